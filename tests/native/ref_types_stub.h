/* ref_types_stub.h: minimal stand-ins for the reference's host types that the C++
 * shim in INTEGRATION.md reads (field names as in src/powersystem/Bus.h:18-31,
 * Branch.h:15-27, Topology.h and src/pso/Particula.h:26-60), so that the shim can be
 * compiled here against include/mpf.h without the reference tree.  Only the members
 * the shim touches are declared. */
#ifndef REF_TYPES_STUB_H_
#define REF_TYPES_STUB_H_

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstdio>
#include <vector>

struct Bus {
  enum Type { NONE, PQ, PV, SLACK, ISOLATED };
  Type type;
  double V, O, P, Q, Gsh, Bsh;
  int indicePVPQ, indiceEstrutura;
};

struct Branch {
  unsigned int from, to;
  bool inservice;
  double R, X, B, tap, shift;
  int indiceEstrutura;
};

struct Topology {
  std::vector<Bus> buses;
  std::vector<Branch> branches;
};

namespace pso {
class Particula {
 public:
  struct Estrutura {
    enum Tipo { NULO, AVR, OLTC, SHC };
    Tipo tipo;
    double min, max, defaultValue;
  };
  std::vector<double> X;
  double operator[](size_t i) const { return X[i]; }
  void mudarFitness(double f) { fitness_ = f; }

 private:
  double fitness_ = 0;
};
}  // namespace pso

#endif
