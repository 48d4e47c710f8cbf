/* c_abi_smoke.c: a plain C99 caller of libmpf (no C++, no Python), the way a
 * reference-side binding would use the C-ABI of include/mpf.h.  It generates the
 * 30-bus synthetic grid of the smallest workload with the library's seeded
 * generator, defines the base case plus 10 N-1 outages, solves Newton-Raphson in
 * plain FP64 and in mixed precision, and writes the grid and both results to the
 * binary file named by argv[1] for the test that runs it to check against the CPU
 * oracle.  Exit status 0 on success; any failing call prints mpf_last_error. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpf.h"

#define NB 30
#define NBR 41
#define NOUT 10
#define NCASES (NOUT + 1)

static int check(int rc, const char* what, const mpf_handle* h) {
  if (rc != MPF_OK) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, mpf_status_string(rc), h ? mpf_last_error(h) : "");
    return 1;
  }
  return 0;
}

int main(int argc, char** argv) {
  mpf_synth_params p;
  mpf_bus buses[NB];
  mpf_branch branches[NBR];
  int32_t out[NOUT], offs[NCASES + 1], flat[NOUT];
  mpf_options opt;
  mpf_handle* h = NULL;
  static double v[NCASES * NB * 2];
  double mis[NCASES];
  int32_t it[NCASES];
  uint8_t st[NCASES];
  FILE* f;
  int prec, c;

  if (argc != 2) {
    fprintf(stderr, "usage: %s OUTPUT\n", argv[0]);
    return 2;
  }
  if (mpf_abi_version() != MPF_ABI_VERSION) {
    fprintf(stderr, "ABI mismatch: library %d, header %d\n", mpf_abi_version(), MPF_ABI_VERSION);
    return 1;
  }
  mpf_synth_default(&p);
  p.n_bus = NB;
  p.n_branch = NBR;
  p.n_pv = 5;
  p.tap_fraction = 0.0;
  p.seed = 1;
  if (check(mpf_synth_grid(&p, buses, branches), "mpf_synth_grid", NULL)) return 1;
  if (check(mpf_select_outages(branches, NBR, NB, NOUT, 7, out), "mpf_select_outages", NULL)) return 1;
  /* case 0: the base case; case c > 0: branch out[c - 1] outaged */
  offs[0] = 0;
  offs[1] = 0;
  for (c = 0; c < NOUT; ++c) {
    flat[c] = out[c];
    offs[c + 2] = c + 1;
  }
  mpf_default_options(&opt);
  if (check(mpf_create(buses, NB, branches, NBR, &opt, &h), "mpf_create", h)) return 1;
  if (check(mpf_set_cases(h, NCASES, offs, flat, NULL), "mpf_set_cases", h)) return 1;

  f = fopen(argv[1], "wb");
  if (!f) {
    perror(argv[1]);
    return 1;
  }
  fwrite(buses, sizeof(buses), 1, f);
  fwrite(branches, sizeof(branches), 1, f);
  fwrite(offs, sizeof(offs), 1, f);
  fwrite(flat, sizeof(flat), 1, f);
  for (prec = MPF_FP64; prec <= MPF_MIXED; ++prec) {
    if (check(mpf_solve(h, MPF_NR, prec, NULL), "mpf_solve", h)) return 1;
    if (check(mpf_get_results(h, v, it, st, mis), "mpf_get_results", h)) return 1;
    fwrite(st, sizeof(st), 1, f);
    fwrite(it, sizeof(it), 1, f);
    fwrite(mis, sizeof(mis), 1, f);
    fwrite(v, sizeof(v), 1, f);
  }
  fclose(f);
  if (check(mpf_destroy(h), "mpf_destroy", NULL)) return 1;
  printf("c_abi_smoke ok: %d cases\n", NCASES);
  return 0;
}
