"""Benchmark: N-1 power-flow solves/s on the 9241-bus synthetic grid (1000 N-1
contingencies, Newton-Raphson to 1e-8 p.u.), mixed precision vs plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one batched solve of every case of the workload, from the flat start to
convergence.  ours: prints one JSON line (rank 0) with value = mixed-precision
solves/s (all ranks), plain FP64 beside it, per-kernel roofline of the dominant
kernel, the end-to-end figure through the host C-ABI call, the CPU baseline and
the GPU clocks seen during the timed region.  reference: times the reference's
own CPU implementation of the path (mkl_runpf / mkl_newtonpf with its Eigen SparseLU
option, compiled from the reference's sources into oracle/_ref/librefpf.so) on this
host's cores.

Multi-GPU: one process per GPU (torchrun); each rank solves its own 1000-case
N-1 set of the same grid (weak scaling, no data-path collective); the time is
the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cfg3_9241bus"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cases", type=int, default=0,
                    help="solve only the first N cases per GPU (small runs for profiling; 0 = all)")
    ap.add_argument("--profile-solve", choices=["mixed", "fp64"], default=None,
                    help="profiling driver: warm-up solves (which also autotune), then exactly one solve "
                         "of this precision between cudaProfilerStart/Stop (for ncu --profile-from-start "
                         "off); prints that solve's kernel timing and exits")
    return ap.parse_args()


def profile_solve(args):
    import torch

    import mapol_b200 as m

    buses, branches, cases = m.workload(args.workload)
    if args.cases:
        cases = cases[:args.cases]
    prec = m.MIXED if args.profile_solve == "mixed" else m.FP64
    # the host-read Newton loop, whose timing splits the solve by kernel family
    with m.PowerFlow(buses, branches, use_graph=1) as pf:
        pf.set_cases(cases)
        for _ in range(max(1, args.warmup)):
            pf.solve(m.NR, prec)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        pf.solve(m.NR, prec)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        res = pf.results()
        return {"profile_solve": args.profile_solve, "cases": len(cases), "converged": int(res.converged.sum()),
                "timing": pf.timing(), "stats": pf.stats()}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def factor_traffic_per_case():
    """DRAM bytes per case of one factorisation, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "dram_nr_mixed_9241bus_256cases.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("factor_dram_bytes_per_case:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU baselines
def cpu_port_baseline(buses, branches, cases, budget_s=15.0):
    """The oracle (own sparse LU, all host threads) on a bounded sample of the cases."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    n = min(len(cases), max(threads, 8))
    t = time.perf_counter()
    r = oracle.runpf(buses, branches, cases[:n], alg=0, solver=oracle.SOLVER_GP, threads=threads)
    dt = time.perf_counter() - t
    # grow the sample toward the time budget
    if dt < budget_s / 4 and n < len(cases):
        n2 = min(len(cases), int(n * budget_s / max(dt, 1e-3)))
        t = time.perf_counter()
        r = oracle.runpf(buses, branches, cases[:n2], alg=0, solver=oracle.SOLVER_GP, threads=threads)
        dt = time.perf_counter() - t
        n = n2
    line = {"value": n / dt, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{n} of the {len(cases)} N-1 cases, NR FP64 to 1e-8, oracle sparse LU "
                      f"(Gilbert-Peierls, minimum degree), {threads} threads, {dt:.1f} s",
            "converged": int(r["converged"].sum())}
    return line, r


def other_cpu_baselines(buses, branches, cases, budget_s=10.0):
    """The other CPU rows, each on a bounded sample on all host threads: Newton with
    the reference's Eigen SparseLU reusing its symbolic analysis within a case (the
    reference calls compute(), i.e. analysis and factorisation, every iteration;
    newtonpf.h:341-363), and fast-decoupled XB (fdpf.h:450-596) on the oracle's own LU."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    out = {}
    if oracle.has_eigen():
        # one and two iterations of one case per thread: their difference is a
        # factorisation with the analysis reused, the first run the analysis and one
        sample = cases[:threads]
        t = time.perf_counter()
        oracle.runpf(buses, branches, sample, max_it=1, solver=oracle.SOLVER_EIGEN_REUSE, threads=threads)
        t1 = time.perf_counter() - t
        t = time.perf_counter()
        oracle.runpf(buses, branches, sample, max_it=2, solver=oracle.SOLVER_EIGEN_REUSE, threads=threads)
        t2 = time.perf_counter() - t
        iters = 7.0  # every case of the 9241-bus workload converges in 7 (oracle and engine)
        per_solve = t1 + (iters - 1.0) * max(t2 - t1, 0.0)
        out["newton_eigen_symbolic_reused"] = {
            "value": len(sample) / per_solve, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{len(sample)} cases, one per thread: analysis + first iteration {t1:.1f} s, each further "
                      f"iteration {t2 - t1:.1f} s; a 7-iteration solve = first + 6 further"}
    n = min(len(cases), max(threads, 8))
    t = time.perf_counter()
    r = oracle.runpf(buses, branches, cases[:n], alg=1, threads=threads)
    dt = time.perf_counter() - t
    if dt < budget_s / 4 and n < len(cases):
        n = min(len(cases), int(n * budget_s / max(dt, 1e-3)))
        t = time.perf_counter()
        r = oracle.runpf(buses, branches, cases[:n], alg=1, threads=threads)
        dt = time.perf_counter() - t
    out["fdxb_own_lu"] = {"value": n / dt, "unit": "solves/s", "cores": threads, "kind": "port",
                          "sample": f"{n} cases, fast-decoupled XB to 1e-8 on the oracle's sparse LU "
                                    f"(B' and B'' refactorised every iteration, as fdpf.h:483-561), {dt:.1f} s",
                          "converged": int(r["converged"].sum())}
    return out


def accuracy(res, ref):
    """Per-result accuracy of GPU results against the FP64 oracle on the cases both
    solved: max |dV| (p.u., complex difference), max angle error (degrees), flag and
    iteration-count mismatches (iterations: mixed precision may take one more)."""
    n = len(ref["converged"])
    conv_g = res.status[:n] == 1
    conv_o = ref["converged"]
    both = conv_g & conv_o
    dv = np.abs(res.v[:n][both] - ref["v"][both])
    dang = np.abs(np.angle(res.v[:n][both] * np.conj(ref["v"][both]), deg=True))
    d_it = res.iterations[:n] - ref["iterations"]
    return {"n_compared": int(n), "max_dv": float(dv.max()) if dv.size else None,
            "max_dangle_deg": float(dang.max()) if dang.size else None,
            "flag_mismatches": int((conv_g != conv_o).sum()),
            "iter_equal": int((d_it[both] == 0).sum()), "iter_plus_one": int((d_it[both] == 1).sum()),
            "iter_other": int(((d_it[both] != 0) & (d_it[both] != 1)).sum())}


METRIC = "N-1 PF solves/sec @1e-8 pu, 9241-bus synth: mixed vs plain FP64; HBM GB/s"

# Real grids beside the synthetic headline: the reference's bundled MATPOWER cases
# (tests/golden/matpower_cases.npz, converted by tests/golden/make_matpower_fixtures.py),
# N-1 outages of non-bridge branches.
REAL_WORKLOADS = {"pegase9241": ("case9241pegase", 1000), "pegase2869": ("case2869pegase", 1000),
                  "pegase1354": ("case1354pegase", 1000)}


def real_workload(name, rank=0, outage_seed=7):
    import mapol_b200 as m

    case, n_out = REAL_WORKLOADS[name]
    g = np.load(os.path.join(ROOT, "tests", "golden", "matpower_cases.npz"))
    buses, branches = g[case + "_buses"], g[case + "_branches"]
    n_out = min(n_out, int((~m.find_bridges(branches, len(buses))).sum()))
    return buses, branches, m.n1_cases(branches, len(buses), n_out, outage_seed + rank)


def _ref_worker(conn, fixture, case_ids, solver):
    """One host core running the reference's own Newton-Raphson (oracle/_ref/librefpf.so,
    one grid per process: the reference keeps its state in globals).  Each "step"
    command runs one Newton iteration of its current case (starting the next case of
    its share when the last one finished) and answers (seconds, iterations done,
    solves finished, their total iterations, converged count)."""
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    from oracle import refpf

    g = np.load(fixture)
    outs = g["outages"]
    st = refpf.Stepper(g["buses"], g["branches"], solver)
    k = 0
    conn.send("ready")
    while conn.recv() == "step":
        t = time.perf_counter()
        r = st.step([int(outs[case_ids[k % len(case_ids)]])])
        dt = time.perf_counter() - t
        done = (1, r[1], int(r[0])) if r is not None else (0, 0, 0)
        if r is not None:
            k += 1
        conn.send((dt, 1, *done))
    st.close()
    conn.close()


def reference_arm(args):
    """The reference's own CPU path on this host's cores: mkl_runpf / mkl_newtonpf
    (runpf.h:259-352, newtonpf.h:365-523) with its Eigen_SparseLU solver option
    (newtonpf.h:341-363), compiled unmodified from the reference tree into
    oracle/_ref/librefpf.so (MKL routines through the in-project stand-in of
    oracle/refshim/mkl.h).  One process per host core (the reference's state is
    global); a step is one Newton iteration on every core (a 9241-bus iteration takes
    seconds), each core walking through its share of the 1000 N-1 cases; solves/s =
    Newton iterations per second / iterations per solve, both counted from the
    reference's own solves during the run."""
    import multiprocessing as mp

    from oracle import refpf

    fixture = os.path.join(ROOT, "tests", "golden", f"workload_{args.workload}.npz")
    if not os.path.exists(fixture):
        return {"impl": "reference", "unavailable": f"no committed fixture for workload {args.workload}"}
    if not refpf.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/librefpf.so (the reference's CPU path built from "
                                                    "its sources) is not present"}
    n_cases = len(np.load(fixture)["outages"])
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    conns, procs = [], []
    for w in range(cores):
        a, b = ctx.Pipe()
        p = ctx.Process(target=_ref_worker, args=(b, fixture, list(range(w, n_cases, cores)), refpf.SOLVER_EIGEN))
        p.start()
        conns.append(a)
        procs.append(p)
    for c in conns:
        assert c.recv() == "ready"

    def step():
        t = time.perf_counter()
        for c in conns:
            c.send("step")
        rs = [c.recv() for c in conns]
        return time.perf_counter() - t, rs

    finished, fin_iters, fin_conv = 0, 0, 0
    for _ in range(args.warmup):
        _, rs = step()
        for r in rs:
            finished, fin_iters, fin_conv = finished + r[2], fin_iters + r[3], fin_conv + r[4]
    wall, iters = 0.0, 0
    for _ in range(args.steps):
        dt, rs = step()
        wall += dt
        for r in rs:
            iters += r[1]
            finished, fin_iters, fin_conv = finished + r[2], fin_iters + r[3], fin_conv + r[4]
    extra = 0
    while finished == 0 and extra < 12:  # short runs: step on, untimed, until a case finishes
        _, rs = step()
        extra += 1
        for r in rs:
            finished, fin_iters, fin_conv = finished + r[2], fin_iters + r[3], fin_conv + r[4]
    for c in conns:
        c.send("stop")
    for p in procs:
        p.join(timeout=60)
    if finished == 0:
        return {"impl": "reference", "unavailable": "no reference solve finished within the run"}
    per_solve = fin_iters / finished
    value = iters / per_solve / wall
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, committed fixture)",
        "config": {"workload": f"{args.workload}: {n_cases} N-1 contingencies, NR to 1e-8 p.u.", "alg": "NR",
                   "linear_solver": "Eigen 3.2.8 SparseLU<COLAMD>, compute() every iteration (the reference's "
                                    "Eigen_SparseLU option; its default MKL DSS is unavailable on this box)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} timed steps, each one Newton iteration of the reference's own "
                                   f"mkl_* code on each of {cores} cores (one process per core); {finished} solves "
                                   f"finished during the run ({fin_conv} converged), {per_solve:.2f} iterations per "
                                   f"solve; solves/s = iterations / iterations per solve / time"
                                   + ("" if fin_conv else "; the reference converges none of these cases: it takes "
                                      "voltage angles as atan(y/x) (cuCangle, util/complexUtils.h:21-23) and its "
                                      "Newton iterates pass 90 degrees, so each case stops at MAX_IT_NR = 10; value "
                                      "counts finished cases")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world, local_rank):
    import torch

    import mapol_b200 as m
    from mapol_b200 import _types as T
    from mapol_b200._lib import lib, ptr
    from mapol_b200.grid import cases_to_offsets

    from mapol_b200.shard import max_over_ranks as _mor
    from mapol_b200.shard import rank_cases

    torch.cuda.set_device(local_rank)
    if args.workload in REAL_WORKLOADS:
        buses, branches, cases = real_workload(args.workload, rank)
    else:
        buses, branches, cases = rank_cases(args.workload, rank)
    if args.cases:
        cases = cases[: args.cases]
    n_cases = len(cases)
    t_create = time.perf_counter()
    pf = m.PowerFlow(buses, branches, device=local_rank, use_graph=1)  # per-family kernel times
    t_create = time.perf_counter() - t_create
    pf.set_cases(cases)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        return _mor(x, world, "cuda")

    out = {}
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    for prec, name in ((m.MIXED, "mixed"), (m.FP64, "fp64")):
        for _ in range(args.warmup):
            pf.solve(m.NR, prec, stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fam = {k: 0.0 for k in ("mismatch_ms", "jacobian_ms", "factor_ms", "solve_ms", "update_ms", "other_ms")}
        launches, iters_sum, nfact = 0, 0, 0
        e0.record(stream)
        for _ in range(args.steps):
            pf.solve(m.NR, prec, stream.cuda_stream)
            tm = pf.timing()
            for k in fam:
                fam[k] += tm[k]
            launches += tm["launches"]
            nfact += tm["iterations_max"]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        res = pf.results()
        conv = res.status == T.CASE_CONVERGED
        iters_sum = int(res.iterations[conv].sum())
        out[name] = dict(res=res, ms=ms, fam={k: v / args.steps for k, v in fam.items()}, launches=launches,
                         n_conv=int(conv.sum()), iters=np.bincount(res.iterations, minlength=11).tolist(),
                         max_mis=float(res.max_mis[conv].max()) if conv.any() else None,
                         iters_sum=iters_sum, nfact=nfact / args.steps)
    st = pf.stats()  # after the solves: device_bytes includes the factor buffers

    # The headline solves: the same kernels with the whole Newton loop as one CUDA graph
    # (use_graph = 2: a device-side while node instead of one host flag read and four
    # graph launches per iteration).  The host-loop solves above give the per-family
    # kernel times of the roofline (the device loop reports them as one figure) and
    # must equal these bit for bit.
    pf2 = m.PowerFlow(buses, branches, device=local_rank, use_graph=2)
    pf2.set_cases(cases)
    loop = {}
    for prec, name in ((m.MIXED, "mixed"), (m.FP64, "fp64")):
        for _ in range(args.warmup):
            pf2.solve(m.NR, prec, stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        e0.record(stream)
        for _ in range(args.steps):
            pf2.solve(m.NR, prec, stream.cuda_stream)
            launches += pf2.timing()["launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        r2 = pf2.results()
        ref = out[name]["res"]
        loop[name] = dict(ms=max_over_ranks(e0.elapsed_time(e1)), launches=launches,
                          identical=bool(np.array_equal(r2.v, ref.v) and np.array_equal(r2.iterations, ref.iterations)
                                         and np.array_equal(r2.status, ref.status)))
    clocks = sampler.stop() if sampler else None

    # end to end through the host C-ABI call: case definitions in from pinned host
    # memory, voltages / flags / iterations / mismatch back into pinned host memory
    e2e = None
    if not args.no_e2e:
        offs, flat = cases_to_offsets(cases)
        nb = len(buses)
        offs_t = torch.from_numpy(offs).pin_memory()
        flat_t = torch.from_numpy(flat).pin_memory()
        v_t = torch.empty((n_cases, nb, 2), dtype=torch.float64).pin_memory()
        it_t = torch.empty(n_cases, dtype=torch.int32).pin_memory()
        st_t = torch.empty(n_cases, dtype=torch.uint8).pin_memory()
        mm_t = torch.empty(n_cases, dtype=torch.float64).pin_memory()
        L = lib()

        def call():
            rc = L.mpf_runpf_host(pf2._h, m.NR, m.MIXED, n_cases, offs_t.data_ptr(), flat_t.data_ptr(), None,
                                  v_t.data_ptr(), it_t.data_ptr(), st_t.data_ptr(), mm_t.data_ptr())
            if rc != 0:
                raise RuntimeError(L.mpf_last_error(pf2._h).decode())

        for _ in range(args.warmup):
            call()
        torch.cuda.synchronize()
        barrier()
        t = time.perf_counter()
        for _ in range(args.steps):
            call()
        dt = max_over_ranks(time.perf_counter() - t)
        barrier()
        h2d = offs.nbytes + flat.nbytes
        d2h = v_t.numel() * 8 + n_cases * (4 + 1 + 8)
        e2e = {"value": n_cases * world * args.steps / dt, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "precision": "mixed",
               "n_converged": int((st_t.numpy() == T.CASE_CONVERGED).sum())}
    pf.close()
    pf2.close()

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    mixed, fp64 = out["mixed"], out["fp64"]
    value = n_cases * world * args.steps / (loop["mixed"]["ms"] / 1e3)
    value_fp64 = n_cases * world * args.steps / (loop["fp64"]["ms"] / 1e3)
    host_loop = {"value": n_cases * world * args.steps / (mixed["ms"] / 1e3),
                 "fp64": n_cases * world * args.steps / (fp64["ms"] / 1e3),
                 "ms_per_step": mixed["ms"] / args.steps,
                 "note": "use_graph = 1 (one host flag read per Newton iteration): the run whose "
                         "per-family kernel times feed the roofline",
                 "results_identical_to_headline": loop["mixed"]["identical"] and loop["fp64"]["identical"]}

    # roofline of the dominant kernel family of the headline (mixed) solve.
    # Algorithmic bytes per case per Newton iteration (w = bytes per LU value, the
    # precision of the Newton system, its solution x and the Jacobian):
    #   factor:   2 w nnz(L+U) (arrowhead and contribution blocks in, panels out)
    #   solve:    w nnz(U panels) + 2 w n (the backward substitution reads the pivot rows
    #             of each supernode and x, and writes x; the forward one is fused into
    #             the factorisation)
    #   mismatch: 16 nb (V) + 8 n (F) + w nnz(J) (the Jacobian fill is fused into the
    #             mismatch pass, so its own family time is 0)
    #   update:   w n (x) + 32 nb (V read and written)
    def alg_bytes(family, w_lu):
        nb, n, nnz_lu, nnz_j = st["n_bus"], st["n_jac"], st["nnz_lu"], st["nnz_jac"]
        return {"factor_ms": 2 * w_lu * nnz_lu, "solve_ms": w_lu * st["nnz_lu_upper"] + 2 * w_lu * n,
                "mismatch_ms": 16 * nb + 8 * n + w_lu * nnz_j, "jacobian_ms": 0,
                "update_ms": w_lu * n + 32 * nb}.get(family)

    fams = {k: v for k, v in mixed["fam"].items() if k != "other_ms"}
    dom = max(fams, key=fams.get)
    tpc = factor_traffic_per_case() if args.workload == WORKLOAD and dom == "factor_ms" else None
    traffic = round(tpc * n_cases) if tpc else None
    # units processed per step by that family: Newton iterations summed over cases
    units = mixed["iters_sum"]
    achieved = alg_bytes(dom, 4) * units / (fams[dom] / 1e3) / 1e9
    per_family = {}
    for k, v in fams.items():
        b = alg_bytes(k, 4)
        per_family[k.replace("_ms", "")] = {"ms_per_step": round(v, 4),
                                            "GB/s": round(b * units / (v / 1e3) / 1e9, 1) if v > 0 else None}

    line = {
        "metric": METRIC if args.workload == WORKLOAD else METRIC.replace(
            "9241-bus synth", REAL_WORKLOADS[args.workload][0] + " (real grid)" if args.workload in REAL_WORKLOADS
            else args.workload),
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": loop["mixed"]["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 mismatch/update/convergence test, f32 LU factorisation and solves",
        "data": ("synthetic (seeded generator: 9241 buses, 16049 branches, 1445 PV, 15% tapped)"
                 if args.workload == WORKLOAD else
                 f"real grid: the reference's bundled {REAL_WORKLOADS[args.workload][0]}.m"
                 if args.workload in REAL_WORKLOADS else f"synthetic ({args.workload})"),
        "config": {"workload": f"{args.workload}: {n_cases} N-1 contingencies per GPU, NR to 1e-8 p.u.",
                   "n_cases_per_gpu": n_cases, "alg": "NR", "parallelism": f"replicas x{world} (cases sharded)",
                   "l2": "inputs larger than L2 (factor working set %.1f GB per GPU)" % (st["device_bytes"] / 1e9)},
        "plain_fp64": {"value": value_fp64, "ms_per_step": loop["fp64"]["ms"] / args.steps,
                       "converged": fp64["n_conv"], "iterations_hist": fp64["iters"],
                       "max_mismatch": fp64["max_mis"]},
        "mixed_over_plain": value / value_fp64,
        "mixed": {"converged": mixed["n_conv"], "iterations_hist": mixed["iters"], "max_mismatch": mixed["max_mis"]},
        "roofline": {"bound": "hbm", "kernel": dom.replace("_ms", ""), "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "traffic_unit": "DRAM bytes per factorisation of all cases (all its level launches)",
                     "alg_bytes": alg_bytes("factor_ms", 4) * n_cases,
                     "traffic_source": ("ncu dram__bytes_read+write.sum, 256 cases, per case x cases "
                                        "(profiles/dram_nr_mixed_9241bus_256cases.md)") if traffic is not None
                                       else None,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "per_family": per_family},
        "gpu_launches": int(loop["mixed"]["launches"]),
        "clocks": clocks,
        "host_loop": host_loop,
    }
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baselines"] = other_cpu_baselines(buses, branches, cases)
    line["setup"] = {"mpf_create_ms": round(t_create * 1e3, 1),
                     "note": "one-time host symbolic analysis (ordering, supernodes, relative maps) and "
                             "upload of the shared arrays; not inside the timed solves"}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], ref = cpu_port_baseline(buses, branches, cases)
        line["accuracy"] = {"vs": "FP64 CPU oracle on the cpu_baseline sample",
                            "mixed": accuracy(mixed["res"], ref), "fp64": accuracy(fp64["res"], ref)}
    return line


def run_multigrid(args, rank, world, local_rank):
    """Grids of uneven size in one batch (MultiGrid): every stage of the three grids'
    cases runs in shared launches.  Beside it: the same cases on one handle per grid,
    solved back to back on the same stream."""
    import torch

    import mapol_b200 as m
    from mapol_b200 import _types as T
    from mapol_b200.grid import WORKLOAD_SETS, workload_set
    from mapol_b200.shard import max_over_ranks as _mor

    torch.cuda.set_device(local_rank)
    grids, cases = workload_set(args.workload)
    n_cases = sum(len(c) for c in cases)
    stream = torch.cuda.current_stream()

    def timed(solve_all):
        for _ in range(args.warmup):
            solve_all()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            solve_all()
        e1.record(stream)
        torch.cuda.synchronize()
        return _mor(e0.elapsed_time(e1), world, "cuda")

    out = {}
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    # both arms run the whole Newton loop as one CUDA graph (use_graph = 2)
    with m.MultiGrid(grids, device=local_rank, use_graph=2) as mg:
        mg.set_cases(cases)
        for prec, name in ((m.MIXED, "mixed"), (m.FP64, "fp64")):
            ms = timed(lambda: mg.pf.solve(m.NR, prec, stream.cuda_stream))
            res = mg.results()
            out[name] = dict(ms=ms, launches=mg.timing()["launches"],
                             n_conv=int(sum((r.status == T.CASE_CONVERGED).sum() for r in res)))
    pfs = []
    for (b, br), cs in zip(grids, cases):
        pf = m.PowerFlow(b, br, device=local_rank, use_graph=2)
        pf.set_cases(cs)
        pfs.append(pf)

    def separate():
        for pf in pfs:
            pf.solve(m.NR, m.MIXED, stream.cuda_stream)

    sep_ms = timed(separate)
    sep_launches = sum(pf.timing()["launches"] for pf in pfs)
    for pf in pfs:
        pf.close()
    clocks = sampler.stop() if sampler else None
    if rank != 0:
        return None
    value = n_cases * world * args.steps / (out["mixed"]["ms"] / 1e3)
    return {
        "metric": "PF solves/sec @1e-8 pu, grids of uneven size in one batch (%s-bus synth): mixed vs plain FP64"
                  % "/".join(str(len(g[0])) for g in grids),
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["mixed"]["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 mismatch/update/convergence test, f32 LU factorisation and solves",
        "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "grids": WORKLOAD_SETS[args.workload],
                   "cases_per_grid": [len(c) for c in cases], "alg": "NR",
                   "newton_loop": "one CUDA graph per solve (use_graph = 2)"},
        "plain_fp64": {"value": n_cases * world * args.steps / (out["fp64"]["ms"] / 1e3),
                       "ms_per_step": out["fp64"]["ms"] / args.steps},
        "converged": {"mixed": out["mixed"]["n_conv"], "fp64": out["fp64"]["n_conv"], "of": n_cases},
        "launches_per_solve": {"one_batch": out["mixed"]["launches"], "one_handle_per_grid": sep_launches},
        "one_handle_per_grid": {"value": n_cases * world * args.steps / (sep_ms / 1e3),
                                "ms_per_step": sep_ms / args.steps, "precision": "mixed"},
        "clocks": clocks,
    }


def run_extras(args):
    """Throughput of the paths beside the headline, each through the public API:
    particle-swarm fitness evaluations (the reference's hybrid_runpf workflow on the
    IEEE 300-bus case with its AVR / OLTC / ShC structures), N-1 solves with generator
    reactive limits enforced, and adjoint gradients of the overload loss (1354-bus grid,
    4096 load scenarios).  Each: warm-up, then timed runs on the device clock."""
    import torch

    import mapol_b200 as m
    from mapol_b200 import pso
    from oracle import oracle

    g = np.load(os.path.join(ROOT, "tests", "golden", "matpower_cases.npz"))
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) / reps

    out = {"metric": "extras: PSO fitness evaluations/s, Q-limited N-1 solves/s, adjoint gradients/s",
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup}
    # particle swarm: 1024 particles, fitness = active loss or DBL_MAX (runpf.h:748-791)
    buses, branches = g["case300_buses"], g["case300_branches"]
    est, bie, rie = pso.estruturas(buses, branches)
    rng = np.random.default_rng(0)
    lo = np.array([e.min for e in est])
    hi = np.array([e.max for e in est])
    X = lo + (hi - lo) * rng.random((1024, len(est)))
    enxame = [pso.Particula(x) for x in X]
    eng = pso.hybrid_init(buses, branches, len(enxame), 1, est, m.NR, bie, rie, precision=m.MIXED)
    dt = timed(lambda: pso.hybrid_runpf(eng, est, enxame), args.steps)
    fit = np.array([p.fitness for p in enxame])
    pso.hybrid_free(eng)
    controls, cols = pso.bind(est, bie, rie, branches)
    n_cpu = min(64, len(enxame))
    t = time.perf_counter()
    for c in range(n_cpu):
        b, br = buses.copy(), branches.copy()
        for (kind, idx), v in zip(controls, X[c, cols]):
            if kind == m.CTRL_AVR:
                b["vm"][idx] = v
            elif kind == m.CTRL_SHC:
                b["bsh"][idx] = v
            else:
                br["tap"][idx] = v
        oracle.runpf(b, br, [[]], alg=0, threads=1)
    dt_cpu = (time.perf_counter() - t) / n_cpu
    out["pso"] = {"grid": "IEEE 300-bus (reference's case300.m)", "particles": len(enxame),
                  "structures": len(est), "value": len(enxame) / dt, "unit": "fitness evaluations/s",
                  "ms_per_swarm": dt * 1e3, "feasible": int((fit < pso.DBL_MAX).sum()),
                  "cpu_oracle_one_thread": {"value": 1.0 / dt_cpu, "unit": "fitness evaluations/s",
                                            "sample": f"{n_cpu} particles, NR FP64, one host thread"}}
    # generator reactive limits on the IEEE 300-bus case, N-1
    cases = m.n1_cases(branches, len(buses), 256, 5, with_base=True)
    res = {}
    for lim in (False, True):
        with m.PowerFlow(buses, branches) as pf:
            if lim:
                pf.set_q_limits(g["case300_qmin"], g["case300_qmax"])
            pf.set_cases(cases)
            dt = timed(lambda: pf.solve(m.NR, m.MIXED, stream.cuda_stream), args.steps)
            r = pf.results()
            res[lim] = (len(cases) / dt, int(r.converged.sum()),
                        int(((pf.bus_types() == 1) & (buses["type"] == 2)[None]).sum()) if lim else 0)
    out["q_limits"] = {"grid": "IEEE 300-bus, generator Q limits of case300.m", "cases": len(cases),
                       "value": res[True][0], "unit": "solves/s", "without_limits": res[False][0],
                       "converged": res[True][1], "switched_buses_total": res[True][2]}
    # adjoint on the 1354-bus grid, 4096 load scenarios
    b4, br4, _ = m.workload("cfg4_1354bus")
    sb = m.load_scenarios(b4, 4096, 0.05, 11)
    with m.PowerFlow(b4, br4) as pf:
        pf.set_cases([[]])
        pf.solve(m.NR, m.FP64)
        rating = 1.2 * np.abs(pf.branch_flows(flows=True)["sf"][0])
        pf.set_ratings(rating)
        pf.set_cases([[]] * 4096, sbus=sb)
        pf.solve(m.NR, m.MIXED, stream.cuda_stream)
        dt_s = timed(lambda: pf.solve(m.NR, m.MIXED, stream.cuda_stream), args.steps)
        from mapol_b200._lib import lib

        dev = torch.device("cuda")
        gp = torch.empty((4096, len(b4)), dtype=torch.float64, device=dev)
        gq = torch.empty_like(gp)
        gg = torch.empty((4096, len(br4)), dtype=torch.float64, device=dev)
        gb = torch.empty_like(gg)

        def adj():
            rc = lib().mpf_adjoint(pf._h, m.MIXED, gp.data_ptr(), gq.data_ptr(), gg.data_ptr(), gb.data_ptr(),
                                   None)
            if rc != 0:
                raise RuntimeError(lib().mpf_last_error(pf._h).decode())

        dt_a = timed(adj, args.steps)
    out["adjoint"] = {"grid": "1354-bus synthetic, 4096 load scenarios", "solve_ms": dt_s * 1e3,
                      "adjoint_ms": dt_a * 1e3, "value": 4096 / dt_a, "unit": "gradients/s (per scenario)",
                      "note": "mpf_adjoint into device buffers: refactorisation at the solution (FP32), U^T "
                              "and L^T substitutions, gradients w.r.t. P, Q, g, b"}
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return 0
    if args.profile_solve:
        print(json.dumps(profile_solve(args)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from mapol_b200.grid import WORKLOAD_SETS

    if args.workload == "extras":
        if rank == 0:
            print(json.dumps(run_extras(args)), flush=True)
        return 0
    if args.workload in WORKLOAD_SETS:
        line = run_multigrid(args, rank, world, local_rank)
    else:
        line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
