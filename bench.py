"""Benchmark: time to reach 1e-8 relative residual per right-hand side on the
128^3 27-point anisotropic AMG-PBiCGStab problem with 16 RHS (one B200).

A step is one complete solve of the 16 right-hand sides from a zero initial
guess.  Forms:
  plain  - FP64 PBiCGStab + FP64 AMG V-cycle, hybrid-SGS smoothing in the
           reference's single-process row order (parity form);
  mixed  - FP64 iterative refinement around an FP32 PBiCGStab (FP64 inner
           products and recurrences) with an FP32 AMG V-cycle whose SGS runs
           the reference's hybrid block semantics with GPU-sized blocks.
  batch  - 64 independent 7-point lognormal-coefficient systems (sides 16..96,
           nv in {1,2,4,8}) solved together in one CUDA-graph launch (FP64
           Krylov, FP32 AMG, autotuned SpMV per group); reported beside;
  learned - held-out 64^3 bump-coefficient systems (nv = 8) from a zero guess
           and from the trained network's guess; reported beside.
The headline `value` is the faster of plain/mixed's device time per RHS on the
128^3 problem; `e2e` repeats it through the XAMG C API with host buffers
(pinned), copies included.  `gpu_launches` is the library's own count of the
kernels it launched in the timed steps of that form.  `true_rel_residual`
checks every form's solution in FP64 on the host (max over columns of
||b - A x|| / ||b||).  The SpMV kernel is tuned first (CSR variants and the
shifted-row run kernel, `--spmv` fixes it); `roofline` reports the FP64
NV=16 product of the tuned kernel on the same operator.

--impl reference times the CPU restatement of the reference's algorithm (the
reference itself cannot be built here: it needs MPI, hypre, argsparser and
yaml-cpp) on the host cores on a bounded sample of the same workload.
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
sys.path.insert(0, os.path.join(ROOT, "xamg-test_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
os.environ.setdefault("XAMG_QUIET", "1")

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
N_GRID, NV, SEED = 128, 16, 2024


def plain_spec():
    return {
        "solver": {"method": "PBiCGStab", "max_iters": 200, "abs_tolerance": 0.0, "rel_tolerance": 1e-8,
                   "convergence_details": "check-L2,noprint"},
        "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 10, "mg_interpolation_type": 6,
                           "mg_strength_threshold": 0.25, "mg_max_levels": 6, "mg_agg_num_levels": 0},
        "pre_smoother": {"method": "HSGS", "max_iters": 1},
        "post_smoother": {"method": "HSGS", "max_iters": 1},
        "coarse_grid_solver": {"method": "Direct"},
    }


def gpu_sms():
    try:
        import torch
        return torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:
        return 148


def mixed_spec(blocks=None, inner_rel=1e-4):
    """Precision form.  Hybrid SGS on two blocks per SM on every level (two
    resident CTAs per SM interleave their latency-bound block sweeps)."""
    blocks = blocks or 2 * gpu_sms()
    s = plain_spec()
    s["meta_solver"] = {"method": "IterativeRefinement", "max_iters": 20, "abs_tolerance": 0.0,
                        "rel_tolerance": 1e-8, "subsolver_reduced_precision": True,
                        "inner_rel_tolerance": inner_rel, "convergence_details": "check-L2,noprint"}
    s["pre_smoother"]["hybrid_blocks"] = blocks
    s["post_smoother"]["hybrid_blocks"] = blocks
    return s


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, idx):
        self.idx = idx
        self.rows = []
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peak_hbm():
    try:
        return json.load(open(PEAKS))["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def build_problem():
    import xamg
    csr = xamg.CsrMatrix.aniso27(N_GRID, 1.0, 1.0, 1e-3)
    rng = np.random.default_rng(SEED)
    B = rng.uniform(-1.0, 1.0, (csr.nrows, NV))
    return csr, B


# SpMV kernels timed for the roofline: CSR variants of xamg_spmv_set_variant,
# and RUN8 = the shifted-row run kernel (chunks of 8 rows)
RUN8 = 108


def spmv_time(csr, prec=0, variant=-1, iters=20, info=None):
    """Live CUDA-event timing of the NV=16 SpMV on the benchmark matrix,
    launched on a torch stream through the C ABI; returns ms per launch.  For
    the run kernel `info` (a dict) receives the plan's sizes."""
    import ctypes as C
    import torch
    import xamg
    rp, ci, v = csr.arrays()
    n = csr.nrows
    dt = torch.float64 if prec == 0 else torch.float32
    x = torch.rand(n, NV, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    st = torch.cuda.Stream()
    P = lambda t: C.c_void_p(t.data_ptr())
    L = xamg.lib()
    plan = None
    if variant == RUN8:
        plan = L.xamg_spmv_runs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), xamg._ptr(np.ascontiguousarray(v)),
                                            8, int(prec == 1))
        assert plan, L.XAMG_b200_last_error()
        if info is not None:
            a = np.zeros(4, np.int64)
            cov = np.zeros(1)
            xamg.check(L.xamg_spmv_runs_plan_info(plan, xamg._ptr(a[0:]), xamg._ptr(cov), xamg._ptr(a[1:]),
                                                  xamg._ptr(a[2:])))
            info.update(nchunks=int(a[0]), coverage=float(cov[0]), segments=int(a[1]), value_slots=int(a[2]))
        launch = lambda: L.xamg_spmv_runs(plan, prec, NV, P(x), P(y), 0, None, C.c_void_p(st.cuda_stream))
    else:
        d = [torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).to(dt).cuda()]
        launch = lambda: L.xamg_csr_spmv(prec, NV, n, P(d[0]), P(d[1]), P(d[2]), P(x), P(y), 0, None,
                                         C.c_void_p(st.cuda_stream))
    torch.cuda.synchronize()
    old = L.xamg_spmv_set_variant(variant if plan is None else -1)
    try:
        with torch.cuda.stream(st):
            for _ in range(3):
                xamg.check(launch())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(iters):
                launch()
            e1.record(st)
        st.synchronize()
    finally:
        L.xamg_spmv_set_variant(old)
        if plan:
            L.xamg_spmv_runs_plan_destroy(plan)
    return e0.elapsed_time(e1) / iters


def tune_spmv(csr, prec=0):
    """Autotune the SpMV kernel on this matrix (results are identical for
    every kernel; only the data layout and launch shape differ)."""
    res = {}
    for var in (0, 3, 5, 6, RUN8):
        res[var] = spmv_time(csr, prec, var, iters=10)
    best = min(res, key=res.get)
    return best, res


def apply_spmv_choice(var):
    """Make the library use the tuned kernel: the run kernel (through the run
    plans built at matrix construction) or a CSR variant everywhere."""
    import xamg
    L = xamg.lib()
    if var == RUN8:
        L.xamg_spmv_set_run_rows(8)
        L.xamg_spmv_set_variant(-1)
    else:
        L.xamg_spmv_set_run_rows(0)
        L.xamg_spmv_set_variant(var)


def spmv_roofline(csr, variant):
    info = {}
    ms = spmv_time(csr, 0, variant, iters=20, info=info)
    n, nnz = csr.nrows, csr.nnz
    xy = 2 * n * NV * 8
    if variant == RUN8:
        # run format: each value once, each chunk's segments once (4 B), the
        # chunk descriptors (16 B) and tile offsets (16 B per four chunks), x and y
        byts = nnz * 8 + info["segments"] * 4 + info["nchunks"] * 20 + xy
        kern = "k_spmv_runs<double,16,0>"
    else:
        byts = nnz * (8 + 4) + (n + 1) * 4 + xy
        kern = {0: "k_spmv<double,16,0,4>", 1: "k_spmv<double,16,0,8>", 2: "k_spmv<double,16,0,16>",
                3: "k_spmv_tile<double,16,0,4,0>", 4: "k_spmv_tile<double,16,0,8,0>",
                5: "k_spmv_tile<double,16,0,4,1>", 6: "k_spmv_tile<double,16,0,8,1>"}.get(
                    variant, "k_spmv_stream<double,16,0>")
    peak, src = peak_hbm()
    ach = byts / (ms * 1e-3) / 1e9
    # DRAM traffic per launch: the ncu capture of the same kernel on the 96^3
    # operator measured TRAFFIC_RATIO x its algorithmic bytes; traffic scales
    # with the operator, so the 128^3 figure is that ratio times the
    # algorithmic bytes
    ratio = TRAFFIC_RATIO.get(variant)
    traffic = round(ratio * byts) if ratio else None
    out = {"bound": "hbm", "kernel": kern, "variant": variant, "achieved": round(ach, 1), "peak": peak,
           "peak_source": src, "unit": "GB/s", "frac": round(ach / peak, 4),
           "traffic": traffic, "traffic_source": "ncu capture at 96^3 scaled to 128^3" if traffic else None,
           "algorithmic_bytes": byts, "launch_ms": round(ms, 4)}
    if info:
        out["run_plan"] = info
    return out


# DRAM bytes / algorithmic bytes of one launch in the ncu captures on the 96^3
# operator (profiles/k_spmv_tile_fp64_nv16_27pt_96cube.md: 483.3 of 510.8 MB;
# profiles/k_spmv_runs_fp64_nv16_27pt_96cube.md: 433.9 of 421.8 MB)
TRAFFIC_RATIO = {5: 0.9457, 6: 0.9457, RUN8: 1.0287}


def run_form(csr, B, spec, warmup, steps):
    import xamg
    xamg.set_nv(NV)
    A = xamg.Matrix(csr)
    x = xamg.Vector(csr.nrows, NV)
    b = xamg.Vector(csr.nrows, NV)
    b.upload(B)
    t0 = time.time()
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    setup_s = time.time() - t0
    for _ in range(warmup):
        x.set(0.0)
        s.solve()
    times = []
    k0 = xamg.kernel_launches()
    for _ in range(steps):
        x.set(0.0)
        s.solve()
        times.append(s.last_ms())
    launches = xamg.kernel_launches() - k0
    X = x.download()
    it = s.iters()
    return {"ms": float(np.mean(times)), "ms_all": [round(t, 3) for t in times], "iters": it[0],
            "sub_iters": it[1], "converged": all(s.converged()), "setup_s": round(setup_s, 1),
            "levels": s.info(), "launches": launches}, X, (s, A, x, b)


def e2e_form(csr, B, spec, warmup, steps):
    """Same solve through the C API with pinned host buffers, copies timed."""
    import torch
    import xamg
    xamg.set_nv(NV)
    A = xamg.Matrix(csr)
    x = xamg.Vector(csr.nrows, NV)
    b = xamg.Vector(csr.nrows, NV)
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    hb = torch.from_numpy(B).pin_memory()
    hx = torch.empty((csr.nrows, NV), dtype=torch.float64).pin_memory()
    L = xamg.lib()
    import ctypes as C

    def step():
        xamg.check(L.XAMG_vector_upload_d(C.c_void_p(hb.data_ptr()), csr.nrows, 0, NV, b.h))
        x.set(0.0)
        s.solve()
        xamg.check(L.XAMG_vector_download_d(C.c_void_p(hx.data_ptr()), csr.nrows, 0, NV, x.h))

    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    return (time.perf_counter() - t0) / steps * 1e3


def batch_form(rank, world, warmup, steps):
    """Batching form: 64 independent 7-point lognormal-coefficient systems
    (sides log-uniform in [16, 96], nv in {1, 2, 4, 8}) solved together, one
    CUDA-graph launch per solve; whole systems are sharded over the ranks."""
    import scipy.sparse as sp
    import xamg
    import families
    mem = [families.batch_member(sd) for sd in range(1, 65)]
    w = [A.nnz * nv for A, nv, _ in mem]
    mine = families.shard(w, world)[rank]
    t0 = time.time()
    batch = xamg.Batch([(mem[i][0], mem[i][1]) for i in mine], xamg.Params(families.batch_spec(blocks=gpu_sms())))
    setup_s = time.time() - t0

    def load():
        for q, i in enumerate(mine):
            batch.upload(q, mem[i][2])

    for _ in range(max(warmup, 1)):
        load()
        batch.solve()
    ms, kern = [], 0
    for _ in range(steps):
        load()
        batch.solve()
        ms.append(batch.last_ms())
        kern += batch.last_kernels()
    # end to end: host right-hand sides in, host solutions out
    t0 = time.perf_counter()
    load()
    batch.solve()
    Xs = [batch.download(q) for q in range(len(mine))]
    e2e_ms = (time.perf_counter() - t0) * 1e3
    its, res = [], []
    for q, i in enumerate(mine):
        A, nv, B = mem[i]
        it, _ = batch.stats(q)
        its.append(it)
        rp, ci, v = A.arrays()
        M = sp.csr_matrix((v, ci, rp), shape=(A.nrows, A.nrows))
        res.append(float(np.max(np.linalg.norm(B - M @ Xs[q], axis=0) / np.linalg.norm(B, axis=0))))
    its = np.concatenate(its)
    rhs = sum(mem[i][1] for i in mine)
    return {"ms": float(np.mean(ms)), "ms_all": [round(t, 2) for t in ms], "systems": len(mine), "rhs": int(rhs),
            "rows": int(sum(mem[i][0].nrows for i in mine)), "iters_min": int(its.min()), "iters_max": int(its.max()),
            "converged": bool(np.all(its >= 0)), "max_true_rel_residual": max(res), "setup_s": round(setup_s, 1),
            "groups": batch.groups(), "e2e_ms": round(e2e_ms, 2), "launches": int(kern),
            "h2d_bytes": int(sum(mem[i][2].nbytes for i in mine)), "d2h_bytes": int(sum(x.nbytes for x in Xs))}


LEARNED_WEIGHTS = os.path.join(ROOT, "xamg-test_b200", "weights", "learned_64.npz")


def learned_form(nsys=16):
    """Learned form: held-out 64^3 bump-coefficient systems (nv = 8) solved
    from a zero guess and from the trained network's guess (2 symmetric
    Gauss-Seidel sweeps on it first); time to 1e-8 relative to ||b|| with the
    inference and the sweeps included."""
    if not os.path.exists(LEARNED_WEIGHTS):
        return {"unavailable": "no trained weights at xamg-test_b200/weights/learned_64.npz"}
    import learned
    net = learned.Net(seed=1)
    net.load(LEARNED_WEIGHTS)
    ev = learned.evaluate(net, list(range(200001, 200001 + nsys)), 64, 8)
    out = {"systems": nsys, "rhs": nsys * 8, "n": 64}
    for k in ("its_zero", "its_x0", "ms_zero", "ms_x0", "ms_infer", "ms_smooth", "guess_rel_res", "guess_rel_err",
              "rel_diff"):
        out["mean_" + k] = float("%.5g" % np.mean([e[k] for e in ev]))
    out["ms_per_rhs_zero"] = round(out["mean_ms_zero"] / 8, 4)
    out["ms_per_rhs_x0"] = round(out["mean_ms_x0"] / 8, 4)
    out["converged"] = all(e["converged"] for e in ev)
    return out


def cpu_sample(csr, B, s_plain):
    """One FP64 PBiCGStab iteration of the oracle (the reference's
    single-process order: Gauss-Seidel sequential, products, inner products
    and vector updates on all host threads) on the same matrix, RHS and
    hierarchy; per-iteration time x the GPU iteration count estimates
    time-to-solution.  Returns (seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    rp, ci, v = csr.arrays()
    levels = [s_plain.level(l) for l in range(s_plain.num_levels())]
    mg = orc.MG(levels)
    t0 = time.perf_counter()
    orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg=mg, max_iters=1, rel_tol=1e-8)
    return time.perf_counter() - t0, orc.num_threads()


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import xamg
    xamg.set_nv(NV)  # host-only: generator, AMG setup and the oracle need no device
    csr, B = build_problem()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    rp, ci, v = csr.arrays()
    spec = plain_spec()
    lv = xamg.amg_host(csr, xamg.Params(spec))
    mg = orc.MG(lv)
    per_iter = []
    # one sampled iteration per step, at most 3 (each takes tens of seconds)
    for _ in range(min(max(args.steps, 1), 3)):
        t0 = time.perf_counter()
        orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg=mg, max_iters=1, rel_tol=1e-8)
        per_iter.append(time.perf_counter() - t0)
    # iterations to 1e-8 of this FP64 method on this workload: 4, the count of
    # the GPU parity form, whose arithmetic is identical bit for bit (a full
    # oracle solve would take minutes per step)
    iters = args.ref_iters
    ms_rhs = float(np.mean(per_iter)) * iters / NV * 1e3
    line = {"impl": "reference", "metric": "time-to-1e-8 residual per RHS", "value": round(ms_rhs, 3),
            "unit": "ms/RHS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "27pt-aniso-128^3 AMG-PBiCGStab nv=16", "n": N_GRID, "nv": NV},
            "cpu_baseline": {"value": round(ms_rhs, 3), "unit": "ms/RHS", "cores": orc.num_threads(), "kind": "port",
                             "sample": "%d timed single PBiCGStab iterations (FP64 oracle on %d host threads, "
                                       "Gauss-Seidel sweeps sequential), x %d iterations"
                             % (len(per_iter), orc.num_threads(), iters)},
            "e2e": {"value": round(ms_rhs, 3), "unit": "ms/RHS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_case(args):
    """One hot kernel alone on a grid of side --n (for profiler captures):
    spmv = the NV=16 FP64 CSR product (variant --variant), gs = one forward +
    backward sequential Gauss-Seidel sweep (cooperative level-ordered kernel)."""
    import ctypes as C
    import torch
    import xamg
    global N_GRID
    N_GRID = args.n
    xamg.init(NV)
    csr, B = build_problem()
    if args.kernel == "spmv":
        ms = spmv_time(csr, 0, args.variant, iters=args.steps)
        print(json.dumps({"kernel": "spmv", "n": args.n, "variant": args.variant, "ms": round(ms, 4)}))
        return
    L = xamg.lib()
    rp, ci, v = csr.arrays()
    n = csr.nrows
    plan = L.xamg_gs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), 0, 1)
    assert plan
    try:
        xamg.check(L.xamg_gs_plan_set_values(plan, xamg._ptr(np.ascontiguousarray(v)), 0))
        rows = np.repeat(np.arange(n), np.diff(rp))
        diag = ci == rows
        invd = np.zeros(n)
        invd[rows[diag]] = 1.0 / v[diag]
        d = [torch.from_numpy(a).cuda() for a in (rp, ci, v, invd, B, np.zeros_like(B), np.ones(NV))]
        P = lambda t: C.c_void_p(t.data_ptr())
        times = []
        for _ in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            xamg.check(L.xamg_hsgs(plan, 0, NV, P(d[0]), P(d[1]), P(d[2]), P(d[3]), P(d[4]), P(d[5]),
                                   P(d[6]), None, None))
            xamg.check(L.XAMG_b200_synchronize())
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        assert L.xamg_gs_plan_error(plan) == 0
        print(json.dumps({"kernel": "gs", "n": args.n, "ms": round(float(np.mean(times[args.warmup:])), 4)}))
    finally:
        L.xamg_gs_plan_destroy(plan)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--forms", default="plain,mixed,batch,learned")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-iters", type=int, default=4,
                    help="PBiCGStab iterations to 1e-8 on the benchmark problem (scales the sampled iteration)")
    ap.add_argument("--kernel", choices=["spmv", "gs"], help="time one hot kernel alone (profiling)")
    ap.add_argument("--n", type=int, default=96, help="grid side of --kernel")
    ap.add_argument("--variant", type=int, default=-1, help="SpMV variant of --kernel spmv")
    ap.add_argument("--spmv", type=int, default=None,
                    help="use this SpMV kernel instead of tuning (0-6: CSR variants, 108: run kernel)")
    args = ap.parse_args()
    if args.kernel:
        return kernel_case(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import xamg
    xamg.init(NV)
    csr, B = build_problem()
    if args.spmv is not None:  # fixed kernel (profiler runs: timing under a profiler misleads the tuner)
        best_var, var_ms = args.spmv, {}
    else:
        best_var, var_ms = tune_spmv(csr, 0)
    apply_spmv_choice(best_var)
    allforms = args.forms.split(",")
    forms = [f for f in allforms if f in ("plain", "mixed")]
    res = {}
    keep = {}
    X = {}
    clocks = None
    for f in forms:
        spec = plain_spec() if f == "plain" else mixed_spec()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with Clocks(local) as ck:
            r, Xf, k = run_form(csr, B, spec, args.warmup, args.steps)
        res[f], keep[f], X[f] = r, k, Xf
        r["clocks"] = ck.summary()
        if f == forms[-1]:
            clocks = r["clocks"]
    if dist:
        t = torch.tensor([res[f]["ms"] for f in forms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        for i, f in enumerate(forms):
            res[f]["ms"] = float(t[i])
    extra = {}
    if "batch" in allforms:
        extra["batch"] = batch_form(rank, world, args.warmup, args.steps)
        if dist:
            t = torch.tensor([extra["batch"]["ms"], extra["batch"]["rhs"]], device="cuda", dtype=torch.float64)
            mx = t.clone()
            dist.all_reduce(mx, op=dist.ReduceOp.MAX)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            extra["batch"]["ms"], extra["batch"]["rhs_all_ranks"] = float(mx[0]), int(t[1])
        tot = extra["batch"].get("rhs_all_ranks", extra["batch"]["rhs"])
        extra["batch"]["ms_per_rhs"] = round(extra["batch"]["ms"] / tot, 4)
    if "learned" in allforms and rank == 0:
        extra["learned"] = learned_form()
    best = min(forms, key=lambda f: res[f]["ms"])
    spec_best = plain_spec() if best == "plain" else mixed_spec()
    e2e_ms = e2e_form(csr, B, spec_best, 1, max(2, args.steps // 2))
    roof = spmv_roofline(csr, best_var)
    roof["variants_ms"] = {str(k): round(v, 4) for k, v in var_ms.items()}
    err = None
    if "plain" in X and "mixed" in X:
        err = float(np.linalg.norm(X["mixed"] - X["plain"]) / np.linalg.norm(X["plain"]))
    # FP64 check of every form's solution on the host: max over columns of
    # ||b - A x|| / ||b||
    true_res = {}
    if rank == 0:
        import scipy.sparse as sp
        rp, ci, v = csr.arrays()
        Ah = sp.csr_matrix((v, ci, rp), shape=(csr.nrows, csr.nrows))
        for f, Xf in X.items():
            R = B - Ah @ Xf
            true_res[f] = float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)))
    cpu = None
    if rank == 0 and not args.no_cpu and "plain" in keep:
        sec, thr = cpu_sample(csr, B, keep["plain"][0])
        iters = res["plain"]["iters"]
        cpu = {"value": round(sec * iters / NV * 1e3, 3), "unit": "ms/RHS", "cores": thr, "kind": "port",
               "sample": "1 FP64 PBiCGStab iteration of the same problem and hierarchy on %d host threads "
                         "(Gauss-Seidel sweeps sequential) (%.1f s), x %d iterations / %d RHS" % (thr, sec, iters, NV)}
    value = res[best]["ms"] / (NV * world) if world > 1 else res[best]["ms"] / NV
    line = {
        "metric": "time-to-1e-8 residual per RHS", "value": round(value, 4), "unit": "ms/RHS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(res[best]["ms"], 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if best == "plain" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": "27pt-aniso-128^3 AMG-PBiCGStab nv=16", "n": N_GRID, "nv": NV,
                   "rows": csr.nrows, "nnz": csr.nnz, "parallelism": "replicas" if world > 1 else "1gpu",
                   "form": best, "l2": "inputs larger than L2 (matrix 669 MB)"},
        "forms": dict({f: {k: res[f][k] for k in ("ms", "iters", "sub_iters", "converged", "setup_s", "launches")}
                       for f in forms}, **extra),
        "mixed_vs_plain_rel_err": err, "true_rel_residual": true_res,
        "e2e": {"value": round(e2e_ms / NV, 4), "unit": "ms/RHS", "h2d_bytes_per_step": csr.nrows * NV * 8,
                "d2h_bytes_per_step": csr.nrows * NV * 8},
        "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": res[best]["launches"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
