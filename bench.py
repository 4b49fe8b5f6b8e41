"""Benchmark: H2 assembly of the Laplace single- and double-layer operators (FP64) on the
Dirichlet benchmark mesh, plus the GMRES solve, on B200.

Workload (default): unit sphere refined x64 (32768 triangles, 16386 vertices), piecewise linear
basis, Sauter-Schwab quadrature q = 2 / 4, leaf size 64, admissibility eta = 1.4, Chebyshev
interpolation m = 4.  One step = assemble both H2 matrices V (SLP) and K (DLP, alpha = 1/2): row and
column cluster bases, coupling matrices and the nearfield blocks (the nearfield of both operators
in one fused pass).  metric = nearfield entries of V and K per second ("BEM entries/s").  The
solve V u = (K + M/2) g_D, g_D = 1/|x - z|, z = (1.2, 1.2, 1.2), GMRES(50) to 1e-8, is timed
after the steps and reported under "solve".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: the path has no exchange step in this form, so N ranks run N independent replicas
(weak scaling, no collective on the data path).
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

METRIC = "BEM entries/s (FP64 nearfield entries of the SLP+DLP H2 assembly)"
UNIT = "entries/s"
Z = (1.2, 1.2, 1.2)
# algorithmic FP64 operations per quadrature point (reference source, + - * / sqrt counted as 1):
# linear-basis single layer 64, double layer 72
FLOPS_PER_POINT = {"slp": 64, "dlp": 72}
# flops the tensor-factored distant-pair sum executes per triangle pair for SLP+DLP, linear basis,
# q = 2 (FMA = 2), from the staged quadrature points: 16 point pairs x 37 (difference 3, r^2 5,
# rsqrt 13, normal part 4, three column weights per channel 12) + 4 row points x 41 (<x_a, n> 5,
# 3 x 3 x 2 outer FMAs 36) + 20 for the scaling.  The points themselves and their normal
# components are formed once per staged triangle (about 1 flop per pair, not counted).
EXECUTED_FLOPS_PER_PAIR = 16 * 37 + 4 * 41 + 20
# the same for the constant-basis single layer (dense cc SLP leg): 16 point pairs x 23
# (difference 3, r^2 5, rsqrt 13, weighted sum 2) + 4 row points x 2 (outer sum) + 2 (scaling);
# the reference counts 46 per point
CC_SLP_FLOPS_PER_PAIR = 16 * 23 + 4 * 2 + 2
CC_SLP_REF_FLOPS_PER_POINT = 46
# reference count per point of the Helmholtz kernels, constant basis (sin, cos and exp counted
# as 1): single layer 54, double layer 66
HELM_FLOPS_PER_POINT = {"slp": 54, "dlp": 66}
# DRAM bytes (read 5,998,336 + write 214,822,656) of one near_dist_kernel launch on the default
# workload (sphere split 64), from an ncu capture of the full-size run (single-pass metrics
# dram__bytes_read.sum + dram__bytes_write.sum)
NEAR_DIST_TRAFFIC = 5998336 + 214822656
# DRAM bytes (read + write) of one FP64 matvec product per algorithmic byte: 301.7 MB for
# 284.3 MB on the sphere split 48 (ncu, dram__bytes_read.sum + dram__bytes_write.sum of the three
# item-kernel launches of a product), applied to the bench's workload by its stored entries
MATVEC_TRAFFIC_RATIO = 301.7 / 284.3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--split", type=int, default=64)
    p.add_argument("--clf", type=int, default=64)
    p.add_argument("--eta", type=float, default=1.4)
    p.add_argument("--m", type=int, default=4)
    p.add_argument("--no-solve", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--batched-meshes", type=int, default=256)
    p.add_argument("--plain-sample", type=int, default=16)
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-helmholtz", action="store_true")
    p.add_argument("--no-mixed", action="store_true")
    p.add_argument("--no-dense", action="store_true")
    p.add_argument("--no-green", action="store_true")
    p.add_argument("--dense-split", type=int, default=32)
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes (profiling runs: no tuning launches)")
    p.add_argument("--serve-requests", type=int, default=500)
    p.add_argument("--cpu-batch-sample", type=int, default=8)
    p.add_argument("--cpu-serve-budget", type=float, default=60.0)
    p.add_argument("--serve-rates", default="50,200,1000,2000")
    return p.parse_args()


def workload(a):
    return {"workload": f"Laplace SLP+DLP H2 assembly, sphere split {a.split} "
                        f"({8 * a.split * a.split} triangles), linear basis, q=2/4, "
                        f"leaf {a.clf}, eta {a.eta}, m {a.m}; GMRES(50) to 1e-8",
            "triangles": 8 * a.split * a.split, "basis": "linear", "q_regular": 2,
            "q_singular": 4, "leaf_size": a.clf, "eta": a.eta, "interpolation_order": a.m,
            "l2_flush": "256 MiB buffer written between timed assembly steps; matvec products "
                        "back to back (operator larger than L2)"}


# --------------------------------------------------------------------------------------------
# distributed plumbing (replicas)
# --------------------------------------------------------------------------------------------

def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def dist_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True,
                    timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# --------------------------------------------------------------------------------------------
# CPU baseline: the unmodified reference (oracle/_ref/ref_bench, OpenMP + AVX) on the host
# --------------------------------------------------------------------------------------------

REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
REF_BENCH_CX = os.path.join(ROOT, "oracle", "_ref", "ref_bench_complex")
# reference GMRES iteration counts of config 3 (the reference's own runs, tests/golden/config3*.npz)
REF_BW_ITERATIONS = {2.0: 22, 8.0: 32}


def run_ref(exe, args, timeout=1800):
    """One run of the reference harness (oracle/ref_bench.c); None if it was not built."""
    if not os.path.exists(exe):
        return None
    out = subprocess.run([exe, *[str(x) for x in args]], capture_output=True, text=True,
                         timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed: {out.stderr[-2000:]}")
    return json.loads(out.stdout)


def run_reference_assembly(a, steps, warmup, solve=False):
    return run_ref(REF_BENCH, ["assembly", a.split, a.clf, a.eta, a.m, steps, warmup] +
                   (["--solve"] if solve else []))


def write_requests(path, reqs):
    """Request file of ref_bench's `requests` mode: (pde, kmax, k, srcs, x, t) per request."""
    import struct
    with open(path, "wb") as fh:
        fh.write(struct.pack("<I", len(reqs)))
        for pde, kmax, k, srcs, x, t in reqs:
            srcs = np.ascontiguousarray(srcs, dtype=np.float64).reshape(-1, 3)
            fh.write(struct.pack("<IIIddI", pde, kmax, 1000, k, 1e-8, srcs.shape[0]))
            fh.write(srcs.tobytes())
            fh.write(struct.pack("<II", x.shape[0], t.shape[0]))
            fh.write(np.ascontiguousarray(x, dtype=np.float64).tobytes())
            fh.write(np.ascontiguousarray(t, dtype=np.uint32).tobytes())


def run_reference_requests(reqs, budget_s):
    """Serve `reqs` one after the other with the reference (Laplace requests by the real build,
    Helmholtz ones by the complex build); per request the set-up, assembly, right-hand side and
    solve seconds, None for requests that the budget left unserved."""
    import tempfile
    out, threads = [None] * len(reqs), None
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "requests.bin")
        write_requests(path, reqs)
        for exe in (REF_BENCH, REF_BENCH_CX):
            if not any(r[0] == (exe == REF_BENCH_CX) for r in reqs):
                continue
            r = run_ref(exe, ["requests", path, budget_s])
            if r is None:
                continue
            for q in r["requests"]:
                out[q["index"]] = q
            threads = r["threads"]
    return out, threads


def cpu_baseline(a):
    """The reference on the host cores (OpenMP + AVX build, all threads): the config-2 assembly of
    V and K with H2Lib's own drivers on every block (one warm-up step, one timed step) and the
    GMRES(50) solve; config 3 (Helmholtz BW, k = 2 and 8) assembly and operator applications;
    config 4 on a sample of the ellipsoids.  The serial config-5 stream is timed in run_serving."""
    r = run_reference_assembly(a, 1, 1, solve=True)
    if r is None:
        return None
    s = r["steps"][0]
    sol = r["solve"]
    out = {"value": r["entries_per_step"] / s["seconds"], "unit": UNIT, "cores": r["threads"],
           "kind": "reference",
           "sample": f"H2Lib OpenMP+AVX build, its own drivers (cluster bases, "
                     f"assemble_bem3d_nearfield_h2matrix, assemble_bem3d_farfield_h2matrix) on "
                     f"every block of V and K, sphere split {a.split}: one warm-up step, one timed "
                     f"step ({r['entries_per_step']:.0f} entries in {s['seconds']:.2f} s)",
           "phase_s": {k: s[k] for k in ("bases", "nearfield", "farfield")},
           "solve": {"seconds": sol["seconds"], "solves_per_s": 1.0 / sol["seconds"],
                     "iterations": sol["iterations"], "matvec_seconds": sol["matvec_seconds"],
                     "what": "solve_gmres_h2matrix_avector, GMRES(50) to 1e-8 (config 2)"}}
    if not a.no_helmholtz:
        hel = []
        for k in (2.0, 8.0):
            h = run_ref(REF_BENCH_CX, ["helmholtz", 64, k, 64, 1.4, 5, 1])
            if h is None:
                break
            it = REF_BW_ITERATIONS[k]
            hel.append({"k": k, "assembly_s": h["assembly"]["seconds"],
                        "near_entries_per_s": h["entries"] / h["assembly"]["seconds"],
                        "application_s": h["application_seconds"],
                        "solve_s_estimate": it * h["application_seconds"],
                        "solves_per_s_estimate": 1.0 / (it * h["application_seconds"]),
                        "estimate": f"{it} reference GMRES iterations x one timed "
                                    "Brakhage-Werner operator application"})
        out["helmholtz"] = hel
    if not a.no_batched:
        work = batched_workload(a.batched_meshes)[:a.cpu_batch_sample]
        reqs = []
        from h2lib_b200 import bem3d as hb
        for split, axes, zs in work:
            g = hb.new_ellipsoid_surface3d(split, axes)
            reqs.append((0, 50, 0.0, zs, g.x, g.t))
        res, _ = run_reference_requests(reqs, 1e9)
        tot = sum(q["setup"] + q["assembly"] + q["rhs"] + q["solve"] for q in res)
        ns = sum(q["solves"] for q in res)
        out["batched"] = {"sample_meshes": len(res), "solves": ns, "seconds": tot,
                          "solves_per_s": ns / tot,
                          "what": "first meshes of the config-4 workload, one after the other: "
                                  "per mesh set-up, assembly of V and K, and 4 GMRES(50) solves"}
    return out


# --------------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------------

def fp64_peak_tflops(torch):
    """cuBLAS DGEMM 8192^3, best of 5 (the FP64 roofline denominator, measured in-run)."""
    n = 8192
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    B = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(A, B)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(A, B)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del A, B
    torch.cuda.empty_cache()
    return best


def run_ours(a, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    from h2lib_b200 import bem3d as hb
    from h2lib_b200._lib import check, lib
    check(lib.h2b_device_init(local), "device_init")
    L = hb.BASIS_LINEAR_BEM3D

    # ---- setup (untimed): mesh, operators, trees, H2 structure on the device
    gr = hb.new_sphere_surface3d(a.split)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    dlp = hb.new_dlp_laplace_bem3d(gr, 2, 4, L, L, 0.5)
    tree = hb.build_tree(gr, L, L, a.clf, a.eta)
    V = hb.H2Matrix(slp, tree, a.m)
    # ---- autotuner (untimed): matvec launch shape and leaf-basis split, timed on V itself; K,
    # made like V afterwards, starts from the same shape
    V.assemble()
    tune = None if a.no_autotune else V.autotune(matvec=True, leaf=True)
    K = hb.H2Matrix(dlp, tree, a.m, like=V)  # shares V's device structure
    entries = V.info()["near_entries"] + K.info()["near_entries"]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        for h in (V, K):
            check(lib.h2b_h2matrix_assemble_row_clusterbasis(h.handle), "row basis")
            check(lib.h2b_h2matrix_assemble_col_clusterbasis(h.handle), "col basis")
            check(lib.h2b_h2matrix_assemble_farfield(h.handle), "coupling")
        check(lib.h2b_h2matrix_assemble_nearfield_pair(V.handle, K.handle), "nearfield pair")
        tv, tk = V.timings(), K.timings()
        dev = sum(tv[p] + tk[p] for p in ("row_basis", "col_basis", "coupling", "near_distant",
                                           "near_singular"))
        return dev, tv, tk

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    dev_ms, wall_ms, phases = [], [], []
    import ctypes
    launches = [ctypes.c_uint64(0), ctypes.c_uint64(0)]
    with ClockSampler(local) as clocks:
        dist_barrier(world)
        torch.cuda.synchronize()
        check(lib.h2b_launch_count(ctypes.byref(launches[0])), "launch count")
        for _ in range(a.steps):
            flush.fill_(1.0)  # evict L2 between steps
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dev, tv, tk = step()
            wall_ms.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(dev)
            phases.append((tv, tk))
        check(lib.h2b_launch_count(ctypes.byref(launches[1])), "launch count")
        torch.cuda.synchronize()
        dist_barrier(world)
    step_ms = dist_max(statistics.mean(dev_ms), world)
    value = world * entries / (step_ms * 1e-3)

    # ---- roofline of the dominant kernel: fused nearfield distant-pair quadrature (FP64)
    pc = V.pair_counts()
    near_dist_ms = statistics.mean(p[0]["near_distant"] for p in phases)
    near_sing_ms = statistics.mean(p[0]["near_singular"] for p in phases)
    dist_flops = pc["distant"] * 16 * (FLOPS_PER_POINT["slp"] + FLOPS_PER_POINT["dlp"])
    sing_points = pc["vertex"] * 512 + pc["edge"] * 1536 + pc["identical"] * 1536
    # kernel evaluations the singular kernel executes for q2 = 4: the edge and identical rules
    # merged to 384 and 96 points (the kernel argument does not depend on the merged variables)
    sing_evals = pc["vertex"] * 512 + pc["edge"] * 384 + pc["identical"] * 96
    peak = fp64_peak_tflops(torch)
    # achieved: the flops the kernel's algorithm (tensor-factored pair sum) executes per launch;
    # the reference's point-by-point count of the same quadrature is reported beside it
    executed = pc["distant"] * EXECUTED_FLOPS_PER_PAIR
    achieved = executed / (near_dist_ms * 1e-3) / 1e12
    ref_tflops = dist_flops / (near_dist_ms * 1e-3) / 1e12
    # distinct triangle pairs: a pair that several nearfield blocks touch (linear basis) is
    # evaluated once per block, as in the reference; counted once here
    up = V.unique_pairs()
    uniq = {"pairs": up, "evaluations_per_distant_pair": pc["distant"] / up["distant"],
            "executed_flops": up["distant"] * EXECUTED_FLOPS_PER_PAIR,
            "reference_count_flops": up["distant"] * 16 * (FLOPS_PER_POINT["slp"] +
                                                           FLOPS_PER_POINT["dlp"])}
    uniq["executed_tflops"] = uniq["executed_flops"] / (near_dist_ms * 1e-3) / 1e12
    uniq["reference_count_tflops"] = uniq["reference_count_flops"] / (near_dist_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64", "kernel": "near_dist_kernel (fused SLP+DLP, linear basis)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": NEAR_DIST_TRAFFIC if (a.split, a.clf, a.m) == (64, 64, 4) else None,
                "flops_per_launch": executed, "flops_per_pair": EXECUTED_FLOPS_PER_PAIR,
                "distant_pairs": pc["distant"], "launch_ms": near_dist_ms,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json "
                               "has no FP64 figure)",
                "reference_count": {"flops_per_launch": dist_flops,
                                    "flops_per_pair": 16 * (FLOPS_PER_POINT["slp"] +
                                                            FLOPS_PER_POINT["dlp"]),
                                    "tflops": ref_tflops, "frac": ref_tflops / peak},
                "unique_pairs": uniq}

    # ---- matvec roofline (HBM): bytes of S, N, V, E read once per product.  The operator
    # (0.55 GB of algorithmic bytes, 0.63 GB read) is five times L2, so products run back to back
    # without a flush: a flush leaves L2 full of dirty lines whose write-back the next product
    # would pay for.
    x = torch.randn(V.cols, dtype=torch.float64, device="cuda")
    y = torch.zeros(V.rows, dtype=torch.float64, device="cuda")

    def time_mv(fn):
        for _ in range(3):
            fn(1.0, V, x, y)
        mv = []
        for _ in range(20):
            fn(1.0, V, x, y)
            mv.append(V.timings()["matvec"])
        return statistics.mean(mv)

    inf = V.info()
    mv_bytes = 8 * (inf["near_entries"] + inf["coupling_entries"] + inf["leaf_entries"]
                    + inf["transfer_entries"])
    mv_ms = time_mv(hb.addeval_h2matrix_avector)
    V.make_single()
    mv32_ms = time_mv(hb.addeval_h2matrix_avector_single)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    roof_mv = {"bound": "hbm", "kernel": "H2 matvec (all kernels of one product)",
               "achieved": mv_bytes / (mv_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
               "frac": mv_bytes / (mv_ms * 1e-3) / 1e9 / hbm,
               "traffic": int(MATVEC_TRAFFIC_RATIO * mv_bytes),
               "traffic_source": "ncu on the sphere split 48, scaled by the stored entries",
               "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s",
               "bytes_per_launch": mv_bytes, "launch_ms": mv_ms,
               "l2": "no flush between products (operator 4x larger than L2)",
               "launches_per_product": 5}
    roof_mv32 = {"bound": "hbm", "kernel": "H2 matvec from the FP32 copies (FP64 vectors/sums)",
                 "achieved": mv_bytes / 2 / (mv32_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                 "frac": mv_bytes / 2 / (mv32_ms * 1e-3) / 1e9 / hbm,
                 "bytes_per_launch": mv_bytes // 2, "launch_ms": mv32_ms,
                 "time_vs_fp64": mv32_ms / mv_ms}

    # ---- solve (FP64 GMRES(50) to 1e-8)
    solve = None
    if not a.no_solve:
        gD = hb.project_l2_harmonic(dlp, Z)
        b = hb.addeval_h2matrix_avector(1.0, K, gD, np.zeros(K.rows))
        u = np.zeros(V.rows)
        hb.solve_gmres_h2matrix_avector(V, b, u, 1e-8, 1000, 50)  # warm-up
        u[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it = hb.solve_gmres_h2matrix_avector(V, b, u, 1e-8, 1000, 50)
        t_solve = time.perf_counter() - t0
        err, nrm = hb.l2_error_harmonic(slp, Z, u)
        solve = {"seconds": t_solve, "solves_per_s": 1.0 / t_solve, "iterations": it,
                 "rel_l2_error_neumann": err / nrm,
                 "rel_residual": hb.residual_norm([V], [1.0], b, u),
                 "reference_iterations": 161, "reference_rel_l2_error": 2.297e-2}

    # ---- mixed precision: the same assembly with FP32 distant-pair quadrature (singular pairs,
    # bases and coupling FP64), then GMRES with FP32 Arnoldi products and FP64 residuals
    mixed = None
    if not a.no_mixed:
        for h in (V, K):
            h.set_precision(True)
        for _ in range(a.warmup):
            step()
        mdev = []
        for _ in range(a.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            mdev.append(step()[0])
        m_ms = dist_max(statistics.mean(mdev), world)
        tv, tk = V.timings(), K.timings()
        mixed = {"value": world * entries / (m_ms * 1e-3), "unit": UNIT, "ms_per_step": m_ms,
                 "near_distant_ms": tv["near_distant"] + tk["near_distant"],
                 "quadrature": "distant pairs FP32 (q=2), singular pairs / bases / coupling FP64"}
        if not a.no_solve:
            gD = hb.project_l2_harmonic(dlp, Z)
            bm = hb.addeval_h2matrix_avector(1.0, K, gD, np.zeros(K.rows))
            V.make_single()
            um = np.zeros(V.rows)
            hb.solve_gmres_mixed([V], [1.0], bm, um, 1e-8, 1000, 50)  # warm-up
            um[:] = 0.0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            itm = hb.solve_gmres_mixed([V], [1.0], bm, um, 1e-8, 1000, 50)
            t_m = time.perf_counter() - t0
            err, nrm = hb.l2_error_harmonic(slp, Z, um)
            mixed["solve"] = {"seconds": t_m, "solves_per_s": 1.0 / t_m, "iterations": itm,
                              "rel_residual_fp64": hb.residual_norm([V], [1.0], bm, um),
                              "rel_l2_error_neumann": err / nrm,
                              "rel_diff_to_fp64_solution":
                                  float(np.linalg.norm(um - u) / np.linalg.norm(u))
                                  if solve else None}
        for h in (V, K):
            h.set_precision(False)

    # ---- e2e: the same assembly through the C ABI from host arrays, results copied to host
    e2e = None
    if not a.no_e2e:
        pin = {}
        inf_k = K.info()
        for name, h, part in (("Vn", V, 5), ("Kn", K, 5), ("Vs", V, 4), ("Ks", K, 4)):
            n = inf["near_entries"] if part == 5 else inf["coupling_entries"]
            pin[name] = torch.empty(n, dtype=torch.float64, pin_memory=True)
        e2e_times, e2e_phases = [], []
        h2d = d2h = 0
        import ctypes
        for rep in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = hb.Surface3d(gr.x, gr.t)
            s2 = hb.new_slp_laplace_bem3d(g2, 2, 4, L, L)
            d2 = hb.new_dlp_laplace_bem3d(g2, 2, 4, L, L, 0.5)
            t1 = time.perf_counter()
            tr2 = hb.build_tree(g2, L, L, a.clf, a.eta, device=True)
            t2 = time.perf_counter()
            V2 = hb.H2Matrix(s2, tr2, a.m)
            K2 = hb.H2Matrix(d2, tr2, a.m, like=V2)
            t3 = time.perf_counter()
            for h in (V2, K2):
                check(lib.h2b_h2matrix_assemble_row_clusterbasis(h.handle), "row basis")
                check(lib.h2b_h2matrix_assemble_col_clusterbasis(h.handle), "col basis")
                check(lib.h2b_h2matrix_assemble_farfield(h.handle), "coupling")
            # the coupling matrices travel to the host while the nearfield is assembled
            for name, h in (("Vs", V2), ("Ks", K2)):
                check(lib.h2b_h2matrix_export_async(h.handle, 4, 0xFFFFFFFF,
                                                    ctypes.c_void_p(pin[name].data_ptr())),
                      "export")
            check(lib.h2b_h2matrix_assemble_nearfield_pair(V2.handle, K2.handle), "near pair")
            t4 = time.perf_counter()
            for name, h in (("Vn", V2), ("Kn", K2)):
                check(lib.h2b_h2matrix_export_async(h.handle, 5, 0xFFFFFFFF,
                                                    ctypes.c_void_p(pin[name].data_ptr())),
                      "export")
            for h in (V2, K2):
                check(lib.h2b_h2matrix_export_wait(h.handle), "export wait")
            t5 = time.perf_counter()
            e2e_times.append(t5 - t0)
            e2e_phases.append({"surface_and_operators": t1 - t0, "trees": t2 - t1,
                               "h2_structure": t3 - t2, "assembly": t4 - t3,
                               "copy_to_host": t5 - t4})
            d2h = 8 * (2 * inf["near_entries"] + 2 * inf["coupling_entries"])
            h2d = gr.x.nbytes + gr.t.nbytes + gr.n.nbytes + gr.g.nbytes
            del V2, K2, tr2, s2, d2, g2
        e2e_s = dist_max(min(e2e_times), world)
        e2e = {"value": world * entries / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "includes": "mesh upload, operators, cluster/block trees (h2b_tree_new_device), "
                           "H2 structure "
                           "upload, assembly of V and K, copy of all nearfield and coupling "
                           "blocks to pinned host memory (coupling copies overlap the nearfield "
                           "assembly; 'assembly' then includes that overlap)",
               "phase_ms": {k: 1e3 * e2e_phases[e2e_times.index(min(e2e_times))][k]
                            for k in e2e_phases[0]}}

    res = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload(a), parallelism=f"replicas{world}"),
        "entries_per_step": entries, "wall_ms_per_step": statistics.mean(wall_ms),
        "phase_ms": {k: statistics.mean(p[0][k] + p[1][k] for p in phases)
                     for k in ("row_basis", "col_basis", "coupling")} |
                    {"near_distant_fused": near_dist_ms, "near_singular_fused": near_sing_ms},
        "pairs_per_operator": pc, "singular_points": sing_points,
        "singular_kernel_evaluations": sing_evals,
        "roofline": roofline, "roofline_matvec": roof_mv, "roofline_matvec_fp32": roof_mv32,
        "autotune": None if tune is None else {
            "shape": tune["shape"], "matvec_ms_start": tune["matvec_ms"][0],
            "matvec_ms_tuned": tune["matvec_ms"][1], "bases_ms_start": tune["bases_ms"][0],
            "bases_ms_tuned": tune["bases_ms"][1],
            "what": "h2b_h2matrix_autotune on V before the warm-up (matvec launch shape and "
                    "leaf-basis CTAs per leaf); K is made like V afterwards"},
        "solve": solve, "mixed": mixed,
        "e2e": e2e,
        "clocks": clocks.summary(),
        # kernels the library launched in the timed steps (its own launch counter)
        "gpu_launches": int(launches[1].value - launches[0].value),
    }
    return res


BATCH_SEED = 20261203


def batched_workload(nmesh, seed=BATCH_SEED):
    """Uneven ellipsoids: semi-axes U[0.5, 2]^3, triangle counts log-uniform in [128, 8192]
    realised as sphere refinements split = round(sqrt(T / 8)) in [4, 32], 4 point sources each,
    uniform on the sphere of radius 3 x the largest semi-axis (numpy PCG64, fixed seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nmesh):
        axes = rng.uniform(0.5, 2.0, 3)
        tri = float(np.exp(rng.uniform(np.log(128.0), np.log(8192.0))))
        split = int(np.clip(round(np.sqrt(tri / 8.0)), 4, 32))
        v = rng.standard_normal((4, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        out.append((split, axes, 3.0 * axes.max() * v))
    return out


def run_batched(a):
    """Batched uneven Laplace Dirichlet solves (all meshes as one forest H2 matrix, one assembly,
    the 4 right-hand sides of every mesh solved together with FP32 Arnoldi steps and FP64
    residuals to 1e-8) against the plain FP64 path (one mesh and one right-hand side per call) on
    a sample of the same meshes."""
    import torch
    from h2lib_b200 import bem3d as hb
    from h2lib_b200._lib import check, lib
    L = hb.BASIS_LINEAR_BEM3D
    work = batched_workload(a.batched_meshes)
    nrhs = 4

    def one_batch(meshes):
        t0 = time.perf_counter()
        surfs = [hb.new_ellipsoid_surface3d(s, ax) for s, ax, _ in meshes]
        gu, voff, toff = hb.union_surface3d(surfs)
        slp = hb.new_slp_laplace_bem3d(gu, 2, 4, L, L)
        dlp = hb.new_dlp_laplace_bem3d(gu, 2, 4, L, L, 0.5)
        forest = hb.build_forest(gu, voff, toff, L, L, a.clf, a.eta)
        th = time.perf_counter()
        V = hb.H2Matrix(slp, forest, a.m)
        K = hb.H2Matrix(dlp, forest, a.m, like=V)
        V.set_precision(True)   # FP32 distant-pair quadrature (singular pairs FP64)
        K.set_precision(True)
        t1 = time.perf_counter()
        for h in (V, K):
            check(lib.h2b_h2matrix_assemble_row_clusterbasis(h.handle), "row basis")
            check(lib.h2b_h2matrix_assemble_col_clusterbasis(h.handle), "col basis")
            check(lib.h2b_h2matrix_assemble_farfield(h.handle), "coupling")
        check(lib.h2b_h2matrix_assemble_nearfield_pair(V.handle, K.handle), "near pair")
        V.make_single()
        t2 = time.perf_counter()
        zs = np.stack([np.stack([z[r] for _, _, z in meshes]) for r in range(nrhs)])
        gD = hb.project_l2_harmonic_multi(dlp, toff, zs)
        n = gu.vertices
        B = np.zeros((nrhs, n))
        check(lib.h2b_h2matrix_addeval_multi(1.0, 0.0, K.handle, nrhs, hb._ptr(gD), n,
                                             hb._ptr(B), n), "rhs")
        X = np.zeros((nrhs, n))
        t3 = time.perf_counter()
        its = hb.solve_gmres_batch([V], [1.0], voff, B, X, 1e-8, 1000, 50, nrhs=nrhs, mixed=True)
        t4 = time.perf_counter()
        err, nrm = hb.l2_error_harmonic_multi(slp, toff, zs, X)
        res = []
        for r in range(nrhs):
            y = hb.addeval_h2matrix_avector(1.0, V, X[r].copy(), np.zeros(n))
            for m in range(len(meshes)):
                lo, hi = int(voff[m]), int(voff[m + 1])
                res.append(np.linalg.norm(B[r, lo:hi] - y[lo:hi]) / np.linalg.norm(B[r, lo:hi]))
        return {"seconds": t4 - t0, "setup_s": t1 - t0, "setup_h2_structure_s": t1 - th,
                "assembly_s": t2 - t1,
                "rhs_s": t3 - t2, "solve_s": t4 - t3, "iterations": its,
                "max_rel_residual_fp64": float(max(res)), "rel_l2_error": err / nrm,
                "unknowns": int(n) * nrhs, "triangles": int(gu.triangles)}

    # warm-up on the same meshes: module load, graph code paths, and the device memory pool
    # grown to the batch's size (a batched solve service reuses its pool)
    one_batch(work)
    torch.cuda.synchronize()
    b = one_batch(work)

    # plain FP64 path on a sample: one mesh per H2 matrix, one right-hand side per GMRES call
    sample = work[:a.plain_sample]
    t0 = time.perf_counter()
    plain_its, plain_err = [], []
    for s, ax, zs in sample:
        g = hb.new_ellipsoid_surface3d(s, ax)
        slp = hb.new_slp_laplace_bem3d(g, 2, 4, L, L)
        dlp = hb.new_dlp_laplace_bem3d(g, 2, 4, L, L, 0.5)
        tree = hb.build_tree(g, L, L, a.clf, a.eta)
        V = hb.H2Matrix(slp, tree, a.m).assemble()
        K = hb.H2Matrix(dlp, tree, a.m, like=V).assemble()
        for r in range(nrhs):
            gD = hb.project_l2_harmonic(dlp, zs[r])
            rhs = hb.addeval_h2matrix_avector(1.0, K, gD, np.zeros(K.rows))
            u = np.zeros(V.rows)
            plain_its.append(hb.solve_gmres_h2matrix_avector(V, rhs, u, 1e-8, 1000, 50))
            e, nn = hb.l2_error_harmonic(slp, zs[r], u)
            plain_err.append(e / nn)
    t_plain = time.perf_counter() - t0
    nsolves = nrhs * len(work)
    its = b["iterations"]
    return {
        "workload": f"{len(work)} ellipsoids (semi-axes U[0.5,2]^3, {min(w[0] for w in work)}.."
                    f"{max(w[0] for w in work)} splits, {b['triangles']} triangles), 4 point-source "
                    f"Dirichlet RHS each, linear basis, q 2/4, leaf {a.clf}, eta {a.eta}, m {a.m}, "
                    f"GMRES(50) to 1e-8 (FP64 residual); seed {BATCH_SEED}",
        "solves": nsolves, "seconds": b["seconds"], "solves_per_s": nsolves / b["seconds"],
        "phase_s": {k: b[k] for k in ("setup_s", "setup_h2_structure_s", "assembly_s", "rhs_s",
                                      "solve_s")},
        "iterations": {"min": int(its.min()), "median": float(np.median(its)),
                       "max": int(its.max())},
        "max_rel_residual_fp64": b["max_rel_residual_fp64"],
        "rel_l2_error_neumann": {"median": float(np.median(b["rel_l2_error"])),
                                 "max": float(np.max(b["rel_l2_error"]))},
        "precision": "FP32 distant-pair quadrature (singular pairs FP64), FP32 H2 matrix copies "
                     "in the Arnoldi steps, FP64 residuals and stopping test",
        "plain_fp64": {"sample_meshes": len(sample), "solves": nrhs * len(sample),
                       "seconds": t_plain, "solves_per_s": nrhs * len(sample) / t_plain,
                       "iterations_median": float(np.median(plain_its)),
                       "rel_l2_error_neumann_median": float(np.median(plain_err)),
                       "path": "per mesh: h2b_tree_new + 2 H2 matrices + per RHS "
                               "h2b_solve_gmres (FP64)"},
        "speedup_vs_plain_fp64": (nsolves / b["seconds"]) / (nrhs * len(sample) / t_plain),
    }


def run_dense(a, peak):
    """Dense constant-basis single layer on the sphere split 32 (8192 triangles, q = 2 / 4;
    assemble_bem3d_amatrix, Library/bem3d.c:9988) into device memory: every triangle pair once,
    no shared-memory scatter.  The distant-pair kernel is timed by the operator's own events."""
    import scipy.sparse as sps
    import torch
    from h2lib_b200 import bem3d as hb
    gr = hb.new_sphere_surface3d(a.dense_split)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, hb.BASIS_CONSTANT_BEM3D, hb.BASIS_CONSTANT_BEM3D)
    n = gr.triangles
    G = torch.empty((n, n), dtype=torch.float64, device="cuda")  # 512 MB: larger than L2
    # pairs by vertices shared, from the incidence matrix
    t = gr.t.astype(np.int64)
    M = sps.csr_matrix((np.ones(3 * n), (np.repeat(np.arange(n), 3), t.ravel())),
                       shape=(n, gr.vertices))
    S = (M @ M.T).tocoo()
    sing = np.bincount(np.minimum(S.data.astype(np.int64), 3), minlength=4)
    distant = n * n - int(S.nnz)
    for _ in range(3):
        hb.assemble_bem3d_amatrix(slp, G)
    dist_ms, sing_ms, wall = [], [], []
    for _ in range(5):
        t0 = time.perf_counter()
        hb.assemble_bem3d_amatrix(slp, G)
        wall.append((time.perf_counter() - t0) * 1e3)
        ms = slp.timings()
        dist_ms.append(ms["near_distant"])
        sing_ms.append(ms["near_singular"])
    d = statistics.mean(dist_ms)
    executed = distant * CC_SLP_FLOPS_PER_PAIR
    ref = distant * 16 * CC_SLP_REF_FLOPS_PER_POINT
    del G
    torch.cuda.empty_cache()
    return {"workload": f"dense cc SLP, sphere split {a.dense_split} ({n} triangles), q 2 / 4, "
                        "FP64, output in device memory",
            "pairs": {"distant": distant, "vertex": int(sing[1]), "edge": int(sing[2]),
                      "identical": int(sing[3])},
            "near_distant_ms": d, "near_singular_ms": statistics.mean(sing_ms),
            "call_wall_ms": statistics.mean(wall),
            "roofline": {"bound": "fp64", "kernel": "near_dist_kernel (constant basis SLP)",
                         "flops_per_pair": CC_SLP_FLOPS_PER_PAIR,
                         "achieved": executed / (d * 1e-3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": executed / (d * 1e-3) / 1e12 / peak,
                         "reference_count": {
                             "flops_per_pair": 16 * CC_SLP_REF_FLOPS_PER_POINT,
                             "tflops": ref / (d * 1e-3) / 1e12,
                             "frac": ref / (d * 1e-3) / 1e12 / peak}}}


def run_green(a):
    """Laplace single layer with the greenhybrid farfield (setup_h2matrix_aprx_greenhybrid_bem3d,
    Library/bem3d.c:9689; the reference test's m 2, l 1, delta 1, accuracy 5e-3) on the sphere
    and tree of the headline workload (split 64, 32768 triangles, leaf 64, eta 1.4 by default):
    per-phase device times of the assembly, the matvec, the ranks, the product's
    distance from the interpolation H2 matrix (m 4), and the reference's CPU assembly of the same
    matrix (oracle/_ref/ref_bench green)."""
    from h2lib_b200 import bem3d as hb
    L = hb.BASIS_LINEAR_BEM3D
    gr = hb.new_sphere_surface3d(a.split)
    tree = hb.build_tree(gr, L, L, a.clf, a.eta)
    slp = hb.new_slp_laplace_bem3d(gr, 2, 4, L, L)
    H = hb.H2Matrix(slp, tree, 2, green=(1, 1.0, 5e-3))
    H.assemble()
    walls, phases = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        H.assemble()
        walls.append(time.perf_counter() - t0)
        phases.append(H.timings())
    ph = {k: statistics.mean(p[k] for p in phases) for k in phases[0]}
    rng = np.random.default_rng(4)
    x = rng.standard_normal(H.cols)
    y = hb.addeval_h2matrix_avector(1.0, H, x.copy(), np.zeros(H.rows))
    mv = []
    for _ in range(5):
        hb.addeval_h2matrix_avector(1.0, H, x.copy(), np.zeros(H.rows))
        mv.append(H.timings()["matvec"])
    Vi = hb.H2Matrix(slp, tree, 4).assemble()
    yi = hb.addeval_h2matrix_avector(1.0, Vi, x.copy(), np.zeros(H.rows))
    rk = H.green_ranks(0)
    out = {"workload": f"Laplace SLP, sphere split {a.split} ({gr.triangles} triangles), linear "
                       f"basis, q 2/4, leaf {a.clf}, eta {a.eta}, greenhybrid m 2 l 1 delta 1 "
                       "accuracy 5e-3 (k = 48)",
           "assembly_wall_s": statistics.mean(walls),
           "phase_ms": {"bases": ph["row_basis"] + ph["col_basis"], "coupling": ph["coupling"],
                        "near_distant": ph["near_distant"], "near_singular": ph["near_singular"]},
           "matvec_ms": statistics.mean(mv),
           "ranks": {"root": int(rk[0]), "mean": float(rk.mean()), "max": int(rk.max())},
           "rel_diff_vs_interpolation_m4": float(np.linalg.norm(y - yi) / np.linalg.norm(yi))}
    ref = run_ref(REF_BENCH, ["green", a.split, a.clf, a.eta, 2, 1, 1.0, 5e-3])
    if ref is not None:
        out["cpu_reference"] = ref
        out["assembly_speedup_vs_cpu_reference"] = ref["seconds"] / out["assembly_wall_s"]
    return out


def run_helmholtz(a, peak):
    """Brakhage-Werner solves of config 3: unit cube split 64 (49152 triangles), constant basis,
    q 2/4, leaf 64, eta 1.4, m 5, plane wave along (1,1,1)/sqrt(3), GMRES(80) to 1e-8, k = 2
    and 8; FP64 with the reference's Givens rotations, FP64 with unitary rotations, and mixed
    precision (unitary)."""
    import torch
    from h2lib_b200 import bem3d as hb
    from h2lib_b200._lib import check, lib
    C = hb.BASIS_CONSTANT_BEM3D
    d = np.ones(3) / np.sqrt(3.0)
    out = []
    gr = hb.new_cube_surface3d(64)
    tree = hb.build_tree(gr, C, C, 64, 1.4)
    for k in (2.0, 8.0):
        slp = hb.new_slp_helmholtz_bem3d(k, gr, 2, 4, C, C)
        dlp = hb.new_dlp_helmholtz_bem3d(k, gr, 2, 4, C, C, 0.5)
        V = hb.H2Matrix(slp, tree, 5)
        K = hb.H2Matrix(dlp, tree, 5, like=V)  # shares V's device structure
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for h in (V, K):
            check(lib.h2b_h2matrix_assemble_row_clusterbasis(h.handle), "row basis")
            check(lib.h2b_h2matrix_assemble_col_clusterbasis(h.handle), "col basis")
            check(lib.h2b_h2matrix_assemble_farfield(h.handle), "coupling")
        # one nearfield pass for both operators (one sine and cosine per point for both kernels)
        check(lib.h2b_h2matrix_assemble_nearfield_pair(V.handle, K.handle), "nearfield pair")
        t_asm = time.perf_counter() - t0
        b = hb.integrate_plane_wave(slp, k * d, coef=-1.0)
        u64 = np.zeros(V.rows, dtype=np.complex128)
        t0 = time.perf_counter()
        it64 = hb.solve_gmres([K, V], [1.0, -1j * k], b, u64, 1e-8, 1000, 80)
        t64 = time.perf_counter() - t0
        # unitary complex Givens rotations: the stop at 1e-8 holds for the true residual
        uu = np.zeros(V.rows, dtype=np.complex128)
        t0 = time.perf_counter()
        itu = hb.solve_gmres([K, V], [1.0, -1j * k], b, uu, 1e-8, 1000, 80, unitary=True)
        tu = time.perf_counter() - t0
        V.make_single()
        K.make_single()
        u32 = np.zeros(V.rows, dtype=np.complex128)
        t0 = time.perf_counter()
        it32 = hb.solve_gmres_mixed([K, V], [1.0, -1j * k], b, u32, 1e-8, 1000, 80)
        t32 = time.perf_counter() - t0
        # the reference's exterior test problem (Tests/test_helmholtzbem3d.c:422) on this mesh: a
        # point source at (0, 0, 0.2) inside the cube, its field as Dirichlet datum, and the
        # solution's exterior field against the exact one at the reference's evaluation points
        # (max_rel_outer_error, Tests/test_helmholtzbem3d.c:224)
        src = (0.0, 0.0, 0.2)
        bp = hb.integrate_point_source(K.bem, src, k)
        up = np.zeros(V.rows, dtype=np.complex128)
        t0 = time.perf_counter()
        itp = hb.solve_gmres([K, V], [1.0, -1j * k], bp, up, 1e-8, 1000, 80, unitary=True)
        tp = time.perf_counter() - t0
        pts = hb.outer_points()
        field = hb.eval_brakhage_werner(slp, up, pts, k)
        exact = hb.point_source_field(pts, src, k)
        point = {"iterations": itp, "seconds": tp,
                 "max_rel_field_error": float(np.max(np.abs(field - exact) / np.abs(exact))),
                 "points": len(pts),
                 "what": "exterior Dirichlet problem with the field of a point source at (0, 0, "
                         "0.2) as datum, FP64 GMRES(80) to 1e-8 (unitary rotations); maximal "
                         "relative error of the Brakhage-Werner field against e^{ikr}/r on the "
                         "reference test's 20 x 20 grid of the plane y = 0, |x| <= 10, outside "
                         "the unit disc"}
        ent = V.info()["near_entries"] + K.info()["near_entries"]
        # distant-pair kernels of V and K, in the reference's count (sin / cos / exp = 1 flop):
        # 16 points per pair x 54 (single layer) or 66 (double layer)
        tv, tk, pcv = V.timings(), K.timings(), V.pair_counts()
        ref_flops = pcv["distant"] * 16 * (HELM_FLOPS_PER_POINT["slp"] +
                                           HELM_FLOPS_PER_POINT["dlp"])
        near = {"pairs": pcv, "phase_ms": {"V": tv, "K": tk},
                "fused": "one pass for V and K, timed on V", "slp_distant_ms": tv["near_distant"],
                "slp_singular_ms": tv["near_singular"], "dlp_distant_ms": tk["near_distant"],
                "dlp_singular_ms": tk["near_singular"],
                "reference_count_tflops": ref_flops / ((tv["near_distant"] + tk["near_distant"])
                                                       * 1e-3) / 1e12}
        near["reference_count_frac"] = near["reference_count_tflops"] / peak
        out.append({"k": k, "assembly_s": t_asm, "near_entries_per_s": ent / t_asm,
                    "nearfield": near, "point_source": point,
                    "fp64": {"iterations": it64, "seconds": t64,
                             "rel_residual": hb.residual_norm([K, V], [1.0, -1j * k], b, u64)},
                    "fp64_unitary": {"iterations": itu, "seconds": tu,
                                     "rel_residual": hb.residual_norm([K, V], [1.0, -1j * k], b,
                                                                      uu)},
                    "mixed": {"iterations": it32, "seconds": t32,
                              "rel_residual": hb.residual_norm([K, V], [1.0, -1j * k], b, u32),
                              "rel_diff_to_fp64": float(np.linalg.norm(u32 - u64) /
                                                        np.linalg.norm(u64))},
                    "reference_iterations": {2.0: 22, 8.0: 32}[k]})
        del V, K, slp, dlp
    return {"workload": "config 3: cube 49152 triangles, Helmholtz Brakhage-Werner, constant "
                        "basis, m 5, GMRES(80) to 1e-8", "runs": out}


def serving_workload(n, seed):
    """Request stream: geometry uniform over sphere / cube / ellipsoid (semi-axes U[0.5, 2]^3),
    triangle counts log-uniform in [512, 32768], Laplace (point source at 3x the extent) or
    Helmholtz (k ~ U[1, 6], random plane-wave direction) with equal probability."""
    from h2lib_b200 import bem3d as hb
    from h2lib_b200.serve import HELMHOLTZ, LAPLACE
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        kind = int(rng.integers(3))
        tri = float(np.exp(rng.uniform(np.log(512.0), np.log(32768.0))))
        axes = rng.uniform(0.5, 2.0, 3)
        if kind == 1:
            g = hb.new_cube_surface3d(max(3, int(round(np.sqrt(tri / 12.0)))))
            ext = np.sqrt(3.0)
        elif kind == 0:
            g = hb.new_sphere_surface3d(max(4, int(round(np.sqrt(tri / 8.0)))))
            ext = 1.0
        else:
            g = hb.new_ellipsoid_surface3d(max(4, int(round(np.sqrt(tri / 8.0)))), axes)
            ext = float(axes.max())
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        if rng.random() < 0.5:
            out.append((g, LAPLACE, 3.0 * ext * d, 0.0))
        else:
            out.append((g, HELMHOLTZ, d, float(rng.uniform(1.0, 6.0))))
    return out


def run_serving(a):
    """Poisson request streams through the solve server (8 slots, 150 GB budget, mixed
    precision), then the plain FP64 form (one slot, FP64) on the same requests."""
    from h2lib_b200.serve import Server
    rates = [float(r) for r in a.serve_rates.split(",")]
    reqs = serving_workload(a.serve_requests, BATCH_SEED + 1)
    rng = np.random.default_rng(BATCH_SEED + 2)

    def serve(requests, slots, mixed, rate, batching=64):
        srv = Server(slots=slots, hbm_budget=150 << 30, batching=batching)
        try:
            for g, pde, src, k in requests[:2]:  # warm-up of the code paths
                srv.wait(srv.submit(g, pde, src, k=k, mixed=mixed))
            gaps = rng.exponential(1.0 / rate, len(requests)) if rate else np.zeros(len(requests))
            t0 = time.perf_counter()
            ids, due = [], 0.0
            for (g, pde, src, k), gap in zip(requests, gaps):
                due += gap
                dt = t0 + due - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(g, pde, src, k=k, mixed=mixed))
            res = [srv.wait(i)[1] for i in ids]
        finally:
            srv.close()
        lat = np.array([r["t_done"] - r["t_submit"] for r in res])
        span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        return {"rate_req_s": rate, "requests": len(res), "solves_per_s": len(res) / span,
                "latency_p50_s": float(np.percentile(lat, 50)),
                "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.median([r["t_start"] - r["t_submit"] for r in res])),
                "mean_phase_s": {p: float(np.mean([r["t_" + p] for r in res]))
                                 for p in ("setup", "assembly", "rhs", "solve")},
                "max_rel_residual_fp64": float(max(r["rel_residual"] for r in res)),
                "iterations_median": float(np.median([r["iterations"] for r in res]))}

    sweep = [serve(reqs, 8, True, r) for r in rates]
    plain = serve(reqs, 1, False, 0.0, batching=1)
    best = max(s["solves_per_s"] for s in sweep)
    cpu = None if a.no_cpu_baseline else cpu_serving(a, reqs, rates)
    return {"workload": f"{len(reqs)} requests per rate: sphere/cube/ellipsoid, 512..32768 "
                        f"triangles, Laplace (linear, m 4) or Helmholtz BW (k 1..6, constant, m 5),"
                        f" GMRES to 1e-8 (FP64 residual); seed {BATCH_SEED + 1}",
            "server": "8 slots, 150 GB HBM budget, FP32 Arnoldi steps + FP64 residuals, queued "
                      "Laplace requests batched (forest H2 matrix, batched GMRES)",
            "sweep": sweep,
            "plain_fp64": dict(plain, path="1 slot, FP64, no batching, requests back to back"),
            "speedup_vs_plain_fp64": best / plain["solves_per_s"],
            "cpu_reference": cpu}


def cpu_serving(a, reqs, rates):
    """The same stream served one request at a time by the reference (OpenMP + AVX build, all
    host threads): the requests of the stream in arrival order are served until the time budget
    is spent, and first-in first-out queueing at each arrival rate is replayed from the measured
    service times (seeded exponential gaps)."""
    from h2lib_b200.serve import HELMHOLTZ
    rr = [(1 if pde == HELMHOLTZ else 0, 80 if pde == HELMHOLTZ else 50, k, src, g.x, g.t)
          for g, pde, src, k in reqs]
    res, threads = run_reference_requests(rr, a.cpu_serve_budget)
    served = [i for i, q in enumerate(res) if q is not None]
    if not served:
        return None
    # requests before the first unserved one keep the stream's order
    prefix = []
    for i, q in enumerate(res):
        if q is None:
            break
        prefix.append(q["setup"] + q["assembly"] + q["rhs"] + q["solve"])
    rng = np.random.default_rng(BATCH_SEED + 3)
    sweep = []
    for rate in rates:
        arr = np.cumsum(rng.exponential(1.0 / rate, len(prefix)))
        done, free = [], 0.0
        for t_arr, svc in zip(arr, prefix):
            free = max(free, t_arr) + svc
            done.append(free)
        lat = np.array(done) - arr
        sweep.append({"rate_req_s": rate, "requests": len(prefix),
                      "solves_per_s": len(prefix) / (done[-1] - arr[0]),
                      "latency_p50_s": float(np.percentile(lat, 50)),
                      "latency_p99_s": float(np.percentile(lat, 99))})
    return {"cores": threads, "kind": "reference", "served": len(served),
            "service_s": {"median": float(np.median(prefix)), "max": float(np.max(prefix))},
            "sample": f"the first {len(prefix)} requests of the stream (budget "
                      f"{a.cpu_serve_budget:.0f} s), one after the other; FIFO queueing replayed "
                      f"at each rate from the measured service times",
            "sweep": sweep}


def main():
    a = parse()
    rank, world, local = dist_init(a.gpus)
    if a.impl == "reference":
        if rank != 0:
            return 0
        r = run_reference_assembly(a, a.steps, a.warmup)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/ref_bench not built (H2Lib sources absent at build)"}))
            return 0
        secs = [s["seconds"] for s in r["steps"]]
        value = r["entries_per_step"] / statistics.mean(secs)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": statistics.mean(secs) * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(workload(a), parallelism="cpu"), "impl": "reference",
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"],
                                 "kind": "reference",
                                 "sample": "every block of V and K per step, H2Lib's own drivers "
                                           "(cluster bases, assemble_bem3d_nearfield_h2matrix, "
                                           "assemble_bem3d_farfield_h2matrix), OpenMP+AVX build"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    res = run_ours(a, rank, world, local)
    if rank == 0:
        if not a.no_batched:
            try:
                res["batched"] = run_batched(a)
            except Exception as e:  # reported, never hides the headline line
                res["batched"] = {"error": str(e)[:300]}
        if not a.no_dense:
            try:
                res["dense_cc_slp"] = run_dense(a, res["roofline"]["peak"])
            except Exception as e:  # reported, never hides the headline line
                res["dense_cc_slp"] = {"error": str(e)[:300]}
        if not a.no_helmholtz:
            try:
                res["helmholtz"] = run_helmholtz(a, res["roofline"]["peak"])
            except Exception as e:  # reported, never hides the headline line
                res["helmholtz"] = {"error": str(e)[:300]}
        if not a.no_green:
            try:
                res["greenhybrid"] = run_green(a)
            except Exception as e:  # reported, never hides the headline line
                res["greenhybrid"] = {"error": str(e)[:300]}
        if not a.no_serving:
            try:
                res["serving"] = run_serving(a)
            except Exception as e:  # reported, never hides the headline line
                res["serving"] = {"error": str(e)[:300]}
        if not a.no_cpu_baseline:
            try:
                res["cpu_baseline"] = cpu_baseline(a)
            except Exception as e:  # the baseline is reported, never required
                res["cpu_baseline"] = {"unavailable": str(e)[:200]}
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
