"""Benchmark: worst-case topology-optimisation design iterations per second
on a 256^3 voxel box (the adjoint-through-spline configuration): tricubic
B-spline density (32^3 coefficients ~ N(0.5, 0.15)), Heaviside beta=8,
bottom face clamped, free-force worst case over the top-face nodes (20
Lanczos steps, each a multigrid solve to relative residual 1e-6), 45 degree
self-support constraint, volume fraction 0.3, MMA update.

One step = one full design iteration through the C ABI.  The mixed path
(FP32 V-cycle inside FP64 CG) is the headline; the plain FP64 GPU path is
measured beside it.  Data are synthetic and seeded.  Inputs (17M nodes)
exceed the 126 MB L2, so no flush is inserted between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--size S]
  python bench.py --mode solve [--precision mixed|fp64] [--size S]
  python bench.py --mode batch|problems|scale|mesh|surface

`--mode solve` times single multigrid-preconditioned CG solves (to relative
residual 1e-6) on the density of the seeded initial design, with a seeded
load on the top-face nodes, and reports per-iteration time and the live
per-kernel-class CUDA-event profile (the kernel mix of one Lanczos step).

With torchrun each rank runs an independent replica (the path does not
shard: one design problem per GPU), timing is max over ranks.
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

METRIC = ("worst-case TO design iterations/s @256^3 (mixed: FP32 V-cycle and CG recurrence, FP64 residual "
          "replacement; true rel.resid 1e-6)")
UNIT = "iter/s"
# V-cycle smoother: 2 + 2 Chebyshev steps for D^-1 K on [0.07 lambda_max,
# lambda_max].  On this workload a 256^3 solve of the seeded design's density
# takes 11 PCG iterations with it (32.3 ms), 11 with 0.05, 12 with 0.1
# (34.8 ms), 16 with 0.03 and 37 with 0.02 (the interval then reaches below
# what the power-iteration estimate of lambda_max supports), 14 with
# [lambda_max/4, lambda_max], 16 with damped Jacobi (omega = 0.8) and 18 with
# omega = 0.6, at the same cost per iteration; 3 + 3 and 4 + 4 steps take 9
# and 8 iterations but longer (33.8 and 36.5 ms with 0.05).  A design
# iteration's 20 Lanczos solves take 265 PCG iterations at 0.07, 275 at 0.1.
SMOOTHER = "chebyshev"
OMEGA = 0.8
CHEB_LOWER = 0.07
SMOOTH_STEPS = 2  # Chebyshev steps before and after the coarse correction


def problem(n, seed=2026):
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[0] = 1
    la = np.zeros((n + 1,) * 3, np.uint8)
    la[n] = 1
    order = 4
    parts = 32 - order
    rng = np.random.default_rng(seed)
    coeff = np.clip(rng.normal(0.5, 0.15, 32 ** 3), 0.0, 1.0)
    return em, fa, la, order, parts, coeff


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                          "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and "Active" in s[5 + i]
                          and "Not" not in s[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(backend=None):
    """One process per GPU (torchrun env); replicas exchange only barriers and
    the max of their timings.  NCCL on GPUs, gloo for host-only runs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.barrier()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, world, rank):
    """CPU reference arm: the FP64 oracle restatement of the reference method
    (the reference itself cannot be built here), one bounded design iteration
    per step at args.ref_size^3, scaled to 256^3 by the element count."""
    if rank != 0:
        return
    from oracle import oracle as O
    n = args.ref_size
    em, fa, la, order, parts, coeff = problem(n)
    cores = os.cpu_count()
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle_design_iteration(O, n, em, fa, la, order, parts, coeff)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    per_iter = statistics.mean(times) * (256.0 / n) ** 3
    value = 1.0 / per_iter
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_iter * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "256^3 worst-case spline TO iteration (config 4 shape)", "sample_size": n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"FP64 oracle design iteration at {n}^3 (20 Lanczos steps, MG-PCG to 1e-6), "
                                       f"time scaled by (256/{n})^3"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def oracle_design_iteration(O, n, em, fa, la, order, parts, coeff, beta=8.0):
    """The FP64 oracle's design iteration: spline -> Heaviside -> operators ->
    Lanczos worst case -> self-support -> adjoint chain -> MMA."""
    p = O.Problem(em, fa, la, None, nu=0.3, n_levels=0, first_factor=4)
    p.spline_setup(order, (parts, parts, parts))
    rh = p.coeff2density(coeff)
    rho = O.heaviside(rh, beta, 1e-3)
    p.set_density(rho)
    p.update_stencil()
    lam, fw, uw, _ = p.lanczos(20, 0, tol=1e-6)
    ssv, _, dss, _, _ = p.selfsupport(coeff, beta, 4)
    s = p.sensitivity(uw)
    s = O.heaviside_chain(rh, beta, s)
    v = O.heaviside_chain(rh, beta, np.full(p.ne, 1.0 / p.ne))
    s = p.filter(2.0, s)
    v = p.filter(2.0, v)
    dc = p.density2coeff_adjoint(s)
    dv = p.density2coeff_adjoint(v)
    m = O.MMA(len(coeff), 2, 0.0, 1.0)
    m.set_x(coeff)
    m.update(dc * 1e6, np.stack([dv * 1e3, dss * 1e3]), np.array([1e3 * (rho.mean() - 0.3), 1e3 * ssv]))
    return lam, p.solve_iterations()


def cpu_samples(O, sizes, coeff):
    """One FP64 oracle design iteration per sample size: seconds, PCG
    iterations over the 20 Lanczos solves, and microseconds per element and
    PCG iteration (flat when the cost scales with elements x iterations)."""
    out = []
    for nr in sizes:
        emr, far, lar, order, parts, _ = problem(nr)
        t0 = time.perf_counter()
        _, its = oracle_design_iteration(O, nr, emr, far, lar, order, parts, coeff)
        dt = time.perf_counter() - t0
        out.append({"n": nr, "s": dt, "pcg_iterations": int(its), "us_per_element_iteration": 1e6 * dt / (nr ** 3 * its)})
    return out


def smoother_id(R):
    return {"chebyshev": R.rso.SMOOTH_CHEBYSHEV, "jacobi": R.rso.SMOOTH_JACOBI, "gs": R.rso.SMOOTH_GS}[SMOOTHER]


def kernel_classes(g):
    """Per-class CUDA-event profile recorded on handle g: launches, mean
    microseconds and algorithmic GB/s of each class that ran."""
    import ctypes
    lib = g.lib
    name = ctypes.create_string_buffer(64)
    cnt, tot, b, fl = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    classes = {}
    for cls in range(16):
        if lib.rso_profile_class(g.h, cls, name, 64, ctypes.byref(cnt), ctypes.byref(tot), ctypes.byref(b),
                                 ctypes.byref(fl)) != 0:
            break
        if cnt.value:
            avg = tot.value / cnt.value / 1e3
            classes[name.value.decode()] = {"launches": cnt.value, "avg_us": avg * 1e6,
                                            "algorithmic_GBps": b.value / avg / 1e9}
    return classes


def run_solves(args):
    """Multigrid-preconditioned CG solves on the initial design's density."""
    import ctypes
    import torch
    import robustoptspline3d_b200 as R
    n = args.size
    em, fa, la, order, parts, coeff = problem(n)
    prec = R.rso.MIXED if args.precision == "mixed" else R.rso.FP64
    g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=prec, smoother=smoother_id(R), omega=OMEGA, cheb_lower=CHEB_LOWER,
                                                    pre=SMOOTH_STEPS, post=SMOOTH_STEPS, poisson_ratio=0.3))
    nc = g.set_spline_partition(parts, parts, parts, order)
    rho = g.projectDensities(g.coeff2density(np.asarray(coeff, np.float32)[:nc]), 8.0)
    g.set_density(rho)
    g.update_stencil()
    tuned = g.autotune() if prec == R.rso.MIXED and not args.no_autotune else None
    if args.fine_rows or args.bottom_level != -3:
        sh = g.launch_shapes()
        g.set_launch_shapes(fine_rows=args.fine_rows or sh["fine_rows"],
                            bottom_level=sh["bottom_level"] if args.bottom_level == -3 else args.bottom_level,
                            row_split=sh["row_split"])
    if args.bottom_kernel >= 0:
        g.set_bottom_kernel(args.bottom_kernel)
    if prec == R.rso.MIXED:
        g.set_krylov_fp32(args.krylov32)
    f = torch.zeros(3 * g.nn, dtype=torch.float64, device="cuda")
    ln = torch.as_tensor(g.load_nodes(), device="cuda").long()
    f[2 * g.nn + ln] = torch.as_tensor(np.random.default_rng(1).standard_normal(len(ln)), device="cuda")
    for _ in range(args.warmup):
        g.solve(f, tol=1e-6, max_iter=500)
    lib = g.lib
    lib.rso_profile_reset(g.h)
    lib.rso_set_profiling(g.h, 1)
    its, ms, worst = 0, 0.0, 0.0
    for _ in range(args.steps):
        _, it, rr, t = g.solve(f, tol=1e-6, max_iter=500)
        its += it
        ms += t
        worst = max(worst, rr)
    lib.rso_set_profiling(g.h, 0)
    classes = kernel_classes(g)
    print(json.dumps({"metric": f"multigrid PCG solve @{n}^3 to rel.resid 1e-6 ({args.precision})",
                      "value": ms / args.steps, "unit": "ms/solve", "higher_is_better": False,
                      "iterations_per_solve": its / args.steps, "ms_per_iteration": ms / its,
                      "max_true_rel_residual": worst, "krylov32_replace_factor": args.krylov32,
                      "levels": g_levels(n), "kernel_classes": classes, "launch_shapes": g.launch_shapes()}), flush=True)
    g.close()


def batch_problem(n, k, seed=2026):
    """16 load cases on an n^3 box (all voxels active, z = 0 nodes clamped):
    load b is a unit total force spread over a seeded 8 x 8-node patch of the
    top face, in a seeded random unit direction.  Density: i.i.d. U[0.2, 1]
    followed by one 3x3x3 mean over the in-box neighbours."""
    from scipy.ndimage import uniform_filter
    rng = np.random.default_rng(seed)
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[0] = 1
    la = np.zeros((n + 1,) * 3, np.uint8)
    la[n] = 1
    rho = rng.uniform(0.2, 1.0, (n, n, n))
    ones = np.ones_like(rho)
    rho = (uniform_filter(rho, 3, mode="constant") / uniform_filter(ones, 3, mode="constant")).astype(np.float32)
    nn = (n + 1) ** 3
    loads = []
    for _ in range(k):
        x0, y0 = rng.integers(0, n + 1 - 8, size=2)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        f = np.zeros(3 * nn)
        ys, xs = np.meshgrid(np.arange(y0, y0 + 8), np.arange(x0, x0 + 8), indexing="ij")
        ids = (xs + (n + 1) * (ys + (n + 1) * n)).ravel()
        for c in range(3):
            f[c * nn + ids] = d[c] / 64.0
        loads.append(f)
    return em, fa, la, rho, np.stack(loads)


def run_batch(args):
    """Config 3a: k load cases solved as one batch (every V-cycle launch carries
    all k systems) against the same systems solved one after another."""
    import torch
    import robustoptspline3d_b200 as R
    n, k = args.size, args.systems
    em, fa, la, rho, F = batch_problem(n, k)
    prec = R.rso.MIXED if args.precision == "mixed" else R.rso.FP64
    g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=prec, smoother=smoother_id(R), omega=OMEGA,
                                                    cheb_lower=CHEB_LOWER, pre=SMOOTH_STEPS, post=SMOOTH_STEPS, poisson_ratio=0.3))
    g.set_density(rho.ravel())
    g.update_stencil()
    if prec == R.rso.MIXED and not args.no_autotune:
        g.autotune()
    Ft = torch.as_tensor(F, device="cuda")
    for _ in range(max(1, args.warmup)):
        g.solve_batch(Ft, tol=1e-6, max_iter=500)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        U, infos = g.solve_batch(Ft, tol=1e-6, max_iter=500)
    torch.cuda.synchronize()
    t_batch = (time.perf_counter() - t0) / args.steps
    t0 = time.perf_counter()
    its = []
    for b in range(k):
        _, it, _, _ = g.solve(Ft[b], tol=1e-6, max_iter=500)
        its.append(it)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    print(json.dumps({"metric": f"{k} load cases @{n}^3 to rel.resid 1e-6 ({args.precision}), batched",
                      "value": k / t_batch, "unit": "solves/s", "higher_is_better": True,
                      "ms_per_batch": t_batch * 1e3, "sequential_solves_per_s": k / t_seq,
                      "batch_vs_sequential": t_seq / t_batch,
                      "iterations": [i for i, _ in infos], "sequential_iterations": its,
                      "data": "synthetic", "config": {"workload": "config 3a (16 top-face patch loads, bottom clamped)",
                                                      "smoother": f"{SMOOTHER} {SMOOTH_STEPS}+{SMOOTH_STEPS}", "levels": g_levels(n)}}),
          flush=True)
    g.close()


def cube_problem(n, seed):
    """Config-0 style cube: all voxels active, x = 0 nodes clamped, a unit total
    -z load spread over the nodes of the x = n face's mid-height line, density
    i.i.d. U[0.2, 1] followed by one 3x3x3 mean over the in-box neighbours."""
    from scipy.ndimage import uniform_filter
    rng = np.random.default_rng(seed)
    em = np.ones((n, n, n), np.uint8)
    fa = np.zeros((n + 1,) * 3, np.uint8)
    fa[:, :, 0] = 1
    la = np.zeros((n + 1,) * 3, np.uint8)
    rho = rng.uniform(0.2, 1.0, (n, n, n))
    rho = (uniform_filter(rho, 3, mode="constant") / uniform_filter(np.ones_like(rho), 3, mode="constant"))
    nn = (n + 1) ** 3
    f = np.zeros(3 * nn)
    ids = n + (n + 1) * (np.arange(n + 1) + (n + 1) * (n // 2))
    f[2 * nn + ids] = -1.0 / (n + 1)
    return em, fa, la, rho.astype(np.float32), f


def run_problems(args):
    """Config 3b: 32 independent cubes of uneven size (edges drawn from
    {32, 48, 64, 96, 128}), one handle and CUDA stream each, solved one after
    another and then concurrently from host threads (ctypes releases the GIL,
    so the problems' kernels overlap on the GPU)."""
    import concurrent.futures
    import torch
    import robustoptspline3d_b200 as R
    rng = np.random.default_rng(2026)
    sizes = rng.choice([32, 48, 64, 96, 128], size=32)
    grids, loads = [], []
    for i, n in enumerate(sizes):
        em, fa, la, rho, f = cube_problem(int(n), 100 + i)
        g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=R.rso.MIXED, smoother=smoother_id(R), omega=OMEGA,
                                                        cheb_lower=CHEB_LOWER, pre=SMOOTH_STEPS, post=SMOOTH_STEPS, poisson_ratio=0.4,
                                                        youngs_modulus=1e6))
        g.set_density(rho.ravel())
        g.update_stencil()
        if not args.no_autotune:
            g.autotune()
        grids.append(g)
        loads.append(torch.as_tensor(f, device="cuda"))

    def solve(i):
        return grids[i].solve(loads[i], tol=1e-6, max_iter=500)[1]

    for i in range(len(grids)):
        solve(i)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = [solve(i) for i in range(len(grids))]
    t_seq = time.perf_counter() - t0
    def concurrent_run():
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(grids)) as ex:
            list(ex.map(solve, range(len(grids))))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            its_c = list(ex.map(solve, range(len(grids))))
            torch.cuda.synchronize()
            return time.perf_counter() - t0, its_c

    t_con, its_c = concurrent_run()
    # Concurrent problems hide one another's latency, so the launch shapes a
    # problem measures alone are not always the best together: the run is
    # repeated with the small levels of every hierarchy (from the first level of
    # at most 6000 nodes down) in the cluster kernel, which needs fewer launches
    # and 8 SMs, and the faster of the two runs is reported.
    for g in grids:
        nl = g.n_levels()
        lb = nl - 1
        while lb - 1 >= 1 and int(np.prod(g.level_dims(lb - 1)[3:6])) <= 6000:
            lb -= 1
        if lb <= nl - 2:
            ch = g.launch_shapes()
            g.set_launch_shapes(ch["fine_rows"], lb, ch["row_split"])
    t_con_b, its_cb = concurrent_run()
    best = min(t_con, t_con_b)
    print(json.dumps({"metric": "32 uneven cubes (edges 32-128) to rel.resid 1e-6 (mixed), concurrent handles",
                      "value": len(grids) / best, "unit": "solves/s", "higher_is_better": True,
                      "sequential_solves_per_s": len(grids) / t_seq, "concurrent_vs_sequential": t_seq / best,
                      "concurrent_tuned_solves_per_s": len(grids) / t_con,
                      "concurrent_bottom_cluster_solves_per_s": len(grids) / t_con_b,
                      "sizes": [int(n) for n in sizes], "iterations": its, "iterations_concurrent": its_c,
                      "iterations_concurrent_bottom_cluster": its_cb,
                      "data": "synthetic", "config": {"workload": "config 3b", "smoother": f"{SMOOTHER} {SMOOTH_STEPS}+{SMOOTH_STEPS}"}}),
          flush=True)
    for g in grids:
        g.close()


def scale_problem(seed=2027, nvoids=200):
    """Mixed precision at scale: a 511 x 256 x 256 voxel box embedded as 512 x 256
    x 256 with the last x element plane inactive, with `nvoids` spherical voids
    (radius ~ U[4, 20], centres ~ U(box), seeded), nodes of x = 0 clamped, load
    set = the node plane x = 511 with the force along +x (constrained-direction
    worst case)."""
    ex, ey, ez = 512, 256, 256
    rng = np.random.default_rng(seed)
    em = np.ones((ez, ey, ex), np.uint8)
    em[:, :, ex - 1] = 0
    for _ in range(nvoids):
        r = rng.uniform(4.0, 20.0)
        cx, cy, cz = rng.uniform(0.0, 511.0), rng.uniform(0.0, ey), rng.uniform(0.0, ez)
        lo = [max(int(np.floor(c - r - 1)), 0) for c in (cz, cy, cx)]
        hi = [min(int(np.ceil(c + r + 1)), m) for c, m in zip((cz, cy, cx), (ez, ey, ex))]
        z, y, x = np.ogrid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        inside = (x + 0.5 - cx) ** 2 + (y + 0.5 - cy) ** 2 + (z + 0.5 - cz) ** 2 <= r * r
        em[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]][inside] = 0
    fa = np.zeros((ez + 1, ey + 1, ex + 1), np.uint8)
    fa[:, :, 0] = 1
    la = np.zeros((ez + 1, ey + 1, ex + 1), np.uint8)
    la[:, :, ex - 1] = 1
    normals = np.zeros(((ez + 1) * (ey + 1) * (ex + 1), 3))
    normals[:, 0] = 1.0
    return em, fa, la, normals


def torus_mesh(R=2.0, r=0.7, nu=512, nv=256):
    """Closed torus surface of 2 nu nv triangles, outward winding."""
    a = 2 * np.pi * np.arange(nu) / nu
    b = 2 * np.pi * np.arange(nv) / nv
    A, Bm = np.meshgrid(a, b, indexing="ij")
    v = np.stack([(R + r * np.cos(Bm)) * np.cos(A), (R + r * np.cos(Bm)) * np.sin(A), r * np.sin(Bm)], axis=-1)
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    p, q = i * nv + j, ((i + 1) % nu) * nv + j
    p1, q1 = i * nv + (j + 1) % nv, ((i + 1) % nu) * nv + (j + 1) % nv
    f = np.concatenate([np.stack([p, q, q1], -1).reshape(-1, 3), np.stack([p, q1, p1], -1).reshape(-1, 3)])
    return v.reshape(-1, 3).astype(np.float32), f.astype(np.int32)


def run_mesh(args):
    """The mesh -> HierarchyGrid input chain at 256^3: a 262,144-triangle torus
    voxelised at preferred resolution 200 (R = 256), shell elements of width 3
    voxels, fixed and load node masks from two half-spaces on the 257^3 nodes,
    outward normals and a constant load field at the load nodes.  Each stage is
    timed through its C-ABI entry point with host buffers (copies included),
    the median of --steps runs after --warmup; the CPU column is the numpy
    restatement on a bounded sample of faces / points scaled to the full
    count (its cost is linear in faces and points)."""
    import robustoptspline3d_b200 as R
    from robustoptspline3d_b200 import boundary as B
    from robustoptspline3d_b200.voxelize import voxelize
    v, f = torus_mesh()
    fix = [B.halfspace(0, 0, -1, -0.5, closed=True)]
    load = [B.halfspace(0, 0, 1, -0.5)]
    force = [B.Field(load[0], ("constant", 1.0), ("constant", (0.0, 0.0, -1.0)))]
    stages = {}

    def timed(name, fn):
        for _ in range(max(args.warmup, 1)):
            out = fn()
        ts = []
        for _ in range(max(args.steps, 1)):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        stages[name] = float(np.median(ts)) * 1e3
        return out

    l0 = R.rso.load_library().rso_launch_count()
    solid, Rg, bx = timed("voxelize", lambda: voxelize(v, f, 200))
    origin, h = B.node_grid(bx, Rg)
    dims = (Rg + 1,) * 3
    shell = timed("shell_w3", lambda: B.shell_elements(v, f, bx, Rg, 3.0, solid))
    fixed = timed("region_masks", lambda: (B.region_mask(fix, origin, h, dims), B.region_mask(load, origin, h, dims)))
    fm, lm = fixed
    surf = B.surface_nodes(solid)
    ln = np.flatnonzero(surf & (lm > 0) & (fm == 0))
    pts = origin[None, :] + np.stack([ln % (Rg + 1), (ln // (Rg + 1)) % (Rg + 1), ln // (Rg + 1) ** 2], 1) * h
    timed("normals", lambda: B.mesh_normals(v, f, pts))
    timed("load_field", lambda: B.region_field(force, pts))
    launches = R.rso.load_library().rso_launch_count() - l0
    total = sum(stages.values())
    out = {"metric": "mesh input chain @256^3 (voxelise, shell, region masks, normals, load field)",
           "value": 1e3 / total, "unit": "chains/s", "higher_is_better": True, "ms_per_chain": total,
           "stages_ms": stages, "gpu_launches": int(launches),
           "sizes": {"triangles": int(len(f)), "resolution": int(Rg), "solid": int(solid.sum()),
                     "shell": int(shell.sum()), "load_nodes": int(len(ln)), "fixed_area_nodes": int(fm.sum())},
           "data": "synthetic torus (R 2, r 0.7)",
           "config": {"workload": "torus 262,144 triangles, preferred 200 -> 256^3, shell width 3",
                      "timing": "host buffers in and out through the C ABI (copies and scratch included)"}}
    if not args.no_cpu_baseline:
        from oracle import boundary as OB
        from oracle import voxel as OV
        cpu = {}
        sel = np.random.default_rng(1).choice(len(f), 400, replace=False)
        t0 = time.perf_counter()
        OB.shell_elements(v, f[sel], bx, Rg, 3.0, solid)
        cpu["shell_w3"] = (time.perf_counter() - t0) * 1e3 * len(f) / len(sel)
        t0 = time.perf_counter()
        OB.region_mask([(r.kind, r.p, r.closed, r.complement) for r in fix + load], origin, h, dims)
        cpu["region_masks"] = (time.perf_counter() - t0) * 1e3
        pk = pts[:64]
        fk = f[:4096]
        t0 = time.perf_counter()
        OB.mesh_normals(v, fk, pk)
        cpu["normals"] = (time.perf_counter() - t0) * 1e3 * (len(f) / len(fk)) * (len(pts) / len(pk))
        vs = f[sel]
        t0 = time.perf_counter()
        OV.voxelize(v, vs, 200)
        cpu["voxelize"] = (time.perf_counter() - t0) * 1e3 * len(f) / len(vs)
        out["cpu_baseline"] = {"value": 1e3 / sum(cpu.values()), "unit": "chains/s", "cores": 1, "kind": "port",
                               "stages_ms": cpu,
                               "sample": "400 faces (shell, voxelise), 64 points x 4096 faces (normals), full "
                                         "region masks; scaled linearly to the full counts",
                               "note": "the port's normals scan every face for every point; the reference "
                                       "queries a CGAL AABB tree, so that stage of the port is no measure of "
                                       "the reference"}
    print(json.dumps(out), flush=True)


def run_surface(args):
    """Surface-point self-support on the seeded 256^3 design (32^3 tricubic
    coefficients): the rho = 0.5 crossings of the 66^3 background grid thinned
    to 200,000 points (rso_surface_points), then the overhang constraint
    (mode 4, 135 degrees) with its coefficient gradient at those points
    (rso_surface_selfsupport).  Both are synchronous C-ABI calls with device
    coefficients; the median host wall time of --steps calls after --warmup.
    The CPU column runs the oracle's restatement of the same two steps once,
    at the full size, on one core."""
    import torch
    import robustoptspline3d_b200 as R
    n = args.size
    em, fa, la, order, parts, coeff = problem(n)
    g = R.HierarchyGrid(em, fa, la, None, R.Config())
    g.set_spline_partition(parts, parts, parts, order)
    c = torch.as_tensor(coeff, dtype=torch.float32, device="cuda")
    mc, npts = 64, 200000
    lib = g.lib

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            out = fn()
        ts = []
        for _ in range(max(args.steps, 1)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)) * 1e3, out

    l0 = lib.rso_launch_count()
    ms_pts, (_, counts) = timed(lambda: g.generate_spline_surface_nodes(c, mc_res=mc, n_points=npts))
    l1 = lib.rso_launch_count()
    ms_ss, res = timed(lambda: g.deal_surface_points(c, 8.0, 4))
    l2 = lib.rso_launch_count()
    calls = max(args.warmup, 1) + max(args.steps, 1)
    out = {"metric": "surface-point self-support @256^3 (sampling + constraint + gradient)",
           "value": 1e3 / (ms_pts + ms_ss), "unit": "evaluations/s", "higher_is_better": True,
           "ms_sampling": ms_pts, "ms_constraint": ms_ss, "counts": counts,
           "constraint": {"value": res[0], "count": res[3], "probe_sum": res[4]},
           "gpu_launches_per_call": {"sampling": (l1 - l0) // calls, "constraint": (l2 - l1) // calls},
           "data": "synthetic (seeded design of the design-iteration bench)",
           "config": {"workload": f"{n}^3 box, order {order}, {parts + order}^3 coefficients, background {mc}^3 "
                                  f"(+2), {npts} points, mode 4 (overhang sigmoid), beta 8",
                      "timing": "host wall clock around synchronous C-ABI calls, device coefficients"}}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        o = O.Problem(em, fa, la, n_levels=1)   # the spline and the mask only; no hierarchy
        o.spline_setup(order, [parts] * 3)
        cd = np.asarray(coeff, np.float32).astype(np.float64)
        t0 = time.perf_counter()
        pts, _ = o.surface_points(cd, mc=mc, n_points=npts)
        t1 = time.perf_counter()
        o.surface_selfsupport(cd, pts, 8.0, 4)
        t2 = time.perf_counter()
        out["cpu_baseline"] = {"value": 1.0 / (t2 - t0), "unit": "evaluations/s", "cores": 1, "kind": "port",
                               "ms_sampling": (t1 - t0) * 1e3, "ms_constraint": (t2 - t1) * 1e3,
                               "sample": "one full evaluation (same sizes)"}
    g.close()
    print(json.dumps(out), flush=True)


def run_scale(args):
    """One worst-case design iteration on the 512 x 256 x 256 voids box (the
    FP32-operator-at-scale configuration), mixed and plain FP64; the FP64 path
    solves to relative residual 1e-10 and serves as the reference the mixed
    path's worst-case eigenvalue, compliance and coefficient gradients are
    compared against (the CPU oracle is checked against the GPU at small sizes
    in the tests)."""
    import torch
    import robustoptspline3d_b200 as R
    em, fa, la, normals = scale_problem()
    order = 4
    parts = (60, 28, 28)
    rng = np.random.default_rng(2026)
    res = {}
    for prec, tol in ((R.rso.MIXED, 1e-6), (R.rso.FP64, 1e-10)):
        t0 = time.perf_counter()
        g = R.HierarchyGrid(em, fa, la, normals, R.Config(precision=prec, smoother=smoother_id(R), omega=OMEGA,
                                                          cheb_lower=CHEB_LOWER, pre=SMOOTH_STEPS, post=SMOOTH_STEPS, poisson_ratio=0.3,
                                                          mode=R.rso.WITH_SUPPORT_CF))
        nc = g.set_spline_partition(*parts, order)
        coeff = np.clip(np.random.default_rng(2026).normal(0.5, 0.15, nc), 0.0, 1.0)
        setup_s = time.perf_counter() - t0
        prm = R.IterParams(lanczos_steps=20, solve_tol=tol, ss_mode=4, constrain_direction=1, filter_mode=1)
        c0 = torch.as_tensor(coeff, dtype=torch.float64, device="cuda")
        vals, gl, gv, gs = g.design_gradient(c0, prm)
        mma = R.MMA(nc, 2, 0.0, 1.0)
        times, info = [], None
        for _ in range(1 + max(1, min(args.steps, 2))):
            mma.set_x(c0)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            info = g.design_iteration(mma, prm)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t1)
        x_new = mma.get()[0]
        # one more iteration with per-class CUDA-event timing (not among the timed ones)
        g.lib.rso_profile_reset(g.h)
        g.lib.rso_set_profiling(g.h, 1)
        mma.set_x(c0)
        g.design_iteration(mma, prm)
        g.lib.rso_set_profiling(g.h, 0)
        res[prec] = dict(vals=vals, gl=gl.cpu().numpy(), x=x_new, s=min(times[1:]), info=info, setup_s=setup_s,
                         levels=[g.level_dims(i)[:3].tolist() for i in range(g.n_levels())],
                         classes=kernel_classes(g), nodes=int(np.prod(g.level_dims(0)[3:6])))
        mma.close()
        g.close()
        del g, gl, gv, gs, c0
        torch.cuda.empty_cache()
    m, d = res[R.rso.MIXED], res[R.rso.FP64]
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))
    out = {"metric": "worst-case design iteration @512x256x256 with 200 voids (mixed vs FP64)",
           "value": 1.0 / m["s"], "unit": "iter/s", "higher_is_better": True,
           "fp64_iters_per_s": 1.0 / d["s"], "mixed_vs_fp64": d["s"] / m["s"],
           "active_elements": int(em.sum()), "levels": m["levels"],
           "pcg_iterations": {"mixed": m["info"]["solve_iterations"], "fp64": d["info"]["solve_iterations"]},
           "errors_vs_fp64": {"lambda_max": abs(m["vals"]["lambda"] - d["vals"]["lambda"]) / abs(d["vals"]["lambda"]),
                              "compliance_worst": abs(m["info"]["c_worst"] - d["info"]["c_worst"]) / abs(d["info"]["c_worst"]),
                              "dlambda_dcoeff": rel(m["gl"], d["gl"]),
                              "coefficients_after_mma": rel(m["x"], d["x"])},
           "setup_s": {"mixed": m["setup_s"], "fp64": d["setup_s"]},
           "kernel_classes": {"mixed": m["classes"], "fp64": d["classes"]},
           "fine_ns_per_node": {k: v["avg_us"] * 1e3 / m["nodes"] for k, v in m["classes"].items()
                                if k.startswith("fine_")},
           "config": {"workload": "511x256x256 voxels (embedded 512x256x256), 200 spherical voids r~U[4,20]",
                      "load": "x=511 node plane, force along +x (constrained direction)", "support": "x=0 nodes",
                      "spline": f"order {order}, partition {parts}", "solve_tol": {"mixed": 1e-6, "fp64": 1e-10},
                      "smoother": f"{SMOOTHER} {SMOOTH_STEPS}+{SMOOTH_STEPS} on [{CHEB_LOWER}, 1] x lambda_max",
                      "smoother_state": "FP32 (BF16/FP16 state not built)", "filter": "none (exact gradients)"},
           "data": "synthetic"}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--fine-rows", type=int, default=0,
                    help="--mode solve: thread rows of the packed fine kernel's CTA (2, 4 or 8; 0: as tuned)")
    ap.add_argument("--bottom-level", type=int, default=-3,
                    help="--mode solve: first level of the bottom kernel (-1 none, -2 built-in rule; default as tuned)")
    ap.add_argument("--bottom-kernel", type=int, default=-1,
                    help="--mode solve: bottom kernel kind (1 persistent grid-wide, 0 cluster; default as tuned)")
    ap.add_argument("--ref-size", type=int, default=24)
    ap.add_argument("--ref-sizes", default="24,32,48",
                    help="sample sizes of the CPU baseline leg (the largest is scaled to 256^3)")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--krylov32", type=float, default=1e-2,
                    help="mixed PCG with the FP32 Krylov recurrence, true-residual replacement factor (0: FP64 recurrence)")
    ap.add_argument("--cheb-lower", type=float, default=None,
                    help="lower end of the Chebyshev smoother's interval as a fraction of lambda_max")
    ap.add_argument("--smooth-steps", type=int, default=2,
                    help="Chebyshev smoothing steps before and after each coarse correction")
    ap.add_argument("--mode", default="design", choices=["design", "solve", "batch", "problems", "scale", "mesh",
                                                          "surface"])
    ap.add_argument("--systems", type=int, default=16)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    args = ap.parse_args()
    global CHEB_LOWER, SMOOTH_STEPS
    if args.cheb_lower is not None:
        CHEB_LOWER = args.cheb_lower
    SMOOTH_STEPS = args.smooth_steps
    if args.mode == "solve":
        run_solves(args)
        return
    if args.mode == "batch":
        run_batch(args)
        return
    if args.mode == "problems":
        run_problems(args)
        return
    if args.mode == "scale":
        run_scale(args)
        return
    if args.mode == "mesh":
        run_mesh(args)
        return
    if args.mode == "surface":
        run_surface(args)
        return
    if args.impl == "reference":
        # host-only arm: rank 0 times the CPU path, other ranks exit at once
        # (no process group is needed for that)
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    import robustoptspline3d_b200 as R

    n = args.size
    em, fa, la, order, parts, coeff = problem(n)
    prm = R.IterParams(lanczos_steps=20, solve_tol=1e-6, ss_mode=4)

    def make(precision):
        g = R.HierarchyGrid(em, fa, la, None, R.Config(precision=precision, smoother=smoother_id(R), omega=OMEGA, cheb_lower=CHEB_LOWER,
                                                        pre=SMOOTH_STEPS, post=SMOOTH_STEPS, poisson_ratio=0.3))
        nc = g.set_spline_partition(parts, parts, parts, order)
        if precision == R.rso.MIXED:
            g.set_krylov_fp32(args.krylov32)
        mma = R.MMA(nc, 2, 0.0, 1.0)
        mma.set_x(coeff)
        return g, mma

    g, mma = make(R.rso.MIXED)
    lib = g.lib
    c0 = torch.as_tensor(coeff, dtype=torch.float64, device="cuda")

    def step(gg, mm):
        # every step is one full design iteration from the seeded initial design
        mm.set_x(c0)
        return gg.design_iteration(mm, prm)

    # warm-up (device path); the last warm-up step times every kernel class
    # to find the dominant one, and the timed steps record only that class
    import ctypes
    kname = ctypes.create_string_buffer(64)
    cnt = ctypes.c_longlong(0)
    tot = ctypes.c_double(0)
    bytes_per = ctypes.c_double(0)
    flops_per = ctypes.c_double(0)
    tuned = None
    for w in range(args.warmup):
        if w == args.warmup - 1:
            lib.rso_profile_reset(g.h)
            lib.rso_set_profiling(g.h, 1)
        step(g, mma)
        if w == 0 and not args.no_autotune:
            # launch shapes measured on this hierarchy once its operators exist
            tuned = g.autotune()
    top_cls, top_ms, stencil_cls = 0, -1.0, None
    for cls in range(16):
        if lib.rso_profile_class(g.h, cls, kname, 64, ctypes.byref(cnt), ctypes.byref(tot), ctypes.byref(bytes_per),
                                 ctypes.byref(flops_per)) != 0:
            break
        if tot.value > top_ms:
            top_cls, top_ms = cls, tot.value
        if kname.value.decode() == "coarse_stencil_fp32_streamed" and cnt.value > 0:
            stencil_cls = cls
    lib.rso_set_profiling(g.h, 0)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lib.rso_profile_reset(g.h)
    # the dominant kernel and the coarse stencil kernel are timed in the timed steps
    lib.rso_set_profiling_classes(g.h, (1 << top_cls) | ((1 << stencil_cls) if stencil_cls is not None else 0))
    launches0 = lib.rso_launch_count()
    barrier_max(world, 0.0)
    infos = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev0.record()
        for _ in range(args.steps):
            infos.append(step(g, mma))
        ev1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    launches = lib.rso_launch_count() - launches0
    lib.rso_set_profiling(g.h, 0)
    ms_dev = ev0.elapsed_time(ev1)
    ms = barrier_max(world, max(ms_dev, wall * 1e3))
    value = world * args.steps / (ms / 1e3)
    # dominant-kernel roofline from the live event timings of the timed steps
    stencil = None
    if stencil_cls is not None:
        lib.rso_profile_class(g.h, stencil_cls, kname, 64, ctypes.byref(cnt), ctypes.byref(tot), ctypes.byref(bytes_per),
                              ctypes.byref(flops_per))
        s_ms = tot.value / max(cnt.value, 1)
        stencil = {"kernel": kname.value.decode(), "launches": cnt.value, "avg_ms": s_ms,
                   "algorithmic_bytes_per_launch": bytes_per.value,
                   "achieved": bytes_per.value / (s_ms / 1e3) / 1e9 if s_ms > 0 else 0.0}
    lib.rso_profile_top(g.h, kname, 64, ctypes.byref(cnt), ctypes.byref(tot), ctypes.byref(bytes_per),
                        ctypes.byref(flops_per))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    avg_ms = tot.value / max(cnt.value, 1)
    achieved = bytes_per.value / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    # DRAM bytes per fine node of one launch, measured by ncu
    # (dram__bytes_read.sum + dram__bytes_write.sum) on a 193^3 case whose
    # working set exceeds L2, where traffic grows with the node count
    traffic_per_node = {"fine_jacobi_fp32": 284.1e6 / 193 ** 3}
    kn = kname.value.decode()
    traffic = traffic_per_node[kn] * (n + 1) ** 3 if kn in traffic_per_node else None
    roofline = {"kernel": kn, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "launches": cnt.value, "avg_ms": avg_ms,
                "algorithmic_bytes_per_launch": bytes_per.value,
                "fp_flops_per_launch": flops_per.value,
                "fp_tflops": flops_per.value / (avg_ms / 1e3) / 1e12 if avg_ms > 0 else 0.0,
                "peak_source": "measured" if peaks else "fallback"}
    # end-to-end through the host-buffer C ABI call: coefficients in from
    # pinned host memory, updated coefficients back to pinned host memory
    cin = torch.as_tensor(np.ascontiguousarray(coeff, np.float64)).pin_memory()
    cout = torch.empty_like(cin).pin_memory()
    host_iteration(g, mma, cin, cout, prm)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host_iteration(g, mma, cin, cout, prm)
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_s = barrier_max(world, e2e_s)
    e2e = {"value": world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": cin.numel() * 8,
           "d2h_bytes_per_step": cout.numel() * 8}
    g.close()
    mma.close()
    # plain FP64 GPU path for the mixed-vs-FP64 comparison
    fp64 = fp64_tight = None
    if args.fp64_steps > 0:
        g64, mma64 = make(R.rso.FP64)
        step(g64, mma64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.fp64_steps):
            step(g64, mma64)
        torch.cuda.synchronize()
        fp64 = barrier_max(world, (time.perf_counter() - t0) / args.fp64_steps)
        # the FP64 path at the tolerance the FP64 reference method is run to
        # (relative residual 1e-10), and the mixed result's distance from it
        prm10 = R.IterParams(lanczos_steps=20, solve_tol=1e-10, ss_mode=4)
        mma64.set_x(c0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info10 = g64.design_iteration(mma64, prm10)
        torch.cuda.synchronize()
        fp64_tight = {"iters_per_s": world / barrier_max(world, time.perf_counter() - t0), "solve_tol": 1e-10,
                      "solve_iterations": info10["solve_iterations"],
                      "mixed_lambda_rel_err": abs(infos[-1]["lam"] - info10["lam"]) / abs(info10["lam"]),
                      "mixed_c_worst_rel_err": abs(infos[-1]["c_worst"] - info10["c_worst"]) / abs(info10["c_worst"])}
        g64.close()
        mma64.close()
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        sizes = [int(v) for v in args.ref_sizes.split(",")]
        samples = cpu_samples(O, sizes, coeff)
        big = samples[-1]
        # scaled from the largest sample by the element count and by the PCG
        # iterations of this run's own 256^3 iteration (the oracle's count
        # grows slowly with size; the samples show by how much)
        its256 = infos[-1]["solve_iterations"]
        per = big["s"] * (256.0 / big["n"]) ** 3 * max(1.0, its256 / big["pcg_iterations"])
        cpu = {"value": 1.0 / per, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": (f"one FP64 oracle design iteration at each of {', '.join(f'{v}^3' for v in sizes)}; "
                          f"the {big['n']}^3 one ({big['s']:.2f} s, {big['pcg_iterations']} PCG iterations) scaled by "
                          f"(256/{big['n']})^3 and by max(1, {its256} / {big['pcg_iterations']}) iterations"),
               "samples": samples}
    clocks = clk.summary()
    # the fine operator's binding roof is the FP32 CUDA-core pipe, not HBM:
    # algorithmic flops per second against 148 SMs x 128 lanes x 2 flop per
    # cycle at the SM clock sampled during the timed region
    mhz = clocks.get("sm_mhz") or 1965.0
    simt_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    if stencil is not None:
        # the coarse stencil operator (HBM-bound), the kernel the stencil-bandwidth target is about
        stencil.update({"bound": "hbm", "peak": hbm, "unit": "GB/s", "frac": stencil["achieved"] / hbm,
                        "peak_source": roofline["peak_source"]})
        roofline["coarse_stencil"] = stencil
    roofline["compute"] = {"bound": "fp32_simt", "achieved_tflops": roofline["fp_tflops"], "peak_tflops": simt_peak,
                           "frac": roofline["fp_tflops"] / simt_peak,
                           "note": "algorithmic 1260 flop per node (576 FMA of K0 + smoother); the kernel executes "
                                   "about 200 additions and multiplications per node in the sum/difference basis"}
    if rank == 0:
        last = infos[-1]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 V-cycle and CG recurrence + f64 iterate, residual replacement, Lanczos, MMA", "data": "synthetic",
                "config": {"workload": f"{n}^3 worst-case spline TO iteration (config 4 shape)", "elements": n ** 3,
                           "spline": "order 4, 32^3 coefficients", "lanczos_steps": 20, "solve_tol": 1e-6,
                           "smoother": f"{SMOOTHER} {SMOOTH_STEPS}+{SMOOTH_STEPS} on [{CHEB_LOWER}, 1] x lambda_max",
                           "preconditioner": "one V-cycle per CG iteration",
                           "krylov": (f"FP32 recurrence, true FP64 residual replacing it every {args.krylov32:g} "
                                      "reduction and at the end") if args.krylov32 > 0 else "FP64 recurrence",
                           "levels": g_levels(n), "parallelism": f"replicas x{world}",
                           "l2_flush": "inputs larger than L2",
                           "step": "one design iteration from the seeded initial design"},
                "fp64_iters_per_s": (1.0 / fp64) if fp64 else None,
                "mixed_vs_fp64": (fp64 / (ms / 1e3 / args.steps)) if fp64 else None,
                "fp64_rel_resid_1e-10": dict(fp64_tight, mixed_vs_fp64=value / fp64_tight["iters_per_s"]) if fp64_tight else None,
                "last_iteration": {k: last[k] for k in ("c_worst", "lam", "volume", "ss_value", "solve_iterations",
                                                        "ms_operators", "ms_worst", "ms_selfsupport", "ms_adjoint",
                                                        "ms_mma")},
                "launch_shapes": tuned,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def g_levels(n):
    lv = [n]
    m = n
    while (m ** 3) > 400:
        m = (m + 1) // 2
        lv.append(m)
    return [lv[0]] + lv[2:]


def host_iteration(g, mma, cin, cout, prm):
    return g.design_iteration_host(mma, cin, prm, coeff_out=cout, density=False)


if __name__ == "__main__":
    main()
