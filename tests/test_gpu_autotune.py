"""Launch-shape autotuner (rso_autotune / rso_set_launch_shapes) through the C ABI.
The alternatives compute the same arithmetic in other launch shapes, so every
forced combination of fine tile height, coarse kernel variant, bottom-kernel
level and bottom-kernel kind must solve to the same answer: the solves run to relative residual 1e-10
and must agree to 1e-8 relative with iteration counts within one."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def make(prob):
    from robustoptspline3d_b200 import Config, HierarchyGrid
    g = HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],
                      Config(precision=1, smoother=2, poisson_ratio=0.4, cheb_lower=0.1))
    g.set_density(prob["rho"].astype(np.float32).ravel())
    g.update_stencil()
    return g


def rhs(g, seed=31):
    rng = np.random.default_rng(seed)
    f = np.zeros(3 * g.nn)
    ln = g.load_nodes()
    for c in range(3):
        f[c * g.nn + ln] = rng.standard_normal(len(ln))
    return f


@pytest.mark.parametrize("gen", [lambda: P.cantilever(64, 32, 32), lambda: P.ellipsoid(40, 24, 24)])
def test_autotune_choices_solve_alike(cuda, gen):
    prob = gen()
    g = make(prob)
    nl = g.n_levels()
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    u_ref, it_ref, _, _ = g.solve(f, tol=1e-10, max_iter=300)
    u_ref = u_ref.cpu().numpy()
    ch = g.autotune()
    assert ch["fine_rows"] in (2, 4, 8)
    assert ch["fine_zchunk"] in (4, 8, 16, 32)
    assert ch["bottom_level"] == -1 or 1 <= ch["bottom_level"] <= nl - 2
    assert len(ch["row_split"]) == nl and all(r in (-1, 0, 1, 2) for r in ch["row_split"])
    u, it, _, _ = g.solve(f, tol=1e-10, max_iter=300)
    assert abs(it - it_ref) <= 1 and rel(u.cpu().numpy(), u_ref) < 1e-8
    assert ch["bottom_kernel"] in (0, 1)
    for rows in (2, 4):
        for bottom in [-1] + list(range(1, nl - 1)):
            for kind in ((1, 0) if bottom > 0 else (1,)):
                g.set_bottom_kernel(kind)
                for split in (0, 1, 2):
                    g.set_launch_shapes(rows, bottom, [-1] + [split] * (nl - 1))
                    u, it, rr, _ = g.solve(f, tol=1e-10, max_iter=300)
                    assert rr < 1e-10
                    assert abs(it - it_ref) <= 1, (rows, bottom, kind, split)
                    assert rel(u.cpu().numpy(), u_ref) < 1e-8, (rows, bottom, kind, split)
    g.close()


def test_bottom_kernels_agree(cuda):
    """The persistent grid-wide bottom kernel and the cluster kernel run the same
    phases (their sweeps in other launch shapes): V-cycle-preconditioned solves
    from every first level agree with per-level launches to 1e-8, repeated
    solves replay captured V-cycles, and an unknown kind is refused."""
    from robustoptspline3d_b200 import RSOError
    g = make(P.ellipsoid(48, 32, 32))
    nl = g.n_levels()
    f = cuda.tensor(rhs(g, 7), dtype=cuda.float64, device="cuda")
    g.set_launch_shapes(4, -1)
    u_ref, it_ref, _, _ = g.solve(f, tol=1e-10, max_iter=300)
    u_ref = u_ref.cpu().numpy()
    for kind in (1, 0):
        g.set_bottom_kernel(kind)
        assert g.bottom_kernel() == kind
        for bottom in range(1, nl - 1):
            g.set_launch_shapes(4, bottom)
            assert g.launch_shapes()["bottom_kernel"] == kind
            for _ in range(3):  # captured on the second occurrence, replayed on the third
                u, it, rr, _ = g.solve(f, tol=1e-10, max_iter=300)
                assert rr < 1e-10 and abs(it - it_ref) <= 1, (kind, bottom, it, it_ref)
                assert rel(u.cpu().numpy(), u_ref) < 1e-8, (kind, bottom)
    with pytest.raises(RSOError):
        g.set_bottom_kernel(2)
    g.close()


def test_launch_shapes_rejected(cuda):
    from robustoptspline3d_b200 import RSOError
    g = make(P.cantilever(32, 16, 16))
    with pytest.raises(RSOError):
        g.set_launch_shapes(3)
    with pytest.raises(RSOError):
        g.set_launch_shapes(4, bottom_level=g.n_levels())
    g.close()


@pytest.mark.parametrize("rows", [2, 4, 8])
def test_fine_zchunk_sweeps_identical(cuda, rows):
    """The z chunk only cuts the march into pieces that re-read the plane below
    them: residual, K u and Jacobi / Chebyshev sweeps are bit-identical for
    chunks of 4, 8, 16 and 32 node planes (with 41 planes the last chunk is
    short), and PCG solves agree to 1e-8 with iteration counts within one
    (the p.q partial sums are grouped by chunk)."""
    g = make(P.cantilever(40, 24, 40))
    g.set_launch_shapes(fine_rows=rows)
    rng = np.random.default_rng(7)
    u = cuda.tensor(rng.standard_normal(3 * g.nn), dtype=cuda.float64, device="cuda")
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    ref = None
    for zc in (32, 16, 8, 4):
        g.set_fine_zchunk(zc)
        assert g.fine_zchunk() == zc
        out = [g.fine_sweep_fp32(0, u, f).cpu().numpy(), g.fine_sweep_fp32(1, u).cpu().numpy(),
               g.fine_sweep_fp32(2, u, f, uprev=u, omega=0.7, c1=0.3).cpu().numpy()]
        x, it, rr, _ = g.solve(f, tol=1e-10, max_iter=300)
        if ref is None:
            ref = (out, x.cpu().numpy(), it)
            continue
        for a, b in zip(out, ref[0]):
            assert np.array_equal(a, b), zc
        assert abs(it - ref[2]) <= 1 and rel(x.cpu().numpy(), ref[1]) < 1e-8
    g.set_fine_zchunk(0)
    assert g.fine_zchunk() in (4, 8, 16, 32)
    g.close()


def test_coarse_variants_sweep_alike(cuda):
    """The three coarse kernels (one thread per node, per (node, row), nine per
    node) compute the same residual and Jacobi / Chebyshev step on every
    coarse level: equal to FP32 rounding of the stencil sums."""
    g = make(P.cantilever(64, 32, 32))
    nl = g.n_levels()
    rng = np.random.default_rng(3)
    for li in range(1, nl - 1):
        nn = int(np.prod(g.level_dims(li)[3:6]))
        u = cuda.tensor(rng.standard_normal(3 * nn), dtype=cuda.float64, device="cuda")
        f = cuda.tensor(rng.standard_normal(3 * nn), dtype=cuda.float64, device="cuda")
        outs = []
        for v in (0, 1, 2):
            g.set_launch_shapes(4, -1, [-1] + [v] * (nl - 1))
            outs.append((g.coarse_sweep_fp32(li, 0, u, f).cpu().numpy(),
                         g.coarse_sweep_fp32(li, 2, u, f, uprev=u, omega=0.6, c1=0.2).cpu().numpy()))
        for a, b in outs[1:]:
            assert rel(a, outs[0][0]) < 1e-5 and rel(b, outs[0][1]) < 1e-5, li
    g.close()


def test_grid_barrier_wait_gives_up(cuda):
    """The persistent bottom kernel's barrier waits are bounded: with an
    arrival target one above the grid no barrier completes, every wait gives up
    after the limit and the launch returns (no fault, no hang); barriers that
    complete report nothing; the handle then solves with the persistent kernel
    as before."""
    import time
    g = make(P.cantilever(48, 24, 24))
    f = cuda.tensor(rhs(g), dtype=cuda.float64, device="cuda")
    g.set_bottom_kernel(1)
    g.set_launch_shapes(4, 1)
    u_ref, it_ref, _, _ = g.solve(f, tol=1e-10, max_iter=300)
    assert g.grid_barrier_selftest(short_by=0, limit_ms=50.0) == 0
    t0 = time.perf_counter()
    assert g.grid_barrier_selftest(short_by=1, limit_ms=5.0) == 1
    assert time.perf_counter() - t0 < 5.0
    assert g.grid_barrier_selftest(short_by=0, limit_ms=50.0) == 0
    u, it, rr, _ = g.solve(f, tol=1e-10, max_iter=300)
    assert rr < 1e-10 and it == it_ref
    assert np.array_equal(u.cpu().numpy(), u_ref.cpu().numpy())
    g.close()
