"""CPU tests: the FP64 oracle against the known-answer checks the reference
carries (it ships no golden vectors) and against independent scipy
assemblies.  No GPU needed."""
import numpy as np
import pytest
import scipy.optimize as so
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import problems as P


def rigid_modes(xyz):
    """6 rigid motions at the given node coordinates (templateMatrix.cpp:105-123)."""
    n = len(xyz)
    R = np.zeros((3 * n, 6))
    for a, p in enumerate(xyz):
        R[3 * a:3 * a + 3, :3] = np.eye(3)
        R[3 * a:3 * a + 3, 3:] = [[0, -p[2], p[1]], [p[2], 0, -p[0]], [-p[1], p[0], 0]]
    return R


def test_k0_rigid_null_space(oracle):
    for E, nu in [(1e6, 0.3), (1e6, 0.4), (2.5, 0.1)]:
        K = oracle.k0(E, nu)
        assert np.allclose(K, K.T, rtol=0, atol=1e-12 * abs(K).max())
        xyz = [(a & 1, (a >> 1) & 1, a >> 2) for a in range(8)]
        assert abs(K @ rigid_modes(xyz)).max() < 1e-10 * abs(K).max()
        w = np.linalg.eigvalsh(K)
        assert np.sum(w > 1e-8 * w.max()) == 18 and w.min() > -1e-8 * w.max()


def test_k0_matches_library(oracle):
    """The library's host-side element matrix equals the oracle's (no GPU call)."""
    from robustoptspline3d_b200 import element_matrix
    for nu in (0.3, 0.4):
        assert np.array_equal(element_matrix(1e6, nu), oracle.k0(1e6, nu))


def assemble(o, prob, K0):
    """scipy assembly of K(rho) with the reference's support treatment (applyK_OTFA_kernel)."""
    ex, ey, ez = o.ex, o.ey, o.ez
    nx, ny = ex + 1, ey + 1
    nn = o.nn
    rows, cols, vals = [], [], []
    em = prob["emask"].ravel()
    rho = o.rho
    for z in range(ez):
        for y in range(ey):
            for x in range(ex):
                e = x + ex * (y + ey * z)
                if not em[e]:
                    continue
                nodes = [(x + (a & 1)) + nx * ((y + ((a >> 1) & 1)) + ny * (z + (a >> 2))) for a in range(8)]
                dofs = np.array([c * nn + n for n in nodes for c in range(3)])
                rows.append(np.repeat(dofs, 24))
                cols.append(np.tile(dofs, 24))
                vals.append((rho[e] ** o.penal * K0).ravel())
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(3 * nn, 3 * nn))
    cls = o.node_class()
    free = np.tile(((cls & 4) == 0) & ((cls & 1) > 0), 3)
    return K, free


def test_apply_k_and_solve_vs_scipy(oracle):
    prob = P.ellipsoid(16, 12, 10)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=2, first_factor=2)
    o.set_density(prob["rho"].ravel())
    K, free = assemble(o, prob, oracle.k0())
    rng = np.random.default_rng(0)
    u = rng.standard_normal(3 * o.nn) * free
    ref = K @ u
    ref[~free] = u[~free]
    assert np.linalg.norm(o.apply_K(u) - ref) < 1e-12 * np.linalg.norm(ref)
    f = rng.standard_normal(3 * o.nn) * free
    o.update_stencil()
    ug, it, rr = o.solve(f, tol=1e-12)
    uref = np.zeros_like(f)
    uref[free] = spl.spsolve(K[free][:, free].tocsc(), f[free])
    assert rr < 1e-12
    assert np.linalg.norm(ug - uref) < 1e-9 * np.linalg.norm(uref)


def test_patch_uniform_strain(oracle):
    """A uniform strain field is in equilibrium: interior forces vanish."""
    n = 6
    em = np.ones((n, n, n), np.uint8)
    z = np.zeros((n + 1,) * 3, np.uint8)
    o = oracle.Problem(em, z, z, None, n_levels=1, first_factor=2)
    o.set_density(np.ones(n ** 3))
    eps = np.array([[1e-3, 2e-4, 0], [2e-4, -5e-4, 3e-4], [0, 3e-4, 7e-4]])
    zz, yy, xx = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    X = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(float)
    u = (X @ eps.T).T.ravel()
    f = o.apply_K(u).reshape(3, n + 1, n + 1, n + 1)
    assert abs(f[:, 1:-1, 1:-1, 1:-1]).max() < 1e-9 * abs(f).max()
    # and rigid motions produce no force at all (optimization.cpp:1167-1179)
    R = rigid_modes(X)
    for k in range(6):
        r = R[:, k].reshape(-1, 3).T.ravel()
        assert abs(o.apply_K(r)).max() < 1e-8


def dense_P(fine_dims, F):
    """trilinear interpolation from the coarse node grid (factor F) to the fine node grid"""
    nxf, nyf, nzf = fine_dims
    exc = [-(-(n - 1) // F) for n in fine_dims]
    nxc, nyc, nzc = [e + 1 for e in exc]
    rows, cols, vals = [], [], []
    for z in range(nzf):
        for y in range(nyf):
            for x in range(nxf):
                i = x + nxf * (y + nyf * z)
                for A in range(8):
                    X, Y, Z = x // F + (A & 1), y // F + ((A >> 1) & 1), z // F + (A >> 2)
                    w = 1.0
                    for c, C in ((x, X), (y, Y), (z, Z)):
                        w *= max(F - abs(c - F * C), 0) / F
                    if w > 0 and X < nxc and Y < nyc and Z < nzc:
                        rows.append(i)
                        cols.append(X + nxc * (Y + nyc * Z))
                        vals.append(w)
    Pn = sp.csr_matrix((vals, (rows, cols)), shape=(nxf * nyf * nzf, nxc * nyc * nzc))
    return sp.kron(sp.eye(3), Pn).tocsr()


def stencil_matrix(S, dims):
    nx, ny, nz = dims
    nn = nx * ny * nz
    rows, cols, vals = [], [], []
    for d in range(27):
        dx, dy, dz = d % 3 - 1, d // 3 % 3 - 1, d // 9 - 1
        for r in range(3):
            for c in range(3):
                v = S[d, r, c]
                for n in np.nonzero(v)[0]:
                    x, y, z = n % nx, n // nx % ny, n // (nx * ny)
                    j = (x + dx) + nx * ((y + dy) + ny * (z + dz))
                    rows.append(r * nn + n)
                    cols.append(c * nn + j)
                    vals.append(v[n])
    return sp.csr_matrix((vals, (rows, cols)), shape=(3 * nn, 3 * nn))


@pytest.mark.parametrize("ff", [2, 4])
def test_galerkin_equals_rkp(oracle, ff):
    """Coarse stencils equal R K_mod P with K_mod the support-modified fine
    operator (restrict_stencil_nondyadic_OTFA_WS_kernel Grid.cu:1154-1268) and
    the dyadic stencil recursion (restrict_stencil_dyadic_kernel :882-939)."""
    prob = P.ellipsoid(16, 12, 8)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=3, first_factor=ff)
    o.set_density(prob["rho"].ravel())
    o.update_stencil()
    K0 = oracle.k0()
    K, free = assemble(o, prob, K0)
    cls = o.node_class()
    sup = np.tile((cls & 4) > 0, 3)
    # element-wise modification: support rows/cols zeroed, diagonal 1e6 per incident active element
    Kl = K.tolil()
    cnt = np.zeros(3 * o.nn)
    em = prob["emask"]
    for z in range(o.ez):
        for y in range(o.ey):
            for x in range(o.ex):
                if em[z, y, x]:
                    for a in range(8):
                        n = (x + (a & 1)) + (o.ex + 1) * ((y + ((a >> 1) & 1)) + (o.ey + 1) * (z + (a >> 2)))
                        for c in range(3):
                            cnt[c * o.nn + n] += 1
    Kc = K.tocsr()
    D = sp.diags(np.where(sup, 0.0, 1.0))
    Kmod = (D @ Kc @ D + sp.diags(np.where(sup, 1e6 * cnt, 0.0))).tocsr()
    fine = (o.ex + 1, o.ey + 1, o.ez + 1)
    A = Kmod
    for lvl in range(1, o.n_levels()):
        F = ff if lvl == 1 else 2
        Pm = dense_P(fine, F)
        A = (Pm.T @ A @ Pm).tocsr()
        d = o.level_dims(lvl)
        fine = (int(d[3]), int(d[4]), int(d[5]))
        S = stencil_matrix(o.stencil(lvl), fine)
        diff = abs(S - A).max()
        assert diff < 1e-9 * abs(A).max(), (lvl, diff)


def test_vcycle_convergence(oracle):
    """test_vcycle (grid/Grid.cpp:2311-2404): random force, V(1,1) cycles with
    the reference hierarchy reach r_rel 1e-4 within 20 cycles; on the rough
    cantilever density the contraction factor stays below 0.75."""
    prob = P.cantilever(32, 16, 16)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, nu=0.3, n_levels=0, first_factor=4)
    o.set_density(np.ones(o.ne))
    o.update_stencil()
    rng = np.random.default_rng(0)
    cls = o.node_class()
    f = rng.uniform(-1, 1, 3 * o.nn) * np.tile((cls & 4) == 0, 3)
    u = np.zeros(3 * o.nn)
    for k in range(20):
        u, rr = o.vcycle(u, f, 1, 1, 0, 1.0, 0)
        if rr < 1e-4:
            break
    assert rr < 1e-4
    o.set_density(prob["rho"].ravel())
    o.update_stencil()
    u = np.zeros(3 * o.nn)
    hist = []
    for k in range(12):
        u, rr = o.vcycle(u, prob["f"], 1, 1, 0, 1.0, 0)
        hist.append(rr)
    assert (hist[-1] / hist[2]) ** (1 / 9) < 0.75


def test_numbering_rank_property(oracle):
    """BitSAT rank (selfTest, optimization.cu:712-765) and the GS colour order."""
    prob = P.voids_box(20, 12, 12, 4)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=3, first_factor=2)
    for lvl in range(o.n_levels()):
        d = o.level_dims(lvl)
        em, vm = o.level_masks(lvl)
        eb, vb = o.level_bitwords(lvl)
        bits = np.unpackbits(vb.view(np.uint8), bitorder="little")[: len(vm)]
        assert np.array_equal(bits, vm)
        num = o.ref_numbering(lvl)
        nx, ny = int(d[3]), int(d[4])
        ids = np.nonzero(vm)[0]
        col = (ids % nx % 2) + 2 * (ids // nx % ny % 2) + 4 * (ids // (nx * ny) % 2)
        assert np.all(num["gs_num"] % 32 == 0)
        gs = num["vlexi2gs"]
        assert len(np.unique(gs)) == len(gs)
        off = np.concatenate([[0], np.cumsum(num["gs_num"])])
        for c in range(8):
            sel = gs[col == c]
            assert np.array_equal(sel, off[c] + np.arange(len(sel)))
        flags = num["vflag"]
        assert np.all(flags[np.setdiff1d(np.arange(len(flags)), gs)] == -1)
        assert np.all(((flags[gs] >> 9) & 7) == col)


def test_worst_case_dense_lanczos_pm(oracle):
    """modifiedPM vs the dense aggregated eigenproblem (verifyModifiedPM,
    utils/test_utils.cpp:2598-2645) and Lanczos vs both."""
    prob = P.top_loaded_cube(8)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, n_levels=3, first_factor=2)
    o.set_density(prob["rho"].ravel())
    o.update_stencil()
    lam, fw, uw = o.dense_worst(0)
    lam_l, fl, ul, ritz = o.lanczos(40, 0, tol=1e-11)
    assert abs(lam_l - lam) < 1e-8 * lam
    c, fp, up, itn = o.modified_pm(0, seed=3, max_itn=500)
    assert abs(c - lam) < 1e-4 * lam
    assert abs(fw @ uw - lam) < 1e-8 * lam


def test_sensitivity_fd(oracle):
    """dC/drho from the adjoint equals central finite differences (h = 1e-6)."""
    prob = P.cantilever(8, 4, 4)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, nu=0.3, n_levels=2, first_factor=2)
    rho = prob["rho"].ravel().copy()
    f = prob["f"]

    def comp(r):
        o.set_density(r)
        o.update_stencil()
        u, _, _ = o.solve(f, tol=1e-13, max_iter=500)
        return f @ u, u

    c0, u0 = comp(rho)
    o.set_density(rho)
    s = o.sensitivity(u0)
    for e in [0, 17, 63, 100]:
        rp, rm = rho.copy(), rho.copy()
        rp[e] += 1e-6
        rm[e] -= 1e-6
        fd = (comp(rp)[0] - comp(rm)[0]) / 2e-6
        assert abs(fd - s[e]) < 1e-5 * abs(s).max()


def test_spline_properties(oracle):
    prob = P.cantilever(20, 12, 10)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, n_levels=1)
    for order in (3, 4):
        nc = o.spline_setup(order, (5, 4, 3))
        for ax in range(3):
            idx, N, dN = o.spline_axis(ax)
            assert np.all(idx >= order)
            assert np.allclose(N.sum(1), 1.0, atol=1e-12)    # partition of unity
            assert np.allclose(dN.sum(1), 0.0, atol=1e-10)
        assert np.allclose(o.coeff2density(np.full(nc, 0.6)), 0.6)
        rng = np.random.default_rng(1)
        c = rng.uniform(0.1, 0.9, nc)
        g = rng.standard_normal(o.ne)
        # adjoint is the transpose of the (unclamped) forward map
        lhs = o.coeff2density(c) @ g
        rhs = c @ o.density2coeff_adjoint(g)
        assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_density_filter_adjoint(oracle):
    prob = P.ellipsoid(14, 10, 10)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=1)
    rng = np.random.default_rng(2)
    em = prob["emask"].ravel() > 0
    a, b = rng.standard_normal(o.ne) * em, rng.standard_normal(o.ne) * em
    assert abs(o.density_filter(2.0, a) @ b - a @ o.density_filter_adjoint(2.0, b)) < 1e-10


def test_selfsupport_gradient_fd(oracle):
    """analytic dcoeff of the overhang constraint vs central differences"""
    prob = P.cantilever(12, 10, 10)
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], None, n_levels=1)
    nc = o.spline_setup(3, (4, 3, 3))
    rng = np.random.default_rng(3)
    c = rng.uniform(0.2, 0.8, nc)
    for mode in (5, 3):
        v, per, dc, cnt, ds = o.selfsupport(c, 8.0, mode)
        for k in rng.choice(nc, 6, replace=False):
            cp, cm = c.copy(), c.copy()
            cp[k] += 1e-6
            cm[k] -= 1e-6
            fd = (o.selfsupport(cp, 8.0, mode)[0] - o.selfsupport(cm, 8.0, mode)[0]) / 2e-6
            assert abs(fd - dc[k]) < 1e-4 * max(abs(dc).max(), 1e-12)


def run_mma(oracle, n, m, lo, hi, f, df, g, dg, x0=None, iters=200):
    s = oracle.MMA(n, m, lo, hi)
    if x0 is not None:
        s.set_x(x0)
    for _ in range(iters):
        x = s.get()[0]
        conv, _ = s.update(df(x), dg(x), g(x))
        if conv:
            break
    return s.get()[0]


def test_mma_case1(oracle):
    """test_mma case 1 (optimization/mma_t.cpp:167-200): 1 variable, 1 constraint."""
    f = lambda x: x * np.exp(-x * x) + np.sin(x)
    df = lambda x: np.exp(-x * x) * (1 - 2 * x * x) + np.cos(x)
    g = lambda x: np.array([(x[0] - 1.5) ** 2 - 1])
    dg = lambda x: np.array([[2 * x[0] - 3]])
    x = run_mma(oracle, 1, 1, 0.5, 2.0, f, df, g, dg)
    # from the box midpoint 1.25, f' < 0: descent leads to the local minimum at the upper bound
    # (a KKT point with f'(2) < 0 and g(2) < 0 inactive)
    assert df(1.25) < 0 and df(2.0) < 0
    assert abs(x[0] - 2.0) < 1e-3


def test_mma_case3(oracle):
    """test_mma case 3 (optimization/mma_t.cpp:240-330): 2 variables, 4 constraints."""
    f = lambda v: v[0] / 2 + v[1] * np.sqrt(3) / 2 + np.exp(10 * (v[0] - v[1]) ** 2)
    df = lambda v: np.array([0.5 + 20 * (v[0] - v[1]) * np.exp(10 * (v[0] - v[1]) ** 2),
                             np.sqrt(3) / 2 + 20 * (v[1] - v[0]) * np.exp(10 * (v[0] - v[1]) ** 2)])
    g = lambda v: np.array([v[0] ** 2 + v[1] ** 2 - 1, v[0] ** 2 - 0.75, v[1] ** 2 - 0.75, (v[0] + v[1]) ** 2 - 1])
    dg = lambda v: np.array([[2 * v[0], 2 * v[1]], [2 * v[0], 0], [0, 2 * v[1]], [2 * (v[0] + v[1])] * 2])
    x = run_mma(oracle, 2, 4, -1.0, 1.0, f, df, g, dg)
    cons = [{"type": "ineq", "fun": lambda v, i=i: -g(v)[i]} for i in range(4)]
    ref = so.minimize(f, [0.0, 0.0], jac=df, bounds=[(-1, 1)] * 2, constraints=cons, method="SLSQP", tol=1e-12)
    assert np.allclose(x, ref.x, atol=2e-3)
    assert f(x) - ref.fun < 1e-4


def free_box(ex=6, ey=4, ez=4):
    """A support-free box, load set the x = ex face (normal +x)."""
    em = np.ones((ez, ey, ex), np.uint8)
    fa = np.zeros((ez + 1, ey + 1, ex + 1), np.uint8)
    la = np.zeros_like(fa)
    la[:, :, ex] = 1
    nrm = np.zeros((fa.size, 3))
    nrm[:, 0] = 1.0
    rho = np.random.default_rng(8).uniform(0.3, 1.0, em.shape)
    return dict(emask=em, fixed=fa, load=la, normals=nrm, rho=rho)


@pytest.mark.parametrize("cf", [0, 1])
def test_support_free_worst_case_vs_pseudo_inverse(oracle, cf):
    """Support-free modes (nsff, nscf; optimization/optimization.cpp:99-117):
    the oracle's coarsest pseudo-inverse, rigid-motion removal of loads
    (forceProject, projection.cpp:289-360) and of displacements
    (displacementProject, :374-411) against a dense pseudo-inverse of the
    scipy-assembled K: solutions of consistent loads, the dense aggregated
    worst case and Lanczos."""
    prob = free_box()
    o = oracle.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], n_levels=2, first_factor=2)
    o.set_density(prob["rho"].ravel())
    o.update_stencil()
    K, _ = assemble(o, prob, oracle.k0())
    Kp = np.linalg.pinv(K.toarray(), rcond=1e-10)
    nn = o.nn
    zz, yy, xx = np.meshgrid(np.arange(o.ez + 1), np.arange(o.ey + 1), np.arange(o.ex + 1), indexing="ij")
    X = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(float)
    R = rigid_modes(X)
    Rf = np.stack([R[:, k].reshape(-1, 3).T.ravel() for k in range(6)], 1)  # SoA rows (c nn + n)
    # consistent load: a random load on the load nodes without rigid part
    rng = np.random.default_rng(3)
    f = o.force_project(rng.standard_normal(3 * nn), cf)
    assert np.abs(Rf.T @ f).max() < 1e-10 * np.linalg.norm(f) * np.abs(Rf).max()
    u, _, rr = o.solve(f, tol=1e-12)
    assert rr < 1e-12
    assert np.abs(Rf.T @ u).max() < 1e-9 * np.linalg.norm(u) * np.abs(Rf).max()
    assert np.linalg.norm(u - Kp @ f) < 1e-7 * np.linalg.norm(Kp @ f)
    # dense worst case: lambda_max of K^+ over unit admissible loads
    ln = o.load_nodes()
    if cf:
        B = np.zeros((3 * nn, len(ln)))
        for k, n in enumerate(ln):
            B[n, k] = 1.0  # normal +x
    else:
        B = np.zeros((3 * nn, 3 * len(ln)))
        for k, n in enumerate(ln):
            for c in range(3):
                B[c * nn + n, 3 * k + c] = 1.0
    # admissible subspace: span(B) without the rigid motions of the load set
    Rl = B.T @ Rf  # in cf mode only the normal components: some motions vanish there
    Ul, sl, _ = np.linalg.svd(Rl, full_matrices=False)
    qr = Ul[:, sl > 1e-8 * sl.max()]
    Pm = np.eye(B.shape[1]) - qr @ qr.T
    w, V = np.linalg.eigh(Pm)
    Z = V[:, w > 0.5]
    lam_ref = np.linalg.eigvalsh(Z.T @ B.T @ Kp @ B @ Z).max()
    lam_o, fo, uo = o.dense_worst(cf, tol=1e-12)
    assert abs(lam_o - lam_ref) <= 1e-7 * lam_ref
    assert abs(np.linalg.norm(fo) - 1) < 1e-9
    lam_l, _, _, _ = o.lanczos(40, cf, tol=1e-11)
    assert abs(lam_l - lam_ref) <= 1e-6 * lam_ref
