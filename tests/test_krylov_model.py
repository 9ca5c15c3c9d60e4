"""Host model of the mixed-precision PCG recurrence of solver.cu
(solve_pcg_k32): p, q = K p, r and z in FP32, the sums in FP64, the iterate
in FP64, and the true FP64 residual replacing the recursive one whenever it
has dropped by the replacement factor, after at most 30 iterations, and
before stopping; a replacement whose true residual is not below
max(0.5, sqrt(factor), sqrt(claimed)) of the previous one (claimed: the
reduction the recursive residual showed over the cycle) hands the solve over
to the FP64 recurrence from the current iterate.  On a well-conditioned system the FP32
recurrence reaches a true relative residual of 1e-10 on its own, in about
the FP64 recurrence's iteration count.  On an ill-conditioned one (a 2-D
diffusion operator with a 1e6 coefficient contrast, Jacobi-preconditioned)
it stalls, and the hand-over ends where the FP64 recurrence alone would.
This checks the algorithm, not the kernels."""
import numpy as np
import pytest
import scipy.sparse as sp


def operator(n=48, seed=3):
    rng = np.random.default_rng(seed)
    c = np.where(rng.uniform(size=(n + 1, n)) < 0.5, 1.0, 1e-6)  # face coefficients, 1e6 contrast
    d = np.where(rng.uniform(size=(n, n + 1)) < 0.5, 1.0, 1e-6)
    N = n * n
    idx = np.arange(N).reshape(n, n)
    rows, cols, vals = [], [], []
    diag = np.zeros(N)
    for i in range(n):
        for j in range(n):
            k = idx[i, j]
            for (ii, jj, w) in ((i - 1, j, c[i, j]), (i + 1, j, c[i + 1, j]), (i, j - 1, d[i, j]), (i, j + 1, d[i, j + 1])):
                diag[k] += w
                if 0 <= ii < n and 0 <= jj < n:
                    rows.append(k); cols.append(idx[ii, jj]); vals.append(-w)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(N, N)) + sp.diags(diag)
    return A.tocsr(), diag


def pcg64(A, dinv, f, tol, max_iter, x0=None):
    x = np.zeros_like(f) if x0 is None else x0.copy()
    r = f - A @ x
    z = dinv * r
    p = z.copy()
    rz = r @ z
    fn = np.linalg.norm(f)
    for it in range(1, max_iter + 1):
        q = A @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) / fn < tol:
            return x, it
        z = dinv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iter


def stall_ratio(factor, claimed):
    return max(0.5, np.sqrt(factor), np.sqrt(max(claimed, 0.0)))


def pcg_k32(A, dinv, f, tol, max_iter, factor, cycle_max=30, max_cycles=0):
    """(x, iterations, true relative residual, stalled)"""
    f32 = np.float32
    cycles = 0
    A32 = A.astype(f32)
    d32 = dinv.astype(f32)
    x = np.zeros_like(f)
    rt = f - A @ x
    fn = np.linalg.norm(f)
    rbase = np.linalg.norm(rt)
    r = rt.astype(f32)
    z = d32 * r
    p = z.copy()
    rz = float(r.astype(np.float64) @ z.astype(np.float64))
    it = since = 0
    rel = rbase / fn
    while it < max_iter:
        q = A32 @ p
        a = rz / float(p.astype(np.float64) @ q.astype(np.float64))
        r = (r - f32(a) * q).astype(f32)
        rn = float(np.sqrt(r.astype(np.float64) @ r.astype(np.float64)))
        it += 1
        since += 1
        replace = rn < factor * rbase or rn < tol * fn or it >= max_iter or since >= cycle_max
        x += a * p.astype(np.float64)
        if replace:
            rt = f - A @ x
            rtrue = np.linalg.norm(rt)
            rel = rtrue / fn
            if rel < tol or it >= max_iter:
                break
            cycles += 1
            if rtrue > stall_ratio(factor, rn / rbase) * rbase or (max_cycles and cycles >= max_cycles):
                return x, it, rel, True
            rbase = rtrue
            since = 0
            r = rt.astype(f32)
        z = d32 * r
        rz_new = float(r.astype(np.float64) @ z.astype(np.float64))
        p = (z + f32(rz_new / rz) * p).astype(f32)
        rz = rz_new
    return x, it, rel, False


def solve_mixed(A, dinv, f, tol, max_iter, factor, max_cycles=0):
    x, it, rel, stalled = pcg_k32(A, dinv, f, tol, max_iter, factor, max_cycles=max_cycles)
    if stalled:
        x, it2 = pcg64(A, dinv, f, tol, max_iter - it, x0=x)
        it += it2
        rel = np.linalg.norm(f - A @ x) / np.linalg.norm(f)
    return x, it, rel, stalled


def laplacian(n=48):
    return sp.diags([-1.0, -1.0, 4.0, -1.0, -1.0], [-n, -1, 0, 1, n], shape=(n * n, n * n)).tocsr()


@pytest.mark.parametrize("factor", [1e-1, 1e-2, 1e-3])
def test_fp32_recurrence_on_a_well_conditioned_system(factor):
    A = laplacian()
    f = np.random.default_rng(1).standard_normal(A.shape[0])
    dinv = 1.0 / A.diagonal()
    x64, it64 = pcg64(A, dinv, f, 1e-10, 5000)
    x, it, rel, stalled = solve_mixed(A, dinv, f, 1e-10, 5000, factor)
    true = np.linalg.norm(f - A @ x) / np.linalg.norm(f)
    assert not stalled
    assert rel < 1e-10 and abs(true - rel) <= 1e-3 * rel
    assert it <= 1.2 * it64, (it, it64)
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-6


@pytest.mark.parametrize("factor", [1e-2, 1e-3])
def test_stalled_fp32_recurrence_hands_over(factor):
    A, diag = operator()
    f = np.random.default_rng(1).standard_normal(A.shape[0])
    dinv = 1.0 / diag
    x64, it64 = pcg64(A, dinv, f, 1e-9, 20000)
    true64 = np.linalg.norm(f - A @ x64) / np.linalg.norm(f)
    x, it, rel, stalled = solve_mixed(A, dinv, f, 1e-9, 20000, factor)
    assert stalled  # 1e6 contrast with a Jacobi preconditioner is beyond the FP32 recurrence
    # the FP64 recurrence stops on its recursive residual, whose gap to the true one on this
    # system is a factor of a few: the hand-over ends as close to the tolerance as it does
    assert rel < 2 * max(1e-9, true64), (rel, true64)
    assert it <= it64 + 200, (it, it64)


def test_short_last_cycle_is_not_a_stall():
    """A cycle that the tolerance ends after a small reduction of the recursive
    residual (0.9 here) may leave the true residual at 0.93 of the previous
    one: above 0.5, but within sqrt(0.9), so no hand-over."""
    assert stall_ratio(1e-2, 0.9) * 1.0 > 0.93
    assert stall_ratio(1e-2, 1e-2) == 0.5
    assert stall_ratio(1e-3, 0.3) == pytest.approx(np.sqrt(0.3))


@pytest.mark.parametrize("max_cycles", [1, 2])
def test_cycle_bound_hands_over(max_cycles):
    A = laplacian()
    f = np.random.default_rng(2).standard_normal(A.shape[0])
    dinv = 1.0 / A.diagonal()
    x64, it64 = pcg64(A, dinv, f, 1e-10, 5000)
    x, it, rel, stalled = solve_mixed(A, dinv, f, 1e-10, 5000, 1e-2, max_cycles=max_cycles)
    assert stalled
    assert rel < 1e-10 * 1.5
    assert it <= 1.2 * it64 + 5
