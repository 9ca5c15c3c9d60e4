"""MMA checkpoint and resume (rso_mma_save / rso_mma_load) through the C ABI:
an MMA run stopped after three updates, saved, loaded into a fresh MMA and
continued must give bit-identical iterates to the run that never stopped;
a checkpoint of the wrong size is refused.  Density restart from saved
records (rso_get_density / rso_set_density_points)."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def _inputs(x, k, n):
    df = -np.exp(-x) * (1 + 0.05 * np.cos(np.arange(n) + k))
    dg = np.stack([np.full(n, 1.0 / n), 0.1 * np.sin(np.arange(n) * 0.3 + k)])
    g = np.array([x.mean() - 0.4, 0.05 * np.sin(k)])
    return df, dg, g


def test_mma_resume_is_exact(cuda):
    import torch
    from robustoptspline3d_b200 import MMA, RSOError
    n, m = 700, 2
    x0 = np.random.default_rng(3).uniform(0.2, 0.8, n)

    def step(mma, k):
        x = mma.get()[0]
        df, dg, g = _inputs(x, k, n)
        mma.update(torch.as_tensor(df, device="cuda"), torch.as_tensor(dg, device="cuda"), g)

    a = MMA(n, m, 0.0, 1.0)
    a.set_x(x0)
    for k in range(3):
        step(a, k)
    state = a.save()
    assert state.size == 6 * n + 1
    for k in range(3, 6):
        step(a, k)
    b = MMA(n, m, 0.0, 1.0)
    b.set_x(np.full(n, 0.5))  # a different start, replaced by the checkpoint
    b.load(state)
    for k in range(3, 6):
        step(b, k)
    for va, vb in zip(a.get(), b.get()):
        assert np.array_equal(va, vb)
    with pytest.raises(RSOError):
        b.load(state[:-1])
    a.close()
    b.close()


def test_density_restart(cuda, tmp_path):
    """writeDensity / readDensity (grid/Grid.cpp:1267-1300, :1914-1945) through
    raw records: a second handle restarted from the saved densities holds the
    same field bit for bit and solves alike; a point on an inactive element or
    outside the grid is refused (the reference exits: "unmatched grid and file")."""
    from robustoptspline3d_b200 import Config, HierarchyGrid, records
    from robustoptspline3d_b200.rso import RSOError
    prob = P.ellipsoid(24, 16, 12)
    mk = lambda: HierarchyGrid(prob["emask"], prob["fixed"], prob["load"], prob["normals"],  # noqa: E731
                               Config(precision=0, smoother=1))
    a, b = mk(), mk()
    rho = (prob["rho"] * np.random.default_rng(3).uniform(0.5, 1.0, prob["rho"].shape)).astype(np.float32)
    a.set_density(rho.ravel())
    prefix = str(tmp_path / "density0003")
    a.writeDensity(prefix)
    b.readDensity(prefix)
    da, db = a.get_density().cpu().numpy(), b.get_density().cpu().numpy()
    assert np.array_equal(da, db)
    assert np.array_equal(db, (rho * prob["emask"]).ravel())
    f = np.zeros(3 * a.nn)
    f[2 * a.nn + a.load_nodes()] = -1.0
    out = []
    for g in (a, b):
        g.update_stencil()
        u, _, rr, _ = g.solve(cuda.tensor(f, dtype=cuda.float64, device="cuda"), tol=1e-10)
        out.append(u.cpu().numpy())
    assert np.array_equal(out[0], out[1])
    pos, val = records.read_density(prefix)
    inactive = np.argwhere(prob["emask"] == 0)[0][::-1].astype(np.int32)  # (x, y, z) of an inactive element
    for bad in (inactive, np.array([prob["emask"].shape[2], 0, 0], np.int32)):
        records.write_vector(prefix + ".pos", np.concatenate([pos.ravel(), bad]), np.int32)
        records.write_vector(prefix + ".val", np.concatenate([val, [0.5]]), np.float32)
        with pytest.raises(RSOError):
            b.readDensity(prefix)
    a.close()
    b.close()
