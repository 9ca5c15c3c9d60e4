"""MMA checkpoint and resume (rso_mma_save / rso_mma_load) through the C ABI:
an MMA run stopped after three updates, saved, loaded into a fresh MMA and
continued must give bit-identical iterates to the run that never stopped;
a checkpoint of the wrong size is refused."""
import numpy as np
import pytest

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
