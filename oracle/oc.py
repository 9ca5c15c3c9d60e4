"""Optimality-criteria updaters restated in numpy (FP32 arithmetic where the
reference computes in FP32).

TEST INFRASTRUCTURE ONLY: the checker of the library's OC entry points; the
product library never imports it.  Parity unpinned: the reference ships no OC
fixtures and cannot be built here, so this restatement of its code is the only
anchor.

Follows optimization/optimization.cu of the reference:
  trySensMultiplier_kernel  :366-392  (the per-element update)
  updateDensities           :394-471  (bisection, at most 31 trials)
  updateDensities2          :473-598  (built without ENABLE_HEAVISIDE: the
                                       same update, extra bracket-width stop,
                                       at most 51 trials)
  tryCSensMultiplier_kernel :560-598  (the per-coefficient update)
  updateCoeff               :600-706  (bisection with coeff2density per trial;
                                       the final threshold is applied to the
                                       last trial's coefficients)
"""
import numpy as np

f32 = np.float32


def _try(src, sens, g, step, damp, lo, hi, shell=None):
    gi = np.abs(np.minimum(sens.astype(f32), f32(0)))
    old = src.astype(f32)
    v = (old * np.power(gi / f32(g), f32(damp))).astype(f32)
    v = np.minimum(np.maximum(v, old - f32(step)), old + f32(step))
    v = np.minimum(np.maximum(v, f32(lo)), f32(hi))
    if shell is not None:
        v = np.where(shell.astype(bool), f32(1), v)
    return v.astype(f32)


def update_density(rho, sens, active, vgoal, step, damp, rho_min, shell=None, variant=0):
    """(new rho, g, volume, trials); rho, sens dense over the box, active a boolean mask."""
    active = active.astype(bool)
    n = int(active.sum())
    gmax = f32(np.max(np.abs(sens[active].astype(f32))))
    lo, hi = f32(0), gmax
    goal = f32(vgoal)
    g = f32((lo + hi) / f32(2))
    V = f32(2)
    itn = trials = 0

    def trial(gg):
        out = _try(rho, sens, gg, step, damp, rho_min, 1.0, shell)
        out = np.where(active, out, rho.astype(f32))
        return out, f32(np.sum(out[active], dtype=np.float64) / n)

    while True:
        g = f32((lo + hi) / f32(2))
        _, V = trial(g)
        trials += 1
        if V > goal:
            lo = g
        elif V < goal:
            hi = g
        if variant == 0:
            go = abs(V - goal) > f32(1e-4)
            if go:
                go = itn < 30
                itn += 1
        else:
            go = abs(V - goal) > f32(1e-4) and (hi - lo) / (lo + hi) > f32(1e-3)
            if go:
                go = itn < 50
                itn += 1
        if not go:
            break
    out, Vf = trial(g)
    return out, float(g), float(Vf), trials


def update_coeff(problem, coeff, csens, vgoal, step, damp, cmin, cmax):
    """(new coefficients, densities, g, volume, trials) with the oracle's coeff2density."""
    active = problem.level_masks(0)[0].astype(bool)
    n = int(active.sum())
    copy = coeff.astype(f32).copy()
    gmax = f32(np.max(np.abs(csens.astype(f32))))
    lo, hi = f32(0), gmax
    goal = f32(vgoal)
    g = f32((lo + hi) / f32(2))
    itn = trials = 0

    def volume(c):
        rho = problem.coeff2density(c.astype(np.float64))
        return rho, f32(np.sum(rho[active].astype(f32), dtype=np.float64) / n)

    cur = copy
    while True:
        g = f32((lo + hi) / f32(2))
        cur = _try(copy, csens, g, step, damp, cmin, cmax)
        _, V = volume(cur)
        trials += 1
        if V > goal:
            lo = g
        elif V < goal:
            hi = g
        go = abs(V - goal) > f32(1e-4)
        if go:
            go = itn < 30
            itn += 1
        if not go:
            break
    final = _try(cur, csens, g, step, damp, cmin, cmax)
    rho, Vf = volume(final)
    return final, rho, float(g), float(Vf), trials
