"""Writes tests/golden/config1.npz: the FP64 oracle's worst case on the
128x64x64 ellipsoid (semi-axes 60, 30, 30 voxels, centred; lowest active
node layer clamped; load set the surface nodes of the 3-voxel outer shell,
load directed along the analytic outward normal; rho = 0.4 + U[-0.05, 0.05];
E = 1e6, nu = 0.4, SIMP p = 3, rho_min = 1e-3), computed as 20 Lanczos steps
with full FP64 reorthogonalisation and one multigrid solve to relative
residual 1e-10 per step, from the seeded start vector (seed 1234) the
library uses too.

Stored: lambda_max and the 20 Ritz values, the norms of f_worst and u_worst,
and f_worst, u_worst and d lambda / d rho at seeded samples of their
non-zero entries (the full fields would be megabytes).  The oracle takes a
few minutes here, too long for a test run, hence the fixture.  Run:
  python tests/golden/make_config1.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

NU = 0.4
SEED = 1234
STEPS = 20
TOL = 1e-10
NSAMPLE = 8192


def config1_problem():
    return P.ellipsoid(128, 64, 64, seed=1, shell=3, axes=(60.0, 30.0, 30.0))


def main():
    prob = config1_problem()
    o = O.Problem(prob["emask"], prob["fixed"], prob["load"], prob["normals"], nu=NU)
    o.set_density(prob["rho"].astype(np.float32).astype(np.float64).ravel())
    o.update_stencil()
    t0 = time.time()
    lam, fw, uw, ritz = o.lanczos(STEPS, 1, tol=TOL, seed=SEED)
    sens = o.sensitivity(uw)
    rng = np.random.default_rng(77)
    iu = np.sort(rng.choice(np.flatnonzero(uw), NSAMPLE, replace=False))
    nzf = np.flatnonzero(fw)
    jf = np.sort(rng.choice(nzf, min(NSAMPLE, nzf.size), replace=False))
    ks = np.sort(rng.choice(np.flatnonzero(sens), NSAMPLE, replace=False))
    np.savez_compressed(os.path.join(HERE, "config1.npz"), lam=lam, ritz=ritz, f_norm=np.linalg.norm(fw),
                        u_norm=np.linalg.norm(uw), iu=iu, u=uw[iu], jf=jf, f=fw[jf], ks=ks, sens=sens[ks],
                        sens_sum=sens.sum(), sens_norm=np.linalg.norm(sens), n_levels=o.n_levels(),
                        active=int(prob["emask"].sum()), nu=NU, seed=SEED, tol=TOL)
    print(f"lambda_max {lam:.12e}, {o.n_levels()} levels, {int(prob['emask'].sum())} active elements, "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
