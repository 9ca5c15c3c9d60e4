"""Writes the golden fixtures of tests/golden/ from the reference's own code.

Builds oracle/_ref/ref_golden (`make -C oracle ref`: definitions extracted
unmodified from the reference's sources and compiled on the host, see
oracle/ref_golden.cpp), feeds it seeded inputs and stores inputs and outputs
as .npz files beside this script:

  funcs.npz   Heaviside, Dirac and the self-support penalty functions
              (grid/Grid.cu:76-190) on a grid of points, for several
              parameter sets (including the sigmoid midpoint and width of
              HierarchyGrid::setPrintAngle, grid/Grid.cu:3161-3185)
  proj.npz    computeProjection_kernel and computeProjectionSensitivity_kernel
              (optimization/optimization.cu:324-348, :167-189), shell flags set
  spline.npz  the knot series (grid/Grid.cpp:3307-3431), SplineBasisX/Y/Z and
              SplineBasisDeri* at the element centres (grid/Grid.cu:427-857)
              and coeff2density (grid/Grid.cu:3405-3502) on a masked 16^3 grid
  filter.npz  filterSensitivity_kernel (grid/Grid.cu:4210-4309) on a masked
              16^3 grid at four radii
  surface.npz the surface-point self-support pieces on a 16^3 box: background
              marching-cubes values and positions (grid/Grid.cu:4109-4160),
              generateEquidistantIntegers (grid/Grid.cpp:3831-3847), and at
              seeded points the normals, orientation probes, flags, per-point
              constraint values, means and coefficient gradients of all six
              modes (grid/Grid.cu:5709-6505, grid/Grid.cpp:4263-4280)

Needs the reference's sources (REF, default /root/reference) and g++; the
fixtures it writes are committed, so the tests need neither.  Run:
  python tests/golden/make_golden.py [fixture ...]   (default: all)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle")
EXE = os.path.join(ORACLE, "_ref", "ref_golden")
SHELL_BIT = 1 << 12  # mask_shellelement, grid/Grid.h:412


def run(args):
    subprocess.run([EXE] + [str(a) for a in args], check=True)


def sigmoid_params(default_angle_ratio):
    """adapt_sigmoid_mid and adapt_sigmoid_c as HierarchyGrid::setPrintAngle
    forms them (float arithmetic)."""
    s = np.float32(default_angle_ratio * np.pi)
    mid = np.float32(np.cos(np.float32(np.pi), dtype=np.float32) / np.cos(s, dtype=np.float32))
    c = np.float32((mid - np.float32(1)) / np.log(1 / 0.004 - 1))
    return float(mid), float(c)


def bit_words(mask_zyx):
    """eActiveBits and its chunk prefix sums: bit id x + y e + z e^2."""
    flat = mask_zyx.ravel().astype(np.uint64)
    nword = (flat.size + 31) // 32
    pad = np.zeros(nword * 32, np.uint64)
    pad[:flat.size] = flat
    words = (pad.reshape(nword, 32) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)
    counts = pad.reshape(nword, 32).sum(axis=1).astype(np.int64)
    sat = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return words, sat


def masked_cube(e, seed):
    """An ellipsoid in an e^3 box with a few random voids and extra voxels."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(e), np.arange(e), np.arange(e), indexing="ij")
    c = (e - 1) / 2
    m = ((x - c) / (0.48 * e)) ** 2 + ((y - c) / (0.40 * e)) ** 2 + ((z - c) / (0.45 * e)) ** 2 <= 1
    m ^= rng.uniform(size=m.shape) < 0.06
    return m.astype(np.uint8)


def surface_fixture(p):
    e, order, parts, mc = 16, 3, (4, 3, 5), 16
    nb = [order + q for q in parts]
    rng = np.random.default_rng(31)
    coeff = rng.normal(0.5, 0.15, nb[0] * nb[1] * nb[2]).astype(np.float32)
    # points inside the box where the spline support holds every one of them
    pts = rng.uniform(0.25, e - 0.25, (3, 500)).astype(np.float32)
    coeff.tofile(p("coeff")); pts.tofile(p("pts"))
    beta, opt_ratio, default_ratio = 8.0, 0.75, 0.75
    run(["surface", e, order, *parts, p("coeff"), mc, pts.shape[1], p("pts"), beta, opt_ratio, default_ratio,
         p("mc"), p("eq"), p("po"), p("dc"), p("sc")])
    n3 = (mc + 2) ** 3
    npt = pts.shape[1]
    po = np.fromfile(p("po"), np.float32)
    out = dict(ereso=e, order=order, parts=np.array(parts, np.int32), mc=mc, coeff=coeff, pts=pts, beta=beta,
               opt_ratio=opt_ratio, default_ratio=default_ratio,
               mc_out=np.fromfile(p("mc"), np.float32).reshape(4, n3),
               equi_pairs=np.array([[100, 10], [1000, 300], [1574, 1500], [12345, 600], [50, 49], [7, 3]], np.int64),
               equi=np.fromfile(p("eq"), np.int32),
               normals=po[:3 * npt].reshape(3, npt), direction=po[3 * npt:4 * npt], flag=po[4 * npt:5 * npt],
               per=po[5 * npt:].reshape(6, npt),
               dc=np.fromfile(p("dc"), np.float32).reshape(6, -1),
               scalars=np.fromfile(p("sc"), np.float32))
    np.savez_compressed(os.path.join(HERE, "surface.npz"), **out)


def main(which=()):
    subprocess.run(["make", "-s", "-C", ORACLE, "ref"], check=True)
    with tempfile.TemporaryDirectory() as td:
        p = lambda name: os.path.join(td, name)  # noqa: E731
        if which:
            if "surface" in which:
                surface_fixture(p)
            print("wrote", ", ".join(f"{w}.npz" for w in which))
            return 0

        # ------------------------------------------------------------- functions
        x = np.concatenate([np.linspace(-0.5, 2.5, 601), np.random.default_rng(1).uniform(-1, 3, 200),
                            [0.0, 0.5, 1.0, 1.5]]).astype(np.float32)
        x.tofile(p("x"))
        sets = []
        for beta, a, ang in ((1.0, 1.0, 0.75), (8.0, 5.0, 0.75), (16.0, 20.0, 0.7), (32.0, 0.5, 0.8)):
            mid, c = sigmoid_params(ang)
            run(["funcs", x.size, p("x"), beta, a, mid, c, p("o")])
            sets.append(((beta, a, mid, c), np.fromfile(p("o"), np.float32).reshape(10, x.size)))
        np.savez_compressed(os.path.join(HERE, "funcs.npz"), x=x,
                            params=np.array([s[0] for s in sets], np.float64),
                            out=np.stack([s[1] for s in sets]))

        # ------------------------------------------------------------ projection
        rng = np.random.default_rng(2)
        n = 4096
        rho = rng.uniform(-0.1, 1.1, n).astype(np.float32)
        flag = rng.integers(0, 1 << 22, n).astype(np.int32) & ~SHELL_BIT
        flag[rng.uniform(size=n) < 0.125] |= SHELL_BIT
        sens = rng.standard_normal(n).astype(np.float32)
        rho.tofile(p("rho")); flag.tofile(p("flag")); sens.tofile(p("sens"))
        outs = []
        betas = (1.0, 8.0, 32.0)
        rhomin = 1e-3
        for beta in betas:
            run(["proj", n, beta, rhomin, p("rho"), p("flag"), p("sens"), p("or"), p("os")])
            outs.append((np.fromfile(p("or"), np.float32), np.fromfile(p("os"), np.float32)))
        np.savez_compressed(os.path.join(HERE, "proj.npz"), rho=rho, flag=flag, sens=sens,
                            betas=np.array(betas), rhomin=rhomin,
                            out_rho=np.stack([o[0] for o in outs]), out_sens=np.stack([o[1] for o in outs]))

        # ---------------------------------------------------------------- spline
        e = 16
        mask = masked_cube(e, 3)
        words, sat = bit_words(mask)
        words.tofile(p("bits")); sat.tofile(p("sat"))
        na = int(sat[-1])
        cases = {}
        for ci, parts in enumerate(((3, 4, 5), (6, 6, 6))):
            order = 3
            nb = [order + q for q in parts]
            coeff = np.random.default_rng(10 + ci).uniform(0, 1, nb[0] * nb[1] * nb[2]).astype(np.float32)
            eflag = np.zeros(na, np.int32)
            eflag[np.random.default_rng(20 + ci).uniform(size=na) < 0.1] = SHELL_BIT
            coeff.tofile(p("coeff")); eflag.tofile(p("eflag"))
            run(["spline", e, order, *parts, words.size, p("bits"), p("sat"), p("coeff"), p("eflag"), rhomin,
                 p("kn"), p("ax"), p("rh")])
            cases[f"parts{ci}"] = np.array(parts, np.int32)
            cases[f"coeff{ci}"] = coeff
            cases[f"eflag{ci}"] = eflag
            cases[f"knots{ci}"] = np.fromfile(p("kn"), np.float32)
            cases[f"axis{ci}"] = np.fromfile(p("ax"), np.float32).reshape(3, e, 2 * order + order + 1)
            cases[f"rho{ci}"] = np.fromfile(p("rh"), np.float32)
        np.savez_compressed(os.path.join(HERE, "spline.npz"), ereso=e, order=3, rhomin=rhomin, mask=mask,
                            **cases)

        # ---------------------------------------------------------------- filter
        mask = masked_cube(e, 4)
        words, sat = bit_words(mask)
        words.tofile(p("bits")); sat.tofile(p("sat"))
        na = int(sat[-1])
        g = np.random.default_rng(5).standard_normal(na).astype(np.float32)
        g.tofile(p("g"))
        radii = (1.0, 1.5, 2.0, 2.6)
        outs = []
        for r in radii:
            run(["filter", e, words.size, p("bits"), p("sat"), na, p("g"), r, p("o")])
            outs.append(np.fromfile(p("o"), np.float32))
        np.savez_compressed(os.path.join(HERE, "filter.npz"), ereso=e, mask=mask, sens=g,
                            radii=np.array(radii), out=np.stack(outs))
        surface_fixture(p)
    print("wrote", ", ".join(f for f in sorted(os.listdir(HERE)) if f.endswith(".npz")))


if __name__ == "__main__":
    sys.exit(main(tuple(sys.argv[1:])))
