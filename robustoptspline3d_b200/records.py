"""Run records in the reference's on-disk layout.

bio::write_vector (utils/binaryIO.h:69-78) writes a std::vector as its raw
native-endian elements, no header; bio::read_vector (:93-107) reads a file
back as len / sizeof(T) elements.  The spline design driver
(optimization/optimization.cpp:822-1097) keeps std::vector<double> records
of the worst-case compliance (cRecord), volume (volRecord), self-support
value (ssRecord), iteration time in ms (tRecord) and the sensitivity-phase
time (testRecord), rewrites them after every iteration as crec_iter, vrec_iter,
ssrec_iter, trec_iter, testrec_iter and at the end as cworst, vrec, ssrec,
trec, and writes the last worst-case force and displacement (flast, ulast).
"""
import os

import numpy as np


def write_vector(path, values, dtype=np.float64):
    """Raw elements of `values` as `dtype` (bio::write_vector)."""
    np.ascontiguousarray(values, dtype=dtype).tofile(path)


def read_vector(path, dtype=np.float64):
    """A file written by write_vector (bio::read_vector)."""
    return np.fromfile(path, dtype=dtype)


class RunRecords:
    """Per-iteration records of a design run, written like the reference's driver."""

    FIELDS = (("c_worst", "crec_iter", "cworst"), ("volume", "vrec_iter", "vrec"),
              ("ss_value", "ssrec_iter", "ssrec"), ("ms_total", "trec_iter", "trec"),
              ("ms_adjoint", "testrec_iter", None))

    def __init__(self, directory):
        self.dir = directory
        os.makedirs(directory, exist_ok=True)
        self.rec = {k: [] for k, _, _ in self.FIELDS}

    def append(self, info):
        """Record one iteration from a design_iteration info dict and rewrite the *_iter files."""
        for key, it_name, _ in self.FIELDS:
            self.rec[key].append(float(info[key]))
            write_vector(os.path.join(self.dir, it_name), self.rec[key])

    def finish(self, f_last=None, u_last=None):
        """Final records (cworst, vrec, ssrec, trec) and, when given, the last worst-case
        force and displacement as flast / ulast (nodal vectors, float64)."""
        for key, _, final in self.FIELDS:
            if final:
                write_vector(os.path.join(self.dir, final), self.rec[key])
        if f_last is not None:
            write_vector(os.path.join(self.dir, "flast"), np.asarray(f_last, np.float64))
        if u_last is not None:
            write_vector(os.path.join(self.dir, "ulast"), np.asarray(u_last, np.float64))


def write_density(prefix, emask, rho):
    """The densities of the active elements with their integer positions: what
    HierarchyGrid::writeDensity (grid/Grid.cpp:1267-1300) stores in an
    OpenVDB grid (absent here), as two raw records: <prefix>.pos, int32
    x, y, z per element in the layout of bio::write_vectors
    (utils/binaryIO.h:80-91), and <prefix>.val, float32 values.  emask is the
    (ez, ey, ex) element mask, rho the dense element field."""
    emask = np.asarray(emask)
    z, y, x = np.nonzero(emask)
    rho = np.asarray(rho, np.float32).reshape(emask.shape)
    write_vector(prefix + ".pos", np.stack([x, y, z], 1).ravel(), np.int32)
    write_vector(prefix + ".val", rho[z, y, x], np.float32)


def read_density(prefix):
    """(positions (n, 3) int32 x, y, z; values (n,) float32) written by write_density."""
    pos = read_vector(prefix + ".pos", np.int32).reshape(-1, 3)
    val = read_vector(prefix + ".val", np.float32)
    if len(pos) != len(val):
        raise ValueError("density records of different lengths")
    return pos, val


def write_coeff(path, coeff):
    """The spline coefficients as float32 raw elements (HierarchyGrid::writeCoeff,
    grid/Grid.cpp:2140-2156, written by the drivers as <out>/coeff)."""
    write_vector(path, np.asarray(coeff, np.float32).ravel(), np.float32)


def read_coeff(path, n_coeff=None):
    """Coefficients written by write_coeff; with n_coeff, the count is checked
    against the handle's spline (a file of another partition is refused)."""
    c = read_vector(path, np.float32)
    if n_coeff is not None and c.size != n_coeff:
        raise ValueError(f"coefficient file holds {c.size} values, the spline has {n_coeff}")
    return c
