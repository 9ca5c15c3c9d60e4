"""Run records in the reference's raw binary layout (bio::write_vector /
read_vector): raw native-endian elements, no header, file names as the
reference's spline driver writes them."""
import os

import numpy as np

from robustoptspline3d_b200.records import RunRecords, read_vector, write_vector


def test_vector_round_trip(tmp_path):
    p = os.path.join(tmp_path, "v")
    a = np.array([1.5, -2.0, 3.25])
    write_vector(p, a)
    assert os.path.getsize(p) == 3 * 8
    assert np.array_equal(read_vector(p), a)
    write_vector(p, [1, 2, 3], dtype=np.float32)
    assert os.path.getsize(p) == 12 and np.array_equal(read_vector(p, np.float32), [1, 2, 3])


def test_run_records_layout(tmp_path):
    r = RunRecords(str(tmp_path))
    infos = [dict(c_worst=0.1 * k, volume=0.3, ss_value=0.2, ms_total=100.0 + k, ms_adjoint=5.0) for k in range(3)]
    for i in infos:
        r.append(i)
    assert np.array_equal(read_vector(os.path.join(tmp_path, "crec_iter")), [0.0, 0.1, 0.2])
    r.finish(f_last=np.ones(6), u_last=np.zeros(6))
    for name in ("cworst", "vrec", "ssrec", "trec", "crec_iter", "vrec_iter", "ssrec_iter", "trec_iter",
                 "testrec_iter", "flast", "ulast"):
        assert os.path.exists(os.path.join(tmp_path, name)), name
    assert np.array_equal(read_vector(os.path.join(tmp_path, "trec")), [100.0, 101.0, 102.0])
    assert read_vector(os.path.join(tmp_path, "flast")).size == 6


def test_density_records_round_trip(tmp_path):
    from robustoptspline3d_b200 import records
    rng = np.random.default_rng(4)
    em = (rng.uniform(size=(5, 6, 7)) < 0.6).astype(np.uint8)
    rho = rng.uniform(0, 1, em.shape).astype(np.float32)
    prefix = str(tmp_path / "density0001")
    records.write_density(prefix, em, rho)
    pos, val = records.read_density(prefix)
    assert len(val) == em.sum()
    back = np.zeros_like(rho)
    back[pos[:, 2], pos[:, 1], pos[:, 0]] = val
    assert np.array_equal(back, rho * em)


def test_coeff_round_trip(tmp_path):
    """writeCoeff's layout: float32 raw elements; a file of another size is refused."""
    import pytest
    from robustoptspline3d_b200 import records
    c = np.random.default_rng(3).uniform(0, 1, 7 * 8 * 9)
    p = str(tmp_path / "coeff")
    records.write_coeff(p, c)
    assert os.path.getsize(p) == 4 * c.size
    back = records.read_coeff(p, c.size)
    assert back.dtype == np.float32 and np.array_equal(back, c.astype(np.float32))
    with pytest.raises(ValueError):
        records.read_coeff(p, c.size + 1)
