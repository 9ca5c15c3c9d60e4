"""OBJ reading for the mesh input (robustoptspline3d_b200.voxelize.read_obj): polygons fanned into
triangles, texture/normal index suffixes and negative indices handled."""
from robustoptspline3d_b200.voxelize import read_obj


def test_read_obj(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("# comment\nmtllib x.mtl\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
                 "f 1/1/1 2/2/2 3/3/3 4/4/4\nf -1 -2 -3\n")
    v, f = read_obj(str(p))
    assert v.shape == (5, 3) and f.shape == (3, 3)
    assert f[0].tolist() == [0, 1, 2] and f[1].tolist() == [0, 2, 3] and f[2].tolist() == [4, 3, 2]
