"""EnSight Gold output of the library's host writers against the reference's own
writers (golden fixtures made by tests/golden/make_golden.py from Mesh::write
and Field<T>::write, src/Mesh/Mesh.cpp:224-355, src/Field/Field.hxx:404-453).
Header lines are compared as text up to the first NUL (the reference leaves
the rest of each 80-byte line unspecified); everything else byte for byte.
These entry points are host code: no GPU needed."""
import os

import numpy as np
import pytest

from conftest import load_golden


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


@pytest.mark.parametrize("name", ["ensight_7x5x6.npz", "ensight_walls_6x8x5.npz"])
def test_writers_match_the_reference(nova, oracle, tmp_path, name):
    g = load_golden(name)
    walls = (0, int(g["walls"]), 0)
    md = nova.ensight.mesh_desc(tuple(int(v) for v in g["N"]), L=tuple(g["L"]), origin=tuple(g["origin"]),
                                walls=walls)
    d = str(tmp_path)
    nova.ensight.write_geometry(md, d)
    nova.ensight.write_case(d, g["times"])
    nova.ensight.write_host(md, g["U"], d, "U", 2)
    nova.ensight.write_host(md, g["p"], d, "p", 2)

    geo = oracle.ensight_parse(os.path.join(d, "geom.p0000.geo"), "geo")
    assert geo["lines"] == list(g["geo_lines"]) and geo["part"] == 1
    assert np.array_equal(geo["dims"], g["geo_dims"]) and np.array_equal(geo["coords"], g["geo_coords"])
    assert geo["size"] == int(g["geo_size"])
    for f in ("U", "p"):
        dat = oracle.ensight_parse(os.path.join(d, "%s.0000.00002.dat" % f), "dat")
        assert dat["lines"] == list(g["dat_lines"]) and dat["part"] == 1
        assert np.array_equal(dat["values"], g[f + "_values"]), f
    assert open(os.path.join(d, "fd.p0000.case")).read() == str(g["case_text"])
    assert open(os.path.join(d, "restart.p.0000.case")).read() == str(g["restart_text"])


def test_read_restores_the_float32_values(nova, tmp_path):
    g = load_golden("ensight_walls_6x8x5.npz")
    md = nova.ensight.mesh_desc(tuple(int(v) for v in g["N"]), L=tuple(g["L"]), walls=(0, 1, 0))
    nova.ensight.write_host(md, g["U"], str(tmp_path), "U", 7)
    back = nova.ensight.read_host(md, 3, str(tmp_path), "U", 7)
    assert np.array_equal(back, g["U"].astype(np.float32).astype(np.float64))


def test_bad_arguments_are_refused(nova, tmp_path):
    md = nova.ensight.mesh_desc((4, 4, 4))
    with pytest.raises(nova.NovaError):
        nova.ensight.read_host(md, 1, str(tmp_path), "missing", 1)
    with pytest.raises(nova.NovaError):
        nova.ensight.write_geometry(md, str(tmp_path / "no" / "such" / "dir"))
