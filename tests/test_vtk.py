"""The VTK writer against the layout of VTK_OUTPUT.F90 (header, points,
vertex cells, scalar blocks) and gfortran's E-format output."""
import numpy as np

from taylor_b200.vtk import fortran_e, write_vtk


def test_fortran_e_format():
    assert fortran_e(1.5, 13, 5) == "  0.15000E+01"
    assert fortran_e(-1.23456e-4, 13, 5) == " -0.12346E-03"
    assert fortran_e(0.0, 20, 5) == "         0.00000E+00"
    assert fortran_e(9.999996, 13, 5) == "  0.10000E+02"     # rounding carries into the exponent
    assert fortran_e(1.0e-120, 13, 5) == "  0.10000-119"     # three-digit exponents drop the E


def test_vtk_layout_round_trips(tmp_path):
    rng = np.random.default_rng(1)
    x = rng.normal(size=(7, 3))
    eps = rng.uniform(size=7)
    elems = np.array([[0, 1, 2, 3, 4, 5, 6, 0]])
    p = tmp_path / "MEGAOUT_0001.vtk"
    write_vtk(p, x, [("eps", eps), ("velocity_x", x[:, 0])], elements=elems)
    lines = p.read_text().splitlines()
    assert lines[0] == "# vtk DataFile Version 2.0"
    assert lines[2] == "ASCII" and lines[3] == "DATASET UNSTRUCTURED_GRID"
    assert lines[4].split() == ["POINTS", "7", "double"]
    pts = np.array([[float(l[13 * k:13 * (k + 1)]) for k in range(3)] for l in lines[5:12]])
    np.testing.assert_allclose(pts, x, rtol=6e-5)  # five significant digits
    i = lines.index("  ", 12) + 1
    assert lines[i].split() == ["CELLS", "8", str(2 * 7 + 9)]
    assert [int(v) for v in lines[i + 1].split()] == [1, 0]
    assert [int(v) for v in lines[i + 8].split()] == [8, 0, 1, 2, 3, 4, 5, 6, 0]
    j = next(k for k, l in enumerate(lines) if l.startswith("CELL_TYPES"))
    assert lines[j].split() == ["CELL_TYPES", "8"] and lines[j + 8].strip() == "12"
    k = next(k for k, l in enumerate(lines) if l.startswith("POINT_DATA"))
    assert lines[k].split() == ["POINT_DATA", "7"]
    assert lines[k + 2].split() == ["SCALARS", "eps", "double", "1"] and lines[k + 3] == "LOOKUP_TABLE default"
    np.testing.assert_allclose([float(v) for v in lines[k + 4:k + 11]], eps, rtol=6e-5)
    assert lines[k + 12].split()[1] == "velocity_x"
