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


def test_list_directed_format():
    from taylor_b200.vtk import fortran_list_int, fortran_list_real
    assert fortran_list_real(1.0) == "   1.0000000000000000     "
    assert fortran_list_real(0.1) == "  0.10000000000000001     "
    assert fortran_list_real(-2.5) == "  -2.5000000000000000     "
    assert fortran_list_real(123.456) == "   123.45600000000000     "
    assert fortran_list_real(1.0e-5) == "   1.0000000000000001E-005"
    assert fortran_list_real(-3.0e20) == "  -3.0000000000000000E+020"
    assert fortran_list_real(0.0) == "   0.0000000000000000     "
    assert fortran_list_int(12) == "          12"


def test_list_directed_file_keeps_every_double(tmp_path):
    """UNF_OUTPUT_STEP_VTK's layout; 17 significant digits read back to the
    same doubles."""
    from taylor_b200.vtk import write_vtk_list_directed
    rng = np.random.default_rng(2)
    x = rng.normal(scale=1e-3, size=(5, 3))
    s = rng.normal(scale=4e8, size=5)
    p = tmp_path / "MEGAOUT_0002.vtk"
    write_vtk_list_directed(p, x, [("stress_xx", s)], elements=np.array([[0, 1, 2, 3, 4, 0, 1, 2]]))
    lines = p.read_text().splitlines()
    assert lines[4].split() == ["POINTS", "5", "double"]
    pts = np.array([[float(v) for v in l.split()] for l in lines[5:10]])
    np.testing.assert_array_equal(pts, x)
    k = next(k for k, l in enumerate(lines) if l.startswith("POINT_DATA"))
    assert lines[k + 2].split() == ["SCALARS", "stress_xx", "double", "1"]
    np.testing.assert_array_equal([float(v) for v in lines[k + 4:k + 9]], s)
    c = next(k for k, l in enumerate(lines) if l.startswith("CELLS"))
    assert [int(v) for v in lines[c + 6].split()] == [8, 0, 1, 2, 3, 4, 0, 1, 2]
