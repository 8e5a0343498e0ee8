"""Output steps as legacy ASCII VTK files in the layouts MEGA writes
(MEGAOUT_####.vtk): the header (VTK_OUTPUT_HEADER), the current coordinates
as POINTS, one vertex cell per node (and the elements when a mesh is given),
POINT_DATA with one SCALARS block per component.  Two number formats, as the
reference has two writers:
  write_vtk               VTK_OUTPUT.F90: points in 3E13.5, scalars in E20.5
                          (five significant digits);
  write_vtk_list_directed VTK_OUTPUT_UNFORMATTED.F90 (UNF_OUTPUT_STEP_VTK):
                          every number in list-directed free format
                          (WRITE(unit,*)), 17 significant digits for doubles,
                          so the file keeps every double exactly.
The arrays come from one device-to-host copy (Mega.snapshot); this module
only formats them.
"""
import numpy as np

from taylor_b200 import _lib


def fortran_e(x, w, d):
    """Fortran Ew.d output of x: 0.<d digits>E+ee, right-justified in w
    (a three-digit exponent drops the E, as gfortran writes it)."""
    if x == 0.0 or not np.isfinite(x):
        if not np.isfinite(x):
            return ("NaN" if np.isnan(x) else ("-Infinity" if x < 0 else "Infinity")).rjust(w)
        return ("0." + "0" * d + "E+00").rjust(w)
    t = f"{abs(x):.{d - 1}e}"                     # d significant digits: m.mmmme+XX
    mant = t[0] + t[2:2 + d - 1]
    e = int(t[t.index("e") + 1:]) + 1             # 0.mmmmm x 10^e
    ex = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    return (("-" if x < 0 else "") + "0." + mant + ex).rjust(w)


def fortran_list_real(x):
    """One DOUBLE PRECISION item of gfortran list-directed output: a blank,
    then the value in G25.17E3 editing -- F20.(17-k) followed by five blanks
    when 0.1 <= |x| < 1e17 after rounding to 17 digits (k digits before the
    point; zero counts as k = 1), else 1PE25.16E3."""
    if not np.isfinite(x):
        return " " + ("NaN" if np.isnan(x) else ("-Infinity" if x < 0 else "Infinity")).rjust(25)
    d = 17
    sign = "-" if np.signbit(x) else ""
    if x == 0.0:
        return " " + (sign + "0." + "0" * (d - 1)).rjust(20) + " " * 5
    t = f"{abs(x):.{d - 1}e}"                     # d significant digits: m.mmm...e+XX
    e10 = int(t[t.index("e") + 1:])
    if -1 <= e10 < d:                             # F editing, d - k decimals
        k = e10 + 1
        return " " + (sign + f"{abs(x):.{d - k}f}").rjust(20) + " " * 5
    mant = t[:t.index("e")]
    ex = f"E{'+' if e10 >= 0 else '-'}{abs(e10):03d}"
    return " " + (sign + mant + ex).rjust(25)


def fortran_list_int(v):
    """One default INTEGER item of gfortran list-directed output: width 12."""
    return f"{int(v):12d}"


def _scalars(lines, name, values):
    lines.append("  ")                                     # START_DATA: WRITE(*,*) ' '
    lines.append("SCALARS " + name.rjust(30) + "double 1".rjust(10))
    lines.append("LOOKUP_TABLE default")
    lines.extend(fortran_e(v, 20, 5) for v in values)


# the reference's names for the fields this library holds (VTK_OUTPUT.F90:190-260)
FIELD_NAMES = {
    _lib.F_DSP_TOT: ("displacement_x", "displacement_y", "displacement_z"),
    _lib.F_VEL: ("velocity_x", "velocity_y", "velocity_z"),
    _lib.F_ACL: ("acceleration_x", "acceleration_y", "acceleration_z"),
    _lib.F_FINT: ("fint_x", "fint_y", "fint_z"),
    _lib.F_PRFORCE: ("pre_disp_force_x", "pre_disp_force_y", "pre_disp_force_z"),
    _lib.F_STRESS: ("stress_xx", "stress_yy", "stress_zz", "stress_yz", "stress_xz", "stress_xy"),
    _lib.F_STRAIN: ("strain_xx", "strain_yy", "strain_zz", "strain_yz", "strain_xz", "strain_xy"),
    _lib.F_EPS: ("eps",),
    _lib.F_WAVE_VEL: ("max_wave_vel",),
    _lib.F_STRAIN_EQ: ("strain_eq",),
}


def write_vtk(path, coo_current, data, elements=None):
    """coo_current (n, 3); data: ordered (name, values (n,)) pairs;
    elements (E, 8) 0-based hexes, written after the vertex cells as the
    reference does with LFEM_OUTPUT."""
    x = np.asarray(coo_current, np.float64).reshape(-1, 3)
    n = len(x)
    ne = 0 if elements is None else len(elements)
    lines = ["# vtk DataFile Version 2.0", "(MEGA VTK FILE)".rjust(30), "ASCII", "DATASET UNSTRUCTURED_GRID",
             "POINTS " + str(n).rjust(10) + "double".rjust(10)]
    lines.extend(fortran_e(a, 13, 5) + fortran_e(b, 13, 5) + fortran_e(c, 13, 5) for a, b, c in x)
    lines.append("  ")
    lines.append("CELLS " + str(n + ne).rjust(10) + str(2 * n + 9 * ne).rjust(20))
    lines.extend(f"{1:8d}{i:8d}" for i in range(n))
    if ne:
        lines.extend(f"{8:8d}" + "".join(f"{v:8d}" for v in el) for el in np.asarray(elements))
    lines.append("  ")
    lines.append("CELL_TYPES" + str(n + ne).rjust(8))
    lines.extend([f"{1:8d}"] * n)
    lines.extend([f"{12:8d}"] * ne)
    lines.append("  ")
    lines.append("  ")
    lines.append("POINT_DATA " + str(n).rjust(10))
    for name, values in data:
        _scalars(lines, name, np.asarray(values, np.float64).reshape(-1))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_vtk_list_directed(path, coo_current, data, elements=None):
    """The layout of UNF_OUTPUT_STEP_VTK (VTK_OUTPUT_UNFORMATTED.F90): as
    write_vtk, with every number written list-directed (fortran_list_real,
    fortran_list_int) -- points three per record, cells as (count, ids...),
    cell types and scalar values one per record."""
    x = np.asarray(coo_current, np.float64).reshape(-1, 3)
    n = len(x)
    ne = 0 if elements is None else len(elements)
    lines = ["# vtk DataFile Version 2.0", "(MEGA VTK FILE)".rjust(30), "ASCII", "DATASET UNSTRUCTURED_GRID",
             "POINTS " + str(n).rjust(10) + "double".rjust(10)]
    lines.extend(fortran_list_real(a) + fortran_list_real(b) + fortran_list_real(c) for a, b, c in x)
    lines.append("  ")
    lines.append("CELLS " + str(n + ne).rjust(10) + str(2 * n + 9 * ne).rjust(20))
    lines.extend(fortran_list_int(1) + fortran_list_int(i) for i in range(n))
    if ne:
        lines.extend(fortran_list_int(8) + "".join(fortran_list_int(v) for v in el) for el in np.asarray(elements))
    lines.append("  ")
    lines.append("CELL_TYPES" + str(n + ne).rjust(8))
    lines.extend([fortran_list_int(1)] * n)
    lines.extend([fortran_list_int(12)] * ne)
    lines.append("  ")
    lines.append("  ")
    lines.append("POINT_DATA " + str(n).rjust(10))
    for name, values in data:
        lines.append("  ")
        lines.append("SCALARS " + name.rjust(30) + "double 1".rjust(10))
        lines.append("LOOKUP_TABLE default")
        lines.extend(fortran_list_real(v) for v in np.asarray(values, np.float64).reshape(-1))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_output_step(m, path, fields=(_lib.F_DSP_TOT, _lib.F_VEL, _lib.F_STRESS, _lib.F_EPS), elements=None):
    """One output step of a resident context: the current coordinates and
    the given fields from a single device-to-host copy, written as VTK."""
    snap = m.snapshot((_lib.F_COO_CURRENT,) + tuple(fields))
    data = []
    for f in fields:
        a = snap[int(f)]
        a = a.reshape(m.n, -1)
        for k, name in enumerate(FIELD_NAMES[int(f)]):
            data.append((name, a[:, k]))
    write_vtk(path, snap[_lib.F_COO_CURRENT], data, elements)
    return snap
