"""Output steps as legacy ASCII VTK files in the layout VTK_OUTPUT.F90
writes (MEGAOUT_####.vtk): the header (VTK_OUTPUT_HEADER), the current
coordinates as POINTS (3E13.5), one vertex cell per node (and the hexes when
a mesh is given), POINT_DATA with one SCALARS block per component (E20.5),
as VTK_WRITE_DBL / VTK_WRITE_DBL_THREE lay them out.  The arrays come from
one device-to-host copy (Mega.snapshot); this module only formats them.
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
