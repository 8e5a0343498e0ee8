// mega_oracle.cpp -- CPU FP64 restatement of MEGA's explicit meshfree step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU library is
// checked against and the CPU baseline that bench.py times.  Nothing in the
// product (taylor_b200/, libmega_gpu.so) links or calls it.
//
// It restates, in C++, the Fortran subroutines of the reference
// (XieZhengTing/Taylor) that sit on the hot path.  Each function names the
// file:line it follows.  The reference cannot be compiled here (no Fortran
// compiler), so parity of this restatement against the reference binary is
// UNPINNED; it is pinned instead by the reference's own identity checks
// (TEST.F90 reproducing conditions and rigid rotation), which the tests run
// against it.
//
// Operation order follows the Fortran where it affects rounding: CSR order
// from BIN_INODE, summation order of the MATMULs, INV3 as written
// (det^2 * A^-1), single-precision literals 1.0E-05 and 1.0E-015 widened to
// double as gfortran does.  With nthreads == 1 the force assembly is the
// serial order; with nthreads > 1 it keeps the reference's per-thread
// FINT_TEMP(NCORES,3,N) buffers and their reduction (FINT.F90:233-240,
// 1238-1247), which is the cost structure the CPU baseline must keep.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../include/mega_gpu.h"

namespace {

typedef double M3[3][3];

// ---------------------------------------------------------------- helpers
// FINT_FUNCTIONS.F90:10-38  Voigt (xx,yy,zz,yz,xz,xy) -> symmetric tensor
inline void v2t(const double v[6], M3 t) {
  t[0][0] = v[0]; t[1][1] = v[1]; t[2][2] = v[2];
  t[2][1] = v[3]; t[1][2] = v[3];
  t[0][2] = v[4]; t[2][0] = v[4];
  t[0][1] = v[5]; t[1][0] = v[5];
}
// FINT_FUNCTIONS.F90:41-65
inline void t2v(const M3 t, double v[6]) {
  v[0] = t[0][0]; v[1] = t[1][1]; v[2] = t[2][2];
  v[3] = t[1][2]; v[4] = t[0][2]; v[5] = t[0][1];
}
// FINT_FUNCTIONS.F90:94-114 (engineering shear counted twice)
inline double tensor_norm(const double v[6]) {
  double s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] +
             2.0 * (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
  return std::sqrt(s);
}
// FINT_FUNCTIONS.F90:69-92
inline double tensor_norm_strain(const double v[6]) {
  double s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] +
             (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
  return std::sqrt(s);
}
// FINT_FUNCTIONS.F90:138-165
inline void dev_proj(const double v[6], double o[6]) {
  double kk = v[0] + v[1] + v[2];
  o[0] = v[0] - kk / 3.0; o[1] = v[1] - kk / 3.0; o[2] = v[2] - kk / 3.0;
  o[3] = v[3]; o[4] = v[4]; o[5] = v[5];
}
// FINT_FUNCTIONS.F90:168-195 -- note the sign: returns -tr/3
inline void sphr_proj(const double v[6], double o[6]) {
  double kk = v[0] + v[1] + v[2];
  o[0] = -kk / 3.0; o[1] = -kk / 3.0; o[2] = -kk / 3.0;
  o[3] = 0.0; o[4] = 0.0; o[5] = 0.0;
}
inline double bulk_mod(double e, double nu) { return e / (3.0 * (1.0 - 2.0 * nu)); }   // :197-211
inline double shear_mod(double e, double nu) { return e / (2.0 * (1.0 + nu)); }        // :215-229

// MATMUL for 3x3 (k ascending)
inline void mm3(const M3 a, const M3 b, M3 c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      c[i][j] = s;
    }
}

// INVERSE.F90:119-152 -- INV3 exactly as written: the adjugate is MULTIPLIED
// by the determinant, so it returns det(A)^2 * A^-1.  exact != 0 divides.
inline void inv3(const M3 a, M3 r, bool exact) {
  double det = a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1] -
               a[0][1] * a[1][0] * a[2][2] + a[0][1] * a[1][2] * a[2][0] +
               a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
  double c[3][3];
  c[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  c[1][0] = -(a[1][0] * a[2][2] - a[1][2] * a[2][0]);
  c[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  c[0][1] = -(a[0][1] * a[2][2] - a[0][2] * a[2][1]);
  c[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
  c[2][1] = -(a[0][0] * a[2][1] - a[0][1] * a[2][0]);
  c[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
  c[1][2] = -(a[0][0] * a[1][2] - a[0][2] * a[1][0]);
  c[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = exact ? c[i][j] / det : c[i][j] * det;
}

// DETERMINANT.F90:18-35 (absolute value)
inline double det_abs(const M3 a) {
  return std::fabs(a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) +
                   a[0][1] * (a[2][0] * a[1][2] - a[1][0] * a[2][2]) +
                   a[0][2] * (a[1][0] * a[2][1] - a[2][0] * a[1][1]));
}

// INVERSE.F90:17-99 -- Gauss-Jordan with full pivoting, n x n, A(i,j) at
// a[i*n+j].  Returns false where the reference sets L=0 (pivot negligible).
bool inverse_gj(const double* a, int n, double* r) {
  int is[16], js[16];
  for (int i = 0; i < n * n; ++i) r[i] = a[i];
  for (int k = 0; k < n; ++k) {
    double d = 0.0;
    for (int i = k; i < n; ++i)
      for (int j = k; j < n; ++j)
        if (std::fabs(r[i * n + j]) > d) { d = std::fabs(r[i * n + j]); is[k] = i; js[k] = j; }
    if (d + 1.0 == 1.0) return false;
    for (int j = 0; j < n; ++j) std::swap(r[k * n + j], r[is[k] * n + j]);
    for (int i = 0; i < n; ++i) std::swap(r[i * n + k], r[i * n + js[k]]);
    r[k * n + k] = 1.0 / r[k * n + k];
    for (int j = 0; j < n; ++j) if (j != k) r[k * n + j] = r[k * n + j] * r[k * n + k];
    for (int i = 0; i < n; ++i)
      if (i != k)
        for (int j = 0; j < n; ++j)
          if (j != k) r[i * n + j] = r[i * n + j] - r[i * n + k] * r[k * n + j];
    for (int i = 0; i < n; ++i) if (i != k) r[i * n + k] = -r[i * n + k] * r[k * n + k];
  }
  for (int k = n - 1; k >= 0; --k) {
    for (int j = 0; j < n; ++j) std::swap(r[k * n + j], r[js[k] * n + j]);
    for (int i = 0; i < n; ++i) std::swap(r[i * n + k], r[i * n + is[k]]);
  }
  return true;
}

// 3x3 determinant of rows (r0, r1, r2) expanded on the first row
inline double det3r(const double* r0, const double* r1, const double* r2) {
  return r0[0] * (r1[1] * r2[2] - r1[2] * r2[1]) + r0[1] * (r1[2] * r2[0] - r1[0] * r2[2]) +
         r0[2] * (r1[0] * r2[1] - r1[1] * r2[0]);
}

// INVERSE.F90:185-223 -- M44INV: cofactor expansion, AINV = COF^T / DET.
// Returns the determinant.
double m44inv(const double a[4][4], double r[4][4]) {
  double cof[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double m[3][3];
      int ri = 0;
      for (int p = 0; p < 4; ++p) {
        if (p == i) continue;
        int cj = 0;
        for (int q = 0; q < 4; ++q) {
          if (q == j) continue;
          m[ri][cj++] = a[p][q];
        }
        ++ri;
      }
      double d = det3r(m[0], m[1], m[2]);
      cof[i][j] = ((i + j) & 1) ? -d : d;
    }
  double det = a[0][0] * cof[0][0] + a[0][1] * cof[0][1] + a[0][2] * cof[0][2] + a[0][3] * cof[0][3];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r[i][j] = cof[j][i] / det;
  return det;
}

// KERNEL.F90:57-71 -- cubic B-spline (ISPLINE = 3) and its derivative.
inline void mls_kernel0(double xsa, double& phi, double& phix) {
  if (xsa <= 0.5) {
    phi = 2.0 / 3.0 - 4.0 * xsa * xsa + 4.0 * xsa * xsa * xsa;
    phix = -8.0 * xsa + 12.0 * xsa * xsa;
  } else if (xsa <= 1.0) {
    phi = 4.0 / 3.0 - 4.0 * xsa + 4.0 * xsa * xsa - 4.0 / 3.0 * xsa * xsa * xsa;
    phix = -4.0 + 8.0 * xsa - 4.0 * xsa * xsa;
  } else {
    phi = 0.0;
    phix = 0.0;
  }
}

// single-precision literals of the reference, widened as gfortran widens them
const double kTolVM = (double)1.0e-5f;    // CONSTITUTE_VONMISES.F90:109  1.0E-05
const double kEpsSK = (double)1.0e-15f;   // RK.f90:219  1.0E-015

// --------------------------------------------------------- RK shape build
// RK.f90:16-453 (RK1), DEG = 1 (MSIZE = 4).  x = evaluation point, nb[ln]
// are 0-based neighbour ids.  shp[ln], shpd[3*ln] (AoS).  Returns false when
// the moment matrix is singular.
bool rk1(const double x[3], const double* gcoo, const double* gwin, const int* nb, int ln,
         const int32_t* ebcs, bool ql, double ql_coef, double ql_len, bool shsup,
         double* shp, double* shpd, std::vector<double>& work) {
  work.resize((size_t)ln * 4);
  double* PHI = work.data();
  double* PX = PHI + ln;
  double* PY = PX + ln;
  double* PZ = PY + ln;
  double phi_sum = 0.0;
  double M[4][4] = {}, Mx[4][4] = {}, My[4][4] = {}, Mz[4][4] = {};
  const double Hx[4] = {0, 1, 0, 0}, Hy[4] = {0, 0, 1, 0}, Hz[4] = {0, 0, 0, 1};
  for (int i = 0; i < ln; ++i) {
    int ii = nb[i];
    const double* xj = gcoo + 3 * (size_t)ii;
    const double* aj = gwin + 3 * (size_t)ii;
    double dx = x[0] - xj[0], dy = x[1] - xj[1], dz = x[2] - xj[2];
    double H[4] = {1.0, dx, dy, dz};                                  // FILL_H RK.f90:474-479
    double nx = dx / aj[0], ny = dy / aj[1], nz = dz / aj[2];          // RK.f90:132-134
    double phi, phx, phy, phz;
    if (shsup) {                                                      // RK.f90:136-166
      double dia = std::sqrt(nx * nx + ny * ny + nz * nz);
      double k, kx;
      mls_kernel0(dia, k, kx);
      double drdx, drdy, drdz;
      if (dia <= 1.0e-13) { drdx = drdy = drdz = 0.0; }
      else {
        drdx = dx / (aj[0] * aj[0]) / dia;
        drdy = dy / (aj[1] * aj[1]) / dia;
        drdz = dz / (aj[2] * aj[2]) / dia;
      }
      phi = k; phx = kx * drdx; phy = kx * drdy; phz = kx * drdz;
    } else {                                                          // RK.f90:168-230
      double kx, kxx, ky, kyy, kz, kzz;
      mls_kernel0(std::fabs(nx), kx, kxx);
      mls_kernel0(std::fabs(ny), ky, kyy);
      mls_kernel0(std::fabs(nz), kz, kzz);
      phi = kx * ky * kz;
      // RK.f90:183-205: every axis uses GWIN(1,II) (quirk kept)
      double drdx = (nx == 0.0) ? 0.0 : (nx >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
      double drdy = (ny == 0.0) ? 0.0 : (ny >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
      double drdz = (nz == 0.0) ? 0.0 : (nz >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
      phx = kxx * ky * kz * drdx;
      phy = kx * kyy * kz * drdy;
      phz = kx * ky * kzz * drdz;
      if (ebcs && ebcs[ii]) {                                         // RK.f90:217-228 singular kernel
        double wm = 1.0 / (std::sqrt(nx * nx + ny * ny + nz * nz) + kEpsSK);
        phx = phx * wm - phi * wm * wm * wm * nx / aj[0];
        phy = phy * wm - phi * wm * wm * wm * ny / aj[1];
        phz = phz * wm - phi * wm * wm * wm * nz / aj[2];
        phi = phi * wm;
      }
    }
    phi_sum += phi;
    PHI[i] = phi; PX[i] = phx; PY[i] = phy; PZ[i] = phz;
    for (int j = 0; j < 4; ++j)                                       // RK.f90:231-242
      for (int k = 0; k < 4; ++k) {
        M[j][k] += H[j] * H[k] * phi;
        Mx[j][k] += Hx[j] * H[k] * phi + H[j] * Hx[k] * phi + H[j] * H[k] * phx;
        My[j][k] += Hy[j] * H[k] * phi + H[j] * Hy[k] * phi + H[j] * H[k] * phy;
        Mz[j][k] += Hz[j] * H[k] * phi + H[j] * Hz[k] * phi + H[j] * H[k] * phz;
      }
  }
  double qlp[6][3];
  if (ql) {                                                           // RK.f90:251-303
    for (int m = 0; m < 6; ++m) { qlp[m][0] = x[0]; qlp[m][1] = x[1]; qlp[m][2] = x[2]; }
    qlp[0][0] = x[0] + ql_len; qlp[1][0] = x[0] - ql_len;
    qlp[2][1] = x[1] + ql_len; qlp[3][1] = x[1] - ql_len;
    qlp[4][2] = x[2] + ql_len; qlp[5][2] = x[2] - ql_len;
    double Ms[4][4] = {};
    for (int m = 0; m < 6; ++m) {
      double H[4] = {1.0, x[0] - qlp[m][0], x[1] - qlp[m][1], x[2] - qlp[m][2]};
      for (int j = 0; j < 4; ++j)
        for (int k = 0; k < 4; ++k) Ms[j][k] += H[j] * H[k];
    }
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) M[j][k] = M[j][k] + Ms[j][k] * phi_sum * ql_coef;
  }
  double Mi[4][4];
  double det = m44inv(M, Mi);                                         // RK.f90:305-309
  bool ok = std::isfinite(det) && det != 0.0;
  double B[4], BX[4], BY[4], BZ[4];
  for (int k = 0; k < 4; ++k) B[k] = Mi[0][k];                        // RK.f90:311-314
  // RK.f90:332-342: BX = H0 * ((-MINV * M_X) * MINV)
  auto dbx = [&](const double Md[4][4], double out[4]) {
    double t[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double s = 0.0;
        for (int k = 0; k < 4; ++k) s += (-Mi[i][k]) * Md[k][j];
        t[i][j] = s;
      }
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += t[0][k] * Mi[k][j];
      out[j] = s;
    }
  };
  dbx(Mx, BX); dbx(My, BY); dbx(Mz, BZ);
  double Hs[4] = {0, 0, 0, 0};
  if (ql) {                                                           // RK.f90:357-377
    for (int m = 0; m < 6; ++m) {
      Hs[0] += 1.0;
      Hs[1] += x[0] - qlp[m][0];
      Hs[2] += x[1] - qlp[m][1];
      Hs[3] += x[2] - qlp[m][2];
    }
  }
  for (int i = 0; i < ln; ++i) {                                      // RK.f90:346-405
    int ii = nb[i];
    const double* xj = gcoo + 3 * (size_t)ii;
    double H[4] = {1.0, x[0] - xj[0], x[1] - xj[1], x[2] - xj[2]};
    if (ql) for (int k = 0; k < 4; ++k) H[k] = H[k] + Hs[k] * ql_coef;
    double C = 0.0, CX = 0.0, CY = 0.0, CZ = 0.0, bhx = 0.0, bhy = 0.0, bhz = 0.0;
    for (int k = 0; k < 4; ++k) C += B[k] * H[k];
    for (int k = 0; k < 4; ++k) CX += BX[k] * H[k];
    for (int k = 0; k < 4; ++k) bhx += B[k] * Hx[k];
    for (int k = 0; k < 4; ++k) CY += BY[k] * H[k];
    for (int k = 0; k < 4; ++k) bhy += B[k] * Hy[k];
    for (int k = 0; k < 4; ++k) CZ += BZ[k] * H[k];
    for (int k = 0; k < 4; ++k) bhz += B[k] * Hz[k];
    CX = CX + bhx; CY = CY + bhy; CZ = CZ + bhz;
    shp[i] = C * PHI[i];
    shpd[3 * i + 0] = CX * PHI[i] + C * PX[i];
    shpd[3 * i + 1] = CY * PHI[i] + C * PY[i];
    shpd[3 * i + 2] = CZ * PHI[i] + C * PZ[i];
  }
  return ok;
}

// ------------------------------------------------- objective rotation (HW)
// HUGHES_WINGET.F90:16-81
void hughes_winget(const M3 L, M3 rot, double strain[6], double d[6], bool exact) {
  M3 A, Ai, G, W, IW, IWi, E;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = (i == j ? 1.0 : 0.0) + 0.5 * L[i][j];
  inv3(A, Ai, exact);
  mm3(L, Ai, G);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) W[i][j] = 0.5 * (G[i][j] - G[j][i]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) IW[i][j] = (i == j ? 1.0 : 0.0) - 0.5 * W[i][j];
  inv3(IW, IWi, exact);
  M3 t;
  mm3(IWi, W, t);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rot[i][j] = (i == j ? 1.0 : 0.0) + t[i][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) E[i][j] = 0.5 * (G[i][j] + G[j][i]);
  t2v(E, strain);
  for (int k = 0; k < 6; ++k) d[k] = strain[k];
  strain[3] = 2.0 * strain[3]; strain[4] = 2.0 * strain[4]; strain[5] = 2.0 * strain[5];
}

// ROTATE_TENSOR.F90:21-87
void rotate_tensor(const M3 rot, double v[6]) {
  M3 T, tmp, rt, out;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rt[i][j] = rot[j][i];
  v2t(v, T);
  mm3(rot, T, tmp);
  mm3(tmp, rt, out);
  t2v(out, v);
}

// ------------------------------------------------------- constitutive laws
// CONSTITUTE_VONMISES.F90:21-158.  Returns Newton passes (0 = elastic);
// *capped set when the 20-iteration cap is reached.
int von_mises(double stress[6], const double spred[6], double state[20], const double* props,
              int maxit, bool* capped) {
  double poiss = props[0], young = props[1], sig0 = props[3];
  double mu = shear_mod(young, poiss);
  double B = props[4], CE = props[5];
  double eps = state[2];
  double dev[6], sph[6];
  dev_proj(spred, dev);
  sphr_proj(spred, sph);
  double tn = tensor_norm(dev);
  double sig23 = std::sqrt(2.0 / 3.0) * sig0;
  double xk = sig23 * std::pow(1.0 + B * eps, CE);
  double yld = tn - xk;
  int iters = 0;
  if (yld > 0.0) {
    double dg = 0.0, epst = eps;
    for (int i = 1; i <= maxit; ++i) {
      ++iters;
      xk = sig23 * std::pow(1.0 + B * eps, CE);
      yld = tn - xk - (2.0 * mu * dg);
      if (std::fabs(yld) > sig23 * kTolVM) {
        double xkp = B * CE * sig0 * std::pow(1.0 + B * eps, CE - 1.0);
        double dyld = -2.0 * mu * (1.0 + xkp / 3.0 / mu);
        dg = dg - yld / dyld;
        if (i == maxit && capped) *capped = true;
      } else {
        eps = epst + std::sqrt(2.0 / 3.0) * dg;
        break;
      }
      eps = epst + std::sqrt(2.0 / 3.0) * dg;
    }
    for (int k = 0; k < 6; ++k) dev[k] = dev[k] - dg * 2.0 * mu * dev[k] / tn;
  }
  state[2] = eps;
  for (int k = 0; k < 6; ++k) stress[k] = -sph[k] + dev[k];
  return iters;
}

// Power-law rate-dependent J2 (no reference counterpart; new physics of the
// learned-guess configuration).  sigma_y(ep, epdot) = A + B*ep^n*(1 + C*ln(
// max(epdot, epdot0)/epdot0)), epdot = sqrt(2/3)*dgamma/dt.  Radial return
// (Simo & Hughes, Computational Inelasticity, box 3.1) solved by Newton on
// dgamma, safeguarded by bisection on the bracket [0, q_tr/(2 mu)], to
// |f| <= rtol * sqrt(2/3)*sigma_y.  Starts from dg0 (< 0: the elastic-
// perfectly-plastic guess f_tr / (2 mu)).  Returns Newton passes.
int vm_rate(double stress[6], const double spred[6], double state[20], const double* props,
            double dt, double rtol, int maxit, int solver, double dg0, bool* capped, double* dg_out) {
  double poiss = props[0], young = props[1];
  double A = props[3], Bh = props[4], n = props[5], C = props[6], ed0 = props[7];
  double mu = shear_mod(young, poiss);
  double eps0 = state[2];
  double dev[6], sph[6];
  dev_proj(spred, dev);
  sphr_proj(spred, sph);
  double tn = tensor_norm(dev);
  const double s23 = std::sqrt(2.0 / 3.0);
  auto sigy = [&](double dg, double* dsig) {
    double ep = eps0 + s23 * dg;
    double ed = s23 * dg / dt;
    double rate = 1.0, drate = 0.0;
    if (ed > ed0) { rate = 1.0 + C * std::log(ed / ed0); drate = C / dg; }
    double epn = (ep > 0.0) ? std::pow(ep, n) : 0.0;
    double depn = (ep > 0.0) ? n * std::pow(ep, n - 1.0) * s23 : 0.0;
    *dsig = Bh * (depn * rate + epn * drate);
    return A + Bh * epn * rate;
  };
  double d0;
  double f0 = tn - s23 * sigy(0.0, &d0);
  int iters = 0;
  double dg = 0.0;
  if (f0 > 0.0) {
    // f(dg) = tn - 2 mu dg - sqrt(2/3) sy(dg) decreases in dg.  Two upper
    // bounds of the root (sy >= A + B (eps0 + sqrt(2/3) dg)^n because the
    // rate factor is >= 1, and 2 mu dg >= 0): the perfectly plastic
    // multiplier and the pure power-law one; start at the smaller.
    // solver 1 (textbook, for comparison): Newton in dg from the perfectly
    // plastic estimate, bracket [0, tn / (2 mu)], arithmetic bisection.
    const bool textbook = solver == 1;
    double hi = f0 / (2.0 * mu);
    if (Bh > 0.0) {
      const double epn0 = (eps0 > 0.0) ? std::pow(eps0, n) : 0.0;
      const double pw = (std::pow(epn0 + f0 / (s23 * Bh), 1.0 / n) - eps0) / s23;
      if (pw > 0.0 && pw < hi) hi = pw;
    }
    if (textbook) hi = tn / (2.0 * mu);
    double lo = 0.0;
    dg = (dg0 >= 0.0) ? dg0 : (textbook ? f0 / (2.0 * mu) : hi);
    if (textbook ? !(dg > lo && dg < hi) : !(dg > lo && dg <= hi)) dg = textbook ? 0.5 * (lo + hi) : hi;
    // Newton in y = ln(dg): f is concave in y, so from the right of the root
    // the iterates decrease monotonically onto it; dg > 0 always.  The
    // bracket guards the start from the left; outside it, bisect in y.
    bool conv = false;
    if (textbook) {
      for (int i = 1; i <= maxit; ++i) {
        ++iters;
        double ds;
        double sy = sigy(dg, &ds);
        double f = tn - 2.0 * mu * dg - s23 * sy;
        if (std::fabs(f) <= rtol * s23 * sy) { conv = true; break; }
        if (f > 0.0) lo = dg; else hi = dg;
        double df = -2.0 * mu - s23 * ds;
        double nd = dg - f / df;
        if (!(nd > lo && nd < hi) || !std::isfinite(nd)) nd = 0.5 * (lo + hi);
        const bool stalled = std::fabs(nd - dg) <= 4.0e-16 * dg;  // below the rounding of dg
        dg = nd;
        if (stalled) { conv = true; break; }
      }
    } else {
      // the iterate is y = ln(dg); ln(epsdot / epsdot0) = y - ythr, and
      // eps^n = exp(n ln eps)
      const double ythr = std::log(ed0 * dt / s23);
      double y = std::log(dg), ylo = -INFINITY, yhi = std::log(hi);
      for (int i = 1; i <= maxit; ++i) {
        ++iters;
        const double ep = eps0 + s23 * dg;
        const double epn = std::exp(n * std::log(ep));
        const double depn = n * epn / ep * s23;
        double rate = 1.0, drate = 0.0;
        if (y > ythr) { rate = 1.0 + C * (y - ythr); drate = C / dg; }
        const double sy = A + Bh * epn * rate;
        const double f = tn - 2.0 * mu * dg - s23 * sy;
        if (std::fabs(f) <= rtol * s23 * sy) { conv = true; break; }
        if (f > 0.0) ylo = y; else yhi = y;
        const double df = -2.0 * mu - s23 * Bh * (depn * rate + epn * drate);
        double yn = y + std::fmax(std::fmin(-f / (df * dg), 50.0), -50.0);
        if (!(yn > ylo && yn < yhi) || !std::isfinite(yn))
          yn = std::isfinite(ylo) ? 0.5 * (ylo + yhi) : yhi - 0.69314718055994530942;  // bisect in y
        const bool stalled = std::fabs(yn - y) <= 4.0e-16;  // below the rounding of dg
        y = yn;
        dg = std::exp(y);
        if (stalled) { conv = true; break; }
      }
    }
    if (!conv && capped) *capped = true;
    for (int k = 0; k < 6; ++k) dev[k] = dev[k] - dg * 2.0 * mu * dev[k] / tn;
    state[2] = eps0 + s23 * dg;
  }
  if (dg_out) *dg_out = dg;
  for (int k = 0; k < 6; ++k) stress[k] = -sph[k] + dev[k];
  return iters;
}

// ESTIMATE_MODULI.F90:16-86 (NSNI_FLAG = .FALSE.)
void estimate_moduli(const double sinc[6], const double einc[6], double& shear, double& bulk) {
  double sd[6], ss[6], ed[6], es[6];
  dev_proj(sinc, sd); sphr_proj(sinc, ss);
  dev_proj(einc, ed); sphr_proj(einc, es);
  double nsd = tensor_norm(sd), nss = tensor_norm(ss);
  double ned = tensor_norm_strain(ed), nes = tensor_norm_strain(es);
  double st = (ned > 1.0e-8 && nsd > 1.0e-8) ? nsd / ned / 2.0 : shear;
  st = std::max(st, shear * 0.5);
  st = std::min(st, shear);
  shear = st;
  double bt = (nes > 1.0e-8 && nss > 1.0e-8) ? nss / nes / 3.0 : bulk;
  bt = std::max(bt, bulk * 0.5);
  bt = std::min(bt, bulk);
  bulk = bt;
}

// ESTIMATE_MODULI with NSNI_FLAG = .TRUE. (no clamp to half the elastic
// moduli), then capped at the elastic moduli.
void estimate_moduli_nsni(const double sinc[6], const double einc[6], double& shear, double& bulk) {
  double sd[6], ss[6], ed[6], es[6];
  dev_proj(sinc, sd); sphr_proj(sinc, ss);
  dev_proj(einc, ed); sphr_proj(einc, es);
  double nsd = tensor_norm(sd), nss = tensor_norm(ss);
  double ned = tensor_norm_strain(ed), nes = tensor_norm_strain(es);
  if (ned > 1.0e-8 && nsd > 1.0e-8) shear = std::min(nsd / ned / 2.0, shear);
  if (nes > 1.0e-8 && nss > 1.0e-8) bulk = std::min(nss / nes / 3.0, bulk);
}

// Damage shared by both damaged models (CONSTITUTE_VONMISES_DAM.F90:94-125,
// CONSTITUTE_DRUCKPRAG.F90:84-113): eta = TENSOR_NORM(total strain) (the
// stress norm, as written); between K_I and K_C the damage follows
// K_C (eta - K_I) / (eta (K_C - K_I)), capped at DAM_MAX.
static void damage_update(const double total_strain[6], double k_i, double k_c, double dam_max, double& dam,
                          double& dam_sv) {
  const double eta = tensor_norm(total_strain);
  const double k_i_check = dam_sv + k_i;
  if (eta < k_i_check) {
  } else if (eta > k_i && eta < k_c) {
    dam = k_c * (eta - k_i) / (eta * (k_c - k_i));
    dam_sv = eta;
    dam_sv = dam_sv - k_i;
  }
  if (dam > dam_max) dam = dam_max;
}

// effective predictor STRESS / (1 - DAM) + MATMUL(ELAS_MAT, INC_STRAIN)
static void effective_predictor(const double stress[6], double dam, const double* props, const double inc[6],
                                double eff[6]) {
  double lam = props[27], mu = props[28], l2m = props[29];
  double C[6][6] = {};
  C[0][0] = C[1][1] = C[2][2] = l2m;
  C[3][3] = C[4][4] = C[5][5] = mu;
  C[0][1] = C[1][0] = C[0][2] = C[2][0] = C[2][1] = C[1][2] = lam;
  for (int r = 0; r < 6; ++r) {
    double v = 0.0;
    for (int c = 0; c < 6; ++c) v += C[r][c] * inc[c];
    eff[r] = stress[r] / (1.0 - dam) + v;
  }
}

// VON_MISES_DAM (CONSTITUTE_VONMISES_DAM.F90:21-196): J2 with the power
// hardening of VON_MISES in effective-stress space, isotropic damage.
// stress: the rotated old stress in, the new stress out.
int von_mises_dam(double stress[6], const double total_strain[6], const double inc[6], double state[20],
                  const double* props, int maxit, bool* capped) {
  const double poiss = props[0], young = props[1], sig0 = props[3], B = props[4], ce = props[5];
  const double k_i = props[8], k_c = props[9], dam_max = props[10];
  const double mu = shear_mod(young, poiss);
  double eps = state[2], dam = state[3], dam_sv = state[4];
  double eff[6], dev[6], sph[6];
  effective_predictor(stress, dam, props, inc, eff);
  dev_proj(eff, dev);
  damage_update(total_strain, k_i, k_c, dam_max, dam, dam_sv);
  sphr_proj(eff, sph);
  const double tn = tensor_norm(dev);
  const double s23 = std::sqrt(2.0 / 3.0);
  const double sig23 = s23 * sig0;
  double xk = sig23 * std::pow(1.0 + B * eps, ce);
  double yld = tn - xk;
  int it = 0;
  if (yld > 0.0) {
    double dg = 0.0;
    const double epst = eps;
    for (int i = 1; i <= maxit; ++i) {
      ++it;
      xk = sig23 * std::pow(1.0 + B * eps, ce);
      yld = tn - xk - (2.0 * mu * dg);
      if (std::fabs(yld) > sig23 * (double)1.0e-5f) {
        const double xkp = B * ce * sig0 * std::pow(1.0 + B * eps, ce - 1.0);
        const double dy = -2.0 * mu * (1.0 + xkp / 3.0 / mu);
        dg = dg - yld / dy;
        if (i == maxit && capped) *capped = true;
      } else {
        eps = epst + s23 * dg;
        break;
      }
      eps = epst + s23 * dg;
    }
    for (int k = 0; k < 6; ++k) dev[k] = dev[k] - dg * 2.0 * mu * dev[k] / tn;
  }
  state[2] = eps;
  state[3] = dam;
  state[4] = dam_sv;
  for (int k = 0; k < 6; ++k) stress[k] = (-sph[k] + dev[k]) * (1.0 - dam);
  return it;
}

// DRUCK_PRAG (CONSTITUTE_DRUCKPRAG.F90:17-241): Drucker-Prager shear yield
// with non-associated flow and isotropic damage in effective-stress space.
// The tension branch is unreachable as written (its flag is never set) and
// is not restated.  stress: the rotated old stress in, the new stress out.
int druck_prag(double stress[6], const double total_strain[6], const double inc[6], double state[20],
               const double* props) {
  const double poiss = props[0], young = props[1];
  const double q_phi = props[24], k_phi = props[25], q_psi = props[26];
  const double k_i = props[8], k_c = props[9], dam_max = props[10];
  double eps_shear = state[0], eps_vol = state[1], eps = state[2], dam = state[3], dam_sv = state[4];
  double eff[6], dev[6];
  effective_predictor(stress, dam, props, inc, eff);
  damage_update(total_strain, k_i, k_c, dam_max, dam, dam_sv);
  dev_proj(eff, dev);
  const double tau_pre = tensor_norm(dev);
  const double sph_pre = (eff[0] + eff[1] + eff[2]) / 3.0;
  const double f_shear = tau_pre + q_phi * sph_pre - k_phi;
  int plastic = 0;
  if (f_shear < 0.0) {
    for (int k = 0; k < 6; ++k) stress[k] = eff[k];
  } else {
    plastic = 1;
    const double tau = k_phi - q_phi * sph_pre;
    const double bulk = bulk_mod(young, poiss), shear = shear_mod(young, poiss);
    const double gamma = f_shear / (2.0 * shear + bulk * q_phi * q_psi);
    const double sph = sph_pre - bulk * q_psi * gamma;
    for (int k = 0; k < 6; ++k) stress[k] = dev[k] * tau / tau_pre;
    stress[0] += sph; stress[1] += sph; stress[2] += sph;
    eps_shear = eps_shear + gamma * std::sqrt(2.0 / 3.0 + 2.0 / 9.0 * q_psi * q_psi);
    eps = eps + eps_shear;
  }
  for (int k = 0; k < 6; ++k) stress[k] = stress[k] * (1.0 - dam);
  state[0] = eps_shear;
  state[1] = eps_vol;
  state[2] = eps;
  state[3] = dam;
  state[4] = dam_sv;
  return plastic;  // a closed-form return counts as one pass
}

// CONSTITUTION.F90:46-85 dispatch.  status bits as in mega_gpu.h.  The
// damaged models (3, 6) also need the rotated old stress (in stress), the
// total and the incremental strain; without them they are rejected.
int constitution(const double spred[6], int mat, const double* props, double dlt, double state[20],
                 double stress[6], int maxit, double rtol, int* status, int* iters_out, int solver = 0,
                 const double* total_strain = nullptr, const double* inc_strain = nullptr) {
  int it = 0;
  bool capped = false;
  switch (mat) {
    case MEGA_MAT_ELASTIC:
      for (int k = 0; k < 6; ++k) stress[k] = spred[k];
      break;
    case MEGA_MAT_VONMISES:
      it = von_mises(stress, spred, state, props, maxit, &capped);
      break;
    case MEGA_MAT_VM_RATE:
      it = vm_rate(stress, spred, state, props, dlt, rtol, maxit, solver, -1.0, &capped, nullptr);
      break;
    case MEGA_MAT_DRUCKER_PRAGER:
      if (!total_strain || !inc_strain) { *status |= MEGA_ST_BAD_MATERIAL; break; }
      it = druck_prag(stress, total_strain, inc_strain, state, props);
      break;
    case MEGA_MAT_VM_DAMAGE:
      if (!total_strain || !inc_strain) { *status |= MEGA_ST_BAD_MATERIAL; break; }
      it = von_mises_dam(stress, total_strain, inc_strain, state, props, maxit, &capped);
      break;
    default:
      *status |= MEGA_ST_BAD_MATERIAL;
      for (int k = 0; k < 6; ++k) stress[k] = spred[k];
  }
  if (capped) *status |= MEGA_ST_NEWTON_CAP;
  if (iters_out) *iters_out = it;
  return it;
}

}  // namespace

// ============================================================ exported API
extern "C" {

// Bin geometry of HANDELER.F90:187-243 and GET_BINS/SOFT_SEARCH of
// BIN_SEARCH.F90:2-64, 69-133, 153-328.  gstart/gstack are 1-based.
// Returns a MEGA_ST_* bitmask.
int orc_bin_search(int n, const double* coo, const double* win, const double* sm_len,
                   const double* dist_max, int itype_int, int shsup, int* gn, int* gstart,
                   int* gstack, int64_t cap, int64_t* nnz_out, int* gmaxn, int* ijk,
                   double* geom_out /* xmin,ymin,zmin,xbin,ybin,zbin,nx,ny,nz */,
                   const double* geom_in /* the same, kept from LINIT (semi-Lagrangian re-search) or null */) {
  if (n <= 0) return 0;
  double xbin = 0, ybin = 0, zbin = 0;
  double xmax = coo[0], ymax = coo[1], zmax = coo[2];
  double xmin = coo[0], ymin = coo[1], zmin = coo[2];
  for (int i = 0; i < n; ++i) {                                       // HANDELER.F90:200-219
    const double* w = win + 3 * (size_t)i;
    const double* x = coo + 3 * (size_t)i;
    if (w[0] > xbin) xbin = w[0];
    if (w[1] > ybin) ybin = w[1];
    if (w[2] > zbin) zbin = w[2];
    if (w[0] + dist_max[0] > xbin) xbin = w[0] + dist_max[0];
    if (w[1] + dist_max[1] > ybin) ybin = w[1] + dist_max[1];
    if (w[2] + dist_max[2] > zbin) zbin = w[2] + dist_max[2];
    if (x[0] > xmax) xmax = x[0];
    if (x[1] > ymax) ymax = x[1];
    if (x[2] > zmax) zmax = x[2];
    if (x[0] < xmin) xmin = x[0];
    if (x[1] < ymin) ymin = x[1];
    if (x[2] < zmin) zmin = x[2];
  }
  xmin = xmin - xbin * 10.0; ymin = ymin - ybin * 10.0; zmin = zmin - zbin * 10.0;   // :226-232
  xmax = xmax + xbin * 10.0; ymax = ymax + ybin * 10.0; zmax = zmax + zbin * 10.0;
  int nx = (int)std::ceil((xmax - xmin) / xbin);                      // :235-241
  int ny = (int)std::ceil((ymax - ymin) / ybin);
  int nz = (int)std::ceil((zmax - zmin) / zbin);
  if (geom_in) {  // the bins of HANDELER.F90:181-250 are laid out at LINIT only
    xmin = geom_in[0]; ymin = geom_in[1]; zmin = geom_in[2];
    xbin = geom_in[3]; ybin = geom_in[4]; zbin = geom_in[5];
    nx = (int)geom_in[6]; ny = (int)geom_in[7]; nz = (int)geom_in[8];
  }
  if (geom_out) {
    geom_out[0] = xmin; geom_out[1] = ymin; geom_out[2] = zmin;
    geom_out[3] = xbin; geom_out[4] = ybin; geom_out[5] = zbin;
    geom_out[6] = nx; geom_out[7] = ny; geom_out[8] = nz;
  }
  const int max_neigh = 1000;
  int status = 0;
  size_t nbins = (size_t)nx * ny * nz;
  // GET_BINS: bins hold node ids in index order
  std::vector<int> cnt(nbins, 0), is(n), js(n), ks(n);
  for (int i = 0; i < n; ++i) {
    const double* x = coo + 3 * (size_t)i;
    int a = (int)std::floor((x[0] - xmin) / xbin) + 1; a = std::max(1, a); a = std::min(a, nx);
    int b = (int)std::floor((x[1] - ymin) / ybin) + 1; b = std::max(1, b); b = std::min(b, ny);
    int c = (int)std::floor((x[2] - zmin) / zbin) + 1; c = std::max(1, c); c = std::min(c, nz);
    is[i] = a; js[i] = b; ks[i] = c;
    if (ijk) { ijk[3 * i] = a; ijk[3 * i + 1] = b; ijk[3 * i + 2] = c; }
    size_t m = (size_t)ny * nx * (c - 1) + (size_t)nx * (b - 1) + (a - 1);
    cnt[m] += 1;
    if (cnt[m] >= max_neigh) status |= MEGA_ST_BIN_OVERFLOW;
  }
  std::vector<int64_t> off(nbins + 1, 0);
  for (size_t m = 0; m < nbins; ++m) off[m + 1] = off[m] + cnt[m];
  std::vector<int> lst(n), fill(nbins, 0);
  for (int i = 0; i < n; ++i) {
    size_t m = (size_t)ny * nx * (ks[i] - 1) + (size_t)nx * (js[i] - 1) + (is[i] - 1);
    lst[off[m] + fill[m]++] = i;
  }
  int mmax = (itype_int == 0) ? 1 : 7;                                // BIN_SEARCH.F90:204-208
  int64_t k = 0;
  int maxn = 0;
  std::vector<int> cand;
  cand.reserve(10000);
  for (int i = 0; i < n; ++i) {                                       // BIN_SEARCH.F90:210-321
    const double* xi = coo + 3 * (size_t)i;
    // BIN_INODE :94-127
    int i0 = std::max(is[i] - 1, 1), i1 = std::min(is[i] + 1, nx);
    int j0 = std::max(js[i] - 1, 1), j1 = std::min(js[i] + 1, ny);
    int k0 = std::max(ks[i] - 1, 1), k1 = std::min(ks[i] + 1, nz);
    cand.clear();
    for (int ix = i0; ix <= i1; ++ix)
      for (int iy = j0; iy <= j1; ++iy)
        for (int iz = k0; iz <= k1; ++iz) {
          size_t m = (size_t)(iz - 1) * nx * ny + (size_t)(iy - 1) * nx + (ix - 1);
          for (int64_t p = off[m]; p < off[m + 1]; ++p) cand.push_back(lst[p]);
        }
    if ((int)cand.size() > 10000) status |= MEGA_ST_CAND_OVERFLOW;
    const double* sl = sm_len + 6 * (size_t)i;
    int cnt_i = 0;
    bool first = true;
    for (int j : cand) {
      const double* xj = coo + 3 * (size_t)j;
      const double* wj = win + 3 * (size_t)j;
      double pts[7][3];
      for (int m = 0; m < 7; ++m) { pts[m][0] = xj[0]; pts[m][1] = xj[1]; pts[m][2] = xj[2]; }
      pts[1][0] = xj[0] + sl[0]; pts[2][0] = xj[0] - sl[1];
      pts[3][1] = xj[1] + sl[2]; pts[4][1] = xj[1] - sl[3];
      pts[5][2] = xj[2] + sl[4]; pts[6][2] = xj[2] - sl[5];
      bool add = false;
      for (int m = 0; m < mmax && !add; ++m) {
        double dx = std::fabs(pts[m][0] - xi[0]), dy = std::fabs(pts[m][1] - xi[1]),
               dz = std::fabs(pts[m][2] - xi[2]);
        if (shsup) {
          double a = dx / wj[0], b = dy / wj[1], c = dz / wj[2];
          if (std::sqrt(a * a + b * b + c * c) < 1.0) add = true;
        } else {
          if (dx / wj[0] < 1.0 && dy / wj[1] < 1.0 && dz / wj[2] < 1.0) add = true;
        }
      }
      if (add) {
        ++k;
        if (k <= cap) gstack[k - 1] = j + 1;
        else status |= MEGA_ST_STACK_OVERFLOW;
        if (first) { gstart[i] = (int)k; first = false; }
        ++cnt_i;
      }
    }
    gn[i] = cnt_i;
    if (cnt_i > maxn) maxn = cnt_i;
  }
  *nnz_out = k;
  *gmaxn = maxn;
  return status;
}

// RK1 for all nodes (FINT.F90:400-408, 580-587).  CSR 1-based.  shp(nnz),
// dshp(3,nnz).  OpenMP over nodes (each node writes its own row).
int orc_rk_shapes(const mega_params* p, int n, const double* coo, const double* win,
                  const int32_t* ebc_nodes, const int* gn, const int* gstart, const int* gstack,
                  double* shp, double* dshp, int nthreads) {
  int status = 0;
#pragma omp parallel num_threads(nthreads) reduction(| : status)
  {
    std::vector<double> work;
    std::vector<int> nb;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      int ln = gn[i];
      if (ln == 0) continue;
      int64_t s = gstart[i] - 1;
      nb.resize(ln);
      for (int j = 0; j < ln; ++j) nb[j] = gstack[s + j] - 1;
      bool ok = rk1(coo + 3 * (size_t)i, coo, win, nb.data(), ln, ebc_nodes, p->ql != 0, p->ql_coef,
                    p->ql_len, p->shsup != 0, shp + s, dshp + 3 * s, work);
      if (!ok) status |= MEGA_ST_SINGULAR_MOMENT;
    }
  }
  return status;
}

// Batched HUGHES_WINGET; lmat/rot column-major (3,3,n).
void orc_hughes_winget(int n, const double* lmat, double* rot, double* strain, double* d, int exact) {
  for (int i = 0; i < n; ++i) {
    M3 L, R;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) L[r][c] = lmat[9 * (size_t)i + c * 3 + r];
    hughes_winget(L, R, strain + 6 * (size_t)i, d + 6 * (size_t)i, exact != 0);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) rot[9 * (size_t)i + c * 3 + r] = R[r][c];
  }
}

void orc_rotate_tensor(int n, const double* rot, double* v) {
  for (int i = 0; i < n; ++i) {
    M3 R;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) R[r][c] = rot[9 * (size_t)i + c * 3 + r];
    rotate_tensor(R, v + 6 * (size_t)i);
  }
}

int orc_constitution(int n, const double* spred, const int* mat, const double* props, double dlt,
                     double* state, double* stress, int* iters, int maxit, double rtol, int solver) {
  int status = 0;
  for (int i = 0; i < n; ++i)
    constitution(spred + 6 * (size_t)i, mat[i], props + 30 * (size_t)i, dlt, state + 20 * (size_t)i,
                 stress + 6 * (size_t)i, maxit, rtol, &status, iters ? iters + i : nullptr, solver);
  return status;
}

// The damaged models on their own: stress holds the rotated old stress on
// entry and the new stress on return; tot = total strain after the step,
// inc = the strain increment (the LSTRAIN and STRAIN of CONSTITUTION).
int orc_damaged(int n, const int* mat, const double* props, const double* tot, const double* inc, double* state,
                double* stress, int* iters, int maxit) {
  int status = 0;
  for (int i = 0; i < n; ++i) {
    double spred[6];  // unused by the damaged models (they form their own predictor)
    for (int k = 0; k < 6; ++k) spred[k] = stress[6 * (size_t)i + k];
    constitution(spred, mat[i], props + 30 * (size_t)i, 0.0, state + 20 * (size_t)i, stress + 6 * (size_t)i,
                 maxit, 0.0, &status, iters ? iters + i : nullptr, 0, tot + 6 * (size_t)i, inc + 6 * (size_t)i);
  }
  return status;
}

// Rate-dependent return mapping with an explicit Newton start (the learned
// guess enters here).  dg0 < 0 selects the plain start.
int orc_vm_rate(int n, const double* spred, const double* props, double dt, double rtol,
                int maxit, const double* dg0, double* state, double* stress, int* iters,
                double* dg_out, int solver) {
  int status = 0;
  for (int i = 0; i < n; ++i) {
    bool capped = false;
    int it = vm_rate(stress + 6 * (size_t)i, spred + 6 * (size_t)i, state + 20 * (size_t)i,
                     props + 30 * (size_t)i, dt, rtol, maxit, solver, dg0 ? dg0[i] : -1.0, &capped,
                     dg_out ? dg_out + i : nullptr);
    if (iters) iters[i] = it;
    if (capped) status |= MEGA_ST_NEWTON_CAP;
  }
  return status;
}

// ------------------------------------------------------------------ NSNI
// Naturally stabilised nodal integration (ITYPE_INT = 2).  The reference's
// NSNI is unfinished (its second derivatives are never formed on the live
// path and its moments never assigned, FINT.F90:441-576, 707-753, 1120-1222),
// so this restates the published method (Hillman & Chen 2016, IJNME 107:603)
// in the form the reference lays out: smoothed second derivatives from the
// shape-function gradients on the faces of each node's smoothing cell
// (FINT.F90:446-535), the strain-gradient increments of D_HUGHES_WINGET
// (HUGHES_WINGET.F90:84-165), stress gradients kept per node
// (LOCAL_DX_STRESS, MAIN.F90:62, 206) and the force term
// B_{,a}^T sigma_{,a} V J M_a (FINT.F90:1127-1208) with the second moments
// M_a = (cell width_a)^2 / 12 of SECOND_MOMENT (PRE_MODEL_SECOND_MOMENT.F90).
// Stress gradients evolve with an isotropic tangent probed from this step's
// stress and strain increments: ESTIMATE_MODULI with NSNI_FLAG set
// (ESTIMATE_MODULI.F90:16-86, the lower clamp off), kept at most elastic so
// the stable step of the elastic moduli still holds.

// Smoothed second derivatives of node i's shape functions (6 per neighbour,
// order XX, YY, ZZ, XY, YZ, XZ as SHPDD_SM): RK1 gradients at the six face
// points x +- SM_LEN (order +X, -X, +Y, -Y, +Z, -Z), differenced over the
// cell width.  Returns false if a moment matrix was singular.
static bool nsni_second_derivatives(const double x[3], const double sml[6], const double* gcoo,
                                    const double* gwin, const int* nb, int ln, const int32_t* ebcs,
                                    const mega_params* p, double* dd, std::vector<double>& work) {
  std::vector<double> g(6 * 3 * (size_t)ln), sh(ln);
  bool ok = true;
  for (int f = 0; f < 6; ++f) {
    double pt[3] = {x[0], x[1], x[2]};
    const int a = f / 2;
    pt[a] = (f % 2 == 0) ? x[a] + sml[f] : x[a] - sml[f];
    ok = rk1(pt, gcoo, gwin, nb, ln, ebcs, p->ql != 0, p->ql_coef, p->ql_len, p->shsup != 0, sh.data(),
             g.data() + 3 * (size_t)ln * f, work) && ok;
  }
  for (int j = 0; j < ln; ++j) {
    double D[3][3];  // D[a][b]: difference along a of the b-derivative
    for (int a = 0; a < 3; ++a) {
      const double w = sml[2 * a] + sml[2 * a + 1];
      for (int b = 0; b < 3; ++b)
        D[a][b] = (g[3 * ((size_t)ln * (2 * a) + j) + b] - g[3 * ((size_t)ln * (2 * a + 1) + j) + b]) / w;
    }
    double* o = dd + 6 * (size_t)j;
    o[0] = D[0][0];
    o[1] = D[1][1];
    o[2] = D[2][2];
    o[3] = 0.5 * (D[0][1] + D[1][0]);
    o[4] = 0.5 * (D[1][2] + D[2][1]);
    o[5] = 0.5 * (D[0][2] + D[2][0]);
  }
  return ok;
}

// index of S_(m a) in the XX, YY, ZZ, XY, YZ, XZ order (XMAP/YMAP/ZMAP of
// FINT.F90:714-726)
static const int kDD[3][3] = {{0, 3, 5}, {3, 1, 4}, {5, 4, 2}};

// D_HUGHES_WINGET (HUGHES_WINGET.F90:84-165): the derivative of the
// objective strain increment along one direction, DG = DL A^-1 -
// L A^-1 (DL / 2) A^-1 with A = I + L / 2; engineering shear.
static void d_hughes_winget(const M3 L, const M3 DL, double de[6], bool exact) {
  M3 A, Ai, DA, t, ida, t1, t2, E;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i][j] = (i == j ? 1.0 : 0.0) + 0.5 * L[i][j];
      DA[i][j] = 0.5 * DL[i][j];
    }
  inv3(A, Ai, exact);
  M3 nAi;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) nAi[i][j] = -Ai[i][j];
  mm3(nAi, DA, t);
  mm3(t, Ai, ida);
  mm3(DL, Ai, t1);
  mm3(L, ida, t2);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) E[i][j] = 0.5 * ((t1[i][j] + t2[i][j]) + (t1[j][i] + t2[j][i]));
  t2v(E, de);
  de[3] = 2.0 * de[3]; de[4] = 2.0 * de[4]; de[5] = 2.0 * de[5];
}

// CONSTRUCT_FINT (FINT.F90:16-1336), Lagrangian DNI path.  When linit, the
// shape functions are built (RK1) and stored; otherwise they are recalled.
// nthreads > 1 keeps the per-thread FINT_TEMP/FEXT_TEMP buffers.
// newton_iters (n, may be NULL) receives the Newton passes per node.
int orc_construct_fint(const mega_params* p, int n, const double* gcoo, const double* gwin,
                       const double* gvol, const double* gprop, const int* gmat,
                       const int32_t* gebc_nodes, const double* bodyforce, double* gstate,
                       double* gstress, double* gstrain, const double* gdinc,
                       const double* gdinc_tot, const int* gn, const int* gstart,
                       const int* gstack, double* shp_stack, double* dshp_stack, int linit,
                       double dlt, double* fint, double* fext, double* gmax_wvel,
                       double* gstrain_eq, double* gint_work, int nthreads, int* newton_iters,
                       const double* sm_len, double* ddshp, double* sgrad, const double* gcoo_current) {
  const bool exact = p->inv3_exact != 0;
  const bool nsni = p->itype_int == 2;
  // semi-Lagrangian (LLAGRANGIAN = .FALSE.): RK1 on the current coordinates
  // every call (FINT.F90:410-436), gradients used as they are (no push-
  // forward), DET left at its initial 1 (FINT.F90:230: only the Lagrangian
  // branches set it)
  const bool semi = p->lagrangian == 0;
  if (nsni && (!sm_len || !ddshp || !sgrad)) return -2;
  if (semi && (!gcoo_current || nsni)) return -2;
  int status = 0;
  int nt = std::max(1, nthreads);
  std::vector<double> fint_t((size_t)nt * 3 * n, 0.0), fext_t((size_t)nt * 3 * n, 0.0);
  std::vector<double> work_t(nt, 0.0);
#pragma omp parallel num_threads(nt) reduction(| : status)
  {
    int tid = omp_get_thread_num();
    double* FT = fint_t.data() + (size_t)tid * 3 * n;
    double* ET = fext_t.data() + (size_t)tid * 3 * n;
    std::vector<double> work, shpd, shp0;
    std::vector<int> nb;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      int ln = gn[i];
      int64_t s = gstart[i] - 1;
      nb.resize(ln);
      for (int j = 0; j < ln; ++j) nb[j] = gstack[s + j] - 1;
      const double* lprop = gprop + 30 * (size_t)i;
      double vol = gvol[i];
      double lstress[6], lstrain[6], lstate[20];
      for (int k = 0; k < 6; ++k) { lstress[k] = gstress[6 * (size_t)i + k]; lstrain[k] = gstrain[6 * (size_t)i + k]; }
      for (int k = 0; k < 20; ++k) lstate[k] = gstate[20 * (size_t)i + k];
      shpd.resize(3 * (size_t)ln);
      shp0.resize(ln);
      if (linit || semi) {                                            // FINT.F90:400-436, 580-587
        const double* xs = semi ? gcoo_current : gcoo;
        if (!rk1(xs + 3 * (size_t)i, xs, gwin, nb.data(), ln, gebc_nodes, p->ql != 0, p->ql_coef,
                 p->ql_len, p->shsup != 0, shp_stack + s, dshp_stack + 3 * s, work))
          status |= MEGA_ST_SINGULAR_MOMENT;
        if (nsni && !nsni_second_derivatives(gcoo + 3 * (size_t)i, sm_len + 6 * (size_t)i, gcoo, gwin, nb.data(),
                                             ln, gebc_nodes, p, ddshp + 6 * s, work))
          status |= MEGA_ST_SINGULAR_MOMENT;
      }
      for (int j = 0; j < ln; ++j) {                                  // FINT.F90:354-359
        shp0[j] = shp_stack[s + j];
        for (int c = 0; c < 3; ++c) shpd[3 * j + c] = dshp_stack[3 * (s + j) + c];
      }
      double det = 1.0;
      M3 fm, ifm_s = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, L_s = {}, R_s = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      if (p->finite_strain && !semi) {                                // FINT.F90:361-391
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) {
            double v = (k == l) ? 1.0 : 0.0;
            for (int j = 0; j < ln; ++j) v += shpd[3 * j + l] * gdinc_tot[3 * (size_t)nb[j] + k];
            fm[k][l] = v;
          }
        det = det_abs(fm);
        M3 ifm;
        inv3(fm, ifm, exact);
        std::memcpy(ifm_s, ifm, sizeof(M3));
        for (int j = 0; j < ln; ++j) {
          double t[3] = {shpd[3 * j], shpd[3 * j + 1], shpd[3 * j + 2]};
          double o[3] = {0, 0, 0};
          for (int k = 0; k < 3; ++k) {
            o[0] += t[k] * ifm[k][0];
            o[1] += t[k] * ifm[k][1];
            o[2] += t[k] * ifm[k][2];
          }
          shpd[3 * j] = o[0]; shpd[3 * j + 1] = o[1]; shpd[3 * j + 2] = o[2];
        }
      }
      double strain[6], D[6] = {0, 0, 0, 0, 0, 0};
      if (p->finite_strain) {                                         // FINT.F90:665-766
        M3 L;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) {
            double v = 0.0;
            for (int j = 0; j < ln; ++j) v += shpd[3 * j + l] * gdinc[3 * (size_t)nb[j] + k];
            L[k][l] = v;
          }
        M3 R;
        hughes_winget(L, R, strain, D, exact);
        rotate_tensor(R, lstress);
        rotate_tensor(R, lstrain);
        std::memcpy(L_s, L, sizeof(M3));
        std::memcpy(R_s, R, sizeof(M3));
      } else {                                                        // FINT.F90:772-783
        for (int k = 0; k < 6; ++k) strain[k] = 0.0;
        for (int j = 0; j < ln; ++j) {
          const double* du = gdinc + 3 * (size_t)nb[j];
          const double* g = &shpd[3 * j];
          strain[0] += g[0] * du[0];
          strain[1] += g[1] * du[1];
          strain[2] += g[2] * du[2];
          strain[3] += g[1] * du[2] + g[2] * du[1];
          strain[4] += g[0] * du[2] + g[2] * du[0];
          strain[5] += g[0] * du[1] + g[1] * du[0];
        }
      }
      for (int k = 0; k < 6; ++k) lstrain[k] = lstrain[k] + strain[k];   // FINT.F90:789
      double srot[6];  // the rotated old stress (NSNI probes the material's increment from it)
      std::memcpy(srot, lstress, sizeof(srot));
      double lam = lprop[27], mu = lprop[28], l2m = lprop[29];            // FORM_CMAT :252-288
      double C[6][6] = {};
      C[0][0] = C[1][1] = C[2][2] = l2m;
      C[3][3] = C[4][4] = C[5][5] = mu;
      C[0][1] = C[1][0] = C[0][2] = C[2][0] = C[2][1] = C[1][2] = lam;
      double spred[6];
      for (int r = 0; r < 6; ++r) {
        double v = 0.0;
        for (int c = 0; c < 6; ++c) v += C[r][c] * strain[c];
        spred[r] = lstress[r] + v;
      }
      int it = 0;
      constitution(spred, gmat[i], lprop, dlt, lstate, lstress, p->newton_max_iter, p->newton_rtol,
                   &status, &it, p->rate_solver, lstrain, strain);
      if (newton_iters) newton_iters[i] = it;
      for (int k = 0; k < 20; ++k) gstate[20 * (size_t)i + k] = lstate[k];   // FINT.F90:809-811
      double sinc[6], einc[6];
      for (int k = 0; k < 6; ++k) {                                   // FINT.F90:813-828
        sinc[k] = lstress[k] - gstress[6 * (size_t)i + k];
        einc[k] = lstrain[k] - gstrain[6 * (size_t)i + k];
        gstress[6 * (size_t)i + k] = lstress[k];
        gstrain[6 * (size_t)i + k] = lstrain[k];
      }
      double eq = lstrain[0] * lstrain[0] + lstrain[1] * lstrain[1] + lstrain[2] * lstrain[2] +
                  2.0 * (lstrain[3] * lstrain[3] + lstrain[4] * lstrain[4] + lstrain[5] * lstrain[5]);
      gstrain_eq[i] = std::sqrt(eq * 2.0 / 3.0);                      // FINT.F90:831-834
      if (p->finite_strain) {                                         // FINT.F90:837-847
        for (int k = 0; k < 6; ++k) work_t[tid] += 0.5 * D[k] * (2.0 * lstress[k] - sinc[k]) * vol * det;
      } else {
        for (int k = 0; k < 6; ++k) work_t[tid] += 0.5 * einc[k] * sinc[k] * vol * det;
      }
      double bulk = bulk_mod(lprop[1], lprop[0]), shear = shear_mod(lprop[1], lprop[0]);  // :850-870
      if (gmat[i] > 1) estimate_moduli(sinc, einc, shear, bulk);
      double pmod = bulk + 4.0 * shear / 3.0;
      gmax_wvel[i] = std::sqrt(std::max(pmod, shear) / lprop[2]);
      const double* lbod = bodyforce ? bodyforce + 3 * (size_t)i : nullptr;
      double dens = lprop[2];
      for (int j = 0; j < ln; ++j) {                                  // FINT.F90:999-1116
        const double* g = &shpd[3 * j];
        double f0 = g[0] * lstress[0] + g[2] * lstress[4] + g[1] * lstress[5];
        double f1 = g[1] * lstress[1] + g[2] * lstress[3] + g[0] * lstress[5];
        double f2 = g[2] * lstress[2] + g[1] * lstress[3] + g[0] * lstress[4];
        size_t jj = (size_t)nb[j];
        FT[3 * jj + 0] += f0 * vol * det;
        FT[3 * jj + 1] += f1 * vol * det;
        FT[3 * jj + 2] += f2 * vol * det;
        for (int c = 0; c < 3; ++c) {
          double fg = shp0[j] * p->gravity[c] * dens;
          double fb = lbod ? shp0[j] * lbod[c] * dens : 0.0;
          ET[3 * jj + c] += (fb + fg) * vol * det;
        }
      }
      if (nsni) {
        // the gradients along a of the incremental displacement gradient,
        // (H_a)_km = sum_J S_(m a)(J) du_J,k (XLMAT/YLMAT/ZLMAT, FINT.F90:728-737)
        const double* dd = ddshp + 6 * s;
        double* sg = sgrad + 18 * (size_t)i;
        M3 H[3];
        for (int a = 0; a < 3; ++a)
          for (int k = 0; k < 3; ++k)
            for (int m = 0; m < 3; ++m) {
              double v = 0.0;
              for (int j = 0; j < ln; ++j) v += dd[6 * (size_t)j + kDD[m][a]] * gdinc[3 * (size_t)nb[j] + k];
              H[a][k][m] = v;
            }
        const double* sml = sm_len + 6 * (size_t)i;
        double gs = shear_mod(lprop[1], lprop[0]), ks = bulk_mod(lprop[1], lprop[0]);
        {
          double dso[6];
          for (int k = 0; k < 6; ++k) dso[k] = lstress[k] - srot[k];
          estimate_moduli_nsni(dso, strain, gs, ks);
        }
        double Cs[6][6] = {};
        {
          const double lam_s = ks - 2.0 * gs / 3.0, l2m_s = ks + 4.0 * gs / 3.0;
          Cs[0][0] = Cs[1][1] = Cs[2][2] = l2m_s;
          Cs[3][3] = Cs[4][4] = Cs[5][5] = gs;
          Cs[0][1] = Cs[1][0] = Cs[0][2] = Cs[2][0] = Cs[2][1] = Cs[1][2] = lam_s;
        }
        double fac[3], W[3][3][3];  // W[a] = M_a / V * V J sigma_a INV3(F)^T
        for (int a = 0; a < 3; ++a) {
          const double wd = sml[2 * a] + sml[2 * a + 1];
          fac[a] = wd * wd / 12.0;
          double de[6];
          if (p->finite_strain) {
            M3 La;
            mm3(H[a], ifm_s, La);
            d_hughes_winget(L_s, La, de, exact);
            rotate_tensor(R_s, sg + 6 * a);
          } else {
            de[0] = H[a][0][0]; de[1] = H[a][1][1]; de[2] = H[a][2][2];
            de[3] = H[a][2][1] + H[a][1][2]; de[4] = H[a][2][0] + H[a][0][2]; de[5] = H[a][1][0] + H[a][0][1];
          }
          double ds[6];
          for (int r = 0; r < 6; ++r) {
            double v = 0.0;
            for (int c = 0; c < 6; ++c) v += Cs[r][c] * de[c];
            ds[r] = v;
          }
          for (int k = 0; k < 6; ++k) sg[6 * a + k] += ds[k];
          for (int k = 0; k < 6; ++k) work_t[tid] += 0.5 * fac[a] * de[k] * (2.0 * sg[6 * a + k] - ds[k]) * vol * det;
          M3 Sa;
          v2t(sg + 6 * a, Sa);
          for (int k = 0; k < 3; ++k)
            for (int m = 0; m < 3; ++m) {
              double v = 0.0;
              for (int q = 0; q < 3; ++q) v += Sa[k][q] * ifm_s[m][q];
              W[a][k][m] = fac[a] * vol * det * v;
            }
        }
        for (int j = 0; j < ln; ++j) {                                // FINT.F90:1127-1208
          const double* d = dd + 6 * (size_t)j;
          double f[3] = {0.0, 0.0, 0.0};
          for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 3; ++k)
              for (int m = 0; m < 3; ++m) f[k] += W[a][k][m] * d[kDD[m][a]];
          const size_t jj = (size_t)nb[j];
          FT[3 * jj + 0] += f[0];
          FT[3 * jj + 1] += f[1];
          FT[3 * jj + 2] += f[2];
        }
        for (int k = 0; k < 18; ++k)
          if (!std::isfinite(sg[k])) status |= MEGA_ST_NONFINITE;
      }
      for (int k = 0; k < 6; ++k)
        if (!std::isfinite(lstress[k])) status |= MEGA_ST_NONFINITE;
    }
  }
  double w = 0.0;
  for (int t = 0; t < nt; ++t) w += work_t[t];
  *gint_work += w;                                                    // FINT.F90:1232
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int i = 0; i < 3 * n; ++i) {                                   // FINT.F90:1238-1247
    double a = 0.0, b = 0.0;
    for (int t = 0; t < nt; ++t) {
      a += fint_t[(size_t)t * 3 * n + i];
      b += fext_t[(size_t)t * 3 * n + i];
    }
    fint[i] = a;
    fext[i] = b;
  }
  return status;
}

// HANDELER.F90:114-133 DO_INTERP: physical values from generalised ones.
void orc_interp(int n, const int* gn, const int* gstart, const int* gstack, const double* shp,
                const double* dinc, double* dinc_phy, int nthreads) {
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(static)
  for (int i = 0; i < n; ++i) {
    int64_t s = gstart[i] - 1;
    for (int k = 0; k < 3; ++k) {
      double v = 0.0;
      for (int j = 0; j < gn[i]; ++j) v += shp[s + j] * dinc[3 * (size_t)(gstack[s + j] - 1) + k];
      dinc_phy[3 * (size_t)i + k] = v;
    }
  }
}

// UDFM_SHAPE_TENSOR (RK.f90:579-726): influence function (box cubic spline)
// and K^-1 (INVERSE, full pivot).  ginvk (3,3,n) column-major.
int orc_pd_shape(int n, const double* gcoo, const double* gwin, const double* gvol, const int* gn,
                 const int* gstart, const int* gstack, double* shp, double* ginvk, int nthreads) {
  int status = 0;
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(static) reduction(| : status)
  for (int i = 0; i < n; ++i) {
    int64_t s = gstart[i] - 1;
    const double* x = gcoo + 3 * (size_t)i;
    double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < gn[i]; ++j) {
      int ii = gstack[s + j] - 1;
      const double* xj = gcoo + 3 * (size_t)ii;
      const double* aj = gwin + 3 * (size_t)ii;
      double h[3] = {-(x[0] - xj[0]), -(x[1] - xj[1]), -(x[2] - xj[2])};
      double kx, d0, ky, d1, kz, d2;
      mls_kernel0(std::fabs(-(x[0] - xj[0]) / aj[0]), kx, d0);
      mls_kernel0(std::fabs(-(x[1] - xj[1]) / aj[1]), ky, d1);
      mls_kernel0(std::fabs(-(x[2] - xj[2]) / aj[2]), kz, d2);
      double phi = kx * ky * kz;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) K[a * 3 + b] += h[a] * h[b] * phi * gvol[ii];
      shp[s + j] = phi;
    }
    double Ki[9];
    if (!inverse_gj(K, 3, Ki)) status |= MEGA_ST_SINGULAR_SHAPE;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) ginvk[9 * (size_t)i + b * 3 + a] = Ki[a * 3 + b];
  }
  return status;
}

// CONSTRUCT_FINT_PD (FINT_PD.F90:214-684), Lagrangian, HODIV = .FALSE.
// Requires orc_pd_shape done (shp, ginvk).  linit: F = I, DET = 1.
int orc_construct_fint_pd(const mega_params* p, int n, const double* gcoo, const double* gcur,
                          const double* gvol, const double* gprop, const int* gmat, double* gstate,
                          double* gstress, double* gstrain, const double* gdinc, const int* gn,
                          const int* gstart, const int* gstack, const double* shp,
                          const double* ginvk, int linit, double dlt, double* fint,
                          double* gmax_wvel, int nthreads) {
  const bool exact = p->inv3_exact != 0;
  int status = 0;
  int nt = std::max(1, nthreads);
  std::vector<double> ft((size_t)nt * 3 * n, 0.0);
#pragma omp parallel num_threads(nt) reduction(| : status)
  {
    int tid = omp_get_thread_num();
    double* FT = ft.data() + (size_t)tid * 3 * n;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {
      int64_t s = gstart[i] - 1;
      int ln = gn[i];
      const double* X0 = gcoo + 3 * (size_t)i;
      const double* lprop = gprop + 30 * (size_t)i;
      M3 invk, fm, ifm;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) invk[a][b] = ginvk[9 * (size_t)i + b * 3 + a];
      double det = 1.0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) ifm[a][b] = fm[a][b] = (a == b) ? 1.0 : 0.0;
      // DFM_SHAPE_TENSOR (RK.f90:730-807) with current coordinates -> S
      auto dfm = [&](const double* Xt, const double* cur_base, bool use_gdinc, M3 S) {
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) S[a][b] = 0.0;
        for (int j = 0; j < ln; ++j) {
          int ii = gstack[s + j] - 1;
          const double* xj = gcoo + 3 * (size_t)ii;
          const double* cj = (use_gdinc ? gdinc : cur_base) + 3 * (size_t)ii;
          double h[3] = {xj[0] - X0[0], xj[1] - X0[1], xj[2] - X0[2]};
          double hs[3] = {cj[0] - Xt[0], cj[1] - Xt[1], cj[2] - Xt[2]};
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) S[a][b] += hs[a] * h[b] * shp[s + j] * gvol[ii];
        }
      };
      if (!linit) {                                                   // FINT_PD.F90:377-404
        M3 S;
        dfm(gcur + 3 * (size_t)i, gcur, false, S);
        mm3(S, invk, fm);
        det = det_abs(fm);
        double a9[9], r9[9];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) a9[a * 3 + b] = fm[a][b];
        if (!inverse_gj(a9, 3, r9)) status |= MEGA_ST_SINGULAR_SHAPE;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) ifm[a][b] = r9[a * 3 + b];
      }
      M3 L, t;                                                        // FINT_PD.F90:456-470
      dfm(gdinc + 3 * (size_t)i, nullptr, true, L);
      mm3(L, invk, t);
      if (!linit) mm3(t, ifm, L); else std::memcpy(L, t, sizeof(M3));
      double lstress[6], lstrain[6], lstate[20], strain[6], D[6];
      for (int k = 0; k < 6; ++k) { lstress[k] = gstress[6 * (size_t)i + k]; lstrain[k] = gstrain[6 * (size_t)i + k]; }
      for (int k = 0; k < 20; ++k) lstate[k] = gstate[20 * (size_t)i + k];
      M3 R;
      hughes_winget(L, R, strain, D, exact);                          // :475-494
      rotate_tensor(R, lstress);
      rotate_tensor(R, lstrain);
      for (int k = 0; k < 6; ++k) lstrain[k] += strain[k];
      double lam = lprop[27], mu = lprop[28], l2m = lprop[29];
      double C[6][6] = {};
      C[0][0] = C[1][1] = C[2][2] = l2m;
      C[3][3] = C[4][4] = C[5][5] = mu;
      C[0][1] = C[1][0] = C[0][2] = C[2][0] = C[2][1] = C[1][2] = lam;
      double spred[6];
      for (int r = 0; r < 6; ++r) {
        double v = 0.0;
        for (int c = 0; c < 6; ++c) v += C[r][c] * strain[c];
        spred[r] = lstress[r] + v;
      }
      constitution(spred, gmat[i], lprop, dlt, lstate, lstress, p->newton_max_iter, p->newton_rtol,
                   &status, nullptr, p->rate_solver, lstrain, strain);
      for (int k = 0; k < 20; ++k) gstate[20 * (size_t)i + k] = lstate[k];
      double sinc[6], einc[6];
      for (int k = 0; k < 6; ++k) {                                   // :505-518 (STRAIN_INC uses
        sinc[k] = lstress[k] - gstress[6 * (size_t)i + k];            //  the old stress, as written)
        einc[k] = lstrain[k] - gstress[6 * (size_t)i + k];
        gstress[6 * (size_t)i + k] = lstress[k];
        gstrain[6 * (size_t)i + k] = lstrain[k];
      }
      double bulk = bulk_mod(lprop[1], lprop[0]), shear = shear_mod(lprop[1], lprop[0]);
      if (gmat[i] > 1) estimate_moduli(sinc, einc, shear, bulk);
      double pmod = bulk + 4.0 * shear / 3.0;
      gmax_wvel[i] = std::sqrt(std::max(pmod, shear) / lprop[2]);
      if (gmat[i] == 3) gmax_wvel[i] = gmax_wvel[i] / 0.15;
      M3 sig, ifmT, pk, ts;                                           // :629-655
      v2t(lstress, sig);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) ifmT[a][b] = ifm[b][a];
      mm3(sig, ifmT, pk);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) pk[a][b] = det * pk[a][b];
      mm3(pk, invk, ts);
      for (int j = 0; j < ln; ++j) {
        int jj = gstack[s + j] - 1;
        const double* xj = gcoo + 3 * (size_t)jj;
        double dx[3] = {X0[0] - xj[0], X0[1] - xj[1], X0[2] - xj[2]};
        for (int k = 0; k < 3; ++k) {
          double f3 = ts[k][0] * dx[0] + ts[k][1] * dx[1] + ts[k][2] * dx[2];
          FT[3 * (size_t)jj + k] = FT[3 * (size_t)jj + k] - f3 * gvol[i] * shp[s + j] * gvol[jj];
          FT[3 * (size_t)i + k] = FT[3 * (size_t)i + k] + f3 * gvol[jj] * shp[s + j] * gvol[i];
        }
      }
    }
  }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int i = 0; i < 3 * n; ++i) {
    double a = 0.0;
    for (int t = 0; t < nt; ++t) a += ft[(size_t)t * 3 * n + i];
    fint[i] = a;
  }
  return status;
}

// Prescribed velocity of the fixity-2 DOFs at TIME (MAIN.F90:448-462): the
// first window k with FIXITY2_TIME(k,1) < TIME < FIXITY2_TIME(k,2) gives
// FIXITY2_NONZERO_EBC(k,j) / (FIXITY2_TIME(k,2) - FIXITY2_TIME(k,1)) for
// direction j; outside every window the velocity is zero.  ftime is
// (steps,2) and fdisp (steps,3), column-major as MODEL.F90:62 holds them.
void orc_fixity2_velocity(int steps, const double* ftime, const double* fdisp, double time, double* vel2) {
  int step_num = 0;
  for (int k = 1; k <= steps; ++k)
    if (ftime[k - 1] < time && time < ftime[steps + k - 1]) { step_num = k; break; }
  for (int j = 0; j < 3; ++j) {
    if (1 <= step_num && step_num <= steps)
      vel2[j] = fdisp[(size_t)j * steps + step_num - 1] / (ftime[steps + step_num - 1] - ftime[step_num - 1]);
    else
      vel2[j] = 0.0;
  }
}

// Central-difference update of MAIN.F90:432-488 for fixity codes 0, 1 and 2
// (vel2 = the prescribed velocities of this step's TIME, from
// orc_fixity2_velocity; may be null when no DOF has code 2).
// total_force (3,2) accumulates as TOTAL_FORCE does.
void orc_corrector(int n, const int* ebc, const double* prop21, const double* mass, const double* fint,
                   double* fext, double* vel, double* acl, double* prforce, const int* body_id,
                   double* total_force, double dlt, const double* vel2) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 3; ++j) {
      size_t m = 3 * (size_t)i + j;
      if (ebc[m] == 1) {
        vel[m] = 0.0;
        acl[m] = 0.0;
        prforce[m] = -fint[m];
        fext[m] = -fint[m];
      } else if (ebc[m] == 2) {                                       // MAIN.F90:447-470
        vel[m] = vel2 ? vel2[j] : 0.0;
        acl[m] = 0.0;
        prforce[m] = -fint[m];
        fext[m] = -fint[m];
      } else {
        double mpdc = prop21[i] * mass[m];
        acl[m] = (fext[m] - fint[m] - mpdc * vel[m]) / (mass[m] + 0.5 * dlt * mpdc);
        vel[m] = vel[m] + 0.5 * dlt * acl[m];
        prforce[m] = 0.0;
      }
      int b = body_id ? body_id[i] : 1;
      if (b >= 1 && b <= 2) total_force[(b - 1) * 3 + j] += prforce[m];
    }
}

// One pass of MAIN.F90's time loop after LINIT (MAIN.F90:348-555): predictor
// (:353-355), DO_INTERP (HANDELER.F90:114-133, serial like the reference),
// current coordinates (:377-386), CONSTRUCT_FINT (:407-416), fixity /
// acceleration / corrector (:432-488) and the energy sums (:524-555).
// en[0..3] = internal (accumulated work), kinetic, external (accumulated),
// int_work accumulator; total_force (3,2) accumulates.
int orc_step(const mega_params* p, int n, const double* coo, const double* win, const double* vol,
             const double* mass, const int* ebc, const double* props, const int* mat,
             const int32_t* ebc_nodes, const double* bodyforce, const int* body_id, const int* gn,
             const int* gstart, const int* gstack, double* shp, double* dshp, double* state,
             double* stress, double* strain, double* dsp, double* dsp_tot, double* dsp_tot_phy,
             double* vel, double* acl, double* fint, double* fext, double* prforce, double* coo_cur,
             double* wvel, double* strain_eq, double* en, double* total_force, double dlt,
             int nthreads, int serial_interp, int* newton_iters, const double* sm_len, double* ddshp,
             double* sgrad, const double* vel2) {
  size_t n3 = 3 * (size_t)n;
  for (size_t m = 0; m < n3; ++m) {                                  // predictor
    dsp[m] = dlt * vel[m] + dlt * dlt * 0.5 * acl[m];
    dsp_tot[m] = dsp_tot[m] + dsp[m];
    vel[m] = vel[m] + dlt * 0.5 * acl[m];
  }
  std::vector<double> dphy(n3);
  orc_interp(n, gn, gstart, gstack, shp, dsp, dphy.data(), serial_interp ? 1 : nthreads);
  for (size_t m = 0; m < n3; ++m) {
    dsp_tot_phy[m] += dphy[m];
    coo_cur[m] = coo[m] + dsp_tot_phy[m];
  }
  std::vector<double> fext_nmo(fext, fext + n3);
  int st = orc_construct_fint(p, n, coo, win, vol, props, mat, ebc_nodes, bodyforce, state, stress,
                              strain, dsp, dsp_tot, gn, gstart, gstack, shp, dshp, 0, dlt, fint,
                              fext, wvel, strain_eq, &en[3], nthreads, newton_iters, sm_len, ddshp, sgrad,
                              nullptr);
  std::vector<double> p21(n);
  for (int i = 0; i < n; ++i) p21[i] = props[30 * (size_t)i + 20];
  orc_corrector(n, ebc, p21.data(), mass, fint, fext, vel, acl, prforce, body_id, total_force, dlt, vel2);
  double ke = 0.0, ee = en[2];
  for (size_t m = 0; m < n3; ++m) {
    ke += 0.5 * mass[m] * vel[m] * vel[m];
    ee += 0.5 * (fext[m] + fext_nmo[m]) * dsp[m];
  }
  en[0] = en[3];
  en[1] = ke;
  en[2] = ee;
  return st;
}

// Bond-based prototype microelastic brittle peridynamics (no reference
// counterpart; Silling & Askari 2005).  Pairwise force density on i:
//   f_i = sum_j c * s_ij * mu_ij * (y_j - y_i)/|y_j - y_i| * V_j,
//   s = (|y_j - y_i| - |xi|)/|xi|; a bond whose stretch exceeds s_c breaks
// for good (broken[e] = 1 for CSR entry e).  Row i excludes nothing: the
// self entry has |xi| = 0 and is skipped.  Returns the newly broken count.
int64_t orc_pmb_force(int n, const double* X, const double* u, const double* vol, const int* gn,
                      const int* gstart, const int* gstack, double c, double s_c,
                      uint8_t* broken, double* f, int nthreads) {
  int64_t nb = 0;
#pragma omp parallel for num_threads(std::max(1, nthreads)) schedule(static) reduction(+ : nb)
  for (int i = 0; i < n; ++i) {
    int64_t s = gstart[i] - 1;
    double fi[3] = {0, 0, 0};
    const double* xi = X + 3 * (size_t)i;
    const double* ui = u + 3 * (size_t)i;
    for (int jj = 0; jj < gn[i]; ++jj) {
      int64_t e = s + jj;
      int j = gstack[e] - 1;
      if (j == i || broken[e]) continue;
      const double* xj = X + 3 * (size_t)j;
      const double* uj = u + 3 * (size_t)j;
      double xi_[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      double eta[3] = {xi_[0] + (uj[0] - ui[0]), xi_[1] + (uj[1] - ui[1]), xi_[2] + (uj[2] - ui[2])};
      double l0 = std::sqrt(xi_[0] * xi_[0] + xi_[1] * xi_[1] + xi_[2] * xi_[2]);
      double l = std::sqrt(eta[0] * eta[0] + eta[1] * eta[1] + eta[2] * eta[2]);
      double st = (l - l0) / l0;
      if (st > s_c) { broken[e] = 1; ++nb; continue; }
      double w = c * st * vol[j] / l;
      fi[0] += w * eta[0]; fi[1] += w * eta[1]; fi[2] += w * eta[2];
    }
    f[3 * (size_t)i] = fi[0]; f[3 * (size_t)i + 1] = fi[1]; f[3 * (size_t)i + 2] = fi[2];
  }
  return nb;
}

// --------------------------------------------------------------- MLP (FP64)
// 4 -> H -> H -> 1, tanh hidden activations, linear output.  Parameters are
// packed [W1 (H x 4), b1 (H), W2 (H x H), b2 (H), W3 (1 x H), b3 (1)], row-
// major (out, in).  Forward for a batch; loss = mean((y - t)^2) / 2;
// backward writes dL/dtheta.  Used as the gradient oracle of the CUDA MLP.
int64_t orc_mlp_nparams(int H) { return (int64_t)H * 4 + H + (int64_t)H * H + H + H + 1; }

double orc_mlp_forward_backward(int H, const double* theta, int nb, const double* x, const double* t,
                                double* y, double* grad) {
  const double* W1 = theta;
  const double* b1 = W1 + H * 4;
  const double* W2 = b1 + H;
  const double* b2 = W2 + (size_t)H * H;
  const double* W3 = b2 + H;
  const double* b3 = W3 + H;
  double* gW1 = grad; double* gb1 = gW1 ? gW1 + H * 4 : nullptr;
  double* gW2 = gb1 ? gb1 + H : nullptr; double* gb2 = gW2 ? gW2 + (size_t)H * H : nullptr;
  double* gW3 = gb2 ? gb2 + H : nullptr; double* gb3 = gW3 ? gW3 + H : nullptr;
  if (grad) std::memset(grad, 0, sizeof(double) * orc_mlp_nparams(H));
  std::vector<double> h1(H), h2(H), d1(H), d2(H);
  double loss = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double* xb = x + 4 * (size_t)b;
    for (int o = 0; o < H; ++o) {
      double a = b1[o];
      for (int k = 0; k < 4; ++k) a += W1[o * 4 + k] * xb[k];
      h1[o] = std::tanh(a);
    }
    for (int o = 0; o < H; ++o) {
      double a = b2[o];
      for (int k = 0; k < H; ++k) a += W2[(size_t)o * H + k] * h1[k];
      h2[o] = std::tanh(a);
    }
    double out = b3[0];
    for (int k = 0; k < H; ++k) out += W3[k] * h2[k];
    if (y) y[b] = out;
    if (t) {
      double r = out - t[b];
      loss += 0.5 * r * r / nb;
      if (grad) {
        double go = r / nb;
        gb3[0] += go;
        for (int k = 0; k < H; ++k) { gW3[k] += go * h2[k]; d2[k] = go * W3[k] * (1.0 - h2[k] * h2[k]); }
        for (int o = 0; o < H; ++o) {
          gb2[o] += d2[o];
          for (int k = 0; k < H; ++k) gW2[(size_t)o * H + k] += d2[o] * h1[k];
        }
        for (int k = 0; k < H; ++k) {
          double a = 0.0;
          for (int o = 0; o < H; ++o) a += W2[(size_t)o * H + k] * d2[o];
          d1[k] = a * (1.0 - h1[k] * h1[k]);
        }
        for (int o = 0; o < H; ++o) {
          gb1[o] += d1[o];
          for (int k = 0; k < 4; ++k) gW1[o * 4 + k] += d1[o] * xb[k];
        }
      }
    }
  }
  return loss;
}

// Adam (Kingma & Ba 2015), step index t >= 1, in place.
void orc_adam(int64_t np, double* theta, const double* g, double* m, double* v, double lr, double b1,
              double b2, double eps, int t) {
  double c1 = 1.0 - std::pow(b1, t), c2 = 1.0 - std::pow(b2, t);
  for (int64_t i = 0; i < np; ++i) {
    m[i] = b1 * m[i] + (1.0 - b1) * g[i];
    v[i] = b2 * v[i] + (1.0 - b2) * g[i] * g[i];
    double mh = m[i] / c1, vh = v[i] / c2;
    theta[i] -= lr * mh / (std::sqrt(vh) + eps);
  }
}

}  // extern "C"
