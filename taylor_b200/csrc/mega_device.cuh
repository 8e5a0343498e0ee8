// mega_device.cuh -- per-node device math of the explicit meshfree step.
//
// Restates, for one node per thread, the small dense kernels the reference
// calls inside its force loop: INV3 (INVERSE.F90:119-152), DETERMINANT
// (DETERMINANT.F90:18-35), HUGHES_WINGET (HUGHES_WINGET.F90:16-81),
// ROTATE_TENSOR (ROTATE_TENSOR.F90:21-87), VON_MISES
// (CONSTITUTE_VONMISES.F90:21-158), ESTIMATE_MODULI (ESTIMATE_MODULI.F90:
// 16-86), the cubic B-spline MLS_KERNEL0 (KERNEL.F90:57-71) and the 4x4
// cofactor inverse M44INV (INVERSE.F90:185-223).  Templated on the working
// type T so the mixed-precision path runs the same code in float.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/mega_gpu.h"

namespace mega {

template <typename T> __device__ __forceinline__ T dsqrt(T x);
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }

// 3x3 row-major in registers
template <typename T> struct Mat3 { T a[3][3]; };

template <typename T>
__device__ __forceinline__ void mm3(const T a[3][3], const T b[3][3], T c[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}

// INV3 as written returns det*adj(A) = det^2 * A^-1; exact divides instead.
template <typename T>
__device__ __forceinline__ void inv3(const T a[3][3], T r[3][3], bool exact) {
  T det = a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1] - a[0][1] * a[1][0] * a[2][2] +
          a[0][1] * a[1][2] * a[2][0] + a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
  T s = exact ? T(1) / det : det;
  r[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * s;
  r[1][0] = -(a[1][0] * a[2][2] - a[1][2] * a[2][0]) * s;
  r[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * s;
  r[0][1] = -(a[0][1] * a[2][2] - a[0][2] * a[2][1]) * s;
  r[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * s;
  r[2][1] = -(a[0][0] * a[2][1] - a[0][1] * a[2][0]) * s;
  r[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * s;
  r[1][2] = -(a[0][0] * a[1][2] - a[0][2] * a[1][0]) * s;
  r[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * s;
}

template <typename T>
__device__ __forceinline__ T det_abs(const T a[3][3]) {
  return fabs(a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2]) +
              a[0][1] * (a[2][0] * a[1][2] - a[1][0] * a[2][2]) +
              a[0][2] * (a[1][0] * a[2][1] - a[2][0] * a[1][1]));
}

// Gauss-Jordan with full pivoting (INVERSE.F90:17-99) for 3x3; false when a
// pivot is negligible (the reference's L = 0).
__device__ __forceinline__ bool inverse3_gj(const double a[3][3], double r[3][3]) {
  int is[3], js[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i][j] = a[i][j];
  for (int k = 0; k < 3; ++k) {
    double d = 0.0;
    is[k] = k; js[k] = k;
    for (int i = k; i < 3; ++i)
      for (int j = k; j < 3; ++j)
        if (fabs(r[i][j]) > d) { d = fabs(r[i][j]); is[k] = i; js[k] = j; }
    if (d + 1.0 == 1.0) return false;
    for (int j = 0; j < 3; ++j) { double t = r[k][j]; r[k][j] = r[is[k]][j]; r[is[k]][j] = t; }
    for (int i = 0; i < 3; ++i) { double t = r[i][k]; r[i][k] = r[i][js[k]]; r[i][js[k]] = t; }
    r[k][k] = 1.0 / r[k][k];
    for (int j = 0; j < 3; ++j) if (j != k) r[k][j] = r[k][j] * r[k][k];
    for (int i = 0; i < 3; ++i)
      if (i != k)
        for (int j = 0; j < 3; ++j)
          if (j != k) r[i][j] = r[i][j] - r[i][k] * r[k][j];
    for (int i = 0; i < 3; ++i) if (i != k) r[i][k] = -r[i][k] * r[k][k];
  }
  for (int k = 2; k >= 0; --k) {
    for (int j = 0; j < 3; ++j) { double t = r[k][j]; r[k][j] = r[js[k]][j]; r[js[k]][j] = t; }
    for (int i = 0; i < 3; ++i) { double t = r[i][k]; r[i][k] = r[i][is[k]]; r[i][is[k]] = t; }
  }
  return true;
}

// Voigt (xx,yy,zz,yz,xz,xy) <-> tensor (FINT_FUNCTIONS.F90:10-65)
template <typename T>
__device__ __forceinline__ void v2t(const T v[6], T t[3][3]) {
  t[0][0] = v[0]; t[1][1] = v[1]; t[2][2] = v[2];
  t[2][1] = v[3]; t[1][2] = v[3];
  t[0][2] = v[4]; t[2][0] = v[4];
  t[0][1] = v[5]; t[1][0] = v[5];
}
template <typename T>
__device__ __forceinline__ void t2v(const T t[3][3], T v[6]) {
  v[0] = t[0][0]; v[1] = t[1][1]; v[2] = t[2][2];
  v[3] = t[1][2]; v[4] = t[0][2]; v[5] = t[0][1];
}

// HUGHES_WINGET.F90:16-81
template <typename T>
__device__ __forceinline__ void hughes_winget(const T L[3][3], T rot[3][3], T strain[6], T d[6],
                                              bool exact) {
  T A[3][3], Ai[3][3], G[3][3], W[3][3], IW[3][3], IWi[3][3], t[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) A[i][j] = (i == j ? T(1) : T(0)) + T(0.5) * L[i][j];
  inv3(A, Ai, exact);
  mm3(L, Ai, G);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) W[i][j] = T(0.5) * (G[i][j] - G[j][i]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) IW[i][j] = (i == j ? T(1) : T(0)) - T(0.5) * W[i][j];
  inv3(IW, IWi, exact);
  mm3(IWi, W, t);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) rot[i][j] = (i == j ? T(1) : T(0)) + t[i][j];
  d[3] = T(0.5) * (G[1][2] + G[2][1]);
  d[4] = T(0.5) * (G[0][2] + G[2][0]);
  d[5] = T(0.5) * (G[0][1] + G[1][0]);
  d[0] = T(0.5) * (G[0][0] + G[0][0]);
  d[1] = T(0.5) * (G[1][1] + G[1][1]);
  d[2] = T(0.5) * (G[2][2] + G[2][2]);
#pragma unroll
  for (int k = 0; k < 6; ++k) strain[k] = d[k];
  strain[3] = T(2) * strain[3]; strain[4] = T(2) * strain[4]; strain[5] = T(2) * strain[5];
}

// ROTATE_TENSOR.F90:21-87: v <- R v R^T (shear entries treated as tensor
// components, as the reference does for the engineering-shear strain too)
template <typename T>
__device__ __forceinline__ void rotate_tensor(const T R[3][3], T v[6]) {
  T S[3][3], tmp[3][3], o[3][3];
  v2t(v, S);
  mm3(R, S, tmp);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) o[i][j] = tmp[i][0] * R[j][0] + tmp[i][1] * R[j][1] + tmp[i][2] * R[j][2];
  t2v(o, v);
}

template <typename T>
__device__ __forceinline__ T tensor_norm(const T v[6]) {
  return dsqrt<T>(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + T(2) * (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]));
}
template <typename T>
__device__ __forceinline__ T tensor_norm_strain(const T v[6]) {
  return dsqrt<T>(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]));
}

// The per-node deformation gradient F and increment gradient G0 between the
// row gather and the stress update.  FP64: 18 doubles, F with its identity.
// Mixed precision: 18 floats holding F - I and G0 (half the bytes; the
// identity is added back in double when read, so F keeps its FP64 unit part
// and the float carries only the displacement gradient, itself a float sum).
// h[0..8] = F - I, h[9..17] = G0, row-major.
__device__ __forceinline__ void store_fg(double* fg, int64_t i, bool mixed, const double h[18]) {
  if (mixed) {
    float2* o = reinterpret_cast<float2*>(reinterpret_cast<float*>(fg) + 18 * i);
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = make_float2((float)h[2 * k], (float)h[2 * k + 1]);
  } else {
    double* o = fg + 18 * i;
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = ((k % 4) == 0 ? 1.0 : 0.0) + h[k];
#pragma unroll
    for (int k = 9; k < 18; ++k) o[k] = h[k];
  }
}
// F (with its identity) in f[0..8], G0 in f[9..17]
__device__ __forceinline__ void load_fg(const double* fg, int64_t i, bool mixed, double f[18]) {
  if (mixed) {
    const float2* g = reinterpret_cast<const float2*>(reinterpret_cast<const float*>(fg) + 18 * i);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float2 v = g[k];
      f[2 * k] = (double)v.x;
      f[2 * k + 1] = (double)v.y;
    }
#pragma unroll
    for (int k = 0; k < 9; k += 4) f[k] = 1.0 + f[k];
  } else {
    const double2* g = reinterpret_cast<const double2*>(fg + 18 * i);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double2 v = g[k];
      f[2 * k] = v.x;
      f[2 * k + 1] = v.y;
    }
  }
}

// Per-node material constants the force kernel needs (from PROPS(30,N)).
struct NodeMat {
  int32_t type;
  double nu, E, rho, sig0, B, C;     // PROPS(1..6)
  double lam, mu, l2m;                // PROPS(28..30)
  double p7, p8;                      // PROPS(7..8) (rate-dependent law)
};

// Radial return of CONSTITUTE_VONMISES.F90:21-158 in FP64 (the residual
// check stays FP64 in every mode).  spred = elastic predictor; returns the
// Newton passes; *cap set on hitting maxit.
__device__ __forceinline__ int von_mises(const double spred[6], double& eps, const NodeMat& m,
                                         int maxit, double stress[6], bool& cap) {
  const double mu = m.E / (2.0 * (1.0 + m.nu));
  const double kk = spred[0] + spred[1] + spred[2];
  double dev[6];
  dev[0] = spred[0] - kk / 3.0; dev[1] = spred[1] - kk / 3.0; dev[2] = spred[2] - kk / 3.0;
  dev[3] = spred[3]; dev[4] = spred[4]; dev[5] = spred[5];
  const double sph = -kk / 3.0;
  const double tn = tensor_norm(dev);
  const double s23 = sqrt(2.0 / 3.0);
  const double sig23 = s23 * m.sig0;
  const double tol = sig23 * (double)1.0e-5f;  // single-precision literal 1.0E-05
  // (1 + B eps)^C and its derivative factor (1 + B eps)^(C - 1); linear
  // hardening (C = 1) needs neither power: x^1 = x and x^0 = 1 exactly
  const bool lin = m.C == 1.0;
  double xk = sig23 * (lin ? 1.0 + m.B * eps : pow(1.0 + m.B * eps, m.C));
  int it = 0;
  if (tn - xk > 0.0) {
    double dg = 0.0;
    const double epst = eps;
    for (int i = 1; i <= maxit; ++i) {
      ++it;
      xk = sig23 * (lin ? 1.0 + m.B * eps : pow(1.0 + m.B * eps, m.C));
      const double y = tn - xk - (2.0 * mu * dg);
      if (fabs(y) > tol) {
        const double xkp = m.B * m.C * m.sig0 * (lin ? 1.0 : pow(1.0 + m.B * eps, m.C - 1.0));
        const double dy = -2.0 * mu * (1.0 + xkp / 3.0 / mu);
        dg = dg - y / dy;
        if (i == maxit) cap = true;
      } else {
        eps = epst + s23 * dg;
        break;
      }
      eps = epst + s23 * dg;
    }
    const double sc = dg * 2.0 * mu / tn;
#pragma unroll
    for (int k = 0; k < 6; ++k) dev[k] = dev[k] - sc * dev[k];
  }
  stress[0] = -sph + dev[0]; stress[1] = -sph + dev[1]; stress[2] = -sph + dev[2];
  stress[3] = dev[3]; stress[4] = dev[4]; stress[5] = dev[5];
  return it;
}

// The damaged models keep four more state values per node,
// aux = {EPS_SHEAR, EPS_VOL, DAM, DAM_SV} = STATE(1, 2, 4, 5), and read
// PROPS(9..11) and PROPS(25..27).
struct DamageMat {
  double ki, kc, dmax;      // K_I, K_C, DAM_MAX
  double qphi, kphi, qpsi;  // Q_PHI, K_PHI, Q_PSI (Drucker-Prager)
};

// Damage of CONSTITUTE_VONMISES_DAM.F90:94-125 / CONSTITUTE_DRUCKPRAG.F90:
// 84-113: eta = TENSOR_NORM(total strain) (the stress-norm weighting, as
// written); once eta passes DAM_SV + K_I and while K_I < eta < K_C the
// damage is K_C (eta - K_I) / (eta (K_C - K_I)) and DAM_SV = eta - K_I;
// capped at DAM_MAX.
__device__ __forceinline__ void damage_update(const double tot[6], const DamageMat& d, double& dam, double& dsv) {
  const double eta = tensor_norm(tot);
  if (eta < dsv + d.ki) {
  } else if (eta > d.ki && eta < d.kc) {
    dam = d.kc * (eta - d.ki) / (eta * (d.kc - d.ki));
    dsv = eta - d.ki;
  }
  if (dam > d.dmax) dam = d.dmax;
}

// VON_MISES_DAM (CONSTITUTE_VONMISES_DAM.F90:21-196).  eff = the effective
// predictor STRESS / (1 - DAM) + C dstrain (formed by the caller from the
// rotated old stress); the radial return of VON_MISES in effective space
// (the same Newton iteration and tolerance), then back to the real stress
// with the new damage.
__device__ __forceinline__ int von_mises_dam(const double eff[6], const double tot[6], double& eps, double aux[4],
                                             const NodeMat& m, const DamageMat& d, int maxit, double stress[6],
                                             bool& cap) {
  damage_update(tot, d, aux[2], aux[3]);
  const int it = von_mises(eff, eps, m, maxit, stress, cap);
  const double keep = 1.0 - aux[2];
#pragma unroll
  for (int k = 0; k < 6; ++k) stress[k] = stress[k] * keep;
  return it;
}

// DRUCK_PRAG (CONSTITUTE_DRUCKPRAG.F90:17-241): shear yield
// f = |dev| + Q_PHI p - K_PHI (p = tr/3 of the effective predictor), a
// closed-form return with non-associated dilatancy Q_PSI, then the real
// stress with the new damage.  The tension cut-off branch is unreachable as
// written (its flag is never set) and is not restated.  Returns 1 on a
// plastic return.
__device__ __forceinline__ int drucker_prager(const double eff[6], const double tot[6], double& eps, double aux[4],
                                              const NodeMat& m, const DamageMat& d, double stress[6]) {
  damage_update(tot, d, aux[2], aux[3]);
  const double kk = eff[0] + eff[1] + eff[2];
  double dev[6];
  dev[0] = eff[0] - kk / 3.0; dev[1] = eff[1] - kk / 3.0; dev[2] = eff[2] - kk / 3.0;
  dev[3] = eff[3]; dev[4] = eff[4]; dev[5] = eff[5];
  const double tau_pre = tensor_norm(dev);
  const double sph_pre = kk / 3.0;
  const double f = tau_pre + d.qphi * sph_pre - d.kphi;
  int plastic = 0;
  if (f < 0.0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) stress[k] = eff[k];
  } else {
    const double tau = d.kphi - d.qphi * sph_pre;
    const double bulk = m.E / (3.0 * (1.0 - 2.0 * m.nu)), shear = m.E / (2.0 * (1.0 + m.nu));
    const double gamma = f / (2.0 * shear + bulk * d.qphi * d.qpsi);
    const double sph = sph_pre - bulk * d.qpsi * gamma;
#pragma unroll
    for (int k = 0; k < 6; ++k) stress[k] = dev[k] * tau / tau_pre;
    stress[0] += sph; stress[1] += sph; stress[2] += sph;
    aux[0] = aux[0] + gamma * sqrt(2.0 / 3.0 + 2.0 / 9.0 * d.qpsi * d.qpsi);
    eps = eps + aux[0];  // EPS accumulates the running EPS_SHEAR, as written
    plastic = 1;
  }
  const double keep = 1.0 - aux[2];
#pragma unroll
  for (int k = 0; k < 6; ++k) stress[k] = stress[k] * keep;
  return plastic;
}

// Power-law rate-dependent J2 return mapping (no reference counterpart):
// sigma_y = A + B*ep^n*(1 + C*ln(max(epdot,epdot0)/epdot0)), epdot =
// sqrt(2/3)*dg/dt.  Safeguarded Newton on dg in [0, q/(2mu)], converged at
// |f| <= rtol*sqrt(2/3)*sigma_y.  dg0 < 0 selects the plain start f_tr/(2mu).
// Upper bound of the rate-dependent plastic multiplier for a trial overstress
// f0 > 0 at plastic strain eps0: the smaller of the perfectly plastic value
// f0 / (2 mu) and the pure power-law value ((eps0^n + f0 / (sqrt(2/3) B))^(1/n)
// - eps0) / sqrt(2/3); both bound the root because the rate factor is >= 1
// and 2 mu dg >= 0.
__device__ __forceinline__ double rate_upper_bound(double f0, double eps0, double mu, double B, double nexp) {
  const double s23 = sqrt(2.0 / 3.0);
  double hi = f0 / (2.0 * mu);
  if (B > 0.0) {
    const double epn0 = (eps0 > 0.0) ? pow(eps0, nexp) : 0.0;
    const double pw = (pow(epn0 + f0 / (s23 * B), 1.0 / nexp) - eps0) / s23;
    if (pw > 0.0 && pw < hi) hi = pw;
  }
  return hi;
}

// Power-law rate-dependent J2 (material 7, no reference counterpart):
// sy = A + B eps^n (1 + C ln(epsdot / epsdot0)) for epsdot > epsdot0, with
// epsdot = sqrt(2/3) dg / dt.  Radial return solved by Newton in y = ln(dg)
// from the upper bound (f is concave in y, so the iterates decrease
// monotonically onto the root from the right), with bracket and bisection
// in y as the guard; converged when |f| <= rtol sqrt(2/3) sy or when an
// update no longer changes dg beyond its rounding.  dg0 >= 0
// starts there instead (clamped into the bracket).  solver = 1 is the
// textbook form kept for comparison: Newton in dg from the perfectly plastic
// estimate f_trial / (2 mu), bracket [0, q / (2 mu)], arithmetic bisection.
// Returns the iterations.
__device__ __forceinline__ int vm_rate(const double spred[6], double& eps, const NodeMat& m, double dt,
                                       double rtol, int maxit, int solver, double dg0, double stress[6],
                                       bool& cap, double& dg_out, double& f_tr) {
  const double mu = m.E / (2.0 * (1.0 + m.nu));
  const double A = m.sig0, Bh = m.B, nexp = m.C, C = m.p7, ed0 = m.p8;
  const double kk = spred[0] + spred[1] + spred[2];
  double dev[6];
  dev[0] = spred[0] - kk / 3.0; dev[1] = spred[1] - kk / 3.0; dev[2] = spred[2] - kk / 3.0;
  dev[3] = spred[3]; dev[4] = spred[4]; dev[5] = spred[5];
  const double sph = -kk / 3.0;
  const double tn = tensor_norm(dev);
  const double s23 = sqrt(2.0 / 3.0);
  const double eps0 = eps;
  double epn0 = (eps0 > 0.0) ? pow(eps0, nexp) : 0.0;
  f_tr = tn - s23 * (A + Bh * epn0);
  int it = 0;
  double dg = 0.0;
  if (f_tr > 0.0) {
    const bool textbook = solver == 1;
    double lo = 0.0, hi = textbook ? tn / (2.0 * mu) : rate_upper_bound(f_tr, eps0, mu, Bh, nexp);
    dg = (dg0 >= 0.0) ? dg0 : (textbook ? f_tr / (2.0 * mu) : hi);
    if (textbook ? !(dg > lo && dg < hi) : !(dg > lo && dg <= hi)) dg = textbook ? 0.5 * (lo + hi) : hi;
    bool conv = false;
    if (textbook) {
      for (int i = 1; i <= maxit; ++i) {
        ++it;
        const double ep = eps0 + s23 * dg;
        const double ed = s23 * dg / dt;
        double rate = 1.0, drate = 0.0;
        if (ed > ed0) { rate = 1.0 + C * log(ed / ed0); drate = C / dg; }
        const double epn = (ep > 0.0) ? pow(ep, nexp) : 0.0;
        const double depn = (ep > 0.0) ? nexp * pow(ep, nexp - 1.0) * s23 : 0.0;
        const double sy = A + Bh * epn * rate;
        const double f = tn - 2.0 * mu * dg - s23 * sy;
        if (fabs(f) <= rtol * s23 * sy) { conv = true; break; }
        if (f > 0.0) lo = dg; else hi = dg;
        const double df = -2.0 * mu - s23 * Bh * (depn * rate + epn * drate);
        double nd = dg - f / df;
        if (!(nd > lo && nd < hi) || !isfinite(nd)) nd = 0.5 * (lo + hi);
        const bool stalled = fabs(nd - dg) <= 4.0e-16 * dg;  // below the rounding of dg
        dg = nd;
        if (stalled) { conv = true; break; }
      }
    } else {
      // the iterate is y = ln(dg); ln(epsdot / epsdot0) = y - ythr, and
      // eps^n = exp(n ln eps): three transcendentals per iteration
      const double ythr = log(ed0 * dt / s23);
      double y = log(dg), ylo = -INFINITY, yhi = log(hi);
      for (int i = 1; i <= maxit; ++i) {
        ++it;
        const double ep = eps0 + s23 * dg;
        const double epn = exp(nexp * log(ep));
        const double depn = nexp * epn / ep * s23;
        double rate = 1.0, drate = 0.0;
        if (y > ythr) { rate = 1.0 + C * (y - ythr); drate = C / dg; }
        const double sy = A + Bh * epn * rate;
        const double f = tn - 2.0 * mu * dg - s23 * sy;
        if (fabs(f) <= rtol * s23 * sy) { conv = true; break; }
        if (f > 0.0) ylo = y; else yhi = y;
        const double df = -2.0 * mu - s23 * Bh * (depn * rate + epn * drate);
        double yn = y + fmax(fmin(-f / (df * dg), 50.0), -50.0);
        if (!(yn > ylo && yn < yhi) || !isfinite(yn))
          yn = isfinite(ylo) ? 0.5 * (ylo + yhi) : yhi - 0.69314718055994530942;  // bisect in y
        const bool stalled = fabs(yn - y) <= 4.0e-16;  // below the rounding of dg
        y = yn;
        dg = exp(y);
        if (stalled) { conv = true; break; }
      }
    }
    if (!conv) cap = true;
    const double sc = dg * 2.0 * mu / tn;
#pragma unroll
    for (int k = 0; k < 6; ++k) dev[k] = dev[k] - sc * dev[k];
    eps = eps0 + s23 * dg;
  }
  dg_out = dg;
  stress[0] = -sph + dev[0]; stress[1] = -sph + dev[1]; stress[2] = -sph + dev[2];
  stress[3] = dev[3]; stress[4] = dev[4]; stress[5] = dev[5];
  return it;
}

// ESTIMATE_MODULI.F90:16-86 with NSNI_FLAG = .FALSE.
__device__ __forceinline__ void estimate_moduli(const double sinc[6], const double einc[6], double& shear,
                                                double& bulk) {
  const double sk = sinc[0] + sinc[1] + sinc[2], ek = einc[0] + einc[1] + einc[2];
  double sd[6] = {sinc[0] - sk / 3.0, sinc[1] - sk / 3.0, sinc[2] - sk / 3.0, sinc[3], sinc[4], sinc[5]};
  double ss[6] = {-sk / 3.0, -sk / 3.0, -sk / 3.0, 0.0, 0.0, 0.0};
  double ed[6] = {einc[0] - ek / 3.0, einc[1] - ek / 3.0, einc[2] - ek / 3.0, einc[3], einc[4], einc[5]};
  double es[6] = {-ek / 3.0, -ek / 3.0, -ek / 3.0, 0.0, 0.0, 0.0};
  const double nsd = tensor_norm(sd), nss = tensor_norm(ss);
  const double ned = tensor_norm_strain(ed), nes = tensor_norm_strain(es);
  double st = (ned > 1.0e-8 && nsd > 1.0e-8) ? nsd / ned / 2.0 : shear;
  st = fmax(st, shear * 0.5);
  st = fmin(st, shear);
  shear = st;
  double bt = (nes > 1.0e-8 && nss > 1.0e-8) ? nss / nes / 3.0 : bulk;
  bt = fmax(bt, bulk * 0.5);
  bt = fmin(bt, bulk);
  bulk = bt;
}

// MLS_KERNEL0 (KERNEL.F90:57-71), cubic B-spline, ISPLINE = 3
template <typename T>
__device__ __forceinline__ void bspline3(T r, T& w, T& dw) {
  if (r <= T(0.5)) {
    w = T(2.0 / 3.0) - T(4) * r * r + T(4) * r * r * r;
    dw = T(-8) * r + T(12) * r * r;
  } else if (r <= T(1)) {
    w = T(4.0 / 3.0) - T(4) * r + T(4) * r * r - T(4.0 / 3.0) * r * r * r;
    dw = T(-4) + T(8) * r - T(4) * r * r;
  } else {
    w = T(0);
    dw = T(0);
  }
}

__device__ __forceinline__ double det3r(const double* r0, const double* r1, const double* r2) {
  return r0[0] * (r1[1] * r2[2] - r1[2] * r2[1]) + r0[1] * (r1[2] * r2[0] - r1[0] * r2[2]) +
         r0[2] * (r1[0] * r2[1] - r1[1] * r2[0]);
}

// M44INV (INVERSE.F90:185-223): cofactor inverse of a symmetric 4x4 moment
// matrix, FP64.  Returns the determinant.
__device__ __forceinline__ double m44inv(const double a[4][4], double r[4][4]) {
  double cof[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double m[3][3];
      int ri = 0;
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        if (p == i) continue;
        int cj = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (q == j) continue;
          m[ri][cj++] = a[p][q];
        }
        ++ri;
      }
      const double d = det3r(m[0], m[1], m[2]);
      cof[i][j] = ((i + j) & 1) ? -d : d;
    }
  const double det = a[0][0] * cof[0][0] + a[0][1] * cof[0][1] + a[0][2] * cof[0][2] + a[0][3] * cof[0][3];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) r[i][j] = cof[j][i] / det;
  return det;
}

}  // namespace mega
