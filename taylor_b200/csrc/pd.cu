// pd.cu -- peridynamic forces.
//
// 1. Correspondence ("non-ordinary state-based") peridynamics of
//    CONSTRUCT_FINT_PD (FINT_PD.F90:214-684), Lagrangian, HODIV = .FALSE.:
//    influence w_iJ = box cubic spline, K_i = sum_J xi xi^T w V_J and its
//    full-pivot inverse (UDFM_SHAPE_TENSOR, RK.f90:579-726); per step
//    F = S K^-1 with S = sum_J (x_J - x_i) xi^T w V_J (DFM_SHAPE_TENSOR,
//    RK.f90:730-807), L = (sum_J (du_J - du_i) xi^T w V_J) K^-1 F^-1, the
//    same Hughes-Winget / return mapping as the RKPM path, P = J sigma F^-T
//    and the pair forces FINT3 = P K^-1 (X_i - X_J):
//       f_J -= FINT3 V_i w V_J,   f_i += FINT3 V_J w V_i   (FINT_PD.F90:629-655).
//    With A_i = P_i K_i^-1 the force on node k is
//       f_k = V_k [ A_k s_k - sum_{i: k in N(i)} A_i (X_i - X_k) w_ik V_i ],
//    s_k = sum_J (X_k - X_J) w_kJ V_J (static), gathered over the transposed
//    list without atomics.
// 2. Bond-based prototype-microelastic-brittle peridynamics (no reference
//    counterpart; Silling & Askari 2005): f_i = sum_j c s mu (y_j - y_i)/|.|
//    V_j, a bond breaks for good when its stretch exceeds s_c.  Each bond is
//    evaluated from both ends with bitwise-identical arithmetic, so both
//    copies break in the same step.  Float force arithmetic, double
//    positions and velocity-Verlet integration.
#include <cstring>
#include <mutex>
#include <set>
#include "mega_internal.cuh"
#include "tiled.cuh"

namespace mega {
namespace {

constexpr int kG = 4;

__device__ __forceinline__ double box_w(double r) {
  double w, dw;
  bspline3(fabs(r), w, dw);
  return w;
}

// UDFM_SHAPE_TENSOR: influence functions, K^-1 (column-major (3,3,n)) and s_i
__global__ void k_pd_shape(int32_t n, const double* __restrict__ X, const double* __restrict__ win,
                           const double* __restrict__ vol, const int64_t* __restrict__ rowptr,
                           const int32_t* __restrict__ col, double* __restrict__ shp, double* __restrict__ ginvk,
                           double* __restrict__ svec, unsigned* __restrict__ status) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kG;
  const int q = threadIdx.x & (kG - 1);
  const unsigned gm = 0xFu << (threadIdx.x & 28);
  if (i >= n) return;
  const double xi0 = X[3 * i], xi1 = X[3 * i + 1], xi2 = X[3 * i + 2];
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, s[3] = {0, 0, 0};
  for (int64_t p = rowptr[i] + q; p < rowptr[i + 1]; p += kG) {
    const int64_t j = col[p];
    const double h0 = -(xi0 - X[3 * j]), h1 = -(xi1 - X[3 * j + 1]), h2 = -(xi2 - X[3 * j + 2]);
    const double w = box_w(h0 / win[3 * j]) * box_w(h1 / win[3 * j + 1]) * box_w(h2 / win[3 * j + 2]);
    const double vw = w * vol[j];
    K[0] += h0 * h0 * vw; K[1] += h0 * h1 * vw; K[2] += h0 * h2 * vw;
    K[4] += h1 * h1 * vw; K[5] += h1 * h2 * vw; K[8] += h2 * h2 * vw;
    s[0] -= h0 * vw; s[1] -= h1 * vw; s[2] -= h2 * vw;
    shp[p] = w;
  }
#pragma unroll
  for (int o = 1; o < kG; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 9; ++k) K[k] += __shfl_xor_sync(gm, K[k], o);
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] += __shfl_xor_sync(gm, s[k], o);
  }
  if (q == 0) {
    double A[3][3] = {{K[0], K[1], K[2]}, {K[1], K[4], K[5]}, {K[2], K[5], K[8]}}, R[3][3];
    if (!inverse3_gj(A, R)) atomicOr(status, (unsigned)MEGA_ST_SINGULAR_SHAPE);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) ginvk[9 * i + 3 * b + a] = R[a][b];
    svec[3 * i] = s[0]; svec[3 * i + 1] = s[1]; svec[3 * i + 2] = s[2];
  }
}

// static s_k when the influence functions come from the caller
__global__ void k_pd_svec(int32_t n, const double* __restrict__ X, const double* __restrict__ vol,
                          const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                          const double* __restrict__ shp, double* __restrict__ svec) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
    const int64_t j = col[p];
    const double vw = shp[p] * vol[j];
    s0 += (X[3 * i] - X[3 * j]) * vw; s1 += (X[3 * i + 1] - X[3 * j + 1]) * vw; s2 += (X[3 * i + 2] - X[3 * j + 2]) * vw;
  }
  svec[3 * i] = s0; svec[3 * i + 1] = s1; svec[3 * i + 2] = s2;
}

// DFM_SHAPE_TENSOR twice: S (current coordinates) and the increment tensor
__global__ void k_pd_defgrad(int32_t n, const double* __restrict__ X, const double* __restrict__ xc,
                             const double* __restrict__ du, const double* __restrict__ vol,
                             const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                             const double* __restrict__ shp, double* __restrict__ fg) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kG;
  const int q = threadIdx.x & (kG - 1);
  const unsigned gm = 0xFu << (threadIdx.x & 28);
  if (i >= n) return;
  double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double X0[3] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
  const double x0[3] = {xc[3 * i], xc[3 * i + 1], xc[3 * i + 2]};
  const double d0[3] = {du[3 * i], du[3 * i + 1], du[3 * i + 2]};
  for (int64_t p = rowptr[i] + q; p < rowptr[i + 1]; p += kG) {
    const int64_t j = col[p];
    const double vw = shp[p] * vol[j];
    const double h[3] = {X[3 * j] - X0[0], X[3 * j + 1] - X0[1], X[3 * j + 2] - X0[2]};
    const double hs[3] = {xc[3 * j] - x0[0], xc[3 * j + 1] - x0[1], xc[3 * j + 2] - x0[2]};
    const double hd[3] = {du[3 * j] - d0[0], du[3 * j + 1] - d0[1], du[3 * j + 2] - d0[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        S[3 * a + b] += hs[a] * h[b] * vw;
        L[3 * a + b] += hd[a] * h[b] * vw;
      }
  }
#pragma unroll
  for (int o = 1; o < kG; o <<= 1)
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      S[k] += __shfl_xor_sync(gm, S[k], o);
      L[k] += __shfl_xor_sync(gm, L[k], o);
    }
  if (q == 0)
    for (int k = 0; k < 9; ++k) { fg[18 * i + k] = S[k]; fg[18 * i + 9 + k] = L[k]; }
}

struct PdStressArgs {
  int32_t n;
  const double* fg;
  const double* ginvk;
  const uint16_t* matidx;
  const MatEntry* mats;
  double* stress;
  double* strain;
  double* eps;
  double* wvel;
  double* amat;  // 9 per node, row-major A_i = P_i K_i^-1
  double* aux;   // 4 per node: STATE(1, 2, 4, 5) of the damaged models (or null)
  int linit;
  int inv3_exact;
  int maxit;
  int rate_solver;
  double rtol;
  double dt;
  unsigned* status;
};

__global__ void k_pd_stress(PdStressArgs a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double* g = a.fg + 18 * i;
  double Ki[3][3], F[3][3], IF[3][3], Ld[3][3], L[3][3], t[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) { Ki[r][c] = a.ginvk[9 * i + 3 * c + r]; Ld[r][c] = g[9 + 3 * r + c]; }
  double det = 1.0;
  unsigned st = 0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) IF[r][c] = (r == c) ? 1.0 : 0.0;
  if (!a.linit) {
    double S[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) S[r][c] = g[3 * r + c];
    mm3(S, Ki, F);
    det = det_abs(F);
    if (!inverse3_gj(F, IF)) st |= MEGA_ST_SINGULAR_SHAPE;
  }
  mm3(Ld, Ki, t);
  if (!a.linit) mm3(t, IF, L);
  else
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) L[r][c] = t[r][c];
  double R[3][3], dstr[6], D[6], sig[6], e6[6], sold[6];
  hughes_winget(L, R, dstr, D, a.inv3_exact != 0);
  for (int k = 0; k < 6; ++k) { sold[k] = a.stress[6 * i + k]; sig[k] = sold[k]; e6[k] = a.strain[6 * i + k]; }
  rotate_tensor(R, sig);
  rotate_tensor(R, e6);
  for (int k = 0; k < 6; ++k) e6[k] += dstr[k];
  const MatEntry me = a.mats[a.matidx[i]];
  NodeMat m;
  m.type = me.type; m.nu = me.nu; m.E = me.E; m.rho = me.rho; m.sig0 = me.sig0; m.B = me.B; m.C = me.C;
  m.lam = me.lam; m.mu = me.mu; m.l2m = me.l2m; m.p7 = me.p7; m.p8 = me.p8;
  if (damaged_type(me.type)) {  // effective-space predictor of the damaged models
    const double keep = 1.0 - a.aux[4 * i + 2];
    for (int k = 0; k < 6; ++k) sig[k] = sig[k] / keep;
  }
  double sp[6];
  sp[0] = sig[0] + (me.l2m * dstr[0] + me.lam * dstr[1] + me.lam * dstr[2]);
  sp[1] = sig[1] + (me.lam * dstr[0] + me.l2m * dstr[1] + me.lam * dstr[2]);
  sp[2] = sig[2] + (me.lam * dstr[0] + me.lam * dstr[1] + me.l2m * dstr[2]);
  sp[3] = sig[3] + me.mu * dstr[3];
  sp[4] = sig[4] + me.mu * dstr[4];
  sp[5] = sig[5] + me.mu * dstr[5];
  double sn[6];
  double ep = a.eps[i];
  bool cap = false;
  if (m.type == MEGA_MAT_ELASTIC) {
    for (int k = 0; k < 6; ++k) sn[k] = sp[k];
  } else if (m.type == MEGA_MAT_VONMISES) {
    von_mises(sp, ep, m, a.maxit, sn, cap);
  } else if (m.type == MEGA_MAT_VM_RATE) {
    double dg, ftr;
    vm_rate(sp, ep, m, a.dt, a.rtol, a.maxit, a.rate_solver, -1.0, sn, cap, dg, ftr);
  } else if (damaged_type(m.type)) {
    double* ax = a.aux + 4 * i;
    const DamageMat d{me.ki, me.kc, me.dmax, me.qphi, me.kphi, me.qpsi};
    if (m.type == MEGA_MAT_VM_DAMAGE) von_mises_dam(sp, e6, ep, ax, m, d, a.maxit, sn, cap);
    else drucker_prager(sp, e6, ep, ax, m, d, sn);
  } else {
    st |= MEGA_ST_BAD_MATERIAL;
    for (int k = 0; k < 6; ++k) sn[k] = sp[k];
  }
  if (cap) st |= MEGA_ST_NEWTON_CAP;
  double sinc[6], einc[6];
  for (int k = 0; k < 6; ++k) {
    sinc[k] = sn[k] - sold[k];
    einc[k] = e6[k] - sold[k];  // FINT_PD.F90:509 subtracts the old STRESS (kept as written)
    a.stress[6 * i + k] = sn[k];
    a.strain[6 * i + k] = e6[k];
  }
  a.eps[i] = ep;
  double bulk = m.E / (3.0 * (1.0 - 2.0 * m.nu)), shear = m.E / (2.0 * (1.0 + m.nu));
  if (m.type > 1) estimate_moduli(sinc, einc, shear, bulk);
  double wv = sqrt(fmax(bulk + 4.0 * shear / 3.0, shear) / m.rho);
  if (m.type == 3) wv = wv / 0.15;
  a.wvel[i] = wv;
  // P = det sigma IF^T ; A = P K^-1
  double Sg[3][3], P[3][3], A[3][3];
  v2t(sn, Sg);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) P[r][c] = det * (Sg[r][0] * IF[c][0] + Sg[r][1] * IF[c][1] + Sg[r][2] * IF[c][2]);
  mm3(P, Ki, A);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a.amat[9 * i + 3 * r + c] = A[r][c];
  for (int k = 0; k < 6; ++k)
    if (!isfinite(sn[k])) st |= MEGA_ST_NONFINITE;
  if (st) atomicOr(a.status, st);
}

__global__ void k_pd_force(int32_t n, const double* __restrict__ X, const double* __restrict__ vol,
                           const int64_t* __restrict__ colptr, const int32_t* __restrict__ trow,
                           const int64_t* __restrict__ tpos, const double* __restrict__ shp,
                           const double* __restrict__ amat, const double* __restrict__ svec,
                           double* __restrict__ fint) {
  const int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kG;
  const int q = threadIdx.x & (kG - 1);
  const unsigned gm = 0xFu << (threadIdx.x & 28);
  if (k >= n) return;
  const double xk0 = X[3 * k], xk1 = X[3 * k + 1], xk2 = X[3 * k + 2];
  double f0 = 0, f1 = 0, f2 = 0;
  for (int64_t e = colptr[k] + q; e < colptr[k + 1]; e += kG) {
    const int64_t i = trow[e];
    const double w = shp[tpos[e]] * vol[i];
    const double d0 = (X[3 * i] - xk0) * w, d1 = (X[3 * i + 1] - xk1) * w, d2 = (X[3 * i + 2] - xk2) * w;
    const double* A = amat + 9 * i;
    f0 -= A[0] * d0 + A[1] * d1 + A[2] * d2;
    f1 -= A[3] * d0 + A[4] * d1 + A[5] * d2;
    f2 -= A[6] * d0 + A[7] * d1 + A[8] * d2;
  }
#pragma unroll
  for (int o = 1; o < kG; o <<= 1) {
    f0 += __shfl_xor_sync(gm, f0, o);
    f1 += __shfl_xor_sync(gm, f1, o);
    f2 += __shfl_xor_sync(gm, f2, o);
  }
  if (q == 0) {
    const double* A = amat + 9 * k;
    const double s0 = svec[3 * k], s1 = svec[3 * k + 1], s2 = svec[3 * k + 2];
    const double vk = vol[k];
    fint[3 * k] = vk * (A[0] * s0 + A[1] * s1 + A[2] * s2 + f0);
    fint[3 * k + 1] = vk * (A[3] * s0 + A[4] * s1 + A[5] * s2 + f1);
    fint[3 * k + 2] = vk * (A[6] * s0 + A[7] * s1 + A[8] * s2 + f2);
  }
}

// ------------------------------------------------------------------ PMB
// Bond-based force density and velocity-Verlet.  The particles are
// renumbered in bin-cell order at set-up, so a tile of R consecutive
// particles has a compact neighbour set; a block per tile stages that set's
// reference positions, displacements and volumes in shared memory and each
// bond then reads only its 2-byte rank in the set (and its broken bit) from
// HBM.  u_in is read, u_out written (double buffered: the kernel reads every
// neighbour's displacement of this step while it advances its own).
struct PmbArgs {
  int32_t n;
  int32_t R;              // particles per tile
  int32_t jmax;           // stride of jset
  const int64_t* rowptr;
  const int32_t* jset;    // per tile: the sorted neighbour set
  const int32_t* jcnt;
  const uint16_t* lidx;   // per bond: rank of its neighbour in the tile's set
  uint32_t* broken;       // bit per bond
  const double* vol;
  const double* X;        // reference positions (double-precision bond geometry)
  const double* u_in;
  double* u_out;
  double* vel;
  double* acl;
  const int8_t* fixed;    // 1: prescribed velocity (kept)
  double c;               // micromodulus
  double s_c;             // critical stretch
  double inv_rho;
  double dt;
  unsigned long long* nbroken;
};

// T = per-bond arithmetic: float (the mixed path: float bond geometry and
// force, the bond vector rounded from the double difference of X and the
// displacements from float offsets to the tile's first particle) or double
// (the oracle's arithmetic, from X and u, for exact parity checks).
//
// FP64 rows are padded to multiples of 4 bonds (pads point at the particle
// itself and start broken), so a lane reads the ranks of 4 consecutive bonds
// as one 8-byte load and their 4 broken bits from one 32-bit word; the float
// path, bound by its shared-memory gathers rather than by these loads, keeps
// unpadded rows and one bond per load.
constexpr int kGP = 8;  // lanes per particle of the bond loop

template <typename T>
__global__ void __launch_bounds__(512) k_pmb_step(PmbArgs a) {
  extern __shared__ double smp[];
  const int64_t t = blockIdx.x;
  const int cnt = a.jcnt[t];
  const int32_t* js = a.jset + t * (int64_t)a.jmax;
  const bool f64 = sizeof(T) == sizeof(double);
  // staged set: FP64 7 arrays of one double per rank (X, u, vol); float: X as
  // 3 doubles (the bond vector is rounded from the exact difference, as the
  // FP64 path forms it: float offsets of X put 1e-6 of the bond length into
  // the stretch and move the break of near-critical bonds), one array per
  // axis so that the eight lanes of a particle, reading neighbours of
  // consecutive rank, read consecutive words (fewer bank conflicts than
  // 24-byte records), and one float4 (u - u_r0, vol)
  double* sd = smp;
  float4* sf = reinterpret_cast<float4*>(smp + ((3 * cnt + 1) & ~1));
  const int64_t r0 = t * a.R;
  const double ur0 = a.u_in[3 * r0], ur1 = a.u_in[3 * r0 + 1], ur2 = a.u_in[3 * r0 + 2];
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
    const int64_t g = js[l];
    const double x0 = a.X[3 * g], x1 = a.X[3 * g + 1], x2 = a.X[3 * g + 2];
    const double u0 = a.u_in[3 * g], u1 = a.u_in[3 * g + 1], u2 = a.u_in[3 * g + 2];
    const double v = a.vol[g];
    if (f64) {  // one array per value: lanes with distinct ranks mod 16 read distinct bank pairs
      sd[l] = x0; sd[cnt + l] = x1; sd[2 * cnt + l] = x2;
      sd[3 * cnt + l] = u0; sd[4 * cnt + l] = u1; sd[5 * cnt + l] = u2; sd[6 * cnt + l] = v;
    } else {
      sd[l] = x0; sd[cnt + l] = x1; sd[2 * cnt + l] = x2;
      sf[l] = make_float4((float)(u0 - ur0), (float)(u1 - ur1), (float)(u2 - ur2), (float)v);
    }
  }
  __syncthreads();
  const int64_t i = t * a.R + threadIdx.x / kGP;
  const int q = threadIdx.x & (kGP - 1);
  const unsigned gm = 0xFFu << (threadIdx.x & 24);
  if (threadIdx.x / kGP >= a.R || i >= a.n) return;
  const double ui0 = a.u_in[3 * i], ui1 = a.u_in[3 * i + 1], ui2 = a.u_in[3 * i + 2];
  const double Xi0 = a.X[3 * i], Xi1 = a.X[3 * i + 1], Xi2 = a.X[3 * i + 2];
  const float fu0 = (float)(ui0 - ur0), fu1 = (float)(ui1 - ur1), fu2 = (float)(ui2 - ur2);
  T f0 = T(0), f1 = T(0), f2 = T(0);
  unsigned nb = 0;
  const T c = (T)a.c, sc = (T)a.s_c;
  constexpr int GB = sizeof(T) == sizeof(double) ? 4 : 1;  // bonds per load group
  constexpr int NQ = GB == 4 ? 2 : 4;                          // groups in flight per lane
  const int64_t p1 = a.rowptr[i + 1];
  for (int64_t pb = a.rowptr[i] + GB * q; pb < p1; pb += GB * kGP * NQ) {
    uint32_t lw[NQ][2];
    uint32_t wd[NQ];
#pragma unroll
    for (int g = 0; g < NQ; ++g) {
      const int64_t p = pb + GB * kGP * g;
      lw[g][0] = lw[g][1] = 0u;
      if (p < p1) {
        if (GB == 4) {
          const uint2 v = *reinterpret_cast<const uint2*>(a.lidx + p);
          lw[g][0] = v.x; lw[g][1] = v.y;
        } else {
          lw[g][0] = a.lidx[p];
        }
        wd[g] = a.broken[p >> 5] >> (p & 31);
      } else {
        wd[g] = 0xFu;  // past the row: skipped
      }
    }
#pragma unroll
    for (int g = 0; g < NQ; ++g)
#pragma unroll
      for (int u = 0; u < GB; ++u) {
        if ((wd[g] >> u) & 1u) continue;  // broken (or a pad)
        const int64_t p = pb + GB * kGP * g + u;
        const int lj = (int)((lw[g][u >> 1] >> (16 * (u & 1))) & 0xFFFFu);
        T s, e0, e1, e2, l, vj;
        if (f64) {
          // the oracle's arithmetic: xi from X, eta = xi + (u_j - u_i), s = (|eta| - |xi|)/|xi|
          const double* d = sd + lj;  // value k of rank lj at d[k cnt]
          const double x0 = d[0] - Xi0, x1 = d[cnt] - Xi1, x2 = d[2 * cnt] - Xi2;
          const double L0d = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
          if (L0d == 0.0) continue;  // the particle itself
          e0 = (T)(x0 + (d[3 * cnt] - ui0));
          e1 = (T)(x1 + (d[4 * cnt] - ui1));
          e2 = (T)(x2 + (d[5 * cnt] - ui2));
          const T L0 = (T)L0d;
          l = (T)sqrt((double)(e0 * e0 + e1 * e1 + e2 * e2));
          s = (l - L0) / L0;
          vj = (T)d[6 * cnt];
        } else {
          const float4 ua = sf[lj];
          const float x0 = (float)(sd[lj] - Xi0), x1 = (float)(sd[cnt + lj] - Xi1), x2 = (float)(sd[2 * cnt + lj] - Xi2);
          const float xx = x0 * x0 + x1 * x1 + x2 * x2;
          if (xx == 0.f) continue;  // the particle itself
          const float d0 = ua.x - fu0, d1 = ua.y - fu1, d2 = ua.z - fu2;
          // stretch without cancellation: (|xi+d|^2 - |xi|^2) / (|xi| (|xi+d| + |xi|)),
          // lengths from the hardware reciprocal square root (about 2 ulp)
          const float f_e0 = x0 + d0, f_e1 = x1 + d1, f_e2 = x2 + d2;
          const float ee = f_e0 * f_e0 + f_e1 * f_e1 + f_e2 * f_e2;
          const float rL0 = rsqrtf(xx), rl = rsqrtf(ee);
          const float fL0 = xx * rL0, fl = ee * rl;
          const float num = 2.f * (x0 * d0 + x1 * d1 + x2 * d2) + (d0 * d0 + d1 * d1 + d2 * d2);
          s = (T)(num * rL0 * __frcp_rn(fl + fL0));
          // eta / |eta| directly, so the force weight needs no division
          e0 = (T)(f_e0 * rl); e1 = (T)(f_e1 * rl); e2 = (T)(f_e2 * rl);
          l = T(1);
          vj = (T)ua.w;
        }
        if (s > sc) {
          atomicOr(&a.broken[p >> 5], 1u << (p & 31));
          ++nb;
          continue;
        }
        const T w = f64 ? c * s * vj / l : c * s * vj;  // the float path's eta is already unit
        f0 += w * e0; f1 += w * e1; f2 += w * e2;
      }
  }
#pragma unroll
  for (int o = 1; o < kGP; o <<= 1) {
    f0 += __shfl_xor_sync(gm, f0, o);
    f1 += __shfl_xor_sync(gm, f1, o);
    f2 += __shfl_xor_sync(gm, f2, o);
    nb += __shfl_xor_sync(gm, nb, o);
  }
  if (q < 3) {
    const int64_t m = 3 * i + q;
    const double f = (double)(q == 0 ? f0 : (q == 1 ? f1 : f2));
    double v = a.vel[m];
    const double aold = a.acl[m];
    double u = a.u_in[m];
    if (a.fixed && a.fixed[i]) {
      u = u + a.dt * v;
    } else {
      const double anew = f * a.inv_rho;
      v = v + 0.5 * a.dt * (aold + anew);            // corrector of this step
      a.acl[m] = anew;
      u = u + a.dt * v + 0.5 * a.dt * a.dt * anew;    // predictor of the next
      a.vel[m] = v;
    }
    a.u_out[m] = u;
  }
  if (q == 0 && nb && a.nbroken) atomicAdd(a.nbroken, (unsigned long long)nb);
}

// ---- renumbering of the particles in bin-cell order
__global__ void k_pmb_iperm(int32_t n, const int32_t* __restrict__ perm, int32_t* __restrict__ iperm) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) iperm[perm[r]] = (int32_t)r;
}
// dst[r w + k] = src[perm[r] w + k] (to = true) or dst[perm[r] w + k] = src[r w + k]
template <typename V>
__global__ void k_pmb_perm(int32_t n, int w, const int32_t* __restrict__ perm, const V* __restrict__ src,
                           V* __restrict__ dst, bool to) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * w) return;
  const int64_t r = e / w, k = e - r * w;
  if (to) dst[e] = src[(int64_t)perm[r] * w + k];
  else dst[(int64_t)perm[r] * w + k] = src[e];
}
// row lengths in the new order, rounded up to whole groups of pad bonds
__global__ void k_pmb_rowlen(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ rowptr0,
                             int32_t pad, int32_t* __restrict__ len) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) len[r] = ((int32_t)(rowptr0[perm[r] + 1] - rowptr0[perm[r]]) + pad - 1) / pad * pad;
}
// warp per new row: the old row's entries in their order, columns renumbered
__global__ void k_pmb_rows(int32_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                           const int64_t* __restrict__ rowptr0, const int32_t* __restrict__ col0,
                           const int64_t* __restrict__ rowptr1, int32_t* __restrict__ col1) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t a0 = rowptr0[perm[r]], len = rowptr0[perm[r] + 1] - a0, b0 = rowptr1[r];
  const int64_t lp = rowptr1[r + 1] - b0;
  for (int64_t k = lane; k < lp; k += 32) col1[b0 + k] = k < len ? iperm[col0[a0 + k]] : (int32_t)r;  // pads: self
}
// the pads of each padded row start broken
__global__ void k_pmb_padbits(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ rowptr0,
                              const int64_t* __restrict__ rowptr1, uint32_t* __restrict__ bits) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t len = rowptr0[perm[r] + 1] - rowptr0[perm[r]];
  for (int64_t p = rowptr1[r] + len; p < rowptr1[r + 1]; ++p) atomicOr(&bits[p >> 5], 1u << (p & 31));
}
// per-bond flags between the two orders: new entry rowptr1[r] + k is old
// entry rowptr0[perm[r]] + k.  to_new: old bytes -> new bits (OR); else new
// bits -> old bytes.
__global__ void k_pmb_flags(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ rowptr0,
                            const int64_t* __restrict__ rowptr1, uint32_t* __restrict__ bits,
                            uint8_t* __restrict__ bytes, bool to_new) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t a0 = rowptr0[perm[r]], len = rowptr0[perm[r] + 1] - a0, b0 = rowptr1[r];
  for (int64_t k = lane; k < len; k += 32) {
    const int64_t p = b0 + k;
    if (to_new) {
      if (bytes[a0 + k]) atomicOr(&bits[p >> 5], 1u << (p & 31));
    } else {
      bytes[a0 + k] = (uint8_t)((bits[p >> 5] >> (p & 31)) & 1u);
    }
  }
}

// Local damage of each particle (Silling & Askari 2005): the fraction of its
// bonds that are broken (the self entry excluded), written in the caller's
// particle order.
__global__ void k_pmb_damage(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ rowptr0,
                             const int64_t* __restrict__ rowptr1, const uint32_t* __restrict__ bits,
                             double* __restrict__ out) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t len = rowptr0[perm[r] + 1] - rowptr0[perm[r]], b0 = rowptr1[r];
  int nb = 0;
  for (int64_t k = lane; k < len; k += 32) {
    const int64_t p = b0 + k;
    nb += (bits[p >> 5] >> (p & 31)) & 1u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nb += __shfl_xor_sync(0xffffffffu, nb, o);
  if (lane == 0) out[perm[r]] = len > 1 ? (double)nb / (double)(len - 1) : 0.0;
}

// Pre-crack: break every bond whose reference segment X_i -> X_j crosses the
// rectangle {p0 + s a + t b : 0 <= s, t <= 1} (strictly between its ends).
__global__ void k_pmb_cut(int32_t n, const double* __restrict__ X, const int64_t* __restrict__ rowptr,
                          const int32_t* __restrict__ col, double3 p0, double3 ea, double3 eb,
                          uint32_t* __restrict__ broken, unsigned long long* __restrict__ ncut) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kG;
  const int q = threadIdx.x & (kG - 1);
  if (i >= n) return;
  const double nx = ea.y * eb.z - ea.z * eb.y, ny = ea.z * eb.x - ea.x * eb.z, nz = ea.x * eb.y - ea.y * eb.x;
  const double aa = ea.x * ea.x + ea.y * ea.y + ea.z * ea.z, bb = eb.x * eb.x + eb.y * eb.y + eb.z * eb.z;
  const double xi0 = X[3 * i], xi1 = X[3 * i + 1], xi2 = X[3 * i + 2];
  const double si = (xi0 - p0.x) * nx + (xi1 - p0.y) * ny + (xi2 - p0.z) * nz;
  unsigned long long cnt = 0;
  for (int64_t p = rowptr[i] + q; p < rowptr[i + 1]; p += kG) {
    const int64_t j = col[p];
    const double d0 = X[3 * j] - xi0, d1 = X[3 * j + 1] - xi1, d2 = X[3 * j + 2] - xi2;
    const double sj = si + d0 * nx + d1 * ny + d2 * nz;
    if (!((si < 0.0 && sj > 0.0) || (si > 0.0 && sj < 0.0))) continue;
    const double t = si / (si - sj);
    const double c0 = xi0 + t * d0 - p0.x, c1 = xi1 + t * d1 - p0.y, c2 = xi2 + t * d2 - p0.z;
    const double s = (c0 * ea.x + c1 * ea.y + c2 * ea.z) / aa, r = (c0 * eb.x + c1 * eb.y + c2 * eb.z) / bb;
    if (s >= 0.0 && s <= 1.0 && r >= 0.0 && r <= 1.0) {
      const uint32_t bit = 1u << (p & 31);
      if (!(atomicOr(&broken[p >> 5], bit) & bit)) ++cnt;
    }
  }
  if (cnt) atomicAdd(ncut, cnt);
}

// predictor of the first step: u1 = u0 + dt v0 + dt^2/2 a0
__global__ void k_pmb_first(int64_t n3, double* __restrict__ u, const double* __restrict__ vel,
                            const double* __restrict__ acl, double dt) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m < n3) u[m] = u[m] + dt * vel[m] + 0.5 * dt * dt * acl[m];
}

inline unsigned gridg(int64_t n) { return (unsigned)((n * kG + 255) / 256); }

}  // namespace

// launchers used by the C ABI (context.cu / pmb ABI below)
int pd_shape(cudaStream_t s, int32_t n, const double* X, const double* win, const double* vol, const DevCSR& csr,
             double* shp, double* ginvk, double* svec, unsigned* status) {
  k_pd_shape<<<gridg(n), 256, 0, s>>>(n, X, win, vol, csr.rowptr, csr.col, shp, ginvk, svec, status);
  MEGA_CHECK_LAUNCH();
  return 0;
}
int pd_svec(cudaStream_t s, int32_t n, const double* X, const double* vol, const DevCSR& csr, const double* shp,
            double* svec) {
  k_pd_svec<<<(n + 127) / 128, 128, 0, s>>>(n, X, vol, csr.rowptr, csr.col, shp, svec);
  MEGA_CHECK_LAUNCH();
  return 0;
}
int pd_step(cudaStream_t s, int32_t n, const double* X, const double* xc, const double* du, const double* vol,
            const DevCSR& csr, const double* shp, const double* ginvk, const double* svec, const uint16_t* matidx,
            const MatEntry* mats, double* stress, double* strain, double* eps, double* aux, double* wvel, double* fg,
            double* amat, double* fint, int linit, const mega_params& p, double dt, unsigned* status) {
  k_pd_defgrad<<<gridg(n), 256, 0, s>>>(n, X, xc, du, vol, csr.rowptr, csr.col, shp, fg);
  MEGA_CHECK_LAUNCH();
  PdStressArgs a{};
  a.n = n; a.fg = fg; a.ginvk = ginvk; a.matidx = matidx; a.mats = mats; a.stress = stress; a.strain = strain;
  a.eps = eps; a.aux = aux; a.wvel = wvel; a.amat = amat; a.linit = linit; a.inv3_exact = p.inv3_exact;
  a.maxit = p.newton_max_iter; a.rate_solver = p.rate_solver; a.rtol = p.newton_rtol; a.dt = dt; a.status = status;
  k_pd_stress<<<(n + 127) / 128, 128, 0, s>>>(a);
  MEGA_CHECK_LAUNCH();
  k_pd_force<<<gridg(n), 256, 0, s>>>(n, X, vol, csr.colptr, csr.trow, csr.tpos, shp, amat, svec, fint);
  MEGA_CHECK_LAUNCH();
  return 0;
}

// ------------------------------------------------- resident PMB context
struct PmbCtx {
  int32_t n = 0;
  cudaStream_t s = nullptr;
  DevPool pool;
  DevCSR csr;          // in the bin-cell numbering (FP64: rows padded to groups of 4 bonds)
  int64_t nreal = 0;   // bonds without the pads
  int32_t* perm = nullptr;      // new particle r = caller's particle perm[r]
  int64_t* rowptr0 = nullptr;   // the caller's row offsets (bond flags map through them)
  TileSet tiles;
  double *X = nullptr, *vol = nullptr, *u[2] = {nullptr, nullptr}, *vel = nullptr, *acl = nullptr;
  uint32_t* broken = nullptr;
  int8_t* fixed = nullptr;
  unsigned long long* nbroken = nullptr;
  unsigned* status = nullptr;
  double c = 0, s_c = 0, rho = 1;
  int f64 = 0;
  int cur = 0;
  int64_t steps = 0;
  cudaGraphExec_t g = nullptr;
  double g_dt = 0;
  ~PmbCtx() {
    if (g) cudaGraphExecDestroy(g);
    pool.free_all();  // stream-ordered frees before the stream goes
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

static PmbArgs pmb_args(PmbCtx* c, double dt) {
  PmbArgs a{};
  a.n = c->n; a.R = c->tiles.R; a.jmax = c->tiles.jmax; a.rowptr = c->csr.rowptr; a.jset = c->tiles.jset;
  a.jcnt = c->tiles.jcnt; a.lidx = c->tiles.lidx; a.broken = c->broken;
  a.vol = c->vol; a.X = c->X; a.u_in = c->u[c->cur]; a.u_out = c->u[1 - c->cur]; a.vel = c->vel; a.acl = c->acl;
  a.fixed = c->fixed; a.c = c->c; a.s_c = c->s_c; a.inv_rho = 1.0 / c->rho; a.dt = dt; a.nbroken = c->nbroken;
  return a;
}

static void launch_pmb(PmbCtx* c, const PmbArgs& a) {
  const unsigned grid = (unsigned)c->tiles.ntiles;
  const int block = c->tiles.R * kGP;
  const size_t smem = (c->f64 ? 64 : 40) * (size_t)c->tiles.maxcnt + 16;
  if (c->f64) k_pmb_step<double><<<grid, block, smem, c->s>>>(a);
  else k_pmb_step<float><<<grid, block, smem, c->s>>>(a);
}

}  // namespace mega

using namespace mega;

extern "C" {

int mega_construct_fint_pd(const mega_params* p, int32_t n, const double* gcoo, const double* gcoo_current,
                           const double* gwin, const double* gvol, const double* gprop, const int32_t* gmat_type,
                           double* gstate, double* gstress, double* gstrain, const double* gdinc, const int32_t* gn,
                           const int32_t* gstart, const int32_t* gstack, int64_t nnz, double* gstack_shp,
                           double* ginvk, int32_t linit, double dlt, double* fint, double* gmax_wvel,
                           double* gint_work) {
  (void)gint_work;
  if (!p || n <= 0 || !gcoo || !gcoo_current || !gwin || !gvol || !gprop || !gmat_type || !gstate || !gstress ||
      !gstrain || !gdinc || !gn || !gstart || !gstack || !gstack_shp || !ginvk || !fint || !gmax_wvel)
    return MEGA_ERR_ARG;
  cudaStream_t s;
  MEGA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{s};
  DevPool pool;
  // CSR in the caller's row order (1-based GSTART/GSTACK)
  std::vector<int64_t> rp(n + 1, 0), hpos;
  for (int32_t i = 0; i < n; ++i) rp[i + 1] = rp[i] + gn[i];
  const int64_t m = rp[n];
  std::vector<int32_t> colh(m);
  hpos.resize(m);
  for (int32_t i = 0; i < n; ++i)
    for (int32_t k = 0; k < gn[i]; ++k) {
      const int64_t q = (int64_t)gstart[i] - 1 + k;
      if (q < 0 || q >= nnz || gstack[q] < 1 || gstack[q] > n) return MEGA_ERR_ARG;
      colh[rp[i] + k] = gstack[q] - 1;
      hpos[rp[i] + k] = q;
    }
  DevCSR csr;
  csr.n = n; csr.nnz = m;
  MEGA_ALLOC(pool, csr.rowptr, n + 1);
  MEGA_ALLOC(pool, csr.col, m);
  MEGA_TRY(cudaMemcpyAsync(csr.rowptr, rp.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(csr.col, colh.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s));
  int r = build_transpose(s, csr, pool);
  if (r) return r;
  const int64_t n3 = 3 * (int64_t)n;
  double *X, *xc, *w, *v, *du, *shp, *ik, *sv, *sig, *eps6, *ep, *wv, *fg, *am, *fi;
  uint16_t* midx;
  MatEntry* dm;
  unsigned* st;
  MEGA_ALLOC(pool, X, n3); MEGA_ALLOC(pool, xc, n3); MEGA_ALLOC(pool, w, n3); MEGA_ALLOC(pool, v, n);
  MEGA_ALLOC(pool, du, n3); MEGA_ALLOC(pool, shp, m); MEGA_ALLOC(pool, ik, 9 * (int64_t)n);
  MEGA_ALLOC(pool, sv, n3); MEGA_ALLOC(pool, sig, 6 * (int64_t)n); MEGA_ALLOC(pool, eps6, 6 * (int64_t)n);
  MEGA_ALLOC(pool, ep, n); MEGA_ALLOC(pool, wv, n); MEGA_ALLOC(pool, fg, 18 * (int64_t)n);
  MEGA_ALLOC(pool, am, 9 * (int64_t)n); MEGA_ALLOC(pool, fi, n3); MEGA_ALLOC(pool, midx, n); MEGA_ALLOC(pool, st, 1);
  // material table
  std::vector<MatEntry> ents;
  std::vector<const double*> rows;  // the PROPS row each entry was made from
  std::vector<uint16_t> idx(n);
  bool damaged = false;
  for (int32_t i = 0; i < n; ++i) {
    const double* pr = gprop + 30 * (size_t)i;
    int found = -1;
    for (size_t e = 0; e < ents.size() && found < 0; ++e)
      if (ents[e].type == gmat_type[i] && std::memcmp(rows[e], pr, 30 * sizeof(double)) == 0) found = (int)e;
    if (found < 0) {
      if (ents.size() >= 1024) return MEGA_ERR_UNSUPPORTED;
      found = (int)ents.size();
      ents.push_back(mat_entry(gmat_type[i], pr));
      rows.push_back(pr);
      damaged = damaged || damaged_type(gmat_type[i]);
    }
    idx[i] = (uint16_t)found;
  }
  MEGA_ALLOC(pool, dm, ents.size());
  std::vector<double> hep(n), hax;
  for (int32_t i = 0; i < n; ++i) hep[i] = gstate[20 * (size_t)i + 2];
  double* aux = nullptr;  // GSTATE(1, 2, 4, 5) when a damaged model is present
  if (damaged) {
    MEGA_ALLOC(pool, aux, 4 * (int64_t)n);
    hax.resize(4 * (size_t)n);
    for (int32_t i = 0; i < n; ++i) {
      const double* g = gstate + 20 * (size_t)i;
      hax[4 * (size_t)i] = g[0]; hax[4 * (size_t)i + 1] = g[1]; hax[4 * (size_t)i + 2] = g[3];
      hax[4 * (size_t)i + 3] = g[4];
    }
    MEGA_TRY(cudaMemcpyAsync(aux, hax.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
  }
  MEGA_TRY(cudaMemcpyAsync(X, gcoo, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(xc, gcoo_current, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(w, gwin, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(v, gvol, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(du, gdinc, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(sig, gstress, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(eps6, gstrain, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(ep, hep.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(midx, idx.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(dm, ents.data(), sizeof(MatEntry) * ents.size(), cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  if (linit) {
    r = pd_shape(s, n, X, w, v, csr, shp, ik, sv, st);
    if (r) return r;
  } else {
    std::vector<double> hs(m);
    for (int64_t k = 0; k < m; ++k) hs[k] = gstack_shp[hpos[k]];
    MEGA_TRY(cudaMemcpyAsync(shp, hs.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
    MEGA_TRY(cudaMemcpyAsync(ik, ginvk, sizeof(double) * 9 * n, cudaMemcpyHostToDevice, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    r = pd_svec(s, n, X, v, csr, shp, sv);
    if (r) return r;
  }
  r = pd_step(s, n, X, xc, du, v, csr, shp, ik, sv, midx, dm, sig, eps6, ep, aux, wv, fg, am, fi, linit, *p, dlt,
              st);
  if (r) return r;
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(fint, fi, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(gstress, sig, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(gstrain, eps6, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(hep.data(), ep, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if (damaged) MEGA_TRY(cudaMemcpyAsync(hax.data(), aux, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(gmax_wvel, wv, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  std::vector<double> hs(m);
  if (linit) {
    MEGA_TRY(cudaMemcpyAsync(hs.data(), shp, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaMemcpyAsync(ginvk, ik, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, s));
  }
  MEGA_TRY(cudaStreamSynchronize(s));
  if (linit)
    for (int64_t k = 0; k < m; ++k) gstack_shp[hpos[k]] = hs[k];
  for (int32_t i = 0; i < n; ++i) gstate[20 * (size_t)i + 2] = hep[i];
  if (damaged)
    for (int32_t i = 0; i < n; ++i) {
      double* g = gstate + 20 * (size_t)i;
      g[0] = hax[4 * (size_t)i]; g[1] = hax[4 * (size_t)i + 1]; g[3] = hax[4 * (size_t)i + 2];
      g[4] = hax[4 * (size_t)i + 3];
    }
  return (int)hst;
}

int construct_fint_pd_gpu(const double* gwin, const double* gvol, const int32_t* gnump, const double* gcoo,
                          const double* gcoo_cuurent, const double* gsm_len, const double* gsm_area,
                          const double* gsm_vol, const double* gnsni_fac, const int32_t* gghost, const double* gprop,
                          double* gstate, double* gstress, double* gstrain, double* g_h_stress, double* g_s_stress,
                          const double* gdinc, const double* gdinc_tot, const int32_t* gmat_type,
                          const int32_t* gebc_nodes, const int32_t* gn, const int32_t* gstart,
                          const int32_t* dim_nn_list, const int32_t* gstack, double* gstack_shp,
                          double* gstack_dshp, double* gstack_ddshp, const int32_t* gmaxn, double* ginvk,
                          const int32_t* linit, double* fint, double* dlt_fint, double* gchar_dist,
                          double* gmax_wvel, double* local_dx_stress, double* local_dy_stress,
                          double* local_dz_stress, const double* g_x_mom, const double* g_y_mom,
                          const double* g_z_mom, const double* model_bodyforce, double* gint_work,
                          const double* dlt) {
  (void)gsm_len; (void)gsm_area; (void)gsm_vol; (void)gnsni_fac; (void)gghost; (void)g_h_stress; (void)g_s_stress;
  (void)gdinc_tot; (void)gebc_nodes; (void)gstack_dshp; (void)gstack_ddshp; (void)gmaxn; (void)local_dx_stress;
  (void)local_dy_stress; (void)local_dz_stress; (void)g_x_mom; (void)g_y_mom; (void)g_z_mom; (void)model_bodyforce;
  mega_params p;
  if (int r = fint_control_get(&p)) return r;
  if (!gnump || !dim_nn_list || !linit || !dlt || *gnump <= 0 || !gcoo_cuurent) return MEGA_ERR_ARG;
  const int32_t n = *gnump;
  const int st = mega_construct_fint_pd(&p, n, gcoo, gcoo_cuurent, gwin, gvol, gprop, gmat_type, gstate, gstress,
                                        gstrain, gdinc, gn, gstart, gstack, *dim_nn_list, gstack_shp, ginvk, *linit,
                                        *dlt, fint, gmax_wvel, gint_work);
  if (st < 0 || !p.auto_ts) return st;
  // AUTO_TS (FINT_PD.F90:690-754): each node's nearest neighbour in the
  // current configuration over its wave speed, the smallest, times DLT_FAC
  if (!gchar_dist || !dlt_fint) return MEGA_ERR_ARG;
  double dmin = 0.0;
  for (int32_t i = 0; i < n; ++i) {
    const double xi = gcoo_cuurent[3 * (size_t)i], yi = gcoo_cuurent[3 * (size_t)i + 1],
                 zi = gcoo_cuurent[3 * (size_t)i + 2];
    bool first = true;
    for (int32_t k = 0; k < gn[i]; ++k) {
      const int32_t jj = gstack[gstart[i] - 1 + k] - 1;
      if (jj == i) continue;
      const double dx = gcoo_cuurent[3 * (size_t)jj] - xi, dy = gcoo_cuurent[3 * (size_t)jj + 1] - yi,
                   dz = gcoo_cuurent[3 * (size_t)jj + 2] - zi;
      const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
      gchar_dist[i] = first ? d : std::min(gchar_dist[i], d);
      first = false;
    }
    const double t = gchar_dist[i] / gmax_wvel[i];
    dmin = (i == 0) ? t : std::min(t, dmin);
  }
  *dlt_fint = dmin * p.dlt_fac;
  return st;
}

static std::mutex g_pmb_mu;
static std::set<PmbCtx*> g_pmbs;
static PmbCtx* get_pmb(int64_t h) {
  std::lock_guard<std::mutex> lk(g_pmb_mu);
  PmbCtx* c = reinterpret_cast<PmbCtx*>(h);
  return g_pmbs.count(c) ? c : nullptr;
}

int mega_pmb_init(int32_t n, const double* coo, const double* vol, const double* vinit, const int32_t* fixed,
                  double horizon, double micromodulus, double s_c, double rho, const uint8_t* broken0,
                  int32_t mode, int64_t* handle, int64_t* nbonds) {
  if (n <= 0 || !coo || !vol || !vinit || !handle || !(horizon > 0) || !(rho > 0)) return MEGA_ERR_ARG;
  PmbCtx* c = new PmbCtx();
  DevPool tmp;  // set-up temporaries, freed (in stream order) before the stream goes
  auto fail = [&](int code) {
    tmp.free_all();
    delete c;
    return code;
  };
  c->n = n; c->c = micromodulus; c->s_c = s_c; c->rho = rho;
  c->f64 = ((mode & 0xff) == MEGA_MODE_FP64);
  if (cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess) return fail(MEGA_ERR_CUDA);
  c->pool.bind(c->s);
  tmp.bind(c->s);
  const int64_t n3 = 3 * (int64_t)n;
#define PA(ptr, cnt) do { if (c->pool.alloc(&(ptr), (size_t)(cnt))) return fail(MEGA_ERR_NOMEM); } while (0)
  double *win = nullptr, *sml = nullptr;
  PA(c->X, n3); PA(c->vol, n); PA(c->u[0], n3); PA(c->u[1], n3); PA(c->vel, n3); PA(c->acl, n3);
  PA(c->fixed, n); PA(c->nbroken, 1); PA(c->status, 1);
  if (tmp.alloc(&win, n3) || tmp.alloc(&sml, 6 * (int64_t)n)) return fail(MEGA_ERR_NOMEM);
  std::vector<double> hw(n3, horizon);
  std::vector<int8_t> hf(n, 0);
  if (fixed)
    for (int32_t i = 0; i < n; ++i) hf[i] = (int8_t)(fixed[i] != 0);
  cudaMemcpyAsync(c->X, coo, sizeof(double) * n3, cudaMemcpyHostToDevice, c->s);
  cudaMemcpyAsync(c->vol, vol, sizeof(double) * n, cudaMemcpyHostToDevice, c->s);
  cudaMemcpyAsync(c->vel, vinit, sizeof(double) * n3, cudaMemcpyHostToDevice, c->s);
  cudaMemcpyAsync(c->fixed, hf.data(), n, cudaMemcpyHostToDevice, c->s);
  cudaMemcpyAsync(win, hw.data(), sizeof(double) * n3, cudaMemcpyHostToDevice, c->s);
  cudaMemsetAsync(sml, 0, sizeof(double) * 6 * n, c->s);
  cudaMemsetAsync(c->u[0], 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->u[1], 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->acl, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->nbroken, 0, sizeof(unsigned long long), c->s);
  cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->s);
  const double dmax[3] = {0.0, 0.0, 0.0};
  // spherical horizon: the ellipsoidal support test of SOFT_SEARCH (SHSUP),
  // in the caller's numbering, with the bin-cell order of the particles
  DevCSR csr0;
  PA(c->perm, n);
  int r = bin_search(c->s, n, c->X, win, sml, dmax, 0, 1, c->status, csr0, nullptr, tmp, nullptr, c->perm);
  if (r) return fail(r);
  const int64_t m = csr0.nnz;
  // renumber the particles in that order: rows keep their entries' order
  int32_t *iperm = nullptr, *len = nullptr;
  double* buf = nullptr;
  int8_t* bf8 = nullptr;
  if (tmp.alloc(&iperm, n) || tmp.alloc(&len, n) || tmp.alloc(&buf, n3) || tmp.alloc(&bf8, n))
    return fail(MEGA_ERR_NOMEM);
  const unsigned gn = (unsigned)((n + 255) / 256), g3 = (unsigned)((n3 + 255) / 256);
  k_pmb_iperm<<<gn, 256, 0, c->s>>>(n, c->perm, iperm);
  cudaMemcpyAsync(buf, c->X, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->s);
  k_pmb_perm<double><<<g3, 256, 0, c->s>>>(n, 3, c->perm, buf, c->X, true);
  cudaMemcpyAsync(buf, c->vel, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->s);
  k_pmb_perm<double><<<g3, 256, 0, c->s>>>(n, 3, c->perm, buf, c->vel, true);
  cudaMemcpyAsync(buf, c->vol, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->s);
  k_pmb_perm<double><<<gn, 256, 0, c->s>>>(n, 1, c->perm, buf, c->vol, true);
  cudaMemcpyAsync(bf8, c->fixed, n, cudaMemcpyDeviceToDevice, c->s);
  k_pmb_perm<int8_t><<<gn, 256, 0, c->s>>>(n, 1, c->perm, bf8, c->fixed, true);
  c->csr.n = n;
  const int32_t pad = c->f64 ? 4 : 1;  // FP64 rows in groups of 4 bonds
  c->csr.gmaxn = (csr0.gmaxn + pad - 1) / pad * pad;
  c->nreal = m;
  PA(c->rowptr0, (int64_t)n + 1);
  cudaMemcpyAsync(c->rowptr0, csr0.rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice, c->s);
  PA(c->csr.rowptr, (int64_t)n + 1);
  k_pmb_rowlen<<<gn, 256, 0, c->s>>>(n, c->perm, csr0.rowptr, pad, len);
  if ((r = scan_counts(c->s, len, c->csr.rowptr, n, tmp))) return fail(r);
  int64_t mp = 0;  // entries with the rows padded
  if (cudaMemcpyAsync(&mp, c->csr.rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->s) != cudaSuccess ||
      cudaStreamSynchronize(c->s) != cudaSuccess)
    return fail(MEGA_ERR_CUDA);
  c->csr.nnz = mp;
  PA(c->csr.col, mp);
  const unsigned gw = (unsigned)(((int64_t)n * 32 + 255) / 256);
  k_pmb_rows<<<gw, 256, 0, c->s>>>(n, c->perm, iperm, csr0.rowptr, csr0.col, c->csr.rowptr, c->csr.col);
  if (cudaGetLastError() != cudaSuccess) return fail(MEGA_ERR_CUDA);
  // tiles of consecutive particles with their neighbour sets
  if ((r = build_tiles(c->s, n, c->csr.rowptr, c->csr.col, mp, c->csr.gmaxn, c->tiles, c->pool, nullptr)))
    return fail(r);
  {
    static bool smem_set = false;  // FP64 stages 64 bytes per particle, float 40: up to 64 KB
    if (!smem_set) {
      if (cudaFuncSetAttribute(k_pmb_step<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024 + 16) !=
              cudaSuccess ||
          cudaFuncSetAttribute(k_pmb_step<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 40 * 1024 + 16) !=
              cudaSuccess)
        return fail(MEGA_ERR_CUDA);
      smem_set = true;
    }
  }
  PA(c->broken, (mp + 31) / 32);
#undef PA
  cudaMemsetAsync(c->broken, 0, sizeof(uint32_t) * ((mp + 31) / 32), c->s);
  k_pmb_padbits<<<gn, 256, 0, c->s>>>(n, c->perm, c->rowptr0, c->csr.rowptr, c->broken);
  if (broken0) {  // the caller's order -> bits in the renumbered order
    uint8_t* b0 = nullptr;
    if (tmp.alloc(&b0, m)) return fail(MEGA_ERR_NOMEM);
    cudaMemcpyAsync(b0, broken0, (size_t)m, cudaMemcpyHostToDevice, c->s);
    k_pmb_flags<<<gw, 256, 0, c->s>>>(n, c->perm, c->rowptr0, c->csr.rowptr, c->broken, b0, true);
  }
  if (cudaStreamSynchronize(c->s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return fail(MEGA_ERR_CUDA);
  if (nbonds) *nbonds = m;
  {
    std::lock_guard<std::mutex> lk(g_pmb_mu);
    g_pmbs.insert(c);
  }
  *handle = reinterpret_cast<int64_t>(c);
  return 0;
}

// nsteps of velocity-Verlet: the first step starts from a = 0 like the
// reference's STATE_INIT (the predictor of step 1 is u = dt v).
int mega_pmb_step(int64_t h, int32_t nsteps, double dt, float* ms) {
  PmbCtx* c = get_pmb(h);
  if (!c) return MEGA_ERR_HANDLE;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    MEGA_TRY(cudaEventCreate(&e0));
    MEGA_TRY(cudaEventCreate(&e1));
    MEGA_TRY(cudaEventRecord(e0, c->s));
  }
  if (c->steps == 0) {
    const int64_t n3 = 3 * (int64_t)c->n;
    k_pmb_first<<<(unsigned)((n3 + 255) / 256), 256, 0, c->s>>>(n3, c->u[c->cur], c->vel, c->acl, dt);
    MEGA_CHECK_LAUNCH();
  }
  int done = 0;
  // graph of two steps (the ping-pong buffers return to where they started)
  if (nsteps >= 2 && (c->g == nullptr || c->g_dt != dt)) {
    if (c->g) { cudaGraphExecDestroy(c->g); c->g = nullptr; }
    cudaGraph_t gr;
    MEGA_TRY(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < 2; ++k) {
      PmbArgs a = pmb_args(c, dt);
      launch_pmb(c, a);
      c->cur = 1 - c->cur;
    }
    cudaError_t e = cudaStreamEndCapture(c->s, &gr);
    if (e != cudaSuccess) { record_cuda_error(e, "capture", __FILE__, __LINE__); return MEGA_ERR_CUDA; }
    e = cudaGraphInstantiate(&c->g, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) { record_cuda_error(e, "instantiate", __FILE__, __LINE__); return MEGA_ERR_CUDA; }
    c->g_dt = dt;
  }
  while (nsteps - done >= 2) {
    MEGA_TRY(cudaGraphLaunch(c->g, c->s));
    done += 2;
  }
  for (; done < nsteps; ++done) {
    PmbArgs a = pmb_args(c, dt);
    launch_pmb(c, a);
    MEGA_CHECK_LAUNCH();
    c->cur = 1 - c->cur;
  }
  c->steps += nsteps;
  if (ms) {
    MEGA_TRY(cudaEventRecord(e1, c->s));
    MEGA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

// what = 0: displacement u (3n), 1: velocity (3n), 2: acceleration (3n),
// 3: broken-bond flags (nnz, as double 0/1).  *nbroken = bonds broken so far.
int mega_pmb_download(int64_t h, int32_t what, double* dst, int64_t* nbroken) {
  PmbCtx* c = get_pmb(h);
  if (!c) return MEGA_ERR_HANDLE;
  const int64_t n3 = 3 * (int64_t)c->n;
  if (nbroken) {
    unsigned long long v = 0;
    MEGA_TRY(cudaMemcpyAsync(&v, c->nbroken, sizeof(v), cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    *nbroken = (int64_t)v;
  }
  if (!dst) return 0;
  // after a step, u[cur] already holds the next step's predictor; the
  // displacement of the last completed step is the one it started from
  const double* ucur = c->steps > 0 ? c->u[1 - c->cur] : c->u[c->cur];
  DevPool tp(c->s);
  if (what >= 0 && what <= 2) {  // back to the caller's particle order
    const double* src = what == 0 ? ucur : (what == 1 ? c->vel : c->acl);
    double* d = nullptr;
    MEGA_ALLOC(tp, d, n3);
    k_pmb_perm<double><<<(unsigned)((n3 + 255) / 256), 256, 0, c->s>>>(c->n, 3, c->perm, src, d, false);
    MEGA_CHECK_LAUNCH();
    MEGA_TRY(cudaMemcpyAsync(dst, d, sizeof(double) * n3, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
  } else if (what == 3) {  // the caller's list order
    const int64_t m = c->nreal;
    uint8_t* d = nullptr;
    MEGA_ALLOC(tp, d, m);
    k_pmb_flags<<<(unsigned)(((int64_t)c->n * 32 + 255) / 256), 256, 0, c->s>>>(c->n, c->perm, c->rowptr0,
                                                                              c->csr.rowptr, c->broken, d, false);
    MEGA_CHECK_LAUNCH();
    std::vector<uint8_t> hb(m);
    MEGA_TRY(cudaMemcpyAsync(hb.data(), d, (size_t)m, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    for (int64_t p = 0; p < m; ++p) dst[p] = hb[p];
  } else if (what == 4) {  // local damage per particle
    double* d = nullptr;
    MEGA_ALLOC(tp, d, c->n);
    k_pmb_damage<<<(unsigned)(((int64_t)c->n * 32 + 255) / 256), 256, 0, c->s>>>(c->n, c->perm, c->rowptr0,
                                                                               c->csr.rowptr, c->broken, d);
    MEGA_CHECK_LAUNCH();
    MEGA_TRY(cudaMemcpyAsync(dst, d, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
  } else return MEGA_ERR_ARG;
  return 0;
}

int mega_pmb_cut(int64_t h, const double* corner, const double* edge_a, const double* edge_b, int64_t* ncut) {
  PmbCtx* c = get_pmb(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!corner || !edge_a || !edge_b) return MEGA_ERR_ARG;
  DevPool tmp(c->s);
  unsigned long long* d = nullptr;
  MEGA_ALLOC(tmp, d, 1);
  MEGA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->s));
  k_pmb_cut<<<gridg(c->n), 256, 0, c->s>>>(c->n, c->X, c->csr.rowptr, c->csr.col,
                                           make_double3(corner[0], corner[1], corner[2]),
                                           make_double3(edge_a[0], edge_a[1], edge_a[2]),
                                           make_double3(edge_b[0], edge_b[1], edge_b[2]), c->broken, d);
  MEGA_CHECK_LAUNCH();
  unsigned long long v = 0;
  MEGA_TRY(cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  if (ncut) *ncut = (int64_t)v;
  return 0;
}

int mega_pmb_finalize(int64_t h) {
  PmbCtx* c = get_pmb(h);
  if (!c) return MEGA_ERR_HANDLE;
  {
    std::lock_guard<std::mutex> lk(g_pmb_mu);
    g_pmbs.erase(c);
  }
  delete c;
  return 0;
}

}  // extern "C"
