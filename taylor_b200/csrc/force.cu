// force.cu -- the per-step internal force of CONSTRUCT_FINT (FINT.F90:
// 259-1247) and the central-difference update of MAIN.F90:348-488.
//
// One explicit step is three kernels:
//   k_defgrad  (row gather, 4 lanes per node): F = I + sum_J u_J (x) grad0 phi_iJ
//              and G0 = sum_J du_J (x) grad0 phi_iJ (FINT.F90:363-376, 673-679)
//              written as sum_J (u_J - u_i)(x)g + u_i (x) sum_J g so the
//              rigid part does not cancel in float;
//   k_stress   (thread per node): |det F|, INV3, L = G0 INV3(F) (the push-
//              forward of FINT.F90:380-391 applied once to the 3x3 instead
//              of per neighbour), Hughes-Winget, rotation of sigma and eps,
//              elastic predictor, return mapping, state write-back, wave
//              speed and internal work (FINT.F90:758-870); it emits
//              T_i = V_i J_i sigma_i INV3(F_i)^T so that the scattered force
//              f_J += B(grad phi_iJ)^T sigma_i V_i J_i (FINT.F90:999-1116)
//              becomes T_i grad0 phi_iJ;
//   k_force    (column gather over the transposed list, 4 lanes per node):
//              f_J = sum_{i: J in N(i)} T_i grad0 phi_iJ -- no atomics, a
//              fixed summation order, no FINT_TEMP(NCORES,3,N) buffers --
//              fused with the fixity / acceleration / corrector of MAIN.F90:
//              432-488, the energy sums of MAIN.F90:524-555 and the next
//              step's predictor (MAIN.F90:353-355).
// FP64 (drop-in) and mixed (float gradients / stress / force arithmetic,
// double moment inverse, positions, integration and return-mapping
// residual) instantiate the same templates.
#include "mega_internal.cuh"
#include "mlp_tc.cuh"

namespace mega {
namespace {

constexpr int kGroup = 4;  // lanes per node in the gathers

__device__ __forceinline__ NodeMat to_nodemat(const MatEntry& e) {
  NodeMat m;
  m.type = e.type; m.nu = e.nu; m.E = e.E; m.rho = e.rho; m.sig0 = e.sig0; m.B = e.B; m.C = e.C;
  m.lam = e.lam; m.mu = e.mu; m.l2m = e.l2m; m.p7 = e.p7; m.p8 = e.p8;
  return m;
}

template <typename G, typename A, bool INTERP>
__global__ void __launch_bounds__(256) k_defgrad(int32_t n, const int64_t* __restrict__ rowptr,
                                                 const int32_t* __restrict__ col, const G* __restrict__ gx,
                                                 const G* __restrict__ gy, const G* __restrict__ gz,
                                                 const double* __restrict__ dsp,
                                                 const double* __restrict__ dsp_tot,
                                                 const double* __restrict__ sdphi,
                                                 const double* __restrict__ shp,
                                                 double* __restrict__ dsp_tot_phy, double* __restrict__ fg,
                                                 StepAccum* __restrict__ acc) {
  if (acc && blockIdx.x == 0 && threadIdx.x < kSlots) {  // per-step counters of the stress kernel
    acc->newton_iters[threadIdx.x] = 0ull;
    acc->plastic[threadIdx.x] = 0ull;
  }
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kGroup;
  const int q = threadIdx.x & (kGroup - 1);
  const unsigned gmask = 0xFu << (threadIdx.x & 28);
  if (i >= n) return;
  const double ui0 = dsp_tot[3 * i], ui1 = dsp_tot[3 * i + 1], ui2 = dsp_tot[3 * i + 2];
  const double di0 = dsp[3 * i], di1 = dsp[3 * i + 1], di2 = dsp[3 * i + 2];
  A F[9], L[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) { F[k] = A(0); L[k] = A(0); }
  double ph0 = 0.0, ph1 = 0.0, ph2 = 0.0;
  const int64_t p1 = rowptr[i + 1];
  for (int64_t p = rowptr[i] + q; p < p1; p += kGroup) {
    const int64_t j = col[p];
    const A g0 = (A)gx[p], g1 = (A)gy[p], g2 = (A)gz[p];
    const A u0 = (A)(dsp_tot[3 * j] - ui0), u1 = (A)(dsp_tot[3 * j + 1] - ui1), u2 = (A)(dsp_tot[3 * j + 2] - ui2);
    const double dj0 = dsp[3 * j], dj1 = dsp[3 * j + 1], dj2 = dsp[3 * j + 2];
    const A d0 = (A)(dj0 - di0), d1 = (A)(dj1 - di1), d2 = (A)(dj2 - di2);
    F[0] += u0 * g0; F[1] += u0 * g1; F[2] += u0 * g2;
    F[3] += u1 * g0; F[4] += u1 * g1; F[5] += u1 * g2;
    F[6] += u2 * g0; F[7] += u2 * g1; F[8] += u2 * g2;
    L[0] += d0 * g0; L[1] += d0 * g1; L[2] += d0 * g2;
    L[3] += d1 * g0; L[4] += d1 * g1; L[5] += d1 * g2;
    L[6] += d2 * g0; L[7] += d2 * g1; L[8] += d2 * g2;
    if (INTERP) {
      const double s = shp[p];
      ph0 += s * dj0; ph1 += s * dj1; ph2 += s * dj2;
    }
  }
#pragma unroll
  for (int o = 1; o < kGroup; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      F[k] += __shfl_xor_sync(gmask, F[k], o);
      L[k] += __shfl_xor_sync(gmask, L[k], o);
    }
    if (INTERP) {
      ph0 += __shfl_xor_sync(gmask, ph0, o);
      ph1 += __shfl_xor_sync(gmask, ph1, o);
      ph2 += __shfl_xor_sync(gmask, ph2, o);
    }
  }
  if (q == 0) {
    const double s0 = sdphi[3 * i], s1 = sdphi[3 * i + 1], s2 = sdphi[3 * i + 2];
    const double ui[3] = {ui0, ui1, ui2}, di[3] = {di0, di1, di2}, sd[3] = {s0, s1, s2};
    double* o = fg + 18 * i;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        o[3 * k + l] = (k == l ? 1.0 : 0.0) + ((double)F[3 * k + l] + ui[k] * sd[l]);
        o[9 + 3 * k + l] = (double)L[3 * k + l] + di[k] * sd[l];
      }
    if (INTERP) {
      dsp_tot_phy[3 * i] += ph0;
      dsp_tot_phy[3 * i + 1] += ph1;
      dsp_tot_phy[3 * i + 2] += ph2;
    }
  }
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  T r = T(0);
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

// State of one node between the trial part of the update (kinematics,
// rotation, elastic predictor) and the rest (return mapping, write-back).
// LEAN: the old stress / strain and the material entry are re-read by the
// second part instead of held (the members stay unused and take no
// registers), which keeps the state small across the learned kernel's
// network evaluation.
template <typename T, bool LEAN>
struct Trial {
  double spred[6];
  T eps6[6], D[6], IF[3][3];
  double det;
  int mi;  // material table index
  double sold[6], eold[6];
  MatEntry me;
};

// FINT.F90:363-794: |det F|, INV3(F), L = G0 INV3(F), Hughes-Winget, rotation
// of sigma and eps, eps += dstrain, elastic predictor.
// DAM: the context holds damaged models (materials 3, 6) and their state;
// without it their branches compile out of the J2 path.
template <typename T, bool LEAN, bool DAM>
__device__ __forceinline__ void stress_trial(const StressArgs& a, int64_t i, Trial<T, LEAN>& w) {
  // F, G0 (18 doubles), stress and strain (6 each) as 16-byte loads
  double fgi[18], sv[6], ev[6];
  load_fg(a.fg, i, sizeof(T) == 4, fgi);  // float F - I and G0 in mixed precision
  {
    const double2* s2 = reinterpret_cast<const double2*>(a.stress + 6 * i);
    const double2* e2 = reinterpret_cast<const double2*>(a.strain + 6 * i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 v = s2[k], u = e2[k];
      sv[2 * k] = v.x; sv[2 * k + 1] = v.y; ev[2 * k] = u.x; ev[2 * k + 1] = u.y;
    }
  }
  w.mi = a.matidx[i];
  if (!LEAN) w.me = a.mats[w.mi];
  const MatEntry& me = LEAN ? a.mats[w.mi] : w.me;
  T G0[3][3], L[3][3], sig[6], dstr[6];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l) G0[k][l] = (T)fgi[9 + 3 * k + l];
  w.det = 1.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double so = sv[k], eo = ev[k];
    if (!LEAN) { w.sold[k] = so; w.eold[k] = eo; }
    sig[k] = (T)so;
    w.eps6[k] = (T)eo;
    w.D[k] = T(0);
  }
  if (a.finite_strain) {
    // |det F| and INV3 in double (F carries the FP64 displacement path)
    double Fd[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) Fd[k][l] = fgi[3 * k + l];
    w.det = det_abs(Fd);
    double IFd[3][3];
    inv3(Fd, IFd, a.inv3_exact != 0);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) w.IF[k][l] = (T)IFd[k][l];
    mm3(G0, w.IF, L);
    T R[3][3];
    hughes_winget(L, R, dstr, w.D, a.inv3_exact != 0);
    rotate_tensor(R, sig);
    rotate_tensor(R, w.eps6);
  } else {
    // FINT.F90:772-783 small strain: engineering shear, no rotation, DET = 1
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) w.IF[k][l] = (k == l) ? T(1) : T(0);
    dstr[0] = G0[0][0]; dstr[1] = G0[1][1]; dstr[2] = G0[2][2];
    dstr[3] = G0[2][1] + G0[1][2]; dstr[4] = G0[2][0] + G0[0][2]; dstr[5] = G0[1][0] + G0[0][1];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) w.eps6[k] = w.eps6[k] + dstr[k];
  // the damaged models predict in effective space: STRESS / (1 - DAM)
  // (CONSTITUTE_VONMISES_DAM.F90:83, CONSTITUTE_DRUCKPRAG.F90:79)
  if (DAM && damaged_type(me.type)) {
    const T keep = T(1) - (T)a.aux[4 * i + 2];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = sig[k] / keep;
  }
  // elastic predictor with FORM_CMAT (FINT_FUNCTIONS.F90:252-288)
  const T lam = (T)me.lam, mu = (T)me.mu, l2m = (T)me.l2m;
  w.spred[0] = (double)(sig[0] + (l2m * dstr[0] + lam * dstr[1] + lam * dstr[2]));
  w.spred[1] = (double)(sig[1] + (lam * dstr[0] + l2m * dstr[1] + lam * dstr[2]));
  w.spred[2] = (double)(sig[2] + (lam * dstr[0] + lam * dstr[1] + l2m * dstr[2]));
  w.spred[3] = (double)(sig[3] + mu * dstr[3]);
  w.spred[4] = (double)(sig[4] + mu * dstr[4]);
  w.spred[5] = (double)(sig[5] + mu * dstr[5]);
}

// Inputs of the surrogate network for a rate-dependent node: with q the
// trial deviatoric norm, sy0 = A + B eps0^n and f = q - sqrt(2/3) sy0,
//   x0 = ln(f / (sqrt(2/3) sy0))            overstress
//   x1 = eps0^n                             hardening state
//   x2 = ln(max(sqrt(2/3) f/(2 mu)/dt, epsdot0)/epsdot0) / 10   rate
//   x3 = 1e3 sqrt(2/3) sy0 / (2 mu)          yield-strain scale
// The target is y = dgamma / ub with ub = rate_upper_bound(f, eps0).
// Returns f (<= 0: elastic) and ub.
__device__ __forceinline__ double rate_features(const double spred[6], double eps0, const MatEntry& me, double dt,
                                                float x[4], double& ub) {
  const double mu = me.E / (2.0 * (1.0 + me.nu));
  const double kk = spred[0] + spred[1] + spred[2];
  const double d0 = spred[0] - kk / 3.0, d1 = spred[1] - kk / 3.0, d2 = spred[2] - kk / 3.0;
  const double q = sqrt(d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (spred[3] * spred[3] + spred[4] * spred[4] +
                                                             spred[5] * spred[5]));
  const double s23 = sqrt(2.0 / 3.0);
  const double epn = (eps0 > 0.0) ? pow(eps0, me.C) : 0.0;
  const double sy0 = me.sig0 + me.B * epn;
  const double f = q - s23 * sy0;
  const double dgpp = f / (2.0 * mu);
  ub = f > 0.0 ? rate_upper_bound(f, eps0, mu, me.B, me.C) : 0.0;
  x[0] = (float)log(fmax(f, 1e-30 * sy0) / (s23 * sy0));
  x[1] = (float)epn;
  x[2] = (float)(log(fmax(s23 * dgpp / dt, me.p8) / me.p8) / 10.0);
  x[3] = (float)(1e3 * s23 * sy0 / (2.0 * mu));
  return f;
}

// FINT.F90:797-870, 999-1116: return mapping (dg0 >= 0 starts the rate law's
// Newton there), state write-back, strain_eq, internal work, wave speed, T_i.
template <typename T, typename TS, bool LEAN, bool DAM>
__device__ __forceinline__ void stress_finish(const StressArgs& a, int64_t i, Trial<T, LEAN>& w, double dg0, double& work,
                                              unsigned long long& nit, unsigned long long& npl, unsigned& st) {
  const MatEntry& me = LEAN ? a.mats[w.mi] : w.me;
  const NodeMat m = to_nodemat(me);
  const double vol = a.vol[i];
  double snew[6];
  double ep = a.eps[i];
  const double ep0 = ep;
  int it = 0;
  bool cap = false;
  if (m.type == MEGA_MAT_ELASTIC) {
#pragma unroll
    for (int k = 0; k < 6; ++k) snew[k] = w.spred[k];
  } else if (m.type == MEGA_MAT_VONMISES) {
    it = von_mises(w.spred, ep, m, a.maxit, snew, cap);
  } else if (m.type == MEGA_MAT_VM_RATE) {
    double dg = 0.0, ftr = 0.0;
    const double dt = a.ndt ? a.ndt[i] : a.dt;
    it = vm_rate(w.spred, ep, m, dt, a.rtol, a.maxit, a.rate_solver, dg0, snew, cap, dg, ftr);
    if (a.log_buf && it > 0) {  // sample (features, converged multiplier) for the surrogate
      const uint64_t sb = (uint64_t)__double_as_longlong(w.spred[0]);
      const uint32_t hsh = ((uint32_t)i * 2654435761u) ^ (uint32_t)(sb ^ (sb >> 29)) ^ a.log_seed;
      if (hsh % a.log_stride == 0) {
        float x[4];
        double ub;
        const double f = rate_features(w.spred, ep0, me, dt, x, ub);
        if (f > 0.0 && ub > 0.0) {
          const unsigned long long k = atomicAdd(a.log_count, 1ull);
          if ((int64_t)k < a.log_cap) {
            float* o = a.log_buf + 5 * k;
            o[0] = x[0]; o[1] = x[1]; o[2] = x[2]; o[3] = x[3];
            o[4] = (float)(dg / ub);
          }
        }
      }
    }
  } else if (DAM && damaged_type(m.type)) {
    // CONSTITUTION.F90:60-64, 72-76: the total strain (already advanced by
    // dstrain) and the four damage-state values ride along; spred is the
    // effective predictor
    double tot[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) tot[k] = (double)w.eps6[k];
    double2* a2 = reinterpret_cast<double2*>(a.aux + 4 * i);
    const double2 x0 = a2[0], x1 = a2[1];
    double ax[4] = {x0.x, x0.y, x1.x, x1.y};
    const DamageMat d{me.ki, me.kc, me.dmax, me.qphi, me.kphi, me.qpsi};
    if (m.type == MEGA_MAT_VM_DAMAGE) it = von_mises_dam(w.spred, tot, ep, ax, m, d, a.maxit, snew, cap);
    else it = drucker_prager(w.spred, tot, ep, ax, m, d, snew);
    a2[0] = make_double2(ax[0], ax[1]);
    a2[1] = make_double2(ax[2], ax[3]);
  } else {
    st |= MEGA_ST_BAD_MATERIAL;
#pragma unroll
    for (int k = 0; k < 6; ++k) snew[k] = w.spred[k];
  }
  if (cap) st |= MEGA_ST_NEWTON_CAP;
  nit += (unsigned long long)it;
  npl += (it > 0) ? 1ull : 0ull;
  if (a.iters) a.iters[i] = it;
  double sinc[6], einc[6], enew[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    enew[k] = (double)w.eps6[k];
    sinc[k] = snew[k] - (LEAN ? a.stress[6 * i + k] : w.sold[k]);
    einc[k] = enew[k] - (LEAN ? a.strain[6 * i + k] : w.eold[k]);
  }
  {
    double2* s2 = reinterpret_cast<double2*>(a.stress + 6 * i);
    double2* e2 = reinterpret_cast<double2*>(a.strain + 6 * i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      s2[k] = make_double2(snew[2 * k], snew[2 * k + 1]);
      e2[k] = make_double2(enew[2 * k], enew[2 * k + 1]);
    }
  }
  a.eps[i] = ep;
  const double eq = enew[0] * enew[0] + enew[1] * enew[1] + enew[2] * enew[2] +
                    2.0 * (enew[3] * enew[3] + enew[4] * enew[4] + enew[5] * enew[5]);
  a.strain_eq[i] = sqrt(eq * 2.0 / 3.0);
  if (a.finite_strain) {
#pragma unroll
    for (int k = 0; k < 6; ++k) work += 0.5 * (double)w.D[k] * (2.0 * snew[k] - sinc[k]) * vol * w.det;
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k) work += 0.5 * einc[k] * sinc[k] * vol * w.det;
  }
  double bulk = m.E / (3.0 * (1.0 - 2.0 * m.nu)), shear = m.E / (2.0 * (1.0 + m.nu));
  if (m.type > 1) estimate_moduli(sinc, einc, shear, bulk);
  const double pmod = bulk + 4.0 * shear / 3.0;
  a.wvel[i] = sqrt(fmax(pmod, shear) / m.rho);
  // T_i = V J sigma IF^T: f_J(k) = sum_m T(k,m) grad0 phi_iJ(m)
  const T vj = (T)(vol * w.det);
  T S[3][3];
  T sn[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) sn[k] = (T)snew[k];
  v2t(sn, S);
  TS tv[12];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int mm = 0; mm < 3; ++mm)
      tv[3 * k + mm] = (TS)(vj * (S[k][0] * w.IF[mm][0] + S[k][1] * w.IF[mm][1] + S[k][2] * w.IF[mm][2]));
  tv[9] = tv[10] = tv[11] = TS(0);
  if (a.has_body) {
    const double rvj = m.rho * vol * w.det;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double b = (a.bodyforce ? a.bodyforce[3 * i + k] : 0.0) + a.grav[k];
      tv[9 + k] = (TS)(b * rvj);
    }
  }
  // the 12-value row (48 or 96 bytes, 16-byte aligned) as vector stores
  if (sizeof(TS) == 4) {
    float4* t4 = reinterpret_cast<float4*>((TS*)a.tmat + 12 * i);
#pragma unroll
    for (int k = 0; k < 3; ++k)
      t4[k] = make_float4((float)tv[4 * k], (float)tv[4 * k + 1], (float)tv[4 * k + 2], (float)tv[4 * k + 3]);
  } else {
    double2* t2 = reinterpret_cast<double2*>((TS*)a.tmat + 12 * i);
#pragma unroll
    for (int k = 0; k < 6; ++k) t2[k] = make_double2((double)tv[2 * k], (double)tv[2 * k + 1]);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    if (!isfinite(snew[k])) st |= MEGA_ST_NONFINITE;
}

template <typename T>
__device__ __forceinline__ void stress_reduce(const StressArgs& a, double work, unsigned long long nit,
                                              unsigned long long npl, unsigned st, double* smd,
                                              unsigned long long* smu) {
  const double wsum = block_sum(work, smd);
  const unsigned long long it_sum = block_sum(nit, smu);
  const unsigned long long pl_sum = block_sum(npl, smu);
  if (threadIdx.x == 0) {
    const int sl = blockIdx.x % kSlots;
    if (wsum != 0.0) atomicAdd(&a.acc->int_work[sl], wsum);
    if (it_sum) { atomicAdd(&a.acc->newton_iters[sl], it_sum); atomicAdd(&a.acc->newton_total[sl], it_sum); }
    if (pl_sum) { atomicAdd(&a.acc->plastic[sl], pl_sum); atomicAdd(&a.acc->plastic_total[sl], pl_sum); }
  }
  if (st) atomicOr(a.status, st);
}

// Overstress f = q - sqrt(2/3) (A + B eps0^n) of a rate-dependent trial
// state (q its deviatoric norm): f > 0 takes a plastic return.
__device__ __forceinline__ double rate_overstress(const double spred[6], double eps0, const MatEntry& me) {
  const double kk = spred[0] + spred[1] + spred[2];
  const double d0 = spred[0] - kk / 3.0, d1 = spred[1] - kk / 3.0, d2 = spred[2] - kk / 3.0;
  const double q = sqrt(d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (spred[3] * spred[3] + spred[4] * spred[4] +
                                                             spred[5] * spred[5]));
  const double epn = (eps0 > 0.0) ? pow(eps0, me.C) : 0.0;
  return q - sqrt(2.0 / 3.0) * (me.sig0 + me.B * epn);
}

// T = arithmetic of kinematics / rotation / predictor, TS = storage of T_i.
// QUEUE (the learned start): plastic rate-dependent nodes are not finished
// here but listed in a.queue (one atomic per warp) for k_stress_queue, so
// the network and its Newton polish run on full warps of plastic nodes only.
template <typename T, typename TS, bool DAM, bool QUEUE>
__global__ void __launch_bounds__(256, 2) k_stress(StressArgs a) {
  __shared__ double smd[32];
  __shared__ unsigned long long smu[32];
  if (blockIdx.x == 0 && threadIdx.x < kSlots) {
    a.acc->ke[threadIdx.x] = 0.0;  // the force kernel of this step accumulates it afresh
  }
  double work = 0.0;
  unsigned long long nit = 0, npl = 0;
  unsigned st = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    Trial<T, false> w;
    stress_trial<T, false, DAM>(a, i, w);
    if (QUEUE) {
      const bool push = w.me.type == MEGA_MAT_VM_RATE && rate_overstress(w.spred, a.eps[i], w.me) > 0.0;
      const unsigned act = __activemask();
      const unsigned bal = __ballot_sync(act, push);
      if (bal) {
        const int lane = threadIdx.x & 31, lead = __ffs(bal) - 1;
        unsigned base = 0;
        if (lane == lead) base = atomicAdd(a.qcount, (unsigned)__popc(bal));
        base = __shfl_sync(act, base, lead);
        if (push) a.queue[base + __popc(bal & ((1u << lane) - 1u))] = (int32_t)i;
      }
      if (push) continue;
    }
    stress_finish<T, TS, false, DAM>(a, i, w, -1.0, work, nit, npl, st);
  }
  stress_reduce<T>(a, work, nit, npl, st, smd, smu);
}

// The learned start: warps of 32 plastic rate-dependent nodes evaluate the
// surrogate together (the 64x64 layer on the tensor cores, mlp_tc.cuh) and
// each node starts its Newton iteration from dgamma0 = clamp(y, 1e-3, 1) ub
// (ub = rate_upper_bound).
constexpr int kLearnBlock = 128;

// The queued plastic rate-dependent nodes of k_stress<..., QUEUE>: warps of
// 32 queued nodes recompute their trial states (the stored state is still
// the old one), evaluate the surrogate together and start Newton from it.
template <typename T, typename TS, bool DAM>
__global__ void __launch_bounds__(kLearnBlock, 4) k_stress_queue(StressArgs a) {
  __shared__ double smd[32];
  __shared__ unsigned long long smu[32];
  __shared__ __align__(16) MlpSmem net;
  __shared__ __align__(16) uint16_t sH1[kLearnBlock * kMlpLd];
  __shared__ float sOut[kLearnBlock];
  const int64_t count = *a.qcount;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t first = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
  double work = 0.0;
  unsigned long long nit = 0, npl = 0;
  unsigned st = 0;
  if (first < count) {  // a block with queued nodes loads the network
    mlp_load(net, a.mlp_w2, a.mlp_small);
  }
  __syncthreads();
  uint16_t* hw = sH1 + (wid * 32) * kMlpLd;
  float* ow = sOut + wid * 32;
  for (int64_t base = first; base < count; base += nwarps * 32) {
    const int64_t k = base + lane;
    const bool act = k < count;
    const int64_t i = act ? a.queue[k] : 0;
    Trial<T, true> w;
    float x[4] = {0.f, 0.f, 0.f, 0.f};
    double ub = 0.0, f = -1.0;
    if (act) {
      stress_trial<T, true, DAM>(a, i, w);
      f = rate_features(w.spred, a.eps[i], a.mats[w.mi], a.ndt ? a.ndt[i] : a.dt, x, ub);
    }
    const float y = warp_mlp(x, act && f > 0.0, net, hw, ow);
    if (act) {
      const double dg0 = f > 0.0 ? (double)fminf(fmaxf(y, 1e-3f), 1.0f) * ub : -1.0;
      stress_finish<T, TS, true, DAM>(a, i, w, dg0, work, nit, npl, st);
    }
  }
  stress_reduce<T>(a, work, nit, npl, st, smd, smu);
}

// G = storage of grad phi, TS = storage of T_i, A = accumulation
template <typename G, typename TS, typename A>
__global__ void __launch_bounds__(256) k_force(ForceArgs a) {
  __shared__ double smd[32];
  const int64_t* __restrict__ colptr = a.csr->colptr;
  const int32_t* __restrict__ trow = a.csr->trow;
  const G* __restrict__ tgx = (const G*)a.tgx;
  const G* __restrict__ tgy = (const G*)a.tgy;
  const G* __restrict__ tgz = (const G*)a.tgz;
  const TS* __restrict__ tm = (const TS*)a.tmat;
  const int q = threadIdx.x & (kGroup - 1);
  const unsigned gmask = 0xFu << (threadIdx.x & 28);
  double ke = 0.0, ee = 0.0, tf[6] = {0, 0, 0, 0, 0, 0};
  unsigned st = 0;
  const int64_t groups = ((int64_t)gridDim.x * blockDim.x) / kGroup;
  // every lane of a group runs the same iterations, so group shuffles are safe
  for (int64_t J = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kGroup; J < a.n; J += groups) {
    A f0 = A(0), f1 = A(0), f2 = A(0);
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    const int64_t c1 = colptr[J + 1];
    for (int64_t e = colptr[J] + q; e < c1; e += kGroup) {
      const int64_t i = trow[e];
      const A g0 = (A)tgx[e], g1 = (A)tgy[e], g2 = (A)tgz[e];
      const TS* t = tm + 12 * i;
      f0 += (A)t[0] * g0 + (A)t[1] * g1 + (A)t[2] * g2;
      f1 += (A)t[3] * g0 + (A)t[4] * g1 + (A)t[5] * g2;
      f2 += (A)t[6] * g0 + (A)t[7] * g1 + (A)t[8] * g2;
      if (a.has_body) {
        const double s = a.tshp[e];
        e0 += s * (double)t[9]; e1 += s * (double)t[10]; e2 += s * (double)t[11];
      }
    }
#pragma unroll
    for (int o = 1; o < kGroup; o <<= 1) {
      f0 += __shfl_xor_sync(gmask, f0, o);
      f1 += __shfl_xor_sync(gmask, f1, o);
      f2 += __shfl_xor_sync(gmask, f2, o);
      if (a.has_body) {
        e0 += __shfl_xor_sync(gmask, e0, o);
        e1 += __shfl_xor_sync(gmask, e1, o);
        e2 += __shfl_xor_sync(gmask, e2, o);
      }
    }
    if (q < 3) {
      const int64_t m = 3 * J + q;
      const double fi = (double)(q == 0 ? f0 : (q == 1 ? f1 : f2));
      double fe = (q == 0 ? e0 : (q == 1 ? e1 : e2));
      if (!isfinite(fi)) st |= MEGA_ST_NONFINITE;
      if (!a.integrate) {
        a.fint[m] = fi;
        a.fext[m] = fe;
      } else {
        const double mass = a.mass[m];
        const double fe_old = a.fext[m];
        double v = a.vel[m], acc, pr;
        const int code = a.ebc[m];
        if (code == 1 || code == 2) {  // MAIN.F90:438-445 (fixed), 447-470 (prescribed velocity)
          v = code == 1 ? 0.0 : a.vel2[q];
          acc = 0.0;
          pr = -fi;
          fe = -fi;
        } else {  // MAIN.F90:472-481
          const double mpdc = a.mats[a.matidx[J]].damp * mass;
          acc = (fe - fi - mpdc * v) / (mass + 0.5 * a.dt * mpdc);
          v = v + 0.5 * a.dt * acc;
          pr = 0.0;
        }
        const double d_old = a.dsp[m];
        ee += 0.5 * (fe + fe_old) * d_old;
        ke += 0.5 * mass * v * v;
        const int b = a.body_id ? a.body_id[J] : 1;
        if (b == 1) tf[q] += pr;
        else if (b == 2) tf[3 + q] += pr;
        a.fint[m] = fi;
        a.fext[m] = fe;
        a.acl[m] = acc;
        a.prforce[m] = pr;
        if (a.predict) {  // MAIN.F90:353-355 of the next step
          const double d = a.dt * v + a.dt * a.dt * 0.5 * acc;
          a.dsp[m] = d;
          a.dsp_tot[m] = a.dsp_tot[m] + d;
          v = v + a.dt * 0.5 * acc;
        }
        a.vel[m] = v;
      }
    }
  }
  if (a.integrate) {
    const double ks = block_sum(ke, smd);
    const double es = block_sum(ee, smd);
    double ts[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) ts[k] = block_sum(tf[k], smd);
    if (threadIdx.x == 0) {
      const int sl = blockIdx.x % kSlots;
      atomicAdd(&a.acc->ke[sl], ks);
      if (es != 0.0) atomicAdd(&a.acc->ee[sl], es);
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (ts[k] != 0.0) atomicAdd(&a.acc->tf[k][sl], ts[k]);
    }
  }
  if (st) atomicOr(a.status, st);
}

__global__ void k_predict(int64_t n3, double* __restrict__ dsp, double* __restrict__ dsp_tot,
                          double* __restrict__ vel, const double* __restrict__ acl, double dt,
                          const double* __restrict__ ndt) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= n3) return;
  if (ndt) dt = ndt[m / 3];
  const double v = vel[m], a = acl[m];
  const double d = dt * v + dt * dt * 0.5 * a;
  dsp[m] = d;
  dsp_tot[m] = dsp_tot[m] + d;
  vel[m] = v + dt * 0.5 * a;
}

__global__ void k_interp(int32_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                         const double* __restrict__ shp, const double* __restrict__ val,
                         const double* __restrict__ base, double* __restrict__ out) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kGroup;
  const int q = threadIdx.x & (kGroup - 1);
  const unsigned gmask = 0xFu << (threadIdx.x & 28);
  if (i >= n) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t p = rowptr[i] + q; p < rowptr[i + 1]; p += kGroup) {
    const int64_t j = col[p];
    const double w = shp[p];
    s0 += w * val[3 * j]; s1 += w * val[3 * j + 1]; s2 += w * val[3 * j + 2];
  }
#pragma unroll
  for (int o = 1; o < kGroup; o <<= 1) {
    s0 += __shfl_xor_sync(gmask, s0, o);
    s1 += __shfl_xor_sync(gmask, s1, o);
    s2 += __shfl_xor_sync(gmask, s2, o);
  }
  if (q == 0) {
    out[3 * i] = (base ? base[3 * i] : 0.0) + s0;
    out[3 * i + 1] = (base ? base[3 * i + 1] : 0.0) + s1;
    out[3 * i + 2] = (base ? base[3 * i + 2] : 0.0) + s2;
  }
}

inline unsigned grid_for(int64_t work, int block) { return (unsigned)((work + block - 1) / block); }

}  // namespace

int device_sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

int launch_defgrad(cudaStream_t s, bool mixed, bool interp, int32_t n, const DevCSR& csr, const void* gx,
                   const void* gy, const void* gz, const double* dsp, const double* dsp_tot,
                   const double* sdphi, const double* shp, double* dsp_tot_phy, double* fg, StepAccum* acc) {
  const int block = 256;
  const unsigned grid = grid_for((int64_t)n * kGroup, block);
  if (mixed) {
    if (interp)
      k_defgrad<float, float, true><<<grid, block, 0, s>>>(n, csr.rowptr, csr.col, (const float*)gx,
                                                           (const float*)gy, (const float*)gz, dsp, dsp_tot,
                                                           sdphi, shp, dsp_tot_phy, fg, acc);
    else
      k_defgrad<float, float, false><<<grid, block, 0, s>>>(n, csr.rowptr, csr.col, (const float*)gx,
                                                            (const float*)gy, (const float*)gz, dsp, dsp_tot,
                                                            sdphi, shp, dsp_tot_phy, fg, acc);
  } else {
    if (interp)
      k_defgrad<double, double, true><<<grid, block, 0, s>>>(n, csr.rowptr, csr.col, (const double*)gx,
                                                             (const double*)gy, (const double*)gz, dsp,
                                                             dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc);
    else
      k_defgrad<double, double, false><<<grid, block, 0, s>>>(n, csr.rowptr, csr.col, (const double*)gx,
                                                              (const double*)gy, (const double*)gz, dsp,
                                                              dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc);
  }
  MEGA_CHECK_LAUNCH();
  return 0;
}

int launch_stress(cudaStream_t s, bool mixed, const StressArgs& a) {
  const int block = 256;
  const int64_t need = grid_for(a.n, block);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)device_sm_count() * 8));
  if (a.mlp_w2 && a.mlp_small && a.queue && a.qcount) {
    // learned start: elastic nodes finish in the first kernel, plastic
    // rate-dependent ones are queued for the network kernel
    const int64_t lneed = grid_for(a.n, kLearnBlock);
    const unsigned lgrid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(lneed, (int64_t)device_sm_count() * 8));
    MEGA_TRY(cudaMemsetAsync(a.qcount, 0, sizeof(unsigned), s));
    if (a.aux) {
      if (mixed) k_stress<float, float, true, true><<<grid, block, 0, s>>>(a);
      else k_stress<double, double, true, true><<<grid, block, 0, s>>>(a);
      MEGA_CHECK_LAUNCH();
      if (mixed) k_stress_queue<float, float, true><<<lgrid, kLearnBlock, 0, s>>>(a);
      else k_stress_queue<double, double, true><<<lgrid, kLearnBlock, 0, s>>>(a);
    } else {
      if (mixed) k_stress<float, float, false, true><<<grid, block, 0, s>>>(a);
      else k_stress<double, double, false, true><<<grid, block, 0, s>>>(a);
      MEGA_CHECK_LAUNCH();
      if (mixed) k_stress_queue<float, float, false><<<lgrid, kLearnBlock, 0, s>>>(a);
      else k_stress_queue<double, double, false><<<lgrid, kLearnBlock, 0, s>>>(a);
    }
  } else {
    if (a.aux) {
      if (mixed) k_stress<float, float, true, false><<<grid, block, 0, s>>>(a);
      else k_stress<double, double, true, false><<<grid, block, 0, s>>>(a);
    } else {
      if (mixed) k_stress<float, float, false, false><<<grid, block, 0, s>>>(a);
      else k_stress<double, double, false, false><<<grid, block, 0, s>>>(a);
    }
  }
  MEGA_CHECK_LAUNCH();
  return 0;
}

int launch_force(cudaStream_t s, bool mixed, const ForceArgs& a) {
  const int block = 256;
  const int64_t need = grid_for((int64_t)a.n * kGroup, block);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)device_sm_count() * 8));
  if (mixed) k_force<float, float, float><<<grid, block, 0, s>>>(a);
  else k_force<double, double, double><<<grid, block, 0, s>>>(a);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int launch_predict(cudaStream_t s, int64_t n3, double* dsp, double* dsp_tot, double* vel, const double* acl,
                   double dt, const double* ndt) {
  if (n3 <= 0) return 0;
  k_predict<<<grid_for(n3, 256), 256, 0, s>>>(n3, dsp, dsp_tot, vel, acl, dt, ndt);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int launch_interp(cudaStream_t s, int32_t n, const DevCSR& csr, const double* shp, const double* val,
                  const double* base, double* out) {
  k_interp<<<grid_for((int64_t)n * kGroup, 256), 256, 0, s>>>(n, csr.rowptr, csr.col, shp, val, base, out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

}  // namespace mega
