// nsni.cu -- naturally stabilised nodal integration (ITYPE_INT = 2) on the
// resident path.
//
// The reference lays NSNI out but never finishes it (FINT.F90:441-576,
// 707-753, 1120-1222 are commented out or read arrays nothing fills), so
// this follows the published method (Hillman & Chen 2016, IJNME 107:603) in
// the reference's layout:
//   set-up   smoothed second derivatives S of every list entry: RK gradients
//            at the six faces x +- SM_LEN of the node's smoothing cell,
//            differenced over the cell width (FINT.F90:446-535), order
//            XX, YY, ZZ, XY, YZ, XZ (SHPDD_SM);
//   per step (double arithmetic; S and the force weights stored as float in
//            mixed mode)
//            k_nsni_h      (row gather) the gradients of the incremental
//            displacement gradient, H_a(k,m) = sum_J S_(m a)(J) du_J,k
//            (XLMAT/YLMAT/ZLMAT, FINT.F90:728-737); the mixed steps form H
//            in the tiled row gather instead (tiled.cu, NS);
//            k_nsni_stress (node) the strain-gradient increments of
//            D_HUGHES_WINGET (HUGHES_WINGET.F90:84-165), stress gradients
//            sigma_,a rotated with the step's rotation and advanced with an
//            isotropic tangent probed from the node's own stress and strain
//            increments (ESTIMATE_MODULI with NSNI_FLAG, capped at the
//            elastic moduli), their work, and the per-node weights
//            W_a = M_a / V * V J sigma_,a INV3(F)^T with the second moments
//            M_a / V = (cell width_a)^2 / 12 (PRE_MODEL_SECOND_MOMENT.F90);
//            k_nsni_force  (column gather) f_J += sum_a W_a S_(. a)(J)
//            (FINT.F90:1127-1208), added by the force kernel before the
//            corrector; the mixed steps sum it in the tiled column gather.
#include "mega_internal.cuh"

namespace mega {
namespace {

constexpr int kNL = 8;  // lanes per node of the two gathers

// node stride of the force weights W: 18 doubles (144 B, nine 16-byte
// loads) or 18 floats padded to 20 (80 B, five 16-byte loads)
template <typename V>
constexpr int w_stride() { return sizeof(V) == 4 ? 20 : 18; }

// index of S_(m a) in the XX, YY, ZZ, XY, YZ, XZ order
__device__ __forceinline__ int dd_index(int m, int a) {
  if (m == a) return m;
  const int lo = m < a ? m : a, hi = m < a ? a : m;
  return lo == 0 ? (hi == 1 ? 3 : 5) : 4;
}

// One axis of the set-up: gp/gm = RK gradients at the + and - faces along
// axis a.  Pass a = 0 writes XX and the raw x-differences of the y- and
// z-derivatives into XY / XZ; pass 1 writes YY, completes XY as the mean of
// both differences and stores the raw one for YZ; pass 2 completes YZ, XZ.
__global__ void k_nsni_combine(int32_t n, int a, const int64_t* __restrict__ rowptr, const double* __restrict__ sml,
                               const double* __restrict__ gp0, const double* __restrict__ gp1,
                               const double* __restrict__ gp2, const double* __restrict__ gm0,
                               const double* __restrict__ gm1, const double* __restrict__ gm2, NsniS s) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const double w = sml[6 * i + 2 * a] + sml[6 * i + 2 * a + 1];
  for (int64_t p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) {
    const double d0 = (gp0[p] - gm0[p]) / w, d1 = (gp1[p] - gm1[p]) / w, d2 = (gp2[p] - gm2[p]) / w;
    if (a == 0) {
      s.v[0][p] = d0;
      s.v[3][p] = d1;
      s.v[5][p] = d2;
    } else if (a == 1) {
      s.v[1][p] = d1;
      s.v[3][p] = 0.5 * (s.v[3][p] + d0);
      s.v[4][p] = d2;
    } else {
      s.v[2][p] = d2;
      s.v[4][p] = 0.5 * (s.v[4][p] + d1);
      s.v[5][p] = 0.5 * (s.v[5][p] + d0);
    }
  }
}

// hq[18 i + 6 k + q] = sum_J S_q(J) du_J,k (S double or float, sums in double)
template <typename SV>
__global__ void __launch_bounds__(256) k_nsni_h(int32_t n, const int64_t* __restrict__ rowptr,
                                                const int32_t* __restrict__ col, NsniArr<SV> s,
                                                const double* __restrict__ du, double* __restrict__ hq) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kNL;
  const int q = threadIdx.x & (kNL - 1);
  const unsigned gm = 0xFFu << (threadIdx.x & 24);
  if (i >= n) return;
  double h[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) h[k] = 0.0;
  // two entries per pass (p, p + kNL): both gathers are in flight before
  // either is summed; each lane still sums its entries in list order
  auto add = [&](int64_t p, double u0, double u1, double u2) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const double sv = (double)s.v[c][p];
      h[c] += sv * u0;
      h[6 + c] += sv * u1;
      h[12 + c] += sv * u2;
    }
  };
  int64_t p = rowptr[i] + q;
  const int64_t pe = rowptr[i + 1];
  for (; p + kNL < pe; p += 2 * kNL) {
    const int64_t j0 = col[p], j1 = col[p + kNL];
    const double a0 = du[3 * j0], a1 = du[3 * j0 + 1], a2 = du[3 * j0 + 2];
    const double b0 = du[3 * j1], b1 = du[3 * j1 + 1], b2 = du[3 * j1 + 2];
    add(p, a0, a1, a2);
    add(p + kNL, b0, b1, b2);
  }
  if (p < pe) {
    const int64_t j = col[p];
    add(p, du[3 * j], du[3 * j + 1], du[3 * j + 2]);
  }
#pragma unroll
  for (int o = 1; o < kNL; o <<= 1)
#pragma unroll
    for (int k = 0; k < 18; ++k) h[k] += __shfl_xor_sync(gm, h[k], o);
  if (q == 0)
#pragma unroll
    for (int k = 0; k < 18; ++k) hq[18 * i + k] = h[k];
}

// D_HUGHES_WINGET (HUGHES_WINGET.F90:84-165): DG = DL A^-1 - L A^-1 (DL/2)
// A^-1, A = I + L/2; the symmetric part with engineering shear.
__device__ __forceinline__ void d_hughes_winget(const double L[3][3], const double DL[3][3], double de[6],
                                                bool exact) {
  double A[3][3], Ai[3][3], DA[3][3], nAi[3][3], t[3][3], ida[3][3], t1[3][3], t2[3][3], E[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      A[i][j] = (i == j ? 1.0 : 0.0) + 0.5 * L[i][j];
      DA[i][j] = 0.5 * DL[i][j];
    }
  inv3(A, Ai, exact);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) nAi[i][j] = -Ai[i][j];
  mm3(nAi, DA, t);
  mm3(t, Ai, ida);
  mm3(DL, Ai, t1);
  mm3(L, ida, t2);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) E[i][j] = 0.5 * ((t1[i][j] + t2[i][j]) + (t1[j][i] + t2[j][i]));
  t2v(E, de);
  de[3] = 2.0 * de[3]; de[4] = 2.0 * de[4]; de[5] = 2.0 * de[5];
}

// ESTIMATE_MODULI with NSNI_FLAG set (no clamp to half the elastic moduli),
// capped at the elastic moduli
__device__ __forceinline__ void estimate_moduli_nsni(const double sinc[6], const double einc[6], double& shear,
                                                     double& bulk) {
  const double sk = sinc[0] + sinc[1] + sinc[2], ek = einc[0] + einc[1] + einc[2];
  const double sd[6] = {sinc[0] - sk / 3.0, sinc[1] - sk / 3.0, sinc[2] - sk / 3.0, sinc[3], sinc[4], sinc[5]};
  const double ss[6] = {-sk / 3.0, -sk / 3.0, -sk / 3.0, 0.0, 0.0, 0.0};
  const double ed[6] = {einc[0] - ek / 3.0, einc[1] - ek / 3.0, einc[2] - ek / 3.0, einc[3], einc[4], einc[5]};
  const double es[6] = {-ek / 3.0, -ek / 3.0, -ek / 3.0, 0.0, 0.0, 0.0};
  const double nsd = tensor_norm(sd), nss = tensor_norm(ss);
  const double ned = tensor_norm_strain(ed), nes = tensor_norm_strain(es);
  if (ned > 1.0e-8 && nsd > 1.0e-8) shear = fmin(nsd / ned / 2.0, shear);
  if (nes > 1.0e-8 && nss > 1.0e-8) bulk = fmin(nss / nes / 3.0, bulk);
}

template <typename WV>
__global__ void __launch_bounds__(128) k_nsni_stress(NsniStepArgs a) {
  __shared__ double red[4];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double work = 0.0;
  if (i < a.n) {
    double g[18];
    load_fg(a.fg, i, sizeof(WV) == 4, g);  // the mixed step stores F - I and G0 as floats
    double F[3][3], G0[3][3], IF[3][3], L[3][3], R[3][3], dstr[6], D[6];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        F[k][l] = g[3 * k + l];
        G0[k][l] = g[9 + 3 * k + l];
        IF[k][l] = (k == l) ? 1.0 : 0.0;
        R[k][l] = (k == l) ? 1.0 : 0.0;
        L[k][l] = 0.0;
      }
    double det = 1.0;
    double srot[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) srot[k] = a.stress_old[6 * i + k];
    if (a.finite_strain) {
      det = det_abs(F);
      inv3(F, IF, a.inv3_exact != 0);
      mm3(G0, IF, L);
      hughes_winget(L, R, dstr, D, a.inv3_exact != 0);
      rotate_tensor(R, srot);
    } else {
      dstr[0] = G0[0][0]; dstr[1] = G0[1][1]; dstr[2] = G0[2][2];
      dstr[3] = G0[2][1] + G0[1][2]; dstr[4] = G0[2][0] + G0[0][2]; dstr[5] = G0[1][0] + G0[0][1];
    }
    const MatEntry& me = a.mats[a.matidx[i]];
    double gs = me.E / (2.0 * (1.0 + me.nu)), ks = me.E / (3.0 * (1.0 - 2.0 * me.nu));
    {
      double dso[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) dso[k] = a.stress_new[6 * i + k] - srot[k];
      estimate_moduli_nsni(dso, dstr, gs, ks);
    }
    const double lam_s = ks - 2.0 * gs / 3.0, l2m_s = ks + 4.0 * gs / 3.0;
    const double vol = a.vol[i];
    const double* hq = a.hq + 18 * i;
    double* sg = a.sgrad + 18 * i;
    double Wm[3][3][3];  // [a][k][m]
    unsigned st = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const double wd = a.sml[6 * i + 2 * ax] + a.sml[6 * i + 2 * ax + 1];
      const double fac = wd * wd / 12.0;
      double Ha[3][3];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m) Ha[k][m] = hq[6 * k + dd_index(m, ax)];
      double de[6], sa[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) sa[k] = sg[6 * ax + k];
      if (a.finite_strain) {
        double La[3][3];
        mm3(Ha, IF, La);
        d_hughes_winget(L, La, de, a.inv3_exact != 0);
        rotate_tensor(R, sa);
      } else {
        de[0] = Ha[0][0]; de[1] = Ha[1][1]; de[2] = Ha[2][2];
        de[3] = Ha[2][1] + Ha[1][2]; de[4] = Ha[2][0] + Ha[0][2]; de[5] = Ha[1][0] + Ha[0][1];
      }
      double ds[6];
      ds[0] = l2m_s * de[0] + lam_s * de[1] + lam_s * de[2];
      ds[1] = lam_s * de[0] + l2m_s * de[1] + lam_s * de[2];
      ds[2] = lam_s * de[0] + lam_s * de[1] + l2m_s * de[2];
      ds[3] = gs * de[3];
      ds[4] = gs * de[4];
      ds[5] = gs * de[5];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        sa[k] += ds[k];
        work += 0.5 * fac * de[k] * (2.0 * sa[k] - ds[k]) * vol * det;
        sg[6 * ax + k] = sa[k];
        if (!isfinite(sa[k])) st |= MEGA_ST_NONFINITE;
      }
      double S[3][3];
      v2t(sa, S);
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m)
          Wm[ax][k][m] = fac * vol * det * (S[k][0] * IF[m][0] + S[k][1] * IF[m][1] + S[k][2] * IF[m][2]);
    }
    // the weights folded onto the six symmetric second derivatives
    WV* w = reinterpret_cast<WV*>(a.w) + w_stride<WV>() * i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      w[6 * k + 0] = (WV)Wm[0][k][0];
      w[6 * k + 1] = (WV)Wm[1][k][1];
      w[6 * k + 2] = (WV)Wm[2][k][2];
      w[6 * k + 3] = (WV)(Wm[1][k][0] + Wm[0][k][1]);  // XY
      w[6 * k + 4] = (WV)(Wm[2][k][1] + Wm[1][k][2]);  // YZ
      w[6 * k + 5] = (WV)(Wm[2][k][0] + Wm[0][k][2]);  // XZ
    }
    if (st) atomicOr(a.status, st);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) work += __shfl_xor_sync(0xffffffffu, work, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = work;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double t = red[0] + red[1] + red[2] + red[3];
    if (t != 0.0) atomicAdd(&a.acc->int_work[blockIdx.x % kSlots], t);
  }
}

// fstab[3 J + k] = sum over the rows i holding J of sum_q W_i(k, q) S_q(i, J);
// V = the arithmetic and storage type of S and W (double or float)
template <typename V>
__global__ void __launch_bounds__(256) k_nsni_force(int32_t n, const int64_t* __restrict__ colptr,
                                                    const int32_t* __restrict__ trow, NsniArr<V> st,
                                                    const V* __restrict__ w, double* __restrict__ fstab) {
  const int64_t J = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kNL;
  const int q = threadIdx.x & (kNL - 1);
  const unsigned gm = 0xFFu << (threadIdx.x & 24);
  if (J >= n) return;
  V f0 = V(0), f1 = V(0), f2 = V(0);
  // the row's 18 weights as 16-byte loads
  auto load_w = [&](int64_t e, V* wi) {
    if constexpr (sizeof(V) == 4) {
      const float4* src = reinterpret_cast<const float4*>(w + 20 * (int64_t)trow[e]);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const float4 x = src[k];
        wi[4 * k] = x.x; wi[4 * k + 1] = x.y; wi[4 * k + 2] = x.z; wi[4 * k + 3] = x.w;
      }
    } else {
      const double2* src = reinterpret_cast<const double2*>(w + 18 * (int64_t)trow[e]);
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const double2 x = src[k];
        wi[2 * k] = x.x; wi[2 * k + 1] = x.y;
      }
    }
  };
  auto add = [&](int64_t e, const V* wi) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const V sv = st.v[c][e];
      f0 += wi[c] * sv;
      f1 += wi[6 + c] * sv;
      f2 += wi[12 + c] * sv;
    }
  };
  // two entries per pass, both rows requested before either is summed
  int64_t e = colptr[J] + q;
  const int64_t ee = colptr[J + 1];
  for (; e + kNL < ee; e += 2 * kNL) {
    V wa[w_stride<V>()], wb[w_stride<V>()];
    load_w(e, wa);
    load_w(e + kNL, wb);
    add(e, wa);
    add(e + kNL, wb);
  }
  if (e < ee) {
    V wa[w_stride<V>()];
    load_w(e, wa);
    add(e, wa);
  }
#pragma unroll
  for (int o = 1; o < kNL; o <<= 1) {
    f0 += __shfl_xor_sync(gm, f0, o);
    f1 += __shfl_xor_sync(gm, f1, o);
    f2 += __shfl_xor_sync(gm, f2, o);
  }
  if (q == 0) {
    fstab[3 * J] = (double)f0;
    fstab[3 * J + 1] = (double)f1;
    fstab[3 * J + 2] = (double)f2;
  }
}

// dst[6 e + q] = float S_q at list position pos[e] (the record order of the
// tiled gathers; list order without pos)
__global__ void k_nsni_records(int64_t m, const int64_t* __restrict__ pos, NsniS src, float* __restrict__ dst) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m) return;
  const int64_t p = pos ? pos[e] : e;
  float v[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) v[c] = (float)src.v[c][p];
  float2* o = reinterpret_cast<float2*>(dst + 6 * e);
  o[0] = make_float2(v[0], v[1]);
  o[1] = make_float2(v[2], v[3]);
  o[2] = make_float2(v[4], v[5]);
}

// dst[6 i + q] = sum over row i of the float-rounded S_q, in double (so that
// the split sum of the tiled row gather is exact in exact arithmetic)
__global__ void k_nsni_rowsum(int32_t n, const int64_t* __restrict__ rowptr, NsniS src, double* __restrict__ dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
#pragma unroll
    for (int c = 0; c < 6; ++c) t[c] += (double)(float)src.v[c][p];
#pragma unroll
  for (int c = 0; c < 6; ++c) dst[6 * i + c] = t[c];
}

}  // namespace

int nsni_combine(cudaStream_t s, int32_t n, int axis, const int64_t* rowptr, const double* sml, const double* gp[3],
                 const double* gm[3], const NsniS& out) {
  const unsigned grid = (unsigned)(((int64_t)n * 32 + 255) / 256);
  k_nsni_combine<<<grid, 256, 0, s>>>(n, axis, rowptr, sml, gp[0], gp[1], gp[2], gm[0], gm[1], gm[2], out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int nsni_step(cudaStream_t s, const NsniStepArgs& a, const DevCSR& csr, const NsniS& rows, const NsniS& cols,
              bool mixed, const double* du, int stage) {
  const unsigned gg = (unsigned)(((int64_t)a.n * kNL + 255) / 256);
  const unsigned gn = (unsigned)((a.n + 127) / 128);
  if (mixed && stage != 1) return MEGA_ERR_UNSUPPORTED;  // the tiled gathers carry those terms
  if (stage == 0) {
    k_nsni_h<double><<<gg, 256, 0, s>>>(a.n, csr.rowptr, csr.col, rows, du, a.hq);
  } else if (stage == 1) {
    if (mixed) k_nsni_stress<float><<<gn, 128, 0, s>>>(a);
    else k_nsni_stress<double><<<gn, 128, 0, s>>>(a);
  } else {
    k_nsni_force<double><<<gg, 256, 0, s>>>(a.n, csr.colptr, csr.trow, cols, (const double*)a.w, a.fstab);
  }
  MEGA_CHECK_LAUNCH();
  return 0;
}

int nsni_records(cudaStream_t s, int64_t m, const int64_t* pos, const NsniS& src, float* dst) {
  if (m <= 0) return 0;
  k_nsni_records<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, pos, src, dst);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int nsni_rowsum(cudaStream_t s, int32_t n, const int64_t* rowptr, const NsniS& src, double* dst) {
  if (n <= 0) return 0;
  k_nsni_rowsum<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rowptr, src, dst);
  MEGA_CHECK_LAUNCH();
  return 0;
}

}  // namespace mega
