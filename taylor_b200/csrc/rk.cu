// rk.cu -- reproducing-kernel shape functions, one warp per node, FP64.
//
// Restates RK1 (RK.f90:16-453) for DEG = 1: per neighbour the linear basis
// H = (1, X-X_J), the box cubic B-spline kernel phi = w(|dx|/a)w(|dy|/a)
// w(|dz|/a) (or the spherical one with SHSUP) with its gradient, the
// singular-kernel modification for EBC neighbours (RK.f90:217-228); the
// moment matrix M and its x/y/z derivatives (RK.f90:231-242), the
// quasi-linear term (RK.f90:251-303), the cofactor inverse (M44INV), the
// correction vectors b = e1 M^-1 and b_,x = -e1 M^-1 M_,x M^-1
// (RK.f90:311-342), and finally phi_J = (b.H~)phi, grad phi_J =
// (b_,x.H~ + b.H_,x)phi + (b.H~)phi_,x (RK.f90:346-405).
// Three kernels, so that none carries the registers of the others (one
// kernel holding the 41 sums, the inverse and the correction vectors at once
// ran at 12 resident warps per SM):
//   k_rk_moments  a group of kLPN lanes per node strides the neighbour list
//                 and accumulates psum and the 4 symmetric 4x4 matrices M,
//                 M_,x, M_,y, M_,z (41 sums), reduced by a butterfly in the
//                 group and stored per node;
//   k_rk_solve    thread per node: the basis-derivative part of M_,d, the
//                 QL term, the inverse and the correction vectors (16 values
//                 per node);
//   k_rk_values   a group per node again: phi_J and grad phi_J per entry.
// kLPN = 4 lanes per node: the ~60 neighbours give every lane ~15 entries,
// and the butterfly over the 41 sums takes two rounds.
#include "mega_internal.cuh"

namespace mega {
namespace {

struct EntryK {
  double H[4];
  double phi, px, py, pz;
};

// RK.f90:123-230 for one neighbour
__device__ __forceinline__ void rk_entry(const double xi[3], const double xj[3], const double aj[3], bool ebc_j,
                                         int shsup, EntryK& e) {
  const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
  e.H[0] = 1.0; e.H[1] = dx; e.H[2] = dy; e.H[3] = dz;
  const double nx = dx / aj[0], ny = dy / aj[1], nz = dz / aj[2];
  if (shsup) {
    const double dia = sqrt(nx * nx + ny * ny + nz * nz);
    double k, kx;
    bspline3(dia, k, kx);
    double drdx = 0.0, drdy = 0.0, drdz = 0.0;
    if (!(dia <= 1.0e-13)) {
      drdx = dx / (aj[0] * aj[0]) / dia;
      drdy = dy / (aj[1] * aj[1]) / dia;
      drdz = dz / (aj[2] * aj[2]) / dia;
    }
    e.phi = k; e.px = kx * drdx; e.py = kx * drdy; e.pz = kx * drdz;
  } else {
    double kx, kxx, ky, kyy, kz, kzz;
    bspline3(fabs(nx), kx, kxx);
    bspline3(fabs(ny), ky, kyy);
    bspline3(fabs(nz), kz, kzz);
    double phi = kx * ky * kz;
    // RK.f90:183-205: every axis divides by GWIN(1,II) (kept as written)
    const double drdx = (nx == 0.0) ? 0.0 : (nx >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
    const double drdy = (ny == 0.0) ? 0.0 : (ny >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
    const double drdz = (nz == 0.0) ? 0.0 : (nz >= 0.0 ? 1.0 / aj[0] : -1.0 / aj[0]);
    double px = kxx * ky * kz * drdx;
    double py = kx * kyy * kz * drdy;
    double pz = kx * ky * kzz * drdz;
    if (ebc_j) {
      const double wm = 1.0 / (sqrt(nx * nx + ny * ny + nz * nz) + (double)1.0e-15f);
      const double w3 = phi * wm * wm * wm;
      px = px * wm - w3 * nx / aj[0];
      py = py * wm - w3 * ny / aj[1];
      pz = pz * wm - w3 * nz / aj[2];
      phi = phi * wm;
    }
    e.phi = phi; e.px = px; e.py = py; e.pz = pz;
  }
}

// packed symmetric 4x4: (00,01,02,03,11,12,13,22,23,33)
__device__ __forceinline__ int sidx(int j, int k) {
  if (j > k) { int t = j; j = k; k = t; }
  return j == 0 ? k : (j == 1 ? 3 + k : (j == 2 ? 5 + k : 9));
}

constexpr int kLPN = 4;  // lanes per node
constexpr int kMom = 41;  // psum, M, M_,x, M_,y, M_,z (10 packed values each)

// the node's position, or a face point of its smoothing cell, x +- SM_LEN
// (face 0..5: +X, -X, +Y, -Y, +Z, -Z)
__device__ __forceinline__ void node_point(int64_t i, const double* __restrict__ coo,
                                           const double* __restrict__ sml, int face, double xi[3]) {
  xi[0] = coo[3 * i]; xi[1] = coo[3 * i + 1]; xi[2] = coo[3 * i + 2];
  if (face >= 0) {
    const int ax = face >> 1;
    xi[ax] = (face & 1) ? xi[ax] - sml[6 * i + face] : xi[ax] + sml[6 * i + face];
  }
}

__global__ void __launch_bounds__(128) k_rk_moments(int32_t n, const double* __restrict__ coo,
                                                    const double* __restrict__ win,
                                                    const int32_t* __restrict__ ebc_nodes,
                                                    const int64_t* __restrict__ rowptr,
                                                    const int32_t* __restrict__ col, int shsup,
                                                    const double* __restrict__ sml, int face,
                                                    double* __restrict__ mom) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kLPN;
  const int lane = threadIdx.x & (kLPN - 1);
  const unsigned gm = ((1u << kLPN) - 1u) << (threadIdx.x & (32 - kLPN));
  if (i >= n) return;  // whole groups leave together
  double xi[3];
  node_point(i, coo, sml, face, xi);
  const int64_t p0 = rowptr[i], p1 = rowptr[i + 1];
  double M[10], Mx[10], My[10], Mz[10], psum = 0.0;
#pragma unroll
  for (int k = 0; k < 10; ++k) { M[k] = 0.0; Mx[k] = 0.0; My[k] = 0.0; Mz[k] = 0.0; }
  for (int64_t p = p0 + lane; p < p1; p += kLPN) {
    const int64_t j = col[p];
    const double xj[3] = {coo[3 * j], coo[3 * j + 1], coo[3 * j + 2]};
    const double aj[3] = {win[3 * j], win[3 * j + 1], win[3 * j + 2]};
    EntryK e;
    rk_entry(xi, xj, aj, ebc_nodes && ebc_nodes[j], shsup, e);
    psum += e.phi;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = a; b < 4; ++b) {
        const int q = sidx(a, b);
        const double hh = e.H[a] * e.H[b];
        M[q] += hh * e.phi;
        Mx[q] += hh * e.px;
        My[q] += hh * e.py;
        Mz[q] += hh * e.pz;
      }
  }
#pragma unroll
  for (int o = kLPN / 2; o > 0; o >>= 1) {
    psum += __shfl_xor_sync(gm, psum, o);
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      M[k] += __shfl_xor_sync(gm, M[k], o);
      Mx[k] += __shfl_xor_sync(gm, Mx[k], o);
      My[k] += __shfl_xor_sync(gm, My[k], o);
      Mz[k] += __shfl_xor_sync(gm, Mz[k], o);
    }
  }
  // every lane holds the sums; lane l stores values l, l + kLPN, ...
  double* o = mom + kMom * i;
#pragma unroll
  for (int v = 0; v < kMom; ++v) {
    if ((v & (kLPN - 1)) != lane) continue;
    o[v] = v == 0 ? psum : (v <= 10 ? M[v - 1] : (v <= 20 ? Mx[v - 11] : (v <= 30 ? My[v - 21] : Mz[v - 31])));
  }
}

// thread per node: bv[16 i ..] = b, b_,x, b_,y, b_,z
__global__ void __launch_bounds__(128) k_rk_solve(int32_t n, const double* __restrict__ coo, int ql, double ql_coef,
                                                  double ql_len, const double* __restrict__ sml, int face,
                                                  const double* __restrict__ mom, double* __restrict__ bv,
                                                  unsigned* __restrict__ status) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* m = mom + kMom * i;
  const double psum = m[0];
  double M[10], Mx[10], My[10], Mz[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) { M[k] = m[1 + k]; Mx[k] = m[11 + k]; My[k] = m[21 + k]; Mz[k] = m[31 + k]; }
  // the basis-derivative part of M_,d: sum (H_,d H^T + H H_,d^T) phi with
  // H_,d the unit vector e_d adds to entry (a, b) delta(a,d) sum H_b phi +
  // delta(b,d) sum H_a phi, the first moments M(0, b) and M(0, a) (H_0 = 1)
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a; b < 4; ++b) {
      const int q = sidx(a, b);
      Mx[q] += (a == 1 ? M[sidx(0, b)] : 0.0) + (b == 1 ? M[sidx(0, a)] : 0.0);
      My[q] += (a == 2 ? M[sidx(0, b)] : 0.0) + (b == 2 ? M[sidx(0, a)] : 0.0);
      Mz[q] += (a == 3 ? M[sidx(0, b)] : 0.0) + (b == 3 ? M[sidx(0, a)] : 0.0);
    }
  double Mf[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Mf[a][b] = M[sidx(a, b)];
  if (ql) {
    // RK.f90:253-301: the six points X +- QL_LEN e_d, differences evaluated
    // in floating point as the reference does
    double xi[3];
    node_point(i, coo, sml, face, xi);
    double d[6][3];
#pragma unroll
    for (int k = 0; k < 6; ++k) { d[k][0] = 0.0; d[k][1] = 0.0; d[k][2] = 0.0; }
    d[0][0] = xi[0] - (xi[0] + ql_len); d[1][0] = xi[0] - (xi[0] - ql_len);
    d[2][1] = xi[1] - (xi[1] + ql_len); d[3][1] = xi[1] - (xi[1] - ql_len);
    d[4][2] = xi[2] - (xi[2] + ql_len); d[5][2] = xi[2] - (xi[2] - ql_len);
    double Ms[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Ms[a][b] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double H[4] = {1.0, d[k][0], d[k][1], d[k][2]};
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) Ms[a][b] += H[a] * H[b];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Mf[a][b] = Mf[a][b] + Ms[a][b] * psum * ql_coef;
  }
  double Mi[4][4];
  const double det = m44inv(Mf, Mi);
  if (!isfinite(det) || det == 0.0) atomicOr(status, (unsigned)MEGA_ST_SINGULAR_MOMENT);
  double B[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) B[k] = Mi[0][k];
  double* o = bv + 16 * i;
#pragma unroll
  for (int k = 0; k < 4; ++k) o[k] = B[k];
  // b_,d = -(b M_,d) M^-1
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    const double* Md = dd == 0 ? Mx : (dd == 1 ? My : Mz);
    double t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double sacc = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) sacc += B[q] * Md[sidx(q, k)];
      t[k] = -sacc;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o[4 + 4 * dd + k] = t[0] * Mi[0][k] + t[1] * Mi[1][k] + t[2] * Mi[2][k] + t[3] * Mi[3][k];
  }
}

__global__ void __launch_bounds__(128) k_rk_values(int32_t n, const double* __restrict__ coo,
                                                   const double* __restrict__ win,
                                                   const int32_t* __restrict__ ebc_nodes,
                                                   const int64_t* __restrict__ rowptr,
                                                   const int32_t* __restrict__ col, int ql, double ql_coef,
                                                   double ql_len, int shsup, const double* __restrict__ sml,
                                                   int face, const double* __restrict__ bv,
                                                   double* __restrict__ shp, double* __restrict__ gx,
                                                   double* __restrict__ gy, double* __restrict__ gz,
                                                   float4* __restrict__ pk, const uint16_t* __restrict__ lidx) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / kLPN;
  const int lane = threadIdx.x & (kLPN - 1);
  if (i >= n) return;
  double xi[3];
  node_point(i, coo, sml, face, xi);
  double Hs[4] = {0.0, 0.0, 0.0, 0.0};
  if (ql) {  // the QL shift of the basis, RK.f90:357-377
    Hs[0] = 6.0;
    Hs[1] = (xi[0] - (xi[0] + ql_len)) + (xi[0] - (xi[0] - ql_len));
    Hs[2] = (xi[1] - (xi[1] + ql_len)) + (xi[1] - (xi[1] - ql_len));
    Hs[3] = (xi[2] - (xi[2] + ql_len)) + (xi[2] - (xi[2] - ql_len));
  }
  const double* b = bv + 16 * i;
  double B[4], BX[4], BY[4], BZ[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) { B[k] = b[k]; BX[k] = b[4 + k]; BY[k] = b[8 + k]; BZ[k] = b[12 + k]; }
  const int64_t p0 = rowptr[i], p1 = rowptr[i + 1];
  for (int64_t p = p0 + lane; p < p1; p += kLPN) {
    const int64_t j = col[p];
    const double xj[3] = {coo[3 * j], coo[3 * j + 1], coo[3 * j + 2]};
    const double aj[3] = {win[3 * j], win[3 * j + 1], win[3 * j + 2]};
    EntryK e;
    rk_entry(xi, xj, aj, ebc_nodes && ebc_nodes[j], shsup, e);
    double H[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) H[k] = ql ? e.H[k] + Hs[k] * ql_coef : e.H[k];
    const double C = B[0] * H[0] + B[1] * H[1] + B[2] * H[2] + B[3] * H[3];
    const double CX = BX[0] * H[0] + BX[1] * H[1] + BX[2] * H[2] + BX[3] * H[3] + B[1];
    const double CY = BY[0] * H[0] + BY[1] * H[1] + BY[2] * H[2] + BY[3] * H[3] + B[2];
    const double CZ = BZ[0] * H[0] + BZ[1] * H[1] + BZ[2] * H[2] + BZ[3] * H[3] + B[3];
    if (shp) shp[p] = C * e.phi;
    const double vx = CX * e.phi + C * e.px, vy = CY * e.phi + C * e.py, vz = CZ * e.phi + C * e.pz;
    if (pk) {  // the mixed-precision record (gradient in float, tile rank) instead of the doubles
      pk[p] = make_float4((float)vx, (float)vy, (float)vz, __int_as_float((int)lidx[p]));
    } else {
      gx[p] = vx;
      gy[p] = vy;
      gz[p] = vz;
    }
  }
}

// the three kernels in order on stream s, with their per-node scratch
int rk_run(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
           const int32_t* ebc_nodes, const DevCSR& csr, const double* sml, int face, double* shp, double* gx,
           double* gy, double* gz, float4* pk, const uint16_t* lidx, unsigned* status) {
  if (p.rk_degree != 1 || p.rk_cont != 3) return MEGA_ERR_UNSUPPORTED;
  DevPool scratch(s);
  double *mom = nullptr, *bv = nullptr;
  MEGA_ALLOC(scratch, mom, (int64_t)kMom * n);
  MEGA_ALLOC(scratch, bv, 16 * (int64_t)n);
  const int block = 128;
  const unsigned gg = (unsigned)(((int64_t)n * kLPN + block - 1) / block);
  const unsigned gn = (unsigned)((n + block - 1) / block);
  k_rk_moments<<<gg, block, 0, s>>>(n, coo, win, ebc_nodes, csr.rowptr, csr.col, p.shsup, sml, face, mom);
  MEGA_CHECK_LAUNCH();
  k_rk_solve<<<gn, block, 0, s>>>(n, coo, p.ql, p.ql_coef, p.ql_len, sml, face, mom, bv, status);
  MEGA_CHECK_LAUNCH();
  k_rk_values<<<gg, block, 0, s>>>(n, coo, win, ebc_nodes, csr.rowptr, csr.col, p.ql, p.ql_coef, p.ql_len, p.shsup,
                                   sml, face, bv, shp, gx, gy, gz, pk, lidx);
  MEGA_CHECK_LAUNCH();
  return 0;
}

}  // namespace

int rk_shapes(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
              const int32_t* ebc_nodes, const DevCSR& csr, double* shp, double* gx, double* gy, double* gz,
              unsigned* status) {
  return rk_run(s, p, n, coo, win, ebc_nodes, csr, nullptr, -1, shp, gx, gy, gz, nullptr, nullptr, status);
}

int rk_shapes_packed(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
                     const int32_t* ebc_nodes, const DevCSR& csr, const uint16_t* lidx, double* shp, float4* pk,
                     unsigned* status) {
  return rk_run(s, p, n, coo, win, ebc_nodes, csr, nullptr, -1, shp, nullptr, nullptr, nullptr, pk, lidx, status);
}

int rk_grad_at_face(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
                    const int32_t* ebc_nodes, const DevCSR& csr, const double* sml, int face, double* gx, double* gy,
                    double* gz, unsigned* status) {
  return rk_run(s, p, n, coo, win, ebc_nodes, csr, sml, face, nullptr, gx, gy, gz, nullptr, nullptr, status);
}

}  // namespace mega
