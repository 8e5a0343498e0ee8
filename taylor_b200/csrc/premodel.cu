// premodel.cu -- the mesh pre-processing of PRE_MODEL.F90:248-268 and
// PRE_CONTROL.F90:803-871 on the device, for meshes of hexahedral and
// tetrahedral blocks (a tetrahedron is an 8-node connectivity whose last
// nodes repeat, PRE_MODEL.F90:233-240):
//   raw nodal windows  ADIAL = the largest per-axis extent of the hexes
//                      holding the node (GET_ADIAL, PRE_MODEL_ADIAL.F90:64-153)
//   nodal volumes      the sum of 1/8 of every such hex's volume, the hex
//                      split into three tetrahedral wedges about the 1-7
//                      diagonal (GET_VOLUMES / GET_VOL2, PRE_MODEL_VOLUMES.F90:
//                      70-117, PRE_MODEL_VOL2.F90:36-52), and 1/4 of every
//                      tetrahedron's volume (GET_VOL1, PRE_MODEL_VOL1.f90:
//                      37-45); a tetrahedron's window is the extent of its
//                      first four nodes (PRE_MODEL_ADIAL.F90:112-150)
//   smoothing cells    SM_LEN, second moments, DIST_MAX
//                      (GET_SMOOTHING_LENGTHS, PRE_MODEL_SMOOTHING_LENGTHS.F90:
//                      49-99)
//   windows            ADIAL scaled by the per-node normalised window
//                      (PRE_CONTROL.F90:870-872), and the smallest raw
//                      window (the automatic QL_LEN before its reduction,
//                      PRE_CONTROL.F90:803-815).
// The element-to-node sums run over a node-to-element list sorted by element,
// so each node adds its elements' volumes in the reference's element order
// (bit for bit; the element volumes use no fused multiply-adds).
#include "mega_internal.cuh"

namespace mega {
namespace {

inline unsigned grid_of(int64_t work, int block) { return (unsigned)((work + block - 1) / block); }

// DETERMINANT.F90:18-35 on columns c0, c1, c2, rounded as written (no FMA)
__device__ __forceinline__ double det_cols(const double c0[3], const double c1[3], const double c2[3]) {
  // A(r, c): row r, column c; A(1,1) = c0[0], A(2,2) = c1[1], ...
  const double t1 = __dsub_rn(__dmul_rn(c1[1], c2[2]), __dmul_rn(c1[2], c2[1]));
  const double t2 = __dsub_rn(__dmul_rn(c0[2], c2[1]), __dmul_rn(c0[1], c2[2]));
  const double t3 = __dsub_rn(__dmul_rn(c0[1], c1[2]), __dmul_rn(c0[2], c1[1]));
  return fabs(__dadd_rn(__dadd_rn(__dmul_rn(c0[0], t1), __dmul_rn(c1[0], t2)), __dmul_rn(c2[0], t3)));
}

// nodes an element of type t (1 tetrahedron, 2 hexahedron) contributes to
__device__ __forceinline__ int elem_nodes(const int8_t* eltype, int64_t e) {
  return (eltype && eltype[e] == 1) ? 4 : 8;
}

// per element: the per-axis extents and its share of volume per node
// (0.125 DVOL for a hex, 0.25 DVOL for a tetrahedron)
__global__ void k_elem(int32_t n, int32_t ne, const double* __restrict__ coo, const int32_t* __restrict__ conn,
                       const int8_t* __restrict__ eltype, double* __restrict__ ext, double* __restrict__ dvol,
                       unsigned* __restrict__ status) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int nk = elem_nodes(eltype, e);
  double x[8][3];
  for (int k = 0; k < nk; ++k) {
    const int32_t id = conn[8 * e + k] - 1;  // IDELM is 1-based
    if (id < 0 || id >= n) {
      atomicOr(status, (unsigned)MEGA_ST_BAD_MESH);
      ext[3 * e] = ext[3 * e + 1] = ext[3 * e + 2] = 0.0;
      dvol[e] = 0.0;
      return;
    }
    x[k][0] = coo[3 * (int64_t)id]; x[k][1] = coo[3 * (int64_t)id + 1]; x[k][2] = coo[3 * (int64_t)id + 2];
  }
  // max over node pairs of |x_K - x_J| is the range of the nk values
  for (int a = 0; a < 3; ++a) {
    double lo = x[0][a], hi = x[0][a];
    for (int k = 1; k < nk; ++k) { lo = fmin(lo, x[k][a]); hi = fmax(hi, x[k][a]); }
    ext[3 * e + a] = __dsub_rn(hi, lo);
  }
  if (nk == 4) {  // GET_VOL1: rows X4-X3, X1-X3, X2-X3 of A, DVOL = |det A| / 6
    double c[3][3];  // c[col][row]
    for (int a = 0; a < 3; ++a) {
      c[a][0] = __dsub_rn(x[3][a], x[2][a]);
      c[a][1] = __dsub_rn(x[0][a], x[2][a]);
      c[a][2] = __dsub_rn(x[1][a], x[2][a]);
    }
    dvol[e] = __dmul_rn(0.25, __ddiv_rn(det_cols(c[0], c[1], c[2]), 6.0));
    return;
  }
  // GET_VOL2: columns (X7-X1, X2-X1, X3-X6), (X7-X1, X5-X1, X6-X8), (X7-X1, X4-X1, X8-X3)
  double d71[3], d21[3], d36[3], d51[3], d68[3], d41[3], d83[3];
  for (int a = 0; a < 3; ++a) {
    d71[a] = __dsub_rn(x[6][a], x[0][a]);
    d21[a] = __dsub_rn(x[1][a], x[0][a]);
    d36[a] = __dsub_rn(x[2][a], x[5][a]);
    d51[a] = __dsub_rn(x[4][a], x[0][a]);
    d68[a] = __dsub_rn(x[5][a], x[7][a]);
    d41[a] = __dsub_rn(x[3][a], x[0][a]);
    d83[a] = __dsub_rn(x[7][a], x[2][a]);
  }
  const double ad = det_cols(d71, d21, d36), bd = det_cols(d71, d51, d68), cd = det_cols(d71, d41, d83);
  dvol[e] = __dmul_rn(0.125, __ddiv_rn(__dadd_rn(__dadd_rn(ad, bd), cd), 6.0));
}

__global__ void k_adj_count(int32_t n, int32_t ne, const int32_t* __restrict__ conn, const int8_t* __restrict__ eltype,
                            int32_t* __restrict__ cnt) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= 8 * (int64_t)ne) return;
  if ((t & 7) >= elem_nodes(eltype, t >> 3)) return;
  const int32_t id = conn[t] - 1;
  if (id >= 0 && id < n) atomicAdd(&cnt[id], 1);
}

__global__ void k_adj_fill(int32_t n, int32_t ne, const int32_t* __restrict__ conn, const int8_t* __restrict__ eltype,
                           const int64_t* __restrict__ off, int32_t* __restrict__ fill, int32_t* __restrict__ list) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= 8 * (int64_t)ne) return;
  if ((t & 7) >= elem_nodes(eltype, t >> 3)) return;
  const int32_t id = conn[t] - 1;
  if (id < 0 || id >= n) return;
  list[off[id] + atomicAdd(&fill[id], 1)] = (int32_t)(t >> 3);
}

// each node's hexes in element order (a node listed twice by one hex keeps
// both entries, as the reference adds twice)
__global__ void k_adj_sort(int32_t n, const int64_t* __restrict__ off, int32_t* __restrict__ list) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = off[i], b = off[i + 1];
  for (int64_t p = a + 1; p < b; ++p) {
    const int32_t v = list[p];
    int64_t q = p - 1;
    while (q >= a && list[q] > v) { list[q + 1] = list[q]; --q; }
    list[q + 1] = v;
  }
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_nonneg(double* addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

struct PreArgs {
  int32_t n;
  const int64_t* off;
  const int32_t* list;
  const double* ext;
  const double* dvol;
  const double* norm_win;  // per node, or null (1)
  double* win_raw;
  double* win;
  double* vol;
  double* sm_len;
  double* mom;
  double* red;  // [0..2] DIST_MAX (max), [3] the smallest raw window (min)
};

__global__ void __launch_bounds__(256) k_node_pre(PreArgs a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double dmx = 0.0, dmy = 0.0, dmz = 0.0, wmin = 1.0e300;
  if (i < a.n) {
    double w0 = 0.0, w1 = 0.0, w2 = 0.0, v = 0.0;  // ADIAL = 0, VOLUME = 0
    for (int64_t p = a.off[i]; p < a.off[i + 1]; ++p) {
      const int64_t e = a.list[p];
      if (a.ext[3 * e] > w0) w0 = a.ext[3 * e];
      if (a.ext[3 * e + 1] > w1) w1 = a.ext[3 * e + 1];
      if (a.ext[3 * e + 2] > w2) w2 = a.ext[3 * e + 2];
      v = __dadd_rn(v, a.dvol[e]);  // the element's share, 0.125 or 0.25 DVOL
    }
    a.win_raw[3 * i] = w0; a.win_raw[3 * i + 1] = w1; a.win_raw[3 * i + 2] = w2;
    a.vol[i] = v;
    const double s = a.norm_win ? a.norm_win[i] : 1.0;
    if (a.win) { a.win[3 * i] = w0 * s; a.win[3 * i + 1] = w1 * s; a.win[3 * i + 2] = w2 * s; }
    // PRE_MODEL_SMOOTHING_LENGTHS.F90:56-88 (THRD = 0.333333333333333d0)
    const double thrd = 0.333333333333333;
    const double d1 = w0 * 2.0, d2 = w1 * 2.0, d3 = w2 * 2.0;
    const double vw = d1 * d2 * d3;
    const double ratio = pow(v, thrd) / pow(vw, thrd);
    const double m1 = d1 * ratio, m2 = d2 * ratio, m3 = d3 * ratio;
    if (a.mom) { a.mom[3 * i] = m1 * m1 / 12.0; a.mom[3 * i + 1] = m2 * m2 / 12.0; a.mom[3 * i + 2] = m3 * m3 / 12.0; }
    const double s1 = d1 * ratio / 2.0, s2 = d2 * ratio / 2.0, s3 = d3 * ratio / 2.0;
    double* sl = a.sm_len + 6 * i;
    sl[0] = s1; sl[1] = s1; sl[2] = s2; sl[3] = s2; sl[4] = s3; sl[5] = s3;
    dmx = s1; dmy = s2; dmz = s3;
    wmin = fmin(w0, fmin(w1, w2));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dmx = fmax(dmx, __shfl_xor_sync(0xffffffffu, dmx, o));
    dmy = fmax(dmy, __shfl_xor_sync(0xffffffffu, dmy, o));
    dmz = fmax(dmz, __shfl_xor_sync(0xffffffffu, dmz, o));
    wmin = fmin(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(&a.red[0], dmx);
    atomic_max_nonneg(&a.red[1], dmy);
    atomic_max_nonneg(&a.red[2], dmz);
    atomic_min_nonneg(&a.red[3], wmin);
  }
}

}  // namespace
}  // namespace mega

using namespace mega;

extern "C" {

int mega_pre_model_hex(int32_t n, const double* coo, int32_t nelem, const int32_t* conn, const double* norm_win,
                       double* win_raw, double* win, double* vol, double* sm_len, double* mom, double* dist_max,
                       double* min_raw_window) {
  return mega_pre_model(n, coo, nelem, conn, nullptr, norm_win, win_raw, win, vol, sm_len, mom, dist_max,
                        min_raw_window);
}

int mega_pre_model(int32_t n, const double* coo, int32_t nelem, const int32_t* conn, const int32_t* eltype,
                   const double* norm_win, double* win_raw, double* win, double* vol, double* sm_len, double* mom,
                   double* dist_max, double* min_raw_window) {
  if (n <= 0 || nelem <= 0 || !coo || !conn || !win_raw || !vol || !sm_len || !dist_max) return MEGA_ERR_ARG;
  std::vector<int8_t> het;
  if (eltype) {
    het.resize(nelem);
    for (int32_t e = 0; e < nelem; ++e) {
      if (eltype[e] != 1 && eltype[e] != 2) return MEGA_ERR_ARG;  // 1 tetrahedron, 2 hexahedron
      het[e] = (int8_t)eltype[e];
    }
  }
  cudaStream_t s;
  MEGA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SG { cudaStream_t s; ~SG() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{s};
  DevPool pool(s);
  const int64_t n3 = 3 * (int64_t)n;
  double *dc, *dext, *dvol, *dnw = nullptr, *dwr, *dw = nullptr, *dv, *dsl, *dmom = nullptr, *dred;
  int32_t *dconn, *cnt, *fill, *list;
  int8_t* det = nullptr;
  int64_t* off;
  unsigned* st;
  MEGA_ALLOC(pool, dc, n3);
  MEGA_ALLOC(pool, dconn, 8 * (int64_t)nelem);
  MEGA_ALLOC(pool, dext, 3 * (int64_t)nelem);
  MEGA_ALLOC(pool, dvol, nelem);
  MEGA_ALLOC(pool, cnt, n);
  MEGA_ALLOC(pool, fill, n);
  MEGA_ALLOC(pool, off, (int64_t)n + 1);
  MEGA_ALLOC(pool, list, 8 * (int64_t)nelem);
  MEGA_ALLOC(pool, dwr, n3);
  MEGA_ALLOC(pool, dv, n);
  MEGA_ALLOC(pool, dsl, 6 * (int64_t)n);
  MEGA_ALLOC(pool, dred, 4);
  MEGA_ALLOC(pool, st, 1);
  if (win) MEGA_ALLOC(pool, dw, n3);
  if (mom) MEGA_ALLOC(pool, dmom, n3);
  if (eltype) {
    MEGA_ALLOC(pool, det, nelem);
    MEGA_TRY(cudaMemcpyAsync(det, het.data(), (size_t)nelem, cudaMemcpyHostToDevice, s));
  }
  if (norm_win) {
    MEGA_ALLOC(pool, dnw, n);
    MEGA_TRY(cudaMemcpyAsync(dnw, norm_win, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  }
  MEGA_TRY(cudaMemcpyAsync(dc, coo, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemcpyAsync(dconn, conn, sizeof(int32_t) * 8 * (size_t)nelem, cudaMemcpyHostToDevice, s));
  MEGA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * n, s));
  MEGA_TRY(cudaMemsetAsync(fill, 0, sizeof(int32_t) * n, s));
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  const double red0[4] = {0.0, 0.0, 0.0, 1.0e300};
  MEGA_TRY(cudaMemcpyAsync(dred, red0, sizeof(red0), cudaMemcpyHostToDevice, s));
  k_elem<<<grid_of(nelem, 256), 256, 0, s>>>(n, nelem, dc, dconn, det, dext, dvol, st);
  k_adj_count<<<grid_of(8 * (int64_t)nelem, 256), 256, 0, s>>>(n, nelem, dconn, det, cnt);
  MEGA_CHECK_LAUNCH();
  int r = scan_counts(s, cnt, off, n, pool);
  if (r) return r;
  k_adj_fill<<<grid_of(8 * (int64_t)nelem, 256), 256, 0, s>>>(n, nelem, dconn, det, off, fill, list);
  k_adj_sort<<<grid_of(n, 256), 256, 0, s>>>(n, off, list);
  MEGA_CHECK_LAUNCH();
  PreArgs a{};
  a.n = n; a.off = off; a.list = list; a.ext = dext; a.dvol = dvol; a.norm_win = dnw; a.win_raw = dwr; a.win = dw;
  a.vol = dv; a.sm_len = dsl; a.mom = dmom; a.red = dred;
  k_node_pre<<<grid_of(n, 256), 256, 0, s>>>(a);
  MEGA_CHECK_LAUNCH();
  double hred[4];
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(win_raw, dwr, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(vol, dv, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(sm_len, dsl, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  if (win) MEGA_TRY(cudaMemcpyAsync(win, dw, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  if (mom) MEGA_TRY(cudaMemcpyAsync(mom, dmom, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(hred, dred, sizeof(hred), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  dist_max[0] = hred[0]; dist_max[1] = hred[1]; dist_max[2] = hred[2];
  if (min_raw_window) *min_raw_window = hred[3];
  return (int)hst;
}

}  // extern "C"
