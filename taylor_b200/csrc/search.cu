// search.cu -- sort-by-cell neighbour search, bit-exact with BIN_SEARCH.
//
// Replaces GET_BINS / BIN_INODE / SOFT_SEARCH (BIN_SEARCH.F90:2-328) and
// the LINIT bin geometry of HANDELER.F90:187-250:
//   1. bounding box and bin size (block reductions; max/min are exact);
//   2. cell of each node, FLOOR((X-XMIN)/XBIN)+1 clamped (BIN_SEARCH.F90:28-41);
//   3. counting sort by cell: histogram, exclusive scan, scatter, then a
//      per-cell sort by node id so every cell lists its nodes in index order
//      like NODELIST_IN_BIN does (BIN_SEARCH.F90:45-54);
//   4. warp-per-node candidate filter over the 27 cells in BIN_INODE order
//      (IX outer, IZ inner, BIN_SEARCH.F90:105-127), ballot + popc compaction
//      so the output rows keep the reference's order exactly;
//   5. one filter pass into per-node candidate slots, scan, compaction
//      (or, where the slots do not fit in memory and in the allocation-free
//      entry point, a count pass -> scan -> fill pass).
// Every floating-point operation of the test uses __d*_rn intrinsics, so no
// FMA contraction can change a comparison: the lists are bit-exact.
#include <algorithm>
#include <mutex>
#include <climits>
#include "mega_internal.cuh"

namespace mega {

namespace {

__device__ __forceinline__ void atomic_max_int(int32_t* a, int32_t v) { atomicMax(a, v); }

// ---- 1. bounding box / bin size partials: 9 values per block:
// [xbin, ybin, zbin, xmax, ymax, zmax, -xmin, -ymin, -zmin] as maxima
__global__ void k_bbox_partial(int32_t n, const double* __restrict__ coo, const double* __restrict__ win,
                               double d0, double d1, double d2, double* __restrict__ part) {
  __shared__ double sm[9][32];
  double v[9];
  v[0] = 0.0; v[1] = 0.0; v[2] = 0.0;
  v[3] = -INFINITY; v[4] = -INFINITY; v[5] = -INFINITY;
  v[6] = -INFINITY; v[7] = -INFINITY; v[8] = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double w0 = win[3 * i], w1 = win[3 * i + 1], w2 = win[3 * i + 2];
    v[0] = fmax(v[0], fmax(w0, __dadd_rn(w0, d0)));
    v[1] = fmax(v[1], fmax(w1, __dadd_rn(w1, d1)));
    v[2] = fmax(v[2], fmax(w2, __dadd_rn(w2, d2)));
    const double x0 = coo[3 * i], x1 = coo[3 * i + 1], x2 = coo[3 * i + 2];
    v[3] = fmax(v[3], x0); v[4] = fmax(v[4], x1); v[5] = fmax(v[5], x2);
    v[6] = fmax(v[6], -x0); v[7] = fmax(v[7], -x1); v[8] = fmax(v[8], -x2);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 9; ++k) sm[k][wid] = v[k];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double a = (lane < nw) ? sm[k][lane] : (k < 3 ? 0.0 : -INFINITY);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
      if (lane == 0) part[9 * blockIdx.x + k] = a;
    }
  }
}

// HANDELER.F90:221-243, with the same IEEE operations: one warp reduces the
// block partials (max is exact in any order), lane 0 forms the geometry.
__global__ void k_bbox_final(int nb, const double* __restrict__ part, double* __restrict__ geom,
                             int32_t* __restrict__ dims) {
  const int lane = threadIdx.x & 31;
  double v[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) v[k] = (k < 3) ? 0.0 : -INFINITY;
  for (int b = lane; b < nb; b += 32)
#pragma unroll
    for (int k = 0; k < 9; ++k) v[k] = fmax(v[k], part[9 * b + k]);
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
  if (lane != 0) return;
  const double xbin = v[0], ybin = v[1], zbin = v[2];
  const double xmin = __dsub_rn(-v[6], __dmul_rn(xbin, 10.0));
  const double ymin = __dsub_rn(-v[7], __dmul_rn(ybin, 10.0));
  const double zmin = __dsub_rn(-v[8], __dmul_rn(zbin, 10.0));
  const double xmax = __dadd_rn(v[3], __dmul_rn(xbin, 10.0));
  const double ymax = __dadd_rn(v[4], __dmul_rn(ybin, 10.0));
  const double zmax = __dadd_rn(v[5], __dmul_rn(zbin, 10.0));
  geom[0] = xmin; geom[1] = ymin; geom[2] = zmin;
  geom[3] = xbin; geom[4] = ybin; geom[5] = zbin;
  dims[0] = (int32_t)ceil(__ddiv_rn(__dsub_rn(xmax, xmin), xbin));
  dims[1] = (int32_t)ceil(__ddiv_rn(__dsub_rn(ymax, ymin), ybin));
  dims[2] = (int32_t)ceil(__ddiv_rn(__dsub_rn(zmax, zmin), zbin));
}

__device__ __forceinline__ int32_t bin_of(double x, double xmin, double bin, int32_t nb) {
  int32_t c = (int32_t)floor(__ddiv_rn(__dsub_rn(x, xmin), bin)) + 1;
  c = max(1, c);
  return min(c, nb);
}

// ---- 2. cell per node, histogram
__global__ void k_cell_assign(int32_t n, const double* __restrict__ coo, const double* __restrict__ geom,
                              int32_t nx, int32_t ny, int32_t nz, int32_t* __restrict__ cell,
                              int32_t* __restrict__ cnt, int32_t* __restrict__ ijk) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t a = bin_of(coo[3 * i], geom[0], geom[3], nx);
  const int32_t b = bin_of(coo[3 * i + 1], geom[1], geom[4], ny);
  const int32_t c = bin_of(coo[3 * i + 2], geom[2], geom[5], nz);
  const int32_t m = (c - 1) * nx * ny + (b - 1) * nx + (a - 1);
  cell[i] = m;
  atomicAdd(&cnt[m], 1);
  if (ijk) { ijk[3 * i] = a; ijk[3 * i + 1] = b; ijk[3 * i + 2] = c; }
}

// ---- 3. scatter into cells, then restore index order inside each cell
__global__ void k_cell_scatter(int32_t n, const int32_t* __restrict__ cell, const int64_t* __restrict__ cstart,
                               int32_t* __restrict__ fill, int32_t* __restrict__ sorted) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t m = cell[i];
  const int32_t k = atomicAdd(&fill[m], 1);
  sorted[cstart[m] + k] = (int32_t)i;
}

__global__ void k_cell_sort(int64_t nbins, const int64_t* __restrict__ cstart, int32_t* __restrict__ sorted,
                            unsigned* __restrict__ status) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m >= nbins) return;
  const int64_t s = cstart[m], e = cstart[m + 1];
  if (e - s >= kMaxBinCount) atomicOr(status, (unsigned)MEGA_ST_BIN_OVERFLOW);
  for (int64_t a = s + 1; a < e; ++a) {  // insertion sort (cells hold few nodes)
    const int32_t v = sorted[a];
    int64_t b = a - 1;
    while (b >= s && sorted[b] > v) { sorted[b + 1] = sorted[b]; --b; }
    sorted[b + 1] = v;
  }
}

// dx / w < 1 with the quotient rounded to nearest, decided without the
// division for w > 0: the largest double below w divided by w is at most
// 1 - 2^-53, which is a double, so the rounded quotient of any dx < w stays
// below 1, and dx >= w gives a quotient of at least 1.  (NaN dx fails both.)
__device__ __forceinline__ bool quotient_below_one(double dx, double w) {
  return w > 0.0 ? dx < w : __ddiv_rn(dx, w) < 1.0;
}

// SOFT_SEARCH acceptance test (BIN_SEARCH.F90:235-293), exact arithmetic.
__device__ __forceinline__ bool accept(const double xi[3], const double xj[3], const double wj[3],
                                       const double sl[6], int mmax, int shsup) {
  for (int m = 0; m < mmax; ++m) {
    double px = xj[0], py = xj[1], pz = xj[2];
    if (m == 1) px = __dadd_rn(xj[0], sl[0]);
    else if (m == 2) px = __dsub_rn(xj[0], sl[1]);
    else if (m == 3) py = __dadd_rn(xj[1], sl[2]);
    else if (m == 4) py = __dsub_rn(xj[1], sl[3]);
    else if (m == 5) pz = __dadd_rn(xj[2], sl[4]);
    else if (m == 6) pz = __dsub_rn(xj[2], sl[5]);
    const double dx = fabs(__dsub_rn(px, xi[0]));
    const double dy = fabs(__dsub_rn(py, xi[1]));
    const double dz = fabs(__dsub_rn(pz, xi[2]));
    if (shsup) {
      const double a = __ddiv_rn(dx, wj[0]), b = __ddiv_rn(dy, wj[1]), c = __ddiv_rn(dz, wj[2]);
      const double s = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
      if (__dsqrt_rn(s) < 1.0) return true;
    } else {
      if (quotient_below_one(dx, wj[0]) && quotient_below_one(dy, wj[1]) && quotient_below_one(dz, wj[2]))
        return true;
    }
  }
  return false;
}

// ---- 4/5. warp-per-node filter of node i's candidates.  Lane k < 27 owns
// neighbour cell k in the reference's visiting order (IX outer, IY, IZ
// inner; cells outside the grid are empty).  The candidates of all 27 cells
// form one index range [0, total) walked 32 at a time, so the output keeps
// the reference order with every lane busy.  SORTED: candidate coordinates
// and windows come from the cell-sorted copies xs / ws (contiguous within a
// cell; one 48-byte record x, w per node, read as three 16-byte loads, with
// no dependence on the index load); otherwise from coo / win by index.
// WRITE: accepted indices go to out[0 .. count).  Returns the count; the
// candidate total in *total_out (lane values agree).
template <bool WRITE, bool SORTED, int MMAX = 0>
__device__ __forceinline__ int32_t filter_row(int64_t i, int lane, const double* __restrict__ coo,
                                              const double* __restrict__ win, const double* __restrict__ xw,
                                              const double* __restrict__ sm_len,
                                              const int32_t* __restrict__ cell, int32_t nx, int32_t ny, int32_t nz,
                                              const int64_t* __restrict__ cstart, const int32_t* __restrict__ sorted,
                                              int mmax, int shsup, int32_t* __restrict__ out, int32_t* total_out) {
  if (MMAX) mmax = MMAX;  // the seven-point test count fixed at compile time
  const double xi[3] = {coo[3 * i], coo[3 * i + 1], coo[3 * i + 2]};
  double sl[6];  // smoothing cells: read only by the seven-point test (mmax = 7)
#pragma unroll
  for (int k = 0; k < 6; ++k) sl[k] = mmax > 1 ? sm_len[6 * i + k] : 0.0;
  const int32_t m0 = cell[i];
  const int32_t is = m0 % nx + 1, js = (m0 / nx) % ny + 1, ks = m0 / (nx * ny) + 1;
  int64_t cbeg = 0;
  int32_t clen = 0;
  if (lane < 27) {
    const int32_t ix = is - 1 + lane / 9, iy = js - 1 + (lane / 3) % 3, iz = ks - 1 + lane % 3;
    if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
      const int64_t m = (int64_t)(iz - 1) * nx * ny + (int64_t)(iy - 1) * nx + (ix - 1);
      cbeg = cstart[m];
      clen = (int32_t)(cstart[m + 1] - cbeg);
    }
  }
  int32_t pre = clen;  // inclusive scan of the cell lengths
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += y;
  }
  const int32_t total = __shfl_sync(0xffffffffu, pre, 31);
  pre -= clen;  // exclusive
  const unsigned lt = (1u << lane) - 1u;
  int32_t count = 0;
  for (int32_t c0 = 0; c0 < total; c0 += 32) {
    const int32_t c = c0 + lane;
    bool add = false;
    int32_t j = 0;
    // owning cell: the last k with pre_k <= c (binary search over lanes 0..26)
    int k = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int t = k + step;
      const int32_t pt = __shfl_sync(0xffffffffu, pre, t < 27 ? t : 26);
      if (t < 27 && pt <= c) k = t;
    }
    const int64_t cb = __shfl_sync(0xffffffffu, cbeg, k);
    const int32_t pk = __shfl_sync(0xffffffffu, pre, k);
    if (c < total) {
      const int64_t q = cb + (c - pk);
      if (SORTED) {
        if (WRITE) j = sorted[q];  // requested with the record, not after the test
        const double2* r = reinterpret_cast<const double2*>(xw + 6 * q);
        const double2 r0 = r[0], r1 = r[1], r2 = r[2];
        const double xj[3] = {r0.x, r0.y, r1.x};
        const double wj[3] = {r1.y, r2.x, r2.y};
        add = accept(xi, xj, wj, sl, mmax, shsup);
      } else {
        j = sorted[q];
        const double xj[3] = {coo[3 * (int64_t)j], coo[3 * (int64_t)j + 1], coo[3 * (int64_t)j + 2]};
        const double wj[3] = {win[3 * (int64_t)j], win[3 * (int64_t)j + 1], win[3 * (int64_t)j + 2]};
        add = accept(xi, xj, wj, sl, mmax, shsup);
      }
    }
    const unsigned b = __ballot_sync(0xffffffffu, add);
    if (WRITE && add) out[count + __popc(b & lt)] = j;
    count += __popc(b);
  }
  *total_out = total;
  return count;
}

// FILL = false counts, FILL = true writes the row (two-pass form)
template <bool FILL>
__global__ void __launch_bounds__(256) k_soft_search(
    int32_t n, const double* __restrict__ coo, const double* __restrict__ win, const double* __restrict__ sm_len,
    const int32_t* __restrict__ cell, int32_t nx, int32_t ny, int32_t nz, const int64_t* __restrict__ cstart,
    const int32_t* __restrict__ sorted, int mmax, int shsup, int32_t* __restrict__ gn,
    const int64_t* __restrict__ rowptr, int32_t* __restrict__ col, int32_t* __restrict__ gmaxn,
    unsigned* __restrict__ status) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // whole warp leaves together
  int32_t total = 0;
  const int32_t count = filter_row<FILL, false>(i, lane, coo, win, nullptr, sm_len, cell, nx, ny, nz, cstart, sorted,
                                                mmax, shsup, FILL ? col + rowptr[i] : nullptr, &total);
  if (lane == 0 && !FILL) {
    gn[i] = count;
    atomic_max_int(gmaxn, count);
    if (total > kMaxCandidates) atomicOr(status, (unsigned)MEGA_ST_CAND_OVERFLOW);
  }
}

// coordinates and windows in cell-sorted order, (x, w) per node
__global__ void k_sorted_coords(int32_t n, const int32_t* __restrict__ sorted, const double* __restrict__ coo,
                                const double* __restrict__ win, double* __restrict__ xw) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int64_t j = sorted[q];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    xw[6 * q + k] = coo[3 * j + k];
    xw[6 * q + 3 + k] = win[3 * j + k];
  }
}

// candidates of each node: the node counts of its 27 cells
__global__ void k_cand_count(int32_t n, const int32_t* __restrict__ cell, int32_t nx, int32_t ny, int32_t nz,
                             const int64_t* __restrict__ cstart, int32_t* __restrict__ cand,
                             unsigned* __restrict__ status) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t m0 = cell[i];
  const int32_t is = m0 % nx + 1, js = (m0 / nx) % ny + 1, ks = m0 / (nx * ny) + 1;
  int64_t t = 0;
  for (int32_t ix = is - 1; ix <= is + 1; ++ix)
    for (int32_t iy = js - 1; iy <= js + 1; ++iy)
      for (int32_t iz = ks - 1; iz <= ks + 1; ++iz)
        if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
          const int64_t m = (int64_t)(iz - 1) * nx * ny + (int64_t)(iy - 1) * nx + (ix - 1);
          t += cstart[m + 1] - cstart[m];
        }
  cand[i] = (int32_t)t;
  if (t > kMaxCandidates) atomicOr(status, (unsigned)MEGA_ST_CAND_OVERFLOW);
}

// one filter pass: node i's accepted indices into its candidate slots
// buf[coff[i] ..), its count into gn[i]; MMAX = 1 (DNI) or 7
template <int MMAX>
__global__ void __launch_bounds__(256, MMAX == 1 ? 4 : 3) k_search_once(
    int32_t n, const double* __restrict__ coo, const double* __restrict__ win, const double* __restrict__ xw,
    const double* __restrict__ sm_len, const int32_t* __restrict__ cell, int32_t nx,
    int32_t ny, int32_t nz, const int64_t* __restrict__ cstart, const int32_t* __restrict__ sorted, int mmax,
    int shsup, const int64_t* __restrict__ coff, int32_t* __restrict__ buf, int32_t* __restrict__ gn,
    int32_t* __restrict__ gmaxn) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  int32_t total = 0;
  const int32_t count = filter_row<true, true, MMAX>(i, lane, coo, win, xw, sm_len, cell, nx, ny, nz, cstart, sorted,
                                                     mmax, shsup, buf + coff[i], &total);
  if (lane == 0) {
    gn[i] = count;
    atomic_max_int(gmaxn, count);
  }
}

// warp per row: the accepted indices from the candidate slots into the CSR
__global__ void __launch_bounds__(256) k_compact_rows(int32_t n, const int64_t* __restrict__ coff,
                                                      const int32_t* __restrict__ buf,
                                                      const int64_t* __restrict__ rowptr, int32_t* __restrict__ col) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t a = coff[i], d = rowptr[i], len = rowptr[i + 1] - d;
  for (int64_t k = lane; k < len; k += 32) col[d + k] = buf[a + k];
}

// ---- scan helpers
constexpr int kScanBlock = 1024;

__global__ void k_scan_block_sums(int64_t m, const int32_t* __restrict__ cnt, int64_t* __restrict__ bsum) {
  __shared__ int64_t sm[32];
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  int64_t v = (i < m) ? cnt[i] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t a = sm[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) bsum[blockIdx.x] = a;
  }
}

// single block: exclusive scan of nb block sums in place, total at [nb]
__global__ void k_scan_bsums(int64_t nb, int64_t* __restrict__ bsum) {
  __shared__ int64_t carry_s;
  __shared__ int64_t wsum[32];
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nb; b0 += kScanBlock) {
    const int64_t b = b0 + threadIdx.x;
    const int64_t v = (b < nb) ? bsum[b] : 0;
    int64_t x = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int64_t w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const int64_t incl = x + (wid > 0 ? wsum[wid - 1] : 0);
    const int64_t carry = carry_s;
    if (b < nb) bsum[b] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry_s = carry + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[nb] = carry_s;
}

__global__ void k_scan_apply(int64_t m, const int32_t* __restrict__ cnt, const int64_t* __restrict__ bsum,
                             int64_t* __restrict__ off) {
  __shared__ int64_t wsum[32];
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  const int64_t v = (i < m) ? cnt[i] : 0;
  int64_t x = v;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t w = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  const int64_t incl = x + (wid > 0 ? wsum[wid - 1] : 0);
  if (i < m) off[i] = bsum[blockIdx.x] + incl - v;
  if (i == m - 1) off[m] = bsum[blockIdx.x] + incl;
}

// ---- transpose (CSC) helpers
__global__ void k_col_count(int64_t nnz, const int32_t* __restrict__ col, int32_t* __restrict__ ccnt) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < nnz) atomicAdd(&ccnt[col[p]], 1);
}

// the largest of n counts into *mx (zeroed by the caller)
__global__ void k_max_count(int32_t n, const int32_t* __restrict__ cnt, int32_t* __restrict__ mx) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int32_t v = i < n ? cnt[i] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0) atomicMax(mx, v);
}
// Entry (i, j) of the lists into column j at an arbitrary free slot: its row
// i and its offset inside row i (the order is restored by k_col_sort).
__global__ void k_col_scatter(int32_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ colptr, int32_t* __restrict__ cfill,
                              int32_t* __restrict__ toff, int32_t* __restrict__ trow) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t r0 = rowptr[i];
  for (int64_t p = r0 + lane; p < rowptr[i + 1]; p += 32) {
    const int32_t j = col[p];
    const int64_t e = colptr[j] + atomicAdd(&cfill[j], 1);
    toff[e] = (int32_t)(p - r0);
    trow[e] = (int32_t)i;
  }
}

// Bitonic sort of 32 * PER (row, offset) pairs by row across one warp:
// element e = k * 32 + lane; stages of stride >= 32 compare a lane's own
// registers, the others exchange by shuffles.  Rows are distinct within a
// column, so the order is total.
template <int PER>
__device__ __forceinline__ void warp_bitonic(int32_t (&key)[PER], int32_t (&val)[PER], int lane) {
#pragma unroll
  for (int size = 2; size <= 32 * PER; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int ks = stride >> 5;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          if (k & ks) continue;
          const int k2 = k | ks;
          const bool up = ((k * 32 + lane) & size) == 0;
          if ((key[k] > key[k2]) == up) {
            const int32_t tk = key[k]; key[k] = key[k2]; key[k2] = tk;
            const int32_t tv = val[k]; val[k] = val[k2]; val[k2] = tv;
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          const int32_t ok = __shfl_xor_sync(0xffffffffu, key[k], stride);
          const int32_t ov = __shfl_xor_sync(0xffffffffu, val[k], stride);
          const bool up = ((k * 32 + lane) & size) == 0;
          const bool lower = (lane & stride) == 0;
          const bool take_min = (lower == up);
          if (take_min ? (ok < key[k]) : (ok > key[k])) { key[k] = ok; val[k] = ov; }
        }
      }
    }
  }
}

template <int PER>
__device__ __forceinline__ void sort_column(int64_t s, int64_t len, int lane, const int64_t* __restrict__ rowptr,
                                            const int32_t* __restrict__ toff, int64_t* __restrict__ tpos,
                                            int32_t* __restrict__ trow) {
  int32_t key[PER], val[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int idx = k * 32 + lane;
    key[k] = idx < len ? trow[s + idx] : INT_MAX;
    val[k] = idx < len ? toff[s + idx] : 0;
  }
  warp_bitonic<PER>(key, val, lane);
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int idx = k * 32 + lane;
    if (idx < len) {
      trow[s + idx] = key[k];
      tpos[s + idx] = rowptr[key[k]] + val[k];
    }
  }
}

// Order each column by row (equivalently by CSR position, rows being
// contiguous and ascending), so the CSC sums are deterministic, and form
// the CSR position of every entry.  Warp per column: up to 256 entries
// sorted in registers by a network sized to the column; longer columns by
// one lane's insertion sort.
__global__ void __launch_bounds__(256) k_col_sort(int32_t n, const int64_t* __restrict__ colptr,
                                                  const int64_t* __restrict__ rowptr,
                                                  const int32_t* __restrict__ toff, int64_t* __restrict__ tpos,
                                                  int32_t* __restrict__ trow) {
  const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  const int64_t s = colptr[j], e = colptr[j + 1];
  const int64_t len = e - s;
  if (len <= 32) sort_column<1>(s, len, lane, rowptr, toff, tpos, trow);
  else if (len <= 64) sort_column<2>(s, len, lane, rowptr, toff, tpos, trow);
  else if (len <= 128) sort_column<4>(s, len, lane, rowptr, toff, tpos, trow);
  else if (len <= 256) sort_column<8>(s, len, lane, rowptr, toff, tpos, trow);
  else if (lane == 0) {
    for (int64_t a = s; a < e; ++a) {
      const int32_t r = trow[a];
      const int64_t v = rowptr[r] + toff[a];
      int64_t b = a - 1;
      while (b >= s && trow[b] > r) { tpos[b + 1] = tpos[b]; trow[b + 1] = trow[b]; --b; }
      tpos[b + 1] = v;
      trow[b + 1] = r;
    }
  }
}

inline unsigned grid_for(int64_t work, int block) { return (unsigned)((work + block - 1) / block); }

}  // namespace

int scan_counts(cudaStream_t s, const int32_t* cnt, int64_t* off, int64_t m, DevPool& scratch) {
  if (m <= 0) {
    MEGA_TRY(cudaMemsetAsync(off, 0, sizeof(int64_t), s));
    return 0;
  }
  const int64_t nb = (m + kScanBlock - 1) / kScanBlock;
  int64_t* bsum = nullptr;
  MEGA_ALLOC(scratch, bsum, nb + 1);
  k_scan_block_sums<<<(unsigned)nb, kScanBlock, 0, s>>>(m, cnt, bsum);
  MEGA_CHECK_LAUNCH();
  k_scan_bsums<<<1, kScanBlock, 0, s>>>(nb, bsum);
  MEGA_CHECK_LAUNCH();
  k_scan_apply<<<(unsigned)nb, kScanBlock, 0, s>>>(m, cnt, bsum, off);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int bin_search(cudaStream_t s, int32_t n, const double* coo, const double* win, const double* sm_len,
               const double dist_max[3], int32_t itype_int, int32_t shsup, unsigned* status, DevCSR& csr,
               int32_t* ijk, DevPool& pool, BinGeom* geom_out, int32_t* cell_order, const BinGeom* fixed) {
  DevPool scratch(s);  // freed on return
  csr.n = n;
  const int nbb = 148 * 2;
  double* part = nullptr;
  double* geom = nullptr;
  int32_t* dims = nullptr;
  MEGA_ALLOC(scratch, part, 9 * nbb);
  MEGA_ALLOC(scratch, geom, 6);
  MEGA_ALLOC(scratch, dims, 3);
  BinGeom bg;
  if (fixed) {  // the semi-Lagrangian re-search keeps the LINIT bins (HANDELER.F90:181-250 run at LINIT only)
    bg = *fixed;
    MEGA_TRY(cudaMemcpyAsync(geom, bg.g, sizeof(double) * 6, cudaMemcpyHostToDevice, s));
  } else {
    k_bbox_partial<<<nbb, 256, 0, s>>>(n, coo, win, dist_max[0], dist_max[1], dist_max[2], part);
    MEGA_CHECK_LAUNCH();
    k_bbox_final<<<1, 32, 0, s>>>(nbb, part, geom, dims);
    MEGA_CHECK_LAUNCH();
    MEGA_TRY(cudaMemcpyAsync(bg.g, geom, sizeof(double) * 6, cudaMemcpyDeviceToHost, s));
    int32_t hd[3];
    MEGA_TRY(cudaMemcpyAsync(hd, dims, sizeof(hd), cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    bg.nx = hd[0]; bg.ny = hd[1]; bg.nz = hd[2];
  }
  if (geom_out) *geom_out = bg;
  const int64_t nbins = (int64_t)bg.nx * bg.ny * bg.nz;
  if (bg.nx <= 0 || bg.ny <= 0 || bg.nz <= 0 || nbins > INT32_MAX) return MEGA_ERR_UNSUPPORTED;

  int32_t *cell = nullptr, *cnt = nullptr, *fill = nullptr, *sorted = nullptr, *gn = nullptr;
  int64_t* cstart = nullptr;
  MEGA_ALLOC(scratch, cell, n);
  MEGA_ALLOC(scratch, cnt, nbins);
  MEGA_ALLOC(scratch, fill, nbins);
  MEGA_ALLOC(scratch, cstart, nbins + 1);
  MEGA_ALLOC(scratch, sorted, n);
  MEGA_ALLOC(scratch, gn, n);
  MEGA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * nbins, s));
  MEGA_TRY(cudaMemsetAsync(fill, 0, sizeof(int32_t) * nbins, s));
  k_cell_assign<<<grid_for(n, 256), 256, 0, s>>>(n, coo, geom, bg.nx, bg.ny, bg.nz, cell, cnt, ijk);
  MEGA_CHECK_LAUNCH();
  int r = scan_counts(s, cnt, cstart, nbins, scratch);
  if (r) return r;
  k_cell_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, cell, cstart, fill, sorted);
  MEGA_CHECK_LAUNCH();
  k_cell_sort<<<grid_for(nbins, 256), 256, 0, s>>>(nbins, cstart, sorted, status);
  MEGA_CHECK_LAUNCH();
  if (cell_order)  // nodes by bin cell (cell id order, index order inside a cell)
    MEGA_TRY(cudaMemcpyAsync(cell_order, sorted, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));

  const int mmax = (itype_int == 0) ? 1 : 7;  // BIN_SEARCH.F90:204-208
  int32_t* gmaxn = nullptr;
  MEGA_ALLOC(scratch, gmaxn, 1);
  MEGA_TRY(cudaMemsetAsync(gmaxn, 0, sizeof(int32_t), s));
  MEGA_ALLOC(pool, csr.rowptr, (int64_t)n + 1);
  const unsigned gw = grid_for((int64_t)n * 32, 256);
  // One filter pass into per-node candidate slots (4 bytes per candidate,
  // about 27 cells x 8 nodes per node), then a compaction; the two-pass form
  // where the slots do not fit.
  int32_t* cand = nullptr;
  int64_t* coff = nullptr;
  MEGA_ALLOC(scratch, cand, n);
  MEGA_ALLOC(scratch, coff, (int64_t)n + 1);
  k_cand_count<<<grid_for(n, 256), 256, 0, s>>>(n, cell, bg.nx, bg.ny, bg.nz, cstart, cand, status);
  MEGA_CHECK_LAUNCH();
  r = scan_counts(s, cand, coff, n, scratch);
  if (r) return r;
  int64_t ctot = 0;
  MEGA_TRY(cudaMemcpyAsync(&ctot, coff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  int32_t* buf = nullptr;
  double* xw = nullptr;
  size_t fr = 0, tot = 0;
  const bool once = cudaMemGetInfo(&fr, &tot) == cudaSuccess &&
                    (size_t)ctot * sizeof(int32_t) + 48 * (size_t)n + ((size_t)1 << 30) < fr;
  if (once) {
    MEGA_ALLOC(scratch, buf, ctot);
    MEGA_ALLOC(scratch, xw, 6 * (int64_t)n);
    k_sorted_coords<<<grid_for(n, 256), 256, 0, s>>>(n, sorted, coo, win, xw);
    MEGA_CHECK_LAUNCH();
    auto k = mmax == 1 ? k_search_once<1> : k_search_once<7>;
    k<<<gw, 256, 0, s>>>(n, coo, win, xw, sm_len, cell, bg.nx, bg.ny, bg.nz, cstart, sorted, mmax, shsup, coff, buf, gn,
                         gmaxn);
  } else {
    k_soft_search<false><<<gw, 256, 0, s>>>(n, coo, win, sm_len, cell, bg.nx, bg.ny, bg.nz, cstart, sorted, mmax,
                                            shsup, gn, nullptr, nullptr, gmaxn, status);
  }
  MEGA_CHECK_LAUNCH();
  r = scan_counts(s, gn, csr.rowptr, n, scratch);
  if (r) return r;
  int64_t nnz = 0;
  MEGA_TRY(cudaMemcpyAsync(&nnz, csr.rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&csr.gmaxn, gmaxn, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  csr.nnz = nnz;
  MEGA_ALLOC(pool, csr.col, nnz);
  if (once)
    k_compact_rows<<<gw, 256, 0, s>>>(n, coff, buf, csr.rowptr, csr.col);
  else
    k_soft_search<true><<<gw, 256, 0, s>>>(n, coo, win, sm_len, cell, bg.nx, bg.ny, bg.nz, cstart, sorted, mmax,
                                           shsup, gn, csr.rowptr, csr.col, gmaxn, status);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaStreamSynchronize(s));
  return 0;
}

int build_transpose(cudaStream_t s, DevCSR& csr, DevPool& pool) {
  DevPool scratch(s);
  const int32_t n = csr.n;
  int32_t *ccnt = nullptr, *cfill = nullptr;
  int32_t* cmax = nullptr;
  MEGA_ALLOC(scratch, ccnt, n);
  MEGA_ALLOC(scratch, cfill, n);
  MEGA_ALLOC(scratch, cmax, 1);
  MEGA_ALLOC(pool, csr.colptr, (int64_t)n + 1);
  MEGA_ALLOC(pool, csr.trow, csr.nnz);
  MEGA_ALLOC(pool, csr.tpos, csr.nnz);
  MEGA_TRY(cudaMemsetAsync(ccnt, 0, sizeof(int32_t) * n, s));
  MEGA_TRY(cudaMemsetAsync(cfill, 0, sizeof(int32_t) * n, s));
  MEGA_TRY(cudaMemsetAsync(cmax, 0, sizeof(int32_t), s));
  k_col_count<<<grid_for(csr.nnz, 256), 256, 0, s>>>(csr.nnz, csr.col, ccnt);
  MEGA_CHECK_LAUNCH();
  k_max_count<<<grid_for(n, 256), 256, 0, s>>>(n, ccnt, cmax);
  MEGA_CHECK_LAUNCH();
  int r = scan_counts(s, ccnt, csr.colptr, n, scratch);
  if (r) return r;
  int32_t* toff = nullptr;
  MEGA_ALLOC(scratch, toff, csr.nnz);
  k_col_scatter<<<grid_for((int64_t)n * 32, 256), 256, 0, s>>>(n, csr.rowptr, csr.col, csr.colptr, cfill, toff,
                                                              csr.trow);
  MEGA_CHECK_LAUNCH();
  k_col_sort<<<grid_for((int64_t)n * 32, 256), 256, 0, s>>>(n, csr.colptr, csr.rowptr, toff, csr.tpos, csr.trow);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaMemcpyAsync(&csr.gmaxc, cmax, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace mega

// ===========================================================================
// Neighbour search that allocates nothing.
//
// Some callers cannot call cudaMalloc at the moment they need a neighbour
// list: a host code whose GPU memory is owned by another allocator (a
// framework's caching pool, a Fortran code that maps one arena at start-up),
// a real-time loop where an allocation's implicit synchronisation is not
// allowed, or a process that has hit its device-memory quota.  This variant
// takes its inputs and outputs in device memory the caller already owns and
// takes every temporary (bounding-box partials, bin histogram and offsets,
// cell-sorted node list, row offsets) from one fixed array that is part of
// the library image.
//
// The array is a file-scope __device__ object of kNoAllocScratchBytes; every
// GPU that loads the library holds it until the process exits.  Host code
// cannot use the symbol g_noalloc_scratch as a device address (on the host it
// names a stand-in object), so the first call on each device looks the
// address up with cudaGetSymbolAddress while that device is current and
// caches it; make that first call before any stream capture.  All calls
// share the array and it keeps the previous call's contents: the counters
// that must start at zero are cleared on every call.  Calls whose work
// overlaps on the GPU (other streams, other host threads) race on the array,
// so serialise them.
// ===========================================================================

namespace mega {

constexpr int64_t kNoAllocScratchBytes = 48ll << 20;  // 48 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {nullptr};

// set-up, once per device, with that device current
int noalloc_scratch_address(void** out) {
  int dev = 0;
  MEGA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return MEGA_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    MEGA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return MEGA_ERR_CUDA;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

// bump allocator over the fixed array (256-byte aligned slices)
struct Carve {
  unsigned char* base;
  int64_t used = 0;
  template <typename T>
  T* take(int64_t count) {
    T* p = (T*)(base + used);
    used += ((count * (int64_t)sizeof(T) + 255) / 256) * 256;
    return p;
  }
};

int64_t scan_scratch_count(int64_t m) { return (m + kScanBlock - 1) / kScanBlock + 1; }

int scan_counts_into(cudaStream_t s, const int32_t* cnt, int64_t* off, int64_t m, int64_t* bsum) {
  if (m <= 0) {
    MEGA_TRY(cudaMemsetAsync(off, 0, sizeof(int64_t), s));
    return 0;
  }
  const int64_t nb = (m + kScanBlock - 1) / kScanBlock;
  k_scan_block_sums<<<(unsigned)nb, kScanBlock, 0, s>>>(m, cnt, bsum);
  MEGA_CHECK_LAUNCH();
  k_scan_bsums<<<1, kScanBlock, 0, s>>>(nb, bsum);
  MEGA_CHECK_LAUNCH();
  k_scan_apply<<<(unsigned)nb, kScanBlock, 0, s>>>(m, cnt, bsum, off);
  MEGA_CHECK_LAUNCH();
  return 0;
}

// 0-based device CSR -> the reference's GN / GSTART / GSTACK (1-based)
__global__ void k_noalloc_fortran(int32_t n, const int64_t* __restrict__ rowptr, int32_t* __restrict__ gn,
                                  int32_t* __restrict__ gstart) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  gn[i] = (int32_t)(rowptr[i + 1] - rowptr[i]);
  gstart[i] = (int32_t)(rowptr[i] + 1);
}
__global__ void k_noalloc_plus_one(int64_t m, int32_t* __restrict__ v) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < m) v[p] += 1;
}

// scratch bytes for n nodes and nbins bins (each slice rounded to 256 B)
int64_t noalloc_bytes(int64_t n, int64_t nbins, int nbb) {
  auto r = [](int64_t b) { return ((b + 255) / 256) * 256; };
  return r(9 * 8 * (int64_t)nbb) + r(6 * 8) + r(3 * 4) + r(4) + r(4) + r(4 * n) + r(4 * n) + r(4 * n) +
         r(8 * (n + 1)) + r(4 * nbins) + r(4 * nbins) + r(8 * (nbins + 1)) +
         r(8 * scan_scratch_count(std::max<int64_t>(nbins, n)));
}

}  // namespace
}  // namespace mega

extern "C" int mega_bin_search_noalloc(int32_t n, const double* d_coo, const double* d_win,
                                       const double* d_sm_len, const double* dist_max, int32_t itype_int,
                                       int32_t shsup, int32_t* d_gn, int32_t* d_gstart, int32_t* d_gstack,
                                       int64_t dim_nn_list, int32_t* d_ijk, int32_t* gmaxn, int64_t* nnz,
                                       void* stream) {
  using namespace mega;
  if (n <= 0 || !d_coo || !d_win || !d_sm_len || !dist_max || !d_gn || !d_gstart || !d_gstack || !gmaxn || !nnz)
    return MEGA_ERR_ARG;
  const int nbb = 148 * 2;
  // reject before touching any input when the nodes alone exceed the array
  if (noalloc_bytes(n, 1, nbb) > kNoAllocScratchBytes) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "mega_bin_search_noalloc: %d nodes need more than its fixed %lld-byte scratch array", (int)n,
             (long long)kNoAllocScratchBytes);
    record_error_text(msg);
    return MEGA_ERR_UNSUPPORTED;
  }
  void* base = nullptr;
  int r = noalloc_scratch_address(&base);
  if (r) return r;
  cudaStream_t s = (cudaStream_t)stream;
  Carve cv{(unsigned char*)base};
  double* part = cv.take<double>(9 * nbb);
  double* geom = cv.take<double>(6);
  int32_t* dims = cv.take<int32_t>(3);
  unsigned* status = cv.take<unsigned>(1);
  int32_t* dmax = cv.take<int32_t>(1);
  int32_t* cell = cv.take<int32_t>(n);
  int32_t* sorted = cv.take<int32_t>(n);
  int32_t* gnw = cv.take<int32_t>(n);
  int64_t* rowptr = cv.take<int64_t>((int64_t)n + 1);
  const int64_t head = cv.used;
  k_bbox_partial<<<nbb, 256, 0, s>>>(n, d_coo, d_win, dist_max[0], dist_max[1], dist_max[2], part);
  MEGA_CHECK_LAUNCH();
  k_bbox_final<<<1, 32, 0, s>>>(nbb, part, geom, dims);
  MEGA_CHECK_LAUNCH();
  int32_t hd[3];
  MEGA_TRY(cudaMemcpyAsync(hd, dims, sizeof(hd), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  const int64_t nbins = (int64_t)hd[0] * hd[1] * hd[2];
  if (hd[0] <= 0 || hd[1] <= 0 || hd[2] <= 0 || nbins > INT32_MAX) return MEGA_ERR_UNSUPPORTED;
  if (noalloc_bytes(n, nbins, nbb) > kNoAllocScratchBytes) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "mega_bin_search_noalloc: %d nodes in %lld bins need %lld bytes of scratch, the fixed array has %lld",
             (int)n, (long long)nbins, (long long)noalloc_bytes(n, nbins, nbb), (long long)kNoAllocScratchBytes);
    record_error_text(msg);
    return MEGA_ERR_UNSUPPORTED;
  }
  cv.used = head;
  int32_t* cnt = cv.take<int32_t>(nbins);
  int32_t* fill = cv.take<int32_t>(nbins);
  int64_t* cstart = cv.take<int64_t>(nbins + 1);
  int64_t* bsum = cv.take<int64_t>(scan_scratch_count(std::max<int64_t>(nbins, n)));
  // the array keeps the previous call's contents: clear the counters
  MEGA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * nbins, s));
  MEGA_TRY(cudaMemsetAsync(fill, 0, sizeof(int32_t) * nbins, s));
  MEGA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned), s));
  MEGA_TRY(cudaMemsetAsync(dmax, 0, sizeof(int32_t), s));
  k_cell_assign<<<grid_for(n, 256), 256, 0, s>>>(n, d_coo, geom, hd[0], hd[1], hd[2], cell, cnt, d_ijk);
  MEGA_CHECK_LAUNCH();
  r = scan_counts_into(s, cnt, cstart, nbins, bsum);
  if (r) return r;
  k_cell_scatter<<<grid_for(n, 256), 256, 0, s>>>(n, cell, cstart, fill, sorted);
  MEGA_CHECK_LAUNCH();
  k_cell_sort<<<grid_for(nbins, 256), 256, 0, s>>>(nbins, cstart, sorted, status);
  MEGA_CHECK_LAUNCH();
  const int mmax = (itype_int == 0) ? 1 : 7;  // BIN_SEARCH.F90:204-208
  const unsigned gw = grid_for((int64_t)n * 32, 256);
  k_soft_search<false><<<gw, 256, 0, s>>>(n, d_coo, d_win, d_sm_len, cell, hd[0], hd[1], hd[2], cstart, sorted,
                                          mmax, shsup, gnw, nullptr, nullptr, dmax, status);
  MEGA_CHECK_LAUNCH();
  r = scan_counts_into(s, gnw, rowptr, n, bsum);
  if (r) return r;
  int64_t total = 0;
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(&total, rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(gmaxn, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hst, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  *nnz = total;
  if (total > (int64_t)INT32_MAX) {  // GSTART is a default INTEGER (int32): 1-based starts would wrap
    char msg[256];
    snprintf(msg, sizeof(msg),
             "mega_bin_search_noalloc: %lld list entries exceed the 32-bit GSTART range", (long long)total);
    record_error_text(msg);
    return MEGA_ERR_UNSUPPORTED;
  }
  k_noalloc_fortran<<<grid_for(n, 256), 256, 0, s>>>(n, rowptr, d_gn, d_gstart);
  MEGA_CHECK_LAUNCH();
  if (total > dim_nn_list) {  // the caller's GSTACK is too small: lists not written
    MEGA_TRY(cudaStreamSynchronize(s));
    return (int)(hst | MEGA_ST_STACK_OVERFLOW);
  }
  k_soft_search<true><<<gw, 256, 0, s>>>(n, d_coo, d_win, d_sm_len, cell, hd[0], hd[1], hd[2], cstart, sorted,
                                         mmax, shsup, gnw, rowptr, d_gstack, dmax, status);
  MEGA_CHECK_LAUNCH();
  k_noalloc_plus_one<<<grid_for(total, 256), 256, 0, s>>>(total, d_gstack);
  MEGA_CHECK_LAUNCH();
  // the fill pass ORs into the same status word: report both passes
  MEGA_TRY(cudaMemcpyAsync(&hst, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  return (int)hst;
}
