// tiled.cu -- shared-memory tiled gathers for the per-step kernels.
//
// The untiled gathers (force.cu) issue ten to thirteen scattered loads per
// neighbour entry and run at the L1 throughput limit with HBM far from busy.
// Here nodes are renumbered in bin-cell order (spatially compact), rows are
// grouped into tiles of R consecutive nodes, and each tile's neighbour set
// (the union of its rows, "J-set") is listed once.  Every neighbour entry
// then carries its gradient and a 16-bit tile-local index in one 16-byte
// (float) or 32-byte (double) record, and the neighbour data the tile needs
// -- (u_tot, du) for the deformation gradient, T_i for the force -- is staged
// in shared memory once per tile:
//   k_defgrad_t  F = I + sum_J (u_J - u_i) (x) g + u_i (x) sum g,  G0 likewise
//   k_force_t    f_J = sum_i T_i g^T_iJ, then the corrector / predictor
// The summation order is fixed by the list order, so results are
// deterministic, and identical in exact arithmetic to force.cu's.
#include "mega_internal.cuh"
#include "tiled.cuh"
#include "bulk.cuh"

namespace mega {
namespace {

// Launch variants of the two gathers (picked per context by the autotuner):
// KG lanes per row / column (4, 8 or 16), KU packed records in flight per
// lane (1, 2 or 4).  A block serves one tile of R rows with R * KG threads.
template <int KG>
__device__ __forceinline__ unsigned group_mask() {
  return ((1u << KG) - 1u) << (threadIdx.x & (32 - KG));
}

__device__ __forceinline__ unsigned hash_u32(unsigned x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}

// Block per tile: list the distinct neighbours of the tile's rows, sort them,
// and give each entry its rank in that list.  HS hash slots in shared memory;
// a tile with more than jmax distinct neighbours reports overflow.
template <int HS>
__global__ void __launch_bounds__(256) k_build_tiles(int32_t n, int32_t R, const int64_t* __restrict__ ptr,
                                                     const int32_t* __restrict__ idx, int32_t jmax,
                                                     int32_t* __restrict__ jset, int32_t* __restrict__ jcnt,
                                                     uint16_t* __restrict__ lidx, int16_t* __restrict__ slot_tmp,
                                                     int32_t* __restrict__ overflow) {
  __shared__ int32_t keys[HS];
  __shared__ int16_t rank[HS];
  __shared__ int32_t sk[HS / 2];
  __shared__ int32_t wsum[8];
  __shared__ int32_t s_total, s_full;
  const int tid = threadIdx.x;
  const int64_t t = blockIdx.x;
  const int64_t r0 = t * R, r1 = min((int64_t)n, r0 + R);
  const int64_t p0 = ptr[r0], p1 = ptr[r1];
  for (int s = tid; s < HS; s += blockDim.x) keys[s] = -1;
  if (tid == 0) s_full = 0;
  __syncthreads();
  for (int64_t p = p0 + tid; p < p1; p += blockDim.x) {
    const int32_t j = idx[p];
    unsigned h = hash_u32((unsigned)j) & (HS - 1);
    int16_t slot = -1;
    for (int probe = 0; probe < HS; ++probe) {  // bounded: a full table stops
      const int32_t prev = atomicCAS(&keys[h], -1, j);
      if (prev == -1 || prev == j) { slot = (int16_t)h; break; }
      h = (h + 1) & (HS - 1);
    }
    if (slot < 0) s_full = 1;
    slot_tmp[p] = slot;
  }
  __syncthreads();
  // compaction of the occupied slots: each thread owns HS/256 consecutive slots
  constexpr int PER = HS / 256;
  int cnt = 0;
  for (int k = 0; k < PER; ++k) cnt += (keys[tid * PER + k] != -1);
  int x = cnt;
  const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (tid == 0) {
    int a = 0;
    for (int w = 0; w < 8; ++w) { const int v = wsum[w]; wsum[w] = a; a += v; }
    s_total = a;
  }
  __syncthreads();
  const int total = s_total;
  if (total > jmax || s_full) {  // the whole block leaves together
    if (tid == 0) {
      jcnt[t] = total;
      atomicMax(overflow, s_full ? HS : total);
    }
    return;
  }
  int pos = wsum[wid] + x - cnt;
  for (int k = 0; k < PER; ++k) {
    const int32_t key = keys[tid * PER + k];
    if (key != -1) sk[pos++] = key;
  }
  int np2 = 1;
  while (np2 < total) np2 <<= 1;
  for (int s = total + tid; s < np2; s += blockDim.x) sk[s] = INT32_MAX;
  __syncthreads();
  // bitonic sort of sk[0..np2)
  for (int k = 2; k <= np2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < np2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int32_t a = sk[i], b = sk[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) { sk[i] = b; sk[l] = a; }
        }
      }
      __syncthreads();
    }
  // rank of each slot = position of its key in the sorted list
  for (int r = tid; r < total; r += blockDim.x) {
    const int32_t key = sk[r];
    unsigned h = hash_u32((unsigned)key) & (HS - 1);
    for (int probe = 0; probe < HS; ++probe) {
      if (keys[h] == key) { rank[h] = (int16_t)r; break; }
      h = (h + 1) & (HS - 1);
    }
    jset[t * (int64_t)jmax + r] = key;
  }
  if (tid == 0) jcnt[t] = total;
  __syncthreads();
  for (int64_t p = p0 + tid; p < p1; p += blockDim.x) lidx[p] = (uint16_t)rank[slot_tmp[p]];
}

// list entries of each tile of R consecutive rows
__global__ void k_tile_entries(int32_t n, int32_t R, int64_t ntiles, const int64_t* __restrict__ ptr,
                               int32_t* __restrict__ ent) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int64_t r0 = t * R, r1 = min((int64_t)n, r0 + R);
  ent[t] = (int32_t)(ptr[r1] - ptr[r0]);
}

__global__ void k_pack_f32(int64_t m, const uint16_t* __restrict__ lidx, const double* __restrict__ gx,
                           const double* __restrict__ gy, const double* __restrict__ gz,
                           const int64_t* __restrict__ pos, float4* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m) return;
  const int64_t p = pos ? pos[e] : e;
  out[e] = make_float4((float)gx[p], (float)gy[p], (float)gz[p], __int_as_float((int)lidx[e]));
}

__global__ void k_pack_t32(int64_t m, const uint16_t* __restrict__ lidx, const float4* __restrict__ in,
                           const int64_t* __restrict__ pos, float4* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m) return;
  const float4 v = in[pos[e]];
  out[e] = make_float4(v.x, v.y, v.z, __int_as_float((int)lidx[e]));
}

__global__ void k_pack_f64(int64_t m, const uint16_t* __restrict__ lidx, const double* __restrict__ gx,
                           const double* __restrict__ gy, const double* __restrict__ gz,
                           const int64_t* __restrict__ pos, double2* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m) return;
  const int64_t p = pos ? pos[e] : e;
  out[2 * e] = make_double2(gx[p], gy[p]);
  out[2 * e + 1] = make_double2(gz[p], __longlong_as_double((long long)lidx[e]));
}

// Entry order for conflict-free reads of the staged neighbour data.  In the
// gathers the KG lanes of a row (column) take its entries KG at a time, and
// the 32 lanes of a warp read the staged values of their current entries in
// one instruction: lanes whose tile ranks l differ but agree modulo NC (the
// bank period of the staged layout) are served one after another, lanes with
// the same l by one broadcast.  This reorders the entries within each row so
// that, at every step, the lanes of each group of GL lanes hold, per class
// l mod NC, one rank only wherever the row's remaining entries allow (greedy,
// lanes in order, each taking its first entry whose class is free or holds
// the same rank); a row keeps all its entries, only their order changes.
// pos, when given, is permuted with lidx.  One warp per warp of the gather's
// blocks, four warps per block.
constexpr int kBankCap = 2048;  // entries of one warp's rows that its pass stages in shared memory

template <int KG, int NC, int GL>
__global__ void __launch_bounds__(128) k_bank_order(int32_t n, int32_t R, int64_t nwarps,
                                                    const int64_t* __restrict__ ptr, uint16_t* lidx,
                                                    const int64_t* __restrict__ pos_src, int64_t* pos) {
  __shared__ int held_s[4][32];
  __shared__ uint16_t sl_s[4][kBankCap], so_s[4][kBankCap];  // ranks, and offsets in the row before
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (w >= nwarps) return;  // whole warps leave together
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  int* held = held_s[wi] + (lane / GL) * NC;  // this lane's group: the rank held per class
  const int wpt = R * KG / 32;  // warps per tile
  const int64_t c = (w / wpt) * R + (w % wpt) * (32 / KG) + lane / KG;
  const int q = lane & (KG - 1);
  int64_t b = 0, e = 0;
  if (c < n) { b = ptr[c]; e = ptr[c + 1]; }
  const int len = (int)(e - b);
  // the warp's rows one after another in shared memory, where they fit
  int x = q == 0 ? len : 0;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const int total = __shfl_sync(0xffffffffu, x, 31);
  const int off = __shfl_sync(0xffffffffu, x - (q == 0 ? len : 0), lane & ~(KG - 1));
  const bool fast = total <= kBankCap;  // warp-uniform
  uint16_t* sl = sl_s[wi] + off;
  uint16_t* so = so_s[wi] + off;
  if (fast)
    for (int k = q; k < len; k += KG) { sl[k] = lidx[b + k]; so[k] = (uint16_t)k; }
  __syncwarp();
  int steps = (len + KG - 1) / KG;
#pragma unroll
  for (int o = 16; o; o >>= 1) steps = max(steps, __shfl_xor_sync(0xffffffffu, steps, o));
  for (int s = 0; s < steps; ++s) {
    const int slot = s * KG + q;
    held_s[wi][lane] = -1;
    __syncwarp();
    for (int turn = 0; turn < 32; ++turn) {
      if (lane == turn && slot < len) {
        if (fast) {
          int pick = slot;
          for (int k = slot; k < len; ++k) {
            const int l = sl[k], h = held[l & (NC - 1)];
            if (h < 0 || h == l) { pick = k; break; }
          }
          if (pick != slot) {
            const uint16_t t1 = sl[pick]; sl[pick] = sl[slot]; sl[slot] = t1;
            const uint16_t t2 = so[pick]; so[pick] = so[slot]; so[slot] = t2;
          }
          const int l = sl[slot];
          if (held[l & (NC - 1)] < 0) held[l & (NC - 1)] = l;
        } else {  // rows too long for shared memory: the same pass in place
          int64_t pick = b + slot;
          for (int64_t k = b + slot; k < e; ++k) {
            const int l = lidx[k], h = held[l & (NC - 1)];
            if (h < 0 || h == l) { pick = k; break; }
          }
          if (pick != b + slot) {
            const uint16_t t1 = lidx[pick]; lidx[pick] = lidx[b + slot]; lidx[b + slot] = t1;
            const int64_t t2 = pos[pick]; pos[pick] = pos[b + slot]; pos[b + slot] = t2;
          }
          const int l = lidx[b + slot];
          if (held[l & (NC - 1)] < 0) held[l & (NC - 1)] = l;
        }
      }
      __syncwarp();
    }
  }
  if (fast)
    for (int k = q; k < len; k += KG) {
      lidx[b + k] = sl[k];
      pos[b + k] = pos_src ? pos_src[b + so[k]] : b + so[k];
    }
}

__global__ void k_gather_rec32(int64_t m, const int64_t* __restrict__ pos, const float4* __restrict__ in,
                               float4* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m) out[e] = in[pos[e]];
}

// the tile rank carried by each float record
__global__ void k_rec_ranks(int64_t m, const float4* __restrict__ rec, uint16_t* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m) out[e] = (uint16_t)__float_as_int(rec[e].w);
}

// out[6 e + k] = in[6 pos[e] + k]
__global__ void k_gather_f6(int64_t m, const int64_t* __restrict__ pos, const float2* __restrict__ in,
                            float2* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m) return;
  const int64_t p = pos[e];
  out[3 * e] = in[3 * p]; out[3 * e + 1] = in[3 * p + 1]; out[3 * e + 2] = in[3 * p + 2];
}

__global__ void k_iota64(int64_t m, int64_t* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m) out[e] = e;
}

template <bool F64>
__device__ __forceinline__ void load_entry(const void* pk, int64_t p, float& g0, float& g1, float& g2, int& l);
template <>
__device__ __forceinline__ void load_entry<false>(const void* pk, int64_t p, float& g0, float& g1, float& g2,
                                                  int& l) {
  const float4 v = __ldg((const float4*)pk + p);
  g0 = v.x; g1 = v.y; g2 = v.z; l = __float_as_int(v.w);
}
__device__ __forceinline__ void load_entry64(const void* pk, int64_t p, double& g0, double& g1, double& g2, int& l) {
  const double2 a = __ldg((const double2*)pk + 2 * p);
  const double2 b = __ldg((const double2*)pk + 2 * p + 1);
  g0 = a.x; g1 = a.y; g2 = b.x; l = (int)__double_as_longlong(b.y);
}

// The six float S values of one NSNI record (three 8-byte loads).
struct SRec {
  float2 a, b, c;
};
__device__ __forceinline__ SRec load_srec(const float* base, int64_t p) {
  const float2* sp = reinterpret_cast<const float2*>(base) + 3 * p;
  return SRec{__ldg(sp), __ldg(sp + 1), __ldg(sp + 2)};
}

// NS: the NSNI gradients of the incremental displacement gradient ride
// along, H_i(k, q) = sum_J S_q(i, J) du_J,k, formed like L as
// sum_J S_q (du_J - du_i) + du_i,k sum_J S_q (FINT.F90:728-737 layout).
template <typename A, bool F64, bool INTERP, int KG, int KU, bool NS = false>
__global__ void __launch_bounds__(64 * KG, (F64 ? 12 : (NS ? 8 : 16)) / KG > 0 ? (F64 ? 12 : (NS ? 8 : 16)) / KG : 1) k_defgrad_t(int32_t n, int32_t R, int32_t jmax,
                                                   NsniTiles ns,
                                                   const int64_t* __restrict__ rowptr, const void* __restrict__ pk,
                                                   const int32_t* __restrict__ jset, const int32_t* __restrict__ jcnt,
                                                   const double* __restrict__ dsp, const double* __restrict__ dsp_tot,
                                                   const double* __restrict__ sdphi, const double* __restrict__ shp,
                                                   double* __restrict__ dsp_tot_phy, double* __restrict__ fg,
                                                   StepAccum* __restrict__ acc) {
  extern __shared__ double sm[];
  if (acc && blockIdx.x == 0 && threadIdx.x < kSlots) {
    acc->newton_iters[threadIdx.x] = 0ull;
    acc->plastic[threadIdx.x] = 0ull;
  }
  const int64_t t = blockIdx.x;
  const int cnt = jcnt[t];
  const int32_t* js = jset + t * (int64_t)jmax;
  // Staged neighbour displacements.  FP64: u_J and du_J as doubles.  Mixed:
  // float offsets from the tile's first node r0 (u_J - u_r0, du_J - du_r0),
  // half the shared-memory traffic, one array per component (value k of
  // rank l at sf[k * cnt + l]: lanes with distinct l mod 32 read distinct
  // banks); the differences u_J - u_i are formed between offsets, exact up
  // to float rounding of the offsets.
  double* su = sm;
  double* sd = sm + 3 * cnt;
  float* sf = reinterpret_cast<float*>(sm);
  const int64_t r0 = t * R;
  const int64_t i = t * R + threadIdx.x / KG;
  const int q = threadIdx.x & (KG - 1);
  const unsigned gmask = group_mask<KG>();
  const bool valid = threadIdx.x / KG < R && i < n;
  // this lane's first KU packed records are requested before the staging,
  // so their latency overlaps it
  int64_t p = 0, pend = 0;
  bool pre = false;
  float4 pf[KU];
  double2 pfa[KU], pfb[KU];
  SRec psr[NS ? KU : 1];
  if (valid) {
    p = rowptr[i] + q;
    pend = rowptr[i + 1];
    pre = p + (KU - 1) * KG < pend;
    if (pre) {
#pragma unroll
      for (int u = 0; u < KU; ++u) {
        if (F64) {
          pfa[u] = __ldg((const double2*)pk + 2 * (p + u * KG));
          pfb[u] = __ldg((const double2*)pk + 2 * (p + u * KG) + 1);
        } else {
          pf[u] = __ldg((const float4*)pk + p + u * KG);
        }
        if constexpr (NS) psr[u] = load_srec(ns.srow, p + u * KG);
      }
    }
  }
  double ur0 = 0.0, ur1 = 0.0, ur2 = 0.0, dr0 = 0.0, dr1 = 0.0, dr2 = 0.0;
  if (!F64) {
    ur0 = dsp_tot[3 * r0]; ur1 = dsp_tot[3 * r0 + 1]; ur2 = dsp_tot[3 * r0 + 2];
    dr0 = dsp[3 * r0]; dr1 = dsp[3 * r0 + 1]; dr2 = dsp[3 * r0 + 2];
  }
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
    const int64_t g = js[l];
    const double a0 = dsp_tot[3 * g], a1 = dsp_tot[3 * g + 1], a2 = dsp_tot[3 * g + 2];
    const double b0 = dsp[3 * g], b1 = dsp[3 * g + 1], b2 = dsp[3 * g + 2];
    if (F64) {
      su[3 * l] = a0; su[3 * l + 1] = a1; su[3 * l + 2] = a2;
      sd[3 * l] = b0; sd[3 * l + 1] = b1; sd[3 * l + 2] = b2;
    } else {
      sf[l] = (float)(a0 - ur0); sf[cnt + l] = (float)(a1 - ur1); sf[2 * cnt + l] = (float)(a2 - ur2);
      sf[3 * cnt + l] = (float)(b0 - dr0); sf[4 * cnt + l] = (float)(b1 - dr1); sf[5 * cnt + l] = (float)(b2 - dr2);
    }
  }
  __syncthreads();
  if (!valid) return;
  const double ui0 = dsp_tot[3 * i], ui1 = dsp_tot[3 * i + 1], ui2 = dsp_tot[3 * i + 2];
  const double di0 = dsp[3 * i], di1 = dsp[3 * i + 1], di2 = dsp[3 * i + 2];
  const float fu0 = (float)(ui0 - ur0), fu1 = (float)(ui1 - ur1), fu2 = (float)(ui2 - ur2);
  const float fd0 = (float)(di0 - dr0), fd1 = (float)(di1 - dr1), fd2 = (float)(di2 - dr2);
  A F[9], L[9];
  double H[NS ? 18 : 1];  // NSNI: exact products of the float S and differences, summed in double
#pragma unroll
  for (int k = 0; k < 9; ++k) { F[k] = A(0); L[k] = A(0); }
#pragma unroll
  for (int k = 0; k < (NS ? 18 : 1); ++k) H[k] = 0.0;
  double ph0 = 0.0, ph1 = 0.0, ph2 = 0.0;
  // One entry: F += (u_J - u_i) (x) g, L += (d_J - d_i) (x) g (+ phi d_J),
  // H(k, q) += S_q (d_J - d_i)_k.
  auto body = [&](int64_t p, A g0, A g1, A g2, int l, const SRec& sr) {
    A u0, u1, u2, d0, d1, d2;
    double dj0, dj1, dj2;  // du_J itself, for the per-step interpolation
    if (F64) {
      u0 = (A)(su[3 * l] - ui0); u1 = (A)(su[3 * l + 1] - ui1); u2 = (A)(su[3 * l + 2] - ui2);
      dj0 = sd[3 * l]; dj1 = sd[3 * l + 1]; dj2 = sd[3 * l + 2];
      d0 = (A)(dj0 - di0); d1 = (A)(dj1 - di1); d2 = (A)(dj2 - di2);
    } else {
      const float* v = sf + l;
      const float v3 = v[3 * cnt], v4 = v[4 * cnt], v5 = v[5 * cnt];
      u0 = (A)(v[0] - fu0); u1 = (A)(v[cnt] - fu1); u2 = (A)(v[2 * cnt] - fu2);
      d0 = (A)(v3 - fd0); d1 = (A)(v4 - fd1); d2 = (A)(v5 - fd2);
      if (INTERP) { dj0 = dr0 + (double)v3; dj1 = dr1 + (double)v4; dj2 = dr2 + (double)v5; }
      else { dj0 = dj1 = dj2 = 0.0; }
    }
    F[0] += u0 * g0; F[1] += u0 * g1; F[2] += u0 * g2;
    F[3] += u1 * g0; F[4] += u1 * g1; F[5] += u1 * g2;
    F[6] += u2 * g0; F[7] += u2 * g1; F[8] += u2 * g2;
    L[0] += d0 * g0; L[1] += d0 * g1; L[2] += d0 * g2;
    L[3] += d1 * g0; L[4] += d1 * g1; L[5] += d1 * g2;
    L[6] += d2 * g0; L[7] += d2 * g1; L[8] += d2 * g2;
    if constexpr (NS) {
      const double sq[6] = {(double)sr.a.x, (double)sr.a.y, (double)sr.b.x, (double)sr.b.y, (double)sr.c.x,
                            (double)sr.c.y};
      const double e0 = (double)d0, e1 = (double)d1, e2 = (double)d2;
#pragma unroll
      for (int c = 0; c < 6; ++c) { H[c] += sq[c] * e0; H[6 + c] += sq[c] * e1; H[12 + c] += sq[c] * e2; }
    }
    if (INTERP) {
      const double s = shp[p];
      ph0 += s * dj0; ph1 += s * dj1; ph2 += s * dj2;
    }
  };
  // KU records in flight per lane before any is used (the loop is bound by
  // DRAM latency otherwise); each lane still sums its entries in list order.
  const SRec s0{};
  if (pre) {
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      if (F64)
        body(p + u * KG, (A)pfa[u].x, (A)pfa[u].y, (A)pfb[u].x, (int)__double_as_longlong(pfb[u].y), s0);
      else
        body(p + u * KG, (A)pf[u].x, (A)pf[u].y, (A)pf[u].z, __float_as_int(pf[u].w), NS ? psr[NS ? u : 0] : s0);
    }
    p += KU * KG;
  }
  if (F64) {
    for (; p + (KU - 1) * KG < pend; p += KU * KG) {
      double2 ra[KU], rb[KU];
#pragma unroll
      for (int u = 0; u < KU; ++u) {
        ra[u] = __ldg((const double2*)pk + 2 * (p + u * KG));
        rb[u] = __ldg((const double2*)pk + 2 * (p + u * KG) + 1);
      }
#pragma unroll
      for (int u = 0; u < KU; ++u)
        body(p + u * KG, (A)ra[u].x, (A)ra[u].y, (A)rb[u].x, (int)__double_as_longlong(rb[u].y), s0);
    }
  } else if constexpr (!NS) {
    // software-pipelined: the next KU records are requested before this
    // KU's sums, so a lane keeps loads in flight while it computes
    float4 cur[KU];
    bool have = p + (KU - 1) * KG < pend;
    if (have) {
#pragma unroll
      for (int u = 0; u < KU; ++u) cur[u] = __ldg((const float4*)pk + p + u * KG);
    }
    while (have) {
      const int64_t pn = p + KU * KG;
      const bool hn = pn + (KU - 1) * KG < pend;
      float4 nxt[KU];
#pragma unroll
      for (int u = 0; u < KU; ++u) nxt[u] = hn ? __ldg((const float4*)pk + pn + u * KG) : cur[u];
#pragma unroll
      for (int u = 0; u < KU; ++u)
        body(p + u * KG, (A)cur[u].x, (A)cur[u].y, (A)cur[u].z, __float_as_int(cur[u].w), s0);
#pragma unroll
      for (int u = 0; u < KU; ++u) cur[u] = nxt[u];
      p = pn;
      have = hn;
    }
  } else {
    for (; p + (KU - 1) * KG < pend; p += KU * KG) {
      float4 r[KU];
      SRec sr[NS ? KU : 1];
#pragma unroll
      for (int u = 0; u < KU; ++u) {
        r[u] = __ldg((const float4*)pk + p + u * KG);
        if constexpr (NS) sr[u] = load_srec(ns.srow, p + u * KG);
      }
#pragma unroll
      for (int u = 0; u < KU; ++u)
        body(p + u * KG, (A)r[u].x, (A)r[u].y, (A)r[u].z, __float_as_int(r[u].w), NS ? sr[NS ? u : 0] : s0);
    }
  }
  for (; p < pend; p += KG) {
    if (F64) {
      double a0, a1, a2;
      int l;
      load_entry64(pk, p, a0, a1, a2, l);
      body(p, (A)a0, (A)a1, (A)a2, l, s0);
    } else {
      float a0, a1, a2;
      int l;
      load_entry<false>(pk, p, a0, a1, a2, l);
      body(p, (A)a0, (A)a1, (A)a2, l, NS ? load_srec(ns.srow, p) : s0);
    }
  }
#pragma unroll
  for (int o = 1; o < KG; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      F[k] += __shfl_xor_sync(gmask, F[k], o);
      L[k] += __shfl_xor_sync(gmask, L[k], o);
    }
    if constexpr (NS) {
#pragma unroll
      for (int k = 0; k < 18; ++k) H[k] += __shfl_xor_sync(gmask, H[k], o);
    }
    if (INTERP) {
      ph0 += __shfl_xor_sync(gmask, ph0, o);
      ph1 += __shfl_xor_sync(gmask, ph1, o);
      ph2 += __shfl_xor_sync(gmask, ph2, o);
    }
  }
  if (q == 0) {
    const double ui[3] = {ui0, ui1, ui2}, di[3] = {di0, di1, di2};
    if constexpr (NS) {
      double ss[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) ss[c] = ns.ssum[6 * i + c];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) ns.hq[18 * i + 6 * k + c] = H[6 * k + c] + di[k] * ss[c];
    }
    const double sd3[3] = {sdphi[3 * i], sdphi[3 * i + 1], sdphi[3 * i + 2]};
    double h[18];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        h[3 * k + l] = (double)F[3 * k + l] + ui[k] * sd3[l];
        h[9 + 3 * k + l] = (double)L[3 * k + l] + di[k] * sd3[l];
      }
    store_fg(fg, i, !F64, h);
    if (INTERP) {
      dsp_tot_phy[3 * i] += ph0;
      dsp_tot_phy[3 * i + 1] += ph1;
      dsp_tot_phy[3 * i + 2] += ph2;
    }
  }
}

// One DOF m = 3 J + q after its column sum fi (and body-force sum fe):
// fixity, acceleration and corrector (MAIN.F90:432-488), the energy and
// reaction sums, and the next step's predictor (MAIN.F90:353-355).
__device__ __forceinline__ void correct_dof(const TiledForceArgs& a, int64_t J, int q, double fi, double fe,
                                            double& ke, double& ee, double* tf, unsigned& st) {
  const int64_t m = 3 * J + q;
  const double dt = a.ndt ? a.ndt[J] : a.dt;
  if (a.fadd) fi += a.fadd[m];
  if (!isfinite(fi)) st |= MEGA_ST_NONFINITE;
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
    acc = (fe - fi - mpdc * v) / (mass + 0.5 * dt * mpdc);
    v = v + 0.5 * dt * acc;
    pr = 0.0;
  }
  ee += 0.5 * (fe + fe_old) * a.dsp[m];
  ke += 0.5 * mass * v * v;
  const int b = a.body_id ? a.body_id[J] : 1;
#pragma unroll
  for (int k = 0; k < 3; ++k)  // constant indices: the sums stay in registers
    if (q == k) {
      if (b == 1) tf[k] += pr;
      else if (b == 2) tf[3 + k] += pr;
    }
  a.fint[m] = fi;
  a.fext[m] = fe;
  a.acl[m] = acc;
  a.prforce[m] = pr;
  if (a.predict) {  // MAIN.F90:353-355 of the next step
    const double d = dt * v + dt * dt * 0.5 * acc;
    a.dsp[m] = d;
    a.dsp_tot[m] = a.dsp_tot[m] + d;
    v = v + dt * 0.5 * acc;
  }
  a.vel[m] = v;
}

// One block reduction of the eight step sums, then one atomic per sum into
// this block's slot.  Every thread of the block takes part.
__device__ __forceinline__ void step_sums(const TiledForceArgs& a, double ke, double ee, const double* tf,
                                          double* red) {
  double v[8] = {ke, ee, tf[0], tf[1], tf[2], tf[3], tf[4], tf[5]};
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 8; ++k) red[wid * 8 + k] = v[k];
  __syncthreads();
  if (threadIdx.x < 8) {
    const int nw = (blockDim.x + 31) >> 5;
    double tsum = 0.0;
    for (int w = 0; w < nw; ++w) tsum += red[w * 8 + threadIdx.x];
    const int sl = blockIdx.x % kSlots;
    double* dst = threadIdx.x == 0 ? &a.acc->ke[sl] : (threadIdx.x == 1 ? &a.acc->ee[sl] : &a.acc->tf[threadIdx.x - 2][sl]);
    if (tsum != 0.0) atomicAdd(dst, tsum);
  }
}

// TS = storage of T_i (float / double), A = accumulation, F64 = record width
// NS (mixed): the NSNI stabilisation force rides along,
// f_J += sum_i sum_q W_i(k, q) S_q(i, J) (FINT.F90:1127-1208 layout), with the
// row weights W_i staged beside T_i.
template <typename TS, typename A, bool F64, int KG, int KU, bool NS = false>
__global__ void __launch_bounds__(64 * KG) k_force_t(TiledForceArgs a) {
  extern __shared__ double smx[];
  __shared__ double red[32 * 8];  // eight sums per warp, up to 32 warps (KG = 16)
  const int64_t t = blockIdx.x;
  const int cnt = a.jcnt[t];
  const int nv = a.has_body ? 12 : 9;
  TS* sT = (TS*)smx;
  const int32_t* js = a.jset + t * (int64_t)a.jmax;
  const TS* tm = (const TS*)a.tmat;
  const int64_t J = t * a.R + threadIdx.x / KG;
  const int q = threadIdx.x & (KG - 1);
  const unsigned gmask = group_mask<KG>();
  const bool valid = threadIdx.x / KG < a.R && J < a.n;
  // this lane's first KU packed records are requested before the staging,
  // so their latency overlaps it (FP64 records only)
  int64_t e = 0, c1 = 0;
  bool pre = false;
  float4 pf[KU];
  double2 pfa[KU], pfb[KU];
  if (F64 && valid) {  // measured: pays in FP64, costs occupancy in mixed
    e = a.colptr[J] + q;
    c1 = a.colptr[J + 1];
    pre = e + (KU - 1) * KG < c1;
    if (pre) {
#pragma unroll
      for (int u = 0; u < KU; ++u) {
        if (F64) {
          pfa[u] = __ldg((const double2*)a.pk + 2 * (e + u * KG));
          pfb[u] = __ldg((const double2*)a.pk + 2 * (e + u * KG) + 1);
        } else {
          pf[u] = __ldg((const float4*)a.pk + e + u * KG);
        }
      }
    }
  }
  // thread per staged node: one index load, then its T row (12 values,
  // 48 or 96 bytes, 16-byte aligned) as independent vector loads
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
    const TS* src = tm + 12 * (int64_t)js[l];
    TS v[12];
    if (sizeof(TS) == 4) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 x = __ldg(s4 + k);
        v[4 * k] = (TS)x.x; v[4 * k + 1] = (TS)x.y; v[4 * k + 2] = (TS)x.z; v[4 * k + 3] = (TS)x.w;
      }
    } else {
      const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 x = __ldg(s2 + k);
        v[2 * k] = (TS)x.x; v[2 * k + 1] = (TS)x.y;
      }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) sT[k * cnt + l] = v[k];
    if (nv == 12) { sT[9 * cnt + l] = v[9]; sT[10 * cnt + l] = v[10]; sT[11 * cnt + l] = v[11]; }
    if constexpr (NS) {  // W_l: 18 of its 20 floats, as five 16-byte loads
      const float4* w4 = reinterpret_cast<const float4*>(a.ns_w + 20 * (int64_t)js[l]);
      TS* sW = sT + nv * cnt;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const float4 x = __ldg(w4 + k);
        sW[(4 * k) * cnt + l] = x.x; sW[(4 * k + 1) * cnt + l] = x.y;
        if (4 * k + 2 < 18) { sW[(4 * k + 2) * cnt + l] = x.z; sW[(4 * k + 3) * cnt + l] = x.w; }
      }
    }
  }
  __syncthreads();
  if (!F64 && valid) {
    e = a.colptr[J] + q;
    c1 = a.colptr[J + 1];
  }
  double ke = 0.0, ee = 0.0, tf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  unsigned st = 0;
  if (valid) {
    A f0 = A(0), f1 = A(0), f2 = A(0);
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    auto body = [&](int64_t e, A g0, A g1, A g2, int l, const SRec& sr) {
      const TS* T = sT + l;  // component k of T_l at T[k * cnt]
      f0 += (A)T[0] * g0 + (A)T[cnt] * g1 + (A)T[2 * cnt] * g2;
      f1 += (A)T[3 * cnt] * g0 + (A)T[4 * cnt] * g1 + (A)T[5 * cnt] * g2;
      f2 += (A)T[6 * cnt] * g0 + (A)T[7 * cnt] * g1 + (A)T[8 * cnt] * g2;
      if constexpr (NS) {
        const A sq[6] = {(A)sr.a.x, (A)sr.a.y, (A)sr.b.x, (A)sr.b.y, (A)sr.c.x, (A)sr.c.y};
        const TS* W = T + nv * cnt;  // W_l(k, q) at W[(6 k + q) * cnt]
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          f0 += (A)W[c * cnt] * sq[c];
          f1 += (A)W[(6 + c) * cnt] * sq[c];
          f2 += (A)W[(12 + c) * cnt] * sq[c];
        }
      }
      if (a.has_body) {
        const double s = a.tshp[e];
        e0 += s * (double)T[9 * cnt]; e1 += s * (double)T[10 * cnt]; e2 += s * (double)T[11 * cnt];
      }
    };
    const SRec s0{};
    if (pre) {  // (FP64 only)
#pragma unroll
      for (int u = 0; u < KU; ++u) {
        if (F64)
          body(e + u * KG, (A)pfa[u].x, (A)pfa[u].y, (A)pfb[u].x, (int)__double_as_longlong(pfb[u].y), s0);
        else
          body(e + u * KG, (A)pf[u].x, (A)pf[u].y, (A)pf[u].z, __float_as_int(pf[u].w), s0);
      }
      e += KU * KG;
    }
    if (F64) {
      for (; e + (KU - 1) * KG < c1; e += KU * KG) {
        double2 ra[KU], rb[KU];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          ra[u] = __ldg((const double2*)a.pk + 2 * (e + u * KG));
          rb[u] = __ldg((const double2*)a.pk + 2 * (e + u * KG) + 1);
        }
#pragma unroll
        for (int u = 0; u < KU; ++u)
          body(e + u * KG, (A)ra[u].x, (A)ra[u].y, (A)rb[u].x, (int)__double_as_longlong(rb[u].y), s0);
      }
    } else if constexpr (!NS) {
      // software-pipelined: the next KU records are requested before this
      // KU's sums, so a lane keeps loads in flight while it computes
      float4 cur[KU];
      bool have = e + (KU - 1) * KG < c1;
      if (have) {
#pragma unroll
        for (int u = 0; u < KU; ++u) cur[u] = __ldg((const float4*)a.pk + e + u * KG);
      }
      while (have) {
        const int64_t en = e + KU * KG;
        const bool hn = en + (KU - 1) * KG < c1;
        float4 nxt[KU];
#pragma unroll
        for (int u = 0; u < KU; ++u) nxt[u] = hn ? __ldg((const float4*)a.pk + en + u * KG) : cur[u];
#pragma unroll
        for (int u = 0; u < KU; ++u)
          body(e + u * KG, (A)cur[u].x, (A)cur[u].y, (A)cur[u].z, __float_as_int(cur[u].w), s0);
#pragma unroll
        for (int u = 0; u < KU; ++u) cur[u] = nxt[u];
        e = en;
        have = hn;
      }
    } else {
      for (; e + (KU - 1) * KG < c1; e += KU * KG) {
        float4 r[KU];
        SRec sr[NS ? KU : 1];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
          r[u] = __ldg((const float4*)a.pk + e + u * KG);
          if constexpr (NS) sr[u] = load_srec(a.ns_scol, e + u * KG);
        }
#pragma unroll
        for (int u = 0; u < KU; ++u)
          body(e + u * KG, (A)r[u].x, (A)r[u].y, (A)r[u].z, __float_as_int(r[u].w), NS ? sr[NS ? u : 0] : s0);
      }
    }
    for (; e < c1; e += KG) {
      if (F64) {
        double b0, b1, b2;
        int l;
        load_entry64(a.pk, e, b0, b1, b2, l);
        body(e, (A)b0, (A)b1, (A)b2, l, s0);
      } else {
        float b0, b1, b2;
        int l;
        load_entry<false>(a.pk, e, b0, b1, b2, l);
        body(e, (A)b0, (A)b1, (A)b2, l, NS ? load_srec(a.ns_scol, e) : s0);
      }
    }
#pragma unroll
    for (int o = 1; o < KG; o <<= 1) {
      f0 += __shfl_xor_sync(gmask, f0, o);
      f1 += __shfl_xor_sync(gmask, f1, o);
      f2 += __shfl_xor_sync(gmask, f2, o);
      if (a.has_body) {
        e0 += __shfl_xor_sync(gmask, e0, o);
        e1 += __shfl_xor_sync(gmask, e1, o);
        e2 += __shfl_xor_sync(gmask, e2, o);
      }
    }
    if (q < 3) correct_dof(a, J, q, (double)(q == 0 ? f0 : (q == 1 ? f1 : f2)), q == 0 ? e0 : (q == 1 ? e1 : e2), ke, ee, tf, st);
  }
  step_sums(a, ke, ee, tf, red);
  if (st) atomicOr(a.status, st);
}

// ---- record streams through the copy engine ------------------------------
// The variants below ask the copy engine (cp.async.bulk) for the tile's
// whole record range, in kChunks chunks with an mbarrier each, before the
// block stages its neighbour data: the records stream into shared memory
// while the threads gather, and the entry loop then reads them from shared
// memory.  Sources are this GPU's record arrays (no peer memory, no
// multicast).  Every wait is bounded; a wait that gives up raises
// MEGA_ST_WAIT_TIMEOUT and the lane skips its sums.
constexpr int kChunks = 4;
constexpr int kPollLimit = 1 << 16;

// Thread 0: the barriers, then the copies of entries [0, ne) of the tile
// (src points at its first record, RB bytes each) into rec.
template <int RB>
__device__ __forceinline__ void issue_records(uint64_t* bar, unsigned char* rec, const unsigned char* src,
                                              int64_t ne) {
  if (threadIdx.x != 0) return;
#pragma unroll
  for (int c = 0; c < kChunks; ++c) mbar_init(&bar[c], 1);
  mbar_fence_init();
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int64_t lo = c * ne / kChunks, hi = (c + 1) * ne / kChunks;
    const uint32_t bytes = (uint32_t)((hi - lo) * RB);
    mbar_arrive_expect(&bar[c], bytes);
    for (uint32_t off = 0; off < bytes; off += 32768u)
      bulk_load(rec + lo * RB + off, src + lo * RB + off, min(32768u, bytes - off), &bar[c]);
  }
}

// Wait for the chunks holding entries [a, b) of the tile.
__device__ __forceinline__ bool wait_records(uint64_t* bar, int64_t ne, int64_t a, int64_t b) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int64_t lo = c * ne / kChunks, hi = (c + 1) * ne / kChunks;
    if (ok && lo < b && hi > a) ok = mbar_wait_bounded(&bar[c], 0, kPollLimit);
  }
  return ok;
}

// Thread 0 before the block retires: no copy of the block is left in flight.
__device__ __forceinline__ void drain_records(uint64_t* bar) {
  if (threadIdx.x != 0) return;
#pragma unroll
  for (int c = 0; c < kChunks; ++c) mbar_wait_bounded(&bar[c], 0, kPollLimit);
}

template <typename A, bool F64, bool INTERP, int KG>
__global__ void __launch_bounds__(64 * KG) k_defgrad_b(int32_t n, int32_t R, int32_t jmax, int32_t recmax,
                                                       const int64_t* __restrict__ rowptr, const void* __restrict__ pk,
                                                       const int32_t* __restrict__ jset, const int32_t* __restrict__ jcnt,
                                                       const double* __restrict__ dsp, const double* __restrict__ dsp_tot,
                                                       const double* __restrict__ sdphi, const double* __restrict__ shp,
                                                       double* __restrict__ dsp_tot_phy, double* __restrict__ fg,
                                                       StepAccum* __restrict__ acc, unsigned* __restrict__ status) {
  constexpr int RB = F64 ? 32 : 16;
  extern __shared__ __align__(128) unsigned char smb[];
  __shared__ uint64_t bar[kChunks];
  if (acc && blockIdx.x == 0 && threadIdx.x < kSlots) {
    acc->newton_iters[threadIdx.x] = 0ull;
    acc->plastic[threadIdx.x] = 0ull;
  }
  const int64_t t = blockIdx.x;
  const int64_t r0 = t * R, r1 = min((int64_t)n, r0 + R);
  const int64_t e0 = rowptr[r0], ne = rowptr[r1] - e0;
  issue_records<RB>(bar, smb, (const unsigned char*)pk + e0 * RB, ne);
  const int cnt = jcnt[t];
  const int32_t* js = jset + t * (int64_t)jmax;
  unsigned char* stg = smb + (size_t)recmax * RB;
  double* su = reinterpret_cast<double*>(stg);
  double* sd = su + 3 * cnt;
  float* sf = reinterpret_cast<float*>(stg);  // mixed: value k of rank l at sf[k * cnt + l]
  const int64_t i = r0 + threadIdx.x / KG;
  const int q = threadIdx.x & (KG - 1);
  const unsigned gmask = group_mask<KG>();
  const bool valid = threadIdx.x / KG < R && i < n;
  double ur0 = 0.0, ur1 = 0.0, ur2 = 0.0, dr0 = 0.0, dr1 = 0.0, dr2 = 0.0;
  if (!F64) {
    ur0 = dsp_tot[3 * r0]; ur1 = dsp_tot[3 * r0 + 1]; ur2 = dsp_tot[3 * r0 + 2];
    dr0 = dsp[3 * r0]; dr1 = dsp[3 * r0 + 1]; dr2 = dsp[3 * r0 + 2];
  }
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
    const int64_t g = js[l];
    const double a0 = dsp_tot[3 * g], a1 = dsp_tot[3 * g + 1], a2 = dsp_tot[3 * g + 2];
    const double b0 = dsp[3 * g], b1 = dsp[3 * g + 1], b2 = dsp[3 * g + 2];
    if (F64) {
      su[3 * l] = a0; su[3 * l + 1] = a1; su[3 * l + 2] = a2;
      sd[3 * l] = b0; sd[3 * l + 1] = b1; sd[3 * l + 2] = b2;
    } else {
      sf[l] = (float)(a0 - ur0); sf[cnt + l] = (float)(a1 - ur1); sf[2 * cnt + l] = (float)(a2 - ur2);
      sf[3 * cnt + l] = (float)(b0 - dr0); sf[4 * cnt + l] = (float)(b1 - dr1); sf[5 * cnt + l] = (float)(b2 - dr2);
    }
  }
  __syncthreads();
  if (!valid) {
    drain_records(bar);
    return;
  }
  const int64_t pa = rowptr[i] - e0, pb = rowptr[i + 1] - e0;
  const bool ok = __all_sync(gmask, wait_records(bar, ne, pa, pb));
  const double ui0 = dsp_tot[3 * i], ui1 = dsp_tot[3 * i + 1], ui2 = dsp_tot[3 * i + 2];
  const double di0 = dsp[3 * i], di1 = dsp[3 * i + 1], di2 = dsp[3 * i + 2];
  const float fu0 = (float)(ui0 - ur0), fu1 = (float)(ui1 - ur1), fu2 = (float)(ui2 - ur2);
  const float fd0 = (float)(di0 - dr0), fd1 = (float)(di1 - dr1), fd2 = (float)(di2 - dr2);
  A F[9], L[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) { F[k] = A(0); L[k] = A(0); }
  double ph0 = 0.0, ph1 = 0.0, ph2 = 0.0;
  if (ok) {
    const float4* rec32 = reinterpret_cast<const float4*>(smb);
    const double2* rec64 = reinterpret_cast<const double2*>(smb);
#pragma unroll 4
    for (int64_t p = pa + q; p < pb; p += KG) {
      A g0, g1, g2;
      int l;
      if (F64) {
        const double2 ra = rec64[2 * p], rb = rec64[2 * p + 1];
        g0 = (A)ra.x; g1 = (A)ra.y; g2 = (A)rb.x; l = (int)__double_as_longlong(rb.y);
      } else {
        const float4 r = rec32[p];
        g0 = (A)r.x; g1 = (A)r.y; g2 = (A)r.z; l = __float_as_int(r.w);
      }
      A u0, u1, u2, d0, d1, d2;
      double dj0, dj1, dj2;
      if (F64) {
        u0 = (A)(su[3 * l] - ui0); u1 = (A)(su[3 * l + 1] - ui1); u2 = (A)(su[3 * l + 2] - ui2);
        dj0 = sd[3 * l]; dj1 = sd[3 * l + 1]; dj2 = sd[3 * l + 2];
        d0 = (A)(dj0 - di0); d1 = (A)(dj1 - di1); d2 = (A)(dj2 - di2);
      } else {
        const float* v = sf + l;
        const float v3 = v[3 * cnt], v4 = v[4 * cnt], v5 = v[5 * cnt];
        u0 = (A)(v[0] - fu0); u1 = (A)(v[cnt] - fu1); u2 = (A)(v[2 * cnt] - fu2);
        d0 = (A)(v3 - fd0); d1 = (A)(v4 - fd1); d2 = (A)(v5 - fd2);
        if (INTERP) { dj0 = dr0 + (double)v3; dj1 = dr1 + (double)v4; dj2 = dr2 + (double)v5; }
        else { dj0 = dj1 = dj2 = 0.0; }
      }
      F[0] += u0 * g0; F[1] += u0 * g1; F[2] += u0 * g2;
      F[3] += u1 * g0; F[4] += u1 * g1; F[5] += u1 * g2;
      F[6] += u2 * g0; F[7] += u2 * g1; F[8] += u2 * g2;
      L[0] += d0 * g0; L[1] += d0 * g1; L[2] += d0 * g2;
      L[3] += d1 * g0; L[4] += d1 * g1; L[5] += d1 * g2;
      L[6] += d2 * g0; L[7] += d2 * g1; L[8] += d2 * g2;
      if (INTERP) {
        const double s = shp[e0 + p];
        ph0 += s * dj0; ph1 += s * dj1; ph2 += s * dj2;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < KG; o <<= 1) {
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
    if (!ok) {
      atomicOr(status, (unsigned)MEGA_ST_WAIT_TIMEOUT);
    } else {
      const double ui[3] = {ui0, ui1, ui2}, di[3] = {di0, di1, di2};
      const double sd3[3] = {sdphi[3 * i], sdphi[3 * i + 1], sdphi[3 * i + 2]};
      double h[18];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) {
          h[3 * k + l] = (double)F[3 * k + l] + ui[k] * sd3[l];
          h[9 + 3 * k + l] = (double)L[3 * k + l] + di[k] * sd3[l];
        }
      store_fg(fg, i, !F64, h);
      if (INTERP) {
        dsp_tot_phy[3 * i] += ph0;
        dsp_tot_phy[3 * i + 1] += ph1;
        dsp_tot_phy[3 * i + 2] += ph2;
      }
    }
  }
  drain_records(bar);
}

template <typename TS, typename A, bool F64, int KG>
__global__ void __launch_bounds__(64 * KG) k_force_b(TiledForceArgs a) {
  constexpr int RB = F64 ? 32 : 16;
  extern __shared__ __align__(128) unsigned char smb[];
  __shared__ uint64_t bar[kChunks];
  __shared__ double red[32 * 8];  // eight sums per warp, up to 32 warps (KG = 16)
  const int64_t t = blockIdx.x;
  const int64_t c0 = t * a.R, c1 = min((int64_t)a.n, c0 + a.R);
  const int64_t e0 = a.colptr[c0], ne = a.colptr[c1] - e0;
  issue_records<RB>(bar, smb, (const unsigned char*)a.pk + e0 * RB, ne);
  const int cnt = a.jcnt[t];
  const int nv = a.has_body ? 12 : 9;
  TS* sT = reinterpret_cast<TS*>(smb + (size_t)a.recmax * RB);
  const int32_t* js = a.jset + t * (int64_t)a.jmax;
  const TS* tm = (const TS*)a.tmat;
  const int64_t J = c0 + threadIdx.x / KG;
  const int q = threadIdx.x & (KG - 1);
  const unsigned gmask = group_mask<KG>();
  const bool valid = threadIdx.x / KG < a.R && J < a.n;
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
    const TS* src = tm + 12 * (int64_t)js[l];
    TS v[12];
    if (sizeof(TS) == 4) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 x = __ldg(s4 + k);
        v[4 * k] = (TS)x.x; v[4 * k + 1] = (TS)x.y; v[4 * k + 2] = (TS)x.z; v[4 * k + 3] = (TS)x.w;
      }
    } else {
      const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double2 x = __ldg(s2 + k);
        v[2 * k] = (TS)x.x; v[2 * k + 1] = (TS)x.y;
      }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) sT[k * cnt + l] = v[k];
    if (nv == 12) { sT[9 * cnt + l] = v[9]; sT[10 * cnt + l] = v[10]; sT[11 * cnt + l] = v[11]; }
  }
  __syncthreads();
  double ke = 0.0, ee = 0.0, tf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  unsigned st = 0;
  if (valid) {
    const int64_t pa = a.colptr[J] - e0, pb = a.colptr[J + 1] - e0;
    const bool ok = __all_sync(gmask, wait_records(bar, ne, pa, pb));
    A f0 = A(0), f1 = A(0), f2 = A(0);
    double b0 = 0.0, b1 = 0.0, b2 = 0.0;
    if (ok) {
      const float4* rec32 = reinterpret_cast<const float4*>(smb);
      const double2* rec64 = reinterpret_cast<const double2*>(smb);
#pragma unroll 4
      for (int64_t p = pa + q; p < pb; p += KG) {
        A g0, g1, g2;
        int l;
        if (F64) {
          const double2 ra = rec64[2 * p], rb = rec64[2 * p + 1];
          g0 = (A)ra.x; g1 = (A)ra.y; g2 = (A)rb.x; l = (int)__double_as_longlong(rb.y);
        } else {
          const float4 r = rec32[p];
          g0 = (A)r.x; g1 = (A)r.y; g2 = (A)r.z; l = __float_as_int(r.w);
        }
        const TS* T = sT + l;  // component k of T_l at T[k * cnt]
        f0 += (A)T[0] * g0 + (A)T[cnt] * g1 + (A)T[2 * cnt] * g2;
        f1 += (A)T[3 * cnt] * g0 + (A)T[4 * cnt] * g1 + (A)T[5 * cnt] * g2;
        f2 += (A)T[6 * cnt] * g0 + (A)T[7 * cnt] * g1 + (A)T[8 * cnt] * g2;
        if (a.has_body) {
          const double s = a.tshp[e0 + p];
          b0 += s * (double)T[9 * cnt]; b1 += s * (double)T[10 * cnt]; b2 += s * (double)T[11 * cnt];
        }
      }
    }
#pragma unroll
    for (int o = 1; o < KG; o <<= 1) {
      f0 += __shfl_xor_sync(gmask, f0, o);
      f1 += __shfl_xor_sync(gmask, f1, o);
      f2 += __shfl_xor_sync(gmask, f2, o);
      if (a.has_body) {
        b0 += __shfl_xor_sync(gmask, b0, o);
        b1 += __shfl_xor_sync(gmask, b1, o);
        b2 += __shfl_xor_sync(gmask, b2, o);
      }
    }
    if (!ok) {
      if (q == 0) st |= MEGA_ST_WAIT_TIMEOUT;
    } else if (q < 3) {
      correct_dof(a, J, q, (double)(q == 0 ? f0 : (q == 1 ? f1 : f2)), q == 0 ? b0 : (q == 1 ? b1 : b2), ke, ee, tf,
                  st);
    }
  }
  step_sums(a, ke, ee, tf, red);
  if (st) atomicOr(a.status, st);
  drain_records(bar);
}

inline unsigned grid_for(int64_t work, int block) { return (unsigned)((work + block - 1) / block); }

}  // namespace

int build_tiles(cudaStream_t s, int32_t n, const int64_t* ptr, const int32_t* idx, int64_t nnz, int32_t gmaxn,
                TileSet& ts, DevPool& pool, int32_t* maxcnt_out) {
  constexpr int HS = 2048;
  const int32_t jmax = HS / 2;
  if (gmaxn > jmax) return MEGA_ERR_UNSUPPORTED;
  DevPool scratch(s);
  int16_t* slot_tmp = nullptr;
  int32_t* ovf = nullptr;
  MEGA_ALLOC(scratch, slot_tmp, nnz);
  MEGA_ALLOC(scratch, ovf, 1);
  for (int32_t R = 64; R >= 8; R >>= 1) {  // >= 8 keeps every block a whole warp
    const int64_t ntiles = (n + R - 1) / R;
    int32_t *jset = nullptr, *jcnt = nullptr;
    uint16_t* lidx = nullptr;
    DevPool trial;
    if (pool.ordered) trial.bind(pool.stream);
    MEGA_ALLOC(trial, jset, ntiles * jmax);
    MEGA_ALLOC(trial, jcnt, ntiles);
    MEGA_ALLOC(trial, lidx, nnz);
    MEGA_TRY(cudaMemsetAsync(ovf, 0, sizeof(int32_t), s));
    k_build_tiles<HS><<<(unsigned)ntiles, 256, 0, s>>>(n, R, ptr, idx, jmax, jset, jcnt, lidx, slot_tmp, ovf);
    MEGA_CHECK_LAUNCH();
    int32_t hovf = 0;
    MEGA_TRY(cudaMemcpyAsync(&hovf, ovf, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> hc(ntiles);
    MEGA_TRY(cudaMemcpyAsync(hc.data(), jcnt, sizeof(int32_t) * ntiles, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    if (hovf) continue;  // too many distinct neighbours: halve the tile
    int32_t mx = 0;
    for (int32_t v : hc) mx = std::max(mx, v);
    // the longest record range of any tile (sizes the streamed variants)
    int32_t* ent = nullptr;
    MEGA_ALLOC(scratch, ent, ntiles);
    k_tile_entries<<<grid_for(ntiles, 256), 256, 0, s>>>(n, R, ntiles, ptr, ent);
    MEGA_CHECK_LAUNCH();
    std::vector<int32_t> he(ntiles);
    MEGA_TRY(cudaMemcpyAsync(he.data(), ent, sizeof(int32_t) * ntiles, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    int32_t emax = 0;
    for (int32_t v : he) emax = std::max(emax, v);
    // keep the trial buffers: move ownership into the persistent pool
    pool.adopt(trial);
    ts.R = R;
    ts.ntiles = ntiles;
    ts.jmax = jmax;
    ts.maxcnt = mx;
    ts.recmax = emax;
    ts.jset = jset;
    ts.jcnt = jcnt;
    ts.lidx = lidx;
    if (maxcnt_out) *maxcnt_out = mx;
    return 0;
  }
  return MEGA_ERR_UNSUPPORTED;
}

int pack_transposed32(cudaStream_t s, int64_t m, const uint16_t* lidx, const float4* in, const int64_t* pos,
                      float4* out) {
  if (m <= 0) return 0;
  k_pack_t32<<<grid_for(m, 256), 256, 0, s>>>(m, lidx, in, pos, out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int pack_entries(cudaStream_t s, int64_t m, const uint16_t* lidx, const double* gx, const double* gy,
                 const double* gz, const int64_t* pos, bool f64, void* out) {
  if (m <= 0) return 0;
  if (f64) k_pack_f64<<<grid_for(m, 256), 256, 0, s>>>(m, lidx, gx, gy, gz, pos, (double2*)out);
  else k_pack_f32<<<grid_for(m, 256), 256, 0, s>>>(m, lidx, gx, gy, gz, pos, (float4*)out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int bank_order(cudaStream_t s, int32_t n, const TileSet& ts, const int64_t* ptr, uint16_t* lidx,
               const int64_t* pos_src, int64_t* pos, int lanes) {
  if (n <= 0) return 0;
  if ((lanes != 4 && lanes != 8) || ts.R * lanes < 32) return MEGA_ERR_UNSUPPORTED;
  const int64_t nwarps = ts.ntiles * (int64_t)(ts.R * lanes / 32);
  const unsigned grid = (unsigned)((nwarps * 32 + 127) / 128);
  if (lanes == 4) k_bank_order<4, 32, 32><<<grid, 128, 0, s>>>(n, ts.R, nwarps, ptr, lidx, pos_src, pos);
  else k_bank_order<8, 32, 32><<<grid, 128, 0, s>>>(n, ts.R, nwarps, ptr, lidx, pos_src, pos);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int iota64(cudaStream_t s, int64_t m, int64_t* out) {
  if (m <= 0) return 0;
  k_iota64<<<grid_for(m, 256), 256, 0, s>>>(m, out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int record_ranks(cudaStream_t s, int64_t m, const float4* rec, uint16_t* out) {
  if (m <= 0) return 0;
  k_rec_ranks<<<grid_for(m, 256), 256, 0, s>>>(m, rec, out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int gather_f6(cudaStream_t s, int64_t m, const int64_t* pos, const float* in, float* out) {
  if (m <= 0) return 0;
  k_gather_f6<<<grid_for(m, 256), 256, 0, s>>>(m, pos, (const float2*)in, (float2*)out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

int gather_records32(cudaStream_t s, int64_t m, const int64_t* pos, const float4* in, float4* out) {
  if (m <= 0) return 0;
  k_gather_rec32<<<grid_for(m, 256), 256, 0, s>>>(m, pos, in, out);
  MEGA_CHECK_LAUNCH();
  return 0;
}

// The launch variants, in the order the autotuner tries them:
// (KG, KU) = (4, 4), (4, 2), (4, 1), (8, 2) with register-held record
// streams, then KG = 4, 8 with the records streamed into shared memory, then
// (16, 1), (16, 2) with register-held streams (four times the threads per
// staged neighbour of KG = 4: the NSNI force gather stages 27 values a node).
constexpr int kVariants = kTiledVariants;
// dynamic shared memory a streamed-variant block may ask for: sm_100's 227 KB
// per block less room for the kernels' static shared memory (under 1 KB)
constexpr int kBulkSmemMax = 227 * 1024 - 1024;

template <typename K>
static int raise_smem(K k, int lim) {
  MEGA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  return 0;
}

template <int KG, int KU>
static int configure_variant(int lim) {
  int r = 0;
  if ((r = raise_smem(k_defgrad_t<float, false, true, KG, KU>, lim))) return r;
  if ((r = raise_smem(k_defgrad_t<float, false, false, KG, KU>, lim))) return r;
  if ((r = raise_smem(k_defgrad_t<float, false, true, KG, KU, true>, lim))) return r;
  if ((r = raise_smem(k_defgrad_t<float, false, false, KG, KU, true>, lim))) return r;
  if ((r = raise_smem(k_defgrad_t<double, true, true, KG, KU>, lim))) return r;
  if ((r = raise_smem(k_defgrad_t<double, true, false, KG, KU>, lim))) return r;
  if ((r = raise_smem(k_force_t<float, float, false, KG, KU>, lim))) return r;
  if ((r = raise_smem(k_force_t<float, float, false, KG, KU, true>, lim))) return r;
  return raise_smem(k_force_t<double, double, true, KG, KU>, lim);
}

static int g_bulk_lim = kBulkSmemMax;  // what the device grants, set by configure_tiled_kernels

template <typename K>
static int raise_smem_upto(K k, int lim) {
  cudaFuncAttributes fa{};
  MEGA_TRY(cudaFuncGetAttributes(&fa, k));
  const int room = lim - (int)fa.sharedSizeBytes;
  g_bulk_lim = std::min(g_bulk_lim, room);
  return raise_smem(k, room);
}

template <int KG>
static int configure_bulk(int lim) {
  int dev = 0, optin = 0;
  MEGA_TRY(cudaGetDevice(&dev));
  MEGA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  lim = std::min(lim + 1024, optin);  // the kernels' static shared memory comes off this
  int r = 0;
  if ((r = raise_smem_upto(k_defgrad_b<float, false, true, KG>, lim))) return r;
  if ((r = raise_smem_upto(k_defgrad_b<float, false, false, KG>, lim))) return r;
  if ((r = raise_smem_upto(k_defgrad_b<double, true, true, KG>, lim))) return r;
  if ((r = raise_smem_upto(k_defgrad_b<double, true, false, KG>, lim))) return r;
  if ((r = raise_smem_upto(k_force_b<float, float, false, KG>, lim))) return r;
  return raise_smem_upto(k_force_b<double, double, true, KG>, lim);
}

// Raise the dynamic shared-memory limit of the tiled kernels once (outside
// any stream capture): a tile stages at most 1024 neighbours, 96 KB for the
// double-precision T_i of the force kernel (120 KB for the float T_i and
// NSNI weights); the streamed variants add the tile's records.
int configure_tiled_kernels() {
  static bool done = false;
  if (done) return 0;
  const int lim = 30 * 4 * 1024 + 1024;
  int r = 0;
  if ((r = configure_variant<4, 4>(lim)) || (r = configure_variant<4, 2>(lim)) ||
      (r = configure_variant<4, 1>(lim)) || (r = configure_variant<8, 2>(lim)) ||
      (r = configure_variant<16, 1>(lim)) || (r = configure_variant<16, 2>(lim)) ||
      (r = configure_bulk<4>(kBulkSmemMax)) || (r = configure_bulk<8>(kBulkSmemMax)))
    return r;
  done = true;
  return 0;
}

int tiled_variants() { return kVariants; }

bool tiled_variant_fits(const TileSet& ts, bool mixed, int variant, bool force, bool has_body) {
  if (variant < 0 || variant >= kVariants) return false;
  if (variant < 4 || variant > 5) return true;  // register variants
  const size_t stage = force ? (mixed ? sizeof(float) : sizeof(double)) * (has_body ? 12 : 9) : (mixed ? 24 : 48);
  return (size_t)ts.recmax * (mixed ? 16 : 32) + stage * (size_t)ts.maxcnt <= (size_t)g_bulk_lim;
}

template <int KG>
static int defgrad_bulk(cudaStream_t s, bool mixed, bool interp, int32_t n, const TileSet& ts,
                        const int64_t* rowptr, const void* pk, const double* dsp, const double* dsp_tot,
                        const double* sdphi, const double* shp, double* dsp_tot_phy, double* fg, StepAccum* acc,
                        unsigned* status) {
  const size_t smem = (size_t)ts.recmax * (mixed ? 16 : 32) + (mixed ? 24 : 48) * (size_t)ts.maxcnt;
  if (smem > (size_t)g_bulk_lim) return MEGA_ERR_UNSUPPORTED;
  const unsigned grid = (unsigned)ts.ntiles;
  const int block = ts.R * KG;
  if (mixed) {
    auto k = interp ? k_defgrad_b<float, false, true, KG> : k_defgrad_b<float, false, false, KG>;
    k<<<grid, block, smem, s>>>(n, ts.R, ts.jmax, ts.recmax, rowptr, pk, ts.jset, ts.jcnt, dsp, dsp_tot, sdphi, shp,
                                dsp_tot_phy, fg, acc, status);
  } else {
    auto k = interp ? k_defgrad_b<double, true, true, KG> : k_defgrad_b<double, true, false, KG>;
    k<<<grid, block, smem, s>>>(n, ts.R, ts.jmax, ts.recmax, rowptr, pk, ts.jset, ts.jcnt, dsp, dsp_tot, sdphi, shp,
                                dsp_tot_phy, fg, acc, status);
  }
  return 0;
}

template <int KG, int KU>
static void defgrad_variant(cudaStream_t s, bool mixed, bool interp, int32_t n, const TileSet& ts,
                            const NsniTiles* ns, const int64_t* rowptr, const void* pk, const double* dsp,
                            const double* dsp_tot, const double* sdphi, const double* shp, double* dsp_tot_phy,
                            double* fg, StepAccum* acc) {
  const size_t smem = (mixed ? 24 : 48) * (size_t)ts.maxcnt;
  const unsigned grid = (unsigned)ts.ntiles;
  const int block = ts.R * KG;
  const NsniTiles nz = ns ? *ns : NsniTiles();
  if (mixed) {
    auto k = ns ? (interp ? k_defgrad_t<float, false, true, KG, KU, true> : k_defgrad_t<float, false, false, KG, KU, true>)
                : (interp ? k_defgrad_t<float, false, true, KG, KU> : k_defgrad_t<float, false, false, KG, KU>);
    k<<<grid, block, smem, s>>>(n, ts.R, ts.jmax, nz, rowptr, pk, ts.jset, ts.jcnt, dsp, dsp_tot, sdphi, shp,
                                dsp_tot_phy, fg, acc);
  } else {
    auto k = interp ? k_defgrad_t<double, true, true, KG, KU> : k_defgrad_t<double, true, false, KG, KU>;
    k<<<grid, block, smem, s>>>(n, ts.R, ts.jmax, nz, rowptr, pk, ts.jset, ts.jcnt, dsp, dsp_tot, sdphi, shp,
                                dsp_tot_phy, fg, acc);
  }
}

int launch_defgrad_tiled(cudaStream_t s, bool mixed, bool interp, int32_t n, const TileSet& ts,
                         const NsniTiles* ns, const int64_t* rowptr, const void* pk, const double* dsp,
                         const double* dsp_tot, const double* sdphi, const double* shp, double* dsp_tot_phy,
                         double* fg, StepAccum* acc, unsigned* status, int variant) {
  int r = 0;
  if (ns && (!mixed || variant == 4 || variant == 5)) return MEGA_ERR_UNSUPPORTED;  // NSNI: register variants
  switch (variant) {
    case 4: r = defgrad_bulk<4>(s, mixed, interp, n, ts, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc,
                                status);
      break;
    case 5: r = defgrad_bulk<8>(s, mixed, interp, n, ts, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc,
                                status);
      break;
    case 1: defgrad_variant<4, 2>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc);
      break;
    case 2: defgrad_variant<4, 1>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc);
      break;
    case 3: defgrad_variant<8, 2>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg, acc);
      break;
    case 6: defgrad_variant<16, 1>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg,
                                   acc);
      break;
    case 7: defgrad_variant<16, 2>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg,
                                   acc);
      break;
    default: defgrad_variant<4, 4>(s, mixed, interp, n, ts, ns, rowptr, pk, dsp, dsp_tot, sdphi, shp, dsp_tot_phy, fg,
                                   acc);
  }
  if (r) return r;
  MEGA_CHECK_LAUNCH();
  return 0;
}

template <int KG>
static int force_bulk(cudaStream_t s, bool mixed, const TiledForceArgs& a) {
  const int nv = a.has_body ? 12 : 9;
  const size_t smem = (size_t)a.recmax * (mixed ? 16 : 32) + (mixed ? sizeof(float) : sizeof(double)) * nv *
                      (size_t)a.maxcnt;
  if (smem > (size_t)g_bulk_lim) return MEGA_ERR_UNSUPPORTED;
  const unsigned grid = (unsigned)a.ntiles;
  const int block = a.R * KG;
  if (mixed) k_force_b<float, float, false, KG><<<grid, block, smem, s>>>(a);
  else k_force_b<double, double, true, KG><<<grid, block, smem, s>>>(a);
  return 0;
}

template <int KG, int KU>
static void force_variant(cudaStream_t s, bool mixed, const TiledForceArgs& a) {
  const int nv = (a.has_body ? 12 : 9) + (a.ns_scol ? 18 : 0);
  const size_t smem = (mixed ? sizeof(float) : sizeof(double)) * nv * (size_t)a.maxcnt;
  const unsigned grid = (unsigned)a.ntiles;
  const int block = a.R * KG;
  if (mixed && a.ns_scol) k_force_t<float, float, false, KG, KU, true><<<grid, block, smem, s>>>(a);
  else if (mixed) k_force_t<float, float, false, KG, KU><<<grid, block, smem, s>>>(a);
  else k_force_t<double, double, true, KG, KU><<<grid, block, smem, s>>>(a);
}

int launch_force_tiled(cudaStream_t s, bool mixed, const TiledForceArgs& a, int variant) {
  int r = 0;
  if (a.ns_scol && (!mixed || variant == 4 || variant == 5)) return MEGA_ERR_UNSUPPORTED;  // NSNI: register variants
  switch (variant) {
    case 1: force_variant<4, 2>(s, mixed, a); break;
    case 2: force_variant<4, 1>(s, mixed, a); break;
    case 3: force_variant<8, 2>(s, mixed, a); break;
    case 6: force_variant<16, 1>(s, mixed, a); break;
    case 7: force_variant<16, 2>(s, mixed, a); break;
    case 4: r = force_bulk<4>(s, mixed, a); break;
    case 5: r = force_bulk<8>(s, mixed, a); break;
    default: force_variant<4, 4>(s, mixed, a);
  }
  if (r) return r;
  MEGA_CHECK_LAUNCH();
  return 0;
}

}  // namespace mega
