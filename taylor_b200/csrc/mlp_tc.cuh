// mlp_tc.cuh -- warp-level inference of the 4 -> 64 -> 64 -> 1 surrogate with
// the 64x64 layer on the tensor cores (mma.sync m16n8k16, bf16 operands, fp32
// accumulation).  Shared by the learned stress kernel and the standalone
// evaluation entry, so the layout below is tested on its own.
//
// Shared-memory image of the network (MlpSmem):
//   W2  [out][in] bf16, rows padded to kMlpLd (72) elements: the fragment
//       loads of 8 rows x 4 lanes then hit 32 distinct banks;
//   P   fp32: W1 (64x4, row-major by output), b1 (64), b2 (64), W3 (64), b3.
// Per warp, 32 x kMlpLd bf16 of scratch holds the lanes' first hidden layers
// (row = lane) and 32 floats the outputs.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace mega {

constexpr int kMlpH = 64;
constexpr int kMlpLd = 72;
constexpr int kMlpSmall = 4 * kMlpH + 3 * kMlpH + 1;  // 449

struct MlpSmem {
  uint16_t W2[kMlpH * kMlpLd];
  float P[kMlpSmall + 3];
};

__device__ __forceinline__ void mma_16816_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// hardware tanh (one SFU instruction, max error about 2^-11): the network
// runs in bf16 anyway, and training uses the accurate tanhf
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint32_t bf16_bits(float f) {
  const __nv_bfloat16 b = __float2bfloat16_rn(f);
  return (uint32_t) * reinterpret_cast<const uint16_t*>(&b);
}

// Block-cooperative copy of the packed network (w2: 64x64 bf16 bits, small:
// kMlpSmall floats) into shared memory; the caller synchronises.
__device__ __forceinline__ void mlp_load(MlpSmem& m, const uint16_t* __restrict__ w2,
                                         const float* __restrict__ small) {
  for (int e = threadIdx.x; e < kMlpH * kMlpH; e += blockDim.x) m.W2[(e >> 6) * kMlpLd + (e & 63)] = w2[e];
  for (int e = threadIdx.x; e < kMlpSmall; e += blockDim.x) m.P[e] = small[e];
}

// Warp-collective: every lane passes its 4 features (on = false gives a zero
// hidden row and an unused output) and receives the network output.  All 32
// lanes must call it together.
__device__ __forceinline__ float warp_mlp(const float x[4], bool on, const MlpSmem& m, uint16_t* __restrict__ hw,
                                          float* __restrict__ out) {
  const float* W1 = m.P;
  const float* b1 = m.P + 4 * kMlpH;
  const float* b2 = m.P + 5 * kMlpH;
  const float* W3 = m.P + 6 * kMlpH;
  const float b3 = m.P[7 * kMlpH];
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  // layer 1 on the CUDA cores, stored as this lane's bf16 row
  uint16_t* row = hw + lane * kMlpLd;
#pragma unroll 4
  for (int o = 0; o < kMlpH; o += 2) {
    float h0 = 0.f, h1 = 0.f;
    if (on) {
      h0 = tanh_sfu(b1[o] + W1[4 * o] * x[0] + W1[4 * o + 1] * x[1] + W1[4 * o + 2] * x[2] +
                    W1[4 * o + 3] * x[3]);
      h1 = tanh_sfu(b1[o + 1] + W1[4 * o + 4] * x[0] + W1[4 * o + 5] * x[1] + W1[4 * o + 6] * x[2] +
                    W1[4 * o + 7] * x[3]);
    }
    *reinterpret_cast<uint32_t*>(row + o) = bf16_bits(h0) | (bf16_bits(h1) << 16);
  }
  __syncwarp();
  // layer 2: D[32 x 64] = H1[32 x 64] W2^T, as 2 (M) x 8 (N) tiles of 16x8,
  // K = 64 in 4 steps of 16.  A fragment (row-major 16x16): a0 = (g, 2t..2t+1),
  // a1 = (g+8, 2t..), a2 = (g, 2t+8..), a3 = (g+8, 2t+8..); B fragment
  // (col-major 16x8, column n = output neuron): b0 = (k 2t..2t+1, n g),
  // b1 = (k 2t+8.., n g); C: c0,c1 = (g, 2t..2t+1), c2,c3 = (g+8, 2t..).
  uint32_t af[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const uint16_t* r0 = hw + (mt * 16 + g) * kMlpLd + ks * 16 + 2 * tq;
      const uint16_t* r1 = r0 + 8 * kMlpLd;
      af[mt][ks][0] = *reinterpret_cast<const uint32_t*>(r0);
      af[mt][ks][1] = *reinterpret_cast<const uint32_t*>(r1);
      af[mt][ks][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
      af[mt][ks][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
    }
  // tanh(D + b2) . W3 folded into the epilogue, one partial per row half
  float rs[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    uint32_t bf[4][2];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const uint16_t* q = m.W2 + (nt * 8 + g) * kMlpLd + ks * 16 + 2 * tq;
      bf[ks][0] = *reinterpret_cast<const uint32_t*>(q);
      bf[ks][1] = *reinterpret_cast<const uint32_t*>(q + 8);
    }
    const int c0 = nt * 8 + 2 * tq;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) mma_16816_bf16(c, af[mt][ks], bf[ks]);
      rs[mt][0] += tanh_sfu(c[0] + b2[c0]) * W3[c0] + tanh_sfu(c[1] + b2[c0 + 1]) * W3[c0 + 1];
      rs[mt][1] += tanh_sfu(c[2] + b2[c0]) * W3[c0] + tanh_sfu(c[3] + b2[c0 + 1]) * W3[c0 + 1];
    }
  }
  // the 4 lanes of a quad hold the 4 column pairs of the same rows
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      rs[mt][h] += __shfl_xor_sync(0xffffffffu, rs[mt][h], 1);
      rs[mt][h] += __shfl_xor_sync(0xffffffffu, rs[mt][h], 2);
    }
  if (tq == 0) {
    out[g] = rs[0][0] + b3;
    out[g + 8] = rs[0][1] + b3;
    out[16 + g] = rs[1][0] + b3;
    out[24 + g] = rs[1][1] + b3;
  }
  __syncwarp();
  const float y = out[lane];
  __syncwarp();  // hw / out may be rewritten by the next call
  return y;
}

}  // namespace mega
