// mlp.cu -- the surrogate network that starts the rate-dependent return
// mapping (no reference counterpart).
//
// A 4 -> 64 -> 64 -> 1 perceptron, tanh hidden layers, linear output,
// parameters packed [W1 (64x4), b1 (64), W2 (64x64), b2 (64), W3 (64), b3]
// row-major (out, in).  It maps the trial state of a plastic node to the
// converged plastic multiplier as a fraction of the perfectly plastic
// estimate, y = dgamma * 2 mu / f_trial (see rate_features in force.cu).
// Training data are logged by the plain Newton solver; training runs here
// with hand-written forward / backward / Adam kernels (Kingma & Ba 2015) in
// FP32; inference (force.cu) uses the weights rounded to bf16 with the 64x64
// layer on the tensor cores (mma.sync bf16, fp32 accumulation).
#include <algorithm>
#include <cmath>
#include <vector>
#include "mega_internal.cuh"
#include "mlp_tc.cuh"

namespace mega {
namespace {

constexpr int H = 64;
constexpr int NP = H * 4 + H + H * H + H + H + 1;  // 4545
constexpr int kB = 128;                           // samples per block
constexpr int LD = H + 1;                         // padded row of the activation tiles

struct Off {
  static constexpr int W1 = 0, B1 = H * 4, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H;
};

// Forward + backward of one block of samples; gradients summed over the block
// and added to grad; loss accumulates 0.5 r^2 / nb.
// Sample q has features X[xs q .. xs q + 3] and target T[ts q].
__global__ void __launch_bounds__(kB) k_mlp_grad(int64_t nb, int64_t s0, const int64_t* __restrict__ order,
                                                 const float* __restrict__ theta, const float* __restrict__ X, int xs,
                                                 const float* __restrict__ T, int ts, float inv_nb,
                                                 float* __restrict__ grad, float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* th = sm;                 // NP
  float* H1 = th + NP + 3;        // [kB][LD]
  float* D2 = H1 + kB * LD;       // [kB][LD]
  float* D1 = D2 + kB * LD;       // [kB][LD]
  float* G2 = D1 + kB * LD;       // [kB][LD] go * h2
  float* XS = G2 + kB * LD;       // [kB][4]
  float* GO = XS + kB * 4;        // [kB]
  const int tid = threadIdx.x;
  for (int k = tid; k < NP; k += kB) th[k] = theta[k];
  const int64_t s = blockIdx.x * (int64_t)kB + tid;
  const bool act = s < nb;
  float x[4] = {0.f, 0.f, 0.f, 0.f}, t = 0.f;
  if (act) {
    const int64_t q = order ? order[s0 + s] : s0 + s;
    x[0] = X[xs * q]; x[1] = X[xs * q + 1]; x[2] = X[xs * q + 2]; x[3] = X[xs * q + 3];
    t = T[ts * q];
  }
  XS[4 * tid] = x[0]; XS[4 * tid + 1] = x[1]; XS[4 * tid + 2] = x[2]; XS[4 * tid + 3] = x[3];
  __syncthreads();
  float* h1 = H1 + tid * LD;
  float* d2 = D2 + tid * LD;
  float* d1 = D1 + tid * LD;
  float* g2 = G2 + tid * LD;
  for (int o = 0; o < H; ++o) {
    const float* w = th + Off::W1 + 4 * o;
    h1[o] = tanhf(th[Off::B1 + o] + w[0] * x[0] + w[1] * x[1] + w[2] * x[2] + w[3] * x[3]);
  }
  float out = th[Off::B3];
  for (int o = 0; o < H; ++o) {
    const float* w = th + Off::W2 + H * o;
    float a = th[Off::B2 + o];
    for (int k = 0; k < H; ++k) a += w[k] * h1[k];
    const float h2 = tanhf(a);
    g2[o] = h2;  // h2 kept here until go is known
    out += th[Off::W3 + o] * h2;
  }
  const float r = act ? out - t : 0.f;
  const float go = r * inv_nb;
  GO[tid] = go;
  if (act) atomicAdd(loss, 0.5f * r * r * inv_nb);
  for (int o = 0; o < H; ++o) {
    const float h2 = g2[o];
    d2[o] = go * th[Off::W3 + o] * (1.f - h2 * h2);
    g2[o] = go * h2;
  }
  for (int k = 0; k < H; ++k) {
    float a = 0.f;
    for (int o = 0; o < H; ++o) a += th[Off::W2 + H * o + k] * d2[o];
    d1[k] = a * (1.f - h1[k] * h1[k]);
  }
  __syncthreads();
  // block sums of the parameter gradients (each thread owns a set of outputs)
  for (int e = tid; e < H * H; e += kB) {  // dW2[o][k] = sum_s d2[s][o] h1[s][k]
    const int o = e / H, k = e - o * H;
    float a = 0.f;
    for (int q = 0; q < kB; ++q) a += D2[q * LD + o] * H1[q * LD + k];
    atomicAdd(&grad[Off::W2 + e], a);
  }
  for (int e = tid; e < H * 4; e += kB) {  // dW1[o][k] = sum_s d1[s][o] x[s][k]
    const int o = e / 4, k = e - o * 4;
    float a = 0.f;
    for (int q = 0; q < kB; ++q) a += D1[q * LD + o] * XS[4 * q + k];
    atomicAdd(&grad[Off::W1 + e], a);
  }
  if (tid < H) {
    float b1 = 0.f, b2 = 0.f, w3 = 0.f;
    for (int q = 0; q < kB; ++q) {
      b1 += D1[q * LD + tid];
      b2 += D2[q * LD + tid];
      w3 += G2[q * LD + tid];
    }
    atomicAdd(&grad[Off::B1 + tid], b1);
    atomicAdd(&grad[Off::B2 + tid], b2);
    atomicAdd(&grad[Off::W3 + tid], w3);
  }
  if (tid == 0) {
    float b3 = 0.f;
    for (int q = 0; q < kB; ++q) b3 += GO[q];
    atomicAdd(&grad[Off::B3], b3);
  }
}

__global__ void k_adam(int np, float* __restrict__ theta, float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  grad[i] = 0.f;
}

__global__ void k_mlp_eval(int64_t n, const float* __restrict__ theta, const float* __restrict__ X,
                           float* __restrict__ Y) {
  __shared__ float th[NP];
  for (int k = threadIdx.x; k < NP; k += blockDim.x) th[k] = theta[k];
  __syncthreads();
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float x0 = X[4 * s], x1 = X[4 * s + 1], x2 = X[4 * s + 2], x3 = X[4 * s + 3];
  float h1[H];
  for (int o = 0; o < H; ++o) {
    const float* w = th + Off::W1 + 4 * o;
    h1[o] = tanhf(th[Off::B1 + o] + w[0] * x0 + w[1] * x1 + w[2] * x2 + w[3] * x3);
  }
  float out = th[Off::B3];
  for (int o = 0; o < H; ++o) {
    const float* w = th + Off::W2 + H * o;
    float a = th[Off::B2 + o];
    for (int k = 0; k < H; ++k) a += w[k] * h1[k];
    out += th[Off::W3 + o] * tanhf(a);
  }
  Y[s] = out;
}

// The inference form used by the learned stress kernel (bf16 W2 on the
// tensor cores), for testing it on its own.
__global__ void __launch_bounds__(128) k_mlp_eval_tc(int64_t n, const uint16_t* __restrict__ w2,
                                                     const float* __restrict__ small, const float* __restrict__ X,
                                                     float* __restrict__ Y) {
  __shared__ __align__(16) MlpSmem net;
  __shared__ __align__(16) uint16_t sH1[128 * kMlpLd];
  __shared__ float sOut[128];
  mlp_load(net, w2, small);
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += nwarps * 32) {
    const int64_t s = base + lane;
    float x[4] = {0.f, 0.f, 0.f, 0.f};
    if (s < n) { x[0] = X[4 * s]; x[1] = X[4 * s + 1]; x[2] = X[4 * s + 2]; x[3] = X[4 * s + 3]; }
    const float y = warp_mlp(x, s < n, net, sH1 + wid * 32 * kMlpLd, sOut + wid * 32);
    if (s < n) Y[s] = y;
  }
}

// theta (fp32, packed as above) -> W2 as bf16 bits + the fp32 small parameters
__global__ void k_mlp_pack(const float* __restrict__ theta, uint16_t* __restrict__ w2, float* __restrict__ small) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < H * H + kMlpSmall; e += gridDim.x * blockDim.x) {
    if (e < H * H) {
      w2[e] = (uint16_t)bf16_bits(theta[Off::W2 + e]);
    } else {
      const int k = e - H * H;  // small = W1, b1, b2, W3, b3
      int src;
      if (k < 4 * H + H) src = k;                 // W1, b1
      else if (k < 4 * H + 2 * H) src = Off::B2 + (k - 5 * H);
      else if (k < 4 * H + 3 * H) src = Off::W3 + (k - 6 * H);
      else src = Off::B3;
      small[k] = theta[src];
    }
  }
}

// order[k] = (a k + b) mod n with gcd(a, n) = 1: a cheap per-epoch shuffle
__global__ void k_shuffle(int64_t n, uint64_t a, uint64_t b, int64_t* __restrict__ order) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < n) order[k] = (int64_t)((a * (uint64_t)k + b) % (uint64_t)n);
}

size_t grad_smem() { return sizeof(float) * (NP + 3 + 4 * kB * LD + kB * 4 + kB); }

uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) { const uint64_t t = a % b; a = b; b = t; }
  return a;
}

}  // namespace

int mlp_nparams() { return NP; }

int mlp_pack(cudaStream_t s, const float* dtheta, uint16_t* w2, float* small) {
  k_mlp_pack<<<(H * H + kMlpSmall + 255) / 256, 256, 0, s>>>(dtheta, w2, small);
  MEGA_CHECK_LAUNCH();
  return 0;
}

// Mini-batch Adam (Kingma & Ba 2015, beta 0.9 / 0.999, eps 1e-8) over ns
// device-resident samples; dth (NP floats, device) is updated in place and
// loss_host (epochs floats, or null) receives each epoch's mean batch loss.
int mlp_train_dev(cudaStream_t s, float* dth, int64_t ns, const float* X, int xs, const float* T, int ts,
                  int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss_host) {
  static_assert(H == kMlpH, "inference and training widths differ");
  DevPool pool(s);
  float *dg, *dm, *dv, *dl;
  int64_t* order;
  MEGA_ALLOC(pool, dg, NP);
  MEGA_ALLOC(pool, dm, NP);
  MEGA_ALLOC(pool, dv, NP);
  MEGA_ALLOC(pool, dl, epochs);
  MEGA_ALLOC(pool, order, ns);
  MEGA_TRY(cudaMemsetAsync(dg, 0, sizeof(float) * NP, s));
  MEGA_TRY(cudaMemsetAsync(dm, 0, sizeof(float) * NP, s));
  MEGA_TRY(cudaMemsetAsync(dv, 0, sizeof(float) * NP, s));
  MEGA_TRY(cudaMemsetAsync(dl, 0, sizeof(float) * epochs, s));
  const size_t sm = grad_smem();
  MEGA_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  uint64_t rng = seed * 6364136223846793005ull + 1442695040888963407ull;
  int step = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  const int64_t nbatches = (ns + batch - 1) / batch;
  for (int32_t ep = 0; ep < epochs; ++ep) {
    rng = rng * 6364136223846793005ull + 1442695040888963407ull;
    uint64_t a = (rng >> 17) % (uint64_t)ns + 1;
    while (gcd64(a, (uint64_t)ns) != 1) a = a % (uint64_t)ns + 1;
    rng = rng * 6364136223846793005ull + 1442695040888963407ull;
    k_shuffle<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(ns, a, rng >> 11, order);
    for (int64_t b0 = 0; b0 < ns; b0 += batch) {
      const int64_t nb = std::min<int64_t>(batch, ns - b0);
      k_mlp_grad<<<(unsigned)((nb + kB - 1) / kB), kB, sm, s>>>(nb, b0, order, dth, X, xs, T, ts,
                                                                1.0f / (float)nb, dg, dl + ep);
      ++step;
      const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
      k_adam<<<(NP + 255) / 256, 256, 0, s>>>(NP, dth, dg, dm, dv, lr, b1, b2, 1e-8f, c1, c2);
    }
    MEGA_CHECK_LAUNCH();
  }
  if (loss_host) {
    MEGA_TRY(cudaMemcpyAsync(loss_host, dl, sizeof(float) * epochs, cudaMemcpyDeviceToHost, s));
  }
  MEGA_TRY(cudaStreamSynchronize(s));
  if (loss_host)
    for (int32_t ep = 0; ep < epochs; ++ep) loss_host[ep] /= (float)nbatches;
  return 0;
}

}  // namespace mega

using namespace mega;

extern "C" {

int mega_mlp_nparams(int32_t hidden) { return hidden == H ? NP : MEGA_ERR_UNSUPPORTED; }

int mega_mlp_grad(int32_t hidden, const float* theta, int64_t nb, const float* x, const float* t, float* grad,
                  float* loss) {
  if (hidden != H) return MEGA_ERR_UNSUPPORTED;
  if (!theta || nb <= 0 || !x || !t || !grad || !loss) return MEGA_ERR_ARG;
  DevPool pool;
  float *dth, *dx, *dt, *dg, *dl;
  MEGA_ALLOC(pool, dth, NP);
  MEGA_ALLOC(pool, dx, 4 * nb);
  MEGA_ALLOC(pool, dt, nb);
  MEGA_ALLOC(pool, dg, NP);
  MEGA_ALLOC(pool, dl, 1);
  MEGA_TRY(cudaMemcpy(dth, theta, sizeof(float) * NP, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemcpy(dx, x, sizeof(float) * 4 * nb, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemcpy(dt, t, sizeof(float) * nb, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemset(dg, 0, sizeof(float) * NP));
  MEGA_TRY(cudaMemset(dl, 0, sizeof(float)));
  const size_t sm = grad_smem();
  MEGA_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_mlp_grad<<<(unsigned)((nb + kB - 1) / kB), kB, sm>>>(nb, 0, nullptr, dth, dx, 4, dt, 1, 1.0f / (float)nb, dg,
                                                         dl);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaMemcpy(grad, dg, sizeof(float) * NP, cudaMemcpyDeviceToHost));
  MEGA_TRY(cudaMemcpy(loss, dl, sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int mega_mlp_eval(int32_t hidden, const float* theta, int64_t n, const float* x, float* y, int32_t tensor_cores) {
  if (hidden != H) return MEGA_ERR_UNSUPPORTED;
  if (!theta || n <= 0 || !x || !y) return MEGA_ERR_ARG;
  DevPool pool;
  float *dth, *dx, *dy, *small;
  uint16_t* w2;
  MEGA_ALLOC(pool, dth, NP);
  MEGA_ALLOC(pool, dx, 4 * n);
  MEGA_ALLOC(pool, dy, n);
  MEGA_ALLOC(pool, w2, H * H);
  MEGA_ALLOC(pool, small, kMlpSmall);
  MEGA_TRY(cudaMemcpy(dth, theta, sizeof(float) * NP, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemcpy(dx, x, sizeof(float) * 4 * n, cudaMemcpyHostToDevice));
  if (tensor_cores) {
    int r = mlp_pack(0, dth, w2, small);
    if (r) return r;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 127) / 128, (int64_t)device_sm_count() * 8);
    k_mlp_eval_tc<<<grid, 128>>>(n, w2, small, dx, dy);
  } else {
    k_mlp_eval<<<(unsigned)((n + 127) / 128), 128>>>(n, dth, dx, dy);
  }
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaMemcpy(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return 0;
}

// Mini-batch Adam on the GPU.  theta (NP floats) in/out; ns samples x (ns,4),
// t (ns); loss_per_epoch (epochs) out, the mean of the batch losses.
int mega_mlp_train(int32_t hidden, float* theta, int64_t ns, const float* x, const float* t, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float* loss_per_epoch) {
  if (hidden != H) return MEGA_ERR_UNSUPPORTED;
  if (!theta || ns <= 0 || !x || !t || epochs <= 0 || batch <= 0) return MEGA_ERR_ARG;
  DevPool pool;
  float *dth, *dx, *dt;
  MEGA_ALLOC(pool, dth, NP);
  MEGA_ALLOC(pool, dx, 4 * ns);
  MEGA_ALLOC(pool, dt, ns);
  MEGA_TRY(cudaMemcpy(dth, theta, sizeof(float) * NP, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemcpy(dx, x, sizeof(float) * 4 * ns, cudaMemcpyHostToDevice));
  MEGA_TRY(cudaMemcpy(dt, t, sizeof(float) * ns, cudaMemcpyHostToDevice));
  int r = mlp_train_dev(0, dth, ns, dx, 4, dt, 1, epochs, batch, lr, seed, loss_per_epoch);
  if (r) return r;
  MEGA_TRY(cudaMemcpy(theta, dth, sizeof(float) * NP, cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
