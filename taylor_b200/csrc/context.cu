// context.cu -- the C ABI of libmega_gpu.so: resident context (the whole
// MAIN.F90:304-658 time loop on the device, captured in CUDA graphs) and the
// copy-in/copy-out drop-ins for the reference's subroutines.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>
#include "mega_internal.cuh"
#include "tiled.cuh"

namespace mega {

static thread_local char g_err[512] = {0};
void record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  snprintf(g_err, sizeof(g_err), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}
const char* last_error_text() { return g_err; }
void record_error_text(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

namespace {

__global__ void k_gather_pos(int64_t m, const int64_t* __restrict__ pos, const double* __restrict__ src,
                             double* __restrict__ dst) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m) dst[e] = src[pos[e]];
}
// row sums of the stored gradients: sum_J grad0 phi_iJ (FP64 of the values
// as stored, so the split sum of k_defgrad is exact in exact arithmetic)
template <typename G>
__global__ void k_rowsum3(int32_t n, const int64_t* __restrict__ rowptr, const G* __restrict__ gx,
                          const G* __restrict__ gy, const G* __restrict__ gz, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
    a += (double)gx[p]; b += (double)gy[p]; c += (double)gz[p];
  }
  out[3 * i] = a; out[3 * i + 1] = b; out[3 * i + 2] = c;
}
__global__ void k_hw(int32_t n, const double* __restrict__ lmat, double* __restrict__ rot,
                     double* __restrict__ strain, double* __restrict__ d, int exact) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double L[3][3], R[3][3], s6[6], d6[6];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) L[r][c] = lmat[9 * i + 3 * c + r];
  hughes_winget(L, R, s6, d6, exact != 0);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) rot[9 * i + 3 * c + r] = R[r][c];
  for (int k = 0; k < 6; ++k) { strain[6 * i + k] = s6[k]; d[6 * i + k] = d6[k]; }
}
__global__ void k_rotate(int32_t n, const double* __restrict__ rot, double* __restrict__ v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double R[3][3], s[6];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) R[r][c] = rot[9 * i + 3 * c + r];
  for (int k = 0; k < 6; ++k) s[k] = v[6 * i + k];
  rotate_tensor(R, s);
  for (int k = 0; k < 6; ++k) v[6 * i + k] = s[k];
}
__global__ void k_constitution(int32_t n, const double* __restrict__ spred, const int32_t* __restrict__ mat,
                               const double* __restrict__ props, double dlt, int maxit, int solver, double rtol,
                               double* __restrict__ state, double* __restrict__ stress, int32_t* __restrict__ iters,
                               unsigned* __restrict__ status) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* pr = props + 30 * i;
  NodeMat m;
  m.type = mat[i]; m.nu = pr[0]; m.E = pr[1]; m.rho = pr[2]; m.sig0 = pr[3]; m.B = pr[4]; m.C = pr[5];
  m.p7 = pr[6]; m.p8 = pr[7]; m.lam = pr[27]; m.mu = pr[28]; m.l2m = pr[29];
  double sp[6], out[6];
  for (int k = 0; k < 6; ++k) sp[k] = spred[6 * i + k];
  double ep = state[20 * i + 2];
  bool cap = false;
  int it = 0;
  if (m.type == MEGA_MAT_ELASTIC) {
    for (int k = 0; k < 6; ++k) out[k] = sp[k];
  } else if (m.type == MEGA_MAT_VONMISES) {
    it = von_mises(sp, ep, m, maxit, out, cap);
  } else if (m.type == MEGA_MAT_VM_RATE) {
    double dg, ftr;
    it = vm_rate(sp, ep, m, dlt, rtol, maxit, solver, -1.0, out, cap, dg, ftr);
  } else {
    atomicOr(status, (unsigned)MEGA_ST_BAD_MATERIAL);
    for (int k = 0; k < 6; ++k) out[k] = sp[k];
  }
  if (cap) atomicOr(status, (unsigned)MEGA_ST_NEWTON_CAP);
  state[20 * i + 2] = ep;
  for (int k = 0; k < 6; ++k) stress[6 * i + k] = out[k];
  if (iters) iters[i] = it;
}

// renumbering: new node r is old node perm[r]
__global__ void k_iperm(int32_t n, const int32_t* __restrict__ perm, int32_t* __restrict__ iperm) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) iperm[perm[r]] = (int32_t)r;
}
// dst[r*w + k] = src[perm[r]*w + k]  (gather = old -> new), element size es bytes
__global__ void k_i32_to_f64(int64_t m, const int32_t* __restrict__ a, double* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) out[k] = (double)a[k];
}
__global__ void k_add_kernel(int64_t m, const double* __restrict__ a, const double* __restrict__ b,
                             double* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) out[k] = a[k] + b[k];
}
__global__ void k_perm_gather(int32_t n, int w, int es, const int32_t* __restrict__ perm,
                              const unsigned char* __restrict__ src, unsigned char* __restrict__ dst) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * w) return;
  const int64_t r = t / w, k = t - r * w;
  const unsigned char* a = src + ((int64_t)perm[r] * w + k) * es;
  unsigned char* b = dst + t * es;
  for (int q = 0; q < es; ++q) b[q] = a[q];
}
__global__ void k_newrow_len(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ rowptr0,
                             int32_t* __restrict__ len) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) len[r] = (int32_t)(rowptr0[perm[r] + 1] - rowptr0[perm[r]]);
}
// warp per new row: copy the old row (same entry order), columns renumbered
__global__ void k_permute_rows(int32_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                               const int64_t* __restrict__ rowptr0, const int32_t* __restrict__ col0,
                               const double* __restrict__ v0, const double* __restrict__ v1,
                               const double* __restrict__ v2, const double* __restrict__ v3,
                               const int64_t* __restrict__ rowptr1, int32_t* __restrict__ col1,
                               double* __restrict__ w0, double* __restrict__ w1, double* __restrict__ w2,
                               double* __restrict__ w3) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t a0 = rowptr0[perm[r]], len = rowptr0[perm[r] + 1] - a0, b0 = rowptr1[r];
  for (int64_t k = lane; k < len; k += 32) {
    col1[b0 + k] = iperm[col0[a0 + k]];
    w0[b0 + k] = v0[a0 + k]; w1[b0 + k] = v1[a0 + k]; w2[b0 + k] = v2[a0 + k]; w3[b0 + k] = v3[a0 + k];
  }
}
// the lists in the new numbering without values: rows in the new order, each
// keeping its entries' order, columns renumbered
__global__ void k_renumber_cols(int32_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                                const int64_t* __restrict__ rowptr0, const int32_t* __restrict__ col0,
                                const int64_t* __restrict__ rowptr1, int32_t* __restrict__ col1) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t a0 = rowptr0[perm[r]], len = rowptr0[perm[r] + 1] - a0, b0 = rowptr1[r];
  for (int64_t k = lane; k < len; k += 32) col1[b0 + k] = iperm[col0[a0 + k]];
}
// row sums of the float-rounded packed gradients (the mixed path's sum_J g)
__global__ void k_rowsum_pk32(int32_t n, const int64_t* __restrict__ rowptr, const float4* __restrict__ pk,
                              double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
    const float4 v = pk[p];
    a += (double)v.x; b += (double)v.y; c += (double)v.z;
  }
  out[3 * i] = a; out[3 * i + 1] = b; out[3 * i + 2] = c;
}

inline unsigned grid_for(int64_t work, int block) { return (unsigned)((work + block - 1) / block); }

// Worker threads for the host-side set-up loops, started once per process
// (up to 15 besides the caller) and kept: starting threads for every loop
// cost more than the copies they split.  Tasks from concurrent callers share
// one queue; a caller waiting for its own tasks runs queued ones meanwhile,
// so a call completes even with every worker busy elsewhere.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool* p = new HostPool();  // never destroyed: the workers block in wait() at exit
    return *p;
  }
  int workers() const { return nw_; }
  void submit(std::function<void()> f) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(std::move(f));
    }
    cv_.notify_one();
  }
  bool run_one() {
    std::function<void()> f;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (q_.empty()) return false;
      f = std::move(q_.front());
      q_.pop_front();
    }
    f();
    return true;
  }

 private:
  HostPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    nw_ = (int)std::min(15u, hw - 1);
    for (int k = 0; k < nw_; ++k) std::thread([this] { loop(); }).detach();
  }
  void loop() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return !q_.empty(); });
        f = std::move(q_.front());
        q_.pop_front();
      }
      f();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> q_;
  int nw_ = 0;
};

// fn(lo, hi) over [0, n) in contiguous chunks on the host's cores (the
// per-node set-up scans of a million-node model), at least `grain` items
// per chunk; the caller runs the first chunk
template <typename F>
void host_parallel(int64_t n, F fn, int64_t grain = 65536) {
  HostPool& pool = HostPool::get();
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(pool.workers() + 1, n / grain));
  if (nt == 1) { fn((int64_t)0, n); return; }
  std::atomic<int64_t> left(nt - 1);
  for (int64_t t = 1; t < nt; ++t)
    pool.submit([&fn, &left, n, nt, t] {
      fn(n * t / nt, n * (t + 1) / nt);
      left.fetch_sub(1, std::memory_order_release);
    });
  fn((int64_t)0, n / nt);
  while (left.load(std::memory_order_acquire) > 0)
    if (!pool.run_one()) std::this_thread::yield();
}

// Bulk host <-> device copies go through one pinned buffer kept for the
// process: the host's cores copy the caller's (pageable) arrays into it in
// 4 MiB pieces and each piece moves with its own DMA as soon as it is there
// (downloads the other way round), instead of the driver staging pageable
// memory on the calling thread.  One user at a time; a failed pinned
// allocation falls back to plain pageable copies.
struct PinnedStage {
  std::mutex mu;
  unsigned char* p = nullptr;
  size_t cap = 0;
};
PinnedStage g_stage;

// one array to upload: copied from src, or written by fill(staging) when
// the host array is formed on the way (fill writes `bytes` bytes)
struct HostToDevice {
  void* dst;
  const void* src;
  size_t bytes;
  std::function<void(void*)> fill = nullptr;
};

// the copies in order on stream s, complete on return
int upload_staged(cudaStream_t s, const std::vector<HostToDevice>& items) {
  size_t total = 0;
  for (const auto& it : items) total += (it.bytes + 255) & ~(size_t)255;
  std::lock_guard<std::mutex> lk(g_stage.mu);
  if (g_stage.cap < total) {
    if (g_stage.p) cudaFreeHost(g_stage.p);
    g_stage.p = nullptr;
    g_stage.cap = 0;
    if (cudaHostAlloc((void**)&g_stage.p, total, cudaHostAllocDefault) == cudaSuccess) g_stage.cap = total;
    else { g_stage.p = nullptr; cudaGetLastError(); }
  }
  if (!g_stage.p) {
    for (const auto& it : items) {
      if (it.fill) {
        std::vector<unsigned char> tmp(it.bytes);
        it.fill(tmp.data());
        MEGA_TRY(cudaMemcpy(it.dst, tmp.data(), it.bytes, cudaMemcpyHostToDevice));
      } else {
        MEGA_TRY(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyHostToDevice, s));
      }
    }
    MEGA_TRY(cudaStreamSynchronize(s));
    return 0;
  }
  // Pieces of at most 4 MiB (a filled array is one piece), each copied into
  // its place in the stage by a pool thread and sent as soon as it is there,
  // so the DMA runs while the host is still copying the rest.
  struct Piece { const HostToDevice* it; size_t at, bytes; unsigned char* stage; };
  constexpr size_t kPiece = (size_t)4 << 20;
  std::vector<Piece> pieces;
  size_t off = 0;
  for (const auto& it : items) {
    if (it.fill) pieces.push_back({&it, 0, it.bytes, g_stage.p + off});
    else
      for (size_t a = 0; a < it.bytes; a += kPiece)
        pieces.push_back({&it, a, std::min(kPiece, it.bytes - a), g_stage.p + off + a});
    off += (it.bytes + 255) & ~(size_t)255;
  }
  std::atomic<int> err(0);
  host_parallel((int64_t)pieces.size(), [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      const Piece& pc = pieces[k];
      if (pc.it->fill) pc.it->fill(pc.stage);
      else std::memcpy(pc.stage, (const unsigned char*)pc.it->src + pc.at, pc.bytes);
      const cudaError_t e = cudaMemcpyAsync((unsigned char*)pc.it->dst + pc.at, pc.stage, pc.bytes,
                                            cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) err.store((int)e);
    }
  }, 1);
  if (err.load()) {
    record_cuda_error((cudaError_t)err.load(), "cudaMemcpyAsync", __FILE__, __LINE__);
    return MEGA_ERR_CUDA;
  }
  MEGA_TRY(cudaStreamSynchronize(s));
  return 0;
}

// device -> host through the pinned buffer (stream s ordered, complete on return)
int download_staged(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_stage.mu);
  if (g_stage.cap < bytes) {
    if (g_stage.p) cudaFreeHost(g_stage.p);
    g_stage.p = nullptr;
    g_stage.cap = 0;
    if (cudaHostAlloc((void**)&g_stage.p, bytes, cudaHostAllocDefault) == cudaSuccess) g_stage.cap = bytes;
    else { g_stage.p = nullptr; cudaGetLastError(); }
  }
  if (!g_stage.p) {
    MEGA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    return 0;
  }
  // 4 MiB pieces, each copied out by a pool thread as soon as its DMA is done
  constexpr size_t kPiece = (size_t)4 << 20;
  const int64_t np = (int64_t)((bytes + kPiece - 1) / kPiece);
  std::vector<cudaEvent_t> ev(np, nullptr);
  int r = 0;
  for (int64_t k = 0; k < np && !r; ++k) {
    const size_t a = (size_t)k * kPiece, len = std::min(kPiece, bytes - a);
    if (cudaMemcpyAsync(g_stage.p + a, (const unsigned char*)src + a, len, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ev[k], s) != cudaSuccess)
      r = MEGA_ERR_CUDA;
  }
  std::atomic<int> bad(0);
  if (!r)
    host_parallel(np, [&](int64_t lo, int64_t hi) {
      for (int64_t k = lo; k < hi; ++k) {
        const size_t a = (size_t)k * kPiece, len = std::min(kPiece, bytes - a);
        if (cudaEventSynchronize(ev[k]) != cudaSuccess) { bad.store(1); continue; }
        std::memcpy((unsigned char*)dst + a, g_stage.p + a, len);
      }
    }, 1);
  if (r || bad.load()) {
    cudaStreamSynchronize(s);  // no DMA may still write the stage
    record_cuda_error(cudaGetLastError(), "download_staged", __FILE__, __LINE__);
    r = MEGA_ERR_CUDA;
  }
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  return r;
}

// Deduplication of PROPS(30,N) and the material type into a table of
// entries and a per-node index.  Rows equal to their predecessor (the usual
// case: materials come in blocks) reuse its entry; that comparison runs in
// parallel, the table lookups of the remaining rows serially.
static int material_table(int32_t n, const double* props, const int32_t* mat_type, size_t cap,
                          std::vector<MatEntry>& ents, std::vector<uint16_t>& idx, bool& damaged) {
  std::vector<uint8_t> same(n, 0);
  host_parallel(n, [&](int64_t lo, int64_t hi) {
    for (int64_t i = std::max<int64_t>(lo, 1); i < hi; ++i)
      same[i] = mat_type[i] == mat_type[i - 1] &&
                std::memcmp(props + 30 * (size_t)i, props + 30 * (size_t)(i - 1), 30 * sizeof(double)) == 0;
  });
  std::map<std::vector<double>, uint16_t> tab;
  idx.assign(n, 0);
  ents.clear();
  damaged = false;
  for (int32_t i = 0; i < n; ++i) {
    if (same[i]) { idx[i] = idx[i - 1]; continue; }
    std::vector<double> key(props + 30 * (size_t)i, props + 30 * (size_t)i + 30);
    key.push_back((double)mat_type[i]);
    auto it = tab.find(key);
    if (it == tab.end()) {
      if (ents.size() >= cap) return MEGA_ERR_UNSUPPORTED;
      const MatEntry e = mat_entry(mat_type[i], props + 30 * (size_t)i);
      damaged = damaged || damaged_type(e.type);
      it = tab.emplace(key, (uint16_t)ents.size()).first;
      ents.push_back(e);
    }
    idx[i] = it->second;
  }
  return 0;
}

}  // namespace

// ------------------------------------------------------------- context
struct Ctx {
  mega_params p{};
  int32_t n = 0;
  cudaStream_t s = nullptr;
  DevPool pool;      // model + state
  DevPool nbpool;    // neighbour structure and shapes
  DevPool mixpool;   // float copies for the mixed mode
  // model
  double *coo = nullptr, *win = nullptr, *vol = nullptr, *mass = nullptr, *sm_len = nullptr;
  double* bodyforce = nullptr;
  int8_t *ebc = nullptr, *body_id = nullptr;
  int32_t* ebc_nodes = nullptr;
  uint16_t* matidx = nullptr;
  MatEntry* mats = nullptr;
  bool has_body = false;
  // neighbours and shapes, in the renumbered (bin-cell) node order
  DevCSR csr;
  bool searched = false;
  int32_t* perm = nullptr;   // new node r = original node perm[r]
  int32_t* iperm = nullptr;  // original node i = new node iperm[i]
  TileSet rt, ct;            // row tiles (deformation gradient), column tiles (force)
  double *shp = nullptr, *sdphi = nullptr, *sdphi32 = nullptr, *tshp = nullptr, *tshp32 = nullptr;
  double* shp32 = nullptr;   // shp in the order of the float row records once reordered (else shp)
  bool banked = false;       // the float records reordered for the gathers' banks (bank_layout)
  void *pk64 = nullptr, *tpk64 = nullptr, *pk32 = nullptr, *tpk32 = nullptr;
  // state
  double *dsp = nullptr, *dsp_tot = nullptr, *dsp_tot_phy = nullptr, *vel = nullptr, *acl = nullptr;
  double *fint = nullptr, *fext = nullptr, *prforce = nullptr, *stress = nullptr, *strain = nullptr;
  double *eps = nullptr, *strain_eq = nullptr, *wvel = nullptr, *fg = nullptr, *scratch3 = nullptr;
  void* tmat = nullptr;
  int32_t* iters = nullptr;
  double* aux = nullptr;  // 4 per node, STATE(1, 2, 4, 5), when a damaged model is present
  // NSNI (ITYPE_INT = 2): second derivatives per entry in CSR and CSC order,
  // stress gradients (18 per node) and per-step scratch
  bool nsni = false;
  NsniS nsr{}, nsc{};
  // mixed NSNI: S as six floats per record in the float row / column record
  // orders, and its row sums (the tiled gathers carry the NSNI terms)
  float *ns_srow = nullptr, *ns_scol = nullptr;
  double* ns_ssum = nullptr;
  // semi-Lagrangian (LLAGRANGIAN = .FALSE.): lists and shapes rebuilt on the
  // current coordinates every step, in the caller's numbering, FP64
  bool semi = false;
  BinGeom sgeom{};           // the LINIT bins
  DevPool sempool;           // this step's lists and shapes
  DevCSR scsr;
  DevCSR* dscsr = nullptr;   // device copy of scsr (read by the force kernel)
  double *sshp = nullptr, *sgx = nullptr, *sgy = nullptr, *sgz = nullptr, *ssd = nullptr;
  double *stgx = nullptr, *stgy = nullptr, *stgz = nullptr, *stshp = nullptr;
  double *coo_cur = nullptr, *zero3 = nullptr;
  double *sgrad = nullptr, *hq = nullptr, *nsw = nullptr, *fstab = nullptr, *stress_prev = nullptr;
  StepAccum* acc = nullptr;
  unsigned* status = nullptr;
  bool phy_valid = true;
  // fixity code 2 (prescribed velocity, MAIN.F90:447-470): the windows of
  // FIXITY2_TIME / FIXITY2_NONZERO_EBC on the device (time (steps,2) then
  // displacement (steps,3), column-major), the device copy of TIME and the
  // three velocities of the current step
  bool has_ebc2 = false;
  int32_t f2_steps = 0;
  double *f2 = nullptr, *dtime = nullptr, *vel2 = nullptr;
  double time = 0.0;
  int64_t steps = 0;
  int64_t launches = 0;
  // independent instances sharing the context (node ranges searched apart)
  std::vector<int32_t> inst_off;  // ninst + 1 prefix offsets, empty = one instance
  std::vector<double> inst_dmax;  // 3 per instance: DIST_MAX of its bin grid
  double* ndt = nullptr;          // per-node step (renumbered order) when the instances step apart
  int prec_mask = 3;              // bit 0: FP64 records built, bit 1: mixed records
  int var_defgrad[2] = {0, 0};    // launch variant of the row gather, [FP64, mixed]
  int var_force[2] = {0, 0};      // launch variant of the column gather
  // surrogate of the rate-dependent return mapping and its sample log
  DevPool mlppool;
  float* mlp_theta = nullptr;  // fp32 parameters (training copy)
  uint16_t* mlp_w2 = nullptr;  // bf16 W2 for the tensor cores
  float* mlp_small = nullptr;
  int32_t* mlp_queue = nullptr;    // plastic rate-dependent nodes of a learned step (n)
  unsigned* mlp_qcount = nullptr;
  bool mlp_on = false;
  float* log_buf = nullptr;
  unsigned long long* log_count = nullptr;
  int64_t log_cap = 0;
  uint32_t log_stride = 1, log_seed = 0;
  // graph cache
  cudaGraphExec_t gexec = nullptr;
  int g_mode = -1;
  double g_dt = 0.0;
  int g_len = 0;
  ~Ctx() {
    if (gexec) cudaGraphExecDestroy(gexec);
    // stream-ordered frees first, then the stream
    sempool.free_all();
    mlppool.free_all();
    mixpool.free_all();
    nbpool.free_all();
    pool.free_all();
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

// Phase timing of the set-up entry points, printed to stderr when the
// environment variable MEGA_TRACE is set (each mark synchronises the stream).
struct PhaseTrace {
  bool on;
  cudaStream_t s;
  const char* what;
  std::chrono::steady_clock::time_point t0, t;
  PhaseTrace(cudaStream_t st, const char* w) : on(std::getenv("MEGA_TRACE") != nullptr), s(st), what(w) {
    t0 = t = std::chrono::steady_clock::now();
  }
  void mark(const char* phase) {
    if (!on) return;
    cudaStreamSynchronize(s);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[mega] %s %-24s %8.3f ms (total %8.3f ms)\n", what, phase,
                 std::chrono::duration<double, std::milli>(now - t).count(),
                 std::chrono::duration<double, std::milli>(now - t0).count());
    t = now;
  }
};

static std::mutex g_ctx_mu;
static std::set<Ctx*> g_ctxs;

static Ctx* get_ctx(int64_t h) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  Ctx* c = reinterpret_cast<Ctx*>(h);
  return g_ctxs.count(c) ? c : nullptr;
}

static int read_status(Ctx* c, bool reset) {
  unsigned st = 0;
  MEGA_TRY(cudaMemcpyAsync(&st, c->status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  if (reset && st) MEGA_TRY(cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->s));
  return (int)st;
}

// The records of a precision are packed at search time only when the
// context's precision mask asks for them.
static int ensure_mixed(Ctx* c) { return (c->prec_mask & 2) ? 0 : MEGA_ERR_STATE; }
static int ensure_fp64(Ctx* c) { return (c->prec_mask & 1) ? 0 : MEGA_ERR_STATE; }

static StressArgs stress_args(Ctx* c, double dt, int mode) {
  StressArgs a{};
  a.n = c->n; a.fg = c->fg; a.matidx = c->matidx; a.mats = c->mats; a.vol = c->vol;
  a.stress = c->stress; a.strain = c->strain; a.eps = c->eps; a.strain_eq = c->strain_eq; a.wvel = c->wvel;
  a.tmat = c->tmat; a.bodyforce = c->bodyforce;
  a.grav[0] = c->p.gravity[0]; a.grav[1] = c->p.gravity[1]; a.grav[2] = c->p.gravity[2];
  a.has_body = c->has_body; a.inv3_exact = c->p.inv3_exact; a.finite_strain = c->p.finite_strain;
  a.maxit = c->p.newton_max_iter; a.rate_solver = c->p.rate_solver; a.rtol = c->p.newton_rtol; a.dt = dt; a.iters = c->iters;
  a.aux = c->aux; a.acc = c->acc; a.status = c->status; a.ndt = c->ndt;
  if ((mode & MEGA_FLAG_LEARNED_GUESS) && c->mlp_on) {
    a.mlp_w2 = c->mlp_w2; a.mlp_small = c->mlp_small; a.queue = c->mlp_queue; a.qcount = c->mlp_qcount;
  }
  if (c->log_cap > 0) {
    a.log_buf = c->log_buf; a.log_count = c->log_count; a.log_cap = c->log_cap;
    a.log_stride = c->log_stride; a.log_seed = c->log_seed;
  }
  return a;
}

static TiledForceArgs force_args(Ctx* c, double dt, int mode, int predict) {
  const bool mixed = (mode & 0xff) == MEGA_MODE_MIXED;
  TiledForceArgs f{};
  f.n = c->n; f.R = c->ct.R; f.ntiles = c->ct.ntiles; f.jmax = c->ct.jmax; f.maxcnt = c->ct.maxcnt;
  f.recmax = c->ct.recmax;
  f.jset = c->ct.jset; f.jcnt = c->ct.jcnt; f.colptr = c->csr.colptr;
  f.pk = mixed ? c->tpk32 : c->tpk64;
  f.tshp = mixed ? c->tshp32 : c->tshp; f.tmat = c->tmat; f.has_body = c->has_body; f.predict = predict;
  f.ebc = c->ebc; f.mass = c->mass; f.matidx = c->matidx; f.mats = c->mats; f.body_id = c->body_id;
  f.fint = c->fint; f.fext = c->fext; f.vel = c->vel; f.acl = c->acl; f.dsp = c->dsp; f.dsp_tot = c->dsp_tot;
  f.prforce = c->prforce; f.fadd = (c->nsni && !mixed) ? c->fstab : nullptr; f.dt = dt; f.acc = c->acc;
  f.status = c->status;
  f.ns_scol = (c->nsni && mixed) ? c->ns_scol : nullptr;
  f.ns_w = (c->nsni && mixed) ? (const float*)c->nsw : nullptr;
  f.vel2 = c->vel2;
  f.ndt = c->ndt;
  return f;
}

// The prescribed velocities of the fixity-2 DOFs at the step's TIME
// (MAIN.F90:448-462: the first window with FIXITY2_TIME(k,1) < TIME <
// FIXITY2_TIME(k,2), FIXITY2_NONZERO_EBC(k,j) over its length, else zero),
// then TIME = TIME + DLT (MAIN.F90:644).  One thread; launched once per step
// between the stress and force kernels of contexts with code-2 DOFs.
__global__ void k_fixity2(int32_t steps, const double* __restrict__ f2, double* time, double* vel2, double dt) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double t = *time;
  int32_t k = 0;
  for (int32_t i = 1; i <= steps; ++i)
    if (f2[i - 1] < t && t < f2[steps + i - 1]) { k = i; break; }
  for (int j = 0; j < 3; ++j)
    vel2[j] = k ? f2[(int64_t)(2 + j) * steps + k - 1] / (f2[steps + k - 1] - f2[k - 1]) : 0.0;
  *time = t + dt;
}

static int launch_fixity2(Ctx* c, double dt) {
  if (!c->has_ebc2) return 0;
  k_fixity2<<<1, 32, 0, c->s>>>(c->f2_steps, c->f2, c->dtime, c->vel2, dt);
  MEGA_CHECK_LAUNCH();
  return 0;
}

// The device's TIME from the host's before a run of steps (the device copy
// advances with the steps; timing and tuning calls step it too).
static int sync_time(Ctx* c) {
  if (c->has_ebc2) MEGA_TRY(cudaMemcpyAsync(c->dtime, &c->time, sizeof(double), cudaMemcpyHostToDevice, c->s));
  return 0;
}

// the NSNI terms of the mixed tiled row gather (null: none)
static const NsniTiles* nsni_tiles(Ctx* c, bool mixed, NsniTiles& buf) {
  if (!c->nsni || !mixed) return nullptr;
  buf.srow = c->ns_srow;
  buf.ssum = c->ns_ssum;
  buf.hq = c->hq;
  return &buf;
}

static NsniStepArgs nsni_args(Ctx* c) {
  NsniStepArgs a{};
  a.n = c->n; a.fg = c->fg; a.stress_old = c->stress_prev; a.stress_new = c->stress; a.sml = c->sm_len;
  a.vol = c->vol; a.matidx = c->matidx; a.mats = c->mats; a.hq = c->hq; a.sgrad = c->sgrad; a.w = c->nsw;
  a.fstab = c->fstab; a.finite_strain = c->p.finite_strain; a.inv3_exact = c->p.inv3_exact; a.acc = c->acc;
  a.status = c->status;
  return a;
}

// kernels one step launches (the learned start splits the stress kernel in
// two; NSNI adds the stress-gradient kernel, and in FP64 its two gathers)
static int kernels_per_step(const Ctx* c, int mode = 0) {
  const bool mixed = (mode & 0xff) == MEGA_MODE_MIXED;
  return (c->nsni ? (mixed ? 4 : 6) : 3) + (c->has_ebc2 ? 1 : 0) +
         (((mode & MEGA_FLAG_LEARNED_GUESS) && c->mlp_on) ? 1 : 0);
}

static int step_once(Ctx* c, double dt, int mode, int predict, cudaEvent_t* ev) {
  const bool mixed = (mode & 0xff) == MEGA_MODE_MIXED;
  const bool interp = (mode & MEGA_FLAG_INTERP_EACH_STEP) != 0;
  if (ev) MEGA_TRY(cudaEventRecord(ev[0], c->s));
  if (c->nsni)
    MEGA_TRY(cudaMemcpyAsync(c->stress_prev, c->stress, sizeof(double) * 6 * c->n, cudaMemcpyDeviceToDevice, c->s));
  NsniTiles nt;
  int r = launch_defgrad_tiled(c->s, mixed, interp, c->n, c->rt, nsni_tiles(c, mixed, nt), c->csr.rowptr,
                               mixed ? c->pk32 : c->pk64, c->dsp, c->dsp_tot, mixed ? c->sdphi32 : c->sdphi,
                               (mixed && c->shp32) ? c->shp32 : c->shp, c->dsp_tot_phy, c->fg, c->acc, c->status,
                               c->var_defgrad[mixed]);
  if (r) return r;
  if (c->nsni && !mixed && (r = nsni_step(c->s, nsni_args(c), c->csr, c->nsr, c->nsc, false, c->dsp, 0))) return r;
  if (ev) MEGA_TRY(cudaEventRecord(ev[1], c->s));
  r = launch_stress(c->s, mixed, stress_args(c, dt, mode));
  if (r) return r;
  if (c->nsni && (r = nsni_step(c->s, nsni_args(c), c->csr, c->nsr, c->nsc, mixed, c->dsp, 1))) return r;
  if (c->nsni && !mixed && (r = nsni_step(c->s, nsni_args(c), c->csr, c->nsr, c->nsc, false, c->dsp, 2))) return r;
  if ((r = launch_fixity2(c, dt))) return r;
  if (ev) MEGA_TRY(cudaEventRecord(ev[2], c->s));
  r = launch_force_tiled(c->s, mixed, force_args(c, dt, mode, predict), c->var_force[mixed]);
  if (r) return r;
  if (ev) MEGA_TRY(cudaEventRecord(ev[3], c->s));
  c->launches += kernels_per_step(c, mode);
  return 0;
}

static int graph_for(Ctx* c, double dt, int mode, int len) {
  if (c->gexec && c->g_mode == mode && c->g_dt == dt && c->g_len == len) return 0;
  if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
  cudaGraph_t g = nullptr;
  MEGA_TRY(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
  const int64_t before = c->launches;
  int r = 0;
  for (int k = 0; k < len && !r; ++k) r = step_once(c, dt, mode, 1, nullptr);
  cudaError_t e = cudaStreamEndCapture(c->s, &g);
  c->launches = before;
  if (r) { if (g) cudaGraphDestroy(g); return r; }
  if (e != cudaSuccess) { record_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__); return MEGA_ERR_CUDA; }
  e = cudaGraphInstantiate(&c->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { record_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__); return MEGA_ERR_CUDA; }
  c->g_mode = mode; c->g_dt = dt; c->g_len = len;
  return 0;
}

static int semi_steps(Ctx* c, int32_t nsteps, double dt, int mode);

static int run_steps(Ctx* c, int32_t nsteps, double dt, int mode) {
  if (!c->searched) return MEGA_ERR_STATE;
  if (nsteps <= 0) return 0;
  if (c->semi) return semi_steps(c, nsteps, dt, mode);
  const int prec = mode & 0xff;
  if (prec != MEGA_MODE_FP64 && prec != MEGA_MODE_MIXED) return MEGA_ERR_ARG;
  if ((mode & MEGA_FLAG_LEARNED_GUESS) && !c->mlp_on) return MEGA_ERR_STATE;
  { int r = (prec == MEGA_MODE_MIXED) ? ensure_mixed(c) : ensure_fp64(c); if (r) return r; }
  if (!(mode & MEGA_FLAG_INTERP_EACH_STEP)) c->phy_valid = false;
  int r = sync_time(c);
  if (r) return r;
  r = launch_predict(c->s, 3 * (int64_t)c->n, c->dsp, c->dsp_tot, c->vel, c->acl, dt, c->ndt);
  if (r) return r;
  c->launches += 1;
  int32_t rem = nsteps - 1;
  const int len = 16;
  if (rem >= len) {
    r = graph_for(c, dt, mode, len);
    if (r) return r;
    while (rem >= len) {
      MEGA_TRY(cudaGraphLaunch(c->gexec, c->s));
      c->launches += kernels_per_step(c, mode) * len;
      rem -= len;
    }
  }
  for (; rem > 0 && !r; --rem) r = step_once(c, dt, mode, 1, nullptr);
  if (r) return r;
  r = step_once(c, dt, mode, 0, nullptr);
  if (r) return r;
  for (int32_t k = 0; k < nsteps; ++k) c->time = c->time + dt;  // TIME = TIME + DLT
  c->steps += nsteps;
  return 0;
}

// The deduplicated PROPS(30,N) table and per-node index onto the device.
static int install_materials(Ctx* c, const std::vector<MatEntry>& ents, const std::vector<uint16_t>& idx,
                             bool damaged) {
  MEGA_ALLOC(c->pool, c->matidx, c->n);
  MEGA_ALLOC(c->pool, c->mats, ents.size());
  if (damaged) {  // STATE(1, 2, 4, 5) start at zero (STATE_INIT.f90)
    MEGA_ALLOC(c->pool, c->aux, 4 * (int64_t)c->n);
    MEGA_TRY(cudaMemsetAsync(c->aux, 0, sizeof(double) * 4 * c->n, c->s));
  }
  MEGA_TRY(cudaMemcpyAsync(c->matidx, idx.data(), sizeof(uint16_t) * c->n, cudaMemcpyHostToDevice, c->s));
  MEGA_TRY(cudaMemcpyAsync(c->mats, ents.data(), sizeof(MatEntry) * ents.size(), cudaMemcpyHostToDevice, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

template <typename T>
static int upload(cudaStream_t s, T* d, const T* h, size_t count) {
  MEGA_TRY(cudaMemcpyAsync(d, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
  return 0;
}

// Device CSR from the reference's 1-based (GN, GSTART, GSTACK); rows are
// re-packed contiguously in node order.  hpos[k] = 0-based GSTACK position
// of packed entry k (for writing per-entry values back).
static int csr_from_host(cudaStream_t s, int32_t n, const int32_t* gn, const int32_t* gstart,
                         const int32_t* gstack, int64_t nnz_cap, DevPool& pool, DevCSR& csr,
                         std::vector<int64_t>& hpos) {
  std::vector<int64_t> rp(n + 1, 0);
  for (int32_t i = 0; i < n; ++i) {
    if (gn[i] < 0) return MEGA_ERR_ARG;
    rp[i + 1] = rp[i] + gn[i];
  }
  const int64_t nnz = rp[n];
  std::vector<int32_t> col(nnz);
  hpos.resize(nnz);
  for (int32_t i = 0; i < n; ++i) {
    const int64_t s0 = (int64_t)gstart[i] - 1;
    if (gn[i] > 0 && (s0 < 0 || s0 + gn[i] > nnz_cap)) return MEGA_ERR_ARG;
    for (int32_t k = 0; k < gn[i]; ++k) {
      const int32_t j = gstack[s0 + k] - 1;
      if (j < 0 || j >= n) return MEGA_ERR_ARG;
      col[rp[i] + k] = j;
      hpos[rp[i] + k] = s0 + k;
    }
  }
  csr.n = n;
  csr.nnz = nnz;
  csr.gmaxn = 0;
  for (int32_t i = 0; i < n; ++i) csr.gmaxn = std::max(csr.gmaxn, gn[i]);
  MEGA_ALLOC(pool, csr.rowptr, n + 1);
  MEGA_ALLOC(pool, csr.col, nnz);
  int r = upload(s, csr.rowptr, rp.data(), n + 1);
  if (r) return r;
  return upload(s, csr.col, col.data(), nnz);
}

static int make_stream(cudaStream_t* s) {
  MEGA_TRY(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  return 0;
}

// Contexts and their set-up temporaries allocate from the device's default
// memory pool; with the release threshold at its maximum, memory a context
// or a temporary frees stays in the pool and the next allocation reuses it
// without a driver round trip.  The pool's previous threshold is kept per
// device; mega_release_cached_memory puts it back, hands the block cache
// below to the pool and trims the pool, so a host program with its own
// allocator gets the memory back without ending the process.
bool trace_on() {
  static const bool on = std::getenv("MEGA_TRACE") != nullptr;
  return on;
}

void trace_alloc(size_t bytes, double ms, bool ordered) {
  if (ms > 5.0)
    std::fprintf(stderr, "[mega] slow %s of %.1f MB: %.3f ms\n", ordered ? "cudaMallocAsync" : "cudaMalloc",
                 bytes / 1048576.0, ms);
}

static std::mutex g_pool_mu;
static std::map<int, uint64_t> g_prev_threshold;  // device -> release threshold before the library set it

void retain_pool_memory() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_prev_threshold.count(dev)) return;
  cudaMemPool_t mp;
  if (cudaDeviceGetDefaultMemPool(&mp, dev) != cudaSuccess) { cudaGetLastError(); return; }
  uint64_t prev = 0;
  if (cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &prev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  uint64_t thr = UINT64_MAX;
  if (cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  g_prev_threshold[dev] = prev;
}

namespace {
struct CachedBlock {
  void* p;
  size_t bytes;
  int dev;
  cudaEvent_t ev;  // recorded after the block's last use
};
std::mutex g_blk_mu;
std::multimap<size_t, CachedBlock> g_blk;  // by block size
size_t g_blk_total = 0;
std::map<int, size_t> g_blk_dev_total;     // bytes cached per device
std::map<int, size_t> g_blk_cap;           // per device: a quarter of its memory

// Size classes: 512 bytes below 1 MiB; above, an eighth of the size's
// power of two (at least 2 MiB), so a list that grew by some entries since
// the last search (semi-Lagrangian re-search under compression) still finds
// the block of the last one
size_t block_round(size_t b) {
  if (b < ((size_t)1 << 20)) return (b + 511) & ~(size_t)511;
  size_t top = (size_t)1 << 20;
  while (top * 2 <= b) top *= 2;
  const size_t g = std::max(top >> 3, (size_t)2 << 20);
  return (b + g - 1) / g * g;
}

// hand every cached block of device dev back to the memory pool
void flush_blocks(int dev, cudaStream_t s) {
  std::vector<CachedBlock> out;
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    for (auto it = g_blk.begin(); it != g_blk.end();) {
      if (it->second.dev == dev) {
        out.push_back(it->second);
        g_blk_total -= it->second.bytes;
        g_blk_dev_total[dev] -= it->second.bytes;
        it = g_blk.erase(it);
      } else {
        ++it;
      }
    }
  }
  for (auto& b : out) {
    cudaStreamWaitEvent(s, b.ev, 0);
    cudaEventDestroy(b.ev);
    cudaFreeAsync(b.p, s);
  }
}
}  // namespace

int cached_alloc(void** p, size_t bytes, cudaStream_t s, size_t* got) {
  const size_t want = block_round(bytes);
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::unique_lock<std::mutex> lk(g_blk_mu);
    // the same size class first (a repeated set-up finds all its blocks so
    // and takes none that another of its requests will ask for); failing
    // that, the smallest block up to a quarter larger (an array that grew)
    auto pick = g_blk.end();
    for (auto it = g_blk.lower_bound(want); it != g_blk.end() && it->first == want; ++it)
      if (it->second.dev == dev) { pick = it; break; }
    if (pick == g_blk.end())
      for (auto it = g_blk.upper_bound(want); it != g_blk.end() && it->first <= want + want / 4; ++it)
        if (it->second.dev == dev) { pick = it; break; }
    if (pick != g_blk.end()) {
      const CachedBlock b = pick->second;
      g_blk.erase(pick);
      g_blk_total -= b.bytes;
      g_blk_dev_total[dev] -= b.bytes;
      lk.unlock();
      cudaStreamWaitEvent(s, b.ev, 0);
      cudaEventDestroy(b.ev);
      *p = b.p;
      *got = b.bytes;
      return 0;
    }
  }
  if (want >= ((size_t)64 << 20)) {
    // a large miss: blocks of this device between half the request and the
    // request are the predecessors of a grown array; hand them back first
    std::vector<CachedBlock> stale;
    {
      std::lock_guard<std::mutex> lk(g_blk_mu);
      for (auto it = g_blk.lower_bound(want / 2); it != g_blk.end() && it->first < want;) {
        if (it->second.dev == dev) {
          stale.push_back(it->second);
          g_blk_total -= it->second.bytes;
          g_blk_dev_total[dev] -= it->second.bytes;
          it = g_blk.erase(it);
        } else {
          ++it;
        }
      }
    }
    for (auto& b : stale) {
      cudaStreamWaitEvent(s, b.ev, 0);
      cudaEventDestroy(b.ev);
      cudaFreeAsync(b.p, s);
    }
  }
  cudaError_t e = cudaMallocAsync(p, want, s);
  if (e != cudaSuccess) {  // give the cache back to the pool and try once more
    cudaGetLastError();
    flush_blocks(dev, s);
    e = cudaMallocAsync(p, want, s);
  }
  if (e != cudaSuccess) {
    record_cuda_error(e, "cudaMallocAsync", __FILE__, __LINE__);
    *p = nullptr;
    return MEGA_ERR_NOMEM;
  }
  *got = want;
  return 0;
}

void cached_free(void* p, size_t block_bytes, cudaStream_t s) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaEvent_t ev = nullptr;
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(ev, s) != cudaSuccess) {
    cudaGetLastError();
    if (ev) cudaEventDestroy(ev);
    cudaFreeAsync(p, s);
    return;
  }
  // at most a quarter of this device's memory waits in the cache
  std::vector<CachedBlock> evict;
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    auto ci = g_blk_cap.find(dev);
    if (ci == g_blk_cap.end()) {
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { cudaGetLastError(); tot = 0; }
      ci = g_blk_cap.emplace(dev, tot / 4).first;
    }
    const size_t cap = ci->second;
    g_blk.emplace(block_bytes, CachedBlock{p, block_bytes, dev, ev});
    size_t& held = g_blk_dev_total[dev];
    held += block_bytes;
    g_blk_total += block_bytes;
    // the largest blocks of this device go first
    for (auto it = g_blk.end(); cap && held > cap && it != g_blk.begin();) {
      --it;
      if (it->second.dev != dev) continue;
      evict.push_back(it->second);
      held -= it->second.bytes;
      g_blk_total -= it->second.bytes;
      it = g_blk.erase(it);
    }
  }
  for (auto& b : evict) {
    cudaStreamWaitEvent(s, b.ev, 0);
    cudaEventDestroy(b.ev);
    cudaFreeAsync(b.p, s);
  }
}

struct StreamGuard {
  cudaStream_t s = nullptr;
  ~StreamGuard() { if (s) cudaStreamDestroy(s); }
};

// ---- semi-Lagrangian steps
__global__ void k_iota(int32_t n, int32_t* __restrict__ a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = (int32_t)i;
}

// Lists and shapes on the coordinates x (the LINIT bins are laid out when
// linit, reused afterwards), their transposed gradients and row sums.
static int semi_build(Ctx* c, const double* x, bool linit) {
  const int32_t n = c->n;
  c->sempool.free_all();
  c->scsr = DevCSR();
  int r = bin_search(c->s, n, x, c->win, c->sm_len, c->p.dist_max, 0, c->p.shsup, c->status, c->scsr, nullptr,
                     c->sempool, linit ? &c->sgeom : nullptr, nullptr, linit ? nullptr : &c->sgeom);
  if (r) return r;
  const int64_t m = c->scsr.nnz;
  MEGA_ALLOC(c->sempool, c->sshp, m);
  MEGA_ALLOC(c->sempool, c->sgx, m);
  MEGA_ALLOC(c->sempool, c->sgy, m);
  MEGA_ALLOC(c->sempool, c->sgz, m);
  if ((r = rk_shapes(c->s, c->p, n, x, c->win, c->ebc_nodes, c->scsr, c->sshp, c->sgx, c->sgy, c->sgz, c->status)))
    return r;
  if ((r = build_transpose(c->s, c->scsr, c->sempool))) return r;
  MEGA_ALLOC(c->sempool, c->stgx, m);
  MEGA_ALLOC(c->sempool, c->stgy, m);
  MEGA_ALLOC(c->sempool, c->stgz, m);
  k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->scsr.tpos, c->sgx, c->stgx);
  k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->scsr.tpos, c->sgy, c->stgy);
  k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->scsr.tpos, c->sgz, c->stgz);
  c->stshp = nullptr;
  if (c->has_body) {
    MEGA_ALLOC(c->sempool, c->stshp, m);
    k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->scsr.tpos, c->sshp, c->stshp);
  }
  MEGA_ALLOC(c->sempool, c->ssd, 3 * (int64_t)n);
  k_rowsum3<double><<<grid_for(n, 256), 256, 0, c->s>>>(n, c->scsr.rowptr, c->sgx, c->sgy, c->sgz, c->ssd);
  MEGA_CHECK_LAUNCH();
  MEGA_ALLOC(c->sempool, c->dscsr, 1);
  MEGA_TRY(cudaMemcpyAsync(c->dscsr, &c->scsr, sizeof(DevCSR), cudaMemcpyHostToDevice, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));  // (the host copy of scsr goes with this scope's changes)
  return 0;
}

// LINIT of the semi-Lagrangian context: lists and shapes on the initial
// coordinates, the caller's numbering kept (identity permutation).
static int semi_search(Ctx* c, int32_t* gn, int32_t* gstart, int32_t* gstack, int64_t dim_nn_list, double* shp,
                       double* dshp, int64_t* nnz, int32_t* gmaxn) {
  const int32_t n = c->n;
  if (!c->perm) {
    MEGA_ALLOC(c->nbpool, c->perm, n);
    MEGA_ALLOC(c->nbpool, c->iperm, n);
    k_iota<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->perm);
    k_iota<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->iperm);
    MEGA_CHECK_LAUNCH();
  }
  MEGA_TRY(cudaMemcpyAsync(c->coo_cur, c->coo, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, c->s));
  int r = semi_build(c, c->coo_cur, true);
  if (r) return r;
  const int64_t m = c->scsr.nnz;
  int st = 0;
  if (gn || gstart) {
    std::vector<int64_t> rp(n + 1);
    MEGA_TRY(cudaMemcpyAsync(rp.data(), c->scsr.rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    for (int32_t i = 0; i < n; ++i) {
      if (gn) gn[i] = (int32_t)(rp[i + 1] - rp[i]);
      if (gstart) gstart[i] = (int32_t)(rp[i] + 1);
    }
  }
  if (gstack) {
    if (m > dim_nn_list) st |= MEGA_ST_STACK_OVERFLOW;
    else {
      MEGA_TRY(cudaMemcpyAsync(gstack, c->scsr.col, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, c->s));
      MEGA_TRY(cudaStreamSynchronize(c->s));
      for (int64_t k = 0; k < m; ++k) gstack[k] += 1;
    }
  }
  if (shp) MEGA_TRY(cudaMemcpyAsync(shp, c->sshp, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
  if (dshp) {
    std::vector<double> a(m), b(m), d(m);
    MEGA_TRY(cudaMemcpyAsync(a.data(), c->sgx, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaMemcpyAsync(b.data(), c->sgy, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaMemcpyAsync(d.data(), c->sgz, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    for (int64_t k = 0; k < m; ++k) { dshp[3 * k] = a[k]; dshp[3 * k + 1] = b[k]; dshp[3 * k + 2] = d[k]; }
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  c->searched = true;
  c->phy_valid = true;
  if (nnz) *nnz = m;
  if (gmaxn) *gmaxn = c->scsr.gmaxn;
  int ds = read_status(c, true);
  if (ds < 0) return ds;
  return st | ds;
}

// MAIN.F90:348-488 with LLAGRANGIAN = .FALSE. (HANDELER.F90:145, FINT.F90:
// 410-436): predictor; the physical increment from the last lists and
// shapes; the current coordinates; a re-search on them in the LINIT bins
// and shapes on them; the force with those gradients as they are (F = I:
// no push-forward, J = 1 as the reference's DET stays 1 on this path);
// corrector.  FP64.
static int semi_steps(Ctx* c, int32_t nsteps, double dt, int mode) {
  if ((mode & 0xff) != MEGA_MODE_FP64 || (mode & MEGA_FLAG_INTERP_EACH_STEP)) return MEGA_ERR_UNSUPPORTED;
  if ((mode & MEGA_FLAG_LEARNED_GUESS) && !c->mlp_on) return MEGA_ERR_STATE;
  const int32_t n = c->n;
  const int64_t n3 = 3 * (int64_t)n;
  if (int r = sync_time(c)) return r;
  for (int32_t k = 0; k < nsteps; ++k) {
    int r = launch_predict(c->s, n3, c->dsp, c->dsp_tot, c->vel, c->acl, dt);
    if (r) return r;
    if ((r = launch_interp(c->s, n, c->scsr, c->sshp, c->dsp, c->dsp_tot_phy, c->dsp_tot_phy))) return r;
    k_add_kernel<<<grid_for(n3, 256), 256, 0, c->s>>>(n3, c->coo, c->dsp_tot_phy, c->coo_cur);
    MEGA_CHECK_LAUNCH();
    if ((r = semi_build(c, c->coo_cur, false))) return r;
    if ((r = launch_defgrad(c->s, false, false, n, c->scsr, c->sgx, c->sgy, c->sgz, c->dsp, c->zero3, c->ssd,
                            c->sshp, nullptr, c->fg, c->acc)))
      return r;
    if ((r = launch_stress(c->s, false, stress_args(c, dt, mode)))) return r;
    if ((r = launch_fixity2(c, dt))) return r;
    ForceArgs f{};
    f.n = n; f.csr = c->dscsr; f.tgx = c->stgx; f.tgy = c->stgy; f.tgz = c->stgz; f.tshp = c->stshp;
    f.tmat = c->tmat; f.has_body = c->has_body; f.integrate = 1; f.predict = 0;
    f.ebc = c->ebc; f.mass = c->mass; f.matidx = c->matidx; f.mats = c->mats; f.body_id = c->body_id;
    f.fint = c->fint; f.fext = c->fext; f.vel = c->vel; f.acl = c->acl; f.dsp = c->dsp; f.dsp_tot = c->dsp_tot;
    f.prforce = c->prforce; f.dt = dt; f.acc = c->acc; f.status = c->status; f.vel2 = c->vel2;
    if ((r = launch_force(c->s, false, f))) return r;
    c->launches += 6 + (c->has_ebc2 ? 1 : 0);
    c->time = c->time + dt;
    c->steps += 1;
  }
  c->phy_valid = true;
  return 0;
}

}  // namespace mega

using namespace mega;

extern "C" {

void mega_params_default(mega_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->rk_degree = 1;
  p->rk_cont = 3;
  p->rk_impl = 0;
  p->itype_int = 0;
  p->ql = 1;
  p->lagrangian = 1;
  p->finite_strain = 1;
  p->shsup = 0;
  p->peridynamics = 0;
  p->inv3_exact = 0;
  p->newton_max_iter = 20;
  p->ql_coef = 0.001;
  p->ql_len = 0.0;
  p->newton_rtol = 1e-10;
  p->auto_ts = 0;
  p->dlt_fac = 1.0;
}

const char* mega_status_string(int32_t st) {
  static thread_local char buf[768];
  if (st == 0) return "ok";
  if (st < 0) {
    const char* w = st == MEGA_ERR_CUDA ? "CUDA error" : st == MEGA_ERR_ARG ? "invalid argument"
                  : st == MEGA_ERR_HANDLE ? "invalid handle" : st == MEGA_ERR_STATE ? "call out of order"
                  : st == MEGA_ERR_NOMEM ? "device allocation failed"
                  : st == MEGA_ERR_UNSUPPORTED ? "configuration not supported on this path" : "error";
    snprintf(buf, sizeof(buf), "%s%s%s", w, last_error_text()[0] ? ": " : "", last_error_text());
    return buf;
  }
  buf[0] = 0;
  struct { int bit; const char* t; } tab[] = {
      {MEGA_ST_NEWTON_CAP, "PLASTICITY MATERIAL MODEL DID NOT CONVERGE"},
      {MEGA_ST_SINGULAR_MOMENT, "singular RK moment matrix"},
      {MEGA_ST_BIN_OVERFLOW, "(NODES_IN_BIN(M).GE.MAX_NEIGH)"},
      {MEGA_ST_CAND_OVERFLOW, "IP.GT.10000"},
      {MEGA_ST_NONFINITE, "non-finite force or stress"},
      {MEGA_ST_BAD_MATERIAL, "INVALID MATERIAL TYPE IN SUBROUTINE CONSTITUTION"},
      {MEGA_ST_STACK_OVERFLOW, "neighbour stack larger than DIM_NN_LIST"},
      {MEGA_ST_SINGULAR_SHAPE, "PROBLEM INVERTING MATRIX"},
      {MEGA_ST_BAD_MESH, "element connectivity names a node outside the model"},
      {MEGA_ST_WAIT_TIMEOUT, "a kernel timed out waiting for its asynchronous copies"}};
  for (auto& t : tab)
    if (st & t.bit) {
      if (buf[0]) strncat(buf, "; ", sizeof(buf) - strlen(buf) - 1);
      strncat(buf, t.t, sizeof(buf) - strlen(buf) - 1);
    }
  return buf;
}

int mega_gpu_init(const mega_params* p, int32_t n, const double* coo, const double* win, const double* vol,
                  const double* mass, const int32_t* ebc, const double* vinit, const double* props,
                  const int32_t* mat_type, const int32_t* body_id, const double* bodyforce,
                  const double* sm_len, int64_t* handle) {
  if (!p || n <= 0 || !coo || !win || !vol || !mass || !ebc || !vinit || !props || !mat_type || !sm_len || !handle)
    return MEGA_ERR_ARG;
  if ((p->lagrangian != 1 && p->lagrangian != 0) || p->peridynamics != 0) return MEGA_ERR_UNSUPPORTED;
  if (p->itype_int != 0 && p->itype_int != 2) return MEGA_ERR_UNSUPPORTED;  // DNI or NSNI
  if (p->lagrangian == 0 && p->itype_int != 0) return MEGA_ERR_UNSUPPORTED;  // semi-Lagrangian: DNI
  bool has_ebc2 = false;
  for (int64_t m = 0; m < 3 * (int64_t)n; ++m) {
    if (ebc[m] < 0 || ebc[m] > 2) return MEGA_ERR_ARG;  // fixity codes 0 free, 1 fixed, 2 prescribed velocity
    has_ebc2 = has_ebc2 || ebc[m] == 2;
  }
  Ctx* c = new Ctx();
  c->has_ebc2 = has_ebc2;
  c->p = *p;
  c->n = n;
  int r = make_stream(&c->s);
  const int64_t n3 = 3 * (int64_t)n;
  auto fail = [&](int code) { delete c; return code; };
  if (r) return fail(r);
  c->pool.bind(c->s);
  c->nbpool.bind(c->s);
  c->mixpool.bind(c->s);
  c->mlppool.bind(c->s);
  PhaseTrace tr(c->s, "gpu_init");
#define CA(ptr, cnt) do { if (c->pool.alloc(&(ptr), (size_t)(cnt))) return fail(MEGA_ERR_NOMEM); } while (0)
  CA(c->coo, n3); CA(c->win, n3); CA(c->vol, n); CA(c->mass, n3);
  if (p->itype_int != 0) CA(c->sm_len, 6 * (int64_t)n);  // DNI never reads the smoothing cells
  CA(c->ebc, n3); CA(c->body_id, n); CA(c->ebc_nodes, n);
  CA(c->dsp, n3); CA(c->dsp_tot, n3); CA(c->dsp_tot_phy, n3); CA(c->vel, n3); CA(c->acl, n3);
  CA(c->fint, n3); CA(c->fext, n3); CA(c->prforce, n3); CA(c->scratch3, n3);
  CA(c->stress, 6 * (int64_t)n); CA(c->strain, 6 * (int64_t)n); CA(c->eps, n); CA(c->strain_eq, n);
  CA(c->wvel, n); CA(c->fg, 18 * (int64_t)n); CA(c->iters, n); CA(c->acc, 1); CA(c->status, 1);
  if (has_ebc2) {  // no windows until mega_set_fixity2: the prescribed velocity is zero (MAIN.F90:458-462)
    CA(c->dtime, 1); CA(c->vel2, 3);
    cudaMemsetAsync(c->vel2, 0, sizeof(double) * 3, c->s);
  }
  c->semi = p->lagrangian == 0;
  if (c->semi) {
    c->sempool.bind(c->s);
    CA(c->coo_cur, n3); CA(c->zero3, n3);
    cudaMemsetAsync(c->zero3, 0, sizeof(double) * n3, c->s);
  }
  c->nsni = p->itype_int == 2;
  if (c->nsni) {
    CA(c->sgrad, 18 * (int64_t)n); CA(c->hq, 18 * (int64_t)n); CA(c->nsw, 18 * (int64_t)n);
    CA(c->fstab, n3); CA(c->stress_prev, 6 * (int64_t)n);
    cudaMemsetAsync(c->sgrad, 0, sizeof(double) * 18 * n, c->s);
    cudaMemsetAsync(c->fstab, 0, sizeof(double) * n3, c->s);
  }
  {
    double* t = nullptr;
    CA(t, 12 * (int64_t)n);
    c->tmat = t;
  }
  c->has_body = p->gravity[0] != 0.0 || p->gravity[1] != 0.0 || p->gravity[2] != 0.0;
  if (bodyforce) {
    for (int64_t m = 0; m < n3 && !c->has_body; ++m) c->has_body = bodyforce[m] != 0.0;
    if (c->has_body) {
      CA(c->bodyforce, n3);
      if (upload(c->s, c->bodyforce, bodyforce, n3)) return fail(MEGA_ERR_CUDA);
    }
  }
#undef CA
  tr.mark("allocate");
  // the material table is built on another host thread while this one
  // converts the fixity and copies the node arrays (pageable copies hold
  // the calling thread)
  std::vector<uint16_t> midx;
  std::vector<MatEntry> ments;
  bool mdamaged = false;
  int mres = 0;
  std::thread mt([&] { mres = material_table(n, props, mat_type, 65535, ments, midx, mdamaged); });
  // fixity codes, body ids, EBC node flags and the initial velocity
  // (zero on fixed components, STATE_INIT.f90:97-105) are formed straight
  // into the staging buffer
  auto fill_ebc = [&](void* d) {
    int8_t* o = (int8_t*)d;
    host_parallel(n3, [&](int64_t lo, int64_t hi) { for (int64_t m = lo; m < hi; ++m) o[m] = (int8_t)ebc[m]; });
  };
  auto fill_body = [&](void* d) {
    int8_t* o = (int8_t*)d;
    host_parallel(n, [&](int64_t lo, int64_t hi) {
      for (int64_t i = lo; i < hi; ++i) o[i] = (int8_t)(body_id ? body_id[i] : 1);
    });
  };
  auto fill_en = [&](void* d) {
    int32_t* o = (int32_t*)d;
    host_parallel(n, [&](int64_t lo, int64_t hi) {
      for (int64_t i = lo; i < hi; ++i) o[i] = (ebc[3 * i] == 1 || ebc[3 * i + 1] == 1 || ebc[3 * i + 2] == 1);
    });
  };
  auto fill_vel = [&](void* d) {
    double* o = (double*)d;
    host_parallel(n3, [&](int64_t lo, int64_t hi) {
      for (int64_t m = lo; m < hi; ++m) o[m] = ebc[m] == 1 ? 0.0 : vinit[m];
    });
  };
  std::vector<HostToDevice> items = {
      {c->coo, coo, 8 * (size_t)n3}, {c->win, win, 8 * (size_t)n3}, {c->vol, vol, 8 * (size_t)n},
      {c->mass, mass, 8 * (size_t)n3}, {c->ebc, nullptr, (size_t)n3, fill_ebc},
      {c->body_id, nullptr, (size_t)n, fill_body}, {c->ebc_nodes, nullptr, 4 * (size_t)n, fill_en},
      {c->vel, nullptr, 8 * (size_t)n3, fill_vel}};
  if (c->sm_len) items.push_back({c->sm_len, sm_len, 48 * (size_t)n});
  tr.mark("fixity");
  const bool up_fail = upload_staged(c->s, items) != 0;
  tr.mark("copies");
  mt.join();
  if (up_fail) return fail(MEGA_ERR_CUDA);
  cudaMemsetAsync(c->dsp, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->dsp_tot, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->dsp_tot_phy, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->acl, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->fint, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->fext, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->prforce, 0, sizeof(double) * n3, c->s);
  cudaMemsetAsync(c->stress, 0, sizeof(double) * 6 * n, c->s);
  cudaMemsetAsync(c->strain, 0, sizeof(double) * 6 * n, c->s);
  cudaMemsetAsync(c->eps, 0, sizeof(double) * n, c->s);
  cudaMemsetAsync(c->strain_eq, 0, sizeof(double) * n, c->s);
  cudaMemsetAsync(c->wvel, 0, sizeof(double) * n, c->s);
  cudaMemsetAsync(c->acc, 0, sizeof(StepAccum), c->s);
  cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->s);
  cudaMemsetAsync(c->tmat, 0, sizeof(double) * 12 * n, c->s);
  if (cudaStreamSynchronize(c->s) != cudaSuccess) return fail(MEGA_ERR_CUDA);
  tr.mark("upload");
  r = mres ? mres : install_materials(c, ments, midx, mdamaged);
  if (r) return fail(r);
  tr.mark("materials");
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    g_ctxs.insert(c);
  }
  *handle = reinterpret_cast<int64_t>(c);
  return 0;
}

__global__ void k_offset_i32(int64_t m, const int32_t* __restrict__ src, int32_t add, int32_t* __restrict__ dst) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) dst[k] = src[k] + add;
}
__global__ void k_offset_i64(int64_t m, const int64_t* __restrict__ src, int64_t add, int64_t* __restrict__ dst) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) dst[k] = src[k] + add;
}

// Instances searched one at a time, each with its own bin grid (their node
// ranges may overlap in space; no instance sees another's nodes), then their
// lists merged into one block-diagonal CSR in the global numbering, with the
// cell orders concatenated into the renumbering.
static int search_instances(Ctx* c, DevCSR& csr, DevPool& out) {
  const int K = (int)c->inst_off.size() - 1;
  DevPool parts_pool(c->s);
  std::vector<DevCSR> parts(K);
  std::vector<int64_t> base(K + 1, 0);
  int32_t gmax = 0;
  for (int k = 0; k < K; ++k) {
    const int32_t o = c->inst_off[k], nk = c->inst_off[k + 1] - o;
    const double* dmax = c->inst_dmax.empty() ? c->p.dist_max : c->inst_dmax.data() + 3 * k;
    int r = bin_search(c->s, nk, c->coo + 3 * (int64_t)o, c->win + 3 * (int64_t)o,
                       c->sm_len ? c->sm_len + 6 * (int64_t)o : nullptr,
                       dmax, c->p.itype_int, c->p.shsup, c->status, parts[k], nullptr, parts_pool, nullptr,
                       c->perm + o);
    if (r) return r;
    k_offset_i32<<<grid_for(nk, 256), 256, 0, c->s>>>(nk, c->perm + o, o, c->perm + o);
    MEGA_CHECK_LAUNCH();
    base[k + 1] = base[k] + parts[k].nnz;
    gmax = std::max(gmax, parts[k].gmaxn);
  }
  const int32_t n = c->n;
  csr.n = n;
  csr.nnz = base[K];
  csr.gmaxn = gmax;
  MEGA_ALLOC(out, csr.rowptr, (int64_t)n + 1);
  MEGA_ALLOC(out, csr.col, csr.nnz);
  for (int k = 0; k < K; ++k) {
    const int32_t o = c->inst_off[k], nk = c->inst_off[k + 1] - o;
    // rows 0..nk of the part (its last offset doubles as the next part's first)
    k_offset_i64<<<grid_for((int64_t)nk + 1, 256), 256, 0, c->s>>>((int64_t)nk + 1, parts[k].rowptr, base[k],
                                                                    csr.rowptr + o);
    k_offset_i32<<<grid_for(parts[k].nnz, 256), 256, 0, c->s>>>(parts[k].nnz, parts[k].col, o, csr.col + base[k]);
    MEGA_CHECK_LAUNCH();
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

// Gather every per-node array through map (dst[r] = src[map[r]]): perm moves
// the original numbering to the bin-cell numbering, iperm moves it back.
static int permute_nodes(Ctx* c, const int32_t* map) {
  const int32_t n = c->n;
  struct Arr { void* p; int w; int es; };
  const Arr list[] = {
      {c->coo, 3, 8}, {c->win, 3, 8}, {c->mass, 3, 8}, {c->dsp, 3, 8}, {c->dsp_tot, 3, 8}, {c->dsp_tot_phy, 3, 8},
      {c->vel, 3, 8}, {c->acl, 3, 8}, {c->fint, 3, 8}, {c->fext, 3, 8}, {c->prforce, 3, 8}, {c->bodyforce, 3, 8},
      {c->sm_len, 6, 8}, {c->stress, 6, 8}, {c->strain, 6, 8}, {c->vol, 1, 8}, {c->eps, 1, 8},
      {c->strain_eq, 1, 8}, {c->wvel, 1, 8}, {c->ebc, 3, 1}, {c->body_id, 1, 1}, {c->ebc_nodes, 1, 4},
      {c->iters, 1, 4}, {c->matidx, 1, 2}, {c->aux, 4, 8}, {c->sgrad, 18, 8}};
  int64_t row_bytes = 0;  // the widest per-node row
  for (const Arr& a : list)
    if (a.p) row_bytes = std::max<int64_t>(row_bytes, (int64_t)a.w * a.es);
  DevPool tp(c->s);
  unsigned char* tmp = nullptr;
  MEGA_ALLOC(tp, tmp, (int64_t)n * row_bytes);
  for (const Arr& a : list) {
    if (!a.p) continue;
    k_perm_gather<<<grid_for((int64_t)n * a.w, 256), 256, 0, c->s>>>(n, a.w, a.es, map, (const unsigned char*)a.p,
                                                                       tmp);
    MEGA_CHECK_LAUNCH();
    MEGA_TRY(cudaMemcpyAsync(a.p, tmp, (size_t)n * a.w * a.es, cudaMemcpyDeviceToDevice, c->s));
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

int mega_search_and_shapes(int64_t h, int32_t* gn, int32_t* gstart, int32_t* gstack, int64_t dim_nn_list,
                           double* shp, double* dshp, int64_t* nnz, int32_t* gmaxn) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  const int32_t n = c->n;
  if (c->semi) return semi_search(c, gn, gstart, gstack, dim_nn_list, shp, dshp, nnz, gmaxn);
  if (c->searched) {  // back to the original numbering, then search afresh
    int r = permute_nodes(c, c->iperm);
    if (r) return r;
    c->nbpool.free_all();
    c->mixpool.free_all();
    c->csr = DevCSR();
    c->rt = TileSet();
    c->ct = TileSet();
    c->perm = c->iperm = nullptr;
    c->shp = c->sdphi = c->sdphi32 = c->tshp = c->tshp32 = c->shp32 = nullptr;
    c->pk64 = c->tpk64 = c->pk32 = c->tpk32 = nullptr;
    c->ns_srow = c->ns_scol = nullptr;
    c->ns_ssum = nullptr;
    c->banked = false;
    c->searched = false;
    if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
  }
  PhaseTrace tr(c->s, "search_and_shapes");
  // 1. search and shapes in the reference's numbering (what the caller may download)
  DevPool tmp0(c->s);
  DevCSR csr0;
  MEGA_ALLOC(c->nbpool, c->perm, n);
  MEGA_ALLOC(c->nbpool, c->iperm, n);
  int r = (c->inst_off.size() > 2) ? search_instances(c, csr0, tmp0)
                                   : bin_search(c->s, n, c->coo, c->win, c->sm_len, c->p.dist_max, c->p.itype_int,
                                                c->p.shsup, c->status, csr0, nullptr, tmp0, nullptr, c->perm);
  if (r) return r;
  tr.mark("bin_search");
  const int64_t m = csr0.nnz;
  // NSNI's smoothed second derivatives on the lists `csr` of the current
  // node order, one axis (two faces) at a time
  auto second_derivatives = [&](const DevCSR& csr, const NsniS& out) -> int {
    DevPool faces(c->s);
    double* g[6];
    for (int k = 0; k < 6; ++k) MEGA_ALLOC(faces, g[k], m);
    for (int ax = 0; ax < 3; ++ax) {
      int q;
      if ((q = rk_grad_at_face(c->s, c->p, n, c->coo, c->win, c->ebc_nodes, csr, c->sm_len, 2 * ax, g[0], g[1],
                               g[2], c->status)) ||
          (q = rk_grad_at_face(c->s, c->p, n, c->coo, c->win, c->ebc_nodes, csr, c->sm_len, 2 * ax + 1, g[3], g[4],
                               g[5], c->status)))
        return q;
      const double* gp[3] = {g[0], g[1], g[2]};
      const double* gm[3] = {g[3], g[4], g[5]};
      if ((q = nsni_combine(c->s, n, ax, csr.rowptr, c->sm_len, gp, gm, out))) return q;
    }
    MEGA_TRY(cudaStreamSynchronize(c->s));
    return 0;
  };
  // The shapes are computed in the caller's numbering only when the caller
  // asks for the lists; otherwise directly on the renumbered lists (each row
  // keeps its entries' order, so the values are the same to the bit).
  const bool want = gn || gstart || gstack || shp || dshp;
  double *shp0 = nullptr, *g0x = nullptr, *g0y = nullptr, *g0z = nullptr;
  NsniS s0{};
  int st = 0;
  if (want) {
    MEGA_ALLOC(tmp0, shp0, m);
    MEGA_ALLOC(tmp0, g0x, m);
    MEGA_ALLOC(tmp0, g0y, m);
    MEGA_ALLOC(tmp0, g0z, m);
    r = rk_shapes(c->s, c->p, n, c->coo, c->win, c->ebc_nodes, csr0, shp0, g0x, g0y, g0z, c->status);
    if (r) return r;
    tr.mark("rk_shapes");
    if (c->nsni) {
      for (int k = 0; k < 6; ++k) MEGA_ALLOC(tmp0, s0.v[k], m);
      if ((r = second_derivatives(csr0, s0))) return r;
      tr.mark("nsni_second_derivatives");
    }
    std::vector<int64_t> rp(n + 1);
    MEGA_TRY(cudaMemcpyAsync(rp.data(), csr0.rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    for (int32_t i = 0; i < n; ++i) {
      if (gn) gn[i] = (int32_t)(rp[i + 1] - rp[i]);
      if (gstart) gstart[i] = (int32_t)(rp[i] + 1);
    }
    if (gstack) {
      if (m > dim_nn_list) st |= MEGA_ST_STACK_OVERFLOW;
      else {
        MEGA_TRY(cudaMemcpyAsync(gstack, csr0.col, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, c->s));
        MEGA_TRY(cudaStreamSynchronize(c->s));
        for (int64_t k = 0; k < m; ++k) gstack[k] += 1;
      }
    }
    if (shp) MEGA_TRY(cudaMemcpyAsync(shp, shp0, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
    if (dshp) {
      std::vector<double> a(m), b(m), d(m);
      MEGA_TRY(cudaMemcpyAsync(a.data(), g0x, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
      MEGA_TRY(cudaMemcpyAsync(b.data(), g0y, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
      MEGA_TRY(cudaMemcpyAsync(d.data(), g0z, sizeof(double) * m, cudaMemcpyDeviceToHost, c->s));
      MEGA_TRY(cudaStreamSynchronize(c->s));
      for (int64_t k = 0; k < m; ++k) { dshp[3 * k] = a[k]; dshp[3 * k + 1] = b[k]; dshp[3 * k + 2] = d[k]; }
    }
    MEGA_TRY(cudaStreamSynchronize(c->s));
    tr.mark("downloads");
  }
  // 2. renumber the nodes in bin-cell order (spatially compact rows and tiles)
  k_iperm<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->perm, c->iperm);
  MEGA_CHECK_LAUNCH();
  r = permute_nodes(c, c->perm);
  if (r) return r;
  DevPool tmp1(c->s);
  int32_t* len1;
  MEGA_ALLOC(tmp1, len1, n);
  c->csr.n = n;
  c->csr.nnz = m;
  c->csr.gmaxn = csr0.gmaxn;
  MEGA_ALLOC(c->nbpool, c->csr.rowptr, (int64_t)n + 1);
  MEGA_ALLOC(c->nbpool, c->csr.col, m);
  MEGA_ALLOC(c->nbpool, c->shp, m);
  // Mixed precision alone (DNI, shapes not asked for): the shape kernel
  // writes the packed row records itself, so no double gradients are kept.
  const bool packed = !want && c->prec_mask == 2 && !c->nsni;
  double *g1x = nullptr, *g1y = nullptr, *g1z = nullptr;
  if (!packed) {
    MEGA_ALLOC(tmp1, g1x, m);
    MEGA_ALLOC(tmp1, g1y, m);
    MEGA_ALLOC(tmp1, g1z, m);
  }
  k_newrow_len<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->perm, csr0.rowptr, len1);
  MEGA_CHECK_LAUNCH();
  r = scan_counts(c->s, len1, c->csr.rowptr, n, tmp1);
  if (r) return r;
  if (c->nsni)
    for (int k = 0; k < 6; ++k) {
      MEGA_ALLOC(c->nbpool, c->nsr.v[k], m);
      MEGA_ALLOC(c->nbpool, c->nsc.v[k], m);
    }
  if (want) {
    k_permute_rows<<<grid_for((int64_t)n * 32, 256), 256, 0, c->s>>>(n, c->perm, c->iperm, csr0.rowptr, csr0.col,
                                                                      shp0, g0x, g0y, g0z, c->csr.rowptr, c->csr.col,
                                                                      c->shp, g1x, g1y, g1z);
    MEGA_CHECK_LAUNCH();
    if (c->nsni) {
      for (int k = 0; k < 6; k += 2)  // (the column indices are rewritten with the same values)
        k_permute_rows<<<grid_for((int64_t)n * 32, 256), 256, 0, c->s>>>(
            n, c->perm, c->iperm, csr0.rowptr, csr0.col, s0.v[k], s0.v[k + 1], s0.v[k], s0.v[k + 1], c->csr.rowptr,
            c->csr.col, c->nsr.v[k], c->nsr.v[k + 1], c->nsr.v[k], c->nsr.v[k + 1]);
      MEGA_CHECK_LAUNCH();
    }
  } else {
    k_renumber_cols<<<grid_for((int64_t)n * 32, 256), 256, 0, c->s>>>(n, c->perm, c->iperm, csr0.rowptr, csr0.col,
                                                                       c->csr.rowptr, c->csr.col);
    MEGA_CHECK_LAUNCH();
    if (packed) {  // the row tiles first: the records carry the tile ranks
      if ((r = configure_tiled_kernels())) return r;
      r = build_tiles(c->s, n, c->csr.rowptr, c->csr.col, m, c->csr.gmaxn, c->rt, c->nbpool, nullptr);
      if (r) return r;
      float4* a = nullptr;
      MEGA_ALLOC(c->nbpool, a, m);
      c->pk32 = a;
      r = rk_shapes_packed(c->s, c->p, n, c->coo, c->win, c->ebc_nodes, c->csr, c->rt.lidx, c->shp, a, c->status);
    } else {
      r = rk_shapes(c->s, c->p, n, c->coo, c->win, c->ebc_nodes, c->csr, c->shp, g1x, g1y, g1z, c->status);
    }
    if (r) return r;
    tr.mark("rk_shapes");
    if (c->nsni) {
      if ((r = second_derivatives(c->csr, c->nsr))) return r;
      tr.mark("nsni_second_derivatives");
    }
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  tmp0.free_all();
  tr.mark("renumber");
  // 3. transposed view, tiles, packed records
  r = configure_tiled_kernels();
  if (r) return r;
  r = build_transpose(c->s, c->csr, c->nbpool);
  if (r) return r;
  if (c->nsni) {
    for (int k = 0; k < 6; ++k)
      k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->csr.tpos, c->nsr.v[k], c->nsc.v[k]);
    MEGA_CHECK_LAUNCH();
  }
  tr.mark("transpose");
  if (!packed) {
    r = build_tiles(c->s, n, c->csr.rowptr, c->csr.col, m, c->csr.gmaxn, c->rt, c->nbpool, nullptr);
    if (r) return r;
  }
  tr.mark("row_tiles");
  // the longest column bounds a column tile's set from below
  r = build_tiles(c->s, n, c->csr.colptr, c->csr.trow, m, c->csr.gmaxc, c->ct, c->nbpool, nullptr);
  if (r) return r;
  tr.mark("column_tiles");
  if (c->prec_mask & 1) {
    double *a = nullptr, *b = nullptr;  // 4 doubles per entry
    MEGA_ALLOC(c->nbpool, a, 4 * m);
    MEGA_ALLOC(c->nbpool, b, 4 * m);
    c->pk64 = a;
    c->tpk64 = b;
    if ((r = pack_entries(c->s, m, c->rt.lidx, g1x, g1y, g1z, nullptr, true, c->pk64)) ||
        (r = pack_entries(c->s, m, c->ct.lidx, g1x, g1y, g1z, c->csr.tpos, true, c->tpk64)))
      return r;
    MEGA_ALLOC(c->nbpool, c->sdphi, 3 * (int64_t)n);
    k_rowsum3<double><<<grid_for(n, 256), 256, 0, c->s>>>(n, c->csr.rowptr, g1x, g1y, g1z, c->sdphi);
    MEGA_CHECK_LAUNCH();
  }
  // The float records are packed in list order here (rows in CSR order,
  // columns ascending rows); mega_autotune in mixed precision reorders them
  // once for the gathers' shared-memory banks (bank_layout).
  if (c->prec_mask & 2) {
    float4* b = nullptr;
    MEGA_ALLOC(c->nbpool, b, m);
    c->tpk32 = b;
    if (packed) {
      if ((r = pack_transposed32(c->s, m, c->ct.lidx, (const float4*)c->pk32, c->csr.tpos, b))) return r;
    } else {
      float4* a = nullptr;
      MEGA_ALLOC(c->nbpool, a, m);
      c->pk32 = a;
      if ((r = pack_entries(c->s, m, c->rt.lidx, g1x, g1y, g1z, nullptr, false, c->pk32)) ||
          (r = pack_entries(c->s, m, c->ct.lidx, g1x, g1y, g1z, c->csr.tpos, false, c->tpk32)))
        return r;
    }
    MEGA_ALLOC(c->nbpool, c->sdphi32, 3 * (int64_t)n);
    k_rowsum_pk32<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->csr.rowptr, (const float4*)c->pk32, c->sdphi32);
    MEGA_CHECK_LAUNCH();
    if (c->nsni) {  // S in both float record orders, and its row sums
      MEGA_ALLOC(c->nbpool, c->ns_srow, 6 * m);
      MEGA_ALLOC(c->nbpool, c->ns_scol, 6 * m);
      MEGA_ALLOC(c->nbpool, c->ns_ssum, 6 * (int64_t)n);
      if ((r = nsni_records(c->s, m, nullptr, c->nsr, c->ns_srow)) ||
          (r = nsni_records(c->s, m, c->csr.tpos, c->nsr, c->ns_scol)) ||
          (r = nsni_rowsum(c->s, n, c->csr.rowptr, c->nsr, c->ns_ssum)))
        return r;
    }
  }
  if (c->has_body && (c->prec_mask & 1)) {
    MEGA_ALLOC(c->nbpool, c->tshp, m);
    k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->csr.tpos, c->shp, c->tshp);
    MEGA_CHECK_LAUNCH();
  }
  if (c->has_body && (c->prec_mask & 2)) {
    MEGA_ALLOC(c->nbpool, c->tshp32, m);
    k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, c->csr.tpos, c->shp, c->tshp32);
    MEGA_CHECK_LAUNCH();
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  // the per-step kernels read neither the transposed row ids (but NSNI's
  // column gather) nor the positions
  if (!c->nsni) {
    c->nbpool.release(c->csr.trow);
    c->csr.trow = nullptr;
  }
  c->nbpool.release(c->csr.tpos);
  c->csr.tpos = nullptr;
  tmp1.free_all();
  tr.mark("pack_and_release");
  // the mixed NSNI force gather stages 27 values a node: its measured best is
  // 8 lanes per column (variant 3); mega_autotune may pick another
  if (c->nsni) c->var_force[1] = 3;
  c->searched = true;
  if (nnz) *nnz = m;
  if (gmaxn) *gmaxn = c->csr.gmaxn;
  int ds = read_status(c, true);
  if (ds < 0) return ds;
  return st | ds;
}

int mega_step_resident(int64_t h, int32_t nsteps, double dt, int32_t mode) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  int r = run_steps(c, nsteps, dt, mode);
  if (r) return r;
  return read_status(c, true);
}

int mega_step_timed(int64_t h, int32_t nsteps, double dt, int32_t mode, float* ms) {
  Ctx* c = get_ctx(h);
  if (!c || !ms) return c ? MEGA_ERR_ARG : MEGA_ERR_HANDLE;
  if (c->searched) { int r = ((mode & 0xff) == MEGA_MODE_MIXED) ? ensure_mixed(c) : ensure_fp64(c); if (r) return r; }
  if (c->searched && !c->semi && nsteps > 16) { int r = graph_for(c, dt, mode, 16); if (r) return r; }
  cudaEvent_t e0, e1;
  MEGA_TRY(cudaEventCreate(&e0));
  MEGA_TRY(cudaEventCreate(&e1));
  MEGA_TRY(cudaEventRecord(e0, c->s));
  int r = run_steps(c, nsteps, dt, mode);
  if (!r) {
    cudaEventRecord(e1, c->s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  return read_status(c, true);
}

int mega_kernel_times(int64_t h, int32_t reps, double dt, int32_t mode, float* out_ms) {
  Ctx* c = get_ctx(h);
  if (!c || !out_ms || reps <= 0) return c ? MEGA_ERR_ARG : MEGA_ERR_HANDLE;
  if (c->semi) return MEGA_ERR_UNSUPPORTED;  // the tiled gathers and instances are Lagrangian only
  if (!c->searched) return MEGA_ERR_STATE;
  { int r = ((mode & 0xff) == MEGA_MODE_MIXED) ? ensure_mixed(c) : ensure_fp64(c); if (r) return r; }
  if (!(mode & MEGA_FLAG_INTERP_EACH_STEP)) c->phy_valid = false;
  if (int r = sync_time(c)) return r;
  cudaEvent_t ev[4];
  for (auto& e : ev) MEGA_TRY(cudaEventCreate(&e));
  double acc[3] = {0, 0, 0};
  int r = launch_predict(c->s, 3 * (int64_t)c->n, c->dsp, c->dsp_tot, c->vel, c->acl, dt, c->ndt);
  for (int32_t k = 0; k < reps && !r; ++k) {
    r = step_once(c, dt, mode, k < reps - 1 ? 1 : 0, ev);
    if (r) break;
    cudaEventSynchronize(ev[3]);
    float t;
    for (int q = 0; q < 3; ++q) {
      cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
      acc[q] += t;
    }
    c->time = c->time + dt;
    c->steps += 1;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (r) return r;
  for (int q = 0; q < 3; ++q) out_ms[q] = (float)(acc[q] / reps);
  return read_status(c, true);
}

// Device array in the renumbered order -> host array in the caller's order.
static int download_nodes(Ctx* c, const void* src, int w, int es, void* dst) {
  const int32_t n = c->n;
  const size_t bytes = (size_t)n * w * es;
  if (!c->searched) {
    MEGA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    return 0;
  }
  DevPool tp(c->s);
  unsigned char* tmp = nullptr;
  MEGA_ALLOC(tp, tmp, bytes);
  k_perm_gather<<<grid_for((int64_t)n * w, 256), 256, 0, c->s>>>(n, w, es, c->iperm, (const unsigned char*)src, tmp);
  MEGA_CHECK_LAUNCH();
  return download_staged(c->s, dst, tmp, bytes);
}

int mega_download(int64_t h, int32_t field, double* dst) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!dst) return MEGA_ERR_ARG;
  const int64_t n = c->n, n3 = 3 * n;
  const double* src = nullptr;
  int w = 0;
  switch (field) {
    case MEGA_F_DSP: src = c->dsp; w = 3; break;
    case MEGA_F_DSP_TOT: src = c->dsp_tot; w = 3; break;
    case MEGA_F_VEL: src = c->vel; w = 3; break;
    case MEGA_F_ACL: src = c->acl; w = 3; break;
    case MEGA_F_FINT: src = c->fint; w = 3; break;
    case MEGA_F_FEXT: src = c->fext; w = 3; break;
    case MEGA_F_STRESS: src = c->stress; w = 6; break;
    case MEGA_F_STRAIN: src = c->strain; w = 6; break;
    case MEGA_F_EPS: src = c->eps; w = 1; break;
    case MEGA_F_STRAIN_EQ: src = c->strain_eq; w = 1; break;
    case MEGA_F_WAVE_VEL: src = c->wvel; w = 1; break;
    case MEGA_F_PRFORCE: src = c->prforce; w = 3; break;
    case MEGA_F_STATE_AUX:
      if (!c->aux) return MEGA_ERR_STATE;
      src = c->aux; w = 4; break;
    case MEGA_F_NSNI_SGRAD:
      if (!c->sgrad) return MEGA_ERR_STATE;
      src = c->sgrad; w = 18; break;
    case MEGA_F_NEWTON_IT: {
      std::vector<int32_t> it(n);
      int r = download_nodes(c, c->iters, 1, 4, it.data());
      if (r) return r;
      for (int64_t i = 0; i < n; ++i) dst[i] = it[i];
      return 0;
    }
    case MEGA_F_DSP_TOT_PHY:
    case MEGA_F_COO_CURRENT: {
      const double* phy = c->dsp_tot_phy;
      if (!c->phy_valid) {
        if (!c->searched) return MEGA_ERR_STATE;
        int r = launch_interp(c->s, c->n, c->csr, c->shp, c->dsp_tot, nullptr, c->scratch3);
        if (r) return r;
        phy = c->scratch3;
      }
      if (field == MEGA_F_COO_CURRENT) {  // x = X + the physical displacement (MAIN.F90:382-386), one copy out
        DevPool tp(c->s);
        double* x = nullptr;
        MEGA_ALLOC(tp, x, n3);
        k_add_kernel<<<grid_for(n3, 256), 256, 0, c->s>>>(n3, c->coo, phy, x);
        MEGA_CHECK_LAUNCH();
        return download_nodes(c, x, 3, 8, dst);
      }
      return download_nodes(c, phy, 3, 8, dst);
    }
    default: return MEGA_ERR_ARG;
  }
  return download_nodes(c, src, w, 8, dst);
}

// Several fields in one copy to the host (the output step of MAIN: the
// VTK writer's arrays), each in the caller's node order, one after another.
int mega_snapshot(int64_t h, int32_t nfields, const int32_t* fields, double* dst) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (nfields <= 0 || !fields || !dst) return MEGA_ERR_ARG;
  const int64_t n = c->n, n3 = 3 * n;
  std::vector<int> width(nfields);
  int64_t total = 0;
  for (int32_t f = 0; f < nfields; ++f) {
    int w = 0;
    switch (fields[f]) {
      case MEGA_F_DSP: case MEGA_F_DSP_TOT: case MEGA_F_VEL: case MEGA_F_ACL: case MEGA_F_FINT: case MEGA_F_FEXT:
      case MEGA_F_PRFORCE: case MEGA_F_COO_CURRENT: case MEGA_F_DSP_TOT_PHY: w = 3; break;
      case MEGA_F_STRESS: case MEGA_F_STRAIN: w = 6; break;
      case MEGA_F_EPS: case MEGA_F_STRAIN_EQ: case MEGA_F_WAVE_VEL: case MEGA_F_NEWTON_IT: w = 1; break;
      case MEGA_F_STATE_AUX: if (!c->aux) return MEGA_ERR_STATE; w = 4; break;
      case MEGA_F_NSNI_SGRAD: if (!c->sgrad) return MEGA_ERR_STATE; w = 18; break;
      default: return MEGA_ERR_ARG;
    }
    width[f] = w;
    total += n * w;
  }
  DevPool tp(c->s);
  double *out = nullptr, *tmp = nullptr;
  MEGA_ALLOC(tp, out, total);
  MEGA_ALLOC(tp, tmp, n3);
  int64_t off = 0;
  for (int32_t f = 0; f < nfields; ++f) {
    const int w = width[f];
    const double* src = nullptr;
    switch (fields[f]) {
      case MEGA_F_DSP: src = c->dsp; break;
      case MEGA_F_DSP_TOT: src = c->dsp_tot; break;
      case MEGA_F_VEL: src = c->vel; break;
      case MEGA_F_ACL: src = c->acl; break;
      case MEGA_F_FINT: src = c->fint; break;
      case MEGA_F_FEXT: src = c->fext; break;
      case MEGA_F_PRFORCE: src = c->prforce; break;
      case MEGA_F_STRESS: src = c->stress; break;
      case MEGA_F_STRAIN: src = c->strain; break;
      case MEGA_F_EPS: src = c->eps; break;
      case MEGA_F_STRAIN_EQ: src = c->strain_eq; break;
      case MEGA_F_WAVE_VEL: src = c->wvel; break;
      case MEGA_F_STATE_AUX: src = c->aux; break;
      case MEGA_F_NSNI_SGRAD: src = c->sgrad; break;
      case MEGA_F_NEWTON_IT:
        k_i32_to_f64<<<grid_for(n, 256), 256, 0, c->s>>>(n, c->iters, tmp);
        MEGA_CHECK_LAUNCH();
        src = tmp;
        break;
      default: {  // the physical displacement, or the current coordinates
        const double* phy = c->dsp_tot_phy;
        if (!c->phy_valid) {
          if (!c->searched) return MEGA_ERR_STATE;
          int r = launch_interp(c->s, c->n, c->csr, c->shp, c->dsp_tot, nullptr, tmp);
          if (r) return r;
          phy = tmp;
        }
        if (fields[f] == MEGA_F_COO_CURRENT) {
          k_add_kernel<<<grid_for(n3, 256), 256, 0, c->s>>>(n3, c->coo, phy, tmp);
          MEGA_CHECK_LAUNCH();
          phy = tmp;
        }
        src = phy;
      }
    }
    if (c->searched)
      k_perm_gather<<<grid_for(n * w, 256), 256, 0, c->s>>>((int32_t)n, w, 8, c->iperm, (const unsigned char*)src,
                                                             (unsigned char*)(out + off));
    else
      MEGA_TRY(cudaMemcpyAsync(out + off, src, sizeof(double) * n * w, cudaMemcpyDeviceToDevice, c->s));
    MEGA_CHECK_LAUNCH();
    off += n * w;
  }
  return download_staged(c->s, dst, out, sizeof(double) * (size_t)total);
}

int mega_upload(int64_t h, int32_t field, const double* src) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!src) return MEGA_ERR_ARG;
  const int32_t n = c->n;
  double* dst = nullptr;
  int w = 0;
  switch (field) {
    case MEGA_F_DSP: dst = c->dsp; w = 3; break;
    case MEGA_F_DSP_TOT: dst = c->dsp_tot; w = 3; c->phy_valid = false; break;
    case MEGA_F_VEL: dst = c->vel; w = 3; break;
    case MEGA_F_ACL: dst = c->acl; w = 3; break;
    case MEGA_F_FEXT: dst = c->fext; w = 3; break;
    case MEGA_F_STRESS: dst = c->stress; w = 6; break;
    case MEGA_F_STRAIN: dst = c->strain; w = 6; break;
    case MEGA_F_EPS: dst = c->eps; w = 1; break;
    case MEGA_F_STATE_AUX:
      if (!c->aux) return MEGA_ERR_STATE;
      dst = c->aux; w = 4; break;
    case MEGA_F_NSNI_SGRAD:
      if (!c->sgrad) return MEGA_ERR_STATE;
      dst = c->sgrad; w = 18; break;
    default: return MEGA_ERR_ARG;
  }
  const size_t bytes = (size_t)n * w * sizeof(double);
  if (!c->searched) {
    MEGA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    return 0;
  }
  DevPool tp(c->s);
  unsigned char* tmp = nullptr;
  MEGA_ALLOC(tp, tmp, bytes);
  MEGA_TRY(cudaMemcpyAsync(tmp, src, bytes, cudaMemcpyHostToDevice, c->s));
  k_perm_gather<<<grid_for((int64_t)n * w, 256), 256, 0, c->s>>>(n, w, 8, c->perm, tmp, (unsigned char*)dst);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

int mega_get_scalars(int64_t h, mega_scalars_t* out) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!out) return MEGA_ERR_ARG;
  StepAccum a;
  MEGA_TRY(cudaMemcpyAsync(&a, c->acc, sizeof(a), cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  out->time = c->time;
  out->int_energy = slot_sum(a.int_work);
  out->kin_energy = slot_sum(a.ke);
  out->ext_energy = slot_sum(a.ee);
  for (int k = 0; k < 6; ++k) out->total_force[k] = slot_sum(a.tf[k]);
  out->steps = c->steps;
  out->newton_iters = (int64_t)slot_sum(a.newton_iters);
  out->plastic_nodes = (int64_t)slot_sum(a.plastic);
  out->newton_iters_total = (int64_t)slot_sum(a.newton_total);
  out->plastic_nodes_total = (int64_t)slot_sum(a.plastic_total);
  return 0;
}

int64_t mega_device_bytes(int64_t h) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  return c->pool.bytes + c->nbpool.bytes + c->mixpool.bytes + c->mlppool.bytes;
}

int64_t mega_kernel_launches(int64_t h) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  return c->launches;
}

// Autotuner: time every launch variant of the two gathers on this context's
// own lists (reps launches each, CUDA events), keep the fastest, and put the
// state back as it was (the force kernel integrates when it runs).
// One-time reordering of a context's float records (at its first mixed
// autotune): the entries of each row and column take the order in which a
// warp's lanes read distinct shared-memory banks of the staged data
// (bank_order), and what travels with the records follows them (the
// interpolation and body-force shape values, the NSNI S values).  About 6 ms
// per gather on a 1 M-node bar; it pays back over a few hundred steps.
static void drop_graph(Ctx* c);

static int bank_layout(Ctx* c) {
  if (c->banked || !(c->prec_mask & 2) || !c->pk32 || !c->tpk32) return 0;
  const int64_t m = c->csr.nnz;
  const int32_t n = c->n;
  DevPool tmp(c->s);
  uint16_t* l = nullptr;
  int64_t* pos = nullptr;
  MEGA_ALLOC(tmp, l, m);
  MEGA_ALLOC(tmp, pos, m);
  int r = 0;
  // columns (the lanes per column of the force variant the context favours)
  if ((r = record_ranks(c->s, m, (const float4*)c->tpk32, l)) || (r = iota64(c->s, m, pos)) ||
      (r = bank_order(c->s, n, c->ct, c->csr.colptr, l, nullptr, pos, c->nsni ? 8 : 4)))
    return r;
  float4* tp = nullptr;
  MEGA_ALLOC(c->nbpool, tp, m);
  if ((r = gather_records32(c->s, m, pos, (const float4*)c->tpk32, tp))) return r;
  double* ts = nullptr;
  if (c->tshp32) {
    MEGA_ALLOC(c->nbpool, ts, m);
    k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, pos, c->tshp32, ts);
    MEGA_CHECK_LAUNCH();
  }
  float* sc = nullptr;
  if (c->ns_scol) {
    MEGA_ALLOC(c->nbpool, sc, 6 * m);
    if ((r = gather_f6(c->s, m, pos, c->ns_scol, sc))) return r;
  }
  // rows
  if ((r = record_ranks(c->s, m, (const float4*)c->pk32, l)) || (r = iota64(c->s, m, pos)) ||
      (r = bank_order(c->s, n, c->rt, c->csr.rowptr, l, nullptr, pos, 4)))
    return r;
  float4* rp = nullptr;
  double* sh = nullptr;
  MEGA_ALLOC(c->nbpool, rp, m);
  MEGA_ALLOC(c->nbpool, sh, m);
  if ((r = gather_records32(c->s, m, pos, (const float4*)c->pk32, rp))) return r;
  k_gather_pos<<<grid_for(m, 256), 256, 0, c->s>>>(m, pos, c->shp, sh);
  MEGA_CHECK_LAUNCH();
  float* sr = nullptr;
  if (c->ns_srow) {
    MEGA_ALLOC(c->nbpool, sr, 6 * m);
    if ((r = gather_f6(c->s, m, pos, c->ns_srow, sr))) return r;
  }
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);  // captured steps hold the old arrays
  c->nbpool.release(c->tpk32); c->tpk32 = tp;
  if (ts) { c->nbpool.release(c->tshp32); c->tshp32 = ts; }
  if (sc) { c->nbpool.release(c->ns_scol); c->ns_scol = sc; }
  c->nbpool.release(c->pk32); c->pk32 = rp;
  c->shp32 = sh;
  if (sr) { c->nbpool.release(c->ns_srow); c->ns_srow = sr; }
  c->banked = true;
  return 0;
}

int mega_autotune(int64_t h, double dt, int32_t mode, int32_t reps, int32_t* choice, float* times_ms) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (c->semi) return MEGA_ERR_UNSUPPORTED;  // the tiled gathers and instances are Lagrangian only
  if (!c->searched) return MEGA_ERR_STATE;
  if (reps <= 0) return MEGA_ERR_ARG;
  const bool mixed = (mode & 0xff) == MEGA_MODE_MIXED;
  { int r = mixed ? ensure_mixed(c) : ensure_fp64(c); if (r) return r; }
  if (mixed) { int r = bank_layout(c); if (r) return r; }
  const int nvar = tiled_variants();
  const size_t n = (size_t)c->n, n3 = 3 * n;
  // snapshot of everything a step writes
  struct Arr { void* p; size_t bytes; };
  const size_t ts = mixed ? sizeof(float) : sizeof(double);
  std::vector<Arr> arrs = {
      {c->dsp, 8 * n3}, {c->dsp_tot, 8 * n3}, {c->dsp_tot_phy, 8 * n3}, {c->vel, 8 * n3}, {c->acl, 8 * n3},
      {c->fint, 8 * n3}, {c->fext, 8 * n3}, {c->prforce, 8 * n3}, {c->stress, 48 * n}, {c->strain, 48 * n},
      {c->eps, 8 * n}, {c->strain_eq, 8 * n}, {c->wvel, 8 * n}, {c->fg, 144 * n}, {c->tmat, 12 * ts * n},
      {c->iters, 4 * n}, {c->acc, sizeof(StepAccum)}, {c->status, sizeof(unsigned)}};
  if (c->aux) arrs.push_back({c->aux, 32 * n});
  if (c->sgrad) arrs.push_back({c->sgrad, 144 * n});
  DevPool snap(c->s);
  std::vector<unsigned char*> copies;
  for (const Arr& a : arrs) {
    unsigned char* d = nullptr;
    MEGA_ALLOC(snap, d, a.bytes);
    MEGA_TRY(cudaMemcpyAsync(d, a.p, a.bytes, cudaMemcpyDeviceToDevice, c->s));
    copies.push_back(d);
  }
  cudaEvent_t e0, e1;
  MEGA_TRY(cudaEventCreate(&e0));
  MEGA_TRY(cudaEventCreate(&e1));
  std::vector<float> tdef(nvar, 0.f), tfor(nvar, 0.f);
  std::vector<bool> fits(nvar, true);
  int r = 0;
  const StressArgs sa = stress_args(c, dt, mode & 0xff);
  for (int v = 0; v < nvar && !r; ++v) {
    NsniTiles nt;
    const NsniTiles* ns = nsni_tiles(c, mixed, nt);
    const auto def = [&]() {
      return launch_defgrad_tiled(c->s, mixed, false, c->n, c->rt, ns, c->csr.rowptr, mixed ? c->pk32 : c->pk64,
                                  c->dsp, c->dsp_tot, mixed ? c->sdphi32 : c->sdphi, c->shp, c->dsp_tot_phy, c->fg,
                                  c->acc, c->status, v);
    };
    r = def();  // warm-up (twice: the first launch of a variant may also load its code)
    if (r == MEGA_ERR_UNSUPPORTED) {  // a streamed variant whose tiles do not fit shared memory
      fits[v] = false;
      r = 0;
      continue;
    }
    if (!r) r = def();
    if (r) break;
    MEGA_TRY(cudaStreamSynchronize(c->s));
    cudaEventRecord(e0, c->s);
    for (int k = 0; k < reps && !r; ++k) r = def();
    cudaEventRecord(e1, c->s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&tdef[v], e0, e1);
    if (r) break;
    r = launch_stress(c->s, mixed, sa);
    if (r) break;
    const TiledForceArgs fa = force_args(c, dt, mode & 0xff, 0);
    r = launch_force_tiled(c->s, mixed, fa, v);  // warm-up
    if (r == MEGA_ERR_UNSUPPORTED) {
      fits[v] = false;
      r = 0;
      continue;
    }
    if (!r) r = launch_force_tiled(c->s, mixed, fa, v);
    if (r) break;
    MEGA_TRY(cudaStreamSynchronize(c->s));
    cudaEventRecord(e0, c->s);
    for (int k = 0; k < reps && !r; ++k) r = launch_force_tiled(c->s, mixed, fa, v);
    cudaEventRecord(e1, c->s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&tfor[v], e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (size_t k = 0; k < arrs.size(); ++k)
    MEGA_TRY(cudaMemcpyAsync(arrs[k].p, copies[k], arrs[k].bytes, cudaMemcpyDeviceToDevice, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  if (r) return r;
  int bd = 0, bf = 0;
  for (int v = 1; v < nvar; ++v) {
    if (!fits[v]) { tdef[v] = tfor[v] = -1.f; continue; }  // reported as -1: not launchable on these tiles
    if (tdef[v] < tdef[bd]) bd = v;
    if (tfor[v] < tfor[bf]) bf = v;
  }
  c->var_defgrad[mixed] = bd;
  c->var_force[mixed] = bf;
  if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
  c->g_mode = -1;
  if (choice) { choice[0] = bd; choice[1] = bf; }
  if (times_ms)
    for (int v = 0; v < nvar; ++v) {
      times_ms[v] = fits[v] ? tdef[v] / reps : -1.f;
      times_ms[nvar + v] = fits[v] ? tfor[v] / reps : -1.f;
    }
  return read_status(c, true);
}

int mega_set_instances(int64_t h, int32_t ninst, const int32_t* inst_nodes, const double* dist_max) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (c->semi) return MEGA_ERR_UNSUPPORTED;  // the tiled gathers and instances are Lagrangian only
  if (ninst < 1 || !inst_nodes) return MEGA_ERR_ARG;
  std::vector<int32_t> off(ninst + 1, 0);
  for (int32_t k = 0; k < ninst; ++k) {
    if (inst_nodes[k] <= 0) return MEGA_ERR_ARG;
    off[k + 1] = off[k] + inst_nodes[k];
  }
  if (off[ninst] != c->n) return MEGA_ERR_ARG;
  c->inst_off = off;
  c->inst_dmax.clear();
  if (dist_max) c->inst_dmax.assign(dist_max, dist_max + 3 * (size_t)ninst);
  return 0;
}

int mega_set_precisions(int64_t h, int32_t mask) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (mask < 1 || mask > 3) return MEGA_ERR_ARG;
  if (c->searched && (mask & ~c->prec_mask)) return MEGA_ERR_STATE;  // records not built
  c->prec_mask = mask;
  return 0;
}

static void drop_graph(Ctx* c) {
  if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
  c->g_mode = -1;
}

__global__ void k_gather_inst_dt(int32_t n, const int32_t* __restrict__ perm, const double* __restrict__ src,
                                 double* __restrict__ dst) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) dst[r] = src[perm[r]];
}

int mega_set_instance_dt(int64_t h, const double* dt_inst) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!c->searched || c->semi) return MEGA_ERR_STATE;
  if (c->inst_off.size() < 2) return MEGA_ERR_STATE;  // not declared as instances
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);
  if (!dt_inst) { c->ndt = nullptr; return 0; }      // back to the call's dt for every node
  const size_t ninst = c->inst_off.size() - 1;
  std::vector<double> hd(c->n);
  for (size_t k = 0; k < ninst; ++k) {
    if (!(dt_inst[k] > 0.0)) return MEGA_ERR_ARG;
    for (int32_t i = c->inst_off[k]; i < c->inst_off[k + 1]; ++i) hd[i] = dt_inst[k];
  }
  if (!c->ndt) MEGA_ALLOC(c->pool, c->ndt, c->n);
  DevPool tp(c->s);
  double* tmp = nullptr;
  MEGA_ALLOC(tp, tmp, c->n);
  MEGA_TRY(cudaMemcpyAsync(tmp, hd.data(), sizeof(double) * c->n, cudaMemcpyHostToDevice, c->s));
  k_gather_inst_dt<<<grid_for(c->n, 256), 256, 0, c->s>>>(c->n, c->perm, tmp, c->ndt);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaStreamSynchronize(c->s));
  return 0;
}

int mega_set_variants(int64_t h, int32_t mode, int32_t defgrad_variant, int32_t force_variant) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!c->searched) return MEGA_ERR_STATE;
  const bool mixed = (mode & 0xff) == MEGA_MODE_MIXED;
  if ((mode & 0xff) != MEGA_MODE_FP64 && !mixed) return MEGA_ERR_ARG;
  if (defgrad_variant < 0 || defgrad_variant >= tiled_variants() || force_variant < 0 ||
      force_variant >= tiled_variants())
    return MEGA_ERR_ARG;
  if (!tiled_variant_fits(c->rt, mixed, defgrad_variant, false, c->has_body) ||
      !tiled_variant_fits(c->ct, mixed, force_variant, true, c->has_body))
    return MEGA_ERR_UNSUPPORTED;
  if (c->nsni && mixed && (defgrad_variant >= 4 || force_variant >= 4))  // the NSNI terms: register variants
    return MEGA_ERR_UNSUPPORTED;
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);
  c->var_defgrad[mixed] = defgrad_variant;
  c->var_force[mixed] = force_variant;
  return 0;
}

int mega_set_fixity2(int64_t h, int32_t steps, const double* ftime, const double* fdisp) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (steps < 0 || (steps > 0 && (!ftime || !fdisp))) return MEGA_ERR_ARG;
  for (int32_t k = 0; k < steps; ++k)  // READ.F90:265: a window may not end before it starts
    if (!(ftime[k] <= ftime[steps + k])) return MEGA_ERR_ARG;
  if (!c->has_ebc2) return MEGA_ERR_STATE;  // no DOF has fixity code 2
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);  // the captured window kernel names the old table
  if (steps > c->f2_steps || !c->f2) MEGA_ALLOC(c->pool, c->f2, 5 * (int64_t)std::max(steps, 1));
  std::vector<double> t(5 * (size_t)steps);
  std::memcpy(t.data(), ftime, sizeof(double) * 2 * steps);
  std::memcpy(t.data() + 2 * (size_t)steps, fdisp, sizeof(double) * 3 * steps);
  if (steps) MEGA_TRY(cudaMemcpyAsync(c->f2, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  c->f2_steps = steps;
  return 0;
}

int mega_set_surrogate(int64_t h, int32_t hidden, const float* theta) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);
  if (!theta) { c->mlp_on = false; return 0; }
  if (hidden != 64) return MEGA_ERR_UNSUPPORTED;
  const int np = mlp_nparams();
  if (!c->mlp_theta) {
    MEGA_ALLOC(c->mlppool, c->mlp_theta, np);
    MEGA_ALLOC(c->mlppool, c->mlp_w2, 64 * 64);
    MEGA_ALLOC(c->mlppool, c->mlp_small, 4 * 64 + 3 * 64 + 1);
    MEGA_ALLOC(c->mlppool, c->mlp_queue, c->n);
    MEGA_ALLOC(c->mlppool, c->mlp_qcount, 1);
  }
  MEGA_TRY(cudaMemcpyAsync(c->mlp_theta, theta, sizeof(float) * np, cudaMemcpyHostToDevice, c->s));
  int r = mlp_pack(c->s, c->mlp_theta, c->mlp_w2, c->mlp_small);
  if (r) return r;
  MEGA_TRY(cudaStreamSynchronize(c->s));
  c->mlp_on = true;
  return 0;
}

int mega_log_rate_samples(int64_t h, int64_t cap, int32_t stride, uint32_t seed) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (cap < 0 || stride <= 0) return MEGA_ERR_ARG;
  MEGA_TRY(cudaStreamSynchronize(c->s));
  drop_graph(c);
  if (c->log_buf) { c->mlppool.release(c->log_buf); c->log_buf = nullptr; }
  if (c->log_count) { c->mlppool.release(c->log_count); c->log_count = nullptr; }
  c->log_cap = 0;
  if (cap == 0) return 0;
  MEGA_ALLOC(c->mlppool, c->log_buf, 5 * cap);
  MEGA_ALLOC(c->mlppool, c->log_count, 1);
  MEGA_TRY(cudaMemsetAsync(c->log_count, 0, sizeof(unsigned long long), c->s));
  c->log_cap = cap;
  c->log_stride = (uint32_t)stride;
  c->log_seed = seed;
  return 0;
}

int mega_rate_samples(int64_t h, float* out, int64_t cap, int64_t* count) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!count || cap < 0) return MEGA_ERR_ARG;
  if (c->log_cap == 0) { *count = 0; return 0; }
  unsigned long long k = 0;
  MEGA_TRY(cudaMemcpyAsync(&k, c->log_count, sizeof(k), cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  const int64_t held = std::min<int64_t>((int64_t)k, c->log_cap);
  *count = held;
  if (out && held > 0) {
    const int64_t m = std::min<int64_t>(held, cap);
    MEGA_TRY(cudaMemcpyAsync(out, c->log_buf, sizeof(float) * 5 * m, cudaMemcpyDeviceToHost, c->s));
    MEGA_TRY(cudaStreamSynchronize(c->s));
    *count = m;
  }
  return 0;
}

int mega_train_surrogate(int64_t h, float* theta, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                         float* loss_per_epoch) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  if (!theta || epochs <= 0 || batch <= 0) return MEGA_ERR_ARG;
  if (c->log_cap == 0) return MEGA_ERR_STATE;
  unsigned long long k = 0;
  MEGA_TRY(cudaMemcpyAsync(&k, c->log_count, sizeof(k), cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  const int64_t ns = std::min<int64_t>((int64_t)k, c->log_cap);
  if (ns <= 0) return MEGA_ERR_STATE;
  const int np = mlp_nparams();
  if (!c->mlp_theta) {
    MEGA_ALLOC(c->mlppool, c->mlp_theta, np);
    MEGA_ALLOC(c->mlppool, c->mlp_w2, 64 * 64);
    MEGA_ALLOC(c->mlppool, c->mlp_small, 4 * 64 + 3 * 64 + 1);
    MEGA_ALLOC(c->mlppool, c->mlp_queue, c->n);
    MEGA_ALLOC(c->mlppool, c->mlp_qcount, 1);
  }
  drop_graph(c);
  MEGA_TRY(cudaMemcpyAsync(c->mlp_theta, theta, sizeof(float) * np, cudaMemcpyHostToDevice, c->s));
  int r = mlp_train_dev(c->s, c->mlp_theta, ns, c->log_buf, 5, c->log_buf + 4, 5, epochs, batch, lr, seed,
                        loss_per_epoch);
  if (r) return r;
  r = mlp_pack(c->s, c->mlp_theta, c->mlp_w2, c->mlp_small);
  if (r) return r;
  MEGA_TRY(cudaMemcpyAsync(theta, c->mlp_theta, sizeof(float) * np, cudaMemcpyDeviceToHost, c->s));
  MEGA_TRY(cudaStreamSynchronize(c->s));
  c->mlp_on = true;
  return 0;
}

int mega_release_cached_memory(void) {
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) { cudaGetLastError(); return MEGA_ERR_CUDA; }
  std::map<int, uint64_t> prev;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    prev.swap(g_prev_threshold);
  }
  std::set<int> devs;
  for (const auto& kv : prev) devs.insert(kv.first);
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    for (const auto& kv : g_blk) devs.insert(kv.second.dev);
  }
  int rc = 0;
  for (int dev : devs) {
    cudaStream_t s = nullptr;
    if (cudaSetDevice(dev) != cudaSuccess || make_stream(&s)) { cudaGetLastError(); rc = MEGA_ERR_CUDA; continue; }
    flush_blocks(dev, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = MEGA_ERR_CUDA;
    cudaStreamDestroy(s);
    cudaMemPool_t mp;
    if (cudaDeviceGetDefaultMemPool(&mp, dev) == cudaSuccess) {
      const auto it = prev.find(dev);
      if (it != prev.end()) {
        uint64_t thr = it->second;
        if (cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr) != cudaSuccess) rc = MEGA_ERR_CUDA;
      }
      if (cudaMemPoolTrimTo(mp, 0) != cudaSuccess) rc = MEGA_ERR_CUDA;
    } else {
      rc = MEGA_ERR_CUDA;
    }
    cudaGetLastError();
  }
  cudaSetDevice(cur);
  return rc;
}

int mega_gpu_finalize(int64_t h) {
  Ctx* c = get_ctx(h);
  if (!c) return MEGA_ERR_HANDLE;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    g_ctxs.erase(c);
  }
  cudaStreamSynchronize(c->s);
  delete c;
  return 0;
}

// ------------------------------------------------ stateless drop-ins
int mega_bin_search(int32_t n, const double* coo, const double* win, const double* sm_len, const double* dist_max,
                    int32_t itype_int, int32_t shsup, int32_t* gn, int32_t* gstart, int32_t* gstack,
                    int64_t dim_nn_list, int32_t* gmaxn, int32_t* ijk, int64_t* nnz) {
  if (n <= 0 || !coo || !win || !sm_len || !dist_max || !gn || !gstart || !gstack || !gmaxn) return MEGA_ERR_ARG;
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  cudaStream_t s = sg.s;
  DevPool pool;
  double *dc, *dw, *ds;
  int32_t* dijk = nullptr;
  unsigned* st;
  MEGA_ALLOC(pool, dc, 3 * (int64_t)n);
  MEGA_ALLOC(pool, dw, 3 * (int64_t)n);
  MEGA_ALLOC(pool, ds, 6 * (int64_t)n);
  MEGA_ALLOC(pool, st, 1);
  if (ijk) MEGA_ALLOC(pool, dijk, 3 * (int64_t)n);
  if ((r = upload(s, dc, coo, 3 * (size_t)n)) || (r = upload(s, dw, win, 3 * (size_t)n)) ||
      (r = upload(s, ds, sm_len, 6 * (size_t)n)))
    return r;
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  DevCSR csr;
  r = bin_search(s, n, dc, dw, ds, dist_max, itype_int, shsup, st, csr, dijk, pool, nullptr);
  if (r) return r;
  std::vector<int64_t> rp(n + 1);
  MEGA_TRY(cudaMemcpyAsync(rp.data(), csr.rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  if (ijk) MEGA_TRY(cudaMemcpyAsync(ijk, dijk, sizeof(int32_t) * 3 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  for (int32_t i = 0; i < n; ++i) {
    gn[i] = (int32_t)(rp[i + 1] - rp[i]);
    gstart[i] = (int32_t)(rp[i] + 1);
  }
  *gmaxn = csr.gmaxn;
  if (nnz) *nnz = csr.nnz;
  if (csr.nnz > dim_nn_list) return (int)(hst | MEGA_ST_STACK_OVERFLOW);
  MEGA_TRY(cudaMemcpyAsync(gstack, csr.col, sizeof(int32_t) * csr.nnz, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  for (int64_t k = 0; k < csr.nnz; ++k) gstack[k] += 1;
  return (int)hst;
}

int mega_rk_shapes(const mega_params* p, int32_t n, const double* coo, const double* win, const int32_t* ebc_nodes,
                   const int32_t* gn, const int32_t* gstart, const int32_t* gstack, int64_t nnz, double* shp,
                   double* dshp) {
  if (!p || n <= 0 || !coo || !win || !gn || !gstart || !gstack || !shp || !dshp) return MEGA_ERR_ARG;
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  cudaStream_t s = sg.s;
  DevPool pool;
  DevCSR csr;
  std::vector<int64_t> hpos;
  r = csr_from_host(s, n, gn, gstart, gstack, nnz, pool, csr, hpos);
  if (r) return r;
  double *dc, *dw, *dshp0, *dgx, *dgy, *dgz;
  int32_t* den = nullptr;
  unsigned* st;
  MEGA_ALLOC(pool, dc, 3 * (int64_t)n);
  MEGA_ALLOC(pool, dw, 3 * (int64_t)n);
  MEGA_ALLOC(pool, st, 1);
  if (ebc_nodes) MEGA_ALLOC(pool, den, n);
  MEGA_ALLOC(pool, dshp0, csr.nnz);
  MEGA_ALLOC(pool, dgx, csr.nnz);
  MEGA_ALLOC(pool, dgy, csr.nnz);
  MEGA_ALLOC(pool, dgz, csr.nnz);
  if ((r = upload(s, dc, coo, 3 * (size_t)n)) || (r = upload(s, dw, win, 3 * (size_t)n))) return r;
  if (ebc_nodes && (r = upload(s, den, ebc_nodes, (size_t)n))) return r;
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  r = rk_shapes(s, *p, n, dc, dw, den, csr, dshp0, dgx, dgy, dgz, st);
  if (r) return r;
  std::vector<double> a(csr.nnz), b(csr.nnz), d(csr.nnz), e(csr.nnz);
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(a.data(), dshp0, sizeof(double) * csr.nnz, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(b.data(), dgx, sizeof(double) * csr.nnz, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(d.data(), dgy, sizeof(double) * csr.nnz, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(e.data(), dgz, sizeof(double) * csr.nnz, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaStreamSynchronize(s));
  for (int64_t k = 0; k < csr.nnz; ++k) {
    const int64_t q = hpos[k];
    shp[q] = a[k];
    dshp[3 * q] = b[k]; dshp[3 * q + 1] = d[k]; dshp[3 * q + 2] = e[k];
  }
  return (int)hst;
}

int mega_hughes_winget(const mega_params* p, int32_t n, const double* lmat, double* rot, double* strain, double* d) {
  if (!p || n <= 0 || !lmat || !rot || !strain || !d) return MEGA_ERR_ARG;
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  DevPool pool;
  double *dl, *dr, *ds, *dd;
  MEGA_ALLOC(pool, dl, 9 * (int64_t)n);
  MEGA_ALLOC(pool, dr, 9 * (int64_t)n);
  MEGA_ALLOC(pool, ds, 6 * (int64_t)n);
  MEGA_ALLOC(pool, dd, 6 * (int64_t)n);
  if ((r = upload(sg.s, dl, lmat, 9 * (size_t)n))) return r;
  k_hw<<<grid_for(n, 128), 128, 0, sg.s>>>(n, dl, dr, ds, dd, p->inv3_exact);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaMemcpyAsync(rot, dr, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaMemcpyAsync(strain, ds, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaMemcpyAsync(d, dd, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaStreamSynchronize(sg.s));
  return 0;
}

int mega_rotate_tensor(int32_t n, const double* rot, double* vtensor) {
  if (n <= 0 || !rot || !vtensor) return MEGA_ERR_ARG;
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  DevPool pool;
  double *dr, *dv;
  MEGA_ALLOC(pool, dr, 9 * (int64_t)n);
  MEGA_ALLOC(pool, dv, 6 * (int64_t)n);
  if ((r = upload(sg.s, dr, rot, 9 * (size_t)n)) || (r = upload(sg.s, dv, vtensor, 6 * (size_t)n))) return r;
  k_rotate<<<grid_for(n, 128), 128, 0, sg.s>>>(n, dr, dv);
  MEGA_CHECK_LAUNCH();
  MEGA_TRY(cudaMemcpyAsync(vtensor, dv, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaStreamSynchronize(sg.s));
  return 0;
}

int mega_constitution(const mega_params* p, int32_t n, const double* stress_pred, const int32_t* mat_type,
                      const double* props, double dlt, double* state, double* stress, int32_t* iters) {
  if (!p || n <= 0 || !stress_pred || !mat_type || !props || !state || !stress) return MEGA_ERR_ARG;
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  DevPool pool;
  double *dp, *dprop, *dst, *dsig;
  int32_t *dm, *dit = nullptr;
  unsigned* st;
  MEGA_ALLOC(pool, dp, 6 * (int64_t)n);
  MEGA_ALLOC(pool, dprop, 30 * (int64_t)n);
  MEGA_ALLOC(pool, dst, 20 * (int64_t)n);
  MEGA_ALLOC(pool, dsig, 6 * (int64_t)n);
  MEGA_ALLOC(pool, dm, n);
  MEGA_ALLOC(pool, st, 1);
  if (iters) MEGA_ALLOC(pool, dit, n);
  if ((r = upload(sg.s, dp, stress_pred, 6 * (size_t)n)) || (r = upload(sg.s, dprop, props, 30 * (size_t)n)) ||
      (r = upload(sg.s, dst, state, 20 * (size_t)n)) || (r = upload(sg.s, dm, mat_type, (size_t)n)))
    return r;
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), sg.s));
  k_constitution<<<grid_for(n, 128), 128, 0, sg.s>>>(n, dp, dm, dprop, dlt, p->newton_max_iter, p->rate_solver,
                                                     p->newton_rtol, dst,
                                                     dsig, dit, st);
  MEGA_CHECK_LAUNCH();
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(state, dst, sizeof(double) * 20 * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaMemcpyAsync(stress, dsig, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, sg.s));
  if (iters) MEGA_TRY(cudaMemcpyAsync(iters, dit, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, sg.s));
  MEGA_TRY(cudaStreamSynchronize(sg.s));
  return (int)hst;
}

// The inputs and outputs of one CONSTRUCT_FINT call (FINT.F90:16-25); the
// pointers after `gint_work` may be null unless the path needs them.
struct FintIO {
  int32_t n;
  const double *gcoo, *gwin, *gvol, *gprop, *bodyforce;
  const int32_t *gmat_type, *gebc_nodes, *gn, *gstart, *gstack;
  int64_t nnz;
  double *gstate, *gstress, *gstrain;
  const double *gdinc, *gdinc_tot;
  double *gstack_shp, *gstack_dshp;
  int32_t linit;
  double dlt;
  double *fint, *fext, *gmax_wvel, *gstrain_eq, *gint_work;
  const double* gcoo_current;   // semi-Lagrangian: shapes on the current coordinates
  const double* gsm_len;        // NSNI: smoothing cells (6, n)
  double* gstack_ddshp;         // NSNI: smoothed second derivatives (6, nnz)
  double *dx_stress, *dy_stress, *dz_stress;  // NSNI: LOCAL_DX/DY/DZ_STRESS (6, n) in/out
};

static int construct_fint_impl(const mega_params* p, const FintIO& io) {
  const int32_t n = io.n;
  const bool semi = p->lagrangian == 0, nsni = p->itype_int == 2;
  if (p->itype_int != 0 && p->itype_int != 2) return MEGA_ERR_UNSUPPORTED;
  if (semi && nsni) return MEGA_ERR_UNSUPPORTED;  // the semi-Lagrangian path is DNI (as the resident one)
  if (semi && !io.gcoo_current) return MEGA_ERR_ARG;
  if (nsni && (!io.gsm_len || !io.gstack_ddshp || !io.dx_stress || !io.dy_stress || !io.dz_stress))
    return MEGA_ERR_ARG;
  const bool shapes_here = io.linit || semi;  // RK1 in this call (FINT.F90:387-436)
  StreamGuard sg;
  int r = make_stream(&sg.s);
  if (r) return r;
  cudaStream_t s = sg.s;
  DevPool pool;
  DevCSR csr;
  std::vector<int64_t> hpos;
  r = csr_from_host(s, n, io.gn, io.gstart, io.gstack, io.nnz, pool, csr, hpos);
  if (r) return r;
  r = build_transpose(s, csr, pool);
  if (r) return r;
  const int64_t n3 = 3 * (int64_t)n, m = csr.nnz;
  double *dc, *dw, *dv, *dsh, *dgx, *dgy, *dgz, *tgx, *tgy, *tgz, *tsh = nullptr, *sd, *ddsp, *dtot, *dsig, *deps6,
         *dep, *deq, *dwv, *dfg, *dT, *dfi, *dfe, *dbf = nullptr, *dcur = nullptr, *dsml = nullptr;
  int32_t* den = nullptr;
  uint16_t* midx;
  StepAccum* acc;
  unsigned* st;
  MEGA_ALLOC(pool, dc, n3); MEGA_ALLOC(pool, dw, n3); MEGA_ALLOC(pool, dv, n);
  MEGA_ALLOC(pool, dsh, m); MEGA_ALLOC(pool, dgx, m); MEGA_ALLOC(pool, dgy, m); MEGA_ALLOC(pool, dgz, m);
  MEGA_ALLOC(pool, tgx, m); MEGA_ALLOC(pool, tgy, m); MEGA_ALLOC(pool, tgz, m);
  MEGA_ALLOC(pool, sd, n3); MEGA_ALLOC(pool, ddsp, n3); MEGA_ALLOC(pool, dtot, n3);
  MEGA_ALLOC(pool, dsig, 6 * (int64_t)n); MEGA_ALLOC(pool, deps6, 6 * (int64_t)n); MEGA_ALLOC(pool, dep, n);
  MEGA_ALLOC(pool, deq, n); MEGA_ALLOC(pool, dwv, n); MEGA_ALLOC(pool, dfg, 18 * (int64_t)n);
  MEGA_ALLOC(pool, dT, 12 * (int64_t)n); MEGA_ALLOC(pool, dfi, n3); MEGA_ALLOC(pool, dfe, n3);
  MEGA_ALLOC(pool, midx, n); MEGA_ALLOC(pool, acc, 1); MEGA_ALLOC(pool, st, 1);
  bool has_body = p->gravity[0] != 0.0 || p->gravity[1] != 0.0 || p->gravity[2] != 0.0;
  if (io.bodyforce)
    for (int64_t k = 0; k < n3 && !has_body; ++k) has_body = io.bodyforce[k] != 0.0;
  if (has_body) {
    MEGA_ALLOC(pool, tsh, m);
    if (io.bodyforce) { MEGA_ALLOC(pool, dbf, n3); if ((r = upload(s, dbf, io.bodyforce, n3))) return r; }
  }
  if (io.gebc_nodes) { MEGA_ALLOC(pool, den, n); if ((r = upload(s, den, io.gebc_nodes, (size_t)n))) return r; }
  if (semi) { MEGA_ALLOC(pool, dcur, n3); if ((r = upload(s, dcur, io.gcoo_current, n3))) return r; }
  if (nsni) { MEGA_ALLOC(pool, dsml, 6 * (int64_t)n); if ((r = upload(s, dsml, io.gsm_len, 6 * (size_t)n))) return r; }
  // material table (per call)
  std::vector<uint16_t> hidx;
  std::vector<MatEntry> ents;
  bool damaged = false;
  if ((r = material_table(n, io.gprop, io.gmat_type, 65535, ents, hidx, damaged))) return r;
  MatEntry* dmat;
  MEGA_ALLOC(pool, dmat, ents.size());
  std::vector<double> hs(n), hax;
  for (int32_t i = 0; i < n; ++i) hs[i] = io.gstate[20 * (size_t)i + 2];
  double* dax = nullptr;  // GSTATE(1, 2, 4, 5) when a damaged model is present
  if (damaged) {
    MEGA_ALLOC(pool, dax, 4 * (int64_t)n);
    hax.resize(4 * (size_t)n);
    for (int32_t i = 0; i < n; ++i) {
      const double* g = io.gstate + 20 * (size_t)i;
      hax[4 * (size_t)i] = g[0]; hax[4 * (size_t)i + 1] = g[1]; hax[4 * (size_t)i + 2] = g[3];
      hax[4 * (size_t)i + 3] = g[4];
    }
    if ((r = upload(s, dax, hax.data(), hax.size()))) return r;
  }
  if ((r = upload(s, dc, io.gcoo, n3)) || (r = upload(s, dw, io.gwin, n3)) || (r = upload(s, dv, io.gvol, (size_t)n)) ||
      (r = upload(s, ddsp, io.gdinc, n3)) || (r = upload(s, dsig, io.gstress, 6 * (size_t)n)) ||
      (r = upload(s, deps6, io.gstrain, 6 * (size_t)n)) || (r = upload(s, dep, hs.data(), (size_t)n)) ||
      (r = upload(s, midx, hidx.data(), (size_t)n)) || (r = upload(s, dmat, ents.data(), ents.size())))
    return r;
  // the total displacement pushes the gradients forward; on the
  // semi-Lagrangian path they are current already (F = I, FINT.F90:410-436)
  if (semi) MEGA_TRY(cudaMemsetAsync(dtot, 0, sizeof(double) * n3, s));
  else if ((r = upload(s, dtot, io.gdinc_tot, n3))) return r;
  MEGA_TRY(cudaMemsetAsync(acc, 0, sizeof(StepAccum), s));
  MEGA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  if (shapes_here) {
    r = rk_shapes(s, *p, n, semi ? dcur : dc, dw, den, csr, dsh, dgx, dgy, dgz, st);
    if (r) return r;
  } else {
    std::vector<double> a(m), b(m), d(m), e(m);
    for (int64_t k = 0; k < m; ++k) {
      const int64_t q = hpos[k];
      a[k] = io.gstack_shp[q];
      b[k] = io.gstack_dshp[3 * q]; d[k] = io.gstack_dshp[3 * q + 1]; e[k] = io.gstack_dshp[3 * q + 2];
    }
    if ((r = upload(s, dsh, a.data(), m)) || (r = upload(s, dgx, b.data(), m)) || (r = upload(s, dgy, d.data(), m)) ||
        (r = upload(s, dgz, e.data(), m)))
      return r;
    MEGA_TRY(cudaStreamSynchronize(s));
  }
  // NSNI: second derivatives (computed at LINIT, read otherwise) in CSR and
  // CSC order, stress gradients, per-call scratch
  NsniS nsr{}, nsc{};
  double *sgrad = nullptr, *hq = nullptr, *nsw = nullptr, *fstab = nullptr, *sprev = nullptr;
  if (nsni) {
    for (int k = 0; k < 6; ++k) { MEGA_ALLOC(pool, nsr.v[k], m); MEGA_ALLOC(pool, nsc.v[k], m); }
    MEGA_ALLOC(pool, sgrad, 18 * (int64_t)n); MEGA_ALLOC(pool, hq, 18 * (int64_t)n);
    MEGA_ALLOC(pool, nsw, 18 * (int64_t)n); MEGA_ALLOC(pool, fstab, n3); MEGA_ALLOC(pool, sprev, 6 * (int64_t)n);
    if (io.linit) {
      DevPool faces(s);
      double* g[6];
      for (int k = 0; k < 6; ++k) MEGA_ALLOC(faces, g[k], m);
      for (int ax = 0; ax < 3; ++ax) {
        if ((r = rk_grad_at_face(s, *p, n, dc, dw, den, csr, dsml, 2 * ax, g[0], g[1], g[2], st)) ||
            (r = rk_grad_at_face(s, *p, n, dc, dw, den, csr, dsml, 2 * ax + 1, g[3], g[4], g[5], st)))
          return r;
        const double* gp[3] = {g[0], g[1], g[2]};
        const double* gm[3] = {g[3], g[4], g[5]};
        if ((r = nsni_combine(s, n, ax, csr.rowptr, dsml, gp, gm, nsr))) return r;
      }
      MEGA_TRY(cudaStreamSynchronize(s));
    } else {
      std::vector<double> v(m);
      for (int k = 0; k < 6; ++k) {
        for (int64_t e = 0; e < m; ++e) v[e] = io.gstack_ddshp[6 * hpos[e] + k];
        if ((r = upload(s, nsr.v[k], v.data(), m))) return r;
        MEGA_TRY(cudaStreamSynchronize(s));
      }
    }
    for (int k = 0; k < 6; ++k) k_gather_pos<<<grid_for(m, 256), 256, 0, s>>>(m, csr.tpos, nsr.v[k], nsc.v[k]);
    MEGA_CHECK_LAUNCH();
    std::vector<double> hg(18 * (size_t)n);
    for (int32_t i = 0; i < n; ++i)
      for (int k = 0; k < 6; ++k) {
        hg[18 * (size_t)i + k] = io.dx_stress[6 * (size_t)i + k];
        hg[18 * (size_t)i + 6 + k] = io.dy_stress[6 * (size_t)i + k];
        hg[18 * (size_t)i + 12 + k] = io.dz_stress[6 * (size_t)i + k];
      }
    if ((r = upload(s, sgrad, hg.data(), hg.size()))) return r;
    MEGA_TRY(cudaMemcpyAsync(sprev, dsig, sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, s));
    MEGA_TRY(cudaStreamSynchronize(s));
  }
  const unsigned g = grid_for(m, 256);
  k_gather_pos<<<g, 256, 0, s>>>(m, csr.tpos, dgx, tgx);
  k_gather_pos<<<g, 256, 0, s>>>(m, csr.tpos, dgy, tgy);
  k_gather_pos<<<g, 256, 0, s>>>(m, csr.tpos, dgz, tgz);
  if (has_body) k_gather_pos<<<g, 256, 0, s>>>(m, csr.tpos, dsh, tsh);
  k_rowsum3<double><<<grid_for(n, 256), 256, 0, s>>>(n, csr.rowptr, dgx, dgy, dgz, sd);
  MEGA_CHECK_LAUNCH();
  r = launch_defgrad(s, false, false, n, csr, dgx, dgy, dgz, ddsp, dtot, sd, dsh, nullptr, dfg, acc);
  if (r) return r;
  StressArgs a{};
  a.n = n; a.fg = dfg; a.matidx = midx; a.mats = dmat; a.vol = dv; a.stress = dsig; a.strain = deps6; a.eps = dep;
  a.strain_eq = deq; a.wvel = dwv; a.tmat = dT; a.bodyforce = dbf; a.aux = dax;
  a.grav[0] = p->gravity[0]; a.grav[1] = p->gravity[1]; a.grav[2] = p->gravity[2];
  a.has_body = has_body; a.inv3_exact = p->inv3_exact; a.finite_strain = p->finite_strain;
  a.maxit = p->newton_max_iter; a.rate_solver = p->rate_solver; a.rtol = p->newton_rtol; a.dt = io.dlt; a.acc = acc;
  a.status = st;
  NsniStepArgs na{};
  if (nsni) {
    na.n = n; na.fg = dfg; na.stress_old = sprev; na.stress_new = dsig; na.sml = dsml; na.vol = dv; na.matidx = midx;
    na.mats = dmat; na.hq = hq; na.sgrad = sgrad; na.w = nsw; na.fstab = fstab; na.finite_strain = p->finite_strain;
    na.inv3_exact = p->inv3_exact; na.acc = acc; na.status = st;
    if ((r = nsni_step(s, na, csr, nsr, nsc, false, ddsp, 0))) return r;
  }
  r = launch_stress(s, false, a);
  if (r) return r;
  if (nsni && ((r = nsni_step(s, na, csr, nsr, nsc, false, ddsp, 1)) || (r = nsni_step(s, na, csr, nsr, nsc, false,
                                                                                       ddsp, 2))))
    return r;
  DevCSR* dcsr;
  MEGA_ALLOC(pool, dcsr, 1);
  if ((r = upload(s, dcsr, &csr, 1))) return r;
  ForceArgs f{};
  f.n = n; f.csr = dcsr; f.tgx = tgx; f.tgy = tgy; f.tgz = tgz; f.tshp = tsh; f.tmat = dT; f.has_body = has_body;
  f.integrate = 0; f.predict = 0; f.fint = dfi; f.fext = dfe; f.acc = acc; f.status = st;
  r = launch_force(s, false, f);
  if (r) return r;
  if (nsni) {  // the stabilisation force joins the internal force (FINT.F90:1127-1208)
    k_add_kernel<<<grid_for(n3, 256), 256, 0, s>>>(n3, dfi, fstab, dfi);
    MEGA_CHECK_LAUNCH();
  }
  StepAccum hacc;
  unsigned hst = 0;
  MEGA_TRY(cudaMemcpyAsync(io.fint, dfi, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(io.fext, dfe, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(io.gstress, dsig, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(io.gstrain, deps6, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(hs.data(), dep, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if (damaged) MEGA_TRY(cudaMemcpyAsync(hax.data(), dax, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(io.gmax_wvel, dwv, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(io.gstrain_eq, deq, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, s));
  MEGA_TRY(cudaMemcpyAsync(&hst, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  if (shapes_here) {  // GSTACK_SHP / GSTACK_DSHP written where RK1 ran (FINT.F90:427-434, 580-587)
    std::vector<double> a2(m), b(m), d(m), e(m);
    MEGA_TRY(cudaMemcpyAsync(a2.data(), dsh, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaMemcpyAsync(b.data(), dgx, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaMemcpyAsync(d.data(), dgy, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaMemcpyAsync(e.data(), dgz, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    MEGA_TRY(cudaStreamSynchronize(s));
    for (int64_t k = 0; k < m; ++k) {
      const int64_t q = hpos[k];
      io.gstack_shp[q] = a2[k];
      io.gstack_dshp[3 * q] = b[k]; io.gstack_dshp[3 * q + 1] = d[k]; io.gstack_dshp[3 * q + 2] = e[k];
    }
  }
  if (nsni) {
    std::vector<double> hg(18 * (size_t)n);
    MEGA_TRY(cudaMemcpyAsync(hg.data(), sgrad, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost, s));
    std::vector<std::vector<double>> dd;
    if (io.linit) {
      dd.assign(6, std::vector<double>(m));
      for (int k = 0; k < 6; ++k)
        MEGA_TRY(cudaMemcpyAsync(dd[k].data(), nsr.v[k], sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    }
    MEGA_TRY(cudaStreamSynchronize(s));
    for (int32_t i = 0; i < n; ++i)
      for (int k = 0; k < 6; ++k) {
        io.dx_stress[6 * (size_t)i + k] = hg[18 * (size_t)i + k];
        io.dy_stress[6 * (size_t)i + k] = hg[18 * (size_t)i + 6 + k];
        io.dz_stress[6 * (size_t)i + k] = hg[18 * (size_t)i + 12 + k];
      }
    if (io.linit)
      for (int64_t e = 0; e < m; ++e)
        for (int k = 0; k < 6; ++k) io.gstack_ddshp[6 * hpos[e] + k] = dd[k][e];
  }
  MEGA_TRY(cudaStreamSynchronize(s));
  for (int32_t i = 0; i < n; ++i) io.gstate[20 * (size_t)i + 2] = hs[i];
  if (damaged)
    for (int32_t i = 0; i < n; ++i) {
      double* gs = io.gstate + 20 * (size_t)i;
      gs[0] = hax[4 * (size_t)i]; gs[1] = hax[4 * (size_t)i + 1]; gs[3] = hax[4 * (size_t)i + 2];
      gs[4] = hax[4 * (size_t)i + 3];
    }
  *io.gint_work += slot_sum(hacc.int_work);
  return (int)hst;
}

int mega_construct_fint(const mega_params* p, int32_t n, const double* gcoo, const double* gwin, const double* gvol,
                        const double* gprop, const int32_t* gmat_type, const int32_t* gebc_nodes,
                        const double* bodyforce, double* gstate, double* gstress, double* gstrain,
                        const double* gdinc, const double* gdinc_tot, const int32_t* gn, const int32_t* gstart,
                        const int32_t* gstack, int64_t nnz, double* gstack_shp, double* gstack_dshp,
                        int32_t linit, double dlt, double* fint, double* fext, double* gmax_wvel,
                        double* gstrain_eq, double* gint_work) {
  if (!p || n <= 0 || !gcoo || !gwin || !gvol || !gprop || !gmat_type || !gstate || !gstress || !gstrain ||
      !gdinc || !gdinc_tot || !gn || !gstart || !gstack || !gstack_shp || !gstack_dshp || !fint || !fext ||
      !gmax_wvel || !gstrain_eq || !gint_work)
    return MEGA_ERR_ARG;
  // this short list has no room for the NSNI arrays or the current
  // coordinates: construct_fint_gpu takes the full list
  if (p->lagrangian != 1 || p->itype_int == 2) return MEGA_ERR_UNSUPPORTED;
  FintIO io{};
  io.n = n; io.gcoo = gcoo; io.gwin = gwin; io.gvol = gvol; io.gprop = gprop; io.bodyforce = bodyforce;
  io.gmat_type = gmat_type; io.gebc_nodes = gebc_nodes; io.gn = gn; io.gstart = gstart; io.gstack = gstack;
  io.nnz = nnz; io.gstate = gstate; io.gstress = gstress; io.gstrain = gstrain; io.gdinc = gdinc;
  io.gdinc_tot = gdinc_tot; io.gstack_shp = gstack_shp; io.gstack_dshp = gstack_dshp; io.linit = linit; io.dlt = dlt;
  io.fint = fint; io.fext = fext; io.gmax_wvel = gmax_wvel; io.gstrain_eq = gstrain_eq; io.gint_work = gint_work;
  return construct_fint_impl(p, io);
}

static std::mutex g_control_mu;
static mega_params g_control{};
static bool g_control_set = false;

int mega_fint_control(const mega_params* p) {
  if (!p) return MEGA_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_control_mu);
  g_control = *p;
  g_control_set = true;
  return 0;
}

}  // extern "C"

namespace mega {
int fint_control_get(mega_params* out) {
  std::lock_guard<std::mutex> lk(g_control_mu);
  if (!g_control_set) return MEGA_ERR_STATE;
  *out = g_control;
  return 0;
}
}  // namespace mega

extern "C" {

int construct_fint_gpu(const double* gwin, const double* gvol, const int32_t* gnump, const double* gcoo,
                       const double* gcoo_cuurent, const double* gsm_len, const double* gsm_area,
                       const double* gsm_vol, const double* gnsni_fac, const int32_t* gghost, const double* gprop,
                       double* gstate, double* gstress, double* gstrain, double* g_h_stress, double* g_s_stress,
                       const double* gdinc, const double* gdinc_tot, const int32_t* gmat_type,
                       const int32_t* gebc_nodes, const int32_t* gn, const int32_t* gstart,
                       const int32_t* dim_nn_list, const int32_t* gstack, double* gstack_shp, double* gstack_dshp,
                       double* gstack_ddshp, const int32_t* gmaxn, double* ginvk, const int32_t* linit, double* fint,
                       double* fext, double* dlt_fint, double* gchar_dist, double* gmax_wvel,
                       double* local_dx_stress, double* local_dy_stress, double* local_dz_stress,
                       const double* g_x_mom, const double* g_y_mom, const double* g_z_mom,
                       const double* model_bodyforce, double* gint_work, const int32_t* model_body_id,
                       double* gstrain_eq, const double* dlt) {
  (void)gsm_area; (void)gsm_vol; (void)gnsni_fac; (void)gghost; (void)g_h_stress; (void)g_s_stress;
  (void)gmaxn; (void)ginvk; (void)dlt_fint; (void)gchar_dist; (void)g_x_mom; (void)g_y_mom; (void)g_z_mom;
  (void)model_body_id;
  mega_params p;
  {
    std::lock_guard<std::mutex> lk(g_control_mu);
    if (!g_control_set) return MEGA_ERR_STATE;  // mega_fint_control first
    p = g_control;
  }
  if (!gnump || !dim_nn_list || !linit || !dlt || *gnump <= 0 || !gcoo || !gwin || !gvol || !gprop || !gmat_type ||
      !gstate || !gstress || !gstrain || !gdinc || !gdinc_tot || !gn || !gstart || !gstack || !gstack_shp ||
      !gstack_dshp || !fint || !fext || !gmax_wvel || !gstrain_eq || !gint_work)
    return MEGA_ERR_ARG;
  FintIO io{};
  io.n = *gnump; io.gcoo = gcoo; io.gwin = gwin; io.gvol = gvol; io.gprop = gprop; io.bodyforce = model_bodyforce;
  io.gmat_type = gmat_type; io.gebc_nodes = gebc_nodes; io.gn = gn; io.gstart = gstart; io.gstack = gstack;
  io.nnz = *dim_nn_list; io.gstate = gstate; io.gstress = gstress; io.gstrain = gstrain; io.gdinc = gdinc;
  io.gdinc_tot = gdinc_tot; io.gstack_shp = gstack_shp; io.gstack_dshp = gstack_dshp; io.linit = *linit;
  io.dlt = *dlt; io.fint = fint; io.fext = fext; io.gmax_wvel = gmax_wvel; io.gstrain_eq = gstrain_eq;
  io.gint_work = gint_work; io.gcoo_current = gcoo_cuurent; io.gsm_len = gsm_len; io.gstack_ddshp = gstack_ddshp;
  io.dx_stress = local_dx_stress; io.dy_stress = local_dy_stress; io.dz_stress = local_dz_stress;
  return construct_fint_impl(&p, io);
}

}  // extern "C"
