// mega_internal.cuh -- host-side plumbing shared by the library's .cu files:
// device allocation tracking, error capture, the resident context and the
// launchers each translation unit exports.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <chrono>
#include <vector>
#include <cuda_runtime.h>
#include "mega_device.cuh"

namespace mega {

constexpr int kMaxBinCount = 1000;     // MAX_NEIGH, HANDELER.F90:245
constexpr int kMaxCandidates = 10000;  // INODE(10000), BIN_SEARCH.F90:80

void record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
// the CONTROL values construct_fint_gpu / construct_fint_pd_gpu read (set
// once by mega_fint_control); MEGA_ERR_STATE before that call
int fint_control_get(mega_params* out);
const char* last_error_text();
void record_error_text(const char* msg);

#define MEGA_TRY(x)                                                   \
  do {                                                                \
    cudaError_t e_ = (x);                                             \
    if (e_ != cudaSuccess) {                                          \
      ::mega::record_cuda_error(e_, #x, __FILE__, __LINE__);          \
      return MEGA_ERR_CUDA;                                           \
    }                                                                 \
  } while (0)

#define MEGA_CHECK_LAUNCH() MEGA_TRY(cudaGetLastError())

// Keep freed stream-ordered memory in the device's default pool for reuse
// instead of returning it to the driver (once per device and process).
void retain_pool_memory();
// With MEGA_TRACE set: report allocations slower than 5 ms to stderr.
bool trace_on();
void trace_alloc(size_t bytes, double ms, bool ordered);

// Stream-ordered device blocks kept for reuse by the process: a freed block
// waits in a cache (with an event marking the end of its last use) and a
// later request of about its size, on any stream, takes it after waiting on
// that event.  Set-up passes that run again with the same sizes (a new
// context on the same model, a re-search) then reach no driver allocation,
// whose cost grows with the pool's fragmentation.  *got = the block's size.
int cached_alloc(void** p, size_t bytes, cudaStream_t s, size_t* got);
void cached_free(void* p, size_t block_bytes, cudaStream_t s);

// Device allocations owned by one object; freed together.  A pool bound to a
// stream allocates and frees in that stream's order (through the block cache
// over cudaMallocAsync / cudaFreeAsync): every user of its memory must run on
// that stream.  An unbound pool uses cudaMalloc / cudaFree.
struct DevPool {
  std::vector<void*> ptrs;
  std::vector<size_t> blocks;  // block size of each pointer (bound pools)
  int64_t bytes = 0;
  cudaStream_t stream = nullptr;
  bool ordered = false;
  DevPool() = default;
  explicit DevPool(cudaStream_t s) { bind(s); }
  DevPool(const DevPool&) = delete;
  DevPool& operator=(const DevPool&) = delete;
  void bind(cudaStream_t s) {
    stream = s;
    ordered = true;
    retain_pool_memory();
  }
  template <typename T>
  int alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    const bool tr = trace_on();
    const auto t0 = tr ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point();
    size_t blk = count * sizeof(T);
    cudaError_t e = cudaSuccess;
    if (ordered) {
      if (cached_alloc((void**)p, count * sizeof(T), stream, &blk)) e = cudaErrorMemoryAllocation;
    } else {
      e = cudaMalloc((void**)p, count * sizeof(T));
    }
    if (tr) {
      if (ordered) cudaStreamSynchronize(stream);
      trace_alloc(count * sizeof(T),
                  std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(), ordered);
    }
    if (e != cudaSuccess) {
      record_cuda_error(e, ordered ? "cudaMallocAsync" : "cudaMalloc", __FILE__, __LINE__);
      *p = nullptr;
      return MEGA_ERR_NOMEM;
    }
    ptrs.push_back((void*)*p);
    blocks.push_back(blk);
    bytes += (int64_t)(count * sizeof(T));
    return 0;
  }
  void drop(void* p, size_t blk) {
    if (ordered) cached_free(p, blk, stream);
    else cudaFree(p);
  }
  void release(void* p) {
    for (size_t k = 0; k < ptrs.size(); ++k)
      if (ptrs[k] == p) {
        drop(p, blocks[k]);
        ptrs.erase(ptrs.begin() + k);
        blocks.erase(blocks.begin() + k);
        return;
      }
  }
  // move every allocation of o into this pool (same binding required)
  void adopt(DevPool& o) {
    for (size_t k = 0; k < o.ptrs.size(); ++k) {
      ptrs.push_back(o.ptrs[k]);
      blocks.push_back(o.blocks[k]);
    }
    bytes += o.bytes;
    o.ptrs.clear();
    o.blocks.clear();
    o.bytes = 0;
  }
  void free_all() {
    for (size_t k = 0; k < ptrs.size(); ++k) drop(ptrs[k], blocks[k]);
    ptrs.clear();
    blocks.clear();
    bytes = 0;
  }
  ~DevPool() { free_all(); }
};

#define MEGA_ALLOC(pool, ptr, count)                  \
  do {                                                \
    int r_ = (pool).alloc(&(ptr), (size_t)(count));   \
    if (r_) return r_;                                \
  } while (0)

// Compressed neighbour structure on the device.  CSR rows are the
// reference's GSTACK rows (0-based); the CSC view lists, for every node J,
// the rows i whose list contains J (ascending i) and the CSR position of
// that entry, which is how values stored per CSR entry are transposed.
struct DevCSR {
  int32_t n = 0;
  int64_t nnz = 0;
  int32_t gmaxn = 0;
  int32_t gmaxc = 0;          // longest column (set with the transposed view)
  int64_t* rowptr = nullptr;  // n + 1
  int32_t* col = nullptr;     // nnz
  int64_t* colptr = nullptr;  // n + 1
  int32_t* trow = nullptr;    // nnz
  int64_t* tpos = nullptr;    // nnz
};

// Bin geometry of HANDELER.F90:187-243 (doubles: xmin,ymin,zmin,xbin,ybin,zbin)
struct BinGeom {
  double g[6];
  int32_t nx, ny, nz;
};

// ---------------- launchers (search.cu)
// Exclusive scan of m int32 counts into int64 offsets (off[m] = total).
int scan_counts(cudaStream_t s, const int32_t* cnt, int64_t* off, int64_t m, DevPool& scratch);
// Bin search into csr (rowptr/col, gmaxn) with the reference's ordering.
// ijk (3,n) 1-based may be null.  status is a device word (OR-ed).
int bin_search(cudaStream_t s, int32_t n, const double* coo, const double* win, const double* sm_len,
               const double dist_max[3], int32_t itype_int, int32_t shsup, unsigned* status,
               DevCSR& csr, int32_t* ijk, DevPool& pool, BinGeom* geom_out, int32_t* cell_order = nullptr,
               const BinGeom* fixed = nullptr);  // fixed: reuse these bins instead of laying them out
// Build the CSC view of csr.
int build_transpose(cudaStream_t s, DevCSR& csr, DevPool& pool);

// ---------------- launchers (rk.cu)
int rk_shapes(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
              const int32_t* ebc_nodes, const DevCSR& csr, double* shp, double* gx, double* gy, double* gz,
              unsigned* status);

// the same shapes with the gradients written straight as mixed-precision
// records (float gradient + lidx[p]) into pk; shp as doubles
int rk_shapes_packed(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
                     const int32_t* ebc_nodes, const DevCSR& csr, const uint16_t* lidx, double* shp, float4* pk,
                     unsigned* status);

int rk_grad_at_face(cudaStream_t s, const mega_params& p, int32_t n, const double* coo, const double* win,
                    const int32_t* ebc_nodes, const DevCSR& csr, const double* sml, int face, double* gx, double* gy,
                    double* gz, unsigned* status);

// Per-material constants, deduplicated from PROPS(30,N) at init.
struct MatEntry {
  int32_t type;
  int32_t pad;
  double nu, E, rho, sig0, B, C, p7, p8, lam, mu, l2m, damp;
  double ki, kc, dmax;      // PROPS(9..11): damage thresholds K_I, K_C and DAM_MAX
  double qphi, kphi, qpsi;  // PROPS(25..27): Drucker-Prager Q_PHI, K_PHI, Q_PSI
};
inline MatEntry mat_entry(int32_t type, const double* pr) {
  MatEntry e{};
  e.type = type;
  e.nu = pr[0]; e.E = pr[1]; e.rho = pr[2]; e.sig0 = pr[3]; e.B = pr[4]; e.C = pr[5];
  e.p7 = pr[6]; e.p8 = pr[7]; e.damp = pr[20]; e.lam = pr[27]; e.mu = pr[28]; e.l2m = pr[29];
  e.ki = pr[8]; e.kc = pr[9]; e.dmax = pr[10]; e.qphi = pr[24]; e.kphi = pr[25]; e.qpsi = pr[26];
  return e;
}
// the models that carry STATE(1, 2, 4, 5) besides the plastic strain
__host__ __device__ inline bool damaged_type(int32_t t) { return t == MEGA_MAT_DRUCKER_PRAGER || t == MEGA_MAT_VM_DAMAGE; }

// Reductions the step kernels accumulate on the device.  Each quantity has
// kSlots partial sums (a block adds into slot blockIdx % kSlots) so that
// thousands of blocks do not serialise on one address; readers sum the slots.
constexpr int kSlots = 64;
struct StepAccum {
  double int_work[kSlots];        // GINT_WORK, accumulated over calls (FINT.F90:1232)
  double ke[kSlots];              // kinetic energy of the last step
  double ee[kSlots];              // accumulated external energy (MAIN.F90:539)
  double tf[6][kSlots];           // TOTAL_FORCE(3,2), running sum (MAIN.F90:485)
  unsigned long long newton_iters[kSlots];  // last step
  unsigned long long plastic[kSlots];       // last step
  unsigned long long newton_total[kSlots];  // over all steps (never reset by a step)
  unsigned long long plastic_total[kSlots];
};
inline double slot_sum(const double* v) {
  double s = 0.0;
  for (int k = 0; k < kSlots; ++k) s += v[k];
  return s;
}
inline unsigned long long slot_sum(const unsigned long long* v) {
  unsigned long long s = 0;
  for (int k = 0; k < kSlots; ++k) s += v[k];
  return s;
}

// ---------------- launchers (force.cu)
struct StressArgs {
  int32_t n;
  const double* fg;          // 18 per node: F (row-major 3x3), G0 (3x3)
  const uint16_t* matidx;
  const MatEntry* mats;
  const double* vol;
  double* stress;            // (6,n)
  double* strain;            // (6,n)
  double* eps;               // (n)
  double* strain_eq;         // (n)
  double* wvel;              // (n)
  void* tmat;                // 12 per node (double or float)
  const double* bodyforce;   // (3,n) or null
  double grav[3];
  int has_body;
  int inv3_exact;
  int finite_strain;
  int maxit;
  int rate_solver;           // material 7: 0 bounded Newton in ln(dgamma), 1 textbook
  double rtol;
  double dt;
  int32_t* iters;            // per-node Newton passes (or null)
  double* aux;               // 4 per node: STATE(1, 2, 4, 5) of the damaged models (or null)
  const uint16_t* mlp_w2;    // surrogate network: W2 (64x64) as bf16 bits, or null
  const float* mlp_small;    // W1 (64x4), b1, b2, W3, b3 as fp32, or null
  const double* ndt;         // per-node step of independent instances, or null (dt for all)
  int32_t* queue;            // learned start: plastic rate-dependent nodes of this step (n), or null
  unsigned* qcount;          // their count (zeroed before the step's stress kernels)
  float* log_buf;            // sample log: 5 floats (4 features, target) per sample, or null
  unsigned long long* log_count;
  int64_t log_cap;
  uint32_t log_stride;
  uint32_t log_seed;
  StepAccum* acc;
  unsigned* status;
};
int launch_defgrad(cudaStream_t s, bool mixed, bool interp, int32_t n, const DevCSR& csr, const void* gx,
                   const void* gy, const void* gz, const double* dsp, const double* dsp_tot,
                   const double* sdphi, const double* shp, double* dsp_tot_phy, double* fg,
                   StepAccum* acc);
int launch_stress(cudaStream_t s, bool mixed, const StressArgs& a);

// ---------------- NSNI (nsni.cu)
// smoothed second derivatives per list entry, one array per component:
// XX, YY, ZZ, XY, YZ, XZ (double for the set-up and FP64 steps, float for
// the mixed steps)
template <typename V>
struct NsniArr {
  V* v[6];
};
using NsniS = NsniArr<double>;
using NsniSF = NsniArr<float>;
struct NsniStepArgs {
  int32_t n;
  const double* fg;          // F, G0 of this step
  const double* stress_old;  // the stress before this step's update
  const double* stress_new;
  const double* sml;         // SM_LEN (6, n)
  const double* vol;
  const uint16_t* matidx;
  const MatEntry* mats;
  double* hq;                // 18 per node: sum_J S_q du_J,k
  double* sgrad;             // 18 per node: sigma_,x, sigma_,y, sigma_,z (Voigt)
  void* w;                   // 18 per node: force weights on the six S components (double, or float when mixed)
  double* fstab;             // 3 per node: the stabilisation force
  int finite_strain;
  int inv3_exact;
  StepAccum* acc;
  unsigned* status;
};
int nsni_combine(cudaStream_t s, int32_t n, int axis, const int64_t* rowptr, const double* sml, const double* gp[3],
                 const double* gm[3], const NsniS& out);
// stage 0: the row gather of H (after the displacement increment is known);
// stage 1: stress gradients and weights (mixed: float weights);
// stage 2: the column gather of the stabilisation force.
// Stages 0 and 2 are the FP64 steps' own kernels: the mixed steps form H and
// the stabilisation force in the tiled gathers (NsniTiles).
int nsni_step(cudaStream_t s, const NsniStepArgs& a, const DevCSR& csr, const NsniS& rows, const NsniS& cols,
              bool mixed, const double* du, int stage);
// dst[6 e + q] = float S_q at list position pos[e] (e when pos is null)
int nsni_records(cudaStream_t s, int64_t m, const int64_t* pos, const NsniS& src, float* dst);
// dst[6 i + q] = sum over row i of the float-rounded S_q, in double
int nsni_rowsum(cudaStream_t s, int32_t n, const int64_t* rowptr, const NsniS& src, double* dst);

// surrogate network of the rate-dependent return mapping (mlp.cu)
int mlp_nparams();
int mlp_pack(cudaStream_t s, const float* dtheta, uint16_t* w2, float* small);
int mlp_train_dev(cudaStream_t s, float* dth, int64_t ns, const float* X, int xs, const float* T, int ts,
                  int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss_host);
struct ForceArgs {
  int32_t n;
  const DevCSR* csr;
  const void* tgx;
  const void* tgy;
  const void* tgz;
  const double* tshp;   // transposed shape values (body force) or null
  const void* tmat;
  int has_body;
  int integrate;        // 0: only fint / fext (CONSTRUCT_FINT drop-in)
  int predict;          // fuse the next step's predictor
  const int8_t* ebc;
  const double* vel2;   // prescribed velocities of fixity code 2 for this step (3), or null
  const double* mass;
  const uint16_t* matidx;
  const MatEntry* mats;
  const int8_t* body_id;
  double* fint;
  double* fext;
  double* vel;
  double* acl;
  double* dsp;
  double* dsp_tot;
  double* prforce;
  double dt;
  StepAccum* acc;
  unsigned* status;
};
int launch_force(cudaStream_t s, bool mixed, const ForceArgs& a);
int launch_predict(cudaStream_t s, int64_t n3, double* dsp, double* dsp_tot, double* vel, const double* acl,
                   double dt, const double* ndt = nullptr);
// out[3i+k] = base[3i+k] + sum_J shp_iJ * val[3J+k]
int launch_interp(cudaStream_t s, int32_t n, const DevCSR& csr, const double* shp, const double* val,
                  const double* base, double* out);
int device_sm_count();

}  // namespace mega
