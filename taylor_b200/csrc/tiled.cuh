// tiled.cuh -- tiles of consecutive rows (or columns) with their neighbour
// sets, for the shared-memory staged gathers of tiled.cu.
#pragma once
#include "mega_internal.cuh"

namespace mega {

struct TileSet {
  int32_t R = 0;           // rows (columns) per tile; the kernels run R*4 threads per tile
  int64_t ntiles = 0;
  int32_t jmax = 0;        // stride of jset per tile
  int32_t maxcnt = 0;      // largest neighbour set of any tile
  int32_t recmax = 0;      // most list entries of any tile (its packed-record range)
  int32_t* jset = nullptr; // [ntiles][jmax] sorted node ids
  int32_t* jcnt = nullptr; // [ntiles]
  uint16_t* lidx = nullptr;  // per entry: rank of its neighbour in the tile's set
};

// NSNI terms carried by the mixed-precision tiled gathers: the smoothed
// second derivatives S_q (XX, YY, ZZ, XY, YZ, XZ) of every list entry as six
// floats in the order of the float row records (srow) and of the float
// column records (scol), their row sums, and the per-node H output (row
// gather) and force weights (column gather)
struct NsniTiles {
  const float* srow = nullptr;   // 6 per row record
  const double* ssum = nullptr;  // 6 per node: sum_J S_q(i, J) in double
  double* hq = nullptr;          // 18 per node out: sum_J S_q(i, J) du_J,k at [18 i + 6 k + q]
};

struct TiledForceArgs {
  int32_t n;
  int32_t R;
  int64_t ntiles;
  int32_t jmax;
  int32_t maxcnt;
  int32_t recmax;
  const int32_t* jset;
  const int32_t* jcnt;
  const int64_t* colptr;
  const void* pk;         // packed transposed entries (gradient + local index)
  const double* tshp;     // transposed shape values (body force) or null
  const void* tmat;       // 12 values per node
  int has_body;
  int predict;
  const int8_t* ebc;
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
  const double* fadd;     // 3 per node added to the internal force (NSNI), or null
  const float* ns_scol;   // NSNI (mixed): 6 S values per column record, or null
  const float* ns_w;      // NSNI (mixed): force weights, 20 floats per node (18 used)
  const double* vel2;     // prescribed velocities of fixity code 2 for this step (3), or null
  const double* ndt;      // per-node step of independent instances, or null (dt for all)
  double dt;
  StepAccum* acc;
  unsigned* status;
};

// Tiles of R consecutive rows of (ptr, idx), R halved from 64 down to 8
// until every tile's neighbour set fits jmax = 1024.
int build_tiles(cudaStream_t s, int32_t n, const int64_t* ptr, const int32_t* idx, int64_t nnz, int32_t gmaxn,
                TileSet& ts, DevPool& pool, int32_t* maxcnt_out);
// out[e] = (g[pos[e]], lidx[e]) as float4 (f64 = false) or 2 x double2
int pack_entries(cudaStream_t s, int64_t m, const uint16_t* lidx, const double* gx, const double* gy,
                 const double* gz, const int64_t* pos, bool f64, void* out);
// out[e] = (in[pos[e]] gradient, lidx[e]): mixed records of the transposed
// view from those of the rows
int pack_transposed32(cudaStream_t s, int64_t m, const uint16_t* lidx, const float4* in, const int64_t* pos,
                      float4* out);
// Reorder the entries within each row (column) of the tiles ts so that the
// lanes of a warp of a gather with `lanes` (4 or 8) lanes per row read
// distinct shared-memory banks of the staged neighbour data (one 32-bit
// word per rank and value) where possible.  lidx is reordered in place;
// pos[e] receives pos_src (or, when null, the identity) at the entry's
// position before, and must hold that same array on entry.
int bank_order(cudaStream_t s, int32_t n, const TileSet& ts, const int64_t* ptr, uint16_t* lidx,
               const int64_t* pos_src, int64_t* pos, int lanes);
// out[e] = e;  out[e] = in[pos[e]]
int iota64(cudaStream_t s, int64_t m, int64_t* out);
int gather_records32(cudaStream_t s, int64_t m, const int64_t* pos, const float4* in, float4* out);
// out[e] = the tile rank of float record e;  out[6 e + k] = in[6 pos[e] + k]
int record_ranks(cudaStream_t s, int64_t m, const float4* rec, uint16_t* out);
int gather_f6(cudaStream_t s, int64_t m, const int64_t* pos, const float* in, float* out);
int configure_tiled_kernels();
// launch variants of the two gathers: lanes per row x records in flight
// (register streams, variants 0-3 and 6, 7), and lanes per row with the
// tile's records streamed into shared memory by the copy engine (variants
// 4, 5)
constexpr int kTiledVariants = 8;
int tiled_variants();
// whether a variant's shared memory fits the row (defgrad) or column (force) tiles
bool tiled_variant_fits(const TileSet& ts, bool mixed, int variant, bool force, bool has_body);
// MEGA_ERR_UNSUPPORTED when the variant's shared memory does not fit the tiles
// ns (mixed only, register variants 0-3): the NSNI H gather rides along
int launch_defgrad_tiled(cudaStream_t s, bool mixed, bool interp, int32_t n, const TileSet& ts,
                         const NsniTiles* ns, const int64_t* rowptr, const void* pk, const double* dsp,
                         const double* dsp_tot,
                         const double* sdphi, const double* shp, double* dsp_tot_phy, double* fg, StepAccum* acc,
                         unsigned* status, int variant = 0);
int launch_force_tiled(cudaStream_t s, bool mixed, const TiledForceArgs& a, int variant = 0);

}  // namespace mega
