/*
 * mega_gpu.h -- C ABI of the B200 explicit meshfree step (libmega_gpu.so).
 *
 * The library replaces the hot path of MEGA (Meshfree Explicit Galerkin
 * Analysis, XieZhengTing/Taylor): the bin neighbour search, the RK shape
 * function build, the nodal-integration internal force with Hughes-Winget
 * rotation and von Mises return mapping, the displacement interpolation,
 * the central-difference update and the peridynamic force.
 *
 * Conventions (they mirror gfortran's defaults, so an ISO_C_BINDING
 * interface block binds every entry point without wrappers):
 *   - arrays are host pointers to Fortran column-major storage: (3,N) is
 *     xyz-interleaved per node, (6,N) is Voigt (xx,yy,zz,yz,xz,xy) per node,
 *     (30,N) material properties, (20,N) state variables;
 *   - LOGICAL is int32_t (0 / 1); INTEGER is int32_t; DOUBLE PRECISION is double;
 *   - neighbour lists (GN, GSTART, GSTACK) are 1-based like the reference;
 *   - every entry returns int: 0 = success, >0 = bitmask of MEGA_ST_* raised
 *     by the device, <0 = MEGA_ERR_* (CUDA or argument error).  Kernels never
 *     trap; the caller maps a nonzero status onto EXIT_PROGRAM.
 * One context owns one CUDA stream and all device buffers; calls on one
 * context are not re-entrant.  The host arrays are never freed or resized.
 */
#ifndef MEGA_GPU_H
#define MEGA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status bits (device status word, OR-ed by kernels) ----------------- */
#define MEGA_ST_NEWTON_CAP      0x0001 /* return mapping hit its iteration cap
                                          (CONSTITUTE_VONMISES.F90:115-119) */
#define MEGA_ST_SINGULAR_MOMENT 0x0002 /* RK moment matrix determinant is 0 or
                                          not finite (INVERSE.F90:185-223) */
#define MEGA_ST_BIN_OVERFLOW    0x0004 /* >= 1000 nodes in one bin
                                          (BIN_SEARCH.F90:48-51) */
#define MEGA_ST_CAND_OVERFLOW   0x0008 /* > 10000 candidates for one node
                                          (BIN_SEARCH.F90:117-120) */
#define MEGA_ST_NONFINITE       0x0010 /* NaN/Inf in a force or stress */
#define MEGA_ST_BAD_MATERIAL    0x0020 /* material type not on this path
                                          (CONSTITUTION.F90:79-83) */
#define MEGA_ST_STACK_OVERFLOW  0x0040 /* neighbour stack larger than the
                                          caller's DIM_NN_LIST */
#define MEGA_ST_SINGULAR_SHAPE  0x0080 /* PD shape tensor K not invertible
                                          (INVERSE.F90:41-45) */
#define MEGA_ST_BAD_MESH        0x0100 /* element connectivity names a node
                                          outside 1..N */
#define MEGA_ST_WAIT_TIMEOUT    0x0200 /* a kernel gave up waiting for its own
                                          asynchronous copies (bounded wait);
                                          its outputs of that step are void */

/* ---- API errors (negative return codes) --------------------------------- */
#define MEGA_ERR_CUDA     (-1)
#define MEGA_ERR_ARG      (-2)
#define MEGA_ERR_HANDLE   (-3)
#define MEGA_ERR_STATE    (-4)  /* call out of order (e.g. step before search) */
#define MEGA_ERR_NOMEM    (-5)
#define MEGA_ERR_UNSUPPORTED (-6)

/* ---- precision / physics modes for the resident stepper ----------------- */
#define MEGA_MODE_FP64    0  /* plain FP64 drop-in */
#define MEGA_MODE_MIXED   1  /* FP32 gradients, stress, strain and force
                                accumulation; FP64 moment inverse, positions,
                                displacements, time integration and return-
                                mapping residual */
#define MEGA_FLAG_INTERP_EACH_STEP 0x100 /* accumulate the physical displacement
                                            every step as HANDELER.F90:114-139
                                            and MAIN.F90:377-386 do, instead of
                                            evaluating it when downloaded */
#define MEGA_FLAG_LEARNED_GUESS    0x200 /* rate-dependent return mapping starts
                                            Newton from the surrogate network */

/* ---- material types handled by the fused force kernel ------------------- */
#define MEGA_MAT_ELASTIC      1  /* CONSTITUTION.F90:48-52 */
#define MEGA_MAT_VONMISES     2  /* CONSTITUTE_VONMISES.F90:21-158 */
#define MEGA_MAT_DRUCKER_PRAGER 3 /* CONSTITUTE_DRUCKPRAG.F90:17-241 (shear yield, damage) */
#define MEGA_MAT_VM_DAMAGE    6  /* CONSTITUTE_VONMISES_DAM.F90:21-196 (J2 + damage) */
#define MEGA_MAT_VM_RATE      7  /* power-law rate-dependent J2 (no reference
                                    counterpart): sigma_y = A + B*ep^n *
                                    (1 + C*ln(max(epdot,epdot0)/epdot0));
                                    PROPS(4..8) = A, B, n, C, epdot0 */

/* ---- fields for mega_download / mega_upload ----------------------------- */
enum mega_field {
  MEGA_F_COO_CURRENT = 0, /* (3,N) x = X + physical total displacement       */
  MEGA_F_DSP         = 1, /* (3N) generalised displacement increment (LOCAL_DSP) */
  MEGA_F_DSP_TOT     = 2, /* (3N) generalised total displacement             */
  MEGA_F_VEL         = 3, /* (3N) generalised velocity                       */
  MEGA_F_ACL         = 4, /* (3N) generalised acceleration                   */
  MEGA_F_FINT        = 5, /* (3N) internal force                             */
  MEGA_F_FEXT        = 6, /* (3N) external force                             */
  MEGA_F_STRESS      = 7, /* (6,N) Cauchy stress                             */
  MEGA_F_STRAIN      = 8, /* (6,N) strain                                    */
  MEGA_F_EPS         = 9, /* (N) equivalent plastic strain, STATE(3,:)       */
  MEGA_F_STRAIN_EQ   = 10,/* (N) GSTRAIN_EQ                                  */
  MEGA_F_WAVE_VEL    = 11,/* (N) GMAX_WVEL                                   */
  MEGA_F_DSP_TOT_PHY = 12,/* (3N) physical total displacement                */
  MEGA_F_PRFORCE     = 13,/* (3,N) reaction force on fixed DOFs              */
  MEGA_F_NEWTON_IT   = 14,/* (N) Newton iterations of the last step (int32 stored as double) */
  MEGA_F_STATE_AUX   = 15,/* (4,N) STATE(1,2,4,5) = EPS_SHEAR, EPS_VOL, DAM, DAM_SV of the damaged
                             models (materials 3, 6); MEGA_ERR_STATE when no node has one */
  MEGA_F_NSNI_SGRAD  = 16 /* (18,N) NSNI stress gradients d sigma/dx, d sigma/dy, d sigma/dz
                             (Voigt each; the reference's LOCAL_DX/DY/DZ_STRESS), ITYPE_INT = 2 */
};

/* Scalars reported by mega_scalars (energies are those MAIN.F90:524-555 writes). */
typedef struct mega_scalars_t {
  double time;            /* simulated time after the last step               */
  double int_energy;      /* internal work (LOCAL_INT_WORK, finite strain)    */
  double kin_energy;      /* 0.5 m v^2                                        */
  double ext_energy;      /* accumulated 0.5 (fext + fext_prev) dsp           */
  double total_force[6];  /* reaction sums for bodies 1 and 2 (TOTAL_FORCE)   */
  int64_t steps;          /* explicit steps taken                             */
  int64_t newton_iters;   /* total return-mapping Newton iterations, last step*/
  int64_t plastic_nodes;  /* nodes that returned plastically, last step       */
  int64_t newton_iters_total;  /* Newton iterations over all resident steps    */
  int64_t plastic_nodes_total; /* plastic node updates over all resident steps */
} mega_scalars_t;

/* Hot-path switches of the reference's CONTROL module (CONTROL.F90:27-95)
 * plus the values PRE_CONTROL derives from the model.  Passed once. */
typedef struct mega_params {
  int32_t rk_degree;       /* RK_DEGREE; only 1 (linear basis) is live        */
  int32_t rk_cont;         /* RK_CONT; 3 = cubic B-spline (KERNEL.F90:57-71)   */
  int32_t rk_impl;         /* RK_IMPL; read, no effect on the live path        */
  int32_t itype_int;       /* ITYPE_INT; 0 = direct nodal integration, 2 = NSNI (resident contexts) */
  int32_t ql;              /* QL (logical): quasi-linear moment regularisation */
  int32_t lagrangian;      /* LLAGRANGIAN (logical); 0 = semi-Lagrangian (resident, DNI, FP64) */
  int32_t finite_strain;   /* LFINITE_STRAIN (logical)                         */
  int32_t shsup;           /* SHSUP (logical): 1 = ellipsoidal support         */
  int32_t peridynamics;    /* PERIDYNAMICS (logical)                          */
  int32_t inv3_exact;      /* 0 = reproduce INV3 as written (det^2 * A^-1,
                              INVERSE.F90:119-152); 1 = true 3x3 inverse      */
  int32_t newton_max_iter; /* return-mapping iteration cap; 20 in the reference */
  int32_t rate_solver;      /* material 7 return mapping: 0 Newton in ln(dgamma) from
                                the upper bound (default), 1 textbook: Newton in dgamma
                                from the perfectly plastic estimate */
  double  ql_coef;         /* QL_COEF                                         */
  double  ql_len;          /* QL_LEN                                          */
  double  gravity[3];      /* IGRAVITY                                        */
  double  dist_max[3];     /* GXDIST_MAX, GYDIST_MAX, GZDIST_MAX              */
  double  newton_rtol;     /* rate-dependent law: relative residual tolerance */
  int32_t auto_ts;         /* AUTO_TS (logical): construct_fint_pd_gpu returns the
                              step of its CFL rule in DLT_FINT (FINT_PD.F90:690-754) */
  int32_t reserved;
  double  dlt_fac;         /* DLT_FAC, the factor of that step                 */
} mega_params;

/* Fill p with the reference's defaults for the Taylor-bar deck
 * (Control.dat: RK 1/3/0, QL on 0.001, DNI, Lagrangian, finite strain). */
void mega_params_default(mega_params* p);

/* ======================================================================== */
/* Stateless drop-ins (copy in, compute on the GPU, copy out, synchronous)  */
/* ======================================================================== */

/* GET_BINS + SOFT_SEARCH (BIN_SEARCH.F90:2-64, 153-328) with the bin
 * geometry HANDELER computes at LINIT (HANDELER.F90:187-250).
 *   coo (3,n), win (3,n), sm_len (6,n), dist_max[3];
 *   out: gn(n), gstart(n), gstack(dim_nn_list) (1-based), *gmaxn, ijk (3,n)
 *   (GIJKSPC), *nnz.  The neighbour order is BIN_INODE's: cells IX-outer /
 *   IZ-inner, node index order inside a cell. */
int mega_bin_search(int32_t n, const double* coo, const double* win,
                    const double* sm_len, const double* dist_max,
                    int32_t itype_int, int32_t shsup,
                    int32_t* gn, int32_t* gstart, int32_t* gstack,
                    int64_t dim_nn_list, int32_t* gmaxn, int32_t* ijk,
                    int64_t* nnz);

/* No counterpart in the reference: the same search as mega_bin_search for
 * callers that cannot allocate GPU memory when they search (their device
 * memory belongs to another allocator or arena, or allocation is not allowed
 * in their loop).  It allocates nothing: inputs and outputs are device
 * pointers the caller owns -- d_coo (3,n), d_win (3,n), d_sm_len (6,n);
 * out d_gn (n), d_gstart (n), d_gstack (dim_nn_list) 1-based, d_ijk (3,n)
 * or NULL -- and every temporary lives in one fixed 48 MiB __device__ array
 * compiled into the library, held by every GPU that loads it until exit.
 * Problems that do not fit (about 16 bytes per bin plus 20 per node, e.g.
 * 1.04 M nodes in 0.32 M bins fit), or whose lists hold more than
 * INT32_MAX entries (GSTART is 32-bit), are rejected with
 * MEGA_ERR_UNSUPPORTED and a message.  dist_max, *gmaxn and *nnz are host memory; stream is a
 * cudaStream_t (NULL = default stream); the call returns after the work on
 * that stream finished.  The first call on a device looks the array up
 * (cudaGetSymbolAddress), so make it before any stream capture.  Calls share
 * the array: calls that overlap on the GPU race, serialise them.  When nnz
 * exceeds dim_nn_list, GN/GSTART are written, GSTACK is not, and
 * MEGA_ST_STACK_OVERFLOW is returned. */
int mega_bin_search_noalloc(int32_t n, const double* d_coo, const double* d_win,
                            const double* d_sm_len, const double* dist_max,
                            int32_t itype_int, int32_t shsup, int32_t* d_gn,
                            int32_t* d_gstart, int32_t* d_gstack, int64_t dim_nn_list,
                            int32_t* d_ijk, int32_t* gmaxn, int64_t* nnz, void* stream);

/* RK1 for every node (RK.f90:16-453 via FINT.F90:404-408): shape functions
 * and gradients at X_i for the neighbours in (gn, gstart, gstack).
 *   ebc_nodes (n) logical; out: shp (nnz), dshp (3,nnz). */
int mega_rk_shapes(const mega_params* p, int32_t n, const double* coo,
                   const double* win, const int32_t* ebc_nodes,
                   const int32_t* gn, const int32_t* gstart,
                   const int32_t* gstack, int64_t nnz,
                   double* shp, double* dshp);

/* HUGHES_WINGET (HUGHES_WINGET.F90:16-81) for n independent nodes.
 *   lmat (3,3,n) column-major; out: rot (3,3,n), strain (6,n), d (6,n). */
int mega_hughes_winget(const mega_params* p, int32_t n, const double* lmat,
                       double* rot, double* strain, double* d);

/* ROTATE_TENSOR (ROTATE_TENSOR.F90:21-87) for n nodes: v <- R v R^T. */
int mega_rotate_tensor(int32_t n, const double* rot, double* vtensor);

/* CONSTITUTION (CONSTITUTION.F90:18-89) for n nodes:
 *   stress_pred (6,n), mat_type (n), props (30,n), dlt; state (20,n) in/out;
 *   out: stress (6,n), iters (n) Newton iterations used (may be NULL). */
int mega_constitution(const mega_params* p, int32_t n,
                      const double* stress_pred, const int32_t* mat_type,
                      const double* props, double dlt, double* state,
                      double* stress, int32_t* iters);

/* CONSTRUCT_FINT (FINT.F90:16-25) with the reference's argument meaning in a
 * shorter list (the arrays the Lagrangian DNI path reads), scalars by value;
 * construct_fint_gpu below takes the full list.  When linit != 0 the shape functions are computed
 * (RK1) and written to gstack_shp / gstack_dshp; otherwise they are read.
 * In/out arrays follow FINT.F90: gstress, gstrain (6,n), gstate (20,n).
 * Outputs: fint, fext (3n), gmax_wvel (n), gstrain_eq (n), *gint_work
 * (accumulated, as GINT_WORK is). */
int mega_construct_fint(const mega_params* p, int32_t n,
                        const double* gcoo, const double* gwin,
                        const double* gvol, const double* gprop,
                        const int32_t* gmat_type, const int32_t* gebc_nodes,
                        const double* bodyforce,
                        double* gstate, double* gstress, double* gstrain,
                        const double* gdinc, const double* gdinc_tot,
                        const int32_t* gn, const int32_t* gstart,
                        const int32_t* gstack, int64_t nnz,
                        double* gstack_shp, double* gstack_dshp,
                        int32_t linit, double dlt,
                        double* fint, double* fext,
                        double* gmax_wvel, double* gstrain_eq,
                        double* gint_work);

/* ---- the two force subroutines with the reference's own argument lists --
 * construct_fint_gpu and construct_fint_pd_gpu take CONSTRUCT_FINT's
 * (FINT.F90:16-25) and CONSTRUCT_FINT_PD's (FINT_PD.F90:16-25) arguments in
 * their order, every one by reference as gfortran passes them (INTEGER
 * int32_t*, LOGICAL LINIT int32_t*, DOUBLE PRECISION double*, arrays
 * column-major), so HANDELER's calls (HANDELER.F90:285-306) bind them
 * unchanged through BIND(C).  The CONTROL module values the reference
 * reads as globals (RK_*, QL*, ITYPE_INT, LLAGRANGIAN, LFINITE_STRAIN,
 * SHSUP, IGRAVITY, AUTO_TS, DLT_FAC, ...) come from one earlier
 * mega_fint_control call.  Paths: Lagrangian DNI and NSNI (ITYPE_INT = 2:
 * GSM_LEN in, GSTACK_DDSHP written at LINIT and read after, LOCAL_DX/DY/
 * DZ_STRESS in/out) and semi-Lagrangian DNI (LLAGRANGIAN = .FALSE.: RK1 on
 * GCOO_CUURENT in every call, GSTACK_SHP/DSHP written).  Accepted and not
 * read, as on the reference's live path: GSM_AREA, GSM_VOL, GNSNI_FAC,
 * GGHOST, G_H_STRESS, G_S_STRESS, GMAXN, GINVK (CONSTRUCT_FINT),
 * MODEL_BODY_ID, G_X/Y/Z_MOM (the NSNI weights come from GSM_LEN);
 * CONSTRUCT_FINT leaves DLT_FINT and GCHAR_DIST untouched (their block is
 * commented out, FINT.F90:1250-1330), CONSTRUCT_FINT_PD sets them when
 * AUTO_TS. */
int mega_fint_control(const mega_params* p);
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
                       double* gstrain_eq, const double* dlt);
int construct_fint_pd_gpu(const double* gwin, const double* gvol, const int32_t* gnump, const double* gcoo,
                          const double* gcoo_cuurent, const double* gsm_len, const double* gsm_area,
                          const double* gsm_vol, const double* gnsni_fac, const int32_t* gghost, const double* gprop,
                          double* gstate, double* gstress, double* gstrain, double* g_h_stress, double* g_s_stress,
                          const double* gdinc, const double* gdinc_tot, const int32_t* gmat_type,
                          const int32_t* gebc_nodes, const int32_t* gn, const int32_t* gstart,
                          const int32_t* dim_nn_list, const int32_t* gstack, double* gstack_shp,
                          double* gstack_dshp, double* gstack_ddshp, const int32_t* gmaxn, double* ginvk,
                          const int32_t* linit, double* fint, double* dlt_fint, double* gchar_dist,
                          double* gmax_wvel, double* local_dx_stress, double* local_dy_stress,
                          double* local_dz_stress, const double* g_x_mom, const double* g_y_mom,
                          const double* g_z_mom, const double* model_bodyforce, double* gint_work,
                          const double* dlt);

/* CONSTRUCT_FINT_PD (FINT_PD.F90:16-759), correspondence peridynamics,
 * Lagrangian path.  At linit != 0 the influence functions and K^-1 are built
 * (UDFM_SHAPE_TENSOR, RK.f90:579-726) into gstack_shp and ginvk (3,3,n).
 * gcoo_current (3,n) are the current coordinates. */
/* Mesh pre-processing of PRE_MODEL.F90:248-268 and PRE_CONTROL.F90:803-871
 * for hexahedral meshes, on the device: conn = IDELM(8,NELEM), 1-based.
 * Out: win_raw (3,N) = ADIAL (GET_ADIAL, PRE_MODEL_ADIAL.F90:64-153), vol (N)
 * (GET_VOLUMES / GET_VOL2, PRE_MODEL_VOLUMES.F90:70-117), sm_len (6,N),
 * mom (3,N) = X/Y/Z_MOM and dist_max (3) (GET_SMOOTHING_LENGTHS,
 * PRE_MODEL_SMOOTHING_LENGTHS.F90:49-99), win (3,N) = ADIAL * norm_win
 * (PRE_CONTROL.F90:870-872; norm_win (N) may be NULL for 1) and the smallest
 * raw window (the automatic QL_LEN before QL_LEN_REDUCE_AUTO,
 * PRE_CONTROL.F90:803-815).  win, mom and min_raw_window may be NULL.
 * Windows and volumes are bit-exact with the reference's element-order
 * loops. */
int mega_pre_model_hex(int32_t n, const double* coo, int32_t nelem, const int32_t* conn, const double* norm_win,
                       double* win_raw, double* win, double* vol, double* sm_len, double* mom, double* dist_max,
                       double* min_raw_window);
/* As mega_pre_model_hex for meshes of hexahedral and tetrahedral blocks:
 * eltype (nelem) 2 = hexahedron, 1 = tetrahedron (the reference's block
 * type, PRE_MODEL.F90:233-240: a block whose last element repeats its
 * seventh node as its eighth; kfile.read_k applies that rule), NULL = all
 * hexahedra.  A tetrahedron counts its first four nodes: its window is
 * their largest per-axis extent (PRE_MODEL_ADIAL.F90:112-150) and each gets
 * 1/4 of its volume (GET_VOL1, PRE_MODEL_VOL1.f90:37-45,
 * PRE_MODEL_VOLUMES.F90:99-115). */
int mega_pre_model(int32_t n, const double* coo, int32_t nelem, const int32_t* conn, const int32_t* eltype,
                   const double* norm_win, double* win_raw, double* win, double* vol, double* sm_len, double* mom,
                   double* dist_max, double* min_raw_window);

int mega_construct_fint_pd(const mega_params* p, int32_t n,
                           const double* gcoo, const double* gcoo_current,
                           const double* gwin, const double* gvol,
                           const double* gprop, const int32_t* gmat_type,
                           double* gstate, double* gstress, double* gstrain,
                           const double* gdinc,
                           const int32_t* gn, const int32_t* gstart,
                           const int32_t* gstack, int64_t nnz,
                           double* gstack_shp, double* ginvk,
                           int32_t linit, double dlt,
                           double* fint, double* gmax_wvel, double* gint_work);

/* ======================================================================== */
/* Resident context: the whole MAIN.F90:304-658 loop on the device          */
/* ======================================================================== */

/* Upload the model and create a context.  Arrays as in MAIN.F90:146-221:
 *   coo (3,n), win (3,n) normalised windows, vol (n), mass (3n), ebc (3,n)
 *   fixity codes (0 free, 1 fixed, 2 prescribed velocity: see
 *   mega_set_fixity2), vinit (3,n), props (30,n), mat_type (n),
 *   body_id (n), bodyforce (3,n) (may be NULL), sm_len (6,n).
 * Velocity starts at vinit except on fixed DOFs (STATE_INIT.f90:97-105);
 * only code-1 nodes take the singular kernel (LOCAL_EBC_NODES). */
int mega_gpu_init(const mega_params* p, int32_t n, const double* coo,
                  const double* win, const double* vol, const double* mass,
                  const int32_t* ebc, const double* vinit, const double* props,
                  const int32_t* mat_type, const int32_t* body_id,
                  const double* bodyforce, const double* sm_len,
                  int64_t* handle);

/* Declare that the context's n nodes are ninst independent instances (for
 * example many bars stepped together), instance k owning the next
 * inst_nodes[k] nodes.  Call before mega_search_and_shapes: each instance is
 * then searched with its own bin grid (dist_max (3,ninst) its DIST_MAX, or
 * NULL for the params' value) and sees no other instance's nodes, so
 * instances may overlap in space; its lists equal those of a search of the
 * instance alone.  The other params (QL length among them) are shared.
 * Energies and reaction sums in mega_get_scalars are totals over all
 * instances. */
int mega_set_instances(int64_t h, int32_t ninst, const int32_t* inst_nodes, const double* dist_max);
/* Give each instance of a mega_set_instances context its own explicit step
 * (after mega_search_and_shapes): dt_inst (ninst) > 0.  The steps of
 * mega_step_resident then advance instance k by dt_inst[k] each (its own
 * stable step instead of the smallest instance's); the call's dt is still
 * what TIME advances by and what the fixity-2 windows see.  NULL goes back to
 * one dt for all.  MEGA_ERR_STATE for a context without instances. */
int mega_set_instance_dt(int64_t h, const double* dt_inst);
/* Autotuner: time each launch variant of the two per-step gathers for the
 * given precision on this context's lists, reps launches each, keep the
 * fastest, and leave the state as it was.  Variants 0..3, 6 and 7 hold the
 * packed records in registers (lanes per row x records in flight: (4, 4),
 * (4, 2), (4, 1), (8, 2), (16, 1), (16, 2)); 4 and 5 have the copy engine
 * stream each tile's records into shared memory (4 or 8 lanes per row),
 * where the tiles fit (not with NSNI in mixed precision).  choice
 * (2) receives the deformation-gradient and force variants, times_ms
 * (2 x MEGA_TUNE_VARIANTS, may be NULL) the mean launch times, -1 for a
 * variant that does not fit. */
#define MEGA_TUNE_VARIANTS 8
/* Pin the launch variants of the two gathers for one precision (after
 * mega_search_and_shapes), e.g. to repeat a run bit for bit: variants with
 * the same lanes per row (0, 1, 2, 4; 3, 5; 6, 7) sum in the same order and
 * give identical results.  MEGA_ERR_UNSUPPORTED when a streamed variant
 * does not fit the context's tiles. */
int mega_set_variants(int64_t h, int32_t mode, int32_t defgrad_variant, int32_t force_variant);
int mega_autotune(int64_t h, double dt, int32_t mode, int32_t reps, int32_t* choice, float* times_ms);
/* The windows of fixity code 2 (MODEL.F90:61-62, read by READ.F90:185-266):
 * ftime = FIXITY2_TIME (steps,2) and fdisp = FIXITY2_NONZERO_EBC (steps,3),
 * column-major.  In every step the corrector gives each code-2 DOF in
 * direction j the velocity fdisp(k,j) / (ftime(k,2) - ftime(k,1)) of the
 * first window k with ftime(k,1) < TIME < ftime(k,2), TIME the step's start
 * time, or 0 outside every window, with zero acceleration and the reaction
 * -FINT (MAIN.F90:447-470).  Without a call there is no window and the
 * prescribed velocity is 0.  MEGA_ERR_ARG when a window ends
 * before it starts (READ.F90:265), MEGA_ERR_STATE when no DOF has code 2. */
int mega_set_fixity2(int64_t h, int32_t steps, const double* ftime, const double* fdisp);
/* Precisions the context will step: mask bit 0 FP64, bit 1 mixed (default
 * 3).  Call before mega_search_and_shapes; only the asked-for packed records
 * are built (the FP64 records are 32 B per list entry, the mixed 16 B).
 * Stepping a precision that was not built returns MEGA_ERR_STATE. */
int mega_set_precisions(int64_t h, int32_t mask);

/* Step 0 (LINIT): neighbour search and RK shapes on the device.  Optional
 * downloads (any pointer may be NULL): gn, gstart, gstack (1-based; gstack
 * sized dim_nn_list), shp (nnz), dshp (3,nnz). *nnz and *gmaxn returned. */
int mega_search_and_shapes(int64_t h, int32_t* gn, int32_t* gstart,
                           int32_t* gstack, int64_t dim_nn_list,
                           double* shp, double* dshp, int64_t* nnz,
                           int32_t* gmaxn);

/* Advance nsteps explicit steps of size dt (IAUTO_TS = 0 semantics) in
 * mode (MEGA_MODE_* | MEGA_FLAG_*).  Device resident; the step sequence is
 * captured in a CUDA graph.  Returns the accumulated device status. */
int mega_step_resident(int64_t h, int32_t nsteps, double dt, int32_t mode);

/* As mega_step_resident, and time the stepping with CUDA events recorded on
 * the context's stream: *ms = device milliseconds for the nsteps. */
int mega_step_timed(int64_t h, int32_t nsteps, double dt, int32_t mode,
                    float* ms);

/* Time one launch of each per-step kernel averaged over reps launches on the
 * context stream (state is advanced reps times): out_ms[0] = stress/force
 * kernel, out_ms[1] = force-gather/integrator kernel. */
int mega_kernel_times(int64_t h, int32_t reps, double dt, int32_t mode,
                      float* out_ms);

/* Copy a field (enum mega_field) to host memory (sizes in the enum). */
int mega_download(int64_t h, int32_t field, double* dst);
/* Several fields at an output step in one device-to-host copy: the fields
 * (MEGA_F_* codes) one after another in dst, each in its mega_download
 * layout and the caller's node order (the arrays VTK_OUTPUT.F90 writes at
 * MAIN's output steps, gathered without one round trip per field). */
int mega_snapshot(int64_t h, int32_t nfields, const int32_t* fields, double* dst);
/* Replace a field from host memory (DSP_TOT, VEL, ACL, STRESS, STRAIN, EPS). */
int mega_upload(int64_t h, int32_t field, const double* src);
int mega_get_scalars(int64_t h, mega_scalars_t* out);
/* Device bytes held by the context. */
int64_t mega_device_bytes(int64_t h);
/* Number of kernels launched by the context since creation. */
int64_t mega_kernel_launches(int64_t h);

/* ======================================================================== */
/* Surrogate start of the rate-dependent return mapping (material 7; no    */
/* reference counterpart).  A 4 -> 64 -> 64 -> 1 tanh perceptron predicts   */
/* the converged plastic multiplier as a fraction y of its upper bound     */
/* ub = min(f / (2 mu), ((eps^n + f / (sqrt(2/3) B))^(1/n) - eps) /         */
/* sqrt(2/3)), where the plain solver starts; the Newton iteration (in      */
/* ln dgamma) then starts at clamp(y, 1e-3, 1) ub instead and converges to  */
/* the same tolerance.  Parameters theta (4545 floats)                      */
/* packed [W1 (64x4), b1 (64), W2 (64x64), b2 (64), W3 (64), b3], weights   */
/* row-major (output, input).  Features of a plastic node, with q the      */
/* trial deviatoric norm, sy0 = A + B eps^n, f = q - sqrt(2/3) sy0:         */
/*   x0 = ln(f / (sqrt(2/3) sy0)), x1 = eps^n,                              */
/*   x2 = ln(max(sqrt(2/3) f / (2 mu dt), epsdot0) / epsdot0) / 10,          */
/*   x3 = 1e3 sqrt(2/3) sy0 / (2 mu).                                       */
/* ======================================================================== */

/* Parameter count for the given hidden width (only 64 is built). */
int mega_mlp_nparams(int32_t hidden);
/* Mean-squared-error loss 0.5 mean (y - t)^2 over nb samples x (4,nb),
 * t (nb) and its gradient (nparams floats) in FP32. */
int mega_mlp_grad(int32_t hidden, const float* theta, int64_t nb, const float* x,
                  const float* t, float* grad, float* loss);
/* y (n) = network(x (4,n)); tensor_cores != 0 evaluates it as the learned
 * stress kernel does (bf16 W2 on the tensor cores, fp32 accumulation). */
int mega_mlp_eval(int32_t hidden, const float* theta, int64_t n, const float* x,
                  float* y, int32_t tensor_cores);
/* Mini-batch Adam (beta 0.9 / 0.999, eps 1e-8) on the device; theta in/out,
 * loss_per_epoch (epochs) out (may be NULL). */
int mega_mlp_train(int32_t hidden, float* theta, int64_t ns, const float* x,
                   const float* t, int32_t epochs, int32_t batch, float lr,
                   uint64_t seed, float* loss_per_epoch);
/* Install theta (host) in the context; steps whose mode has
 * MEGA_FLAG_LEARNED_GUESS then use it.  theta = NULL removes it. */
int mega_set_surrogate(int64_t h, int32_t hidden, const float* theta);
/* Log (features, y) of plastic rate-dependent nodes solved by plain Newton
 * into a device buffer of cap samples: a node is sampled when a hash of its
 * index and trial stress is 0 mod stride.  cap = 0 stops logging and frees
 * the buffer. */
int mega_log_rate_samples(int64_t h, int64_t cap, int32_t stride, uint32_t seed);
/* Copy up to cap logged samples, 5 floats each (x0..x3, y), to out (host,
 * may be NULL); *count = samples copied (or held, when out is NULL). */
int mega_rate_samples(int64_t h, float* out, int64_t cap, int64_t* count);
/* Train on the logged samples without leaving the device, starting from
 * theta (host, in/out), then install the result as by mega_set_surrogate. */
int mega_train_surrogate(int64_t h, float* theta, int32_t epochs, int32_t batch,
                         float lr, uint64_t seed, float* loss_per_epoch);

/* ======================================================================== */
/* Bond-based peridynamics (no reference counterpart: the reference's        */
/* FINT_PD is correspondence-based).  Prototype microelastic brittle model  */
/* (Silling & Askari 2005) with bond breaking, resident on the device.      */
/* ======================================================================== */

/* coo (3,n) reference positions, vol (n), vinit (3,n), fixed (n) particles
 * that keep their velocity (may be NULL); spherical horizon; micromodulus
 * c; critical stretch s_c; density rho; broken0 (nnz) initial broken flags
 * per neighbour-list entry (may be NULL; the list is the SOFT_SEARCH
 * ellipsoidal-support list with window = horizon, as mega_bin_search(...,
 * shsup = 1) returns it).  mode: MEGA_MODE_MIXED = float bond arithmetic,
 * MEGA_MODE_FP64 = double.  *nbonds = list entries (self included). */
int mega_pmb_init(int32_t n, const double* coo, const double* vol, const double* vinit,
                  const int32_t* fixed, double horizon, double micromodulus, double s_c,
                  double rho, const uint8_t* broken0, int32_t mode, int64_t* handle,
                  int64_t* nbonds);
/* nsteps of velocity-Verlet (float force, double positions); *ms device time
 * of the call when ms is not NULL. */
int mega_pmb_step(int64_t h, int32_t nsteps, double dt, float* ms);
/* what: 0 displacement (3,n), 1 velocity, 2 acceleration, 3 broken flags (nnz),
 * 4 local damage (n): the fraction of each particle's bonds (self excluded)
 * that are broken; *nbroken = bond copies broken so far (each bond breaks at
 * both ends). */
int mega_pmb_download(int64_t h, int32_t what, double* dst, int64_t* nbroken);
/* Pre-crack on the device: break every bond whose reference segment crosses
 * the rectangle corner + s edge_a + t edge_b (0 <= s, t <= 1), each a
 * double[3]; *ncut = list entries newly broken (may be NULL). */
int mega_pmb_cut(int64_t h, const double* corner, const double* edge_a, const double* edge_b, int64_t* ncut);
int mega_pmb_finalize(int64_t h);

const char* mega_status_string(int32_t status);
int mega_gpu_finalize(int64_t h);

/* No counterpart in the reference (device memory of this library).  Set-up
 * temporaries and finalised contexts leave their device blocks in a
 * process-wide cache (at most a quarter of each device's memory) and in the
 * device's default memory pool, whose release threshold the library raises
 * to its maximum, so a repeated set-up allocates nothing from the driver.
 * This call hands every cached block to the pool, puts back each device's
 * previous release threshold and trims the pool to what live contexts hold,
 * for a host program whose own allocator needs the memory.  Contexts stay
 * valid; a later set-up caches again.  Call it with no library call in
 * flight on another thread. */
int mega_release_cached_memory(void);

#ifdef __cplusplus
}
#endif
#endif /* MEGA_GPU_H */
