/*
 * pyib_b200.h -- C ABI of the B200 per-step hot path of PyIB.
 *
 * The reference has no plugin API; its per-step path is the Python object graph
 * built by src/pyib/solver/ib_case.py:build_runtime (ib_case.py:633-809), and the
 * device is chosen by the import-time backend module (backend.py:10-45).  Each
 * entry point below replaces one method on that graph; the comment names it
 * (paths relative to src/pyib/solver of the reference).  A ctypes binding of
 * exactly these symbols (pyib_b200/_lib.py) backs the Driver-compatible Python
 * class B200Driver.
 *
 * Conventions
 *  - Every function returns 0 on success and a positive PYIB_E_* code on error;
 *    pyib_last_error() copies the message.  No function aborts the process.
 *  - The library owns device memory.  Host buffers are caller-owned and copied
 *    (synchronously) on the context's stream.
 *  - One context per host thread; the library starts no host threads.
 *  - Fields use the dense nested-level layout (levels innermost first; per level
 *    cells, then faces of axis x,y,z, then edges of axis x,y,z, all x-fastest),
 *    with every face and edge oriented along +axis.  Absent slots hold zero.
 */
#ifndef PYIB_B200_H
#define PYIB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYIB_MAX_LEVELS 8

enum pyib_status {
  PYIB_OK = 0,
  PYIB_E_ARG = 1,        /* invalid argument (size, id, range)                  */
  PYIB_E_CUDA = 2,       /* a CUDA runtime call failed                           */
  PYIB_E_STATE = 3,      /* call out of order (e.g. step before tables uploaded) */
  PYIB_E_NOCONV = 4,     /* strict CG did not converge (ib_driver_np.py:357-376) */
  PYIB_E_NONFINITE = 5,  /* non-finite value detected                            */
  PYIB_E_DEVICE = 6      /* kernel-side check failed (index out of range)       */
};

typedef struct pyib_ctx pyib_ctx;

/* Nested-level layout (replaces the mesh handed to IBCore, ib_core_np.py:24). */
typedef struct pyib_layout {
  int32_t nlevels;
  int32_t n[PYIB_MAX_LEVELS][3];       /* cells per axis of every level box       */
  int32_t hole_lo[PYIB_MAX_LEVELS][3]; /* first hole cell (levels > 0), else 0     */
  int32_t hole_n[PYIB_MAX_LEVELS][3];  /* hole cells per axis (levels > 0), else 0 */
  double h[PYIB_MAX_LEVELS];           /* spacing of every level                  */
  double lo[PYIB_MAX_LEVELS][3];       /* lower corner of every level box         */
  int64_t ncell, nface, nedge;         /* dense slot counts                       */
  int32_t nbface;                      /* boundary (ghost) faces                   */
  int32_t device;                      /* CUDA device ordinal                      */
} pyib_layout;

/* Physics and solver parameters (Driver.__init__, ib_driver_np.py:104-153;
 * ib_case.py:698-718). */
typedef struct pyib_params {
  double rou, visc, ac, ad;  /* density, dynamic viscosity, CN weights          */
  double tol1, tol2;         /* mixed stopping test (ib_driver_np.py:311)       */
  int32_t cavity;            /* 1: no-slip walls (set_cavity(U_lid=0))          */
  int32_t check;             /* cg_check_interval (ib_case.py:714)              */
  int32_t cg_max;            /* cg_max_iterations                               */
  int32_t strict;            /* fail_on_cg_nonconvergence                       */
  int32_t precision;         /* 0: float64 throughout; 1: float32 bulk CG inside
                                float64 iterative refinement                   */
  int32_t nmarkers;          /* Lagrangian markers                              */
  double hh;                 /* delta-kernel width (ImmersedBoundary.hh)        */
  double hh3;                /* hh**3 as the host computes it (ib_immersed.py:89) */
  double mixed_tol;          /* precision 1: inner float32 solve reduces the
                                preconditioned residual norm by this factor      */
  int32_t mixed_max_sweeps;  /* precision 1: cap on float64 refinement sweeps   */
  int32_t ib_mode;           /* 0: accumulated_explicit (ib_driver_np.py:447-525);
                                1: direct, explicit; 2: direct, implicit -- the force
                                of every inner iteration replaces the last, times
                                rou*ib_alpha (ib_driver_np.py:466-486)             */
  double ib_alpha;           /* ib_mode 1, 2: force relaxation (Driver.ib_alpha)   */
} pyib_params;

/* Per-solve statistics (Driver.helm_solve finish(), ib_driver_np.py:338-377). */
typedef struct pyib_solve_stats {
  int32_t iterations;
  int32_t converged;
  double rel_residual;       /* sqrt(|r_true|^2 / |r_0|^2)                      */
  double tol_ratio;          /* sqrt(eta_true / threshold)                      */
  double eta0, threshold;
  int32_t refinements;       /* outer float64 refinement sweeps (precision 1)   */
  int32_t pad;
} pyib_solve_stats;

/* Per-step statistics (Driver.step diagnostics, ib_driver_np.py:498-509). */
typedef struct pyib_step_stats {
  int32_t max_iterations;    /* helmholtz_iterations_last_step                  */
  int32_t total_iterations;  /* sum over the inner solves                       */
  int32_t all_converged;
  int32_t ib_updates;        /* ib_force_updates_last_step                      */
  double max_rel_residual, max_tol_ratio;
} pyib_step_stats;

/* Table ids for pyib_upload (host-built operator tables). */
enum pyib_table {
  PYIB_T_PREC = 0,          /* f64[nedge] diagonal preconditioner, 0 = masked (ib_driver_np.py:78-88) */
  PYIB_T_INLET_IDX,         /* i32[n] inlet edges                                 */
  PYIB_T_INLET_VAL,         /* f64[n] inlet stream values y*te_z (ib_driver_np.py:271) */
  PYIB_T_CURL_PTR, PYIB_T_CURL_COL, PYIB_T_CURL_VAL,     /* CSR faces x edges           */
  PYIB_T_ROT_PTR, PYIB_T_ROT_COL, PYIB_T_ROT_VAL,        /* CSR edges x faces           */
  PYIB_T_P_PTR, PYIB_T_P_COL, PYIB_T_P_VAL3,             /* CSR cells x faces, 3 values */
  PYIB_T_I_PTR, PYIB_T_I_COL, PYIB_T_I_VAL3,             /* CSR faces x cells, 3 values */
  PYIB_T_CF_PTR, PYIB_T_CF_FACE,                         /* cell -> signed face list    */
  PYIB_T_F_LO, PYIB_T_F_HI, PYIB_T_F_AOL,                /* face cells (ghost ext), AoL */
  PYIB_T_VOLCI,                                          /* f64[ncell] 1/volume (0 absent) */
  PYIB_T_BF_FACE, PYIB_T_BF_CELL, PYIB_T_BF_INFO, PYIB_T_BF_AF, /* boundary (ghost) faces */
  PYIB_T_PA_BITS, PYIB_T_PA_ROW, PYIB_T_PA_PTR, PYIB_T_PA_COL, PYIB_T_PA_VAL, /* matvec patch A */
  PYIB_T_PV_BITS, PYIB_T_PV_ROW, PYIB_T_PV_PTR, PYIB_T_PV_COL, PYIB_T_PV_VAL, /* matvec patch V */
  PYIB_T_PR_BITS, PYIB_T_PR_ROW, PYIB_T_PR_PTR, PYIB_T_PR_COL, PYIB_T_PR_VAL, /* matvec patch RI */
  PYIB_T_LC_CAND, PYIB_T_LC_FIDX,                        /* load-correction cell lists  */
  PYIB_T_LC_CPOS,                                        /* f64[ncell*3] cell centres   */
  PYIB_T_PREC_BITS,         /* u32 bitmask: edges whose PREC differs from their level's value */
  PYIB_T_PREC_REG,          /* f64[nlevels] PREC of a level's regular edges              */
  PYIB_T_PA_IDS, PYIB_T_PV_IDS, PYIB_T_PR_IDS, /* i32 dense ids of the patch rows (A, V, RI) */
  PYIB_T_COUNT
};

/* Field ids for pyib_set_field / pyib_get_field. */
enum pyib_field {
  PYIB_F_S = 0,        /* f64[nedge] stream function s                        */
  PYIB_F_S_OLD,        /* f64[nedge] previous s                               */
  PYIB_F_U,            /* f64[nface] face flux (last_face_flux)               */
  PYIB_F_VC,           /* f64[3*ncell] cell velocity, component-major         */
  PYIB_F_VC_GHOST,     /* f64[3*nbface] ghost-cell velocity                   */
  PYIB_F_RES_C,        /* f64[3*ncell] last momentum residual                 */
  PYIB_F_RES_E,        /* f64[nedge] edge residual (solve right-hand side)    */
  PYIB_F_FE,           /* f64[3*ncell] Eulerian IB force ib_force_E           */
  PYIB_F_FL,           /* f64[3*M] Lagrangian IB force ib_force_L (marker-major) */
  PYIB_F_MARKERS,      /* f64[3*M] marker positions (marker-major)            */
  PYIB_F_MVEL,         /* f64[3*M] desired marker velocity                    */
  PYIB_F_DS,           /* f64[M] marker volume ds**3 as the host computes it (ib_immersed.py:106) */
  PYIB_F_WORK_E,       /* f64[nedge] scratch edge vector (operator tests)     */
  PYIB_F_WORK_E2,      /* f64[nedge] scratch edge vector (operator tests)     */
  PYIB_F_WORK_C3,      /* f64[3*ncell] scratch cell vector (operator tests)   */
  PYIB_F_WORK_F,       /* f64[nface] scratch face vector (operator tests)     */
  PYIB_F_IB_CELL,      /* i32[125*M] stencil cells (dense ids), read only     */
  PYIB_F_IB_W,         /* f64[125*M] stencil weights, read only               */
  PYIB_F_IB_BASE,      /* i32[3*M] rint((x - pos_ref)/dx), read only          */
  PYIB_F_LAG_TMP,      /* f64[3*M] last interpolated marker velocity          */
  PYIB_F_DINV,         /* f32[nedge] mixed solver's 1/diag(A), read only      */
  PYIB_F_COUNT
};

/* ---- lifetime ------------------------------------------------------------ */
int pyib_create(const pyib_layout* layout, pyib_ctx** out);
int pyib_destroy(pyib_ctx* ctx);
int pyib_last_error(const pyib_ctx* ctx, char* buf, size_t n);
int pyib_version(char* buf, size_t n);

/* Host tables (IBCore.__init__ device transfer, ib_core_np.py:123-126;
 * build_A upload, ib_sparse.py:93-95).  bytes must match the table's type. */
int pyib_upload(pyib_ctx* ctx, int32_t table, const void* host, size_t bytes);
/* Patch-table row counts {A rows, V rows, RI rows[, upper faces exact]}; call after
 * uploads.  A fourth count != 0 states that every edge of the nodes on a level's
 * upper faces is an RI patch row or masked, so the RI template skips those nodes. */
int pyib_finalize(pyib_ctx* ctx, const int64_t* counts, int32_t ncounts);
int pyib_set_params(pyib_ctx* ctx, const pyib_params* params);
/* Marker-stencil geometry (ImmersedBoundary.__init__, ib_immersed.py:25-44). */
int pyib_set_ib_geometry(pyib_ctx* ctx, const double* pos_ref, double dx);

/* ---- fields ---------------------------------------------------------------- */
int pyib_set_field(pyib_ctx* ctx, int32_t field, const void* host, size_t count);
int pyib_get_field(pyib_ctx* ctx, int32_t field, void* host, size_t count);

/* ---- operators (tests and the Python driver) ------------------------------ */
/* w = (R I V P C) p with Dirichlet/absent rows zeroed: IBCore.flow_mat +
 * DirBC (ib_core_np.py:168-175, ib_driver_np.py:29-33) / Asp @ pp
 * (ib_driver_np.py:387).  alpd 1 selects the viscous block (0: without it);
 * alpd 3 computes the same product (viscous block on) with the single-pass fused
 * kernel the float64 CG uses, whose rows are bit-identical to the three-kernel path.
 * alpd 5 and 9 pin the form of the curl+interp and viscous stencils (viscous block
 * on): 5 runs them as one fused kernel, 9 as two kernels; both give the same bits,
 * and alpd 1 uses whichever form the autotuner picked (two kernels before tuning). */
int pyib_matvec(pyib_ctx* ctx, int32_t in_field, int32_t out_field, double dt, int32_t alpd);
/* Single-component operators on the scratch fields:
 *  op 0: curl   WORK_E  -> WORK_F  (ib_core_np.py:133)
 *  op 1: rot    WORK_F  -> WORK_E  (ib_core_np.py:129)
 *  op 2: interp WORK_F  -> WORK_C3 (ib_core_np.py:150)
 *  op 3: integr WORK_C3 -> WORK_F  (ib_core_np.py:144)                        */
int pyib_operator(pyib_ctx* ctx, int32_t op);
/* Driver.calc_vel (ib_driver_np.py:267-291): reads S, writes S (boundary-set),
 * U, VC and VC_GHOST. */
int pyib_calc_vel(pyib_ctx* ctx);
/* Driver.conv_diff (ib_driver_np.py:293-303) on U, VC: writes conv to WORK_C3
 * and diff to RES_C (test entry point). */
int pyib_conv_diff(pyib_ctx* ctx);
/* Driver.helm_solve (ib_driver_np.py:311-410): RES_E and S in, S out. */
int pyib_helm_solve(pyib_ctx* ctx, double dt, pyib_solve_stats* stats);
/* Driver.step (ib_driver_np.py:412-532), accumulated explicit forcing.
 * markers/vel: host positions and velocities at the new time level (the
 * prescribed motion, ib_driver_np.py:441-451), or NULL for a fixed body. */
int pyib_step(pyib_ctx* ctx, double dt, double dt_old, int32_t inner,
              const double* markers, const double* vel, pyib_step_stats* stats);

/* ---- batches of independent cases on one GPU ------------------------------- */
/* No counterpart in the reference, which runs one case per process
 * (ib_case.py:1413-1648).  A batch steps many cases of uneven size together: each
 * step runs pyib_step's parts per case, and the CG iterations of every case's
 * Helmholtz solves run together, one launch per kernel stage (curl+interp, viscous
 * and integr+rot templates with their exact rows, residual update, direction
 * update) over the tiles of all cases still iterating, `check` iterations to one
 * CUDA graph.  Each case computes exactly what pyib_step computes on its own
 * context (same kernels, grids and reduction orders).  The contexts stay owned by
 * the caller, share one device, one precision and one CG check interval, and must
 * not be used from another thread while a batch call runs. */
typedef struct pyib_batch pyib_batch;
int pyib_batch_create(pyib_ctx* const* ctxs, int32_t n, pyib_batch** out);
int pyib_batch_destroy(pyib_batch* batch);
int pyib_batch_last_error(const pyib_batch* batch, char* buf, size_t n);
/* One step of every case: dt[c], dt_old[c] and (when markers is not NULL) the
 * prescribed marker positions and velocities of case c, as pyib_step; stats[c]
 * receives case c's statistics.  A failing case stops the call with its status and
 * its message (pyib_batch_last_error). */
int pyib_batch_step(pyib_batch* batch, const double* dt, const double* dt_old, int32_t inner,
                    const double* const* markers, const double* const* vel, pyib_step_stats* stats);
/* out[0] CUDA-event seconds of the batched iteration chunks, out[1] batched kernels
 * launched, out[2] graph captures (out holds 3 doubles); reset clears them. */
int pyib_batch_timing(pyib_batch* batch, double* out, int32_t reset);

/* ---- immersed boundary (ib_immersed.py) ------------------------------------ */
/* 5^3 stencil ids and weights (ImmersedBoundary._build_cells_weights, 63-81). */
int pyib_ib_stencil(pyib_ctx* ctx);
/* Eulerian -> Lagrangian: LAG_TMP = interp(VC) (_interp_stencil, 87-93). */
int pyib_ib_interp(pyib_ctx* ctx);
/* Lagrangian -> Eulerian: FE = spread(FL) with ds^3 weights (_spread_stencil,
 * 103-111).  Deterministic: contributions sorted by cell, summed in input order. */
int pyib_ib_spread(pyib_ctx* ctx);
/* Derivative of the interpolation with respect to the marker positions, for adjoint
 * gradients: jac[9*m + 3*c + d] = d u_L[m, c] / d x_m[d] (M*9 doubles, host buffer) at
 * the current markers and PYIB_F_VC.  The derivative of ImmersedBoundary's weights
 * and interpolation (ib_immersed.py:12-19, 63-93); the reference has no derivative. */
int pyib_ib_interp_dx(pyib_ctx* ctx, double* jac);

/* Offline pressure recovery (ib_postprocess.py:49-107, recover_pressure): Jacobi-
 * preconditioned CG from x = 0 on a caller's symmetric positive definite CSR matrix
 * (n rows; ptr[n+1], col, val on the host), stopping when |b - A x| <= rtol |b| (the
 * test of scipy.sparse.linalg.cg with atol = 0), checked every 10 iterations.  The
 * matrix and vectors are copied into the context's grow-only workspace (indices
 * are checked on the host first); x (n doubles, host) receives the solution, *iterations the
 * iterations run, *solve_ms (nullable) the device time from the first kernel to
 * the last (CUDA events).  Not converged: PYIB_E_NOCONV, x holding the last iterate. */
int pyib_graph_pcg(pyib_ctx* ctx, int64_t n, const int64_t* ptr, const int32_t* col, const double* val,
                   const double* rhs, double* x, double rtol, int32_t max_iterations, int32_t* iterations,
                   double* solve_ms);

/* ---- loads (ib_interior.py) ------------------------------------------------- */
/* ClosedSphereLoadCorrection.evaluate + fluid force/moment integrals
 * (ib_interior.py:216-239, 291-296).  out[0:3] force_fluid, [3:6] moment_fluid,
 * [6:9] linear momentum, [9:12] angular momentum, [12] indicator volume. */
/* Offline pressure recovery, all of it on the device (ib_postprocess.py:49-107,
 * recover_pressure): input checks with the reference's messages (PYIB_E_ARG),
 * the face weights A/|x2-x1| and jumps 0.5 (g1+g2).(x2-x1), the Laplacian with
 * cell 0 pinned, the connectivity check, Jacobi-preconditioned CG from zero with
 * the stop |r| < rtol |b| (scipy's cg, atol = 0; PYIB_E_NOCONV after
 * max_iterations), the boundary-adjacent zero-mean gauge and the weighted
 * projection residual.  Host arrays: positions and gradient ncell x 3, face_cells
 * nface x 2 (second cell -1 on boundary faces), face_area nface; pressure
 * receives ncell doubles.  info (nullable, 7 doubles): weighted residual rms,
 * iterations, 1 if the gauge used boundary cells, CG device ms, whole-call device
 * ms (copies included), connectivity sweeps, CSR nonzeros.  All sums are in fixed
 * orders, so repeated calls give the same bits. */
int pyib_recover_pressure(pyib_ctx* ctx, int64_t ncell, const double* positions, int64_t nface,
                          const int64_t* face_cells, const double* face_area, const double* gradient, double rtol,
                          int32_t max_iterations, double* pressure, double* info);

int pyib_loads(pyib_ctx* ctx, const double* centre, double radius, double width,
               double density, int32_t fixed_centre, const double* centre0, double* out);

/* Diagnostics for a sampled step (ib_case.py:1129-1224): out[0] max speed,
 * out[1] max |vol*cdiv(U)|, out[2] max slip, out[3] rms slip. */
int pyib_diagnostics(pyib_ctx* ctx, double* out);

/* Device timing of the CG solves since the last reset: out[0] CG seconds
 * (CUDA events around each solve), out[1] CG iterations, out[2] kernels launched
 * by this context, out[3] and out[4] the z-chunk depths of the cell and node
 * stencil tiles the autotuner picked (out holds 5 doubles). */
int pyib_cg_timing(pyib_ctx* ctx, double* out, int32_t reset);
/* The matvec plan the autotuner chose (benchmark support; the reference has no
 * tiles to tune).  out holds 8 int32: for the float64 matvec, then the float32
 * matvec of the mixed solver, each [tuned (0/1), cell-tile z depth, node-tile z
 * depth, curl+interp and viscous templates fused (1) or two kernels (0)]. */
int pyib_matvec_plan(pyib_ctx* ctx, int32_t* out);
/* CUDA events on the context's stream: which=0 records the start, which=1 records
 * the end, waits for it and returns the elapsed milliseconds. */
int pyib_event(pyib_ctx* ctx, int32_t which, double* elapsed_ms);
/* Times reps back-to-back matvecs (WORK_E -> WORK_E2, viscous block) with CUDA
 * events (benchmark support).  ms_per holds 7 doubles: [0] one matvec, then one
 * launch of each of its kernels alone: [1] curl+interp template, [2] its patch
 * rows, [3] viscous template, [4] its patch rows, [5] integr+rot template with the
 * dot, [6] its patch rows with the final reduction.  When the tuned matvec runs the
 * curl+interp and viscous templates as one kernel, [1] times that kernel and [3] is 0.  With params.precision = 1 the
 * float32 matvec of the mixed solver is timed instead (on a float32 copy of WORK_E). */
int pyib_bench_matvec(pyib_ctx* ctx, int32_t reps, double dt, double* ms_per);

/* The single-pass float64 matvec of the CG (k_mvF with its exact-row kernels),
 * timed with CUDA events over reps calls on WORK_E: ms_per[0] the whole matvec,
 * [1] exact vc rows plus the listed template vc, [2] exact vq rows, [3] k_mvF,
 * [4] exact w rows with the final dot; ms_per[5] = the tuned node planes per block.
 * Counterpart: the operator timed is Asp @ pp / IBCore.flow_mat (ib_driver_np.py:387). */
int pyib_bench_matvec_fused(pyib_ctx* ctx, int32_t reps, double dt, double* ms_per);

/* Deterministic spreading that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc (a code running inside a device-memory
 * budget fixed at start-up, or one whose framework allocator owns all device
 * memory).  Same result as pyib_ib_spread: out[d*ncell + c] = sum over the
 * contributions with cell c, in (marker, offset) order, of f[3*m+d] * w * ds3[m].
 * All pointers are device pointers: cell/w are the 125*nmarkers stencil cells and
 * weights (PYIB_F_IB_CELL, PYIB_F_IB_W), ds3 the marker volumes, f the marker-major
 * forces, out 3*ncell doubles (component-major, fully overwritten).
 *  - Scratch: one fixed file-scope device array of 17,408,256 bytes, enough for at
 *    most 8192 markers; larger counts return PYIB_E_ARG.  Every GPU that loads the
 *    library holds this array until the process exits.
 *  - Cell ids are checked on the device: a contribution whose id lies outside
 *    [0, ncell) is skipped (nothing is written outside out) and the call returns
 *    PYIB_E_DEVICE; the valid contributions are still summed into out.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call before
 *    any stream capture.
 *  - Calls share the array: calls that overlap on the GPU (different streams, or
 *    threads without ordering) race.  Run them in one stream or serialize them.
 *  - stream is a cudaStream_t (NULL: the legacy default stream).  The call reads
 *    the count of rejected ids back in stream order, so it returns only after its
 *    work on that stream has finished. */
int pyib_spread_noalloc(const int32_t* cell, const double* w, const double* ds3, const double* f,
                        int32_t nmarkers, int64_t ncell, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PYIB_B200_H */
