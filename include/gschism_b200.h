/* gschism_b200: B200-native SCHISM semi-implicit hydrodynamic step, C ABI.
 *
 * One context (gs_ctx) holds a batch of ensemble members (independent meshes of any size that
 * share the vertical grid and the physics constants) resident in the HBM of one GPU.  Every
 * phase of the step runs as one launch over all members; the whole step is a fixed launch
 * sequence on the context's stream, which gs_step captures once in a CUDA graph and replays.
 *
 * Conventions: every entry point returns a gs_status (0 = GS_OK) and never aborts the process;
 * gs_last_error() describes the last failure.  Host pointers are caller-owned and only read
 * during the call.  Contexts are independent (thread-safe across contexts, not within one).
 * Field exchange (gs_state_get/put) uses the reference numbering of the member's own input and
 * level-major layout: per-level fields [nvrt][n], vectors [nvrt][n][2], tracers [ntr][nvrt][n].
 *
 * Reference interfaces replaced (paths within schism-dev/gschism):
 *   src/grid/read_and_process_grid.cpp:829-855   readHGrid connectivity        -> gs_grid_build
 *   src/solver/pcg_solver.py:538-1148            PCGSolverMultiGPU             -> gs_jcg_*
 *   src/solver/pcg_loop.cpp:182-291,467-479      NativePCG.add_partition/solve -> gs_jcg_solve_csr
 *   src/python/schism_step.py:95-334             schism_step                   -> gs_step
 *   src/python/cuda_functions.py:140-257         cufunc.<kernel>(...)          -> gs_phase
 *   src/kernels/meshdata.cu:7560-8000            get{Node,Side,Element}Var*    -> gs_state_get/put
 */
#ifndef GSCHISM_B200_H
#define GSCHISM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gs_status;
enum {
    GS_OK = 0,
    GS_ERR_ARG = 1,            /* bad argument or call order */
    GS_ERR_CUDA = 2,           /* CUDA runtime error (message in gs_last_error) */
    GS_ERR_OOM = 3,            /* device allocation failed */
    GS_ERR_NOT_CONVERGED = 4,  /* JCG reached maxiter without meeting the tolerance */
    GS_ERR_TIMEOUT = 5,        /* a bounded device wait gave up (error flag set by a kernel) */
    GS_ERR_BAD_MESH = 6,       /* connectivity check failed (hanging node, broken ball, ...) */
    GS_ERR_STATE = 7           /* field or member unknown, or buffer size mismatch */
};

enum { GS_FP64 = 0, GS_FP32_IR = 1 };   /* JCG precision: plain FP64, or FP32 inner + FP64 refinement */

/* ------------------------------------------------------------------ grid ---- */

/* Mesh connectivity exactly as readHGrid builds it (read_and_process_grid.cpp:27-574):
 * node->elements in counter-clockwise order, element-side-element table ic3, side numbering,
 * isdel/isidenode, node->nodes in counter-clockwise order.
 * elnode[ne*4] (-1 padded), i34[ne], isbnd[np] (open segment index, -2 land, -1 interior).
 * Output capacities: nne[4*ne], nnp[4*ne+np], ic3/elside[4*ne], isdel/isidenode[2*4*ne]. */
gs_status gs_grid_build(int np, int ne, const int32_t* elnode, const int32_t* i34, const int32_t* isbnd,
                        int32_t* nne_start, int32_t* nne, int32_t* nnp_start, int32_t* nnp,
                        int32_t* ic3, int32_t* elside, int32_t* isdel, int32_t* isidenode,
                        int32_t* ns_out);

/* ------------------------------------------------------------------ model ---- */

typedef struct {
    int nvrt, ntr;                         /* levels and tracers (shared by all members) */
    int nz; double h_s, h_c, theta_b, theta_f;
    const double* ztot;                    /* [nz], ztot[nz-1] = -h_s (vgrid.in, ivcor = 2) */
    const double* sigma;                   /* [nvrt-nz+1] */
    double dt, thetai, h0, dtb_min, dtb_max, velmin_btrack, rmaxvel, dfv0, coricoef, rho0, grav, dramp;
    int ihhat;
    double rtol; int maxiter, check_every; /* JCG: pcg_solver.py:1075 solve(rtol, maxiter, checkEvery) */
    int precision;                         /* GS_FP64 or GS_FP32_IR */
    double ir_inner_rtol;                  /* FP32 inner solve: each refinement sweep reduces the
                                              residual by this factor (<= 0: 0.1).  At >= 1e-2 the
                                              sweeps replace the inner CG's residual with the FP64
                                              one and continue its recurrence; tighter values
                                              restart the inner CG every sweep. */
    int ir_inner_maxiter;                  /* iteration cap of one sweep (< 1: 200) */
    int device;                            /* CUDA device ordinal */
    int itr_met;                           /* tracer transport: 1 (or 0) first-order upwind, the
                                              reference's scheme; 3 TVD (flux-limited horizontal
                                              advection, Casulli & Zanolli 2005); 4 the TVD of 3
                                              with a flux-corrected vertical step (Zalesak FCT
                                              over the implicit upwind solve) */
    int tvd_limiter;                       /* itr_met = 3, 4: 0 none (first order), 1 minmod,
                                              2 Osher (beta = 2), 3 van Leer, 4 superbee */
    double dfh0;                           /* constant vertical tracer diffusivity (m^2/s), implicit;
                                              0 = none (the reference has none) */
} gs_config;

typedef struct {
    int np, ne, nope, nland, nbfr;
    const double* x; const double* y; const double* depth;
    const double* drag;                    /* [np] bottom drag coefficient (nchi = 0) */
    const double* tau;                     /* [np][2] kinematic surface stress, m^2/s^2 */
    const double* tr_init;                 /* [ntr][nvrt][np] initial nodal tracers */
    const int32_t* elnode;                 /* [ne][3] counter-clockwise triangles */
    const int32_t* open_start;             /* [nope+1] */
    const int32_t* open_nodes;
    const int32_t* land_start;             /* [nland+1] */
    const int32_t* land_nodes;
    const int32_t* iettype;                /* [nope]: 0 none, 3 tidal harmonics */
    const double* amig; const double* ff; const double* face;   /* [nbfr] */
    const double* emo; const double* efa;  /* [open_start[nope]][nbfr] in open_nodes order */
} gs_member_desc;

typedef struct gs_ctx gs_ctx;

gs_status gs_ctx_create(const gs_config* cfg, gs_ctx** out);
gs_status gs_member_add(gs_ctx* ctx, const gs_member_desc* desc, int* member_id);
/* Host half of gs_ctx_finalize: connectivity, space-filling-curve order, matrix layout and
 * geometry of every added member, with no CUDA call (so it can run on a worker thread while the
 * GPU steps other contexts).  Optional: gs_ctx_finalize runs it when it has not been run. */
gs_status gs_ctx_prepare(gs_ctx* ctx);
/* Allocate device state for every added member, upload, build geometry and cold-start levels. */
gs_status gs_ctx_finalize(gs_ctx* ctx);
gs_status gs_ctx_destroy(gs_ctx* ctx);
const char* gs_last_error(const gs_ctx* ctx);
gs_status gs_sync(gs_ctx* ctx);
/* Run the context's work on a caller-owned cudaStream_t (passed as void*; NULL restores the
 * context's own stream).  Lets a caller order the step with its own work and time it with
 * events recorded on that stream. */
gs_status gs_set_stream(gs_ctx* ctx, void* stream);

/* Advance every member by nsteps steps (schism_step.py:95-334): replays of one captured step
 * (a CUDA graph; the step clock, time and ramp live on the device).  The first call captures it,
 * and again after gs_set_vortex switches storm forcing on or off for the first/last member;
 * it must therefore not be made while the stream is being captured by the caller. */
gs_status gs_step(gs_ctx* ctx, int nsteps);

/* Individual phases of one step, in call order (the cufunc kernels of schism_step.py). */
enum {
    GS_PHASE_BEGIN = 0,        /* time ramps and forcing for step `it` (arg) */
    GS_PHASE_BTRACK = 1,       /* backtrackAllNodes, meshdata.cu:3547 */
    GS_PHASE_PREPARE = 2,      /* elevation BCs, U, hhat/chi, ghat1 (meshdata.cu:4276-4725, 6183) */
    GS_PHASE_ASSEMBLE = 3,     /* setupCoefficientMatrixAndRHS + rollUp + setEssentialBC */
    GS_PHASE_SOLVE = 4,        /* solveWaveEquation (JCG) */
    GS_PHASE_UPDATE_ELEV = 5,  /* updateElevation */
    GS_PHASE_MOMENTUM = 6,     /* computeHorGradientAtSide, solveMomentumEquations, applyMomentumBC */
    GS_PHASE_VVEL = 7,         /* computeVerticalVelocity */
    GS_PHASE_TRANSPORT = 8,    /* computeTransport(dt) */
    GS_PHASE_LEVELS = 9,       /* ul0* wet/dry and levels (arg = it) */
    GS_PHASE_NODAL_VEL = 10    /* nodal velocities */
};
gs_status gs_phase(gs_ctx* ctx, int phase, int arg);

/* State exchange in reference numbering (see the header comment for layouts). */
enum {
    GS_F_ETA1 = 0, GS_F_ETA2 = 1, GS_F_NODE_Z = 2, GS_F_NODE_U2 = 3, GS_F_NODE_W2 = 4,
    GS_F_NODE_TR = 5, GS_F_NODE_KB = 6, GS_F_NODE_DRY = 7, GS_F_QEL = 8,
    GS_F_NODE_TAU = 9,                   /* surface stress [np][2] (kinematic) */
    GS_F_SIDE_U2 = 10, GS_F_SIDE_BTU = 11, GS_F_SIDE_ZC = 12, GS_F_SIDE_KB = 13, GS_F_SIDE_DRY = 14,
    GS_F_SIDE_U = 15, GS_F_SIDE_HHAT = 16, GS_F_SIDE_CHI = 17, GS_F_SIDE_QH = 18,
    GS_F_SIDE_BTELEM = 19, GS_F_SIDE_GRADETA1 = 20, GS_F_SIDE_GRADETA2 = 21,
    GS_F_ELEM_Z = 30, GS_F_ELEM_W = 31, GS_F_ELEM_QV = 32, GS_F_ELEM_TR = 33, GS_F_ELEM_KB = 34,
    GS_F_ELEM_DRY = 35, GS_F_ELEM_GHAT = 36,
    GS_F_CSR_DATA = 40, GS_F_CSR_INDPTR = 41, GS_F_CSR_INDICES = 42, GS_F_JCG_X = 43, GS_F_ELBC = 44,
    GS_F_JCG_X1 = 45, GS_F_JCG_X2 = 46,  /* JCG solution history x0 (last), x1, x2 */
    GS_F_NODE_RHO = 47, GS_F_ELEM_RHO = 48  /* density [nvrt][n] from tracers 0, 1 (T, S); -99 when dry */
};
/* bytes must equal the field's size (int32 for *_KB, *_DRY, SIDE_BTELEM, CSR_INDPTR/INDICES).
 * The numbering permutation runs on the device and a field crosses to the host as one copy
 * through page-locked staging.  gs_state_get returns when the data is in `host` (it waits for
 * the work queued before it); gs_state_put copies `host` to staging before it returns (the buffer
 * may be reused at once) and queues the upload on the context's stream.  A page-locked `host`
 * (gs_host_alloc, cudaHostAlloc) skips the staging copy: the DMA engine reads or writes it
 * directly, and gs_state_put / gs_set_tau then return once their copy is done. */
gs_status gs_state_get(gs_ctx* ctx, int member, int field, void* host, size_t bytes);
gs_status gs_state_put(gs_ctx* ctx, int member, int field, const void* host, size_t bytes);
/* Per-step host forcing: replace a member's surface stress [np][2] (host buffer, copied before
 * the call returns; the upload is queued on the context's stream, no synchronisation). */
gs_status gs_set_tau(gs_ctx* ctx, int member, const double* tau_host);

/* Output path (replaces DeviceToHost, src/iop/deviceToHost.py:37-224, the reference's per-field
 * device-to-host reads for writeOutput, src/iop/writeOutput.py:53-280).
 * gs_state_get_async queues the read of one field into `host`, which must be page-locked memory
 * (gs_host_alloc), and returns at once; CSR fields are not available this way.  gs_output_mark
 * records a point on the context's stream and gs_output_wait blocks the calling host thread until
 * everything queued before that mark is done (the reads included).  A writer thread can wait
 * for one record while the stepping thread queues the next steps. */
gs_status gs_state_get_async(gs_ctx* ctx, int member, int field, void* host, size_t bytes);
gs_status gs_output_mark(gs_ctx* ctx, uint64_t* ticket);
gs_status gs_output_wait(gs_ctx* ctx, uint64_t ticket);
/* Page-locked host memory for gs_state_get_async (NULL on failure) and its release. */
void* gs_host_alloc(size_t bytes);
gs_status gs_host_free(void* p);

/* Parametric storm forcing for a member (storm-surge scenarios): a radial vortex moving along a
   straight track, evaluated on the device at the start of every step.  Wind speed at distance r
   from the centre W(r) = vmax * sqrt((rmax/r)^B exp(1 - (rmax/r)^B)) (Holland profile, W(rmax) =
   vmax), counter-clockwise, plus the track velocity weighted by W/vmax; drag coefficient
   1e-3 (0.75 + 0.067 |W|), at most 3e-3; the member's surface stress (kinematic, per node) becomes
   rho_air/rho0 * Cd |W| W times the step's ramp.  No counterpart in the reference, whose wind comes
   from forcing files; this generates the synthetic input on the device.  NULL switches it off
   (the stress set by gs_set_tau / the member description is used again). */
typedef struct {
    double x0, y0;        /* centre at time 0 (m, mesh coordinates) */
    double heading;       /* direction of motion (radians from +x, counter-clockwise) */
    double speed;         /* translation speed (m/s) */
    double vmax, rmax;    /* maximum wind (m/s) and its radius (m) */
    double holland_b;     /* profile shape B (typically 1..2.5) */
    double rho_air;       /* air density (kg/m^3) */
} gs_vortex;
gs_status gs_set_vortex(gs_ctx* ctx, int member, const gs_vortex* vortex);

/* Slot-level admission.  A member's own step is the context's step minus its start step (default
   0), and its tide, ramp and storm track follow that step: a member given start K while the
   context is at step K, with its cold-start state put back (gs_state_put), steps from there on as
   a context of its own would from its step 1, bit for bit.  A start above the context's step
   parks the member: no tide, no storm, so a member at rest (cold-start state, zero stress) stays
   at rest and its solve converges at once.  GS_MEMBER_PARKED parks for good.  Between steps
   only (the call synchronises the context's stream).  No counterpart in the reference, which
   runs one forecast per process. */
#define GS_MEMBER_PARKED 2000000000
gs_status gs_set_member_start(gs_ctx* ctx, int member, int start_step);
/* The context's step index (the last BEGIN phase's argument, advanced by every gs_step). */
gs_status gs_get_step(gs_ctx* ctx, int* step);

/* Device memory a context holding members of these sizes allocates (bytes, an upper bound used
   for admission by HBM footprint).  np/ne/ns/nnz are the sums over the members.  A TVD context
   (itr_met = 3) allocates ne * nvrt * ntr * 8 bytes more, one with the vertical FCT (itr_met = 4)
   ne * nvrt * (ntr + 1) * 8 bytes more. */
size_t gs_footprint_bytes(int nvrt, int ntr, int nmem, int64_t np, int64_t ne, int64_t ns, int64_t nnz);

typedef struct {
    int64_t jcg_iters;         /* iterations of the last solve (inner FP32 iterations for IR) */
    int64_t jcg_outer;         /* FP64 refinement sweeps of the last solve (IR) */
    double jcg_relres;         /* |b - Ax| / |b| of the last solve (FP64) */
    int64_t transport_substeps;
    int64_t walk_cap_hits;     /* celestial walks that reached 40 iterations */
    int64_t btrack_stops;      /* backtracks stopped at the 38th sub-step */
    int32_t error_flags;       /* device error bits (bounded waits, non-convergence) */
} gs_stats;
gs_status gs_get_stats(gs_ctx* ctx, int member, gs_stats* out);
/* Launch shapes of the step's kernels, for the autotuner (no counterpart in the reference, whose
   launch shapes are fixed in its kernel wrappers).  For the stream kernels a = threads per block
   (a multiple of 32, at most what the compiled kernel allows) and b = the grid cap in blocks per
   SM (1..64); the kernels stride over their entities, so results do not depend on the shape.
   GS_K_JCG_TILES: a = tiles a large member is cut into, b = the smallest tile in rows (a
   multiple of 32); this changes the order of the solver's partial sums.  A change takes effect
   at the next launch (the captured step is recaptured). */
enum {
    GS_K_BTRACK = 0, GS_K_SIDE_PREP = 1, GS_K_GHAT = 2, GS_K_ASSEMBLE = 3, GS_K_MOMENTUM = 4,
    GS_K_VVEL = 5, GS_K_NODAL_VEL = 6, GS_K_NODAL_TRACER = 7, GS_K_LEVELS = 8, GS_K_JCG_TILES = 9
};
gs_status gs_set_launch(gs_ctx* ctx, int kernel, int a, int b);
gs_status gs_get_launch(gs_ctx* ctx, int kernel, int* a, int* b);

/* Tracer mass of a member: for each of the ntr tracers, the sum over the member's wet prisms of
   volume x concentration (out[ntr]), in FP64 with compensated (Neumaier two-sum) accumulation in a
   fixed order, so the value does not depend on the GPU or the launch.  The reference has no mass
   budget; this is the FP64 budget the mass-conservation checks read. */
gs_status gs_tracer_mass(gs_ctx* ctx, int member, double* out);

/* Bound of every device wait of the context's persistent kernels (the grid barrier of the
 * transport and the solver's member-level waits), in polls: after 4,096 plain polls each poll
 * sleeps about 128 ns, so the default (0 selects it: 2^24 polls) is about 2 s.  A wait that runs
 * out sets a flag; every block then leaves its kernel, later launches of the step return at
 * once, and the next gs_sync / gs_get_stats / gs_state_get returns GS_ERR_TIMEOUT and clears the
 * flag and the barrier word, so the context is usable again (its state is that of an unfinished
 * step: put a saved state back before stepping on).  No counterpart in the reference, whose
 * native solver loop bounds its host-side wait by `timeout_seconds` (pcg_loop.cpp:182-291). */
gs_status gs_set_wait_limit(gs_ctx* ctx, long long polls);

/* For tests of the recovery path only: the next solves of `member` wait for one block arrival
 * that never comes, so their bounded waits run out (see gs_set_wait_limit) and the step reports
 * GS_ERR_TIMEOUT; -1 switches it off.  No device fault or endless wait is involved.  No
 * counterpart in the reference. */
gs_status gs_test_stall_solve(gs_ctx* ctx, int member);
/* sizes of a member: np, ne, ns, nnz (CSR of the elevation matrix) */
gs_status gs_member_sizes(gs_ctx* ctx, int member, int* np, int* ne, int* ns, int* nnz);

/* ------------------------------------------------------------------ JCG on a caller CSR ---- */

/* Stand-alone Jacobi-PCG on one CSR matrix, with the semantics of PCGSolverMultiGPU.solve
 * (pcg_solver.py:1075-1124): b, x live in solver-owned device buffers; the solve computes
 * invD = 1/diag(A), atol = rtol*|b|, the parabolic guess x = 3x0 - 3x1 + x2 from the previous
 * three solutions, iterates, and rolls the history.  Device pointers returned by gs_jcg_buffers
 * are owned by the solver and stay valid until gs_jcg_destroy. */
typedef struct gs_jcg gs_jcg;
gs_status gs_jcg_create(int n, int nnz, int precision, int device, gs_jcg** out);
gs_status gs_jcg_buffers(gs_jcg* s, int32_t** indptr, int32_t** indices, double** data,
                         double** b, double** x);
gs_status gs_jcg_solve_csr(gs_jcg* s, double rtol, int maxiter, int check_every, int* iters);
/* |b - A x| / |b| of the current solution (pcg_solver.py:1127-1143) */
gs_status gs_jcg_check(gs_jcg* s, double* relres);
gs_status gs_jcg_destroy(gs_jcg* s);
const char* gs_jcg_last_error(const gs_jcg* s);

/* FP64 JCG on a caller CSR that allocates no device memory.  No counterpart in the reference.
 * For callers that cannot allocate: a host whose device memory is entirely handed out by its own
 * pool, or a loop that must not pay allocation latency mid-run.  Every argument except iters is
 * a device pointer the caller owns; x holds the initial guess on entry and the solution on exit
 * (no solution history is kept).  Same rules as gs_jcg_solve_csr: atol = rtol*|b|, test every
 * check_every iterations, *iters = maxiter when the tolerance is not met.  The work space is a
 * fixed array inside the library (about 3.1 MiB on every GPU that loads it, kept until the
 * process exits), so n is limited to 65536 rows; larger n returns GS_ERR_ARG.  The first call on
 * a device looks up that array's device address (a one-time set-up per device); that first call
 * should come before any stream capture.  The address is kept for the life of the process, so
 * the entry point must not be used on a device after that device was reset (cudaDeviceReset or a
 * reset of its primary context) in the same process.  All calls share the array: calls that
 * overlap in time on the GPU (other streams, other host threads) race and must be serialised by
 * the caller.  stream may be NULL. */
gs_status gs_jcg_solve_csr_noalloc(int n, const int32_t* indptr, const int32_t* indices, const double* data,
                                   const double* b, double* x, double rtol, int maxiter, int check_every,
                                   void* stream, int* iters);

#ifdef __cplusplus
}
#endif
#endif
