/* CPU oracle of the SCHISM semi-implicit step (test infrastructure only; see oracle.h).
 *
 * Scope (same as the CUDA product): triangles, ics = 1 (planar coordinates), ivcor = 2 (SZ),
 * itur = 0 (constant vertical viscosity), no vegetation, no baroclinic force (ibc = 1),
 * nchi = 0 (drag coefficient per node), imm = 0, ihorcon = 0, ntip = 0 (no tidal potential),
 * no atmospheric pressure, open boundaries with iettype 0/3 (none / tidal harmonics) and
 * ifltype = 0, first-order upwind transport (itr_met = 1, the reference's scheme) or flux-limited
 * TVD horizontal transport (itr_met = 3, restated from Casulli & Zanolli 2005: the reference has
 * no TVD), the same with a flux-corrected vertical step (itr_met = 4, Zalesak's FCT over the
 * implicit upwind solve), optional constant vertical tracer diffusivity.
 */
#ifndef GS_ORACLE_STEP_H
#define GS_ORACLE_STEP_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int np, ne, nvrt, ntr, nope, nland, nbfr;
    const double* x;  const double* y;  const double* depth;
    const double* drag;          /* [np] */
    const double* tau;           /* [np][2] kinematic surface stress */
    const double* tr_init;       /* [ntr][nvrt][np] initial nodal tracers */
    const int32_t* elnode;       /* [ne][3] */
    const int32_t* open_start;   /* [nope+1] */
    const int32_t* open_nodes;
    const int32_t* land_start;   /* [nland+1] */
    const int32_t* land_nodes;
    const int32_t* iettype;      /* [nope] */
    const double* amig; const double* ff; const double* face;   /* [nbfr] */
    const double* emo;  const double* efa;  /* [open_start[nope]][nbfr], same order as open_nodes */
    int nz; double h_s, h_c, theta_b, theta_f;
    const double* ztot;          /* [nz] */
    const double* sigma;         /* [nvrt-nz+1] */
    double dt, thetai, h0, dtb_min, dtb_max, velmin_btrack, rmaxvel, dfv0, coricoef, rho0, grav, dramp;
    int ihhat;
    int itr_met, tvd_limiter;    /* transport: 1 upwind, 3 TVD, 4 TVD + vertical FCT; limiter 0 .. 4 */
    double dfh0;                 /* constant vertical tracer diffusivity (implicit) */
} og_input;

/* Exchange field codes (level-major [nvrt][n] for per-level fields, components interleaved
 * last for vectors, tracers [ntr][nvrt][n]).  The CUDA product uses the same numbers. */
enum {
    OGF_ETA1 = 0, OGF_ETA2 = 1, OGF_NODE_Z = 2, OGF_NODE_U2 = 3, OGF_NODE_W2 = 4,
    OGF_NODE_TR = 5, OGF_NODE_KB = 6, OGF_NODE_DRY = 7, OGF_QEL = 8, OGF_NODE_TAU = 9,
    OGF_SIDE_U2 = 10, OGF_SIDE_BTU = 11, OGF_SIDE_ZC = 12, OGF_SIDE_KB = 13, OGF_SIDE_DRY = 14,
    OGF_SIDE_U = 15, OGF_SIDE_HHAT = 16, OGF_SIDE_CHI = 17, OGF_SIDE_QH = 18,
    OGF_SIDE_BTELEM = 19, OGF_SIDE_GRADETA1 = 20, OGF_SIDE_GRADETA2 = 21,
    OGF_ELEM_Z = 30, OGF_ELEM_W = 31, OGF_ELEM_QV = 32, OGF_ELEM_TR = 33, OGF_ELEM_KB = 34,
    OGF_ELEM_DRY = 35, OGF_ELEM_GHAT = 36,
    OGF_CSR_DATA = 40, OGF_CSR_INDPTR = 41, OGF_CSR_INDICES = 42, OGF_JCG_X = 43,
    OGF_ELBC = 44, OGF_JCG_X1 = 45, OGF_JCG_X2 = 46,
    OGF_NODE_RHO = 47, OGF_ELEM_RHO = 48
};

typedef struct og_model og_model;

og_model* og_model_create(const og_input* in, int* status);
void og_model_free(og_model* m);
int og_model_sizes(const og_model* m, int* np, int* ne, int* ns, int* nnz);
/* copy a field out / in (doubles or int32 according to the field) */
int og_get(const og_model* m, int field, void* out);
int og_put(og_model* m, int field, const void* in);

/* phases of the step (schism_step.py:95-334), callable one by one for parity tests */
void og_begin_step(og_model* m, int it);                       /* time ramps, forcing */
/* storm forcing: p = {x0, y0, heading, speed, vmax, rmax, B, rho_air}, NULL = off (stress kept) */
void og_set_vortex(og_model* m, const double* p);
void og_btrack(og_model* m);                                   /* mdc:3547-3660 */
void og_prepare_elevation(og_model* m, double time);           /* BCs, U, hhat/chi, ghat1 */
void og_assemble(og_model* m, double time);                    /* mdc:3182-3474 */
void og_essential_bc(og_model* m);                             /* roll-up + mdc:4400-4446 */
int  og_jcg_solve(og_model* m, double rtol, int maxiter, int check_every, double* relres);
void og_update_elevation(og_model* m);                         /* mdc:4449-4456 */
void og_momentum(og_model* m, double time);                    /* mdc:5045-5454 */
void og_vertical_velocity(og_model* m);                        /* mdc:5978-6103 */
int  og_transport(og_model* m, double dt);                     /* step:78-93 */
void og_levels(og_model* m, int it);                           /* ul0*, mdc:5521-5762 */
void og_nodal_velocities(og_model* m);                         /* mdc:5765-5929 */
void og_density(og_model* m);                                  /* mdc:6776-6812 (end of og_levels) */
double og_eqstate(double T, double S);                         /* eqstate.h:12-52 */
/* one whole step; returns the JCG iteration count */
int  og_step(og_model* m, int it);
/* diagnostics: [0] JCG iterations of the last solve, [1] transport sub-steps of the last
 * transport, [2] btrack walks that hit the iteration cap, [3] btrack sub-step hard stops */
void og_counters(const og_model* m, int64_t* out4);
/* tracer mass sum_e sum_k V_ek C_ek per tracer, with a compensated (two-sum) accumulator */
void og_tracer_mass(const og_model* m, double* out_ntr);
/* the flux-corrected vertical step of itr_met = 4 on one column of n prisms (0 at the bottom):
 * q[j] the flux between prisms j and j+1, v the volumes, co the field before the step, cl the
 * implicit upwind result; out the corrected field (may be cl).  Returns 0, or -1 for n < 1. */
int og_fct_column(int n, double dt, const double* q, const double* v, const double* co, const double* cl,
                  double* out);
/* initialise: geometry, CSR pattern, cold-start levels (schism_init.py:78-103) */
int og_model_init(og_model* m);

#ifdef __cplusplus
}
#endif
#endif
