/* Internal state of the CPU oracle (test infrastructure only). */
#ifndef GS_ORACLE_STEP_INTERNAL_H
#define GS_ORACLE_STEP_INTERNAL_H
#include <math.h>
#include <stdint.h>
#include "step.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double x, y; } v2;
static inline v2 V2(double x, double y) { v2 r; r.x = x; r.y = y; return r; }
static inline v2 V2ADD(v2 a, v2 b) { return V2(a.x + b.x, a.y + b.y); }
static inline v2 V2SUB(v2 a, v2 b) { return V2(a.x - b.x, a.y - b.y); }
static inline v2 V2S(v2 a, double s) { return V2(a.x * s, a.y * s); }      /* v*s and s*v */
static inline v2 V2DIV(v2 a, double s) { return V2(a.x / s, a.y / s); }
static inline double V2DOT(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline double V2CROSS(v2 a, v2 b) { return a.x * b.y - a.y * b.x; }

struct og_model {
    int np, ne, ns, nvrt, ntr, nope, nland, nbfr, nnz;
    double dt, thetai, h0, dtb_min, dtb_max, velmin, rmaxvel, dfv0, coricoef, rho0, grav, dramp;
    int ihhat;
    int itr_met, tvd_limiter; double dfh0;
    double rtol; int maxiter, check_every;
    int nz; double h_s, h_c, theta_b, theta_f;
    double *ztot, *sigma, *cs;
    double time, ramp;
    /* connectivity, reference numbering */
    int32_t *isbnd, *nne_s, *nne, *nnp_s, *nnp, *el, *es, *isdel, *isn;
    int32_t *open_start, *open_nodes, *land_start, *land_nodes, *seg_iettype;
    double *amig, *ff, *face;
    /* nodes */
    double *x, *y, *depth, *drag, *Cd, *grav2, *tau, *eta1, *eta2, *qel, *mX, *elbc;
    double vortex[8]; int has_vortex;   /* storm forcing (og_set_vortex) */
    int32_t* kb; uint8_t *ndry, *nwas, *ess;
    double* z; v2* u2; double* w2; double* tr; double* tr_init;
    double *nbfr_emo, *nbfr_efa;
    int32_t *sb1, *sb2;
    /* JCG */
    double *x0, *x1, *x2, *xs, *jr, *jz, *jp, *jq, *jinvD, *jb, jrz_new;
    int32_t *indptr, *indices, *slot, *dslot; double* data;
    /* sides */
    double *len, *snx, *sny, *scx, *scy, *cori;
    int32_t* kbs; uint8_t* sdry; int8_t* sbt;
    double* zc; v2* su2; v2* btu; int32_t* btel; v2* U; double *hhat, *chi, *chi2;
    v2 *gE1, *gE2; double* Qh;
    /* elements */
    double *area, *edepth; v2* gphi; double* ssign;
    int32_t* kbe; uint8_t* edry;
    double *ez, *ew, *Qv, *etr, *prev, *inflow, *maxDt; v2* ghat;
    double *rho_n, *rho_e;       /* [np*nvrt], [ne*nvrt] densities (ntr >= 2: T and S) */
    double* tvds;                 /* TVD: inflow sum per prism and tracer [ne][nvrt][ntr] */
    int64_t cnt[4];
};

double og_compz(const og_model* m, int i, int k);
int og_update_kb_value(const og_model* m, int i);
void og_set_solver(og_model* m, double rtol, int maxiter, int check_every);

#endif
