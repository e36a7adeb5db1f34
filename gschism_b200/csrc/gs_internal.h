// Internal declarations of gschism_b200 (host C++ and CUDA).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gschism_b200.h"

#include <vector_types.h>   // double2 (plain struct, usable from host-only translation units)

namespace gs {

struct Connectivity {
    std::vector<int32_t> nne_start, nne, nnp_start, nnp, ic3, elside, isdel, isidenode;
    int ns = 0;
};
int build_connectivity(int np, int ne, const int32_t* elnode, const int32_t* i34, const int32_t* isbnd,
                       Connectivity& c);
void hilbert_order(int n, const double* x, const double* y, std::vector<int32_t>& perm);

constexpr int kMaxTracers = 8;
constexpr int kMaxLevels = 64;
// default bound of a device wait, in polls: about 2 s of polling
constexpr long long kWaitPolls = 1ll << 24;
constexpr int kMaxBfr = 8;
constexpr int kMaxDeg = 24;        // max node degree supported by the per-row assembly
constexpr int kVortexParams = 9;  // x0, y0, heading, speed, vmax, rmax, B, rho_air, enabled
constexpr int kMassBlocks = 256;    // fixed grid of the tracer mass budget (deterministic sums)
constexpr int kIrVectors = 9;      // FP32 vectors of the refinement solve: (u, w, s, p) x 2, d

// Device error bits (gs_stats.error_flags)
enum : int {
    ERR_BARRIER_TIMEOUT = 1,
    ERR_JCG_NOT_CONVERGED = 2,
    ERR_DEGREE = 4,
};

// Static geometry of one element for the backtracking gathers: the corner positions and node ids
// in element node order, the area, and in perm which node starts each of the element's sides in
// the element's orientation (bits 2j..2j+1 for side j) and whether sides j and j+1 meet at an
// obtuse corner (bit 8+j).  One 80-byte record replaces the side -> node -> x/y chains of
// dependent loads of the walk and the interpolation.
struct alignas(16) ElemGeo {
    double2 p[3];
    double area;
    int32_t n[3];
    int32_t perm;
};
static_assert(sizeof(ElemGeo) == 80, "ElemGeo layout");

// Launch shapes of the step's stream kernels: threads per block and the grid cap in blocks per
// SM (the kernels loop over their entities with a grid stride, so any shape gives the same
// results), and the tiling of the JCG work list.  The defaults are hand-chosen; gs_set_launch
// (the autotuner) replaces them.  The kernel ids equal the GS_K_* codes of the C ABI.
enum : int {
    LK_BTRACK = 0, LK_SIDE_PREP, LK_GHAT, LK_ASSEMBLE, LK_MOMENTUM, LK_VVEL, LK_NODAL_VEL,
    LK_NODAL_TRACER, LK_LEVELS, LK_COUNT
};
struct LaunchShape { int block, per_sm; };
struct JcgTiling {
    int tiles = 592;        // tiles of a large member (one per block of a 4-blocks-per-SM grid)
    int min_rows = 1024;    // smallest tile (four rows per thread of a 256-thread block)
    int per_sm = 4;         // cap of the cooperative grid in blocks per SM
};
struct LaunchTable {
    // the node gathers (nodal velocities, nodal tracers) at 512 threads: the tuner's choice on
    // both the 1M basin and the 64-member ensemble (nodal velocities 20% faster than at 128)
    LaunchShape k[LK_COUNT] = {{128, 32}, {256, 16}, {256, 16}, {128, 16}, {128, 32},
                               {128, 32}, {512, 32}, {512, 16}, {256, 16}};
    JcgTiling jcg;
};

// Batch-wide constants shared by all members (copied into kernel arguments).
struct Phys {
    int nvrt, ntr, nz;
    double h_s, h_c, theta_f;
    double dt, thetai, h0, dtb_min, dtb_max, velmin, rmaxvel, dfv0, coricoef, rho0, grav, dramp;
    int ihhat;
    int tvd, tvd_limiter;          // TVD horizontal transport and its limiter (0 none .. 4 superbee)
    int tvd_vert;                  // flux-corrected vertical step (itr_met = 4)
    double dfh0;                   // constant vertical tracer diffusivity (implicit; 0 = none)
};

// Device state of a batch: members concatenated entity-wise, SFC order inside each member.
// Per-level fields are level-major: f[k * N + i].
struct Dev {
    int NP, NE, NS, NNZ, NB, nmem;
    // nodes
    double *x, *y, *depth, *drag, *tau, *eta1, *eta2, *qel, *elbc;
    double *tau_own;               // [NP][2] the members' own surface stress (restored after a storm)
    int32_t *pn_ref, *ps_ref, *pe_ref;   // internal entity -> reference index within its member
    int32_t *kb;
    uint8_t *ndry, *nwas, *ess;
    int32_t *nbnd;                 // -1 interior, -2 land-only, >= 0 open
    double *z, *w2, *tr;           // [nvrt][NP], [ntr][nvrt][NP]
    double2 *u2;                   // [nvrt][NP]
    int32_t *nne_s, *nne, *nne_loc; // node -> elements (CCW) and the node's local index there
    int32_t *nnp_s, *nnp, *nbr_slot, *diag_slot;
    int32_t *sb1, *sb2;            // open-boundary node -> linked boundary sides
    // open boundary nodes (elevation BC)
    int32_t *bn_node, *bn_ietype, *bn_nbfr;
    double *bn_emo, *bn_efa, *bn_amig, *bn_ff, *bn_face;   // [NB][kMaxBfr]
    // CSR of the elevation matrix (rows = nodes)
    // elevation matrix (rows = nodes) in SELL-32 layout: slices of 32 consecutive rows; entry k
    // of row i sits at sell[i/32].x + 32*k + i%32 for k < sell[i/32].y (the slice's widest row).
    // A row's entries are in increasing column order; padding entries hold the row's own column
    // and a zero value.
    int2* sell;
    int32_t *indices;
    double *A;
    float *A32;                    // D^-1 A in FP32 (refinement solve)
    // JCG vectors
    double *b, *xs, *r, *zz, *p0, *p1, *q, *invD, *xh0, *xh1, *xh2;
    float *ir32, *diag32;          // ir32: kIrVectors FP32 vectors of the refinement solve
    // sides
    int32_t *sn, *se;              // [2][NS]
    double *len, *snx, *sny, *scx, *scy, *cori;
    int32_t *kbs;
    uint8_t *sdry;
    int8_t *sbt;                   // 0 interior, 1 land, 2 open
    double *zc, *Qh;               // [nvrt][NS]
    double2 *su2, *btu;            // [nvrt][NS]
    int32_t *btel;                 // [nvrt][NS]
    double2 *U, *gE1, *gE2;
    double2 *sgh;                  // [3][NS] a side's terms of the element-averaged ghat
    double *hhat, *chi, *chi2;
    // elements
    int32_t *en, *es;              // [3][NE]
    ElemGeo* egeo;                 // [NE]
    double *area;
    double2 *gphi;                 // [3][NE]
    int8_t *ssgn;                  // [3][NE]
    int32_t *kbe;
    uint8_t *edry;
    double *ez, *ew, *Qv;          // [nvrt][NE]
    double *etr, *prev;            // [ntr][nvrt][NE]
    double *tvds;                  // [ntr][nvrt][NE] TVD inflow sums (allocated with TVD only)
    double *vgam;                  // [nvrt][NE] vertical sweep scratch (allocated with vertical FCT only)
    double *maxDt;
    double2 *ghat;
    double *rho_n, *rho_e;         // [nvrt][NP], [nvrt][NE] densities (allocated with >= 2 tracers)
    // members
    int32_t *mem_np0, *mem_ne0;    // entity offsets [nmem+1]
    double *mem_start;             // [nmem] start step of each member (its step = clk[0] - start)
    double *vort;                  // [nmem][kVortexParams] storm parameters (gs_vortex + enabled flag)
    int32_t *elem_member;          // [NE]
    double *mem_rem, *mem_dtb;     // transport sub-cycling per member
    unsigned long long *mem_mindt; // positive doubles ordered as unsigned
    int32_t *mem_nsub;
    // JCG work list: tiles of rows inside one member
    int ntiles;
    int32_t *tile_r0, *tile_r1, *tile_mem, *mem_t0, *mem_t1;
    double *tile_part;             // [4][ntiles] partial sums
    double *mem_scal;              // per member scalars (see jcg.cu)
    int32_t *mem_iters, *mem_outer;
    // global control
    double* clk;                   // [3] step, time = step * dt, ramp (set on the device each step)
    unsigned* bar;                  // grid barrier word (zero between launches)
    int32_t *err;                  // ERR_* flags: set on the device, cleared by the host after reporting
    long long wait_polls;          // bound of every device wait, in polls (~128 ns each after 4096)
    unsigned long long *counters;  // [4]: walk cap hits, btrack stops, ...
};

}  // namespace gs

#ifdef __CUDACC__
#define GS_HD __host__ __device__ __forceinline__
#else
#define GS_HD inline
#endif
