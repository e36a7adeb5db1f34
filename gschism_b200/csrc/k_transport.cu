// Tracer transport, first-order upwind (computeTransport, schism_step.py:78-93; kernels
// meshdata.cu:6493-6665, 6739-6774, 6842-6863).
//
// The sub-cycling loop runs inside one cooperative launch: every member keeps its own
// remaining time and sub-step on the device (the reference reads minTransportDt back to the
// host once per sub-step).  The minimum admissible sub-step of a member is reduced with an
// integer atomicMin on the bit pattern of non-negative doubles, which is order-independent.
//
// The reference copies every element's tracers into a snapshot before each sub-step and reads
// the neighbours from it.  Here the two tracer arrays alternate instead: sub-step s reads one
// (etr for even s, prev for odd s) and writes the other, so no copy is made; after a member's
// last sub-step its result sits in prev when it took an odd number of sub-steps.  The implicit
// vertical advection runs after every member has finished sub-cycling, reads the result from
// where it sits and writes etr; its Thomas sweep recomputes each row's coefficients and keeps the
// forward-sweep values in etr and the eliminated super-diagonal in prev (both level-major, so a
// warp's accesses are coalesced), instead of per-thread arrays in local memory.  The tracer count
// is a template parameter, so per-tracer values stay in registers.
//
// TVD (itr_met = 3; the reference has only upwind): flux-limited horizontal advection restated
// from Casulli & Zanolli (2005).  On a face between the upwind prism U and the downwind prism D
// the face value is C_U + psi(r)/2 (C_D - C_U), r = S_U / (|Q| (C_U - C_D)), S_U = sum over U's
// interior inflow faces g of |Q_g| (C_g - C_U).  A sub-step is three passes: the inflow sums of
// the snapshot, the admissible sub-step (every update coefficient non-negative:
// dt <= V / sum_in |Q| (1 - psi/2 + sum_out psi/(2r))), and the update
// C_P += dt/V [sum_in |Q| (1 - psi/2)(C_U - C_P) + sum_out |Q| psi/2 (C_P - C_D)].  Limiter 0
// (psi = 0) reproduces the upwind scheme bit for bit.  The vertical solve optionally adds a
// constant diffusivity between prism centres.  This file is compiled with -fmad=false so that
// the limiter's branches see the same rounding as the FP64 CPU restatement.
//
// Vertical FCT (itr_met = 4: the TVD horizontal passes plus a flux-corrected vertical step; no
// counterpart in the reference either): Zalesak's (1979) flux-corrected transport with the
// implicit upwind solve as the low-order scheme.  After the Thomas sweep gives C^L, interior
// interface j of a column carries the anti-diffusive transfer a_j = dt |Qv| (C^L_{j+1} - C^L_j)/2
// (central minus upwind flux), scaled by min(R+ of the receiver, R- of the giver), R+/- =
// min(1, Q+/-/P+/-) from the prism's incoming / outgoing transfers P and its room to the bounds Q
// = V (C_max/min - C^L) over the prism and its column neighbours, of C^L and of the field before
// the vertical step.  The transfers are antisymmetric, so the column's tracer mass is unchanged,
// and no new extremum appears whatever the vertical Courant number.  The field before the step is
// kept in prev (copied there by the forward sweep when the horizontal result sits in etr) and
// the sweep's eliminated super-diagonal goes to its own column scratch.
#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

constexpr double kHuge = 1.79e+308;

struct TrArgs {
    double* rem;                 // [2][nmem] remaining time by parity
    unsigned long long* mindt;   // [2][nmem]
    int32_t* nsub;               // [nmem]
    unsigned* active;            // members still sub-cycling
    double dt;
    int maxsub;
};

__device__ __forceinline__ double evol(const Dev& d, int e, int k) {
    return d.area[e] * (d.ez[(size_t)(k + 1) * d.NE + e] - d.ez[(size_t)k * d.NE + e]);
}

// flux limiter psi(r): 0 none, 1 minmod, 2 Osher (beta = 2), 3 van Leer, 4 superbee; 0 for r <= 0,
// the limit value for r beyond 1e300
__device__ __forceinline__ double tvd_psi(int lim, double r) {
    if (!(r > 0.0)) return 0.0;
    if (!(r < 1.0e300)) return lim == 0 ? 0.0 : (lim == 1 ? 1.0 : 2.0);
    switch (lim) {
    case 1: return fmin(r, 1.0);
    case 2: return fmin(r, 2.0);
    case 3: return (r + r) / (1.0 + r);
    case 4: return fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0));
    default: return 0.0;
    }
}

// psi of a face with upwind value cu, downwind value cd, flux magnitude aq and upwind inflow sum
// su; psir = psi / (2 r) (0 when psi = 0)
__device__ __forceinline__ double tvd_face(int lim, double su, double aq, double cu, double cd, double& psir) {
    const double dd = cu - cd;
    if (dd == 0.0) { psir = 0.0; return 0.0; }
    const double r = su / (aq * dd);
    const double psi = tvd_psi(lim, r);
    psir = (psi > 0.0) ? psi / (2.0 * r) : 0.0;
    return psi;
}

// Minimum of non-negative doubles (compared as their bit patterns) into slot[m] for each lane's
// member m (m < 0: none): a warp whose lanes share one member reduces with shuffles and issues
// one atomic, instead of one per element on the same word.  All 32 lanes must call it.
__device__ __forceinline__ void warp_min_to_member(unsigned long long* slot, int m, double v) {
    const unsigned full = 0xffffffffu;
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    const int m0 = __shfl_sync(full, m, 0);
    if (__all_sync(full, m == m0 || m < 0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(full, b, o);
            b = w < b ? w : b;
        }
        if ((threadIdx.x & 31) == 0 && m0 >= 0) atomicMin(slot + m0, b);
    } else if (m >= 0) {
        atomicMin(slot + m, b);
    }
}

// The three sides of element e as the horizontal update needs them (loaded once per element).
struct ElemSides {
    int s[3], kbs[3], nb[3];
    double sg[3];
    bool nbwet[3];
    int8_t bt[3];
};

__device__ __forceinline__ ElemSides elem_sides(const Dev& d, int e) {
    ElemSides q;
    const int NE = d.NE, NS = d.NS;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int s = d.es[j * NE + e];
        q.s[j] = s;
        q.kbs[j] = d.kbs[s];
        const int e0 = d.se[s], e1 = d.se[NS + s];
        const int nb = (e0 == e) ? e1 : e0;
        q.nb[j] = nb;
        q.nbwet[j] = nb >= 0 && !d.edry[nb];
        q.sg[j] = (double)d.ssgn[j * NE + e];
        q.bt[j] = d.sbt[s];
    }
    return q;
}

// Flux-corrected vertical step of element e's column (FCT above): dst holds C^L and co the field
// before the vertical step; streamed from the bed up with a window of three prisms, each prism's
// corrected value written two levels behind the read.  The expression order is the CPU
// restatement's.
template <int NTR>
__device__ void vertical_fct(const Dev& d, const Phys& P, int e, double dt, const double* co_all, double* dst) {
    const int NE = d.NE, nvrt = P.nvrt;
    const size_t trs = (size_t)nvrt * NE;
    const int k0 = d.kbe[e] + 1;
    const int n = nvrt - k0;
    if (n < 2) return;
#pragma unroll 1
    for (int t = 0; t < NTR; t++) {
        const double* co = co_all + t * trs;
        double* cl = dst + t * trs;
        // prisms i-2 (m2) and i-1 (m1); raw transfer of face (i-2, i-1); scaled transfer of face
        // (i-3, i-2); limiter factors of prism i-2
        double cl_m2 = 0.0, cl_m1 = 0.0, co_m2 = 0.0, co_m1 = 0.0, v_m2 = 1.0, v_m1 = 1.0;
        double a_m2 = 0.0, fa_m3 = 0.0, rp_m2 = 1.0, rm_m2 = 1.0;
        for (int i = 0; i <= n + 1; i++) {
            double cl_i = 0.0, co_i = 0.0, v_i = 1.0, a_m1 = 0.0;
            if (i < n) {
                const size_t ix = (size_t)(k0 + i) * NE + e;
                cl_i = cl[ix]; co_i = co[ix]; v_i = evol(d, e, k0 + i - 1);
                if (i >= 1) a_m1 = 0.5 * dt * fabs(d.Qv[(size_t)(k0 + i - 1) * NE + e]) * (cl_i - cl_m1);
            }
            double rp_m1 = 1.0, rm_m1 = 1.0, fa_m2 = 0.0;
            if (i >= 1 && i <= n) {
                // limiter factors of prism i-1: transfers a_m2 (below) and a_m1 (above)
                double cmax = fmax(cl_m1, co_m1), cmin = fmin(cl_m1, co_m1);
                if (i >= 2) { cmax = fmax(cmax, fmax(cl_m2, co_m2)); cmin = fmin(cmin, fmin(cl_m2, co_m2)); }
                if (i < n) { cmax = fmax(cmax, fmax(cl_i, co_i)); cmin = fmin(cmin, fmin(cl_i, co_i)); }
                const double pp = fmax(0.0, a_m2) + fmax(0.0, -a_m1);
                const double pm = fmin(0.0, a_m2) + fmin(0.0, -a_m1);
                const double qp = v_m1 * (cmax - cl_m1), qm = v_m1 * (cmin - cl_m1);
                rp_m1 = pp > 0.0 ? fmin(1.0, qp / pp) : 1.0;
                rm_m1 = pm < 0.0 ? fmin(1.0, qm / pm) : 1.0;
                if (i >= 2) fa_m2 = a_m2 * (a_m2 > 0.0 ? fmin(rp_m1, rm_m2) : fmin(rm_m1, rp_m2));
            }
            if (i >= 2) cl[(size_t)(k0 + i - 2) * NE + e] = cl_m2 + (fa_m3 - fa_m2) / v_m2;
            fa_m3 = fa_m2; a_m2 = a_m1; rp_m2 = rp_m1; rm_m2 = rm_m1;
            cl_m2 = cl_m1; co_m2 = co_m1; v_m2 = v_m1;
            cl_m1 = cl_i; co_m1 = co_i; v_m1 = v_i;
        }
    }
}

// verticalAdvectionUpdate, meshdata.cu:6611-6665 (upwind: phi = 0) for the NTR tracers of
// element e: reads the column from src, writes it to dst (src may equal dst), uses scr (one
// level-major slice) for the eliminated super-diagonal.  Same arithmetic as the reference's
// tridag_sch<1> (meshdata.cu:3664-3716) row by row; with FCT, scr is the column scratch and the
// flux correction follows.
template <int NTR, bool FCT>
__device__ void vertical_upwind(const Dev& d, const Phys& P, int e, double dt, const double* src, double* dst,
                                double* scr) {
    const int NE = d.NE, nvrt = P.nvrt;
    const size_t trs = (size_t)nvrt * NE;
    const int kb = d.kbe[e];
    const int k0 = kb + 1;
    if (k0 >= nvrt) return;          // a wet element has at least one layer
    double bet = 0.0, cprev = 0.0;
    double up[NTR];
    for (int k = k0; k < nvrt; k++) {
        double alow = 0.0, cupp = 0.0, bdia = 0.0;
        const double dbv = dt / evol(d, e, k - 1);
        bdia += 1.0;
        const double qk = d.Qv[(size_t)k * NE + e], qm = d.Qv[(size_t)(k - 1) * NE + e];
        if (k != nvrt - 1 && qk < 0.0) { const double tmp = dbv * fabs(qk); cupp -= tmp; bdia += tmp; }
        if (k - 1 != kb && qm > 0.0) { const double tmp = dbv * fabs(qm); alow -= tmp; bdia += tmp; }
        if (P.dfh0 > 0.0) {
            // diffusion across the interfaces with the prisms above and below, over the distance
            // between prism centres
            const double ar = d.area[e];
            if (k != nvrt - 1) {
                const double zp = d.ez[(size_t)(k + 1) * NE + e], zm = d.ez[(size_t)(k - 1) * NE + e];
                const double tmp = dbv * (P.dfh0 * ar / (0.5 * (zp - zm)));
                cupp -= tmp; bdia += tmp;
            }
            if (k - 1 != kb) {
                const double zp = d.ez[(size_t)k * NE + e], zm = d.ez[(size_t)(k - 2) * NE + e];
                const double tmp = dbv * (P.dfh0 * ar / (0.5 * (zp - zm)));
                alow -= tmp; bdia += tmp;
            }
        }
        const size_t ix = (size_t)k * NE + e;
        if (k == k0) {
            bet = bdia;
#pragma unroll
            for (int t = 0; t < NTR; t++) {
                const double c = src[t * trs + ix];
                if (FCT && src == dst) d.prev[t * trs + ix] = c;   // keep the field before the step
                up[t] = (c * 1.0) / bet;
                dst[t * trs + ix] = up[t];
            }
        } else {
            const double gam = cprev / bet;
            bet = bdia - alow * gam;
#pragma unroll
            for (int t = 0; t < NTR; t++) {
                const double c = src[t * trs + ix];
                if (FCT && src == dst) d.prev[t * trs + ix] = c;
                up[t] = (c * 1.0 - alow * up[t]) / bet;
                dst[t * trs + ix] = up[t];
            }
            scr[ix] = gam;           // after the reads: scr may be src's first tracer slice
        }
        cprev = cupp;
    }
    // back substitution: u_j -= gam_{j+1} u_{j+1}; up holds the top level's value
    for (int k = nvrt - 2; k >= k0; k--) {
        const double gam = scr[(size_t)(k + 1) * NE + e];
        const size_t ix = (size_t)k * NE + e;
#pragma unroll
        for (int t = 0; t < NTR; t++) {
            up[t] = dst[t * trs + ix] - gam * up[t];
            dst[t * trs + ix] = up[t];
        }
    }
    if (FCT) {
        vertical_fct<NTR>(d, P, e, dt, d.prev, dst);
#pragma unroll
        for (int t = 0; t < NTR; t++) up[t] = dst[t * trs + (size_t)k0 * NE + e];
    }
    // levels at and below the bed take the bottom prism's value
    for (int k = 0; k <= kb; k++)
#pragma unroll
        for (int t = 0; t < NTR; t++) dst[t * trs + (size_t)k * NE + e] = up[t];
}

template <int NTR, bool TVD, bool FCT>
__global__ void __launch_bounds__(256) k_transport(Dev d, Phys P, TrArgs T) {
    const int NE = d.NE, NS = d.NS, nvrt = P.nvrt, nmem = d.nmem;
    const size_t trs = (size_t)nvrt * NE;
    const int G = gridDim.x * blockDim.x;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;   // blockDim is a multiple of 32: warps start at gid - lane
    const unsigned long long seed = (unsigned long long)__double_as_longlong(1e34);
    for (int m = gid; m < nmem; m += G) {
        T.rem[m] = T.dt; T.rem[nmem + m] = T.dt;
        T.mindt[m] = seed; T.mindt[nmem + m] = seed;
        T.nsub[m] = 0;
    }
    if (gid == 0) *T.active = (unsigned)nmem;
    if (!grid_sync(d.bar, d.err, d.wait_polls)) return;
    for (int sub = 0; sub < T.maxsub; sub++) {
        if (*((volatile unsigned*)T.active) == 0u) break;
        const int par = sub & 1, nxt = par ^ 1;
        const double* src = par ? d.prev : d.etr;     // the sub-step's snapshot
        double* dst = par ? d.etr : d.prev;
        if (TVD) {
            const int lim = P.tvd_limiter;
            // TVD pass 1: inflow sums of the snapshot (interior inflow faces, side order)
            for (int e = gid; e < NE; e += G) {
                const int m = d.elem_member[e];
                if (!(((volatile double*)T.rem)[par * nmem + m] > 0.0) || d.edry[e]) continue;
                const ElemSides q = elem_sides(d, e);
                for (int k = d.kbe[e] + 1; k < nvrt; k++) {
                    const size_t ix = (size_t)k * NE + e;
                    double own[NTR], su[NTR];
#pragma unroll
                    for (int t = 0; t < NTR; t++) { own[t] = src[t * trs + ix]; su[t] = 0.0; }
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        if (k <= q.kbs[j] || !q.nbwet[j]) continue;
                        const double fq = d.Qh[(size_t)k * NS + q.s[j]];
                        if (q.sg[j] * fq < 0.0) {
                            const size_t nx = (size_t)k * NE + q.nb[j];
#pragma unroll
                            for (int t = 0; t < NTR; t++) su[t] += fabs(fq) * (src[t * trs + nx] - own[t]);
                        }
                    }
#pragma unroll
                    for (int t = 0; t < NTR; t++) d.tvds[t * trs + ix] = su[t];
                }
            }
            if (!grid_sync(d.bar, d.err, d.wait_polls)) return;
            // TVD pass 2: admissible sub-step per element (warp-uniform loop: the warp reduces
            // its minimum before the member's atomic)
            for (int eb = gid - lane; eb < NE; eb += G) {
                const int e = eb + lane;
                int mm = -1;
                double md = kHuge;
                if (e < NE) mm = d.elem_member[e];
                if (e < NE && ((volatile double*)T.rem)[par * nmem + mm] > 0.0 && !d.edry[e]) {
                    const ElemSides q = elem_sides(d, e);
                    for (int k = d.kbe[e] + 1; k < nvrt; k++) {
                        const size_t ix = (size_t)k * NE + e;
                        const double vol = evol(d, e, k - 1);
                        double own[NTR], so[NTR], den[NTR];
#pragma unroll
                        for (int t = 0; t < NTR; t++) { own[t] = src[t * trs + ix]; so[t] = 0.0; den[t] = 0.0; }
#pragma unroll
                        for (int j = 0; j < 3; j++) {
                            if (k <= q.kbs[j] || !q.nbwet[j]) continue;
                            const double fq = d.Qh[(size_t)k * NS + q.s[j]];
                            if (q.sg[j] * fq > 0.0) {
                                const size_t nx = (size_t)k * NE + q.nb[j];
#pragma unroll
                                for (int t = 0; t < NTR; t++) {
                                    double psir;
                                    tvd_face(lim, d.tvds[t * trs + ix], fabs(fq), own[t], src[t * trs + nx], psir);
                                    so[t] += psir;
                                }
                            }
                        }
#pragma unroll
                        for (int j = 0; j < 3; j++) {
                            if (k <= q.kbs[j] || !q.nbwet[j]) continue;
                            const double fq = d.Qh[(size_t)k * NS + q.s[j]];
                            if (q.sg[j] * fq < 0.0) {
                                const size_t nx = (size_t)k * NE + q.nb[j];
#pragma unroll
                                for (int t = 0; t < NTR; t++) {
                                    double psir;
                                    const double psi = tvd_face(lim, d.tvds[t * trs + nx], fabs(fq), src[t * trs + nx], own[t], psir);
                                    den[t] += fabs(fq) * (1.0 - 0.5 * psi + so[t]);
                                }
                            }
                        }
#pragma unroll
                        for (int t = 0; t < NTR; t++) {
                            const double pd = (den[t] == 0.0) ? kHuge : vol / den[t] * (1.0 - 1.0e-6);
                            md = fmin(md, pd);
                        }
                    }
                    d.maxDt[e] = md;
                }
                warp_min_to_member(T.mindt + par * nmem, mm, md);
            }
        } else
        // horizontalAdvectionPrepare (meshdata.cu:6493-6559): inflow and max sub-step per element
        // (warp-uniform loop: the warp reduces its minimum before the member's atomic)
        for (int eb = gid - lane; eb < NE; eb += G) {
            const int e = eb + lane;
            int mm = -1;
            double md = kHuge;
            if (e < NE) mm = d.elem_member[e];
            if (e < NE && ((volatile double*)T.rem)[par * nmem + mm] > 0.0 && !d.edry[e]) {
                const int kb = d.kbe[e];
                const ElemSides q = elem_sides(d, e);
                for (int k = kb + 1; k < nvrt; k++) {
                    double in = 0.0;
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        if (k <= q.kbs[j]) continue;
                        if (!q.nbwet[j]) continue;
                        const double fq = d.Qh[(size_t)k * NS + q.s[j]];
                        const bool influx = (q.sg[j] * fq) < 0.0;
                        if (q.bt[j] == 1 || !influx) continue;
                        in += fabs(fq);
                    }
                    const double pd = (in == 0.0) ? kHuge : evol(d, e, k - 1) / in * (1.0 - 1.0e-6);
                    md = fmin(md, pd);
                }
                d.maxDt[e] = md;
            }
            warp_min_to_member(T.mindt + par * nmem, mm, md);
        }
        if (!grid_sync(d.bar, d.err, d.wait_polls)) return;
        // horizontalAdvectionUpdate (meshdata.cu:6561-6609) with dtb = min(remaining, min maxDt)
        for (int e = gid; e < NE; e += G) {
            const int m = d.elem_member[e];
            const double rem = ((volatile double*)T.rem)[par * nmem + m];
            if (!(rem > 0.0)) {
                // a finished member stays finished: carry its remaining time into the next
                // parity slot, which otherwise still holds its value from before its last
                // sub-step and would make it run (and leave the count of active members) again
                if (e == d.mem_ne0[m]) T.rem[nxt * nmem + m] = rem;
                continue;
            }
            const double mdt = __longlong_as_double((long long)((volatile unsigned long long*)T.mindt)[par * nmem + m]);
            const double dtb = fmin(rem, mdt);
            const bool last = !((rem - dtb) > 0.0);
            if (e == d.mem_ne0[m]) {                       // member bookkeeping, once per member
                T.rem[nxt * nmem + m] = rem - dtb;
                T.mindt[nxt * nmem + m] = seed;
                T.nsub[m] = sub + 1;
                if (last) atomicSub(T.active, 1u);
            }
            if (d.edry[e]) continue;
            const int kb = d.kbe[e];
            const ElemSides q = elem_sides(d, e);
            for (int k = kb + 1; k < nvrt; k++) {
                const size_t ix = (size_t)k * NE + e;
                const double vol = evol(d, e, k - 1);
                const double dbv = dtb / vol;
                double own[NTR], adv[NTR];
#pragma unroll
                for (int t = 0; t < NTR; t++) { own[t] = src[t * trs + ix]; adv[t] = own[t]; }
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    if (k <= q.kbs[j]) continue;
                    const double fq = d.Qh[(size_t)k * NS + q.s[j]];
                    const double sQ = q.sg[j] * fq;
                    if (TVD) {
                        const int lim = P.tvd_limiter;
                        const double coef = dbv * fabs(fq);
                        const size_t nx = (size_t)k * NE + q.nb[j];
                        if (sQ < 0.0) {
                            if (q.nbwet[j]) {
#pragma unroll
                                for (int t = 0; t < NTR; t++) {
                                    const double cu = src[t * trs + nx];
                                    double psir;
                                    const double psi = tvd_face(lim, d.tvds[t * trs + nx], fabs(fq), cu, own[t], psir);
                                    adv[t] += coef * (1.0 - 0.5 * psi) * (cu - own[t]);
                                }
                            } else if (q.bt[j] == 2) {
#pragma unroll
                                for (int t = 0; t < NTR; t++) adv[t] += coef * (adv[t] - own[t]);
                            }
                        } else if (sQ > 0.0 && q.nbwet[j]) {
#pragma unroll
                            for (int t = 0; t < NTR; t++) {
                                const double cd = src[t * trs + nx];
                                double psir;
                                const double psi = tvd_face(lim, d.tvds[t * trs + ix], fabs(fq), own[t], cd, psir);
                                adv[t] += coef * (0.5 * psi) * (own[t] - cd);
                            }
                        }
                        continue;
                    }
                    if (sQ >= 0.0) continue;
                    const double coef = dbv * fabs(fq);
                    if (q.nbwet[j]) {
                        const size_t nx = (size_t)k * NE + q.nb[j];
#pragma unroll
                        for (int t = 0; t < NTR; t++) adv[t] += coef * (src[t * trs + nx] - own[t]);
                    } else if (q.bt[j] == 2) {
#pragma unroll
                        for (int t = 0; t < NTR; t++) {
                            const double cout = adv[t];
                            adv[t] += coef * (cout - own[t]);
                        }
                    }
                }
#pragma unroll
                for (int t = 0; t < NTR; t++) dst[t * trs + ix] = adv[t];
            }
#pragma unroll
            for (int t = 0; t < NTR; t++) {
                const double v = dst[t * trs + (size_t)(kb + 1) * NE + e];
                for (int k = 0; k <= kb; k++) dst[t * trs + (size_t)k * NE + e] = v;
            }
        }
        if (!grid_sync(d.bar, d.err, d.wait_polls)) return;
    }
    // verticalAdvectionUpdate for every wet element, once its member has finished sub-cycling:
    // after n sub-steps the horizontal result is in prev when n is odd, in etr when it is even
    for (int e = gid; e < NE; e += G) {
        if (d.edry[e]) continue;
        const int m = d.elem_member[e];
        const double* res = (T.nsub[m] & 1) ? d.prev : d.etr;
        vertical_upwind<NTR, FCT>(d, P, e, T.dt, res, d.etr, FCT ? d.vgam : d.prev);
    }
}

// Tracer mass budget of one member (elements [e0, e1)): per tracer, the sum over wet prisms of
// volume x concentration in FP64 with Neumaier's compensated summation.  Every thread sums its
// prisms, the block merges its threads in a fixed tree and a final one-thread pass merges the
// blocks in order: the grid is fixed (kMassBlocks), so the result does not depend on the GPU.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
}

__global__ void __launch_bounds__(256) k_tracer_mass(Dev d, int nvrt, int ntr, int e0, int e1, double* part) {
    __shared__ double sh_s[256], sh_c[256];
    const int tid = threadIdx.x, NE = d.NE;
    for (int t = 0; t < ntr; t++) {
        double s = 0.0, c = 0.0;
        for (int e = e0 + blockIdx.x * blockDim.x + tid; e < e1; e += gridDim.x * blockDim.x) {
            if (d.edry[e]) continue;
            for (int k = d.kbe[e] + 1; k < nvrt; k++)
                neumaier_add(s, c, evol(d, e, k - 1) * d.etr[((size_t)t * nvrt + k) * NE + e]);
        }
        sh_s[tid] = s; sh_c[tid] = c;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (tid < w) {
                double a = sh_s[tid], ca = sh_c[tid];
                neumaier_add(a, ca, sh_s[tid + w]);
                sh_s[tid] = a; sh_c[tid] = ca + sh_c[tid + w];
            }
            __syncthreads();
        }
        if (tid == 0) {
            part[((size_t)blockIdx.x * ntr + t) * 2] = sh_s[0];
            part[((size_t)blockIdx.x * ntr + t) * 2 + 1] = sh_c[0];
        }
        __syncthreads();
    }
}

__global__ void k_tracer_mass_final(int nblk, int ntr, const double* part, double* out) {
    const int t = threadIdx.x;
    if (t >= ntr) return;
    double s = 0.0, c = 0.0;
    for (int b = 0; b < nblk; b++) {
        neumaier_add(s, c, part[((size_t)b * ntr + t) * 2]);
        c += part[((size_t)b * ntr + t) * 2 + 1];
    }
    out[t] = s + c;
}

cudaError_t launch_tracer_mass(const Dev& d, const Phys& P, int e0, int e1, double* part, double* out,
                               cudaStream_t st) {
    k_tracer_mass<<<kMassBlocks, 256, 0, st>>>(d, P.nvrt, P.ntr, e0, e1, part);
    k_tracer_mass_final<<<1, 32, 0, st>>>(kMassBlocks, P.ntr, part, out);
    return cudaGetLastError();
}

template <int NTR>
__global__ void k_nodal_tracer(Dev d, Phys P) {
    // nodalTracerUpdate, meshdata.cu:6739-6774 (node-centred gather, no atomics).  One thread per
    // (node, level), the level in blockIdx.y; each (node, level) sums its elements in the same
    // order as a node-by-node loop.
    const int NP = d.NP, NE = d.NE, nvrt = P.nvrt, ivrt = nvrt - 1, k = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        if (d.ndry[i]) continue;
        const int q0 = d.nne_s[i], q1 = d.nne_s[i + 1];
        double sum[NTR];
#pragma unroll
        for (int t = 0; t < NTR; t++) sum[t] = 0.0;
        double sumA = 0.0;
        for (int q = q0; q < q1; q++) {
            const int e = d.nne[q];
            if (d.edry[e]) continue;
            const int kb = d.kbe[e];
            const int kin = k > kb ? k : kb;
            int kLo = kin, kHi = kin + 1;
            double zrat = 0.0;
            if (kin == ivrt) { kLo = ivrt; kHi = ivrt; }
            else if (kin == kb) { kLo = kb + 1; kHi = kb + 1; }
            else {
                const double zp = d.ez[(size_t)(kin + 1) * NE + e], zc = d.ez[(size_t)kin * NE + e],
                             zm = d.ez[(size_t)(kin - 1) * NE + e];
                zrat = (zp - zc) / (zp - zm);
            }
            const double A = d.area[e];
#pragma unroll
            for (int t = 0; t < NTR; t++) {
                const double* tr = d.etr + (size_t)t * nvrt * NE;
                sum[t] += A * ((1.0 - zrat) * tr[(size_t)kHi * NE + e] + zrat * tr[(size_t)kLo * NE + e]);
            }
            sumA += A;
        }
        if (sumA == 0.0) continue;
        const double inv = 1.0 / sumA;
#pragma unroll
        for (int t = 0; t < NTR; t++) d.tr[((size_t)t * nvrt + k) * NP + i] = inv * sum[t];
    }
}

template <int NTR>
static cudaError_t launch_ntr(const Dev& d, const Phys& P, TrArgs& T, cudaStream_t st, int nsm, const LaunchShape& nt) {
    // the TVD passes live in their own instantiation, so the upwind one keeps its smaller
    // register budget and its occupancy
    const void* fn = P.tvd_vert ? (const void*)k_transport<NTR, true, true>
                     : P.tvd    ? (const void*)k_transport<NTR, true, false>
                                : (const void*)k_transport<NTR, false, false>;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0);
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    int grid = std::min(nsm * per_sm, (d.NE + 255) / 256);
    if (grid < 1) grid = 1;
    Dev dd = d;
    Phys pp = P;
    void* args[] = {&dd, &pp, &T};
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, 0, st);
    if (e != cudaSuccess) return e;
    k_nodal_tracer<NTR><<<dim3(grid_of(d.NP, nt, nsm), P.nvrt), nt.block, 0, st>>>(d, P);
    return cudaGetLastError();
}

template <int NTR>
static int nodal_tracer_max_threads() {
    cudaFuncAttributes a{};
    return cudaFuncGetAttributes(&a, k_nodal_tracer<NTR>) == cudaSuccess ? a.maxThreadsPerBlock : 0;
}

int transport_max_threads(int ntr) {
    switch (ntr) {
    case 1: return nodal_tracer_max_threads<1>();
    case 2: return nodal_tracer_max_threads<2>();
    case 3: return nodal_tracer_max_threads<3>();
    case 4: return nodal_tracer_max_threads<4>();
    case 5: return nodal_tracer_max_threads<5>();
    case 6: return nodal_tracer_max_threads<6>();
    case 7: return nodal_tracer_max_threads<7>();
    default: return nodal_tracer_max_threads<8>();
    }
}

cudaError_t launch_transport(const Dev& d, const Phys& P, double dt, cudaStream_t st, int nsm, const LaunchTable& L) {
    if (P.ntr <= 0) return cudaSuccess;
    TrArgs T;
    T.rem = d.mem_rem; T.mindt = d.mem_mindt; T.nsub = d.mem_nsub; T.active = (unsigned*)(d.mem_mindt + 2 * d.nmem);
    T.dt = dt; T.maxsub = 100000;
    static_assert(kMaxTracers == 8, "one instantiation per tracer count");
    switch (P.ntr) {
    case 1: return launch_ntr<1>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 2: return launch_ntr<2>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 3: return launch_ntr<3>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 4: return launch_ntr<4>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 5: return launch_ntr<5>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 6: return launch_ntr<6>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    case 7: return launch_ntr<7>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    default: return launch_ntr<8>(d, P, T, st, nsm, L.k[LK_NODAL_TRACER]);
    }
}

}  // namespace gs
