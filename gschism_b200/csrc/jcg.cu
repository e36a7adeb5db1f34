// Jacobi-preconditioned CG for the elevation system, one persistent cooperative launch per
// solve for every member of a batch (replaces PCGSolverMultiGPU.solve / NativePCG,
// src/solver/pcg_solver.py:1075-1124 and src/solver/pcg_loop.cpp:334-416).
//
// Work decomposition.  A member's rows are cut into tiles whose size depends only on that
// member's row count, and every block owns a contiguous run of tiles.  A phase writes one
// partial per tile (fixed block tree); after the grid barrier each block forms the member totals
// it needs by summing that member's tile partials in tile order.  Every reduction is therefore
// deterministic and independent of the batch composition and of the grid size: a member gives
// bit-identical results alone and inside any batch.  Scalars stay on the device; convergence is
// tested every check_every iterations on the device, so a solve never returns to the host.
//
// GS_FP64: per iteration two phases separated by grid barriers:
//   A: beta = rz/rz_old; p_new = z + beta p; q = A p_new (p_new of neighbour rows is formed on
//      the fly from z and the previous p, so no barrier is needed between p and q); p.q partials
//   B: alpha = rz/p.q; x += alpha p; r -= alpha q; z = invD r; r.r and r.z partials.
// GS_FP32_IR solves the residual equation A d = r in FP32 (FP32 matrix and vectors, FP64 dot
// products) inside FP64 refinement sweeps r = b - A x, x += d, with the single-reduction form of
// the iteration (one barrier per iteration; see k_jcg_ir).
#include <algorithm>
#include <mutex>

#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

constexpr int kThreads = 256;

enum { R_BB = 0, R_PQ = 1, R_RR0 = 2, R_RZ0 = 3, R_RR1 = 4, R_RZ1 = 5, R_OUT = 6, R_WU0 = 7, R_WU1 = 8, R_KINDS = 9 };

struct JcgView {
    int n, nmem, ntiles;
    const int32_t *indptr, *indices;   // CSR rows (indptr), or SELL-32 slices when sell is set
    const int2* sell;
    const double* A;
    const float* A32;              // D^-1 A in FP32 (refinement solve)
    const double* b;
    const double* invD;
    double *x, *r, *z, *q, *p0, *p1;
    float* ir32;                   // kIrVectors FP32 vectors of the refinement solve
    const float* diag32;           // D in FP32
    const int32_t *tile_r0, *tile_r1, *tile_mem, *mem_t0, *mem_t1, *blk_t0;   // blk_t0: [grid+1]
    double* tile_part;             // [R_KINDS][ntiles]
    double* mem_atol2;             // [nmem]
    int32_t* mdone;                // [nmem] iterations at convergence, -1 while active
    int32_t* mouter;               // [nmem] refinement sweeps (IR)
    int32_t* minner;               // [nmem] inner iterations so far (IR)
    int32_t* mret;                 // [nmem] inner iteration at which the sweep's solve finished, -1 before
    double* mem_ab;                // [9][nmem] inner solve: alpha (parity 0, 1), gamma (parity 0, 1),
                                   // [4..6) published (alpha, beta) pairs, [6] alpha, [7] gamma and
                                   // [8] recursive r.r of the previous sweep's last iteration
    double* mpub;                  // [nmem][2] published (alpha, beta) of the member's current inner iteration
    int32_t* mgen;                 // [nmem] inner iteration whose scalars are published (kRetired: finished)
    unsigned* mcnt;                // [nmem] block arrivals of the inner solve
    const int32_t* mnblk;          // [nmem] blocks of the refinement grid that hold tiles of the member
    unsigned* ndone;
    unsigned* bar;
    int32_t* err;                  // ERR_BARRIER_TIMEOUT (shared with the context's other launches)
    int32_t* status;               // ERR_JCG_NOT_CONVERGED of this solve (zeroed at every launch)
    long long wait_polls;          // bound of every wait
    int stall_member;              // recovery tests: one more arrival expected for this member (-1: none)
    double rtol;
    int maxiter, check_every;
    double inner_rtol;
    int inner_maxiter;
};

// Fixed-order block sum of NV values; every thread returns the totals.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double s = v[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k * 32 + w] = s;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double s = (lane < (kThreads >> 5)) ? sh[k * 32 + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        v[k] = s;
    }
    __syncthreads();
}

template <int NV>
__device__ __forceinline__ void put_partials(const JcgView& J, int t, const int (&kinds)[NV], double (&v)[NV],
                                             double* sh) {
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) J.tile_part[(size_t)kinds[k] * J.ntiles + t] = v[k];
    }
}

// Member totals of NV kinds: the member's tile partials summed in tile order (fixed tree).
template <int NV>
__device__ __forceinline__ void member_totals(const JcgView& J, int m, const int (&kinds)[NV], double (&out)[NV],
                                              double* sh) {
    const int t0 = J.mem_t0[m], t1 = J.mem_t1[m];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double s = 0.0;
        const volatile double* tp = J.tile_part + (size_t)kinds[k] * J.ntiles;
        for (int t = t0 + threadIdx.x; t < t1; t += kThreads) s += tp[t];
        out[k] = s;
    }
    block_sum<NV>(out, sh);
}

// The same totals, bit for bit, with a thread's loads of a chunk (up to four tiles per kind, L2
// reads) issued before it adds them in tile order: one L2 round trip per chunk instead of one per
// tile.  Used by the FP64 solve (8% faster on a 1M-row system); in the FP32 solve the larger
// register footprint cost more than it saved on the 64-member ensemble.
template <int NV>
__device__ __forceinline__ void member_totals_wide(const JcgView& J, int m, const int (&kinds)[NV],
                                                   double (&out)[NV], double* sh) {
    constexpr int kChunk = 4;
    const int t0 = J.mem_t0[m], t1 = J.mem_t1[m];
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = 0.0;
    for (int base = t0 + threadIdx.x; base < t1; base += kChunk * kThreads) {
        double v[NV][kChunk];
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double* tp = J.tile_part + (size_t)kinds[k] * J.ntiles;
#pragma unroll
            for (int j = 0; j < kChunk; j++) {
                const int t = base + j * kThreads;
                v[k][j] = t < t1 ? __ldcg(tp + t) : 0.0;
            }
        }
#pragma unroll
        for (int k = 0; k < NV; k++)
#pragma unroll
            for (int j = 0; j < kChunk; j++)
                if (base + j * kThreads < t1) out[k] += v[k][j];
    }
    block_sum<NV>(out, sh);
}

__device__ __forceinline__ int ld_done(const JcgView& J, int m) { return *((volatile int32_t*)&J.mdone[m]); }

// generation word of a finished member (mgen), in both solves
constexpr int kGenRetired = 0x7fffffff;

// Block-uniform read of a word another block may update in the same phase: thread 0 reads,
// the block agrees on that value (either value leads every block to the same decision).
__device__ __forceinline__ int uniform_ld(const int32_t* p, int* shv) {
    __syncthreads();
    if (threadIdx.x == 0) *shv = *((const volatile int32_t*)p);
    __syncthreads();
    return *shv;
}

// Entries of row i: positions off + k * stride for k < n, in increasing column order.
struct RowRange { int off, n, stride; };

template <bool SELL>
__device__ __forceinline__ RowRange row_range(const JcgView& J, int i) {
    if constexpr (SELL) {
        const int2 sw = __ldg(J.sell + (i >> 5));
        return {sw.x + (i & 31), sw.y, 32};
    } else {
        const int a0 = __ldg(J.indptr + i), a1 = __ldg(J.indptr + i + 1);
        return {a0, a1 - a0, 1};
    }
}

// Row product sum_k vals[e_k] * g(indices[e_k]) over the row's entries e_k, in entry order.
// Entries are fetched eight at a time and all index and value loads of a chunk are issued before
// its gathers, so a row of up to eight entries costs about two memory latencies rather than two
// per entry.  Slots past the row's end gather the row itself with a zero weight, which leaves the
// sum unchanged.  In SELL-32 layout the loads of one slot are contiguous across a warp.
template <bool SELL, typename T, typename G>
__device__ __forceinline__ T row_dot(const JcgView& J, const T* __restrict__ vals, int i, G g) {
    const RowRange rr = row_range<SELL>(J, i);
    T s = (T)0;
    for (int base = 0; base < rr.n; base += 8) {
        int c[8];
        T v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const bool ok = base + k < rr.n;
            const int e = rr.off + (base + k) * rr.stride;
            c[k] = ok ? __ldg(J.indices + e) : i;
            v[k] = ok ? __ldg(vals + e) : (T)0;
        }
        T gv[8];
#pragma unroll
        for (int k = 0; k < 8; k++) gv[k] = g(c[k]);
#pragma unroll
        for (int k = 0; k < 8; k++) s += v[k] * gv[k];
    }
    return s;
}

__device__ __forceinline__ bool checkpoint(const JcgView& J, int it, int maxit) {
    return ((it + 1) % J.check_every == 0) || (it == maxit - 1);
}

// |b|^2 partials (and zero the search directions of both precisions)
__device__ void phase_bb(const JcgView& J, double* sh) {
    const int tb0 = J.blk_t0[blockIdx.x], tb1 = J.blk_t0[blockIdx.x + 1];
    for (int t = tb0; t < tb1; t++) {
        const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
        double v[1] = {0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += kThreads) {
            const double bi = J.b[i];
            v[0] += bi * bi;
            J.p0[i] = 0.0; J.p1[i] = 0.0;
        }
        const int kinds[1] = {R_BB};
        put_partials<1>(J, t, kinds, v, sh);
    }
}

// atol^2 per member (owner = block holding the member's first tile); atol = 0 retires it
__device__ void phase_atol(const JcgView& J, double* sh) {
    const int tb0 = J.blk_t0[blockIdx.x], tb1 = J.blk_t0[blockIdx.x + 1];
    for (int t = tb0; t < tb1; t++) {
        const int m = J.tile_mem[t];
        if (t != J.mem_t0[m]) continue;
        const int kinds[1] = {R_BB};
        double tot[1];
        member_totals<1>(J, m, kinds, tot, sh);
        if (threadIdx.x == 0) {
            const double atol = J.rtol * sqrt(tot[0]);
            J.mem_atol2[m] = atol * atol;
            // a zero right-hand side: the member is done before the first iteration, and its
            // generation word says so to every block that holds its tiles
            if (atol == 0.0) { J.mdone[m] = 0; J.mgen[m] = kGenRetired; __threadfence(); atomicAdd(J.ndone, 1u); }
        }
    }
}

#define GSYNC() do { if (!grid_sync(J.bar, J.err, J.wait_polls)) return; } while (0)

// Arrivals that complete member m's count: its blocks, plus one that never comes when the
// recovery test stalls the member (its waits then run out and the solve reports a timeout).
__device__ __forceinline__ unsigned arrivals(const JcgView& J, int m) {
    return (unsigned)J.mnblk[m] + (m == J.stall_member ? 1u : 0u);
}

// ------------------------------------------------------------------------------- FP64 ----
//
// The reference's two-phase iteration with member-level synchronisation instead of grid
// barriers (as the FP32 solve, below): after its tiles of member m a block adds one to mcnt[m];
// the member's last arriver sums the member's partials in tile order and publishes the scalar
// the next phase needs in mpub[2m] (alpha) or mpub[2m+1] (beta), with mgen[m] = 2 it + 2 (alpha of
// iteration it) or 2 it + 3 (beta of iteration it + 1); mgen = 0 means nothing published yet and
// kRetired a finished member.  The totals, and so alpha, beta, the iterates and the iteration
// counts, are those of the grid-barrier form bit for bit.

constexpr int kRetired64 = kGenRetired;

__device__ __forceinline__ int ld_acquire_s32(const int32_t* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Wait until member m has published generation g.  Returns the published scalar in *val and
// 1 = on, 0 = finished, -1 = failed (bounded) wait.
__device__ __forceinline__ int wait64(const JcgView& J, int m, int g, int slot, double* shd, int* shv) {
    __syncthreads();
    if (threadIdx.x == 0) {
        long long spins = 0;
        int cur, st = 1;
        while ((cur = ld_acquire_s32(&J.mgen[m])) < g) {
            if (++spins > 4096) __nanosleep(128);
            if (spins > J.wait_polls) { atomicOr(J.err, ERR_BARRIER_TIMEOUT); st = -1; break; }
            if ((spins & 255) == 0 && (*((volatile int32_t*)J.err) & ERR_BARRIER_TIMEOUT)) { st = -1; break; }
        }
        __threadfence();
        if (st == 1 && cur == kRetired64) st = 0;
        if (st == 1) *shd = __ldcg(&J.mpub[2 * m + slot]);
        *shv = st;
    }
    __syncthreads();
    return *shv;
}

__device__ __forceinline__ void publish64(const JcgView& J, int m, int g, int slot, double val) {
    J.mpub[2 * m + slot] = val;
    __threadfence();
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(&J.mgen[m]), "r"(g) : "memory");
}

// Arrival of this block at member m; returns true in the whole block for the last arriver.
__device__ __forceinline__ bool arrive64(const JcgView& J, int m, int* shv) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned old = atomicAdd(&J.mcnt[m], 1u);
        const bool last = ((old + 1u) % arrivals(J, m)) == 0u;
        if (last) __threadfence();
        *shv = last ? 1 : 0;
    }
    __syncthreads();
    return *shv != 0;
}

// Scalars of phase A of iteration nit (nit >= 1) from the partials of iteration nit - 1's phase B,
// published by the member's last arriver: the checkpoint test, then beta.
__device__ void publish_beta(const JcgView& J, int m, int nit, double* sh) {
    const int cur = (nit + 1) & 1, old = nit & 1;
    const int kinds[3] = {cur ? R_RR1 : R_RR0, cur ? R_RZ1 : R_RZ0, old ? R_RZ1 : R_RZ0};
    double tot[3];
    member_totals_wide<3>(J, m, kinds, tot, sh);
    if (threadIdx.x != 0) return;
    if (checkpoint(J, nit - 1, J.maxiter) && tot[0] <= J.mem_atol2[m]) {
        J.mdone[m] = nit;
        __threadfence();
        atomicAdd(J.ndone, 1u);
        publish64(J, m, kRetired64, 1, 0.0);
        return;
    }
    if (nit == J.maxiter) {
        // still active after the last iteration: the reference returns maxiter
        J.mdone[m] = J.maxiter;
        atomicOr(J.status, ERR_JCG_NOT_CONVERGED);
        __threadfence();
        atomicAdd(J.ndone, 1u);
        publish64(J, m, kRetired64, 1, 0.0);
        return;
    }
    publish64(J, m, 2 * nit + 1, 1, (tot[2] == 0.0) ? 0.0 : tot[1] / tot[2]);
}

// rows of the FP64 loop (p update and q = A p) unrolled per thread
#ifndef GS_JCG64_ROW_UNROLL
#define GS_JCG64_ROW_UNROLL 1
#endif
constexpr int kRowUnroll64 = GS_JCG64_ROW_UNROLL;

template <bool SELL>
__global__ void __launch_bounds__(kThreads) k_jcg64(JcgView J) {
    __shared__ double sh[4 * 32];
    __shared__ double shd;
    __shared__ int shv;
    const int tid = threadIdx.x;
    const int tb0 = J.blk_t0[blockIdx.x], tb1 = J.blk_t0[blockIdx.x + 1];
    phase_bb(J, sh);
    GSYNC();
    phase_atol(J, sh);
    GSYNC();
    // r = b - A x; z = invD r; (r.r, r.z) into the parity-1 slots (iteration -1); iteration 0 of
    // a member starts with beta = 0 once all its blocks are here
    {
        int cm = -1;
        bool on = false;
        for (int t = tb0; t < tb1; t++) {
            const int m = J.tile_mem[t];
            if (m != cm) {
                if (cm >= 0 && on && arrive64(J, cm, &shv) && tid == 0) publish64(J, cm, 1, 1, 0.0);
                cm = m;
                on = uniform_ld(&J.mdone[m], &shv) < 0;
            }
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            if (!on) {
                for (int i = r0 + tid; i < r1; i += kThreads) { J.x[i] = 0.0; J.r[i] = 0.0; J.z[i] = 0.0; }
                continue;
            }
            double v[2] = {0.0, 0.0};
            for (int i = r0 + tid; i < r1; i += kThreads) {
                const double s = row_dot<SELL, double>(J, J.A, i, [&](int c) { return J.x[c]; });
                const double ri = J.b[i] - s, zi = J.invD[i] * ri;
                J.r[i] = ri; J.z[i] = zi;
                v[0] += ri * ri; v[1] += ri * zi;
            }
            const int kinds[2] = {R_RR1, R_RZ1};
            put_partials<2>(J, t, kinds, v, sh);
        }
        if (cm >= 0 && on && arrive64(J, cm, &shv) && tid == 0) publish64(J, cm, 1, 1, 0.0);
    }
    for (int it = 0; it < J.maxiter; it++) {
        const double* pc = (it & 1) ? J.p1 : J.p0;
        double* pn = (it & 1) ? J.p0 : J.p1;
        const int cur = (it + 1) & 1;
        bool any = false;
        // phase A: p_new = z + beta p; q = A p_new; p.q partials; the last arriver publishes alpha
        {
            int cm = -1;
            bool on = false;
            double beta = 0.0;
            for (int t = tb0; t < tb1; t++) {
                const int m = J.tile_mem[t];
                if (m != cm) {
                    if (cm >= 0 && on && arrive64(J, cm, &shv)) {
                        const int kinds[2] = {R_PQ, cur ? R_RZ1 : R_RZ0};
                        double tot[2];
                        member_totals_wide<2>(J, cm, kinds, tot, sh);
                        if (tid == 0) publish64(J, cm, 2 * it + 2, 0, (tot[0] != 0.0) ? tot[1] / tot[0] : 0.0);
                    }
                    cm = m;
                    on = false;
                    // a member with mdone >= 0 (zero right-hand side, or retired) publishes no
                    // more; either value of mdone a block reads leads to the same decision
                    if (uniform_ld(&J.mdone[m], &shv) < 0) {
                        const int st = wait64(J, m, 2 * it + 1, 1, &shd, &shv);
                        if (st < 0) return;
                        on = st == 1;
                        beta = (it == 0) ? 0.0 : shd;
                    }
                }
                if (!on) continue;
                any = true;
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                double v[1] = {0.0};
#pragma unroll kRowUnroll64
                for (int i = r0 + tid; i < r1; i += kThreads) {
                    const double s = row_dot<SELL, double>(J, J.A, i, [&](int c) { return J.z[c] + beta * pc[c]; });
                    const double pi = J.z[i] + beta * pc[i];
                    pn[i] = pi; J.q[i] = s;
                    v[0] += pi * s;
                }
                const int kinds[1] = {R_PQ};
                put_partials<1>(J, t, kinds, v, sh);
            }
            if (cm >= 0 && on && arrive64(J, cm, &shv)) {
                const int kinds[2] = {R_PQ, cur ? R_RZ1 : R_RZ0};
                double tot[2];
                member_totals_wide<2>(J, cm, kinds, tot, sh);
                if (tid == 0) publish64(J, cm, 2 * it + 2, 0, (tot[0] != 0.0) ? tot[1] / tot[0] : 0.0);
            }
        }
        if (!any) break;
        // phase B: x += alpha p; r -= alpha q; z = invD r; (r.r, r.z) partials; the last arriver
        // takes the checkpoint decision and publishes the next beta
        {
            const int srr = (it & 1) ? R_RR1 : R_RR0, srz = (it & 1) ? R_RZ1 : R_RZ0;
            int cm = -1;
            bool on = false;
            double alpha = 0.0;
            for (int t = tb0; t < tb1; t++) {
                const int m = J.tile_mem[t];
                if (m != cm) {
                    if (cm >= 0 && on && arrive64(J, cm, &shv)) publish_beta(J, cm, it + 1, sh);
                    cm = m;
                    on = false;
                    if (uniform_ld(&J.mdone[m], &shv) < 0) {
                        const int st = wait64(J, m, 2 * it + 2, 0, &shd, &shv);
                        if (st < 0) return;
                        on = st == 1;
                        alpha = shd;
                    }
                }
                if (!on) continue;
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                double v[2] = {0.0, 0.0};
                for (int i = r0 + tid; i < r1; i += kThreads) {
                    J.x[i] += alpha * pn[i];
                    const double ri = J.r[i] - alpha * J.q[i];
                    const double zi = J.invD[i] * ri;
                    J.r[i] = ri; J.z[i] = zi;
                    v[0] += ri * ri; v[1] += ri * zi;
                }
                const int kinds[2] = {srr, srz};
                put_partials<2>(J, t, kinds, v, sh);
            }
            if (cm >= 0 && on && arrive64(J, cm, &shv)) publish_beta(J, cm, it + 1, sh);
        }
    }
}

// ---------------------------------------------------------------------- FP32 + refinement ----
//
// Outer FP64 sweeps r = b - A x, x += d around an inner FP32 solve of A d = r.  The inner solve is
// the single-reduction form of Jacobi-PCG (Chronopoulos and Gear, 1989): with u = D^-1 r and
// w = A u the recurrences
//   s_i = w_i + beta_i s_{i-1},   p_i = u_i + beta_i p_{i-1},   d += alpha_i p_i,
//   r_{i+1} = r_i - alpha_i s_i,  w_{i+1} = A u_{i+1},
//   gamma = (r, u), delta = (w, u),  beta_i = gamma_i / gamma_{i-1},
//   alpha_i = gamma_i / (delta_i - beta_i gamma_i / alpha_{i-1})
// give the iterates of the two-reduction loop with one grid-wide reduction per iteration.  The
// vectors are kept scaled by D^-1 (u, w~ = D^-1 w, s~ = D^-1 s) and the FP32 matrix copy holds
// D^-1 A, so u_{i+1} = u_i - alpha_i s~_i and w~_{i+1} = (D^-1 A) u_{i+1}; the dot products use
// the FP32 diagonal D: gamma = sum D u^2, delta = sum D w~ u, r.r = sum (D u)^2.  A row's
// w~_{i+1} needs u_{i+1} of its neighbours; each block forms those on the fly from the neighbours'
// (u_i, w~_i, s~_{i-1}), so u, w~ and s~ are double-buffered by iteration parity and no barrier
// separates the vector update from the matrix product.

// FP32 vectors in ir32: (u, w~, s~, p) packed per row for iteration parities 0 and 1 (4 n floats
// each, so a neighbour's three values arrive in one 16-byte load and a row's own four in one),
// then d.
static_assert(kIrVectors == 9, "ir32 layout");

// rows of the FP32 inner loop in flight per thread, bit for bit the same result whatever the
// count: two for a system whose working set fits in L2 (13% faster than one on a 1M-row system;
// three and four were not faster there), four beyond it (5% faster than two on the 64-member
// ensemble's 9M rows, where DRAM latency has to be covered)
#ifndef GS_JCG_IR_ROW_UNROLL
#define GS_JCG_IR_ROW_UNROLL 2
#endif
#ifndef GS_JCG_IR_ROW_UNROLL_LARGE
#define GS_JCG_IR_ROW_UNROLL_LARGE 4
#endif
constexpr int kRowUnroll = GS_JCG_IR_ROW_UNROLL;
constexpr int kRowUnrollLarge = GS_JCG_IR_ROW_UNROLL_LARGE;
// bytes an FP32 inner iteration touches per row (matrix slots, indices, the row's float4 state,
// d and the diagonal), for the L2 test that picks the row count in flight
constexpr double kIrBytesPerRow = 100.0;

// resident blocks per SM the refinement solve is compiled for (register budget)
#ifndef GS_JCG_IR_MIN_BLOCKS
#define GS_JCG_IR_MIN_BLOCKS 4
#endif
__device__ __forceinline__ float4* ir_uws(const JcgView& J, int parity) {
    return reinterpret_cast<float4*>(J.ir32) + (size_t)parity * J.n;
}
__device__ __forceinline__ float* ir_d(const JcgView& J) { return J.ir32 + (size_t)8 * J.n; }

// u_{i+1} of a row from its (u_i, w~_i, s~_{i-1}); the same expression for a row and its neighbours
__device__ __forceinline__ float u_next(float4 q, float al, float bt) { return q.x - al * (q.y + bt * q.z); }

__device__ __forceinline__ int ld_i32(const int32_t* p) { return *((const volatile int32_t*)p); }

// ---- member-level synchronisation of the inner solve.  Rows of a member only couple to rows of
// the same member, so the inner iterations need no grid-wide barrier: after its tiles of member m
// a block adds one to mcnt[m]; the block whose arrival completes the member's count (mnblk[m]
// blocks hold its tiles) sums the member's tile partials in tile order, takes the convergence
// decision, computes the next (alpha, beta) and publishes them with mgen[m] = next iteration (or
// kRetired).  Blocks wait only for the members they hold.  Every wait is bounded.
constexpr int kRetired = kGenRetired;

__device__ __forceinline__ int ld_acquire_i32(const int32_t* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i32(int32_t* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until member m has published inner iteration it.  pub receives (alpha, beta, state) with
// state 1 = on, 0 = finished, -1 = failed wait (the caller leaves the kernel).
__device__ __forceinline__ void member_wait(const JcgView& J, int m, int it, double* pub) {
    __syncthreads();
    if (threadIdx.x == 0) {
        long long spins = 0;
        int g;
        bool ok = true;
        while ((g = ld_acquire_i32(&J.mgen[m])) < it) {
            if (++spins > 4096) __nanosleep(128);
            if (spins > J.wait_polls) { atomicOr(J.err, ERR_BARRIER_TIMEOUT); ok = false; break; }
            if ((spins & 255) == 0 && (*((volatile int32_t*)J.err) & ERR_BARRIER_TIMEOUT)) { ok = false; break; }
        }
        __threadfence();
        if (!ok) {
            pub[2] = -1.0;
        } else if (g == kRetired) {
            pub[2] = 0.0;
        } else {
            pub[0] = __ldcg(&J.mpub[2 * m]);
            pub[1] = __ldcg(&J.mpub[2 * m + 1]);
            pub[2] = 1.0;
        }
    }
    __syncthreads();
}

// This block's tiles of member m are done for inner iteration it (their partials of iteration
// it + 1 are in parity slot np).  The member's last arriver publishes iteration it + 1.
// WIDE: the last arriver sums the partials with member_totals_wide (same bits): 4% faster on a
// system that fits in L2, but 8% slower beyond it, where the larger register footprint costs more
// than the shorter reduction saves; so only the two-rows-in-flight instantiation uses it.
template <bool WIDE>
__device__ __forceinline__ void member_arrive(const JcgView& J, int m, int it, int np, double* sh, int* shv) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned old = atomicAdd(&J.mcnt[m], 1u);
        const bool last = ((old + 1u) % arrivals(J, m)) == 0u;
        if (last) __threadfence();
        *shv = last ? 1 : 0;
    }
    __syncthreads();
    if (!*shv) return;
    const int kinds[3] = {np ? R_RZ1 : R_RZ0, np ? R_WU1 : R_WU0, np ? R_RR1 : R_RR0};
    double tot[3];
    if constexpr (WIDE) member_totals_wide<3>(J, m, kinds, tot, sh);
    else member_totals<3>(J, m, kinds, tot, sh);
    if (threadIdx.x != 0) return;
    const int nmem = J.nmem, nit = it + 1;
    const int cp = np ^ 1;
    const bool done = checkpoint(J, it, J.inner_maxiter) && tot[2] <= J.mem_atol2[nmem + m];
    if (done || nit == J.inner_maxiter) {
        // the sweep ends after iteration it: keep its (alpha, gamma) and recursive r.r for the
        // next sweep; a sweep stopped by the iteration cap leaves r.r = 0, so the next sweep
        // restarts the recurrence instead of continuing a stalled one
        J.mem_ab[(size_t)6 * nmem + m] = J.mem_ab[(size_t)cp * nmem + m];
        J.mem_ab[(size_t)7 * nmem + m] = J.mem_ab[(size_t)(2 + cp) * nmem + m];
        J.mem_ab[(size_t)8 * nmem + m] = done ? tot[2] : 0.0;
    }
    if (done) {
        J.mret[m] = nit;
        J.minner[m] += nit;
        __threadfence();
        st_release_i32(&J.mgen[m], kRetired);
        return;
    }
    const double ap = J.mem_ab[(size_t)cp * nmem + m];
    const double gp = J.mem_ab[(size_t)(2 + cp) * nmem + m];
    const double beta = (gp != 0.0) ? tot[0] / gp : 0.0;
    const double den = tot[1] - ((ap != 0.0) ? beta * tot[0] / ap : 0.0);
    const double alpha = (den != 0.0) ? tot[0] / den : 0.0;
    J.mem_ab[(size_t)np * nmem + m] = alpha;
    J.mem_ab[(size_t)(2 + np) * nmem + m] = tot[0];
    J.mpub[2 * m] = alpha;
    J.mpub[2 * m + 1] = beta;
    __threadfence();
    st_release_i32(&J.mgen[m], nit);
}

template <bool SELL, int UNR>
__global__ void __launch_bounds__(kThreads, GS_JCG_IR_MIN_BLOCKS) k_jcg_ir(JcgView J) {
    __shared__ double sh[4 * 32];
    __shared__ double pub[3];
    __shared__ int shv;
    const int tid = threadIdx.x;
    const int tb0 = J.blk_t0[blockIdx.x], tb1 = J.blk_t0[blockIdx.x + 1];
    const int nmem = J.nmem;
    float* const dd = ir_d(J);
    phase_bb(J, sh);
    GSYNC();
    phase_atol(J, sh);
    GSYNC();
    for (int outer = 0; outer < 64; outer++) {
        // O1: FP64 residual r = b - A x; u_0 = D^-1 r in FP32 replaces the inner solve's recursive
        // residual, d = 0; the search direction p and s~ = D^-1 A p carry over from the previous
        // sweep (residual replacement: the inner CG continues instead of restarting; the first
        // sweep starts from p = s~ = 0); outer r.r partials
        {
            float4* uw0 = ir_uws(J, 0);
            for (int t = tb0; t < tb1; t++) {
                const int m = J.tile_mem[t];
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                const int dn = uniform_ld(&J.mdone[m], &shv);
                if (dn >= 0) {
                    if (outer == 0 && dn == 0)
                        for (int i = r0 + tid; i < r1; i += kThreads) J.x[i] = 0.0;
                    continue;
                }
                // parity holding the previous sweep's last s~ (its final inner iteration index)
                int last = 0;
                if (outer > 0) {
                    const int rt = uniform_ld(&J.mret[m], &shv);
                    last = (rt >= 0 ? rt : J.inner_maxiter) & 1;
                }
                const float4* uwl = ir_uws(J, last);
                double v[1] = {0.0};
                for (int i = r0 + tid; i < r1; i += kThreads) {
                    const double s = row_dot<SELL, double>(J, J.A, i, [&](int c) { return J.x[c]; });
                    const double ri = J.b[i] - s;
                    // s~ and p of the previous sweep's last iteration (zero in the first sweep)
                    float sprev = 0.0f, pprev = 0.0f;
                    if (outer > 0) { const float4 l = uwl[i]; sprev = l.z; pprev = l.w; }
                    uw0[i] = make_float4((float)(J.invD[i] * ri), 0.0f, sprev, pprev);
                    dd[i] = 0.0f;
                    v[0] += ri * ri;
                }
                const int kinds[1] = {R_OUT};
                put_partials<1>(J, t, kinds, v, sh);
            }
        }
        GSYNC();
        // O2: outer convergence test; w~_0 = (D^-1 A) u_0 and (gamma, delta, r.r) of iteration 0
        {
            float4* uw0 = ir_uws(J, 0);
            const float* u0 = J.ir32;          // u components of parity 0 (stride 4)
            for (int t = tb0; t < tb1; t++) {
                const int m = J.tile_mem[t];
                if (uniform_ld(&J.mdone[m], &shv) >= 0) continue;
                const int kinds1[1] = {R_OUT};
                double tot[1];
                member_totals<1>(J, m, kinds1, tot, sh);
                const bool owner = (t == J.mem_t0[m] && tid == 0);
                if (tot[0] <= J.mem_atol2[m]) {
                    if (owner) {
                        // retired at the outer test: blocks that hold its tiles beside another
                        // member's see kRetired at every inner iteration instead of waiting
                        J.mdone[m] = J.minner[m]; J.mouter[m] = outer;
                        J.mgen[m] = kRetired;
                        __threadfence(); atomicAdd(J.ndone, 1u);
                    }
                    continue;
                }
                if (owner) {
                    // a sweep that did not halve the FP64 residual restarts the next one's
                    // recurrence (the continued search directions have gone stale)
                    if (outer > 0 && tot[0] > 0.25 * J.mem_atol2[nmem + m] / (J.inner_rtol * J.inner_rtol))
                        J.mem_ab[(size_t)8 * nmem + m] = 0.0;
                    J.mem_atol2[nmem + m] = J.inner_rtol * J.inner_rtol * tot[0];
                    J.mouter[m] = outer + 1;
                    J.mret[m] = -1;
                    J.mgen[m] = 0;
                    J.mcnt[m] = 0u;
                }
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                double v[3] = {0.0, 0.0, 0.0};
                for (int i = r0 + tid; i < r1; i += kThreads) {
                    // neighbours read only the u component, this row writes only its w~ component
                    const float w = row_dot<SELL, float>(J, J.A32, i, [&](int c) { return u0[4 * (size_t)c]; });
                    uw0[i].y = w;
                    const double ui = u0[4 * (size_t)i], dg = J.diag32[i], du = dg * ui;
                    v[0] += du * ui; v[1] += dg * (double)w * ui; v[2] += du * du;
                }
                const int kinds[3] = {R_RZ0, R_WU0, R_RR0};
                put_partials<3>(J, t, kinds, v, sh);
            }
        }
        GSYNC();
        if (*((volatile unsigned*)J.ndone) >= (unsigned)nmem) break;
        // inner iterations: iteration 0's scalars come from the O2 totals (every block forms them);
        // later ones are published per member by its last arriver
        for (int it = 0; it < J.inner_maxiter; it++) {
            const int cp = it & 1, np = cp ^ 1;
            const float4* __restrict__ uwc = ir_uws(J, cp);
            float4* __restrict__ uwn = ir_uws(J, np);
            bool any = false;
            int cm = -1;
            bool on = false;
            float al = 0.0f, bt = 0.0f;
            for (int t = tb0; t < tb1; t++) {
                const int m = J.tile_mem[t];
                if (m != cm) {
                    if (cm >= 0 && on) member_arrive<UNR == kRowUnroll>(J, cm, it, np, sh, &shv);
                    cm = m;
                    if (it == 0) {
                        on = uniform_ld(&J.mdone[m], &shv) < 0;
                        if (on) {
                            const int kinds[3] = {R_RZ0, R_WU0, R_RR0};
                            double tot[3];
                            member_totals<3>(J, m, kinds, tot, sh);
                            // first sweep: beta = 0.  Later sweeps continue the recurrence from the
                            // previous sweep's last (alpha, gamma) -- residual replacement every
                            // inner_rtol reduction, which keeps the FP32 recursion accurate when
                            // inner_rtol >= 1e-2 -- unless the replaced residual is more than 4x the
                            // recursive one it replaces (r.r more than 16x), the previous sweep hit
                            // the iteration cap, or it did not halve the FP64 residual.  Tighter
                            // inner tolerances, or any of these, restart the recurrence (beta = 0):
                            // plain restarted refinement.
                            const bool reliable = J.inner_rtol >= 1e-2;
                            const double ac = (outer > 0) ? J.mem_ab[(size_t)6 * nmem + m] : 0.0;
                            const double gc = (outer > 0) ? J.mem_ab[(size_t)7 * nmem + m] : 0.0;
                            const double rc = (outer > 0) ? J.mem_ab[(size_t)8 * nmem + m] : 0.0;
                            const bool cont = reliable && gc != 0.0 && ac != 0.0 && tot[2] <= 16.0 * rc;
                            const double beta = cont ? tot[0] / gc : 0.0;
                            const double den = tot[1] - ((beta != 0.0) ? beta * tot[0] / ac : 0.0);
                            const double alpha = (den != 0.0) ? tot[0] / den : 0.0;
                            if (t == J.mem_t0[m] && tid == 0) {
                                J.mem_ab[m] = alpha;
                                J.mem_ab[(size_t)2 * nmem + m] = tot[0];
                            }
                            al = (float)alpha; bt = (float)beta;
                        }
                    } else {
                        member_wait(J, m, it, pub);
                        if (pub[2] < -0.5) return;
                        on = pub[2] > 0.5;
                        al = (float)pub[0]; bt = (float)pub[1];
                    }
                }
                if (!on) continue;
                any = true;
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                double v[3] = {0.0, 0.0, 0.0};
#pragma unroll UNR
                for (int i = r0 + tid; i < r1; i += kThreads) {
                    // a row's (u, w~, s~, p) travel together: one 16-byte load and store per row
                    const float4 o = uwc[i];
                    const float snew = o.y + bt * o.z;
                    const float pnew = o.x + bt * o.w;
                    dd[i] += al * pnew;
                    const float unew = u_next(o, al, bt);
                    const float w = row_dot<SELL, float>(J, J.A32, i, [&](int c) { return u_next(uwc[c], al, bt); });
                    uwn[i] = make_float4(unew, w, snew, pnew);
                    const double dg = J.diag32[i], du = dg * unew;
                    v[0] += du * unew; v[1] += dg * (double)w * unew; v[2] += du * du;
                }
                const int kinds[3] = {np ? R_RZ1 : R_RZ0, np ? R_WU1 : R_WU0, np ? R_RR1 : R_RR0};
                put_partials<3>(J, t, kinds, v, sh);
            }
            if (cm >= 0 && on) member_arrive<UNR == kRowUnroll>(J, cm, it, np, sh, &shv);
            if (!any) break;
        }
        // x += d for the members of this sweep; the sweep's owner closes the member's count
        // (members still on at the iteration cap count it in full)
        for (int t = tb0; t < tb1; t++) {
            const int m = J.tile_mem[t];
            if (uniform_ld(&J.mdone[m], &shv) >= 0) continue;
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            for (int i = r0 + tid; i < r1; i += kThreads) J.x[i] += (double)dd[i];
            if (t == J.mem_t0[m] && tid == 0 && J.mret[m] < 0) J.minner[m] += J.inner_maxiter;
        }
        GSYNC();
    }
    for (int t = tb0; t < tb1; t++) {
        const int m = J.tile_mem[t];
        if (t == J.mem_t0[m] && tid == 0 && ld_done(J, m) < 0) {
            J.mdone[m] = J.minner[m];
            atomicOr(J.status, ERR_JCG_NOT_CONVERGED);
        }
    }
}

// ------------------------------------------------------------------------------ host ----

static const void* ir_kernel(bool sell, bool large) {
    if (sell) return large ? (const void*)k_jcg_ir<true, kRowUnrollLarge> : (const void*)k_jcg_ir<true, kRowUnroll>;
    return large ? (const void*)k_jcg_ir<false, kRowUnrollLarge> : (const void*)k_jcg_ir<false, kRowUnroll>;
}

struct JcgWork {
    int n = 0, nmem = 0, ntiles = 0, grid = 0, grid64 = 0, gridir = 0;
    bool ir_large = false;           // the FP32 inner solve's working set exceeds the L2
    bool sell = false;               // kernels instantiated for the SELL-32 layout
    int32_t *tile_r0 = nullptr, *tile_r1 = nullptr, *tile_mem = nullptr, *mem_t0 = nullptr, *mem_t1 = nullptr;
    int32_t *blk64 = nullptr, *blkir = nullptr;
    double *tile_part = nullptr, *mem_atol2 = nullptr, *mem_ab = nullptr;
    // per-member control words in one array: mdone, mouter, minner, mret, mgen, mcnt ([nmem] each),
    // ndone, status (ERR_JCG_NOT_CONVERGED of the last solve)
    int32_t* mctl = nullptr;
    int32_t* status = nullptr;
    int32_t *mdone = nullptr, *mouter = nullptr, *minner = nullptr, *mret = nullptr, *mgen = nullptr;
    unsigned* mcnt = nullptr;
    int32_t *mnblk = nullptr, *mnblk64 = nullptr;   // blocks holding each member's tiles (IR, FP64 grids)
    unsigned* ndone = nullptr;
};

// Tile rows of a member: a function of the member's own size and the tiling only (batch
// independence).  By default a large member is cut into about 592 tiles, i.e. one per block of a
// 4-blocks-per-SM grid on a 148-SM part, so its rows spread evenly over the SMs, and tiles never
// go below 1,024 rows (four rows per thread): every tile ends in a block-wide reduction, and
// smaller tiles leave too little independent work between those reductions.  The autotuner may
// choose other values (JcgTiling).
static int tile_rows_for(int rows, const JcgTiling& tl) {
    const long long per = ((long long)rows + tl.tiles - 1) / tl.tiles;
    return (int)std::max((long long)tl.min_rows, (per + 31) / 32 * 32);
}

// Contiguous tile ranges per block with about the same number of rows in each.
static void block_ranges(const std::vector<int32_t>& tr0, const std::vector<int32_t>& tr1, int grid,
                         std::vector<int32_t>& bt) {
    const int T = (int)tr0.size();
    std::vector<long long> cum(T + 1, 0);
    for (int t = 0; t < T; t++) cum[t + 1] = cum[t] + (tr1[t] - tr0[t]);
    bt.assign(grid + 1, T);
    bt[0] = 0;
    int t = 0;
    for (int b = 1; b < grid; b++) {
        const long long target = cum[T] * b / grid;
        while (t < T && cum[t] + (tr1[t] - tr0[t]) / 2 < target) t++;
        bt[b] = std::max(bt[b - 1], t);
    }
}

static int coop_blocks(const void* fn, int nsm, int cap = 4) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    if (per_sm > cap) per_sm = cap;
    return nsm * per_sm;
}

cudaError_t jcg_work_alloc(JcgWork*& w, const std::vector<int>& row0, const std::vector<int>& rows, bool sell,
                           cudaStream_t st, const JcgTiling& tiling) {
    w = new JcgWork();
    const int nmem = (int)rows.size();
    std::vector<int32_t> tr0, tr1, tm, mt0(nmem), mt1(nmem);
    for (int m = 0; m < nmem; m++) {
        const int tr = tile_rows_for(rows[m], tiling);
        mt0[m] = (int)tr0.size();
        for (int r = 0; r < rows[m]; r += tr) {
            tr0.push_back(row0[m] + r);
            tr1.push_back(row0[m] + std::min(rows[m], r + tr));
            tm.push_back(m);
        }
        mt1[m] = (int)tr0.size();
    }
    w->nmem = nmem;
    w->ntiles = (int)tr0.size();
    const int T = w->ntiles;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    long long nrows = 0;
    for (int r : rows) nrows += r;
    w->ir_large = (double)nrows * kIrBytesPerRow > (double)l2;
    w->sell = sell;
    const void* f64 = sell ? (const void*)k_jcg64<true> : (const void*)k_jcg64<false>;
    const void* fir = ir_kernel(sell, w->ir_large);
    w->grid64 = std::max(1, std::min(T, coop_blocks(f64, nsm, tiling.per_sm)));
    w->gridir = std::max(1, std::min(T, coop_blocks(fir, nsm, tiling.per_sm)));
    std::vector<int32_t> b64, bir;
    block_ranges(tr0, tr1, w->grid64, b64);
    block_ranges(tr0, tr1, w->gridir, bir);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 8); };
    A((void**)&w->tile_r0, 4 * T); A((void**)&w->tile_r1, 4 * T); A((void**)&w->tile_mem, 4 * T);
    A((void**)&w->mem_t0, 4 * nmem); A((void**)&w->mem_t1, 4 * nmem);
    A((void**)&w->blk64, 4 * b64.size()); A((void**)&w->blkir, 4 * bir.size());
    A((void**)&w->tile_part, 8 * (size_t)R_KINDS * T);
    A((void**)&w->mem_atol2, 16 * (size_t)nmem);
    A((void**)&w->mem_ab, 72 * (size_t)nmem);
    A((void**)&w->mctl, 4 * (6 * (size_t)nmem + 2));
    A((void**)&w->mnblk, 4 * (size_t)nmem);
    A((void**)&w->mnblk64, 4 * (size_t)nmem);
    if (e != cudaSuccess) return e;
    w->mdone = w->mctl; w->mouter = w->mctl + nmem; w->minner = w->mctl + 2 * nmem; w->mret = w->mctl + 3 * nmem;
    w->mgen = w->mctl + 4 * nmem; w->mcnt = (unsigned*)(w->mctl + 5 * nmem);
    w->ndone = (unsigned*)(w->mctl + 6 * nmem);
    w->status = w->mctl + 6 * nmem + 1;
    {
        // blocks of each grid holding tiles of each member
        auto count = [&](const std::vector<int32_t>& bt, int grid, int32_t* dst) {
            std::vector<int32_t> nb(nmem, 0);
            for (int b = 0; b < grid; b++) {
                int last = -1;
                for (int t = bt[b]; t < bt[b + 1]; t++)
                    if (tm[t] != last) { last = tm[t]; nb[last]++; }
            }
            cudaMemcpyAsync(dst, nb.data(), 4 * (size_t)nmem, cudaMemcpyHostToDevice, st);
        };
        count(bir, w->gridir, w->mnblk);
        count(b64, w->grid64, w->mnblk64);
    }
    // uploads on the caller's stream, never the legacy default stream (pageable sources are
    // staged before each call returns)
    cudaMemcpyAsync(w->tile_r0, tr0.data(), 4 * T, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->tile_r1, tr1.data(), 4 * T, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->tile_mem, tm.data(), 4 * T, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->mem_t0, mt0.data(), 4 * nmem, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->mem_t1, mt1.data(), 4 * nmem, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->blk64, b64.data(), 4 * b64.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(w->blkir, bir.data(), 4 * bir.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(w->tile_part, 0, 8 * (size_t)R_KINDS * T, st);
    cudaMemsetAsync(w->mctl, 0, 4 * (6 * (size_t)nmem + 2), st);
    cudaStreamSynchronize(st);
    return cudaGetLastError();
}

void jcg_work_free(JcgWork* w) {
    if (!w) return;
    void* ps[] = {w->tile_r0, w->tile_r1, w->tile_mem, w->mem_t0, w->mem_t1, w->blk64, w->blkir,
                  w->tile_part, w->mem_atol2, w->mem_ab, w->mctl, w->mnblk, w->mnblk64};
    for (void* p : ps) cudaFree(p);
    delete w;
}

cudaError_t jcg_launch(const JcgArgs& a, JcgWork* w, cudaStream_t st, int nsm) {
    (void)nsm;
    JcgView J{};
    J.n = a.n; J.nmem = w->nmem; J.ntiles = w->ntiles;
    J.indptr = a.indptr; J.sell = a.sell; J.indices = a.indices; J.A = a.A; J.A32 = a.A32; J.b = a.b; J.invD = a.invD;
    J.x = a.x; J.r = a.r; J.z = a.z; J.q = a.q; J.p0 = a.p0; J.p1 = a.p1;
    J.ir32 = a.ir32; J.diag32 = a.diag32;
    J.tile_r0 = w->tile_r0; J.tile_r1 = w->tile_r1; J.tile_mem = w->tile_mem;
    J.mem_t0 = w->mem_t0; J.mem_t1 = w->mem_t1;
    const bool ir = (a.precision == GS_FP32_IR);
    J.blk_t0 = ir ? w->blkir : w->blk64;
    J.tile_part = w->tile_part; J.mem_atol2 = w->mem_atol2;
    J.mdone = w->mdone; J.mouter = w->mouter; J.minner = w->minner; J.mret = w->mret; J.ndone = w->ndone;
    J.mem_ab = w->mem_ab; J.mpub = w->mem_ab + 4 * (size_t)w->nmem;
    J.mgen = w->mgen; J.mcnt = w->mcnt; J.mnblk = ir ? w->mnblk : w->mnblk64;
    J.bar = a.bar; J.err = a.err; J.status = w->status;
    J.wait_polls = a.wait_polls > 0 ? a.wait_polls : kWaitPolls;
    J.stall_member = (a.stall_member >= 0 && a.stall_member < w->nmem) ? a.stall_member : -1;
    J.rtol = a.rtol; J.maxiter = a.maxiter; J.check_every = a.check_every > 0 ? a.check_every : 1;
    J.inner_rtol = a.inner_rtol; J.inner_maxiter = a.inner_maxiter;
    cudaMemsetAsync(w->mdone, 0xFF, 4 * (size_t)w->nmem, st);
    cudaMemsetAsync(w->mouter, 0, 4 * (5 * (size_t)w->nmem + 2), st);   // mouter .. mcnt, ndone, status
    void* args[] = {&J};
    if ((a.sell != nullptr) != w->sell) return cudaErrorInvalidValue;
    const void* fn = ir ? ir_kernel(w->sell, w->ir_large)
                        : (w->sell ? (const void*)k_jcg64<true> : (const void*)k_jcg64<false>);
    const int grid = ir ? w->gridir : w->grid64;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, st);
}

cudaError_t jcg_read_iters(JcgWork* w, std::vector<int>& iters, std::vector<int>& outer, cudaStream_t st) {
    iters.resize(w->nmem);
    outer.resize(w->nmem);
    cudaMemcpyAsync(iters.data(), w->mdone, 4 * (size_t)w->nmem, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(outer.data(), w->mouter, 4 * (size_t)w->nmem, cudaMemcpyDeviceToHost, st);
    return cudaStreamSynchronize(st);
}

int32_t* jcg_iters_device(JcgWork* w) { return w->mdone; }

cudaError_t jcg_read_status(JcgWork* w, int32_t* flags, cudaStream_t st) {
    cudaMemcpyAsync(flags, w->status, 4, cudaMemcpyDeviceToHost, st);
    return cudaStreamSynchronize(st);
}

// ------------------------------------------------------------- solve without allocating ----
//
// gs_jcg_solve_csr_noalloc: the FP64 solve of k_jcg64 on a caller CSR for callers that cannot
// allocate device memory.  Its scratch (residual, search directions, inverse diagonal, tile
// partials, tile tables and control words) lives in the file-scope array below; every GPU that
// loads the library holds it until the process exits.

constexpr int kNoAllocMaxRows = 65536;
constexpr int kNoAllocTileRows = 256;
constexpr int kNoAllocMaxTiles = kNoAllocMaxRows / kNoAllocTileRows;     // 256
constexpr int kNoAllocMaxBlocks = kNoAllocMaxTiles;
// byte offsets inside the scratch array (all 256-byte aligned)
constexpr size_t kNaVec = sizeof(double) * kNoAllocMaxRows;              // one FP64 vector
constexpr size_t kNaOffPart = 6 * kNaVec;
constexpr size_t kNaOffAtol = kNaOffPart + sizeof(double) * R_KINDS * kNoAllocMaxTiles;
constexpr size_t kNaOffTiles = kNaOffAtol + 256;
constexpr size_t kNaOffBlk = kNaOffTiles + 3 * sizeof(int32_t) * kNoAllocMaxTiles;
constexpr size_t kNaOffCtl = kNaOffBlk + sizeof(int32_t) * (kNoAllocMaxBlocks + 64);
constexpr size_t kNaCtlBytes = 256;
constexpr size_t kNoAllocBytes = kNaOffCtl + kNaCtlBytes;                // about 3.1 MiB

static __device__ __align__(256) unsigned char gs_noalloc_scratch[kNoAllocBytes];

// control words at kNaOffCtl: [0] mem_t0, [1] mem_t1, [2] mdone, [3] mouter, [4] ndone,
// [5] grid barrier word, [6] solve status, [7] err, [8] mgen, [9] mcnt, [10] mnblk (= grid: every
// block holds tiles of the one member); published scalars at kNaOffAtol + 64

__global__ void k_noalloc_setup(unsigned char* base, int n, const int32_t* indptr, const int32_t* indices,
                                const double* A, int ntiles, int grid) {
    // tile tables of one member, block ranges, cleared control words, inverse diagonal
    int32_t* tr0 = (int32_t*)(base + kNaOffTiles);
    int32_t* tr1 = tr0 + kNoAllocMaxTiles;
    int32_t* tm = tr1 + kNoAllocMaxTiles;
    int32_t* bt = (int32_t*)(base + kNaOffBlk);
    int32_t* ctl = (int32_t*)(base + kNaOffCtl);
    double* invD = (double*)(base + 5 * kNaVec);
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, G = gridDim.x * blockDim.x;
    for (int t = gid; t < ntiles; t += G) {
        tr0[t] = t * kNoAllocTileRows;
        tr1[t] = min(n, (t + 1) * kNoAllocTileRows);
        tm[t] = 0;
    }
    for (int b = gid; b <= grid; b += G) bt[b] = (int32_t)((long long)ntiles * b / grid);
    if (gid < (int)(kNaCtlBytes / 4)) ctl[gid] = (gid == 1) ? ntiles : (gid == 2 ? -1 : (gid == 10 ? grid : 0));
    for (int i = gid; i < n; i += G) {
        double dg = 0.0;
        for (int a = indptr[i]; a < indptr[i + 1]; a++)
            if (indices[a] == i) dg = A[a];
        invD[i] = 1.0 / dg;
    }
}

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once per device.
static cudaError_t noalloc_base(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, gs_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = (unsigned char*)p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace gs

extern "C" gs_status gs_jcg_solve_csr_noalloc(int n, const int32_t* indptr, const int32_t* indices,
                                              const double* data, const double* b, double* x, double rtol,
                                              int maxiter, int check_every, void* stream, int* iters) {
    using namespace gs;
    if (n <= 0 || n > kNoAllocMaxRows || !indptr || !indices || !data || !b || !x || maxiter < 1)
        return GS_ERR_ARG;
    unsigned char* base = nullptr;
    if (noalloc_base(&base) != cudaSuccess) return GS_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = (n + kNoAllocTileRows - 1) / kNoAllocTileRows;
    const int grid = std::max(1, std::min(ntiles, coop_blocks((const void*)k_jcg64<false>, nsm)));
    k_noalloc_setup<<<std::max(1, std::min(64, (n + 255) / 256)), 256, 0, st>>>(base, n, indptr, indices, data,
                                                                               ntiles, grid);
    int32_t* ctl = (int32_t*)(base + kNaOffCtl);
    JcgView J{};
    J.n = n; J.nmem = 1; J.ntiles = ntiles;
    J.indptr = indptr; J.indices = indices; J.A = data; J.b = b; J.x = x;
    J.r = (double*)(base + 0 * kNaVec); J.z = (double*)(base + 1 * kNaVec); J.q = (double*)(base + 2 * kNaVec);
    J.p0 = (double*)(base + 3 * kNaVec); J.p1 = (double*)(base + 4 * kNaVec);
    J.invD = (const double*)(base + 5 * kNaVec);
    J.tile_part = (double*)(base + kNaOffPart);
    J.mem_atol2 = (double*)(base + kNaOffAtol);
    J.tile_r0 = (const int32_t*)(base + kNaOffTiles);
    J.tile_r1 = J.tile_r0 + kNoAllocMaxTiles;
    J.tile_mem = J.tile_r1 + kNoAllocMaxTiles;
    J.blk_t0 = (const int32_t*)(base + kNaOffBlk);
    J.mem_t0 = ctl + 0; J.mem_t1 = ctl + 1; J.mdone = ctl + 2; J.mouter = ctl + 3;
    J.ndone = (unsigned*)(ctl + 4); J.bar = (unsigned*)(ctl + 5);
    J.err = ctl + 7; J.status = ctl + 6;
    J.wait_polls = kWaitPolls; J.stall_member = -1;
    J.mgen = ctl + 8; J.mcnt = (unsigned*)(ctl + 9); J.mnblk = ctl + 10;
    J.mpub = (double*)(base + kNaOffAtol + 64);
    J.rtol = rtol; J.maxiter = maxiter; J.check_every = check_every > 0 ? check_every : 1;
    void* args[] = {&J};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_jcg64<false>, dim3(grid), dim3(kThreads), args, 0, st);
    if (e != cudaSuccess) return GS_ERR_CUDA;
    int32_t h[8] = {0};
    e = cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GS_ERR_CUDA;
    if (iters) *iters = h[2];
    if (h[7] & ERR_BARRIER_TIMEOUT) return GS_ERR_TIMEOUT;
    return GS_OK;
}
