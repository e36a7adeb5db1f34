// Jacobi-preconditioned CG for the elevation system, one persistent cooperative launch per
// solve for every member of a batch (replaces PCGSolverMultiGPU.solve / NativePCG,
// src/solver/pcg_solver.py:1075-1124 and src/solver/pcg_loop.cpp:334-416).
//
// Rows are cut into tiles of kTile rows that never straddle two members.  Every reduction is
// deterministic and independent of the batch: each tile writes a partial from a fixed
// block tree, and the last tile of a member to finish sums that member's tile partials in a
// fixed order (threadfence-reduction pattern).  Scalars stay on the device; convergence is
// tested every check_every iterations on the device, so a solve never round-trips to the host.
//
// Per iteration two phases separated by grid barriers:
//   A: beta = rz/rz_old; p_new = z + beta p; q = A p_new (p_new of neighbour rows is formed on
//      the fly from z and the previous p, so no barrier is needed between p and q); p.q partials
//   B: alpha = rz/p.q; x += alpha p; r -= alpha q; z = invD r; r.r and r.z partials.
// FP32_IR mode runs the same iteration in FP32 on the residual equation A d = r (FP32 matrix
// copy and vectors, FP64 dot products) inside FP64 refinement sweeps r = b - A x.
#include <cooperative_groups.h>

#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

constexpr int kTile = 1024;        // rows per tile
constexpr int kThreads = 256;      // threads per block (4 rows per thread per tile)
constexpr int kRPT = kTile / kThreads;

enum { R_BB = 0, R_PQ = 1, R_RR0 = 2, R_RZ0 = 3, R_RR1 = 4, R_RZ1 = 5, R_KINDS = 6 };
enum { G_BB = 0, G_PQ = 1, G_RRZ0 = 2, G_RRZ1 = 3, G_GROUPS = 4 };

struct JcgView {
    int n, nmem, ntiles;
    const int32_t *indptr, *indices;
    const double* A;
    const float* A32;
    const double* b;
    const double* invD;
    double *x, *r, *z, *q, *p0, *p1;
    float *r32, *z32, *q32, *p032, *p132, *d32, *invD32;
    const int32_t *tile_r0, *tile_r1, *tile_mem, *mem_t0, *mem_t1;
    double* tile_part;             // [R_KINDS][ntiles]
    double* mem_tot;               // [R_KINDS][nmem]
    double* mem_atol2;             // [nmem]
    unsigned* mem_cnt;             // [G_GROUPS][nmem]
    int32_t* mdone;                // [nmem] iterations at convergence, -1 while active
    int32_t* mouter;               // [nmem] refinement sweeps (IR)
    unsigned* ndone;
    unsigned *bar_count, *bar_gen;
    int32_t* err;
    double rtol;
    int maxiter, check_every;
    double inner_rtol;
    int inner_maxiter;
};

// block-wide fixed-order sum of NV values per thread; result valid in thread 0
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
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = (lane < (kThreads >> 5)) ? sh[k * 32 + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    }
    __syncthreads();
}

// Publish a tile's partials and, in the last tile of the member to arrive, the member totals.
// Returns true in the block that computed the totals.
template <int NV>
__device__ bool publish(const JcgView& J, int t, int m, int grp, const int (&kinds)[NV], double (&v)[NV],
                        double* sh, int* shflag) {
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) J.tile_part[(size_t)kinds[k] * J.ntiles + t] = v[k];
        __threadfence();
        const unsigned nt = (unsigned)(J.mem_t1[m] - J.mem_t0[m]);
        const unsigned old = atomicAdd(&J.mem_cnt[grp * J.nmem + m], 1u);
        *shflag = (old == nt - 1);
    }
    __syncthreads();
    const bool last = *shflag;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    const int t0 = J.mem_t0[m], t1 = J.mem_t1[m];
    double s[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        s[k] = 0.0;
        const volatile double* tp = J.tile_part + (size_t)kinds[k] * J.ntiles;
        for (int tt = t0 + threadIdx.x; tt < t1; tt += kThreads) s[k] += tp[tt];
    }
    block_sum<NV>(s, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) J.mem_tot[(size_t)kinds[k] * J.nmem + m] = s[k];
        J.mem_cnt[grp * J.nmem + m] = 0u;
        __threadfence();
    }
    __syncthreads();
    return true;
}

__device__ __forceinline__ double ld_tot(const JcgView& J, int kind, int m) {
    return *((volatile double*)&J.mem_tot[(size_t)kind * J.nmem + m]);
}
__device__ __forceinline__ int ld_done(const JcgView& J, int m) {
    return *((volatile int32_t*)&J.mdone[m]);
}

// ------------------------------------------------------------------------------- FP64 ----

__global__ void __launch_bounds__(kThreads) k_jcg64(JcgView J) {
    __shared__ double sh[4 * 32];
    __shared__ int shflag;
    const int G = gridDim.x;
    const int tid = threadIdx.x;

    // I0: |b|^2 per member; p = 0
    for (int t = blockIdx.x; t < J.ntiles; t += G) {
        const int m = J.tile_mem[t], r0 = J.tile_r0[t], r1 = J.tile_r1[t];
        double v[1] = {0.0};
        for (int j = 0; j < kRPT; j++) {
            const int i = r0 + tid + j * kThreads;
            if (i < r1) { const double bi = J.b[i]; v[0] += bi * bi; J.p0[i] = 0.0; J.p1[i] = 0.0; }
        }
        const int kinds[1] = {R_BB};
        if (publish<1>(J, t, m, G_BB, kinds, v, sh, &shflag) && tid == 0) {
            const double atol = J.rtol * sqrt(J.mem_tot[(size_t)R_BB * J.nmem + m]);
            J.mem_atol2[m] = atol * atol;
            if (atol == 0.0) { J.mdone[m] = 0; atomicAdd(J.ndone, 1u); }
        }
    }
    if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;

    // I1: r = b - A x; z = invD r; (r.r, r.z) into the parity-1 slots (iteration -1)
    for (int t = blockIdx.x; t < J.ntiles; t += G) {
        const int m = J.tile_mem[t], r0 = J.tile_r0[t], r1 = J.tile_r1[t];
        const bool zero = ld_done(J, m) == 0;
        double v[2] = {0.0, 0.0};
        for (int j = 0; j < kRPT; j++) {
            const int i = r0 + tid + j * kThreads;
            if (i >= r1) continue;
            if (zero) { J.x[i] = 0.0; J.r[i] = 0.0; J.z[i] = 0.0; continue; }
            double s = 0.0;
            for (int a = J.indptr[i]; a < J.indptr[i + 1]; a++) s += J.A[a] * J.x[J.indices[a]];
            const double ri = J.b[i] - s, zi = J.invD[i] * ri;
            J.r[i] = ri; J.z[i] = zi;
            v[0] += ri * ri; v[1] += ri * zi;
        }
        const int kinds[2] = {R_RR1, R_RZ1};
        publish<2>(J, t, m, G_RRZ1, kinds, v, sh, &shflag);
    }
    if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;

    for (int it = 0; it < J.maxiter; it++) {
        if (*((volatile unsigned*)J.ndone) >= (unsigned)J.nmem) break;
        const int cur = (it + 1) & 1;            // parity slot of iteration it-1
        const int old = it & 1;                  // parity slot of iteration it-2
        double* pc = (it & 1) ? J.p1 : J.p0;     // p of iteration it-1
        double* pn = (it & 1) ? J.p0 : J.p1;     // p of iteration it
        // phase A
        for (int t = blockIdx.x; t < J.ntiles; t += G) {
            const int m = J.tile_mem[t];
            if (ld_done(J, m) >= 0) continue;
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            const double rzc = ld_tot(J, cur ? R_RZ1 : R_RZ0, m);
            const double rzo = ld_tot(J, old ? R_RZ1 : R_RZ0, m);
            const double beta = (it == 0 || rzo == 0.0) ? 0.0 : rzc / rzo;
            double v[1] = {0.0};
            for (int j = 0; j < kRPT; j++) {
                const int i = r0 + tid + j * kThreads;
                if (i >= r1) continue;
                double s = 0.0;
                for (int a = J.indptr[i]; a < J.indptr[i + 1]; a++) {
                    const int c = J.indices[a];
                    s += J.A[a] * (J.z[c] + beta * pc[c]);
                }
                const double pi = J.z[i] + beta * pc[i];
                pn[i] = pi; J.q[i] = s;
                v[0] += pi * s;
            }
            const int kinds[1] = {R_PQ};
            publish<1>(J, t, m, G_PQ, kinds, v, sh, &shflag);
        }
        if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
        // phase B
        const int slot_rr = (it & 1) ? R_RR1 : R_RR0, slot_rz = (it & 1) ? R_RZ1 : R_RZ0;
        const int grp = (it & 1) ? G_RRZ1 : G_RRZ0;
        for (int t = blockIdx.x; t < J.ntiles; t += G) {
            const int m = J.tile_mem[t];
            if (ld_done(J, m) >= 0) continue;
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            const double pq = ld_tot(J, R_PQ, m);
            const double rz = ld_tot(J, cur ? R_RZ1 : R_RZ0, m);
            const double alpha = (pq != 0.0) ? rz / pq : 0.0;
            double v[2] = {0.0, 0.0};
            for (int j = 0; j < kRPT; j++) {
                const int i = r0 + tid + j * kThreads;
                if (i >= r1) continue;
                J.x[i] += alpha * pn[i];
                const double ri = J.r[i] - alpha * J.q[i];
                const double zi = J.invD[i] * ri;
                J.r[i] = ri; J.z[i] = zi;
                v[0] += ri * ri; v[1] += ri * zi;
            }
            const int kinds[2] = {slot_rr, slot_rz};
            if (publish<2>(J, t, m, grp, kinds, v, sh, &shflag) && tid == 0) {
                if ((it + 1) % J.check_every == 0 || it == J.maxiter - 1) {
                    const double rr = J.mem_tot[(size_t)slot_rr * J.nmem + m];
                    if (rr <= J.mem_atol2[m]) {
                        J.mdone[m] = it + 1;
                        __threadfence();
                        atomicAdd(J.ndone, 1u);
                    }
                }
            }
        }
        if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
    }
    if (blockIdx.x == 0) {
        for (int m = tid; m < J.nmem; m += kThreads)
            if (J.mdone[m] < 0) { J.mdone[m] = J.maxiter; atomicOr(J.err, ERR_JCG_NOT_CONVERGED); }
    }
}

// ---------------------------------------------------------------------- FP32 + refinement ----

__global__ void __launch_bounds__(kThreads) k_jcg_ir(JcgView J) {
    // Outer FP64 sweeps: r = b - A x (FP64 matrix), stop when r.r <= (rtol |b|)^2 (tested every
    // sweep), else solve A d = r in FP32 JCG to inner_rtol (FP64 dot products), x += d.
    __shared__ double sh[4 * 32];
    __shared__ int shflag;
    const int G = gridDim.x;
    const int tid = threadIdx.x;
    // |b|^2
    for (int t = blockIdx.x; t < J.ntiles; t += G) {
        const int m = J.tile_mem[t], r0 = J.tile_r0[t], r1 = J.tile_r1[t];
        double v[1] = {0.0};
        for (int j = 0; j < kRPT; j++) {
            const int i = r0 + tid + j * kThreads;
            if (i < r1) { const double bi = J.b[i]; v[0] += bi * bi; }
        }
        const int kinds[1] = {R_BB};
        if (publish<1>(J, t, m, G_BB, kinds, v, sh, &shflag) && tid == 0) {
            const double atol = J.rtol * sqrt(J.mem_tot[(size_t)R_BB * J.nmem + m]);
            J.mem_atol2[m] = atol * atol;
            J.mouter[m] = 0;
            if (atol == 0.0) { J.mdone[m] = 0; atomicAdd(J.ndone, 1u); }
        }
    }
    if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
    int total_inner = 0;
    for (int outer = 0; outer < 64; outer++) {
        if (*((volatile unsigned*)J.ndone) >= (unsigned)J.nmem) break;
        // O1: FP64 residual; r32 = r; z32 = invD32 r32; inner (r.r, r.z) into parity 1
        for (int t = blockIdx.x; t < J.ntiles; t += G) {
            const int m = J.tile_mem[t];
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            const bool done = ld_done(J, m) >= 0;
            double v[3] = {0.0, 0.0, 0.0};
            for (int j = 0; j < kRPT; j++) {
                const int i = r0 + tid + j * kThreads;
                if (i >= r1) continue;
                if (done) { if (ld_done(J, m) == 0 && outer == 0) J.x[i] = 0.0; continue; }
                double s = 0.0;
                for (int a = J.indptr[i]; a < J.indptr[i + 1]; a++) s += J.A[a] * J.x[J.indices[a]];
                const double ri = J.b[i] - s;
                const float r32 = (float)ri, z32 = J.invD32[i] * r32;
                J.r32[i] = r32; J.z32[i] = z32; J.d32[i] = 0.0f; J.p032[i] = 0.0f; J.p132[i] = 0.0f;
                v[0] += ri * ri;
                v[1] += (double)r32 * (double)r32;
                v[2] += (double)r32 * (double)z32;
            }
            const int kinds[3] = {R_BB, R_RR1, R_RZ1};   // BB slot now holds the outer r.r
            if (publish<3>(J, t, m, G_RRZ1, kinds, v, sh, &shflag) && tid == 0) {
                const double rr = J.mem_tot[(size_t)R_BB * J.nmem + m];
                if (ld_done(J, m) < 0 && rr <= J.mem_atol2[m]) {
                    J.mdone[m] = total_inner;
                    __threadfence();
                    atomicAdd(J.ndone, 1u);
                } else if (ld_done(J, m) < 0) {
                    J.mouter[m] = outer + 1;   // > 0: the member's inner solve is running
                }
            }
        }
        if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
        if (*((volatile unsigned*)J.ndone) >= (unsigned)J.nmem) break;
        // inner FP32 JCG; member m stops when its inner r.r falls below inner_rtol^2 times the
        // outer r.r (kept in the BB slot); mouter[m] is negated when that happens
        int inner_it = 0;
        for (; inner_it < J.inner_maxiter; inner_it++) {
            const int cur = (inner_it + 1) & 1, old = inner_it & 1;
            float* pc = (inner_it & 1) ? J.p132 : J.p032;
            float* pn = (inner_it & 1) ? J.p032 : J.p132;
            for (int t = blockIdx.x; t < J.ntiles; t += G) {
                const int m = J.tile_mem[t];
                if (ld_done(J, m) >= 0) continue;
                // inner-done marker: the member's tiles stop once mouter[m] is negated
                if (*((volatile int32_t*)&J.mouter[m]) < 0) continue;
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                const double rzc = ld_tot(J, cur ? R_RZ1 : R_RZ0, m);
                const double rzo = ld_tot(J, old ? R_RZ1 : R_RZ0, m);
                const float beta = (inner_it == 0 || rzo == 0.0) ? 0.0f : (float)(rzc / rzo);
                double v[1] = {0.0};
                for (int j = 0; j < kRPT; j++) {
                    const int i = r0 + tid + j * kThreads;
                    if (i >= r1) continue;
                    float s = 0.0f;
                    for (int a = J.indptr[i]; a < J.indptr[i + 1]; a++) {
                        const int c = J.indices[a];
                        s += J.A32[a] * (J.z32[c] + beta * pc[c]);
                    }
                    const float pi = J.z32[i] + beta * pc[i];
                    pn[i] = pi; J.q32[i] = s;
                    v[0] += (double)pi * (double)s;
                }
                const int kinds[1] = {R_PQ};
                publish<1>(J, t, m, G_PQ, kinds, v, sh, &shflag);
            }
            if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
            const int slot_rr = (inner_it & 1) ? R_RR1 : R_RR0, slot_rz = (inner_it & 1) ? R_RZ1 : R_RZ0;
            const int grp = (inner_it & 1) ? G_RRZ1 : G_RRZ0;
            for (int t = blockIdx.x; t < J.ntiles; t += G) {
                const int m = J.tile_mem[t];
                if (ld_done(J, m) >= 0) continue;
                if (*((volatile int32_t*)&J.mouter[m]) < 0) continue;
                const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
                const double pq = ld_tot(J, R_PQ, m);
                const double rz = ld_tot(J, cur ? R_RZ1 : R_RZ0, m);
                const float alpha = (pq != 0.0) ? (float)(rz / pq) : 0.0f;
                double v[2] = {0.0, 0.0};
                for (int j = 0; j < kRPT; j++) {
                    const int i = r0 + tid + j * kThreads;
                    if (i >= r1) continue;
                    J.d32[i] += alpha * pn[i];
                    const float ri = J.r32[i] - alpha * J.q32[i];
                    const float zi = J.invD32[i] * ri;
                    J.r32[i] = ri; J.z32[i] = zi;
                    v[0] += (double)ri * (double)ri; v[1] += (double)ri * (double)zi;
                }
                const int kinds[2] = {slot_rr, slot_rz};
                if (publish<2>(J, t, m, grp, kinds, v, sh, &shflag) && tid == 0) {
                    if ((inner_it + 1) % J.check_every == 0 || inner_it == J.inner_maxiter - 1) {
                        const double rr = J.mem_tot[(size_t)slot_rr * J.nmem + m];
                        if (rr <= J.mem_tot[(size_t)R_BB * J.nmem + m] * J.inner_rtol * J.inner_rtol) {
                            J.mouter[m] = -J.mouter[m];           // inner solve of m finished
                        }
                    }
                }
            }
            if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
            // stop the inner loop when no member is still iterating
            bool active = false;
            for (int m = 0; m < J.nmem && !active; m++)
                if (ld_done(J, m) < 0 && *((volatile int32_t*)&J.mouter[m]) > 0) active = true;
            if (!active) { inner_it++; break; }
        }
        total_inner += inner_it;
        // x += d; restore the sweep counters
        for (int t = blockIdx.x; t < J.ntiles; t += G) {
            const int m = J.tile_mem[t];
            if (ld_done(J, m) >= 0) continue;
            const int r0 = J.tile_r0[t], r1 = J.tile_r1[t];
            for (int j = 0; j < kRPT; j++) {
                const int i = r0 + tid + j * kThreads;
                if (i < r1) J.x[i] += (double)J.d32[i];
            }
        }
        if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
        if (blockIdx.x == 0)
            for (int m = tid; m < J.nmem; m += kThreads)
                if (J.mouter[m] < 0) J.mouter[m] = -J.mouter[m];
        if (!grid_sync(J.bar_count, J.bar_gen, J.err)) return;
    }
    if (blockIdx.x == 0)
        for (int m = tid; m < J.nmem; m += kThreads)
            if (J.mdone[m] < 0) { J.mdone[m] = total_inner; atomicOr(J.err, ERR_JCG_NOT_CONVERGED); }
}

// ------------------------------------------------------------------------------ host ----

static int coop_grid(const void* fn, int nsm, int ntiles) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    int g = nsm * per_sm;
    if (g > ntiles) g = ntiles;
    return g < 1 ? 1 : g;
}

struct JcgWork {
    // work list and reduction scratch shared by the mesh path and the stand-alone solver
    int n = 0, nmem = 0, ntiles = 0;
    int32_t *tile_r0 = nullptr, *tile_r1 = nullptr, *tile_mem = nullptr, *mem_t0 = nullptr, *mem_t1 = nullptr;
    double *tile_part = nullptr, *mem_tot = nullptr, *mem_atol2 = nullptr;
    unsigned* mem_cnt = nullptr;
    int32_t *mdone = nullptr, *mouter = nullptr;
    unsigned* ndone = nullptr;
};

cudaError_t jcg_work_alloc(JcgWork*& w, const std::vector<int>& row0, const std::vector<int>& rows) {
    w = new JcgWork();
    const int nmem = (int)rows.size();
    std::vector<int32_t> tr0, tr1, tm, mt0(nmem), mt1(nmem);
    for (int m = 0; m < nmem; m++) {
        mt0[m] = (int)tr0.size();
        for (int r = 0; r < rows[m]; r += kTile) {
            tr0.push_back(row0[m] + r);
            tr1.push_back(row0[m] + std::min(rows[m], r + kTile));
            tm.push_back(m);
        }
        mt1[m] = (int)tr0.size();
    }
    w->nmem = nmem;
    w->ntiles = (int)tr0.size();
    const int T = w->ntiles;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 8); };
    A((void**)&w->tile_r0, 4 * T); A((void**)&w->tile_r1, 4 * T); A((void**)&w->tile_mem, 4 * T);
    A((void**)&w->mem_t0, 4 * nmem); A((void**)&w->mem_t1, 4 * nmem);
    A((void**)&w->tile_part, 8 * (size_t)R_KINDS * T); A((void**)&w->mem_tot, 8 * (size_t)R_KINDS * nmem);
    A((void**)&w->mem_atol2, 8 * nmem); A((void**)&w->mem_cnt, 4 * (size_t)G_GROUPS * nmem);
    A((void**)&w->mdone, 4 * nmem); A((void**)&w->mouter, 4 * nmem); A((void**)&w->ndone, 8);
    if (e != cudaSuccess) return e;
    cudaMemcpy(w->tile_r0, tr0.data(), 4 * T, cudaMemcpyHostToDevice);
    cudaMemcpy(w->tile_r1, tr1.data(), 4 * T, cudaMemcpyHostToDevice);
    cudaMemcpy(w->tile_mem, tm.data(), 4 * T, cudaMemcpyHostToDevice);
    cudaMemcpy(w->mem_t0, mt0.data(), 4 * nmem, cudaMemcpyHostToDevice);
    cudaMemcpy(w->mem_t1, mt1.data(), 4 * nmem, cudaMemcpyHostToDevice);
    cudaMemset(w->mem_cnt, 0, 4 * (size_t)G_GROUPS * nmem);
    cudaMemset(w->mem_tot, 0, 8 * (size_t)R_KINDS * nmem);
    return cudaGetLastError();
}

void jcg_work_free(JcgWork* w) {
    if (!w) return;
    void* ps[] = {w->tile_r0, w->tile_r1, w->tile_mem, w->mem_t0, w->mem_t1, w->tile_part, w->mem_tot,
                  w->mem_atol2, w->mem_cnt, w->mdone, w->mouter, w->ndone};
    for (void* p : ps) cudaFree(p);
    delete w;
}

cudaError_t jcg_launch(const JcgArgs& a, JcgWork* w, cudaStream_t st, int nsm) {
    JcgView J{};
    J.n = a.n; J.nmem = w->nmem; J.ntiles = w->ntiles;
    J.indptr = a.indptr; J.indices = a.indices; J.A = a.A; J.A32 = a.A32; J.b = a.b; J.invD = a.invD;
    J.x = a.x; J.r = a.r; J.z = a.z; J.q = a.q; J.p0 = a.p0; J.p1 = a.p1;
    J.r32 = a.r32; J.z32 = a.z32; J.q32 = a.q32; J.p032 = a.p032; J.p132 = a.p132; J.d32 = a.d32;
    J.invD32 = a.invD32;
    J.tile_r0 = w->tile_r0; J.tile_r1 = w->tile_r1; J.tile_mem = w->tile_mem;
    J.mem_t0 = w->mem_t0; J.mem_t1 = w->mem_t1;
    J.tile_part = w->tile_part; J.mem_tot = w->mem_tot; J.mem_atol2 = w->mem_atol2; J.mem_cnt = w->mem_cnt;
    J.mdone = w->mdone; J.mouter = w->mouter; J.ndone = w->ndone;
    J.bar_count = a.bar_count; J.bar_gen = a.bar_gen; J.err = a.err;
    J.rtol = a.rtol; J.maxiter = a.maxiter; J.check_every = a.check_every > 0 ? a.check_every : 1;
    J.inner_rtol = a.inner_rtol; J.inner_maxiter = a.inner_maxiter;
    cudaMemsetAsync(w->mdone, 0xFF, 4 * (size_t)w->nmem, st);
    cudaMemsetAsync(w->ndone, 0, 8, st);
    cudaMemsetAsync(w->mem_cnt, 0, 4 * (size_t)G_GROUPS * w->nmem, st);
    void* args[] = {&J};
    const void* fn = (a.precision == GS_FP32_IR) ? (const void*)k_jcg_ir : (const void*)k_jcg64;
    const int grid = coop_grid(fn, nsm, w->ntiles);
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

}  // namespace gs
