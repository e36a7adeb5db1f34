// Device helpers shared by the gschism_b200 kernels.
//
// Every FP64 expression that feeds a compared field keeps the operand order of the reference
// kernels (src/kernels/meshdata.cu), so the FP64 form reproduces the CPU restatement to
// rounding; the backtracking file is compiled without FMA contraction so its predicates and
// element indices match bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gs_internal.h"

namespace gs {

struct VG {
    int nvrt, nz;
    double h_s, h_c, h0;
    double ztot[kMaxLevels + 1];
    double sigma[kMaxLevels];
    double cs[kMaxLevels];
};

__device__ __forceinline__ double2 v2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return v2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return v2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator*(double2 a, double s) { return v2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 operator/(double2 a, double s) { return v2(a.x / s, a.y / s); }
__device__ __forceinline__ double dot2(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double cross2(double2 a, double2 b) { return a.x * b.y - a.y * b.x; }

// z of level k at a node (Node::compZCoord, ivcor = 2)
__device__ __forceinline__ double compz(const VG& vg, double eta2, double depth, int kb, int k) {
    if (eta2 + depth <= vg.h0) return 0.0;
    const double hmod2 = fmin(depth, vg.h_s);
    if (k == vg.nvrt - 1) return eta2;
    if (k == vg.nz - 1) return -hmod2;
    if (k == kb) return -depth;
    if (k < vg.nz - 1) return vg.ztot[k];
    const int ks = k - (vg.nz - 1);
    if (hmod2 <= vg.h_c) return vg.sigma[ks] * (hmod2 + eta2) + eta2;
    return eta2 * (1.0 + vg.sigma[ks]) + vg.h_c * vg.sigma[ks] + (hmod2 - vg.h_c) * vg.cs[ks];
}

// bottom level of a node (Node::updateKb, ivcor = 2)
__device__ __forceinline__ int node_kb(const VG& vg, double depth) {
    if (depth <= vg.h_s) return vg.nz - 1;
    int kb = -1, L = 0, R = vg.nz;
    while (L <= R) {
        const int M = (R + L) / 2;
        if (-depth >= vg.ztot[L] && -depth < vg.ztot[M]) R = M;
        else L = M;
        if (R - L == 1) { kb = L; break; }
    }
    return kb;
}

__device__ __forceinline__ double2 clampvel(double2 v, double rmaxvel) {
    const double ry = rmaxvel * 1.013;
    return v2(fmin(fmax(v.x, -rmaxvel), rmaxvel), fmin(fmax(v.y, -ry), ry));
}

// Grid-wide barrier for cooperative launches on one 32-bit word that starts at zero.  Each
// block adds 1, except block 0, which adds 2^31 - (blocks - 1): the increments of one round sum
// to 2^31, so the word's top bit flips exactly when the last block arrives and the low bits are
// back at zero for the next round.  A waiting block polls until the top bit differs from the one
// its own add returned: one atomic per block and no reset store.  The wait is bounded: after
// `polls` polls (kWaitPolls, about 2 s, unless the context sets another bound) the block records
// ERR_BARRIER_TIMEOUT and returns false, and every caller then leaves the kernel (the host clears
// the word and the flag after reporting the timeout).
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(unsigned* bar, int32_t* err, long long polls) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
        const bool first = (blockIdx.x | blockIdx.y | blockIdx.z) == 0;
        const unsigned inc = first ? (0x80000000u - (nb - 1u)) : 1u;
        __threadfence();
        const unsigned old = atomicAdd(bar, inc);
        long long spins = 0;
        while (((ld_acquire_u32(bar) ^ old) & 0x80000000u) == 0u) {
            if (++spins > 4096) __nanosleep(128);
            if (spins > polls) { atomicOr(err, ERR_BARRIER_TIMEOUT); break; }
            if ((spins & 255) == 0 && (*((volatile int32_t*)err) & ERR_BARRIER_TIMEOUT)) break;
        }
        __threadfence();
    }
    __syncthreads();
    return (*((volatile int32_t*)err) & ERR_BARRIER_TIMEOUT) == 0;
}

// Deterministic sum of n doubles by one warp: lane-strided partial sums, then a fixed
// xor-shuffle tree; every lane returns the same value.
__device__ __forceinline__ double warp_sum_fixed(const double* v, int n, int lane) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += v[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

inline int grid_for(int n, int block, int max_blocks) {
    int g = (n + block - 1) / block;
    if (g > max_blocks) g = max_blocks;
    return g < 1 ? 1 : g;
}
// grid of a stream kernel with launch shape s over n entities
inline int grid_of(long long n, const LaunchShape& s, int nsm) {
    long long g = (n + s.block - 1) / s.block;
    const long long cap = (long long)nsm * s.per_sm;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

}  // namespace gs
