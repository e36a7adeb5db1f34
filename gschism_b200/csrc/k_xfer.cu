// Field exchange between the device state (internal space-filling-curve order, level-major,
// members concatenated) and the caller's reference numbering, done on the device so that a
// field crosses PCIe/C2C as one contiguous copy through pinned staging memory.
//
// A field of one member is a block of nt x nl slices (tracers x levels) of n entities with nc
// components.  gather writes the reference-ordered block out[t][k][perm[i]][c] from the device
// slices src[t][k][off + i][c] (stride N per slice); scatter is the inverse.  Element kinds: 0 =
// double, 1 = int32, 2 = uint8 on the device exchanged as int32.  With remap set (backtracked
// element ids), non-negative int32 values v are replaced by remap[v].
#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

__global__ void k_gather(const void* __restrict__ src, void* __restrict__ dst, int kind, int n, int N, int off,
                         int nslices, int nc, const int32_t* __restrict__ perm, const int32_t* __restrict__ remap) {
    const long long total = (long long)nslices * n;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const long long sl = g / n;
        const int i = (int)(g - sl * n);
        const size_t s = ((size_t)sl * N + off + i) * nc;
        const size_t o = ((size_t)sl * n + perm[i]) * nc;
        if (kind == 0) {
            const double* a = (const double*)src;
            double* b = (double*)dst;
            for (int c = 0; c < nc; c++) b[o + c] = a[s + c];
        } else if (kind == 1) {
            const int32_t* a = (const int32_t*)src;
            int32_t* b = (int32_t*)dst;
            for (int c = 0; c < nc; c++) {
                int32_t v = a[s + c];
                if (remap && v >= 0) v = remap[v];
                b[o + c] = v;
            }
        } else {
            const uint8_t* a = (const uint8_t*)src;
            int32_t* b = (int32_t*)dst;
            for (int c = 0; c < nc; c++) b[o + c] = (int32_t)a[s + c];
        }
    }
}

__global__ void k_scatter(const void* __restrict__ src, void* __restrict__ dst, int kind, int n, int N, int off,
                          int nslices, int nc, const int32_t* __restrict__ perm) {
    const long long total = (long long)nslices * n;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const long long sl = g / n;
        const int i = (int)(g - sl * n);
        const size_t d = ((size_t)sl * N + off + i) * nc;
        const size_t o = ((size_t)sl * n + perm[i]) * nc;
        if (kind == 0) {
            const double* a = (const double*)src;
            double* b = (double*)dst;
            for (int c = 0; c < nc; c++) b[d + c] = a[o + c];
        } else if (kind == 1) {
            const int32_t* a = (const int32_t*)src;
            int32_t* b = (int32_t*)dst;
            for (int c = 0; c < nc; c++) b[d + c] = a[o + c];
        } else {
            const int32_t* a = (const int32_t*)src;
            uint8_t* b = (uint8_t*)dst;
            for (int c = 0; c < nc; c++) b[d + c] = (uint8_t)a[o + c];
        }
    }
}

void launch_gather(const void* src, void* dst, int kind, int n, int N, int off, int nslices, int nc,
                   const int32_t* perm, const int32_t* remap, cudaStream_t st, int nsm) {
    const long long total = (long long)nslices * n;
    const int grid = (int)std::min<long long>((total + 255) / 256, (long long)nsm * 8);
    k_gather<<<grid > 0 ? grid : 1, 256, 0, st>>>(src, dst, kind, n, N, off, nslices, nc, perm, remap);
}

void launch_scatter(const void* src, void* dst, int kind, int n, int N, int off, int nslices, int nc,
                    const int32_t* perm, cudaStream_t st, int nsm) {
    const long long total = (long long)nslices * n;
    const int grid = (int)std::min<long long>((total + 255) / 256, (long long)nsm * 8);
    k_scatter<<<grid > 0 ? grid : 1, 256, 0, st>>>(src, dst, kind, n, N, off, nslices, nc, perm);
}

}  // namespace gs
