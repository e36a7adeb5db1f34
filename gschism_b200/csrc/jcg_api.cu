// Stand-alone JCG on a caller-filled CSR matrix: the drop-in for PCGSolverMultiGPU
// (src/solver/pcg_solver.py:538-1148), one partition per device.  The caller writes the CSR
// arrays and b into solver-owned device buffers (as the reference's populate kernels write
// into csr_data/csr_indices/csr_indptr), then calls gs_jcg_solve_csr.
#include <string>
#include <vector>

#include "dev_common.cuh"
#include "kernels.h"

using namespace gs;

struct gs_jcg {
    int n = 0, nnz = 0, precision = GS_FP64, dev = 0, nsm = 148;
    cudaStream_t st = nullptr;
    int32_t *indptr = nullptr, *indices = nullptr;
    double *A = nullptr, *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p0 = nullptr,
           *p1 = nullptr, *invD = nullptr, *x0 = nullptr, *x1 = nullptr, *x2 = nullptr, *scratch = nullptr;
    float *A32 = nullptr, *ir32 = nullptr, *diag32 = nullptr;
    unsigned *bar = nullptr;
    int32_t* err = nullptr;
    JcgWork* w = nullptr;
    std::vector<void*> allocs;
    std::string msg;
};

namespace gs {

__global__ void k_jcg_prep(int n, const int32_t* indptr, const int32_t* indices, const double* A, double* invD,
                           float* diag32, float* A32, double* x, const double* x0, const double* x1,
                           const double* x2) {
    // computeInvDiag (pcg_solver.py:933-938) and extrapolateGuess (:881-886); with A32 set, also
    // the FP32 rows of D^-1 A and the FP32 diagonal of the refinement solve
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double dg = 0.0;
        for (int a = indptr[i]; a < indptr[i + 1]; a++)
            if (indices[a] == i) dg = A[a];
        const double inv = 1.0 / dg;
        invD[i] = inv;
        if (A32) {
            diag32[i] = (float)dg;
            for (int a = indptr[i]; a < indptr[i + 1]; a++) A32[a] = (float)(A[a] * inv);
        }
        x[i] = 3.0 * x0[i] - 3.0 * x1[i] + x2[i];
    }
}

__global__ void k_roll(int n, const double* x, double* x0, double* x1, double* x2) {
    // rollHistory, pcg_solver.py:941-947
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x2[i] = x1[i]; x1[i] = x0[i]; x0[i] = x[i];
    }
}

__global__ void k_resid2(int n, const int32_t* indptr, const int32_t* indices, const double* A, const double* x,
                         const double* b, double* out) {
    // single block: |b - A x|^2 and |b|^2 in a fixed order
    __shared__ double sh[2][32];
    double rr = 0.0, bb = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int a = indptr[i]; a < indptr[i + 1]; a++) s += A[a] * x[indices[a]];
        const double r = b[i] - s;
        rr += r * r; bb += b[i] * b[i];
    }
    for (int o = 16; o > 0; o >>= 1) { rr += __shfl_xor_sync(0xffffffffu, rr, o); bb += __shfl_xor_sync(0xffffffffu, bb, o); }
    if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = rr; sh[1][threadIdx.x >> 5] = bb; }
    __syncthreads();
    if (threadIdx.x < 32) {
        rr = threadIdx.x < (blockDim.x >> 5) ? sh[0][threadIdx.x] : 0.0;
        bb = threadIdx.x < (blockDim.x >> 5) ? sh[1][threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) { rr += __shfl_xor_sync(0xffffffffu, rr, o); bb += __shfl_xor_sync(0xffffffffu, bb, o); }
        if (threadIdx.x == 0) { out[0] = rr; out[1] = bb; }
    }
}

}  // namespace gs

template <typename T>
static cudaError_t jalloc(gs_jcg* s, T*& p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) { cudaMemsetAsync(q, 0, (n ? n : 1) * sizeof(T), s->st); s->allocs.push_back(q); p = (T*)q; }
    return e;
}

extern "C" {

gs_status gs_jcg_create(int n, int nnz, int precision, int device, gs_jcg** out) {
    if (n <= 0 || nnz < n || !out || (precision != GS_FP64 && precision != GS_FP32_IR)) return GS_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GS_ERR_CUDA;
    gs_jcg* s = new gs_jcg();
    s->n = n; s->nnz = nnz; s->precision = precision; s->dev = device;
    cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
#define J(f, k) if (e == cudaSuccess) e = jalloc(s, s->f, k)
    J(indptr, n + 1); J(indices, nnz); J(A, nnz); J(A32, nnz);
    J(b, n); J(x, n); J(r, n); J(z, n); J(q, n); J(p0, n); J(p1, n); J(invD, n); J(x0, n); J(x1, n); J(x2, n);
    J(scratch, 2); J(ir32, (size_t)kIrVectors * n); J(diag32, n);
    J(bar, 2); J(err, 1);
#undef J
    if (e == cudaSuccess) e = jcg_work_alloc(s->w, std::vector<int>{0}, std::vector<int>{n}, false, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) {
        gs_status st = (e == cudaErrorMemoryAllocation) ? GS_ERR_OOM : GS_ERR_CUDA;
        gs_jcg_destroy(s);
        return st;
    }
    *out = s;
    return GS_OK;
}

gs_status gs_jcg_buffers(gs_jcg* s, int32_t** indptr, int32_t** indices, double** data, double** b, double** x) {
    if (!s) return GS_ERR_ARG;
    if (indptr) *indptr = s->indptr;
    if (indices) *indices = s->indices;
    if (data) *data = s->A;
    if (b) *b = s->b;
    if (x) *x = s->x;
    return GS_OK;
}

gs_status gs_jcg_solve_csr(gs_jcg* s, double rtol, int maxiter, int check_every, int* iters) {
    // PCGSolverMultiGPU.solve, pcg_solver.py:1075-1124
    if (!s || maxiter < 1) return GS_ERR_ARG;
    cudaSetDevice(s->dev);
    const int n = s->n;
    const int g = grid_for(n, 256, s->nsm * 8);
    float* a32 = (s->precision == GS_FP32_IR) ? s->A32 : nullptr;
    k_jcg_prep<<<g, 256, 0, s->st>>>(n, s->indptr, s->indices, s->A, s->invD, s->diag32, a32, s->x, s->x0, s->x1,
                                     s->x2);
    JcgArgs a{};
    a.n = n; a.precision = s->precision;
    a.indptr = s->indptr; a.indices = s->indices; a.A = s->A; a.A32 = s->A32; a.b = s->b; a.invD = s->invD;
    a.x = s->x; a.r = s->r; a.z = s->z; a.q = s->q; a.p0 = s->p0; a.p1 = s->p1;
    a.ir32 = s->ir32;
    a.diag32 = s->diag32;
    a.bar = s->bar; a.err = s->err;
    a.rtol = rtol; a.maxiter = maxiter; a.check_every = check_every < 1 ? 1 : check_every;
    a.inner_rtol = 0.1; a.inner_maxiter = 400;
    a.wait_polls = kWaitPolls; a.stall_member = -1;
    cudaError_t e = jcg_launch(a, s->w, s->st, s->nsm);
    if (e != cudaSuccess) { s->msg = cudaGetErrorString(e); return GS_ERR_CUDA; }
    k_roll<<<g, 256, 0, s->st>>>(n, s->x, s->x0, s->x1, s->x2);
    std::vector<int> it, outer;
    e = jcg_read_iters(s->w, it, outer, s->st);
    if (e != cudaSuccess) { s->msg = cudaGetErrorString(e); return GS_ERR_CUDA; }
    int32_t flags = 0;
    cudaMemcpyAsync(&flags, s->err, 4, cudaMemcpyDeviceToHost, s->st);
    cudaStreamSynchronize(s->st);
    if (iters) *iters = it[0];
    if (flags & ERR_BARRIER_TIMEOUT) {
        // the barrier word is left mid-round; both words are cleared so the next solve starts clean
        cudaMemsetAsync(s->bar, 0, sizeof(unsigned), s->st);
        cudaMemsetAsync(s->err, 0, sizeof(int32_t), s->st);
        cudaStreamSynchronize(s->st);
        s->msg = "device barrier timed out";
        return GS_ERR_TIMEOUT;
    }
    return GS_OK;
}

gs_status gs_jcg_check(gs_jcg* s, double* relres) {
    // checkSolution, pcg_solver.py:1127-1143
    if (!s || !relres) return GS_ERR_ARG;
    k_resid2<<<1, 1024, 0, s->st>>>(s->n, s->indptr, s->indices, s->A, s->x, s->b, s->scratch);
    double h[2] = {0.0, 0.0};
    cudaError_t e = cudaMemcpyAsync(h, s->scratch, 16, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) { s->msg = cudaGetErrorString(e); return GS_ERR_CUDA; }
    const double rn = sqrt(h[0]), bn = sqrt(h[1]);
    *relres = bn > 0 ? rn / bn : rn;
    return GS_OK;
}

gs_status gs_jcg_destroy(gs_jcg* s) {
    if (!s) return GS_ERR_ARG;
    if (s->st) { cudaStreamSynchronize(s->st); cudaStreamDestroy(s->st); }
    jcg_work_free(s->w);
    for (void* p : s->allocs) cudaFree(p);
    delete s;
    return GS_OK;
}

const char* gs_jcg_last_error(const gs_jcg* s) { return s ? s->msg.c_str() : "null solver"; }

}  // extern "C"
