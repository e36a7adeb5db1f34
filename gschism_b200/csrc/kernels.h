// Launch entry points of the gschism_b200 kernels (host side).
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "gs_internal.h"

namespace gs {

struct VG;

struct JcgArgs {
    int n, precision;
    const int32_t *indptr, *indices;     // CSR rows, or SELL-32 slices when sell is set
    const int2* sell;
    const double* A;
    const float* A32;                    // D^-1 A in FP32
    const double *b, *invD;
    double *x, *r, *z, *q, *p0, *p1;
    float* ir32;                         // kIrVectors * n floats
    const float* diag32;                 // matrix diagonal in FP32
    unsigned* bar;
    int32_t* err;
    double rtol;
    int maxiter, check_every;
    double inner_rtol;
    int inner_maxiter;
    long long wait_polls;                // bound of every wait of the solve (0: kWaitPolls)
    int stall_member;                    // recovery tests: this member's arrivals never complete (-1: off)
};
struct JcgWork;
cudaError_t jcg_work_alloc(JcgWork*& w, const std::vector<int>& row0, const std::vector<int>& rows, bool sell,
                           cudaStream_t st, const JcgTiling& tiling = JcgTiling());
void jcg_work_free(JcgWork* w);
cudaError_t jcg_launch(const JcgArgs& a, JcgWork* w, cudaStream_t st, int nsm);
cudaError_t jcg_read_iters(JcgWork* w, std::vector<int>& iters, std::vector<int>& outer, cudaStream_t st);
// ERR_JCG_NOT_CONVERGED of the last solve (cleared at every launch); 0 or the flag
cudaError_t jcg_read_status(JcgWork* w, int32_t* flags, cudaStream_t st);
int32_t* jcg_iters_device(JcgWork* w);

// k_xfer.cu: one member's field between device slices and a reference-ordered block
void launch_gather(const void* src, void* dst, int kind, int n, int N, int off, int nslices, int nc,
                   const int32_t* perm, const int32_t* remap, cudaStream_t st, int nsm);
void launch_scatter(const void* src, void* dst, int kind, int n, int N, int off, int nslices, int nc,
                    const int32_t* perm, cudaStream_t st, int nsm);

// k_elev.cu
void launch_clock_set(const Dev& d, const Phys& P, int it, cudaStream_t st);
void launch_clock_advance(const Dev& d, const Phys& P, cudaStream_t st);
void launch_elev_prepare(const Dev& d, const Phys& P, bool vortex, cudaStream_t st, int nsm, const LaunchTable& L);
void launch_assemble(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L);
void launch_update_elev(const Dev& d, const VG& vg, cudaStream_t st, int nsm);
// k_btrack.cu
void launch_btrack(const Dev& d, const Phys& P, const VG& vg, cudaStream_t st, int nsm, const LaunchTable& L);
// k_mom.cu
void launch_momentum(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L);
void launch_vvel(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L);
// k_transport.cu
cudaError_t launch_transport(const Dev& d, const Phys& P, double dt, cudaStream_t st, int nsm, const LaunchTable& L);
// per-tracer mass of elements [e0, e1): part holds kMassBlocks * ntr * 2 doubles, out ntr
cudaError_t launch_tracer_mass(const Dev& d, const Phys& P, int e0, int e1, double* part, double* out,
                               cudaStream_t st);
// k_levels.cu
void launch_geometry(const Dev& d, const Phys& P, cudaStream_t st, int nsm);
void launch_levels(const Dev& d, const Phys& P, const VG& vg, int it, cudaStream_t st, int nsm, const LaunchTable& L);
void launch_nodal_vel(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L);
// largest block each stream kernel of the launch table can run with (its compiled limits)
int btrack_max_threads();
int elev_max_threads(int kernel);
int mom_max_threads(int kernel);
int levels_max_threads(int kernel);
int transport_max_threads(int ntr);

}  // namespace gs
