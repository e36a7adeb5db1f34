// Tracer transport, first-order upwind (computeTransport, schism_step.py:78-93; kernels
// meshdata.cu:6493-6665, 6739-6774, 6842-6863).
//
// The sub-cycling loop runs inside one cooperative launch: every member keeps its own
// remaining time and sub-step on the device (the reference reads minTransportDt back to the
// host once per sub-step).  The minimum admissible sub-step of a member is reduced with an
// integer atomicMin on the bit pattern of non-negative doubles, which is order-independent.
// The implicit vertical advection of an element is fused into its member's last sub-step.
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

__device__ void vertical_upwind(const Dev& d, const Phys& P, int e, double dt) {
    // verticalAdvectionUpdate, meshdata.cu:6611-6665 (upwind: phi = 0)
    const int NE = d.NE, nvrt = P.nvrt, ntr = P.ntr;
    const int kb = d.kbe[e];
    const int nEq = nvrt - (kb + 1);
    double alow[kMaxLevels], bdia[kMaxLevels], cupp[kMaxLevels], gam[kMaxLevels], u[kMaxLevels];
    for (int k = kb + 1; k < nvrt; k++) {
        const int kin = k - (kb + 1);
        alow[kin] = 0.0; cupp[kin] = 0.0; bdia[kin] = 0.0;
        const double dbv = dt / evol(d, e, k - 1);
        bdia[kin] += 1.0;
        const double qk = d.Qv[(size_t)k * NE + e], qm = d.Qv[(size_t)(k - 1) * NE + e];
        if (k != nvrt - 1 && qk < 0.0) { const double tmp = dbv * fabs(qk); cupp[kin] -= tmp; bdia[kin] += tmp; }
        if (k - 1 != kb && qm > 0.0) { const double tmp = dbv * fabs(qm); alow[kin] -= tmp; bdia[kin] += tmp; }
    }
    for (int t = 0; t < ntr; t++) {
        double* tr = d.etr + (size_t)t * nvrt * NE;
        double bet = bdia[0];
        u[0] = (tr[(size_t)(kb + 1) * NE + e] * 1.0) / bet;
        for (int j = 1; j < nEq; j++) {
            gam[j] = cupp[j - 1] / bet;
            bet = bdia[j] - alow[j] * gam[j];
            u[j] = (tr[(size_t)(kb + 1 + j) * NE + e] * 1.0 - alow[j] * u[j - 1]) / bet;
        }
        for (int j = nEq - 2; j >= 0; j--) u[j] = u[j] - gam[j + 1] * u[j + 1];
        for (int k = kb + 1; k < nvrt; k++) tr[(size_t)k * NE + e] = u[k - (kb + 1)];
        for (int k = 0; k <= kb; k++) tr[(size_t)k * NE + e] = u[0];
    }
}

__global__ void __launch_bounds__(256) k_transport(Dev d, Phys P, TrArgs T) {
    const int NE = d.NE, NS = d.NS, nvrt = P.nvrt, ntr = P.ntr, nmem = d.nmem;
    const int G = gridDim.x * blockDim.x;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long seed = (unsigned long long)__double_as_longlong(1e34);
    for (int m = gid; m < nmem; m += G) {
        T.rem[m] = T.dt; T.rem[nmem + m] = T.dt;
        T.mindt[m] = seed; T.mindt[nmem + m] = seed;
        T.nsub[m] = 0;
    }
    if (gid == 0) *T.active = (unsigned)nmem;
    if (!grid_sync(d.bar, d.err)) return;
    for (int sub = 0; sub < T.maxsub; sub++) {
        if (*((volatile unsigned*)T.active) == 0u) break;
        const int par = sub & 1, nxt = par ^ 1;
        // horizontalAdvectionPrepare (meshdata.cu:6493-6559): snapshot, inflow, max sub-step
        for (int e = gid; e < NE; e += G) {
            const int m = d.elem_member[e];
            if (!(((volatile double*)T.rem)[par * nmem + m] > 0.0) || d.edry[e]) continue;
            const int kb = d.kbe[e];
            for (int t = 0; t < ntr; t++)
                for (int k = 0; k < nvrt; k++) {
                    const size_t ix = ((size_t)t * nvrt + k) * NE + e;
                    d.prev[ix] = d.etr[ix];
                }
            double md = kHuge;
            for (int k = kb + 1; k < nvrt; k++) {
                double in = 0.0;
                for (int j = 0; j < 3; j++) {
                    const int s = d.es[j * NE + e];
                    if (k <= d.kbs[s]) continue;
                    const int e0 = d.se[s], e1 = d.se[NS + s];
                    const int nb = (e0 == e) ? e1 : e0;
                    if (nb < 0 || d.edry[nb]) continue;
                    const double fq = d.Qh[(size_t)k * NS + s];
                    const bool influx = ((double)d.ssgn[j * NE + e] * fq) < 0.0;
                    if (d.sbt[s] == 1 || !influx) continue;
                    in += fabs(fq);
                }
                const double pd = (in == 0.0) ? kHuge : evol(d, e, k - 1) / in * (1.0 - 1.0e-6);
                md = fmin(md, pd);
            }
            d.maxDt[e] = md;
            atomicMin(&T.mindt[par * nmem + m], (unsigned long long)__double_as_longlong(md));
        }
        if (!grid_sync(d.bar, d.err)) return;
        // horizontalAdvectionUpdate (meshdata.cu:6561-6609) with dtb = min(remaining, min maxDt)
        for (int e = gid; e < NE; e += G) {
            const int m = d.elem_member[e];
            const double rem = ((volatile double*)T.rem)[par * nmem + m];
            if (!(rem > 0.0)) continue;
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
            for (int k = kb + 1; k < nvrt; k++) {
                const double vol = evol(d, e, k - 1);
                const double dbv = dtb / vol;
                double adv[kMaxTracers];
                for (int t = 0; t < ntr; t++) adv[t] = d.prev[((size_t)t * nvrt + k) * NE + e];
                for (int j = 0; j < 3; j++) {
                    const int s = d.es[j * NE + e];
                    if (k <= d.kbs[s]) continue;
                    const double fq = d.Qh[(size_t)k * NS + s];
                    const double sQ = (double)d.ssgn[j * NE + e] * fq;
                    if (sQ >= 0.0) continue;
                    const int e0 = d.se[s], e1 = d.se[NS + s];
                    const int nb = (e0 == e) ? e1 : e0;
                    const double coef = dbv * fabs(fq);
                    if (nb >= 0 && !d.edry[nb]) {
                        for (int t = 0; t < ntr; t++)
                            adv[t] += coef * (d.prev[((size_t)t * nvrt + k) * NE + nb] - d.prev[((size_t)t * nvrt + k) * NE + e]);
                    } else if (d.sbt[s] == 2) {
                        for (int t = 0; t < ntr; t++) {
                            const double cout = adv[t];
                            adv[t] += coef * (cout - d.prev[((size_t)t * nvrt + k) * NE + e]);
                        }
                    }
                }
                for (int t = 0; t < ntr; t++) d.etr[((size_t)t * nvrt + k) * NE + e] = adv[t];
            }
            for (int t = 0; t < ntr; t++) {
                const double v = d.etr[((size_t)t * nvrt + kb + 1) * NE + e];
                for (int k = 0; k <= kb; k++) d.etr[((size_t)t * nvrt + k) * NE + e] = v;
            }
            if (last) vertical_upwind(d, P, e, T.dt);
        }
        if (!grid_sync(d.bar, d.err)) return;
    }
}

__global__ void k_nodal_tracer(Dev d, Phys P) {
    // nodalTracerUpdate, meshdata.cu:6739-6774 (node-centred gather, no atomics)
    const int NP = d.NP, NE = d.NE, nvrt = P.nvrt, ntr = P.ntr, ivrt = nvrt - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        if (d.ndry[i]) continue;
        const int q0 = d.nne_s[i], q1 = d.nne_s[i + 1];
        for (int k = 0; k < nvrt; k++) {
            double sum[kMaxTracers];
            for (int t = 0; t < ntr; t++) sum[t] = 0.0;
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
                for (int t = 0; t < ntr; t++) {
                    const double* tr = d.etr + (size_t)t * nvrt * NE;
                    sum[t] += A * ((1.0 - zrat) * tr[(size_t)kHi * NE + e] + zrat * tr[(size_t)kLo * NE + e]);
                }
                sumA += A;
            }
            if (sumA == 0.0) continue;
            const double inv = 1.0 / sumA;
            for (int t = 0; t < ntr; t++) d.tr[((size_t)t * nvrt + k) * NP + i] = inv * sum[t];
        }
    }
}

cudaError_t launch_transport(const Dev& d, const Phys& P, double dt, cudaStream_t st, int nsm) {
    TrArgs T;
    T.rem = d.mem_rem; T.mindt = d.mem_mindt; T.nsub = d.mem_nsub; T.active = (unsigned*)(d.mem_mindt + 2 * d.nmem);
    T.dt = dt; T.maxsub = 100000;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_transport, 256, 0);
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    int grid = std::min(nsm * per_sm, (d.NE + 255) / 256);
    if (grid < 1) grid = 1;
    Dev dd = d;
    Phys pp = P;
    void* args[] = {&dd, &pp, &T};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_transport, dim3(grid), dim3(256), args, 0, st);
    if (e != cudaSuccess) return e;
    k_nodal_tracer<<<grid_for(d.NP, 128, nsm * 16), 128, 0, st>>>(d, P);
    return cudaGetLastError();
}

}  // namespace gs
