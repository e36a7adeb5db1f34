// Wet/dry state and vertical levels (ul0* kernels, meshdata.cu:5521-5762) and nodal
// velocities (meshdata.cu:5765-5929).  The reference accumulates nodal velocities with FP64
// atomics in thread order; here every node gathers over its counter-clockwise element ball,
// so the sums are deterministic.
#include <algorithm>

#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

__global__ void k_lev_nodes(Dev d, VG vg) {
    // ul0UpdateZCoords, meshdata.cu:5521-5547
    const int NP = d.NP;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        const double depth = d.depth[i], eta = d.eta2[i];
        const int kb = node_kb(vg, depth);
        d.kb[i] = kb;
        for (int k = kb; k < vg.nvrt; k++) d.z[(size_t)k * NP + i] = compz(vg, eta, depth, kb, k);
        d.nwas[i] = d.ndry[i];
        d.ndry[i] = 1;
    }
}

__global__ void k_lev_elems(Dev d, Phys P) {
    // ul0ComputeDryElements, meshdata.cu:5550-5593
    const int NE = d.NE, NP = d.NP, nvrt = P.nvrt;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NE; e += gridDim.x * blockDim.x) {
        const int n0 = d.en[e], n1 = d.en[NE + e], n2 = d.en[2 * NE + e];
        const bool dry = (d.eta2[n0] + d.depth[n0] <= P.h0) || (d.eta2[n1] + d.depth[n1] <= P.h0) ||
                         (d.eta2[n2] + d.depth[n2] <= P.h0);
        d.edry[e] = dry;
        if (dry) { d.kbe[e] = 0; continue; }
        const int k1 = d.kb[n0], k2 = d.kb[n1], k3 = d.kb[n2];
        int kb = k1 < k2 ? k1 : k2;
        kb = kb < k3 ? kb : k3;
        d.kbe[e] = kb;
        for (int k = kb; k < nvrt; k++) {
            double zz = d.z[(size_t)(k > k1 ? k : k1) * NP + n0] + d.z[(size_t)(k > k2 ? k : k2) * NP + n1] +
                        d.z[(size_t)(k > k3 ? k : k3) * NP + n2];
            zz /= 3;
            d.ez[(size_t)k * NE + e] = zz;
        }
    }
}

__global__ void k_lev_nodes_dry(Dev d) {
    // ul0ComputeDryNodes, meshdata.cu:5596-5613
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.NP; i += gridDim.x * blockDim.x) {
        uint8_t dry = 1;
        for (int q = d.nne_s[i]; q < d.nne_s[i + 1]; q++)
            if (!d.edry[d.nne[q]]) { dry = 0; break; }
        d.ndry[i] = dry;
    }
}

__global__ void k_lev_rewet_nodes(Dev d, Phys P) {
    // ul0UpdateRewettedNodes, meshdata.cu:5616-5676 (every tracer is averaged, not only T and S)
    const int NP = d.NP, nvrt = P.nvrt, ntr = P.ntr;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        if (!(!d.ndry[i] && d.nwas[i])) continue;
        for (int k = 0; k < nvrt; k++) {
            double ux = 0.0, uy = 0.0, uw = 0.0, ts[kMaxTracers];
            for (int t = 0; t < ntr; t++) ts[t] = 0.0;
            int icount = 0;
            for (int a = d.nnp_s[i]; a < d.nnp_s[i + 1]; a++) {
                const int nb = d.nnp[a];
                if (d.nwas[nb]) continue;
                icount++;
                const double2 u = d.u2[(size_t)k * NP + nb];
                ux += u.x; uy += u.y; uw += d.w2[(size_t)k * NP + nb];
                for (int t = 0; t < ntr; t++) ts[t] += d.tr[((size_t)t * nvrt + k) * NP + nb];
            }
            if (icount > 0) {
                const double inv = 1.0 / icount;
                d.u2[(size_t)k * NP + i] = v2(inv * ux, inv * uy);
                d.w2[(size_t)k * NP + i] = inv * uw;
                for (int t = 0; t < ntr; t++) d.tr[((size_t)t * nvrt + k) * NP + i] = inv * ts[t];
            } else {
                d.u2[(size_t)k * NP + i] = v2(0.0, 0.0);
                d.w2[(size_t)k * NP + i] = 0.0;
            }
        }
    }
}

__global__ void k_lev_sides(Dev d, Phys P, int it) {
    // ul0UpdateSides, meshdata.cu:5679-5745
    const int NS = d.NS, NP = d.NP, NE = d.NE, nvrt = P.nvrt;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < NS; s += gridDim.x * blockDim.x) {
        const int e0 = d.se[s], e1 = d.se[NS + s];
        const bool wet = !d.edry[e0] || (e1 >= 0 && !d.edry[e1]);
        const int a = d.sn[s], b = d.sn[NS + s];
        const int kb1 = d.kb[a], kb2 = d.kb[b];
        if (!wet) { d.kbs[s] = 0; continue; }
        const int kb = kb1 < kb2 ? kb1 : kb2;
        d.kbs[s] = kb;
        for (int k = 0; k < kb; k++) d.zc[(size_t)k * NS + s] = 0.0;
        const bool rewet = (it != 0) && d.sdry[s];
        for (int k = kb; k < nvrt; k++) {
            d.zc[(size_t)k * NS + s] = 0.5 * (d.z[(size_t)(k > kb1 ? k : kb1) * NP + a] + d.z[(size_t)(k > kb2 ? k : kb2) * NP + b]);
            if (rewet) {
                double2 ut = v2(0.0, 0.0);
                int icount = 0;
                for (int j = 0; j < 2; j++) {
                    const int e = (j == 0) ? e0 : e1;
                    if (e < 0) continue;
                    for (int jj = 0; jj < 3; jj++) {
                        const int ss = d.es[jj * NE + e];
                        if (d.sdry[ss]) continue;
                        icount++;
                        ut = ut + d.su2[(size_t)k * NS + ss];
                    }
                }
                d.su2[(size_t)k * NS + s] = (icount > 0) ? ut / icount : v2(0.0, 0.0);
            }
        }
    }
}

__global__ void k_lev_sides_dry(Dev d) {
    // ul0UpdateSides2, meshdata.cu:5748-5762
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < d.NS; s += gridDim.x * blockDim.x) {
        const int e0 = d.se[s], e1 = d.se[d.NS + s];
        const bool wet = !d.edry[e0] || (e1 >= 0 && !d.edry[e1]);
        d.sdry[s] = !wet;
    }
}

__global__ void k_nodal_vel(Dev d, Phys P) {
    // zeroNodalVelocities .. computeNodalHorizontalVelocities2 (indvel <= 0, triangles)
    const int NP = d.NP, NE = d.NE, NS = d.NS, nvrt = P.nvrt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        const int q0 = d.nne_s[i], q1 = d.nne_s[i + 1];
        const int kbn = d.kb[i];
        double asum = 0.0;
        for (int q = q0; q < q1; q++) asum += d.area[d.nne[q]];
        const double inv = 1.0 / asum;
        for (int k = 0; k < nvrt; k++) {
            double w = 0.0;
            if (k >= kbn) {
                for (int q = q0; q < q1; q++) {
                    const int e = d.nne[q];
                    w += d.ew[(size_t)k * NE + e] * d.area[e];
                }
                w = inv * w;
            }
            d.w2[(size_t)k * NP + i] = w;
        }
        int count = 0;
        if (!d.ndry[i])
            for (int q = q0; q < q1; q++) count += d.edry[d.nne[q]] ? 0 : 1;
        for (int k = 0; k < nvrt; k++) {
            double2 u = v2(0.0, 0.0);
            if (count > 0 && k >= kbn) {
                for (int q = q0; q < q1; q++) {
                    const int e = d.nne[q];
                    if (d.edry[e] || k < d.kbe[e]) continue;
                    const int j = d.nne_loc[q];
                    const int s1 = d.es[j * NE + e], s2 = d.es[((j + 1) % 3) * NE + e], s3 = d.es[((j + 2) % 3) * NE + e];
                    const double2 ue = clampvel((d.su2[(size_t)k * NS + s2] + d.su2[(size_t)k * NS + s3]) -
                                                d.su2[(size_t)k * NS + s1], P.rmaxvel);
                    u = u + ue;
                }
                u = u * (1.0 / count);
            }
            d.u2[(size_t)k * NP + i] = u;
        }
    }
}

// eqstate, src/kernels/eqstate.h:12-52 (ieos_type = 0, ieos_pres = 0): UNESCO 1980 one-atmosphere
// density (Millero & Poisson 1981), T and S clamped to their validity range [-2, 40] C, [0, 42] psu
__device__ __forceinline__ double eqstate(double T, double S) {
    T = fmax(-2.0, fmin(T, 40.0));
    S = fmax(0.0, fmin(S, 42.0));
    const double sqrtS = sqrt(S);
    const double rhow = 999.842594 + T * (6.793952e-2 + T * (-9.095290e-3 + T * (1.001685e-4
                        + T * (-1.120083e-6 + T * 6.536332e-9))));
    const double A = 8.24493e-1 + T * (-4.0899e-3 + T * (7.6438e-5 + T * (-8.2467e-7 + T * 5.3875e-9)));
    const double B = -5.72466e-3 + T * (1.0227e-4 + T * (-1.6546e-6));
    return rhow + S * (A + B * sqrtS + 4.8314e-4 * S);
}

// computeNodeDensity / computeElemDensity, meshdata.cu:6776-6812: density of every (entity, level)
// from the first two tracers (T, S); -99 on dry entities.  One thread per (entity, level): the
// tracer slices [t][k][n] are read with unit stride.
__global__ void k_density(const double* __restrict__ tr, const uint8_t* __restrict__ dry, double* __restrict__ rho,
                          int n, int nvrt) {
    const long long total = (long long)n * nvrt;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(g % n);
        rho[g] = dry[i] ? -99.0 : eqstate(tr[g], tr[total + g]);
    }
}

void launch_density(const Dev& d, const Phys& P, cudaStream_t st, int nsm) {
    if (!d.rho_n || P.ntr < 2) return;
    const long long tn = (long long)d.NP * P.nvrt, te = (long long)d.NE * P.nvrt;
    k_density<<<(int)std::min<long long>((tn + 255) / 256, (long long)nsm * 8), 256, 0, st>>>(d.tr, d.ndry, d.rho_n,
                                                                                            d.NP, P.nvrt);
    k_density<<<(int)std::min<long long>((te + 255) / 256, (long long)nsm * 8), 256, 0, st>>>(d.etr, d.edry, d.rho_e,
                                                                                            d.NE, P.nvrt);
}

void launch_levels(const Dev& d, const Phys& P, const VG& vg, int it, cudaStream_t st, int nsm, const LaunchTable& L) {
    const LaunchShape& s = L.k[LK_LEVELS];
    const int b = s.block;
    k_lev_nodes<<<grid_of(d.NP, s, nsm), b, 0, st>>>(d, vg);
    k_lev_elems<<<grid_of(d.NE, s, nsm), b, 0, st>>>(d, P);
    k_lev_nodes_dry<<<grid_of(d.NP, s, nsm), b, 0, st>>>(d);
    if (it != 0) k_lev_rewet_nodes<<<grid_of(d.NP, s, nsm), b, 0, st>>>(d, P);
    k_lev_sides<<<grid_of(d.NS, s, nsm), b, 0, st>>>(d, P, it);
    k_lev_sides_dry<<<grid_of(d.NS, s, nsm), b, 0, st>>>(d);
    launch_density(d, P, st, nsm);
}

void launch_nodal_vel(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L) {
    const LaunchShape& s = L.k[LK_NODAL_VEL];
    k_nodal_vel<<<grid_of(d.NP, s, nsm), s.block, 0, st>>>(d, P);
}

int levels_max_threads(int kernel) {
    cudaFuncAttributes a{};
    if (kernel == LK_NODAL_VEL)
        return cudaFuncGetAttributes(&a, k_nodal_vel) == cudaSuccess ? a.maxThreadsPerBlock : 0;
    if (kernel != LK_LEVELS) return 0;
    const void* fs[] = {(const void*)k_lev_nodes, (const void*)k_lev_elems, (const void*)k_lev_nodes_dry,
                        (const void*)k_lev_rewet_nodes, (const void*)k_lev_sides, (const void*)k_lev_sides_dry};
    int m = 1024;
    for (const void* f : fs) {
        if (cudaFuncGetAttributes(&a, f) != cudaSuccess) return 0;
        m = std::min(m, a.maxThreadsPerBlock);
    }
    return m;
}

}  // namespace gs
