// Elevation phase of the step: boundary values, side terms, element ghat1 and the per-node
// assembly of the wave-equation row (meshdata.cu:3182-3474, 4276-4476, 4615-4725, 6183-6424).
//
// Assembly is a node-centred gather: one thread owns one matrix row and walks the node's
// elements in counter-clockwise order, accumulating the row in registers in the same order
// as the reference's addToSparseMatrix (no atomics, deterministic).  Roll-up of eta, the
// essential boundary conditions and the JCG set-up values are fused into the same pass.
#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

// Step clock on the device (computeTimeRamps, mdh:2036-2077): step index, time and the tanh
// ramp, so the step's launch sequence has no per-step host arguments and replays as a graph.
__device__ __forceinline__ void clock_at(Dev& d, const Phys& P, int it) {
    const double time = it * P.dt;
    d.clk[0] = it;
    d.clk[1] = time;
    d.clk[2] = (P.dramp > 0.0) ? tanh(2.0 * time / 86400.0 / P.dramp) : 1.0;
}
__global__ void k_clock_set(Dev d, Phys P, int it) { clock_at(d, P, it); }
__global__ void k_clock_advance(Dev d, Phys P) { clock_at(d, P, (int)d.clk[0] + 1); }

// Member of node i (mem_np0[m] <= i < mem_np0[m + 1]).
__device__ __forceinline__ int member_of_node(const Dev& d, int i) {
    int lo = 0, hi = d.nmem;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (d.mem_np0[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// A member's own clock: its step is the context's step minus the member's start step
// (gs_set_member_start; 0 unless the member was admitted later), with the time and ramp of that
// step, so a member admitted into a running context sees the clock of a run of its own.  A
// member whose start lies ahead of the context's step is parked: time 0, ramp 0 (no tide, no
// storm).
__device__ __forceinline__ void member_clock(const Dev& d, const Phys& P, int m, double& time, double& ramp) {
    const double ls = d.clk[0] - d.mem_start[m];
    if (ls < 0.0) { time = 0.0; ramp = 0.0; return; }
    const int it = (int)ls;
    time = it * P.dt;
    ramp = (P.dramp > 0.0) ? tanh(2.0 * time / 86400.0 / P.dramp) : 1.0;
}

__global__ void k_elev_bc(Dev d, Phys P) {
    // computeElevationBoundaryConditions, mdc:4276-4339 (iettype 3: tidal harmonics)
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < d.NB; b += gridDim.x * blockDim.x) {
        const int i = d.bn_node[b];
        double time, ramp;
        member_clock(d, P, member_of_node(d, i), time, ramp);
        const int iettype = d.bn_ietype[b];
        const double eic = 0.0;
        const double r_eic = (1.0 - ramp) * eic;
        const double r_eth = ramp * 0.0;
        double r_eta1_bar = 0.0;
        if (iettype == 3 || iettype == 5) {
            const int nb = d.bn_nbfr[b];
            for (int f = 0; f < nb; f++) {
                const double amig = d.bn_amig[b * kMaxBfr + f];
                const double efa = d.bn_efa[b * kMaxBfr + f];
                const double emo = d.bn_emo[b * kMaxBfr + f];
                const int ncyc = (int)(amig * time / (2.0 * 3.14159265358979323846));
                const double arg = amig * time - (2.0 * 3.14159265358979323846) * ncyc + d.bn_face[b * kMaxBfr + f] - efa;
                r_eta1_bar += ramp * d.bn_ff[b * kMaxBfr + f] * emo * cos(arg);
            }
        }
        double v = 0.0;
        if (iettype == 1 || iettype == 2 || iettype == 4) v = r_eic + r_eth;
        else if (iettype == 3) v = r_eic + r_eta1_bar;
        else if (iettype == 5) v = r_eic + r_eta1_bar + r_eth;
        d.elbc[i] = v;
    }
}

__global__ void k_side_prep(Dev d, Phys P) {
    // computeVerticallyIntegratedVelocity (mdc:4459-4476) and
    // computeVegetationAndDragParameters (mdc:4615-4725, iveg = 0); then, for every side of a wet
    // element, the side's three terms of computeElemAverageGhat (mdc:6183-6424): its
    // backtracked-velocity column integral and its stress, drag and Coriolis terms, so that the
    // element pass adds three stored terms per side instead of integrating both columns of every
    // side once per adjacent element.  Side-parallel: each level's reads are coalesced.
    const int nvrt = P.nvrt, NS = d.NS;
    const double dt = P.dt;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < NS; s += gridDim.x * blockDim.x) {
        double2 U = v2(0.0, 0.0);
        double hhat = 0.0, chi = 0.0, chi2 = 0.0;
        const int e0 = d.se[s], e1 = d.se[NS + s];
        const bool ghat_side = (e0 >= 0 && !d.edry[e0]) || (e1 >= 0 && !d.edry[e1]);
        const int kb = d.kbs[s];
        const bool is2d = (kb == nvrt - 2);
        const bool wet = !d.sdry[s];
        // one pass over the column: the depth integral of the velocity (wet sides) and of the
        // backtracked velocity (3-D sides of wet elements) over the same level pairs
        double2 Ustar = v2(0.0, 0.0);
        const bool col_u = wet, col_b = ghat_side && !is2d;
        if (col_u || col_b) {
            double zlo = d.zc[(size_t)kb * NS + s];
            double2 ulo = col_u ? d.su2[(size_t)kb * NS + s] : v2(0.0, 0.0);
            double2 blo = col_b ? d.btu[(size_t)kb * NS + s] : v2(0.0, 0.0);
            for (int k = kb + 1; k < nvrt; k++) {
                const double zhi = d.zc[(size_t)k * NS + s];
                if (col_u) {
                    const double2 uhi = d.su2[(size_t)k * NS + s];
                    const double2 uc = (ulo + uhi) * 0.5;
                    U = U + uc * (zhi - zlo);
                    ulo = uhi;
                }
                if (col_b) {
                    const double2 bhi = d.btu[(size_t)k * NS + s];
                    const double2 w2 = ((bhi + blo) / 2.0) * (zhi - zlo);
                    Ustar = Ustar + w2;
                    blo = bhi;
                }
                zlo = zhi;
            }
        }
        const int a = d.sn[s], b = d.sn[NS + s];
        const double htot = 0.5 * (d.eta2[a] + d.eta2[b]) + 0.5 * (d.depth[a] + d.depth[b]);
        if (wet) {
            const double2 bt = d.btu[(size_t)(kb + 1) * NS + s];
            const double vmag1 = sqrt(bt.x * bt.x + bt.y * bt.y);
            const double cd = 0.5 * (d.drag[a] + d.drag[b]);
            chi2 = cd * vmag1;
            chi = chi2;
            if (kb == nvrt - 2) {
                const double fricH = htot + chi2 * P.dt;
                hhat = htot * htot / fricH;
            } else {
                hhat = htot - chi * P.dt;
                if (P.ihhat == 1) hhat = fmax(0.0, hhat);
            }
        }
        d.U[s] = U; d.hhat[s] = hhat; d.chi[s] = chi; d.chi2[s] = chi2;
        if (!ghat_side) continue;
        const double cff1 = is2d ? hhat / htot : 1.0;
        const double cff2 = is2d ? 0.0 : 1.0;
        if (is2d) {
            const double dz = d.zc[(size_t)(nvrt - 1) * NS + s] - d.zc[(size_t)(nvrt - 2) * NS + s];
            Ustar = Ustar + d.btu[(size_t)(nvrt - 1) * NS + s] * dz;
        }
        const double2 tau = (v2(d.tau[2 * a], d.tau[2 * a + 1]) + v2(d.tau[2 * b], d.tau[2 * b + 1])) * 0.5;
        const double2 ubstar = d.btu[(size_t)(kb + 1) * NS + s];
        const double cor = d.cori[s];
        const double2 F = U * cor;
        const double2 fb = d.su2[(size_t)(kb + 1) * NS + s] * cor;
        d.sgh[s] = Ustar * cff1;
        d.sgh[NS + s] = ubstar * (chi * dt * cff2) + tau * (dt * cff1);
        d.sgh[2 * (size_t)NS + s] = F * (cff1 * dt) - fb * (cff2 * chi * dt * dt);
    }
}

__global__ void k_ghat(Dev d, Phys P) {
    // computeElemAverageGhat, mdc:6183-6424 (ics = 1, iveg = 0, ibc = 1, no horizontal
    // viscosity, atmospheric pressure or tidal potential): per side j of the element, in the
    // reference's order, g += Ustar_j cff1_j; g -= (drag + stress)_j; g += (Coriolis)_j, with the
    // side terms made by k_side_prep.
    const int NS = d.NS, NE = d.NE;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NE; e += gridDim.x * blockDim.x) {
        double2 g = v2(0.0, 0.0);
        if (!d.edry[e]) {
            for (int j = 0; j < 3; j++) {
                const int s = d.es[j * NE + e];
                g = g + d.sgh[s];
                g = g - d.sgh[NS + s];
                g = g + d.sgh[2 * (size_t)NS + s];
            }
            g = g * (1.0 / 3);
        }
        d.ghat[e] = g;
    }
}

__global__ void k_assemble(Dev d, Phys P) {
    // setupCoefficientMatrixAndRHS (mdc:3182-3474) for one row per thread, then rollUpElevation
    // (mdc:3538) and setEssentialBC (mdc:4400-4446) on the same row, then the per-solve set-up
    // of PCGSolverMultiGPU.solve (b, invD, parabolic guess; pcg_solver.py:881-938).
    const int NE = d.NE, NP = d.NP;
    const double dt = P.dt, th = P.thetai;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NP; i += gridDim.x * blockDim.x) {
        const int q0 = d.nne_s[i], q1 = d.nne_s[i + 1];
        const int s0 = d.nnp_s[i], nn = d.nnp_s[i + 1] - s0;
        if (nn > kMaxDeg) { atomicOr(d.err, ERR_DEGREE); continue; }
        double vals[kMaxDeg];
        for (int p = 0; p < nn; p++) vals[p] = 0.0;
        double diag = 0.0, qel = 0.0;
        for (int q = q0; q < q1; q++) {
            const int e = d.nne[q];
            const int id1 = d.nne_loc[q];
            const int n0 = d.en[e], n1 = d.en[NE + e], n2 = d.en[2 * NE + e];
            const int sa = d.es[e], sb = d.es[NE + e], sc = d.es[2 * NE + e];
            const double grav3 = (P.grav + P.grav + P.grav + 0.0) / 3;
            const double hhatb = (d.hhat[sa] + d.hhat[sb] + d.hhat[sc] + 0.0) / 3;
            const double area = d.area[e];
            const double2 U = (((d.U[sa] + d.U[sb]) + d.U[sc]) + v2(0.0, 0.0)) / 3;
            const double2 gp1 = d.gphi[id1 * NE + e];
            const double I41 = dot2(gp1, U);
            const double I42 = dot2(gp1, d.ghat[e]);
            qel += dt * area * ((1 - th) * I41 + th * I42);
            const double fric = grav3 * th * (1.0 - th) * dt * dt * hhatb;
            const int ids[3] = {n0, n1, n2};
            const int ia = ids[id1], ib = ids[(id1 + 1) % 3], ic = ids[(id1 + 2) % 3];
            const double2 p0 = v2(d.x[ia], d.y[ia]);
            const double2 p1 = v2(d.x[ib], d.y[ib]);
            const double2 p2 = v2(d.x[ic], d.y[ic]);
            const double ipp_ii = (1.0 / 6.0) * area, ipp_ij = (1.0 / 12.0) * area, ipp_ik = (1.0 / 12.0) * area;
            const double g_ii = ((1.0 / 4.0) / area) * dot2(p2 - p1, p2 - p1);
            const double g_ij = ((1.0 / 4.0) / area) * dot2(p2 - p1, p0 - p2);
            const double g_ik = -g_ii - g_ij;
            const double c = grav3 * th * th * dt * dt * hhatb;
            const int pos = q - q0;
            const int pos2 = (pos + 1 == nn) ? 0 : pos + 1;
            diag += ipp_ii + c * g_ii;
            vals[pos] += ipp_ij + c * g_ij;
            vals[pos2] += ipp_ik + c * g_ik;
            const double wet = d.edry[e] ? 0.0 : 1.0;
            for (int l = 0; l < 3; l++) {
                const int nl = ids[l];
                const double ipp = ((id1 == l) ? (2.0 / 12.0) : (1.0 / 12.0)) * area;
                const double igpgp = area * dot2(d.gphi[id1 * NE + e], d.gphi[l * NE + e]);
                const double eta = d.eta2[nl];
                qel += (eta + 0.0) * ipp - eta * fric * igpgp * wet;
            }
            qel += (dt / 3) * 0.0;
        }
        if (d.nbnd[i] >= 0) {
            const int sl[2] = {d.sb1[i], d.sb2[i]};
            for (int l = 0; l < 2; l++) {
                const int s = sl[l];
                if (s < 0 || d.sdry[s]) continue;
                const double Unbar = d.U[s].x * d.snx[s] + d.U[s].y * d.sny[s];
                qel -= 0.5 * (1.0 - th) * dt * d.len[s] * Unbar;
            }
        }
        // roll-up and essential boundary conditions
        d.eta1[i] = d.eta2[i];
        if (d.nbnd[i] >= 0 && d.ess[i]) {
            for (int p = 0; p < nn; p++) vals[p] = 0.0;
            diag = 1.0;
            qel = d.elbc[i];
        } else {
            for (int p = 0; p < nn; p++) {
                const int nb = d.nnp[s0 + p];
                if (d.nbnd[nb] >= 0 && d.ess[nb]) {
                    qel -= vals[p] * d.elbc[nb];
                    vals[p] = 0.0;
                }
            }
        }
        // FP64 row, and the row of D^-1 A in FP32 for the refinement solve
        const double inv = 1.0 / diag;
        for (int p = 0; p < nn; p++) {
            const int at = d.nbr_slot[s0 + p];
            d.A[at] = vals[p];
            d.A32[at] = (float)(vals[p] * inv);
        }
        d.A[d.diag_slot[i]] = diag;
        d.A32[d.diag_slot[i]] = 1.0f;
        d.qel[i] = qel;
        d.b[i] = qel;
        d.invD[i] = inv;
        d.diag32[i] = (float)diag;
        d.xs[i] = 3.0 * d.xh0[i] - 3.0 * d.xh1[i] + d.xh2[i];
    }
}

__global__ void k_update_elev(Dev d, VG vg) {
    // scatterXToMesh + rollHistory (pcg_solver.py:941-954), updateElevation (mdc:4449-4456)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.NP; i += gridDim.x * blockDim.x) {
        const double x = d.xs[i];
        d.xh2[i] = d.xh1[i]; d.xh1[i] = d.xh0[i]; d.xh0[i] = x;
        d.eta2[i] = x;
        if (!d.ndry[i]) d.kb[i] = node_kb(vg, d.depth[i]);
    }
}

// Storm forcing: kinematic surface stress of a radial vortex on a straight track (gs_vortex in the
// C ABI) for the nodes of members that have one; other members keep their stress.
__global__ void k_vortex_tau(Dev d, Phys P) {
    const double rho0 = P.rho0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.NP; i += gridDim.x * blockDim.x) {
        const int lo = member_of_node(d, i);
        const double* v = d.vort + (size_t)kVortexParams * lo;
        if (v[8] == 0.0) continue;
        double time, ramp;
        member_clock(d, P, lo, time, ramp);
        const double x0 = v[0], y0 = v[1], hd = v[2], sp = v[3], vmax = v[4], rmax = v[5], B = v[6], rho_air = v[7];
        const double ch = cos(hd), sh = sin(hd);
        const double cx = x0 + sp * time * ch, cy = y0 + sp * time * sh;
        const double dx = d.x[i] - cx, dy = d.y[i] - cy;
        const double r = sqrt(dx * dx + dy * dy);
        double W = 0.0, tx = 0.0, ty = 0.0;
        if (r > 1.0) {
            const double q = pow(rmax / r, B);
            W = vmax * sqrt(q * exp(1.0 - q));
            tx = -dy / r; ty = dx / r;
        }
        const double f = W / vmax;
        const double wx = W * tx + f * sp * ch, wy = W * ty + f * sp * sh;
        const double ws = sqrt(wx * wx + wy * wy);
        double cd = 1e-3 * (0.75 + 0.067 * ws);
        if (cd > 3e-3) cd = 3e-3;
        const double k = ramp * rho_air / rho0 * cd * ws;
        d.tau[2 * (size_t)i] = k * wx;
        d.tau[2 * (size_t)i + 1] = k * wy;
    }
}

void launch_clock_set(const Dev& d, const Phys& P, int it, cudaStream_t st) { k_clock_set<<<1, 1, 0, st>>>(d, P, it); }
void launch_clock_advance(const Dev& d, const Phys& P, cudaStream_t st) { k_clock_advance<<<1, 1, 0, st>>>(d, P); }

void launch_elev_prepare(const Dev& d, const Phys& P, bool vortex, cudaStream_t st, int nsm, const LaunchTable& L) {
    if (vortex) k_vortex_tau<<<grid_for(d.NP, 256, nsm * 8), 256, 0, st>>>(d, P);
    if (d.NB > 0) k_elev_bc<<<grid_for(d.NB, 128, nsm * 4), 128, 0, st>>>(d, P);
    const LaunchShape &sp = L.k[LK_SIDE_PREP], &gh = L.k[LK_GHAT];
    k_side_prep<<<grid_of(d.NS, sp, nsm), sp.block, 0, st>>>(d, P);
    k_ghat<<<grid_of(d.NE, gh, nsm), gh.block, 0, st>>>(d, P);
}

void launch_assemble(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L) {
    const LaunchShape& s = L.k[LK_ASSEMBLE];
    k_assemble<<<grid_of(d.NP, s, nsm), s.block, 0, st>>>(d, P);
}

int elev_max_threads(int kernel) {
    cudaFuncAttributes a{};
    cudaError_t e = cudaErrorInvalidValue;
    if (kernel == LK_SIDE_PREP) e = cudaFuncGetAttributes(&a, k_side_prep);
    else if (kernel == LK_GHAT) e = cudaFuncGetAttributes(&a, k_ghat);
    else if (kernel == LK_ASSEMBLE) e = cudaFuncGetAttributes(&a, k_assemble);
    return e == cudaSuccess ? a.maxThreadsPerBlock : 0;
}

void launch_update_elev(const Dev& d, const VG& vg, cudaStream_t st, int nsm) {
    k_update_elev<<<grid_for(d.NP, 256, nsm * 16), 256, 0, st>>>(d, vg);
}

}  // namespace gs
