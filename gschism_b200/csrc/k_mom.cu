// Momentum and vertical velocity (meshdata.cu:5045-5454, 5978-6103) plus the horizontal
// advective fluxes of transport (computeHorizAdvecFluxes, :6461-6491), fused per side: one
// thread owns one side column, solves its vertical tridiagonal system with the intermediate
// values kept in the level-major output arrays (coalesced across sides, no local memory) and
// writes u2 and Qh level by level.
#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

__device__ __forceinline__ double2 side_grad_eta(const Dev& d, const Phys& P, int s, const double* f, int which) {
    // Side::grad2 (meshdata.cu:1330-1373): average of the gradients of the wet neighbours;
    // which = 1 tests element dryness (isDry), 2 tests the updated depth (isDry2)
    const int NE = d.NE, NS = d.NS;
    double2 g = v2(0.0, 0.0);
    int count = 0;
    for (int l = 0; l < 2; l++) {
        const int e = d.se[l * NS + s];
        if (e < 0) continue;
        const int n0 = d.en[e], n1 = d.en[NE + e], n2 = d.en[2 * NE + e];
        bool ok;
        if (which == 1) ok = !d.edry[e];
        else ok = !((d.eta2[n0] + d.depth[n0] <= P.h0) || (d.eta2[n1] + d.depth[n1] <= P.h0) ||
                    (d.eta2[n2] + d.depth[n2] <= P.h0));
        if (!ok) continue;
        const double2 g0 = d.gphi[e], g1 = d.gphi[NE + e], g2 = d.gphi[2 * NE + e];
        const double gx = f[n0] * g0.x + f[n1] * g1.x + f[n2] * g2.x;
        const double gy = f[n0] * g0.y + f[n1] * g1.y + f[n2] * g2.y;
        g = g + v2(gx, gy);
        count++;
    }
    if (count > 0) g = g * (1.0 / count);
    return g;
}

// Horizontal advective flux through side s between levels k-1 and k (computeHorizAdvecFluxes)
__device__ __forceinline__ double side_flux(double len, double nx, double ny, double zk, double zkm1, double2 uk,
                                            double2 ukm1) {
    const double area = len * (zk - zkm1);
    const double vn1 = nx * uk.x + ny * uk.y;
    const double vn2 = nx * ukm1.x + ny * ukm1.y;
    return area * (0.5 * (vn1 + vn2));
}

// applyMomentumBC on a land side: free slip (islip = 0) keeps the tangential component
__device__ __forceinline__ double2 slip(double2 u, int8_t bt, double nx, double ny) {
    if (bt != 1) return u;
    const double2 t = v2(-ny, nx), nn = v2(nx, ny);
    const double vnorm = 0.0;
    const double vtan = dot2(u, t);
    return t * vtan - nn * vnorm;
}

__global__ void __launch_bounds__(128, 8) k_momentum(Dev d, Phys P) {
    const int NS = d.NS, nvrt = P.nvrt;
    const double dt = P.dt, th = P.thetai;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < NS; s += gridDim.x * blockDim.x) {
        double2* u2 = d.su2;
        const double2* btu = d.btu;
        double* Qh = d.Qh;
        if (d.sdry[s]) {
            for (int k = 0; k < nvrt; k++) { u2[(size_t)k * NS + s] = v2(0.0, 0.0); Qh[(size_t)k * NS + s] = -1.0e34; }
            continue;
        }
        // computeHorGradientAtSide (pressure and tidal potential gradients are zero)
        const double2 gE1 = side_grad_eta(d, P, s, d.eta1, 1);
        const double2 gE2 = side_grad_eta(d, P, s, d.eta2, 2);
        d.gE1[s] = gE1; d.gE2[s] = gE2;
        const int kb = d.kbs[s];
        const int a = d.sn[s], b = d.sn[NS + s];
        const double grav3 = 0.5 * (P.grav + P.grav);
        const double cor = d.cori[s];
        const double2 tau2 = (v2(d.tau[2 * a], d.tau[2 * a + 1]) + v2(d.tau[2 * b], d.tau[2 * b + 1])) * 0.5;
        const double cd = 0.5 * (d.drag[a] + d.drag[b]);
        const int8_t bt = d.sbt[s];
        const double nx = d.snx[s], ny = d.sny[s], len = d.len[s];
        const bool two_d = (kb == nvrt - 2);
        double2 vel2d = v2(0.0, 0.0);   // 2D column: one velocity for every level
        double2 rtop = v2(0.0, 0.0);    // 3D column: the top row's value after the forward sweep
        if (two_d) {
            const double htot = d.zc[(size_t)(nvrt - 1) * NS + s] - d.zc[(size_t)kb * NS + s];
            const double hhat = d.hhat[s];
            const double2 un = u2[(size_t)(nvrt - 1) * NS + s];
            const double2 corT = v2(un.y, -un.x) * cor;
            const double2 inner = (corT + tau2 / htot) - (gE1 * (1 - th) + gE2 * th) * grav3;
            const double2 hat_gam = btu[(size_t)(nvrt - 1) * NS + s] + inner * dt;
            vel2d = clampvel((hat_gam * hhat) / htot, P.rmaxvel);
        } else {
            // assembly of row k (solveMomentumEquations, meshdata.cu:5076-5354) and the forward
            // sweep of tridag_sch<2> (meshdata.cu:3664-3716); the sweep's values replace u2[k]
            // (the old u2[k] stays in a register for row k+1), the eliminated super-diagonal goes
            // to Qh[k] until the fluxes overwrite it
            const double2 grad2D = (gE2 * th + gE1 * (1.0 - th)) * grav3;
            const double dfz = 0.5 * (P.dfv0 + P.dfv0);
            double2 ukm1 = v2(0.0, 0.0), bkm1 = v2(0.0, 0.0);
            double2 uk = u2[(size_t)(kb + 1) * NS + s], bk = btu[(size_t)(kb + 1) * NS + s];
            double zkm1 = d.zc[(size_t)kb * NS + s], zk = d.zc[(size_t)(kb + 1) * NS + s];
            double bet = 0.0, cprev = 0.0;
            double2 rprev = v2(0.0, 0.0);
            for (int k = kb + 1; k < nvrt; k++) {
                const bool top = (k == nvrt - 1);
                const double2 ukp1 = top ? v2(0.0, 0.0) : u2[(size_t)(k + 1) * NS + s];
                const double2 bkp1 = top ? v2(0.0, 0.0) : btu[(size_t)(k + 1) * NS + s];
                const double zkp1 = top ? 0.0 : d.zc[(size_t)(k + 1) * NS + s];
                double alow = 0.0, cupp = 0.0, bdia = 0.0;
                const double cff1 = 1.0;
                const double dz_0 = zk - zkm1;
                const double dz_1 = !top ? zkp1 - zk : 0.0;
                if (!top) {
                    const double tmp = dt * dfz / dz_1;
                    cupp += cff1 * dz_1 / 6.0 - tmp;
                    bdia += cff1 * dz_1 / 3.0 + tmp;
                }
                if (k > kb + 1) {
                    const double tmp = dt * dfz / dz_0;
                    alow += cff1 * dz_0 / 6.0 - tmp;
                    bdia += cff1 * dz_0 / 3.0 + tmp;
                } else {
                    bdia += dt * d.chi2[s];
                }
                double dz = 0.0;
                dz += dz_1;
                if (k > kb + 1) dz += dz_0;
                double2 r = grad2D * (-(0.5 * dz) * dt);
                if (!top) {
                    const double2 uu = uk * 2.0 + ukp1;
                    const double2 ct = v2(uu.y, -uu.x) * cor;
                    const double2 in = (bk * 2.0 + bkp1) + ct * dt;
                    r = r + in * (dz_1 / 6.0);
                } else {
                    r = r + tau2 * dt;
                }
                if (k > kb + 1) {
                    const double2 uu = uk * 2.0 + ukm1;
                    const double2 ct = v2(uu.y, -uu.x) * cor;
                    const double2 in = (bk * 2.0 + bkm1) + ct * dt;
                    r = r + in * (dz_0 / 6.0);
                }
                if (k == kb + 1) {
                    bet = bdia;
                    r = v2(r.x / bet, r.y / bet);
                } else {
                    const double gam = cprev / bet;
                    bet = bdia - alow * gam;
                    r = v2((r.x - alow * rprev.x) / bet, (r.y - alow * rprev.y) / bet);
                    Qh[(size_t)k * NS + s] = gam;
                }
                u2[(size_t)k * NS + s] = r;
                rprev = r;
                cprev = cupp;
                ukm1 = uk; uk = ukp1; bkm1 = bk; bk = bkp1; zkm1 = zk; zk = zkp1;
            }
            rtop = rprev;
        }
        // top-down: back substitution (3D), clamp, the bottom level's value, free slip on land
        // sides, and the stores of u2 and of the fluxes Qh (land sides carry zero flux)
        double2 r = rtop, uabove = v2(0.0, 0.0);
        double zabove = 0.0;
        for (int k = nvrt - 1; k >= kb; k--) {
            double2 u;
            if (k > kb) {
                if (two_d) {
                    u = vel2d;
                } else {
                    if (k < nvrt - 1) {
                        const double gam = Qh[(size_t)(k + 1) * NS + s];
                        const double2 x = u2[(size_t)k * NS + s];
                        r = v2(x.x - gam * r.x, x.y - gam * r.y);
                    }
                    u = clampvel(r, P.rmaxvel);
                }
            } else {
                // ucol[kb]: the level above when there is no bottom drag, else 0 (3D) / the 2D value
                if (cd == 0.0) u = two_d ? vel2d : clampvel(r, P.rmaxvel);
                else u = two_d ? vel2d : v2(0.0, 0.0);
            }
            u = slip(u, bt, nx, ny);
            u2[(size_t)k * NS + s] = u;
            const double zk = d.zc[(size_t)k * NS + s];
            if (k < nvrt - 1)
                Qh[(size_t)(k + 1) * NS + s] = (bt == 1) ? 0.0 : side_flux(len, nx, ny, zabove, zk, uabove, u);
            uabove = u;
            zabove = zk;
        }
        Qh[(size_t)kb * NS + s] = -1.0e34;
        for (int k = 0; k < kb; k++) { u2[(size_t)k * NS + s] = v2(0.0, 0.0); Qh[(size_t)k * NS + s] = -1.0e34; }
    }
}

__global__ void __launch_bounds__(128, 6) k_vvel(Dev d, Phys P) {
    // computeVerticalVelocity, meshdata.cu:5978-6103 (imm = 0, triangles, ics = 1)
    const int NE = d.NE, NS = d.NS, NP = d.NP, nvrt = P.nvrt;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NE; e += gridDim.x * blockDim.x) {
        if (d.edry[e]) {
            for (int l = 0; l < nvrt; l++) d.ew[(size_t)l * NE + e] = 0.0;
            continue;
        }
        const int kb = d.kbe[e];
        const int n0 = d.en[e], n1 = d.en[NE + e], n2 = d.en[2 * NE + e];
        const int sd[3] = {d.es[e], d.es[NE + e], d.es[2 * NE + e]};
        const double2 g0 = d.gphi[e], g1 = d.gphi[NE + e], g2 = d.gphi[2 * NE + e];
        const double ghx = d.depth[n0] * g0.x + d.depth[n1] * g1.x + d.depth[n2] * g2.x;
        const double ghy = d.depth[n0] * g0.y + d.depth[n1] * g1.y + d.depth[n2] * g2.y;
        double2 ub = v2(0.0, 0.0);
        for (int j = 0; j < 3; j++) ub = ub + d.su2[(size_t)d.kbs[sd[j]] * NS + sd[j]];
        ub = (ub + v2(0.0, 0.0)) / 3;
        for (int l = 0; l < kb; l++) d.ew[(size_t)l * NE + e] = 0.0;
        d.ew[(size_t)kb * NE + e] = 0.0 + (-(ghx * ub.x + ghy * ub.y));
        double bottomFlux = 0.0;
        d.Qv[(size_t)kb * NE + e] = 0.0;
        const double x0 = d.x[n0], y0 = d.y[n0], x1 = d.x[n1], y1 = d.y[n1], x2 = d.x[n2], y2 = d.y[n2];
        const int kb0 = d.kb[n0], kb1 = d.kb[n1], kb2 = d.kb[n2];
        const double az = 2.0 * d.area[e];
        for (int l = kb; l < nvrt - 1; l++) {
            const int k = l + 1;
            const double z0 = d.z[(size_t)(k > kb0 ? k : kb0) * NP + n0];
            const double z1 = d.z[(size_t)(k > kb1 ? k : kb1) * NP + n1];
            const double z2 = d.z[(size_t)(k > kb2 ? k : kb2) * NP + n2];
            const double n20x = x2 - x0, n20y = y2 - y0, n20z = z2 - z0;
            const double n10x = x1 - x0, n10y = y1 - y0, n10z = z1 - z0;
            const double ax = n10y * n20z - n20y * n10z;
            const double ay = n20x * n10z - n10x * n20z;
            const double len = sqrt(ax * ax + ay * ay + az * az);
            const double tA = 0.5 * len;
            const double inv = 1.0 / len;
            const double tnx = ax * inv, tny = ay * inv, tnz = az * inv;
            double sideFlux = 0.0;
            double2 um = v2(0.0, 0.0);
            for (int j = 0; j < 3; j++) {
                const int s = sd[j];
                const int kbs = d.kbs[s];
                const int ka = (l + 1 > kbs) ? l + 1 : kbs, kc = (l > kbs) ? l : kbs;
                const double2 ut = d.su2[(size_t)ka * NS + s], ubt = d.su2[(size_t)kc * NS + s];
                const double2 u2c = (ut + ubt) * 0.5;
                const double sideArea = d.len[s] * (d.zc[(size_t)ka * NS + s] - d.zc[(size_t)kc * NS + s]);
                const double sign = (double)d.ssgn[j * NE + e];
                sideFlux += sign * (u2c.x * d.snx[s] + u2c.y * d.sny[s]) * sideArea;
            }
            for (int j = 0; j < 3; j++) {
                const int s = sd[j];
                const int kk = (l + 1 > d.kbs[s]) ? l + 1 : d.kbs[s];
                um = um + d.su2[(size_t)kk * NS + s];
            }
            um = (um + v2(0.0, 0.0)) / 3;
            const double topFlux = -sideFlux - bottomFlux;
            d.Qv[(size_t)(l + 1) * NE + e] = topFlux;
            const double topH = (um.x * tnx + um.y * tny) * tA;
            d.ew[(size_t)(l + 1) * NE + e] = (topFlux - topH) / (tnz * tA);
            bottomFlux = -topFlux;
        }
    }
}

void launch_momentum(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L) {
    const LaunchShape& s = L.k[LK_MOMENTUM];
    k_momentum<<<grid_of(d.NS, s, nsm), s.block, 0, st>>>(d, P);
}

void launch_vvel(const Dev& d, const Phys& P, cudaStream_t st, int nsm, const LaunchTable& L) {
    const LaunchShape& s = L.k[LK_VVEL];
    k_vvel<<<grid_of(d.NE, s, nsm), s.block, 0, st>>>(d, P);
}

int mom_max_threads(int kernel) {
    cudaFuncAttributes a{};
    cudaError_t e = cudaErrorInvalidValue;
    if (kernel == LK_MOMENTUM) e = cudaFuncGetAttributes(&a, k_momentum);
    else if (kernel == LK_VVEL) e = cudaFuncGetAttributes(&a, k_vvel);
    return e == cudaSuccess ? a.maxThreadsPerBlock : 0;
}

}  // namespace gs
