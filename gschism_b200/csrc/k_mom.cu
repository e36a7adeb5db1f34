// Momentum and vertical velocity (meshdata.cu:5045-5454, 5978-6103) plus the horizontal
// advective fluxes of transport (computeHorizAdvecFluxes, :6461-6491), fused per side: one
// thread owns one side column, solves its vertical tridiagonal system in registers/local
// memory and writes u2 and Qh level by level (level-major arrays, coalesced across sides).
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

__global__ void __launch_bounds__(128) k_momentum(Dev d, Phys P) {
    const int NS = d.NS, nvrt = P.nvrt;
    const double dt = P.dt, th = P.thetai;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < NS; s += gridDim.x * blockDim.x) {
        double2* u2 = d.su2;
        const double2* btu = d.btu;
        if (d.sdry[s]) {
            for (int k = 0; k < nvrt; k++) { u2[(size_t)k * NS + s] = v2(0.0, 0.0); d.Qh[(size_t)k * NS + s] = -1.0e34; }
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
        double2 ucol[kMaxLevels];
        if (kb == nvrt - 2) {
            const double htot = d.zc[(size_t)(nvrt - 1) * NS + s] - d.zc[(size_t)kb * NS + s];
            const double hhat = d.hhat[s];
            const double2 un = u2[(size_t)(nvrt - 1) * NS + s];
            const double2 corT = v2(un.y, -un.x) * cor;
            const double2 inner = (corT + tau2 / htot) - (gE1 * (1 - th) + gE2 * th) * grav3;
            const double2 hat_gam = btu[(size_t)(nvrt - 1) * NS + s] + inner * dt;
            const double2 vel = clampvel((hat_gam * hhat) / htot, P.rmaxvel);
            for (int k = 0; k < nvrt; k++) ucol[k] = vel;
        } else {
            double alow[kMaxLevels], cupp[kMaxLevels], bdia[kMaxLevels], gam[kMaxLevels];
            double2 rh[kMaxLevels];
            const double2 grad2D = (gE2 * th + gE1 * (1.0 - th)) * grav3;
            const double dfz = 0.5 * (P.dfv0 + P.dfv0);
            for (int k = kb + 1; k < nvrt; k++) {
                const int kin = k - (kb + 1);
                alow[kin] = 0.0; cupp[kin] = 0.0; bdia[kin] = 0.0;
                const double cff1 = 1.0;
                const double dz_0 = d.zc[(size_t)k * NS + s] - d.zc[(size_t)(k - 1) * NS + s];
                const double dz_1 = (k < nvrt - 1) ? d.zc[(size_t)(k + 1) * NS + s] - d.zc[(size_t)k * NS + s] : 0.0;
                if (k < nvrt - 1) {
                    const double tmp = dt * dfz / dz_1;
                    cupp[kin] += cff1 * dz_1 / 6.0 - tmp;
                    bdia[kin] += cff1 * dz_1 / 3.0 + tmp;
                }
                if (k > kb + 1) {
                    const double tmp = dt * dfz / dz_0;
                    alow[kin] += cff1 * dz_0 / 6.0 - tmp;
                    bdia[kin] += cff1 * dz_0 / 3.0 + tmp;
                } else {
                    bdia[kin] += dt * d.chi2[s];
                }
                double dz = 0.0;
                dz += dz_1;
                if (k > kb + 1) dz += dz_0;
                double2 r = grad2D * (-(0.5 * dz) * dt);
                const double2 uk = u2[(size_t)k * NS + s];
                const double2 bk = btu[(size_t)k * NS + s];
                if (k < nvrt - 1) {
                    const double2 uu = uk * 2.0 + u2[(size_t)(k + 1) * NS + s];
                    const double2 ct = v2(uu.y, -uu.x) * cor;
                    const double2 in = (bk * 2.0 + btu[(size_t)(k + 1) * NS + s]) + ct * dt;
                    r = r + in * (dz_1 / 6.0);
                } else {
                    r = r + tau2 * dt;
                }
                if (k > kb + 1) {
                    const double2 uu = uk * 2.0 + u2[(size_t)(k - 1) * NS + s];
                    const double2 ct = v2(uu.y, -uu.x) * cor;
                    const double2 in = (bk * 2.0 + btu[(size_t)(k - 1) * NS + s]) + ct * dt;
                    r = r + in * (dz_0 / 6.0);
                }
                rh[kin] = r;
            }
            // tridag_sch<2>, meshdata.cu:3664-3716
            const int n = nvrt - kb - 1;
            double bet = bdia[0];
            rh[0] = v2(rh[0].x / bet, rh[0].y / bet);
            for (int j = 1; j < n; j++) {
                gam[j] = cupp[j - 1] / bet;
                bet = bdia[j] - alow[j] * gam[j];
                rh[j] = v2((rh[j].x - alow[j] * rh[j - 1].x) / bet, (rh[j].y - alow[j] * rh[j - 1].y) / bet);
            }
            for (int j = n - 2; j >= 0; j--)
                rh[j] = v2(rh[j].x - gam[j + 1] * rh[j + 1].x, rh[j].y - gam[j + 1] * rh[j + 1].y);
            for (int k = kb + 1; k < nvrt; k++) ucol[k] = clampvel(rh[k - kb - 1], P.rmaxvel);
        }
        if (cd == 0.0) ucol[kb] = ucol[kb + 1];
        else if (kb != nvrt - 2) ucol[kb] = v2(0.0, 0.0);
        for (int k = 0; k < kb; k++) ucol[k] = v2(0.0, 0.0);
        // applyMomentumBC: free slip on land sides (islip = 0)
        const int8_t bt = d.sbt[s];
        const double nx = d.snx[s], ny = d.sny[s];
        if (bt == 1) {
            const double2 t = v2(-ny, nx), nn = v2(nx, ny);
            for (int k = kb; k < nvrt; k++) {
                const double vnorm = 0.0;
                const double vtan = dot2(ucol[k], t);
                ucol[k] = t * vtan - nn * vnorm;
            }
        }
        // store u2 and the horizontal advective fluxes Qh (land sides carry zero flux)
        const double len = d.len[s];
        double zprev = d.zc[(size_t)kb * NS + s];
        for (int k = 0; k < nvrt; k++) {
            u2[(size_t)k * NS + s] = ucol[k];
            double qh = -1.0e34;
            if (k > kb) {
                const double zk = d.zc[(size_t)k * NS + s];
                if (bt == 1) qh = 0.0;
                else {
                    const double area = len * (zk - zprev);
                    const double vn1 = nx * ucol[k].x + ny * ucol[k].y;
                    const double vn2 = nx * ucol[k - 1].x + ny * ucol[k - 1].y;
                    qh = area * (0.5 * (vn1 + vn2));
                }
                zprev = zk;
            }
            d.Qh[(size_t)k * NS + s] = qh;
        }
    }
}

__global__ void __launch_bounds__(128) k_vvel(Dev d, Phys P) {
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

void launch_momentum(const Dev& d, const Phys& P, cudaStream_t st, int nsm) {
    k_momentum<<<grid_for(d.NS, 128, nsm * 32), 128, 0, st>>>(d, P);
}

void launch_vvel(const Dev& d, const Phys& P, cudaStream_t st, int nsm) {
    k_vvel<<<grid_for(d.NE, 128, nsm * 32), 128, 0, st>>>(d, P);
}

}  // namespace gs
