// Eulerian-Lagrangian backtracking (backtrackAllNodes, meshdata.cu:3547-3660; Side::btrack,
// :1449-1629; leaded celestial walk, :85-127 and :651-746; interpolateVelocities, :1209-1291).
//
// One thread per (side, level) query, level-major so a warp handles neighbouring sides of one
// level (coalesced side data, cache-local element walks).  This file is compiled with
// -fmad=false: the walk predicates and the shape coordinates must round exactly like the FP64
// CPU restatement so that the element reached by every walk matches it bit for bit.
#include "dev_common.cuh"
#include "kernels.h"

namespace gs {

namespace {

constexpr double kSmall = 1.0e-7;
constexpr int kWalkMax = 40;

__device__ __forceinline__ double2 npos(const Dev& d, int i) { return v2(d.x[i], d.y[i]); }

__device__ __forceinline__ double signed_area(double2 p1, double2 p2, double2 p3) {
    return 0.5 * ((p1.x - p3.x) * (p2.y - p3.y) - (p2.x - p3.x) * (p1.y - p3.y));
}

__device__ __forceinline__ double2 corner(const double2 (&p)[3], int j) {
    return j == 0 ? p[0] : (j == 1 ? p[1] : p[2]);
}

// Exits of element e through which the walk from x0 towards xt may leave (one bit per side, in
// the element's side order); 0 when xt is inside.  The corners are taken in the element's
// orientation: corner j starts side j.  Of the reference's four-corner predicate masks only the
// three triangle bits can be set (its fourth "left" bit is always set, which masks the rest), and
// the obtuse-corner bits depend on the element alone, so they come with the element record.
__device__ unsigned valid_exits(const ElemGeo* geo, int e, double2 x0, double2 xt, double& fac) {
    double2 p[3];
    p[0] = geo[e].p[0]; p[1] = geo[e].p[1]; p[2] = geo[e].p[2];
    const int pm = geo[e].perm;
    double2 C[3];
    C[0] = corner(p, pm & 3);
    C[1] = corner(p, (pm >> 2) & 3);
    C[2] = corner(p, (pm >> 4) & 3);
    const double2 vt0 = xt - x0;
    double mp = fmax(dot2(vt0, C[0] - x0), dot2(vt0, C[1] - x0));
    mp = fmax(mp, dot2(vt0, C[2] - x0));
    fac = fmax(1.00001 * fac, fmin(1.0, (mp / dot2(vt0, vt0)) * 1.00001));
    const double2 ixt = x0 + (xt - x0) * fac;
    const double2 s0 = C[1] - C[0], s1 = C[2] - C[1], s2 = C[0] - C[2];
    unsigned left = 0u, bis = 0u;
    left |= (unsigned)(cross2(s0, ixt - C[0]) > -kSmall);
    left |= (unsigned)(cross2(s1, ixt - C[1]) > -kSmall) << 1;
    left |= (unsigned)(cross2(s2, ixt - C[2]) > -kSmall) << 2;
    const unsigned obt = (unsigned)(pm >> 8) & 7u;
    bis |= (unsigned)(dot2(ixt - C[1], s0 + s1) < 0.0);
    bis |= (unsigned)(dot2(ixt - C[2], s1 + s2) < 0.0) << 1;
    bis |= (unsigned)(dot2(ixt - C[0], s2 + s0) < 0.0) << 2;
    return (~left & 7u) & ((~obt & 7u) | bis);
}

// returns 1 if xt was found inside *cur, 0 if the walk stopped at a boundary or dry element
__device__ int celestial_walk(const Dev& d, int& cur, double2 x0, double2 xt, int& lastCross) {
    double fac = 0.00001;
    for (int iter = 0; iter < kWalkMax; iter++) {
        const unsigned valid = valid_exits(d.egeo, cur, x0, xt, fac);
        if (valid == 0u) return 1;
        const int j = __ffs(valid) - 1;
        const int s = d.es[j * d.NE + cur];
        lastCross = s;
        const int e0 = d.se[s], e1 = d.se[d.NS + s];
        const int nxt = (e0 == cur) ? e1 : e0;
        if (nxt < 0 || d.edry[nxt]) return 0;
        cur = nxt;
    }
    atomicAdd(&d.counters[0], 1ull);
    return 1;
}

// Velocity at (px, py, pz) inside element e (interpolateVelocities).  The vertical bracket is
// the pair of levels (L, L+1) with z(L) < pz <= z(L+1) of the element-interpolated level
// heights, or the bottom (pz <= z(kbe-1)) or top (pz >= z(nvrt-1)) case.  z is non-decreasing
// in the level (the vertical grid's levels are ordered at every wet node; a dry node's levels
// all sit at 0 and rounding keeps a weighted sum of non-decreasing terms non-decreasing), so
// that pair is unique and any search that keeps z(L) < pz <= z(R) ends on the same one as the
// reference's bisection over [kbe-1, nvrt-1].  The search starts at `hint` (the previous
// bracket of this trajectory), steps at most one level either way and bisects the rest.
__device__ void interp_vel(const Dev& d, const VG& vg, int e, double px, double py, double pz, double* out,
                           int& hint) {
    const int NP = d.NP;
    const ElemGeo& g = d.egeo[e];
    const double2 x0 = g.p[0], x1 = g.p[1], x2 = g.p[2];
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const double2 xt = v2(px, py);
    const double area = g.area;
    double s0 = signed_area(xt, x1, x2) / area;
    double s1 = signed_area(x0, xt, x2) / area;
    double s2 = 1.0 - s0 - s1;
    const double s3 = 0.0;
    const double tmpmin = fmin(s0, fmin(s1, s2));
    if (tmpmin < 0) {
        const double a = -tmpmin + 1.0e-8;
        const double b = 1.0 / (s0 + s1 + s2 + 3.0 * a);
        s0 = (s0 + a) * b; s1 = (s1 + a) * b; s2 = (s2 + a) * b;
    }
    const int kb0 = d.kb[n0], kb1 = d.kb[n1], kb2 = d.kb[n2];
    const double e0 = d.eta2[n0], e1 = d.eta2[n1], e2 = d.eta2[n2];
    const double h0 = d.depth[n0], h1 = d.depth[n1], h2 = d.depth[n2];
    auto zat = [&](int k) {
        const double z0 = compz(vg, e0, h0, kb0, k > kb0 ? k : kb0);
        const double z1 = compz(vg, e1, h1, kb1, k > kb1 ? k : kb1);
        const double z2 = compz(vg, e2, h2, kb2, k > kb2 ? k : kb2);
        return s0 * z0 + s1 * z1 + s2 * z2 + s3 * 0.0;
    };
    // L* = the highest level in [lo, hi] with z < pz (lo - 1 when there is none), searched
    // between the sentinels lo - 1 and hi + 1: two one-level steps from the hint, then bisection
    const int lo = d.kbe[e] - 1, hi = vg.nvrt - 1;
    int Lk = lo - 1, Rk = hi + 1;
    double zL = 0.0, zR = 0.0;
    int k = min(max(hint, lo), hi);
    for (int probe = 0; Rk - Lk > 1; probe++) {
        const double zk = zat(k);
        const bool below = zk < pz;
        if (below) { Lk = k; zL = zk; } else { Rk = k; zR = zk; }
        k = (probe < 2) ? (below ? k + 1 : k - 1) : (Lk + Rk) / 2;
        if (k <= Lk || k >= Rk) k = (Lk + Rk) / 2;
    }
    hint = Lk;
    // bottom when no level lies below pz; top when pz reaches the top height
    int mode = (Lk < lo) ? 1 : (Lk == hi) ? 2 : 0;
    if (mode == 0 && zR == pz && (Rk == hi || pz >= zat(hi))) mode = 2;
    int L = Lk, R = Rk;
    double w1, w2;
    if (mode == 0) {
        w2 = (pz - zL) / (zR - zL);
        w1 = 1.0 - w2;
    } else {
        L = lo; R = hi;
        w1 = (mode == 1) ? 1.0 : 0.0;
        w2 = 1.0 - w1;
    }
    const int kl0 = L > kb0 ? L : kb0, kl1 = L > kb1 ? L : kb1, kl2 = L > kb2 ? L : kb2;
    const int kr0 = R > kb0 ? R : kb0, kr1 = R > kb1 ? R : kb1, kr2 = R > kb2 ? R : kb2;
    const double2 zero = v2(0.0, 0.0);
    const double2 uL = ((d.u2[(size_t)kl0 * NP + n0] * s0 + d.u2[(size_t)kl1 * NP + n1] * s1) +
                        d.u2[(size_t)kl2 * NP + n2] * s2) + zero * s3;
    const double2 uR = ((d.u2[(size_t)kr0 * NP + n0] * s0 + d.u2[(size_t)kr1 * NP + n1] * s1) +
                        d.u2[(size_t)kr2 * NP + n2] * s2) + zero * s3;
    const double wL = s0 * d.w2[(size_t)kl0 * NP + n0] + s1 * d.w2[(size_t)kl1 * NP + n1] +
                      s2 * d.w2[(size_t)kl2 * NP + n2] + s3 * 0.0;
    const double wR = s0 * d.w2[(size_t)kr0 * NP + n0] + s1 * d.w2[(size_t)kr1 * NP + n1] +
                      s2 * d.w2[(size_t)kr2 * NP + n2] + s3 * 0.0;
    const double2 uv = uL * w1 + uR * w2;
    out[0] = uv.x; out[1] = uv.y;
    out[2] = w1 * wL + w2 * wR;
}

__device__ void side_btrack(const Dev& d, const VG& vg, const Phys& P, int s, int jlev, double dtbk,
                            double* u_int, int& elem_out) {
    const int NS = d.NS, NP = d.NP;
    double x0[3] = {d.scx[s], d.scy[s], d.zc[(size_t)jlev * NS + s]};
    double time_rm = P.dt, t1 = 1e10, t2 = 2e10, t3 = 3e10;
    const int a = d.sn[s], b = d.sn[NS + s];
    const double2 u0 = d.su2[(size_t)jlev * NS + s];
    u_int[0] = u0.x; u_int[1] = u0.y;
    u_int[2] = 0.5 * (d.w2[(size_t)jlev * NP + a] + d.w2[(size_t)jlev * NP + b]);
    const int ea = d.se[s], eb = d.se[NS + s];
    int cur = !d.edry[ea] ? ea : eb;
    int iter = 0, hint = jlev - 1;
    bool fresh = false;   // u_int holds the interpolation at (cur, xt) of this sub-step
    double xt[3] = {-1.0e25, -1.0e25, -1.0e25};
    const double vm2 = P.velmin * P.velmin;
    for (;;) {
        const double dtb = fmin(dtbk, time_rm);
        xt[0] = x0[0] - dtb * u_int[0];
        xt[1] = x0[1] - dtb * u_int[1];
        xt[2] = x0[2] - dtb * u_int[2];
        int lc = -1;
        const int found = celestial_walk(d, cur, v2(x0[0], x0[1]), v2(xt[0], xt[1]), lc);
        fresh = false;
        if (t3 <= time_rm) { xt[0] = x0[0]; xt[1] = x0[1]; xt[2] = x0[2]; break; }
        if (!found) {
            const double2 p1 = npos(d, d.sn[lc]), p2 = npos(d, d.sn[NS + lc]);
            const double2 p0 = v2(x0[0], x0[1]), pt = v2(xt[0], xt[1]);
            const double2 v1 = pt - p0, vv = p2 - p1;
            const double denom = cross2(vv, v1);
            double t, sp;
            if (fabs(denom) < kSmall) {
                t = fmin(fmax(dot2(pt - p1, vv) / dot2(vv, vv), 0.0), 1.0);
                if (t < 0.0000000001) t = 0.0;
                if (t > 0.9999999999) t = 1.0;
                sp = fmin(fmax(dot2((p1 + vv * t) - p0, v1) / dot2(v1, v1), 0.0), 1.0);
            } else {
                t = fmin(fmax(cross2(p0 - p1, v1) / denom, 0.0), 1.0);
                if (t < 0.0000000001) t = 0.0;
                if (t > 0.9999999999) t = 1.0;
                sp = fmin(fmax(dot2((p1 + vv * t) - p0, v1) / dot2(v1, v1), 0.0), 1.0);
                if (sp < 0.0000000001) sp = 0.0;
            }
            time_rm -= sp * dtb;
            const double2 xi = p1 + vv * t;
            xt[2] = x0[2] + sp * (xt[2] - x0[2]);
            xt[0] = xi.x; xt[1] = xi.y;
            if (d.sbt[lc] == 2) break;
            const double ln = sqrt(vv.x * vv.x + vv.y * vv.y);
            const double2 tg = v2(vv.x / ln, vv.y / ln);
            double u[3];
            interp_vel(d, vg, cur, xt[0], xt[1], xt[2], u, hint);
            const double dd = u[0] * tg.x + u[1] * tg.y;
            u_int[0] = tg.x * dd; u_int[1] = tg.y * dd; u_int[2] = u[2];
        } else {
            time_rm -= dtb;
            interp_vel(d, vg, cur, xt[0], xt[1], xt[2], u_int, hint);
            fresh = true;
        }
        if (time_rm <= 0.0) break;
        const double vmag2 = u_int[0] * u_int[0] + u_int[1] * u_int[1];
        if (vmag2 <= vm2) { elem_out = cur; return; }
        x0[0] = xt[0]; x0[1] = xt[1]; x0[2] = xt[2];
        iter++;
        if (iter == 38) { atomicAdd(&d.counters[1], 1ull); elem_out = cur; return; }
        t3 = t2; t2 = t1; t1 = time_rm;
    }
    // the final interpolation at (cur, xt); when the last sub-step ended inside an element it has
    // just been computed with these same arguments
    if (!fresh) interp_vel(d, vg, cur, xt[0], xt[1], xt[2], u_int, hint);
    elem_out = cur;
}

}  // namespace

// resident blocks per SM the backtracking is compiled for (register budget)
#ifndef GS_BTRACK_MIN_BLOCKS
#define GS_BTRACK_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(128, GS_BTRACK_MIN_BLOCKS) k_btrack(Dev d, Phys P, VG vg) {
    const int NS = d.NS, NP = d.NP, NE = d.NE, nvrt = P.nvrt;
    const long long total = (long long)NS * nvrt;
    const int ndelt_max = (int)fmax(1.0, P.dt / P.dtb_min);
    const int ndelt_min = (int)fmax(1.0, P.dt / P.dtb_max);
    const double vm2 = P.velmin * P.velmin;
    if (NS <= 0) return;
    // query q = k * NS + s, visited with a grid stride; (k, s) carried instead of divided
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long q0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int k = (int)(q0 / NS), s = (int)(q0 - (long long)k * NS);
    const int dk = (int)(stride / NS), ds = (int)(stride - (long long)dk * NS);
    for (long long qi = q0; qi < total; qi += stride, k += dk, s += ds) {
        if (s >= NS) { s -= NS; k++; }
        const double2 u = d.su2[(size_t)k * NS + s];
        double2 bt = u;
        int be = -1;
        if (!d.sdry[s] && k >= d.kbs[s] && !(u.x * u.x + u.y * u.y <= vm2)) {
            double suma = 0.0;
            int icount = 0;
            for (int l = 0; l < 2; l++) {
                const int e = d.se[l * NS + s];
                if (e < 0) continue;
                icount++;
                const int n0 = d.en[e], n1 = d.en[NE + e], n2 = d.en[2 * NE + e];
                const double2 g0 = d.gphi[e], g1 = d.gphi[NE + e], g2 = d.gphi[2 * NE + e];
                const double2 a0 = d.u2[(size_t)k * NP + n0], a1 = d.u2[(size_t)k * NP + n1], a2 = d.u2[(size_t)k * NP + n2];
                const double gux = a0.x * g0.x + a1.x * g1.x + a2.x * g2.x;
                const double guy = a0.x * g0.y + a1.x * g1.y + a2.x * g2.y;
                const double gvx = a0.y * g0.x + a1.y * g1.x + a2.y * g2.x;
                const double gvy = a0.y * g0.y + a1.y * g1.y + a2.y * g2.y;
                suma += P.dt * sqrt((gux * gux + guy * guy) + (gvx * gvx + gvy * gvy));
            }
            int nd4 = (int)(suma / icount) * 4;
            if (nd4 > ndelt_max) nd4 = ndelt_max;
            if (nd4 < ndelt_min) nd4 = ndelt_min;
            const double dtbk = P.dt / nd4;
            double ui[3];
            side_btrack(d, vg, P, s, k, dtbk, ui, be);
            bt = v2(ui[0], ui[1]);
        }
        d.btu[(size_t)k * NS + s] = bt;
        d.btel[(size_t)k * NS + s] = be;
    }
}

void launch_btrack(const Dev& d, const Phys& P, const VG& vg, cudaStream_t st, int nsm, const LaunchTable& L) {
    cudaMemsetAsync(d.counters, 0, 2 * sizeof(unsigned long long), st);
    const LaunchShape& s = L.k[LK_BTRACK];
    k_btrack<<<grid_of((long long)d.NS * P.nvrt, s, nsm), s.block, 0, st>>>(d, P, vg);
}

int btrack_max_threads() {
    cudaFuncAttributes a{};
    return cudaFuncGetAttributes(&a, k_btrack) == cudaSuccess ? a.maxThreadsPerBlock : 0;
}

}  // namespace gs
