/* CPU oracle: Eulerian-Lagrangian backtracking (test infrastructure only).
 * Restates backtrackAllNodes (mdc:3547-3660), Side::btrack (mdc:1449-1629), the leaded
 * celestial walk (mdc:85-127) with Element::computePredicates (mdc:651-746), triangle shape
 * coordinates with the fiAnywhere fix (mdc:990-1050) and Element::interpolateVelocities
 * (mdc:1209-1291), for triangles and ics = 1.  The element that holds each foot point is
 * recorded as an extra output (the reference keeps it only inside the walk). */
#include <math.h>
#include <stdlib.h>
#include "step_internal.h"

#define SMALL 1.0e-7          /* mdh:6 */
#define WALK_MAX 40           /* mdc:87 */

static inline v2 npos(const og_model* m, int i) { return V2(m->x[i], m->y[i]); }

static inline double signed_area(v2 p1, v2 p2, v2 p3) {
    /* signedArea, mdh:378-381 */
    return 0.5 * ((p1.x - p3.x) * (p2.y - p3.y) - (p2.x - p3.x) * (p1.y - p3.y));
}

static int node_in_order(const og_model* m, int e, int idx) {
    /* Element::getNodeInOrder, mdc:647-649 */
    const int s = m->es[3 * e + idx];
    return (m->ssign[3 * e + idx] > 0) ? m->isn[2 * s] : m->isn[2 * s + 1];
}

static unsigned valid_exits(const og_model* m, int e, v2 x0, v2 xt, double* fac) {
    /* Element::computePredicates, mdc:651-746, reduced to the validity mask of mdc:102 */
    v2 C[4];
    for (int j = 0; j < 4; j++) C[j] = npos(m, node_in_order(m, e, j == 3 ? 2 : j));
    const v2 vt0 = V2SUB(xt, x0);
    double mp = fmax(V2DOT(vt0, V2SUB(C[0], x0)), V2DOT(vt0, V2SUB(C[1], x0)));
    mp = fmax(mp, V2DOT(vt0, V2SUB(C[2], x0)));
    *fac = fmax(1.00001 * (*fac), fmin(1.0, (mp / V2DOT(vt0, vt0)) * 1.00001));
    const v2 ixt = V2ADD(x0, V2S(V2SUB(xt, x0), *fac));
    const int i3 = 0;                                      /* nxq(3) for a triangle */
    const v2 s0 = V2SUB(C[1], C[0]), s1 = V2SUB(C[2], C[1]), s2 = V2SUB(C[i3], C[2]), s3 = V2SUB(C[0], C[i3]);
    unsigned left = 0, obt = 0, bis = 0;
    left |= (unsigned)(V2CROSS(s0, V2SUB(ixt, C[0])) > -SMALL) << 0;
    left |= (unsigned)(V2CROSS(s1, V2SUB(ixt, C[1])) > -SMALL) << 1;
    left |= (unsigned)(V2CROSS(s2, V2SUB(ixt, C[2])) > -SMALL) << 2;
    left |= 1u << 3;                                       /* triangles: side 3 never valid */
    const v2 s3t = s0;
    obt |= (unsigned)(V2DOT(s0, s1) > 0.0) << 0;
    obt |= (unsigned)(V2DOT(s1, s2) > 0.0) << 1;
    obt |= (unsigned)(V2DOT(s2, s3t) > 0.0) << 2;
    obt |= (unsigned)(V2DOT(s3, s0) > 0.0) << 3;
    bis |= (unsigned)(V2DOT(V2SUB(ixt, C[1]), V2ADD(s0, s1)) < 0.0) << 0;
    bis |= (unsigned)(V2DOT(V2SUB(ixt, C[2]), V2ADD(s1, s2)) < 0.0) << 1;
    bis |= (unsigned)(V2DOT(V2SUB(ixt, C[i3]), V2ADD(s2, s3t)) < 0.0) << 2;
    bis |= (unsigned)(V2DOT(V2SUB(ixt, C[0]), V2ADD(s3, s0)) < 0.0) << 3;
    return (~left & 0xFu) & ((~obt & 0xFu) | bis);
}

static int celestial_walk(og_model* m, int* cur, v2 x0, v2 xt, int* lastCross) {
    /* celestialWalk, mdc:85-127.  The reference asserts past 40 iterations; the oracle
     * stops there, keeps the current element and counts the event. */
    double fac = 0.00001;
    for (int iter = 0; iter < WALK_MAX; iter++) {
        const unsigned valid = valid_exits(m, *cur, x0, xt, &fac);
        if (valid == 0) return 1;
        const int j = __builtin_ctz(valid);
        *lastCross = m->es[3 * (*cur) + j];
        const int prev = *cur;
        const int s = *lastCross;
        const int nxt = (m->isdel[2 * s] == prev) ? m->isdel[2 * s + 1] : m->isdel[2 * s];
        if (nxt < 0 || m->edry[nxt]) { *cur = prev; return 0; }
        *cur = nxt;
    }
#pragma omp atomic
    m->cnt[2]++;
    return 1;
}

static void interp_vel(const og_model* m, int e, double px, double py, double pz, double* out) {
    /* Element::interpolateVelocities, mdc:1209-1291 with computeShapeCoords(fiAnywhere) */
    const int* nd = &m->el[3 * e];
    const int nvrt = m->nvrt;
    const v2 x0 = npos(m, nd[0]), x1 = npos(m, nd[1]), x2 = npos(m, nd[2]);
    const v2 xt = V2(px, py);
    const double area = m->area[e];
    double shp[4];
    shp[0] = signed_area(xt, x1, x2) / area;
    shp[1] = signed_area(x0, xt, x2) / area;
    shp[2] = 1.0 - shp[0] - shp[1];
    shp[3] = 0.0;
    const double tmpmin = fmin(shp[0], fmin(shp[1], shp[2]));
    if (tmpmin < 0) {
        const double a = -tmpmin + 1.0e-8;
        const double b = 1.0 / (shp[0] + shp[1] + shp[2] + 3.0 * a);
        shp[0] = (shp[0] + a) * b;
        shp[1] = (shp[1] + a) * b;
        shp[2] = (shp[2] + a) * b;
    }
    int L = m->kbe[e] - 1, R = nvrt - 1;
    double zL = 0.0, zR = 0.0;
    {
        double zn[4];
        for (int j = 0; j < 3; j++) zn[j] = og_compz(m, nd[j], L > m->kb[nd[j]] ? L : m->kb[nd[j]]);
        zn[3] = 0.0;
        zL = shp[0] * zn[0] + shp[1] * zn[1] + shp[2] * zn[2] + shp[3] * zn[3];
        for (int j = 0; j < 3; j++) zn[j] = og_compz(m, nd[j], R > m->kb[nd[j]] ? R : m->kb[nd[j]]);
        zR = shp[0] * zn[0] + shp[1] * zn[1] + shp[2] * zn[2] + shp[3] * zn[3];
    }
    double w1, w2;
    if (pz <= zL) { w1 = 1.0; w2 = 0.0; }
    else if (pz >= zR) { w1 = 0.0; w2 = 1.0; }
    else {
        while (R - L > 1) {
            const int M = (L + R) / 2;
            double zn[4];
            for (int j = 0; j < 3; j++) zn[j] = og_compz(m, nd[j], M > m->kb[nd[j]] ? M : m->kb[nd[j]]);
            zn[3] = 0.0;
            const double zM = shp[0] * zn[0] + shp[1] * zn[1] + shp[2] * zn[2] + shp[3] * zn[3];
            if (zM < pz) { L = M; zL = zM; } else { R = M; zR = zM; }
        }
        w2 = (pz - zL) / (zR - zL);
        w1 = 1.0 - w2;
    }
    /* s0*v0 + s1*v1 + s2*v2 + s3*v3 with the absent fourth node's value 0 (mdh getNodalValues) */
    const int kl0 = L > m->kb[nd[0]] ? L : m->kb[nd[0]], kr0 = R > m->kb[nd[0]] ? R : m->kb[nd[0]];
    const int kl1 = L > m->kb[nd[1]] ? L : m->kb[nd[1]], kr1 = R > m->kb[nd[1]] ? R : m->kb[nd[1]];
    const int kl2 = L > m->kb[nd[2]] ? L : m->kb[nd[2]], kr2 = R > m->kb[nd[2]] ? R : m->kb[nd[2]];
    const v2* U = m->u2; const double* W = m->w2;
    const v2 uL = V2ADD(V2ADD(V2ADD(V2S(U[(size_t)nd[0] * nvrt + kl0], shp[0]), V2S(U[(size_t)nd[1] * nvrt + kl1], shp[1])),
                              V2S(U[(size_t)nd[2] * nvrt + kl2], shp[2])), V2S(V2(0.0, 0.0), shp[3]));
    const v2 uR = V2ADD(V2ADD(V2ADD(V2S(U[(size_t)nd[0] * nvrt + kr0], shp[0]), V2S(U[(size_t)nd[1] * nvrt + kr1], shp[1])),
                              V2S(U[(size_t)nd[2] * nvrt + kr2], shp[2])), V2S(V2(0.0, 0.0), shp[3]));
    const double wL = shp[0] * W[(size_t)nd[0] * nvrt + kl0] + shp[1] * W[(size_t)nd[1] * nvrt + kl1] +
                      shp[2] * W[(size_t)nd[2] * nvrt + kl2] + shp[3] * 0.0;
    const double wR = shp[0] * W[(size_t)nd[0] * nvrt + kr0] + shp[1] * W[(size_t)nd[1] * nvrt + kr1] +
                      shp[2] * W[(size_t)nd[2] * nvrt + kr2] + shp[3] * 0.0;
    const v2 uv = V2ADD(V2S(uL, w1), V2S(uR, w2));
    out[0] = uv.x; out[1] = uv.y;
    out[2] = w1 * wL + w2 * wR;
}

static void side_btrack(og_model* m, int s, int jlev, double dt, double dtbk, double* u_int, int* elem_out) {
    /* Side::btrack, mdc:1449-1629 */
    const int nvrt = m->nvrt;
    double x0[3] = {m->scx[s], m->scy[s], m->zc[(size_t)s * nvrt + jlev]};
    double time_rm = dt, t1 = 1e10, t2 = 2e10, t3 = 3e10;
    const int a = m->isn[2 * s], b = m->isn[2 * s + 1];
    u_int[0] = m->su2[(size_t)s * nvrt + jlev].x;
    u_int[1] = m->su2[(size_t)s * nvrt + jlev].y;
    u_int[2] = 0.5 * (m->w2[(size_t)a * nvrt + jlev] + m->w2[(size_t)b * nvrt + jlev]);
    int cur = !m->edry[m->isdel[2 * s]] ? m->isdel[2 * s] : m->isdel[2 * s + 1];
    int iter = 0;
    double xt[3] = {-1.0e25, -1.0e25, -1.0e25};
    for (;;) {
        const double dtb = fmin(dtbk, time_rm);
        xt[0] = x0[0] - dtb * u_int[0];
        xt[1] = x0[1] - dtb * u_int[1];
        xt[2] = x0[2] - dtb * u_int[2];
        int lc = -1;
        const int found = celestial_walk(m, &cur, V2(x0[0], x0[1]), V2(xt[0], xt[1]), &lc);
        if (t3 <= time_rm) { xt[0] = x0[0]; xt[1] = x0[1]; xt[2] = x0[2]; break; }
        if (!found) {
            const v2 p1 = npos(m, m->isn[2 * lc]), p2 = npos(m, m->isn[2 * lc + 1]);
            const v2 p0 = V2(x0[0], x0[1]), pt = V2(xt[0], xt[1]);
            const v2 v1 = V2SUB(pt, p0), v2v = V2SUB(p2, p1);
            const double denom = V2CROSS(v2v, v1);
            double t, sp;
            if (fabs(denom) < SMALL) {
                t = fmin(fmax(V2DOT(V2SUB(pt, p1), v2v) / V2DOT(v2v, v2v), 0.0), 1.0);
                if (t < 0.0000000001) t = 0.0;
                if (t > 0.9999999999) t = 1.0;
                sp = fmin(fmax(V2DOT(V2SUB(V2ADD(p1, V2S(v2v, t)), p0), v1) / V2DOT(v1, v1), 0.0), 1.0);
            } else {
                t = fmin(fmax(V2CROSS(V2SUB(p0, p1), v1) / denom, 0.0), 1.0);
                if (t < 0.0000000001) t = 0.0;
                if (t > 0.9999999999) t = 1.0;
                sp = fmin(fmax(V2DOT(V2SUB(V2ADD(p1, V2S(v2v, t)), p0), v1) / V2DOT(v1, v1), 0.0), 1.0);
                if (sp < 0.0000000001) sp = 0.0;
            }
            time_rm -= sp * dtb;
            const v2 xi = V2ADD(p1, V2S(v2v, t));
            xt[2] = x0[2] + sp * (xt[2] - x0[2]);
            xt[0] = xi.x; xt[1] = xi.y;
            if (m->sbt[lc] == 2) break;                     /* open boundary: stop */
            const double ln = sqrt(v2v.x * v2v.x + v2v.y * v2v.y);
            const v2 tg = V2(v2v.x / ln, v2v.y / ln);
            double u[3];
            interp_vel(m, cur, xt[0], xt[1], xt[2], u);
            const double d = u[0] * tg.x + u[1] * tg.y;
            u_int[0] = tg.x * d; u_int[1] = tg.y * d; u_int[2] = u[2];
        } else {
            time_rm -= dtb;
            interp_vel(m, cur, xt[0], xt[1], xt[2], u_int);
        }
        if (time_rm <= 0.0) break;
        const double vmag2 = u_int[0] * u_int[0] + u_int[1] * u_int[1];
        if (vmag2 <= m->velmin * m->velmin) { *elem_out = cur; return; }
        x0[0] = xt[0]; x0[1] = xt[1]; x0[2] = xt[2];
        iter++;
        if (iter == 38) {                                            /* mdc:1610-1611 */
#pragma omp atomic
            m->cnt[3]++;
            *elem_out = cur;
            return;
        }
        t3 = t2; t2 = t1; t1 = time_rm;
    }
    interp_vel(m, cur, xt[0], xt[1], xt[2], u_int);
    *elem_out = cur;
}

void og_btrack(og_model* m) {
    /* backtrackAllNodes, mdc:3547-3660 */
    const int nvrt = m->nvrt;
    const double dt = m->dt;
    const int ndelt_max = (int)fmax(1.0, dt / m->dtb_min);
    const int ndelt_min = (int)fmax(1.0, dt / m->dtb_max);
    const double vm2 = m->velmin * m->velmin;
    m->cnt[2] = 0; m->cnt[3] = 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (int s = 0; s < m->ns; s++) {
        for (int k = 0; k < nvrt; k++) {
            m->btu[(size_t)s * nvrt + k] = m->su2[(size_t)s * nvrt + k];
            m->btel[(size_t)s * nvrt + k] = -1;
        }
        if (m->sdry[s]) continue;
        for (int k = m->kbs[s]; k < nvrt; k++) {
            const v2 u = m->su2[(size_t)s * nvrt + k];
            if (u.x * u.x + u.y * u.y <= vm2) continue;
            double suma = 0.0;
            int icount = 0;
            for (int l = 0; l < 2; l++) {
                const int e = m->isdel[2 * s + l];
                if (e < 0) continue;
                icount++;
                const int* nd = &m->el[3 * e];
                const v2* gp = &m->gphi[3 * e];
                double ut[3], vt[3];
                for (int j = 0; j < 3; j++) { ut[j] = m->u2[(size_t)nd[j] * nvrt + k].x; vt[j] = m->u2[(size_t)nd[j] * nvrt + k].y; }
                const double gux = ut[0] * gp[0].x + ut[1] * gp[1].x + ut[2] * gp[2].x;
                const double guy = ut[0] * gp[0].y + ut[1] * gp[1].y + ut[2] * gp[2].y;
                const double gvx = vt[0] * gp[0].x + vt[1] * gp[1].x + vt[2] * gp[2].x;
                const double gvy = vt[0] * gp[0].y + vt[1] * gp[1].y + vt[2] * gp[2].y;
                suma += dt * sqrt((gux * gux + guy * guy) + (gvx * gvx + gvy * gvy));
            }
            int nd4 = (int)(suma / icount) * 4;
            if (nd4 > ndelt_max) nd4 = ndelt_max;
            if (nd4 < ndelt_min) nd4 = ndelt_min;
            const double dtbk = dt / nd4;
            double ui[3];
            int eo = -1;
            side_btrack(m, s, k, dt, dtbk, ui, &eo);
            m->btu[(size_t)s * nvrt + k] = V2(ui[0], ui[1]);
            m->btel[(size_t)s * nvrt + k] = eo;
        }
    }
}
