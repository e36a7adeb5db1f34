/* CPU oracle: tracer transport (test infrastructure only).
 * Restates computeTransport (schism_step.py:78-93): computeHorizAdvecFluxes (mdc:6461-6491),
 * the sub-cycled horizontalAdvectionPrepare / minTransportDt / horizontalAdvectionUpdate
 * (mdc:6493-6609, 6842-6863), verticalAdvectionUpdate (mdc:6611-6665) and nodalTracerUpdate
 * (mdc:6739-6774); first-order upwind (TransportModel::Upwind, mdh:469-483).
 *
 * The TVD option (itr_met = 3) has no counterpart in the reference and is restated from the
 * published scheme (Casulli & Zanolli 2005, as used by SCHISM's TVD transport): on a horizontal
 * face f between the upwind prism U and the downwind prism D the face value is
 * C_U + psi(r_f)/2 (C_D - C_U), with r_f = S_U / (|Q_f| (C_U - C_D)) and S_U the sum over U's
 * interior inflow faces g of |Q_g| (C_g - C_U).  In the non-conservative form of the reference's
 * upwind update this gives, for prism P,
 *   C_P' = C_P + dt/V [ sum_in |Q| (1 - psi/2) (C_U - C_P) + sum_out |Q| psi/2 (C_P - C_D) ],
 * and the sub-step keeps every coefficient non-negative: dt <= V / sum_in |Q| (1 - psi/2 + so)
 * with so = sum_out psi/(2 r) (the outflow terms rewritten through r), times (1 - 1e-6).  With
 * limiter 0 (psi = 0) it is the upwind scheme bit for bit.  The vertical solve optionally adds a
 * constant diffusivity dfh0 between prism centres, implicitly (symmetric, conservative).
 *
 * itr_met = 4 keeps the horizontal TVD of itr_met = 3 and makes the vertical step flux-corrected
 * (Zalesak 1979, FCT, with the implicit upwind solve as the low-order scheme; also no counterpart
 * in the reference, which has only upwind): after the implicit solve gives C^L, each interior
 * interface j of a column (between prisms j and j+1, flux Qv) carries the anti-diffusive transfer
 * a_j = dt |Qv| (C^L_{j+1} - C^L_j) / 2 (the central minus the upwind flux), scaled by
 * alpha_j = min(R+ of the receiving prism, R- of the giving one), where R+/- = min(1, Q+/-/P+/-),
 * P+/- the sums of the prism's incoming / outgoing transfers and Q+/- = V (C_max/min - C^L) with
 * C_max/min over the prism and its column neighbours, of C^L and of the field before the vertical
 * step.  The transfers are antisymmetric, so the column's tracer mass is that of C^L, and no new
 * extremum is made. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "step_internal.h"

#define HUGE_D 1.79e+308   /* huge_double, mdh:8 */

static inline double evol(const og_model* m, int e, int k) {
    /* Element::volume(k) = area * (z[k+1] - z[k]), mdh:1023 */
    return m->area[e] * (m->ez[(size_t)e * m->nvrt + k + 1] - m->ez[(size_t)e * m->nvrt + k]);
}

/* Flux-corrected vertical step of one column of n prisms (index 0 at the bottom): cl = the implicit
 * upwind result, co = the field before the vertical step, v = prism volumes, q[j] = Qv of the
 * interface between prisms j and j+1; out = the corrected field (may be cl).  a, rp, rm are
 * scratch of n entries. */
static void fct_column(int n, double dt, const double* q, const double* v, const double* co, const double* cl,
                       double* out, double* a, double* rp, double* rm) {
    for (int j = 0; j + 1 < n; j++) a[j] = 0.5 * dt * fabs(q[j]) * (cl[j + 1] - cl[j]);
    for (int i = 0; i < n; i++) {
        const double below = i > 0 ? a[i - 1] : 0.0, above = i + 1 < n ? a[i] : 0.0;
        double cmax = fmax(cl[i], co[i]), cmin = fmin(cl[i], co[i]);
        if (i > 0) { cmax = fmax(cmax, fmax(cl[i - 1], co[i - 1])); cmin = fmin(cmin, fmin(cl[i - 1], co[i - 1])); }
        if (i + 1 < n) { cmax = fmax(cmax, fmax(cl[i + 1], co[i + 1])); cmin = fmin(cmin, fmin(cl[i + 1], co[i + 1])); }
        const double pp = fmax(0.0, below) + fmax(0.0, -above);
        const double pm = fmin(0.0, below) + fmin(0.0, -above);
        const double qp = v[i] * (cmax - cl[i]), qm = v[i] * (cmin - cl[i]);
        rp[i] = pp > 0.0 ? fmin(1.0, qp / pp) : 1.0;
        rm[i] = pm < 0.0 ? fmin(1.0, qm / pm) : 1.0;
    }
    /* alpha_j a_j in a, then the update from the bottom up (out may alias cl) */
    for (int j = 0; j + 1 < n; j++) a[j] *= a[j] > 0.0 ? fmin(rp[j + 1], rm[j]) : fmin(rm[j + 1], rp[j]);
    for (int i = 0; i < n; i++) {
        const double fin = i > 0 ? a[i - 1] : 0.0, fout = i + 1 < n ? a[i] : 0.0;
        out[i] = cl[i] + (fin - fout) / v[i];
    }
}

static void tridag1(int n, const double* a, const double* b, const double* c, const double* rhs,
                    double* u, double* gam) {
    double bet = b[0];
    u[0] = rhs[0] / bet;
    for (int j = 1; j < n; j++) {
        gam[j] = c[j - 1] / bet;
        bet = b[j] - a[j] * gam[j];
        u[j] = (rhs[j] - a[j] * u[j - 1]) / bet;
    }
    for (int j = n - 2; j >= 0; j--) u[j] = u[j] - gam[j + 1] * u[j + 1];
}

/* flux limiter psi(r): 0 none, 1 minmod, 2 Osher (beta = 2), 3 van Leer, 4 superbee; every
 * limiter is 0 for r <= 0, and r beyond 1e300 takes the limit value */
static double tvd_psi(int lim, double r) {
    if (!(r > 0.0)) return 0.0;
    if (!(r < 1.0e300)) return lim == 0 ? 0.0 : (lim == 1 ? 1.0 : 2.0);
    switch (lim) {
    case 1: return fmin(r, 1.0);
    case 2: return fmin(r, 2.0);
    case 3: return (r + r) / (1.0 + r);
    case 4: return fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0));
    default: return 0.0;
    }
}

/* psi of a face with upwind value cu, downwind value cd, flux magnitude aq and upwind inflow
 * sum su; *psir = psi / (2 r) (0 when psi = 0) */
static double tvd_face(int lim, double su, double aq, double cu, double cd, double* psir) {
    const double d = cu - cd;
    if (d == 0.0) { *psir = 0.0; return 0.0; }
    const double r = su / (aq * d);
    const double psi = tvd_psi(lim, r);
    *psir = (psi > 0.0) ? psi / (2.0 * r) : 0.0;
    return psi;
}

static inline int face_nb(const og_model* m, int e, int s) {
    return (m->isdel[2 * s] == e) ? m->isdel[2 * s + 1] : m->isdel[2 * s];
}

/* one TVD sub-step of the horizontal advection: snapshot, inflow sums, admissible sub-step,
 * update; returns the sub-step taken */
static double tvd_substep(og_model* m, double remaining) {
    const int ne = m->ne, nvrt = m->nvrt, ntr = m->ntr, lim = m->tvd_limiter;
#define PV(e, k, t) m->prev[((size_t)(e) * nvrt + (k)) * ntr + (t)]
#define SV(e, k, t) m->tvds[((size_t)(e) * nvrt + (k)) * ntr + (t)]
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        if (m->edry[e]) continue;
        memcpy(&m->prev[(size_t)e * nvrt * ntr], &m->etr[(size_t)e * nvrt * ntr], sizeof(double) * nvrt * ntr);
    }
    /* S_P: interior inflow faces, in side order */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        if (m->edry[e]) continue;
        for (int k = m->kbe[e] + 1; k < nvrt; k++)
            for (int t = 0; t < ntr; t++) {
                double su = 0.0;
                for (int j = 0; j < 3; j++) {
                    const int s = m->es[3 * e + j];
                    if (k <= m->kbs[s]) continue;
                    const int nb = face_nb(m, e, s);
                    if (nb < 0 || m->edry[nb]) continue;
                    const double fq = m->Qh[(size_t)s * nvrt + k];
                    if (m->ssign[3 * e + j] * fq < 0.0) su += fabs(fq) * (PV(nb, k, t) - PV(e, k, t));
                }
                SV(e, k, t) = su;
            }
    }
    /* admissible sub-step per element */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        if (m->edry[e]) continue;
        double md = HUGE_D;
        for (int k = m->kbe[e] + 1; k < nvrt; k++) {
            const double vol = evol(m, e, k - 1);
            for (int t = 0; t < ntr; t++) {
                double so = 0.0, den = 0.0, psir;
                for (int j = 0; j < 3; j++) {
                    const int s = m->es[3 * e + j];
                    if (k <= m->kbs[s]) continue;
                    const int nb = face_nb(m, e, s);
                    if (nb < 0 || m->edry[nb]) continue;
                    const double fq = m->Qh[(size_t)s * nvrt + k];
                    if (m->ssign[3 * e + j] * fq > 0.0) {
                        tvd_face(lim, SV(e, k, t), fabs(fq), PV(e, k, t), PV(nb, k, t), &psir);
                        so += psir;
                    }
                }
                for (int j = 0; j < 3; j++) {
                    const int s = m->es[3 * e + j];
                    if (k <= m->kbs[s]) continue;
                    const int nb = face_nb(m, e, s);
                    if (nb < 0 || m->edry[nb]) continue;
                    const double fq = m->Qh[(size_t)s * nvrt + k];
                    if (m->ssign[3 * e + j] * fq < 0.0) {
                        const double psi = tvd_face(lim, SV(nb, k, t), fabs(fq), PV(nb, k, t), PV(e, k, t), &psir);
                        den += fabs(fq) * (1.0 - 0.5 * psi + so);
                    }
                }
                const double pd = (den == 0.0) ? HUGE_D : vol / den * (1.0 - 1.0e-6);
                md = fmin(md, pd);
            }
        }
        m->maxDt[e] = md;
    }
    double mdt = 1e34;
    for (int e = 0; e < ne; e++) mdt = fmin(mdt, m->edry[e] ? HUGE_D : m->maxDt[e]);
    const double dtb = fmin(remaining, mdt);
    /* update, faces in side order, tracers inner */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        if (m->edry[e]) continue;
        const int kb = m->kbe[e];
        double* tr = &m->etr[(size_t)e * nvrt * ntr];
        for (int k = kb + 1; k < nvrt; k++) {
            const double dbv = dtb / evol(m, e, k - 1);
            double adv[64];
            for (int t = 0; t < ntr; t++) adv[t] = PV(e, k, t);
            for (int j = 0; j < 3; j++) {
                const int s = m->es[3 * e + j];
                if (k <= m->kbs[s]) continue;
                const double fq = m->Qh[(size_t)s * nvrt + k];
                const double sQ = m->ssign[3 * e + j] * fq;
                const int nb = face_nb(m, e, s);
                const int interior = nb >= 0 && !m->edry[nb];
                const double coef = dbv * fabs(fq);
                double psir;
                if (sQ < 0.0) {
                    if (interior) {
                        for (int t = 0; t < ntr; t++) {
                            const double own = PV(e, k, t), cu = PV(nb, k, t);
                            const double psi = tvd_face(lim, SV(nb, k, t), fabs(fq), cu, own, &psir);
                            adv[t] += coef * (1.0 - 0.5 * psi) * (cu - own);
                        }
                    } else if (m->sbt[s] == 2) {
                        /* open boundary inflow: Cout keeps the running value (mdc:6585-6592) */
                        for (int t = 0; t < ntr; t++) adv[t] += coef * (adv[t] - PV(e, k, t));
                    }
                } else if (sQ > 0.0 && interior) {
                    for (int t = 0; t < ntr; t++) {
                        const double own = PV(e, k, t), cd = PV(nb, k, t);
                        const double psi = tvd_face(lim, SV(e, k, t), fabs(fq), own, cd, &psir);
                        adv[t] += coef * (0.5 * psi) * (own - cd);
                    }
                }
            }
            for (int t = 0; t < ntr; t++) tr[k * ntr + t] = adv[t];
        }
        for (int k = 0; k <= kb; k++)
            for (int t = 0; t < ntr; t++) tr[k * ntr + t] = tr[(kb + 1) * ntr + t];
    }
#undef PV
#undef SV
    return dtb;
}

int og_transport(og_model* m, double dt) {
    const int ne = m->ne, ns = m->ns, nvrt = m->nvrt, ntr = m->ntr;
    /* computeHorizAdvecFluxes */
    for (int s = 0; s < ns; s++) {
        double* Qh = &m->Qh[(size_t)s * nvrt];
        for (int k = 0; k < nvrt; k++) Qh[k] = -1.0e34;
        if (m->sdry[s]) continue;
        const int land = (m->sbt[s] == 1);
        for (int k = m->kbs[s] + 1; k < nvrt; k++) {
            if (land) { Qh[k] = 0.0; continue; }
            const double area = m->len[s] * (m->zc[(size_t)s * nvrt + k] - m->zc[(size_t)s * nvrt + k - 1]);
            const v2 u1 = m->su2[(size_t)s * nvrt + k], u0 = m->su2[(size_t)s * nvrt + k - 1];
            const double vn1 = m->snx[s] * u1.x + m->sny[s] * u1.y;
            const double vn2 = m->snx[s] * u0.x + m->sny[s] * u0.y;
            const double vc = 0.5 * (vn1 + vn2);
            Qh[k] = area * vc;
        }
    }
    double remaining = dt;
    int nsub = 0;
    while (m->itr_met >= 3 && remaining > 0.0) {
        remaining -= tvd_substep(m, remaining);
        nsub++;
    }
    while (m->itr_met < 3 && remaining > 0.0) {
        /* horizontalAdvectionPrepare */
#pragma omp parallel for schedule(static)
        for (int e = 0; e < ne; e++) {
            if (m->edry[e]) continue;
            const int kb = m->kbe[e];
            memcpy(&m->prev[(size_t)e * nvrt * ntr], &m->etr[(size_t)e * nvrt * ntr], sizeof(double) * nvrt * ntr);
            m->maxDt[e] = HUGE_D;
            for (int k = 0; k < kb + 1; k++) m->inflow[(size_t)e * nvrt + k] = 0.0;
            for (int k = kb + 1; k < nvrt; k++) {
                double in = 0.0;
                for (int j = 0; j < 3; j++) {
                    const int s = m->es[3 * e + j];
                    if (k <= m->kbs[s]) continue;
                    const int nb = (m->isdel[2 * s] == e) ? m->isdel[2 * s + 1] : m->isdel[2 * s];
                    if (nb < 0 || m->edry[nb]) continue;
                    const double fq = m->Qh[(size_t)s * nvrt + k];
                    const int influx = (m->ssign[3 * e + j] * fq) < 0.0;
                    if (m->sbt[s] == 1 || !influx) continue;
                    in += fabs(fq);
                }
                m->inflow[(size_t)e * nvrt + k] = in;
                const double pd = (in == 0.0) ? HUGE_D : evol(m, e, k - 1) / in * (1.0 - 1.0e-6);
                m->maxDt[e] = fmin(m->maxDt[e], pd);
            }
        }
        /* minTransportDt: minimum over wet elements, seeded with 1e34 (schism_step.py:73) */
        double mdt = 1e34;
        for (int e = 0; e < ne; e++) mdt = fmin(mdt, m->edry[e] ? HUGE_D : m->maxDt[e]);
        const double dtb = fmin(remaining, mdt);
        /* horizontalAdvectionUpdate(dtb) */
#pragma omp parallel for schedule(static)
        for (int e = 0; e < ne; e++) {
            if (m->edry[e]) continue;
            const int kb = m->kbe[e];
            const double* pv = &m->prev[(size_t)e * nvrt * ntr];
            double* tr = &m->etr[(size_t)e * nvrt * ntr];
            for (int k = kb + 1; k < nvrt; k++) {
                const double vol = evol(m, e, k - 1);
                const double dbv = dtb / vol;
                double adv[64];
                for (int t = 0; t < ntr; t++) adv[t] = pv[k * ntr + t];
                for (int j = 0; j < 3; j++) {
                    const int s = m->es[3 * e + j];
                    if (k <= m->kbs[s]) continue;
                    const double fq = m->Qh[(size_t)s * nvrt + k];
                    const double sQ = m->ssign[3 * e + j] * fq;
                    if (sQ >= 0.0) continue;
                    double cout[64];
                    for (int t = 0; t < ntr; t++) cout[t] = adv[t];
                    const int nb = (m->isdel[2 * s] == e) ? m->isdel[2 * s + 1] : m->isdel[2 * s];
                    if (nb >= 0 && !m->edry[nb]) {
                        for (int t = 0; t < ntr; t++) cout[t] = m->prev[((size_t)nb * nvrt + k) * ntr + t];
                    } else if (m->sbt[s] == 2) {
                        /* open boundary inflow: Cout keeps the running value (mdc:6585-6592) */
                    } else {
                        continue;
                    }
                    const double coef = dbv * fabs(fq);
                    for (int t = 0; t < ntr; t++) adv[t] += coef * (cout[t] - pv[k * ntr + t]);
                }
                for (int t = 0; t < ntr; t++) tr[k * ntr + t] = adv[t];
            }
            for (int k = 0; k <= kb; k++)
                for (int t = 0; t < ntr; t++) tr[k * ntr + t] = tr[(kb + 1) * ntr + t];
        }
        remaining -= dtb;
        nsub++;
    }
    m->cnt[1] = nsub;
    /* verticalAdvectionUpdate(dt) */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; e++) {
        double alow[nvrt], bdia[nvrt], cupp[nvrt], rrhs[nvrt], soln[nvrt], gam[nvrt], vol[nvrt], fa[nvrt],
            frp[nvrt], frm[nvrt];
        if (m->edry[e]) continue;
        const int kb = m->kbe[e];
        double* tr = &m->etr[(size_t)e * nvrt * ntr];
        double* pv = &m->prev[(size_t)e * nvrt * ntr];
        memcpy(pv, tr, sizeof(double) * nvrt * ntr);
        const double* Qv = &m->Qv[(size_t)e * nvrt];
        for (int t = 0; t < ntr; t++) {
            const int nEq = nvrt - (kb + 1);
            for (int kin = 0; kin < nEq; kin++) { alow[kin] = 0.0; cupp[kin] = 0.0; bdia[kin] = 0.0; }
            for (int k = kb + 1; k < nvrt; k++) {
                const int kin = k - (kb + 1);
                const double dbv = dt / evol(m, e, k - 1);
                bdia[kin] += 1.0;
                rrhs[kin] = pv[k * ntr + t] * 1.0;
                if (k != nvrt - 1 && Qv[k] < 0.0) {
                    const double tmp = dbv * fabs(Qv[k]);
                    cupp[kin] -= tmp; bdia[kin] += tmp;
                }
                if (k - 1 != kb && Qv[k - 1] > 0.0) {
                    const double tmp = dbv * fabs(Qv[k - 1]);
                    alow[kin] -= tmp; bdia[kin] += tmp;
                }
                if (m->dfh0 > 0.0) {
                    /* diffusion across the interfaces with the prisms above and below, over the
                       distance between prism centres */
                    const double* z = &m->ez[(size_t)e * nvrt];
                    if (k != nvrt - 1) {
                        const double tmp = dbv * (m->dfh0 * m->area[e] / (0.5 * (z[k + 1] - z[k - 1])));
                        cupp[kin] -= tmp; bdia[kin] += tmp;
                    }
                    if (k - 1 != kb) {
                        const double tmp = dbv * (m->dfh0 * m->area[e] / (0.5 * (z[k] - z[k - 2])));
                        alow[kin] -= tmp; bdia[kin] += tmp;
                    }
                }
            }
            tridag1(nEq, alow, bdia, cupp, rrhs, soln, gam);
            if (m->itr_met == 4) {
                for (int k = kb + 1; k < nvrt; k++) vol[k - (kb + 1)] = evol(m, e, k - 1);
                fct_column(nEq, dt, Qv + kb + 1, vol, rrhs, soln, soln, fa, frp, frm);
            }
            for (int k = kb + 1; k < nvrt; k++) tr[k * ntr + t] = soln[k - (kb + 1)];
        }
        for (int k = 0; k <= kb; k++)
            for (int t = 0; t < ntr; t++) tr[k * ntr + t] = tr[(kb + 1) * ntr + t];
    }
    /* nodalTracerUpdate */
    const int ivrt = nvrt - 1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m->np; i++) {
        if (m->ndry[i]) continue;
        for (int k = 0; k < nvrt; k++) {
            double sum[64];
            for (int t = 0; t < ntr; t++) sum[t] = 0.0;
            double sumA = 0.0;
            for (int q = m->nne_s[i]; q < m->nne_s[i + 1]; q++) {
                const int e = m->nne[q];
                if (m->edry[e]) continue;
                const int kb = m->kbe[e];
                const int kin = k > kb ? k : kb;
                int kLo = kin, kHi = kin + 1;
                double zrat = 0.0;
                const double* z = &m->ez[(size_t)e * nvrt];
                if (kin == ivrt) { kLo = ivrt; kHi = ivrt; }
                else if (kin == kb) { kLo = kb + 1; kHi = kb + 1; }
                else zrat = (z[kin + 1] - z[kin]) / (z[kin + 1] - z[kin - 1]);
                const double A = m->area[e];
                const double* tr = &m->etr[(size_t)e * nvrt * ntr];
                for (int t = 0; t < ntr; t++)
                    sum[t] += A * ((1.0 - zrat) * tr[kHi * ntr + t] + zrat * tr[kLo * ntr + t]);
                sumA += A;
            }
            if (sumA == 0.0) continue;
            const double inv = 1.0 / sumA;
            for (int t = 0; t < ntr; t++) m->tr[((size_t)i * nvrt + k) * ntr + t] = inv * sum[t];
        }
    }
    return nsub;
}

int og_fct_column(int n, double dt, const double* q, const double* v, const double* co, const double* cl,
                  double* out) {
    if (n < 1) return -1;
    double* scr = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    if (!scr) return -1;
    fct_column(n, dt, q, v, co, cl, out, scr, scr + n, scr + 2 * (size_t)n);
    free(scr);
    return 0;
}

void og_tracer_mass(const og_model* m, double* out) {
    /* sum over wet prisms of volume x concentration, two-sum compensated (Neumaier) */
    const int nvrt = m->nvrt, ntr = m->ntr;
    for (int t = 0; t < ntr; t++) {
        double s = 0.0, c = 0.0;
        for (int e = 0; e < m->ne; e++) {
            if (m->edry[e]) continue;
            for (int k = m->kbe[e] + 1; k < nvrt; k++) {
                const double v = evol(m, e, k - 1) * m->etr[((size_t)e * nvrt + k) * ntr + t];
                const double tt = s + v;
                if (fabs(s) >= fabs(v)) c += (s - tt) + v; else c += (v - tt) + s;
                s = tt;
            }
        }
        out[t] = s + c;
    }
}
