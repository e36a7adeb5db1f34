/* CPU oracle: tracer transport (test infrastructure only).
 * Restates computeTransport (schism_step.py:78-93): computeHorizAdvecFluxes (mdc:6461-6491),
 * the sub-cycled horizontalAdvectionPrepare / minTransportDt / horizontalAdvectionUpdate
 * (mdc:6493-6609, 6842-6863), verticalAdvectionUpdate (mdc:6611-6665) and nodalTracerUpdate
 * (mdc:6739-6774); first-order upwind (TransportModel::Upwind, mdh:469-483). */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "step_internal.h"

#define HUGE_D 1.79e+308   /* huge_double, mdh:8 */

static inline double evol(const og_model* m, int e, int k) {
    /* Element::volume(k) = area * (z[k+1] - z[k]), mdh:1023 */
    return m->area[e] * (m->ez[(size_t)e * m->nvrt + k + 1] - m->ez[(size_t)e * m->nvrt + k]);
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
    while (remaining > 0.0) {
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
        double alow[nvrt], bdia[nvrt], cupp[nvrt], rrhs[nvrt], soln[nvrt], gam[nvrt];
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
            }
            tridag1(nEq, alow, bdia, cupp, rrhs, soln, gam);
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
