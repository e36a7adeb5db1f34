/* CPU oracle: state exchange in level-major layout (test infrastructure only).
 * Per-level fields travel as [nvrt][n] (vectors [nvrt][n][2], tracers [ntr][nvrt][n]); the
 * oracle stores them per entity ([i*nvrt + k]) like the reference's structs. */
#include <string.h>
#include "step_internal.h"

typedef struct { int kind; int n; int lev; int comp; int isint; } fdesc;
/* kind: pointer selector below; lev: per-level; comp: 1 scalar, 2 vector, -1 tracer */

static void* fptr(const og_model* m, int f, fdesc* d) {
    memset(d, 0, sizeof(*d));
    d->comp = 1;
    switch (f) {
    case OGF_ETA1: d->n = m->np; return m->eta1;
    case OGF_ETA2: d->n = m->np; return m->eta2;
    case OGF_QEL: d->n = m->np; return m->qel;
    case OGF_NODE_TAU: d->n = m->np; d->comp = 2; return m->tau;
    case OGF_ELBC: d->n = m->np; return m->elbc;
    case OGF_JCG_X: d->n = m->np; return m->x0;
    case OGF_JCG_X1: d->n = m->np; return m->x1;
    case OGF_JCG_X2: d->n = m->np; return m->x2;
    case OGF_NODE_Z: d->n = m->np; d->lev = 1; return m->z;
    case OGF_NODE_U2: d->n = m->np; d->lev = 1; d->comp = 2; return m->u2;
    case OGF_NODE_W2: d->n = m->np; d->lev = 1; return m->w2;
    case OGF_NODE_TR: d->n = m->np; d->lev = 1; d->comp = -1; return m->tr;
    case OGF_NODE_KB: d->n = m->np; d->isint = 1; return m->kb;
    case OGF_NODE_DRY: d->n = m->np; d->isint = 2; return m->ndry;
    case OGF_SIDE_U2: d->n = m->ns; d->lev = 1; d->comp = 2; return m->su2;
    case OGF_SIDE_BTU: d->n = m->ns; d->lev = 1; d->comp = 2; return m->btu;
    case OGF_SIDE_ZC: d->n = m->ns; d->lev = 1; return m->zc;
    case OGF_SIDE_QH: d->n = m->ns; d->lev = 1; return m->Qh;
    case OGF_SIDE_BTELEM: d->n = m->ns; d->lev = 1; d->isint = 1; return m->btel;
    case OGF_SIDE_KB: d->n = m->ns; d->isint = 1; return m->kbs;
    case OGF_SIDE_DRY: d->n = m->ns; d->isint = 2; return m->sdry;
    case OGF_SIDE_U: d->n = m->ns; d->comp = 2; return m->U;
    case OGF_SIDE_HHAT: d->n = m->ns; return m->hhat;
    case OGF_SIDE_CHI: d->n = m->ns; return m->chi;
    case OGF_SIDE_GRADETA1: d->n = m->ns; d->comp = 2; return m->gE1;
    case OGF_SIDE_GRADETA2: d->n = m->ns; d->comp = 2; return m->gE2;
    case OGF_ELEM_Z: d->n = m->ne; d->lev = 1; return m->ez;
    case OGF_ELEM_W: d->n = m->ne; d->lev = 1; return m->ew;
    case OGF_ELEM_QV: d->n = m->ne; d->lev = 1; return m->Qv;
    case OGF_ELEM_TR: d->n = m->ne; d->lev = 1; d->comp = -1; return m->etr;
    case OGF_ELEM_KB: d->n = m->ne; d->isint = 1; return m->kbe;
    case OGF_ELEM_DRY: d->n = m->ne; d->isint = 2; return m->edry;
    case OGF_ELEM_GHAT: d->n = m->ne; d->comp = 2; return m->ghat;
    case OGF_NODE_RHO: d->n = m->np; d->lev = 1; return m->rho_n;
    case OGF_ELEM_RHO: d->n = m->ne; d->lev = 1; return m->rho_e;
    case OGF_CSR_DATA: d->n = m->nnz; return m->data;
    case OGF_CSR_INDPTR: d->n = m->np + 1; d->isint = 1; return m->indptr;
    case OGF_CSR_INDICES: d->n = m->nnz; d->isint = 1; return m->indices;
    default: return NULL;
    }
}

static int xfer(og_model* m, int f, void* ext, int to_ext) {
    fdesc d;
    void* p = fptr(m, f, &d);
    if (!p) return -1;
    const int nvrt = m->nvrt, ntr = m->ntr, n = d.n;
    if (d.isint == 1 && !d.lev) {
        if (to_ext) memcpy(ext, p, 4 * (size_t)n); else memcpy(p, ext, 4 * (size_t)n);
        return 0;
    }
    if (d.isint == 2) {
        int32_t* e = (int32_t*)ext; uint8_t* q = (uint8_t*)p;
        for (int i = 0; i < n; i++) { if (to_ext) e[i] = q[i]; else q[i] = (uint8_t)e[i]; }
        return 0;
    }
    if (d.isint == 1 && d.lev) {
        int32_t* e = (int32_t*)ext; int32_t* q = (int32_t*)p;
        for (int k = 0; k < nvrt; k++)
            for (int i = 0; i < n; i++) {
                if (to_ext) e[(size_t)k * n + i] = q[(size_t)i * nvrt + k];
                else q[(size_t)i * nvrt + k] = e[(size_t)k * n + i];
            }
        return 0;
    }
    double* e = (double*)ext; double* q = (double*)p;
    if (!d.lev) {
        const size_t cnt = (size_t)n * d.comp;
        if (to_ext) memcpy(e, q, 8 * cnt); else memcpy(q, e, 8 * cnt);
        return 0;
    }
    if (d.comp == 1 || d.comp == 2) {
        const int c = d.comp;
        for (int k = 0; k < nvrt; k++)
            for (int i = 0; i < n; i++)
                for (int j = 0; j < c; j++) {
                    double* a = &e[((size_t)k * n + i) * c + j];
                    double* b = &q[((size_t)i * nvrt + k) * c + j];
                    if (to_ext) *a = *b; else *b = *a;
                }
        return 0;
    }
    for (int t = 0; t < ntr; t++)
        for (int k = 0; k < nvrt; k++)
            for (int i = 0; i < n; i++) {
                double* a = &e[((size_t)t * nvrt + k) * n + i];
                double* b = &q[((size_t)i * nvrt + k) * ntr + t];
                if (to_ext) *a = *b; else *b = *a;
            }
    return 0;
}

int og_get(const og_model* m, int field, void* out) { return xfer((og_model*)m, field, out, 1); }
int og_put(og_model* m, int field, const void* in) { return xfer(m, field, (void*)in, 0); }
