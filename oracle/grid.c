/* Oracle: mesh connectivity exactly as the reference's readHGrid builds it.
 * Test infrastructure only (see oracle.h).  Restates grid = src/grid/read_and_process_grid.cpp. */
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* misc.h:20-25: local index at offset from another, modulo size */
static inline int nxq(int offset, int index, int size) {
    return (index + offset + 10 * size) % size;
}

void og_grid_isbnd(int np, int nope, const int32_t* open_start, const int32_t* open_nodes,
                   int nland, const int32_t* land_start, const int32_t* land_nodes,
                   int32_t* isbnd) {
    /* grid:946-950 and 990-996: open nodes carry their segment index (last segment wins) */
    for (int i = 0; i < np; i++) isbnd[i] = -1;
    for (int k = 0; k < nope; k++)
        for (int j = open_start[k]; j < open_start[k + 1]; j++) isbnd[open_nodes[j]] = k;
    /* grid:1071-1077: land nodes not already open become -2 */
    for (int k = 0; k < nland; k++)
        for (int j = land_start[k]; j < land_start[k + 1]; j++)
            if (isbnd[land_nodes[j]] == -1) isbnd[land_nodes[j]] = -2;
}

int og_grid_build(int np, int ne, const int32_t* elnode, const int32_t* i34, const int32_t* isbnd,
                  int32_t* nne_start, int32_t* nne, int32_t* nnp_start, int32_t* nnp,
                  int32_t* ic3, int32_t* elside, int32_t* isdel, int32_t* isidenode, int32_t* ns_out) {
#define ELNODE(j, e) elnode[(e) * 4 + (j)]
#define IC3(j, e) ic3[(e) * 4 + (j)]
#define ELSIDE(j, e) elside[(e) * 4 + (j)]
    int32_t* cnt = (int32_t*)calloc((size_t)np + 1, sizeof(int32_t));
    if (!cnt) return -100;

    /* buildListsOfElementNeighbors, grid:27-84: count, check hanging nodes, fill in element order */
    for (int e = 0; e < ne; e++)
        for (int j = 0; j < i34[e]; j++) cnt[ELNODE(j, e)]++;
    for (int i = 0; i < np; i++)
        if (cnt[i] == 0) { free(cnt); return -1; }
    nne_start[0] = 0;
    for (int i = 0; i < np; i++) nne_start[i + 1] = nne_start[i] + cnt[i];
    memset(cnt, 0, sizeof(int32_t) * (size_t)np);
    for (int e = 0; e < ne; e++)
        for (int j = 0; j < i34[e]; j++) {
            const int v = ELNODE(j, e);
            nne[nne_start[v] + cnt[v]] = e;
            cnt[v]++;
        }

    /* buildElementSideElementTable, grid:272-437 */
    for (int ie = 0; ie < ne; ie++) {
        for (int j = 0; j < 4; j++) { IC3(j, ie) = -1; ELSIDE(j, ie) = -1; }
    }
    for (int ie = 0; ie < ne; ie++) {
        for (int k = 0; k < i34[ie]; k++) {
            IC3(k, ie) = -1;
            const int n1 = ELNODE(nxq(1, k, i34[ie]), ie);
            const int n2 = ELNODE(nxq(2, k, i34[ie]), ie);
            for (int l = nne_start[n1]; l < nne_start[n1 + 1]; l++) {
                const int je = nne[l];
                if (je == ie) continue;
                int found = 0;
                for (int m = 0; m < i34[je]; m++)
                    if (ELNODE(m, je) == n2) { found = 1; break; }
                if (found) { IC3(k, ie) = je; break; }
            }
            const int je = IC3(k, ie);
            if (je != -1) {                   /* grid:315-326: opposite orientation check */
                for (int l = 0; l < i34[je]; l++) {
                    if (ELNODE(nxq(0, l, i34[je]), je) == n1 && ELNODE(nxq(1, l, i34[je]), je) == n2) {
                        free(cnt);
                        return -2;
                    }
                }
            }
        }
    }
    int ns = 0;                               /* grid:331-375: global side numbering */
    for (int ie = 0; ie < ne; ie++) {
        for (int j = 0; j < i34[ie]; j++) {
            const int je = IC3(j, ie);
            if (je != -1) {
                if (ie < je) {
                    ELSIDE(j, ie) = ns;
                    int l = -1;
                    for (int k = 0; k < i34[je]; k++)
                        if (IC3(k, je) == ie) { l = k; break; }
                    if (l == -1) { free(cnt); return -3; }
                    ELSIDE(l, je) = ns;
                    ns++;
                }
            } else {
                ELSIDE(j, ie) = ns;
                ns++;
            }
        }
    }
    if (ns < ne || ns < np) { free(cnt); return -4; }
    for (int ie = 0; ie < ne; ie++) {         /* grid:392-428: isdel / isidenode */
        for (int j = 0; j < i34[ie]; j++) {
            const int jsj = ELSIDE(j, ie);
            if (jsj == -1) { free(cnt); return -5; }
            const int n1 = ELNODE(nxq(1, j, i34[ie]), ie);
            const int n2 = ELNODE(nxq(2, j, i34[ie]), ie);
            const int je = IC3(j, ie);
            if (je == -1 || (je > -1 && ie < je)) {
                isdel[2 * jsj] = ie;     isdel[2 * jsj + 1] = je;
                isidenode[2 * jsj] = n1; isidenode[2 * jsj + 1] = n2;
            } else {
                isdel[2 * jsj] = je;     isdel[2 * jsj + 1] = ie;
                isidenode[2 * jsj] = n2; isidenode[2 * jsj + 1] = n1;
            }
        }
    }
    *ns_out = ns;

    /* reorderElementsCounterClockwise, grid:496-574 */
    for (int i = 0; i < np; i++) {
        const int s0 = nne_start[i], s1 = nne_start[i + 1];
        if (isbnd[i] != -1) {
            int icount = 0;
            for (int q = s0; q < s1; q++) {
                const int ie = nne[q];
                int il = -1;
                for (int l = 0; l < i34[ie]; l++)
                    if (ELNODE(l, ie) == i) { il = l; break; }
                if (il == -1) { free(cnt); return -6; }
                if (IC3(nxq(-1, il, i34[ie]), ie) == -1) { icount++; nne[s0] = ie; }
            }
            if (icount != 1) { free(cnt); return -7; }
        }
        for (int q = s0 + 1; q < s1; q++) {
            const int ie = nne[q - 1];
            int il = -1;
            for (int l = 0; l < i34[ie]; l++)
                if (ELNODE(l, ie) == i) { il = l; break; }
            if (il == -1) { free(cnt); return -6; }
            const int nxt = IC3(nxq(-2, il, i34[ie]), ie);
            if (nxt == -1) { free(cnt); return -8; }
            nne[q] = nxt;
        }
    }

    /* buildListsOfNodeNeighbors, grid:87-174 */
    nnp_start[0] = 0;
    for (int i = 0; i < np; i++) {
        int c = 0;
        const int s0 = nne_start[i], s1 = nne_start[i + 1];
        for (int q = s0; q < s1; q++) {
            const int ie = nne[q];
            if (q == s1 - 1) c += (isbnd[i] == -1) ? i34[ie] - 2 : i34[ie] - 1;
            else c += i34[ie] - 2;
        }
        nnp_start[i + 1] = nnp_start[i] + c;
    }
    for (int i = 0; i < np; i++) {
        int cur = nnp_start[i];
        const int s0 = nne_start[i], s1 = nne_start[i + 1];
        for (int q = s0; q < s1; q++) {
            const int ie = nne[q];
            int ii = -1;
            for (int k = 0; k < i34[ie]; k++)
                if (ELNODE(k, ie) == i) { ii = k; break; }
            if (ii == -1) { free(cnt); return -9; }
            for (int k = 1; k < i34[ie] - 1; k++) nnp[cur++] = ELNODE(nxq(k, ii, i34[ie]), ie);
            if (q == s1 - 1) {
                const int last = ELNODE(nxq(i34[ie] - 1, ii, i34[ie]), ie);
                if (isbnd[i] == -1) {
                    if (last != nnp[nnp_start[i]]) { free(cnt); return -10; }
                } else {
                    nnp[cur++] = last;
                }
            }
        }
    }
    free(cnt);
    return 0;
#undef ELNODE
#undef IC3
#undef ELSIDE
}
