// Mesh connectivity and space-filling-curve ordering (host side of gschism_b200).
//
// gs_grid_build reproduces the numbering of the reference grid reader exactly
// (src/grid/read_and_process_grid.cpp:27-574): the side numbering, isdel/isidenode orientation
// and the counter-clockwise node->element / node->node orders are part of the drop-in contract,
// because every per-node sum of the step runs in that element order.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "gs_internal.h"

namespace gs {

namespace {
inline int wrap(int i, int n) { return ((i % n) + n) % n; }

inline int local_of(const int32_t* el, int i34, int node) {
    for (int l = 0; l < i34; ++l)
        if (el[l] == node) return l;
    return -1;
}
}  // namespace

int build_connectivity(int np, int ne, const int32_t* elnode, const int32_t* i34, const int32_t* isbnd,
                       Connectivity& c) {
    // node -> elements, element order (read_and_process_grid.cpp:27-84)
    c.nne_start.assign(np + 1, 0);
    for (int e = 0; e < ne; ++e)
        for (int j = 0; j < i34[e]; ++j) c.nne_start[elnode[4 * e + j] + 1]++;
    for (int i = 0; i < np; ++i) {
        if (c.nne_start[i + 1] == 0) return -1;                    // hanging node
        c.nne_start[i + 1] += c.nne_start[i];
    }
    c.nne.assign(c.nne_start[np], 0);
    {
        std::vector<int32_t> fill(c.nne_start.begin(), c.nne_start.end() - 1);
        for (int e = 0; e < ne; ++e)
            for (int j = 0; j < i34[e]; ++j) c.nne[fill[elnode[4 * e + j]]++] = e;
    }
    // neighbour element across each local side: the first element in the (element-ordered)
    // ball of the side's first node that also holds its second node (:272-328)
    c.ic3.assign(4 * (size_t)ne, -1);
    for (int e = 0; e < ne; ++e) {
        const int n = i34[e];
        for (int k = 0; k < n; ++k) {
            const int a = elnode[4 * e + wrap(k + 1, n)], b = elnode[4 * e + wrap(k + 2, n)];
            int other = -1;
            for (int q = c.nne_start[a]; q < c.nne_start[a + 1] && other < 0; ++q) {
                const int je = c.nne[q];
                if (je != e && local_of(&elnode[4 * je], i34[je], b) >= 0) other = je;
            }
            c.ic3[4 * e + k] = other;
            if (other >= 0) {                                          // same orientation -> error
                for (int l = 0; l < i34[other]; ++l)
                    if (elnode[4 * other + l] == a && elnode[4 * other + wrap(l + 1, i34[other])] == b) return -2;
            }
        }
    }
    // global side numbering in element order; an interior side takes its number at the
    // element with the smaller index (:331-375)
    c.elside.assign(4 * (size_t)ne, -1);
    int ns = 0;
    for (int e = 0; e < ne; ++e) {
        for (int j = 0; j < i34[e]; ++j) {
            const int je = c.ic3[4 * e + j];
            if (je < 0) { c.elside[4 * e + j] = ns++; continue; }
            if (e > je) continue;
            int l = -1;
            for (int k = 0; k < i34[je] && l < 0; ++k)
                if (c.ic3[4 * je + k] == e) l = k;
            if (l < 0) return -3;
            c.elside[4 * e + j] = ns;
            c.elside[4 * je + l] = ns;
            ++ns;
        }
    }
    if (ns < ne || ns < np) return -4;
    c.ns = ns;
    c.isdel.assign(2 * (size_t)ns, -1);
    c.isidenode.assign(2 * (size_t)ns, -1);
    for (int e = 0; e < ne; ++e) {                                     // :392-428
        const int n = i34[e];
        for (int j = 0; j < n; ++j) {
            const int s = c.elside[4 * e + j];
            if (s < 0) return -5;
            const int a = elnode[4 * e + wrap(j + 1, n)], b = elnode[4 * e + wrap(j + 2, n)];
            const int je = c.ic3[4 * e + j];
            const bool owner = (je < 0) || (e < je);
            c.isdel[2 * s] = owner ? e : je;
            c.isdel[2 * s + 1] = owner ? je : e;
            c.isidenode[2 * s] = owner ? a : b;
            c.isidenode[2 * s + 1] = owner ? b : a;
        }
    }
    // counter-clockwise ball: boundary nodes start at their boundary element; each next
    // element lies across local side (i-2) of the previous one (:496-574)
    for (int i = 0; i < np; ++i) {
        const int s0 = c.nne_start[i], s1 = c.nne_start[i + 1];
        if (isbnd[i] != -1) {
            int found = 0;
            int first = -1;
            for (int q = s0; q < s1; ++q) {
                const int e = c.nne[q];
                const int il = local_of(&elnode[4 * e], i34[e], i);
                if (il < 0) return -6;
                if (c.ic3[4 * e + wrap(il - 1, i34[e])] == -1) { ++found; first = e; }
            }
            if (found != 1) return -7;
            c.nne[s0] = first;
        }
        for (int q = s0 + 1; q < s1; ++q) {
            const int e = c.nne[q - 1];
            const int il = local_of(&elnode[4 * e], i34[e], i);
            if (il < 0) return -6;
            const int nx = c.ic3[4 * e + wrap(il - 2, i34[e])];
            if (nx < 0) return -8;
            c.nne[q] = nx;
        }
    }
    // node -> nodes, counter-clockwise (:87-174)
    c.nnp_start.assign(np + 1, 0);
    for (int i = 0; i < np; ++i) {
        int cnt = 0;
        const int s0 = c.nne_start[i], s1 = c.nne_start[i + 1];
        for (int q = s0; q < s1; ++q) cnt += i34[c.nne[q]] - ((q == s1 - 1 && isbnd[i] != -1) ? 1 : 2);
        c.nnp_start[i + 1] = c.nnp_start[i] + cnt;
    }
    c.nnp.assign(c.nnp_start[np], 0);
    for (int i = 0; i < np; ++i) {
        int w = c.nnp_start[i];
        const int s0 = c.nne_start[i], s1 = c.nne_start[i + 1];
        for (int q = s0; q < s1; ++q) {
            const int e = c.nne[q];
            const int n = i34[e];
            const int il = local_of(&elnode[4 * e], n, i);
            if (il < 0) return -9;
            for (int k = 1; k < n - 1; ++k) c.nnp[w++] = elnode[4 * e + wrap(il + k, n)];
            if (q == s1 - 1) {
                const int last = elnode[4 * e + wrap(il + n - 1, n)];
                if (isbnd[i] == -1) {
                    if (last != c.nnp[c.nnp_start[i]]) return -10;       // broken ball
                } else {
                    c.nnp[w++] = last;
                }
            }
        }
    }
    return 0;
}

// Hilbert index of (x, y) on a 2^order grid (iterative quadrant rotation).
static uint64_t hilbert_d(uint32_t x, uint32_t y, int order) {
    uint64_t d = 0;
    for (uint32_t s = 1u << (order - 1); s > 0; s >>= 1) {
        const uint32_t rx = (x & s) ? 1u : 0u;
        const uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) { x = s - 1 - x; y = s - 1 - y; }
            std::swap(x, y);
        }
    }
    return d;
}

void hilbert_order(int n, const double* x, const double* y, std::vector<int32_t>& perm) {
    // perm[new] = old, sorted by the Hilbert index of the point in the bounding box
    double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
    for (int i = 0; i < n; ++i) {
        x0 = std::min(x0, x[i]); x1 = std::max(x1, x[i]);
        y0 = std::min(y0, y[i]); y1 = std::max(y1, y[i]);
    }
    const int order = 16;
    const double sx = (x1 > x0) ? ((1u << order) - 1) / (x1 - x0) : 0.0;
    const double sy = (y1 > y0) ? ((1u << order) - 1) / (y1 - y0) : 0.0;
    std::vector<std::pair<uint64_t, int32_t>> key(n);
    for (int i = 0; i < n; ++i) {
        const uint32_t hx = (uint32_t)((x[i] - x0) * sx), hy = (uint32_t)((y[i] - y0) * sy);
        key[i] = {hilbert_d(hx, hy, order), i};
    }
    std::sort(key.begin(), key.end());
    perm.resize(n);
    for (int i = 0; i < n; ++i) perm[i] = key[i].second;
}

}  // namespace gs

extern "C" gs_status gs_grid_build(int np, int ne, const int32_t* elnode, const int32_t* i34,
                                   const int32_t* isbnd, int32_t* nne_start, int32_t* nne,
                                   int32_t* nnp_start, int32_t* nnp, int32_t* ic3, int32_t* elside,
                                   int32_t* isdel, int32_t* isidenode, int32_t* ns_out) {
    if (np <= 0 || ne <= 0 || !elnode || !i34 || !isbnd) return GS_ERR_ARG;
    gs::Connectivity c;
    const int rc = gs::build_connectivity(np, ne, elnode, i34, isbnd, c);
    if (rc != 0) return GS_ERR_BAD_MESH;
    std::memcpy(nne_start, c.nne_start.data(), sizeof(int32_t) * (np + 1));
    std::memcpy(nne, c.nne.data(), sizeof(int32_t) * c.nne.size());
    std::memcpy(nnp_start, c.nnp_start.data(), sizeof(int32_t) * (np + 1));
    std::memcpy(nnp, c.nnp.data(), sizeof(int32_t) * c.nnp.size());
    std::memcpy(ic3, c.ic3.data(), sizeof(int32_t) * c.ic3.size());
    std::memcpy(elside, c.elside.data(), sizeof(int32_t) * c.elside.size());
    std::memcpy(isdel, c.isdel.data(), sizeof(int32_t) * c.isdel.size());
    std::memcpy(isidenode, c.isidenode.data(), sizeof(int32_t) * c.isidenode.size());
    *ns_out = c.ns;
    return GS_OK;
}
