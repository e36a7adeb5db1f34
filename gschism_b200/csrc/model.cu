// Context of gschism_b200: batch set-up, device state, phases of the step, CUDA-graph step,
// state exchange in reference numbering, and the stand-alone CSR JCG solver.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dev_common.cuh"
#include "kernels.h"

using namespace gs;

namespace {

struct MemberHost {
    // input copy (reference numbering)
    int np = 0, ne = 0, nope = 0, nland = 0, nbfr = 0;
    std::vector<double> x, y, depth, drag, tau, tr_init;
    std::vector<int32_t> elnode, open_start, open_nodes, land_start, land_nodes, iettype;
    std::vector<double> amig, ff, face, emo, efa;
    // derived
    Connectivity con;
    std::vector<int32_t> isbnd;
    std::vector<int32_t> pn, pe, ps;      // new -> old
    std::vector<int32_t> qn, qe, qs;      // old -> new
    int nnz = 0;
    int np0 = 0, ne0 = 0, ns0 = 0, nnz0 = 0, nb0 = 0;   // batch offsets
    std::vector<int32_t> csr_row_perm;    // helper for CSR export
};

struct HostBatch {
    // concatenated arrays in batch (new) numbering
    std::vector<double> x, y, depth, drag, tau, eta;
    std::vector<int32_t> nbnd, nne_s, nne, nne_loc, nnp_s, nnp, nbr_slot, diag_slot, sb1, sb2;
    std::vector<uint8_t> ess;
    std::vector<int32_t> indptr, indices;
    std::vector<int32_t> sn, se;         // [2][NS]
    std::vector<double> len, snx, sny, scx, scy, cori;
    std::vector<int8_t> sbt;
    std::vector<int32_t> en, es;         // [3][NE]
    std::vector<double> area, gphi;      // gphi: [3][NE] x,y interleaved
    std::vector<int8_t> ssgn;
    std::vector<int32_t> elem_member, mem_np0, mem_ne0;
    std::vector<int32_t> bn_node, bn_ietype, bn_nbfr;
    std::vector<double> bn_emo, bn_efa, bn_amig, bn_ff, bn_face;
    std::vector<double> tr, etr;         // [ntr][nvrt][NP], [ntr][nvrt][NE]
};

// Host-side result of gs_ctx_prepare, consumed (and released) by gs_ctx_finalize.
struct Prepared {
    HostBatch B;
    int NP = 0, NE = 0, NS = 0;
    std::vector<int32_t> en, es;          // [3][NE]
    std::vector<double> gphi;             // [3][NE][2]
    std::vector<int8_t> ssg;              // [3][NE]
    std::vector<ElemGeo> egeo;            // [NE]
    std::vector<int2> sell;               // SELL-32 slices
    std::vector<int32_t> sidx;            // SELL entries' columns
};

}  // namespace

struct gs_ctx {
    gs_config cfg{};
    std::vector<double> ztot, sigma;
    std::vector<MemberHost> mem;
    bool finalized = false;
    int dev = 0, nsm = 148;
    cudaStream_t st = nullptr;
    cudaStream_t own_st = nullptr;
    Dev d{};
    VG vg{};
    Phys P{};
    JcgWork* jw = nullptr;
    std::vector<void*> allocs;
    int it = 0;
    // gs_step replays one captured step; recaptured when storm forcing switches on or off
    cudaGraphExec_t graph = nullptr;
    int graph_vortex = -1;
    bool graph_failed = false;       // capture refused: gs_step launches the phases directly
    std::string err;
    std::vector<int> last_iters, last_outer;
    // batch CSR of the elevation matrix on the host (export) and each CSR entry's SELL position
    std::vector<int32_t> h_indptr, h_indices, h_csr2sell;
    // storm parameters per member ([nmem][kVortexParams]) and how many members have one
    std::vector<double> h_vort;
    int nvortex = 0;
    Prepared* prep = nullptr;        // host preparation awaiting gs_ctx_finalize
    LaunchTable launch;              // launch shapes (defaults or the autotuner's)
    double* mass_part = nullptr;     // tracer mass budget: per-block partials and result
    double* mass_out = nullptr;
    int stall_member = -1;           // recovery tests: the member whose solve waits run out
    // field exchange staging: one device block, two pinned host blocks used in turn (an event
    // per host block marks when its last copy has finished)
    void* dstage = nullptr;
    size_t dstage_bytes = 0;
    void* hstage[2] = {nullptr, nullptr};
    size_t hstage_bytes[2] = {0, 0};
    cudaEvent_t hev[2] = {nullptr, nullptr};
    int hnext = 0;
    // output marks (gs_output_mark / gs_output_wait): ticket -> event, and recycled events; a
    // writer thread may wait on a mark while the stepping thread records the next ones
    std::mutex marks_mu;
    uint64_t next_ticket = 1;
    std::map<uint64_t, cudaEvent_t> marks;
    std::vector<cudaEvent_t> free_events;
    gs_status fail(gs_status s, const std::string& m) { err = m; return s; }
};

namespace {

template <typename T>
cudaError_t dalloc(gs_ctx* c, T*& p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) { cudaMemsetAsync(q, 0, (n ? n : 1) * sizeof(T), c->own_st); c->allocs.push_back(q); p = (T*)q; }
    return e;
}

template <typename T>
cudaError_t dup(gs_ctx* c, T*& p, const std::vector<T>& h) {
    cudaError_t e = dalloc(c, p, h.size());
    if (e == cudaSuccess && !h.empty()) e = cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->own_st);
    return e;
}

void compute_isbnd(MemberHost& m) {
    // open nodes carry their segment index (last wins), land-only nodes -2, interior -1
    m.isbnd.assign(m.np, -1);
    for (int k = 0; k < m.nope; k++)
        for (int j = m.open_start[k]; j < m.open_start[k + 1]; j++) m.isbnd[m.open_nodes[j]] = k;
    for (int k = 0; k < m.nland; k++)
        for (int j = m.land_start[k]; j < m.land_start[k + 1]; j++)
            if (m.isbnd[m.land_nodes[j]] == -1) m.isbnd[m.land_nodes[j]] = -2;
}

int seg_of_pair(const std::vector<int32_t>& start, const std::vector<int32_t>& nodes, int nseg, int a, int b) {
    for (int k = 0; k < nseg; k++)
        for (int j = start[k]; j < start[k + 1] - 1; j++) {
            const int b1 = nodes[j], b2 = nodes[j + 1];
            if ((b1 == a && b2 == b) || (b1 == b && b2 == a)) return k;
        }
    return -1;
}

}  // namespace

// ============================================================================ C ABI ====

extern "C" {

gs_status gs_ctx_create(const gs_config* cfg, gs_ctx** out) {
    if (!cfg || !out) return GS_ERR_ARG;
    if (cfg->nvrt < 2 || cfg->nvrt > kMaxLevels || cfg->ntr < 0 || cfg->ntr > kMaxTracers || cfg->nz < 1 ||
        cfg->nz > cfg->nvrt)
        return GS_ERR_ARG;
    if ((cfg->itr_met != 0 && cfg->itr_met != 1 && cfg->itr_met != 3 && cfg->itr_met != 4) || cfg->tvd_limiter < 0 ||
        cfg->tvd_limiter > 4 || !(cfg->dfh0 >= 0.0))
        return GS_ERR_ARG;
    gs_ctx* c = new gs_ctx();
    c->cfg = *cfg;
    c->ztot.assign(cfg->ztot, cfg->ztot + cfg->nz);
    c->sigma.assign(cfg->sigma, cfg->sigma + (cfg->nvrt - cfg->nz + 1));
    c->cfg.ztot = c->ztot.data();
    c->cfg.sigma = c->sigma.data();
    if (c->cfg.check_every < 1) c->cfg.check_every = 1;
    if (c->cfg.maxiter < 1) c->cfg.maxiter = 1;
    if (c->cfg.ir_inner_maxiter < 1) c->cfg.ir_inner_maxiter = 200;
    if (!(c->cfg.ir_inner_rtol > 0.0)) c->cfg.ir_inner_rtol = 0.1;
    *out = c;
    return GS_OK;
}

gs_status gs_member_add(gs_ctx* c, const gs_member_desc* m, int* id) {
    if (!c || !m || c->finalized) return GS_ERR_ARG;
    if (m->np < 3 || m->ne < 1 || m->nbfr < 0 || m->nbfr > kMaxBfr) return c->fail(GS_ERR_ARG, "bad member sizes");
    MemberHost h;
    h.np = m->np; h.ne = m->ne; h.nope = m->nope; h.nland = m->nland; h.nbfr = m->nbfr;
    const int nvrt = c->cfg.nvrt, ntr = c->cfg.ntr;
    h.x.assign(m->x, m->x + m->np); h.y.assign(m->y, m->y + m->np); h.depth.assign(m->depth, m->depth + m->np);
    h.drag.assign(m->drag, m->drag + m->np); h.tau.assign(m->tau, m->tau + 2 * (size_t)m->np);
    h.tr_init.assign(m->tr_init, m->tr_init + (size_t)ntr * nvrt * m->np);
    h.elnode.assign(m->elnode, m->elnode + 3 * (size_t)m->ne);
    h.open_start.assign(m->open_start, m->open_start + m->nope + 1);
    const int non = m->nope ? m->open_start[m->nope] : 0;
    h.open_nodes.assign(m->open_nodes, m->open_nodes + non);
    h.land_start.assign(m->land_start, m->land_start + m->nland + 1);
    h.land_nodes.assign(m->land_nodes, m->land_nodes + (m->nland ? m->land_start[m->nland] : 0));
    h.iettype.assign(m->iettype, m->iettype + m->nope);
    h.amig.assign(m->amig, m->amig + m->nbfr); h.ff.assign(m->ff, m->ff + m->nbfr); h.face.assign(m->face, m->face + m->nbfr);
    h.emo.assign(m->emo, m->emo + (size_t)non * m->nbfr); h.efa.assign(m->efa, m->efa + (size_t)non * m->nbfr);
    for (int v : h.elnode) if (v < 0 || v >= m->np) return c->fail(GS_ERR_ARG, "element node out of range");
    *id = (int)c->mem.size();
    c->mem.push_back(std::move(h));
    return GS_OK;
}

const char* gs_last_error(const gs_ctx* c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"

// ----------------------------------------------------------------------- finalize ----

static gs_status build_member(gs_ctx* c, MemberHost& m, HostBatch& B, int mid) {
    const int nvrt = c->cfg.nvrt, ntr = c->cfg.ntr;
    compute_isbnd(m);
    std::vector<int32_t> el4(4 * (size_t)m.ne, -1), i34(m.ne, 3);
    for (int e = 0; e < m.ne; e++)
        for (int j = 0; j < 3; j++) el4[4 * e + j] = m.elnode[3 * e + j];
    if (build_connectivity(m.np, m.ne, el4.data(), i34.data(), m.isbnd.data(), m.con) != 0)
        return c->fail(GS_ERR_BAD_MESH, "mesh connectivity check failed");
    const Connectivity& C = m.con;
    const int np = m.np, ne = m.ne, ns = C.ns;
    // space-filling-curve order of nodes, elements (centroids) and sides (midpoints)
    hilbert_order(np, m.x.data(), m.y.data(), m.pn);
    {
        std::vector<double> cx(ne), cy(ne);
        for (int e = 0; e < ne; e++) {
            cx[e] = (m.x[m.elnode[3 * e]] + m.x[m.elnode[3 * e + 1]] + m.x[m.elnode[3 * e + 2]]) / 3.0;
            cy[e] = (m.y[m.elnode[3 * e]] + m.y[m.elnode[3 * e + 1]] + m.y[m.elnode[3 * e + 2]]) / 3.0;
        }
        hilbert_order(ne, cx.data(), cy.data(), m.pe);
        std::vector<double> sx(ns), sy(ns);
        for (int s = 0; s < ns; s++) {
            sx[s] = 0.5 * (m.x[C.isidenode[2 * s]] + m.x[C.isidenode[2 * s + 1]]);
            sy[s] = 0.5 * (m.y[C.isidenode[2 * s]] + m.y[C.isidenode[2 * s + 1]]);
        }
        hilbert_order(ns, sx.data(), sy.data(), m.ps);
    }
    m.qn.assign(np, 0); m.qe.assign(ne, 0); m.qs.assign(ns, 0);
    for (int i = 0; i < np; i++) m.qn[m.pn[i]] = i;
    for (int i = 0; i < ne; i++) m.qe[m.pe[i]] = i;
    for (int i = 0; i < ns; i++) m.qs[m.ps[i]] = i;
    const int NP0 = (int)B.x.size(), NE0 = (int)B.area.size(), NS0 = (int)B.len.size();
    m.np0 = NP0; m.ne0 = NE0; m.ns0 = NS0;
    m.nnz0 = (int)B.indices.size();
    // nodes
    for (int i = 0; i < np; i++) {
        const int o = m.pn[i];
        B.x.push_back(m.x[o]); B.y.push_back(m.y[o]); B.depth.push_back(m.depth[o]); B.drag.push_back(m.drag[o]);
        B.tau.push_back(m.tau[2 * o]); B.tau.push_back(m.tau[2 * o + 1]);
        B.nbnd.push_back(m.isbnd[o]);
    }
    // node -> elements with the node's local index, node -> nodes, CSR rows sorted by column
    for (int i = 0; i < np; i++) {
        const int o = m.pn[i];
        for (int q = C.nne_start[o]; q < C.nne_start[o + 1]; q++) {
            const int eo = C.nne[q];
            int loc = -1;
            for (int j = 0; j < 3; j++) if (m.elnode[3 * eo + j] == o) loc = j;
            B.nne.push_back(NE0 + m.qe[eo]);
            B.nne_loc.push_back(loc);
        }
        B.nne_s.push_back((int)B.nne.size());
        const int rs = (int)B.indices.size();
        std::vector<std::pair<int, int>> cols;   // (new column, position in the ball or -1 for diag)
        const int s0 = C.nnp_start[o], s1 = C.nnp_start[o + 1];
        if (s1 - s0 > kMaxDeg) return c->fail(GS_ERR_BAD_MESH, "node degree above the supported maximum");
        cols.push_back({i, -1});
        for (int a = s0; a < s1; a++) cols.push_back({m.qn[C.nnp[a]], a - s0});
        std::sort(cols.begin(), cols.end());
        std::vector<int32_t> slot(s1 - s0, 0);
        int dslot = 0;
        for (size_t r = 0; r < cols.size(); r++) {
            B.indices.push_back(NP0 + cols[r].first);
            if (cols[r].second < 0) dslot = rs + (int)r;
            else slot[cols[r].second] = rs + (int)r;
        }
        B.diag_slot.push_back(dslot);
        for (int a = s0; a < s1; a++) { B.nnp.push_back(NP0 + m.qn[C.nnp[a]]); B.nbr_slot.push_back(slot[a - s0]); }
        B.nnp_s.push_back((int)B.nnp.size());
        B.indptr.push_back((int)B.indices.size());
        B.sb1.push_back(-1); B.sb2.push_back(-1);
        B.ess.push_back(0);
    }
    m.nnz = (int)B.indices.size() - m.nnz0;
    // open boundary nodes: the last matching (segment, position) provides the constituents
    std::vector<int> bn_pos(np, -1);
    for (int k = 0; k < m.nope; k++)
        for (int j = m.open_start[k]; j < m.open_start[k + 1]; j++) {
            const int o = m.open_nodes[j];
            B.ess[NP0 + m.qn[o]] = (m.iettype[k] != 0);
            bn_pos[o] = j;
        }
    m.nb0 = (int)B.bn_node.size();
    for (int i = 0; i < np; i++) {
        const int o = m.pn[i];
        if (m.isbnd[o] < 0) continue;
        const int j = bn_pos[o];
        B.bn_node.push_back(NP0 + i);
        B.bn_ietype.push_back(m.iettype[m.isbnd[o]]);
        B.bn_nbfr.push_back(m.nbfr);
        for (int f = 0; f < kMaxBfr; f++) {
            const bool ok = f < m.nbfr && j >= 0;
            B.bn_emo.push_back(ok ? m.emo[(size_t)j * m.nbfr + f] : 0.0);
            B.bn_efa.push_back(ok ? m.efa[(size_t)j * m.nbfr + f] : 0.0);
            B.bn_amig.push_back(f < m.nbfr ? m.amig[f] : 0.0);
            B.bn_ff.push_back(f < m.nbfr ? m.ff[f] : 0.0);
            B.bn_face.push_back(f < m.nbfr ? m.face[f] : 0.0);
        }
    }
    // sides (geometry as populateSides, meshdata.cu:2146-2347; boundary type and open-node links
    // in reference side order)
    std::vector<int8_t> sbt_old(ns, 0);
    std::vector<int32_t> sb1(np, -1), sb2(np, -1);
    for (int s = 0; s < ns; s++) {
        const int a = C.isidenode[2 * s], b = C.isidenode[2 * s + 1];
        if (m.isbnd[a] != -1 && m.isbnd[b] != -1) {
            if (seg_of_pair(m.land_start, m.land_nodes, m.nland, a, b) >= 0) sbt_old[s] = 1;
            else if (seg_of_pair(m.open_start, m.open_nodes, m.nope, a, b) >= 0) sbt_old[s] = 2;
            if (sbt_old[s]) {
                const int nn[2] = {a, b};
                for (int qq = 0; qq < 2; qq++) {
                    const int i = nn[qq];
                    if (m.isbnd[i] < 0) continue;
                    if (sb1[i] < 0) sb1[i] = s; else if (sb2[i] < 0) sb2[i] = s;
                }
            }
        }
    }
    for (int i = 0; i < np; i++) {
        const int o = m.pn[i];
        B.sb1[NP0 + i] = sb1[o] >= 0 ? NS0 + m.qs[sb1[o]] : -1;
        B.sb2[NP0 + i] = sb2[o] >= 0 ? NS0 + m.qs[sb2[o]] : -1;
    }
    for (int s = 0; s < ns; s++) {
        const int so = m.ps[s];
        const int a = C.isidenode[2 * so], b = C.isidenode[2 * so + 1];
        const int e0 = C.isdel[2 * so], e1 = C.isdel[2 * so + 1];
        B.sn.push_back(NP0 + m.qn[a]);
        B.se.push_back(e0 >= 0 ? NE0 + m.qe[e0] : -1);
        B.scx.push_back(0.5 * (m.x[a] + m.x[b]));
        B.scy.push_back(0.5 * (m.y[a] + m.y[b]));
        const double nx = -(m.y[a] - m.y[b]), ny = (m.x[a] - m.x[b]);
        const double ln = std::sqrt(nx * nx + ny * ny);
        B.snx.push_back(nx / ln); B.sny.push_back(ny / ln);
        const double dx = m.x[b] - m.x[a], dy = m.y[b] - m.y[a], dz = 0.0 - 0.0;
        B.len.push_back(std::sqrt(dx * dx + dy * dy + dz * dz));
        B.cori.push_back(c->cfg.coricoef);
        B.sbt.push_back(sbt_old[so]);
        (void)e1;
    }
    // second rows of the [2][NS] side arrays are appended after all members (see finalize)
    // elements (populateElements, meshdata.cu:2350-2480)
    for (int e = 0; e < ne; e++) {
        const int eo = m.pe[e];
        const int* nd = &m.elnode[3 * eo];
        const double x0 = m.x[nd[0]], y0 = m.y[nd[0]], x1 = m.x[nd[1]], y1 = m.y[nd[1]], x2 = m.x[nd[2]], y2 = m.y[nd[2]];
        const double area = 0.5 * ((x0 - x2) * (y1 - y2) - (x1 - x2) * (y0 - y2));
        B.area.push_back(area);
        B.elem_member.push_back(mid);
    }
    (void)nvrt; (void)ntr;
    return GS_OK;
}

// Host half of finalize: connectivity, space-filling-curve order, batch arrays, matrix layout and
// element geometry, with no CUDA call, so it can run on any thread while the GPU is busy.
static gs_status prepare_host(gs_ctx* c) {
    const int nvrt = c->cfg.nvrt, ntr = c->cfg.ntr;
    Prepared* pr = new Prepared();
    std::unique_ptr<Prepared> guard(pr);
    HostBatch& B = pr->B;
    B.nne_s.push_back(0); B.nnp_s.push_back(0); B.indptr.push_back(0);
    for (size_t k = 0; k < c->mem.size(); k++) {
        B.mem_np0.push_back((int)B.x.size());
        B.mem_ne0.push_back((int)B.area.size());
        gs_status s = build_member(c, c->mem[k], B, (int)k);
        if (s != GS_OK) return s;
    }
    const int NP = (int)B.x.size(), NE = (int)B.area.size(), NS = (int)B.len.size();
    pr->NP = NP; pr->NE = NE; pr->NS = NS;
    B.mem_np0.push_back(NP); B.mem_ne0.push_back(NE);
    // second halves of [2][NS] and the [3][NE] arrays, geometry of elements, initial tracers
    std::vector<int32_t> sn2(NS), se2(NS);
    std::vector<int32_t>& en = pr->en;
    std::vector<int32_t>& es = pr->es;
    std::vector<double>& gphi = pr->gphi;
    std::vector<int8_t>& ssg = pr->ssg;
    en.assign(3 * (size_t)NE, 0); es.assign(3 * (size_t)NE, 0);
    gphi.assign(6 * (size_t)NE, 0.0);
    ssg.assign(3 * (size_t)NE, 0);
    B.tr.assign((size_t)ntr * nvrt * NP, 0.0);
    B.etr.assign((size_t)ntr * nvrt * NE, 0.0);
    for (auto& m : c->mem) {
        const Connectivity& C = m.con;
        for (int s = 0; s < C.ns; s++) {
            const int so = m.ps[s];
            sn2[m.ns0 + s] = m.np0 + m.qn[C.isidenode[2 * so + 1]];
            const int e1 = C.isdel[2 * so + 1];
            se2[m.ns0 + s] = e1 >= 0 ? m.ne0 + m.qe[e1] : -1;
        }
        for (int e = 0; e < m.ne; e++) {
            const int eo = m.pe[e], E = m.ne0 + e;
            const int* nd = &m.elnode[3 * eo];
            const double area = B.area[E];
            for (int j = 0; j < 3; j++) {
                en[(size_t)j * NE + E] = m.np0 + m.qn[nd[j]];
                const int so = C.elside[4 * eo + j];
                es[(size_t)j * NE + E] = m.ns0 + m.qs[so];
                ssg[(size_t)j * NE + E] = (C.isdel[2 * so] == eo) ? 1 : -1;
                const int p2 = nd[(j + 1) % 3], p3 = nd[(j + 2) % 3];
                gphi[2 * ((size_t)j * NE + E)] = (m.y[p2] - m.y[p3]) / (2 * area);
                gphi[2 * ((size_t)j * NE + E) + 1] = (m.x[p3] - m.x[p2]) / (2 * area);
            }
            // initial element tracers: node levels k and k-1 averaged, level 0 = level 1
            const double inv = 1.0 / (2.0 * 3);
            for (int t = 0; t < ntr; t++) {
                for (int k = 1; k < nvrt; k++) {
                    double sum = 0.0;
                    for (int j = 0; j < 3; j++)
                        sum += m.tr_init[((size_t)t * nvrt + k) * m.np + nd[j]] +
                               m.tr_init[((size_t)t * nvrt + k - 1) * m.np + nd[j]];
                    B.etr[((size_t)t * nvrt + k) * NE + E] = inv * sum;
                }
                B.etr[((size_t)t * nvrt + 0) * NE + E] = B.etr[((size_t)t * nvrt + 1) * NE + E];
            }
        }
        for (int t = 0; t < ntr; t++)
            for (int k = 0; k < nvrt; k++)
                for (int i = 0; i < m.np; i++)
                    B.tr[((size_t)t * nvrt + k) * NP + m.np0 + i] = m.tr_init[((size_t)t * nvrt + k) * m.np + m.pn[i]];
    }
    B.sn.insert(B.sn.end(), sn2.begin(), sn2.end());
    B.se.insert(B.se.end(), se2.begin(), se2.end());
    // backtracking records: corners in node order, and the node that starts each side in the
    // element's orientation (the side's first node when the element is the side's first element)
    pr->egeo.resize(NE);
    for (int E = 0; E < NE; E++) {
        ElemGeo& g = pr->egeo[E];
        std::memset(&g, 0, sizeof(g));
        for (int j = 0; j < 3; j++) {
            const int n = en[(size_t)j * NE + E];
            g.p[j].x = B.x[n]; g.p[j].y = B.y[n];
            g.n[j] = n;
        }
        g.area = B.area[E];
        for (int j = 0; j < 3; j++) {
            const int s = es[(size_t)j * NE + E];
            const int start = ssg[(size_t)j * NE + E] > 0 ? B.sn[s] : B.sn[(size_t)NS + s];
            const int c = (start == g.n[0]) ? 0 : (start == g.n[1]) ? 1 : 2;
            g.perm |= c << (2 * j);
        }
        // obtuse-corner flags of the walk predicates: side j and side j+1 (in side order) make an
        // obtuse angle at their shared corner when their direction vectors point the same way
        double2 C[3];
        for (int j = 0; j < 3; j++) C[j] = g.p[(g.perm >> (2 * j)) & 3];
        double2 sv[3];
        for (int j = 0; j < 3; j++) {
            const double2 a = C[j], b = C[(j + 1) % 3];
            sv[j].x = b.x - a.x; sv[j].y = b.y - a.y;
        }
        for (int j = 0; j < 3; j++) {
            const double2 u = sv[j], w = sv[(j + 1) % 3];
            if (u.x * w.x + u.y * w.y > 0.0) g.perm |= 1 << (8 + j);
        }
    }

    // SELL-32 layout of the batch matrix; assembly slots move to their SELL positions
    std::vector<int2>& sell = pr->sell;
    std::vector<int32_t>& sidx = pr->sidx;
    {
        const int nsl = (NP + 31) / 32;
        sell.resize(nsl);
        c->h_csr2sell.assign(B.indices.size(), 0);
        long long off = 0;
        for (int s = 0; s < nsl; s++) {
            int w = 0;
            for (int i = 32 * s; i < std::min(NP, 32 * s + 32); i++) w = std::max(w, B.indptr[i + 1] - B.indptr[i]);
            sell[s].x = (int)off; sell[s].y = w;
            off += 32LL * w;
            if (off > 0x7fffffffLL) return c->fail(GS_ERR_ARG, "elevation matrix too large for 32-bit offsets");
        }
        sidx.assign((size_t)off, 0);
        for (int s = 0; s < nsl; s++)
            for (int l = 0; l < 32; l++) {
                const int i = 32 * s + l;
                for (int k = 0; k < sell[s].y; k++) {
                    const size_t pos = (size_t)sell[s].x + 32 * (size_t)k + l;
                    if (i < NP && k < B.indptr[i + 1] - B.indptr[i]) {
                        sidx[pos] = B.indices[B.indptr[i] + k];
                        c->h_csr2sell[B.indptr[i] + k] = (int32_t)pos;
                    } else {
                        sidx[pos] = std::min(i, NP - 1);
                    }
                }
            }
        for (auto& v : B.nbr_slot) v = c->h_csr2sell[v];
        for (auto& v : B.diag_slot) v = c->h_csr2sell[v];
        c->h_indptr = B.indptr;
        c->h_indices = B.indices;
    }
    c->prep = guard.release();
    return GS_OK;
}

extern "C" gs_status gs_ctx_prepare(gs_ctx* c) {
    if (!c || c->finalized) return GS_ERR_ARG;
    if (c->prep) return GS_OK;
    if (c->mem.empty()) return c->fail(GS_ERR_ARG, "no members");
    return prepare_host(c);
}

extern "C" gs_status gs_ctx_finalize(gs_ctx* c) {
    if (!c || c->finalized) return GS_ERR_ARG;
    if (c->mem.empty()) return c->fail(GS_ERR_ARG, "no members");
    if (!c->prep) {
        const gs_status ps = prepare_host(c);
        if (ps != GS_OK) return ps;
    }
    std::unique_ptr<Prepared> pr(c->prep);     // released when finalize returns
    c->prep = nullptr;
    cudaError_t ce = cudaSetDevice(c->cfg.device);
    if (ce != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(ce));
    c->dev = c->cfg.device;
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->dev);
    if (!coop) return c->fail(GS_ERR_CUDA, "device lacks cooperative launch");
    // uploads, clears and set-up kernels go to the context's own non-blocking stream
    if (cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking) != cudaSuccess) return c->fail(GS_ERR_CUDA, "stream");
    c->st = c->own_st;
    const int nvrt = c->cfg.nvrt, ntr = c->cfg.ntr;
    HostBatch& B = pr->B;
    const int NP = pr->NP, NE = pr->NE, NS = pr->NS;
    const std::vector<int32_t>& en = pr->en;
    const std::vector<int32_t>& es = pr->es;
    const std::vector<double>& gphi = pr->gphi;
    const std::vector<int8_t>& ssg = pr->ssg;
    const std::vector<int2>& sell = pr->sell;
    const std::vector<int32_t>& sidx = pr->sidx;
    Dev& d = c->d;
    d.NP = NP; d.NE = NE; d.NS = NS; d.NNZ = (int)sidx.size(); d.NB = (int)B.bn_node.size();
    d.nmem = (int)c->mem.size();
    cudaError_t e = cudaSuccess;
#define UP(field, vec) if (e == cudaSuccess) e = dup(c, d.field, vec)
#define AL(field, n) if (e == cudaSuccess) e = dalloc(c, d.field, n)
    UP(x, B.x); UP(y, B.y); UP(depth, B.depth); UP(drag, B.drag); UP(tau, B.tau); UP(tau_own, B.tau);
    {
        std::vector<int32_t> pn(NP), ps(NS), pe(NE);
        for (const MemberHost& m : c->mem) {
            for (int i = 0; i < m.np; i++) pn[m.np0 + i] = m.pn[i];
            for (int i = 0; i < m.con.ns; i++) ps[m.ns0 + i] = m.ps[i];
            for (int i = 0; i < m.ne; i++) pe[m.ne0 + i] = m.pe[i];
        }
        UP(pn_ref, pn); UP(ps_ref, ps); UP(pe_ref, pe);
    }
    AL(eta1, NP); AL(eta2, NP); AL(qel, NP); AL(elbc, NP); AL(kb, NP); AL(ndry, NP); AL(nwas, NP);
    UP(ess, B.ess); UP(nbnd, B.nbnd);
    AL(z, (size_t)nvrt * NP); AL(w2, (size_t)nvrt * NP); AL(u2, (size_t)nvrt * NP);
    UP(tr, B.tr);
    UP(nne_s, B.nne_s); UP(nne, B.nne); UP(nne_loc, B.nne_loc); UP(nnp_s, B.nnp_s); UP(nnp, B.nnp);
    UP(nbr_slot, B.nbr_slot); UP(diag_slot, B.diag_slot); UP(sb1, B.sb1); UP(sb2, B.sb2);
    UP(bn_node, B.bn_node); UP(bn_ietype, B.bn_ietype); UP(bn_nbfr, B.bn_nbfr);
    UP(bn_emo, B.bn_emo); UP(bn_efa, B.bn_efa); UP(bn_amig, B.bn_amig); UP(bn_ff, B.bn_ff); UP(bn_face, B.bn_face);
    UP(sell, sell); UP(indices, sidx); AL(A, d.NNZ); AL(A32, d.NNZ);
    AL(b, NP); AL(xs, NP); AL(r, NP); AL(zz, NP); AL(p0, NP); AL(p1, NP); AL(q, NP); AL(invD, NP);
    AL(xh0, NP); AL(xh1, NP); AL(xh2, NP);
    AL(ir32, (size_t)kIrVectors * NP); AL(diag32, NP);
    UP(sn, B.sn); UP(se, B.se); UP(len, B.len); UP(snx, B.snx); UP(sny, B.sny); UP(scx, B.scx); UP(scy, B.scy);
    UP(cori, B.cori); AL(kbs, NS); AL(sdry, NS); UP(sbt, B.sbt);
    AL(zc, (size_t)nvrt * NS); AL(Qh, (size_t)nvrt * NS); AL(su2, (size_t)nvrt * NS); AL(btu, (size_t)nvrt * NS);
    AL(btel, (size_t)nvrt * NS); AL(U, NS); AL(gE1, NS); AL(gE2, NS); AL(sgh, 3 * (size_t)NS); AL(hhat, NS); AL(chi, NS); AL(chi2, NS);
    UP(en, en); UP(es, es); UP(area, B.area);
    if (e == cudaSuccess) { e = dalloc(c, d.gphi, 3 * (size_t)NE); if (e == cudaSuccess) e = cudaMemcpyAsync(d.gphi, gphi.data(), gphi.size() * 8, cudaMemcpyHostToDevice, c->own_st); }
    UP(ssgn, ssg); AL(kbe, NE); AL(edry, NE);
    if (e == cudaSuccess) { e = dalloc(c, d.egeo, NE); if (e == cudaSuccess) e = cudaMemcpyAsync(d.egeo, pr->egeo.data(), pr->egeo.size() * sizeof(ElemGeo), cudaMemcpyHostToDevice, c->own_st); }
    AL(ez, (size_t)nvrt * NE); AL(ew, (size_t)nvrt * NE); AL(Qv, (size_t)nvrt * NE);
    UP(etr, B.etr); AL(prev, (size_t)ntr * nvrt * NE);
    if (c->cfg.itr_met >= 3) AL(tvds, (size_t)ntr * nvrt * NE);
    if (c->cfg.itr_met == 4) AL(vgam, (size_t)nvrt * NE);
    AL(maxDt, NE); AL(ghat, NE);
    if (ntr >= 2) { AL(rho_n, (size_t)nvrt * NP); AL(rho_e, (size_t)nvrt * NE); }
    UP(mem_np0, B.mem_np0); UP(mem_ne0, B.mem_ne0); UP(elem_member, B.elem_member);
    c->h_vort.assign((size_t)kVortexParams * c->mem.size(), 0.0);
    UP(vort, c->h_vort);
    AL(mem_start, d.nmem);
    AL(mem_rem, 2 * (size_t)d.nmem); AL(mem_dtb, d.nmem); AL(mem_mindt, 2 * (size_t)d.nmem + 1); AL(mem_nsub, d.nmem);
    AL(clk, 3); AL(bar, 1); AL(err, 1); AL(counters, 4);
    d.wait_polls = kWaitPolls;
    if (e == cudaSuccess) e = dalloc(c, c->mass_part, (size_t)kMassBlocks * kMaxTracers * 2);
    if (e == cudaSuccess) e = dalloc(c, c->mass_out, (size_t)kMaxTracers);
#undef UP
#undef AL
    if (e != cudaSuccess) return c->fail(e == cudaErrorMemoryAllocation ? GS_ERR_OOM : GS_ERR_CUDA, cudaGetErrorString(e));
    {
        std::vector<int> row0, rows;
        for (auto& m : c->mem) { row0.push_back(m.np0); rows.push_back(m.np); }
        e = jcg_work_alloc(c->jw, row0, rows, true, c->own_st, c->launch.jcg);
        if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    }
    // constants
    Phys& P = c->P;
    const gs_config& g = c->cfg;
    P.nvrt = nvrt; P.ntr = ntr; P.nz = g.nz; P.h_s = g.h_s; P.h_c = g.h_c; P.theta_f = g.theta_f;
    P.dt = g.dt; P.thetai = g.thetai; P.h0 = g.h0; P.dtb_min = g.dtb_min; P.dtb_max = g.dtb_max;
    P.velmin = g.velmin_btrack; P.rmaxvel = g.rmaxvel; P.dfv0 = g.dfv0; P.coricoef = g.coricoef;
    P.rho0 = g.rho0; P.grav = g.grav; P.dramp = g.dramp; P.ihhat = g.ihhat;
    P.tvd = (g.itr_met >= 3); P.tvd_vert = (g.itr_met == 4); P.tvd_limiter = g.tvd_limiter; P.dfh0 = g.dfh0;
    VG& vg = c->vg;
    std::memset(&vg, 0, sizeof(vg));
    vg.nvrt = nvrt; vg.nz = g.nz; vg.h_s = g.h_s; vg.h_c = g.h_c; vg.h0 = g.h0;
    for (int k = 0; k < g.nz; k++) vg.ztot[k] = c->ztot[k];
    for (int k = 0; k < nvrt - g.nz + 1; k++) {
        const double s = c->sigma[k], tb = g.theta_b, tf = g.theta_f;
        vg.sigma[k] = s;
        vg.cs[k] = (1.0 - tb) * std::sinh(tf * s) / std::sinh(tf) +
                   tb * (std::tanh(tf * (s + 0.5)) - std::tanh(tf * 0.5)) / 2.0 / std::tanh(tf * 0.5);
    }
    // cold start levels (schism_init.py:81-91)
    launch_levels(c->d, c->P, c->vg, 0, c->st, c->nsm, c->launch);
    e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    c->finalized = true;
    return GS_OK;
}

// ------------------------------------------------------------------------- phases ----

static gs_status run_phase(gs_ctx* c, int phase, int arg) {
    const int nsm = c->nsm;
    cudaStream_t st = c->st;
    switch (phase) {
    case GS_PHASE_BEGIN: c->it = arg; launch_clock_set(c->d, c->P, arg, st); break;
    case GS_PHASE_BTRACK: launch_btrack(c->d, c->P, c->vg, st, nsm, c->launch); break;
    case GS_PHASE_PREPARE: launch_elev_prepare(c->d, c->P, c->nvortex > 0, st, nsm, c->launch); break;
    case GS_PHASE_ASSEMBLE:
        launch_assemble(c->d, c->P, st, nsm, c->launch);
        break;
    case GS_PHASE_SOLVE: {
        JcgArgs a{};
        Dev& d = c->d;
        a.n = d.NP; a.precision = c->cfg.precision;
        a.indptr = nullptr; a.sell = d.sell; a.indices = d.indices; a.A = d.A; a.A32 = d.A32; a.b = d.b; a.invD = d.invD;
        a.x = d.xs; a.r = d.r; a.z = d.zz; a.q = d.q; a.p0 = d.p0; a.p1 = d.p1;
        a.ir32 = d.ir32; a.diag32 = d.diag32;
        a.bar = d.bar; a.err = d.err;
        a.rtol = c->cfg.rtol; a.maxiter = c->cfg.maxiter; a.check_every = c->cfg.check_every;
        a.inner_rtol = c->cfg.ir_inner_rtol; a.inner_maxiter = c->cfg.ir_inner_maxiter;
        a.wait_polls = c->d.wait_polls; a.stall_member = c->stall_member;
        cudaError_t e = jcg_launch(a, c->jw, st, nsm);
        if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, std::string("jcg launch: ") + cudaGetErrorString(e));
        break;
    }
    case GS_PHASE_UPDATE_ELEV: launch_update_elev(c->d, c->vg, st, nsm); break;
    case GS_PHASE_MOMENTUM: launch_momentum(c->d, c->P, st, nsm, c->launch); break;
    case GS_PHASE_VVEL: launch_vvel(c->d, c->P, st, nsm, c->launch); break;
    case GS_PHASE_TRANSPORT: {
        cudaError_t e = launch_transport(c->d, c->P, c->cfg.dt, st, nsm, c->launch);
        if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, std::string("transport launch: ") + cudaGetErrorString(e));
        break;
    }
    case GS_PHASE_LEVELS: launch_levels(c->d, c->P, c->vg, arg, st, nsm, c->launch); break;
    case GS_PHASE_NODAL_VEL: launch_nodal_vel(c->d, c->P, st, nsm, c->launch); break;
    default: return c->fail(GS_ERR_ARG, "unknown phase");
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    return GS_OK;
}

static gs_status check_err(gs_ctx* c) {
    int32_t flags = 0;
    cudaError_t e = cudaMemcpyAsync(&flags, c->d.err, 4, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    if (flags & (ERR_BARRIER_TIMEOUT | ERR_DEGREE)) {
        // reported once: the barrier word (left mid-round by a timeout) and the flags are cleared,
        // so the context's next launches start clean
        cudaMemsetAsync(c->d.bar, 0, sizeof(unsigned), c->st);
        cudaMemsetAsync(c->d.err, 0, sizeof(int32_t), c->st);
        cudaStreamSynchronize(c->st);
        if (flags & ERR_BARRIER_TIMEOUT) return c->fail(GS_ERR_TIMEOUT, "a bounded device wait timed out");
        return c->fail(GS_ERR_BAD_MESH, "node degree above the supported maximum");
    }
    return GS_OK;
}

extern "C" {

gs_status gs_phase(gs_ctx* c, int phase, int arg) {
    if (!c || !c->finalized) return GS_ERR_ARG;
    return run_phase(c, phase, arg);
}

}  // extern "C"

// One step as a fixed launch sequence: advance the device clock, then every phase.  The LEVELS
// phase only tells the cold start (step 0) from a step, so any step index >= 1 gives the same
// launches.
static gs_status launch_step(gs_ctx* c) {
    launch_clock_advance(c->d, c->P, c->st);
    const int seq[] = {GS_PHASE_BTRACK, GS_PHASE_PREPARE, GS_PHASE_ASSEMBLE, GS_PHASE_SOLVE, GS_PHASE_UPDATE_ELEV,
                       GS_PHASE_MOMENTUM, GS_PHASE_VVEL, GS_PHASE_TRANSPORT, GS_PHASE_LEVELS, GS_PHASE_NODAL_VEL};
    for (int ph : seq) {
        const gs_status s = run_phase(c, ph, 1);
        if (s != GS_OK) return s;
    }
    return GS_OK;
}

// Capture one step into a CUDA graph (once, and again when storm forcing switches on or off).
// A refused capture leaves gs_step on direct launches.
static void ensure_graph(gs_ctx* c) {
    const int vort = c->nvortex > 0 ? 1 : 0;
    if (c->graph_failed || (c->graph && c->graph_vortex == vort)) return;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
    gs_status s = GS_OK;
    if (e == cudaSuccess) {
        s = launch_step(c);
        e = cudaStreamEndCapture(c->st, &g);
    }
    if (e == cudaSuccess && s == GS_OK) e = cudaGraphInstantiate(&c->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess || s != GS_OK) {
        c->graph = nullptr;
        c->graph_failed = true;
        cudaGetLastError();
        return;
    }
    c->graph_vortex = vort;
}

extern "C" {

gs_status gs_step(gs_ctx* c, int nsteps) {
    if (!c || !c->finalized || nsteps < 0) return GS_ERR_ARG;
    if (nsteps > 0) ensure_graph(c);
    for (int n = 0; n < nsteps; n++) {
        if (c->graph) {
            const cudaError_t e = cudaGraphLaunch(c->graph, c->st);
            if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(e));
        } else {
            const gs_status s = launch_step(c);
            if (s != GS_OK) return s;
        }
        c->it++;
    }
    return GS_OK;
}

gs_status gs_sync(gs_ctx* c) {
    if (!c || !c->finalized) return GS_ERR_ARG;
    return check_err(c);
}

gs_status gs_set_stream(gs_ctx* c, void* stream) {
    if (!c || !c->finalized) return GS_ERR_ARG;
    cudaStreamSynchronize(c->st);
    c->st = stream ? (cudaStream_t)stream : c->own_st;
    return GS_OK;
}

gs_status gs_member_sizes(gs_ctx* c, int member, int* np, int* ne, int* ns, int* nnz) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size()) return GS_ERR_ARG;
    const MemberHost& m = c->mem[member];
    *np = m.np; *ne = m.ne; *ns = m.con.ns; *nnz = m.nnz;
    return GS_OK;
}

gs_status gs_get_stats(gs_ctx* c, int member, gs_stats* out) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !out) return GS_ERR_ARG;
    gs_status s = check_err(c);
    std::vector<int> iters, outer;
    cudaError_t e = jcg_read_iters(c->jw, iters, outer, c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    unsigned long long cnt[4] = {0, 0, 0, 0};
    int32_t nsub = 0, flags = 0, jflags = 0;
    cudaMemcpyAsync(cnt, c->d.counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(&nsub, c->d.mem_nsub + member, 4, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(&flags, c->d.err, 4, cudaMemcpyDeviceToHost, c->st);
    cudaStreamSynchronize(c->st);
    jcg_read_status(c->jw, &jflags, c->st);
    flags |= jflags;   // non-convergence of the last solve (ERR_BARRIER_TIMEOUT was reported above)
    if (s == GS_ERR_TIMEOUT) flags |= ERR_BARRIER_TIMEOUT;
    std::memset(out, 0, sizeof(*out));
    out->jcg_iters = iters[member];
    out->jcg_outer = outer[member];
    out->transport_substeps = nsub;
    out->walk_cap_hits = (int64_t)cnt[0];
    out->btrack_stops = (int64_t)cnt[1];
    out->error_flags = flags;
    return s == GS_OK ? GS_OK : s;
}

static_assert((int)GS_K_BTRACK == (int)LK_BTRACK && (int)GS_K_SIDE_PREP == (int)LK_SIDE_PREP &&
                  (int)GS_K_GHAT == (int)LK_GHAT && (int)GS_K_ASSEMBLE == (int)LK_ASSEMBLE &&
                  (int)GS_K_MOMENTUM == (int)LK_MOMENTUM && (int)GS_K_VVEL == (int)LK_VVEL &&
                  (int)GS_K_NODAL_VEL == (int)LK_NODAL_VEL && (int)GS_K_NODAL_TRACER == (int)LK_NODAL_TRACER &&
                  (int)GS_K_LEVELS == (int)LK_LEVELS && (int)GS_K_JCG_TILES == (int)LK_COUNT,
              "launch ids of the C ABI");

static int max_threads_of(int kernel, int ntr) {
    switch (kernel) {
    case LK_BTRACK: return btrack_max_threads();
    case LK_SIDE_PREP: case LK_GHAT: case LK_ASSEMBLE: return elev_max_threads(kernel);
    case LK_MOMENTUM: case LK_VVEL: return mom_max_threads(kernel);
    case LK_NODAL_VEL: case LK_LEVELS: return levels_max_threads(kernel);
    case LK_NODAL_TRACER: return transport_max_threads(ntr);
    default: return 0;
    }
}

gs_status gs_set_launch(gs_ctx* c, int kernel, int a, int b) {
    if (!c || !c->finalized || kernel < 0 || kernel > GS_K_JCG_TILES) return GS_ERR_ARG;
    cudaSetDevice(c->dev);
    if (kernel == GS_K_JCG_TILES) {
        // a = tiles of a large member, b = smallest tile (rows, a multiple of 32); the cap of the
        // cooperative grid stays at its default
        if (a < 1 || a > 65536 || b < 32 || b > (1 << 24) || b % 32 != 0) return GS_ERR_ARG;
        JcgTiling tl = c->launch.jcg;
        tl.tiles = a; tl.min_rows = b;
        cudaError_t e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
        std::vector<int> row0, rows;
        for (auto& m : c->mem) { row0.push_back(m.np0); rows.push_back(m.np); }
        JcgWork* w = nullptr;
        e = jcg_work_alloc(w, row0, rows, true, c->own_st, tl);
        if (e != cudaSuccess) {
            jcg_work_free(w);
            return c->fail(e == cudaErrorMemoryAllocation ? GS_ERR_OOM : GS_ERR_CUDA, cudaGetErrorString(e));
        }
        jcg_work_free(c->jw);
        c->jw = w;
        c->launch.jcg = tl;
    } else {
        const int mx = max_threads_of(kernel, c->cfg.ntr);
        if (a < 32 || a % 32 != 0 || a > mx || b < 1 || b > 64) return GS_ERR_ARG;
        c->launch.k[kernel] = LaunchShape{a, b};
    }
    // the captured step holds the old shapes
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    c->graph_vortex = -1;
    return GS_OK;
}

gs_status gs_set_wait_limit(gs_ctx* c, long long polls) {
    if (!c || !c->finalized || polls < 0) return GS_ERR_ARG;
    c->d.wait_polls = polls > 0 ? polls : kWaitPolls;
    // the captured step holds the old bound in its kernel parameters
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    c->graph_vortex = -1;
    return GS_OK;
}

gs_status gs_test_stall_solve(gs_ctx* c, int member) {
    if (!c || !c->finalized || member < -1 || member >= (int)c->mem.size()) return GS_ERR_ARG;
    c->stall_member = member;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    c->graph_vortex = -1;
    return GS_OK;
}

gs_status gs_get_launch(gs_ctx* c, int kernel, int* a, int* b) {
    if (!c || !c->finalized || kernel < 0 || kernel > GS_K_JCG_TILES || !a || !b) return GS_ERR_ARG;
    if (kernel == GS_K_JCG_TILES) { *a = c->launch.jcg.tiles; *b = c->launch.jcg.min_rows; }
    else { *a = c->launch.k[kernel].block; *b = c->launch.k[kernel].per_sm; }
    return GS_OK;
}

gs_status gs_tracer_mass(gs_ctx* c, int member, double* out) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !out) return GS_ERR_ARG;
    const int ntr = c->cfg.ntr;
    if (ntr == 0) return GS_OK;
    const MemberHost& m = c->mem[member];
    cudaError_t e = launch_tracer_mass(c->d, c->P, m.ne0, m.ne0 + m.ne, c->mass_part, c->mass_out, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, c->mass_out, sizeof(double) * ntr, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    return GS_OK;
}

gs_status gs_ctx_destroy(gs_ctx* c) {
    if (!c) return GS_ERR_ARG;
    delete c->prep;
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->own_st) cudaStreamDestroy(c->own_st);
    jcg_work_free(c->jw);
    for (void* p : c->allocs) cudaFree(p);
    if (c->dstage) cudaFree(c->dstage);
    for (int k = 0; k < 2; k++) {
        if (c->hstage[k]) cudaFreeHost(c->hstage[k]);
        if (c->hev[k]) cudaEventDestroy(c->hev[k]);
    }
    for (auto& kv : c->marks) cudaEventDestroy(kv.second);
    for (cudaEvent_t ev : c->free_events) cudaEventDestroy(ev);
    delete c;
    return GS_OK;
}

}  // extern "C"

// --------------------------------------------------------------------- state exchange ----

namespace {

struct FieldInfo {
    char ent;       // 'N', 'S', 'E', 'C' (CSR), 'R' (CSR rows + 1)
    int lev;        // per-level
    int comp;       // 1, 2 (vector), -1 tracers
    int isint;      // 0 double, 1 int32, 2 uint8 (exchanged as int32)
    void* ptr;
};

bool field_info(gs_ctx* c, int f, FieldInfo& fi) {
    Dev& d = c->d;
    fi = FieldInfo{'N', 0, 1, 0, nullptr};
    switch (f) {
    case GS_F_ETA1: fi.ptr = d.eta1; return true;
    case GS_F_ETA2: fi.ptr = d.eta2; return true;
    case GS_F_QEL: fi.ptr = d.qel; return true;
    case GS_F_NODE_TAU: fi.comp = 2; fi.ptr = d.tau; return true;
    case GS_F_ELBC: fi.ptr = d.elbc; return true;
    case GS_F_JCG_X: fi.ptr = d.xh0; return true;
    case GS_F_JCG_X1: fi.ptr = d.xh1; return true;
    case GS_F_JCG_X2: fi.ptr = d.xh2; return true;
    case GS_F_NODE_Z: fi.lev = 1; fi.ptr = d.z; return true;
    case GS_F_NODE_U2: fi.lev = 1; fi.comp = 2; fi.ptr = d.u2; return true;
    case GS_F_NODE_W2: fi.lev = 1; fi.ptr = d.w2; return true;
    case GS_F_NODE_TR: fi.lev = 1; fi.comp = -1; fi.ptr = d.tr; return true;
    case GS_F_NODE_KB: fi.isint = 1; fi.ptr = d.kb; return true;
    case GS_F_NODE_DRY: fi.isint = 2; fi.ptr = d.ndry; return true;
    case GS_F_SIDE_U2: fi.ent = 'S'; fi.lev = 1; fi.comp = 2; fi.ptr = d.su2; return true;
    case GS_F_SIDE_BTU: fi.ent = 'S'; fi.lev = 1; fi.comp = 2; fi.ptr = d.btu; return true;
    case GS_F_SIDE_ZC: fi.ent = 'S'; fi.lev = 1; fi.ptr = d.zc; return true;
    case GS_F_SIDE_QH: fi.ent = 'S'; fi.lev = 1; fi.ptr = d.Qh; return true;
    case GS_F_SIDE_BTELEM: fi.ent = 'S'; fi.lev = 1; fi.isint = 1; fi.ptr = d.btel; return true;
    case GS_F_SIDE_KB: fi.ent = 'S'; fi.isint = 1; fi.ptr = d.kbs; return true;
    case GS_F_SIDE_DRY: fi.ent = 'S'; fi.isint = 2; fi.ptr = d.sdry; return true;
    case GS_F_SIDE_U: fi.ent = 'S'; fi.comp = 2; fi.ptr = d.U; return true;
    case GS_F_SIDE_HHAT: fi.ent = 'S'; fi.ptr = d.hhat; return true;
    case GS_F_SIDE_CHI: fi.ent = 'S'; fi.ptr = d.chi; return true;
    case GS_F_SIDE_GRADETA1: fi.ent = 'S'; fi.comp = 2; fi.ptr = d.gE1; return true;
    case GS_F_SIDE_GRADETA2: fi.ent = 'S'; fi.comp = 2; fi.ptr = d.gE2; return true;
    case GS_F_ELEM_Z: fi.ent = 'E'; fi.lev = 1; fi.ptr = d.ez; return true;
    case GS_F_ELEM_W: fi.ent = 'E'; fi.lev = 1; fi.ptr = d.ew; return true;
    case GS_F_ELEM_QV: fi.ent = 'E'; fi.lev = 1; fi.ptr = d.Qv; return true;
    case GS_F_ELEM_TR: fi.ent = 'E'; fi.lev = 1; fi.comp = -1; fi.ptr = d.etr; return true;
    case GS_F_ELEM_KB: fi.ent = 'E'; fi.isint = 1; fi.ptr = d.kbe; return true;
    case GS_F_ELEM_DRY: fi.ent = 'E'; fi.isint = 2; fi.ptr = d.edry; return true;
    case GS_F_ELEM_GHAT: fi.ent = 'E'; fi.comp = 2; fi.ptr = d.ghat; return true;
    case GS_F_NODE_RHO: fi.lev = 1; fi.ptr = d.rho_n; return d.rho_n != nullptr;
    case GS_F_ELEM_RHO: fi.ent = 'E'; fi.lev = 1; fi.ptr = d.rho_e; return d.rho_e != nullptr;
    case GS_F_CSR_DATA: fi.ent = 'C'; fi.ptr = d.A; return true;
    case GS_F_CSR_INDPTR: fi.ent = 'R'; fi.isint = 1; return true;
    case GS_F_CSR_INDICES: fi.ent = 'C'; fi.isint = 1; return true;
    default: return false;
    }
}

// reference-numbered CSR of one member: rows in reference node order, columns sorted by
// reference index, values gathered from the device matrix
void member_csr(gs_ctx* c, MemberHost& m, std::vector<int32_t>& indptr, std::vector<int32_t>& indices,
                std::vector<int32_t>& src) {
    const Connectivity& C = m.con;
    indptr.assign(m.np + 1, 0);
    indices.clear(); src.clear();
    const std::vector<int32_t>& hptr = c->h_indptr;
    const std::vector<int32_t>& hind = c->h_indices;
    for (int o = 0; o < m.np; o++) {
        const int i = m.np0 + m.qn[o];
        std::vector<std::pair<int, int>> row;
        for (int a = hptr[i]; a < hptr[i + 1]; a++) row.push_back({m.pn[hind[a] - m.np0], c->h_csr2sell[a]});
        std::sort(row.begin(), row.end());
        for (auto& pr : row) { indices.push_back(pr.first); src.push_back(pr.second); }
        indptr[o + 1] = (int)indices.size();
    }
    (void)C;
}

// One member's field as the exchange kernels see it (k_xfer.cu).
struct Block {
    int kind, n, N, off, nslices, nc;
    const int32_t* perm;
};

gs_status field_block(gs_ctx* c, const MemberHost& m, const FieldInfo& fi, size_t bytes, Block& k) {
    const Dev& d = c->d;
    k.kind = fi.isint == 2 ? 2 : (fi.isint ? 1 : 0);
    k.N = fi.ent == 'N' ? d.NP : fi.ent == 'S' ? d.NS : d.NE;
    k.n = fi.ent == 'N' ? m.np : fi.ent == 'S' ? m.con.ns : m.ne;
    k.off = fi.ent == 'N' ? m.np0 : fi.ent == 'S' ? m.ns0 : m.ne0;
    k.perm = (fi.ent == 'N' ? d.pn_ref : fi.ent == 'S' ? d.ps_ref : d.pe_ref) + k.off;
    k.nc = fi.comp == 2 ? 2 : 1;
    k.nslices = (fi.comp == -1 ? c->cfg.ntr : 1) * (fi.lev ? c->cfg.nvrt : 1);
    const size_t esz = fi.isint ? 4 : 8;
    if (bytes != (size_t)k.nslices * k.n * k.nc * esz) return c->fail(GS_ERR_STATE, "size mismatch for field");
    return GS_OK;
}

// Staging blocks of at least `bytes`: the device block and the next pinned host block (after its
// previous copy has finished).  Grows them on demand.
cudaError_t stage(gs_ctx* c, size_t bytes, int& h) {
    cudaError_t e = cudaSuccess;
    if (c->dstage_bytes < bytes) {
        if (c->dstage) { cudaStreamSynchronize(c->st); cudaFree(c->dstage); }
        c->dstage = nullptr; c->dstage_bytes = 0;
        e = cudaMalloc(&c->dstage, bytes);
        if (e != cudaSuccess) return e;
        c->dstage_bytes = bytes;
    }
    h = c->hnext;
    c->hnext ^= 1;
    if (!c->hev[h]) {
        e = cudaEventCreateWithFlags(&c->hev[h], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    } else {
        e = cudaEventSynchronize(c->hev[h]);
        if (e != cudaSuccess) return e;
    }
    if (c->hstage_bytes[h] < bytes) {
        if (c->hstage[h]) cudaFreeHost(c->hstage[h]);
        c->hstage[h] = nullptr; c->hstage_bytes[h] = 0;
        e = cudaHostAlloc(&c->hstage[h], bytes, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        c->hstage_bytes[h] = bytes;
    }
    return cudaSuccess;
}

bool page_locked(const void* p) {
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return pa.type == cudaMemoryTypeHost;
}

// Host block (reference order) -> device field, stream-ordered.  Pageable memory is copied to
// pinned staging before the call returns; page-locked memory is copied by the DMA engine straight
// from the caller's buffer and the call returns once that copy is done.  The upload and the
// scatter run on the context stream either way.
cudaError_t put_block(gs_ctx* c, const void* host, size_t bytes, void* dst, const Block& k) {
    int h = 0;
    cudaError_t e = stage(c, bytes, h);
    if (e != cudaSuccess) return e;
    const bool direct = page_locked(host);
    if (!direct) std::memcpy(c->hstage[h], host, bytes);
    e = cudaMemcpyAsync(c->dstage, direct ? host : c->hstage[h], bytes, cudaMemcpyHostToDevice, c->st);
    if (e != cudaSuccess) return e;
    cudaEventRecord(c->hev[h], c->st);
    launch_scatter(c->dstage, dst, k.kind, k.n, k.N, k.off, k.nslices, k.nc, k.perm, c->st, c->nsm);
    e = cudaGetLastError();
    if (e == cudaSuccess && direct) e = cudaEventSynchronize(c->hev[h]);
    return e;
}

}  // namespace

extern "C" gs_status gs_state_get(gs_ctx* c, int member, int field, void* host, size_t bytes) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !host) return GS_ERR_ARG;
    FieldInfo fi;
    if (!field_info(c, field, fi)) return c->fail(GS_ERR_STATE, "unknown field");
    // a bounded wait that ran out in the steps before (their results are incomplete) is
    // reported here, once, like gs_sync
    {
        const gs_status s = check_err(c);
        if (s != GS_OK) return s;
    }
    MemberHost& m = c->mem[member];
    if (fi.ent == 'C' || fi.ent == 'R') {
        if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->fail(GS_ERR_CUDA, "sync");
        std::vector<int32_t> ip, ix, src;
        member_csr(c, m, ip, ix, src);
        if (fi.ent == 'R') {
            if (bytes != 4 * ip.size()) return c->fail(GS_ERR_STATE, "size");
            std::memcpy(host, ip.data(), bytes);
        } else if (fi.isint) {
            if (bytes != 4 * ix.size()) return c->fail(GS_ERR_STATE, "size");
            std::memcpy(host, ix.data(), bytes);
        } else {
            if (bytes != 8 * src.size()) return c->fail(GS_ERR_STATE, "size");
            std::vector<double> all(c->d.NNZ);
            cudaMemcpyAsync(all.data(), c->d.A, 8 * (size_t)c->d.NNZ, cudaMemcpyDeviceToHost, c->st);
            cudaStreamSynchronize(c->st);
            double* out = (double*)host;
            for (size_t a = 0; a < src.size(); a++) out[a] = all[src[a]];
        }
        return GS_OK;
    }
    Block k;
    gs_status st = field_block(c, m, fi, bytes, k);
    if (st != GS_OK) return st;
    int h = 0;
    cudaError_t e = stage(c, bytes, h);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    launch_gather(fi.ptr, c->dstage, k.kind, k.n, k.N, k.off, k.nslices, k.nc, k.perm,
                  field == GS_F_SIDE_BTELEM ? c->d.pe_ref : nullptr, c->st, c->nsm);
    // page-locked destinations take the copy directly, others through pinned staging
    const bool direct = page_locked(host);
    e = cudaMemcpyAsync(direct ? host : c->hstage[h], c->dstage, bytes, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    if (!direct) std::memcpy(host, c->hstage[h], bytes);
    return GS_OK;
}

extern "C" gs_status gs_state_get_async(gs_ctx* c, int member, int field, void* host, size_t bytes) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !host) return GS_ERR_ARG;
    FieldInfo fi;
    if (!field_info(c, field, fi)) return c->fail(GS_ERR_STATE, "unknown field");
    if (fi.ent == 'C' || fi.ent == 'R') return c->fail(GS_ERR_STATE, "CSR fields have no asynchronous read");
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, host) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        return c->fail(GS_ERR_ARG, "gs_state_get_async needs page-locked host memory (gs_host_alloc)");
    }
    Block k;
    gs_status st = field_block(c, c->mem[member], fi, bytes, k);
    if (st != GS_OK) return st;
    cudaError_t e = cudaSuccess;
    if (c->dstage_bytes < bytes) {
        if (c->dstage) { cudaStreamSynchronize(c->st); cudaFree(c->dstage); }
        c->dstage = nullptr; c->dstage_bytes = 0;
        e = cudaMalloc(&c->dstage, bytes);
        if (e != cudaSuccess) return c->fail(GS_ERR_OOM, cudaGetErrorString(e));
        c->dstage_bytes = bytes;
    }
    launch_gather(fi.ptr, c->dstage, k.kind, k.n, k.N, k.off, k.nslices, k.nc, k.perm,
                  field == GS_F_SIDE_BTELEM ? c->d.pe_ref : nullptr, c->st, c->nsm);
    e = cudaMemcpyAsync(host, c->dstage, bytes, cudaMemcpyDeviceToHost, c->st);
    return e == cudaSuccess ? GS_OK : c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" gs_status gs_output_mark(gs_ctx* c, uint64_t* ticket) {
    if (!c || !c->finalized || !ticket) return GS_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->marks_mu);
    cudaEvent_t ev = nullptr;
    if (!c->free_events.empty()) { ev = c->free_events.back(); c->free_events.pop_back(); }
    else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return GS_ERR_CUDA;
    if (cudaEventRecord(ev, c->st) != cudaSuccess) { c->free_events.push_back(ev); return GS_ERR_CUDA; }
    *ticket = c->next_ticket++;
    c->marks[*ticket] = ev;
    return GS_OK;
}

extern "C" gs_status gs_output_wait(gs_ctx* c, uint64_t ticket) {
    if (!c || !c->finalized) return GS_ERR_ARG;
    cudaEvent_t ev = nullptr;
    {
        std::lock_guard<std::mutex> lk(c->marks_mu);
        auto it = c->marks.find(ticket);
        if (it == c->marks.end()) return GS_ERR_ARG;
        ev = it->second;
        c->marks.erase(it);
    }
    const cudaError_t e = cudaEventSynchronize(ev);
    std::lock_guard<std::mutex> lk(c->marks_mu);
    c->free_events.push_back(ev);
    return e == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}

extern "C" void* gs_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0 || cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    return p;
}

extern "C" gs_status gs_host_free(void* p) {
    if (!p) return GS_ERR_ARG;
    return cudaFreeHost(p) == cudaSuccess ? GS_OK : GS_ERR_CUDA;
}

extern "C" gs_status gs_state_put(gs_ctx* c, int member, int field, const void* host, size_t bytes) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !host) return GS_ERR_ARG;
    FieldInfo fi;
    if (!field_info(c, field, fi)) return c->fail(GS_ERR_STATE, "unknown field");
    if (fi.ent == 'C' || fi.ent == 'R') return c->fail(GS_ERR_STATE, "CSR fields are read-only");
    Block k;
    gs_status st = field_block(c, c->mem[member], fi, bytes, k);
    if (st != GS_OK) return st;
    cudaError_t e = put_block(c, host, bytes, fi.ptr, k);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    return GS_OK;
}

extern "C" gs_status gs_set_tau(gs_ctx* c, int member, const double* tau_host) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || !tau_host) return GS_ERR_ARG;
    FieldInfo fi;
    field_info(c, GS_F_NODE_TAU, fi);
    const MemberHost& m = c->mem[member];
    const size_t bytes = 16 * (size_t)m.np;
    Block k;
    gs_status st = field_block(c, m, fi, bytes, k);
    if (st != GS_OK) return st;
    // the member's own stress (kept for when a storm is switched off), then the live field
    cudaError_t e = put_block(c, tau_host, bytes, c->d.tau_own, k);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d.tau + 2 * (size_t)m.np0, c->d.tau_own + 2 * (size_t)m.np0, bytes,
                            cudaMemcpyDeviceToDevice, c->st);
    return e == cudaSuccess ? GS_OK : c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" gs_status gs_set_vortex(gs_ctx* c, int member, const gs_vortex* v) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size()) return GS_ERR_ARG;
    if (v && !(v->vmax > 0.0 && v->rmax > 0.0 && v->holland_b > 0.0 && v->rho_air > 0.0))
        return c->fail(GS_ERR_ARG, "vortex: vmax, rmax, holland_b and rho_air must be positive");
    double* p = c->h_vort.data() + (size_t)kVortexParams * member;
    const bool was = p[8] != 0.0;
    if (v) {
        const double q[kVortexParams] = {v->x0, v->y0, v->heading, v->speed, v->vmax, v->rmax, v->holland_b, v->rho_air, 1.0};
        for (int k = 0; k < kVortexParams; k++) p[k] = q[k];
    } else {
        for (int k = 0; k < kVortexParams; k++) p[k] = 0.0;
    }
    c->nvortex += (v ? 1 : 0) - (was ? 1 : 0);
    cudaError_t e = cudaMemcpyAsync(c->d.vort + (size_t)kVortexParams * member, p, sizeof(double) * kVortexParams,
                                    cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    if (!v && was) {
        // back to the member's own stress
        const MemberHost& m = c->mem[member];
        e = cudaMemcpyAsync(c->d.tau + 2 * (size_t)m.np0, c->d.tau_own + 2 * (size_t)m.np0, 16 * (size_t)m.np,
                            cudaMemcpyDeviceToDevice, c->st);
        if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    }
    return GS_OK;
}

extern "C" gs_status gs_set_member_start(gs_ctx* c, int member, int start_step) {
    if (!c || !c->finalized || member < 0 || member >= (int)c->mem.size() || start_step < 0) return GS_ERR_ARG;
    const double t0 = (double)start_step;
    cudaError_t e = cudaMemcpyAsync(c->d.mem_start + member, &t0, sizeof(double), cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    return GS_OK;
}

extern "C" gs_status gs_get_step(gs_ctx* c, int* step) {
    if (!c || !c->finalized || !step) return GS_ERR_ARG;
    double clk = 0.0;
    cudaError_t e = cudaMemcpyAsync(&clk, c->d.clk, sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return c->fail(GS_ERR_CUDA, cudaGetErrorString(e));
    *step = (int)clk;
    return GS_OK;
}

// Upper bound of the device bytes gs_ctx_finalize allocates for members of these total sizes
// (the allocation list of gs_ctx_finalize and jcg_work_alloc; boundary nodes counted as all nodes,
// SELL padding as a quarter of the entries, plus allocation granularity).
extern "C" size_t gs_footprint_bytes(int nvrt, int ntr, int nmem, int64_t np, int64_t ne, int64_t ns, int64_t nnz) {
    if (nvrt < 1 || ntr < 0 || nmem < 1 || np < 0 || ne < 0 || ns < 0 || nnz < 0) return 0;
    const double L = nvrt, T = ntr;
    const double sell = (double)nnz * 1.25 + 32.0 * kMaxDeg;
    double b = 0.0;
    const double R = ntr >= 2 ? 8.0 : 0.0;      // densities
    b += (double)np * (91.0 + L * (8 + 8 + 16 + 8 * T + R) + 20.0 + 88.0 + 4.0 * kIrVectors + 4.0 + 332.0 + 20.0);
    b += (double)ne * (24.0 + 88.0 + 24.0 + 4.0 + 80.0 + L * (24.0 + 16.0 * T + R) + 4.0);
    b += (double)ns * (16.0 + 70.0 + 72.0 + 16.0 + 48.0 + L * 52.0 + 4.0);
    b += std::max(L * 16.0 * (double)ns, L * 8.0 * T * (double)ne);   // field exchange staging (largest field)
    b += sell * 16.0 + (double)np / 32.0 * 8.0;
    b += ((double)np / 1024.0 + nmem) * 84.0 + (double)nmem * (16.0 + 72.0 + 40.0 + 8.0 * kVortexParams + 64.0 + 8.0);
    b += (double)kMassBlocks * kMaxTracers * 16.0 + kMaxTracers * 8.0;
    b += 256.0 * 1024 * 1024;                   // allocation granularity of ~120 allocations
    return (size_t)b;
}
