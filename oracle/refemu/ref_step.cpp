/* Host driver of the reference's own step kernels (test infrastructure only).
 *
 * This translation unit includes the reference's kernel source, src/kernels/meshdata.cu, with
 * the host stand-in for the CUDA vocabulary (oracle/refemu/cuda_runtime.h) and a constants.h
 * generated for one case from the reference's own template (oracle/refemu/build.py).  The
 * kernels run unchanged on the CPU, one global thread index after the other, so this library
 * computes exactly what the reference's kernels compute, with atomics applied in index order
 * and no FMA contraction.  It is the pinned reference the CPU restatement (oracle/step.c) and
 * the CUDA product are compared with; nothing in the product links it.
 *
 * The driver mirrors the host code around the kernels:
 *   - mesh construction: src/python/main.py:505-778 (struct memory, createMesh, populate phases);
 *   - cold start: src/python/schism_init.py:78-103 (ul0* levels, densities);
 *   - one step: src/python/schism_step.py:95-334, kernel by kernel (rd_kernel);
 *   - the elevation solve: PCGSolverMultiGPU.solve, src/solver/pcg_solver.py:1075-1124 (gather
 *     b from qel, Jacobi-preconditioned CG with the parabolic initial guess and the compiled
 *     loop's scalar rules, pcg_solver.py:208-276, scatter x to mX, roll the history);
 *   - the transport sub-step minimum: minTransportDt, meshdata.cu:6842-6863, restated as a
 *     sequential minimum (the kernel itself needs a whole thread block).
 */
#include "meshdata.cu"


thread_local gs_dim3 threadIdx, blockIdx, blockDim, gridDim;

namespace {

struct RefInput {
    int np, ne, ns, nope, nland, mnond, mnlnd, nbfr, nbnd_nodes, nbnd_sides;
    const int* i34;          /* [ne] */
    const int* elnode;       /* (4, ne) F-order: [e*4 + j] */
    const int* elside;       /* (4, ne) F-order */
    const double* coords;    /* (3, np) F-order: [i*3 + c] */
    const int* isdel;        /* (2, ns) F-order: [s*2 + l] */
    const int* isidenode;    /* (2, ns) F-order */
    const int* isbnd;        /* [np] */
    const int* nond;         /* [nope] */
    const int* nlnd;         /* [nland] */
    const int* iond;         /* (nope, mnond) F-order: [seg + i*nope] */
    const int* ilnd;         /* (nland, mnlnd) F-order */
    const int* nnp_start; const int* nnp;   /* node -> nodes CSR */
    const int* nne_start; const int* nne;   /* node -> elements CSR */
    const double* drag;      /* [np] */
    const double* temp;      /* [np] */
    const double* salt;      /* [np] */
    int* kb;                 /* readVGrid kb (ivcor = 1 only) */
    double* sigma_lcl;
    double h_c, h_s, theta_b, theta_f;
    double* sigma; double* ztot; double* cs; double* dcs;
    int n_sigma, n_ztot;
    double* amig; double* face; double* ff;                /* [nbfr] */
    double* emo; double* efa; double* umo; double* ufa; double* vmo; double* vfa;  /* (nope, mnond, nbfr) F */
    int* ifltype; int* iettype; double* qthcon; double* eth; /* [nope] */
};

struct RefModel {
    int np = 0, ne = 0, ns = 0, nnz = 0;
    std::vector<int> i34, elnode, elside, isdel, isidenode, isbnd, nond, nlnd, iond, ilnd;
    std::vector<int> nnp_start, nnp, nne_start, nne, gidx_n, gidx_e, gidx_s, lidx_n, lidx_e, lidx_s;
    std::vector<int> part_n, part_e, part_s, lnn_start, lne_start, shared_nb, shared_sb;
    std::vector<int> kb, ifltype, iettype, csr_indptr, csr_indices;
    std::vector<double> coords, coords_ll, wind_rot, drag, temp, salt, sigma_lcl;
    std::vector<double> sigma, ztot, cs, dcs, amig, face, ff, emo, efa, umo, ufa, vmo, vfa, qthcon, eth;
    std::vector<double> csr_data, zeros1;
    /* struct memory (zero-filled like the reference's cp.zeros buffers) */
    Node* nodes = nullptr; Element* elems = nullptr; Side* sides = nullptr;
    NodeBoundary* nbmem = nullptr; SideBoundary* sbmem = nullptr; BoundarySegment* segmem = nullptr;
    NodeBoundary* land_nb = nullptr; BoundarySegment* land_seg = nullptr;
    Node** nn_mem = nullptr; Element** ne_mem = nullptr; int16_t* perm_mem = nullptr; double* coeff_mem = nullptr;
    Node* node_ptrs[1]; Element* elem_ptrs[1]; Side* side_ptrs[1];
    double debug_plot[8]; int debug_plot_idx[8];
    /* solver state (pcg_solver.py): parabolic history and work vectors */
    std::vector<double> x0, x1, x2, xs, b, r, z, p, q, invD;
    double rtol = 1e-12; int maxiter = 1000, check_every = 10, last_iters = 0, last_substeps = 0;
};

RefModel* g_model = nullptr;

/* Thread order of the kernels whose sums are atomic updates: 0 = index order, 1 = reversed.
 * On a GPU that order is whatever the scheduler gives; both are orders a GPU may produce, so
 * two runs that differ only in it bound how far the reference departs from itself. */
int g_atomic_order = 0;

/* Summation order of the solver's dot products: 0 = sequential, 1 = warp-shaped (sequential
 * sums of 32 entries, then the partial sums added pairwise), the shape of a GPU library
 * reduction.  The reference's dot products run in cuBLAS/CuPy, whose order is not specified. */
int g_dot_order = 0;

double dot_sum(const double* a, const double* b, int n) {
    if (g_dot_order == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    }
    std::vector<double> part;
    for (int i0 = 0; i0 < n; i0 += 32) {
        double s = 0.0;
        const int i1 = i0 + 32 < n ? i0 + 32 : n;
        for (int i = i0; i < i1; ++i) s += a[i] * b[i];
        part.push_back(s);
    }
    while (part.size() > 1) {
        std::vector<double> nx;
        for (size_t j = 0; j < part.size(); j += 2) nx.push_back(j + 1 < part.size() ? part[j] + part[j + 1] : part[j]);
        part.swap(nx);
    }
    return part.empty() ? 0.0 : part[0];
}

template <class F> void launch(int n, F&& f, bool reverse = false) {
    blockDim.x = 1; blockDim.y = blockDim.z = 1; threadIdx.x = threadIdx.y = threadIdx.z = 0;
    gridDim.x = n > 0 ? n : 1; gridDim.y = gridDim.z = 1;
    if (reverse) { for (int i = n - 1; i >= 0; --i) { blockIdx.x = i; f(); } }
    else { for (int i = 0; i < n; ++i) { blockIdx.x = i; f(); } }
}

template <class T> T* zalloc(size_t n) {
    void* p = calloc(n ? n : 1, sizeof(T));
    return static_cast<T*>(p);
}

template <class T> std::vector<T> vec(const T* p, size_t n) { return p ? std::vector<T>(p, p + n) : std::vector<T>(n ? n : 1, T()); }

void spmv(const RefModel& m, const double* v, double* out) {
    for (int i = 0; i < m.np; ++i) {
        double s = 0.0;
        for (int a = m.csr_indptr[i]; a < m.csr_indptr[i + 1]; ++a) s += m.csr_data[a] * v[m.csr_indices[a]];
        out[i] = s;
    }
}

}  // namespace

extern "C" {

int rd_sizes(int* out6) {
    /* getStructSizes, meshdata.cu:7461-7471 */
    out6[0] = (int)sizeof(Node); out6[1] = (int)sizeof(Element); out6[2] = (int)sizeof(Side);
    out6[3] = (int)sizeof(NodeBoundary); out6[4] = (int)sizeof(SideBoundary); out6[5] = (int)sizeof(BoundarySegment);
    return nvrt * 1000 + ntracers;
}

int rd_create(const RefInput* in) {
    /* main.py:505-778 for one partition (global index = local index) */
    if (g_model != nullptr || mesh != nullptr) return -1;
    RefModel& m = *(g_model = new RefModel());
    const int np_ = in->np, ne_ = in->ne, ns_ = in->ns;
    m.np = np_; m.ne = ne_; m.ns = ns_;
    m.i34 = vec(in->i34, ne_); m.elnode = vec(in->elnode, 4 * (size_t)ne_); m.elside = vec(in->elside, 4 * (size_t)ne_);
    m.coords = vec(in->coords, 3 * (size_t)np_); m.isdel = vec(in->isdel, 2 * (size_t)ns_);
    m.isidenode = vec(in->isidenode, 2 * (size_t)ns_); m.isbnd = vec(in->isbnd, np_);
    m.nond = vec(in->nond, in->nope); m.nlnd = vec(in->nlnd, in->nland);
    m.iond = vec(in->iond, (size_t)in->nope * in->mnond); m.ilnd = vec(in->ilnd, (size_t)in->nland * in->mnlnd);
    m.nnp_start = vec(in->nnp_start, np_ + 1); m.nnp = vec(in->nnp, in->nnp_start[np_]);
    m.nne_start = vec(in->nne_start, np_ + 1); m.nne = vec(in->nne, in->nne_start[np_]);
    m.drag = vec(in->drag, np_); m.temp = vec(in->temp, np_); m.salt = vec(in->salt, np_);
    m.kb = vec(in->kb, np_); m.sigma_lcl = vec(in->sigma_lcl, (size_t)np_ * nvrt);
    m.sigma = vec(in->sigma, in->n_sigma); m.ztot = vec(in->ztot, in->n_ztot); m.cs = vec(in->cs, in->n_sigma);
    m.dcs = vec(in->dcs, in->n_sigma);
    const size_t nb = (size_t)(in->nbfr > 0 ? in->nbfr : 1);
    m.amig = vec(in->amig, nb); m.face = vec(in->face, nb); m.ff = vec(in->ff, nb);
    const size_t ne3 = (size_t)in->nope * in->mnond * nb;
    m.emo = vec(in->emo, ne3); m.efa = vec(in->efa, ne3); m.umo = vec(in->umo, ne3); m.ufa = vec(in->ufa, ne3);
    m.vmo = vec(in->vmo, ne3); m.vfa = vec(in->vfa, ne3);
    m.ifltype = vec(in->ifltype, in->nope); m.iettype = vec(in->iettype, in->nope);
    m.qthcon = vec(in->qthcon, in->nope); m.eth = vec(in->eth, in->nope);
    m.coords_ll.assign(2, 0.0); m.wind_rot.assign(np_, 0.0); m.zeros1.assign(np_ + 1, 0.0);

    m.gidx_n.resize(np_); m.gidx_e.resize(ne_); m.gidx_s.resize(ns_);
    for (int i = 0; i < np_; ++i) m.gidx_n[i] = i;
    for (int i = 0; i < ne_; ++i) m.gidx_e[i] = i;
    for (int i = 0; i < ns_; ++i) m.gidx_s[i] = i;
    m.lidx_n = m.gidx_n; m.lidx_e = m.gidx_e; m.lidx_s = m.gidx_s;
    m.part_n.assign(np_, 0); m.part_e.assign(ne_, 0); m.part_s.assign(ns_, 0);
    m.lnn_start = m.nnp_start; m.lne_start = m.nne_start;
    m.shared_nb.assign(1, -1); m.shared_sb.assign(1, -1);

    const int nn_tot = m.nnp_start[np_], ne_tot = m.nne_start[np_];
    m.nnz = nn_tot + np_;
    m.csr_data.assign(m.nnz, 0.0); m.csr_indices.assign(m.nnz, 0); m.csr_indptr.assign(np_ + 1, 0);
    m.csr_indptr[np_] = m.nnz;   /* PCGSolverMultiGPU.__init__, pcg_solver.py:622-623 */

    /* struct memory; boundary arrays sized generously (the host has no silent overrun) */
    m.nodes = zalloc<Node>(np_); m.elems = zalloc<Element>(ne_); m.sides = zalloc<Side>(ns_);
    m.nbmem = zalloc<NodeBoundary>((size_t)np_ + 1); m.sbmem = zalloc<SideBoundary>((size_t)ns_ + 1);
    m.segmem = zalloc<BoundarySegment>((size_t)in->nope + in->nland + 1);
    m.land_nb = zalloc<NodeBoundary>(1); m.land_seg = zalloc<BoundarySegment>(1);
    m.nn_mem = zalloc<Node*>(nn_tot); m.ne_mem = zalloc<Element*>(ne_tot);
    m.perm_mem = zalloc<int16_t>(nn_tot); m.coeff_mem = zalloc<double>(nn_tot);
    m.node_ptrs[0] = m.nodes; m.elem_ptrs[0] = m.elems; m.side_ptrs[0] = m.sides;

    initTidalHarmonicConstituents(m.amig.data(), m.face.data(), m.ff.data());
    launch(1, [&] {
        createMesh(0, np_, ne_, ns_, in->nland, np_, ne_, ns_, np_, ne_, ns_, m.land_nb, m.land_seg,
                   m.node_ptrs, m.elem_ptrs, m.side_ptrs, m.nodes, m.elems, m.sides, m.nn_mem, m.ne_mem,
                   m.perm_mem, m.coeff_mem, m.nbmem, m.sbmem, m.segmem, m.kb.data(), in->h_c, in->h_s,
                   in->theta_b, in->theta_f, m.sigma.data(), m.ztot.data(), m.cs.data(), m.dcs.data(),
                   m.debug_plot, m.debug_plot_idx);
    });
    double* dnull = m.zeros1.data();
    launch(np_, [&] {
        populateNodes(m.i34.data(), m.isbnd.data(), m.shared_nb.data(), m.coords.data(), m.coords_ll.data(), false,
                      m.wind_rot.data(), m.nnp_start.data(), m.nnp.data(), m.nne_start.data(), m.nne.data(),
                      m.perm_mem, m.csr_data.data(), m.lnn_start.data(), m.lne_start.data(), m.gidx_n.data(),
                      m.gidx_e.data(), m.gidx_s.data(), m.lidx_n.data(), m.lidx_e.data(), m.lidx_s.data(),
                      m.part_n.data(), m.part_e.data(), m.part_s.data(), m.drag.data(), dnull, dnull, dnull, dnull,
                      m.temp.data(), m.salt.data(), m.kb.data(), m.sigma_lcl.data());
    });
    launch(np_, [&] { populateNodes2(m.lnn_start.data(), m.csr_indices.data(), m.csr_indptr.data()); });
    launch(ns_, [&] {
        populateSides(m.i34.data(), m.shared_sb.data(), m.coords.data(), m.coords_ll.data(), false, m.wind_rot.data(),
                      m.isdel.data(), m.isidenode.data(), m.isbnd.data(), m.nond.data(), m.nlnd.data(), m.iond.data(),
                      m.ilnd.data(), m.nnp_start.data(), m.nnp.data(), m.nne_start.data(), m.nne.data(),
                      m.gidx_n.data(), m.gidx_e.data(), m.gidx_s.data(), m.lidx_n.data(), m.lidx_e.data(),
                      m.lidx_s.data(), m.part_n.data(), m.part_e.data(), m.part_s.data(), m.drag.data(), dnull);
    });
    launch(ne_, [&] {
        populateElements(m.i34.data(), m.elnode.data(), m.elside.data(), m.coords.data(), m.coords_ll.data(), false,
                         m.wind_rot.data(), m.isdel.data(), m.isidenode.data(), m.isbnd.data(), m.nond.data(),
                         m.nlnd.data(), m.iond.data(), m.ilnd.data(), m.nnp_start.data(), m.nnp.data(),
                         m.nne_start.data(), m.nne.data(), m.gidx_n.data(), m.gidx_e.data(), m.gidx_s.data(),
                         m.lidx_n.data(), m.lidx_e.data(), m.lidx_s.data(), m.part_n.data(), m.part_e.data(),
                         m.part_s.data(), m.drag.data(), dnull);
    });
    launch(1, [&] {
        populateMesh(m.i34.data(), m.elnode.data(), m.elside.data(), m.coords.data(), m.coords_ll.data(), false,
                     m.wind_rot.data(), m.shared_nb.data(), m.shared_sb.data(), m.isdel.data(), m.isidenode.data(),
                     m.isbnd.data(), m.nond.data(), m.nlnd.data(), m.iond.data(), m.ilnd.data(), m.nnp_start.data(),
                     m.nnp.data(), m.nne_start.data(), m.nne.data(), m.gidx_n.data(), m.gidx_e.data(),
                     m.gidx_s.data(), m.lidx_n.data(), m.lidx_e.data(), m.lidx_s.data(), m.part_n.data(),
                     m.part_e.data(), m.part_s.data(), m.drag.data(), dnull, m.emo.data(), m.efa.data(),
                     m.umo.data(), m.ufa.data(), m.vmo.data(), m.vfa.data());
    });
    launch(mesh->nbp, [&] {
        populateBoundaryNodes(m.nond.data(), m.iond.data(), m.emo.data(), m.efa.data(), m.umo.data(), m.ufa.data(),
                              m.vmo.data(), m.vfa.data(), m.ifltype.data(), m.iettype.data(), m.qthcon.data(),
                              m.eth.data());
    });
    launch(mesh->nbs, [&] {
        populateBoundarySides(m.nond.data(), m.iond.data(), m.emo.data(), m.efa.data(), m.umo.data(), m.ufa.data(),
                              m.vmo.data(), m.vfa.data(), m.ifltype.data(), m.iettype.data(), m.qthcon.data());
    });
    m.x0.assign(np_, 0.0); m.x1.assign(np_, 0.0); m.x2.assign(np_, 0.0); m.xs.assign(np_, 0.0);
    m.b.assign(np_, 0.0); m.r.assign(np_, 0.0); m.z.assign(np_, 0.0); m.p.assign(np_, 0.0);
    m.q.assign(np_, 0.0); m.invD.assign(np_, 0.0);
    return 0;
}

void rd_counts(int* out) {
    out[0] = mesh->np; out[1] = mesh->ne; out[2] = mesh->ns; out[3] = mesh->nbp; out[4] = mesh->nbs;
    out[5] = g_model->nnz; out[6] = g_model->last_iters; out[7] = g_model->last_substeps;
}

void rd_set_atomic_order(int order) { g_atomic_order = order; }
void rd_set_dot_order(int order) { g_dot_order = order; }

void rd_set_solver(double rtol, int maxiter, int check_every) {
    g_model->rtol = rtol; g_model->maxiter = maxiter; g_model->check_every = check_every;
}

/* One reference kernel over its launch domain (cuda_functions.py:140-257 kernel types). */
int rd_kernel(const char* name, double t, int i1, int i2) {
    RefModel& m = *g_model;
    const int NP = mesh->np, NE = mesh->ne, NS = mesh->ns, NBP = mesh->nbp, NBS = mesh->nbs;
    const std::string k(name);
    const bool atomic_kernel = (k == "computeNodalVerticalVelocities1" || k == "computeNodalHorizontalVelocities1" ||
                                k == "setVelocityOpenBndNodes" || k == "computeBoundaryAreas");
    const bool rev = atomic_kernel && g_atomic_order == 1;
#define K(NAME, N, CALL) if (k == #NAME) { launch(N, [&] { CALL; }, rev); return 0; }
    K(scaleGravity, NP, scaleGravity(t))
    K(computeBedDeformation, 1, computeBedDeformation())
    K(computeTidalPotential, NP, computeTidalPotential(t, nullptr, nullptr, nullptr, nullptr, nullptr))
    K(getBoundaryConditions, NBP, getBoundaryConditions(t))
    K(resetBoundaryAreas, NBS, resetBoundaryAreas())
    K(computeBoundaryAreas, NBS, computeBoundaryAreas())
    K(computeFlowBcVelocities, NBS, computeFlowBcVelocities(t))
    K(computeBottomDragVegetation, NP, computeBottomDragVegetation())
    K(computeTurbulence, NP, computeTurbulence())
    K(computeHorizontalViscosity, NS, computeHorizontalViscosity())
    K(backtrackAllNodes, NS, backtrackAllNodes())
    K(computeElevationBoundaryConditions, NBP, computeElevationBoundaryConditions(t))
    K(computeVerticallyIntegratedVelocity, NS, computeVerticallyIntegratedVelocity())
    K(computeVegetationAndDragParameters, NS, computeVegetationAndDragParameters())
    K(computeDensityGradient, NE, computeDensityGradient())
    K(computeBaroclinicTerm, NS, computeBaroclinicTerm())
    K(computeElemAverageGhat, NE, computeElemAverageGhat())
    K(setupCoefficientMatrixAndRHS, NP, setupCoefficientMatrixAndRHS(t))
    K(rollUpElevation, NP, rollUpElevation())
    K(setEssentialBC, NP, setEssentialBC())
    K(updateElevation, NP, updateElevation())
    K(computeHorGradientAtSide, NS, computeHorGradientAtSide())
    K(solveMomentumEquations, NS, solveMomentumEquations(t))
    K(applyMomentumBC, NBS, applyMomentumBC())
    K(shapiroFilter1, NS, shapiroFilter1())
    K(shapiroFilter2, NS, shapiroFilter2())
    K(computeVerticalVelocity, NE, computeVerticalVelocity())
    K(computeHorizAdvecFluxes, NS, computeHorizAdvecFluxes())
    K(horizontalAdvectionPrepare, NE, horizontalAdvectionPrepare())
    K(horizontalAdvectionUpdate, NE, horizontalAdvectionUpdate(t))
    K(verticalAdvectionUpdate, NE, verticalAdvectionUpdate(t))
    K(nodalTracerUpdate, NP, nodalTracerUpdate())
    K(ul0UpdateZCoords, NP, ul0UpdateZCoords())
    K(ul0ComputeDryElements, NE, ul0ComputeDryElements())
    K(ul0ComputeDryNodes, NP, ul0ComputeDryNodes())
    K(ul0UpdateRewettedNodes, NP, ul0UpdateRewettedNodes(i1, i2))
    K(ul0UpdateSides, NS, ul0UpdateSides(i1, i2))
    K(ul0UpdateSides2, NS, ul0UpdateSides2())
    K(computeNodeDensity, NP, computeNodeDensity())
    K(computeElemDensity, NE, computeElemDensity())
    K(zeroNodalVelocities, NP, zeroNodalVelocities())
    K(computeNodalVerticalVelocities1, NE, computeNodalVerticalVelocities1())
    K(computeNodalVerticalVelocities2, NP, computeNodalVerticalVelocities2())
    K(computeNodalHorizontalVelocities1, NE, computeNodalHorizontalVelocities1())
    K(computeNodalHorizontalVelocities2, NP, computeNodalHorizontalVelocities2())
    K(resetVelocityOpenBndNodes, NBP, resetVelocityOpenBndNodes())
    K(setVelocityOpenBndNodes, NBS, setVelocityOpenBndNodes())
#undef K
    return -1;
}

void rd_time_ramps(double time, double dramp) {
    /* computeTimeRamps (meshdata.h:2036-2076) with nws = 0, no sources: only dramp matters */
    launch(1, [&] { computeTimeRamps(time, 0, false, 0.0, 0.0, 0.0, 0.0, dramp); });
}

double rd_min_transport_dt(void) {
    /* minTransportDt, meshdata.cu:6842-6863: min over wet elements of transport.maxDt, the
     * result buffer starting at 1e34 (schism_step.py:70-72) */
    double v = 1e34;
    for (int e = 0; e < mesh->ne; ++e) {
        const Element& el = mesh->localElemData[e];
        const double d = el.isDry ? huge_double : el.transport.maxDt;
        v = fmin(v, d);
    }
    return v;
}

int rd_transport(double dt) {
    /* computeTransport, schism_step.py:78-93 */
    rd_kernel("computeHorizAdvecFluxes", 0, 0, 0);
    double remaining = dt;
    int n = 0;
    while (remaining > 0.0 && n < 100000) {
        rd_kernel("horizontalAdvectionPrepare", 0, 0, 0);
        const double dtb = fmin(remaining, rd_min_transport_dt());
        rd_kernel("horizontalAdvectionUpdate", dtb, 0, 0);
        remaining -= dtb;
        ++n;
    }
    rd_kernel("verticalAdvectionUpdate", dt, 0, 0);
    rd_kernel("nodalTracerUpdate", 0, 0, 0);
    g_model->last_substeps = n;
    return n;
}

int rd_solve(void) {
    /* PCGSolverMultiGPU.solve, pcg_solver.py:1075-1124 */
    RefModel& m = *g_model;
    const int n = m.np;
    launch(n, [&] { gatherBFromMesh(m.b.data()); });
    const double bb = dot_sum(m.b.data(), m.b.data(), n);
    for (int i = 0; i < n; ++i) {
        double d = 0.0;
        for (int a = m.csr_indptr[i]; a < m.csr_indptr[i + 1]; ++a)
            if (m.csr_indices[a] == i) d = m.csr_data[a];
        m.invD[i] = 1.0 / d;
    }
    const double atol = m.rtol * sqrt(bb);
    int iters = 0;
    if (atol == 0.0) {
        for (int i = 0; i < n; ++i) m.xs[i] = 0.0;
    } else {
        for (int i = 0; i < n; ++i) { m.xs[i] = 3.0 * m.x0[i] - 3.0 * m.x1[i] + m.x2[i]; m.p[i] = 0.0; }
        spmv(m, m.xs.data(), m.q.data());
        for (int i = 0; i < n; ++i) m.r[i] = m.b[i] - m.q[i];
        const double atol2 = atol * atol;
        for (int i = 0; i < n; ++i) m.z[i] = m.invD[i] * m.r[i];
        double rr = dot_sum(m.r.data(), m.r.data(), n), rz = dot_sum(m.r.data(), m.z.data(), n);
        double rho = rz, rz_new = rz;
        iters = m.maxiter;
        for (int it = 0; it < m.maxiter; ++it) {
            const double beta = (it == 0 || rho == 0.0) ? 0.0 : rz_new / rho;
            if (it > 0) rho = rz_new;
            for (int i = 0; i < n; ++i) m.p[i] = m.z[i] + beta * m.p[i];
            spmv(m, m.p.data(), m.q.data());
            const double pq = dot_sum(m.p.data(), m.q.data(), n);
            const double alpha = (pq != 0.0) ? rho / pq : 0.0;
            for (int i = 0; i < n; ++i) {
                m.xs[i] += alpha * m.p[i];
                m.r[i] = m.r[i] - alpha * m.q[i];
                m.z[i] = m.invD[i] * m.r[i];
            }
            rr = dot_sum(m.r.data(), m.r.data(), n);
            rz = dot_sum(m.r.data(), m.z.data(), n);
            rz_new = rz;
            if ((it + 1) % m.check_every == 0 || it == m.maxiter - 1) {
                if (rr <= atol2) { iters = it + 1; break; }
            }
        }
    }
    launch(n, [&] { scatterXToMesh(m.xs.data()); });
    for (int i = 0; i < n; ++i) { m.x2[i] = m.x1[i]; m.x1[i] = m.x0[i]; m.x0[i] = m.xs[i]; }
    m.last_iters = iters;
    return iters;
}

/* Field exchange in the oracle's layout (level-major [nvrt][n], vectors [.][n][2], tracers
 * [ntr][nvrt][n]); field codes are the oracle's (oracle/step.h, OGF_*).  to_ext = 1 reads the
 * reference's structs, 0 writes them.  Returns -1 for a field the reference does not keep. */
int rd_xfer(int f, void* ext, int to_ext) {
    RefModel& m = *g_model;
    const int NP = mesh->np, NE = mesh->ne, NS = mesh->ns;
    double* d = static_cast<double*>(ext);
    int32_t* q = static_cast<int32_t*>(ext);
#define SC(N, EXPR) for (int i = 0; i < (N); ++i) { if (to_ext) d[i] = (EXPR); else (EXPR) = d[i]; } return 0;
#define V2(N, EXPR) for (int i = 0; i < (N); ++i) { if (to_ext) { d[2*i] = (EXPR).x; d[2*i+1] = (EXPR).y; } \
                                                   else { (EXPR).x = d[2*i]; (EXPR).y = d[2*i+1]; } } return 0;
#define LV(N, EXPR) for (int k = 0; k < nvrt; ++k) for (int i = 0; i < (N); ++i) { \
        double& v_ = (EXPR); if (to_ext) d[(size_t)k*(N)+i] = v_; else v_ = d[(size_t)k*(N)+i]; } return 0;
#define LV2(N, EXPR) for (int k = 0; k < nvrt; ++k) for (int i = 0; i < (N); ++i) { \
        double2& v_ = (EXPR); size_t o_ = ((size_t)k*(N)+i)*2; \
        if (to_ext) { d[o_] = v_.x; d[o_+1] = v_.y; } else { v_.x = d[o_]; v_.y = d[o_+1]; } } return 0;
#define TR(N, EXPR) for (int t = 0; t < ntracers; ++t) for (int k = 0; k < nvrt; ++k) for (int i = 0; i < (N); ++i) { \
        double& v_ = (EXPR); size_t o_ = ((size_t)t*nvrt + k)*(N) + i; if (to_ext) d[o_] = v_; else v_ = d[o_]; } return 0;
#define IS(N, EXPR, T) for (int i = 0; i < (N); ++i) { if (to_ext) q[i] = (int32_t)(EXPR); else (EXPR) = (T)q[i]; } return 0;
    Node* nd = mesh->localNodeData; Side* sd = mesh->localSideData; Element* el = mesh->localElemData;
    switch (f) {
    case 0: SC(NP, nd[i].eta1)
    case 1: SC(NP, nd[i].eta2)
    case 2: LV(NP, nd[i].z[k])
    case 3: LV2(NP, nd[i].u2[k])
    case 4: LV(NP, nd[i].w2[k])
    case 5: TR(NP, nd[i].tracers[k].tracer[t])
    case 6: IS(NP, nd[i].kb, int16_t)
    case 7: IS(NP, nd[i].isDry, bool)
    case 8: SC(NP, nd[i].qel)
    case 9: V2(NP, nd[i].tau)
    case 10: LV2(NS, sd[i].u2[k])
    case 11: LV2(NS, sd[i].btu[k])
    case 12: LV(NS, sd[i].zc[k])
    case 13: IS(NS, sd[i].kb, int16_t)
    case 14: IS(NS, sd[i].isDry, bool)
    case 15: V2(NS, sd[i].U)
    case 16: SC(NS, sd[i].hhat)
    case 17: SC(NS, sd[i].chi)
    case 18: LV(NS, sd[i].transport.Qh[k])
    case 20: V2(NS, sd[i].gradEta1)
    case 21: V2(NS, sd[i].gradEta2)
    case 30: LV(NE, el[i].z[k])
    case 31: LV(NE, el[i].w[k])
    case 32: LV(NE, el[i].transport.Qv[k])
    case 33: TR(NE, el[i].tracers[k].tracer[t])
    case 34: IS(NE, el[i].kb, int16_t)
    case 35: IS(NE, el[i].isDry, bool)
    case 36: V2(NE, el[i].ghat1)
    case 40: SC(m.nnz, m.csr_data[i])
    case 41: IS(NP + 1, m.csr_indptr[i], int)
    case 42: IS(m.nnz, m.csr_indices[i], int)
    case 43: SC(NP, m.x0[i])
    case 44:
        for (int i = 0; i < NP; ++i) {
            NodeBoundary* b_ = nd[i].nodeBnd;
            if (to_ext) d[i] = b_ ? b_->elbc : 0.0; else if (b_) b_->elbc = d[i];
        }
        return 0;
    case 45: SC(NP, m.x1[i])
    case 46: SC(NP, m.x2[i])
    case 47: LV(NP, nd[i].rho[k])
    case 48: LV(NE, el[i].rho[k])
    default: return -1;
    }
#undef SC
#undef V2
#undef LV
#undef LV2
#undef TR
#undef IS
}

}  // extern "C"
