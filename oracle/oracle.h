/* CPU oracle for the SCHISM hydrodynamic step (test infrastructure only).
 *
 * This library restates, in plain C and FP64, the reference algorithm of the hot path so that
 * the CUDA implementation can be checked against it.  It is linked only by the tests, by the
 * smoke check and by the CPU-baseline leg of the benchmark; the product never calls it.
 * Every function names the reference file:line it follows ("mdc" = src/kernels/meshdata.cu,
 * "mdh" = src/kernels/meshdata.h, "grid" = src/grid/read_and_process_grid.cpp,
 * "pcg" = src/solver/pcg_solver.py, "step" = src/python/schism_step.py).
 *
 * Parity pins: the connectivity part is pinned bit-exactly against the reference's own
 * readHGrid compiled from its sources (recipe oracle/build_ref.py).  The step part has no
 * reference golden vectors (the reference ships no tests or fixtures and needs a GPU), so it
 * is pinned by analytic known-answer tests (lake at rest, uniform-flow backtracking, closed-basin
 * mass conservation) in tests/.
 */
#ifndef GS_ORACLE_H
#define GS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- grid (readHGrid) ---- */
/* Inputs: elnode[ne*4] (row e = 4 local nodes, -1 padded), i34[ne], isbnd[np].
 * Outputs (caller-allocated, capacities in comments):
 *   nne_start[np+1], nne[<=4*ne]      node -> elements, CCW order (grid:27-84, 496-574)
 *   nnp_start[np+1], nnp[<=4*ne+np]   node -> nodes, CCW order (grid:87-174)
 *   ic3[ne*4], elside[ne*4]           element-side-element and element-side tables (grid:272-437)
 *   isdel[2*ns], isidenode[2*ns]      side -> elements / nodes (capacity 4*ne sides)
 *   *ns                               number of sides
 * Returns 0 on success, a negative code on a malformed mesh. */
int og_grid_build(int np, int ne, const int32_t* elnode, const int32_t* i34, const int32_t* isbnd,
                  int32_t* nne_start, int32_t* nne, int32_t* nnp_start, int32_t* nnp,
                  int32_t* ic3, int32_t* elside, int32_t* isdel, int32_t* isidenode, int32_t* ns);

/* isbnd from the boundary segment lists (grid:946-1079): open node -> segment index,
 * land-only node -> -2, interior -> -1.  open_nodes/land_nodes are the concatenated
 * segments with starts arrays of length nseg+1. */
void og_grid_isbnd(int np, int nope, const int32_t* open_start, const int32_t* open_nodes,
                   int nland, const int32_t* land_start, const int32_t* land_nodes,
                   int32_t* isbnd);

#ifdef __cplusplus
}
#endif
#endif
