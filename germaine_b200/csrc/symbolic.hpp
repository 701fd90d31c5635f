// Host symbolic phase of the multifrontal LU that replaces UMFPACK's
// umfpack_zi_symbolic (called at src/AC/forward_shot_AC.c:58 and in every
// per-frequency driver).  The reference hands UMFPACK a generic CSC matrix
// and lets it pick a fill-reducing ordering; the matrices here are always
// the 9-point stencil on an NX x NY grid, so the ordering is a geometric
// nested dissection with one-line separators (a line of grid points cuts a
// 9-point stencil graph) and the whole front structure follows in closed
// form from the rectangles of the dissection.
#pragma once
#include <cstdint>
#include <vector>

namespace gm {

// direction q of the 9-point stencil: di = q % 3 - 1, dj = q / 3 - 1
// (NW, N, NE, W, C, E, SW, S, SE -- the reference's triplet order within a
// row, src/AC/init_A_AC_9p_pml.c:68-214).
inline int stencil_di(int q) { return q % 3 - 1; }
inline int stencil_dj(int q) { return q / 3 - 1; }

struct Symbolic {
    int nx = 0, ny = 0, n = 0;
    int leaf_max = 0;          // largest leaf rectangle (grid points)
    int nnodes = 0;
    int nlevels = 0;           // heights 0 .. nlevels-1 (leaves at 0)

    std::vector<int> perm;     // elimination position -> grid index
    std::vector<int> iperm;    // grid index -> elimination position

    // per node (postorder: children before parents)
    std::vector<int> npiv, nfront, parent, height, child0, child1;
    std::vector<int> owner;          // grid index -> node that eliminates it
    std::vector<int64_t> var_off;    // vars[var_off[v] .. + nfront[v]): pivots first, then ring
    std::vector<int> vars;           // grid indices
    std::vector<int64_t> front_off;  // column-major nfront x nfront block per node
    int64_t front_total = 0;         // sum nfront^2 (elements per frequency)
    std::vector<int64_t> inv_off;    // inv[inv_off[v] + t*nfront[v] + i], t = child slot 0/1
    std::vector<int> inv;            // child contribution-block index feeding front position i, or -1
    std::vector<int64_t> rhs_off;    // per-node offset of its update vector (the ring rows, sum nfront - npiv)
    int64_t rhs_total = 0;

    // matrix entries of the REF operator M = A^T scattered into fronts:
    // for node v, ent[ent_off[v] .. ent_off[v+1]) = (pos = i + j*nfront, id)
    // with id = q*n + c addressing the assembled stencil value A[c][c+off(q)]
    // (stored direction-major), so that M[c+off(q)][c] = A[c][c+off(q)].
    std::vector<int64_t> ent_off;
    std::vector<int> ent_pos, ent_id;

    // level schedule: nodes of height h are lvl_nodes[lvl_off[h] .. lvl_off[h+1])
    std::vector<int> lvl_off, lvl_nodes;
    std::vector<int> lvl_max_piv, lvl_max_front;

    // exact operation counts (real flops, a complex FMA = 8)
    double factor_flops = 0;       // partial LU of every front
    double solve_flops_per_rhs = 0;// forward + backward substitution, one RHS
    int64_t factor_entries = 0;    // stored L+U entries (sum f^2 - (f-s)^2)
    int64_t u_entries = 0;         // stored U entries (pivot rows from the diagonal on: s(s+1)/2 + s(f-s))
};

// Builds the nested-dissection symbolic structure of an nx x ny 9-point grid.
// leaf_max: rectangles with at most this many points are not cut further.
void build_symbolic(int nx, int ny, int leaf_max, Symbolic &s);

}  // namespace gm
