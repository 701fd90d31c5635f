// Geometric nested dissection + multifrontal symbolic analysis for the
// 9-point stencil (see symbolic.hpp).
#include "symbolic.hpp"

#include <algorithm>
#include <stdexcept>

namespace gm {

namespace {

struct Rect { int x0, x1, y0, y1; };  // half-open, 0-based grid coordinates

struct Builder {
    Symbolic &s;
    std::vector<Rect> region;          // rectangle whose points the node's subtree eliminates
    std::vector<std::vector<int>> piv; // pivots (grid indices) of each node
    int next_pos = 0;

    explicit Builder(Symbolic &sym) : s(sym) {}

    int new_node(const Rect &r, std::vector<int> &&pivots, int c0, int c1) {
        int id = (int)piv.size();
        for (int k : pivots) { s.perm[next_pos] = k; s.iperm[k] = next_pos; ++next_pos; }
        piv.push_back(std::move(pivots));
        region.push_back(r);
        s.child0.push_back(c0); s.child1.push_back(c1);
        int h = 0;
        if (c0 >= 0) h = std::max(h, s.height[c0] + 1);
        if (c1 >= 0) h = std::max(h, s.height[c1] + 1);
        s.height.push_back(h);
        return id;
    }

    int build(const Rect &r) {
        const int w = r.x1 - r.x0, h = r.y1 - r.y0;
        const bool can_cut_x = w >= 3, can_cut_y = h >= 3;
        if (w * h <= s.leaf_max || (!can_cut_x && !can_cut_y)) {
            std::vector<int> p;
            p.reserve(w * h);
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x) p.push_back(y * s.nx + x);
            return new_node(r, std::move(p), -1, -1);
        }
        std::vector<int> sep;
        int c0, c1;
        if ((w >= h && can_cut_x) || !can_cut_y) {
            const int xm = r.x0 + w / 2;
            c0 = build({r.x0, xm, r.y0, r.y1});
            c1 = build({xm + 1, r.x1, r.y0, r.y1});
            for (int y = r.y0; y < r.y1; ++y) sep.push_back(y * s.nx + xm);
        } else {
            const int ym = r.y0 + h / 2;
            c0 = build({r.x0, r.x1, r.y0, ym});
            c1 = build({r.x0, r.x1, ym + 1, r.y1});
            for (int x = r.x0; x < r.x1; ++x) sep.push_back(ym * s.nx + x);
        }
        return new_node(r, std::move(sep), c0, c1);
    }
};

}  // namespace

void build_symbolic(int nx, int ny, int leaf_max, Symbolic &s) {
    if (nx < 1 || ny < 1) throw std::invalid_argument("grid must be at least 1 x 1");
    if ((int64_t)nx * ny > (int64_t)1 << 28) throw std::invalid_argument("grid too large");
    s = Symbolic();
    s.nx = nx; s.ny = ny; s.n = nx * ny; s.leaf_max = std::max(leaf_max, 4);
    s.perm.assign(s.n, -1); s.iperm.assign(s.n, -1);

    Builder b(s);
    b.build({0, nx, 0, ny});
    s.nnodes = (int)b.piv.size();
    if (b.next_pos != s.n) throw std::logic_error("dissection did not cover the grid");

    const int nn = s.nnodes;
    s.parent.assign(nn, -1);
    for (int v = 0; v < nn; ++v) {
        if (s.child0[v] >= 0) s.parent[s.child0[v]] = v;
        if (s.child1[v] >= 0) s.parent[s.child1[v]] = v;
    }

    // front variables: pivots, then the ring of the node's rectangle
    // (points outside it at Chebyshev distance 1), all eliminated later,
    // sorted by elimination position.
    s.npiv.resize(nn); s.nfront.resize(nn);
    s.var_off.assign(nn + 1, 0);
    std::vector<int> ring;
    for (int v = 0; v < nn; ++v) {
        const Rect &r = b.region[v];
        ring.clear();
        for (int y = r.y0 - 1; y <= r.y1; ++y) {
            if (y < 0 || y >= ny) continue;
            for (int x = r.x0 - 1; x <= r.x1; ++x) {
                if (x < 0 || x >= nx) continue;
                if (x >= r.x0 && x < r.x1 && y >= r.y0 && y < r.y1) continue;
                ring.push_back(y * nx + x);
            }
        }
        std::sort(ring.begin(), ring.end(), [&](int a, int c) { return s.iperm[a] < s.iperm[c]; });
        const auto &p = b.piv[v];
        s.npiv[v] = (int)p.size();
        s.nfront[v] = (int)(p.size() + ring.size());
        s.var_off[v + 1] = s.var_off[v] + s.nfront[v];
        s.vars.insert(s.vars.end(), p.begin(), p.end());
        s.vars.insert(s.vars.end(), ring.begin(), ring.end());
    }

    // storage offsets
    s.front_off.assign(nn, 0); s.rhs_off.assign(nn, 0);
    int64_t fo = 0, ro = 0;
    for (int v = 0; v < nn; ++v) {
        s.front_off[v] = fo; fo += (int64_t)s.nfront[v] * s.nfront[v];
        s.rhs_off[v] = ro; ro += s.nfront[v] - s.npiv[v];
    }
    s.front_total = fo; s.rhs_total = ro;

    // extend-add inverse maps: for parent p and child slot t, position i of
    // p's front is fed by the child's contribution-block entry inv[...] (or -1)
    std::vector<int> pos(s.n, -1);
    s.inv_off.assign(nn, 0);
    int64_t io = 0;
    for (int v = 0; v < nn; ++v) { s.inv_off[v] = io; io += 2 * (int64_t)s.nfront[v]; }
    s.inv.assign(io, -1);
    for (int p = 0; p < nn; ++p) {
        const int f = s.nfront[p];
        for (int i = 0; i < f; ++i) pos[s.vars[s.var_off[p] + i]] = i;
        for (int t = 0; t < 2; ++t) {
            const int c = t == 0 ? s.child0[p] : s.child1[p];
            if (c < 0) continue;
            const int sc = s.npiv[c], fc = s.nfront[c];
            for (int a = 0; a < fc - sc; ++a) {
                const int g = s.vars[s.var_off[c] + sc + a];
                const int i = pos[g];
                if (i < 0) throw std::logic_error("child contribution variable missing from parent front");
                s.inv[s.inv_off[p] + (int64_t)t * f + i] = a;
            }
        }
        for (int i = 0; i < f; ++i) pos[s.vars[s.var_off[p] + i]] = -1;
    }

    // owner node of every pivot
    s.owner.assign(s.n, -1);
    std::vector<int> &owner = s.owner;
    for (int v = 0; v < nn; ++v)
        for (int i = 0; i < s.npiv[v]; ++i) owner[s.vars[s.var_off[v] + i]] = v;

    // matrix entries of M = A^T assigned to the front of the earlier-eliminated end
    s.ent_off.assign(nn + 1, 0);
    s.ent_pos.clear(); s.ent_id.clear();
    s.ent_pos.reserve((size_t)9 * s.n); s.ent_id.reserve((size_t)9 * s.n);
    for (int v = 0; v < nn; ++v) {
        const int f = s.nfront[v];
        for (int i = 0; i < f; ++i) pos[s.vars[s.var_off[v] + i]] = i;
        for (int ip = 0; ip < s.npiv[v]; ++ip) {
            const int p = s.vars[s.var_off[v] + ip];
            const int px = p % nx, py = p / nx;
            for (int q = 0; q < 9; ++q) {
                const int cx = px + stencil_di(q), cy = py + stencil_dj(q);
                if (cx < 0 || cx >= nx || cy < 0 || cy >= ny) continue;
                const int c = cy * nx + cx;
                if (s.iperm[c] < s.iperm[p]) continue;   // owned by c's front
                const int jc = pos[c];
                if (jc < 0) throw std::logic_error("stencil neighbour missing from front");
                // M[p][c] = A[c][p]; p = c + off(8-q)
                s.ent_pos.push_back(ip + jc * f);
                s.ent_id.push_back((8 - q) * s.n + c);
                if (c != p) {   // M[c][p] = A[p][c]; c = p + off(q)
                    s.ent_pos.push_back(jc + ip * f);
                    s.ent_id.push_back(q * s.n + p);
                }
            }
        }
        for (int i = 0; i < f; ++i) pos[s.vars[s.var_off[v] + i]] = -1;
        s.ent_off[v + 1] = (int64_t)s.ent_pos.size();
    }

    // level schedule by height
    int hmax = 0;
    for (int v = 0; v < nn; ++v) hmax = std::max(hmax, s.height[v]);
    s.nlevels = hmax + 1;
    s.lvl_off.assign(s.nlevels + 1, 0);
    for (int v = 0; v < nn; ++v) s.lvl_off[s.height[v] + 1]++;
    for (int h = 0; h < s.nlevels; ++h) s.lvl_off[h + 1] += s.lvl_off[h];
    s.lvl_nodes.assign(nn, 0);
    std::vector<int> fill(s.lvl_off.begin(), s.lvl_off.end() - 1);
    for (int v = 0; v < nn; ++v) s.lvl_nodes[fill[s.height[v]]++] = v;
    s.lvl_max_piv.assign(s.nlevels, 0); s.lvl_max_front.assign(s.nlevels, 0);
    for (int v = 0; v < nn; ++v) {
        s.lvl_max_piv[s.height[v]] = std::max(s.lvl_max_piv[s.height[v]], s.npiv[v]);
        s.lvl_max_front[s.height[v]] = std::max(s.lvl_max_front[s.height[v]], s.nfront[v]);
    }

    // exact flop and storage counts
    s.factor_flops = 0; s.solve_flops_per_rhs = 0; s.factor_entries = 0; s.u_entries = 0;
    for (int v = 0; v < nn; ++v) {
        const double f = s.nfront[v], sp = s.npiv[v];
        for (int k = 0; k < s.npiv[v]; ++k) {
            const double m = f - k - 1;
            s.factor_flops += 8.0 * m * m + 6.0 * m;  // rank-1 update + column scaling by 1/pivot
        }
        s.factor_entries += (int64_t)(f * f - (f - sp) * (f - sp));
        s.u_entries += (int64_t)(sp * (sp + 1) / 2 + sp * (f - sp));
        s.solve_flops_per_rhs += 8.0 * (f * f - (f - sp) * (f - sp));
    }
}

}  // namespace gm
