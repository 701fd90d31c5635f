// gm_symbolic_*: host-only introspection of the nested-dissection analysis
// (the counterpart of inspecting UMFPACK's Symbolic object), used by the
// tests to check the extend-add maps without a GPU.
#include <cstring>
#include <exception>
#include <new>

#include "../../include/germaine_gpu.h"
#include "common.hpp"
#include "symbolic.hpp"

struct gm_symbolic {
    gm::Symbolic s;
};

extern "C" int gm_symbolic_create(int nx, int ny, int leaf_max, gm_symbolic **out) {
    if (!out || nx < 1 || ny < 1) return gm::fail(GM_ERROR_INVALID, "gm_symbolic_create: bad argument");
    try {
        auto *h = new gm_symbolic();
        gm::build_symbolic(nx, ny, leaf_max > 0 ? leaf_max : 64, h->s);
        *out = h;
    } catch (const std::bad_alloc &) {
        return gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_symbolic_create: out of host memory");
    } catch (const std::exception &ex) {
        return gm::fail(GM_ERROR_INVALID, ex.what());
    }
    return GM_OK;
}

extern "C" int gm_symbolic_destroy(gm_symbolic *s) {
    delete s;
    return GM_OK;
}

extern "C" int gm_symbolic_sizes(const gm_symbolic *h, int64_t *sz) {
    if (!h || !sz) return gm::fail(GM_ERROR_INVALID, "gm_symbolic_sizes: null argument");
    const gm::Symbolic &s = h->s;
    std::memset(sz, 0, 16 * sizeof(int64_t));
    int mf = 0, mp = 0;
    for (int v = 0; v < s.nnodes; ++v) {
        if (s.nfront[v] > mf) mf = s.nfront[v];
        if (s.npiv[v] > mp) mp = s.npiv[v];
    }
    sz[0] = s.n; sz[1] = s.nnodes; sz[2] = s.nlevels; sz[3] = (int64_t)s.vars.size();
    sz[4] = s.front_total; sz[5] = (int64_t)s.inv.size(); sz[6] = (int64_t)s.ent_pos.size();
    sz[7] = s.rhs_total; sz[8] = s.factor_entries; sz[9] = mf; sz[10] = mp;
    return GM_OK;
}

template <class T>
static void copy_vec(const std::vector<T> &v, void *dst) {
    std::memcpy(dst, v.data(), v.size() * sizeof(T));
}

extern "C" int gm_symbolic_export(const gm_symbolic *h, int what, void *dst) {
    if (!h || !dst) return gm::fail(GM_ERROR_INVALID, "gm_symbolic_export: null argument");
    const gm::Symbolic &s = h->s;
    switch (what) {
        case 0: copy_vec(s.perm, dst); break;
        case 1: copy_vec(s.iperm, dst); break;
        case 2: copy_vec(s.npiv, dst); break;
        case 3: copy_vec(s.nfront, dst); break;
        case 4: copy_vec(s.parent, dst); break;
        case 5: copy_vec(s.height, dst); break;
        case 6: copy_vec(s.child0, dst); break;
        case 7: copy_vec(s.child1, dst); break;
        case 8: copy_vec(s.var_off, dst); break;
        case 9: copy_vec(s.vars, dst); break;
        case 10: copy_vec(s.front_off, dst); break;
        case 11: copy_vec(s.inv_off, dst); break;
        case 12: copy_vec(s.inv, dst); break;
        case 13: copy_vec(s.ent_off, dst); break;
        case 14: copy_vec(s.ent_pos, dst); break;
        case 15: copy_vec(s.ent_id, dst); break;
        case 16: copy_vec(s.rhs_off, dst); break;
        case 17: copy_vec(s.lvl_off, dst); break;
        case 18: copy_vec(s.lvl_nodes, dst); break;
        default: return gm::fail(GM_ERROR_INVALID, "gm_symbolic_export: unknown array");
    }
    return GM_OK;
}

extern "C" double gm_symbolic_flops(const gm_symbolic *h, int which) {
    if (!h) return -1.0;
    return which == 0 ? h->s.factor_flops : h->s.solve_flops_per_rhs;
}
