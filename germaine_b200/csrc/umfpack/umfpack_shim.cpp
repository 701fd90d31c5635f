// libgermaine_umfpack.so: the six UMFPACK calls of GERMAINE's drivers
// (include/germaine_umfpack.h) served by the B200 engine of
// libgermaine_gpu.so.  Host code only: the pattern analysis maps the
// compressed columns onto the 9-point stencil of the detected grid, the
// values go to gm_factor_values, the solves to gm_solve.
//
// Reference call sites: src/AC/forward_shot_AC.c:41,58,61,62,88,120 (and the
// same sequence in grad_obj_AC.c, obj_AC.c, hessian_AC.c, hessian_shin_AC.c
// and the SH/TE drivers).
#include "germaine_umfpack.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "germaine_gpu.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int info_status(double *Info, int st) {
    if (Info) Info[UMFPACK_STATUS] = (double)st;
    return st;
}

constexpr unsigned kSymMagic = 0x53594d47u;   // "GMYS"
constexpr unsigned kNumMagic = 0x4e554d47u;   // "GMUN"

struct Symbolic {
    unsigned magic = kSymMagic;
    int n = 0, nx = 0, ny = 0, nnz = 0;
};

struct Numeric {
    unsigned magic = kNumMagic;
    int n = 0, nx = 0, ny = 0;
    gm_engine *e = nullptr;
};

// Engines are kept per grid between numeric objects: the symbolic analysis
// and the device workspaces are reused by the next frequency of a driver.
std::mutex g_pool_mu;
std::map<std::pair<int, int>, std::vector<gm_engine *>> g_pool;
constexpr size_t kPoolKeep = 2;

int env_device() {
    const char *s = std::getenv("GM_UMFPACK_DEVICE");
    return s ? std::atoi(s) : 0;
}

int env_precision() {
    const char *s = std::getenv("GM_UMFPACK_PRECISION");
    return (s && (std::strcmp(s, "c64") == 0 || std::strcmp(s, "C64") == 0)) ? GM_PREC_C64_IR : GM_PREC_FP64;
}

gm_engine *take_engine(int nx, int ny, int *rc) {
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto &v = g_pool[{nx, ny}];
        if (!v.empty()) {
            gm_engine *e = v.back();
            v.pop_back();
            *rc = UMFPACK_OK;
            return e;
        }
    }
    gm_config c{};
    c.nx = nx;
    c.ny = ny;
    c.dh = 1.f;            // geometry-free: the operator arrives by value
    c.npml = 0;
    c.free_surf = 1;
    c.physics = GM_PHYS_AC;
    c.precision = env_precision();
    c.op_mode = GM_OP_REF; // entry [q][c] of gm_factor_values = column c of the matrix
    gm_engine *e = nullptr;
    const int st = gm_engine_create(env_device(), &c, &e);
    if (st != GM_OK) {
        *rc = st == GM_ERROR_OUT_OF_MEMORY ? UMFPACK_ERROR_out_of_memory : UMFPACK_ERROR_internal_error;
        fail(*rc, "engine creation failed: %s", gm_last_error());
        return nullptr;
    }
    *rc = UMFPACK_OK;
    return e;
}

void give_engine(int nx, int ny, gm_engine *e) {
    if (!e) return;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto &v = g_pool[{nx, ny}];
        if (v.size() < kPoolKeep) {
            v.push_back(e);
            return;
        }
    }
    gm_engine_destroy(e);
}

// Direction q of row r relative to column c on an nx-wide grid, or -1 when
// r is not one of c's 9-point neighbours.
inline int stencil_dir(int r, int c, int nx) {
    const int ci = c % nx, cj = c / nx, ri = r % nx, rj = r / nx;
    const int di = ri - ci, dj = rj - cj;
    if (di < -1 || di > 1 || dj < -1 || dj > 1) return -1;
    return (di + 1) + 3 * (dj + 1);
}

// Checks that (Ap, Ai) is a valid compressed-column pattern of an n x n
// matrix contained in the 9-point stencil of an nx-wide grid.
int check_pattern(int n, int nx, const int *Ap, const int *Ai) {
    if (Ap[0] != 0) return fail(UMFPACK_ERROR_invalid_matrix, "Ap[0] = %d, not 0", Ap[0]);
    for (int c = 0; c < n; ++c) {
        if (Ap[c + 1] < Ap[c]) return fail(UMFPACK_ERROR_invalid_matrix, "Ap decreases at column %d", c);
        if (Ap[c + 1] - Ap[c] > 9)
            return fail(UMFPACK_ERROR_invalid_matrix, "column %d has %d entries: not a 9-point grid matrix", c,
                        Ap[c + 1] - Ap[c]);
        int last = -1;
        for (int p = Ap[c]; p < Ap[c + 1]; ++p) {
            const int r = Ai[p];
            if (r < 0 || r >= n) return fail(UMFPACK_ERROR_invalid_matrix, "row index %d out of range in column %d", r, c);
            if (r <= last) return fail(UMFPACK_ERROR_invalid_matrix, "rows not ascending in column %d", c);
            last = r;
            if (stencil_dir(r, c, nx) < 0)
                return fail(UMFPACK_ERROR_invalid_matrix,
                            "entry (%d, %d) is outside the 9-point stencil of a %d-wide grid", r, c, nx);
        }
    }
    return UMFPACK_OK;
}

}  // namespace

extern "C" const char *gm_umfpack_last_error(void) { return g_err.c_str(); }

extern "C" int umfpack_zi_triplet_to_col(int n_row, int n_col, int nz, const int Ti[], const int Tj[],
                                         const double Tx[], const double Tz[], int Ap[], int Ai[],
                                         double Ax[], double Az[], int Map[]) {
    if (!Ti || !Tj || !Ap || !Ai) return fail(UMFPACK_ERROR_argument_missing, "triplet_to_col: missing array");
    if (n_row <= 0 || n_col <= 0) return fail(UMFPACK_ERROR_n_nonpositive, "triplet_to_col: n_row/n_col must be positive");
    if (nz < 0) return fail(UMFPACK_ERROR_invalid_matrix, "triplet_to_col: nz < 0");
    for (int k = 0; k < nz; ++k)
        if (Ti[k] < 0 || Ti[k] >= n_row || Tj[k] < 0 || Tj[k] >= n_col)
            return fail(UMFPACK_ERROR_invalid_matrix, "triplet %d = (%d, %d) out of range", k, Ti[k], Tj[k]);
    const bool values = Tx && Ax;
    const bool packed = values && !Tz && !Az;   // interleaved complex in Tx / Ax
    try {
        // counting sort by column, then by row within each column (stable
        // in the triplet order, so duplicates are summed in input order)
        std::vector<int> cnt(n_col + 1, 0), order(nz);
        for (int k = 0; k < nz; ++k) ++cnt[Tj[k] + 1];
        for (int c = 0; c < n_col; ++c) cnt[c + 1] += cnt[c];
        {
            std::vector<int> pos(cnt.begin(), cnt.end() - 1);
            for (int k = 0; k < nz; ++k) order[pos[Tj[k]]++] = k;
        }
        int nnz = 0;
        std::vector<std::pair<int, int>> col;
        for (int c = 0; c < n_col; ++c) {
            Ap[c] = nnz;
            col.clear();
            for (int t = cnt[c]; t < cnt[c + 1]; ++t) col.emplace_back(Ti[order[t]], order[t]);
            std::stable_sort(col.begin(), col.end(),
                             [](const std::pair<int, int> &a, const std::pair<int, int> &b) { return a.first < b.first; });
            for (size_t t = 0; t < col.size(); ++t) {
                const int r = col[t].first, k = col[t].second;
                const bool dup = t > 0 && col[t - 1].first == r;
                if (!dup) {
                    Ai[nnz] = r;
                    if (values) {
                        if (packed) {
                            Ax[2 * nnz] = 0.0;
                            Ax[2 * nnz + 1] = 0.0;
                        } else {
                            Ax[nnz] = 0.0;
                            if (Az) Az[nnz] = 0.0;
                        }
                    }
                    ++nnz;
                }
                const int p = nnz - 1;
                if (values) {
                    if (packed) {
                        Ax[2 * p] += Tx[2 * k];
                        Ax[2 * p + 1] += Tx[2 * k + 1];
                    } else {
                        Ax[p] += Tx[k];
                        if (Az) Az[p] += Tz ? Tz[k] : 0.0;
                    }
                }
                if (Map) Map[k] = p;
            }
        }
        Ap[n_col] = nnz;
    } catch (const std::bad_alloc &) {
        return fail(UMFPACK_ERROR_out_of_memory, "triplet_to_col: out of host memory");
    }
    return UMFPACK_OK;
}

extern "C" int umfpack_zi_symbolic(int n_row, int n_col, const int Ap[], const int Ai[], const double Ax[],
                                   const double Az[], void **Symbolic_out, const double Control[], double Info[]) {
    (void)Ax; (void)Az; (void)Control;
    if (!Symbolic_out || !Ap || !Ai) return info_status(Info, fail(UMFPACK_ERROR_argument_missing, "symbolic: missing argument"));
    *Symbolic_out = nullptr;
    if (n_row <= 0 || n_col <= 0) return info_status(Info, fail(UMFPACK_ERROR_n_nonpositive, "symbolic: n must be positive"));
    if (n_row != n_col)
        return info_status(Info, fail(UMFPACK_ERROR_invalid_matrix, "symbolic: only square grid matrices (%d x %d)", n_row, n_col));
    const int n = n_col;
    // column 0 is grid point (0, 0): its rows are {0, 1, NX, NX + 1}
    int nx = 0;
    for (int p = Ap[0]; p < Ap[1]; ++p)
        if (Ai[p] >= 2) { nx = Ai[p]; break; }
    if (nx < 3 || n % nx != 0 || n / nx < 3)
        return info_status(Info, fail(UMFPACK_ERROR_invalid_matrix,
                                      "symbolic: cannot read a grid width from column 0 (n = %d): not a 9-point grid matrix", n));
    int st = check_pattern(n, nx, Ap, Ai);
    if (st) return info_status(Info, st);
    auto *s = new (std::nothrow) Symbolic();
    if (!s) return info_status(Info, fail(UMFPACK_ERROR_out_of_memory, "symbolic: out of host memory"));
    s->n = n;
    s->nx = nx;
    s->ny = n / nx;
    s->nnz = Ap[n];
    *Symbolic_out = s;
    return info_status(Info, UMFPACK_OK);
}

extern "C" int umfpack_zi_numeric(const int Ap[], const int Ai[], const double Ax[], const double Az[],
                                  void *Symbolic_in, void **Numeric_out, const double Control[], double Info[]) {
    (void)Control;
    if (!Numeric_out || !Ap || !Ai || !Ax) return info_status(Info, fail(UMFPACK_ERROR_argument_missing, "numeric: missing argument"));
    *Numeric_out = nullptr;
    const Symbolic *s = static_cast<const Symbolic *>(Symbolic_in);
    if (!s || s->magic != kSymMagic) return info_status(Info, fail(UMFPACK_ERROR_invalid_Symbolic_object, "numeric: invalid Symbolic object"));
    const int n = s->n, nx = s->nx;
    if (Ap[n] != s->nnz) return info_status(Info, fail(UMFPACK_ERROR_different_pattern, "numeric: pattern differs from the symbolic one"));
    const bool packed = !Az;
    std::vector<double> re, im;
    try {
        re.assign((size_t)9 * n, 0.0);
        im.assign((size_t)9 * n, 0.0);
    } catch (const std::bad_alloc &) {
        return info_status(Info, fail(UMFPACK_ERROR_out_of_memory, "numeric: out of host memory"));
    }
    for (int c = 0; c < n; ++c)
        for (int p = Ap[c]; p < Ap[c + 1]; ++p) {
            const int r = Ai[p];
            const int q = (r >= 0 && r < n) ? stencil_dir(r, c, nx) : -1;
            if (q < 0) return info_status(Info, fail(UMFPACK_ERROR_different_pattern, "numeric: entry (%d, %d) not in the symbolic pattern", r, c));
            re[(size_t)q * n + c] = packed ? Ax[2 * (size_t)p] : Ax[p];
            im[(size_t)q * n + c] = packed ? Ax[2 * (size_t)p + 1] : Az[p];
        }
    int rc = 0;
    gm_engine *e = take_engine(nx, s->ny, &rc);
    if (!e) return info_status(Info, rc);
    const int st = gm_factor_values(e, 1, re.data(), im.data());
    if (st < 0) {
        fail(UMFPACK_ERROR_internal_error, "numeric: %s", gm_last_error());
        gm_engine_destroy(e);
        return info_status(Info, st == GM_ERROR_OUT_OF_MEMORY ? UMFPACK_ERROR_out_of_memory : UMFPACK_ERROR_internal_error);
    }
    auto *num = new (std::nothrow) Numeric();
    if (!num) {
        give_engine(nx, s->ny, e);
        return info_status(Info, fail(UMFPACK_ERROR_out_of_memory, "numeric: out of host memory"));
    }
    num->n = n;
    num->nx = nx;
    num->ny = s->ny;
    num->e = e;
    *Numeric_out = num;
    return info_status(Info, st == GM_WARNING_PERTURBED ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK);
}

extern "C" int umfpack_zi_solve(int sys, const int Ap[], const int Ai[], const double Ax[], const double Az[],
                                double Xx[], double Xz[], const double Bx[], const double Bz[], void *Numeric_in,
                                const double Control[], double Info[]) {
    (void)Ap; (void)Ai; (void)Ax; (void)Az; (void)Control;
    Numeric *num = static_cast<Numeric *>(Numeric_in);
    if (!num || num->magic != kNumMagic) return info_status(Info, fail(UMFPACK_ERROR_invalid_Numeric_object, "solve: invalid Numeric object"));
    if (!Xx || !Bx) return info_status(Info, fail(UMFPACK_ERROR_argument_missing, "solve: missing X or B"));
    if (sys != UMFPACK_A && sys != UMFPACK_At && sys != UMFPACK_Aat)
        return info_status(Info, fail(UMFPACK_ERROR_invalid_system, "solve: sys %d is not supported (A, At, Aat only)", sys));
    const bool packed = !Xz && !Bz;
    if (!packed && (!Xz || !Bz)) return info_status(Info, fail(UMFPACK_ERROR_argument_missing, "solve: only one imaginary array given"));
    const int n = num->n;
    // A^H x = b  <=>  A^T conj(x) = conj(b)
    const bool conj = sys == UMFPACK_At;
    const int gsys = sys == UMFPACK_A ? GM_SYS_A : GM_SYS_AT;
    std::vector<double> b, x;
    try {
        b.resize(2 * (size_t)n);
        x.resize(2 * (size_t)n);
    } catch (const std::bad_alloc &) {
        return info_status(Info, fail(UMFPACK_ERROR_out_of_memory, "solve: out of host memory"));
    }
    const double sg = conj ? -1.0 : 1.0;
    for (int k = 0; k < n; ++k) {
        b[2 * (size_t)k] = packed ? Bx[2 * (size_t)k] : Bx[k];
        b[2 * (size_t)k + 1] = sg * (packed ? Bx[2 * (size_t)k + 1] : Bz[k]);
    }
    const int st = gm_solve(num->e, gsys, 1, b.data(), x.data());
    if (st < 0) return info_status(Info, fail(UMFPACK_ERROR_internal_error, "solve: %s", gm_last_error()));
    for (int k = 0; k < n; ++k) {
        const double xr = x[2 * (size_t)k], xi = sg * x[2 * (size_t)k + 1];
        if (packed) {
            Xx[2 * (size_t)k] = xr;
            Xx[2 * (size_t)k + 1] = xi;
        } else {
            Xx[k] = xr;
            Xz[k] = xi;
        }
    }
    // refinement short of the target is reported, like UMFPACK's
    // ill-conditioning warning, with the singular-matrix code
    return info_status(Info, st == GM_WARNING_NOT_CONVERGED ? UMFPACK_WARNING_singular_matrix : UMFPACK_OK);
}

extern "C" void umfpack_zi_free_symbolic(void **Symbolic_io) {
    if (!Symbolic_io || !*Symbolic_io) return;
    Symbolic *s = static_cast<Symbolic *>(*Symbolic_io);
    if (s->magic == kSymMagic) {
        s->magic = 0;
        delete s;
    }
    *Symbolic_io = nullptr;
}

extern "C" void umfpack_zi_free_numeric(void **Numeric_io) {
    if (!Numeric_io || !*Numeric_io) return;
    Numeric *num = static_cast<Numeric *>(*Numeric_io);
    if (num->magic == kNumMagic) {
        give_engine(num->nx, num->ny, num->e);
        num->magic = 0;
        delete num;
    }
    *Numeric_io = nullptr;
}
