// On-disk formats of the reference, so that the engine's outputs and inputs
// are byte-compatible with GERMAINE's files:
//   seismograms  <PICKS_FILE>_p_stage_<n>.bin  write_seis_AC (src/AC/write_seis_AC.c:53-67),
//                read back by read_seis_AC (src/AC/read_seis_AC.c:24-37):
//                float (re, im) pairs, frequency outer, shot, receiver inner --
//                the [nf][nshots][ntr] complex64 layout gm_forward returns.
//                write_seis_AC reduces its 1-based arrays from element 0
//                (src/AC/write_seis_AC.c:43-44: the count is n but the NR
//                vectors hold data in [1..n]), so the gathered copy never
//                receives element n and the LAST sample of every file is
//                written as 0 + 0i; gm_write_seis does the same unless
//                GM_SEIS_KEEP_LAST is given;
//   models and snapshots without the PML frame  writemod_true
//                (src/writemod_true.c:26-34): the interior NX0 x NY0 floats,
//                x outer, y inner, every IDX-th column and IDY-th row;
//   models with the frame  writemod (src/writemod.c:24-30) in binary
//                format 3 (src/writedsk.c:32-40): the full NX x NY grid,
//                same order and subsampling;
//   full grids read back  the layout writemod and the reference's l-BFGS
//                "*.old" files (src/LBFGS.c:183-216) and Hessian files
//                (src/AC/hessian_AC.c:178-188) are written in: NX x NY
//                floats, x outer (gm_read_grid);
//   material models  readmod (src/readmod.c:43-104; readmod_SH, readmod_TE
//                alike): the interior layout of writemod_true, extended into
//                the PML frame by copying the nearest interior value (left /
//                right columns, then top rows unless FREE_SURF, then bottom
//                rows);
//   source wavelet  the SU trace read_stf_dft reads (src/read_stf_dft.c:
//                24-52): a 240-byte trace header (sample count and
//                interval as unsigned shorts at bytes 114 and 116), then the
//                samples as floats (gm_stf_dft).
// Host code only (plain stdio); grids are flat row-major [NY][NX] over the
// full grid including the frame.
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "germaine_gpu.h"
#include "host_setup.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

int frame(int nx, int ny, int npml, int free_surf, int &nx0, int &ny0, int &yshift) {
    yshift = free_surf ? 0 : npml;
    nx0 = nx - 2 * npml;
    ny0 = ny - npml - yshift;
    if (nx <= 0 || ny <= 0 || npml < 0 || nx0 <= 0 || ny0 <= 0)
        return gm::fail(GM_ERROR_INVALID, "grid %d x %d with NPML %d has no interior", nx, ny, npml);
    return GM_OK;
}

// x-outer columns of rows [y0, y0 + nyw) and columns [x0, x0 + nxw) of a
// row-major grid, every idx-th column and idy-th row
int write_columns(const char *who, const char *path, const float *grid, int nx, int x0, int nxw, int y0, int nyw,
                  int idx, int idy) {
    File fp(path, "wb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "%s: cannot open %s", who, path);
    std::vector<float> col;
    for (int i = 0; i < nxw; i += idx) {
        col.clear();
        for (int j = 0; j < nyw; j += idy) col.push_back(grid[(size_t)(j + y0) * nx + (i + x0)]);
        if (std::fwrite(col.data(), sizeof(float), col.size(), fp.f) != col.size())
            return gm::fail(GM_ERROR_INVALID, "%s: write to %s failed", who, path);
    }
    return GM_OK;
}

}  // namespace

extern "C" int gm_write_seis(const char *path, int nf, int nshots, int ntr, int flags, const float *seis) {
    if (!path || !seis || nf <= 0 || nshots <= 0 || ntr <= 0 || (flags & ~GM_SEIS_KEEP_LAST))
        return gm::fail(GM_ERROR_INVALID, "gm_write_seis: bad argument");
    File fp(path, "wb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "gm_write_seis: cannot open %s", path);
    const size_t cnt = (size_t)2 * nf * nshots * ntr;
    const size_t head = (flags & GM_SEIS_KEEP_LAST) ? cnt : cnt - 2;
    const float zero[2] = {0.0f, 0.0f};
    if (std::fwrite(seis, sizeof(float), head, fp.f) != head ||
        (head < cnt && std::fwrite(zero, sizeof(float), 2, fp.f) != 2))
        return gm::fail(GM_ERROR_INVALID, "gm_write_seis: write to %s failed", path);
    return GM_OK;
}

extern "C" int gm_read_seis(const char *path, int nf, int nshots, int ntr, float *seis) {
    if (!path || !seis || nf <= 0 || nshots <= 0 || ntr <= 0) return gm::fail(GM_ERROR_INVALID, "gm_read_seis: bad argument");
    File fp(path, "rb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "gm_read_seis: cannot open %s", path);
    const size_t cnt = (size_t)2 * nf * nshots * ntr;
    if (std::fread(seis, sizeof(float), cnt, fp.f) != cnt)
        return gm::fail(GM_ERROR_INVALID, "gm_read_seis: %s holds fewer than %zu floats", path, cnt);
    return GM_OK;
}

extern "C" int gm_write_model_true(const char *path, int nx, int ny, int npml, int free_surf, int idx, int idy,
                                   const float *grid) {
    int nx0, ny0, yshift;
    if (!path || !grid || idx <= 0 || idy <= 0) return gm::fail(GM_ERROR_INVALID, "gm_write_model_true: bad argument");
    if (int rc = frame(nx, ny, npml, free_surf, nx0, ny0, yshift)) return rc;
    return write_columns("gm_write_model_true", path, grid, nx, npml, nx0, yshift, ny0, idx, idy);
}

extern "C" int gm_write_model(const char *path, int nx, int ny, int idx, int idy, const float *grid) {
    if (!path || !grid || nx <= 0 || ny <= 0 || idx <= 0 || idy <= 0)
        return gm::fail(GM_ERROR_INVALID, "gm_write_model: bad argument");
    return write_columns("gm_write_model", path, grid, nx, 0, nx, 0, ny, idx, idy);
}

extern "C" int gm_read_model(const char *path, int nx, int ny, int npml, int free_surf, float *grid) {
    int nx0, ny0, yshift;
    if (!path || !grid) return gm::fail(GM_ERROR_INVALID, "gm_read_model: bad argument");
    if (int rc = frame(nx, ny, npml, free_surf, nx0, ny0, yshift)) return rc;
    File fp(path, "rb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "gm_read_model: cannot open %s", path);
    std::vector<float> col(ny0);
    for (int i = 0; i < nx0; ++i) {
        if (std::fread(col.data(), sizeof(float), ny0, fp.f) != (size_t)ny0)
            return gm::fail(GM_ERROR_INVALID, "gm_read_model: %s holds fewer than %d x %d floats", path, nx0, ny0);
        for (int j = 0; j < ny0; ++j) grid[(size_t)(j + yshift) * nx + (i + npml)] = col[j];
    }
    auto at = [&](int j, int i) -> float & { return grid[(size_t)j * nx + i]; };   // 0-based
    for (int j = yshift; j < yshift + ny0; ++j) {
        for (int i = 0; i < npml; ++i) at(j, i) = at(j, npml);
        for (int i = npml + nx0; i < nx; ++i) at(j, i) = at(j, npml + nx0 - 1);
    }
    for (int j = 0; j < yshift; ++j)
        for (int i = 0; i < nx; ++i) at(j, i) = at(yshift, i);
    for (int j = yshift + ny0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) at(j, i) = at(yshift + ny0 - 1, i);
    return GM_OK;
}

extern "C" int gm_read_grid(const char *path, int nx, int ny, float *grid) {
    if (!path || !grid || nx <= 0 || ny <= 0) return gm::fail(GM_ERROR_INVALID, "gm_read_grid: bad argument");
    File fp(path, "rb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "gm_read_grid: cannot open %s", path);
    std::vector<float> col(ny);
    for (int i = 0; i < nx; ++i) {
        if (std::fread(col.data(), sizeof(float), ny, fp.f) != (size_t)ny)
            return gm::fail(GM_ERROR_INVALID, "gm_read_grid: %s holds fewer than %d x %d floats", path, nx, ny);
        for (int j = 0; j < ny; ++j) grid[(size_t)j * nx + i] = col[j];
    }
    return GM_OK;
}

extern "C" int gm_stf_dft(const char *path, int physics, float freq, float *amp) {
    if (!path || !amp) return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: bad argument");
    if (physics < 1 || physics > 4) return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: unknown physics %d", physics);
    File fp(path, "rb");
    if (!fp.f) return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: cannot open %s", path);
    unsigned char hdr[240];
    if (std::fread(hdr, 1, sizeof hdr, fp.f) != sizeof hdr)
        return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: %s has no 240-byte SU trace header", path);
    unsigned short ns = 0, ndt = 0;
    std::memcpy(&ns, hdr + 114, sizeof ns);
    std::memcpy(&ndt, hdr + 116, sizeof ndt);
    if (ns == 0) return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: %s holds no samples", path);
    std::vector<float> w(ns);
    if (std::fread(w.data(), sizeof(float), ns, fp.f) != ns)
        return gm::fail(GM_ERROR_INVALID, "gm_stf_dft: %s holds fewer than %d samples", path, (int)ns);
    gmh_stf_dft(w.data(), (int)ns, (int)ndt, physics, freq, amp);
    return GM_OK;
}
