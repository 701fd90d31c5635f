// Gradient post-processing on the device: the Gaussian smoothing of the
// gradient that precond() applies before the l-BFGS step when SPATFILTER = 1
// (src/precond.c:18, src/gauss_filt.c:10-141).  The filter weights are built
// on the host with the reference's own float / double arithmetic
// (host_setup.c: gmh_gauss_kernel); the device convolution accumulates in
// float in the reference's order (taps along x outer, along y inner) with
// separately rounded products and sums, so the result is bit-identical.
// HBM-bound: the gradient is read through L1 (each value is reused by every
// output cell whose window covers it), one float per cell written.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "host_setup.h"
#include "kernels.cuh"

namespace gm {

constexpr int GAUSS_WMAX = 12288;   // weights held in shared memory (48 KB)

__global__ void __launch_bounds__(256) k_gauss_filt(const float *__restrict__ in, float *__restrict__ out, int nx,
                                                    int ny, const float *__restrict__ wg, int hfsx, int hfsy) {
    extern __shared__ float w[];
    const int nwx = 2 * hfsx + 1, nw = nwx * (2 * hfsy + 1);
    for (int t = threadIdx.x; t < nw; t += blockDim.x) w[t] = wg[t];
    __syncthreads();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nx * ny) return;
    const int i = k % nx, j = k / nx;
    float conv = 0.0f;
    for (int ii = -hfsx; ii <= hfsx; ++ii) {
        const int xi = min(max(i + ii, 0), nx - 1);   // the edge extension of gauss_filt.c:72-100
        for (int jj = -hfsy; jj <= hfsy; ++jj) {
            const int yj = min(max(j + jj, 0), ny - 1);
            conv = __fadd_rn(conv, __fmul_rn(__ldg(in + (size_t)yj * nx + xi), w[(jj + hfsy) * nwx + ii + hfsx]));
        }
    }
    out[k] = conv;
}

}  // namespace gm

extern "C" int gm_gauss_filt(int device, int nx, int ny, float dh, float vref, float fc_low, float filt_size_grad,
                             float filt_size_grad1, const float *grad, float *out) {
    if (nx <= 0 || ny <= 0 || !grad || !out || !(dh > 0.f) || !(fc_low > 0.f))
        return gm::fail(GM_ERROR_INVALID, "gm_gauss_filt: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_gauss_filt: bad device %d", device);
    const size_t n = (size_t)nx * ny;
    std::vector<float> w(gm::GAUSS_WMAX);
    int hfs[2] = {0, 0};
    const int nw = gmh_gauss_kernel(dh, vref, fc_low, filt_size_grad, filt_size_grad1, hfs, w.data(), gm::GAUSS_WMAX);
    if (nw < 0) return gm::fail(GM_ERROR_INVALID, "gm_gauss_filt: filter window larger than %d taps", gm::GAUSS_WMAX);
    if (nw == 0) {   // filter size 0: gauss_filt returns without touching the gradient
        if (out != grad && cudaMemcpy(out, grad, n * sizeof(float), cudaMemcpyDefault) != cudaSuccess)
            return gm::fail(GM_ERROR_CUDA, "gm_gauss_filt: copy failed");
        return GM_OK;
    }
    float *din = nullptr, *dout = nullptr, *dw = nullptr;
    int rc = GM_OK;
    if (cudaMalloc(&din, n * sizeof(float)) != cudaSuccess || cudaMalloc(&dout, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dw, nw * sizeof(float)) != cudaSuccess) {
        rc = gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_gauss_filt: device allocation failed");
    } else if (cudaMemcpy(din, grad, n * sizeof(float), cudaMemcpyDefault) != cudaSuccess ||
               cudaMemcpy(dw, w.data(), nw * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = gm::fail(GM_ERROR_CUDA, "gm_gauss_filt: upload failed");
    } else {
        const int tpb = 256;
        gm::k_gauss_filt<<<(unsigned)((n + tpb - 1) / tpb), tpb, nw * sizeof(float)>>>(din, dout, nx, ny, dw, hfs[0],
                                                                                      hfs[1]);
        gm::note_launch();
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * sizeof(float), cudaMemcpyDefault);
        if (e != cudaSuccess) rc = gm::fail(GM_ERROR_CUDA, "gm_gauss_filt: %s", cudaGetErrorString(e));
    }
    cudaFree(din);
    cudaFree(dout);
    cudaFree(dw);
    return rc;
}

// ---- apply_hess_AC (src/AC/apply_hess_AC.c:11-40) ----
// MAX_HESS = max |hess| (NaN entries never pass the reference's ">" test,
// fmaxf skips them alike); grad *= 1.0 / (hess + EPS_HESS * MAX_HESS) with
// the reference's types: the denominator summed in float, the reciprocal and
// the product in double, the result rounded to float.  The maximum of
// non-negative floats is the maximum of their bit patterns, so the
// reduction is an atomicMax on the bits and does not depend on the order.
namespace gm {

__global__ void __launch_bounds__(256) k_hess_max(const float *__restrict__ hess, size_t n, unsigned *maxbits) {
    float m = 0.0f;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(hess[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
}

__global__ void __launch_bounds__(256) k_apply_hess(float *__restrict__ grad, const float *__restrict__ hess, size_t n,
                                                    float eps_hess, const unsigned *maxbits) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float em = __fmul_rn(eps_hess, __uint_as_float(*maxbits));
    const double q = __ddiv_rn(1.0, (double)__fadd_rn(hess[k], em));
    grad[k] = __double2float_rn(__dmul_rn((double)grad[k], q));
}

}  // namespace gm

extern "C" int gm_apply_hess(int device, int n, float eps_hess, float *grad, const float *hess, float *max_hess) {
    if (n <= 0 || !grad || !hess) return gm::fail(GM_ERROR_INVALID, "gm_apply_hess: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_apply_hess: bad device %d", device);
    const size_t bytes = (size_t)n * sizeof(float);
    float *dg = nullptr, *dh = nullptr;
    unsigned *dmax = nullptr;
    int rc = GM_OK;
    if (cudaMalloc(&dg, bytes) != cudaSuccess || cudaMalloc(&dh, bytes) != cudaSuccess ||
        cudaMalloc(&dmax, sizeof(unsigned)) != cudaSuccess) {
        rc = gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_apply_hess: device allocation failed");
    } else if (cudaMemcpy(dg, grad, bytes, cudaMemcpyDefault) != cudaSuccess ||
               cudaMemcpy(dh, hess, bytes, cudaMemcpyDefault) != cudaSuccess ||
               cudaMemset(dmax, 0, sizeof(unsigned)) != cudaSuccess) {
        rc = gm::fail(GM_ERROR_CUDA, "gm_apply_hess: upload failed");
    } else {
        const int tpb = 256;
        const unsigned nblk = (unsigned)std::min<size_t>(((size_t)n + tpb - 1) / tpb, 148 * 8);
        gm::k_hess_max<<<nblk, tpb>>>(dh, (size_t)n, dmax);
        gm::note_launch();
        gm::k_apply_hess<<<(unsigned)(((size_t)n + tpb - 1) / tpb), tpb>>>(dg, dh, (size_t)n, eps_hess, dmax);
        gm::note_launch();
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(grad, dg, bytes, cudaMemcpyDefault);
        unsigned bits = 0;
        if (e == cudaSuccess && max_hess) {
            e = cudaMemcpy(&bits, dmax, sizeof(unsigned), cudaMemcpyDeviceToHost);
            std::memcpy(max_hess, &bits, sizeof(float));
        }
        if (e != cudaSuccess) rc = gm::fail(GM_ERROR_CUDA, "gm_apply_hess: %s", cudaGetErrorString(e));
    }
    cudaFree(dg);
    cudaFree(dh);
    cudaFree(dmax);
    return rc;
}

// ---- precond (src/precond.c:10-24): gauss_filt, taper_grad_hor, taper_grad_file ----
// taper_grad_hor (src/taper_grad_hor.c:20-31): rows j <= GRADT2 + FSSHIFT
// (1-based) set to zero.  taper_grad_file (src/taper_grad_file.c:18-70):
// the interior multiplied by the taper read from "taper.bin" (NX0 x NY0
// floats, x outer), then the frame filled from the nearest interior column
// (left, right: every row), the top NPML rows from row NPML+1 when
// FREE_SURF == 1 (for a free surface those are interior rows -- the
// reference overwrites them; it leaves the frame rows of FREE_SURF == 0
// as the column copies left them) and the bottom rows from row
// FSSHIFT+NY0.  All float multiplications and copies: bit-identical.
namespace gm {

__global__ void k_taper_hor(float *g, int nx, int rows) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < rows * nx) g[t] = 0.0f;
}

__global__ void k_taper_file_mul(float *g, const float *__restrict__ tap, int nx, int npml, int fsshift, int nx0,
                                 int ny0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;   // t = i * ny0 + j: file order
    if (t >= nx0 * ny0) return;
    const int i = t / ny0, j = t % ny0;
    float &v = g[(size_t)(j + fsshift) * nx + (i + npml)];
    v = __fmul_rn(v, tap[t]);
}

__global__ void k_taper_file_lr(float *g, int nx, int ny, int npml, int nx0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ny) return;
    float *row = g + (size_t)j * nx;
    const float l = row[npml], r = row[npml + nx0 - 1];
    for (int i = 0; i < npml; ++i) row[i] = l;
    for (int i = npml + nx0; i < nx; ++i) row[i] = r;
}

__global__ void k_taper_file_tb(float *g, int nx, int ny, int npml, int free_surf, int fsshift, int ny0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    if (free_surf == 1)
        for (int j = 0; j < npml; ++j) g[(size_t)j * nx + i] = g[(size_t)npml * nx + i];
    for (int j = fsshift + ny0; j < ny; ++j) g[(size_t)j * nx + i] = g[(size_t)(fsshift + ny0 - 1) * nx + i];
}

}  // namespace gm

extern "C" int gm_precond(int device, int nx, int ny, int npml, int free_surf, float dh, int spatfilter, float vref,
                          float fc_low, float filt_size_grad, float filt_size_grad1, int taper_hor, int gradt2,
                          const float *taper, float *grad) {
    if (nx <= 0 || ny <= 0 || npml < 0 || !grad) return gm::fail(GM_ERROR_INVALID, "gm_precond: bad argument");
    const int fsshift = free_surf ? 0 : npml, nx0 = nx - 2 * npml, ny0 = ny - npml - fsshift;
    if (taper && (nx0 <= 0 || ny0 <= 0)) return gm::fail(GM_ERROR_INVALID, "gm_precond: grid without interior");
    int rc;
    if (spatfilter == 1 && (rc = gm_gauss_filt(device, nx, ny, dh, vref, fc_low, filt_size_grad, filt_size_grad1, grad, grad)))
        return rc;
    if (!taper_hor && !taper) return GM_OK;
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_precond: bad device %d", device);
    const size_t n = (size_t)nx * ny;
    float *dg = nullptr, *dt = nullptr;
    rc = GM_OK;
    cudaError_t e = cudaMalloc(&dg, n * sizeof(float));
    if (e == cudaSuccess && taper) e = cudaMalloc(&dt, (size_t)nx0 * ny0 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(dg, grad, n * sizeof(float), cudaMemcpyDefault);
    if (e == cudaSuccess && taper) e = cudaMemcpy(dt, taper, (size_t)nx0 * ny0 * sizeof(float), cudaMemcpyDefault);
    if (e == cudaSuccess && taper_hor) {
        const int rows = std::min(ny, std::max(0, gradt2 + fsshift));
        if (rows > 0) {
            gm::k_taper_hor<<<(rows * nx + 255) / 256, 256>>>(dg, nx, rows);
            gm::note_launch();
        }
    }
    if (e == cudaSuccess && taper) {
        gm::k_taper_file_mul<<<(nx0 * ny0 + 255) / 256, 256>>>(dg, dt, nx, npml, fsshift, nx0, ny0);
        gm::k_taper_file_lr<<<(ny + 127) / 128, 128>>>(dg, nx, ny, npml, nx0);
        gm::k_taper_file_tb<<<(nx + 127) / 128, 128>>>(dg, nx, ny, npml, free_surf, fsshift, ny0);
        gm::note_launch();
        gm::note_launch();
        gm::note_launch();
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(grad, dg, n * sizeof(float), cudaMemcpyDefault);
    if (e != cudaSuccess) rc = gm::fail(GM_ERROR_CUDA, "gm_precond: %s", cudaGetErrorString(e));
    cudaFree(dg);
    cudaFree(dt);
    return rc;
}
