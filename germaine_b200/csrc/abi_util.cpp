// gm_cgemm_sub_c64: the batched complex GEMM of the factorisation as a
// stand-alone C-ABI call (device pointers), for testing the tensor-core
// kernel against the CUDA-core one.
#include <vector>

#include "common.hpp"
#include "kernels_tc.cuh"

extern "C" int gm_cgemm_sub_c64(int device, int backend, int nprob, const int32_t *dims, void *const *A,
                                void *const *B, void *const *C) {
    if (nprob <= 0 || !dims || !A || !B || !C || (backend != 0 && backend != 1))
        return gm::fail(GM_ERROR_INVALID, "gm_cgemm_sub_c64: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_cgemm_sub_c64: bad device");
    std::vector<gm::CgemmProb> probs(nprob);
    std::vector<int4> tiles;
    const int tm = gm::cgemm_tile_rows(), tn = gm::cgemm_tile_cols();
    for (int i = 0; i < nprob; ++i) {
        const int32_t *d = dims + 6 * i;   // m, n, k, lda, ldb, ldc
        if (d[0] < 0 || d[1] < 0 || d[2] < 0 || d[3] < d[0] || d[4] < d[2] || d[5] < d[0])
            return gm::fail(GM_ERROR_INVALID, "gm_cgemm_sub_c64: bad dimensions for problem %d", i);
        probs[i] = {static_cast<const float2 *>(A[i]), static_cast<const float2 *>(B[i]), static_cast<float2 *>(C[i]),
                    d[3], d[4], d[5], d[0], d[1], d[2]};
        for (int a = 0; a < (d[0] + tm - 1) / tm; ++a)
            for (int b = 0; b < (d[1] + tn - 1) / tn; ++b) tiles.push_back(make_int4(i, a, b, 0));
    }
    gm::CgemmProb *dp = nullptr;
    int4 *dt = nullptr;
    int *derr = nullptr;
    int rc = GM_OK;
    if (cudaMalloc(&dp, probs.size() * sizeof(gm::CgemmProb)) != cudaSuccess ||
        cudaMalloc(&dt, (tiles.size() + 1) * sizeof(int4)) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
        rc = gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_cgemm_sub_c64: device allocation failed");
    } else {
        cudaMemcpy(dp, probs.data(), probs.size() * sizeof(gm::CgemmProb), cudaMemcpyHostToDevice);
        cudaMemcpy(dt, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice);
        cudaMemset(derr, 0, sizeof(int));
        gm::launch_cgemm_sub(backend, dp, dt, (int)tiles.size(), derr, 0);
        cudaError_t e = cudaDeviceSynchronize();
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = gm::fail(GM_ERROR_CUDA, "gm_cgemm_sub_c64: %s", cudaGetErrorString(e));
        else if (herr) rc = gm::fail(GM_ERROR_CUDA, "gm_cgemm_sub_c64: tensor-core wait timed out");
    }
    cudaFree(dp);
    cudaFree(dt);
    cudaFree(derr);
    return rc;
}

extern "C" int gm_wait_probe(int device, long long polls, int *timed_out) {
    if (!timed_out || polls < 1 || polls > (1ll << 24))
        return gm::fail(GM_ERROR_INVALID, "gm_wait_probe: polls must be in 1 .. 2^24");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_wait_probe: bad device");
    int *d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_wait_probe: allocation");
    cudaMemset(d, 0xff, sizeof(int));
    gm::launch_wait_probe(polls, d, 0);
    cudaError_t e = cudaDeviceSynchronize();
    int h = -1;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_wait_probe: %s", cudaGetErrorString(e));
    *timed_out = h;
    return GM_OK;
}
