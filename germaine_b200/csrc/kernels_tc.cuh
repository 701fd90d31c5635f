// Batched complex-FP32 GEMM C -= A * B (tcgen05 tensor cores or CUDA cores).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace gm {

struct CgemmProb {
    const float2 *A;   // m x k, column-major, leading dimension lda
    const float2 *B;   // k x n, column-major, ldb
    float2 *C;         // m x n, column-major, ldc
    int lda, ldb, ldc, m, n, k;
};

// tiles[t] = (problem, tile row, tile column) of a 128 x 64 output tile;
// backend 1 = tcgen05 (3xTF32), 0 = CUDA cores.  *d_err is set to 1 if a
// tensor-core wait timed out.
void launch_cgemm_sub(int backend, const CgemmProb *d_probs, const int4 *d_tiles, int ntiles, int *d_err,
                      cudaStream_t st);
int cgemm_tile_rows();
int cgemm_tile_cols();

}  // namespace gm
