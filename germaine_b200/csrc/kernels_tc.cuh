// Batched complex-FP32 GEMM C -= A * B (tcgen05 tensor cores or CUDA cores).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace gm {

// A: m x k, B: k x n, C: m x n, column-major with leading dimensions lda/ldb/ldc
using CgemmProb = GemmProb<float>;

// tiles[t] = (problem, tile row, tile column) of a 128 x 64 output tile;
// backend 1 = tcgen05 (3xTF32), 0 = CUDA cores.  *d_err is set to 1 if a
// tensor-core wait timed out.
void launch_cgemm_sub(int backend, const CgemmProb *d_probs, const int4 *d_tiles, int ntiles, int *d_err,
                      cudaStream_t st);
// one CTA waits, with the tensor-core kernels' bounded wait, on an mbarrier
// that nothing signals; *d_status = 1 when the wait ran out (device memory)
void launch_wait_probe(long long limit, int *d_status, cudaStream_t st);
int cgemm_tile_rows();
int cgemm_tile_cols();

}  // namespace gm
