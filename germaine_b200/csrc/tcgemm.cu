// Complex-FP32 GEMM  C -= A * B  on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulator in tensor memory), batched over a
// list of problems; the CUDA-core twin (k_cgemm_cc) computes the same thing
// for checking and for shapes too small for a 128-row tile.
//
// A: m x k, B: k x n, C: m x n, complex64, column-major with leading
// dimensions lda/ldb/ldc -- the layout of the dense fronts, so A = L21 and
// B = U12 of a front are read in place.
//
// One CTA (4 warps) owns a 128 x 64 complex output tile:
//   * the complex product is one real MMA stream through the embedding
//       [Pr | Pi] = [Ar | Ai] * [[Br, Bi]; [-Bi, Br]]
//     i.e. real A' (128 x 2k), real B' (128 x 2k, rows 0..63 give Re P,
//     rows 64..127 give Im P), D = A' B'^T (M = 128, N = 128);
//   * each real operand is split into three TF32 pieces x = x1 + x2 + x3
//     (round to nearest, ~33 significant bits in total) and D accumulates
//     the six products of order <= 2 (x1y1, x1y2, x2y1, x1y3, x2y2, x3y1)
//     in FP32 in TMEM: more accurate than an FP32 FMA (a two-piece split,
//     ~22 bits, roughly doubled the refinement sweeps of the
//     mixed-precision solve), still at tensor-core rate;
//   * operands are staged per 16-complex K chunk into shared memory in the
//     canonical K-major, no-swizzle layout (8-row x 16-byte core matrices:
//     leading byte offset = 128 rows x 16 B between the two 16-B K halves
//     of one MMA, stride byte offset = 128 B between 8-row groups);
//   * one elected thread issues the 24 MMAs of a chunk (smallest products
//     first) and commits them to an mbarrier; all threads wait (bounded: on
//     timeout an error flag is set and the kernel winds down) before the
//     shared memory is reused;
//   * the tensor core's FP32 accumulation is not round-to-nearest: its error
//     grows linearly with the number of accumulated products (measured: at
//     K = 454 real terms of one sign, 30x the error of FP32 FMA chains, all
//     of it bias).  So TMEM accumulates one K chunk only; after each chunk
//     every thread moves its accumulator row to registers (tcgen05.ld
//     32x32b: warp w owns lanes 32w..32w+31 = rows of the tile) and adds it
//     to an FP32 register accumulator with ordinary round-to-nearest adds;
//   * epilogue: C -= accumulator with coalesced column-major stores.
#include "kernels_tc.cuh"
#include "cplx.cuh"

namespace gm {

namespace {

constexpr int TM = 128;          // tile rows (M of the MMA)
constexpr int TN = 64;           // complex tile columns (N of the MMA = 2 TN)
constexpr int KC = 16;           // complex K per staged chunk -> 2 KC = 32 real
constexpr int KR = 2 * KC;       // real K per chunk
constexpr int NCHUNK16 = KR / 4; // 16-byte K chunks per operand row
constexpr int OPER_BYTES = NCHUNK16 * 128 * 16;   // one operand piece: 16 KB
constexpr uint32_t TMEM_COLS = 128;
constexpr long long WAIT_LIMIT = 1ll << 26;       // mbarrier polls before giving up

constexpr int NSPLIT = 3;

struct __align__(1024) TcSmem {
    unsigned char a[NSPLIT][OPER_BYTES];
    unsigned char b[NSPLIT][OPER_BYTES];
    unsigned long long mbar;
    uint32_t tmem_addr;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x -> three TF32 pieces (round to nearest each); x - p1 and r1 - p2 are exact
__device__ __forceinline__ void split3(float x, float &p1, float &p2, float &p3) {
    p1 = tf32_rna(x);
    const float r1 = x - p1;
    p2 = tf32_rna(r1);
    p3 = tf32_rna(r1 - p2);
}

// shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// version 1 (Blackwell), base offset 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: kind::tf32, D f32, A/B tf32, both K-major,
// N = 128 (>> 3 at bit 17), M = 128 (>> 4 at bit 24)
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit = WAIT_LIMIT) {
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(addr));
}

// row r (0..127), real K index kr (0..31) -> byte offset in an operand
__device__ __forceinline__ int oper_off(int r, int chunk16) { return chunk16 * (128 * 16) + r * 16; }

}  // namespace

__global__ void __launch_bounds__(128) k_cgemm_tc(const CgemmProb *__restrict__ probs, const int4 *__restrict__ tiles,
                                                  int *err) {
    extern __shared__ unsigned char smem_raw[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int4 tl = tiles[blockIdx.x];
    const CgemmProb p = probs[tl.x];
    const int m0 = tl.y * TM, n0 = tl.z * TN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&sm.tmem_addr)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&sm.mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem_addr;
    const uint32_t mbar = smem_u32(&sm.mbar);
    bool ok = true;

    const int nk = (p.k + KC - 1) / KC;
    float accr[TN], acci[TN];   // this thread's tile row: Re, Im of the product
#pragma unroll
    for (int q = 0; q < TN; ++q) { accr[q] = 0.f; acci[q] = 0.f; }
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int kc = 0; kc < nk && ok; ++kc) {
        const int k0 = kc * KC;
        // ---- stage A': row i = tid, K' = [Re A(i, k0..k0+15) | Im A(i, ...)] ----
        {
            const int i = m0 + tid;
            float re[KC], im[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                float2 v = make_float2(0.f, 0.f);
                if (i < p.m && k0 + q < p.k) v = p.A[(size_t)i + (size_t)(k0 + q) * p.lda];
                re[q] = v.x;
                im[q] = v.y;
            }
#pragma unroll
            for (int c = 0; c < NCHUNK16; ++c) {
                float q1[4], q2[4], q3[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int kr = 4 * c + e;
                    split3(kr < KC ? re[kr] : im[kr - KC], q1[e], q2[e], q3[e]);
                }
                *reinterpret_cast<float4 *>(sm.a[0] + oper_off(tid, c)) = make_float4(q1[0], q1[1], q1[2], q1[3]);
                *reinterpret_cast<float4 *>(sm.a[1] + oper_off(tid, c)) = make_float4(q2[0], q2[1], q2[2], q2[3]);
                *reinterpret_cast<float4 *>(sm.a[2] + oper_off(tid, c)) = make_float4(q3[0], q3[1], q3[2], q3[3]);
            }
        }
        // ---- stage B': row j' = tid; j' < 64: [Re B(:, j) ; -Im B(:, j)], j' >= 64: [Im B(:, j) ; Re B(:, j)] ----
        {
            const int half = tid >> 6, j = n0 + (tid & 63);
            float re[KC], im[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                float2 v = make_float2(0.f, 0.f);
                if (j < p.n && k0 + q < p.k) v = p.B[(size_t)(k0 + q) + (size_t)j * p.ldb];
                re[q] = v.x;
                im[q] = v.y;
            }
#pragma unroll
            for (int c = 0; c < NCHUNK16; ++c) {
                float q1[4], q2[4], q3[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int kr = 4 * c + e;
                    float x;
                    if (half == 0) x = kr < KC ? re[kr] : -im[kr - KC];
                    else x = kr < KC ? im[kr] : re[kr - KC];
                    split3(x, q1[e], q2[e], q3[e]);
                }
                *reinterpret_cast<float4 *>(sm.b[0] + oper_off(tid, c)) = make_float4(q1[0], q1[1], q1[2], q1[3]);
                *reinterpret_cast<float4 *>(sm.b[1] + oper_off(tid, c)) = make_float4(q2[0], q2[1], q2[2], q2[3]);
                *reinterpret_cast<float4 *>(sm.b[2] + oper_off(tid, c)) = make_float4(q3[0], q3[1], q3[2], q3[3]);
            }
        }
        // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t lbo = 128 * 16, sbo = 128;
            uint32_t ab[NSPLIT], bb[NSPLIT];
#pragma unroll
            for (int q = 0; q < NSPLIT; ++q) { ab[q] = smem_u32(sm.a[q]); bb[q] = smem_u32(sm.b[q]); }
            // products of order <= 2, smallest first, each over the chunk's K;
            // the chunk starts from a zero accumulator
            const int pa[6] = {0, 1, 2, 0, 1, 0}, pb[6] = {2, 1, 0, 1, 0, 0};
#pragma unroll
            for (int u = 0; u < 6; ++u) {
#pragma unroll
                for (int t = 0; t < KR / 8; ++t) {
                    const uint32_t off = (uint32_t)t * 2u * (128u * 16u);   // two 16-B K chunks per MMA (K = 8)
                    const uint32_t acc = (t > 0 || u > 0) ? 1u : 0u;
                    mma_tf32(tmem, smem_desc(ab[pa[u]] + off, lbo, sbo), smem_desc(bb[pb[u]] + off, lbo, sbo), acc);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(mbar) : "memory");
        }
        ok = mbar_wait(mbar, (uint32_t)(kc & 1));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!__syncthreads_and(ok)) { ok = false; break; }
        // flush the chunk's accumulator into the register accumulator
#pragma unroll
        for (int js = 0; js < TN; js += 32) {
            uint32_t vr[32], vi[32];
            tmem_ld32(lane_base + (uint32_t)js, vr);
            tmem_ld32(lane_base + (uint32_t)(TN + js), vi);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                accr[js + q] += __uint_as_float(vr[q]);
                acci[js + q] += __uint_as_float(vi[q]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else if (nk > 0) {
        const int i = m0 + warp * 32 + lane;
        if (i < p.m) {
#pragma unroll
            for (int q = 0; q < TN; ++q) {
                const int j = n0 + q;
                if (j < p.n) {
                    float2 &c = p.C[(size_t)i + (size_t)j * p.ldc];
                    c.x -= accr[q];
                    c.y -= acci[q];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS) : "memory");
}

// CUDA-core twin: one thread per output element of the tile (same tiles)
__global__ void __launch_bounds__(128) k_cgemm_cc(const CgemmProb *__restrict__ probs, const int4 *__restrict__ tiles) {
    const int4 tl = tiles[blockIdx.x];
    const CgemmProb p = probs[tl.x];
    const int i = tl.y * TM + threadIdx.x;
    if (i >= p.m) return;
    for (int jj = 0; jj < TN; ++jj) {
        const int j = tl.z * TN + jj;
        if (j >= p.n) break;
        float2 acc = make_float2(0.f, 0.f);
        for (int q = 0; q < p.k; ++q) cfma(acc, p.A[(size_t)i + (size_t)q * p.lda], p.B[(size_t)q + (size_t)j * p.ldb]);
        float2 &c = p.C[(size_t)i + (size_t)j * p.ldc];
        c.x -= acc.x;
        c.y -= acc.y;
    }
}

// The bounded wait of k_cgemm_tc on an mbarrier that no thread ever
// signals: phase 0 never completes, so the wait gives up after `limit`
// polls and the kernel reports it in *status (1 = timed out, 0 = the wait
// returned early, which would be a defect).  Nothing else is in flight:
// no tensor-core work, no memory copies, no TMEM.
__global__ void k_wait_probe(long long limit, int *status) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&bar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait(smem_u32(&bar), 0u, limit);
    __syncthreads();
    if (threadIdx.x == 0) *status = ok ? 0 : 1;
}

void launch_wait_probe(long long limit, int *d_status, cudaStream_t st) {
    (k_wait_probe<<<1, 32, 0, st>>>(limit, d_status), note_launch());
}

size_t cgemm_tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

void launch_cgemm_sub(int backend, const CgemmProb *d_probs, const int4 *d_tiles, int ntiles, int *d_err,
                      cudaStream_t st) {
    if (ntiles <= 0) return;
    if (backend == 1) {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute((const void *)k_cgemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cgemm_tc_smem_bytes());
            attr = true;
        }
        (k_cgemm_tc<<<ntiles, 128, cgemm_tc_smem_bytes(), st>>>(d_probs, d_tiles, d_err), note_launch());
    } else {
        (k_cgemm_cc<<<ntiles, 128, 0, st>>>(d_probs, d_tiles), note_launch());
    }
}

int cgemm_tile_rows() { return TM; }
int cgemm_tile_cols() { return TN; }

}  // namespace gm
