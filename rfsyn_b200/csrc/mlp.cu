// mlp.cu -- the learned surrogate's network: a multilayer perceptron
// (GELU hidden layers) trained and evaluated entirely on the GPU with
// hand-written kernels.  rfsyn has no learned component; this maps a scene's
// parameter vector to its tx -> rx transfer function.
//
// Kernels:
//   k_gemm_nt   C[M,N] = A[M,K] . B[N,K]^T on the tensor cores (BF16 operands,
//               mma.sync m16n8k16, FP32 accumulation), 64x64 CTA tiles, A/B
//               tiles staged by cp.async (two stages), fused epilogues: bias +
//               GELU (hidden layers, pre-activation kept in FP32), bias (output
//               layer), GELU' (backward through a hidden layer, dZ in FP32,
//               BF16 and transposed BF16), plain FP32 (weight gradients);
//   k_gemm_tc   the same products and epilogues on tcgen05 (accumulators in
//               tensor memory), selectable; slower on this network's products;
//   k_mse       loss gradient 2 (out - y) / (M N), FP32 / BF16 / transposed,
//               per-block loss partials (deterministic);
//   k_colsum    bias gradients as deterministic column sums of dZ;
//   k_adam      Adam with bias correction and a cosine learning rate taken
//               from the device step counter; writes the BF16 weights and
//               their transposes used by the next step's GEMMs;
//   k_gather    a training batch from the resident data set through a
//               per-epoch permutation and the device step counter.
// One training step is ~8 launches per layer; the whole step is captured in
// a CUDA graph and replayed.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "engine.h"

typedef __nv_bfloat16 bf16;

namespace {

constexpr int GT = 64;   // CTA tile (M and N)
constexpr int GK = 32;   // K per stage
constexpr int SROW = 40; // shared row length (bf16): 80 bytes, conflict-free fragment loads

enum { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_BWD_GELU = 2, EPI_F32 = 3 };

struct Epi {
    const float *bias;   // [N] (HIDDEN, OUT)
    float *f32;          // HIDDEN: pre-activation; OUT: output; BWD_GELU: dZ; F32: C
    bf16 *b16;           // HIDDEN: GELU(pre); BWD_GELU: dZ
    bf16 *b16t;          // BWD_GELU: dZ^T ([N][M])
    const float *pre;    // BWD_GELU: pre-activation of the layer whose output gradient this is
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

__device__ __forceinline__ void cp16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void mma_bf16(float c[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// C = A . B^T.  A: [M][lda] bf16 row-major, B: [N][ldb] bf16 row-major.
// M, N multiples of 64, K a multiple of 32, lda / ldb multiples of 8.
template <int EPI>
__global__ void __launch_bounds__(128) k_gemm_nt(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B,
                                                 int ldb, int M, int N, int K, Epi epi) {
    __shared__ __align__(16) bf16 As[2][GT][SROW];
    __shared__ __align__(16) bf16 Bs[2][GT][SROW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[2][4][4] = {};

    auto load = [&](int st, int k0) {
        // 64 rows x 32 bf16 = 64 x 4 chunks of 16 bytes, per operand
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int c = tid + 128 * q, row = c >> 2, col = (c & 3) * 8;
            cp16(&As[st][row][col], A + (size_t)(m0 + row) * lda + k0 + col);
            cp16(&Bs[st][row][col], B + (size_t)(n0 + row) * ldb + k0 + col);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    const int nk = K / GK;
    load(0, 0);
    for (int kt = 0; kt < nk; kt++) {
        const int st = kt & 1;
        if (kt + 1 < nk) {
            load(st ^ 1, (kt + 1) * GK);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk += 16) {
            unsigned a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                const int r = 32 * wm + 16 * mi + g;
                a[mi][0] = *reinterpret_cast<const unsigned *>(&As[st][r][kk + 2 * t]);
                a[mi][1] = *reinterpret_cast<const unsigned *>(&As[st][r + 8][kk + 2 * t]);
                a[mi][2] = *reinterpret_cast<const unsigned *>(&As[st][r][kk + 2 * t + 8]);
                a[mi][3] = *reinterpret_cast<const unsigned *>(&As[st][r + 8][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ni++) {
                const int c = 32 * wn + 8 * ni + g;
                b[ni][0] = *reinterpret_cast<const unsigned *>(&Bs[st][c][kk + 2 * t]);
                b[ni][1] = *reinterpret_cast<const unsigned *>(&Bs[st][c][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
                    mma_bf16(acc[mi][ni], a[mi][0], a[mi][1], a[mi][2], a[mi][3], b[ni][0], b[ni][1]);
        }
        __syncthreads();  // the stage may be refilled
    }
    // epilogue: acc[mi][ni] covers rows r, r+8 and columns c, c+1
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = m0 + 32 * wm + 16 * mi + g + 8 * h;
                const int c = n0 + 32 * wn + 8 * ni + 2 * t;
                float v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
                const size_t o = (size_t)r * N + c;
                if (EPI == EPI_HIDDEN || EPI == EPI_OUT) {
                    v0 += epi.bias[c];
                    v1 += epi.bias[c + 1];
                    epi.f32[o] = v0;
                    epi.f32[o + 1] = v1;
                    if (EPI == EPI_HIDDEN) {
                        __nv_bfloat162 p;
                        p.x = __float2bfloat16_rn(gelu(v0));
                        p.y = __float2bfloat16_rn(gelu(v1));
                        *reinterpret_cast<__nv_bfloat162 *>(epi.b16 + o) = p;
                    }
                } else if (EPI == EPI_BWD_GELU) {
                    v0 *= gelu_grad(epi.pre[o]);
                    v1 *= gelu_grad(epi.pre[o + 1]);
                    epi.f32[o] = v0;
                    epi.f32[o + 1] = v1;
                    const bf16 b0 = __float2bfloat16_rn(v0), b1 = __float2bfloat16_rn(v1);
                    epi.b16[o] = b0;
                    epi.b16[o + 1] = b1;
                    epi.b16t[(size_t)c * M + r] = b0;
                    epi.b16t[(size_t)(c + 1) * M + r] = b1;
                } else {
                    epi.f32[o] = v0;
                    epi.f32[o + 1] = v1;
                }
            }
}

// ---- the same contraction on the 5th-generation tensor cores ----------------
// k_gemm_tc: C = A . B^T with one tcgen05.mma (M 128, N 32, K 16, BF16 in,
// FP32 accumulation in tensor memory) stream per CTA tile of 128 x 32.
// K is staged 64 at a time (one 128-byte row per tile row) by cp.async into
// a four-stage ring in the 128-byte-swizzled K-major layout the MMA's shared
// memory descriptors describe (16-byte chunk c of row r at chunk c ^ (r % 8)
// of the row, 8-row groups 1024 bytes apart).  One thread issues the four
// MMAs of a stage and commits them to the stage's mbarrier, which frees the
// stage for a later load; the last commit releases the accumulator, which
// eight warps read back (tcgen05.ld, warp w lanes 32 (w % 4) .. +31 = tile
// rows, columns 16 (w / 4) .. +15) into the same fused epilogues as
// k_gemm_nt.  Every wait is bounded: on a timeout the CTA records it,
// waits (bounded) for its MMAs in flight, frees its tensor memory and
// returns.  Measured on the surrogate's network (54-512x4-512, one B200):
// a training step takes 0.226-0.233 ms at batch 256 against 0.189-0.191
// ms on k_gemm_nt, and 0.51 against 0.42 ms at batch 2048 -- products of
// at most 512 x 2048 x 512 are latency-bound on staging their tiles, which
// this cp.async-fed form does no faster than the mma.sync tiles -- so it
// runs only when asked for (RFSYN_FDTD_MLP_GEMM=tcgen05).
namespace tc {
// Tiles of 128 rows x BN columns (BN 32: more CTAs on these small products
// -- 128 x 128 tiles, fewer CTAs and fewer re-reads of A, measured slower
// even on 2048-row batches), K staged 64 at a time in a 4-stage ring filled
// three steps ahead (a refill waits for the MMAs of the step before, which
// take far less than a load)
constexpr int BM = 128, BK = 64, STAGES = 4, DIST = 3, THREADS = 256;
template <int BN>
struct Shape {
    static constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
    static_assert(STAGE_BYTES % 1024 == 0 && A_BYTES % 1024 == 0, "swizzle atoms stay 1024-byte aligned");
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 64;  // tiles 1024-aligned, then barriers, TMEM address
    static constexpr uint32_t TMEM_COLS = BN;                     // FP32 accumulator: a column per output column
    // instruction descriptor: F32 accumulator, BF16 A and B, both K-major,
    // N >> 3 at bit 17, M >> 4 at bit 24
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};
constexpr long long WAIT = 2000000000LL;  // SM cycles, about a second
}  // namespace tc

__device__ __forceinline__ unsigned sm_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory descriptor of a K-major, 128-byte-swizzled operand tile at
// shared address `a`: start address >> 4, leading offset 16 bytes (unused
// with swizzling), stride offset 1024 bytes (one 8-row group), descriptor
// version 1, layout 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t a) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(sm_addr(bar)));
}

__device__ __forceinline__ bool tc_mbar_wait(uint64_t *bar, unsigned parity) {
    const long long t0 = clock64();
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(sm_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > tc::WAIT) return false;
    }
}

template <int EPI>
__device__ __forceinline__ void epi_store(const Epi &epi, int M, int N, int r, int c, float v) {
    const size_t o = (size_t)r * N + c;
    if (EPI == EPI_HIDDEN || EPI == EPI_OUT) {
        v += epi.bias[c];
        epi.f32[o] = v;
        if (EPI == EPI_HIDDEN) epi.b16[o] = __float2bfloat16_rn(gelu(v));
    } else if (EPI == EPI_BWD_GELU) {
        v *= gelu_grad(epi.pre[o]);
        epi.f32[o] = v;
        const bf16 b = __float2bfloat16_rn(v);
        epi.b16[o] = b;
        epi.b16t[(size_t)c * M + r] = b;
    } else {
        epi.f32[o] = v;
    }
}

// C = A . B^T.  A: [M][lda], B: [N][ldb], BF16 row-major (K-major); M a
// multiple of 128, N of 32, K of 64, lda / ldb multiples of 8.
template <int EPI, int BN>
__global__ void __launch_bounds__(tc::THREADS) k_gemm_tc(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B,
                                                 int ldb, int M, int N, int K, Epi epi, int *err) {
    using S = tc::Shape<BN>;
    extern __shared__ unsigned char tc_smem[];
    const unsigned pad = (1024u - (sm_addr(tc_smem) & 1023u)) & 1023u;
    unsigned char *tiles = tc_smem + pad;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tiles + tc::STAGES * S::STAGE_BYTES);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + tc::STAGES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * tc::BM, n0 = blockIdx.x * BN;
    if (tid == 0) {
        for (int s = 0; s < tc::STAGES; s++) tc_mbar_init(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sm_addr(tmem_slot)),
                     "r"(S::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    auto load = [&](int s, int k0) {
        unsigned char *as = tiles + s * S::STAGE_BYTES, *bs = as + S::A_BYTES;
        for (int q = tid; q < tc::BM * 8; q += tc::THREADS) {
            const int r = q >> 3, c = q & 7;
            cp16(as + r * 128 + ((c ^ (r & 7)) << 4), A + (size_t)(m0 + r) * lda + k0 + c * 8);
        }
        for (int q = tid; q < BN * 8; q += tc::THREADS) {
            const int r = q >> 3, c = q & 7;
            cp16(bs + r * 128 + ((c ^ (r & 7)) << 4), B + (size_t)(n0 + r) * ldb + k0 + c * 8);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    const int nk = K / tc::BK;
    bool failed = false;
    int committed = -1;  // the last K step whose MMAs were committed
    for (int p = 0; p < tc::DIST && p < nk; p++) load(p % tc::STAGES, p * tc::BK);
    for (int kt = 0; kt < nk; kt++) {
        const int s = kt % tc::STAGES, nxt = kt + tc::DIST;
        if (nxt < nk) {
            // stage nxt % STAGES was last read by the MMAs of step nxt - STAGES
            const int ns = nxt % tc::STAGES, prev = nxt - tc::STAGES;
            if (prev >= 0 && !tc_mbar_wait(&bar[ns], (prev / tc::STAGES) & 1)) failed = true;
            if (__syncthreads_or(failed)) break;
            load(ns, nxt * tc::BK);
        }
        // step kt's copies are complete once at most the copies of the steps
        // loaded after it are pending
        const int after = nk - 1 - kt < tc::DIST ? nk - 1 - kt : tc::DIST;
        static_assert(tc::DIST <= 3, "the waits below cover up to three later groups");
        if (after >= 3) asm volatile("cp.async.wait_group 3;\n" ::: "memory");
        else if (after == 2) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
        else if (after == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        // make them visible to the tensor core's (async-proxy) reads, then to
        // the issuing thread
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t as = sm_addr(tiles + s * S::STAGE_BYTES), bs = as + S::A_BYTES;
#pragma unroll
            for (int kk = 0; kk < tc::BK / 16; kk++) {
                const uint64_t da = sw128_desc(as + 32 * kk), db = sw128_desc(bs + 32 * kk);
                const uint32_t acc = (kt | kk) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(S::IDESC), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             sm_addr(&bar[s]))
                         : "memory");
        }
        committed = kt;
    }
    // the last commit covers every MMA this CTA issued; copies still in
    // flight (after an early exit) land before the shared memory is released
    if (committed >= 0 && !tc_mbar_wait(&bar[committed % tc::STAGES], (committed / tc::STAGES) & 1)) failed = true;
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (__syncthreads_or(failed)) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // warp w reads TMEM lanes 32 (w % 4) .. (the tile rows it may
        // access) and the BN / 2 columns of half w / 4, 16 at a time
        static_assert(tc::THREADS == 256 && BN % 32 == 0, "eight warps: four lane groups x two column halves");
        const int r = m0 + 32 * (warp & 3) + lane;  // TMEM lane = tile row
#pragma unroll
        for (int cc = (BN / 2) * (warp >> 2); cc < (BN / 2) * ((warp >> 2) + 1); cc += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)cc));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; q++) epi_store<EPI>(epi, M, N, r, n0 + cc + q, __uint_as_float(v[q]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(S::TMEM_COLS)
                     : "memory");
}

// Loss gradient of the mean squared error over M x N outputs; per-block
// partial sums of the squared error (fixed order: deterministic).
__global__ void k_mse(const float *out, const float *y, int M, int N, float *d32, bf16 *d16, bf16 *d16t,
                      float *partial) {
    __shared__ float red[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float se = 0.f;
    if (i < M * N) {
        const float e = out[i] - y[i];
        se = e * e;
        const float gr = 2.0f * e / (float)(M * N);
        d32[i] = gr;
        const bf16 b = __float2bfloat16_rn(gr);
        d16[i] = b;
        const int r = i / N, c = i - r * N;
        d16t[(size_t)c * M + r] = b;
    }
    red[threadIdx.x] = se;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Column sums of d [M][N] (bias gradients), one thread per column.
// Block of 32 columns x 8 warps: warp w sums rows w, w + 8, ... of its
// lane's column, then the eight partial sums are added in warp order (a
// fixed order: deterministic).
__global__ void __launch_bounds__(256) k_colsum(const float *d, int M, int N, float *out) {
    __shared__ float part[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, c = blockIdx.x * 32 + lane;
    float s = 0.f;
    if (c < N)
        for (int r = w; r < M; r += 8) s += d[(size_t)r * N + c];
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && c < N) {
        float t = part[0][lane];
        for (int q = 1; q < 8; q++) t += part[q][lane];
        out[c] = t;
    }
}

struct AdamArgs {
    float *w, *m, *v;
    const float *g;
    bf16 *w16, *w16t;    // weights as [rows][cols] and [cols][rows] BF16 (null for biases)
    int n, rows, cols;
    float lr0, beta1, beta2, eps;
    long long total_steps;
    const long long *step;  // steps done before this update
};

// Adam with bias correction; learning rate lr0 * 0.5 (1 + cos(pi s / S)).
__global__ void k_adam(AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const long long s = *a.step + 1;
    const float frac = (float)min(1.0, (double)(s - 1) / (double)max(1LL, a.total_steps));
    const float lr = a.lr0 * 0.5f * (1.0f + cospif(frac));
    const float g = a.g[i];
    const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    const float mh = m / (1.0f - powf(a.beta1, (float)s));
    const float vh = v / (1.0f - powf(a.beta2, (float)s));
    const float w = a.w[i] - lr * mh / (sqrtf(vh) + a.eps);
    a.w[i] = w;
    if (a.w16) {
        const bf16 b = __float2bfloat16_rn(w);
        a.w16[i] = b;
        const int r = i / a.cols, c = i - r * a.cols;
        a.w16t[(size_t)c * a.rows + r] = b;
    }
}

__global__ void k_step_inc(long long *step) { *step += 1; }

// Batch of B rows from the resident set: row q of the batch is sample
// perm[(step * B + q) mod n]; X as BF16 [B][kin] and its transpose, Y FP32.
__global__ void k_gather(const bf16 *X, const float *Y, const int *perm, long long n, const long long *step, int B,
                         int kin, int nout, bf16 *xb, bf16 *xbt, float *yb) {
    const int q = blockIdx.x;
    const long long idx = perm[((*step) * B + q) % n];
    for (int c = threadIdx.x; c < kin; c += blockDim.x) {
        const bf16 v = X[idx * kin + c];
        xb[(size_t)q * kin + c] = v;
        xbt[(size_t)c * B + q] = v;
    }
    for (int c = threadIdx.x; c < nout; c += blockDim.x) yb[(size_t)q * nout + c] = Y[idx * nout + c];
}

__global__ void k_f2bf(const float *in, bf16 *out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

// Rows of X [n][n_in] FP32 into BF16 [n][kin] (zero padding).
__global__ void k_pack_x(const float *in, int n_in, bf16 *out, int kin, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kin) return;
    const size_t r = i / kin;
    const int c = (int)(i - r * kin);
    out[i] = __float2bfloat16_rn(c < n_in ? in[r * n_in + c] : 0.f);
}

}  // namespace

extern unsigned long long rfb_launch_count(void);

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Layer {
    int in, out;             // out x in weights
    float *w = nullptr, *b = nullptr, *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;
    float *gw = nullptr, *gb = nullptr;
    bf16 *w16 = nullptr, *w16t = nullptr;
};

struct fdtd_b200_mlp {
    int n_in, kin, width, depth, n_out;
    std::vector<Layer> L;
    int bmax = 0;                          // batch buffers sized for this many rows
    std::vector<float *> pre;              // per hidden layer [B][width]
    std::vector<bf16 *> act, actt;         // per layer input: act[0] = x, act[l] = GELU(pre[l-1]); transposes
    float *out = nullptr, *y = nullptr, *d32 = nullptr, *partial = nullptr;
    bf16 *d16 = nullptr, *d16t = nullptr;
    float *dz32 = nullptr;
    bf16 *dz16 = nullptr, *dz16t = nullptr;
    // resident training set
    bf16 *X = nullptr;
    float *Y = nullptr;
    int *perm = nullptr;
    size_t n_data = 0;
    long long *step = nullptr;
    cudaStream_t st = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_b = 0;
    AdamArgs adam_cfg{};
    unsigned long long launches = 0;
    // tensor-core products: enabled (the shared memory attribute was set),
    // their launches, and the device flag a timed-out wait sets
    int tc = 0;
    unsigned long long tc_launches = 0;
    int *d_err = nullptr;
};

typedef struct fdtd_b200_mlp fdtd_b200_mlp_t;

#define MCK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            rfb_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return -1;                                                                        \
        }                                                                                     \
    } while (0)

static void mlp_free_batch(fdtd_b200_mlp *m) {
    for (auto p : m->pre) cudaFree(p);
    for (auto p : m->act) cudaFree(p);
    for (auto p : m->actt) cudaFree(p);
    m->pre.clear();
    m->act.clear();
    m->actt.clear();
    cudaFree(m->out); cudaFree(m->y); cudaFree(m->d32); cudaFree(m->partial);
    cudaFree(m->d16); cudaFree(m->d16t); cudaFree(m->dz32); cudaFree(m->dz16); cudaFree(m->dz16t);
    m->out = m->y = m->d32 = m->partial = m->dz32 = nullptr;
    m->d16 = m->d16t = m->dz16 = m->dz16t = nullptr;
    if (m->graph) cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
    m->bmax = 0;
}

static int mlp_batch_buffers(fdtd_b200_mlp *m, int B) {
    if (B <= m->bmax) return 0;
    mlp_free_batch(m);
    const int nl = (int)m->L.size();
    m->pre.assign(nl - 1, nullptr);
    m->act.assign(nl, nullptr);
    m->actt.assign(nl, nullptr);
    for (int l = 0; l < nl; l++) {
        MCK(cudaMalloc(&m->act[l], (size_t)B * m->L[l].in * sizeof(bf16)));
        MCK(cudaMalloc(&m->actt[l], (size_t)B * m->L[l].in * sizeof(bf16)));
        if (l < nl - 1) MCK(cudaMalloc(&m->pre[l], (size_t)B * m->L[l].out * sizeof(float)));
    }
    // the two gradient buffer sets alternate between output-sized and
    // hidden-sized gradients: both hold the larger
    const size_t no = (size_t)B * m->n_out, nw = (size_t)B * std::max(m->width, m->n_out);
    MCK(cudaMalloc(&m->out, no * sizeof(float)));
    MCK(cudaMalloc(&m->y, no * sizeof(float)));
    MCK(cudaMalloc(&m->d32, nw * sizeof(float)));
    MCK(cudaMalloc(&m->d16, nw * sizeof(bf16)));
    MCK(cudaMalloc(&m->d16t, nw * sizeof(bf16)));
    MCK(cudaMalloc(&m->partial, (no / 256 + 1) * sizeof(float)));
    MCK(cudaMalloc(&m->dz32, nw * sizeof(float)));
    MCK(cudaMalloc(&m->dz16, nw * sizeof(bf16)));
    MCK(cudaMalloc(&m->dz16t, nw * sizeof(bf16)));
    m->bmax = B;
    return 0;
}

// The network's products: k_gemm_nt (64 x 64 tiles, mma.sync), or with
// RFSYN_FDTD_MLP_GEMM=tcgen05 k_gemm_tc where the shapes fit its tiles (M a
// multiple of 128, N of 32, K of 64 -- every training-step product of the
// surrogate does).
template <int EPI>
static void gemm(fdtd_b200_mlp *m, const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, Epi epi) {
    if (m->tc && M > 0 && N > 0 && K > 0 && M % tc::BM == 0 && N % 32 == 0 && K % tc::BK == 0 && lda % 8 == 0 &&
        ldb % 8 == 0) {
        dim3 grid(N / 32, M / tc::BM);
        k_gemm_tc<EPI, 32><<<grid, tc::THREADS, tc::Shape<32>::SMEM, m->st>>>(A, lda, B, ldb, M, N, K, epi,
                                                                            m->d_err);
        m->tc_launches++;
    } else {
        dim3 grid(N / GT, M / GT);
        k_gemm_nt<EPI><<<grid, 128, 0, m->st>>>(A, lda, B, ldb, M, N, K, epi);
    }
    m->launches++;
}

// The tensor-core products need more than 48 KB of shared memory.
template <int BN>
static bool tc_attrs() {
    const int sm = tc::Shape<BN>::SMEM;
    return cudaFuncSetAttribute(k_gemm_tc<EPI_HIDDEN, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_gemm_tc<EPI_OUT, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_gemm_tc<EPI_BWD_GELU, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_gemm_tc<EPI_F32, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
               cudaSuccess;
}

// A timed-out wait in a tensor-core product, reported once per call.
static int mlp_check_err(fdtd_b200_mlp *m) {
    int e = 0;
    if (cudaMemcpy(&e, m->d_err, sizeof e, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rfb_set_error("surrogate: reading the error flag failed");
        return -1;
    }
    if (e) {
        cudaMemset(m->d_err, 0, sizeof(int));
        rfb_set_error("surrogate: a tensor-core product's wait timed out");
        return -1;
    }
    return 0;
}

// Forward pass of B rows whose input is already in act[0].
static void mlp_forward(fdtd_b200_mlp *m, int B) {
    const int nl = (int)m->L.size();
    for (int l = 0; l < nl; l++) {
        const Layer &ly = m->L[l];
        Epi e{};
        e.bias = ly.b;
        if (l < nl - 1) {
            e.f32 = m->pre[l];
            e.b16 = m->act[l + 1];
            gemm<EPI_HIDDEN>(m, m->act[l], ly.in, ly.w16, ly.in, B, ly.out, ly.in, e);
        } else {
            e.f32 = m->out;
            gemm<EPI_OUT>(m, m->act[l], ly.in, ly.w16, ly.in, B, ly.out, ly.in, e);
        }
    }
}

// Transposes of the hidden activations (B x width, BF16) for the weight
// gradients: written by a small kernel.
__global__ void k_transpose_bf16(const bf16 *in, int rows, int cols, bf16 *out) {
    __shared__ bf16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        if (r0 + y < rows && c0 + threadIdx.x < cols) tile[y][threadIdx.x] = in[(size_t)(r0 + y) * cols + c0 + threadIdx.x];
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        if (c0 + y < cols && r0 + threadIdx.x < rows) out[(size_t)(c0 + y) * rows + r0 + threadIdx.x] = tile[threadIdx.x][y];
}

// Backward pass after the forward (dOut already in d32 / d16 / d16t): weight
// and bias gradients of every layer.  The gradient flowing backwards
// alternates between the (d*) and (dz*) buffer sets.
static void mlp_backward(fdtd_b200_mlp *m, int B) {
    const int nl = (int)m->L.size();
    // transposes of the layer inputs (act[0]^T is written by the gather)
    for (int l = 1; l < nl; l++) {
        dim3 grid((m->L[l].in + 31) / 32, (B + 31) / 32);
        k_transpose_bf16<<<grid, dim3(32, 8), 0, m->st>>>(m->act[l], B, m->L[l].in, m->actt[l]);
        m->launches++;
    }
    float *g32[2] = {m->d32, m->dz32};
    bf16 *g16[2] = {m->d16, m->dz16}, *g16t[2] = {m->d16t, m->dz16t};
    int cur = 0;
    for (int l = nl - 1; l >= 0; l--) {
        const Layer &ly = m->L[l];
        // dW = dZ^T . X: [out][in] = (dZ^T [out][B]) . (X^T [in][B])^T
        Epi e{};
        e.f32 = ly.gw;
        gemm<EPI_F32>(m, g16t[cur], B, m->actt[l], B, ly.out, ly.in, B, e);
        k_colsum<<<(ly.out + 31) / 32, 256, 0, m->st>>>(g32[cur], B, ly.out, ly.gb);
        m->launches++;
        if (l > 0) {
            // dX = dZ . W = dZ [B][out] . (W^T [in][out])^T, times GELU' of the
            // previous layer's pre-activation
            Epi eb{};
            eb.f32 = g32[cur ^ 1];
            eb.b16 = g16[cur ^ 1];
            eb.b16t = g16t[cur ^ 1];
            eb.pre = m->pre[l - 1];
            gemm<EPI_BWD_GELU>(m, g16[cur], ly.out, ly.w16t, ly.out, B, ly.in, ly.out, eb);
            cur ^= 1;
        }
    }
}

static void mlp_loss(fdtd_b200_mlp *m, int B) {
    const int n = B * m->n_out;
    k_mse<<<(n + 255) / 256, 256, 0, m->st>>>(m->out, m->y, B, m->n_out, m->d32, m->d16, m->d16t, m->partial);
    m->launches++;
}

static void mlp_adam(fdtd_b200_mlp *m) {
    for (Layer &ly : m->L) {
        AdamArgs a = m->adam_cfg;
        a.w = ly.w; a.m = ly.mw; a.v = ly.vw; a.g = ly.gw;
        a.w16 = ly.w16; a.w16t = ly.w16t;
        a.n = ly.out * ly.in; a.rows = ly.out; a.cols = ly.in;
        k_adam<<<(a.n + 255) / 256, 256, 0, m->st>>>(a);
        AdamArgs b = m->adam_cfg;
        b.w = ly.b; b.m = ly.mb; b.v = ly.vb; b.g = ly.gb;
        b.w16 = nullptr; b.w16t = nullptr;
        b.n = ly.out; b.rows = 1; b.cols = ly.out;
        k_adam<<<(b.n + 255) / 256, 256, 0, m->st>>>(b);
        m->launches += 2;
    }
    k_step_inc<<<1, 1, 0, m->st>>>(m->step);
    m->launches++;
}

// BF16 copies (and transposes) of the FP32 master weights.
static int mlp_sync_bf16(fdtd_b200_mlp *m) {
    for (Layer &ly : m->L) {
        const size_t n = (size_t)ly.out * ly.in;
        k_f2bf<<<(unsigned)((n + 255) / 256), 256, 0, m->st>>>(ly.w, ly.w16, n);
        dim3 grid((ly.in + 31) / 32, (ly.out + 31) / 32);
        k_transpose_bf16<<<grid, dim3(32, 8), 0, m->st>>>(ly.w16, ly.out, ly.in, ly.w16t);
        m->launches += 2;
    }
    MCK(cudaGetLastError());
    return 0;
}

extern "C" void fdtd_b200_mlp_destroy(fdtd_b200_mlp_t *m) {
    if (!m) return;
    if (m->st) cudaStreamSynchronize(m->st);
    mlp_free_batch(m);
    for (Layer &ly : m->L) {
        cudaFree(ly.w); cudaFree(ly.b); cudaFree(ly.mw); cudaFree(ly.vw); cudaFree(ly.mb); cudaFree(ly.vb);
        cudaFree(ly.gw); cudaFree(ly.gb); cudaFree(ly.w16); cudaFree(ly.w16t);
    }
    cudaFree(m->X); cudaFree(m->Y); cudaFree(m->perm); cudaFree(m->step); cudaFree(m->d_err);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
}

// splitmix64: the initial weights' random stream
static uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

extern "C" fdtd_b200_mlp_t *fdtd_b200_mlp_create(int n_in, int width, int depth, int n_out, uint64_t seed) {
    if (n_in < 1 || width < 64 || width % 64 || n_out < 64 || n_out % 64 || depth < 1 || n_in > 4096) {
        rfb_set_error("mlp: n_in >= 1, width and n_out multiples of 64, depth >= 1");
        return nullptr;
    }
    fdtd_b200_mlp *m = new fdtd_b200_mlp();
    m->n_in = n_in;
    m->kin = (n_in + 63) / 64 * 64;
    m->width = width;
    m->depth = depth;
    m->n_out = n_out;
    for (int l = 0; l <= depth; l++) {
        Layer ly;
        ly.in = l == 0 ? m->kin : width;
        ly.out = l == depth ? n_out : width;
        m->L.push_back(ly);
    }
    uint64_t rs = seed;
    auto fail = [&]() -> fdtd_b200_mlp_t * {
        fdtd_b200_mlp_destroy(m);
        return nullptr;
    };
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess) return fail();
    for (int l = 0; l <= depth; l++) {
        Layer &ly = m->L[l];
        const size_t nw = (size_t)ly.out * ly.in;
        float **f32s[] = {&ly.w, &ly.mw, &ly.vw, &ly.gw};
        for (float **p : f32s)
            if (cudaMalloc(p, nw * sizeof(float)) != cudaSuccess) return fail();
        float **b32s[] = {&ly.b, &ly.mb, &ly.vb, &ly.gb};
        for (float **p : b32s)
            if (cudaMalloc(p, ly.out * sizeof(float)) != cudaSuccess) return fail();
        if (cudaMalloc(&ly.w16, nw * sizeof(bf16)) != cudaSuccess) return fail();
        if (cudaMalloc(&ly.w16t, nw * sizeof(bf16)) != cudaSuccess) return fail();
        // uniform(-lim, lim), lim = sqrt(6 / fan_in) (He); only the real inputs
        // of the first layer count, padded columns start at zero
        const int fan_in = l == 0 ? n_in : ly.in;
        const double lim = sqrt(6.0 / fan_in) * (l == depth ? 0.5 : 1.0);
        std::vector<float> w(nw, 0.f), z(nw, 0.f), zb(ly.out, 0.f);
        for (int r = 0; r < ly.out; r++)
            for (int c = 0; c < ly.in; c++) {
                const double u = (double)(splitmix(rs) >> 11) * (1.0 / 9007199254740992.0);
                w[(size_t)r * ly.in + c] = (l == 0 && c >= n_in) ? 0.f : (float)((2.0 * u - 1.0) * lim);
            }
        if (cudaMemcpy(ly.w, w.data(), nw * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
        if (cudaMemcpy(ly.mw, z.data(), nw * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
        if (cudaMemcpy(ly.vw, z.data(), nw * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
        if (cudaMemcpy(ly.b, zb.data(), ly.out * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
        if (cudaMemcpy(ly.mb, zb.data(), ly.out * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
        if (cudaMemcpy(ly.vb, zb.data(), ly.out * 4, cudaMemcpyHostToDevice) != cudaSuccess) return fail();
    }
    if (cudaMalloc(&m->step, sizeof(long long)) != cudaSuccess) return fail();
    if (cudaMemset(m->step, 0, sizeof(long long)) != cudaSuccess) return fail();
    if (cudaMalloc(&m->d_err, sizeof(int)) != cudaSuccess) return fail();
    if (cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess) return fail();
    {
        // RFSYN_FDTD_MLP_GEMM=tcgen05 puts the products whose shapes fit on
        // k_gemm_tc; by default every product runs on k_gemm_nt, which is
        // faster on this network's products at every batch measured (see
        // k_gemm_tc)
        const char *v = getenv("RFSYN_FDTD_MLP_GEMM");
        const bool want = v && !strcmp(v, "tcgen05");
        m->tc = want && tc_attrs<32>();
        if (want && !m->tc) {
            rfb_set_error("mlp: cannot configure the tensor-core products' shared memory");
            return fail();
        }
    }
    if (mlp_sync_bf16(m) != 0) return fail();
    if (cudaStreamSynchronize(m->st) != cudaSuccess) return fail();
    return m;
}

extern "C" size_t fdtd_b200_mlp_n_params(const fdtd_b200_mlp_t *m) {
    size_t n = 0;
    for (const Layer &ly : m->L) n += (size_t)ly.out * ly.in + ly.out;
    return n;
}

// Parameters in layer order: W (out x in, row-major, first layer with its
// zero-padded input columns), then b.
extern "C" int fdtd_b200_mlp_get_params(fdtd_b200_mlp_t *m, float *out) {
    MCK(cudaStreamSynchronize(m->st));
    size_t o = 0;
    for (const Layer &ly : m->L) {
        const size_t nw = (size_t)ly.out * ly.in;
        MCK(cudaMemcpy(out + o, ly.w, nw * 4, cudaMemcpyDeviceToHost));
        o += nw;
        MCK(cudaMemcpy(out + o, ly.b, ly.out * 4, cudaMemcpyDeviceToHost));
        o += ly.out;
    }
    return 0;
}

extern "C" int fdtd_b200_mlp_set_params(fdtd_b200_mlp_t *m, const float *in) {
    MCK(cudaStreamSynchronize(m->st));
    size_t o = 0;
    for (const Layer &ly : m->L) {
        const size_t nw = (size_t)ly.out * ly.in;
        MCK(cudaMemcpy(ly.w, in + o, nw * 4, cudaMemcpyHostToDevice));
        o += nw;
        MCK(cudaMemcpy(ly.b, in + o, ly.out * 4, cudaMemcpyHostToDevice));
        o += ly.out;
    }
    return mlp_sync_bf16(m);
}

// Reads the gradients of the last backward pass in parameter layout.
static int mlp_read_grads(fdtd_b200_mlp *m, float *out) {
    MCK(cudaStreamSynchronize(m->st));
    size_t o = 0;
    for (const Layer &ly : m->L) {
        const size_t nw = (size_t)ly.out * ly.in;
        MCK(cudaMemcpy(out + o, ly.gw, nw * 4, cudaMemcpyDeviceToHost));
        o += nw;
        MCK(cudaMemcpy(out + o, ly.gb, ly.out * 4, cudaMemcpyDeviceToHost));
        o += ly.out;
    }
    return 0;
}

static int mlp_upload_x(fdtd_b200_mlp *m, const float *X, size_t n, bf16 *dst) {
    float *tmp = nullptr;
    MCK(cudaMalloc(&tmp, n * m->n_in * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(tmp, X, n * m->n_in * sizeof(float), cudaMemcpyHostToDevice, m->st);
    if (e == cudaSuccess) {
        const size_t tot = n * m->kin;
        k_pack_x<<<(unsigned)((tot + 255) / 256), 256, 0, m->st>>>(tmp, m->n_in, dst, m->kin, n);
        m->launches++;
        e = cudaStreamSynchronize(m->st);
    }
    cudaFree(tmp);
    if (e != cudaSuccess) {
        rfb_set_error("mlp: input upload failed: %s", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

// One forward + backward pass on the given batch (B a multiple of 64):
// loss = mean squared error, grads in parameter layout.
extern "C" int fdtd_b200_mlp_grad(fdtd_b200_mlp_t *m, const float *X, const float *Y, int B, double *loss,
                                  float *grads) {
    if (B < 64 || B % 64) {
        rfb_set_error("mlp: batch must be a positive multiple of 64");
        return -1;
    }
    if (mlp_batch_buffers(m, B) != 0) return -1;
    if (mlp_upload_x(m, X, B, m->act[0]) != 0) return -1;
    dim3 grid((m->kin + 31) / 32, (B + 31) / 32);
    k_transpose_bf16<<<grid, dim3(32, 8), 0, m->st>>>(m->act[0], B, m->kin, m->actt[0]);
    MCK(cudaMemcpyAsync(m->y, Y, (size_t)B * m->n_out * 4, cudaMemcpyHostToDevice, m->st));
    mlp_forward(m, B);
    mlp_loss(m, B);
    mlp_backward(m, B);
    MCK(cudaGetLastError());
    std::vector<float> part((size_t)B * m->n_out / 256 + 1);
    const int nb = (B * m->n_out + 255) / 256;
    MCK(cudaMemcpyAsync(part.data(), m->partial, nb * 4, cudaMemcpyDeviceToHost, m->st));
    if (mlp_read_grads(m, grads) != 0) return -1;
    if (mlp_check_err(m) != 0) return -1;
    double se = 0;
    for (int q = 0; q < nb; q++) se += part[q];
    if (loss) *loss = se / ((double)B * m->n_out);
    return 0;
}

extern "C" int fdtd_b200_mlp_set_data(fdtd_b200_mlp_t *m, const float *X, const float *Y, size_t n) {
    MCK(cudaStreamSynchronize(m->st));
    cudaFree(m->X);
    cudaFree(m->Y);
    cudaFree(m->perm);
    m->X = nullptr;
    m->Y = nullptr;
    m->perm = nullptr;
    m->n_data = 0;
    if (n == 0) return 0;
    MCK(cudaMalloc(&m->X, n * m->kin * sizeof(bf16)));
    MCK(cudaMalloc(&m->Y, n * m->n_out * sizeof(float)));
    MCK(cudaMalloc(&m->perm, n * sizeof(int)));
    if (mlp_upload_x(m, X, n, m->X) != 0) return -1;
    MCK(cudaMemcpy(m->Y, Y, n * m->n_out * sizeof(float), cudaMemcpyHostToDevice));
    m->n_data = n;
    if (m->graph) cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
    return 0;
}

static void mlp_train_step(fdtd_b200_mlp *m, int B) {
    k_gather<<<B, 128, 0, m->st>>>(m->X, m->Y, m->perm, (long long)m->n_data, m->step, B, m->kin, m->n_out,
                                   m->act[0], m->actt[0], m->y);
    m->launches++;
    mlp_forward(m, B);
    mlp_loss(m, B);
    mlp_backward(m, B);
    mlp_adam(m);
}

// `steps` Adam steps of batch B over the resident data set, sampled through a
// permutation that is reshuffled (seeded) every pass over the data; the
// learning rate follows lr0 * 0.5 (1 + cos(pi s / steps)).  Each step is a
// CUDA graph replay.  *final_loss: mean squared error of the last batch.
extern "C" int fdtd_b200_mlp_train(fdtd_b200_mlp_t *m, size_t steps, int B, double lr, double beta1, double beta2,
                                   double eps, uint64_t shuffle_seed, double *final_loss) {
    if (!m->n_data) {
        rfb_set_error("mlp: no training data (fdtd_b200_mlp_set_data)");
        return -1;
    }
    if (B < 64 || B % 64) {
        rfb_set_error("mlp: batch must be a positive multiple of 64");
        return -1;
    }
    if (mlp_batch_buffers(m, B) != 0) return -1;
    MCK(cudaMemsetAsync(m->step, 0, sizeof(long long), m->st));
    m->adam_cfg.lr0 = (float)lr;
    m->adam_cfg.beta1 = (float)beta1;
    m->adam_cfg.beta2 = (float)beta2;
    m->adam_cfg.eps = (float)eps;
    m->adam_cfg.total_steps = (long long)steps;
    m->adam_cfg.step = m->step;
    // first and second moments restart
    for (Layer &ly : m->L) {
        MCK(cudaMemsetAsync(ly.mw, 0, (size_t)ly.out * ly.in * 4, m->st));
        MCK(cudaMemsetAsync(ly.vw, 0, (size_t)ly.out * ly.in * 4, m->st));
        MCK(cudaMemsetAsync(ly.mb, 0, ly.out * 4, m->st));
        MCK(cudaMemsetAsync(ly.vb, 0, ly.out * 4, m->st));
    }
    if (m->graph && m->graph_b != B) {
        cudaGraphExecDestroy(m->graph);
        m->graph = nullptr;
    }
    if (m->graph) {
        // the captured Adam arguments hold the old schedule: capture again
        cudaGraphExecDestroy(m->graph);
        m->graph = nullptr;
    }
    {
        cudaGraph_t g = nullptr;
        MCK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
        mlp_train_step(m, B);
        MCK(cudaStreamEndCapture(m->st, &g));
        const cudaError_t e = cudaGraphInstantiate(&m->graph, g, 0);
        cudaGraphDestroy(g);
        MCK(e);
        m->graph_b = B;
    }
    const size_t per_pass = std::max<size_t>(1, m->n_data / B);
    std::vector<int> perm(m->n_data);
    uint64_t rs = shuffle_seed;
    size_t done = 0;
    while (done < steps) {
        // permutation of this pass (Fisher-Yates on splitmix64)
        for (size_t q = 0; q < m->n_data; q++) perm[q] = (int)q;
        for (size_t q = m->n_data - 1; q > 0; q--) std::swap(perm[q], perm[splitmix(rs) % (q + 1)]);
        MCK(cudaMemcpyAsync(m->perm, perm.data(), m->n_data * sizeof(int), cudaMemcpyHostToDevice, m->st));
        const size_t run = std::min(per_pass, steps - done);
        for (size_t s = 0; s < run; s++) {
            MCK(cudaGraphLaunch(m->graph, m->st));
            m->launches += 0;
        }
        // the permutation buffer is rewritten for the next pass only after
        // this pass's steps have read it
        MCK(cudaStreamSynchronize(m->st));
        done += run;
    }
    if (final_loss) {
        const int nb = (B * m->n_out + 255) / 256;
        std::vector<float> part(nb);
        MCK(cudaMemcpy(part.data(), m->partial, nb * 4, cudaMemcpyDeviceToHost));
        double se = 0;
        for (float v : part) se += v;
        *final_loss = se / ((double)B * m->n_out);
    }
    return mlp_check_err(m);
}

// Network outputs of n inputs (any n; evaluated in batches of up to 1024).
extern "C" int fdtd_b200_mlp_predict(fdtd_b200_mlp_t *m, const float *X, size_t n, float *Y) {
    const int B = 1024;
    if (mlp_batch_buffers(m, B) != 0) return -1;
    std::vector<float> xb((size_t)B * m->n_in, 0.f);
    for (size_t r0 = 0; r0 < n; r0 += B) {
        const size_t rows = std::min<size_t>(B, n - r0);
        std::fill(xb.begin(), xb.end(), 0.f);
        memcpy(xb.data(), X + r0 * m->n_in, rows * m->n_in * sizeof(float));
        // rows padded to the tensor-core tile height (zero rows)
        const int Bp = (int)((rows + tc::BM - 1) / tc::BM * tc::BM);
        if (mlp_upload_x(m, xb.data(), Bp, m->act[0]) != 0) return -1;
        mlp_forward(m, Bp);
        MCK(cudaGetLastError());
        MCK(cudaMemcpyAsync(Y + r0 * m->n_out, m->out, rows * m->n_out * sizeof(float), cudaMemcpyDeviceToHost,
                            m->st));
        MCK(cudaStreamSynchronize(m->st));
    }
    return mlp_check_err(m);
}

extern "C" unsigned long long fdtd_b200_mlp_launch_count(const fdtd_b200_mlp_t *m) { return m->launches; }

extern "C" unsigned long long fdtd_b200_mlp_tensor_core_launches(const fdtd_b200_mlp_t *m) { return m->tc_launches; }
