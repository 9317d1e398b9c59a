// tma.cuh -- interior sweep fed by the Tensor Memory Accelerator.
//
// Same march and arithmetic as k_sweep_interior (fused.cuh), but each plane
// arrives as whole boxes: one elected thread issues, per plane, one tiled
// cp.async.bulk.tensor load per field component (E: rows j0-1 .. j0+TJ,
// columns k0-4 .. k0+35; H: rows j0-1 .. j0+TJ-1, columns k0-4 .. k0+31) and
// one for the material codes, all completing on the stage's mbarrier.  The
// boxes start at column k0-4 so that the first element of every box row is
// 16-byte aligned (k0 is a multiple of 32); their out-of-range rows are
// zero-filled by the hardware.  Loads never use cluster multicast.  Work
// items whose halo would wrap around a periodic axis are never given to this
// kernel (the plan builder keeps them on the edge sweep).
//
// Compared with the per-thread cp.async ring this removes ~14 copy
// instructions per thread per plane and their address arithmetic; the SM's
// issue slots go to the stencil itself.
//
// Every mbarrier wait is bounded (about one second of SM clock).  On timeout
// the CTA records an error code in *err, waits (bounded) for its own copies
// still in flight and returns, so a stalled copy can never hang the GPU.
#pragma once
#include <cuda.h>

#include "fused.cuh"

namespace rfb {

// One tensor map per input array of one buffer parity, for the wide (TJ x
// 32) tiles and for the narrow (2 TJ x 16) tiles of the work-queue sweep.
struct TmaMaps {
    CUtensorMap e[3], h[3], code;
    CUtensorMap en[3], hn[3], coden;
    CUtensorMap e2[3], h2[3], code2;  // interior tiles of 2 TJ rows x 32 columns
};

constexpr int TMA_EW = 40;  // E box width (k0-4 .. k0+35)
constexpr int TMA_HW = 36;  // H box width (k0-4 .. k0+31)

__host__ __device__ constexpr size_t round128(size_t b) { return (b + 127) / 128 * 128; }

// Shared-memory layout: NS stages (3 E boxes, 3 H boxes, codes), then the NS
// mbarriers, the H tile of the current plane and the (Ca, Cb) table.
template <typename T, int TJ, int NS>
struct TmaLayout {
    static constexpr unsigned ebytes = sizeof(T) * TMA_EW * (TJ + 2);
    static constexpr unsigned hbytes = sizeof(T) * TMA_HW * (TJ + 1);
    static constexpr unsigned cbytes = 32 * TJ;
    static constexpr size_t ebox = round128(ebytes);
    static constexpr size_t hbox = round128(hbytes);
    static constexpr size_t cbox = round128(cbytes);
    static constexpr size_t stage = 3 * ebox + 3 * hbox + cbox;
    static constexpr size_t bars = NS * stage;
    static constexpr size_t sh = bars + round128(8 * NS);
    static constexpr size_t tab = sh + round128(sizeof(T) * 3 * (TJ + 1) * 33);
    static constexpr size_t total = tab + sizeof(T) * 512;
};

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity: false
// after `limit` SM cycles without it (every sweep waits ~2e9 cycles, about a
// second, before it reports a stalled copy).
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, unsigned parity, long long limit) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    return mbar_wait_for(bar, parity, 2000000000LL);
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB)
    k_sweep_interior_tma(Args<T> a, const SweepItem *items, const __grid_constant__ TmaMaps maps, int *err) {
    static_assert(NS >= 3, "the ring must hold the current, the next and one prefetched plane");
    using L = TmaLayout<T, TJ, NS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + L::bars);
    T(*sH)[TJ + 1][33] = reinterpret_cast<T(*)[TJ + 1][33]>(smem_raw + L::sh);
    T *s_tab = reinterpret_cast<T *>(smem_raw + L::tab);
    auto E = [&](int s, int c) { return reinterpret_cast<T(*)[TMA_EW]>(smem_raw + s * L::stage + c * L::ebox); };
    auto H = [&](int s, int c) {
        return reinterpret_cast<T(*)[TMA_HW]>(smem_raw + s * L::stage + 3 * L::ebox + c * L::hbox);
    };
    auto CODE = [&](int s) {
        return reinterpret_cast<uint8_t(*)[32]>(smem_raw + s * L::stage + 3 * L::ebox + 3 * L::hbox);
    };

    const SweepItem it = items[blockIdx.x];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const bool px = a.per & 1u;
    const int r = ty + 1, q = tx + 4;  // stage coordinates of the own cell
    const bool with_codes = a.codes != nullptr;
    const unsigned tx_bytes = 3 * L::ebytes + 3 * L::hbytes + (with_codes ? L::cbytes : 0u);

    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    for (int t = tid; t < 256; t += 32 * TJ) {
        s_tab[t] = a.tca[t];
        s_tab[256 + t] = a.tcb[t];
    }
    __syncthreads();

    // uniform bookkeeping: phase bit s = parity of slot s's next completion,
    // pending bit s = slot s has a load in flight that nobody waited for
    unsigned phase = 0, pending = 0;
    bool failed = false;
    auto issue = [&](int s, int p) {
        if (tid == 0) {
            mbar_expect_tx(&bars[s], tx_bytes);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                tma_load_3d(E(s, c), &maps.e[c], k0 - 4, j0 - 1, p, &bars[s]);
                tma_load_3d(H(s, c), &maps.h[c], k0 - 4, j0 - 1, p, &bars[s]);
            }
            if (with_codes) tma_load_3d(CODE(s), &maps.code, k0, j0, p, &bars[s]);
        }
        pending |= 1u << s;
    };
    auto wait_slot = [&](int s) {
        if (!mbar_wait(&bars[s], (phase >> s) & 1u)) failed = true;
        phase ^= 1u << s;
        pending &= ~(1u << s);
    };

    const T cbh = a.cbh;
    const int pprev = ib > 0 ? ib - 1 : a.nx - 1;  // ib == 0 only on a periodic x axis
    int pf = ib;
    issue(NS - 1, pprev);
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) issue(s, pf);
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    // H(pprev) needs plane pprev (slot NS-1) and plane ib (slot 0)
    wait_slot(NS - 1);
    wait_slot(0);
    if (__syncthreads_or(failed)) goto bail;
    {
        // unstretched H of component c at stage position (rr, qq) of the
        // plane in slot sc (the plane after it is in slot sn)
        auto hval = [&](int c, int sc, int sn, int rr, int qq) -> T {
            if (c == 0)
                return upd_h(H(sc, 0)[rr][qq], cbh, xs(xs(E(sc, 2)[rr + 1][qq], E(sc, 2)[rr][qq]),
                                                      xs(E(sc, 1)[rr][qq + 1], E(sc, 1)[rr][qq])));
            if (c == 1)
                return upd_h(H(sc, 1)[rr][qq], cbh, xs(xs(E(sc, 0)[rr][qq + 1], E(sc, 0)[rr][qq]),
                                                      xs(E(sn, 2)[rr][qq], E(sc, 2)[rr][qq])));
            return upd_h(H(sc, 2)[rr][qq], cbh, xs(xs(E(sn, 1)[rr][qq], E(sc, 1)[rr][qq]),
                                                  xs(E(sc, 0)[rr + 1][qq], E(sc, 0)[rr][qq])));
        };
        T prevHy = hval(1, NS - 1, 0, r, q);
        T prevHz = hval(2, NS - 1, 0, r, q);
        __syncthreads();  // slot NS-1 may now be refilled

        int sc = 0;
        for (int i = ib; i < ie; i++) {
            const int sn = sc == NS - 1 ? 0 : sc + 1;
            const int sf = sc == 0 ? NS - 1 : sc - 1;  // held plane i-1, read by nobody any more
            if (pf >= 0 && i + NS - 1 <= ie) issue(sf, pf);
            if (pf >= 0 && i + NS - 1 <= ie) pf = plane_after(pf, a.nx, px);
            wait_slot(sn);  // plane i+1 (plane i landed before the previous barrier)
            if (__syncthreads_or(failed)) goto bail;
            const T e0 = E(sc, 0)[r][q], e1 = E(sc, 1)[r][q], e2 = E(sc, 2)[r][q];
            const int code = with_codes ? (int)CODE(sc)[ty][tx] : 0;
            const long long c = (long long)i * a.plane + (long long)(j0 + ty) * a.pitch + (k0 + tx);
            const T hx = hval(0, sc, sn, r, q);
            const T hy = hval(1, sc, sn, r, q);
            const T hz = hval(2, sc, sn, r, q);
            a.Ho[0][c] = hx;
            a.Ho[1][c] = hy;
            a.Ho[2][c] = hz;
            const int qs = tx + 1;  // sH column of the own cell
            sH[0][r][qs] = hx;
            sH[1][r][qs] = hy;
            sH[2][r][qs] = hz;
            if (ty == 0) {
                sH[0][0][qs] = hval(0, sc, sn, 0, q);
                sH[2][0][qs] = hval(2, sc, sn, 0, q);
            } else if (ty == 1 && tx < TJ) {
                sH[0][tx + 1][0] = hval(0, sc, sn, tx + 1, 3);
                sH[1][tx + 1][0] = hval(1, sc, sn, tx + 1, 3);
            }
            __syncthreads();
            if (!with_codes || code != LIST_CODE) {
                const T ca = s_tab[code], cb = s_tab[256 + code];
                a.Eo[0][c] = upd_e(ca, e0, cb, xs(xs(sH[2][r][qs], sH[2][r - 1][qs]), xs(sH[1][r][qs], sH[1][r][qs - 1])));
                a.Eo[1][c] = upd_e(ca, e1, cb, xs(xs(sH[0][r][qs], sH[0][r][qs - 1]), xs(hz, prevHz)));
                a.Eo[2][c] = upd_e(ca, e2, cb, xs(xs(hy, prevHy), xs(sH[0][r][qs], sH[0][r - 1][qs])));
            }
            prevHy = hy;
            prevHz = hz;
            sc = sn;
        }
    }
    return;
bail:
    // a copy did not complete in time: report it, then let the copies still
    // in flight land (bounded) before the CTA's shared memory is released
    if (tid == 0) {
        atomicExch(err, 1);
        for (int s = 0; s < NS; s++)
            if (pending & (1u << s)) mbar_wait(&bars[s], (phase >> s) & 1u);
    }
    __syncthreads();
}

// Variants (element type, TJ, NS, CTAs per SM) the autotuner chooses from.
#define RFB_TMA_VARIANTS_FP32(X) X(float, 8, 4, 5) X(float, 8, 3, 6) X(float, 16, 3, 3)
#define RFB_TMA_VARIANTS_FP64(X) X(double, 8, 3, 3) X(double, 8, 4, 2)

template <typename T>
void launch_interior_tma(const Args<T> &a, const FusedPlan &p, const TmaMaps &m, int *err, cudaStream_t st);

#define RFB_LAUNCH_TMA(TT, TJ_, NS_, MB_)                                                                     \
    if (p.tj == TJ_ && p.ns == NS_)                                                                           \
        k_sweep_interior_tma<TT, TJ_, NS_, MB_><<<p.n_int, dim3(32, TJ_), TmaLayout<TT, TJ_, NS_>::total, st>>>( \
            a, p.d_int, m, err);
template <>
inline void launch_interior_tma<float>(const Args<float> &a, const FusedPlan &p, const TmaMaps &m, int *err,
                                       cudaStream_t st) {
    if (!p.n_int) return;
    RFB_TMA_VARIANTS_FP32(RFB_LAUNCH_TMA)
}
template <>
inline void launch_interior_tma<double>(const Args<double> &a, const FusedPlan &p, const TmaMaps &m, int *err,
                                        cudaStream_t st) {
    if (!p.n_int) return;
    RFB_TMA_VARIANTS_FP64(RFB_LAUNCH_TMA)
}

#define RFB_PREP_TMA(TT, TJ_, NS_, MB_)                                                                     \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_interior_tma<TT, TJ_, NS_, MB_>,                                  \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TmaLayout<TT, TJ_, NS_>::total);
static inline int tma_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaSuccess;
    RFB_TMA_VARIANTS_FP32(RFB_PREP_TMA)
    RFB_TMA_VARIANTS_FP64(RFB_PREP_TMA)
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

#define RFB_TMA_ENTRY(TT, TJ_, NS_, MB_) {TJ_, NS_, MB_},
static const InteriorVariant kTmaVariantsFp32[] = {RFB_TMA_VARIANTS_FP32(RFB_TMA_ENTRY)};
static const InteriorVariant kTmaVariantsFp64[] = {RFB_TMA_VARIANTS_FP64(RFB_TMA_ENTRY)};

}  // namespace rfb
