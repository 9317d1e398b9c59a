// engine.cu -- device memory, uploads, CUDA-graph time loop and the step-wise
// update entry points behind rfsyn's fdtd_update_* functions.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <iterator>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "kernels.cuh"
#include "fused.cuh"
#include "tma.cuh"
#include "sweep.cuh"
#include "energy.cuh"
#include "iq.cuh"
#include "sphere_frac.cuh"

using namespace rfb;

// ---------------------------------------------------------------------------
// errors and launch accounting
// ---------------------------------------------------------------------------
static thread_local char g_err[512];
static std::atomic<unsigned long long> g_launches{0};

extern "C" void rfb_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
extern "C" const char *rfb_last_error(void) { return g_err; }
extern "C" unsigned long long rfb_launch_count(void) { return g_launches.load(); }
extern "C" void rfb_count_launch(void) { g_launches++; }

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            rfb_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            goto fail;                                                                  \
        }                                                                               \
    } while (0)

#define MU0_ 1.25663706212e-6

// ---------------------------------------------------------------------------
// Device memory cache.  cudaMalloc / cudaFree of megabyte blocks cost one to
// a few milliseconds each on B200 (measured), and one scene holds dozens of
// them, so a process that creates and destroys simulations again and again
// (end-to-end runs, batches, sweeps of scenes) spent most of its set-up time
// in the driver.  Blocks of 1 MB and more are rounded up to 2 MB, smaller
// ones to a power of two (at least 256 bytes; the driver calls for small
// blocks were seen to stall a session's set-up or destroy by tens of
// milliseconds now and then), and, when freed, kept per device for the next
// allocation of a size within a quarter of theirs.  A freed block enters the cache after a device synchronisation,
// the same implicit synchronisation cudaFree performs, so no pending work
// can still touch it when it is handed out again.  The cache holds at most a
// quarter of the device's memory; an allocation that fails empties the
// cache and retries.
// ---------------------------------------------------------------------------
namespace {
struct MemCache {
    std::mutex mu;
    std::multimap<size_t, void *> free_blocks[64];  // per device, by size
    size_t free_bytes[64] = {};
    size_t cap[64] = {};
    std::unordered_map<void *, std::pair<int, size_t>> live;  // cached-class block -> device, size
};
MemCache &mem_cache() {
    static MemCache *c = new MemCache();  // never destroyed: frees may run at exit
    return *c;
}
constexpr size_t MC_MIN = 1ull << 20, MC_GRAIN = 2ull << 20;

void mc_release_device(MemCache &c, int dev) {
    for (auto &kv : c.free_blocks[dev]) cudaFree(kv.second);
    c.free_blocks[dev].clear();
    c.free_bytes[dev] = 0;
}
}  // namespace

// Host-side fault injection (no device fault): RFSYN_FDTD_FAIL_ALLOC=n makes
// the n-th device allocation that the creating thread makes inside one
// single-scene engine creation (rfb_engine_create: field buffers, CPML,
// scene upload, plan, graphs) report cudaErrorMemoryAllocation without
// calling the driver, so every error path of engine creation can be driven
// from a test.  The countdown belongs to the creating thread, so allocations
// other threads make meanwhile never take the injected failure; allocations
// made before the engine exists (host scene building, the sphere
// rasteriser's staging) are outside the armed window.  Unset or 0: off.
static thread_local long long g_fail_countdown = 0;

static void arm_alloc_failure(bool on) {
    const char *v = on ? getenv("RFSYN_FDTD_FAIL_ALLOC") : nullptr;
    g_fail_countdown = v ? atoll(v) : 0;
}

static cudaError_t dmalloc_raw(void **p, size_t n) {
    *p = nullptr;
    if (g_fail_countdown > 0 && --g_fail_countdown == 0) return cudaErrorMemoryAllocation;
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return ce;
    if (dev < 0 || dev >= 64) return cudaMalloc(p, n);
    // size classes: powers of two from 256 bytes below MC_MIN, multiples
    // of MC_GRAIN above, so a block freed by one session fits the same
    // request of the next and steady-state sessions make no driver calls
    size_t want;
    if (n < MC_MIN) {
        want = 256;
        while (want < n) want *= 2;
    } else {
        want = (n + MC_GRAIN - 1) / MC_GRAIN * MC_GRAIN;
    }
    MemCache &c = mem_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto &fb = c.free_blocks[dev];
    auto it = fb.lower_bound(want);
    if (it != fb.end() && it->first <= want + want / 4) {
        *p = it->second;
        c.free_bytes[dev] -= it->first;
        c.live[*p] = {dev, it->first};
        fb.erase(it);
        return cudaSuccess;
    }
    ce = cudaMalloc(p, want);
    if (ce == cudaErrorMemoryAllocation && c.free_bytes[dev]) {
        cudaGetLastError();
        mc_release_device(c, dev);
        ce = cudaMalloc(p, want);
    }
    if (ce != cudaSuccess) {
        *p = nullptr;
        return ce;
    }
    c.live[*p] = {dev, want};
    return cudaSuccess;
}

template <typename X>
static cudaError_t dmalloc(X **p, size_t n) {
    return dmalloc_raw(reinterpret_cast<void **>(p), n);
}

static cudaError_t dfree(void *p) {
    if (!p) return cudaSuccess;
    MemCache &c = mem_cache();
    std::unique_lock<std::mutex> lk(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) {
        lk.unlock();
        return cudaFree(p);
    }
    const int dev = it->second.first;
    const size_t size = it->second.second;
    c.live.erase(it);
    // the block is cached only once no work queued before this call can
    // still touch it; the wait runs without the lock, so other threads'
    // allocations and frees are not held up behind this device's work
    lk.unlock();
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaError_t ce = cudaDeviceSynchronize();
    lk.lock();
    if (!c.cap[dev]) {
        size_t fr = 0, tot = 0;
        c.cap[dev] = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? tot / 4 : 0;
    }
    if (ce == cudaSuccess && c.free_bytes[dev] + size <= c.cap[dev]) {
        c.free_blocks[dev].emplace(size, p);
        c.free_bytes[dev] += size;
    } else {
        ce = cudaFree(p);
    }
    if (cur != dev) cudaSetDevice(cur);
    return ce;
}

// Returns every cached block of every device to the driver.
extern "C" void rfb_release_cached_memory(void) {
    MemCache &c = mem_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < 64; d++)
        if (!c.free_blocks[d].empty()) {
            cudaSetDevice(d);
            mc_release_device(c, d);
        }
    cudaSetDevice(cur);
}

extern "C" unsigned long long rfb_cached_bytes(void) {
    MemCache &c = mem_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    unsigned long long s = 0;
    for (int d = 0; d < 64; d++) s += c.free_bytes[d];
    return s;
}

// Device error codes the sweeps record in their error word.
extern "C" double rfb_now(void) {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

// -1 until first read: RFSYN_FDTD_TRACE=1 or the trace setting turns it on
static std::atomic<int> g_trace{-1};

extern "C" int rfb_trace_enabled(void) {
    int on = g_trace.load();
    if (on < 0) {
        const char *v = getenv("RFSYN_FDTD_TRACE");
        on = v && v[0] == '1';
        int expect = -1;
        g_trace.compare_exchange_strong(expect, on);
        on = g_trace.load();
    }
    return on;
}

extern "C" void rfb_set_trace(int on) { g_trace.store(on < 0 ? -1 : on ? 1 : 0); }

extern "C" void rfb_trace(const char *phase, double t0) {
    if (rfb_trace_enabled()) fprintf(stderr, "rfsyn_b200 trace: %s %.3f ms\n", phase, 1e3 * (rfb_now() - t0));
}

static const char *sweep_error_text(int err) {
    return err == 2 ? "a sweep CTA's shared memory did not start on a 128-byte boundary (no copy issued)"
                    : "a sweep's tensor copies did not complete in time";
}

static long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// Row pitch (elements) of the device layout: a multiple of 32 elements, so
// every row starts on a 128-byte line and a 32-wide k tile never runs past
// the end of its row (also for the one-byte code volume).
static long long pitch_for(int nz, size_t esz) {
    (void)esz;
    return round_up(nz + 1, 32);
}

// ---------------------------------------------------------------------------
// CPML on the device: profiles in the run precision, psi over slabs only.
// ---------------------------------------------------------------------------
struct SlabExt {
    int lo, hi, ns;
};

// Leading / trailing non-identity runs of a profile (kappa_inv, b, a) =
// (1, 1, 0) marks the unstretched interior (rfsyn cpml.c:50-52).
static SlabExt slab_extent(const double *kinv, const double *b, const double *a, int len) {
    auto ident = [&](int q) { return kinv[q] == 1.0 && b[q] == 1.0 && a[q] == 0.0; };
    int lead = 0;
    while (lead < len && !ident(lead)) lead++;
    int trail = 0;
    while (trail < len - lead && !ident(len - 1 - trail)) trail++;
    bool interior_ok = true;
    for (int q = lead; q < len - trail; q++)
        if (!ident(q)) interior_ok = false;
    SlabExt s;
    if (!interior_ok) {
        s.lo = len; s.hi = len;
    } else {
        s.lo = lead; s.hi = len - trail;
    }
    s.ns = s.lo + (len - s.hi);
    return s;
}

struct DevCpml {
    int on = 0;
    int prec = RFB_FP64;
    void *prof[3][6] = {};  // kinv_m b_m a_m kinv_h b_h a_h
    SlabExt em[3], eh[3];
    void *psi_e[6] = {};
    void *psi_h[2][6] = {};
    size_t psi_e_bytes[6] = {}, psi_h_bytes[6] = {};
    // the profiles share one allocation and the psi arrays another, each
    // array starting on a 256-byte boundary
    void *prof_base = nullptr, *psi_base = nullptr;
    size_t psi_total = 0;
};

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

static void *dev_upload_conv(const double *src, size_t n, int prec) {
    void *d = nullptr;
    size_t esz = prec == RFB_FP64 ? 8 : 4;
    if (dmalloc(&d, n * esz) != cudaSuccess) return nullptr;
    if (prec == RFB_FP64) {
        if (cudaMemcpy(d, src, n * 8, cudaMemcpyHostToDevice) != cudaSuccess) { dfree(d); return nullptr; }
    } else {
        std::vector<float> tmp(n);
        for (size_t q = 0; q < n; q++) tmp[q] = (float)src[q];
        if (cudaMemcpy(d, tmp.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess) { dfree(d); return nullptr; }
    }
    return d;
}

static void devcpml_free(DevCpml &c) {
    dfree(c.prof_base);
    dfree(c.psi_base);
    c = DevCpml();
}

// nbuf_h: 1 for in-place schedules, 2 for ping-pong H psi.
static int devcpml_init(DevCpml &c, const rfb_geom_t *g, const rfb_cpml_desc_t *d, int prec, long long pitch,
                        int nbuf_h) {
    c.prec = prec;
    c.on = 1;
    const int n[3] = {g->nx, g->ny, g->nz};
    const size_t esz = prec == RFB_FP64 ? 8 : 4;
    // profiles: staged in the run precision on the host, one upload
    size_t prof_off[3][6], prof_bytes = 0;
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 6; q++) {
            prof_off[a][q] = prof_bytes;
            prof_bytes += align256((q < 3 ? (size_t)n[a] + 1 : (size_t)n[a]) * esz);
        }
    {
        std::vector<unsigned char> stage(prof_bytes, 0);
        for (int a = 0; a < 3; a++) {
            const double *src[6] = {d->kinv_m[a], d->b_m[a], d->a_m[a], d->kinv_h[a], d->b_h[a], d->a_h[a]};
            for (int q = 0; q < 6; q++) {
                const size_t len = q < 3 ? (size_t)n[a] + 1 : (size_t)n[a];
                unsigned char *dst = stage.data() + prof_off[a][q];
                if (prec == RFB_FP64) {
                    memcpy(dst, src[q], len * 8);
                } else {
                    float *f = reinterpret_cast<float *>(dst);
                    for (size_t k = 0; k < len; k++) f[k] = (float)src[q][k];
                }
            }
            c.em[a] = slab_extent(d->kinv_m[a], d->b_m[a], d->a_m[a], n[a] + 1);
            c.eh[a] = slab_extent(d->kinv_h[a], d->b_h[a], d->a_h[a], n[a]);
        }
        if (dmalloc(&c.prof_base, prof_bytes) != cudaSuccess ||
            cudaMemcpy(c.prof_base, stage.data(), prof_bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            rfb_set_error("cpml profile upload failed");
            return -1;
        }
        for (int a = 0; a < 3; a++)
            for (int q = 0; q < 6; q++) c.prof[a][q] = static_cast<char *>(c.prof_base) + prof_off[a][q];
    }
    // extents of a psi array with slab axis ax and ns slab cells
    auto bytes = [&](int ax, int ns) -> size_t {
        size_t e;
        if (ax == 0) e = (size_t)ns * (g->ny + 1) * pitch;
        else if (ax == 1) e = (size_t)(g->nx + 1) * ns * pitch;
        else e = (size_t)(g->nx + 1) * (g->ny + 1) * ns;
        return e * esz;
    };
    // psi: offsets first, then one allocation cleared once
    size_t off_e[6], off_h[2][6], total = 0;
    for (int p = 0; p < 6; p++) {
        const int ax = psi_axis_e(p), ah = psi_axis_h(p);
        c.psi_e_bytes[p] = bytes(ax, c.em[ax].ns);
        c.psi_h_bytes[p] = bytes(ah, c.eh[ah].ns);
        off_e[p] = total;
        total += align256(c.psi_e_bytes[p]);
        for (int b = 0; b < nbuf_h; b++) {
            off_h[b][p] = total;
            total += align256(c.psi_h_bytes[p]);
        }
    }
    c.psi_total = total;
    if (total) {
        if (dmalloc(&c.psi_base, total) != cudaSuccess || cudaMemset(c.psi_base, 0, total) != cudaSuccess) {
            rfb_set_error("psi alloc failed");
            return -1;
        }
        char *base = static_cast<char *>(c.psi_base);
        for (int p = 0; p < 6; p++) {
            if (c.psi_e_bytes[p]) c.psi_e[p] = base + off_e[p];
            if (c.psi_h_bytes[p])
                for (int b = 0; b < nbuf_h; b++) c.psi_h[b][p] = base + off_h[b][p];
        }
    }
    return 0;
}

template <typename T>
static void fill_cpml_args(Args<T> &a, const DevCpml &c, int hin, int hout) {
    a.cpml_on = c.on;
    if (!c.on) return;
    for (int ax = 0; ax < 3; ax++) {
        a.kinv_m[ax] = (const T *)c.prof[ax][0];
        a.b_m[ax] = (const T *)c.prof[ax][1];
        a.a_m[ax] = (const T *)c.prof[ax][2];
        a.kinv_h[ax] = (const T *)c.prof[ax][3];
        a.b_h[ax] = (const T *)c.prof[ax][4];
        a.a_h[ax] = (const T *)c.prof[ax][5];
        a.lo_m[ax] = c.em[ax].lo; a.hi_m[ax] = c.em[ax].hi; a.ns_m[ax] = c.em[ax].ns;
        a.lo_h[ax] = c.eh[ax].lo; a.hi_h[ax] = c.eh[ax].hi; a.ns_h[ax] = c.eh[ax].ns;
    }
    for (int p = 0; p < 6; p++) {
        a.psi_e[p] = (T *)c.psi_e[p];
        a.psi_hi[p] = (T *)c.psi_h[hin][p];
        a.psi_ho[p] = (T *)(c.psi_h[hout][p] ? c.psi_h[hout][p] : c.psi_h[hin][p]);
    }
}

// Contiguous rows of `row` bytes into rows of `pitch` bytes.
__global__ void k_repack_u8(uint8_t *dst, const uint8_t *src, long long row, long long pitch, long long n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    dst[(t / row) * pitch + (t % row)] = src[t];
}

// ---------------------------------------------------------------------------
// Scene on the device: code volume, coefficient table, interface list.
// ---------------------------------------------------------------------------
struct DevScene {
    int prec = RFB_FP64;
    uint8_t *codes = nullptr;
    void *tca = nullptr, *tcb = nullptr;
    int n_cells = 0;
    int *lc_ijk = nullptr;
    uint8_t *l_kind = nullptr;
    void *l_ca = nullptr, *l_cb = nullptr;
    int *l_tix = nullptr, *l_src = nullptr, *l_aix = nullptr;
    void *ade_c = nullptr, *ade_s = nullptr;
    size_t ade_s_bytes = 0;
    void *t_m11 = nullptr, *t_scale = nullptr, *t_w = nullptr;
    int *t_main = nullptr, *t_nq = nullptr, *t_uv = nullptr, *t_sign = nullptr;
    void *t3 = nullptr;
    int n_skip = 0;
    long long skip[MAX_SKIP] = {};
    double *cb64_tab = nullptr, *cb64_list = nullptr;  // FP64 Cb for the energy audit
};

static void devscene_free(DevScene &s) {
    dfree(s.codes); dfree(s.tca); dfree(s.tcb);
    dfree(s.lc_ijk); dfree(s.l_kind); dfree(s.l_ca); dfree(s.l_cb);
    dfree(s.l_tix); dfree(s.l_src); dfree(s.l_aix); dfree(s.ade_c); dfree(s.ade_s);
    dfree(s.t_m11); dfree(s.t_scale); dfree(s.t_w);
    dfree(s.t_main); dfree(s.t_nq); dfree(s.t_uv); dfree(s.t_sign);
    dfree(s.cb64_tab); dfree(s.cb64_list); dfree(s.t3);
    s = DevScene();
}

template <typename X>
static X *dev_copy(const X *src, size_t n) {
    if (!n || !src) return nullptr;
    X *d = nullptr;
    if (dmalloc(&d, n * sizeof(X)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, src, n * sizeof(X), cudaMemcpyHostToDevice) != cudaSuccess) { dfree(d); return nullptr; }
    return d;
}

static int devscene_init(DevScene &s, const rfb_geom_t *g, const rfb_scene_image_t *img, int prec,
                         long long pitch) {
    s.prec = prec;
    double tca[256], tcb[256];
    for (int q = 0; q < 256; q++) { tca[q] = 1.0; tcb[q] = 0.0; }
    int tc = img ? img->table_count : 0;
    for (int q = 0; q < tc; q++) { tca[q] = img->table_ca[q]; tcb[q] = img->table_cb[q]; }
    s.tca = dev_upload_conv(tca, 256, prec);
    s.tcb = dev_upload_conv(tcb, 256, prec);
    s.cb64_tab = (double *)dev_upload_conv(tcb, 256, RFB_FP64);
    if (!s.tca || !s.tcb || !s.cb64_tab) { rfb_set_error("table upload failed"); return -1; }
    const size_t plane_b = (size_t)(g->ny + 1) * pitch;
    const size_t total_b = plane_b * (g->nx + 1);
    s.n_cells = img ? (int)img->n_cells : 0;
    if (img && img->codes) {
        if (dmalloc(&s.codes, total_b) != cudaSuccess) { rfb_set_error("code volume alloc failed"); return -1; }
        const size_t rows = (size_t)(g->nx + 1) * (g->ny + 1), row = (size_t)g->nz + 1;
        if (pitch == (long long)row) {
            if (cudaMemcpy(s.codes, img->codes, rows * row, cudaMemcpyHostToDevice) != cudaSuccess) {
                rfb_set_error("code volume upload failed");
                return -1;
            }
        } else {
            // one contiguous upload, then a device-side repack into the
            // pitched layout (a strided host copy of short rows is slow)
            uint8_t *tmp = nullptr;
            if (dmalloc(&tmp, rows * row) != cudaSuccess) { rfb_set_error("code volume staging failed"); return -1; }
            cudaError_t ce = cudaMemcpy(tmp, img->codes, rows * row, cudaMemcpyHostToDevice);
            if (ce == cudaSuccess) {
                const long long n = (long long)(rows * row);
                k_repack_u8<<<(unsigned)((n + 255) / 256), 256>>>(s.codes, tmp, (long long)row, pitch, n);
                g_launches++;
                ce = cudaDeviceSynchronize();
            }
            dfree(tmp);
            if (ce != cudaSuccess) { rfb_set_error("code volume upload failed"); return -1; }
        }
    }
    if (s.n_cells) {
        const size_t ne = 3 * (size_t)s.n_cells;
        s.lc_ijk = dev_copy(img->cell_ijk, 3 * (size_t)s.n_cells);
        s.l_kind = dev_copy(img->kind, ne);
        s.l_ca = dev_upload_conv(img->ca, ne, prec);
        s.l_cb = dev_upload_conv(img->cb, ne, prec);
        s.cb64_list = (double *)dev_upload_conv(img->cb, ne, RFB_FP64);
        s.l_tix = dev_copy(img->tix, ne);
        s.l_src = dev_copy(img->src, ne);
        s.l_aix = dev_copy(img->aix, ne);
        if (!s.lc_ijk || !s.l_kind || !s.l_ca || !s.l_cb || !s.l_tix || !s.l_src || !s.l_aix || !s.cb64_list) {
            rfb_set_error("interface list upload failed");
            return -1;
        }
        if (img->n_tensors) {
            size_t nt = img->n_tensors;
            s.t_m11 = dev_upload_conv(img->t_m11, nt, prec);
            s.t_scale = dev_upload_conv(img->t_scale, nt, prec);
            s.t_w = dev_upload_conv(img->t_w, 4 * nt, prec);
            s.t_main = dev_copy(img->t_main, 4 * nt);
            s.t_nq = dev_copy(img->t_nq, nt);
            s.t_uv = dev_copy(img->t_uv, 16 * nt);
            s.t_sign = dev_copy(img->t_sign, nt);
            if (!s.t_m11 || !s.t_scale || !s.t_w || !s.t_main || !s.t_nq || !s.t_uv || !s.t_sign) {
                rfb_set_error("tensor list upload failed");
                return -1;
            }
        }
        if (img->n_t3) {
            s.t3 = dev_upload_conv(img->t3, 5 * img->n_t3, prec);
            if (!s.t3) {
                rfb_set_error("3x3 tensor upload failed");
                return -1;
            }
        }
        if (img->n_ade) {
            s.ade_c = dev_upload_conv(img->ade_c, img->n_ade * RFB_ADE_NC, prec);
            s.ade_s_bytes = ne * 5 * (prec == RFB_FP64 ? 8 : 4);
            if (!s.ade_c || dmalloc(&s.ade_s, s.ade_s_bytes) != cudaSuccess) {
                rfb_set_error("dispersive state allocation failed");
                return -1;
            }
            cudaMemset(s.ade_s, 0, s.ade_s_bytes);
        }
        if (!s.codes) {
            if (s.n_cells <= MAX_SKIP) {
                s.n_skip = s.n_cells;
                for (int q = 0; q < s.n_cells; q++)
                    s.skip[q] = ((long long)img->cell_ijk[3 * q] * (g->ny + 1) + img->cell_ijk[3 * q + 1]) * pitch +
                                img->cell_ijk[3 * q + 2];
            } else {
                if (dmalloc(&s.codes, total_b) != cudaSuccess) { rfb_set_error("code volume alloc failed"); return -1; }
                cudaMemset(s.codes, 0, total_b);
                k_mark_list<<<(s.n_cells + 255) / 256, 256>>>(s.codes, s.lc_ijk, s.n_cells, g->ny, pitch);
                g_launches++;
                if (cudaDeviceSynchronize() != cudaSuccess) { rfb_set_error("mark list failed"); return -1; }
            }
        }
    }
    return 0;
}

template <typename T>
static void fill_scene_args(Args<T> &a, const DevScene &s) {
    a.codes = s.codes;
    a.tca = (const T *)s.tca;
    a.tcb = (const T *)s.tcb;
    a.n_skip = s.n_skip;
    for (int q = 0; q < MAX_SKIP; q++) a.skip[q] = s.skip[q];
    a.n_cells = s.n_cells;
    a.lc_ijk = s.lc_ijk;
    a.l_kind = s.l_kind;
    a.l_ca = (const T *)s.l_ca;
    a.l_cb = (const T *)s.l_cb;
    a.l_tix = s.l_tix;
    a.l_src = s.l_src;
    a.l_aix = s.l_aix;
    a.ade_c = (const T *)s.ade_c;
    a.ade_s = (T *)s.ade_s;
    a.t_m11 = (const T *)s.t_m11;
    a.t_scale = (const T *)s.t_scale;
    a.t_w = (const T *)s.t_w;
    a.t_main = s.t_main;
    a.t_nq = s.t_nq;
    a.t_uv = s.t_uv;
    a.t_sign = s.t_sign;
    a.t3 = (const T *)s.t3;
}

template <typename T>
static void fill_geom_args(Args<T> &a, const rfb_geom_t *g, long long pitch) {
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.per = g->periodic;
    a.pitch = pitch;
    a.plane = (long long)(g->ny + 1) * pitch;
    a.cbh = (T)(g->dt / (MU0_ * g->dx));
    a.dx = (T)g->dx;
}

// ---------------------------------------------------------------------------
// Engine (device time loop)
// ---------------------------------------------------------------------------
struct rfb_engine {
    rfb_geom_t g;
    int prec, sched;
    long long pitch;
    size_t esz, total;
    void *fld[2][6] = {};
    void *fld_base = nullptr;  // one allocation holds every field buffer
    int nbuf = 1;
    DevCpml cpml;
    DevScene scene;
    int n_src = 0;
    void *src_val = nullptr;
    int *src_hard = nullptr;
    int n_probes = 0;
    long long *probe_cell = nullptr;
    int *probe_comp = nullptr;
    void *ts = nullptr;
    int *d_step = nullptr;
    size_t n_steps = 0, steps_done = 0;
    double *d_omega = nullptr, *d_re = nullptr, *d_im = nullptr;
    size_t dft_cap = 0;
    // plane probes: series n_probes .. n_probes + n_planes - 1 of ts
    int n_planes = 0;
    PlaneDesc *d_planes = nullptr;
    // the gather's per-chunk sums (n_planes x plane_chunks) and per-plane
    // counters of finished chunks (zero between launches)
    int plane_chunks = 0;
    double *d_plane_part = nullptr;
    int *d_plane_count = nullptr;
    void **d_fout[2] = {nullptr, nullptr};  // per parity: the six output components, for the plane gather
    // running DFT of every series: the bins (rad/s), t offset (steps), the
    // per (series, bin) sums (FP64: re, im; FP32: re, im, compensations)
    int n_freqs = 0;
    std::vector<double> dft_freqs;
    double dft_t_off = 0.0;
    double *d_run_omega = nullptr;
    void *d_acc = nullptr;
    cudaStream_t stream = nullptr, stream2 = nullptr, stream3 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join3 = nullptr;
    int own_stream = 0;
    int parity = 0;
    static constexpr int CHUNK = 16;
    cudaGraphExec_t g1[2] = {nullptr, nullptr}, gk[2] = {nullptr, nullptr};
    int launches_per_step = 0;
    FusedPlan plan;
    TmaMaps tmaps[2];       // tensor maps of the input buffers per parity (TMA interior sweep)
    int *d_err = nullptr;   // set by a sweep whose copies did not complete in time
    double *d_energy = nullptr;  // energy audit: block partials + result
    float *d_iq = nullptr;       // stage output: n_steps I/Q pairs, then the noise scale (a double)
    // cells whose three E samples are 3x3 samples without source or TF/SF
    // term, updated per cell by k_list_cells (their list entries are kind 5);
    // t3_kinds keeps the image's kinds to undo it
    int *t3_cells = nullptr;
    int n_t3_cells = 0;
    // cells whose three E samples are dispersive samples outside the CPML
    // without source or TF/SF term, updated per cell by k_list_cells (their
    // list entries are kind 6)
    int *ade_cells = nullptr;
    int n_ade_cells = 0;
    std::vector<int> ade_host;
    // the list entries outside those cells (k_e_list's work), or none
    int *list_work = nullptr;
    int n_list_work = 0;
    std::vector<uint8_t> t3_kinds;
    std::vector<int> t3_host;
    size_t h2d_bytes = 0, n_ade = 0;
    // plane wave (TF/SF): line, H-target terms, per-entry E terms
    int tf_on = 0, tf_n_h = 0, tf_m_len = 0;
    double tf_ce = 0, tf_ch = 0;
    void *tf_inc_e = nullptr, *tf_inc_h = nullptr, *tf_src = nullptr;
    long long *tf_h_cell = nullptr;
    int *tf_h_comp = nullptr, *tf_h_first = nullptr, *tf_h_count = nullptr, *tf_h_idx = nullptr;
    void *tf_h_coef = nullptr, *tf_h_w = nullptr;
    int *tf_e_first = nullptr, *tf_e_count = nullptr, *tf_e_idx = nullptr;
    void *tf_e_coef = nullptr, *tf_e_w = nullptr;
    int active = 0;          // a source sits on a padded boundary plane
    int member = 0;          // scene of a batch: no plan, graphs or second stream of its own
};

template <typename T>
static Args<T> engine_args(const rfb_engine *e, int par) {
    Args<T> a;
    memset(&a, 0, sizeof a);
    fill_geom_args(a, &e->g, e->pitch);
    const int in = e->nbuf == 2 ? par : 0, out = e->nbuf == 2 ? 1 - par : 0;
    for (int c = 0; c < 3; c++) {
        a.E[c] = (T *)e->fld[in][c];
        a.H[c] = (T *)e->fld[in][3 + c];
        a.Eo[c] = (T *)e->fld[out][c];
        a.Ho[c] = (T *)e->fld[out][3 + c];
    }
    fill_cpml_args(a, e->cpml, in, e->cpml.psi_h[1][0] || e->nbuf == 2 ? out : in);
    fill_scene_args(a, e->scene);
    a.src_val = (const T *)e->src_val;
    a.src_hard = e->src_hard;
    if (e->n_t3_cells || e->n_ade_cells) {
        a.l_work = e->list_work;
        a.n_work = e->n_list_work;
    }
    a.n_steps = (long long)e->n_steps;
    a.d_step = e->d_step;
    if (e->tf_on) {
        a.tf_first = e->tf_e_first;
        a.tf_count = e->tf_e_count;
        a.tf_idx = e->tf_e_idx;
        a.tf_coef = (const T *)e->tf_e_coef;
        a.tf_w = (const T *)e->tf_e_w;
        a.inc_h = (const T *)e->tf_inc_h;
    }
    return a;
}

template <typename T>
static TfArgs<T> tf_args(const rfb_engine *e, int par) {
    TfArgs<T> t;
    memset(&t, 0, sizeof t);
    const int out = e->nbuf == 2 ? 1 - par : 0;
    t.n_h = e->tf_n_h;
    t.h_cell = e->tf_h_cell;
    t.h_comp = e->tf_h_comp;
    t.h_first = e->tf_h_first;
    t.h_count = e->tf_h_count;
    t.h_idx = e->tf_h_idx;
    t.h_coef = (const T *)e->tf_h_coef;
    t.h_w = (const T *)e->tf_h_w;
    for (int c = 0; c < 3; c++) t.Ho[c] = (T *)e->fld[out][3 + c];
    t.inc_e = (T *)e->tf_inc_e;
    t.inc_h = (T *)e->tf_inc_h;
    t.m_len = e->tf_m_len;
    t.ce = (T)e->tf_ce;
    t.ch = (T)e->tf_ch;
    t.src = (const T *)e->tf_src;
    t.d_step = e->d_step;
    t.n_steps = (long long)e->n_steps;
    return t;
}

// Plane wave: H corrections from the line's E^n, then the line's H to n+1/2
// (before the interface list, whose boundary entries read it).
template <typename T>
static void tf_before_list(rfb_engine *e, int par) {
    if (!e->tf_on) return;
    TfArgs<T> t = tf_args<T>(e, par);
    if (t.n_h) k_tfsf_h<T><<<(t.n_h + 255) / 256, 256, 0, e->stream>>>(t);
    k_inc_h<T><<<(t.m_len + 255) / 256, 256, 0, e->stream>>>(t);
}
// ... and the line's E to n+1 after the step counter advanced.
template <typename T>
static void tf_after_step(rfb_engine *e, int par) {
    if (!e->tf_on) return;
    TfArgs<T> t = tf_args<T>(e, par);
    k_inc_e<T><<<(t.m_len + 255) / 256, 256, 0, e->stream>>>(t);
}

// Interior sweep of the plan: TMA-fed or cp.async-fed variant, or (mode 2)
// the persistent work-queue sweep over the interior items.
template <typename T>
static void launch_q_t(const Args<T> &a, const FusedPlan &p, int kind, const TmaMaps &m, int *err, cudaStream_t st);
template <>
void launch_q_t<float>(const Args<float> &a, const FusedPlan &p, int kind, const TmaMaps &m, int *err,
                       cudaStream_t st) {
    if (kind == 2 && p.uni) launch_q_f<5>(a, p.d, p.tj, p.ns, p.d_qe, p.n_qe, m, p.d_queue + 2, err, st);
    else if (kind == 2) launch_q_f<2>(a, p.d, p.tj, p.ns, p.d_qe, p.n_qe, m, p.d_queue + 2, err, st);
    else if (kind == 1) launch_q_f<1>(a, p.d, p.tj, p.ns, p.d_qx, p.n_qx, m, p.d_queue + 4, err, st);
    else launch_q_f<0>(a, p.d, p.tj, p.ns, p.d_int, p.n_int, m, p.d_queue, err, st);
}
template <>
void launch_q_t<double>(const Args<double> &a, const FusedPlan &p, int kind, const TmaMaps &m, int *err,
                        cudaStream_t st) {
    if (kind == 2 && p.uni) launch_q_d<5>(a, p.d, p.tj, p.ns, p.d_qe, p.n_qe, m, p.d_queue + 2, err, st);
    else if (kind == 2) launch_q_d<2>(a, p.d, p.tj, p.ns, p.d_qe, p.n_qe, m, p.d_queue + 2, err, st);
    else if (kind == 1) launch_q_d<1>(a, p.d, p.tj, p.ns, p.d_qx, p.n_qx, m, p.d_queue + 4, err, st);
    else launch_q_d<0>(a, p.d, p.tj, p.ns, p.d_int, p.n_int, m, p.d_queue, err, st);
}

// The two-rows interior sweep (FP32 plans only).
static void launch_interior_i2(const Args<float> &a, const FusedPlan &p, const TmaMaps &m, int *err, cudaStream_t st) {
    launch_q_i2(a, p.i2, p.d_int, p.n_int, m, p.d_queue, err, st);
}
static void launch_interior_i2(const Args<double> &, const FusedPlan &, const TmaMaps &, int *, cudaStream_t) {}

template <typename T>
static void launch_int(rfb_engine *e, const Args<T> &a, int par, cudaStream_t st) {
    const TmaMaps &m = e->tmaps[e->nbuf == 2 ? par : 0];
    if (e->plan.tma >= 2) {
        if (e->plan.i2) launch_interior_i2(a, e->plan, m, e->d_err, st);
        else launch_q_t<T>(a, e->plan, 0, m, e->d_err, st);
        launch_q_t<T>(a, e->plan, 1, m, e->d_err, st);
    } else if (e->plan.tma) launch_interior_tma<T>(a, e->plan, m, e->d_err, st);
    else launch_interior<T>(a, e->plan, st);
}
// Work-queue plans that also hold cp.async-fed edge items (the tiles whose
// halo wraps around a periodic y / z axis) run those on a third stream:
// both edge launches are bound by the march of one item, so one after the
// other they would take twice as long as side by side.
static bool edge_on_third_stream(const rfb_engine *e) {
    return e->plan.tma >= 2 && e->plan.n_edge > 0 && e->stream3 != nullptr;
}

// Everything else of the sweep: the slab / boundary queue (modes 2-4) and
// the cp.async-fed edge sweep (mode 0 and 1 edge tiles; in modes 2-4 the
// items whose halo wraps, unless they have the third stream).
template <typename T>
static void launch_rest(rfb_engine *e, const Args<T> &a, int par, cudaStream_t st) {
    if (e->plan.tma >= 2) launch_q_t<T>(a, e->plan, 2, e->tmaps[e->nbuf == 2 ? par : 0], e->d_err, st);
    if (!edge_on_third_stream(e)) launch_edge<T>(a, e->plan, st);
}

// One fused sweep: the interior kinds on the engine stream, the slab /
// boundary kinds on the second stream, side by side (they touch disjoint
// cells); a work-queue plan's cp.async-fed edge items on a third.  A third
// stream for the x-slab kind measured slower on C2.
template <typename T>
static void launch_sweep(rfb_engine *e, const Args<T> &a, int par) {
    const bool third = edge_on_third_stream(e);
    cudaEventRecord(e->ev_fork, e->stream);
    cudaStreamWaitEvent(e->stream2, e->ev_fork, 0);
    if (third) cudaStreamWaitEvent(e->stream3, e->ev_fork, 0);
    launch_int<T>(e, a, par, e->stream);
    launch_rest<T>(e, a, par, e->stream2);
    if (third) {
        launch_edge<T>(a, e->plan, e->stream3);
        cudaEventRecord(e->ev_join3, e->stream3);
    }
    cudaEventRecord(e->ev_join, e->stream2);
    cudaStreamWaitEvent(e->stream, e->ev_join, 0);
    if (third) cudaStreamWaitEvent(e->stream, e->ev_join3, 0);
}

// Threads of the interface-list launch: the entries left to it when some
// cells go to the per-cell kernels (none when all do), else every entry.
static int list_threads(const rfb_engine *e) {
    return (e->n_t3_cells || e->n_ade_cells) ? e->n_list_work : 3 * e->scene.n_cells;
}

// Launches of the step's interface list: one (k_list_cells when some cells
// have per-cell updates, else k_e_list), or none without list work.
static int list_launches(const rfb_engine *e) {
    return (e->scene.n_cells && list_threads(e)) || e->n_t3_cells || e->n_ade_cells ? 1 : 0;
}

template <typename T>
static void launch_list(rfb_engine *e, const Args<T> &a) {
    if (e->n_t3_cells || e->n_ade_cells) {
        const int nb3 = (e->n_t3_cells + 255) / 256, nba = (e->n_ade_cells + 255) / 256;
        const int nbl = (list_threads(e) + 255) / 256;
        k_list_cells<T><<<nb3 + nba + nbl, 256, 0, e->stream>>>(a, e->t3_cells, e->n_t3_cells, nb3, e->ade_cells,
                                                                e->n_ade_cells, nba);
    } else if (a.n_cells && list_threads(e)) {
        k_e_list<T><<<(list_threads(e) + 255) / 256, 256, 0, e->stream>>>(a);
    }
}

// Plane probes of the step: their means join the series before the point
// probes advance the step counter.
template <typename T>
static void launch_plane_gather(rfb_engine *e, int par) {
    if (!e->n_planes) return;
    const int out = e->nbuf == 2 ? 1 - par : 0;
    k_plane_gather<T><<<dim3(e->plane_chunks, e->n_planes), kPlaneThreads, 0, e->stream>>>(
        e->d_planes, e->n_planes, (const T *const *)e->d_fout[out], (T *)e->ts, e->n_probes, (long long)e->n_steps,
        e->d_step, e->d_plane_part, e->d_plane_count, e->plane_chunks);
}

template <typename T>
static void enqueue_step(rfb_engine *e, int par) {
    Args<T> a = engine_args<T>(e, par);
    const rfb_geom_t &g = e->g;
    if (e->sched == RFB_SCHED_FUSED) {
        launch_sweep<T>(e, a, par);
    } else {
        dim3 blk(32, 8);
        dim3 grd((g.nz + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nx + 1);
        k_h_split<T><<<grd, blk, 0, e->stream>>>(a);
        k_e_split<T><<<grd, blk, 0, e->stream>>>(a);
    }
    tf_before_list<T>(e, par);
    launch_list<T>(e, a);
    ProbeArgs<T> p;
    p.n = e->n_probes;
    p.cell = e->probe_cell;
    p.comp = e->probe_comp;
    const int out = e->nbuf == 2 ? 1 - par : 0;
    for (int c = 0; c < 6; c++) p.F[c] = (const T *)e->fld[out][c];
    p.ts = (T *)e->ts;
    p.n_steps = (long long)e->n_steps;
    p.d_step = e->d_step;
    launch_plane_gather<T>(e, par);
    k_probe_gather<T><<<1, 128, 0, e->stream>>>(p);
    tf_after_step<T>(e, par);
}

// The running DFT over the last `count` recorded samples of every series.
template <typename T>
static void launch_dft_run(rfb_engine *e, int count) {
    const int ns = e->n_probes + e->n_planes;
    if (!e->n_freqs || !ns) return;
    dim3 grd((unsigned)((e->n_freqs + 127) / 128), (unsigned)ns);
    k_dft_run<T><<<grd, 128, 0, e->stream>>>((const T *)e->ts, ns, (long long)e->n_steps, e->d_step, count,
                                             e->n_freqs, e->d_run_omega, e->g.dt, e->dft_t_off, e->d_acc);
}

static int count_step_launches(const rfb_engine *e) {
    int n = (e->sched == RFB_SCHED_FUSED)
                ? (e->plan.n_int > 0) + (e->plan.n_edge > 0) + (e->plan.n_qe > 0) + (e->plan.n_qx > 0)
                : 2;
    n += list_launches(e);
    if (e->tf_on) n += 2 + (e->tf_n_h > 0);
    if (e->n_planes) n++;
    return n + 1;
}

static int build_graph(rfb_engine *e, int par, int steps, cudaGraphExec_t *out) {
    cudaGraph_t graph = nullptr;
    int p = par;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < steps; s++) {
        if (e->prec == RFB_FP64) enqueue_step<double>(e, p);
        else enqueue_step<float>(e, p);
        if (e->nbuf == 2) p ^= 1;
    }
    if (e->prec == RFB_FP64) launch_dft_run<double>(e, steps);
    else launch_dft_run<float>(e, steps);
    CK(cudaStreamEndCapture(e->stream, &graph));
    CK(cudaGraphInstantiate(out, graph, 0));
    cudaGraphDestroy(graph);
    return 0;
fail:
    if (graph) cudaGraphDestroy(graph);
    return -1;
}

// Work lists of the sweep.  Interior items: column tiles of (tj x 32) cells
// in (j, k) whose cells, halo row and halo column lie outside every CPML
// slab and PEC boundary (and hold no code-less list cell), over the interior
// plane range; edge items: (8 x 32) tiles over everything else.
static void free_plan_lists(FusedPlan &p) {
    dfree(p.d_int);
    dfree(p.d_edge);
    dfree(p.d_qe);
    dfree(p.d_qx);
    p.d_int = p.d_edge = p.d_qe = p.d_qx = nullptr;
    p.n_int = p.n_edge = p.n_qe = p.n_qx = 0;
}

// ---- tensor maps of the TMA interior sweep -----------------------------------
// Each field array (and the code volume) is a 3-D tensor (pitch, ny+1, nx+1),
// k fastest; boxes are (40 | 36 | 32) x rows x 1 plane.  Out-of-range boxes
// parts read as zero (no NaN fill).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)f;
    });
    return fn;
}

static int encode_map(CUtensorMap *m, void *base, CUtensorMapDataType dt, size_t esz, const rfb_geom_t &g,
                      size_t pitch, unsigned box_w, unsigned box_h) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        rfb_set_error("the CUDA driver does not provide cuTensorMapEncodeTiled");
        return -1;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)g.ny + 1, (cuuint64_t)g.nx + 1};
    const cuuint64_t strides[2] = {(cuuint64_t)(pitch * esz), (cuuint64_t)(pitch * esz * (g.ny + 1))};
    const cuuint32_t box[3] = {box_w, box_h, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        rfb_set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return -1;
    }
    return 0;
}

static int build_tma_maps(rfb_engine *e, int tj) {
    const CUtensorMapDataType dt =
        e->prec == RFB_FP64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    for (int par = 0; par < 2; par++) {
        const int in = e->nbuf == 2 ? par : 0;
        TmaMaps &m = e->tmaps[par];
        memset(&m, 0, sizeof m);
        for (int c = 0; c < 3; c++) {
            if (encode_map(&m.e[c], e->fld[in][c], dt, e->esz, e->g, e->pitch, TMA_EW, tj + 2)) return -1;
            if (encode_map(&m.h[c], e->fld[in][3 + c], dt, e->esz, e->g, e->pitch, TMA_HW, tj + 1)) return -1;
            // narrow tiles: 2 tj rows x 16 columns (E 24 x (2 tj + 2), H 20 x (2 tj + 1))
            if (encode_map(&m.en[c], e->fld[in][c], dt, e->esz, e->g, e->pitch, 24, 2 * tj + 2)) return -1;
            if (encode_map(&m.hn[c], e->fld[in][3 + c], dt, e->esz, e->g, e->pitch, 20, 2 * tj + 1)) return -1;
        }
        // interior tiles of 2 tj rows x 32 columns (two rows per thread)
        for (int c = 0; c < 3; c++) {
            if (encode_map(&m.e2[c], e->fld[in][c], dt, e->esz, e->g, e->pitch, TMA_EW, 2 * tj + 2)) return -1;
            if (encode_map(&m.h2[c], e->fld[in][3 + c], dt, e->esz, e->g, e->pitch, TMA_HW, 2 * tj + 1)) return -1;
        }
        if (e->scene.codes &&
            (encode_map(&m.code, e->scene.codes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, e->g, e->pitch, 32, tj) ||
             encode_map(&m.coden, e->scene.codes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, e->g, e->pitch, 16, 2 * tj) ||
             encode_map(&m.code2, e->scene.codes, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, e->g, e->pitch, 32, 2 * tj)))
            return -1;
    }
    return 0;
}

// The work-queue sweeps address psi arrays and field planes with 32-bit
// offsets: admitted only when each has fewer than 2^31 elements.
static bool q_fits(const rfb_engine *e) {
    const long long lim = 1LL << 31;
    const rfb_geom_t &g = e->g;
    const long long plane = (long long)(g.ny + 1) * e->pitch;
    if (plane >= lim) return false;
    if (!e->cpml.on) return true;
    const long long x = (long long)e->cpml.eh[0].ns * plane, xm = (long long)e->cpml.em[0].ns * plane;
    const long long y = (long long)(g.nx + 1) * std::max(e->cpml.eh[1].ns, e->cpml.em[1].ns) * e->pitch;
    const long long z = (long long)(g.nx + 1) * (g.ny + 1) * std::max(e->cpml.eh[2].ns, e->cpml.em[2].ns);
    return x < lim && xm < lim && y < lim && z < lim;
}

// Work items of a sweep plan (host lists): vi interior, vx x-slab planes of
// interior tiles (modes 2, 3), vq slab / boundary tiles of the work-queue
// edge sweep (modes 2, 3), ve tiles of the cp.async-fed edge sweep.
struct PlanLists {
    std::vector<SweepItem> vi, vx, vq, ve;
    FusedDims d;
};

static void plan_items(const rfb_engine *e, int active, int tj, int tma, int seg_int, int seg_edge, PlanLists &out,
                       int i2 = 0) {
    const rfb_geom_t &g = e->g;
    const bool px = g.periodic & 1u, py = g.periodic & 2u, pz = g.periodic & 4u;
    PlanLists &p = out;
    p.d.cj = g.ny + ((active && !py) ? 1 : 0);
    p.d.ck = g.nz + ((active && !pz) ? 1 : 0);
    p.d.ci = g.nx + ((active && !px) ? 1 : 0);
    std::vector<SweepItem> &vi = p.vi, &ve = p.ve, &vq = p.vq, &vx = p.vx;
    const bool on = e->cpml.on != 0;
    int xlo, xhi, ylo, yhi, zlo, zhi;
    auto ext = [&](int ax, int *lo, int *hi, int n, bool per) {
        interior_axis(on ? e->cpml.eh[ax].lo : 0, on ? e->cpml.eh[ax].hi : n, on ? e->cpml.em[ax].lo : 0,
                      on ? e->cpml.em[ax].hi : n + 1, n, per, on, lo, hi);
    };
    ext(0, &xlo, &xhi, g.nx, px);
    ext(1, &ylo, &yhi, g.ny, py);
    ext(2, &zlo, &zhi, g.nz, pz);
    const int xa = px ? 0 : xlo + 1, xb = std::max(xa, xhi);
    auto add = [](std::vector<SweepItem> &v, int j0, int k0, int b, int en, int seg, int sub = 0) {
        for (int s = b; s < en; s += seg) v.push_back(SweepItem{j0, k0, s, std::min(en, s + seg), sub});
    };
    // does [q0, q1] hold a slab cell of axis ax on the H or the E grid (the
    // kernels' slab_in: inside [0, len) and outside [lo, hi))
    auto touches = [&](int ax, int q0, int q1) {
        if (!on) return false;
        const int n = ax == 1 ? g.ny : g.nz;
        const SlabExt &h = e->cpml.eh[ax], &m = e->cpml.em[ax];
        for (int q = q0; q <= q1; q++) {
            if (q >= 0 && q < n && (q < h.lo || q >= h.hi)) return true;
            if (q >= 0 && q < n + 1 && (q < m.lo || q >= m.hi)) return true;
        }
        return false;
    };
    auto add_edge = [&](int j0, int rows, int k0, int b, int en) {
        // modes 2, 3: tiles whose halo stays inside the grid go to the TMA-fed
        // slab / boundary queue; tiles whose halo wraps around a periodic
        // axis to the cp.async-fed edge sweep (8-row tiles)
        const bool wraps = (py && (j0 <= 0 || j0 + rows >= g.ny)) || (pz && (k0 <= 0 || k0 + 32 >= g.nz));
        if (tma >= 2 && !wraps) {
            // rows j0-1 .. j0+rows-1 and columns k0-1 .. k0+31 cover the
            // tile, its halo row and its halo column
            const bool ty = touches(1, j0 - 1, j0 + rows - 1), tz = touches(2, k0 - 1, k0 + 31);
            add(vq, j0, k0, b, en, seg_edge, ty && tz ? 0 : tz ? 2 : 1);
            return;
        }
        for (int jj = j0; jj < j0 + rows && jj < p.d.cj; jj += 8) add(ve, jj, k0, b, en, seg_edge);
    };
    // tile origins: multiples of (tj, 32) from 0, or in modes 3 and 4, on
    // axes without wrap, shifted so that the first interior tile starts right
    // after the low slab (j0 any row, k0 a multiple of 16 for the TMA boxes);
    // the tiles below it may start at negative coordinates, their cells
    // outside the grid are idle lanes.  Mode 4 (no periodic y / z) covers
    // the z-slab columns with narrow (2 tj x 16) tiles instead: 32-wide
    // columns only where they are z-interior, 16-wide columns below and
    // above them.
    int js = 0, ks = 0;
    std::vector<std::pair<int, int>> cols;  // (k0, width)
    if (tma == 4) {
        const int ja = ylo + 1;
        js = ja - tj * ((ja + tj - 1) / tj);
        const int ka = (zlo + 1 + 15) / 16 * 16;
        int kb = ka;
        while (kb + 32 <= std::min(zhi, p.d.ck)) kb += 32;
        for (int k0 = ka - 16; k0 + 16 > 0; k0 -= 16) cols.push_back({k0, 16});
        for (int k0 = ka; k0 < kb; k0 += 32) cols.push_back({k0, 32});
        for (int k0 = kb; k0 < p.d.ck; k0 += 16) cols.push_back({k0, 16});
    }
    if (tma == 3) {
        if (!py) {
            const int ja = ylo + 1;
            js = ja - tj * ((ja + tj - 1) / tj);
        }
        if (!pz) {
            const int ka = (zlo + 1 + 15) / 16 * 16;
            ks = ka - 32 * ((ka + 31) / 32);
        }
    }
    if (tma != 4)
        for (int k0 = ks; k0 < p.d.ck; k0 += 32) cols.push_back({k0, 32});
    for (const auto &cw : cols) {
        const int k0 = cw.first;
        if (cw.second == 16) {
            // narrow z-slab tiles: always slab / boundary work
            for (int j0 = 0; j0 < p.d.cj; j0 += 2 * tj)
                add(vq, j0, k0, 0, p.d.ci, seg_edge, touches(1, j0 - 1, j0 + 2 * tj - 1) ? 4 : 3);
            continue;
        }
        for (int j0 = js; j0 < p.d.cj; j0 += tj) {
            const bool full = j0 >= 0 && k0 >= 0 && j0 + tj <= p.d.cj && k0 + 32 <= p.d.ck;
            // the interior sweeps read the halo without wrapping it: on a
            // periodic axis the tiles at either end stay on the edge sweep
            const bool yok = py ? (j0 >= 1 && j0 + tj < g.ny) : (j0 - 1 >= ylo && j0 + tj <= yhi);
            const bool zok = pz ? (k0 >= 32 && k0 + 32 < g.nz) : (k0 - 1 >= zlo && k0 + 32 <= zhi);
            bool skipcell = false;
            for (int s = 0; s < e->scene.n_skip; s++) {
                const long long c = e->scene.skip[s];
                const int sk = (int)(c % e->pitch), sj = (int)((c / e->pitch) % (g.ny + 1));
                if (sj >= j0 && sj < j0 + tj && sk >= k0 && sk < k0 + 32) skipcell = true;
            }
            if (tma >= 2 && full && yok && zok && !skipcell && xb > xa) {
                // interior planes to the interior sweep, x-slab and
                // x-boundary planes to the x-slab sweep
                add(vi, j0, k0, xa, xb, seg_int);
                add(vx, j0, k0, 0, xa, seg_edge);
                add(vx, j0, k0, xb, p.d.ci, seg_edge);
            } else if (full && yok && zok && !skipcell && xb > xa) {
                add(vi, j0, k0, xa, xb, seg_int);
                add_edge(j0, tj, k0, 0, xa);
                add_edge(j0, tj, k0, xb, p.d.ci);
            } else {
                add_edge(j0, tj, k0, 0, p.d.ci);
            }
        }
    }
    if (i2) {
        // two-rows interior: pair each interior tile with the one below it
        // (same column, same planes) into one item of 2 tj rows; a tile
        // left without a partner goes to the slab / boundary queue, whose
        // full body sweeps any tile
        std::vector<SweepItem> paired;
        std::vector<bool> used(vi.size(), false);
        for (size_t a = 0; a < vi.size(); a++) {
            if (used[a]) continue;
            size_t b = a + 1;
            for (; b < vi.size(); b++)
                if (!used[b] && vi[b].k0 == vi[a].k0 && vi[b].j0 == vi[a].j0 + tj && vi[b].ib == vi[a].ib &&
                    vi[b].ie == vi[a].ie)
                    break;
            used[a] = true;
            if (b < vi.size()) {
                used[b] = true;
                paired.push_back(vi[a]);
            } else {
                SweepItem it = vi[a];
                it.sub = 0;
                vq.push_back(it);
            }
        }
        vi.swap(paired);
    }
    // queue order: longest items first, so the last items to start are
    // short; among equal lengths, items of one body together
    std::stable_sort(vq.begin(), vq.end(), [](const SweepItem &x, const SweepItem &y) {
        if (x.ie - x.ib != y.ie - y.ib) return x.ie - x.ib > y.ie - y.ib;
        return x.sub < y.sub;
    });
}

static int build_sweep_plan(rfb_engine *e, int active, int tj, int ns, int tma, int seg_int, int seg_edge,
                            int uni = 0, int i2 = 0) {
    if (i2 && (tma < 2 || uni || e->prec != RFB_FP32 || tj != 8 || (i2 != 3 && i2 != 4))) {
        rfb_set_error("the two-rows interior sweep needs an FP32 plan of mode 2 or 3, three launches, 8-row tiles "
                      "and ring depth 3 or 4");
        return -1;
    }
    if (tma >= 2 && !q_fits(e)) {
        rfb_set_error("grid too large for the work-queue sweep (32-bit offsets)");
        return -1;
    }
    if (tma == 4 && (e->g.periodic & 6u)) {
        rfb_set_error("sweep mode 4 (narrow z-slab tiles) needs non-periodic y and z axes");
        return -1;
    }
    FusedPlan &p = e->plan;
    free_plan_lists(p);
    p.tj = tj;
    p.ns = ns;
    p.tma = tma;
    p.seg_int = seg_int;
    p.seg_edge = seg_edge;
    p.uni = tma >= 2 ? uni : 0;
    p.i2 = i2;
    PlanLists pl;
    plan_items(e, active, tj, tma, seg_int, seg_edge, pl, i2);
    p.d = pl.d;
    if (p.uni) {
        // one queue: interior and x-slab items join the slab / boundary
        // items, costliest first (a slab or boundary plane costs about four
        // interior planes)
        for (SweepItem it : pl.vi) it.sub = 5, pl.vq.push_back(it);
        for (SweepItem it : pl.vx) it.sub = 6, pl.vq.push_back(it);
        pl.vi.clear();
        pl.vx.clear();
        // among equal costs, items of one body together (fewer
        // instruction-fetch stalls)
        auto cost = [](const SweepItem &x) { return (x.ie - x.ib) * (x.sub == 5 ? 1 : 4); };
        std::stable_sort(pl.vq.begin(), pl.vq.end(), [&](const SweepItem &x, const SweepItem &y) {
            if (cost(x) != cost(y)) return cost(x) > cost(y);
            return x.sub < y.sub;
        });
    }
    const std::vector<SweepItem> &vi = pl.vi, &ve = pl.ve, &vq = pl.vq, &vx = pl.vx;
    p.n_int = (int)vi.size();
    p.n_edge = (int)ve.size();
    p.n_qe = (int)vq.size();
    p.n_qx = (int)vx.size();
    if (p.n_int) CK(dmalloc(&p.d_int, vi.size() * sizeof(SweepItem)));
    if (p.n_edge) CK(dmalloc(&p.d_edge, ve.size() * sizeof(SweepItem)));
    if (p.n_qe) CK(dmalloc(&p.d_qe, vq.size() * sizeof(SweepItem)));
    if (p.n_qx) CK(dmalloc(&p.d_qx, vx.size() * sizeof(SweepItem)));
    if (p.n_int) CK(cudaMemcpy(p.d_int, vi.data(), vi.size() * sizeof(SweepItem), cudaMemcpyHostToDevice));
    if (p.n_edge) CK(cudaMemcpy(p.d_edge, ve.data(), ve.size() * sizeof(SweepItem), cudaMemcpyHostToDevice));
    if (p.n_qe) CK(cudaMemcpy(p.d_qe, vq.data(), vq.size() * sizeof(SweepItem), cudaMemcpyHostToDevice));
    if (p.n_qx) CK(cudaMemcpy(p.d_qx, vx.data(), vx.size() * sizeof(SweepItem), cudaMemcpyHostToDevice));
    if (tma >= 2 && !p.d_queue) {
        CK(dmalloc(&p.d_queue, 6 * sizeof(int)));
        CK(cudaMemset(p.d_queue, 0, 6 * sizeof(int)));
    }
    if (tma && (p.n_int || p.n_qe || p.n_qx) && build_tma_maps(e, tj) != 0) return -1;
    return 0;
fail:
    return -1;
}

static bool plan_variant_known(int prec, int tj, int ns, int tma) {
    const InteriorVariant *v;
    size_t n;
    if (tma < 0 || tma > 4) return false;
    if (tma >= 2) {
        v = prec == RFB_FP32 ? kQVariantsFp32 : kQVariantsFp64;
        n = prec == RFB_FP32 ? std::size(kQVariantsFp32) : std::size(kQVariantsFp64);
    } else if (prec == RFB_FP32) {
        v = tma ? kTmaVariantsFp32 : kIntVariantsFp32;
        n = tma ? std::size(kTmaVariantsFp32) : std::size(kIntVariantsFp32);
    } else {
        v = tma ? kTmaVariantsFp64 : kIntVariantsFp64;
        n = tma ? std::size(kTmaVariantsFp64) : std::size(kIntVariantsFp64);
    }
    for (size_t q = 0; q < n; q++)
        if (v[q].tj == tj && v[q].ns == ns) return true;
    return false;
}

// ---- autotuner ---------------------------------------------------------------
// Picks the interior variant (rows per tile, ring depth, CTAs per SM) and the
// segment lengths of both work lists by timing a few sweeps of each candidate
// on the engine's own scene; the choice is cached per geometry.  Every
// candidate computes bit-identical fields, so tuning changes speed only.
struct TunedPlan {
    int tj, ns, tma, seg_int, seg_edge, uni, i2;
};

static std::mutex g_tune_mu;
static std::vector<std::pair<std::vector<long long>, TunedPlan>> g_tune_cache;

template <typename T>
static void enqueue_sweep(rfb_engine *e, int par) {
    Args<T> a = engine_args<T>(e, par);
    launch_sweep<T>(e, a, par);
}

static int autotune(rfb_engine *e, int active) {
    const rfb_geom_t &g = e->g;
    std::vector<long long> key = {g.nx, g.ny, g.nz, (long long)g.periodic, e->prec, active, e->cpml.on};
    if (e->cpml.on)
        for (int a = 0; a < 3; a++) {
            key.push_back(e->cpml.eh[a].lo); key.push_back(e->cpml.eh[a].hi);
            key.push_back(e->cpml.em[a].lo); key.push_back(e->cpml.em[a].hi);
        }
    for (int s = 0; s < e->scene.n_skip; s++) key.push_back(e->scene.skip[s]);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (auto &kv : g_tune_cache)
            if (kv.first == key)
                return build_sweep_plan(e, active, kv.second.tj, kv.second.ns, kv.second.tma, kv.second.seg_int,
                                        kv.second.seg_edge, kv.second.uni, kv.second.i2);
    }
    struct Cand {
        InteriorVariant v;
        int tma;
    };
    std::vector<Cand> vars;
    const bool qok = q_fits(e), narrow = qok && !(e->g.periodic & 6u);
    if (e->prec == RFB_FP32) {
        if (qok)
            for (const InteriorVariant &v : kQVariantsFp32) vars.push_back({v, 2}), vars.push_back({v, 3});
        if (narrow)
            for (const InteriorVariant &v : kQVariantsFp32) vars.push_back({v, 4});
        for (const InteriorVariant &v : kTmaVariantsFp32) vars.push_back({v, 1});
        for (const InteriorVariant &v : kIntVariantsFp32) vars.push_back({v, 0});
    } else {
        if (qok)
            for (const InteriorVariant &v : kQVariantsFp64) vars.push_back({v, 2}), vars.push_back({v, 3});
        if (narrow)
            for (const InteriorVariant &v : kQVariantsFp64) vars.push_back({v, 4});
        for (const InteriorVariant &v : kTmaVariantsFp64) vars.push_back({v, 1});
        for (const InteriorVariant &v : kIntVariantsFp64) vars.push_back({v, 0});
    }
    const int segs_int[] = {32, 64, 128};
    const int segs_edge[] = {16, 32};
    TunedPlan best = {vars[0].v.tj, vars[0].v.ns, vars[0].tma, 64, 32, 0, 0};
    float best_ms = 1e30f;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    {
        const long long cells = (long long)g.nx * g.ny * g.nz;
        const int reps = cells > (1 << 22) ? 3 : 6;
        int par = 0;
        for (const Cand &cv : vars)
            for (int si : segs_int)
                for (int se : segs_edge)
                    for (int form = 0; form <= (cv.tma >= 2 ? 3 : 0); form++) {
                        // form 0: three launches; 1: one queue; 2, 3: three
                        // launches, two-rows interior of ring depth 3, 4
                        const InteriorVariant &v = cv.v;
                        const int uni = form == 1, i2 = form >= 2 ? form + 1 : 0;
                        if (i2 && (e->prec != RFB_FP32 || v.tj != 8)) continue;
                        if (build_sweep_plan(e, active, v.tj, v.ns, cv.tma, si, se, uni, i2) != 0) goto fail;
                        for (int w = 0; w < 2; w++) {
                            if (e->prec == RFB_FP64) enqueue_sweep<double>(e, par);
                            else enqueue_sweep<float>(e, par);
                            par ^= 1;
                        }
                        CK(cudaEventRecord(t0, e->stream));
                        for (int w = 0; w < reps; w++) {
                            if (e->prec == RFB_FP64) enqueue_sweep<double>(e, par);
                            else enqueue_sweep<float>(e, par);
                            par ^= 1;
                        }
                        CK(cudaEventRecord(t1, e->stream));
                        CK(cudaEventSynchronize(t1));
                        float ms = 0.f;
                        CK(cudaEventElapsedTime(&ms, t0, t1));
                        if (ms < best_ms) {
                            best_ms = ms;
                            best = TunedPlan{v.tj, v.ns, cv.tma, si, se, uni, i2};
                        }
                    }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache.push_back({key, best});
    }
    if (build_sweep_plan(e, active, best.tj, best.ns, best.tma, best.seg_int, best.seg_edge, best.uni, best.i2) != 0)
        return -1;
    {
        // a timed-out copy during tuning would have left the error flag set
        int err = 0;
        CK(cudaMemcpy(&err, e->d_err, sizeof err, cudaMemcpyDeviceToHost));
        if (err) {
            rfb_set_error("%s", sweep_error_text(err));
            return -1;
        }
    }
    // the tuning sweeps advanced the fields: start from the zero state again
    if (rfb_engine_reset(e) != 0) return -1;
    CK(cudaStreamSynchronize(e->stream));
    return 0;
fail:
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    return -1;
}

extern "C" void rfb_engine_destroy(rfb_engine_t *e) {
    if (!e) return;
    double t_phase = rfb_now();
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (int q = 0; q < 2; q++) {
        if (e->g1[q]) cudaGraphExecDestroy(e->g1[q]);
        if (e->gk[q]) cudaGraphExecDestroy(e->gk[q]);
    }
    rfb_trace("destroy: graphs", t_phase);
    t_phase = rfb_now();
    dfree(e->fld_base);
    devcpml_free(e->cpml);
    devscene_free(e->scene);
    dfree(e->src_val); dfree(e->src_hard);
    dfree(e->probe_cell); dfree(e->probe_comp); dfree(e->ts); dfree(e->d_step); dfree(e->d_err); dfree(e->d_energy); dfree(e->d_iq);
    dfree(e->t3_cells);
    dfree(e->ade_cells);
    dfree(e->list_work);
    dfree(e->d_planes);
    dfree(e->d_plane_part);
    dfree(e->d_plane_count);
    dfree(e->d_fout[0]);
    dfree(e->d_fout[1]);
    dfree(e->d_run_omega);
    dfree(e->d_acc);
    dfree(e->d_omega); dfree(e->d_re); dfree(e->d_im);
    dfree(e->plan.d_int); dfree(e->plan.d_edge); dfree(e->plan.d_qe); dfree(e->plan.d_qx); dfree(e->plan.d_queue);
    dfree(e->tf_inc_e); dfree(e->tf_inc_h); dfree(e->tf_src); dfree(e->tf_h_cell); dfree(e->tf_h_comp);
    dfree(e->tf_h_first); dfree(e->tf_h_count); dfree(e->tf_h_idx); dfree(e->tf_h_coef); dfree(e->tf_h_w);
    dfree(e->tf_e_first); dfree(e->tf_e_count); dfree(e->tf_e_idx); dfree(e->tf_e_coef);
    dfree(e->tf_e_w);
    rfb_trace("destroy: device buffers", t_phase);
    t_phase = rfb_now();
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    if (e->ev_join3) cudaEventDestroy(e->ev_join3);
    if (e->stream2) cudaStreamDestroy(e->stream2);
    if (e->stream3) cudaStreamDestroy(e->stream3);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    rfb_trace("destroy: streams and host state", t_phase);
}

// Cells whose three list entries are 3x3 samples without a source go to the
// per-cell kernel; their entries become kind 5, which the list kernel skips.
static int group_t3_cells(rfb_engine *e, const rfb_scene_image_t *img) {
    const size_t ne = 3 * (size_t)img->n_cells;
    // an E sample outside every CPML slab (the list kernel's e_term is then
    // the plain difference)
    auto outside = [&](int ax, int q) {
        return !e->cpml.on || (q >= e->cpml.em[ax].lo && q < e->cpml.em[ax].hi);
    };
    std::vector<int> cells, ade;
    for (size_t q = 0; q < (size_t)img->n_cells; q++) {
        bool all3 = true, allade = true;
        for (int c = 0; c < 3; c++) {
            all3 &= img->kind[3 * q + c] == RFB_LK_TENSOR3 && img->src[3 * q + c] < 0;
            allade &= img->kind[3 * q + c] == RFB_LK_ADE && img->src[3 * q + c] < 0 && img->aix[3 * q + c] >= 0;
        }
        if (all3) cells.push_back((int)q);
        else if (allade && outside(0, img->cell_ijk[3 * q]) && outside(1, img->cell_ijk[3 * q + 1]) &&
                 outside(2, img->cell_ijk[3 * q + 2]))
            ade.push_back((int)q);
    }
    if (cells.empty() && ade.empty()) return 0;
    e->t3_kinds.assign(img->kind, img->kind + ne);
    std::vector<uint8_t> kinds = e->t3_kinds;
    for (int q : cells)
        for (int c = 0; c < 3; c++) kinds[3 * (size_t)q + c] = RFB_LK_CELL3;
    for (int q : ade)
        for (int c = 0; c < 3; c++) kinds[3 * (size_t)q + c] = RFB_LK_CELLADE;
    if (!cells.empty() && !(e->t3_cells = dev_copy(cells.data(), cells.size()))) {
        rfb_set_error("3x3 cell list upload failed");
        return -1;
    }
    if (!ade.empty() && !(e->ade_cells = dev_copy(ade.data(), ade.size()))) {
        rfb_set_error("dispersive cell list upload failed");
        return -1;
    }
    {
        // the list kernel runs only over the entries left to it
        std::vector<int> work;
        work.reserve(ne - 3 * (cells.size() + ade.size()));
        for (size_t q = 0; q < ne; q++)
            if (kinds[q] != RFB_LK_CELL3 && kinds[q] != RFB_LK_CELLADE) work.push_back((int)q);
        if (!work.empty()) {
            e->list_work = dev_copy(work.data(), work.size());
            if (!e->list_work) {
                rfb_set_error("list work upload failed");
                return -1;
            }
        }
        e->n_list_work = (int)work.size();
    }
    CK(cudaMemcpy(e->scene.l_kind, kinds.data(), ne, cudaMemcpyHostToDevice));
    e->n_t3_cells = (int)cells.size();
    e->t3_host = cells;
    e->n_ade_cells = (int)ade.size();
    e->ade_host = ade;
    return 0;
fail:
    return -1;
}

// Gives every 3x3 cell back to the list kernel (a TF/SF term landed on one).
static int ungroup_t3_cells(rfb_engine *e) {
    if (!e->n_t3_cells && !e->n_ade_cells) return 0;
    CK(cudaMemcpy(e->scene.l_kind, e->t3_kinds.data(), e->t3_kinds.size(), cudaMemcpyHostToDevice));
    e->n_t3_cells = 0;
    e->n_ade_cells = 0;
    dfree(e->list_work);
    e->list_work = nullptr;
    e->n_list_work = 0;
    return 0;
fail:
    return -1;
}

static rfb_engine_t *engine_create(const rfb_geom_t *geom, int precision, int schedule, const rfb_cpml_desc_t *cpml,
                                   const rfb_scene_image_t *scene, size_t n_sources, const rfb_source_desc_t *sources,
                                   size_t n_probes, const rfb_probe_desc_t *probes, size_t n_steps, void *stream,
                                   int member) {
    rfb_engine *e = new rfb_engine();
    e->member = member;
    e->g = *geom;
    e->prec = precision;
    e->sched = schedule;
    e->esz = precision == RFB_FP64 ? 8 : 4;
    e->pitch = pitch_for(geom->nz, e->esz);
    e->total = (size_t)(geom->nx + 1) * (geom->ny + 1) * e->pitch;
    e->nbuf = schedule == RFB_SCHED_FUSED ? 2 : 1;
    e->n_steps = n_steps;
    if (stream) {
        e->stream = (cudaStream_t)stream;
    } else {
        CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = 1;
    }
    double t_phase;
    t_phase = rfb_now();
    {
        // every buffer is a multiple of 128 bytes (whole pitched rows), so
        // the sub-buffers keep the alignment the tensor copies need
        const size_t one = e->total * e->esz;
        CK(dmalloc(&e->fld_base, one * 6 * e->nbuf));
        CK(cudaMemsetAsync(e->fld_base, 0, one * 6 * e->nbuf, e->stream));
        for (int b = 0; b < e->nbuf; b++)
            for (int c = 0; c < 6; c++) e->fld[b][c] = static_cast<char *>(e->fld_base) + (size_t)(6 * b + c) * one;
    }
    rfb_trace("engine: field buffers", t_phase);
    t_phase = rfb_now();
    if (cpml && devcpml_init(e->cpml, geom, cpml, precision, e->pitch, e->nbuf) != 0) goto fail_noset;
    rfb_trace("engine: cpml", t_phase);
    t_phase = rfb_now();
    if (devscene_init(e->scene, geom, scene, precision, e->pitch) != 0) goto fail_noset;
    if (!member && scene && scene->n_cells && group_t3_cells(e, scene) != 0) goto fail_noset;
    rfb_trace("engine: scene upload", t_phase);
    e->n_src = (int)n_sources;
    if (n_sources) {
        std::vector<double> vals(n_sources * n_steps);
        std::vector<int> hard(n_sources);
        for (size_t s = 0; s < n_sources; s++) {
            memcpy(&vals[s * n_steps], sources[s].values, n_steps * sizeof(double));
            hard[s] = sources[s].hard;
        }
        e->src_val = dev_upload_conv(vals.data(), vals.size(), precision);
        e->src_hard = dev_copy(hard.data(), n_sources);
        if (!e->src_val || !e->src_hard) { rfb_set_error("source upload failed"); goto fail_noset; }
    }
    e->n_probes = (int)n_probes;
    if (n_probes) {
        std::vector<long long> cell(n_probes);
        std::vector<int> comp(n_probes);
        for (size_t q = 0; q < n_probes; q++) {
            cell[q] = ((long long)probes[q].i * (geom->ny + 1) + probes[q].j) * e->pitch + probes[q].k;
            comp[q] = probes[q].component;
        }
        e->probe_cell = dev_copy(cell.data(), n_probes);
        e->probe_comp = dev_copy(comp.data(), n_probes);
        CK(dmalloc(&e->ts, n_probes * n_steps * e->esz));
        CK(cudaMemset(e->ts, 0, n_probes * n_steps * e->esz));
        if (!e->probe_cell || !e->probe_comp) { rfb_set_error("probe upload failed"); goto fail_noset; }
    }
    CK(dmalloc(&e->d_step, sizeof(int)));
    CK(cudaMemset(e->d_step, 0, sizeof(int)));
    CK(dmalloc(&e->d_err, sizeof(int)));
    CK(cudaMemset(e->d_err, 0, sizeof(int)));
    if (schedule == RFB_SCHED_FUSED) {
        if (fused_prepare() != 0) {
            rfb_set_error("cannot configure the sweep kernels' shared memory");
            goto fail_noset;
        }
        int active = 0;
        for (size_t s = 0; s < n_sources; s++) {
            if ((sources[s].i == geom->nx && !(geom->periodic & 1u)) ||
                (sources[s].j == geom->ny && !(geom->periodic & 2u)) ||
                (sources[s].k == geom->nz && !(geom->periodic & 4u)))
                active = 1;
        }
        e->active = active;
        if (member) {
            // a batch scene: the batch builds the plans and owns the streams
            if (tma_prepare() != 0 || q_prepare() != 0 || qi2_prepare() != 0) {
                rfb_set_error("cannot configure the TMA sweep kernels' shared memory");
                goto fail_noset;
            }
            goto created;
        }
        CK(cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&e->stream3, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_join3, cudaEventDisableTiming));
        if (tma_prepare() != 0 || q_prepare() != 0 || qi2_prepare() != 0) {
            rfb_set_error("cannot configure the TMA sweep kernels' shared memory");
            goto fail_noset;
        }
        // plan: "tj,ns,seg_interior,seg_edge[,mode[,single_queue[,i2]]]" from RFSYN_FDTD_PLAN,
        // the autotuner (default) or, with RFSYN_FDTD_TUNE=0, the first
        // TMA variant
        const char *ov = rfb_plan_override();
        int a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0;
        int rc;
        const int nov = ov ? sscanf(ov, "%d,%d,%d,%d,%d,%d,%d", &a1, &a2, &a3, &a4, &a5, &a6, &a7) : 0;
        if (nov >= 4 && a3 > 0 && a4 > 0 && plan_variant_known(precision, a1, a2, nov >= 5 ? a5 : 0) &&
            (a6 == 0 || (a6 == 1 && a5 >= 2)))
            rc = build_sweep_plan(e, active, a1, a2, nov >= 5 ? a5 : 0, a3, a4, a6, a7);
        else if (ov)
            rc = (rfb_set_error("sweep plan \"%s\" names no sweep variant", ov), -1);
        else if (!rfb_tune_enabled())
            rc = build_sweep_plan(e, active, precision == RFB_FP32 ? kTmaVariantsFp32[0].tj : kTmaVariantsFp64[0].tj,
                                  precision == RFB_FP32 ? kTmaVariantsFp32[0].ns : kTmaVariantsFp64[0].ns, 1, 64,
                                  32);
        else {
            const double t_tune = rfb_now();
            rc = autotune(e, active);
            rfb_trace("engine: plan (autotune or cached)", t_tune);
        }
        if (rc != 0) goto fail_noset;
    }
created:
    CK(cudaDeviceSynchronize());
    e->launches_per_step = count_step_launches(e);
    if (scene) {
        const size_t ne = 3 * scene->n_cells;
        e->h2d_bytes += (scene->codes ? (size_t)(geom->nx + 1) * (geom->ny + 1) * (geom->nz + 1) : 0) +
                        2 * 256 * e->esz + 3 * scene->n_cells * 4 + ne * (1 + 2 * e->esz + 3 * 4) +
                        scene->n_tensors * (6 * e->esz + 25 * 4) + scene->n_ade * RFB_ADE_NC * e->esz;
        for (size_t q = 0; q < ne; q++)
            if (scene->kind[q] == RFB_LK_ADE) e->n_ade++;
    }
    e->h2d_bytes += n_sources * n_steps * e->esz + n_probes * 12;
    if (cpml)
        e->h2d_bytes += 6 * e->esz * ((size_t)geom->nx + geom->ny + geom->nz + 3);
    return e;
fail:
fail_noset:
    rfb_engine_destroy(e);
    return nullptr;
}

extern "C" rfb_engine_t *rfb_engine_create(const rfb_geom_t *geom, int precision, int schedule,
                                           const rfb_cpml_desc_t *cpml, const rfb_scene_image_t *scene,
                                           size_t n_sources, const rfb_source_desc_t *sources, size_t n_probes,
                                           const rfb_probe_desc_t *probes, size_t n_steps, void *stream) {
    arm_alloc_failure(true);
    rfb_engine_t *e = engine_create(geom, precision, schedule, cpml, scene, n_sources, sources, n_probes, probes,
                                    n_steps, stream, 0);
    arm_alloc_failure(false);
    return e;
}

extern "C" rfb_engine_t *rfb_engine_create_member(const rfb_geom_t *geom, int precision,
                                                  const rfb_cpml_desc_t *cpml, const rfb_scene_image_t *scene,
                                                  size_t n_sources, const rfb_source_desc_t *sources,
                                                  size_t n_probes, const rfb_probe_desc_t *probes, size_t n_steps,
                                                  void *stream) {
    if (!stream) {
        rfb_set_error("a batch scene needs the batch's stream");
        return nullptr;
    }
    return engine_create(geom, precision, RFB_SCHED_FUSED, cpml, scene, n_sources, sources, n_probes, probes,
                         n_steps, stream, 1);
}

extern "C" int rfb_engine_set_tfsf(rfb_engine_t *e, const rfb_tfsf_desc_t *d) {
    if (e->tf_on || e->member) {
        rfb_set_error("a plane wave is attached once, to a session");
        return -1;
    }
    const int prec = e->prec;
    const size_t ne = 3 * (size_t)e->scene.n_cells;
    const rfb_geom_t &g = e->g;
    std::vector<long long> cell(d->n_h);
    std::vector<int> comp(d->n_h);
    for (size_t q = 0; q < d->n_h; q++) {
        cell[q] = ((long long)d->h_ijkc[4 * q] * (g.ny + 1) + d->h_ijkc[4 * q + 1]) * e->pitch + d->h_ijkc[4 * q + 2];
        comp[q] = d->h_ijkc[4 * q + 3];
    }
    // a 3x3 or dispersive cell that carries a TF/SF E term stays with the
    // list kernel
    if ((e->n_t3_cells || e->n_ade_cells) && d->entry_first) {
        bool hit = false;
        for (int q : e->t3_host)
            for (int c = 0; c < 3; c++) hit |= d->entry_first[3 * (size_t)q + c] >= 0;
        for (int q : e->ade_host)
            for (int c = 0; c < 3; c++) hit |= d->entry_first[3 * (size_t)q + c] >= 0;
        if (hit && ungroup_t3_cells(e) != 0) goto fail;
    }
    e->tf_m_len = (int)d->m_len;
    e->tf_ce = d->ce;
    e->tf_ch = d->ch;
    e->tf_n_h = (int)d->n_h;
    CK(dmalloc(&e->tf_inc_e, d->m_len * e->esz));
    CK(dmalloc(&e->tf_inc_h, d->m_len * e->esz));
    CK(cudaMemset(e->tf_inc_e, 0, d->m_len * e->esz));
    CK(cudaMemset(e->tf_inc_h, 0, d->m_len * e->esz));
    e->tf_src = dev_upload_conv(d->src, e->n_steps + 1, prec);
    if (!e->tf_src) goto fail;
    if (d->n_h) {
        e->tf_h_cell = dev_copy(cell.data(), d->n_h);
        e->tf_h_comp = dev_copy(comp.data(), d->n_h);
        e->tf_h_first = dev_copy(d->h_first, d->n_h);
        e->tf_h_count = dev_copy(d->h_count, d->n_h);
        e->tf_h_idx = dev_copy(d->h_idx, d->n_hterms);
        e->tf_h_coef = dev_upload_conv(d->h_coef, d->n_hterms, prec);
        e->tf_h_w = dev_upload_conv(d->h_w, 4 * d->n_hterms, prec);
        if (!e->tf_h_cell || !e->tf_h_comp || !e->tf_h_first || !e->tf_h_count || !e->tf_h_idx || !e->tf_h_coef ||
            !e->tf_h_w)
            goto fail;
    }
    if (ne) {
        e->tf_e_first = dev_copy(d->entry_first, ne);
        e->tf_e_count = dev_copy(d->entry_count, ne);
        if (!e->tf_e_first || !e->tf_e_count) goto fail;
    }
    if (d->n_eterms) {
        e->tf_e_idx = dev_copy(d->e_idx, d->n_eterms);
        e->tf_e_coef = dev_upload_conv(d->e_coef, d->n_eterms, prec);
        e->tf_e_w = dev_upload_conv(d->e_w, 4 * d->n_eterms, prec);
        if (!e->tf_e_idx || !e->tf_e_coef || !e->tf_e_w) goto fail;
    }
    e->tf_on = 1;
    // graphs captured before the plane wave would lack its kernels
    for (int q = 0; q < 2; q++) {
        if (e->g1[q]) cudaGraphExecDestroy(e->g1[q]);
        if (e->gk[q]) cudaGraphExecDestroy(e->gk[q]);
        e->g1[q] = e->gk[q] = nullptr;
    }
    e->launches_per_step = count_step_launches(e);
    e->h2d_bytes += (size_t)(e->n_steps + 1) * e->esz + d->n_h * 24 + (d->n_hterms + d->n_eterms) * (5 * e->esz + 4) +
                    ne * 8;
    return 0;
fail:
    rfb_set_error("plane-wave upload failed");
    return -1;
}

extern "C" int rfb_engine_reset(rfb_engine_t *e) {
    CK(cudaMemsetAsync(e->fld_base, 0, e->total * e->esz * 6 * e->nbuf, e->stream));
    if (e->cpml.psi_base) CK(cudaMemsetAsync(e->cpml.psi_base, 0, e->cpml.psi_total, e->stream));
    if (e->scene.ade_s) CK(cudaMemsetAsync(e->scene.ade_s, 0, e->scene.ade_s_bytes, e->stream));
    if (e->tf_on) {
        CK(cudaMemsetAsync(e->tf_inc_e, 0, (size_t)e->tf_m_len * e->esz, e->stream));
        CK(cudaMemsetAsync(e->tf_inc_h, 0, (size_t)e->tf_m_len * e->esz, e->stream));
    }
    if (e->d_acc)
        CK(cudaMemsetAsync(e->d_acc, 0, (size_t)(e->n_probes + e->n_planes) * e->n_freqs * 4 * e->esz, e->stream));
    // the plane gather's counters are zero between launches; a launch cut
    // short by an error would leave them counting
    if (e->d_plane_count) CK(cudaMemsetAsync(e->d_plane_count, 0, (size_t)e->n_planes * sizeof(int), e->stream));
    CK(cudaMemsetAsync(e->d_step, 0, sizeof(int), e->stream));
    e->steps_done = 0;
    e->parity = 0;
    return 0;
fail:
    return -1;
}

// Running-DFT launches per replayed graph (one, after its steps).
static unsigned dft_launches(const rfb_engine *e) { return (e->n_freqs && (e->n_probes + e->n_planes)) ? 1u : 0u; }

extern "C" int rfb_engine_advance(rfb_engine_t *e, size_t n) {
    if (e->steps_done + n > e->n_steps) {
        rfb_set_error("advance past the configured step count (%zu + %zu > %zu)", e->steps_done, n, e->n_steps);
        return -1;
    }
    const int per_parity = e->nbuf == 2 ? 2 : 1;
    while (n > 0) {
        const int par = per_parity == 2 ? e->parity : 0;
        if (n >= (size_t)rfb_engine::CHUNK) {
            if (!e->gk[par] && build_graph(e, par, rfb_engine::CHUNK, &e->gk[par]) != 0) return -1;
            CK(cudaGraphLaunch(e->gk[par], e->stream));
            g_launches += (unsigned long long)rfb_engine::CHUNK * e->launches_per_step + dft_launches(e);
            n -= rfb_engine::CHUNK;
            e->steps_done += rfb_engine::CHUNK;
            // CHUNK is even: parity unchanged
        } else {
            if (!e->g1[par] && build_graph(e, par, 1, &e->g1[par]) != 0) return -1;
            CK(cudaGraphLaunch(e->g1[par], e->stream));
            g_launches += e->launches_per_step + dft_launches(e);
            n -= 1;
            e->steps_done += 1;
            if (per_parity == 2) e->parity ^= 1;
        }
    }
    return 0;
fail:
    return -1;
}

extern "C" int rfb_engine_advance_timed(rfb_engine_t *e, size_t n, double *ms) {
    cudaEvent_t a = nullptr, b = nullptr;
    float t = 0.f;
    int rc = -1;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, e->stream));
    if (rfb_engine_advance(e, n) != 0) goto out;
    CK(cudaEventRecord(b, e->stream));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&t, a, b));
    if (ms) *ms = t;
    rc = 0;
    goto out;
fail:
out:
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return rc;
}

extern "C" int rfb_engine_info(rfb_engine_t *e, rfb_engine_info_t *out) {
    out->list_cells = (size_t)e->scene.n_cells;
    out->dispersive = e->n_ade;
    out->h2d_bytes = e->h2d_bytes;
    out->tile_j = e->plan.tj;
    out->seg_len = e->plan.seg_int;
    out->ring_depth = e->plan.ns;
    out->tma = e->plan.tma;
    out->unified = e->plan.uni;
    out->interior_ring2 = e->plan.i2;
    out->seg_edge = e->plan.seg_edge;
    out->interior_items = e->plan.n_int;
    out->edge_items = e->plan.n_edge + e->plan.n_qe + e->plan.n_qx;
    size_t sca = 0;
    if (e->cpml.on) {
        // cells of the swept volume inside the slab of each axis (H profiles)
        const int n[3] = {e->g.nx, e->g.ny, e->g.nz};
        for (int a = 0; a < 3; a++) {
            const size_t others = (size_t)e->g.nx * e->g.ny * e->g.nz / (size_t)n[a];
            sca += (size_t)e->cpml.eh[a].ns * others;
        }
    }
    out->slab_cell_axes = sca;
    return 0;
}

// Launches the step kernels one by one with events around each, outside any
// graph, to attribute GPU time to the sweep and to the list / probe kernels.
template <typename T>
static int time_kernels_t(rfb_engine *e, size_t n, double *sweep_ms, double *other_ms) {
    cudaEvent_t ev[4] = {};
    double sw = 0.0, ot = 0.0;
    int rc = -1;
    for (int q = 0; q < 4; q++) CK(cudaEventCreate(&ev[q]));
    for (size_t s = 0; s < n; s++) {
        const int par = e->nbuf == 2 ? e->parity : 0;
        Args<T> a = engine_args<T>(e, par);
        const rfb_geom_t &g = e->g;
        CK(cudaEventRecord(ev[0], e->stream));
        if (e->sched == RFB_SCHED_FUSED) {
            launch_sweep<T>(e, a, par);
            g_launches += (e->plan.n_int > 0) + (e->plan.n_edge > 0) + (e->plan.n_qe > 0) + (e->plan.n_qx > 0);
        } else {
            dim3 blk(32, 8), grd((g.nz + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nx + 1);
            k_h_split<T><<<grd, blk, 0, e->stream>>>(a);
            k_e_split<T><<<grd, blk, 0, e->stream>>>(a);
            g_launches += 2;
        }
        CK(cudaEventRecord(ev[1], e->stream));
        tf_before_list<T>(e, par);
        launch_list<T>(e, a);
        g_launches += list_launches(e);
        ProbeArgs<T> p;
        p.n = e->n_probes;
        p.cell = e->probe_cell;
        p.comp = e->probe_comp;
        const int out = e->nbuf == 2 ? 1 - par : 0;
        for (int c = 0; c < 6; c++) p.F[c] = (const T *)e->fld[out][c];
        p.ts = (T *)e->ts;
        p.n_steps = (long long)e->n_steps;
        p.d_step = e->d_step;
        launch_plane_gather<T>(e, par);
        k_probe_gather<T><<<1, 128, 0, e->stream>>>(p);
        tf_after_step<T>(e, par);
        launch_dft_run<T>(e, 1);
        g_launches += 1 + (e->tf_on ? 2 + (e->tf_n_h > 0) : 0) + (e->n_planes > 0) + dft_launches(e);
        CK(cudaEventRecord(ev[2], e->stream));
        CK(cudaEventSynchronize(ev[2]));
        float t1 = 0.f, t2 = 0.f;
        CK(cudaEventElapsedTime(&t1, ev[0], ev[1]));
        CK(cudaEventElapsedTime(&t2, ev[1], ev[2]));
        sw += t1;
        ot += t2;
        e->steps_done++;
        if (e->nbuf == 2) e->parity ^= 1;
    }
    *sweep_ms = sw;
    *other_ms = ot;
    rc = 0;
fail:
    for (int q = 0; q < 4; q++)
        if (ev[q]) cudaEventDestroy(ev[q]);
    return rc;
}

// ---- energy audit ------------------------------------------------------------
static int check_sweep_error(rfb_engine *e);

template <typename T>
static void enqueue_energy(rfb_engine *e, double dt, double dx, int x_lo, int x_hi, bool prev) {
    EnergyArgs<T> a;
    memset(&a, 0, sizeof a);
    const int cur = e->nbuf == 2 ? e->parity : 0;
    for (int m = 0; m < 3; m++) {
        a.E[m] = (const T *)e->fld[cur][m];
        a.H[m] = (const T *)e->fld[cur][3 + m];
        a.Ep[m] = prev ? (const T *)e->fld[1 - cur][m] : nullptr;
        a.Hp[m] = prev ? (const T *)e->fld[1 - cur][3 + m] : nullptr;
    }
    a.codes = e->scene.codes;
    a.cb_tab = e->scene.cb64_tab;
    a.n_cells = e->scene.n_cells;
    a.lc_ijk = e->scene.lc_ijk;
    a.cb_list = e->scene.cb64_list;
    a.n_skip = e->scene.n_skip;
    for (int q = 0; q < MAX_SKIP; q++) a.skip[q] = e->scene.skip[q];
    a.nx = e->g.nx;
    a.ny = e->g.ny;
    a.nz = e->g.nz;
    a.pitch = e->pitch;
    a.x_lo = x_lo;
    a.x_hi = x_hi;
    a.dt_over_dx = dt / dx;
    a.partial = e->d_energy;
    k_energy<T><<<EN_BLOCKS, EN_THREADS, 0, e->stream>>>(a);
}

extern "C" int rfb_engine_energy(rfb_engine_t *e, double dt, double dx, int x_lo, int x_hi, double q[RFB_EN_COUNT]) {
    const bool prev = e->nbuf == 2 && e->steps_done > 0;
    if (!e->d_energy) CK(dmalloc(&e->d_energy, (size_t)(EN_BLOCKS + 1) * RFB_EN_COUNT * sizeof(double)));
    if (e->prec == RFB_FP64) enqueue_energy<double>(e, dt, dx, x_lo, x_hi, prev);
    else enqueue_energy<float>(e, dt, dx, x_lo, x_hi, prev);
    k_energy_final<<<1, 32, 0, e->stream>>>(e->d_energy, EN_BLOCKS, pow(dx, 3.0), prev ? 1 : 0,
                                            e->d_energy + (size_t)EN_BLOCKS * RFB_EN_COUNT);
    g_launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q, e->d_energy + (size_t)EN_BLOCKS * RFB_EN_COUNT, RFB_EN_COUNT * sizeof(double),
                       cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return check_sweep_error(e);
fail:
    return -1;
}

extern "C" int rfb_engine_time_kernels(rfb_engine_t *e, size_t n, double *sweep_ms, double *other_ms) {
    if (e->steps_done + n > e->n_steps) {
        rfb_set_error("time_kernels past the configured step count");
        return -1;
    }
    return e->prec == RFB_FP64 ? time_kernels_t<double>(e, n, sweep_ms, other_ms)
                               : time_kernels_t<float>(e, n, sweep_ms, other_ms);
}

// After the stream drained: did a sweep give up on its copies?
static int check_sweep_error(rfb_engine *e) {
    int err = 0;
    CK(cudaMemcpy(&err, e->d_err, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
        rfb_set_error("%s", sweep_error_text(err));
        return -1;
    }
    return 0;
fail:
    return -1;
}

extern "C" int rfb_engine_sync(rfb_engine_t *e) {
    CK(cudaStreamSynchronize(e->stream));
    return check_sweep_error(e);
fail:
    return -1;
}

extern "C" void *rfb_engine_stream(rfb_engine_t *e) { return (void *)e->stream; }
extern "C" size_t rfb_engine_steps_done(rfb_engine_t *e) { return e->steps_done; }
extern "C" int rfb_engine_launches_per_step(rfb_engine_t *e) { return e->launches_per_step; }

// The FDTD stage's signal of one probe, optionally with rfsyn's AWGN, as
// interleaved float I/Q (2 n_steps floats) in host memory.
extern "C" int rfb_engine_read_iq(rfb_engine_t *e, int probe, int noise, double snr_linear, unsigned long long seed,
                                  unsigned long long stream, float *out) {
    const long long n = (long long)e->n_steps;
    if (probe < 0 || probe >= e->n_probes + e->n_planes || !out) {
        rfb_set_error("read_iq: no probe %d", probe);
        return -1;
    }
    // samples, then the noise scale in an 8-byte slot at float offset 2 n + 2
    if (!e->d_iq) CK(dmalloc(&e->d_iq, (size_t)(2 * n + 4) * sizeof(float)));
    {
        double *d_std = noise ? reinterpret_cast<double *>(e->d_iq + 2 * n + 2) : nullptr;
        const size_t off = (size_t)probe * (size_t)n * e->esz;
        const unsigned blocks = (unsigned)((n + 255) / 256);
        if (e->prec == RFB_FP64) {
            const double *x = reinterpret_cast<const double *>(reinterpret_cast<const char *>(e->ts) + off);
            if (noise) k_iq_power<double><<<1, 1, 0, e->stream>>>(x, n, snr_linear, d_std);
            k_iq_noise<double><<<blocks, 256, 0, e->stream>>>(x, n, d_std, seed, stream, e->d_iq);
        } else {
            const float *x = reinterpret_cast<const float *>(reinterpret_cast<const char *>(e->ts) + off);
            if (noise) k_iq_power<float><<<1, 1, 0, e->stream>>>(x, n, snr_linear, d_std);
            k_iq_noise<float><<<blocks, 256, 0, e->stream>>>(x, n, d_std, seed, stream, e->d_iq);
        }
        g_launches += 1 + (noise ? 1 : 0);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, e->d_iq, (size_t)(2 * n) * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
        CK(cudaStreamSynchronize(e->stream));
        if (check_sweep_error(e) != 0) return -1;
    }
    return 0;
fail:
    return -1;
}

// Failure-path check of the sweeps' bounded wait: one thread arms an mbarrier
// for 16 bytes of a copy that is never issued and waits on it with the given
// cycle limit; the wait gives up, the thread records it and the kernel ends
// (no copy is in flight, so nothing lands after the exit).
__global__ void k_wait_selftest(long long limit, int *status, long long *cycles) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    mbar_expect_tx(&bar, 16);
    const long long t0 = clock64();
    const bool done = mbar_wait_for(&bar, 0, limit);
    *cycles = clock64() - t0;
    *status = done ? 0 : 1;
}

extern "C" int fdtd_b200_selftest_bounded_wait(long long limit_cycles, int *timed_out, long long *cycles) {
    int *d_status = nullptr;
    long long *d_cycles = nullptr;
    int rc = -1;
    if (!timed_out || !cycles || limit_cycles <= 0 || limit_cycles > 4000000000LL) {
        rfb_set_error("selftest: limit must lie in (0, 4e9] cycles");
        return -1;
    }
    if (dmalloc(&d_status, sizeof(int)) != cudaSuccess || dmalloc(&d_cycles, sizeof(long long)) != cudaSuccess) {
        rfb_set_error("selftest: device allocation failed");
        goto out;
    }
    k_wait_selftest<<<1, 32>>>(limit_cycles, d_status, d_cycles);
    g_launches++;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(timed_out, d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(cycles, d_cycles, sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess) {
        rfb_set_error("selftest: %s", cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    rc = 0;
out:
    dfree(d_status);
    dfree(d_cycles);
    return rc;
}

extern "C" int rfb_engine_read_probes(rfb_engine_t *e, double *out) {
    size_t n = (size_t)(e->n_probes + e->n_planes) * e->n_steps;
    if (!n) return 0;
    CK(cudaStreamSynchronize(e->stream));
    if (check_sweep_error(e) != 0) return -1;
    if (e->prec == RFB_FP64) {
        CK(cudaMemcpy(out, e->ts, n * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(n);
        CK(cudaMemcpy(tmp.data(), e->ts, n * 4, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < n; q++) out[q] = tmp[q];
    }
    return 0;
fail:
    return -1;
}

// Plane probes (axis 0..2, index, component 0..5 of ex..hz): their series
// follow the point probes'.  Before the first step only.
extern "C" int rfb_engine_set_planes(rfb_engine_t *e, size_t n, const int *axis_index_comp) {
    std::vector<PlaneDesc> pd(n);
    const int nn[3] = {e->g.nx, e->g.ny, e->g.nz};
    const long long st[3] = {(long long)(e->g.ny + 1) * e->pitch, e->pitch, 1};
    const size_t ns = (size_t)e->n_probes + n;
    if (e->steps_done) {
        rfb_set_error("plane probes must be set before the first step");
        return -1;
    }
    for (size_t q = 0; q < n; q++) {
        const int a = axis_index_comp[3 * q], idx = axis_index_comp[3 * q + 1], c = axis_index_comp[3 * q + 2];
        if (a < 0 || a > 2 || idx < 0 || idx > nn[a] || c < 0 || c > 5) {
            rfb_set_error("plane probe %zu: axis %d, index %d, component %d out of range", q, a, idx, c);
            return -1;
        }
        const int u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
        pd[q] = PlaneDesc{(long long)idx * st[a], st[u], st[v], nn[u], nn[v], c};
    }
    for (int q = 0; q < 2; q++) {
        if (e->g1[q]) cudaGraphExecDestroy(e->g1[q]);
        if (e->gk[q]) cudaGraphExecDestroy(e->gk[q]);
        e->g1[q] = e->gk[q] = nullptr;
    }
    dfree(e->d_planes);
    dfree(e->d_plane_part);
    dfree(e->d_plane_count);
    e->d_planes = nullptr;
    e->d_plane_part = nullptr;
    e->d_plane_count = nullptr;
    e->n_planes = 0;
    e->plane_chunks = 0;
    if (n) {
        e->d_planes = dev_copy(pd.data(), n);
        if (!e->d_planes) {
            rfb_set_error("plane probe upload failed");
            return -1;
        }
        for (size_t q = 0; q < n; q++) {
            const long long npts = (long long)pd[q].nu * pd[q].nv;
            e->plane_chunks = std::max(e->plane_chunks, (int)((npts + kPlaneChunk - 1) / kPlaneChunk));
        }
        if (dmalloc(&e->d_plane_part, n * e->plane_chunks * sizeof(double)) != cudaSuccess ||
            dmalloc(&e->d_plane_count, n * sizeof(int)) != cudaSuccess ||
            cudaMemset(e->d_plane_count, 0, n * sizeof(int)) != cudaSuccess) {
            rfb_set_error("plane probe upload failed");
            return -1;
        }
        for (int b = 0; b < e->nbuf; b++) {
            void *ptrs[6];
            for (int c = 0; c < 6; c++) ptrs[c] = e->fld[e->nbuf == 2 ? b : 0][c];
            dfree(e->d_fout[b]);
            e->d_fout[b] = dev_copy(ptrs, 6);
            if (!e->d_fout[b]) {
                rfb_set_error("plane probe upload failed");
                return -1;
            }
        }
        if (e->nbuf == 1) e->d_fout[1] = nullptr;
        // the pass over stored series sizes its buffers by the series count
        dfree(e->d_omega); dfree(e->d_re); dfree(e->d_im);
        e->d_omega = e->d_re = e->d_im = nullptr;
        e->dft_cap = 0;
        // series of every probe, point and plane
        dfree(e->ts);
        e->ts = nullptr;
        CK(dmalloc(&e->ts, ns * e->n_steps * e->esz));
        CK(cudaMemset(e->ts, 0, ns * e->n_steps * e->esz));
    }
    e->n_planes = (int)n;
    e->launches_per_step = count_step_launches(e);
    if (e->n_freqs) {
        // the sums follow the series: resize them
        std::vector<double> f = e->dft_freqs;
        return rfb_engine_set_dft(e, f.size(), f.data(), e->dft_t_off);
    }
    return 0;
fail:
    return -1;
}

// Bins of the running DFT (Hz) and the time offset of sample n, t = (n +
// t_off) dt.  Before the first step only; 0 bins: no running DFT.
extern "C" int rfb_engine_set_dft(rfb_engine_t *e, size_t n_freqs, const double *freqs_hz, double t_offset_steps) {
    const size_t ns = (size_t)e->n_probes + e->n_planes;
    if (e->steps_done) {
        rfb_set_error("DFT bins must be set before the first step");
        return -1;
    }
    for (int q = 0; q < 2; q++) {
        if (e->g1[q]) cudaGraphExecDestroy(e->g1[q]);
        if (e->gk[q]) cudaGraphExecDestroy(e->gk[q]);
        e->g1[q] = e->gk[q] = nullptr;
    }
    dfree(e->d_run_omega);
    dfree(e->d_acc);
    e->d_run_omega = nullptr;
    e->d_acc = nullptr;
    e->n_freqs = 0;
    e->dft_freqs.assign(freqs_hz, freqs_hz + n_freqs);
    e->dft_t_off = t_offset_steps;
    if (n_freqs && ns) {
        std::vector<double> om(n_freqs);
        for (size_t f = 0; f < n_freqs; f++) om[f] = 2.0 * 3.14159265358979323846 * freqs_hz[f];
        e->d_run_omega = dev_copy(om.data(), n_freqs);
        if (!e->d_run_omega) {
            rfb_set_error("DFT bin upload failed");
            return -1;
        }
        CK(dmalloc(&e->d_acc, ns * n_freqs * 4 * e->esz));
        CK(cudaMemset(e->d_acc, 0, ns * n_freqs * 4 * e->esz));
        e->n_freqs = (int)n_freqs;
    }
    return 0;
fail:
    return -1;
}

// The running sums, accumulated with the steps.
static int read_running_dft(rfb_engine *e, size_t nout, double *out_re, double *out_im) {
    CK(cudaStreamSynchronize(e->stream));
    if (check_sweep_error(e) != 0) return -1;
    if (e->prec == RFB_FP64) {
        std::vector<double> acc(2 * nout);
        CK(cudaMemcpy(acc.data(), e->d_acc, 2 * nout * sizeof(double), cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < nout; q++) {
            out_re[q] = acc[2 * q];
            out_im[q] = acc[2 * q + 1];
        }
    } else {
        std::vector<float> acc(4 * nout);
        CK(cudaMemcpy(acc.data(), e->d_acc, 4 * nout * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < nout; q++) {
            out_re[q] = acc[4 * q];
            out_im[q] = acc[4 * q + 1];
        }
    }
    return 0;
fail:
    return -1;
}

extern "C" int rfb_engine_probe_dft(rfb_engine_t *e, size_t n_freqs, const double *freqs_hz, double t_offset_steps,
                                    double *out_re, double *out_im) {
    const size_t n_series = (size_t)e->n_probes + e->n_planes;
    if (!n_series || !n_freqs) return 0;
    if ((size_t)e->n_freqs == n_freqs && e->dft_t_off == t_offset_steps &&
        memcmp(e->dft_freqs.data(), freqs_hz, n_freqs * sizeof(double)) == 0)
        return read_running_dft(e, n_series * n_freqs, out_re, out_im);
    // other bins: a pass over the stored series
    std::vector<double> om(n_freqs);
    const size_t nout = n_series * n_freqs;
    for (size_t f = 0; f < n_freqs; f++) om[f] = 2.0 * 3.14159265358979323846 * freqs_hz[f];
    if (e->dft_cap < n_freqs || !e->d_re) {
        dfree(e->d_omega); dfree(e->d_re); dfree(e->d_im);
        e->d_omega = e->d_re = e->d_im = nullptr;
        CK(dmalloc(&e->d_omega, n_freqs * 8));
        CK(dmalloc(&e->d_re, nout * 8));
        CK(dmalloc(&e->d_im, nout * 8));
        e->dft_cap = n_freqs;
    }
    CK(cudaMemcpyAsync(e->d_omega, om.data(), n_freqs * 8, cudaMemcpyHostToDevice, e->stream));
    {
        dim3 grd((unsigned)((n_freqs + 127) / 128), (unsigned)n_series);
        if (e->prec == RFB_FP64)
            k_probe_dft<double><<<grd, 128, 0, e->stream>>>((const double *)e->ts, (long long)e->n_steps, (int)n_series,
                                                            (int)e->steps_done, (int)n_freqs, e->d_omega, e->g.dt,
                                                            t_offset_steps, e->d_re, e->d_im);
        else
            k_probe_dft<float><<<grd, 128, 0, e->stream>>>((const float *)e->ts, (long long)e->n_steps, (int)n_series,
                                                           (int)e->steps_done, (int)n_freqs, e->d_omega, e->g.dt,
                                                           t_offset_steps, e->d_re, e->d_im);
        g_launches++;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out_re, e->d_re, nout * 8, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(out_im, e->d_im, nout * 8, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return 0;
fail:
    return -1;
}

extern "C" int rfb_engine_read_field(rfb_engine_t *e, int component, double *host) {
    const rfb_geom_t &g = e->g;
    const int buf = e->nbuf == 2 ? e->parity : 0;
    const size_t rows = (size_t)(g.nx + 1) * (g.ny + 1);
    CK(cudaStreamSynchronize(e->stream));
    if (check_sweep_error(e) != 0) return -1;
    if (e->prec == RFB_FP64) {
        CK(cudaMemcpy2D(host, (g.nz + 1) * 8, e->fld[buf][component], e->pitch * 8, (g.nz + 1) * 8, rows,
                        cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(rows * (g.nz + 1));
        CK(cudaMemcpy2D(tmp.data(), (g.nz + 1) * 4, e->fld[buf][component], e->pitch * 4, (g.nz + 1) * 4, rows,
                        cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < tmp.size(); q++) host[q] = tmp[q];
    }
    return 0;
fail:
    return -1;
}

// ---------------------------------------------------------------------------
// Sphere fill fractions (FP64 subpixel construction on the GPU)
// ---------------------------------------------------------------------------
__global__ void k_sphere_fractions(double cx, double cy, double cz, double r, int i0, int j0, int k0, int ni, int nj,
                                   int nk, double *f, double *n2) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncell = (long long)ni * nj * nk;
    if (t >= 3 * ncell) return;
    const long long cell = t / 3;
    const int comp = (int)(t - 3 * cell);
    const int k = k0 + (int)(cell % nk);
    const int j = j0 + (int)((cell / nk) % nj);
    const int i = i0 + (int)(cell / ((long long)nk * nj));
    double p[3];
    rfb_sample_pos(i, j, k, comp, p);
    double nrm[3];
    f[t] = rfb_sphere_cube_fraction(p, cx, cy, cz, r, nrm);
    n2[t] = __dmul_rn(nrm[comp], nrm[comp]);
}

// Sphere set-up runs once per sphere of every scene (tens of thousands of
// calls when a batch of scenes is built): the device results and their
// pinned host staging are kept per device and grown on demand, so a call is
// one launch, two copies and one synchronisation.
namespace {
struct FracScratch {
    double *dev = nullptr, *host = nullptr;
    size_t cap = 0;  // doubles per output
};
std::mutex g_frac_mu;
FracScratch g_frac[64];
}  // namespace

extern "C" int rfb_sphere_fractions(const double centre[3], double radius, int i0, int j0, int k0, int ni, int nj,
                                    int nk, double *f, double *n2) {
    const size_t n = 3 * (size_t)ni * nj * nk;
    int rc = -1, dev = 0;
    if (!n) return 0;
    std::lock_guard<std::mutex> lock(g_frac_mu);
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        rfb_set_error("sphere fractions: device index %d out of range", dev);
        return -1;
    }
    {
        FracScratch &s = g_frac[dev];
        if (s.cap < n) {
            dfree(s.dev);
            cudaFreeHost(s.host);
            s.dev = nullptr;
            s.host = nullptr;
            s.cap = 0;
            const size_t want = std::max(n, (size_t)1 << 18);
            CK(dmalloc(&s.dev, 2 * want * sizeof(double)));
            CK(cudaMallocHost(&s.host, 2 * want * sizeof(double)));
            s.cap = want;
        }
        k_sphere_fractions<<<(unsigned)((n + 255) / 256), 256>>>(centre[0], centre[1], centre[2], radius, i0, j0, k0,
                                                                 ni, nj, nk, s.dev, s.dev + s.cap);
        g_launches++;
        CK(cudaGetLastError());
        CK(cudaMemcpy(s.host, s.dev, n * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(s.host + s.cap, s.dev + s.cap, n * 8, cudaMemcpyDeviceToHost));
        memcpy(f, s.host, n * 8);
        memcpy(n2, s.host + s.cap, n * 8);
    }
    rc = 0;
fail:
    return rc;
}

// ---------------------------------------------------------------------------
// Step-wise API: FP64 device mirror of a host grid.
// ---------------------------------------------------------------------------
struct rfb_fields {
    rfb_geom_t g;
    long long pitch;
    size_t total;
    double *f[6] = {};
    cudaStream_t stream = nullptr;
};
struct rfb_cpml_dev {
    DevCpml c;
    int nx, ny, nz;
};
struct rfb_scene_dev {
    DevScene s;
};

// The step-wise API keeps rfsyn's own unpadded layout (pitch nz+1) on the
// device, so each host array moves with one contiguous copy.
static long long step_pitch(int nz) { return nz + 1; }

extern "C" rfb_fields_t *rfb_fields_create(const rfb_geom_t *geom) {
    rfb_fields *f = new rfb_fields();
    f->g = *geom;
    f->pitch = step_pitch(geom->nz);
    f->total = (size_t)(geom->nx + 1) * (geom->ny + 1) * f->pitch;
    CK(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
    for (int c = 0; c < 6; c++) CK(dmalloc(&f->f[c], f->total * 8));
    return f;
fail:
    rfb_fields_destroy(f);
    return nullptr;
}

extern "C" void rfb_fields_destroy(rfb_fields_t *f) {
    if (!f) return;
    for (int c = 0; c < 6; c++) dfree(f->f[c]);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

extern "C" rfb_cpml_dev_t *rfb_cpml_dev_create(const rfb_geom_t *geom, const rfb_cpml_desc_t *desc) {
    rfb_cpml_dev *c = new rfb_cpml_dev();
    c->nx = geom->nx; c->ny = geom->ny; c->nz = geom->nz;
    if (devcpml_init(c->c, geom, desc, RFB_FP64, step_pitch(geom->nz), 1) != 0) {
        devcpml_free(c->c);
        delete c;
        return nullptr;
    }
    return c;
}
extern "C" void rfb_cpml_dev_destroy(rfb_cpml_dev_t *c) {
    if (!c) return;
    devcpml_free(c->c);
    delete c;
}
extern "C" rfb_scene_dev_t *rfb_scene_dev_create(const rfb_geom_t *geom, const rfb_scene_image_t *img) {
    rfb_scene_dev *s = new rfb_scene_dev();
    if (devscene_init(s->s, geom, img, RFB_FP64, step_pitch(geom->nz)) != 0) {
        devscene_free(s->s);
        delete s;
        return nullptr;
    }
    return s;
}
extern "C" void rfb_scene_dev_destroy(rfb_scene_dev_t *s) {
    if (!s) return;
    devscene_free(s->s);
    delete s;
}

static int fields_xfer(rfb_fields *f, double *const host[6], int first, int count, bool up) {
    const rfb_geom_t &g = f->g;
    const size_t rows = (size_t)(g.nx + 1) * (g.ny + 1);
    const size_t bytes = rows * (size_t)(g.nz + 1) * 8;
    for (int c = first; c < first + count; c++) {
        if (up) CK(cudaMemcpyAsync(f->f[c], host[c], bytes, cudaMemcpyHostToDevice, f->stream));
        else CK(cudaMemcpyAsync(host[c], f->f[c], bytes, cudaMemcpyDeviceToHost, f->stream));
    }
    return 0;
fail:
    return -1;
}

static Args<double> step_args(rfb_fields *f, const rfb_geom_t *geom) {
    Args<double> a;
    memset(&a, 0, sizeof a);
    fill_geom_args(a, geom, f->pitch);
    for (int c = 0; c < 3; c++) {
        a.E[c] = a.Eo[c] = f->f[c];
        a.H[c] = a.Ho[c] = f->f[3 + c];
    }
    return a;
}

extern "C" int rfb_step_update_h(rfb_fields_t *f, const rfb_geom_t *geom, rfb_cpml_dev_t *cpml,
                                 double *const host[6]) {
    f->g = *geom;
    Args<double> a = step_args(f, geom);
    if (cpml) fill_cpml_args(a, cpml->c, 0, 0);
    dim3 blk(32, 8), grd((geom->nz + 1 + 31) / 32, (geom->ny + 1 + 7) / 8, geom->nx + 1);
    if (fields_xfer(f, host, 0, 6, true)) return -1;
    k_h_split<double><<<grd, blk, 0, f->stream>>>(a);
    g_launches++;
    CK(cudaGetLastError());
    if (fields_xfer(f, host, 3, 3, false)) return -1;
    CK(cudaStreamSynchronize(f->stream));
    return 0;
fail:
    return -1;
}

extern "C" int rfb_step_update_e(rfb_fields_t *f, const rfb_geom_t *geom, rfb_cpml_dev_t *cpml,
                                 rfb_scene_dev_t *scene, double vacuum_cb, double *const host[6]) {
    f->g = *geom;
    Args<double> a = step_args(f, geom);
    if (cpml) fill_cpml_args(a, cpml->c, 0, 0);
    DevScene vac;
    double *vca = nullptr, *vcb = nullptr;
    if (scene) {
        fill_scene_args(a, scene->s);
    } else {
        // vacuum table: Ca = 1, Cb = dt/(eps0 dx) (grid.c:92-118)
        double one = 1.0;
        vca = dev_copy(&one, 1);
        vcb = dev_copy(&vacuum_cb, 1);
        if (!vca || !vcb) { rfb_set_error("vacuum table upload failed"); dfree(vca); dfree(vcb); return -1; }
        a.tca = vca;
        a.tcb = vcb;
    }
    dim3 blk(32, 8), grd((geom->nz + 1 + 31) / 32, (geom->ny + 1 + 7) / 8, geom->nx + 1);
    int rc = -1;
    if (fields_xfer(f, host, 0, 6, true)) goto out;
    k_e_split<double><<<grd, blk, 0, f->stream>>>(a);
    g_launches++;
    if (a.n_cells) {
        // the step-wise list carries no sources: d_step is unused
        k_e_list<double><<<(3 * a.n_cells + 255) / 256, 256, 0, f->stream>>>(a);
        g_launches++;
    }
    if (cudaGetLastError() != cudaSuccess) { rfb_set_error("E update launch failed"); goto out; }
    if (fields_xfer(f, host, 0, 3, false)) goto out;
    if (cudaStreamSynchronize(f->stream) != cudaSuccess) { rfb_set_error("E update failed"); goto out; }
    rc = 0;
out:
    cudaStreamSynchronize(f->stream);
    dfree(vca);
    dfree(vcb);
    (void)vac;
    return rc;
}

#include "batch.cuh"
