// batch.cuh -- many independent scenes advanced together (included by
// engine.cu after the single-scene engine).
//
// rfsyn runs its examples one at a time (cli/main.c:362-417); a scene of a
// few hundred thousand cells cannot fill a B200, and each of its steps pays
// the launch latency of four kernels.  A batch keeps every scene resident in
// its own buffers (an engine created as a batch member: fields, slab psi,
// codes, interface list, sources, probes) and advances all of them with the
// same launches per step:
//   k_sweep_qb<KIND 0, 1> and k_sweep_qb<KIND 2> -- the work-queue sweeps of
//     sweep.cuh over queues of (scene, tile, plane range) items of every
//     scene, or with the single-queue plan one k_sweep_qb<KIND 5> over every
//     item; a CTA switching scenes copies the scene's parameters (Args) and
//     (Ca, Cb) table into shared memory;
//   k_e_list_b -- the interface-list entries of every scene, one block per
//     256 entries of one scene;
//   k_probe_gather_b -- every probe of every scene, then the shared step
//     counter.
// Steps are captured in CUDA graphs (16 steps per graph), and the tile
// height, ring depth, tile origins and segment lengths are chosen by timing
// candidate plans on the batch itself.  Scenes whose tile halos would wrap
// around a periodic y or z axis are not admitted (their tiles need the
// cp.async edge sweep, which takes one scene per launch).
#pragma once

namespace rfb {

struct BatchItem {
    int scene;
    SweepItem t;
};

// Copies one scene's Args into the CTA's shared copy (32-bit words).
template <typename T>
__device__ __forceinline__ void load_args(Args<T> &dst, const Args<T> *src, int nthreads, int tid) {
    const unsigned *s = reinterpret_cast<const unsigned *>(src);
    unsigned *d = reinterpret_cast<unsigned *>(&dst);
    for (int t = tid; t < (int)(sizeof(Args<T>) / 4); t += nthreads) d[t] = s[t];
}

// Tensor maps written by the host before the launch are read through the
// tensormap proxy: order the generic-proxy copy before their first use.
__device__ __forceinline__ void tensormap_acquire(const TmaMaps *m) {
    const CUtensorMap *maps[14] = {&m->e[0],  &m->e[1],  &m->e[2],  &m->h[0],  &m->h[1],  &m->h[2],  &m->code,
                                   &m->en[0], &m->en[1], &m->en[2], &m->hn[0], &m->hn[1], &m->hn[2], &m->coden};
#pragma unroll
    for (int q = 0; q < 14; q++)
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(maps[q]) : "memory");
}

// Dynamic shared memory of the batched sweep: the single-scene layout, then
// the CTA's copy of the current scene's parameters.  No static shared
// memory: it would precede the dynamic region and break the 128-byte
// alignment the tensor copies need.
template <typename T, int TJ, int NS>
struct QBLayout {
    static constexpr size_t args = round128(QLayout<T, TJ, NS>::total);
    static constexpr size_t total = args + sizeof(Args<T>);
};

template <typename T, int TJ, int NS, int MINB, int KIND>
__global__ void __launch_bounds__(32 * TJ, MINB)
    k_sweep_qb(const Args<T> *args, const FusedDims *dims, const TmaMaps *maps, const BatchItem *items, int n_items,
               int *queue, int *err) {
    static_assert(NS >= 3, "the ring must hold the current, the next and one prefetched plane");
    static_assert(TJ >= 5, "warps 0-3 share the halo recomputation, warp 4 issues the copies");
    using S = QLayout<T, TJ, NS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (q_misaligned(smem_raw, err)) return;
    Args<T> &sa = *reinterpret_cast<Args<T> *>(smem_raw + QBLayout<T, TJ, NS>::args);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::bars);
    volatile int *s_item = reinterpret_cast<volatile int *>(smem_raw + S::misc);
    const int tid = threadIdx.y * 32 + threadIdx.x;
    q_init_bars<NS>(bars);
    unsigned phase = 0, pending = 0;
    bool failed = false;
    int cur = -1;
    for (;;) {
        if (tid == 0) *s_item = atomicAdd(&queue[0], 1);
        __syncthreads();
        const int w = *s_item;
        if (w >= n_items) break;
        const BatchItem bi = items[w];
        if (bi.scene != cur) {
            load_args(sa, args + bi.scene, 32 * TJ, tid);
            // the fence orders the maps for the thread that issues the copies
            if (tid == kCopyIssueTid) tensormap_acquire(maps + bi.scene);
            __syncthreads();
            q_load_table<T, TJ, NS>(sa, smem_raw);
            __syncthreads();
            cur = bi.scene;
        }
        if (!q_run<T, TJ, NS, KIND>(sa, dims[bi.scene], maps[bi.scene], bi.t, smem_raw, phase, pending, failed)) {
            q_bail<NS>(bars, phase, pending, err);
            break;
        }
        __syncthreads();  // the ring, the tables and the item slot are free again
    }
    q_leave(queue);
}

// Interface-list entries of many scenes: block b updates entries
// blocks[b].y .. +255 of scene blocks[b].x.
template <typename T>
__global__ void __launch_bounds__(256) k_e_list_b(const Args<T> *args, const int2 *blocks) {
    __shared__ Args<T> sa;
    const int2 b = blocks[blockIdx.x];
    load_args(sa, args + b.x, 256, threadIdx.x);
    __syncthreads();
    const int e = b.y + threadIdx.x;
    if (e < 3 * sa.n_cells) e_list_entry(sa, e);
}

template <typename T>
struct ProbeRefB {
    const T *f[2];     // the probed component in field buffer 0 and 1
    long long cell;
    T *ts;             // the probe's time series (n_steps samples)
};

// Records sample n of every probe of every scene from the output buffer of
// the step, then advances the batch's step counter (single block).
template <typename T>
__global__ void k_probe_gather_b(const ProbeRefB<T> *p, int n, int out_buf, long long n_steps, int *d_step) {
    __shared__ int step;
    if (threadIdx.x == 0) step = *d_step;
    __syncthreads();
    if (step < n_steps)
        for (int q = threadIdx.x; q < n; q += blockDim.x) p[q].ts[step] = p[q].f[out_buf][p[q].cell];
    __syncthreads();
    if (threadIdx.x == 0) *d_step = step + 1;
}

// CTAs per SM of the batched sweeps: the interior as in the single-scene
// plan; the FP32 x-slab and edge kinds, which keep the scene's parameters in
// registers loaded from shared memory, at 3 (8-row tiles) or 1 (16-row);
// the FP32 single-queue kind with 8-row tiles at 4 (64 registers, 176 bytes
// of spills, against 80 registers at 3: stalled on waits, barriers and
// instruction fetch, it gains from the extra warps -- C4's step 4.681 ->
// 4.616 ms); FP64 as in the single-scene plan.
#define RFB_QB_MINB(TT, TJ_, MBI_, MBE_, KIND_) \
    ((KIND_) == 0 ? (MBI_) : sizeof(TT) == 8 ? (MBE_) : ((TJ_) == 16 ? 1 : (KIND_) == 5 ? 4 : 3))
#define RFB_LAUNCH_QB(TT, TJ_, NS_, MBI_, MBE_)                                                            \
    if (tj == TJ_ && ns == NS_) {                                                                          \
        constexpr int MB_ = RFB_QB_MINB(TT, TJ_, MBI_, MBE_, KIND);                                                  \
        const int g = std::min(n, qb_grid<TT, TJ_, NS_, MB_, KIND>());                                     \
        k_sweep_qb<TT, TJ_, NS_, MB_, KIND><<<g, dim3(32, TJ_), QBLayout<TT, TJ_, NS_>::total, st>>>(      \
            args, dims, maps, items, n, queue, err);                                                       \
    }

template <typename T, int TJ, int NS, int MINB, int KIND>
inline int qb_grid() {
    static int g = 0;
    if (!g) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweep_qb<T, TJ, NS, MINB, KIND>, 32 * TJ,
                                                      QBLayout<T, TJ, NS>::total);
        g = (sms > 0 ? sms : 148) * (per > 0 ? per : 1);
    }
    return g;
}

template <int KIND, typename T>
inline void launch_qb(const Args<T> *args, const FusedDims *dims, const TmaMaps *maps, int tj, int ns,
                      const BatchItem *items, int n, int *queue, int *err, cudaStream_t st) {
    if (n <= 0) return;
    if constexpr (sizeof(T) == 4) {
        RFB_Q_VARIANTS_FP32(RFB_LAUNCH_QB)
    } else {
        RFB_Q_VARIANTS_FP64(RFB_LAUNCH_QB)
    }
}

#define RFB_PREP_QB(TT, TJ_, NS_, MBI_, MBE_)                                                               \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_qb<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 0), 0>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QBLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_qb<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 1), 1>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QBLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_qb<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 2), 2>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QBLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_qb<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 5), 5>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QBLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess) {                                                                                 \
        (void)qb_grid<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 5), 5>();                                       \
        (void)qb_grid<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 0), 0>();                                       \
        (void)qb_grid<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 1), 1>();                                       \
        (void)qb_grid<TT, TJ_, NS_, RFB_QB_MINB(TT, TJ_, MBI_, MBE_, 2), 2>();                                       \
    }
static inline int qb_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaSuccess;
    RFB_Q_VARIANTS_FP32(RFB_PREP_QB)
    RFB_Q_VARIANTS_FP64(RFB_PREP_QB)
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

}  // namespace rfb

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct rfb_batch {
    std::vector<rfb_engine *> m;  // members (owned)
    int prec = RFB_FP32;
    size_t n_steps = 0, steps_done = 0;
    int parity = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int own_stream = 0;
    int *d_step = nullptr, *d_err = nullptr, *d_queue = nullptr;
    void *d_args[2] = {};          // Args<T>[n] per parity
    FusedDims *d_dims = nullptr;
    TmaMaps *d_maps[2] = {};
    BatchItem *d_items[3] = {};    // interior, x slab, edge (uni: every item in the edge list)
    int n_items[3] = {};
    int uni = 0;
    int2 *d_lblocks = nullptr;
    int n_lblocks = 0;
    void *d_probes = nullptr;
    int n_probes = 0;
    int tj = 8, ns = 4, mode = 2, seg_int = 64, seg_edge = 32;
    size_t cells = 0, list_cells = 0, slab_cell_axes = 0;
    static constexpr int CHUNK = 16;
    cudaGraphExec_t g1[2] = {nullptr, nullptr}, gk[2] = {nullptr, nullptr};
};

static void batch_free_plan(rfb_batch *b) {
    for (int k = 0; k < 3; k++) {
        dfree(b->d_items[k]);
        b->d_items[k] = nullptr;
        b->n_items[k] = 0;
    }
    for (int q = 0; q < 2; q++) {
        if (b->g1[q]) cudaGraphExecDestroy(b->g1[q]);
        if (b->gk[q]) cudaGraphExecDestroy(b->gk[q]);
        b->g1[q] = b->gk[q] = nullptr;
        dfree(b->d_maps[q]);
        b->d_maps[q] = nullptr;
    }
    dfree(b->d_dims);
    b->d_dims = nullptr;
}

// Work lists and per-scene tensor maps / dims of one plan.
static int batch_build_plan(rfb_batch *b, int tj, int ns, int mode, int seg_int, int seg_edge, int uni = 0) {
    batch_free_plan(b);
    b->tj = tj;
    b->ns = ns;
    b->mode = mode;
    b->uni = uni;
    b->seg_int = seg_int;
    b->seg_edge = seg_edge;
    const size_t n = b->m.size();
    std::vector<BatchItem> lists[3];
    std::vector<FusedDims> dims(n);
    std::vector<TmaMaps> maps[2];
    maps[0].resize(n);
    maps[1].resize(n);
    for (size_t s = 0; s < n; s++) {
        rfb_engine *e = b->m[s];
        if (mode == 4 && (e->g.periodic & 6u)) {
            rfb_set_error("batch scene %zu: sweep mode 4 needs non-periodic y and z axes", s);
            return -1;
        }
        PlanLists pl;
        plan_items(e, e->active, tj, mode, seg_int, seg_edge, pl);
        if (!pl.ve.empty()) {
            rfb_set_error("batch scene %zu: a tile halo wraps around a periodic y or z axis", s);
            return -1;
        }
        dims[s] = pl.d;
        for (const SweepItem &it : pl.vi) lists[0].push_back(BatchItem{(int)s, it});
        for (const SweepItem &it : pl.vx) lists[1].push_back(BatchItem{(int)s, it});
        for (const SweepItem &it : pl.vq) lists[2].push_back(BatchItem{(int)s, it});
        if (build_tma_maps(e, tj) != 0) return -1;
        maps[0][s] = e->tmaps[0];
        maps[1][s] = e->tmaps[1];
    }
    if (uni) {
        // one queue for every item (interior sub 5, x slab sub 6)
        for (BatchItem it : lists[0]) it.t.sub = 5, lists[2].push_back(it);
        for (BatchItem it : lists[1]) it.t.sub = 6, lists[2].push_back(it);
        lists[0].clear();
        lists[1].clear();
    }
    for (int k = 0; k < 3; k++) {
        // costliest items first across the whole batch (a slab or boundary
        // plane costs about four interior planes); among equal costs, items
        // of one body together, so that the SMs run few bodies at a time
        // (fewer instruction-fetch stalls: 4 % faster on C4)
        auto cost = [](const BatchItem &x) { return (x.t.ie - x.t.ib) * (x.t.sub == 5 ? 1 : 4); };
        std::stable_sort(lists[k].begin(), lists[k].end(), [&](const BatchItem &x, const BatchItem &y) {
            if (cost(x) != cost(y)) return cost(x) > cost(y);
            return x.t.sub < y.t.sub;
        });
        b->n_items[k] = (int)lists[k].size();
        if (b->n_items[k]) {
            CK(dmalloc(&b->d_items[k], lists[k].size() * sizeof(BatchItem)));
            CK(cudaMemcpy(b->d_items[k], lists[k].data(), lists[k].size() * sizeof(BatchItem),
                          cudaMemcpyHostToDevice));
        }
    }
    CK(dmalloc(&b->d_dims, n * sizeof(FusedDims)));
    CK(cudaMemcpy(b->d_dims, dims.data(), n * sizeof(FusedDims), cudaMemcpyHostToDevice));
    for (int q = 0; q < 2; q++) {
        CK(dmalloc(&b->d_maps[q], n * sizeof(TmaMaps)));
        CK(cudaMemcpy(b->d_maps[q], maps[q].data(), n * sizeof(TmaMaps), cudaMemcpyHostToDevice));
    }
    return 0;
fail:
    return -1;
}

template <typename T>
static void batch_sweep(rfb_batch *b, int par) {
    const Args<T> *args = (const Args<T> *)b->d_args[par];
    const TmaMaps *maps = b->d_maps[par];
    if (b->uni) {
        launch_qb<5, T>(args, b->d_dims, maps, b->tj, b->ns, b->d_items[2], b->n_items[2], b->d_queue + 2, b->d_err,
                        b->stream);
        return;
    }
    cudaEventRecord(b->ev_fork, b->stream);
    cudaStreamWaitEvent(b->stream2, b->ev_fork, 0);
    launch_qb<0, T>(args, b->d_dims, maps, b->tj, b->ns, b->d_items[0], b->n_items[0], b->d_queue, b->d_err,
                    b->stream);
    launch_qb<1, T>(args, b->d_dims, maps, b->tj, b->ns, b->d_items[1], b->n_items[1], b->d_queue + 4, b->d_err,
                    b->stream);
    launch_qb<2, T>(args, b->d_dims, maps, b->tj, b->ns, b->d_items[2], b->n_items[2], b->d_queue + 2, b->d_err,
                    b->stream2);
    cudaEventRecord(b->ev_join, b->stream2);
    cudaStreamWaitEvent(b->stream, b->ev_join, 0);
}

template <typename T>
static void batch_rest(rfb_batch *b, int par) {
    if (b->n_lblocks)
        k_e_list_b<T><<<b->n_lblocks, 256, 0, b->stream>>>((const Args<T> *)b->d_args[par], b->d_lblocks);
    k_probe_gather_b<T><<<1, 1024, 0, b->stream>>>((const ProbeRefB<T> *)b->d_probes, b->n_probes, 1 - par,
                                                   (long long)b->n_steps, b->d_step);
}

static int batch_launches_per_step(const rfb_batch *b) {
    return (b->n_items[0] > 0) + (b->n_items[1] > 0) + (b->n_items[2] > 0) + (b->n_lblocks > 0) + 1;
}

static void batch_enqueue_step(rfb_batch *b, int par) {
    if (b->prec == RFB_FP64) {
        batch_sweep<double>(b, par);
        batch_rest<double>(b, par);
    } else {
        batch_sweep<float>(b, par);
        batch_rest<float>(b, par);
    }
}

static int batch_graph(rfb_batch *b, int par, int steps, cudaGraphExec_t *out) {
    cudaGraph_t graph = nullptr;
    int p = par;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < steps; s++) {
        batch_enqueue_step(b, p);
        p ^= 1;
    }
    CK(cudaStreamEndCapture(b->stream, &graph));
    CK(cudaGraphInstantiate(out, graph, 0));
    cudaGraphDestroy(graph);
    return 0;
fail:
    if (graph) cudaGraphDestroy(graph);
    return -1;
}

extern "C" int rfb_batch_reset(rfb_batch_t *b) {
    for (rfb_engine *e : b->m)
        if (rfb_engine_reset(e) != 0) return -1;
    CK(cudaMemsetAsync(b->d_step, 0, sizeof(int), b->stream));
    b->steps_done = 0;
    b->parity = 0;
    return 0;
fail:
    return -1;
}

// Picks the plan (tile height, ring depth, tile origins, segment lengths) by
// timing a few batched sweeps of each candidate; every candidate computes
// bit-identical fields, so the choice changes speed only.
// Plans chosen for batches of the same scene geometries (in order), so that
// a batch built again -- the next set of examples of a stage, an end-to-end
// run -- skips the tuning.
struct BatchCand {
    int tj, ns, mode, si, se, uni;
};
static std::mutex g_btune_mu;
static std::vector<std::pair<std::vector<long long>, BatchCand>> g_btune_cache;

static std::vector<long long> batch_key(const rfb_batch *b) {
    std::vector<long long> key = {b->prec, (long long)b->m.size()};
    for (const rfb_engine *e : b->m) {
        const rfb_geom_t &g = e->g;
        key.insert(key.end(), {g.nx, g.ny, g.nz, (long long)g.periodic, e->active, e->cpml.on});
        if (e->cpml.on)
            for (int a = 0; a < 3; a++)
                key.insert(key.end(), {e->cpml.eh[a].lo, e->cpml.eh[a].hi, e->cpml.em[a].lo, e->cpml.em[a].hi});
        key.push_back(e->scene.n_skip);
        for (int s = 0; s < e->scene.n_skip; s++) key.push_back(e->scene.skip[s]);
    }
    return key;
}

static int batch_autotune(rfb_batch *b) {
    using Cand = BatchCand;
    std::vector<Cand> cands;
    const InteriorVariant *v = b->prec == RFB_FP32 ? kQVariantsFp32 : kQVariantsFp64;
    const size_t nv = b->prec == RFB_FP32 ? std::size(kQVariantsFp32) : std::size(kQVariantsFp64);
    bool wrap_yz = false;
    for (const rfb_engine *e : b->m) wrap_yz |= (e->g.periodic & 6u) != 0;
    // two stages: variant, tile origins and queue form at (64, 32)-plane
    // items, then the segment lengths of the winner
    for (size_t q = 0; q < nv; q++)
        for (int mode = 2; mode <= (wrap_yz ? 3 : 4); mode++)
            for (int uni : {0, 1}) cands.push_back(Cand{v[q].tj, v[q].ns, mode, 64, 32, uni});
    const char *ov = rfb_plan_override();
    if (ov) {
        int a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
        const int nov = sscanf(ov, "%d,%d,%d,%d,%d,%d", &a1, &a2, &a3, &a4, &a5, &a6);
        if (nov < 5 || a5 < 2 || a3 <= 0 || a4 <= 0 || a6 < 0 || a6 > 1 || !plan_variant_known(b->prec, a1, a2, a5)) {
            rfb_set_error("sweep plan \"%s\" names no work-queue sweep variant", ov);
            return -1;
        }
        return batch_build_plan(b, a1, a2, a5, a3, a4, a6);
    }
    const std::vector<long long> key = batch_key(b);
    {
        std::lock_guard<std::mutex> lock(g_btune_mu);
        for (const auto &kv : g_btune_cache)
            if (kv.first == key) {
                const Cand &c = kv.second;
                return batch_build_plan(b, c.tj, c.ns, c.mode, c.si, c.se, c.uni);
            }
    }
    Cand best = cands[0];
    const size_t first_stage = cands.size();
    float best_ms = 1e30f;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int par = 0;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    for (size_t ci = 0; ci < cands.size(); ci++) {
        const Cand c = cands[ci];
        if (batch_build_plan(b, c.tj, c.ns, c.mode, c.si, c.se, c.uni) != 0) goto fail;
        for (int w = 0; w < 5; w++) {
            if (w == 2) CK(cudaEventRecord(t0, b->stream));
            if (b->prec == RFB_FP64) batch_sweep<double>(b, par);
            else batch_sweep<float>(b, par);
            par ^= 1;
        }
        CK(cudaEventRecord(t1, b->stream));
        CK(cudaEventSynchronize(t1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, t0, t1));
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
        if (ci + 1 == first_stage)
            for (int si : {32, 64})
                for (int se : {16, 32})
                    if (si != best.si || se != best.se)
                        cands.push_back(Cand{best.tj, best.ns, best.mode, si, se, best.uni});
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    {
        int err = 0;
        CK(cudaMemcpy(&err, b->d_err, sizeof err, cudaMemcpyDeviceToHost));
        if (err) {
            rfb_set_error("batch: %s", sweep_error_text(err));
            return -1;
        }
    }
    {
        std::lock_guard<std::mutex> lock(g_btune_mu);
        g_btune_cache.push_back({key, best});
    }
    if (batch_build_plan(b, best.tj, best.ns, best.mode, best.si, best.se, best.uni) != 0) return -1;
    // the tuning sweeps advanced the fields: start from the zero state again
    if (rfb_batch_reset(b) != 0) return -1;
    CK(cudaStreamSynchronize(b->stream));
    return 0;
fail:
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    return -1;
}

extern "C" void rfb_batch_destroy(rfb_batch_t *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free_plan(b);
    for (rfb_engine *e : b->m) rfb_engine_destroy(e);
    dfree(b->d_step); dfree(b->d_err); dfree(b->d_queue);
    dfree(b->d_args[0]); dfree(b->d_args[1]);
    dfree(b->d_lblocks); dfree(b->d_probes);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->stream2) cudaStreamDestroy(b->stream2);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

template <typename T>
static int batch_upload_args(rfb_batch *b) {
    const size_t n = b->m.size();
    std::vector<Args<T>> a[2];
    std::vector<ProbeRefB<T>> probes;
    std::vector<int2> lblocks;
    for (int par = 0; par < 2; par++) {
        a[par].resize(n);
        for (size_t s = 0; s < n; s++) {
            a[par][s] = engine_args<T>(b->m[s], par);
            a[par][s].d_step = b->d_step;
        }
        CK(dmalloc(&b->d_args[par], n * sizeof(Args<T>)));
        CK(cudaMemcpy(b->d_args[par], a[par].data(), n * sizeof(Args<T>), cudaMemcpyHostToDevice));
    }
    for (size_t s = 0; s < n; s++) {
        rfb_engine *e = b->m[s];
        const int ne = 3 * e->scene.n_cells;
        for (int e0 = 0; e0 < ne; e0 += 256) lblocks.push_back(make_int2((int)s, e0));
        std::vector<long long> cell(e->n_probes);
        std::vector<int> comp(e->n_probes);
        if (e->n_probes) {
            CK(cudaMemcpy(cell.data(), e->probe_cell, e->n_probes * sizeof(long long), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(comp.data(), e->probe_comp, e->n_probes * sizeof(int), cudaMemcpyDeviceToHost));
        }
        for (int q = 0; q < e->n_probes; q++) {
            ProbeRefB<T> r;
            r.f[0] = (const T *)e->fld[0][comp[q]];
            r.f[1] = (const T *)e->fld[1][comp[q]];
            r.cell = cell[q];
            r.ts = (T *)e->ts + (size_t)q * e->n_steps;
            probes.push_back(r);
        }
    }
    b->n_lblocks = (int)lblocks.size();
    if (b->n_lblocks) {
        CK(dmalloc(&b->d_lblocks, lblocks.size() * sizeof(int2)));
        CK(cudaMemcpy(b->d_lblocks, lblocks.data(), lblocks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }
    b->n_probes = (int)probes.size();
    if (b->n_probes) {
        CK(dmalloc(&b->d_probes, probes.size() * sizeof(ProbeRefB<T>)));
        CK(cudaMemcpy(b->d_probes, probes.data(), probes.size() * sizeof(ProbeRefB<T>), cudaMemcpyHostToDevice));
    }
    return 0;
fail:
    return -1;
}

extern "C" void *rfb_stream_create(void) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        rfb_set_error("cannot create a CUDA stream");
        return nullptr;
    }
    return (void *)st;
}
extern "C" void rfb_stream_destroy(void *stream) {
    if (stream) cudaStreamDestroy((cudaStream_t)stream);
}

extern "C" rfb_batch_t *rfb_batch_create(rfb_engine_t **members, size_t n, void *stream, int own_stream) {
    rfb_batch *b = new rfb_batch();
    b->stream = (cudaStream_t)stream;
    b->own_stream = own_stream;
    for (size_t s = 0; s < n; s++) b->m.push_back(members[s]);
    if (n == 0) {
        rfb_set_error("a batch needs at least one scene");
        goto fail;
    }
    b->prec = members[0]->prec;
    b->n_steps = members[0]->n_steps;
    for (size_t s = 0; s < n; s++) {
        rfb_engine *e = members[s];
        if (!e->member || e->prec != b->prec || e->n_steps != b->n_steps || e->nbuf != 2) {
            rfb_set_error("batch scene %zu: scenes must be batch members of one precision and step count", s);
            goto fail;
        }
        b->cells += (size_t)e->g.nx * e->g.ny * e->g.nz;
        b->list_cells += (size_t)e->scene.n_cells;
        if (e->cpml.on) {
            const int nn[3] = {e->g.nx, e->g.ny, e->g.nz};
            for (int a = 0; a < 3; a++)
                b->slab_cell_axes += (size_t)e->cpml.eh[a].ns * ((size_t)e->g.nx * e->g.ny * e->g.nz / nn[a]);
        }
    }
    if (!b->stream) {
        rfb_set_error("a batch needs the stream its scenes were created on");
        goto fail;
    }
    CK(cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    CK(dmalloc(&b->d_step, sizeof(int)));
    CK(cudaMemset(b->d_step, 0, sizeof(int)));
    CK(dmalloc(&b->d_err, sizeof(int)));
    CK(cudaMemset(b->d_err, 0, sizeof(int)));
    CK(dmalloc(&b->d_queue, 6 * sizeof(int)));
    CK(cudaMemset(b->d_queue, 0, 6 * sizeof(int)));
    if (qb_prepare() != 0) {
        rfb_set_error("cannot configure the batched sweep kernels' shared memory");
        goto fail;
    }
    for (size_t s = 0; s < n; s++)
        if (!q_fits(members[s])) {
            rfb_set_error("batch scene %zu too large for the work-queue sweep (32-bit offsets)", s);
            goto fail;
        }
    if ((b->prec == RFB_FP64 ? batch_upload_args<double>(b) : batch_upload_args<float>(b)) != 0) goto fail;
    CK(cudaDeviceSynchronize());
    {
        const double t_tune = rfb_now();
        const int rc = batch_autotune(b);
        rfb_trace("batch: plan (tuned or cached)", t_tune);
        if (rc != 0) goto fail;
    }
    return b;
fail:
    rfb_batch_destroy(b);
    return nullptr;
}

static int batch_check_error(rfb_batch *b) {
    int err = 0;
    if (cudaMemcpy(&err, b->d_err, sizeof err, cudaMemcpyDeviceToHost) != cudaSuccess) {
        rfb_set_error("batch: %s", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (err) {
        rfb_set_error("batch: %s", sweep_error_text(err));
        return -1;
    }
    return 0;
}

extern "C" int rfb_batch_advance(rfb_batch_t *b, size_t n) {
    if (b->steps_done + n > b->n_steps) {
        rfb_set_error("advance past the configured step count (%zu + %zu > %zu)", b->steps_done, n, b->n_steps);
        return -1;
    }
    const int lps = batch_launches_per_step(b);
    while (n > 0) {
        const int par = b->parity;
        if (n >= (size_t)rfb_batch::CHUNK) {
            if (!b->gk[par] && batch_graph(b, par, rfb_batch::CHUNK, &b->gk[par]) != 0) return -1;
            CK(cudaGraphLaunch(b->gk[par], b->stream));
            g_launches += (unsigned long long)rfb_batch::CHUNK * lps;
            n -= rfb_batch::CHUNK;
            b->steps_done += rfb_batch::CHUNK;
        } else {
            if (!b->g1[par] && batch_graph(b, par, 1, &b->g1[par]) != 0) return -1;
            CK(cudaGraphLaunch(b->g1[par], b->stream));
            g_launches += lps;
            n -= 1;
            b->steps_done += 1;
            b->parity ^= 1;
        }
    }
    for (rfb_engine *e : b->m) {
        e->steps_done = b->steps_done;
        e->parity = b->parity;
    }
    return 0;
fail:
    return -1;
}

extern "C" int rfb_batch_sync(rfb_batch_t *b) {
    CK(cudaStreamSynchronize(b->stream));
    return batch_check_error(b);
fail:
    return -1;
}

extern "C" int rfb_batch_advance_timed(rfb_batch_t *b, size_t n, double *ms) {
    cudaEvent_t a = nullptr, c = nullptr;
    float t = 0.f;
    int rc = -1;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&c));
    CK(cudaEventRecord(a, b->stream));
    if (rfb_batch_advance(b, n) != 0) goto out;
    CK(cudaEventRecord(c, b->stream));
    CK(cudaEventSynchronize(c));
    CK(cudaEventElapsedTime(&t, a, c));
    if (ms) *ms = t;
    rc = batch_check_error(b);
    goto out;
fail:
out:
    if (a) cudaEventDestroy(a);
    if (c) cudaEventDestroy(c);
    return rc;
}

// Runs n more steps launching each kernel separately (no graph) with events
// around the sweep and around the rest, to attribute GPU time.
extern "C" int rfb_batch_time_kernels(rfb_batch_t *b, size_t n, double *sweep_ms, double *other_ms) {
    cudaEvent_t ev[3] = {};
    double sw = 0.0, ot = 0.0;
    int rc = -1;
    if (b->steps_done + n > b->n_steps) {
        rfb_set_error("advance past the configured step count");
        return -1;
    }
    for (int q = 0; q < 3; q++) CK(cudaEventCreate(&ev[q]));
    for (size_t s = 0; s < n; s++) {
        const int par = b->parity;
        CK(cudaEventRecord(ev[0], b->stream));
        if (b->prec == RFB_FP64) batch_sweep<double>(b, par);
        else batch_sweep<float>(b, par);
        CK(cudaEventRecord(ev[1], b->stream));
        if (b->prec == RFB_FP64) batch_rest<double>(b, par);
        else batch_rest<float>(b, par);
        CK(cudaEventRecord(ev[2], b->stream));
        CK(cudaEventSynchronize(ev[2]));
        float a = 0.f, c = 0.f;
        CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
        CK(cudaEventElapsedTime(&c, ev[1], ev[2]));
        sw += a;
        ot += c;
        g_launches += batch_launches_per_step(b);
        b->steps_done++;
        b->parity ^= 1;
    }
    for (rfb_engine *e : b->m) {
        e->steps_done = b->steps_done;
        e->parity = b->parity;
    }
    *sweep_ms = sw;
    *other_ms = ot;
    rc = batch_check_error(b);
fail:
    for (int q = 0; q < 3; q++)
        if (ev[q]) cudaEventDestroy(ev[q]);
    return rc;
}

extern "C" rfb_engine_t *rfb_batch_member(rfb_batch_t *b, size_t s) {
    return s < b->m.size() ? b->m[s] : nullptr;
}
extern "C" size_t rfb_batch_size(rfb_batch_t *b) { return b->m.size(); }
extern "C" size_t rfb_batch_steps_done(rfb_batch_t *b) { return b->steps_done; }
extern "C" void *rfb_batch_stream(rfb_batch_t *b) { return (void *)b->stream; }

extern "C" int rfb_batch_info(rfb_batch_t *b, rfb_batch_info_t *out) {
    out->scenes = b->m.size();
    out->cells = b->cells;
    out->list_cells = b->list_cells;
    out->slab_cell_axes = b->slab_cell_axes;
    out->tile_j = b->tj;
    out->ring_depth = b->ns;
    out->mode = b->mode;
    out->unified = b->uni;
    out->seg_interior = b->seg_int;
    out->seg_edge = b->seg_edge;
    out->items_interior = b->n_items[0];
    out->items_xslab = b->n_items[1];
    out->items_edge = b->n_items[2];
    out->launches_per_step = batch_launches_per_step(b);
    return 0;
}
