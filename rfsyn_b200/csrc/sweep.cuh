// sweep.cuh -- persistent, TMA-fed H+E sweep over a device work queue.
//
// One step of the fused schedule is three launches of k_sweep_q on two
// streams, one per kind of work item:
//   KIND 0 (interior) -- tiles whose cells, halos and planes lie outside
//     every CPML slab and PEC boundary: branch-free, no psi;
//   KIND 1 (x slab) -- the same tiles' planes inside the x slab or on an x
//     boundary: x-slab psi and plane conditions, both uniform per plane;
//   KIND 2 (edge) -- all other tiles whose halo does not wrap around a
//     periodic axis, with rfsyn's per-component update ranges
//     (engine/fdtd/cpml.c:176-219, materials.c:911-1060) and every slab
//     psi recursion (cpml.h:46-51).  An edge item is marched by one of
//     three bodies chosen by its `sub` field: tiles that touch only the y
//     slab (KIND 3 body) or only the z slab (KIND 4 body) carry no code
//     for the other axis; the rest take the full body.
// Items whose halo wraps stay on the cp.async-fed k_sweep_edge (fused.cuh).
// Each kind is compiled separately so the interior keeps the lean
// instruction stream it needs to stay bandwidth-bound.
//
// The grid is sized to the resident CTAs (SM count x CTAs per SM); each CTA
// pops items from a device counter until the list is exhausted, so uneven
// items (interior vs slab tiles, segment remainders) balance across SMs.  The
// last CTA to leave zeroes the counters, so every launch starts from a clean
// queue whatever ran before it.
//
// Per item the march is the one of k_sweep_interior_tma (tma.cuh): per plane
// one elected thread issues one tiled cp.async.bulk.tensor load per field
// component and one for the codes into an NS-deep ring of shared-memory
// stages completing on mbarriers; H of the plane is computed for the tile and
// its low-j / low-k halo (recomputed, never stored), then E follows from the
// shared H and the previous plane's H kept in registers.  psi values of slab
// cells are read with plain loads issued before the plane's barrier wait, so
// their latency overlaps the wait; profile values of the tile's rows and
// columns sit in shared memory.  Only slab cells touch psi or profiles, so
// the bytes moved are the algorithmic ones.
//
// Every mbarrier wait is bounded (tma.cuh: mbar_wait); on a timeout the CTA
// records an error code, lets its own copies in flight land (bounded) and
// leaves the queue.  No load uses cluster multicast.
#pragma once
#include "tma.cuh"

namespace rfb {

// The thread that issues a CTA's tensor copies (warp 4, lane 0; warps 0-3
// recompute the halo H).  Where the tensor maps live in global memory (the
// batched sweep), this thread is also the one that acquires them through the
// tensormap proxy before its first copy of a scene.
constexpr int kCopyIssueTid = 4 * 32;

template <typename T, int TJ>
struct TileTables {
    T tab[512];           // Ca (0..255), Cb (256..511)
    T py[6][2 * TJ + 1];  // y profiles at rows j0-1 .. j0+rows-1: H grid (kinv b a), E grid (kinv b a)
    T pz[6][33];          // z profiles at cols k0-1 .. k0+cols-1
};

// Boxes of one stage for a tile of TR rows x W columns: E rows j0-1 ..
// j0+TR, columns k0-4 .. k0+W+3; H rows j0-1 .. j0+TR-1, columns k0-4 ..
// k0+W-1; codes TR x W.  Wide tiles are (TJ x 32), one row per warp;
// narrow tiles (2 TJ x 16), two rows per warp.
template <typename T, int TR, int W>
struct QShape {
    static constexpr int EW = W + 8, HW = W + 4;
    static constexpr unsigned ebytes = sizeof(T) * EW * (TR + 2);
    static constexpr unsigned hbytes = sizeof(T) * HW * (TR + 1);
    static constexpr unsigned cbytes = W * TR;
    static constexpr size_t ebox = round128(ebytes);
    static constexpr size_t hbox = round128(hbytes);
    static constexpr size_t cbox = round128(cbytes);
    static constexpr size_t stage = 3 * ebox + 3 * hbox + cbox;
};

__host__ __device__ constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }

template <typename T, int TJ, int NS>
struct QLayout {
    using Wd = QShape<T, TJ, 32>;
    using Nr = QShape<T, 2 * TJ, 16>;
    static constexpr size_t stage = cmax(Wd::stage, Nr::stage);
    static constexpr size_t bars = NS * stage;
    static constexpr size_t sh = bars + round128(8 * NS);
    static constexpr size_t tabs = sh + round128(sizeof(T) * 2 * 3 * cmax((TJ + 1) * 33, (2 * TJ + 1) * 17));
    static constexpr size_t misc = tabs + round128(sizeof(TileTables<T, TJ>));
    static constexpr size_t total = misc + 16;
};

// One work item: the march over planes [ib, ie) of the (TJ x 32) tile (W =
// 32) or the (2 TJ x 16) tile (W = 16) at (j0, k0) of the scene described by
// `a`, `d` and `maps`.  `phase`,
// `pending` and `failed` are the CTA's ring bookkeeping, carried across
// items.  Returns false when a copy did not complete in time (the caller
// drains the ring and leaves the queue).
template <typename T, int TJ, int NS, int KIND, int W = 32>
__device__ __forceinline__ bool q_item(const Args<T> &a, const FusedDims &d, const TmaMaps &maps, const SweepItem &it,
                                       unsigned char *smem_raw, unsigned &phase, unsigned &pending, bool &failed) {
    constexpr bool EDGE = KIND >= 2;             // per-cell y / z conditions
    constexpr bool YS = KIND == 2 || KIND == 3;  // y-slab psi
    constexpr bool ZS = KIND == 2 || KIND == 4;  // z-slab psi
    constexpr bool XS = KIND >= 1;               // x-slab psi and plane conditions
    static_assert(W == 32 || (W == 16 && KIND >= 2), "narrow tiles are edge tiles");
    constexpr int RPW = 32 / W;       // tile rows per warp
    constexpr int TR = TJ * RPW;      // tile rows
    using L = QShape<T, TR, W>;
    using S = QLayout<T, TJ, NS>;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::bars);
    // H of the current plane (tile + halo), double-buffered by plane parity
    // so one block barrier per plane separates its writes from its reads
    T(*sHb)[3][TR + 1][W + 1] = reinterpret_cast<T(*)[3][TR + 1][W + 1]>(smem_raw + S::sh);
    TileTables<T, TJ> &tt = *reinterpret_cast<TileTables<T, TJ> *>(smem_raw + S::tabs);
    auto E = [&](int s, int c) { return reinterpret_cast<T(*)[L::EW]>(smem_raw + s * S::stage + c * L::ebox); };
    auto H = [&](int s, int c) {
        return reinterpret_cast<T(*)[L::HW]>(smem_raw + s * S::stage + 3 * L::ebox + c * L::hbox);
    };
    auto CODE = [&](int s) {
        return reinterpret_cast<uint8_t(*)[W]>(smem_raw + s * S::stage + 3 * L::ebox + 3 * L::hbox);
    };
    const CUtensorMap *me = W == 32 ? maps.e : maps.en, *mh = W == 32 ? maps.h : maps.hn;
    const CUtensorMap *mc = W == 32 ? &maps.code : &maps.coden;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const int row = ty * RPW + (RPW > 1 ? tx / W : 0), col = RPW > 1 ? tx % W : tx;  // own cell in the tile
    const int r = row + 1, q = col + 4;  // stage coordinates of the own cell
    const int qs = col + 1;              // sH / z-table column of the own cell
    const bool with_codes = a.codes != nullptr;
    const unsigned tx_bytes = 3 * L::ebytes + 3 * L::hbytes + (with_codes ? L::cbytes : 0u);
    const T cbh = a.cbh;
    const int on = a.cpml_on;
    const long long ny1 = a.ny + 1;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;

    // warps 0-3 recompute the halo H of the plane (one piece each); warp 4
    // issues the copies, so no warp carries two extra jobs per plane
    auto issue = [&](int s, int p) {
        if (p < 0 || failed) return;  // a failed CTA issues no further copies
        if (tid == kCopyIssueTid) {
            mbar_expect_tx(&bars[s], tx_bytes);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                tma_load_3d(E(s, c), &me[c], k0 - 4, j0 - 1, p, &bars[s]);
                tma_load_3d(H(s, c), &mh[c], k0 - 4, j0 - 1, p, &bars[s]);
            }
            if (with_codes) tma_load_3d(CODE(s), mc, k0, j0, p, &bars[s]);
        }
        pending |= 1u << s;
    };
    // a wait that timed out marks the CTA failed; later waits return at
    // once and the item ends with garbage, reported at its end
    auto wait_slot = [&](int s) {
        if (!(pending & (1u << s))) return;
        if (failed || !mbar_wait(&bars[s], (phase >> s) & 1u)) {
            failed = true;
            return;  // still pending: drained (bounded) on the bail path
        }
        phase ^= 1u << s;
        pending &= ~(1u << s);
    };

    // ---- per-thread geometry of the item ----
    // The interior instantiation takes tiles whose cells and halos lie
    // outside the y / z slabs and boundaries: every component is swept
    // at every (j, k), only the plane (x) conditions and x-slab psi
    // remain, both uniform per plane.  The edge instantiation adds the
    // per-cell y / z conditions and y / z slab psi.
    const int j = j0 + row, k = k0 + col;
    const bool own = !EDGE || (j >= 0 && k >= 0 && j < d.cj && k < d.ck);
    const int pitch = (int)a.pitch;
    const int plane32 = (int)a.plane;
    // halo cells recomputed per plane: the row (j0-1, k0 .. k0+W-1), Hx by
    // warp 0 and Hz by warp 2, the column (j0 .. j0+TR-1, k0-1), Hx by warp
    // 1 and Hy by warp 3; lane tx takes halo column tx / halo row tx
    const int jh = j0 - 1, jc = j0 + tx, kh = k0 - 1;
    unsigned mjk = 0x3f;                   // bits 0-2 H, 3-5 E at (j, k), plane apart
    bool rowh = tx < W, colh = tx < TR;    // halo cells this thread recomputes
    int sjh = -1, skh = -1, sjm = -1, skm = -1;
    int sjh_row = -1, sjh_col = -1, skh_col = -1;
    unsigned mrow_jk = 5u, mcol_jk = 3u;   // halo components at (j, k), plane apart
    if constexpr (EDGE) {
        const int jmin = py ? 0 : 1, kmin = pz ? 0 : 1;
        mjk = 0;
        if (own) {
            if (j < a.ny && k < a.nz) mjk |= 1u;
            if (j < a.ny + (py ? 0 : 1) && k < a.nz) mjk |= 2u;
            if (j < a.ny && k < a.nz + (pz ? 0 : 1)) mjk |= 4u;
            if (j < a.ny && k < a.nz) {
                if (j >= jmin && k >= kmin) mjk |= 8u;
                if (k >= kmin) mjk |= 16u;
                if (j >= jmin) mjk |= 32u;
            }
        }
        rowh = tx < W && j0 > 0 && k >= 0 && k < d.ck;
        colh = tx < TR && k0 > 0 && jc >= 0 && jc < d.cj;
        mrow_jk = (k < a.nz ? 1u : 0u) | (k < a.nz + (pz ? 0 : 1) ? 4u : 0u);
        mcol_jk = (jc < a.ny ? 1u : 0u) | (jc < a.ny + (py ? 0 : 1) ? 2u : 0u);
        // a body without one axis's slab code serves only tiles whose
        // cells and halos lie outside that slab (the host classifies them)
        if constexpr (YS) {
            sjh = slab_in(j, a.lo_h[1], a.hi_h[1], a.ny, on);
            sjm = slab_in(j, a.lo_m[1], a.hi_m[1], a.ny, on);
            sjh_row = slab_in(jh, a.lo_h[1], a.hi_h[1], a.ny, on);
            sjh_col = slab_in(jc, a.lo_h[1], a.hi_h[1], a.ny, on);
            for (int t = tid; t < TR + 1; t += 32 * TJ) {
                T v[3];
                prof_at(on ? a.kinv_h[1] : (const T *)nullptr, a.b_h[1], a.a_h[1], j0 - 1 + t, a.ny, v);
                tt.py[0][t] = v[0]; tt.py[1][t] = v[1]; tt.py[2][t] = v[2];
                prof_at(on ? a.kinv_m[1] : (const T *)nullptr, a.b_m[1], a.a_m[1], j0 - 1 + t, a.ny + 1, v);
                tt.py[3][t] = v[0]; tt.py[4][t] = v[1]; tt.py[5][t] = v[2];
            }
        }
        if constexpr (ZS) {
            skh = slab_in(k, a.lo_h[2], a.hi_h[2], a.nz, on);
            skm = slab_in(k, a.lo_m[2], a.hi_m[2], a.nz, on);
            skh_col = slab_in(kh, a.lo_h[2], a.hi_h[2], a.nz, on);
            for (int t = tid; t < W + 1; t += 32 * TJ) {
                T v[3];
                prof_at(on ? a.kinv_h[2] : (const T *)nullptr, a.b_h[2], a.a_h[2], k0 - 1 + t, a.nz, v);
                tt.pz[0][t] = v[0]; tt.pz[1][t] = v[1]; tt.pz[2][t] = v[2];
                prof_at(on ? a.kinv_m[2] : (const T *)nullptr, a.b_m[2], a.a_m[2], k0 - 1 + t, a.nz + 1, v);
                tt.pz[3][t] = v[0]; tt.pz[4][t] = v[1]; tt.pz[5][t] = v[2];
            }
        }
    }
    const int nshy = a.ns_h[1], nshz = a.ns_h[2], nsmy = a.ns_m[1], nsmz = a.ns_m[2];
    // 32-bit element offsets (the plan admits these sweeps only when every
    // field plane and psi array has fewer than 2^31 elements): in-plane
    // offsets (x-slab psi arrays are planes of the field layout), y-slab
    // offsets s*pitch + k, z-slab offsets j*ns + s; per plane a uniform
    // base is added
    struct Cell {
        int ox, oy, oz;  // x-, y-, z-slab array offsets (plane / slab bases apart)
        int sy, sz;      // H-grid y / z slab indices (-1 outside)
    };
    const Cell own_c = {j * pitch + k, sjh * pitch + k, j * nshz + skh, sjh, skh};
    const Cell row_c = {jh * pitch + k, sjh_row * pitch + k, jh * nshz + skh, sjh_row, skh};
    const Cell col_c = {jc * pitch + kh, sjh_col * pitch + kh, jc * nshz + skh_col, sjh_col, skh_col};
    const int oym = sjm * pitch + k, ozm = j * nsmz + skm;
    // per-plane uniform bases of the H-side psi arrays and the plane's x
    // profile (kappa_inv, b, a) on the H and E grids
    struct PlaneB {
        int by, bz, bx, sx;
    };
    auto plane_b = [&](int i) -> PlaneB {
        const int sx = (XS && on) ? slab_in(i, a.lo_h[0], a.hi_h[0], a.nx, on) : -1;
        return PlaneB{i * nshy * pitch, i * (int)ny1 * nshz, sx * plane32, sx};
    };
    T xph[3] = {T(1), T(1), T(0)}, xpm[3] = {T(1), T(1), T(0)};
    auto load_xprof = [&](int i, int sxh_, int sxm_) {
        if constexpr (!XS) return;
        if (sxh_ >= 0) {
            xph[0] = a.kinv_h[0][i];
            xph[1] = a.b_h[0][i];
            xph[2] = a.a_h[0][i];
        }
        if (sxm_ >= 0) {
            xpm[0] = a.kinv_m[0][i];
            xpm[1] = a.b_m[0][i];
            xpm[2] = a.a_m[0][i];
        }
    };

    // H of component c at plane i (slots sc / sn) for the cell at stage
    // position (rr, qq) described by `cl`; yi / zi are its rows in the
    // profile tables.  pA / pB are the cell's psi inputs of the two terms
    // (used where a slab applies); the updated psi are stored when `store`.
    auto hcell = [&](int c, const PlaneB &pb, int sc, int sn, int rr, int qq, const Cell &cl, int yi, int zi,
                     T pA, T pB, bool store) -> T {
        const T hin = H(sc, c)[rr][qq];
        T dA, dB;
        if (c == 0) {
            dA = xs(E(sc, 2)[rr + 1][qq], E(sc, 2)[rr][qq]);
            dB = xs(E(sc, 1)[rr][qq + 1], E(sc, 1)[rr][qq]);
        } else if (c == 1) {
            dA = xs(E(sc, 0)[rr][qq + 1], E(sc, 0)[rr][qq]);
            dB = xs(E(sn, 2)[rr][qq], E(sc, 2)[rr][qq]);
        } else {
            dA = xs(E(sn, 1)[rr][qq], E(sc, 1)[rr][qq]);
            dB = xs(E(sc, 0)[rr + 1][qq], E(sc, 0)[rr][qq]);
        }
        T pn;
        if (c == 0) {
            if (YS && cl.sy >= 0) {
                dA = stretch(dA, tt.py[0][yi], tt.py[1][yi], tt.py[2][yi], a.dx, pA, &pn);
                if (store) a.psi_ho[0][pb.by + cl.oy] = pn;
            }
            if (ZS && cl.sz >= 0) {
                dB = stretch(dB, tt.pz[0][zi], tt.pz[1][zi], tt.pz[2][zi], a.dx, pB, &pn);
                if (store) a.psi_ho[1][pb.bz + cl.oz] = pn;
            }
        } else if (c == 1) {
            if (ZS && cl.sz >= 0) {
                dA = stretch(dA, tt.pz[0][zi], tt.pz[1][zi], tt.pz[2][zi], a.dx, pA, &pn);
                if (store) a.psi_ho[2][pb.bz + cl.oz] = pn;
            }
            if (pb.sx >= 0) {
                dB = stretch(dB, xph[0], xph[1], xph[2], a.dx, pB, &pn);
                if (store) a.psi_ho[3][pb.bx + cl.ox] = pn;
            }
        } else {
            if (pb.sx >= 0) {
                dA = stretch(dA, xph[0], xph[1], xph[2], a.dx, pA, &pn);
                if (store) a.psi_ho[4][pb.bx + cl.ox] = pn;
            }
            if (YS && cl.sy >= 0) {
                dB = stretch(dB, tt.py[0][yi], tt.py[1][yi], tt.py[2][yi], a.dx, pB, &pn);
                if (store) a.psi_ho[5][pb.by + cl.oy] = pn;
            }
        }
        return upd_h(hin, cbh, xs(dA, dB));
    };
    // psi inputs of H component c at a cell (zero where no slab applies)
    auto hpsi = [&](int c, const PlaneB &pb, const Cell &cl, T &pA, T &pB) {
        pA = T(0);
        pB = T(0);
        if (c == 0) {
            if (YS && cl.sy >= 0) pA = a.psi_hi[0][pb.by + cl.oy];
            if (ZS && cl.sz >= 0) pB = a.psi_hi[1][pb.bz + cl.oz];
        } else if (c == 1) {
            if (ZS && cl.sz >= 0) pA = a.psi_hi[2][pb.bz + cl.oz];
            if (pb.sx >= 0) pB = a.psi_hi[3][pb.bx + cl.ox];
        } else {
            if (pb.sx >= 0) pA = a.psi_hi[4][pb.bx + cl.ox];
            if (YS && cl.sy >= 0) pB = a.psi_hi[5][pb.by + cl.oy];
        }
    };
    // plane conditions: H bits (Hx to nx inclusive on a PEC x axis), E bits
    auto plane_mask = [&](int i) -> unsigned {
        if constexpr (!XS) return 0x3fu;
        unsigned m = 0;
        if (i < a.nx + (px ? 0 : 1)) m |= 1u;
        if (i < a.nx) m |= 2u | 4u | 8u;
        if (i < a.nx && i >= (px ? 0 : 1)) m |= 16u | 32u;
        return m;
    };

    // ---- prologue: previous plane and the first NS-1 planes ----
    int pprev = ib > 0 ? ib - 1 : (px ? a.nx - 1 : -1);
    int pf = ib;
    issue(NS - 1, pprev);
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) issue(s, pf);
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    wait_slot(NS - 1);
    wait_slot(0);
    if (__syncthreads_or(failed)) return false;
    {
        T prevHy = T(0), prevHz = T(0);
        if (pprev >= 0) {
            const unsigned mp = plane_mask(pprev) & mjk;
            const PlaneB pb = plane_b(pprev);
            load_xprof(pprev, pb.sx, -1);
            // psi are read only for components swept at the cell, so
            // every offset used addresses a cell of the grid
            T pA = T(0), pB = T(0);
            prevHy = H(NS - 1, 1)[r][q];
            if (mp & 2u) {
                hpsi(1, pb, own_c, pA, pB);
                prevHy = hcell(1, pb, NS - 1, 0, r, q, own_c, r, qs, pA, pB, false);
            }
            prevHz = H(NS - 1, 2)[r][q];
            if (mp & 4u) {
                hpsi(2, pb, own_c, pA, pB);
                prevHz = hcell(2, pb, NS - 1, 0, r, q, own_c, r, qs, pA, pB, false);
            }
        }
        __syncthreads();  // slot NS-1 may now be refilled

        int sc = 0;
        for (int i = ib; i < ie; i++) {
            const int sn = sc == NS - 1 ? 0 : sc + 1;
            const int sf = sc == 0 ? NS - 1 : sc - 1;  // held plane i-1, read by nobody any more
            if (pf >= 0 && i + NS - 1 <= ie) {
                issue(sf, pf);
                pf = plane_after(pf, a.nx, px);
            }
            const unsigned mpl = plane_mask(i);
            const unsigned m = mpl & mjk;
            const PlaneB pb = plane_b(i);
            const int sxm = (XS && on) ? slab_in(i, a.lo_m[0], a.hi_m[0], a.nx, on) : -1;
            const int bym = i * nsmy * pitch, bzm = i * (int)ny1 * nsmz, bxm = sxm * plane32;
            // halo cells recomputed this plane: row (j0-1, k) Hx by warp 0,
            // Hz by warp 2; column (j0+tx, k0-1) Hx by warp 1, Hy by warp 3
            const unsigned mrow = (ty == 0 && rowh) ? (mpl & mrow_jk & 1u)
                                  : (ty == 2 && rowh) ? (mpl & mrow_jk & 4u) : 0u;
            const unsigned mcol = (ty == 1 && colh) ? (mpl & mcol_jk & 1u)
                                  : (ty == 3 && colh) ? (mpl & mcol_jk & 2u) : 0u;
            // psi inputs of the own cell and of the halo cells and the
            // plane's x profile, all loaded before the wait; psi are read
            // only for components swept at the cell, so every offset
            // used addresses a cell of the grid
            T hp[6], ep[6], hh[4];
#pragma unroll
            for (int t = 0; t < 6; t++) hp[t] = ep[t] = T(0);
#pragma unroll
            for (int t = 0; t < 4; t++) hh[t] = T(0);
            load_xprof(i, pb.sx, sxm);
            if (m & 1u) hpsi(0, pb, own_c, hp[0], hp[1]);
            if (m & 2u) hpsi(1, pb, own_c, hp[2], hp[3]);
            if (m & 4u) hpsi(2, pb, own_c, hp[4], hp[5]);
            if (mrow & 1u) hpsi(0, pb, row_c, hh[0], hh[1]);
            if (mrow & 4u) hpsi(2, pb, row_c, hh[2], hh[3]);
            if (mcol & 1u) hpsi(0, pb, col_c, hh[0], hh[1]);
            if (mcol & 2u) hpsi(1, pb, col_c, hh[2], hh[3]);
            if (m & 8u) {
                if (YS && sjm >= 0) ep[0] = a.psi_e[0][bym + oym];
                if (ZS && skm >= 0) ep[1] = a.psi_e[1][bzm + ozm];
            }
            if (m & 16u) {
                if (ZS && skm >= 0) ep[2] = a.psi_e[2][bzm + ozm];
                if (sxm >= 0) ep[3] = a.psi_e[3][bxm + own_c.ox];
            }
            if (m & 32u) {
                if (sxm >= 0) ep[4] = a.psi_e[4][bxm + own_c.ox];
                if (YS && sjm >= 0) ep[5] = a.psi_e[5][bym + oym];
            }
            wait_slot(sn);  // plane i+1 (plane i landed before the previous barrier)
            T(*sH)[TR + 1][W + 1] = sHb[(i - ib) & 1];
            const T e0 = E(sc, 0)[r][q], e1 = E(sc, 1)[r][q], e2 = E(sc, 2)[r][q];
            const int code = with_codes ? (int)CODE(sc)[row][col] : 0;
            const long long c = (long long)i * a.plane + own_c.ox;
            T hx = H(sc, 0)[r][q], hy = H(sc, 1)[r][q], hz = H(sc, 2)[r][q];
            if (m & 1u) hx = hcell(0, pb, sc, sn, r, q, own_c, r, qs, hp[0], hp[1], true);
            if (m & 2u) hy = hcell(1, pb, sc, sn, r, q, own_c, r, qs, hp[2], hp[3], true);
            if (m & 4u) hz = hcell(2, pb, sc, sn, r, q, own_c, r, qs, hp[4], hp[5], true);
            if (own) {
                a.Ho[0][c] = hx;
                a.Ho[1][c] = hy;
                a.Ho[2][c] = hz;
            }
            sH[0][r][qs] = hx;
            sH[1][r][qs] = hy;
            sH[2][r][qs] = hz;
            if (ty == 0 && rowh) {
                // row halo (j0-1, k): Hx
                T v = H(sc, 0)[0][q];
                if (mrow & 1u) v = hcell(0, pb, sc, sn, 0, q, row_c, 0, qs, hh[0], hh[1], false);
                sH[0][0][qs] = v;
            } else if (ty == 2 && rowh) {
                // row halo (j0-1, k): Hz
                T v = H(sc, 2)[0][q];
                if (mrow & 4u) v = hcell(2, pb, sc, sn, 0, q, row_c, 0, qs, hh[2], hh[3], false);
                sH[2][0][qs] = v;
            } else if (ty == 1 && colh) {
                // column halo (j0+tx, k0-1): Hx
                T v = H(sc, 0)[tx + 1][3];
                if (mcol & 1u) v = hcell(0, pb, sc, sn, tx + 1, 3, col_c, tx + 1, 0, hh[0], hh[1], false);
                sH[0][tx + 1][0] = v;
            } else if (ty == 3 && colh) {
                // column halo (j0+tx, k0-1): Hy
                T v = H(sc, 1)[tx + 1][3];
                if (mcol & 2u) v = hcell(1, pb, sc, sn, tx + 1, 3, col_c, tx + 1, 0, hh[2], hh[3], false);
                sH[1][tx + 1][0] = v;
            }
            __syncthreads();
            if (!with_codes || code != LIST_CODE) {
                bool skip = false;
                if constexpr (EDGE) {
                    if (!with_codes)
                        for (int s = 0; s < a.n_skip; s++) skip |= a.skip[s] == c;
                }
                if (!skip) {
                    const T ca = tt.tab[code], cb = tt.tab[256 + code];
                    T pn;
                    if (m & 8u) {
                        T tA = xs(sH[2][r][qs], sH[2][r - 1][qs]);
                        T tB = xs(sH[1][r][qs], sH[1][r][qs - 1]);
                        if (YS && sjm >= 0) {
                            tA = stretch(tA, tt.py[3][r], tt.py[4][r], tt.py[5][r], a.dx, ep[0], &pn);
                            a.psi_e[0][bym + oym] = pn;
                        }
                        if (ZS && skm >= 0) {
                            tB = stretch(tB, tt.pz[3][qs], tt.pz[4][qs], tt.pz[5][qs], a.dx, ep[1], &pn);
                            a.psi_e[1][bzm + ozm] = pn;
                        }
                        a.Eo[0][c] = upd_e(ca, e0, cb, xs(tA, tB));
                    }
                    if (m & 16u) {
                        T tA = xs(sH[0][r][qs], sH[0][r][qs - 1]);
                        T tB = xs(hz, prevHz);
                        if (ZS && skm >= 0) {
                            tA = stretch(tA, tt.pz[3][qs], tt.pz[4][qs], tt.pz[5][qs], a.dx, ep[2], &pn);
                            a.psi_e[2][bzm + ozm] = pn;
                        }
                        if (sxm >= 0) {
                            tB = stretch(tB, xpm[0], xpm[1], xpm[2], a.dx, ep[3], &pn);
                            a.psi_e[3][bxm + own_c.ox] = pn;
                        }
                        a.Eo[1][c] = upd_e(ca, e1, cb, xs(tA, tB));
                    }
                    if (m & 32u) {
                        T tA = xs(hy, prevHy);
                        T tB = xs(sH[0][r][qs], sH[0][r - 1][qs]);
                        if (sxm >= 0) {
                            tA = stretch(tA, xpm[0], xpm[1], xpm[2], a.dx, ep[4], &pn);
                            a.psi_e[4][bxm + own_c.ox] = pn;
                        }
                        if (YS && sjm >= 0) {
                            tB = stretch(tB, tt.py[3][r], tt.py[4][r], tt.py[5][r], a.dx, ep[5], &pn);
                            a.psi_e[5][bym + oym] = pn;
                        }
                        a.Eo[2][c] = upd_e(ca, e2, cb, xs(tA, tB));
                    }
                }
            }
            prevHy = hy;
            prevHz = hz;
            sc = sn;
        }
    }
    return !__syncthreads_or(failed);
}

// The march of one item: an edge item takes the body its `sub` names; KIND 5
// (the single-queue sweep) takes interior (sub 5) and x-slab (sub 6) items
// too.
template <typename T, int TJ, int NS, int KIND>
__device__ __forceinline__ bool q_run(const Args<T> &a, const FusedDims &d, const TmaMaps &maps, const SweepItem &it,
                                      unsigned char *smem_raw, unsigned &phase, unsigned &pending, bool &failed) {
    if constexpr (KIND == 5) {
        switch (it.sub) {
            case 5: return q_item<T, TJ, NS, 0>(a, d, maps, it, smem_raw, phase, pending, failed);
            case 6: return q_item<T, TJ, NS, 1>(a, d, maps, it, smem_raw, phase, pending, failed);
            case 1: return q_item<T, TJ, NS, 3>(a, d, maps, it, smem_raw, phase, pending, failed);
            case 2: return q_item<T, TJ, NS, 4>(a, d, maps, it, smem_raw, phase, pending, failed);
            case 3: return q_item<T, TJ, NS, 4, 16>(a, d, maps, it, smem_raw, phase, pending, failed);
            case 4: return q_item<T, TJ, NS, 2, 16>(a, d, maps, it, smem_raw, phase, pending, failed);
            default: return q_item<T, TJ, NS, 2>(a, d, maps, it, smem_raw, phase, pending, failed);
        }
    }
    if constexpr (KIND == 2) {
        if (it.sub == 1) return q_item<T, TJ, NS, 3>(a, d, maps, it, smem_raw, phase, pending, failed);
        if (it.sub == 2) return q_item<T, TJ, NS, 4>(a, d, maps, it, smem_raw, phase, pending, failed);
        if (it.sub == 3) return q_item<T, TJ, NS, 4, 16>(a, d, maps, it, smem_raw, phase, pending, failed);
        if (it.sub == 4) return q_item<T, TJ, NS, 2, 16>(a, d, maps, it, smem_raw, phase, pending, failed);
    }
    return q_item<T, TJ, NS, KIND>(a, d, maps, it, smem_raw, phase, pending, failed);
}

// Loads the scene's (Ca, Cb) table into the CTA's shared tables.
template <typename T, int TJ, int NS>
__device__ __forceinline__ void q_load_table(const Args<T> &a, unsigned char *smem_raw) {
    using S = QLayout<T, TJ, NS>;
    TileTables<T, TJ> &tt = *reinterpret_cast<TileTables<T, TJ> *>(smem_raw + S::tabs);
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int t = tid; t < 256; t += 32 * TJ) {
        tt.tab[t] = a.tca[t];
        tt.tab[256 + t] = a.tcb[t];
    }
}

// Tensor copies need their shared destinations on 128-byte boundaries; the
// layouts keep every box at a multiple of 128 from the dynamic region's
// start.  A CTA whose region does not start on such a boundary records
// error 2 and returns before issuing anything.
__device__ __forceinline__ bool q_misaligned(const unsigned char *smem, int *err) {
    if ((__cvta_generic_to_shared(smem) & 127u) == 0) return false;
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(err, 2);
    return true;
}

template <int NS>
__device__ __forceinline__ void q_init_bars(uint64_t *bars) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
}

// A copy did not complete in time: report it, let the CTA's copies still in
// flight land (bounded) before its shared memory is reused or released.
template <int NS>
__device__ __forceinline__ void q_bail(uint64_t *bars, unsigned phase, unsigned pending, int *err) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        atomicExch(err, 1);
        for (int s = 0; s < NS; s++)
            if (pending & (1u << s)) mbar_wait(&bars[s], (phase >> s) & 1u);
    }
    __syncthreads();
}

// Leaves the queue; the last CTA out rewinds it for the next launch.
__device__ __forceinline__ void q_leave(int *queue) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        if (atomicAdd(&queue[1], 1) == (int)gridDim.x - 1) {
            queue[0] = 0;
            queue[1] = 0;
            __threadfence();
        }
    }
}

template <typename T, int TJ, int NS, int MINB, int KIND>
__global__ void __launch_bounds__(32 * TJ, MINB)
    k_sweep_q(Args<T> a, FusedDims d, const SweepItem *items, int n_items, const __grid_constant__ TmaMaps maps,
              int *queue, int *err) {
    static_assert(NS >= 3, "the ring must hold the current, the next and one prefetched plane");
    static_assert(TJ >= 5, "warps 0-3 share the halo recomputation, warp 4 issues the copies");
    using S = QLayout<T, TJ, NS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (q_misaligned(smem_raw, err)) return;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::bars);
    volatile int *s_item = reinterpret_cast<volatile int *>(smem_raw + S::misc);
    q_init_bars<NS>(bars);
    q_load_table<T, TJ, NS>(a, smem_raw);
    __syncthreads();
    // ring bookkeeping: phase bit s = parity of slot s's next completion,
    // pending bit s = slot s has a load in flight that nobody waited for
    unsigned phase = 0, pending = 0;
    bool failed = false;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) *s_item = atomicAdd(&queue[0], 1);
        __syncthreads();
        const int w = *s_item;
        if (w >= n_items) break;
        const SweepItem it = items[w];
        if (!q_run<T, TJ, NS, KIND>(a, d, maps, it, smem_raw, phase, pending, failed)) {
            q_bail<NS>(bars, phase, pending, err);
            break;
        }
        __syncthreads();  // the ring, the tables and the item slot are free again
    }
    q_leave(queue);
}

// ---- interior tiles of two rows per thread ---------------------------------------
// The interior march of q_item (KIND 0: no slab, no boundary) over a tile of
// 2 TJ rows x 32 columns with TJ warps: thread (tx, ty) owns the cells of
// rows ty and ty + TJ, so the plane's fixed work -- the copy wait, the block
// barrier, the ring bookkeeping, the halo row and column -- is shared by
// twice the cells, and each thread has two independent cells' arithmetic to
// interleave.  Same operations in the same order per cell as q_item, so the
// results are bit-identical.
template <typename T, int TJ, int NS>
struct QLayoutI2 {
    using S = QShape<T, 2 * TJ, 32>;
    static constexpr size_t stage = S::stage;
    static constexpr size_t bars = NS * stage;
    static constexpr size_t sh = bars + round128(8 * NS);
    static constexpr size_t tabs = sh + round128(sizeof(T) * 2 * 3 * (2 * TJ + 1) * 33);
    static constexpr size_t misc = tabs + round128(sizeof(TileTables<T, TJ>));
    static constexpr size_t total = misc + 16;
};

template <typename T, int TJ, int NS>
__device__ __forceinline__ bool q_item_i2(const Args<T> &a, const TmaMaps &maps, const SweepItem &it,
                                          unsigned char *smem_raw, unsigned &phase, unsigned &pending, bool &failed) {
    constexpr int TR = 2 * TJ;
    using L = QShape<T, TR, 32>;
    using S = QLayoutI2<T, TJ, NS>;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::bars);
    T(*sHb)[3][TR + 1][33] = reinterpret_cast<T(*)[3][TR + 1][33]>(smem_raw + S::sh);
    TileTables<T, TJ> &tt = *reinterpret_cast<TileTables<T, TJ> *>(smem_raw + S::tabs);
    auto E = [&](int s, int c) { return reinterpret_cast<T(*)[L::EW]>(smem_raw + s * S::stage + c * L::ebox); };
    auto H = [&](int s, int c) {
        return reinterpret_cast<T(*)[L::HW]>(smem_raw + s * S::stage + 3 * L::ebox + c * L::hbox);
    };
    auto CODE = [&](int s) {
        return reinterpret_cast<uint8_t(*)[32]>(smem_raw + s * S::stage + 3 * L::ebox + 3 * L::hbox);
    };
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const bool px = a.per & 1u;
    const bool with_codes = a.codes != nullptr;
    const unsigned tx_bytes = 3 * L::ebytes + 3 * L::hbytes + (with_codes ? L::cbytes : 0u);
    const T cbh = a.cbh;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const int q = tx + 4, qs = tx + 1;
    const bool colh = tx < TR;

    auto issue = [&](int s, int p) {
        if (p < 0 || failed) return;
        if (tid == kCopyIssueTid) {
            mbar_expect_tx(&bars[s], tx_bytes);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                tma_load_3d(E(s, c), &maps.e2[c], k0 - 4, j0 - 1, p, &bars[s]);
                tma_load_3d(H(s, c), &maps.h2[c], k0 - 4, j0 - 1, p, &bars[s]);
            }
            if (with_codes) tma_load_3d(CODE(s), &maps.code2, k0, j0, p, &bars[s]);
        }
        pending |= 1u << s;
    };
    auto wait_slot = [&](int s) {
        if (!(pending & (1u << s))) return;
        if (failed || !mbar_wait(&bars[s], (phase >> s) & 1u)) {
            failed = true;
            return;
        }
        phase ^= 1u << s;
        pending &= ~(1u << s);
    };
    // unstretched H of component c at stage position (rr, qq) of the plane
    // in slot sc (the plane after it in slot sn): q_item's arithmetic
    auto hval = [&](int c, int sc, int sn, int rr, int qq) -> T {
        T dA, dB;
        if (c == 0) {
            dA = xs(E(sc, 2)[rr + 1][qq], E(sc, 2)[rr][qq]);
            dB = xs(E(sc, 1)[rr][qq + 1], E(sc, 1)[rr][qq]);
        } else if (c == 1) {
            dA = xs(E(sc, 0)[rr][qq + 1], E(sc, 0)[rr][qq]);
            dB = xs(E(sn, 2)[rr][qq], E(sc, 2)[rr][qq]);
        } else {
            dA = xs(E(sn, 1)[rr][qq], E(sc, 1)[rr][qq]);
            dB = xs(E(sc, 0)[rr + 1][qq], E(sc, 0)[rr][qq]);
        }
        return upd_h(H(sc, c)[rr][qq], cbh, xs(dA, dB));
    };

    int pprev = ib > 0 ? ib - 1 : (px ? a.nx - 1 : -1);
    int pf = ib;
    issue(NS - 1, pprev);
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) issue(s, pf);
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    wait_slot(NS - 1);
    wait_slot(0);
    if (__syncthreads_or(failed)) return false;
    T prevHy[2] = {T(0), T(0)}, prevHz[2] = {T(0), T(0)};
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int r = ty + u * TJ + 1;
        prevHy[u] = H(NS - 1, 1)[r][q];
        prevHz[u] = H(NS - 1, 2)[r][q];
        if (pprev >= 0) {
            prevHy[u] = hval(1, NS - 1, 0, r, q);
            prevHz[u] = hval(2, NS - 1, 0, r, q);
        }
    }
    __syncthreads();  // slot NS-1 may now be refilled

    int sc = 0;
    for (int i = ib; i < ie; i++) {
        const int sn = sc == NS - 1 ? 0 : sc + 1;
        const int sf = sc == 0 ? NS - 1 : sc - 1;
        if (pf >= 0 && i + NS - 1 <= ie) {
            issue(sf, pf);
            pf = plane_after(pf, a.nx, px);
        }
        wait_slot(sn);
        T(*sH)[TR + 1][33] = sHb[(i - ib) & 1];
        T e0[2], e1[2], e2[2], hy[2], hz[2];
        int code[2];
        long long c[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int row = ty + u * TJ, r = row + 1;
            e0[u] = E(sc, 0)[r][q];
            e1[u] = E(sc, 1)[r][q];
            e2[u] = E(sc, 2)[r][q];
            code[u] = with_codes ? (int)CODE(sc)[row][tx] : 0;
            c[u] = (long long)i * a.plane + (long long)(j0 + row) * a.pitch + (k0 + tx);
            const T hx = hval(0, sc, sn, r, q);
            hy[u] = hval(1, sc, sn, r, q);
            hz[u] = hval(2, sc, sn, r, q);
            a.Ho[0][c[u]] = hx;
            a.Ho[1][c[u]] = hy[u];
            a.Ho[2][c[u]] = hz[u];
            sH[0][r][qs] = hx;
            sH[1][r][qs] = hy[u];
            sH[2][r][qs] = hz[u];
        }
        // halo: row (j0-1) Hx by warp 0, Hz by warp 2; column (k0-1) Hx by
        // warp 1, Hy by warp 3 (lanes of the tile's 2 TJ rows)
        if (ty == 0) sH[0][0][qs] = hval(0, sc, sn, 0, q);
        else if (ty == 2) sH[2][0][qs] = hval(2, sc, sn, 0, q);
        else if (ty == 1 && colh) sH[0][tx + 1][0] = hval(0, sc, sn, tx + 1, 3);
        else if (ty == 3 && colh) sH[1][tx + 1][0] = hval(1, sc, sn, tx + 1, 3);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int r = ty + u * TJ + 1;
            if (!with_codes || code[u] != LIST_CODE) {
                const T ca = tt.tab[code[u]], cb = tt.tab[256 + code[u]];
                a.Eo[0][c[u]] = upd_e(ca, e0[u], cb, xs(xs(sH[2][r][qs], sH[2][r - 1][qs]),
                                                          xs(sH[1][r][qs], sH[1][r][qs - 1])));
                a.Eo[1][c[u]] = upd_e(ca, e1[u], cb, xs(xs(sH[0][r][qs], sH[0][r][qs - 1]), xs(hz[u], prevHz[u])));
                a.Eo[2][c[u]] = upd_e(ca, e2[u], cb, xs(xs(hy[u], prevHy[u]), xs(sH[0][r][qs], sH[0][r - 1][qs])));
            }
            prevHy[u] = hy[u];
            prevHz[u] = hz[u];
        }
        sc = sn;
    }
    return !__syncthreads_or(failed);
}

// The interior queue with tiles of two rows per thread (KIND 0 items of
// 2 TJ rows).
template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB)
    k_sweep_q_i2(Args<T> a, const SweepItem *items, int n_items, const __grid_constant__ TmaMaps maps, int *queue,
                 int *err) {
    static_assert(NS >= 3 && TJ >= 5, "ring of three planes; warps 0-3 recompute halos, warp 4 issues copies");
    using S = QLayoutI2<T, TJ, NS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (q_misaligned(smem_raw, err)) return;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::bars);
    volatile int *s_item = reinterpret_cast<volatile int *>(smem_raw + S::misc);
    q_init_bars<NS>(bars);
    {
        TileTables<T, TJ> &tt = *reinterpret_cast<TileTables<T, TJ> *>(smem_raw + S::tabs);
        const int tid = threadIdx.y * 32 + threadIdx.x;
        for (int t = tid; t < 256; t += 32 * TJ) {
            tt.tab[t] = a.tca[t];
            tt.tab[256 + t] = a.tcb[t];
        }
    }
    __syncthreads();
    unsigned phase = 0, pending = 0;
    bool failed = false;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) *s_item = atomicAdd(&queue[0], 1);
        __syncthreads();
        const int w = *s_item;
        if (w >= n_items) break;
        const SweepItem it = items[w];
        if (!q_item_i2<T, TJ, NS>(a, maps, it, smem_raw, phase, pending, failed)) {
            q_bail<NS>(bars, phase, pending, err);
            break;
        }
        __syncthreads();
    }
    q_leave(queue);
}

// Variants of the two-rows interior (FP32 only): (TJ, NS, CTAs per SM).
#define RFB_QI2_VARIANTS(X) X(8, 3, 3) X(8, 4, 2)

template <typename T>
inline int qi2_grid(int ns) {
    static int g[8] = {};
    int &gv = g[ns & 7];
    if (!gv) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
#define RFB_QI2_OCC(TJ_, NS_, MB_)                                                                         \
        if (ns == NS_)                                                                                     \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweep_q_i2<float, TJ_, NS_, MB_>, 32 * TJ_, \
                                                          QLayoutI2<float, TJ_, NS_>::total);
        RFB_QI2_VARIANTS(RFB_QI2_OCC)
#undef RFB_QI2_OCC
        gv = (sms > 0 ? sms : 148) * (per > 0 ? per : 1);
    }
    return gv;
}

// Launch over n two-row interior items (FP32; plan variant `ns`).
inline void launch_q_i2(const Args<float> &a, int ns, const SweepItem *items, int n, const TmaMaps &m, int *queue,
                        int *err, cudaStream_t st) {
    if (n <= 0) return;
#define RFB_QI2_LAUNCH(TJ_, NS_, MB_)                                                                      \
    if (ns == NS_) {                                                                                       \
        const int g = std::min(n, qi2_grid<float>(NS_));                                                   \
        k_sweep_q_i2<float, TJ_, NS_, MB_><<<g, dim3(32, TJ_), QLayoutI2<float, TJ_, NS_>::total, st>>>(    \
            a, items, n, m, queue, err);                                                                   \
    }
    RFB_QI2_VARIANTS(RFB_QI2_LAUNCH)
#undef RFB_QI2_LAUNCH
}

static inline int qi2_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaSuccess;
#define RFB_QI2_PREP(TJ_, NS_, MB_)                                                                        \
    if (e == cudaSuccess)                                                                                  \
        e = cudaFuncSetAttribute(k_sweep_q_i2<float, TJ_, NS_, MB_>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)QLayoutI2<float, TJ_, NS_>::total);                                  \
    if (e == cudaSuccess) (void)qi2_grid<float>(NS_);
    RFB_QI2_VARIANTS(RFB_QI2_PREP)
#undef RFB_QI2_PREP
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

// Variants (element type, TJ, NS, CTAs per SM of the interior and of the
// edge instantiation): interior and edge share the tile height and ring
// depth of a plan.
#define RFB_Q_VARIANTS_FP32(X) X(float, 8, 4, 4, 4) X(float, 8, 3, 5, 3) X(float, 16, 3, 2, 2)
#define RFB_Q_VARIANTS_FP64(X) X(double, 8, 3, 3, 2) X(double, 8, 4, 2, 2)

template <typename T, int TJ, int NS, int MINB, int KIND>
inline int q_grid() {
    static int g = 0;
    if (!g) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweep_q<T, TJ, NS, MINB, KIND>, 32 * TJ,
                                                      QLayout<T, TJ, NS>::total);
        g = (sms > 0 ? sms : 148) * (per > 0 ? per : 1);
    }
    return g;
}

// Launch of one instantiation over n items; the grid never exceeds the items.
// q_grid is first evaluated in q_prepare, outside any stream capture.
#define RFB_LAUNCH_Q(TT, TJ_, NS_, MBI_, MBE_)                                                               \
    if (tj == TJ_ && ns == NS_) {                                                                            \
        constexpr int MB_ = KIND == 0 ? MBI_ : MBE_;                                                         \
        const int g = std::min(n, q_grid<TT, TJ_, NS_, MB_, KIND>());                                        \
        k_sweep_q<TT, TJ_, NS_, MB_, KIND><<<g, dim3(32, TJ_), QLayout<TT, TJ_, NS_>::total, st>>>(          \
            a, d, items, n, m, queue, err);                                                                  \
    }
template <typename T, int KIND>
void launch_q(const Args<T> &a, const FusedDims &d, int tj, int ns, const SweepItem *items, int n, const TmaMaps &m,
              int *queue, int *err, cudaStream_t st);
template <int KIND>
inline void launch_q_f(const Args<float> &a, const FusedDims &d, int tj, int ns, const SweepItem *items, int n,
                       const TmaMaps &m, int *queue, int *err, cudaStream_t st) {
    if (n <= 0) return;
    RFB_Q_VARIANTS_FP32(RFB_LAUNCH_Q)
}
template <int KIND>
inline void launch_q_d(const Args<double> &a, const FusedDims &d, int tj, int ns, const SweepItem *items, int n,
                       const TmaMaps &m, int *queue, int *err, cudaStream_t st) {
    if (n <= 0) return;
    RFB_Q_VARIANTS_FP64(RFB_LAUNCH_Q)
}

#define RFB_PREP_Q(TT, TJ_, NS_, MBI_, MBE_)                                                                \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_q<TT, TJ_, NS_, MBI_, 0>,                                         \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_q<TT, TJ_, NS_, MBE_, 1>,                                         \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_q<TT, TJ_, NS_, MBE_, 2>,                                         \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_sweep_q<TT, TJ_, NS_, MBE_, 5>,                                         \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QLayout<TT, TJ_, NS_>::total); \
    if (e == cudaSuccess) {                                                                                 \
        (void)q_grid<TT, TJ_, NS_, MBI_, 0>();                                                             \
        (void)q_grid<TT, TJ_, NS_, MBE_, 1>();                                                             \
        (void)q_grid<TT, TJ_, NS_, MBE_, 2>();                                                             \
        (void)q_grid<TT, TJ_, NS_, MBE_, 5>();                                                             \
    }
static inline int q_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaSuccess;
    RFB_Q_VARIANTS_FP32(RFB_PREP_Q)
    RFB_Q_VARIANTS_FP64(RFB_PREP_Q)
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

#define RFB_Q_ENTRY(TT, TJ_, NS_, MBI_, MBE_) {TJ_, NS_, MBI_},
static const InteriorVariant kQVariantsFp32[] = {RFB_Q_VARIANTS_FP32(RFB_Q_ENTRY)};
static const InteriorVariant kQVariantsFp64[] = {RFB_Q_VARIANTS_FP64(RFB_Q_ENTRY)};

}  // namespace rfb
