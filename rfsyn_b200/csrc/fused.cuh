// fused.cuh -- one-launch-per-step H+E sweep (2.5D march along i).
//
// The grid is cut into column tiles of (TJ x 32) cells in (j, k); a work item
// is one tile and a range of i planes.  A CTA marches its range plane by
// plane.  Per plane p a stage of shared memory holds E^n(p) with a one-cell
// halo in j and k, H^{n-1/2}(p) of the tile plus its low-j / low-k halo cells
// and the tile's material codes; stages form an NS-deep ring filled by
// cp.async NS-1 planes ahead, so while plane i is computed the next planes
// are in flight from HBM.
//
// Plane i: H^{n+1/2}(i) is computed for the tile (stored) and for its halo
// (recomputed, never stored) from E(i), E(i+1) and H_in(i); E^{n+1}(i) then
// follows from shared H(i) and the H(i-1) values of the previous plane kept
// in registers.  Fields and the H-side psi are ping-ponged between two
// buffers, so a halo recomputation always reads step-n data even when the
// owning CTA has already written step n+1.  Per cell-step the sweep moves the
// compulsory 6 reads + 6 writes of the field components (48 B in FP32).
//
// Two kernels make up one step's sweep (they run concurrently on two streams
// and touch disjoint cells):
//   k_sweep_interior -- items whose tiles and planes lie outside every CPML
//     slab and PEC boundary: branch-free, no psi;
//   k_sweep_edge -- all other items: rfsyn's per-component update ranges and
//     the slab psi recursions, with psi and profile values staged in shared
//     memory by the same cp.async ring, so no global load sits on the
//     compute path.
#pragma once
#include <algorithm>

#include "engine.h"
#include "kernels.cuh"

namespace rfb {

struct FusedDims {
    int cj, ck, ci;   // covered extents: j in [0,cj), k in [0,ck), planes [0,ci)
};

struct SweepItem {
    int j0, k0, ib, ie;
    // slab / boundary tiles of the work-queue sweep: 0 any (y and z slabs,
    // boundaries), 1 no z-slab cell in the tile or its halo, 2 no y-slab
    // cell, 3 narrow tile without y-slab cells, 4 any narrow tile; in the
    // single-queue sweep also 5 interior and 6 x-slab items
    int sub = 0;
};

struct FusedPlan {
    int tj = 8, ns = 6;   // interior variant (rows per tile, ring depth)
    // interior planes staged per thread by cp.async (0), by the TMA (1), or
    // (2, 3) interior and slab tiles both by the TMA in the persistent
    // work-queue sweeps k_sweep_q (sweep.cuh); 3 shifts the tile origins of
    // axes without wrap so that interior tiles start right after the slab
    int tma = 0;
    FusedDims d;
    int seg_int = 64, seg_edge = 32;
    int n_int = 0, n_edge = 0;
    SweepItem *d_int = nullptr, *d_edge = nullptr;  // device work lists
    // modes >= 2, uni = 1: every item (interior sub 5, x slab sub 6, slab /
    // boundary subs 0-4) in the one edge list, one launch of k_sweep_q<KIND 5>
    int uni = 0;
    // modes 2, 3, FP32: 0, or the ring depth of the interior sweep whose
    // threads own two rows of a 2 tj-row tile (k_sweep_q_i2); its interior
    // items are then 2 tj rows high
    int i2 = 0;
    int n_qe = 0, n_qx = 0;                         // modes 2, 3: edge and x-slab items of k_sweep_q
    SweepItem *d_qe = nullptr, *d_qx = nullptr;
    int *d_queue = nullptr;                         // counters (interior 0-1, edge 2-3, x slab 4-5)
};

template <typename T>
__device__ __forceinline__ void cp_async(T *smem, const T *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = valid ? (int)sizeof(T) : 0;
    if (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_u32(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T, int TJ>
struct FusedStage {
    T e[3][TJ + 2][34];   // E^n(p): rows j0-1 .. j0+TJ, cols k0-1 .. k0+32
    T h[3][TJ + 1][33];   // H_in(p): rows j0-1 .. j0+TJ-1, cols k0-1 .. k0+31
    uint32_t code[TJ][8]; // material codes of the tile (32 bytes per row)
};

// Edge stage: the fields plus the psi of plane p at the positions of h:
// slots 0-5 hold the H-side psi arrays (hx_y hx_z hy_z hy_x hz_x hz_y),
// slots 6-11 the E-side ones (ex_y ex_z ey_z ey_x ez_x ez_y, own cells only).
template <typename T, int TJ>
struct EdgeStage {
    FusedStage<T, TJ> f;
    T psi[12][TJ + 1][33];
};

__device__ __forceinline__ int wrap_coord(int q, int n, bool periodic, bool &valid) {
    valid = true;
    if (periodic) {
        if (q < 0) return q + n;
        if (q >= n) return q - n;
        return q;
    }
    if (q < 0 || q > n) valid = false;
    return q;
}

// In-plane element offsets a thread copies every plane, computed once.
struct IssuePlan {
    int own_off;   // own (j, k) offset or -1
    int job;       // 0 none, 1 E halo, 2 H halo row, 3 H halo column, 4 codes
    int job_off;   // offset (elements; bytes for codes) or -1
    int job_r, job_q;
};

template <typename T, int TJ>
__device__ __forceinline__ IssuePlan make_issue_plan(const Args<T> &a, int j0, int k0, int tid) {
    const bool py = a.per & 2u, pz = a.per & 4u;
    IssuePlan ip;
    const int tx = tid & 31, ty = tid >> 5;
    bool vj, vk;
    int jj = wrap_coord(j0 + ty, a.ny, py, vj);
    int kk = wrap_coord(k0 + tx, a.nz, pz, vk);
    ip.own_off = (vj && vk) ? jj * (int)a.pitch + kk : -1;
    ip.job = 0;
    ip.job_off = -1;
    ip.job_r = ip.job_q = 0;
    int jb = tid;
    constexpr int J_EROW = 64, J_ECOL = 2 * (TJ + 2), J_HROW = 32, J_HCOL = TJ, J_CODE = 8 * TJ;
    if (jb < J_EROW) {
        ip.job = 1;
        ip.job_r = jb < 32 ? 0 : TJ + 1;
        ip.job_q = (jb & 31) + 1;
    } else if ((jb -= J_EROW) < J_ECOL) {
        ip.job = 1;
        ip.job_r = jb >> 1;
        ip.job_q = (jb & 1) ? 33 : 0;
    } else if ((jb -= J_ECOL) < J_HROW) {
        ip.job = 2;
        ip.job_r = 0;
        ip.job_q = jb + 1;
    } else if ((jb -= J_HROW) < J_HCOL) {
        ip.job = 3;
        ip.job_r = jb + 1;
        ip.job_q = 0;
    } else if ((jb -= J_HCOL) < J_CODE) {
        ip.job = 4;
        ip.job_r = jb >> 3;
        ip.job_q = jb & 7;
    }
    if (ip.job == 1 || ip.job == 2 || ip.job == 3) {
        jj = wrap_coord(j0 - 1 + ip.job_r, a.ny, py, vj);
        kk = wrap_coord(k0 - 1 + ip.job_q, a.nz, pz, vk);
        ip.job_off = (vj && vk) ? jj * (int)a.pitch + kk : -1;
    } else if (ip.job == 4) {
        const int j = j0 + ip.job_r, k = k0 + 4 * ip.job_q;
        ip.job_off = (a.codes && j >= 0 && k >= 0 && j <= a.ny && k <= a.nz) ? j * (int)a.pitch + k : -1;
    }
    return ip;
}

// Issues the cp.async copies of the fields of plane p into stage st (p < 0:
// zeros).
template <typename T, int TJ>
__device__ __forceinline__ void fused_issue(const Args<T> &a, FusedStage<T, TJ> &st, int p, const IssuePlan &ip,
                                            int r, int q) {
    const bool vp = p >= 0;
    const long long pb = vp ? (long long)p * a.plane : 0;
    const T *zero = a.E[0];
    {
        const bool v = vp && ip.own_off >= 0;
        const long long o = pb + ip.own_off;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            cp_async(&st.e[c][r][q], v ? a.E[c] + o : zero, v);
            cp_async(&st.h[c][r][q], v ? a.H[c] + o : zero, v);
        }
    }
    const bool v = vp && ip.job_off >= 0;
    const long long o = pb + ip.job_off;
    if (ip.job == 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) cp_async(&st.e[c][ip.job_r][ip.job_q], v ? a.E[c] + o : zero, v);
    } else if (ip.job == 2) {
        cp_async(&st.h[0][0][ip.job_q], v ? a.H[0] + o : zero, v);
        cp_async(&st.h[2][0][ip.job_q], v ? a.H[2] + o : zero, v);
    } else if (ip.job == 3) {
        cp_async(&st.h[0][ip.job_r][0], v ? a.H[0] + o : zero, v);
        cp_async(&st.h[1][ip.job_r][0], v ? a.H[1] + o : zero, v);
    } else if (ip.job == 4) {
        cp_async_u32(&st.code[ip.job_r][ip.job_q], v ? (const void *)(a.codes + o) : (const void *)zero, v);
    }
}

__device__ __forceinline__ int plane_after(int i, int nx, bool px) {
    int p = i + 1;
    if (p == nx && px) return 0;
    if (p > nx) return -1;
    return p;
}

// Unstretched H of component c at stage position (r, q).
template <typename T, int TJ>
__device__ __forceinline__ T h_interior(int c, T cbh, const FusedStage<T, TJ> &cur, const FusedStage<T, TJ> &nxt,
                                        int r, int q) {
    if (c == 0)
        return upd_h(cur.h[0][r][q], cbh, xs(xs(cur.e[2][r + 1][q], cur.e[2][r][q]), xs(cur.e[1][r][q + 1], cur.e[1][r][q])));
    if (c == 1)
        return upd_h(cur.h[1][r][q], cbh, xs(xs(cur.e[0][r][q + 1], cur.e[0][r][q]), xs(nxt.e[2][r][q], cur.e[2][r][q])));
    return upd_h(cur.h[2][r][q], cbh, xs(xs(nxt.e[1][r][q], cur.e[1][r][q]), xs(cur.e[0][r + 1][q], cur.e[0][r][q])));
}

// ---------------------------------------------------------------------------
// Interior sweep: every cell of every plane of the item is updated with the
// unstretched formulas (the host-built item list guarantees it).
// ---------------------------------------------------------------------------
template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB) k_sweep_interior(Args<T> a, FusedDims d, const SweepItem *items) {
    extern __shared__ __align__(16) unsigned char smem_cp[];
    FusedStage<T, TJ> *stage = reinterpret_cast<FusedStage<T, TJ> *>(smem_cp);
    T(*sH)[TJ + 1][33] = reinterpret_cast<T(*)[TJ + 1][33]>(smem_cp + NS * sizeof(FusedStage<T, TJ>));
    T *s_tab = reinterpret_cast<T *>(smem_cp + NS * sizeof(FusedStage<T, TJ>) + sizeof(T) * 3 * (TJ + 1) * 33);

    const SweepItem it = items[blockIdx.x];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const bool px = a.per & 1u;
    const int r = ty + 1, q = tx + 1;
    const IssuePlan ip = make_issue_plan<T, TJ>(a, j0, k0, tid);
    (void)d;
    for (int t = tid; t < 256; t += 32 * TJ) {
        s_tab[t] = a.tca[t];
        s_tab[256 + t] = a.tcb[t];
    }
    const T cbh = a.cbh;
    const int pprev = ib > 0 ? ib - 1 : a.nx - 1;  // ib == 0 only on a periodic x axis
    fused_issue<T, TJ>(a, stage[NS - 1], pprev, ip, r, q);
    cp_async_commit();
    int pf = ib;
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) fused_issue<T, TJ>(a, stage[s], pf, ip, r, q);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    cp_async_wait<NS - 2>();
    __syncthreads();
    T prevHy = h_interior<T, TJ>(1, cbh, stage[NS - 1], stage[0], r, q);
    T prevHz = h_interior<T, TJ>(2, cbh, stage[NS - 1], stage[0], r, q);
    __syncthreads();

    int sc = 0;
    for (int i = ib; i < ie; i++) {
        const int sn = sc == NS - 1 ? 0 : sc + 1;
        const int sf = sc == 0 ? NS - 1 : sc - 1;
        if (pf >= 0 && i + NS - 1 <= ie) fused_issue<T, TJ>(a, stage[sf], pf, ip, r, q);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
        cp_async_wait<NS - 2>();
        __syncthreads();
        const FusedStage<T, TJ> &cur = stage[sc];
        const FusedStage<T, TJ> &nxt = stage[sn];
        const T e0 = cur.e[0][r][q], e1 = cur.e[1][r][q], e2 = cur.e[2][r][q];
        const int code = (int)((cur.code[ty][tx >> 2] >> (8 * (tx & 3))) & 0xffu);
        const long long c = (long long)i * a.plane + (long long)ip.own_off;
        const T hx = h_interior<T, TJ>(0, cbh, cur, nxt, r, q);
        const T hy = h_interior<T, TJ>(1, cbh, cur, nxt, r, q);
        const T hz = h_interior<T, TJ>(2, cbh, cur, nxt, r, q);
        a.Ho[0][c] = hx;
        a.Ho[1][c] = hy;
        a.Ho[2][c] = hz;
        sH[0][r][q] = hx;
        sH[1][r][q] = hy;
        sH[2][r][q] = hz;
        if (ty == 0) {
            sH[0][0][q] = h_interior<T, TJ>(0, cbh, cur, nxt, 0, q);
            sH[2][0][q] = h_interior<T, TJ>(2, cbh, cur, nxt, 0, q);
        } else if (ty == 1 && tx < TJ) {
            sH[0][tx + 1][0] = h_interior<T, TJ>(0, cbh, cur, nxt, tx + 1, 0);
            sH[1][tx + 1][0] = h_interior<T, TJ>(1, cbh, cur, nxt, tx + 1, 0);
        }
        __syncthreads();
        if (!a.codes || code != LIST_CODE) {
            const T ca = s_tab[code], cb = s_tab[256 + code];
            a.Eo[0][c] = upd_e(ca, e0, cb, xs(xs(sH[2][r][q], sH[2][r - 1][q]), xs(sH[1][r][q], sH[1][r][q - 1])));
            a.Eo[1][c] = upd_e(ca, e1, cb, xs(xs(sH[0][r][q], sH[0][r][q - 1]), xs(hz, prevHz)));
            a.Eo[2][c] = upd_e(ca, e2, cb, xs(xs(hy, prevHy), xs(sH[0][r][q], sH[0][r - 1][q])));
        }
        prevHy = hy;
        prevHz = hz;
        sc = sn;
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Edge sweep
// ---------------------------------------------------------------------------
// Profile triple (kappa_inv, b, a) at index q of an axis profile of length
// len, identity outside it or when the axis has no CPML.
template <typename T>
__device__ __forceinline__ void prof_at(const T *kinv, const T *b, const T *ac, int q, int len, T *out) {
    if (kinv && q >= 0 && q < len) {
        out[0] = kinv[q];
        out[1] = b[q];
        out[2] = ac[q];
    } else {
        out[0] = T(1);
        out[1] = T(1);
        out[2] = T(0);
    }
}

// Slab index of q, -1 in the unstretched interior or outside [0, len).
__device__ __forceinline__ int slab_in(int q, int lo, int hi, int len, int on) {
    if (!on || q < 0 || q >= len) return -1;
    return slab_of(q, lo, hi);
}

// Per-CTA profile tables in shared memory.
template <typename T, int TJ>
struct EdgeShared {
    T py[6][TJ + 1];   // y profile (h: kinv b a, m: kinv b a) at rows j0-1 .. j0+TJ-1
    T pz[6][33];       // z profile at cols k0-1 .. k0+31
};

// rfsyn's cpml_term with the psi state passed by value: psi_new = b psi +
// a d (written to *psi_out), returns d kappa_inv + dx psi_new.
template <typename T>
__device__ __forceinline__ T stretch(T d, T kinv, T b, T ac, T dx, T psi_old, T *psi_out) {
    T pn = cpml_psi(b, psi_old, ac, d);
    *psi_out = pn;
    return cpml_out(d, kinv, dx, pn);
}

template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB) k_sweep_edge(Args<T> a, FusedDims d, const SweepItem *items) {
    extern __shared__ __align__(16) unsigned char smem_cp[];
    EdgeStage<T, TJ> *stage = reinterpret_cast<EdgeStage<T, TJ> *>(smem_cp);
    unsigned char *after = smem_cp + NS * sizeof(EdgeStage<T, TJ>);
    T(*sH)[TJ + 1][33] = reinterpret_cast<T(*)[TJ + 1][33]>(after);
    T *s_tab = reinterpret_cast<T *>(after + sizeof(T) * 3 * (TJ + 1) * 33);
    EdgeShared<T, TJ> &es =
        *reinterpret_cast<EdgeShared<T, TJ> *>(after + sizeof(T) * 3 * (TJ + 1) * 33 + sizeof(T) * 512);

    const SweepItem it = items[blockIdx.x];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int j0 = it.j0, k0 = it.k0, ib = it.ib, ie = it.ie;
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const int j = j0 + ty, k = k0 + tx;
    // tiles may start at negative coordinates on an axis without wrap (the
    // work-queue plans shift the tile origins); cells outside the grid idle
    const bool own = j >= 0 && k >= 0 && j < d.cj && k < d.ck;
    const bool row_halo = (j0 > 0 || py);
    const bool col_halo = (k0 > 0 || pz);
    const int jh = j0 > 0 ? j0 - 1 : a.ny - 1;
    const int kh = k0 > 0 ? k0 - 1 : a.nz - 1;
    const int r = ty + 1, q = tx + 1;
    const IssuePlan ip = make_issue_plan<T, TJ>(a, j0, k0, tid);
    const int on = a.cpml_on;
    const long long ny1 = a.ny + 1;

    for (int t = tid; t < 256; t += 32 * TJ) {
        s_tab[t] = a.tca[t];
        s_tab[256 + t] = a.tcb[t];
    }
    for (int t = tid; t < TJ + 1; t += 32 * TJ) {
        const int jj = j0 - 1 + t;
        T v[3];
        prof_at(on ? a.kinv_h[1] : (const T *)nullptr, a.b_h[1], a.a_h[1], jj, a.ny, v);
        es.py[0][t] = v[0]; es.py[1][t] = v[1]; es.py[2][t] = v[2];
        prof_at(on ? a.kinv_m[1] : (const T *)nullptr, a.b_m[1], a.a_m[1], jj, a.ny + 1, v);
        es.py[3][t] = v[0]; es.py[4][t] = v[1]; es.py[5][t] = v[2];
    }
    for (int t = tid; t < 33; t += 32 * TJ) {
        const int kk = k0 - 1 + t;
        T v[3];
        prof_at(on ? a.kinv_h[2] : (const T *)nullptr, a.b_h[2], a.a_h[2], kk, a.nz, v);
        es.pz[0][t] = v[0]; es.pz[1][t] = v[1]; es.pz[2][t] = v[2];
        prof_at(on ? a.kinv_m[2] : (const T *)nullptr, a.b_m[2], a.a_m[2], kk, a.nz + 1, v);
        es.pz[3][t] = v[0]; es.pz[4][t] = v[1]; es.pz[5][t] = v[2];
    }
    // slab indices of the own cell (H side: q < n; E side: only swept samples
    // use them, and those have q < n)
    const int sjh = slab_in(j, a.lo_h[1], a.hi_h[1], a.ny, on);
    const int skh = slab_in(k, a.lo_h[2], a.hi_h[2], a.nz, on);
    const int sjm = slab_in(j, a.lo_m[1], a.hi_m[1], a.ny, on);
    const int skm = slab_in(k, a.lo_m[2], a.hi_m[2], a.nz, on);
    // halo cells: row (j0-1, k) for warp 0, column (j0+tx, k0-1) for warp 1
    const int sjh_row = slab_in(j0 - 1, a.lo_h[1], a.hi_h[1], a.ny, on);
    const int jc = j0 + tx;
    const int sjh_col = slab_in(jc, a.lo_h[1], a.hi_h[1], a.ny, on);
    const int skh_col = slab_in(k0 - 1, a.lo_h[2], a.hi_h[2], a.nz, on);
    const int nshy = a.ns_h[1], nshz = a.ns_h[2], nsmy = a.ns_m[1], nsmz = a.ns_m[2];

    // psi copies of plane p into stage st
    auto issue_psi = [&](EdgeStage<T, TJ> &st, int p) {
        if (!on || p < 0) return;
        const int sxh = slab_in(p, a.lo_h[0], a.hi_h[0], a.nx, on);
        const int sxm = slab_in(p, a.lo_m[0], a.hi_m[0], a.nx, on);
        if (own) {
            if (sjh >= 0) {
                const long long o = ((long long)p * nshy + sjh) * a.pitch + k;
                cp_async(&st.psi[0][r][q], a.psi_hi[0] + o, true);
                cp_async(&st.psi[5][r][q], a.psi_hi[5] + o, true);
            }
            if (skh >= 0) {
                const long long o = ((long long)p * ny1 + j) * nshz + skh;
                cp_async(&st.psi[1][r][q], a.psi_hi[1] + o, true);
                cp_async(&st.psi[2][r][q], a.psi_hi[2] + o, true);
            }
            if (sxh >= 0) {
                const long long o = ((long long)sxh * ny1 + j) * a.pitch + k;
                cp_async(&st.psi[3][r][q], a.psi_hi[3] + o, true);
                cp_async(&st.psi[4][r][q], a.psi_hi[4] + o, true);
            }
            if (sjm >= 0) {
                const long long o = ((long long)p * nsmy + sjm) * a.pitch + k;
                cp_async(&st.psi[6][r][q], a.psi_e[0] + o, true);
                cp_async(&st.psi[11][r][q], a.psi_e[5] + o, true);
            }
            if (skm >= 0) {
                const long long o = ((long long)p * ny1 + j) * nsmz + skm;
                cp_async(&st.psi[7][r][q], a.psi_e[1] + o, true);
                cp_async(&st.psi[8][r][q], a.psi_e[2] + o, true);
            }
            if (sxm >= 0) {
                const long long o = ((long long)sxm * ny1 + j) * a.pitch + k;
                cp_async(&st.psi[9][r][q], a.psi_e[3] + o, true);
                cp_async(&st.psi[10][r][q], a.psi_e[4] + o, true);
            }
        }
        if (ty == 0 && row_halo && k >= 0 && k < d.ck) {
            // row halo (j0-1, k): Hx (hx_y, hx_z), Hz (hz_x, hz_y)
            if (sjh_row >= 0) {
                const long long o = ((long long)p * nshy + sjh_row) * a.pitch + k;
                cp_async(&st.psi[0][0][q], a.psi_hi[0] + o, true);
                cp_async(&st.psi[5][0][q], a.psi_hi[5] + o, true);
            }
            if (skh >= 0) {
                const long long o = ((long long)p * ny1 + jh) * nshz + skh;
                cp_async(&st.psi[1][0][q], a.psi_hi[1] + o, true);
            }
            if (sxh >= 0) {
                const long long o = ((long long)sxh * ny1 + jh) * a.pitch + k;
                cp_async(&st.psi[4][0][q], a.psi_hi[4] + o, true);
            }
        } else if (ty == 1 && tx < TJ && col_halo && jc >= 0 && jc < d.cj) {
            // column halo (j0+tx, k0-1): Hx (hx_y, hx_z), Hy (hy_z, hy_x)
            if (sjh_col >= 0) {
                const long long o = ((long long)p * nshy + sjh_col) * a.pitch + kh;
                cp_async(&st.psi[0][tx + 1][0], a.psi_hi[0] + o, true);
            }
            if (skh_col >= 0) {
                const long long o = ((long long)p * ny1 + jc) * nshz + skh_col;
                cp_async(&st.psi[1][tx + 1][0], a.psi_hi[1] + o, true);
                cp_async(&st.psi[2][tx + 1][0], a.psi_hi[2] + o, true);
            }
            if (sxh >= 0) {
                const long long o = ((long long)sxh * ny1 + jc) * a.pitch + kh;
                cp_async(&st.psi[3][tx + 1][0], a.psi_hi[3] + o, true);
            }
        }
    };
    auto issue = [&](EdgeStage<T, TJ> &st, int p) {
        fused_issue<T, TJ>(a, st.f, p, ip, r, q);
        issue_psi(st, p);
    };

    // H of component c at plane i for the cell at stage (rr, qq) with
    // coordinates (jj, kk); sy / sz its H-side y / z slab indices, yi / zi
    // its rows in the profile tables; store: the owner writes the new psi.
    auto h_edge = [&](int c, int i, int jj, int kk, int rr, int qq, int sy, int sz, int yi, int zi,
                      const EdgeStage<T, TJ> &cs, const EdgeStage<T, TJ> &ns, bool store) -> T {
        const FusedStage<T, TJ> &cur = cs.f, &nxt = ns.f;
        const T hin = cur.h[c][rr][qq];
        const int sx = slab_in(i, a.lo_h[0], a.hi_h[0], a.nx, on);
        T dA, dB;
        if (c == 0) {
            if (!(i < a.nx + (px ? 0 : 1) && jj < a.ny && kk < a.nz)) return hin;
            dA = xs(cur.e[2][rr + 1][qq], cur.e[2][rr][qq]);
            dB = xs(cur.e[1][rr][qq + 1], cur.e[1][rr][qq]);
            if (sy >= 0) {
                T pn;
                dA = stretch(dA, es.py[0][yi], es.py[1][yi], es.py[2][yi], a.dx, cs.psi[0][rr][qq], &pn);
                if (store) a.psi_ho[0][((long long)i * nshy + sy) * a.pitch + kk] = pn;
            }
            if (sz >= 0) {
                T pn;
                dB = stretch(dB, es.pz[0][zi], es.pz[1][zi], es.pz[2][zi], a.dx, cs.psi[1][rr][qq], &pn);
                if (store) a.psi_ho[1][((long long)i * ny1 + jj) * nshz + sz] = pn;
            }
        } else if (c == 1) {
            if (!(i < a.nx && jj < a.ny + (py ? 0 : 1) && kk < a.nz)) return hin;
            dA = xs(cur.e[0][rr][qq + 1], cur.e[0][rr][qq]);
            dB = xs(nxt.e[2][rr][qq], cur.e[2][rr][qq]);
            if (sz >= 0) {
                T pn;
                dA = stretch(dA, es.pz[0][zi], es.pz[1][zi], es.pz[2][zi], a.dx, cs.psi[2][rr][qq], &pn);
                if (store) a.psi_ho[2][((long long)i * ny1 + jj) * nshz + sz] = pn;
            }
            if (sx >= 0) {
                T pn;
                dB = stretch(dB, a.kinv_h[0][i], a.b_h[0][i], a.a_h[0][i], a.dx, cs.psi[3][rr][qq], &pn);
                if (store) a.psi_ho[3][((long long)sx * ny1 + jj) * a.pitch + kk] = pn;
            }
        } else {
            if (!(i < a.nx && jj < a.ny && kk < a.nz + (pz ? 0 : 1))) return hin;
            dA = xs(nxt.e[1][rr][qq], cur.e[1][rr][qq]);
            dB = xs(cur.e[0][rr + 1][qq], cur.e[0][rr][qq]);
            if (sx >= 0) {
                T pn;
                dA = stretch(dA, a.kinv_h[0][i], a.b_h[0][i], a.a_h[0][i], a.dx, cs.psi[4][rr][qq], &pn);
                if (store) a.psi_ho[4][((long long)sx * ny1 + jj) * a.pitch + kk] = pn;
            }
            if (sy >= 0) {
                T pn;
                dB = stretch(dB, es.py[0][yi], es.py[1][yi], es.py[2][yi], a.dx, cs.psi[5][rr][qq], &pn);
                if (store) a.psi_ho[5][((long long)i * nshy + sy) * a.pitch + kk] = pn;
            }
        }
        return upd_h(hin, a.cbh, xs(dA, dB));
    };

    T prevHy = 0, prevHz = 0;
    int pprev = -1;
    if (ib > 0) pprev = ib - 1;
    else if (px) pprev = a.nx - 1;
    if (pprev >= 0) {
        issue(stage[NS - 1], pprev);
        cp_async_commit();
    }
    int pf = ib;
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) issue(stage[s], pf);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    if (pprev >= 0) {
        cp_async_wait<NS - 2>();
        __syncthreads();
        if (own) {
            prevHy = h_edge(1, pprev, j, k, r, q, sjh, skh, r, q, stage[NS - 1], stage[0], false);
            prevHz = h_edge(2, pprev, j, k, r, q, sjh, skh, r, q, stage[NS - 1], stage[0], false);
        }
    }
    __syncthreads();  // profile tables visible; prologue slot free

    int sc = 0;
    for (int i = ib; i < ie; i++) {
        const int sn = sc == NS - 1 ? 0 : sc + 1;
        const int sf = sc == 0 ? NS - 1 : sc - 1;
        if (pf >= 0 && i + NS - 1 <= ie) issue(stage[sf], pf);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
        cp_async_wait<NS - 2>();
        __syncthreads();
        const EdgeStage<T, TJ> &cs = stage[sc];
        const EdgeStage<T, TJ> &ns = stage[sn];
        const FusedStage<T, TJ> &cur = cs.f;
        const T e0 = cur.e[0][r][q], e1 = cur.e[1][r][q], e2 = cur.e[2][r][q];
        const int code = (int)((cur.code[ty][tx >> 2] >> (8 * (tx & 3))) & 0xffu);
        const long long c = (long long)i * a.plane + (long long)ip.own_off;
        T hx = 0, hy = 0, hz = 0;
        if (own) {
            hx = h_edge(0, i, j, k, r, q, sjh, skh, r, q, cs, ns, true);
            hy = h_edge(1, i, j, k, r, q, sjh, skh, r, q, cs, ns, true);
            hz = h_edge(2, i, j, k, r, q, sjh, skh, r, q, cs, ns, true);
            a.Ho[0][c] = hx;
            a.Ho[1][c] = hy;
            a.Ho[2][c] = hz;
        }
        sH[0][r][q] = hx;
        sH[1][r][q] = hy;
        sH[2][r][q] = hz;
        if (ty == 0 && row_halo && k >= 0 && k < d.ck) {
            sH[0][0][q] = h_edge(0, i, jh, k, 0, q, sjh_row, skh, 0, q, cs, ns, false);
            sH[2][0][q] = h_edge(2, i, jh, k, 0, q, sjh_row, skh, 0, q, cs, ns, false);
        } else if (ty == 1 && tx < TJ && col_halo && jc >= 0 && jc < d.cj) {
            sH[0][tx + 1][0] = h_edge(0, i, jc, kh, tx + 1, 0, sjh_col, skh_col, tx + 1, 0, cs, ns, false);
            sH[1][tx + 1][0] = h_edge(1, i, jc, kh, tx + 1, 0, sjh_col, skh_col, tx + 1, 0, cs, ns, false);
        }
        __syncthreads();
        if (own && i < a.nx) {
            bool skip;
            if (a.codes) {
                skip = code == LIST_CODE;
            } else {
                skip = false;
                for (int s = 0; s < a.n_skip; s++) skip |= a.skip[s] == c;
            }
            if (!skip) {
                const T ca = s_tab[code], cb = s_tab[256 + code];
                const int sxm = slab_in(i, a.lo_m[0], a.hi_m[0], a.nx, on);
                if (e_updated(a, 0, i, j, k)) {
                    T tA = xs(sH[2][r][q], sH[2][r - 1][q]);
                    T tB = xs(sH[1][r][q], sH[1][r][q - 1]);
                    if (sjm >= 0) {
                        T pn;
                        tA = stretch(tA, es.py[3][r], es.py[4][r], es.py[5][r], a.dx, cs.psi[6][r][q], &pn);
                        a.psi_e[0][((long long)i * nsmy + sjm) * a.pitch + k] = pn;
                    }
                    if (skm >= 0) {
                        T pn;
                        tB = stretch(tB, es.pz[3][q], es.pz[4][q], es.pz[5][q], a.dx, cs.psi[7][r][q], &pn);
                        a.psi_e[1][((long long)i * ny1 + j) * nsmz + skm] = pn;
                    }
                    a.Eo[0][c] = upd_e(ca, e0, cb, xs(tA, tB));
                }
                if (e_updated(a, 1, i, j, k)) {
                    T tA = xs(sH[0][r][q], sH[0][r][q - 1]);
                    T tB = xs(hz, prevHz);
                    if (skm >= 0) {
                        T pn;
                        tA = stretch(tA, es.pz[3][q], es.pz[4][q], es.pz[5][q], a.dx, cs.psi[8][r][q], &pn);
                        a.psi_e[2][((long long)i * ny1 + j) * nsmz + skm] = pn;
                    }
                    if (sxm >= 0) {
                        T pn;
                        tB = stretch(tB, a.kinv_m[0][i], a.b_m[0][i], a.a_m[0][i], a.dx, cs.psi[9][r][q], &pn);
                        a.psi_e[3][((long long)sxm * ny1 + j) * a.pitch + k] = pn;
                    }
                    a.Eo[1][c] = upd_e(ca, e1, cb, xs(tA, tB));
                }
                if (e_updated(a, 2, i, j, k)) {
                    T tA = xs(hy, prevHy);
                    T tB = xs(sH[0][r][q], sH[0][r - 1][q]);
                    if (sxm >= 0) {
                        T pn;
                        tA = stretch(tA, a.kinv_m[0][i], a.b_m[0][i], a.a_m[0][i], a.dx, cs.psi[10][r][q], &pn);
                        a.psi_e[4][((long long)sxm * ny1 + j) * a.pitch + k] = pn;
                    }
                    if (sjm >= 0) {
                        T pn;
                        tB = stretch(tB, es.py[3][r], es.py[4][r], es.py[5][r], a.dx, cs.psi[11][r][q], &pn);
                        a.psi_e[5][((long long)i * nsmy + sjm) * a.pitch + k] = pn;
                    }
                    a.Eo[2][c] = upd_e(ca, e2, cb, xs(tA, tB));
                }
            }
        }
        prevHy = hy;
        prevHz = hz;
        sc = sn;
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Instantiations and launch
// ---------------------------------------------------------------------------
template <typename T, int TJ, int NS>
constexpr size_t interior_smem() {
    return NS * sizeof(FusedStage<T, TJ>) + sizeof(T) * 3 * (TJ + 1) * 33 + sizeof(T) * 512;
}
template <typename T, int TJ, int NS>
constexpr size_t edge_smem() {
    return NS * sizeof(EdgeStage<T, TJ>) + sizeof(T) * 3 * (TJ + 1) * 33 + sizeof(T) * 512 +
           sizeof(EdgeShared<T, TJ>);
}

// Interior variants (TJ, NS, CTAs per SM) the autotuner chooses from, and
// the edge kernels: FP32 edge 3 stages at 3 CTAs/SM, FP64 edge 2 at 2.
#define RFB_INT_VARIANTS_FP32(X) X(float, 8, 6, 4) X(float, 8, 5, 5) X(float, 16, 4, 3) X(float, 16, 3, 4)
#define RFB_INT_VARIANTS_FP64(X) X(double, 8, 4, 3) X(double, 16, 2, 2)
#define RFB_EDGE_FP32 k_sweep_edge<float, 8, 3, 3>
#define RFB_EDGE_FP64 k_sweep_edge<double, 8, 2, 2>

struct InteriorVariant {
    int tj, ns, minb;
};
static const InteriorVariant kIntVariantsFp32[] = {{8, 6, 4}, {8, 5, 5}, {16, 4, 3}, {16, 3, 4}};
static const InteriorVariant kIntVariantsFp64[] = {{8, 4, 3}, {16, 2, 2}};

template <typename T>
void launch_interior(const Args<T> &a, const FusedPlan &p, cudaStream_t st);
template <typename T>
void launch_edge(const Args<T> &a, const FusedPlan &p, cudaStream_t st);

#define RFB_LAUNCH_INT(TT, TJ_, NS_, MB_)                                                                    \
    if (p.tj == TJ_ && p.ns == NS_)                                                                          \
        k_sweep_interior<TT, TJ_, NS_, MB_><<<p.n_int, dim3(32, TJ_), interior_smem<TT, TJ_, NS_>(), st>>>( \
            a, p.d, p.d_int);
template <>
inline void launch_interior<float>(const Args<float> &a, const FusedPlan &p, cudaStream_t st) {
    if (!p.n_int) return;
    RFB_INT_VARIANTS_FP32(RFB_LAUNCH_INT)
}
template <>
inline void launch_interior<double>(const Args<double> &a, const FusedPlan &p, cudaStream_t st) {
    if (!p.n_int) return;
    RFB_INT_VARIANTS_FP64(RFB_LAUNCH_INT)
}
template <>
inline void launch_edge<float>(const Args<float> &a, const FusedPlan &p, cudaStream_t st) {
    if (p.n_edge) RFB_EDGE_FP32<<<p.n_edge, dim3(32, 8), edge_smem<float, 8, 3>(), st>>>(a, p.d, p.d_edge);
}
template <>
inline void launch_edge<double>(const Args<double> &a, const FusedPlan &p, cudaStream_t st) {
    if (p.n_edge) RFB_EDGE_FP64<<<p.n_edge, dim3(32, 8), edge_smem<double, 8, 2>(), st>>>(a, p.d, p.d_edge);
}

// Raises the dynamic shared-memory limit of every sweep instantiation once.
#define RFB_PREP_INT(TT, TJ_, NS_, MB_)                                                            \
    if (e == cudaSuccess)                                                                          \
        e = cudaFuncSetAttribute(k_sweep_interior<TT, TJ_, NS_, MB_>,                             \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)interior_smem<TT, TJ_, NS_>());
static inline int fused_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaSuccess;
    RFB_INT_VARIANTS_FP32(RFB_PREP_INT)
    RFB_INT_VARIANTS_FP64(RFB_PREP_INT)
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(RFB_EDGE_FP32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)edge_smem<float, 8, 3>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(RFB_EDGE_FP64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)edge_smem<double, 8, 2>());
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

// Interior range [lo, hi) of an axis: indices whose profiles are the identity
// on both staggered grids and where every component is swept (index >= 1 on a
// non-periodic axis).
static inline void interior_axis(int lo_h, int hi_h, int lo_m, int hi_m, int n, bool periodic, bool cpml, int *lo,
                                 int *hi) {
    if (periodic) {
        *lo = 0;
        *hi = n;
        return;
    }
    *lo = 1;
    *hi = n;
    if (cpml) {
        *lo = std::max(*lo, std::max(lo_h, lo_m));
        *hi = std::min(*hi, std::min(hi_h, hi_m));
    }
}

}  // namespace rfb
