// fused.cuh -- one-kernel-per-step H+E sweep (2.5D march along i).
//
// Each CTA owns a (TJ x 32) tile of (j, k) and a segment of i planes and
// marches the segment plane by plane.  Per plane p a stage of shared memory
// holds E^n(p) with a one-cell halo in j and k, H^{n-1/2}(p) of the tile plus
// the low-j / low-k halo cells, and the material codes of the tile.  Stages
// live in an NS-deep ring filled by cp.async NS-1 planes ahead, so while
// plane i is computed planes i+1 .. i+NS-1 are in flight from HBM (enough
// bytes in flight per SM to cover HBM latency at full bandwidth).
//
// Plane i: H^{n+1/2}(i) is computed for the tile (stored) and for its halo
// (recomputed redundantly, never stored) from E(i), E(i+1) and H_in(i); then
// E^{n+1}(i) follows from shared H(i) and the H(i-1) values of the previous
// plane kept in registers.  Fields and the H-side psi are ping-ponged between
// two buffers, so a halo recomputation always reads step-n data even when the
// owning CTA has already written step n+1.  Per cell-step the kernel moves the
// compulsory 6 reads + 6 writes of the field components (48 B in FP32).
//
// A (tile, plane) with no CPML slab, no PEC boundary and no skipped cell takes
// a branch-free interior path (uniform per CTA, so no divergence); all other
// planes take the general path with rfsyn's per-component update ranges and
// the slab-stored psi recursions.  Both evaluate identical arithmetic.
#pragma once
#include "engine.h"
#include "kernels.cuh"

namespace rfb {

struct FusedDims {
    int cj, ck, ci;   // covered extents: j in [0,cj), k in [0,ck), planes [0,ci)
    int seg_len;      // planes per CTA segment
};

struct FusedPlan {
    int tj = 8;
    FusedDims d;
    dim3 grid;
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
        ip.job_off = (a.codes && j <= a.ny && k <= a.nz) ? j * (int)a.pitch + k : -1;
    }
    return ip;
}

// Issues the cp.async copies of plane p into stage st (p < 0: zeros).
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

// General-path H^{n+1/2} of component c at plane i from stage-resident E(i)
// (cur), E(i+1) (nxt) and H_in(i); (r, q) is the stage position.  Components
// that rfsyn's loops do not update keep their input value.  store: write the
// new psi (owner) or only use it (halo).
template <typename T, int TJ>
__device__ __forceinline__ T fused_h(const Args<T> &a, int c, int i, int j, int k, const FusedStage<T, TJ> &cur,
                                     const FusedStage<T, TJ> &nxt, int r, int q, bool store) {
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const T hin = cur.h[c][r][q];
    T dA, dB;
    int pA, pB, axA, axB, qA, qB;
    if (c == 0) {
        if (!(i < a.nx + (px ? 0 : 1) && j < a.ny && k < a.nz)) return hin;
        dA = xs(cur.e[2][r + 1][q], cur.e[2][r][q]);
        dB = xs(cur.e[1][r][q + 1], cur.e[1][r][q]);
        pA = 0; axA = 1; qA = j;
        pB = 1; axB = 2; qB = k;
    } else if (c == 1) {
        if (!(i < a.nx && j < a.ny + (py ? 0 : 1) && k < a.nz)) return hin;
        dA = xs(cur.e[0][r][q + 1], cur.e[0][r][q]);
        dB = xs(nxt.e[2][r][q], cur.e[2][r][q]);
        pA = 2; axA = 2; qA = k;
        pB = 3; axB = 0; qB = i;
    } else {
        if (!(i < a.nx && j < a.ny && k < a.nz + (pz ? 0 : 1))) return hin;
        dA = xs(nxt.e[1][r][q], cur.e[1][r][q]);
        dB = xs(cur.e[0][r + 1][q], cur.e[0][r][q]);
        pA = 4; axA = 0; qA = i;
        pB = 5; axB = 1; qB = j;
    }
    T tA = dA, tB = dB;
    if (a.cpml_on) {
        int s = slab_of(qA, a.lo_h[axA], a.hi_h[axA]);
        if (s >= 0) {
            const long long pi = psi_idx(a, axA, a.ns_h[axA], s, i, j, k);
            T pn;
            tA = cpml_step(dA, a.kinv_h[axA][qA], a.b_h[axA][qA], a.a_h[axA][qA], a.dx, a.psi_hi[pA][pi], &pn);
            if (store) a.psi_ho[pA][pi] = pn;
        }
        s = slab_of(qB, a.lo_h[axB], a.hi_h[axB]);
        if (s >= 0) {
            const long long pi = psi_idx(a, axB, a.ns_h[axB], s, i, j, k);
            T pn;
            tB = cpml_step(dB, a.kinv_h[axB][qB], a.b_h[axB][qB], a.a_h[axB][qB], a.dx, a.psi_hi[pB][pi], &pn);
            if (store) a.psi_ho[pB][pi] = pn;
        }
    }
    return xs(hin, xm(a.cbh, xs(tA, tB)));
}

__device__ __forceinline__ int plane_after(int i, int nx, bool px) {
    int p = i + 1;
    if (p == nx && px) return 0;
    if (p > nx) return -1;
    return p;
}

// Range [lo, hi) of a non-periodic axis where both profiles are the identity
// and every component is swept, for tiles that also read index lo-1.
__device__ __forceinline__ void interior_range(int lo_h, int hi_h, int lo_m, int hi_m, int n, bool periodic, int cpml,
                                               int &lo, int &hi) {
    if (periodic) {
        lo = 0;
        hi = n;
        return;
    }
    lo = 1;
    hi = n;
    if (cpml) {
        lo = max(lo, max(lo_h, lo_m));
        hi = min(hi, min(hi_h, hi_m));
    }
}

// NS stages: planes i .. i+NS-2 are resident or in flight while plane i is
// computed (prefetch distance NS-1).
template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB) k_fused(Args<T> a, FusedDims d) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FusedStage<T, TJ> *stage = reinterpret_cast<FusedStage<T, TJ> *>(smem_raw);
    T(*sH)[TJ + 1][33] = reinterpret_cast<T(*)[TJ + 1][33]>(smem_raw + NS * sizeof(FusedStage<T, TJ>));
    T *s_tab = reinterpret_cast<T *>(smem_raw + NS * sizeof(FusedStage<T, TJ>) + sizeof(T) * 3 * (TJ + 1) * 33);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int k0 = blockIdx.x * 32, j0 = blockIdx.y * TJ;
    const int ib = blockIdx.z * d.seg_len;
    const int ie = min(ib + d.seg_len, d.ci);
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const int j = j0 + ty, k = k0 + tx;
    const bool own = j < d.cj && k < d.ck;
    const bool row_halo = (j0 > 0 || py);
    const bool col_halo = (k0 > 0 || pz);
    const int jh = j0 > 0 ? j0 - 1 : a.ny - 1;
    const int kh = k0 > 0 ? k0 - 1 : a.nz - 1;
    const int r = ty + 1, q = tx + 1;
    const IssuePlan ip = make_issue_plan<T, TJ>(a, j0, k0, tid);

    // coefficient table in shared memory
    for (int t = tid; t < 256; t += 32 * TJ) {
        s_tab[t] = a.tca[t];
        s_tab[256 + t] = a.tcb[t];
    }
    // interior test: y / z per CTA, x per plane
    int ylo, yhi, zlo, zhi, xlo, xhi;
    interior_range(a.lo_h[1], a.hi_h[1], a.lo_m[1], a.hi_m[1], a.ny, py, a.cpml_on, ylo, yhi);
    interior_range(a.lo_h[2], a.hi_h[2], a.lo_m[2], a.hi_m[2], a.nz, pz, a.cpml_on, zlo, zhi);
    interior_range(a.lo_h[0], a.hi_h[0], a.lo_m[0], a.hi_m[0], a.nx, px, a.cpml_on, xlo, xhi);
    const bool tile_fast = (py ? j0 + TJ <= a.ny : (j0 - 1 >= ylo && j0 + TJ <= yhi)) &&
                           (pz ? k0 + 32 <= a.nz : (k0 - 1 >= zlo && k0 + 32 <= zhi));
    // skipped cells (code-less scenes) in this tile: their planes take the general path
    int skip_plane[MAX_SKIP];
#pragma unroll
    for (int s = 0; s < MAX_SKIP; s++) {
        skip_plane[s] = -1;
        if (s < a.n_skip) {
            const long long c = a.skip[s];
            const int sk = (int)(c % a.pitch), sj = (int)((c / a.pitch) % (a.ny + 1));
            if (sj >= j0 && sj < j0 + TJ && sk >= k0 && sk < k0 + 32) skip_plane[s] = (int)(c / a.plane);
        }
    }

    T prevHy = 0, prevHz = 0;
    int pprev = -1;
    if (ib > 0) pprev = ib - 1;
    else if (px) pprev = a.nx - 1;
    // one commit group per plane: [pprev], ib, ib+1, ..., ib+NS-2; the
    // plane before the segment borrows the slot of plane ib+NS-1
    if (pprev >= 0) {
        fused_issue<T, TJ>(a, stage[NS - 1], pprev, ip, r, q);
        cp_async_commit();
    }
    int pf = ib;  // next plane to fetch (in march order, possibly wrapped)
#pragma unroll
    for (int s = 0; s < NS - 1; s++) {
        if (pf >= 0 && ib + s <= ie) fused_issue<T, TJ>(a, stage[s], pf, ip, r, q);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
    }
    if (pprev >= 0) {
        cp_async_wait<NS - 2>();
        __syncthreads();
        if (own) {
            prevHy = fused_h<T, TJ>(a, 1, pprev, j, k, stage[NS - 1], stage[0], r, q, false);
            prevHz = fused_h<T, TJ>(a, 2, pprev, j, k, stage[NS - 1], stage[0], r, q, false);
        }
        __syncthreads();
    }

    int sc = 0;
    for (int i = ib; i < ie; i++) {
        const int sn = sc == NS - 1 ? 0 : sc + 1;
        const int sf = sc == 0 ? NS - 1 : sc - 1;  // slot of plane i+NS-1
        // fetch plane i+NS-1 (needed as E(i+NS-1) by plane i+NS-2 <= ie-1)
        if (pf >= 0 && i + NS - 1 <= ie) fused_issue<T, TJ>(a, stage[sf], pf, ip, r, q);
        cp_async_commit();
        if (pf >= 0) pf = plane_after(pf, a.nx, px);
        cp_async_wait<NS - 2>();
        __syncthreads();
        const FusedStage<T, TJ> &cur = stage[sc];
        const FusedStage<T, TJ> &nxt = stage[sn];
        bool fast = tile_fast && i >= xlo && i < xhi;
#pragma unroll
        for (int s = 0; s < MAX_SKIP; s++) fast = fast && skip_plane[s] != i;
        const T e0 = cur.e[0][r][q], e1 = cur.e[1][r][q], e2 = cur.e[2][r][q];
        const int code = (int)((cur.code[ty][tx >> 2] >> (8 * (tx & 3))) & 0xffu);
        const long long c = (long long)i * a.plane + (long long)ip.own_off;
        T hx = 0, hy = 0, hz = 0;
        if (fast) {
            const T cbh = a.cbh;
            hx = xs(cur.h[0][r][q], xm(cbh, xs(xs(cur.e[2][r + 1][q], cur.e[2][r][q]), xs(cur.e[1][r][q + 1], cur.e[1][r][q]))));
            hy = xs(cur.h[1][r][q], xm(cbh, xs(xs(cur.e[0][r][q + 1], cur.e[0][r][q]), xs(nxt.e[2][r][q], cur.e[2][r][q]))));
            hz = xs(cur.h[2][r][q], xm(cbh, xs(xs(nxt.e[1][r][q], cur.e[1][r][q]), xs(cur.e[0][r + 1][q], cur.e[0][r][q]))));
            a.Ho[0][c] = hx;
            a.Ho[1][c] = hy;
            a.Ho[2][c] = hz;
            sH[0][r][q] = hx;
            sH[1][r][q] = hy;
            sH[2][r][q] = hz;
            if (ty == 0) {
                sH[0][0][q] = xs(cur.h[0][0][q], xm(cbh, xs(xs(cur.e[2][1][q], cur.e[2][0][q]), xs(cur.e[1][0][q + 1], cur.e[1][0][q]))));
                sH[2][0][q] = xs(cur.h[2][0][q], xm(cbh, xs(xs(nxt.e[1][0][q], cur.e[1][0][q]), xs(cur.e[0][1][q], cur.e[0][0][q]))));
            } else if (ty == 1 && tx < TJ) {
                const int rr = tx + 1;
                sH[0][rr][0] = xs(cur.h[0][rr][0], xm(cbh, xs(xs(cur.e[2][rr + 1][0], cur.e[2][rr][0]), xs(cur.e[1][rr][1], cur.e[1][rr][0]))));
                sH[1][rr][0] = xs(cur.h[1][rr][0], xm(cbh, xs(xs(cur.e[0][rr][1], cur.e[0][rr][0]), xs(nxt.e[2][rr][0], cur.e[2][rr][0]))));
            }
        } else {
            if (own) {
                hx = fused_h<T, TJ>(a, 0, i, j, k, cur, nxt, r, q, true);
                hy = fused_h<T, TJ>(a, 1, i, j, k, cur, nxt, r, q, true);
                hz = fused_h<T, TJ>(a, 2, i, j, k, cur, nxt, r, q, true);
                a.Ho[0][c] = hx;
                a.Ho[1][c] = hy;
                a.Ho[2][c] = hz;
            }
            sH[0][r][q] = hx;
            sH[1][r][q] = hy;
            sH[2][r][q] = hz;
            if (ty == 0 && row_halo && k < d.ck) {
                sH[0][0][q] = fused_h<T, TJ>(a, 0, i, jh, k, cur, nxt, 0, q, false);
                sH[2][0][q] = fused_h<T, TJ>(a, 2, i, jh, k, cur, nxt, 0, q, false);
            } else if (ty == 1 && tx < TJ && col_halo && j0 + tx < d.cj) {
                const int rr = tx + 1;
                sH[0][rr][0] = fused_h<T, TJ>(a, 0, i, j0 + tx, kh, cur, nxt, rr, 0, false);
                sH[1][rr][0] = fused_h<T, TJ>(a, 1, i, j0 + tx, kh, cur, nxt, rr, 0, false);
            }
        }
        __syncthreads();
        if (fast) {
            if (!a.codes || code != LIST_CODE) {
                const T ca = s_tab[code], cb = s_tab[256 + code];
                a.Eo[0][c] = xa(xm(ca, e0), xm(cb, xs(xs(sH[2][r][q], sH[2][r - 1][q]), xs(sH[1][r][q], sH[1][r][q - 1]))));
                a.Eo[1][c] = xa(xm(ca, e1), xm(cb, xs(xs(sH[0][r][q], sH[0][r][q - 1]), xs(hz, prevHz))));
                a.Eo[2][c] = xa(xm(ca, e2), xm(cb, xs(xs(hy, prevHy), xs(sH[0][r][q], sH[0][r - 1][q]))));
            }
        } else if (own && i < a.nx) {
            bool skip;
            if (a.codes) {
                skip = code == LIST_CODE;
            } else {
                skip = false;
                for (int s = 0; s < a.n_skip; s++) skip |= a.skip[s] == c;
            }
            if (!skip) {
                const T ca = s_tab[code], cb = s_tab[256 + code];
                if (e_updated(a, 0, i, j, k)) {
                    T tA = e_term(a, 0, 1, j, xs(sH[2][r][q], sH[2][r - 1][q]), i, j, k);
                    T tB = e_term(a, 1, 2, k, xs(sH[1][r][q], sH[1][r][q - 1]), i, j, k);
                    a.Eo[0][c] = xa(xm(ca, e0), xm(cb, xs(tA, tB)));
                }
                if (e_updated(a, 1, i, j, k)) {
                    T tA = e_term(a, 2, 2, k, xs(sH[0][r][q], sH[0][r][q - 1]), i, j, k);
                    T tB = e_term(a, 3, 0, i, xs(hz, prevHz), i, j, k);
                    a.Eo[1][c] = xa(xm(ca, e1), xm(cb, xs(tA, tB)));
                }
                if (e_updated(a, 2, i, j, k)) {
                    T tA = e_term(a, 4, 0, i, xs(hy, prevHy), i, j, k);
                    T tB = e_term(a, 5, 1, j, xs(sH[0][r][q], sH[0][r - 1][q]), i, j, k);
                    a.Eo[2][c] = xa(xm(ca, e2), xm(cb, xs(tA, tB)));
                }
            }
        }
        prevHy = hy;
        prevHz = hz;
        sc = sn;
    }
    cp_async_wait<0>();
}

template <typename T, int TJ, int NS>
constexpr size_t fused_smem() {
    return NS * sizeof(FusedStage<T, TJ>) + sizeof(T) * 3 * (TJ + 1) * 33 + sizeof(T) * 512;
}

// Instantiations: FP32 keeps six planes in flight at four CTAs per SM (64
// registers); FP64 four planes at three CTAs per SM.  TJ = 16 halves the
// relative halo at the cost of fewer column tiles.
#define RFB_FUSED_FP32_8 k_fused<float, 8, 6, 4>
#define RFB_FUSED_FP32_16 k_fused<float, 16, 4, 2>
#define RFB_FUSED_FP64_8 k_fused<double, 8, 4, 3>
#define RFB_FUSED_FP64_16 k_fused<double, 16, 3, 1>

template <typename T>
void launch_fused(const Args<T> &a, const FusedPlan &p, cudaStream_t st);

template <>
inline void launch_fused<float>(const Args<float> &a, const FusedPlan &p, cudaStream_t st) {
    if (p.tj == 16)
        RFB_FUSED_FP32_16<<<p.grid, dim3(32, 16), fused_smem<float, 16, 4>(), st>>>(a, p.d);
    else
        RFB_FUSED_FP32_8<<<p.grid, dim3(32, 8), fused_smem<float, 8, 6>(), st>>>(a, p.d);
}

template <>
inline void launch_fused<double>(const Args<double> &a, const FusedPlan &p, cudaStream_t st) {
    if (p.tj == 16)
        RFB_FUSED_FP64_16<<<p.grid, dim3(32, 16), fused_smem<double, 16, 3>(), st>>>(a, p.d);
    else
        RFB_FUSED_FP64_8<<<p.grid, dim3(32, 8), fused_smem<double, 8, 4>(), st>>>(a, p.d);
}

// Raises the dynamic shared-memory limit of every fused instantiation once.
static inline int fused_prepare() {
    static int done = 0;
    if (done) return 0;
    cudaError_t e = cudaFuncSetAttribute(RFB_FUSED_FP32_8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fused_smem<float, 8, 6>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(RFB_FUSED_FP32_16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fused_smem<float, 16, 4>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(RFB_FUSED_FP64_8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fused_smem<double, 8, 4>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(RFB_FUSED_FP64_16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fused_smem<double, 16, 3>());
    if (e != cudaSuccess) return -1;
    done = 1;
    return 0;
}

// Plans the fused sweep.  boundary_active: some source sits on a padded
// boundary plane (i = nx, j = ny or k = nz of a non-periodic axis), so those
// planes must be swept too; otherwise they stay zero for the whole run and
// are skipped.
static inline int fused_plan_dims(FusedPlan *p, const rfb_geom_t *g, int boundary_active, int tj, int seg_len) {
    const bool px = g->periodic & 1u, py = g->periodic & 2u, pz = g->periodic & 4u;
    p->tj = tj;
    p->d.cj = g->ny + ((boundary_active && !py) ? 1 : 0);
    p->d.ck = g->nz + ((boundary_active && !pz) ? 1 : 0);
    p->d.ci = g->nx + ((boundary_active && !px) ? 1 : 0);
    if (seg_len <= 0 || seg_len > p->d.ci) seg_len = p->d.ci;
    p->d.seg_len = seg_len;
    const int nseg = (p->d.ci + seg_len - 1) / seg_len;
    p->grid = dim3((p->d.ck + 31) / 32, (p->d.cj + tj - 1) / tj, nseg);
    if (nseg > 65535 || p->grid.y > 65535) return -1;
    return 0;
}

// Default plan: TJ = 8 and i-segments sized so the grid holds about
// eight CTAs per SM of a 148-SM B200.
static inline int fused_plan_default(FusedPlan *p, const rfb_geom_t *g, int boundary_active) {
    if (fused_plan_dims(p, g, boundary_active, 8, 0) != 0) return -1;
    const long long cols = (long long)p->grid.x * p->grid.y;
    const long long target = 148LL * 8;
    long long nseg = (target + cols - 1) / cols;
    long long max_seg = p->d.ci / 8 > 0 ? p->d.ci / 8 : 1;
    if (nseg > max_seg) nseg = max_seg;
    if (nseg < 1) nseg = 1;
    const int seg_len = (int)((p->d.ci + nseg - 1) / nseg);
    return fused_plan_dims(p, g, boundary_active, 8, seg_len);
}

}  // namespace rfb
