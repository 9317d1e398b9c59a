// fused.cuh -- one-kernel-per-step H+E sweep (2.5D march along i).
//
// Each CTA owns a (TJ x 32) tile of (j, k) and a segment of i planes.  It
// marches the segment plane by plane: E^n of planes i and i+1 sit in shared
// memory with a one-cell halo in j and k; H^{n+1/2} of plane i is computed for
// the tile plus its low j / low k halo (the halo redundantly, never stored),
// and E^{n+1} of plane i follows from shared H and the plane i-1 values kept in
// registers.  Fields and the H-side psi are ping-ponged between two buffers, so
// a halo recomputation always reads the step-n state even when the owning CTA
// has already written step n+1.  Per cell-step the kernel moves the compulsory
// 6 reads + 6 writes of the field components (48 B in FP32).
#pragma once
#include "kernels.cuh"
#include "engine.h"

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

// H value of component c at plane i, tile position (r, q) of the shared E
// planes: cur (plane i) and nxt (plane i+1).  Returns H^{n+1/2} (or the input
// value where the component is not updated there); store selects whether the
// new psi is written (owner) or only used (halo).
template <typename T, int TJ>
__device__ __forceinline__ T fused_h(const Args<T> &a, int c, int i, int j, int k, const T (*cur)[TJ + 2][34],
                                     const T (*nxt)[TJ + 2][34], int r, int q, bool store) {
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const long long ci = cidx(a, i, j, k);
    const T hin = a.H[c][ci];
    T dA, dB;
    int pA, pB, axA, axB, qA, qB;
    if (c == 0) {
        if (!(i < a.nx + (px ? 0 : 1) && j < a.ny && k < a.nz)) return hin;
        dA = xs(cur[2][r + 1][q], cur[2][r][q]);
        dB = xs(cur[1][r][q + 1], cur[1][r][q]);
        pA = 0; axA = 1; qA = j;
        pB = 1; axB = 2; qB = k;
    } else if (c == 1) {
        if (!(i < a.nx && j < a.ny + (py ? 0 : 1) && k < a.nz)) return hin;
        dA = xs(cur[0][r][q + 1], cur[0][r][q]);
        dB = xs(nxt[2][r][q], cur[2][r][q]);
        pA = 2; axA = 2; qA = k;
        pB = 3; axB = 0; qB = i;
    } else {
        if (!(i < a.nx && j < a.ny && k < a.nz + (pz ? 0 : 1))) return hin;
        dA = xs(nxt[1][r][q], cur[1][r][q]);
        dB = xs(cur[0][r + 1][q], cur[0][r][q]);
        pA = 4; axA = 0; qA = i;
        pB = 5; axB = 1; qB = j;
    }
    T tA = dA, tB = dB;
    if (a.cpml_on) {
        int s = slab_of(qA, a.lo_h[axA], a.hi_h[axA]);
        if (s >= 0) {
            long long pi = psi_idx(a, axA, a.ns_h[axA], s, i, j, k);
            T pn;
            tA = cpml_step(dA, a.kinv_h[axA][qA], a.b_h[axA][qA], a.a_h[axA][qA], a.dx, a.psi_hi[pA][pi], &pn);
            if (store) a.psi_ho[pA][pi] = pn;
        }
        s = slab_of(qB, a.lo_h[axB], a.hi_h[axB]);
        if (s >= 0) {
            long long pi = psi_idx(a, axB, a.ns_h[axB], s, i, j, k);
            T pn;
            tB = cpml_step(dB, a.kinv_h[axB][qB], a.b_h[axB][qB], a.a_h[axB][qB], a.dx, a.psi_hi[pB][pi], &pn);
            if (store) a.psi_ho[pB][pi] = pn;
        }
    }
    return xs(hin, xm(a.cbh, xs(tA, tB)));
}

template <typename T>
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

template <typename T, int TJ>
__device__ __forceinline__ void fused_load_plane(const Args<T> &a, T (*dst)[TJ + 2][34], int p, int j0, int k0,
                                                 int tx, int ty) {
    const bool py = a.per & 2u, pz = a.per & 4u;
    // own cells (coalesced rows)
    {
        bool vj, vk;
        const int jj = wrap_coord<T>(j0 + ty, a.ny, py, vj);
        const int kk = wrap_coord<T>(k0 + tx, a.nz, pz, vk);
        T ex = 0, ey = 0, ez = 0;
        if (p >= 0 && vj && vk) {
            const long long c = cidx(a, p, jj, kk);
            ex = a.E[0][c]; ey = a.E[1][c]; ez = a.E[2][c];
        }
        dst[0][ty + 1][tx + 1] = ex; dst[1][ty + 1][tx + 1] = ey; dst[2][ty + 1][tx + 1] = ez;
    }
    // halo rows r = 0 (j0-1) and r = TJ+1 (j0+TJ)
    if (ty < 2) {
        const int r = ty == 0 ? 0 : TJ + 1;
        bool vj, vk;
        const int jj = wrap_coord<T>(j0 - 1 + r, a.ny, py, vj);
        const int kk = wrap_coord<T>(k0 + tx, a.nz, pz, vk);
        T ex = 0, ey = 0, ez = 0;
        if (p >= 0 && vj && vk) {
            const long long c = cidx(a, p, jj, kk);
            ex = a.E[0][c]; ey = a.E[1][c]; ez = a.E[2][c];
        }
        dst[0][r][tx + 1] = ex; dst[1][r][tx + 1] = ey; dst[2][r][tx + 1] = ez;
    } else if (ty == 2 && tx < 2 * (TJ + 2)) {
        // halo columns q = 0 (k0-1) and q = 33 (k0+32), all TJ+2 rows
        const int r = tx >> 1;
        const int q = (tx & 1) ? 33 : 0;
        bool vj, vk;
        const int jj = wrap_coord<T>(j0 - 1 + r, a.ny, py, vj);
        const int kk = wrap_coord<T>(k0 - 1 + q, a.nz, pz, vk);
        T ex = 0, ey = 0, ez = 0;
        if (p >= 0 && vj && vk) {
            const long long c = cidx(a, p, jj, kk);
            ex = a.E[0][c]; ey = a.E[1][c]; ez = a.E[2][c];
        }
        dst[0][r][q] = ex; dst[1][r][q] = ey; dst[2][r][q] = ez;
    }
}

template <typename T, int TJ>
__global__ void __launch_bounds__(32 * TJ) k_fused(Args<T> a, FusedDims d) {
    __shared__ T sE[2][3][TJ + 2][34];
    __shared__ T sH[3][TJ + 1][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int k0 = blockIdx.x * 32, j0 = blockIdx.y * TJ;
    const int ib = blockIdx.z * d.seg_len;
    const int ie = min(ib + d.seg_len, d.ci);
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const int j = j0 + ty, k = k0 + tx;
    const bool own = j < d.cj && k < d.ck;
    // halo cells of H: row j0-1 (Hx, Hz) and column k0-1 (Hx, Hy)
    const bool row_halo = (j0 > 0 || py);
    const bool col_halo = (k0 > 0 || pz);
    const int jh = j0 > 0 ? j0 - 1 : a.ny - 1;   // used only when row_halo
    const int kh = k0 > 0 ? k0 - 1 : a.nz - 1;   // used only when col_halo

    int cur = 0;
    T prevHy = 0, prevHz = 0;
    // prologue: H of the plane before the segment (Hy, Hz only)
    int pprev = -1;
    if (ib > 0) pprev = ib - 1;
    else if (px) pprev = a.nx - 1;
    if (pprev >= 0) {
        fused_load_plane<T, TJ>(a, sE[0], pprev, j0, k0, tx, ty);
        fused_load_plane<T, TJ>(a, sE[1], ib, j0, k0, tx, ty);
        __syncthreads();
        if (own) {
            prevHy = fused_h<T, TJ>(a, 1, pprev, j, k, sE[0], sE[1], ty + 1, tx + 1, false);
            prevHz = fused_h<T, TJ>(a, 2, pprev, j, k, sE[0], sE[1], ty + 1, tx + 1, false);
        }
        __syncthreads();
        cur = 1;
    } else {
        fused_load_plane<T, TJ>(a, sE[0], ib, j0, k0, tx, ty);
        cur = 0;
    }

    for (int i = ib; i < ie; i++) {
        const int nxt = cur ^ 1;
        int pn = i + 1;
        if (pn == a.nx && px) pn = 0;
        else if (pn > a.nx) pn = -1;
        fused_load_plane<T, TJ>(a, sE[nxt], pn, j0, k0, tx, ty);
        __syncthreads();
        T e0 = sE[cur][0][ty + 1][tx + 1], e1 = sE[cur][1][ty + 1][tx + 1], e2 = sE[cur][2][ty + 1][tx + 1];
        T hx = 0, hy = 0, hz = 0;
        if (own) {
            const long long c = cidx(a, i, j, k);
            hx = fused_h<T, TJ>(a, 0, i, j, k, sE[cur], sE[nxt], ty + 1, tx + 1, true);
            hy = fused_h<T, TJ>(a, 1, i, j, k, sE[cur], sE[nxt], ty + 1, tx + 1, true);
            hz = fused_h<T, TJ>(a, 2, i, j, k, sE[cur], sE[nxt], ty + 1, tx + 1, true);
            a.Ho[0][c] = hx; a.Ho[1][c] = hy; a.Ho[2][c] = hz;
        }
        sH[0][ty + 1][tx + 1] = hx;
        sH[1][ty + 1][tx + 1] = hy;
        sH[2][ty + 1][tx + 1] = hz;
        if (ty == 0 && row_halo && k < d.ck) {
            sH[0][0][tx + 1] = fused_h<T, TJ>(a, 0, i, jh, k, sE[cur], sE[nxt], 0, tx + 1, false);
            sH[2][0][tx + 1] = fused_h<T, TJ>(a, 2, i, jh, k, sE[cur], sE[nxt], 0, tx + 1, false);
        }
        if (tx == 31 && col_halo && j < d.cj) {
            sH[0][ty + 1][0] = fused_h<T, TJ>(a, 0, i, j, kh, sE[cur], sE[nxt], ty + 1, 0, false);
            sH[1][ty + 1][0] = fused_h<T, TJ>(a, 1, i, j, kh, sE[cur], sE[nxt], ty + 1, 0, false);
        }
        __syncthreads();
        if (own && i < a.nx) {
            const long long c = cidx(a, i, j, k);
            int code = 0;
            bool skip = false;
            if (a.codes) {
                code = a.codes[c];
                skip = code == LIST_CODE;
            } else {
                for (int s = 0; s < a.n_skip; s++) skip |= a.skip[s] == c;
            }
            if (!skip) {
                const T ca = a.tca[code], cb = a.tcb[code];
                const int r = ty + 1, q = tx + 1;
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
        cur = nxt;
    }
}

template <typename T>
void launch_fused(const Args<T> &a, const FusedPlan &p, cudaStream_t st) {
    if (p.tj == 4) k_fused<T, 4><<<p.grid, dim3(32, 4), 0, st>>>(a, p.d);
    else k_fused<T, 8><<<p.grid, dim3(32, 8), 0, st>>>(a, p.d);
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
    if (seg_len <= 0) seg_len = p->d.ci;
    p->d.seg_len = seg_len;
    const int nseg = (p->d.ci + seg_len - 1) / seg_len;
    p->grid = dim3((p->d.ck + 31) / 32, (p->d.cj + tj - 1) / tj, nseg);
    if (nseg > 65535 || p->grid.y > 65535) return -1;
    return 0;
}

// Default tile plan: TJ = 8 and i-segments sized so the grid holds about
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
