// energy.cuh -- FP64 energy audit of the resident fields.
//
// rfsyn audits energy on the host (validate_long_term_stability.c:166-209,
// audit_periodic_energy.c:43-71): U = sum over i < nx, j < ny, k < nz and the
// three components of 0.5 (eps E^2 + mu0 H^2), times dx^3, with eps recovered
// from the component's scalar Cb as dt / (dx Cb).  Here the same sums run on
// the GPU in FP64 whatever the field precision: each thread accumulates a
// grid-stride share, warps combine with shuffles, blocks with shared memory,
// and one final pass adds the block partials in a fixed order, so repeated
// calls are bit-for-bit identical.
//
// Code cells take Cb from the FP64 table; interface-list cells (code 255, or
// the few skip cells of a code-less scene) take it from the list, in a
// second loop over list entries.  With ping-pong buffers the previous step's
// E and H are still resident, which gives the audit's "modified" energy
// (audit_periodic_energy.c:53-62): E^{n-1} energy + 0.5 mu0 H^{n-3/2} . H^{n-1/2}.
#pragma once
#include "engine.h"
#include "kernels.cuh"

namespace rfb {

constexpr int EN_BLOCKS = 592;  // 4 per SM
constexpr int EN_THREADS = 256;
constexpr double EN_MU0 = 1.25663706212e-6;

template <typename T>
struct EnergyArgs {
    const T *E[3], *H[3];    // current fields
    const T *Ep[3], *Hp[3];  // previous step, or null
    const uint8_t *codes;    // null: table entry 0 except skip cells
    const double *cb_tab;    // 256 FP64 Cb
    int n_cells;
    const int *lc_ijk;
    const double *cb_list;   // 3 per list cell
    int n_skip;
    long long skip[MAX_SKIP];
    int nx, ny, nz;
    long long pitch;
    int x_lo, x_hi;
    double dt_over_dx;       // eps = dt_over_dx / Cb
    double *partial;         // [EN_BLOCKS][RFB_EN_COUNT]
};

struct EnAcc {
    double v[RFB_EN_COUNT];
};

__device__ __forceinline__ void en_electric(EnAcc &acc, double eps, double e, double ep, bool prev, bool inside) {
    if (!isfinite(e)) acc.v[RFB_EN_NONFINITE] += 1.0;
    acc.v[RFB_EN_MAX_E] = fmax(acc.v[RFB_EN_MAX_E], fabs(e));
    const double u = 0.5 * eps * e * e;
    acc.v[RFB_EN_E] += u;
    if (inside) acc.v[RFB_EN_E_INT] += u;
    if (prev) acc.v[RFB_EN_E_PREV] += 0.5 * eps * ep * ep;
}

template <typename T>
__global__ void __launch_bounds__(EN_THREADS) k_energy(EnergyArgs<T> a) {
    EnAcc acc;
#pragma unroll
    for (int q = 0; q < RFB_EN_COUNT; q++) acc.v[q] = 0.0;
    const bool prev = a.Ep[0] != nullptr;
    const long long plane_cells = (long long)a.ny * a.nz;
    const long long n = (long long)a.nx * plane_cells;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int i = (int)(t / plane_cells);
        const long long r = t - (long long)i * plane_cells;
        const int j = (int)(r / a.nz), k = (int)(r - (long long)j * a.nz);
        const long long c = ((long long)i * (a.ny + 1) + j) * a.pitch + k;
        const bool inside = i >= a.x_lo && i < a.x_hi;
        // magnetic energy of every cell
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const double h = (double)a.H[m][c];
            if (!isfinite(h)) acc.v[RFB_EN_NONFINITE] += 1.0;
            acc.v[RFB_EN_MAX_H] = fmax(acc.v[RFB_EN_MAX_H], fabs(h));
            const double u = 0.5 * EN_MU0 * h * h;
            acc.v[RFB_EN_H] += u;
            if (inside) acc.v[RFB_EN_H_INT] += u;
            if (prev) acc.v[RFB_EN_CROSS] += 0.5 * EN_MU0 * (double)a.Hp[m][c] * h;
        }
        // electric energy of code cells
        int code = 0;
        bool listed = false;
        if (a.codes) {
            code = a.codes[c];
            listed = code == LIST_CODE;
        } else {
            for (int s = 0; s < a.n_skip; s++) listed |= a.skip[s] == c;
        }
        if (listed) continue;
        const double eps = a.dt_over_dx / a.cb_tab[code];
#pragma unroll
        for (int m = 0; m < 3; m++)
            en_electric(acc, eps, (double)a.E[m][c], prev ? (double)a.Ep[m][c] : 0.0, prev, inside);
    }
    // electric energy of interface-list cells
    const long long ne = 3LL * a.n_cells;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ne; t += stride) {
        const long long q = t / 3;
        const int m = (int)(t - 3 * q);
        const int i = a.lc_ijk[3 * q], j = a.lc_ijk[3 * q + 1], k = a.lc_ijk[3 * q + 2];
        if (i >= a.nx || j >= a.ny || k >= a.nz) continue;
        const long long c = ((long long)i * (a.ny + 1) + j) * a.pitch + k;
        const double eps = a.dt_over_dx / a.cb_list[t];
        en_electric(acc, eps, (double)a.E[m][c], prev ? (double)a.Ep[m][c] : 0.0, prev, i >= a.x_lo && i < a.x_hi);
    }
    // warp, then block
    __shared__ double red[EN_THREADS / 32][RFB_EN_COUNT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < RFB_EN_COUNT; q++) {
        double v = acc.v[q];
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = (q == RFB_EN_MAX_E || q == RFB_EN_MAX_H) ? fmax(v, o) : v + o;
        }
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < RFB_EN_COUNT) {
        const int q = threadIdx.x;
        double v = red[0][q];
        for (int w = 1; w < EN_THREADS / 32; w++)
            v = (q == RFB_EN_MAX_E || q == RFB_EN_MAX_H) ? fmax(v, red[w][q]) : v + red[w][q];
        a.partial[(long long)blockIdx.x * RFB_EN_COUNT + q] = v;
    }
}

// Adds the block partials in block order and applies the cell volume.
__global__ void k_energy_final(const double *partial, int nblocks, double volume, int have_prev, double *out) {
    const int q = threadIdx.x;
    if (q >= RFB_EN_COUNT) return;
    double v = partial[q];
    for (int b = 1; b < nblocks; b++) {
        const double o = partial[(long long)b * RFB_EN_COUNT + q];
        v = (q == RFB_EN_MAX_E || q == RFB_EN_MAX_H) ? fmax(v, o) : v + o;
    }
    if (q == RFB_EN_E || q == RFB_EN_H || q == RFB_EN_E_INT || q == RFB_EN_H_INT || q == RFB_EN_E_PREV ||
        q == RFB_EN_CROSS)
        v *= volume;
    if (!have_prev && (q == RFB_EN_E_PREV || q == RFB_EN_CROSS)) v = nan("");
    out[q] = v;
}

}  // namespace rfb
