// smooth.cu -- smoothed permittivity tensors of cut cells, built on the GPU in
// FP64: the fill fraction of the unit cube around every E sample near a
// sphere's or a slab's surface (8^3 lattice, sphere_frac.cuh) and, for the
// samples the surface cuts, the row of the smoothed relative inverse
// permittivity between the sample's background and the inclusion along the
// surface normal (Kottke, Farjadpour and Johnson's tau average, smooth3.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "engine.h"
#include "smooth3.h"
#include "sphere_frac.cuh"

namespace {

// One sphere's box of cells: f[3 cell + c], rows[9 cell + 3 c + b] = M_cb of
// sample c; eps_bg[cell] is the cell's isotropic background.
__global__ void k_sphere_rows(double cx, double cy, double cz, double r, double eps_in, int i0, int j0, int k0,
                              int ni, int nj, int nk, const double *eps_bg, double *f, double *rows, int *bad) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncell = (long long)ni * nj * nk;
    if (t >= 3 * ncell) return;
    const long long cell = t / 3;
    const int comp = (int)(t - 3 * cell);
    const int k = k0 + (int)(cell % nk);
    const int j = j0 + (int)((cell / nk) % nj);
    const int i = i0 + (int)(cell / ((long long)nk * nj));
    double p[3], n[3];
    rfb_sample_pos(i, j, k, comp, p);
    const double fr = rfb_sphere_cube_fraction(p, cx, cy, cz, r, n);
    f[t] = fr;
    if (n[0] == 0.0 && n[1] == 0.0 && n[2] == 0.0) n[comp] = 1.0;  // the centre itself: any normal
    const double eb = eps_bg[cell];
    const double bg[9] = {eb, 0, 0, 0, eb, 0, 0, 0, eb}, in[9] = {eps_in, 0, 0, 0, eps_in, 0, 0, 0, eps_in};
    double m[9];
    if (rfb_sm_mix(fr, bg, in, n, m) != 0) {
        atomicExch(bad, 1);
        m[3 * comp] = m[3 * comp + 1] = m[3 * comp + 2] = 0.0;
    }
    for (int b = 0; b < 3; b++) rows[3 * t + b] = m[3 * comp + b];
}

struct SlabGeom {
    double o[3], u[3], half;
    double eps_in[9];
};

// Listed samples (i, j, k, c) near a slab's faces: f[s] and row c of M.
__global__ void k_slab_rows(SlabGeom g, const int *ijkc, const double *eps_bg, int n, double *f, double *rows,
                            int *bad) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int c = ijkc[4 * s + 3];
    double p[3];
    rfb_sample_pos(ijkc[4 * s], ijkc[4 * s + 1], ijkc[4 * s + 2], c, p);
    const double fr = rfb_slab_cube_fraction(p, g.o, g.u, g.half);
    f[s] = fr;
    const double eb = eps_bg[s];
    const double bg[9] = {eb, 0, 0, 0, eb, 0, 0, 0, eb};
    double m[9];
    if (rfb_sm_mix(fr, bg, g.eps_in, g.u, m) != 0) {
        atomicExch(bad, 1);
        m[3 * c] = m[3 * c + 1] = m[3 * c + 2] = 0.0;
    }
    for (int b = 0; b < 3; b++) rows[3 * s + b] = m[3 * c + b];
}

// Per-device staging, grown on demand (set-up code: one launch, a few copies
// and one synchronisation per call).
struct Stage {
    double *dev = nullptr;
    int *dflag = nullptr;
    size_t cap = 0;  // doubles
};
std::mutex g_mu;
Stage g_stage[64];

int stage_for(size_t doubles, Stage **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        rfb_set_error("subpixel smoothing: no usable CUDA device");
        return -1;
    }
    Stage &s = g_stage[dev];
    if (!s.dflag && cudaMalloc(&s.dflag, sizeof(int)) != cudaSuccess) {
        s.dflag = nullptr;
        rfb_set_error("subpixel smoothing: device allocation failed");
        return -1;
    }
    if (s.cap < doubles) {
        cudaFree(s.dev);
        s.dev = nullptr;
        s.cap = 0;
        const size_t want = std::max(doubles, (size_t)1 << 20);
        if (cudaMalloc(&s.dev, want * sizeof(double)) != cudaSuccess) {
            s.dev = nullptr;
            rfb_set_error("subpixel smoothing: device allocation of %zu bytes failed", want * sizeof(double));
            return -1;
        }
        s.cap = want;
    }
    *out = &s;
    return 0;
}

int finish(Stage *s, double *f, size_t nf, double *rows, size_t nr, double *dev_f, double *dev_rows) {
    int bad = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) rfb_count_launch();
    if (e == cudaSuccess) e = cudaMemcpy(f, dev_f, nf * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(rows, dev_rows, nr * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&bad, s->dflag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        rfb_set_error("subpixel smoothing: %s", cudaGetErrorString(e));
        return -1;
    }
    if (bad) {
        rfb_set_error("subpixel smoothing: a permittivity is not positive definite");
        return -1;
    }
    return 0;
}

}  // namespace

extern "C" int rfb_sphere_rows(const double centre[3], double radius, double eps_in, int i0, int j0, int k0, int ni,
                               int nj, int nk, const double *eps_bg, double *f, double *rows) {
    const size_t ncell = (size_t)ni * nj * nk, n = 3 * ncell;
    if (!n) return 0;
    std::lock_guard<std::mutex> lock(g_mu);
    Stage *s = nullptr;
    if (stage_for(ncell + 4 * n, &s) != 0) return -1;
    double *d_bg = s->dev, *d_f = s->dev + ncell, *d_rows = d_f + n;
    if (cudaMemcpy(d_bg, eps_bg, ncell * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(s->dflag, 0, sizeof(int)) != cudaSuccess) {
        rfb_set_error("subpixel smoothing: upload failed");
        return -1;
    }
    k_sphere_rows<<<(unsigned)((n + 255) / 256), 256>>>(centre[0], centre[1], centre[2], radius, eps_in, i0, j0, k0,
                                                         ni, nj, nk, d_bg, d_f, d_rows, s->dflag);
    return finish(s, f, n, rows, 3 * n, d_f, d_rows);
}

extern "C" int rfb_slab_rows(const double point[3], const double unit_normal[3], double thickness,
                             const double eps_in[9], const int *ijkc, const double *eps_bg, int n, double *f,
                             double *rows) {
    if (n <= 0) return 0;
    std::lock_guard<std::mutex> lock(g_mu);
    Stage *s = nullptr;
    // sample coordinates (4 ints = 2 doubles each), background, f, rows
    if (stage_for((size_t)n * 7, &s) != 0) return -1;
    int *d_ijkc = reinterpret_cast<int *>(s->dev);
    double *d_bg = s->dev + 2 * (size_t)n, *d_f = d_bg + n, *d_rows = d_f + n;
    if (cudaMemcpy(d_ijkc, ijkc, 4 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_bg, eps_bg, (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(s->dflag, 0, sizeof(int)) != cudaSuccess) {
        rfb_set_error("subpixel smoothing: upload failed");
        return -1;
    }
    SlabGeom g;
    for (int a = 0; a < 3; a++) {
        g.o[a] = point[a];
        g.u[a] = unit_normal[a];
    }
    g.half = 0.5 * thickness;
    for (int q = 0; q < 9; q++) g.eps_in[q] = eps_in[q];
    k_slab_rows<<<(unsigned)((n + 255) / 256), 256>>>(g, d_ijkc, d_bg, n, d_f, d_rows, s->dflag);
    return finish(s, f, (size_t)n, rows, 3 * (size_t)n, d_f, d_rows);
}
