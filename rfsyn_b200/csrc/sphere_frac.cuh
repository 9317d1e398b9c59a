// sphere_frac.cuh -- fill fraction of the unit cube around an E sample,
// inside a sphere or a slab (FP64, every operation rounded separately so the
// CPU restatement of the oracle reproduces it bit for bit).
#pragma once
#include <cuda_runtime.h>

// Position of the E sample of component comp of cell (i, j, k), cell units:
// Ex at (i + 1/2, j, k), Ey at (i, j + 1/2, k), Ez at (i, j, k + 1/2).
__device__ __forceinline__ void rfb_sample_pos(int i, int j, int k, int comp, double p[3]) {
    p[0] = __dadd_rn((double)i, comp == 0 ? 0.5 : 0.0);
    p[1] = __dadd_rn((double)j, comp == 1 ? 0.5 : 0.0);
    p[2] = __dadd_rn((double)k, comp == 2 ? 0.5 : 0.0);
}

// Offset of lattice point a (0..7) from the cube centre: (a + 1/2)/8 - 1/2.
__device__ __forceinline__ double rfb_lattice(int a) { return __dsub_rn(__ddiv_rn(__dadd_rn((double)a, 0.5), 8.0), 0.5); }

// Unit cube around p and the sphere (centre c, radius r): exact 0 / 1 when
// the half diagonal sqrt(3)/2 clears the surface, else the share of an 8^3
// lattice of points whose squared distance is <= r^2.  nrm: the outward unit
// normal (p - c)/|p - c| (zero at the centre).
__device__ __forceinline__ double rfb_sphere_cube_fraction(const double p[3], double cx, double cy, double cz,
                                                           double r, double nrm[3]) {
    const double dx = __dsub_rn(p[0], cx), dy = __dsub_rn(p[1], cy), dz = __dsub_rn(p[2], cz);
    const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    nrm[0] = nrm[1] = nrm[2] = 0.0;
    if (d > 0.0) {
        nrm[0] = __ddiv_rn(dx, d);
        nrm[1] = __ddiv_rn(dy, d);
        nrm[2] = __ddiv_rn(dz, d);
    }
    const double h = 0.8660254037844386;
    if (__dadd_rn(d, h) <= r) return 1.0;
    if (__dsub_rn(d, h) >= r) return 0.0;
    const double r2 = __dmul_rn(r, r);
    int count = 0;
    for (int a = 0; a < 8; a++) {
        const double px = __dsub_rn(__dadd_rn(p[0], rfb_lattice(a)), cx);
        for (int b = 0; b < 8; b++) {
            const double py = __dsub_rn(__dadd_rn(p[1], rfb_lattice(b)), cy);
            for (int e = 0; e < 8; e++) {
                const double pz = __dsub_rn(__dadd_rn(p[2], rfb_lattice(e)), cz);
                const double q = __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz));
                count += q <= r2;
            }
        }
    }
    return __ddiv_rn((double)count, 512.0);
}

// Unit cube around p and the slab |(x - o) . u| <= half (u unit): exact 0 / 1
// when the cube's support sum_a |u_a| / 2 clears both faces, else the share
// of the 8^3 lattice inside.
__device__ __forceinline__ double rfb_slab_cube_fraction(const double p[3], const double o[3], const double u[3],
                                                         double half) {
    const double d = __dadd_rn(__dadd_rn(__dmul_rn(u[0], __dsub_rn(p[0], o[0])), __dmul_rn(u[1], __dsub_rn(p[1], o[1]))),
                               __dmul_rn(u[2], __dsub_rn(p[2], o[2])));
    const double reach = __dmul_rn(0.5, __dadd_rn(__dadd_rn(fabs(u[0]), fabs(u[1])), fabs(u[2])));
    const double ad = fabs(d);
    if (__dadd_rn(ad, reach) <= half) return 1.0;
    if (__dsub_rn(ad, reach) > half) return 0.0;
    int count = 0;
    for (int a = 0; a < 8; a++) {
        const double ox = __dmul_rn(u[0], rfb_lattice(a));
        for (int b = 0; b < 8; b++) {
            const double oy = __dadd_rn(ox, __dmul_rn(u[1], rfb_lattice(b)));
            for (int e = 0; e < 8; e++) {
                const double q = __dadd_rn(d, __dadd_rn(oy, __dmul_rn(u[2], rfb_lattice(e))));
                count += fabs(q) <= half;
            }
        }
    }
    return __ddiv_rn((double)count, 512.0);
}
