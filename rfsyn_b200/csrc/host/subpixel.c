/*
 * subpixel.c -- rfsyn's 2-D subpixel helpers (engine/fdtd/subpixel_te.h:18-71)
 * and their 3-D generalisation.
 *
 * rfsyn's helpers describe a rotated rectangle in the (x, y) plane of a
 * z-invariant TE/TM problem: the share of a sample's dx x dy cell that the
 * rectangle covers, the share of an edge segment inside it, and the
 * arithmetic, harmonic and normal-aligned tensor mixes of two permittivities
 * (subpixel_te.c:27-505).  The same contracts are kept here -- argument
 * checks, status codes, outputs left untouched on failure, the clamping of
 * results into [0, 1] -- with an implementation of this library's own: the
 * cell is the unit square in cell units, clipped by the rectangle's four
 * half-planes one after the other (Sutherland-Hodgman polygon clipping), and
 * the covered share is the clipped polygon's shoelace area.
 *
 * fdtd_b200_subpixel_tensor3 is the 3-D form of the tensor mix.  For two
 * isotropic media it is rfsyn's rule with the rotation taken to three
 * dimensions, M = lambda_n n n^T + lambda_t (I - n n^T), lambda_n = <1/eps>,
 * lambda_t = 1/<eps> (subpixel_te.c:106-132 in the plane); for anisotropic
 * media it averages Kottke, Farjadpour and Johnson's tau transform of the
 * permittivity in the frame of the interface normal (Phys. Rev. E 77, 036611,
 * 2008, eqs. 23-24), which reduces to the same rule when both media are
 * isotropic.  The GPU kernels that smooth spheres and slabs evaluate the same
 * operations (engine.cu, k_smooth_rows).
 */
#include <float.h>
#include <math.h>
#include <stddef.h>

#include "host.h"

enum { ST_OK = 0, ST_INVALID = -1, ST_NUMERIC = -2 };

typedef struct {
    double x, y;
} vtx_t;

/* A convex polygon clipped by one half-plane keeps at most one vertex more
 * than it had; the unit square clipped four times has at most 8. */
#define CLIP_MAX 16

static int finite_all(double a, double b, double c) { return isfinite(a) && isfinite(b) && isfinite(c); }

/* Keeps the part of polygon `in` (n vertices) where nx x + ny y <= off;
 * writes it to `out` and returns its vertex count, or -1 on overflow or a
 * non-finite crossing. */
static int clip_half_plane(const vtx_t *in, int n, double nx, double ny, double off, vtx_t *out) {
    int m = 0;
    if (n == 0) return 0;
    /* scale the plane so its largest coefficient is 1: distances stay O(1) */
    const double s = fmax(fmax(fabs(nx), fabs(ny)), fabs(off));
    if (s == 0.0) {
        for (int q = 0; q < n; q++) out[q] = in[q];
        return n;
    }
    nx /= s;
    ny /= s;
    off /= s;
    for (int q = 0; q < n; q++) {
        const vtx_t a = in[q == 0 ? n - 1 : q - 1], b = in[q];
        const double da = nx * a.x + ny * a.y - off, db = nx * b.x + ny * b.y - off;
        const int ina = da <= 0.0, inb = db <= 0.0;
        if (ina != inb) {
            const double den = da - db;
            if (!(den != 0.0) || !isfinite(den)) return -1;
            double t = da / den;
            if (!isfinite(t)) return -1;
            t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
            if (m >= CLIP_MAX) return -1;
            out[m].x = a.x + t * (b.x - a.x);
            out[m].y = a.y + t * (b.y - a.y);
            if (!isfinite(out[m].x) || !isfinite(out[m].y)) return -1;
            m++;
        }
        if (inb) {
            if (m >= CLIP_MAX) return -1;
            out[m++] = b;
        }
    }
    return m;
}

static int rect_ok(const subpixel_te_rectangle_t *r) {
    return r && isfinite(r->center_x) && isfinite(r->center_y) && isfinite(r->size_u) && r->size_u > 0.0 &&
           isfinite(r->size_v) && r->size_v > 0.0 && isfinite(r->angle_rad);
}

int subpixel_te_rectangle_fraction(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                   double dx, double dy, double *fraction_out) {
    if (!fraction_out || !rect_ok(rectangle) || !isfinite(sample_x) || !isfinite(sample_y) || !isfinite(dx) ||
        !(dx > 0.0) || !isfinite(dy) || !(dy > 0.0))
        return ST_INVALID;
    const double hu = 0.5 * rectangle->size_u, hv = 0.5 * rectangle->size_v;
    const double rx = sample_x - rectangle->center_x, ry = sample_y - rectangle->center_y;
    if (!(hu > 0.0) || !(hv > 0.0) || !isfinite(rx) || !isfinite(ry)) return ST_NUMERIC;
    const double c = cos(rectangle->angle_rad), s = sin(rectangle->angle_rad);
    /* the sample in the rectangle's frame; a point (a dx, b dy) away from
     * the sample, a and b in [-1/2, 1/2], sits at (u0 + c dx a + s dy b,
     * v0 - s dx a + c dy b) */
    const double u0 = c * rx + s * ry, v0 = c * ry - s * rx;
    const double plane[4][3] = {
        {c * dx, s * dy, hu - u0},    /*  u <= hu */
        {-c * dx, -s * dy, hu + u0},  /* -u <= hu */
        {-s * dx, c * dy, hv - v0},   /*  v <= hv */
        {s * dx, -c * dy, hv + v0},   /* -v <= hv */
    };
    for (int p = 0; p < 4; p++)
        if (!finite_all(plane[p][0], plane[p][1], plane[p][2])) return ST_NUMERIC;
    vtx_t buf[2][CLIP_MAX] = {{{-0.5, -0.5}, {0.5, -0.5}, {0.5, 0.5}, {-0.5, 0.5}}};
    int n = 4, cur = 0;
    for (int p = 0; p < 4 && n > 0; p++) {
        n = clip_half_plane(buf[cur], n, plane[p][0], plane[p][1], plane[p][2], buf[1 - cur]);
        if (n < 0) return ST_NUMERIC;
        cur = 1 - cur;
    }
    double area2 = 0.0; /* shoelace, fanned from the first vertex */
    for (int q = 1; q + 1 < n; q++) {
        const vtx_t o = buf[cur][0], a = buf[cur][q], b = buf[cur][q + 1];
        area2 += (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x);
    }
    const double f = 0.5 * fabs(area2);
    if (!isfinite(f) || f > 1.0 + 128.0 * DBL_EPSILON) return ST_NUMERIC;
    *fraction_out = f > 1.0 ? 1.0 : f;
    return ST_OK;
}

/* The parameter interval [lo, hi] of t where |w0 + dw t| <= half; returns 0
 * when no t qualifies. */
static int slab_interval(double w0, double dw, double half, double len, double *lo, double *hi) {
    if (fabs(dw) < 1e-300) {
        if (fabs(w0) > half * (1.0 + 1e-12)) return 0;
        *lo = 0.0;
        *hi = len;
        return 1;
    }
    const double t1 = (-half - w0) / dw, t2 = (half - w0) / dw;
    *lo = fmin(t1, t2);
    *hi = fmax(t1, t2);
    return 1;
}

int subpixel_te_rectangle_edge_fraction(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                        int edge_axis, double length, double *fraction_out) {
    if (!rectangle || !fraction_out || !isfinite(sample_x) || !isfinite(sample_y)) return ST_INVALID;
    if (edge_axis != 1 && edge_axis != 2) return ST_INVALID;
    if (!isfinite(length) || !(length > 0.0)) return ST_INVALID;
    if (!isfinite(rectangle->center_x) || !isfinite(rectangle->center_y) || !isfinite(rectangle->size_u) ||
        !(rectangle->size_u >= 0.0) || !isfinite(rectangle->size_v) || !(rectangle->size_v >= 0.0) ||
        !isfinite(rectangle->angle_rad))
        return ST_INVALID;
    const double rx = sample_x - rectangle->center_x, ry = sample_y - rectangle->center_y;
    if (!isfinite(rx) || !isfinite(ry)) return ST_NUMERIC;
    if (rectangle->size_u == 0.0) return ST_NUMERIC;
    const double c = cos(rectangle->angle_rad), s = sin(rectangle->angle_rad);
    /* the edge runs from the sample along +x (axis 1) or +y (axis 2) */
    const double ex = edge_axis == 1 ? 1.0 : 0.0, ey = edge_axis == 1 ? 0.0 : 1.0;
    const double u0 = rx * c + ry * s, v0 = ry * c - rx * s;
    const double du = ex * c + ey * s, dv = ey * c - ex * s;
    double alo, ahi, blo, bhi;
    if (!slab_interval(u0, du, 0.5 * rectangle->size_u, length, &alo, &ahi) ||
        !slab_interval(v0, dv, 0.5 * rectangle->size_v, length, &blo, &bhi)) {
        *fraction_out = 0.0;
        return ST_OK;
    }
    const double lo = fmax(fmax(alo, blo), 0.0), hi = fmin(fmin(ahi, bhi), length);
    *fraction_out = hi > lo ? (hi - lo) / length : 0.0;
    return ST_OK;
}

static int mix_args_ok(double f, double eb, double ei) {
    return isfinite(f) && f >= 0.0 && f <= 1.0 && isfinite(eb) && eb >= 1.0 && isfinite(ei) && ei >= 1.0;
}

int subpixel_te_mix_epsilon_harmonic(double fraction, double eps_background, double eps_inside,
                                     double *epsilon_r_out) {
    if (!epsilon_r_out || !mix_args_ok(fraction, eps_background, eps_inside)) return ST_INVALID;
    const double inv = (1.0 - fraction) / eps_background + fraction / eps_inside;
    if (!isfinite(inv) || !(inv > 0.0)) return ST_NUMERIC;
    *epsilon_r_out = 1.0 / inv;
    return ST_OK;
}

int subpixel_te_mix_epsilon(double fraction, double eps_background, double eps_inside, double *epsilon_r_out) {
    if (!epsilon_r_out || !mix_args_ok(fraction, eps_background, eps_inside)) return ST_INVALID;
    double e;
    if (fraction == 0.0) {
        e = eps_background;
    } else if (fraction == 1.0) {
        e = eps_inside;
    } else {
        /* step up from the smaller permittivity by the larger one's share,
         * one rounding, so the mix never leaves [min, max] */
        const int in_hi = eps_inside >= eps_background;
        const double lo = in_hi ? eps_background : eps_inside, hi = in_hi ? eps_inside : eps_background;
        e = fma(in_hi ? fraction : 1.0 - fraction, hi - lo, lo);
    }
    if (!isfinite(e) || e < 1.0) return ST_NUMERIC;
    *epsilon_r_out = e;
    return ST_OK;
}

int subpixel_te_rectangle_epsilon(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                  double dx, double dy, double eps_background, double eps_inside,
                                  double *fraction_out, double *epsilon_r_out) {
    double f, e;
    if (!fraction_out || !epsilon_r_out || fraction_out == epsilon_r_out) return ST_INVALID;
    int st = subpixel_te_rectangle_fraction(rectangle, sample_x, sample_y, dx, dy, &f);
    if (st != ST_OK) return st;
    st = subpixel_te_mix_epsilon(f, eps_background, eps_inside, &e);
    if (st != ST_OK) return st;
    *fraction_out = f;
    *epsilon_r_out = e;
    return ST_OK;
}

int subpixel_te_mix_epsilon_tensor(double fraction, double eps_background, double eps_inside, double normal_rad,
                                   double *minv_xx, double *minv_xy, double *minv_yy) {
    if (!minv_xx || !minv_xy || !minv_yy || !mix_args_ok(fraction, eps_background, eps_inside) ||
        !isfinite(normal_rad))
        return ST_INVALID;
    /* along the normal the layers are in series (harmonic mean of eps),
     * along the interface in parallel (arithmetic mean) */
    const double lam_n = (1.0 - fraction) / eps_background + fraction / eps_inside;
    const double eps_t = (1.0 - fraction) * eps_background + fraction * eps_inside;
    if (!isfinite(lam_n) || !(lam_n > 0.0) || !isfinite(eps_t) || !(eps_t > 0.0)) return ST_NUMERIC;
    const double lam_t = 1.0 / eps_t;
    const double c = cos(normal_rad), s = sin(normal_rad);
    *minv_xx = lam_n * c * c + lam_t * s * s;
    *minv_yy = lam_n * s * s + lam_t * c * c;
    *minv_xy = (lam_n - lam_t) * c * s;
    return ST_OK;
}

/* ---- three dimensions ---------------------------------------------------------- */
#include "../smooth3.h"

int fdtd_b200_subpixel_tensor3(double fraction, const double eps_background[9], const double eps_inside[9],
                               const double normal[3], double minv_out[9]) {
    double m[9];
    if (!eps_background || !eps_inside || !normal || !minv_out || !isfinite(fraction)) return ST_INVALID;
    for (int q = 0; q < 9; q++)
        if (!isfinite(eps_background[q]) || !isfinite(eps_inside[q])) return ST_INVALID;
    for (int a = 0; a < 3; a++)
        for (int b = a + 1; b < 3; b++)
            if (eps_background[3 * a + b] != eps_background[3 * b + a] ||
                eps_inside[3 * a + b] != eps_inside[3 * b + a])
                return ST_INVALID;
    if (rfb_sm_mix(fraction, eps_background, eps_inside, normal, m) != 0) return ST_INVALID;
    for (int q = 0; q < 9; q++)
        if (!isfinite(m[q])) return ST_NUMERIC;
    for (int q = 0; q < 9; q++) minv_out[q] = m[q];
    return ST_OK;
}
