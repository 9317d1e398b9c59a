/*
 * sphere_raster.h -- TEST INFRASTRUCTURE (oracle).  CPU restatement of the
 * sphere rasteriser (fill fraction of the unit cube around each E sample by
 * 8^3 supersampling, FP64; diagonal of the smoothed inverse permittivity,
 * Farjadpour et al., Opt. Lett. 31, 2972 (2006), or with smoothing 2 its
 * full row, eps^-1 = <1/eps> n n^T + (1/<eps>) (I - n n^T), where the 3x3
 * update may run) into a dense per-sample
 * state, sphere by sphere in list order.  Shared by the oracle and by the
 * scene driver built over rfsyn (which then hands the state to rfsyn's own
 * materials API).
 */
#ifndef RFSYN_ORACLE_SPHERE_RASTER_H
#define RFSYN_ORACLE_SPHERE_RASTER_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include "scene.h"

/* Fill fraction of the unit cube centred at (x, y, z) inside sphere sp and
 * the squared normal component along `axis` at that point. */
static double sr_cube_fraction(double x, double y, double z, const scn_sphere_t *sp, double *n2, int axis) {
    double dx = x - sp->cx, dy = y - sp->cy, dz = z - sp->cz;
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    double comp = axis == 0 ? dx : axis == 1 ? dy : dz;
    *n2 = d > 0.0 ? (comp / d) * (comp / d) : 0.0;
    const double h = 0.8660254037844386;
    if (d + h <= sp->radius) return 1.0;
    if (d - h >= sp->radius) return 0.0;
    double r2 = sp->radius * sp->radius;
    int count = 0;
    for (int a = 0; a < 8; a++) {
        double px = x + (((double)a + 0.5) / 8.0 - 0.5) - sp->cx;
        for (int b = 0; b < 8; b++) {
            double py = y + (((double)b + 0.5) / 8.0 - 0.5) - sp->cy;
            for (int e = 0; e < 8; e++) {
                double pz = z + (((double)e + 0.5) / 8.0 - 0.5) - sp->cz;
                if (px * px + py * py + pz * pz <= r2) count++;
            }
        }
    }
    return (double)count / 512.0;
}

/* Callbacks into the caller's dense material state. */
typedef struct {
    void *ctx;
    /* table material of canonical cell w */
    void (*background)(void *ctx, size_t w, double *eps_r, double *sigma);
    /* whole cell inside a dielectric sphere: id <- sphere, clear samples */
    int (*fill_cell)(void *ctx, size_t w, const scn_sphere_t *sp);
    /* whole cell inside a dispersive sphere: clear samples, 3 dispersive */
    int (*fill_cell_disp)(void *ctx, size_t w, const scn_disp_t *d);
    /* sample c of cell w: scalar override (clears a dispersive sample) */
    int (*set_sample)(void *ctx, size_t w, int c, double eps_r, double sigma);
    int (*set_sample_disp)(void *ctx, size_t w, int c, const scn_disp_t *d);
    /* sample c of cell w: row of a 3x3 sample with loss sigma (clears the
     * sample's other descriptions); NULL: not supported */
    int (*set_sample_t3)(void *ctx, size_t w, int c, const double row[3], double sigma);
} sr_target_t;

/* Rasterises every sphere of s into the target.  n: nx, ny, nz; periodic
 * bits; `canon` maps (i, j, k) to the canonical padded index. */
static int sr_rasterise(const scn_scene_t *s, const size_t n[3], unsigned periodic,
                        size_t (*canon)(const void *geo, size_t i, size_t j, size_t k), const void *geo,
                        const sr_target_t *t) {
    for (size_t q = 0; q < s->n_spheres; q++) {
        const scn_sphere_t *sp = &s->spheres[q];
        const scn_disp_t *dm = sp->disp >= 0 ? &s->disp[sp->disp] : NULL;
        long lo[3], hi[3];
        double cen[3] = {sp->cx, sp->cy, sp->cz};
        for (int a = 0; a < 3; a++) {
            lo[a] = (long)floor(cen[a] - sp->radius) - 2;
            hi[a] = (long)ceil(cen[a] + sp->radius) + 2;
            if (lo[a] < 0) lo[a] = 0;
            if (hi[a] > (long)n[a]) hi[a] = (long)n[a];
        }
        for (long i = lo[0]; i <= hi[0]; i++)
            for (long j = lo[1]; j <= hi[1]; j++)
                for (long k = lo[2]; k <= hi[2]; k++) {
                    double f[3], n2[3];
                    f[0] = sr_cube_fraction((double)i + 0.5, (double)j, (double)k, sp, &n2[0], 0);
                    f[1] = sr_cube_fraction((double)i, (double)j + 0.5, (double)k, sp, &n2[1], 1);
                    f[2] = sr_cube_fraction((double)i, (double)j, (double)k + 0.5, sp, &n2[2], 2);
                    int valid[3];
                    for (int c = 0; c < 3; c++) {
                        size_t ni = n[0] + ((c != 0 && !(periodic & 1u)) ? 1 : 0);
                        size_t nj = n[1] + ((c != 1 && !(periodic & 2u)) ? 1 : 0);
                        size_t nk = n[2] + ((c != 2 && !(periodic & 4u)) ? 1 : 0);
                        valid[c] = (size_t)i < ni && (size_t)j < nj && (size_t)k < nk;
                    }
                    size_t w = canon(geo, (size_t)i, (size_t)j, (size_t)k);
                    if (f[0] == 1.0 && f[1] == 1.0 && f[2] == 1.0 && valid[0] && valid[1] && valid[2]) {
                        int rc = dm ? t->fill_cell_disp(t->ctx, w, dm) : t->fill_cell(t->ctx, w, sp);
                        if (rc != 0) return -1;
                        continue;
                    }
                    for (int c = 0; c < 3; c++) {
                        if (!valid[c] || f[c] <= 0.0) continue;
                        if (dm) {
                            if (f[c] >= 0.5 && t->set_sample_disp(t->ctx, w, c, dm) != 0) return -1;
                            continue;
                        }
                        double eps_c, sig_c;
                        if (s->smoothing == 2 && f[c] < 1.0) {
                            /* full row; the 3x3 update needs the cell in
                             * [1, n-1] on every axis without wrap */
                            double eb, sb;
                            t->background(t->ctx, w, &eb, &sb);
                            const double p[3] = {(double)i + (c == 0 ? 0.5 : 0.0), (double)j + (c == 1 ? 0.5 : 0.0),
                                                 (double)k + (c == 2 ? 0.5 : 0.0)};
                            double nv[3] = {p[0] - sp->cx, p[1] - sp->cy, p[2] - sp->cz};
                            const double d = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                            if (d > 0.0) {
                                nv[0] /= d; nv[1] /= d; nv[2] /= d;
                            } else {
                                nv[0] = nv[1] = nv[2] = 0.0;
                                nv[c] = 1.0;
                            }
                            const double lam_n = (1.0 - f[c]) / eb + f[c] / sp->eps_r;
                            const double lam_t = 1.0 / ((1.0 - f[c]) * eb + f[c] * sp->eps_r);
                            double row[3];
                            for (int b = 0; b < 3; b++) row[b] = (lam_n - lam_t) * nv[c] * nv[b] + (b == c ? lam_t : 0.0);
                            sig_c = f[c] * sp->sigma + (1.0 - f[c]) * sb;
                            const long pi[3] = {i, j, k};
                            int margin = 1;
                            for (int a = 0; a < 3; a++)
                                if (!(periodic & (1u << a)) && (pi[a] < 1 || pi[a] + 1 > (long)n[a])) margin = 0;
                            if (margin) {
                                if (!t->set_sample_t3 || t->set_sample_t3(t->ctx, w, c, row, sig_c) != 0) return -1;
                                continue;
                            }
                            eps_c = 1.0 / row[c];
                        } else if (!s->smoothing || f[c] == 1.0) {
                            if (f[c] < 0.5) continue;
                            eps_c = sp->eps_r;
                            sig_c = sp->sigma;
                        } else {
                            double eb, sb;
                            t->background(t->ctx, w, &eb, &sb);
                            double mean = f[c] * sp->eps_r + (1.0 - f[c]) * eb;
                            double minv = f[c] / sp->eps_r + (1.0 - f[c]) / eb;
                            double inv = n2[c] * minv + (1.0 - n2[c]) / mean;
                            eps_c = 1.0 / inv;
                            sig_c = f[c] * sp->sigma + (1.0 - f[c]) * sb;
                        }
                        if (t->set_sample(t->ctx, w, c, eps_c, sig_c) != 0) return -1;
                    }
                }
    }
    return 0;
}

#endif
