/* cpml.c -- CPML parameters and graded profiles (host, FP64, rfsyn's formulas
 * of engine/fdtd/cpml.c:10-150) and the CPML step-wise sweeps (GPU). */
#include <math.h>
#include <stdlib.h>

#include "host.h"

rfb_fields_t *rfb_grid_device(fdtd_grid_t *g, rfb_geom_t *geom, double *h[6]);

rfb_cpml_ext_t *rfb_cpml_ext(const cpml_t *p) {
    rfb_cpml_ext_t *x = (rfb_cpml_ext_t *)p;
    return (x && x->magic == RFB_CPML_MAGIC) ? x : NULL;
}

cpml_params_t cpml_default_params(size_t npml) {
    cpml_params_t p;
    p.npml = npml;
    p.m = 3.0;
    p.ma = 1.0;
    p.kappa_max = 7.0;
    p.alpha_max = 0.05;
    p.r0 = 1e-6;
    return p;
}

/* One graded coefficient triple at depth rho into a layer of thickness d
 * (rfsyn cpml.c:41-57): sigma = sigma_max r^m, kappa = 1 + (kappa_max-1) r^m,
 * alpha = alpha_max (1-r)^ma, b = exp(-(sigma/kappa + alpha) dt / eps0),
 * a = sigma (b-1) / (dx kappa (sigma + kappa alpha)). */
static void graded(double rho, double d, double dx, double dt, double sigma_max, const cpml_params_t *p,
                   double *kinv, double *b, double *a) {
    if (rho < 0.0) {
        *kinv = 1.0; *b = 1.0; *a = 0.0;
        return;
    }
    double r = rho / d;
    if (r > 1.0) r = 1.0;
    double sigma = sigma_max * pow(r, p->m);
    double kappa = 1.0 + (p->kappa_max - 1.0) * pow(r, p->m);
    double alpha = p->alpha_max * pow(1.0 - r, p->ma);
    double bb = exp(-(sigma / kappa + alpha) * dt / EPS0);
    double aa = (sigma > 0.0) ? sigma * (bb - 1.0) / (dx * kappa * (sigma + kappa * alpha)) : 0.0;
    *kinv = 1.0 / kappa;
    *b = bb;
    *a = aa;
}

/* Integer positions x = q dx (q = 0..n) and half positions (q + 1/2) dx
 * (q = 0..n-1); depth measured from the nearer absorbing face. */
static int axis_profiles(size_t n, double dx, double dt, double sigma_max, const cpml_params_t *p, double **km,
                         double **bm, double **am, double **kh, double **bh, double **ah) {
    *km = malloc((n + 1) * sizeof(double));
    *bm = malloc((n + 1) * sizeof(double));
    *am = malloc((n + 1) * sizeof(double));
    *kh = malloc(n * sizeof(double));
    *bh = malloc(n * sizeof(double));
    *ah = malloc(n * sizeof(double));
    if (!*km || !*bm || !*am || !*kh || !*bh || !*ah) return -1;
    const double d = (double)p->npml * dx;
    const double len = (double)n * dx;
    for (size_t q = 0; q <= n; q++) {
        double x = (double)q * dx, rho = -1.0;
        if (x < d) rho = d - x;
        else if (x > len - d) rho = x - (len - d);
        graded(rho, d, dx, dt, sigma_max, p, &(*km)[q], &(*bm)[q], &(*am)[q]);
    }
    for (size_t q = 0; q < n; q++) {
        double x = ((double)q + 0.5) * dx, rho = -1.0;
        if (x < d) rho = d - x;
        else if (x > len - d) rho = x - (len - d);
        graded(rho, d, dx, dt, sigma_max, p, &(*kh)[q], &(*bh)[q], &(*ah)[q]);
    }
    return 0;
}

static void set_identity(double *k, double *b, double *a, size_t n) {
    for (size_t q = 0; q < n; q++) { k[q] = 1.0; b[q] = 1.0; a[q] = 0.0; }
}

cpml_t *cpml_create(const fdtd_grid_t *g, cpml_params_t params) {
    if (!g || params.npml == 0 || !isfinite(params.r0) || params.r0 <= 0.0 || params.r0 >= 1.0 ||
        !isfinite(params.m) || params.m <= 0.0 || !isfinite(params.ma) || params.ma < 0.0 ||
        !isfinite(params.kappa_max) || params.kappa_max < 1.0 || !isfinite(params.alpha_max) ||
        params.alpha_max < 0.0)
        return NULL;
    if ((!(g->periodic_axes & 1u) && params.npml >= (g->nx + 1) / 2) ||
        (!(g->periodic_axes & 2u) && params.npml >= (g->ny + 1) / 2) ||
        (!(g->periodic_axes & 4u) && params.npml >= (g->nz + 1) / 2))
        return NULL;
    rfb_cpml_ext_t *x = calloc(1, sizeof(*x));
    if (!x) return NULL;
    x->magic = RFB_CPML_MAGIC;
    x->nx = g->nx; x->ny = g->ny; x->nz = g->nz;
    x->periodic = g->periodic_axes;
    x->dt = g->dt;
    cpml_t *p = &x->pub;
    p->npml = params.npml;
    p->dx = g->dx;
    /* optimal sigma_max for reflection r0 (cpml.c:103-105) */
    double eta0 = sqrt(MU0 / EPS0);
    double sigma_max = -(params.m + 1.0) * log(params.r0) / (2.0 * eta0 * (double)params.npml * g->dx);
    int ok = 1;
    ok &= axis_profiles(g->nx, g->dx, g->dt, sigma_max, &params, &p->kappa_inv_m_x, &p->b_m_x, &p->a_m_x,
                        &p->kappa_inv_h_x, &p->b_h_x, &p->a_h_x) == 0;
    ok &= axis_profiles(g->ny, g->dx, g->dt, sigma_max, &params, &p->kappa_inv_m_y, &p->b_m_y, &p->a_m_y,
                        &p->kappa_inv_h_y, &p->b_h_y, &p->a_h_y) == 0;
    ok &= axis_profiles(g->nz, g->dx, g->dt, sigma_max, &params, &p->kappa_inv_m_z, &p->b_m_z, &p->a_m_z,
                        &p->kappa_inv_h_z, &p->b_h_z, &p->a_h_z) == 0;
    if (!ok) {
        cpml_destroy(p);
        return NULL;
    }
    /* periodic axes: identity stretching, no memory (cpml.c:113-125) */
    if (g->periodic_axes & 1u) {
        set_identity(p->kappa_inv_m_x, p->b_m_x, p->a_m_x, g->nx + 1);
        set_identity(p->kappa_inv_h_x, p->b_h_x, p->a_h_x, g->nx);
    }
    if (g->periodic_axes & 2u) {
        set_identity(p->kappa_inv_m_y, p->b_m_y, p->a_m_y, g->ny + 1);
        set_identity(p->kappa_inv_h_y, p->b_h_y, p->a_h_y, g->ny);
    }
    if (g->periodic_axes & 4u) {
        set_identity(p->kappa_inv_m_z, p->b_m_z, p->a_m_z, g->nz + 1);
        set_identity(p->kappa_inv_h_z, p->b_h_z, p->a_h_z, g->nz);
    }
    return p;
}

void cpml_destroy(cpml_t *p) {
    if (!p) return;
    free(p->kappa_inv_m_x); free(p->b_m_x); free(p->a_m_x);
    free(p->kappa_inv_m_y); free(p->b_m_y); free(p->a_m_y);
    free(p->kappa_inv_m_z); free(p->b_m_z); free(p->a_m_z);
    free(p->kappa_inv_h_x); free(p->b_h_x); free(p->a_h_x);
    free(p->kappa_inv_h_y); free(p->b_h_y); free(p->a_h_y);
    free(p->kappa_inv_h_z); free(p->b_h_z); free(p->a_h_z);
    rfb_cpml_ext_t *x = rfb_cpml_ext(p);
    if (x) {
        rfb_cpml_dev_destroy(x->dev);
        x->magic = 0;
        free(x);
    }
}

void rfb_cpml_desc_from(const cpml_t *p, rfb_cpml_desc_t *d) {
    d->kinv_m[0] = p->kappa_inv_m_x; d->b_m[0] = p->b_m_x; d->a_m[0] = p->a_m_x;
    d->kinv_m[1] = p->kappa_inv_m_y; d->b_m[1] = p->b_m_y; d->a_m[1] = p->a_m_y;
    d->kinv_m[2] = p->kappa_inv_m_z; d->b_m[2] = p->b_m_z; d->a_m[2] = p->a_m_z;
    d->kinv_h[0] = p->kappa_inv_h_x; d->b_h[0] = p->b_h_x; d->a_h[0] = p->a_h_x;
    d->kinv_h[1] = p->kappa_inv_h_y; d->b_h[1] = p->b_h_y; d->a_h[1] = p->a_h_y;
    d->kinv_h[2] = p->kappa_inv_h_z; d->b_h[2] = p->b_h_z; d->a_h[2] = p->a_h_z;
}

/* Device CPML state (profiles + slab psi) of a cpml_t used with grid g. */
rfb_cpml_dev_t *rfb_cpml_device(cpml_t *p, const fdtd_grid_t *g) {
    rfb_cpml_ext_t *x = rfb_cpml_ext(p);
    if (!x || x->nx != g->nx || x->ny != g->ny || x->nz != g->nz) return NULL;
    if (!x->dev) {
        rfb_geom_t geom;
        rfb_geom_from_grid(g, &geom);
        rfb_cpml_desc_t d;
        rfb_cpml_desc_from(p, &d);
        x->dev = rfb_cpml_dev_create(&geom, &d);
    }
    return x->dev;
}

void fdtd_update_h_cpml(fdtd_grid_t *g, cpml_t *pml) {
    if (!g || !pml) return;
    rfb_cpml_dev_t *c = rfb_cpml_device(pml, g);
    if (!c) return;
    rfb_geom_t geom;
    double *h[6];
    rfb_fields_t *f = rfb_grid_device(g, &geom, h);
    if (!f) return;
    rfb_step_update_h(f, &geom, c, h);
}

void fdtd_update_e_cpml(fdtd_grid_t *g, cpml_t *pml) {
    if (!g || !pml) return;
    rfb_cpml_dev_t *c = rfb_cpml_device(pml, g);
    if (!c) return;
    rfb_geom_t geom;
    double *h[6];
    rfb_fields_t *f = rfb_grid_device(g, &geom, h);
    if (!f) return;
    rfb_step_update_e(f, &geom, c, NULL, g->dt / (EPS0 * g->dx), h);
}
