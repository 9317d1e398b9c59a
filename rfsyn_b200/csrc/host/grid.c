/* grid.c -- fdtd_grid_t lifecycle and the vacuum step-wise sweeps.
 * Semantics follow rfsyn engine/fdtd/grid.c:7-130; the sweeps run on the GPU. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "host.h"

rfb_grid_ext_t *rfb_grid_ext(const fdtd_grid_t *g) {
    rfb_grid_ext_t *x = (rfb_grid_ext_t *)g;
    return (x && x->magic == RFB_GRID_MAGIC) ? x : NULL;
}

/* Same acceptance rules as rfsyn's fdtd_grid_create (grid.c:7-46). */
int rfb_grid_geometry(fdtd_grid_t *g, size_t nx, size_t ny, size_t nz, double dx, double courant) {
    if (!nx || !ny || !nz || !isfinite(dx) || dx <= 0.0 || !isfinite(courant) || courant <= 0.0 || courant > 1.0)
        return -1;
    if (nx > SIZE_MAX - 1 || ny > SIZE_MAX - 1 || nz > SIZE_MAX - 1) return -1;
    size_t nx1 = nx + 1, ny1 = ny + 1, nz1 = nz + 1;
    if (nx1 > SIZE_MAX / ny1 || (nx1 * ny1) > SIZE_MAX / nz1) return -1;
    size_t total = nx1 * ny1 * nz1;
    g->periodic_axes = 0;
    g->nx = nx;
    g->ny = ny;
    g->nz = nz;
    g->dx = dx;
    /* dt = S * dx / (c sqrt 3), evaluated as rfsyn does (grid.c:27-28). */
    double dt_max = dx / (C0 * sqrt(3.0));
    g->dt = courant * dt_max;
    if (total > SIZE_MAX / sizeof(double) || !isfinite(g->dt) || g->dt <= 0.0) return -1;
    g->ex = g->ey = g->ez = g->hx = g->hy = g->hz = NULL;
    return 0;
}

fdtd_grid_t *fdtd_grid_create(size_t nx, size_t ny, size_t nz, double dx, double courant_safety_factor) {
    rfb_grid_ext_t *x = calloc(1, sizeof(*x));
    if (!x) return NULL;
    if (rfb_grid_geometry(&x->pub, nx, ny, nz, dx, courant_safety_factor) != 0) {
        free(x);
        return NULL;
    }
    x->magic = RFB_GRID_MAGIC;
    size_t total = (nx + 1) * (ny + 1) * (nz + 1);
    fdtd_grid_t *g = &x->pub;
    g->ex = calloc(total, sizeof(double));
    g->ey = calloc(total, sizeof(double));
    g->ez = calloc(total, sizeof(double));
    g->hx = calloc(total, sizeof(double));
    g->hy = calloc(total, sizeof(double));
    g->hz = calloc(total, sizeof(double));
    if (!g->ex || !g->ey || !g->ez || !g->hx || !g->hy || !g->hz) {
        fdtd_grid_destroy(g);
        return NULL;
    }
    return g;
}

void fdtd_grid_destroy(fdtd_grid_t *g) {
    if (!g) return;
    rfb_grid_ext_t *x = rfb_grid_ext(g);
    free(g->ex); free(g->ey); free(g->ez);
    free(g->hx); free(g->hy); free(g->hz);
    if (x) {
        rfb_fields_destroy(x->dev);
        x->magic = 0;
        free(x);
    }
}

int fdtd_grid_set_periodic(fdtd_grid_t *g, unsigned axes) {
    if (!g || (axes & ~7u)) return -1;
    g->periodic_axes = axes;
    return 0;
}

void rfb_geom_from_grid(const fdtd_grid_t *g, rfb_geom_t *out) {
    out->nx = (int)g->nx;
    out->ny = (int)g->ny;
    out->nz = (int)g->nz;
    out->periodic = g->periodic_axes;
    out->dx = g->dx;
    out->dt = g->dt;
}

/* Device mirror of a host grid, created on first use. */
static rfb_fields_t *grid_device(fdtd_grid_t *g, rfb_geom_t *geom) {
    rfb_grid_ext_t *x = rfb_grid_ext(g);
    if (!x || !g->ex) return NULL;
    if (g->nx > INT32_MAX - 2 || g->ny > INT32_MAX - 2 || g->nz > INT32_MAX - 2) return NULL;
    rfb_geom_from_grid(g, geom);
    if (!x->dev) x->dev = rfb_fields_create(geom);
    return x->dev;
}

static void host_fields(fdtd_grid_t *g, double *h[6]) {
    h[0] = g->ex; h[1] = g->ey; h[2] = g->ez;
    h[3] = g->hx; h[4] = g->hy; h[5] = g->hz;
}

void fdtd_update_h(fdtd_grid_t *g) {
    if (!g) return;
    rfb_geom_t geom;
    rfb_fields_t *f = grid_device(g, &geom);
    if (!f) return;
    double *h[6];
    host_fields(g, h);
    rfb_step_update_h(f, &geom, NULL, h);
}

void fdtd_update_e(fdtd_grid_t *g) {
    if (!g) return;
    rfb_geom_t geom;
    rfb_fields_t *f = grid_device(g, &geom);
    if (!f) return;
    double *h[6];
    host_fields(g, h);
    /* ca = dt / (eps0 dx): grid.c:93 */
    rfb_step_update_e(f, &geom, NULL, NULL, g->dt / (EPS0 * g->dx), h);
}

/* Used by cpml.c and materials.c. */
rfb_fields_t *rfb_grid_device(fdtd_grid_t *g, rfb_geom_t *geom, double *h[6]) {
    rfb_fields_t *f = grid_device(g, geom);
    if (f) host_fields(g, h);
    return f;
}
