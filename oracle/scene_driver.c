/*
 * scene_driver.c -- TEST INFRASTRUCTURE (oracle).  Replays a scn_scene_t
 * through rfsyn's public C API: fdtd_grid_create, cpml_create,
 * materials_*, source_apply, fdtd_update_{h,e}*_cpml / _materials,
 * probe_td_record and probe_dft_record.  The same source is compiled
 *   - with rfsyn's own sources into oracle/_ref/librfsyn_ref.so (golden runs),
 *   - against librfsyn_fdtd_b200.so into oracle/lib/libscene_driver_b200.so
 *     (exercises the GPU behind rfsyn's step-wise functions).
 * scn_setup() is also usable as an fdtd_material_setup_fn.
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "rfsyn_fdtd.h"
#include "scene.h"
#include "sphere_raster.h"
#ifdef SCN_WITH_B200_EXT
#include "rfsyn_fdtd_b200.h"
#endif

static field_component_t comp_of(int c) { return (field_component_t)c; }

#ifndef SCN_WITH_B200_EXT
static double static_eps(const scn_disp_t *d) {
    double e = d->eps_inf;
    for (int p = 0; p < d->npoles; p++) e += d->delta_eps[p];
    return e;
}

/* Spheres for rfsyn: rasterised into a shadow state with the shared
 * rasteriser, then handed to rfsyn's own API as column boxes of equal id
 * followed by per-component overrides in increasing key order (rfsyn keeps
 * overrides sorted, so in-order insertion appends). */
typedef struct {
    const fdtd_grid_t *g;
    materials_t *m;
    uint8_t *ids;
    double teps[256], tsig[256];
    int ntab;
    int32_t *ovr;   /* per (cell, comp): index into oe/os or -1 */
    double *oe, *os;
    size_t no, cap;
} shadow_t;

static int sh_id(shadow_t *h, double eps, double sig) {
    material_id_t id;
    if (materials_register(h->m, eps, sig, &id) != 0) return -1;
    h->teps[id] = eps;
    h->tsig[id] = sig;
    if ((int)id >= h->ntab) h->ntab = (int)id + 1;
    return (int)id;
}
static void sh_bg(void *ctx, size_t w, double *eps, double *sig) {
    shadow_t *h = (shadow_t *)ctx;
    *eps = h->teps[h->ids[w]];
    *sig = h->tsig[h->ids[w]];
}
static int sh_set(shadow_t *h, size_t w, int c, double eps, double sig) {
    if (h->ovr[3 * w + (size_t)c] < 0) {
        if (h->no == h->cap) {
            h->cap = h->cap ? 2 * h->cap : 1024;
            double *ne = realloc(h->oe, h->cap * sizeof(double));
            if (ne) h->oe = ne;
            double *ns = realloc(h->os, h->cap * sizeof(double));
            if (ns) h->os = ns;
            if (!ne || !ns) return -1;
        }
        h->ovr[3 * w + (size_t)c] = (int32_t)h->no++;
    }
    h->oe[h->ovr[3 * w + (size_t)c]] = eps;
    h->os[h->ovr[3 * w + (size_t)c]] = sig;
    return 0;
}
static int sh_fill(void *ctx, size_t w, const scn_sphere_t *sp) {
    shadow_t *h = (shadow_t *)ctx;
    int id = sh_id(h, sp->eps_r, sp->sigma);
    if (id < 0) return -1;
    h->ids[w] = (uint8_t)id;
    for (int c = 0; c < 3; c++) h->ovr[3 * w + (size_t)c] = -1;
    return 0;
}
static int sh_fill_disp(void *ctx, size_t w, const scn_disp_t *d) {
    shadow_t *h = (shadow_t *)ctx;
    int id = sh_id(h, static_eps(d), d->sigma);
    if (id < 0) return -1;
    h->ids[w] = (uint8_t)id;
    for (int c = 0; c < 3; c++) h->ovr[3 * w + (size_t)c] = -1;
    return 0;
}
static int sh_sample(void *ctx, size_t w, int c, double eps, double sig) { return sh_set((shadow_t *)ctx, w, c, eps, sig); }
static int sh_sample_disp(void *ctx, size_t w, int c, const scn_disp_t *d) {
    return sh_set((shadow_t *)ctx, w, c, static_eps(d), d->sigma);
}
static size_t sh_canon(const void *geo, size_t i, size_t j, size_t k) { return fdtd_index((const fdtd_grid_t *)geo, i, j, k); }

static int ref_spheres(const fdtd_grid_t *g, materials_t *m, const scn_scene_t *s) {
    int rc = -1;
    size_t total = (g->nx + 1) * (g->ny + 1) * (g->nz + 1);
    shadow_t h;
    memset(&h, 0, sizeof h);
    h.g = g;
    h.m = m;
    h.ids = calloc(total, 1);
    h.ovr = malloc(3 * total * sizeof(int32_t));
    if (!h.ids || !h.ovr) goto out;
    for (size_t q = 0; q < 3 * total; q++) h.ovr[q] = -1;
    if (sh_id(&h, 1.0, 0.0) != 0) goto out;
    /* the spheres are applied after the scene's boxes, which this shadow does
     * not track: scenes given to rfsyn with spheres carry no boxes */
    if (s->n_boxes) goto out;
    {
        const size_t n[3] = {g->nx, g->ny, g->nz};
        sr_target_t tg = {&h, sh_bg, sh_fill, sh_fill_disp, sh_sample, sh_sample_disp};
        if (sr_rasterise(s, n, g->periodic_axes, sh_canon, g, &tg) != 0) goto out;
    }
    /* ids: runs of equal non-vacuum id along k become boxes */
    for (size_t i = 0; i <= g->nx; i++)
        for (size_t j = 0; j <= g->ny; j++) {
            size_t base = (i * (g->ny + 1) + j) * (g->nz + 1);
            size_t k = 0;
            while (k <= g->nz) {
                uint8_t id = h.ids[base + k];
                size_t k1 = k + 1;
                while (k1 <= g->nz && h.ids[base + k1] == id) k1++;
                if (id != 0 && materials_assign_box(m, g, i, i + 1, j, j + 1, k, k1, id) != 0) goto out;
                k = k1;
            }
        }
    for (size_t q = 0; q < 3 * total; q++) {
        if (h.ovr[q] < 0) continue;
        size_t w = q / 3, c = q % 3, kk = w % (g->nz + 1), row = w / (g->nz + 1);
        if (materials_set_component(m, g, comp_of((int)c), row / (g->ny + 1), row % (g->ny + 1), kk, h.oe[h.ovr[q]],
                                    h.os[h.ovr[q]]) != 0)
            goto out;
    }
    rc = 0;
out:
    free(h.ids);
    free(h.ovr);
    free(h.oe);
    free(h.os);
    return rc;
}
#endif

/* Applies boxes, then scalar overrides, then tensor edges (in list order). */
int scn_setup(const fdtd_grid_t *g, materials_t *m, void *ctx) {
    const scn_scene_t *s = (const scn_scene_t *)ctx;
    /* the plane wave is a run option (fdtd_b200_config_t), not a material */
    for (size_t q = 0; q < s->n_boxes; q++) {
        const scn_box_t *b = &s->boxes[q];
        if (materials_set_box(m, g, b->i0, b->i1, b->j0, b->j1, b->k0, b->k1, b->eps_r, b->sigma) != 0) return -1;
    }
    for (size_t q = 0; q < s->n_comps; q++) {
        const scn_comp_t *c = &s->comps[q];
        if (materials_set_component(m, g, comp_of(c->comp), c->i, c->j, c->k, c->eps_r, c->sigma) != 0) return -1;
    }
    for (size_t q = 0; q < s->n_tensors; q++) {
        const scn_tensor_t *t = &s->tensors[q];
        if (materials_set_component_tensor(m, g, comp_of(t->comp), t->i, t->j, t->k, t->m11, t->m12, t->m22) != 0)
            return -1;
    }
#ifdef SCN_WITH_B200_EXT
    for (size_t q = 0; q < s->n_disp; q++) {
        const scn_disp_t *d = &s->disp[q];
        fdtd_b200_dispersive_t md;
        memset(&md, 0, sizeof md);
        md.eps_inf = d->eps_inf;
        md.sigma = d->sigma;
        md.n_poles = d->npoles;
        for (int p = 0; p < 2; p++) {
            md.kind[p] = d->kind[p];
            md.delta_eps[p] = d->delta_eps[p];
            md.tau[p] = d->tau[p];
            md.omega_p[p] = d->omega_p[p];
            md.gamma[p] = d->gamma[p];
        }
        if (d->i <= g->nx && fdtd_b200_materials_set_component_dispersive(m, g, comp_of(d->comp), d->i, d->j, d->k, &md) != 0)
            return -1;
    }
    if (s->n_spheres) {
        fdtd_b200_sphere_t *sp = calloc(s->n_spheres, sizeof(*sp));
        fdtd_b200_dispersive_t *md = calloc(s->n_spheres, sizeof(*md));
        if (!sp || !md) { free(sp); free(md); return -1; }
        for (size_t q = 0; q < s->n_spheres; q++) {
            const scn_sphere_t *b = &s->spheres[q];
            sp[q].cx = b->cx; sp[q].cy = b->cy; sp[q].cz = b->cz; sp[q].radius = b->radius;
            sp[q].eps_r = b->eps_r; sp[q].sigma = b->sigma;
            if (b->disp >= 0) {
                const scn_disp_t *d = &s->disp[b->disp];
                md[q].eps_inf = d->eps_inf; md[q].sigma = d->sigma; md[q].n_poles = d->npoles;
                for (int p = 0; p < 2; p++) {
                    md[q].kind[p] = d->kind[p]; md[q].delta_eps[p] = d->delta_eps[p]; md[q].tau[p] = d->tau[p];
                    md[q].omega_p[p] = d->omega_p[p]; md[q].gamma[p] = d->gamma[p];
                }
                sp[q].model = &md[q];
            }
        }
        int rc = fdtd_b200_materials_add_spheres(m, g, sp, s->n_spheres, s->smoothing);
        free(sp);
        free(md);
        if (rc != 0) return -1;
    }
    for (size_t q = 0; q < s->n_tensor3; q++) {
        const scn_tensor3_t *t = &s->tensor3[q];
        /* the public setter takes lossless rows */
        if (t->sigma != 0.0) return -1;
        if (fdtd_b200_materials_set_component_tensor3(m, g, comp_of(t->comp), t->i, t->j, t->k, t->m) != 0) return -1;
    }
#else
    /* rfsyn has no 3x3 samples */
    if (s->n_tensor3) return -1;
    /* rfsyn has no dispersive media: dispersive samples enter rfsyn at their
     * static permittivity eps_inf + sum delta_eps */
    for (size_t q = 0; q < s->n_disp; q++) {
        const scn_disp_t *d = &s->disp[q];
        if (d->i > g->nx) continue;
        if (materials_set_component(m, g, comp_of(d->comp), d->i, d->j, d->k, static_eps(d), d->sigma) != 0) return -1;
    }
    if (s->n_spheres && ref_spheres(g, m, s) != 0) return -1;
#endif
    return 0;
}

typedef union {
    source_gaussian_deriv_params_t gd;
    source_ricker_params_t rk;
    source_modulated_gaussian_params_t mg;
} wave_params_t;

/* Returns 0 on success; probe_td: n_probes * n_steps (probe-major);
 * dft_re/dft_im: n_probes * n_freqs (may be NULL). */
int scn_run(const scn_scene_t *s, double *probe_td, double *dft_re, double *dft_im) {
    int rc = -1;
    if (s->n_planes) return -1; /* rfsyn's probes are single cells */
    fdtd_grid_t *g = fdtd_grid_create(s->nx, s->ny, s->nz, s->dx, s->courant);
    cpml_t *p = NULL;
    materials_t *m = NULL;
    source_t *src = NULL;
    wave_params_t *wp = NULL;
    probe_td_t *ptd = NULL;
    probe_dft_t *pdft = NULL;
    size_t made_td = 0, made_dft = 0;
    if (!g) return -1;
    if (fdtd_grid_set_periodic(g, s->periodic) != 0) goto out;
    if (s->npml) {
        cpml_params_t cp = {s->npml, s->m, s->ma, s->kappa_max, s->alpha_max, s->r0};
        p = cpml_create(g, cp);
        if (!p) goto out;
    }
    m = materials_create(g);
    if (!m || scn_setup(g, m, (void *)s) != 0) goto out;
    src = calloc(s->n_sources + 1, sizeof(*src));
    wp = calloc(s->n_sources + 1, sizeof(*wp));
    ptd = calloc(s->n_probes + 1, sizeof(*ptd));
    pdft = calloc(s->n_probes + 1, sizeof(*pdft));
    if (!src || !wp || !ptd || !pdft) goto out;
    for (size_t q = 0; q < s->n_sources; q++) {
        const scn_source_t *d = &s->sources[q];
        source_waveform_fn fn;
        if (d->waveform == 0) { wp[q].gd.t0 = d->p0; wp[q].gd.tau = d->p1; fn = source_waveform_gaussian_derivative; }
        else if (d->waveform == 1) { wp[q].rk.f0_hz = d->p0; wp[q].rk.t0 = d->p1; fn = source_waveform_ricker; }
        else { wp[q].mg.freq_hz = d->p0; wp[q].mg.t0 = d->p1; wp[q].mg.tau = d->p2; fn = source_waveform_modulated_gaussian; }
        src[q] = source_make_point(d->i, d->j, d->k, comp_of(d->comp), d->mode ? SRC_HARD : SRC_SOFT, d->amplitude, fn,
                                   &wp[q]);
    }
    for (size_t q = 0; q < s->n_probes; q++, made_td++)
        if (probe_td_create(&ptd[q], s->probes[q].i, s->probes[q].j, s->probes[q].k, comp_of(s->probes[q].comp),
                            s->n_steps) != 0)
            goto out;
    if (s->n_freqs)
        for (size_t q = 0; q < s->n_probes; q++, made_dft++)
            if (probe_dft_create(&pdft[q], s->probes[q].i, s->probes[q].j, s->probes[q].k, comp_of(s->probes[q].comp),
                                 s->freqs, s->n_freqs) != 0)
                goto out;
    for (size_t n = 0; n < s->n_steps; n++) {
        if (p) fdtd_update_h_cpml(g, p);
        else fdtd_update_h(g);
        double t = ((double)n + s->src_t_offset) * g->dt;
        for (size_t q = 0; q < s->n_sources; q++) source_apply(&src[q], g, t);
        if (p) fdtd_update_e_cpml_materials(g, p, m);
        else fdtd_update_e_materials(g, m);
        double td = ((double)n + s->dft_t_offset) * g->dt;
        for (size_t q = 0; q < s->n_probes; q++) {
            probe_td_record(&ptd[q], g);
            if (s->n_freqs) probe_dft_record(&pdft[q], g, td, g->dt);
        }
    }
    for (size_t q = 0; q < s->n_probes; q++) {
        if (probe_td) memcpy(probe_td + q * s->n_steps, ptd[q].buffer, s->n_steps * sizeof(double));
        if (s->n_freqs && dft_re && dft_im) {
            memcpy(dft_re + q * s->n_freqs, pdft[q].acc_re, s->n_freqs * sizeof(double));
            memcpy(dft_im + q * s->n_freqs, pdft[q].acc_im, s->n_freqs * sizeof(double));
        }
    }
    rc = 0;
out:
    for (size_t q = 0; q < made_td; q++) probe_td_destroy(&ptd[q]);
    for (size_t q = 0; q < made_dft; q++) probe_dft_destroy(&pdft[q]);
    free(src); free(wp); free(ptd); free(pdft);
    materials_destroy(m);
    cpml_destroy(p);
    fdtd_grid_destroy(g);
    return rc;
}

/* The full field state after a run, for element-wise comparisons: six arrays
 * of (nx+1)(ny+1)(nz+1) doubles (ex, ey, ez, hx, hy, hz).  initial (may be
 * NULL) seeds all six fields before the first step. */
int scn_run_fields(const scn_scene_t *s, const double *initial, double *fields_out) {
    int rc = -1;
    fdtd_grid_t *g = fdtd_grid_create(s->nx, s->ny, s->nz, s->dx, s->courant);
    cpml_t *p = NULL;
    materials_t *m = NULL;
    if (!g) return -1;
    size_t total = (s->nx + 1) * (s->ny + 1) * (s->nz + 1);
    double *f[6] = {g->ex, g->ey, g->ez, g->hx, g->hy, g->hz};
    if (fdtd_grid_set_periodic(g, s->periodic) != 0) goto out;
    if (s->npml) {
        cpml_params_t cp = {s->npml, s->m, s->ma, s->kappa_max, s->alpha_max, s->r0};
        p = cpml_create(g, cp);
        if (!p) goto out;
    }
    m = materials_create(g);
    if (!m || scn_setup(g, m, (void *)s) != 0) goto out;
    if (initial)
        for (int c = 0; c < 6; c++) memcpy(f[c], initial + c * total, total * sizeof(double));
    for (size_t n = 0; n < s->n_steps; n++) {
        if (p) fdtd_update_h_cpml(g, p);
        else fdtd_update_h(g);
        if (p) fdtd_update_e_cpml_materials(g, p, m);
        else fdtd_update_e_materials(g, m);
    }
    for (int c = 0; c < 6; c++) memcpy(fields_out + c * total, f[c], total * sizeof(double));
    rc = 0;
out:
    materials_destroy(m);
    cpml_destroy(p);
    fdtd_grid_destroy(g);
    return rc;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* A resident copy of the scene for timing rfsyn's loop (H, sources, E,
 * without probes): scn_bench_create builds it (grid, CPML, materials and the
 * first source) and returns the build's wall-clock seconds in *setup_s;
 * scn_bench_steps advances `steps` more steps and returns their wall-clock
 * seconds in *loop_s.  rfsyn allocates its fields and the twelve full-grid
 * psi arrays with calloc (engine/fdtd/grid.c, engine/fdtd/cpml.c:126-138),
 * so the first step over them pays the page faults of first touch: callers
 * run untimed warm-up steps before the timed ones. */
typedef struct {
    const scn_scene_t *s;
    fdtd_grid_t *g;
    cpml_t *p;
    materials_t *m;
    source_t src;
    source_modulated_gaussian_params_t mg;
    source_gaussian_deriv_params_t gd;
    size_t n;
} scn_bench_t;

void scn_bench_destroy(scn_bench_t *b) {
    if (!b) return;
    materials_destroy(b->m);
    cpml_destroy(b->p);
    fdtd_grid_destroy(b->g);
    free(b);
}

scn_bench_t *scn_bench_create(const scn_scene_t *s, double *setup_s) {
    double t0 = now_s();
    scn_bench_t *b = calloc(1, sizeof *b);
    if (!b) return NULL;
    b->s = s;
    b->g = fdtd_grid_create(s->nx, s->ny, s->nz, s->dx, s->courant);
    if (!b->g || fdtd_grid_set_periodic(b->g, s->periodic) != 0) goto fail;
    if (s->npml) {
        cpml_params_t cp = {s->npml, s->m, s->ma, s->kappa_max, s->alpha_max, s->r0};
        b->p = cpml_create(b->g, cp);
        if (!b->p) goto fail;
    }
    b->m = materials_create(b->g);
    if (!b->m || scn_setup(b->g, b->m, (void *)s) != 0) goto fail;
    if (s->n_sources) {
        const scn_source_t *d = &s->sources[0];
        if (d->waveform == 2) {
            b->mg.freq_hz = d->p0; b->mg.t0 = d->p1; b->mg.tau = d->p2;
            b->src = source_make_point(d->i, d->j, d->k, comp_of(d->comp), SRC_SOFT, d->amplitude,
                                       source_waveform_modulated_gaussian, &b->mg);
        } else {
            b->gd.t0 = d->p0; b->gd.tau = d->p1;
            b->src = source_make_point(d->i, d->j, d->k, comp_of(d->comp), SRC_SOFT, d->amplitude,
                                       source_waveform_gaussian_derivative, &b->gd);
        }
    }
    if (setup_s) *setup_s = now_s() - t0;
    return b;
fail:
    scn_bench_destroy(b);
    return NULL;
}

int scn_bench_steps(scn_bench_t *b, size_t steps, double *loop_s) {
    if (!b) return -1;
    double t0 = now_s();
    for (size_t q = 0; q < steps; q++, b->n++) {
        if (b->p) fdtd_update_h_cpml(b->g, b->p);
        else fdtd_update_h(b->g);
        if (b->s->n_sources) source_apply(&b->src, b->g, (double)b->n * b->g->dt);
        if (b->p) fdtd_update_e_cpml_materials(b->g, b->p, b->m);
        else fdtd_update_e_materials(b->g, b->m);
    }
    if (loop_s) *loop_s = now_s() - t0;
    return 0;
}
