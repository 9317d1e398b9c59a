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

#include "rfsyn_fdtd.h"
#include "scene.h"

static field_component_t comp_of(int c) { return (field_component_t)c; }

/* Applies boxes, then scalar overrides, then tensor edges (in list order). */
int scn_setup(const fdtd_grid_t *g, materials_t *m, void *ctx) {
    const scn_scene_t *s = (const scn_scene_t *)ctx;
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
