/* run.c -- the device time loop behind rfsyn's fdtd_simulate_echo*,
 * fdtd_stage_create and the extension API (fdtd_b200_*).
 *
 * rfsyn's loop (engine/fdtd/simulate.c:48-54) is, per step n:
 *   H update with CPML; source at t = n dt; E update with CPML + materials;
 *   probe record.
 * Here the whole loop runs on the GPU: the engine replays a CUDA graph of
 * the step kernels, sources are injected by the interface-list kernel and
 * probes are gathered on the device; only the time series comes back. */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "host.h"

static int g_prec = -1, g_sched = -1;

int rfb_default_precision(void) {
    if (g_prec < 0) {
        const char *v = getenv("RFSYN_FDTD_PRECISION");
        g_prec = (v && (!strcmp(v, "fp32") || !strcmp(v, "FP32"))) ? RFB_FP32 : RFB_FP64;
    }
    return g_prec;
}

int rfb_default_schedule(void) {
    if (g_sched < 0) {
        const char *v = getenv("RFSYN_FDTD_SCHEDULE");
        g_sched = (v && !strcmp(v, "split")) ? RFB_SCHED_SPLIT : RFB_SCHED_FUSED;
    }
    return g_sched;
}

int fdtd_b200_set_default_precision(int precision) {
    if (precision != FDTD_B200_FP64 && precision != FDTD_B200_FP32) return -1;
    g_prec = precision;
    return 0;
}

int fdtd_b200_set_default_schedule(int schedule) {
    if (schedule != FDTD_B200_SCHED_SPLIT && schedule != FDTD_B200_SCHED_FUSED) return -1;
    g_sched = schedule;
    return 0;
}

/* ---- fdtd.gpu.* settings ------------------------------------------------------
 * rfsyn's pipeline config keeps the FDTD stage's keys in its "fdtd" section
 * (cli/settings.c:6-33, read with config.c's typed getters); the GPU options
 * live beside them as "gpu.<name>" keys, which rfsyn's `config set
 * fdtd.gpu.<name> <value>` (cli/main.c:233-290) stores as text, a number or
 * a boolean.  These are the process-wide ones; the per-run ones (DFT bins,
 * batching, per-example scenes) are read by the job runner above the ABI. */
static char g_plan[96];
static int g_plan_set = 0;  /* 0: RFSYN_FDTD_PLAN decides; 1: g_plan ("" = autotune) */
static int g_tune = -1;     /* -1: RFSYN_FDTD_TUNE decides */

const char *rfb_plan_override(void) { return g_plan_set ? (g_plan[0] ? g_plan : NULL) : getenv("RFSYN_FDTD_PLAN"); }

int rfb_tune_enabled(void) {
    if (g_tune >= 0) return g_tune;
    const char *v = getenv("RFSYN_FDTD_TUNE");
    return !(v && !strcmp(v, "0"));
}

static const char *setting_name(const char *key) {
    if (!strncmp(key, "fdtd.", 5)) key += 5;
    if (!strncmp(key, "gpu.", 4)) key += 4;
    return key;
}

static int parse_flag(const char *v, int *out) {
    if (!strcmp(v, "1") || !strcmp(v, "true")) return *out = 1, 0;
    if (!strcmp(v, "0") || !strcmp(v, "false")) return *out = 0, 0;
    return -1;
}

/* 4 to 7 comma-separated integers >= 0, nothing else */
static int plan_text_ok(const char *v) {
    int n = 0;
    const char *p = v;
    while (*p) {
        if (*p < '0' || *p > '9') return 0;
        while (*p >= '0' && *p <= '9') p++;
        n++;
        if (*p == ',') {
            p++;
            if (!*p) return 0;
        } else if (*p) {
            return 0;
        }
    }
    return n >= 4 && n <= 7;
}

int fdtd_b200_apply_setting(const char *key, const char *value) {
    if (!key || !value) {
        rfb_set_error("NULL setting key or value");
        return -1;
    }
    const char *k = setting_name(key);
    int flag = 0;
    if (!strcmp(value, "default")) {
        /* back to the initial state: the environment variable decides */
        if (!strcmp(k, "precision")) return g_prec = -1, 0;
        if (!strcmp(k, "schedule")) return g_sched = -1, 0;
        if (!strcmp(k, "plan")) return g_plan_set = 0, 0;
        if (!strcmp(k, "tune")) return g_tune = -1, 0;
        if (!strcmp(k, "trace")) return rfb_set_trace(-1), 0;
    }
    if (!strcmp(k, "precision")) {
        if (!strcmp(value, "fp32") || !strcmp(value, "FP32")) return fdtd_b200_set_default_precision(FDTD_B200_FP32);
        if (!strcmp(value, "fp64") || !strcmp(value, "FP64")) return fdtd_b200_set_default_precision(FDTD_B200_FP64);
    } else if (!strcmp(k, "schedule")) {
        if (!strcmp(value, "fused")) return fdtd_b200_set_default_schedule(FDTD_B200_SCHED_FUSED);
        if (!strcmp(value, "split")) return fdtd_b200_set_default_schedule(FDTD_B200_SCHED_SPLIT);
    } else if (!strcmp(k, "plan")) {
        if (!strcmp(value, "auto")) {
            g_plan[0] = '\0';
            g_plan_set = 1;
            return 0;
        }
        if (strlen(value) < sizeof g_plan && plan_text_ok(value)) {
            strcpy(g_plan, value);
            g_plan_set = 1;
            return 0;
        }
    } else if (!strcmp(k, "tune")) {
        if (parse_flag(value, &flag) == 0) return g_tune = flag, 0;
    } else if (!strcmp(k, "trace")) {
        if (parse_flag(value, &flag) == 0) return rfb_set_trace(flag), 0;
    } else {
        rfb_set_error("unknown setting \"%s\"", key);
        return -1;
    }
    rfb_set_error("invalid value \"%s\" for setting \"%s\"", value, key);
    return -1;
}

int fdtd_b200_get_setting(const char *key, char *buf, size_t len) {
    if (!key || !buf || !len) {
        rfb_set_error("NULL setting key or buffer");
        return -1;
    }
    const char *k = setting_name(key);
    const char *v;
    if (!strcmp(k, "precision")) v = rfb_default_precision() == RFB_FP32 ? "fp32" : "fp64";
    else if (!strcmp(k, "schedule")) v = rfb_default_schedule() == RFB_SCHED_SPLIT ? "split" : "fused";
    else if (!strcmp(k, "plan")) v = rfb_plan_override() ? rfb_plan_override() : "auto";
    else if (!strcmp(k, "tune")) v = rfb_tune_enabled() ? "true" : "false";
    else if (!strcmp(k, "trace")) v = rfb_trace_enabled() ? "true" : "false";
    else {
        rfb_set_error("unknown setting \"%s\"", key);
        return -1;
    }
    if (strlen(v) + 1 > len) {
        rfb_set_error("buffer too short for setting \"%s\"", key);
        return -1;
    }
    strcpy(buf, v);
    return 0;
}

const char *fdtd_b200_last_error(void) { return rfb_last_error(); }
unsigned long long fdtd_b200_launch_count(void) { return rfb_launch_count(); }
unsigned long long fdtd_b200_cached_bytes(void) { return rfb_cached_bytes(); }
void fdtd_b200_release_cached_memory(void) { rfb_release_cached_memory(); }
const char *fdtd_b200_version(void) { return "rfsyn-b200 0.1 (sm_100a)"; }

void fdtd_b200_config_init(fdtd_b200_config_t *cfg, size_t nx, size_t ny, size_t nz, double dx, size_t n_steps,
                           size_t npml) {
    memset(cfg, 0, sizeof(*cfg));
    cfg->nx = nx;
    cfg->ny = ny;
    cfg->nz = nz;
    cfg->dx = dx;
    cfg->courant_safety = 0.99;
    cfg->n_steps = n_steps;
    cfg->cpml = cpml_default_params(npml);
    cfg->precision = FDTD_B200_FP64;
    cfg->schedule = FDTD_B200_SCHED_FUSED;
    cfg->source_time_offset_steps = 0.0;
    cfg->dft_time_offset_steps = 1.0;
}

struct fdtd_b200_sim {
    rfb_engine_t *eng;
    int borrowed;          /* a batch scene: the batch owns the engine */
    size_t n_steps, n_probes, n_freqs;
    double dt, dx;
    double *freqs;
    double dft_offset;
    size_t nx, ny, nz;
    int precision, schedule;
};

static double wave_value(const fdtd_b200_source_t *s, double t, size_t n) {
    switch (s->waveform) {
    case FDTD_B200_WAVE_GAUSSIAN_DERIV: {
        source_gaussian_deriv_params_t p = {s->p0, s->p1};
        return s->amplitude * source_waveform_gaussian_derivative(t, &p);
    }
    case FDTD_B200_WAVE_RICKER: {
        source_ricker_params_t p = {s->p0, s->p1};
        return s->amplitude * source_waveform_ricker(t, &p);
    }
    case FDTD_B200_WAVE_MOD_GAUSSIAN: {
        source_modulated_gaussian_params_t p = {s->p0, s->p1, s->p2};
        return s->amplitude * source_waveform_modulated_gaussian(t, &p);
    }
    default:
        return s->samples[n];
    }
}

/* amplitude * waveform(t) of a plane wave (waveforms 0..2 as for sources) */
double rfb_wave_value(int waveform, double amplitude, double p0, double p1, double p2, double t) {
    fdtd_b200_source_t s;
    memset(&s, 0, sizeof s);
    s.waveform = waveform;
    s.amplitude = amplitude;
    s.p0 = p0;
    s.p1 = p1;
    s.p2 = p2;
    return wave_value(&s, t, 0);
}

static size_t canon(size_t q, size_t n, int periodic) { return periodic ? q % n : q; }

/* member: create the engine as a scene of a batch (FUSED, on the batch's
 * stream, no plan of its own). */
static fdtd_b200_sim_t *sim_create(const fdtd_b200_config_t *cfg, fdtd_material_setup_fn setup, void *context,
                                   void *cuda_stream, int member) {
    fdtd_grid_t g;
    cpml_t *pml = NULL;
    materials_t *mat = NULL;
    rfb_scene_build_t scene;
    int have_scene = 0;
    double *vals = NULL;
    rfb_source_desc_t *sd = NULL;
    rfb_extra_cell_t *extra = NULL;
    rfb_probe_desc_t *pd = NULL;
    fdtd_b200_sim_t *sim = NULL;
    rfb_tfsf_build_t tf;
    int32_t *tf_first = NULL, *tf_count = NULL;
    memset(&tf, 0, sizeof tf);

    if (!cfg) { rfb_set_error("NULL config"); return NULL; }
    if (cfg->n_steps == 0) { rfb_set_error("n_steps must be positive"); return NULL; }
    if (cfg->precision != FDTD_B200_FP64 && cfg->precision != FDTD_B200_FP32) {
        rfb_set_error("unknown precision %d", cfg->precision);
        return NULL;
    }
    if (rfb_grid_geometry(&g, cfg->nx, cfg->ny, cfg->nz, cfg->dx, cfg->courant_safety) != 0) {
        rfb_set_error("invalid grid geometry");
        return NULL;
    }
    if (cfg->nx > 60000 || cfg->ny > 60000 || cfg->nz > 60000) {
        rfb_set_error("grid axis longer than 60000 cells");
        return NULL;
    }
    if (fdtd_grid_set_periodic(&g, cfg->periodic_axes) != 0) {
        rfb_set_error("invalid periodic axes");
        return NULL;
    }
    const int px = g.periodic_axes & 1u, py = g.periodic_axes & 2u, pz = g.periodic_axes & 4u;
    if (cfg->cpml.npml > 0) {
        pml = cpml_create(&g, cfg->cpml);
        if (!pml) { rfb_set_error("invalid CPML parameters for this grid"); return NULL; }
    }
    mat = materials_create(&g);
    if (!mat) { rfb_set_error("materials_create failed"); goto fail; }
    double t_phase = rfb_now();
    if (setup && setup(&g, mat, context) != 0) { rfb_set_error("scene setup callback failed"); goto fail; }
    rfb_trace("create: setup callback", t_phase);

    const size_t ns = cfg->n_sources, np = cfg->n_probes, nt = cfg->n_steps;
    if (cfg->plane_wave) {
        if (member) {
            rfb_set_error("a plane wave is not supported in a batch scene");
            goto fail;
        }
        t_phase = rfb_now();
        if (rfb_tfsf_build(&g, mat, cfg->plane_wave, nt, pml ? (int)cfg->cpml.npml : 0, &tf) != 0) goto fail;
        rfb_trace("create: plane wave", t_phase);
    }
    if (ns || tf.n_cells) {
        vals = malloc((ns ? ns : 1) * nt * sizeof(double));
        sd = calloc(ns ? ns : 1, sizeof(*sd));
        extra = calloc(ns + tf.n_cells, sizeof(*extra));
        if (!vals || !sd || !extra) { rfb_set_error("out of host memory"); goto fail; }
    }
    for (size_t q = 0; q < tf.n_cells; q++) {
        /* cells next to the plane-wave boundary: on the interface list */
        extra[ns + q].i = tf.cells[3 * q];
        extra[ns + q].j = tf.cells[3 * q + 1];
        extra[ns + q].k = tf.cells[3 * q + 2];
        extra[ns + q].component = -1;
        extra[ns + q].slot = -1;
    }
    for (size_t s = 0; s < ns; s++) {
        const fdtd_b200_source_t *src = &cfg->sources[s];
        if (src->i > g.nx || src->j > g.ny || src->k > g.nz) { rfb_set_error("source %zu outside the grid", s); goto fail; }
        if (src->component > FIELD_EZ) { rfb_set_error("source %zu drives a non-E component", s); goto fail; }
        if (src->waveform == FDTD_B200_WAVE_SAMPLES && !src->samples) { rfb_set_error("source %zu has no samples", s); goto fail; }
        if (src->waveform < 0 || src->waveform > FDTD_B200_WAVE_SAMPLES) { rfb_set_error("source %zu: unknown waveform", s); goto fail; }
        for (size_t n = 0; n < nt; n++) {
            double t = ((double)n + cfg->source_time_offset_steps) * g.dt;
            vals[s * nt + n] = wave_value(src, t, n);
        }
        sd[s].i = (int)canon(src->i, g.nx, px);
        sd[s].j = (int)canon(src->j, g.ny, py);
        sd[s].k = (int)canon(src->k, g.nz, pz);
        sd[s].component = (int)src->component;
        sd[s].hard = src->mode == SRC_HARD;
        sd[s].values = vals + s * nt;
        extra[s].i = sd[s].i;
        extra[s].j = sd[s].j;
        extra[s].k = sd[s].k;
        extra[s].component = sd[s].component;
        extra[s].slot = (int)s;
    }
    if (np) {
        pd = calloc(np, sizeof(*pd));
        if (!pd) { rfb_set_error("out of host memory"); goto fail; }
    }
    for (size_t q = 0; q < np; q++) {
        const fdtd_b200_probe_t *p = &cfg->probes[q];
        if (p->i > g.nx || p->j > g.ny || p->k > g.nz) { rfb_set_error("probe %zu outside the grid", q); goto fail; }
        if (p->component > FIELD_HZ) { rfb_set_error("probe %zu: unknown component", q); goto fail; }
        pd[q].i = (int)canon(p->i, g.nx, px);
        pd[q].j = (int)canon(p->j, g.ny, py);
        pd[q].k = (int)canon(p->k, g.nz, pz);
        pd[q].component = (int)p->component;
    }
    t_phase = rfb_now();
    if (materials_build_image(mat, &g, ns + tf.n_cells, extra, &scene) != 0) goto fail;
    have_scene = 1;
    rfb_trace("create: scene image", t_phase);
    t_phase = rfb_now();
    if (cfg->plane_wave) {
        /* E corrections per list entry: find each E target's cell */
        const size_t ne = 3 * scene.img.n_cells;
        tf_first = malloc((ne + 1) * sizeof(int32_t));
        tf_count = calloc(ne + 1, sizeof(int32_t));
        if (!tf_first || !tf_count) { rfb_set_error("out of host memory"); goto fail; }
        for (size_t e = 0; e < ne; e++) tf_first[e] = -1;
        const size_t nz1 = g.nz + 1, ny1 = g.ny + 1;
        for (size_t q = 0; q < tf.n_e; q++) {
            const size_t key = ((size_t)tf.e_ijkc[4 * q] * ny1 + (size_t)tf.e_ijkc[4 * q + 1]) * nz1 +
                               (size_t)tf.e_ijkc[4 * q + 2];
            size_t lo = 0, hi = scene.img.n_cells;
            while (lo < hi) {
                const size_t mid = (lo + hi) / 2;
                const int32_t *c = scene.img.cell_ijk + 3 * mid;
                const size_t km = ((size_t)c[0] * ny1 + (size_t)c[1]) * nz1 + (size_t)c[2];
                if (km < key) lo = mid + 1;
                else hi = mid;
            }
            const int32_t *hit = scene.img.cell_ijk + 3 * lo;
            if (lo == scene.img.n_cells || hit[0] != tf.e_ijkc[4 * q] || hit[1] != tf.e_ijkc[4 * q + 1] ||
                hit[2] != tf.e_ijkc[4 * q + 2]) {
                rfb_set_error("plane wave: a boundary sample is not on the list");
                goto fail;
            }
            const size_t e = 3 * lo + (size_t)tf.e_ijkc[4 * q + 3];
            if (scene.img.kind[e] != RFB_LK_SCALAR) {
                rfb_set_error("plane wave: the boundary must lie in scalar media");
                goto fail;
            }
            tf_first[e] = tf.e_first[q];
            tf_count[e] = tf.e_count[q];
        }
        rfb_trace("create: plane-wave targets", t_phase);
    }

    sim = calloc(1, sizeof(*sim));
    if (!sim) { rfb_set_error("out of host memory"); goto fail; }
    sim->n_steps = nt;
    sim->n_probes = np;
    sim->dt = g.dt;
    sim->dx = g.dx;
    sim->nx = g.nx; sim->ny = g.ny; sim->nz = g.nz;
    sim->dft_offset = cfg->dft_time_offset_steps;
    sim->precision = cfg->precision;
    sim->schedule = cfg->schedule;
    sim->n_freqs = cfg->n_freqs;
    if (cfg->n_freqs) {
        if (!cfg->freqs_hz) { rfb_set_error("n_freqs without freqs_hz"); goto fail; }
        sim->freqs = malloc(cfg->n_freqs * sizeof(double));
        if (!sim->freqs) { rfb_set_error("out of host memory"); goto fail; }
        memcpy(sim->freqs, cfg->freqs_hz, cfg->n_freqs * sizeof(double));
    }
    rfb_geom_t geom;
    rfb_geom_from_grid(&g, &geom);
    rfb_cpml_desc_t cd;
    if (pml) rfb_cpml_desc_from(pml, &cd);
    if (member) {
        sim->schedule = FDTD_B200_SCHED_FUSED;
        sim->borrowed = 1;
        sim->eng = rfb_engine_create_member(&geom, cfg->precision, pml ? &cd : NULL, &scene.img, ns, sd, np, pd, nt,
                                            cuda_stream);
    } else {
        sim->eng = rfb_engine_create(&geom, cfg->precision, cfg->schedule, pml ? &cd : NULL, &scene.img, ns, sd, np,
                                     pd, nt, cuda_stream);
    }
    if (!sim->eng) goto fail;
    rfb_trace("create: engine", t_phase);
    if (cfg->n_planes) {
        if (member) { rfb_set_error("plane probes are not supported in batches"); goto fail; }
        if (!cfg->planes) { rfb_set_error("n_planes without planes"); goto fail; }
        int *aic = malloc(3 * cfg->n_planes * sizeof(int));
        if (!aic) { rfb_set_error("out of host memory"); goto fail; }
        for (size_t q = 0; q < cfg->n_planes; q++) {
            aic[3 * q] = cfg->planes[q].axis;
            aic[3 * q + 1] = cfg->planes[q].index > (size_t)INT32_MAX ? -1 : (int)cfg->planes[q].index;
            aic[3 * q + 2] = (int)cfg->planes[q].component;
        }
        const int prc = rfb_engine_set_planes(sim->eng, cfg->n_planes, aic);
        free(aic);
        if (prc != 0) goto fail;
        sim->n_probes += cfg->n_planes;
    }
    /* the probe spectra accumulate with the steps (sessions; a batch's
     * scenes transform their stored series when read) */
    if (!member && cfg->n_freqs &&
        rfb_engine_set_dft(sim->eng, cfg->n_freqs, cfg->freqs_hz, cfg->dft_time_offset_steps) != 0)
        goto fail;
    if (cfg->plane_wave) {
        rfb_tfsf_desc_t td;
        memset(&td, 0, sizeof td);
        td.m_len = tf.m_len;
        td.ce = tf.ce;
        td.ch = tf.ch;
        td.src = tf.src;
        td.n_h = tf.n_h;
        td.h_ijkc = tf.h_ijkc;
        td.h_first = tf.h_first;
        td.h_count = tf.h_count;
        td.n_hterms = tf.n_hterms;
        td.n_eterms = tf.n_eterms;
        td.h_coef = tf.h_coef; td.h_w = tf.h_w; td.h_idx = tf.h_idx;
        td.e_coef = tf.e_coef; td.e_w = tf.e_w; td.e_idx = tf.e_idx;
        td.entry_first = tf_first;
        td.entry_count = tf_count;
        if (rfb_engine_set_tfsf(sim->eng, &td) != 0) {
            rfb_engine_destroy(sim->eng);
            sim->eng = NULL;
            goto fail;
        }
    }
    rfb_tfsf_free(&tf);
    free(tf_first);
    free(tf_count);
    rfb_scene_build_free(&scene);
    free(vals); free(sd); free(extra); free(pd);
    materials_destroy(mat);
    cpml_destroy(pml);
    return sim;
fail:
    if (sim) {
        free(sim->freqs);
        free(sim);
    }
    if (have_scene) rfb_scene_build_free(&scene);
    rfb_tfsf_free(&tf);
    free(tf_first);
    free(tf_count);
    free(vals); free(sd); free(extra); free(pd);
    materials_destroy(mat);
    cpml_destroy(pml);
    return NULL;
}

fdtd_b200_sim_t *fdtd_b200_sim_create(const fdtd_b200_config_t *cfg, fdtd_material_setup_fn setup, void *context,
                                      void *cuda_stream) {
    return sim_create(cfg, setup, context, cuda_stream, 0);
}

void fdtd_b200_sim_destroy(fdtd_b200_sim_t *sim) {
    if (!sim) return;
    if (!sim->borrowed) rfb_engine_destroy(sim->eng);
    free(sim->freqs);
    free(sim);
}

int fdtd_b200_sim_reset(fdtd_b200_sim_t *sim) { return sim ? rfb_engine_reset(sim->eng) : -1; }
int fdtd_b200_sim_advance(fdtd_b200_sim_t *sim, size_t n) { return sim ? rfb_engine_advance(sim->eng, n) : -1; }
int fdtd_b200_sim_advance_timed(fdtd_b200_sim_t *sim, size_t n, double *ms) {
    return sim ? rfb_engine_advance_timed(sim->eng, n, ms) : -1;
}
int fdtd_b200_sim_synchronize(fdtd_b200_sim_t *sim) { return sim ? rfb_engine_sync(sim->eng) : -1; }
size_t fdtd_b200_sim_steps_done(const fdtd_b200_sim_t *sim) { return sim ? rfb_engine_steps_done(sim->eng) : 0; }
void *fdtd_b200_sim_stream(const fdtd_b200_sim_t *sim) { return sim ? rfb_engine_stream(sim->eng) : NULL; }
int fdtd_b200_sim_launches_per_step(const fdtd_b200_sim_t *sim) {
    return sim ? rfb_engine_launches_per_step(sim->eng) : 0;
}

int fdtd_b200_sim_info(const fdtd_b200_sim_t *sim, fdtd_b200_sim_info_t *info) {
    if (!sim || !info) return -1;
    rfb_engine_info_t ei;
    if (rfb_engine_info(sim->eng, &ei) != 0) return -1;
    info->cells = sim->nx * sim->ny * sim->nz;
    info->list_cells = ei.list_cells;
    info->dispersive = ei.dispersive;
    info->slab_cell_axes = ei.slab_cell_axes;
    info->h2d_bytes = ei.h2d_bytes;
    info->precision = sim->precision;
    info->schedule = sim->schedule;
    info->tile_j = ei.tile_j;
    info->seg_len = ei.seg_len;
    info->ring_depth = ei.ring_depth;
    info->tma = ei.tma;
    info->unified = ei.unified;
    info->interior_items = ei.interior_items;
    info->edge_items = ei.edge_items;
    info->interior_ring2 = ei.interior_ring2;
    info->seg_edge = ei.seg_edge;
    return 0;
}

int fdtd_b200_sim_time_kernels(fdtd_b200_sim_t *sim, size_t n, double *sweep_ms, double *other_ms) {
    if (!sim || !sweep_ms || !other_ms) return -1;
    return rfb_engine_time_kernels(sim->eng, n, sweep_ms, other_ms);
}

int fdtd_b200_sim_energy(fdtd_b200_sim_t *sim, int x_lo, int x_hi, fdtd_b200_energy_t *out) {
    if (!sim || !out) return -1;
    double q[RFB_EN_COUNT];
    if (rfb_engine_energy(sim->eng, sim->dt, sim->dx, x_lo, x_hi, q) != 0) return -1;
    out->electric_j = q[RFB_EN_E];
    out->magnetic_j = q[RFB_EN_H];
    out->total_j = q[RFB_EN_E] + q[RFB_EN_H];
    out->interior_j = q[RFB_EN_E_INT] + q[RFB_EN_H_INT];
    out->electric_prev_j = q[RFB_EN_E_PREV];
    out->cross_j = q[RFB_EN_CROSS];
    out->modified_prev_j = q[RFB_EN_E_PREV] + q[RFB_EN_CROSS];
    out->max_abs_e = q[RFB_EN_MAX_E];
    out->max_abs_h = q[RFB_EN_MAX_H];
    out->nonfinite = (size_t)q[RFB_EN_NONFINITE];
    return 0;
}

int fdtd_b200_sim_read_probes(fdtd_b200_sim_t *sim, double *probe_td) {
    if (!sim || !probe_td) return -1;
    return rfb_engine_read_probes(sim->eng, probe_td);
}

int fdtd_b200_sim_read_iq(fdtd_b200_sim_t *sim, size_t probe, const fdtd_b200_awgn_t *awgn, float *iq_out) {
    if (!sim || !iq_out) {
        rfb_set_error("read_iq: NULL argument");
        return -1;
    }
    /* awgn.c:28: snr_linear from the float snr_db, in double */
    const double snr_linear = awgn ? pow(10.0, (double)awgn->snr_db / 10.0) : 0.0;
    return rfb_engine_read_iq(sim->eng, (int)probe, awgn != NULL, snr_linear, awgn ? awgn->seed : 0,
                              awgn ? awgn->stream : 0, iq_out);
}

int fdtd_b200_iq_write(const char *path, const float *iq, size_t n_samples) {
    if (!path || (n_samples && !iq)) return -1;
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    const size_t written = n_samples ? fwrite(iq, 2 * sizeof(float), n_samples, f) : 0;
    const int closed = fclose(f);
    return (written == n_samples && closed == 0) ? 0 : -1;
}

int fdtd_b200_sim_dft(fdtd_b200_sim_t *sim, double *re, double *im) {
    if (!sim || !re || !im) return -1;
    return rfb_engine_probe_dft(sim->eng, sim->n_freqs, sim->freqs, sim->dft_offset, re, im);
}

int fdtd_b200_sim_read_field(fdtd_b200_sim_t *sim, field_component_t c, double *host) {
    if (!sim || !host || c > FIELD_HZ) return -1;
    return rfb_engine_read_field(sim->eng, (int)c, host);
}

int fdtd_b200_run(const fdtd_b200_config_t *cfg, fdtd_material_setup_fn setup, void *context,
                  fdtd_b200_result_t *result) {
    if (!result) { rfb_set_error("NULL result"); return -1; }
    double t_phase = rfb_now();
    fdtd_b200_sim_t *sim = fdtd_b200_sim_create(cfg, setup, context, NULL);
    rfb_trace("run: create", t_phase);
    if (!sim) return -1;
    int rc = -1;
    double ms = 0.0;
    t_phase = rfb_now();
    if (rfb_engine_advance_timed(sim->eng, cfg->n_steps, &ms) != 0) goto out;
    rfb_trace("run: time loop", t_phase);
    t_phase = rfb_now();
    if (result->probe_td && rfb_engine_read_probes(sim->eng, result->probe_td) != 0) goto out;
    if (result->dft_re && result->dft_im && sim->n_freqs &&
        rfb_engine_probe_dft(sim->eng, sim->n_freqs, sim->freqs, sim->dft_offset, result->dft_re, result->dft_im) != 0)
        goto out;
    rfb_trace("run: series + spectra", t_phase);
    result->sample_rate_hz = 1.0 / sim->dt;
    result->device_ms = ms;
    rc = 0;
out:
    t_phase = rfb_now();
    fdtd_b200_sim_destroy(sim);
    rfb_trace("run: destroy", t_phase);
    return rc;
}

/* ---- rfsyn's entry points --------------------------------------------------- */

int fdtd_simulate_echo_with_setup(const fdtd_sim_config_t *cfg, double *out_td, double *sample_rate_out,
                                  fdtd_material_setup_fn setup, void *context) {
    if (!cfg || !out_td) return -1;
    if (cfg->n_steps == 0) return -1;
    fdtd_grid_t g;
    if (rfb_grid_geometry(&g, cfg->nx, cfg->ny, cfg->nz, cfg->dx, cfg->courant_safety) != 0) return -1;
    if (cfg->src_i > g.nx || cfg->src_j > g.ny || cfg->src_k > g.nz || cfg->probe_i > g.nx ||
        cfg->probe_j > g.ny || cfg->probe_k > g.nz)
        return -1;
    fdtd_b200_config_t b;
    fdtd_b200_config_init(&b, cfg->nx, cfg->ny, cfg->nz, cfg->dx, cfg->n_steps, cfg->npml);
    b.courant_safety = cfg->courant_safety;
    b.cpml = cpml_default_params(cfg->npml);
    b.precision = rfb_default_precision();
    b.schedule = rfb_default_schedule();
    /* simulate.c:37-38: soft Gaussian-derivative source, amplitude 1, t = n dt;
     * a non-E source component is ignored, as rfsyn's source_apply does */
    fdtd_b200_source_t src;
    memset(&src, 0, sizeof src);
    src.i = cfg->src_i; src.j = cfg->src_j; src.k = cfg->src_k;
    src.component = cfg->src_component;
    src.mode = SRC_SOFT;
    src.amplitude = 1.0;
    src.waveform = FDTD_B200_WAVE_GAUSSIAN_DERIV;
    src.p0 = cfg->t0_over_dt * g.dt;
    src.p1 = cfg->tau_over_dt * g.dt;
    b.n_sources = (cfg->src_component <= FIELD_EZ) ? 1 : 0;
    b.sources = &src;
    b.source_time_offset_steps = 0.0;
    fdtd_b200_probe_t probe = {cfg->probe_i, cfg->probe_j, cfg->probe_k, cfg->probe_component};
    int valid_probe = cfg->probe_component <= FIELD_HZ;
    b.n_probes = valid_probe ? 1 : 0;
    b.probes = &probe;
    fdtd_b200_result_t r;
    memset(&r, 0, sizeof r);
    r.probe_td = valid_probe ? out_td : NULL;
    if (!valid_probe) memset(out_td, 0, cfg->n_steps * sizeof(double));
    if (fdtd_b200_run(&b, setup, context, &r) != 0) return -1;
    if (sample_rate_out) *sample_rate_out = 1.0 / g.dt;
    return 0;
}

int fdtd_simulate_echo(const fdtd_sim_config_t *cfg, double *out_td, double *sample_rate_out) {
    return fdtd_simulate_echo_with_setup(cfg, out_td, sample_rate_out, NULL, NULL);
}

/* ---- the stage (cli/fdtd_stage.c:10-41) and its signal type ------------------ */

typedef struct {
    fdtd_sim_config_t cfg;
} stage_ctx_t;

static int stage_apply(void *ctx_v, signal_t *sig) {
    stage_ctx_t *ctx = (stage_ctx_t *)ctx_v;
    if (!ctx || !sig) return -1;
    if (signal_resize(sig, ctx->cfg.n_steps) != 0) return -1;
    double *buf = malloc(ctx->cfg.n_steps * sizeof(double));
    if (!buf) return -1;
    double fs = 0.0;
    if (fdtd_simulate_echo(&ctx->cfg, buf, &fs) != 0) {
        free(buf);
        return -1;
    }
    for (size_t n = 0; n < sig->n_samples; n++) sig->samples[n] = (float)buf[n];
    free(buf);
    sig->sample_rate_hz = fs;
    return 0;
}

static void stage_destroy(void *ctx) { free(ctx); }

transform_t fdtd_stage_create(const fdtd_sim_config_t *cfg) {
    transform_t none = {NULL, NULL, NULL};
    if (!cfg) return none;
    stage_ctx_t *ctx = malloc(sizeof(*ctx));
    if (!ctx) return none;
    ctx->cfg = *cfg;
    transform_t t = {stage_apply, stage_destroy, ctx};
    return t;
}

signal_t *signal_create(size_t n_samples, double sample_rate_hz, double center_freq_hz) {
    if (n_samples > SIZE_MAX / sizeof(rfsyn_float_complex)) return NULL;
    signal_t *sig = calloc(1, sizeof(*sig));
    if (!sig) return NULL;
    sig->samples = calloc(n_samples, sizeof(rfsyn_float_complex));
    if (!sig->samples && n_samples > 0) {
        free(sig);
        return NULL;
    }
    sig->n_samples = n_samples;
    sig->sample_rate_hz = sample_rate_hz;
    sig->center_freq_hz = center_freq_hz;
    return sig;
}

void signal_destroy(signal_t *sig) {
    if (!sig) return;
    free(sig->samples);
    if (sig->metadata && sig->meta_free) sig->meta_free(sig->metadata);
    free(sig);
}

int signal_resize(signal_t *sig, size_t n) {
    if (!sig) return -1;
    if (n > SIZE_MAX / sizeof(rfsyn_float_complex)) return -1;
    rfsyn_float_complex *grown = realloc(sig->samples, n * sizeof(rfsyn_float_complex));
    if (!grown && n > 0) return -1;
    if (n > sig->n_samples) memset(grown + sig->n_samples, 0, (n - sig->n_samples) * sizeof(rfsyn_float_complex));
    sig->samples = grown;
    sig->n_samples = n;
    return 0;
}

signal_t *signal_copy(const signal_t *sig) {
    if (!sig) return NULL;
    signal_t *c = signal_create(sig->n_samples, sig->sample_rate_hz, sig->center_freq_hz);
    if (!c) return NULL;
    memcpy(c->samples, sig->samples, sig->n_samples * sizeof(rfsyn_float_complex));
    c->metadata = sig->metadata;
    return c;
}

/* ---- batches of independent scenes ------------------------------------------ */
/* Member scenes are built by a few host threads: each scene's set-up
 * callback, material maps, interface list and device buffers are its own,
 * and the engine's shared state (memory cache, launch counter, fill-fraction
 * scratch) is locked or atomic.  The error reported is the one of the
 * lowest-numbered scene that failed, as a sequential loop would report:
 * scenes are taken in increasing order, so every lower scene was tried. */
typedef struct {
    const fdtd_b200_config_t *configs;
    const fdtd_material_setup_fn *setups;
    void *const *contexts;
    void *stream;
    fdtd_b200_sim_t **sims;
    size_t n;
    atomic_size_t next;
    atomic_int failed;
    size_t fail_at;
    char msg[480];
    pthread_mutex_t mu;
} member_job_t;

static void *member_worker(void *arg) {
    member_job_t *j = (member_job_t *)arg;
    while (!atomic_load(&j->failed)) {
        const size_t s = atomic_fetch_add(&j->next, 1);
        if (s >= j->n) break;
        fdtd_material_setup_fn fn = j->setups ? j->setups[s] : NULL;
        void *ctx = j->contexts ? j->contexts[s] : NULL;
        j->sims[s] = sim_create(&j->configs[s], fn, ctx, j->stream, 1);
        if (!j->sims[s]) {
            pthread_mutex_lock(&j->mu);
            if (!atomic_load(&j->failed) || s < j->fail_at) {
                j->fail_at = s;
                snprintf(j->msg, sizeof j->msg, "batch scene %zu: %s", s, rfb_last_error());
            }
            atomic_store(&j->failed, 1);
            pthread_mutex_unlock(&j->mu);
        }
    }
    return NULL;
}

/* Threads for member creation: RFSYN_FDTD_CREATE_THREADS, else the online
 * cores up to 16, never more than the scenes. */
static size_t member_threads(size_t n) {
    long t = 0;
    const char *v = getenv("RFSYN_FDTD_CREATE_THREADS");
    if (v && *v) t = strtol(v, NULL, 10);
    if (t <= 0) {
        t = sysconf(_SC_NPROCESSORS_ONLN);
        if (t > 16) t = 16;
    }
    if (t < 1) t = 1;
    return (size_t)t < n ? (size_t)t : n;
}

static int create_members(member_job_t *j) {
    pthread_t th[64];
    size_t nt = member_threads(j->n);
    if (nt > 64) nt = 64;
    size_t started = 0;
    for (size_t q = 1; q < nt; q++) {
        if (pthread_create(&th[q], NULL, member_worker, j) != 0) break;
        started = q;
    }
    member_worker(j);  /* the calling thread works too */
    for (size_t q = 1; q <= started; q++) pthread_join(th[q], NULL);
    return atomic_load(&j->failed) ? -1 : 0;
}

struct fdtd_b200_batch {
    rfb_batch_t *b;
    size_t n;
    fdtd_b200_sim_t **sims;   /* per scene: its configuration; engines owned by b */
};

fdtd_b200_batch_t *fdtd_b200_batch_create(size_t n_scenes, const fdtd_b200_config_t *configs,
                                          const fdtd_material_setup_fn *setups, void *const *contexts,
                                          void *cuda_stream) {
    fdtd_b200_batch_t *bt = NULL;
    rfb_engine_t **engs = NULL;
    void *stream = cuda_stream;
    int own = 0;
    size_t made = 0;
    if (!configs || n_scenes == 0) {
        rfb_set_error("a batch needs at least one scene configuration");
        return NULL;
    }
    for (size_t s = 0; s < n_scenes; s++) {
        if (configs[s].precision != configs[0].precision || configs[s].n_steps != configs[0].n_steps) {
            rfb_set_error("batch scene %zu: every scene must share precision and step count", s);
            return NULL;
        }
    }
    if (!stream) {
        stream = rfb_stream_create();
        if (!stream) return NULL;
        own = 1;
    }
    bt = calloc(1, sizeof(*bt));
    engs = calloc(n_scenes, sizeof(*engs));
    if (bt) bt->sims = calloc(n_scenes, sizeof(*bt->sims));
    if (!bt || !engs || !bt->sims) {
        rfb_set_error("out of host memory");
        goto fail;
    }
    bt->n = n_scenes;
    const double t_members = rfb_now();
    {
        member_job_t job;
        memset(&job, 0, sizeof job);
        job.configs = configs;
        job.setups = setups;
        job.contexts = contexts;
        job.stream = stream;
        job.sims = bt->sims;
        job.n = n_scenes;
        atomic_init(&job.next, 0);
        atomic_init(&job.failed, 0);
        pthread_mutex_init(&job.mu, NULL);
        const int rc = create_members(&job);
        pthread_mutex_destroy(&job.mu);
        for (size_t s = 0; s < n_scenes; s++) engs[s] = bt->sims[s] ? bt->sims[s]->eng : NULL;
        made = n_scenes;  /* engines of the scenes that were made (NULL elsewhere) */
        if (rc != 0) {
            rfb_set_error("%s", job.msg);
            goto fail;
        }
    }
    rfb_trace("batch: member scenes", t_members);
    bt->b = rfb_batch_create(engs, n_scenes, stream, own);
    own = 0;      /* the batch owns the stream now, on failure too */
    made = 0;     /* ... and the engines */
    if (!bt->b) goto fail;
    free(engs);
    return bt;
fail:
    if (bt) {
        for (size_t s = 0; s < made; s++) rfb_engine_destroy(engs[s]);
        if (bt->sims)
            for (size_t s = 0; s < n_scenes; s++) fdtd_b200_sim_destroy(bt->sims[s]);
        free(bt->sims);
        free(bt);
    }
    free(engs);
    if (own) rfb_stream_destroy(stream);
    return NULL;
}

void fdtd_b200_batch_destroy(fdtd_b200_batch_t *bt) {
    if (!bt) return;
    rfb_batch_destroy(bt->b);
    for (size_t s = 0; s < bt->n; s++) fdtd_b200_sim_destroy(bt->sims[s]);
    free(bt->sims);
    free(bt);
}

size_t fdtd_b200_batch_size(const fdtd_b200_batch_t *bt) { return bt ? bt->n : 0; }
int fdtd_b200_batch_reset(fdtd_b200_batch_t *bt) { return bt ? rfb_batch_reset(bt->b) : -1; }
int fdtd_b200_batch_advance(fdtd_b200_batch_t *bt, size_t n) { return bt ? rfb_batch_advance(bt->b, n) : -1; }
int fdtd_b200_batch_advance_timed(fdtd_b200_batch_t *bt, size_t n, double *ms) {
    return bt ? rfb_batch_advance_timed(bt->b, n, ms) : -1;
}
int fdtd_b200_batch_synchronize(fdtd_b200_batch_t *bt) { return bt ? rfb_batch_sync(bt->b) : -1; }
size_t fdtd_b200_batch_steps_done(const fdtd_b200_batch_t *bt) { return bt ? rfb_batch_steps_done(bt->b) : 0; }
void *fdtd_b200_batch_stream(const fdtd_b200_batch_t *bt) { return bt ? rfb_batch_stream(bt->b) : NULL; }

int fdtd_b200_batch_time_kernels(fdtd_b200_batch_t *bt, size_t n, double *sweep_ms, double *other_ms) {
    if (!bt || !sweep_ms || !other_ms) return -1;
    return rfb_batch_time_kernels(bt->b, n, sweep_ms, other_ms);
}

int fdtd_b200_batch_read_probes(fdtd_b200_batch_t *bt, size_t scene, double *probe_td) {
    if (!bt || scene >= bt->n || !probe_td) {
        rfb_set_error("batch: bad scene index or output");
        return -1;
    }
    if (rfb_batch_sync(bt->b) != 0) return -1;
    return rfb_engine_read_probes(bt->sims[scene]->eng, probe_td);
}

int fdtd_b200_batch_read_iq(fdtd_b200_batch_t *bt, size_t scene, size_t probe, const fdtd_b200_awgn_t *awgn,
                            float *iq_out) {
    if (!bt || scene >= bt->n || !iq_out) {
        rfb_set_error("batch: bad scene index or output");
        return -1;
    }
    if (rfb_batch_sync(bt->b) != 0) return -1;
    return fdtd_b200_sim_read_iq(bt->sims[scene], probe, awgn, iq_out);
}

int fdtd_b200_batch_dft(fdtd_b200_batch_t *bt, size_t scene, double *re, double *im) {
    if (!bt || scene >= bt->n || !re || !im) {
        rfb_set_error("batch: bad scene index or output");
        return -1;
    }
    if (rfb_batch_sync(bt->b) != 0) return -1;
    fdtd_b200_sim_t *sim = bt->sims[scene];
    return rfb_engine_probe_dft(sim->eng, sim->n_freqs, sim->freqs, sim->dft_offset, re, im);
}

int fdtd_b200_batch_info(const fdtd_b200_batch_t *bt, fdtd_b200_batch_info_t *info) {
    if (!bt || !info) return -1;
    rfb_batch_info_t bi;
    if (rfb_batch_info(bt->b, &bi) != 0) return -1;
    info->scenes = bi.scenes;
    info->cells = bi.cells;
    info->list_cells = bi.list_cells;
    info->slab_cell_axes = bi.slab_cell_axes;
    info->tile_j = bi.tile_j;
    info->ring_depth = bi.ring_depth;
    info->mode = bi.mode;
    info->seg_interior = bi.seg_interior;
    info->seg_edge = bi.seg_edge;
    info->items_interior = bi.items_interior;
    info->items_xslab = bi.items_xslab;
    info->items_edge = bi.items_edge;
    info->launches_per_step = bi.launches_per_step;
    info->unified = bi.unified;
    return 0;
}
