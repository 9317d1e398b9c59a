/* source_probe.c -- point sources, waveforms and host-side probes with
 * rfsyn's semantics (engine/fdtd/source.c:8-57, engine/fdtd/probe.c:21-105).
 * These act on the caller-visible host arrays of the step-wise API; the
 * device time loop evaluates the same waveforms once per step on the host
 * and injects / records on the GPU. */
#include <math.h>
#include <stdlib.h>

#include "host.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* -2u exp(-u^2), u = (t - t0)/tau */
double source_waveform_gaussian_derivative(double t, const void *params) {
    const source_gaussian_deriv_params_t *p = (const source_gaussian_deriv_params_t *)params;
    double u = (t - p->t0) / p->tau;
    return -2.0 * u * exp(-u * u);
}

/* (1 - 2a^2) exp(-a^2), a = pi f0 (t - t0) */
double source_waveform_ricker(double t, const void *params) {
    const source_ricker_params_t *p = (const source_ricker_params_t *)params;
    double a = M_PI * p->f0_hz * (t - p->t0);
    double a2 = a * a;
    return (1.0 - 2.0 * a2) * exp(-a2);
}

/* exp(-u^2) sin(2 pi f (t - t0)) */
double source_waveform_modulated_gaussian(double t, const void *params) {
    const source_modulated_gaussian_params_t *p = (const source_modulated_gaussian_params_t *)params;
    double u = (t - p->t0) / p->tau;
    double envelope = exp(-u * u);
    return envelope * sin(2.0 * M_PI * p->freq_hz * (t - p->t0));
}

source_t source_make_point(size_t i, size_t j, size_t k, field_component_t component, source_mode_t mode,
                           double amplitude, source_waveform_fn waveform, const void *params) {
    source_t s;
    s.i = i; s.j = j; s.k = k;
    s.component = component;
    s.mode = mode;
    s.amplitude = amplitude;
    s.waveform = waveform;
    s.params = params;
    return s;
}

void source_apply(const source_t *src, fdtd_grid_t *g, double t) {
    if (!src || !g || !src->waveform) return;
    if (src->i > g->nx || src->j > g->ny || src->k > g->nz) return;
    double *field;
    switch (src->component) {
    case FIELD_EX: field = g->ex; break;
    case FIELD_EY: field = g->ey; break;
    case FIELD_EZ: field = g->ez; break;
    default: return;
    }
    if (!field) return;
    double val = src->amplitude * src->waveform(t, src->params);
    size_t idx = fdtd_index(g, src->i, src->j, src->k);
    if (src->mode == SRC_SOFT) field[idx] += val;
    else field[idx] = val;
}

static const double *field_of(const fdtd_grid_t *g, field_component_t c) {
    switch (c) {
    case FIELD_EX: return g->ex;
    case FIELD_EY: return g->ey;
    case FIELD_EZ: return g->ez;
    case FIELD_HX: return g->hx;
    case FIELD_HY: return g->hy;
    case FIELD_HZ: return g->hz;
    default: return NULL;
    }
}

int probe_td_create(probe_td_t *probe, size_t i, size_t j, size_t k, field_component_t component, size_t n_steps) {
    if (!probe || n_steps == 0) return -1;
    probe->buffer = malloc(n_steps * sizeof(double));
    if (!probe->buffer) return -1;
    probe->i = i; probe->j = j; probe->k = k;
    probe->component = component;
    probe->n_steps = n_steps;
    probe->next_index = 0;
    return 0;
}

void probe_td_destroy(probe_td_t *probe) {
    if (!probe) return;
    free(probe->buffer);
    probe->buffer = NULL;
}

void probe_td_record(probe_td_t *probe, const fdtd_grid_t *g) {
    if (!probe || !g || !probe->buffer) return;
    if (probe->next_index >= probe->n_steps) return;
    const double *f = field_of(g, probe->component);
    if (!f) return;
    probe->buffer[probe->next_index++] = f[fdtd_index(g, probe->i, probe->j, probe->k)];
}

int probe_dft_create(probe_dft_t *probe, size_t i, size_t j, size_t k, field_component_t component,
                     const double *freqs_hz, size_t n_freqs) {
    if (!probe || !freqs_hz || n_freqs == 0) return -1;
    probe->acc_re = calloc(n_freqs, sizeof(double));
    probe->acc_im = calloc(n_freqs, sizeof(double));
    if (!probe->acc_re || !probe->acc_im) {
        free(probe->acc_re);
        free(probe->acc_im);
        return -1;
    }
    probe->i = i; probe->j = j; probe->k = k;
    probe->component = component;
    probe->freqs_hz = freqs_hz;
    probe->n_freqs = n_freqs;
    return 0;
}

void probe_dft_destroy(probe_dft_t *probe) {
    if (!probe) return;
    free(probe->acc_re);
    free(probe->acc_im);
    probe->acc_re = NULL;
    probe->acc_im = NULL;
}

/* Riemann-sum DFT: re += v cos(w t) dt, im -= v sin(w t) dt. */
void probe_dft_record(probe_dft_t *probe, const fdtd_grid_t *g, double t, double dt) {
    if (!probe || !g) return;
    const double *f = field_of(g, probe->component);
    if (!f) return;
    double v = f[fdtd_index(g, probe->i, probe->j, probe->k)];
    for (size_t q = 0; q < probe->n_freqs; q++) {
        double w = 2.0 * M_PI * probe->freqs_hz[q];
        probe->acc_re[q] += v * cos(w * t) * dt;
        probe->acc_im[q] -= v * sin(w * t) * dt;
    }
}

void probe_dft_result(const probe_dft_t *probe, size_t f_idx, double *out_magnitude, double *out_phase_rad) {
    if (!probe || f_idx >= probe->n_freqs) {
        if (out_magnitude) *out_magnitude = 0.0;
        if (out_phase_rad) *out_phase_rad = 0.0;
        return;
    }
    double re = probe->acc_re[f_idx], im = probe->acc_im[f_idx];
    if (out_magnitude) *out_magnitude = sqrt(re * re + im * im);
    if (out_phase_rad) *out_phase_rad = atan2(im, re);
}
