/*
 * rfsyn_fdtd_b200.h -- extensions of the B200 FDTD stage beyond rfsyn's ABI.
 *
 * rfsyn's fdtd_simulate_echo (engine/fdtd/simulate.c:10-69) fixes one
 * Gaussian-derivative source, one time-domain probe, the default CPML
 * parameters and FP64.  The run configuration below lifts those limits
 * (several sources and probes, probe DFTs, chosen waveform and CPML
 * parameters, periodic axes, FP32 or FP64) and a session object keeps a
 * scene resident on the GPU across repeated runs.  Every entry point returns
 * 0 / a valid pointer on success and -1 / NULL on failure, with the reason
 * in fdtd_b200_last_error().
 */
#ifndef RFSYN_FDTD_B200_H
#define RFSYN_FDTD_B200_H

#include "rfsyn_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { FDTD_B200_FP64 = 0, FDTD_B200_FP32 = 1 } fdtd_b200_precision_t;

/* SPLIT: separate H and E kernels (fields updated in place).
 * FUSED: one H+E march per step over ping-pong buffers. */
typedef enum { FDTD_B200_SCHED_SPLIT = 0, FDTD_B200_SCHED_FUSED = 1 } fdtd_b200_schedule_t;

typedef enum {
    FDTD_B200_WAVE_GAUSSIAN_DERIV = 0, /* p0 = t0, p1 = tau (s): source.c:8-13       */
    FDTD_B200_WAVE_RICKER = 1,         /* p0 = f0 (Hz), p1 = t0 (s): source.c:15-20  */
    FDTD_B200_WAVE_MOD_GAUSSIAN = 2,   /* p0 = f (Hz), p1 = t0, p2 = tau: source.c:21-26 */
    FDTD_B200_WAVE_SAMPLES = 3         /* samples[n] used as is (already scaled)     */
} fdtd_b200_waveform_t;

typedef struct {
    size_t i, j, k;
    field_component_t component;   /* FIELD_EX..FIELD_EZ */
    source_mode_t mode;
    double amplitude;
    int waveform;                  /* fdtd_b200_waveform_t */
    double p0, p1, p2;
    const double *samples;         /* n_steps values for FDTD_B200_WAVE_SAMPLES */
} fdtd_b200_source_t;

typedef struct {
    size_t i, j, k;
    field_component_t component;   /* FIELD_EX..FIELD_HZ */
} fdtd_b200_probe_t;

typedef struct {
    size_t nx, ny, nz;
    double dx;
    double courant_safety;
    size_t n_steps;
    unsigned periodic_axes;        /* x=1, y=2, z=4 */
    cpml_params_t cpml;            /* cpml.npml == 0: no absorbing layer */
    int precision;                 /* fdtd_b200_precision_t */
    int schedule;                  /* fdtd_b200_schedule_t */
    size_t n_sources;
    const fdtd_b200_source_t *sources;
    /* Source value of step n is taken at t = (n + source_time_offset_steps) dt
     * and added after the H update, before the E update (simulate.c:48-54). */
    double source_time_offset_steps;
    size_t n_probes;
    const fdtd_b200_probe_t *probes;
    /* Probe DFT bins (shared by every probe).  Sample n (recorded after the
     * E update of step n) enters at t = (n + dft_time_offset_steps) dt. */
    size_t n_freqs;
    const double *freqs_hz;
    double dft_time_offset_steps;
} fdtd_b200_config_t;

/* Defaults: courant 0.99, cpml = cpml_default_params(npml), FP64, FUSED,
 * offsets 0 (source) and 1 (DFT). */
void fdtd_b200_config_init(fdtd_b200_config_t *cfg, size_t nx, size_t ny, size_t nz, double dx,
                           size_t n_steps, size_t npml);

typedef struct {
    double *probe_td;              /* n_probes * n_steps, probe-major, or NULL */
    double *dft_re, *dft_im;       /* n_probes * n_freqs, or NULL */
    double sample_rate_hz;         /* 1 / dt */
    double device_ms;              /* GPU time of the step loop (CUDA events) */
} fdtd_b200_result_t;

/* One complete run (upload, loop, download).  `setup` may be NULL. */
int fdtd_b200_run(const fdtd_b200_config_t *cfg, fdtd_material_setup_fn setup, void *context,
                  fdtd_b200_result_t *result);

/* ---- resident session ----------------------------------------------------- */
typedef struct fdtd_b200_sim fdtd_b200_sim_t;

/* Uploads the scene once.  cuda_stream: a cudaStream_t to run on, or NULL
 * for a private stream. */
fdtd_b200_sim_t *fdtd_b200_sim_create(const fdtd_b200_config_t *cfg, fdtd_material_setup_fn setup,
                                      void *context, void *cuda_stream);
void fdtd_b200_sim_destroy(fdtd_b200_sim_t *sim);
/* Zero fields / CPML state and rewind to step 0 (asynchronous). */
int fdtd_b200_sim_reset(fdtd_b200_sim_t *sim);
/* Enqueue n more steps (asynchronous; CUDA-graph replay). */
int fdtd_b200_sim_advance(fdtd_b200_sim_t *sim, size_t n_steps);
int fdtd_b200_sim_synchronize(fdtd_b200_sim_t *sim);
size_t fdtd_b200_sim_steps_done(const fdtd_b200_sim_t *sim);
void *fdtd_b200_sim_stream(const fdtd_b200_sim_t *sim);
/* n_probes * n_steps doubles, probe-major (blocking). */
int fdtd_b200_sim_read_probes(fdtd_b200_sim_t *sim, double *probe_td);
/* n_probes * n_freqs each, over the steps done so far (blocking). */
int fdtd_b200_sim_dft(fdtd_b200_sim_t *sim, double *dft_re, double *dft_im);
/* One field component in rfsyn's padded layout, (nx+1)(ny+1)(nz+1) doubles. */
int fdtd_b200_sim_read_field(fdtd_b200_sim_t *sim, field_component_t component, double *host);
/* Kernels launched per time step by this session. */
int fdtd_b200_sim_launches_per_step(const fdtd_b200_sim_t *sim);

/* ---- process-wide settings and diagnostics ---------------------------------- */
/* Precision / schedule used by rfsyn's own entry points (fdtd_simulate_echo,
 * fdtd_stage_create).  Initial values: FP64 and FUSED, or the environment
 * variables RFSYN_FDTD_PRECISION=fp32|fp64 and RFSYN_FDTD_SCHEDULE=split|fused. */
int fdtd_b200_set_default_precision(int precision);
int fdtd_b200_set_default_schedule(int schedule);
const char *fdtd_b200_last_error(void);
/* Kernel launches issued by this process through the library. */
unsigned long long fdtd_b200_launch_count(void);
/* Library version string. */
const char *fdtd_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RFSYN_FDTD_B200_H */
