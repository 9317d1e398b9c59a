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

#include <stdint.h>

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

/* A plane wave injected by a total-field / scattered-field boundary (no
 * counterpart in rfsyn, whose validators drive soft sheets or modal lines,
 * engine/fdtd/validation_common.h:16-18).  Direction k = (sin t cos p,
 * sin t sin p, cos t) for theta t, phi p (radians); E along
 * cos(psi) theta_hat + sin(psi) phi_hat; amplitude * waveform(t) drives
 * the line's source (waveform and p0..p2 as for sources, samples not
 * allowed).  The total field fills the box of sample positions
 * [i0, i1] x [j0, j1] x [k0, k1] (cell units; the whole axis on a periodic
 * axis); the box grown by two cells must lie outside the CPML and inside
 * the grid, in scalar media.  The incident field comes from a 1-D FDTD line
 * along k with the grid's dt and spacing dx sqrt(sum_a k_a^4), which gives
 * it the grid's numerical phase velocity along k to second order in k dx,
 * read by cubic interpolation at each sample's projected distance (Taflove
 * & Hagness, Computational Electrodynamics 3rd ed., ch. 5).  At normal
 * incidence and along a body diagonal the injection is exact; at other
 * angles the scattered region sees about -60 dB of the incident peak at 17
 * cells per wavelength.  The line's source sits 8 line cells before the
 * first corner, so E there is the waveform delayed by that distance.  A
 * wave with a component of k along a periodic axis is rejected (no Floquet
 * boundaries). */
typedef struct {
    double theta, phi, psi;
    double amplitude;
    int waveform;                  /* fdtd_b200_waveform_t, not SAMPLES */
    double p0, p1, p2;
    size_t i0, i1, j0, j1, k0, k1;
} fdtd_b200_plane_wave_t;

/* A plane probe: every step, the mean of one field component over a whole
 * grid plane -- axis (0 = x, 1 = y, 2 = z) at cell index `index`, every
 * cell of the other two axes (u < n_u, v < n_v).  In a cell periodic across
 * the plane, at normal incidence, that mean is the amplitude of the
 * specular reflected or transmitted wave, so a plane probe's running DFT is
 * a reflection / transmission spectrum.  No counterpart in rfsyn (its
 * probes are single cells, engine/fdtd/probe.h:8-39). */
typedef struct {
    int axis;
    size_t index;
    field_component_t component;   /* FIELD_EX..FIELD_HZ */
} fdtd_b200_plane_probe_t;

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
     * E update of step n) enters at t = (n + dft_time_offset_steps) dt.  In
     * sessions the sums accumulate on the GPU as the steps run (FP64 runs:
     * FP64 sums with direct sincos, rfsyn's probe_dft_record arithmetic,
     * engine/fdtd/probe.c:78-92; FP32 runs: Kahan-compensated FP32 sums with
     * an FP64 phase recurrence); batches transform the stored series when
     * read. */
    size_t n_freqs;
    const double *freqs_hz;
    double dft_time_offset_steps;
    /* NULL, or a plane wave injected through a TF/SF boundary (sessions and
     * fdtd_b200_run; not in batches) */
    const fdtd_b200_plane_wave_t *plane_wave;
    /* Plane probes (sessions and fdtd_b200_run; not in batches): their
     * series and spectra follow the point probes', so every probe output
     * holds n_probes + n_planes series. */
    size_t n_planes;
    const fdtd_b200_plane_probe_t *planes;
} fdtd_b200_config_t;

/* Defaults: courant 0.99, cpml = cpml_default_params(npml), FP64, FUSED,
 * offsets 0 (source) and 1 (DFT). */
void fdtd_b200_config_init(fdtd_b200_config_t *cfg, size_t nx, size_t ny, size_t nz, double dx,
                           size_t n_steps, size_t npml);

typedef struct {
    double *probe_td;              /* (n_probes + n_planes) * n_steps, probe-major, or NULL */
    double *dft_re, *dft_im;       /* (n_probes + n_planes) * n_freqs, or NULL */
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
/* advance + synchronise; *ms = GPU time of the n steps, from CUDA events
 * recorded on the session stream around them. */
int fdtd_b200_sim_advance_timed(fdtd_b200_sim_t *sim, size_t n_steps, double *ms);
size_t fdtd_b200_sim_steps_done(const fdtd_b200_sim_t *sim);
void *fdtd_b200_sim_stream(const fdtd_b200_sim_t *sim);
/* (n_probes + n_planes) * n_steps doubles, probe-major (blocking). */
int fdtd_b200_sim_read_probes(fdtd_b200_sim_t *sim, double *probe_td);
/* (n_probes + n_planes) * n_freqs each, over the steps done so far (blocking). */
int fdtd_b200_sim_dft(fdtd_b200_sim_t *sim, double *dft_re, double *dft_im);

/* ---- the stage's output signal, AWGN and .iq files ---------------------------
 * rfsyn's CLI chain after the FDTD stage: the probe series becomes a complex
 * float signal (float)td[n] + 0i (cli/fdtd_stage.c:23-24), awgn_create(snr_db,
 * seed, stream) adds white Gaussian noise of per-axis deviation
 * sqrt(P / 10^(snr_db/10) / 2), P the mean power, drawn with rfsyn's PCG32
 * stream and Box-Muller pair per sample (engine/noise/awgn.c:16-44), and
 * write_signal stores the samples as interleaved float32 I/Q
 * (cli/main.c:70-85).  fdtd_b200_sim_read_iq computes the same samples on
 * the GPU from the resident probe series and returns 2 n_steps floats (I, Q
 * per sample); awgn NULL leaves the noise out.  fdtd_b200_iq_write writes n
 * samples to a file as write_signal does (0, or -1). */
typedef struct {
    float snr_db;
    uint64_t seed, stream;
} fdtd_b200_awgn_t;
int fdtd_b200_sim_read_iq(fdtd_b200_sim_t *sim, size_t probe, const fdtd_b200_awgn_t *awgn, float *iq_out);
int fdtd_b200_iq_write(const char *path, const float *iq, size_t n_samples);

/* ---- failure detection ----------------------------------------------------------
 * Every wait of the sweeps on a tensor copy is bounded (~2e9 SM cycles); a
 * copy that never completes makes the sweep record an error that the next
 * blocking call returns as -1 with its text.  This runs the same wait on an
 * mbarrier armed for a copy that is never issued, with the given limit
 * (cycles, at most 4e9): *timed_out = 1 and *cycles the time waited.  No
 * copy is in flight, so the device stays usable. */
int fdtd_b200_selftest_bounded_wait(long long limit_cycles, int *timed_out, long long *cycles);
/* One field component in rfsyn's padded layout, (nx+1)(ny+1)(nz+1) doubles. */
int fdtd_b200_sim_read_field(fdtd_b200_sim_t *sim, field_component_t component, double *host);
/* Kernels launched per time step by this session. */
int fdtd_b200_sim_launches_per_step(const fdtd_b200_sim_t *sim);

/* Shape of a session's device work, for roofline accounting. */
typedef struct {
    size_t cells;            /* nx * ny * nz */
    size_t list_cells;       /* cells on the interface list (overrides, tensors, dispersive, sources) */
    size_t dispersive;       /* dispersive (ADE) samples */
    size_t slab_cell_axes;   /* sum over cells of the CPML slab axes containing them */
    size_t h2d_bytes;        /* scene bytes uploaded at creation */
    int precision, schedule;
    int tile_j, seg_len;     /* fused sweep plan: rows per interior tile, planes per work item */
    int ring_depth;          /* planes staged per interior CTA */
    int tma;                 /* 1: interior planes staged by the Tensor Memory Accelerator */
    int interior_items;      /* work items of the interior sweep (CTAs per step) */
    int edge_items;          /* work items of the edge sweep */
    int unified;             /* 1: every sweep item in one work queue, one launch per step */
    int interior_ring2;      /* 0, or the ring depth of the interior sweep whose threads own two
                                rows of a 2 tile_j-row tile */
    int seg_edge;            /* planes per slab / boundary work item */
} fdtd_b200_sim_info_t;

int fdtd_b200_sim_info(const fdtd_b200_sim_t *sim, fdtd_b200_sim_info_t *info);

/* Runs n more steps launching each kernel separately (no graph) with CUDA
 * events around every launch; *sweep_ms = summed GPU time of the H/E sweep
 * kernel(s), *other_ms = the interface-list and probe kernels. */
int fdtd_b200_sim_time_kernels(fdtd_b200_sim_t *sim, size_t n_steps, double *sweep_ms, double *other_ms);

/* FP64 energy audit of the resident fields after `steps_done` = n steps
 * (replaces the host loops of validate_long_term_stability.c:166-209 and
 * audit_periodic_energy.c:43-71): sums over i < nx, j < ny, k < nz of
 * 0.5 eps E^2 and 0.5 mu0 H^2 times dx^3, eps = dt / (dx Cb) from each
 * component's scalar Cb (validate_long_term_stability.c:74-75).  FP64
 * accumulation whatever the field precision; deterministic.  interior_j
 * covers planes x_lo <= i < x_hi.  With the fused schedule the previous
 * step's fields are resident too: electric_prev_j is the energy of E^{n-1},
 * cross_j = 0.5 mu0 H^{n-3/2} . H^{n-1/2} dx^3, and modified_prev_j their sum,
 * the audit's modified energy at step n-1; NaN with the split schedule or
 * before the first step. */
typedef struct {
    double electric_j, magnetic_j, total_j, interior_j;
    double electric_prev_j, cross_j, modified_prev_j;
    double max_abs_e, max_abs_h;
    size_t nonfinite;
} fdtd_b200_energy_t;

int fdtd_b200_sim_energy(fdtd_b200_sim_t *sim, int x_lo, int x_hi, fdtd_b200_energy_t *out);

/* ---- batches of independent scenes ------------------------------------------
 * No counterpart in rfsyn, whose job loop simulates its examples one after
 * the other (cli/main.c:362-417).  A batch uploads many scenes -- each with
 * its own size, CPML, materials (setup callback), sources and probes, as for
 * fdtd_b200_sim_create -- and advances all of them together: every step is
 * five kernel launches for the whole batch (three work-queue sweeps over the
 * tiles of every scene, the interface lists, the probes), replayed from CUDA
 * graphs.  Every scene yields exactly the probe series and spectra of its own
 * session (the same kernels, the same arithmetic).  All scenes share the
 * precision and step count; the FUSED schedule is used whatever the
 * configuration says; a scene periodic in y or z whose tile halos would wrap
 * is rejected.  Creation times candidate tile plans on the batch
 * (RFSYN_FDTD_PLAN "rows,ring,seg_interior,seg_edge,mode" with mode 2 or 3
 * fixes one).  setups / contexts may be NULL, or hold NULL entries. */
typedef struct fdtd_b200_batch fdtd_b200_batch_t;

fdtd_b200_batch_t *fdtd_b200_batch_create(size_t n_scenes, const fdtd_b200_config_t *configs,
                                          const fdtd_material_setup_fn *setups, void *const *contexts,
                                          void *cuda_stream);
void fdtd_b200_batch_destroy(fdtd_b200_batch_t *batch);
size_t fdtd_b200_batch_size(const fdtd_b200_batch_t *batch);
int fdtd_b200_batch_reset(fdtd_b200_batch_t *batch);
int fdtd_b200_batch_advance(fdtd_b200_batch_t *batch, size_t n_steps);
int fdtd_b200_batch_advance_timed(fdtd_b200_batch_t *batch, size_t n_steps, double *ms);
int fdtd_b200_batch_synchronize(fdtd_b200_batch_t *batch);
size_t fdtd_b200_batch_steps_done(const fdtd_b200_batch_t *batch);
void *fdtd_b200_batch_stream(const fdtd_b200_batch_t *batch);
/* As fdtd_b200_sim_time_kernels, for the whole batch. */
int fdtd_b200_batch_time_kernels(fdtd_b200_batch_t *batch, size_t n_steps, double *sweep_ms, double *other_ms);
/* Probe series / spectra of one scene (blocking), as the session calls. */
int fdtd_b200_batch_read_probes(fdtd_b200_batch_t *batch, size_t scene, double *probe_td);
/* fdtd_b200_sim_read_iq for one scene of the batch (2 n_steps floats). */
int fdtd_b200_batch_read_iq(fdtd_b200_batch_t *batch, size_t scene, size_t probe, const fdtd_b200_awgn_t *awgn,
                            float *iq_out);
int fdtd_b200_batch_dft(fdtd_b200_batch_t *batch, size_t scene, double *dft_re, double *dft_im);

typedef struct {
    size_t scenes, cells, list_cells, slab_cell_axes;
    int tile_j, ring_depth;
    int mode;                    /* 2: tiles from the origin; 3: origins shifted to the slab edges;
                                    4: narrow tiles over the z slabs */
    int seg_interior, seg_edge;  /* planes per work item */
    int items_interior, items_xslab, items_edge;
    int launches_per_step;
    int unified;                 /* 1: every sweep item in one work queue, one launch per step */
} fdtd_b200_batch_info_t;

int fdtd_b200_batch_info(const fdtd_b200_batch_t *batch, fdtd_b200_batch_info_t *info);

/* ---- learned surrogate network -------------------------------------------------
 * No counterpart in rfsyn.  A multilayer perceptron trained and evaluated on
 * the GPU by this library's own kernels (BF16 tensor-core GEMMs with FP32
 * accumulation, fused bias / GELU epilogues, FP32 Adam master weights): the
 * network of the transfer-function surrogate (rfsyn_b200.surrogate), which
 * maps a scene's parameter vector to its tx -> rx transfer function.
 * Layers: n_in -> width (GELU), depth-1 times width -> width (GELU),
 * width -> n_out.  width and n_out are multiples of 64; the input is padded
 * with zeros to a multiple of 64.  Training batches are multiples of 64. */
typedef struct fdtd_b200_mlp fdtd_b200_mlp_t;

/* He-uniform initial weights from splitmix64(seed), zero biases. */
fdtd_b200_mlp_t *fdtd_b200_mlp_create(int n_in, int width, int depth, int n_out, uint64_t seed);
void fdtd_b200_mlp_destroy(fdtd_b200_mlp_t *mlp);
/* Parameters in layer order: W (out x in, row-major; the first layer's in is
 * the padded input width), then b. */
size_t fdtd_b200_mlp_n_params(const fdtd_b200_mlp_t *mlp);
int fdtd_b200_mlp_get_params(fdtd_b200_mlp_t *mlp, float *params);
int fdtd_b200_mlp_set_params(fdtd_b200_mlp_t *mlp, const float *params);
/* One forward + backward pass of a batch (X: batch x n_in, Y: batch x
 * n_out): mean squared error and its gradient in parameter layout. */
int fdtd_b200_mlp_grad(fdtd_b200_mlp_t *mlp, const float *X, const float *Y, int batch, double *loss,
                       float *grads);
/* Uploads the training set (kept on the device). */
int fdtd_b200_mlp_set_data(fdtd_b200_mlp_t *mlp, const float *X, const float *Y, size_t n);
/* `steps` Adam steps (betas, eps) of `batch` samples drawn through a
 * permutation reshuffled every pass (splitmix64(shuffle_seed)), learning
 * rate lr * 0.5 (1 + cos(pi s / steps)); each step replays one CUDA graph.
 * final_loss: mean squared error of the last batch. */
int fdtd_b200_mlp_train(fdtd_b200_mlp_t *mlp, size_t steps, int batch, double lr, double beta1, double beta2,
                        double eps, uint64_t shuffle_seed, double *final_loss);
/* Outputs of n inputs (n x n_out). */
int fdtd_b200_mlp_predict(fdtd_b200_mlp_t *mlp, const float *X, size_t n, float *Y);
unsigned long long fdtd_b200_mlp_launch_count(const fdtd_b200_mlp_t *mlp);
/* How many of those launches were products on the tcgen05 tensor cores
 * (accumulators in tensor memory).  The products run on mma.sync tiles of
 * 64 x 64, faster on this network's small products; with the environment
 * variable RFSYN_FDTD_MLP_GEMM=tcgen05 set when the network is created,
 * every product whose rows are a multiple of 128, columns of 32 and depth
 * of 64 runs on tcgen05 tiles of 128 x 32 instead. */
unsigned long long fdtd_b200_mlp_tensor_core_launches(const fdtd_b200_mlp_t *mlp);

/* ---- dispersive media (auxiliary differential equations) ----------------------
 * rfsyn models only static eps_r and sigma (engine/fdtd/materials.c:92-125);
 * these entry points add per-component dispersive samples integrated with
 * polarisation-current ADEs (Taflove & Hagness, Computational
 * Electrodynamics, 3rd ed., ch. 9):
 *   eps(w) = eps_inf + sum_p chi_p(w),   sigma static conductivity,
 *   Debye   chi_p = delta_eps_p / (1 + j w tau_p),
 *   Lorentz chi_p = delta_eps_p w_p^2 / (w_p^2 + 2 j w gamma_p - w^2).
 * A dispersive sample takes precedence over a scalar override of the same
 * component; a 2x2 tensor edge takes precedence over both; box assignment
 * clears dispersive samples inside the box, as it clears overrides. */
#define FDTD_B200_MAX_POLES 2
typedef enum { FDTD_B200_POLE_DEBYE = 0, FDTD_B200_POLE_LORENTZ = 1 } fdtd_b200_pole_kind_t;

typedef struct {
    double eps_inf;                          /* >= 1 */
    double sigma;                            /* >= 0, S/m */
    int n_poles;                             /* 1 .. FDTD_B200_MAX_POLES */
    int kind[FDTD_B200_MAX_POLES];           /* fdtd_b200_pole_kind_t */
    double delta_eps[FDTD_B200_MAX_POLES];   /* > 0 */
    double tau[FDTD_B200_MAX_POLES];         /* Debye relaxation time (s) */
    double omega_p[FDTD_B200_MAX_POLES];     /* Lorentz resonance (rad/s) */
    double gamma[FDTD_B200_MAX_POLES];       /* Lorentz damping (1/s) */
} fdtd_b200_dispersive_t;

int fdtd_b200_materials_set_component_dispersive(materials_t *mat, const fdtd_grid_t *g,
                                                 field_component_t component, size_t i, size_t j, size_t k,
                                                 const fdtd_b200_dispersive_t *model);
/* Every component of every cell of a half-open box gets the model. */
int fdtd_b200_materials_set_dispersive_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0,
                                           size_t j1, size_t k0, size_t k1, const fdtd_b200_dispersive_t *model);
int fdtd_b200_materials_clear_component_dispersive(materials_t *mat, const fdtd_grid_t *g,
                                                   field_component_t component, size_t i, size_t j, size_t k);

/* ---- full 3x3 anisotropic permittivity -----------------------------------------
 * rfsyn's tensor edges (materials_set_component_tensor, materials.c:658-903)
 * are 2x2 (Ex, Ey; a z-invariant TM scope).  These samples carry a full row
 * of the relative inverse permittivity m = eps_r^-1: component c of a cell
 * is updated as
 *   E_c += dt/(eps0 dx) (m_cc D_c + sum_{b != c} m_cb <D_b>),
 * D_b = (curl H)_b dx at the b sample, <D_b> its mean over the four b
 * samples surrounding the E_c sample (which keeps the coupling reciprocal
 * for a symmetric m).  Lossless as set here (spheres smoothed with smoothing 2
 * carry a loss, see below); for cells outside the CPML; on an axis
 * without wrap the cell lies in [1, n-1].  A 3x3 sample takes precedence
 * over every other description of the same component; box assignment clears
 * them.  set_component_tensor3 takes the row (3 values, m_cc > 0);
 * set_tensor3_box inverts a symmetric positive-definite eps_r (9 values,
 * row-major) and sets all three components of every cell of the box. */
int fdtd_b200_materials_set_component_tensor3(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                              size_t i, size_t j, size_t k, const double row[3]);
int fdtd_b200_materials_clear_component_tensor3(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                                size_t i, size_t j, size_t k);
int fdtd_b200_materials_set_tensor3_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0,
                                        size_t j1, size_t k0, size_t k1, const double eps_r[9]);
/* Every E sample (cell units: Ex of cell (i,j,k) at (i+1/2, j, k), ...)
 * within thickness / 2 of the plane through `point` with `normal`, and
 * admitted by the margin rule, gets the row of eps_r^-1 (a staircased
 * anisotropic slab). */
int fdtd_b200_materials_set_tensor3_slab(materials_t *mat, const fdtd_grid_t *g, const double point[3],
                                         const double normal[3], double thickness, const double eps_r[9]);
/* The same slab with its faces smoothed: samples whose unit cube lies inside
 * get the row of eps_r^-1 as above; samples whose cube a face may cut get,
 * when their fill fraction f (8^3 lattice) is positive, the row of the
 * smoothed inverse permittivity between the cell's table material and eps_r
 * along the normal (fdtd_b200_subpixel_tensor3, Kottke et al.'s average for
 * the anisotropic slab), with sigma (1 - f) sigma_table, built on the GPU in
 * FP64.  The margin rule applies. */
int fdtd_b200_materials_set_tensor3_slab_smoothed(materials_t *mat, const fdtd_grid_t *g, const double point[3],
                                                  const double normal[3], double thickness, const double eps_r[9]);
/* The row of a 3x3 sample: 0, or 1 when the component has none. */
int fdtd_b200_materials_get_tensor3(const materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                    size_t i, size_t j, size_t k, double row[3]);

/* ---- spheres with subpixel smoothing -------------------------------------------
 * Rasterises spheres (centre and radius in cell units: the E_x sample of cell
 * (i,j,k) sits at (i+1/2, j, k), E_y at (i, j+1/2, k), E_z at (i, j, k+1/2))
 * in list order, later spheres over earlier ones.  The fill fraction f of the
 * unit cube around every E sample near a surface is computed on the GPU in
 * FP64 (supersampled, 8^3 points).  A cell whose three samples are inside
 * takes the sphere's material id; a sample cut by the surface gets, by
 * `smoothing`:
 *   0  the inside material when f >= 1/2 (staircase);
 *   1  a scalar override with the diagonal of the smoothed inverse
 *      permittivity 1/eps_c = n_c^2 <1/eps> + (1 - n_c^2) / <eps>;
 *   2  the full row of the smoothed inverse permittivity as a 3x3 sample,
 *      M = <1/eps> n n^T + (1/<eps>) (I - n n^T) (fdtd_b200_subpixel_tensor3
 *      with two isotropic media), built on the GPU in FP64, off-diagonal
 *      terms included; where the 3x3 update cannot run (the margin rule of
 *      fdtd_b200_materials_set_component_tensor3) its diagonal as in 1;
 * with <.> weighted by f against the cell's table material, n the outward
 * surface normal at the sample, and sigma mixed by f (a lossy 3x3 sample
 * takes its loss at the component's permittivity 1/M_cc, as rfsyn's
 * make_coeff does for a scalar one).  Dispersive spheres (model != NULL) are
 * always staircased onto dispersive samples. */
typedef struct {
    double cx, cy, cz, radius;
    double eps_r, sigma;
    const fdtd_b200_dispersive_t *model;     /* NULL: plain dielectric */
} fdtd_b200_sphere_t;

int fdtd_b200_materials_add_spheres(materials_t *mat, const fdtd_grid_t *g, const fdtd_b200_sphere_t *spheres,
                                    size_t n_spheres, int smoothing);

/* ---- three-dimensional subpixel smoothing -------------------------------------
 * rfsyn's tensor mix (subpixel_te_mix_epsilon_tensor, engine/fdtd/
 * subpixel_te.c:106-132) is two-dimensional: an interface normal in the
 * (x, y) plane and isotropic media.  fdtd_b200_subpixel_tensor3 gives the
 * smoothed relative inverse permittivity M (9 values, row-major) of a cell of
 * which a share `fraction` holds eps_inside behind an interface of normal
 * `normal` (any length > 0), the rest eps_background; both permittivities are
 * symmetric positive-definite 3x3 matrices (row-major), so anisotropic media
 * are allowed.  It averages Kottke, Farjadpour and Johnson's tau transform of
 * eps in the frame of the normal (Phys. Rev. E 77, 036611, 2008), which for
 * two isotropic media is M = <1/eps> n n^T + (1/<eps>) (I - n n^T), rfsyn's
 * rule in three dimensions: with n in the (x, y) plane the (x, y) block of M
 * is rfsyn's (m_xx, m_xy, m_yy).  Returns SUBPIXEL_TE_OK, or
 * SUBPIXEL_TE_INVALID_ARGUMENT (NULL, fraction outside [0, 1], zero normal, a
 * permittivity that is not symmetric positive definite). */
int fdtd_b200_subpixel_tensor3(double fraction, const double eps_background[9], const double eps_inside[9],
                               const double normal[3], double minv_out[9]);

/* ---- heightmap world -----------------------------------------------------------
 * rfsyn's terrain description (engine/world/world.h:10-17, world.c:49-135):
 * column (i, j) is solid material column_materials[i ny + j] up to height
 * heights_m[i ny + j] (0 .. nz dx; air columns have height 0).  rfsyn loads
 * such worlds and a material catalog but never applies them to an FDTD grid
 * (cli/main.c:325-333).  This maps one onto the materials of a grid with the
 * same cells: media[id] gives eps_r and sigma of world material id (for
 * example rfsyn's material_catalog_evaluate at the simulation frequency).
 * Cells take world.c's bulk id (solid where the solid fraction is >= 1/2);
 * with smoothing, every E component of a cell cut by the surface gets the
 * diagonal of the smoothed inverse permittivity along the world's surface
 * normal, the rule fdtd_b200_materials_add_spheres uses.  Box assignment
 * semantics: the columns' earlier descriptions are replaced.  Returns 0 (and
 * the number of cut cells in *mixed_out) or -1 with fdtd_b200_last_error(),
 * rejecting what world_create_heightmap rejects. */
typedef struct {
    size_t nx, ny, nz;                 /* world cells: the grid's */
    double dx;                         /* the grid's */
    const double *heights_m;           /* nx * ny */
    const uint8_t *column_materials;   /* nx * ny world material ids */
    uint8_t air_id;
} fdtd_b200_heightmap_t;
typedef struct {
    double eps_r, sigma;
} fdtd_b200_medium_t;
int fdtd_b200_materials_apply_heightmap(materials_t *mat, const fdtd_grid_t *g, const fdtd_b200_heightmap_t *hm,
                                        const fdtd_b200_medium_t *media, size_t n_media, int smoothing,
                                        size_t *mixed_out);

/* ---- sphere fill fractions without device allocation --------------------------
 * No counterpart in rfsyn.  For callers that cannot allocate device memory
 * when they rasterise a sphere: a thread building scenes while another
 * thread of the process captures a CUDA graph (an allocation would break the
 * capture), a real-time loop that must not enter the allocator, or a process
 * whose device memory belongs to another framework's pool allocator.
 * Computes, for every cell of the box [i0, i0+ni) x [j0, j0+nj) x [k0, k0+nk),
 * the fill fraction f[3*cell + c] and squared normal component n2[3*cell + c]
 * of the three E samples, cell = ((i-i0)*nj + (j-j0))*nk + (k-k0), exactly as
 * fdtd_b200_materials_add_spheres does; f and n2 are host arrays of
 * 3*ni*nj*nk doubles.  Nothing is allocated: the device staging is a fixed
 * array of 2^20 samples per output (16 MiB in all) that the library keeps on
 * every GPU that loads it until the process exits; a box of more than 2^20
 * samples is rejected with -1.  The first call on a device sets that device
 * up (once): it looks the staging array up, which may load the part of the
 * library that holds it and so commit its 16 MiB at that moment (CUDA loads
 * a library's device code lazily by default; with CUDA_MODULE_LOADING=EAGER
 * in the environment the array is committed with the device's context
 * instead), and it creates the non-blocking stream the calls run on.  Make that first call at
 * start-up: before any stream capture, and before another framework's pool
 * takes the device's memory.  Later calls launch on that stream and copy back
 * with asynchronous copies on it, so they never wait on the legacy default
 * stream or on a stream another thread is capturing; for the duration of a
 * call the calling thread's capture mode is thread-local, so a capture
 * another thread runs in the global mode is not disturbed by it (the
 * caller's mode is restored on return).  Every call shares the
 * one array: calls that overlap on the GPU (from several host threads) race,
 * so serialise them. */
int fdtd_b200_sphere_fractions_noalloc(const double centre[3], double radius, int i0, int j0, int k0,
                                       int ni, int nj, int nk, double *f, double *n2);

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
/* Device memory blocks that destroyed simulations, stages and batches freed
 * (1 MB and more rounded to 2 MB, smaller ones to a power of two) are kept
 * by the library for the next creation (up to a
 * quarter of each device's memory; an allocation that fails empties the
 * cache first).  fdtd_b200_cached_bytes reports what is held;
 * fdtd_b200_release_cached_memory returns all of it to the driver. */
unsigned long long fdtd_b200_cached_bytes(void);
void fdtd_b200_release_cached_memory(void);

/* ---- fdtd.gpu.* settings ------------------------------------------------------
 * The config surface's GPU section.  rfsyn's pipeline config keeps the FDTD
 * stage's keys in its "fdtd" section (cli/settings.c:6-33); the GPU options
 * sit beside them as "gpu.<name>" (set with `config set fdtd.gpu.<name> v`,
 * cli/main.c:233-290).  key: "fdtd.gpu.<name>", "gpu.<name>" or "<name>";
 * value as text (a boolean as true/false or 1/0):
 *   precision  fp32 | fp64          default precision of rfsyn's entry points
 *   schedule   fused | split        default schedule of rfsyn's entry points
 *   plan       auto | tj,ns,seg_interior,seg_edge[,mode[,single_queue[,two_rows_ring]]]
 *                                   the sweep plan (auto = the autotuner)
 *   tune       true | false         false: the first tensor-copy variant, no tuning
 *   trace      true | false         per-phase host times on stderr
 * "default" restores a setting's initial state (its RFSYN_FDTD_* environment
 * variable decides).  Returns 0, or -1 with fdtd_b200_last_error() for an
 * unknown key or a value it does not accept (the setting is unchanged).
 * fdtd_b200_get_setting writes the current value as text. */
int fdtd_b200_apply_setting(const char *key, const char *value);
int fdtd_b200_get_setting(const char *key, char *buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* RFSYN_FDTD_B200_H */
