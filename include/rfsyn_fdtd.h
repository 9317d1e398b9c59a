/*
 * rfsyn_fdtd.h -- reference-compatible C ABI of the B200 FDTD stage.
 *
 * Every type and function below keeps the exact layout, signature, argument
 * meaning and error convention of the rfsyn declaration it replaces (cited
 * per item as reference-project file:line), so code written against rfsyn's
 * engine/fdtd and cli/fdtd_stage headers links against librfsyn_fdtd_b200.so
 * unchanged.  The numerics run on the GPU (sm_100a); the host side only keeps
 * the scene description and the caller-visible field arrays.
 *
 * Field-array contract of the step-wise update functions
 * (fdtd_update_h/e, fdtd_update_h/e_cpml, fdtd_update_e[_cpml]_materials):
 * the six double arrays of an fdtd_grid_t stay authoritative on the host,
 * exactly as in rfsyn: callers may read or write them between calls.  Each
 * call uploads the fields it reads, runs the update kernel on the GPU and
 * writes the updated components back before returning.
 *
 * CPML memory: the psi recursions live in device memory, stored only over the
 * absorbing slabs.  The psi_* pointers of struct cpml are kept for layout
 * compatibility and are NULL in this implementation; the profile arrays
 * (kappa_inv_*, b_*, a_*) are valid host arrays with rfsyn's values.
 */
#ifndef RFSYN_FDTD_H
#define RFSYN_FDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#include <complex>
extern "C" {
typedef std::complex<float> rfsyn_float_complex;
#else
#include <complex.h>
typedef float complex rfsyn_float_complex;
#endif

/* ---- physical constants: engine/core/constants.h:4-6 ------------------- */
#define C0    299792458.0
#define EPS0  8.8541878128e-12
#define MU0   1.25663706212e-6

/* ---- engine/fdtd/field_component.h:4-7 --------------------------------- */
typedef enum {
    FIELD_EX, FIELD_EY, FIELD_EZ,
    FIELD_HX, FIELD_HY, FIELD_HZ
} field_component_t;

/* ---- grid: engine/fdtd/grid.h:6-33 -------------------------------------- */
typedef struct {
    size_t nx, ny, nz;
    double dx;
    double dt;
    unsigned periodic_axes;
    double *ex, *ey, *ez;
    double *hx, *hy, *hz;
} fdtd_grid_t;

/* engine/fdtd/grid.h:15 -- NULL on invalid sizes/dx/safety factor. */
fdtd_grid_t *fdtd_grid_create(size_t nx, size_t ny, size_t nz, double dx,
                              double courant_safety_factor);
/* engine/fdtd/grid.h:17 -- bits x=1, y=2, z=4; -1 on NULL or stray bits. */
int fdtd_grid_set_periodic(fdtd_grid_t *g, unsigned axes);
/* engine/fdtd/grid.h:19 */
void fdtd_grid_destroy(fdtd_grid_t *g);

/* engine/fdtd/grid.h:21-23 */
static inline size_t grid_previous(size_t q, size_t extent) {
    return q == 0 ? extent - 1 : q - 1;
}

/* engine/fdtd/grid.h:25-30 -- padded (nx+1)(ny+1)(nz+1) layout, k fastest,
 * periodic axes wrapped by modulo. */
static inline size_t fdtd_index(const fdtd_grid_t *g, size_t i, size_t j, size_t k) {
    if (g->periodic_axes & 1u) i %= g->nx;
    if (g->periodic_axes & 2u) j %= g->ny;
    if (g->periodic_axes & 4u) k %= g->nz;
    return (i * (g->ny + 1) + j) * (g->nz + 1) + k;
}

/* engine/fdtd/grid.h:32-33 -- vacuum Yee sweeps (GPU). */
void fdtd_update_h(fdtd_grid_t *g);
void fdtd_update_e(fdtd_grid_t *g);

/* ---- CPML: engine/fdtd/cpml.h:7-51 -------------------------------------- */
struct cpml {
    size_t npml;
    double dx;

    double *kappa_inv_m_x, *b_m_x, *a_m_x;
    double *kappa_inv_m_y, *b_m_y, *a_m_y;
    double *kappa_inv_m_z, *b_m_z, *a_m_z;

    double *kappa_inv_h_x, *b_h_x, *a_h_x;
    double *kappa_inv_h_y, *b_h_y, *a_h_y;
    double *kappa_inv_h_z, *b_h_z, *a_h_z;

    /* Device-resident in this implementation (see header comment): NULL. */
    double *psi_hx_y, *psi_hx_z;
    double *psi_hy_z, *psi_hy_x;
    double *psi_hz_x, *psi_hz_y;
    double *psi_ex_y, *psi_ex_z;
    double *psi_ey_z, *psi_ey_x;
    double *psi_ez_x, *psi_ez_y;
};

typedef struct cpml cpml_t;

typedef struct {
    size_t npml;
    double m;
    double ma;
    double kappa_max;
    double alpha_max;
    double r0;
} cpml_params_t;

/* engine/fdtd/cpml.h:38 -- m=3, ma=1, kappa_max=7, alpha_max=0.05, r0=1e-6. */
cpml_params_t cpml_default_params(size_t npml);
/* engine/fdtd/cpml.h:40 -- NULL on bad params or npml >= (n+1)/2 on an
 * absorbing axis. */
cpml_t *cpml_create(const fdtd_grid_t *g, cpml_params_t params);
/* engine/fdtd/cpml.h:41 */
void cpml_destroy(cpml_t *pml);
/* engine/fdtd/cpml.h:43-44 (GPU). */
void fdtd_update_h_cpml(fdtd_grid_t *g, cpml_t *pml);
void fdtd_update_e_cpml(fdtd_grid_t *g, cpml_t *pml);

/* engine/fdtd/cpml.h:46-51 -- one psi recursion step; returns the
 * stretched difference. */
static inline double cpml_term(double diff, double kappa_inv, double b, double a,
                               double dx, double *psi)
{
    *psi = b * (*psi) + a * diff;
    return diff * kappa_inv + dx * (*psi);
}

/* ---- materials: engine/fdtd/materials.h:10-36 --------------------------- */
typedef struct materials materials_t;
typedef uint8_t material_id_t;
typedef struct { double Ca, Cb; } material_coeff_t;

/* engine/fdtd/materials.h:14-15 -- id 0 is vacuum (eps_r 1, sigma 0). */
materials_t *materials_create(const fdtd_grid_t *g);
void materials_destroy(materials_t *mat);

/* engine/fdtd/materials.h:17 -- dedupes (eps_r, sigma); at most 256 entries;
 * rejects eps_r < 1, sigma < 0 and non-finite input. */
int materials_register(materials_t *mat, double eps_r, double sigma, material_id_t *id_out);

/* engine/fdtd/materials.h:19-20 -- half-open boxes; clears scalar and tensor
 * overrides inside the box; periodic ends are clipped. */
int materials_assign_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1,
                         size_t j0, size_t j1, size_t k0, size_t k1, material_id_t id);
int materials_set_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1,
                      size_t j0, size_t j1, size_t k0, size_t k1, double eps_r, double sigma);

/* engine/fdtd/materials.h:22-24 -- per-component scalar overrides. */
int materials_set_component(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                            size_t i, size_t j, size_t k, double eps_r, double sigma);
int materials_clear_component(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                              size_t i, size_t j, size_t k);
int materials_get_coefficients(const materials_t *mat, const fdtd_grid_t *g,
                               field_component_t component, size_t i, size_t j, size_t k,
                               material_coeff_t *out);

/* engine/fdtd/materials.h:26-27 (GPU). */
void fdtd_update_e_materials(fdtd_grid_t *g, const materials_t *mat);
void fdtd_update_e_cpml_materials(fdtd_grid_t *g, cpml_t *pml, const materials_t *mat);

/* engine/fdtd/materials.h:29-32 */
typedef struct {
    double m11, m12, m22;
    double scale; /* dt/(eps0*dx) */
} material_tensor_t;

/* engine/fdtd/materials.h:34-36 -- 2x2 inverse-permittivity tensor on Ex/Ey
 * (Ex: m11=xx, m22=yy; Ey: m11=yy, m22=xx).  get returns 1 when absent. */
int materials_set_component_tensor(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                   size_t i, size_t j, size_t k, double m11, double m12, double m22);
int materials_clear_component_tensor(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                     size_t i, size_t j, size_t k);
int materials_get_tensor(const materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                         size_t i, size_t j, size_t k, material_tensor_t *out);

/* ---- 2-D subpixel helpers: engine/fdtd/subpixel_te.h:4-71 --------------------
 * Set-up helpers rfsyn's tilted-interface validator calls directly
 * (engine/fdtd/validate_materials_tilted.c:163-241): the share of a sample's
 * dx x dy cell covered by a rotated rectangle, the covered share of an edge
 * segment, and arithmetic, harmonic and normal-aligned 2x2 tensor mixes of
 * two relative permittivities.  Same status codes, argument checks and
 * output conventions (outputs untouched on failure). */
typedef enum {
    SUBPIXEL_TE_OK = 0,
    SUBPIXEL_TE_INVALID_ARGUMENT = -1,
    SUBPIXEL_TE_NUMERIC_ERROR = -2
} subpixel_te_status_t;

typedef struct {
    double center_x, center_y;
    double size_u, size_v;   /* full side lengths along the rotated axes */
    double angle_rad;        /* rotation of the u axis from x */
} subpixel_te_rectangle_t;

/* subpixel_te.h:18-25 */
int subpixel_te_rectangle_fraction(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                   double dx, double dy, double *fraction_out);
/* subpixel_te.h:27-34: edge from the sample along +x (axis 1) or +y (2) */
int subpixel_te_rectangle_edge_fraction(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                        int edge_axis, double length, double *fraction_out);
/* subpixel_te.h:37-42: 1 / ((1-f)/eps_bg + f/eps_in) */
int subpixel_te_mix_epsilon_harmonic(double fraction, double eps_background, double eps_inside,
                                     double *epsilon_r_out);
/* subpixel_te.h:44-49: (1-f) eps_bg + f eps_in */
int subpixel_te_mix_epsilon(double fraction, double eps_background, double eps_inside, double *epsilon_r_out);
/* subpixel_te.h:51-61 */
int subpixel_te_rectangle_epsilon(const subpixel_te_rectangle_t *rectangle, double sample_x, double sample_y,
                                  double dx, double dy, double eps_background, double eps_inside,
                                  double *fraction_out, double *epsilon_r_out);
/* subpixel_te.h:63-71: inverse-permittivity tensor harmonic along the normal
 * at angle normal_rad, 1/arithmetic along the interface */
int subpixel_te_mix_epsilon_tensor(double fraction, double eps_background, double eps_inside, double normal_rad,
                                   double *minv_xx, double *minv_xy, double *minv_yy);

/* ---- sources: engine/fdtd/source.h:8-35 --------------------------------- */
typedef enum {
    SRC_SOFT,
    SRC_HARD
} source_mode_t;

typedef double (*source_waveform_fn)(double t, const void *params);

typedef struct {
    size_t i, j, k;
    field_component_t component;
    source_mode_t mode;
    double amplitude;
    source_waveform_fn waveform;
    const void *params;
} source_t;

typedef struct { double t0, tau; } source_gaussian_deriv_params_t;
double source_waveform_gaussian_derivative(double t, const void *params);

typedef struct { double f0_hz, t0; } source_ricker_params_t;
double source_waveform_ricker(double t, const void *params);

typedef struct { double freq_hz, t0, tau; } source_modulated_gaussian_params_t;
double source_waveform_modulated_gaussian(double t, const void *params);

source_t source_make_point(size_t i, size_t j, size_t k, field_component_t component,
                           source_mode_t mode, double amplitude,
                           source_waveform_fn waveform, const void *params);

/* engine/fdtd/source.h:35 -- adds (SOFT) or assigns (HARD) on the host
 * field array; the next update call carries it to the GPU. */
void source_apply(const source_t *src, fdtd_grid_t *g, double t);

/* ---- probes: engine/fdtd/probe.h:8-39 ----------------------------------- */
typedef struct {
    size_t i, j, k;
    field_component_t component;
    double *buffer;
    size_t n_steps;
    size_t next_index;
} probe_td_t;

int  probe_td_create(probe_td_t *probe, size_t i, size_t j, size_t k,
                     field_component_t component, size_t n_steps);
void probe_td_destroy(probe_td_t *probe);
void probe_td_record(probe_td_t *probe, const fdtd_grid_t *g);

typedef struct {
    size_t i, j, k;
    field_component_t component;

    const double *freqs_hz;
    size_t n_freqs;

    double *acc_re;
    double *acc_im;
} probe_dft_t;

int  probe_dft_create(probe_dft_t *probe, size_t i, size_t j, size_t k, field_component_t component,
                      const double *freqs_hz, size_t n_freqs);
void probe_dft_destroy(probe_dft_t *probe);
void probe_dft_record(probe_dft_t *probe, const fdtd_grid_t *g, double t, double dt);
void probe_dft_result(const probe_dft_t *probe, size_t f_idx, double *out_magnitude,
                      double *out_phase_rad);

/* ---- time loop: engine/fdtd/simulate.h:9-29 ----------------------------- */
typedef struct {
    size_t nx, ny, nz;
    double dx;
    double courant_safety;
    size_t n_steps;

    size_t npml;

    size_t src_i, src_j, src_k;
    field_component_t src_component;
    double t0_over_dt, tau_over_dt;

    size_t probe_i, probe_j, probe_k;
    field_component_t probe_component;
} fdtd_sim_config_t;

/* engine/fdtd/simulate.h:25 -- runs the whole loop on the GPU; -1 on NULL
 * cfg/out, n_steps 0, source/probe outside the padded grid, or any
 * allocation / CUDA failure (message via fdtd_b200_last_error()). */
int fdtd_simulate_echo(const fdtd_sim_config_t *cfg, double *out_td, double *sample_rate_out);

/* engine/fdtd/simulate.h:27 -- the callback edits the host-side scene
 * description (materials API) before the description is uploaded.  The
 * grid it receives carries the geometry (sizes, dx, dt, periodic bits); its
 * field pointers are NULL because the fields live on the GPU for the whole
 * run. */
typedef int (*fdtd_material_setup_fn)(const fdtd_grid_t *grid, materials_t *materials, void *context);

/* engine/fdtd/simulate.h:29 */
int fdtd_simulate_echo_with_setup(const fdtd_sim_config_t *cfg, double *out_td, double *sample_rate_out,
                                  fdtd_material_setup_fn setup, void *context);

/* ---- stage boundary types: engine/core/rf_signal.h:10-28,
 *      engine/core/transform.h:6-10 ----------------------------------------- */
typedef void *(*metadata_copy_fn)(const void *metadata);
typedef void  (*metadata_free_fn)(void *metadata);

typedef struct signal {
    rfsyn_float_complex *samples;
    size_t n_samples;
    double sample_rate_hz;
    double center_freq_hz;

    void *metadata;
    metadata_copy_fn meta_copy;
    metadata_free_fn meta_free;
} signal_t;

/* engine/core/rf_signal.h:21-27.  Exported with default visibility so a host
 * program that links rfsyn's own rf_signal.c interposes its definitions. */
signal_t *signal_create(size_t n_samples, double sample_rate_hz, double center_freq_hz);
void signal_destroy(signal_t *sig);
int signal_resize(signal_t *sig, size_t new_n_samples);
signal_t *signal_copy(const signal_t *sig);

typedef struct {
    int (*apply)(void *ctx, signal_t *sig);
    void (*destroy)(void *ctx);
    void *ctx;
} transform_t;

/* ---- the drop-in entry point: cli/fdtd_stage.h:7 ------------------------- */
/* Copies *cfg.  apply() resizes the signal to n_steps, runs the GPU loop and
 * writes (float)probe[n] + 0i with sample_rate_hz = 1/dt; -1 on failure.
 * {NULL, NULL, NULL} on NULL cfg or allocation failure. */
transform_t fdtd_stage_create(const fdtd_sim_config_t *cfg);

#ifdef __cplusplus
}
#endif

#endif /* RFSYN_FDTD_H */
