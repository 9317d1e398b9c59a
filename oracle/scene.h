/*
 * scene.h -- TEST INFRASTRUCTURE (oracle).  A flat, self-contained scene
 * description shared by
 *   - fdtd_oracle.c   : the CPU restatement of rfsyn's FDTD loop (FP64),
 *   - scene_driver.c  : a driver that replays the scene through rfsyn's public
 *                       C API, linked either against rfsyn itself (compiled
 *                       from its sources into oracle/_ref) or against
 *                       librfsyn_fdtd_b200.so (step-wise GPU path),
 * so one case runs identically on every implementation.  Never linked into
 * the product.
 *
 * Loop of one run (rfsyn engine/fdtd/simulate.c:48-54 generalised):
 *   for n in 0..n_steps-1:
 *     H update (CPML when npml > 0)
 *     every source applied at t = (n + src_t_offset) dt
 *     E update with materials (CPML when npml > 0)
 *     probes record; DFT accumulates at t = (n + dft_t_offset) dt
 */
#ifndef RFSYN_ORACLE_SCENE_H
#define RFSYN_ORACLE_SCENE_H

#include <stddef.h>

typedef struct { size_t i0, i1, j0, j1, k0, k1; double eps_r, sigma; } scn_box_t;
typedef struct { int comp; size_t i, j, k; double eps_r, sigma; } scn_comp_t;
typedef struct { int comp; size_t i, j, k; double m11, m12, m22; } scn_tensor_t;
/* full 3x3 sample (no rfsyn counterpart): row `comp` of the relative
 * inverse permittivity */
typedef struct { int comp; size_t i, j, k; double m[3]; double sigma; } scn_tensor3_t;
/* waveform: 0 Gaussian derivative (p0 t0, p1 tau), 1 Ricker (p0 f0, p1 t0),
 *           2 modulated Gaussian (p0 f, p1 t0, p2 tau).  mode 0 soft, 1 hard. */
typedef struct { size_t i, j, k; int comp, mode; double amplitude; int waveform; double p0, p1, p2; } scn_source_t;
typedef struct { size_t i, j, k; int comp; } scn_probe_t;
/* mean of component comp over the whole plane axis = index (cells u < n_u, v < n_v) */
typedef struct { int axis; size_t index; int comp; } scn_plane_t;
/* dispersive sample (no rfsyn counterpart): kind 0 Debye (tau), 1 Lorentz
 * (omega_p, gamma) per pole */
typedef struct {
    int comp; size_t i, j, k;
    double eps_inf, sigma;
    int npoles;
    int kind[2];
    double delta_eps[2], tau[2], omega_p[2], gamma[2];
} scn_disp_t;
/* sphere in cell units (no rfsyn counterpart); disp >= 0 selects a
 * dispersive model from the disp list (its position fields are ignored) */
typedef struct {
    double cx, cy, cz, radius, eps_r, sigma;
    int disp;
} scn_sphere_t;

/* plane wave through a total-field / scattered-field box (no rfsyn
 * counterpart): direction theta / phi, E polarisation psi, waveform as a
 * source's, total field in the box of sample positions [i0,i1]x[j0,j1]x[k0,k1] */
typedef struct {
    double theta, phi, psi, amplitude;
    int waveform;
    double p0, p1, p2;
    size_t i0, i1, j0, j1, k0, k1;
} scn_plane_wave_t;

typedef struct {
    size_t nx, ny, nz;
    double dx, courant;
    size_t n_steps;
    unsigned periodic;
    size_t npml;                        /* 0: no CPML */
    double m, ma, kappa_max, alpha_max, r0;
    size_t n_boxes;   const scn_box_t *boxes;       /* applied first, in order */
    size_t n_comps;   const scn_comp_t *comps;      /* then scalar overrides */
    size_t n_tensors; const scn_tensor_t *tensors;  /* then tensor edges */
    size_t n_disp;    const scn_disp_t *disp;       /* then dispersive samples */
    size_t n_spheres; const scn_sphere_t *spheres;  /* then spheres, in order */
    int smoothing;                                  /* sphere smoothing: 0 off, 1 diagonal, 2 full 3x3 */
    size_t n_sources; const scn_source_t *sources;
    size_t n_probes;  const scn_probe_t *probes;
    size_t n_freqs;   const double *freqs;
    double src_t_offset, dft_t_offset;
    size_t n_tensor3; const scn_tensor3_t *tensor3; /* applied last */
    const scn_plane_wave_t *plane_wave;             /* NULL: none */
    size_t n_planes;  const scn_plane_t *planes;    /* plane probes: series after the point probes */
} scn_scene_t;

#endif
