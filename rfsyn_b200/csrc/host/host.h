/* host.h -- internal structures of the host library (not public ABI). */
#ifndef RFSYN_B200_HOST_H
#define RFSYN_B200_HOST_H

#include "../../../include/rfsyn_fdtd.h"
#include "../../../include/rfsyn_fdtd_b200.h"
#include "../engine.h"

#define RFB_GRID_MAGIC 0x52464247u /* "RFBG" */
#define RFB_CPML_MAGIC 0x52464243u /* "RFBC" */

/* A grid handed out by fdtd_grid_create: the public struct first, then the
 * device mirror used by the step-wise update functions. */
typedef struct {
    fdtd_grid_t pub;
    unsigned magic;
    rfb_fields_t *dev;
} rfb_grid_ext_t;

typedef struct {
    cpml_t pub;
    unsigned magic;
    size_t nx, ny, nz;
    unsigned periodic;
    double dt;
    rfb_cpml_dev_t *dev;
} rfb_cpml_ext_t;

rfb_grid_ext_t *rfb_grid_ext(const fdtd_grid_t *g);
rfb_cpml_ext_t *rfb_cpml_ext(const cpml_t *p);

/* Geometry-only grid (no field arrays) for the device time loop. */
int rfb_grid_geometry(fdtd_grid_t *g, size_t nx, size_t ny, size_t nz, double dx, double courant);
void rfb_geom_from_grid(const fdtd_grid_t *g, rfb_geom_t *out);
void rfb_cpml_desc_from(const cpml_t *p, rfb_cpml_desc_t *out);

/* Scene image of a materials description for grid g.  extra_cells (canonical
 * i, j, k triples) are forced onto the interface list (point sources);
 * src_slot_of_extra gives, per extra cell, the component (0..2) and source
 * slot to attach (comp < 0: none). */
typedef struct {
    rfb_scene_image_t img;
    /* storage owned by the image */
    uint8_t *codes;
    int32_t *cell_ijk;
    uint8_t *kind;
    double *ca, *cb;
    int32_t *tix, *src, *aix;
    double *t_m11, *t_scale, *t_w;
    int32_t *t_main, *t_nq, *t_uv, *t_sign;
    double *ade_c;
    double *t3;             /* 3x3 samples: 5 doubles per record */
} rfb_scene_build_t;

void rfb_ade_record(const double *model, double dt, double dx, double *out);

typedef struct {
    int i, j, k;
    int component; /* 0..2 */
    int slot;
} rfb_extra_cell_t;

int materials_build_image(const materials_t *mat, const fdtd_grid_t *g, size_t n_extra,
                          const rfb_extra_cell_t *extra, rfb_scene_build_t *out);
void rfb_scene_build_free(rfb_scene_build_t *b);
/* Device copy of the scene for the step-wise API (rebuilt when stale). */
rfb_scene_dev_t *materials_device(const materials_t *mat, const fdtd_grid_t *g);
int materials_matches(const materials_t *mat, const fdtd_grid_t *g);

/* Component c of canonical cell (i,j,k) is swept by rfsyn's E loops
 * (materials.c:915-1059). */
int rfb_e_swept(const fdtd_grid_t *g, int c, size_t i, size_t j, size_t k);

/* Plane-wave TF/SF boundary (tfsf.c): the 1-D incident line and the
 * correction terms of the H samples (applied after the sweep) and of the E
 * samples (applied by the interface-list kernel). */
typedef struct {
    size_t m_len;            /* E samples of the line (H: m_len - 1) */
    double ce, ch;           /* dt / (eps0 d1), dt / (mu0 d1), d1 the line spacing */
    double *src;             /* E1D[0] at steps 0 .. n_steps */
    size_t n_h;              /* H targets: i, j, k, comp; first term, count */
    int32_t *h_ijkc, *h_first, *h_count;
    size_t n_e;              /* E targets, likewise */
    int32_t *e_ijkc, *e_first, *e_count;
    size_t n_hterms, n_eterms;
    double *h_coef, *h_w, *e_coef, *e_w;   /* w: 4 cubic weights per term */
    int32_t *h_idx, *e_idx;
    size_t n_cells;          /* cells whose E samples go on the interface list */
    int32_t *cells;
} rfb_tfsf_build_t;

int rfb_tfsf_build(const fdtd_grid_t *g, const materials_t *mat, const fdtd_b200_plane_wave_t *pw, size_t n_steps,
                   int cpml_npml, rfb_tfsf_build_t *out);
void rfb_tfsf_free(rfb_tfsf_build_t *b);
double rfb_wave_value(int waveform, double amplitude, double p0, double p1, double p2, double t);

/* Inverse of a symmetric positive-definite 3x3 matrix (row-major); -1 when
 * the matrix is not symmetric positive definite. */
int rfb_spd3_inverse(const double e[9], double out[9]);
int rfb_default_precision(void);
int rfb_default_schedule(void);

#endif
