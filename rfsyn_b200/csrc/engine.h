/*
 * engine.h -- internal C interface between the host library (C) and the
 * CUDA engine (engine.cu).  Not part of the public ABI.
 *
 * Device layout shared by every kernel: a field component of a grid with
 * sizes nx, ny, nz is one array of (nx+1)*(ny+1)*pitch elements, index
 * (i*(ny+1) + j)*pitch + k, i.e. rfsyn's padded (i, j, k)-order with k
 * fastest (engine/fdtd/grid.h:25-30) and the k row padded to `pitch`
 * elements so every row starts on a 128-byte boundary.
 */
#ifndef RFSYN_B200_ENGINE_H
#define RFSYN_B200_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { RFB_FP64 = 0, RFB_FP32 = 1 };

/* Loop schedule of the device time loop. */
enum {
    RFB_SCHED_SPLIT = 0,  /* H kernel, then E kernel, in place              */
    RFB_SCHED_FUSED = 1   /* one H+E march per step, ping-pong buffers      */
};

/* Host geometry of one grid. */
typedef struct {
    int nx, ny, nz;
    unsigned periodic;      /* x=1, y=2, z=4 */
    double dx, dt;
} rfb_geom_t;

/* CPML profiles on the host, rfsyn's per-axis arrays (engine/fdtd/cpml.c:21-89):
 * index 0..2 = x, y, z; *_m have n+1 entries (integer positions), *_h have n
 * (half-integer positions). */
typedef struct {
    const double *kinv_m[3], *b_m[3], *a_m[3];
    const double *kinv_h[3], *b_h[3], *a_h[3];
} rfb_cpml_desc_t;

/* Per-(cell, component) entry kinds of the interface list. */
enum {
    RFB_LK_COPY   = 0,  /* component not updated (PEC or padded): keep value */
    RFB_LK_SCALAR = 1,  /* E = Ca E + Cb (dA - dB) with CPML where present    */
    RFB_LK_TENSOR = 2,  /* rfsyn 2x2 tensor edge (materials.c:847-903)        */
    RFB_LK_ADE    = 3,  /* dispersive (Debye / Lorentz) cell                  */
    RFB_LK_TENSOR3 = 4, /* full 3x3 anisotropic sample (no rfsyn counterpart) */
    RFB_LK_CELL3  = 5,  /* 3x3 sample updated by the per-cell kernel, not here */
    RFB_LK_CELLADE = 6  /* dispersive sample updated by the per-cell kernel    */
};

/* Scene image produced by the host materials description and consumed by the
 * engine.  Everything is double on the host; the engine converts to the run
 * precision on upload. */
typedef struct {
    /* Code volume, rfsyn's padded layout (pitch nz+1).  NULL means every cell
     * uses table entry 0 and no cell is diverted to the list. */
    const uint8_t *codes;
    int table_count;
    double table_ca[256], table_cb[256];

    /* Interface list: n_entries = 3 * n_cells, entry e = 3*cell + component. */
    size_t n_cells;
    const int32_t *cell_ijk;    /* 3 per cell: i, j, k (canonical)            */
    const uint8_t *kind;        /* per entry                                  */
    const double *ca, *cb;      /* per entry (scalar kind)                    */
    const int32_t *tix;         /* per entry: tensor record or -1             */
    const int32_t *src;         /* per entry: source slot or -1               */
    const int32_t *aix;         /* per entry: ADE record or -1                */

    /* Tensor records (2x2 edges).  Each record: main coefficient (m11 for Ex,
     * -m11 for Ey), the difference Hz(main0) - Hz(main1), scale and up to four
     * couplings value += w * sign * (Hz(a) - Hz(b)). */
    size_t n_tensors;
    const double *t_m11, *t_scale;
    const int32_t *t_main;      /* 4 per record: u0, v0, u1, v1               */
    const int32_t *t_nq;        /* couplings used                              */
    const double *t_w;          /* 4 per record                               */
    const int32_t *t_uv;        /* 16 per record: ua, va, ub, vb per coupling  */
    const int32_t *t_sign;      /* per record: +1 or -1 applied to couplings   */

    /* 3x3 records: row c of the relative inverse permittivity of the
     * sample's component c, then dt / (eps0 dx).  The update is
     *   E_c += s (m_cc D_c + sum_{b != c} m_cb <D_b>)
     * with D_b the curl difference of component b at its own sample and
     * <D_b> its mean over the four b samples around the E_c sample. */
    size_t n_t3;
    const double *t3;           /* 5 per record                                */

    /* ADE records (dispersive cells), see rfb_ade_desc in the engine. */
    size_t n_ade;
    const double *ade_c;        /* RFB_ADE_NC coefficients per record          */
    int ade_npoles;             /* poles per record (all records share it)     */
} rfb_scene_image_t;

#define RFB_ADE_NC 16

/* One point source: the per-step values s_n = amplitude * waveform(t_n) are
 * evaluated on the host (rfsyn's source.c:40-57 semantics) and uploaded. */
typedef struct {
    int i, j, k, component;
    int hard;               /* 0 = SOFT (add), 1 = HARD (assign) */
    const double *values;   /* n_steps values */
} rfb_source_desc_t;

typedef struct {
    int i, j, k, component; /* component 0..5 = Ex..Hz */
} rfb_probe_desc_t;

typedef struct rfb_engine rfb_engine_t;

/* Creation of a device engine for one simulation.  `stream` may be NULL
 * (the engine creates its own) or a cudaStream_t owned by the caller. */
rfb_engine_t *rfb_engine_create(const rfb_geom_t *geom, int precision, int schedule,
                                const rfb_cpml_desc_t *cpml,      /* NULL: no CPML  */
                                const rfb_scene_image_t *scene,   /* NULL: vacuum   */
                                size_t n_sources, const rfb_source_desc_t *sources,
                                size_t n_probes, const rfb_probe_desc_t *probes,
                                size_t n_steps, void *stream);
void rfb_engine_destroy(rfb_engine_t *e);
/* Plane probes, n triples (axis 0..2, index, component 0..5 = ex..hz): each
 * records the mean of the component over the whole grid plane every step,
 * as series n_probes .. n_probes + n - 1.  Bins (Hz) of the running DFT of
 * every series, accumulated with the steps, sample n at t = (n + t_off) dt.
 * Both before the first step. */
int rfb_engine_set_planes(rfb_engine_t *e, size_t n, const int *axis_index_comp);
int rfb_engine_set_dft(rfb_engine_t *e, size_t n_freqs, const double *freqs_hz, double t_offset_steps);
/* An engine for one scene of a batch (FUSED schedule): device state only;
 * the batch builds the sweep plans and owns the kernels' launches.  `stream`
 * must be the batch's stream. */
rfb_engine_t *rfb_engine_create_member(const rfb_geom_t *geom, int precision, const rfb_cpml_desc_t *cpml,
                                       const rfb_scene_image_t *scene, size_t n_sources,
                                       const rfb_source_desc_t *sources, size_t n_probes,
                                       const rfb_probe_desc_t *probes, size_t n_steps, void *stream);

/* ---- batches of scenes advanced together (batch.cuh) ----------------------- */
typedef struct rfb_batch rfb_batch_t;
typedef struct {
    size_t scenes, cells, list_cells, slab_cell_axes;
    int tile_j, ring_depth, mode, seg_interior, seg_edge;
    int items_interior, items_xslab, items_edge;
    int launches_per_step;
    int unified;
} rfb_batch_info_t;
/* Takes ownership of the members (and of `stream` when own_stream). */
rfb_batch_t *rfb_batch_create(rfb_engine_t **members, size_t n, void *stream, int own_stream);
void rfb_batch_destroy(rfb_batch_t *b);
int rfb_batch_reset(rfb_batch_t *b);
int rfb_batch_advance(rfb_batch_t *b, size_t n);
int rfb_batch_advance_timed(rfb_batch_t *b, size_t n, double *ms);
int rfb_batch_sync(rfb_batch_t *b);
int rfb_batch_time_kernels(rfb_batch_t *b, size_t n, double *sweep_ms, double *other_ms);
rfb_engine_t *rfb_batch_member(rfb_batch_t *b, size_t s);
size_t rfb_batch_size(rfb_batch_t *b);
size_t rfb_batch_steps_done(rfb_batch_t *b);
void *rfb_batch_stream(rfb_batch_t *b);
int rfb_batch_info(rfb_batch_t *b, rfb_batch_info_t *out);
/* A non-blocking stream (for a batch's members), or NULL. */
void *rfb_stream_create(void);
void rfb_stream_destroy(void *stream);

/* Plane wave through a TF/SF boundary: the 1-D incident line and the
 * correction terms (see tfsf.c).  H targets are corrected after the sweep
 * from the line's E; E targets are list entries (entry_first / entry_count
 * per entry of the scene image, -1 / 0 for none) corrected from its H. */
typedef struct {
    size_t m_len;
    double ce, ch;
    const double *src;                       /* n_steps + 1 */
    size_t n_h;
    const int32_t *h_ijkc, *h_first, *h_count;
    size_t n_hterms, n_eterms;
    const double *h_coef, *h_w, *e_coef, *e_w;  /* w: 4 weights per term */
    const int32_t *h_idx, *e_idx;
    const int32_t *entry_first, *entry_count;  /* 3 * n_cells of the scene image */
} rfb_tfsf_desc_t;
/* Attaches a plane wave to an engine before its first step. */
int rfb_engine_set_tfsf(rfb_engine_t *e, const rfb_tfsf_desc_t *d);

/* Zero fields, psi and ADE state and rewind the step counter (async). */
int rfb_engine_reset(rfb_engine_t *e);
/* Enqueue n steps on the engine stream (CUDA graph replay). */
int rfb_engine_advance(rfb_engine_t *e, size_t n);
/* Blocking copy of the probe time series (n_probes * n_steps doubles, probe
 * major).  Only the first `steps_done` samples of each probe are valid. */
int rfb_engine_read_probes(rfb_engine_t *e, double *out);
/* One probe's stage signal as interleaved float I/Q (2 n_steps floats),
 * with rfsyn's AWGN when noise != 0 (snr_linear = 10^(snr_db/10)). */
int rfb_engine_read_iq(rfb_engine_t *e, int probe, int noise, double snr_linear, unsigned long long seed,
                       unsigned long long stream, float *out);
/* Running DFT of every probe series over bins freqs (Kahan-compensated FP32
 * accumulation in FP32 runs, FP64 otherwise; FP64 phase recurrence); sample n
 * is taken at t = (n + t_offset_steps) * dt and weighted by dt. */
int rfb_engine_probe_dft(rfb_engine_t *e, size_t n_freqs, const double *freqs_hz,
                         double t_offset_steps, double *out_re, double *out_im);
int rfb_engine_sync(rfb_engine_t *e);
/* advance + synchronise, returning the GPU time of the n steps (CUDA events
 * recorded on the engine stream). */
int rfb_engine_advance_timed(rfb_engine_t *e, size_t n, double *ms);
void *rfb_engine_stream(rfb_engine_t *e);
size_t rfb_engine_steps_done(rfb_engine_t *e);
/* Kernel launches per time step (for launch accounting). */
int rfb_engine_launches_per_step(rfb_engine_t *e);
typedef struct {
    size_t list_cells, dispersive, slab_cell_axes, h2d_bytes;
    int tile_j, seg_len, ring_depth, tma, interior_items, edge_items, unified;
    int interior_ring2;  /* 0, or the ring depth of the two-rows interior sweep */
    int seg_edge;        /* planes per slab / boundary work item */
} rfb_engine_info_t;
int rfb_engine_info(rfb_engine_t *e, rfb_engine_info_t *out);
int rfb_engine_time_kernels(rfb_engine_t *e, size_t n, double *sweep_ms, double *other_ms);
/* Download one field component (0..5) into a host array in rfsyn layout. */
int rfb_engine_read_field(rfb_engine_t *e, int component, double *host);

/* ---- step-wise API support (rfsyn's fdtd_update_* on host arrays) -------- */
typedef struct rfb_fields rfb_fields_t;      /* FP64 device mirror of a grid  */
typedef struct rfb_cpml_dev rfb_cpml_dev_t;  /* device profiles + slab psi    */
typedef struct rfb_scene_dev rfb_scene_dev_t;/* device codes + list           */

rfb_fields_t *rfb_fields_create(const rfb_geom_t *geom);
void rfb_fields_destroy(rfb_fields_t *f);
rfb_cpml_dev_t *rfb_cpml_dev_create(const rfb_geom_t *geom, const rfb_cpml_desc_t *desc);
void rfb_cpml_dev_destroy(rfb_cpml_dev_t *c);
rfb_scene_dev_t *rfb_scene_dev_create(const rfb_geom_t *geom, const rfb_scene_image_t *img);
void rfb_scene_dev_destroy(rfb_scene_dev_t *s);

/* host arrays: ex, ey, ez, hx, hy, hz in rfsyn layout (double). */
int rfb_step_update_h(rfb_fields_t *f, const rfb_geom_t *geom, rfb_cpml_dev_t *cpml,
                      double *const host[6]);
/* vacuum_cb: Cb of the vacuum table used when scene is NULL. */
int rfb_step_update_e(rfb_fields_t *f, const rfb_geom_t *geom, rfb_cpml_dev_t *cpml,
                      rfb_scene_dev_t *scene, double vacuum_cb, double *const host[6]);

/* FP64 energy audit of an engine's resident fields (rfsyn
 * validate_long_term_stability.c:166-209, audit_periodic_energy.c:43-71):
 * sums over i < nx, j < ny, k < nz of 0.5 eps E^2 and 0.5 mu0 H^2 times
 * dx^3, eps = dt / (dx Cb) per (cell, component) with Cb the component's
 * scalar coefficient.  q[] receives RFB_EN_COUNT values (RFB_EN_*). */
enum {
    RFB_EN_E = 0,        /* electric energy of the current E (step n)            */
    RFB_EN_H,            /* magnetic energy of the current H (step n - 1/2)      */
    RFB_EN_E_INT,        /* electric, planes x_lo <= i < x_hi                    */
    RFB_EN_H_INT,        /* magnetic, planes x_lo <= i < x_hi                    */
    RFB_EN_E_PREV,       /* electric energy of E at step n - 1 (ping-pong only)  */
    RFB_EN_CROSS,        /* 0.5 mu0 H^{n-3/2} . H^{n-1/2} dx^3 (ping-pong only)  */
    RFB_EN_MAX_E,        /* max |E| (current)                                    */
    RFB_EN_MAX_H,        /* max |H| (current)                                    */
    RFB_EN_NONFINITE,    /* number of non-finite current samples                 */
    RFB_EN_COUNT
};
int rfb_engine_energy(rfb_engine_t *e, double dt, double dx, int x_lo, int x_hi, double q[RFB_EN_COUNT]);

/* Fill fractions of a sphere (centre / radius in cell units) for the three E
 * samples of every cell of the box [i0, i0+ni) x [j0, j0+nj) x [k0, k0+nk):
 * f[3*cell + c] and the squared normal component n2[3*cell + c] along the
 * sample's own axis; cell = ((i-i0)*nj + (j-j0))*nk + (k-k0).  FP64 on the
 * GPU, every operation rounded separately (bit-identical to the oracle). */
int rfb_sphere_fractions(const double centre[3], double radius, int i0, int j0, int k0, int ni, int nj, int nk,
                         double *f, double *n2);

/* Smoothed permittivity of cut cells, FP64 on the GPU (smooth.cu).
 * rfb_sphere_rows: for every cell of the box as rfb_sphere_fractions, the
 * fill fraction f[3 cell + c] of each E sample and row c of the smoothed
 * relative inverse permittivity rows[9 cell + 3 c + b] between the cell's
 * isotropic background eps_bg[cell] and eps_in, along the sphere's normal.
 * rfb_slab_rows: the same for n listed samples ijkc[4 s ..] = (i, j, k, c)
 * against the slab |(x - point) . u| <= thickness / 2 (u unit) holding the
 * 3x3 eps_in: f[s], rows[3 s + b]. */
int rfb_sphere_rows(const double centre[3], double radius, double eps_in, int i0, int j0, int k0, int ni, int nj,
                    int nk, const double *eps_bg, double *f, double *rows);
int rfb_slab_rows(const double point[3], const double unit_normal[3], double thickness, const double eps_in[9],
                  const int *ijkc, const double *eps_bg, int n, double *f, double *rows);

/* Last error message of the calling thread ("" if none). */
const char *rfb_last_error(void);
void rfb_set_error(const char *fmt, ...);

/* Host wall clock (s) and, with RFSYN_FDTD_TRACE=1 in the environment, one
 * stderr line "rfsyn_b200 trace: <phase> <ms>" per traced phase. */
double rfb_now(void);
void rfb_trace(const char *phase, double t0);

/* Number of kernels this process has launched through the engine;
 * rfb_count_launch adds one for a launch made outside engine.cu. */
unsigned long long rfb_launch_count(void);
void rfb_count_launch(void);
unsigned long long rfb_cached_bytes(void);
/* process-wide settings (host/run.c, engine.cu) */
const char *rfb_plan_override(void);
int rfb_tune_enabled(void);
void rfb_set_trace(int on);
int rfb_trace_enabled(void);
void rfb_release_cached_memory(void);

#ifdef __cplusplus
}
#endif

#endif
