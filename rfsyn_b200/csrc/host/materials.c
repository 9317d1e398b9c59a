/* materials.c -- host-side scene description (rfsyn materials API,
 * engine/fdtd/materials.c:27-799 semantics) and its compilation into the
 * device image: a per-cell code volume plus a compact interface list that
 * carries every per-component override and tensor edge.
 *
 * Storage here is B200-first rather than rfsyn's: overrides live in
 * open-addressing hash maps keyed by padded_index*3 + component (O(1) set /
 * clear / lookup instead of sorted arrays with memmove), and are sorted only
 * once, when the device image is built. */
#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "host.h"

#define MATERIAL_LIMIT 256
/* dispersive model packed as doubles: eps_inf, sigma, n_poles, then per pole
 * kind, delta_eps, tau, omega_p, gamma */
#define DISP_W 13

typedef struct {
    double eps_r, sigma;
    material_coeff_t coeff;
} mat_entry_t;

/* ---- open-addressing map: uint64 key -> fixed-size value ------------------ */
typedef struct {
    uint64_t *keys;    /* UINT64_MAX = empty */
    double *vals;      /* vw doubles per slot */
    size_t cap, count, vw;
    uint8_t *mark;     /* per-cell flag set by every put of key cell * 3 + c (or NULL) */
} omap_t;

#define OMAP_EMPTY UINT64_MAX

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

/* Home slot of a key.  Keys are cell * 3 + component, and scenes describe
 * cells in runs along k, so runs of 32 consecutive keys keep consecutive
 * slots and only the run is hashed: filling or reading a slab, a box or a
 * shell walks the table (and its values) nearly sequentially instead of
 * taking a cache miss per key. */
static size_t omap_home(uint64_t key, size_t mask) {
    return (size_t)((mix64(key >> 5) << 5) | (key & 31u)) & mask;
}

static int omap_init(omap_t *m, size_t vw) {
    m->vw = vw;
    m->cap = 0;
    m->count = 0;
    m->keys = NULL;
    m->vals = NULL;
    m->mark = NULL;
    return 0;
}

static void omap_free(omap_t *m) {
    free(m->keys);
    free(m->vals);
    m->keys = NULL;
    m->vals = NULL;
    m->cap = m->count = 0;
}

static long omap_find(const omap_t *m, uint64_t key) {
    if (!m->count) return -1; /* an empty map: no probe (deletes and lookups in maps a scene never filled) */
    size_t mask = m->cap - 1, h = omap_home(key, mask);
    for (;;) {
        if (m->keys[h] == OMAP_EMPTY) return -1;
        if (m->keys[h] == key) return (long)h;
        h = (h + 1) & mask;
    }
}

static int omap_grow(omap_t *m, size_t want_cap) {
    uint64_t *ok = m->keys;
    double *ov = m->vals;
    size_t ocap = m->cap;
    uint64_t *nk = malloc(want_cap * sizeof(uint64_t));
    double *nv = malloc(want_cap * m->vw * sizeof(double));
    if (!nk || !nv) {
        free(nk);
        free(nv);
        return -1;
    }
    for (size_t q = 0; q < want_cap; q++) nk[q] = OMAP_EMPTY;
    size_t mask = want_cap - 1;
    for (size_t q = 0; q < ocap; q++) {
        if (ok[q] == OMAP_EMPTY) continue;
        size_t h = omap_home(ok[q], mask);
        while (nk[h] != OMAP_EMPTY) h = (h + 1) & mask;
        nk[h] = ok[q];
        memcpy(nv + h * m->vw, ov + q * m->vw, m->vw * sizeof(double));
    }
    free(ok);
    free(ov);
    m->keys = nk;
    m->vals = nv;
    m->cap = want_cap;
    return 0;
}

/* Room for n_more new keys without a rehash on the way (a bulk setter
 * reserves once instead of growing through every power of two). */
static int omap_reserve(omap_t *m, size_t n_more) {
    const size_t need = 2 * (m->count + n_more);
    if (need <= m->cap) return 0;
    size_t cap = m->cap ? m->cap : 64;
    while (cap < need) cap *= 2;
    return omap_grow(m, cap);
}

static int omap_put(omap_t *m, uint64_t key, const double *val) {
    if (m->mark) m->mark[key / 3] = 1;
    if ((m->count + 1) * 2 > m->cap) {
        if (omap_grow(m, m->cap ? m->cap * 2 : 64) != 0) return -1;
    }
    /* one probe: the key's slot, or the empty slot that ends its chain */
    size_t mask = m->cap - 1, h = omap_home(key, mask);
    while (m->keys[h] != OMAP_EMPTY && m->keys[h] != key) h = (h + 1) & mask;
    if (m->keys[h] == OMAP_EMPTY) {
        m->keys[h] = key;
        m->count++;
    }
    memcpy(m->vals + h * m->vw, val, m->vw * sizeof(double));
    return 0;
}

/* Backward-shift deletion keeps probe chains intact without tombstones. */
static void omap_del_slot(omap_t *m, size_t h) {
    size_t mask = m->cap - 1;
    size_t hole = h;
    size_t q = (h + 1) & mask;
    while (m->keys[q] != OMAP_EMPTY) {
        size_t home = omap_home(m->keys[q], mask);
        /* can the entry at q move into the hole? (home not in (hole, q]) */
        int movable = (q > hole) ? (home <= hole || home > q) : (home <= hole && home > q);
        if (movable) {
            m->keys[hole] = m->keys[q];
            memcpy(m->vals + hole * m->vw, m->vals + q * m->vw, m->vw * sizeof(double));
            hole = q;
        }
        q = (q + 1) & mask;
    }
    m->keys[hole] = OMAP_EMPTY;
    m->count--;
}

static void omap_del(omap_t *m, uint64_t key) {
    long at = omap_find(m, key);
    if (at >= 0) omap_del_slot(m, (size_t)at);
}

/* ---- the description --------------------------------------------------------- */
struct materials {
    size_t nx, ny, nz, total;
    double dx, dt;
    uint8_t *ids;
    /* 1 for every cell that ever held a per-component description (set by
     * the maps' puts, never cleared): cells without it need no map lookups */
    uint8_t *touched;
    mat_entry_t table[MATERIAL_LIMIT];
    size_t table_count;
    omap_t scalar;  /* key -> (Ca, Cb) */
    omap_t tensor;  /* key -> (m11, m12, m22, scale) */
    omap_t disp;    /* key -> dispersive model (DISP_W doubles) */
    omap_t tensor3; /* key -> row of the 3x3 relative inverse permittivity, then sigma (4 doubles) */
    unsigned long version;
    /* device copy for the step-wise API */
    rfb_scene_dev_t *dev;
    unsigned long dev_version;
    unsigned dev_periodic;
};

int materials_matches(const materials_t *mat, const fdtd_grid_t *g) {
    return mat && g && mat->nx == g->nx && mat->ny == g->ny && mat->nz == g->nz && mat->dx == g->dx &&
           mat->dt == g->dt;
}

static int component_number(field_component_t c) {
    switch (c) {
    case FIELD_EX: return 0;
    case FIELD_EY: return 1;
    case FIELD_EZ: return 2;
    default: return -1;
    }
}

/* Valid padded coordinates of an E component; periodic axes omit the
 * duplicate endpoint (materials.c:70-90). */
static int component_valid(const fdtd_grid_t *g, int c, size_t i, size_t j, size_t k) {
    if (!g || c < 0 || c > 2) return 0;
    size_t ni = g->nx, nj = g->ny, nk = g->nz;
    if (c != 0 && !(g->periodic_axes & 1u)) ni++;
    if (c != 1 && !(g->periodic_axes & 2u)) nj++;
    if (c != 2 && !(g->periodic_axes & 4u)) nk++;
    return i < ni && j < nj && k < nk;
}

/* Lossy update coefficients (materials.c:92-125): loss = sigma dt / (2 eps),
 * Ca = (1 - loss)/(1 + loss), Cb = dt/(eps dx)/(1 + loss). */
static int make_coeff(const materials_t *mat, double eps_r, double sigma, material_coeff_t *out) {
    if (!mat || !out || !isfinite(eps_r) || eps_r < 1.0 || !isfinite(sigma) || sigma < 0.0) return -1;
    double eps = eps_r * EPS0;
    double loss = (sigma * mat->dt) / (2.0 * eps);
    double cb = mat->dt / (eps * mat->dx);
    if (!isfinite(eps) || eps <= 0.0 || !isfinite(loss) || !isfinite(cb) || cb <= 0.0) return -1;
    material_coeff_t coeff = {.Ca = (1.0 - loss) / (1.0 + loss), .Cb = cb / (1.0 + loss)};
    if (!isfinite(coeff.Ca) || !isfinite(coeff.Cb) || coeff.Cb <= 0.0) return -1;
    *out = coeff;
    return 0;
}

materials_t *materials_create(const fdtd_grid_t *g) {
    if (!g || g->nx == 0 || g->ny == 0 || g->nz == 0) return NULL;
    if (!isfinite(g->dx) || g->dx <= 0.0 || !isfinite(g->dt) || g->dt <= 0.0) return NULL;
    if (g->nx == SIZE_MAX || g->ny == SIZE_MAX || g->nz == SIZE_MAX) return NULL;
    size_t nx1 = g->nx + 1, ny1 = g->ny + 1, nz1 = g->nz + 1;
    if (nx1 > SIZE_MAX / ny1) return NULL;
    size_t total = nx1 * ny1;
    if (total > SIZE_MAX / nz1) return NULL;
    total *= nz1;
    if (total > SIZE_MAX / 3) return NULL;
    materials_t *mat = calloc(1, sizeof(*mat));
    if (!mat) return NULL;
    mat->nx = g->nx;
    mat->ny = g->ny;
    mat->nz = g->nz;
    mat->total = total;
    mat->dx = g->dx;
    mat->dt = g->dt;
    omap_init(&mat->scalar, 2);
    omap_init(&mat->tensor, 4);
    omap_init(&mat->disp, DISP_W);
    omap_init(&mat->tensor3, 4);
    mat->ids = calloc(total, 1);
    mat->touched = calloc(total, 1);
    if (!mat->ids || !mat->touched) {
        materials_destroy(mat);
        return NULL;
    }
    mat->scalar.mark = mat->tensor.mark = mat->disp.mark = mat->tensor3.mark = mat->touched;
    material_id_t vacuum;
    if (materials_register(mat, 1.0, 0.0, &vacuum) != 0) {
        materials_destroy(mat);
        return NULL;
    }
    return mat;
}

void materials_destroy(materials_t *mat) {
    if (!mat) return;
    free(mat->ids);
    free(mat->touched);
    omap_free(&mat->scalar);
    omap_free(&mat->tensor);
    omap_free(&mat->disp);
    omap_free(&mat->tensor3);
    rfb_scene_dev_destroy(mat->dev);
    free(mat);
}

int materials_register(materials_t *mat, double eps_r, double sigma, material_id_t *id_out) {
    material_coeff_t coeff;
    if (!mat || !id_out || make_coeff(mat, eps_r, sigma, &coeff) != 0) return -1;
    for (size_t n = 0; n < mat->table_count; n++) {
        if (mat->table[n].eps_r == eps_r && mat->table[n].sigma == sigma) {
            *id_out = (material_id_t)n;
            return 0;
        }
    }
    if (mat->table_count >= MATERIAL_LIMIT) return -1;
    size_t n = mat->table_count++;
    mat->table[n].eps_r = eps_r;
    mat->table[n].sigma = sigma;
    mat->table[n].coeff = coeff;
    mat->version++;
    *id_out = (material_id_t)n;
    return 0;
}

/* Padded ends accepted; periodic starts must be canonical (materials.c:425-454). */
static int box_valid(const materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0, size_t j1,
                     size_t k0, size_t k1) {
    if (!materials_matches(mat, g)) return 0;
    if (i0 >= i1 || j0 >= j1 || k0 >= k1) return 0;
    if (i1 > g->nx + 1 || j1 > g->ny + 1 || k1 > g->nz + 1) return 0;
    if ((g->periodic_axes & 1u) && i0 >= g->nx) return 0;
    if ((g->periodic_axes & 2u) && j0 >= g->ny) return 0;
    if ((g->periodic_axes & 4u) && k0 >= g->nz) return 0;
    return 1;
}

static int key_in_box(const materials_t *mat, uint64_t key, size_t i0, size_t i1, size_t j0, size_t j1, size_t k0,
                      size_t k1) {
    size_t idx = (size_t)(key / 3);
    size_t k = idx % (mat->nz + 1);
    size_t row = idx / (mat->nz + 1);
    size_t j = row % (mat->ny + 1);
    size_t i = row / (mat->ny + 1);
    return i >= i0 && i < i1 && j >= j0 && j < j1 && k >= k0 && k < k1;
}

static void clear_box_overrides(materials_t *mat, omap_t *m, size_t i0, size_t i1, size_t j0, size_t j1, size_t k0,
                                size_t k1) {
    if (!m->count) return;
    /* collect then delete, so deletion shifts cannot skip entries */
    uint64_t *victims = malloc(m->count * sizeof(uint64_t));
    size_t nv = 0;
    if (!victims) return;
    for (size_t q = 0; q < m->cap; q++)
        if (m->keys[q] != OMAP_EMPTY && key_in_box(mat, m->keys[q], i0, i1, j0, j1, k0, k1))
            victims[nv++] = m->keys[q];
    for (size_t q = 0; q < nv; q++) omap_del(m, victims[q]);
    free(victims);
}

int materials_assign_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0, size_t j1,
                         size_t k0, size_t k1, material_id_t id) {
    if (!box_valid(mat, g, i0, i1, j0, j1, k0, k1) || (size_t)id >= mat->table_count) return -1;
    if ((g->periodic_axes & 1u) && i1 > g->nx) i1 = g->nx;
    if ((g->periodic_axes & 2u) && j1 > g->ny) j1 = g->ny;
    if ((g->periodic_axes & 4u) && k1 > g->nz) k1 = g->nz;
    for (size_t i = i0; i < i1; i++)
        for (size_t j = j0; j < j1; j++) {
            uint8_t *row = mat->ids + fdtd_index(g, i, j, 0);
            if (!(g->periodic_axes & 4u)) {
                memset(row + k0, id, k1 - k0);
            } else {
                for (size_t k = k0; k < k1; k++) mat->ids[fdtd_index(g, i, j, k)] = id;
            }
        }
    clear_box_overrides(mat, &mat->scalar, i0, i1, j0, j1, k0, k1);
    clear_box_overrides(mat, &mat->tensor, i0, i1, j0, j1, k0, k1);
    clear_box_overrides(mat, &mat->disp, i0, i1, j0, j1, k0, k1);
    clear_box_overrides(mat, &mat->tensor3, i0, i1, j0, j1, k0, k1);
    mat->version++;
    return 0;
}

int materials_set_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0, size_t j1, size_t k0,
                      size_t k1, double eps_r, double sigma) {
    if (!box_valid(mat, g, i0, i1, j0, j1, k0, k1)) return -1;
    material_id_t id;
    if (materials_register(mat, eps_r, sigma, &id) != 0) return -1;
    return materials_assign_box(mat, g, i0, i1, j0, j1, k0, k1, id);
}

int materials_set_component(materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i, size_t j,
                            size_t k, double eps_r, double sigma) {
    int c = component_number(component);
    material_coeff_t coeff;
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k) || make_coeff(mat, eps_r, sigma, &coeff) != 0)
        return -1;
    uint64_t key = (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c;
    double v[2] = {coeff.Ca, coeff.Cb};
    if (omap_put(&mat->scalar, key, v) != 0) return -1;
    mat->version++;
    return 0;
}

int materials_clear_component(materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i, size_t j,
                              size_t k) {
    int c = component_number(component);
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    omap_del(&mat->scalar, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c);
    mat->version++;
    return 0;
}

static material_coeff_t lookup(const materials_t *mat, size_t idx, int c) {
    long at = omap_find(&mat->scalar, (uint64_t)idx * 3 + (uint64_t)c);
    if (at >= 0) {
        material_coeff_t r = {mat->scalar.vals[2 * at], mat->scalar.vals[2 * at + 1]};
        return r;
    }
    return mat->table[mat->ids[idx]].coeff;
}

int materials_get_coefficients(const materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i,
                               size_t j, size_t k, material_coeff_t *out) {
    int c = component_number(component);
    if (!out || !materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    *out = lookup(mat, fdtd_index(g, i, j, k), c);
    return 0;
}

/* x/y interior margins for the 4-neighbour tensor stencil (materials.c:273-294). */
static int tensor_margin_ok(const fdtd_grid_t *g, size_t i, size_t j) {
    if (!(g->periodic_axes & 1u) && (g->nx < 3 || i == 0 || i >= g->nx - 1)) return 0;
    if (!(g->periodic_axes & 2u) && (g->ny < 3 || j == 0 || j >= g->ny - 1)) return 0;
    return 1;
}

/* Positive definiteness of [[a b][b c]] without forming ac - b^2
 * (materials.c:296-308). */
static int tensor_spd(double a, double b, double c) {
    if (!isfinite(a) || !isfinite(b) || !isfinite(c) || a <= 0.0 || c <= 0.0) return 0;
    return fabs(b) / sqrt(a) < sqrt(c);
}

int materials_set_component_tensor(materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i,
                                   size_t j, size_t k, double m11, double m12, double m22) {
    int c = component_number(component);
    if (c != 0 && c != 1) return -1;
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k) || !tensor_margin_ok(g, i, j) ||
        !tensor_spd(m11, m12, m22))
        return -1;
    double scale = mat->dt / (EPS0 * mat->dx);
    if (!isfinite(scale) || scale <= 0.0) return -1;
    double v[4] = {m11, m12, m22, scale};
    if (omap_put(&mat->tensor, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) != 0) return -1;
    mat->version++;
    return 0;
}

int materials_clear_component_tensor(materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i,
                                     size_t j, size_t k) {
    int c = component_number(component);
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    omap_del(&mat->tensor, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c);
    mat->version++;
    return 0;
}

static const double *tensor_at(const materials_t *mat, size_t idx, int c) {
    long at = omap_find(&mat->tensor, (uint64_t)idx * 3 + (uint64_t)c);
    return at >= 0 ? mat->tensor.vals + 4 * (size_t)at : NULL;
}

int materials_get_tensor(const materials_t *mat, const fdtd_grid_t *g, field_component_t component, size_t i, size_t j,
                         size_t k, material_tensor_t *out) {
    int c = component_number(component);
    if (!out || !materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    const double *t = tensor_at(mat, fdtd_index(g, i, j, k), c);
    if (!t) return 1;
    out->m11 = t[0];
    out->m12 = t[1];
    out->m22 = t[2];
    out->scale = t[3];
    return 0;
}

/* ---- dispersive samples ------------------------------------------------------ */
static int pack_model(const fdtd_b200_dispersive_t *m, double *v) {
    if (!m || !isfinite(m->eps_inf) || m->eps_inf < 1.0 || !isfinite(m->sigma) || m->sigma < 0.0 || m->n_poles < 1 ||
        m->n_poles > FDTD_B200_MAX_POLES)
        return -1;
    memset(v, 0, DISP_W * sizeof(double));
    v[0] = m->eps_inf;
    v[1] = m->sigma;
    v[2] = (double)m->n_poles;
    for (int p = 0; p < m->n_poles; p++) {
        double *w = v + 3 + 5 * p;
        if (!isfinite(m->delta_eps[p]) || m->delta_eps[p] <= 0.0) return -1;
        if (m->kind[p] == FDTD_B200_POLE_DEBYE) {
            if (!isfinite(m->tau[p]) || m->tau[p] <= 0.0) return -1;
        } else if (m->kind[p] == FDTD_B200_POLE_LORENTZ) {
            if (!isfinite(m->omega_p[p]) || m->omega_p[p] <= 0.0 || !isfinite(m->gamma[p]) || m->gamma[p] < 0.0)
                return -1;
        } else {
            return -1;
        }
        w[0] = (double)m->kind[p];
        w[1] = m->delta_eps[p];
        w[2] = m->tau[p];
        w[3] = m->omega_p[p];
        w[4] = m->gamma[p];
    }
    return 0;
}

int fdtd_b200_materials_set_component_dispersive(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                                 size_t i, size_t j, size_t k, const fdtd_b200_dispersive_t *model) {
    int c = component_number(component);
    double v[DISP_W];
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k) || pack_model(model, v) != 0) return -1;
    if (omap_put(&mat->disp, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) != 0) return -1;
    mat->version++;
    return 0;
}

int fdtd_b200_materials_clear_component_dispersive(materials_t *mat, const fdtd_grid_t *g,
                                                   field_component_t component, size_t i, size_t j, size_t k) {
    int c = component_number(component);
    if (!materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    omap_del(&mat->disp, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c);
    mat->version++;
    return 0;
}

/* ---- full 3x3 anisotropic samples ---------------------------------------------
 * No counterpart in rfsyn, whose tensor edges are 2x2 (materials.c:658-903).
 * A sample of component c holds row c of the relative inverse permittivity
 * m = eps_r^-1 (3x3).  Its update needs the H samples of the neighbouring
 * cells one step away on every axis: on an axis without wrap the cell must
 * lie in [1, n-1].  Like rfsyn's tensor edges the samples are lossless and
 * meant for cells outside the CPML. */
static int tensor3_margin_ok(const fdtd_grid_t *g, size_t i, size_t j, size_t k) {
    const size_t n[3] = {g->nx, g->ny, g->nz}, p[3] = {i, j, k};
    for (int a = 0; a < 3; a++)
        if (!(g->periodic_axes & (1u << a)) && (p[a] < 1 || p[a] + 1 > n[a])) return 0;
    return 1;
}

int fdtd_b200_materials_set_component_tensor3(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                              size_t i, size_t j, size_t k, const double row[3]) {
    int c = component_number(component);
    if (c < 0 || c > 2 || !row || !materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    if (!tensor3_margin_ok(g, i, j, k)) return -1;
    for (int q = 0; q < 3; q++)
        if (!isfinite(row[q])) return -1;
    if (!(row[c] > 0.0)) return -1;
    const double v[4] = {row[0], row[1], row[2], 0.0};
    if (omap_put(&mat->tensor3, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) != 0) return -1;
    mat->version++;
    return 0;
}

int fdtd_b200_materials_clear_component_tensor3(materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                                size_t i, size_t j, size_t k) {
    int c = component_number(component);
    if (c < 0 || c > 2 || !materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    omap_del(&mat->tensor3, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c);
    mat->version++;
    return 0;
}

int fdtd_b200_materials_set_tensor3_slab(materials_t *mat, const fdtd_grid_t *g, const double point[3],
                                         const double normal[3], double thickness, const double eps_r[9]) {
    double m[9];
    if (!point || !normal || !eps_r || !(thickness > 0.0) || rfb_spd3_inverse(eps_r, m) != 0) return -1;
    if (!materials_matches(mat, g)) return -1;
    const double nn = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
    if (!(nn > 0.0)) return -1;
    const double u[3] = {normal[0] / nn, normal[1] / nn, normal[2] / nn};
    const size_t n[3] = {g->nx, g->ny, g->nz};
    size_t lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        const int per = (g->periodic_axes >> a) & 1u;
        lo[a] = per ? 0 : 1;
        hi[a] = per ? n[a] : n[a];  /* cells [lo, hi): the margin rule keeps index n - 1 at most */
    }
    /* Per (i, j) column only the k range the slab can reach is tested: the
     * sample offsets move d by at most 0.5 (|u0| + |u1| + |u2|), and a cell
     * of margin on each side keeps the bound conservative; every sample
     * then passes the exact test below.  Pass 0 counts, pass 1 stores. */
    const double half = 0.5 * thickness, slack = 0.5 * (fabs(u[0]) + fabs(u[1]) + fabs(u[2]));
    for (int pass = 0; pass < 2; pass++) {
        size_t count = 0;
        for (size_t i = lo[0]; i < hi[0]; i++)
            for (size_t j = lo[1]; j < hi[1]; j++) {
                size_t ka = lo[2], kb = hi[2];
                if (fabs(u[2]) > 1e-9) {
                    const double r0 = u[0] * ((double)i - point[0]) + u[1] * ((double)j - point[1]) - u[2] * point[2];
                    double a = (-half - slack - r0) / u[2], b = (half + slack - r0) / u[2];
                    if (a > b) { const double s = a; a = b; b = s; }
                    a = floor(a) - 1.0;
                    b = ceil(b) + 2.0;
                    if (a > (double)ka) ka = a >= (double)hi[2] ? hi[2] : (size_t)a;
                    if (b < (double)kb) kb = b <= (double)ka ? ka : (size_t)b;
                }
                for (size_t k = ka; k < kb; k++)
                    for (int c = 0; c < 3; c++) {
                        double p[3] = {(double)i, (double)j, (double)k};
                        p[c] += 0.5;
                        const double d =
                            u[0] * (p[0] - point[0]) + u[1] * (p[1] - point[1]) + u[2] * (p[2] - point[2]);
                        if (fabs(d) > half) continue;
                        if (!component_valid(g, c, i, j, k) || !tensor3_margin_ok(g, i, j, k)) continue;
                        const double v[4] = {m[3 * c], m[3 * c + 1], m[3 * c + 2], 0.0};
                        if (pass == 0) {
                            count++;
                        } else if (omap_put(&mat->tensor3, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) !=
                                   0) {
                            return -1;
                        }
                    }
            }
        if (pass == 0 && omap_reserve(&mat->tensor3, count) != 0) return -1;
    }
    mat->version++;
    return 0;
}

/* The slab with subpixel smoothing of its faces.  Every valid E sample
 * (component_valid, tensor3_margin_ok) whose unit cube lies inside the slab
 * -- |d| + r <= thickness / 2, d the sample's signed distance from the mid
 * plane and r = (|u0| + |u1| + |u2|) / 2 the cube's reach along the normal u
 * -- gets the row of eps_r^-1 as the staircased slab gives it; every sample
 * whose cube the faces may cut (|d| - r <= thickness / 2 < |d| + r) gets, when
 * its fill fraction f (8^3 lattice) is positive, the row of the smoothed
 * inverse permittivity between the cell's table material (isotropic, the
 * background) and eps_r along u, with sigma (1 - f) sigma_background; both
 * computed on the GPU in FP64 (rfb_slab_rows).  Samples outside stay as
 * they are. */
int fdtd_b200_materials_set_tensor3_slab_smoothed(materials_t *mat, const fdtd_grid_t *g, const double point[3],
                                                  const double normal[3], double thickness, const double eps_r[9]) {
    double m[9];
    if (!point || !normal || !eps_r || !(thickness > 0.0) || rfb_spd3_inverse(eps_r, m) != 0) return -1;
    if (!materials_matches(mat, g)) return -1;
    const double nn = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
    if (!(nn > 0.0)) return -1;
    const double u[3] = {normal[0] / nn, normal[1] / nn, normal[2] / nn};
    const size_t n[3] = {g->nx, g->ny, g->nz};
    size_t lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = ((g->periodic_axes >> a) & 1u) ? 0 : 1;
        hi[a] = n[a];
    }
    const double half = 0.5 * thickness;
    const double reach = 0.5 * ((fabs(u[0]) + fabs(u[1])) + fabs(u[2]));
    /* column k ranges as the staircased slab, widened by the cube's reach */
    const double slack = reach + reach;
    size_t n_in = 0, cap_in = 1024, n_cut = 0, cap_cut = 1024;
    uint64_t *in_keys = malloc(cap_in * sizeof(uint64_t));
    int32_t *cut = malloc(4 * cap_cut * sizeof(int32_t));
    double *cut_bg = NULL, *f = NULL, *rows = NULL;
    int rc = -1, gpu_failed = 0;
    if (!in_keys || !cut) goto out;
    for (size_t i = lo[0]; i < hi[0]; i++)
        for (size_t j = lo[1]; j < hi[1]; j++) {
            size_t ka = lo[2], kb = hi[2];
            if (fabs(u[2]) > 1e-9) {
                const double r0 = u[0] * ((double)i - point[0]) + u[1] * ((double)j - point[1]) - u[2] * point[2];
                double a = (-half - slack - r0) / u[2], b = (half + slack - r0) / u[2];
                if (a > b) { const double t = a; a = b; b = t; }
                a = floor(a) - 1.0;
                b = ceil(b) + 2.0;
                if (a > (double)ka) ka = a >= (double)hi[2] ? hi[2] : (size_t)a;
                if (b < (double)kb) kb = b <= (double)ka ? ka : (size_t)b;
            }
            for (size_t k = ka; k < kb; k++)
                for (int c = 0; c < 3; c++) {
                    double p[3] = {(double)i, (double)j, (double)k};
                    p[c] += 0.5;
                    /* the device's operation order (sphere_frac.cuh) */
                    const double d = (u[0] * (p[0] - point[0]) + u[1] * (p[1] - point[1])) + u[2] * (p[2] - point[2]);
                    const double ad = fabs(d);
                    if (ad - reach > half) continue;
                    if (!component_valid(g, c, i, j, k) || !tensor3_margin_ok(g, i, j, k)) continue;
                    const uint64_t key = (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c;
                    if (ad + reach <= half) {
                        if (n_in == cap_in) {
                            cap_in *= 2;
                            uint64_t *nk2 = realloc(in_keys, cap_in * sizeof(uint64_t));
                            if (!nk2) goto out;
                            in_keys = nk2;
                        }
                        in_keys[n_in++] = key;
                    } else {
                        if (n_cut == cap_cut) {
                            cap_cut *= 2;
                            int32_t *nc = realloc(cut, 4 * cap_cut * sizeof(int32_t));
                            if (!nc) goto out;
                            cut = nc;
                        }
                        cut[4 * n_cut] = (int32_t)i;
                        cut[4 * n_cut + 1] = (int32_t)j;
                        cut[4 * n_cut + 2] = (int32_t)k;
                        cut[4 * n_cut + 3] = c;
                        n_cut++;
                    }
                }
        }
    if (n_cut > (size_t)INT32_MAX) goto out;
    cut_bg = malloc((n_cut + 1) * sizeof(double));
    f = malloc((n_cut + 1) * sizeof(double));
    rows = malloc((3 * n_cut + 1) * sizeof(double));
    if (!cut_bg || !f || !rows) goto out;
    for (size_t q = 0; q < n_cut; q++) {
        const size_t w = fdtd_index(g, (size_t)cut[4 * q], (size_t)cut[4 * q + 1], (size_t)cut[4 * q + 2]);
        cut_bg[q] = mat->table[mat->ids[w]].eps_r;
    }
    if (rfb_slab_rows(point, u, thickness, eps_r, cut, cut_bg, (int)n_cut, f, rows) != 0) {
        gpu_failed = 1;
        goto out;
    }
    if (omap_reserve(&mat->tensor3, n_in + n_cut) != 0) goto out;
    for (size_t q = 0; q < n_in; q++) {
        const int c = (int)(in_keys[q] % 3);
        const double v[4] = {m[3 * c], m[3 * c + 1], m[3 * c + 2], 0.0};
        if (omap_put(&mat->tensor3, in_keys[q], v) != 0) goto out;
    }
    for (size_t q = 0; q < n_cut; q++) {
        if (!(f[q] > 0.0)) continue;
        const size_t w = fdtd_index(g, (size_t)cut[4 * q], (size_t)cut[4 * q + 1], (size_t)cut[4 * q + 2]);
        const double v[4] = {rows[3 * q], rows[3 * q + 1], rows[3 * q + 2],
                             (1.0 - f[q]) * mat->table[mat->ids[w]].sigma};
        if (omap_put(&mat->tensor3, (uint64_t)w * 3 + (uint64_t)cut[4 * q + 3], v) != 0) goto out;
    }
    rc = 0;
out:
    if (rc != 0 && !gpu_failed) rfb_set_error("smoothed slab: out of host memory");
    free(in_keys);
    free(cut);
    free(cut_bg);
    free(f);
    free(rows);
    mat->version++;
    return rc;
}

int fdtd_b200_materials_set_dispersive_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0,
                                           size_t j1, size_t k0, size_t k1, const fdtd_b200_dispersive_t *model) {
    double v[DISP_W];
    if (!model || pack_model(model, v) != 0 || !box_valid(mat, g, i0, i1, j0, j1, k0, k1)) return -1;
    if (omap_reserve(&mat->disp, 3 * (i1 - i0) * (j1 - j0) * (k1 - k0)) != 0) return -1;
    for (size_t i = i0; i < i1; i++)
        for (size_t j = j0; j < j1; j++)
            for (size_t k = k0; k < k1; k++)
                for (int c = 0; c < 3; c++) {
                    if (!component_valid(g, c, i, j, k)) continue;
                    if (omap_put(&mat->disp, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) != 0) return -1;
                }
    mat->version++;
    return 0;
}

int fdtd_b200_materials_get_tensor3(const materials_t *mat, const fdtd_grid_t *g, field_component_t component,
                                     size_t i, size_t j, size_t k, double row[3]) {
    int c = component_number(component);
    if (c < 0 || c > 2 || !row || !materials_matches(mat, g) || !component_valid(g, c, i, j, k)) return -1;
    long long q = omap_find(&mat->tensor3, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c);
    if (q < 0) return 1;
    memcpy(row, mat->tensor3.vals + (size_t)q * 4, 3 * sizeof(double));
    return 0;
}

/* Inverse of a symmetric positive-definite 3x3 matrix (row-major), by the
 * adjugate; -1 when the matrix is not symmetric or not positive definite
 * (leading principal minors). */
int rfb_spd3_inverse(const double e[9], double out[9]) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            if (!isfinite(e[3 * a + b]) || fabs(e[3 * a + b] - e[3 * b + a]) > 1e-12 * (fabs(e[3 * a + b]) + 1.0))
                return -1;
    const double m1 = e[0], m2 = e[0] * e[4] - e[1] * e[3];
    const double det = e[0] * (e[4] * e[8] - e[5] * e[7]) - e[1] * (e[3] * e[8] - e[5] * e[6]) +
                       e[2] * (e[3] * e[7] - e[4] * e[6]);
    if (!(m1 > 0.0 && m2 > 0.0 && det > 0.0)) return -1;
    out[0] = (e[4] * e[8] - e[5] * e[7]) / det;
    out[1] = (e[2] * e[7] - e[1] * e[8]) / det;
    out[2] = (e[1] * e[5] - e[2] * e[4]) / det;
    out[3] = out[1];
    out[4] = (e[0] * e[8] - e[2] * e[6]) / det;
    out[5] = (e[2] * e[3] - e[0] * e[5]) / det;
    out[6] = out[2];
    out[7] = out[5];
    out[8] = (e[0] * e[4] - e[1] * e[3]) / det;
    return 0;
}

int fdtd_b200_materials_set_tensor3_box(materials_t *mat, const fdtd_grid_t *g, size_t i0, size_t i1, size_t j0,
                                        size_t j1, size_t k0, size_t k1, const double eps_r[9]) {
    double m[9];
    if (!eps_r || rfb_spd3_inverse(eps_r, m) != 0) return -1;
    if (!box_valid(mat, g, i0, i1, j0, j1, k0, k1)) return -1;
    for (size_t i = i0; i < i1; i++)
        for (size_t j = j0; j < j1; j++)
            for (size_t k = k0; k < k1; k++)
                for (int c = 0; c < 3; c++) {
                    if (!component_valid(g, c, i, j, k) || !tensor3_margin_ok(g, i, j, k)) return -1;
                    const double v[4] = {m[3 * c], m[3 * c + 1], m[3 * c + 2], 0.0};
                    if (omap_put(&mat->tensor3, (uint64_t)fdtd_index(g, i, j, k) * 3 + (uint64_t)c, v) != 0)
                        return -1;
                }
    mat->version++;
    return 0;
}

/* ADE update record of a dispersive sample (RFB_ADE_NC doubles):
 *   [0] ca  [1] cb  [2] ce  [3] n_poles, then per pole
 *   kind, cj, cjm, aJ, aJm, aE
 * for  E+ = ca E + cb (dA - dB) + ce E- - sum_p (cj J_p + cjm J_p-)
 *      J_p+ = aJ J_p + aJm J_p- + aE (E+ - E_ref),  E_ref = E (Debye) or E- (Lorentz)
 * where - / + denote the previous / next time level.  Derivation: Ampere's
 * law at n+1/2 with the centred Debye update J+ = k J + beta (E+ - E)/dt and
 * the centred Lorentz update J+ = a J + xi J- + g (E+ - E-)/(2 dt) (Taflove &
 * Hagness 3rd ed. sec. 9.4). */
void rfb_ade_record(const double *m, double dt, double dx, double *out) {
    const double e0ei = EPS0 * m[0], sigma = m[1];
    const int np = (int)m[2];
    double kJ[FDTD_B200_MAX_POLES], kJm[FDTD_B200_MAX_POLES], kE[FDTD_B200_MAX_POLES];
    double half_beta = 0.0, quarter_g = 0.0;
    for (int p = 0; p < np; p++) {
        const double *w = m + 3 + 5 * p;
        if ((int)w[0] == FDTD_B200_POLE_DEBYE) {
            double den = 1.0 + dt / (2.0 * w[2]);
            double beta = (EPS0 * w[1] * dt / w[2]) / den;
            kJ[p] = (1.0 - dt / (2.0 * w[2])) / den;
            kJm[p] = 0.0;
            kE[p] = beta / dt;
            half_beta += 0.5 * beta;
        } else {
            double den = 1.0 + w[4] * dt;
            double g = EPS0 * w[1] * w[3] * w[3] * dt * dt / den;
            kJ[p] = (2.0 - w[3] * w[3] * dt * dt) / den;
            kJm[p] = (w[4] * dt - 1.0) / den;
            kE[p] = g / (2.0 * dt);
            quarter_g += 0.25 * g;
        }
    }
    const double A = e0ei + 0.5 * sigma * dt + half_beta + quarter_g;
    memset(out, 0, RFB_ADE_NC * sizeof(double));
    out[0] = (e0ei - 0.5 * sigma * dt + half_beta) / A;
    out[1] = dt / (A * dx);
    out[2] = quarter_g / A;
    out[3] = (double)np;
    for (int p = 0; p < np; p++) {
        double *r = out + 4 + 6 * p;
        r[0] = m[3 + 5 * p];
        r[1] = 0.5 * dt * (1.0 + kJ[p]) / A;
        r[2] = 0.5 * dt * kJm[p] / A;
        r[3] = kJ[p];
        r[4] = kJm[p];
        r[5] = kE[p];
    }
}

/* ---- spheres ------------------------------------------------------------------ */
static int sample_valid(const fdtd_grid_t *g, int c, size_t i, size_t j, size_t k) {
    return component_valid(g, c, i, j, k);
}

int fdtd_b200_materials_add_spheres(materials_t *mat, const fdtd_grid_t *g, const fdtd_b200_sphere_t *spheres,
                                    size_t n_spheres, int smoothing) {
    if (!materials_matches(mat, g) || (!spheres && n_spheres)) return -1;
    const size_t n[3] = {g->nx, g->ny, g->nz};
    {
        /* room in the maps for every sphere's samples at once (a surface
         * shell about 1.3 cells thick, three samples a cell; a dispersive
         * sphere's whole volume), so the maps are not rehashed sphere after
         * sphere as they grow */
        double shell = 0.0, vol = 0.0;
        for (size_t q = 0; q < n_spheres; q++) {
            const fdtd_b200_sphere_t *sp = &spheres[q];
            const double r = sp->radius, cen[3] = {sp->cx, sp->cy, sp->cz};
            if (!isfinite(r) || r <= 0.0 || !isfinite(cen[0]) || !isfinite(cen[1]) || !isfinite(cen[2])) continue;
            /* the part of its box inside the grid bounds both: its volume
             * the dispersive samples, its surface area the sphere's surface
             * inside it (the part of a convex surface inside a box has no
             * more area than the box) */
            double e[3];
            for (int a = 0; a < 3; a++)
                e[a] = fmax(0.0, fmin(cen[a] + r + 2.0, (double)n[a]) - fmax(cen[a] - r - 2.0, 0.0) + 1.0);
            const double box_vol = e[0] * e[1] * e[2], box_area = 2.0 * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0]);
            if (sp->model)
                vol += 3.0 * fmin((4.0 / 3.0) * M_PI * (r + 1.0) * (r + 1.0) * (r + 1.0), box_vol);
            else
                shell += 3.0 * 1.3 * fmin(4.0 * M_PI * (r + 1.0) * (r + 1.0), box_area);
        }
        const double cap = 3.0 * (double)mat->total;
        omap_t *dst = smoothing == 2 ? &mat->tensor3 : &mat->scalar;
        if (omap_reserve(dst, (size_t)fmin(shell, cap)) != 0 || omap_reserve(&mat->disp, (size_t)fmin(vol, cap)) != 0) {
            rfb_set_error("out of host memory rasterising spheres");
            return -1;
        }
    }
    for (size_t q = 0; q < n_spheres; q++) {
        const fdtd_b200_sphere_t *sp = &spheres[q];
        if (!isfinite(sp->cx) || !isfinite(sp->cy) || !isfinite(sp->cz) || !isfinite(sp->radius) || sp->radius <= 0.0)
            return -1;
        double dmodel[DISP_W];
        material_id_t sid = 0;
        if (sp->model) {
            if (pack_model(sp->model, dmodel) != 0) return -1;
        } else if (materials_register(mat, sp->eps_r, sp->sigma, &sid) != 0) {
            return -1;
        }
        const double cen[3] = {sp->cx, sp->cy, sp->cz};
        long lo[3], hi[3];
        for (int a = 0; a < 3; a++) {
            lo[a] = (long)floor(cen[a] - sp->radius) - 2;
            hi[a] = (long)ceil(cen[a] + sp->radius) + 2;
            if (lo[a] < 0) lo[a] = 0;
            if (hi[a] > (long)n[a]) hi[a] = (long)n[a];
        }
        if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) continue;
        const int ni = (int)(hi[0] - lo[0] + 1), nj = (int)(hi[1] - lo[1] + 1), nk = (int)(hi[2] - lo[2] + 1);
        const size_t ncell = (size_t)ni * nj * nk;
        /* smoothing 2 (full tensor) on a plain dielectric: fractions and the
         * rows of the smoothed inverse permittivity against each cell's
         * table material, from the GPU; otherwise fractions and squared
         * normal components */
        const int full = smoothing == 2 && !sp->model;
        double *f = malloc(3 * ncell * sizeof(double)), *n2 = malloc((full ? 9 : 3) * ncell * sizeof(double));
        double *ebg = full ? malloc(ncell * sizeof(double)) : NULL;
        int frc = !f || !n2 || (full && !ebg);
        if (!frc && full) {
            for (int di = 0; di < ni; di++)
                for (int dj = 0; dj < nj; dj++)
                    for (int dk = 0; dk < nk; dk++)
                        ebg[((size_t)di * nj + (size_t)dj) * nk + (size_t)dk] =
                            mat->table[mat->ids[fdtd_index(g, (size_t)(lo[0] + di), (size_t)(lo[1] + dj),
                                                            (size_t)(lo[2] + dk))]].eps_r;
            frc = rfb_sphere_rows(cen, sp->radius, sp->eps_r, (int)lo[0], (int)lo[1], (int)lo[2], ni, nj, nk, ebg, f,
                                  n2);
        } else if (!frc) {
            frc = rfb_sphere_fractions(cen, sp->radius, (int)lo[0], (int)lo[1], (int)lo[2], ni, nj, nk, f, n2);
        }
        free(ebg);
        if (frc) {
            free(f);
            free(n2);
            return -1;
        }
        {
            /* room for this sphere's surface samples in the map they go to,
             * reserved once instead of grown through every power of two */
            size_t cut = 0;
            if (sp->model)
                for (size_t q3 = 0; q3 < 3 * ncell; q3++) cut += f[q3] >= 0.5;
            else
                for (size_t q3 = 0; q3 < 3 * ncell; q3++) cut += f[q3] > 0.0 && f[q3] < 1.0;
            omap_t *dst = sp->model ? &mat->disp : (full ? &mat->tensor3 : &mat->scalar);
            if (omap_reserve(dst, cut) != 0) goto oom;
        }
        for (int di = 0; di < ni; di++)
            for (int dj = 0; dj < nj; dj++)
                for (int dk = 0; dk < nk; dk++) {
                    const size_t i = (size_t)(lo[0] + di), j = (size_t)(lo[1] + dj), k = (size_t)(lo[2] + dk);
                    const size_t cell = ((size_t)di * nj + (size_t)dj) * nk + (size_t)dk;
                    const double *fc = f + 3 * cell, *nc = n2 + (full ? 9 : 3) * cell;
                    if (fc[0] <= 0.0 && fc[1] <= 0.0 && fc[2] <= 0.0) continue; /* outside the sphere */
                    int valid[3] = {1, 1, 1};  /* every sample of a cell below the last planes */
                    if (i + 1 >= n[0] || j + 1 >= n[1] || k + 1 >= n[2])
                        for (int c = 0; c < 3; c++) valid[c] = sample_valid(g, c, i, j, k);
                    const size_t w = fdtd_index(g, i, j, k);
                    if (fc[0] == 1.0 && fc[1] == 1.0 && fc[2] == 1.0 && valid[0] && valid[1] && valid[2]) {
                        if (mat->touched[w]) {
                            for (int c = 0; c < 3; c++) {
                                omap_del(&mat->scalar, (uint64_t)w * 3 + (uint64_t)c);
                                omap_del(&mat->disp, (uint64_t)w * 3 + (uint64_t)c);
                                omap_del(&mat->tensor3, (uint64_t)w * 3 + (uint64_t)c);
                            }
                            for (int c = 0; c < 2; c++) omap_del(&mat->tensor, (uint64_t)w * 3 + (uint64_t)c);
                        }
                        if (sp->model) {
                            for (int c = 0; c < 3; c++)
                                if (omap_put(&mat->disp, (uint64_t)w * 3 + (uint64_t)c, dmodel) != 0) goto oom;
                        } else {
                            mat->ids[w] = sid;
                        }
                        continue;
                    }
                    for (int c = 0; c < 3; c++) {
                        if (!valid[c] || fc[c] <= 0.0) continue;
                        const uint64_t key = (uint64_t)w * 3 + (uint64_t)c;
                        if (sp->model) {
                            if (fc[c] >= 0.5 && omap_put(&mat->disp, key, dmodel) != 0) goto oom;
                            continue;
                        }
                        double eps_c, sig_c;
                        if (full && fc[c] < 1.0) {
                            /* the row of the smoothed tensor where the 3x3
                             * update may run, else its diagonal */
                            const double *row = nc + 3 * c;
                            const double eb = mat->table[mat->ids[w]].eps_r, sb = mat->table[mat->ids[w]].sigma;
                            sig_c = fc[c] * sp->sigma + (1.0 - fc[c]) * sb;
                            if (tensor3_margin_ok(g, i, j, k)) {
                                const double v[4] = {row[0], row[1], row[2], sig_c};
                                if (omap_put(&mat->tensor3, key, v) != 0) goto oom;
                                omap_del(&mat->scalar, key);
                                omap_del(&mat->disp, key);
                                if (c < 2) omap_del(&mat->tensor, key);
                                continue;
                            }
                            eps_c = row[c] > 0.0 ? 1.0 / row[c] : eb;
                        } else if (!smoothing || fc[c] == 1.0) {
                            if (fc[c] < 0.5) continue;
                            eps_c = sp->eps_r;
                            sig_c = sp->sigma;
                        } else {
                            /* diagonal of the smoothed inverse permittivity */
                            const double eb = mat->table[mat->ids[w]].eps_r, sb = mat->table[mat->ids[w]].sigma;
                            const double mean = fc[c] * sp->eps_r + (1.0 - fc[c]) * eb;
                            const double minv = fc[c] / sp->eps_r + (1.0 - fc[c]) / eb;
                            const double inv = nc[c] * minv + (1.0 - nc[c]) / mean;
                            eps_c = 1.0 / inv;
                            sig_c = fc[c] * sp->sigma + (1.0 - fc[c]) * sb;
                        }
                        material_coeff_t co;
                        if (make_coeff(mat, eps_c, sig_c, &co) != 0) goto fail;
                        double v[2] = {co.Ca, co.Cb};
                        if (omap_put(&mat->scalar, key, v) != 0) goto oom;
                        omap_del(&mat->disp, key);
                        omap_del(&mat->tensor3, key);
                    }
                }
        free(f);
        free(n2);
        mat->version++;
        continue;
    oom:
        rfb_set_error("out of host memory rasterising spheres");
    fail:
        free(f);
        free(n2);
        mat->version++;
        return -1;
    }
    return 0;
}

/* ---- heightmap world -> materials --------------------------------------------
 * rfsyn describes terrain as a heightmap world (engine/world/world.c:49-135):
 * column (i, j) holds solid material column_materials[i ny + j] up to height
 * h; cell (i, j, k) has the solid fraction f = clamp(h/dx - k, 0, 1) (height
 * clipped to the domain, world.c:23-28, :94-95), its bulk id is the solid
 * where f >= 0.5 and air elsewhere (:98), and a cell with 0 < f < 1 carries
 * the surface normal (-gx, -gy, 1) / |.| from central differences of the
 * heights, one-sided at the edges (:30-47).  rfsyn never applies a world to
 * its FDTD grid (cli/main.c:325-333); this maps it onto the materials: bulk
 * ids per column run, and with smoothing, every E component of a mixed cell
 * gets the diagonal of the smoothed inverse permittivity used for spheres,
 *   1/eps_c = n_c^2 (f/eps_s + (1-f)/eps_a) + (1 - n_c^2) / (f eps_s + (1-f) eps_a),
 *   sigma_c = f sigma_s + (1 - f) sigma_a. */
static double hm_fraction(double hc, size_t k) {
    double f = hc - (double)k;
    if (f <= 0.0) return 0.0;
    if (f >= 1.0) return 1.0;
    return f;
}

static int hm_normal(const fdtd_b200_heightmap_t *hm, size_t i, size_t j, double n[3]) {
    const size_t il = i ? i - 1 : i, ir = i + 1 < hm->nx ? i + 1 : i;
    const size_t jl = j ? j - 1 : j, jr = j + 1 < hm->ny ? j + 1 : j;
    double gx = 0.0, gy = 0.0;
    if (ir != il) gx = (hm->heights_m[ir * hm->ny + j] - hm->heights_m[il * hm->ny + j]) / ((double)(ir - il) * hm->dx);
    if (jr != jl) gy = (hm->heights_m[i * hm->ny + jr] - hm->heights_m[i * hm->ny + jl]) / ((double)(jr - jl) * hm->dx);
    const double len = hypot(hypot(gx, gy), 1.0);
    if (!isfinite(len) || len <= 0.0) return -1;
    n[0] = -gx / len;
    n[1] = -gy / len;
    n[2] = 1.0 / len;
    return 0;
}

int fdtd_b200_materials_apply_heightmap(materials_t *mat, const fdtd_grid_t *g, const fdtd_b200_heightmap_t *hm,
                                        const fdtd_b200_medium_t *media, size_t n_media, int smoothing,
                                        size_t *mixed_out) {
    if (mixed_out) *mixed_out = 0;
    if (!materials_matches(mat, g) || !hm || !hm->heights_m || !hm->column_materials || !media) {
        rfb_set_error("heightmap: NULL argument or materials of another grid");
        return -1;
    }
    if (hm->nx != g->nx || hm->ny != g->ny || hm->nz != g->nz || !isfinite(hm->dx) || hm->dx <= 0.0 ||
        fabs(hm->dx - g->dx) > 1e-12 * g->dx) {
        rfb_set_error("heightmap: its cells must be the grid's (nx, ny, nz, dx)");
        return -1;
    }
    if ((size_t)hm->air_id >= n_media) {
        rfb_set_error("heightmap: no medium for the air id %d", (int)hm->air_id);
        return -1;
    }
    const size_t cols = hm->nx * hm->ny;
    const double top = (double)hm->nz * hm->dx;
    for (size_t q = 0; q < cols; q++) {
        const double h = hm->heights_m[q];
        if (!isfinite(h) || h < 0.0 || h > top || (h > 0.0 && hm->column_materials[q] == hm->air_id) ||
            (size_t)hm->column_materials[q] >= n_media) {
            rfb_set_error("heightmap: column %zu has an invalid height or material", q);
            return -1;
        }
    }
    /* media -> material ids, registered on first use */
    int id_of[256];
    for (int q = 0; q < 256; q++) id_of[q] = -1;
    for (size_t q = 0; q <= cols; q++) {
        const uint8_t w = q < cols ? hm->column_materials[q] : hm->air_id;
        if (id_of[w] >= 0) continue;
        material_id_t id;
        if (materials_register(mat, media[w].eps_r, media[w].sigma, &id) != 0) {
            rfb_set_error("heightmap: medium %d rejected (eps_r >= 1, sigma >= 0, at most 256 materials)", (int)w);
            return -1;
        }
        id_of[w] = id;
    }
    /* bulk ids: the solid run below, air above (box assignment clears any
     * description the cells had) */
    for (size_t i = 0; i < hm->nx; i++)
        for (size_t j = 0; j < hm->ny; j++) {
            const size_t q = i * hm->ny + j;
            const double hc = fmin(hm->heights_m[q] / hm->dx, (double)hm->nz);
            size_t kb = 0;
            while (kb < hm->nz && hm_fraction(hc, kb) >= 0.5) kb++;
            if (kb > 0 &&
                materials_assign_box(mat, g, i, i + 1, j, j + 1, 0, kb, (material_id_t)id_of[hm->column_materials[q]]))
                return -1;
            if (kb < hm->nz &&
                materials_assign_box(mat, g, i, i + 1, j, j + 1, kb, hm->nz, (material_id_t)id_of[hm->air_id]))
                return -1;
        }
    /* mixed cells */
    size_t mixed = 0;
    const fdtd_b200_medium_t air = media[hm->air_id];
    for (size_t i = 0; i < hm->nx; i++)
        for (size_t j = 0; j < hm->ny; j++) {
            const size_t q = i * hm->ny + j;
            const double hc = fmin(hm->heights_m[q] / hm->dx, (double)hm->nz);
            const fdtd_b200_medium_t sol = media[hm->column_materials[q]];
            for (size_t k = 0; k < hm->nz; k++) {
                const double f = hm_fraction(hc, k);
                if (!(f > 0.0 && f < 1.0)) continue;
                mixed++;
                if (!smoothing) continue;
                double n[3];
                if (hm_normal(hm, i, j, n) != 0) {
                    rfb_set_error("heightmap: no surface normal at column %zu", q);
                    return -1;
                }
                const size_t w = fdtd_index(g, i, j, k);
                for (int c = 0; c < 3; c++) {
                    if (!sample_valid(g, c, i, j, k)) continue;
                    const double n2 = n[c] * n[c];
                    const double mean = f * sol.eps_r + (1.0 - f) * air.eps_r;
                    const double minv = f / sol.eps_r + (1.0 - f) / air.eps_r;
                    const double inv = n2 * minv + (1.0 - n2) / mean;
                    material_coeff_t co;
                    if (make_coeff(mat, 1.0 / inv, f * sol.sigma + (1.0 - f) * air.sigma, &co) != 0) {
                        rfb_set_error("heightmap: smoothed medium out of range");
                        return -1;
                    }
                    const double v[2] = {co.Ca, co.Cb};
                    if (omap_put(&mat->scalar, (uint64_t)w * 3 + (uint64_t)c, v) != 0) {
                        rfb_set_error("out of host memory mapping the heightmap");
                        return -1;
                    }
                }
            }
        }
    mat->version++;
    if (mixed_out) *mixed_out = mixed;
    return 0;
}

/* Symmetric Ex/Ey coupling weight of two tensor edges (materials.c:836-845):
 * 0.25 * rho * sqrt(m11_x) * sqrt(m11_y) with rho the mean normalised
 * off-diagonal correlation; evaluated in the same order for bit parity. */
static double pair_weight(const double *ex, const double *ey) {
    double rx = (ex[1] / sqrt(ex[0])) / sqrt(ex[2]);
    double ry = (ey[1] / sqrt(ey[0])) / sqrt(ey[2]);
    double rho = 0.5 * rx + 0.5 * ry;
    return (0.25 * rho * sqrt(ex[0])) * sqrt(ey[0]);
}

static size_t prev_q(size_t q, size_t n) { return q == 0 ? n - 1 : q - 1; }
static size_t next_q(size_t q, size_t n) { return q + 1 == n ? 0 : q + 1; }

/* Component c of canonical cell (i,j,k) is swept by rfsyn's E loops
 * (materials.c:915-1059). */
int rfb_e_swept(const fdtd_grid_t *g, int c, size_t i, size_t j, size_t k) {
    size_t i0 = (g->periodic_axes & 1u) ? 0 : 1, j0 = (g->periodic_axes & 2u) ? 0 : 1,
           k0 = (g->periodic_axes & 4u) ? 0 : 1;
    if (i >= g->nx || j >= g->ny || k >= g->nz) return 0;
    if (c != 0 && i < i0) return 0;
    if (c != 1 && j < j0) return 0;
    if (c != 2 && k < k0) return 0;
    return 1;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

void rfb_scene_build_free(rfb_scene_build_t *b) {
    if (!b) return;
    free(b->codes); free(b->cell_ijk); free(b->kind); free(b->ca); free(b->cb);
    free(b->tix); free(b->src); free(b->aix);
    free(b->t_m11); free(b->t_scale); free(b->t_w); free(b->t_main); free(b->t_nq); free(b->t_uv); free(b->t_sign);
    free(b->ade_c);
    free(b->t3);
    memset(b, 0, sizeof(*b));
}


/* Record dedupe of 3x3 samples: an open-addressing table over the records
 * built so far, keyed by their five values' bits. */
typedef struct {
    int32_t *slot;  /* record index + 1, 0 empty */
    size_t mask;
} t3_dedupe_t;

static uint64_t t3_hash(const double *r) {
    uint64_t h = 1469598103934665603ull;
    for (int q = 0; q < 5; q++) {
        uint64_t b;
        memcpy(&b, &r[q], sizeof b);
        h = (h ^ b) * 1099511628211ull;
        h ^= h >> 29;
    }
    return h;
}

/* The index of the record just written at recs[5 * *n]: an earlier equal
 * record's, or *n (then *n grows). */
static int32_t t3_record_index(t3_dedupe_t *d, double *recs, size_t *n) {
    const double *r = recs + 5 * *n;
    for (size_t h = t3_hash(r) & d->mask;; h = (h + 1) & d->mask) {
        const int32_t s = d->slot[h];
        if (!s) {
            d->slot[h] = (int32_t)(*n + 1);
            return (int32_t)(*n)++;
        }
        if (!memcmp(recs + 5 * (size_t)(s - 1), r, 5 * sizeof(double))) return s - 1;
    }
}

/* Pass 1 of the image's list entries over list cells [q0, q1): cell
 * coordinates, the scalar (Ca, Cb) of every entry and its kind -- COPY for
 * components the sweep does not update, TENSOR3 (map slot in tix), TENSOR,
 * ADE (map slot in aix) or SCALAR, in that precedence.  It only reads the
 * maps, so ranges run on several threads. */
typedef struct {
    const materials_t *mat;
    const fdtd_grid_t *g;
    const uint64_t *cells;
    rfb_scene_build_t *out;
    size_t q0, q1;
} image_range_t;

static void *image_pass1_range(void *arg) {
    const image_range_t *p = arg;
    const materials_t *mat = p->mat;
    const fdtd_grid_t *g = p->g;
    rfb_scene_build_t *out = p->out;
    const size_t nz1 = g->nz + 1;
    for (size_t q = p->q0; q < p->q1; q++) {
        const size_t idx = (size_t)p->cells[q];
        const size_t k = idx % nz1, row = idx / nz1, j = row % (g->ny + 1), i = row / (g->ny + 1);
        out->cell_ijk[3 * q] = (int32_t)i;
        out->cell_ijk[3 * q + 1] = (int32_t)j;
        out->cell_ijk[3 * q + 2] = (int32_t)k;
        for (int c = 0; c < 3; c++) {
            const size_t e = 3 * q + (size_t)c;
            out->tix[e] = -1;
            out->src[e] = -1;
            out->aix[e] = -1;
            const material_coeff_t co = lookup(mat, idx, c);
            out->ca[e] = co.Ca;
            out->cb[e] = co.Cb;
            if (!rfb_e_swept(g, c, i, j, k)) {
                out->kind[e] = RFB_LK_COPY;
                continue;
            }
            const long t3 = omap_find(&mat->tensor3, (uint64_t)idx * 3 + (uint64_t)c);
            if (t3 >= 0) {
                out->kind[e] = RFB_LK_TENSOR3;
                out->tix[e] = (int32_t)t3;
                continue;
            }
            if (c < 2 && tensor_at(mat, idx, c)) {
                out->kind[e] = RFB_LK_TENSOR;
                continue;
            }
            const long dm = omap_find(&mat->disp, (uint64_t)idx * 3 + (uint64_t)c);
            if (dm < 0) {
                out->kind[e] = RFB_LK_SCALAR;
            } else {
                out->kind[e] = RFB_LK_ADE;
                out->aix[e] = (int32_t)dm;
            }
        }
    }
    return NULL;
}

/* Pass 1 over all nc list cells on up to 16 threads (the online cores;
 * one for short lists); a thread that cannot start leaves its range to
 * the calling thread. */
static void image_pass1(const materials_t *mat, const fdtd_grid_t *g, const uint64_t *cells, size_t nc,
                        rfb_scene_build_t *out) {
    enum { MAX_T = 16 };
    long nt = sysconf(_SC_NPROCESSORS_ONLN);
    if (nt > MAX_T) nt = MAX_T;
    if (nt > (long)(nc / 16384) + 1) nt = (long)(nc / 16384) + 1;
    if (nt < 1) nt = 1;
    image_range_t job[MAX_T];
    pthread_t th[MAX_T];
    int started[MAX_T] = {0};
    for (long t = 0; t < nt; t++)
        job[t] = (image_range_t){mat, g, cells, out, nc * (size_t)t / (size_t)nt, nc * (size_t)(t + 1) / (size_t)nt};
    for (long t = 1; t < nt; t++) started[t] = pthread_create(&th[t], NULL, image_pass1_range, &job[t]) == 0;
    image_pass1_range(&job[0]);
    for (long t = 1; t < nt; t++) {
        if (started[t]) pthread_join(th[t], NULL);
        else image_pass1_range(&job[t]);
    }
}

int materials_build_image(const materials_t *mat, const fdtd_grid_t *g, size_t n_extra, const rfb_extra_cell_t *extra,
                          rfb_scene_build_t *out) {
    memset(out, 0, sizeof(*out));
    if (!materials_matches(mat, g)) {
        rfb_set_error("materials do not match the grid");
        return -1;
    }
    t3_dedupe_t t3d = {NULL, 0};
    const size_t nz1 = g->nz + 1;
    /* 1. cells on the interface list (padded linear index) */
    size_t cap = mat->scalar.count + mat->tensor.count + mat->disp.count + mat->tensor3.count + n_extra;
    int id255 = 0;
    if (mat->table_count == MATERIAL_LIMIT) {
        /* code 255 marks list cells: cells of material 255 go to the list too */
        for (size_t q = 0; q < mat->total; q++)
            if (mat->ids[q] == 255) { id255 = 1; cap++; }
    }
    uint64_t *cells = malloc((cap ? cap : 1) * sizeof(uint64_t));
    if (!cells) goto oom;
    size_t nc = 0;
    for (size_t q = 0; q < mat->scalar.cap; q++)
        if (mat->scalar.keys[q] != OMAP_EMPTY) cells[nc++] = mat->scalar.keys[q] / 3;
    for (size_t q = 0; q < mat->tensor.cap; q++)
        if (mat->tensor.keys[q] != OMAP_EMPTY) cells[nc++] = mat->tensor.keys[q] / 3;
    for (size_t q = 0; q < mat->disp.cap; q++)
        if (mat->disp.keys[q] != OMAP_EMPTY) cells[nc++] = mat->disp.keys[q] / 3;
    for (size_t q = 0; q < mat->tensor3.cap; q++)
        if (mat->tensor3.keys[q] != OMAP_EMPTY) cells[nc++] = mat->tensor3.keys[q] / 3;
    for (size_t q = 0; q < n_extra; q++)
        cells[nc++] = ((uint64_t)extra[q].i * (g->ny + 1) + (uint64_t)extra[q].j) * nz1 + (uint64_t)extra[q].k;
    if (id255)
        for (size_t q = 0; q < mat->total; q++)
            if (mat->ids[q] == 255) cells[nc++] = q;
    /* sorted, unique: by a sort for few candidates, else through a byte per
     * cell scanned in order (linear in the grid, no n log n sort of the
     * three keys per override) */
    uint8_t *mask = nc > 4096 ? calloc(mat->total, 1) : NULL;
    if (mask) {
        for (size_t q = 0; q < nc; q++) mask[cells[q]] = 1;
        size_t nu = 0;
        const size_t words = mat->total / 8;
        for (size_t w8 = 0; w8 < words; w8++) {
            uint64_t v;
            memcpy(&v, mask + 8 * w8, 8);
            if (!v) continue;
            for (size_t b = 0; b < 8; b++)
                if (mask[8 * w8 + b]) cells[nu++] = 8 * w8 + b;
        }
        for (size_t q = 8 * words; q < mat->total; q++)
            if (mask[q]) cells[nu++] = q;
        nc = nu;
        free(mask);
    } else {
        qsort(cells, nc, sizeof(uint64_t), cmp_u64);
        size_t nu = 0;
        for (size_t q = 0; q < nc; q++)
            if (nu == 0 || cells[nu - 1] != cells[q]) cells[nu++] = cells[q];
        nc = nu;
    }

    /* 2. code volume: needed when any cell uses a non-vacuum material or the
     *    list is long; otherwise the engine works code-less */
    int uniform = 1;
    for (size_t q = 0; q < mat->total && uniform; q++)
        if (mat->ids[q] != 0) uniform = 0;
    if (!uniform) {
        out->codes = malloc(mat->total);
        if (!out->codes) goto oom;
        memcpy(out->codes, mat->ids, mat->total);
        for (size_t q = 0; q < nc; q++) out->codes[cells[q]] = 255;
    }
    rfb_scene_image_t *img = &out->img;
    img->codes = out->codes;
    img->table_count = (int)mat->table_count;
    for (size_t q = 0; q < mat->table_count; q++) {
        img->table_ca[q] = mat->table[q].coeff.Ca;
        img->table_cb[q] = mat->table[q].coeff.Cb;
    }
    /* 3. list entries */
    const size_t ne = 3 * nc;
    out->cell_ijk = malloc((3 * nc + 1) * sizeof(int32_t));
    out->kind = malloc(ne + 1);
    out->ca = malloc((ne + 1) * sizeof(double));
    out->cb = malloc((ne + 1) * sizeof(double));
    out->tix = malloc((ne + 1) * sizeof(int32_t));
    out->src = malloc((ne + 1) * sizeof(int32_t));
    out->aix = malloc((ne + 1) * sizeof(int32_t));
    size_t tcap = mat->tensor.count + 1;
    out->t_m11 = malloc(tcap * sizeof(double));
    out->t_scale = malloc(tcap * sizeof(double));
    out->t_w = calloc(4 * tcap, sizeof(double));
    out->t_main = calloc(4 * tcap, sizeof(int32_t));
    out->t_nq = calloc(tcap, sizeof(int32_t));
    out->t_uv = calloc(16 * tcap, sizeof(int32_t));
    out->t_sign = calloc(tcap, sizeof(int32_t));
    out->t3 = malloc((5 * mat->tensor3.count + 5) * sizeof(double));
    size_t t3cap = 2;
    while (t3cap < 2 * mat->tensor3.count + 2) t3cap *= 2;
    t3d.slot = calloc(t3cap, sizeof(int32_t));
    t3d.mask = t3cap - 1;
    if (!out->cell_ijk || !out->kind || !out->ca || !out->cb || !out->tix || !out->src || !out->aix || !out->t_m11 ||
        !out->t_scale || !out->t_w || !out->t_main || !out->t_nq || !out->t_uv || !out->t_sign || !out->t3 || !t3d.slot)
        goto oom;
    size_t nt = 0, nt3 = 0;
    /* ADE records, deduplicated by model */
    size_t n_models = 0, model_cap = 16;
    double *models = malloc(model_cap * DISP_W * sizeof(double));
    double *records = malloc(model_cap * RFB_ADE_NC * sizeof(double));
    out->ade_c = records; /* owned by the image from here on */
    if (!models || !records) {
        free(models);
        goto oom;
    }
    /* pass 1, in parallel over ranges of list cells: coordinates, scalar
     * coefficients and each entry's kind; a 3x3 or dispersive sample keeps
     * its map slot in tix / aix for pass 2 */
    if (mat->tensor3.cap >= (size_t)INT32_MAX || mat->disp.cap >= (size_t)INT32_MAX) {
        free(models);
        goto oom;
    }
    image_pass1(mat, g, cells, nc, out);
    /* pass 2, in entry order: the records, numbered as the entries meet
     * them (3x3 records deduplicated, ADE models, 2x2 tensor records); the
     * last 3x3 record of each component and the last model are tried
     * first (neighbouring cells of a uniform region share them) */
    int32_t last3[3] = {-1, -1, -1};
    size_t last_model = 0;
    for (size_t q = 0; q < nc; q++) {
        const size_t idx = (size_t)cells[q];
        const size_t i = (size_t)out->cell_ijk[3 * q], j = (size_t)out->cell_ijk[3 * q + 1],
                     k = (size_t)out->cell_ijk[3 * q + 2];
        for (int c = 0; c < 3; c++) {
            const size_t e = 3 * q + (size_t)c;
            const uint8_t kind = out->kind[e];
            if (kind == RFB_LK_TENSOR3) {
                /* full 3x3 sample: its row of eps_r^-1, then the update's
                 * coefficients E+ = ca E + s value with the loss of sigma
                 * taken at the component's own permittivity 1/m_cc, as
                 * make_coeff takes it for a scalar sample:
                 * s = dt/(eps0 dx) / (1 + loss), ca = (1 - loss)/(1 + loss),
                 * loss = sigma dt / (2 eps0 / m_cc); lossless: s = dt/(eps0
                 * dx), ca = 1 */
                const double *row = mat->tensor3.vals + (size_t)out->tix[e] * 4;
                double *rec = out->t3 + 5 * nt3;
                rec[0] = row[0];
                rec[1] = row[1];
                rec[2] = row[2];
                const double loss = (row[3] * mat->dt) / (2.0 * (EPS0 / row[c]));
                rec[3] = (mat->dt / (EPS0 * mat->dx)) / (1.0 + loss);
                rec[4] = (1.0 - loss) / (1.0 + loss);
                /* samples with the same record share it (a uniform anisotropic
                 * region is one record per component): fewer record bytes
                 * for the list kernels to read */
                if (last3[c] >= 0 && !memcmp(out->t3 + 5 * (size_t)last3[c], rec, 5 * sizeof(double)))
                    out->tix[e] = last3[c];
                else
                    out->tix[e] = last3[c] = t3_record_index(&t3d, out->t3, &nt3);
                continue;
            }
            if (kind == RFB_LK_ADE) {
                const double *mv = mat->disp.vals + (size_t)out->aix[e] * DISP_W;
                size_t r = 0;
                if (last_model < n_models && !memcmp(models + last_model * DISP_W, mv, DISP_W * sizeof(double)))
                    r = last_model;
                else
                    while (r < n_models && memcmp(models + r * DISP_W, mv, DISP_W * sizeof(double)) != 0) r++;
                last_model = r;
                if (r == n_models) {
                    if (n_models == model_cap) {
                        model_cap *= 2;
                        double *nm = realloc(models, model_cap * DISP_W * sizeof(double));
                        if (nm) models = nm;
                        double *nr = realloc(records, model_cap * RFB_ADE_NC * sizeof(double));
                        if (nr) records = out->ade_c = nr;
                        if (!nm || !nr) {
                            free(models);
                            goto oom;
                        }
                    }
                    memcpy(models + r * DISP_W, mv, DISP_W * sizeof(double));
                    rfb_ade_record(mv, mat->dt, mat->dx, records + r * RFB_ADE_NC);
                    n_models++;
                }
                out->aix[e] = (int32_t)r;
                continue;
            }
            if (kind != RFB_LK_TENSOR) continue;
            const double *t = tensor_at(mat, idx, c);
            /* tensor edge record (materials.c:847-903) */
            out->kind[e] = RFB_LK_TENSOR;
            out->tix[e] = (int32_t)nt;
            out->t_scale[nt] = t[3];
            int32_t *mn = out->t_main + 4 * nt;
            int nq = 0;
            if (c == 0) {
                size_t ip = next_q(i, g->nx), jm = prev_q(j, g->ny);
                out->t_m11[nt] = t[0];
                mn[0] = (int32_t)i; mn[1] = (int32_t)j; mn[2] = (int32_t)i; mn[3] = (int32_t)jm;
                size_t ni[4] = {i, ip, i, ip}, nj[4] = {j, j, jm, jm};
                out->t_sign[nt] = -1;
                for (int s = 0; s < 4; s++) {
                    const double *o = tensor_at(mat, fdtd_index(g, ni[s], nj[s], k), 1);
                    if (!o) continue;
                    size_t um = prev_q(ni[s], g->nx);
                    out->t_w[4 * nt + nq] = pair_weight(t, o);
                    int32_t *uv = out->t_uv + 16 * nt + 4 * nq;
                    uv[0] = (int32_t)ni[s]; uv[1] = (int32_t)nj[s]; uv[2] = (int32_t)um; uv[3] = (int32_t)nj[s];
                    nq++;
                }
            } else {
                size_t im = prev_q(i, g->nx), jp = next_q(j, g->ny);
                out->t_m11[nt] = -t[0];
                mn[0] = (int32_t)i; mn[1] = (int32_t)j; mn[2] = (int32_t)im; mn[3] = (int32_t)j;
                size_t ni[4] = {i, im, i, im}, nj[4] = {j, j, jp, jp};
                out->t_sign[nt] = 1;
                for (int s = 0; s < 4; s++) {
                    const double *o = tensor_at(mat, fdtd_index(g, ni[s], nj[s], k), 0);
                    if (!o) continue;
                    size_t vm = prev_q(nj[s], g->ny);
                    out->t_w[4 * nt + nq] = pair_weight(o, t);
                    int32_t *uv = out->t_uv + 16 * nt + 4 * nq;
                    uv[0] = (int32_t)ni[s]; uv[1] = (int32_t)nj[s]; uv[2] = (int32_t)ni[s]; uv[3] = (int32_t)vm;
                    nq++;
                }
            }
            out->t_nq[nt] = nq;
            nt++;
        }
    }
    /* sources attached to extra cells */
    for (size_t q = 0; q < n_extra; q++) {
        if (extra[q].component < 0 || extra[q].slot < 0) continue;
        uint64_t key = ((uint64_t)extra[q].i * (g->ny + 1) + (uint64_t)extra[q].j) * nz1 + (uint64_t)extra[q].k;
        uint64_t *hit = bsearch(&key, cells, nc, sizeof(uint64_t), cmp_u64);
        if (!hit) continue;
        size_t e = 3 * (size_t)(hit - cells) + (size_t)extra[q].component;
        if (out->src[e] >= 0) {
            rfb_set_error("two sources on the same field sample");
            free(models);
            free(cells);
            free(t3d.slot);
            rfb_scene_build_free(out);
            return -1;
        }
        out->src[e] = extra[q].slot;
    }
    free(cells);
    free(models);
    img->n_ade = n_models;
    img->ade_c = records;
    img->n_cells = nc;
    img->cell_ijk = out->cell_ijk;
    img->kind = out->kind;
    img->ca = out->ca;
    img->cb = out->cb;
    img->tix = out->tix;
    img->src = out->src;
    img->aix = out->aix;
    img->n_tensors = nt;
    img->n_t3 = nt3;
    img->t3 = out->t3;
    img->t_m11 = out->t_m11;
    img->t_scale = out->t_scale;
    img->t_main = out->t_main;
    img->t_nq = out->t_nq;
    img->t_w = out->t_w;
    img->t_uv = out->t_uv;
    img->t_sign = out->t_sign;
    free(t3d.slot);
    return 0;
oom:
    free(cells);
    free(t3d.slot);
    rfb_scene_build_free(out);
    rfb_set_error("out of host memory building the scene image");
    return -1;
}

rfb_scene_dev_t *materials_device(const materials_t *cmat, const fdtd_grid_t *g) {
    materials_t *mat = (materials_t *)cmat;
    if (mat->dev && mat->dev_version == mat->version && mat->dev_periodic == g->periodic_axes) return mat->dev;
    rfb_scene_dev_destroy(mat->dev);
    mat->dev = NULL;
    rfb_scene_build_t b;
    if (materials_build_image(mat, g, 0, NULL, &b) != 0) return NULL;
    rfb_geom_t geom;
    rfb_geom_from_grid(g, &geom);
    mat->dev = rfb_scene_dev_create(&geom, &b.img);
    rfb_scene_build_free(&b);
    mat->dev_version = mat->version;
    mat->dev_periodic = g->periodic_axes;
    return mat->dev;
}

rfb_fields_t *rfb_grid_device(fdtd_grid_t *g, rfb_geom_t *geom, double *h[6]);
rfb_cpml_dev_t *rfb_cpml_device(cpml_t *p, const fdtd_grid_t *g);

void fdtd_update_e_materials(fdtd_grid_t *g, const materials_t *mat) {
    if (!materials_matches(mat, g)) return;
    rfb_scene_dev_t *s = materials_device(mat, g);
    if (!s) return;
    rfb_geom_t geom;
    double *h[6];
    rfb_fields_t *f = rfb_grid_device(g, &geom, h);
    if (!f) return;
    rfb_step_update_e(f, &geom, NULL, s, g->dt / (EPS0 * g->dx), h);
}

void fdtd_update_e_cpml_materials(fdtd_grid_t *g, cpml_t *pml, const materials_t *mat) {
    if (!materials_matches(mat, g) || !pml || pml->dx != g->dx) return;
    rfb_cpml_dev_t *c = rfb_cpml_device(pml, g);
    if (!c) return;
    rfb_scene_dev_t *s = materials_device(mat, g);
    if (!s) return;
    rfb_geom_t geom;
    double *h[6];
    rfb_fields_t *f = rfb_grid_device(g, &geom, h);
    if (!f) return;
    rfb_step_update_e(f, &geom, c, s, g->dt / (EPS0 * g->dx), h);
}
