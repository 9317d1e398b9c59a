/* tfsf.c -- total-field / scattered-field plane-wave injection (host side).
 *
 * No counterpart in rfsyn.  The incident field comes from a 1-D FDTD line
 * along the propagation direction k (Taflove & Hagness, Computational
 * Electrodynamics 3rd ed., ch. 5, the incident-field-array method): E1D at
 * integer positions m d1, H1D at (m + 1/2) d1, the grid's dt, a hard source
 * at m = 0.  A grid sample at position p (cell units) sees the incident
 * field at s = k . (p - r_ref) dx / d1 + M0 on the line (r_ref the corner of
 * the total-field box the wave reaches first), interpolated by a cubic
 * Lagrange polynomial through the four line samples around s.
 *
 * Line spacing (dispersion matching): the Yee grid's numerical dispersion
 * along k, 4/dx^2 sum_a sin^2(k k_a dx / 2), expands to
 * k^2 - k^4 dx^2 / 12 sum_a k_a^4, and the line's to k^2 - k^4 d1^2 / 12, so
 * d1 = dx sqrt(sum_a k_a^4) gives both the same phase velocity to second
 * order in k dx; the time-discretisation term is the same for both (same
 * dt).  Along an axis d1 = dx and every s is a whole or half line cell, so
 * normal incidence is injected exactly; along a body diagonal d1 = dx / sqrt 3
 * and the line reproduces the grid exactly as well.  sum_a k_a^4 >= 1/3, so
 * c dt / d1 <= courant_safety and the line is stable whenever the grid is.
 *
 * Corrections, generated from the update stencils themselves so that edges
 * and corners need no special cases:
 *   E_c update (E += Cb (tA - tB)) of a sample whose H neighbour q lies on
 *   the other side of the boundary: + Cb sigma (+1 inside / -1 outside) H_inc(q);
 *   H_c update (H -= cbh (dA - dB)) of a sample whose E neighbour q lies on
 *   the other side: - cbh sigma (+1 inside / -1 outside) E_inc(q);
 * sigma the sign of q in the stencil.  Each term is
 * coef * (((w0 X[idx-1] + w1 X[idx]) + w2 X[idx+1]) + w3 X[idx+2]) with X the
 * 1-D line's E (for H targets) or H (for E targets) and the unit-vector
 * component folded into coef; its four weights are stored together.  Terms
 * of one target are applied in the order generated here (the oracle
 * restates the same order). */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "host.h"

/* line cells between the source and the first box corner: a sample may sit
 * sqrt(3) cells before that corner, 3 line cells at the smallest d1, and
 * the cubic stencil reaches one more sample back */
#define M0 8.0
#define TF_C0 299792458.0
#define TF_MU0 1.25663706212e-6

/* position of sample (comp, cell) in cell units: E (c < 3) at cell + e_c / 2,
 * H (c >= 3) at cell + (1,1,1)/2 - e_{c-3}/2 */
static void sample_pos(int comp, const long p[3], double out[3]) {
    for (int a = 0; a < 3; a++) out[a] = (double)p[a];
    if (comp < 3) {
        out[comp] += 0.5;
    } else {
        for (int a = 0; a < 3; a++)
            if (a != comp - 3) out[a] += 0.5;
    }
}

typedef struct {
    double lo[3], hi[3];
    unsigned per;
    long n[3];
    double k[3], e[3], h[3], ref[3];
    double r;   /* line spacing / dx */
} tf_geo_t;

static int inside(const tf_geo_t *t, const double pos[3]) {
    for (int a = 0; a < 3; a++) {
        if (t->per & (1u << a)) continue;
        if (pos[a] < t->lo[a] || pos[a] > t->hi[a]) return 0;
    }
    return 1;
}

static double line_pos(const tf_geo_t *t, const double pos[3]) {
    double s = 0.0;
    for (int a = 0; a < 3; a++) s += t->k[a] * (pos[a] - t->ref[a]);
    return s / t->r + M0;
}

static void tf_geometry(const fdtd_grid_t *g, const fdtd_b200_plane_wave_t *pw, tf_geo_t *t) {
    memset(t, 0, sizeof(*t));
    t->per = g->periodic_axes;
    t->n[0] = (long)g->nx;
    t->n[1] = (long)g->ny;
    t->n[2] = (long)g->nz;
    const double lo[3] = {(double)pw->i0, (double)pw->j0, (double)pw->k0};
    const double hi[3] = {(double)pw->i1, (double)pw->j1, (double)pw->k1};
    const double st = sin(pw->theta), ct = cos(pw->theta), sp = sin(pw->phi), cp = cos(pw->phi);
    t->k[0] = st * cp;
    t->k[1] = st * sp;
    t->k[2] = ct;
    const double th[3] = {ct * cp, ct * sp, -st}, ph[3] = {-sp, cp, 0.0};
    for (int a = 0; a < 3; a++) t->e[a] = cos(pw->psi) * th[a] + sin(pw->psi) * ph[a];
    t->h[0] = t->k[1] * t->e[2] - t->k[2] * t->e[1];
    t->h[1] = t->k[2] * t->e[0] - t->k[0] * t->e[2];
    t->h[2] = t->k[0] * t->e[1] - t->k[1] * t->e[0];
    double k4 = 0.0;
    for (int a = 0; a < 3; a++) k4 += (t->k[a] * t->k[a]) * (t->k[a] * t->k[a]);
    t->r = sqrt(k4);
    for (int a = 0; a < 3; a++) {
        t->lo[a] = lo[a];
        t->hi[a] = hi[a];
        t->ref[a] = (t->per & (1u << a)) ? 0.0 : (t->k[a] >= 0.0 ? lo[a] : hi[a]);
    }
}

static long wrapc(const tf_geo_t *t, int a, long q) {
    if (!(t->per & (1u << a))) return q;
    if (q < 0) return q + t->n[a];
    if (q >= t->n[a]) return q - t->n[a];
    return q;
}

/* growable arrays */
typedef struct {
    size_t n, cap;
    int32_t *ijkc;   /* i, j, k, comp per target */
    int32_t *first, *count;
} targets_t;

typedef struct {
    size_t n, cap;
    double *coef, *w;   /* w: 4 weights per term */
    int32_t *idx;
} terms_t;

static int push_term(terms_t *T, double coef, double s) {
    if (T->n == T->cap) {
        size_t nc = T->cap ? 2 * T->cap : 256;
        double *a = realloc(T->coef, nc * sizeof(double));
        if (a) T->coef = a;
        double *b = realloc(T->w, 4 * nc * sizeof(double));
        if (b) T->w = b;
        int32_t *d = realloc(T->idx, nc * sizeof(int32_t));
        if (d) T->idx = d;
        if (!a || !b || !d) return -1;
        T->cap = nc;
    }
    /* cubic Lagrange weights of the samples idx-1 .. idx+2 at u = s - idx;
     * u = 0 gives exactly (0, 1, 0, 0) */
    const double f = floor(s), u = s - f;
    double *w = T->w + 4 * T->n;
    T->coef[T->n] = coef;
    T->idx[T->n] = (int32_t)f;
    w[0] = -u * (u - 1.0) * (u - 2.0) / 6.0;
    w[1] = (u + 1.0) * (u - 1.0) * (u - 2.0) / 2.0;
    w[2] = -(u + 1.0) * u * (u - 2.0) / 2.0;
    w[3] = (u + 1.0) * u * (u - 1.0) / 6.0;
    T->n++;
    return 0;
}

static int push_target(targets_t *R, long i, long j, long k, int comp, size_t first, size_t count) {
    if (R->n == R->cap) {
        size_t nc = R->cap ? 2 * R->cap : 256;
        int32_t *a = realloc(R->ijkc, 4 * nc * sizeof(int32_t));
        if (a) R->ijkc = a;
        int32_t *b = realloc(R->first, nc * sizeof(int32_t));
        if (b) R->first = b;
        int32_t *c = realloc(R->count, nc * sizeof(int32_t));
        if (c) R->count = c;
        if (!a || !b || !c) return -1;
        R->cap = nc;
    }
    R->ijkc[4 * R->n] = (int32_t)i;
    R->ijkc[4 * R->n + 1] = (int32_t)j;
    R->ijkc[4 * R->n + 2] = (int32_t)k;
    R->ijkc[4 * R->n + 3] = comp;
    R->first[R->n] = (int32_t)first;
    R->count[R->n] = (int32_t)count;
    R->n++;
    return 0;
}

void rfb_tfsf_free(rfb_tfsf_build_t *b) {
    free(b->src);
    free(b->h_ijkc); free(b->h_first); free(b->h_count);
    free(b->e_ijkc); free(b->e_first); free(b->e_count);
    free(b->h_coef); free(b->h_w); free(b->h_idx);
    free(b->e_coef); free(b->e_w); free(b->e_idx);
    free(b->cells);
    memset(b, 0, sizeof(*b));
}

double rfb_wave_value(int waveform, double amplitude, double p0, double p1, double p2, double t);

int rfb_tfsf_build(const fdtd_grid_t *g, const materials_t *mat, const fdtd_b200_plane_wave_t *pw, size_t n_steps,
                   int cpml_npml, rfb_tfsf_build_t *out) {
    memset(out, 0, sizeof(*out));
    if (pw->waveform < 0 || pw->waveform > 2) {
        rfb_set_error("plane wave: unknown waveform");
        return -1;
    }
    tf_geo_t t;
    tf_geometry(g, pw, &t);
    for (int a = 0; a < 3; a++) {
        /* a wave with a component of k along a periodic axis has a phase
         * shift across the period (Floquet); without that boundary the
         * wrapped grid would not carry it */
        if ((t.per & (1u << a)) && fabs(t.k[a]) > 1e-12) {
            rfb_set_error("plane wave: oblique incidence along periodic axis %d is not supported (normal incidence "
                          "only along periodic axes)", a);
            return -1;
        }
    }
    const long n[3] = {(long)g->nx, (long)g->ny, (long)g->nz};
    long lo[3], hi[3];
    const size_t bl[3] = {pw->i0, pw->j0, pw->k0}, bh[3] = {pw->i1, pw->j1, pw->k1};
    for (int a = 0; a < 3; a++) {
        if (t.per & (1u << a)) {
            lo[a] = 0;
            hi[a] = n[a] - 1;
            continue;
        }
        const long margin = 2 + (long)cpml_npml;
        if (bl[a] >= bh[a] || (long)bl[a] < margin || (long)bh[a] + margin > n[a]) {
            rfb_set_error("plane wave: the total-field box grown by two cells must lie inside the grid and outside "
                          "the CPML (axis %d)", a);
            return -1;
        }
        lo[a] = (long)bl[a] - 2;
        hi[a] = (long)bh[a] + 2;
    }
    const double cb_h = g->dt / (TF_MU0 * g->dx);
    targets_t HT = {0}, ET = {0};
    terms_t HX = {0}, EX = {0};
    double smax = 0.0;
    /* shell: cells within two of a face on a non-periodic axis, the box
     * grown by two on every axis */
    for (long i = lo[0]; i <= hi[0]; i++)
        for (long j = lo[1]; j <= hi[1]; j++)
            for (long k = lo[2]; k <= hi[2]; k++) {
                const long p[3] = {i, j, k};
                int near = 0;
                for (int a = 0; a < 3; a++)
                    if (!(t.per & (1u << a)) && (p[a] <= (long)bl[a] + 2 || p[a] >= (long)bh[a] - 2)) near = 1;
                if (!near) {
                    /* a column that is near no x / y face meets the shell
                     * again only at the high z face: skip to it */
                    if (!(t.per & 4u) && k < (long)bh[2] - 2) k = (long)bh[2] - 3;
                    continue;
                }
                for (int c = 0; c < 3; c++) {
                    /* ---- H_c at p: H -= cbh (dA - dB), dA = E_fa(p+e_axa) - E_fa(p), dB likewise */
                    {
                        const int fa = (c + 2) % 3, axa = (c + 1) % 3, fb = (c + 1) % 3, axb = (c + 2) % 3;
                        double hp[3];
                        sample_pos(3 + c, p, hp);
                        const int hin = inside(&t, hp);
                        const int qc[4] = {fa, fa, fb, fb};
                        const double sg[4] = {1.0, -1.0, -1.0, 1.0};
                        long q[4][3];
                        for (int u = 0; u < 4; u++)
                            for (int a = 0; a < 3; a++) q[u][a] = p[a];
                        q[0][axa] += 1;
                        q[2][axb] += 1;
                        const size_t first = HX.n;
                        for (int u = 0; u < 4; u++) {
                            double ep[3];
                            sample_pos(qc[u], q[u], ep);
                            if (inside(&t, ep) == hin) continue;
                            const double s = line_pos(&t, ep);
                            if (s > smax) smax = s;
                            if (push_term(&HX, -cb_h * sg[u] * (hin ? 1.0 : -1.0) * t.e[qc[u]], s) != 0) goto oom;
                        }
                        if (HX.n > first &&
                            push_target(&HT, wrapc(&t, 0, i), wrapc(&t, 1, j), wrapc(&t, 2, k), c, first,
                                        HX.n - first) != 0)
                            goto oom;
                    }
                    /* ---- E_c at p: E += Cb (tA - tB), tA = H_fa(p) - H_fa(p-e_axa), tB likewise */
                    {
                        const size_t ci = (size_t)wrapc(&t, 0, i), cj = (size_t)wrapc(&t, 1, j),
                                     ck = (size_t)wrapc(&t, 2, k);
                        if (!rfb_e_swept(g, c, ci, cj, ck)) continue;
                        const int fa = (c + 2) % 3, axa = (c + 1) % 3, fb = (c + 1) % 3, axb = (c + 2) % 3;
                        double epos[3];
                        sample_pos(c, p, epos);
                        const int ein = inside(&t, epos);
                        const int qc[4] = {fa, fa, fb, fb};
                        const double sg[4] = {1.0, -1.0, -1.0, 1.0};
                        long q[4][3];
                        for (int u = 0; u < 4; u++)
                            for (int a = 0; a < 3; a++) q[u][a] = p[a];
                        q[1][axa] -= 1;
                        q[3][axb] -= 1;
                        material_coeff_t co;
                        if (materials_get_coefficients(mat, g, (field_component_t)c, ci, cj, ck, &co) != 0) {
                            rfb_set_error("plane wave: no coefficients at a boundary sample");
                            goto fail;
                        }
                        const size_t first = EX.n;
                        for (int u = 0; u < 4; u++) {
                            double hpq[3];
                            sample_pos(3 + qc[u], q[u], hpq);
                            if (inside(&t, hpq) == ein) continue;
                            const double s = line_pos(&t, hpq) - 0.5;
                            if (s + 0.5 > smax) smax = s + 0.5;
                            if (push_term(&EX, co.Cb * sg[u] * (ein ? 1.0 : -1.0) * t.h[qc[u]], s) != 0) goto oom;
                        }
                        if (EX.n > first && push_target(&ET, (long)ci, (long)cj, (long)ck, c, first, EX.n - first) != 0)
                            goto oom;
                    }
                }
            }
    /* every term reads the line inside [0, m_len) */
    for (size_t q = 0; q < HX.n; q++)
        if (HX.idx[q] < 1) {
            rfb_set_error("plane wave: the line does not reach a boundary sample");
            goto fail;
        }
    for (size_t q = 0; q < EX.n; q++)
        if (EX.idx[q] < 1) {
            rfb_set_error("plane wave: the line does not reach a boundary sample");
            goto fail;
        }
    {
        const double cells_per_step = TF_C0 * g->dt / g->dx;
        out->m_len = (size_t)ceil(smax) + 4 + (size_t)ceil((double)n_steps * cells_per_step / t.r) + 4;
    }
    out->ce = g->dt / (8.8541878128e-12 * (g->dx * t.r));
    out->ch = g->dt / (TF_MU0 * (g->dx * t.r));
    /* hard source E1D[0] at steps 0..n_steps: amplitude * waveform(n dt) */
    out->src = malloc((n_steps + 1) * sizeof(double));
    if (!out->src) goto oom;
    for (size_t s = 0; s <= n_steps; s++)
        out->src[s] = rfb_wave_value(pw->waveform, pw->amplitude, pw->p0, pw->p1, pw->p2, (double)s * g->dt);
    out->n_h = HT.n;
    out->h_ijkc = HT.ijkc; out->h_first = HT.first; out->h_count = HT.count;
    out->n_e = ET.n;
    out->e_ijkc = ET.ijkc; out->e_first = ET.first; out->e_count = ET.count;
    out->n_hterms = HX.n;
    out->h_coef = HX.coef; out->h_w = HX.w; out->h_idx = HX.idx;
    out->n_eterms = EX.n;
    out->e_coef = EX.coef; out->e_w = EX.w; out->e_idx = EX.idx;
    /* list cells: every E target, and every E sample reading a corrected H
     * sample: H_c(p) is read by E_{c+1}(p), E_{c+1}(p + e_{c+2}),
     * E_{c+2}(p), E_{c+2}(p + e_{c+1}) */
    {
        size_t cap = ET.n + 4 * HT.n + 1;
        out->cells = malloc(3 * cap * sizeof(int32_t));
        if (!out->cells) goto oom;
        size_t nc = 0;
        for (size_t q = 0; q < ET.n; q++) {
            memcpy(out->cells + 3 * nc, ET.ijkc + 4 * q, 3 * sizeof(int32_t));
            nc++;
        }
        for (size_t q = 0; q < HT.n; q++) {
            const int c = HT.ijkc[4 * q + 3];
            const long base[3] = {HT.ijkc[4 * q], HT.ijkc[4 * q + 1], HT.ijkc[4 * q + 2]};
            for (int v = 0; v < 4; v++) {
                long cell[3] = {base[0], base[1], base[2]};
                if (v == 1) cell[(c + 2) % 3] += 1;
                if (v == 3) cell[(c + 1) % 3] += 1;
                for (int a = 0; a < 3; a++) cell[a] = wrapc(&t, a, cell[a]);
                for (int a = 0; a < 3; a++) out->cells[3 * nc + a] = (int32_t)cell[a];
                nc++;
            }
        }
        out->n_cells = nc;
    }
    return 0;
oom:
    rfb_set_error("out of host memory building the plane-wave boundary");
fail:
    free(HT.ijkc); free(HT.first); free(HT.count);
    free(ET.ijkc); free(ET.first); free(ET.count);
    free(HX.coef); free(HX.w); free(HX.idx);
    free(EX.coef); free(EX.w); free(EX.idx);
    rfb_tfsf_free(out);
    return -1;
}
