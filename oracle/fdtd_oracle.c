/*
 * fdtd_oracle.c -- TEST INFRASTRUCTURE.  CPU restatement (FP64, plain loops)
 * of rfsyn's FDTD time loop, used only by tests/, smoke() and the CPU leg of
 * bench.py as the checker.  Never linked into the product.
 *
 * Parity pin: tests compare every function here against rfsyn itself built
 * from its sources (oracle/_ref, recipe in oracle/Makefile) and against the
 * committed golden fixtures in tests/golden/.
 *
 * Followed, line by line in arithmetic order:
 *   grid / dt / index wrap ....... engine/fdtd/grid.c:7-46, grid.h:21-30
 *   CPML profiles ................ engine/fdtd/cpml.c:21-150
 *   cpml_term .................... engine/fdtd/cpml.h:46-51
 *   H update (CPML, vacuum) ...... engine/fdtd/cpml.c:176-219, grid.c:62-90
 *   E update with materials ...... engine/fdtd/materials.c:911-1060
 *   material coefficients ........ engine/fdtd/materials.c:92-125
 *   box / override semantics ..... engine/fdtd/materials.c:476-636
 *   2x2 tensor edge .............. engine/fdtd/materials.c:836-903
 *   sources ...................... engine/fdtd/source.c:8-57
 *   probes, DFT .................. engine/fdtd/probe.c:40-92
 * Beyond rfsyn (no reference counterpart; pinned by physics checks in tests):
 *   dispersive ADE samples ....... Taflove & Hagness, Computational
 *                                  Electrodynamics 3rd ed. sec. 9.4 (Debye
 *                                  and Lorentz polarisation currents)
 *   sphere fill fractions and the diagonal of the smoothed inverse
 *   permittivity (Farjadpour et al., Opt. Lett. 31, 2972 (2006))
 *   full 3x3 anisotropic samples: the 2x2 tensor edge generalised to a
 *                                  full row of eps_r^-1, off-diagonal curls
 *                                  averaged over the four surrounding samples
 *   plane wave, TF/SF boundary ... Taflove & Hagness 3rd ed. ch. 5: a 1-D
 *                                  incident line with spacing
 *                                  dx sqrt(sum k_a^4) (the grid's dispersion
 *                                  along k to second order), cubic Lagrange
 *                                  interpolation, corrections generated from
 *                                  the update stencils (the product's term
 *                                  order, restated)
 * The data structures are the plainest possible (dense per-component override
 * and tensor planes, full-grid psi) so the restatement is easy to audit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "scene.h"
#include "sphere_raster.h"

#define O_C0 299792458.0
#define O_EPS0 8.8541878128e-12
#define O_MU0 1.25663706212e-6
#define O_PI 3.14159265358979323846

typedef struct {
    size_t n[3];          /* nx, ny, nz */
    unsigned per;
    double dx, dt;
    size_t total;
    double *E[3], *H[3];
    /* CPML: per axis, integer (m) and half (h) profiles */
    int cpml;
    double *km[3], *bm[3], *am[3], *kh[3], *bh[3], *ah[3];
    double *psiH[3][2], *psiE[3][2];
    /* materials */
    uint8_t *id;
    double tca[256], tcb[256], teps[256], tsig[256];
    size_t ntab;
    uint8_t *has_ovr[3];
    double *oca[3], *ocb[3];
    uint8_t *has_t[2];
    double *tm11[2], *tm12[2], *tm22[2], *tscale[2];
    /* dispersive samples: per-component index into the ADE arrays (-1) */
    int *dix[3];
    size_t nd, dcap;
    double *drec;   /* 16 per sample */
    double *dst;    /* 5 per sample: J0 J1 J0- J1- E- */
    /* full 3x3 samples: per component a flag and the row of eps_r^-1 */
    uint8_t *has_t3[3];
    double *t3m[3], *t3s[3];
    /* plane wave: the 1-D line, H targets, per-sample E term ranges, terms */
    int tf;
    size_t tf_len;
    double tf_ce, tf_ch, *tf_e, *tf_h, *tf_src;
    size_t tf_nh, tf_hcap;
    size_t *tf_hw;      /* canonical index of each H target */
    int *tf_hc, *tf_hfirst, *tf_hcount;
    int *tf_efirst[3], *tf_ecount[3];
    size_t tf_nt, tf_tcap;
    double *tf_coef, *tf_w;   /* 4 weights per term */
    int *tf_idx;
} orc_t;

static int periodic(const orc_t *o, int a) { return (o->per >> a) & 1u; }

/* grid.h:25-30 */
static size_t at(const orc_t *o, size_t i, size_t j, size_t k) {
    if (periodic(o, 0)) i %= o->n[0];
    if (periodic(o, 1)) j %= o->n[1];
    if (periodic(o, 2)) k %= o->n[2];
    return (i * (o->n[1] + 1) + j) * (o->n[2] + 1) + k;
}

static size_t back(size_t q, size_t n) { return q == 0 ? n - 1 : q - 1; }

/* cpml.c:21-89, one axis */
static void profiles(orc_t *o, int a, const scn_scene_t *s, double sigma_max) {
    size_t n = o->n[a];
    o->km[a] = malloc((n + 1) * 8); o->bm[a] = malloc((n + 1) * 8); o->am[a] = malloc((n + 1) * 8);
    o->kh[a] = malloc(n * 8); o->bh[a] = malloc(n * 8); o->ah[a] = malloc(n * 8);
    double d = (double)s->npml * o->dx, len = (double)n * o->dx;
    for (size_t q = 0; q < 2 * n + 1; q++) {
        /* even q: integer position q/2; odd q: half position */
        int half = q & 1;
        size_t idx = q / 2;
        double x = half ? ((double)idx + 0.5) * o->dx : (double)idx * o->dx;
        double rho = -1.0;
        if (x < d) rho = d - x;
        else if (x > len - d) rho = x - (len - d);
        double kinv = 1.0, b = 1.0, av = 0.0;
        if (rho >= 0.0 && !periodic(o, a)) {
            double r = rho / d;
            if (r > 1.0) r = 1.0;
            double sg = sigma_max * pow(r, s->m);
            double kp = 1.0 + (s->kappa_max - 1.0) * pow(r, s->m);
            double al = s->alpha_max * pow(1.0 - r, s->ma);
            b = exp(-(sg / kp + al) * o->dt / O_EPS0);
            av = (sg > 0.0) ? sg * (b - 1.0) / (o->dx * kp * (sg + kp * al)) : 0.0;
            kinv = 1.0 / kp;
        }
        if (half) { o->kh[a][idx] = kinv; o->bh[a][idx] = b; o->ah[a][idx] = av; }
        else { o->km[a][idx] = kinv; o->bm[a][idx] = b; o->am[a][idx] = av; }
    }
}

static void orc_free(orc_t *o) {
    for (int c = 0; c < 3; c++) {
        free(o->E[c]); free(o->H[c]);
        free(o->km[c]); free(o->bm[c]); free(o->am[c]); free(o->kh[c]); free(o->bh[c]); free(o->ah[c]);
        for (int t = 0; t < 2; t++) { free(o->psiH[c][t]); free(o->psiE[c][t]); }
        free(o->has_ovr[c]); free(o->oca[c]); free(o->ocb[c]);
    }
    for (int c = 0; c < 2; c++) { free(o->has_t[c]); free(o->tm11[c]); free(o->tm12[c]); free(o->tm22[c]); free(o->tscale[c]); }
    for (int c = 0; c < 3; c++) free(o->dix[c]), free(o->has_t3[c]), free(o->t3m[c]), free(o->t3s[c]);
    for (int c = 0; c < 3; c++) free(o->tf_efirst[c]), free(o->tf_ecount[c]);
    free(o->tf_e); free(o->tf_h); free(o->tf_src); free(o->tf_hw); free(o->tf_hc); free(o->tf_hfirst);
    free(o->tf_hcount); free(o->tf_coef); free(o->tf_w); free(o->tf_idx);
    free(o->drec);
    free(o->dst);
    free(o->id);
}

/* ADE coefficients of a dispersive sample (see the product's record layout):
 * E+ = ca E + cb (dA - dB) + ce E- - sum_p (cj J + cjm J-),
 * J+ = aJ J + aJm J- + aE (E+ - E_ref).  Debye: k = (1 - dt/2tau)/(1 + dt/2tau),
 * beta = eps0 de dt/tau / (1 + dt/2tau); Lorentz: a = (2 - wp^2 dt^2)/(1+g dt),
 * xi = (g dt - 1)/(1 + g dt), gl = eps0 de wp^2 dt^2/(1 + g dt); Ampere at
 * n+1/2 gives A = eps0 eps_inf + sigma dt/2 + sum beta/2 + sum gl/4. */
static void ade_coeffs(const scn_disp_t *d, double dt, double dx, double *r) {
    double e0ei = O_EPS0 * d->eps_inf, hb = 0.0, qg = 0.0;
    double kJ[2] = {0, 0}, kJm[2] = {0, 0}, kE[2] = {0, 0};
    for (int p = 0; p < d->npoles; p++) {
        if (d->kind[p] == 0) {
            double den = 1.0 + dt / (2.0 * d->tau[p]);
            double beta = (O_EPS0 * d->delta_eps[p] * dt / d->tau[p]) / den;
            kJ[p] = (1.0 - dt / (2.0 * d->tau[p])) / den;
            kE[p] = beta / dt;
            hb += 0.5 * beta;
        } else {
            double den = 1.0 + d->gamma[p] * dt;
            double gl = O_EPS0 * d->delta_eps[p] * d->omega_p[p] * d->omega_p[p] * dt * dt / den;
            kJ[p] = (2.0 - d->omega_p[p] * d->omega_p[p] * dt * dt) / den;
            kJm[p] = (d->gamma[p] * dt - 1.0) / den;
            kE[p] = gl / (2.0 * dt);
            qg += 0.25 * gl;
        }
    }
    double A = e0ei + 0.5 * d->sigma * dt + hb + qg;
    memset(r, 0, 16 * sizeof(double));
    r[0] = (e0ei - 0.5 * d->sigma * dt + hb) / A;
    r[1] = dt / (A * dx);
    r[2] = qg / A;
    r[3] = (double)d->npoles;
    for (int p = 0; p < d->npoles; p++) {
        double *w = r + 4 + 6 * p;
        w[0] = (double)d->kind[p];
        w[1] = 0.5 * dt * (1.0 + kJ[p]) / A;
        w[2] = 0.5 * dt * kJm[p] / A;
        w[3] = kJ[p];
        w[4] = kJm[p];
        w[5] = kE[p];
    }
}

static int set_disp(orc_t *o, int c, size_t w, const scn_disp_t *d) {
    if (o->dix[c][w] < 0) {
        if (o->nd == o->dcap) {
            o->dcap = o->dcap ? 2 * o->dcap : 64;
            double *nr = realloc(o->drec, o->dcap * 16 * sizeof(double));
            if (nr) o->drec = nr;
            double *ns = realloc(o->dst, o->dcap * 5 * sizeof(double));
            if (ns) o->dst = ns;
            if (!nr || !ns) return -1;
        }
        o->dix[c][w] = (int)o->nd++;
    }
    size_t q = (size_t)o->dix[c][w];
    ade_coeffs(d, o->dt, o->dx, o->drec + 16 * q);
    memset(o->dst + 5 * q, 0, 5 * sizeof(double));
    return 0;
}

static int coeff(const orc_t *o, double eps_r, double sigma, double *ca, double *cb);
static int table_id(orc_t *o, double eps_r, double sigma);

/* oracle-side callbacks of the shared sphere rasteriser */
static void sr_bg(void *ctx, size_t w, double *eps, double *sig) {
    orc_t *o = (orc_t *)ctx;
    *eps = o->teps[o->id[w]];
    *sig = o->tsig[o->id[w]];
}
static void clear_samples(orc_t *o, size_t w) {
    for (int c = 0; c < 3; c++) o->has_ovr[c][w] = 0, o->dix[c][w] = -1, o->has_t3[c][w] = 0;
    for (int c = 0; c < 2; c++) o->has_t[c][w] = 0;
}
static int sr_fill(void *ctx, size_t w, const scn_sphere_t *sp) {
    orc_t *o = (orc_t *)ctx;
    int id = table_id(o, sp->eps_r, sp->sigma);
    if (id < 0) return -1;
    clear_samples(o, w);
    o->id[w] = (uint8_t)id;
    return 0;
}
static int sr_fill_disp(void *ctx, size_t w, const scn_disp_t *d) {
    orc_t *o = (orc_t *)ctx;
    clear_samples(o, w);
    for (int c = 0; c < 3; c++)
        if (set_disp(o, c, w, d) != 0) return -1;
    return 0;
}
static int sr_sample(void *ctx, size_t w, int c, double eps, double sig) {
    orc_t *o = (orc_t *)ctx;
    if (coeff(o, eps, sig, &o->oca[c][w], &o->ocb[c][w]) != 0) return -1;
    o->has_ovr[c][w] = 1;
    o->dix[c][w] = -1;
    o->has_t3[c][w] = 0;
    return 0;
}
static int sr_sample_disp(void *ctx, size_t w, int c, const scn_disp_t *d) {
    return set_disp((orc_t *)ctx, c, w, d);
}
static int sr_sample_t3(void *ctx, size_t w, int c, const double row[3], double sigma) {
    orc_t *o = (orc_t *)ctx;
    o->has_ovr[c][w] = 0;
    o->dix[c][w] = -1;
    if (c < 2) o->has_t[c][w] = 0;
    o->has_t3[c][w] = 1;
    memcpy(o->t3m[c] + 3 * w, row, 3 * sizeof(double));
    o->t3s[c][w] = sigma;
    return 0;
}
static size_t sr_canon(const void *geo, size_t i, size_t j, size_t k) { return at((const orc_t *)geo, i, j, k); }

/* materials.c:92-125 */
static int coeff(const orc_t *o, double eps_r, double sigma, double *ca, double *cb) {
    if (!isfinite(eps_r) || eps_r < 1.0 || !isfinite(sigma) || sigma < 0.0) return -1;
    double eps = eps_r * O_EPS0;
    double loss = (sigma * o->dt) / (2.0 * eps);
    double b = o->dt / (eps * o->dx);
    *ca = (1.0 - loss) / (1.0 + loss);
    *cb = b / (1.0 + loss);
    return 0;
}

static int table_id(orc_t *o, double eps_r, double sigma) {
    for (size_t q = 0; q < o->ntab; q++)
        if (o->teps[q] == eps_r && o->tsig[q] == sigma) return (int)q;
    if (o->ntab >= 256) return -1;
    if (coeff(o, eps_r, sigma, &o->tca[o->ntab], &o->tcb[o->ntab]) != 0) return -1;
    o->teps[o->ntab] = eps_r;
    o->tsig[o->ntab] = sigma;
    return (int)o->ntab++;
}

/* ---- plane wave (TF/SF) ---------------------------------------------------- */
static double wave(const scn_source_t *s, double t);

static void tf_pos(int comp, const long p[3], double out[3]) {
    for (int a = 0; a < 3; a++) out[a] = (double)p[a];
    if (comp < 3) out[comp] += 0.5;
    else
        for (int a = 0; a < 3; a++)
            if (a != comp - 3) out[a] += 0.5;
}

typedef struct {
    double lo[3], hi[3], k[3], e[3], h[3], ref[3];
    double r;   /* line spacing / dx */
    unsigned per;
} tf_t;

static int tf_in(const tf_t *t, const double p[3]) {
    for (int a = 0; a < 3; a++)
        if (!(t->per & (1u << a)) && (p[a] < t->lo[a] || p[a] > t->hi[a])) return 0;
    return 1;
}

static double tf_s(const tf_t *t, const double p[3]) {
    double s = 0.0;
    for (int a = 0; a < 3; a++) s += t->k[a] * (p[a] - t->ref[a]);
    return s / t->r + 8.0;
}

static int tf_term(orc_t *o, double coef, double s) {
    if (o->tf_nt == o->tf_tcap) {
        o->tf_tcap = o->tf_tcap ? 2 * o->tf_tcap : 256;
        o->tf_coef = realloc(o->tf_coef, o->tf_tcap * 8);
        o->tf_w = realloc(o->tf_w, 4 * o->tf_tcap * 8);
        o->tf_idx = realloc(o->tf_idx, o->tf_tcap * sizeof(int));
        if (!o->tf_coef || !o->tf_w || !o->tf_idx) return -1;
    }
    /* cubic Lagrange weights of line samples f-1 .. f+2 at u = s - f */
    double f = floor(s), u = s - f;
    double *w = o->tf_w + 4 * o->tf_nt;
    o->tf_coef[o->tf_nt] = coef;
    o->tf_idx[o->tf_nt] = (int)f;
    w[0] = -u * (u - 1.0) * (u - 2.0) / 6.0;
    w[1] = (u + 1.0) * (u - 1.0) * (u - 2.0) / 2.0;
    w[2] = -(u + 1.0) * u * (u - 2.0) / 2.0;
    w[3] = (u + 1.0) * u * (u - 1.0) / 6.0;
    o->tf_nt++;
    return 0;
}

static long tf_wrap(const orc_t *o, int a, long q) {
    if (!periodic(o, a)) return q;
    long n = (long)o->n[a];
    return q < 0 ? q + n : (q >= n ? q - n : q);
}

static int tf_init(orc_t *o, const scn_scene_t *s) {
    const scn_plane_wave_t *pw = s->plane_wave;
    tf_t t;
    memset(&t, 0, sizeof t);
    t.per = o->per;
    double st = sin(pw->theta), ct = cos(pw->theta), sp = sin(pw->phi), cp = cos(pw->phi);
    t.k[0] = st * cp; t.k[1] = st * sp; t.k[2] = ct;
    double th[3] = {ct * cp, ct * sp, -st}, ph[3] = {-sp, cp, 0.0};
    for (int a = 0; a < 3; a++) t.e[a] = cos(pw->psi) * th[a] + sin(pw->psi) * ph[a];
    t.h[0] = t.k[1] * t.e[2] - t.k[2] * t.e[1];
    t.h[1] = t.k[2] * t.e[0] - t.k[0] * t.e[2];
    t.h[2] = t.k[0] * t.e[1] - t.k[1] * t.e[0];
    t.r = sqrt(t.k[0] * t.k[0] * (t.k[0] * t.k[0]) + t.k[1] * t.k[1] * (t.k[1] * t.k[1]) +
               t.k[2] * t.k[2] * (t.k[2] * t.k[2]));
    const size_t bl[3] = {pw->i0, pw->j0, pw->k0}, bh[3] = {pw->i1, pw->j1, pw->k1};
    long lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        t.lo[a] = (double)bl[a];
        t.hi[a] = (double)bh[a];
        t.ref[a] = periodic(o, a) ? 0.0 : (t.k[a] >= 0.0 ? (double)bl[a] : (double)bh[a]);
        lo[a] = periodic(o, a) ? 0 : (long)bl[a] - 2;
        hi[a] = periodic(o, a) ? (long)o->n[a] - 1 : (long)bh[a] + 2;
    }
    const double cbh = o->dt / (O_MU0 * o->dx);
    double smax = 0.0;
    for (int c = 0; c < 3; c++) {
        o->tf_efirst[c] = malloc(o->total * sizeof(int));
        o->tf_ecount[c] = calloc(o->total, sizeof(int));
        if (!o->tf_efirst[c] || !o->tf_ecount[c]) return -1;
        for (size_t q = 0; q < o->total; q++) o->tf_efirst[c][q] = -1;
    }
    for (long i = lo[0]; i <= hi[0]; i++)
        for (long j = lo[1]; j <= hi[1]; j++)
            for (long k = lo[2]; k <= hi[2]; k++) {
                const long p[3] = {i, j, k};
                int near = 0;
                for (int a = 0; a < 3; a++)
                    if (!periodic(o, a) && (p[a] <= (long)bl[a] + 2 || p[a] >= (long)bh[a] - 2)) near = 1;
                if (!near) continue;
                for (int c = 0; c < 3; c++) {
                    const int fa = (c + 2) % 3, axa = (c + 1) % 3, fb = (c + 1) % 3, axb = (c + 2) % 3;
                    const int qc[4] = {fa, fa, fb, fb};
                    const double sg[4] = {1.0, -1.0, -1.0, 1.0};
                    /* H_c at p */
                    {
                        double hp[3];
                        tf_pos(3 + c, p, hp);
                        int hin = tf_in(&t, hp);
                        long q[4][3];
                        for (int u = 0; u < 4; u++) for (int a = 0; a < 3; a++) q[u][a] = p[a];
                        q[0][axa] += 1;
                        q[2][axb] += 1;
                        size_t first = o->tf_nt;
                        for (int u = 0; u < 4; u++) {
                            double ep[3];
                            tf_pos(qc[u], q[u], ep);
                            if (tf_in(&t, ep) == hin) continue;
                            double sv = tf_s(&t, ep);
                            if (sv > smax) smax = sv;
                            if (tf_term(o, -cbh * sg[u] * (hin ? 1.0 : -1.0) * t.e[qc[u]], sv) != 0) return -1;
                        }
                        if (o->tf_nt > first) {
                            if (o->tf_nh == o->tf_hcap) {
                                o->tf_hcap = o->tf_hcap ? 2 * o->tf_hcap : 256;
                                o->tf_hw = realloc(o->tf_hw, o->tf_hcap * sizeof(size_t));
                                o->tf_hc = realloc(o->tf_hc, o->tf_hcap * sizeof(int));
                                o->tf_hfirst = realloc(o->tf_hfirst, o->tf_hcap * sizeof(int));
                                o->tf_hcount = realloc(o->tf_hcount, o->tf_hcap * sizeof(int));
                                if (!o->tf_hw || !o->tf_hc || !o->tf_hfirst || !o->tf_hcount) return -1;
                            }
                            o->tf_hw[o->tf_nh] = at(o, (size_t)tf_wrap(o, 0, i), (size_t)tf_wrap(o, 1, j),
                                                    (size_t)tf_wrap(o, 2, k));
                            o->tf_hc[o->tf_nh] = c;
                            o->tf_hfirst[o->tf_nh] = (int)first;
                            o->tf_hcount[o->tf_nh] = (int)(o->tf_nt - first);
                            o->tf_nh++;
                        }
                    }
                    /* E_c at p */
                    {
                        size_t ci = (size_t)tf_wrap(o, 0, i), cj = (size_t)tf_wrap(o, 1, j), ck = (size_t)tf_wrap(o, 2, k);
                        size_t cc[3] = {ci, cj, ck};
                        int swept = ci < o->n[0] && cj < o->n[1] && ck < o->n[2];
                        for (int a = 0; a < 3 && swept; a++)
                            if (a != c && !periodic(o, a) && cc[a] < 1) swept = 0;
                        if (!swept) continue;
                        double epos[3];
                        tf_pos(c, p, epos);
                        int ein = tf_in(&t, epos);
                        long q[4][3];
                        for (int u = 0; u < 4; u++) for (int a = 0; a < 3; a++) q[u][a] = p[a];
                        q[1][axa] -= 1;
                        q[3][axb] -= 1;
                        size_t w = at(o, ci, cj, ck);
                        double cb = o->has_ovr[c][w] ? o->ocb[c][w] : o->tcb[o->id[w]];
                        size_t first = o->tf_nt;
                        for (int u = 0; u < 4; u++) {
                            double hq[3];
                            tf_pos(3 + qc[u], q[u], hq);
                            if (tf_in(&t, hq) == ein) continue;
                            double sv = tf_s(&t, hq) - 0.5;
                            if (sv + 0.5 > smax) smax = sv + 0.5;
                            if (tf_term(o, cb * sg[u] * (ein ? 1.0 : -1.0) * t.h[qc[u]], sv) != 0) return -1;
                        }
                        if (o->tf_nt > first) {
                            o->tf_efirst[c][w] = (int)first;
                            o->tf_ecount[c][w] = (int)(o->tf_nt - first);
                        }
                    }
                }
            }
    double cps = O_C0 * o->dt / o->dx;
    o->tf_len = (size_t)ceil(smax) + 4 + (size_t)ceil((double)s->n_steps * cps / t.r) + 4;
    o->tf_ce = o->dt / (O_EPS0 * (o->dx * t.r));
    o->tf_ch = o->dt / (O_MU0 * (o->dx * t.r));
    o->tf_e = calloc(o->tf_len, 8);
    o->tf_h = calloc(o->tf_len, 8);
    o->tf_src = malloc((s->n_steps + 1) * 8);
    if (!o->tf_e || !o->tf_h || !o->tf_src) return -1;
    scn_source_t ws;
    memset(&ws, 0, sizeof ws);
    ws.waveform = pw->waveform;
    ws.p0 = pw->p0; ws.p1 = pw->p1; ws.p2 = pw->p2;
    for (size_t n = 0; n <= s->n_steps; n++) o->tf_src[n] = pw->amplitude * wave(&ws, (double)n * o->dt);
    o->tf = 1;
    return 0;
}

/* H corrections from the line's E^n, then the line's H to n+1/2 */
static void tf_after_h(orc_t *o) {
    for (size_t q = 0; q < o->tf_nh; q++) {
        double *f = &o->H[o->tf_hc[q]][o->tf_hw[q]];
        double h = *f;
        for (int t = o->tf_hfirst[q]; t < o->tf_hfirst[q] + o->tf_hcount[q]; t++) {
            int m = o->tf_idx[t];
            const double *w = o->tf_w + 4 * t;
            h = h + o->tf_coef[t] * (w[0] * o->tf_e[m - 1] + w[1] * o->tf_e[m] + w[2] * o->tf_e[m + 1] +
                                     w[3] * o->tf_e[m + 2]);
        }
        *f = h;
    }
    for (size_t m = 0; m + 1 < o->tf_len; m++) o->tf_h[m] = o->tf_h[m] - o->tf_ch * (o->tf_e[m + 1] - o->tf_e[m]);
}

/* the line's E to n+1 (hard source at m = 0) */
static void tf_after_e(orc_t *o, size_t n1, size_t n_steps) {
    for (size_t m = 1; m + 1 < o->tf_len; m++) o->tf_e[m] = o->tf_e[m] - o->tf_ce * (o->tf_h[m] - o->tf_h[m - 1]);
    o->tf_e[0] = o->tf_src[n1 < n_steps ? n1 : n_steps];
}

static int orc_init(orc_t *o, const scn_scene_t *s) {
    memset(o, 0, sizeof(*o));
    o->n[0] = s->nx; o->n[1] = s->ny; o->n[2] = s->nz;
    o->per = s->periodic;
    o->dx = s->dx;
    o->dt = s->courant * (s->dx / (O_C0 * sqrt(3.0)));
    o->total = (s->nx + 1) * (s->ny + 1) * (s->nz + 1);
    for (int c = 0; c < 3; c++) {
        o->E[c] = calloc(o->total, 8);
        o->H[c] = calloc(o->total, 8);
        o->has_ovr[c] = calloc(o->total, 1);
        o->oca[c] = calloc(o->total, 8);
        o->ocb[c] = calloc(o->total, 8);
        if (!o->E[c] || !o->H[c] || !o->has_ovr[c] || !o->oca[c] || !o->ocb[c]) return -1;
    }
    for (int c = 0; c < 2; c++) {
        o->has_t[c] = calloc(o->total, 1);
        o->tm11[c] = calloc(o->total, 8); o->tm12[c] = calloc(o->total, 8);
        o->tm22[c] = calloc(o->total, 8); o->tscale[c] = calloc(o->total, 8);
        if (!o->has_t[c] || !o->tm11[c] || !o->tm12[c] || !o->tm22[c] || !o->tscale[c]) return -1;
    }
    o->id = calloc(o->total, 1);
    if (!o->id) return -1;
    for (int c = 0; c < 3; c++) {
        o->has_t3[c] = calloc(o->total, 1);
        o->t3m[c] = calloc(3 * o->total, 8);
        o->t3s[c] = calloc(o->total, 8);
        if (!o->has_t3[c] || !o->t3m[c] || !o->t3s[c]) return -1;
    }
    for (int c = 0; c < 3; c++) {
        o->dix[c] = malloc(o->total * sizeof(int));
        if (!o->dix[c]) return -1;
        for (size_t q = 0; q < o->total; q++) o->dix[c][q] = -1;
    }
    table_id(o, 1.0, 0.0);
    if (s->npml) {
        o->cpml = 1;
        double eta0 = sqrt(O_MU0 / O_EPS0);
        double sigma_max = -(s->m + 1.0) * log(s->r0) / (2.0 * eta0 * (double)s->npml * o->dx);
        for (int a = 0; a < 3; a++) profiles(o, a, s, sigma_max);
        for (int c = 0; c < 3; c++)
            for (int t = 0; t < 2; t++) {
                o->psiH[c][t] = calloc(o->total, 8);
                o->psiE[c][t] = calloc(o->total, 8);
                if (!o->psiH[c][t] || !o->psiE[c][t]) return -1;
            }
    }
    /* scene: boxes clear overrides inside them (materials.c:476-528) */
    for (size_t q = 0; q < s->n_boxes; q++) {
        const scn_box_t *b = &s->boxes[q];
        int id = table_id(o, b->eps_r, b->sigma);
        if (id < 0) return -1;
        size_t i1 = b->i1, j1 = b->j1, k1 = b->k1;
        if (periodic(o, 0) && i1 > o->n[0]) i1 = o->n[0];
        if (periodic(o, 1) && j1 > o->n[1]) j1 = o->n[1];
        if (periodic(o, 2) && k1 > o->n[2]) k1 = o->n[2];
        for (size_t i = b->i0; i < i1; i++)
            for (size_t j = b->j0; j < j1; j++)
                for (size_t k = b->k0; k < k1; k++) {
                    /* keys of the box use unwrapped coordinates */
                    size_t raw = (i * (o->n[1] + 1) + j) * (o->n[2] + 1) + k;
                    size_t w = at(o, i, j, k);
                    o->id[w] = (uint8_t)id;
                    for (int c = 0; c < 3; c++) o->has_ovr[c][raw] = 0, o->dix[c][raw] = -1;
                    for (int c = 0; c < 2; c++) o->has_t[c][raw] = 0;
                }
    }
    for (size_t q = 0; q < s->n_comps; q++) {
        const scn_comp_t *c = &s->comps[q];
        size_t w = at(o, c->i, c->j, c->k);
        if (coeff(o, c->eps_r, c->sigma, &o->oca[c->comp][w], &o->ocb[c->comp][w]) != 0) return -1;
        o->has_ovr[c->comp][w] = 1;
    }
    for (size_t q = 0; q < s->n_tensors; q++) {
        const scn_tensor_t *t = &s->tensors[q];
        size_t w = at(o, t->i, t->j, t->k);
        o->has_t[t->comp][w] = 1;
        o->tm11[t->comp][w] = t->m11;
        o->tm12[t->comp][w] = t->m12;
        o->tm22[t->comp][w] = t->m22;
        o->tscale[t->comp][w] = o->dt / (O_EPS0 * o->dx);
    }
    for (size_t q = 0; q < s->n_disp; q++) {
        const scn_disp_t *d = &s->disp[q];
        if (d->i > o->n[0]) continue;  /* model-only entry (sphere material) */
        if (set_disp(o, d->comp, at(o, d->i, d->j, d->k), d) != 0) return -1;
    }
    /* spheres in list order (oracle/sphere_raster.h) */
    if (s->n_spheres) {
        for (size_t q = 0; q < s->n_spheres; q++)
            if (s->spheres[q].disp < 0 && table_id(o, s->spheres[q].eps_r, s->spheres[q].sigma) < 0) return -1;
        sr_target_t tg = {o, sr_bg, sr_fill, sr_fill_disp, sr_sample, sr_sample_disp, sr_sample_t3};
        if (sr_rasterise(s, o->n, o->per, sr_canon, o, &tg) != 0) return -1;
    }
    for (size_t q = 0; q < s->n_tensor3; q++) {
        const scn_tensor3_t *t = &s->tensor3[q];
        size_t w = at(o, t->i, t->j, t->k);
        o->has_t3[t->comp][w] = 1;
        memcpy(o->t3m[t->comp] + 3 * w, t->m, 3 * sizeof(double));
        o->t3s[t->comp][w] = t->sigma;
    }
    if (s->plane_wave && tf_init(o, s) != 0) return -1;
    return 0;
}

/* cpml.h:46-51 */
static double stretch(double diff, double kinv, double b, double a, double dx, double *psi) {
    *psi = b * (*psi) + a * diff;
    return diff * kinv + dx * (*psi);
}

/* H update (cpml.c:176-219).  Component c: H_c -= cb (dA - dB) with
 * A = d E_{c+2} / d x_{c+1} and B = d E_{c+1} / d x_{c+2} (forward). */
static void update_h(orc_t *o) {
    const double cb = o->dt / (O_MU0 * o->dx);
    for (int c = 0; c < 3; c++) {
        const int fa = (c + 2) % 3, axa = (c + 1) % 3;
        const int fb = (c + 1) % 3, axb = (c + 2) % 3;
        size_t lim[3] = {o->n[0], o->n[1], o->n[2]};
        if (!periodic(o, c)) lim[c]++;
        for (size_t i = 0; i < lim[0]; i++)
            for (size_t j = 0; j < lim[1]; j++)
                for (size_t k = 0; k < lim[2]; k++) {
                    size_t p[3] = {i, j, k};
                    size_t here = at(o, i, j, k);
                    size_t qa[3] = {i, j, k}, qb[3] = {i, j, k};
                    qa[axa]++;
                    qb[axb]++;
                    double dA = o->E[fa][at(o, qa[0], qa[1], qa[2])] - o->E[fa][here];
                    double dB = o->E[fb][at(o, qb[0], qb[1], qb[2])] - o->E[fb][here];
                    double tA = dA, tB = dB;
                    if (o->cpml) {
                        tA = stretch(dA, o->kh[axa][p[axa]], o->bh[axa][p[axa]], o->ah[axa][p[axa]], o->dx,
                                     &o->psiH[c][0][here]);
                        tB = stretch(dB, o->kh[axb][p[axb]], o->bh[axb][p[axb]], o->ah[axb][p[axb]], o->dx,
                                     &o->psiH[c][1][here]);
                    }
                    o->H[c][here] -= cb * (tA - tB);
                }
    }
}

/* materials.c:836-845 */
static double pair_w(double x11, double x12, double x22, double y11, double y12, double y22) {
    double rx = (x12 / sqrt(x11)) / sqrt(x22);
    double ry = (y12 / sqrt(y11)) / sqrt(y22);
    double rho = 0.5 * rx + 0.5 * ry;
    return (0.25 * rho * sqrt(x11)) * sqrt(y11);
}

/* materials.c:847-903 */
static void tensor_edge(orc_t *o, int c, size_t i, size_t j, size_t k) {
    size_t w = at(o, i, j, k);
    const double m11 = o->tm11[c][w], m12 = o->tm12[c][w], m22 = o->tm22[c][w];
    double *Hz = o->H[2];
    double value;
    if (c == 0) {
        size_t ip = (i + 1 == o->n[0]) ? 0 : i + 1, jm = back(j, o->n[1]);
        size_t ni[4] = {i, ip, i, ip}, nj[4] = {j, j, jm, jm};
        value = m11 * (Hz[at(o, i, j, k)] - Hz[at(o, i, jm, k)]);
        for (int q = 0; q < 4; q++) {
            size_t ow = at(o, ni[q], nj[q], k);
            if (!o->has_t[1][ow]) continue;
            size_t um = back(ni[q], o->n[0]);
            double curl = -(Hz[at(o, ni[q], nj[q], k)] - Hz[at(o, um, nj[q], k)]);
            value += pair_w(m11, m12, m22, o->tm11[1][ow], o->tm12[1][ow], o->tm22[1][ow]) * curl;
        }
        o->E[0][w] += o->tscale[0][w] * value;
    } else {
        size_t im = back(i, o->n[0]), jp = (j + 1 == o->n[1]) ? 0 : j + 1;
        size_t ni[4] = {i, im, i, im}, nj[4] = {j, j, jp, jp};
        value = -m11 * (Hz[at(o, i, j, k)] - Hz[at(o, im, j, k)]);
        for (int q = 0; q < 4; q++) {
            size_t ow = at(o, ni[q], nj[q], k);
            if (!o->has_t[0][ow]) continue;
            size_t vm = back(nj[q], o->n[1]);
            double curl = Hz[at(o, ni[q], nj[q], k)] - Hz[at(o, ni[q], vm, k)];
            value += pair_w(o->tm11[0][ow], o->tm12[0][ow], o->tm22[0][ow], m11, m12, m22) * curl;
        }
        o->E[1][w] += o->tscale[1][w] * value;
    }
}

/* Curl difference of E component b at cell (i, j, k): the unstretched
 * (dA - dB) of the E update below. */
static double curl_d(const orc_t *o, int b, size_t i, size_t j, size_t k) {
    const int fa = (b + 2) % 3, axa = (b + 1) % 3, fb = (b + 1) % 3, axb = (b + 2) % 3;
    size_t pa[3] = {i, j, k}, pb[3] = {i, j, k};
    pa[axa] = back(pa[axa], o->n[axa]);
    pb[axb] = back(pb[axb], o->n[axb]);
    double tA = o->H[fa][at(o, i, j, k)] - o->H[fa][at(o, pa[0], pa[1], pa[2])];
    double tB = o->H[fb][at(o, i, j, k)] - o->H[fb][at(o, pb[0], pb[1], pb[2])];
    return tA - tB;
}

/* Full 3x3 sample: value = m_cc D_c, then for each b != c (ascending)
 * value += m_cb (0.25 (((D_b(w) + D_b(w+e_c)) + D_b(w-e_b)) + D_b(w+e_c-e_b)));
 * E_c = ca E_c + s value with the loss of sigma at the component's
 * permittivity 1/m_cc (rfsyn's make_coeff form, materials.c:92-125):
 * loss = sigma dt / (2 eps0 / m_cc), s = dt/(eps0 dx) / (1 + loss),
 * ca = (1 - loss) / (1 + loss). */
static void tensor3(orc_t *o, int c, size_t i, size_t j, size_t k) {
    size_t w = at(o, i, j, k);
    const double *r = o->t3m[c] + 3 * w;
    double value = r[c] * curl_d(o, c, i, j, k);
    for (int b = 0; b < 3; b++) {
        if (b == c) continue;
        size_t p0[3] = {i, j, k}, p1[3] = {i, j, k};
        p1[c] += 1;
        size_t p2[3] = {p0[0], p0[1], p0[2]}, p3[3] = {p1[0], p1[1], p1[2]};
        p2[b] = back(p2[b], o->n[b]);
        p3[b] = back(p3[b], o->n[b]);
        double s4 = ((curl_d(o, b, p0[0], p0[1], p0[2]) + curl_d(o, b, p1[0], p1[1], p1[2])) +
                     curl_d(o, b, p2[0], p2[1], p2[2])) +
                    curl_d(o, b, p3[0], p3[1], p3[2]);
        value = value + r[b] * (0.25 * s4);
    }
    const double loss = (o->t3s[c][w] * o->dt) / (2.0 * (O_EPS0 / r[c]));
    const double sc = (o->dt / (O_EPS0 * o->dx)) / (1.0 + loss), ca = (1.0 - loss) / (1.0 + loss);
    o->E[c][w] = ca * o->E[c][w] + sc * value;
}

/* E update (materials.c:911-1060).  Component c: E_c = Ca E_c + Cb (dA - dB)
 * with A = d H_{c+2} / d x_{c+1}, B = d H_{c+1} / d x_{c+2} (backward);
 * index 0 of an axis other than c is swept only when that axis is periodic. */
static void update_e(orc_t *o) {
    for (int c = 0; c < 3; c++) {
        const int fa = (c + 2) % 3, axa = (c + 1) % 3;
        const int fb = (c + 1) % 3, axb = (c + 2) % 3;
        size_t lo[3];
        for (int a = 0; a < 3; a++) lo[a] = (a == c || periodic(o, a)) ? 0 : 1;
        for (size_t i = lo[0]; i < o->n[0]; i++)
            for (size_t j = lo[1]; j < o->n[1]; j++)
                for (size_t k = lo[2]; k < o->n[2]; k++) {
                    size_t here = at(o, i, j, k);
                    if (o->has_t3[c][here]) {
                        tensor3(o, c, i, j, k);
                        continue;
                    }
                    if (c < 2 && o->has_t[c][here]) {
                        tensor_edge(o, c, i, j, k);
                        continue;
                    }
                    size_t p[3] = {i, j, k};
                    size_t qa[3] = {i, j, k}, qb[3] = {i, j, k};
                    qa[axa] = back(qa[axa], o->n[axa]);
                    qb[axb] = back(qb[axb], o->n[axb]);
                    double ca, cb;
                    if (o->has_ovr[c][here]) { ca = o->oca[c][here]; cb = o->ocb[c][here]; }
                    else { ca = o->tca[o->id[here]]; cb = o->tcb[o->id[here]]; }
                    double tA = o->H[fa][here] - o->H[fa][at(o, qa[0], qa[1], qa[2])];
                    double tB = o->H[fb][here] - o->H[fb][at(o, qb[0], qb[1], qb[2])];
                    if (o->cpml) {
                        tA = stretch(tA, o->km[axa][p[axa]], o->bm[axa][p[axa]], o->am[axa][p[axa]], o->dx,
                                     &o->psiE[c][0][here]);
                        tB = stretch(tB, o->km[axb][p[axb]], o->bm[axb][p[axb]], o->am[axb][p[axb]], o->dx,
                                     &o->psiE[c][1][here]);
                    }
                    if (o->dix[c][here] >= 0) {
                        /* polarisation-current ADE (Debye / Lorentz poles) */
                        const double *r = o->drec + 16 * (size_t)o->dix[c][here];
                        double *st = o->dst + 5 * (size_t)o->dix[c][here];
                        double v = o->E[c][here], em = st[4];
                        double en = r[0] * v + r[1] * (tA - tB);
                        en = en + r[2] * em;
                        int np = (int)r[3];
                        for (int q = 0; q < np; q++) en = en - (r[5 + 6 * q] * st[q] + r[6 + 6 * q] * st[2 + q]);
                        for (int q = 0; q < np; q++) {
                            const double *w = r + 4 + 6 * q;
                            double eref = w[0] != 0.0 ? em : v;
                            double jn = (w[3] * st[q] + w[4] * st[2 + q]) + w[5] * (en - eref);
                            st[2 + q] = st[q];
                            st[q] = jn;
                        }
                        st[4] = v;
                        o->E[c][here] = en;
                        continue;
                    }
                    o->E[c][here] = ca * o->E[c][here] + cb * (tA - tB);
                    if (o->tf && o->tf_efirst[c][here] >= 0) {
                        double v = o->E[c][here];
                        for (int t = o->tf_efirst[c][here]; t < o->tf_efirst[c][here] + o->tf_ecount[c][here]; t++) {
                            int m = o->tf_idx[t];
                            const double *w = o->tf_w + 4 * t;
                            v = v + o->tf_coef[t] * (w[0] * o->tf_h[m - 1] + w[1] * o->tf_h[m] +
                                                     w[2] * o->tf_h[m + 1] + w[3] * o->tf_h[m + 2]);
                        }
                        o->E[c][here] = v;
                    }
                }
    }
}

/* source.c:8-26 */
static double wave(const scn_source_t *s, double t) {
    if (s->waveform == 0) {
        double u = (t - s->p0) / s->p1;
        return -2.0 * u * exp(-u * u);
    }
    if (s->waveform == 1) {
        double a = O_PI * s->p0 * (t - s->p1);
        double a2 = a * a;
        return (1.0 - 2.0 * a2) * exp(-a2);
    }
    double u = (t - s->p1) / s->p2;
    double env = exp(-u * u);
    return env * sin(2.0 * O_PI * s->p0 * (t - s->p1));
}

static double *field(orc_t *o, int comp) { return comp < 3 ? o->E[comp] : o->H[comp - 3]; }

static void step(orc_t *o, const scn_scene_t *s, size_t n) {
    update_h(o);
    if (o->tf) tf_after_h(o);
    double t = ((double)n + s->src_t_offset) * o->dt;
    for (size_t q = 0; q < s->n_sources; q++) {
        const scn_source_t *src = &s->sources[q];
        if (src->i > o->n[0] || src->j > o->n[1] || src->k > o->n[2] || src->comp > 2) continue;
        double v = src->amplitude * wave(src, t);
        double *f = o->E[src->comp];
        size_t w = at(o, src->i, src->j, src->k);
        if (src->mode == 0) f[w] += v;
        else f[w] = v;
    }
    update_e(o);
    if (o->tf) tf_after_e(o, n + 1, s->n_steps);
}

/* Mean of one component over a whole plane (plane probe), FP64, summed in
 * the order of the GPU's reduction so FP64 runs compare bit for bit: the
 * points t = u n_v + v (u outer) are cut into chunks of 1024; within a
 * chunk, point t goes to partial sum (t - chunk start) mod 256 in increasing
 * t; each group of 32 partials is reduced by halving (p[l] += p[l + h] for
 * h = 16, 8, 4, 2, 1) and the 8 group sums are added in order, giving the
 * chunk's sum; the chunks' sums are added in chunk order; the total is
 * divided by n_u n_v. */
static double plane_mean(const orc_t *o, const scn_plane_t *pl) {
    const int a = pl->axis, u = a == 0 ? 1 : 0, v = a == 2 ? 1 : 2;
    const double *f = field((orc_t *)o, pl->comp);
    const size_t nu = o->n[u], nv = o->n[v], npts = nu * nv;
    double total = 0.0;
    for (size_t t0 = 0; t0 < npts; t0 += 1024) {
        const size_t t1 = t0 + 1024 < npts ? t0 + 1024 : npts;
        double part[256];
        for (int t = 0; t < 256; t++) part[t] = 0.0;
        for (size_t t = t0; t < t1; t++) {
            size_t ijk[3];
            ijk[a] = pl->index;
            ijk[u] = t / nv;
            ijk[v] = t % nv;
            part[(t - t0) % 256] = part[(t - t0) % 256] + f[at(o, ijk[0], ijk[1], ijk[2])];
        }
        double chunk = 0.0;
        for (int w = 0; w < 8; w++) {
            double *g = part + 32 * w;
            for (int h = 16; h > 0; h >>= 1)
                for (int l = 0; l < 32 - h; l++) g[l] = g[l] + g[l + h];
            chunk = chunk + g[0];
        }
        total = total + chunk;
    }
    return total / (double)npts;
}

/* Runs the scene; probe_td (n_probes + n_planes) * n_steps, dft_re/im
 * (n_probes + n_planes) * n_freqs: point probes, then plane probes. */
int orc_run(const scn_scene_t *s, double *probe_td, double *dft_re, double *dft_im) {
    orc_t o;
    int rc = -1;
    const size_t ns = s->n_probes + s->n_planes;
    if (orc_init(&o, s) != 0) goto out;
    if (dft_re && dft_im && s->n_freqs) {
        memset(dft_re, 0, ns * s->n_freqs * 8);
        memset(dft_im, 0, ns * s->n_freqs * 8);
    }
    for (size_t n = 0; n < s->n_steps; n++) {
        step(&o, s, n);
        double td = ((double)n + s->dft_t_offset) * o.dt;
        for (size_t q = 0; q < ns; q++) {
            double v;
            if (q < s->n_probes) {
                const scn_probe_t *p = &s->probes[q];
                v = field(&o, p->comp)[at(&o, p->i, p->j, p->k)];
            } else {
                v = plane_mean(&o, &s->planes[q - s->n_probes]);
            }
            if (probe_td) probe_td[q * s->n_steps + n] = v;
            if (dft_re && dft_im)
                for (size_t f = 0; f < s->n_freqs; f++) {
                    double w = 2.0 * O_PI * s->freqs[f];
                    dft_re[q * s->n_freqs + f] += v * cos(w * td) * o.dt;
                    dft_im[q * s->n_freqs + f] -= v * sin(w * td) * o.dt;
                }
        }
    }
    rc = 0;
out:
    orc_free(&o);
    return rc;
}

int orc_run_fields(const scn_scene_t *s, const double *initial, double *fields_out) {
    orc_t o;
    int rc = -1;
    if (orc_init(&o, s) != 0) goto out;
    if (initial)
        for (int c = 0; c < 6; c++) memcpy(field(&o, c), initial + c * o.total, o.total * 8);
    for (size_t n = 0; n < s->n_steps; n++) {
        update_h(&o);
        update_e(&o);
    }
    for (int c = 0; c < 6; c++) memcpy(fields_out + c * o.total, field(&o, c), o.total * 8);
    rc = 0;
out:
    orc_free(&o);
    return rc;
}

/* Energy audit after the scene's n_steps steps, in the loop order of rfsyn's
 * validate_long_term_stability.c:166-209 (eps = dt / (dx Cb) from the
 * component's scalar coefficient, :74-75) and, for the modified energy, of
 * audit_periodic_energy.c:53-62 applied to the last step: E^{n-1} energy and
 * 0.5 mu0 H^{n-3/2} . H^{n-1/2}.  q: electric, magnetic, electric and
 * magnetic over planes x_lo <= i < x_hi, electric of E^{n-1}, cross term,
 * max |E|, max |H|, non-finite count (energies times dx^3). */
int orc_energy(const scn_scene_t *s, int x_lo, int x_hi, double *q) {
    orc_t o;
    int rc = -1;
    double *prev = NULL;
    if (orc_init(&o, s) != 0) goto out;
    prev = malloc(6 * o.total * sizeof(double));
    if (!prev) goto out;
    for (size_t n = 0; n < s->n_steps; n++) {
        if (n + 1 == s->n_steps)
            for (int c = 0; c < 6; c++) memcpy(prev + c * o.total, field(&o, c), o.total * 8);
        step(&o, s, n);
    }
    for (int v = 0; v < 9; v++) q[v] = 0.0;
    for (size_t i = 0; i < o.n[0]; i++)
        for (size_t j = 0; j < o.n[1]; j++)
            for (size_t k = 0; k < o.n[2]; k++) {
                size_t w = at(&o, i, j, k);
                int inside = (int)i >= x_lo && (int)i < x_hi;
                for (int c = 0; c < 3; c++) {
                    double cb = o.has_ovr[c][w] ? o.ocb[c][w] : o.tcb[o.id[w]];
                    double eps = o.dt / (o.dx * cb);
                    double ev = o.E[c][w], hv = o.H[c][w];
                    double ep = prev[c * o.total + w], hp = prev[(3 + c) * o.total + w];
                    if (!isfinite(ev)) q[8] += 1.0;
                    if (!isfinite(hv)) q[8] += 1.0;
                    q[6] = fmax(q[6], fabs(ev));
                    q[7] = fmax(q[7], fabs(hv));
                    double ue = 0.5 * eps * ev * ev, uh = 0.5 * O_MU0 * hv * hv;
                    q[0] += ue;
                    q[1] += uh;
                    if (inside) q[2] += ue, q[3] += uh;
                    q[4] += 0.5 * eps * ep * ep;
                    q[5] += 0.5 * O_MU0 * hp * hv;
                }
            }
    double vol = pow(o.dx, 3.0);
    for (int v = 0; v < 6; v++) q[v] *= vol;
    rc = 0;
out:
    free(prev);
    orc_free(&o);
    return rc;
}

/* dt of a scene (grid.c:27-28) */
double orc_dt(double dx, double courant) { return courant * (dx / (O_C0 * sqrt(3.0))); }
