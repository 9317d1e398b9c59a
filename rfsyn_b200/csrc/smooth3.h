/*
 * smooth3.h -- the smoothed permittivity of a cell cut by a planar
 * interface, in three dimensions (FP64).  Shared by the host entry point
 * fdtd_b200_subpixel_tensor3 (host/subpixel.c) and the GPU kernels that
 * smooth sphere and slab surfaces (engine.cu); plain C, compiled for the host
 * by gcc and for the device by nvcc.
 *
 * A fraction f of the cell holds eps_in, the rest eps_bg (3x3, symmetric
 * positive definite), and the interface has unit normal n.  Kottke,
 * Farjadpour and Johnson (Phys. Rev. E 77, 036611, 2008, eqs. 23-24) average
 * not eps but its transform tau in the frame (n, p, q) of the normal:
 *   tau_nn = -1/e_nn,  tau_na = e_na/e_nn,  tau_an = e_an/e_nn,
 *   tau_ab = e_ab - e_an e_nb / e_nn            (a, b in {p, q}),
 * then invert the transform of <tau> = (1-f) tau(eps_bg) + f tau(eps_in).
 * For two isotropic media this is rfsyn's rule (engine/fdtd/subpixel_te.c:
 * 106-132) taken to three dimensions: eps_nn = 1/<1/eps> (layers in series
 * along the normal), eps_pp = eps_qq = <eps> (in parallel along the
 * interface), i.e. eps^-1 = <1/eps> n n^T + (1/<eps>) (I - n n^T).  The
 * caller gets M = eps^-1, the relative inverse permittivity the 3x3 update
 * multiplies the curl with.
 */
#ifndef RFB_SMOOTH3_H
#define RFB_SMOOTH3_H

#ifdef __CUDACC__
#define RFB_HD __host__ __device__ __forceinline__
#else
#define RFB_HD static inline
#endif

/* Inverse of a symmetric 3x3 matrix by its adjugate; 0, or -1 when its
 * determinant is not positive (not positive definite) or not finite. */
RFB_HD int rfb_sm_inverse(const double a[9], double out[9]) {
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(det > 0.0) || !(det < 1e300)) return -1;
    out[0] = c00 / det;
    out[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    out[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    out[3] = c01 / det;
    out[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    out[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    out[6] = c02 / det;
    out[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    out[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    return 0;
}

/* Orthonormal frame with first vector n (unit): r[3*axis + m] is component
 * `axis` of frame vector m (m = 0: n, 1: p, 2: q).  p is n crossed with the
 * coordinate axis least aligned with n, normalised; q = n x p. */
RFB_HD void rfb_sm_frame(const double n[3], double r[9]) {
    const double ax = n[0] < 0 ? -n[0] : n[0], ay = n[1] < 0 ? -n[1] : n[1], az = n[2] < 0 ? -n[2] : n[2];
    const int e = (ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2);
    double p[3];
    /* p = e_axis x n */
    if (e == 0) { p[0] = 0.0; p[1] = -n[2]; p[2] = n[1]; }
    else if (e == 1) { p[0] = n[2]; p[1] = 0.0; p[2] = -n[0]; }
    else { p[0] = -n[1]; p[1] = n[0]; p[2] = 0.0; }
    const double pl = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    p[0] /= pl; p[1] /= pl; p[2] /= pl;
    const double q[3] = {n[1] * p[2] - n[2] * p[1], n[2] * p[0] - n[0] * p[2], n[0] * p[1] - n[1] * p[0]};
    for (int a = 0; a < 3; a++) {
        r[3 * a] = n[a];
        r[3 * a + 1] = p[a];
        r[3 * a + 2] = q[a];
    }
}

/* out = R^T e R (to the frame) when `to_frame`, else R e R^T (back). */
RFB_HD void rfb_sm_rotate(const double r[9], const double e[9], double out[9], int to_frame) {
    double t[9];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double s = 0.0;
            for (int m = 0; m < 3; m++) s += (to_frame ? r[3 * m + a] : r[3 * a + m]) * e[3 * m + b];
            t[3 * a + b] = s;
        }
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double s = 0.0;
            for (int m = 0; m < 3; m++) s += t[3 * a + m] * (to_frame ? r[3 * m + b] : r[3 * b + m]);
            out[3 * a + b] = s;
        }
}

/* The tau transform of e (in the normal's frame, index 0 = n), added to
 * acc with weight w. */
RFB_HD void rfb_sm_tau_acc(const double e[9], double w, double acc[9]) {
    const double inn = 1.0 / e[0];
    acc[0] += w * (-inn);
    for (int a = 1; a < 3; a++) {
        acc[a] += w * (e[a] * inn);          /* tau_na */
        acc[3 * a] += w * (e[3 * a] * inn);  /* tau_an */
        for (int b = 1; b < 3; b++) acc[3 * a + b] += w * (e[3 * a + b] - e[3 * a] * e[b] * inn);
    }
}

/* Smoothed relative inverse permittivity M (9 values, row-major) of a cell
 * with fraction f of eps_in behind an interface of normal n (need not be
 * unit), the rest eps_bg.  0, or -1 for an invalid argument (f outside
 * [0, 1], a zero normal, a permittivity that is not positive definite). */
RFB_HD int rfb_sm_mix(double f, const double eps_bg[9], const double eps_in[9], const double n_in[3], double m[9]) {
    if (!(f >= 0.0 && f <= 1.0)) return -1;
    const double nl = sqrt(n_in[0] * n_in[0] + n_in[1] * n_in[1] + n_in[2] * n_in[2]);
    if (!(nl > 0.0) || !(nl < 1e300)) return -1;
    const double n[3] = {n_in[0] / nl, n_in[1] / nl, n_in[2] / nl};
    double chk[9];
    if (rfb_sm_inverse(eps_bg, chk) != 0 || rfb_sm_inverse(eps_in, chk) != 0) return -1;
    if (f == 0.0) return rfb_sm_inverse(eps_bg, m);
    if (f == 1.0) return rfb_sm_inverse(eps_in, m);
    double r[9], eb[9], ei[9], tau[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ef[9], e[9];
    rfb_sm_frame(n, r);
    rfb_sm_rotate(r, eps_bg, eb, 1);
    rfb_sm_rotate(r, eps_in, ei, 1);
    if (!(eb[0] > 0.0) || !(ei[0] > 0.0)) return -1;
    rfb_sm_tau_acc(eb, 1.0 - f, tau);
    rfb_sm_tau_acc(ei, f, tau);
    /* invert the transform: e_nn = -1/tau_nn, e_na = -tau_na/tau_nn,
     * e_an = -tau_an/tau_nn, e_ab = tau_ab - tau_an tau_nb / tau_nn */
    const double it = 1.0 / tau[0];
    ef[0] = -it;
    for (int a = 1; a < 3; a++) {
        ef[a] = -tau[a] * it;
        ef[3 * a] = -tau[3 * a] * it;
        for (int b = 1; b < 3; b++) ef[3 * a + b] = tau[3 * a + b] - tau[3 * a] * tau[b] * it;
    }
    rfb_sm_rotate(r, ef, e, 0);
    /* symmetric by construction up to rounding: average the halves */
    for (int a = 0; a < 3; a++)
        for (int b = a + 1; b < 3; b++) e[3 * a + b] = e[3 * b + a] = 0.5 * (e[3 * a + b] + e[3 * b + a]);
    return rfb_sm_inverse(e, m);
}

#endif /* RFB_SMOOTH3_H */
