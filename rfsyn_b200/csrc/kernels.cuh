// kernels.cuh -- sm_100a kernels of the FDTD time loop.
//
// One templated source serves FP64 (bit-for-bit with rfsyn's CPU loops: the
// same operation order, every multiply and add rounded separately through
// __dmul_rn/__dadd_rn so nothing is contracted into an FMA) and FP32 (the
// same order, rounded separately through __fmul_rn/__fadd_rn: every sweep
// variant the autotuner may pick yields bit-identical FP32 fields, so runs
// are reproducible whatever variant a process picks).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rfb {

__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xs(float a, float b) { return __fsub_rn(a, b); }

// The update expressions H - cbh d, Ca E + Cb t and rfsyn's cpml_term
// (psi' = b psi + a d, result d kappa_inv + dx psi'), every product and sum
// rounded on its own in rfsyn's operation order (FP64 bit-exact with rfsyn;
// FP32 identical in every kernel, so all sweep variants agree bit for bit).
// Contracting the FP32 forms into fused multiply-adds measured no faster on
// B200: the edge sweep gained register spills.
template <typename T>
__device__ __forceinline__ T upd_h(T h, T cbh, T d) { return xs(h, xm(cbh, d)); }
template <typename T>
__device__ __forceinline__ T upd_e(T ca, T e, T cb, T t) { return xa(xm(ca, e), xm(cb, t)); }
template <typename T>
__device__ __forceinline__ T cpml_psi(T b, T psi, T ac, T d) { return xa(xm(b, psi), xm(ac, d)); }
template <typename T>
__device__ __forceinline__ T cpml_out(T d, T kinv, T dx, T p) { return xa(xm(d, kinv), xm(dx, p)); }

// The incident line at a TF/SF term: cubic Lagrange interpolation through
// x[-1] .. x[2] with the term's weights, ((w0 x[-1] + w1 x[0]) + w2 x[1]) + w3 x[2].
template <typename T>
__device__ __forceinline__ T tf_interp(const T *w, const T *x) {
    return xa(xa(xa(xm(w[0], x[-1]), xm(w[1], x[0])), xm(w[2], x[1])), xm(w[3], x[2]));
}

constexpr int LIST_CODE = 255;
constexpr int MAX_SKIP = 4;

// psi arrays (slab storage).  H: hx_y hx_z hy_z hy_x hz_x hz_y,
// E: ex_y ex_z ey_z ey_x ez_x ez_y.  Axis of the slab of each array:
__host__ __device__ constexpr int psi_axis_h(int p) { return p == 0 ? 1 : p == 1 ? 2 : p == 2 ? 2 : p == 3 ? 0 : p == 4 ? 0 : 1; }
__host__ __device__ constexpr int psi_axis_e(int p) { return psi_axis_h(p); }

template <typename T>
struct Args {
    int nx, ny, nz;
    unsigned per;
    long long pitch, plane;  // plane = (ny+1)*pitch
    T *E[3], *H[3];          // inputs (split: updated in place)
    T *Eo[3], *Ho[3];        // outputs (split: same as inputs)
    T cbh, dx;
    // CPML
    int cpml_on;
    const T *kinv_m[3], *b_m[3], *a_m[3];
    const T *kinv_h[3], *b_h[3], *a_h[3];
    int lo_m[3], hi_m[3], ns_m[3];
    int lo_h[3], hi_h[3], ns_h[3];
    T *psi_e[6];
    T *psi_hi[6], *psi_ho[6];
    // scene
    const uint8_t *codes;    // NULL: table entry 0 everywhere except skip cells
    const T *tca, *tcb;      // 256 entries
    int n_skip;
    long long skip[MAX_SKIP];
    // interface list
    int n_cells;
    // NULL, or the n_work entries the per-entry update takes (the others
    // belong to cells k_list_cells updates whole)
    const int *l_work;
    int n_work;
    const int *lc_ijk;
    const uint8_t *l_kind;
    const T *l_ca, *l_cb;
    const int *l_tix, *l_src, *l_aix;
    const T *ade_c;          // RFB_ADE_NC coefficients per dispersive model
    T *ade_s;                // 5 state values per list entry: J0 J1 J0- J1- E-
    const T *t_m11, *t_scale, *t_w;
    const int *t_main, *t_nq, *t_uv, *t_sign;
    const T *t3;             // 3x3 samples: row of eps_r^-1, then s and ca of E+ = ca E + s value
    // plane-wave boundary: per list entry its first correction term (-1:
    // none) and count; terms coef * (w0 H1D[idx] + w1 H1D[idx + 1])
    const int *tf_first, *tf_count, *tf_idx;
    const T *tf_coef, *tf_w;  // 4 cubic weights per term
    const T *inc_h;          // the incident line's H at n + 1/2
    // sources
    const T *src_val;
    const int *src_hard;
    long long n_steps;
    const int *d_step;
};

template <typename T>
__device__ __forceinline__ long long cidx(const Args<T> &a, int i, int j, int k) {
    return ((long long)i * (a.ny + 1) + j) * a.pitch + k;
}

__device__ __forceinline__ int slab_of(int q, int lo, int hi) {
    return q < lo ? q : (q >= hi ? lo + (q - hi) : -1);
}

// Index of slab cell s of a psi array whose slab axis is `axis`.
template <typename T>
__device__ __forceinline__ long long psi_idx(const Args<T> &a, int axis, int ns, int s, int i, int j, int k) {
    if (axis == 0) return ((long long)s * (a.ny + 1) + j) * a.pitch + k;
    if (axis == 1) return ((long long)i * ns + s) * a.pitch + k;
    return ((long long)i * (a.ny + 1) + j) * ns + s;
}

// rfsyn's cpml_term (engine/fdtd/cpml.h:46-51): psi = b psi + a diff;
// returns diff kappa_inv + dx psi.
template <typename T>
__device__ __forceinline__ T cpml_step(T diff, T kinv, T b, T ac, T dx, T psi_old, T *psi_new) {
    T p = cpml_psi(b, psi_old, ac, diff);
    *psi_new = p;
    return cpml_out(diff, kinv, dx, p);
}

// Stretched difference for an H component along `axis` at position q, using
// psi array p (ping-pong in/out).
template <typename T>
__device__ __forceinline__ T h_term(const Args<T> &a, int p, int axis, int q, T diff, int i, int j, int k) {
    if (!a.cpml_on) return diff;
    int s = slab_of(q, a.lo_h[axis], a.hi_h[axis]);
    if (s < 0) return diff;
    long long pi = psi_idx(a, axis, a.ns_h[axis], s, i, j, k);
    T pn;
    T r = cpml_step(diff, a.kinv_h[axis][q], a.b_h[axis][q], a.a_h[axis][q], a.dx, a.psi_hi[p][pi], &pn);
    a.psi_ho[p][pi] = pn;
    return r;
}

template <typename T>
__device__ __forceinline__ T e_term(const Args<T> &a, int p, int axis, int q, T diff, int i, int j, int k) {
    if (!a.cpml_on) return diff;
    int s = slab_of(q, a.lo_m[axis], a.hi_m[axis]);
    if (s < 0) return diff;
    long long pi = psi_idx(a, axis, a.ns_m[axis], s, i, j, k);
    T pn;
    T r = cpml_step(diff, a.kinv_m[axis][q], a.b_m[axis][q], a.a_m[axis][q], a.dx, a.psi_e[p][pi], &pn);
    a.psi_e[p][pi] = pn;
    return r;
}

// ---- H update (rfsyn cpml.c:176-219; vacuum grid.c:62-90) ----------------
// One thread per padded cell, all three components; reads E and H from the
// input buffers and writes H to the output buffers.
template <typename T>
__device__ __forceinline__ void h_cell(const Args<T> &a, int i, int j, int k) {
    const bool px = a.per & 1u, py = a.per & 2u, pz = a.per & 4u;
    const long long c = cidx(a, i, j, k);
    const int jp = (py && j + 1 == a.ny) ? 0 : j + 1;
    const int kp = (pz && k + 1 == a.nz) ? 0 : k + 1;
    const int ip = (px && i + 1 == a.nx) ? 0 : i + 1;
    if (i < a.nx + (px ? 0 : 1) && j < a.ny && k < a.nz) {
        T dA = xs(a.E[2][cidx(a, i, jp, k)], a.E[2][c]);
        T dB = xs(a.E[1][cidx(a, i, j, kp)], a.E[1][c]);
        T tA = h_term(a, 0, 1, j, dA, i, j, k);
        T tB = h_term(a, 1, 2, k, dB, i, j, k);
        a.Ho[0][c] = upd_h(a.H[0][c], a.cbh, xs(tA, tB));
    }
    if (i < a.nx && j < a.ny + (py ? 0 : 1) && k < a.nz) {
        T dA = xs(a.E[0][cidx(a, i, j, kp)], a.E[0][c]);
        T dB = xs(a.E[2][cidx(a, ip, j, k)], a.E[2][c]);
        T tA = h_term(a, 2, 2, k, dA, i, j, k);
        T tB = h_term(a, 3, 0, i, dB, i, j, k);
        a.Ho[1][c] = upd_h(a.H[1][c], a.cbh, xs(tA, tB));
    }
    if (i < a.nx && j < a.ny && k < a.nz + (pz ? 0 : 1)) {
        T dA = xs(a.E[1][cidx(a, ip, j, k)], a.E[1][c]);
        T dB = xs(a.E[0][cidx(a, i, jp, k)], a.E[0][c]);
        T tA = h_term(a, 4, 0, i, dA, i, j, k);
        T tB = h_term(a, 5, 1, j, dB, i, j, k);
        a.Ho[2][c] = upd_h(a.H[2][c], a.cbh, xs(tA, tB));
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_h_split(Args<T> a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k > a.nz || j > a.ny || i > a.nx) return;
    h_cell(a, i, j, k);
}

// Scalar E update of component comp at (i,j,k): rfsyn materials.c:920-1059.
// `v` is the current E value (source already applied).
template <typename T>
__device__ __forceinline__ T e_scalar(const Args<T> &a, int comp, int i, int j, int k, T v, T ca, T cb) {
    const long long c = cidx(a, i, j, k);
    const int im = i == 0 ? a.nx - 1 : i - 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1;
    const int km = k == 0 ? a.nz - 1 : k - 1;
    T tA, tB;
    if (comp == 0) {
        tA = e_term(a, 0, 1, j, xs(a.Ho[2][c], a.Ho[2][cidx(a, i, jm, k)]), i, j, k);
        tB = e_term(a, 1, 2, k, xs(a.Ho[1][c], a.Ho[1][cidx(a, i, j, km)]), i, j, k);
    } else if (comp == 1) {
        tA = e_term(a, 2, 2, k, xs(a.Ho[0][c], a.Ho[0][cidx(a, i, j, km)]), i, j, k);
        tB = e_term(a, 3, 0, i, xs(a.Ho[2][c], a.Ho[2][cidx(a, im, j, k)]), i, j, k);
    } else {
        tA = e_term(a, 4, 0, i, xs(a.Ho[1][c], a.Ho[1][cidx(a, im, j, k)]), i, j, k);
        tB = e_term(a, 5, 1, j, xs(a.Ho[0][c], a.Ho[0][cidx(a, i, jm, k)]), i, j, k);
    }
    return upd_e(ca, v, cb, xs(tA, tB));
}

template <typename T>
__device__ __forceinline__ bool e_updated(const Args<T> &a, int comp, int i, int j, int k) {
    const int i0 = (a.per & 1u) ? 0 : 1, j0 = (a.per & 2u) ? 0 : 1, k0 = (a.per & 4u) ? 0 : 1;
    if (i >= a.nx || j >= a.ny || k >= a.nz) return false;
    if (comp != 0 && i < i0) return false;
    if (comp != 1 && j < j0) return false;
    if (comp != 2 && k < k0) return false;
    return true;
}

// ---- bulk E update (cells not on the interface list) ---------------------
template <typename T>
__global__ void __launch_bounds__(256) k_e_split(Args<T> a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= a.nz || j >= a.ny || i >= a.nx) return;
    const long long c = cidx(a, i, j, k);
    int code = 0;
    if (a.codes) {
        code = a.codes[c];
        if (code == LIST_CODE) return;
    } else {
        for (int s = 0; s < a.n_skip; s++)
            if (a.skip[s] == c) return;
    }
    const T ca = a.tca[code], cb = a.tcb[code];
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
        if (e_updated(a, comp, i, j, k))
            a.Eo[comp][c] = e_scalar(a, comp, i, j, k, a.E[comp][c], ca, cb);
    }
}

// Dispersive E update (record layout of rfb_ade_record):
//   E+ = ca E + cb (dA - dB) + ce E- - sum_p (cj J_p + cjm J_p-)
//   J_p+ = aJ J_p + aJm J_p- + aE (E+ - E_ref), E_ref = E (Debye), E- (Lorentz)
// The ADE update of one dispersive sample from its two curl terms: r is
// the model's record (Ca-like, Cb-like and E-history coefficients, the pole
// count, 6 per pole), v the sample's E before the step, st its 5 state
// values (pole currents now and one step back, E one step back), updated in
// place.  At most two poles (RFB_ADE_NC = 4 + 6 x 2).
template <typename T>
__device__ __forceinline__ T ade_core(const T *r, T v, T tA, T tB, T *st) {
    const T em = st[4];
    T en = xa(xm(r[0], v), xm(r[1], xs(tA, tB)));
    en = xa(en, xm(r[2], em));
    const int np = (int)r[3];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        if (p >= np) break;
        const T *w = r + 4 + 6 * p;
        en = xs(en, xa(xm(w[1], st[p]), xm(w[2], st[2 + p])));
    }
#pragma unroll
    for (int p = 0; p < 2; p++) {
        if (p >= np) break;
        const T *w = r + 4 + 6 * p;
        const T eref = (w[0] != T(0)) ? em : v;
        const T jn = xa(xa(xm(w[3], st[p]), xm(w[4], st[2 + p])), xm(w[5], xs(en, eref)));
        st[2 + p] = st[p];
        st[p] = jn;
    }
    st[4] = v;
    return en;
}

template <typename T>
__device__ __forceinline__ T e_ade(const Args<T> &a, int e, int comp, int i, int j, int k, T v) {
    const T *r = a.ade_c + 16 * a.l_aix[e];
    T *st = a.ade_s + 5 * (long long)e;
    // curl with CPML where present: reuse the scalar update with (1, 1)
    // coefficients would change rounding, so form the stretched difference here
    const long long c = cidx(a, i, j, k);
    const int im = i == 0 ? a.nx - 1 : i - 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1;
    const int km = k == 0 ? a.nz - 1 : k - 1;
    T tA, tB;
    if (comp == 0) {
        tA = e_term(a, 0, 1, j, xs(a.Ho[2][c], a.Ho[2][cidx(a, i, jm, k)]), i, j, k);
        tB = e_term(a, 1, 2, k, xs(a.Ho[1][c], a.Ho[1][cidx(a, i, j, km)]), i, j, k);
    } else if (comp == 1) {
        tA = e_term(a, 2, 2, k, xs(a.Ho[0][c], a.Ho[0][cidx(a, i, j, km)]), i, j, k);
        tB = e_term(a, 3, 0, i, xs(a.Ho[2][c], a.Ho[2][cidx(a, im, j, k)]), i, j, k);
    } else {
        tA = e_term(a, 4, 0, i, xs(a.Ho[1][c], a.Ho[1][cidx(a, im, j, k)]), i, j, k);
        tB = e_term(a, 5, 1, j, xs(a.Ho[0][c], a.Ho[0][cidx(a, i, jm, k)]), i, j, k);
    }
    return ade_core(r, v, tA, tB, st);
}

// Full 3x3 sample of component c at (i, j, k), record r = (m_c0, m_c1, m_c2,
// s, ca): value = m_cc D_c, then for b = 0, 1, 2 (b != c) value += m_cb (0.25
// (((D_b(w) + D_b(w + e_c)) + D_b(w - e_b)) + D_b(w + e_c - e_b))); the
// result is ca E + s value (a lossless sample has ca = 1, s = dt/(eps0 dx)).  D_b(p) is the curl difference of E component b
// from the advanced H, (H_{b+2}(p) - H_{b+2}(p - e_{b+1})) - (H_{b+1}(p) -
// H_{b+1}(p - e_{b+2})), the unstretched terms of the E update
// (materials.c:920-1059).  Neighbours wrap on periodic axes only (the host
// admits samples in [1, n-1] on the other axes, so every index used is in
// the padded grid: a step back never leaves it, a step forward reaches at
// most the padded boundary sample n).
template <typename T>
__device__ __forceinline__ T e_tensor3(const Args<T> &a, const T *r, int c, int i, int j, int k, T v) {
    // linear indices by strides from the sample's own; a step back from
    // coordinate 0 wraps to n - 1 (reached only on periodic axes)
    const int n[3] = {a.nx, a.ny, a.nz};
    const long long st[3] = {(long long)(a.ny + 1) * a.pitch, a.pitch, 1};
    auto curl_at = [&](int b, long long q, const int p[3]) {
        const int fa = (b + 2) % 3, axa = (b + 1) % 3, fb = (b + 1) % 3, axb = (b + 2) % 3;
        const long long qa = p[axa] == 0 ? q + (long long)(n[axa] - 1) * st[axa] : q - st[axa];
        const long long qb = p[axb] == 0 ? q + (long long)(n[axb] - 1) * st[axb] : q - st[axb];
        return xs(xs(a.Ho[fa][q], a.Ho[fa][qa]), xs(a.Ho[fb][q], a.Ho[fb][qb]));
    };
    const int p0[3] = {i, j, k};
    const long long c0 = cidx(a, i, j, k);
    T value = xm(r[c], curl_at(c, c0, p0));
    const bool wrap = ((a.per >> c) & 1u) && p0[c] + 1 == n[c];
    int p1[3] = {i, j, k};
    p1[c] = wrap ? 0 : p1[c] + 1;
    const long long c1 = wrap ? c0 - (long long)(n[c] - 1) * st[c] : c0 + st[c];
    for (int b = 0; b < 3; b++) {
        if (b == c) continue;
        int p2[3] = {p0[0], p0[1], p0[2]};
        p2[b] = p2[b] == 0 ? n[b] - 1 : p2[b] - 1;
        int p3[3] = {p1[0], p1[1], p1[2]};
        p3[b] = p3[b] == 0 ? n[b] - 1 : p3[b] - 1;
        const long long back = p0[b] == 0 ? (long long)(n[b] - 1) * st[b] : -st[b];
        const T s4 = xa(xa(xa(curl_at(b, c0, p0), curl_at(b, c1, p1)), curl_at(b, c0 + back, p2)),
                        curl_at(b, c1 + back, p3));
        value = xa(value, xm(r[b], xm(T(0.25), s4)));
    }
    return xa(xm(r[4], v), xm(r[3], value));
}

// The three components of a cell whose samples are all 3x3 samples (no
// source, no TF/SF term): e_tensor3 for c = 0, 1, 2 with the same operation
// order, the curl differences they share computed once -- D_b at the cell
// and at the cell one step back along b serve both components c != b -- so
// a cell takes 18 curl evaluations instead of 27.
template <typename T>
__device__ __forceinline__ void t3_cell(const Args<T> &a, int cell) {
    const int i = a.lc_ijk[3 * cell], j = a.lc_ijk[3 * cell + 1], k = a.lc_ijk[3 * cell + 2];
    const int n[3] = {a.nx, a.ny, a.nz};
    const long long st[3] = {(long long)(a.ny + 1) * a.pitch, a.pitch, 1};
    auto curl_at = [&](int b, long long q, const int p[3]) {
        const int fa = (b + 2) % 3, axa = (b + 1) % 3, fb = (b + 1) % 3, axb = (b + 2) % 3;
        const long long qa = p[axa] == 0 ? q + (long long)(n[axa] - 1) * st[axa] : q - st[axa];
        const long long qb = p[axb] == 0 ? q + (long long)(n[axb] - 1) * st[axb] : q - st[axb];
        return xs(xs(a.Ho[fa][q], a.Ho[fa][qa]), xs(a.Ho[fb][q], a.Ho[fb][qb]));
    };
    const int p0[3] = {i, j, k};
    const long long c0 = cidx(a, i, j, k);
    T dw[3], dm[3];
    long long back[3];
    for (int b = 0; b < 3; b++) {
        dw[b] = curl_at(b, c0, p0);
        int p2[3] = {i, j, k};
        p2[b] = p2[b] == 0 ? n[b] - 1 : p2[b] - 1;
        back[b] = p0[b] == 0 ? (long long)(n[b] - 1) * st[b] : -st[b];
        dm[b] = curl_at(b, c0 + back[b], p2);
    }
    for (int c = 0; c < 3; c++) {
        const T *r = a.t3 + 5 * (long long)a.l_tix[3 * cell + c];
        T value = xm(r[c], dw[c]);
        const bool wrap = ((a.per >> c) & 1u) && p0[c] + 1 == n[c];
        int p1[3] = {i, j, k};
        p1[c] = wrap ? 0 : p1[c] + 1;
        const long long c1 = wrap ? c0 - (long long)(n[c] - 1) * st[c] : c0 + st[c];
        for (int b = 0; b < 3; b++) {
            if (b == c) continue;
            int p3[3] = {p1[0], p1[1], p1[2]};
            p3[b] = p3[b] == 0 ? n[b] - 1 : p3[b] - 1;
            const T s4 = xa(xa(xa(dw[b], curl_at(b, c1, p1)), dm[b]), curl_at(b, c1 + back[b], p3));
            value = xa(value, xm(r[b], xm(T(0.25), s4)));
        }
        a.Eo[c][c0] = xa(xm(r[4], a.E[c][c0]), xm(r[3], value));
    }
}

// Cells whose three samples are dispersive (ADE) samples outside every CPML
// slab, with no source and no TF/SF term: one thread per cell takes its
// three components -- the nine H values they read loaded once, the 15 state
// values of the cell's samples (contiguous) loaded together -- with the
// operations of e_ade per sample (ade_core), so the results are
// bit-identical to the per-entry form.
template <typename T>
__device__ __forceinline__ void ade_cell(const Args<T> &a, int cell) {
    const int i = a.lc_ijk[3 * cell], j = a.lc_ijk[3 * cell + 1], k = a.lc_ijk[3 * cell + 2];
    const long long c = cidx(a, i, j, k);
    const int im = i == 0 ? a.nx - 1 : i - 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1;
    const int km = k == 0 ? a.nz - 1 : k - 1;
    const long long ci = cidx(a, im, j, k), cj = cidx(a, i, jm, k), ck = cidx(a, i, j, km);
    const T hx = a.Ho[0][c], hy = a.Ho[1][c], hz = a.Ho[2][c];
    const T hx_j = a.Ho[0][cj], hx_k = a.Ho[0][ck], hy_k = a.Ho[1][ck], hy_i = a.Ho[1][ci], hz_j = a.Ho[2][cj],
            hz_i = a.Ho[2][ci];
    const T e0 = a.E[0][c], e1 = a.E[1][c], e2 = a.E[2][c];
    const T *r0 = a.ade_c + 16 * a.l_aix[3 * cell], *r1 = a.ade_c + 16 * a.l_aix[3 * cell + 1],
            *r2 = a.ade_c + 16 * a.l_aix[3 * cell + 2];
    T *st = a.ade_s + 15 * (long long)cell;
    T s[15];
#pragma unroll
    for (int q = 0; q < 15; q++) s[q] = st[q];
    const T n0 = ade_core(r0, e0, xs(hz, hz_j), xs(hy, hy_k), s);
    const T n1 = ade_core(r1, e1, xs(hx, hx_k), xs(hz, hz_i), s + 5);
    const T n2 = ade_core(r2, e2, xs(hy, hy_i), xs(hx, hx_j), s + 10);
#pragma unroll
    for (int q = 0; q < 15; q++) st[q] = s[q];
    a.Eo[0][c] = n0;
    a.Eo[1][c] = n1;
    a.Eo[2][c] = n2;
}

// ---- interface list: overrides, tensor edges, sources --------------------
// One thread per (cell, component) entry.  Reads E from the input buffers,
// H from the output buffers (already advanced), writes E output.
template <typename T>
__device__ __forceinline__ void e_list_entry(const Args<T> &a, int e) {
    const int cell = e / 3, comp = e - 3 * cell;
    const int i = a.lc_ijk[3 * cell], j = a.lc_ijk[3 * cell + 1], k = a.lc_ijk[3 * cell + 2];
    const long long c = cidx(a, i, j, k);
    const int kind = a.l_kind[e];
    if (kind == 5 || kind == 6) return;  // a 3x3 / ADE cell: k_list_cells updates it per cell
    T v = a.E[comp][c];
    const int s = a.l_src[e];
    if (s >= 0) {
        const int n = *a.d_step;
        const T sv = (n < a.n_steps) ? a.src_val[(long long)s * a.n_steps + n] : T(0);
        v = a.src_hard[s] ? sv : xa(v, sv);
    }
    if (kind == 1) {
        v = e_scalar(a, comp, i, j, k, v, a.l_ca[e], a.l_cb[e]);
    } else if (kind == 2) {
        // rfsyn materials.c:847-903: value = m11 dHz + sum_q w_q curl_q,
        // E += scale * value.
        const int t = a.l_tix[e];
        const int *mn = a.t_main + 4 * t;
        T value = xm(a.t_m11[t], xs(a.Ho[2][cidx(a, mn[0], mn[1], k)], a.Ho[2][cidx(a, mn[2], mn[3], k)]));
        const int nq = a.t_nq[t];
        const bool neg = a.t_sign[t] < 0;
        for (int q = 0; q < nq; q++) {
            const int *uv = a.t_uv + 16 * t + 4 * q;
            T d = xs(a.Ho[2][cidx(a, uv[0], uv[1], k)], a.Ho[2][cidx(a, uv[2], uv[3], k)]);
            if (neg) d = -d;
            value = xa(value, xm(a.t_w[4 * t + q], d));
        }
        v = xa(v, xm(a.t_scale[t], value));
    } else if (kind == 3) {
        // dispersive sample: polarisation-current ADE (Debye / Lorentz poles)
        v = e_ade(a, e, comp, i, j, k, v);
    } else if (kind == 4) {
        // full 3x3 anisotropic sample
        v = e_tensor3(a, a.t3 + 5 * (long long)a.l_tix[e], comp, i, j, k, v);
    }
    if (a.tf_first) {
        // a sample next to the total-field / scattered-field boundary
        const int f = a.tf_first[e];
        if (f >= 0)
            for (int t = f; t < f + a.tf_count[e]; t++) {
                const int m = a.tf_idx[t];
                v = xa(v, xm(a.tf_coef[t], tf_interp(a.tf_w + 4 * t, a.inc_h + m)));
            }
    }
    a.Eo[comp][c] = v;
}

// ---- plane wave through a TF/SF boundary -----------------------------------
template <typename T>
struct TfArgs {
    int n_h;
    const long long *h_cell;
    const int *h_comp, *h_first, *h_count, *h_idx;
    const T *h_coef, *h_w;  // 4 cubic weights per term
    T *Ho[3];              // H after the sweep of the step
    T *inc_e, *inc_h;      // the 1-D line
    int m_len;
    T ce, ch;
    const T *src;          // E1D[0] per step, n_steps + 1 values
    const int *d_step;
    long long n_steps;
};

// H samples next to the boundary: H += coef * interp(E1D around idx) for
// each of their terms, in order (E1D at step n).
template <typename T>
__global__ void k_tfsf_h(TfArgs<T> a) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n_h) return;
    T *f = a.Ho[a.h_comp[q]] + a.h_cell[q];
    T h = *f;
    for (int t = a.h_first[q]; t < a.h_first[q] + a.h_count[q]; t++) {
        const int m = a.h_idx[t];
        h = xa(h, xm(a.h_coef[t], tf_interp(a.h_w + 4 * t, a.inc_e + m)));
    }
    *f = h;
}

// The line's H: H1D[m] -= ch (E1D[m+1] - E1D[m]).
template <typename T>
__global__ void k_inc_h(TfArgs<T> a) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < a.m_len - 1; m += gridDim.x * blockDim.x)
        a.inc_h[m] = xs(a.inc_h[m], xm(a.ch, xs(a.inc_e[m + 1], a.inc_e[m])));
}

// The line's E: E1D[m] -= ce (H1D[m] - H1D[m-1]); E1D[0] is the hard source
// of the step just completed (the step counter already advanced).
template <typename T>
__global__ void k_inc_e(TfArgs<T> a) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < a.m_len - 1; m += gridDim.x * blockDim.x) {
        if (m == 0) {
            const long long n = *a.d_step;
            a.inc_e[0] = a.src[n < a.n_steps ? n : a.n_steps];
        } else {
            a.inc_e[m] = xs(a.inc_e[m], xm(a.ce, xs(a.inc_h[m], a.inc_h[m - 1])));
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_e_list(Args<T> a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (a.l_work) {
        if (t < a.n_work) e_list_entry(a, a.l_work[t]);
        return;
    }
    if (t >= 3 * a.n_cells) return;
    e_list_entry(a, t);
}

// The whole interface list of a step in one launch when some cells have
// per-cell updates: blocks [0, nb_t3) take the whole 3x3 cells (t3_cell),
// the next nb_ade blocks the dispersive cells (ade_cell), the rest the list
// entries left to the per-entry update (a.l_work).  The three parts touch
// disjoint samples and read only the step's advanced H and the previous E,
// so running them side by side changes no result, and their dependent
// gathers overlap instead of ending one launch before the next begins.
// The kernel is bound by the latency of those gathers, so in FP32 it is
// held to 40 registers (6 blocks of 256 per SM, against 4 at its natural
// 60; 32 bytes of spills): C3's step 0.2233 -> 0.2181 ms, C2's ~1 % faster.
// FP64 keeps the 3 blocks per SM of its natural 78-80 registers.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 3) k_list_cells(Args<T> a, const int *t3, int n_t3, int nb_t3, const int *ade,
                                                    int n_ade, int nb_ade) {
    const int b = blockIdx.x;
    if (b < nb_t3) {
        const int t = b * blockDim.x + threadIdx.x;
        if (t < n_t3) t3_cell(a, t3[t]);
    } else if (b < nb_t3 + nb_ade) {
        const int t = (b - nb_t3) * blockDim.x + threadIdx.x;
        if (t < n_ade) ade_cell(a, ade[t]);
    } else {
        const int t = (b - nb_t3 - nb_ade) * blockDim.x + threadIdx.x;
        if (t < a.n_work) e_list_entry(a, a.l_work[t]);
    }
}

// ---- probes ---------------------------------------------------------------
template <typename T>
struct ProbeArgs {
    int n;
    const long long *cell;
    const int *comp;
    const T *F[6];
    T *ts;
    long long n_steps;
    int *d_step;
};

// Records sample n of every probe after the step, then advances the device
// step counter (single block).
template <typename T>
__global__ void k_probe_gather(ProbeArgs<T> p) {
    __shared__ int n;
    if (threadIdx.x == 0) n = *p.d_step;
    __syncthreads();
    if (n < p.n_steps)
        for (int q = threadIdx.x; q < p.n; q += blockDim.x)
            p.ts[(long long)q * p.n_steps + n] = p.F[p.comp[q]][p.cell[q]];
    __syncthreads();
    if (threadIdx.x == 0) *p.d_step = n + 1;
}

// ---- plane probes ------------------------------------------------------------
// Sample n of a plane probe is the mean of one field component over a whole
// grid plane (axis a at index q: every (u, v) of the other two axes, u < n_u,
// v < n_v): for a periodic cell at normal incidence, the amplitude of the
// specular (zeroth-order) reflected or transmitted wave.  The plane's points
// t = u n_v + v are cut into chunks of kPlaneChunk, one block each (grid:
// chunks x planes), so the gather spreads over the SMs.  Each thread sums
// its points of the chunk (t0 + x, t0 + x + kPlaneThreads, ...) in FP64,
// warp shuffles and one pass over the warps' sums reduce the block in a
// fixed tree, and the last block of the plane to finish (a per-plane
// counter, reset by that block) adds the chunks' sums in chunk order: the
// mean is deterministic.  Runs before k_probe_gather (same step index).
struct PlaneDesc {
    long long base, su, sv;  // element offset of (u, v) = (0, 0) and the strides
    int nu, nv, comp;
};

constexpr int kPlaneChunk = 1024, kPlaneThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kPlaneThreads) k_plane_gather(const PlaneDesc *planes, int n_planes,
                                                                const T *const *F, T *ts, int series0,
                                                                long long n_steps, const int *d_step, double *part,
                                                                int *count, int max_chunks) {
    __shared__ double warp_sum[kPlaneThreads / 32];
    const int q = blockIdx.y, b = blockIdx.x;
    if (q >= n_planes) return;
    const int n = *d_step;
    if (n >= n_steps) return;
    const PlaneDesc pd = planes[q];
    const long long npts = (long long)pd.nu * pd.nv;
    const int nchunk = (int)((npts + kPlaneChunk - 1) / kPlaneChunk);
    if (b >= nchunk) return;
    const T *f = F[pd.comp];
    const long long t0 = (long long)b * kPlaneChunk, t1 = t0 + kPlaneChunk < npts ? t0 + kPlaneChunk : npts;
    double acc = 0.0;
    for (long long t = t0 + threadIdx.x; t < t1; t += kPlaneThreads) {
        const long long u = t / pd.nv, v = t - u * pd.nv;
        acc = __dadd_rn(acc, (double)f[pd.base + u * pd.su + v * pd.sv]);
    }
    for (int off = 16; off > 0; off >>= 1) acc = __dadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, off));
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kPlaneThreads / 32; w++) s = __dadd_rn(s, warp_sum[w]);
        part[(long long)q * max_chunks + b] = s;
        __threadfence();
        if (atomicAdd(&count[q], 1) == nchunk - 1) {
            // every chunk's sum is visible: the other blocks fenced before
            // their increments
            __threadfence();
            const volatile double *pp = part + (long long)q * max_chunks;
            double m = 0.0;
            for (int c = 0; c < nchunk; c++) m = __dadd_rn(m, pp[c]);
            ts[(long long)(series0 + q) * n_steps + n] = (T)__ddiv_rn(m, (double)npts);
            count[q] = 0;
        }
    }
}

// ---- running DFT --------------------------------------------------------------
// Accumulates the DFT bins of every series (point probes, then plane probes)
// over the `count` samples the step loop recorded last, [step - count, step),
// into acc: rfsyn's running sums re += v cos(w t) dt, im -= v sin(w t) dt
// with t = (n + t_off) dt (engine/fdtd/probe.c:78-92).  Thread per (series,
// bin); launched once per replayed chunk of steps, so the sums advance with
// the run instead of in a pass over the stored series afterwards.  FP64 runs:
// FP64 sums with direct sincos (the order and arithmetic of rfsyn's loop).
// FP32 runs: Kahan-compensated FP32 sums (acc holds re, im and their
// compensations), the phasor advanced by an FP64 recurrence anchored with a
// direct sincos at the first sample of each launch.
template <typename T>
__global__ void k_dft_run(const T *ts, int n_series, long long n_steps, const int *d_step, int count, int n_freqs,
                          const double *omega, double dt, double t_off, void *acc) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (f >= n_freqs || p >= n_series) return;
    const int n1 = min((long long)*d_step, n_steps), n0 = max(n1 - count, 0);
    const T *s = ts + (long long)p * n_steps;
    const double w = omega[f];
    const long long a = (long long)p * n_freqs + f;
    if (sizeof(T) == 8) {
        double *r = static_cast<double *>(acc) + 2 * a;
        double re = r[0], im = r[1];
        for (int n = n0; n < n1; n++) {
            double t = ((double)n + t_off) * dt;
            double sn, cn;
            sincos(w * t, &sn, &cn);
            double v = (double)s[n];
            re = __dadd_rn(re, __dmul_rn(__dmul_rn(v, cn), dt));
            im = __dsub_rn(im, __dmul_rn(__dmul_rn(v, sn), dt));
        }
        r[0] = re;
        r[1] = im;
    } else {
        float4 *r = static_cast<float4 *>(acc) + a;
        float4 st = *r;  // re, im, Kahan compensations of re and im
        if (n1 > n0) {
            double cw, sw, cn, sn;
            sincos(w * dt, &sw, &cw);
            sincos(w * (((double)n0 + t_off) * dt), &sn, &cn);
            const float fdt = (float)dt;
            for (int n = n0; n < n1; n++) {
                const float v = (float)s[n] * fdt;
                const float yr = v * (float)cn - st.z;
                const float tr = st.x + yr;
                st.z = (tr - st.x) - yr;
                st.x = tr;
                const float yi = -v * (float)sn - st.w;
                const float ti = st.y + yi;
                st.w = (ti - st.y) - yi;
                st.y = ti;
                const double c2 = cn * cw - sn * sw;
                sn = sn * cw + cn * sw;
                cn = c2;
            }
        }
        *r = st;
    }
}

// ---- running DFT of the probe series -------------------------------------
// Thread per (probe, bin).  FP64 runs: acc += v cos(w t) dt in FP64 with
// direct sincos (rfsyn probe.c:78-92).  FP32 runs: Kahan-compensated FP32
// accumulation, phasor advanced by an FP64 recurrence re-anchored every 64
// samples.
template <typename T>
__global__ void k_probe_dft(const T *ts, long long n_steps, int n_probes, int steps_done, int n_freqs,
                            const double *omega, double dt, double t_off, double *out_re, double *out_im) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (f >= n_freqs || p >= n_probes) return;
    const T *s = ts + (long long)p * n_steps;
    const double w = omega[f];
    if (sizeof(T) == 8) {
        double re = 0.0, im = 0.0;
        for (int n = 0; n < steps_done; n++) {
            double t = ((double)n + t_off) * dt;
            double sn, cn;
            sincos(w * t, &sn, &cn);
            double v = (double)s[n];
            re = __dadd_rn(re, __dmul_rn(__dmul_rn(v, cn), dt));
            im = __dsub_rn(im, __dmul_rn(__dmul_rn(v, sn), dt));
        }
        out_re[(long long)p * n_freqs + f] = re;
        out_im[(long long)p * n_freqs + f] = im;
    } else {
        float re = 0.f, im = 0.f, cre = 0.f, cim = 0.f;  // Kahan compensation
        double cw, sw;
        sincos(w * dt, &sw, &cw);
        double cn = 1.0, sn = 0.0;
        const float fdt = (float)dt;
        for (int n = 0; n < steps_done; n++) {
            if ((n & 63) == 0) sincos(w * (((double)n + t_off) * dt), &sn, &cn);
            const float v = (float)s[n] * fdt;
            float yr = v * (float)cn - cre;
            float tr = re + yr;
            cre = (tr - re) - yr;
            re = tr;
            float yi = -v * (float)sn - cim;
            float ti = im + yi;
            cim = (ti - im) - yi;
            im = ti;
            const double c2 = cn * cw - sn * sw;
            sn = sn * cw + cn * sw;
            cn = c2;
        }
        out_re[(long long)p * n_freqs + f] = (double)re;
        out_im[(long long)p * n_freqs + f] = (double)im;
    }
}

// Marks list cells in a code volume (code-less scenes with many list cells).
__global__ void k_mark_list(uint8_t *codes, const int *ijk, int n, int ny, long long pitch) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    codes[((long long)ijk[3 * q] * (ny + 1) + ijk[3 * q + 1]) * pitch + ijk[3 * q + 2]] = LIST_CODE;
}

}  // namespace rfb
