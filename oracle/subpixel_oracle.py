"""TEST INFRASTRUCTURE (oracle).  numpy FP64 restatement of the smoothed
inverse permittivity of a cut cell in three dimensions.

Kottke, Farjadpour and Johnson, Phys. Rev. E 77, 036611 (2008), eqs. 23-24:
in an orthonormal frame (n, p, q) whose first vector is the interface normal,
the transform

    tau(e) = [[-1/e_nn,      e_np/e_nn,                 e_nq/e_nn               ],
              [ e_pn/e_nn,   e_pp - e_pn e_np / e_nn,   e_pq - e_pn e_nq / e_nn ],
              [ e_qn/e_nn,   e_qp - e_qn e_np / e_nn,   e_qq - e_qn e_nq / e_nn ]]

is averaged over the cell, <tau> = (1 - f) tau(eps_bg) + f tau(eps_in), and
inverted (tau is an involution up to the sign conventions: applying the
same formulas to <tau> with e_nn = -1/<tau>_nn gives eps).  The frame here
comes from a QR factorisation (any orthonormal completion of n gives the same
eps), so the restatement shares no arithmetic with the product's own frame.
For isotropic media it reduces to rfsyn's rule (engine/fdtd/subpixel_te.c:
106-132): eps^-1 = <1/eps> n n^T + (1/<eps>) (I - n n^T).
"""
from __future__ import annotations

import numpy as np


def _frame(n: np.ndarray) -> np.ndarray:
    """3x3 orthonormal matrix whose first column is n (unit)."""
    q, _ = np.linalg.qr(np.column_stack([n, np.eye(3)]))  # 3 x 4, rank 3: Q's first column is +-n
    if np.dot(q[:, 0], n) < 0:
        q = -q
    return q


def _tau(e: np.ndarray) -> np.ndarray:
    t = np.empty((3, 3))
    t[0, 0] = -1.0 / e[0, 0]
    t[0, 1:] = e[0, 1:] / e[0, 0]
    t[1:, 0] = e[1:, 0] / e[0, 0]
    t[1:, 1:] = e[1:, 1:] - np.outer(e[1:, 0], e[0, 1:]) / e[0, 0]
    return t


def _tau_inverse(t: np.ndarray) -> np.ndarray:
    e = np.empty((3, 3))
    e[0, 0] = -1.0 / t[0, 0]
    e[0, 1:] = -t[0, 1:] / t[0, 0]
    e[1:, 0] = -t[1:, 0] / t[0, 0]
    e[1:, 1:] = t[1:, 1:] - np.outer(t[1:, 0], t[0, 1:]) / t[0, 0]
    return e


def smoothed_minv(f: float, eps_bg, eps_in, normal) -> np.ndarray:
    """eps^-1 (3x3) of a cell with fraction f of eps_in behind an interface of
    normal `normal`, the rest eps_bg; eps given as scalars or 3x3."""
    eb = np.asarray(eps_bg, dtype=float) * (np.eye(3) if np.ndim(eps_bg) == 0 else 1.0)
    ei = np.asarray(eps_in, dtype=float) * (np.eye(3) if np.ndim(eps_in) == 0 else 1.0)
    n = np.asarray(normal, dtype=float)
    n = n / np.linalg.norm(n)
    if f == 0.0:
        return np.linalg.inv(eb)
    if f == 1.0:
        return np.linalg.inv(ei)
    r = _frame(n)
    tau = (1.0 - f) * _tau(r.T @ eb @ r) + f * _tau(r.T @ ei @ r)
    e = r @ _tau_inverse(tau) @ r.T
    return np.linalg.inv(0.5 * (e + e.T))


def isotropic_minv(f: float, eps_bg: float, eps_in: float, normal) -> np.ndarray:
    """rfsyn's isotropic rule in three dimensions (closed form)."""
    n = np.asarray(normal, dtype=float)
    n = n / np.linalg.norm(n)
    lam_n = (1.0 - f) / eps_bg + f / eps_in
    lam_t = 1.0 / ((1.0 - f) * eps_bg + f * eps_in)
    return lam_n * np.outer(n, n) + lam_t * (np.eye(3) - np.outer(n, n))


def _lattice() -> np.ndarray:
    return (np.arange(8) + 0.5) / 8.0 - 0.5


def slab_rows(nx: int, ny: int, nz: int, periodic: int, point, normal, thickness: float, eps_r,
              eps_bg: float = 1.0, sigma_bg: float = 0.0) -> list:
    """3x3 samples of a slab |(x - point) . u| <= thickness / 2 of eps_r
    (3x3) with smoothed faces, in a uniform isotropic background, as rows
    (comp, i, j, k, (m0, m1, m2), sigma): samples whose unit cube lies inside
    take the row of eps_r^-1; samples whose cube a face may cut take, when
    their fill fraction f (8^3 lattice) is positive, the row of the smoothed
    inverse permittivity along u with sigma (1 - f) sigma_bg.  Samples lie
    in [1, n-1] on every axis without wrap (the 3x3 update's margin)."""
    n = np.array([nx, ny, nz])
    o = np.asarray(point, dtype=float)
    nv = np.asarray(normal, dtype=float)
    nn = np.sqrt((nv[0] * nv[0] + nv[1] * nv[1]) + nv[2] * nv[2])
    u = nv / nn
    half = 0.5 * thickness
    reach = 0.5 * ((abs(u[0]) + abs(u[1])) + abs(u[2]))
    minv_in = np.linalg.inv(np.asarray(eps_r, dtype=float).reshape(3, 3))
    lat = _lattice()
    rows = []
    lo = [0 if (periodic >> a) & 1 else 1 for a in range(3)]
    I, J, K = np.meshgrid(*[np.arange(lo[a], n[a]) for a in range(3)], indexing="ij")
    for c in range(3):
        p = [I.astype(float), J.astype(float), K.astype(float)]
        p[c] = p[c] + 0.5
        d = (u[0] * (p[0] - o[0]) + u[1] * (p[1] - o[1])) + u[2] * (p[2] - o[2])
        ad = np.abs(d)
        inside = ad + reach <= half
        cut = ~inside & ~(ad - reach > half)
        for (i, j, k) in zip(I[inside], J[inside], K[inside]):
            rows.append((c, int(i), int(j), int(k), tuple(minv_in[c]), 0.0))
        dc = d[cut]
        ox = u[0] * lat
        oy = ox[:, None] + u[1] * lat[None, :]
        off = oy[:, :, None] + u[2] * lat[None, None, :]
        q = dc[:, None] + off.reshape(1, -1)
        f = np.count_nonzero(np.abs(q) <= half, axis=1) / 512.0
        for (i, j, k, fr) in zip(I[cut], J[cut], K[cut], f):
            if fr > 0.0:
                m = smoothed_minv(float(fr), eps_bg, eps_r if np.ndim(eps_r) == 2 else
                                  np.asarray(eps_r, dtype=float).reshape(3, 3), u)
                rows.append((c, int(i), int(j), int(k), tuple(m[c]), (1.0 - fr) * sigma_bg))
    return rows
