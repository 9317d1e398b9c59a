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
