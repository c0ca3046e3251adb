"""FP64 NumPy restatement of the reference's conductivity-draw initial guess. TEST INFRASTRUCTURE
ONLY: the checker of the study's per-placement coefficient map (cunibs_sigma_coefficients).

The reference (uq/conductivity/run.py) starts every draw of a conductivity Monte Carlo at

    x0 = x_nom + W E^-1 W^T r0,   r0 = b(sigma) - A(sigma) x_nom,   E = W^T A_nom W,

W an orthonormal basis of the dominant column space of the sensitivities (run.py:104-123: a
reduced QR, then the SVD of R, keeping singular values above rtol times the largest) and r0, by
linearity in sigma, the sum over the perturbed tissues of (sigma_t - sigma_nom_t) c_t with
c_t = b_t - A_t x_nom (run.py:157-200).
"""

from __future__ import annotations

import numpy as np


def dominant_left_basis(a: np.ndarray, rtol: float = 1e-8) -> np.ndarray:
    """Orthonormal basis of the dominant column space of a tall a (run.py:104-123)."""
    q, r = np.linalg.qr(a, mode="reduced")
    u, s, _ = np.linalg.svd(r, full_matrices=False)
    keep = int((s > rtol * s[0]).sum()) if s.size and s[0] > 0 else 0
    return q @ u[:, :keep]


def galerkin_correction(a_nom: np.ndarray, sens: np.ndarray, r0: np.ndarray, rtol: float = 1e-8) -> np.ndarray:
    """x0 - x_nom = W E^-1 W^T r0 (run.py:139-200)."""
    w = dominant_left_basis(sens, rtol)
    if w.shape[1] == 0:
        return np.zeros(a_nom.shape[0])
    e = w.T @ (a_nom @ w)
    return w @ np.linalg.solve(e, w.T @ r0)
