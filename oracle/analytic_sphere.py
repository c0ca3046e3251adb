"""Closed-form TMS E-field inside a spherically symmetric conductor. TEST INFRASTRUCTURE ONLY.

For magnetic dipoles outside a sphere centred at the origin, the induced field inside does not
depend on the radial conductivity profile (Heller & van Hulsteyn 1992, J. Appl. Phys. 71:4;
Eaton 1992, Med. Biol. Eng. Comput. 30:433). By reciprocity with Sarvas's field of a current
dipole in a sphere (Phys. Med. Biol. 32:11, 1987), with a = r0 - r (dipole at r0, field point r),

    F      = |a| (|r0| |a| + |r0|^2 - r0 . r)
    grad F = (|a|^2 / |r0| + a . r0 / |a| + 2 |a| + 2 |r0|) r0 - (|a| + 2 |r0| + a . r0 / |a|) r
    E(r)   = -mu0/(4 pi) dI/dt / F^2 * (F (r x m) - (m . grad F) (r x r0))

summed over the dipoles (grad F is the gradient of F with respect to r0). The field is everywhere tangential (r . E = 0), divergence-free, and
differs from the primary field -dA/dt by a gradient; tests/test_analytic_sphere.py checks those
three properties before using it as a sanity bound on the finite-element solution.
"""

from __future__ import annotations

import numpy as np

MU0_OVER_4PI = 1e-7


def sphere_efield(points_m, dip_pos_m, dip_moment, didt: float = 1e6) -> np.ndarray:
    """E (V/m) at points (N, 3) in metres, for dipoles at dip_pos_m (M, 3) with moments (M, 3)."""
    r = np.asarray(points_m, np.float64).reshape(-1, 3)
    out = np.zeros_like(r)
    for r0, m in zip(np.asarray(dip_pos_m, np.float64).reshape(-1, 3), np.asarray(dip_moment, np.float64).reshape(-1, 3)):
        a = r0 - r
        an = np.linalg.norm(a, axis=1)
        r0n = float(np.linalg.norm(r0))
        ar0 = a @ r0
        F = an * (r0n * an + r0n * r0n - r @ r0)
        c_0 = an * an / r0n + ar0 / an + 2.0 * an + 2.0 * r0n
        c_r = an + 2.0 * r0n + ar0 / an
        m_grad = c_0 * (r0 @ m) - c_r * (r @ m)
        term = F[:, None] * np.cross(r, m) - m_grad[:, None] * np.cross(r, r0)
        out += -MU0_OVER_4PI * didt * term / (F * F)[:, None]
    return out


def primary_efield(points_m, dip_pos_m, dip_moment, didt: float = 1e6) -> np.ndarray:
    """-dA/dt of the dipoles alone: -mu0/(4 pi) dI/dt sum m x (r - r0) / |r - r0|^3."""
    r = np.asarray(points_m, np.float64).reshape(-1, 3)
    out = np.zeros_like(r)
    for r0, m in zip(np.asarray(dip_pos_m, np.float64).reshape(-1, 3), np.asarray(dip_moment, np.float64).reshape(-1, 3)):
        d = r - r0
        dn = np.linalg.norm(d, axis=1)
        out += -MU0_OVER_4PI * didt * np.cross(m, d) / (dn ** 3)[:, None]
    return out


def head_frame_dipoles(coil, transform):
    """A coil's dipoles (metres, coil frame) placed by a (4, 4) coil-to-head transform in mm."""
    T = np.asarray(transform, np.float64).reshape(4, 4)
    pos = (np.asarray(coil.positions_m) * 1e3) @ T[:3, :3].T + T[:3, 3]
    mom = np.asarray(coil.moments) @ T[:3, :3].T
    return pos * 1e-3, mom
