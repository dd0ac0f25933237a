"""Synthetic problem builders for the unit-cube workloads.

All randomness is numpy's PCG64 (``numpy.random.default_rng``) with the
fixed seeds below, so every machine builds bit-identical inputs:

* mesh: the reference's structured unit cube, 6 tets per hex
  (generate_unit_cube_mesh, FEM/adaptive_fem_engine.hpp:2219), optionally with
  the interior nodes (0 < i,j,k < N) jittered by U(-a h, a h) per coordinate;
* material: uniform E, nu, or a per-element log-normal shear modulus
  mu_e = mu_0 exp(sigma z_e) with lambda/mu fixed by nu (given to the
  library as E_e = 2 mu_e (1 + nu));
* Dirichlet data: bottom face z = 0 clamped (all DOFs), top face z = 1 with
  u_z prescribed, applied in equal load fractions s / n_steps.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ._lib import unit_cube

SEED_JITTER = 0x4A2
SEED_MAT = 0x3D2
SEED_MAT_3 = 0x3D3
SEED_PHASE_3 = 0x9F3
SEED_TRUE_4 = 0xA4
SEED_MODEL_4 = 0xB4
SEED_FD_4 = 0x5F4
SEED_JITTER_5 = 0x4A5
SEED_TRUE_5 = 0xA5


@dataclass
class Problem:
    name: str
    N: int
    xyz: np.ndarray
    conn: np.ndarray
    nu: float
    E: float = 1.0
    E_elem: np.ndarray | None = None   # per-element Young's modulus (None: uniform E)
    mask: np.ndarray = field(default=None)
    bc_value: np.ndarray = field(default=None)
    # the mesh generator's stored TetraElement::volume (computed before any
    # jitter, as generate_unit_cube_mesh stores it); the assembly skips
    # elements whose stored volume is < 1e-30, i.e. the slivers of the split
    elem_volume: np.ndarray | None = None
    n_steps: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self):
        return self.xyz.size // 3

    @property
    def n_elems(self):
        return self.conn.size // 4

    def lame(self):
        """per-element (mu, lambda) as the reference derives them from (E, nu)"""
        E = self.E_elem if self.E_elem is not None else np.full(self.n_elems, self.E)
        nu = self.nu
        mu = E / (2.0 * (1.0 + nu))
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        return mu, lam


def tet_volumes(xyz, conn):
    """|triple product| / 6 per tet (tet_volume, FEM/mesh_adaptation.hpp:111-126)"""
    X = xyz.reshape(-1, 3)
    c = conn.reshape(-1, 4)
    a, b, cc, d = X[c[:, 0]], X[c[:, 1]], X[c[:, 2]], X[c[:, 3]]
    u, v, w = b - a, cc - a, d - a
    s6 = (u[:, 0] * (v[:, 1] * w[:, 2] - v[:, 2] * w[:, 1])
          - u[:, 1] * (v[:, 0] * w[:, 2] - v[:, 2] * w[:, 0])
          + u[:, 2] * (v[:, 0] * w[:, 1] - v[:, 1] * w[:, 0]))
    return np.abs(s6) / 6.0


def jitter_interior(xyz, N, amp, seed):
    """Move nodes with 0 < i,j,k < N by U(-amp h, amp h) per coordinate."""
    s = N + 1
    idx = np.arange(xyz.size // 3)
    i, j, k = idx % s, (idx // s) % s, idx // (s * s)
    interior = (i > 0) & (i < N) & (j > 0) & (j < N) & (k > 0) & (k < N)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-amp / N, amp / N, size=(interior.sum(), 3))
    out = xyz.reshape(-1, 3).copy()
    out[interior] += d
    return out.reshape(-1)


def lognormal_E(n_elems, sigma, seed, nu, E0=1.0):
    """E_e with mu_e = mu_0 exp(sigma z), z ~ N(0,1); lambda/mu fixed by nu."""
    mu0 = E0 / (2.0 * (1.0 + nu))
    z = np.random.default_rng(seed).standard_normal(n_elems)
    mu = mu0 * np.exp(sigma * z)
    return 2.0 * mu * (1.0 + nu)


def clamp_top_bc(xyz, uz_total):
    """bottom z=0 clamped; top z=1 u_z = uz_total at full load"""
    z = xyz[2::3]
    mask = np.zeros(xyz.size, np.uint8)
    val = np.zeros(xyz.size, np.float64)
    bottom = z < 1e-12
    top = z > 1.0 - 1e-12
    mask[np.repeat(bottom, 3)] = 1
    mask[2::3][top] = 1
    val[2::3][top] = uz_total
    return mask, val


def top_face_xy_dofs(xyz):
    """DOF indices of u_x, u_y on the top face (the loss's support)"""
    top = np.nonzero(xyz[2::3] > 1.0 - 1e-12)[0]
    return np.sort(np.concatenate([3 * top, 3 * top + 1]))


def unit_cube_problem(name, N, *, jitter=0.0, seed_jitter=SEED_JITTER, sigma_log=0.0,
                      seed_mat=SEED_MAT, nu=0.3, E=1.0, uz_total=-0.1, n_steps=5, mesher=None):
    """mesher(N) -> (xyz, conn): the unit-cube generator to use (default: the
    library's fm_unit_cube; a CPU caller that must not load the library
    passes another generator of the same mesh)"""
    xyz, conn = (mesher or unit_cube)(N)
    vol = tet_volumes(xyz, conn)
    if jitter:
        xyz = jitter_interior(xyz, N, jitter, seed_jitter)
    E_elem = lognormal_E(conn.size // 4, sigma_log, seed_mat, nu, E) if sigma_log else None
    mask, val = clamp_top_bc(xyz, uz_total)
    return Problem(name=name, N=N, xyz=xyz, conn=conn, nu=nu, E=E, E_elem=E_elem, mask=mask,
                   bc_value=val, n_steps=n_steps, elem_volume=vol,
                   meta={"jitter": jitter, "sigma_log": sigma_log, "uz_total": uz_total})


# ---- the five unit-cube workloads ------------------------------------------------
def small_block(N=8):
    """8^3 hexes x 6 tets, E=1, nu=0.3, top u_z=-0.1 in 5 steps (FP64 parity case)"""
    return unit_cube_problem("small", N, uz_total=-0.1, n_steps=5)


def scaleup_block(N=64, n_steps=10, mesher=None):
    """64^3 x 6 tets, interior jitter 0.15 h, log-normal mu (sigma 0.3), u_z=-0.2 in 10 steps"""
    return unit_cube_problem("scaleup", N, jitter=0.15, sigma_log=0.3, uz_total=-0.2,
                             n_steps=n_steps, mesher=mesher)


def assembly_block(N=128):
    """128^3 x 6 tets, log-normal mu, and the sinusoidal displacement field
    u_c = 0.05 sin(2 pi x + p1c) sin(2 pi y + p2c) sin(2 pi z + p3c), nine phases
    U[0, 2pi) (one triple per component)."""
    P = unit_cube_problem("assembly", N, sigma_log=0.3, seed_mat=SEED_MAT_3)
    ph = np.random.default_rng(SEED_PHASE_3).uniform(0.0, 2.0 * np.pi, size=(3, 3))
    x, y, z = P.xyz[0::3], P.xyz[1::3], P.xyz[2::3]
    u = np.zeros_like(P.xyz)
    for c in range(3):
        u[c::3] = 0.05 * (np.sin(2 * np.pi * x + ph[c, 0]) * np.sin(2 * np.pi * y + ph[c, 1]) *
                          np.sin(2 * np.pi * z + ph[c, 2]))
    P.meta["u"] = u
    P.meta["phases"] = ph
    return P


def adjoint_block(N=32):
    """32^3 x 6 tets, true/model log-normal mu (seeds A/B), u_z=-0.1 in 5 steps"""
    P = unit_cube_problem("adjoint", N, sigma_log=0.3, seed_mat=SEED_MODEL_4, uz_total=-0.1,
                          n_steps=5)
    P.meta["E_true"] = lognormal_E(P.n_elems, 0.3, SEED_TRUE_4, P.nu)
    return P


def near_incompressible_block(N=48):
    """48^3 x 6 tets, jitter 0.1 h, nu=0.49, E=1, u_z=-0.4 in 20 steps"""
    P = unit_cube_problem("near_incompressible", N, jitter=0.1, seed_jitter=SEED_JITTER_5,
                          nu=0.49, uz_total=-0.4, n_steps=20)
    P.meta["E_true"] = lognormal_E(P.n_elems, 0.2, SEED_TRUE_5, P.nu)
    return P
