"""Independent numpy restatement of the fTWA / HF trajectory engine (small N only).

TEST INFRASTRUCTURE ONLY.  Written separately from oracle/fps_oracle.c (numpy
matrix products instead of explicit loops) so the two oracles cross-check each
other.  Follows:
  FHfTWASolver::derivative   src/FHfTWASolver.cpp:568-600
  FHHFSolver::derivative     src/FHHFSolver.cpp:575-608
  step_RK4_38                src/FHfTWASolver.cpp:629-661 (k3 time uses dt, :653)
  runSimulation time loops   src/FHfTWASolver.cpp:366-426, src/FHHFSolver.cpp:306-401
  normalisation              src/FHfTWASolver.cpp:489-551
Also restates the Hamiltonian builders used for the configurations:
  FHLattice grid generator   src/FHLattice.cpp:872-895 (x fastest)
  minimum-image distance     src/FHLattice.cpp:516-539
  FHTunnelingInteraction::addTunneling  src/FHTunnelingInteraction.cpp:293-312
  FHCoulombInteraction::addCoulombinU/V src/FHCoulombInteraction.cpp:246-288
"""
from __future__ import annotations

import numpy as np

METHOD_FTWA, METHOD_HF = 0, 1
COUL_NULL, COUL_ONSITE, COUL_DISTANCE = 0, 1, 2


# ---------------------------------------------------------------- builders
def grid_positions(nx: int, ny: int, nz: int = 1, a: float = 1.0) -> np.ndarray:
    pts = [(a * x, a * y, a * z) for z in range(nz) for y in range(ny) for x in range(nx)]
    return np.array(pts, dtype=np.float64)


def distance_matrix(pos: np.ndarray, periodic: bool = False, latmat: np.ndarray | None = None) -> np.ndarray:
    d = pos[:, None, :] - pos[None, :, :]
    D = np.sqrt((d ** 2).sum(-1))
    if periodic:
        L = np.asarray(latmat, dtype=np.float64)
        for zs in (-1, 0, 1):
            for ys in (-1, 0, 1):
                for xs in (-1, 0, 1):
                    shift = xs * L[:, 0] + ys * L[:, 1] + zs * L[:, 2]
                    D = np.minimum(D, np.sqrt(((d + shift) ** 2).sum(-1)))
    return D


def tunneling(D: np.ndarray, shells, same_point: float = 1e-4) -> np.ndarray:
    """shells: list of (distance, energy); adds energy to i<j pairs (and mirror)."""
    n = D.shape[0]
    T = np.zeros((n, n))
    iu = np.triu_indices(n, 1)
    for dist, E in shells:
        m = (D[iu] - dist) ** 2 < same_point
        T[iu[0][m], iu[1][m]] += E
        T[iu[1][m], iu[0][m]] += E
    return T


def coulomb_onsite(D: np.ndarray, U0: float, same_point: float = 1e-4):
    U = np.where(D ** 2 < same_point, U0, 0.0)
    V = np.where((D ** 2 < same_point) & ~np.eye(D.shape[0], dtype=bool), U0, 0.0)
    return U, V


# ---------------------------------------------------------------- dynamics
def delta(tM, U, V, ext, coul, ext_null, method, same, other, pulse_diag=None):
    shift = 0.5 if method == METHOD_FTWA else 0.0
    D = np.array(tM, dtype=np.complex128)
    if coul != COUL_NULL:
        D = D + np.diag(U @ (np.real(np.diag(other)) + shift))
        if coul == COUL_DISTANCE:
            if method == METHOD_FTWA:
                D = D + np.diag(V @ (np.real(np.diag(same)) + shift))
            else:
                D = D + np.diag(V @ np.real(np.diag(same))) - same * V
    if not ext_null and ext is not None:
        D = D + ext
    if pulse_diag is not None:
        D = D + np.diag(pulse_diag)
    return D


def run(tM, U, V, ext, coul, ext_null, method, dt, S, Tp, rho0, pulse=None):
    """rho0: [B,2,n,n]. Returns dict of normalised observables and final states."""
    tM = np.asarray(tM, dtype=np.float64)
    n = tM.shape[0]
    U = np.asarray(U, dtype=np.float64)
    V = np.zeros((n, n)) if V is None else np.asarray(V, dtype=np.float64)
    rho0 = np.array(rho0, dtype=np.complex128)
    B = rho0.shape[0]
    h = dt / S

    def pdiag(t):
        if not pulse:
            return None
        nb = pulse["n_bins"]
        b = int(np.clip(np.floor(t / pulse["bin_width"]), 0, nb - 1))
        x = (t - pulse["t0"]) / pulse["td"]
        return pulse["amp"][b] * np.exp(-0.5 * x * x) * np.asarray(pulse["proj"])

    def f(t, ru, rd):
        Du = delta(tM, U, V, ext, coul, ext_null, method, ru, rd, pdiag(t))
        Dd = delta(tM, U, V, ext, coul, ext_null, method, rd, ru, pdiag(t))
        return -1j * (ru @ Du - Du @ ru), -1j * (rd @ Dd - Dd @ rd)

    def step(t, ru, rd):
        k1u, k1d = f(t, ru, rd)
        k2u, k2d = f(t + h / 3, ru + k1u * h / 3, rd + k1d * h / 3)
        k3u, k3d = f(t + 2 * dt / 3, ru + (-k1u / 3 + k2u) * h, rd + (-k1d / 3 + k2d) * h)
        k4u, k4d = f(t + h, ru + (k1u - k2u + k3u) * h, rd + (k1d - k2d + k3d) * h)
        return (ru + (k1u + 3 * k2u + 3 * k3u + k4u) * h / 8,
                rd + (k1d + 3 * k2d + 3 * k3d + k4d) * h / 8)

    du = np.zeros((n, Tp)); dd = np.zeros((n, Tp))
    d2u = np.zeros((n, Tp)); d2d = np.zeros((n, Tp)); dud = np.zeros((n, Tp))
    final = np.zeros_like(rho0)
    for b in range(B):
        ru = rho0[b, 0].copy(); rd = rho0[b, 1].copy()
        # the engine's Hermitian projection of injected states
        for r in (ru, rd):
            iu = np.triu_indices(n, 1)
            r[iu[1], iu[0]] = np.conj(r[iu])
            r[np.diag_indices(n)] = np.real(np.diag(r))
        t = 0.0
        for it in range(Tp):
            if method == METHOD_HF and it > 0:
                for _ in range(S):
                    ru, rd = step(t, ru, rd); t += h
            a = np.real(np.diag(ru)); c = np.real(np.diag(rd))
            du[:, it] += a; dd[:, it] += c
            d2u[:, it] += a * a; d2d[:, it] += c * c; dud[:, it] += a * c
            if method == METHOD_FTWA:
                for _ in range(S):
                    ru, rd = step(t, ru, rd); t += h
        final[b, 0] = ru; final[b, 1] = rd
    out = {"final": final}
    if method == METHOD_FTWA:
        out["niiu"] = du / B + 0.5
        out["niid"] = dd / B + 0.5
        out["n2iiu"] = d2u / B + du / B + 0.25
        out["n2iid"] = d2d / B + dd / B + 0.25
        out["nund"] = dud / B + (du + dd) / (2 * B) + 0.25
    else:
        out["niiu"] = du / B; out["niid"] = dd / B
        out["n2iiu"] = d2u / B; out["n2iid"] = d2d / B; out["nund"] = dud / B
    return out
