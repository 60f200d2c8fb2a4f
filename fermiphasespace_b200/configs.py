"""Synthetic systems of the benchmark workloads, built as FermiPhaseSpace would.

Geometry follows makeBCGrid (src/FHLattice.cpp:872-895: x fastest, then y, z,
spacing a); hopping follows FHTunnelingInteraction::addTunneling
(src/FHTunnelingInteraction.cpp:293-312: +E on i<j pairs whose distance matches
a shell within (d - dist)^2 < samePointDistance, mirrored); on-site Coulomb
follows FHCoulombInteraction::addCoulombinU (src/FHCoulombInteraction.cpp:246-264:
U_ij += U0 where d_ij^2 < samePointDistance, i.e. the diagonal for ordinary
lattices).  samePointDistance is the JSON-lattice default 1e-4
(include/FHLattice.h:77).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SAME_POINT = 1e-4


def grid_positions(nx: int, ny: int, nz: int = 1, a: float = 1.0) -> np.ndarray:
    return np.array([(a * x, a * y, a * z) for z in range(nz) for y in range(ny) for x in range(nx)],
                    dtype=np.float64)


def distances(pos: np.ndarray) -> np.ndarray:
    d = pos[:, None, :] - pos[None, :, :]
    return np.sqrt((d * d).sum(-1))


def hopping(D: np.ndarray, shells) -> np.ndarray:
    n = D.shape[0]
    T = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            for dist, E in shells:
                if (D[i, j] - dist) ** 2 < SAME_POINT:
                    T[i, j] += E
                    T[j, i] += E
    return T


def onsite(D: np.ndarray, U0: float) -> tuple[np.ndarray, np.ndarray]:
    n = D.shape[0]
    close = D ** 2 < SAME_POINT
    U = np.where(close, U0, 0.0)
    V = np.where(close & ~np.eye(n, dtype=bool), U0, 0.0)
    return U, V


@dataclass
class Workload:
    name: str
    tM: np.ndarray
    U: np.ndarray
    V: np.ndarray
    ext: np.ndarray | None
    occ_up: np.ndarray
    occ_dn: np.ndarray
    dt: float
    S: int
    t_max: float
    n_traj: int

    @property
    def n(self) -> int:
        return self.tM.shape[0]

    @property
    def n_snapshots(self) -> int:
        # FHSolver::setTimeParameters, src/FHSolver.cpp:100
        return int(np.floor(self.t_max / self.dt + 1))

    @property
    def nnz_offdiag(self) -> int:
        return int(np.count_nonzero(self.tM - np.diag(np.diag(self.tM))))


def grid_3x2(n_traj: int = 1000) -> Workload:
    """3x2 grid, t=1 (E=-1), U=4, no potential, Neel product state, dt=0.01,
    stepsParTimePoints=10, t_max=10 (the CPU-runnable plain fTWA case)."""
    pos = grid_positions(3, 2)
    D = distances(pos)
    T = hopping(D, [(1.0, -1.0)])
    U, V = onsite(D, 4.0)
    # spinWave (src/FHSystem.cpp:559-570): up on even sites, down on odd
    occ_u = np.array([1.0 if i % 2 == 0 else 0.0 for i in range(6)])
    return Workload("grid3x2_U4_neel", T, U, V, None, occ_u, 1.0 - occ_u, 0.01, 10, 10.0, n_traj)


def grid_10x10(U0: float = 4.0, W: float = 2.0, seed: int = 0, n_traj: int = 16384,
               t_max: float = 20.0) -> Workload:
    """10x10 grid, t=1, on-site U, static random site potential uniform in
    [-W/2, W/2] (seeded), domain wall (both spins on x < 5), dt=0.005, S=1."""
    pos = grid_positions(10, 10)
    D = distances(pos)
    T = hopping(D, [(1.0, -1.0)])
    U, V = onsite(D, U0)
    rng = np.random.default_rng(seed)
    w = rng.uniform(-W / 2, W / 2, size=100)
    ext = np.diag(w)
    occ = np.array([1.0 if (i % 10) < 5 else 0.0 for i in range(100)])
    return Workload(f"grid10x10_U{U0:g}_W{W:g}_domainwall", T, U, V, ext, occ, occ.copy(), 0.005, 1, t_max, n_traj)


def grid(nx: int, ny: int, U0: float = 4.0, seed: int = 0, n_traj: int = 1024, dt: float = 0.01,
         S: int = 1, t_max: float = 2.0) -> Workload:
    """nx x ny grid, t=1, on-site U, seeded random half-filled product state."""
    pos = grid_positions(nx, ny)
    D = distances(pos)
    T = hopping(D, [(1.0, -1.0)])
    U, V = onsite(D, U0)
    n = nx * ny
    rng = np.random.default_rng(seed)
    occ_u = np.zeros(n); occ_u[rng.permutation(n)[: (n + 1) // 2]] = 1.0
    occ_d = np.zeros(n); occ_d[rng.permutation(n)[: n // 2]] = 1.0
    return Workload(f"grid{nx}x{ny}_U{U0:g}", T, U, V, None, occ_u, occ_d, dt, S, t_max, n_traj)


def adjoint_8x8(n_traj: int = 2048, n_bins: int = 50, seed: int = 0, t_max: float = 10.0, dt: float = 0.01):
    """8x8 grid, t=1, on-site U=4, seeded half-filled product state, and a per-time-bin
    site pulse v_i(t) = a_b(t) exp(-((t - t0)/td)^2 / 2) (x_i - <x>), n_bins bins over
    [0, t_max], a_b ~ N(0, 0.5^2) seeded, t0 = t_max/2, td = t_max/5.  The loss of
    the adjoint is the time-integrated doublon occupancy over [0, t_max]."""
    w = grid(8, 8, U0=4.0, seed=seed, n_traj=n_traj, dt=dt, S=1, t_max=t_max)
    w.name = f"grid8x8_U4_pulse{n_bins}"
    pos = grid_positions(8, 8)
    rng = np.random.default_rng(seed + 17)
    pulse = {"n_bins": n_bins, "amp": rng.normal(0.0, 0.5, n_bins), "bin_width": t_max / n_bins,
             "t0": t_max / 2, "td": t_max / 5, "proj": pos[:, 0] - pos[:, 0].mean()}
    return w, pulse


def moire_positions(nx: int = 8, ny: int = 8, a: float = 1.42, d: float = 3.35, theta_deg: float = 5.0) -> np.ndarray:
    """Site positions of the twisted-bilayer honeycomb from the engine's own
    system generator (`makeSitesSystem <name> <folder> moire nx ny a d theta`)."""
    import tempfile

    from . import hostlib
    with tempfile.TemporaryDirectory() as tmp:
        hostlib.make_sites_system("moire", tmp + "/", "moire", [nx, ny, a, d, theta_deg])
        s = hostlib.System(tmp + "/moire.json")
        return s.positions(s.n)


def moire_8x8(U0: float = 1.0, n_traj: int = 2048, seed: int = 0, dt: float = 0.005, t_max: float = 2.0,
              a: float = 1.42, pos: np.ndarray | None = None) -> Workload:
    """Twisted bilayer honeycomb, 8x8 cells per layer, theta = 5 deg, interlayer
    distance 3.35, a = 1.42 (256 sites).  Distance-decaying hopping
    t(r) = exp(-(r - a)/0.45) for 0 < r <= 4a (tM_ij = -t(r)), long-range Coulomb
    U_ij = U0/(1 + r) (r = 0 included) and V_ij = U0/(1 + r) for i != j
    (coulomb kind DISTANCE), seeded random half-filled product state."""
    if pos is None:
        pos = moire_positions(a=a)
    D = distances(pos)
    n = pos.shape[0]
    T = np.where((D > 1e-6) & (D <= 4 * a + 1e-9), -np.exp(-(D - a) / 0.45), 0.0)
    U = U0 / (1.0 + D)
    V = U0 / (1.0 + D)
    np.fill_diagonal(V, 0.0)
    rng = np.random.default_rng(seed)
    occ_u = np.zeros(n); occ_u[rng.permutation(n)[: n // 2]] = 1.0
    occ_d = np.zeros(n); occ_d[rng.permutation(n)[: n // 2]] = 1.0
    return Workload(f"moire8x8_theta5_U{U0:g}", T, U, V, None, occ_u, occ_d, dt, 1, t_max, n_traj)


def _system_from_generator(tmp: str, name: str, geometry: str, params, U0: float, neighbor: float | None = None):
    """(tM, U, V) of a generated system, through the engine's JSON loader."""
    import json

    from . import hostlib
    hostlib.make_sites_system(name, tmp + "/", geometry, params)
    path = f"{tmp}/{name}.json"
    doc = json.load(open(path))
    tun = doc["system"]["tunnelingInteraction"]
    if neighbor is not None:
        tun["neighborDistance"] = neighbor
    doc["system"]["coulombInteraction"] = {"type": "onSite", "onSiteInteraction": U0}
    with open(path, "w") as fh:
        json.dump(doc, fh)
    m = hostlib.System(path).matrices()
    return m["tM"].real.copy(), m["U"].real.copy(), m["V"].real.copy()


def uneven_batch(U0: float = 4.0, seed: int = 0, scale: float = 1.0) -> list[Workload]:
    """The uneven batch: kagome 6x6 (108 sites), honeycomb (graphene 3x4, 24 sites),
    periodic fcc 3x3x3 conventional cells (108 sites, nearest neighbours at a/sqrt 2),
    8x8 and 12x12 grids; t = 1 (nearest neighbours, E = -1), on-site U, each with
    its own seeded random half-filled product state; 2048 / 1024 / 1024 / 2048 /
    2048 trajectories (8192 in all, times `scale`); dt = 0.01, S = 1, t_max = 2."""
    import tempfile
    specs = [("kagome6x6", "kagome", [6, 6], None, 2048), ("honeycomb24", "graphene", [3, 4], None, 1024),
             ("fcc3x3x3p", "fccPeriodic", [3, 3, 3], 0.5 ** 0.5, 1024), ("grid8x8", "grid", [8, 8], None, 2048),
             ("grid12x12", "grid", [12, 12], None, 2048)]
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for k, (name, geo, prm, nb, B) in enumerate(specs):
            tM, U, V = _system_from_generator(tmp, name, geo, prm, U0, nb)
            n = tM.shape[0]
            rng = np.random.default_rng(seed + 101 * k)
            occ_u = np.zeros(n); occ_u[rng.permutation(n)[: (n + 1) // 2]] = 1.0
            occ_d = np.zeros(n); occ_d[rng.permutation(n)[: n // 2]] = 1.0
            out.append(Workload(f"{name}_U{U0:g}", tM, U, V, None, occ_u, occ_d, 0.01, 1, 2.0,
                                max(1, int(round(B * scale)))))
    return out
