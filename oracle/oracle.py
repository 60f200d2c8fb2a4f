"""ctypes front-end of the FP64 C oracle (oracle/fps_oracle.c).

TEST INFRASTRUCTURE ONLY — imported by tests/, by ``__graft_entry__.smoke()`` and
by the CPU-baseline leg of ``bench.py``, always as the checker or the timed CPU
restatement, never by the product.  The C file cites the FermiPhaseSpace functions
it restates (src/FHfTWASolver.cpp, src/FHHFSolver.cpp).  Parity of the oracle with
the reference is unpinned (the reference cannot be built here and ships no golden
outputs); it is pinned by analytic known-answer tests and by oracle/oracle_np.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

METHOD_FTWA, METHOD_HF = 0, 1
COUL_NULL, COUL_ONSITE, COUL_DISTANCE = 0, 1, 2
OBS_DIAG, OBS_DIAG2, OBS_DOUB, OBS_WHOLE, OBS_ENER = 1, 2, 4, 8, 16

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_run.restype = ctypes.c_int
        L.oracle_run.argtypes = [
            ctypes.c_int, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ctypes.c_uint,
            dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int,
            ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp,
        ]
        L.oracle_sample.restype = ctypes.c_int
        L.oracle_sample.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, dp, dp, dp]
        L.oracle_sample_range.restype = ctypes.c_int
        L.oracle_sample_range.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_uint64, dp, dp, dp]
        L.oracle_gauss_pair.restype = None
        L.oracle_gauss_pair.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, dp, dp]
        L.oracle_gpsr_drift.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp,
                                        ctypes.c_double, dp, ctypes.c_int]
        L.oracle_gpsr_drift.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _cx(m, n):
    if m is None:
        return None
    a = np.asfortranarray(np.asarray(m, dtype=np.complex128).reshape(n, n))
    return np.ascontiguousarray(a.T).reshape(-1).view(np.float64).copy()  # col-major interleaved


@dataclass
class System:
    """Dense Hamiltonian inputs (the matrices FHSystem hands the solvers)."""
    tM: np.ndarray
    U: np.ndarray
    V: np.ndarray | None = None
    ext: np.ndarray | None = None
    coulomb: int = COUL_ONSITE
    ext_null: bool = True
    pulse: dict | None = field(default=None)

    @property
    def n(self) -> int:
        return int(self.tM.shape[0])


def run(system: System, method: int, dt: float, S: int, Tp: int, rho0: np.ndarray,
        obs: int = OBS_DIAG | OBS_DIAG2 | OBS_DOUB | OBS_ENER, nthreads: int = 0,
        want_final: bool = True) -> dict:
    """Integrates rho0 ([B,2,n,n] complex) and returns normalised observables."""
    n = system.n
    rho0 = np.asarray(rho0, dtype=np.complex128)
    B = rho0.shape[0]
    # [B][2][n][n] complex, col-major per matrix: store the transpose row-major
    r0 = np.ascontiguousarray(np.transpose(rho0, (0, 1, 3, 2))).view(np.float64).reshape(-1)
    tM, U = _cx(system.tM, n), _cx(system.U, n)
    V = _cx(system.V if system.V is not None else np.zeros((n, n)), n)
    ext = _cx(system.ext, n) if system.ext is not None else None
    out = {k: np.zeros((n, Tp)) for k in ("niiu", "niid", "n2iiu", "n2iid", "nund")}
    out["time"] = np.zeros(Tp)
    out["energies"] = np.zeros((5, Tp))
    whole_u = whole_d = None
    if obs & OBS_WHOLE:
        whole_u = np.zeros((Tp, n, n, 2))
        whole_d = np.zeros((Tp, n, n, 2))
    final = np.zeros(B * 4 * n * n) if want_final else None
    pl = system.pulse or {}
    nb = int(pl.get("n_bins", 0))
    amp = np.ascontiguousarray(pl.get("amp", np.zeros(1)), dtype=np.float64)
    proj = np.ascontiguousarray(pl.get("proj", np.zeros(n)), dtype=np.float64)
    lib().oracle_run(
        n, _p(tM), _p(U), _p(V), _p(ext), int(system.coulomb), int(bool(system.ext_null)),
        int(method), float(dt), int(S), int(Tp), int(B), _p(r0), int(obs),
        _p(out["time"]), _p(out["niiu"]), _p(out["niid"]), _p(out["n2iiu"]), _p(out["n2iid"]),
        _p(out["nund"]), _p(out["energies"]), _p(whole_u), _p(whole_d), _p(final), int(nthreads),
        nb, _p(amp), float(pl.get("bin_width", 1.0)), float(pl.get("t0", 0.0)),
        float(pl.get("td", 1.0)), _p(proj))
    if final is not None:
        f = final.view(np.complex128).reshape(B, 2, n, n)
        out["final"] = np.transpose(f, (0, 1, 3, 2)).copy()
    if whole_u is not None:
        out["whole_u"] = np.transpose(whole_u.view(np.complex128)[..., 0], (0, 2, 1)).copy()
        out["whole_d"] = np.transpose(whole_d.view(np.complex128)[..., 0], (0, 2, 1)).copy()
    return out


def sample(n: int, B: int, seed: int, occ_up, occ_dn, first: int = 0) -> np.ndarray:
    """Product-state fTWA samples [B,2,n,n] from the engine's Philox convention:
    trajectories first .. first+B-1 of the seed's ensemble."""
    ou = np.ascontiguousarray(occ_up, dtype=np.float64)
    od = np.ascontiguousarray(occ_dn, dtype=np.float64)
    buf = np.zeros(B * 4 * n * n)
    lib().oracle_sample_range(n, int(first), B, seed, _p(ou), _p(od), _p(buf))
    f = buf.view(np.complex128).reshape(B, 2, n, n)
    return np.transpose(f, (0, 1, 3, 2)).copy()


def gauss_pair(seed: int, b: int, e: int) -> tuple[float, float]:
    g1, g2 = ctypes.c_double(), ctypes.c_double()
    lib().oracle_gauss_pair(seed, b, e, ctypes.byref(g1), ctypes.byref(g2))
    return g1.value, g2.value


def gpsr_drift(system: System, rho: np.ndarray, d_t: float, nthreads: int = 0) -> np.ndarray:
    """GPSR drift increments (src/FHGPSRSolver.cpp:168-206) of general complex states
    rho [B,2,n,n] over one step d_t; static potentials only."""
    n = system.n
    rho = np.asarray(rho, dtype=np.complex128)
    B = rho.shape[0]
    r0 = np.ascontiguousarray(np.transpose(rho, (0, 1, 3, 2))).view(np.float64).reshape(-1)
    tM, U = _cx(system.tM, n), _cx(system.U, n)
    ext = _cx(system.ext, n) if system.ext is not None else None
    out = np.zeros(B * 4 * n * n)
    lib().oracle_gpsr_drift(n, _p(tM), _p(U), _p(ext), int(system.coulomb), int(bool(system.ext_null)), int(B),
                            _p(r0), float(d_t), _p(out), int(nthreads))
    f = out.view(np.complex128).reshape(B, 2, n, n)
    return np.transpose(f, (0, 1, 3, 2)).copy()
