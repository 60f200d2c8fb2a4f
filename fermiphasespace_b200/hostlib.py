"""ctypes front-end of libfpshost.so (include/fps_host.h): the C++ system loader,
the `fps` driver and the system generator, for Python callers and tests."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfpshost.so")
FPS_EXE = os.path.join(HERE, "_lib", "fps")
MAKE_SITES_EXE = os.path.join(HERE, "_lib", "makeSitesSystem")

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build the package first")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.fpsh_system_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        L.fpsh_system_free.argtypes = [vp]
        L.fpsh_system_free.restype = None
        L.fpsh_system_n.argtypes = [vp]
        L.fpsh_system_matrices.argtypes = [vp, _dp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int)]
        L.fpsh_system_occupations.argtypes = [vp, _dp, _dp]
        L.fpsh_system_ground_state.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp]
        L.fpsh_system_positions.argtypes = [vp, _dp]
        L.fpsh_run_fps.argtypes = [ctypes.c_char_p]
        L.fpsh_make_sites_system.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _dp, ctypes.c_int,
                                             ctypes.c_char_p]
        L.fpsh_last_error.restype = ctypes.c_char_p
        L.fpsh_shard_range.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
        L.fpsh_shard_sum.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                     ctypes.c_longlong, ctypes.c_double]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _colmajor(buf: np.ndarray, n: int) -> np.ndarray:
    return buf.reshape(n, n).T.copy()


class System:
    """An FHSystem loaded by the C++ host layer from a simulation JSON file."""

    def __init__(self, json_path: str):
        self.L = load()
        h = ctypes.c_void_p()
        if self.L.fpsh_system_load(json_path.encode(), ctypes.byref(h)) != 0:
            raise RuntimeError(self.L.fpsh_last_error().decode())
        self.h = h
        self.n = int(self.L.fpsh_system_n(h))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.fpsh_system_free(self.h)
            self.h = None

    def matrices(self):
        n = self.n
        bufs = [np.zeros(n * n) for _ in range(4)]
        flags = (ctypes.c_int * 3)()
        self.L.fpsh_system_matrices(self.h, *[_p(b) for b in bufs], flags)
        tM, U, V, ext = (_colmajor(b, n) for b in bufs)
        return {"tM": tM, "U": U, "V": V, "ext": ext, "coulomb": flags[0], "ext_null": bool(flags[1]),
                "core_hole": bool(flags[2])}

    def occupations(self, n_lattice: int):
        up, dn = np.zeros(n_lattice), np.zeros(n_lattice)
        self.L.fpsh_system_occupations(self.h, _p(up), _p(dn))
        return up, dn

    def ground_state(self, which: int, n_lattice: int):
        nu, nd = np.zeros(n_lattice * n_lattice), np.zeros(n_lattice * n_lattice)
        eu, ed = np.zeros(n_lattice), np.zeros(n_lattice)
        self.L.fpsh_system_ground_state(self.h, which, _p(nu), _p(nd), _p(eu), _p(ed))
        return _colmajor(nu, n_lattice), _colmajor(nd, n_lattice), eu, ed

    def positions(self, n_lattice: int):
        xyz = np.zeros(3 * n_lattice)
        self.L.fpsh_system_positions(self.h, _p(xyz))
        return xyz.reshape(n_lattice, 3)


def make_sites_system(name: str, folder: str, geometry: str, params, ic: str = "ic_sw"):
    L = load()
    prm = np.ascontiguousarray(params, dtype=np.float64)
    rc = L.fpsh_make_sites_system(name.encode(), folder.encode(), geometry.encode(), _p(prm), len(prm), ic.encode())
    if rc != 0:
        raise RuntimeError(L.fpsh_last_error().decode())


def shard_range(n_traj: int, rank: int, world: int) -> tuple[int, int]:
    """[first, end) of rank's trajectories, as the C++ fps shards them."""
    L = load()
    a, b = ctypes.c_longlong(), ctypes.c_longlong()
    if L.fpsh_shard_range(n_traj, rank, world, ctypes.byref(a), ctypes.byref(b)) != 0:
        raise RuntimeError(L.fpsh_last_error().decode())
    return a.value, b.value


def shard_sum(data: np.ndarray, rank: int, world: int, port: int, addr: str = "127.0.0.1",
              timeout_s: float = 30.0) -> np.ndarray:
    """Element-wise sum over `world` processes (the exchange sharded fps runs use)."""
    L = load()
    buf = np.ascontiguousarray(data, dtype=np.float64).copy()
    if L.fpsh_shard_sum(addr.encode(), port, rank, world, _p(buf), buf.size, timeout_s) != 0:
        raise RuntimeError(L.fpsh_last_error().decode())
    return buf
