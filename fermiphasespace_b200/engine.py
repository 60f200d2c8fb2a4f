"""ctypes front-end of libfpsg.so (the C ABI in include/fpsg.h).

This module is plumbing for tests, the benchmark and Python callers; the C++ host
layer (fermiphasespace_b200/host) binds the same ABI directly.  It loads the
in-tree library and fails loudly when it is missing — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfpsg.so")

OK, ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_DIVERGED, ERR_STATE, ERR_UNSUPPORTED, ERR_NO_DEVICE = \
    0, -1, -2, -3, -4, -5, -6, -7, -8
METHOD_FTWA, METHOD_HF = 0, 1
PREC_FP64, PREC_FP32, PREC_SPLIT_BF16X3, PREC_SPLIT_TF32X3 = 0, 1, 2, 3
COUL_NULL, COUL_ONSITE, COUL_DISTANCE = 0, 1, 2
PATH_AUTO, PATH_STREAM, PATH_RESIDENT, PATH_DENSE = 0, 1, 2, 3
OBS_DIAG, OBS_DIAG2, OBS_DOUBLONS, OBS_WHOLE, OBS_ENERGIES = 1, 2, 4, 8, 16
OBS_DEFAULT = OBS_DIAG | OBS_DIAG2 | OBS_DOUBLONS | OBS_ENERGIES
FLAG_TEST_EXPIRE_WAIT = 0x1
FLAG_FP32_PLAIN_STATE = 0x2

# every symbol include/fpsg.h declares
EXPORTS = (
    "fpsg_create", "fpsg_destroy", "fpsg_last_error", "fpsg_set_memory_cap", "fpsg_set_system",
    "fpsg_set_pulse", "fpsg_set_initial_samples", "fpsg_sample", "fpsg_run", "fpsg_advance",
    "fpsg_get_state", "fpsg_num_trajectories", "fpsg_version", "fpsg_ensemble_sums_noalloc", "fpsg_grad",
    "fpsg_sample_range", "fpsg_run_batch", "fpsg_set_grad_memory", "fpsg_last_grad_info", "fpsg_gpsr_drift",
)

_dp = ctypes.POINTER(ctypes.c_double)


class GradInfo(ctypes.Structure):
    _fields_ = [("chunk_traj", ctypes.c_int), ("chunks", ctypes.c_int), ("segments", ctypes.c_int),
                ("kept_segments", ctypes.c_int)]


class Outputs(ctypes.Structure):
    _fields_ = [
        ("time", _dp), ("niiu", _dp), ("niid", _dp), ("n2iiu", _dp), ("n2iid", _dp), ("nund", _dp),
        ("energies", _dp), ("whole_u", _dp), ("whole_d", _dp),
        ("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
        ("traj_steps", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
        ("path_used", ctypes.c_int), ("reserved", ctypes.c_int),
    ]


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("tM", _dp), ("U", _dp), ("V", _dp), ("extpot", _dp),
        ("coulomb_kind", ctypes.c_int), ("extpot_is_null", ctypes.c_int), ("n_traj", ctypes.c_int),
        ("seed", ctypes.c_uint64), ("occ_up", _dp), ("occ_dn", _dp), ("out", ctypes.POINTER(Outputs)),
    ]


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("block_threads", ctypes.c_int), ("schedule", ctypes.c_int), ("grid", ctypes.c_int),
        ("graph_nodes", ctypes.c_int), ("tune_ms", ctypes.c_double), ("device_ms", ctypes.c_double),
        ("traj_steps", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
    ]


class FpsgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fpsg error {code}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libfpsg.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.fpsg_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_uint64]
    L.fpsg_create.restype = ctypes.c_int
    L.fpsg_destroy.argtypes = [vp]
    L.fpsg_destroy.restype = None
    L.fpsg_last_error.argtypes = [vp]
    L.fpsg_last_error.restype = ctypes.c_char_p
    L.fpsg_set_memory_cap.argtypes = [vp, ctypes.c_uint64]
    L.fpsg_set_memory_cap.restype = ctypes.c_int
    L.fpsg_set_grad_memory.argtypes = [vp, ctypes.c_int64]
    L.fpsg_set_grad_memory.restype = ctypes.c_int
    L.fpsg_last_grad_info.argtypes = [vp, ctypes.POINTER(GradInfo)]
    L.fpsg_last_grad_info.restype = ctypes.c_int
    L.fpsg_gpsr_drift.argtypes = [vp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, _dp]
    L.fpsg_gpsr_drift.restype = ctypes.c_int
    L.fpsg_set_system.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
    L.fpsg_set_system.restype = ctypes.c_int
    L.fpsg_set_pulse.argtypes = [vp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp]
    L.fpsg_set_pulse.restype = ctypes.c_int
    L.fpsg_set_initial_samples.argtypes = [vp, ctypes.c_int, _dp]
    L.fpsg_set_initial_samples.restype = ctypes.c_int
    L.fpsg_sample.argtypes = [vp, ctypes.c_int, ctypes.c_uint64, _dp, _dp, _dp, _dp]
    L.fpsg_sample.restype = ctypes.c_int
    L.fpsg_sample_range.argtypes = [vp, ctypes.c_int64, ctypes.c_int, ctypes.c_uint64, _dp, _dp, _dp, _dp]
    L.fpsg_sample_range.restype = ctypes.c_int
    L.fpsg_run_batch.argtypes = [vp, ctypes.POINTER(SystemDesc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(BatchInfo)]
    L.fpsg_run_batch.restype = ctypes.c_int
    L.fpsg_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                           ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(Outputs)]
    L.fpsg_run.restype = ctypes.c_int
    L.fpsg_advance.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                               ctypes.c_double, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int64)]
    L.fpsg_advance.restype = ctypes.c_int
    L.fpsg_get_state.argtypes = [vp, _dp]
    L.fpsg_get_state.restype = ctypes.c_int
    L.fpsg_num_trajectories.argtypes = [vp]
    L.fpsg_num_trajectories.restype = ctypes.c_int
    L.fpsg_version.argtypes = []
    L.fpsg_version.restype = ctypes.c_char_p
    L.fpsg_ensemble_sums_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p]
    L.fpsg_grad.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            _dp, _dp, _dp, _dp, _dp, _dp]
    L.fpsg_grad.restype = ctypes.c_int
    L.fpsg_ensemble_sums_noalloc.restype = ctypes.c_int
    _lib = L
    return L


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def to_colmajor_cx(m, n: int) -> np.ndarray:
    """n x n (real or complex) -> interleaved complex col-major float64 buffer."""
    a = np.asarray(m, dtype=np.complex128).reshape(n, n)
    return np.ascontiguousarray(a.T).view(np.float64).reshape(-1).copy()


def states_to_buffer(rho: np.ndarray) -> np.ndarray:
    """[B,2,n,n] complex -> [B][2][n][n] col-major interleaved float64."""
    r = np.asarray(rho, dtype=np.complex128)
    return np.ascontiguousarray(np.transpose(r, (0, 1, 3, 2))).view(np.float64).reshape(-1).copy()


def buffer_to_states(buf: np.ndarray, B: int, n: int) -> np.ndarray:
    f = buf.view(np.complex128).reshape(B, 2, n, n)
    return np.transpose(f, (0, 1, 3, 2)).copy()


@dataclass
class RunResult:
    time: np.ndarray
    niiu: np.ndarray
    niid: np.ndarray
    n2iiu: np.ndarray
    n2iid: np.ndarray
    nund: np.ndarray
    energies: np.ndarray
    whole_u: np.ndarray | None
    whole_d: np.ndarray | None
    device_ms: float
    total_ms: float
    traj_steps: int
    launches: int
    path_used: int


class Engine:
    """One fpsg context on one CUDA device."""

    def __init__(self, device: int = 0, flags: int = 0):
        self.L = load()
        h = ctypes.c_void_p()
        rc = self.L.fpsg_create(ctypes.byref(h), int(device), int(flags))
        if rc != OK:
            raise FpsgError(rc, "fpsg_create failed (no CUDA device?)")
        self.h = h
        self.n = 0
        self._n_bins = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.fpsg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OK:
            raise FpsgError(rc, self.L.fpsg_last_error(self.h).decode())

    def set_memory_cap(self, nbytes: int):
        self._check(self.L.fpsg_set_memory_cap(self.h, int(nbytes)))

    def set_grad_memory(self, nbytes: int):
        """Bytes fpsg_grad may keep for stage inputs from its forward pass
        (-1 automatic, 0 recompute every segment)."""
        self._check(self.L.fpsg_set_grad_memory(self.h, int(nbytes)))

    def set_system(self, tM, U, V=None, ext=None, coulomb: int = COUL_ONSITE, ext_null: bool | None = None):
        tM = np.asarray(tM)
        n = tM.shape[0]
        if ext_null is None:
            ext_null = ext is None
        bufs = [to_colmajor_cx(tM, n), to_colmajor_cx(U, n),
                to_colmajor_cx(V, n) if V is not None else None,
                to_colmajor_cx(ext, n) if ext is not None else None]
        self._check(self.L.fpsg_set_system(self.h, n, *[_ptr(b) for b in bufs], int(coulomb), int(bool(ext_null))))
        self.n = n

    def set_pulse(self, amp, bin_width: float, t0: float, td: float, proj):
        amp = np.ascontiguousarray(amp, dtype=np.float64)
        proj = np.ascontiguousarray(proj, dtype=np.float64)
        self._check(self.L.fpsg_set_pulse(self.h, len(amp), _ptr(amp), bin_width, t0, td, _ptr(proj)))
        self._n_bins = len(amp)

    def clear_pulse(self):
        self._check(self.L.fpsg_set_pulse(self.h, 0, None, 1.0, 0.0, 1.0, None))
        self._n_bins = 0

    def set_initial_samples(self, rho0: np.ndarray):
        buf = states_to_buffer(rho0)
        self._check(self.L.fpsg_set_initial_samples(self.h, int(rho0.shape[0]), _ptr(buf)))

    def sample(self, B: int, seed: int, occ_up, occ_dn, rot_up=None, rot_dn=None, first: int = 0):
        """Draws trajectories first .. first+B-1 of the seed's ensemble."""
        ou = np.ascontiguousarray(occ_up, dtype=np.float64)
        od = np.ascontiguousarray(occ_dn, dtype=np.float64)
        ru = to_colmajor_cx(rot_up, self.n) if rot_up is not None else None
        rd = to_colmajor_cx(rot_dn, self.n) if rot_dn is not None else None
        self._check(self.L.fpsg_sample_range(self.h, int(first), int(B), int(seed), _ptr(ou), _ptr(od), _ptr(ru),
                                             _ptr(rd)))

    def num_trajectories(self) -> int:
        return int(self.L.fpsg_num_trajectories(self.h))

    def get_state(self) -> np.ndarray:
        B = self.num_trajectories()
        buf = np.zeros(B * 4 * self.n * self.n)
        self._check(self.L.fpsg_get_state(self.h, _ptr(buf)))
        return buffer_to_states(buf, B, self.n)

    def run(self, method: int, precision: int, dt: float, S: int, Tp: int, obs: int = OBS_DEFAULT,
            path: int = PATH_AUTO) -> RunResult:
        n = self.n
        arrs = {k: np.zeros((n, Tp)) for k in ("niiu", "niid", "n2iiu", "n2iid", "nund")}
        tarr = np.zeros(Tp)
        en = np.zeros((5, Tp))
        wu = wd = None
        if obs & OBS_WHOLE:
            wu = np.zeros((Tp, n, n, 2))
            wd = np.zeros((Tp, n, n, 2))
        o = Outputs()
        o.time = _ptr(tarr)
        for k, v in arrs.items():
            setattr(o, k, _ptr(v))
        o.energies = _ptr(en)
        o.whole_u = _ptr(wu)
        o.whole_d = _ptr(wd)
        self._check(self.L.fpsg_run(self.h, int(method), int(precision), int(path), float(dt), int(S), int(Tp),
                                    int(obs), ctypes.byref(o)))

        def whole(w):
            if w is None:
                return None
            return np.transpose(w.view(np.complex128)[..., 0], (0, 2, 1)).copy()

        return RunResult(time=tarr, energies=en, whole_u=whole(wu), whole_d=whole(wd), device_ms=o.device_ms,
                         total_ms=o.total_ms, traj_steps=o.traj_steps, launches=o.kernel_launches,
                         path_used=o.path_used, **arrs)

    def run_batch(self, systems: list, method: int, precision: int, dt: float, S: int, Tp: int,
                  obs: int = OBS_DEFAULT) -> tuple[list, dict]:
        """Integrates several systems together (fpsg_run_batch).  Each entry of
        `systems` is a dict with tM, U, V (or None), ext (or None), coulomb,
        n_traj, seed, occ_up, occ_dn.  Returns one RunResult per system and the
        batch information (autotuner choice, graph size, device time)."""
        keep, descs, results = [], (SystemDesc * len(systems))(), []
        for k, sy in enumerate(systems):
            tM = np.asarray(sy["tM"])
            n = tM.shape[0]
            mats = [to_colmajor_cx(tM, n), to_colmajor_cx(sy["U"], n),
                    to_colmajor_cx(sy["V"], n) if sy.get("V") is not None else None,
                    to_colmajor_cx(sy["ext"], n) if sy.get("ext") is not None else None]
            ou = np.ascontiguousarray(sy["occ_up"], dtype=np.float64)
            od = np.ascontiguousarray(sy["occ_dn"], dtype=np.float64)
            arrs = {key: np.zeros((n, Tp)) for key in ("niiu", "niid", "n2iiu", "n2iid", "nund")}
            tarr, en = np.zeros(Tp), np.zeros((5, Tp))
            o = Outputs()
            o.time = _ptr(tarr)
            for key, v in arrs.items():
                setattr(o, key, _ptr(v))
            o.energies = _ptr(en)
            d = descs[k]
            d.n, d.tM, d.U, d.V, d.extpot = n, _ptr(mats[0]), _ptr(mats[1]), _ptr(mats[2]), _ptr(mats[3])
            d.coulomb_kind = int(sy.get("coulomb", COUL_ONSITE))
            d.extpot_is_null = int(sy.get("ext") is None)
            d.n_traj, d.seed = int(sy["n_traj"]), int(sy["seed"])
            d.occ_up, d.occ_dn = _ptr(ou), _ptr(od)
            d.out = ctypes.pointer(o)
            keep.append((mats, ou, od, o))
            results.append((o, tarr, en, arrs))
        info = BatchInfo()
        self._check(self.L.fpsg_run_batch(self.h, descs, len(systems), int(method), int(precision), float(dt), int(S),
                                          int(Tp), int(obs), ctypes.byref(info)))
        out = [RunResult(time=tarr, energies=en, whole_u=None, whole_d=None, device_ms=o.device_ms, total_ms=o.total_ms,
                         traj_steps=o.traj_steps, launches=o.kernel_launches, path_used=o.path_used, **arrs)
               for (o, tarr, en, arrs) in results]
        return out, {f: getattr(info, f) for f, _ in BatchInfo._fields_}

    def grad(self, precision: int, dt: float, S: int, Tp: int, checkpoint_every: int = 16) -> dict:
        """Loss L = sum_t w_t mean_i <n_up n_dn>(t) and its gradient with respect to the
        U scale, the tM scale and the pulse amplitudes (fpsg_grad); the state is kept."""
        loss, gu, gt, ms, fms = (ctypes.c_double() for _ in range(5))
        n_bins = self._n_bins
        gp = np.zeros(max(1, n_bins))
        self._check(self.L.fpsg_grad(self.h, int(precision), float(dt), int(S), int(Tp), int(checkpoint_every),
                                     ctypes.byref(loss), ctypes.byref(gu), ctypes.byref(gt), _ptr(gp),
                                     ctypes.byref(ms), ctypes.byref(fms)))
        gi = GradInfo()
        self._check(self.L.fpsg_last_grad_info(self.h, ctypes.byref(gi)))
        return {"loss": loss.value, "dU": gu.value, "dt": gt.value, "dpulse": gp[:n_bins].copy(),
                "device_ms": ms.value, "forward_ms": fms.value, "chunk_traj": gi.chunk_traj,
                "chunks": gi.chunks, "segments": gi.segments, "kept_segments": gi.kept_segments}

    def gpsr_drift(self, rho: np.ndarray, d_t: float, t: float = 0.0) -> np.ndarray:
        """GPSR drift increments (fpsg_gpsr_drift) of general complex states
        rho [B, 2, n, n] over one step d_t, with the context's system."""
        rho = np.asarray(rho, dtype=np.complex128)
        B, n = rho.shape[0], rho.shape[-1]
        buf = np.ascontiguousarray(np.transpose(rho, (0, 1, 3, 2))).view(np.float64).reshape(-1)
        out = np.zeros_like(buf)
        self._check(self.L.fpsg_gpsr_drift(self.h, int(B), _ptr(buf), float(t), float(d_t), _ptr(out)))
        f = out.view(np.complex128).reshape(B, 2, n, n)
        return np.transpose(f, (0, 1, 3, 2)).copy()

    def advance(self, method: int, precision: int, dt: float, S: int, n_steps: int, t_start: float = 0.0,
                path: int = PATH_AUTO) -> tuple[float, int]:
        ms = ctypes.c_double()
        launches = ctypes.c_int64()
        self._check(self.L.fpsg_advance(self.h, int(method), int(precision), int(path), float(dt), int(S),
                                        float(t_start), int(n_steps), ctypes.byref(ms), ctypes.byref(launches)))
        return ms.value, launches.value
