"""fpsg_ensemble_sums_noalloc: the ensemble sums for callers that cannot allocate.

Callers that run while a CUDA graph is captured, or whose device memory belongs
to another runtime's allocator, cannot let a library call cudaMalloc.  This entry
point takes their device buffers and keeps its partial sums in a static device
array instead.  Its sums, normalised as the reference normalises them
(src/FHfTWASolver.cpp:506-532), must equal what fpsg_run's stream path reports for
the same states at t = 0 bit for bit (same chunking, same Kahan combine), and the
plain NumPy sums of the same diagonals to rounding.  Here the test owns the device
buffers (allocated with torch); the entry point itself allocates nothing.  Every
case makes two calls in a row, the second reusing the array the first left
behind.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same tolerance as the FP64 observable parity tests


def normalise(sums: np.ndarray, B: int, n: int) -> dict:
    su, sd, s2u, s2d, sud = (sums[o * n:(o + 1) * n] for o in range(5))
    return {
        "niiu": su / B + 0.5,
        "niid": sd / B + 0.5,
        "n2iiu": (s2u / B + (su + su) / (2.0 * B)) + 0.25,
        "n2iid": (s2d / B + (sd + sd) / (2.0 * B)) + 0.25,
        "nund": (sud / B + (su + sd) / (2.0 * B)) + 0.25,
    }


def numpy_sums(states: np.ndarray) -> np.ndarray:
    d = np.real(np.diagonal(states, axis1=2, axis2=3))   # [B][2][n]
    du, dd = d[:, 0], d[:, 1]
    return np.concatenate([du.sum(0), dd.sum(0), (du * du).sum(0), (dd * dd).sum(0), (du * dd).sum(0)])


def call(L, E, rho, B, n, sums, stream):
    s = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    return L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), B, n, ctypes.c_void_p(sums.data_ptr()), s)


@pytest.mark.parametrize("nx,ny,cases,use_null", [
    (4, 3, [(37, 11), (130, 12)], False),      # several chunks, a ragged last one
    (4, 3, [(1, 13), (4097, 14)], False),      # one trajectory; 65 chunks
    (4, 3, [(5, 15), (70, 16)], True),         # the legacy NULL stream
    (32, 16, [(2, 17), (3, 18)], False),       # n = 512, the largest n the header names
], ids=["ragged", "B1_B4097", "null_stream", "n512"])
def test_noalloc_sums_match_stream_path_and_numpy(engine_lib, nx, ny, cases, use_null):
    import torch
    from fermiphasespace_b200 import configs
    E = engine_lib
    L = E.load()
    w = configs.grid(nx, ny, U0=4.0, seed=2)
    n = w.n
    eng = E.Engine(0)
    try:
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        stream = None if use_null else torch.cuda.current_stream()
        for k, (B, seed) in enumerate(cases):
            eng.sample(B, seed, w.occ_up, w.occ_dn)
            states = eng.get_state()
            # the existing entry point: observables of snapshot 0 of a stream-path run
            ref = eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 1, obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS,
                          path=E.PATH_STREAM)
            rho = torch.from_numpy(E.states_to_buffer(states)).cuda()
            sums = torch.full((5 * n,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = call(L, E, rho, B, n, sums, stream)
            assert rc == E.OK, (k, rc)
            torch.cuda.synchronize()
            raw = sums.cpu().numpy()
            got = normalise(raw, B, n)
            for key, v in got.items():
                assert np.array_equal(v, getattr(ref, key)[:, 0]), (k, key, np.abs(v - getattr(ref, key)[:, 0]).max())
            want = numpy_sums(states)
            assert np.abs(raw - want).max() <= TOL * max(1.0, B), (k, np.abs(raw - want).max())
    finally:
        eng.close()


def test_noalloc_rejects_sizes_beyond_its_array(engine_lib):
    import torch
    E = engine_lib
    L = E.load()
    rho = torch.zeros(64, dtype=torch.float64, device="cuda")
    sums = torch.zeros(64, dtype=torch.float64, device="cuda")
    # n = 512 fits 102 chunks of 64 trajectories: B = 6528 is the largest accepted
    # request, B = 6529 needs a 103rd chunk (both are rejected or accepted before
    # anything is read, so small buffers stand in for the states)
    assert L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), 6529, 512,
                                        ctypes.c_void_p(sums.data_ptr()), None) == E.ERR_INVALID
    assert L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), 1, 60000,
                                        ctypes.c_void_p(sums.data_ptr()), None) == E.ERR_INVALID
    assert L.fpsg_ensemble_sums_noalloc(None, 2, 6, ctypes.c_void_p(sums.data_ptr()), None) == E.ERR_INVALID
    assert L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), 0, 6,
                                        ctypes.c_void_p(sums.data_ptr()), None) == E.ERR_INVALID
