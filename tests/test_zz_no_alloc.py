"""fpsg_ensemble_sums_noalloc: the ensemble sums for callers that cannot allocate.

Callers that run while a CUDA graph is captured, or whose device memory belongs
to another runtime's allocator, cannot let a library call cudaMalloc.  This entry
point takes their device buffers and keeps its partial sums in a static device
array instead.  Its sums, normalised as the reference normalises them
(src/FHfTWASolver.cpp:506-532), must equal what fpsg_run reports for the same
states at t = 0.  Here the test owns the device buffers (allocated with torch);
the entry point itself allocates nothing.
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


def test_noalloc_sums_match_run(engine_lib):
    import torch
    from fermiphasespace_b200 import configs
    E = engine_lib
    L = E.load()
    w = configs.grid(4, 3, U0=4.0, seed=2)
    eng = E.Engine(0)
    try:
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        stream = torch.cuda.current_stream()
        for call, (B, seed) in enumerate([(37, 11), (130, 12)]):
            eng.sample(B, seed, w.occ_up, w.occ_dn)
            states = eng.get_state()
            # the existing entry point: observables of snapshot 0 of a run
            ref = eng.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 1, obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS)
            rho = torch.from_numpy(E.states_to_buffer(states)).cuda()
            sums = torch.full((5 * w.n,), float("nan"), dtype=torch.float64, device="cuda")
            rc = L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), B, w.n,
                                              ctypes.c_void_p(sums.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert rc == E.OK, (call, rc)
            torch.cuda.synchronize()
            got = normalise(sums.cpu().numpy(), B, w.n)
            for k, v in got.items():
                err = np.abs(v - getattr(ref, k)[:, 0]).max()
                assert err <= TOL, (call, k, err)
    finally:
        eng.close()


def test_noalloc_rejects_sizes_beyond_its_array(engine_lib):
    import torch
    E = engine_lib
    L = E.load()
    rho = torch.zeros(2 * 2 * 513 * 513 * 2, dtype=torch.float64, device="cuda")
    sums = torch.zeros(5 * 513, dtype=torch.float64, device="cuda")
    rc = L.fpsg_ensemble_sums_noalloc(ctypes.c_void_p(rho.data_ptr()), 2, 513, ctypes.c_void_p(sums.data_ptr()), None)
    assert rc == E.ERR_INVALID
    rc = L.fpsg_ensemble_sums_noalloc(None, 2, 6, ctypes.c_void_p(sums.data_ptr()), None)
    assert rc == E.ERR_INVALID
