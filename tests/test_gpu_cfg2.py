"""The 10x10 headline system at every on-site U it is quoted for (U = 2, 4, 8),
fTWA and Hartree-Fock, against the FP64 oracle on the same inputs.

Shape: 10x10 grid, t = 1, on-site U, static disorder W = 2 (seed 0), domain wall
(both spins on x < 5), dt = 0.005, stepsParTimePoints = 1.  fTWA: 8 trajectories,
50 snapshots (50 RK4 steps, src/FHfTWASolver.cpp:366-426).  HF: the deterministic
density matrix started from N0 = diag(occ) (src/FHHFSolver.cpp:75-88), 50
snapshots (49 steps, src/FHHFSolver.cpp:306-401).

FP64 paths: bit-identical states (np.array_equal); observables bit-identical on
the stream path, whose ensemble sums run in the oracle's order, and within 1e-13
on the resident path, which sums per CTA first.  FP32 paths:
within 1e-5 of the oracle (FP32 stages over 50 steps of h = 0.005; the
trajectories have not yet left their FP64 twins at t = 0.25).
"""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu

US = (2.0, 4.0, 8.0)
OBS_KEYS = ("niiu", "niid", "n2iiu", "n2iid", "nund")


def system(O, w):
    return O.System(tM=w.tM, U=w.U, V=w.V, ext=w.ext, coulomb=O.COUL_ONSITE, ext_null=False)


@pytest.fixture(scope="module", params=US, ids=lambda u: f"U{u:g}")
def ftwa_case(request, oracle_lib):
    O = oracle_lib
    w = configs.grid_10x10(U0=request.param, n_traj=8)
    rho0 = O.sample(w.n, 8, 50 + int(request.param), w.occ_up, w.occ_dn)
    ref = O.run(system(O, w), O.METHOD_FTWA, w.dt, 1, 50, rho0,
                obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
    return w, rho0, ref


@pytest.fixture(scope="module", params=US, ids=lambda u: f"U{u:g}")
def hf_case(request, oracle_lib):
    O = oracle_lib
    w = configs.grid_10x10(U0=request.param, n_traj=1)
    N0 = np.zeros((1, 2, w.n, w.n), dtype=complex)
    N0[0, 0] = np.diag(w.occ_up)
    N0[0, 1] = np.diag(w.occ_dn)
    ref = O.run(system(O, w), O.METHOD_HF, w.dt, 1, 50, N0,
                obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
    return w, N0, ref


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_cfg2_ftwa_fp64_bit_identical(engine, engine_lib, ftwa_case, path):
    E = engine_lib
    w, rho0, ref = ftwa_case
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 50, path=getattr(E, "PATH_" + path),
                   obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == getattr(E, "PATH_" + path)
    assert np.array_equal(engine.get_state(), ref["final"])
    tol = 0.0 if path == "STREAM" else 1e-13
    for k in OBS_KEYS:
        assert np.abs(getattr(r, k) - ref[k]).max() <= tol, k
    # energies: per-matrix partial sums on the GPU, one whole-matrix sum in the oracle
    assert np.abs(r.energies - ref["energies"]).max() < 1e-11 * max(1.0, np.abs(ref["energies"]).max())
    # the window moved the state (the comparison is not vacuous)
    assert np.abs(ref["final"] - rho0).max() > 1e-3


def test_cfg2_ftwa_fp32_resident(engine, engine_lib, ftwa_case):
    E = engine_lib
    w, rho0, ref = ftwa_case
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, 50, obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_RESIDENT
    for k in OBS_KEYS:
        assert np.abs(getattr(r, k) - ref[k]).max() < 1e-5, k
    assert np.abs(engine.get_state() - ref["final"]).max() < 1e-5


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_cfg2_hf_fp64_bit_identical(engine, engine_lib, hf_case, path):
    E = engine_lib
    w, N0, ref = hf_case
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(N0)
    r = engine.run(E.METHOD_HF, E.PREC_FP64, w.dt, 1, 50, path=getattr(E, "PATH_" + path),
                   obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == getattr(E, "PATH_" + path)
    assert np.array_equal(engine.get_state(), ref["final"])
    for k in OBS_KEYS:     # one trajectory: every reduction order gives the same sums
        assert np.array_equal(getattr(r, k), ref[k]), k
    assert np.abs(r.energies - ref["energies"]).max() < 1e-11 * max(1.0, np.abs(ref["energies"]).max())
    assert np.abs(ref["final"] - N0).max() > 1e-3
    # HF keeps each spin's particle number (trace) exactly up to rounding
    tr = np.einsum("bsii->bs", engine.get_state()).real
    assert np.abs(tr - np.array([[w.occ_up.sum(), w.occ_dn.sum()]])).max() < 1e-10


def test_cfg2_hf_fp32_resident(engine, engine_lib, hf_case):
    E = engine_lib
    w, N0, ref = hf_case
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(N0)
    r = engine.run(E.METHOD_HF, E.PREC_FP32, w.dt, 1, 50, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_RESIDENT
    for k in ("niiu", "niid", "nund"):
        assert np.abs(getattr(r, k) - ref[k]).max() < 1e-5, k


def test_cfg2_fp32_compensated_update_beats_plain(engine_lib):
    """The FP32 resident path keeps each state element as FP32 plus the bf16
    residual of its last update.  Against the FP64 path (bit-identical to the
    oracle) over 400 steps of the U = 4 system, its state error must be well below
    that of the same path with plain FP32 updates (FPSG_FLAG_FP32_PLAIN_STATE), and
    its observables closer too."""
    E = engine_lib
    w = configs.grid_10x10(U0=4.0, n_traj=16)
    Tp = 400
    res, states = {}, {}
    for name, prec, flags in (("fp64", E.PREC_FP64, 0), ("comp", E.PREC_FP32, 0),
                              ("plain", E.PREC_FP32, E.FLAG_FP32_PLAIN_STATE)):
        eng = E.Engine(0, flags=flags)
        try:
            eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
            eng.sample(16, 808, w.occ_up, w.occ_dn)
            res[name] = eng.run(E.METHOD_FTWA, prec, w.dt, 1, Tp, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
            states[name] = eng.get_state()
        finally:
            eng.close()
    assert res["comp"].path_used == E.PATH_RESIDENT and res["plain"].path_used == E.PATH_RESIDENT
    e_comp = np.abs(states["comp"] - states["fp64"]).max()
    e_plain = np.abs(states["plain"] - states["fp64"]).max()
    assert e_comp < e_plain / 4, (e_comp, e_plain)
    o_comp = max(np.abs(res["comp"].niiu - res["fp64"].niiu).max(), np.abs(res["comp"].nund - res["fp64"].nund).max())
    o_plain = max(np.abs(res["plain"].niiu - res["fp64"].niiu).max(), np.abs(res["plain"].nund - res["fp64"].nund).max())
    assert o_comp < o_plain, (o_comp, o_plain)


def test_cfg2_ftwa_fp64_long_window_bit_identical(engine, engine_lib, oracle_lib):
    """200 RK steps of 32 trajectories of the U = 4 system on the resident FP64
    path, bit-identical to the oracle: every RK stage's divisions by 3 (computed as a
    correctly rounded multiply-and-correct) and scalings by 1/8 must round exactly as
    the oracle's divisions do, over about 2.6e8 of them."""
    E, O = engine_lib, oracle_lib
    w = configs.grid_10x10(U0=4.0, n_traj=32)
    rho0 = O.sample(w.n, 32, 77, w.occ_up, w.occ_dn)
    ref = O.run(system(O, w), O.METHOD_FTWA, w.dt, 1, 200, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 200, path=E.PATH_RESIDENT, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_RESIDENT
    assert np.array_equal(engine.get_state(), ref["final"])
    assert np.abs(ref["final"] - rho0).max() > 1e-2
