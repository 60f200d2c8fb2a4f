"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

FP64 path: per-trajectory states must be bit-identical to the oracle (the kernels
follow the oracle's arithmetic contract), ensemble observables within 1e-12.
FP32 path: compared against the oracle with the tolerances written in each test
(FP32 stages, FP64 ensemble reduction).
"""
import math

import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu

OBS_KEYS = ("niiu", "niid", "n2iiu", "n2iid", "nund")


def oracle_system(O, w, coul=None, ext_null=None):
    return O.System(tM=w.tM, U=w.U, V=w.V, ext=w.ext,
                    coulomb=O.COUL_ONSITE if coul is None else coul,
                    ext_null=(w.ext is None) if ext_null is None else ext_null)


def set_engine_system(eng, E, w, coul=None):
    eng.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE if coul is None else coul)


def assert_obs_close(res, ref, atol, keys=OBS_KEYS):
    for k in keys:
        got = getattr(res, k)
        want = ref[k]
        err = np.abs(got - want).max()
        assert err <= atol, (k, err)


def test_sampler_matches_oracle(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    set_engine_system(engine, E, w)
    engine.sample(64, 7, w.occ_up, w.occ_dn)
    got = engine.get_state()
    want = O.sample(w.n, 64, 7, w.occ_up, w.occ_dn)
    # Box-Muller uses the device's log/sincos: a few ulp from the host libm
    assert np.abs(got - want).max() < 1e-14
    assert np.array_equal(got, np.conj(np.transpose(got, (0, 1, 3, 2))))
    d = np.real(np.diagonal(got, axis1=2, axis2=3))
    assert np.array_equal(d[:, 0], np.tile(w.occ_up - 0.5, (64, 1)))


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_fp64_grid3x2_bit_identical(engine, engine_lib, oracle_lib, path):
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    B, Tp = 24, 41
    rho0 = O.sample(w.n, B, 0, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, w.dt, w.S, Tp, rho0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, w.S, Tp, path=getattr(E, "PATH_" + path))
    assert res.path_used == getattr(E, "PATH_" + path)
    got = engine.get_state()
    assert np.array_equal(got, ref["final"]), np.abs(got - ref["final"]).max()
    assert_obs_close(res, ref, 1e-12)
    assert np.abs(res.energies - ref["energies"]).max() < 1e-12
    assert res.traj_steps == B * Tp * w.S


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_fp64_golden_fixture(engine, engine_lib, path):
    """Against the committed oracle golden file (tests/golden/grid3x2_ftwa.npz)."""
    import os
    E = engine_lib
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "grid3x2_ftwa.npz"))
    w = configs.grid_3x2()
    set_engine_system(engine, E, w)
    engine.set_initial_samples(g["rho0"])
    res = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, w.S, g["niiu"].shape[1], path=getattr(E, "PATH_" + path))
    assert np.array_equal(engine.get_state(), g["final"])
    for k in OBS_KEYS:
        assert np.abs(getattr(res, k) - g[k]).max() < 1e-12
    assert np.abs(res.energies - g["energies"]).max() < 1e-12


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_fp64_potential_and_random_state(engine, engine_lib, oracle_lib, path):
    E, O = engine_lib, oracle_lib
    w = configs.grid(4, 3, U0=6.0, seed=3)
    rng = np.random.default_rng(9)
    w.ext = np.diag(rng.uniform(-1, 1, w.n))
    B, Tp, S, dt = 10, 21, 3, 0.02
    rho0 = O.sample(w.n, B, 5, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, dt, S, Tp, rho0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP64, dt, S, Tp, path=getattr(E, "PATH_" + path))
    assert np.array_equal(engine.get_state(), ref["final"])
    assert_obs_close(res, ref, 1e-12)
    assert np.abs(res.energies - ref["energies"]).max() < 1e-12


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_fp64_distance_coulomb_and_pulse(engine, engine_lib, oracle_lib, path):
    E, O = engine_lib, oracle_lib
    pos = configs.grid_positions(3, 3)
    D = configs.distances(pos)
    T = configs.hopping(D, [(1.0, -1.0), (math.sqrt(2.0), -0.25)])
    U = 2.0 / (1.0 + D)
    V = np.where(np.eye(9, dtype=bool), 0.0, 2.0 / (1.0 + D))
    occ_u = np.array([1.0, 0, 1, 0, 1, 0, 1, 0, 1])
    occ_d = 1.0 - occ_u
    pulse = {"n_bins": 7, "amp": np.array([0.3, -0.2, 0.5, 0.1, -0.4, 0.2, 0.0]), "bin_width": 0.05,
             "t0": 0.15, "td": 0.1, "proj": pos[:, 0] - 1.0}
    sysm = O.System(tM=T, U=U, V=V, coulomb=O.COUL_DISTANCE, ext_null=True, pulse=pulse)
    B, Tp, S, dt = 6, 31, 2, 0.01
    rho0 = O.sample(9, B, 13, occ_u, occ_d)
    ref = O.run(sysm, O.METHOD_FTWA, dt, S, Tp, rho0)
    engine.set_system(T, U, V, None, coulomb=E.COUL_DISTANCE)
    engine.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP64, dt, S, Tp, path=getattr(E, "PATH_" + path))
    assert np.array_equal(engine.get_state(), ref["final"])
    assert_obs_close(res, ref, 1e-12)
    assert np.abs(res.energies - ref["energies"]).max() < 1e-12


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_hf_onsite_bit_identical(engine, engine_lib, oracle_lib, path):
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    rng = np.random.default_rng(0)
    N0 = np.zeros((1, 2, 6, 6), dtype=complex)
    N0[0, 0] = np.diag(w.occ_up)
    N0[0, 1] = np.diag(w.occ_dn)
    for s in range(2):
        X = 0.05 * (rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)))
        N0[0, s] += X + X.conj().T
    Tp = 51
    ref = O.run(oracle_system(O, w), O.METHOD_HF, w.dt, w.S, Tp, N0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(N0)
    res = engine.run(E.METHOD_HF, E.PREC_FP64, w.dt, w.S, Tp, path=getattr(E, "PATH_" + path))
    assert np.array_equal(engine.get_state(), ref["final"])
    assert_obs_close(res, ref, 1e-12)
    assert np.abs(res.energies - ref["energies"]).max() < 1e-12
    assert res.traj_steps == (Tp - 1) * w.S


def test_fp64_split_cluster_kernel_8x8(engine, engine_lib, oracle_lib):
    """n = 64 in FP64 does not fit one CTA: the resident path runs one spin per CTA
    in a 2-CTA cluster (diagonals through distributed shared memory)."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(8, 8, U0=4.0, seed=1)
    B, Tp, S, dt = 3, 4, 2, 0.01
    rho0 = O.sample(w.n, B, 2, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, dt, S, Tp, rho0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP64, dt, S, Tp, path=E.PATH_RESIDENT)
    assert np.array_equal(engine.get_state(), ref["final"])
    assert_obs_close(res, ref, 1e-12)


def test_whole_density_matrix(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    B, Tp = 8, 11
    rho0 = O.sample(w.n, B, 4, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, w.dt, w.S, Tp, rho0, obs=O.OBS_DIAG | O.OBS_WHOLE)
    for path in (E.PATH_STREAM, E.PATH_RESIDENT):
        set_engine_system(engine, E, w)
        engine.set_initial_samples(rho0)
        res = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, w.S, Tp, obs=E.OBS_DIAG | E.OBS_WHOLE, path=path)
        assert np.abs(res.whole_u - ref["whole_u"]).max() < 1e-12
        assert np.abs(res.whole_d - ref["whole_d"]).max() < 1e-12


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_fp32_short_run_close_to_fp64(engine, engine_lib, oracle_lib, path):
    """FP32 stages: within 2e-5 of the FP64 oracle over 50 RK steps on the 3x2 grid."""
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    B, Tp = 64, 6
    rho0 = O.sample(w.n, B, 1, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, w.dt, w.S, Tp, rho0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, w.S, Tp, path=getattr(E, "PATH_" + path))
    assert_obs_close(res, ref, 2e-5)
    assert np.abs(engine.get_state() - ref["final"]).max() < 1e-4


def test_fp32_split_cluster_10x10(engine, engine_lib, oracle_lib):
    """The 10x10 domain-wall system on the FP32 resident path (2-CTA clusters)."""
    E, O = engine_lib, oracle_lib
    w = configs.grid_10x10(U0=4.0, n_traj=4)
    B, Tp, S = 4, 5, 2
    rho0 = O.sample(w.n, B, 3, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, w.dt, S, Tp, rho0)
    set_engine_system(engine, E, w)
    engine.set_initial_samples(rho0)
    res = engine.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, S, Tp, path=E.PATH_RESIDENT)
    assert res.path_used == E.PATH_RESIDENT
    assert_obs_close(res, ref, 2e-5)
    assert np.abs(engine.get_state() - ref["final"]).max() < 1e-4
    # and the FP64 stream path on the same input is bit-identical
    engine.set_initial_samples(rho0)
    engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, S, Tp, path=E.PATH_STREAM)
    assert np.array_equal(engine.get_state(), ref["final"])


def test_advance_matches_run(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w = configs.grid_3x2()
    rho0 = O.sample(w.n, 16, 6, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, w.dt, 1, 30, rho0)
    for path in (E.PATH_STREAM, E.PATH_RESIDENT):
        set_engine_system(engine, E, w)
        engine.set_initial_samples(rho0)
        ms, launches = engine.advance(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 30, path=path)
        assert launches >= 1 and ms > 0
        assert np.array_equal(engine.get_state(), ref["final"])


def test_errors_are_reported(engine, engine_lib):
    E = engine_lib
    w = configs.grid_3x2()
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.01, 1, 2)
    assert ei.value.code == E.ERR_STATE
    with pytest.raises(E.FpsgError) as ei:
        engine.set_system(w.tM + 1j * np.eye(6), w.U)
    assert ei.value.code == E.ERR_UNSUPPORTED
    set_engine_system(engine, E, w)
    bad = np.zeros((1, 2, 6, 6), dtype=complex)
    bad[0, 0, 0, 1] = np.nan
    with pytest.raises(E.FpsgError) as ei:
        engine.set_initial_samples(bad)
    assert ei.value.code == E.ERR_INVALID
    engine.sample(4, 1, w.occ_up, w.occ_dn)
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP64, -0.01, 1, 2)
    assert ei.value.code == E.ERR_INVALID
    engine.set_system(w.tM, w.U, w.V, coulomb=E.COUL_DISTANCE)
    engine.sample(4, 1, w.occ_up, w.occ_dn)
    with pytest.raises(E.FpsgError) as ei:        # the Fock term has no tensor-core form here
        engine.run(E.METHOD_HF, E.PREC_SPLIT_BF16X3, 0.01, 1, 2)
    assert ei.value.code == E.ERR_UNSUPPORTED
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_HF, E.PREC_FP64, 0.01, 1, 2, path=E.PATH_RESIDENT)
    assert ei.value.code == E.ERR_UNSUPPORTED


def test_memory_cap_gives_oom(engine, engine_lib):
    E = engine_lib
    w = configs.grid_3x2()
    set_engine_system(engine, E, w)
    engine.set_memory_cap(1)
    with pytest.raises(E.FpsgError) as ei:
        engine.sample(1000, 0, w.occ_up, w.occ_dn)
    assert ei.value.code == E.ERR_OOM
    engine.set_memory_cap(0)
    engine.sample(1000, 0, w.occ_up, w.occ_dn)


def test_divergence_is_detected(engine, engine_lib):
    """A step far beyond stability drives the state to inf/nan: the record pass
    flags it and the call returns FPSG_ERR_DIVERGED instead of garbage."""
    E = engine_lib
    w = configs.grid_3x2()
    engine.set_system(w.tM * 1e3, w.U * 1e3, w.V)
    engine.sample(8, 0, w.occ_up, w.occ_dn)
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP32, 10.0, 20, 40)
    assert ei.value.code == E.ERR_DIVERGED


@pytest.mark.parametrize("sizes", [(3, 2), (6, 5)])
def test_hf_fock_term_bit_exact(engine, engine_lib, oracle_lib, sizes):
    """HF with distance Coulomb: Delta = tM + diag(U n_other + V n_same) - N o V
    (src/FHHFSolver.cpp:583-590), dense and complex, with a static potential and
    a pulse; exchange energy -sum V |N|^2 / 2 (:271-272)."""
    E, O = engine_lib, oracle_lib
    nx, ny = sizes
    pos = configs.grid_positions(nx, ny)
    D = configs.distances(pos)
    n = nx * ny
    T = configs.hopping(D, [(1.0, -1.0)])
    U = 2.0 / (1.0 + D)
    V = 2.0 / (1.0 + D)
    np.fill_diagonal(V, 0.0)
    rng = np.random.default_rng(3)
    ext = np.diag(rng.uniform(-1, 1, n))
    pulse = {"n_bins": 3, "amp": rng.normal(0, 0.5, 3), "bin_width": 0.02, "t0": 0.03, "td": 0.02,
             "proj": pos[:, 0] - pos[:, 0].mean()}
    _, R = np.linalg.eigh(T)
    N0 = np.zeros((1, 2, n, n), dtype=complex)
    N0[0, 0] = R[:, : (n + 1) // 2] @ R[:, : (n + 1) // 2].T
    N0[0, 1] = R[:, : n // 2] @ R[:, : n // 2].T
    sysm = O.System(tM=T, U=U, V=V, ext=ext, coulomb=O.COUL_DISTANCE, ext_null=False, pulse=pulse)
    ref = O.run(sysm, O.METHOD_HF, 0.01, 3, 6, N0, obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(T, U, V, ext, coulomb=E.COUL_DISTANCE)
    engine.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    engine.set_initial_samples(N0)
    r = engine.run(E.METHOD_HF, E.PREC_FP64, 0.01, 3, 6, obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == E.PATH_STREAM
    assert np.array_equal(engine.get_state(), ref["final"])
    for k in ("niiu", "niid", "n2iiu", "nund"):
        assert np.array_equal(getattr(r, k), ref[k]), k
    assert np.abs(r.energies - ref["energies"]).max() < 1e-12 * max(1.0, np.abs(ref["energies"]).max())
    # the exchange term is present: V row of the energies differs from the Hartree-only value
    assert np.abs(ref["energies"][2]).max() > 0
