"""The dense tensor-core path (split BF16x3, tcgen05) and the global-memory stream
path for matrices too large for shared memory, on the moire lattice (n = 256,
distance-decaying hopping, long-range Coulomb), checked against the FP64 oracle
on the same injected samples.

Tolerances: the split product keeps ~16 significant bits per operand and drops
lo*lo (relative error ~2^-16 of each commutator entry); over a few RK steps of
h = 0.005 the state error stays below 1e-5 of its scale.  The FP64 global-memory
stream path is bit-identical to the oracle."""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def moire():
    return configs.moire_8x8(U0=1.0, n_traj=4)


def oracle_system(O, w, coul, pulse=None):
    return O.System(tM=w.tM, U=w.U, V=w.V, ext=w.ext, coulomb=coul, ext_null=w.ext is None, pulse=pulse)


def rel_state_err(a, b):
    return np.abs(a - b).max() / max(1e-30, np.abs(b).max())


def test_moire_fp64_global_stream_bit_exact(engine, engine_lib, oracle_lib, moire):
    E, O = engine_lib, oracle_lib
    w = moire
    rho0 = O.sample(w.n, 2, 3, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w, O.COUL_DISTANCE), O.METHOD_FTWA, w.dt, 1, 3, rho0,
                obs=O.OBS_DIAG | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_DISTANCE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 3, obs=E.OBS_DIAG | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == E.PATH_STREAM
    assert np.array_equal(r.niiu, ref["niiu"]) and np.array_equal(r.nund, ref["nund"])
    assert np.array_equal(engine.get_state(), ref["final"])


def test_moire_dense_bf16x3_close_to_fp64(engine, engine_lib, oracle_lib, moire):
    E, O = engine_lib, oracle_lib
    w = moire
    rho0 = O.sample(w.n, 4, 5, w.occ_up, w.occ_dn)
    Tp = 4
    ref = O.run(oracle_system(O, w, O.COUL_DISTANCE), O.METHOD_FTWA, w.dt, 1, Tp, rho0,
                obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_DISTANCE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, w.dt, 1, Tp,
                   obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == E.PATH_DENSE
    got = engine.get_state()
    err = rel_state_err(got, ref["final"])
    assert err < 2e-5, err
    # the step actually moved the state (the check is not vacuous)
    assert rel_state_err(ref["final"], rho0) > 1e-3
    for k in ("niiu", "niid", "nund", "n2iiu"):
        assert np.abs(r.__dict__[k] - ref[k]).max() < 2e-5, k
    assert np.abs(r.energies - ref["energies"]).max() < 1e-3 * max(1.0, np.abs(ref["energies"]).max())
    # Hermiticity: the imaginary diagonal stays zero
    d = np.einsum("bsii->bsi", got)
    assert np.abs(d.imag).max() == 0.0


def test_dense_padded_small_lattice_with_pulse_and_potential(engine, engine_lib, oracle_lib):
    """n = 30 < 256 exercises the zero padding; pulse and static potential enter Delta's diagonal."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(6, 5, U0=3.0, seed=4, n_traj=3)
    rng = np.random.default_rng(1)
    ext = np.diag(rng.uniform(-1, 1, w.n))
    pos = configs.grid_positions(6, 5)
    pulse = {"n_bins": 4, "amp": rng.normal(0, 0.5, 4), "bin_width": 0.01, "t0": 0.02, "td": 0.02,
             "proj": pos[:, 0] - pos[:, 0].mean()}
    rho0 = O.sample(w.n, 3, 2, w.occ_up, w.occ_dn)
    sysm = O.System(tM=w.tM, U=w.U, V=w.V, ext=ext, coulomb=O.COUL_ONSITE, ext_null=False, pulse=pulse)
    ref = O.run(sysm, O.METHOD_FTWA, 0.01, 2, 4, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    engine.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 2, 4, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_DENSE
    assert rel_state_err(engine.get_state(), ref["final"]) < 2e-5
    assert np.abs(r.niiu - ref["niiu"]).max() < 2e-5


def test_dense_hf_matches_oracle(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w = configs.grid(6, 6, U0=4.0, seed=7, n_traj=1)
    N0 = np.zeros((1, 2, w.n, w.n), dtype=complex)
    N0[0, 0] = np.diag(w.occ_up)
    N0[0, 1] = np.diag(w.occ_dn)
    # a non-diagonal start so the hopping acts at once
    _, R = np.linalg.eigh(w.tM)
    N0[0, 0] = R[:, :18] @ R[:, :18].T
    ref = O.run(O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True), O.METHOD_HF,
                0.01, 3, 5, N0, obs=O.OBS_DIAG | O.OBS_DOUB)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(N0)
    r = engine.run(E.METHOD_HF, E.PREC_SPLIT_BF16X3, 0.01, 3, 5, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert np.abs(r.niiu - ref["niiu"]).max() < 2e-5
    assert rel_state_err(engine.get_state(), ref["final"]) < 2e-5


def test_dense_rejects_other_precisions_and_large_n(engine, engine_lib):
    E = engine_lib
    w = configs.grid(4, 4, n_traj=2)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.sample(2, 1, w.occ_up, w.occ_dn)
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, 2, path=E.PATH_DENSE)
    assert ei.value.code == E.ERR_INVALID
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 1, 2, path=E.PATH_STREAM)
    assert ei.value.code == E.ERR_INVALID


def test_moire_fp32_global_stream_close_to_fp64(engine, engine_lib, oracle_lib, moire):
    E, O = engine_lib, oracle_lib
    w = moire
    rho0 = O.sample(w.n, 2, 9, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w, O.COUL_DISTANCE), O.METHOD_FTWA, w.dt, 1, 3, rho0, obs=O.OBS_DIAG)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_DISTANCE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP32, w.dt, 1, 3, obs=E.OBS_DIAG)
    assert r.path_used == E.PATH_STREAM
    assert rel_state_err(engine.get_state(), ref["final"]) < 1e-6


def test_moire_dense_tf32x3_and_bf16x3_vs_fp64(engine, engine_lib, moire):
    """Split TF32x3 (kind::tf32, ~21 significant bits per operand) and split BF16x3
    against the FP64 GPU path (bit-identical to the oracle at this n) over 50 steps
    on the same samples.  Both stay within 2e-6 of the state's scale: at this
    system the FP32 rounding of the long-range Hartree diagonal (~50) and of the
    FP32 state dominates the error of either split."""
    E = engine_lib
    w = moire
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_DISTANCE)
    Tp = 51
    states, niiu = {}, {}
    for name, prec in (("fp64", E.PREC_FP64), ("tf32", E.PREC_SPLIT_TF32X3), ("bf16", E.PREC_SPLIT_BF16X3)):
        engine.sample(8, 13, w.occ_up, w.occ_dn)
        r = engine.run(E.METHOD_FTWA, prec, w.dt, 1, Tp, obs=E.OBS_DIAG)
        if name != "fp64":
            assert r.path_used == E.PATH_DENSE
        states[name], niiu[name] = engine.get_state(), r.niiu
    errs = {k: rel_state_err(states[k], states["fp64"]) for k in ("tf32", "bf16")}
    assert errs["tf32"] < 2e-6 and errs["bf16"] < 2e-6, errs
    assert np.abs(niiu["tf32"] - niiu["fp64"]).max() < 2e-6


def test_dense_bounded_wait_reports_timeout(engine_lib, oracle_lib):
    """A device-side wait that runs out is reported, not hung: a context made with
    FPSG_FLAG_TEST_EXPIRE_WAIT has the first stage launch of each dense call wait on
    a barrier nothing arrives at (before it holds tensor memory or issues a copy).
    The call returns FPSG_ERR_TIMEOUT, and the device stays usable: the same context
    (without the hook, a fresh one) then integrates correctly."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(6, 5, U0=3.0, seed=4, n_traj=2)
    rho0 = O.sample(w.n, 2, 2, w.occ_up, w.occ_dn)
    eng = E.Engine(0, flags=E.FLAG_TEST_EXPIRE_WAIT)
    try:
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        eng.set_initial_samples(rho0)
        with pytest.raises(E.FpsgError) as ei:
            eng.run(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 1, 3, obs=E.OBS_DIAG)
        assert ei.value.code == E.ERR_TIMEOUT
        # the hook touches only the dense path: the FP64 path of the same context still runs
        eng.set_initial_samples(rho0)
        eng.run(E.METHOD_FTWA, E.PREC_FP64, 0.01, 1, 3, obs=E.OBS_DIAG)
    finally:
        eng.close()
    ref = O.run(O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True), O.METHOD_FTWA,
                0.01, 1, 3, rho0, obs=O.OBS_DIAG)
    eng = E.Engine(0)
    try:
        eng.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        eng.set_initial_samples(rho0)
        r = eng.run(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 1, 3, obs=E.OBS_DIAG)
        assert r.path_used == E.PATH_DENSE
        assert rel_state_err(eng.get_state(), ref["final"]) < 2e-5
    finally:
        eng.close()
    with pytest.raises(E.FpsgError):
        E.Engine(0, flags=1 << 40)       # unknown flags are refused
