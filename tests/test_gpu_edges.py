"""Edge cases of the CUDA paths against the FP64 oracle: a single site, one
trajectory, a single snapshot, trajectory counts that leave the last resident
group or cluster partly empty, long snapshot intervals, and the size and argument
limits each path reports as errors.  Per-trajectory states are compared bit for
bit; ensemble observables to 1e-12 (the oracle sums its trajectories per thread,
the GPU in fixed 64-trajectory chunks, so the last bits of a mean can differ)."""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu

OBS = 1 | 2 | 4 | 16


def osys(O, tM, U, V, coul=None):
    return O.System(tM=tM, U=U, V=V, coulomb=O.COUL_ONSITE if coul is None else coul, ext_null=True)


@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_single_site(engine, engine_lib, oracle_lib, path):
    """n = 1: Delta is a number, the commutator vanishes, rho stays constant."""
    E, O = engine_lib, oracle_lib
    tM, U, V = np.array([[0.3]]), np.array([[4.0]]), np.zeros((1, 1))
    rho0 = O.sample(1, 3, 2, np.array([1.0]), np.array([0.0]))
    ref = O.run(osys(O, tM, U, V), O.METHOD_FTWA, 0.01, 2, 5, rho0, obs=O.OBS_DIAG | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(tM, U, V, None, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.01, 2, 5, obs=E.OBS_DIAG | E.OBS_DOUBLONS,
                   path=getattr(E, "PATH_" + path))
    assert np.array_equal(r.niiu, ref["niiu"]) and np.array_equal(r.nund, ref["nund"])
    assert np.array_equal(engine.get_state(), rho0)


@pytest.mark.parametrize("B", [1, 37])
@pytest.mark.parametrize("path", ["STREAM", "RESIDENT"])
def test_odd_trajectory_counts_bit_exact(engine, engine_lib, oracle_lib, B, path):
    """One trajectory, and a count that leaves the last group of the resident path
    partly empty: every trajectory still matches the oracle bit for bit."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(4, 3, U0=3.0, seed=5, n_traj=B)
    rho0 = O.sample(w.n, B, 8, w.occ_up, w.occ_dn)
    ref = O.run(osys(O, w.tM, w.U, w.V), O.METHOD_FTWA, 0.02, 3, 4, rho0,
                obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.02, 3, 4, obs=OBS, path=getattr(E, "PATH_" + path))
    assert r.path_used == getattr(E, "PATH_" + path)
    assert np.array_equal(engine.get_state(), ref["final"])
    for k in ("niiu", "niid", "n2iiu", "nund"):
        assert np.abs(getattr(r, k) - ref[k]).max() < 1e-12, k


def test_one_snapshot_and_long_intervals(engine, engine_lib, oracle_lib):
    """n_snapshots = 1 records t = 0 and (fTWA) still integrates S steps after it;
    a long interval (S = 50) between two snapshots."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(3, 3, U0=4.0, seed=1, n_traj=4)
    rho0 = O.sample(w.n, 4, 4, w.occ_up, w.occ_dn)
    for S, Tp in ((7, 1), (50, 2)):
        ref = O.run(osys(O, w.tM, w.U, w.V), O.METHOD_FTWA, 0.05, S, Tp, rho0, obs=O.OBS_DIAG)
        engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        engine.set_initial_samples(rho0)
        r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.05, S, Tp, obs=E.OBS_DIAG)
        assert r.niiu.shape == (w.n, Tp)
        assert np.array_equal(engine.get_state(), ref["final"])
        assert np.abs(r.niiu - ref["niiu"]).max() < 1e-12
        assert r.traj_steps == 4 * Tp * S


def test_limits_are_reported(engine, engine_lib):
    E = engine_lib
    # the dense path handles n <= 256
    n = 260
    tM = np.zeros((n, n))
    tM[np.arange(n - 1), np.arange(1, n)] = -1.0
    tM = tM + tM.T
    engine.set_system(tM, np.eye(n) * 2.0, np.zeros((n, n)), None, coulomb=E.COUL_ONSITE)
    engine.sample(2, 1, np.ones(n) * (np.arange(n) % 2), np.ones(n) * ((np.arange(n) + 1) % 2))
    with pytest.raises(E.FpsgError) as ei:
        engine.advance(E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 1, 1)
    assert ei.value.code == E.ERR_UNSUPPORTED
    # the resident path does not fit this n: asking for it is an error, auto falls back
    with pytest.raises(E.FpsgError) as ei:
        engine.advance(E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, 1, path=E.PATH_RESIDENT)
    assert ei.value.code == E.ERR_UNSUPPORTED
    r = engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, 2, obs=E.OBS_DIAG)
    assert r.path_used == E.PATH_STREAM and np.all(np.isfinite(r.niiu))
    # argument errors
    with pytest.raises(E.FpsgError) as ei:
        engine.sample(0, 1, np.zeros(n), np.zeros(n))
    assert ei.value.code == E.ERR_INVALID
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 0, 2)
    assert ei.value.code == E.ERR_INVALID
    with pytest.raises(E.FpsgError) as ei:
        engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, 0)
    assert ei.value.code == E.ERR_INVALID


def test_scratch_reuse_across_calls(engine, engine_lib, oracle_lib):
    """Per-call scratch stays pooled in the context: calls of other paths,
    precisions and sizes in the same context take each other's buffers back,
    and each call still matches the oracle (FP64) or repeats itself (FP32)."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(4, 3, U0=3.0, seed=2, n_traj=37)
    rho0 = O.sample(w.n, 37, 9, w.occ_up, w.occ_dn)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    f32 = []
    for Tp, path in ((4, "STREAM"), (6, "RESIDENT"), (3, "STREAM"), (6, "RESIDENT")):
        ref = O.run(osys(O, w.tM, w.U, w.V), O.METHOD_FTWA, 0.02, 2, Tp, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
        engine.set_initial_samples(rho0)
        r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.02, 2, Tp, obs=E.OBS_DIAG | E.OBS_DOUBLONS,
                       path=getattr(E, "PATH_" + path))
        assert np.array_equal(engine.get_state(), ref["final"]), (Tp, path)
        assert np.abs(r.niiu - ref["niiu"]).max() < 1e-12
        engine.set_initial_samples(rho0)
        f32.append(engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.02, 2, 6, obs=E.OBS_DIAG).niiu)
    assert all(np.array_equal(f32[0], x) for x in f32[1:])


def test_pooled_tables_across_systems(engine, engine_lib, oracle_lib):
    """fpsg_set_system hands its old tables back to the context's pool and takes
    blocks from it: switching between systems of different sizes in one context
    keeps every run on the oracle."""
    E, O = engine_lib, oracle_lib
    for nx, ny, seed in ((4, 3, 1), (6, 5, 2), (4, 3, 3), (2, 2, 4)):
        w = configs.grid(nx, ny, U0=3.5, seed=seed, n_traj=6)
        rho0 = O.sample(w.n, 6, seed, w.occ_up, w.occ_dn)
        ref = O.run(osys(O, w.tM, w.U, w.V), O.METHOD_FTWA, 0.02, 2, 4, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
        engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        engine.set_initial_samples(rho0)
        r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.02, 2, 4, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
        assert np.array_equal(engine.get_state(), ref["final"]), (nx, ny)
        assert np.abs(r.nund - ref["nund"]).max() < 1e-12
