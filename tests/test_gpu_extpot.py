"""A static potential with off-diagonal entries (a real symmetric tridiagonal
extPot), which the reference adds to Delta as a whole matrix
(src/FHfTWASolver.cpp:586-596) and whose energy row `pe` it sums over every
element (src/FHfTWASolver.cpp:401-411).  Every path must carry the off-diagonal
part into the commutator and keep it out of the hopping energy `tH`:

* FP64 stream and resident paths: bit-identical to the FP64 oracle;
* FP32 resident path: within 1e-5 of the oracle after a few steps;
* dense tensor-core path (split BF16x3 and TF32x3): within 2e-5 of the state's
  scale, as in the other dense tests;
* fpsg_grad, whose tM-scale identity needs Delta = tM off the diagonal, refuses
  the system with FPSG_ERR_UNSUPPORTED instead of returning a wrong gradient.
"""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu


def tridiag_potential(n, seed):
    rng = np.random.default_rng(seed)
    ext = np.diag(rng.uniform(-1.0, 1.0, n))
    off = rng.uniform(-0.4, 0.4, n - 1)
    ext += np.diag(off, 1) + np.diag(off, -1)
    return ext


@pytest.fixture(scope="module")
def case():
    w = configs.grid(6, 5, U0=3.0, seed=4, n_traj=3)
    return w, tridiag_potential(w.n, 11)


def oracle_ref(O, w, ext, method, dt, S, Tp, rho0, obs):
    sysm = O.System(tM=w.tM, U=w.U, V=w.V, ext=ext, coulomb=O.COUL_ONSITE, ext_null=False)
    return O.run(sysm, method, dt, S, Tp, rho0, obs=obs)


def rel_state_err(a, b):
    return np.abs(a - b).max() / max(1e-30, np.abs(b).max())


def test_offdiag_potential_fp64_paths_bit_exact(engine, engine_lib, oracle_lib, case):
    E, O = engine_lib, oracle_lib
    w, ext = case
    rho0 = O.sample(w.n, 3, 2, w.occ_up, w.occ_dn)
    obs_o = O.OBS_DIAG | O.OBS_DOUB | O.OBS_ENER
    ref = oracle_ref(O, w, ext, O.METHOD_FTWA, 0.01, 2, 6, rho0, obs_o)
    # the off-diagonal part moves the dynamics: without it the state differs
    plain = O.run(O.System(tM=w.tM, U=w.U, V=w.V, ext=np.diag(np.diag(ext)), coulomb=O.COUL_ONSITE,
                           ext_null=False), O.METHOD_FTWA, 0.01, 2, 6, rho0, obs=O.OBS_DIAG)
    assert rel_state_err(plain["final"], ref["final"]) > 1e-4
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    for path in (E.PATH_STREAM, E.PATH_RESIDENT):
        engine.set_initial_samples(rho0)
        r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.01, 2, 6, path=path,
                       obs=E.OBS_DIAG | E.OBS_DOUBLONS | E.OBS_ENERGIES)
        assert r.path_used == path
        assert np.array_equal(engine.get_state(), ref["final"]), path
        # the stream path sums trajectories in the oracle's order; the resident path
        # sums per CTA first (a fixed order of its own, equal to rounding)
        tol = 0.0 if path == E.PATH_STREAM else 1e-13
        assert np.abs(r.niiu - ref["niiu"]).max() <= tol and np.abs(r.nund - ref["nund"]).max() <= tol, path
        # energies: the GPU sums per matrix and column, the oracle over the whole matrix
        assert np.abs(r.energies - ref["energies"]).max() < 1e-12 * max(1.0, np.abs(ref["energies"]).max()), path


def test_offdiag_potential_energy_rows_apart(engine, engine_lib, oracle_lib, case):
    """fTWA energies are written for core-hole systems only; the computed rows are
    compared here directly: tH must not contain the potential's off-diagonal part."""
    E, O = engine_lib, oracle_lib
    w, ext = case
    N0 = np.zeros((1, 2, w.n, w.n), dtype=complex)
    _, R = np.linalg.eigh(w.tM + ext)
    N0[0, 0] = R[:, :15] @ R[:, :15].T
    N0[0, 1] = R[:, :14] @ R[:, :14].T
    ref = oracle_ref(O, w, ext, O.METHOD_HF, 0.01, 1, 3, N0, O.OBS_DIAG | O.OBS_ENER)
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    for path in (E.PATH_STREAM, E.PATH_RESIDENT):
        engine.set_initial_samples(N0)
        r = engine.run(E.METHOD_HF, E.PREC_FP64, 0.01, 1, 3, path=path, obs=E.OBS_DIAG | E.OBS_ENERGIES)
        scale = max(1.0, np.abs(ref["energies"]).max())
        assert np.abs(r.energies - ref["energies"]).max() < 1e-12 * scale, path
        # the potential row carries the off-diagonal part (it differs from the diagonal-only sum)
        diag_only = np.einsum("ii,sii->", ext, N0[0]).real
        assert abs(ref["energies"][3, 0] - diag_only) > 1e-3


def test_offdiag_potential_fp32_resident(engine, engine_lib, oracle_lib, case):
    E, O = engine_lib, oracle_lib
    w, ext = case
    rho0 = O.sample(w.n, 3, 5, w.occ_up, w.occ_dn)
    ref = oracle_ref(O, w, ext, O.METHOD_FTWA, 0.01, 2, 6, rho0, O.OBS_DIAG)
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 2, 6, obs=E.OBS_DIAG)
    assert r.path_used == E.PATH_RESIDENT
    assert rel_state_err(engine.get_state(), ref["final"]) < 1e-5
    assert np.abs(r.niiu - ref["niiu"]).max() < 1e-5


@pytest.mark.parametrize("prec_name", ["bf16x3", "tf32x3"])
def test_offdiag_potential_dense_path(engine, engine_lib, oracle_lib, case, prec_name):
    E, O = engine_lib, oracle_lib
    prec = {"bf16x3": E.PREC_SPLIT_BF16X3, "tf32x3": E.PREC_SPLIT_TF32X3}[prec_name]
    w, ext = case
    rho0 = O.sample(w.n, 3, 7, w.occ_up, w.occ_dn)
    ref = oracle_ref(O, w, ext, O.METHOD_FTWA, 0.01, 2, 4, rho0, O.OBS_DIAG | O.OBS_DOUB)
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, prec, 0.01, 2, 4, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_DENSE
    assert rel_state_err(engine.get_state(), ref["final"]) < 2e-5
    assert np.abs(r.niiu - ref["niiu"]).max() < 2e-5
    assert np.abs(r.nund - ref["nund"]).max() < 2e-5


def test_offdiag_potential_grad_refused(engine, engine_lib, case):
    E = engine_lib
    w, ext = case
    engine.set_system(w.tM, w.U, w.V, ext, coulomb=E.COUL_ONSITE)
    engine.sample(2, 1, w.occ_up, w.occ_dn)
    with pytest.raises(E.FpsgError) as ei:
        engine.grad(E.PREC_FP64, 0.01, 1, 3, 2)
    assert ei.value.code == E.ERR_UNSUPPORTED
    # a diagonal potential is still served
    engine.set_system(w.tM, w.U, w.V, np.diag(np.diag(ext)), coulomb=E.COUL_ONSITE)
    engine.sample(2, 1, w.occ_up, w.occ_dn)
    g = engine.grad(E.PREC_FP64, 0.01, 1, 3, 2)
    assert np.isfinite(g["loss"])
