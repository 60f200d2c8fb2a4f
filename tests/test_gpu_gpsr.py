"""GPSR drift (fpsg_gpsr_drift): the 3/8-rule RK4 drift increment of FHGPSRSolver
(src/FHGPSRSolver.cpp:168-206) for general complex (non-Hermitian) states, against
the oracle's restatement, bit for bit; the diagonal of Delta is complex here
(Delta_up = tM + diagmat(U diag(rho_dn)) + extPot, src/FHGPSRSolver.cpp:111-134).
"""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu


def random_states(n, B, seed, scale=0.3):
    rng = np.random.default_rng(seed)
    rho = scale * (rng.normal(size=(B, 2, n, n)) + 1j * rng.normal(size=(B, 2, n, n)))
    for b in range(B):
        for s in range(2):
            rho[b, s] += np.diag(rng.uniform(0.0, 1.0, n) + 1j * rng.normal(0.0, 0.1, n))
    return rho


def distance_U(pos, U0):
    r = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=-1)
    return U0 / (1.0 + r)


@pytest.mark.parametrize("case", ["grid3x3_onsite", "grid6x5_ext", "grid6x5_distance", "grid12x10_global"])
def test_gpsr_drift_matches_oracle(engine, engine_lib, oracle_lib, case):
    E, O = engine_lib, oracle_lib
    if case == "grid3x3_onsite":
        w = configs.grid(3, 3, U0=4.0, seed=2, n_traj=4)
        U, coul, ext, B = w.U, E.COUL_ONSITE, None, 4
    elif case == "grid6x5_ext":
        w = configs.grid(6, 5, U0=3.0, seed=4, n_traj=3)
        rng = np.random.default_rng(5)
        ext = np.diag(rng.uniform(-1, 1, w.n)) + 0.2 * (np.eye(w.n, k=1) + np.eye(w.n, k=-1))
        U, coul, B = w.U, E.COUL_ONSITE, 3
    elif case == "grid6x5_distance":
        w = configs.grid(6, 5, U0=3.0, seed=4, n_traj=3)
        U, coul, ext, B = distance_U(configs.grid_positions(6, 5), 2.0), E.COUL_DISTANCE, None, 3
    else:   # n = 120: the stage input does not fit shared memory and is read from global memory
        w = configs.grid(12, 10, U0=4.0, seed=6, n_traj=2)
        U, coul, ext, B = w.U, E.COUL_ONSITE, None, 2
    n = w.n
    rho = random_states(n, B, 11)
    V = np.zeros((n, n))
    engine.set_system(w.tM, U, V, ext, coulomb=coul)
    d = engine.gpsr_drift(rho, 0.01)
    ref = O.gpsr_drift(O.System(tM=w.tM, U=U, V=V, ext=ext, coulomb=coul, ext_null=ext is None), rho, 0.01)
    assert np.array_equal(d, ref), np.abs(d - ref).max()
    assert np.abs(d).max() > 1e-4          # not vacuous
    # the diagonal of the drift is complex (the state is not Hermitian)
    assert np.abs(np.einsum("bsii->bsi", d).imag).max() > 1e-8


def test_gpsr_drift_of_a_hermitian_state_is_the_hf_step(engine, engine_lib, oracle_lib):
    """For a Hermitian state with on-site U, the GPSR derivative is the HF one (shift
    0, real diagonal), so the drift equals the increment of one HF RK4 step."""
    E, O = engine_lib, oracle_lib
    w = configs.grid(4, 4, U0=4.0, seed=3, n_traj=2)
    n = w.n
    A = random_states(n, 2, 21, scale=0.1)
    H = 0.5 * (A + np.conj(np.transpose(A, (0, 1, 3, 2))))
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    d = engine.gpsr_drift(H, 0.02)
    engine.set_initial_samples(H)
    engine.run(E.METHOD_HF, E.PREC_FP64, 0.02, 1, 2, obs=E.OBS_DIAG)
    assert np.abs(d - (engine.get_state() - H)).max() < 1e-14


def test_gpsr_drift_refuses_a_pulse(engine, engine_lib):
    E = engine_lib
    w = configs.grid(3, 3, U0=4.0, seed=2, n_traj=1)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.set_pulse(np.ones(2), 0.1, 0.1, 0.1, np.zeros(w.n))
    with pytest.raises(E.FpsgError) as ei:
        engine.gpsr_drift(random_states(w.n, 1, 1), 0.01)
    assert ei.value.code == E.ERR_UNSUPPORTED
