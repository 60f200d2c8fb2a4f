"""The 4-CTA-cluster resident kernel (k_resident_quad): matrices too large for one
CTA per spin — FP64 at n = 100, FP32 from n = 101 to n = 144.  Two CTAs share a
spin matrix, each integrating half of its elements and writing them into the other
one's copy through distributed shared memory.

FP64: bit-identical to the FP64 oracle (and to the FP64 stream path) for on-site
Coulomb (the next stage's Hartree diagonal written by the pass) and for a
long-range Coulomb matrix with a pulse (the diagonal formed after each stage).
FP32: within 1e-5 of the oracle over a short window."""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu


def osys(O, w, coul, ext=None, pulse=None):
    return O.System(tM=w.tM, U=w.U, V=w.V, ext=ext, coulomb=coul, ext_null=ext is None, pulse=pulse)


def test_quad_fp64_onsite_bit_identical(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w = configs.grid_10x10(U0=4.0, n_traj=6)
    rho0 = O.sample(w.n, 6, 31, w.occ_up, w.occ_dn)
    obs = O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER | O.OBS_WHOLE
    ref = O.run(osys(O, w, O.COUL_ONSITE, w.ext), O.METHOD_FTWA, w.dt, 2, 12, rho0, obs=obs)
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 2, 12, path=E.PATH_RESIDENT,
                   obs=E.OBS_DIAG | E.OBS_DIAG2 | E.OBS_DOUBLONS | E.OBS_ENERGIES | E.OBS_WHOLE)
    assert r.path_used == E.PATH_RESIDENT
    assert np.array_equal(engine.get_state(), ref["final"])
    for k in ("niiu", "niid", "n2iiu", "n2iid", "nund"):       # per-CTA ensemble sums
        assert np.abs(getattr(r, k) - ref[k]).max() < 1e-13, k
    assert np.abs(r.energies - ref["energies"]).max() < 1e-11 * max(1.0, np.abs(ref["energies"]).max())
    assert np.abs(r.whole_u - ref["whole_u"]).max() < 1e-13


def test_quad_fp64_long_range_coulomb_and_pulse(engine, engine_lib, oracle_lib):
    """Distance Coulomb U_ij = U0/(1 + r_ij): the Hartree diagonal needs the whole
    other-spin diagonal, so each CTA forms it after the stage from both spins'
    diagonals (the partner's read from its shared memory)."""
    E, O = engine_lib, oracle_lib
    w = configs.grid_10x10(U0=1.5, n_traj=4)
    pos = configs.grid_positions(10, 10)
    D = configs.distances(pos)
    U = 1.5 / (1.0 + D)
    V = U.copy()
    np.fill_diagonal(V, 0.0)
    rng = np.random.default_rng(3)
    pulse = {"n_bins": 5, "amp": rng.normal(0, 0.5, 5), "bin_width": 0.01, "t0": 0.02, "td": 0.03,
             "proj": pos[:, 0] - pos[:, 0].mean()}
    rho0 = O.sample(w.n, 4, 32, w.occ_up, w.occ_dn)
    sysm = O.System(tM=w.tM, U=U, V=V, ext=w.ext, coulomb=O.COUL_DISTANCE, ext_null=False, pulse=pulse)
    ref = O.run(sysm, O.METHOD_FTWA, 0.005, 2, 6, rho0, obs=O.OBS_DIAG | O.OBS_DOUB | O.OBS_ENER)
    engine.set_system(w.tM, U, V, w.ext, coulomb=E.COUL_DISTANCE)
    engine.set_pulse(pulse["amp"], pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, 0.005, 2, 6, path=E.PATH_RESIDENT,
                   obs=E.OBS_DIAG | E.OBS_DOUBLONS | E.OBS_ENERGIES)
    assert r.path_used == E.PATH_RESIDENT
    assert np.array_equal(engine.get_state(), ref["final"])
    assert np.abs(r.niiu - ref["niiu"]).max() < 1e-13 and np.abs(r.nund - ref["nund"]).max() < 1e-13
    assert np.abs(r.energies - ref["energies"]).max() < 1e-11 * max(1.0, np.abs(ref["energies"]).max())


def test_quad_fp64_many_trajectories_match_stream(engine, engine_lib):
    """More trajectories than clusters (each cluster takes several in turn) and a
    long launch: equal to the FP64 stream path bit for bit."""
    E = engine_lib
    w = configs.grid_10x10(U0=8.0, n_traj=600)
    engine.set_system(w.tM, w.U, w.V, w.ext, coulomb=E.COUL_ONSITE)
    out = {}
    for path in (E.PATH_STREAM, E.PATH_RESIDENT):
        engine.sample(600, 44, w.occ_up, w.occ_dn)
        r = engine.run(E.METHOD_FTWA, E.PREC_FP64, w.dt, 1, 20, obs=E.OBS_DIAG | E.OBS_DOUBLONS, path=path)
        assert r.path_used == path
        out[path] = (engine.get_state(), r)
    assert np.array_equal(out[E.PATH_STREAM][0], out[E.PATH_RESIDENT][0])
    for k in ("niiu", "niid", "nund"):
        a, b = getattr(out[E.PATH_STREAM][1], k), getattr(out[E.PATH_RESIDENT][1], k)
        assert np.abs(a - b).max() < 1e-13, k      # per-CTA vs per-chunk ensemble sums


@pytest.mark.parametrize("nx,ny", [(12, 9), (12, 12)], ids=["n108", "n144"])
def test_quad_fp32_large_grids(engine, engine_lib, oracle_lib, nx, ny):
    E, O = engine_lib, oracle_lib
    w = configs.grid(nx, ny, U0=4.0, seed=5, n_traj=3, dt=0.01)
    rho0 = O.sample(w.n, 3, 33, w.occ_up, w.occ_dn)
    ref = O.run(osys(O, w, O.COUL_ONSITE), O.METHOD_FTWA, 0.01, 2, 8, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.set_initial_samples(rho0)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP32, 0.01, 2, 8, obs=E.OBS_DIAG | E.OBS_DOUBLONS)
    assert r.path_used == E.PATH_RESIDENT
    assert np.abs(engine.get_state() - ref["final"]).max() < 1e-5
    assert np.abs(r.niiu - ref["niiu"]).max() < 1e-5 and np.abs(r.nund - ref["nund"]).max() < 1e-5
