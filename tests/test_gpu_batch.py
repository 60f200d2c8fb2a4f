"""fpsg_run_batch: several lattices of different size integrated together.  Systems
that fit a resident kernel (one CTA or 2-CTA cluster per matrix group, or two CTAs
per spin matrix) run it, all of them in one captured CUDA graph; the others share
one persistent stream-stage launch per RK stage, replayed from a graph per
snapshot.  Each system's observables must be bit-identical to the same system run
alone (same device sampler, same kernel and configuration), and the FP64 batch
must match the FP64 oracle on the same samples."""
import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu

OBS = 1 | 2 | 4 | 16   # diag, diag2, doublons, energies


@pytest.fixture(scope="module")
def batch():
    return configs.uneven_batch(scale=1 / 512)      # 4 / 2 / 2 / 4 / 4 trajectories


def descs(ws, seed0=10):
    from fermiphasespace_b200 import engine as E
    return [{"tM": w.tM, "U": w.U, "V": w.V, "ext": None, "coulomb": E.COUL_ONSITE, "n_traj": w.n_traj,
             "seed": seed0 + k, "occ_up": w.occ_up, "occ_dn": w.occ_dn} for k, w in enumerate(ws)]


def alone(engine, E, w, seed, method, prec, dt, S, Tp):
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.sample(w.n_traj, seed, w.occ_up, w.occ_dn)
    r = engine.run(method, prec, dt, S, Tp, obs=OBS)
    return r, engine.get_state()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batch_equals_each_system_alone(engine, engine_lib, batch, prec):
    E = engine_lib
    P = E.PREC_FP64 if prec == "fp64" else E.PREC_FP32
    res, info = engine.run_batch(descs(batch), E.METHOD_FTWA, P, 0.01, 2, 5, obs=OBS)
    assert info["traj_steps"] == sum(w.n_traj for w in batch) * 5 * 2
    paths = [r.path_used for r in res]
    if prec == "fp32":
        # every system of the batch fits a resident kernel in FP32 (n = 108 and 144
        # on two CTAs per spin)
        assert paths == [E.PATH_RESIDENT] * len(batch)
    else:
        # FP64: the 24- and 64-site systems resident, the others on the stream stage
        assert E.PATH_RESIDENT in paths and E.PATH_STREAM in paths
    for k, w in enumerate(batch):
        ref, _ = alone(engine, E, w, 10 + k, E.METHOD_FTWA, P, 0.01, 2, 5)
        assert ref.path_used == res[k].path_used, w.name
        for key in ("niiu", "niid", "n2iiu", "n2iid", "nund"):
            assert np.array_equal(getattr(res[k], key), getattr(ref, key)), (w.name, key)
        # energy partials are summed across the CTA's threads, whose count the autotuner picks
        tol = 1e-12 if prec == "fp64" else 1e-5
        assert np.allclose(res[k].energies, ref.energies, rtol=tol, atol=tol), w.name


def test_batch_fp64_matches_oracle(engine, engine_lib, oracle_lib, batch):
    E, O = engine_lib, oracle_lib
    res, _ = engine.run_batch(descs(batch, 30), E.METHOD_FTWA, E.PREC_FP64, 0.01, 1, 4, obs=OBS)
    for k, w in enumerate(batch):
        engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        engine.sample(w.n_traj, 30 + k, w.occ_up, w.occ_dn)
        rho0 = engine.get_state()
        ref = O.run(O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True), O.METHOD_FTWA,
                    0.01, 1, 4, rho0, obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER)
        # states are bit-identical on either path; ensemble sums in the oracle's order
        # on the stream stage, per CTA (equal to rounding) on the resident kernels
        tol = 0.0 if res[k].path_used == E.PATH_STREAM else 1e-13
        for key in ("niiu", "nund", "n2iiu"):
            assert np.abs(getattr(res[k], key) - ref[key]).max() <= tol, (w.name, key)


def test_batch_hf(engine, engine_lib, batch):
    E = engine_lib
    ws = batch[:3]
    ds = descs(ws)
    for d in ds:
        d["n_traj"] = 1
    res, _ = engine.run_batch(ds, E.METHOD_HF, E.PREC_FP64, 0.01, 3, 4, obs=OBS)
    for k, w in enumerate(ws):
        engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
        engine.sample(1, 10 + k, w.occ_up, w.occ_dn)
        ref = engine.run(E.METHOD_HF, E.PREC_FP64, 0.01, 3, 4, obs=OBS)
        assert ref.path_used == res[k].path_used
        assert np.array_equal(res[k].niiu, ref.niiu)
        assert np.allclose(res[k].energies, ref.energies, rtol=1e-12, atol=1e-12)


def test_batch_autotuner_choice_is_cached(engine, engine_lib, batch):
    """The stream-stage part (FP64: the 108- and 144-site systems) picks threads per
    CTA and work order by timing them once per batch shape."""
    E = engine_lib
    _, a = engine.run_batch(descs(batch), E.METHOD_FTWA, E.PREC_FP64, 0.01, 1, 3, obs=1)
    _, b = engine.run_batch(descs(batch, 50), E.METHOD_FTWA, E.PREC_FP64, 0.01, 1, 3, obs=1)
    assert a["block_threads"] in (128, 256, 512) and a["schedule"] in (0, 1)
    assert (b["block_threads"], b["schedule"]) == (a["block_threads"], a["schedule"])
    assert b["tune_ms"] == 0.0
    assert a["kernel_launches"] >= a["graph_nodes"] > 0


def test_batch_rejects_what_it_does_not_do(engine, engine_lib, batch):
    E = engine_lib
    with pytest.raises(E.FpsgError) as ei:
        engine.run_batch(descs(batch[:1]), E.METHOD_FTWA, E.PREC_FP32, 0.01, 1, 2, obs=E.OBS_WHOLE)
    assert ei.value.code == E.ERR_UNSUPPORTED
    with pytest.raises(E.FpsgError) as ei:
        engine.run_batch(descs(batch[:1]), E.METHOD_FTWA, E.PREC_SPLIT_BF16X3, 0.01, 1, 2)
    assert ei.value.code == E.ERR_UNSUPPORTED
