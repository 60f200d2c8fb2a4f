"""The drop-in path on the GPU: makeSitesSystem -> edited JSON -> `fps` -> result JSON,
checked against the FP64 oracle on the same initial samples.

Mirrors the reference's own smoke script (tests.py: generate with makeSitesSystem,
run fps with HF, patch the JSON, run fTWA) with assertions on the numbers.
"""
import json
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tools():
    from fermiphasespace_b200 import build, hostlib
    build.build_cuda()
    build.build_host()
    return hostlib


def make_case(tools, tmp_path, method, extra_params=None, results=None, gpu=None, U=4.0):
    tools.make_sites_system("grid6", str(tmp_path), "grid", [3, 2])
    p = tmp_path / "grid6.json"
    doc = json.load(open(p))
    doc["method"] = method
    doc["parameters"] = {"dt": 0.01, "t_max": 0.3, "stepsParTimePoints": 10, "n_traj": 32}
    doc["parameters"].update(extra_params or {})
    doc["system"]["coulombInteraction"]["onSiteInteraction"] = U
    doc["results"] = results or {"diagDMatrix": True, "diag2DMatrix": True, "onSiteDoublons": True,
                                 "energies": True, "wholeDMatrix": True}
    if gpu is not None:
        doc["gpu"] = gpu
    p.write_text(json.dumps(doc))
    return p


def run_fps(tools, path):
    r = subprocess.run([tools.FPS_EXE, str(path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def oracle_system(O, w):
    return O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True)


def test_fps_ftwa_matches_oracle(tools, oracle_lib, tmp_path):
    from fermiphasespace_b200 import configs
    O = oracle_lib
    p = make_case(tools, tmp_path, "fTWA", gpu={"seed": 5, "fTWAEnergies": "computed"})
    run_fps(tools, p)
    res = json.load(open(tmp_path / "grid6_fTWA_res.json"))
    sim = res["simulation"]
    assert res["fpsVersion"] == "0.5.0"
    Tp = 31
    assert len(sim["t"]) == Tp and abs(sim["t"][-1] - 0.3) < 1e-12
    w = configs.grid_3x2()
    rho0 = O.sample(6, 32, 5, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, 0.01, 10, Tp, rho0, obs=O.OBS_DIAG | O.OBS_ENER | O.OBS_WHOLE)
    # the device sampler's log/sincos differ from the host libm by a few ulp; 300 RK steps
    for key, rk in (("Niiu", "niiu"), ("Niid", "niid"), ("N2iiu", "n2iiu"), ("NuNd", "nund")):
        assert np.abs(np.array(sim[key]) - ref[rk]).max() < 1e-9, key
    E = sim["E"]
    for row, name in enumerate(("tH", "U", "V", "pe", "tot")):
        assert np.abs(np.array(E[name]) - ref["energies"][row]).max() < 1e-9, name
    n1 = np.array(sim["N1hu"]["r"]) + 1j * np.array(sim["N1hu"]["i"])
    assert np.abs(n1 - ref["whole_u"][:, 0, 5]).max() < 1e-9


def test_fps_ftwa_reference_energy_rows(tools, tmp_path):
    """Without a core hole the reference never merges the energy sums: all rows zero."""
    p = make_case(tools, tmp_path, "fTWA", gpu={"seed": 1})
    run_fps(tools, p)
    sim = json.load(open(tmp_path / "grid6_fTWA_res.json"))["simulation"]
    for name in ("tH", "U", "V", "pe", "tot"):
        assert not np.any(sim["E"][name])


def test_fps_hf_bit_exact(tools, oracle_lib, tmp_path):
    from fermiphasespace_b200 import configs
    O = oracle_lib
    p = make_case(tools, tmp_path, "HF")
    run_fps(tools, p)
    sim = json.load(open(tmp_path / "grid6_HF_res.json"))["simulation"]
    w = configs.grid_3x2()
    N0 = np.zeros((1, 2, 6, 6), dtype=complex)
    N0[0, 0] = np.diag(w.occ_up)
    N0[0, 1] = np.diag(w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_HF, 0.01, 10, 31, N0)
    assert np.array_equal(np.array(sim["Niiu"]), ref["niiu"])
    assert np.array_equal(np.array(sim["NuNd"]), ref["nund"])
    assert np.abs(np.array(sim["E"]["tot"]) - ref["energies"][4]).max() < 1e-12


def test_fps_rejects_methods_outside_the_engine(tools, tmp_path):
    p = make_case(tools, tmp_path, "ED")
    r = subprocess.run([tools.FPS_EXE, str(p)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "not part of this engine" in (r.stdout + r.stderr)


def test_sampler_rotation_matches_numpy(engine, engine_lib, oracle_lib):
    """Rotated (ground-state) initial conditions: rho = R (diag(n - 1/2) + W) R^H."""
    E, O = engine_lib, oracle_lib
    from fermiphasespace_b200 import configs
    w = configs.grid_3x2()
    occ = np.array([1.0, 1, 1, 0, 0, 0])
    _, R = np.linalg.eigh(w.tM)
    engine.set_system(w.tM, w.U, w.V, None, coulomb=E.COUL_ONSITE)
    engine.sample(16, 3, occ, occ, R, R)
    got = engine.get_state()
    base = O.sample(6, 16, 3, occ, occ)
    want = np.einsum("ij,bsjk,lk->bsil", R, base, R.conj())
    assert np.abs(got - want).max() < 1e-13


def test_fps_tensor_core_precision(tools, oracle_lib, tmp_path):
    """`"gpu": {"precision": "bf16x3"}` runs the dense tensor-core path from `fps`."""
    from fermiphasespace_b200 import configs
    O = oracle_lib
    p = make_case(tools, tmp_path, "fTWA", gpu={"seed": 5, "precision": "bf16x3"})
    run_fps(tools, p)
    sim = json.load(open(tmp_path / "grid6_fTWA_res.json"))["simulation"]
    w = configs.grid_3x2()
    rho0 = O.sample(6, 32, 5, w.occ_up, w.occ_dn)
    ref = O.run(oracle_system(O, w), O.METHOD_FTWA, 0.01, 10, 31, rho0, obs=O.OBS_DIAG | O.OBS_DOUB)
    for key, rk in (("Niiu", "niiu"), ("NuNd", "nund")):
        assert np.abs(np.array(sim[key]) - ref[rk]).max() < 5e-5, key


def oracle_snapshots(O, sysm, dt, S, Tp, rho0):
    """Per-trajectory fTWA states at every snapshot t = 0 .. Tp-1, by chaining
    one-snapshot oracle runs (each records, then takes S steps); for a static
    Hamiltonian the chain is the same computation as one long run."""
    states = [rho0]
    cur = rho0
    for _ in range(1, Tp):
        cur = O.run(sysm, O.METHOD_FTWA, dt, S, 1, cur, obs=O.OBS_DIAG)["final"]
        states.append(cur)
    return states


def test_fps_core_hole_states_nich_and_ground_state_blocks(tools, oracle_lib, tmp_path):
    """fTWA through `fps` on the 3x2 grid with a core hole (src/FHSystem.cpp:296-324)
    and every result the reference can write: TB- and MF-basis occupations
    Mkk = diag(V^H N V) (src/FHfTWASolver.cpp:386-395, normalised at :535-541),
    NiCh = N(site, n-1) (src/FHSolver.cpp:285-291), energies (merged for core-hole
    systems, src/FHfTWASolver.cpp:470-476) and the tbGroundState / mfGroundState
    blocks (src/FHSolver.cpp:178-185).  The engine forms Mkk from the ensemble-mean
    density matrix; the check forms it as the reference does, per trajectory from the
    oracle's states and then averaged.  Tolerance 1e-9 as in the other fps tests
    (device sampler vs host libm in the last ulp)."""
    O = oracle_lib
    B, Tp, dt, S, seed = 16, 11, 0.01, 5, 9
    tools.make_sites_system("ch6", str(tmp_path), "grid", [3, 2])
    p = tmp_path / "ch6.json"
    doc = json.load(open(p))
    doc["method"] = "fTWA"
    doc["parameters"] = {"dt": dt, "t_max": dt * (Tp - 1), "stepsParTimePoints": S, "n_traj": B}
    doc["system"]["coulombInteraction"]["onSiteInteraction"] = 3.0
    doc["system"]["coreHole"] = {"presence": True, "site": 2, "eps": -2.0, "X": -0.5, "Uc": 1.5, "G": 0.7,
                                 "IC": [1, 0]}
    doc["results"] = {"diagDMatrix": True, "onSiteDoublons": True, "energies": True, "tbStates": True,
                      "mfStates": True}
    doc["gpu"] = {"seed": seed}
    p.write_text(json.dumps(doc))
    run_fps(tools, p)
    res = json.load(open(tmp_path / "ch6_fTWA_res.json"))
    sim = res["simulation"]

    sysh = tools.System(str(p))
    m = sysh.matrices()
    assert m["core_hole"] and sysh.n == 7
    ou, od = sysh.occupations(6)
    ou = np.append(ou, 1.0)
    od = np.append(od, 0.0)
    sysm = O.System(tM=m["tM"], U=m["U"], V=m["V"], ext=m["ext"], coulomb=m["coulomb"], ext_null=m["ext_null"])
    rho0 = O.sample(7, B, seed, ou, od)
    ref = O.run(sysm, O.METHOD_FTWA, dt, S, Tp, rho0, obs=O.OBS_DIAG | O.OBS_DOUB | O.OBS_ENER | O.OBS_WHOLE)
    for key, rk in (("Niiu", "niiu"), ("Niid", "niid"), ("NuNd", "nund")):
        assert np.abs(np.array(sim[key]) - ref[rk]).max() < 1e-9, key
    # core-hole systems merge the energies (they are not all zero here)
    for row, name in enumerate(("tH", "U", "V", "pe", "tot")):
        assert np.abs(np.array(sim["E"][name]) - ref["energies"][row]).max() < 1e-9, name
    assert np.abs(np.array(sim["E"]["tot"])).max() > 1e-3
    # NiCh: the ensemble mean of rho(site, n-1), complex
    for spin, key in ((0, "u"), (1, "d")):
        got = np.array(sim["NiCh"][key]["r"]) + 1j * np.array(sim["NiCh"][key]["i"])
        want = ref["whole_u" if spin == 0 else "whole_d"][:, 2, 6]
        assert np.abs(got - want).max() < 1e-9, key
    assert np.abs(np.array(sim["NiCh"]["u"]["r"])).max() > 1e-6

    # ground-state blocks: TB eigenpairs of the lattice hopping, MF self-consistent
    T6 = m["tM"][:6, :6]
    tb = res["tbGroundState"]
    Vt, Et = np.array(tb["rotationMatrix"]), np.array(tb["energyVector"])
    assert np.allclose(Vt.T @ Vt, np.eye(6), atol=1e-12)
    assert np.allclose(T6 @ Vt, Vt * Et, atol=1e-12)
    assert np.all(np.diff(Et) >= -1e-12)
    mf = res["mfGroundState"]
    Vu, Vd = np.array(mf["rotationMatrixUp"]), np.array(mf["rotationMatrixDown"])
    for V in (Vu, Vd):
        assert np.allclose(V.T @ V, np.eye(6), atol=1e-12)

    # Mkk and Mukk, per trajectory as the reference accumulates them
    def ext(V):
        X = np.eye(7)
        X[:6, :6] = V
        return X
    snaps = oracle_snapshots(O, sysm, dt, S, Tp, rho0)
    for key, V, spin in (("Mkku", Vt, 0), ("Mkkd", Vt, 1), ("Mukku", Vu, 0), ("Mukkd", Vd, 1)):
        Vx = ext(V)
        want = np.stack([np.real(np.einsum("ik,bij,jk->bk", Vx.conj(), st[:, spin], Vx)).mean(0) + 0.5
                         for st in snaps], axis=1)
        got = np.array(sim[key])
        assert got.shape == (7, Tp), (key, got.shape)
        assert np.abs(got - want).max() < 1e-9, (key, np.abs(got - want).max())


def test_fps_sharded_over_two_processes_equals_one(tools, tmp_path):
    """`fps` launched as two ranks (WORLD_SIZE=2, as torchrun or mpirun would) splits
    the trajectories like the reference's MPI solver, each rank draws its range of
    the seeded ensemble, the ranks sum their observables over the native exchange
    and rank 0 writes the result file.  Both ranks run on the one GPU here (their
    kernels never wait on each other); the result equals the single-process run of
    the same file to rounding (the ensemble sums are split differently)."""
    import os
    import shutil
    import socket
    one = tmp_path / "one"
    two = tmp_path / "two"
    one.mkdir()
    two.mkdir()
    p1 = make_case(tools, one, "fTWA", gpu={"seed": 5, "fTWAEnergies": "computed"},
                   extra_params={"n_traj": 37})
    shutil.copy(one / "grid6.xyz", two / "grid6.xyz")
    p2 = two / "grid6.json"
    shutil.copy(p1, p2)
    run_fps(tools, p1)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
                   FPS_SHARD_PORT=str(port), FPS_SHARD_TIMEOUT="120")
        procs.append(subprocess.Popen([tools.FPS_EXE, str(p2)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [pr.communicate(timeout=300)[0] for pr in procs]
    assert all(pr.returncode == 0 for pr in procs), outs
    assert "trajectories from 0 to 17" in outs[0] and "trajectories from 18 to 36" in outs[1], outs
    ref = json.load(open(one / "grid6_fTWA_res.json"))["simulation"]
    got = json.load(open(two / "grid6_fTWA_res.json"))["simulation"]
    for key in ("Niiu", "Niid", "N2iiu", "N2iid", "NuNd"):
        assert np.abs(np.array(got[key]) - np.array(ref[key])).max() < 1e-12, key
    for name in ("tH", "U", "V", "pe", "tot"):
        assert np.abs(np.array(got["E"][name]) - np.array(ref["E"][name])).max() < 1e-12, name
    for part in ("r", "i"):
        assert np.abs(np.array(got["N1hu"][part]) - np.array(ref["N1hu"][part])).max() < 1e-12
