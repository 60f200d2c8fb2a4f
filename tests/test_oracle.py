"""Known-answer tests pinning the FP64 oracle (CPU only).

The reference ships no usable golden outputs and cannot be built here (it needs
Armadillo + BLAS/LAPACK), so the oracle is pinned by analytic properties of the
equations it restates (src/FHfTWASolver.cpp:568-661, src/FHHFSolver.cpp:527-608),
by an independent numpy restatement, and by committed golden files.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle_np as ON

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def grid_system(nx, ny, U0=4.0, coul=O.COUL_ONSITE):
    pos = ON.grid_positions(nx, ny)
    D = ON.distance_matrix(pos)
    T = ON.tunneling(D, [(1.0, -1.0)])
    U, V = ON.coulomb_onsite(D, U0)
    return O.System(tM=T, U=U, V=V, coulomb=coul, ext_null=True), D


def neel(n):
    u = np.array([1.0 if i % 2 == 0 else 0.0 for i in range(n)])
    return u, 1.0 - u


def test_linear_step_is_degree4_taylor(oracle_lib):
    """U = 0: one 3/8-rule step of L(rho) = -i(rho T - T rho) equals sum_{k<=4} h^k L^k / k!."""
    sysm, _ = grid_system(3, 2, coul=O.COUL_NULL)
    T = sysm.tM
    rho0 = O.sample(6, 3, 11, *neel(6))
    h = 0.05
    out = O.run(sysm, O.METHOD_FTWA, h, 1, 1, rho0)
    L = lambda r: -1j * (r @ T - T @ r)
    for b in range(3):
        for s in range(2):
            r = rho0[b, s]
            acc, term = r.copy(), r.copy()
            for k in range(1, 5):
                term = L(term) * h / k
                acc = acc + term
            assert np.abs(out["final"][b, s] - acc).max() < 1e-14


def test_linear_matches_exact_propagator(oracle_lib):
    """U = 0: rho(t) = e^{iTt} rho0 e^{-iTt}; the RK4 error is O(h^4)."""
    sysm, _ = grid_system(3, 2, coul=O.COUL_NULL)
    w, Q = np.linalg.eigh(sysm.tM)
    rho0 = O.sample(6, 2, 5, *neel(6))
    errs = []
    for h in (0.04, 0.02):
        Tp = int(round(1.0 / h))
        out = O.run(sysm, O.METHOD_FTWA, h, 1, Tp, rho0)
        t = Tp * h
        Ut = Q @ np.diag(np.exp(1j * w * t)) @ Q.conj().T
        exact = np.einsum("ij,bsjk,lk->bsil", Ut, rho0, Ut.conj())
        errs.append(np.abs(out["final"] - exact).max())
    assert errs[0] < 1e-4  # ~ |T|^5 h^4 t / 120
    assert errs[0] / errs[1] > 12.0  # fourth order: ideal ratio 16


def test_trace_and_hermiticity_conserved(oracle_lib):
    sysm, _ = grid_system(3, 2, U0=4.0)
    rho0 = O.sample(6, 8, 3, *neel(6))
    out = O.run(sysm, O.METHOD_FTWA, 0.01, 10, 101, rho0)
    f = out["final"]
    assert np.array_equal(f, np.conj(np.transpose(f, (0, 1, 3, 2))))  # exact, by construction of the order
    tr0 = np.trace(rho0, axis1=2, axis2=3)
    tr1 = np.trace(f, axis1=2, axis2=3)
    assert np.abs(tr1 - tr0).max() < 1e-12


def test_diagonal_hamiltonian_freezes_densities(oracle_lib):
    n = 5
    sysm = O.System(tM=np.zeros((n, n)), U=4.0 * np.eye(n), V=np.zeros((n, n)), coulomb=O.COUL_ONSITE)
    rho0 = O.sample(n, 4, 9, *neel(n))
    out = O.run(sysm, O.METHOD_FTWA, 0.02, 3, 21, rho0)
    d0 = np.real(np.diagonal(rho0, axis1=2, axis2=3))
    d1 = np.real(np.diagonal(out["final"], axis1=2, axis2=3))
    assert np.array_equal(d0, d1)


def hf_energy(T, U, N):
    nu, nd = np.real(np.diag(N[0])), np.real(np.diag(N[1]))
    return np.real(np.sum(T * (N[0] + N[1]))) + nu @ U @ nd


def test_hf_energy_conserved(oracle_lib):
    sysm, _ = grid_system(3, 2, U0=4.0)
    u, d = neel(6)
    rng = np.random.default_rng(1)
    # a non-stationary HF state: small random Hermitian coherences on a Neel density
    N0 = np.zeros((1, 2, 6, 6), dtype=complex)
    for s, occ in enumerate((u, d)):
        X = 0.05 * (rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)))
        N0[0, s] = np.diag(occ) + X + X.conj().T
    errs = []
    for S in (5, 10):
        out = O.run(sysm, O.METHOD_HF, 0.05, S, 41, N0, obs=O.OBS_ENER)
        E = out["energies"][4]
        errs.append(np.abs(E - E[0]).max())
        # the engine's energy rows agree with a direct evaluation
        assert abs(E[0] - hf_energy(sysm.tM, sysm.U, N0[0])) < 1e-12
    assert errs[1] < 1e-7
    assert errs[0] / max(errs[1], 1e-300) > 10.0


def scf_hartree(T, U, nup, ndn, iters=500):
    n = T.shape[0]
    du = np.full(n, nup / n)
    dd = np.full(n, ndn / n)
    for _ in range(iters):
        eu, vu = np.linalg.eigh(T + np.diag(U @ dd))
        ed, vd = np.linalg.eigh(T + np.diag(U @ du))
        Nu = vu[:, :nup] @ vu[:, :nup].T
        Nd = vd[:, :ndn] @ vd[:, :ndn].T
        du_new, dd_new = np.diag(Nu), np.diag(Nd)
        if np.abs(du_new - du).max() + np.abs(dd_new - dd).max() < 1e-14:
            break
        du = 0.5 * du + 0.5 * du_new
        dd = 0.5 * dd + 0.5 * dd_new
    return Nu, Nd


def test_mean_field_ground_state_is_stationary(oracle_lib):
    sysm, _ = grid_system(3, 2, U0=2.0)
    Nu, Nd = scf_hartree(sysm.tM, sysm.U, 3, 3)
    N0 = np.array([[Nu, Nd]], dtype=complex)
    out = O.run(sysm, O.METHOD_HF, 0.05, 4, 41, N0)
    assert np.abs(out["final"][0] - N0[0]).max() < 1e-9


def test_mirror_symmetry_preserved(oracle_lib):
    sysm, _ = grid_system(3, 2, U0=4.0)
    # mirror x -> 2 - x on the 3x2 grid (site = x + 3y)
    perm = np.array([2, 1, 0, 5, 4, 3])
    P = np.eye(6)[perm]
    occ = np.array([1.0, 0.0, 1.0, 0.0, 1.0, 0.0])  # mirror-symmetric
    N0 = np.array([[np.diag(occ), np.diag(1 - occ)]], dtype=complex)
    rng = np.random.default_rng(2)
    X = 0.1 * rng.normal(size=(6, 6))
    X = X + X.T
    X = 0.5 * (X + P @ X @ P.T)
    N0[0, 0] += X
    out = O.run(sysm, O.METHOD_HF, 0.02, 5, 51, N0)
    f = out["final"][0, 0]
    assert np.abs(P @ f @ P.T - f).max() < 1e-12


@pytest.mark.parametrize("method", [O.METHOD_FTWA, O.METHOD_HF])
def test_c_oracle_matches_numpy_twin(oracle_lib, method):
    sysm, _ = grid_system(3, 2, U0=4.0)
    rng = np.random.default_rng(4)
    w = rng.uniform(-1, 1, 6)
    sysm.ext = np.diag(w)
    sysm.ext_null = False
    rho0 = O.sample(6, 4, 21, *neel(6))
    if method == O.METHOD_HF:
        rho0 = rho0 + 0.5 * np.eye(6)
    a = O.run(sysm, method, 0.01, 4, 31, rho0)
    b = ON.run(sysm.tM, sysm.U, sysm.V, sysm.ext, sysm.coulomb, False, method, 0.01, 4, 31, rho0)
    for k in ("niiu", "niid", "n2iiu", "n2iid", "nund"):
        assert np.abs(a[k] - b[k]).max() < 1e-12, k
    assert np.abs(a["final"] - b["final"]).max() < 1e-12


def test_c_oracle_matches_numpy_twin_distance_coulomb_and_pulse(oracle_lib):
    pos = ON.grid_positions(2, 2)
    D = ON.distance_matrix(pos)
    T = ON.tunneling(D, [(1.0, -1.0), (math.sqrt(2), -0.3)])
    U = 3.0 / (1.0 + D)
    V = np.where(np.eye(4, dtype=bool), 0.0, 3.0 / (1.0 + D))
    pulse = {"n_bins": 5, "amp": np.array([0.3, -0.2, 0.5, 0.1, -0.4]), "bin_width": 0.1, "t0": 0.2,
             "td": 0.15, "proj": pos[:, 0].copy()}
    sysm = O.System(tM=T, U=U, V=V, coulomb=O.COUL_DISTANCE, ext_null=True, pulse=pulse)
    rho0 = O.sample(4, 3, 8, np.array([1.0, 0, 1, 0]), np.array([0.0, 1, 0, 1]))
    a = O.run(sysm, O.METHOD_FTWA, 0.01, 3, 51, rho0)
    b = ON.run(T, U, V, None, O.COUL_DISTANCE, True, O.METHOD_FTWA, 0.01, 3, 51, rho0, pulse=pulse)
    assert np.abs(a["final"] - b["final"]).max() < 1e-12
    for k in ("niiu", "nund"):
        assert np.abs(a[k] - b[k]).max() < 1e-12


def test_sampler_statistics(oracle_lib):
    n = 6
    u, d = neel(n)
    rho = O.sample(n, 4000, 123, u, d)
    assert np.array_equal(np.real(np.diagonal(rho[:, 0], axis1=1, axis2=2)), np.tile(u - 0.5, (4000, 1)))
    # sigma^2 = (n_i + n_j - 2 n_i n_j)/2: 1/2 where occupations differ, 0 otherwise
    m = np.abs(rho[:, 0]) ** 2
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            want = 0.5 if u[i] != u[j] else 0.0
            assert abs(m[:, i, j].mean() - want) < 0.04
    off = rho[:, 0][:, 0, 1]
    assert abs(off.mean()) < 0.03
    assert abs(np.var(off.real) - 0.25) < 0.03 and abs(np.var(off.imag) - 0.25) < 0.03
    # spin up and spin down draw from disjoint triangles of one matrix
    assert abs(np.corrcoef(rho[:, 0][:, 0, 1].real, rho[:, 1][:, 0, 1].real)[0, 1]) < 0.05


def test_golden_fixtures(oracle_lib):
    """The committed golden files (tests/golden/make_golden.py) still reproduce."""
    import json
    with open(os.path.join(GOLDEN, "manifest.json")) as fh:
        manifest = json.load(fh)
    from tests.golden import make_golden
    for case in manifest["cases"]:
        ref = np.load(os.path.join(GOLDEN, case["file"]))
        got = make_golden.compute(case["name"])
        for k in ref.files:
            assert np.array_equal(ref[k], got[k]), (case["name"], k)


def test_gpsr_drift_restatement_is_the_hf_increment_on_hermitian_states(oracle_lib):
    """The GPSR derivative (src/FHGPSRSolver.cpp:111-134) with on-site U equals the HF
    one (no 1/2 shift) when the state is Hermitian, so the GPSR drift of one step
    equals the increment of one HF RK4 step of the same state (static potential, so
    the HF k3 time convention does not enter)."""
    O = oracle_lib
    from fermiphasespace_b200 import configs
    w = configs.grid(3, 3, U0=4.0, seed=2, n_traj=3)
    n = w.n
    rng = np.random.default_rng(1)
    A = rng.normal(size=(3, 2, n, n)) + 1j * rng.normal(size=(3, 2, n, n))
    H = 0.05 * (A + np.conj(np.transpose(A, (0, 1, 3, 2))))
    for b in range(3):
        for s in range(2):
            H[b, s] += np.diag(rng.uniform(0, 1, n))
    sysm = O.System(tM=w.tM, U=w.U, V=np.zeros_like(w.U), coulomb=O.COUL_ONSITE, ext_null=True)
    d = O.gpsr_drift(sysm, H, 0.01)
    ref = O.run(sysm, O.METHOD_HF, 0.01, 1, 2, H, obs=O.OBS_DIAG)
    assert np.abs(d - (ref["final"] - H)).max() < 1e-15
    # and a non-Hermitian state gets a complex diagonal drift
    Z = H + 0.1 * (rng.normal(size=H.shape) + 1j * rng.normal(size=H.shape))
    dz = O.gpsr_drift(sysm, Z, 0.01)
    assert np.abs(np.einsum("bsii->bsi", dz).imag).max() > 1e-6
