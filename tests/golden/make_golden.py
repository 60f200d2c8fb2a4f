"""Generates the golden fixtures of the FP64 oracle (tests/golden/*.npz).

These are outputs of this project's own FP64 restatement (oracle/fps_oracle.c),
not reference data: FermiPhaseSpace ships no usable golden outputs and cannot be
built here.  They freeze the oracle's bits so that any change to it is visible,
and they are what the GPU parity tests compare the CUDA path against when the
oracle library is not rebuilt.  Regenerate with:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from fermiphasespace_b200 import configs  # noqa: E402

CASES = {
    # 3x2 grid Neel state, U=4 (the plain CPU-runnable case) with 16 trajectories
    # and 2 time units instead of 1000 trajectories and 10
    "grid3x2_ftwa": dict(cfg="grid_3x2", B=16, seed=0, Tp=201, method=O.METHOD_FTWA),
    # the same lattice under HF, one trajectory (N itself)
    "grid3x2_hf": dict(cfg="grid_3x2", B=1, seed=0, Tp=201, method=O.METHOD_HF),
}


def system_of(name: str):
    w = configs.grid_3x2()
    return w, O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True)


def initial(case) -> np.ndarray:
    w, _ = system_of(case["cfg"])
    if case["method"] == O.METHOD_HF:
        N0 = np.zeros((1, 2, w.n, w.n), dtype=complex)
        N0[0, 0] = np.diag(w.occ_up)
        N0[0, 1] = np.diag(w.occ_dn)
        rng = np.random.default_rng(case["seed"])
        for s in range(2):
            X = 0.05 * (rng.normal(size=(w.n, w.n)) + 1j * rng.normal(size=(w.n, w.n)))
            N0[0, s] += X + X.conj().T
        return N0
    return O.sample(w.n, case["B"], case["seed"], w.occ_up, w.occ_dn)


def compute(name: str) -> dict:
    case = CASES[name]
    w, sysm = system_of(case["cfg"])
    rho0 = initial(case)
    out = O.run(sysm, case["method"], w.dt, w.S, case["Tp"], rho0, obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER,
                nthreads=1)
    res = {"rho0": rho0, "final": out["final"]}
    for k in ("niiu", "niid", "n2iiu", "n2iid", "nund", "energies"):
        res[k] = out[k]
    return res


def main():
    manifest = {"cases": []}
    for name in CASES:
        res = compute(name)
        fn = f"{name}.npz"
        np.savez_compressed(os.path.join(HERE, fn), **res)
        manifest["cases"].append({"name": name, "file": fn, **{k: v for k, v in CASES[name].items()}})
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)


if __name__ == "__main__":
    main()
