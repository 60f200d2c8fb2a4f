"""Discrete adjoint (fpsg_grad): gradients of the time-integrated doublon occupancy
with respect to the U scale, the t scale and the per-bin pulse amplitudes.

Checked against central finite differences (h = 1e-4, FP64) of the FP64 oracle and
of the GPU forward pass, and wrapped in a torch.autograd.Function (test harness
only) whose backward must return the same numbers.
"""
import math

import numpy as np
import pytest

from fermiphasespace_b200 import configs

pytestmark = pytest.mark.gpu

H = 1e-4


def pulse_case():
    w = configs.grid(3, 3, U0=4.0, seed=2, n_traj=4)
    pos = configs.grid_positions(3, 3)
    proj = pos[:, 0] - pos[:, 0].mean()
    rng = np.random.default_rng(7)
    pulse = {"n_bins": 5, "amp": rng.normal(0, 0.5, 5), "bin_width": 0.04, "t0": 0.1, "td": 0.06, "proj": proj}
    return w, pulse


def oracle_loss(O, w, pulse, rho0, dt, S, Tp, su=1.0, st=1.0, amp=None):
    p = dict(pulse)
    if amp is not None:
        p["amp"] = amp
    sysm = O.System(tM=w.tM * st, U=w.U * su, V=w.V * su, coulomb=O.COUL_ONSITE, ext_null=True, pulse=p)
    out = O.run(sysm, O.METHOD_FTWA, dt, S, Tp, rho0, obs=O.OBS_DOUB, want_final=False)
    wts = np.full(Tp, dt)
    wts[0] = wts[-1] = dt / 2
    return float((wts * out["nund"].mean(axis=0)).sum())


def setup(engine, E, w, pulse, rho0, su=1.0, st=1.0, amp=None):
    engine.set_system(w.tM * st, w.U * su, w.V * su, None, coulomb=E.COUL_ONSITE)
    engine.set_pulse(pulse["amp"] if amp is None else amp, pulse["bin_width"], pulse["t0"], pulse["td"], pulse["proj"])
    engine.set_initial_samples(rho0)


def test_adjoint_fp64_matches_oracle_finite_differences(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    dt, S, Tp = 0.02, 2, 11
    rho0 = O.sample(w.n, 4, 3, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    g = engine.grad(E.PREC_FP64, dt, S, Tp, checkpoint_every=3)
    L0 = oracle_loss(O, w, pulse, rho0, dt, S, Tp)
    assert abs(g["loss"] - L0) < 1e-12 * max(1.0, abs(L0))
    fdU = (oracle_loss(O, w, pulse, rho0, dt, S, Tp, su=1 + H) - oracle_loss(O, w, pulse, rho0, dt, S, Tp, su=1 - H)) / (2 * H)
    fdT = (oracle_loss(O, w, pulse, rho0, dt, S, Tp, st=1 + H) - oracle_loss(O, w, pulse, rho0, dt, S, Tp, st=1 - H)) / (2 * H)
    assert abs(g["dU"] - fdU) < 1e-6 * max(1.0, abs(fdU)), (g["dU"], fdU)
    assert abs(g["dt"] - fdT) < 1e-6 * max(1.0, abs(fdT)), (g["dt"], fdT)
    for b in range(5):
        ap, am = pulse["amp"].copy(), pulse["amp"].copy()
        ap[b] += H
        am[b] -= H
        fd = (oracle_loss(O, w, pulse, rho0, dt, S, Tp, amp=ap) - oracle_loss(O, w, pulse, rho0, dt, S, Tp, amp=am)) / (2 * H)
        assert abs(g["dpulse"][b] - fd) < 1e-6 * max(1e-3, abs(fd)) + 1e-10, (b, g["dpulse"][b], fd)
    # the context state is untouched by fpsg_grad
    assert np.array_equal(engine.get_state()[:, :, np.arange(9), np.arange(9)].real,
                          rho0[:, :, np.arange(9), np.arange(9)].real)


def test_adjoint_checkpoint_interval_does_not_change_the_gradient(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    rho0 = O.sample(w.n, 4, 5, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    a = engine.grad(E.PREC_FP64, 0.02, 1, 16, checkpoint_every=1)
    b = engine.grad(E.PREC_FP64, 0.02, 1, 16, checkpoint_every=7)
    c = engine.grad(E.PREC_FP64, 0.02, 1, 16, checkpoint_every=64)
    for k in ("dU", "dt"):
        assert abs(a[k] - b[k]) < 1e-12 and abs(a[k] - c[k]) < 1e-12
    assert np.abs(a["dpulse"] - c["dpulse"]).max() < 1e-12


def test_adjoint_fp32_close_to_fp64(engine, engine_lib, oracle_lib):
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    rho0 = O.sample(w.n, 16, 9, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    g64 = engine.grad(E.PREC_FP64, 0.02, 2, 11)
    g32 = engine.grad(E.PREC_FP32, 0.02, 2, 11)
    assert abs(g32["loss"] - g64["loss"]) < 1e-6
    for k in ("dU", "dt"):
        assert abs(g32[k] - g64[k]) < 1e-4 * max(1.0, abs(g64[k]))
    assert np.abs(g32["dpulse"] - g64["dpulse"]).max() < 1e-4


def test_torch_autograd_wrapper(engine, engine_lib, oracle_lib):
    """The adjoint as the backward of a torch.autograd.Function (harness only)."""
    import torch
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    rho0 = O.sample(w.n, 4, 3, w.occ_up, w.occ_dn)

    class DoublonLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u_scale, t_scale, amps):
            setup(engine, E, w, pulse, rho0, su=float(u_scale), st=float(t_scale), amp=amps.detach().cpu().numpy())
            g = engine.grad(E.PREC_FP64, 0.02, 2, 11)
            ctx.save_for_backward(torch.tensor(g["dU"] / float(u_scale), dtype=torch.float64),
                                  torch.tensor(g["dt"] / float(t_scale), dtype=torch.float64),
                                  torch.from_numpy(g["dpulse"]))
            return torch.tensor(g["loss"], dtype=torch.float64)

        @staticmethod
        def backward(ctx, go):
            gu, gt, gp = ctx.saved_tensors
            return go * gu, go * gt, go * gp

    u = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    t = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    a = torch.tensor(pulse["amp"], dtype=torch.float64, requires_grad=True)
    L = DoublonLoss.apply(u, t, a)
    L.backward()
    fd = (oracle_loss(O, w, pulse, rho0, 0.02, 2, 11, su=1 + H) - oracle_loss(O, w, pulse, rho0, 0.02, 2, 11, su=1 - H)) / (2 * H)
    assert abs(u.grad.item() - fd) < 1e-6 * max(1.0, abs(fd))
    assert a.grad.shape == (5,)


@pytest.mark.parametrize("prec,tol", [("FP64", 1e-11), ("FP32", 2e-5)])
def test_segment_reverse_kernel_matches_per_stage_kernels(engine, engine_lib, oracle_lib, prec, tol):
    """With an on-site U the reverse sweep runs one segment-resident launch per
    checkpoint segment; the same U given as a distance Coulomb matrix with V = 0
    (the same dynamics and loss) takes the per-stage kernels.  The gradients agree.
    The small systems take the variant with the stage adjoints in shared memory;
    the 8x8 grid in FP64 does not fit two clusters per SM pair that way and takes
    the variant with them in registers."""
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    w2 = configs.grid(6, 5, U0=3.0, seed=4, n_traj=24)
    w3 = configs.grid(8, 8, U0=4.0, seed=6, n_traj=24)
    for sysw, pl in ((w, pulse), (w2, None), (w3, None)):
        rho0 = O.sample(sysw.n, 24, 11, sysw.occ_up, sysw.occ_dn)
        res = []
        for coul in (E.COUL_ONSITE, E.COUL_DISTANCE):
            engine.set_system(sysw.tM, sysw.U, np.zeros_like(sysw.V), None, coulomb=coul)
            if pl is not None:
                engine.set_pulse(pl["amp"], pl["bin_width"], pl["t0"], pl["td"], pl["proj"])
            engine.set_initial_samples(rho0)
            res.append(engine.grad(getattr(E, "PREC_" + prec), 0.02, 2, 9, checkpoint_every=5))
        a, b = res
        assert abs(a["loss"] - b["loss"]) < 1e-12 * max(1.0, abs(b["loss"]))
        for k in ("dU", "dt"):
            assert abs(a[k] - b[k]) < tol * max(1.0, abs(b[k])), (prec, k, a[k], b[k])
        if pl is not None:
            assert np.abs(a["dpulse"] - b["dpulse"]).max() < tol * max(1.0, np.abs(b["dpulse"]).max())


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_kept_segments_give_the_same_gradient(engine, engine_lib, oracle_lib, prec):
    """The forward pass may keep the stage inputs of its last segments instead of
    recomputing them in the backward pass (fpsg_set_grad_memory).  All segments
    kept, two kept, and none kept give the same gradient to the bit: the kept
    inputs come from the same kernel arithmetic as the recomputed ones."""
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    B, C, S, Tp = 16, 5, 1, 31
    rho0 = O.sample(w.n, B, 13, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    elem = 16 if prec == "FP64" else 8
    segbytes = elem * B * 2 * (w.n * (w.n + 1) // 2) * 4 * C
    res = []
    for budget in (-1, 2 * segbytes + 64, 0):
        engine.set_grad_memory(budget)
        res.append(engine.grad(getattr(E, "PREC_" + prec), 0.02, S, Tp, checkpoint_every=C))
    engine.set_grad_memory(-1)
    for r in res[1:]:
        for k in ("loss", "dU", "dt"):
            assert r[k] == res[0][k], (prec, k, r[k], res[0][k])
        assert np.array_equal(r["dpulse"], res[0]["dpulse"])


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_trajectory_chunks_give_the_same_gradient(engine, engine_lib, oracle_lib, prec):
    """When the stage inputs of every segment of the whole ensemble do not fit the
    kept-segment budget, fpsg_grad runs the trajectories in chunks (each a multiple
    of one trajectory per SM) so that every segment of a chunk is kept.  Three
    chunks, one chunk with every segment kept, and one chunk with none kept give
    the same parameter gradients to the bit (the per-trajectory partials do not
    depend on the chunking) and the same loss to rounding."""
    import torch
    E, O = engine_lib, oracle_lib
    w, pulse = pulse_case()
    sm = torch.cuda.get_device_properties(0).multi_processor_count
    B, C, S, Tp = 3 * sm, 5, 1, 31
    rho0 = O.sample(w.n, B, 17, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    elem = 16 if prec == "FP64" else 8
    nseg = (Tp - 1 + C - 1) // C
    per_traj = elem * 2 * (w.n * (w.n + 1) // 2) * 4 * C * nseg     # every segment of one trajectory
    res = []
    for budget in (-1, per_traj * sm, 0):
        engine.set_grad_memory(budget)
        res.append(engine.grad(getattr(E, "PREC_" + prec), 0.02, S, Tp, checkpoint_every=C))
    engine.set_grad_memory(-1)
    assert (res[0]["chunks"], res[0]["kept_segments"]) == (1, nseg)
    assert (res[1]["chunks"], res[1]["chunk_traj"], res[1]["kept_segments"]) == (3, sm, nseg)
    assert (res[2]["chunks"], res[2]["kept_segments"]) == (1, 0)
    for r in res[1:]:
        assert abs(r["loss"] - res[0]["loss"]) <= 1e-13 * abs(res[0]["loss"]), (prec, r["loss"], res[0]["loss"])
        for k in ("dU", "dt"):
            assert r[k] == res[0][k], (prec, k, r[k], res[0][k])
        assert np.array_equal(r["dpulse"], res[0]["dpulse"])
    # and the chunked gradient is the oracle's (FP64) to the tolerance of the FD test
    if prec == "FP64":
        fd = (oracle_loss(O, w, pulse, rho0, 0.02, S, Tp, su=1 + H) - oracle_loss(O, w, pulse, rho0, 0.02, S, Tp, su=1 - H)) / (2 * H)
        assert abs(res[1]["dU"] - fd) < 1e-6 * max(1.0, abs(fd))


def gpu_loss(engine, E, w, pulse, rho0, dt, S, Tp, su=1.0, st=1.0, amp=None):
    """The loss from the FP64 forward pass (bit-identical to the oracle's)."""
    setup(engine, E, w, pulse, rho0, su=su, st=st, amp=amp)
    r = engine.run(E.METHOD_FTWA, E.PREC_FP64, dt, S, Tp, obs=E.OBS_DOUBLONS)
    wts = np.full(Tp, dt)
    wts[0] = wts[-1] = dt / 2
    return float((wts * r.nund.mean(axis=0)).sum())


def test_adjoint_full_shape_finite_differences(engine, engine_lib, oracle_lib):
    """The adjoint workload's shape (8x8 grid, on-site U = 4, 50-bin Gaussian-envelope
    site pulse, dt = 0.01, checkpoints every 16 steps) over t in [0, 5] (500 RK
    steps), with 16 trajectories.  Over this window the loss is sensitive enough
    that the central difference at h = 1e-4 still carries a truncation error of
    about 1e-3 (relative): its error against the adjoint must fall about 100-fold
    from h = 1e-4 to h = 1e-5 (second order, converging on the adjoint value), and
    the adjoint must agree with the difference at h = 1e-6 for the U scale, the t
    scale and three pulse bins.  The FP32 gradient against the FP64 one."""
    E, O = engine_lib, oracle_lib
    w, pulse = configs.adjoint_8x8(n_traj=16, t_max=5.0)
    dt, S, Tp = w.dt, 1, 501
    rho0 = O.sample(w.n, 16, 23, w.occ_up, w.occ_dn)
    setup(engine, E, w, pulse, rho0)
    g = engine.grad(E.PREC_FP64, dt, S, Tp, checkpoint_every=16)
    g32 = engine.grad(E.PREC_FP32, dt, S, Tp, checkpoint_every=16)
    L0 = gpu_loss(engine, E, w, pulse, rho0, dt, S, Tp)
    assert abs(g["loss"] - L0) < 1e-12 * abs(L0)

    def fd(h, **kw_pm):
        (name, (vp, vm)), = kw_pm.items()
        return (gpu_loss(engine, E, w, pulse, rho0, dt, S, Tp, **{name: vp}) -
                gpu_loss(engine, E, w, pulse, rho0, dt, S, Tp, **{name: vm})) / (2 * h)

    e4 = abs(fd(1e-4, su=(1 + 1e-4, 1 - 1e-4)) - g["dU"])
    e5 = abs(fd(1e-5, su=(1 + 1e-5, 1 - 1e-5)) - g["dU"])
    assert 30 < e4 / e5 < 300, (e4, e5)
    h6 = 1e-6
    fdU = fd(h6, su=(1 + h6, 1 - h6))
    fdT = fd(h6, st=(1 + h6, 1 - h6))
    assert abs(g["dU"] - fdU) < 1e-6 * max(1.0, abs(fdU)), (g["dU"], fdU)
    assert abs(g["dt"] - fdT) < 1e-6 * max(1.0, abs(fdT)), (g["dt"], fdT)
    for b in (10, 25, 40):
        ap, am = pulse["amp"].copy(), pulse["amp"].copy()
        ap[b] += h6
        am[b] -= h6
        f = fd(h6, amp=(ap, am))
        assert abs(g["dpulse"][b] - f) < 1e-6 * max(1e-2, abs(f)), (b, g["dpulse"][b], f)
    print("fp32-vs-fp64", abs(g32["loss"] - g["loss"]), abs(g32["dU"] - g["dU"]) / abs(g["dU"]),
          abs(g32["dt"] - g["dt"]) / abs(g["dt"]), np.abs(g32["dpulse"] - g["dpulse"]).max() / np.abs(g["dpulse"]).max())
    # measured: loss 1.1e-7 relative, dU / dt 1.5e-5, pulse bins 7e-5 of the largest
    assert abs(g32["loss"] - g["loss"]) < 1e-6 * abs(g["loss"])
    for k in ("dU", "dt"):
        assert abs(g32[k] - g[k]) < 2e-4 * abs(g[k]), (k, g32[k], g[k])
    assert np.abs(g32["dpulse"] - g["dpulse"]).max() < 5e-4 * np.abs(g["dpulse"]).max()
