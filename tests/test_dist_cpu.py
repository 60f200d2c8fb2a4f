"""Trajectory shards on two gloo ranks (CPU): each rank integrates its range of the
seed's ensemble with the FP64 oracle, the ranks sum their weighted observables
with one all_reduce, and the result must equal the oracle run on the whole
ensemble.  Also covers a rank that fails before the collective."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fermiphasespace_b200 import shards


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_range_partitions_like_the_mpi_solver():
    for B in (1, 7, 16, 1000, 1001):
        for ws in (1, 2, 3, 8):
            if ws > B:
                continue
            rs = [shards.shard_range(B, r, ws) for r in range(ws)]
            assert rs[0][0] == 0 and rs[-1][1] == B
            assert all(rs[i][1] == rs[i + 1][0] for i in range(ws - 1))
            sizes = [e - f for f, e in rs]
            # B // ws each, the last B % ws ranks one more
            assert sizes == [B // ws] * (ws - B % ws) + [B // ws + 1] * (B % ws)
    with pytest.raises(ValueError):
        shards.shard_range(10, 2, 2)


def test_pack_unpack_weighted_mean():
    a = {k: np.full((3, 4), 1.0) for k in shards.OBS_KEYS}
    b = {k: np.full((3, 4), 4.0) for k in shards.OBS_KEYS}
    out = shards.unpack(shards.pack(a, 1) + shards.pack(b, 2), a)
    assert out["n_traj"] == 3
    assert np.allclose(out["niiu"], 3.0)


def _worker(rank, ws, port, B, seed, result_q, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from fermiphasespace_b200 import configs
    from oracle import oracle as O
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before the collective")
        w = configs.grid_3x2()
        first, end = shards.shard_range(B, rank, ws)
        rho0 = O.sample(w.n, end - first, seed, w.occ_up, w.occ_dn, first=first)
        sysm = O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True)
        r = O.run(sysm, O.METHOD_FTWA, 0.01, 2, 6, rho0, obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER,
                  nthreads=1, want_final=False)
        out = shards.combine(r, end - first, shards.torch_all_reduce_sum())
        if rank == 0:
            result_q.put({k: out[k] for k in shards.OBS_KEYS} | {"n_traj": out["n_traj"]})
        dist.barrier()
    except RuntimeError as e:
        result_q.put({"rank": rank, "error": str(e)})
    finally:
        dist.destroy_process_group()


def _run_world(ws, B, seed, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, B, seed, q, fail_rank)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    outs = []
    while not q.empty():
        outs.append(q.get())
    return outs, [p.exitcode for p in procs]


def test_two_rank_shards_equal_the_whole_ensemble():
    from fermiphasespace_b200 import configs
    from oracle import oracle as O
    B, seed = 13, 4
    outs, codes = _run_world(2, B, seed)
    assert codes == [0, 0], outs
    got = [o for o in outs if "niiu" in o][0]
    assert got["n_traj"] == B
    w = configs.grid_3x2()
    rho0 = O.sample(w.n, B, seed, w.occ_up, w.occ_dn)
    sysm = O.System(tM=w.tM, U=w.U, V=w.V, coulomb=O.COUL_ONSITE, ext_null=True)
    ref = O.run(sysm, O.METHOD_FTWA, 0.01, 2, 6, rho0, obs=O.OBS_DIAG | O.OBS_DIAG2 | O.OBS_DOUB | O.OBS_ENER,
                nthreads=1, want_final=False)
    for k in shards.OBS_KEYS:
        assert np.abs(got[k] - ref[k]).max() < 1e-13, k


def test_sample_range_is_a_slice_of_the_ensemble():
    from fermiphasespace_b200 import configs
    from oracle import oracle as O
    w = configs.grid_3x2()
    whole = O.sample(w.n, 10, 9, w.occ_up, w.occ_dn)
    part = O.sample(w.n, 4, 9, w.occ_up, w.occ_dn, first=5)
    assert np.array_equal(whole[5:9], part)


def test_a_failed_rank_ends_the_job_with_an_error():
    """Rank 1 raises before the all_reduce; rank 0's collective must end with an
    error (gloo timeout or a closed peer), not hang."""
    outs, codes = _run_world(2, 8, 1, fail_rank=1)
    assert any(o.get("rank") == 1 and "failed" in o.get("error", "") for o in outs)
    assert all(c is not None for c in codes)
    assert not any("niiu" in o for o in outs)


# ---- the native exchange of sharded `fps` runs (C++ host layer, TCP, no GPU needed)

def test_native_shard_range_equals_python_split():
    from fermiphasespace_b200 import build, hostlib
    build.build_host()
    for B in (1, 7, 16, 1000, 1001, 16384):
        for ws in (1, 2, 3, 8):
            for r in range(ws):
                assert hostlib.shard_range(B, r, ws) == shards.shard_range(B, r, ws), (B, ws, r)


def _sum_worker(rank, ws, port, result_q, skip_ranks):
    from fermiphasespace_b200 import hostlib
    if rank in skip_ranks:
        result_q.put((rank, "skipped"))
        return
    data = np.arange(7, dtype=np.float64) * (rank + 1) + 0.1 * rank
    try:
        out = hostlib.shard_sum(data, rank, ws, port, timeout_s=3.0 if skip_ranks else 30.0)
        result_q.put((rank, out))
    except RuntimeError as e:
        result_q.put((rank, "error: " + str(e)))


def test_native_shard_sum_three_ranks_rank_order():
    ws, port = 3, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sum_worker, args=(r, ws, port, q, ())) for r in range(ws)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
    want = np.zeros(7)
    for r in range(ws):                      # the sum in rank order, as rank 0 forms it
        want = want + (np.arange(7, dtype=np.float64) * (r + 1) + 0.1 * r)
    for r in range(ws):
        assert isinstance(got[r], np.ndarray), got[r]
        assert np.array_equal(got[r], want), r


@pytest.mark.parametrize("missing", [1, 0], ids=["peer_never_arrives", "rank0_never_listens"])
def test_native_shard_sum_missing_rank_ends_with_an_error(missing):
    """A rank that never joins: the others give up at their deadline with an error
    (no hang), whichever side is missing."""
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sum_worker, args=(r, ws, port, q, (missing,))) for r in range(ws)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
    other = 1 - missing
    assert got[missing] == "skipped"
    assert isinstance(got[other], str) and got[other].startswith("error:") and "timed out" in got[other], got[other]
