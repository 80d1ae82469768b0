"""The multi-rank path on CPU: two gloo ranks shard a job's spectra, agree on
the max-over-ranks time and merge their per-spectrum results on rank 0 --
the same calls bench.py and the service make over NCCL on GPUs."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from prestozl_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    env = replicas.rank_env()
    ids = list(range(7))
    mine = replicas.shard(ids, env.rank, env.world)
    # each rank "searches" its spectra: results keyed by spectrum id
    local = {i: [(float(i), env.rank)] for i in mine}
    t = replicas.max_over_ranks(10.0 + env.rank, dist)
    merged = replicas.gather_results(local, dist)
    q.put((env.rank, mine, t, merged))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_time_and_merge():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, mine, t, merged = q.get(timeout=120)
        out[r] = (mine, t, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out[0][0] + out[1][0]) == list(range(7))
    assert not set(out[0][0]) & set(out[1][0])
    assert out[0][1] == out[1][1] == 11.0
    merged = out[0][2]
    assert sorted(merged) == list(range(7))
    assert all(merged[i][0][1] == i % 2 for i in range(7))
    assert out[1][2] is None


def test_rstep_ranges_cover_a_spectrum():
    for n, w in ((23364, 8), (5, 8), (100, 3)):
        rr = replicas.rstep_ranges(n, w)
        assert sum(c for _, c in rr) == n
        assert all(rr[i][0] + rr[i][1] == rr[i + 1][0] for i in range(w - 1))


def _dedisp_worker(rank, world, port, q, numdms=11):
    import datetime

    import numpy as np
    import torch.distributed as dist

    from oracle import bindings as ob

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    env = replicas.rank_env()
    rng = np.random.default_rng(5)  # every rank reads the same subband blocks
    worklen, nsub = 500, 12
    cur = rng.standard_normal((worklen, nsub)).astype(np.float32)
    last = rng.standard_normal((worklen, nsub)).astype(np.float32)
    off = rng.integers(0, worklen + 1, (numdms, nsub)).astype(np.int32)
    first, count = replicas.dm_ranges(numdms, env.world)[env.rank]
    # a rank without trials (more ranks than DMs) dedisperses nothing
    rows = ob.dedisp_subbands(cur, last, off[first:first + count]) if count else []
    local = {first + i: [rows[i].tobytes()] for i in range(count)}
    merged = replicas.gather_results(local, dist)
    full = ob.dedisp_subbands(cur, last, off) if env.rank == 0 else None
    ok = None
    if env.rank == 0:
        ok = sorted(merged) == list(range(numdms)) and all(
            merged[d][0] == full[d].tobytes() for d in range(numdms))
    q.put((env.rank, (first, count), ok))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,numdms", [(2, 11), (3, 2)])
def test_gloo_ranks_split_dm_trials(world, numdms):
    """Dedispersion over several ranks: each takes a contiguous range of the
    DM trials (replicas.dm_ranges) over the same subband blocks, with no data
    exchange; the trials merged on rank 0 equal the one-rank result bit for
    bit.  With more ranks than DMs the rank left without trials searches
    nothing and still joins the gather.  (The oracle's dedispersion stands in
    for each rank's GPU.)"""
    from tests import helpers as H

    H.ensure_oracle()
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dedisp_worker, args=(r, world, port, q, numdms))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, rng_, ok = q.get(timeout=120)
        out[r] = (rng_, ok)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [out[r][0] for r in range(world)] == replicas.dm_ranges(numdms, world)
    assert out[0][1] is True
    assert replicas.dm_ranges(3, 4) == [(0, 1), (1, 1), (2, 1), (3, 0)]


def _split_worker(rank, world, port, q, workdir, first, count):
    import datetime

    import torch.distributed as dist

    from prestozl_b200 import jerk
    from tests import helpers as H

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    os.makedirs(os.path.join(workdir, f"rank{rank}"), exist_ok=True)
    pb = H.small_problem(os.path.join(workdir, f"rank{rank}"))
    obs = jerk.obs_from_refobs(pb.obs)
    searched = []

    def search(f, n):
        searched.append((f, n))
        _, _, keys, pows = pb.oracle.search_hits(f, n)
        return keys, pows

    merged = replicas.split_search(search, obs, pb.subs[0], first, count, dist)
    res = None
    if rank == 0:
        whole = replicas.split_search(search, obs, pb.subs[0], first, count, None)
        orc, done, _ = pb.oracle.search(first, count)
        res = (merged, whole, orc, list(pb.obs.powcut))
    q.put((rank, searched[:1], res))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,first,count", [(2, 0, 48), (3, 4, 9)])
def test_gloo_ranks_split_one_spectrum_and_merge_in_order(world, first, count, tmp_path):
    """One spectrum searched by several ranks: each takes a contiguous share
    of the rsteps (replicas.rstep_ranges) and returns its raw hits; rank 0
    merges them in the reference's insertion order (sort by key, then the
    ordered insertion, jerk_merge_hits).  The merged list equals, bit for
    bit, the list from one rank's hits over the whole range, and equals the
    oracle's own list of that range (except within 1e-4 of a cutoff; powers
    and sigmas to 1e-5).  The oracle's search stands in for each rank's GPU."""
    from tests import helpers as H

    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q, str(tmp_path), first,
                                                     count)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, searched, res = q.get(timeout=300)
        out[r] = (searched, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ranges = replicas.rstep_ranges(count, world)
    for r in range(world):
        assert out[r][0] == [(first + ranges[r][0], ranges[r][1])]
    merged, whole, orc, powcut = out[0][1]
    assert len(merged) > 0
    assert len(merged) == len(whole)
    for f in merged.dtype.names:  # field by field (the records carry padding)
        assert np.array_equal(merged[f], whole[f]), f
    probs = H.compare_cands(merged, orc, powcut)
    assert not probs, probs[:10]
