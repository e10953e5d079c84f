"""The N>1 path on CPU: world-size-2 gloo ranks split a K range, each
accumulates its reports' hash with the library's ReportSolution, the
partials are all-gathered and merged -- the result must equal a single
process over the whole range.  The reports come from the reference's own
raw-report fixtures, so no GPU is involved."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import GOLDEN, ref_raw

from ap26_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _available_ks():
    d = os.path.join(GOLDEN, "ref_raw", "shift0")
    return sorted(int(f[:-4]) for f in os.listdir(d) if f.endswith(".txt"))


def _worker(rank, world, port, ks, out):
    import torch
    import ap26_b200 as A
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    a, b = replicas.split_range(0, len(ks) - 1, world, rank)
    r = A.Reporter()
    for K in ks[a:b + 1]:
        r.report_all(ref_raw(K))
    t = torch.tensor([r.hash.value], dtype=torch.int64)
    gathered = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(gathered, t)
    dev_ms = torch.tensor([float(10 + rank)], dtype=torch.float64)
    dist.all_reduce(dev_ms, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((replicas.merge_hash([g.item() for g in gathered]), dev_ms.item()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_split_merges_to_single_process_hash():
    ks = _available_ks()
    assert len(ks) >= 3
    single = __import__("ap26_b200").Reporter()
    for K in ks:
        single.report_all(ref_raw(K))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ks, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert merged == single.hash.value
    assert tmax == 11.0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_range_partitions_exactly(world):
    kmin, kmax = 43241056, 43241056 + 63
    seen = []
    for r in range(world):
        a, b = replicas.split_range(kmin, kmax, world, r)
        seen += list(range(a, b + 1))
    assert seen == list(range(kmin, kmax + 1))


def test_merge_hash_reduction_matches_sequential():
    vals = [1_999_999_000, 1_500, 2_000_000_000, 7]
    h = 0
    for v in vals:  # one process adding the same totals
        h += v
        if h > replicas.MAXINTV:
            h -= replicas.MAXINTV
    assert replicas.merge_hash(vals) == h
