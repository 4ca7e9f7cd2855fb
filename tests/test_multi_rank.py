"""Multi-GPU host logic on CPU: the C ABI's slab partition (the reference's
contiguous ceil(n/ngpus) split) and, with two gloo ranks, the benchmark's
distributed pieces (per-rank distinct inputs, max-over-ranks timing)."""
import os
import socket
import sys

import numpy as np
import pytest


def part(n, g):
    from sscRaft.rafttypes import libraft, _ptr
    st = np.zeros(g, np.int32)
    ct = np.zeros(g, np.int32)
    assert libraft.raft_slab_partition(n, g, _ptr(st), _ptr(ct)) == 0
    return st, ct


@pytest.mark.parametrize("n,g", [(512, 1), (512, 8), (7, 3), (2, 4), (0, 2), (1000, 7)])
def test_slab_partition_covers_once(n, g):
    st, ct = part(n, g)
    sub = -(-n // g) if n else 0
    assert ct.sum() == n and np.all(ct >= 0) and np.all(ct <= sub)
    covered = np.concatenate([np.arange(s, s + c) for s, c in zip(st, ct)]) if n else np.array([])
    np.testing.assert_array_equal(covered, np.arange(n))
    # reference rule: full slabs first, then the remainder, then empty ones
    nz = ct[ct > 0]
    assert np.all(nz[:-1] == sub)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    t = bench.max_over_ranks(10.0 + rank)          # slowest rank decides the step time
    seeds = bench.slice_seed_base(rank, 512)
    out.put((rank, t, seeds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_timing_and_seeds():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[0][2] + 512 <= res[1][2]               # disjoint per-rank slice seeds


def _slab_worker(rank, world, port, out):
    """One rank of a slab-split reconstruction: its slices (the C ABI's slab
    partition), reconstructed by the FP64 oracle standing in for the rank's
    GPU, gathered on every rank."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in ("ssc-raft_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(root, p))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from helpers import sino_case
    n, N, A = 5, 48, 40
    sino, ang = sino_case(N, A, n, seed=77)
    st, ct = part(n, world)
    mine = oracle.fbp(sino[st[rank]:st[rank] + ct[rank]], ang, oracle.MODE_LIN, 5, 2) if ct[rank] else \
        np.zeros((0, N, N))
    parts = [None] * world
    dist.all_gather_object(parts, (int(st[rank]), mine))
    vol = np.zeros((n, N, N))
    for s0, blk in parts:
        vol[s0:s0 + len(blk)] = blk
    out.put((rank, vol))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_slab_split_reconstruction_equals_whole():
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle
    from helpers import sino_case
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sino, ang = sino_case(48, 40, 5, seed=77)
    whole = oracle.fbp(sino, ang, oracle.MODE_LIN, 5, 2)
    for _, vol in res:
        np.testing.assert_array_equal(vol, whole)


def test_bench_inputs_do_not_import_the_package():
    """The reference arm makes its inputs with synthetic.py loaded by path, so
    that process maps no library of this repository."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r); import bench; S = bench.synthetic_module(); "
            "S.ellipse_params(1, 3); assert 'sscRaft' not in sys.modules, sorted(sys.modules)" % root)
    subprocess.run([sys.executable, "-c", code], check=True, timeout=120)
