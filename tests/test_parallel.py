"""Multi-process path on CPU (gloo, world size 2): instance sharding covers
the ensemble exactly once, per-rank tracking of the shards reproduces a
single-process run, and the timing/work reductions are max/sum."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from elegant_b200.parallel import reduce_timing, shard_instances


def test_shard_instances_partition():
    rng = np.random.default_rng(0)
    counts = rng.integers(500, 4001, size=37)
    offsets = np.concatenate([[0], np.cumsum(counts)])
    for world in (1, 2, 3, 8):
        seen = []
        sizes = []
        for r in range(world):
            i0, i1, local = shard_instances(offsets, r, world)
            seen += list(range(i0, i1))
            sizes.append(local[-1])
            assert local[0] == 0 and np.all(np.diff(local) == counts[i0:i1])
        assert seen == list(range(37))
        if world > 1:
            assert max(sizes) - min(sizes) <= 2 * counts.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from reforacle import PortOracle
    from elegant_b200 import Element, Lattice, workloads as w
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lat, beam, offsets, overrides = w.ensemble(n_instances=6, n_min=20, n_max=40, seed=3)
    i0, i1, _ = shard_instances(offsets, rank, world)
    oracle = PortOracle("b2e")
    work = 0.0
    results = {}
    for i in range(i0, i1):
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        sl = slice(offsets[i], offsets[i + 1])
        rows, nl, eff = oracle.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), 4)
        work += eff
        results[i] = rows
    t, total = reduce_timing(1.0 + rank, work, dist)
    gathered = [None] * world
    dist.all_gather_object(gathered, results)
    if rank == 0:
        merged = {}
        for g in gathered:
            merged.update(g)
        np.save(os.path.join(out_dir, "t.npy"), np.array([t, total]))
        np.save(os.path.join(out_dir, "rows.npy"), np.concatenate([merged[i] for i in range(6)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_run(tmp_path):
    from reforacle import PortOracle
    from elegant_b200 import Element, Lattice, workloads as w
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    t, total = np.load(tmp_path / "t.npy")
    assert t == 2.0
    rows = np.load(tmp_path / "rows.npy")
    lat, beam, offsets, overrides = w.ensemble(n_instances=6, n_min=20, n_max=40, seed=3)
    oracle = PortOracle("b2e")
    expect, work = [], 0.0
    for i in range(6):
        els = []
        for j, e in enumerate(lat.elements):
            params = dict(e.params)
            for (ie, name, vals) in overrides:
                if ie == j:
                    params[name] = float(vals[i])
            els.append(Element(e.name, e.type, params))
        sl = slice(offsets[i], offsets[i + 1])
        r, nl, eff = oracle.track(Lattice(els), beam.coords[sl], beam.ids[sl], w.ring_p_central(), 4)
        expect.append(r)
        work += eff
    assert total == work
    assert np.array_equal(rows, np.concatenate(expect))


def _keys_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from elegant_b200.parallel import (REDUCE_MAX_U64, REDUCE_MIN_U64, REDUCE_SUM_U32, REDUCE_SUM_U64,
                                       allreduce_keys_and_counts)
    # order-preserving keys: values with the top bit set compare above the others
    keys = np.array([[0x8000000000000005, 0x7FFFFFFFFFFFFFF0, 3], [0x8000000000000001, 0xFFFFFFFFFFFFFFFF, 9]],
                    dtype=np.uint64)[rank]
    t = torch.from_numpy(keys.view(np.int64).copy())
    allreduce_keys_and_counts(t, REDUCE_MIN_U64, dist)
    mn = t.numpy().view(np.uint64).tolist()
    t = torch.from_numpy(keys.view(np.int64).copy())
    allreduce_keys_and_counts(t, REDUCE_MAX_U64, dist)
    mx = t.numpy().view(np.uint64).tolist()
    c32 = torch.tensor([rank + 1, 10 * rank, 7], dtype=torch.int32)
    allreduce_keys_and_counts(c32, REDUCE_SUM_U32, dist)
    c64 = torch.tensor([2 ** 40 + rank], dtype=torch.int64)
    allreduce_keys_and_counts(c64, REDUCE_SUM_U64, dist)
    np.save(os.path.join(out_dir, f"keys{rank}.npy"), np.array([mn, mx], dtype=np.uint64))
    np.save(os.path.join(out_dir, f"counts{rank}.npy"), np.concatenate([c32.numpy(), c64.numpy()]).astype(np.int64))
    dist.destroy_process_group()


def test_csr_exchange_reductions_two_ranks(tmp_path):
    """The CSR exchange (a bunch spread over two ranks): unsigned min/max of
    order-preserving c*t keys and sums of histogram and particle counts."""
    port = _free_port()
    mp.start_processes(_keys_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        k = np.load(tmp_path / f"keys{r}.npy")
        assert k[0].tolist() == [0x8000000000000001, 0x7FFFFFFFFFFFFFF0, 3]
        assert k[1].tolist() == [0x8000000000000005, 0xFFFFFFFFFFFFFFFF, 9]
        c = np.load(tmp_path / f"counts{r}.npy")
        assert c.tolist() == [3, 10, 14, 2 ** 41 + 1]
