"""The N > 1 bench path on CPU: two gloo ranks run the whole-job reduction of independent
replicas (max of the device times, sum of the event counts) and the reference arm prints from
rank 0 only."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import datetime

    import torch
    sys.path.insert(0, str(ROOT))
    import bench
    torch.distributed.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                         world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_ms = [12.5, 30.25][rank]
        out = bench.reduce_over_ranks(t_ms, events=100 * (rank + 1), spikes=7 + rank, device="cpu")
        results[rank] = out
    finally:
        torch.distributed.destroy_process_group()


def test_replica_reduction_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(results) == {0: (30.25, 300, 15), 1: (30.25, 300, 15)}


def _shard_rank(rank, world, port, results):
    import datetime

    import numpy as np
    import torch
    sys.path.insert(0, str(ROOT))
    import bench
    import bsnn
    torch.distributed.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                         world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        full = bsnn.config4_batch(24, steps=50, seed=5)
        mine = bench.shard_of(len(full.instances), rank, world)
        part = full.subset(mine)
        # what the shard would report: a per-instance count that identifies the instance
        counts = np.array([[i.seed % 1000, i.seed % 7] for i in part.instances])
        gathered = bench.gather_instance_counts(counts, mine, len(full.instances), "cpu")
        results[rank] = (mine, [i.seed for i in part.instances], gathered.tolist())
    finally:
        torch.distributed.destroy_process_group()


def test_batch_sharding_two_gloo_ranks():
    """The batched workload over two ranks: the shards' instances are disjoint, their union is the
    one-GPU spec (same seeds, parameters and weight sets), and the single all-reduce at the end gives
    every rank every instance's counts at its global index."""
    import numpy as np

    import bsnn
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(results)
    full = bsnn.config4_batch(24, steps=50, seed=5)
    seeds = {}
    for r in range(2):
        mine, shard_seeds, _ = res[r]
        seeds.update(zip(mine, shard_seeds))
    assert sorted(res[0][0] + res[1][0]) == list(range(24)) and not set(res[0][0]) & set(res[1][0])
    assert [seeds[b] for b in range(24)] == [i.seed for i in full.instances]
    want = np.array([[i.seed % 1000, i.seed % 7] for i in full.instances])
    for r in range(2):
        np.testing.assert_array_equal(np.array(res[r][2]), want)
    part = full.subset([3, 1])
    for k, b in enumerate((3, 1)):
        a, c = part.instance_network(k), full.instance_network(b)
        assert a.groups == c.groups and a.rng_seed == c.rng_seed
        for x, y in zip(a.conns, c.conns):
            np.testing.assert_array_equal(x.weights, y.weights)


@pytest.mark.parametrize("rank,expect_line", [(0, True), (1, False)])
def test_reference_arm_prints_on_rank_zero_only(rank, expect_line):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    if rank != 0:
        res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                             env=env, capture_output=True, text=True, timeout=120)
        assert res.returncode == 0 and res.stdout.strip() == ""
    else:
        # rank 0 runs the bounded CPU sample (no GPU here); keep it short
        res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                              "--workload", "small_plastic_500", "--cpu-seconds", "0.5"],
                             env=env, capture_output=True, text=True, timeout=300)
        assert res.returncode == 0, res.stderr[-2000:]
        import json
        line = json.loads(res.stdout.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"


def _undefined_names(path):
    """Names that a function of `path` reads as globals but that neither the module nor the
    builtins define (what a linter reports as an undefined name)."""
    import builtins
    import symtable
    src = path.read_text()
    top = symtable.symtable(src, str(path), "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()
               or s.is_namespace()} | set(dir(builtins))
    missing = []

    def walk(table):
        for child in table.get_children():
            if child.get_type() == "function":
                for s in child.get_symbols():
                    if s.is_global() and s.is_referenced() and s.get_name() not in defined:
                        missing.append(f"{child.get_name()}: {s.get_name()}")
            walk(child)
    walk(top)
    return missing


_PY_FILES = sorted(["bench.py", "__graft_entry__.py"]
                   + [str(p.relative_to(ROOT)) for d in ("example-cuda-spiking-nn_b200/bsnn", "oracle", "tests",
                                                         "tests/golden") for p in (ROOT / d).glob("*.py")])


@pytest.mark.parametrize("name", _PY_FILES)
def test_no_undefined_names(name):
    """The bench and most of the package run only on a GPU, so a name left undefined by an edit
    would first show there; catch it here."""
    assert _undefined_names(ROOT / name) == []
