"""Ensembles over several ranks: member partition and the host-side
collectives of a multi-GPU run (gloo, world size 2, CPU)."""
import json
import socket

import numpy as np
import pytest

import dist_worker as W
import ensemble as E
import scenario as S


def test_partition_covers_and_balances():
    sizes = S.config3_sizes(seed=3, members=256)
    for nr in (1, 2, 4, 8):
        parts = E.partition(sizes, nr)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(256))
        assert E.imbalance(sizes, parts) < 1.01
        assert parts == E.partition(sizes, nr)  # deterministic
    assert E.partition([5, 1, 1], 4)[3] == []


def test_partition_rejects_bad_rank_count():
    with pytest.raises(ValueError):
        E.partition([1, 2], 0)


def test_gather_single_process():
    out = E.gather_members({1: "b", 0: "a"}, 2)
    assert out == ["a", "b"]
    with pytest.raises(RuntimeError):
        E.gather_members({0: "a"}, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    nm, steps = 6, 2
    mp.start_processes(W.run, args=(2, _free_port(), nm, steps, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    res = json.loads((tmp_path / "result.json").read_text())
    sizes = W.member_sizes(nm)
    # every member solved once, on the rank the partition gave it, and equal
    # to the same member solved in this process
    assert sorted(k for p in res["parts"] for k in p) == list(range(nm))
    for k in (0, nm - 1):
        ref = W.solve_member(k, sizes[k], steps)
        assert res["members"][k] == ref
    assert res["work"] == sum(m["cells"] * m["iters"] for m in res["members"])
    assert res["max"] == 2.0
