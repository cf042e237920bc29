"""Rank body of the two-process ensemble test (gloo, CPU): the host path of
bench.py's multi-GPU run, with the oracle standing in for the GPU solve."""
import os

import numpy as np


def member_sizes(n):
    rng = np.random.default_rng(7)
    return [int(x) for x in rng.integers(300, 2500, n)]


def solve_member(k, size, steps):
    import efdc_xm as X
    import oracle as O
    import scenario as S
    scn = S.config3_member(k, size, seed=5)
    orc = O.Oracle(scn.grid)
    st = scn.copy_state()
    iters = 0
    for n in range(1, steps + 1):
        iters += orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st).iters_total
    orc.close()
    return {"cells": scn.ncell, "iters": iters, "p_sum": float(st["p"][1:scn.la].sum())}


def run(rank, world, port, nmembers, steps, out_dir):
    import torch.distributed as dist
    import ensemble as E
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    sizes = member_sizes(nmembers)
    parts = E.partition(sizes, world)
    local = {k: solve_member(k, sizes[k], steps) for k in parts[rank]}
    work = sum(v["cells"] * v["iters"] for v in local.values())
    allm = E.gather_members(local, nmembers)
    tot, = E.sum_over_ranks([work])
    mx, = E.max_over_ranks([float(rank + 1)])
    if rank == 0:
        import json
        with open(os.path.join(out_dir, "result.json"), "w") as f:
            json.dump({"members": allm, "work": tot, "max": mx, "parts": parts}, f)
    dist.barrier()
    dist.destroy_process_group()
