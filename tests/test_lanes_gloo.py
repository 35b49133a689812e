"""Multi-GPU sharding, checked on the CPU with two gloo ranks.

bench.py --gpus N (under torchrun) gives rank r lane r of the tile range
(lane_range, the reference's --prefix-lanes split, v13:3533-3554), runs the
filter on it with no data exchange, and reduces only the elapsed time (max
over ranks).  Here each rank filters its lane with the oracle; the gathered
lanes must be disjoint, cover the range and together equal one filter pass
over the whole range, and the max-reduction must return the slowest rank's
time on every rank."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, t0, n_tiles, out_dir):
    import importlib
    import torch
    import torch.distributed as dist
    sys.path.insert(0, HERE)
    sys.path.insert(0, ROOT)
    import oracle_bind as ob
    ccs = importlib.import_module("cunningham-chain-search_b200")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lo, hi = ccs.lane_range(t0, t0 + n_tiles, world, rank)
    lat = ob.Lattice()
    surv = lat.filter_range(lo, hi - lo)
    # survivors in whole-range coordinates (tile index relative to t0)
    recs = sorted((int(b), int(k), int(t) + (lo - t0)) for b, k, t, _ in surv)
    gathered = [None] * world
    dist.all_gather_object(gathered, {"lane": (lo, hi), "recs": recs})
    ms = torch.tensor([10.0 + 5.0 * rank])
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    dist.barrier()
    if rank == 0:
        import json
        with open(os.path.join(out_dir, "lanes.json"), "w") as f:
            json.dump({"gathered": gathered, "max_ms": float(ms.item())}, f)
    else:
        assert float(ms.item()) == 10.0 + 5.0 * (world - 1)
    dist.destroy_process_group()


def test_two_rank_lanes_cover_the_range(ob, tmp_path):
    import json
    import torch.multiprocessing as mp
    world = 2
    t0 = (1 << 60) // (20677 * 1616615) + 4242
    n_tiles = 1501                                  # odd: the remainder goes to lane 0
    mp.start_processes(_rank_main, args=(world, _free_port(), t0, n_tiles, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    res = json.load(open(tmp_path / "lanes.json"))
    lanes = [tuple(g["lane"]) for g in res["gathered"]]
    assert lanes[0][0] == t0 and lanes[-1][1] == t0 + n_tiles
    assert all(lanes[i][1] == lanes[i + 1][0] for i in range(world - 1))
    assert lanes[0][1] - lanes[0][0] == n_tiles // world + 1
    merged = sorted(tuple(r) for g in res["gathered"] for r in g["recs"])
    whole = sorted((int(b), int(k), int(t)) for b, k, t, _ in ob.Lattice().filter_range(t0, n_tiles))
    assert merged == whole and len(whole) > 50
    assert res["max_ms"] == 10.0 + 5.0 * (world - 1)
