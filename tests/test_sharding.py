"""Multi-GPU plumbing on the host: world-size-2 gloo process groups on CPU.

Shards cover every item once, BFV shards keep response groups whole, the
maximum over ranks is what every rank sees, and Paillier-Lookup decode
results computed shard by shard (with the CPU oracle standing in for each
GPU) and gathered in rank order equal the unsharded results."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from cuhepy_b200.sharding import group_shard_bounds, gather_in_rank_order, max_over_ranks, shard_bounds


def test_shard_bounds_cover_each_item_once():
    for total in (0, 1, 7, 65536, 1000003):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def test_group_shards_keep_response_groups_whole():
    for tiles, padded in ((1024, 512), (1025, 512), (3, 512), (1024, 256), (4096, 512)):
        for world in (1, 2, 3, 8):
            spans = [group_shard_bounds(tiles, padded, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == tiles
            for lo, hi in spans:
                assert lo % padded == 0 or lo == hi == tiles      # empty shards sit at the end
                assert hi % padded == 0 or hi == tiles


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import random
        import sys

        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from conftest import hx, load_golden
        from oracle import paillier as oracle

        data = load_golden("lookup_512.json")
        pk = {k: hx(v) for k, v in data["pk"].items()}
        keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
        rng = random.Random(5)
        items = [rng.randrange(pk["n_squared"]) for _ in range(9)]
        lo, hi = shard_bounds(len(items), rank, world)
        local = [oracle.decode_distance([oracle.lookup_decrypt(c, keys)], data["key_len"]) for c in items[lo:hi]]
        gathered = gather_in_rank_order(local, dist)
        slowest = max_over_ranks(1.0 + rank, dist)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"gathered": gathered, "max": slowest, "items": [str(c) for c in items]}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_unsharded_result(tmp_path):
    import json

    from conftest import hx, load_golden
    from oracle import paillier as oracle

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    data = load_golden("lookup_512.json")
    pk = {k: hx(v) for k, v in data["pk"].items()}
    keys = {"pk": pk, "sk": {k: hx(v) for k, v in data["sk"].items()}}
    results = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    items = [int(c) for c in results[0]["items"]]
    whole = [oracle.decode_distance([oracle.lookup_decrypt(c, keys)], data["key_len"]) for c in items]
    for r in results:
        assert r["gathered"] == whole
        assert r["max"] == float(world)
