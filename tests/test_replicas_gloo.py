"""Multi-GPU host logic of bench.py on CPU: two ranks over gloo (127.0.0.1).

The path has no exchange step (frames are independent), so N GPUs run N
replicas: each rank takes its own frames, the timed region is bracketed by
barriers, the whole-job rate uses the maximum device time over ranks, and the
reference arm runs on rank 0 only. These are the collective steps bench.py takes
under torchrun; here they run on gloo with fake per-rank timings."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import datetime

    sys.path.insert(0, ROOT)
    import bench
    from turboransac_b200 import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cpu = torch.device("cpu")
    frames = 8
    mine = scenes.batched_frames(frames, first=rank * frames)  # the rank's replica slice, as bench.main takes it
    seeds = torch.tensor([f.seed & 0x7FFFFFFFFFFFFFFF for f in mine], dtype=torch.int64)
    allseeds = [torch.zeros_like(seeds) for _ in range(world)]
    dist.all_gather(allseeds, seeds)
    bench.barrier(dist)
    local_ms = 100.0 * (rank + 1)              # fake device time of this rank's steps
    total_ms = bench.max_over_ranks(dist, local_ms, cpu)
    value = world * frames * 3 / (total_ms / 1000.0)
    bench.barrier(dist)

    class A:  # the reference arm's arguments
        frames, warmup, steps, gpus = 4, 0, 1, world
    ref_ret = bench.run_reference(A, world, rank) if rank != 0 else None
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as fh:
        flat = sorted(int(s) for t in allseeds for s in t.tolist())
        fh.write(f"{total_ms} {value} {len(set(flat))} {len(flat)} {ref_ret}\n")
    dist.destroy_process_group()


def test_two_rank_replicas_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    lines = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    for total_ms, value, uniq, n, ref_ret in lines:
        assert float(total_ms) == 200.0                         # max over ranks, seen by every rank
        assert abs(float(value) - 2 * 8 * 3 / 0.2) < 1e-9       # whole-job frames / slowest rank's time
        assert int(uniq) == int(n) == 16                        # disjoint replica frames
        assert ref_ret == "None"                                # reference arm: rank 1 does no work
