"""The N > 1 path of bench.py on CPU: two ranks over gloo.

bench.py --gpus N runs one process per GPU (torchrun), each a replica of the
workload (weak scaling, no collective on the data path); the ranks meet at a
barrier on both sides of the timed region and report the maximum time over
ranks.  These tests run that host logic as two CPU processes over gloo on
127.0.0.1: the rendezvous, the barrier, the max over ranks, and that only
rank 0 runs the reference arm.
"""
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


def _rank_main(rank, world, port, out_dir):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    ws, r, local = bench._dist_init()
    assert (ws, r, local) == (world, rank, rank)
    bench._barrier(ws)
    # each rank's "device time" differs; every rank must see the maximum
    m = bench._allmax(1.5 * (rank + 1), ws)
    bench._barrier(ws)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(repr(m))
    dist.destroy_process_group()


def test_two_ranks_meet_and_take_the_maximum(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [float(open(tmp_path / f"rank{r}.txt").read()) for r in range(2)]
    assert got == [3.0, 3.0]


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the other ranks return at once, without work."""
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        workload = "ot128"
    assert bench.run_reference(Args(), 2, 1) is None


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    saved = {k: os.environ.pop(k, None) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        assert bench._dist_init() == (1, 0, 0)
        assert bench._allmax(2.5, 1) == 2.5
        bench._barrier(1)
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
