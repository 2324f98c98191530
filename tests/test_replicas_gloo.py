"""The multi-rank path on CPU: two gloo ranks run independent replicas of the
matcher (the oracle stands in for the device on a host without a GPU), each
on its own pairs, and reduce only their timing: the slowest rank sets the
job's time and the rate counts every rank's pairs."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world_size, port, out_dir):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from nx_stereo_b200 import replicas
    from oracle import oracle

    replicas.init("gloo", rank=rank, world_size=world_size,
                  init_method=f"tcp://127.0.0.1:{port}", timeout_s=60)
    left, right = oracle.scene(64, 48, replicas.seed(rank, 0))
    disparity = oracle.fast_sgm(left, right, 64, 8)
    replicas.barrier()
    seconds = 0.5 + 0.25 * rank  # the ranks' timed regions, as they measured them
    slowest = replicas.max_over_ranks(seconds)
    rate = replicas.whole_job_rate(10, world_size, slowest)
    # A loop whose length rank 0 decides (the end-to-end loop's rounds): every
    # rank takes as many rounds as rank 0, whatever its own flag says.
    rounds = 0
    while True:
        rounds += 1
        if not replicas.agree(rounds < 3 if rank == 0 else rounds < 10):
            break
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), disparity)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{slowest} {rate} {rounds}")
    replicas.barrier()
    import torch.distributed as dist

    dist.destroy_process_group()


def test_two_gloo_ranks_run_independent_replicas_and_reduce_only_time(tmp_path, oracle):
    import torch.multiprocessing as mp

    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    results = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]
    assert all(float(slowest) == 0.75 for slowest, _, _ in results)
    assert all(float(rate) == pytest.approx(20 / 0.75) for _, rate, _ in results)
    assert [int(rounds) for _, _, rounds in results] == [3, 3]
    from nx_stereo_b200 import replicas

    outputs = [np.load(tmp_path / f"rank{r}.npy") for r in range(2)]
    assert not np.array_equal(outputs[0], outputs[1])  # each rank had its own pairs
    for r in range(2):
        left, right = oracle.scene(64, 48, replicas.seed(r, 0))
        assert np.array_equal(outputs[r].view(np.uint32),
                              oracle.sgm(left, right, 64, 8).view(np.uint32))
