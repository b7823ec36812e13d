"""The multi-GPU replica logic (yahmc_b200.replicas, used by bench.py under torchrun) on two
gloo ranks on the CPU: per-rank inputs differ, the timed region's duration is the maximum
over the ranks, the job time per solve divides it by the ranks, and a rank that leaves
before a barrier ends the other's barrier with an error instead of a hang."""
import datetime
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, mode):
    import torch
    import torch.distributed as dist
    from yahmc_b200 import fields, replicas
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    result = {}
    if mode == "normal":
        replicas.barrier(dist)
        result["max"] = replicas.max_over_ranks(1.0 + 0.5 * rank, dist)
        src = fields.gaussian_spinor(64, 3, np.random.default_rng(replicas.rank_seed(11, rank)))
        mine = torch.tensor([float(np.real(src.ravel()[0]))], dtype=torch.float64)
        got = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(got, mine)
        result["firsts"] = [float(g.item()) for g in got]
        result["job"] = replicas.job_time_per_solve(result["max"], world)
        replicas.barrier(dist)
        dist.destroy_process_group()
    else:                                   # rank 1 leaves without meeting the barrier
        if rank == 1:
            np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([0.0]))
            os._exit(0)
        try:
            replicas.barrier(dist)
            result["error"] = 0.0
        except Exception:
            result["error"] = 1.0
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.array([result.get("max", 0.0), result.get("job", 0.0), result.get("error", 0.0)]
                     + result.get("firsts", [])))


def _spawn(mode, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path), mode), nprocs=2, join=True,
                       start_method="spawn")
    return [np.load(tmp_path / f"r{r}.npy") for r in range(2)]


def test_two_rank_replicas(tmp_path):
    r0, r1 = _spawn("normal", tmp_path)
    for r in (r0, r1):
        assert r[0] == 1.5                  # max over ranks of 1.0 and 1.5
        assert r[1] == 0.75                 # two solves ran concurrently
        assert r[3] != r[4]                 # each rank solves its own source
    assert np.array_equal(r0[3:], r1[3:])


def test_rank_that_leaves_ends_the_barrier_with_an_error(tmp_path):
    r0, _ = _spawn("leave", tmp_path)
    assert r0[2] == 1.0


def test_helpers():
    from yahmc_b200 import replicas
    assert replicas.rank_seed(5, 0) != replicas.rank_seed(5, 1)
    assert replicas.max_over_ranks(3.25) == 3.25
    with pytest.raises(ValueError):
        replicas.job_time_per_solve(1.0, 0)

