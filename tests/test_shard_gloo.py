"""Multi-rank screening path on CPU: two gloo ranks each screen their own
contiguous step range (the oracle stands in for the GPU) and the stitched
result equals the unsharded screen; the timing reduction is a max over
ranks."""

import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

import cases


def _worker(rank, world, port, outdir):
    import torch
    import torch.distributed as dist

    import oracle
    from mizuba_b200.shard import max_over_ranks, step_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pj = cases.random_linear_pj(80, seed=17, box=6.0, speed=10.0)
        full = oracle.run(pj, 1.0, 0.05, n_threads=1)
        b, e = step_range(rank, world, full["n_cd_steps"])
        part = oracle.run(pj, 1.0, 0.05, step_begin=b, step_end=e, n_threads=1)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), b=b, e=e, aabbs=part["aabbs"],
                 srt_idx=part["srt_idx"], conj=part["conjunctions"].view(np.uint8),
                 bp=np.concatenate([x.view(np.uint8) for x in part["bp"]] + [np.zeros(0, np.uint8)]))
        t = max_over_ranks(float(rank + 1))
        assert t == float(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_unsharded_screen():
    import oracle

    world = 2
    port = 29500 + (os.getpid() % 2000)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, port, d), nprocs=world, join=True, start_method="spawn")
        pj = cases.random_linear_pj(80, seed=17, box=6.0, speed=10.0)
        full = oracle.run(pj, 1.0, 0.05, n_threads=1)
        parts = [np.load(os.path.join(d, f"r{r}.npz")) for r in range(world)]
    assert parts[0]["b"] == 0 and parts[0]["e"] == parts[1]["b"] and parts[1]["e"] == full["n_cd_steps"]
    assert np.array_equal(np.concatenate([p["aabbs"] for p in parts]), full["aabbs"])
    assert np.array_equal(np.concatenate([p["srt_idx"] for p in parts]), full["srt_idx"])
    assert np.array_equal(np.concatenate([p["conj"] for p in parts]), full["conjunctions"].view(np.uint8))
    bp_full = np.concatenate([x.view(np.uint8) for x in full["bp"]])
    assert np.array_equal(np.concatenate([p["bp"] for p in parts]), bp_full)


@pytest.mark.parametrize("n,world", [(480, 1), (480, 2), (480, 8), (7, 3), (3, 4)])
def test_step_ranges_partition(n, world):
    from mizuba_b200.shard import step_range

    rs = [step_range(r, world, n) for r in range(world)]
    assert rs[0][0] == 0 and rs[-1][1] == n
    assert all(rs[k][1] == rs[k + 1][0] for k in range(world - 1))
    assert max(e - b for b, e in rs) - min(e - b for b, e in rs) <= 1
