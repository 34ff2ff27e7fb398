"""CPU: the cross-rank sharding of a volume batch with 2 gloo ranks.

Each rank segments its share of a small batch with the CPU checker (standing in for
the GPU, which this test does not need) and the job figures are combined with the
same collectives bench.py uses; the union of the shards must be the whole batch,
disjoint, and the combined result must equal a single-process run."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import sys

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    shard = importlib.import_module("3dimagetoolkit_b200.shard")
    synth = importlib.import_module("3dimagetoolkit_b200.synth")
    import oracle_py as O

    shapes = [(10, 9, 8), (8, 8, 8), (12, 7, 9), (9, 11, 8), (7, 8, 10)]
    mine = shard.volume_shard(len(shapes), rank, world)
    vox_iters = 0.0
    p = O.default_params(sigma=1.5, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=3, tol=0.0, bc=2,
                         ls_steps=1)
    for q in mine:
        u0 = synth.ellipsoids(shapes[q], q, n=1, semi_axes=(2, 3))
        r = O.rsfe_apply(u0, synth.sphere_phi0(shapes[q], 3.0), p)
        np.save(os.path.join(out_dir, f"phi{q}.npy"), r["phi"])
        vox_iters += u0.size * r["stats"]["iterations"]
    total, secs = shard.job_throughput(vox_iters, 1.0 + rank)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array([total, secs, len(mine)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_the_batch(tmp_path, pkg, O):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    shard = importlib.import_module("3dimagetoolkit_b200.shard")
    shapes = [(10, 9, 8), (8, 8, 8), (12, 7, 9), (9, 11, 8), (7, 8, 10)]
    parts = [shard.volume_shard(len(shapes), r, world) for r in range(world)]
    assert sorted(sum(parts, [])) == list(range(len(shapes)))
    totals = [np.load(tmp_path / f"rank{r}.npy") for r in range(world)]
    want_total = sum(np.prod(s) * 3 for s in shapes)
    for t in totals:
        assert t[0] == want_total and t[1] == 2.0
    p = O.default_params(sigma=1.5, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=3, tol=0.0, bc=2,
                         ls_steps=1)
    for q, s in enumerate(shapes):
        u0 = pkg.synth.ellipsoids(s, q, n=1, semi_axes=(2, 3))
        want = O.rsfe_apply(u0, pkg.synth.sphere_phi0(s, 3.0), p)["phi"]
        assert np.array_equal(np.load(tmp_path / f"phi{q}.npy"), want)


def test_shard_rejects_bad_rank():
    shard = importlib.import_module("3dimagetoolkit_b200.shard")
    with pytest.raises(ValueError):
        shard.volume_shard(4, 2, 2)
