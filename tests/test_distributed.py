"""Multi-rank sample sharding and film reduction on CPU (gloo, world size 2),
with the oracle as the per-rank renderer."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from xyz_b200.distributed import sample_range, weak_range


def test_sample_ranges_cover_every_sample_once():
    for total in (1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, n = sample_range(total, r, world)
                seen.extend(range(a, a + n))
            assert seen == list(range(total))
    assert weak_range(64, 3) == (192, 64)
    with pytest.raises(ValueError):
        sample_range(8, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir, fail_rank):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from tests.helpers import ensure_port
    from xyz_b200 import scenes
    from xyz_b200.distributed import render_and_reduce, sample_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        sd = scenes.cornell_box()
        P = ensure_port()
        P.scene_create(sd)
        P.set_camera(sd.camera, 24, 16)
        P.set_path_params(max_depth=6)
        if rank == fail_rank:
            raise SystemExit(3)  # this rank leaves before the reduce
        a, n = sample_range(6, rank, world)
        film = render_and_reduce(lambda f, c: torch.from_numpy(P.render(c, seed=5, s0=f, nthreads=1)), a, n)
        if rank == 0:
            np.save(os.path.join(out_dir, "film.npy"), film.numpy())
    except RuntimeError as e:
        with open(os.path.join(out_dir, f"error{rank}.txt"), "w") as f:
            f.write(str(e))
    finally:
        if dist.is_initialized() and rank != fail_rank:
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def test_two_ranks_reduce_to_the_single_process_image(tmp_path):
    from tests.helpers import ensure_port
    from xyz_b200 import scenes
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), -1)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    film = np.load(tmp_path / "film.npy")
    sd = scenes.cornell_box()
    P = ensure_port()
    P.scene_create(sd)
    P.set_camera(sd.camera, 24, 16)
    P.set_path_params(max_depth=6)
    ref = P.render(6, seed=5, nthreads=1)
    # the same samples, summed in two groups: equal up to float association
    assert np.allclose(film, ref, rtol=1e-5, atol=1e-6)


def test_a_rank_that_leaves_is_reported_not_waited_for(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), 1)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert procs[1].exitcode == 3
    # rank 0's reduce fails with an error instead of hanging
    assert procs[0].exitcode == 0
    assert (tmp_path / "error0.txt").exists()


def test_jobs_assigned_by_cost_once_each_and_balanced():
    from xyz_b200 import scenes
    from xyz_b200.distributed import assign_by_cost, job_cost
    work = [(e.scene.n_tris, e.width, e.height, e.spp) for e in scenes.batch_workload(16)]
    costs = [job_cost(*w) for w in work]
    for world in (1, 2, 3, 8):
        parts = assign_by_cost(costs, world)
        assert sorted(j for p in parts for j in p) == list(range(len(costs)))
        loads = [sum(costs[j] for j in p) for p in parts]
        # longest-first greedy: no rank exceeds the mean by more than one job
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
        assert parts == assign_by_cost(costs, world)
    assert assign_by_cost([5.0, 1.0, 4.0, 2.0], 2) == [[0, 1], [2, 3]]
    with pytest.raises(ValueError):
        assign_by_cost([1.0], 0)


class _FakeGuide:
    """Stands in for api.Guide on CPU: a parameter vector."""

    def __init__(self, p):
        self.p = np.asarray(p, np.float32)

    def params(self):
        return self.p.copy()

    def set_params(self, p):
        self.p = np.asarray(p, np.float32).copy()


def _guide_worker(rank, world, port, out_dir):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from xyz_b200.distributed import broadcast_guide
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        g = _FakeGuide(np.full(28992, float(rank + 1), np.float32) * np.arange(28992, dtype=np.float32))
        broadcast_guide(g, src=0)
        np.save(os.path.join(out_dir, f"params{rank}.npy"), g.p)
    finally:
        dist.destroy_process_group()


def test_guide_weights_broadcast_from_the_training_rank(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_guide_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    p0, p1 = np.load(tmp_path / "params0.npy"), np.load(tmp_path / "params1.npy")
    assert np.array_equal(p0, np.arange(28992, dtype=np.float32))
    assert np.array_equal(p1, p0)
