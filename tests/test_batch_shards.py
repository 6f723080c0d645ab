"""Splitting a batch of geometries over several GPUs (host logic, no GPU):
the work estimate, the longest-processing-time partition, and the host-side
gather of per-geometry results between two gloo ranks, with a stand-in for
the GPU batch that 'converges' each geometry to a value derived from it."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

LABELS = {75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}


def geometries(n=11, seed=4):
    rng = np.random.default_rng(seed)
    out, taus = [], []
    for k in range(n):
        shape = tuple(int(v) for v in rng.integers(4, 12, 3))
        out.append(np.where(rng.random(shape) < 0.4, 75, 255).astype(np.uint8))
        taus.append(float(rng.uniform(0.6, 1.4)))
    return out, taus


class FakeBatch:
    """Stands in for lbflow_b200.batch.Batch: K of a geometry = its fluid
    count times tau, steps = its edge sum, one update per fluid voxel-step."""

    def __init__(self, geoms, taus, labels, collision='MRT', storage='fp64', device=0):
        self.geoms, self.taus = geoms, taus

    def converge(self, g, report=1000, tol=1e-6, max_steps=200000):
        nf = np.array([(x == 75).sum() for x in self.geoms])
        steps = np.array([sum(x.shape) for x in self.geoms])
        return dict(steps=steps, K=nf * np.array(self.taus), converged=np.ones(len(self.geoms), bool),
                    seconds=float(steps.sum()) * 1e-3, updates=int((nf * steps).sum()))

    def fluid_nodes(self):
        return int(sum((x == 75).sum() for x in self.geoms))

    def close(self):
        pass


def test_partition_is_complete_balanced_and_deterministic():
    from lbflow_b200.batch import estimated_work, partition
    geoms, taus = geometries(23)
    work = estimated_work(geoms, taus, LABELS)
    assert all(w > 0 for w in work)
    for parts in (1, 2, 3, 8):
        split = partition(work, parts)
        assert sorted(k for p in split for k in p) == list(range(len(work)))
        loads = [sum(work[k] for k in p) for p in split]
        # LPT bound: no part exceeds the mean by more than the largest item.
        assert max(loads) <= sum(work) / parts + max(work) + 1e-9
        assert split == partition(work, parts)
    # More parts than items: the extra parts are empty.
    assert partition([3.0, 1.0], 4) == [[0], [1], [], []]


def test_work_counts_fluid_voxels_and_viscous_time():
    from lbflow_b200.batch import estimated_work
    g = np.full((4, 4, 8), 75, np.uint8)
    w1, w2 = estimated_work([g, g], [1.0, 0.75], LABELS)
    assert w1 == pytest.approx(128 * 64 / (0.5 / 3)) and w2 == pytest.approx(2 * w1)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        from lbflow_b200.batch import converge_sharded
        geoms, taus = geometries()
        r = converge_sharded(geoms, taus, LABELS, 1e-5, rank=rank, world=world, batch_factory=FakeBatch)
        out[rank] = dict(K=r['K'].tolist(), steps=r['steps'].tolist(), parts=r['parts'], seconds=r['seconds'],
                         updates=r['updates'], rank_seconds=r['rank_seconds'])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_two_ranks_gather_the_single_process_result():
    from lbflow_b200.batch import converge_sharded
    geoms, taus = geometries()
    single = converge_sharded(geoms, taus, LABELS, 1e-5, batch_factory=FakeBatch)
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0] == res[1]                      # every rank holds the gathered result
    r = res[0]
    assert np.allclose(r['K'], single['K']) and r['steps'] == single['steps'].tolist()
    assert sorted(r['parts'][0] + r['parts'][1]) == list(range(len(geoms)))
    assert r['updates'] == single['updates']
    assert r['seconds'] == max(r['rank_seconds']) and r['seconds'] < single['seconds']
