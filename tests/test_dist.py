"""Grid partition over ranks and the reduction of partial builds, with two
gloo ranks on the CPU: every rank builds its Morton block of the grid with the
FP64 oracle, the partial results are all-reduced, and the sum must equal the
whole-grid build (the reduction ParaGauss does in xc_sndrcv)."""
import os
import socket

import numpy as np
import pytest

import oracle as O
from pgxc import cases, dist as D


def test_spatial_shards_partition_the_grid():
    c = cases.small_case(functional="PBE", seed=3)
    for world in (1, 2, 3, 8):
        parts = D.spatial_shards(c.grid_xyz, world)
        assert len(parts) == world
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(c.npts))
        assert all(len(p) % 128 == 0 for p in parts[:-1])


def test_shards_are_spatially_compact():
    """Each shard's bounding box is much smaller than the whole grid's."""
    c = cases.small_case(functional="VWN", seed=4, natoms=5)
    parts = D.spatial_shards(c.grid_xyz, 8)
    full = np.prod(np.ptp(c.grid_xyz, axis=0))
    vols = [np.prod(np.ptp(c.grid_xyz[p], axis=0)) for p in parts if len(p)]
    assert np.median(vols) < 0.5 * full


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, functional, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = cases.small_case(functional=functional, seed=11, natoms=5, nocc=7)
        O.weight_case(c)
        idx = D.spatial_shards(c.grid_xyz, world)[rank]
        ham, exc, nel = O.xc_build(D.shard_case(c, idx), nthreads=1)
        ham, exc, nel = D.reduce_build(ham, exc, nel)
        if rank == 0:
            np.save(out, np.concatenate([ham, [exc, nel]]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("functional", ["VWN", "PBE"])
def test_two_rank_reduction_equals_whole_grid(functional, tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r0.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), functional, out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    c = cases.small_case(functional=functional, seed=11, natoms=5, nocc=7)
    O.weight_case(c)
    ham, exc, nel = O.xc_build(c, nthreads=1)
    # the sums differ from the single build only by the order of additions
    assert abs(got[-2] - exc) < 1e-11 and abs(got[-1] - nel) < 1e-11
    assert np.max(np.abs(got[:-2] - ham)) < 1e-11
