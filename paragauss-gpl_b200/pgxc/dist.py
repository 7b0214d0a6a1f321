"""Grid partition over ranks and the reduction of their partial builds.

ParaGauss hands grid batches to MPI ranks (dynamic load balancing,
dlb/dlb_impl_static.f90:124-166) and sums each rank's packed V_xc and its
E_xc / N_el contributions with one reduction per SCF cycle (xc_sndrcv,
modules/xc_hamiltonian.f90:769-798).  Here each GPU rank owns one spatially
compact block of the grid -- a contiguous range of the points in Morton
order, so that its 128-point tiles list few basis functions -- builds it with
its own context, and the partial results are summed with a single all-reduce
of [packed V, E_xc, N_el].  Becke weights depend only on the point and the
atoms, so every rank computes the weights of its own points.
"""
import numpy as np

from . import cases as C


def morton_keys(xyz, bits=21):
    """64-bit Morton codes of points (n, 3) quantised on their bounding box."""
    xyz = np.asarray(xyz, dtype=np.float64)
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    span = np.where(hi > lo, hi - lo, 1.0)
    q = np.clip(((xyz - lo) / span * ((1 << bits) - 1)).astype(np.int64), 0, (1 << bits) - 1).astype(np.uint64)
    key = np.zeros(len(xyz), dtype=np.uint64)
    for b in range(bits):
        for d in range(3):
            key |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + d)
    return key


def spatial_shards(xyz, world, align=128):
    """Point indices of each rank: contiguous ranges of the Morton order made
    of whole `align`-point tiles, the tiles shared out as evenly as possible
    (only the last range may end in a partial tile)."""
    order = np.argsort(morton_keys(xyz), kind="stable")
    n = len(order)
    tiles = -(-n // align)
    bounds = [min(n, (r * tiles // world) * align) for r in range(world + 1)]
    bounds[-1] = n
    return [order[bounds[r]:bounds[r + 1]] for r in range(world)]


def shard_case(case, idx):
    """The case restricted to the grid points idx (same geometry, basis, orbitals)."""
    sub = C.Case(**{**case.__dict__})
    sub.grid_xyz = case.grid_xyz[idx]
    sub.grid_wraw = case.grid_wraw[idx]
    sub.point_atom = case.point_atom[idx]
    sub.grid_w = None if case.grid_w is None else case.grid_w[idx]
    return sub


def reduce_build(ham, exc, nel, group=None):
    """Sum the ranks' packed V_xc, E_xc and N_el with one all-reduce.

    ham may be a numpy array (host buffers, reduced through a CPU tensor with
    the gloo backend) or a torch tensor on the device of an NCCL group.
    Returns (ham, exc, nel) summed over the group."""
    import torch
    import torch.distributed as dist

    if isinstance(ham, np.ndarray):
        buf = torch.from_numpy(np.concatenate([ham, [exc, nel]]).astype(np.float64))
        dist.all_reduce(buf, group=group)
        out = buf.numpy()
        return out[:-2].copy(), float(out[-2]), float(out[-1])
    buf = torch.cat([ham.reshape(-1), torch.stack([torch.as_tensor(exc, dtype=ham.dtype, device=ham.device),
                                                   torch.as_tensor(nel, dtype=ham.dtype, device=ham.device)])])
    dist.all_reduce(buf, group=group)
    return buf[:-2], buf[-2], buf[-1]
