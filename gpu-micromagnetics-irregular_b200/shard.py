"""Multi-GPU split of a batch of independent LLG instances.

One process per GPU.  The instances are independent (no coupling between
geometries), so the split needs no collective in the hot path: every rank
builds the same seeded instance list, computes the same longest-processing-
time partition (llg_partition_lpt in libllg.so) and integrates only its own
instances; one host-side gather of the final states and counters to rank 0
follows the run.  The reference has no multi-GPU path (one geometry per
process, src/irregular/2d_fft/2d_i2/2d_fft.cu:523 creates its SUNDIALS
context without a communicator).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import llg


def instance_cost(params) -> float:
    """Cost estimate of one instance: cells x expected BDF steps.  Work per
    step is proportional to the cell count (stencils, vectors, the padded
    FFT); the step count grows with the demag strength, which sets the
    stiffness (a linear proxy, 1 + strength / 4)."""
    cells = float(params.ng) * float(params.ny)
    strength = float(params.demag_strength) if params.demag_mode != llg.DEMAG_OFF else 0.0
    return cells * (1.0 + 0.25 * strength)


def partition_lpt(costs, nparts: int):
    """part_of[i] for each instance and the summed cost per part."""
    lib = llg.load()
    c = np.ascontiguousarray(costs, dtype=np.float64)
    part = np.zeros(len(c), np.int32)
    load = np.zeros(nparts, np.float64)
    llg._check(lib.llg_partition_lpt(len(c), c.ctypes.data_as(C.POINTER(C.c_double)), int(nparts),
                                     part.ctypes.data_as(C.POINTER(C.c_int32)),
                                     load.ctypes.data_as(C.POINTER(C.c_double))), "llg_partition_lpt")
    return part, load


def my_instances(instances, world: int, rank: int):
    """Indices of the instances this rank integrates (same on every rank's view)."""
    part, _ = partition_lpt([instance_cost(x["params"]) for x in instances], world)
    return [i for i in range(len(instances)) if part[i] == rank]


def gather_results(local: dict, world: int, rank: int, dst: int = 0):
    """Host gather of per-instance results {index: value} to rank dst over the
    default process group (one call after the run).  Returns the merged dict
    ordered by instance index on dst, None elsewhere."""
    if world == 1:
        return dict(sorted(local.items()))
    import torch.distributed as dist
    bucket = [None] * world if rank == dst else None
    dist.gather_object(local, bucket, dst=dst)
    if rank != dst:
        return None
    merged = {}
    for part in bucket:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"instance {k} integrated on two ranks")
            merged[k] = v
    return dict(sorted(merged.items()))
