"""One data set's score pass split over processes (one per GPU).

Every rank uploads the same sequences, scores its own group of tiles
(Engine.set_partition(rank, world), groups of nearly equal cost, the same in
every rank) and then takes part in one exchange: the bytewise minimum of all
ranks' distance storage.  A pair is scored by exactly one group and every
other rank holds 0xFF bytes for it, so the minimum is the full matrix; each
rank copies it back and can run DBSCAN or the adaptive sweep as after a whole
pass.  The exchange is an all-reduce over torch.distributed (NCCL over
NVLink on GPUs, gloo on CPU)."""
from __future__ import annotations


def combine_bytes(buf, dist):
    """In place: the bytewise minimum of `buf` (a uint8 tensor) over all ranks."""
    dist.all_reduce(buf, op=dist.ReduceOp.MIN)
    return buf


def combine_parts(eng, dist, device):
    """After this rank's partitioned score pass: the full matrix in `eng`."""
    import torch
    nbytes = eng.distance_bytes()
    buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)
    if nbytes:
        eng.distance_copy(buf.data_ptr(), to_engine=False)
    combine_bytes(buf, dist)
    if buf.is_cuda:
        torch.cuda.current_stream(buf.device).synchronize()  # the engine's stream copies it back
    if nbytes:
        eng.distance_copy(buf.data_ptr(), to_engine=True)
    return nbytes
