"""One data set's score pass split over processes (one per GPU).

Every rank uploads the same sequences and scores its own group of tiles
(Engine.set_partition(rank, world): tiles in descending cost go one by one to
the least loaded group, the same in every rank); every other pair of the
packed path holds 0xFF bytes until the exchange.

The exchange is sized to the result, the counterpart of the reference's
gather of per-rank distance stripes (dbscan.c:374-379, 457-458): a rank sends
only the distance rectangles of its own tiles (about one triangle divided by
the number of ranks), receives the other ranks' rectangles and writes them
into both triangles of its matrix.  Payload sizes are exchanged first and
must agree with what the shared layout predicts; payloads then move in
fixed-size chunks with all-gathers (NCCL over NVLink on GPUs, gloo on CPU),
so no rank holds a second full-size matrix.

``combine_bytes`` / ``combine_parts`` are the earlier exchange (an all-reduce
with the bytewise minimum over the whole matrix), kept for comparison."""
from __future__ import annotations

CHUNK_BYTES = 256 << 20


def exchange_tiles(eng, dist, device, chunk_bytes: int = CHUNK_BYTES) -> dict:
    """After this rank's partitioned score pass: every other rank's tile
    rectangles unpacked into `eng`, so its matrix is the whole pass's.
    `eng` needs partition_bytes / partition_pack / partition_unpack (the
    engine, or a stand-in with the same methods).  Returns byte counts."""
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    sizes = [int(eng.partition_bytes(p)) for p in range(world)]
    # sizes first: every rank must see the same layout and the same payloads
    mine = torch.tensor(sizes, dtype=torch.int64, device=device)
    seen = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(seen, mine)
    for r, s in enumerate(seen):
        if s.tolist() != sizes:
            raise RuntimeError(f"rank {r} predicts payload sizes {s.tolist()}, this rank {sizes}")
    own = torch.empty(max(sizes[rank], 16), dtype=torch.uint8, device=device)
    eng.partition_pack(own.data_ptr())
    top = max(sizes) if sizes else 0
    chunk = max(16, min(int(chunk_bytes), (top + 15) // 16 * 16))
    send = torch.zeros(chunk, dtype=torch.uint8, device=device)
    recv = [torch.empty(chunk, dtype=torch.uint8, device=device) for _ in range(world)]
    received = 0
    for off in range(0, top, chunk):
        n = max(0, min(sizes[rank] - off, chunk))
        if n:
            send[:n].copy_(own[off:off + n])
        dist.all_gather(recv, send)
        if send.is_cuda:
            torch.cuda.current_stream(send.device).synchronize()  # the engine's stream reads recv
        for p in range(world):
            m = max(0, min(sizes[p] - off, chunk))
            if p != rank and m:
                eng.partition_unpack(p, recv[p].data_ptr(), off, m)
                received += m
    return {"sent": sizes[rank], "received": received, "chunk": chunk, "rounds": (top + chunk - 1) // chunk}


def combine_bytes(buf, dist):
    """In place: the bytewise minimum of `buf` (a uint8 tensor) over all ranks."""
    dist.all_reduce(buf, op=dist.ReduceOp.MIN)
    return buf


def combine_parts(eng, dist, device):
    """The whole-matrix exchange: the bytewise minimum of every rank's storage."""
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
