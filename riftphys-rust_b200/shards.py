"""The batched-worlds table split across ranks (one process per GPU): rank r of N steps the
contiguous world range [r*W/N, (r+1)*W/N) of one table built from one seed, with no exchange during
the ticks; the per-world 32-byte tick hashes are gathered once per rollback window so every rank
holds the whole table's hashes in world order."""


def world_range(rank, world_size, n_worlds):
    """[first, end) of the worlds rank `rank` of `world_size` steps."""
    return rank * n_worlds // world_size, (rank + 1) * n_worlds // world_size


def gather_world_hashes(local, n_worlds, dist=None, device="cpu"):
    """All ranks' hashes (lists of 32-byte digests of their world ranges, in world order) gathered
    into the whole table's list on every rank. One all_gather of a fixed-size uint8 tensor per rank
    (padded to the largest range); every rank makes the same call."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(local)
    ws, rank = dist.get_world_size(), dist.get_rank()
    lo, hi = world_range(rank, ws, n_worlds)
    assert len(local) == hi - lo, "local hashes must cover this rank's world range"
    most = max(world_range(r, ws, n_worlds)[1] - world_range(r, ws, n_worlds)[0] for r in range(ws))
    buf = torch.zeros((max(most, 1), 32), dtype=torch.uint8)
    for i, h in enumerate(local):
        buf[i] = torch.frombuffer(bytearray(h), dtype=torch.uint8)
    buf = buf.to(device)
    parts = [torch.empty_like(buf) for _ in range(ws)]
    dist.all_gather(parts, buf)
    out = []
    for r in range(ws):
        a, b = world_range(r, ws, n_worlds)
        rows = parts[r].cpu()
        out.extend(bytes(rows[i].numpy().tobytes()) for i in range(b - a))
    return out
