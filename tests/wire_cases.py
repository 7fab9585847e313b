"""The riftnet wire snapshot (riftphys-riftnet/src/wire.rs) over any library exporting the C ABI:
the chunks parse with the reference's parse_chunk rules (restated here), carry every live body once
in id order with its pose and shape scale, and the edge cases (no body, exactly a chunk, a removed
body, a short buffer) behave as the header says."""
import struct

import numpy as np

from conftest import rp

HDR = struct.Struct("<IHBBQQHHI")  # NetHdr, repr(C): 32 bytes
ENT = struct.Struct("<I3f4f3fI")   # NetEnt: 48 bytes


def parse_chunk(buf):
    """wire.rs:56-64: the header, then the entities; None when the chunk is not a v2 snapshot."""
    if len(buf) < HDR.size:
        return None
    magic, ver, kind, flags, tick, epoch, total, index, plen = HDR.unpack_from(buf, 0)
    if magic != 0x30535052 or kind != 1 or ver != 2 or plen != len(buf) - HDR.size or plen % ENT.size:
        return None
    ents = [ENT.unpack_from(buf, HDR.size + k * ENT.size) for k in range(plen // ENT.size)]
    return (tick, epoch, total, index), ents


def split(data, chunks):
    """The back-to-back chunks: full chunks of 25 entities, the last one shorter."""
    out, off = [], 0
    for c in range(chunks):
        n = min(25, (len(data) - off - HDR.size) // ENT.size)
        out.append(data[off: off + HDR.size + n * ENT.size])
        off += HDR.size + n * ENT.size
    assert off == len(data)
    return out


def scene(lib, n):
    w = lib.world(max(n + 4, 8), max(n + 4, 8))
    rng = np.random.default_rng(n)
    if n:
        kinds = np.arange(n) % 3
        dims = np.column_stack([rng.uniform(0.1, 0.5, n), rng.uniform(0.1, 0.5, n), rng.uniform(0.1, 0.5, n)])
        for k in range(n):
            d = rp.desc_array(np.array([[k * 1.5, 2.0 + 0.1 * k, 0.0]]), np.array([[0.0, 0.0, 0.0, 1.0]]), dims[k:k + 1],
                              int(kinds[k]), np.array([1000.0]), np.ones(1, dtype=np.uint32))
            w.add_bodies_array(d)
    return w, (kinds if n else np.zeros(0)), (dims if n else np.zeros((0, 3)))


def case_snapshot_parses_and_carries_every_body(lib):
    for n in (0, 1, 25, 26, 60):
        w, kinds, dims = scene(lib, n)
        for _ in range(5):
            w.step(1.0 / 60.0)
        data, chunks = w.pack_snapshot(77, 3)
        assert chunks == (n + 24) // 25 and len(data) == 32 * chunks + 48 * n, (n, chunks, len(data))
        ids = []
        for c, buf in enumerate(split(data, chunks)):
            parsed = parse_chunk(buf)
            assert parsed is not None, f"{n} bodies: chunk {c} does not parse"
            (tick, epoch, total, index), ents = parsed
            assert (tick, epoch, total, index) == (77, 3, chunks, c)
            for e in ents:
                bid = e[0]
                ids.append(bid)
                (p, q) = w.pose(bid)
                assert np.array_equal(np.float32(e[1:4]), np.float32(p)) and np.array_equal(np.float32(e[4:8]), np.float32(q))
                k = int(kinds[bid - 1])
                r, h, z = (float(np.float32(v)) for v in dims[bid - 1])
                want = {0: ((r, r, r), 1), 1: ((r, h, z), 2), 2: ((r, float((np.float32(h) + np.float32(r)) * np.float32(0.5)), r), 3)}[k]
                assert tuple(np.float32(e[8:11])) == tuple(np.float32(want[0])) and e[11] == want[1], (bid, e, want)
        assert ids == list(range(1, n + 1))
        w.close()


def case_snapshot_skips_removed_bodies(lib):
    w, _, _ = scene(lib, 30)
    w.remove_body(5)
    w.remove_body(26)
    data, chunks = w.pack_snapshot(1, 1)
    ids = [e[0] for buf in split(data, chunks) for e in parse_chunk(buf)[1]]
    assert ids == [i for i in range(1, 31) if i not in (5, 26)] and chunks == 2
    w.close()


def case_snapshot_buffer_checks(lib):
    import ctypes
    w, _, _ = scene(lib, 30)
    n, c = ctypes.c_uint64(0), ctypes.c_uint32(0)
    w.c("rphys_ext_pack_snapshot", 0, 0, None, 0, ctypes.byref(n), ctypes.byref(c))
    assert n.value == 32 * 2 + 48 * 30 and c.value == 2
    short = ctypes.create_string_buffer(n.value - 1)
    try:
        w.c("rphys_ext_pack_snapshot", 0, 0, short, n.value - 1, ctypes.byref(n), ctypes.byref(c))
    except rp.RPhysError:
        pass
    else:
        raise AssertionError("a short buffer was accepted")
    w.close()
