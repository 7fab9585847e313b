"""Generates tests/golden/blake3_kat.json: BLAKE3 digests of seeded byte strings, computed with the
Python `blake3` module (the reference hashes with the Rust `blake3` crate, same algorithm). Lengths
cover the single-block, single-chunk, multi-chunk and uneven-tree cases. Run from the repo root."""
import json
import os
import random

import blake3

LENGTHS = [0, 1, 55, 56, 63, 64, 65, 127, 128, 1023, 1024, 1025, 2047, 2048, 2049, 3072, 3073, 4096, 5121,
           7168, 8191, 8192, 8193, 16384, 31745, 65536, 100000]


def data(n, seed=1234):
    r = random.Random(seed + n)
    return bytes(r.getrandbits(8) for _ in range(n))


if __name__ == "__main__":
    out = {"seed": 1234, "cases": [{"len": n, "blake3": blake3.blake3(data(n)).hexdigest()} for n in LENGTHS]}
    path = os.path.join(os.path.dirname(__file__), "blake3_kat.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, len(LENGTHS), "cases")
