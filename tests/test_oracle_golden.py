"""The oracle against its golden fixtures: BLAKE3 known answers from the Python `blake3` module, and
the committed tick-hash sequences of two seeded scenes (regression pin)."""
import ctypes
import json
import os
import random

from conftest import oracle_lib, rp, scenes

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_blake3_known_answers():
    lib = oracle_lib()
    f = lib.dll.rphys_oracle_blake3
    f.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
    kat = json.load(open(os.path.join(HERE, "blake3_kat.json")))
    for case in kat["cases"]:
        n = case["len"]
        r = random.Random(kat["seed"] + n)
        data = bytes(r.getrandbits(8) for _ in range(n))
        out = ctypes.create_string_buffer(32)
        f(data, n, out)
        assert out.raw.hex() == case["blake3"], n


def test_scene_hash_sequences():
    lib = oracle_lib()
    g = json.load(open(os.path.join(HERE, "scene_hashes.json")))
    for name, spec in g["scenes"].items():
        w = lib.world(*spec["cap"])
        dt, _ = getattr(scenes, spec["build"])(rp, w, **spec["kw"])
        got = []
        for t in range(spec["ticks"]):
            h = w.step_hash(dt)
            if (t + 1) % 10 == 0:
                got.append(h.hex())
        assert got == g["hashes"][name], name
