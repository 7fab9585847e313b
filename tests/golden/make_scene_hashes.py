"""Generates tests/golden/scene_hashes.json: the tick hashes (every 10th tick) of two seeded scenes,
computed by the CPU oracle (oracle/build/liboracle_rphys.so). They pin the oracle against
regressions and give the GPU tests a committed fixture to match without running the oracle.
Run from the repo root after `make -C oracle`."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import oracle_lib, rp, scenes  # noqa: E402

SCENES = {
    "box_drop_27": {"cap": [64, 64], "ticks": 120, "build": "box_drop", "kw": {"n_side": 3}},
    "terrain_300": {"cap": [512, 512], "ticks": 120, "build": "terrain",
                    "kw": {"n_bodies": 300, "hf_n": 48, "area": 30.0}},
}


def run(lib, spec):
    w = lib.world(*spec["cap"])
    fn = getattr(scenes, spec["build"])
    dt, _ = fn(rp, w, **spec["kw"])
    out = []
    for t in range(spec["ticks"]):
        h = w.step_hash(dt)
        if (t + 1) % 10 == 0:
            out.append(h.hex())
    return out


if __name__ == "__main__":
    lib = oracle_lib()
    data = {"scenes": SCENES, "hashes": {k: run(lib, v) for k, v in SCENES.items()}}
    with open(os.path.join(HERE, "scene_hashes.json"), "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", {k: len(v) for k, v in data["hashes"].items()})
