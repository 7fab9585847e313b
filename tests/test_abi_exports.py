"""The CUDA library loads (no GPU needed to load it) and exports every entry point declared in
include/*.h; the ctypes bindings cover the same set."""
import os
import re
import subprocess

from conftest import PKG_DIR, ROOT, rp


def declared():
    names = set()
    for h in ("riftphys_c.h", "rphys_ext.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(rphys_\w+)\s*\(", src))
    return names


def test_headers_declare_the_v1_abi():
    names = declared()
    for n in ("rphys_world_create", "rphys_world_step_ex", "rphys_world_get_step_hash", "rphys_world_snapshot_create",
              "rphys_world_snapshot_restore", "rphys_world_get_contacts", "rphys_add_box_body"):
        assert n in names


def test_product_library_exports_every_declared_symbol():
    if not os.path.exists(rp.PRODUCT_LIB):
        subprocess.run(["make", "-C", PKG_DIR, "-j8"], check=True, capture_output=True)
    lib = rp.Lib(rp.PRODUCT_LIB)  # also binds every ctypes signature
    missing = [n for n in sorted(declared()) if not hasattr(lib.dll, n)]
    assert not missing, missing
    bound = {n for n, _, _ in rp.ABI}
    assert declared() <= bound, sorted(declared() - bound)


def test_desc_array_matches_struct_layout():
    import ctypes
    import numpy as np
    a = rp.desc_array(np.array([[1.0, 2.0, 3.0]]), np.array([[0.0, 0.0, 0.0, 1.0]]), np.array([[0.5, 0.25, 0.75]]),
                      rp.SHAPE_BOX, np.array([1000.0]), np.array([rp.RPHYS_BODY_DYNAMIC]), 4, 1)
    d = rp.BodyDescEx(rp.iso(1.0, 2.0, 3.0), rp.vel(), rp.SHAPE_BOX, (0.5, 0.25, 0.75), 1000.0, rp.RPHYS_BODY_DYNAMIC, 4, 1)
    assert bytes(a.tobytes()) == ctypes.string_at(ctypes.addressof(d), ctypes.sizeof(d))


def test_batch_scene_is_deterministic():
    import numpy as np
    from conftest import scenes
    a = scenes.batch_world_descs(rp, 3, n_min=16, n_max=300)
    b = scenes.batch_world_descs(rp, 3, n_min=16, n_max=300)
    assert np.array_equal(a, b) and 17 <= len(a) <= 301
