"""The C-ABI library loads on a host without a GPU and exports every function wgpt.h declares;
host-side entry points (validation, builders) work without a device."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np

from webgpuraytracer_b200 import _lib
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:int|void\s*\*|const char\s*\*|void)\s+(wgpt_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 25
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"
    assert set(names) <= set(_lib.EXPORTS), "every exported function has a ctypes signature"
    assert _lib.lib().wgpt_abi_version() == 1


def test_struct_sizes_match_layout_header():
    text = (ROOT / "include" / "wgpt_layout.h").read_text()
    for struct_name, size in (("wgpt_scene_params", 112), ("wgpt_material", 144), ("wgpt_object", 96),
                              ("wgpt_plane", 32), ("wgpt_mesh_instance", 80), ("wgpt_bvh_node", 32),
                              ("wgpt_triangle", 128), ("wgpt_light", 80), ("wgpt_gbuffer_texel", 48),
                              ("wgpt_denoise_uniforms", 48)):
        assert f"sizeof({struct_name}) == {size}" in text


def test_scene_descriptor_matches_the_header(tmp_path):
    """The ctypes wgpt_scene_desc has the C header's field offsets and size (gcc prints them)."""
    fields = [f[0] for f in _lib.SceneDesc._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "wgpt.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof(wgpt_scene_desc, {f}));\n' for f in fields)
                   + '  printf("%zu\\n", sizeof(wgpt_scene_desc));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [getattr(_lib.SceneDesc, f).offset for f in fields] + [C.sizeof(_lib.SceneDesc)]
    assert got == want


def _desc(p):
    return rd.scene_desc(p)


def test_validate_accepts_generated_scenes_and_rejects_bad_indices():
    L = _lib.lib()
    s = synth.small_scene(1, 64, 64, 4)
    p = sc.pack_scene_data(s)
    msg = C.create_string_buffer(256)
    d = _desc(p)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 0, msg.value
    # a TLAS child out of range
    bad = sc.PackedScene(**{**p.__dict__})
    tl = p.tlas.copy().view(np.uint32).reshape(-1, 8)
    tl[0, 7] = 999
    bad.tlas = tl.view(np.uint8).reshape(-1).copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2
    assert b"tlas" in msg.value
    # a material index beyond the material buffer
    bad = sc.PackedScene(**{**p.__dict__})
    ob = p.objects.copy().view(np.int32).reshape(-1, 24)
    ob[0, 16] = 50
    bad.objects = ob.view(np.uint8).reshape(-1).copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2
    # a texture index beyond the texture array (here: no array at all) is a layout error
    bad = sc.PackedScene(**{**p.__dict__})
    mt = p.materials.copy().view(np.int32).reshape(-1, 36)
    mt[0, 24] = 0                    # albedo_idx
    bad.materials = mt.view(np.uint8).reshape(-1).copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2
    assert b"texture index" in msg.value
    # ... and accepted once the array has that layer
    bad.textures = np.zeros((1, 8, 8, 4), np.uint8)
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 0, msg.value
    # parallax maps are accepted; a height-map index beyond the array is a layout error too
    bad = sc.PackedScene(**{**p.__dict__})
    bad.flags = p.flags | _lib.HAS_HEIGHTMAPS
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 0, msg.value
    mt = p.materials.copy().view(np.int32).reshape(-1, 36)
    mt[0, 26] = 0                    # height_idx
    bad.materials = mt.view(np.uint8).reshape(-1).copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2
    assert b"texture index" in msg.value
    # a size that is not a whole number of records
    bad = sc.PackedScene(**{**p.__dict__})
    bad.objects = p.objects[:-4].copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2


def test_validate_rejects_cyclic_blas():
    L = _lib.lib()
    s = synth.flagship_scene(1, 64, 36, 8, instances=2, prims=3, subdivisions=2, sky=False)
    p = sc.pack_scene_data(s)
    msg = C.create_string_buffer(256)
    d = _desc(p)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 0, msg.value
    bad = sc.PackedScene(**{**p.__dict__})
    nodes = p.bvh.copy().view(np.uint32).reshape(-1, 8)
    inner = np.nonzero(nodes[:, 3] == 0)[0]
    nodes[inner[3], 7] = inner[3]    # right child pointing at itself: a cycle
    bad.bvh = nodes.view(np.uint8).reshape(-1).copy()
    d = _desc(bad)
    assert L.wgpt_validate_scene(C.byref(d), msg, 256) == 2


def test_l2_probe_rejects_bad_arguments_before_touching_a_device():
    L = _lib.lib()
    out = C.c_double(0.0)
    assert L.wgpt_probe_l2_read(0, 0, 1, C.byref(out)) == 1              # below 1 MiB
    assert L.wgpt_probe_l2_read(0, 128 << 20, 1, C.byref(out)) == 1      # above 96 MiB
    assert L.wgpt_probe_l2_read(0, (1 << 20) + 8, 1, C.byref(out)) == 1  # not a multiple of 16
    assert L.wgpt_probe_l2_read(0, 1 << 20, 0, C.byref(out)) == 1        # no repetitions
    assert L.wgpt_probe_l2_read(0, 1 << 20, 1, None) == 1
