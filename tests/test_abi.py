"""The C ABI: the library loads without a GPU and exports every entry point
that include/*.h declares; the structs keep the engine's byte layouts
(GpuFrame 352 bytes, GpuChunk 96 bytes, src/render/mod.rs:458-488)."""
import ctypes as C
import re
from pathlib import Path

from voxelcraft_menu_b200 import native

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(vmw?_[a-z_0-9]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_entry_point_is_exported():
    L = native.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert len(declared_functions()) >= 40


def test_binding_covers_the_headers():
    assert declared_functions() <= set(native.EXPORTED)


def test_struct_layouts():
    assert C.sizeof(native.VmFrame) == 352
    assert native.VmFrame.cloud_cover.offset == 192
    assert native.VmFrame.godray_strength.offset == 208
    assert native.VmFrame.tint_strength.offset == 224
    assert native.VmFrame.wave_amp.offset == 240
    assert native.VmFrame.shaft_origin.offset == 256
    assert native.VmFrame.cloud_patch.offset == 272
    assert native.VmFrame.prev_view_proj.offset == 288
    assert C.sizeof(native.VmChunk) == 96 and native.VmChunk.root.offset == 48
    assert native.CHUNK_DTYPE.itemsize == 96


def test_create_without_a_gpu_reports_an_error():
    import torch
    if torch.cuda.is_available():
        return
    L = native.lib()
    caps = native.VmCaps(64, 64, 8191, 0, 0)
    h = C.c_void_p()
    assert L.vm_create(0, C.byref(caps), C.byref(h)) != 0
    assert not h.value
