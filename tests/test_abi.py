"""The C ABI library loads and exports every symbol its header declares (no GPU needed)."""
import ctypes
import os
import re

from conftest import PKG_DIR, ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(wfb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "wfb_renderer_render" in names and "wfb_scene_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(wfb):
    lib = ctypes.CDLL(os.path.join(PKG_DIR, "libwfb200.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_abi_version_and_errors(wfb):
    lib = wfb.load_library()
    assert lib.wfb_abi_version() == 1
    import pytest
    with pytest.raises(wfb.WfbError) as e:
        wfb.Scene.generate("no-such-scene", 8, 8)
    assert e.value.status == wfb.ERR_INVALID_ARGUMENT
    assert "unknown scene" in str(e.value)
