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


STRUCTS = [("wfb_scene_desc", "SceneDesc"), ("wfb_scene_info", "SceneInfo"),
           ("wfb_render_params", "_CRenderParams"), ("wfb_render_stats", "_CRenderStats"),
           ("wfb_tune_result", "_CTuneResult"), ("wfb_job_desc", "_CJobDesc"),
           ("wfb_server_config", "_CServerConfig"), ("wfb_server_stats", "_CServerStats"),
           ("wfb_launch_config", "_CLaunchConfig"), ("wfb_device_facts", "_CDeviceFacts")]


def test_ctypes_mirrors_match_c_layout(wfb, tmp_path):
    """Every ctypes structure has the size and field offsets the C compiler gives the header."""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wfb200.h"', "int main(void) {"]
    for c_name, py_name in STRUCTS:
        lines.append(f'printf("{py_name} size %zu\\n", sizeof({c_name}));')
        for fname, _ in getattr(wfb, py_name)._fields_:
            lines.append(f'printf("{py_name} {fname} %zu\\n", offsetof({c_name}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c_layout = {(ln.split()[0], ln.split()[1]): int(ln.split()[2]) for ln in out if ln.strip()}
    for _, py_name in STRUCTS:
        cls = getattr(wfb, py_name)
        assert ctypes.sizeof(cls) == c_layout[(py_name, "size")], py_name
        for fname, _ in cls._fields_:
            assert getattr(cls, fname).offset == c_layout[(py_name, fname)], (py_name, fname)


def test_python_parameter_objects_construct(wfb):
    p = wfb.RenderParams(spp=3, seed=9, max_depth=4, count_rays=True)
    assert (p.spp, p.seed, p.max_depth, p.count_rays) == (3, 9, 4, True)
    c = p._c()
    assert c.seed == 9 and c.max_depth == 4
    st = wfb.RenderStats()
    assert st.kernel_launches == 0 and st.node_visits == 0
    j = wfb.JobDesc((0.0, 1.0, 5.0), (0.0, 0.0, 0.0), width=8, height=4, spp=2)
    assert j._c().width == 8


def _dynamic_symbols(path):
    import subprocess
    out = subprocess.run(["nm", "-DC", "--defined-only", path], check=True, capture_output=True, text=True).stdout
    return [ln.split(" ", 2)[2] for ln in out.splitlines() if len(ln.split(" ", 2)) == 3]


def test_engine_library_exports_only_the_c_abi():
    syms = _dynamic_symbols(os.path.join(PKG_DIR, "libwfb200.so"))
    assert syms and all(s.startswith("wfb_") for s in syms), [s for s in syms if not s.startswith("wfb_")][:10]


def test_cpp_dropin_exports_the_reference_gpu_interface():
    """libwf_gpu.so provides exactly what code written against WVM/include/wf/renderer.hpp and
    WVM/src/gpu/queues.cuh links to (the reference's GPU library surface), and nothing else."""
    syms = _dynamic_symbols(os.path.join(PKG_DIR, "libwf_gpu.so"))
    need = ["wf::GpuRenderer::GpuRenderer(wf::Scene const&, wf::GpuMode)", "wf::GpuRenderer::~GpuRenderer()",
            "wf::GpuRenderer::render(wf::RenderParams const&, wf::RenderStats*)", "wf::GpuRenderer::reset()",
            "wf::GpuRenderer::run_passes(int, int, wf::RenderParams const&, wf::RenderStats*)",
            "wf::GpuRenderer::download(int)",
            "wf::GpuRenderer::download_mean(int, std::vector<float, std::allocator<float> >*)",
            "wf::GpuRenderer::device_bytes() const", "wf::query_cuda_device()",
            "wf::gpu::scan_workspace_create(wf::gpu::ScanWorkspace*, int)",
            "wf::gpu::scan_workspace_destroy(wf::gpu::ScanWorkspace*)"]
    for n in need:
        assert n in syms, n
    assert any(s.startswith("wf::GpuRenderer::device_name") for s in syms)
    for fn in ("scan_exclusive_u32", "compact_u32", "test_queue_push"):
        assert any(s.startswith(f"wf::gpu::{fn}(") for s in syms), fn
    assert all(s.startswith(("wf::GpuRenderer::", "wf::query_cuda_device", "wf::gpu::")) for s in syms)
