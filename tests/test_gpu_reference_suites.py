"""The reference's own GPU test programs (WVM/tests/test_gpu_render.cu, WVM/tests/test_gpu_queues.cu),
compiled unchanged from the reference sources and linked against this engine's drop-in C++ library
(libwf_gpu.so: wf::GpuRenderer, wf::query_cuda_device, wf::gpu queue primitives over the C ABI)
instead of the reference's GPU library. Every reference test must pass except the one that
asserts the reference author's GPU model (compute capability 7.5), which a B200 (10.0) cannot
satisfy."""
import os
import re
import subprocess

import pytest

from conftest import ORACLE_DIR

pytestmark = pytest.mark.gpu

HARDWARE_PINNED = {"query_cuda_device_reports_gtx_1650_ti_facts"}  # CHECK(compute_capability == "7.5")


def run_suite(name, timeout):
    exe = os.path.join(ORACLE_DIR, "_ref", name)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is missing: build it with `make -C oracle` where the reference sources exist")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=timeout)
    results = dict((m.group(2), m.group(1).strip()) for m in re.finditer(r"^\[\s*(ok|FAIL)\s*\] (\S+)$", p.stdout, re.M))
    return p, results


def test_reference_gpu_render_suite_passes_on_engine():
    p, results = run_suite("test_gpu_render_shim", 900)
    assert len(results) >= 15, p.stdout[-2000:]
    failed = {k for k, v in results.items() if v != "ok"}
    assert failed <= HARDWARE_PINNED, f"reference tests failing on the engine: {sorted(failed)}\n{p.stdout[-4000:]}"
    assert "megakernel_and_wavefront_produce_bitwise_identical_images" in results


def test_reference_gpu_queue_suite_passes_on_engine():
    p, results = run_suite("test_gpu_queues_shim", 600)
    assert len(results) >= 15, p.stdout[-2000:]
    failed = {k for k, v in results.items() if v != "ok"}
    assert not failed, f"reference queue tests failing on the engine: {sorted(failed)}\n{p.stdout[-4000:]}"
    assert p.returncode == 0
