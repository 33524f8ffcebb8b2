"""wfb_render_passes_noalloc: the render entry point for callers that cannot allocate device memory
(a host that owns all device memory through its own pool, or a real-time loop where an allocation
would break the frame budget). The test owns the film buffers (allocated here with torch, as such a caller's pool
would), calls the entry point through the C ABI and checks the film against the renderer's, bit for
bit -- the tolerance every film test in this suite uses -- on two calls in a row."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(wfb):
    lib = wfb.load_library()
    fn = lib.wfb_render_passes_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _film(torch, w, h):
    return [torch.zeros(n, dtype=torch.float32, device="cuda") for n in (3 * w * h, w * h, w * h)]


def _call(wfb, fn, scene, first, count, seed, depth, film):
    st = fn(scene.handle, first, count, seed, depth, film[0].data_ptr(), film[1].data_ptr(), film[2].data_ptr(), None)
    if st != wfb.OK:
        raise wfb.WfbError(st, wfb.load_library().wfb_last_error().decode())


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _expected(wfb, scene, first, count, seed, depth):
    """Film sums of the existing entry point (a renderer's run_passes) for the same samples."""
    r = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    r.run_passes(first, count, wfb.RenderParams(spp=count, seed=seed, max_depth=depth))
    rgb, lum, lum2 = r.download_sums()
    return r, [rgb.reshape(-1), lum.reshape(-1), lum2.reshape(-1)]


def test_noalloc_equals_renderer_on_two_calls_in_a_row(wfb):
    torch = pytest.importorskip("torch")
    fn = _noalloc(wfb)
    w, h, spp = 64, 36, 8
    scene = wfb.Scene.generate("cornell36", w, h, 1234, 16)
    keep, want = _expected(wfb, scene, 0, spp, 1234, 8)  # creating the renderer uploads the scene
    for call in range(2):
        film = _film(torch, w, h)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _call(wfb, fn, scene, 0, spp, 1234, 8, film)
        torch.cuda.synchronize()
        if call == 1:  # the first call on a device may load the module holding the static array
            assert torch.cuda.mem_get_info()[0] == free_before, "the no-alloc entry point allocated device memory"
        for got, exp in zip(film, want):
            assert np.array_equal(_bits(got.cpu().numpy()), _bits(exp)), f"call {call}: film differs"


def test_noalloc_progressive_and_large_image(wfb):
    torch = pytest.importorskip("torch")
    fn = _noalloc(wfb)
    # progressive: [0, 3) then [3, 8) on one film == [0, 8) rendered by a renderer
    w, h = 40, 24
    scene = wfb.Scene.generate("icospheres", w, h, 1234, 16)
    keep, want = _expected(wfb, scene, 0, 8, 77, 8)
    film = _film(torch, w, h)
    _call(wfb, fn, scene, 0, 3, 77, 8, film)
    _call(wfb, fn, scene, 3, 5, 77, 8, film)
    torch.cuda.synchronize()
    for got, exp in zip(film, want):
        assert np.array_equal(_bits(got.cpu().numpy()), _bits(exp))
    # a full-resolution pass (921,600 samples) runs in direct mode, twice in a row
    big = wfb.Scene.generate("icospheres", 1280, 720, 1234, 16)
    keep_big, want_big = _expected(wfb, big, 5, 1, 1234, 8)
    for _ in range(2):
        film = _film(torch, 1280, 720)
        _call(wfb, fn, big, 5, 1, 1234, 8, film)
        torch.cuda.synchronize()
        for got, exp in zip(film, want_big):
            assert np.array_equal(_bits(got.cpu().numpy()), _bits(exp))


def test_noalloc_rejects_oversize_and_non_resident_scene(wfb):
    torch = pytest.importorskip("torch")
    fn = _noalloc(wfb)
    scene = wfb.Scene.generate("cornell36", 64, 36, 1234, 16)
    film = _film(torch, 64, 36)
    with pytest.raises(wfb.WfbError, match="not resident"):
        _call(wfb, fn, scene, 0, 1, 1, 8, film)  # no renderer yet: never uploaded
    keep = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    with pytest.raises(wfb.WfbError, match="WFB_NOALLOC_MAX_SAMPLES") as e:
        _call(wfb, fn, scene, 0, 1048576 // (64 * 36) + 1, 1, 8, film)
    assert e.value.status == wfb.ERR_INVALID_ARGUMENT


def test_noalloc_on_a_non_blocking_stream_with_the_scene_destroyed_at_once(wfb):
    """The call returns without waiting; the caller may destroy the scene right away. The scene's
    device memory must outlive the queued render, which runs on a stream that the library's own
    (legacy default) stream does not wait for."""
    torch = pytest.importorskip("torch")
    fn = _noalloc(wfb)
    w, h = 1280, 720  # 921,600 samples: one call of the largest size the scratch array takes
    scene = wfb.Scene.generate("icospheres", w, h, 1234, 16)
    keep, want = _expected(wfb, scene, 2, 1, 99, 8)
    film = _film(torch, w, h)
    stream = torch.cuda.Stream()  # created with cudaStreamNonBlocking
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        st = fn(scene.handle, 2, 1, 99, 8, film[0].data_ptr(), film[1].data_ptr(), film[2].data_ptr(),
                ctypes.c_void_p(stream.cuda_stream))
    assert st == wfb.OK, wfb.load_library().wfb_last_error().decode()
    keep.close()
    scene.close()  # last owner gone: the arena release is queued behind the render
    # an identical scene uploaded at once may take the released memory from the same pool
    again = wfb.Scene.generate("icospheres", w, h, 1234, 16)
    keep_again = wfb.GpuRenderer(again, wfb.MEGAKERNEL)
    stream.synchronize()
    for got, exp in zip(film, want):
        assert np.array_equal(_bits(got.cpu().numpy()), _bits(exp))
    keep_again.close()
