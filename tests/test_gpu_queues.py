"""Queue primitives on a B200 against numpy and against the reference's own kernels
(WVM/tests/test_gpu_queues.cu: sizes incl. 921,600 and 1,000,003, in-place, canaries, capacity
rejection, stable compaction, queue_push popcount / overflow / capacity 0)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 31, 32, 33, 255, 256, 1023, 1024, 1025, 4097, 65536, 921600, 1000003]
CANARY = 0xDEADBEEF


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", SIZES)
def test_scan_matches_numpy_and_reference(wfb, ref, torch, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 2**31, n, dtype=np.uint64).astype(np.uint32)
    csum = np.cumsum(x, dtype=np.uint64) & np.uint64(0xFFFFFFFF)  # sums wrap mod 2^32
    want = np.concatenate([np.zeros(1, np.uint64), csum[:-1]]).astype(np.uint32)
    total_want = np.uint32(np.sum(x, dtype=np.uint64) & 0xFFFFFFFF)
    ws = wfb.ScanWorkspace(n)
    d_in = dev(torch, x)
    d_out = dev(torch, np.full(n + 64, CANARY, np.uint32))
    d_tot = dev(torch, np.zeros(1, np.uint32))
    assert ws.scan_exclusive_u32(d_in.data_ptr(), d_out.data_ptr(), n, d_tot.data_ptr()) == 0
    torch.cuda.synchronize()
    ws.check()
    out = host(d_out)
    assert np.array_equal(out[:n], want)
    assert (out[n:] == CANARY).all(), "wrote past the end"
    assert host(d_tot)[0] == total_want
    # the reference scan gives the same bits
    r_out = dev(torch, np.zeros(n, np.uint32))
    r_tot = dev(torch, np.zeros(1, np.uint32))
    assert ref.ref_lib().ref_scan(d_in.data_ptr(), r_out.data_ptr(), n, r_tot.data_ptr(), n) == 0
    assert np.array_equal(host(r_out), want) and host(r_tot)[0] == total_want


def test_scan_in_place_repeated_and_capacity(wfb, torch):
    ws = wfb.ScanWorkspace(300000)
    rng = np.random.default_rng(7)
    for k in range(40):  # the same workspace over many scans (epoch-tagged status words)
        n = int(rng.integers(1, 300000))
        x = rng.integers(0, 1000, n).astype(np.uint32)
        d = dev(torch, x)
        assert ws.scan_exclusive_u32(d.data_ptr(), d.data_ptr(), n) == 0
        torch.cuda.synchronize()
        want = np.concatenate([np.zeros(1, np.uint64), np.cumsum(x, dtype=np.uint64)[:-1]]).astype(np.uint32)
        assert np.array_equal(host(d), want), k
    ws.check()
    d = dev(torch, np.full(300001, CANARY, np.uint32))
    assert ws.scan_exclusive_u32(d.data_ptr(), d.data_ptr(), 300001) == 1  # n > capacity: rejected
    torch.cuda.synchronize()
    assert (host(d) == CANARY).all(), "a rejected call must not touch memory"
    tot = dev(torch, np.full(1, CANARY, np.uint32))
    assert ws.scan_exclusive_u32(d.data_ptr(), d.data_ptr(), 0, tot.data_ptr()) == 0
    torch.cuda.synchronize()
    assert host(tot)[0] == 0


@pytest.mark.parametrize("n,density", [(1, 1.0), (1000, 0.5), (921600, 0.3), (1000003, 0.9), (50000, 0.0)])
def test_compaction_is_stable_and_matches_reference(wfb, ref, torch, n, density):
    rng = np.random.default_rng(n)
    flags = (rng.random(n) < density).astype(np.uint32) * rng.integers(1, 5, n).astype(np.uint32)
    vals = rng.integers(0, 2**32 - 1, n, dtype=np.uint64).astype(np.uint32)
    want = vals[flags != 0]
    ws = wfb.ScanWorkspace(n)
    d_v, d_f = dev(torch, vals), dev(torch, flags)
    d_o = dev(torch, np.full(n + 16, CANARY, np.uint32))
    d_c = dev(torch, np.zeros(1, np.uint32))
    assert ws.compact_u32(d_v.data_ptr(), d_f.data_ptr(), d_o.data_ptr(), d_c.data_ptr(), n) == 0
    torch.cuda.synchronize()
    ws.check()
    out = host(d_o)
    assert host(d_c)[0] == len(want)
    assert np.array_equal(out[: len(want)], want)
    assert (out[len(want):] == CANARY).all()
    r_o = dev(torch, np.zeros(n, np.uint32))
    r_c = dev(torch, np.zeros(1, np.uint32))
    scratch = dev(torch, np.zeros(n, np.uint32))
    assert ref.ref_lib().ref_compact(d_v.data_ptr(), d_f.data_ptr(), r_o.data_ptr(), r_c.data_ptr(),
                                     scratch.data_ptr(), n, n) == 0
    assert host(r_c)[0] == len(want) and np.array_equal(host(r_o)[: len(want)], want)


@pytest.mark.parametrize("pattern", ["all", "none", "even", "lane0", "random"])
@pytest.mark.parametrize("capacity", [0, 7, 1000, 1 << 20])
def test_queue_push_multiset_and_overflow(wfb, ref, torch, pattern, capacity):
    n = 5000
    idx = np.arange(n)
    flags = {"all": np.ones(n), "none": np.zeros(n), "even": idx % 2 == 0, "lane0": idx % 32 == 0,
             "random": np.random.default_rng(3).random(n) < 0.37}[pattern].astype(np.uint32)
    want = np.flatnonzero(flags)
    for impl in ("engine", "reference"):
        items = dev(torch, np.full(max(capacity, 1) + 8, CANARY, np.uint32))
        counter = dev(torch, np.zeros(1, np.uint32))
        overflow = dev(torch, np.zeros(1, np.uint32))
        d_f = dev(torch, flags)
        if impl == "engine":
            st = wfb.test_queue_push(d_f.data_ptr(), n, items.data_ptr(), capacity, counter.data_ptr(),
                                     overflow.data_ptr())
        else:
            st = ref.ref_lib().ref_queue_push(d_f.data_ptr(), n, items.data_ptr(), capacity, counter.data_ptr(),
                                              overflow.data_ptr())
        torch.cuda.synchronize()
        assert st == 0
        got = host(items)
        stored = min(len(want), capacity)
        assert host(counter)[0] == len(want), impl  # reservations count dropped pushes too
        assert host(overflow)[0] == len(want) - stored, impl
        assert (got[capacity:] == CANARY).all() if capacity else (got == CANARY).all()
        kept = np.sort(got[:stored])
        assert len(np.unique(kept)) == stored and np.isin(kept, want).all(), impl


def test_a_look_back_that_cannot_complete_gives_up(wfb, torch):
    """The next scan claims tiles from 1 on, so no tile publishes the first prefix and every look-back
    waits for it; with a 1 ms limit the waits give up, the kernel returns, the workspace reports
    WFB_ERR_DEVICE_WAIT, and a scan on a fresh workspace is exact."""
    n = 100000
    x = np.arange(n, dtype=np.uint32) % 7
    want = np.concatenate([np.zeros(1, np.uint64), np.cumsum(x, dtype=np.uint64)[:-1]]).astype(np.uint32)
    ws = wfb.ScanWorkspace(n)
    d = dev(torch, x)
    out = dev(torch, np.zeros(n, np.uint32))
    try:
        wfb.set_bounded_wait_test(1_000_000, unsatisfiable=True)
        assert ws.scan_exclusive_u32(d.data_ptr(), out.data_ptr(), n) == 0
        torch.cuda.synchronize()
    finally:
        wfb.set_bounded_wait_test(0)
    with pytest.raises(wfb.WfbError) as e:
        ws.check()
    assert e.value.status == wfb.ERR_DEVICE_WAIT
    ws2 = wfb.ScanWorkspace(n)
    assert ws2.scan_exclusive_u32(d.data_ptr(), out.data_ptr(), n) == 0
    torch.cuda.synchronize()
    ws2.check()
    assert np.array_equal(host(out), want)
