"""Batched and served rendering on a B200: every job's film is bit-identical to the same job rendered
alone, through graph replay, slicing, admission limits and cancellation."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL_RES = ((64, 64), (96, 54), (40, 30), (128, 72), (33, 17))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def scenes(wfb):
    return {name: wfb.Scene.generate(name, 64, 64, 1234, 16) for name in ("cornell36", "icospheres")}


def small_jobs(wfb, scenes, n, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        name = ("cornell36", "icospheres")[i % 2]
        w, h = SMALL_RES[int(rng.integers(len(SMALL_RES)))]
        job = {"scene": name, "width": w, "height": h, "spp": int(rng.choice([1, 3, 4, 8])),
               "max_depth": int(rng.choice([4, 8])), "seed": i + 1,
               "azimuth": float(rng.uniform(0, 360)), "elevation": float(rng.uniform(10, 40))}
        out.append((scenes[name], wfb.mix_job_desc(job, scenes[name])))
    return out


def solo(wfb, scene, job):
    r = wfb.GpuRenderer(scene, wfb.MEGAKERNEL)
    r.set_camera(job.cam_position, job.cam_look_at, job.cam_up, job.cam_vfov_deg, job.width, job.height)
    return r.render(wfb.RenderParams(spp=job.spp, seed=job.seed, max_depth=job.max_depth))


def test_batch_jobs_equal_solo_renders(wfb, scenes):
    jobs = small_jobs(wfb, scenes, 12)
    b = wfb.Batch(max_jobs=16)
    ids = [b.add(s, j) for s, j in jobs]
    st = b.run(count_rays=True)
    assert st.extension_rays > 0 and st.invalid_hits == 0
    for jid, (s, j) in zip(ids, jobs):
        got = b.download(jid)
        want = solo(wfb, s, j)
        assert np.array_equal(bits(got.rgb), bits(want.rgb)), f"job {jid} differs from its solo render"
        assert np.array_equal(bits(got.lum_var), bits(want.lum_var))


@pytest.mark.parametrize("pool", [1 << 12, 1 << 20])
def test_wavefront_batch_jobs_equal_solo_renders(wfb, scenes, pool):
    """The 64-job batch on the other arm: the paths of every job share one persistent wavefront pool (each
    slot carries its job); small pools force split jobs and slot reuse across jobs."""
    jobs = small_jobs(wfb, scenes, 12, seed=7)
    b = wfb.Batch(max_jobs=16, mode=wfb.WAVEFRONT, paths_in_flight=pool)
    ids = [b.add(s, j) for s, j in jobs]
    st = b.run(count_rays=True)
    assert st.extension_rays > 0 and st.invalid_hits == 0 and st.queue_overflows == 0
    assert st.kernel_launches == 4
    mk = wfb.Batch(max_jobs=16)
    for s, j in jobs:
        mk.add(s, j)
    mst = mk.run(count_rays=True)
    assert (mst.extension_rays, mst.shadow_rays) == (st.extension_rays, st.shadow_rays)
    for jid, (s, j) in zip(ids, jobs):
        got = b.download(jid)
        want = solo(wfb, s, j)
        assert np.array_equal(bits(got.rgb), bits(want.rgb)), f"job {jid} differs from its solo render"
        assert np.array_equal(bits(got.lum_var), bits(want.lum_var))


def test_wavefront_server_results_equal_solo_renders(wfb, scenes):
    jobs = small_jobs(wfb, scenes, 6, seed=11)
    srv = wfb.Server(mode=wfb.WAVEFRONT, paths_in_flight=1 << 18, launch_target_ms=5.0)
    tickets = [srv.submit(s, j) for s, j in jobs]
    for t, (s, j) in zip(tickets, jobs):
        assert srv.wait(t, 60000)
        res, _ = srv.result(t)
        assert np.array_equal(bits(res.rgb), bits(solo(wfb, s, j).rgb))
    srv.close()


def test_graph_replay_with_changing_batches(wfb, scenes):
    b = wfb.Batch(max_jobs=16, use_graph=True)
    nog = wfb.Batch(max_jobs=16, use_graph=False)
    for rnd, n in enumerate((5, 11, 3)):
        jobs = small_jobs(wfb, scenes, n, seed=100 + rnd)
        b.clear()
        nog.clear()
        for s, j in jobs:
            b.add(s, j)
            nog.add(s, j)
        b.run()
        nog.run()
        for jid in range(n):
            assert np.array_equal(bits(b.download(jid).rgb), bits(nog.download(jid).rgb))
        # replaying the same batch gives the same films
        first = [b.download(j).rgb.copy() for j in range(n)]
        b.run()
        for jid in range(n):
            assert np.array_equal(bits(b.download(jid).rgb), bits(first[jid]))


def test_batch_rejects_overfull_and_bad_jobs(wfb, scenes):
    b = wfb.Batch(max_jobs=2)
    s, j = small_jobs(wfb, scenes, 1)[0]
    b.add(s, j)
    b.add(s, j)
    with pytest.raises(wfb.WfbError, match="full"):
        b.add(s, j)
    bad = wfb.JobDesc(cam_position=j.cam_position, cam_look_at=j.cam_look_at, width=0, height=4)
    with pytest.raises(wfb.WfbError):
        wfb.Batch(max_jobs=2).add(s, bad)


@pytest.mark.parametrize("kw", [dict(fixed_slice=2), dict(launch_target_ms=1.0), dict(one_job_per_launch=True),
                                dict(use_graph=False, fixed_slice=3), dict(launch_target_ms=1.0, schedule="shared"),
                                dict(launch_target_ms=0.2, schedule="express")])
def test_served_jobs_equal_solo_renders(wfb, scenes, kw):
    jobs = small_jobs(wfb, scenes, 10, seed=11)
    srv = wfb.Server(**kw)
    tickets = []
    for s, j in jobs:  # arrivals spread over time so later jobs join launches already running
        tickets.append(srv.submit(s, j))
        time.sleep(0.002)
    for t, (s, j) in zip(tickets, jobs):
        assert srv.wait(t, 60000)
        assert srv.poll(t) == wfb.JOB_DONE
        got, latency = srv.result(t)
        assert latency > 0.0
        want = solo(wfb, s, j)
        assert np.array_equal(bits(got.rgb), bits(want.rgb))
        assert np.array_equal(bits(got.lum_var), bits(want.lum_var))
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0
    if kw.get("one_job_per_launch"):
        assert st["launches"] == len(jobs)
    srv.close()


def test_results_collected_while_the_server_keeps_launching(wfb, scenes):
    """A collector takes each result as soon as its job is done while later jobs still arrive and
    launch (graph replay): finished jobs leave the server while their films' memory is still to be
    freed by the worker, and every job completes with its solo render's film."""
    jobs = small_jobs(wfb, scenes, 48, seed=23)
    srv = wfb.Server(launch_target_ms=2.0)
    tickets, got, errors = [], {}, []
    ready = threading.Condition()

    def collector():
        for k in range(len(jobs)):
            with ready:
                ready.wait_for(lambda: len(tickets) > k)
                t = tickets[k]
            try:
                assert srv.wait(t, 60000)
                got[k] = srv.result(t)[0]
            except Exception as e:  # surfaced below
                errors.append((k, repr(e)))

    th = threading.Thread(target=collector)
    th.start()
    for s, j in jobs:
        t = srv.submit(s, j)
        with ready:
            tickets.append(t)
            ready.notify_all()
        time.sleep(0.003)
    th.join()
    assert errors == []
    for k in (0, 1, 17, 47):
        s, j = jobs[k]
        assert np.array_equal(bits(got[k].rgb), bits(solo(wfb, s, j).rgb))
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    srv.close()


def test_server_budget_cancel_and_concurrent_submitters(wfb, scenes):
    s = scenes["icospheres"]
    job = wfb.JobDesc(cam_position=(0.0, 6.0, 17.0), cam_look_at=(0.0, 0.5, 0.0), width=128, height=72, spp=8,
                      seed=3, max_depth=8)
    one_job_bytes = 5 * 128 * 72 * 4 + 3 * 128 * 72 * 8 * 4
    srv = wfb.Server(budget_bytes=2 * one_job_bytes + 1024, fixed_slice=1)
    tickets, lock = [], threading.Lock()

    def submitter():
        for _ in range(4):
            t = srv.submit(s, job)
            with lock:
                tickets.append(t)

    threads = [threading.Thread(target=submitter) for _ in range(3)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    srv.cancel(tickets[-1])
    want = solo(wfb, s, job)
    for t in tickets[:-1]:
        assert srv.wait(t, 60000)
        got, _ = srv.result(t)
        assert np.array_equal(bits(got.rgb), bits(want.rgb))
    st = srv.stats()
    assert st["peak_bytes"] <= 2 * one_job_bytes + 1024
    assert st["completed"] == len(tickets) - 1 and st["cancelled"] == 1
    with pytest.raises(wfb.WfbError, match="budget"):
        wfb.Server(budget_bytes=1024).submit(s, job)
    srv.close()


def test_config4_mix_every_job_bitwise_equal_to_solo(wfb):
    """The 64-job batched workload (scenes 1-3, resolutions up to 1920x1080, spp up to 64): one
    launch, and every job equals its solo render bit for bit."""
    mix = wfb.job_mix(64, 1234)
    sc = {name: wfb.Scene.generate(name, 64, 64, 1234, 16) for name in wfb.MIX_SCENES}
    b = wfb.Batch(max_jobs=64)
    jobs = [(sc[m["scene"]], wfb.mix_job_desc(m, sc[m["scene"]])) for m in mix]
    for s, j in jobs:
        b.add(s, j)
    st = b.run()
    assert st.invalid_hits == 0
    for jid, (s, j) in enumerate(jobs):
        got = b.download(jid)
        want = solo(wfb, s, j)
        assert np.array_equal(bits(got.rgb), bits(want.rgb)), f"job {jid} {mix[jid]}"
