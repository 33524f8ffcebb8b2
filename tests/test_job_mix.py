"""The batched/served job list (64 jobs, PRNG seed 1234) is pinned: the committed JSON that
`wf batch` / `wf serve` read equals what the package's job_mix + mix_job_desc draw now."""
import json
import os
import sys

from conftest import GOLDEN_DIR

sys.path.insert(0, GOLDEN_DIR)
import make_job_mix  # noqa: E402


def test_job_mix_matches_committed_list(wfb):
    with open(make_job_mix.OUT) as f:
        committed = json.load(f)
    assert committed == json.loads(json.dumps(make_job_mix.job_list(wfb)))
    jobs = committed["jobs"]
    assert len(jobs) == 64 and [j["seed"] for j in jobs] == list(range(1, 65))
    assert {j["scene"] for j in jobs} == set(wfb.MIX_SCENES)
    assert all((j["width"], j["height"]) in wfb.MIX_RESOLUTIONS and j["spp"] in wfb.MIX_SPP for j in jobs)
    assert os.path.basename(make_job_mix.OUT) == "job_mix_64_seed1234.json"
