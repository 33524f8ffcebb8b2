"""Writes the batched/served job list (64 jobs, PRNG seed 1234) as JSON, cameras resolved.

The list is drawn once by the package's `job_mix` (numpy PCG64, documented there) and each job's
orbit camera is resolved against its scene's default camera (`mix_job_desc`). Cameras are stored as
the exact float32 values (shortest decimal that reads back to the same float32), so every reader --
this package, `wf batch` / `wf serve`, or another tool -- renders the same jobs bit for bit.
Run from the repository root:
    python tests/golden/make_job_mix.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import load_engine  # noqa: E402

N_JOBS, SEED = 64, 1234
OUT = os.path.join(HERE, f"job_mix_{N_JOBS}_seed{SEED}.json")


def f32(v):
    return float(np.float32(v))


def job_list(wfb, n=N_JOBS, seed=SEED):
    scenes = {name: wfb.Scene.generate(name, 64, 64, 1234, 16) for name in wfb.MIX_SCENES}
    jobs = []
    for m in wfb.job_mix(n, seed):
        d = wfb.mix_job_desc(m, scenes[m["scene"]])
        jobs.append({"scene": m["scene"], "width": d.width, "height": d.height, "spp": d.spp,
                     "max_depth": d.max_depth, "seed": d.seed,
                     "azimuth": m["azimuth"], "elevation": m["elevation"],
                     "cam_position": [f32(v) for v in d.cam_position],
                     "cam_look_at": [f32(v) for v in d.cam_look_at],
                     "cam_up": [f32(v) for v in d.cam_up], "cam_vfov_deg": f32(d.cam_vfov_deg)})
    for s in scenes.values():
        s.close()
    return {"generator": "job_mix", "n": n, "prng_seed": seed,
            "scenes": "engine generators, seed 1234, 16-bin SAH", "jobs": jobs}


def main():
    wfb = load_engine()
    wfb.load_library()
    with open(OUT, "w") as f:
        json.dump(job_list(wfb), f, indent=1)
        f.write("\n")
    print(OUT)


if __name__ == "__main__":
    main()
