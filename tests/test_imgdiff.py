"""`imgdiff` (the reference's image comparison tool, WVM/tools/imgdiff.cpp) on this engine's PFM reader:
same printed metrics, messages and exit codes as the reference's own tool built from its sources
(oracle/_ref/imgdiff), over identical, close, distant, non-finite, zero and mismatched images."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ORACLE_DIR, PKG_DIR

OURS = os.path.join(PKG_DIR, "imgdiff")
THEIRS = os.path.join(ORACLE_DIR, "_ref", "imgdiff")


def write_pfm(path, rgb):
    h, w, _ = rgb.shape
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(rgb[::-1], "<f4").tobytes())


def run(tool, *args):
    p = subprocess.run([tool, *map(str, args)], capture_output=True, text=True, timeout=60)
    return p.returncode, p.stdout, p.stderr.splitlines()[0] if p.stderr else ""


def cases(tmp):
    rng = np.random.default_rng(5)
    a = rng.uniform(0.0, 2.0, (9, 16, 3)).astype(np.float32)
    b = a.copy()
    b[3, 4, 1] *= np.float32(1.0 + 3e-6)
    c = a.copy()
    c[0, 0, 0] += np.float32(0.25)
    nan_a, nan_b = a.copy(), a.copy()
    nan_a[1, 1, 1] = nan_b[1, 1, 1] = np.nan
    inf_a, inf_b = a.copy(), a.copy()
    inf_a[2, 2, 2] = inf_b[2, 2, 2] = np.inf
    inf_c = a.copy()
    inf_c[2, 2, 2] = -np.inf
    zero = np.zeros_like(a)
    tiny = zero.copy()
    tiny[0, 0, 0] = 1e-30
    neg = -a
    small = a[:8]
    files = {}
    for name, img in [("a", a), ("b", b), ("c", c), ("nan_a", nan_a), ("nan_b", nan_b), ("inf_a", inf_a),
                      ("inf_b", inf_b), ("inf_c", inf_c), ("zero", zero), ("tiny", tiny), ("neg", neg),
                      ("small", small)]:
        files[name] = tmp / (name + ".pfm")
        write_pfm(files[name], img)
    f = files
    return [
        (f["a"], f["a"]), (f["a"], f["b"]), (f["a"], f["c"]), (f["a"], f["c"], "--tol", "0.5"),
        (f["a"], f["b"], "--tol", "1e-7"), (f["nan_a"], f["nan_b"]), (f["inf_a"], f["inf_b"]),
        (f["inf_a"], f["inf_c"]), (f["zero"], f["tiny"]), (f["zero"], f["zero"]), (f["neg"], f["a"]),
        (f["a"], f["small"]), (f["a"], f["b"], "--bogus"), (f["a"],), (f["a"], tmp / "missing.pfm"),
    ]


def test_imgdiff_known_answers(tmp_path):
    if not os.path.exists(OURS):
        pytest.fail("imgdiff is missing: build it with `make -C graphics-book-tutorials_b200`")
    c = cases(tmp_path)
    assert run(OURS, *c[0])[:2] == (0, "max_abs_rel=0\nmean_rel=0\n")
    code, out, _ = run(OURS, *c[1])
    assert code == 0 and 2.9e-6 < float(out.split()[0].split("=")[1]) < 3.1e-6
    assert run(OURS, *c[2])[0] == 1 and run(OURS, *c[3])[0] == 0
    assert run(OURS, *c[5]) == (2, "", "Non-finite pixel mismatch")
    assert run(OURS, *c[6])[0] == 0 and run(OURS, *c[7])[0] == 2
    assert run(OURS, *c[11]) == (2, "", "Image dimensions mismatch")
    assert run(OURS, *c[12]) == (2, "", "Unknown option: --bogus")
    assert run(OURS, *c[13])[0] == 2 and run(OURS, *c[14])[2].startswith("Error:")


def test_imgdiff_matches_the_reference_tool(tmp_path):
    if not os.path.exists(THEIRS):
        pytest.skip("oracle/_ref/imgdiff not built (the reference sources are absent)")
    for args in cases(tmp_path):
        ours, theirs = run(OURS, *args), run(THEIRS, *args)
        if args[-1] == tmp_path / "missing.pfm":  # both fail to read; the wording of the reader differs
            assert ours[0] == theirs[0] == 2 and ours[2].startswith("Error:") and theirs[2].startswith("Error:")
            continue
        assert ours == theirs, args
