"""ncusum: the reference tool's JSON contract (WVM/tools/ncusum.cpp:143-365) and the launch-list and
raw-page modes used for the committed profile summaries. CPU only."""
import importlib.util
import json
import os
import subprocess
import sys

from conftest import PKG_DIR

TOOL = os.path.join(PKG_DIR, "ncusum.py")
HEADER = '"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size",' \
         '"Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n'


def row(i, kernel, metric, unit, value):
    return f'"{i}","1","p","h","{kernel}","1","7","(128, 1, 1)","(148, 1, 1)","0","10.0","S","{metric}","{unit}","{value}"\n'


def run(*args):
    return subprocess.run([sys.executable, TOOL, *args], capture_output=True, text=True)


def load():
    spec = importlib.util.spec_from_file_location("ncusum", TOOL)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_json_contract(tmp_path):
    csv = tmp_path / "p.csv"
    csv.write_text(HEADER
                   + row(0, "kb", "sm__warps_active.avg.pct_of_peak_sustained_active", "%", "40")
                   + row(0, "kb", "launch__registers_per_thread", "register/thread", "64")
                   + row(1, "kb", "sm__warps_active.avg.pct_of_peak_sustained_active", "%", "50")
                   + row(1, "kb", "launch__registers_per_thread", "register/thread", "64")
                   + row(2, "ka", "sm__warps_active.avg.pct_of_peak_sustained_active", "%", "1,000.5")
                   + row(2, "ka", "launch__cache_config", "", "PreferL1")
                   + row(2, "ka", "dram__throughput.avg.pct_of_peak_sustained_elapsed", "%", "n/a"))
    out = tmp_path / "s.json"
    p = run(str(csv), "--out", str(out))
    assert p.returncode == 0, p.stderr
    d = json.loads(out.read_text())
    assert d["schema_version"] == 1
    assert [k["name"] for k in d["kernels"]] == ["ka", "kb"]
    ka, kb = d["kernels"]
    assert ka["invocations"] == 1 and kb["invocations"] == 2
    m = {x["name"]: x for x in kb["metrics"]}
    assert m["sm__warps_active.avg.pct_of_peak_sustained_active"]["value"] == 45.0
    assert m["sm__warps_active.avg.pct_of_peak_sustained_active"]["samples"] == 2
    ma = {x["name"]: x for x in ka["metrics"]}
    assert ma["launch__cache_config"]["value"] is None and ma["launch__cache_config"]["samples"] == 0
    assert ma["dram__throughput.avg.pct_of_peak_sustained_elapsed"]["value"] is None
    s = d["summary"]
    assert s["achieved_occupancy_pct"] == (1000.5 + 45.0) / 2
    assert s["registers_per_thread"] == 64.0
    assert s["dram_throughput_pct"] is None and s["sm_throughput_pct"] is None


def test_errors_exit_2_without_output(tmp_path):
    out = tmp_path / "o.json"
    assert run(str(tmp_path / "missing.csv")).returncode == 2
    empty = tmp_path / "e.csv"
    empty.write_text("")
    p = run(str(empty), "--out", str(out))
    assert p.returncode == 2 and "is empty" in p.stderr and not out.exists()
    bad = tmp_path / "b.csv"
    bad.write_text('"ID","Kernel Name","Metric Name","Metric Value"\n"0","k","m","1"\n')
    p = run(str(bad))
    assert p.returncode == 2 and "missing required column 'Metric Unit'" in p.stderr
    short = tmp_path / "s.csv"
    short.write_text(HEADER + '"0","1"\n')
    p = run(str(short))
    assert p.returncode == 2 and "fewer than 5 fields" in p.stderr


def test_launch_list_shares(tmp_path):
    csv = tmp_path / "l.csv"
    k = "void ns::<unnamed>::megakernel_persistent<128, 0, 8, 0>(ns::<unnamed>::MkArgs)"
    csv.write_text("==PROF== Connected\n" + HEADER + row(0, "warm", "gpu__time_duration.sum", "ns", "5")
                   + row(1, k, "gpu__time_duration.sum", "ms", "3") + row(2, "fill", "gpu__time_duration.sum", "us", "1000")
                   + row(3, k, "gpu__time_duration.sum", "ns", "1,000,000"))
    text = load().launches(str(csv), skip_launches=1)
    lines = text.splitlines()
    assert lines[1].startswith("megakernel_persistent<128, 0, 8, 0>")
    assert " 2 " in lines[1] and "4.000" in lines[1] and "80.00%" in lines[1]
    assert lines[2].startswith("fill") and "20.00%" in lines[2]


def test_raw_page_bytes_per_unit(tmp_path):
    csv = tmp_path / "r.csv"
    csv.write_text('"ID","Kernel Name","dram__bytes_read.sum","dram__bytes_write.sum","gpu__time_duration.sum"\n'
                   '"","","Mbyte","Kbyte","ms"\n'
                   '"0","void k(int)","2.5","500","1.5"\n')
    text = load().raw(str(csv), ["dram__bytes_read.sum", "gpu__time_duration.sum", "absent"], per_unit=1000)
    assert "kernel: k" in text and "dram__bytes_read.sum: 2.5 Mbyte" in text and "absent: n/a" in text
    assert "dram_bytes_total: 3000000" in text and "dram_bytes_per_unit: 3000.000" in text
