#!/usr/bin/env python3
"""Nsight Compute CSV summariser.

Default mode follows the reference tool's contract (WVM/tools/ncusum.cpp:143-365, usage in
WVM/tools/README.md): read a long-format CSV (`ncu --csv`, one row per kernel x metric with the
columns ID, Kernel Name, Metric Name, Metric Unit, Metric Value) and write a schema_version 1
JSON object:

    {"schema_version": 1,
     "kernels": [{"name", "invocations", "metrics": [{"name", "unit", "value" (mean), "samples"}]}],
     "summary": {"achieved_occupancy_pct", "warp_execution_efficiency", "registers_per_thread",
                 "dram_throughput_pct", "sm_throughput_pct"}}

Kernels and metrics are sorted by name. Values like "1,234.5" parse as 1234.5. "n/a" and empty
values count as missing ("value": null, "samples": 0). Text-valued metrics are skipped. Each
summary entry is the mean over kernels of that metric's per-kernel mean, or null. Errors (an
unreadable or empty file, a missing column, a row with fewer than 5 fields) print one line to
stderr, write nothing and exit with status 2.

Two more modes:
  --launches   a launch list (`--metrics gpu__time_duration.sum`): per kernel, its launches, total
               device time, mean per launch and share of the total, as a text table.
  --raw        a wide CSV from `ncu -i rep --page raw --csv` (header row, units row, one row per
               captured launch): the named metrics (--metric, repeatable; default: the traffic,
               occupancy, issue and stall set), one block per launch.

  python ncusum.py profile.csv [--out summary.json]
  python ncusum.py launches.csv --launches [--skip-regex R] [--skip-launches N]
  python ncusum.py raw.csv --raw [--metric NAME ...] [--per-unit N]
"""
import argparse
import csv
import io
import json
import re
import sys

REQUIRED = ["ID", "Kernel Name", "Metric Name", "Metric Unit", "Metric Value"]
SUMMARY = {
    "achieved_occupancy_pct": "sm__warps_active.avg.pct_of_peak_sustained_active",
    "warp_execution_efficiency": "smsp__thread_inst_executed_per_inst_executed.ratio",
    "registers_per_thread": "launch__registers_per_thread",
    "dram_throughput_pct": "dram__throughput.avg.pct_of_peak_sustained_elapsed",
    "sm_throughput_pct": "sm__throughput.avg.pct_of_peak_sustained_elapsed",
}
RAW_DEFAULT = [
    "gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum",
    "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "lts__t_sector_hit_rate.pct",
    "launch__registers_per_thread", "launch__grid_size", "launch__block_size",
    "sm__warps_active.avg.pct_of_peak_sustained_active", "smsp__issue_active.avg.pct_of_peak_sustained_active",
    "smsp__thread_inst_executed_per_inst_executed.ratio", "sm__throughput.avg.pct_of_peak_sustained_elapsed",
    "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active",
    "smsp__average_warps_issue_stalled_long_scoreboard_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_wait_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_not_selected_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_branch_resolving_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_short_scoreboard_per_issue_active.ratio",
]
UNIT_SCALE = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "ns": 1e-9, "us": 1e-6, "usecond": 1e-6,
              "ms": 1e-3, "msecond": 1e-3, "s": 1.0, "second": 1.0, "nsecond": 1e-9}


class Fail(Exception):
    pass


def is_null(s: str) -> bool:
    return s == "" or s.lower() == "n/a"


def parse_number(s: str) -> float:
    return float(s.replace(",", ""))


def read_rows(path: str):
    try:
        with open(path, "rb") as f:
            text = f.read().decode("utf-8", errors="replace")
    except OSError:
        raise Fail(f"Error: cannot open file {path}")
    lines = [ln[:-1] if ln.endswith("\r") else ln for ln in text.split("\n")]
    while lines and lines[-1] == "":
        lines.pop()
    if not lines:
        raise Fail(f"Error: {path} is empty")
    # ncu may print ==PROF== / ==WARNING== lines before the table in a --log-file.
    start = next((i for i, ln in enumerate(lines) if ln.startswith('"')), 0)
    return [next(csv.reader(io.StringIO(ln))) if ln else [] for ln in lines[start:]]


def long_table(path: str):
    rows = read_rows(path)
    header = rows[0]
    idx = {}
    for col in REQUIRED:
        if col not in header:
            raise Fail(f"Error: missing required column '{col}' in header")
        idx[col] = header.index(col)
    out = []
    for n, row in enumerate(rows[1:], start=2):
        if not row:
            continue
        if len(row) < 5:
            raise Fail(f"Error: row {n} in {path} has fewer than 5 fields")
        out.append({c: row[i] if i < len(row) else "" for c, i in idx.items()})
    return out


def summarise(path: str) -> dict:
    kernels = {}
    for r in long_table(path):
        k = kernels.setdefault(r["Kernel Name"], {"ids": set(), "metrics": {}})
        k["ids"].add(r["ID"])
        m = k["metrics"].setdefault(r["Metric Name"], {"unit": "", "samples": []})
        m["unit"] = r["Metric Unit"]
        if not is_null(r["Metric Value"]):
            try:
                m["samples"].append(parse_number(r["Metric Value"]))
            except ValueError:
                pass  # text-valued metric
    out_kernels = []
    for name in sorted(kernels):
        k = kernels[name]
        metrics = []
        for mname in sorted(k["metrics"]):
            m = k["metrics"][mname]
            s = m["samples"]
            metrics.append({"name": mname, "unit": m["unit"], "value": (sum(s) / len(s)) if s else None,
                            "samples": len(s)})
        out_kernels.append({"name": name, "invocations": len(k["ids"]), "metrics": metrics})

    def across(metric):
        vals = []
        for k in kernels.values():
            m = k["metrics"].get(metric)
            if m and m["samples"]:
                vals.append(sum(m["samples"]) / len(m["samples"]))
        return sum(vals) / len(vals) if vals else None

    return {"schema_version": 1, "kernels": out_kernels, "summary": {k: across(v) for k, v in SUMMARY.items()}}


def short_name(kernel: str) -> str:
    """`void ns::<unnamed>::k<128, 0, 8, 0>(ns::Args)` -> `k<128, 0, 8, 0>`."""
    base = re.sub(r"<?unnamed>::|\(anonymous namespace\)::", "", kernel).split("(")[0]
    base = re.sub(r"^void\s+", "", base)
    head, sep, tmpl = base.partition("<")
    if sep:
        # keep the template arguments, drop the namespace of the function name
        return head.split("::")[-1] + "<" + tmpl
    return head.split("::")[-1]


def launches(path: str, skip_regex: str = None, skip_launches: int = 0) -> str:
    per = {}
    order = []
    total = 0.0
    seen = 0
    for r in long_table(path):
        if r["Metric Name"] != "gpu__time_duration.sum" or is_null(r["Metric Value"]):
            continue
        seen += 1
        if seen <= skip_launches:
            continue
        name = short_name(r["Kernel Name"])
        if skip_regex and re.search(skip_regex, name):
            continue
        sec = parse_number(r["Metric Value"]) * UNIT_SCALE.get(r["Metric Unit"], 1e-9)
        if name not in per:
            per[name] = [0, 0.0]
            order.append(name)
        per[name][0] += 1
        per[name][1] += sec
        total += sec
    lines = [f"{'kernel':60s} {'launches':>8s} {'total ms':>11s} {'mean ms':>10s} {'share':>7s}"]
    for name in sorted(order, key=lambda n: -per[n][1]):
        n, t = per[name]
        lines.append(f"{name[:60]:60s} {n:8d} {t * 1e3:11.3f} {t * 1e3 / n:10.3f} {100.0 * t / total:6.2f}%")
    lines.append(f"{'total':60s} {sum(v[0] for v in per.values()):8d} {total * 1e3:11.3f}")
    return "\n".join(lines)


def raw(path: str, metrics, per_unit: float = None) -> str:
    rows = read_rows(path)
    if len(rows) < 3:
        raise Fail(f"Error: {path} has no launch rows (expected header, units, data)")
    header, units = rows[0], rows[1]
    if "Kernel Name" not in header:
        raise Fail("Error: missing required column 'Kernel Name' in header")
    kcol = header.index("Kernel Name")
    out = []
    for row in rows[2:]:
        if not row:
            continue
        out.append(f"kernel: {short_name(row[kcol])}")
        for m in metrics:
            if m not in header:
                out.append(f"  {m}: n/a")
                continue
            i = header.index(m)
            out.append(f"  {m}: {row[i]} {units[i]}".rstrip())
        if per_unit:
            tot = 0.0
            for m in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
                if m in header:
                    i = header.index(m)
                    tot += parse_number(row[i]) * UNIT_SCALE.get(units[i], 1.0)
            out.append(f"  dram_bytes_total: {tot:.0f}")
            out.append(f"  dram_bytes_per_unit: {tot / per_unit:.3f}")
    return "\n".join(out)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("input")
    ap.add_argument("--out")
    ap.add_argument("--launches", action="store_true")
    ap.add_argument("--skip-regex")
    ap.add_argument("--skip-launches", type=int, default=0, help="launches mode: ignore the first N launches")
    ap.add_argument("--raw", action="store_true")
    ap.add_argument("--metric", action="append")
    ap.add_argument("--per-unit", type=float, help="raw mode: units the launch processed, for DRAM bytes per unit")
    a = ap.parse_args(argv)
    try:
        if a.launches:
            text = launches(a.input, a.skip_regex, a.skip_launches)
        elif a.raw:
            text = raw(a.input, a.metric or RAW_DEFAULT, a.per_unit)
        else:
            text = json.dumps(summarise(a.input), indent=2)
    except Fail as e:
        print(str(e), file=sys.stderr)
        return 2
    if a.out:
        try:
            with open(a.out, "w") as f:
                f.write(text + "\n")
        except OSError:
            print(f"Error: cannot write to {a.out}", file=sys.stderr)
            return 2
    else:
        print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
