"""Summaries of Nsight Compute output for the profiles/ notes.

  python -m gravity_b200.ncu_summary launches <launches.csv> [--skip-init]
      per kernel: launches, total device time and share (from a
      `--metrics gpu__time_duration.sum --csv` launch list).
  python -m gravity_b200.ncu_summary raw <report.ncu-rep> [...]
      the headline counters of a `--set full` capture (DRAM bytes and
      throughput, SM/warp activity, stalls, registers), read with
      `ncu -i <report> --page raw --csv`.
"""

from __future__ import annotations

import argparse
import collections
import csv
import io
import re
import subprocess
import sys

RAW_METRICS = [
    "gpu__time_duration.sum",
    "dram__bytes_read.sum",
    "dram__bytes_write.sum",
    "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed",
    "dram__throughput.avg.pct_of_peak_sustained_elapsed",
    "lts__t_bytes.sum",
    "l1tex__t_bytes.sum",
    "sm__throughput.avg.pct_of_peak_sustained_elapsed",
    "sm__warps_active.avg.pct_of_peak_sustained_active",
    "sm__maximum_warps_per_active_cycle_pct",
    "launch__registers_per_thread",
    "launch__occupancy_limit_registers",
    "launch__shared_mem_per_block_dynamic",
    "launch__grid_size",
    "launch__block_size",
    "smsp__average_warps_issue_stalled_long_scoreboard_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_short_scoreboard_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_mio_throttle_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_lg_throttle_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_barrier_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_wait_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_math_pipe_throttle_per_issue_active.ratio",
    "smsp__issue_active.avg.pct_of_peak_sustained_active",
    "l1tex__data_bank_conflicts_pipe_lsu_mem_shared.sum",
    "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active",
]


def short_name(full: str) -> str:
    name = full.split("(")[0]
    name = re.sub(r"<[^<>]*>", "", name)
    name = re.sub(r"<[^<>]*>", "", name)
    return name.split("::")[-1].strip() or full


def launches(path: str, skip_init: bool = False) -> str:
    rows = list(csv.reader(open(path, newline="")))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    hdr = rows[hi]
    ki, mi, vi, ui = (hdr.index(c) for c in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    tot = collections.defaultdict(float)
    cnt = collections.Counter()
    scale = {"ns": 1.0, "nsecond": 1.0, "usecond": 1e3, "us": 1e3, "msecond": 1e6, "ms": 1e6}
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[mi] != "gpu__time_duration.sum":
            continue
        name = short_name(r[ki])
        if skip_init and name in ("green_real_kernel", "fft64_line_kernel", "green_final_kernel",
                                  "direct_accel_kernel"):
            continue
        tot[name] += float(r[vi].replace(",", "")) * scale.get(r[ui], 1.0)
        cnt[name] += 1
    total = sum(tot.values()) or 1.0
    out = io.StringIO()
    out.write(f"{'kernel':40s} {'launches':>8s} {'total us':>10s} {'share':>7s}\n")
    for k, v in sorted(tot.items(), key=lambda x: -x[1]):
        out.write(f"{k:40s} {cnt[k]:8d} {v / 1e3:10.1f} {100 * v / total:6.1f}%\n")
    out.write(f"{'(all)':40s} {sum(cnt.values()):8d} {total / 1e3:10.1f}\n")
    return out.getvalue()


def raw(report: str) -> str:
    res = subprocess.run(["ncu", "-i", report, "--page", "raw", "--csv"], capture_output=True, text=True)
    if res.returncode != 0:
        raise SystemExit(res.stderr)
    rows = list(csv.reader(io.StringIO(res.stdout)))
    hdr, units = rows[0], rows[1]
    out = io.StringIO()
    for r in rows[2:]:
        d = dict(zip(hdr, r))
        u = dict(zip(hdr, units))
        out.write(f"kernel: {short_name(d.get('Kernel Name', '?'))}\n")
        for m in RAW_METRICS:
            if m in d:
                out.write(f"  {m} = {d[m]} {u.get(m, '')}\n")
        rd, wr = d.get("dram__bytes_read.sum"), d.get("dram__bytes_write.sum")
        if rd and wr:
            mult = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
            b = float(rd.replace(",", "")) * mult.get(u.get("dram__bytes_read.sum", "byte"), 1) + \
                float(wr.replace(",", "")) * mult.get(u.get("dram__bytes_write.sum", "byte"), 1)
            out.write(f"  traffic_bytes_per_launch: {b:.0f}\n")
    return out.getvalue()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("launches")
    a.add_argument("csv")
    a.add_argument("--skip-init", action="store_true")
    b = sub.add_parser("raw")
    b.add_argument("reports", nargs="+")
    args = ap.parse_args(argv)
    if args.cmd == "launches":
        sys.stdout.write(launches(args.csv, args.skip_init))
    else:
        for r in args.reports:
            sys.stdout.write(raw(r))


if __name__ == "__main__":
    main()
