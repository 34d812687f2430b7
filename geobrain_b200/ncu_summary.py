"""Summaries of Nsight Compute CSV output for the profiles of this package.

    python -m geobrain_b200.ncu_summary launches <launches.csv>
        per kernel: launches, total device ms and share of an
        ``ncu --metrics gpu__time_duration.sum --csv`` launch list;
    python -m geobrain_b200.ncu_summary metrics <raw.csv>
        the DRAM, issue, occupancy and stall figures of one captured launch
        from ``ncu -i <rep> --page raw --csv``.
"""
from __future__ import annotations

import collections
import csv
import re
import sys

METRICS = [
    "gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum",
    "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "sm__throughput.avg.pct_of_peak_sustained_elapsed",
    "smsp__issue_active.avg.pct_of_peak_sustained_active", "sm__warps_active.avg.pct_of_peak_sustained_active",
    "launch__registers_per_thread", "launch__grid_size", "launch__occupancy_limit_registers",
    "launch__occupancy_limit_shared_mem", "smsp__inst_executed.sum", "l1tex__data_pipe_lsu_wavefronts_mem_shared.sum",
    "lts__t_sectors_srcunit_tex.sum",
]


def _rows(path):
    with open(path) as f:
        return list(csv.reader([l for l in f if l.startswith('"')]))


def launches(path: str) -> str:
    rows = _rows(path)
    hdr = rows[0]
    ik, im, iv, iu = (hdr.index(k) for k in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    tot = collections.OrderedDict()
    for r in rows[1:]:
        if r[im] != "gpu__time_duration.sum":
            continue
        name = re.sub(r"^void ", "", re.sub(r"\(.*", "", r[ik]))
        v = float(r[iv].replace(",", ""))
        ms = {"nsecond": 1e-6, "ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "msecond": 1.0, "ms": 1.0}.get(r[iu], 1e-6) * v
        c, t = tot.get(name, (0, 0.0))
        tot[name] = (c + 1, t + ms)
    total = sum(t for _, t in tot.values())
    out = ["| kernel | launches | total ms | share |", "|---|---|---|---|"]
    for k, (c, t) in sorted(tot.items(), key=lambda kv: -kv[1][1]):
        out.append(f"| `{k}` | {c} | {t:.3f} | {t / total:.1%} |")
    out.append(f"| all | {sum(c for c, _ in tot.values())} | {total:.3f} | 100% |")
    return "\n".join(out)


def metrics(path: str) -> str:
    rows = _rows(path)
    hdr, units = rows[0], rows[1]
    out = []
    for vals in rows[2:]:
        out.append(f"kernel: {vals[hdr.index('Kernel Name')]}" if "Kernel Name" in hdr else "kernel:")
        for m in METRICS:
            if m in hdr:
                i = hdr.index(m)
                out.append(f"  {m} = {vals[i]} {units[i]}")
        stalls = []
        for i, h in enumerate(hdr):
            if h.startswith("smsp__average_warps_issue_stalled_") and h.endswith("_per_issue_active.ratio"):
                try:
                    stalls.append((float(vals[i].replace(",", "")), h[len("smsp__average_warps_issue_stalled_"):-len(
                        "_per_issue_active.ratio")]))
                except ValueError:
                    pass
        out.append("  stalls per issued instruction: " +
                   ", ".join(f"{n} {v:.2f}" for v, n in sorted(stalls, reverse=True)[:8]))
    return "\n".join(out)


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2 or argv[0] not in ("launches", "metrics"):
        raise SystemExit(__doc__)
    print(launches(argv[1]) if argv[0] == "launches" else metrics(argv[1]))


if __name__ == "__main__":
    main()
