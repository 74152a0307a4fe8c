"""Per-kernel launches, total device time and share from an ncu launch list.

Input: the CSV that `ncu --metrics gpu__time_duration.sum --csv --log-file X`
writes.  Output: a markdown table, one row per kernel name, sorted by time.

    python -m spiffe_b200.launch_summary launches.csv [--top N]
"""
import argparse
import csv
import re
from collections import defaultdict


def short_name(name):
    # "<unnamed>::k_push32<1, 1>(int, ...)" -> "k_push32<1, 1>"
    name = re.sub(r"^\(anonymous namespace\)::|^<unnamed>::", "", name)
    depth, out = 0, []
    for ch in name:
        if ch == "(" and depth == 0 and out and not "".join(out).startswith("void cub"):
            break
        depth += ch == "<"
        depth -= ch == ">"
        out.append(ch)
    s = "".join(out).strip()
    return s if len(s) <= 60 else s[:57] + "..."


def read(path):
    per = defaultdict(lambda: [0, 0.0])
    with open(path, newline="") as fh:
        lines = [ln for ln in fh if ln.startswith('"')]
    for row in csv.DictReader(lines):
        if row.get("Metric Name") != "gpu__time_duration.sum":
            continue
        scale = {"ns": 1e-6, "us": 1e-3, "usecond": 1e-3, "ms": 1.0, "msecond": 1.0, "nsecond": 1e-6}[
            row["Metric Unit"]]
        k = short_name(row["Kernel Name"])
        per[k][0] += 1
        per[k][1] += float(row["Metric Value"].replace(",", "")) * scale
    return per


def main():
    p = argparse.ArgumentParser()
    p.add_argument("csv")
    p.add_argument("--top", type=int, default=30)
    a = p.parse_args()
    per = read(a.csv)
    total = sum(v[1] for v in per.values())
    print("| kernel | launches | total ms | share |")
    print("|---|---:|---:|---:|")
    for k, (n, ms) in sorted(per.items(), key=lambda kv: -kv[1][1])[: a.top]:
        print(f"| {k} | {n} | {ms:.3f} | {100 * ms / total:.2f}% |")
    print(f"\ntotal {total:.3f} ms over {sum(v[0] for v in per.values())} launches")


if __name__ == "__main__":
    main()
