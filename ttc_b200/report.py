"""Report of the tuned transpositions stored in a plan database (TTC's ttc.db schema).

TTC's generatePlots.py (createBenchmarkPerfPlots, generatePlots.py:141-265 in the TTC project)
reads the `fastest0Percent` view - the fastest variant of every measurement - joined with the size
table, and summarises it per tensor rank: the minimum, mean, maximum and standard deviation of the
attained bandwidth, and of the speedup over the measurement's reference bandwidth where one was
recorded. This module runs the same query on a database the tuner wrote and prints the summary as
a table, optionally also as CSV (matplotlib is not part of this library's dependencies, so no
figure is drawn).

    python -m ttc_b200.report [--db ttc.db] [--where "floatTypeA = 'float'"] [--csv out.csv]
"""
from __future__ import annotations

import argparse
import csv
import math
import sys
from typing import Optional

from .sql_util import DatabaseUnavailable, connect


def benchmark_summary(db: str, where: str = "1") -> list[dict]:
    """Per rank: count, min/mean/max/std bandwidth (GiB/s) of the fastest variants and their
    speedup over the reference bandwidth (measurements without one are left out of the speedup)."""
    con = connect(db)
    try:
        rows = con.execute(
            "SELECT dim, bandwidth, IFNULL(referenceBandwidth, 0) FROM fastest0Percent "
            "JOIN size ON fastest0Percent.size_id = size.size_id WHERE " + where).fetchall()
    finally:
        con.close()
    by_dim: dict[int, list] = {}
    for dim, bw, ref in rows:
        by_dim.setdefault(int(dim), []).append((float(bw), float(ref)))

    def stats(xs):
        if not xs:
            return None, None, None, None
        m = sum(xs) / len(xs)
        return min(xs), m, max(xs), math.sqrt(sum((x - m) ** 2 for x in xs) / len(xs))

    out = []
    for dim in sorted(by_dim):
        bws = [b for b, _ in by_dim[dim]]
        sps = [b / r for b, r in by_dim[dim] if r > 0]
        bmin, bavg, bmax, bstd = stats(bws)
        smin, savg, smax, sstd = stats(sps)
        out.append({"dim": dim, "count": len(bws), "bw_min": bmin, "bw_avg": bavg, "bw_max": bmax, "bw_std": bstd,
                    "speedup_count": len(sps), "speedup_min": smin, "speedup_avg": savg, "speedup_max": smax,
                    "speedup_std": sstd})
    return out


def format_table(rows: list[dict]) -> str:
    head = f"{'dim':>3} {'n':>5} {'min GiB/s':>10} {'avg GiB/s':>10} {'max GiB/s':>10} {'std':>8}  " \
           f"{'speedup min/avg/max':>24}"
    lines = [head, "-" * len(head)]
    for r in rows:
        sp = "-" if not r["speedup_count"] else \
            f"{r['speedup_min']:.2f}/{r['speedup_avg']:.2f}/{r['speedup_max']:.2f}"
        lines.append(f"{r['dim']:>3} {r['count']:>5} {r['bw_min']:>10.2f} {r['bw_avg']:>10.2f} {r['bw_max']:>10.2f} "
                     f"{r['bw_std']:>8.2f}  {sp:>24}")
    return "\n".join(lines)


def main(argv: Optional[list] = None) -> int:
    ap = argparse.ArgumentParser(description="Summary of the fastest tuned variants per tensor rank")
    ap.add_argument("--db", default=None, help="plan database (default: the tuner's ttc.db)")
    ap.add_argument("--where", default="1", help="SQL constraint on the joined rows, as in generatePlots.py")
    ap.add_argument("--csv", default=None, help="also write the summary to this CSV file")
    a = ap.parse_args(argv)
    if a.db is None:
        from .ttc import database_path
        a.db = database_path()
    db = a.db
    try:
        rows = benchmark_summary(db, a.where)
    except DatabaseUnavailable as e:
        print(f"[TTC] ERROR: database {db} unavailable: {e}", file=sys.stderr)
        return 1
    print(format_table(rows))
    if a.csv:
        with open(a.csv, "w", newline="") as f:
            w = csv.DictWriter(f, fieldnames=list(rows[0].keys()) if rows else ["dim"])
            w.writeheader()
            w.writerows(rows)
    return 0


if __name__ == "__main__":
    sys.exit(main())
