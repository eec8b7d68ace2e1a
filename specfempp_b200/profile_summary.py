"""Summarise an ncu launch list (``--metrics gpu__time_duration.sum --csv``)
into per-kernel launches, total time and share.

  python -m specfempp_b200.profile_summary launches.csv
"""
from __future__ import annotations

import collections
import csv
import sys

_UNIT = {"ns": 1e-3, "nsecond": 1e-3, "us": 1.0, "usecond": 1.0, "ms": 1e3, "msecond": 1e3}


def summarise(path):
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, mi, vi, ui = (h.index(k) for k in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    agg = collections.OrderedDict()
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[mi] != "gpu__time_duration.sum":
            continue
        name = r[ki].split("(")[0].replace("void ", "").replace("(anonymous namespace)::", "").replace("unnamed>::", "")
        t = float(r[vi].replace(",", "")) * _UNIT.get(r[ui], 1.0)
        a = agg.setdefault(name.strip(), [0, 0.0])
        a[0] += 1
        a[1] += t
    total = sum(a[1] for a in agg.values())
    out = ["%-44s %8s %12s %7s %10s" % ("kernel", "launches", "total us", "share", "avg us")]
    for k, (n, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        out.append("%-44s %8d %12.1f %6.1f%% %10.2f" % (k[:44], n, t, 100 * t / total, t / n))
    return out


if __name__ == "__main__":
    print("\n".join(summarise(sys.argv[1])))
