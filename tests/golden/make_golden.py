"""Regenerate the gauge fixtures from the reference's regression data.

Reads tests/<case>/regression_data/gauge*.txt of the reference checkout
(gauge rows "level time q(1..meqn)", printed e15.7) and writes one compact
fixture per case here: rows "gauge_id level time q...". Usage:

    python tests/golden/make_golden.py <path of the reference checkout>

The fixtures are committed so the tests never read the reference at run time.
"""
import glob
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <path of the reference checkout>")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {"advection_2d_square": [1, 2], "acoustics_2d_radial": [0, 1, 2], "advection_3d_swirl": [1, 2],
         "advection_2d_annulus": [1, 2], "acoustics_1d_homogeneous": [0, 1], "advection_1d_example1": [0, 1],
         "euler_1d_wcblast": [1, 2]}

for case, ids in CASES.items():
    rows = []
    for gid in ids:
        path = os.path.join(REF, "tests", case, "regression_data", "gauge%05d.txt" % gid)
        with open(path) as f:
            for line in f:
                if line.startswith("#") or not line.strip():
                    continue
                rows.append("%d %s" % (gid, " ".join(line.split())))
    out = os.path.join(HERE, "%s_gauges.txt" % case)
    with open(out, "w") as f:
        f.write("# gauge rows of the reference regression data: gauge_id level time q(1..meqn)\n")
        f.write("\n".join(rows) + "\n")
    print(out, len(rows))
