"""Readers for the committed golden fixtures (tests/golden)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gauge_rows(case: str) -> np.ndarray:
    rows = []
    with open(os.path.join(GOLDEN, "%s_gauges.txt" % case)) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


def assert_gauges_match(mine: np.ndarray, golden: np.ndarray, rel: float = 6e-7, absol: float = 1e-7) -> None:
    """Rows (gauge, level, time, q...) must match the 7-digit (e15.7) regression data."""
    for gid in np.unique(golden[:, 0]):
        g = golden[golden[:, 0] == gid]
        m = mine[mine[:, 0] == gid]
        assert len(m) == len(g), "gauge %d: %d rows, expected %d" % (gid, len(m), len(g))
        np.testing.assert_array_equal(m[:, 1], g[:, 1], err_msg="gauge %d levels" % gid)
        np.testing.assert_allclose(m[:, 2], g[:, 2], rtol=rel, atol=1e-12, err_msg="gauge %d times" % gid)
        tol = rel * np.abs(g[:, 3:]) + absol
        bad = np.abs(m[:, 3:] - g[:, 3:]) > tol
        assert not bad.any(), "gauge %d values differ at rows %s" % (gid, np.nonzero(bad.any(axis=1))[0][:5])
