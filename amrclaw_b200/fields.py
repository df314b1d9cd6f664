"""Hierarchy read-back helpers: a level's grids assembled into one array, and the L1
error and mass drift of one solution against another on that level.

Two runs whose fine grids differ (the FP32 form may flag a cell the FP64 run does not)
still share the base level, which every run covers completely and which carries the
averages of the finer levels (update.f); comparisons are made there.
"""
from __future__ import annotations

import numpy as np


def level_array(grids: np.ndarray, values: np.ndarray, nvar: int, level: int, dims) -> np.ndarray:
    """Values of every grid of `level` placed in a [nvar][nz?][ny][nx] array of the level's
    index space (dims = (nx, ny) or (nx, ny, nz)); cells no grid covers are NaN.

    grids: rows (grid_number, level, ilo, ihi, jlo, jhi[, klo, khi]) in output order;
    values: the interiors in the same order, [m][j][i] (2D) or [m][k][j][i] (3D)."""
    nd = len(dims)
    shape = (nvar,) + tuple(reversed(dims))
    out = np.full(shape, np.nan)
    off = 0
    for row in grids:
        lo = [int(row[2 + 2 * d]) for d in range(nd)]
        hi = [int(row[3 + 2 * d]) for d in range(nd)]
        n = [hi[d] - lo[d] + 1 for d in range(nd)]
        size = nvar * int(np.prod(n))
        if int(row[1]) == level:
            block = values[off:off + size].reshape((nvar,) + tuple(reversed(n)))
            sl = tuple(slice(lo[d], hi[d] + 1) for d in reversed(range(nd)))
            out[(slice(None),) + sl] = block
        off += size
    return out


def l1_error(test: np.ndarray, ref: np.ndarray, cell_volume: float):
    """Per component: absolute L1 error sum|test-ref|*dV and relative error / sum|ref|*dV."""
    diff = np.abs(test - ref).reshape(test.shape[0], -1)
    mag = np.abs(ref).reshape(ref.shape[0], -1)
    absl1 = diff.sum(axis=1) * cell_volume
    refl1 = mag.sum(axis=1) * cell_volume
    rel = np.where(refl1 > 0, absl1 / np.where(refl1 > 0, refl1, 1.0), absl1)
    return absl1, rel
