"""Richardson error estimation of the 3D path (src/3d errest.f, coarsen.f, errf1.f, with
setflags.f from bufnst.f and the extra step of setgrd.f).

The device path runs the big step (2*dt on the old values coarsened by 2, ghost ring of
twice the width filled at the previous time) and the regular step (dt on the values the
gradient test reads) as virtual patches of the level step kernels, and adds errf1's
flags to the level flag array. FP64 results must equal the oracle's bit for bit. No test
of the reference runs this option; the oracle's restatement is checked by properties.
"""
import tempfile

import numpy as np
import pytest

import configs
from oracle.pyoracle import Oracle3D


def _blast(tol, gradient=True, levels=3, n=16, tfinal=0.1):
    rd = configs.euler_blast(n=n, levels=levels, tfinal=tfinal, max1d=16)
    rd.amrdata.flag_richardson = True
    rd.amrdata.flag_richardson_tol = tol
    rd.amrdata.flag2refine = gradient
    return rd


def _oracle(rd):
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d)
        o.run(0)
        out = dict(grids=o.grids(), values=o.values(), time=o.time(), cells=o.cell_updates())
        o.close()
    return out


def _gpu(rd, **kw):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d, **kw) as s:
            s.run(0)
            return dict(grids=s.grids(), values=s.values(), info=s.info())


def _assert_identical(ref, gpu):
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells" % diff.size
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]


# ---------------------------------------------------------------- oracle properties (CPU)

def test_oracle_smaller_tolerance_refines_at_least_as_much():
    loose = _oracle(_blast(1e30, gradient=False, levels=2, tfinal=0.05))
    tight = _oracle(_blast(2e-3, gradient=False, levels=2, tfinal=0.05))
    assert (loose["grids"][:, 1] > 1).sum() == 0  # nothing reaches an unreachable tolerance
    assert (tight["grids"][:, 1] > 1).sum() > 0
    assert tight["cells"] > loose["cells"]


def test_oracle_rejects_a_tolerance_without_richardson():
    # data.py writes -1 when Richardson is off; a hand-written positive tolerance would
    # make bufnst.f add the old solution to the flags, so the input is refused
    rd = configs.euler_blast(n=8, levels=2, tfinal=0.05, max1d=16)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        path = d + "/amr.data"
        Oracle3D(d).close()  # the file as written loads
        lines = open(path).read().splitlines(True)
        k = next(i for i, l in enumerate(lines) if l.rstrip().endswith("=: flag_richardson_tol"))
        lines[k] = "1.0e-2" + lines[k][len(lines[k].split()[0]):]
        open(path, "w").write("".join(lines))
        with pytest.raises(RuntimeError, match="create failed"):
            Oracle3D(d)


# ---------------------------------------------------------------- device vs oracle (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_blast_richardson_and_gradient_matches_oracle(batched):
    mk = lambda: _blast(2e-3)
    _assert_identical(_oracle(mk()), _gpu(mk(), batched=batched))


@pytest.mark.gpu
def test_blast_richardson_only_matches_oracle():
    mk = lambda: _blast(2e-3, gradient=False)
    ref = _oracle(mk())
    assert (ref["grids"][:, 1] > 1).sum() > 0
    _assert_identical(ref, _gpu(mk()))


@pytest.mark.gpu
def test_fp32_richardson_runs_and_refines():
    g32 = _gpu(_blast(2e-3, gradient=False), precision="fp32")
    assert (g32["grids"][:, 1] > 1).sum() > 0
    assert np.isfinite(g32["values"]).all()
