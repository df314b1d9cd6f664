"""The output contract: fort.qNNNN / fort.tNNNN / fort.aNNNN files.

The plotting tools read these files by layout, so the device path must write what the
reference's valout writes (src/2d/valout.f90:51-65,149-165; src/3d/valout.f90:45-62,
136-160,190-260,290-296). The oracle's writer restates those edit descriptors; the GPU
tests require the device path's files to be byte-identical to the oracle's for the same
run, frame by frame. The CPU tests pin the Ew.d text and the block layout to the Fortran
format rules themselves.
"""
import os
import re
import tempfile

import numpy as np
import pytest

import configs
from amrclaw_b200 import problems
from oracle.pyoracle import Oracle2D, Oracle3D

E26 = r"[ -]*-?0\.\d{16}(E[+-]\d\d|[+-]\d{3})"


def _binary(rd):
    rd.clawdata.output_format = "binary"
    return rd


def _files(d):
    return sorted(f for f in os.listdir(d) if re.fullmatch(r"fort\.[qtab]\d{4}", f))


def _run_both(rd, ndim, tmp):
    from amrclaw_b200 import Solver
    run, og, dg = (os.path.join(tmp, x) for x in ("run", "oracle", "device"))
    for x in (run, og, dg):
        os.makedirs(x)
    rd.write(run)
    o = (Oracle3D if ndim == 3 else Oracle2D)(run, outdir=og, write_output=True, threads=8)
    o.run(0)
    o.close()
    with Solver(run, outdir=dg, write_output=True) as s:
        s.run(0)
        extra = os.path.join(tmp, "valout")
        s.valout(extra)  # the entry point, on the final state
    return og, dg, extra


def _assert_same_files(og, dg):
    fo, fd = _files(og), _files(dg)
    assert fo == fd and len(fo) >= 3, (fo, fd)
    for name in fo:
        a = open(os.path.join(og, name), "rb").read()
        b = open(os.path.join(dg, name), "rb").read()
        if a != b and name[5] == "b" or (a != b and len(a) % 8 == 0 and b"\n" not in a[:64]):
            x, y = np.frombuffer(a, dtype="<f8"), np.frombuffer(b, dtype="<f8")
            if x.size != y.size:
                raise AssertionError("%s: %d doubles from the oracle, %d from the device" % (name, x.size, y.size))
            k = np.nonzero(x != y)[0]
            raise AssertionError("%s differs at %d of %d doubles, first at %d: oracle %r device %r" % (
                name, k.size, x.size, k[0], x[k[0]], y[k[0]]))
        if a != b:
            la, lb = a.split(b"\n"), b.split(b"\n")
            k = next(i for i, (x, y) in enumerate(zip(la, lb)) if x != y) if len(la) == len(lb) else min(len(la), len(lb))
            raise AssertionError("%s differs at line %d: oracle %r device %r" % (
                name, k + 1, la[k] if k < len(la) else None, lb[k] if k < len(lb) else None))


def _assert_valout_entry_matches_last_frame(og, extra):
    """amrgpu_valout writes the final state as the next frame: same text as the run's last frame."""
    last = [f for f in _files(og) if f.startswith("fort.q")][-1]
    got = [f for f in _files(extra) if f.startswith("fort.q")]
    assert len(got) == 1 and int(got[0][6:]) == int(last[6:]) + 1
    assert open(os.path.join(extra, got[0]), "rb").read() == open(os.path.join(og, last), "rb").read()
    tl = open(os.path.join(og, "fort.t" + last[6:])).read()
    tg = open(os.path.join(extra, "fort.t" + got[0][6:])).read()
    assert tl == tg


@pytest.mark.gpu
def test_2d_frames_byte_identical_to_the_oracle():
    rd = configs.acoustics_radial_regression()
    rd.clawdata.num_output_times = 2
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, extra = _run_both(rd, 2, tmp)
        _assert_same_files(og, dg)
        _assert_valout_entry_matches_last_frame(og, extra)


@pytest.mark.gpu
def test_2d_periodic_frames_byte_identical_to_the_oracle():
    rd = configs.advection_square_bench(n=24, tfinal=0.3, levels=3)
    rd.clawdata.num_output_times = 3
    rd.clawdata.output_t0 = True
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 2, tmp)
        _assert_same_files(og, dg)


@pytest.mark.gpu
def test_3d_frames_byte_identical_to_the_oracle():
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.1, max1d=12)
    rd.clawdata.num_output_times = 2
    rd.clawdata.output_t0 = True
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, extra = _run_both(rd, 3, tmp)
        _assert_same_files(og, dg)
        _assert_valout_entry_matches_last_frame(og, extra)


@pytest.mark.gpu
def test_3d_aux_frames_byte_identical_to_the_oracle():
    """Swirl (3 face-velocity aux arrays): fort.a every frame, naux = 3 in fort.t."""
    rd = problems.advection_swirl3d(n=16, levels=2, tfinal=0.1)
    c = rd.clawdata
    c.num_output_times = 2; c.output_t0 = True
    c.output_aux_components = "all"; c.output_aux_onlyonce = False
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 3, tmp)
        _assert_same_files(og, dg)
        names = _files(dg)
        assert sum(n.startswith("fort.a") for n in names) == 3
        assert re.search(r"^\s+3\s+naux$", open(os.path.join(dg, "fort.t0001")).read(), re.M)


@pytest.mark.gpu
@pytest.mark.parametrize("binary", [False, True], ids=["ascii", "binary"])
def test_2d_aux_frames_byte_identical_to_the_oracle(binary):
    """The annulus (aux: u, v, kappa): fort.a at t0 only (output_aux_onlyonce), naux = 3."""
    rd = configs.advection_annulus_regression()
    c = rd.clawdata
    c.num_output_times = 2; c.output_t0 = True
    c.output_aux_components = "all"; c.output_aux_onlyonce = True
    if binary:
        _binary(rd)
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 2, tmp)
        _assert_same_files(og, dg)
        names = _files(dg)
        assert [n for n in names if n.startswith("fort.a")] == ["fort.a0000"]
        assert re.search(r"^\s+3\s+naux$", open(os.path.join(dg, "fort.t0001")).read(), re.M)


# ----------------------------------------------------------------- CPU: the oracle's layout
def _fortran_float(field):
    """Value of an Ew.d field: 0.ddddE+xx, or 0.dddd+xxx when the exponent has 3 digits."""
    f = field.strip()
    return float(f if "E" in f else re.sub(r"(\d)([+-]\d{3})$", r"\1e\2", f))


def _oracle_frames(rd, ndim, tmp):
    run = os.path.join(tmp, "run")
    out = os.path.join(tmp, "out")
    os.makedirs(run); os.makedirs(out)
    rd.write(run)
    o = (Oracle3D if ndim == 3 else Oracle2D)(run, outdir=out, write_output=True, threads=2)
    o.run(0)
    g, v = o.grids(), o.values()
    o.close()
    return out, g, v


def test_fort_t_layout_follows_t_file_format():
    rd = configs.euler_blast(n=8, levels=2, tfinal=0.02, max1d=12)
    rd.clawdata.output_t0 = True
    with tempfile.TemporaryDirectory() as tmp:
        out, g, _ = _oracle_frames(rd, 3, tmp)
        lines = open(os.path.join(out, "fort.t0001")).read().split("\n")
    # (e18.8,'    time', /, i6,'                 meqn'/, ... 'nghost'/,/)
    assert re.fullmatch(r"[ -]*-?0\.\d{8}E[+-]\d\d    time", lines[0]) and len(lines[0]) == 18 + 8
    for k, (name, val) in enumerate([("meqn", 5), ("ngrids", len(g)), ("naux", 0), ("ndim", 3), ("nghost", 2)]):
        assert lines[k + 1] == "%6d                 %s" % (val, name)
    assert lines[6:] == ["", ""]


def test_fort_q_layout_follows_header_format_and_rows():
    """2D: 8 header lines and a blank, then my rows of mx lines of meqn e26.16 fields,
    each row closed by a list-directed blank record ('  '); 3D adds mz, zlow, dz, a
    blank record per k-plane and one per grid."""
    for ndim, rd in ((2, configs.acoustics_radial_regression()), (3, configs.euler_blast(n=8, levels=2, tfinal=0.02, max1d=12))):
        rd.clawdata.output_t0 = True
        rd.clawdata.tfinal = 0.02
        with tempfile.TemporaryDirectory() as tmp:
            out, g, v = _oracle_frames(rd, ndim, tmp)
            lines = open(os.path.join(out, "fort.q0001")).read().split("\n")
        meqn = 3 if ndim == 2 else 5
        pos, vpos = 0, 0
        for row in g:
            n = [row[3] - row[2] + 1, row[5] - row[4] + 1] + ([row[7] - row[6] + 1] if ndim == 3 else [])
            assert lines[pos] == "%6d                 grid_number" % row[0]
            assert lines[pos + 1] == "%6d                 AMR_level" % row[1]
            for d in range(ndim):
                assert lines[pos + 2 + d] == "%6d                 %s" % (n[d], ("mx", "my", "mz")[d])
            for d in range(2 * ndim):
                assert re.fullmatch(E26 + r"    (xlow|ylow|zlow|dx|dy|dz)", lines[pos + 2 + ndim + d]), lines[pos + 2 + ndim + d]
            pos += 2 + 3 * ndim
            assert lines[pos] == ""
            pos += 1
            cells = int(np.prod(n))
            vals = v[vpos:vpos + cells * meqn].reshape(meqn, cells)
            c = 0
            for _ in range(n[2] if ndim == 3 else 1):
                for _ in range(n[1]):
                    for _ in range(n[0]):
                        ln = lines[pos]
                        assert len(ln) == 26 * meqn
                        got = [_fortran_float(ln[26 * m:26 * (m + 1)]) for m in range(meqn)]
                        np.testing.assert_allclose(got, vals[:, c], rtol=1e-15, atol=0)
                        c += 1
                        pos += 1
                    assert lines[pos] == "  "
                    pos += 1
                if ndim == 3:
                    assert lines[pos] == "  "
                    pos += 1
            if ndim == 3:
                assert lines[pos] == "  "
                pos += 1
            vpos += cells * meqn
        assert lines[pos:] == [""]


# ----------------------------------------------------------------- binary form (output_format 3)
@pytest.mark.gpu
@pytest.mark.parametrize("split", [False, True])
def test_2d_binary_frames_byte_identical_to_the_oracle(split):
    """fort.b holds every grid's whole array (ghost cells as the last step left them)."""
    rd = _binary(configs.euler_quadrants(n=32, levels=3, tfinal=0.15))
    rd.clawdata.num_output_times = 2
    rd.clawdata.output_t0 = True
    if split:
        rd.clawdata.dimensional_split = "godunov"
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 2, tmp)
        _assert_same_files(og, dg)
        assert sum(n.startswith("fort.b") for n in _files(dg)) == 3


@pytest.mark.gpu
@pytest.mark.parametrize("split", [False, True])
def test_3d_binary_frames_byte_identical_to_the_oracle(split):
    rd = _binary(configs.euler_blast(n=16, levels=2, tfinal=0.08, max1d=12))
    rd.clawdata.num_output_times = 2
    rd.clawdata.output_t0 = True
    if split:
        rd.clawdata.dimensional_split = "godunov"
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 3, tmp)
        _assert_same_files(og, dg)


@pytest.mark.gpu
def test_3d_binary_aux_frames_byte_identical_to_the_oracle():
    rd = _binary(problems.advection_swirl3d(n=16, levels=2, tfinal=0.1))
    c = rd.clawdata
    c.num_output_times = 2; c.output_t0 = True
    c.output_aux_components = "all"; c.output_aux_onlyonce = False
    with tempfile.TemporaryDirectory() as tmp:
        og, dg, _ = _run_both(rd, 3, tmp)
        _assert_same_files(og, dg)
        assert sum(n.startswith("fort.a") for n in _files(dg)) == 3


def test_binary_layout_whole_arrays_with_ghost_cells():
    """The oracle's fort.b: per grid nvar * (mx+4) * (my+4) doubles, q(m,i,j) with m fastest;
    the interior matches the run's values and fort.q holds the headers only."""
    rd = _binary(configs.acoustics_radial_regression())
    rd.clawdata.output_t0 = True
    rd.clawdata.tfinal = 0.02
    with tempfile.TemporaryDirectory() as tmp:
        out, g, v = _oracle_frames(rd, 2, tmp)
        raw = np.fromfile(os.path.join(out, "fort.b0001"), dtype="<f8")
        lines = open(os.path.join(out, "fort.q0001")).read().split("\n")
    assert len(lines) == 9 * len(g) + 1
    pos, vpos = 0, 0
    for row in g:
        mx, my = row[3] - row[2] + 1, row[5] - row[4] + 1
        a = raw[pos:pos + 3 * (mx + 4) * (my + 4)].reshape(my + 4, mx + 4, 3)
        inner = np.transpose(a[2:-2, 2:-2, :], (2, 0, 1)).ravel()
        np.testing.assert_array_equal(inner, v[vpos:vpos + 3 * mx * my])
        pos += a.size
        vpos += 3 * mx * my
    assert pos == raw.size
