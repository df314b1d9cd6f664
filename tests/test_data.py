"""The setrun.py boundary writes the reference's data files in its read order."""
import configs

# Field order of claw.data as read by src/2d/amr2.f90:148-335 (2D) and of
# amr.data as written by src/python/amrclaw/data.py:62-123.
CLAW_ORDER = ["num_dim", "lower", "upper", "num_cells", "num_eqn", "num_waves", "num_aux", "t0", "output_style",
              "num_output_times", "tfinal", "output_t0", "output_format", "output_q_components", "dt_initial",
              "dt_max", "cfl_max", "cfl_desired", "steps_max", "dt_variable", "order", "transverse_waves",
              "dimensional_split", "verbosity", "source_split", "capa_index", "use_fwaves", "limiter", "num_ghost",
              "bc_lower", "bc_upper", "restart", "restart_file", "checkpt_style"]
AMR_ORDER = ["amr_levels_max", "refinement_ratios_x", "refinement_ratios_y", "refinement_ratios_t",
             "flag_richardson", "flag_richardson_tol", "flag2refine", "flag2refine_tol", "regrid_interval",
             "regrid_buffer_width", "clustering_cutoff", "verbosity_regrid"]


def _names(path):
    out = []
    for line in open(path):
        if "=:" in line:
            out.append(line.split("=:")[1].split()[0])
    return out


def test_claw_and_amr_data_order(tmp_path):
    rd = configs.advection_square_regression()
    rd.write(str(tmp_path))
    assert _names(tmp_path / "claw.data") == CLAW_ORDER
    assert _names(tmp_path / "amr.data")[: len(AMR_ORDER)] == AMR_ORDER


def test_codes(tmp_path):
    rd = configs.advection_square_regression()
    rd.write(str(tmp_path))
    vals = {}
    for line in open(tmp_path / "claw.data"):
        if "=:" in line:
            v, k = line.split("=:")
            vals[k.split()[0]] = v.split()
    assert vals["limiter"] == ["3"]          # vanleer
    assert vals["bc_lower"] == ["2", "2"]    # periodic
    assert vals["transverse_waves"] == ["2"]
    regions = [l for l in open(tmp_path / "regions.data") if l.strip() and not l.startswith("#") and "=:" not in l]
    assert len(regions) == 2


def test_checkpoint_fields_follow_the_style(tmp_path):
    """amr3.f90:311-325: style 2 is followed by the checkpoint times, style 3 by the interval."""
    rd = configs.euler_blast(n=8, levels=2, tfinal=0.1)
    rd.clawdata.checkpt_style = 2
    rd.clawdata.checkpt_times = [0.05, 0.08]
    rd.write(str(tmp_path))
    names = _names(tmp_path / "claw.data")
    assert names[-3:] == ["checkpt_style", "num_checkpt_times", "checkpt_times"]
    rd.clawdata.checkpt_style = 3
    rd.clawdata.checkpt_interval = 4
    rd.write(str(tmp_path))
    assert _names(tmp_path / "claw.data")[-2:] == ["checkpt_style", "checkpt_interval"]
