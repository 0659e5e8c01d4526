"""Host-side logic without a GPU: the -group.param front end and the
per-profile defaults (paramsParser.hxx, initGen_*::defaultGridParams)."""
import math

import pytest

from vlasolve_b200.params import ParamsParser
from vlasolve_b200.solver import config_from_dict, config_from_params


def test_cli_values_and_lists():
    p = ParamsParser(["-init.type", "Plummer", "-grid.Ures", "64", "32",
                      "-grid.Umin", "-3", "0", "-solver.noLinking"])
    assert p.get("type", "init", "UDF") == "Plummer"
    assert p.get("Ures", "grid", 0, 1) == 32
    assert p.get("Umin", "grid", 0.0, 0) == -3.0  # "-3" is a value, not a key
    assert p.get("noLinking", "solver", False) is True  # bare key reads as true
    assert p.get("dt", "solver", 0.25) == 0.25


def test_first_definition_wins_and_cli_beats_file(tmp_path):
    f = tmp_path / "p.ini"
    f.write_text("solver.dt 0.1\nsolver.dt 0.2\ngrid.Pres = 64 # comment\n")
    p = ParamsParser([str(f), "-solver.dt", "0.05"])
    assert p.get("dt", "solver", 1.0) == 0.05
    assert p.get("Pres", "grid", 0) == 64


def test_bad_command_line():
    # after the optional parameter file, every argument must start a key
    with pytest.raises(ValueError):
        ParamsParser(["params_file.ini", "oops"])


def test_udf_defaults():
    c = config_from_params(ParamsParser([]))
    assert c.init_type == "UDF"
    assert c.grid["Pres"] == 200 and c.grid["Ures"] == (200, 200)
    assert c.grid["Pscale"] == "logarithmic" and c.grid["Uscale"] == ("linear", "quadratic")
    assert c.solver["dt"] == 0.005 and c.solver["statsEvery"] == 25
    assert c.init["R0"] == 2 and c.init["alpha"] == 0.5


def test_pldf_velocity_range_from_dispersion():
    c = config_from_dict({"type": "PLDF", "alpha": 1.0, "eta": 0.1})
    n, M, eta, alpha = 1.0, 1.0, 0.1, 1.0
    R0 = 1 / eta
    sigO2 = (3 - n) / (5 - 2 * n) * (M * eta) / (R0 * (alpha * 0.5 + 1))
    sig2 = sigO2 + 2 * (sigO2 * 0.5 * alpha)
    assert c.grid["Umax"][0] == pytest.approx(16 * math.sqrt(sig2), rel=1e-15)
    assert c.init["R0_given"] == 0


def test_hernquist_defaults_use_log_J():
    c = config_from_dict({"type": "Hernquist"})
    assert c.grid["Uscale"][1] == "logarithmic"
    assert c.solver["dt"] == 0.025


def test_uppercase_scale_rejected():
    # scale names are lowercase in the reference (scale.hxx:25-29)
    with pytest.raises(ValueError):
        config_from_params(ParamsParser(["-grid.Pscale", "LOGARITHMIC"]))


def test_unknown_profile_rejected():
    with pytest.raises(ValueError):
        config_from_params(ParamsParser(["-init.type", "PLUMMER"]))
