"""The .vls restart reader on the reference's own restart files (no GPU
needed for vls_restart_info), and its error behaviour on damaged files."""
import os

import pytest

from conftest import GOLDEN


def info(name):
    from vlasolve_b200.build import build
    from vlasolve_b200.solver import restart_info
    build()
    return restart_info(os.path.join(GOLDEN, name))


def test_restart_info_of_reference_files():
    a = info("udf_tiny_restart_step2.vls")
    assert (a["time"], a["step"]) == (0.01, 2)
    assert (a["Pmin"], a["Pmax"], a["Pres"], a["Pscale"]) == (0.01, 25.0, 16, "logarithmic")
    # the J minimum is not in the file (paramT::write, grid_base.hxx:129-130)
    assert a["Umin"] == (-2.0, 0.0) and a["Umax"] == (2.0, 1.6)
    assert a["Ures"] == (16, 8) and a["Uscale"] == ("linear", "quadratic")
    assert (a["G"], a["dt"], a["Tmax"], a["noLinking"]) == (1.0, 0.005, 0.0125, 0)
    assert (a["kernelType"], a["kernelBufferSize"]) == ("delayed", 0)
    assert (a["snapshotEvery"], a["restartEvery"], a["statsEvery"]) == (-1, 2, -1)
    b = info("udf_tiny_final_step3.vls")
    assert (b["time"], b["step"]) == (0.015, 3)


def test_damaged_restart_files_are_errors(tmp_path):
    from vlasolve_b200._lib import VlsError
    src = open(os.path.join(GOLDEN, "udf_tiny_restart_step2.vls"), "rb").read()
    short = tmp_path / "short.vls"
    short.write_bytes(src[:100])
    with pytest.raises(VlsError):
        info(str(short))
    bad = bytearray(src)
    bad[8] ^= 0xFF  # inside the first tag
    p = tmp_path / "badtag.vls"
    p.write_bytes(bytes(bad))
    with pytest.raises(VlsError):
        info(str(p))
    with pytest.raises(VlsError):
        info(str(tmp_path / "missing.vls"))
