"""The NDfield snapshot the reference wrote (tests/golden/udf_tiny_snapshot_step1.ND,
Save_NDfield NDfield.hxx:308-363 of NDfieldFromData vlasovSolver21.hxx:717-773),
read field by field on the host: the layout the library's writer must
reproduce byte for byte (tests/test_gpu_parity.py compares the two files)."""
import os
import struct

import numpy as np

from conftest import GOLDEN, load_golden

ND = os.path.join(GOLDEN, "udf_tiny_snapshot_step1.ND")


def test_reference_ndfield_layout():
    b = open(ND, "rb").read()
    g, cfg = load_golden("udf_tiny")
    nj, nu, nr = (int(x) for x in g["shape"])
    n = nr * nu * nj
    # tag record: 16-byte tag framed by int markers
    assert struct.unpack_from("<i16si", b, 0) == (16, b"NDFIELD" + b"\0" * 9, 16)
    # header record of 652 bytes: comment[80], ndims, dims[20], fdims_index,
    # datatype, x0[20], delta[20], dummy[160]
    off = 24
    assert struct.unpack_from("<i", b, off)[0] == 652
    comment = b[off + 4: off + 84]
    assert comment.rstrip(b"\0") == b"1 1 0 1 2 0"  # Rscale VERTEX Uscale VERTEX Jscale CELL
    ndims = struct.unpack_from("<i", b, off + 84)[0]
    dims = struct.unpack_from("<20i", b, off + 88)
    assert ndims == 3 and dims[:3] == (nr, nu, nj) and not any(dims[3:])
    fdi, dtype = struct.unpack_from("<2i", b, off + 168)
    assert fdi == 0 and dtype == 1 << 9  # ND_DOUBLE
    x0 = struct.unpack_from("<20d", b, off + 176)
    delta = struct.unpack_from("<20d", b, off + 336)
    assert x0[:3] == (cfg["Pmin"], cfg["Umin"][0], cfg["Umin"][1])
    assert delta[:3] == (cfg["Pmax"] - cfg["Pmin"], cfg["Umax"][0] - cfg["Umin"][0],
                         cfg["Umax"][1] - cfg["Umin"][1])
    assert struct.unpack_from("<i", b, off + 656)[0] == 652
    # data record: int marker n*8, n doubles [j][u][r], marker
    d0 = off + 660
    assert d0 == 684 and len(b) == d0 + 4 + 8 * n + 4
    assert struct.unpack_from("<i", b, d0)[0] == 8 * n
    assert struct.unpack_from("<i", b, len(b) - 4)[0] == 8 * n
    f = np.frombuffer(b[d0 + 4: d0 + 4 + 8 * n], "<f8").reshape(nj, nu, nr)
    # the same binary's run of the same case after one step
    np.testing.assert_array_equal(f, g["f_1"])


def test_record_marker_wraps_like_a_c_int():
    """The reference stores the data record's byte count in an int
    (NDfield.hxx:355), so above 2 GiB the marker is the count modulo 2^32 read
    as a signed int; the library writes the same bits (checked on a grid of
    1025 x 1025 x 256 cells in tests/test_gpu_parity.py)."""
    n = 1025 * 1025 * 256
    wrapped = struct.unpack("<i", struct.pack("<I", (8 * n) % 2 ** 32))[0]
    assert 8 * n > 2 ** 31 and wrapped == 8 * n - 2 ** 32
