"""The .u field file (simson_b200/ufile.py) on the CPU: the byte layout of
bla/wdiscbl.f, the round trip, the resolution changes of bla/rdiscbl.f (x/z
modes truncated or padded, y refined by Chebyshev re-expansion, which is
exact for the polynomials the coarse grid resolves) and the files the
reader must refuse (corrupt markers, truncation, unknown flow type, a y
resolution reduction)."""
import struct

import numpy as np
import pytest

from simson_b200.ufile import UFileError, read_u, write_u


def fields(nx, ny, nz, seed=0, m=3):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((nz, ny, nx // 2)) + 1j * rng.standard_normal((nz, ny, nx // 2)) for _ in range(m)]


def test_byte_layout(tmp_path):
    nx, ny, nz = 8, 9, 6
    q = fields(nx, ny, nz)
    p = tmp_path / "a.u"
    write_u(p, q, re=4200.0, xl=12.5, zl=6.25, t=1.5, dstar=1.0, fltype=1)
    b = p.read_bytes()
    rec = [(44, 0), (16, 52), (12, 76)]
    for n, off in rec:
        assert struct.unpack_from("<i", b, off)[0] == n and struct.unpack_from("<i", b, off + 4 + n)[0] == n
    assert struct.unpack_from("<di4d", b, 4) == (4200.0, 0, 12.5, 6.25, 1.5, 0.0)
    assert struct.unpack_from("<4i", b, 56) == (nx, ny, nz, 0)
    assert struct.unpack_from("<id", b, 80) == (1, 1.0)
    data0 = 96
    assert len(b) == data0 + 3 * nz * ny * (8 + 8 * nx)
    # second record of the data: field 1, z = 1, y = 2, re/im interleaved
    off = data0 + (8 + 8 * nx) + 4
    row = np.frombuffer(b, "<f8", nx, off)
    assert np.array_equal(row[0::2], q[0][0, 1].real) and np.array_equal(row[1::2], q[0][0, 1].imag)


def test_round_trip(tmp_path):
    q = fields(16, 17, 12, 3)
    p = tmp_path / "b.u"
    write_u(p, q, 3000.0, 6.0, 3.0, 7.25, fltype=2)
    head, back = read_u(p)
    assert head["re"] == 3000.0 and head["t"] == 7.25 and head["fltype"] == 2 and head["nzc"] == 12
    for a, c in zip(q, back):
        assert np.array_equal(a, c)


def test_extra_header_records(tmp_path):
    q = fields(8, 9, 4)
    p = tmp_path / "c.u"
    write_u(p, q, 400.0, 100.0, 10.0, 0.0, fltype=7, bstart=10.0, blength=20.0, rlam=0.1, spanv=0.2)
    head, back = read_u(p)
    assert (head["bstart"], head["blength"], head["rlam"], head["spanv"]) == (10.0, 20.0, 0.1, 0.2)
    assert np.array_equal(back[1], q[1])


def test_resolution_change_x_z(tmp_path):
    nx, ny, nz = 8, 9, 8
    q = fields(nx, ny, nz, 5)
    for f in q:
        f[nz // 2] = 0.0
    p = tmp_path / "d.u"
    write_u(p, q, 1.0, 1.0, 1.0, 0.0)
    _, big = read_u(p, nx=16, nz=16)
    for a, c in zip(q, big):
        assert np.array_equal(c[:4, :, :4], a[:4])          # kz = 0..3
        assert np.array_equal(c[-3:, :, :4], a[-3:])        # kz = -3..-1
        assert not c[4:13].any() and not c[:, :, 4:].any()  # new modes, and the file's kz = -4
    _, small = read_u(p, nx=4, nz=4)
    for a, c in zip(q, small):
        assert np.array_equal(c[:2], a[:2, :, :2]) and np.array_equal(c[2:], a[-2:, :, :2])


def test_y_refinement_is_exact_for_resolved_polynomials(tmp_path):
    nx, nz = 4, 4
    y9 = np.cos(np.pi * np.arange(9) / 8)
    y17 = np.cos(np.pi * np.arange(17) / 16)
    prof = lambda y: 1 - y ** 2 + 0.3 * y ** 5 - 0.1 * y ** 8  # degree 8 < 9 points
    q = np.zeros((nz, 9, nx // 2), complex)
    q[0, :, 0] = prof(y9)
    q[1, :, 1] = (1 + 2j) * prof(y9)
    p = tmp_path / "e.u"
    write_u(p, [q, q, q], 1.0, 1.0, 1.0, 0.0)
    _, fine = read_u(p, nyp=17)
    assert np.abs(fine[0][0, :, 0] - prof(y17)).max() < 1e-13
    assert np.abs(fine[0][1, :, 1] - (1 + 2j) * prof(y17)).max() < 1e-13
    with pytest.raises(UFileError):
        read_u(p, nyp=5)  # rdiscbl cannot reduce y


def test_refuses_corrupt_files(tmp_path):
    q = fields(8, 9, 4)
    p = tmp_path / "f.u"
    write_u(p, q, 1.0, 1.0, 1.0, 0.0)
    good = p.read_bytes()
    bad = tmp_path / "g.u"
    bad.write_bytes(good[:-5])                       # truncated
    with pytest.raises(UFileError):
        read_u(bad)
    b = bytearray(good)
    b[48:52] = struct.pack("<i", 40)                 # trailing marker of the first record
    bad.write_bytes(bytes(b))
    with pytest.raises(UFileError):
        read_u(bad)
    b = bytearray(good)
    b[80:84] = struct.pack("<i", 42)                 # unknown flow type
    bad.write_bytes(bytes(b))
    with pytest.raises(UFileError):
        read_u(bad)
    b = bytearray(good)
    b[56:60] = struct.pack("<i", 7)                  # odd nx
    bad.write_bytes(bytes(b))
    with pytest.raises(UFileError):
        read_u(bad)
    with pytest.raises(UFileError):
        read_u(p, nx=16, varsiz=False)


def test_pressure_file(tmp_path):
    """bla/wdiscp.f's .p file: the velocity file's header and one field; its
    flow-type record differs for fltype >= 6 (four values, 20 included)."""
    from simson_b200.ufile import write_p
    (p,) = fields(8, 9, 6, 11, m=1)
    f = tmp_path / "field.u.p"
    write_p(f, p, 4200.0, 12.5, 6.25, 3.0)
    b = f.read_bytes()
    assert len(b) == 96 + 6 * 9 * (8 + 8 * 8)   # header as the .u file, one field
    head, (back,) = read_u(f, m=1, pressure_file=True)
    assert head["t"] == 3.0 and np.array_equal(back, p)
    write_p(f, p, 400.0, 100.0, 10.0, 0.0, fltype=20, bstart=1.0, blength=2.0, rlam=0.5, spanv=0.25)
    head, (back,) = read_u(f, m=1, pressure_file=True)
    assert (head["bstart"], head["blength"], head["rlam"], head["spanv"]) == (1.0, 2.0, 0.5, 0.25)
    assert np.array_equal(back, p)
    with pytest.raises(UFileError):  # read as a velocity file the fltype-20 record does not fit
        read_u(f, m=1)
