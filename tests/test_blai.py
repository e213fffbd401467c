"""The bla.i / sgs.i readers (simson_b200.blai) on the CPU: the record order
and branches of bla/rparambl.f and bla/rparamles.f, the derived values
(icfl, vart, dtmax, cflmax), the reference's own example decks where the
reference sources are present, and the errors for decks the reference
rejects or this library does not run; the amp.stat number format and the
variable-time-step rule of the driver."""
import os

import pytest

from deck import bla_i
from simson_b200 import blai


def _reference_root():
    from build_ref import REF_ROOT  # where the oracle recipe finds the reference sources
    return REF_ROOT


REF = _reference_root()


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_channel_deck_records_and_derived_values(tmp_path):
    p = write(tmp_path, "bla.i", bla_i(tmax=50.0, maxit=-40, dt=0.0, nst=4, icfl=6, iamp=16, ixys=30,
                                       saves=((10.0, "t10.u"), (20.5, "t20.u"))))
    b = blai.read_bla_i(p)
    assert (b.namnin, b.namnut, b.tmax, b.maxit, b.nst) == ("init.u", "end.u", 50.0, 0, 4)
    assert b.vart and b.dtmax == 1.0e30
    assert abs(b.cflmax - 0.8 * 8 ** 0.5) < 1e-15
    assert b.icfl == 4          # min(icfl/nst*nst, 3 nst)
    assert b.ixys == 28         # max(ixys, nst)/nst*nst
    assert (b.iamp, b.namamp) == (16, "amp.stat")
    assert b.tsave == [10.0, 20.5] and b.nmsave == ["t10.u", "t20.u"]
    assert blai.unsupported(b) == []


def test_fixed_and_bounded_time_steps(tmp_path):
    b = blai.read_bla_i(write(tmp_path, "a.i", bla_i(dt=0.01, nst=3, icfl=0)))
    assert not b.vart and b.icfl == 0 and abs(b.cflmax - 0.8 * 3 ** 0.5) < 1e-15
    b = blai.read_bla_i(write(tmp_path, "b.i", bla_i(dt=-0.02, nst=3, icfl=0)))
    assert b.vart and b.dtmax == 0.02 and b.icfl == 3  # dt <= 0 and icfl <= 0: icfl = nst
    b = blai.read_bla_i(write(tmp_path, "c.i", bla_i(dt=0.01, nst=3, icfl=2)))
    assert b.icfl == 3  # 0 < icfl < nst: icfl = nst


def test_constant_re_tau_branch_reads_retau(tmp_path):
    b = blai.read_bla_i(write(tmp_path, "bla.i", bla_i(cflux=False, retau=395.0)))
    assert not b.cflux and b.retau == 395.0
    assert blai.unsupported(b) == []  # px = -(Re_tau/Re)^2 (bla/bla.f:1645)


def test_spatial_deck_records(tmp_path):
    b = blai.read_bla_i(write(tmp_path, "bla.i", bla_i(spat=True, cflux=False, retau=0.0, rbfl="baseflow.u",
                                                       xl=48.0, fringe=(2.0, -10.0, -1.0, 5.0, 2.0))))
    assert b.spat and b.rbfl and b.nambfl == "baseflow.u" and not b.tabfre
    assert (b.fmax, b.fstart, b.fend, b.frise, b.ffall) == (2.0, -10.0, -1.0, 5.0, 2.0)
    assert b.cdev == 0.0 and blai.unsupported(b) == []
    b = blai.read_bla_i(write(tmp_path, "w.i", bla_i(spat=True, xl=48.0, ampob=0.1)))
    assert "wave forcing in the fringe (ampob, amp2d)" in blai.unsupported(b)
    # rparambl.f:1898-1912: fstart < fend inside the box, positive distances and strength
    for bad in ((1.0, 0.0, -13.0, 7.0, 3.0), (0.0, -13.0, 0.0, 7.0, 3.0), (1.0, -13.0, 0.0, -7.0, 3.0),
                (1.0, -13.0, 7.0, 7.0, 3.0)):
        with pytest.raises(blai.DeckError, match="fstart < fend"):
            blai.read_bla_i(write(tmp_path, "f.i", bla_i(spat=True, xl=12.0, fringe=bad)))


def test_rejected_decks(tmp_path):
    with pytest.raises(blai.DeckError, match="Wrong version"):
        blai.read_bla_i(write(tmp_path, "v.i", bla_i().replace("20070716", "20060101")))
    with pytest.raises(blai.DeckError, match="nst must be 3"):
        blai.read_bla_i(write(tmp_path, "n.i", bla_i(nst=2)))
    with pytest.raises(blai.DeckError, match="end of file"):
        blai.read_bla_i(write(tmp_path, "t.i", "\n".join(bla_i().splitlines()[:12]) + "\n"))
    with pytest.raises(blai.DeckError, match="expected a logical"):
        blai.read_bla_i(write(tmp_path, "l.i", bla_i().replace(".true.         Variable", "maybe  Variable")))


def test_sgs_deck(tmp_path):
    s = blai.read_sgs_i(write(tmp_path, "sgs.i", "20060909\n# ADM-RT\n 1\n1.5\n5\n0.2\n"))
    assert (s.iles, s.cutoff_inv, s.iord, s.chi) == (1, 1.5, 5, 0.2)
    s = blai.read_sgs_i(write(tmp_path, "sgs2.i", "20060909\n2\n0.\n2\n"))
    assert (s.iles, s.cs, s.ineg) == (2, 0.0, 2)
    s = blai.read_sgs_i(write(tmp_path, "sgs3.i", "20060909\n2\n0.1\n"))
    assert (s.iles, s.cs, s.ineg) == (2, 0.1, 1)
    with pytest.raises(blai.DeckError, match="Wrong version of sgs.i"):
        blai.read_sgs_i(write(tmp_path, "sgs4.i", "20070716\n1\n"))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "examples")), reason="reference sources not present")
@pytest.mark.parametrize("example", ["channel", "temporal-channel-retau180"])
def test_reference_example_decks(example):
    b = blai.read_bla_i(os.path.join(REF, "examples", example, "bla.i"))
    assert b.nst == 4 and b.vart and b.icfl == 4 and b.msave == 5
    assert blai.unsupported(b) == []
    s = blai.read_sgs_i(os.path.join(REF, "examples", "spatial-blasius-les", "sgs.i"))
    assert (s.iles, s.cutoff_inv, s.iord, s.chi) == (1, 1.5, 5, 0.2)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "examples")), reason="reference sources not present")
def test_reference_spatial_example_decks():
    b = blai.read_bla_i(os.path.join(REF, "examples", "spatial-channel-couette", "bla.i"))
    assert b.spat and b.rbfl and b.nambfl == "baseflow.u" and not b.cflux and b.nst == 4
    assert (b.fmax, b.fstart, b.fend, b.frise, b.ffall) == (1.0, -13.0, 0.0, 7.0, 3.0)
    assert blai.unsupported(b) == []
    b = blai.read_bla_i(os.path.join(REF, "examples", "spatial-blasius-les", "bla.i"))
    assert b.spat and b.fstart == -70.0 and b.sgs
    bad = blai.unsupported(b)
    assert "boundary condition ibc = 110" in bad and "trip forcing" in bad


def test_amp_stat_number_format():
    from simson_b200.driver import fortran_e
    assert fortran_e(1.0) == "  0.1000000000000000E+001"
    assert fortran_e(-1.23456789e-4) == " -0.1234567890000000E-003"
    assert fortran_e(0.0) == "  0.0000000000000000E+000"
    assert fortran_e(9.99999999999999999) == "  0.1000000000000000E+002"
    assert all(len(fortran_e(v)) == 25 for v in (3.5e200, -7.25e-150, 1.0))


def test_next_time_step_rule():
    from simson_b200.driver import next_dt
    cflmax = 0.8 * 8 ** 0.5
    # far from the next save: the CFL rule alone (bla/bla.f:2362-2367)
    assert next_dt(0.1, 2 * cflmax, cflmax, 1e30, 0.0, 1e30, 0.0) == 0.1 * cflmax / (2 * cflmax)
    assert abs(next_dt(0.1, cflmax, cflmax, 1e30, 0.0, 1e30, 0.0) - 0.1) < 1e-15
    assert next_dt(0.1, 0.5 * cflmax, cflmax, 0.05, 0.0, 1e30, 0.0) == 0.05
    # a save time two and a half steps ahead: the step is shortened to land on it
    dt = next_dt(0.1, cflmax, cflmax, 1e30, 0.0, 0.35, 0.0)
    assert abs(dt - 0.25 / 3) < 1e-15
