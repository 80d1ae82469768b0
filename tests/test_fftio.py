"""Host-side fault injection on the search's input files (no GPU): a truncated
or padded .fft and malformed .inf files are reported as JERK_EINVAL errors
naming the file and the field, where the reference either searches the wrong
number of bins silently (the bin count comes from the .fft's length alone,
src/accel_utils.c:1763) or ends the process (readinf, src/ioinf.c:20-240).
Well-formed files load with the N and dt the reference reads."""

import os

import numpy as np
import pytest

from prestozl_b200 import fftio, synth
from prestozl_b200.jerk import JERK_EINVAL, JerkError
from tests import helpers as H

N, DT = 1 << 16, 64e-6


@pytest.fixture
def pair(tmp_path):
    rng = np.random.default_rng(3)
    spec = (rng.standard_normal(N // 2) + 1j * rng.standard_normal(N // 2)).astype(np.complex64)
    root = str(tmp_path / "spec")
    synth.write_fft(root, spec, N, DT)
    return root, spec


def _raises(root, text):
    with pytest.raises(JerkError) as ei:
        fftio.load_fft(root)
    assert ei.value.code == JERK_EINVAL
    assert text in str(ei.value), str(ei.value)


def test_well_formed_pair_loads(pair):
    root, spec = pair
    got, n, dt = fftio.load_fft(root)
    assert (n, dt) == (N, DT)
    assert np.array_equal(np.asarray(got), spec)


def test_real_telescope_form_loads(tmp_path):
    """An .inf of a real observation (instrument, object, RA/DEC, observer,
    MJD and barycentring lines before N), in the layout readinf reads."""
    root = str(tmp_path / "obs")
    np.zeros(N // 2, np.complex64).tofile(root + ".fft")

    def line(k, v):
        return " " + k.ljust(39) + "=  " + str(v) + "\n"

    with open(root + ".inf", "w") as f:
        f.write(line("Data file name without suffix", "obs"))
        f.write(line("Telescope used", "GBT"))
        f.write(line("Instrument used", "GUPPI"))
        f.write(line("Object being observed", "J0000+0000"))
        f.write(line("J2000 Right Ascension (hh:mm:ss.ssss)", "00:00:00.0000"))
        f.write(line("J2000 Declination     (dd:mm:ss.ssss)", "00:00:00.0000"))
        f.write(line("Data observed by", "nobody"))
        f.write(line("Epoch of observation (MJD)", "60000.000000000000000"))
        f.write(line("Barycentered?           (1=yes, 0=no)", 1))
        f.write(line("Number of bins in the time series", N))
        f.write(line("Width of each time series bin (sec)", DT))
        f.write(line("Any breaks in the data? (1=yes, 0=no)", 0))
    _, n, dt = fftio.load_fft(root)
    assert (n, dt) == (N, DT)


@pytest.mark.parametrize("nbins", [N // 2 - 1, N // 2 + 5, 0])
def test_wrong_length_fft_is_rejected(pair, nbins):
    root, spec = pair
    out = np.zeros(nbins, np.complex64)
    out[: min(nbins, len(spec))] = spec[: min(nbins, len(spec))]
    out.tofile(root + ".fft")
    _raises(root, "truncated or from another series")


def test_partial_value_fft_is_rejected(pair):
    root, spec = pair
    with open(root + ".fft", "ab") as f:
        f.write(b"\0\0\0")
    _raises(root, "whole number of complex64")


def test_missing_files_are_reported(pair):
    root, _ = pair
    os.remove(root + ".fft")
    _raises(root, "cannot open")
    _raises(root + "_none", "cannot open")


@pytest.mark.parametrize("edit,text", [
    (lambda L: L[:3], "the bin width"),                                     # ends early
    (lambda L: L[:2] + ["\n"] + L[3:], "blank line while looking for the number of bins"),
    (lambda L: L[:2] + [" Number of bins in the time series 65536\n"] + L[3:],
     "no '=' between key and value of the number of bins"),
    (lambda L: L[:2] + [L[2].replace("65536", "lots")] + L[3:], "number for the number of bins"),
    (lambda L: L[:3] + [L[3].replace("6.4e-05", "-6.4e-05")] + L[4:], "not a positive number"),
    (lambda L: L[:2] + [L[2].replace("65536", "65536.5")] + L[3:], "not an integer"),
], ids=["truncated", "blank", "no-equals", "not-a-number", "negative-dt", "fractional-N"])
def test_malformed_inf_is_rejected(pair, edit, text):
    root, _ = pair
    with open(root + ".inf") as f:
        lines = f.readlines()
    with open(root + ".inf", "w") as f:
        f.writelines(edit(lines))
    _raises(root, text)


def test_values_match_the_reference_reader(pair):
    """N and dt as the reference's readinf / create_accelobs read them."""
    from oracle import bindings as ob

    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) reads the pair")
    root, _ = pair
    ref = ob.RefSearch(root + ".fft", ["-zmax", "0", "-numharm", "1"])
    _, n, dt = fftio.load_fft(root)
    assert (n, dt) == (int(ref.obs.N), ref.obs.dt)
    assert ref.obs.numbins == n // 2
    ref.close()
