"""The search's input from a time series on the GPU (jerk_realfft,
jerk_deredden, jerk_spectrum_from_timeseries): the steps the reference takes
for a ".dat" input (src/accel_utils.c:1696-1753).

Tolerances:
  * real FFT (FP32, like the reference's FFTW single-precision path): as
    accurate as a standard single-precision FFT library on the same input --
    scipy.fft's FP32 transform (pocketfft) -- against the FP64 transform: the
    rms error at most 1.5 times scipy's (the norm-wise FFT accuracy), and the
    largest bin error at most 4 times scipy's, both over the spectrum's rms
    magnitude.  (The largest error sits in one of the few red-noise bins
    hundreds of times the rms, where the rounding of that one value decides
    it; per-bin error profiles also differ between FFT algorithms, as errors
    from those bins spread over the bins that share their butterflies.  A
    defect shows as orders of magnitude.)
  * red-noise removal: bit-exact against the oracle and the reference build
  * search from a .dat file: the candidate list of the reference's CPU
    accelsearch on the same file, except entries within 1e-4 of a cutoff;
    powers and sigmas to 1e-5
"""

import numpy as np
import pytest
import scipy.fft as scipy_fft

from oracle import bindings as ob
from prestozl_b200 import build, jerk, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def built():
    build.build()
    H.ensure_oracle()


def red_series(n: int, seed: int) -> np.ndarray:
    """White noise plus a random walk (red noise) plus two sinusoids."""
    rng = np.random.default_rng(seed)
    t = np.arange(n)
    x = rng.standard_normal(n) + 0.02 * np.cumsum(rng.standard_normal(n))
    x += 0.3 * np.sin(2 * np.pi * 0.1234567 * t) + 0.05 * np.sin(2 * np.pi * 0.0377 * t + 1.0)
    return x.astype(np.float32)


def gpu_realfft(x: np.ndarray) -> np.ndarray:
    d = torch.from_numpy(x).cuda()
    out = jerk.realfft(d)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("n", [1 << 15, 1 << 16, 1 << 20, 3 << 20, 5 << 21, 15 << 20, 1 << 25],
                         ids=["2^15", "2^16", "2^20", "3*2^20", "5*2^21", "15*2^20", "2^25"])
def test_realfft_matches_fp64(n):
    """Powers of two and mixed lengths (M = n/2 = 768 x 2048, 4096 x 1280,
    7680 x 1024)."""
    x = red_series(n, n % 1000003)
    got = gpu_realfft(x).astype(np.complex128)
    want = ob.packed_rfft(x)
    rms = float(np.sqrt(np.mean(np.abs(want) ** 2)))
    X = scipy_fft.rfft(x)
    assert X.dtype == np.complex64
    lib = X[: n // 2].astype(np.complex128)
    lib[0] = complex(X[0].real, X[n // 2].real)
    err, lib_err = np.abs(got - want) / rms, np.abs(lib - want) / rms
    rms_err, lib_rms = float(np.sqrt(np.mean(err ** 2))), float(np.sqrt(np.mean(lib_err ** 2)))
    print(f"n={n}: max err {err.max():.2e} (scipy FP32 {lib_err.max():.2e}), "
          f"rms err {rms_err:.2e} (scipy FP32 {lib_rms:.2e})")
    assert err.max() <= 4.0 * lib_err.max(), (float(err.max()), int(np.argmax(err)))
    assert rms_err <= 1.5 * lib_rms


def test_realfft_largest_size_by_parseval_and_spot_bins():
    """n = 2^27 (R1 = R2 = 8192): Parseval's sum and four bins summed
    directly in FP64."""
    n = 1 << 27
    rng = np.random.default_rng(27)
    x = rng.standard_normal(n, dtype=np.float32)
    got = gpu_realfft(x)
    x64 = x.astype(np.float64)
    dc, nyq = float(got[0].real), float(got[0].imag)
    e_time = float(np.dot(x64, x64))
    e_freq = (dc * dc + nyq * nyq + 2.0 * float(np.sum(np.abs(got[1:].astype(np.complex128)) ** 2))) / n
    assert abs(e_freq - e_time) <= 1e-5 * e_time, (e_freq, e_time)
    assert abs(dc - x64.sum()) <= 1e-5 * np.sqrt(n) * 10
    t = np.arange(n, dtype=np.float64)
    for k in (1, 12345, n // 8 + 3, n // 2 - 1):
        want = complex(np.sum(x64 * np.cos(2 * np.pi * ((k * t) % n) / n)),
                       -np.sum(x64 * np.sin(2 * np.pi * ((k * t) % n) / n)))
        assert abs(complex(got[k]) - want) <= 2e-6 * np.sqrt(n) * 20, (k, got[k], want)


def test_realfft_in_place_equals_out_of_place():
    x = red_series(1 << 20, 5)
    d = torch.from_numpy(x).cuda()
    a = jerk.realfft(d)
    b = jerk.realfft(d, out=d.view(torch.complex64))
    torch.cuda.synchronize()
    assert torch.equal(torch.view_as_real(a), torch.view_as_real(b))


@pytest.mark.parametrize("numamps", [8, 13, 100, 12345, 1000003])
def test_deredden_bit_exact_on_random_spectra(numamps):
    rng = np.random.default_rng(numamps)
    f = np.arange(numamps) + 1.0
    amp = 10.0 / np.sqrt(f) + 1.0
    spec = (rng.standard_normal(numamps) * amp + 1j * rng.standard_normal(numamps) * amp)
    spec = spec.astype(np.complex64)
    d = torch.from_numpy(spec.copy()).cuda()
    jerk.deredden(d)
    got = d.cpu().numpy()
    want = ob.deredden(spec)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if H.have_ref():
        assert np.array_equal(want.view(np.uint32), ob.deredden(spec, True).view(np.uint32))


def test_spectrum_from_timeseries_paper_size():
    """2^25 samples (the paper's length): realfft then deredden on the GPU;
    the deredden step bit-exact against the oracle applied to the GPU's own
    realfft output, bin 0 = (1, 1)."""
    n = 1 << 25
    x = red_series(n, 2025)
    d = torch.from_numpy(x).cuda()
    raw = jerk.realfft(d).cpu().numpy()
    spec = jerk.spectrum_from_timeseries(d)
    torch.cuda.synchronize()
    got = spec.cpu().numpy()
    want = ob.deredden(raw)
    want[0] = 1.0 + 1.0j
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # red noise removed: power levels flat across the band
    p = np.abs(got[1:]) ** 2
    lo, hi = float(np.median(p[100:10000])), float(np.median(p[-100000:]))
    assert 0.5 < lo / hi < 2.0, (lo, hi)


def test_search_from_dat_file_matches_reference(tmp_path):
    """A .dat time series searched end to end: the reference's CPU accelsearch
    reads it, FFTs and dereddens it and searches; here the GPU does all three
    (jerk_spectrum_from_timeseries, then the search)."""
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) runs the .dat search")
    N, dt = 1 << 20, 64e-6
    ts = synth.timeseries(N, dt, synth.small_pulsar(), 20241203)
    ts = ts + (0.02 * np.cumsum(np.random.default_rng(9).standard_normal(N))).astype(np.float32)
    root = str(tmp_path / "series")
    ts.astype(np.float32).tofile(root + ".dat")
    synth.write_inf(root, N, dt)
    args = list(H.golden("small_cands.json")["args"])
    ob.set_threads(1)
    ref = ob.RefSearch(root + ".dat", args)
    obs = jerk.obs_from_refobs(ref.obs)
    subs = []
    for st, h in ref.subharmonics():
        info = ref.shi_info(st, h)
        info["kern"] = ref.kernels(st, h)
        subs.append(info)
    d = torch.from_numpy(ts.astype(np.float32)).cuda()
    spec = jerk.spectrum_from_timeseries(d)
    torch.cuda.synchronize()
    plan = jerk.JerkPlan(obs, subs, batch=16)
    got = plan.search(spec)
    plan.close()
    ref.make_bank()
    want, _ = ref.search()
    ref.close()
    assert len(want) > 0
    probs = H.compare_cands(got, want, list(obs.powcut))
    assert not probs, probs[:10]
    print(f".dat search: {len(got)} candidates (reference {len(want)})")


def test_zap_birdies_bit_exact():
    """Birdie zapping on the GPU equals the oracle's zapbirds loop bitwise on
    a spectrum made on the GPU from a 2^20-sample series: ordinary and
    overlapping birdies, one clamped at the top, one below 301 bins (left
    alone), one at N/2 (stops the list) and one after it (not zapped)."""
    N = 1 << 20
    x = red_series(N, 77)
    spec = jerk.spectrum_from_timeseries(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    before = spec.cpu().numpy()
    lob = [1000.3, 1030.0, 250.0, 88888.25, 200000.0, N / 2 - 20.5, N / 2, 300000.0]
    hib = [1040.7, 1060.2, 260.0, 88890.0, 200000.0, N / 2 + 30.0, N / 2 + 5, 300010.0]
    jerk.zap_birdies(spec, N, lob, hib)
    got = spec.cpu().numpy()
    want = ob.zap_list(before, N, lob, hib)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert got[1020] == got[1000] and got[1020].imag == 0  # zapped
    assert got[300005] == before[300005]  # after the stop
    assert got[255] == before[255]  # below the threshold


def test_spectrum_from_timeseries_mixed_length():
    """A series of 15 * 2^20 samples (M = 7680 x 1024), a length with
    factors 3 and 5 as dedispersion tools choose them: realfft then deredden,
    the deredden step bit-exact against the oracle applied to the GPU's own
    realfft output, bin 0 = (1, 1)."""
    n = 15 << 20
    x = red_series(n, 15)
    d = torch.from_numpy(x).cuda()
    raw = jerk.realfft(d).cpu().numpy()
    got = jerk.spectrum_from_timeseries(d).cpu().numpy()
    want = ob.deredden(raw)
    want[0] = 1.0 + 1.0j
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
