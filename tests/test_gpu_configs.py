"""Parity at the other search configurations (beyond the small spectrum and the
paper-scale run): the mixed geometries of the batched workload -- (zmax, wmax)
in {(50, 150 -> 160), (100, 0), (200, 300)}, numharm 8 / 16, 2^22 .. 2^24
samples -- and the memory-heavy one (zmax 300, wmax 600, numharm 32, fftlen
4096, 2^25 samples).

For each configuration:
  * the plan's geometry (numz, numw, corr_uselen, fftlen, cutoffs, numindep,
    every subharmonic's sizes) equals the reference's create_accelobs;
  * sampled ffdot volumes (first, middle and last rstep; fundamental, a middle
    and the highest subharmonic, and every one at the longest fftlen) from the
    CUDA path agree with the oracle's FP64 recomputation from the same kernel
    rows to 1e-5 relative to max(power, 1) -- whole volumes, or, where the
    kernels of one subharmonic exceed 256 MB, 9 sampled (w, z) rows, each row
    being its own correlation; the worst error is printed per configuration;
  * the candidate list over the first rsteps equals the reference CPU
    search's, except entries within 1e-4 of a stage cutoff (the memory-heavy
    configuration in its own test below, from a red-noise .dat with birdies
    and a zaplist, as that configuration is defined).
Spectra: seeded Gaussian noise plus injected pulsars (prestozl_b200.synth).
"""

import os

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu

DT = 54.6e-6
CONFIGS = {
    # name: (log2 N, zmax, wmax, numharm, sigma, rsteps compared with the reference)
    "n22_z50_w150_h8": (22, 50, 150, 8, 2.0, 8),
    "n22_z100_w0_h16": (22, 100, 0, 16, 2.0, 8),
    "n24_z200_w300_h8": (24, 200, 300, 8, 2.0, 3),
    "n25_z300_w600_h32": (25, 300, 600, 32, 4.0, 0),
    # FFT length 10240
    "n22_z600_w1200_h8": (22, 600, 1200, 8, 3.0, 0),
    # the longest supported FFT length (15360; one rstep per batch under the
    # 32-bit volume limit)
    "n22_z1200_w1500_h2": (22, 1200, 1500, 2, 3.0, 0),
}
POW_TOL = 1e-5


def _spectrum(logn: int, seed: int, extra=()):
    torch = pytest.importorskip("torch")
    N = 1 << logn
    pulsars = synth.random_pulsars(np.random.default_rng(seed), 2) + list(extra)
    spec = synth.presto_fft_torch(synth.timeseries_torch(N, DT, pulsars, seed, device="cuda"))
    out = spec.cpu().numpy()
    torch.cuda.synchronize()
    return out, N


@pytest.mark.parametrize("name", list(CONFIGS))
def test_configuration_matches_reference(name, tmp_path):
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) is needed")
    logn, zmax, wmax, numharm, sigma, nsteps = CONFIGS[name]
    N = 1 << logn
    obs, fftlen, _ = jerk.obs_from_params(N // 2, N, DT, zmax, wmax, numharm, sigma)
    # one more pulsar inside the rsteps compared with the reference search
    # (which starts at the first rstep)
    T = N * DT
    r_in = obs.rlo + (0.4 * max(nsteps, 1)) * (obs.corr_uselen // 2)
    psr = synth.Pulsar(f=r_in / T, z=0.5 * zmax, w=0.5 * wmax, snr=25.0, nharm=3)
    spec, N = _spectrum(logn, 1000 + logn, [psr])
    root = str(tmp_path / "spec")
    synth.write_fft(root, spec, N, DT)
    args = ["-zmax", str(zmax), "-wmax", str(wmax), "-numharm", str(numharm),
            "-sigma", str(sigma)]
    ob.set_threads(1)
    ref = ob.RefSearch(root + ".fft", args)
    ro = ref.obs

    # geometry
    assert (obs.numz, obs.numw, obs.corr_uselen, fftlen, obs.numharmstages) == \
        (ro.numz, ro.numw, ro.corr_uselen, ro.fftlen, ro.numharmstages)
    assert obs.lobin == ro.lobin and obs.highestbin == ro.highestbin
    for i in range(obs.numharmstages):
        assert obs.numindep[i] == ro.numindep[i]
        assert abs(obs.powcut[i] - ro.powcut[i]) <= 1e-6 * ro.powcut[i]
    subs = jerk.subharm_sizes(obs, fftlen)
    for (st, h), s in zip(ref.subharmonics(), subs):
        info = ref.shi_info(st, h)
        for k in ("numharm", "harmnum", "numz", "numw", "fftlen", "halfwidth"):
            assert info[k] == s[k], (name, st, h, k)

    bank = jerk.DeviceBank(subs)
    plan = jerk.JerkPlan(obs, subs, batch=4, device_bank=bank.ptr.value)
    nr = plan.num_rsteps
    geom = ob.geom_from_refobs(ro)
    rstep = ro.corr_uselen // 2
    worst = 0.0
    picks = sorted({0, len(subs) // 2, len(subs) - 1} |
                   {i for i, s in enumerate(subs) if s["fftlen"] == fftlen})
    for i in picks:
        sub = dict(subs[i])
        nrow = sub["numw"] * sub["numz"]
        rows = None
        if nrow * sub["fftlen"] * 8 <= (256 << 20):
            sub["kern"] = bank.rows(subs, i, range(nrow)).reshape(
                sub["numw"], sub["numz"], sub["fftlen"])
        else:
            ws = sorted({0, sub["numw"] // 2, sub["numw"] - 1})
            zs = sorted({0, sub["numz"] // 2, sub["numz"] - 1})
            rows = [w * sub["numz"] + z for w in ws for z in zs]
            sub["kern"] = bank.rows(subs, i, rows).reshape(1, len(rows), sub["fftlen"])
            sub["numw"], sub["numz"] = 1, len(rows)
        orc = ob.Oracle(spec, geom, [sub])
        for k in (0, nr // 2, nr - 1):
            startr = ro.rlo + k * rstep
            got, rlo = plan.volume(spec, k, i)
            h, want, _, _ = orc.fderivs(0, startr, startr + rstep - 0.5)
            if rows is not None:
                got = got.reshape(-1, got.shape[-1])[rows].reshape(want.shape)
            assert rlo == h["rlo"] and got.shape == want.shape
            err = float((np.abs(got.astype(np.float64) - want) / np.maximum(want, 1.0)).max())
            worst = max(worst, err)
            assert err <= POW_TOL, (name, i, k, err)
        del orc, sub
    print(f"{name}: max FP32 power error vs FP64 oracle over sampled volumes {worst:.3e}")

    if nsteps:
        ref.make_bank()
        want, done = ref.search(max_steps=nsteps)
        assert done == nsteps
        got = plan.search(spec, 0, nsteps)
        probs = H.compare_cands(got, want, list(ro.powcut))
        assert not probs, (name, probs[:10])
        assert len(want) > 0
    else:
        # the memory-heavy configuration: a full pass over a few rsteps runs and
        # its candidates are well formed
        got = plan.search(spec, nr // 2, 2)
        assert np.all(got["numharm"] >= 1) and np.all(got["sigma"] > 0)
    plan.close()
    bank.close()
    ref.close()


def test_memory_heavy_red_noise_and_birdies_match_reference(tmp_path):
    """The memory-heavy configuration end to end, as the reference runs it on
    a .dat input with -zaplist: a 2^25-sample series (dt 54.6 us) of red noise
    (power falling as f^-1.5 below 2 Hz over a white floor), 20 single-bin
    birdies and one pulsar, searched at -zmax 300 -wmax 600 -numharm 32
    -sigma 4.0.

    The reference's CPU accelsearch reads the .dat, FFTs it, removes the red
    noise (src/accel_utils.c:1557-1634), zaps the zaplist's birdies
    (src/accelsearch_lib.c:393-418, src/zapping.c:29-81) and searches.  Here
    the GPU does every step: jerk_spectrum_from_timeseries, jerk_zap_birdies,
    the kernel bank (jerk_bank_generate) and the search.
      * The GPU's dereddened and zapped spectrum equals, bitwise, the
        reference's own deredden and zapbirds applied to the GPU's real FFT,
        and differs from the spectrum the reference prepared itself only by
        the real FFT's rounding (rms difference at most 1e-5 of the rms; the
        GPU's FP32 real FFT is held to a single-precision library in
        test_gpu_input).
      * The candidate lists of the first two rsteps (1.0 - 2.7 Hz: the
        whitened red-noise band, two zapped birdies and the pulsar's
        fundamental) are equal except entries within 1e-4 of a cutoff;
        powers and sigmas agree to 1e-5.
    The reference searches on one thread (its threaded search calls
    dcdflib's cdfchi concurrently, which aborts at 32 harmonics)."""
    torch = pytest.importorskip("torch")
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) is needed")
    N, nsteps = 1 << 25, 2
    T = N * DT
    birdies = synth.memory_heavy_birdies()
    psr = synth.Pulsar(f=1.9, z=120.0, w=-200.0, snr=30.0, nharm=4, phase=0.3)
    x = synth.red_noise_timeseries(N, DT, 505, pulsars=[psr], birdies=birdies)
    root = str(tmp_path / "series")
    x.tofile(root + ".dat")
    synth.write_inf(root, N, DT)
    width = 0.003  # Hz: about 5.5 bins
    with open(root + ".zaplist", "w") as f:
        f.write("# freq width (Hz)\n")
        for fb in birdies:
            f.write(f"{fb!r} {width!r}\n")
    # get_birdies (src/birdzap.c:6-80) at zero velocity, sorted by lobin
    lob = sorted((fb - 0.5 * width) * T for fb in birdies)
    hib = sorted((fb + 0.5 * width) * T for fb in birdies)

    args = ["-zmax", "300", "-wmax", "600", "-numharm", "32", "-sigma", "4.0",
            "-zaplist", root + ".zaplist"]
    ob.set_threads(1)
    ref = ob.RefSearch(root + ".dat", args)
    ro = ref.obs
    obs, fftlen, _ = jerk.obs_from_params(N // 2, N, DT, 300, 600, 32, 4.0)
    assert (obs.numz, obs.numw, obs.numharmstages, fftlen) == (ro.numz, ro.numw, 6, ro.fftlen)

    # the spectrum, on the GPU, and its pin against the reference's own steps
    d = torch.from_numpy(x).cuda()
    raw = jerk.realfft(d).cpu().numpy()
    spec = jerk.spectrum_from_timeseries(d)
    jerk.zap_birdies(spec, N, lob, hib)
    got_spec = spec.cpu().numpy()
    want_spec = ob.deredden(raw, reference=True)
    want_spec[0] = 1.0 + 1.0j
    for lo, hi in zip(lob, hib):
        want_spec = ob.zapbirds(want_spec, lo, min(hi, N // 2 - 1), reference=True)
    assert np.array_equal(got_spec.view(np.uint32), want_spec.view(np.uint32))
    # the spectrum the reference prepared itself (its real FFT, deredden and
    # zapping) differs from the GPU's only by the real FFT's rounding
    rs = ref.spectrum()
    diff = np.abs(rs.astype(np.complex128) - got_spec)
    rms = float(np.sqrt(np.mean(np.abs(rs.astype(np.complex128)) ** 2)))
    assert float(np.sqrt(np.mean(diff ** 2))) <= 1e-5 * rms

    subs = jerk.subharm_sizes(obs, fftlen)
    bank = jerk.DeviceBank(subs)
    plan = jerk.JerkPlan(obs, subs, batch=2, device_bank=bank.ptr.value)
    got = plan.search(spec, 0, nsteps)
    torch.cuda.synchronize()
    plan.close()
    bank.close()
    del spec, d

    ref.make_bank()
    want, done = ref.search(max_steps=nsteps)
    ref.close()
    assert done == nsteps and len(want) > 0
    probs = H.compare_cands(got, want, list(ro.powcut))
    assert not probs, probs[:10]
    # the pulsar is found near its fundamental; no birdie survives the zapping
    assert np.any(np.abs(got["r"] - 1.9 * T) < 2.0)
    for fb in birdies[:2]:
        assert not np.any(np.abs(got["r"] - fb * T) < 1.0), fb
    print(f"memory-heavy red noise + birdies: {len(got)} candidates (reference {len(want)})")
