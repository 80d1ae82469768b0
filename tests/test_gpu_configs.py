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
  * (except the memory-heavy one, whose reference bank takes minutes on one
    CPU core) the candidate list over the first rsteps equals the reference
    CPU search's, except entries within 1e-4 of a stage cutoff.
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
