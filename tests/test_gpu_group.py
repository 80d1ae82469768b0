"""The batched form across plans: searches of spectra of uneven length and
geometry advanced together in waves of merged launches (jerk_search_group,
jerk_search_begin + jerk_group_advance).  A wave runs one prep launch, one
correlation launch per FFT length and one harmonic sum per stage count over
every plan's next batch; each plan's CTAs run as in its own launches, so each
plan's candidates and raw hits must equal, bit for bit, that plan searched
alone with jerk_search."""

import numpy as np
import pytest

from prestozl_b200 import build, jerk, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# (log2 N, dt, zmax, wmax, numharm, sigma, seed)
MIX = [
    (20, 64e-6, 20, 60, 8, 2.0, 0),      # the small spectrum
    (20, 64e-6, 20, 60, 8, 2.0, 11),     # same geometry, other data
    (19, 64e-6, 100, 0, 16, 2.5, 12),    # shorter, no -wmax volume, 5 stages
    (21, 54.6e-6, 50, 160, 8, 3.0, 13),  # longer, other geometry
    (20, 64e-6, 20, 60, 4, 2.0, 14),     # 3 stages
]


def _spectrum(logn, dt, seed):
    if seed == 0:
        spec, N, dt = synth.small_spectrum()
        return spec, N
    N = 1 << logn
    ps = synth.random_pulsars(np.random.default_rng(seed), 2, zmax=16.0, wmax=40.0, fmax=300.0)
    return synth.presto_fft(synth.timeseries(N, dt, ps, seed)), N


class Mix:
    def __init__(self, entries, stream, batch=8, harm_modes=None):
        self.banks, self.plans, self.specs = {}, [], []
        for i, (logn, dt, zmax, wmax, nh, sig, seed) in enumerate(entries):
            spec, N = _spectrum(logn, dt, seed)
            obs, fftlen, _ = jerk.obs_from_params(len(spec), N, dt, zmax, wmax, nh, sig)
            subs = jerk.subharm_sizes(obs, fftlen)
            key = (zmax, wmax, nh, fftlen, obs.corr_uselen)
            if key not in self.banks:
                self.banks[key] = jerk.DeviceBank(subs)
            hm = harm_modes[i] if harm_modes else 0
            self.plans.append(jerk.JerkPlan(obs, subs, batch=batch, stream=stream,
                                            device_bank=self.banks[key].ptr.value, harm_mode=hm))
            self.specs.append(torch.from_numpy(spec.view(np.float32).copy()).cuda())

    def close(self):
        for p in self.plans:
            p.close()
        for b in self.banks.values():
            b.close()


def _same(a, b):
    assert len(a) == len(b)
    for f in a.dtype.names:
        assert np.array_equal(a[f], b[f]), f


@pytest.fixture(scope="module")
def stream():
    build.build()
    s = torch.cuda.Stream()
    return s.cuda_stream


def test_group_search_equals_each_search_alone(stream):
    mix = Mix(MIX, stream)
    alone = [p.search(s) for p, s in zip(mix.plans, mix.specs)]
    got = jerk.search_group(mix.plans, mix.specs)
    torch.cuda.synchronize()
    for a, g in zip(alone, got):
        _same(g, a)
    assert all(len(a) > 0 for a in alone)
    mix.close()


def test_incremental_waves_equal_searches_alone(stream):
    """Passes started with begin(), advanced a few waves ahead at a time
    (ahead = 2) until every batch is enqueued, collected with their raw hits;
    one plan uses the harmonic sum's prefetch form (its sum runs in its own
    launch inside each wave)."""
    mix = Mix(MIX, stream, batch=5, harm_modes=[0, 2, 0, 0, 0])
    alone = [p.search(s, want_hits=True) for p, s in zip(mix.plans, mix.specs)]
    for p, s in zip(mix.plans, mix.specs):
        p.begin(s)
    rounds = 0
    while jerk.group_advance(mix.plans, ahead=2):
        rounds += 1
    assert rounds > 0
    got = [p.collect(want_hits=True) for p in mix.plans]
    torch.cuda.synchronize()
    for (ca, ka, pa), (cg, kg, pg) in zip(alone, got):
        _same(cg, ca)
        assert np.array_equal(kg, ka) and np.array_equal(pg, pa)
    mix.close()


def test_more_plans_than_one_wave_holds(stream):
    """14 searches: waves of at most 12 plans, the rest in a second wave."""
    entries = [(18, 64e-6, 20, 60, 8, 2.0, 100 + i) for i in range(14)]
    mix = Mix(entries, stream, batch=4)
    alone = [p.search(s) for p, s in zip(mix.plans, mix.specs)]
    got = jerk.search_group(mix.plans, mix.specs)
    torch.cuda.synchronize()
    for a, g in zip(alone, got):
        _same(g, a)
    mix.close()


def test_plans_on_different_streams_are_refused(stream):
    mix = Mix(MIX[:1], stream)
    other = Mix(MIX[1:2], torch.cuda.Stream().cuda_stream)
    with pytest.raises(jerk.JerkError):
        jerk.search_group(mix.plans + other.plans, mix.specs + other.specs)
    # both plans stay usable
    assert len(mix.plans[0].search(mix.specs[0])) > 0
    assert len(other.plans[0].search(other.specs[0])) > 0
    mix.close()
    other.close()
