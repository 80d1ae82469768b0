"""The served form: spectra of uneven length and uneven (zmax, wmax, numharm)
submitted together must each give exactly the candidate list they give when
searched alone (same kernels, same inputs -- bitwise equal), with banks
shared between requests of equal geometry and admission held to an HBM
budget."""

import numpy as np
import pytest

from prestozl_b200 import build, jerk, synth

pytestmark = pytest.mark.gpu

# (N, dt, zmax, wmax, numharm, sigma, seed)
MIX = [
    (1 << 20, 64e-6, 20, 60, 8, 2.0, 1),
    (1 << 19, 64e-6, 50, 160, 4, 2.5, 2),
    (1 << 20, 64e-6, 20, 60, 8, 2.0, 3),     # shares the first request's bank
    (1 << 18, 128e-6, 100, 0, 16, 3.0, 4),   # -wmax 0
    (1 << 20, 64e-6, 10, 40, 2, 2.0, 5),
]


def spectra():
    out = []
    for N, dt, z, w, nh, sig, seed in MIX:
        rng = np.random.default_rng(seed)
        ps = synth.random_pulsars(rng, 2, zmax=z * 0.8, wmax=max(w, 1) * 0.8, fmax=200.0)
        ts = synth.timeseries(N, dt, ps, seed)
        out.append(synth.presto_fft(ts))
    return out


def alone(spec, N, dt, z, w, nh, sig):
    obs, fftlen, _ = jerk.obs_from_params(len(spec), N, dt, z, w, nh, sig)
    subs = jerk.subharm_sizes(obs, fftlen)
    bank = jerk.DeviceBank(subs)
    plan = jerk.JerkPlan(obs, subs, batch=16, device_bank=bank.ptr.value)
    c = plan.search(spec)
    plan.close()
    bank.close()
    return c


def test_results_alone_equal_results_in_the_mix():
    build.build()
    specs = spectra()
    want = [alone(s, N, dt, z, w, nh, sig) for s, (N, dt, z, w, nh, sig, _) in zip(specs, MIX)]
    srv = jerk.JerkServer(max_active=3, batch=16)
    for i, (s, (N, dt, z, w, nh, sig, _)) in enumerate(zip(specs, MIX)):
        srv.submit(s, N, dt, z, w, nh, sig, tag=i)
    got = {}
    while len(got) < len(MIX):
        r = srv.poll(60000)
        assert r is not None, "server stalled"
        tag, cands, t = r
        assert t["submit"] <= t["start"] <= t["done"]
        got[tag] = cands
    st = srv.stats()
    srv.close()
    assert st["finished"] == len(MIX) and st["failed"] == 0
    for i in range(len(MIX)):
        assert np.array_equal(got[i], want[i]), i
    assert any(len(w) for w in want)


def test_admission_under_a_small_budget_still_finishes_everything():
    build.build()
    specs = spectra()[:3]
    # room for about one request at a time (each needs ~130 MB here)
    srv = jerk.JerkServer(hbm_budget_bytes=300 << 20, max_active=3, batch=4)
    for i, (s, (N, dt, z, w, nh, sig, _)) in enumerate(zip(specs, MIX)):
        srv.submit(s, N, dt, z, w, nh, sig, tag=i)
    tags = []
    while len(tags) < 3:
        r = srv.poll(60000)
        assert r is not None
        tags.append(r[0])
    st = srv.stats()
    srv.close()
    assert sorted(tags) == [0, 1, 2] and st["failed"] == 0
    assert 0 < st["peak_bytes"] <= st["budget"]


def test_requests_that_cannot_fit_or_wait_too_long_fail_alone():
    """Fault handling on the host: a request larger than the whole budget and
    requests left waiting past the queue deadline come back as errors while
    the loop keeps serving the others."""
    build.build()
    specs = spectra()
    # budget too small for any request: every one fails with ENOMEM
    srv = jerk.JerkServer(hbm_budget_bytes=16 << 20, max_active=2, batch=4)
    srv.submit(specs[0], *MIX[0][:6], tag=0)
    with pytest.raises(jerk.JerkError) as ei:
        srv.poll(60000)
    assert ei.value.code == jerk.JERK_ENOMEM
    srv.close()
    # one slot and a deadline of ~zero: the loop admits what fits before it
    # expires what still waits, so the first request takes the slot and the
    # one queued behind it times out; the first still finishes
    srv = jerk.JerkServer(max_active=1, batch=4, queue_timeout_s=1e-9)
    srv.submit(specs[0], *MIX[0][:6], tag=0)
    srv.submit(specs[2], *MIX[2][:6], tag=1)
    outcomes = {}
    for _ in range(2):
        try:
            tag, cands, _ = srv.poll(60000)
            outcomes[tag] = "ok"
        except jerk.JerkError as e:
            outcomes["err"] = e.code
    st = srv.stats()
    srv.close()
    assert outcomes.get(0) == "ok"
    assert outcomes.get("err") == jerk.JERK_TIMEOUT
    assert st["failed"] == 1


def test_poisson_stream_of_dedispersion_trials_peaks_at_the_pulsar_trial():
    """The served stream in miniature: trial spectra arrive at Poisson times
    (40 per second) while earlier ones are on the GPU; one pulsar's SNR peaks
    at trial 5 and falls off as a Gaussian in trial index (sigma 1.5 trials).
    Every trial is answered, latencies are reported, and the pulsar's best
    candidate sigma is highest at the peak trial."""
    import time

    torch = pytest.importorskip("torch")
    build.build()
    N, dt, ntrials, peak = 1 << 22, 64e-6, 10, 5
    psr = synth.Pulsar(f=87.3, z=30.0, w=60.0, snr=30.0, nharm=4)
    specs = []
    for t in range(ntrials):
        snr = psr.snr * float(np.exp(-0.5 * ((t - peak) / 1.5) ** 2))
        p = synth.Pulsar(psr.f, psr.z, psr.w, snr, psr.nharm)
        ts = synth.timeseries_torch(N, dt, [p] if snr > 1.0 else [], 700 + t, device="cuda")
        specs.append(synth.presto_fft_torch(ts).contiguous())
    torch.cuda.synchronize()
    rng = np.random.default_rng(7)
    gaps = rng.exponential(1.0 / 40.0, ntrials)
    srv = jerk.JerkServer(max_active=3, batch=32)
    t0 = time.perf_counter()
    for t in range(ntrials):
        time.sleep(float(gaps[t]))
        srv.submit(specs[t], N, dt, 100, 200, 8, 3.0, tag=t)
    best, lat = {}, []
    for _ in range(ntrials):
        tag, cands, tm = srv.poll(120000)
        lat.append(tm["done"] - tm["submit"])
        # the pulsar's candidates: within its drift (z/2 + w/12 bins) of f * T
        r0 = psr.f * N * dt
        near = cands[np.abs(cands["r"] - r0) < 30.0] if len(cands) else cands
        best[tag] = float(near["sigma"].max()) if len(near) else 0.0
    srv.close()
    wall = time.perf_counter() - t0
    print(f"{ntrials} trials in {wall:.2f} s; latency p50 {np.percentile(lat, 50):.2f} s "
          f"p99 {np.percentile(lat, 99):.2f} s; best sigma by trial "
          f"{[round(best[t], 1) for t in range(ntrials)]}")
    assert sorted(best) == list(range(ntrials))
    assert max(best, key=best.get) == peak
    assert best[peak] > best[0] and best[peak] > best[ntrials - 1]


def test_time_series_requests_equal_their_spectra():
    """Dedispersed trials go straight into the served loop: a request that
    carries the N float32 samples (from host memory or a CUDA tensor) gives
    exactly the candidates of the spectrum the same series makes on the GPU
    (jerk_spectrum_from_timeseries: realfft, deredden, bin 0 -- the
    reference's .dat preparation), in a mix with ordinary spectrum requests;
    the series buffers are reused between requests."""
    torch = pytest.importorskip("torch")
    build.build()
    N, dt = 1 << 20, 64e-6
    series = []
    for seed in (31, 32):
        rng = np.random.default_rng(seed)
        ps = synth.random_pulsars(rng, 2, zmax=16.0, wmax=48.0, fmax=200.0)
        ts = synth.timeseries(N, dt, ps, seed)
        ts = ts + (0.02 * np.cumsum(rng.standard_normal(N))).astype(np.float32)
        series.append(np.ascontiguousarray(ts, dtype=np.float32))
    prepared = []
    for ts in series:
        spec = jerk.spectrum_from_timeseries(torch.from_numpy(ts).cuda())
        torch.cuda.synchronize()
        prepared.append(spec)
    params = (N, dt, 20, 60, 8, 2.0)
    srv = jerk.JerkServer(max_active=3, batch=16)
    dev_series = torch.from_numpy(series[1]).cuda()
    srv.submit(series[0], *params, tag=0, timeseries=True)
    srv.submit(prepared[0], *params, tag=1)
    srv.submit(dev_series, *params, tag=2, timeseries=True)
    srv.submit(prepared[1], *params, tag=3)
    srv.submit(series[1], *params, tag=4, timeseries=True)  # reuses a pooled buffer
    got = {}
    while len(got) < 5:
        r = srv.poll(60000)
        assert r is not None, "server stalled"
        got[r[0]] = r[1]
    st = srv.stats()
    srv.close()
    assert st["failed"] == 0
    assert len(got[1]) > 0 and len(got[3]) > 0
    assert np.array_equal(got[0], got[1])
    assert np.array_equal(got[2], got[3]) and np.array_equal(got[4], got[3])
    with pytest.raises(jerk.JerkError):  # not a supported series length
        s2 = jerk.JerkServer(max_active=1)
        try:
            s2.submit(np.zeros(7 << 16, np.float32), 7 << 16, dt, 20, 60, 8, 2.0,
                      timeseries=True)
        finally:
            s2.close()


def test_time_series_request_with_birdies():
    """A time-series request carrying a birdie list: the server zaps the
    birdies after making the spectrum, as a -zaplist run does, and the
    candidates equal those of the spectrum prepared and zapped beforehand
    (jerk_spectrum_from_timeseries then jerk_zap_birdies)."""
    torch = pytest.importorskip("torch")
    build.build()
    N, dt = 1 << 20, 64e-6
    rng = np.random.default_rng(41)
    ps = synth.random_pulsars(rng, 2, zmax=16.0, wmax=48.0, fmax=200.0)
    ts = np.ascontiguousarray(synth.timeseries(N, dt, ps, 41), dtype=np.float32)
    # zap the strongest pulsar's fundamental region and an empty band
    r0 = ps[0].f * N * dt
    lob, hib = [r0 - 40.0, 120000.0], [r0 + 40.0, 120050.0]
    spec = jerk.spectrum_from_timeseries(torch.from_numpy(ts).cuda())
    jerk.zap_birdies(spec, N, lob, hib)
    torch.cuda.synchronize()
    params = (N, dt, 20, 60, 8, 2.0)
    srv = jerk.JerkServer(max_active=2, batch=16)
    srv.submit(ts, *params, tag=0, timeseries=True, birdies=(lob, hib))
    srv.submit(spec, *params, tag=1)
    srv.submit(ts, *params, tag=2, timeseries=True)  # no birdies
    got = {}
    while len(got) < 3:
        r = srv.poll(60000)
        assert r is not None, "server stalled"
        got[r[0]] = r[1]
    srv.close()
    assert np.array_equal(got[0], got[1])
    assert not np.array_equal(got[0], got[2])  # the zapping changed the result
