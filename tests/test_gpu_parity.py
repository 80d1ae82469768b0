"""CUDA path vs the oracle and the reference's golden results, through the
C ABI (libjerk.so).  Small spectrum: 2^20 samples with one binary pulsar,
-zmax 20 -wmax 60 -numharm 8 -sigma 2.0 (546 rsteps).

Tolerances (FP32 CUDA correlation against the oracle's FP64 one):
  * ffdot powers: |gpu - oracle| <= 1e-5 * max(oracle, 1)  (normalised power)
  * summed powers of hits and candidates: 1e-5 relative; sigma 1e-5 relative
  * integer/index work (rlo, rinds, hit keys): exact, except hits whose power
    lies within 1e-4 relative of their stage's cutoff
"""

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk
from tests import helpers as H

pytestmark = pytest.mark.gpu

POW_TOL = 1e-5


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    return H.small_problem(str(tmp_path_factory.mktemp("gpu_small")))


@pytest.fixture(scope="module")
def plan(small):
    p = jerk.JerkPlan(jerk.obs_from_refobs(small.obs), small.subs, batch=8)
    yield p
    p.close()


def test_plan_geometry(small, plan):
    assert plan.num_rsteps == H.golden("small_cands.json")["nrsteps"]


@pytest.mark.parametrize("which", ["first", "pulsar", "late", "last"])
def test_volumes_match_oracle(small, plan, which):
    k = {"first": 0, "pulsar": small.rstep_of(8281.0), "late": 540,
         "last": plan.num_rsteps - 1}[which]
    startr = small.startr(k)
    lastr = startr + small.rstep - 0.5
    worst = 0.0
    for i in range(len(small.subs)):
        got, rlo = plan.volume(small.spec, k, i)
        h, want, _, _ = small.oracle.fderivs(i, startr, lastr)
        assert rlo == h["rlo"]
        assert got.shape == want.shape
        err = np.abs(got.astype(np.float64) - want) / np.maximum(want, 1.0)
        worst = max(worst, float(err.max()))
        assert err.max() <= POW_TOL, (which, i, err.max())
    print(f"max FP32 power error vs FP64 oracle ({which}): {worst:.3e}")


def _oracle_hits(small, first, count):
    _, _, keys, pows = small.oracle.search_hits(first, count)
    return keys, pows


def _compare_hits(small, gk, gp, ok, op):
    powcut = np.array(list(small.obs.powcut))
    S = small.obs.numharmstages
    per = small.obs.corr_uselen * small.subs[0]["numz"] * small.subs[0]["numw"]
    stage_of = lambda k: ((k // per) % S).astype(int)
    gd = dict(zip(gk.tolist(), gp.tolist()))
    od = dict(zip(ok.tolist(), op.tolist()))
    near = lambda k, p: abs(p - powcut[stage_of(np.uint64(k))]) <= 1e-4 * powcut[stage_of(np.uint64(k))]
    missing = [k for k in od if k not in gd and not near(k, od[k])]
    extra = [k for k in gd if k not in od and not near(k, gd[k])]
    assert not missing and not extra, (len(missing), len(extra))
    common = [k for k in od if k in gd]
    rel = max((abs(gd[k] - od[k]) / od[k] for k in common), default=0.0)
    assert rel <= POW_TOL, rel
    # insertion order (sorted keys) equals the oracle's order
    assert np.all(np.diff(gk.astype(np.uint64)) > 0)
    return len(common), rel


def test_hits_match_oracle(small, plan):
    first, count = 0, 48
    cands, gk, gp = plan.search(small.spec, first, count, want_hits=True)
    ok, op = _oracle_hits(small, first, count)
    n, rel = _compare_hits(small, gk, gp, ok, op)
    assert n > 1000
    print(f"{n} hits, max summed-power rel error {rel:.3e}")


def test_hits_around_pulsar_match_oracle(small, plan):
    first = max(0, small.rstep_of(8281.0) - 4)
    cands, gk, gp = plan.search(small.spec, first, 9, want_hits=True)
    ok, op = _oracle_hits(small, first, 9)
    _compare_hits(small, gk, gp, ok, op)


def test_full_search_matches_reference_golden(small, plan):
    g = H.golden("small_cands.json")
    want = np.array([tuple(c) for c in g["cands"]], dtype=jerk.CAND_DTYPE)
    got = plan.search(small.spec)
    probs = H.compare_cands(got, want, g["obs"]["powcut"])
    assert not probs, probs[:10]


def test_batch_size_does_not_change_results(small):
    """The tuning knobs (rsteps per batch; the harmonic sum's kernel -- plain
    gathers, gathers with TMA prefetch into L2, TMA tiles of 8 or 16 z rows)
    change only speed: hits, powers and candidates are bitwise the same."""
    obs = jerk.obs_from_refobs(small.obs)
    res = []
    for b, mode in ((1, 1), (5, 2), (8, 1), (8, 4), (16, 3), (3, 2), (8, 0)):
        p = jerk.JerkPlan(obs, small.subs, batch=b, harm_mode=mode)
        c, k, pw = p.search(small.spec, 100, 23, want_hits=True)
        res.append((c, k, pw))
        p.close()
    for c, k, pw in res[1:]:
        assert np.array_equal(k, res[0][1]) and np.array_equal(pw, res[0][2])
        assert np.array_equal(c, res[0][0])


def test_device_resident_spectrum(small, plan):
    torch = pytest.importorskip("torch")
    d = torch.from_numpy(small.spec.view(np.float32).copy()).cuda()
    c1 = plan.search(small.spec, 200, 16)
    c2 = plan.search(d, 200, 16)
    torch.cuda.synchronize()
    assert np.array_equal(c1, c2)


def test_hit_buffer_overflow_is_recovered(small):
    p = jerk.JerkPlan(jerk.obs_from_refobs(small.obs), small.subs, batch=8, max_hits=64)
    c, k, pw = p.search(small.spec, 0, 30, want_hits=True)
    p.close()
    q = jerk.JerkPlan(jerk.obs_from_refobs(small.obs), small.subs, batch=8)
    c2, k2, pw2 = q.search(small.spec, 0, 30, want_hits=True)
    q.close()
    assert len(k) > 64
    assert np.array_equal(k, k2) and np.array_equal(c, c2)


def test_graph_mode_replays_match_batch_by_batch(small):
    """A pass captured into a CUDA graph and replayed gives, for every
    spectrum, exactly the hits and candidates of the batch-by-batch path;
    the graph is reused across spectra (host or device) and re-captured for
    a new rstep range."""
    torch = pytest.importorskip("torch")
    obs = jerk.obs_from_refobs(small.obs)
    # another spectrum with other hits (a scaled copy would normalise to the same data)
    other = np.ascontiguousarray(np.roll(small.spec, 4099))
    plain = jerk.JerkPlan(obs, small.subs, batch=8)
    graph = jerk.JerkPlan(obs, small.subs, batch=8, use_graph=True)
    dev = torch.from_numpy(other.view(np.float32).copy()).cuda()
    keys = []
    for spec, first, count in ((small.spec, 100, 40), (other, 100, 40), (dev, 100, 40),
                               (small.spec, 0, 24), (small.spec, 100, 40)):
        want = plain.search(spec, first, count, want_hits=True)
        got = graph.search(spec, first, count, want_hits=True)
        torch.cuda.synchronize()
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
        keys.append(got[1])
    assert not np.array_equal(keys[0], keys[1])  # the replays did see new data
    plain.close()
    graph.close()


def test_local_power_normalisation_matches_reference(tmp_path):
    """-locpow (src/accel_utils.c:1186-1203): volumes against the FP64 oracle
    (same normalisation restated) and the whole small search against the
    reference CPU search run with -locpow."""
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    from prestozl_b200 import synth

    spec, N, dt = synth.small_spectrum()
    args = list(H.golden("small_cands.json")["args"]) + ["-locpow"]
    prob = H.Problem(str(tmp_path), spec, N, dt, args)
    assert prob.obs.norm_type == 1
    obs = jerk.obs_from_refobs(prob.obs)
    assert obs.norm_type == 1
    p = jerk.JerkPlan(obs, prob.subs, batch=8)
    worst = 0.0
    for k in (0, prob.rstep_of(8281.0), p.num_rsteps - 1):
        startr = prob.startr(k)
        for i in range(len(prob.subs)):
            got, rlo = p.volume(prob.spec, k, i)
            h, want, _, _ = prob.oracle.fderivs(i, startr, startr + prob.rstep - 0.5)
            err = float((np.abs(got.astype(np.float64) - want) / np.maximum(want, 1.0)).max())
            worst = max(worst, err)
            assert err <= POW_TOL, (k, i, err)
    got = p.search(prob.spec)
    p.close()
    prob.ref.make_bank()
    want, done = prob.ref.search()
    probs = H.compare_cands(got, want, list(prob.obs.powcut))
    assert not probs, probs[:10]
    assert len(want) > 0
    print(f"-locpow: max FP32 power error vs FP64 oracle {worst:.3e}, {len(want)} candidates")


# numharm: rsteps compared (0 = the whole search).  At 16 and 32 harmonics the
# reference's single-threaded search of the whole spectrum takes about a
# minute, so the first 48 rsteps (the pulsar sits in rstep 7) are compared.
FEW_MANY_HARMONICS = {1: 0, 2: 0, 4: 0, 16: 48, 32: 48}


@pytest.mark.parametrize("numharm", list(FEW_MANY_HARMONICS))
def test_harmonic_counts_match_reference(numharm, tmp_path):
    """-numharm 1, 2, 4, 16 and 32 on the small spectrum (the golden run is
    at 8): the candidate list equals the reference CPU search's, except
    entries within 1e-4 of a stage cutoff; powers and sigmas to 1e-5.  At 32
    harmonics the harmonic sum runs six stages and 31 subharmonics.

    The reference runs on one thread: its OpenMP search calls candidate_sigma
    (dcdflib's cdfchi, which keeps static state) from several threads at once
    (src/accel_utils.c:1518-1535), and at 32 harmonics with several threads
    it aborts with "Error in cdfchi()".  The reference's own GPU path returns
    no candidates at -numharm 1: its search sits inside numharmstages > 1."""
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    from prestozl_b200 import synth

    spec, N, dt = synth.small_spectrum()
    args = list(H.golden("small_cands.json")["args"])
    args[args.index("-numharm") + 1] = str(numharm)
    prob = H.Problem(str(tmp_path), spec, N, dt, args)
    assert prob.obs.numharmstages == numharm.bit_length()
    steps = FEW_MANY_HARMONICS[numharm]
    p = jerk.JerkPlan(jerk.obs_from_refobs(prob.obs), prob.subs, batch=16)
    got = p.search(prob.spec, 0, steps) if steps else p.search(prob.spec)
    p.close()
    prob.ref.make_bank()
    ob.set_threads(1)
    want, done = prob.ref.search(max_steps=steps)
    if steps:
        assert done == steps
    assert len(want) > 0
    probs = H.compare_cands(got, want, list(prob.obs.powcut))
    assert not probs, probs[:10]
    print(f"-numharm {numharm}: {len(got)} candidates (reference {len(want)})")


def test_photon_normalisation_matches_reference(tmp_path):
    """-photon (powers over the photon count, the DC bin of the .fft,
    src/accel_utils.c:1798-1808): Poisson counts of mean 4 whose rate
    carries the small spectrum's pulsar; volumes against the FP64 oracle and
    the whole search against the reference CPU search run with -photon.

    The DC bin of photon counts (normalised power about 4e6 here) lies inside
    rstep 0, whose volumes then carry FP32 rounding in proportion to that
    peak, as the reference's FP32 FFTs do: there the bound is
    1e-5 max(oracle, 1) + 1e-6 (the volume's peak); elsewhere the usual
    per-cell 1e-5."""
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    from prestozl_b200 import synth

    N, dt, seed = 1 << 20, 64e-6, 99
    pulsar = synth.timeseries(N, dt, synth.small_pulsar(), seed) - synth.timeseries(N, dt, [],
                                                                                    seed)
    rate = np.maximum(4.0 + 2.0 * pulsar.astype(np.float64), 0.0)
    counts = np.random.default_rng(seed).poisson(rate).astype(np.float32)
    spec = synth.presto_fft(counts)
    args = list(H.golden("small_cands.json")["args"]) + ["-photon"]
    prob = H.Problem(str(tmp_path), spec, N, dt, args)
    assert prob.obs.nph > 0
    obs = jerk.obs_from_refobs(prob.obs)
    assert obs.nph == prob.obs.nph
    p = jerk.JerkPlan(obs, prob.subs, batch=8)
    worst = 0.0
    for k in (0, prob.rstep_of(8281.0), p.num_rsteps - 1):
        startr = prob.startr(k)
        for i in range(len(prob.subs)):
            got, rlo = p.volume(prob.spec, k, i)
            h, want, _, _ = prob.oracle.fderivs(i, startr, startr + prob.rstep - 0.5)
            diff = np.abs(got.astype(np.float64) - want)
            floor = 1e-6 * float(want.max()) if k == 0 else 0.0
            bound = POW_TOL * np.maximum(want, 1.0) + floor
            assert np.all(diff <= bound), (k, i, float((diff / bound).max()))
            if k:
                worst = max(worst, float((diff / np.maximum(want, 1.0)).max()))
    got = p.search(prob.spec)
    p.close()
    prob.ref.make_bank()
    want, _ = prob.ref.search()
    probs = H.compare_cands(got, want, list(prob.obs.powcut))
    assert not probs, probs[:10]
    assert len(want) > 0
    print(f"-photon: nph {prob.obs.nph:.0f}, max FP32 power error vs FP64 oracle past rstep 0 "
          f"{worst:.3e}, {len(want)} candidates")


def test_frequency_band_matches_reference(tmp_path):
    """-flo 10 -fhi 400 on the small spectrum: the band limits set the first
    and last rsteps and the number of independent trials (and so the power
    cutoffs, src/accel_utils.c:1906-1984); the candidate list equals the
    reference CPU search's with the same flags."""
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides the kernel bank")
    from prestozl_b200 import synth

    spec, N, dt = synth.small_spectrum()
    args = list(H.golden("small_cands.json")["args"]) + ["-flo", "10", "-fhi", "400"]
    prob = H.Problem(str(tmp_path), spec, N, dt, args)
    obs = jerk.obs_from_refobs(prob.obs)
    assert prob.obs.rlo > 600 and prob.obs.highestbin < 30000
    p = jerk.JerkPlan(obs, prob.subs, batch=8)
    got = p.search(prob.spec)
    p.close()
    prob.ref.make_bank()
    want, _ = prob.ref.search()
    assert len(want) > 0
    probs = H.compare_cands(got, want, list(prob.obs.powcut))
    assert not probs, probs[:10]
    assert got["r"].min() >= prob.obs.rlo and got["r"].max() <= prob.obs.highestbin


def test_bounded_wait_gives_up_without_fault(small, plan):
    """Every device wait here is bounded.  A pass that runs the correlation's
    bounded wait on an mbarrier nothing completes (a one-thread probe kernel on
    the plan's stream, with no copy in flight) fails with JERK_ECUDA and the
    wait's message instead of hanging;
    the context and the same plan stay usable, and the next pass gives the
    results of a pass that never failed."""
    want = plan.search(small.spec, 100, 8, want_hits=True)
    plan.set_wait_probe(True)
    try:
        with pytest.raises(jerk.JerkError) as ei:
            plan.search(small.spec, 100, 8)
        assert ei.value.code == jerk.JERK_ECUDA
        assert "timed out" in str(ei.value)
    finally:
        plan.set_wait_probe(False)
    got = plan.search(small.spec, 100, 8, want_hits=True)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
