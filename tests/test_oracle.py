"""The oracle pinned against the reference itself (CPU only).

The reference's CPU accelsearch is compiled from its sources into
oracle/_ref (oracle/Makefile).  Where it is present these tests compare the
oracle's restatement with it directly; the golden fixtures (made by
tests/golden/make_golden.py from the same build) pin it everywhere.
"""

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import synth
from tests import helpers as H


@pytest.fixture(scope="module", autouse=True)
def _build():
    H.ensure_oracle()


def test_sizing_matches_reference_golden():
    L = ob.orclib()
    for e in H.golden("sizing.json"):
        o = e["obs"]
        zmax = int(-o["zlo"])
        wmax = int(-o["wlo"])
        out = (ob.C.c_int * 3)()
        L.orc_obs_sizes(zmax, wmax, out)
        assert (out[0], out[1], out[2]) == (o["maxkernlen"], o["fftlen"], o["corr_uselen"]), e
        for i, sub in enumerate(e.get("subs", [])):
            so = (ob.C.c_int * 6)()
            L.orc_sub_sizes(sub["numharm"], sub["harmnum"], zmax, wmax, o["corr_uselen"],
                            o["fftlen"], so)
            got = dict(zip(["zmax", "wmax", "numz", "numw", "fftlen", "halfwidth"], list(so)))
            for k, v in got.items():
                assert v == sub[k], (e["zmax"], e["wmax"], e["numharm"], i, k, v, sub[k])


def test_sigma_matches_reference_golden():
    g = H.golden("sigma.json")
    for power, numsum, numindep, want in g["candidate_sigma"]:
        got = ob.orc_candidate_sigma(power, numsum, numindep)
        if np.isnan(want):
            assert np.isnan(got), (power, numsum, numindep)
            continue
        assert got == pytest.approx(want, rel=1e-9, abs=1e-9), (power, numsum, numindep)
    for sig, numsum, numindep, want in g["power_for_sigma"]:
        got = ob.orc_power_for_sigma(sig, numsum, numindep)
        # the reference inverts the chi^2 CDF to a 1e-8 search tolerance
        assert got == pytest.approx(want, rel=2e-7), (sig, numsum, numindep)


def test_median_rank_matches_reference():
    if not H.have_ref():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 96, 192, 640, 1024, 1025):
        a = (rng.standard_normal(n) ** 2).astype(np.float32)
        scratch = a.copy()  # the reference reorders its input in place
        want = ob.reflib().ref_median(scratch.ctypes.data, n)
        assert np.sort(a)[(n - 1) // 2] == want


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    if not H.have_ref():
        pytest.skip("reference build not present")
    return H.small_problem(str(tmp_path_factory.mktemp("small")))


def test_small_spectrum_is_the_golden_one(small):
    g = H.golden("small_cands.json")
    assert H.golden("small_cands.json")["spectrum_sha256"] == \
        __import__("hashlib").sha256(small.spec.tobytes()).hexdigest()
    assert small.obs.corr_uselen == g["obs"]["corr_uselen"]


def test_oracle_volumes_match_reference(small):
    # the pulsar's rstep, the first rstep and one near the top of the spectrum
    for k in (small.rstep_of(8281.0), 0, 540):
        startr = small.startr(k)
        lastr = startr + small.rstep - 0.5
        for i, (st, h) in enumerate(small.ref.subharmonics()):
            hr, pr, ri, zi = small.ref.fderivs(1 << st, h, startr, lastr)
            ho, po, ri2, zi2 = small.oracle.fderivs(i, startr, lastr)
            assert hr == ho
            if st > 0:
                assert np.array_equal(ri, ri2) and np.array_equal(zi, zi2)
            # the reference correlates in float FFTW, the oracle in double
            err = np.abs(pr - po)
            assert np.all(err <= 2e-6 * np.maximum(po, 1.0)), (k, st, h, err.max())


def test_oracle_candidates_match_reference_prefix(small):
    cr, _ = small.ref.search(max_steps=80)
    co, _, _ = small.oracle.search(0, 80)
    assert not H.compare_cands(co, cr, list(small.obs.powcut))


def test_oracle_full_search_matches_golden(small):
    g = H.golden("small_cands.json")
    want = np.array([tuple(c) for c in g["cands"]], dtype=ob.CAND_DTYPE)
    co, steps, _ = small.oracle.search()
    assert steps == g["nrsteps"]
    assert not H.compare_cands(co, want, g["obs"]["powcut"])


def test_oracle_insert_replays_search(small):
    # replaying the recorded hits through the insertion gives the same list
    co, _, keys, pows = small.oracle.search_hits(0, 40)
    assert len(keys) > 0
    o = small.obs
    nz, nw = small.subs[0]["numz"], small.subs[0]["numw"]
    k = keys.astype(np.uint64)
    kk = k % o.corr_uselen; k //= o.corr_uselen
    jj = k % nz; k //= nz
    ii = k % nw; k //= nw
    st = k % o.numharmstages; rs = k // o.numharmstages
    nh = (1 << st.astype(np.int64))
    rlo = np.floor(np.rint(2 * (o.rlo + rs * small.rstep)) * 0.5)
    hits = np.zeros(len(keys), dtype=ob.CAND_DTYPE)
    hits["power"] = pows
    hits["numharm"] = nh
    hits["r"] = (rlo + kk * 0.5) / nh
    hits["z"] = (o.zlo + jj * 2.0) / nh
    hits["w"] = (o.wlo + ii * 20.0) / nh
    again = ob.insert_hits(hits, list(o.numindep))
    assert len(again) == len(co)
    assert np.array_equal(again["r"], co["r"]) and np.array_equal(again["power"], co["power"])


def test_insertion_walk_matches_reference_on_crafted_sequences(small):
    """Random hit orders, including the ones that leave the reference's list
    unsorted, give the same final list in the oracle as in the reference."""
    rng = np.random.default_rng(5)
    o = small.obs
    unsorted = 0
    for trial in range(15):
        n = int(rng.integers(1, 2500))
        nh = (1 << rng.integers(0, o.numharmstages, n)).astype(np.int32)
        st = np.log2(nh).astype(int)
        pc = np.array(list(o.powcut))[st]
        pows = (pc + rng.uniform(0.01, 40.0, n)).astype(np.float32)
        rlo = rng.integers(0, 4000, n).astype(np.int64)
        want = small.ref.insert_sequence(pows, rlo, nh)
        hits = np.zeros(n, dtype=ob.CAND_DTYPE)
        hits["power"], hits["numharm"] = pows, nh
        hits["r"] = rlo / nh.astype(np.float64)
        hits["z"], hits["w"] = 0.0, 0.0
        got = ob.insert_hits(hits, list(o.numindep))
        assert len(got) == len(want)
        assert np.array_equal(got["r"], want["r"])
        assert np.array_equal(got["power"], want["power"])
        assert np.array_equal(got["sigma"], want["sigma"])
        unsorted += int(np.any(np.diff(want["r"]) < 0))
    assert unsorted > 0


def test_local_power_normalisation_matches_reference():
    """-locpow: the oracle's direct double-top-hat local power equals the
    reference's FFT correlation (src/corr_routines.c:309-366) to 1e-6, for
    every chunk length the FFT lengths give, and its fast inverse square root
    (src/misc_utils.c:293-304) is bit-exact."""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    ob.quiet_wisdom()
    rng = np.random.default_rng(11)
    for n in (64, 96, 192, 256, 384, 512, 640, 1024, 2048, 2560, 3840):
        p = rng.exponential(1.0, n).astype(np.float32)
        want = ob.ref_local_powers(p)
        got = ob.local_powers(p)
        assert np.max(np.abs(got / want - 1.0)) < 1e-6, n
    for x in rng.exponential(2.0, 1000).astype(np.float32):
        assert ob.invsqrtf(float(x)) == ob.invsqrtf(float(x), reference=True)


def test_reference_options_do_not_leak_between_opens(tmp_path):
    """The reference's option parser keeps its options in one static struct;
    the driver restores the defaults before each parse, so a -locpow search
    opened earlier in the process does not turn the next search's
    normalisation into local power."""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    spec, N, dt = synth.small_spectrum()
    root = str(tmp_path / "s")
    synth.write_fft(root, spec, N, dt)
    args = ["-zmax", "20", "-wmax", "60", "-numharm", "8", "-sigma", "2.0"]
    a = ob.RefSearch(root + ".fft", args + ["-locpow"])
    b = ob.RefSearch(root + ".fft", args)
    assert a.obs.norm_type == 1 and b.obs.norm_type == 0
    a.close()
    b.close()


def _reddish_spectrum(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    amp = 10.0 / np.sqrt(np.arange(n) + 1.0) + 1.0
    return (rng.standard_normal(n) * amp + 1j * rng.standard_normal(n) * amp).astype(np.complex64)


def test_deredden_restatement_matches_reference():
    """The oracle's red-noise removal is bit-exact with the reference's
    deredden (src/accel_utils.c:1557-1633) from the smallest spectrum it
    accepts to 2^20 bins."""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    for n in (8, 9, 13, 14, 100, 1000, 4097, 12345, 1 << 16, 1 << 20):
        s = _reddish_spectrum(n, n)
        a, b = ob.deredden(s), ob.deredden(s, reference=True)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), n
        assert a[0] == 1.0


def test_reference_realfft_packing_and_precision():
    """The reference's realfft (as built here) equals the FP64 packed
    transform to FP32 rounding: every bin k within 2e-6 of |X[k]| + |X[M-k]|
    (both come from one pair of complex FFT outputs) plus 1e-5 of the
    spectrum's rms magnitude, and the rms error below 2e-7 of it.  (A packing, sign or scale
    slip would be of order 1.)"""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    ob.quiet_wisdom()
    for logn in (15, 18):
        n = 1 << logn
        rng = np.random.default_rng(logn)
        x = (rng.standard_normal(n) + 0.02 * np.cumsum(rng.standard_normal(n))).astype(np.float32)
        want = ob.packed_rfft(x)
        got = ob.ref_realfft(x).astype(np.complex128)
        rms = np.sqrt(np.mean(np.abs(want) ** 2))
        err = np.abs(got - want)
        assert np.all(err <= 2e-6 * ob.pair_magnitude(want) + 1e-5 * rms), logn
        assert np.sqrt(np.mean(err ** 2)) <= 2e-7 * rms, logn


def test_dat_input_is_realfft_then_deredden_then_bin0(tmp_path):
    """For a .dat input the reference searches realfft -> deredden with bin 0
    then set to (1, 1) (src/accel_utils.c:1696-1753, 1829-1834), nothing
    more: its in-memory spectrum equals those steps applied to the series,
    bitwise, and the oracle's deredden gives the same bits."""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    ob.quiet_wisdom()
    N, dt = 1 << 16, 64e-6
    rng = np.random.default_rng(16)
    ts = (rng.standard_normal(N) + 0.02 * np.cumsum(rng.standard_normal(N))).astype(np.float32)
    root = str(tmp_path / "series")
    ts.tofile(root + ".dat")
    synth.write_inf(root, N, dt)
    ref = ob.RefSearch(root + ".dat", ["-zmax", "20", "-wmax", "60", "-numharm", "4"])
    got = ref.spectrum()
    ref.close()
    raw = ob.ref_realfft(ts)
    for reference in (True, False):
        want = ob.deredden(raw, reference=reference)
        want[0] = 1.0 + 1.0j
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), reference


def test_zapbirds_restatement_matches_reference():
    """The oracle's zapbirds (src/zapping.c:29-81, from memory) is bit-exact
    with the reference build's: random spectra and birdies, including
    birdies below the 301-bin threshold and median windows reaching past the
    spectrum's end (zero padding, as the reference's .dat buffer has)."""
    if not ob.have_reference():
        pytest.skip("reference build absent")
    rng = np.random.default_rng(1)
    for t in range(200):
        n = int(rng.integers(2000, 100000))
        spec = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) *
                rng.uniform(0.5, 30)).astype(np.complex64)
        lo = float(rng.uniform(250, n - 2)) if t % 5 else float(rng.uniform(0, 400))
        hi = min(lo + float(rng.uniform(0, 50)), n - 1)
        a, b = ob.zapbirds(spec, lo, hi), ob.zapbirds(spec, lo, hi, reference=True)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (n, lo, hi)


@pytest.mark.parametrize("worklen,nsub,numdms", [(1000, 32, 20), (257, 13, 7), (64, 1, 3)])
def test_dedisp_oracle_equals_reference_float_dedisp(worklen, nsub, numdms):
    """The oracle's subband dedispersion against the reference's own
    float_dedisp (src/dispersion.c:208-231), called once per DM as
    prepsubband does, bitwise; offsets anywhere in [0, worklen]."""
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) is the comparator")
    rng = np.random.default_rng(worklen + nsub)
    cur = (rng.standard_normal((worklen, nsub)) * 30 + 100).astype(np.float32)
    last = (rng.standard_normal((worklen, nsub)) * 30 + 100).astype(np.float32)
    off = rng.integers(0, worklen + 1, (numdms, nsub)).astype(np.int32)
    off[0] = 0
    off[-1, 0] = worklen
    a = ob.dedisp_subbands(cur, last, off)
    b = ob.dedisp_subbands(cur, last, off, reference=True)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_downsample_oracle_is_the_block_mean():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((600, 5)).astype(np.float32)
    got = ob.downsample_subbands(x, 3)
    want = np.empty((200, 5), dtype=np.float32)
    for t in range(200):
        acc = np.zeros(5, dtype=np.float32)
        for k in range(3):
            acc = (acc + x[3 * t + k]).astype(np.float32)
        want[t] = acc / np.float32(3)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_dedisp_oracle_matches_golden_from_the_reference():
    """The committed fixture (tests/golden/dedisp_small.npz, the reference's
    float_dedisp per DM, made by tests/golden/make_golden.py) pins the
    oracle's dedispersion without the reference build."""
    import os

    g = np.load(os.path.join(H.GOLDEN, "dedisp_small.npz"))
    got = ob.dedisp_subbands(g["cur"], g["last"], g["offsets"])
    assert np.array_equal(got.view(np.uint32), g["out"].view(np.uint32))
