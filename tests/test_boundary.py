"""The C-ABI library: it loads, exports what include/jerk.h declares, and its
host-side logic (geometry, statistics, candidate insertion) matches the
reference -- all without a GPU."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk
from tests import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    H.ensure_oracle()


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            if m.group(1) not in ("if", "while", "for", "return", "sizeof"):
                names.append(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = jerk.lib()
    names = declared_functions()
    assert "jerk_search" in names and "jerk_plan_create" in names
    for n in names:
        assert hasattr(L, n), n


def test_obs_geometry_matches_reference():
    for e in H.golden("sizing.json"):
        o = e["obs"]
        wgiven = e["wmax"] is not None
        obs, fftlen, mk = jerk.obs_from_params(e["numbins"], e["N"], e["dt"], e["zmax"],
                                               e["wmax"] or 0, e["numharm"], e["sigma"],
                                               wmax_given=wgiven)
        assert (fftlen, mk) == (o["fftlen"], o["maxkernlen"])
        for k in ("corr_uselen", "numz", "numw", "numharmstages", "highestbin"):
            assert getattr(obs, k) == o[k], k
        for k in ("rlo", "zlo", "wlo"):
            assert getattr(obs, k) == o[k], k
        assert list(obs.numindep)[: o["numharmstages"]] == o["numindep"]
        for got, want in zip(list(obs.powcut)[: o["numharmstages"]], o["powcut"]):
            # the reference's chi^2 inversion stops at a 1e-8 tolerance: allow one float ulp
            assert abs(got - want) <= np.spacing(np.float32(want)), (got, want)
        for i, sub in enumerate(e.get("subs", [])):
            got = jerk.subharm_sizes(obs, fftlen)[i]
            for k in ("numharm", "harmnum", "zmax", "wmax", "numz", "numw", "fftlen",
                      "halfwidth"):
                assert got[k] == sub[k], (e["zmax"], e["wmax"], i, k)


def test_sigma_matches_reference():
    g = H.golden("sigma.json")
    for power, numsum, numindep, want in g["candidate_sigma"]:
        got = jerk.candidate_sigma(power, numsum, numindep)
        if np.isnan(want):
            assert np.isnan(got)
        else:
            assert got == pytest.approx(want, rel=1e-9, abs=1e-9)
    for sig, numsum, numindep, want in g["power_for_sigma"]:
        assert jerk.power_for_sigma(sig, numsum, numindep) == pytest.approx(want, rel=2e-7)


def test_insertion_matches_oracle_on_random_hits():
    rng = np.random.default_rng(11)
    unsorted = 0
    for trial in range(20):
        n = int(rng.integers(1, 3000))
        hits = np.zeros(n, dtype=jerk.CAND_DTYPE)
        # clustered r values so the 15-bin rule is exercised, ties included
        hits["r"] = np.round(rng.uniform(0, 2000, n) * 4) / 4
        hits["numharm"] = 1 << rng.integers(0, 5, n)
        hits["power"] = rng.uniform(10, 60, n).astype(np.float32)
        numindep = [10 ** 7 >> s for s in range(6)]
        for i in range(n):
            st = int(np.log2(hits["numharm"][i]))
            hits["sigma"][i] = np.float32(
                ob.orc_candidate_sigma(float(hits["power"][i]), int(hits["numharm"][i]),
                                       numindep[st]))
        want = ob.insert_hits(hits, numindep)
        got = jerk.insert_hits(hits)
        assert len(got) == len(want)
        assert np.array_equal(got["r"], want["r"])
        assert np.array_equal(got["power"], want["power"])
        unsorted += int(np.any(np.diff(got["r"]) < 0))
    # the reference's list walk leaves the list unsorted in a corner case;
    # the random sequences must reach it for this test to mean anything
    assert unsorted > 0


def test_errors_are_returned_not_fatal():
    obs = jerk.Obs()
    obs.numharmstages = 3
    with pytest.raises(jerk.JerkError) as ei:
        jerk.JerkPlan(obs, [])
    assert ei.value.code == jerk.JERK_EINVAL
    with pytest.raises(jerk.JerkError):
        jerk.obs_from_params(1 << 10, 1 << 11, 1e-3, 20, 60, 3, 2.0)  # numharm not 2^k


def test_bad_tuning_knob_is_rejected_before_any_device_work():
    obs, fftlen, _ = jerk.obs_from_params(1 << 19, 1 << 20, 64e-6, 20, 60, 8, 2.0)
    subs = jerk.subharm_sizes(obs, fftlen)
    with pytest.raises(jerk.JerkError) as ei:
        jerk.JerkPlan(obs, subs, batch=8, harm_mode=7)
    assert ei.value.code == jerk.JERK_EINVAL
    assert "harm_mode" in str(ei.value)


def test_unsupported_fft_length_is_rejected_before_any_device_work():
    # zmax 1400, wmax 1500 needs fftlen 25600 (the longest supported is 15360)
    obs, fftlen, _ = jerk.obs_from_params(1 << 24, 1 << 25, 54.6e-6, 1400, 1500, 16, 3.0)
    assert fftlen == 25600
    subs = jerk.subharm_sizes(obs, fftlen)
    with pytest.raises(jerk.JerkError) as ei:
        jerk.JerkPlan(obs, subs, batch=4)
    assert ei.value.code == jerk.JERK_EUNSUPPORTED and "25600" in str(ei.value)


def test_input_entry_points_size_and_reject_before_any_device_work():
    """jerk_realfft / jerk_deredden: scratch sizes from the host alone, and
    unsupported lengths, null or misaligned pointers and short scratch come
    back as error codes before anything reaches the device."""
    L = jerk.lib()
    M = 1 << 24
    # the four-step scratch: M complex values plus two twiddle tables
    assert L.jerk_realfft_scratch_bytes(1 << 25) >= 8 * M
    for bad in (0, 3, 1 << 14, (1 << 25) + 2, 1 << 28, 7 << 20, (1 << 20) + 2):
        assert L.jerk_realfft_scratch_bytes(bad) == 0, bad
    # lengths with factors 3 and 5: M = n / 2 = R1 R2 over the block-FFT sizes
    for good in (3 << 20, 5 << 21, 15 << 20, 2 * 10240 * 10240):
        assert L.jerk_realfft_scratch_bytes(good) >= 4 * good, good
    assert L.jerk_deredden_scratch_bytes(7) == 0
    assert L.jerk_deredden_scratch_bytes(8) > 0
    assert L.jerk_deredden_scratch_bytes(1 << 24) >= 4 * ((1 << 24) // 100)
    assert L.jerk_spectrum_scratch_bytes(1 << 25) == max(
        L.jerk_realfft_scratch_bytes(1 << 25), L.jerk_deredden_scratch_bytes(1 << 24))
    big = L.jerk_realfft_scratch_bytes(1 << 20)
    assert L.jerk_realfft(4096, 7 << 20, 4096, 4096, big, None) == jerk.JERK_EUNSUPPORTED
    assert L.jerk_realfft(None, 1 << 20, 4096, 4096, big, None) == jerk.JERK_EINVAL
    assert L.jerk_realfft(4100, 1 << 20, 4096, 4096, big, None) == jerk.JERK_EINVAL  # misaligned
    assert L.jerk_realfft(4096, 1 << 20, 4096, 4096, big - 1, None) == jerk.JERK_EINVAL
    assert "scratch" in jerk.lib().jerk_last_error().decode()
    assert L.jerk_deredden(4096, 7, 4096, 1 << 20, None) == jerk.JERK_EINVAL
    assert L.jerk_deredden(4096, 1 << 20, 4096, 16, None) == jerk.JERK_EINVAL
    assert L.jerk_spectrum_from_timeseries(4096, 100, 4096, 4096, big, None) == jerk.JERK_EUNSUPPORTED


def _disp_offsets(numdms, nsub, worklen, dm0, ddm, dt=64e-6):
    f = 1200.0 + (np.arange(nsub) + 0.5) * 400.0 / nsub
    dms = dm0 + ddm * np.arange(numdms)
    delay = 4.148808e3 * dms[:, None] * (f[None, :] ** -2 - f[-1] ** -2)
    return np.minimum(np.rint(delay / dt), worklen).astype(np.int32)


def test_dedisp_tiling_choice_on_the_host():
    """jerk_dedisp_plan (no CUDA call): the widest tile, then the largest DM
    group, whose subband windows fit two CTAs per SM (100 KB); wide subband
    counts fall back to narrower tiles with up to 227 KB."""
    g, t, b = jerk.dedisp_plan(65536, 64, _disp_offsets(512, 64, 65536, 0.0, 0.5, 256e-6))
    assert (g, t) == (32, 256) and b <= 100 * 1024
    assert jerk.dedisp_plan(8192, 64, _disp_offsets(96, 64, 8192, 10.0, 0.5))[:2] == (16, 256)
    g, t, b = jerk.dedisp_plan(2048, 512, _disp_offsets(24, 512, 2048, 10.0, 0.5))
    assert (g, t) == (8, 64) and 100 * 1024 < b <= 227 * 1024
    # one window row per subband of the tile plus the DM spread: a wide spread
    # within a group shrinks the group
    wide = np.zeros((64, 8), dtype=np.int32)
    wide[1::2] = 3000
    assert jerk.dedisp_plan(4096, 8, wide)[0] == 1


def test_dedisp_plan_rejects_bad_offsets():
    for off in (np.array([[0, 1, 2, 101]]), np.array([[0, -1, 2, 3]])):
        with pytest.raises(jerk.JerkError) as ei:
            jerk.dedisp_plan(100, 4, off)
        assert ei.value.code == jerk.JERK_EINVAL
    with pytest.raises(jerk.JerkError):
        jerk.dedisp_plan(100, 4, np.zeros((2, 3)))
    with pytest.raises(jerk.JerkError) as ei:  # 4096 subband rows of 32 samples: too wide
        jerk.dedisp_plan(64, 4096, np.zeros((1, 4096)))
    assert ei.value.code == jerk.JERK_EUNSUPPORTED


def test_merge_hits_host_only_edges():
    """jerk_merge_hits needs no GPU: no hits give an empty list, a key past
    the last rstep or mismatched lengths are refused."""
    import numpy as np

    from prestozl_b200 import jerk

    obs, fftlen, _ = jerk.obs_from_params(1 << 19, 1 << 20, 64e-6, 20, 60, 8, 2.0)
    fund = jerk.subharm_sizes(obs, fftlen)[0]
    assert len(jerk.merge_hits(obs, fund, np.zeros(0, np.uint64), np.zeros(0, np.float32))) == 0
    per_rstep = obs.numharmstages * fund["numw"] * fund["numz"] * obs.corr_uselen
    with pytest.raises(jerk.JerkError):
        jerk.merge_hits(obs, fund, np.array([per_rstep * 10 ** 6], np.uint64),
                        np.array([50.0], np.float32))
    with pytest.raises(jerk.JerkError):
        jerk.merge_hits(obs, fund, np.array([1, 2], np.uint64), np.array([50.0], np.float32))
