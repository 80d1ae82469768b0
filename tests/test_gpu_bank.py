"""GPU kernel-bank generation (jerk_bank_generate) against the reference's own
bank (create_subharminfos in oracle/_ref) and the golden kernel rows.

Tolerance: per kernel row, max |gpu - ref| <= 1e-5 * max |ref|.  The reference
builds each response from a float cosine series with a float real FFT and
then a float complex FFT; the GPU evaluates the same response bins as a
double-precision DFT and uses its own FP32 FFT, so rows differ by float
rounding (a few 1e-7 relative).
"""

import os

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu

ROW_TOL = 1e-5


def _rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("reference build missing")
    return H.small_problem(str(tmp_path_factory.mktemp("bank_small")))


def test_small_bank_matches_golden_rows(small):
    subs = small.subs
    bank = jerk.DeviceBank(subs)
    g = np.load(os.path.join(H.GOLDEN, "kernels_small.npz"))
    s0 = subs[0]
    n0 = s0["numw"] * s0["numz"]
    got = bank.rows(subs, 0, [0, n0 // 2, n0 - 1])
    for i in range(3):
        assert _rel_err(got[i], g["k_1_1_rows"][i]) <= ROW_TOL
    # subharmonic 1/8: w = 0 only (z-responses and the z = 0 sinc)
    i81 = [k for k, s in enumerate(subs) if (s["numharm"], s["harmnum"]) == (8, 1)][0]
    got = bank.rows(subs, i81, range(len(g["k_8_1_all"])))
    for i in range(len(got)):
        assert _rel_err(got[i], g["k_8_1_all"][i]) <= ROW_TOL
    i87 = [k for k, s in enumerate(subs) if (s["numharm"], s["harmnum"]) == (8, 7)][0]
    n87 = subs[i87]["numw"] * subs[i87]["numz"]
    got = bank.rows(subs, i87, [0, 7, 50, n87 - 1])
    for i in range(4):
        assert _rel_err(got[i], g["k_8_7_rows"][i]) <= ROW_TOL
    bank.close()


def test_small_bank_matches_reference_everywhere(small):
    bank = jerk.DeviceBank(small.subs)
    worst = 0.0
    for i, s in enumerate(small.subs):
        n = s["numw"] * s["numz"]
        got = bank.rows(small.subs, i, range(n))
        ref = s["kern"].reshape(n, s["fftlen"])
        for r in range(n):
            e = _rel_err(got[r], ref[r])
            worst = max(worst, e)
            assert e <= ROW_TOL, (i, r, e)
    bank.close()
    print(f"worst kernel-row error vs reference: {worst:.2e}")


def test_search_with_generated_bank_matches_golden(small):
    bank = jerk.DeviceBank(small.subs)
    subs = [{k: v for k, v in s.items() if k != "kern"} for s in small.subs]
    plan = jerk.JerkPlan(jerk.obs_from_refobs(small.obs), subs, batch=8, device_bank=bank.ptr.value)
    got = plan.search(small.spec)
    plan.close()
    bank.close()
    g = H.golden("small_cands.json")
    want = np.array([tuple(c) for c in g["cands"]], dtype=jerk.CAND_DTYPE)
    assert not H.compare_cands(got, want, g["obs"]["powcut"])


def test_paper_scale_bank_samples_match_reference(tmp_path):
    """-zmax 200 -wmax 300 -numharm 16: sampled rows of every subharmonic."""
    N, dt = 1 << 16, 54.6e-6
    spec = synth.presto_fft(np.random.default_rng(1).standard_normal(N).astype(np.float32))
    root = str(tmp_path / "paper")
    synth.write_fft(root, spec, N, dt)
    ref = ob.RefSearch(root + ".fft", ["-zmax", "200", "-wmax", "300", "-numharm", "16",
                                       "-sigma", "3.0"])
    obs = jerk.obs_from_refobs(ref.obs)
    subs = []
    for st, h in ref.subharmonics():
        subs.append(ref.shi_info(st, h))
    bank = jerk.DeviceBank(subs)
    rng = np.random.default_rng(2)
    worst = 0.0
    for i, (st, h) in enumerate(ref.subharmonics()):
        s = subs[i]
        n = s["numw"] * s["numz"]
        pick = sorted(set([0, n - 1, n // 2] + list(rng.integers(0, n, 6))))
        want = ref.kernels(st, h).reshape(n, s["fftlen"])[pick]
        got = bank.rows(subs, i, pick)
        for a, b in zip(got, want):
            e = _rel_err(a, b)
            worst = max(worst, e)
            assert e <= ROW_TOL, (i, e)
    bank.close()
    ref.close()
    print(f"worst sampled kernel-row error (z200 w300 h16): {worst:.2e}")


def _reference_kernel_row(z: float, w: float, fftlen: int) -> np.ndarray:
    """One bank row as the reference's init_kernel (src/accel_utils.c:151-168)
    makes it: gen_w_response from the reference build, placed wrapped around
    fftlen (src/corr_prep.c:92-114), forward FFT (here in FP64)."""
    import ctypes as C

    lib = ob._ref()
    lib.ref_w_resp_halfwidth.restype = C.c_int
    khw = lib.ref_w_resp_halfwidth(float(z), float(w), 0)  # LOWACC
    numkern = 2 * 2 * khw
    resp = np.zeros(numkern, dtype=np.complex64)
    lib.ref_gen_w_response(0.0, 2, float(z), float(w), numkern, resp.ctypes.data)
    row = np.zeros(fftlen, dtype=np.complex128)
    row[fftlen - numkern // 2:] = resp[: numkern // 2]
    row[: numkern // 2] = resp[numkern // 2:]
    return np.fft.fft(row)


def test_longest_fft_bank_samples_match_reference():
    """-zmax 1200 -wmax 1500 -numharm 2: the fundamental's kernels need fftlen
    15360 (1201 x 151 rows, 22 GB), the subharmonic's 10240.  Sampled rows of
    both against the reference's gen_w_response, placed and FFT'd as
    init_kernel does (the reference's own bank of this size would take hours
    on the CPU)."""
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("reference build missing")
    obs, fftlen, _ = jerk.obs_from_params(1 << 21, 1 << 22, 64e-6, 1200, 1500, 2, 3.0)
    assert fftlen == 15360
    subs = jerk.subharm_sizes(obs, fftlen)
    bank = jerk.DeviceBank(subs)
    rng = np.random.default_rng(3)
    worst = 0.0
    for i, s in enumerate(subs):
        n = s["numw"] * s["numz"]
        pick = sorted(set([0, n - 1, n // 2] + [int(v) for v in rng.integers(0, n, 5)]))
        got = bank.rows(subs, i, pick)
        for g, r in zip(got, pick):
            ii, jj = divmod(r, s["numz"])
            want = _reference_kernel_row(-s["zmax"] + 2 * jj, -s["wmax"] + 20 * ii, s["fftlen"])
            e = _rel_err(g.astype(np.complex128), want)
            worst = max(worst, e)
            assert e <= ROW_TOL, (i, r, e)
    bank.close()
    print(f"worst sampled kernel-row error (z1200 w1500, fftlen 15360): {worst:.2e}")
