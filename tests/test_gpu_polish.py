"""Candidate polishing on the GPU (jerk_polish_rzw) against the reference's
own harmonic polishing, max_rzw_arr_harmonics (src/maximize_rzw.c:84-190),
run from the reference build on the same spectrum with the same local
powers.

The polished (r, z, w) are points of a fixed grid, so they must be equal
exactly: the GPU's FP32 FFTs differ from the reference's in rounding only,
and the maximum moves only if two grid powers tie to that rounding (none in
these cases).  The summed power at the maximum agrees to 1e-4 relative.
"""

import time

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    build.build()
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) is the comparator")


def compare(ref, spec, cands, pol):
    lobin = ref.obs.lobin
    t_ref = t_gpu = 0.0
    rows = []
    for nh, r, z, w in cands:
        t0 = time.perf_counter()
        want, lp = ref.polish(nh, r - lobin, z, w)
        t1 = time.perf_counter()
        got = pol.polish(spec, nh, r - lobin, z, w, lp)
        t2 = time.perf_counter()
        t_ref += t1 - t0
        t_gpu += t2 - t1
        rows.append((nh, r, z, w, want, got[:3]))
    bad = [x for x in rows if x[4] != x[5]]
    return rows, bad, t_ref, t_gpu


def test_polish_small_golden_candidates(tmp_path):
    spec, N, dt = synth.small_spectrum()
    root = str(tmp_path / "small")
    synth.write_fft(root, spec, N, dt)
    g = H.golden("small_cands.json")
    ref = ob.RefSearch(root + ".fft", g["args"])
    cands = [(int(c[2]), c[3], c[4], c[5]) for c in g["cands"]]
    # the same candidates at fewer harmonics, and at w = 0 (the z-only responses)
    cands += [(nh, r, z * nh / 8, w * nh / 8) for nh in (1, 2, 4) for _, r, z, w in cands[:3]]
    cands += [(8, r, z, 0.0) for _, r, z, w in cands[:3]]
    pol = jerk.Polisher()
    rows, bad, t_ref, t_gpu = compare(ref, spec, cands, pol)
    pol.close()
    ref.close()
    print(f"{len(rows)} candidates: reference {t_ref:.2f} s, GPU {t_gpu:.3f} s")
    assert not bad, bad[:5]


def test_polish_paper_scale():
    """2^25 samples, -zmax 200 -wmax 300 -numharm 16: candidates at four
    injected pulsars (all harmonic counts) and at noise positions."""
    torch = pytest.importorskip("torch")
    import tempfile

    N, dt = 1 << 25, 54.6e-6
    pulsars = synth.random_pulsars(np.random.default_rng(0), 4)
    spec = synth.presto_fft_torch(synth.timeseries_torch(N, dt, pulsars, 0, device="cuda"))
    spec = spec.cpu().numpy()
    torch.cuda.synchronize()
    with tempfile.TemporaryDirectory() as d:
        synth.write_fft(d + "/paper", spec, N, dt)
        ref = ob.RefSearch(d + "/paper.fft", ["-zmax", "200", "-wmax", "300", "-numharm", "16",
                                              "-sigma", "3.0"])
        T = N * dt
        cands = []
        for p in pulsars:
            for nh in (1, 2, 4, 8, 16):
                # the search reports the fundamental on its grid: r to 1/2, z to 2/nh, w to 20/nh
                r = round(p.f * T * 2) / 2
                z = round(p.z * nh / 2) * 2 / nh
                w = round(p.w * nh / 20) * 20 / nh
                if abs(z * nh) <= 200 and abs(w * nh) <= 300:
                    cands.append((nh, r, z, w))
        rng = np.random.default_rng(5)
        for nh in (1, 4, 16):
            for _ in range(3):
                r = float(rng.integers(20000, (1 << 24) // nh - 20000)) + 0.5 * rng.integers(2)
                z = float(rng.integers(-100, 101)) * 2 / nh
                w = float(rng.integers(-15, 16)) * 20 / nh
                cands.append((nh, r, z, w))
        pol = jerk.Polisher()
        rows, bad, t_ref, t_gpu = compare(ref, spec, cands, pol)
        pol.close()
        ref.close()
    print(f"{len(rows)} paper-scale candidates: reference {t_ref:.1f} s, GPU {t_gpu:.3f} s "
          f"({t_ref / max(t_gpu, 1e-9):.0f}x)")
    assert not bad, bad[:5]


def test_polish_rejects_before_device_work():
    pol = jerk.Polisher()
    spec = np.zeros(1 << 16, dtype=np.complex64)
    with pytest.raises(jerk.JerkError) as ei:
        pol.polish(spec, 0, 1000.0, 0.0, 0.0, [])
    assert ei.value.code == jerk.JERK_EINVAL
    with pytest.raises(jerk.JerkError) as ei:  # first harmonic below bin 0
        pol.polish(spec, 2, 0.2, 0.0, 0.0, [1.0, 1.0])
    assert ei.value.code == jerk.JERK_EINVAL
    pol.close()


def _ref_optimize(ref, nh, r, z, w, power=20.0):
    """The reference's optimize_accelcand on one candidate: (r, z, w) of the
    fundamental (r absolute) and its per-harmonic derivatives."""
    import ctypes as C

    f = ob._ref().ref_optimize_cand
    f.argtypes = [C.c_void_p, C.c_float, C.c_int, C.c_double, C.c_double, C.c_double,
                  C.c_void_p, C.POINTER(C.c_float)]
    out = np.zeros(11 * nh)
    sig = C.c_float()
    assert f(ref.ctx, power, nh, r, z, w, out.ctypes.data, C.byref(sig)) == 0
    o = out.reshape(nh, 11)
    return (o[0, 1], o[0, 2], o[0, 3]), o[:, 4:11]


def test_optimize_wholly_on_gpu_matches_reference(tmp_path):
    """jerk_optimize_cand -- local powers, the volume search and the peak
    derivatives all on the GPU -- against the reference's optimize_accelcand
    on the golden small-problem candidates.

    Tolerances: polished r, z, w equal; power at the peak and local power to
    2e-5 relative (FP32 rounding of the interpolations, whose responses come
    from FFTs of other rounding); phase to 1e-4 rad; the finite differences
    (steps of 0.003 bins) amplify that rounding by 1 / 0.006 and
    1 / 0.000036, so dpow to 1e-3 and d2pow to 0.1 of the power (the
    reference's own float interpolations carry noise of that order)."""
    spec, N, dt = synth.small_spectrum()
    root = str(tmp_path / "small")
    synth.write_fft(root, spec, N, dt)
    g = H.golden("small_cands.json")
    ref = ob.RefSearch(root + ".fft", g["args"])
    lobin = ref.obs.lobin
    pol = jerk.Polisher()
    worst = {"pow": 0.0, "locpow": 0.0, "phs": 0.0, "dpow": 0.0, "d2pow": 0.0}
    for c in g["cands"]:
        nh, r, z, w = int(c[2]), c[3], c[4], c[5]
        (rr, zz, ww), want = _ref_optimize(ref, nh, r, z, w)
        (gr, gz, gw), got, _ = pol.optimize(spec, nh, r - lobin, z, w)
        assert (gr + lobin, gz, gw) == (rr, zz, ww), (c, (gr + lobin, gz, gw), (rr, zz, ww))
        for h in range(nh):
            p = want[h, 0]
            e_pow = abs(got["pow"][h] - p) / p
            e_lp = abs(got["locpow"][h] - want[h, 6]) / want[h, 6]
            dphs = abs(got["phs"][h] - want[h, 1])
            e_phs = min(dphs, abs(dphs - 2 * np.pi))
            e_dp = abs(got["dpow"][h] - want[h, 2]) / p
            e_d2 = abs(got["d2pow"][h] - want[h, 4]) / p
            for k, v in (("pow", e_pow), ("locpow", e_lp), ("phs", e_phs), ("dpow", e_dp),
                         ("d2pow", e_d2)):
                worst[k] = max(worst[k], v)
            assert e_pow <= 2e-5 and e_lp <= 2e-5 and e_phs <= 1e-4, (c, h, e_pow, e_lp, e_phs)
            assert e_dp <= 1e-3 and e_d2 <= 0.1, (c, h, e_dp, e_d2)
    pol.close()
    ref.close()
    print("worst GPU-optimisation differences vs the reference:",
          {k: f"{v:.2e}" for k, v in worst.items()})


def test_device_spectrum_equals_host_spectrum(tmp_path):
    """The polisher on a spectrum held in device memory (a CUDA tensor: a
    kernel gathers the windows) gives the same bits as on the same spectrum
    in host memory: golden candidates, candidates at the spectrum's two ends
    (windows reaching past them read zeros) and local powers on bin values
    (z = w = 0 at whole r, answered by the values themselves)."""
    torch = pytest.importorskip("torch")
    spec, N, dt = synth.small_spectrum()
    root = str(tmp_path / "small")
    synth.write_fft(root, spec, N, dt)
    g = H.golden("small_cands.json")
    ref = ob.RefSearch(root + ".fft", g["args"])
    lobin = ref.obs.lobin
    ref.close()
    n = len(spec)
    dspec = torch.from_numpy(spec).cuda()
    pol = jerk.Polisher()
    cands = [(int(c[2]), c[3] - lobin, c[4], c[5]) for c in g["cands"]]
    cands += [(2, 3.0, 0.0, 0.0), (1, 40.5, 2.0, -20.0), (1, n - 30.5, -4.0, 20.0)]
    for nh, r, z, w in cands:
        h_rzw, h_d, h_lp = pol.optimize(spec, nh, r, z, w)
        d_rzw, d_d, d_lp = pol.optimize(dspec, nh, r, z, w)
        assert h_rzw == d_rzw, (nh, r, z, w)
        assert h_d.tobytes() == d_d.tobytes() and h_lp.tobytes() == d_lp.tobytes()
        assert pol.polish(spec, nh, r, z, w, h_lp) == pol.polish(dspec, nh, r, z, w, h_lp)
    r = np.array([0.0, 1.0, 17.0, 1000.0, n - 25.0, n - 1.0, 5.5, n + 3.0])
    zw = np.zeros_like(r)
    assert np.array_equal(pol.local_power(spec, r, zw, zw), pol.local_power(dspec, r, zw, zw))
    with pytest.raises(jerk.JerkError):
        pol.optimize(dspec.view(torch.float32), 1, 1000.0, 0.0, 0.0)
    pol.close()
