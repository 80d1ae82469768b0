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
