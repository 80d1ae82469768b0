"""The drop-in, end to end: the reference's own accelsearch_cu main and its
accelsearch_CPU1 / accelsearch_CPU2, around this project's accelsearch_GPU
(oracle/_ref/accelsearch_b200, built by `make -C oracle dropin`), must write
the ACCEL file the reference's CPU accelsearch writes for the same spectrum
and flags (tests/golden/small_ACCEL.txt).

Every field of both ACCEL tables must match as printed, except the search's
summed power and its sigma (columns 2 and 3 of the first table), which come
from FP32 powers and may differ in the last printed digit (tolerance 0.011).
The binary .cand file (one fourierprops record per candidate,
src/accelsearch_lib.c:958-961) must equal the reference's field for field
(tests/golden/small_ACCEL.cand).  Both files are written by the reference's
own CPU2, so downstream tools read them as they read the reference's
(tests/test_sifting.py runs the reference's sifting parser on the ACCEL
file).
"""

import os
import subprocess

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


# fourierprops (include/presto.h:171-189) as the reference writes it (x86-64
# alignment: the doubles on 8-byte boundaries)
FOURIERPROPS = np.dtype([("r", "f8"), ("rerr", "f4"), ("z", "f8"), ("zerr", "f4"), ("w", "f8"),
                         ("werr", "f4"), ("pow", "f4"), ("powerr", "f4"), ("sig", "f4"),
                         ("rawpow", "f4"), ("phs", "f4"), ("phserr", "f4"), ("cen", "f4"),
                         ("cenerr", "f4"), ("pur", "f4"), ("purerr", "f4"), ("locpow", "f4")],
                        align=True)


def read_cand(path: str) -> np.ndarray:
    raw = open(path, "rb").read()
    assert len(raw) % FOURIERPROPS.itemsize == 0, len(raw)
    return np.frombuffer(raw, dtype=FOURIERPROPS)


def accel_rows(text: str):
    rows = []
    for line in text.splitlines():
        t = line.split()
        if t and t[0].isdigit() and len(t) > 5:
            rows.append(t)
        elif line.startswith(" Data file name"):
            break  # the appended .inf
    return rows


def test_dropin_accel_matches_reference(tmp_path):
    build.build()
    if not os.path.exists(ob.DROPIN_CLI):
        pytest.skip("drop-in binary not built (reference sources absent at build time)")
    spec, N, dt = synth.small_spectrum()
    synth.write_fft(str(tmp_path / "small"), spec, N, dt)
    args = H.golden("small_cands.json")["args"]
    env = dict(os.environ, PRESTO=str(tmp_path), OMP_NUM_THREADS="1")
    out = subprocess.run([ob.DROPIN_CLI, *args, "small.fft"], cwd=tmp_path, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    got = accel_rows((tmp_path / "small_ACCEL_20_JERK_60").read_text())
    want = accel_rows(open(os.path.join(H.GOLDEN, "small_ACCEL.txt")).read())
    assert len(got) == len(want) > 0
    fund = True
    for g, w in zip(got, want):
        assert len(g) == len(w)
        for i, (a, b) in enumerate(zip(g, w)):
            if a == b:
                continue
            # first table: Cand, Sigma, Summed Power, ... (sigma/power from FP32 powers)
            assert fund and i in (1, 2), (g, w)
            assert abs(float(a) - float(b)) <= 0.011, (g, w)
        if len(g) > 12 and g[1].isdigit():
            fund = False  # second table rows start "cand harm"
    # the .cand records, field by field (padding bytes are not data)
    gc = read_cand(str(tmp_path / "small_ACCEL_20_JERK_60.cand"))
    wc = read_cand(os.path.join(H.GOLDEN, "small_ACCEL.cand"))
    assert len(gc) == len(wc) > 0
    for f in FOURIERPROPS.names:
        assert np.array_equal(gc[f], wc[f]), (f, gc[f], wc[f])


def test_dropin_many_spectra_in_one_process(tmp_path):
    """A pool worker searches many spectra in one process
    (bin/accelsearch_pipeline_cu.py): the drop-in keeps its GPU kernel bank
    between calls of one geometry.  Three spectra searched in one process
    write the ACCEL files that three separate runs write."""
    import numpy as np

    build.build()
    if not (os.path.exists(ob.DROPIN_CLI) and os.path.exists(ob.DROPIN_MANY_CLI)):
        pytest.skip("drop-in binaries not built (reference sources absent at build time)")
    args = H.golden("small_cands.json")["args"]
    N, dt = 1 << 20, 64e-6
    names = []
    many = tmp_path / "many"
    many.mkdir()
    for i, seed in enumerate((20241203, 5, 6)):
        if i == 0:
            spec, N, dt = synth.small_spectrum()
        else:
            rng = np.random.default_rng(seed)
            ps = synth.random_pulsars(rng, 2, zmax=16.0, wmax=48.0, fmax=200.0)
            spec = synth.presto_fft(synth.timeseries(N, dt, ps, seed))
        name = f"s{i}"
        names.append(name)
        one = tmp_path / name
        one.mkdir()
        for d in (one, many):
            synth.write_fft(str(d / name), spec, N, dt)
        env = dict(os.environ, PRESTO=str(one), OMP_NUM_THREADS="1")
        out = subprocess.run([ob.DROPIN_CLI, *args, name + ".fft"], cwd=one, env=env,
                             capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
    env = dict(os.environ, PRESTO=str(many), OMP_NUM_THREADS="1")
    out = subprocess.run([ob.DROPIN_MANY_CLI, *args, "--", *[n + ".fft" for n in names]],
                         cwd=many, env=env, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    print(out.stderr.strip())
    for n in names:
        a = (tmp_path / n / f"{n}_ACCEL_20_JERK_60").read_text()
        b = (many / f"{n}_ACCEL_20_JERK_60").read_text()
        assert a == b, n
    assert len(accel_rows((many / "s0_ACCEL_20_JERK_60").read_text())) > 0
