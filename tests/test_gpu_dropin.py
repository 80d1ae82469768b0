"""The drop-in, end to end: the reference's own accelsearch_cu main and its
accelsearch_CPU1 / accelsearch_CPU2, around this project's accelsearch_GPU
(oracle/_ref/accelsearch_b200, built by `make -C oracle dropin`), must write
the ACCEL file the reference's CPU accelsearch writes for the same spectrum
and flags (tests/golden/small_ACCEL.txt).

Every field of both ACCEL tables must match as printed, except the search's
summed power and its sigma (columns 2 and 3 of the first table), which come
from FP32 powers and may differ in the last printed digit (tolerance 0.011).
"""

import os
import subprocess

import pytest

from oracle import bindings as ob
from prestozl_b200 import build, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


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
