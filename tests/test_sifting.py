"""Downstream compatibility of the ACCEL output (no GPU): the reference's own
sifting parser, candlist_from_candfile (python/presto/sifting.py:1077-1181),
reads the ACCEL file of the small search.  The drop-in writes its ACCEL file
with the reference's own CPU2 (output_fundamentals / output_harmonics) and
tests/test_gpu_dropin.py holds it equal to this golden file, so this is the
file sifting gets from the drop-in, up to the last printed digit of the
search's summed power and sigma.

sifting.py imports matplotlib (absent here) and presto.presto, the SWIG
wrapper of the C library, for candidate_sigma only; the test gives it a
stand-in for the first and the reference build's own candidate_sigma
(oracle/_ref) for the second.  It reads the parser from the reference
checkout, so it runs where the checkout is and is skipped elsewhere.
"""

import importlib.util
import os
import shutil
import sys
import types

import pytest

from oracle import bindings as ob
from tests import helpers as H


def load_sifting():
    path = os.path.join(ob.REFERENCE_SOURCES, "python", "presto", "sifting.py")
    if not os.path.exists(path):
        pytest.skip("the reference checkout (python/presto) is not here")
    H.ensure_oracle()
    if not H.have_ref():
        pytest.skip("the reference build (oracle/_ref) provides candidate_sigma")
    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot", "presto",
                                             "presto.presto", "presto.infodata",
                                             "presto.sifting")}
    # plotting is never reached by the parser; the module body only defines
    # and registers a plot scale (classes derived from two matplotlib bases)
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    mpl.scale = types.SimpleNamespace(ScaleBase=object, register_scale=lambda *a, **k: None)
    mpl.transforms = types.SimpleNamespace(Transform=object)
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    pkg = types.ModuleType("presto")
    pkg.__path__ = [os.path.dirname(path)]
    swig = types.ModuleType("presto.presto")
    swig.candidate_sigma = ob.candidate_sigma
    sys.modules.update({"matplotlib": mpl, "matplotlib.pyplot": plt, "presto": pkg,
                        "presto.presto": swig})
    try:
        spec = importlib.util.spec_from_file_location("presto.sifting", path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules["presto.sifting"] = mod
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


def fundamental_rows(text: str):
    rows = []
    for line in text.splitlines():
        t = line.split()
        if line.startswith(" Data file name"):
            break
        if t and t[0].isdigit() and len(t) > 9 and not t[1].isdigit() and "(" in t[7]:
            rows.append(t)
    return rows


def test_reference_sifting_reads_the_accel_file(tmp_path):
    sifting = load_sifting()
    # sifting takes the DM from the file name (..._DM<dm>_ACCEL...)
    name = tmp_path / "small_DM0.00_ACCEL_20_JERK_60"
    shutil.copy(os.path.join(H.GOLDEN, "small_ACCEL.txt"), name)
    cl = sifting.candlist_from_candfile(str(name))
    rows = fundamental_rows(name.read_text())
    assert len(cl.cands) == len(rows) > 0
    for c, t in zip(cl.cands, rows):
        assert c.candnum == int(t[0])
        assert c.numharm == int(t[4])
        assert c.r == float(t[7].split("(")[0])
        assert c.z == float(t[9].split("(")[0])
        assert c.DMstr == "0.00"
        # the harmonic table was read and the optimised sigma recomputed
        assert len(c.harm_pows) == c.numharm and c.snr > 0 and c.sigma > 0
    # the pulsar (123.4 Hz, 5 harmonics) is the first candidate
    assert abs(cl.cands[0].f - 123.4) < 0.01
