"""Generate the golden fixtures in this folder by running the REFERENCE.

The reference's own CPU accelsearch objects are compiled from the reference
sources by ``oracle/Makefile`` (``oracle/_ref/libprestoref.so``); this script
drives them on seeded synthetic inputs and stores small results:

* ``small_cands.json``   the full search of the 2^20-sample spectrum with one
                         binary pulsar (-zmax 20 -wmax 60 -numharm 8
                         -sigma 2.0): the candidate list the reference builds
                         before its optimisation stage, plus its geometry.
* ``sizing.json``        accelobs sizing and per-subharmonic kernel sizes of
                         the reference for the benchmark's search parameters.
* ``sigma.json``         candidate_sigma / power_for_sigma on a grid.
* ``kernels_small.npz``  a few response-kernel FFTs of the small search's bank.
* ``small_ACCEL.txt``    the reference CLI's ACCEL output for the small search
                         (after its sort / harmonic removal / optimisation).
* ``small_ACCEL.cand``   the same run's binary .cand file: one fourierprops
                         record per candidate (src/accelsearch_lib.c:958-961).
* ``dedisp_small.npz``   two seeded blocks of 96 samples x 12 subbands, an
                         offsets table of 7 DMs (0 and 96 included) and the
                         reference's float_dedisp (src/dispersion.c:208-231)
                         of them, one call per DM as prepsubband makes them.

Run from the repository root after ``make -C oracle``:

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py dedisp     # only dedisp_small.npz
    python tests/golden/make_golden.py accel      # only small_ACCEL.txt / .cand
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import bindings as ob  # noqa: E402
from prestozl_b200 import synth  # noqa: E402

SMALL_ARGS = ["-zmax", "20", "-wmax", "60", "-numharm", "8", "-sigma", "2.0"]

# (zmax, wmax or None for no -wmax, numharm, sigma, with_subharmonics)
SIZING_SETS = [
    (20, 60, 8, 2.0, True),
    (200, 300, 16, 3.0, True),
    (50, 150, 8, 3.0, True),      # wmax 150 is rounded up to 160 by the reference
    (100, 0, 16, 3.0, True),      # -wmax 0: numw = 0, one w row per subharmonic
    (200, 300, 1, 3.0, True),
    (300, 600, 32, 4.0, False),   # bank too large to build here; geometry only
]


def spectrum_digest(spec: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(spec).tobytes()).hexdigest()


def obs_dict(o) -> dict:
    d = {}
    for name, _ in o._fields_:
        v = getattr(o, name)
        if name in ("powcut", "numindep"):
            v = list(v)[: o.numharmstages]
        d[name] = v
    return d


def small_cands(tmp: str) -> dict:
    spec, N, dt = synth.small_spectrum()
    root = os.path.join(tmp, "small")
    synth.write_fft(root, spec, N, dt)
    ob.set_threads(1)
    r = ob.RefSearch(root + ".fft", SMALL_ARGS)
    cands, nsteps = r.search()
    out = {
        "args": SMALL_ARGS,
        "N": N, "dt": dt, "seed": 20241203,
        "spectrum_sha256": spectrum_digest(spec),
        "obs": obs_dict(r.obs),
        "nrsteps": nsteps,
        "cands": [[float(c["power"]), float(c["sigma"]), int(c["numharm"]), float(c["r"]),
                   float(c["z"]), float(c["w"])] for c in cands],
    }
    # a few kernels of the bank
    ks = {}
    k0 = r.kernels(0, 1)
    ks["k_1_1_rows"] = k0.reshape(-1, k0.shape[-1])[[0, k0.shape[0] * k0.shape[1] // 2, -1]]
    ks["k_8_1_all"] = r.kernels(3, 1).reshape(-1, r.shi_info(3, 1)["fftlen"])
    k37 = r.kernels(3, 7)
    ks["k_8_7_rows"] = k37.reshape(-1, k37.shape[-1])[[0, 7, 50, -1]]
    np.savez_compressed(os.path.join(HERE, "kernels_small.npz"), **ks)
    r.close()
    return out


def accel_small(tmp: str) -> None:
    import shutil
    import subprocess

    spec, N, dt = synth.small_spectrum()
    root = os.path.join(tmp, "small")
    synth.write_fft(root, spec, N, dt)
    env = dict(os.environ, PRESTO=tmp, OMP_NUM_THREADS="1")
    subprocess.run([ob.REF_CLI, *SMALL_ARGS, "small.fft"], cwd=tmp, env=env, check=True,
                   stdout=subprocess.DEVNULL)
    shutil.copy(os.path.join(tmp, "small_ACCEL_20_JERK_60"), os.path.join(HERE, "small_ACCEL.txt"))
    shutil.copy(os.path.join(tmp, "small_ACCEL_20_JERK_60.cand"),
                os.path.join(HERE, "small_ACCEL.cand"))


def sizing(tmp: str) -> list:
    # geometry does not depend on the data: a short white-noise file will do
    N, dt = 1 << 18, 54.6e-6
    spec = synth.presto_fft(np.random.default_rng(7).standard_normal(N).astype(np.float32))
    root = os.path.join(tmp, "geom")
    synth.write_fft(root, spec, N, dt)
    res = []
    for zmax, wmax, nh, sig, with_subs in SIZING_SETS:
        args = ["-zmax", str(zmax), "-numharm", str(nh), "-sigma", str(sig)]
        if wmax is not None:
            args += ["-wmax", str(wmax)]
        r = ob.RefSearch(root + ".fft", args)
        entry = {"zmax": zmax, "wmax": wmax, "numharm": nh, "sigma": sig, "N": N, "dt": dt,
                 "numbins": len(spec), "obs": obs_dict(r.obs)}
        if with_subs:
            entry["subs"] = [r.shi_info(st, h) for st, h in r.subharmonics()]
        res.append(entry)
        r.close()
    return res


def sigma_grid() -> dict:
    rows = []
    for numsum in (1, 2, 4, 8, 16, 32):
        for numindep in (1.0e3, 1.2e7, 5.0e9):
            for power in (0.5, 3.0, 10.0, 20.0, 35.0, 60.0, 120.0, 400.0, 2000.0):
                rows.append([power, numsum, numindep, ob.candidate_sigma(power, numsum, numindep)])
    cuts = []
    for numsum in (1, 2, 4, 8, 16, 32):
        for numindep in (1.0e3, 1.2e7, 5.0e9):
            for sig in (2.0, 3.0, 4.0, 6.0):
                cuts.append([sig, numsum, numindep, ob.power_for_sigma(sig, numsum, numindep)])
    return {"candidate_sigma": rows, "power_for_sigma": cuts}


def dedisp_small() -> None:
    rng = np.random.default_rng(96)
    worklen, nsub, numdms = 96, 12, 7
    cur = (rng.standard_normal((worklen, nsub)) * 25 + 80).astype(np.float32)
    last = (rng.standard_normal((worklen, nsub)) * 25 + 80).astype(np.float32)
    off = rng.integers(0, worklen + 1, (numdms, nsub)).astype(np.int32)
    off[0] = 0
    off[1] = worklen
    out = ob.dedisp_subbands(cur, last, off, reference=True)
    np.savez_compressed(os.path.join(HERE, "dedisp_small.npz"), cur=cur, last=last,
                        offsets=off, out=out)


def main() -> None:
    ob.build()
    if sys.argv[1:] == ["dedisp"]:
        dedisp_small()
        return
    if sys.argv[1:] == ["accel"]:
        with tempfile.TemporaryDirectory() as tmp:
            accel_small(tmp)
        return
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(HERE, "small_cands.json"), "w") as f:
            json.dump(small_cands(tmp), f, indent=1)
        with open(os.path.join(HERE, "sizing.json"), "w") as f:
            json.dump(sizing(tmp), f, indent=1)
    with tempfile.TemporaryDirectory() as tmp:
        accel_small(tmp)
    with open(os.path.join(HERE, "sigma.json"), "w") as f:
        json.dump(sigma_grid(), f, indent=1)
    dedisp_small()


if __name__ == "__main__":
    main()
