"""Shared set-up for the parity tests: seeded spectra on disk, the reference's
kernel bank and geometry (via the oracle's reference build), and comparison
helpers.  The oracle is the checker here and nowhere else."""

from __future__ import annotations

import functools
import json
import os

import numpy as np

from oracle import bindings as ob
from prestozl_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def ensure_oracle() -> None:
    if not os.path.exists(ob.ORACLE_LIB):
        ob.build(reference=False)


def have_ref() -> bool:
    return ob.have_reference()


class Problem:
    """A spectrum written as .fft/.inf plus the reference's view of it."""

    def __init__(self, workdir: str, spec: np.ndarray, N: int, dt: float, args):
        self.spec = np.ascontiguousarray(spec, dtype=np.complex64)
        self.N, self.dt, self.args = N, dt, list(args)
        root = os.path.join(workdir, "spec")
        synth.write_fft(root, self.spec, N, dt)
        ob.set_threads(1)
        self.ref = ob.RefSearch(root + ".fft", self.args)
        self.obs = self.ref.obs
        self.subs = []
        for st, h in self.ref.subharmonics():
            info = self.ref.shi_info(st, h)
            info["kern"] = self.ref.kernels(st, h)
            self.subs.append(info)
        self.geom = ob.geom_from_refobs(self.obs)
        self.oracle = ob.Oracle(self.spec, self.geom, self.subs)

    @property
    def rstep(self) -> int:
        return self.obs.corr_uselen // 2

    def startr(self, k: int) -> float:
        return self.obs.rlo + k * self.rstep

    def rstep_of(self, r: float) -> int:
        return int((r - self.obs.rlo) // self.rstep)


@functools.lru_cache(maxsize=None)
def small_problem(workdir: str) -> Problem:
    spec, N, dt = synth.small_spectrum()
    return Problem(workdir, spec, N, dt, golden("small_cands.json")["args"])


def near_cutoff(power: float, numharm: int, powcut, rel: float = 1e-4) -> bool:
    stage = int(np.log2(numharm))
    return abs(power - powcut[stage]) <= rel * powcut[stage]


def compare_cands(got: np.ndarray, want: np.ndarray, powcut, rel_pow: float = 1e-5,
                  rel_sig: float = 1e-5):
    """Candidate lists must match in (numharm, r, z, w) except entries whose
    power is within 1e-4 of the stage cutoff; matched powers and sigmas must
    agree to the given relative tolerance.  Returns a list of problems."""
    problems = []
    key = lambda c: (int(c["numharm"]), round(float(c["r"]), 6), round(float(c["z"]), 6),
                     round(float(c["w"]), 6))
    gd = {key(c): c for c in got}
    wd = {key(c): c for c in want}
    for k, c in wd.items():
        if k not in gd:
            if not near_cutoff(float(c["power"]), k[0], powcut):
                problems.append(("missing", k, float(c["power"])))
            continue
        g = gd[k]
        if abs(float(g["power"]) - float(c["power"])) > rel_pow * abs(float(c["power"])):
            problems.append(("power", k, float(g["power"]), float(c["power"])))
        if abs(float(g["sigma"]) - float(c["sigma"])) > rel_sig * max(abs(float(c["sigma"])), 1e-3):
            problems.append(("sigma", k, float(g["sigma"]), float(c["sigma"])))
    for k, c in gd.items():
        if k not in wd and not near_cutoff(float(c["power"]), k[0], powcut):
            problems.append(("extra", k, float(c["power"])))
    return problems
