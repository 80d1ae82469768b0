"""Autotuning of rsteps per launch (the batch size B) per search geometry.

B trades kernel-bank reuse (each kernel row is read from HBM once per batch
and kept in registers for B rsteps) against the size of the double-buffered
ffdot volumes (2 x B x ~160 MB at -zmax 200 -wmax 300 -numharm 16) and the
granularity of the overlap between a batch's harmonic sums and the next
batch's correlations.  The best B depends on the geometry (fftlen, numz,
numw, stages, corr_uselen), so it is measured once on a short partial search
and cached in a JSON file (``$JERK_TUNE_CACHE``, default
``~/.cache/prestozl_b200/autotune.json``).

The FFT radix plans are fixed per fftlen (``csrc/jerk_fft.cuh``) and the
kernels' tile shapes are compile-time; the run-time knobs are B and the
harmonic-sum kernel (jerk_config.harm_mode: plain gathers, gathers with TMA
prefetch into L2, or TMA tiles in shared memory).
"""

from __future__ import annotations

import json
import os
from typing import Dict, Optional, Sequence

from . import jerk

DEFAULT_CANDIDATES = (16, 32, 64)
DEFAULT_HARM_MODES = (1, 2, 4)


def cache_path() -> str:
    return os.environ.get("JERK_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "prestozl_b200",
                                       "autotune.json"))


def geometry_key(obs: jerk.Obs, subs: Sequence[dict]) -> str:
    f = subs[0]
    return (f"fftlen={f['fftlen']}:numz={f['numz']}:numw={f['numw']}:"
            f"stages={obs.numharmstages}:uselen={obs.corr_uselen}")


def _load() -> Dict[str, dict]:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(db: Dict[str, dict]) -> None:
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    # one temporary file per process: ranks of one node may store at once;
    # os.replace is atomic, so readers see one whole file or another
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as fh:
        json.dump(db, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def cached(obs: jerk.Obs, subs: Sequence[dict]) -> Optional[dict]:
    """The cached choice for this geometry ({"batch_rsteps", "harm_mode", ...})."""
    return _load().get(geometry_key(obs, subs))


def tune(obs: jerk.Obs, subs: Sequence[dict], bank_ptr: int, spectrum,
         candidates: Sequence[int] = DEFAULT_CANDIDATES,
         harm_modes: Sequence[int] = DEFAULT_HARM_MODES, rsteps: int = 1024,
         use_cache: bool = True) -> dict:
    """Time a partial search of ``rsteps`` rsteps for each (B, harm_mode) pair
    (the spectrum may be a CUDA tensor or a host array) and cache the fastest.
    Both knobs change only speed: the candidates are the same for all."""
    import torch

    key = geometry_key(obs, subs)
    db = _load() if use_cache else {}
    if use_cache and key in db:
        return db[key]
    times = {}
    for B in candidates:
        for hr in harm_modes:
            try:
                plan = jerk.JerkPlan(obs, subs, batch=B, device_bank=bank_ptr, harm_mode=hr)
            except jerk.JerkError:
                continue  # e.g. volumes beyond 32-bit offsets, or out of memory
            n = min(rsteps, plan.num_rsteps)
            plan.search(spectrum, 0, max(B, n // 4))  # warm
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            plan.search(spectrum, 0, n)
            e1.record()
            torch.cuda.synchronize()
            times[(B, hr)] = e0.elapsed_time(e1) / n
            plan.close()
    if not times:
        raise RuntimeError("no batch size could be planned")
    best = min(times, key=times.get)
    entry = {"batch_rsteps": best[0], "harm_mode": best[1],
             "ms_per_rstep": {f"B{k[0]}/mode{k[1]}": v for k, v in times.items()},
             "rsteps_timed": rsteps}
    if use_cache:
        db[key] = entry
        _store(db)
    return entry
