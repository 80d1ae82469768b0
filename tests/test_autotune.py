"""The autotuner's cache (host side, no GPU): keyed by geometry, stored
atomically, read back by any later process; an unreadable file is a miss."""

import os

from prestozl_b200 import autotune, jerk


def test_cache_round_trip_and_geometry_key(tmp_path, monkeypatch):
    monkeypatch.setenv("JERK_TUNE_CACHE", str(tmp_path / "tune.json"))
    obs, fftlen, _ = jerk.obs_from_params(1 << 19, 1 << 20, 64e-6, 20, 60, 8, 2.0)
    subs = jerk.subharm_sizes(obs, fftlen)
    assert autotune.cached(obs, subs) is None
    key = autotune.geometry_key(obs, subs)
    assert key == f"fftlen={fftlen}:numz={obs.numz}:numw={obs.numw}:stages=4:uselen={obs.corr_uselen}"
    autotune._store({key: {"batch_rsteps": 32, "harm_mode": 1}})
    assert autotune.cached(obs, subs) == {"batch_rsteps": 32, "harm_mode": 1}
    assert not [f for f in os.listdir(tmp_path) if f.endswith(".tmp")]
    # another geometry is a miss
    obs2, fftlen2, _ = jerk.obs_from_params(1 << 19, 1 << 20, 64e-6, 50, 160, 8, 2.0)
    assert autotune.cached(obs2, jerk.subharm_sizes(obs2, fftlen2)) is None
    # a damaged file reads as empty
    (tmp_path / "tune.json").write_text("{not json")
    assert autotune.cached(obs, subs) is None
