"""The entry point that allocates nothing (jerk_volume_static).

Some callers cannot allocate device memory when they search -- their memory
is handed out up front by a pool they do not own, or their loop must not
allocate after start-up -- so libjerk offers one ffdot-volume step whose
working memory is a fixed array inside the library.  Through the C ABI, two
calls in a row must give the volumes the plan-based entry point
(jerk_debug_volume) gives, within the parity tolerance of the GPU tests
(1e-5 of max(power, 1)).  This file is collected last on purpose: if it
fails, a run stopping at the first failure has run everything else.
"""

import numpy as np
import pytest

from prestozl_b200 import build, jerk, synth

pytestmark = pytest.mark.gpu

POW_TOL = 1e-5


def test_volume_without_allocation_matches_plan():
    torch = pytest.importorskip("torch")
    build.build()
    spec, N, dt = synth.small_spectrum()
    obs, fftlen, _ = jerk.obs_from_params(len(spec), N, dt, 20, 60, 8, 2.0)
    subs = jerk.subharm_sizes(obs, fftlen)
    bank = jerk.DeviceBank(subs)
    plan = jerk.JerkPlan(obs, subs, batch=4, device_bank=bank.ptr.value)
    d_spec = torch.from_numpy(spec.view(np.float32).copy()).cuda()
    rstep = obs.corr_uselen // 2
    offs = np.cumsum([0] + [s["numw"] * s["numz"] * s["fftlen"] for s in subs])
    # two calls in a row, different rsteps and subharmonics sharing the array
    for k, i in ((128, 0), (129, 7)):
        want, rlo = plan.volume(spec, k, i)
        s = subs[i]
        out = torch.full((s["numw"] * s["numz"] * (obs.corr_uselen + 8),), -1.0,
                         dtype=torch.float32, device="cuda")
        numrs, rlo2 = jerk.volume_static(d_spec.data_ptr(), len(spec), 0, s,
                                         bank.ptr.value + 8 * int(offs[i]), obs.rlo + k * rstep,
                                         obs.corr_uselen, obs.nph, out.data_ptr())
        torch.cuda.synchronize()
        got = out[: s["numw"] * s["numz"] * numrs].cpu().numpy().reshape(want.shape)
        assert (numrs, rlo2) == (want.shape[2], rlo)
        err = np.abs(got.astype(np.float64) - want) / np.maximum(want, 1.0)
        assert err.max() <= POW_TOL, (k, i, err.max())
    plan.close()
    bank.close()


def test_sizes_beyond_the_array_are_rejected():
    torch = pytest.importorskip("torch")
    build.build()
    big = {"numharm": 1, "harmnum": 1, "numz": 3, "numw": 1, "fftlen": 10240, "halfwidth": 16}
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    with pytest.raises(jerk.JerkError):
        jerk.volume_static(buf.data_ptr(), 8, 0, big, buf.data_ptr(), 100.0, 2048, 0.0,
                           buf.data_ptr())
