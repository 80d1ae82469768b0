"""Subband dedispersion on the GPU (jerk_downsample_subbands,
jerk_dedisp_subbands): prepsubband_cu's GPU steps (src/prepsubband_kernels.cu),
whose DM-trial series the search takes.

Bar: bit-exact.  Against the oracle's restatement (itself equal bitwise to
the reference's float_dedisp, tests/test_oracle.py) and, where the reference
build is present, against the reference's own DownsampDataArray / getDedisp
compiled for sm_100a, called through the drop-in's symbols of the same names.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import bindings as ob
from prestozl_b200 import build, jerk
from tests import helpers as H

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def built():
    build.build()
    H.ensure_oracle()


def dispersion_offsets(numdms: int, nsub: int, worklen: int, dm0: float, ddm: float,
                       dt: float = 64e-6, flo: float = 1200.0, bw: float = 400.0) -> np.ndarray:
    """Offsets as prepsubband makes them (src/prepsubband_cu.c:458-467): the
    cold-plasma delay of each subband's centre relative to the top one, in
    samples, rounded to the nearest; clipped to the block."""
    f = flo + (np.arange(nsub) + 0.5) * bw / nsub
    dms = dm0 + ddm * np.arange(numdms)
    delay = 4.148808e3 * dms[:, None] * (f[None, :] ** -2 - f[-1] ** -2)
    return np.minimum(np.rint(delay / dt), worklen).astype(np.int32)


def blocks(worklen: int, nsub: int, seed: int):
    rng = np.random.default_rng(seed)
    cur = (rng.standard_normal((worklen, nsub)) * 20 + 100).astype(np.float32)
    last = (rng.standard_normal((worklen, nsub)) * 20 + 100).astype(np.float32)
    return cur, last


CASES = [
    # worklen, nsub, numdms, offsets
    ("paper-like 64 subbands", 8192, 64, 96, "disp"),
    ("ragged: 13 subbands, 1000 samples, 37 DMs", 1000, 13, 37, "random"),
    ("offsets at 0 and at worklen", 512, 8, 5, "edges"),
    ("wide: 512 subbands", 2048, 512, 24, "disp"),
    ("one subband, one DM", 300, 1, 1, "random"),
]


def make_offsets(kind, numdms, nsub, worklen, seed):
    if kind == "disp":
        return dispersion_offsets(numdms, nsub, worklen, 10.0, 0.5)
    rng = np.random.default_rng(seed)
    if kind == "random":
        return rng.integers(0, worklen + 1, (numdms, nsub)).astype(np.int32)
    off = np.zeros((numdms, nsub), dtype=np.int32)
    off[1] = worklen
    off[2, ::2] = worklen
    off[3] = rng.integers(0, worklen + 1, nsub)
    off[4] = worklen - 1
    return off


@pytest.mark.parametrize("name,worklen,nsub,numdms,kind", CASES, ids=[c[0] for c in CASES])
def test_dedisp_bit_exact(name, worklen, nsub, numdms, kind):
    cur, last = blocks(worklen, nsub, worklen + nsub)
    off = make_offsets(kind, numdms, nsub, worklen, 7)
    dd = jerk.Dedisperser(worklen, nsub, off)
    got = dd(torch.from_numpy(cur).cuda(), torch.from_numpy(last).cuda()).cpu().numpy()
    want = ob.dedisp_subbands(cur, last, off)
    print(name, "tiling (DMs per group, samples per tile):", dd.shape)
    dd.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_dedisp_scalar_path_on_unaligned_blocks():
    """Blocks that do not start on 16 bytes take the one-subband-at-a-time
    window loads; the result is the same."""
    worklen, nsub, numdms = 1024, 16, 12
    cur, last = blocks(worklen, nsub, 3)
    off = dispersion_offsets(numdms, nsub, worklen, 50.0, 1.0)
    dd = jerk.Dedisperser(worklen, nsub, off)
    big = torch.zeros(2 * worklen * nsub + 2, dtype=torch.float32, device="cuda")
    c = big[1: 1 + worklen * nsub].view(worklen, nsub)
    l = big[1 + worklen * nsub: 1 + 2 * worklen * nsub].view(worklen, nsub)
    c.copy_(torch.from_numpy(cur))
    l.copy_(torch.from_numpy(last))
    got = dd(c, l).cpu().numpy()
    dd.close()
    want = ob.dedisp_subbands(cur, last, off)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("bs,nsub", [(1, 64), (2, 64), (3, 13), (8, 128)])
def test_downsample_bit_exact(bs, nsub):
    worklen = 3000
    rng = np.random.default_rng(bs * 100 + nsub)
    x = (rng.standard_normal((worklen * bs, nsub)) * 30 + 7).astype(np.float32)
    got = jerk.downsample_subbands(torch.from_numpy(x).cuda(), bs).cpu().numpy()
    want = ob.downsample_subbands(x, bs)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_offsets_from_device_memory_and_matches():
    worklen, nsub, numdms = 2048, 32, 40
    off = dispersion_offsets(numdms, nsub, worklen, 0.0, 2.0)
    doff = torch.from_numpy(off).cuda()
    L = jerk.lib()
    p = C.c_void_p()
    jerk._check(L.jerk_dedisperser_create(C.byref(p), worklen, nsub, numdms,
                                          C.c_void_p(doff.data_ptr())))
    assert L.jerk_dedisperser_matches(p, worklen, nsub, numdms, off.ctypes.data) == 1
    off2 = off.copy()
    off2[3, 4] += 1
    assert L.jerk_dedisperser_matches(p, worklen, nsub, numdms, off2.ctypes.data) == 0
    assert L.jerk_dedisperser_matches(p, worklen, nsub + 1, numdms, off.ctypes.data) == 0
    cur, last = blocks(worklen, nsub, 11)
    out = torch.empty((numdms, worklen), dtype=torch.float32, device="cuda")
    dc, dl = torch.from_numpy(cur).cuda(), torch.from_numpy(last).cuda()
    jerk._check(L.jerk_dedisp_subbands(p, C.c_void_p(dc.data_ptr()), C.c_void_p(dl.data_ptr()),
                                       C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    L.jerk_dedisperser_destroy(p)
    want = ob.dedisp_subbands(cur, last, off)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_rejects_bad_offsets_and_shapes():
    with pytest.raises(jerk.JerkError) as ei:
        jerk.Dedisperser(100, 4, np.array([[0, 1, 2, 101]]))
    assert ei.value.code == jerk.JERK_EINVAL
    with pytest.raises(jerk.JerkError):
        jerk.Dedisperser(100, 4, np.array([[0, -1, 2, 3]]))
    with pytest.raises(jerk.JerkError):
        jerk.Dedisperser(100, 4, np.zeros((2, 3)))
    dd = jerk.Dedisperser(100, 4, np.zeros((2, 4)))
    x = torch.zeros((100, 4), device="cuda")
    with pytest.raises(jerk.JerkError):
        dd(x, torch.zeros((99, 4), device="cuda"))
    with pytest.raises(jerk.JerkError):
        dd(x.double(), x.double())
    dd.close()


def _load(path):
    lib = C.CDLL(path)
    lib.DownsampDataArray.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.DownsampDataArray.restype = None
    lib.getDedisp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                              C.c_void_p]
    lib.getDedisp.restype = None
    return lib


def test_dropin_symbols_equal_reference_gpu_kernels():
    """The drop-in's DownsampDataArray and getDedisp
    (prestozl_b200/csrc/compat/prepsubband_gpu.c) against the reference's own
    (src/prepsubband_kernels.cu), same device buffers, the way
    prepsubband_cu calls them: downsample the current block, then dedisperse
    it against the previous one, for two consecutive blocks."""
    import os

    if not (os.path.exists(ob.REF_DEDISP_GPU_LIB) and os.path.exists(ob.PREPSUBBAND_DROPIN_LIB)):
        pytest.skip("the reference build (oracle/_ref) has the reference's GPU kernels")
    ref, ours = _load(ob.REF_DEDISP_GPU_LIB), _load(ob.PREPSUBBAND_DROPIN_LIB)
    worklen, bs, nsub, numdms = 4096, 4, 64, 64
    off = dispersion_offsets(numdms, nsub, worklen, 20.0, 1.0, dt=4 * 64e-6)
    doff = torch.from_numpy(off).cuda()
    rng = np.random.default_rng(42)
    raw = [torch.from_numpy((rng.standard_normal((worklen * bs, nsub)) * 10 + 50)
                            .astype(np.float32)).cuda() for _ in range(3)]
    res = {}
    for name, lib in (("ref", ref), ("ours", ours)):
        ds = [torch.empty((worklen, nsub), device="cuda") for _ in range(3)]
        outs = []
        for i in range(3):
            lib.DownsampDataArray(ds[i].data_ptr(), raw[i].data_ptr(), worklen, bs, nsub)
            if i:
                out = torch.empty((numdms, worklen), device="cuda")
                lib.getDedisp(ds[i].data_ptr(), ds[i - 1].data_ptr(), out.data_ptr(), worklen,
                              nsub, numdms, doff.data_ptr())
                outs.append(out)
        torch.cuda.synchronize()
        res[name] = ([d.cpu().numpy() for d in ds], [o.cpu().numpy() for o in outs])
    for a, b in zip(res["ref"][0], res["ours"][0]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for a, b in zip(res["ref"][1], res["ours"][1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_dedispersed_trials_feed_the_search():
    """prepsubband_cu's GPU steps feeding the search with no file in between.
    Raw subband blocks carry a pulsar dispersed at DM 100 (1200-1600 MHz, 16
    subbands, 32 us samples).  Each block is downsampled 2x and dedispersed
    against the previous one into 9 DM trials (DM 0 to 200), block after
    block, into 2^20-sample series in HBM.  Each series then goes to the
    served loop as a time-series request.  The pulsar's best candidate sits
    at its frequency and is strongest in the DM-100 trial."""
    nsub, bs, worklen, nblocks = 16, 2, 1 << 16, 16
    dt_raw, dt = 32e-6, 64e-6
    dm_true, dms = 100.0, np.arange(9) * 25.0
    f_psr = 123.4
    freqs = 1200.0 + (np.arange(nsub) + 0.5) * 400.0 / nsub

    def delay(dm):  # seconds, relative to the top subband
        return 4.148808e3 * dm * (freqs ** -2 - freqs[-1] ** -2)

    off = np.rint(np.array([delay(dm) for dm in dms]) / dt).astype(np.int32)
    dd = jerk.Dedisperser(worklen, nsub, off)
    rng = np.random.default_rng(2024)
    d_true = delay(dm_true)
    raw_len = worklen * bs
    prev = None
    series = torch.empty((len(dms), nblocks * worklen), dtype=torch.float32, device="cuda")
    for k in range(nblocks + 1):
        t = (k * raw_len + np.arange(raw_len))[:, None] * dt_raw - d_true[None, :]
        sig = sum(a * np.cos(2 * np.pi * h * f_psr * t) for h, a in ((1, 1.0), (2, 0.5), (3, 0.3)))
        raw = (rng.standard_normal((raw_len, nsub)) + 0.01 * sig).astype(np.float32)
        ds = jerk.downsample_subbands(torch.from_numpy(raw).cuda(), bs)
        if prev is not None:
            series[:, (k - 1) * worklen: k * worklen] = dd(ds, prev)
        prev = ds
    torch.cuda.synchronize()
    dd.close()
    N = nblocks * worklen
    srv = jerk.JerkServer(max_active=3, batch=16)
    for i in range(len(dms)):
        srv.submit(series[i].contiguous(), N, dt, 20, 60, 8, 2.0, tag=i, timeseries=True)
    r0 = f_psr * N * dt
    best = {}
    for _ in range(len(dms)):
        tag, cands, _ = srv.poll(120000)
        near = cands[np.abs(cands["r"] - r0) < 2.0] if len(cands) else cands
        best[tag] = float(near["sigma"].max()) if len(near) else 0.0
    st = srv.stats()
    srv.close()
    print("best sigma at the pulsar by DM trial:", {float(dms[k]): round(v, 1)
                                                     for k, v in sorted(best.items())})
    assert st["failed"] == 0
    peak = int(np.argmax([best[i] for i in range(len(dms))]))
    assert dms[peak] == dm_true
    assert best[peak] > 10.0 and best[peak] > 2 * max(best[0], best[len(dms) - 1])


def test_dedisp_matches_reference_golden():
    """The GPU against the committed fixture of the reference's float_dedisp
    (tests/golden/dedisp_small.npz): 96 samples x 12 subbands, 7 DMs with
    offsets 0 and 96 among them."""
    import os

    g = np.load(os.path.join(H.GOLDEN, "dedisp_small.npz"))
    worklen, nsub = g["cur"].shape
    dd = jerk.Dedisperser(worklen, nsub, g["offsets"])
    got = dd(torch.from_numpy(g["cur"]).cuda(), torch.from_numpy(g["last"]).cuda()).cpu().numpy()
    dd.close()
    assert np.array_equal(got.view(np.uint32), g["out"].view(np.uint32))
