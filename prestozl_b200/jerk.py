"""Python mirror of libjerk's C ABI (``include/jerk.h``), through ctypes.

This is the host-side interface the tests and the benchmark use; C callers
link ``prestozl_b200/lib/libjerk.so`` directly.  There is no fallback: if the
CUDA library is missing, every entry point raises.

Names follow the reference (``accelobs`` -> ``Obs``, ``subharminfo`` ->
``Subharm``, ``accelcand`` -> ``Cand``; ``include/accel.h`` in PrestoZL).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("JERK_LIB", os.path.join(HERE, "lib", "libjerk.so"))

JERK_OK = 0
JERK_OVERFLOW = 1
JERK_TIMEOUT = 2
JERK_EINVAL = -1
JERK_ECUDA = -2
JERK_ENOMEM = -3
JERK_EUNSUPPORTED = -4

MAX_STAGES = 6


class JerkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libjerk error {code}: {msg}")
        self.code = code


class Obs(C.Structure):
    """jerk_obs: the search geometry (accelobs fields the loop reads)."""
    _fields_ = [
        ("numbins", C.c_longlong), ("lobin", C.c_longlong), ("highestbin", C.c_longlong),
        ("rlo", C.c_double), ("zlo", C.c_double), ("wlo", C.c_double),
        ("corr_uselen", C.c_int), ("numz", C.c_int), ("numw", C.c_int),
        ("numharmstages", C.c_int), ("norm_type", C.c_int), ("nph", C.c_float),
        ("powcut", C.c_float * MAX_STAGES), ("numindep", C.c_longlong * MAX_STAGES),
    ]


class Subharm(C.Structure):
    _fields_ = [("numharm", C.c_int), ("harmnum", C.c_int), ("zmax", C.c_int),
                ("wmax", C.c_int), ("numz", C.c_int), ("numw", C.c_int),
                ("fftlen", C.c_int), ("halfwidth", C.c_int), ("kernels", C.c_void_p)]


class Cand(C.Structure):
    _fields_ = [("power", C.c_float), ("sigma", C.c_float), ("numharm", C.c_int),
                ("r", C.c_double), ("z", C.c_double), ("w", C.c_double)]


class Config(C.Structure):
    _fields_ = [("batch_rsteps", C.c_int), ("max_hits", C.c_longlong),
                ("stream", C.c_void_p), ("device_bank", C.c_void_p), ("harm_mode", C.c_int),
                ("use_graph", C.c_int)]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("ms", C.c_double),
                ("bytes", C.c_double), ("flops", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_longlong), ("max_active", C.c_int),
                ("batch_rsteps", C.c_int), ("device", C.c_int), ("batches_ahead", C.c_int),
                ("queue_timeout_s", C.c_double), ("harm_mode", C.c_int)]


class Request(C.Structure):
    _fields_ = [("spectrum", C.c_void_p), ("on_device", C.c_int), ("numbins", C.c_longlong),
                ("N", C.c_longlong), ("dt", C.c_double), ("zmax", C.c_int), ("wmax", C.c_int),
                ("wmax_given", C.c_int), ("numharm", C.c_int), ("sigma", C.c_float),
                ("flo", C.c_double), ("fhi", C.c_double), ("tag", C.c_longlong),
                ("timeseries", C.c_int), ("bird_lobins", C.c_void_p), ("bird_hibins", C.c_void_p),
                ("numbirds", C.c_int)]


class Result(C.Structure):
    _fields_ = [("tag", C.c_longlong), ("status", C.c_int), ("cands", C.POINTER(Cand)),
                ("ncands", C.c_longlong), ("t_submit", C.c_double), ("t_start", C.c_double),
                ("t_done", C.c_double)]


class Hits(C.Structure):
    _fields_ = [("count", C.c_longlong), ("keys", C.POINTER(C.c_ulonglong)),
                ("powers", C.POINTER(C.c_float))]


CAND_DTYPE = np.dtype([("power", np.float32), ("sigma", np.float32), ("numharm", np.int32),
                       ("r", np.float64), ("z", np.float64), ("w", np.float64)], align=True)
assert CAND_DTYPE.itemsize == C.sizeof(Cand)

_lib = None

EXPORTS = [
    "jerk_obs_from_params", "jerk_subharm_count", "jerk_subharm_sizes", "jerk_plan_create",
    "jerk_plan_destroy", "jerk_search", "jerk_num_rsteps", "jerk_debug_volume",
    "jerk_candidate_sigma", "jerk_power_for_sigma", "jerk_insert_hits", "jerk_free",
    "jerk_last_error", "jerk_bank_elements", "jerk_bank_generate", "jerk_device_alloc",
    "jerk_device_free", "jerk_copy_to_host", "jerk_plan_set_profiling", "jerk_plan_reset_stats",
    "jerk_plan_kernel_stats", "jerk_plan_transfer_stats", "jerk_volume_static",
    "jerk_search_async", "jerk_search_advance", "jerk_search_ready", "jerk_search_collect", "jerk_plan_device_bytes",
    "jerk_server_create", "jerk_server_submit", "jerk_server_poll", "jerk_server_stats",
    "jerk_server_destroy", "jerk_realfft_scratch_bytes", "jerk_realfft",
    "jerk_deredden_scratch_bytes", "jerk_deredden", "jerk_spectrum_scratch_bytes",
    "jerk_spectrum_from_timeseries", "jerk_polisher_create", "jerk_polisher_destroy",
    "jerk_polish_rzw", "jerk_zap_birdies", "jerk_local_power", "jerk_derivs",
    "jerk_optimize_cand", "jerk_downsample_subbands", "jerk_dedisperser_create",
    "jerk_dedisperser_destroy", "jerk_dedisperser_shape", "jerk_dedisperser_matches",
    "jerk_dedisp_subbands", "jerk_dedisp_plan", "jerk_debug_wait_probe", "jerk_merge_hits",
    "jerk_search_begin", "jerk_group_advance", "jerk_search_group", "jerk_server_transfer_stats",
]


def lib() -> C.CDLL:
    """Load libjerk.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise JerkError(JERK_ECUDA, f"{LIB_PATH} is missing; run prestozl_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    L.jerk_last_error.restype = C.c_char_p
    L.jerk_obs_from_params.argtypes = [C.c_longlong, C.c_longlong, C.c_double, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_float, C.c_double, C.c_double,
                                       C.POINTER(Obs), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.jerk_subharm_count.argtypes = [C.c_int]
    L.jerk_subharm_sizes.argtypes = [C.POINTER(Obs), C.c_int, C.c_int, C.POINTER(Subharm)]
    L.jerk_plan_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Obs), C.POINTER(Subharm),
                                   C.c_int, C.POINTER(Config)]
    L.jerk_plan_destroy.argtypes = [C.c_void_p]
    L.jerk_plan_destroy.restype = None
    L.jerk_search.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_longlong,
                              C.POINTER(C.POINTER(Cand)), C.POINTER(C.c_longlong),
                              C.POINTER(Hits)]
    L.jerk_num_rsteps.argtypes = [C.c_void_p]
    L.jerk_num_rsteps.restype = C.c_longlong
    L.jerk_debug_volume.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_int,
                                    C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    L.jerk_debug_wait_probe.argtypes = [C.c_void_p, C.c_int]
    L.jerk_search_begin.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_longlong]
    L.jerk_group_advance.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int]
    L.jerk_search_group.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_int), C.c_int,
                                    C.POINTER(C.POINTER(Cand)), C.POINTER(C.c_longlong)]
    L.jerk_merge_hits.argtypes = [C.POINTER(Obs), C.POINTER(Subharm), C.c_void_p, C.c_void_p,
                                  C.c_longlong, C.POINTER(C.POINTER(Cand)),
                                  C.POINTER(C.c_longlong)]
    L.jerk_candidate_sigma.restype = C.c_double
    L.jerk_candidate_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
    L.jerk_power_for_sigma.restype = C.c_double
    L.jerk_power_for_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
    L.jerk_insert_hits.restype = C.c_longlong
    L.jerk_insert_hits.argtypes = [C.POINTER(Cand), C.c_longlong, C.POINTER(C.POINTER(Cand))]
    L.jerk_free.argtypes = [C.c_void_p]
    L.jerk_free.restype = None
    L.jerk_bank_elements.restype = C.c_longlong
    L.jerk_bank_elements.argtypes = [C.POINTER(Subharm), C.c_int]
    L.jerk_bank_generate.argtypes = [C.POINTER(Subharm), C.c_int, C.c_void_p, C.c_void_p]
    L.jerk_device_alloc.argtypes = [C.c_longlong, C.POINTER(C.c_void_p)]
    L.jerk_device_free.argtypes = [C.c_void_p]
    L.jerk_device_free.restype = None
    L.jerk_copy_to_host.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
    L.jerk_plan_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.jerk_plan_reset_stats.argtypes = [C.c_void_p]
    L.jerk_plan_reset_stats.restype = None
    L.jerk_plan_kernel_stats.argtypes = [C.c_void_p, C.c_int, C.POINTER(KernelStat)]
    L.jerk_plan_transfer_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong),
                                           C.POINTER(C.c_longlong)]
    L.jerk_plan_transfer_stats.restype = None
    L.jerk_search_async.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_longlong]
    L.jerk_search_ready.argtypes = [C.c_void_p]
    L.jerk_search_advance.argtypes = [C.c_void_p, C.c_int]
    L.jerk_search_collect.argtypes = [C.c_void_p, C.POINTER(C.POINTER(Cand)),
                                      C.POINTER(C.c_longlong), C.POINTER(Hits)]
    L.jerk_plan_device_bytes.restype = C.c_longlong
    L.jerk_plan_device_bytes.argtypes = [C.c_void_p]
    L.jerk_server_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(ServerConfig)]
    L.jerk_server_submit.argtypes = [C.c_void_p, C.POINTER(Request)]
    L.jerk_server_poll.argtypes = [C.c_void_p, C.POINTER(Result), C.c_int]
    L.jerk_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    L.jerk_server_stats.restype = None
    L.jerk_server_transfer_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong),
                                             C.POINTER(C.c_longlong)]
    L.jerk_server_transfer_stats.restype = None
    L.jerk_server_destroy.argtypes = [C.c_void_p]
    L.jerk_server_destroy.restype = None
    L.jerk_volume_static.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.POINTER(Subharm),
                                     C.c_void_p, C.c_double, C.c_int, C.c_float, C.c_void_p,
                                     C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.c_void_p]
    for f in ("jerk_realfft_scratch_bytes", "jerk_deredden_scratch_bytes",
              "jerk_spectrum_scratch_bytes"):
        getattr(L, f).restype = C.c_longlong
        getattr(L, f).argtypes = [C.c_longlong]
    for f in ("jerk_realfft", "jerk_spectrum_from_timeseries"):
        getattr(L, f).argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p, C.c_longlong,
                                  C.c_void_p]
    L.jerk_deredden.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p]
    L.jerk_local_power.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]
    L.jerk_derivs.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jerk_optimize_cand.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.jerk_zap_birdies.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_void_p]
    L.jerk_downsample_subbands.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p]
    L.jerk_dedisperser_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int,
                                          C.c_void_p]
    L.jerk_dedisperser_destroy.argtypes = [C.c_void_p]
    L.jerk_dedisperser_destroy.restype = None
    L.jerk_dedisperser_shape.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.jerk_dedisperser_matches.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    L.jerk_dedisp_subbands.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    L.jerk_dedisp_plan.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    L.jerk_polisher_create.argtypes = [C.POINTER(C.c_void_p), C.c_void_p]
    L.jerk_polisher_destroy.argtypes = [C.c_void_p]
    L.jerk_polisher_destroy.restype = None
    L.jerk_polish_rzw.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_double,
                                  C.c_double, C.c_double, C.c_void_p, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_float)]
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != JERK_OK:
        raise JerkError(rc, lib().jerk_last_error().decode())


def obs_from_params(numbins: int, N: int, dt: float, zmax: int, wmax: int, numharm: int,
                    sigma: float, flo: float = 1.0, fhi: float = 10000.0,
                    wmax_given: bool = True) -> Tuple[Obs, int, int]:
    """create_accelobs sizing with accelsearch's defaults (-flo 1 -fhi 10000)."""
    o = Obs()
    fftlen, mk = C.c_int(0), C.c_int(0)
    _check(lib().jerk_obs_from_params(numbins, N, dt, zmax, wmax, int(wmax_given), numharm,
                                      sigma, flo, fhi, C.byref(o), C.byref(fftlen), C.byref(mk)))
    return o, fftlen.value, mk.value


def subharm_sizes(obs: Obs, fftlen: int) -> List[dict]:
    out = []
    for i in range(lib().jerk_subharm_count(obs.numharmstages)):
        s = Subharm()
        _check(lib().jerk_subharm_sizes(C.byref(obs), fftlen, i, C.byref(s)))
        out.append({k: getattr(s, k) for k, _ in Subharm._fields_ if k != "kernels"})
    return out


def candidate_sigma(power: float, numsum: int, numtrials: float) -> float:
    return lib().jerk_candidate_sigma(power, numsum, numtrials)


def power_for_sigma(sigma: float, numsum: int, numtrials: float) -> float:
    return lib().jerk_power_for_sigma(sigma, numsum, numtrials)


def insert_hits(hits: np.ndarray) -> np.ndarray:
    hits = np.ascontiguousarray(hits, dtype=CAND_DTYPE)
    out = C.POINTER(Cand)()
    n = lib().jerk_insert_hits(hits.ctypes.data_as(C.POINTER(Cand)), len(hits), C.byref(out))
    arr = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_byte)), shape=(n * CAND_DTYPE.itemsize,))
    res = np.frombuffer(arr.tobytes(), dtype=CAND_DTYPE).copy()
    lib().jerk_free(out)
    return res


def merge_hits(obs: Obs, fundamental: dict, keys, powers) -> np.ndarray:
    """Candidates of one spectrum from the raw hits of searches of disjoint
    rstep ranges (any order): jerk_merge_hits.  Host only."""
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    pw = np.ascontiguousarray(powers, dtype=np.float32)
    if len(k) != len(pw):
        raise JerkError(JERK_EINVAL, "merge_hits: keys and powers differ in length")
    f = (Subharm * 1)(fundamental) if isinstance(fundamental, Subharm) else \
        _subharm_array([fundamental])
    out = C.POINTER(Cand)()
    n = C.c_longlong(0)
    _check(lib().jerk_merge_hits(C.byref(obs), f, k.ctypes.data, pw.ctypes.data, len(k),
                                 C.byref(out), C.byref(n)))
    nb = n.value * CAND_DTYPE.itemsize
    cands = np.frombuffer(C.string_at(out, nb), dtype=CAND_DTYPE).copy() if nb else \
        np.zeros(0, dtype=CAND_DTYPE)
    lib().jerk_free(out)
    return cands


def _subharm_array(subs: Sequence[dict]):
    arr = (Subharm * len(subs))()
    for i, s in enumerate(subs):
        arr[i] = Subharm(s["numharm"], s["harmnum"], s.get("zmax", 0), s.get("wmax", 0),
                         s["numz"], s["numw"], s["fftlen"], s["halfwidth"], None)
    return arr


class DeviceBank:
    """A kernel bank generated on the device (jerk_bank_generate); pass it to
    JerkPlan(device_bank=bank.ptr) to share it between plans."""

    def __init__(self, subs: Sequence[dict], stream: int = 0):
        arr = _subharm_array(subs)
        self.elements = lib().jerk_bank_elements(arr, len(subs))
        self.ptr = C.c_void_p()
        _check(lib().jerk_device_alloc(self.elements * 8, C.byref(self.ptr)))
        rc = lib().jerk_bank_generate(arr, len(subs), self.ptr, stream or None)
        if rc != JERK_OK:
            self.close()
            _check(rc)

    def close(self) -> None:
        if self.ptr:
            lib().jerk_device_free(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rows(self, subs: Sequence[dict], sub: int, rows: Sequence[int]) -> np.ndarray:
        """Copy kernel rows (flattened w * numz + z) of one subharmonic to the host."""
        off = sum(s["numw"] * s["numz"] * s["fftlen"] for s in subs[:sub])
        n = subs[sub]["fftlen"]
        out = np.zeros((len(rows), n), dtype=np.complex64)
        for i, r in enumerate(rows):
            _check(lib().jerk_copy_to_host(out[i].ctypes.data, self.ptr.value + 8 * (off + int(r) * n),
                                           8 * n))
        return out


def volume_static(spectrum_dev: int, numbins: int, lobin: int, sub: dict, kernels_dev: int,
                  fullrlo: float, corr_uselen: int, nph: float, volume_dev: int,
                  stream: int = 0) -> Tuple[int, int]:
    """One subharmonic's ffdot volume for one rstep through the entry point
    that allocates nothing (jerk_volume_static); all pointers are device
    addresses the caller owns.  Returns (numrs, rlo); asynchronous on stream."""
    s = Subharm(sub["numharm"], sub["harmnum"], sub.get("zmax", 0), sub.get("wmax", 0),
                sub["numz"], sub["numw"], sub["fftlen"], sub["halfwidth"], None)
    numrs, rlo = C.c_int(0), C.c_longlong(0)
    rc = lib().jerk_volume_static(spectrum_dev, numbins, lobin, C.byref(s), kernels_dev, fullrlo,
                                  corr_uselen, nph, volume_dev, C.byref(numrs), C.byref(rlo),
                                  stream or None)
    if rc != JERK_OK:
        raise JerkError(rc, "jerk_volume_static failed (see stderr)")
    return numrs.value, rlo.value


def _input_call(fn: str, size_fn: str, x, n: int, out):
    import torch

    if not (getattr(x, "is_cuda", False) and x.is_contiguous()):
        raise JerkError(JERK_EINVAL, f"{fn}: expects a contiguous CUDA tensor")
    nbytes = getattr(lib(), size_fn)(n)
    if nbytes <= 0:
        raise JerkError(JERK_EUNSUPPORTED, f"{fn}: size {n} not supported")
    scratch = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    if fn == "jerk_deredden":
        _check(lib().jerk_deredden(x.data_ptr(), n, scratch.data_ptr(), nbytes, stream or None))
    else:
        _check(getattr(lib(), fn)(x.data_ptr(), n, out.data_ptr(), scratch.data_ptr(), nbytes,
                                  stream or None))
    return out if out is not None else x


def _series_out(ts, out):
    import torch

    if ts.dtype != torch.float32 or ts.dim() != 1:
        raise JerkError(JERK_EINVAL, "the time series must be a 1-D float32 tensor")
    if out is None:
        out = torch.empty(ts.numel() // 2, dtype=torch.complex64, device=ts.device)
    return out


def realfft(ts, out=None):
    """Forward real FFT of a float32 CUDA time series in PRESTO's packing
    (realfft(data, n, -1), src/fastffts.c:163-235): n/2 complex64 values,
    value 0 = (DC, Nyquist).  ``out`` may be ``ts`` viewed as complex64
    (in place).  Asynchronous on torch's current stream."""
    out = _series_out(ts, out)
    return _input_call("jerk_realfft", "jerk_realfft_scratch_bytes", ts, ts.numel(), out)


def deredden(spec):
    """The reference's red-noise removal (src/accel_utils.c:1557-1633), in
    place on a complex64 CUDA spectrum; bit-exact with the reference."""
    return _input_call("jerk_deredden", "jerk_deredden_scratch_bytes", spec, spec.numel(), None)


def spectrum_from_timeseries(ts, out=None):
    """realfft, deredden and bin 0 set to (1, 1): the spectrum the reference
    searches for a .dat input without -photon (src/accel_utils.c:1747-1753,
    1829-1834)."""
    out = _series_out(ts, out)
    return _input_call("jerk_spectrum_from_timeseries", "jerk_spectrum_scratch_bytes", ts,
                       ts.numel(), out)


RDERIVS_DTYPE = np.dtype([("pow", np.float64), ("phs", np.float64), ("dpow", np.float64),
                          ("dphs", np.float64), ("d2pow", np.float64), ("d2phs", np.float64),
                          ("locpow", np.float64)])


class Polisher:
    """Candidate polishing on the GPU (jerk_polish_rzw): the volume search of
    the reference's harmonic polishing (src/maximize_rzw.c:84-190)."""

    def __init__(self):
        self.ptr = C.c_void_p()
        _check(lib().jerk_polisher_create(C.byref(self.ptr), None))

    @staticmethod
    def _spectrum(spectrum):
        """(pointer, numdata, keepalive): a numpy spectrum is read on the host;
        a complex64 CUDA tensor on the GPU, once the work that wrote it on
        torch's current stream has finished (the polisher has its own
        stream)."""
        if getattr(spectrum, "is_cuda", False):
            import torch

            if spectrum.dtype != torch.complex64 or not spectrum.is_contiguous():
                raise JerkError(JERK_EINVAL, "polisher: expects a contiguous complex64 tensor")
            torch.cuda.current_stream(spectrum.device).synchronize()
            return C.c_void_p(spectrum.data_ptr()), spectrum.numel(), spectrum
        a = np.ascontiguousarray(spectrum, dtype=np.complex64)
        return C.c_void_p(a.ctypes.data), len(a), a

    def polish(self, spectrum: np.ndarray, numharm: int, r: float, z: float, w: float,
               locpow) -> Tuple[float, float, float, float]:
        """(r, z, w, summed power) polished; r relative to the spectrum's bin
        0; locpow[i] the local power of harmonic numharm - i."""
        sp, n, _keep = self._spectrum(spectrum)
        lp = np.ascontiguousarray(locpow, dtype=np.float32)
        ro, zo, wo, mp = C.c_double(), C.c_double(), C.c_double(), C.c_float()
        _check(lib().jerk_polish_rzw(self.ptr, sp, n, numharm, r, z, w,
                                     lp.ctypes.data, C.byref(ro), C.byref(zo), C.byref(wo),
                                     C.byref(mp)))
        return ro.value, zo.value, wo.value, mp.value

    def optimize(self, spectrum: np.ndarray, numharm: int, r: float, z: float, w: float):
        """The reference's default candidate optimisation wholly on the GPU
        (jerk_optimize_cand): ((r, z, w) polished, r relative to the
        spectrum's bin 0; the per-harmonic derivatives, RDERIVS_DTYPE; the
        local powers the volume search used)."""
        sp, n, _keep = self._spectrum(spectrum)
        rzw = np.zeros(3)
        d = np.zeros(numharm, dtype=RDERIVS_DTYPE)
        lp = np.zeros(numharm, dtype=np.float32)
        _check(lib().jerk_optimize_cand(self.ptr, sp, n, numharm, r, z, w,
                                        rzw.ctypes.data, d.ctypes.data, lp.ctypes.data))
        return tuple(float(v) for v in rzw), d, lp

    def local_power(self, spectrum: np.ndarray, r, z, w) -> np.ndarray:
        """get_localpower3d at the given points (jerk_local_power)."""
        sp, n, _keep = self._spectrum(spectrum)
        r, z, w = (np.ascontiguousarray(v, dtype=np.float64) for v in (r, z, w))
        out = np.zeros(len(r))
        _check(lib().jerk_local_power(self.ptr, sp, n, len(r), r.ctypes.data,
                                      z.ctypes.data, w.ctypes.data, out.ctypes.data))
        return out

    def close(self):
        if self.ptr:
            lib().jerk_polisher_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def zap_birdies(spec, N: int, lobins, hibins):
    """The reference's birdie zapping of an in-memory spectrum
    (src/accelsearch_lib.c:393-418, zapbirds src/zapping.c:29-81), in place on
    a complex64 CUDA tensor; lobins/hibins in Fourier bins, in list order.
    Bit-exact with the reference."""
    import torch

    if not (getattr(spec, "is_cuda", False) and spec.is_contiguous()):
        raise JerkError(JERK_EINVAL, "zap_birdies: expects a contiguous CUDA tensor")
    lo = np.ascontiguousarray(lobins, dtype=np.float64)
    hi = np.ascontiguousarray(hibins, dtype=np.float64)
    stream = torch.cuda.current_stream(spec.device).cuda_stream
    _check(lib().jerk_zap_birdies(spec.data_ptr(), spec.numel(), N, lo.ctypes.data,
                                  hi.ctypes.data, len(lo), stream or None))
    return spec


def _stream_of(t):
    import torch

    return torch.cuda.current_stream(t.device).cuda_stream or None


def _check_subbands(t, what: str):
    import torch

    if not (getattr(t, "is_cuda", False) and t.dtype == torch.float32 and t.is_contiguous()
            and t.dim() == 2):
        raise JerkError(JERK_EINVAL, f"{what}: expects a contiguous 2-D float32 CUDA tensor")


def downsample_subbands(data, bs: int, out=None):
    """prepsubband_cu's DownsampDataArray (jerk_downsample_subbands): data
    [worklen * bs, nsub] float32 on the GPU, time-major -> [worklen, nsub],
    each the mean of bs consecutive samples; on torch's current stream."""
    import torch

    _check_subbands(data, "downsample_subbands")
    worklen, nsub = data.shape[0] // bs, data.shape[1]
    if out is None:
        out = torch.empty((worklen, nsub), dtype=torch.float32, device=data.device)
    _check_subbands(out, "downsample_subbands")
    if tuple(out.shape) != (worklen, nsub):
        raise JerkError(JERK_EINVAL, "downsample_subbands: out must be [worklen, nsub]")
    _check(lib().jerk_downsample_subbands(C.c_void_p(out.data_ptr()),
                                          C.c_void_p(data.data_ptr()), worklen, bs, nsub,
                                          C.c_void_p(_stream_of(data))))
    return out


def dedisp_plan(worklen: int, nsub: int, offsets) -> Tuple[int, int, int]:
    """The tiling a Dedisperser would choose for these offsets (host only,
    jerk_dedisp_plan): (DMs per CTA group, samples per tile, shared-memory
    bytes per CTA).  Raises JerkError on offsets outside [0, worklen]."""
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    if off.ndim != 2 or off.shape[1] != nsub:
        raise JerkError(JERK_EINVAL, "dedisp_plan: offsets must be [numdms, nsub]")
    g, t, b = C.c_int(), C.c_int(), C.c_longlong()
    _check(lib().jerk_dedisp_plan(worklen, nsub, off.shape[0], off.ctypes.data_as(C.c_void_p),
                                  C.byref(g), C.byref(t), C.byref(b)))
    return g.value, t.value, b.value


class Dedisperser:
    """prepsubband_cu's getDedisp (jerk_dedisp_subbands) for one offsets
    table: offsets [numdms, nsub] (in samples, each in [0, worklen])."""

    def __init__(self, worklen: int, nsub: int, offsets):
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        if off.ndim != 2 or off.shape[1] != nsub:
            raise JerkError(JERK_EINVAL, "Dedisperser: offsets must be [numdms, nsub]")
        self.worklen, self.nsub, self.numdms = worklen, nsub, off.shape[0]
        self.ptr = C.c_void_p()
        _check(lib().jerk_dedisperser_create(C.byref(self.ptr), worklen, nsub, self.numdms,
                                             off.ctypes.data_as(C.c_void_p)))

    @property
    def shape(self) -> Tuple[int, int]:
        """(DMs per CTA group, samples per tile) that the plan chose."""
        g, t = C.c_int(), C.c_int()
        _check(lib().jerk_dedisperser_shape(self.ptr, C.byref(g), C.byref(t)))
        return g.value, t.value

    def __call__(self, cur, last, out=None):
        """[numdms, worklen] series from the current and the previous block
        ([worklen, nsub] each); on torch's current stream."""
        import torch

        for t in (cur, last):
            _check_subbands(t, "Dedisperser")
            if tuple(t.shape) != (self.worklen, self.nsub):
                raise JerkError(JERK_EINVAL, "Dedisperser: blocks must be [worklen, nsub]")
        if out is None:
            out = torch.empty((self.numdms, self.worklen), dtype=torch.float32, device=cur.device)
        _check_subbands(out, "Dedisperser")
        if tuple(out.shape) != (self.numdms, self.worklen):
            raise JerkError(JERK_EINVAL, "Dedisperser: out must be [numdms, worklen]")
        _check(lib().jerk_dedisp_subbands(self.ptr, C.c_void_p(cur.data_ptr()),
                                          C.c_void_p(last.data_ptr()),
                                          C.c_void_p(out.data_ptr()),
                                          C.c_void_p(_stream_of(cur))))
        return out

    def close(self):
        if self.ptr:
            lib().jerk_dedisperser_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _spectrum_arg(spectrum):
    """(pointer, on_device, keepalive) for a numpy array or a CUDA tensor."""
    if isinstance(spectrum, np.ndarray):
        a = np.ascontiguousarray(spectrum, dtype=np.complex64)
        return C.c_void_p(a.ctypes.data), 0, a
    # a torch tensor on the GPU (complex64 or float32 pairs)
    if getattr(spectrum, "is_cuda", False):
        return C.c_void_p(spectrum.data_ptr()), 1, spectrum
    a = np.ascontiguousarray(np.asarray(spectrum), dtype=np.complex64)
    return C.c_void_p(a.ctypes.data), 0, a


class JerkPlan:
    """A search plan on the current CUDA device (jerk_plan_create)."""

    def __init__(self, obs: Obs, subs: Sequence[dict], batch: int = 8, max_hits: int = 0,
                 stream: int = 0, device_bank: int = 0, harm_mode: int = 0,
                 use_graph: bool = False):
        self.obs = obs
        self._kerns = []
        arr = (Subharm * len(subs))()
        for i, s in enumerate(subs):
            k = s.get("kern")
            kp = None
            if k is not None:
                k = np.ascontiguousarray(k, dtype=np.complex64)
                self._kerns.append(k)
                kp = k.ctypes.data
            arr[i] = Subharm(s["numharm"], s["harmnum"], s.get("zmax", 0), s.get("wmax", 0),
                             s["numz"], s["numw"], s["fftlen"], s["halfwidth"], kp)
        self.subs = arr
        cfg = Config(batch, max_hits, stream or None, device_bank or None, harm_mode,
                     int(bool(use_graph)))
        self._p = C.c_void_p()
        _check(lib().jerk_plan_create(C.byref(self._p), C.byref(obs), arr, len(subs),
                                      C.byref(cfg)))
        self._kerns = []  # the bank is on the device now

    @property
    def num_rsteps(self) -> int:
        return lib().jerk_num_rsteps(self._p)

    def close(self) -> None:
        if self._p:
            lib().jerk_plan_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, spectrum, first_rstep: int = 0, num_rsteps: int = 0,
               want_hits: bool = False):
        """Candidates (CAND_DTYPE, list order) and optionally raw hits
        (keys u64, powers f32) in the reference's insertion order."""
        ptr, dev, keep = _spectrum_arg(spectrum)
        out = C.POINTER(Cand)()
        n = C.c_longlong(0)
        hits = Hits()
        _check(lib().jerk_search(self._p, ptr, dev, first_rstep, num_rsteps, C.byref(out),
                                 C.byref(n), C.byref(hits) if want_hits else None))
        nb = n.value * CAND_DTYPE.itemsize
        cands = np.frombuffer(C.string_at(out, nb), dtype=CAND_DTYPE).copy() if nb else \
            np.zeros(0, dtype=CAND_DTYPE)
        lib().jerk_free(out)
        if not want_hits:
            return cands
        k = np.ctypeslib.as_array(hits.keys, shape=(max(hits.count, 1),))[: hits.count].copy()
        p = np.ctypeslib.as_array(hits.powers, shape=(max(hits.count, 1),))[: hits.count].copy()
        lib().jerk_free(C.cast(hits.keys, C.c_void_p))
        lib().jerk_free(C.cast(hits.powers, C.c_void_p))
        return cands, k, p

    def begin(self, spectrum, first_rstep: int = 0, num_rsteps: int = 0) -> None:
        """Start a pass whose batches come from group_advance (jerk_search_begin).
        The spectrum must stay alive until collect()."""
        ptr, dev, keep = _spectrum_arg(spectrum)
        _check(lib().jerk_search_begin(self._p, ptr, dev, first_rstep, num_rsteps))
        self._inflight_keep = keep

    def collect(self, want_hits: bool = False):
        """Finish the pass in flight (jerk_search_collect): candidates, and
        optionally the raw hits, as search() returns them."""
        out = C.POINTER(Cand)()
        n = C.c_longlong(0)
        hits = Hits()
        try:
            _check(lib().jerk_search_collect(self._p, C.byref(out), C.byref(n),
                                             C.byref(hits) if want_hits else None))
        finally:
            self._inflight_keep = None
        nb = n.value * CAND_DTYPE.itemsize
        cands = np.frombuffer(C.string_at(out, nb), dtype=CAND_DTYPE).copy() if nb else \
            np.zeros(0, dtype=CAND_DTYPE)
        lib().jerk_free(out)
        if not want_hits:
            return cands
        k = np.ctypeslib.as_array(hits.keys, shape=(max(hits.count, 1),))[: hits.count].copy()
        p = np.ctypeslib.as_array(hits.powers, shape=(max(hits.count, 1),))[: hits.count].copy()
        lib().jerk_free(C.cast(hits.keys, C.c_void_p))
        lib().jerk_free(C.cast(hits.powers, C.c_void_p))
        return cands, k, p

    def set_profiling(self, on: bool) -> None:
        _check(lib().jerk_plan_set_profiling(self._p, int(on)))

    def reset_stats(self) -> None:
        lib().jerk_plan_reset_stats(self._p)

    def kernel_stats(self) -> dict:
        n = lib().jerk_plan_kernel_stats(self._p, 0, None)
        arr = (KernelStat * max(n, 1))()
        lib().jerk_plan_kernel_stats(self._p, n, arr)
        return {a.name.decode(): {"launches": a.launches, "ms": a.ms, "bytes": a.bytes,
                                  "flops": a.flops} for a in arr[:n]}

    def transfer_stats(self) -> Tuple[int, int]:
        h, d = C.c_longlong(0), C.c_longlong(0)
        lib().jerk_plan_transfer_stats(self._p, C.byref(h), C.byref(d))
        return h.value, d.value

    def set_wait_probe(self, on: bool) -> None:
        """Test hook: later passes also run one bounded wait that must give
        up, and fail with JERK_ECUDA (jerk_debug_wait_probe)."""
        _check(lib().jerk_debug_wait_probe(self._p, int(bool(on))))

    def volume(self, spectrum, rstep: int, sub: int):
        """ffdot volume [numw][numz][numrs] of one (rstep, subharmonic)."""
        ptr, dev, keep = _spectrum_arg(spectrum)
        s = self.subs[sub]
        fftlen = s.fftlen
        out = np.zeros(s.numw * s.numz * fftlen, dtype=np.float32)
        numrs, rlo = C.c_int(0), C.c_longlong(0)
        _check(lib().jerk_debug_volume(self._p, ptr, dev, rstep, sub, out.ctypes.data,
                                       C.byref(numrs), C.byref(rlo)))
        n = s.numw * s.numz * numrs.value
        return out[:n].reshape(s.numw, s.numz, numrs.value), rlo.value

    def decode(self, keys: np.ndarray):
        """(rstep, stage, w index, z index, r index) of encoded hit keys."""
        k = keys.astype(np.uint64)
        numrs, numz, numw = self.obs.corr_uselen, self.subs[0].numz, self.subs[0].numw
        S = self.obs.numharmstages
        kk = k % numrs; k //= numrs
        jj = k % numz; k //= numz
        ii = k % numw; k //= numw
        st = k % S; rs = k // S
        return rs, st, ii, jj, kk


def group_advance(plans: Sequence["JerkPlan"], ahead: int = 0) -> int:
    """Enqueue waves of merged launches over the plans' passes in flight
    (jerk_group_advance): 1 while batches remain, 0 once all are enqueued."""
    n = len(plans)
    parr = (C.c_void_p * max(n, 1))(*[p._p.value for p in plans])
    rc = lib().jerk_group_advance(parr, n, ahead)
    if rc < 0:
        _check(rc)
    return rc


def search_group(plans: Sequence["JerkPlan"], spectra) -> List[np.ndarray]:
    """Whole-spectrum searches of several plans (any geometries, one shared
    stream) in waves of merged launches (jerk_search_group); returns each
    plan's candidate list, bitwise what plan.search(spectrum) returns."""
    n = len(plans)
    if n != len(spectra) or n < 1:
        raise JerkError(JERK_EINVAL, "search_group: one spectrum per plan")
    args = [_spectrum_arg(s) for s in spectra]
    parr = (C.c_void_p * n)(*[p._p.value for p in plans])
    sarr = (C.c_void_p * n)(*[a[0].value for a in args])
    darr = (C.c_int * n)(*[a[1] for a in args])
    outs = (C.POINTER(Cand) * n)()
    counts = (C.c_longlong * n)()
    rc = lib().jerk_search_group(parr, sarr, darr, n, outs, counts)
    res = []
    for i in range(n):
        nb = counts[i] * CAND_DTYPE.itemsize
        res.append(np.frombuffer(C.string_at(outs[i], nb), dtype=CAND_DTYPE).copy() if nb
                   else np.zeros(0, dtype=CAND_DTYPE))
        if outs[i]:
            lib().jerk_free(outs[i])
    _check(rc)
    return res


def _cands_array(ptr, n: int) -> np.ndarray:
    nb = n * CAND_DTYPE.itemsize
    out = np.frombuffer(C.string_at(ptr, nb), dtype=CAND_DTYPE).copy() if nb else \
        np.zeros(0, dtype=CAND_DTYPE)
    lib().jerk_free(ptr)
    return out


class JerkServer:
    """The served form (jerk_server_*): submit spectra as they arrive, poll
    finished candidate lists.  Spectra (numpy arrays on the host, or CUDA
    tensors) are kept alive here until their result has been polled."""

    def __init__(self, hbm_budget_bytes: int = 0, max_active: int = 0, batch: int = 0,
                 device: int = 0, batches_ahead: int = 0, queue_timeout_s: float = 0.0,
                 harm_mode: int = 0):
        cfg = ServerConfig(hbm_budget_bytes, max_active, batch, device, batches_ahead,
                           queue_timeout_s, harm_mode)
        self._s = C.c_void_p()
        _check(lib().jerk_server_create(C.byref(self._s), C.byref(cfg)))
        self._keep = {}
        self._next = 0

    def submit(self, spectrum, N: int, dt: float, zmax: int, wmax: int, numharm: int,
               sigma: float, wmax_given: bool = True, flo: float = 1.0, fhi: float = 10000.0,
               tag: Optional[int] = None, timeseries: bool = False, birdies=None) -> int:
        """Queue one search.  ``spectrum``: the complex64 spectrum (numpy or a
        CUDA tensor), or with ``timeseries=True`` the N float32 samples of a
        time series, which the server turns into its spectrum on the GPU as
        the reference does for a .dat input; ``birdies`` = (lobins, hibins)
        are then zapped after it, as a -zaplist run zaps them."""
        if timeseries:
            if getattr(spectrum, "is_cuda", False):
                ptr, dev, keep = C.c_void_p(spectrum.data_ptr()), 1, spectrum
                n = int(spectrum.numel())
            else:
                keep = np.ascontiguousarray(spectrum, dtype=np.float32)
                ptr, dev, n = C.c_void_p(keep.ctypes.data), 0, len(keep)
            if n != N:
                raise JerkError(JERK_EINVAL, "a time series request needs N samples")
            numbins = N // 2
        else:
            ptr, dev, keep = _spectrum_arg(spectrum)
            numbins = int(spectrum.shape[0]) if dev else len(keep)
        if tag is None:
            tag = self._next
        self._next = max(self._next, tag) + 1
        req = Request(ptr, dev, numbins, N, dt, zmax, wmax, int(wmax_given), numharm, sigma,
                      flo, fhi, tag, int(timeseries))
        if birdies is not None:
            lo = np.ascontiguousarray(birdies[0], dtype=np.float64)
            hi = np.ascontiguousarray(birdies[1], dtype=np.float64)
            keep = (keep, lo, hi)
            req.bird_lobins, req.bird_hibins, req.numbirds = lo.ctypes.data, hi.ctypes.data, len(lo)
        self._keep[tag] = keep  # alive until the result is polled
        _check(lib().jerk_server_submit(self._s, C.byref(req)))
        return tag

    def poll(self, timeout_ms: int = 1000):
        """(tag, candidates, times dict) of the next finished request, or None."""
        r = Result()
        rc = lib().jerk_server_poll(self._s, C.byref(r), timeout_ms)
        if rc == JERK_TIMEOUT:
            return None
        _check(rc)
        self._keep.pop(r.tag, None)
        if r.status != JERK_OK:
            raise JerkError(r.status, f"request {r.tag} failed")
        cands = _cands_array(r.cands, r.ncands)
        return r.tag, cands, {"submit": r.t_submit, "start": r.t_start, "done": r.t_done}

    def stats(self) -> dict:
        a = (C.c_longlong * 6)()
        lib().jerk_server_stats(self._s, a)
        out = dict(zip(["submitted", "finished", "failed", "queued", "peak_bytes", "budget"],
                       list(a)))
        h, d = C.c_longlong(0), C.c_longlong(0)
        lib().jerk_server_transfer_stats(self._s, C.byref(h), C.byref(d))
        out["h2d_bytes"], out["d2h_bytes"] = h.value, d.value
        return out

    def close(self) -> None:
        if self._s:
            lib().jerk_server_destroy(self._s)
            self._s = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def obs_from_refobs(ro) -> Obs:
    """jerk_obs from the reference's accelobs summary (oracle bindings)."""
    o = Obs()
    o.numbins, o.lobin, o.highestbin = ro.numbins, ro.lobin, ro.highestbin
    o.rlo, o.zlo, o.wlo = ro.rlo, ro.zlo, ro.wlo
    o.corr_uselen, o.numz, o.numw = ro.corr_uselen, ro.numz, ro.numw
    o.numharmstages, o.norm_type, o.nph = ro.numharmstages, ro.norm_type, ro.nph
    for i in range(MAX_STAGES):
        o.powcut[i] = ro.powcut[i]
        o.numindep[i] = ro.numindep[i]
    return o
