"""ctypes bindings for the oracle's two libraries.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` -- never by the product package.

* ``RefSearch`` drives ``oracle/_ref/libprestoref.so``: the reference's own
  accelsearch objects (compiled from the reference sources by
  ``oracle/Makefile``) behind ``oracle/ref_driver.c``.
* ``Oracle`` drives ``oracle/liboracle.so``: this project's CPU restatement of
  the search (``oracle/jerk_oracle.c``), which works on explicit arrays.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libprestoref.so")
REF_CLI = os.path.join(REF_DIR, "accelsearch")
DROPIN_CLI = os.path.join(REF_DIR, "accelsearch_b200")
DROPIN_MANY_CLI = os.path.join(REF_DIR, "accelsearch_b200_many")
REFGPU_CLI = os.path.join(REF_DIR, "accelsearch_refgpu")
REF_DEDISP_GPU_LIB = os.path.join(REF_DIR, "libprestodedisp_gpu.so")
PREPSUBBAND_DROPIN_LIB = os.path.join(REF_DIR, "libprepsubband_dropin.so")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
# Where the reference's sources lie: $PRESTOZL_REFERENCE, by default the
# checkout this build recipe was written against.  Only the build (and CPU
# tests that read the reference's Python) look there; the built oracle/_ref
# travels without it.
REFERENCE_SOURCES = os.environ.get("PRESTOZL_REFERENCE", "/root/reference")


def build(reference: Optional[bool] = None) -> None:
    """Compile the oracle (always) and the reference build (when the
    reference sources are present)."""
    if reference is None:
        reference = os.path.isdir(os.path.join(REFERENCE_SOURCES, "src"))
    targets = ["oracle"] + (["ref", "dropin", "refgpu", "dedispgpu"] if reference else [])
    subprocess.run(["make", "-s", "-C", HERE, "-j8", f"REF={REFERENCE_SOURCES}", *targets],
                   check=True)


def have_reference() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(REF_CLI)


class RefObs(C.Structure):
    _fields_ = [
        ("N", C.c_longlong), ("numbins", C.c_longlong), ("lobin", C.c_longlong),
        ("highestbin", C.c_longlong),
        ("maxkernlen", C.c_int), ("corr_uselen", C.c_int), ("fftlen", C.c_int),
        ("numharmstages", C.c_int), ("numz", C.c_int), ("numw", C.c_int),
        ("norm_type", C.c_int), ("inmem", C.c_int),
        ("dt", C.c_double), ("T", C.c_double), ("rlo", C.c_double), ("rhi", C.c_double),
        ("zlo", C.c_double), ("zhi", C.c_double), ("wlo", C.c_double), ("whi", C.c_double),
        ("nph", C.c_double),
        ("powcut", C.c_float * 6), ("numindep", C.c_longlong * 6),
    ]


class RefCand(C.Structure):
    _fields_ = [("power", C.c_float), ("sigma", C.c_float), ("numharm", C.c_int),
                ("r", C.c_double), ("z", C.c_double), ("w", C.c_double)]


CAND_DTYPE = np.dtype([("power", np.float32), ("sigma", np.float32), ("numharm", np.int32),
                       ("r", np.float64), ("z", np.float64), ("w", np.float64)], align=True)

_reflib = None


def quiet_wisdom() -> None:
    """The reference's FFT wrapper (src/fftcalls.c:13-35) reads a wisdom file
    from $PRESTO/lib and prints a warning to stdout when it is missing; point
    PRESTO at an empty one so the reference prints nothing."""
    d = os.path.join(REF_DIR, "presto_home")
    f = os.path.join(d, "lib", "fftw_wisdom.txt")
    if not os.path.exists(f):
        os.makedirs(os.path.dirname(f), exist_ok=True)
        open(f, "w").close()
    os.environ["PRESTO"] = d


def _ref():
    global _reflib
    if _reflib is None:
        quiet_wisdom()
        lib = C.CDLL(REF_LIB)
        lib.ref_open.restype = C.c_void_p
        lib.ref_open.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        lib.ref_get_obs.argtypes = [C.c_void_p, C.POINTER(RefObs)]
        lib.ref_make_bank.argtypes = [C.c_void_p]
        lib.ref_shi_info.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
        lib.ref_copy_kernels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        lib.ref_fderivs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.POINTER(C.c_longlong), C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        lib.ref_search.restype = C.c_long
        lib.ref_search.argtypes = [C.c_void_p, C.c_long, C.c_void_p, C.c_long,
                                   C.POINTER(C.c_long)]
        lib.ref_candidate_sigma.restype = C.c_double
        lib.ref_candidate_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
        lib.ref_power_for_sigma.restype = C.c_double
        lib.ref_power_for_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
        lib.ref_w_resp_halfwidth.argtypes = [C.c_double, C.c_double, C.c_int]
        lib.ref_next_good_fftlen.argtypes = [C.c_int]
        lib.ref_fftlen_from_kernwidth.argtypes = [C.c_int]
        lib.ref_median.restype = C.c_float
        lib.ref_median.argtypes = [C.c_void_p, C.c_int]
        lib.ref_gen_w_response.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double,
                                           C.c_int, C.c_void_p]
        lib.ref_close.argtypes = [C.c_void_p]
        lib.ref_set_threads.argtypes = [C.c_int]
        lib.ref_insert_sequence.restype = C.c_long
        lib.ref_insert_sequence.argtypes = [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_long]
        lib.ref_set_threads(1)
        _reflib = lib
    return _reflib


def reflib():
    return _ref()


class RefSearch:
    """The reference accelsearch set up on one ``.fft`` file.

    ``args`` are accelsearch command-line flags (e.g. ``-zmax 20``); the file
    name comes last, as on the reference's command line.  The reference opens
    its ``.txtcand`` work file next to the ``.fft``.
    """

    def __init__(self, fftfile: str, args: Sequence[str]):
        argv = ["accelsearch", *[str(a) for a in args], fftfile]
        arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
        self._argv = arr
        self.ctx = _ref().ref_open(len(argv), arr)
        o = RefObs()
        _ref().ref_get_obs(self.ctx, C.byref(o))
        self.obs = o

    def spectrum(self) -> np.ndarray:
        """The spectrum the reference searches (after its .dat preparation)."""
        out = np.zeros(int(self.obs.numbins), dtype=np.complex64)
        f = _ref().ref_copy_spectrum
        f.restype = C.c_long
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
        n = f(self.ctx, out.ctypes.data, len(out))
        if n < 0:
            raise RuntimeError("the reference holds no spectrum in memory")
        return out[:n]

    def polish(self, numharm: int, r: float, z: float, w: float):
        """The reference's polishing volume search for a candidate (r
        relative to obs.lobin): ((r, z, w) polished, locpow per harmonic,
        highest harmonic first)."""
        f = _ref().ref_polish
        f.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p,
                      C.c_void_p]
        rzw = np.zeros(3)
        lp = np.zeros(numharm, dtype=np.float32)
        if f(self.ctx, numharm, r, z, w, rzw.ctypes.data, lp.ctypes.data) != 0:
            raise RuntimeError("the reference holds no spectrum in memory")
        return tuple(float(v) for v in rzw), lp

    def close(self):
        if self.ctx:
            _ref().ref_close(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def make_bank(self):
        _ref().ref_make_bank(self.ctx)

    def subharmonics(self):
        """[(stage, harm)] in the reference's bank order."""
        out = [(0, 1)]
        for stage in range(1, self.obs.numharmstages):
            for harm in range(1, 1 << stage, 2):
                out.append((stage, harm))
        return out

    def shi_info(self, stage: int, harm: int) -> dict:
        self.make_bank()
        info = (C.c_int * 8)()
        _ref().ref_shi_info(self.ctx, stage, harm, info)
        keys = ["numharm", "harmnum", "zmax", "wmax", "numz", "numw", "fftlen", "halfwidth"]
        return dict(zip(keys, list(info)))

    def kernels(self, stage: int, harm: int) -> np.ndarray:
        info = self.shi_info(stage, harm)
        out = np.zeros((info["numw"], info["numz"], info["fftlen"]), dtype=np.complex64)
        _ref().ref_copy_kernels(self.ctx, stage, harm, out.ctypes.data)
        return out

    def fderivs(self, numharm: int, harmnum: int, fullrlo: float, fullrhi: float):
        """(header dict, powers[w][z][r], rinds, zinds) of one subharmonic."""
        self.make_bank()
        hdr = (C.c_longlong * 6)()
        _ref().ref_fderivs(self.ctx, numharm, harmnum, fullrlo, fullrhi, hdr, None, None, None)
        h = dict(zip(["rlo", "zlo", "wlo", "numrs", "numzs", "numws"], list(hdr)))
        pw = np.zeros((h["numws"], h["numzs"], h["numrs"]), dtype=np.float32)
        rinds = np.zeros(self.obs.corr_uselen, dtype=np.uint16)
        zinds = np.zeros(self.obs.numz, dtype=np.uint16)
        _ref().ref_fderivs(self.ctx, numharm, harmnum, fullrlo, fullrhi, hdr,
                           pw.ctypes.data, rinds.ctypes.data, zinds.ctypes.data)
        return h, pw, rinds, zinds

    def insert_sequence(self, pows, rlo, numharm, max_out: int = 1 << 20):
        """The reference's own list insertion over a crafted hit sequence
        (one 1x1x1 volume per hit through search_ffdotpows)."""
        pows = np.ascontiguousarray(pows, dtype=np.float32)
        rlo = np.ascontiguousarray(rlo, dtype=np.int64)
        numharm = np.ascontiguousarray(numharm, dtype=np.int32)
        out = np.zeros(max_out, dtype=CAND_DTYPE)
        n = _ref().ref_insert_sequence(self.ctx, len(pows), pows.ctypes.data, rlo.ctypes.data,
                                       numharm.ctypes.data, out.ctypes.data, max_out)
        return out[: min(n, max_out)].copy()

    def search(self, max_steps: int = 0, max_out: int = 1 << 20):
        out = np.zeros(max_out, dtype=CAND_DTYPE)
        done = C.c_long(0)
        n = _ref().ref_search(self.ctx, max_steps, out.ctypes.data, max_out, C.byref(done))
        if n < 0:
            raise RuntimeError("reference search refused this configuration")
        return out[: min(n, max_out)].copy(), done.value


def set_threads(n: int) -> None:
    """OpenMP threads for the reference's parallel loops (1 = its default)."""
    _ref().ref_set_threads(n)


def candidate_sigma(power: float, numsum: int, numtrials: float) -> float:
    return _ref().ref_candidate_sigma(power, numsum, numtrials)


def power_for_sigma(sigma: float, numsum: int, numtrials: float) -> float:
    return _ref().ref_power_for_sigma(sigma, numsum, numtrials)


# --------------------------------------------------------------------------
# The oracle restatement (oracle/jerk_oracle.c)

class OrcGeom(C.Structure):
    _fields_ = [
        ("numbins", C.c_longlong), ("lobin", C.c_longlong), ("highestbin", C.c_longlong),
        ("rlo", C.c_double), ("zlo", C.c_double), ("wlo", C.c_double),
        ("corr_uselen", C.c_int), ("numz", C.c_int), ("numharmstages", C.c_int),
        ("norm_type", C.c_int), ("nph", C.c_double),
        ("powcut", C.c_float * 6), ("numindep", C.c_longlong * 6),
    ]


class OrcSub(C.Structure):
    _fields_ = [("numharm", C.c_int), ("harmnum", C.c_int), ("numz", C.c_int),
                ("numw", C.c_int), ("fftlen", C.c_int), ("halfwidth", C.c_int),
                ("kern", C.c_void_p)]


_orclib = None


def _orc():
    global _orclib
    if _orclib is None:
        lib = C.CDLL(ORACLE_LIB)
        lib.orc_fderivs.argtypes = [C.POINTER(OrcGeom), C.POINTER(OrcSub), C.c_void_p,
                                    C.c_double, C.c_double, C.POINTER(C.c_longlong),
                                    C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_summed.argtypes = [C.POINTER(OrcGeom), C.POINTER(OrcSub), C.c_void_p,
                                   C.c_double, C.c_int, C.c_void_p]
        lib.orc_search.restype = C.c_long
        lib.orc_search.argtypes = [C.POINTER(OrcGeom), C.POINTER(OrcSub), C.c_void_p,
                                   C.c_long, C.c_long, C.c_void_p, C.c_long,
                                   C.POINTER(C.c_long), C.POINTER(C.c_long)]
        lib.orc_search_hits.restype = C.c_long
        lib.orc_search_hits.argtypes = [C.POINTER(OrcGeom), C.POINTER(OrcSub), C.c_void_p,
                                        C.c_long, C.c_long, C.c_void_p, C.c_long,
                                        C.POINTER(C.c_long), C.POINTER(C.c_long),
                                        C.c_void_p, C.c_void_p, C.c_long]
        lib.orc_insert_hits.restype = C.c_long
        lib.orc_insert_hits.argtypes = [C.c_void_p, C.c_long, C.POINTER(C.c_longlong),
                                        C.c_void_p, C.c_long]
        lib.orc_candidate_sigma.restype = C.c_double
        lib.orc_candidate_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
        lib.orc_power_for_sigma.restype = C.c_double
        lib.orc_power_for_sigma.argtypes = [C.c_double, C.c_int, C.c_double]
        lib.orc_w_resp_halfwidth.argtypes = [C.c_double, C.c_double]
        lib.orc_next_good_fftlen.argtypes = [C.c_int]
        lib.orc_fftlen_from_kernwidth.argtypes = [C.c_int]
        lib.orc_obs_sizes.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int)]
        lib.orc_sub_sizes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_int)]
        lib.orc_calc_required_r.restype = C.c_double
        lib.orc_calc_required_r.argtypes = [C.c_double, C.c_double]
        lib.orc_calc_required_z.argtypes = [C.c_double, C.c_double]
        lib.orc_calc_required_w.argtypes = [C.c_double, C.c_double]
        lib.orc_downsample_subbands.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                C.c_int]
        lib.orc_dedisp_subbands.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                            C.c_int, C.c_void_p]
        _orclib = lib
    return _orclib


def orclib():
    return _orc()


def geom_from_refobs(o: RefObs) -> OrcGeom:
    g = OrcGeom()
    g.numbins, g.lobin, g.highestbin = o.numbins, o.lobin, o.highestbin
    g.rlo, g.zlo, g.wlo = o.rlo, o.zlo, o.wlo
    g.corr_uselen, g.numz, g.numharmstages = o.corr_uselen, o.numz, o.numharmstages
    g.norm_type, g.nph = o.norm_type, o.nph
    for i in range(6):
        g.powcut[i] = o.powcut[i]
        g.numindep[i] = o.numindep[i]
    return g


def local_powers(powers: np.ndarray) -> np.ndarray:
    """The oracle's -locpow local power levels (direct restatement)."""
    p = np.ascontiguousarray(powers, dtype=np.float32)
    out = np.zeros_like(p)
    f = _orc().orc_local_powers
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    f(p.ctypes.data, len(p), out.ctypes.data)
    return out


def ref_local_powers(powers: np.ndarray) -> np.ndarray:
    """The reference's own corr_loc_pow (FFT correlation)."""
    p = np.array(powers, dtype=np.float32)  # the reference may work in place
    out = np.zeros_like(p)
    f = _ref().ref_corr_loc_pow
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    f(p.ctypes.data, len(p), out.ctypes.data)
    return out


def deredden(spectrum: np.ndarray, reference: bool = False) -> np.ndarray:
    """Red-noise removal (src/accel_utils.c:1557-1633) on a copy of a
    complex64 spectrum: the oracle's restatement, or the reference's own."""
    f = _ref().deredden if reference else _orc().orc_deredden
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_int]
    a = np.array(spectrum, dtype=np.complex64)
    f(a.ctypes.data, len(a))
    return a


def zap_list(spectrum: np.ndarray, N: int, lobins, hibins) -> np.ndarray:
    """The oracle's birdie zapping (zapbirds over a birdie list, as the
    reference's CPU1 applies it) on a copy of a complex64 spectrum."""
    f = _orc().orc_zap_list
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_long, C.c_longlong, C.c_void_p, C.c_void_p, C.c_int]
    a = np.array(spectrum, dtype=np.complex64)
    lo = np.ascontiguousarray(lobins, dtype=np.float64)
    hi = np.ascontiguousarray(hibins, dtype=np.float64)
    f(a.ctypes.data, len(a), N, lo.ctypes.data, hi.ctypes.data, len(lo))
    return a


def zapbirds(spectrum: np.ndarray, lobin: float, hibin: float, reference: bool = False):
    """One zapbirds (src/zapping.c:29-81) on a copy of a spectrum, by the
    oracle or by the reference build (which reads up to 100 bins past the end:
    the copy is zero-padded there, as the reference's .dat buffer is)."""
    n = len(spectrum)
    pad = np.zeros(n + 2000, dtype=np.complex64)
    pad[1000:1000 + n] = spectrum
    if reference:
        f = _ref().zapbirds
        f.restype = None
        f.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        f(lobin, hibin, None, pad[1000:].ctypes.data)
    else:
        f = _orc().orc_zapbirds
        f.restype = None
        f.argtypes = [C.c_void_p, C.c_long, C.c_double, C.c_double]
        f(pad[1000:].ctypes.data, n, lobin, hibin)
    return pad[1000:1000 + n].copy()


def ref_realfft(series: np.ndarray) -> np.ndarray:
    """The reference's forward realfft (src/fastffts.c:163-235, isign -1) on a
    copy of a float32 series, as built here (its complex FFT is the FFTW
    stand-in under shim/)."""
    f = _ref().realfft
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_long, C.c_int]
    a = np.array(series, dtype=np.float32)
    f(a.ctypes.data, len(a), -1)
    return a.view(np.complex64)


def packed_rfft(series: np.ndarray) -> np.ndarray:
    """The FP64 forward real FFT in the reference's packing: n/2 complex
    values, value 0 = (DC, Nyquist)."""
    X = np.fft.rfft(np.asarray(series, dtype=np.float64))
    n = len(series)
    out = X[: n // 2].copy()
    out[0] = complex(X[0].real, X[n // 2].real)
    return out


def pair_magnitude(packed: np.ndarray) -> np.ndarray:
    """|X[k]| + |X[M-k]| for a packed spectrum of M values (bin 0 pairs with
    itself): the scale of the rounding a real FFT built on an M-point complex
    FFT leaves in bin k."""
    a = np.abs(np.asarray(packed))
    return a + np.concatenate([a[:1], a[:0:-1]])


def downsample_subbands(data: np.ndarray, bs: int) -> np.ndarray:
    """Subband downsampling (orc_downsample_subbands): data [worklen * bs,
    nsub] float32, time-major -> [worklen, nsub]."""
    x = np.ascontiguousarray(data, dtype=np.float32)
    worklen, nsub = x.shape[0] // bs, x.shape[1]
    out = np.empty((worklen, nsub), dtype=np.float32)
    _orc().orc_downsample_subbands(out.ctypes.data, x.ctypes.data, worklen, bs, nsub)
    return out


def dedisp_subbands(cur: np.ndarray, last: np.ndarray, offsets: np.ndarray,
                    reference: bool = False) -> np.ndarray:
    """Subband dedispersion of one block: cur and last [worklen, nsub]
    float32, offsets [numdms, nsub] -> [numdms, worklen].  The oracle's
    restatement, or with reference=True the reference's own float_dedisp
    (src/dispersion.c:208-231) once per DM, as prepsubband calls it."""
    c = np.ascontiguousarray(cur, dtype=np.float32)
    l = np.ascontiguousarray(last, dtype=np.float32)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    worklen, nsub = c.shape
    numdms = off.shape[0]
    out = np.empty((numdms, worklen), dtype=np.float32)
    if reference:
        f = _ref().float_dedisp
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_void_p]
        for d in range(numdms):
            f(c.ctypes.data, l.ctypes.data, worklen, nsub, off[d].ctypes.data, 0.0,
              out[d].ctypes.data)
    else:
        _orc().orc_dedisp_subbands(c.ctypes.data, l.ctypes.data, out.ctypes.data, worklen, nsub,
                                   numdms, off.ctypes.data)
    return out


def invsqrtf(x: float, reference: bool = False) -> float:
    f = _ref().ref_invsqrtf if reference else _orc().orc_invsqrtf
    f.restype = C.c_float
    f.argtypes = [C.c_float]
    return float(f(x))


class Oracle:
    """The oracle restatement on explicit arrays.

    ``subs`` is a list of dicts (bank order) with keys numharm, harmnum,
    numz, numw, fftlen, halfwidth and ``kern`` (complex64 [numw][numz][fftlen]).
    """

    def __init__(self, spectrum: np.ndarray, geom: OrcGeom, subs: List[dict]):
        self.spec = np.ascontiguousarray(spectrum, dtype=np.complex64)
        self.geom = geom
        self._kerns = [np.ascontiguousarray(s["kern"], dtype=np.complex64) for s in subs]
        self.subs = (OrcSub * len(subs))()
        for i, s in enumerate(subs):
            self.subs[i] = OrcSub(s["numharm"], s["harmnum"], s["numz"], s["numw"],
                                  s["fftlen"], s["halfwidth"], self._kerns[i].ctypes.data)

    def fderivs(self, sub_index: int, fullrlo: float, fullrhi: float):
        hdr = (C.c_longlong * 6)()
        g, s = C.byref(self.geom), C.byref(self.subs[sub_index])
        _orc().orc_fderivs(g, s, self.spec.ctypes.data, fullrlo, fullrhi, hdr, None, None, None)
        h = dict(zip(["rlo", "zlo", "wlo", "numrs", "numzs", "numws"], list(hdr)))
        pw = np.zeros((h["numws"], h["numzs"], h["numrs"]), dtype=np.float32)
        rinds = np.zeros(self.geom.corr_uselen, dtype=np.uint16)
        zinds = np.zeros(self.geom.numz, dtype=np.uint16)
        _orc().orc_fderivs(g, s, self.spec.ctypes.data, fullrlo, fullrhi, hdr,
                           pw.ctypes.data, rinds.ctypes.data, zinds.ctypes.data)
        return h, pw, rinds, zinds

    def summed(self, startr: float, upto_stage: int) -> np.ndarray:
        s0 = self.subs[0]
        pw = np.zeros((s0.numw, s0.numz, self.geom.corr_uselen), dtype=np.float32)
        _orc().orc_summed(C.byref(self.geom), self.subs, self.spec.ctypes.data, startr,
                          upto_stage, pw.ctypes.data)
        return pw

    def search(self, first_step: int = 0, max_steps: int = 0, max_out: int = 1 << 20):
        out = np.zeros(max_out, dtype=CAND_DTYPE)
        done, nh = C.c_long(0), C.c_long(0)
        n = _orc().orc_search(C.byref(self.geom), self.subs, self.spec.ctypes.data,
                              first_step, max_steps, out.ctypes.data, max_out,
                              C.byref(done), C.byref(nh))
        return out[: min(n, max_out)].copy(), done.value, nh.value


    def search_hits(self, first_step: int = 0, max_steps: int = 0, max_out: int = 1 << 20,
                    hit_cap: int = 1 << 22):
        """(cands, steps, hit keys, hit powers): every threshold crossing in
        insertion order, keyed as the product keys its hits."""
        out = np.zeros(max_out, dtype=CAND_DTYPE)
        keys = np.zeros(hit_cap, dtype=np.uint64)
        pows = np.zeros(hit_cap, dtype=np.float32)
        done, nh = C.c_long(0), C.c_long(0)
        n = _orc().orc_search_hits(C.byref(self.geom), self.subs, self.spec.ctypes.data,
                                   first_step, max_steps, out.ctypes.data, max_out,
                                   C.byref(done), C.byref(nh), keys.ctypes.data,
                                   pows.ctypes.data, hit_cap)
        m = min(nh.value, hit_cap)
        return out[: min(n, max_out)].copy(), done.value, keys[:m].copy(), pows[:m].copy()


def insert_hits(hits: np.ndarray, numindep: Sequence[int], max_out: int = 1 << 20):
    """insert_new_accelcand over a decoded hit sequence (CAND_DTYPE; sigma is
    recomputed)."""
    hits = np.ascontiguousarray(hits, dtype=CAND_DTYPE)
    out = np.zeros(max_out, dtype=CAND_DTYPE)
    ni = (C.c_longlong * 6)(*[int(x) for x in list(numindep)[:6]])
    n = _orc().orc_insert_hits(hits.ctypes.data, len(hits), ni, out.ctypes.data, max_out)
    return out[: min(n, max_out)].copy()


def orc_candidate_sigma(power: float, numsum: int, numtrials: float) -> float:
    return _orc().orc_candidate_sigma(power, numsum, numtrials)


def orc_power_for_sigma(sigma: float, numsum: int, numtrials: float) -> float:
    return _orc().orc_power_for_sigma(sigma, numsum, numtrials)
