"""Reading a PRESTO ``.fft`` spectrum and its ``.inf`` for the search, with the
checks the reference leaves out.

The reference's ``create_accelobs`` (src/accel_utils.c:1755-1770) takes N and
dt from the ``.inf`` (``readinf``, src/ioinf.c:121-240) and the bin count from
the ``.fft`` file's length alone (``chkfilelen``), so a truncated or padded
``.fft`` is searched as a shorter or longer spectrum without a word, and a
malformed ``.inf`` ends the process (``exit`` inside ``read_inf_line_valstr``
and ``chk_str2double``).  This reader walks the ``.inf`` lines in the order
``readinf`` does and parses values as it does (the text after the ``=`` in
column 41, or after the last ``=``; numbers by their ``strtod`` prefix), but
reports every problem as a :class:`~prestozl_b200.jerk.JerkError`
(``JERK_EINVAL``) with the file and the field, and it rejects an ``.fft``
whose size is not ``N/2`` complex64 values.
"""

from __future__ import annotations

import os
import re
from typing import Dict, Tuple

import numpy as np

from .jerk import JERK_EINVAL, JerkError

# readinf's first telescope name: the makedata form, without sky/band lines
# (src/ioinf.c:6 scopes[0], :134)
MAKEDATA_SCOPE = "None (Artificial Data Set)"
_NUM = re.compile(r"^\s*[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")


def _fail(path: str, what: str) -> JerkError:
    return JerkError(JERK_EINVAL, f"{path}: {what}")


def _value(line: str, path: str, field: str) -> str:
    """The value string of one .inf line (src/ioinf.c:20-77)."""
    if not line or line == "\n" or not line.strip():
        raise _fail(path, f"end of file or blank line while looking for {field}")
    if len(line) >= 41 and line[40] == "=":
        v = line[41:]
    else:
        i = line.rfind("=")
        if i < 0:
            raise _fail(path, f"no '=' between key and value of {field}")
        v = line[i + 1:]
    v = v.strip()
    return v if v else "Unknown"


def _number(v: str, path: str, field: str) -> float:
    m = _NUM.match(v)
    if not m:
        raise _fail(path, f"cannot read a number for {field} from {v!r}")
    return float(m.group(0))


def read_inf(root: str) -> Dict[str, object]:
    """N, dt, telescope and the on/off count of ``root + '.inf'``."""
    path = root + ".inf"
    try:
        with open(path) as f:
            lines = f.readlines()
    except OSError as e:
        raise _fail(path, f"cannot open ({e.strerror})") from None
    it = iter(lines + [""])
    name = _value(next(it), path, "the data file name")
    scope = _value(next(it), path, "the telescope")
    if scope != MAKEDATA_SCOPE:
        # instrument, object, RA, DEC, observer, MJD, barycentred flag
        for field in ("the instrument", "the object", "RA", "DEC", "the observer", "the MJD",
                      "the barycentred flag"):
            _value(next(it), path, field)
    N = _number(_value(next(it), path, "the number of bins"), path, "the number of bins")
    dt = _number(_value(next(it), path, "the bin width"), path, "the bin width")
    onoff = _number(_value(next(it), path, "the breaks flag"), path, "the breaks flag")
    if N != int(N) or N < 2:
        raise _fail(path, f"number of bins {N!r} is not an integer >= 2")
    if not dt > 0.0 or not np.isfinite(dt):
        raise _fail(path, f"bin width {dt!r} is not a positive number")
    return {"name": name, "telescope": scope, "N": int(N), "dt": dt, "numonoff": int(onoff)}


def load_fft(root: str, mmap: bool = True) -> Tuple[np.ndarray, int, float]:
    """(spectrum, N, dt) of ``root + '.fft'`` / ``root + '.inf'``: the N/2
    complex64 bins of a real FFT (PRESTO packing, bin 0 = DC and Nyquist).
    The file is memory-mapped unless ``mmap`` is false."""
    inf = read_inf(root)
    path = root + ".fft"
    try:
        size = os.path.getsize(path)
    except OSError as e:
        raise _fail(path, f"cannot open ({e.strerror})") from None
    want = inf["N"] // 2
    if size % 8:
        raise _fail(path, f"{size} bytes is not a whole number of complex64 values")
    if size // 8 != want:
        raise _fail(path, f"holds {size // 8} complex64 bins, the .inf's N = {inf['N']} "
                          f"needs {want} (truncated or from another series)")
    spec = np.memmap(path, dtype=np.complex64, mode="r") if mmap else np.fromfile(
        path, dtype=np.complex64)
    return spec, inf["N"], inf["dt"]
