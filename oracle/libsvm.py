"""CPU restatement of the reference's LIBSVM reader, read_input_file<T> (include/read_input.h:8-36).

Test infrastructure only: the product parses on the GPU (db200_libsvm_parse); this module is the checker.

The reference, per line i < n (getline keeps the trailing '\\n'):
  * strtok(line, " ") splits on ' ' only, runs of blanks collapsing (read_input.h:19-33);
  * the first token's atof, converted to T, is the label; Y[i] = 1 when it equals 1, else -1 (:20-22);
  * for every further token, atoi of the part before the first ':' is a 1-based index and atof of the part after
    it is the value (of the whole token when there is no ':'); X[(index - 1) + i*d] = value when index >= 1
    (:25-32).

atof and atoi are prefix parsers: leading C whitespace, then the longest valid number; no number gives 0.  Python's
float() rounds decimal strings correctly, as glibc's strtod does, and numpy's float32 cast rounds the double to
nearest like the C conversion in `T value = atof(...)`.

Cases where the reference's behaviour is undefined, or where the GPU parser declines, raise instead
(LibsvmError): a feature index above d, a last line of blanks only (atof(NULL)), hexadecimal values, "nan(...)"
payloads, more than 38 significant digits, NUL bytes.
"""
from __future__ import annotations

import re
import warnings

import numpy as np

_WS = rb"[ \t\n\v\f\r]*"
_INT = re.compile(_WS + rb"([+-]?[0-9]+)")
_DEC = re.compile(_WS + rb"([+-]?)((?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?)")
_SPECIAL = re.compile(_WS + rb"([+-]?)(inf|nan)(\()?", re.I)
_HEX = re.compile(_WS + rb"[+-]?0[xX](?:[0-9a-fA-F]|\.[0-9a-fA-F])")


class LibsvmError(ValueError):
    pass


def atoi(tok: bytes) -> int:
    m = _INT.match(tok)
    return int(m.group(1)) if m else 0


def _sig_digits(mant: bytes) -> int:
    """Significant digits of a decimal mantissa, up to the last nonzero one."""
    digits = mant.replace(b".", b"").lstrip(b"0").rstrip(b"0")
    return len(digits)


def atof(tok: bytes) -> float:
    if _HEX.match(tok):
        raise LibsvmError("hexadecimal value")
    m = _SPECIAL.match(tok)
    if m:
        if m.group(2).lower() == b"nan":
            if m.group(3):
                raise LibsvmError("NaN payload")
            return -float("nan") if m.group(1) == b"-" else float("nan")
        return float("-inf") if m.group(1) == b"-" else float("inf")
    m = _DEC.match(tok)
    if not m:
        return 0.0
    mant = re.split(rb"[eE]", m.group(2))[0]
    if _sig_digits(mant) > 38:
        raise LibsvmError("more than 38 significant digits")
    return float(m.group(1) + m.group(2))


def _to_t(v: float, dtype):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        return dtype(v)


def read_input_file(data: bytes, n: int, d: int, X: np.ndarray, Y: np.ndarray, dtype=np.float32) -> int:
    """Parse the first n lines of LIBSVM text `data` into X (n x d, row i = point i) and Y (n), in place, with
    the reference's semantics.  Entries the text does not name keep their values.  Returns the lines read."""
    pos, lines = 0, 0
    for i in range(n):
        if pos >= len(data):
            break
        nl = data.find(b"\n", pos)
        end = len(data) if nl < 0 else nl + 1
        line = data[pos:end]
        pos = end
        if b"\0" in line:
            raise LibsvmError(f"line {i + 1}: NUL byte")
        toks = [t for t in line.split(b" ") if t]
        if not toks:
            raise LibsvmError(f"line {i + 1}: no label")
        lab = _to_t(atof(toks[0]), dtype)
        Y[i] = 1 if lab == 1 else -1
        for t in toks[1:]:
            c = t.find(b":")
            idx = atoi(t if c < 0 else t[:c])
            if idx - 1 > -1:
                if idx > d:
                    raise LibsvmError(f"line {i + 1}: feature index {idx} above d = {d}")
                X[i, idx - 1] = _to_t(atof(t if c < 0 else t[c + 1:]), dtype)
        lines += 1
    return lines
