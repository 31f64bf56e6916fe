"""LIBSVM text cases shared by the reader's tests and its golden-fixture generator.

Every case is (name, text, n, d): the first n lines of `text` are read with d features.  All cases are inputs
the reference's read_input_file (include/read_input.h:8-36) handles with defined behaviour.  ERROR_CASES hold
inputs where it does not (or where the GPU parser declines) and both the oracle and the GPU parser must refuse.
"""
from __future__ import annotations

import numpy as np


def _dense(g, n, d, fmt, scale=1.0, labels="pm1"):
    X = g.standard_normal((n, d)) * scale
    y = np.where(g.random(n) < 0.5, 1, -1)
    lines = []
    for i in range(n):
        lab = {"pm1": f"{y[i]:+d}", "plain": f"{y[i]:d}", "float": f"{float(y[i]):.1f}"}[labels]
        feats = " ".join(f"{k + 1}:{fmt(X[i, k])}" for k in range(d))
        lines.append(f"{lab} {feats}\n")
    return "".join(lines).encode()


def _sparse_binary(g, n, d, p):
    lines = []
    for i in range(n):
        idx = np.flatnonzero(g.random(d) < p) + 1
        lines.append(("1" if g.random() < 0.4 else "-1") + "".join(f" {k}:1" for k in idx) + "\n")
    return "".join(lines).encode()


EDGE_VALUES = [
    "0", "-0", "+0.0", "00012.5000", ".5", "5.", "-.5e2", "1e", "1e+", "1E5", "1.e3", "-1.5E-3",
    "3.4028235e38", "3.4028236e38", "3.40282357e38", "1e39", "-1e39", "1.17549435e-38", "1.4e-45", "7e-46",
    "1e-46", "2.4703282292062327e-324", "2.4703282292062328e-324", "4.9406564584124654e-324", "1e-400",
    "1.7976931348623157e308", "1.7976931348623159e308", "1.8e308", "9007199254740993", "9007199254740992.5",
    "0.1", "0.2", "0.30000000000000004", "123456789012345678901234567890", "0.123456789012345678901234567890123",
    "1234567890123456789012345678.9012345678", "1e22", "1e23", "8.98846567431158e307", "5e-324",
    "inf", "-inf", "INFINITY", "nan", "-nan", "NaN", "in", "na", "0x", "0xg", "+", "-", ".", "-.", "e5", "1e5x",
    "12abc", "  \t7", "1.5\r",
]


def cases():
    g = np.random.default_rng(20261203)
    out = []
    out.append(("dense_repr", _dense(g, 120, 32, repr), 120, 32))
    out.append(("dense_6f", _dense(g, 101, 20, lambda v: f"{v:.6f}", labels="plain"), 101, 20))
    out.append(("dense_3e", _dense(g, 129, 9, lambda v: f"{v:.3e}", scale=1e-3, labels="float"), 129, 9))
    out.append(("dense_g_wide", _dense(g, 12, 700, lambda v: f"{v:g}"), 12, 700))  # lines of several windows
    out.append(("sparse_binary", _sparse_binary(g, 300, 123, 0.11), 300, 123))
    # every edge value as a feature, one per line and all in one line
    d = len(EDGE_VALUES)
    per_line = "".join(f"1 {k + 1}:{v}\n" for k, v in enumerate(EDGE_VALUES)).encode()
    one_line = ("-1 " + " ".join(f"{k + 1}:{v}" for k, v in enumerate(EDGE_VALUES)) + "\n").encode()
    out.append(("edge_values_per_line", per_line, d, d))
    out.append(("edge_values_one_line", one_line, 1, d))
    # labels: +1 / -1 / other values (only an exact 1 gives +1)
    labels = ["+1", "1", "1.0", "1.00000001", "1.0000001", "2", "-1", "0", "1e0", "0.1e1", "inf", "nan", "\n",
              "1\r", "+1.000000000000000000000000000000"]
    out.append(("labels", "".join(f"{lab} 1:1\n" if lab != "\n" else "\n" for lab in labels).encode(),
                len(labels), 1))
    # line structure: blanks, CRLF, empty lines, tokens without ':', index 0 / negative, unsorted and repeated
    # indices (the last value wins), "1:2:3", empty value, empty index, tabs inside tokens, fewer lines than n,
    # no final newline
    text = (b"1   1:1.5    3:2.5   \n"
            b"-1 2:1\r\n"
            b"\n"
            b"1 5 4\n"
            b"-1 0:3 -2:4 3:7\n"
            b"1 4:1 2:2 4:3 1:4 2:5\n"
            b"1 1:2:3 2: :5 \t4:2.5\n"
            b"  -1 3:1e-3 5:-0\n"
            b"1 5:1 5:2 5:3 5:4 5:5 5:6 5:7 5:8 5:9 5:10 5:11 5:12 5:13 5:14 5:15 5:16 5:17 5:18 5:19 5:20"
            b" 5:21 5:22 5:23 5:24 5:25 5:26 5:27 5:28 5:29 5:30 5:31 5:32 5:33 5:34 5:35\n"
            b"-1 1:0.25 3:0.75")
    out.append(("structure", text, 14, 5))
    out.append(("structure_first_lines", text, 4, 5))
    # long line whose tokens straddle 512-byte windows, repeated indices across windows
    toks = " ".join(f"{(k * 37) % 300 + 1}:{k * 0.001:.17g}" for k in range(900))
    rev = " ".join(reversed(toks.split(" ")))
    out.append(("long_repeats", f"1 {toks}\n-1 {rev}\n".encode(), 2, 300))
    return out


ERROR_CASES = [
    ("index_above_d", b"1 1:1 6:2\n", 1, 5),
    ("hex_value", b"1 1:0x1p3\n", 1, 5),
    ("nan_payload", b"1 1:nan(123)\n", 1, 5),
    ("too_many_digits", b"1 1:0.1234567890123456789012345678901234567891\n", 1, 5),
    ("nul_byte", b"1 1:1\x00 2:2\n", 1, 5),
    ("blank_last_line", b"1 1:1\n   ", 2, 5),
]
