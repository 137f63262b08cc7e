"""The 4-point cosine delta weights of the spread and the interpolation
(delta4 in preprocess_src_b200/csrc/rbc_internal.cuh) against the mathematical
functions, on the host.

delta4 evaluates sin(pi f / 2) and cos(pi f / 2) on [0, 1) from fitted
polynomials in FP32 with fused multiply-adds.  The coefficients are read from
the header and the evaluation is emulated in numpy (each multiply-add exact in
FP64, then rounded to FP32), so the bounds below hold for what the kernels run.
"""
import re
from pathlib import Path

import numpy as np

HEADER = Path(__file__).resolve().parents[1] / "preprocess_src_b200" / "csrc" / "rbc_internal.cuh"


def _coefficients():
    text = HEADER.read_text()
    body = text[text.index("void delta4(float f, float w[4])"):]
    body = body[:body.index("w[0] =")]
    p_line = body[body.index("const float p ="):body.index("const float s =")]
    c_line = body[body.index("const float c ="):]
    num = r"[-+]?\d+\.\d+(?:e[-+]?\d+)?f"
    p = [float(x[:-1]) for x in re.findall(num, p_line)]
    c = [float(x[:-1]) for x in re.findall(num, c_line)]
    return p, c   # Horner order: highest degree first


def _fma32(a, b, c):
    return (a.astype(np.float64) * b + c).astype(np.float32)


def _eval(f):
    p, c = _coefficients()
    f = f.astype(np.float32)
    t = (f.astype(np.float64) * f).astype(np.float32)
    acc = np.full_like(t, np.float32(p[0]))
    for k in p[1:]:
        acc = _fma32(acc, t, np.float32(k))
    s = (acc.astype(np.float64) * f).astype(np.float32)
    acc = np.full_like(t, np.float32(c[0]))
    for k in c[1:]:
        acc = _fma32(acc, t, np.float32(k))
    return s, acc


def test_delta_weights_match_sin_and_cos():
    p, c = _coefficients()
    assert len(p) == 5 and len(c) == 6 and c[-1] == 1.0
    f = np.linspace(0.0, 1.0, 400001)
    s, co = _eval(f)
    fd = f.astype(np.float32).astype(np.float64)
    es = np.abs(s - np.sin(np.pi * fd / 2)).max()
    ec = np.abs(co - np.cos(np.pi * fd / 2)).max()
    # about one or two FP32 roundings of values up to 1 (2^-24 = 6e-8)
    assert es <= 2.5e-7 and ec <= 2.5e-7, (es, ec)
    # the bounds the spread's fixed-point scale assumes: weights in [0, 1/2], sum 1
    assert s.min() >= 0.0 and s.max() <= 1.0 and co.min() >= 0.0 and co.max() <= 1.0
    w = np.stack([0.25 - 0.25 * s, 0.25 + 0.25 * co, 0.25 + 0.25 * s, 0.25 - 0.25 * co])
    assert np.abs(w.sum(axis=0) - 1.0).max() <= 3e-7
