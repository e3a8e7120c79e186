"""Compensated FP64 accumulation (mnhack8_b200/csrc/hs_csum.h), on the CPU.

The batched mixed-precision solver accumulates its CG dot products, outer
residual and ABFT checksum sums with the Ogita-Rump-Oishi error-free
transformations.  The header compiles for host and device with the same
operation sequence; this test builds it with g++ (-ffp-contract=off, as the
library's host code) and checks, against exact rational arithmetic:

* Dot2 on ill-conditioned dot products (condition numbers up to ~1e20) is
  accurate to about the working precision times (1 + n^2 u cond), where the
  plain recursive sum has lost every digit;
* merging partial sums of arbitrary splits (the kernels' block partials)
  keeps that accuracy, and a merge is symmetric bit for bit (both lanes of
  an xor butterfly hold the same value).
"""
import os
import struct
import subprocess
import tempfile
from fractions import Fraction

import numpy as np
import pytest

from tests.conftest import ROOT

SRC = r"""
#include <cstdio>
#include <vector>
#include "hs_csum.h"
using namespace hs;
int main(int argc, char** argv) {
    FILE* f = std::fopen(argv[1], "rb");
    long n = 0, split = 0;
    if (std::fread(&n, 8, 1, f) != 1 || std::fread(&split, 8, 1, f) != 1) return 2;
    std::vector<double> x(n), y(n);
    if ((long)std::fread(x.data(), 8, n, f) != n || (long)std::fread(y.data(), 8, n, f) != n) return 2;
    std::fclose(f);
    CSum c{0.0, 0.0};
    double plain = 0.0;
    for (long i = 0; i < n; ++i) { csum_fma(c, x[i], y[i]); plain = std::fma(x[i], y[i], plain); }
    // the same sum as merged block partials of `split` terms each
    CSum m{0.0, 0.0};
    for (long b = 0; b < n; b += split) {
        CSum p{0.0, 0.0};
        for (long i = b; i < n && i < b + split; ++i) csum_fma(p, x[i], y[i]);
        csum_merge(m, p);
    }
    // symmetry of a merge
    CSum a{0.0, 0.0}, b2{0.0, 0.0};
    for (long i = 0; i < n / 2; ++i) csum_fma(a, x[i], y[i]);
    for (long i = n / 2; i < n; ++i) csum_fma(b2, x[i], y[i]);
    CSum ab = a, ba = b2;
    csum_merge(ab, b2);
    csum_merge(ba, a);
    std::printf("%a %a %a %d\n", csum_value(c), plain, csum_value(m),
                (ab.hi == ba.hi && ab.lo == ba.lo) ? 1 : 0);
    return 0;
}
"""


@pytest.fixture(scope="module")
def prog():
    d = tempfile.mkdtemp(prefix="csum_")
    src = os.path.join(d, "t.cpp")
    with open(src, "w") as f:
        f.write(SRC)
    exe = os.path.join(d, "t")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-mfma",
                    "-I", os.path.join(ROOT, "mnhack8_b200", "csrc"), src, "-o", exe], check=True)
    return exe, d


def ill_conditioned(n, cond_exp, seed):
    """A dot product whose terms span ~cond_exp decades and cancel (after the
    GenDot construction of Ogita, Rump and Oishi, simplified)."""
    rng = np.random.default_rng(seed)
    h = n // 2
    e = np.round(rng.uniform(0, cond_exp / 2, h)).astype(int)
    e[0], e[-1] = cond_exp // 2, 0
    x = list(rng.uniform(-1, 1, h) * 2.0 ** (e * np.log2(10)))
    y = list(rng.uniform(-1, 1, h) * 2.0 ** (e * np.log2(10)))
    es = np.round(np.linspace(cond_exp / 2, 0, n - h)).astype(int)
    for k in range(n - h):
        xi = rng.uniform(-1, 1) * 2.0 ** (es[k] * np.log2(10))
        exact = sum(Fraction(a) * Fraction(b) for a, b in zip(x, y))
        yi = (rng.uniform(-1, 1) * 2.0 ** (es[k] * np.log2(10)) - float(exact)) / xi
        x.append(xi)
        y.append(yi)
    perm = rng.permutation(n)
    return np.array(x)[perm], np.array(y)[perm]


@pytest.mark.parametrize("cond_exp,seed", [(12, 1), (16, 2), (20, 3), (20, 4)])
def test_dot2_ill_conditioned(prog, cond_exp, seed):
    exe, d = prog
    n, split = 64, 5
    x, y = ill_conditioned(n, cond_exp, seed)
    exact = sum(Fraction(float(a)) * Fraction(float(b)) for a, b in zip(x, y))
    absdot = sum(abs(Fraction(float(a)) * Fraction(float(b))) for a, b in zip(x, y))
    cond = float(2 * absdot / abs(exact))
    path = os.path.join(d, f"v{seed}.bin")
    with open(path, "wb") as f:
        f.write(struct.pack("<qq", n, split))
        f.write(np.asarray(x, dtype="<f8").tobytes())
        f.write(np.asarray(y, dtype="<f8").tobytes())
    out = subprocess.run([exe, path], check=True, capture_output=True, text=True).stdout.split()
    dot2, plain, merged = (float.fromhex(v) for v in out[:3])
    u = 2.0 ** -53
    bound = (u + 2 * (n * u) ** 2 * cond) * abs(float(exact))
    assert abs(Fraction(dot2) - exact) <= Fraction(bound), (dot2, float(exact), cond)
    assert abs(Fraction(merged) - exact) <= Fraction(bound), (merged, float(exact), cond)
    assert out[3] == "1"                               # merge symmetric bit for bit
    if cond > 1e18:
        # the plain recursive sum has no correct digit left at this conditioning
        assert abs(plain - float(exact)) > 1e-3 * abs(float(exact))
