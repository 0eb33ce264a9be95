"""The engine's binary64 emulation (ultrahigh_ann_b200/csrc/exact64.h), which
replays the reference CPU's binary64 sums on the GPU without the FP64 units,
checked bit for bit against the host's IEEE 754 binary64 operations (numpy,
round to nearest even) on millions of operand pairs: random finite bit
patterns, near-cancelling pairs, huge exponent gaps, subnormals, signed zeros,
overflow and underflow. The header is compiled here as plain C++ with g++.
Also the float-float sum's error bound."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parents[1] / "ultrahigh_ann_b200" / "csrc"

HARNESS = r"""
#include "exact64.h"
extern "C" void x64_batch(int op, const uint64_t* a, const uint64_t* b,
                          uint64_t* out, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) {
        out[i] = op == 0 ? uha::x64::add(a[i], b[i])
               : op == 1 ? uha::x64::sub(a[i], b[i])
                         : uha::x64::mul(a[i], b[i]);
    }
}
extern "C" void x64_from_float(const float* f, uint64_t* out, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = uha::x64::from_float(f[i]);
}
extern "C" void x64_to_float(const uint64_t* b, float* out, uint64_t n)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = uha::x64::to_float(b[i]);
}
// float-float sum of (q - r)^2 terms, sequential, as hi and lo
extern "C" void ff_l2(const float* q, const float* r, uint64_t n, float* hi, float* lo)
{
    uha::x64::FF s{0.f, 0.f};
    for (uint64_t i = 0; i < n; ++i) {
        const uha::x64::FF d = uha::x64::two_sum(q[i], -r[i]);
        const uha::x64::FF p = uha::x64::two_prod(d.hi, d.hi);
        const float cross = 2.0f * d.hi * d.lo;
        s = uha::x64::ff_add(s, uha::x64::two_sum(p.hi, p.lo + cross));
    }
    *hi = s.hi;
    *lo = s.lo;
}
"""


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("x64")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    so = d / "libx64.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                    f"-I{CSRC}", str(src), "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    vp = ctypes.c_void_p
    L.x64_batch.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_uint64]
    L.x64_from_float.argtypes = [vp, vp, ctypes.c_uint64]
    L.x64_to_float.argtypes = [vp, vp, ctypes.c_uint64]
    L.ff_l2.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def run(lib, op, a, b):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    out = np.zeros(a.size, np.uint64)
    lib.x64_batch(op, _p(a), _p(b), _p(out), a.size)
    return out


def expect(op, a, b):
    with np.errstate(over="ignore", under="ignore"):
        r = a + b if op == 0 else a - b if op == 1 else a * b
    return r.view(np.uint64)


def finite_bits(rng, n, lo_exp=0, hi_exp=2046):
    sign = rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63)
    exp = rng.integers(lo_exp, hi_exp + 1, n, dtype=np.uint64) << np.uint64(52)
    frac = rng.integers(0, 1 << 52, n, dtype=np.uint64)
    return (sign | exp | frac).view(np.float64)


def cases(rng, n=400_000):
    a = finite_bits(rng, n)
    b = finite_bits(rng, n)
    yield "random", a, b
    # moderate exponents: the replayed sums' range
    a = finite_bits(rng, n, 900, 1150)
    b = finite_bits(rng, n, 900, 1150)
    yield "moderate", a, b
    # near-cancellation: b = -a perturbed by a few ulps
    a = finite_bits(rng, n, 1, 2040)
    ulps = rng.integers(-5, 6, n).astype(np.int64)
    b = -(a.view(np.int64) + ulps).view(np.float64)
    yield "cancel", a, b
    # exponent gaps around the 53/64/128-bit alignment boundaries
    a = finite_bits(rng, n, 1000, 1100)
    gap = rng.choice([1, 2, 52, 53, 54, 63, 64, 65, 66, 116, 117, 127, 128, 129, 200], n)
    b = a * np.ldexp(1.0, -gap) * rng.uniform(0.5, 1.5, n)
    b[rng.random(n) < 0.5] *= -1
    yield "gaps", a, b
    # subnormals and values around the normal boundary
    a = finite_bits(rng, n, 0, 3)
    b = finite_bits(rng, n, 0, 3)
    yield "subnormal", a, b
    # products that underflow into subnormals or overflow
    a = finite_bits(rng, n, 400, 700)
    b = finite_bits(rng, n, 400, 700)
    yield "underflow", a, b
    a = finite_bits(rng, n, 1500, 2046)
    b = finite_bits(rng, n, 1000, 2046)
    yield "overflow", a, b
    # ties: values whose exact sum lies halfway between neighbours
    a = np.ldexp(rng.integers(1 << 52, 1 << 53, n).astype(np.float64), 0)
    b = rng.choice([0.5, 1.5, -0.5, 2.5, 1.0], n)
    yield "halfway", a, b
    z = np.array([0.0, -0.0, 0.0, -0.0, 1.0, -1.0, 5e-324, -5e-324])
    w = np.array([0.0, -0.0, -0.0, 0.0, -1.0, 1.0, -5e-324, 5e-324])
    yield "zeros", z, w


@pytest.mark.parametrize("op", [0, 1, 2])
def test_x64_matches_host_binary64(lib, op):
    rng = np.random.default_rng(op + 1)
    for name, a, b in cases(rng):
        got = run(lib, op, a, b)
        want = expect(op, a, b)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, (name, a[bad[:3]], b[bad[:3]], got[bad[:3]], want[bad[:3]])


def test_x64_from_float_is_exact(lib):
    rng = np.random.default_rng(4)
    bits = rng.integers(0, 0xFFFFFFFF, 1_000_000, dtype=np.uint64).astype(np.uint32)
    f = bits.view(np.float32)
    f = f[np.isfinite(f)]
    f = np.concatenate([f, np.array([0.0, -0.0, 1e-45, -1e-45, 1.17549435e-38], np.float32)])
    out = np.zeros(f.size, np.uint64)
    lib.x64_from_float(_p(f), _p(out), f.size)
    assert np.array_equal(out, f.astype(np.float64).view(np.uint64))


def test_x64_to_float_rounds_like_the_host(lib):
    rng = np.random.default_rng(6)
    parts = [finite_bits(rng, 500_000, 1023 - 160, 1023 + 140),   # binary32 range and beyond
             finite_bits(rng, 200_000),
             # exactly halfway between binary32 neighbours
             (rng.integers(1, 1 << 24, 100_000).astype(np.float64) + 0.5) *
             np.ldexp(1.0, rng.integers(-150, 100, 100_000)),
             np.array([0.0, -0.0, 3.4028235677973366e38, 3.4028235677973366e38 * (1 + 2**-25),
                       1.401298464324817e-45, 7.006492321624085e-46, 7.006492321624087e-46])]
    x = np.concatenate(parts)
    out = np.zeros(x.size, np.float32)
    lib.x64_to_float(_p(x.view(np.uint64)), _p(out), x.size)
    with np.errstate(over="ignore"):
        want = x.astype(np.float32)
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))


def test_float_float_l2_sum_within_stated_bound(lib):
    """Sequential float-float sum of exactly formed (q - r)^2 terms: relative
    error at most (n + 2) * 2^-45 against the exact value (a sorted binary64 sum
    of the exact binary64 terms stands in for it: its own error, below
    n * 2^-53, is far under the bound)."""
    rng = np.random.default_rng(5)
    for n in (1, 7, 1000, 60660):
        q = rng.standard_normal(n).astype(np.float32) * 10
        r = (q + rng.standard_normal(n).astype(np.float32) * 1e-3).astype(np.float32)
        hi = np.zeros(1, np.float32)
        lo = np.zeros(1, np.float32)
        lib.ff_l2(_p(q), _p(r), n, _p(hi), _p(lo))
        d = q.astype(np.float64) - r.astype(np.float64)  # exact
        terms = d * d
        exact = float(np.sum(np.sort(terms)))
        got = float(hi[0]) + float(lo[0])
        assert abs(got - exact) <= (n + 2) * 2.0 ** -45 * exact + 1e-300, n
