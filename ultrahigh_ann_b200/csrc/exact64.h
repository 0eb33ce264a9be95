// Binary64 arithmetic without the FP64 units, for the certified re-score and
// replay paths that keep the GPU's FP64 pipe out of the query path.
//
// Two tools:
//
// * x64::add / x64::sub / x64::mul: IEEE 754 binary64 operations with round
//   to nearest, ties to even, on bit patterns, evaluated with 64- and 128-bit
//   integer arithmetic. Results equal the hardware's __dadd_rn / __dsub_rn /
//   __dmul_rn (and the x86 host's SSE2 double operations) bit for bit for
//   every finite operand, zeros and subnormals included; a result too large
//   overflows to infinity. The operands here are always finite (the scans
//   validate rows and queries). The algorithm is the textbook one: exact
//   integer significand product / aligned sum with a sticky bit, then one
//   rounding of the exact value to 53 significant bits (or to the subnormal
//   grid).
//
// * Float-float (unevaluated sums hi + lo of two binary32 values) for fast
//   sums of exactly formed terms with a small, stated error bound: the
//   error-free TwoSum (Knuth) and TwoProduct (with an FMA) transformations.
//
// The header compiles as CUDA (host and device) and as plain C++ (the host
// tests check x64 against the host's binary64 operations).
#pragma once

#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define UHA_X64 __host__ __device__ __forceinline__
#else
#define UHA_X64 inline
#endif

namespace uha {
namespace x64 {

using u128 = unsigned __int128;

constexpr uint64_t kSignBit = 0x8000000000000000ull;
constexpr uint64_t kFracMask = (1ull << 52) - 1;
constexpr uint64_t kInf = 0x7ff0000000000000ull;

UHA_X64 int bit_length128(u128 v)
{
    const uint64_t hi = static_cast<uint64_t>(v >> 64);
    const uint64_t lo = static_cast<uint64_t>(v);
#ifdef __CUDA_ARCH__
    return hi != 0 ? 128 - __clzll(static_cast<long long>(hi))
                   : (lo != 0 ? 64 - __clzll(static_cast<long long>(lo)) : 0);
#else
    return hi != 0 ? 128 - __builtin_clzll(hi) : (lo != 0 ? 64 - __builtin_clzll(lo) : 0);
#endif
}

// sign, significand and exponent of a finite nonzero binary64: |x| = sig * 2^exp
struct Parts {
    uint64_t sign;
    uint64_t sig;  // < 2^53
    int exp;
};

UHA_X64 Parts unpack(uint64_t bits)
{
    const int biased = static_cast<int>((bits >> 52) & 0x7ff);
    Parts p;
    p.sign = bits & kSignBit;
    if (biased == 0) {  // subnormal
        p.sig = bits & kFracMask;
        p.exp = -1074;
    } else {
        p.sig = (bits & kFracMask) | (1ull << 52);
        p.exp = biased - 1075;
    }
    return p;
}

UHA_X64 bool is_zero(uint64_t bits)
{
    return (bits & ~kSignBit) == 0;
}

// The binary64 nearest (ties to even) to sign * (s + t) * 2^e, where s > 0 is
// an integer and t is a fraction in [0, 1) known only by `sticky` = (t > 0).
// Requires: sticky implies s >= 2^55 (enough bits that the sticky tail lies
// below the rounding position's half unit).
UHA_X64 uint64_t round_pack(uint64_t sign, u128 s, int e, bool sticky)
{
    const int n = bit_length128(s);
    int e_res = e + n - 53;  // exponent of the result's last significand bit
    if (e_res < -1074) {
        e_res = -1074;       // subnormal grid
    }
    const int shift = e_res - e;
    uint64_t sig;
    if (shift <= 0) {
        // exact (s has at most 53 bits here; sticky implies n > 55, shift > 0)
        sig = static_cast<uint64_t>(s << (-shift));
    } else if (shift >= 129) {
        sig = 0;  // far below half of the smallest subnormal
    } else {
        u128 rem;
        u128 half;
        if (shift == 128) {
            sig = 0;
            rem = s;
            half = static_cast<u128>(1) << 127;
        } else {
            sig = static_cast<uint64_t>(s >> shift);
            rem = s & ((static_cast<u128>(1) << shift) - 1);
            half = static_cast<u128>(1) << (shift - 1);
        }
        const bool up = rem > half || (rem == half && (sticky || (sig & 1)));
        if (up) {
            ++sig;
            if (sig == (1ull << 53)) {
                sig >>= 1;
                ++e_res;
            }
        }
    }
    if (sig == 0) {
        return sign;
    }
    if (sig < (1ull << 52)) {
        return sign | sig;  // subnormal (e_res == -1074)
    }
    const int biased = e_res + 1075;
    if (biased >= 2047) {
        return sign | kInf;
    }
    return sign | (static_cast<uint64_t>(biased) << 52) | (sig & kFracMask);
}

UHA_X64 uint64_t mul(uint64_t a, uint64_t b)
{
    const uint64_t sign = (a ^ b) & kSignBit;
    if (is_zero(a) || is_zero(b)) {
        return sign;
    }
    const Parts pa = unpack(a);
    const Parts pb = unpack(b);
    const u128 s = static_cast<u128>(pa.sig) * pb.sig;
    return round_pack(sign, s, pa.exp + pb.exp, false);
}

UHA_X64 uint64_t add(uint64_t a, uint64_t b)
{
    if (is_zero(a)) {
        // -0 + -0 = -0, +0 + -0 = +0; x + 0 = x
        return is_zero(b) ? (a & b) : b;
    }
    if (is_zero(b)) {
        return a;
    }
    Parts pa = unpack(a);
    Parts pb = unpack(b);
    if (pa.exp < pb.exp || (pa.exp == pb.exp && pa.sig < pb.sig)) {
        const Parts t = pa;
        pa = pb;
        pb = t;
    }
    // |a| >= |b|; both significands placed 64 bits up (exact), b aligned to a
    const int d = pa.exp - pb.exp;
    const u128 sa = static_cast<u128>(pa.sig) << 64;
    u128 sb = static_cast<u128>(pb.sig) << 64;
    bool sticky = false;
    if (d >= 128) {
        sb = 0;
        sticky = true;
    } else if (d > 0) {
        const u128 lost = sb & ((static_cast<u128>(1) << d) - 1);
        sticky = lost != 0;
        sb >>= d;
    }
    const int e = pa.exp - 64;
    if (pa.sign == pb.sign) {
        return round_pack(pa.sign, sa + sb, e, sticky);
    }
    // |a| - |b| - t: with a sticky tail t in (0, 1), that is (s - 1) + (1 - t)
    u128 s = sa - sb;
    if (sticky) {
        s -= 1;  // s >= 2^115 here (d > 64)
    }
    if (s == 0) {
        return 0;  // x - x = +0 under round to nearest
    }
    return round_pack(pa.sign, s, e, sticky);
}

UHA_X64 uint64_t sub(uint64_t a, uint64_t b)
{
    return add(a, b ^ kSignBit);
}

// Exact binary64 bits of a binary32 value.
UHA_X64 uint64_t from_float(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    const uint64_t sign = static_cast<uint64_t>(u & 0x80000000u) << 32;
    const int biased = static_cast<int>((u >> 23) & 0xff);
    const uint32_t frac = u & 0x7fffffu;
    if (biased == 0) {
        if (frac == 0) {
            return sign;
        }
        // subnormal binary32: frac * 2^-149, normal in binary64
        return round_pack(sign, frac, -149, false);
    }
    return sign | (static_cast<uint64_t>(biased - 127 + 1023) << 52) |
           (static_cast<uint64_t>(frac) << 29);
}

// The binary32 nearest (ties to even) to a finite binary64, infinity when it
// overflows, with binary32 subnormals.
UHA_X64 float to_float(uint64_t bits)
{
    uint32_t out = static_cast<uint32_t>((bits & kSignBit) >> 32);
    if (!is_zero(bits)) {
        const Parts p = unpack(bits);
        // value = sig * 2^exp, sig < 2^53; round to 24 bits on the binary32 grid
        const int n = bit_length128(p.sig);
        int e_res = p.exp + n - 24;
        if (e_res < -149) {
            e_res = -149;
        }
        const int shift = e_res - p.exp;
        uint64_t sig;
        if (shift <= 0) {
            sig = p.sig << (-shift);
        } else if (shift >= 64) {
            sig = 0;  // p.sig < 2^53: below half of the smallest subnormal
        } else {
            const uint64_t rem = p.sig & ((1ull << shift) - 1);
            const uint64_t half = 1ull << (shift - 1);
            sig = p.sig >> shift;
            if (rem > half || (rem == half && (sig & 1))) {
                ++sig;
                if (sig == (1ull << 24)) {
                    sig >>= 1;
                    ++e_res;
                }
            }
        }
        if (sig != 0) {
            if (sig < (1ull << 23)) {
                out |= static_cast<uint32_t>(sig);  // subnormal
            } else {
                const int biased = e_res + 150;
                out |= biased >= 255 ? 0x7f800000u
                                     : (static_cast<uint32_t>(biased) << 23) |
                                           static_cast<uint32_t>(sig & 0x7fffffu);
            }
        }
    }
    float f;
    std::memcpy(&f, &out, sizeof(f));
    return f;
}

// ------------------------------------------------------------ float-float

struct FF {
    float hi;
    float lo;
};

// a + b = s + err exactly (Knuth's TwoSum; round to nearest, no overflow).
UHA_X64 FF two_sum(float a, float b)
{
#ifdef __CUDA_ARCH__
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float err = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
#else
    volatile float s = a + b;
    volatile float bb = s - a;
    volatile float t1 = s - bb;
    volatile float t2 = a - t1;
    volatile float t3 = b - bb;
    const float err = t2 + t3;
#endif
    return FF{s, err};
}

// a * b = p + err exactly (TwoProduct with an FMA; no underflow of err).
UHA_X64 FF two_prod(float a, float b)
{
#ifdef __CUDA_ARCH__
    const float p = __fmul_rn(a, b);
    return FF{p, __fmaf_rn(a, b, -p)};
#else
    const float p = a * b;
    return FF{p, __builtin_fmaf(a, b, -p)};
#endif
}

// Sum of two nonnegative float-float values with relative error at most
// 2^-46 of the result (the accurate Dekker/Bailey addition).
UHA_X64 FF ff_add(FF a, FF b)
{
    const FF s = two_sum(a.hi, b.hi);
    const FF t = two_sum(a.lo, b.lo);
#ifdef __CUDA_ARCH__
    const float c = __fadd_rn(s.lo, t.hi);
    FF u = two_sum(s.hi, c);
    const float w = __fadd_rn(t.lo, u.lo);
#else
    const float c = s.lo + t.hi;
    FF u = two_sum(s.hi, c);
    const float w = t.lo + u.lo;
#endif
    return two_sum(u.hi, w);
}

}  // namespace x64
}  // namespace uha
