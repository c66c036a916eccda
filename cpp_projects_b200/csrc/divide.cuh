// Correctly rounded division by a small divisor known at compile time.
//
// The level-0 running means divide by r + 1 for every sample; an IEEE
// divide (__fdiv_rn) costs a reciprocal on the special-function unit plus a
// correction sequence, and it dominated the fused head's instruction count.
//
// Method: Brisebarre, Muller and Raina, "Accelerating correctly rounded
// floating-point division when the divisor is known in advance", IEEE
// Transactions on Computers 53(8), 2004.  With zh = RN(1/d) and
// zl ~ (1 - d zh) / d (the part of 1/d that zh misses), the quotient is
// q = RN(x zh + RN(x zl)): one multiply and one fused multiply-add.  The
// paper shows q = RN(x / d) for every x of a normal range when d passes its
// test; here the claim is checked exhaustively instead — every finite float
// x against __fdiv_rn, for each divisor the kernels use (the library's
// self-test entry bfs_selftest_divide).
//
// Outside the range where x zl is a normal number the product underflows and
// the identity fails (e.g. x below 1e-36 for d = 3), so |x| < 2^-64, zeros
// (the method returns +0 for x = -0), infinities and NaNs take __fdiv_rn.
// Powers of two divide exactly as a multiply by 2^-k.
#pragma once

#include <cuda_runtime.h>

namespace bfs {

// hi = RN(1/D); lo = the remainder (1 - D hi) / D rounded to float.  D hi has
// at most 24 + 32 significant bits, so 1 - D hi is exact in double.
template <int D>
struct RecipSplit {
    static constexpr float hi = 1.0f / static_cast<float>(D);
    static constexpr float lo =
        static_cast<float>((1.0 - static_cast<double>(D) * static_cast<double>(hi)) / static_cast<double>(D));
};

// |x| in [2^-64, +inf): bits of |x| minus those of 2^-64, unsigned compare.
__device__ __forceinline__ bool split_div_safe(float x) {
    return (__float_as_uint(x) & 0x7fffffffu) - 0x1f800000u < 0x7f800000u - 0x1f800000u;
}

// RN(x / D), bit-identical to __fdiv_rn(x, D) for every x.
template <int D>
__device__ __forceinline__ float div_const(float x) {
    static_assert(D >= 1, "divisor must be positive");
    if constexpr ((D & (D - 1)) == 0) {
        return __fmul_rn(x, 1.0f / static_cast<float>(D));   // 1/D exact: same real value
    } else {
        if (split_div_safe(x))
            return __fmaf_rn(x, RecipSplit<D>::hi, __fmul_rn(x, RecipSplit<D>::lo));
        return __fdiv_rn(x, static_cast<float>(D));
    }
}

// RN(x / d) for a divisor that is a compile-time constant after unrolling
// (d = 2..8 take div_const; anything else __fdiv_rn).
__device__ __forceinline__ float div_small(float x, int d) {
    switch (d) {
        case 2: return div_const<2>(x);
        case 3: return div_const<3>(x);
        case 4: return div_const<4>(x);
        case 5: return div_const<5>(x);
        case 6: return div_const<6>(x);
        case 7: return div_const<7>(x);
        case 8: return div_const<8>(x);
        default: return __fdiv_rn(x, static_cast<float>(d));
    }
}

}  // namespace bfs
