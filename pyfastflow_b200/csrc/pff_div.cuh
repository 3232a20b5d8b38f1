// Exact f32 division by a per-launch constant (the cell size dx) without the
// general IEEE division sequence, for the stencils whose cost is instructions.
//
// Markstein's correction (P. Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; also Muller et al.,
// Handbook of Floating-Point Arithmetic, on division with a fused multiply-add):
// with y = RN(1/dx), q0 = RN(m y) is within 1.5 ulp of m/dx; one correction
// q1 = RN(q0 + RN(m - dx q0) y) lands within one ulp, and a second one gives RN(m/dx)
// exactly, by Markstein's theorem, as long as nothing underflows or overflows, which
// the range [mlo, mhi] of m ensures.  Outside that range callers use the IEEE
// division.  pff_receivers_div_selfcheck compares the quotient with the IEEE
// division for every float in the range.
#pragma once
#include <algorithm>
#include <cuda_runtime.h>

namespace pff {

struct DivC {
    float dx, y, mlo, mhi;  // y = RN(1/dx); the exact range of the numerator: [mlo, mhi]
};

inline DivC make_divc(float dx)
{
    DivC c;
    c.dx = dx;
    c.y = 1.0f / dx;  // IEEE single division on the host: RN(1/dx)
    // q = m/dx and m itself within [2^-100, 2^100]: no intermediate leaves the normal range
    c.mlo = std::max(dx * 0x1p-100f, 0x1p-100f);
    c.mhi = std::min(dx * 0x1p100f, 0x1p100f);
    return c;
}

__device__ __forceinline__ float div_markstein(float m, const DivC &c)
{
    float q = __fmul_rn(m, c.y);
    float r = __fmaf_rn(-c.dx, q, m);
    q = __fmaf_rn(r, c.y, q);
    r = __fmaf_rn(-c.dx, q, m);
    return __fmaf_rn(r, c.y, q);
}

// RN(m / dx) for any m: the corrected quotient inside its exact range, else IEEE.
__device__ __forceinline__ float div_dx(float m, const DivC &c)
{
    return (m >= c.mlo && m <= c.mhi) ? div_markstein(m, c) : __fdiv_rn(m, c.dx);
}

}  // namespace pff
