// Device helpers shared by the tensor-core Legendre kernels (legendre_tc.cu, legendre_ck.cu):
// the healpy alm index, the FP64 seed of a Legendre / Wigner-d row, coefficient-table
// loads, the f16 hi/lo operand split and the bounded mbarrier wait with abort flag.
#pragma once

#include <math.h>
#include <stdint.h>

#include "tc_common.cuh"

namespace gm {
namespace ltc {

constexpr double kBig = 2.037035976334486e90;      // 2^300
constexpr double kShrink = 2.409919865102884e-181; // 2^-600

struct Coef {
    double alpha, beta, c0;
};

__device__ __forceinline__ int64_t alm_idx(int64_t lmax, int64_t l, int64_t m)
{
    return m * (2 * lmax + 1 - m) / 2 + l;
}

__device__ __forceinline__ void seed_lane(const double *__restrict__ sd, double lsin, double lcos,
                                          double &v, int &k)
{
    double f = sd[0];
    if (sd[2] != 0.0) f += sd[2] * lcos;
    if (sd[3] != 0.0) f += sd[3] * lsin;
    if (!(f > -1.0e300)) {
        v = 0.0;
        k = 0;
        return;
    }
    int kk = 0;
    if (f < -300.0) kk = (int)floor((f + 300.0) / 600.0);
    v = sd[1] * exp2(f - 600.0 * (double)kk);
    k = kk;
}

// Binary-exponent carry, applied once per 8 steps: a lane still below 2^-300 (k < 0) is
// renormalised when it passes 2^300 (growth over 8 steps stays far below 2^700).
__device__ __forceinline__ void rescale(double &v, double &vp, int &k)
{
    if (k < 0 && fabs(v) > kBig) {
        v *= kShrink;
        vp *= kShrink;
        ++k;
    }
}

// Coefficient table entries are 32 bytes: (alpha, beta) then (c0, 0), so one 16-byte load
// fetches (alpha, beta).
__device__ __forceinline__ Coef load_coef(const double *__restrict__ tab, int64_t idx)
{
    const double2 ab = __ldg(reinterpret_cast<const double2 *>(tab) + 2 * idx);
    Coef c;
    c.alpha = ab.x;
    c.beta = ab.y;
    c.c0 = __ldg(tab + 4 * idx + 2);
    return c;
}

// Operands are f16 hi/lo pairs (22 significant bits; the products hi*hi + hi*lo + lo*hi
// run as three kind::f16 MMAs).  The generated rows are bounded by sqrt((2l+1)/4pi); the
// right-hand-side and alm images are scaled by a power of two so their largest entry sits
// near 2^13.
__device__ __forceinline__ void pack8(const float (&v)[8], uint4 &hi, uint4 &lo)
{
    tc::split_f16x2(v[0], v[1], hi.x, lo.x);
    tc::split_f16x2(v[2], v[3], hi.y, lo.y);
    tc::split_f16x2(v[4], v[5], hi.z, lo.z);
    tc::split_f16x2(v[6], v[7], hi.w, lo.w);
}

__device__ __forceinline__ void sts128(uint32_t addr, const uint4 &v)
{
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z),
                 "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ double sgn_of(int sp) { return sp > 0 ? 1.0 : (sp < 0 ? -1.0 : 0.0); }

__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, volatile int *abort,
                                              int *err)
{
    if (*abort) return false;
    if (tc::mbar_wait(bar, parity)) return true;
    *abort = 1;
    atomicExch(err, 1);
    return false;
}

}  // namespace ltc
}  // namespace gm
