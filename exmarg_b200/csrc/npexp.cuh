// numpy's float32 exp on the device, bit for bit.
//
// The reference ranks arrival times by a float32 score formed with numpy's exp
// (exmarg/search/gather.py:407).  numpy (2.x, contiguous float32 arrays on AVX2 / AVX-512 hosts) computes it
// with its SIMD kernel simd_exp_f32 (numpy/_core/src/umath/loops_exponent_log.dispatch.c.src): a Cody-Waite
// reduction by ln 2 and a degree-5 / degree-2 rational minimax approximation.  It is not correctly rounded,
// and neither is CUDA's expf, and the two disagree in the last bit for many inputs; a one-ulp change of a
// score near the n_loud-th place swaps which time is walked.  This function performs numpy's published
// steps in the same order with explicitly rounded operations (no contraction), so the score -- and
// hence the selection -- is the reference's.  Checked against np.exp on every float32 input by the
// host restatement in the test suite's oracle, and on the device through exm_np_exp32.
#pragma once

__device__ __forceinline__ float exm_pow2f(int j)   // 2^j for -126 <= j <= 127
{
    return __int_as_float((j + 127) << 23);
}

__device__ __forceinline__ float exm_np_expf(float x)
{
    if (x != x) return x;
    if (x >= 88.72283935546875f) return __int_as_float(0x7f800000);
    if (x <= -103.97208404541015625f) return 0.0f;
    // k = rint(x log2 e): float32 product, rounded to an integer by adding and removing 1.5 * 2^23
    const float k = __fsub_rn(__fadd_rn(__fmul_rn(x, 0x1.715476p+0f), 0x1.8p+23f), 0x1.8p+23f);
    // r = x - k ln 2 in two fused steps (ln 2 split into a short high part and the remainder)
    float r = __fmaf_rn(k, -6.93145752e-1f, x);
    r = __fmaf_rn(k, -1.42860677e-6f, r);
    float num = __fmaf_rn(5.082762527590693718096e-04f, r, 6.757896990527504603057e-03f);
    num = __fmaf_rn(num, r, 5.114512081637298353406e-02f);
    num = __fmaf_rn(num, r, 2.473615434895520810817e-01f);
    num = __fmaf_rn(num, r, 7.257664613233124478488e-01f);
    num = __fmaf_rn(num, r, 9.999999999980870924916e-01f);
    float den = __fmaf_rn(2.159509375685829852307e-02f, r, -2.742335390411667452936e-01f);
    den = __fmaf_rn(den, r, 1.0f);
    const float p = __fdiv_rn(num, den);
    // p * 2^k with a single rounding (k lies in [-150, 128]): a split keeps each power of two normal
    const int ki = (int)k;
    if (ki > 127) return __fmul_rn(__fmul_rn(p, exm_pow2f(ki - 64)), exm_pow2f(64));
    if (ki < -120) return __fmul_rn(__fmul_rn(p, exm_pow2f(ki + 64)), exm_pow2f(-64));
    return __fmul_rn(p, exm_pow2f(ki));
}
