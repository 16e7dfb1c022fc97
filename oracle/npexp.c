/* ORACLE -- test infrastructure only.
 *
 * numpy's float32 exp, restated in plain C: the function the reference's time selection uses to score
 * arrival times (exmarg/search/gather.py:407, xp.exp(2.0 * lqL) + xp.exp(2.0 * mx) on float32 arrays).
 *
 * numpy 2.3.5 (the version the reference runs with here) dispatches np.exp on contiguous float32 arrays to
 * its SIMD kernel simd_exp_f32 (numpy/_core/src/umath/loops_exponent_log.dispatch.c.src, AVX512F and AVX2
 * builds; constants in npy_simd_data.h).  That kernel is not correctly rounded, so a correctly rounded exp
 * (or CUDA's expf) differs from it in the last bit for many inputs, and the ranking of scores near the
 * n_loud-th place can change.  Its published algorithm:
 *   1. x >= 88.72283935546875 -> +inf; x <= -103.97208404541015625 -> 0; NaN -> NaN
 *   2. k = rint(x * log2(e)), the product rounded to float32 and k rounded by adding and subtracting 1.5*2^23
 *   3. Cody-Waite reduction with two fused multiply-adds: r = fma(k, -ln2_hi, x), r = fma(k, -ln2_lo, r)
 *   4. exp(r) ~ P(r) / Q(r): P of degree 5, Q of degree 2 (minimax), Horner by fused multiply-adds,
 *      then one IEEE float32 division
 *   5. the quotient scaled by 2^k (AVX-512 scalef: one rounding, also into the subnormal range)
 * The device restatement (exmarg_b200/csrc/npexp.cuh) performs the same operations; tests check both
 * bit for bit against np.exp.
 */
#include <math.h>
#include <stdint.h>

static float npexp_scale(float p, int k)
{
    /* p * 2^k with one rounding: the powers of two used are normal floats, the first product is exact */
    if (k > 127) return (p * ldexpf(1.0f, k - 64)) * ldexpf(1.0f, 64);
    if (k < -120) return (p * ldexpf(1.0f, k + 64)) * ldexpf(1.0f, -64);
    return p * ldexpf(1.0f, k);
}

float oracle_npexp32(float x)
{
    const float xmax = 88.72283935546875f, xmin = -103.97208404541015625f;
    const float log2e = 0x1.715476p+0f, magic = 0x1.8p+23f;
    const float c1 = -6.93145752e-1f, c2 = -1.42860677e-6f;
    const float p0 = 9.999999999980870924916e-01f, p1 = 7.257664613233124478488e-01f,
                p2 = 2.473615434895520810817e-01f, p3 = 5.114512081637298353406e-02f,
                p4 = 6.757896990527504603057e-03f, p5 = 5.082762527590693718096e-04f;
    const float q0 = 1.0f, q1 = -2.742335390411667452936e-01f, q2 = 2.159509375685829852307e-02f;
    if (x != x) return x;
    if (x >= xmax) return INFINITY;
    if (x <= xmin) return 0.0f;
    volatile float t = x * log2e;        /* float32 product, no contraction */
    volatile float u = t + magic;
    const float k = u - magic;
    float r = fmaf(k, c1, x);
    r = fmaf(k, c2, r);
    float num = fmaf(p5, r, p4);
    num = fmaf(num, r, p3);
    num = fmaf(num, r, p2);
    num = fmaf(num, r, p1);
    num = fmaf(num, r, p0);
    float den = fmaf(q2, r, q1);
    den = fmaf(den, r, q0);
    return npexp_scale(num / den, (int)k);
}

void oracle_npexp32_array(const float *x, float *y, int64_t n)
{
    for (int64_t i = 0; i < n; ++i) y[i] = oracle_npexp32(x[i]);
}
