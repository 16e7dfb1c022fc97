// numpy's default_rng(seed).integers(0, n, size) reproduced bit for bit, on the host
// (seeding) and on the device (the stream).  Published algorithms, restated:
//  * SeedSequence (numpy.random.SeedSequence, O'Neill's seed_seq_fe hash-mix
//    entropy pool, pool of 4 uint32, INIT/MULT constants of that design),
//  * PCG64 = PCG XSL RR 128/64 (O'Neill 2014): 128-bit LCG, output
//    rotr64(hi ^ lo, hi >> 58) of the stepped state; numpy seeds it with
//    state = 0, inc = 2 initseq + 1, step, state += initstate, step,
//  * the 32-bit draws numpy's bounded generator consumes are the low then the
//    high half of each 64-bit output,
//  * Lemire's nearly-divisionless bounded integers (arXiv:1805.10941): draw x,
//    m = x * n, reject while (m mod 2^32) < (2^32 mod n), return m >> 32.
// The reference draws its random arrival times this way
// (exmarg/search/gather.py:397), so the device visits the same times.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define EXM_HD __host__ __device__ __forceinline__
#else
#define EXM_HD inline
#endif

typedef unsigned __int128 exm_u128;

#define EXM_PCG_MULT ((((exm_u128)0x2360ED051FC65DA4ull) << 64) | (exm_u128)0x4385DF649FCCF645ull)

struct exm_pcg {
    exm_u128 state, inc;
};

EXM_HD void exm_pcg_step(exm_pcg &g) { g.state = g.state * EXM_PCG_MULT + g.inc; }

EXM_HD uint64_t exm_pcg_output(exm_u128 s)
{
    const uint64_t hi = (uint64_t)(s >> 64), lo = (uint64_t)s;
    const uint64_t x = hi ^ lo;
    const unsigned r = (unsigned)(hi >> 58);
    return (x >> r) | (x << ((64u - r) & 63u));
}

// state after `delta` more steps (O'Neill's LCG jump-ahead, O(log delta))
EXM_HD void exm_pcg_advance(exm_pcg &g, uint64_t delta)
{
    exm_u128 acc_mult = 1, acc_plus = 0, cur_mult = EXM_PCG_MULT, cur_plus = g.inc;
    while (delta) {
        if (delta & 1) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1;
    }
    g.state = acc_mult * g.state + acc_plus;
}

// host: the PCG64 state numpy's default_rng(seed) starts from (seed >= 0)
inline exm_pcg exm_pcg_from_seed(uint64_t seed)
{
    const uint32_t INIT_A = 0x43b0d7e5u, MULT_A = 0x931e8875u, INIT_B = 0x8b51f9ddu, MULT_B = 0x58f38dedu;
    const uint32_t MIX_L = 0xca01f9ddu, MIX_R = 0x4973f715u;
    uint32_t words[2];
    int nw = 0;
    uint64_t s = seed;
    do {
        words[nw++] = (uint32_t)s;
        s >>= 32;
    } while (s && nw < 2);
    uint32_t hc = INIT_A;
    auto hashmix = [&hc, MULT_A](uint32_t v) {
        v ^= hc;
        hc *= MULT_A;
        v *= hc;
        v ^= v >> 16;
        return v;
    };
    auto mix = [MIX_L, MIX_R](uint32_t x, uint32_t y) {
        uint32_t r = MIX_L * x - MIX_R * y;
        r ^= r >> 16;
        return r;
    };
    uint32_t pool[4];
    for (int i = 0; i < 4; ++i) pool[i] = hashmix(i < nw ? words[i] : 0u);
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            if (a != b) pool[b] = mix(pool[b], hashmix(pool[a]));
    uint32_t hb = INIT_B, out[8];
    for (int i = 0; i < 8; ++i) {
        uint32_t v = pool[i & 3];
        v ^= hb;
        hb *= MULT_B;
        v *= hb;
        v ^= v >> 16;
        out[i] = v;
    }
    uint64_t w[4];
    for (int i = 0; i < 4; ++i) w[i] = (uint64_t)out[2 * i] | ((uint64_t)out[2 * i + 1] << 32);
    const exm_u128 initstate = ((exm_u128)w[0] << 64) | w[1];
    const exm_u128 initseq = ((exm_u128)w[2] << 64) | w[3];
    exm_pcg g;
    g.state = 0;
    g.inc = (initseq << 1) | 1;
    exm_pcg_step(g);
    g.state += initstate;
    exm_pcg_step(g);
    return g;
}
