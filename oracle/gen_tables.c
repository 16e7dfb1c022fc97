/*
 * ORACLE -- test infrastructure only (inputs of the CPU baselines and the tests).
 *
 * The seeded synthetic node table of exmarg_b200.synth.gen_table_node in plain C:
 * the same float32 operations in the same order (built with -ffp-contract=off, so
 * no FMA is formed) and the same 32-bit hash, giving bit-identical tables, in
 * parallel over the host cores.
 */
#include <stdint.h>

static inline uint32_t mix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    return h ^ (h >> 16);
}

/* out (ntau, nphif, nb, nd) float32; M (nb, nd), P (nphif), Q (ntau) */
void oracle_gen_node(float *out, const float *M, const float *P, const float *Q, float S, uint32_t seed, uint32_t k,
                     int ntau, int nphif, int nb, int nd)
{
    const float scale = 2.384185791015625e-07f; /* 2^-22 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int r = 0; r < ntau; ++r)
        for (int c = 0; c < nphif; ++c) {
            float *o = out + ((int64_t)r * nphif + c) * nb * nd;
            const uint32_t h0 = (seed * 0x9E3779B1u) ^ (k * 0x85EBCA77u);
            const uint32_t hr = mix32(h0 ^ ((uint32_t)r * 0xC2B2AE3Du));
            const uint32_t hc = mix32(hr ^ ((uint32_t)c * 0x27D4EB2Fu));
            for (int b = 0; b < nb; ++b) {
                const uint32_t hb = mix32(hc ^ ((uint32_t)b * 0x165667B1u));
                for (int d = 0; d < nd; ++d) {
                    float v = M[b * nd + d] * P[c];
                    v = v * Q[r];
                    v = v - S;
                    const uint32_t h = mix32(hb ^ ((uint32_t)d * 0xD3A2646Cu));
                    const float pert = (float)((int32_t)(h & 0xFFFFu) - 32768) * scale;
                    o[b * nd + d] = v + pert;
                }
            }
        }
}
