// PCG32 (M. E. O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically Good
// Algorithms for Random Number Generation", 2014): 64-bit LCG state, XSH-RR output.
#ifndef ARC_PCG32_H_
#define ARC_PCG32_H_

#include <stdint.h>

#ifdef __CUDACC__
#define ARC_HD __host__ __device__
#else
#define ARC_HD
#endif

typedef struct arc_pcg32 {
    uint64_t state;
    uint64_t inc;
} arc_pcg32;

static inline ARC_HD uint32_t arc_pcg32_next(arc_pcg32* r) {
    const uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

static inline ARC_HD void arc_pcg32_seed(arc_pcg32* r, uint64_t initstate, uint64_t initseq) {
    r->state = 0u;
    r->inc = (initseq << 1u) | 1u;
    arc_pcg32_next(r);
    r->state += initstate;
    arc_pcg32_next(r);
}

// Uniform float in [0, 1) with 24 random bits.
static inline ARC_HD float arc_pcg32_float(arc_pcg32* r) {
    return (float)(arc_pcg32_next(r) >> 8) * (1.0f / 16777216.0f);
}

// Counter-based uniform float in [0, 1) for tree node `node` under `seed`: one PCG32 output of
// the stream (seed, node).  Used for the stochastic cluster representative, which the
// reference draws from a default-seeded host mt19937 (bvh.cu:27-28, 694-697).
static inline ARC_HD float arc_node_random(uint32_t seed, uint32_t node) {
    arc_pcg32 r;
    arc_pcg32_seed(&r, (uint64_t)seed, (uint64_t)node);
    return arc_pcg32_float(&r);
}

#endif  // ARC_PCG32_H_
