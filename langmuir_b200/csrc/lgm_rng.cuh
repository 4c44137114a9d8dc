// lgm_rng.cuh -- the counter-based random stream of the kMC step.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Every draw of a step is addressed by a counter
// instead of a position in one serial stream, so a carrier's draws do not
// depend on the order threads run in:
//   key = {seed, replica},  counter = {step, index, purpose, 0}
//   purpose 1/2: proposal / decision of electron `index`, 3/4: of hole `index`,
//   16 + k: electrode source k (0 eL, 1 eR, 2 hL, 3 hR) with index 0,
//   64 +: world set-up streams (index = draw number).
// Integers in [0, n): (w0 * n) >> 32.  Uniform [0, 1) with 53 bits:
// ((w_a >> 5) * 2^26 + (w_b >> 6)) / 2^53, (a, b) = (0, 1) for decisions and
// (1, 2) for sources.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define LGM_HD __host__ __device__ __forceinline__
#else
#define LGM_HD inline
#endif

namespace lgm {

enum : uint32_t {
    RNG_CHOOSE_E = 1, RNG_DECIDE_E = 2, RNG_CHOOSE_H = 3, RNG_DECIDE_H = 4,
    RNG_SOURCE = 16, RNG_SETUP = 64
};

struct Philox4 {
    uint32_t w[4];
};

LGM_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                             uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
    }
    Philox4 o;
    o.w[0] = c0; o.w[1] = c1; o.w[2] = c2; o.w[3] = c3;
    return o;
}

LGM_HD uint32_t uint_below(uint32_t w, uint32_t n) {
    return (uint32_t)(((uint64_t)w * n) >> 32);
}

LGM_HD double unit_double(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

}  // namespace lgm
