// mc_rng.cuh - the two random-number modes of the render path.
//
// MC_RNG_PHILOX: counter-based Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
//   "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from the
//   paper: 10 rounds of two 32x32->64 multiplies with the published multipliers
//   and Weyl key increments. Draw k of (pixel p, sample s) is word (k & 3) of
//   philox(counter = (k >> 2, s, p, 0), key = (seed_lo, seed_hi)), mapped to
//   ((word >> 9) + 0.5) * 2^-23 in (0, 1). A path keeps only its draw index.
// MC_RNG_XORWOW: the reference's generator, curand XORWOW seeded per pixel with
//   curand_init(seed, pixel, 0) and carried across samples (PT:2865-2871); the
//   curand device functions are called, not re-implemented.
#pragma once
#include <curand_kernel.h>
#include <stdint.h>

#include "mc_math.cuh"

namespace mc {

MC_HD void philox4x32_10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32), lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

MC_HD float word_to_uniform(uint32_t w) { return ((float)(w >> 9) + 0.5f) * 1.1920928955078125e-07f; }

struct PhiloxRng {
    uint32_t k0, k1, sample, pixel, draw;
    uint32_t block;   // index of the cached 4-word block, 0xffffffff = none
    uint32_t w0, w1, w2, w3;
    MC_D void init(uint32_t seedLo, uint32_t seedHi, uint32_t s, uint32_t p, uint32_t d) {
        k0 = seedLo; k1 = seedHi; sample = s; pixel = p; draw = d; block = 0xffffffffu;
    }
    MC_D float uniform() {
        uint32_t blk = draw >> 2;
        if (blk != block) {
            uint32_t c0 = blk, c1 = sample, c2 = pixel, c3 = 0u;
            philox4x32_10(c0, c1, c2, c3, k0, k1);
            w0 = c0; w1 = c1; w2 = c2; w3 = c3;
            block = blk;
        }
        uint32_t sel = draw & 3u;
        uint32_t w = sel == 0 ? w0 : (sel == 1 ? w1 : (sel == 2 ? w2 : w3));
        draw++;
        return word_to_uniform(w);
    }
};

struct XorwowRng {
    curandState st;
    MC_D float uniform() { return curand_uniform(&st); }
};

}  // namespace mc
