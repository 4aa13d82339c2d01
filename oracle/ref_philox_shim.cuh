// Counter-based RNG shim for the oracle harness (test infrastructure).
//
// Included before the reference translation unit in the "philox" oracle build.
// It defines curand_kernel.h's include guard and the four curand names the
// reference uses (curandState, curand_init, curand_uniform,
// curand_uniform_double; path_tracer.cu:36, 2870, and the samplers), so the
// unmodified reference draws from the same counter-based stream as the
// library's MC_RNG_PHILOX mode: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), key = the 64-bit seed,
// counter = (draw >> 2, sample, pixel, 0), word = draw & 3,
// uniform = ((word >> 9) + 0.5) * 2^-23 in (0, 1).
// The harness sets `sample` and zeroes `draw` before each sample, which makes
// the stream a function of (pixel, sample, draw index) only.
#pragma once
#define CURAND_KERNEL_H_ 1
#include <cuda_runtime.h>
#include <stdint.h>

struct mcrefPhiloxState {
    unsigned int pixel;
    unsigned int seed_lo;
    unsigned int seed_hi;
    unsigned int sample;
    unsigned int draw;
};
typedef mcrefPhiloxState curandState;

__host__ __device__ inline void mcref_philox4x32_10(unsigned int c[4], unsigned int k0, unsigned int k1) {
    for (int round = 0; round < 10; ++round) {
        unsigned long long p0 = (unsigned long long)0xD2511F53u * c[0];
        unsigned long long p1 = (unsigned long long)0xCD9E8D57u * c[2];
        unsigned int hi0 = (unsigned int)(p0 >> 32), lo0 = (unsigned int)p0;
        unsigned int hi1 = (unsigned int)(p1 >> 32), lo1 = (unsigned int)p1;
        unsigned int n0 = hi1 ^ c[1] ^ k0;
        unsigned int n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__host__ __device__ inline void curand_init(unsigned long long seed, unsigned long long subsequence,
                                            unsigned long long /*offset*/, curandState* state) {
    state->pixel = (unsigned int)subsequence;
    state->seed_lo = (unsigned int)seed;
    state->seed_hi = (unsigned int)(seed >> 32);
    state->sample = 0;
    state->draw = 0;
}

__host__ __device__ inline unsigned int mcref_philox_next(curandState* state) {
    unsigned int c[4] = {state->draw >> 2, state->sample, state->pixel, 0u};
    mcref_philox4x32_10(c, state->seed_lo, state->seed_hi);
    unsigned int word = c[state->draw & 3u];
    state->draw += 1u;
    return word;
}

__host__ __device__ inline float curand_uniform(curandState* state) {
    unsigned int word = mcref_philox_next(state);
    return ((float)(word >> 9) + 0.5f) * 1.1920928955078125e-07f;  // 2^-23
}

__host__ __device__ inline double curand_uniform_double(curandState* state) {
    unsigned int a = mcref_philox_next(state) >> 5;
    unsigned int b = mcref_philox_next(state) >> 6;
    return ((double)a * 67108864.0 + (double)b + 0.5) * (1.0 / 9007199254740992.0);
}
