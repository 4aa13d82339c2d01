// mc_guide.cuh - the guiding distribution shared by the MLP kernels and the
// guided shade kernel: parameter layout, input encoding, and the 8-lobe von
// Mises-Fisher mixture (density and sampling).
#pragma once
#include <math.h>
#include <stdint.h>

#include "mc_abi.h"

#ifndef MC_GD
#define MC_GD __device__ __forceinline__
#endif

namespace mc {
namespace guide {

constexpr int kIn = MC_GUIDE_INPUTS;     // 144
constexpr int kHid = MC_GUIDE_HIDDEN;    // 64
constexpr int kOut = MC_GUIDE_OUTPUTS;   // 40
constexpr int kOutPad = 48;              // output rows padded to a multiple of 16
constexpr int kLobes = MC_GUIDE_LOBES;   // 8
constexpr int kFreqs = 12;

// flat FP32 parameter offsets (W[out][in] row-major)
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kHid * kIn;
constexpr int oW2 = oB1 + kHid;
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;
constexpr int oB3 = oW3 + kHid * kHid;
constexpr int oW4 = oB3 + kHid;
constexpr int oB4 = oW4 + kOut * kHid;
constexpr int kParams = oB4 + kOut;
static_assert(kParams == MC_GUIDE_PARAM_COUNT, "parameter layout");

// BF16 weight blob (elements): every layer's weights W[out][in] with the bias
// folded in: each layer's input gains a 16-column block [1, 1, 0, ...] and
// its weight rows the matching block [hi, lo, 0, ...], hi = bf16(b) and
// lo = bf16(b - hi), so the MMA adds the bias (to about 2^-17 of it) and the
// forward epilogues only apply ReLU. W4 is padded to 48 rows. The kernels read
// the same rows MN-major as the backward pass's W operands (dH = dZ W).
constexpr int kInK = kIn + 16;           // 160
constexpr int kHidK = kHid + 16;         // 80
constexpr int bI1 = 0;
constexpr int bI2 = bI1 + kHid * kInK;
constexpr int bI3 = bI2 + kHid * kHidK;
constexpr int bI4 = bI3 + kHid * kHidK;
constexpr int kBlobAll = bI4 + kOutPad * kHidK;

// log-concentration range: kappa in [0.01, 1000]
constexpr float kLogKappaMin = -4.60517019f;
constexpr float kLogKappaMax = 6.90775528f;
constexpr float kTwoPi = 6.28318530718f;

// Inputs: coordinate c (0..2 position in [0,1], 3..5 direction), frequency f:
// in[24c + 2f] = sin(pi 2^f x), in[24c + 2f + 1] = cos(pi 2^f x).
// Frequencies 0 and 6 of a coordinate are evaluated directly, the five after
// each by the double-angle identities sin 2a = 2 sin a cos a, cos 2a =
// (cos a - sin a)(cos a + sin a). Squaring the unit complex number cos a +
// i sin a doubles its error (plus one rounding), so five doublings stay
// within about 4e-6 of the direct values, far below the BF16 spacing (2^-8
// near 1) the network reads the inputs in.
MC_GD void encode_coord(float x, float* out24) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float s, c;
        sincospif(x * (half ? 64.0f : 1.0f), &s, &c);
        out24[12 * half] = s;
        out24[12 * half + 1] = c;
#pragma unroll
        for (int j = 1; j < 6; j++) {
            const float s2 = 2.0f * s * c;
            const float c2 = (c - s) * (c + s);
            s = s2;
            c = c2;
            out24[12 * half + 2 * j] = s;
            out24[12 * half + 2 * j + 1] = c;
        }
    }
}

// von Mises-Fisher density on the unit sphere at cosine c to the mean:
// kappa / (2 pi (1 - exp(-2 kappa))) * exp(kappa (c - 1)).
MC_GD float vmf_pdf(float kappa, float c) {
    return kappa / (kTwoPi * (1.0f - expf(-2.0f * kappa))) * expf(kappa * (c - 1.0f));
}

// Mixture stored as weights[8], unit means[8][3], kappa[8].
MC_GD float mixture_pdf(const float* m, float wx, float wy, float wz) {
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; k++) {
        float c = m[8 + 3 * k] * wx + m[9 + 3 * k] * wy + m[10 + 3 * k] * wz;
        q += m[k] * vmf_pdf(m[32 + k], c);
    }
    return q;
}

// Orthonormal basis around a unit vector (Duff et al., "Building an
// Orthonormal Basis, Revisited", JCGT 2017).
MC_GD void onb(float nx, float ny, float nz, float* t, float* b) {
    float sign = copysignf(1.0f, nz);
    float a = -1.0f / (sign + nz);
    float bb = nx * ny * a;
    t[0] = 1.0f + sign * nx * nx * a; t[1] = sign * bb; t[2] = -sign * nx;
    b[0] = bb; b[1] = sign + ny * ny * a; b[2] = -ny;
}

// Samples a lobe by u0, then a direction of that vMF (inversion of the
// cosine's distribution, Jakob, "Numerically stable sampling of the von
// Mises Fisher distribution on S^2", 2012).
MC_GD void mixture_sample(const float* m, float u0, float u1, float u2, float* dir) {
    int k = kLobes - 1;
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < kLobes; i++) {
        acc += m[i];
        if (u0 < acc) {
            k = i;
            break;
        }
    }
    const float kappa = m[32 + k];
    float w = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kappa)) / kappa;
    w = fminf(1.0f, fmaxf(-1.0f, w));
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    float t[3], b[3];
    const float mx = m[8 + 3 * k], my = m[9 + 3 * k], mz = m[10 + 3 * k];
    onb(mx, my, mz, t, b);
    const float lx = s * cp, ly = s * sp;
    dir[0] = t[0] * lx + b[0] * ly + mx * w;
    dir[1] = t[1] * lx + b[1] * ly + my * w;
    dir[2] = t[2] * lx + b[2] * ly + mz * w;
}

}  // namespace guide
}  // namespace mc
