// mc_guide_oracle.cpp - FP64 restatement of the path-guiding MLP.
//
// TEST INFRASTRUCTURE (see mc_oracle.h): the library never calls it. The
// guiding MLP has no counterpart in the reference; this file states the
// network, the vMF-mixture loss and its gradient directly from their
// definitions so that the tensor-core kernels can be checked:
//   * forward: encoding sin/cos(pi 2^f x), f = 0..11, of the normalized
//     position and the direction; 144 -> 64 -> 64 -> 64 (ReLU) -> 40;
//     outputs -> softmax weights, normalized means, kappa = exp(clamp(.));
//   * loss: sum_i w_i * -log q(next_i), q the mixture density;
//   * gradient by back-propagation in FP64 (checked against finite
//     differences by the tests).
// With emulate_bf16 != 0 the values the GPU rounds to BF16 (weights, encoded
// inputs, hidden activations, output and hidden-layer gradients) are rounded
// the same way (round to nearest even after rounding to FP32), so the GPU
// result differs only by its FP32 accumulation order.
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "mc_oracle.h"

namespace {

constexpr int IN = MC_GUIDE_INPUTS, HID = MC_GUIDE_HIDDEN, OUT = MC_GUIDE_OUTPUTS, LOBES = MC_GUIDE_LOBES;
constexpr int oW1 = 0, oB1 = oW1 + HID * IN, oW2 = oB1 + HID, oB2 = oW2 + HID * HID, oW3 = oB2 + HID,
              oB3 = oW3 + HID * HID, oW4 = oB3 + HID, oB4 = oW4 + OUT * HID, NP = oB4 + OUT;
static_assert(NP == MC_GUIDE_PARAM_COUNT, "parameter layout");
constexpr double kLogKappaMin = (double)-4.60517019f, kLogKappaMax = (double)6.90775528f;

float bf16_round(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return x;
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}
double rb(double v, bool bf) { return bf ? (double)bf16_round((float)v) : v; }

// coordinates exactly as the GPU forms them (FP32 subtract and multiply)
void coords(const float* pos, const float* dir, const float* lo, const float* inv, float* c) {
    for (int i = 0; i < 3; i++) {
        volatile float d = pos[i] - lo[i];
        c[i] = d * inv[i];
        c[3 + i] = dir[i];
    }
}

void encode(const float* c6, bool bf, double* x) {
    for (int c = 0; c < 6; c++)
        for (int f = 0; f < 12; f++) {
            const double y = (double)(c6[c] * (float)(1 << f));
            double s = std::sin(M_PI * y), co = std::cos(M_PI * y);
            x[24 * c + 2 * f] = rb(s, bf);
            x[24 * c + 2 * f + 1] = rb(co, bf);
        }
}

struct Fwd {
    double x[IN], z1[HID], h1[HID], z2[HID], h2[HID], z3[HID], h3[HID], y[OUT];
};

void forward(const double* P, const std::vector<double>& W, bool bf, Fwd& F) {
    auto layer = [&](const double* in, int nin, int ow, int ob, int nout, double* z, double* h) {
        for (int o = 0; o < nout; o++) {
            double s = 0.0;
            for (int i = 0; i < nin; i++) s += W[ow + o * nin + i] * in[i];
            z[o] = s + P[ob + o];
            if (h) h[o] = rb(z[o] > 0.0 ? z[o] : 0.0, bf);
        }
    };
    layer(F.x, IN, oW1, oB1, HID, F.z1, F.h1);
    layer(F.h1, HID, oW2, oB2, HID, F.z2, F.h2);
    layer(F.h2, HID, oW3, oB3, HID, F.z3, F.h3);
    layer(F.h3, HID, oW4, oB4, OUT, F.y, nullptr);
}

// anc: the anchor offset added to every raw lobe mean (zero when unanchored)
void mixture(const double* y, const double* anc, double* m) {
    double mx = y[0];
    for (int k = 1; k < LOBES; k++) mx = std::max(mx, y[k]);
    double s = 0.0;
    for (int k = 0; k < LOBES; k++) s += std::exp(y[k] - mx);
    for (int k = 0; k < LOBES; k++) {
        m[k] = std::exp(y[k] - mx) / s;
        double a = y[8 + 3 * k] + anc[0], b = y[9 + 3 * k] + anc[1], c = y[10 + 3 * k] + anc[2];
        double l = std::sqrt(a * a + b * b + c * c);
        if (l > 1e-20) {
            m[8 + 3 * k] = a / l; m[9 + 3 * k] = b / l; m[10 + 3 * k] = c / l;
        } else {
            m[8 + 3 * k] = 0; m[9 + 3 * k] = 0; m[10 + 3 * k] = 1;
        }
        m[32 + k] = std::exp(std::min(std::max(y[32 + k], kLogKappaMin), kLogKappaMax));
    }
}

double vmf(double kappa, double c) { return kappa / (2.0 * M_PI * (1.0 - std::exp(-2.0 * kappa))) * std::exp(kappa * (c - 1.0)); }

// -W log q(w) and d/dy
double loss_grad(const double* y, const double* anc, const double* w, double W, double* dy) {
    double m[OUT];
    mixture(y, anc, m);
    double len[LOBES], vk[LOBES], cs[LOBES], q = 0.0;
    for (int k = 0; k < LOBES; k++) {
        double a = y[8 + 3 * k] + anc[0], b = y[9 + 3 * k] + anc[1], c = y[10 + 3 * k] + anc[2];
        len[k] = std::sqrt(a * a + b * b + c * c);
        if (!(len[k] > 1e-20)) len[k] = 0.0;
        cs[k] = m[8 + 3 * k] * w[0] + m[9 + 3 * k] * w[1] + m[10 + 3 * k] * w[2];
        vk[k] = vmf(m[32 + k], cs[k]);
        q += m[k] * vk[k];
    }
    q = std::max(q, 1e-30);
    for (int k = 0; k < LOBES; k++) {
        const double kap = m[32 + k];
        const double r = m[k] * vk[k] / q;
        dy[k] = -W * (r - m[k]);
        const bool clamped = y[32 + k] < kLogKappaMin || y[32 + k] > kLogKappaMax;
        const double dlogv = 1.0 / kap - 2.0 / std::expm1(2.0 * kap) + cs[k] - 1.0;
        dy[32 + k] = clamped ? 0.0 : -W * r * kap * dlogv;
        const double g = len[k] > 0.0 ? -W * r * kap / len[k] : 0.0;
        for (int j = 0; j < 3; j++) dy[8 + 3 * k + j] = g * (w[j] - cs[k] * m[8 + 3 * k + j]);
    }
    return W != 0.0 ? -W * std::log(q) : 0.0;
}

std::vector<double> weights(const double* P, bool bf) {
    std::vector<double> W(P, P + NP);
    if (bf)
        for (int i = 0; i < NP; i++) {
            const bool isBias = (i >= oB1 && i < oW2) || (i >= oB2 && i < oW3) || (i >= oB3 && i < oW4) || i >= oB4;
            if (!isBias) W[i] = rb(P[i], true);
        }
    return W;
}

// Anchored lobes (flags bit 1; bit 2 turns the direction back): every raw
// mean is offset by 1.5 times the direction input, FP32 products as the GPU's.
void anchor_of(int flags, const float* dir, double* anc) {
    const float s = (flags & 2) ? ((flags & 4) ? -1.5f : 1.5f) : 0.0f;
    for (int j = 0; j < 3; j++) anc[j] = (double)(s * dir[j]);
}

}  // namespace

extern "C" {

int orc_guide_forward(const double* params, const float* queries, int n, const float* lo, const float* inv,
                      int flags, double* mix) {
    const bool bf = (flags & 1) != 0;
    std::vector<double> W = weights(params, bf);
    Fwd F;
    for (int i = 0; i < n; i++) {
        const float* Q = queries + (size_t)i * 6;
        float c6[6];
        coords(Q, Q + 3, lo, inv, c6);
        encode(c6, bf, F.x);
        forward(params, W, bf, F);
        double anc[3];
        anchor_of(flags, Q + 3, anc);
        mixture(F.y, anc, mix + (size_t)i * OUT);
    }
    return 0;
}

int orc_guide_loss_grad(const double* params, const float* records, int n, const float* lo, const float* inv,
                        int flags, double* grad, double* loss) {
    const bool bf = (flags & 1) != 0;
    std::vector<double> W = weights(params, bf);
    std::memset(grad, 0, sizeof(double) * NP);
    double total = 0.0;
    Fwd F;
    for (int r = 0; r < n; r++) {
        const float* R = records + (size_t)r * MC_GUIDE_RECORD_FLOATS;
        float c6[6];
        coords(R, R + 3, lo, inv, c6);
        encode(c6, bf, F.x);
        forward(params, W, bf, F);
        const double w[3] = {R[6], R[7], R[8]};
        double dy[OUT];
        double anc[3];
        anchor_of(flags, R + 3, anc);
        total += loss_grad(F.y, anc, w, (double)R[9], dy);
        for (int o = 0; o < OUT; o++) dy[o] = rb(dy[o], bf);
        // layer 4
        double dh3[HID] = {0};
        for (int o = 0; o < OUT; o++) {
            grad[oB4 + o] += dy[o];
            for (int i = 0; i < HID; i++) {
                grad[oW4 + o * HID + i] += dy[o] * F.h3[i];
                dh3[i] += dy[o] * W[oW4 + o * HID + i];
            }
        }
        // hidden layers
        auto back = [&](const double* dh, const double* z, const double* hin, int nin, int ow, int ob, double* dhin) {
            double dz[HID];
            for (int o = 0; o < HID; o++) dz[o] = rb(z[o] > 0.0 ? dh[o] : 0.0, bf);
            if (dhin) std::memset(dhin, 0, sizeof(double) * nin);
            for (int o = 0; o < HID; o++) {
                grad[ob + o] += dz[o];
                for (int i = 0; i < nin; i++) {
                    grad[ow + o * nin + i] += dz[o] * hin[i];
                    if (dhin) dhin[i] += dz[o] * W[ow + o * nin + i];
                }
            }
        };
        double dh2[HID], dh1[HID];
        back(dh3, F.z3, F.h2, HID, oW3, oB3, dh2);
        back(dh2, F.z2, F.h1, HID, oW2, oB2, dh1);
        back(dh1, F.z1, F.x, IN, oW1, oB1, nullptr);
    }
    if (loss) *loss = total;
    return 0;
}

}  // extern "C"
