// CPU oracle (double precision) of the learned hash MLP. TEST INFRASTRUCTURE ONLY: the tests
// check the CUDA forward/backward kernels against it; the product never calls it.
//
// No reference counterpart (the learned hash replaces cascade hashing's random projection):
//   x      = desc / 64                                  (128)
//   hpre   = W1 x + b1,  h = bf16(relu(hpre))           (256)   W1 bf16 [256][128], b1 f32
//   o      = W2 h + b2                                  (128)   W2 bf16 [128][256], b2 f32
//   bits   = [o > 0]; bucket key byte s = bits 8s..8s+7; code = all 128 bits
// Training loss on triplets (anchor a, positive p, negative n), z = tanh(o):
//   D(u,v) = sum_c (z_u,c - z_v,c)^2 / 4,   L = mean_b max(0, margin + D(a,p) - D(a,n))
// Gradients flow through the bf16 rounding of h as through the identity.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {

static inline double bf16_round(double v) {
    // round-to-nearest-even to bfloat16 (8-bit mantissa) through float
    float f = float(v);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u = (u + 0x7FFFu + lsb) & 0xFFFF0000u;
    std::memcpy(&f, &u, 4);
    return double(f);
}

// w1 [256*128], w2 [128*256] are the bf16 weights given as float values.
void orc_mlp_forward(const float* w1, const float* b1, const float* w2, const float* b2, const uint8_t* desc,
                     uint32_t n, float* out /* n x 128 */, uint32_t* codes /* n x 4, may be null */) {
    std::vector<double> h(256);
    for (uint32_t i = 0; i < n; ++i) {
        const uint8_t* x = desc + size_t(i) * 128;
        for (int j = 0; j < 256; ++j) {
            double s = b1[j];
            for (int d = 0; d < 128; ++d) s += double(w1[j * 128 + d]) * (double(x[d]) / 64.0);
            h[j] = bf16_round(s > 0 ? s : 0);
        }
        uint32_t c4[4] = {0, 0, 0, 0};
        for (int c = 0; c < 128; ++c) {
            double s = b2[c];
            for (int j = 0; j < 256; ++j) s += double(w2[c * 256 + j]) * h[j];
            out[size_t(i) * 128 + c] = float(s);
            if (s > 0) c4[c / 32] |= 1u << (c % 32);
        }
        if (codes) std::memcpy(codes + size_t(i) * 4, c4, 16);
    }
}

// Loss and gradients (dW1 [256*128], db1 [256], dW2 [128*256], db2 [128]) of one triplet batch.
//   kind 0: triplet hinge on all 128 channels (above).
//   kind 1: bucket-key loss on channels 0..47 (6 tables of 8 bits) plus the triplet hinge on the
//           code channels 48..127. Per table s and pair (u, v): q_k = max((1 + z_u,k z_v,k) / 2, 1e-4),
//           A_s(u, v) = prod_{k in s} q_k (soft probability that the 8-bit keys agree);
//           loss += -log(A_s(a, p) + 1e-6) + lambda * A_s(a, n).
double orc_mlp_loss_grad(const float* w1, const float* b1, const float* w2, const float* b2, const uint8_t* a,
                         const uint8_t* p, const uint8_t* ng, uint32_t batch, float margin, int kind, float lambda,
                         double* dw1, double* db1, double* dw2, double* db2) {
    std::memset(dw1, 0, sizeof(double) * 256 * 128);
    std::memset(db1, 0, sizeof(double) * 256);
    std::memset(dw2, 0, sizeof(double) * 128 * 256);
    std::memset(db2, 0, sizeof(double) * 128);
    double loss = 0;
    std::vector<double> hp(3 * 256), h(3 * 256), z(3 * 128), dz(3 * 128), dh(256);
    for (uint32_t b = 0; b < batch; ++b) {
        const uint8_t* xs[3] = {a + size_t(b) * 128, p + size_t(b) * 128, ng + size_t(b) * 128};
        for (int r = 0; r < 3; ++r) {
            for (int j = 0; j < 256; ++j) {
                double s = b1[j];
                for (int d = 0; d < 128; ++d) s += double(w1[j * 128 + d]) * (double(xs[r][d]) / 64.0);
                hp[r * 256 + j] = s;
                h[r * 256 + j] = bf16_round(s > 0 ? s : 0);
            }
            for (int c = 0; c < 128; ++c) {
                double s = b2[c];
                for (int j = 0; j < 256; ++j) s += double(w2[c * 256 + j]) * h[r * 256 + j];
                z[r * 128 + c] = std::tanh(s);
            }
        }
        const int c0 = kind == 1 ? 48 : 0;  // first channel of the hinge term
        double dap = 0, dan = 0;
        for (int c = c0; c < 128; ++c) {
            const double u = z[c] - z[128 + c], v = z[c] - z[256 + c];
            dap += u * u / 4;
            dan += v * v / 4;
        }
        const double l = margin + dap - dan;
        std::fill(dz.begin(), dz.end(), 0.0);
        if (l > 0) {
            loss += l;
            for (int c = c0; c < 128; ++c) {
                const double u = z[c] - z[128 + c], v = z[c] - z[256 + c];
                dz[c] = (u - v) / 2 / batch;
                dz[128 + c] = -u / 2 / batch;
                dz[256 + c] = v / 2 / batch;
            }
        }
        if (kind == 1) {
            for (int t = 0; t < 6; ++t) {
                double aap = 1, aan = 1;
                for (int k = 8 * t; k < 8 * t + 8; ++k) {
                    aap *= std::max((1 + z[k] * z[128 + k]) / 2, 1e-4);
                    aan *= std::max((1 + z[k] * z[256 + k]) / 2, 1e-4);
                }
                loss += -std::log(aap + 1e-6) + lambda * aan;
                for (int k = 8 * t; k < 8 * t + 8; ++k) {
                    const double qap = std::max((1 + z[k] * z[128 + k]) / 2, 1e-4);
                    const double qan = std::max((1 + z[k] * z[256 + k]) / 2, 1e-4);
                    // d q / d z_u = z_v / 2 where q is not clamped
                    const double cap = (1 + z[k] * z[128 + k]) / 2 > 1e-4 ? -(aap / (aap + 1e-6)) / qap * 0.5 : 0.0;
                    const double can = (1 + z[k] * z[256 + k]) / 2 > 1e-4 ? lambda * aan / qan * 0.5 : 0.0;
                    dz[k] += (cap * z[128 + k] + can * z[256 + k]) / batch;
                    dz[128 + k] += cap * z[k] / batch;
                    dz[256 + k] += can * z[k] / batch;
                }
            }
        }
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 128; ++c) dz[r * 128 + c] *= 1 - z[r * 128 + c] * z[r * 128 + c];  // do
            for (int c = 0; c < 128; ++c) {
                db2[c] += dz[r * 128 + c];
                for (int j = 0; j < 256; ++j) dw2[c * 256 + j] += dz[r * 128 + c] * h[r * 256 + j];
            }
            for (int j = 0; j < 256; ++j) {
                double s = 0;
                for (int c = 0; c < 128; ++c) s += double(w2[c * 256 + j]) * dz[r * 128 + c];
                dh[j] = hp[r * 256 + j] > 0 ? s : 0;
                db1[j] += dh[j];
                for (int d = 0; d < 128; ++d) dw1[j * 128 + d] += dh[j] * (double(xs[r][d]) / 64.0);
            }
        }
    }
    return loss / batch;
}

double orc_mlp_triplet_grad(const float* w1, const float* b1, const float* w2, const float* b2, const uint8_t* a,
                            const uint8_t* p, const uint8_t* ng, uint32_t batch, float margin, double* dw1,
                            double* db1, double* dw2, double* db2) {
    return orc_mlp_loss_grad(w1, b1, w2, b2, a, p, ng, batch, margin, 0, 0.f, dw1, db1, dw2, db2);
}

}  // extern "C"
