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
double orc_mlp_triplet_grad(const float* w1, const float* b1, const float* w2, const float* b2, const uint8_t* a,
                            const uint8_t* p, const uint8_t* ng, uint32_t batch, float margin, double* dw1,
                            double* db1, double* dw2, double* db2) {
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
        double dap = 0, dan = 0;
        for (int c = 0; c < 128; ++c) {
            const double u = z[c] - z[128 + c], v = z[c] - z[256 + c];
            dap += u * u / 4;
            dan += v * v / 4;
        }
        const double l = margin + dap - dan;
        std::fill(dz.begin(), dz.end(), 0.0);
        if (l > 0) {
            loss += l;
            for (int c = 0; c < 128; ++c) {
                const double u = z[c] - z[128 + c], v = z[c] - z[256 + c];
                dz[c] = (u - v) / 2 / batch;
                dz[128 + c] = -u / 2 / batch;
                dz[256 + c] = v / 2 / batch;
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

}  // extern "C"
