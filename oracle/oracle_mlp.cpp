// oracle_mlp.cpp -- CPU restatement of the project's learned gradient
// surrogate.  TEST INFRASTRUCTURE ONLY: the parity tests load it as the
// test oracle of the device MLP kernels; the product library never links it.
//
// No reference counterpart (the surrogate is this project's addition), so
// parity is anchored on the mathematics: the FP64 mode is checked against
// central finite differences of the loss, and the BF16 mode rounds the same
// intermediate values to bfloat16 (round to nearest, ties to even, on the
// upper 16 bits of the binary32 value) as the device kernels do:
//   xb  = bf16((theta - in_mean) / in_scale)                     (binary32 arithmetic)
//   z1  = xb W1b^T + b1;   a1b = bf16(silu(z1));  s1b = bf16(silu'(z1))
//   z2  = a1b W2b^T + b2;  a2b = bf16(silu(z2));  s2b = bf16(silu'(z2))
//   y   = a2b W3b^T + b3;  output = y * out_scale + out_mean
//   t   = (g - out_mean) / out_scale;  loss = sum (y - t)^2 / B
//   dyb = bf16(2 (y - t) / B);  dz2b = bf16((dyb W3b) * s2b);  dz1b = bf16((dz2b W2b) * s1b)
//   dW3 = dyb^T a2b, dW2 = dz2b^T a1b, dW1 = dz1b^T xb, db = column sums.
// Sums are accumulated in FP64 (the device accumulates in FP32 on the tensor
// cores, so the two agree to FP32 accumulation error plus rare one-ulp BF16
// flips of an intermediate value).
#include "oracle_mlp.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace oracle_mlp {

Layout Layout::make(int P) {
    Layout L;
    L.P = P;
    L.Pp = ((P + 15) / 16) * 16;
    L.w1 = 0;
    L.b1 = L.w1 + (int64_t)kH * L.Pp;
    L.w2 = L.b1 + kH;
    L.b2 = L.w2 + (int64_t)kH * kH;
    L.w3 = L.b2 + kH;
    L.b3 = L.w3 + (int64_t)L.Pp * kH;
    L.total = L.b3 + L.Pp;
    return L;
}

namespace {

// bfloat16 rounding of a binary32 value (round to nearest even), returned as binary32.
inline float bf16_round(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) {  // Inf / NaN: keep (quiet NaN)
        if (u & 0x007fffffu) u |= 0x00400000u;
        u &= 0xffff0000u;
    } else {
        u += 0x7fffu + ((u >> 16) & 1u);
        u &= 0xffff0000u;
    }
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

struct Round {
    bool on;
    double operator()(double v) const { return on ? (double)bf16_round((float)v) : v; }
};

double silu(double z) { return z / (1.0 + std::exp(-z)); }
double dsilu(double z) {
    const double s = 1.0 / (1.0 + std::exp(-z));
    return s * (1.0 + z * (1.0 - s));
}

// Weights as doubles, BF16-rounded in BF16 mode.
struct Weights {
    Layout L;
    std::vector<double> w1, b1, w2, b2, w3, b3;
    Weights(const float* params, int P, Round rd) : L(Layout::make(P)) {
        auto take = [&](std::vector<double>& v, int64_t off, int64_t n, bool round) {
            v.resize(n);
            for (int64_t i = 0; i < n; ++i) v[i] = round ? rd(params[off + i]) : (double)params[off + i];
        };
        take(w1, L.w1, (int64_t)kH * L.Pp, true);
        take(b1, L.b1, kH, false);
        take(w2, L.w2, (int64_t)kH * kH, true);
        take(b2, L.b2, kH, false);
        take(w3, L.w3, (int64_t)L.Pp * kH, true);
        take(b3, L.b3, L.Pp, false);
    }
};

// Activations of one row.
struct Row {
    std::vector<double> x, a1, s1, a2, s2, y;
};

void row_forward(const Weights& W, const float* norm, const float* theta, Round rd, Row& r) {
    const int P = W.L.P, Pp = W.L.Pp;
    r.x.assign(Pp, 0.0);
    for (int j = 0; j < P; ++j) {
        const float v = (theta[j] - norm[j]) / norm[P + j];  // binary32, as on the device
        r.x[j] = rd(v);
    }
    r.a1.assign(kH, 0.0); r.s1.assign(kH, 0.0); r.a2.assign(kH, 0.0); r.s2.assign(kH, 0.0);
    for (int h = 0; h < kH; ++h) {
        double z = 0.0;
        for (int j = 0; j < Pp; ++j) z += r.x[j] * W.w1[(size_t)h * Pp + j];
        z += W.b1[h];
        r.a1[h] = rd(silu(z));
        r.s1[h] = rd(dsilu(z));
    }
    for (int h = 0; h < kH; ++h) {
        double z = 0.0;
        for (int k = 0; k < kH; ++k) z += r.a1[k] * W.w2[(size_t)h * kH + k];
        z += W.b2[h];
        r.a2[h] = rd(silu(z));
        r.s2[h] = rd(dsilu(z));
    }
    r.y.assign(Pp, 0.0);
    for (int j = 0; j < P; ++j) {
        double z = 0.0;
        for (int k = 0; k < kH; ++k) z += r.a2[k] * W.w3[(size_t)j * kH + k];
        r.y[j] = z + W.b3[j];
    }
}

}  // namespace

struct Evaluator::Impl {
    Round rd;
    Weights W;
    std::vector<float> norm;
    Impl(const float* params, const float* nrm, int P, int bf16)
        : rd{bf16 != 0}, W(params, P, Round{bf16 != 0}), norm(nrm, nrm + 4 * P) {}
};

Evaluator::Evaluator(const float* params, const float* norm, int P, int bf16)
    : impl_(new Impl(params, norm, P, bf16)) {}
Evaluator::~Evaluator() { delete impl_; }

void Evaluator::operator()(const float* theta, float* out) const {
    const int P = impl_->W.L.P;
    const float* norm = impl_->norm.data();
    Row r;
    row_forward(impl_->W, norm, theta, impl_->rd, r);
    for (int j = 0; j < P; ++j) out[j] = (float)(r.y[j] * norm[3 * P + j] + norm[2 * P + j]);
}

void forward(const float* params, const float* norm, int P, const float* x, int64_t n, float* out, int bf16) {
    const Evaluator ev(params, norm, P, bf16);
    for (int64_t i = 0; i < n; ++i) ev(x + i * P, out + i * P);
}

}  // namespace oracle_mlp

using namespace oracle_mlp;

extern "C" {

int64_t orc_mlp_num_weights(int32_t P) { return Layout::make(P).total; }

// Surrogate gradient at n positions (n x P).  norm: in_mean, in_scale,
// out_mean, out_scale (P each).
void orc_mlp_forward(const float* params, const float* norm, int32_t P, const float* x, int64_t n, float* out,
                     int32_t bf16) {
    forward(params, norm, P, x, n, out, bf16);
}

// Loss and weight gradient (flat layout, FP64) of one batch: pair rows
// index[0..batch), rows outside [0, num_pairs) skipped.
void orc_mlp_loss_gradient(const float* params, const float* norm, int32_t P, const float* theta, const float* grad,
                           int64_t num_pairs, const int32_t* index, int32_t batch, double* weight_grad, double* loss,
                           int32_t bf16) {
    const Round rd{bf16 != 0};
    const Weights W(params, P, rd);
    const Layout& L = W.L;
    const int Pp = L.Pp;
    std::memset(weight_grad, 0, sizeof(double) * (size_t)L.total);
    double lsum = 0.0;
    Row r;
    std::vector<double> dy(Pp), dz2(kH), dz1(kH);
    for (int b = 0; b < batch; ++b) {
        const int64_t row = index[b];
        if (row < 0 || row >= num_pairs) continue;
        row_forward(W, norm, theta + row * P, rd, r);
        std::fill(dy.begin(), dy.end(), 0.0);
        for (int j = 0; j < P; ++j) {
            const float t = (grad[row * P + j] - norm[2 * P + j]) / norm[3 * P + j];  // binary32
            const double e = r.y[j] - (double)t;
            lsum += e * e;
            dy[j] = rd(2.0 * e / (double)batch);
        }
        for (int h = 0; h < kH; ++h) {
            double s = 0.0;
            for (int j = 0; j < Pp; ++j) s += dy[j] * W.w3[(size_t)j * kH + h];
            dz2[h] = rd(s * r.s2[h]);
        }
        for (int k = 0; k < kH; ++k) {
            double s = 0.0;
            for (int h = 0; h < kH; ++h) s += dz2[h] * W.w2[(size_t)h * kH + k];
            dz1[k] = rd(s * r.s1[k]);
        }
        for (int j = 0; j < Pp; ++j) {
            for (int h = 0; h < kH; ++h) weight_grad[L.w3 + (size_t)j * kH + h] += dy[j] * r.a2[h];
            weight_grad[L.b3 + j] += dy[j];
        }
        for (int h = 0; h < kH; ++h) {
            for (int k = 0; k < kH; ++k) weight_grad[L.w2 + (size_t)h * kH + k] += dz2[h] * r.a1[k];
            weight_grad[L.b2 + h] += dz2[h];
            for (int j = 0; j < Pp; ++j) weight_grad[L.w1 + (size_t)h * Pp + j] += dz1[h] * r.x[j];
            weight_grad[L.b1 + h] += dz1[h];
        }
    }
    *loss = lsum / (double)batch;
}

}  // extern "C"
