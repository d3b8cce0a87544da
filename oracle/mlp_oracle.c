/*
 * CPU oracle for the learned pivot proposer -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference has no learned pivot (its pivot is the first vertex of a
 * colour, src/scc_color.cc:64-93), so nothing here is pinned to reference
 * output: the network, its gradient and the features are restated from their
 * definitions, and tests/test_oracle.py pins the gradient below against central
 * finite differences of the loss below.
 *
 * Network: x[8] -> relu(x W1 + b1)[64] -> relu(h1 W2 + b2)[64] -> h2 . w3 + b3.
 * Parameter order: W1[8][64], b1[64], W2[64][64], b2[64], w3[64], b3 (4,801).
 * The engine uses the weights rounded to BF16 (round to nearest, ties to even),
 * so every function here rounds them the same way and accumulates in double.
 * With bf16_acts, the inputs and the first hidden layer are rounded to BF16 as
 * well (the tensor-core inference path stages them as BF16 MMA operands).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define IN 8
#define H 64
#define O_W1 0
#define O_B1 (O_W1 + IN * H)
#define O_W2 (O_B1 + H)
#define O_B2 (O_W2 + H * H)
#define O_W3 (O_B2 + H)
#define O_B3 (O_W3 + H)
#define NPARAM (O_B3 + 1)

/* BF16 keeps the upper 16 bits of an IEEE binary32; round to nearest even on
 * the dropped 16 bits (NaN stays NaN). */
float orc_bf16(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) {
        u |= 0x00400000u;
    } else {
        uint32_t lsb = (u >> 16) & 1u;
        u += 0x7FFFu + lsb;
    }
    u &= 0xFFFF0000u;
    float y;
    memcpy(&y, &u, 4);
    return y;
}

int32_t orc_mlp_num_params(void) { return NPARAM; }

static void rounded(const float* p, double* w) {
    for (int i = 0; i < NPARAM; ++i) w[i] = (double)orc_bf16(p[i]);
}

static double forward1(const double* w, const float* xin, int bf16_acts, double* h1, double* z2, double* h2) {
    double x[IN];
    for (int k = 0; k < IN; ++k) x[k] = bf16_acts ? (double)orc_bf16(xin[k]) : (double)xin[k];
    for (int j = 0; j < H; ++j) {
        double a = w[O_B1 + j];
        for (int k = 0; k < IN; ++k) a += x[k] * w[O_W1 + k * H + j];
        double h = a > 0.0 ? a : 0.0;
        h1[j] = bf16_acts ? (double)orc_bf16((float)h) : h;
    }
    double y = w[O_B3];
    for (int j = 0; j < H; ++j) {
        double a = w[O_B2 + j];
        for (int k = 0; k < H; ++k) a += h1[k] * w[O_W2 + k * H + j];
        z2[j] = a;
        h2[j] = a > 0.0 ? a : 0.0;
        y += h2[j] * w[O_W3 + j];
    }
    return y;
}

void orc_mlp_forward(const float* params, const float* x, int64_t n, int bf16_acts, double* y) {
    double w[NPARAM], h1[H], z2[H], h2[H];
    rounded(params, w);
    for (int64_t i = 0; i < n; ++i) y[i] = forward1(w, x + i * IN, bf16_acts, h1, z2, h2);
}

/* Mean squared error over n rows and its gradient w.r.t. the (BF16-rounded)
 * parameters; FP32-valued activations (no activation rounding). */
double orc_mlp_loss_grad(const float* params, const float* x, const float* t, int64_t n, double* grad) {
    double w[NPARAM], h1[H], z2[H], h2[H], d2[H];
    rounded(params, w);
    memset(grad, 0, sizeof(double) * NPARAM);
    double loss = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const float* xi = x + i * IN;
        double y = forward1(w, xi, 0, h1, z2, h2);
        double diff = y - (double)t[i];
        loss += diff * diff;
        double dy = 2.0 * diff / (double)n;
        grad[O_B3] += dy;
        for (int j = 0; j < H; ++j) {
            grad[O_W3 + j] += h2[j] * dy;
            d2[j] = z2[j] > 0.0 ? dy * w[O_W3 + j] : 0.0;
            grad[O_B2 + j] += d2[j];
        }
        for (int k = 0; k < H; ++k) {
            double a = 0.0;
            for (int j = 0; j < H; ++j) {
                grad[O_W2 + k * H + j] += h1[k] * d2[j];
                a += d2[j] * w[O_W2 + k * H + j];
            }
            double d1 = h1[k] > 0.0 ? a : 0.0;
            grad[O_B1 + k] += d1;
            for (int q = 0; q < IN; ++q) grad[O_W1 + q * H + k] += (double)xi[q] * d1;
        }
    }
    return loss / (double)n;
}

/* Loss with double parameters taken as given (no rounding): the central
 * finite differences that pin orc_mlp_loss_grad perturb these. */
double orc_mlp_loss(const double* w, const float* x, const float* t, int64_t n) {
    double h1[H], z2[H], h2[H];
    double loss = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double diff = forward1(w, x + i * IN, 0, h1, z2, h2) - (double)t[i];
        loss += diff * diff;
    }
    return loss / (double)n;
}

/* Features of vertex v (the engine's k_pivot_features): log1p of out-degree,
 * in-degree, their product, live out/in neighbours (cnt_* may be NULL: the
 * degrees stand in), the class size, the mean log1p-degree of the first 4
 * out-neighbours and the largest log1p-degree of the first 4 in-neighbours;
 * each rounded to BF16. */
void orc_pivot_features(const int32_t* begin, const int32_t* node_idx, const int32_t* r_begin,
                        const int32_t* r_node_idx, const int32_t* cnt_out, const int32_t* cnt_in, int32_t v,
                        int32_t class_size, float* f) {
    float od = (float)(begin[v + 1] - begin[v]), id = (float)(r_begin[v + 1] - r_begin[v]);
    f[0] = log1pf(od);
    f[1] = log1pf(id);
    f[2] = log1pf(od * id);
    f[3] = cnt_out ? log1pf((float)(cnt_out[v] > 0 ? cnt_out[v] : 0)) : f[0];
    f[4] = cnt_in ? log1pf((float)(cnt_in[v] > 0 ? cnt_in[v] : 0)) : f[1];
    f[5] = log1pf((float)class_size);
    float s = 0.f, mx = 0.f;
    int k = 0;
    for (int32_t e = begin[v]; e < begin[v + 1] && k < 4; ++e, ++k) {
        int32_t w = node_idx[e];
        s += log1pf((float)(begin[w + 1] - begin[w]));
    }
    f[6] = k ? s / (float)k : 0.f;
    k = 0;
    for (int32_t e = r_begin[v]; e < r_begin[v + 1] && k < 4; ++e, ++k) {
        int32_t u = r_node_idx[e];
        float d = log1pf((float)(r_begin[u + 1] - r_begin[u]));
        if (d > mx) mx = d;
    }
    f[7] = mx;
    for (int j = 0; j < IN; ++j) f[j] = orc_bf16(f[j]);
}
