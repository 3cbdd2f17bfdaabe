/* CPU restatement of the surrogate MLP (forward, loss, backward).
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the tensor-core kernels in
 * dem_mph_b200/csrc/dmph_mlp.cu; nothing in the product calls it.  The
 * surrogate has no counterpart in the reference (its parity is unpinned);
 * this file states the network the GPU computes:
 *
 *   64 -> 128 -> 128 -> 128 -> 16, ReLU after the three hidden layers,
 *   parameters per layer l: W_l [out][in] then b_l [out], consecutive;
 *   operands rounded to BF16 (round to nearest even) before every product,
 *   hidden activations stored as BF16 after the ReLU, FP32 outputs;
 *   loss = sum over rows and the first n_valid outputs of (y - t)^2 / (rows * n_valid);
 *   gradients of the weights and biases in the same layout as the parameters,
 *   with every backward operand (dY, the gradient through each ReLU) rounded
 *   to BF16 as the GPU stores them.
 *
 * Sums run in double, so results differ from the GPU's FP32 tensor-core
 * accumulation by rounding only.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define IN 64
#define HID 128
#define OUT 16

static const int L_IN[4] = {IN, HID, HID, HID};
static const int L_OUT[4] = {HID, HID, HID, OUT};

static float bf16(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

int mlp_oracle_param_count(void)
{
    int n = 0;
    for (int l = 0; l < 4; l++) n += L_OUT[l] * L_IN[l] + L_OUT[l];
    return n;
}

static int layer_offset(int l)
{
    int n = 0;
    for (int k = 0; k < l; k++) n += L_OUT[k] * L_IN[k] + L_OUT[k];
    return n;
}

/* activations of one row: a[0] input (bf16), a[1..3] hidden (bf16), y output */
static void forward_row(const float *P, const float *x, float a[4][HID], float *y)
{
    for (int k = 0; k < IN; k++) a[0][k] = bf16(x[k]);
    for (int l = 0; l < 4; l++) {
        const float *W = P + layer_offset(l);
        const float *b = W + L_OUT[l] * L_IN[l];
        for (int o = 0; o < L_OUT[l]; o++) {
            double s = 0.0;
            for (int k = 0; k < L_IN[l]; k++) s += (double)bf16(W[o * L_IN[l] + k]) * (double)a[l][k];
            const float z = (float)s + b[o];
            if (l < 3)
                a[l + 1][o] = bf16(z > 0.f ? z : 0.f);
            else
                y[o] = z;
        }
    }
}

void mlp_oracle_forward(const float *P, int n, const float *X, float *Y)
{
    float a[4][HID];
    for (int i = 0; i < n; i++) forward_row(P, X + (size_t)i * IN, a, Y + (size_t)i * OUT);
}

double mlp_oracle_grad(const float *P, int n, const float *X, const float *T, int n_valid, float *G)
{
    const int np = mlp_oracle_param_count();
    double *g = (double *)calloc((size_t)np, sizeof(double));
    double loss = 0.0;
    const double scale = 2.0 / ((double)n * n_valid);
    float a[4][HID], y[OUT], d[HID], dn[HID];
    for (int i = 0; i < n; i++) {
        forward_row(P, X + (size_t)i * IN, a, y);
        for (int o = 0; o < OUT; o++) {
            const float df = o < n_valid ? y[o] - T[(size_t)i * OUT + o] : 0.f;
            loss += (double)df * df;
            d[o] = bf16((float)(df * scale));
        }
        for (int l = 3; l >= 0; l--) {
            const int off = layer_offset(l), in = L_IN[l], out = L_OUT[l];
            for (int o = 0; o < out; o++) {
                for (int k = 0; k < in; k++) g[off + o * in + k] += (double)d[o] * a[l][k];
                g[off + out * in + o] += d[o];
            }
            if (l == 0) break;
            for (int k = 0; k < in; k++) {
                double s = 0.0;
                for (int o = 0; o < out; o++) s += (double)bf16(P[off + o * in + k]) * d[o];
                dn[k] = a[l][k] > 0.f ? bf16((float)s) : 0.f;
            }
            memcpy(d, dn, sizeof(float) * in);
        }
    }
    for (int p = 0; p < np; p++) G[p] = (float)g[p];
    free(g);
    return loss / ((double)n * n_valid);
}
