/*
 * mupsi_mlp_oracle.c -- CPU oracle of the surrogate-mean MLP (test infrastructure).
 *
 * The surrogate has no counterpart in the reference renderer; this file is the
 * checker for the GPU's tensor-core forward and backward kernels. It evaluates
 * the network defined in include/mupsi_gpu.h (mupsi_mlp_desc) in FP64, rounding
 * to BF16 at exactly the points where the GPU kernels store BF16 operands:
 * the Fourier features, the weights, the hidden activations h1..h4, and the
 * pre-activation gradients dz1..dz4 that feed the tensor-core products (the
 * hidden layers' bias gradients are sums of the BF16 dz, as on the GPU). Sums
 * are FP64 (the GPU accumulates in FP32), so GPU and oracle differ by FP32
 * accumulation rounding plus rare BF16 rounding-boundary flips.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "mupsi_oracle.h"

#define NF 48
#define NG 96
#define NH 64

/* BF16 round to nearest even of an FP32 value (NaN not expected here). */
static double bf16(double x) {
  float f = (float)x;
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

typedef struct {
  const float *W1, *b1, *W[3], *b[3], *w5, *b5;
} mo_mlp_view;

static mo_mlp_view view(const float* params) {
  mo_mlp_view v;
  v.W1 = params;
  v.b1 = params + 6144;
  for (int l = 0; l < 3; ++l) {
    v.W[l] = params + 6208 + l * 4160;
    v.b[l] = params + 6208 + l * 4160 + 4096;
  }
  v.w5 = params + 18688;
  v.b5 = params + 18752;
  return v;
}

/* Forward pass of one point; keeps what the backward pass needs. */
typedef struct {
  double g[NG];      /* bf16 Fourier features */
  double h[4][NH];   /* bf16 activations h1..h4 */
  unsigned char m[4][NH];
  double y;          /* network output before y_scale */
} mo_mlp_act;

static void forward1(const mo_mlp_view* v, const float* fourier, const float* center, const float* p,
                     mo_mlp_act* a) {
  /* the GPU computes the phases in FP32: x = p - center, u_f = B_f . x */
  const float x0 = p[0] - center[0], x1 = p[1] - center[1], x2 = p[2] - center[2];
  for (int f = 0; f < NF; ++f) {
    const float u = fourier[3 * f] * x0 + (fourier[3 * f + 1] * x1 + fourier[3 * f + 2] * x2);
    a->g[f] = bf16(sin((double)u));
    a->g[NF + f] = bf16(cos((double)u));
  }
  const double* in = a->g;
  for (int l = 0; l < 4; ++l) {
    const int K = l == 0 ? NG : NH;
    const float* W = l == 0 ? v->W1 : v->W[l - 1];
    const float* b = l == 0 ? v->b1 : v->b[l - 1];
    for (int j = 0; j < NH; ++j) {
      double z = 0.0;
      for (int i = 0; i < K; ++i) z += bf16(W[j * K + i]) * in[i];
      z = (double)(float)z + (double)b[j];
      a->m[l][j] = z > 0.0;
      a->h[l][j] = bf16(z > 0.0 ? z : 0.0);
    }
    in = a->h[l];
  }
  double y = 0.0;
  for (int j = 0; j < NH; ++j) y += bf16(v->w5[j]) * a->h[3][j];
  a->y = y + (double)v->b5[0];
}

void mo_mlp_forward(const float* params, const float* fourier, const float* center, float y_scale, int64_t n,
                    const float* p, float* out) {
  mo_mlp_view v = view(params);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    mo_mlp_act a;
    forward1(&v, fourier, center, p + 3 * i, &a);
    out[i] = (float)((double)y_scale * a.y);
  }
}

/* Gradient of L = (1/n) sum_i (y_i - target_i / y_scale)^2 over the parameter
 * vector (layout of mupsi_mlp_desc.params) and L itself. */
void mo_mlp_grad(const float* params, const float* fourier, const float* center, float y_scale, int64_t n,
                 const float* p, const float* target, double* grad, double* loss) {
  mo_mlp_view v = view(params);
  memset(grad, 0, sizeof(double) * MUPSI_MLP_PARAMS);
  double L = 0.0;
  for (int64_t s = 0; s < n; ++s) {
    mo_mlp_act a;
    forward1(&v, fourier, center, p + 3 * s, &a);
    const double r = a.y - (double)target[s] / (double)y_scale;
    L += r * r;
    const double dy = 2.0 * r / (double)n;
    /* output layer (CUDA cores on the GPU) */
    for (int j = 0; j < NH; ++j) grad[18688 + j] += dy * a.h[3][j];
    grad[18752] += dy;
    double dh[NH], dz[NH];
    for (int j = 0; j < NH; ++j) dh[j] = dy * bf16(v.w5[j]);
    for (int l = 3; l >= 0; --l) {
      const int K = l == 0 ? NG : NH;
      const float* W = l == 0 ? v.W1 : v.W[l - 1];
      double* gW = grad + (l == 0 ? 0 : 6208 + (l - 1) * 4160);
      double* gb = grad + (l == 0 ? 6144 : 6208 + (l - 1) * 4160 + 4096);
      const double* in = l == 0 ? a.g : a.h[l - 1];
      for (int j = 0; j < NH; ++j) {
        const double d = a.m[l][j] ? (double)(float)dh[j] : 0.0;
        dz[j] = bf16(d);
        gb[j] += dz[j]; /* the GPU's bias gradient is the product with a column of ones */
      }
      for (int j = 0; j < NH; ++j)
        for (int i = 0; i < K; ++i) gW[j * K + i] += dz[j] * in[i];
      if (l > 0) {
        for (int i = 0; i < NH; ++i) {
          double acc = 0.0;
          for (int j = 0; j < NH; ++j) acc += dz[j] * bf16(W[j * NH + i]);
          dh[i] = acc;
        }
      }
    }
  }
  *loss = L / (double)n;
}
