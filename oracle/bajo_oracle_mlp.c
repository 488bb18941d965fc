/* bajo_oracle_mlp.c -- TEST INFRASTRUCTURE ONLY: FP64 restatement of the
 * path-guiding network (encoding, forward pass, vMF-mixture negative
 * log-likelihood and its gradient by backpropagation) that checks the
 * tensor-core kernels of the product library.  The guiding network is new on
 * this path (the reference has no counterpart), so this file is anchored on
 * its own published maths: one-blob encoding (Mueller et al., "Neural
 * Importance Sampling", 2019), the von Mises-Fisher density
 * kappa / (2 pi (1 - e^-2kappa)) exp(kappa (mu.w - 1)), softmax mixture
 * weights, and reverse-mode differentiation of a ReLU MLP; gradients are
 * additionally pinned by central finite differences in the tests.
 *
 * Features are computed in float with the same operation order as the CUDA
 * encoder (-ffp-contract=off here, -fmad=false there), so the feature rows
 * agree bit for bit before the kernels round them to half precision. */
#include <math.h>
#include <string.h>

#include "bajo_oracle.h"

#define IN 64
#define HID 64
#define OUT 20
#define OUTPAD 32
#define LAYER (HID * IN + HID)
#define POS_BINS 16
#define DIR_BINS 8

static int off_w(int l) { return l * LAYER; }
static int off_b(int l) { return l < 3 ? l * LAYER + HID * IN : 3 * LAYER + OUTPAD * HID; }

uint32_t bo_mlp_param_count(void) { return 3 * LAYER + OUTPAD * HID + OUTPAD; }

static void blob(float v, int bins, float* out) {
  if (v < 0.0f) v = 0.0f;
  if (v > 1.0f) v = 1.0f;
  float s = v * (float)bins - 0.5f;
  float fl = floorf(s);
  float f = s - fl;
  int i0 = (int)fl < 0 ? 0 : (int)fl;
  int i1 = (int)fl + 1 > bins - 1 ? bins - 1 : (int)fl + 1;
  for (int k = 0; k < bins; ++k) out[k] = (k == i0 ? 1.0f - f : 0.0f) + (k == i1 ? f : 0.0f);
}

static void octahedral(float nx, float ny, float nz, float* u, float* v) {
  float l1 = fabsf(nx) + fabsf(ny) + fabsf(nz);
  float x = l1 > 0.0f ? nx / l1 : 0.0f, y = l1 > 0.0f ? ny / l1 : 0.0f;
  if (nz < 0.0f) {
    float ax = fabsf(x), ay = fabsf(y);
    x = (1.0f - ay) * (x >= 0.0f ? 1.0f : -1.0f);
    y = (1.0f - ax) * (y >= 0.0f ? 1.0f : -1.0f);
  }
  *u = x * 0.5f + 0.5f;
  *v = y * 0.5f + 0.5f;
}

void bo_mlp_encode(const float* p, const float* n, const float* box, float* feat) {
  for (int a = 0; a < 3; ++a) {
    float ext = box[3 + a] - box[a];
    float v = ext > 0.0f ? (p[a] - box[a]) / ext : 0.5f;
    blob(v, POS_BINS, feat + a * POS_BINS);
  }
  float u, w;
  octahedral(n[0], n[1], n[2], &u, &w);
  blob(u, DIR_BINS, feat + 3 * POS_BINS);
  blob(w, DIR_BINS, feat + 3 * POS_BINS + DIR_BINS);
}

/* activations of one sample: a[0] = features, a[1..3] = hidden, o = outputs */
typedef struct {
  double a[4][64];
  double o[OUT];
} fwd_state;

static void forward_one(const double* P, const float* feat, fwd_state* s) {
  for (int k = 0; k < IN; ++k) s->a[0][k] = feat[k];
  for (int l = 0; l < 3; ++l) {
    const double* W = P + off_w(l);
    const double* b = P + off_b(l);
    for (int i = 0; i < HID; ++i) {
      double z = b[i];
      for (int k = 0; k < IN; ++k) z += W[i * IN + k] * s->a[l][k];
      s->a[l + 1][i] = z > 0.0 ? z : 0.0;
    }
  }
  const double* W = P + off_w(3);
  const double* b = P + off_b(3);
  for (int i = 0; i < OUT; ++i) {
    double z = b[i];
    for (int k = 0; k < HID; ++k) z += W[i * HID + k] * s->a[3][k];
    s->o[i] = z;
  }
}

void bo_mlp_forward_f64(const double* params, const float* pos, const float* nrm, const float* box, uint32_t n,
                        double* out20) {
  fwd_state s;
  float feat[IN];
  for (uint32_t i = 0; i < n; ++i) {
    bo_mlp_encode(pos + 3 * (size_t)i, nrm + 3 * (size_t)i, box, feat);
    forward_one(params, feat, &s);
    memcpy(out20 + (size_t)OUT * i, s.o, sizeof(s.o));
  }
}

/* mixture: mean m / len, len = sqrt(|m|^2 + 1e-12), kappa = exp(clamp(s, -2, 8)),
 * softmax weights */
static void mixture(const double* o, double pi[4], double mu[4][3], double kap[4], double len[4], double norm[4]) {
  double mx = -1e300, z = 0.0;
  for (int k = 0; k < 4; ++k) mx = o[5 * k + 4] > mx ? o[5 * k + 4] : mx;
  for (int k = 0; k < 4; ++k) {
    pi[k] = exp(o[5 * k + 4] - mx);
    z += pi[k];
  }
  for (int k = 0; k < 4; ++k) {
    pi[k] /= z;
    len[k] = sqrt(o[5 * k] * o[5 * k] + o[5 * k + 1] * o[5 * k + 1] + o[5 * k + 2] * o[5 * k + 2] + 1e-12);
    for (int a = 0; a < 3; ++a) mu[k][a] = o[5 * k + a] / len[k];
    double s = o[5 * k + 3];
    s = s < -2.0 ? -2.0 : (s > 8.0 ? 8.0 : s);
    kap[k] = exp(s);
    norm[k] = kap[k] / (2.0 * 3.14159265358979323846 * (-expm1(-2.0 * kap[k])));
  }
}

double bo_vmf_mixture_pdf(const double* out20, const float* dir) {
  double pi[4], mu[4][3], kap[4], len[4], norm[4], q = 0.0;
  mixture(out20, pi, mu, kap, len, norm);
  for (int k = 0; k < 4; ++k) {
    double c = mu[k][0] * dir[0] + mu[k][1] * dir[1] + mu[k][2] * dir[2];
    q += pi[k] * norm[k] * exp(kap[k] * (c - 1.0));
  }
  return q;
}

/* -w log pdf(dir) and d/d(outputs) */
static double nll_grad(const double* o, const float* dir, double w, double* g) {
  double pi[4], mu[4][3], kap[4], len[4], norm[4], v[4], c[4], q = 0.0;
  mixture(o, pi, mu, kap, len, norm);
  for (int k = 0; k < 4; ++k) {
    c[k] = mu[k][0] * dir[0] + mu[k][1] * dir[1] + mu[k][2] * dir[2];
    v[k] = norm[k] * exp(kap[k] * (c[k] - 1.0));
    q += pi[k] * v[k];
  }
  if (q < 1e-300) q = 1e-300;
  for (int k = 0; k < 4; ++k) {
    double r = pi[k] * v[k] / q;
    g[5 * k + 4] = w * (pi[k] - r);
    double dlogv = 1.0 - 2.0 * kap[k] * exp(-2.0 * kap[k]) / (-expm1(-2.0 * kap[k])) + kap[k] * (c[k] - 1.0);
    int clamped = o[5 * k + 3] < -2.0 || o[5 * k + 3] > 8.0;
    g[5 * k + 3] = clamped ? 0.0 : -w * r * dlogv;
    for (int a = 0; a < 3; ++a) g[5 * k + a] = -w * r * kap[k] * (dir[a] - mu[k][a] * c[k]) / len[k];
  }
  return -w * log(q);
}

double bo_mlp_loss_f64(const double* params, const float* pos, const float* nrm, const float* dir, const float* w,
                       uint32_t n, const float* box) {
  fwd_state s;
  float feat[IN];
  double loss = 0.0, g[OUT];
  for (uint32_t i = 0; i < n; ++i) {
    bo_mlp_encode(pos + 3 * (size_t)i, nrm + 3 * (size_t)i, box, feat);
    forward_one(params, feat, &s);
    loss += nll_grad(s.o, dir + 3 * (size_t)i, w[i], g);
  }
  return loss;
}

double bo_mlp_grad_f64(const double* params, const float* pos, const float* nrm, const float* dir, const float* w,
                       uint32_t n, const float* box, double* grad) {
  memset(grad, 0, sizeof(double) * bo_mlp_param_count());
  fwd_state s;
  float feat[IN];
  double loss = 0.0, g[OUT], da[HID], dz[HID];
  for (uint32_t i = 0; i < n; ++i) {
    bo_mlp_encode(pos + 3 * (size_t)i, nrm + 3 * (size_t)i, box, feat);
    forward_one(params, feat, &s);
    loss += nll_grad(s.o, dir + 3 * (size_t)i, w[i], g);
    /* output layer */
    double* GW = grad + off_w(3);
    double* Gb = grad + off_b(3);
    const double* W4 = params + off_w(3);
    for (int k = 0; k < HID; ++k) da[k] = 0.0;
    for (int j = 0; j < OUT; ++j) {
      Gb[j] += g[j];
      for (int k = 0; k < HID; ++k) {
        GW[j * HID + k] += g[j] * s.a[3][k];
        da[k] += W4[j * HID + k] * g[j];
      }
    }
    /* hidden layers 2, 1, 0: z_l = W_l a_l + b_l, a_{l+1} = relu(z_l) */
    for (int l = 2; l >= 0; --l) {
      for (int k = 0; k < HID; ++k) dz[k] = s.a[l + 1][k] > 0.0 ? da[k] : 0.0;
      double* GWl = grad + off_w(l);
      double* Gbl = grad + off_b(l);
      const double* Wl = params + off_w(l);
      for (int k = 0; k < IN; ++k) da[k] = 0.0;
      for (int j = 0; j < HID; ++j) {
        Gbl[j] += dz[j];
        for (int k = 0; k < IN; ++k) {
          GWl[j * IN + k] += dz[j] * s.a[l][k];
          da[k] += Wl[j * IN + k] * dz[j];
        }
      }
    }
  }
  return loss;
}
