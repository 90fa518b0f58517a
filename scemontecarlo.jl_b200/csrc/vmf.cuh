// The learned proposal's output head: a 4-component von Mises-Fisher mixture on S^2
// read from the MLP's 20 outputs (per component: logit, 3 raw mean components, raw
// concentration). kappa = softplus(c) / tau + kKappaMin with tau = kT in meV, so the
// network predicts kappa * kT. The FP64 forms serve training and the host; the sweep
// draws and evaluates the mixture in FP32 (MixF below).
#pragma once
#include <math.h>
#include <stdint.h>

namespace vmf {

constexpr int kComp = 4;
constexpr int kOut = 20;
constexpr int kOutPad = 32;
constexpr int kIn = 43;     // 14 neighbour spins x 3 + kT
constexpr int kInPad = 64;
constexpr int kHid = 128;
constexpr double kKappaMin = 1e-3;
constexpr double kTwoPi = 6.283185307179586;

struct Mix {
  double logpi[kComp];
  double mu[kComp][3];
  double mn[kComp];     // |raw mean|
  double kappa[kComp];
  double c[kComp];      // raw concentration
};

__host__ __device__ inline double softplus(double x) { return x > 20.0 ? x : log1p(exp(x)); }
__host__ __device__ inline double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

__host__ __device__ inline void mixture(const float* o, double tau, Mix& m) {
  double amax = -1e300;
  for (int k = 0; k < kComp; ++k) amax = fmax(amax, (double)o[5 * k]);
  double s = 0.0;
  for (int k = 0; k < kComp; ++k) s += exp((double)o[5 * k] - amax);
  const double lse = amax + log(s);
  for (int k = 0; k < kComp; ++k) {
    m.logpi[k] = (double)o[5 * k] - lse;
    const double x = o[5 * k + 1], y = o[5 * k + 2], z = o[5 * k + 3];
    const double n = sqrt(x * x + y * y + z * z);
    m.mn[k] = n;
    const double inv = 1.0 / fmax(n, 1e-12);
    m.mu[k][0] = x * inv;
    m.mu[k][1] = y * inv;
    m.mu[k][2] = z * inv;
    m.c[k] = o[5 * k + 4];
    m.kappa[k] = softplus(m.c[k]) / tau + kKappaMin;
  }
}

// log of kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (mu.x - 1)}
__host__ __device__ inline double log_vmf(const double* mu, double kappa, double x0, double x1, double x2) {
  const double d = mu[0] * x0 + mu[1] * x1 + mu[2] * x2;
  return log(kappa) - log(kTwoPi) - log(-expm1(-2.0 * kappa)) + kappa * (d - 1.0);
}

__host__ __device__ inline double log_q(const Mix& m, double x0, double x1, double x2) {
  double l[kComp], lm = -1e300;
  for (int k = 0; k < kComp; ++k) {
    l[k] = m.logpi[k] + log_vmf(m.mu[k], m.kappa[k], x0, x1, x2);
    lm = fmax(lm, l[k]);
  }
  double s = 0.0;
  for (int k = 0; k < kComp; ++k) s += exp(l[k] - lm);
  return lm + log(s);
}

// One draw: component by the weights' inverse CDF (u_comp), w = mu.x by the
// inverse CDF w = 1 + log(u + (1 - u) e^{-2 kappa}) / kappa (u_w), azimuth
// 2 pi u_phi about mu in the frame t1 = normalised (e_a - mu_a mu) for the axis a
// least aligned with mu, t2 = mu x t1.
__host__ __device__ inline void sample(const Mix& m, double u_comp, double u_w, double u_phi, double* out) {
  int k = 0;
  double acc = exp(m.logpi[0]);
  while (k < kComp - 1 && u_comp >= acc) {
    ++k;
    acc += exp(m.logpi[k]);
  }
  const double kap = m.kappa[k];
  double w = 1.0 + log(u_w + (1.0 - u_w) * exp(-2.0 * kap)) / kap;
  w = fmin(1.0, fmax(-1.0, w));
  const double v = sqrt(fmax(0.0, 1.0 - w * w));
  const double* mu = m.mu[k];
  const double a0 = fabs(mu[0]), a1 = fabs(mu[1]), a2 = fabs(mu[2]);
  const int ax = (a0 <= a1 && a0 <= a2) ? 0 : (a1 <= a2 ? 1 : 2);
  double t1[3] = {-mu[ax] * mu[0], -mu[ax] * mu[1], -mu[ax] * mu[2]};
  t1[ax] += 1.0;
  const double tn = 1.0 / sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
  t1[0] *= tn, t1[1] *= tn, t1[2] *= tn;
  const double t2[3] = {mu[1] * t1[2] - mu[2] * t1[1], mu[2] * t1[0] - mu[0] * t1[2], mu[0] * t1[1] - mu[1] * t1[0]};
  const double ph = kTwoPi * u_phi;
  const double cp = cos(ph), sp = sin(ph);
  double x[3];
  for (int i = 0; i < 3; ++i) x[i] = w * mu[i] + v * (cp * t1[i] + sp * t2[i]);
  const double n = 1.0 / sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  out[0] = x[0] * n, out[1] = x[1] * n, out[2] = x[2] * n;
}

// -log q(y) and its gradient with respect to the 20 outputs (scaled by `scale`).
__host__ __device__ inline double nll_grad(const float* o, double tau, const double* y, double scale, float* dout) {
  Mix m;
  mixture(o, tau, m);
  double l[kComp], d[kComp], lm = -1e300;
  for (int k = 0; k < kComp; ++k) {
    d[k] = m.mu[k][0] * y[0] + m.mu[k][1] * y[1] + m.mu[k][2] * y[2];
    l[k] = m.logpi[k] + log_vmf(m.mu[k], m.kappa[k], y[0], y[1], y[2]);
    lm = fmax(lm, l[k]);
  }
  double s = 0.0;
  for (int k = 0; k < kComp; ++k) s += exp(l[k] - lm);
  const double lq = lm + log(s);
  for (int k = 0; k < kComp; ++k) {
    const double r = exp(l[k] - lq);
    const double pi = exp(m.logpi[k]);
    dout[5 * k] = (float)(scale * (pi - r));
    const double kap = m.kappa[k];
    const double dk = 1.0 / kap - 2.0 / expm1(2.0 * kap) + (d[k] - 1.0);
    dout[5 * k + 4] = (float)(scale * (-r * dk * sigmoid(m.c[k]) / tau));
    const double inv = 1.0 / fmax(m.mn[k], 1e-12);
    for (int i = 0; i < 3; ++i)
      dout[5 * k + 1 + i] = (float)(scale * (-r * kap * (y[i] - d[k] * m.mu[k][i]) * inv));
  }
  return -lq;
}

// Single-precision form of the mixture used inside the sweep (the draw and the
// density ratio of one item; the same function evaluates q(e) and q(e'), so the
// Hastings ratio is exactly that of the distribution sampled up to FP32 rounding).
struct MixF {
  float logpi[kComp];
  float mu[kComp][3];
  float kappa[kComp];
};

__device__ inline float softplus_f(float x) { return x > 20.0f ? x : log1pf(__expf(x)); }

__device__ inline void mixture_f(const float* o, float tau, MixF& m) {
  float amax = o[0];
  for (int k = 1; k < kComp; ++k) amax = fmaxf(amax, o[5 * k]);
  float s = 0.0f;
  for (int k = 0; k < kComp; ++k) s += __expf(o[5 * k] - amax);
  const float lse = amax + __logf(s);
  for (int k = 0; k < kComp; ++k) {
    m.logpi[k] = o[5 * k] - lse;
    const float x = o[5 * k + 1], y = o[5 * k + 2], z = o[5 * k + 3];
    const float inv = 1.0f / fmaxf(sqrtf(x * x + y * y + z * z), 1e-12f);
    m.mu[k][0] = x * inv;
    m.mu[k][1] = y * inv;
    m.mu[k][2] = z * inv;
    m.kappa[k] = softplus_f(o[5 * k + 4]) / tau + (float)kKappaMin;
  }
}

__device__ inline float log_q_f(const MixF& m, float x0, float x1, float x2) {
  float l[kComp], lm = -3.0e38f;
  for (int k = 0; k < kComp; ++k) {
    const float d = m.mu[k][0] * x0 + m.mu[k][1] * x1 + m.mu[k][2] * x2;
    const float kap = m.kappa[k];
    l[k] = m.logpi[k] + __logf(kap) - __logf((float)kTwoPi) - __logf(-expm1f(-2.0f * kap)) + kap * (d - 1.0f);
    lm = fmaxf(lm, l[k]);
  }
  float s = 0.0f;
  for (int k = 0; k < kComp; ++k) s += __expf(l[k] - lm);
  return lm + __logf(s);
}

// the draw of sample() in single precision (same inverse CDFs and frame)
__device__ inline void sample_f(const MixF& m, float u_comp, float u_w, float u_phi, float* out) {
  int k = 0;
  float acc = __expf(m.logpi[0]);
  while (k < kComp - 1 && u_comp >= acc) {
    ++k;
    acc += __expf(m.logpi[k]);
  }
  const float kap = m.kappa[k];
  float w = 1.0f + __logf(u_w + (1.0f - u_w) * __expf(-2.0f * kap)) / kap;
  w = fminf(1.0f, fmaxf(-1.0f, w));
  const float v = sqrtf(fmaxf(0.0f, 1.0f - w * w));
  const float* mu = m.mu[k];
  const float a0 = fabsf(mu[0]), a1 = fabsf(mu[1]), a2 = fabsf(mu[2]);
  const int ax = (a0 <= a1 && a0 <= a2) ? 0 : (a1 <= a2 ? 1 : 2);
  float t1[3] = {-mu[ax] * mu[0], -mu[ax] * mu[1], -mu[ax] * mu[2]};
  t1[ax] += 1.0f;
  const float tn = 1.0f / sqrtf(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
  t1[0] *= tn, t1[1] *= tn, t1[2] *= tn;
  const float t2[3] = {mu[1] * t1[2] - mu[2] * t1[1], mu[2] * t1[0] - mu[0] * t1[2], mu[0] * t1[1] - mu[1] * t1[0]};
  float sp, cp;
  sincosf((float)kTwoPi * u_phi, &sp, &cp);
  float x[3];
  for (int i = 0; i < 3; ++i) x[i] = w * mu[i] + v * (cp * t1[i] + sp * t2[i]);
  const float n = 1.0f / sqrtf(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  out[0] = x[0] * n, out[1] = x[1] * n, out[2] = x[2] * n;
}

}  // namespace vmf
