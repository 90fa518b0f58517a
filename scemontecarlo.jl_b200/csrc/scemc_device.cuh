// scemc_device.cuh — device math of the sweep: the keyed Philox stream, the
// Metropolis proposal, and the real (tesseral) spherical-harmonic rows.
//
// Keyed stream: Philox4x32-10 with key = (lo32(seed), hi32(seed)) and counter
// (site, sweep, slot, tag) — the layout of src/gpu/philox.jl:52-67. Tag 0 is the
// reference's Metropolis stream, so a single chain draws exactly the reference's
// numbers; the fourth counter word (reserved there for update kinds) carries
//   tag 1 = overrelaxation accept uniform, slot = OR pass index;
//   tag 3 = replica-exchange uniform, site = pair index, sweep = exchange count.
// The proposal is evaluated in FP64 (as the reference does), then projected to
// the unit sphere and rounded to FP32 for storage.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace scemc {

constexpr double kTwoPi = 6.283185307179586;  // src/gpu/philox.jl:18
constexpr double kFlipFraction = 0.2;         // src/updates.jl:20
constexpr uint32_t kTagMetro = 0u, kTagOR = 1u, kTagExchange = 3u, kTagLearn = 4u;

// ---------------------------------------------------------------------------
// Philox4x32-10 (src/gpu/philox.jl:26-60)
// ---------------------------------------------------------------------------
struct Blk {
  uint32_t w0, w1, w2, w3;
};

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ __forceinline__ Blk philox10(Blk c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t hi0 = mulhi32(0xd2511f53u, c.w0), lo0 = 0xd2511f53u * c.w0;
    const uint32_t hi1 = mulhi32(0xcd9e8d57u, c.w2), lo1 = 0xcd9e8d57u * c.w2;
    c = Blk{hi1 ^ c.w1 ^ k0, lo1, hi0 ^ c.w3 ^ k1, lo0};
    k0 += 0x9e3779b9u;
    k1 += 0xbb67ae85u;
  }
  return c;
}

__host__ __device__ __forceinline__ Blk philox_block(uint64_t seed, uint32_t site, uint32_t sweep,
                                                     uint32_t slot, uint32_t tag) {
  return philox10(Blk{site, sweep, slot, tag}, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// Open-interval (0,1) uniform from two words: (w>>12 + 0.5) * 2^-52 (philox.jl:78-81).
__host__ __device__ __forceinline__ double philox_uniform(uint32_t hi, uint32_t lo) {
  const uint64_t w = ((uint64_t)hi << 32) | (uint64_t)lo;
  return ((double)(w >> 12) + 0.5) * 0x1p-52;
}

// Box–Muller pair (philox.jl:100-105), FP64.
__device__ __forceinline__ void philox_normal2(const Blk& b, double& n1, double& n2) {
  const double u1 = philox_uniform(b.w0, b.w1);
  const double u2 = philox_uniform(b.w2, b.w3);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincos(kTwoPi * u2, &s, &c);
  n1 = r * c;
  n2 = r * s;
}

// Keyed Metropolis proposal (src/gpu/gpu_sweep.jl:32-41 with the Rodrigues
// rotation of src/updates.jl:25-29), FP64; the result is normalised and rounded
// to FP32. Returns the accept uniform.
__device__ __forceinline__ double keyed_proposal(uint64_t seed, uint32_t site1, uint32_t sweep, float ex,
                                                 float ey, float ez, double step, float& px, float& py,
                                                 float& pz) {
  const Blk b0 = philox_block(seed, site1, sweep, 0u, kTagMetro);
  const double u_flip = philox_uniform(b0.w0, b0.w1);
  const double u_acc = philox_uniform(b0.w2, b0.w3);
  if (u_flip < kFlipFraction) {
    px = -ex;
    py = -ey;
    pz = -ez;
    return u_acc;
  }
  double n1, n2, n3, n4;
  philox_normal2(philox_block(seed, site1, sweep, 1u, kTagMetro), n1, n2);
  philox_normal2(philox_block(seed, site1, sweep, 2u, kTagMetro), n3, n4);
  const double nn = sqrt((n1 * n1 + n2 * n2) + n3 * n3);
  const double a0 = n1 / nn, a1 = n2 / nn, a2 = n3 / nn;
  const double e0 = ex, e1 = ey, e2 = ez;
  double s, c;
  sincos(step * n4, &s, &c);
  const double cr0 = a1 * e2 - a2 * e1, cr1 = a2 * e0 - a0 * e2, cr2 = a0 * e1 - a1 * e0;
  const double d = (a0 * e0 + a1 * e1) + a2 * e2;
  const double f = (1.0 - c) * d;
  double r0 = (c * e0 + s * cr0) + f * a0;
  double r1 = (c * e1 + s * cr1) + f * a1;
  double r2 = (c * e2 + s * cr2) + f * a2;
  const double rn = sqrt((r0 * r0 + r1 * r1) + r2 * r2);
  px = (float)(r0 / rn);
  py = (float)(r1 / rn);
  pz = (float)(r2 / rn);
  return u_acc;
}

// ---------------------------------------------------------------------------
// Tesseral rows. Row order is lm_index order (l-major, m = -l..l); the
// normalisation and sign follow src/gpu/zlm_device.jl:101-109, so that
// Z_1m = N1*(y, z, x) and Z_00 = 1/sqrt(4 pi).
// ---------------------------------------------------------------------------
constexpr float kZ00 = 0.28209479177387814f;
constexpr float kN1 = 0.4886025119029199f;    // sqrt(3/(4 pi))
constexpr float kC2a = 1.0925484305920792f;   // sqrt(15/(4 pi))
constexpr float kC20 = 0.31539156525252005f;  // sqrt(5/(4 pi)) / 2
constexpr float kC22 = 0.5462742152960396f;   // sqrt(15/(16 pi))

__device__ __forceinline__ void zrow_l1(float x, float y, float z, float* o) {
  o[0] = kN1 * y;
  o[1] = kN1 * z;
  o[2] = kN1 * x;
}
__device__ __forceinline__ void zrow_l2(float x, float y, float z, float* o) {
  o[0] = kC2a * (x * y);
  o[1] = kC2a * (y * z);
  o[2] = kC20 * (3.0f * (z * z) - 1.0f);
  o[3] = kC2a * (x * z);
  o[4] = kC22 * (x * x - y * y);
}

// d^n P_l(z)/dz^n for n <= l <= 6 by the zlm_device.jl:66-98 recursion (precision T).
template <typename T>
__device__ __forceinline__ T dnpl_t(int l, int n, T z) {
  T cache[8];
  if (n == l) {
    T p = (T)1;
    for (int i = 2 * l - 1; i >= 1; i -= 2) p *= (T)i;
    cache[0] = p;
  } else {
    T Pl = (T)1, Plm1 = (T)0;
    cache[0] = Pl;
    for (int ll = 1; ll <= l - n; ++ll) {
      const T nPl = ((T)(2 * ll - 1) * z * Pl - (T)(ll - 1) * Plm1) / (T)ll;
      Plm1 = Pl;
      Pl = nPl;
      cache[ll] = Pl;
    }
    for (int ni = 1; ni <= n; ++ni) {
      const T pnn = (T)(2 * ni - 1) * cache[0];
      cache[0] = pnn;
      const int ll = ni + 1;
      cache[1] = ((T)(2 * ll - 1) * (z * pnn + (T)ni * cache[1])) / (T)ll;
      const int hi = (l < l - n + ni) ? l : l - n + ni;
      for (int li = ni + 2; li <= hi; ++li)
        cache[li - ni] = ((T)(2 * li - 1) * (z * cache[li - ni - 1] + (T)ni * cache[li - ni]) -
                          (T)(li - 1) * cache[li - ni - 2]) /
                         (T)li;
    }
  }
  return cache[l - n];
}

template <typename T>
__device__ __forceinline__ T plm_norm_t(int l, int n) {
  T acc = (T)(2 * l + 1) / (T)12.566370614359172;
  for (int i = l - n + 1; i <= l + n; ++i) acc /= (T)i;
  return sqrt(acc);
}

// General tesseral value Z_lm for l <= 6 (zlm_device.jl:20-109 in precision T).
template <typename T>
__device__ __forceinline__ T zlm_general(int l, int m, T x, T y, T z) {
  const int n = m < 0 ? -m : m;
  const T par = (n & 1) ? (T)-1 : (T)1;
  const T plm = par * plm_norm_t<T>(l, n) * dnpl_t<T>(l, n, z);
  if (n == 0) return plm;
  const T c = par * sqrt((T)2) * plm;
  T re = (T)1, im = (T)0;  // (x + iy)^n by repeated multiplication
  for (int k = 0; k < n; ++k) {
    const T nr = re * x - im * y;
    im = re * y + im * x;
    re = nr;
  }
  return m > 0 ? c * re : c * im;
}

// Tangent-projected gradient of Z_lm at u (grad_device.jl:27-67), FP64: the
// Cartesian derivative of par*norm*d^nP_l(z)*sqrt2*Re/Im((x+iy)^n) with the radial
// part (u . dZ) u / |u|^2 removed.
__device__ __forceinline__ void grad_zlm_f64(int l, int m, double x, double y, double z, double* g) {
  const int n = m < 0 ? -m : m;
  const double par = (n & 1) ? -1.0 : 1.0;
  const double nrm = plm_norm_t<double>(l, n);
  const double plm = par * nrm * dnpl_t<double>(l, n, z);
  const double dplm = par * nrm * (l < n + 1 ? 0.0 : dnpl_t<double>(l, n + 1, z));
  const double r2 = x * x + y * y + z * z;
  if (m == 0) {
    const double zz = z * dplm / r2;
    g[0] = -x * zz;
    g[1] = -y * zz;
    g[2] = dplm - z * zz;
    return;
  }
  const double c = par * sqrt(2.0);
  double re = 1.0, im = 0.0, re1 = 1.0, im1 = 0.0;  // (x + iy)^n and (x + iy)^(n - 1)
  for (int k = 0; k < n; ++k) {
    re1 = re, im1 = im;
    const double nr = re * x - im * y;
    im = re * y + im * x;
    re = nr;
  }
  double dx, dy, dz;
  if (m > 0) {
    dx = c * n * plm * re1;
    dy = -c * n * plm * im1;
    dz = c * dplm * re;
  } else {
    dx = c * n * plm * im1;
    dy = c * n * plm * re1;
    dz = c * dplm * im;
  }
  const double zz = (x * dx + y * dy + z * dz) / r2;
  g[0] = dx - x * zz;
  g[1] = dy - y * zz;
  g[2] = dz - z * zz;
}

// Row index -> (l, m).
__host__ __device__ __forceinline__ void row_lm(int row, int& l, int& m) {
  l = 0;
  while ((l + 1) * (l + 1) <= row) ++l;
  m = row - l * l - l;
}

// Full FP32 row up to LMAX into o[(LMAX+1)^2].
template <int LMAX>
__device__ __forceinline__ void zrow_f32(float x, float y, float z, float* o) {
  o[0] = kZ00;
  if (LMAX >= 1) zrow_l1(x, y, z, o + 1);
  if (LMAX >= 2) zrow_l2(x, y, z, o + 4);
#pragma unroll
  for (int l = 3; l <= LMAX; ++l)
#pragma unroll
    for (int m = -l; m <= l; ++m) o[l * l + l + m] = zlm_general<float>(l, m, x, y, z);
}

// Single FP32 value of row `row` (dynamic).
__device__ __forceinline__ float zval_f32(int row, float x, float y, float z) {
  switch (row) {
    case 0: return kZ00;
    case 1: return kN1 * y;
    case 2: return kN1 * z;
    case 3: return kN1 * x;
    case 4: return kC2a * (x * y);
    case 5: return kC2a * (y * z);
    case 6: return kC20 * (3.0f * (z * z) - 1.0f);
    case 7: return kC2a * (x * z);
    case 8: return kC22 * (x * x - y * y);
    default: {
      int l, m;
      row_lm(row, l, m);
      return zlm_general<float>(l, m, x, y, z);
    }
  }
}

// Single FP64 value of row `row`: closed forms for l <= 2, the general recursion above.
__device__ __forceinline__ double zval_f64(int row, double x, double y, double z) {
  switch (row) {
    case 0: return 0.28209479177387814;
    case 1: return 0.4886025119029199 * y;
    case 2: return 0.4886025119029199 * z;
    case 3: return 0.4886025119029199 * x;
    case 4: return 1.0925484305920792 * (x * y);
    case 5: return 1.0925484305920792 * (y * z);
    case 6: return 0.31539156525252005 * (3.0 * (z * z) - 1.0);
    case 7: return 1.0925484305920792 * (x * z);
    case 8: return 0.5462742152960396 * (x * x - y * y);
    default: {
      int l, m;
      row_lm(row, l, m);
      return zlm_general<double>(l, m, x, y, z);
    }
  }
}

}  // namespace scemc
