// oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 CPU restatement of the chain-level spin Monte Carlo path of
// SCEMonteCarlo.jl (v0.1.0). It is the checker for the CUDA library and the
// timed CPU baseline; nothing in the product links or calls it.
//
// Every function cites the reference file:line it restates. Paths are relative
// to the reference project root.
//
// Pinning: the Philox block function is checked against the three Random123
// known-answer vectors the reference's own tests hold
// (test/unit/test_gpu.jl:51-59) and the open-interval edge words (70-71); the
// tesseral row against its analytic l <= 2 forms and S^2 quadrature
// orthonormality; the energy path against exact total-energy differences,
// the rank-generic reference kernels, and closed-form statistics (dimer
// Langevin law, single moment in a field).
//
// Floating-point: compiled with -ffp-contract=off so that a*b+c is never fused,
// matching Julia's default (no implicit muladd).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kFourPi = 12.566370614359172;          // Float64(4π)
constexpr double kTwoPi = 6.283185307179586;            // philox.jl:18
constexpr double kFlipFraction = 0.2;                   // updates.jl:20
// units.jl:17 and :29
const double KB_EV = 1.380649e-23 / 1.602176634e-19;
const double MU_B_EV_T = 9.2740100783e-24 / 1.602176634e-19;

// ---------------------------------------------------------------------------
// Philox4x32-10 — src/gpu/philox.jl:12-60
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t w[4];
};

inline U4 philox_round(const U4& c, uint32_t k0, uint32_t k1) {  // philox.jl:26-35
  const uint64_t p0 = (uint64_t)0xd2511f53u * (uint64_t)c.w[0];
  const uint64_t p1 = (uint64_t)0xcd9e8d57u * (uint64_t)c.w[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  return U4{{hi1 ^ c.w[1] ^ k0, lo1, hi0 ^ c.w[3] ^ k1, lo0}};
}

inline U4 philox10(U4 c, uint32_t k0, uint32_t k1) {  // philox.jl:43-50
  for (int i = 0; i < 9; ++i) {
    c = philox_round(c, k0, k1);
    k0 += 0x9e3779b9u;
    k1 += 0xbb67ae85u;
  }
  return philox_round(c, k0, k1);
}

// ctr = (site, sweep, slot, tag); key = (lo32(seed), hi32(seed)) — philox.jl:55-60.
// The reference's Metropolis stream uses tag 0 (philox.jl:52-54 reserves the
// fourth word for update-kind / replica tags).
inline U4 philox_block(uint64_t seed, int32_t site, int32_t sweep, uint32_t slot,
                       uint32_t tag) {
  U4 c{{(uint32_t)site, (uint32_t)sweep, slot, tag}};
  return philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

inline double philox_uniform(uint32_t hi, uint32_t lo) {  // philox.jl:78-81
  const uint64_t w = ((uint64_t)hi << 32) | (uint64_t)lo;
  return ((double)(w >> 12) + 0.5) * 0x1p-52;
}

inline void philox_normal2(const U4& b, double& n1, double& n2) {  // philox.jl:100-105
  const double u1 = philox_uniform(b.w[0], b.w[1]);
  const double u2 = philox_uniform(b.w[2], b.w[3]);
  const double r = std::sqrt(-2.0 * std::log(u1));
  const double a = kTwoPi * u2;
  n1 = r * std::cos(a);
  n2 = r * std::sin(a);
}

// Rodrigues rotation — src/updates.jl:25-29:
// c*e + s*cross(axis,e) + (1-c)*dot(axis,e)*axis, left-to-right.
inline void rotate(const double* e, const double* ax, double th, double* out) {
  const double c = std::cos(th), s = std::sin(th);
  const double cr0 = ax[1] * e[2] - ax[2] * e[1];
  const double cr1 = ax[2] * e[0] - ax[0] * e[2];
  const double cr2 = ax[0] * e[1] - ax[1] * e[0];
  const double d = ax[0] * e[0] + ax[1] * e[1] + ax[2] * e[2];
  const double f = (1.0 - c) * d;
  out[0] = (c * e[0] + s * cr0) + f * ax[0];
  out[1] = (c * e[1] + s * cr1) + f * ax[1];
  out[2] = (c * e[2] + s * cr2) + f * ax[2];
}

// _keyed_proposal — src/gpu/gpu_sweep.jl:32-41 (slots: philox.jl:65-67).
inline void keyed_proposal(uint64_t seed, int32_t site, int32_t sweep, const double* e,
                           double step, double* e2, double* u_acc) {
  const U4 b0 = philox_block(seed, site, sweep, 0u, 0u);
  const double u_flip = philox_uniform(b0.w[0], b0.w[1]);
  *u_acc = philox_uniform(b0.w[2], b0.w[3]);
  if (u_flip < kFlipFraction) {
    e2[0] = -e[0];
    e2[1] = -e[1];
    e2[2] = -e[2];
    return;
  }
  double n1, n2, n3, n4;
  philox_normal2(philox_block(seed, site, sweep, 1u, 0u), n1, n2);
  philox_normal2(philox_block(seed, site, sweep, 2u, 0u), n3, n4);
  const double nn = std::sqrt((n1 * n1 + n2 * n2) + n3 * n3);
  const double ax[3] = {n1 / nn, n2 / nn, n3 / nn};
  rotate(e, ax, step * n4, e2);
}

// ---------------------------------------------------------------------------
// Tesseral row Z_lm(u) — src/gpu/zlm_device.jl:17-129 (operation order kept)
// ---------------------------------------------------------------------------
inline double plm_norm(int l, int m) {  // zlm_device.jl:20-26
  double acc = (double)(2 * l + 1) / kFourPi;
  for (int i = l - m + 1; i <= l + m; ++i) acc /= (double)i;
  return std::sqrt(acc);
}

struct Cx {
  double re, im;
};
inline Cx cmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

inline Cx cpow(Cx x, int p) {  // zlm_device.jl:34-57 (power_by_squaring value path)
  if (p == 0) return Cx{1.0, 0.0};
  const Cx xsq = cmul(x, x);
  if (p == 1) return x;
  if (p == 2) return xsq;
  int t = __builtin_ctz((unsigned)p) + 1;
  p >>= t;
  if ((t -= 1) > 0) x = xsq;
  while ((t -= 1) > 0) x = cmul(x, x);
  Cx y = x;
  while (p > 0) {
    t = __builtin_ctz((unsigned)p) + 1;
    p >>= t;
    while ((t -= 1) >= 0) x = cmul(x, x);
    y = cmul(y, x);
  }
  return y;
}

// d^n P_l(x)/dx^n — zlm_device.jl:66-98. cache is 0-based here (cache[i-1]).
inline double dnpl(double x, int l, int n, double* cache) {
  if (n == l) {
    double p = 1.0;
    for (int i = 2 * l - 1; i >= 1; i -= 2) p *= (double)i;
    cache[0] = p;
  } else {
    double Pl = 1.0, Plm1 = 0.0;
    cache[0] = Pl;
    for (int ll = 1; ll <= l - n; ++ll) {
      const double nPl = ((double)(2 * ll - 1) * x * Pl - (double)(ll - 1) * Plm1) / (double)ll;
      Plm1 = Pl;
      Pl = nPl;
      cache[ll] = Pl;
    }
    for (int ni = 1; ni <= n; ++ni) {
      const double pnn = (double)(2 * ni - 1) * cache[0];
      cache[0] = pnn;
      const int ll = ni + 1;
      cache[1] = ((double)(2 * ll - 1) * (x * pnn + (double)ni * cache[1])) / (double)ll;
      const int hi = std::min(l, l - n + ni);
      for (int li = ni + 2; li <= hi; ++li) {
        // Julia: cache[li-ni+1] = ((2li-1)*(x*cache[li-ni] + ni*cache[li-ni+1])
        //                          - (li-1)*cache[li-ni-1]) / li   (1-based)
        cache[li - ni] = ((double)(2 * li - 1) * (x * cache[li - ni - 1] + (double)ni * cache[li - ni]) -
                          (double)(li - 1) * cache[li - ni - 2]) /
                         (double)li;
      }
    }
  }
  return cache[l - n];
}

inline double zlm_one(int l, int m, const double* u, double* cache) {  // zlm_device.jl:101-109
  const int n = m < 0 ? -m : m;
  const double par = (n & 1) ? -1.0 : 1.0;
  const double plm = par * plm_norm(l, n) * dnpl(u[2], l, n, cache);
  if (n == 0) return plm;
  const double c = par * std::sqrt(2.0) * plm;
  const Cx zp = cpow(Cx{u[0], u[1]}, n);
  return m > 0 ? c * zp.re : c * zp.im;
}

inline void zlm_row(int lmax, const double* u, double* z) {  // zlm_device.jl:120-129
  double cache[16];
  int i = 0;
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) z[i++] = zlm_one(l, m, u, cache);
}

// Tangent-projected gradient of Z_lm at u — src/gpu/grad_device.jl:27-67 (the
// device twin of Harmonics.grad_Zlm_unsafe): d^{n+1}P_l is +0 when l < n + 1; the
// radial part (u . dZ) u / |u|^2 is removed.
inline void grad_zlm_one(int l, int m, const double* u, double* cache, double* g) {
  const double x = u[0], y = u[1], z = u[2];
  const int n = m < 0 ? -m : m;
  const double par = (n & 1) ? -1.0 : 1.0;
  const double plm = par * plm_norm(l, n) * dnpl(z, l, n, cache);
  const double dplm = par * plm_norm(l, n) * (l < n + 1 ? 0.0 : dnpl(z, l, n + 1, cache));
  const double r2 = x * x + y * y + z * z;
  if (m == 0) {
    const double zz = z * dplm / r2;
    g[0] = -x * zz;
    g[1] = -y * zz;
    g[2] = dplm - z * zz;
    return;
  }
  const double c = par * std::sqrt(2.0);
  const Cx zpn = cpow(Cx{x, y}, n), zpn1 = cpow(Cx{x, y}, n - 1);
  double dx, dy, dz;
  if (m > 0) {
    dx = c * n * plm * zpn1.re;
    dy = -c * n * plm * zpn1.im;
    dz = c * dplm * zpn.re;
  } else {
    dx = c * n * plm * zpn1.im;
    dy = c * n * plm * zpn1.re;
    dz = c * dplm * zpn.im;
  }
  const double zz = (x * dx + y * dy + z * dz) / r2;
  g[0] = dx - x * zz;
  g[1] = dy - y * zz;
  g[2] = dz - z * zz;
}

inline void grad_zlm_row(int lmax, const double* u, double* g) {  // grad_device.jl:77-89, component-fastest
  double cache[16];
  int i = 0;
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m, ++i) grad_zlm_one(l, m, u, cache, g + 3 * i);
}

inline int lm_index0(int l, int m) { return l * l + l + m; }  // Harmonics.lm_index - 1

// ---------------------------------------------------------------------------
// TiledHamiltonian — src/hamiltonian.jl:62-499 (all index arrays 1-based as in Julia)
// ---------------------------------------------------------------------------
struct Term {
  double coef;
  std::vector<int> atoms;   // 1-based
  std::vector<int> shifts;  // 3 per member
  std::vector<int> ls;
  std::vector<double> folded;  // column-major, dims (2l+1)...
};

struct Ham {
  int n_cell_atoms = 0;
  int dims[3] = {1, 1, 1};
  int n_sites = 0, lmax = 0, nlm = 0, n_active = 0, n_colors = 0, n_fitted = 0;
  std::vector<Term> terms;
  std::vector<int32_t> inst_term, inst_ptr, inst_sites, site_ptr, site_inst;
  std::vector<int8_t> site_slot;
  std::vector<uint8_t> site_has_l1, site_active;
  // programs (hamiltonian.jl:62-91)
  std::vector<int32_t> site_prog, sprog_ptr, sent_tgt, sfac_ptr, sfac_row, site_col, site_col2,
      pent_row, pent_row2, eprog_ptr, efac_ptr, efac_row;
  std::vector<double> sent_w, eent_w, term_coef;
  std::vector<int8_t> sfac_slot;
  std::vector<int32_t> color_ptr, color_sites;
  std::vector<double> magmoms;
  bool has_magmoms = false;
  double field[3] = {0, 0, 0};
};

// Column-major multi-index walk of a dense tensor with the given dims.
inline bool next_index(std::vector<int>& idx, const std::vector<int>& dims) {
  for (size_t k = 0; k < dims.size(); ++k) {
    if (++idx[k] < dims[k]) return true;
    idx[k] = 0;
  }
  return false;
}

// _push_term_programs! — hamiltonian.jl:99-133 (idx is 0-based here; μ = idx - l).
void push_term_programs(Ham& H, double coef, const std::vector<int>& ls,
                        const std::vector<double>& folded) {
  const int D = (int)ls.size();
  std::vector<int> dims(D);
  for (int k = 0; k < D; ++k) dims[k] = 2 * ls[k] + 1;
  for (int v = 0; v < D; ++v) {
    std::vector<int> idx(D, 0);
    size_t lin = 0;
    do {
      const double w = coef * folded[lin++];
      if (w != 0.0) {
        H.sent_w.push_back(w);
        H.sent_tgt.push_back(lm_index0(ls[v], idx[v] - ls[v]) + 1);
        for (int k = 0; k < D; ++k) {
          if (k == v) continue;
          H.sfac_row.push_back(lm_index0(ls[k], idx[k] - ls[k]) + 1);
          H.sfac_slot.push_back((int8_t)(k + 1));
        }
        H.sfac_ptr.push_back((int32_t)H.sfac_row.size() + 1);
        const size_t nf = H.sfac_row.size();
        H.pent_row.push_back(D == 2 ? H.sfac_row[nf - 1] : D == 3 ? H.sfac_row[nf - 2] : 0);
        H.pent_row2.push_back(D == 3 ? H.sfac_row[nf - 1] : 0);
      }
    } while (next_index(idx, dims));
    H.sprog_ptr.push_back((int32_t)H.sent_w.size() + 1);
  }
  std::vector<int> idx(D, 0);
  size_t lin = 0;
  do {
    const double w = folded[lin++];
    if (w != 0.0) {
      H.eent_w.push_back(w);
      for (int k = 0; k < D; ++k) H.efac_row.push_back(lm_index0(ls[k], idx[k] - ls[k]) + 1);
      H.efac_ptr.push_back((int32_t)H.efac_row.size() + 1);
    }
  } while (next_index(idx, dims));
  H.eprog_ptr.push_back((int32_t)H.eent_w.size() + 1);
}

// _build_programs — hamiltonian.jl:138-181
void build_programs(Ham& H) {
  const size_t nadj = H.site_inst.size();
  H.site_prog.assign(nadj, 0);
  H.site_col.assign(nadj, 0);
  H.site_col2.assign(nadj, 0);
  H.sprog_ptr = {1};
  H.sfac_ptr = {1};
  H.eprog_ptr = {1};
  H.efac_ptr = {1};
  H.term_coef.clear();
  std::vector<int> pbase(H.terms.size());
  std::vector<int8_t> pslot1, pslot2;
  int np = 0;
  for (size_t k = 0; k < H.terms.size(); ++k) {
    const Term& t = H.terms[k];
    H.term_coef.push_back(t.coef);
    pbase[k] = np;
    const int D = (int)t.ls.size();
    np += D;
    for (int v = 1; v <= D; ++v) {
      pslot1.push_back(D == 2 ? (int8_t)(3 - v) : D == 3 ? (int8_t)(v == 1 ? 2 : 1) : (int8_t)0);
      pslot2.push_back(D == 3 ? (int8_t)(v == 3 ? 2 : 3) : (int8_t)0);
    }
    push_term_programs(H, t.coef, t.ls, t.folded);
  }
  for (size_t j = 0; j < nadj; ++j) {
    const int inst = H.site_inst[j];
    const int pid = pbase[H.inst_term[inst - 1] - 1] + H.site_slot[j];
    H.site_prog[j] = pid;
    const int off = H.inst_ptr[inst - 1] - 1;
    const int sl1 = pslot1[pid - 1], sl2 = pslot2[pid - 1];
    H.site_col[j] = sl1 == 0 ? 0 : sl2 == 0 ? H.inst_sites[off + sl1 - 1] : -H.inst_sites[off + sl1 - 1];
    H.site_col2[j] = sl2 == 0 ? 0 : H.inst_sites[off + sl2 - 1];
  }
}

// _color_sites — hamiltonian.jl:456-499
void color_sites(Ham& H) {
  std::vector<int32_t> colors(H.n_sites, 0);
  std::vector<int> stamp;
  int ncol = 0;
  for (int s = 1; s <= H.n_sites; ++s) {
    if (!H.site_active[s - 1]) continue;
    for (int j = H.site_ptr[s - 1]; j < H.site_ptr[s]; ++j) {
      const int i = H.site_inst[j - 1];
      for (int q = H.inst_ptr[i - 1]; q < H.inst_ptr[i]; ++q) {
        const int c = colors[H.inst_sites[q - 1] - 1];
        if (c > 0) stamp[c - 1] = s;
      }
    }
    int c = 1;
    while (c <= ncol && stamp[c - 1] == s) ++c;
    if (c > ncol) {
      ncol = c;
      stamp.push_back(0);
    }
    colors[s - 1] = c;
  }
  std::vector<int32_t> counts(ncol, 0);
  for (int s = 0; s < H.n_sites; ++s)
    if (colors[s] > 0) counts[colors[s] - 1]++;
  H.color_ptr.assign(ncol + 1, 0);
  H.color_ptr[0] = 1;
  for (int c = 0; c < ncol; ++c) H.color_ptr[c + 1] = H.color_ptr[c] + counts[c];
  H.color_sites.assign(H.color_ptr[ncol] - 1, 0);
  std::vector<int32_t> cursor(H.color_ptr.begin(), H.color_ptr.end() - 1);
  for (int s = 1; s <= H.n_sites; ++s) {
    const int c = colors[s - 1];
    if (c <= 0) continue;
    H.color_sites[cursor[c - 1] - 1] = s;
    cursor[c - 1]++;
  }
  H.n_colors = ncol;
}

inline int imod(int a, int b) {
  const int r = a % b;
  return r < 0 ? r + b : r;
}

// TiledHamiltonian(n_cell_atoms, terms; dims, magmoms, field) — hamiltonian.jl:267-393,
// _resolve_zeeman 405-430, _zeeman_terms 437-448.
bool build_ham(Ham& H, int n_cell_atoms, std::vector<Term> raw, const int* dims,
               const double* magmoms, const double* field, std::string& err) {
  if (n_cell_atoms < 1) {
    err = "n_cell_atoms must be >= 1";
    return false;
  }
  for (int k = 0; k < 3; ++k)
    if (dims[k] < 1) {
      err = "dims must be >= 1";
      return false;
    }
  H.n_cell_atoms = n_cell_atoms;
  for (int k = 0; k < 3; ++k) H.dims[k] = dims[k];
  if (field && !magmoms) {
    err = "field given without magmoms";
    return false;
  }
  H.has_magmoms = magmoms != nullptr;
  if (magmoms) {
    H.magmoms.assign(magmoms, magmoms + n_cell_atoms);
    for (double m : H.magmoms)
      if (!(std::isfinite(m) && m >= 0)) {
        err = "magmoms must be finite and >= 0";
        return false;
      }
  }
  if (field)
    for (int k = 0; k < 3; ++k) H.field[k] = field[k];
  std::vector<Term> zterms;
  const double N1 = std::sqrt(3.0 / kFourPi);
  if (magmoms && (H.field[0] != 0.0 || H.field[1] != 0.0 || H.field[2] != 0.0)) {
    for (int a = 0; a < n_cell_atoms; ++a) {
      const double m = H.magmoms[a];
      if (m == 0.0) continue;
      const double sc = -(MU_B_EV_T * m / N1);
      Term t;
      t.coef = 1.0;
      t.atoms = {a + 1};
      t.shifts = {0, 0, 0};
      t.ls = {1};
      t.folded = {sc * H.field[1], sc * H.field[2], sc * H.field[0]};
      zterms.push_back(t);
    }
  }
  std::vector<Term> mterms;
  for (auto& t : raw)
    if (t.coef != 0.0) mterms.push_back(t);
  if (mterms.empty() && zterms.empty()) {
    err = "the term list is empty";
    return false;
  }
  int lmax = 0;
  for (size_t k = 0; k < mterms.size(); ++k) {
    Term& mt = mterms[k];
    const int body = (int)mt.atoms.size();
    if ((int)mt.ls.size() != body || (int)mt.shifts.size() != 3 * body) {
      err = "atoms/shifts/ls lengths disagree";
      return false;
    }
    for (int a : mt.atoms)
      if (a < 1 || a > n_cell_atoms) {
        err = "term atom outside 1:n_cell_atoms";
        return false;
      }
    for (int i = 0; i < body; ++i)
      for (int j = i + 1; j < body; ++j) {
        bool same = mt.atoms[i] == mt.atoms[j];
        for (int c = 0; c < 3 && same; ++c)
          same = imod(mt.shifts[3 * i + c], dims[c]) == imod(mt.shifts[3 * j + c], dims[c]);
        if (same) {
          err = "term folds two member sites onto one supercell site";
          return false;
        }
      }
    if (mt.shifts[0] != 0 || mt.shifts[1] != 0 || mt.shifts[2] != 0) {
      err = "shifts[1] must be zero";
      return false;
    }
    size_t sz = 1;
    for (int l : mt.ls) {
      if (l < 0) {
        err = "negative angular momentum";
        return false;
      }
      sz *= (size_t)(2 * l + 1);
      lmax = std::max(lmax, l);
    }
    if (sz != mt.folded.size()) {
      err = "size(folded) does not match ls";
      return false;
    }
    mt.coef = mt.coef * std::pow(kFourPi, (double)body / 2.0);  // hamiltonian.jl:316
  }
  H.n_fitted = (int)mterms.size();
  H.terms = mterms;
  if (!zterms.empty()) {
    H.terms.insert(H.terms.end(), zterms.begin(), zterms.end());
    lmax = std::max(lmax, 1);
  }
  const int ncells = dims[0] * dims[1] * dims[2];
  H.n_sites = n_cell_atoms * ncells;
  H.lmax = lmax;
  H.nlm = (lmax + 1) * (lmax + 1);
  const int nterms = (int)H.terms.size();
  const int n_inst = nterms * ncells;
  H.inst_term.assign(n_inst, 0);
  H.inst_ptr.assign(n_inst + 1, 0);
  H.inst_ptr[0] = 1;
  int i = 0;
  for (int c3 = 0; c3 < dims[2]; ++c3)
    for (int c2 = 0; c2 < dims[1]; ++c2)
      for (int c1 = 0; c1 < dims[0]; ++c1)
        for (int k = 0; k < nterms; ++k) {
          const Term& t = H.terms[k];
          H.inst_term[i] = k + 1;
          for (size_t m = 0; m < t.atoms.size(); ++m) {
            const int w1 = imod(c1 + t.shifts[3 * m + 0], dims[0]);
            const int w2 = imod(c2 + t.shifts[3 * m + 1], dims[1]);
            const int w3 = imod(c3 + t.shifts[3 * m + 2], dims[2]);
            H.inst_sites.push_back(t.atoms[m] + n_cell_atoms * (w1 + dims[0] * (w2 + dims[1] * w3)));
          }
          H.inst_ptr[i + 1] = (int32_t)H.inst_sites.size() + 1;
          ++i;
        }
  // per-site adjacency CSR — hamiltonian.jl:355-375
  std::vector<int32_t> counts(H.n_sites, 0);
  for (int32_t s : H.inst_sites) counts[s - 1]++;
  H.site_ptr.assign(H.n_sites + 1, 0);
  H.site_ptr[0] = 1;
  for (int s = 0; s < H.n_sites; ++s) H.site_ptr[s + 1] = H.site_ptr[s] + counts[s];
  H.site_inst.assign(H.inst_sites.size(), 0);
  H.site_slot.assign(H.inst_sites.size(), 0);
  std::vector<int32_t> cursor(H.site_ptr.begin(), H.site_ptr.end() - 1);
  for (int inst = 1; inst <= n_inst; ++inst) {
    int slot = 0;
    for (int q = H.inst_ptr[inst - 1]; q < H.inst_ptr[inst]; ++q) {
      ++slot;
      const int s = H.inst_sites[q - 1];
      H.site_inst[cursor[s - 1] - 1] = inst;
      H.site_slot[cursor[s - 1] - 1] = (int8_t)slot;
      cursor[s - 1]++;
    }
  }
  H.site_has_l1.assign(H.n_sites, 0);
  H.site_active.assign(H.n_sites, 0);
  H.n_active = 0;
  for (int s = 0; s < H.n_sites; ++s) {
    for (int j = H.site_ptr[s]; j < H.site_ptr[s + 1]; ++j) {
      const Term& t = H.terms[H.inst_term[H.site_inst[j - 1] - 1] - 1];
      if (t.ls[H.site_slot[j - 1] - 1] == 1) H.site_has_l1[s] = 1;
    }
    H.site_active[s] = H.site_ptr[s + 1] > H.site_ptr[s];
    H.n_active += H.site_active[s];
  }
  build_programs(H);
  color_sites(H);
  return true;
}

// ---------------------------------------------------------------------------
// Energy contract — src/energy.jl:26-157, reference kernels 283-344
// zrows is nlm x n_sites column-major (column s-1 holds Z(e_s)).
// ---------------------------------------------------------------------------
void zrows_of(const Ham& H, const double* config, double* zrows) {  // energy.jl:41-50
  for (int s = 0; s < H.n_sites; ++s) zlm_row(H.lmax, config + 3 * s, zrows + (size_t)H.nlm * s);
}

inline double Z(const Ham& H, const double* zrows, int row1, int col1) {
  return zrows[(size_t)H.nlm * (col1 - 1) + (row1 - 1)];
}

double total_energy(const Ham& H, const double* zrows) {  // energy.jl:55-75
  double E = 0.0;
  for (size_t i = 0; i < H.inst_term.size(); ++i) {
    const int k = H.inst_term[i];
    const int off = H.inst_ptr[i] - 1;
    double Ei = 0.0;
    for (int e = H.eprog_ptr[k - 1]; e < H.eprog_ptr[k]; ++e) {
      double p = 1.0;
      const int f0 = H.efac_ptr[e - 1] - 1;
      const int nf = H.efac_ptr[e] - 1 - f0;
      for (int m = 1; m <= nf; ++m) p *= Z(H, zrows, H.efac_row[f0 + m - 1], H.inst_sites[off + m - 1]);
      Ei += H.eent_w[e - 1] * p;
    }
    E += H.term_coef[k - 1] * Ei;
  }
  return E;
}

double total_energy_ref(const Ham& H, const double* zrows) {  // energy.jl:283-309
  double E = 0.0;
  for (size_t i = 0; i < H.inst_term.size(); ++i) {
    const Term& t = H.terms[H.inst_term[i] - 1];
    const int off = H.inst_ptr[i] - 1;
    const int D = (int)t.ls.size();
    std::vector<int> dims(D), idx(D, 0);
    for (int k = 0; k < D; ++k) dims[k] = 2 * t.ls[k] + 1;
    double Ei = 0.0;
    size_t lin = 0;
    do {
      const double w = t.folded[lin++];
      if (w == 0.0) continue;
      double p = 1.0;
      for (int k = 0; k < D; ++k)
        p *= Z(H, zrows, lm_index0(t.ls[k], idx[k] - t.ls[k]) + 1, H.inst_sites[off + k]);
      Ei += w * p;
    } while (next_index(idx, dims));
    E += t.coef * Ei;
  }
  return E;
}

void site_coeffs(const Ham& H, int s, const double* zrows, double* c) {  // energy.jl:100-139
  for (int j = H.site_ptr[s - 1]; j < H.site_ptr[s]; ++j) {
    const int pid = H.site_prog[j - 1];
    const int col = H.site_col[j - 1];
    if (col > 0) {
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        const double z = Z(H, zrows, H.pent_row[e - 1], col);
        if (z == 0.0) continue;
        c[H.sent_tgt[e - 1] - 1] += H.sent_w[e - 1] * z;
      }
    } else if (col < 0) {
      const int col2 = H.site_col2[j - 1];
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        const double p = Z(H, zrows, H.pent_row[e - 1], -col) * Z(H, zrows, H.pent_row2[e - 1], col2);
        if (p == 0.0) continue;
        c[H.sent_tgt[e - 1] - 1] += H.sent_w[e - 1] * p;
      }
    } else {
      const int off = H.inst_ptr[H.site_inst[j - 1] - 1] - 1;
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        double p = 1.0;
        for (int f = H.sfac_ptr[e - 1]; f < H.sfac_ptr[e]; ++f)
          p *= Z(H, zrows, H.sfac_row[f - 1], H.inst_sites[off + H.sfac_slot[f - 1] - 1]);
        if (p == 0.0) continue;
        c[H.sent_tgt[e - 1] - 1] += H.sent_w[e - 1] * p;
      }
    }
  }
}

void site_coeffs_ref(const Ham& H, int s, const double* zrows, double* c) {  // energy.jl:313-344
  for (int j = H.site_ptr[s - 1]; j < H.site_ptr[s]; ++j) {
    const int i = H.site_inst[j - 1];
    const Term& t = H.terms[H.inst_term[i - 1] - 1];
    const int slot = H.site_slot[j - 1];
    const int off = H.inst_ptr[i - 1] - 1;
    const int D = (int)t.ls.size();
    std::vector<int> dims(D), idx(D, 0);
    for (int k = 0; k < D; ++k) dims[k] = 2 * t.ls[k] + 1;
    size_t lin = 0;
    do {
      const double w = t.coef * t.folded[lin++];
      if (w == 0.0) continue;
      double p = 1.0;
      for (int k = 1; k <= D; ++k) {
        if (k == slot) continue;
        p *= Z(H, zrows, lm_index0(t.ls[k - 1], idx[k - 1] - t.ls[k - 1]) + 1, H.inst_sites[off + k - 1]);
      }
      if (p == 0.0) continue;
      c[lm_index0(t.ls[slot - 1], idx[slot - 1] - t.ls[slot - 1])] += w * p;
    } while (next_index(idx, dims));
  }
}

inline double delta_energy(int nlm, const double* c, const double* zold, const double* znew) {
  double dE = 0.0;  // energy.jl:148-157
  for (int k = 0; k < nlm; ++k) {
    const double ck = c[k];
    if (ck == 0.0) continue;
    dE += ck * (znew[k] - zold[k]);
  }
  return dE;
}

// _entry_walk_partial — src/gpu/gpu_sweep.jl:48-85 (1-based lane).
double entry_walk_partial(const Ham& H, const double* zrows, const double* znew, int s, int lane,
                          int ws) {
  double a = 0.0;
  const double* zs = zrows + (size_t)H.nlm * (s - 1);
  for (int j = H.site_ptr[s - 1] + lane - 1; j <= H.site_ptr[s] - 1; j += ws) {
    const int pid = H.site_prog[j - 1];
    const int col = H.site_col[j - 1];
    if (col > 0) {
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        const double z = Z(H, zrows, H.pent_row[e - 1], col);
        if (z == 0.0) continue;
        const int tgt = H.sent_tgt[e - 1];
        a += H.sent_w[e - 1] * z * (znew[tgt - 1] - zs[tgt - 1]);
      }
    } else if (col < 0) {
      const int col2 = H.site_col2[j - 1];
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        const double p = Z(H, zrows, H.pent_row[e - 1], -col) * Z(H, zrows, H.pent_row2[e - 1], col2);
        if (p == 0.0) continue;
        const int tgt = H.sent_tgt[e - 1];
        a += H.sent_w[e - 1] * p * (znew[tgt - 1] - zs[tgt - 1]);
      }
    } else {
      const int off = H.inst_ptr[H.site_inst[j - 1] - 1] - 1;
      for (int e = H.sprog_ptr[pid - 1]; e < H.sprog_ptr[pid]; ++e) {
        double p = 1.0;
        for (int f = H.sfac_ptr[e - 1]; f < H.sfac_ptr[e]; ++f)
          p *= Z(H, zrows, H.sfac_row[f - 1], H.inst_sites[off + H.sfac_slot[f - 1] - 1]);
        if (p == 0.0) continue;
        const int tgt = H.sent_tgt[e - 1];
        a += H.sent_w[e - 1] * p * (znew[tgt - 1] - zs[tgt - 1]);
      }
    }
  }
  return a;
}

double reduce_dE(const Ham& H, const double* dE) {  // updates.jl:92-98
  double d = 0.0;
  for (int32_t s : H.color_sites) d += dE[s - 1];
  return d;
}

// _metropolis_sweep_keyed_ref! — src/gpu/gpu_sweep.jl:227-263
int keyed_sweep(const Ham& H, double* config, double* zrows, double* dE, int32_t* acc, double beta,
                double step, uint64_t seed, int32_t sweep, int ws) {
  std::vector<double> znew(H.nlm), partials(ws);
  std::fill(dE, dE + H.n_sites, 0.0);
  std::fill(acc, acc + H.n_sites, 0);
  int nacc = 0;
  for (int32_t s : H.color_sites) {
    double e2[3], u;
    keyed_proposal(seed, s, sweep, config + 3 * (s - 1), step, e2, &u);
    zlm_row(H.lmax, e2, znew.data());
    for (int lane = 1; lane <= ws; ++lane)
      partials[lane - 1] = entry_walk_partial(H, zrows, znew.data(), s, lane, ws);
    double d = 0.0;
    for (int t = 0; t < ws; ++t) d += partials[t];
    if (d <= 0.0 || u < std::exp(-beta * d)) {
      for (int k = 0; k < 3; ++k) config[3 * (s - 1) + k] = e2[k];
      std::copy(znew.begin(), znew.end(), zrows + (size_t)H.nlm * (s - 1));
      dE[s - 1] = d;
      acc[s - 1] = 1;
      ++nacc;
    }
  }
  return nacc;
}

// ---------------------------------------------------------------------------
// CPU sweeps (the timed baseline) — src/updates.jl:37-290 with the keyed Philox
// draws of the device scheme in place of per-site Xoshiro streams:
//   Metropolis: the slots of gpu_sweep.jl:32-41 (tag 0);
//   overrelaxation pass k of a compound sweep: uniform from block
//   (site, sweep, k, tag 1), words 1-2, read only when dE > 0.
// Colour-parallel over OpenMP threads like `sweep_tasks` (updates.jl:172-206):
// dE staged per site and reduced in colour order => thread-count independent.
// ---------------------------------------------------------------------------
struct Chain {
  std::vector<double> config, zrows, dE;
  double energy = 0.0, step = 0.6, max_drift = 0.0;
  uint64_t seed = 0;
  int64_t sweep_index = 0;
  int64_t acc_metro = 0, att_metro = 0, acc_or = 0, att_or = 0;
};

inline int attempt_metro(const Ham& H, Chain& ch, double beta, int s, int32_t sweep, double* c,
                         double* znew) {  // updates.jl:37-58
  std::fill(c, c + H.nlm, 0.0);
  site_coeffs(H, s, ch.zrows.data(), c);
  double e2[3], u;
  keyed_proposal(ch.seed, s, sweep, ch.config.data() + 3 * (s - 1), ch.step, e2, &u);
  zlm_row(H.lmax, e2, znew);
  double* zs = ch.zrows.data() + (size_t)H.nlm * (s - 1);
  const double d = delta_energy(H.nlm, c, zs, znew);
  if (d <= 0.0 || u < std::exp(-beta * d)) {
    for (int k = 0; k < 3; ++k) ch.config[3 * (s - 1) + k] = e2[k];
    std::copy(znew, znew + H.nlm, zs);
    ch.dE[s - 1] = d;
    return 1;
  }
  return 0;
}

inline int attempt_or(const Ham& H, Chain& ch, double beta, int s, int32_t sweep, uint32_t pass,
                      double* c, double* znew, int* attempted) {  // updates.jl:66-87
  std::fill(c, c + H.nlm, 0.0);
  site_coeffs(H, s, ch.zrows.data(), c);
  const double h[3] = {c[3], c[1], c[2]};
  const double hn = std::sqrt((h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]);
  *attempted = 0;
  if (hn < 1e-12) return 0;
  *attempted = 1;
  const double ax[3] = {h[0] / hn, h[1] / hn, h[2] / hn};
  const double* e = ch.config.data() + 3 * (s - 1);
  const double d2 = 2.0 * ((e[0] * ax[0] + e[1] * ax[1]) + e[2] * ax[2]);
  const double e2[3] = {d2 * ax[0] - e[0], d2 * ax[1] - e[1], d2 * ax[2] - e[2]};
  zlm_row(H.lmax, e2, znew);
  double* zs = ch.zrows.data() + (size_t)H.nlm * (s - 1);
  const double d = delta_energy(H.nlm, c, zs, znew);
  bool ok = d <= 0.0;
  if (!ok) {
    const U4 b = philox_block(ch.seed, s, sweep, pass, 1u);
    ok = philox_uniform(b.w[0], b.w[1]) < std::exp(-beta * d);
  }
  if (ok) {
    for (int k = 0; k < 3; ++k) ch.config[3 * (s - 1) + k] = e2[k];
    std::copy(znew, znew + H.nlm, zs);
    ch.dE[s - 1] = d;
    return 1;
  }
  return 0;
}

// One compound sweep (run.jl:143-150): Metropolis, then n_or overrelaxation passes.
void compound_sweep(const Ham& H, Chain& ch, double beta, int n_or, int threads) {
  const int32_t sweep = (int32_t)(ch.sweep_index + 1);
  for (int pass = -1; pass < n_or; ++pass) {
    std::fill(ch.dE.begin(), ch.dE.end(), 0.0);
    int64_t nacc = 0, natt = 0;
#pragma omp parallel num_threads(threads) reduction(+ : nacc, natt)
    {
      std::vector<double> c(H.nlm), znew(H.nlm);
      for (int col = 0; col < H.n_colors; ++col) {
#pragma omp for schedule(static)
        for (int q = H.color_ptr[col]; q < H.color_ptr[col + 1]; ++q) {
          const int s = H.color_sites[q - 1];
          if (pass < 0) {
            nacc += attempt_metro(H, ch, beta, s, sweep, c.data(), znew.data());
          } else {
            if (!H.site_has_l1[s - 1]) continue;
            int at = 0;
            nacc += attempt_or(H, ch, beta, s, sweep, (uint32_t)pass, c.data(), znew.data(), &at);
            natt += at;
          }
        }
      }
    }
    ch.energy += reduce_dE(H, ch.dE.data());
    if (pass < 0) {
      ch.acc_metro += nacc;
      ch.att_metro += H.n_active;
    } else {
      ch.acc_or += nacc;
      ch.att_or += natt;
    }
  }
  ch.sweep_index += 1;
}

void adapt_step(Chain& ch, double target) {  // updates.jl:296-305 (not frozen)
  if (ch.att_metro > 0) {
    const double a = (double)ch.acc_metro / (double)ch.att_metro;
    ch.step = std::min(std::max(ch.step * std::exp(0.5 * (a - target)), 1e-3), M_PI);
  }
  ch.acc_metro = 0;
  ch.att_metro = 0;
}

double renormalize(const Ham& H, Chain& ch) {  // state.jl:168-185
  for (int s = 0; s < H.n_sites; ++s) {
    if (!H.site_active[s]) continue;
    double* e = ch.config.data() + 3 * s;
    const double n = std::sqrt((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2]);
    for (int k = 0; k < 3; ++k) e[k] = e[k] / n;
    zlm_row(H.lmax, e, ch.zrows.data() + (size_t)H.nlm * s);
  }
  const double E = total_energy(H, ch.zrows.data());
  const double drift = std::fabs(ch.energy - E);
  ch.max_drift = std::max(ch.max_drift, drift);
  ch.energy = E;
  return drift;
}

// ---------------------------------------------------------------------------
// Binning and observables — src/binning.jl:13-218, src/observables.jl:85-249
// ---------------------------------------------------------------------------
constexpr int kMinBins = 32, kMaxLevels = 62;

struct LogBinner {  // binning.jl:25-79
  int ncomp;
  std::vector<int64_t> count;
  std::vector<double> sums, sums2, pending;  // level-major: [k*ncomp + j]
  std::vector<uint8_t> pending_full;
  int64_t n = 0;
  explicit LogBinner(int nc)
      : ncomp(nc), count(kMaxLevels, 0), sums(kMaxLevels * nc, 0.0), sums2(kMaxLevels * nc, 0.0),
        pending(kMaxLevels * nc, 0.0), pending_full(kMaxLevels, 0) {}
  void push(const double* xs) {
    n += 1;
    for (int k = 0; k < kMaxLevels; ++k) {
      count[k] += 1;
      for (int j = 0; j < ncomp; ++j) {
        const double x = k == 0 ? xs[j] : pending[(k - 1) * ncomp + j];
        sums[k * ncomp + j] += x;
        sums2[k * ncomp + j] += x * x;
      }
      if (pending_full[k]) {
        for (int j = 0; j < ncomp; ++j) {
          const double x = k == 0 ? xs[j] : pending[(k - 1) * ncomp + j];
          pending[k * ncomp + j] = 0.5 * (pending[k * ncomp + j] + x);
        }
        pending_full[k] = 0;
      } else {
        for (int j = 0; j < ncomp; ++j) {
          const double x = k == 0 ? xs[j] : pending[(k - 1) * ncomp + j];
          pending[k * ncomp + j] = x;
        }
        pending_full[k] = 1;
        break;
      }
    }
  }
  double level_error(int k, int j) const {  // binning.jl:87-92
    const int64_t nn = count[k];
    if (nn < 2) return NAN;
    const double s = sums[k * ncomp + j];
    const double var = (sums2[k * ncomp + j] - s * s / (double)nn) / (double)(nn - 1);
    return std::sqrt(std::max(var, 0.0) / (double)nn);
  }
  int plateau() const {  // binning.jl:95-98 (0-based level)
    for (int k = kMaxLevels - 1; k >= 0; --k)
      if (count[k] >= kMinBins) return k;
    return 0;
  }
  double mean(int j) const { return n == 0 ? NAN : sums[j] / (double)n; }
  double std_error(int j) const { return n >= 2 ? level_error(plateau(), j) : NAN; }
  double tau_int(int j) const {  // binning.jl:120-128
    if (n < 2) return NAN;
    const double e1 = level_error(0, j);
    if (!(e1 > 0)) return NAN;
    const double r = level_error(plateau(), j) / e1;
    return 0.5 * (r * r - 1.0);
  }
};

struct BinStore {  // binning.jl:138-188
  int ncomp;
  int64_t bin_size;
  int nbins;
  std::vector<double> means, acc;
  int nfull = 0;
  int64_t nacc = 0;
  BinStore(int nc, int64_t bs, int nb) : ncomp(nc), bin_size(bs), nbins(nb), means(nb * nc, 0.0), acc(nc, 0.0) {}
  void push(const double* xs) {
    if (nfull >= nbins) return;
    for (int j = 0; j < ncomp; ++j) acc[j] += xs[j];
    nacc += 1;
    if (nacc == bin_size) {
      for (int j = 0; j < ncomp; ++j) {
        means[nfull * ncomp + j] = acc[j] / (double)bin_size;
        acc[j] = 0.0;
      }
      nfull += 1;
      nacc = 0;
    }
  }
};

// Observable ids in the order of standard_observables (observables.jl:85-92).
enum { OBS_E = 0, OBS_E2, OBS_M, OBS_ABSM, OBS_M2, OBS_M4, OBS_SUB, OBS_COUNT };

struct Accums {
  std::vector<LogBinner> bin;
  std::vector<BinStore> store;
};

int obs_ncomp(const Ham& H, int o) {
  if (o == OBS_M) return 3;
  if (o == OBS_SUB) return 3 * H.n_cell_atoms;
  return 1;
}

void measure(const Ham& H, const Chain& ch, Accums& A) {  // observables.jl:104-143,186-193
  double m[3] = {0, 0, 0};
  // pairwise vs sequential summation differ by ULPs only; sequential here
  for (int s = 0; s < H.n_sites; ++s)
    if (H.site_active[s])
      for (int k = 0; k < 3; ++k) m[k] += ch.config[3 * s + k];
  for (int k = 0; k < 3; ++k) m[k] /= (double)H.n_active;
  const double m2 = (m[0] * m[0] + m[1] * m[1]) + m[2] * m[2];
  std::vector<double> sub(3 * H.n_cell_atoms, 0.0);
  for (int s = 0; s < H.n_sites; ++s) {
    if (!H.site_active[s]) continue;
    const int a = s % H.n_cell_atoms;
    for (int k = 0; k < 3; ++k) sub[3 * a + k] += ch.config[3 * s + k];
  }
  const int ncells = H.n_sites / H.n_cell_atoms;
  for (double& v : sub) v /= (double)ncells;
  const double E = ch.energy;
  double v1;
  v1 = E;
  A.bin[OBS_E].push(&v1), A.store[OBS_E].push(&v1);
  v1 = E * E;
  A.bin[OBS_E2].push(&v1), A.store[OBS_E2].push(&v1);
  A.bin[OBS_M].push(m), A.store[OBS_M].push(m);
  v1 = std::sqrt(m2);
  A.bin[OBS_ABSM].push(&v1), A.store[OBS_ABSM].push(&v1);
  v1 = m2;
  A.bin[OBS_M2].push(&v1), A.store[OBS_M2].push(&v1);
  v1 = m2 * m2;
  A.bin[OBS_M4].push(&v1), A.store[OBS_M4].push(&v1);
  A.bin[OBS_SUB].push(sub.data()), A.store[OBS_SUB].push(sub.data());
}

// jackknife — binning.jl:198-218
template <class F>
void jackknife(F f, const std::vector<std::vector<double>>& cols, double& est, double& err) {
  const size_t nb = cols[0].size();
  std::vector<double> tot(cols.size(), 0.0), loo(cols.size()), th(nb);
  for (size_t q = 0; q < cols.size(); ++q)
    for (double v : cols[q]) tot[q] += v;
  std::vector<double> mean(cols.size());
  for (size_t q = 0; q < cols.size(); ++q) mean[q] = tot[q] / (double)nb;
  const double full = f(mean);
  for (size_t i = 0; i < nb; ++i) {
    for (size_t q = 0; q < cols.size(); ++q) loo[q] = (tot[q] - cols[q][i]) / (double)(nb - 1);
    th[i] = f(loo);
  }
  double tbar = 0.0;
  for (double t : th) tbar += t;
  tbar /= (double)nb;
  est = (double)nb * full - (double)(nb - 1) * tbar;
  double ss = 0.0;
  for (double t : th) ss += (t - tbar) * (t - tbar);
  err = std::sqrt((double)(nb - 1) / (double)nb * ss);
}

// Output block of one temperature: for observables E,E2,m(3),absm,m2,m4,sub(3A):
// mean, err, tau per component; then C, chi, U (est, err); then acc_m, acc_or, step, drift.
int stats_len(const Ham& H) { return 3 * (6 + 2 + 3 * H.n_cell_atoms) + 6 + 4; }

void finalize(const Ham& H, const Accums& A, const Chain& ch, double kT, double* out) {
  int w = 0;
  for (int o = 0; o < OBS_COUNT; ++o) {
    const int nc = obs_ncomp(H, o);
    for (int j = 0; j < nc; ++j) {
      out[w++] = A.bin[o].mean(j);
      out[w++] = A.bin[o].std_error(j);
      out[w++] = A.bin[o].tau_int(j);
    }
  }
  auto col = [&](int o) {
    const BinStore& s = A.store[o];
    return std::vector<double>(s.means.begin(), s.means.begin() + s.nfull);
  };
  const double n = (double)H.n_active;
  double est, err;
  // standard_evaluables — observables.jl:160-166
  auto ok = [](const std::vector<std::vector<double>>& c) { return c[0].size() >= 2; };
  std::vector<std::vector<double>> ce = {col(OBS_E), col(OBS_E2)};
  if (ok(ce)) {
    jackknife([&](const std::vector<double>& m) { return (m[1] - m[0] * m[0]) / (n * kT * kT); }, ce, est, err);
  } else {
    est = err = NAN;
  }
  out[w++] = est, out[w++] = err;
  std::vector<std::vector<double>> cx = {col(OBS_M2), col(OBS_ABSM)};
  if (ok(cx)) {
    jackknife([&](const std::vector<double>& m) { return n * (m[0] - m[1] * m[1]) / kT; }, cx, est, err);
  } else {
    est = err = NAN;
  }
  out[w++] = est, out[w++] = err;
  std::vector<std::vector<double>> cu = {col(OBS_M2), col(OBS_M4)};
  if (ok(cu)) {
    jackknife([&](const std::vector<double>& m) { return m[1] / (m[0] * m[0]); }, cu, est, err);
  } else {
    est = err = NAN;
  }
  out[w++] = est, out[w++] = err;
  out[w++] = ch.att_metro == 0 ? NAN : (double)ch.acc_metro / (double)ch.att_metro;
  out[w++] = ch.att_or == 0 ? NAN : (double)ch.acc_or / (double)ch.att_or;
  out[w++] = ch.step;
  out[w++] = ch.max_drift;
}

Accums make_accums(const Ham& H, int64_t planned, int nbins) {  // observables.jl:180-184
  Accums A;
  const int64_t bs = std::max<int64_t>(1, planned / nbins);
  for (int o = 0; o < OBS_COUNT; ++o) {
    A.bin.emplace_back(obs_ncomp(H, o));
    A.store.emplace_back(obs_ncomp(H, o), bs, nbins);
  }
  return A;
}

thread_local std::string g_err;

}  // namespace

// ===========================================================================
// C ABI for the Python test harness (ctypes). Site/instance indices 1-based.
// ===========================================================================
extern "C" {

const char* or_last_error() { return g_err.c_str(); }

void or_philox4x32(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
  U4 c{{ctr[0], ctr[1], ctr[2], ctr[3]}};
  const U4 r = philox10(c, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = r.w[i];
}

void or_philox_block(uint64_t seed, int32_t site, int32_t sweep, uint32_t slot, uint32_t tag,
                     uint32_t* out) {
  const U4 r = philox_block(seed, site, sweep, slot, tag);
  for (int i = 0; i < 4; ++i) out[i] = r.w[i];
}

double or_philox_uniform(uint32_t hi, uint32_t lo) { return philox_uniform(hi, lo); }

void or_philox_normal2(const uint32_t* blk, double* out) {
  U4 b{{blk[0], blk[1], blk[2], blk[3]}};
  philox_normal2(b, out[0], out[1]);
}

void or_keyed_proposal(uint64_t seed, int32_t site, int32_t sweep, const double* e, double step,
                       double* e2, double* u_acc) {
  keyed_proposal(seed, site, sweep, e, step, e2, u_acc);
}

void or_rotate(const double* e, const double* axis, double th, double* out) { rotate(e, axis, th, out); }

void or_zlm_row(int lmax, const double* u, double* out) { zlm_row(lmax, u, out); }

void or_cpow(double re, double im, int p, double* out) {
  const Cx r = cpow(Cx{re, im}, p);
  out[0] = r.re;
  out[1] = r.im;
}

// Term list: atoms/ls concatenated over terms (body[k] each), shifts 3 per member,
// folded concatenated (Π(2l+1) per term, column-major).
void* or_ham_build(int n_cell_atoms, int n_terms, const double* coef, const int32_t* body,
                   const int32_t* atoms, const int32_t* shifts, const int32_t* ls, const double* folded,
                   const int32_t* dims, const double* magmoms, const double* field) {
  std::vector<Term> raw(n_terms);
  size_t am = 0, fo = 0;
  for (int k = 0; k < n_terms; ++k) {
    Term& t = raw[k];
    t.coef = coef[k];
    size_t sz = 1;
    for (int m = 0; m < body[k]; ++m) {
      t.atoms.push_back(atoms[am + m]);
      t.ls.push_back(ls[am + m]);
      for (int c = 0; c < 3; ++c) t.shifts.push_back(shifts[3 * (am + m) + c]);
      sz *= (size_t)(2 * ls[am + m] + 1);
    }
    am += body[k];
    t.folded.assign(folded + fo, folded + fo + sz);
    fo += sz;
  }
  Ham* H = new Ham();
  std::string err;
  if (!build_ham(*H, n_cell_atoms, raw, dims, magmoms, field, err)) {
    g_err = err;
    delete H;
    return nullptr;
  }
  return H;
}

void or_ham_free(void* h) { delete static_cast<Ham*>(h); }

int64_t or_ham_scalar(void* h, const char* name) {
  const Ham& H = *static_cast<Ham*>(h);
  const std::string n(name);
  if (n == "n_sites") return H.n_sites;
  if (n == "nlm") return H.nlm;
  if (n == "lmax") return H.lmax;
  if (n == "n_colors") return H.n_colors;
  if (n == "n_active") return H.n_active;
  if (n == "n_cell_atoms") return H.n_cell_atoms;
  if (n == "n_terms") return (int64_t)H.terms.size();
  if (n == "n_fitted") return H.n_fitted;
  return -1;
}

// Array accessor: returns the length; copies into `out` when non-null.
// dtype code written to *code: 0 = int32, 1 = int8, 2 = uint8, 3 = float64.
int64_t or_ham_array(void* h, const char* name, void* out, int* code) {
  const Ham& H = *static_cast<Ham*>(h);
  const std::string n(name);
  auto i32 = [&](const std::vector<int32_t>& v) {
    *code = 0;
    if (out) std::memcpy(out, v.data(), v.size() * 4);
    return (int64_t)v.size();
  };
  auto i8 = [&](const std::vector<int8_t>& v) {
    *code = 1;
    if (out) std::memcpy(out, v.data(), v.size());
    return (int64_t)v.size();
  };
  auto u8 = [&](const std::vector<uint8_t>& v) {
    *code = 2;
    if (out) std::memcpy(out, v.data(), v.size());
    return (int64_t)v.size();
  };
  auto f64 = [&](const std::vector<double>& v) {
    *code = 3;
    if (out) std::memcpy(out, v.data(), v.size() * 8);
    return (int64_t)v.size();
  };
#define A32(x) \
  if (n == #x) return i32(H.x);
  A32(inst_term) A32(inst_ptr) A32(inst_sites) A32(site_ptr) A32(site_inst) A32(site_prog)
  A32(sprog_ptr) A32(sent_tgt) A32(sfac_ptr) A32(sfac_row) A32(site_col) A32(site_col2) A32(pent_row)
  A32(pent_row2) A32(eprog_ptr) A32(efac_ptr) A32(efac_row) A32(color_ptr) A32(color_sites)
#undef A32
  if (n == "site_slot") return i8(H.site_slot);
  if (n == "sfac_slot") return i8(H.sfac_slot);
  if (n == "site_has_l1") return u8(H.site_has_l1);
  if (n == "site_active") return u8(H.site_active);
  if (n == "sent_w") return f64(H.sent_w);
  if (n == "eent_w") return f64(H.eent_w);
  if (n == "term_coef") return f64(H.term_coef);
  *code = -1;
  return -1;
}

void or_zrows(void* h, const double* config, double* zrows) { zrows_of(*static_cast<Ham*>(h), config, zrows); }

double or_total_energy(void* h, const double* zrows) { return total_energy(*static_cast<Ham*>(h), zrows); }

double or_total_energy_ref(void* h, const double* zrows) {
  return total_energy_ref(*static_cast<Ham*>(h), zrows);
}

void or_grad_zlm_row(int lmax, const double* u, double* g) { grad_zlm_row(lmax, u, g); }

// All-site energy gradient (gpu_gradient.jl:131-243 semantics): G[s] = sum_t c_t(s)
// grad Z_t(e_s), c the leave-one-out coefficients of site s (energy.jl:100-139);
// config and G are 3 x n_sites (payload order).
void or_energy_gradient(void* h, const double* config, double* G) {
  const Ham& H = *static_cast<Ham*>(h);
  std::vector<double> zr((size_t)H.nlm * H.n_sites), c(H.nlm), g(3 * (size_t)H.nlm);
  zrows_of(H, config, zr.data());
  for (int s = 0; s < H.n_sites; ++s) {
    std::fill(c.begin(), c.end(), 0.0);
    site_coeffs(H, s + 1, zr.data(), c.data());
    grad_zlm_row(H.lmax, config + 3 * (size_t)s, g.data());
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int t = 0; t < H.nlm; ++t) {
      gx += c[t] * g[3 * t];
      gy += c[t] * g[3 * t + 1];
      gz += c[t] * g[3 * t + 2];
    }
    G[3 * (size_t)s] = gx;
    G[3 * (size_t)s + 1] = gy;
    G[3 * (size_t)s + 2] = gz;
  }
}

void or_site_coeffs(void* h, int s, const double* zrows, double* c) {
  site_coeffs(*static_cast<Ham*>(h), s, zrows, c);
}

void or_site_coeffs_ref(void* h, int s, const double* zrows, double* c) {
  site_coeffs_ref(*static_cast<Ham*>(h), s, zrows, c);
}

double or_delta_energy(int nlm, const double* c, const double* zold, const double* znew) {
  return delta_energy(nlm, c, zold, znew);
}

double or_entry_walk_partial(void* h, const double* zrows, const double* znew, int s, int lane, int ws) {
  return entry_walk_partial(*static_cast<Ham*>(h), zrows, znew, s, lane, ws);
}

int or_keyed_sweep(void* h, double* config, double* zrows, double* dE, int32_t* acc, double beta,
                   double step, uint64_t seed, int32_t sweep, int ws) {
  return keyed_sweep(*static_cast<Ham*>(h), config, zrows, dE, acc, beta, step, seed, sweep, ws);
}

double or_reduce_dE(void* h, const double* dE) { return reduce_dE(*static_cast<Ham*>(h), dE); }

// One step adaptation (updates.jl:296-305) of a chain whose Metropolis counters since
// the last adaptation are acc / att: returns the new step.
double or_adapt_step(double step, int64_t acc, int64_t att, double target) {
  Chain ch;
  ch.step = step;
  ch.acc_metro = acc;
  ch.att_metro = att;
  adapt_step(ch, target);
  return ch.step;
}

int or_swap_accepts(double kt_a, double kt_b, double E_a, double E_b, double u) {  // pt.jl:92-96
  const double logw = (1.0 / kt_a - 1.0 / kt_b) * (E_a - E_b);
  return u < std::exp(std::min(0.0, logw));
}

// Replay one device sweep through the FP64 energy path.
//   config: pre-sweep spins (3n, the device's FP32 values widened), updated in place
//           with the DEVICE's decisions so that the replay stays on its trajectory;
//   prop:   device proposal per site (3n); u: device accept uniform per site;
//   dev_acc: device accept flag per site.
// Outputs per site: dE64 (oracle ΔE of the device proposal on the current state),
// scale (Σ|c|·(Σ|znew|+Σ|zold|), the reference's tolerance scale, test_gpu.jl:168),
// oracle accept decision. Sites are visited in colour order (updates.jl:157-170).
// kind 0 = Metropolis (uniform read always), 1 = overrelaxation (ΔE<=0 accepts).
void or_replay_sweep(void* h, double* config, const double* prop, const double* u,
                     const uint8_t* dev_acc, double beta, double* dE64, double* scale,
                     uint8_t* or_acc, double* c_out) {
  const Ham& H = *static_cast<Ham*>(h);
  std::vector<double> zrows((size_t)H.nlm * H.n_sites), c(H.nlm), znew(H.nlm);
  zrows_of(H, config, zrows.data());
  for (int32_t s : H.color_sites) {
    std::fill(c.begin(), c.end(), 0.0);
    site_coeffs(H, s, zrows.data(), c.data());
    if (c_out) std::copy(c.begin(), c.end(), c_out + (size_t)H.nlm * (s - 1));
    const double* p = prop + 3 * (s - 1);
    zlm_row(H.lmax, p, znew.data());
    double* zs = zrows.data() + (size_t)H.nlm * (s - 1);
    const double d = delta_energy(H.nlm, c.data(), zs, znew.data());
    double sc = 0, sn = 0, so = 0;
    for (int k = 0; k < H.nlm; ++k) {
      sc += std::fabs(c[k]);
      sn += std::fabs(znew[k]);
      so += std::fabs(zs[k]);
    }
    dE64[s - 1] = d;
    scale[s - 1] = sc * (sn + so);
    or_acc[s - 1] = (d <= 0.0 || u[s - 1] < std::exp(-beta * d)) ? 1 : 0;
    if (dev_acc[s - 1]) {
      for (int k = 0; k < 3; ++k) config[3 * (s - 1) + k] = p[k];
      std::copy(znew.begin(), znew.end(), zs);
    }
  }
}

// Chain API for the CPU baseline and the statistics oracle --------------------
void* or_chain_new(void* h, const double* config, uint64_t seed, double step) {
  const Ham& H = *static_cast<Ham*>(h);
  Chain* ch = new Chain();
  ch->config.assign(config, config + 3 * H.n_sites);
  ch->zrows.assign((size_t)H.nlm * H.n_sites, 0.0);
  zrows_of(H, ch->config.data(), ch->zrows.data());
  ch->dE.assign(H.n_sites, 0.0);
  ch->energy = total_energy(H, ch->zrows.data());
  ch->seed = seed;
  ch->step = step;
  return ch;
}

void or_chain_free(void* c) { delete static_cast<Chain*>(c); }

void or_chain_get(void* c, double* config, double* energy, int64_t* sweep_index, int64_t* counters,
                  double* step) {
  Chain& ch = *static_cast<Chain*>(c);
  if (config) std::copy(ch.config.begin(), ch.config.end(), config);
  if (energy) *energy = ch.energy;
  if (sweep_index) *sweep_index = ch.sweep_index;
  if (counters) {
    counters[0] = ch.acc_metro;
    counters[1] = ch.att_metro;
    counters[2] = ch.acc_or;
    counters[3] = ch.att_or;
  }
  if (step) *step = ch.step;
}

void or_chain_sweeps(void* h, void* c, double beta, int64_t nsweeps, int n_or, int threads) {
  const Ham& H = *static_cast<Ham*>(h);
  Chain& ch = *static_cast<Chain*>(c);
  for (int64_t i = 0; i < nsweeps; ++i) compound_sweep(H, ch, beta, n_or, threads);
}

double or_chain_renormalize(void* h, void* c) {
  return renormalize(*static_cast<Ham*>(h), *static_cast<Chain*>(c));
}

int or_stats_len(void* h) { return stats_len(*static_cast<Ham*>(h)); }

// run_mc at one temperature (run.jl:156-205) on the keyed scheme: thermalise with
// step adaptation, renormalise + freeze, measure. Writes the stats block.
int or_run_mc(void* h, void* c, double kT, int64_t sweeps_therm, int64_t sweeps_measure,
              int64_t measure_interval, int n_or, double adapt_target, int64_t adapt_interval,
              int64_t renorm_interval, int nbins, int threads, double* out) {
  const Ham& H = *static_cast<Ham*>(h);
  Chain& ch = *static_cast<Chain*>(c);
  const double beta = 1.0 / kT;
  ch.max_drift = 0.0;
  for (int64_t sw = 1; sw <= sweeps_therm; ++sw) {
    compound_sweep(H, ch, beta, n_or, threads);
    if (sw % adapt_interval == 0) adapt_step(ch, adapt_target);
    if (sw % renorm_interval == 0) renormalize(H, ch);
  }
  renormalize(H, ch);
  ch.acc_metro = ch.att_metro = ch.acc_or = ch.att_or = 0;
  ch.max_drift = 0.0;
  Accums A = make_accums(H, sweeps_measure / measure_interval, nbins);
  for (int64_t sw = 1; sw <= sweeps_measure; ++sw) {
    compound_sweep(H, ch, beta, n_or, threads);
    if (sw % renorm_interval == 0) renormalize(H, ch);
    if (sw % measure_interval == 0) measure(H, ch, A);
  }
  finalize(H, A, ch, kT, out);
  return 0;
}

// run_pt over R rungs (pt.jl:372-430 schedule, serial reference order of
// gpu_pt.jl:115-140): lanes advance `exchange_interval` sweeps, then adjacent
// pairs of alternating parity attempt a payload swap with one uniform each,
// drawn from Philox (exchange_seed, pair, boundary, slot 0, tag 3).
// Lanes run concurrently over OpenMP threads (one lane per thread).
int or_run_pt(void* h, int R, void** chains, const double* kts, int64_t sweeps_therm,
              int64_t sweeps_measure, int64_t measure_interval, int64_t exchange_interval, int n_or,
              double adapt_target, int64_t adapt_interval, int64_t renorm_interval, int nbins,
              uint64_t exchange_seed, int threads, double* out, int64_t* swap_att, int64_t* swap_acc) {
  const Ham& H = *static_cast<Ham*>(h);
  std::vector<Chain*> ch(R);
  for (int r = 0; r < R; ++r) ch[r] = static_cast<Chain*>(chains[r]);
  std::vector<Accums> acc;
  std::vector<int64_t> phase_sweeps(R, 0);
  int parity = 0;
  int64_t boundary = 0;
  for (int i = 0; i < R - 1; ++i) swap_att[i] = swap_acc[i] = 0;
  for (int phase = 0; phase < 2; ++phase) {
    const bool meas = phase == 1;
    const int64_t total = meas ? sweeps_measure : sweeps_therm;
    if (meas) {
      for (int r = 0; r < R; ++r) {
        renormalize(H, *ch[r]);
        ch[r]->acc_metro = ch[r]->att_metro = ch[r]->acc_or = ch[r]->att_or = 0;
        ch[r]->max_drift = 0.0;
        acc.push_back(make_accums(H, sweeps_measure / measure_interval, nbins));
        phase_sweeps[r] = 0;
      }
    }
    int64_t done = 0;
    while (done < total) {
      const int64_t n = std::min(exchange_interval, total - done);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
      for (int r = 0; r < R; ++r) {
        Chain& c = *ch[r];
        const double beta = 1.0 / kts[r];
        for (int64_t k = 0; k < n; ++k) {
          phase_sweeps[r] += 1;
          compound_sweep(H, c, beta, n_or, 1);
          if (!meas && phase_sweeps[r] % adapt_interval == 0) adapt_step(c, adapt_target);
          if (phase_sweeps[r] % renorm_interval == 0) renormalize(H, c);
          if (meas && phase_sweeps[r] % measure_interval == 0) measure(H, c, acc[r]);
        }
      }
      done += n;
      if (done < total) {
        boundary += 1;
        for (int i = parity; i < R - 1; i += 2) {
          const U4 b = philox_block(exchange_seed, i + 1, (int32_t)boundary, 0u, 3u);
          const double u = philox_uniform(b.w[0], b.w[1]);
          swap_att[i] += 1;
          const double logw = (1.0 / kts[i] - 1.0 / kts[i + 1]) * (ch[i]->energy - ch[i + 1]->energy);
          if (u < std::exp(std::min(0.0, logw))) {
            std::swap(ch[i]->config, ch[i + 1]->config);
            std::swap(ch[i]->zrows, ch[i + 1]->zrows);
            std::swap(ch[i]->energy, ch[i + 1]->energy);
            swap_acc[i] += 1;
          }
        }
        parity = 1 - parity;
      }
    }
  }
  const int L = stats_len(H);
  for (int r = 0; r < R; ++r) finalize(H, acc[r], *ch[r], kts[r], out + (size_t)r * L);
  return 0;
}

// LogBinner / BinStore / jackknife exposed for cross-checks of the host statistics.
void or_logbinner_stats(const double* xs, int64_t n, double* mean, double* err, double* tau) {
  LogBinner b(1);
  for (int64_t i = 0; i < n; ++i) b.push(xs + i);
  *mean = b.mean(0);
  *err = b.std_error(0);
  *tau = b.tau_int(0);
}

double or_kb_ev() { return KB_EV; }
double or_mu_b_ev_t() { return MU_B_EV_T; }

int or_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
