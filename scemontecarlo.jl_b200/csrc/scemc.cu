// scemc.cu — libscemc_cuda.so: the chain-level colour-class Metropolis and
// overrelaxation sweep of SCEMonteCarlo.jl, written for B200 (sm_100a).
//
// Design (see include/scemc.h for the ABI):
//   * Tables. The reference's CSR-by-site tables (src/hamiltonian.jl:62-91,
//     234-265) are compiled once into a device adjacency of 16-byte records
//     {kind|offset, nb0, nb1, nb2}: one per (site, cluster instance), carrying the
//     neighbour site ids of the other members in ascending slot order. Programs
//     whose member l's are all in {1,2} and whose body order is <= 4 get a dense
//     FP32 coefficient tensor (target m first, then the other members' m) and a
//     fully unrolled contraction; every other program walks the reference's
//     sparse entry list (sent_w / sent_tgt / sfac_*), so any model the reference
//     accepts (lmax <= 6, any body order) runs.
//   * State. Spins are FP32 float4, stored site-major / replica-minor
//     (spins[site * R + r]) so that the replicas of one site sit in one 16*R-byte
//     line: the records of a site are read once per warp (broadcast) and the
//     neighbour gathers of consecutive replicas coalesce. Neighbour Z_lm rows are
//     recomputed in registers from the gathered spins (no zrows array).
//   * Sweep. Colour classes are processed in order; inside a class every
//     (site, replica) item is independent. A group of G lanes (1..32) handles one
//     item, striding over its records, and reduces the leave-one-out coefficient
//     vector c (src/energy.jl:100-139) with warp shuffles. dE = sum_k c_k(znew_k -
//     zold_k) in FP32 (energy.jl:148-157); the accept test uses FP64 exp.
//     Two launch forms: one kernel per colour (graph-captured), or one persistent
//     cooperative kernel per compound sweep with a bounded grid barrier between
//     colours.
//   * Energies. Accepted FP32 dE are converted to 2^-40 fixed point and summed in
//     int64 (order-free, so the FP64 running energy is independent of the launch
//     shape); FP64 is used for the running energy, the periodic full recompute
//     (fixed 1024-instance chunks, fixed-order reduction) and the observables.
#include "scemc.h"
#include "scemc_device.cuh"
#include "mlp.h"
#include "umma.cuh"
#include "vmf.cuh"

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

using namespace scemc;

namespace {

thread_local std::string t_err;

int32_t fail(int32_t code, const std::string& m) {
  t_err = m;
  return code;
}

#define CUDA_TRY(x)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess)                                                           \
      return fail(SCEMC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// A host-to-device copy that has landed on the device when it returns. From pageable
// memory cudaMemcpy may return once the source is staged, and the legacy stream's DMA
// is not ordered before kernels on the batches' non-blocking streams; waiting for the
// legacy stream closes that window. Used for tables and run parameters (not per step).
inline cudaError_t h2d_sync(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? cudaStreamSynchronize(0) : e;
}

enum Kind : int {
  K_GEN = 0,
  K_B1_L1 = 1,
  K_B1_L2 = 2,
  K_B2_11 = 3,
  K_B2_12 = 4,
  K_B2_21 = 5,
  K_B2_22 = 6,
  K_B3_111 = 7,
  K_B4_1111 = 8,
  K_B3_L2 = 9  // body 3, every member l in {1, 2}, not all l = 1 (fast tables only; the generic
               // records walk it as a sparse program)
};
constexpr int kKindShift = 26;
constexpr int32_t kOffMask = (1 << kKindShift) - 1;
constexpr double kFixScale = 1099511627776.0;  // 2^40: fixed-point unit of dE sums
constexpr int kMaxSlots = 512;
// Layout of the per-slot readback block (byte offsets per slot count n): energy (8n),
// slot_of_rung (4n, padded to 8n), counters (32n), swaps (16n), steps (8n),
// max_drift (8n).
constexpr size_t kRbEnergy = 0, kRbSlotOfRung = 8, kRbCounters = 16, kRbSwaps = 48, kRbSteps = 64,
                 kRbMaxDrift = 72, kReadbackBytesPerSlot = 80;
constexpr int kChunk = 1024;  // fixed reduction chunk (sites or instances)
constexpr int kMaxCellAtoms = 64;
constexpr int kRecPasses = 4;  // replay record: Metropolis + up to 3 overrelaxation passes

struct DevProg {
  int32_t e_lo, e_hi;  // sparse entries, 0-based half-open
  int32_t own_slot;    // 1-based member slot of the owning site
  int32_t body;
};

struct DevLattice {
  int32_t n_sites, nlm, lmax, n_colors, n_active, n_cell_atoms, R, slot0;
  int64_t spin_off;  // float4 index of (site 0, replica 0)
  int64_t n_inst;
  const int32_t* adj_ptr;  // n_sites+1, 0-based
  const int4* rec;
  const DevProg* prog;
  const float* tensor;
  const float* sent_w;
  const int8_t* sent_tgt;   // 0-based row
  const int32_t* sfac_ptr;  // 0-based, n_sent+1
  const int8_t* sfac_row;   // 0-based row
  const int8_t* sfac_slot;  // 1-based member slot
  const int32_t* inst_ptr;    // 0-based, n_inst+1
  const int32_t* inst_sites;  // 0-based
  const int32_t* color_ptr;    // 0-based, n_colors+1
  const int32_t* color_sites;  // 0-based site ids
  const uint8_t* has_l1;
  const uint8_t* active;
  // energy programs (FP64 recompute)
  const int32_t* inst_term;  // 0-based
  const int32_t* eprog_ptr;  // 0-based, n_terms+1
  const double* eent_w;
  const int32_t* efac_ptr;  // 0-based
  const int8_t* efac_row;   // 0-based
  const double* term_coef;
  // row-parallel fast tables (lmax 1 or 2, every program of a fast kind); fast == 0 otherwise
  int32_t fast, dmax;            // dmax: largest number of distinct neighbours of a site
  int32_t rmax, pad2;            // rmax: largest number of fast records of a site
  const int32_t* nb_ptr;         // n_sites+1: distinct neighbours of site s
  const int32_t* nb_list;        // 0-based site ids
  const int32_t* fr_ptr;         // n_sites+1: fast records of site s
  const uint32_t* fr_cnt;        // per site: n_pair | n_trip << 8 | n_quad << 16 | n_one << 24
  const int4* idesc;             // per colour position: {site | has_l1 << 30 | n_one << 31, nb offset,
                                 //   record offset, n_pair | n_trip << 8 | n_quad << 16 | n_nb << 24}
  const uint2* frec;             // {kind<<26 | tensor offset, local neighbour indices (8 bits each)}
  const float* ftensor;          // dense blocks, rows padded to the kernel's row count
  // learned proposal: environment of every site (n_sites x env_k, 0-based), per batch
  const int32_t* env;
  int32_t env_k, pad3;
  const int16_t* site_colour;  // 1-based colour of every site, 0 = inactive
};

// Grid barrier state (one per ensemble).
struct GridSync {
  unsigned long long arrived;  // monotonically increasing arrival count (never reset)
  int error;
  int pad;
};

// Per-ensemble device scalars.
struct EnsState {
  int32_t exchange_parity;
  int32_t exchange_count;
  int32_t error;
  uint32_t sweep;  // completed sweeps (the keyed stream's counter word is sweep + 1)
};

struct SweepArgs {
  const DevLattice* lat;
  int32_t n_lat;
  int32_t n_slots;
  float4* spins;
  const int32_t* seg;  // (max_colors) x (n_lat+1) item prefix per colour
  int32_t max_colors;
  int32_t colour;  // per-colour launch form
  int32_t pass;    // -1 Metropolis, k >= 0 overrelaxation pass k
  uint32_t sweep;  // 1-based counter word of this sweep
  const int32_t* rung_of_slot;
  const double* beta;   // per rung
  const double* step;   // per rung
  const unsigned long long* seed;  // per rung
  unsigned long long* dE_fix;      // per slot
  unsigned long long* cnt;         // per rung: [acc_metro, att_metro, acc_or, att_or]
  GridSync* gs;
  long long barrier_limit_ns;
  unsigned long long bar_base;  // arrival count at launch (persistent form)
  const EnsState* st;           // device sweep counter (read by every launch, so graphs stay valid)
  // replay recording (replica rec_r of lattice rec_li), may be null
  int32_t rec_li, rec_r, rec_cap;  // rec_cap: sites per recorded pass
  float* rec_prop;
  double* rec_u;
  float* rec_dE;
  uint8_t* rec_acc;
  // fast kernel: precomputed Metropolis proposals (null = computed inline)
  const int32_t* item_base;  // max_colors+1: first global item of each colour
  float4* prop;
  double* propu;
  const double* lqr;  // learned proposals: log q(e | env) - log q(e' | env) per item (null otherwise)
  double* rec_lqr;
  uint32_t* flags;    // data-flow form: per item slot, the pass epoch its update completed (null otherwise)
  int32_t dmax, rmax;
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void red_add_release(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Data-flow form: the pass epoch of a sweep (distinct for every (sweep, pass) with at
// most 6 overrelaxation passes; never 0, the flags' initial value).
__device__ __forceinline__ uint32_t flow_epoch(uint32_t sweep, int pass) { return sweep * 8u + (uint32_t)(pass + 2); }

// Waits until an item slot's flag holds `epoch`; bounded by limit_ns, after which the
// error word is set and every later wait gives up at once.
__device__ __forceinline__ bool wait_flag(const uint32_t* f, uint32_t epoch, int* err, long long limit_ns) {
  if (ld_acquire_u32(f) == epoch) return true;
  const unsigned long long t0 = globaltimer();
  for (unsigned int it = 0;; ++it) {
    if (ld_acquire_u32(f) == epoch) return true;
    if ((it & 15u) == 15u) {
      if (*(volatile int*)err) return false;
      if ((long long)(globaltimer() - t0) > limit_ns) {
        atomicExch(err, 1);
        return false;
      }
    }
    __nanosleep(20);
  }
}

// Barrier across all blocks of a cooperative launch on a monotonically increasing
// arrival counter: barrier k of a launch whose counter started at `base` completes
// when the counter reaches base + (k + 1) * nblocks. One fire-and-forget release
// add per block and acquire polling; the wait is bounded by limit_ns, after which
// the error word is set, every block leaves, and every later barrier fails at once.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, unsigned long long base, int k, unsigned int nblocks,
                                             long long limit_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* verr = &gs->error;
    int ok = *verr ? 0 : 1;
    if (ok) {
      __threadfence();
      red_add_release(&gs->arrived, 1ull);
      const unsigned long long target = base + (unsigned long long)(k + 1) * nblocks;
      const unsigned long long t0 = globaltimer();
      for (unsigned int it = 0;; ++it) {
        if (ld_acquire(&gs->arrived) >= target) break;
        if ((it & 31u) == 31u) {
          if (*verr) {
            ok = 0;
            break;
          }
          if ((long long)(globaltimer() - t0) > limit_ns) {
            atomicExch(&gs->error, 1);
            ok = 0;
            break;
          }
        }
        if (it > 64) __nanosleep(32);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <bool PERSIST>
__device__ __forceinline__ float4 load_spin(const float4* p) {
  if (PERSIST) return __ldcg(p);  // spins change between colours inside the launch
  return __ldg(p);
}

// Predicated add into a register array at a runtime index.
template <int N>
__device__ __forceinline__ void add_at(float* c, int k, float v) {
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (i == k) c[i] += v;
}

// Leave-one-out coefficients of one site over records [j0 + lane, j1) step G.
template <int LMAX, int G, bool PERSIST>
__device__ __forceinline__ void accumulate_c(const DevLattice& L, const float4* __restrict__ sp, int R, int r,
                                             int s, int lane, float* c) {
  constexpr int NLM = (LMAX + 1) * (LMAX + 1);
  const int j0 = L.adj_ptr[s], j1 = L.adj_ptr[s + 1];
  for (int j = j0 + lane; j < j1; j += G) {
    const int4 rc = __ldg(L.rec + j);
    const int kind = (int)((unsigned)rc.x >> kKindShift);
    const float* __restrict__ T = L.tensor + (rc.x & kOffMask);
    if (LMAX >= 1 && kind == K_B2_11) {
      const float4 n = load_spin<PERSIST>(sp + (int64_t)rc.y * R + r);
      float z[3];
      zrow_l1(n.x, n.y, n.z, z);
#pragma unroll
      for (int mt = 0; mt < 3; ++mt) {
        float a = c[1 + mt];
#pragma unroll
        for (int m = 0; m < 3; ++m) a = fmaf(__ldg(T + mt * 3 + m), z[m], a);
        c[1 + mt] = a;
      }
    } else if (LMAX >= 1 && kind == K_B1_L1) {
#pragma unroll
      for (int mt = 0; mt < 3; ++mt) c[1 + mt] += __ldg(T + mt);
    } else if (LMAX >= 1 && kind == K_B3_111) {
      const float4 n1 = load_spin<PERSIST>(sp + (int64_t)rc.y * R + r);
      const float4 n2 = load_spin<PERSIST>(sp + (int64_t)rc.z * R + r);
      float z1[3], z2[3];
      zrow_l1(n1.x, n1.y, n1.z, z1);
      zrow_l1(n2.x, n2.y, n2.z, z2);
#pragma unroll
      for (int mt = 0; mt < 3; ++mt) {
        float a = c[1 + mt];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          float t = 0.0f;
#pragma unroll
          for (int q = 0; q < 3; ++q) t = fmaf(__ldg(T + (mt * 3 + p) * 3 + q), z2[q], t);
          a = fmaf(z1[p], t, a);
        }
        c[1 + mt] = a;
      }
    } else if (LMAX >= 1 && kind == K_B4_1111) {
      const float4 n1 = load_spin<PERSIST>(sp + (int64_t)rc.y * R + r);
      const float4 n2 = load_spin<PERSIST>(sp + (int64_t)rc.z * R + r);
      const float4 n3 = load_spin<PERSIST>(sp + (int64_t)rc.w * R + r);
      float z1[3], z2[3], z3[3];
      zrow_l1(n1.x, n1.y, n1.z, z1);
      zrow_l1(n2.x, n2.y, n2.z, z2);
      zrow_l1(n3.x, n3.y, n3.z, z3);
#pragma unroll
      for (int mt = 0; mt < 3; ++mt) {
        float a = c[1 + mt];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          float t2 = 0.0f;
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            float t3 = 0.0f;
#pragma unroll
            for (int u = 0; u < 3; ++u) t3 = fmaf(__ldg(T + ((mt * 3 + p) * 3 + q) * 3 + u), z3[u], t3);
            t2 = fmaf(z2[q], t3, t2);
          }
          a = fmaf(z1[p], t2, a);
        }
        c[1 + mt] = a;
      }
    } else if (LMAX >= 2 && kind >= K_B2_12 && kind <= K_B2_22) {
      const float4 n = load_spin<PERSIST>(sp + (int64_t)rc.y * R + r);
      if (kind == K_B2_12) {  // target l=1, neighbour l=2
        float z[5];
        zrow_l2(n.x, n.y, n.z, z);
#pragma unroll
        for (int mt = 0; mt < 3; ++mt) {
          float a = c[1 + mt];
#pragma unroll
          for (int m = 0; m < 5; ++m) a = fmaf(__ldg(T + mt * 5 + m), z[m], a);
          c[1 + mt] = a;
        }
      } else if (kind == K_B2_21) {  // target l=2, neighbour l=1
        float z[3];
        zrow_l1(n.x, n.y, n.z, z);
#pragma unroll
        for (int mt = 0; mt < 5; ++mt) {
          float a = c[4 + mt];
#pragma unroll
          for (int m = 0; m < 3; ++m) a = fmaf(__ldg(T + mt * 3 + m), z[m], a);
          c[4 + mt] = a;
        }
      } else {  // K_B2_22
        float z[5];
        zrow_l2(n.x, n.y, n.z, z);
#pragma unroll
        for (int mt = 0; mt < 5; ++mt) {
          float a = c[4 + mt];
#pragma unroll
          for (int m = 0; m < 5; ++m) a = fmaf(__ldg(T + mt * 5 + m), z[m], a);
          c[4 + mt] = a;
        }
      }
    } else if (LMAX >= 2 && kind == K_B1_L2) {
#pragma unroll
      for (int mt = 0; mt < 5; ++mt) c[4 + mt] += __ldg(T + mt);
    } else {
      // Sparse generic walk: the reference's program entries (energy.jl:126-135).
      const DevProg pg = L.prog[rc.x & kOffMask];
      int base = 0;
      if (rc.y < 0) base = L.inst_ptr[-1 - rc.y];
      for (int e = pg.e_lo; e < pg.e_hi; ++e) {
        float p = 1.0f;
        for (int f = L.sfac_ptr[e]; f < L.sfac_ptr[e + 1]; ++f) {
          const int slot = L.sfac_slot[f];
          int nb;
          if (rc.y >= 0) {
            const int idx = slot - 1 - (slot > pg.own_slot ? 1 : 0);
            nb = idx == 0 ? rc.y : (idx == 1 ? rc.z : rc.w);
          } else {
            nb = L.inst_sites[base + slot - 1];
          }
          const float4 n = load_spin<PERSIST>(sp + (int64_t)nb * R + r);
          p *= zval_f32(L.sfac_row[f], n.x, n.y, n.z);
        }
        add_at<NLM>(c, L.sent_tgt[e], L.sent_w[e] * p);
      }
    }
  }
}

template <int NLM>
__device__ __forceinline__ float delta_e(const float* c, const float* zo, const float* zn) {
  float d = 0.0f;  // energy.jl:148-157 (row-difference form, zero coefficients skipped)
#pragma unroll
  for (int k = 0; k < NLM; ++k)
    if (c[k] != 0.0f) d = fmaf(c[k], zn[k] - zo[k], d);
  return d;
}

// Item enumeration of one colour: locate the lattice of a flat item index.
__device__ __forceinline__ int find_lattice(const int32_t* seg_c, int n_lat, int item) {
  int l = 0;
  while (l + 1 < n_lat && item >= seg_c[l + 1]) ++l;
  return l;
}

// Process colour `col` of the current pass: all (site, replica) items, G lanes each.
// Block-local accumulators (shared) collect fixed-point dE and counters per slot.
template <int LMAX, int G, bool PERSIST>
__device__ void sweep_colour(const SweepArgs& a, int col, unsigned long long* s_dE, unsigned int* s_cnt) {
  constexpr int NLM = (LMAX + 1) * (LMAX + 1);
  const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
  const int n_items = seg_c[a.n_lat];
  const int lane = threadIdx.x % G;
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int n_groups = (gridDim.x * blockDim.x) / G;
  const int rounds = (n_items + n_groups - 1) / n_groups;
  const unsigned int gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x % 32) / G * G));
  for (int rd = 0; rd < rounds; ++rd) {
    const int item = rd * n_groups + group;
    const bool valid = item < n_items;
    float c[NLM];
#pragma unroll
    for (int k = 0; k < NLM; ++k) c[k] = 0.0f;
    int li = 0, slot = 0, s = 0, r = 0, R = 1;
    const DevLattice* Lp = a.lat;
    if (valid) {
      li = find_lattice(seg_c, a.n_lat, item);
      Lp = a.lat + li;
      const int local = item - seg_c[li];
      R = Lp->R;
      const int q = local / R;
      r = local - q * R;
      s = Lp->color_sites[Lp->color_ptr[col] + q];
      slot = Lp->slot0 + r;
    }
    const DevLattice& L = *Lp;
    const float4* __restrict__ sp = a.spins + L.spin_off;
    const bool do_or = a.pass >= 0;
    const bool skip = !valid || (do_or && !L.has_l1[s]);
    if (!skip) accumulate_c<LMAX, G, PERSIST>(L, sp, R, r, s, lane, c);
    if (G > 1) {
#pragma unroll
      for (int o = G / 2; o >= 1; o >>= 1)
#pragma unroll
        for (int k = 0; k < NLM; ++k) c[k] += __shfl_xor_sync(gmask, c[k], o);
    }
    if (skip || lane != 0) continue;
    const int rung = a.rung_of_slot[slot];
    const double beta = a.beta[rung];
    const float4 e = load_spin<PERSIST>(sp + (int64_t)s * R + r);
    float px, py, pz;
    double u;
    bool attempted = true;
    if (!do_or) {
      u = keyed_proposal(a.seed[rung], (uint32_t)(s + 1), a.st->sweep + 1u, e.x, e.y, e.z, a.step[rung], px, py, pz);
    } else {
      // Reflection about the l = 1 field axis h = (c4, c2, c3) (updates.jl:66-87).
      const double h0 = LMAX >= 1 ? c[NLM > 3 ? 3 : 0] : 0.0, h1 = LMAX >= 1 ? c[NLM > 1 ? 1 : 0] : 0.0,
                   h2 = LMAX >= 1 ? c[NLM > 2 ? 2 : 0] : 0.0;
      const double hn = sqrt((h0 * h0 + h1 * h1) + h2 * h2);
      if (hn < 1e-12) {
        attempted = false;
        px = e.x, py = e.y, pz = e.z;
      } else {
        const double a0 = h0 / hn, a1 = h1 / hn, a2 = h2 / hn;
        const double d2 = 2.0 * (((double)e.x * a0 + (double)e.y * a1) + (double)e.z * a2);
        double r0 = d2 * a0 - e.x, r1 = d2 * a1 - e.y, r2 = d2 * a2 - e.z;
        const double rn = sqrt((r0 * r0 + r1 * r1) + r2 * r2);
        px = (float)(r0 / rn);
        py = (float)(r1 / rn);
        pz = (float)(r2 / rn);
      }
      const Blk b = philox_block(a.seed[rung], (uint32_t)(s + 1), a.st->sweep + 1u, (uint32_t)a.pass, kTagOR);
      u = philox_uniform(b.w0, b.w1);
    }
    float dE = 0.0f;
    bool acc = false;
    if (attempted) {
      float zo[NLM], zn[NLM];
      zrow_f32<LMAX>(e.x, e.y, e.z, zo);
      zrow_f32<LMAX>(px, py, pz, zn);
      dE = delta_e<NLM>(c, zo, zn);
      acc = dE <= 0.0f || u < exp(-beta * (double)dE);
    }
    if (acc) {
      a.spins[L.spin_off + (int64_t)s * R + r] = make_float4(px, py, pz, 0.0f);
      const long long fx = llrint((double)dE * kFixScale);
      atomicAdd(s_dE + slot, (unsigned long long)fx);
    }
    if (do_or) {
      if (attempted) atomicAdd(s_cnt + 3 * slot + 2, 1u);
      if (acc) atomicAdd(s_cnt + 3 * slot + 1, 1u);
    } else if (acc) {
      atomicAdd(s_cnt + 3 * slot + 0, 1u);
    }
    if (a.rec_prop != nullptr && li == a.rec_li && r == a.rec_r && a.pass + 1 < kRecPasses) {
      const int64_t q = (int64_t)(a.pass + 1) * a.rec_cap + s;
      a.rec_prop[3 * q + 0] = px;
      a.rec_prop[3 * q + 1] = py;
      a.rec_prop[3 * q + 2] = pz;
      a.rec_u[q] = u;
      a.rec_dE[q] = dE;
      a.rec_acc[q] = (uint8_t)(acc ? 1 : (attempted ? 0 : 2));
    }
  }
}

__device__ __forceinline__ void flush_block(const SweepArgs& a, unsigned long long* s_dE, unsigned int* s_cnt) {
  __syncthreads();
  for (int i = threadIdx.x; i < a.n_slots; i += blockDim.x) {
    if (s_dE[i]) atomicAdd(a.dE_fix + i, s_dE[i]);
    const int rung = a.rung_of_slot[i];
    if (s_cnt[3 * i + 0]) atomicAdd(a.cnt + 4 * rung + 0, (unsigned long long)s_cnt[3 * i + 0]);
    if (s_cnt[3 * i + 1]) atomicAdd(a.cnt + 4 * rung + 2, (unsigned long long)s_cnt[3 * i + 1]);
    if (s_cnt[3 * i + 2]) atomicAdd(a.cnt + 4 * rung + 3, (unsigned long long)s_cnt[3 * i + 2]);
    s_dE[i] = 0ull;
    s_cnt[3 * i + 0] = s_cnt[3 * i + 1] = s_cnt[3 * i + 2] = 0u;
  }
  __syncthreads();
}

__device__ __forceinline__ void zero_block(int n_slots, unsigned long long* s_dE, unsigned int* s_cnt) {
  for (int i = threadIdx.x; i < n_slots; i += blockDim.x) {
    s_dE[i] = 0ull;
    s_cnt[3 * i + 0] = s_cnt[3 * i + 1] = s_cnt[3 * i + 2] = 0u;
  }
  __syncthreads();
}

// One colour of one pass per launch.
template <int LMAX, int G>
__global__ void __launch_bounds__(256) k_sweep_colour(SweepArgs a) {
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  sweep_colour<LMAX, G, false>(a, a.colour, s_dE, s_cnt);
  flush_block(a, s_dE, s_cnt);
}

// One compound pass (every colour) per cooperative launch, bounded grid barrier
// between colours.
template <int LMAX, int G>
__global__ void __launch_bounds__(256) k_sweep_persistent(SweepArgs a) {
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  for (int col = 0; col < a.max_colors; ++col) {
    sweep_colour<LMAX, G, true>(a, col, s_dE, s_cnt);
    if (col + 1 < a.max_colors)
      if (!grid_barrier(a.gs, a.bar_base, col, gridDim.x, a.barrier_limit_ns)) break;
  }
  flush_block(a, s_dE, s_cnt);
}

// L2 read-bandwidth probe: each block reads a contiguous share of buf, `reps` times,
// with L2-only loads; the sum keeps the loads alive.
__global__ void __launch_bounds__(256) k_l2_probe(const float4* __restrict__ buf, int64_t n4, int reps, float* sink) {
  const int64_t per = (n4 + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = i0 + per < n4 ? i0 + per : n4;
  float acc = 0.0f;
  for (int k = 0; k < reps; ++k)
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const float4 v = __ldcg(buf + i);
      acc += (v.x + v.y) + (v.z + v.w);
    }
  if (acc == 1234.5f) sink[blockIdx.x] = acc;  // never true for a zeroed buffer; the loads stay
}

// Barrier self-test: nblocks_expected = gridDim.x + 1 can never be reached.
__global__ void k_barrier_selftest(GridSync* gs, long long limit_ns) {
  grid_barrier(gs, 0ull, 0, gridDim.x + 1, limit_ns);
}

// ---------------------------------------------------------------------------
// Row-parallel fast sweep (lmax 1 or 2; every program a dense l in {1,2} kind).
// A group of G lanes owns one (site, replica) item; lane t owns coefficient row
// t+1 (rows 1..NR; the l = 0 row never changes dE). Phase A gathers the site's
// distinct neighbours once and writes their Z rows to shared memory; phase B walks
// the site's records with every lane on the same record (per-neighbour merged
// NR x NR pair blocks, l = 1 triplets and quads, one merged body-1 vector); phase C
// reduces dE = sum_t c_t (znew_t - zold_t) with a fixed butterfly, so the result
// does not depend on the launch shape.
// ---------------------------------------------------------------------------
// F_TRIP2: a merged body-3 block with l in {1, 2} members, NR x NR x NR floats
// W[t][p][q] (t the site's row, p and q the rows of the neighbours with the smaller and
// the larger local index); counted with the l = 1 triplets, told apart by its kind.
constexpr int F_PAIR = 1, F_TRIP = 2, F_QUAD = 3, F_ONE = 4, F_TRIP2 = 5;

template <int NR>
__device__ __forceinline__ void zrow_nr(float x, float y, float z, float* o) {
  zrow_l1(x, y, z, o);
  if (NR > 3) zrow_l2(x, y, z, o + 3);
}

// Per-slot run parameters (beta, step, key) staged at the start of the fast kernel's
// dynamic shared memory: 3 x 8 bytes per slot, rounded to 16 bytes.
__host__ __device__ __forceinline__ size_t fast_param_floats(int n_slots) { return ((size_t)6 * n_slots + 3) & ~(size_t)3; }

__device__ __forceinline__ void stage_params(const SweepArgs& a, float* zsm) {
  double* b = reinterpret_cast<double*>(zsm);
  double* st = b + a.n_slots;
  unsigned long long* sd = reinterpret_cast<unsigned long long*>(st + a.n_slots);
  for (int i = threadIdx.x; i < a.n_slots; i += blockDim.x) {
    const int rung = a.rung_of_slot[i];
    b[i] = a.beta[rung];
    st[i] = a.step[rung];
    sd[i] = a.seed[rung];
  }
  __syncthreads();
}

// Shared-memory floats one warp of the fast kernel uses (host and device agree):
// rmax records (uint2) then dmax Z rows of NR floats, each region a multiple of 16 bytes.
__host__ __device__ __forceinline__ size_t fast_rec_floats(int rmax) { return (2 * (size_t)rmax + 3) & ~(size_t)3; }
__host__ __device__ __forceinline__ size_t fast_nbid_words(int dmax) { return ((size_t)dmax + 3) & ~(size_t)3; }
__host__ __device__ __forceinline__ size_t fast_group_floats(int dmax, int rmax, int NR) {
  return fast_rec_floats(rmax) + fast_nbid_words(dmax) + (((size_t)dmax * NR + 3) & ~(size_t)3);
}

// A warp's first item of the next colour, read before the grid barrier: its
// descriptor and own spin (registers) and its records and neighbour ids (the
// warp's shared memory). None of these change while the current colour updates.
struct FastPre {
  int item;  // -1: nothing prefetched
  int4 dsc;
  float4 e;
};

template <int N>
__device__ __forceinline__ float pick(const float* v, int k) {
  float r = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (i == k) r = v[i];
  return r;
}

__device__ __forceinline__ int find_colour(const int32_t* base, int n, int idx) {
  int lo = 0, hi = n;  // base[lo] <= idx < base[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (base[mid] <= idx) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Metropolis proposals of every item of the pass (they depend only on the item's
// own spin, which no earlier colour changes).
template <bool PERSIST>
__device__ void make_proposals(const SweepArgs& a) {
  const int total = a.item_base[a.max_colors];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int col = find_colour(a.item_base, a.max_colors, idx);
    const int item = idx - a.item_base[col];
    const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
    const int li = find_lattice(seg_c, a.n_lat, item);
    const DevLattice& L = a.lat[li];
    const int local = item - seg_c[li];
    const int q = local / L.R, r = local - (local / L.R) * L.R;
    const int s = L.color_sites[L.color_ptr[col] + q];
    const int rung = a.rung_of_slot[L.slot0 + r];
    const float4 e = load_spin<PERSIST>(a.spins + L.spin_off + (int64_t)s * L.R + r);
    float px, py, pz;
    const double u =
        keyed_proposal(a.seed[rung], (uint32_t)(s + 1), a.st->sweep + 1u, e.x, e.y, e.z, a.step[rung], px, py, pz);
    a.prop[idx] = make_float4(px, py, pz, 0.0f);
    a.propu[idx] = u;
  }
}

// The coefficient rows of one item from its records (rb) and its neighbours' Z rows
// (zb): row lane `row` sums its W rows over the records of slice `slice`; the
// slices are added with a fixed butterfly, so every lane of a row ends with c_row.
template <int NR, int G, int S>
__device__ __forceinline__ float fast_walk(const uint2* rb, const float* zb, const float* __restrict__ ft,
                                           int n_pair, int n_trip, int n_quad, int n_one, int row, int slice) {
  float acc = 0.0f, acc2 = 0.0f;
  // pairs: each row lane dots its W row with the neighbour's Z row
  if (row < NR) {
#pragma unroll 4
    for (int j = slice; j < n_pair; j += S) {
      const uint2 fr = rb[j];
      const float* z = zb + (fr.y & 0xffu) * NR;
      const float* w = ft + (fr.x & kOffMask) + row * NR;
      if (NR == 8) {
        const float4 w0 = __ldg(reinterpret_cast<const float4*>(w));
        const float4 w1 = __ldg(reinterpret_cast<const float4*>(w) + 1);
        const float4 z0 = *reinterpret_cast<const float4*>(z);
        const float4 z1 = *reinterpret_cast<const float4*>(z + 4);
        acc = fmaf(w0.x, z0.x, acc);
        acc2 = fmaf(w0.y, z0.y, acc2);
        acc = fmaf(w0.z, z0.z, acc);
        acc2 = fmaf(w0.w, z0.w, acc2);
        acc = fmaf(w1.x, z1.x, acc);
        acc2 = fmaf(w1.y, z1.y, acc2);
        acc = fmaf(w1.z, z1.z, acc);
        acc2 = fmaf(w1.w, z1.w, acc2);
      } else {
#pragma unroll
        for (int m = 0; m < NR; ++m) acc = fmaf(__ldg(w + m), z[m], acc);
      }
    }
  }
  // triplets: l = 1 blocks feed rows 1..3 only; merged blocks with l = 2 members
  // (NR = 8) feed every row: c_row += sum_p z1_p sum_q W[row][p][q] z2_q
  for (int j = n_pair + slice; j < n_pair + n_trip; j += S) {
    const uint2 fr = rb[j];
    const float* z1 = zb + (fr.y & 0xffu) * NR;
    const float* z2 = zb + ((fr.y >> 8) & 0xffu) * NR;
    if (NR == 8 && (fr.x >> kKindShift) == (uint32_t)F_TRIP2) {
      if (row < NR) {
        const float4* w4 = reinterpret_cast<const float4*>(ft + (fr.x & kOffMask) + row * NR * NR);
        const float4 za = *reinterpret_cast<const float4*>(z2), zc = *reinterpret_cast<const float4*>(z2 + 4);
#pragma unroll
        for (int p = 0; p < NR; ++p) {
          const float4 a0 = __ldg(w4 + 2 * p), a1 = __ldg(w4 + 2 * p + 1);
          float t = a0.x * za.x;
          t = fmaf(a0.y, za.y, t);
          t = fmaf(a0.z, za.z, t);
          t = fmaf(a0.w, za.w, t);
          t = fmaf(a1.x, zc.x, t);
          t = fmaf(a1.y, zc.y, t);
          t = fmaf(a1.z, zc.z, t);
          t = fmaf(a1.w, zc.w, t);
          acc2 = fmaf(z1[p], t, acc2);
        }
      }
    } else if (row < 3) {
      const float4* w4 = reinterpret_cast<const float4*>(ft + (fr.x & kOffMask) + row * 12);
      const float4 a0 = __ldg(w4), a1 = __ldg(w4 + 1), a2 = __ldg(w4 + 2);
      const float w[9] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x};
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const float t = fmaf(w[p * 3 + 0], z2[0], fmaf(w[p * 3 + 1], z2[1], w[p * 3 + 2] * z2[2]));
        acc = fmaf(z1[p], t, acc);
      }
    }
  }
  // l = 1 quads: rows 1..3 only
  if (row < 3) {
    for (int j = n_pair + n_trip + slice; j < n_pair + n_trip + n_quad; j += S) {
      const uint2 fr = rb[j];
      const float* z1 = zb + (fr.y & 0xffu) * NR;
      const float* z2 = zb + ((fr.y >> 8) & 0xffu) * NR;
      const float* z3 = zb + ((fr.y >> 16) & 0xffu) * NR;
      const float4* w4 = reinterpret_cast<const float4*>(ft + (fr.x & kOffMask) + row * 28);
      float w[28];
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        const float4 v = __ldg(w4 + k);
        w[4 * k] = v.x, w[4 * k + 1] = v.y, w[4 * k + 2] = v.z, w[4 * k + 3] = v.w;
      }
      const float z3a = z3[0], z3b = z3[1], z3c = z3[2];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        float t2 = 0.0f;
#pragma unroll
        for (int qq = 0; qq < 3; ++qq) {
          const int o = (p * 3 + qq) * 3;
          const float t3 = fmaf(w[o], z3a, fmaf(w[o + 1], z3b, w[o + 2] * z3c));
          t2 = fmaf(z2[qq], t3, t2);
        }
        acc = fmaf(z1[p], t2, acc);
      }
    }
  }
  if (n_one && slice == 0 && row < NR) {
    const uint2 fr = rb[n_pair + n_trip + n_quad];
    acc += __ldg(ft + (fr.x & kOffMask) + row);
  }
  acc += acc2;
#pragma unroll
  for (int o = G; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

struct FastMove {
  float px, py, pz, dE;
  double u;
  bool attempted, acc_ok;
};

// The move of one item from its coefficient rows (acc, one row per row lane): the
// proposal (Metropolis: precomputed or drawn from the keyed stream; overrelaxation:
// reflection about the l = 1 field h = (c4, c2, c3)), dE = sum_t c_t (znew_t - zold_t)
// summed over the row lanes with a fixed butterfly, and the decision (Metropolis, or
// Metropolis-Hastings with the learned density ratio lq). Every lane gets the result.
template <int NR, int G>
__device__ __forceinline__ FastMove fast_decide(float acc, float4 e, int row, int pass, bool have_prop, float4 p4,
                                                double u_pre, bool mh, double lq, double beta,
                                                unsigned long long seed, double step, uint32_t site1,
                                                uint32_t sweep1) {
  const bool do_or = pass >= 0;
  float px, py, pz;
  double u;
  bool attempted = true;
  if (!do_or) {
    if (have_prop) {
      px = p4.x, py = p4.y, pz = p4.z;
      u = u_pre;
    } else {
      u = keyed_proposal(seed, site1, sweep1, e.x, e.y, e.z, step, px, py, pz);
    }
  } else {
    // reflection about h = (c4, c2, c3): rows 3, 1, 2 live in lanes 2, 0, 1
    const double h0 = __shfl_sync(0xffffffffu, acc, 2);
    const double h1 = __shfl_sync(0xffffffffu, acc, 0);
    const double h2 = __shfl_sync(0xffffffffu, acc, 1);
    const double hn = sqrt((h0 * h0 + h1 * h1) + h2 * h2);
    if (hn < 1e-12) {
      attempted = false;
      px = e.x, py = e.y, pz = e.z;
    } else {
      const double a0 = h0 / hn, a1 = h1 / hn, a2 = h2 / hn;
      const double d2 = 2.0 * (((double)e.x * a0 + (double)e.y * a1) + (double)e.z * a2);
      const double r0 = d2 * a0 - e.x, r1 = d2 * a1 - e.y, r2 = d2 * a2 - e.z;
      const double rn = sqrt((r0 * r0 + r1 * r1) + r2 * r2);
      px = (float)(r0 / rn);
      py = (float)(r1 / rn);
      pz = (float)(r2 / rn);
    }
    const Blk bk = philox_block(seed, site1, sweep1, (uint32_t)pass, kTagOR);
    u = philox_uniform(bk.w0, bk.w1);
  }
  float zo[NR], zn[NR];
  zrow_nr<NR>(e.x, e.y, e.z, zo);
  zrow_nr<NR>(px, py, pz, zn);
  float term = 0.0f;
  if (row < NR && acc != 0.0f) term = acc * (pick<NR>(zn, row) - pick<NR>(zo, row));
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) term += __shfl_xor_sync(0xffffffffu, term, o);
  const float dE = attempted ? term : 0.0f;
  bool acc_ok;
  if (!do_or && mh) {  // Metropolis-Hastings with the learned proposal's density ratio
    const double la = -beta * (double)dE + lq;
    acc_ok = la >= 0.0 || u < exp(la);
  } else {
    acc_ok = attempted && (dE <= 0.0f || u < exp(-beta * (double)dE));
  }
  FastMove m;
  m.px = px, m.py = py, m.pz = pz, m.dE = dE, m.u = u, m.attempted = attempted, m.acc_ok = acc_ok;
  return m;
}

template <int LMAX, bool PERSIST>
__device__ void fast_colour(const SweepArgs& a, int col, unsigned long long* s_dE, unsigned int* s_cnt,
                            float* zsm, FastPre& pre, int next_col) {
  // One warp per (site, replica) item: lane = slice * G + row. The G row lanes own
  // coefficient rows 1..NR; the S = 32 / G slices split the site's records
  // (record j goes to slice j % S) and are summed with a fixed butterfly.
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  constexpr int G = NR <= 4 ? 4 : 8;
  constexpr int S = 32 / G;
  const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
  const int n_items = seg_c[a.n_lat];
  const int lane = threadIdx.x & 31;
  const int row = lane % G, slice = lane / G;
  const int wib = threadIdx.x >> 5;
  const int warps_per_block = blockDim.x >> 5;
  const int warp = blockIdx.x * warps_per_block + wib;
  const int n_warps = gridDim.x * warps_per_block;
  const size_t per_warp = fast_group_floats(a.dmax, a.rmax, NR);
  uint2* rb = reinterpret_cast<uint2*>(zsm + fast_param_floats(a.n_slots) + (size_t)wib * per_warp);
  int* nbid = reinterpret_cast<int*>(zsm + fast_param_floats(a.n_slots) + (size_t)wib * per_warp +
                                     fast_rec_floats(a.rmax));
  float* zb = zsm + fast_param_floats(a.n_slots) + (size_t)wib * per_warp + fast_rec_floats(a.rmax) +
              fast_nbid_words(a.dmax);
  const double* p_beta = reinterpret_cast<const double*>(zsm);
  const double* p_step = p_beta + a.n_slots;
  const unsigned long long* p_seed = reinterpret_cast<const unsigned long long*>(p_step + a.n_slots);
  const bool do_or = a.pass >= 0;
  for (int item = warp; item < n_items; item += n_warps) {  // warp-uniform
    const int li = find_lattice(seg_c, a.n_lat, item);
    const DevLattice& L = a.lat[li];
    const int local = item - seg_c[li];
    const int R = L.R;
    const int q = local / R;
    const int r = local - q * R;
    const bool have = item == pre.item;  // warp-uniform
    const int4 dsc = have ? pre.dsc : __ldg(L.idesc + __ldg(L.color_ptr + col) + q);
    const int s = dsc.x & 0x3fffffff;
    const uint32_t epoch = a.flags ? flow_epoch(a.st->sweep, a.pass) : 0u;
    if (do_or && !(dsc.x & (1 << 30))) {  // warp-uniform: no l = 1 channel
      if (a.flags && lane == 0) st_release_u32(a.flags + L.spin_off + (int64_t)s * R + r, epoch);
      continue;
    }
    const int slot = L.slot0 + r;
    const float4* __restrict__ sp = a.spins + L.spin_off;
    // independent loads of the item, issued before the table walk
    const float4 e = have ? pre.e : load_spin<PERSIST>(sp + (int64_t)s * R + r);
    float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f);
    double u_pre = 0.0, lq = 0.0;
    if (!do_or && a.prop != nullptr) {
      const int idx = a.item_base[col] + item;
      p4 = a.prop[idx];
      u_pre = a.propu[idx];
      if (a.lqr != nullptr) lq = a.lqr[idx];
    }
    const int n0 = dsc.y, j0 = dsc.z;
    const uint32_t cnt = (uint32_t)dsc.w;
    const int nd = (int)(cnt >> 24);
    const int n_pair = (int)(cnt & 0xffu), n_trip = (int)((cnt >> 8) & 0xffu), n_quad = (int)((cnt >> 16) & 0xffu);
    const int n_one = (dsc.x >> 31) & 1;
    const int nrec = n_pair + n_trip + n_quad + n_one;
    // every record and neighbour spin of the site is requested before any is used
    if (have) {
      for (int k = lane; k < nd; k += 32) {
        const float4 v = load_spin<PERSIST>(sp + (int64_t)nbid[k] * R + r);
        zrow_nr<NR>(v.x, v.y, v.z, zb + k * NR);
      }
    } else {
      for (int k = lane; k < nrec; k += 32) rb[k] = __ldg(L.frec + j0 + k);
      for (int k = lane; k < nd; k += 32) {
        const int nb = __ldg(L.nb_list + n0 + k);
        if (a.flags) {  // a neighbour of an earlier colour must have finished this pass
          const int cn = __ldg(L.site_colour + nb);
          if (cn > 0 && cn <= col) wait_flag(a.flags + L.spin_off + (int64_t)nb * R + r, epoch, &a.gs->error,
                                             a.barrier_limit_ns);
        }
        const float4 v = load_spin<PERSIST>(sp + (int64_t)nb * R + r);
        zrow_nr<NR>(v.x, v.y, v.z, zb + k * NR);
      }
    }
    __syncwarp();
    const float acc = fast_walk<NR, G, S>(rb, zb, L.ftensor, n_pair, n_trip, n_quad, n_one, row, slice);
    __syncwarp();  // rb / zb are rewritten for the next item
    const FastMove mv = fast_decide<NR, G>(acc, e, row, a.pass, !do_or && a.prop != nullptr, p4, u_pre,
                                           a.lqr != nullptr, lq, p_beta[slot], p_seed[slot], p_step[slot],
                                           (uint32_t)(s + 1), a.st->sweep + 1u);
    const float px = mv.px, py = mv.py, pz = mv.pz, dE = mv.dE;
    const double u = mv.u;
    const bool attempted = mv.attempted, acc_ok = mv.acc_ok;
    if (lane != 0) continue;
    if (acc_ok) {
      a.spins[L.spin_off + (int64_t)s * R + r] = make_float4(px, py, pz, 0.0f);
      atomicAdd(s_dE + slot, (unsigned long long)llrint((double)dE * kFixScale));
    }
    if (a.flags) st_release_u32(a.flags + L.spin_off + (int64_t)s * R + r, epoch);  // after the spin store
    if (do_or) {
      if (attempted) atomicAdd(s_cnt + 3 * slot + 2, 1u);
      if (acc_ok) atomicAdd(s_cnt + 3 * slot + 1, 1u);
    } else if (acc_ok) {
      atomicAdd(s_cnt + 3 * slot + 0, 1u);
    }
    if (a.rec_prop != nullptr && li == a.rec_li && r == a.rec_r && a.pass + 1 < kRecPasses) {
      const int64_t qq = (int64_t)(a.pass + 1) * a.rec_cap + s;
      a.rec_prop[3 * qq + 0] = px;
      a.rec_prop[3 * qq + 1] = py;
      a.rec_prop[3 * qq + 2] = pz;
      a.rec_u[qq] = u;
      a.rec_dE[qq] = dE;
      a.rec_acc[qq] = (uint8_t)(acc_ok ? 1 : (attempted ? 0 : 2));
      if (a.rec_lqr != nullptr && !do_or) a.rec_lqr[s] = lq;
    }
  }
  // prefetch this warp's first item of the next colour (before the grid barrier)
  pre.item = -1;
  if (next_col < 0) return;
  const int32_t* seg_n = a.seg + (size_t)next_col * (a.n_lat + 1);
  if (warp >= seg_n[a.n_lat]) return;
  __syncwarp();
  const int li = find_lattice(seg_n, a.n_lat, warp);
  const DevLattice& L = a.lat[li];
  const int local = warp - seg_n[li];
  const int q = local / L.R, r = local - q * L.R;
  const int4 dsc = __ldg(L.idesc + __ldg(L.color_ptr + next_col) + q);
  if (do_or && !(dsc.x & (1 << 30))) return;
  const int s = dsc.x & 0x3fffffff;
  const uint32_t cnt = (uint32_t)dsc.w;
  const int nd = (int)(cnt >> 24);
  const int nrec = (int)(cnt & 0xffu) + (int)((cnt >> 8) & 0xffu) + (int)((cnt >> 16) & 0xffu) + ((dsc.x >> 31) & 1);
  for (int k = lane; k < nrec; k += 32) rb[k] = __ldg(L.frec + dsc.z + k);
  for (int k = lane; k < nd; k += 32) nbid[k] = __ldg(L.nb_list + dsc.y + k);
  pre.e = load_spin<PERSIST>(a.spins + L.spin_off + (int64_t)s * L.R + r);
  pre.dsc = dsc;
  pre.item = warp;
  __syncwarp();
}

// 64 registers (eight 128-thread blocks per SM): a colour of the 5-chain bcc 16^3
// workload then runs its items in one wave. Measured on that workload: 108
// registers (two waves) 12 % slower; 80 or 96 registers with 128-thread blocks
// (one wave, fewer spills) 9 % and 13 % slower; 256-thread blocks 1 % slower.
#ifndef SCEMC_FAST_MINB
#define SCEMC_FAST_MINB 8
#endif
#ifndef SCEMC_FAST_THREADS
#define SCEMC_FAST_THREADS 128
#endif
#define SCEMC_FAST_BOUNDS __launch_bounds__(SCEMC_FAST_THREADS, SCEMC_FAST_MINB)

template <int LMAX>
__global__ void SCEMC_FAST_BOUNDS k_fast_colour(SweepArgs a) {
  extern __shared__ __align__(16) float zsm[];
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  stage_params(a, zsm);
  FastPre pre;
  pre.item = -1;
  fast_colour<LMAX, false>(a, a.colour, s_dE, s_cnt, zsm, pre, -1);
  flush_block(a, s_dE, s_cnt);
}

template <int LMAX>
__global__ void SCEMC_FAST_BOUNDS k_fast_persistent(SweepArgs a) {
  extern __shared__ __align__(16) float zsm[];
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  stage_params(a, zsm);
  bool ok = true;
  int k = 0;
  if (a.pass < 0 && a.prop != nullptr) {
    make_proposals<true>(a);
    ok = grid_barrier(a.gs, a.bar_base, k++, gridDim.x, a.barrier_limit_ns);
  }
  FastPre pre;
  pre.item = -1;
  for (int col = 0; ok && col < a.max_colors; ++col) {
    if (a.flags) {  // data flow: items wait on their earlier-colour neighbours' flags instead of a barrier
      fast_colour<LMAX, true>(a, col, s_dE, s_cnt, zsm, pre, -1);
      continue;
    }
    fast_colour<LMAX, true>(a, col, s_dE, s_cnt, zsm, pre, col + 1 < a.max_colors ? col + 1 : -1);
    if (col + 1 < a.max_colors) ok = grid_barrier(a.gs, a.bar_base, k++, gridDim.x, a.barrier_limit_ns);
  }
  flush_block(a, s_dE, s_cnt);
}

__global__ void __launch_bounds__(256) k_proposals(SweepArgs a) { make_proposals<false>(a); }

// ---------------------------------------------------------------------------
// Chain-resident cluster sweep (row-parallel arithmetic, one launch per compound
// sweep). For chains small enough that one replica's spins fit in shared memory
// (16 bytes a site), a thread-block cluster owns one replica slot and every CTA of
// the cluster holds a full copy of that replica's spins. Each colour is split over
// the cluster's warps (one warp per site, the row-parallel record walk of
// fast_walk / fast_decide reading the neighbours from the local copy); an accepted
// spin is written into every CTA's copy through distributed shared memory, and the
// hardware cluster barrier separates the colours, so a colour costs a barrier
// instead of a kernel boundary and its neighbour reads never leave the SM. The
// cluster's CTAs are co-scheduled by construction, and every thread of every CTA
// takes the same barriers, so no wait can be left hanging. The chain's spins are
// loaded at the start and written back at the end of the compound sweep (one
// Metropolis pass, then n_or overrelaxation passes); arithmetic and decisions are
// those of k_fast_colour, bit for bit.
// ---------------------------------------------------------------------------
constexpr int kClusterThreads = 512;

__host__ __device__ __forceinline__ size_t cluster_smem_bytes(int n_sites, int dmax, int rmax, int nr) {
  return (size_t)n_sites * 16 + (size_t)(kClusterThreads / 32) * fast_group_floats(dmax, rmax, nr) * 4;
}

template <int LMAX>
__global__ void __launch_bounds__(kClusterThreads, 1) k_chain_cluster(SweepArgs a, int n_or) {
  namespace cg = cooperative_groups;
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  constexpr int G = NR <= 4 ? 4 : 8;
  constexpr int S = 32 / G;
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int csize = (int)cluster.num_blocks();
  const int slot = blockIdx.x / csize;  // one cluster per replica slot
  int li = 0;
  while (li + 1 < a.n_lat && slot >= a.lat[li + 1].slot0) ++li;
  const DevLattice& L = a.lat[li];
  const int R = L.R, r = slot - L.slot0, ns = L.n_sites;
  const int rung = a.rung_of_slot[slot];
  const double beta = a.beta[rung], step = a.step[rung];
  const unsigned long long seed = a.seed[rung];
  extern __shared__ __align__(16) float zsm[];
  float4* sspin = reinterpret_cast<float4*>(zsm);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int row = lane % G, slice = lane / G;
  const int wpb = blockDim.x >> 5;
  const size_t per_warp = fast_group_floats(a.dmax, a.rmax, NR);
  float* wbase = zsm + (size_t)ns * 4 + (size_t)wib * per_warp;
  uint2* rb = reinterpret_cast<uint2*>(wbase);
  int* nbid = reinterpret_cast<int*>(wbase + fast_rec_floats(a.rmax));
  float* zb = wbase + fast_rec_floats(a.rmax) + fast_nbid_words(a.dmax);
  __shared__ unsigned long long s_dE;
  __shared__ unsigned int s_cnt[3];
  if (threadIdx.x == 0) s_dE = 0ull, s_cnt[0] = s_cnt[1] = s_cnt[2] = 0u;
  float4* __restrict__ gsp = a.spins + L.spin_off;
  for (int s = threadIdx.x; s < ns; s += blockDim.x) sspin[s] = __ldcg(gsp + (int64_t)s * R + r);
  cluster.sync();  // every copy is complete before any CTA writes into another's
  const uint32_t sweep1 = a.st->sweep + 1u;
  // The static tables of a warp's first item of a colour (descriptor, records,
  // neighbour ids) are read before the barrier that ends the previous colour, so
  // their latency overlaps the wait; the spins are read after it.
  int pre_q = -1;
  int4 pre_dsc = make_int4(0, 0, 0, 0);
  auto load_tables = [&](int4 dsc) {
    const uint32_t cnt = (uint32_t)dsc.w;
    const int nrec = (int)(cnt & 0xffu) + (int)((cnt >> 8) & 0xffu) + (int)((cnt >> 16) & 0xffu) + ((dsc.x >> 31) & 1);
    for (int k = lane; k < nrec; k += 32) rb[k] = __ldg(L.frec + dsc.z + k);
    for (int k = lane; k < (int)(cnt >> 24); k += 32) nbid[k] = __ldg(L.nb_list + dsc.y + k);
  };
  auto prefetch = [&](int pass, int col) {
    pre_q = -1;
    if (col >= a.max_colors) return;
    const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
    const int q = crank * wpb + wib;
    if (q >= (seg_c[li + 1] - seg_c[li]) / R) return;
    pre_dsc = __ldg(L.idesc + __ldg(L.color_ptr + col) + q);
    if (pass >= 0 && !(pre_dsc.x & (1 << 30))) return;  // skipped by the overrelaxation pass
    load_tables(pre_dsc);
    pre_q = q;
  };
  prefetch(-1, 0);
  for (int pass = -1; pass < n_or; ++pass) {
    const bool do_or = pass >= 0;
    for (int col = 0; col < a.max_colors; ++col) {
      const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
      const int nq = (seg_c[li + 1] - seg_c[li]) / R;
      for (int q = crank * wpb + wib; q < nq; q += csize * wpb) {  // warp-uniform
        const bool have = q == pre_q;
        const int4 dsc = have ? pre_dsc : __ldg(L.idesc + __ldg(L.color_ptr + col) + q);
        const int site = dsc.x & 0x3fffffff;
        if (do_or && !(dsc.x & (1 << 30))) continue;  // no l = 1 channel
        const float4 e = sspin[site];
        float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f);
        double u_pre = 0.0;
        const bool have_prop = !do_or && a.prop != nullptr;
        if (have_prop) {
          const int idx = a.item_base[col] + seg_c[li] + q * R + r;
          p4 = a.prop[idx];
          u_pre = a.propu[idx];
        }
        const uint32_t cnt = (uint32_t)dsc.w;
        const int nd = (int)(cnt >> 24);
        const int n_pair = (int)(cnt & 0xffu), n_trip = (int)((cnt >> 8) & 0xffu), n_quad = (int)((cnt >> 16) & 0xffu);
        const int n_one = (dsc.x >> 31) & 1;
        if (!have) {
          load_tables(dsc);
          __syncwarp();
        }
        pre_q = -1;
        for (int k = lane; k < nd; k += 32) {
          const float4 v = sspin[nbid[k]];
          zrow_nr<NR>(v.x, v.y, v.z, zb + k * NR);
        }
        __syncwarp();
        const float acc = fast_walk<NR, G, S>(rb, zb, L.ftensor, n_pair, n_trip, n_quad, n_one, row, slice);
        __syncwarp();  // rb / nbid / zb are rewritten for the next item
        const FastMove mv = fast_decide<NR, G>(acc, e, row, pass, have_prop, p4, u_pre, false, 0.0, beta, seed, step,
                                               (uint32_t)(site + 1), sweep1);
        if (mv.acc_ok && lane < csize) {  // the new spin into every CTA's copy
          float4* dst = cluster.map_shared_rank(sspin + site, (unsigned)lane);
          *dst = make_float4(mv.px, mv.py, mv.pz, 0.0f);
        }
        if (lane != 0) continue;
        if (mv.acc_ok) atomicAdd(&s_dE, (unsigned long long)llrint((double)mv.dE * kFixScale));
        if (do_or) {
          if (mv.attempted) atomicAdd(s_cnt + 2, 1u);
          if (mv.acc_ok) atomicAdd(s_cnt + 1, 1u);
        } else if (mv.acc_ok) {
          atomicAdd(s_cnt + 0, 1u);
        }
        if (a.rec_prop != nullptr && li == a.rec_li && r == a.rec_r && pass + 1 < kRecPasses) {
          const int64_t qq = (int64_t)(pass + 1) * a.rec_cap + site;
          a.rec_prop[3 * qq + 0] = mv.px;
          a.rec_prop[3 * qq + 1] = mv.py;
          a.rec_prop[3 * qq + 2] = mv.pz;
          a.rec_u[qq] = mv.u;
          a.rec_dE[qq] = mv.dE;
          a.rec_acc[qq] = (uint8_t)(mv.acc_ok ? 1 : (mv.attempted ? 0 : 2));
        }
      }
      __syncwarp();
      if (col + 1 < a.max_colors) prefetch(pass, col + 1);
      else if (pass + 1 < n_or) prefetch(pass + 1, 0);
      __syncwarp();
      cluster.sync();  // this colour's spins are in every copy before the next colour reads them
    }
  }
  // every copy is identical: each CTA writes back its share of the sites
  const int per = (ns + csize - 1) / csize;
  const int s0 = crank * per, s1 = min(ns, s0 + per);
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) gsp[(int64_t)s * R + r] = sspin[s];
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_dE) atomicAdd(a.dE_fix + slot, s_dE);
    if (s_cnt[0]) atomicAdd(a.cnt + 4 * rung + 0, (unsigned long long)s_cnt[0]);
    if (s_cnt[1]) atomicAdd(a.cnt + 4 * rung + 2, (unsigned long long)s_cnt[1]);
    if (s_cnt[2]) atomicAdd(a.cnt + 4 * rung + 3, (unsigned long long)s_cnt[2]);
  }
}


// ---------------------------------------------------------------------------
// Replica-parallel sweep (same tables as the row-parallel kernel). A thread owns P
// replicas of one site: r = g, g + G, ..., g + (P-1) G with G = ceil(R / P), so the
// G threads of a site read each neighbour's replicas as contiguous float4 runs.
// Every coupling word (descriptor, record, W block) a thread loads serves its P
// replicas. When a colour fills many waves (fcc 64^3 x 32 rungs) the load's register
// writeback, not the FMA pipe, bounds a one-replica thread and P = 2 at 80 registers
// measured fastest (7.7 against 9.3 ms per pass at fcc 48^3). When a colour is small
// (the PT ladders) each thread's record walk is latency-bound: P = 1 at 64
// registers with twice the threads measured 0.49 against 0.54 ms per step, and two
// threads per item (NP = 2, rep_form) 0.41.
// Each replica keeps its NR coefficients in registers, c_t = sum_j W_j[t, :] . z_j,
// and forms
// dE = sum_t c_t (znew_t - zold_t) itself (no shuffles or shared-memory rows). Built
// for large replica counts (many PT rungs of one Hamiltonian).
// ---------------------------------------------------------------------------

// The leave-one-out coefficients c[k][t] = sum_j W_j[t, :] . z_j of P replicas
// (r = g + k G, those with ok[k]) of the site of descriptor `dsc`, from every record's
// W block and its neighbours' Z rows. PF: the neighbour rows are prefetched into L1
// first and read through it (else through L2); a template parameter, so the
// many-wave form carries no per-load branch.
// NP > 1: only the records j with j % NP == part (the one-body record with part 0),
// for NP threads that share one site's walk. PAIRS = false: every record but the
// pair records (whose sum the caller forms on the tensor cores).
template <int LMAX, int P, int NP, bool PF, bool T2 = (LMAX == 2), bool PAIRS = true>
__device__ __forceinline__ void rep_coeffs(const DevLattice& L, const float4* __restrict__ sp, int4 dsc, int R, int G,
                                           int g, const bool (&ok)[P],
                                           float (&c)[P][(LMAX + 1) * (LMAX + 1) - 1], int part = 0) {
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  const int n0 = dsc.y, j0 = dsc.z;
  const uint32_t cnt = (uint32_t)dsc.w;
  const int n_pair = (int)(cnt & 0xffu), n_trip = (int)((cnt >> 8) & 0xffu), n_quad = (int)((cnt >> 16) & 0xffu);
  const int n_one = (dsc.x >> 31) & 1;
  const uint2* __restrict__ fr = L.frec + j0;
  const int32_t* __restrict__ nbl = L.nb_list + n0;
  const float* __restrict__ ft = L.ftensor;
  // the P replicas' spins of neighbour `loc` (unused replicas read replica g)
  auto gather = [&](int loc, float4* v) {
    const float4* b = sp + (int64_t)__ldg(nbl + loc) * R + g;
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = PF ? __ldg(b + (ok[k] ? k * G : 0)) : __ldcg(b + (ok[k] ? k * G : 0));
  };
  if (PF) {  // the site's records and every neighbour row requested at once; the walk then hits L1
    const int nd = (int)(cnt >> 24);
    const int nrec = n_pair + n_trip + n_quad + n_one;
    for (int j = 0; j < nrec; j += 16) asm volatile("prefetch.global.L1 [%0];" ::"l"(fr + j));
    if (nrec > 0) asm volatile("prefetch.global.L1 [%0];" ::"l"(fr + nrec - 1));  // an unaligned run's last line
#pragma unroll 4
    for (int k = 0; k < nd; ++k) {
      const float4* b = sp + (int64_t)__ldg(nbl + k) * R + g;
#pragma unroll
      for (int kk = 0; kk < P; ++kk)
        if (ok[kk]) asm volatile("prefetch.global.L1 [%0];" ::"l"(b + kk * G));
    }
  }
#pragma unroll
  for (int k = 0; k < P; ++k)
#pragma unroll
    for (int t = 0; t < NR; ++t) c[k][t] = 0.0f;
  // merged per-neighbour pair blocks: c += W z_nb
  auto pair = [&](uint2 rec, const float4 (&v)[P]) {
    float z[P][NR];
#pragma unroll
    for (int k = 0; k < P; ++k) zrow_nr<NR>(v[k].x, v[k].y, v[k].z, z[k]);
    const float* w = ft + (rec.x & kOffMask);
    if constexpr (NR == 8) {
      const float4* w4 = reinterpret_cast<const float4*>(w);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const float4 a0 = __ldg(w4 + 2 * t), a1 = __ldg(w4 + 2 * t + 1);
#pragma unroll
        for (int k = 0; k < P; ++k) {
          float x = c[k][t];
          x = fmaf(a0.x, z[k][0], x);
          x = fmaf(a0.y, z[k][1], x);
          x = fmaf(a0.z, z[k][2], x);
          x = fmaf(a0.w, z[k][3], x);
          x = fmaf(a1.x, z[k][4], x);
          x = fmaf(a1.y, z[k][5], x);
          x = fmaf(a1.z, z[k][6], x);
          x = fmaf(a1.w, z[k][7], x);
          c[k][t] = x;
        }
      }
    } else {
      const float4 a0 = __ldg(reinterpret_cast<const float4*>(w)), a1 = __ldg(reinterpret_cast<const float4*>(w) + 1);
      const float a8 = __ldg(w + 8);
      const float ww[9] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a8};
#pragma unroll
      for (int k = 0; k < P; ++k)
#pragma unroll
        for (int t = 0; t < 3; ++t)
          c[k][t] = fmaf(ww[3 * t], z[k][0], fmaf(ww[3 * t + 1], z[k][1], fmaf(ww[3 * t + 2], z[k][2], c[k][t])));
    }
  };
#pragma unroll 1
  for (int j = part; PAIRS && j < n_pair; j += NP) {
    const uint2 rec = __ldg(fr + j);
    float4 v[P];
    gather((int)(rec.y & 0xffu), v);
    pair(rec, v);
  }
  // l = 1 triplets: c_t += sum_p z1_p sum_q W[t][3p + q] z2_q (rows padded to 12)
#pragma unroll 1
  for (int j = n_pair + part; j < n_pair + n_trip; j += NP) {
    const uint2 rec = __ldg(fr + j);
    float4 v1[P], v2[P];
    gather((int)(rec.y & 0xffu), v1);
    gather((int)((rec.y >> 8) & 0xffu), v2);
    if constexpr (NR == 8 && T2) {
      // merged body-3 block with l = 2 members: c_t += sum_p z1_p sum_q W[t][p][q] z2_q
      if ((rec.x >> kKindShift) == (uint32_t)F_TRIP2) {
        float y1[P][NR], y2[P][NR];
#pragma unroll
        for (int k = 0; k < P; ++k) {
          zrow_nr<NR>(v1[k].x, v1[k].y, v1[k].z, y1[k]);
          zrow_nr<NR>(v2[k].x, v2[k].y, v2[k].z, y2[k]);
        }
        const float4* w4 = reinterpret_cast<const float4*>(ft + (rec.x & kOffMask));
#pragma unroll
        for (int t = 0; t < NR; ++t) {
#pragma unroll
          for (int p = 0; p < NR; ++p) {
            const float4 a0 = __ldg(w4 + (t * NR + p) * 2), a1 = __ldg(w4 + (t * NR + p) * 2 + 1);
#pragma unroll
            for (int k = 0; k < P; ++k) {
              float u = a0.x * y2[k][0];
              u = fmaf(a0.y, y2[k][1], u);
              u = fmaf(a0.z, y2[k][2], u);
              u = fmaf(a0.w, y2[k][3], u);
              u = fmaf(a1.x, y2[k][4], u);
              u = fmaf(a1.y, y2[k][5], u);
              u = fmaf(a1.z, y2[k][6], u);
              u = fmaf(a1.w, y2[k][7], u);
              c[k][t] = fmaf(y1[k][p], u, c[k][t]);
            }
          }
        }
        continue;
      }
    }
    float z1[P][3], z2[P][3];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      zrow_l1(v1[k].x, v1[k].y, v1[k].z, z1[k]);
      zrow_l1(v2[k].x, v2[k].y, v2[k].z, z2[k]);
    }
    const float4* w4 = reinterpret_cast<const float4*>(ft + (rec.x & kOffMask));
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const float4 a0 = __ldg(w4 + 3 * t), a1 = __ldg(w4 + 3 * t + 1), a2 = __ldg(w4 + 3 * t + 2);
      const float w[9] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x};
#pragma unroll
      for (int k = 0; k < P; ++k) {
        float x = c[k][t];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const float u = fmaf(w[p * 3 + 0], z2[k][0], fmaf(w[p * 3 + 1], z2[k][1], w[p * 3 + 2] * z2[k][2]));
          x = fmaf(z1[k][p], u, x);
        }
        c[k][t] = x;
      }
    }
  }
  // l = 1 quads (rows padded to 28)
#pragma unroll 1
  for (int j = n_pair + n_trip + part; j < n_pair + n_trip + n_quad; j += NP) {
    const uint2 rec = __ldg(fr + j);
    float z1[P][3], z2[P][3], z3[P][3];
    {
      float4 v[P];
      gather((int)(rec.y & 0xffu), v);
#pragma unroll
      for (int k = 0; k < P; ++k) zrow_l1(v[k].x, v[k].y, v[k].z, z1[k]);
      gather((int)((rec.y >> 8) & 0xffu), v);
#pragma unroll
      for (int k = 0; k < P; ++k) zrow_l1(v[k].x, v[k].y, v[k].z, z2[k]);
      gather((int)((rec.y >> 16) & 0xffu), v);
#pragma unroll
      for (int k = 0; k < P; ++k) zrow_l1(v[k].x, v[k].y, v[k].z, z3[k]);
    }
    const float4* w4 = reinterpret_cast<const float4*>(ft + (rec.x & kOffMask));
#pragma unroll
    for (int t = 0; t < 3; ++t) {
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        // W[t][p][qq][:] for qq = 0..2 lives in floats 9p .. 9p + 8 of row t
        float w[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) w[m] = __ldg(reinterpret_cast<const float*>(w4 + 7 * t) + 9 * p + m);
#pragma unroll
        for (int k = 0; k < P; ++k) {
          float t2 = 0.0f;
#pragma unroll
          for (int qq = 0; qq < 3; ++qq) {
            const float t3 = fmaf(w[qq * 3], z3[k][0], fmaf(w[qq * 3 + 1], z3[k][1], w[qq * 3 + 2] * z3[k][2]));
            t2 = fmaf(z2[k][qq], t3, t2);
          }
          c[k][t] = fmaf(z1[k][p], t2, c[k][t]);
        }
      }
    }
  }
  if (n_one && part == 0) {
    const float* w = ft + (__ldg(fr + n_pair + n_trip + n_quad).x & kOffMask);
#pragma unroll
    for (int t = 0; t < NR; ++t) {
      const float wt = __ldg(w + t);
#pragma unroll
      for (int k = 0; k < P; ++k) c[k][t] += wt;
    }
  }
}

// One replica of a replica-parallel item: the proposal (precomputed, keyed inline or
// the overrelaxation reflection about the site's l = 1 field), dE = c . (znew - zold),
// the Metropolis (or Metropolis-Hastings) test, the write-back, the counters and the
// record. c holds the replica's leave-one-out coefficients.
template <int NR, bool PF>
__device__ __forceinline__ void rep_decide(const SweepArgs& a, const DevLattice& L, int li, int col,
                                           const int32_t* seg_c, int q, int s, int64_t row0, int r,
                                           const float (&c)[NR], const double* p_beta, const double* p_step,
                                           const unsigned long long* p_seed, unsigned long long* s_dE,
                                           unsigned int* s_cnt) {
  const bool do_or = a.pass >= 0;
  const float4* __restrict__ sp = a.spins + L.spin_off;
  const int slot = L.slot0 + r;
  const float4 e = PF ? __ldg(sp + row0 + r) : __ldcg(sp + row0 + r);
  const double beta = p_beta[slot];
  float px, py, pz;
  double u, lq = 0.0;
  bool attempted = true;
  if (!do_or) {
    if (a.prop != nullptr) {
      const int idx = a.item_base[col] + seg_c[li] + q * L.R + r;
      const float4 p4 = a.prop[idx];
      px = p4.x, py = p4.y, pz = p4.z;
      u = a.propu[idx];
      if (a.lqr != nullptr) lq = a.lqr[idx];
    } else {
      u = keyed_proposal(p_seed[slot], (uint32_t)(s + 1), a.st->sweep + 1u, e.x, e.y, e.z, p_step[slot], px, py,
                         pz);
    }
  } else {
    // reflection about h = (c4, c2, c3) = rows (3, 1, 2)
    const double h0 = c[2], h1 = c[0], h2 = c[1];
    const double hn = sqrt((h0 * h0 + h1 * h1) + h2 * h2);
    if (hn < 1e-12) {
      attempted = false;
      px = e.x, py = e.y, pz = e.z;
    } else {
      const double a0 = h0 / hn, a1 = h1 / hn, a2 = h2 / hn;
      const double d2 = 2.0 * (((double)e.x * a0 + (double)e.y * a1) + (double)e.z * a2);
      const double r0 = d2 * a0 - e.x, r1 = d2 * a1 - e.y, r2 = d2 * a2 - e.z;
      const double rn = sqrt((r0 * r0 + r1 * r1) + r2 * r2);
      px = (float)(r0 / rn);
      py = (float)(r1 / rn);
      pz = (float)(r2 / rn);
    }
    const Blk bk = philox_block(p_seed[slot], (uint32_t)(s + 1), a.st->sweep + 1u, (uint32_t)a.pass, kTagOR);
    u = philox_uniform(bk.w0, bk.w1);
  }
  float zo[NR], zn[NR];
  zrow_nr<NR>(e.x, e.y, e.z, zo);
  zrow_nr<NR>(px, py, pz, zn);
  float term = 0.0f;
#pragma unroll
  for (int t = 0; t < NR; ++t) term = fmaf(c[t], zn[t] - zo[t], term);
  const float dE = attempted ? term : 0.0f;
  bool acc_ok;
  if (!do_or && a.lqr != nullptr) {  // Metropolis-Hastings with the learned proposal's density ratio
    const double la = -beta * (double)dE + lq;
    acc_ok = la >= 0.0 || u < exp(la);
  } else {
    acc_ok = attempted && (dE <= 0.0f || u < exp(-beta * (double)dE));
  }
  if (acc_ok) {
    a.spins[L.spin_off + row0 + r] = make_float4(px, py, pz, 0.0f);
    atomicAdd(s_dE + slot, (unsigned long long)llrint((double)dE * kFixScale));
  }
  if (do_or) {
    if (attempted) atomicAdd(s_cnt + 3 * slot + 2, 1u);
    if (acc_ok) atomicAdd(s_cnt + 3 * slot + 1, 1u);
  } else if (acc_ok) {
    atomicAdd(s_cnt + 3 * slot + 0, 1u);
  }
  if (a.rec_prop != nullptr && li == a.rec_li && r == a.rec_r && a.pass + 1 < kRecPasses) {
    const int64_t qq = (int64_t)(a.pass + 1) * a.rec_cap + s;
    a.rec_prop[3 * qq + 0] = px;
    a.rec_prop[3 * qq + 1] = py;
    a.rec_prop[3 * qq + 2] = pz;
    a.rec_u[qq] = u;
    a.rec_dE[qq] = dE;
    a.rec_acc[qq] = (uint8_t)(acc_ok ? 1 : (attempted ? 0 : 2));
    if (a.rec_lqr != nullptr && !do_or) a.rec_lqr[s] = lq;
  }
}

// NP = 2: two adjacent threads share an item's record walk (alternate records) and
// add their halves with one shuffle; the even thread decides. For colours too small
// to fill the GPU, where each thread's walk is the critical path.
template <int LMAX, int P, int NP, bool PF, bool T2 = (LMAX == 2)>
__device__ void rep_colour(const SweepArgs& a, int col, unsigned long long* s_dE, unsigned int* s_cnt,
                           const float* zsm) {
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
  const double* p_beta = reinterpret_cast<const double*>(zsm);
  const double* p_step = p_beta + a.n_slots;
  const unsigned long long* p_seed = reinterpret_cast<const unsigned long long*>(p_step + a.n_slots);
  const bool do_or = a.pass >= 0;
  int n_threads = 0;  // threads of this colour over every lattice (G per site)
  for (int l = 0; l < a.n_lat; ++l) {
    const int R = a.lat[l].R;
    n_threads += (seg_c[l + 1] - seg_c[l]) / R * ((R + P - 1) / P);
  }
  const int stride = gridDim.x * blockDim.x;  // a multiple of 32: the NP threads of an item stay in one warp
  for (int t0 = blockIdx.x * blockDim.x + threadIdx.x; t0 < n_threads * NP; t0 += stride) {
    const int tid = t0 / NP, part = t0 % NP;
    int li = 0, base = 0, G = 1, R = 1;
    for (; li < a.n_lat; ++li) {
      R = a.lat[li].R;
      G = (R + P - 1) / P;
      const int nt = (seg_c[li + 1] - seg_c[li]) / R * G;
      if (tid < base + nt) break;
      base += nt;
    }
    const DevLattice& L = a.lat[li];
    const int q = (tid - base) / G;
    const int g = (tid - base) - q * G;
    const int4 dsc = __ldg(L.idesc + __ldg(L.color_ptr + col) + q);
    const int s = dsc.x & 0x3fffffff;
    if (do_or && !(dsc.x & (1 << 30))) continue;  // no l = 1 channel
    const float4* __restrict__ sp = a.spins + L.spin_off;
    const int64_t row0 = (int64_t)s * R;
    bool ok[P];
#pragma unroll
    for (int k = 0; k < P; ++k) ok[k] = g + k * G < R;
    float c[P][NR];
    rep_coeffs<LMAX, P, NP, PF, T2>(L, sp, dsc, R, G, g, ok, c, part);
    if (NP == 2) {
      const unsigned pair = 3u << (threadIdx.x & 30u);
#pragma unroll
      for (int k = 0; k < P; ++k)
#pragma unroll
        for (int t = 0; t < NR; ++t) c[k][t] += __shfl_xor_sync(pair, c[k][t], 1);
      if (part != 0) continue;
    }
    // per replica: proposal, dE, decision, write-back
#pragma unroll
    for (int k = 0; k < P; ++k)
      if (ok[k])
        rep_decide<NR, PF>(a, L, li, col, seg_c, q, s, row0, g + k * G, c[k], p_beta, p_step, p_seed, s_dE, s_cnt);
  }
}

// ---------------------------------------------------------------------------
// Learned proposal of one colour: network inputs, then (after the tensor-core MLP)
// a draw from each item's vMF mixture with its density ratio. Items are numbered as
// in the sweep kernels (lattice, then site, then replica), row = item.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void item_of(const SweepArgs& a, const int32_t* seg_c, int item, int& li, int& q, int& r) {
  li = find_lattice(seg_c, a.n_lat, item);
  const int local = item - seg_c[li];
  const int R = a.lat[li].R;
  q = local / R;
  r = local - q * R;
}

// kT in meV of a slot, the network's 43rd input and the head's temperature
__device__ __forceinline__ float slot_kt_mev(const SweepArgs& a, int slot) {
  return (float)(1.0e3 / a.beta[a.rung_of_slot[slot]]);
}

// Fused learned proposal of one colour: one warpgroup per tile of 128 items (persistent
// over tiles). Each thread gathers its item's environment into the BF16 input tile;
// the three layers run on the tcgen05 tensor cores (weights resident in shared
// memory, FP32 accumulators in TMEM, bias + SiLU epilogues writing the next layer's
// BF16 operand tile); each thread then reads its 20 outputs and draws from the vMF
// mixture. Shared-memory operand tiles use the K-major no-swizzle layout in 64-column
// chunks (umma.cuh).
struct LearnedNet {
  const __nv_bfloat16* W1;  // [128][64]
  const __nv_bfloat16* W2;  // [128][128]
  const __nv_bfloat16* W3;  // [32][128]
  const float* b1;          // [128]
  const float* b2;          // [128]
  const float* b3;          // [32]
  int* err;
};

constexpr int kTile = 128;
constexpr uint32_t kChunkBytes = 128u * 64u * 2u;  // one 128-row x 64-column BF16 chunk
// dynamic shared memory of k_learned_fused (bytes): W1 (1 chunk), W2 (2), W3 (2 x 32 rows),
// X (1), H (2), biases
constexpr size_t kLearnedSmem = 1024 + kChunkBytes * (1 + 2 + 1 + 2) + 2u * (32u * 64u * 2u) + 4 * (128 + 128 + 32);

__device__ __forceinline__ void stage_rows_kmajor(uint8_t* dst, const __nv_bfloat16* src, int rows, int K) {
  // src [rows][K] row-major -> chunks of 64 columns, each rows x 64 K-major no-swizzle
  const int pieces = rows * (K / 8);
  for (int p = threadIdx.x; p < pieces; p += blockDim.x) {
    const int row = p / (K / 8), kg = p % (K / 8);
    const int chunk = kg >> 3, kk = (kg & 7) * 8;
    const uint4 v = *reinterpret_cast<const uint4*>(src + (int64_t)row * K + kg * 8);
    *reinterpret_cast<uint4*>(dst + (size_t)chunk * rows * 128 + umma::kmajor_offset(row, kk, 64)) = v;
  }
}

// issue one layer: D (TMEM) = A (128 x K, chunks) . B (N x K, chunks)^T
__device__ __forceinline__ void learned_layer(uint32_t tmem_d, const uint8_t* A, const uint8_t* B, int n_rows_b,
                                              int K, int N, uint64_t* mbar) {
  umma::fence_after();
  const uint32_t a0 = umma::smem_u32(A), b0 = umma::smem_u32(B);
  const uint32_t idesc = umma::idesc_bf16_f32(N);
  for (int kk = 0; kk < K / 16; ++kk) {
    const uint32_t ch = (uint32_t)(kk >> 2), in = (uint32_t)(kk & 3) * 256u;
    const uint64_t ad = umma::smem_desc(a0 + ch * (128u * 128u) + in, 128u, 1024u);
    const uint64_t bd = umma::smem_desc(b0 + ch * ((uint32_t)n_rows_b * 128u) + in, 128u, 1024u);
    umma::mma_bf16(tmem_d, ad, bd, idesc, kk > 0 ? 1u : 0u);
  }
  umma::commit(mbar);
}

// Two warpgroups per CTA: both gather half of a row's environment and each runs the
// epilogue of half the hidden columns (a warp reads TMEM lanes 32 (warp % 4) ..);
// warpgroup 0 reads the 20 outputs and draws for its rows.
// MH = false: the draws, uniforms and log-density ratios go to a.prop / a.propu / lqr
// for a sweep kernel to decide. MH = true: the Metropolis-Hastings step runs here as
// well. Warpgroup 1 walks the records of its row's next item (the replica-parallel
// coefficients c_t, one replica per thread) while warpgroup 0 draws, hands them over
// in shared memory, and warpgroup 0 forms dE = sum_t c_t (z_t(new) - z_t(old)),
// decides and writes the spin. Safe within one launch because no site of the colour
// is a Hamiltonian neighbour or an environment site of another.
// SiLU z / (1 + e^-z) with the fast division (the training path in learned.cu uses the
// same form, so the sweep and the training forward agree): for z below about -87,
// e^-z is infinite and the quotient is 0, the function's limit.
__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// FIELD (with MH): the network reads the item's leave-one-out coefficients (rows 1..NR,
// in meV) and kT instead of its environment spins; they fix the site's conditional
// distribution whatever the range of the couplings.
template <int LMAX, bool MH, bool FIELD = false>
__global__ void __launch_bounds__(256, 2) k_learned_fused(SweepArgs a, LearnedNet net, double* lqr) {
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  extern __shared__ __align__(1024) uint8_t lsm[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(lsm) + 1023) & ~(uintptr_t)1023);
  uint8_t* sW1 = base;
  uint8_t* sW2 = sW1 + kChunkBytes;
  uint8_t* sW3 = sW2 + 2 * kChunkBytes;
  uint8_t* sX = sW3 + 2 * (32u * 64u * 2u);
  uint8_t* sH = sX + kChunkBytes;
  float* sb = reinterpret_cast<float*>(sH + 2 * kChunkBytes);
  // MH: per-slot accumulators after the biases (dynamic, sized by n_slots), and the
  // rows' coefficients in the sH tile while it is free (after layer 3 has read it)
  unsigned long long* s_dE = reinterpret_cast<unsigned long long*>(sb + 288);
  unsigned int* s_cnt = reinterpret_cast<unsigned int*>(s_dE + a.n_slots);
  float* sC = reinterpret_cast<float*>(sH);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int row = tid & 127, wg = tid >> 7;
  const int col = a.colour;
  const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
  const int n_items = seg_c[a.n_lat];
  const int n_tiles = (n_items + kTile - 1) / kTile;
  if ((int)blockIdx.x >= n_tiles) return;
  if (MH) zero_block(a.n_slots, s_dE, s_cnt);
  if (warp == 0) umma::tmem_alloc(&tslot, 256u);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  stage_rows_kmajor(sW1, net.W1, 128, 64);
  stage_rows_kmajor(sW2, net.W2, 128, 128);
  stage_rows_kmajor(sW3, net.W3, 32, 128);
  for (int i = tid; i < 128; i += blockDim.x) {
    sb[i] = net.b1[i];
    sb[128 + i] = net.b2[i];
    if (i < 32) sb[256 + i] = net.b3[i];
  }
  umma::fence_async_smem();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;
  // A thread's share of one tile's environment (warpgroup 0: spins 0..7 -> input
  // columns 0..23; warpgroup 1: spins 8..13 and kT -> columns 24..42), gathered for
  // the next tile while this tile draws.
  // A row's item and, written straight into the BF16 input tile sX (free once the
  // previous tile's layer 1 has read it), the row's input columns: warpgroup 0
  // columns 0..23 (environment spins 0..7), warpgroup 1 columns 24..63 (spins 8..
  // k-1, kT in meV at column 3k, zeros after it). k = L.env_k <= 21.
  struct Gather {
    int li, q, r, s;
    bool valid;
    float4 e;
    float tau;
  };
  auto put = [&](int c, float v) {
    *reinterpret_cast<__nv_bfloat16*>(sX + umma::kmajor_offset(row, c, 64)) = __float2bfloat16_rn(v);
  };
  auto gather = [&](int tile, Gather& g) {
    const int item = tile * kTile + row;
    g.valid = tile < n_tiles && item < n_items;
    g.li = g.q = g.r = g.s = 0;
    g.e = make_float4(0.f, 0.f, 1.f, 0.f);
    g.tau = 1.0f;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (int ch = wg ? 3 : 0; ch < (wg ? 8 : 3); ++ch)
      *reinterpret_cast<uint4*>(sX + umma::kmajor_offset(row, ch * 8, 64)) = z;
    if (!g.valid) return;
    item_of(a, seg_c, item, g.li, g.q, g.r);
    const DevLattice& L = a.lat[g.li];
    g.s = L.color_sites[L.color_ptr[col] + g.q];
    const float4* sp = a.spins + L.spin_off;
    const int K = L.env_k;
    const int32_t* env = L.env + (int64_t)g.s * K;
    g.tau = slot_kt_mev(a, L.slot0 + g.r);
    const int j0 = wg ? 8 : 0, j1 = wg ? K : (K < 8 ? K : 8);
    for (int jb = j0; jb < j1; jb += 4) {  // four spins' loads in flight at a time
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        v[u] = jb + u < j1 ? __ldg(sp + (int64_t)__ldg(env + jb + u) * L.R + g.r) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (jb + u < j1) {
          put(3 * (jb + u), v[u].x);
          put(3 * (jb + u) + 1, v[u].y);
          put(3 * (jb + u) + 2, v[u].z);
        }
    }
    if ((3 * K < 24) == (wg == 0)) put(3 * K, g.tau);
    if (!wg) g.e = sp[(int64_t)g.s * L.R + g.r];
  };
  // MH, warpgroup 1: the coefficients of a gathered row's item
  auto coeffs = [&](const Gather& g, float (&cc)[NR]) {
#pragma unroll
    for (int t = 0; t < NR; ++t) cc[t] = 0.0f;
    if (!g.valid) return;
    const DevLattice& L = a.lat[g.li];
    const int4 dsc = __ldg(L.idesc + __ldg(L.color_ptr + col) + g.q);
    const bool one[1] = {true};
    float c1[1][NR];
    rep_coeffs<LMAX, 1, 2, true>(L, a.spins + L.spin_off, dsc, L.R, L.R, g.r, one, c1, wg);
#pragma unroll
    for (int t = 0; t < NR; ++t) cc[t] = c1[0][t];
  };
  // FIELD: the network input row of an item from its two coefficient halves (warpgroup
  // 1's half through shared memory, free between the last layer and the next tile's
  // first): columns 0..NR-1 the coefficients in meV, column NR kT in meV.
  auto field_input = [&](const Gather& g, const float (&cc)[NR]) {
    __syncthreads();  // the previous use of sC (the decisions) is over
    if (wg == 1)
#pragma unroll
      for (int t = 0; t < NR; ++t) sC[row * NR + t] = cc[t];
    __syncthreads();
    if (wg == 0) {
#pragma unroll
      for (int t = 0; t < NR; ++t) put(t, 1.0e3f * (cc[t] + sC[row * NR + t]));
      put(NR, g.valid ? g.tau : 0.0f);
    }
  };
  Gather cur, nxt;
  gather(blockIdx.x, cur);
  float ccur[NR];  // MH: this warpgroup's half of the current tile's coefficients
  if (MH) coeffs(cur, ccur);
  if (FIELD) field_input(cur, ccur);
  for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
    const int item = tile * kTile + row;
    const bool valid = cur.valid;
    const int li = cur.li, r = cur.r, s = cur.s;
    const float4 e = cur.e;
    const float tau = cur.tau;
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    // layer 1 -> TMEM columns 0..127
    if (tid == 0) learned_layer(tmem, sX, sW1, 128, 64, 128, &mbar);
    ok = umma::mbar_wait(&mbar, phase, 1000000000ull);
    phase ^= 1u;
    umma::fence_after();
    for (int c0 = 64 * wg; c0 < 64 * wg + 64; c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + lane_base + (uint32_t)c0, v);
      alignas(16) __nv_bfloat16 h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float z = v[i] + sb[c0 + i];
        h[i] = __float2bfloat16_rn(silu_fast(z));
      }
      *reinterpret_cast<uint4*>(sH + (c0 >> 6) * kChunkBytes + umma::kmajor_offset(row, c0 & 63, 64)) =
          *reinterpret_cast<const uint4*>(h);
    }
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    // layer 2 -> TMEM columns 128..255
    if (tid == 0) learned_layer(tmem + 128u, sH, sW2, 128, 128, 128, &mbar);
    ok = ok && umma::mbar_wait(&mbar, phase, 1000000000ull);
    phase ^= 1u;
    umma::fence_after();
    for (int c0 = 64 * wg; c0 < 64 * wg + 64; c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + lane_base + 128u + (uint32_t)c0, v);
      alignas(16) __nv_bfloat16 h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float z = v[i] + sb[128 + c0 + i];
        h[i] = __float2bfloat16_rn(silu_fast(z));
      }
      *reinterpret_cast<uint4*>(sH + (c0 >> 6) * kChunkBytes + umma::kmajor_offset(row, c0 & 63, 64)) =
          *reinterpret_cast<const uint4*>(h);
    }
    umma::fence_async_smem();
    umma::fence_before();
    __syncthreads();
    // layer 3 -> TMEM columns 0..31
    if (tid == 0) learned_layer(tmem, sH, sW3, 32, 128, 32, &mbar);
    ok = ok && umma::mbar_wait(&mbar, phase, 1000000000ull);
    phase ^= 1u;
    umma::fence_after();
    float o[32];
    if (wg == 0) {
#pragma unroll
      for (int c0 = 0; c0 < 32; c0 += 8) umma::tmem_ld8(tmem + lane_base + (uint32_t)c0, o + c0);
    } else if (MH) {
#pragma unroll
      for (int t = 0; t < NR; ++t) sC[row * NR + t] = ccur[t];
    }
    umma::fence_before();
    __syncthreads();  // every thread has read TMEM and the tiles before the next tile reuses them
    gather(tile + gridDim.x, nxt);  // the next tile's loads are in flight during this tile's draw
    if (MH && wg == 1) coeffs(nxt, ccur);
    cur = nxt;
    auto draw_decide = [&]() {
#pragma unroll
    for (int j = 0; j < 32; ++j) o[j] += sb[256 + j];
    const DevLattice& L = a.lat[li];
    const int slot = L.slot0 + r;
    const int rung = a.rung_of_slot[slot];
    vmf::MixF mix;
    vmf::mixture_f(o, tau, mix);
    const Blk b0 = philox_block(a.seed[rung], (uint32_t)(s + 1), a.st->sweep + 1u, 0u, kTagLearn);
    const Blk b1 = philox_block(a.seed[rung], (uint32_t)(s + 1), a.st->sweep + 1u, 1u, kTagLearn);
    float xs[3];
    vmf::sample_f(mix, (float)philox_uniform(b0.w0, b0.w1), (float)philox_uniform(b0.w2, b0.w3),
                  (float)philox_uniform(b1.w0, b1.w1), xs);
    const double u = philox_uniform(b1.w2, b1.w3);
    const double lq = (double)(vmf::log_q_f(mix, e.x, e.y, e.z) - vmf::log_q_f(mix, xs[0], xs[1], xs[2]));
    if (!MH) {
      const int idx = a.item_base[col] + item;
      a.prop[idx] = make_float4(xs[0], xs[1], xs[2], 0.0f);
      a.propu[idx] = u;
      lqr[idx] = lq;
      return;
    }
    float zo[NR], zn[NR];
    zrow_nr<NR>(e.x, e.y, e.z, zo);
    zrow_nr<NR>(xs[0], xs[1], xs[2], zn);
    float dE = 0.0f;
#pragma unroll
    for (int t = 0; t < NR; ++t) dE = fmaf(ccur[t] + sC[row * NR + t], zn[t] - zo[t], dE);
    const double la = -a.beta[rung] * (double)dE + lq;
    const bool acc_ok = la >= 0.0 || u < exp(la);
    if (acc_ok) {
      a.spins[L.spin_off + (int64_t)s * L.R + r] = make_float4(xs[0], xs[1], xs[2], 0.0f);
      atomicAdd(s_dE + slot, (unsigned long long)llrint((double)dE * kFixScale));
      atomicAdd(s_cnt + 3 * slot + 0, 1u);
    }
    if (a.rec_prop != nullptr && li == a.rec_li && r == a.rec_r && a.pass + 1 < kRecPasses) {
      const int64_t qq = (int64_t)(a.pass + 1) * a.rec_cap + s;
      a.rec_prop[3 * qq + 0] = xs[0];
      a.rec_prop[3 * qq + 1] = xs[1];
      a.rec_prop[3 * qq + 2] = xs[2];
      a.rec_u[qq] = u;
      a.rec_dE[qq] = dE;
      a.rec_acc[qq] = (uint8_t)(acc_ok ? 1 : 0);
      if (a.rec_lqr != nullptr) a.rec_lqr[s] = lq;
    }
    };
    if (wg == 0 && valid && ok) draw_decide();
    if (MH && wg == 0) coeffs(cur, ccur);  // the next tile's half, after this tile's decisions
    if (FIELD) field_input(cur, ccur);
  }
  if (!ok && tid == 0 && net.err) atomicExch(net.err, 1);
  if (MH) flush_block(a, s_dE, s_cnt);
  umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after();
    umma::tmem_free(tmem, 256u);
  }
}

// P = 2 at 80 registers (three 256-thread blocks per SM); P = 1 at 64 registers
// (four blocks per SM).
#ifndef SCEMC_REP_MINB_P2
#define SCEMC_REP_MINB_P2 3
#endif
template <int LMAX, int P, int NP, bool PF, bool T2 = (LMAX == 2)>
__global__ void __launch_bounds__(256, P == 1 ? 4 : SCEMC_REP_MINB_P2) k_rep_colour(SweepArgs a) {
  extern __shared__ __align__(16) float zsm[];
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  stage_params(a, zsm);
  rep_colour<LMAX, P, NP, PF, T2>(a, a.colour, s_dE, s_cnt, zsm);
  flush_block(a, s_dE, s_cnt);
}

// ---------------------------------------------------------------------------
// Replica-parallel pass with the pair records on the tensor cores (lmax 2, kernel 5).
// A warp owns one site and 32 of its replicas. The pair records' share of the
// coefficients, c[rep][i] = sum_rec sum_j W_rec[i][j] z_j(nb_rec, rep), is the product
// of a (replicas x 8K) matrix of neighbour Z rows with the (8K x 8) stack of the
// site's K coupling blocks. It runs as mma.sync m16n8k8 TF32 over groups of eight
// records: for component j, K indexes the group's eight records, the A operand holds
// z_j of their neighbours for 16 replicas and the B operand holds column j of their
// blocks. A lane's A values over the eight components are then four whole Z rows
// (two neighbours x two replicas per 16-replica tile), which it computes from the
// spins it loads, so no operand moves between lanes; its B values are row g of two
// blocks. FP32 accuracy comes from splitting both operands, x = hi + lo with hi = x
// truncated to TF32 (|lo| < 2^-10 |x|), and summing hi.hi + hi.lo + lo.hi; the tensor
// core keeps 11 significant bits of lo and the lo.lo product is dropped, which leaves
// under 2^-19 relative per product (the block rows are read once per group of eight
// records and split in registers: measured faster than reading host-split copies,
// which doubles the block loads). After the last group the accumulators pass through
// shared memory to lane = replica; the lane adds its triplet, quad and one-body
// records (FP32 FMAs, as the replica-parallel kernel) and decides. The sums run in
// another order than the FMA kernels', so the chains agree with theirs to rounding,
// not bit for bit.
// ---------------------------------------------------------------------------
constexpr int kTcRowFloats = 12;  // a row of the 32 x 8 coefficient tile: 16-byte aligned, no bank conflicts

__host__ __device__ __forceinline__ size_t tc_warp_floats(int dmax, int rmax) {
  return fast_rec_floats(rmax) + fast_nbid_words(dmax) + 32 * kTcRowFloats;
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return h;
}

// The head of an operand: its sign, exponent and 10 significand bits (one mask), or
// with SCEMC_TC_RNA = 1 the value rounded to TF32 (cvt.rna, measured 7 % slower per
// compound sweep at fcc 48^3 x 32); the tail is the exact FP32 remainder.
#ifndef SCEMC_TC_RNA
#define SCEMC_TC_RNA 0
#endif
__device__ __forceinline__ uint32_t tf32_head(float x) {
  return SCEMC_TC_RNA ? tf32_rna(x) : (__float_as_uint(x) & 0xffffe000u);
}

// d += a . b: one m16n8k8 product, TF32 operands, FP32 accumulators
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Three 256-thread blocks per SM (80 registers, 112 bytes of spills): measured 7 %
// faster per compound sweep than two blocks at 128 registers at fcc 64^3 x 32, where
// the pass waits on its neighbour gathers.
#ifndef SCEMC_TC_MINB
#define SCEMC_TC_MINB 3
#endif
// SCEMC_TC_FOLD = 1: the Z rows' normalisation constants move into the block columns
// (scaled once per group of records), and each lane evaluates the bare polynomials
// (y, z, x, xy, yz, 3z^2 - 1, xz, x^2 - y^2) of its eight spins per group: measured
// 3 % faster at fcc 64^3 x 32. 0 evaluates the normalised rows.
#ifndef SCEMC_TC_FOLD
#define SCEMC_TC_FOLD 1
#endif
__device__ __forceinline__ float tc_col_scale(int m) {
  if (!SCEMC_TC_FOLD) return 1.0f;
  return m < 3 ? kN1 : (m == 5 ? kC20 : (m == 7 ? kC22 : kC2a));
}
__device__ __forceinline__ void tc_zrow(float4 v, float (&o)[8]) {
  if (SCEMC_TC_FOLD) {
    o[0] = v.y, o[1] = v.z, o[2] = v.x;
    o[3] = v.x * v.y, o[4] = v.y * v.z, o[5] = 3.0f * (v.z * v.z) - 1.0f;
    o[6] = v.x * v.z, o[7] = v.x * v.x - v.y * v.y;
  } else {
    zrow_nr<8>(v.x, v.y, v.z, o);
  }
}

template <bool T2>
__global__ void __launch_bounds__(256, SCEMC_TC_MINB) k_rep_tc(SweepArgs a) {
  constexpr int NR = 8;
  extern __shared__ __align__(16) float zsm[];
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  stage_params(a, zsm);
  const int col = a.colour;
  const int32_t* seg_c = a.seg + (size_t)col * (a.n_lat + 1);
  const double* p_beta = reinterpret_cast<const double*>(zsm);
  const double* p_step = p_beta + a.n_slots;
  const unsigned long long* p_seed = reinterpret_cast<const unsigned long long*>(p_step + a.n_slots);
  const bool do_or = a.pass >= 0;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;  // fragment row group and column of this lane
  float* wbase = zsm + fast_param_floats(a.n_slots) + (size_t)wib * tc_warp_floats(a.dmax, a.rmax);
  uint2* rb = reinterpret_cast<uint2*>(wbase);
  int* nbid = reinterpret_cast<int*>(wbase + fast_rec_floats(a.rmax));
  float* tile = wbase + fast_rec_floats(a.rmax) + fast_nbid_words(a.dmax);
  int n_items = 0;  // (site, 32-replica chunk) items of this colour over every lattice
  for (int l = 0; l < a.n_lat; ++l) {
    const int R = a.lat[l].R;
    n_items += (seg_c[l + 1] - seg_c[l]) / R * ((R + 31) >> 5);
  }
  const int n_warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + wib; w < n_items; w += n_warps) {  // warp-uniform
    int li = 0, base = 0, R = 1, nch = 1;
    for (; li < a.n_lat; ++li) {
      R = a.lat[li].R;
      nch = (R + 31) >> 5;
      const int ni = (seg_c[li + 1] - seg_c[li]) / R * nch;
      if (w < base + ni) break;
      base += ni;
    }
    const DevLattice& L = a.lat[li];
    const int q = (w - base) / nch;
    const int r0 = ((w - base) - q * nch) * 32;
    const int4 dsc = __ldg(L.idesc + __ldg(L.color_ptr + col) + q);
    if (do_or && !(dsc.x & (1 << 30))) continue;  // no l = 1 channel
    const int s = dsc.x & 0x3fffffff;
    const uint32_t cnt = (uint32_t)dsc.w;
    const int n_pair = (int)(cnt & 0xffu);
    const int nd = (int)(cnt >> 24);
    const float4* __restrict__ sp = a.spins + L.spin_off;
    __syncwarp();  // the previous item's readers of rb, nbid and the tile are done
    for (int k = lane; k < n_pair; k += 32) rb[k] = __ldg(L.frec + dsc.z + k);
    for (int k = lane; k < nd; k += 32) nbid[k] = __ldg(L.nb_list + dsc.y + k);
    __syncwarp();
    float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll 1
    for (int j0 = 0; j0 < n_pair; j0 += 8) {
      // this lane's K columns: records j0 + t and j0 + t + 4 (zero blocks past the last)
      const int k1 = j0 + t, k2 = k1 + 4;
      const bool v1 = k1 < n_pair, v2 = k2 < n_pair;
      const uint2 rc1 = rb[v1 ? k1 : 0], rc2 = rb[v2 ? k2 : 0];
      const int nb1 = nbid[rc1.y & 0xffu], nb2 = nbid[rc2.y & 0xffu];
      // rows g of the two blocks, split into head and tail (zero past the last record)
      uint32_t b1h[NR], b1l[NR], b2h[NR], b2l[NR];
      {
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4* w1 = reinterpret_cast<const float4*>(L.ftensor + (rc1.x & kOffMask)) + 2 * g;
        const float4* w2 = reinterpret_cast<const float4*>(L.ftensor + (rc2.x & kOffMask)) + 2 * g;
        const float4 p0 = v1 ? __ldg(w1) : z4, p1 = v1 ? __ldg(w1 + 1) : z4;
        const float4 q0 = v2 ? __ldg(w2) : z4, q1 = v2 ? __ldg(w2 + 1) : z4;
        float x1[NR] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
        float x2[NR] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
        for (int m = 0; m < NR; ++m) {
          x1[m] *= tc_col_scale(m);
          x2[m] *= tc_col_scale(m);
          b1h[m] = tf32_head(x1[m]);
          b1l[m] = __float_as_uint(x1[m] - __uint_as_float(b1h[m]));
          b2h[m] = tf32_head(x2[m]);
          b2l[m] = __float_as_uint(x2[m] - __uint_as_float(b2h[m]));
        }
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        // rows g and g + 8 of this 16-replica tile
        const int ra = r0 + 16 * mt + g, rc = ra + 8;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 s0 = v1 && ra < R ? __ldcg(sp + (int64_t)nb1 * R + ra) : z4;
        const float4 s1 = v1 && rc < R ? __ldcg(sp + (int64_t)nb1 * R + rc) : z4;
        const float4 s2 = v2 && ra < R ? __ldcg(sp + (int64_t)nb2 * R + ra) : z4;
        const float4 s3 = v2 && rc < R ? __ldcg(sp + (int64_t)nb2 * R + rc) : z4;
        float z0[NR], z1[NR], z2[NR], z3[NR];
        tc_zrow(s0, z0);
        tc_zrow(s1, z1);
        tc_zrow(s2, z2);
        tc_zrow(s3, z3);
#pragma unroll
        for (int j = 0; j < NR; ++j) {
          const uint32_t h0 = tf32_head(z0[j]), h1 = tf32_head(z1[j]), h2 = tf32_head(z2[j]), h3 = tf32_head(z3[j]);
          const uint32_t l0 = __float_as_uint(z0[j] - __uint_as_float(h0));
          const uint32_t l1 = __float_as_uint(z1[j] - __uint_as_float(h1));
          const uint32_t l2 = __float_as_uint(z2[j] - __uint_as_float(h2));
          const uint32_t l3 = __float_as_uint(z3[j] - __uint_as_float(h3));
          mma_tf32(acc[mt], l0, l1, l2, l3, b1h[j], b2h[j]);
          mma_tf32(acc[mt], h0, h1, h2, h3, b1l[j], b2l[j]);
          mma_tf32(acc[mt], h0, h1, h2, h3, b1h[j], b2h[j]);
        }
      }
    }
    // accumulator fragments (rows g, g + 8; columns 2t, 2t + 1) to lane = replica
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      float* ta = tile + (16 * mt + g) * kTcRowFloats + 2 * t;
      *reinterpret_cast<float2*>(ta) = make_float2(acc[mt][0], acc[mt][1]);
      *reinterpret_cast<float2*>(ta + 8 * kTcRowFloats) = make_float2(acc[mt][2], acc[mt][3]);
    }
    __syncwarp();
    const int r = r0 + lane;
    if (r < R) {
      const float4 cp0 = *reinterpret_cast<const float4*>(tile + lane * kTcRowFloats);
      const float4 cp1 = *reinterpret_cast<const float4*>(tile + lane * kTcRowFloats + 4);
      float c[1][NR];
      const bool ok[1] = {true};
      rep_coeffs<2, 1, 1, false, T2, false>(L, sp, dsc, R, R, r, ok, c, 0);
      const float cp[NR] = {cp0.x, cp0.y, cp0.z, cp0.w, cp1.x, cp1.y, cp1.z, cp1.w};
#pragma unroll
      for (int m = 0; m < NR; ++m) c[0][m] += cp[m];
      rep_decide<NR, false>(a, L, li, col, seg_c, q, s, (int64_t)s * R, r, c[0], p_beta, p_step, p_seed, s_dE,
                            s_cnt);
    }
  }
  flush_block(a, s_dE, s_cnt);
}

// Persistent replica-parallel pass (mode 2 with kernel 3): one cooperative launch runs
// the pass's proposal precompute (when requested) and every colour, with the bounded
// grid barrier between them. Spins written by other blocks in earlier colours are
// read through L2 (the non-prefetching form's loads), never from a stale L1 line.
template <int LMAX, int P, int NP, bool T2 = (LMAX == 2)>
__global__ void __launch_bounds__(256, P == 1 ? 4 : SCEMC_REP_MINB_P2) k_rep_persistent(SweepArgs a) {
  extern __shared__ __align__(16) float zsm[];
  __shared__ unsigned long long s_dE[kMaxSlots];
  __shared__ unsigned int s_cnt[3 * kMaxSlots];
  zero_block(a.n_slots, s_dE, s_cnt);
  stage_params(a, zsm);
  bool ok = true;
  int k = 0;
  if (a.pass < 0 && a.prop != nullptr) {
    make_proposals<true>(a);
    ok = grid_barrier(a.gs, a.bar_base, k++, gridDim.x, a.barrier_limit_ns);
  }
  for (int col = 0; ok && col < a.max_colors; ++col) {
    rep_colour<LMAX, P, NP, false, T2>(a, col, s_dE, s_cnt, zsm);
    if (col + 1 < a.max_colors) ok = grid_barrier(a.gs, a.bar_base, k++, gridDim.x, a.barrier_limit_ns);
  }
  flush_block(a, s_dE, s_cnt);
}


// Leave-one-out coefficient rows 1..NR of every site of replica r of lattice li, one
// thread per site through the replica-parallel walk (one replica per thread): the
// learned proposal's field inputs for training. Inactive sites get zeros.
template <int LMAX, bool T2>
__global__ void __launch_bounds__(256) k_site_coeffs(const DevLattice* lat, int li, int r, const float4* spins,
                                                     float* out) {
  constexpr int NR = (LMAX + 1) * (LMAX + 1) - 1;
  const DevLattice& L = lat[li];
  const float4* sp = spins + L.spin_off;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.n_sites; s += gridDim.x * blockDim.x) {
    float c[1][NR];
#pragma unroll
    for (int t = 0; t < NR; ++t) c[0][t] = 0.0f;
    if (L.active[s]) {
      const uint32_t cnt = L.fr_cnt[s];
      const int nd = L.nb_ptr[s + 1] - L.nb_ptr[s];
      const int4 dsc = make_int4(s | ((cnt >> 24) ? (int)(1u << 31) : 0), L.nb_ptr[s], L.fr_ptr[s],
                                 (int32_t)((cnt & 0xffffffu) | ((uint32_t)nd << 24)));
      const bool ok[1] = {true};
      rep_coeffs<LMAX, 1, 1, false, T2>(L, sp, dsc, L.R, L.R, r, ok, c, 0);
    }
#pragma unroll
    for (int t = 0; t < NR; ++t) out[(int64_t)s * NR + t] = c[0][t];
  }
}

struct TailArgs {
  int32_t n_slots, n_rungs, n_lat;
  const DevLattice* lat;
  double* energy;               // per slot
  unsigned long long* dE_fix;   // per slot
  unsigned long long* cnt;      // per rung x4
  unsigned long long* win;      // per rung x2 adaptation window {acc, att}
  int add_att;                  // add n_active to att_metro (a Metropolis pass ran)
  int adapt;                    // adapt the step now
  double adapt_target;
  double* step;                 // per rung
  int exchange;                 // attempt swaps now
  int32_t* slot_of_rung;
  int32_t* rung_of_slot;
  const double* beta;
  unsigned long long* swaps;    // per rung x2 {att, acc}
  uint64_t exchange_seed;
  EnsState* st;
  int bump;  // one sweep completed: advance the device sweep counter
};

// Energy fold, counters, adaptation and replica exchange (one block).
// Exchange: src/gpu/gpu_pt.jl:129-134 schedule with the swap rule of src/pt.jl:92-96.
__global__ void k_tail(TailArgs t) {
  for (int i = threadIdx.x; i < t.n_slots; i += blockDim.x) {
    const long long fx = (long long)t.dE_fix[i];
    t.dE_fix[i] = 0ull;
    t.energy[i] += (double)fx / kFixScale;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (t.bump) t.st->sweep += 1u;
  for (int li = 0; li < t.n_lat; ++li) {
    const DevLattice& L = t.lat[li];
    for (int k = 0; k < L.R; ++k) {
      const int rung = L.slot0 + k;
      if (t.add_att) {
        t.cnt[4 * rung + 1] += (unsigned long long)L.n_active;
        t.win[2 * rung + 1] += (unsigned long long)L.n_active;
      }
    }
  }
  // acceptance window for adaptation = metro counters since the last adaptation
  if (t.adapt) {
    for (int rung = 0; rung < t.n_rungs; ++rung) {
      const unsigned long long att = t.win[2 * rung + 1];
      const unsigned long long acc = t.cnt[4 * rung + 0] - t.win[2 * rung + 0];
      if (att > 0) {
        const double a = (double)acc / (double)att;
        double s = t.step[rung] * exp(0.5 * (a - t.adapt_target));
        s = s < 1e-3 ? 1e-3 : (s > 3.141592653589793 ? 3.141592653589793 : s);
        t.step[rung] = s;
      }
      t.win[2 * rung + 0] = t.cnt[4 * rung + 0];
      t.win[2 * rung + 1] = 0ull;
    }
  }
  if (t.exchange) {
    const int parity = t.st->exchange_parity;
    const int count = ++t.st->exchange_count;
    for (int li = 0; li < t.n_lat; ++li) {
      const DevLattice& L = t.lat[li];
      for (int i = parity; i < L.R - 1; i += 2) {
        const int ra = L.slot0 + i, rb = ra + 1;
        const Blk b = philox_block(t.exchange_seed, (uint32_t)(i + 1), (uint32_t)count, (uint32_t)li, kTagExchange);
        const double u = philox_uniform(b.w0, b.w1);
        const int sa = t.slot_of_rung[ra], sb = t.slot_of_rung[rb];
        const double logw = (t.beta[ra] - t.beta[rb]) * (t.energy[sa] - t.energy[sb]);
        t.swaps[2 * ra + 0] += 1ull;
        if (u < exp(logw < 0.0 ? logw : 0.0)) {
          t.slot_of_rung[ra] = sb;
          t.slot_of_rung[rb] = sa;
          t.rung_of_slot[sb] = ra;
          t.rung_of_slot[sa] = rb;
          t.swaps[2 * ra + 1] += 1ull;
        }
      }
    }
    t.st->exchange_parity = 1 - parity;
  }
}

// ---- FP64 energy recompute and renormalisation ------------------------------

// Partial energies of fixed 1024-instance chunks for every slot of lattice li.
// grid: (chunks, R); block 256 (each thread 4 instances, fixed-order reduction).
__global__ void __launch_bounds__(256) k_energy_chunks(const DevLattice* lat, int li, const float4* spins,
                                                       double* partial, int n_chunks) {
  const DevLattice& L = lat[li];
  const int chunk = blockIdx.x, r = blockIdx.y;
  const float4* sp = spins + L.spin_off;
  double acc = 0.0;
  for (int k = 0; k < kChunk / 256; ++k) {
    const int64_t i = (int64_t)chunk * kChunk + k * 256 + threadIdx.x;
    if (i >= L.n_inst) break;
    const int t = L.inst_term[i];
    const int off = L.inst_ptr[i];
    double Ei = 0.0;
    for (int e = L.eprog_ptr[t]; e < L.eprog_ptr[t + 1]; ++e) {
      double p = 1.0;
      const int f0 = L.efac_ptr[e], nf = L.efac_ptr[e + 1] - f0;
      for (int m = 0; m < nf; ++m) {
        const float4 v = sp[(int64_t)L.inst_sites[off + m] * L.R + r];
        p *= zval_f64(L.efac_row[f0 + m], (double)v.x, (double)v.y, (double)v.z);
      }
      Ei += L.eent_w[e] * p;
    }
    acc += L.term_coef[t] * Ei;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o >= 1; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[(size_t)r * n_chunks + chunk] = red[0];
}

// Sum chunk partials in order; mode 0: write E_out; mode 1: renormalisation
// (drift, max_drift, re-anchor the running energy).
__global__ void k_energy_fold(const DevLattice* lat, int li, const double* partial, int n_chunks, double* energy,
                              double* e_out, double* drift, double* max_drift, const int32_t* rung_of_slot,
                              int mode) {
  const DevLattice& L = lat[li];
  const int r = threadIdx.x;
  if (r >= L.R) return;
  double E = 0.0;
  for (int c = 0; c < n_chunks; ++c) E += partial[(size_t)r * n_chunks + c];
  const int slot = L.slot0 + r;
  if (e_out) e_out[slot] = E;
  if (mode == 1) {
    const double d = fabs(energy[slot] - E);
    const int rung = rung_of_slot[slot];
    if (drift) drift[slot] = d;
    if (d > max_drift[rung] || d != d) max_drift[rung] = d;
    energy[slot] = E;
  }
}

// Normalise active spins in FP64 and round to FP32 (state.jl:168-175).
__global__ void k_normalize(const DevLattice* lat, int li, float4* spins) {
  const DevLattice& L = lat[li];
  const int64_t n = (int64_t)L.n_sites * L.R;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / L.R);
    if (!L.active[s]) continue;
    float4 v = spins[L.spin_off + i];
    const double x = v.x, y = v.y, z = v.z;
    const double nn = sqrt((x * x + y * y) + z * z);
    spins[L.spin_off + i] = make_float4((float)(x / nn), (float)(y / nn), (float)(z / nn), 0.0f);
  }
}

// ---- measurements (observables.jl:85-143) -----------------------------------

// Partial sums per (chunk, replica): {m_x, m_y, m_z} over active sites and the
// sublattice sums {x_a, y_a, z_a}; record layout per slot: 3 + 3*n_cell_atoms.
__global__ void __launch_bounds__(256) k_measure_chunks(const DevLattice* lat, int li, const float4* spins,
                                                        double* partial, int n_chunks, int rlen) {
  const DevLattice& L = lat[li];
  const int chunk = blockIdx.x, r = blockIdx.y;
  const int A = L.n_cell_atoms;
  __shared__ double red[256][4];
  __shared__ double out[3 + 3 * kMaxCellAtoms];
  for (int k = threadIdx.x; k < 3 + 3 * A; k += blockDim.x) out[k] = 0.0;
  __syncthreads();
  // each thread sums sites of one sublattice at a time: sites of chunk are
  // [chunk*1024, +1024); sublattice a = s % A.
  for (int a = 0; a < A; ++a) {
    double sx = 0, sy = 0, sz = 0, dummy = 0;
    for (int k = 0; k < kChunk / 256; ++k) {
      const int s = chunk * kChunk + k * 256 + threadIdx.x;
      if (s >= L.n_sites || (s % A) != a || !L.active[s]) continue;
      const float4 v = spins[L.spin_off + (int64_t)s * L.R + r];
      sx += v.x, sy += v.y, sz += v.z;
    }
    red[threadIdx.x][0] = sx, red[threadIdx.x][1] = sy, red[threadIdx.x][2] = sz, red[threadIdx.x][3] = dummy;
    __syncthreads();
    for (int o = 128; o >= 1; o >>= 1) {
      if (threadIdx.x < o)
        for (int q = 0; q < 3; ++q) red[threadIdx.x][q] += red[threadIdx.x + o][q];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      for (int q = 0; q < 3; ++q) {
        out[3 + 3 * a + q] = red[0][q];
        out[q] += red[0][q];
      }
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < 3 + 3 * A; k += blockDim.x)
    partial[((size_t)r * n_chunks + chunk) * rlen + k] = out[k];
}

// Fold the chunk partials in order into one record row per rung:
// {E, m_x, m_y, m_z, sub...} (m averaged over active sites, sub over cells).
__global__ void k_measure_fold(const DevLattice* lat, int li, const double* partial, int n_chunks, int rlen,
                               const double* energy, const int32_t* rung_of_slot, double* rec_row,
                               int rec_len) {
  const DevLattice& L = lat[li];
  const int r = blockIdx.x;
  const int slot = L.slot0 + r;
  const int rung = rung_of_slot[slot];
  const int A = L.n_cell_atoms;
  const double ncells = (double)(L.n_sites / A);
  for (int k = threadIdx.x; k < 3 + 3 * A; k += blockDim.x) {
    double v = 0.0;
    for (int c = 0; c < n_chunks; ++c) v += partial[((size_t)r * n_chunks + c) * rlen + k];
    const double outv = k < 3 ? v / (double)L.n_active : v / ncells;
    rec_row[(size_t)rung * rec_len + 1 + k] = outv;
  }
  if (threadIdx.x == 0) rec_row[(size_t)rung * rec_len] = energy[slot];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename T>
int32_t upload(std::vector<void*>& allocs, const std::vector<T>& v, const T** out) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  CUDA_TRY(cudaMalloc(&p, bytes));
  allocs.push_back(p);
  if (!v.empty()) CUDA_TRY(h2d_sync(p, v.data(), v.size() * sizeof(T)));
  *out = static_cast<const T*>(p);
  return SCEMC_OK;
}

}  // namespace

struct scemc_tables {
  int device = 0;
  DevLattice dl{};
  std::vector<void*> allocs;
  std::vector<int32_t> color_ptr;  // 0-based host copy
  std::vector<int32_t> site_col_of;  // colour (1-based) of every site, 0 = inactive
  std::vector<uint8_t> active;
  int32_t n_sites = 0, nlm = 0, lmax = 0, n_colors = 0, n_active = 0, n_cell_atoms = 1;
  int64_t n_inst = 0;
  double d_mean = 0, a_mean = 0;
  int64_t bytes = 0;
  bool has_generic = true;
  int64_t fast_records = 0;
  bool trip2 = false;  // the fast records hold body-3 blocks with l = 2 members
  ~scemc_tables() {
    for (void* p : allocs) cudaFree(p);
  }
};

struct scemc_ensemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<const scemc_tables*> tabs;
  std::vector<int32_t> R;          // replicas per table
  std::vector<int32_t> slot0;      // first slot per table
  std::vector<int64_t> spin_off;   // float4 offset per table
  int32_t n_slots = 0;
  int64_t n_spins = 0;
  int32_t lmax = 0;
  int32_t max_colors = 0;
  int64_t sweep_index = 0;
  uint64_t exchange_seed = 0x5ce3c0ffee5eedull;
  // device
  DevLattice* d_lat = nullptr;
  float4* d_spins = nullptr;
  int32_t* d_seg = nullptr;
  std::vector<int32_t> seg;  // host copy
  double* d_energy = nullptr;
  unsigned long long* d_dEfix = nullptr;
  unsigned long long* d_cnt = nullptr;
  unsigned long long* d_win = nullptr;
  unsigned long long* d_swaps = nullptr;
  double* d_beta = nullptr;
  double* d_step = nullptr;
  unsigned long long* d_seed = nullptr;
  int32_t* d_slot_of_rung = nullptr;
  int32_t* d_rung_of_slot = nullptr;
  double* d_max_drift = nullptr;
  double* d_drift = nullptr;
  double* d_eout = nullptr;
  GridSync* d_gs = nullptr;
  EnsState* d_st = nullptr;
  double* d_partial = nullptr;
  size_t partial_cap = 0;
  // measurements
  double* d_meas = nullptr;
  int64_t meas_cap = 0, meas_n = 0;
  int32_t rec_len = 0;
  // replay record (replica rec_r of table rec_li; buffers sized for the largest table)
  bool recording = false;
  int32_t rec_li = 0, rec_r = 0;
  int32_t rec_cap = 0;  // sites the record buffers hold
  float* d_rprop = nullptr;
  double* d_ru = nullptr;
  float* d_rdE = nullptr;
  uint8_t* d_racc = nullptr;
  long long barrier_limit_ns = 2000000000ll;
  int coop_blocks = 0;  // cached co-resident grid size for the persistent form
  int coop_G = -1;
  unsigned char* d_readback = nullptr;  // energy, slot_of_rung, counters, swaps, steps, max_drift (one block)
  double* d_energy_in = nullptr;        // energies of an upload, committed on the device
  double* d_cfg64 = nullptr;  // device copy of a host payload (3 x n_spins FP64)
  unsigned long long* d_bad = nullptr;  // first non-finite payload spin
  unsigned char* h_small = nullptr;     // pinned: flag, energies in, per-slot arrays out
  // learned proposal (network not owned)
  const scemc_mlp* mlp = nullptr;
  bool learned_field = false;  // the network reads the site coefficients (set_learned with k = 0)
  std::vector<int32_t*> d_env;
  double* d_lqr = nullptr;
  double* d_rlqr = nullptr;
  uint32_t* d_flags = nullptr;  // data-flow form: per item slot completion epochs
  // row-parallel fast kernel
  bool fast = false;
  bool trip2 = false;  // some table has body-3 blocks with l = 2 members
  int32_t dmax = 0, rmax = 0;
  std::vector<int32_t> item_base;  // max_colors+1
  int32_t* d_item_base = nullptr;
  float4* d_prop = nullptr;
  double* d_propu = nullptr;
  int coop_key[4] = {-1, -1, -1, -1};
  // chain-resident cluster kernel: cluster size and dynamic shared memory (0 = not prepared)
  int cluster_cs = 0;
  size_t cluster_smem = 0;
  unsigned long long bar_base = 0;  // host mirror of GridSync::arrived after the enqueued launches
  int graph_passes_per_launch = 0;
  // autotuned launch form (used when mode, proposals, lanes are 0)
  bool tuned = false;
  int tuned_mode = 2, tuned_proposals = 0, tuned_lanes = 0, tuned_kernel = 0;
  // captured compound-sweep graphs keyed by {n_or, fast, precompute, G, recording}
  struct GraphEntry {
    int key[7];
    cudaGraphExec_t exec;
    int64_t launches;  // kernel nodes in the graph
  };
  int64_t launches = 0;  // kernels enqueued on the stream (a graph replay adds its kernel nodes)
  std::vector<GraphEntry> graphs;
  // live timing of the sweep kernels: one event pair per pass
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending;
  double prof_ms = 0.0;
  int64_t prof_passes = 0;
  ~scemc_ensemble() {
    if (h_small) cudaFreeHost(h_small);
    for (auto& pr : ev_pending) {
      ev_pool.push_back(pr.first);
      ev_pool.push_back(pr.second);
    }
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    void* qs[] = {d_item_base, d_prop, d_propu, d_lqr, d_rlqr, d_flags};
    for (int32_t* p : d_env)
      if (p) cudaFree(p);
    for (void* p : qs)
      if (p) cudaFree(p);
    void* ps[] = {d_lat,   d_spins,   d_seg,  d_readback, d_dEfix, d_win,   d_beta,  d_seed,
                  d_rung_of_slot, d_drift, d_eout, d_gs, d_st, d_partial, d_meas, d_rprop, d_ru, d_rdE, d_racc,
                  d_cfg64, d_bad,   d_energy_in};
    for (void* p : ps)
      if (p) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// ---- table compilation --------------------------------------------------------
int32_t check_ptr(const int32_t* p, int64_t n, int64_t first, int64_t last, const char* name) {
  if (!p) return fail(SCEMC_ERR_ARG, std::string(name) + " is NULL");
  if (p[0] != first) return fail(SCEMC_ERR_ARG, std::string(name) + "[1] must be " + std::to_string(first));
  for (int64_t i = 0; i < n; ++i)
    if (p[i + 1] < p[i]) return fail(SCEMC_ERR_ARG, std::string(name) + " is not monotone");
  if (p[n] != last) return fail(SCEMC_ERR_ARG, std::string(name) + " does not end at its array length + 1");
  return SCEMC_OK;
}

// Row-parallel fast tables: per site the distinct neighbours (first-appearance
// order) and records referencing them by local index. All pair programs of a site
// that share a neighbour merge into one NR x NR block (rows/columns 1..NR of the
// tesseral row); body-1 programs merge into one NR vector; l = 1 triplets and quads
// keep one record each. Blocks are deduplicated by the list of merged program ids.
struct FastBuild {
  std::vector<int32_t> nb_ptr, nb_list, fr_ptr;
  std::vector<uint32_t> fr_cnt;
  std::vector<uint2> frec;
  std::vector<float> ft;
  int32_t dmax = 0, rmax = 0;
  int64_t n_trip2 = 0;  // merged body-3 blocks with l = 2 members
};

// prog_l: per program, the l of its own member and of its other members in slot
// order (three entries; the body-3 block layout needs them).
bool build_fast(const scemc_tables_desc* d, const std::vector<int32_t>& prog_kind,
                const std::vector<int32_t>& prog_toff, const std::vector<int32_t>& prog_l,
                const std::vector<float>& tensor, const std::vector<int32_t>& pbase, FastBuild& F) {
  if (d->lmax != 1 && d->lmax != 2) return false;
  const int NR = d->nlm - 1;
  for (int32_t k : prog_kind)
    if (k == K_GEN) return false;
  auto place = [&](const std::vector<float>& v) {
    while (F.ft.size() % 4) F.ft.push_back(0.0f);
    const int32_t off = (int32_t)F.ft.size();
    F.ft.insert(F.ft.end(), v.begin(), v.end());
    return off;
  };
  std::map<std::vector<int32_t>, int32_t> pair_cache, one_cache, tri2_cache;
  std::vector<int32_t> single_off(prog_kind.size(), -1);
  // program id -> (template, slot) for the l placement of pair blocks
  const int ns = d->n_sites;
  F.nb_ptr.assign(ns + 1, 0);
  F.fr_ptr.assign(ns + 1, 0);
  F.fr_cnt.assign(ns, 0u);
  std::vector<int32_t> nbs;
  std::vector<std::pair<int32_t, std::vector<int32_t>>> pairs;  // (local, pids)
  std::vector<int32_t> ones;
  std::vector<std::array<int32_t, 5>> multi;  // (kind, pid, l0, l1, l2)
  // body-3 programs with l = 2 members, merged per unordered neighbour pair:
  // ((smaller local, larger local), [pid * 2 + (factor order reversed)])
  std::vector<std::pair<std::pair<int32_t, int32_t>, std::vector<int32_t>>> tri2;
  for (int32_t s = 0; s < ns; ++s) {
    nbs.clear();
    pairs.clear();
    ones.clear();
    multi.clear();
    tri2.clear();
    auto local = [&](int32_t site) {
      for (size_t i = 0; i < nbs.size(); ++i)
        if (nbs[i] == site) return (int32_t)i;
      nbs.push_back(site);
      return (int32_t)nbs.size() - 1;
    };
    for (int64_t j = d->site_ptr[s] - 1; j < d->site_ptr[s + 1] - 1; ++j) {
      const int32_t inst = d->site_inst[j] - 1;
      const int32_t pid = d->site_prog[j] - 1;
      const int own = d->site_slot[j];
      const int32_t k = d->inst_term[inst] - 1;
      const int D = d->term_body[k];
      int32_t loc[3] = {0, 0, 0}, q = 0;
      for (int sl = 1; sl <= D; ++sl)
        if (sl != own) loc[q++] = local(d->inst_sites[d->inst_ptr[inst] - 1 + sl - 1] - 1);
      const int kind = prog_kind[pid];
      if (kind == K_B1_L1 || kind == K_B1_L2) {
        ones.push_back(pid);
      } else if (kind >= K_B2_11 && kind <= K_B2_22) {
        bool found = false;
        for (auto& pr : pairs)
          if (pr.first == loc[0]) {
            pr.second.push_back(pid);
            found = true;
            break;
          }
        if (!found) pairs.push_back({loc[0], {pid}});
      } else if (kind == K_B3_L2) {
        const std::pair<int32_t, int32_t> key{std::min(loc[0], loc[1]), std::max(loc[0], loc[1])};
        const int32_t tag = pid * 2 + (loc[0] > loc[1] ? 1 : 0);
        bool found = false;
        for (auto& t : tri2)
          if (t.first == key) {
            t.second.push_back(tag);
            found = true;
            break;
          }
        if (!found) tri2.push_back({key, {tag}});
      } else {
        multi.push_back({kind, pid, loc[0], loc[1], loc[2]});
      }
    }
    if (nbs.size() > 255) return false;
    F.dmax = std::max<int32_t>(F.dmax, (int32_t)nbs.size());
    F.nb_ptr[s] = (int32_t)F.nb_list.size();
    F.nb_list.insert(F.nb_list.end(), nbs.begin(), nbs.end());
    F.fr_ptr[s] = (int32_t)F.frec.size();
    for (auto& pr : pairs) {
      std::vector<int32_t> key = pr.second;
      std::sort(key.begin(), key.end());
      auto it = pair_cache.find(key);
      int32_t off;
      if (it != pair_cache.end()) {
        off = it->second;
      } else {
        std::vector<float> W((size_t)NR * NR, 0.0f);
        for (int32_t pid : key) {
          const int kind = prog_kind[pid];
          const int lt = (kind == K_B2_11 || kind == K_B2_12) ? 1 : 2;
          const int lf = (kind == K_B2_11 || kind == K_B2_21) ? 1 : 2;
          const int rt = lt == 1 ? 0 : 3, rf = lf == 1 ? 0 : 3;
          for (int mt = 0; mt < 2 * lt + 1; ++mt)
            for (int mf = 0; mf < 2 * lf + 1; ++mf)
              W[(size_t)(rt + mt) * NR + rf + mf] += tensor[prog_toff[pid] + mt * (2 * lf + 1) + mf];
        }
        off = place(W);
        pair_cache[key] = off;
      }
      if (off > kOffMask) return false;
      F.frec.push_back(make_uint2(((uint32_t)F_PAIR << kKindShift) | (uint32_t)off, (uint32_t)pr.first));
    }
    std::stable_sort(multi.begin(), multi.end(),
                     [](const std::array<int32_t, 5>& x, const std::array<int32_t, 5>& y) { return x[0] < y[0]; });
    int n_trip = 0, n_quad = 0;
    // merged body-3 blocks with l = 2 members (before the l = 1 triplets, in the triplet range)
    for (auto& t : tri2) {
      std::vector<int32_t> key = t.second;
      std::sort(key.begin(), key.end());
      auto it = tri2_cache.find(key);
      int32_t off;
      if (it != tri2_cache.end()) {
        off = it->second;
      } else {
        std::vector<float> W((size_t)NR * NR * NR, 0.0f);
        for (int32_t tag : key) {
          const int32_t pid = tag >> 1;
          const bool flip = (tag & 1) != 0;
          const int lt = prog_l[3 * pid], l0 = prog_l[3 * pid + 1], l1 = prog_l[3 * pid + 2];
          const int d0 = 2 * l0 + 1, d1 = 2 * l1 + 1;
          const int rt = lt == 1 ? 0 : 3, r0 = l0 == 1 ? 0 : 3, r1 = l1 == 1 ? 0 : 3;
          for (int mt = 0; mt < 2 * lt + 1; ++mt)
            for (int m0 = 0; m0 < d0; ++m0)
              for (int m1 = 0; m1 < d1; ++m1) {
                const float v = tensor[prog_toff[pid] + (mt * d0 + m0) * d1 + m1];
                const int p = flip ? r1 + m1 : r0 + m0, q = flip ? r0 + m0 : r1 + m1;
                W[((size_t)(rt + mt) * NR + p) * NR + q] += v;
              }
        }
        off = place(W);
        tri2_cache[key] = off;
      }
      if (off > kOffMask) return false;
      ++n_trip;
      ++F.n_trip2;
      F.frec.push_back(make_uint2(((uint32_t)F_TRIP2 << kKindShift) | (uint32_t)off,
                                  (uint32_t)t.first.first | ((uint32_t)t.first.second << 8)));
    }
    for (auto& m : multi) {
      const int32_t pid = m[1];
      if (single_off[pid] < 0) {
        // three target rows, each padded to a multiple of 4 floats (16-byte loads)
        const int row = m[0] == K_B3_111 ? 9 : 27, stride = m[0] == K_B3_111 ? 12 : 28;
        std::vector<float> v((size_t)3 * stride, 0.0f);
        for (int t = 0; t < 3; ++t)
          for (int k = 0; k < row; ++k) v[(size_t)t * stride + k] = tensor[prog_toff[pid] + t * row + k];
        single_off[pid] = place(v);
      }
      if (m[0] == K_B3_111) ++n_trip;
      else ++n_quad;
      const uint32_t kind = m[0] == K_B3_111 ? F_TRIP : F_QUAD;
      if (single_off[pid] > kOffMask) return false;
      F.frec.push_back(make_uint2((kind << kKindShift) | (uint32_t)single_off[pid],
                                  (uint32_t)m[2] | ((uint32_t)m[3] << 8) | ((uint32_t)m[4] << 16)));
    }
    if (!ones.empty()) {
      std::vector<int32_t> key = ones;  // merged body-1 vector
      std::sort(key.begin(), key.end());
      auto it = one_cache.find(key);
      int32_t off;
      if (it != one_cache.end()) {
        off = it->second;
      } else {
        std::vector<float> w(NR, 0.0f);
        for (int32_t pid : key) {
          const int lt = prog_kind[pid] == K_B1_L1 ? 1 : 2;
          const int rt = lt == 1 ? 0 : 3;
          for (int mt = 0; mt < 2 * lt + 1; ++mt) w[rt + mt] += tensor[prog_toff[pid] + mt];
        }
        off = place(w);
        one_cache[key] = off;
      }
      if (off > kOffMask) return false;
      F.frec.push_back(make_uint2(((uint32_t)F_ONE << kKindShift) | (uint32_t)off, 0u));
    }
    if (pairs.size() > 255 || n_trip > 255 || n_quad > 255) return false;
    F.fr_cnt[s] = (uint32_t)pairs.size() | ((uint32_t)n_trip << 8) | ((uint32_t)n_quad << 16) |
                  ((uint32_t)(ones.empty() ? 0 : 1) << 24);
  }
  F.nb_ptr[ns] = (int32_t)F.nb_list.size();
  F.fr_ptr[ns] = (int32_t)F.frec.size();
  for (int32_t s = 0; s < ns; ++s) F.rmax = std::max(F.rmax, F.fr_ptr[s + 1] - F.fr_ptr[s]);
  (void)pbase;
  return true;
}

int32_t compile_tables(const scemc_tables_desc* d, scemc_tables* T) {
  if (!d) return fail(SCEMC_ERR_ARG, "desc is NULL");
  if (d->lmax > 6) return fail(SCEMC_ERR_UNSUPPORTED, "lmax = " + std::to_string(d->lmax) +
                                                         " unsupported on the device path (<= 6)");
  if (d->lmax < 0 || d->nlm != (d->lmax + 1) * (d->lmax + 1))
    return fail(SCEMC_ERR_ARG, "nlm must equal (lmax+1)^2");
  if (d->n_sites < 1 || d->n_colors < 0 || d->n_cell_atoms < 1 || d->n_cell_atoms > kMaxCellAtoms ||
      d->n_sites % d->n_cell_atoms != 0)
    return fail(SCEMC_ERR_ARG, "bad n_sites / n_colors / n_cell_atoms");
  const int32_t ns = d->n_sites;
  int32_t rc;
  if ((rc = check_ptr(d->site_ptr, ns, 1, d->n_adj + 1, "site_ptr"))) return rc;
  if ((rc = check_ptr(d->inst_ptr, d->n_inst, 1, d->n_inst_sites + 1, "inst_ptr"))) return rc;
  if ((rc = check_ptr(d->sprog_ptr, d->n_sprog, 1, d->n_sent + 1, "sprog_ptr"))) return rc;
  if ((rc = check_ptr(d->sfac_ptr, d->n_sent, 1, d->n_sfac + 1, "sfac_ptr"))) return rc;
  if ((rc = check_ptr(d->eprog_ptr, d->n_terms, 1, d->n_eent + 1, "eprog_ptr"))) return rc;
  if ((rc = check_ptr(d->efac_ptr, d->n_eent, 1, d->n_efac + 1, "efac_ptr"))) return rc;
  if ((rc = check_ptr(d->color_ptr, d->n_colors, 1, d->n_active + 1, "color_ptr"))) return rc;
  if (!d->term_body || !d->term_ls || !d->site_inst || !d->site_slot || !d->inst_term || !d->inst_sites ||
      !d->site_prog || !d->sent_w || !d->sent_tgt || !d->sfac_row || !d->sfac_slot || !d->eent_w ||
      !d->efac_row || !d->term_coef || !d->color_sites || !d->site_has_l1 || !d->site_active)
    return fail(SCEMC_ERR_ARG, "a table pointer is NULL");
  // templates -> program ids
  std::vector<int32_t> pbase(d->n_terms + 1, 0), lsbase(d->n_terms + 1, 0);
  for (int64_t k = 0; k < d->n_terms; ++k) {
    if (d->term_body[k] < 1) return fail(SCEMC_ERR_ARG, "term_body must be >= 1");
    pbase[k + 1] = pbase[k] + d->term_body[k];
    lsbase[k + 1] = lsbase[k] + d->term_body[k];
  }
  if (pbase[d->n_terms] != d->n_sprog) return fail(SCEMC_ERR_ARG, "sum(term_body) != number of site programs");
  for (int64_t k = 0; k < lsbase[d->n_terms]; ++k)
    if (d->term_ls[k] < 0 || d->term_ls[k] > d->lmax) return fail(SCEMC_ERR_ARG, "term_ls outside 0:lmax");
  for (int64_t e = 0; e < d->n_sent; ++e)
    if (d->sent_tgt[e] < 1 || d->sent_tgt[e] > d->nlm) return fail(SCEMC_ERR_ARG, "sent_tgt outside 1:nlm");
  for (int64_t f = 0; f < d->n_sfac; ++f)
    if (d->sfac_row[f] < 1 || d->sfac_row[f] > d->nlm) return fail(SCEMC_ERR_ARG, "sfac_row outside 1:nlm");
  for (int64_t f = 0; f < d->n_efac; ++f)
    if (d->efac_row[f] < 1 || d->efac_row[f] > d->nlm) return fail(SCEMC_ERR_ARG, "efac_row outside 1:nlm");
  for (int64_t i = 0; i < d->n_inst; ++i)
    if (d->inst_term[i] < 1 || d->inst_term[i] > d->n_terms) return fail(SCEMC_ERR_ARG, "inst_term out of range");
  for (int64_t q = 0; q < d->n_inst_sites; ++q)
    if (d->inst_sites[q] < 1 || d->inst_sites[q] > ns) return fail(SCEMC_ERR_ARG, "inst_sites out of range");
  for (int64_t q = 0; q < d->n_active; ++q)
    if (d->color_sites[q] < 1 || d->color_sites[q] > ns) return fail(SCEMC_ERR_ARG, "color_sites out of range");
  for (int64_t i = 0; i < d->n_inst; ++i) {
    const int32_t k = d->inst_term[i] - 1;
    if (d->inst_ptr[i + 1] - d->inst_ptr[i] != d->term_body[k])
      return fail(SCEMC_ERR_ARG, "instance size differs from its template's body order");
  }
  // programs: kind + dense tensor (fast kinds), sparse descriptors (all)
  std::vector<int32_t> prog_kind(d->n_sprog, K_GEN), prog_toff(d->n_sprog, 0), prog_l(3 * d->n_sprog, 0);
  std::vector<DevProg> progs(d->n_sprog);
  std::vector<float> tensor;
  for (int64_t k = 0; k < d->n_terms; ++k) {
    const int D = d->term_body[k];
    const int32_t* ls = d->term_ls + lsbase[k];
    for (int v = 1; v <= D; ++v) {
      const int32_t pid = pbase[k] + v - 1;  // 0-based
      DevProg pg;
      pg.e_lo = d->sprog_ptr[pid] - 1;
      pg.e_hi = d->sprog_ptr[pid + 1] - 1;
      pg.own_slot = v;
      pg.body = D;
      progs[pid] = pg;
      // factor l's in ascending slot order excluding v
      int lf[8];
      int nf = 0;
      bool small = D <= 4;
      for (int q = 1; q <= D && small; ++q)
        if (q != v) lf[nf++] = ls[q - 1];
      const int lt = ls[v - 1];
      int kind = K_GEN;
      if (small) {
        auto in12 = [](int l) { return l == 1 || l == 2; };
        bool ok = in12(lt);
        for (int q = 0; q < nf; ++q) ok = ok && in12(lf[q]);
        if (ok) {
          if (D == 1) kind = lt == 1 ? K_B1_L1 : K_B1_L2;
          else if (D == 2) kind = lt == 1 ? (lf[0] == 1 ? K_B2_11 : K_B2_12) : (lf[0] == 1 ? K_B2_21 : K_B2_22);
          else if (D == 3 && lt == 1 && lf[0] == 1 && lf[1] == 1) kind = K_B3_111;
          else if (D == 3 && d->lmax == 2) kind = K_B3_L2;
          else if (D == 4 && lt == 1 && lf[0] == 1 && lf[1] == 1 && lf[2] == 1) kind = K_B4_1111;
        }
      }
      if (kind != K_GEN) {
        int dims[4];
        dims[0] = 2 * lt + 1;
        int size = dims[0];
        for (int q = 0; q < nf; ++q) {
          dims[q + 1] = 2 * lf[q] + 1;
          size *= dims[q + 1];
        }
        const int32_t off = (int32_t)tensor.size();
        tensor.resize(tensor.size() + size, 0.0f);
        for (int e = pg.e_lo; e < pg.e_hi; ++e) {
          int idx = d->sent_tgt[e] - 1 - lt * lt;
          const int f0 = d->sfac_ptr[e] - 1, f1 = d->sfac_ptr[e + 1] - 1;
          if (f1 - f0 != nf) return fail(SCEMC_ERR_ARG, "program entry factor count differs from body - 1");
          for (int f = f0; f < f1; ++f) {
            const int q = f - f0;
            const int m = d->sfac_row[f] - 1 - lf[q] * lf[q];
            if (m < 0 || m >= dims[q + 1]) return fail(SCEMC_ERR_ARG, "factor row outside its l block");
            idx = idx * dims[q + 1] + m;
          }
          if (idx < 0 || idx >= size) return fail(SCEMC_ERR_ARG, "target row outside its l block");
          tensor[off + idx] += (float)d->sent_w[e];
        }
        if (off > kOffMask) return fail(SCEMC_ERR_UNSUPPORTED, "coefficient tensors too large");
        prog_toff[pid] = off;
      }
      prog_kind[pid] = kind;
      prog_l[3 * pid] = lt;
      for (int q = 0; q < nf && q < 2; ++q) prog_l[3 * pid + 1 + q] = lf[q];
    }
  }
  if (d->n_sprog > kOffMask) return fail(SCEMC_ERR_UNSUPPORTED, "too many site programs");
  // adjacency records
  std::vector<int4> rec(d->n_adj);
  std::vector<int32_t> adj_ptr(ns + 1);
  int64_t d_sum = 0, a_sum = 0;
  std::vector<int32_t> seen;
  for (int32_t s = 0; s < ns; ++s) {
    adj_ptr[s] = d->site_ptr[s] - 1;
    seen.clear();
    for (int64_t j = d->site_ptr[s] - 1; j < d->site_ptr[s + 1] - 1; ++j) {
      const int32_t inst = d->site_inst[j] - 1;
      if (inst < 0 || inst >= d->n_inst) return fail(SCEMC_ERR_ARG, "site_inst out of range");
      const int32_t pid = d->site_prog[j] - 1;
      if (pid < 0 || pid >= d->n_sprog) return fail(SCEMC_ERR_ARG, "site_prog out of range");
      const int32_t k = d->inst_term[inst] - 1;
      const int D = d->term_body[k];
      const int own = d->site_slot[j];
      if (own < 1 || own > D || pid != pbase[k] + own - 1)
        return fail(SCEMC_ERR_ARG, "site_prog/site_slot inconsistent with the instance's template");
      if (d->inst_sites[d->inst_ptr[inst] - 1 + own - 1] != s + 1)
        return fail(SCEMC_ERR_ARG, "site_slot does not point back at the site");
      int4 r4;
      // body-3 blocks with l = 2 members have a dense form only in the fast tables; the
      // generic walk keeps the reference's sparse program for them
      const int kind = prog_kind[pid] == K_B3_L2 ? (int)K_GEN : prog_kind[pid];
      r4.x = (kind << kKindShift) | (kind == K_GEN ? pid : prog_toff[pid]);
      r4.y = r4.z = r4.w = -1;
      if (D <= 4) {
        int nb[3] = {-1, -1, -1}, q = 0;
        for (int sl = 1; sl <= D; ++sl) {
          if (sl == own) continue;
          nb[q++] = d->inst_sites[d->inst_ptr[inst] - 1 + sl - 1] - 1;
        }
        r4.y = nb[0], r4.z = nb[1], r4.w = nb[2];
        for (int t = 0; t < q; ++t) seen.push_back(nb[t]);
      } else {
        r4.y = -1 - inst;
        for (int sl = 1; sl <= D; ++sl)
          if (sl != own) seen.push_back(d->inst_sites[d->inst_ptr[inst] - 1 + sl - 1] - 1);
      }
      rec[j] = r4;
    }
    if (d->site_active[s]) {
      std::sort(seen.begin(), seen.end());
      d_sum += std::unique(seen.begin(), seen.end()) - seen.begin();
      a_sum += d->site_ptr[s + 1] - d->site_ptr[s];
    }
  }
  adj_ptr[ns] = (int32_t)d->n_adj;
  // 0-based copies of the remaining tables
  auto rebase = [](const int32_t* p, int64_t n) {
    std::vector<int32_t> v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = p[i] - 1;
    return v;
  };
  std::vector<float> sent_w(d->n_sent);
  std::vector<int8_t> sent_tgt(d->n_sent), sfac_row(d->n_sfac), sfac_slot(d->n_sfac), efac_row(d->n_efac);
  for (int64_t e = 0; e < d->n_sent; ++e) {
    sent_w[e] = (float)d->sent_w[e];
    sent_tgt[e] = (int8_t)(d->sent_tgt[e] - 1);
  }
  for (int64_t f = 0; f < d->n_sfac; ++f) {
    sfac_row[f] = (int8_t)(d->sfac_row[f] - 1);
    sfac_slot[f] = d->sfac_slot[f];
  }
  for (int64_t f = 0; f < d->n_efac; ++f) efac_row[f] = (int8_t)(d->efac_row[f] - 1);
  FastBuild F;
  const bool fast = build_fast(d, prog_kind, prog_toff, prog_l, tensor, pbase, F);
  // the generic records are kept for every model that needs them, and for small
  // fast ones (so the generic form can still be selected); huge fast models skip them
  const bool keep_generic = !fast || d->n_adj <= (int64_t)(1 << 24);
  std::vector<int4> rec_v;
  if (keep_generic) rec_v = std::move(rec);
  std::vector<int4>().swap(rec);
  std::vector<uint8_t> has_l1(d->site_has_l1, d->site_has_l1 + ns), active(d->site_active, d->site_active + ns);
  std::vector<double> eent_w(d->eent_w, d->eent_w + d->n_eent), term_coef(d->term_coef, d->term_coef + d->n_terms);
  DevLattice& L = T->dl;
  L.n_sites = ns;
  L.nlm = d->nlm;
  L.lmax = d->lmax;
  L.n_colors = d->n_colors;
  L.n_active = d->n_active;
  L.n_cell_atoms = d->n_cell_atoms;
  L.n_inst = d->n_inst;
  int32_t r = 0;
  if ((r = upload(T->allocs, adj_ptr, &L.adj_ptr))) return r;
  if ((r = upload(T->allocs, rec_v, &L.rec))) return r;
  if ((r = upload(T->allocs, progs, &L.prog))) return r;
  if ((r = upload(T->allocs, tensor, &L.tensor))) return r;
  if ((r = upload(T->allocs, sent_w, &L.sent_w))) return r;
  if ((r = upload(T->allocs, sent_tgt, &L.sent_tgt))) return r;
  if ((r = upload(T->allocs, rebase(d->sfac_ptr, d->n_sent + 1), &L.sfac_ptr))) return r;
  if ((r = upload(T->allocs, sfac_row, &L.sfac_row))) return r;
  if ((r = upload(T->allocs, sfac_slot, &L.sfac_slot))) return r;
  if ((r = upload(T->allocs, rebase(d->inst_ptr, d->n_inst + 1), &L.inst_ptr))) return r;
  if ((r = upload(T->allocs, rebase(d->inst_sites, d->n_inst_sites), &L.inst_sites))) return r;
  std::vector<int32_t> cp = rebase(d->color_ptr, d->n_colors + 1);
  if ((r = upload(T->allocs, cp, &L.color_ptr))) return r;
  // Sites of a colour in tiles of SCEMC_ORDER_TILE_CELLS consecutive cells, and in
  // sublattice order inside a tile (stable): translation-equivalent sites share their
  // coupling blocks, so the threads of one warp, which carry two neighbouring items of
  // a colour, read the same block, and the items in flight together gather from one
  // region of the lattice. The order inside a colour does not change any result (its
  // sites are updated independently and keyed by site; measured bitwise equal). Tiles
  // of 4096 cells measured 3 % faster than one tile at fcc 48^3 x 32 rungs (13.78
  // against 14.23 ms per compound sweep; site order 14.52).
  std::vector<int32_t> cs = rebase(d->color_sites, d->n_active);
#ifndef SCEMC_ORDER_TILE_CELLS
#define SCEMC_ORDER_TILE_CELLS 4096  // 0: one tile (the whole lattice)
#endif
  for (int32_t c = 0; c < d->n_colors; ++c)
    std::stable_sort(cs.begin() + cp[c], cs.begin() + cp[c + 1], [&](int32_t x, int32_t y) {
      const int32_t na = d->n_cell_atoms, tc = SCEMC_ORDER_TILE_CELLS;
      if (tc > 0 && x / (na * tc) != y / (na * tc)) return x / (na * tc) < y / (na * tc);
      return x % na < y % na;
    });
  if ((r = upload(T->allocs, cs, &L.color_sites))) return r;
  if ((r = upload(T->allocs, has_l1, &L.has_l1))) return r;
  if ((r = upload(T->allocs, active, &L.active))) return r;
  if ((r = upload(T->allocs, rebase(d->inst_term, d->n_inst), &L.inst_term))) return r;
  if ((r = upload(T->allocs, rebase(d->eprog_ptr, d->n_terms + 1), &L.eprog_ptr))) return r;
  if ((r = upload(T->allocs, eent_w, &L.eent_w))) return r;
  if ((r = upload(T->allocs, rebase(d->efac_ptr, d->n_eent + 1), &L.efac_ptr))) return r;
  if ((r = upload(T->allocs, efac_row, &L.efac_row))) return r;
  if ((r = upload(T->allocs, term_coef, &L.term_coef))) return r;
  L.fast = fast ? 1 : 0;
  L.dmax = F.dmax;
  L.rmax = F.rmax;
  if (fast) {
    if ((r = upload(T->allocs, F.nb_ptr, &L.nb_ptr))) return r;
    if ((r = upload(T->allocs, F.nb_list, &L.nb_list))) return r;
    if ((r = upload(T->allocs, F.fr_ptr, &L.fr_ptr))) return r;
    if ((r = upload(T->allocs, F.fr_cnt, &L.fr_cnt))) return r;
    std::vector<int4> idesc(d->n_active);
    for (int64_t qpos = 0; qpos < d->n_active; ++qpos) {
      const int32_t site = cs[qpos];
      const uint32_t c = F.fr_cnt[site];
      const int32_t nd = F.nb_ptr[site + 1] - F.nb_ptr[site];
      idesc[qpos] = make_int4(site | (d->site_has_l1[site] ? (1 << 30) : 0) | ((c >> 24) ? (int)(1u << 31) : 0),
                              F.nb_ptr[site], F.fr_ptr[site], (int32_t)((c & 0xffffffu) | ((uint32_t)nd << 24)));
    }
    if ((r = upload(T->allocs, idesc, &L.idesc))) return r;
    if ((r = upload(T->allocs, F.frec, &L.frec))) return r;
    if ((r = upload(T->allocs, F.ft, &L.ftensor))) return r;
  }
  T->has_generic = keep_generic;
  T->fast_records = (int64_t)F.frec.size();
  T->trip2 = F.n_trip2 > 0;
  T->color_ptr = cp;
  T->site_col_of.assign(ns, 0);
  for (int32_t c = 0; c < d->n_colors; ++c)
    for (int32_t q = cp[c]; q < cp[c + 1]; ++q) T->site_col_of[d->color_sites[q] - 1] = c + 1;
  if (d->n_colors > 32767) return fail(SCEMC_ERR_UNSUPPORTED, "more than 32767 colours");
  {
    std::vector<int16_t> sc(T->site_col_of.begin(), T->site_col_of.end());
    if ((r = upload(T->allocs, sc, &L.site_colour))) return r;
  }
  T->active = active;
  T->n_sites = ns;
  T->nlm = d->nlm;
  T->lmax = d->lmax;
  T->n_colors = d->n_colors;
  T->n_active = d->n_active;
  T->n_cell_atoms = d->n_cell_atoms;
  T->n_inst = d->n_inst;
  T->d_mean = d->n_active ? (double)d_sum / d->n_active : 0.0;
  T->a_mean = d->n_active ? (double)a_sum / d->n_active : 0.0;
  T->bytes = (int64_t)(rec_v.size() * 16 + adj_ptr.size() * 4 + tensor.size() * 4 + sent_w.size() * 6 +
                       d->n_inst_sites * 4 + d->n_inst * 8 + F.frec.size() * 8 + F.nb_list.size() * 4 +
                       F.ft.size() * 4 + (F.nb_ptr.size() + F.fr_ptr.size()) * 4);
  return SCEMC_OK;
}

// ---- ensemble helpers ----------------------------------------------------------
template <typename T>
int32_t dalloc(T** p, size_t n) {
  CUDA_TRY(cudaMalloc((void**)p, std::max<size_t>(n * sizeof(T), 16)));
  CUDA_TRY(cudaMemset(*p, 0, std::max<size_t>(n * sizeof(T), 16)));
  // the legacy-stream clear is not ordered before work on the batches' non-blocking
  // streams: wait for it here (allocation happens at set-up, outside any capture)
  CUDA_TRY(cudaStreamSynchronize(0));
  return SCEMC_OK;
}

int sm_count(int dev);

// Host payloads (per table, per replica 3 x n_sites FP64, the tables one after the
// other) cross the bus unchanged, in one copy each way. Kernels check them, round
// them to FP32 and interleave the replicas (spins[site * R + r]) on the device.
__global__ void k_payload_check(const double* cfg, int64_t n, unsigned long long* bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = cfg[3 * i], y = cfg[3 * i + 1], z = cfg[3 * i + 2];
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicMin(bad, (unsigned long long)i);
  }
}

// One table, walked in device order so that the float4 stores coalesce. Writes
// nothing when the check flagged a spin; block 0 of the first table's launch also
// commits the uploaded energies.
__global__ void k_payload_in(const double* cfg, int64_t n_sites, int R, float4* spins, const unsigned long long* bad,
                             const double* energy_in, double* energy, int n_slots) {
  if (*bad != ~0ull) return;
  if (energy_in != nullptr && blockIdx.x == 0)
    for (int i = threadIdx.x; i < n_slots; i += blockDim.x) energy[i] = energy_in[i];
  const int64_t tot = n_sites * R;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < tot; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = j / R;
    const double* c = cfg + 3 * ((j - s * R) * n_sites + s);
    spins[j] = make_float4((float)c[0], (float)c[1], (float)c[2], 0.0f);
  }
}

__global__ void k_payload_out(const float4* spins, int64_t n_sites, int R, double* cfg) {
  const int64_t tot = n_sites * R;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < tot; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = j / R;
    const float4 v = spins[j];
    double* c = cfg + 3 * ((j - s * R) * n_sites + s);
    c[0] = v.x;
    c[1] = v.y;
    c[2] = v.z;
  }
}

unsigned payload_blocks(const scemc_ensemble* E, int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(E->device) * 16));
}

// Pinned host area for the small transfers: the non-finite flag, the energies on
// the way in, and the per-slot readback block on the way out.
constexpr size_t kSmallIn = 16;
size_t small_out_offset(int n_slots) { return kSmallIn + (((size_t)8 * n_slots + 15) & ~(size_t)15); }
size_t small_bytes(int n_slots) { return small_out_offset(n_slots) + kReadbackBytesPerSlot * n_slots + 64; }

// Replaces every chain's spins (and, when `energies` is given, the running
// energies) from a host payload. Nothing on the device changes when an input is
// not finite: the kernels commit only when the check found nothing, and the host
// reads the check's result after one wait. Returns after the host buffers may be
// reused.
int32_t payload_upload(scemc_ensemble* E, const double* cfgs, const double* energies) {
  if (energies)
    for (int i = 0; i < E->n_slots; ++i)
      if (!std::isfinite(energies[i])) return fail(SCEMC_ERR_ARG, "energy must be finite");
  const int64_t n = E->n_spins;
  auto* h_bad = reinterpret_cast<unsigned long long*>(E->h_small);
  CUDA_TRY(cudaMemsetAsync(E->d_bad, 0xff, sizeof(unsigned long long), E->stream));
  if (energies) {
    double* h_en = reinterpret_cast<double*>(E->h_small + kSmallIn);
    std::memcpy(h_en, energies, sizeof(double) * E->n_slots);
    CUDA_TRY(cudaMemcpyAsync(E->d_energy_in, h_en, sizeof(double) * E->n_slots, cudaMemcpyHostToDevice, E->stream));
  }
  if (n > 0) {
    CUDA_TRY(cudaMemcpyAsync(E->d_cfg64, cfgs, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, E->stream));
    k_payload_check<<<payload_blocks(E, n), 256, 0, E->stream>>>(E->d_cfg64, n, E->d_bad);
    CUDA_TRY(cudaGetLastError());
  }
  for (size_t ti = 0; ti < E->tabs.size(); ++ti) {
    const int64_t ns = E->tabs[ti]->n_sites;
    k_payload_in<<<payload_blocks(E, ns * E->R[ti]), 256, 0, E->stream>>>(
        E->d_cfg64 + 3 * E->spin_off[ti], ns, E->R[ti], E->d_spins + E->spin_off[ti], E->d_bad,
        ti == 0 && energies ? E->d_energy_in : nullptr, E->d_energy, E->n_slots);
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaMemcpyAsync(h_bad, E->d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost, E->stream));
  CUDA_TRY(cudaStreamSynchronize(E->stream));
  if (*h_bad != ~0ull) {
    const int64_t p = (int64_t)*h_bad;
    size_t ti = 0;
    while (ti + 1 < E->tabs.size() && p >= E->spin_off[ti + 1]) ++ti;
    const int64_t local = p - E->spin_off[ti], ns = E->tabs[ti]->n_sites;
    return fail(SCEMC_ERR_NUMERIC, "spin column " + std::to_string(local % ns + 1) + " of replica " +
                                       std::to_string(local / ns + 1) + " is not finite");
  }
  return SCEMC_OK;
}

// Destinations of a download (each may be NULL).
struct DownloadDst {
  double* configs = nullptr;
  double* energies = nullptr;
  int32_t* slot_of_rung = nullptr;
  int64_t* counters = nullptr;
  int64_t* swaps = nullptr;
  double* steps = nullptr;
  double* max_drift = nullptr;
};

// Everything is read on the batch stream (after the work enqueued on it) and
// waited for once.
int32_t payload_download(const scemc_ensemble* E, const DownloadDst& d) {
  const int n = E->n_slots;
  if (d.configs && E->n_spins > 0) {
    for (size_t ti = 0; ti < E->tabs.size(); ++ti) {
      const int64_t ns = E->tabs[ti]->n_sites;
      k_payload_out<<<payload_blocks(E, ns * E->R[ti]), 256, 0, E->stream>>>(
          E->d_spins + E->spin_off[ti], ns, E->R[ti], E->d_cfg64 + 3 * E->spin_off[ti]);
      CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaMemcpyAsync(d.configs, E->d_cfg64, sizeof(double) * 3 * E->n_spins, cudaMemcpyDeviceToHost,
                             E->stream));
  }
  struct Part {
    void* dst;
    size_t off, bytes;
  } parts[] = {{d.energies, kRbEnergy * n, (size_t)8 * n}, {d.slot_of_rung, kRbSlotOfRung * n, (size_t)4 * n},
               {d.counters, kRbCounters * n, (size_t)32 * n}, {d.swaps, kRbSwaps * n, (size_t)16 * n},
               {d.steps, kRbSteps * n, (size_t)8 * n}, {d.max_drift, kRbMaxDrift * n, (size_t)8 * n}};
  bool any = false;
  for (const Part& pt : parts) any = any || pt.dst != nullptr;
  unsigned char* h = E->h_small + small_out_offset(n);
  if (any)
    CUDA_TRY(cudaMemcpyAsync(h, E->d_readback, kReadbackBytesPerSlot * (size_t)n, cudaMemcpyDeviceToHost, E->stream));
  CUDA_TRY(cudaStreamSynchronize(E->stream));
  for (const Part& pt : parts)
    if (pt.dst) std::memcpy(pt.dst, h + pt.off, pt.bytes);
  return SCEMC_OK;
}

int32_t create_ensemble(int32_t n_tables, const scemc_tables* const* tables, const int32_t* replicas,
                        const double* configs, const double* energies, const uint64_t* seeds, const double* steps,
                        scemc_ensemble** out) {
  if (!out) return fail(SCEMC_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (n_tables < 1 || !tables || !replicas || !configs || !energies || !seeds || !steps)
    return fail(SCEMC_ERR_ARG, "bad batch arguments");
  auto* E = new scemc_ensemble();
  std::unique_ptr<scemc_ensemble> guard(E);
  CUDA_TRY(cudaGetDevice(&E->device));
  CUDA_TRY(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  int64_t off = 0;
  int32_t slots = 0;
  for (int i = 0; i < n_tables; ++i) {
    if (!tables[i]) return fail(SCEMC_ERR_ARG, "a table set is NULL");
    if (replicas[i] < 1) return fail(SCEMC_ERR_ARG, "replicas must be >= 1");
    E->tabs.push_back(tables[i]);
    E->R.push_back(replicas[i]);
    E->slot0.push_back(slots);
    E->spin_off.push_back(off);
    off += (int64_t)tables[i]->n_sites * replicas[i];
    slots += replicas[i];
    E->lmax = std::max(E->lmax, tables[i]->lmax);
    E->max_colors = std::max(E->max_colors, tables[i]->n_colors);
  }
  if (slots > kMaxSlots) return fail(SCEMC_ERR_ARG, "at most 512 replica slots per batch");
  E->n_slots = slots;
  E->n_spins = off;
  for (int i = 0; i < slots; ++i)
    if (!(steps[i] > 0) || !std::isfinite(energies[i])) return fail(SCEMC_ERR_ARG, "step must be > 0 and energy finite");
  int32_t rc;
  if ((rc = dalloc(&E->d_spins, off))) return rc;
  if ((rc = dalloc(&E->d_cfg64, (size_t)3 * std::max<int64_t>(off, 1))) || (rc = dalloc(&E->d_bad, 1))) return rc;
  CUDA_TRY(cudaHostAlloc((void**)&E->h_small, small_bytes(slots), cudaHostAllocDefault));
  // lattice descriptors with per-batch geometry
  std::vector<DevLattice> lats(n_tables);
  int max_atoms = 1;
  for (int i = 0; i < n_tables; ++i) {
    lats[i] = tables[i]->dl;
    lats[i].R = replicas[i];
    lats[i].slot0 = E->slot0[i];
    lats[i].spin_off = E->spin_off[i];
    max_atoms = std::max(max_atoms, tables[i]->n_cell_atoms);
  }
  if ((rc = dalloc(&E->d_lat, n_tables))) return rc;
  CUDA_TRY(h2d_sync(E->d_lat, lats.data(), sizeof(DevLattice) * n_tables));
  // per-colour item prefixes
  E->seg.assign((size_t)std::max(E->max_colors, 1) * (n_tables + 1), 0);
  for (int c = 0; c < E->max_colors; ++c) {
    int64_t acc = 0;
    for (int i = 0; i < n_tables; ++i) {
      E->seg[(size_t)c * (n_tables + 1) + i] = (int32_t)acc;
      const scemc_tables* T = tables[i];
      if (c < T->n_colors) acc += (int64_t)(T->color_ptr[c + 1] - T->color_ptr[c]) * replicas[i];
    }
    if (acc > 0x7fffffffll) return fail(SCEMC_ERR_UNSUPPORTED, "more than 2^31 items in one colour class");
    E->seg[(size_t)c * (n_tables + 1) + n_tables] = (int32_t)acc;
  }
  if ((rc = dalloc(&E->d_seg, E->seg.size()))) return rc;
  CUDA_TRY(h2d_sync(E->d_seg, E->seg.data(), E->seg.size() * 4));
  E->item_base.assign(E->max_colors + 1, 0);
  for (int c = 0; c < E->max_colors; ++c) {
    const int64_t nb = (int64_t)E->item_base[c] + E->seg[(size_t)c * (n_tables + 1) + n_tables];
    if (nb > 0x7fffffffll) return fail(SCEMC_ERR_UNSUPPORTED, "more than 2^31 items in one pass");
    E->item_base[c + 1] = (int32_t)nb;
  }
  if ((rc = dalloc(&E->d_item_base, E->item_base.size()))) return rc;
  CUDA_TRY(h2d_sync(E->d_item_base, E->item_base.data(), E->item_base.size() * 4));
  E->fast = true;
  for (int i = 0; i < n_tables; ++i) {
    E->fast = E->fast && tables[i]->dl.fast && tables[i]->lmax == E->lmax;
    E->trip2 = E->trip2 || tables[i]->trip2;
    E->dmax = std::max(E->dmax, tables[i]->dl.dmax);
    E->rmax = std::max(E->rmax, tables[i]->dl.rmax);
  }
  // the per-slot arrays a download returns share one allocation, read back in one copy
  if ((rc = dalloc(&E->d_readback, kReadbackBytesPerSlot * (size_t)slots))) return rc;
  {
    unsigned char* rb = E->d_readback;
    const size_t n = (size_t)slots;
    E->d_energy = reinterpret_cast<double*>(rb + kRbEnergy * n);
    E->d_slot_of_rung = reinterpret_cast<int32_t*>(rb + kRbSlotOfRung * n);
    E->d_cnt = reinterpret_cast<unsigned long long*>(rb + kRbCounters * n);
    E->d_swaps = reinterpret_cast<unsigned long long*>(rb + kRbSwaps * n);
    E->d_step = reinterpret_cast<double*>(rb + kRbSteps * n);
    E->d_max_drift = reinterpret_cast<double*>(rb + kRbMaxDrift * n);
  }
  if ((rc = dalloc(&E->d_dEfix, slots)) || (rc = dalloc(&E->d_win, 2 * slots)) || (rc = dalloc(&E->d_beta, slots)) ||
      (rc = dalloc(&E->d_seed, slots)) || (rc = dalloc(&E->d_rung_of_slot, slots)) ||
      (rc = dalloc(&E->d_drift, slots)) || (rc = dalloc(&E->d_energy_in, slots)) || (rc = dalloc(&E->d_eout, slots)) ||
      (rc = dalloc(&E->d_gs, 1)) || (rc = dalloc(&E->d_st, 1)))
    return rc;
  std::vector<int32_t> ident(slots);
  for (int i = 0; i < slots; ++i) ident[i] = i;
  CUDA_TRY(h2d_sync(E->d_slot_of_rung, ident.data(), 4 * slots));
  CUDA_TRY(h2d_sync(E->d_rung_of_slot, ident.data(), 4 * slots));
  CUDA_TRY(h2d_sync(E->d_energy, energies, 8 * slots));
  CUDA_TRY(h2d_sync(E->d_step, steps, 8 * slots));
  CUDA_TRY(h2d_sync(E->d_seed, seeds, 8 * slots));
  std::vector<double> ones(slots, 1.0);
  CUDA_TRY(h2d_sync(E->d_beta, ones.data(), 8 * slots));
  E->rec_len = 4 + 3 * max_atoms;
  if ((rc = payload_upload(E, configs, nullptr))) return rc;
  *out = guard.release();
  return SCEMC_OK;
}

// Sweep launch ----------------------------------------------------------------
using KFn = void (*)(SweepArgs);

template <int LMAX>
KFn pick_colour(int G) {
  switch (G) {
    case 1: return k_sweep_colour<LMAX, 1>;
    case 2: return k_sweep_colour<LMAX, 2>;
    case 4: return k_sweep_colour<LMAX, 4>;
    case 8: return k_sweep_colour<LMAX, 8>;
    case 16: return k_sweep_colour<LMAX, 16>;
    default: return k_sweep_colour<LMAX, 32>;
  }
}
template <int LMAX>
KFn pick_persist(int G) {
  switch (G) {
    case 1: return k_sweep_persistent<LMAX, 1>;
    case 2: return k_sweep_persistent<LMAX, 2>;
    case 4: return k_sweep_persistent<LMAX, 4>;
    case 8: return k_sweep_persistent<LMAX, 8>;
    case 16: return k_sweep_persistent<LMAX, 16>;
    default: return k_sweep_persistent<LMAX, 32>;
  }
}

KFn kernel_for(int lmax, int G, bool persist) {
  switch (lmax) {
    case 0: return persist ? pick_persist<0>(G) : pick_colour<0>(G);
    case 1: return persist ? pick_persist<1>(G) : pick_colour<1>(G);
    case 2: return persist ? pick_persist<2>(G) : pick_colour<2>(G);
    case 3: return persist ? pick_persist<3>(G) : pick_colour<3>(G);
    case 4: return persist ? pick_persist<4>(G) : pick_colour<4>(G);
    case 5: return persist ? pick_persist<5>(G) : pick_colour<5>(G);
    default: return persist ? pick_persist<6>(G) : pick_colour<6>(G);
  }
}

int norm_lanes(int lanes) {
  if (lanes <= 1) return 1;
  int g = 1;
  while (g < lanes && g < 32) g <<= 1;
  return g;
}

SweepArgs make_args(scemc_ensemble* E, int pass) {
  SweepArgs a{};
  a.lat = E->d_lat;
  a.n_lat = (int32_t)E->tabs.size();
  a.n_slots = E->n_slots;
  a.spins = E->d_spins;
  a.seg = E->d_seg;
  a.max_colors = E->max_colors;
  a.pass = pass;
  a.sweep = (uint32_t)(E->sweep_index + 1);
  a.st = E->d_st;
  a.rung_of_slot = E->d_rung_of_slot;
  a.beta = E->d_beta;
  a.step = E->d_step;
  a.seed = E->d_seed;
  a.dE_fix = E->d_dEfix;
  a.cnt = E->d_cnt;
  a.gs = E->d_gs;
  a.barrier_limit_ns = E->barrier_limit_ns;
  if (E->recording) {
    a.rec_li = E->rec_li;
    a.rec_r = E->rec_r;
    a.rec_cap = E->rec_cap;
    a.rec_prop = E->d_rprop;
    a.rec_u = E->d_ru;
    a.rec_dE = E->d_rdE;
    a.rec_acc = E->d_racc;
    a.rec_lqr = E->d_rlqr;
  }
  return a;
}

int sm_count(int dev) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

cudaEvent_t take_event(scemc_ensemble* E) {
  if (!E->ev_pool.empty()) {
    cudaEvent_t e = E->ev_pool.back();
    E->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Folds the elapsed time of completed pass event pairs (after a stream sync).
void harvest_events(scemc_ensemble* E) {
  for (auto& pr : E->ev_pending) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
      E->prof_ms += ms;
      E->prof_passes += E->graph_passes_per_launch > 0 ? E->graph_passes_per_launch : 1;
    }
    E->ev_pool.push_back(pr.first);
    E->ev_pool.push_back(pr.second);
  }
  E->ev_pending.clear();
  E->graph_passes_per_launch = 0;
}

// Resolved launch configuration of a sweep pass.
struct Launch {
  int G = 1;          // lanes per item (generic kernel); the fast kernel fixes its own
  int mode = 2;       // 1 = one launch per colour, 2 = persistent cooperative kernel
  bool graph = false; // per-colour launches of a compound sweep captured in a CUDA graph
  bool fast = false;  // row-parallel fast kernel (one warp per item)
  bool rep = false;   // replica-parallel kernel (one thread per item, per-colour launches)
  bool precompute = false;  // Metropolis proposals computed before the colour loop
  bool learned = false;     // Metropolis proposals from the learned network, per colour
  bool flow = false;        // persistent form with per-item completion flags instead of grid barriers
  int rep_p = 0;            // replica-parallel kernel: replicas per thread (0 = per colour, by its size)
  int rep_np = 0;           // replica-parallel kernel: threads per item (0 = per colour, by its size)
  int rep_pf = 0;           // replica-parallel kernel: 1 prefetch, 2 no prefetch (0 = per colour, by its size)
  bool cluster = false;     // chain-resident cluster kernel: one launch per compound sweep
  bool rep_tc = false;      // replica-parallel pass with the pair records on the tensor cores (kernel 5)
};

using FastFn = void (*)(SweepArgs);

FastFn fast_kernel(int lmax, bool persist) {
  if (lmax == 1) return persist ? k_fast_persistent<1> : k_fast_colour<1>;
  return persist ? k_fast_persistent<2> : k_fast_colour<2>;
}

int fast_rows(int lmax) { return lmax == 1 ? 3 : 8; }
int fast_group(int lmax) { return lmax == 1 ? 4 : 8; }

// Threads per block and dynamic shared memory (neighbour Z rows) of the fast kernel.
void fast_shape(const scemc_ensemble* E, int* threads, size_t* smem) {
  const int NR = fast_rows(E->lmax);
  const size_t per_warp = fast_group_floats(std::max(E->dmax, 1), std::max(E->rmax, 1), NR) * sizeof(float);
  const size_t params = fast_param_floats(E->n_slots) * sizeof(float);
  int t = SCEMC_FAST_THREADS;
  size_t m = params + (size_t)(t / 32) * per_warp;
  while (m > 160 * 1024 && t > 32) {
    t /= 2;
    m = params + (size_t)(t / 32) * per_warp;
  }
  *threads = t;
  *smem = m;
}

int32_t ensure_props(scemc_ensemble* E) {
  if (E->d_prop) return SCEMC_OK;
  const int64_t n = std::max<int32_t>(E->item_base.back(), 1);
  int32_t rc;
  if ((rc = dalloc(&E->d_prop, n)) || (rc = dalloc(&E->d_propu, n))) return rc;
  return SCEMC_OK;
}

int32_t run_pass_impl(scemc_ensemble* E, int pass, const Launch& Lc);

// One pass (Metropolis or OR pass k) over every colour, optionally timed.
int32_t run_pass(scemc_ensemble* E, int pass, const Launch& Lc) {
  if (!E->profiling) return run_pass_impl(E, pass, Lc);
  cudaEvent_t a = take_event(E), b = take_event(E);
  CUDA_TRY(cudaEventRecord(a, E->stream));
  const int32_t rc = run_pass_impl(E, pass, Lc);
  CUDA_TRY(cudaEventRecord(b, E->stream));
  E->ev_pending.emplace_back(a, b);
  return rc;
}

int max_colour_items(const scemc_ensemble* E) {
  int m = 1;
  for (int c = 0; c < E->max_colors; ++c) m = std::max(m, E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()]);
  return m;
}

// Learned Metropolis pass: per colour, the fused network + mixture-draw kernel, then
// the sweep kernel on those proposals.
// The fused learned kernel with the Metropolis-Hastings decision, and its dynamic
// shared memory (the per-slot accumulators follow the network's tiles).
using LearnedFn = void (*)(SweepArgs, LearnedNet, double*);
LearnedFn learned_mh_kernel(int lmax, bool field) {
  if (field) return lmax == 1 ? k_learned_fused<1, true, true> : k_learned_fused<2, true, true>;
  return lmax == 1 ? k_learned_fused<1, true> : k_learned_fused<2, true>;
}
size_t learned_smem(const scemc_ensemble* E, bool mh) {
  return kLearnedSmem + (mh ? (size_t)20 * E->n_slots + 16 : 0);
}

int32_t prepare_learned(scemc_ensemble* E) {
  int32_t rc;
  if ((rc = ensure_props(E))) return rc;
  if (!E->d_lqr && (rc = dalloc(&E->d_lqr, (size_t)std::max<int32_t>(E->item_base.back(), 1)))) return rc;
  CUDA_TRY(cudaFuncSetAttribute((const void*)k_learned_fused<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kLearnedSmem));
  CUDA_TRY(cudaFuncSetAttribute((const void*)learned_mh_kernel(E->lmax, E->learned_field),
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)learned_smem(E, true)));
  return SCEMC_OK;
}

// Threads of a replica-parallel launch of colour c with P replicas per thread.
int64_t rep_threads(const scemc_ensemble* E, int c, int P) {
  int64_t nt = 0;
  const int32_t* sc = E->seg.data() + (size_t)c * (E->tabs.size() + 1);
  for (size_t li = 0; li < E->tabs.size(); ++li)
    nt += (int64_t)(sc[li + 1] - sc[li]) / E->R[li] * ((E->R[li] + P - 1) / P);
  return nt;
}

// The replica-parallel form of one colour launch: replicas per thread P, threads per
// item NP, and whether each thread first prefetches its neighbour rows into L1 (at
// most two waves of resident threads: the record walk is then latency-bound;
// measured 9 % faster on the PT ladders, 7 % slower at fcc 48^3 x 32).
struct RepForm {
  int P;
  int np;  // threads per item
  int64_t nt;
  int32_t pf;
  FastFn fn;
  size_t smem;  // dynamic shared memory (bytes)
};
RepForm rep_form(const scemc_ensemble* E, int c, int forced, int forced_np = 0, int forced_pf = 0, bool tc = false) {
  RepForm f;
  const int64_t sms = sm_count(E->device);
  if (tc) {  // one warp per (site, 32 replicas)
    int64_t items = 0;
    const int32_t* sc = E->seg.data() + (size_t)c * (E->tabs.size() + 1);
    for (size_t li = 0; li < E->tabs.size(); ++li)
      items += (int64_t)(sc[li + 1] - sc[li]) / E->R[li] * ((E->R[li] + 31) / 32);
    f.P = 1;
    f.np = 1;
    f.pf = 0;
    f.nt = items * 32;
    f.fn = E->trip2 ? k_rep_tc<true> : k_rep_tc<false>;
    f.smem = (fast_param_floats(E->n_slots) + 8 * tc_warp_floats(std::max(E->dmax, 1), std::max(E->rmax, 1))) *
             sizeof(float);
    return f;
  }
  f.smem = fast_param_floats(E->n_slots) * sizeof(float);
  const int64_t nt1 = rep_threads(E, c, 1);
  // Small colours (twice the one-replica threads still fit one wave of four
  // 256-thread blocks per SM): one replica per thread and two threads per item, for
  // the most parallel walk. Larger: two replicas per thread, one thread per item.
  // Measured (ms per sweep of 16 rungs, bcc body-4): 32^3 0.49 against 0.55 with
  // P = 2; 40^3 (above the threshold) 0.70 with P = 2 against 0.76 with P = 1.
  // NP depends on the colour's size only, so a forced P does not change the chains.
  const int NP = forced_np == 1 || forced_np == 2 ? forced_np : (2 * nt1 <= sms * 1024 ? 2 : 1);
  f.P = forced == 1 || forced == 2 ? forced : (NP == 2 ? 1 : 2);
  f.np = NP;
  f.nt = rep_threads(E, c, f.P) * NP;
  f.pf = forced_pf == 1 ? 1 : forced_pf == 2 ? 0 : (f.nt <= sms * (f.P == 1 ? 1024 : 768) * 2 ? 1 : 0);
  // [0: lmax 1, 1: lmax 2 without body-3 l = 2 blocks, 2: lmax 2 with them][P - 1][NP - 1][pf]
  // (the block walk costs registers, so tables without such blocks run instances without it)
  static const FastFn forms[3][2][2][2] = {
      {{{k_rep_colour<1, 1, 1, false>, k_rep_colour<1, 1, 1, true>},
        {k_rep_colour<1, 1, 2, false>, k_rep_colour<1, 1, 2, true>}},
       {{k_rep_colour<1, 2, 1, false>, k_rep_colour<1, 2, 1, true>},
        {k_rep_colour<1, 2, 2, false>, k_rep_colour<1, 2, 2, true>}}},
      {{{k_rep_colour<2, 1, 1, false, false>, k_rep_colour<2, 1, 1, true, false>},
        {k_rep_colour<2, 1, 2, false, false>, k_rep_colour<2, 1, 2, true, false>}},
       {{k_rep_colour<2, 2, 1, false, false>, k_rep_colour<2, 2, 1, true, false>},
        {k_rep_colour<2, 2, 2, false, false>, k_rep_colour<2, 2, 2, true, false>}}},
      {{{k_rep_colour<2, 1, 1, false, true>, k_rep_colour<2, 1, 1, true, true>},
        {k_rep_colour<2, 1, 2, false, true>, k_rep_colour<2, 1, 2, true, true>}},
       {{k_rep_colour<2, 2, 1, false, true>, k_rep_colour<2, 2, 1, true, true>},
        {k_rep_colour<2, 2, 2, false, true>, k_rep_colour<2, 2, 2, true, true>}}}};
  f.fn = forms[E->lmax == 1 ? 0 : (E->trip2 ? 2 : 1)][f.P - 1][NP - 1][f.pf];
  return f;
}

int32_t run_learned_pass(scemc_ensemble* E, const Launch& Lc) {
  SweepArgs a = make_args(E, -1);
  int32_t rc;
  if ((rc = prepare_learned(E))) return rc;
  a.item_base = E->d_item_base;
  a.prop = E->d_prop;
  a.propu = E->d_propu;
  a.dmax = std::max(E->dmax, 1);
  a.rmax = std::max(E->rmax, 1);
  const int cap = sm_count(E->device) * 64;
  LearnedNet net;
  net.W1 = E->mlp->d_W1;
  net.W2 = E->mlp->d_W2;
  net.W3 = E->mlp->d_W3;
  net.b1 = E->mlp->d_master + mlpl::oB1;
  net.b2 = E->mlp->d_master + mlpl::oB2;
  net.b3 = E->mlp->d_master + mlpl::oB3;
  net.err = &E->d_gs->error;
  for (int c = 0; c < E->max_colors; ++c) {
    const int n = E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()];
    if (n == 0) continue;
    a.colour = c;
    a.lqr = nullptr;
    const int tiles = (n + kTile - 1) / kTile;
    const unsigned grid = (unsigned)std::min(tiles, 2 * sm_count(E->device));
    ++E->launches;
    if (Lc.rep) {  // the replica-parallel decision runs inside the fused kernel
      const auto fn = learned_mh_kernel(E->lmax, E->learned_field);
      fn<<<grid, 256, learned_smem(E, true), E->stream>>>(a, net, E->d_lqr);
      CUDA_TRY(cudaGetLastError());
      continue;
    }
    k_learned_fused<1, false><<<grid, 256, kLearnedSmem, E->stream>>>(a, net, E->d_lqr);
    CUDA_TRY(cudaGetLastError());
    a.lqr = E->d_lqr;
    ++E->launches;
    {
      int threads;
      size_t smem;
      fast_shape(E, &threads, &smem);
      FastFn fn = fast_kernel(E->lmax, false);
      CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int blocks = (int)std::min<int64_t>(sm_count(E->device) * 16, ((int64_t)n * 32 + threads - 1) / threads);
      fn<<<std::max(blocks, 1), threads, smem, E->stream>>>(a);
    }
    CUDA_TRY(cudaGetLastError());
  }
  return SCEMC_OK;
}

// The persistent replica-parallel pass: its P and NP are the form rep_form picks for
// the colour with the most items (or the forced ones); cooperative launch of at most
// the co-resident blocks.
int32_t run_rep_persistent(scemc_ensemble* E, SweepArgs a, const Launch& Lc) {
  int cbig = 0;
  for (int c = 0; c < E->max_colors; ++c)
    if (E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()] >
        E->seg[(size_t)cbig * (E->tabs.size() + 1) + E->tabs.size()])
      cbig = c;
  const RepForm f = rep_form(E, cbig, Lc.rep_p, Lc.rep_np, 2);
  const int NP = f.np;
  using PFn = void (*)(SweepArgs);
  static const PFn forms[3][2][2] = {{{k_rep_persistent<1, 1, 1>, k_rep_persistent<1, 1, 2>},
                                      {k_rep_persistent<1, 2, 1>, k_rep_persistent<1, 2, 2>}},
                                     {{k_rep_persistent<2, 1, 1, false>, k_rep_persistent<2, 1, 2, false>},
                                      {k_rep_persistent<2, 2, 1, false>, k_rep_persistent<2, 2, 2, false>}},
                                     {{k_rep_persistent<2, 1, 1, true>, k_rep_persistent<2, 1, 2, true>},
                                      {k_rep_persistent<2, 2, 1, true>, k_rep_persistent<2, 2, 2, true>}}};
  if (f.P != 1 && f.P != 2) return fail(SCEMC_ERR_ARG, "the persistent replica-parallel form takes 1 or 2 replicas per thread");
  const PFn fn = forms[E->lmax == 1 ? 0 : (E->trip2 ? 2 : 1)][f.P - 1][NP - 1];
  const int threads = 256;
  const size_t smem = fast_param_floats(E->n_slots) * sizeof(float);
  CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int key[4] = {3, E->lmax, f.P, NP};
  if (!std::equal(key, key + 4, E->coop_key)) {
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, threads, smem));
    if (per_sm < 1) return fail(SCEMC_ERR_CUDA, "persistent replica-parallel kernel cannot be resident");
    E->coop_blocks = per_sm * sm_count(E->device);
    std::copy(key, key + 4, E->coop_key);
  }
  int64_t need = 1;
  for (int c = 0; c < E->max_colors; ++c) need = std::max<int64_t>(need, rep_threads(E, c, f.P) * NP);
  need = (need + threads - 1) / threads;
  if (a.prop) need = std::max<int64_t>(need, ((int64_t)E->item_base.back() + threads - 1) / threads);
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(E->coop_blocks, need));
  a.bar_base = E->bar_base;
  void* params[] = {&a};
  ++E->launches;
  CUDA_TRY(cudaLaunchCooperativeKernel((const void*)fn, dim3(blocks), dim3(threads), params, smem, E->stream));
  E->bar_base += (unsigned long long)blocks * ((a.prop ? 1 : 0) + std::max(E->max_colors - 1, 0));
  return SCEMC_OK;
}

int32_t run_pass_impl(scemc_ensemble* E, int pass, const Launch& Lc) {
  const int lmax = E->lmax;
  if (Lc.learned && pass < 0) return run_learned_pass(E, Lc);
  SweepArgs a = make_args(E, pass);
  const int max_items = max_colour_items(E);
  if (Lc.rep) {
    const int threads = 256;
    a.item_base = E->d_item_base;
    const int cap = sm_count(E->device) * 64;
    if (Lc.precompute && pass < 0) {
      int32_t rc;
      if ((rc = ensure_props(E))) return rc;
      a.prop = E->d_prop;
      a.propu = E->d_propu;
      if (Lc.mode == 2) return run_rep_persistent(E, a, Lc);  // proposals inside the persistent launch
      const int blocks = (int)std::min<int64_t>(cap, ((int64_t)E->item_base.back() + 255) / 256);
      ++E->launches;
      k_proposals<<<std::max(blocks, 1), 256, 0, E->stream>>>(a);
      CUDA_TRY(cudaGetLastError());
    }
    if (Lc.mode == 2) return run_rep_persistent(E, a, Lc);
    a.dmax = std::max(E->dmax, 1);
    a.rmax = std::max(E->rmax, 1);
    for (int c = 0; c < E->max_colors; ++c) {
      const int n = E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()];
      if (n == 0) continue;
      a.colour = c;
      const RepForm f = rep_form(E, c, Lc.rep_p, Lc.rep_np, Lc.rep_pf, Lc.rep_tc);
      CUDA_TRY(cudaFuncSetAttribute((const void*)f.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.smem));
      const int blocks = (int)std::min<int64_t>(cap, (f.nt + threads - 1) / threads);
      ++E->launches;
      f.fn<<<std::max(blocks, 1), threads, f.smem, E->stream>>>(a);
      CUDA_TRY(cudaGetLastError());
    }
    return SCEMC_OK;
  }
  if (Lc.fast) {
    int threads;
    size_t smem;
    fast_shape(E, &threads, &smem);
    const int G = 32;  // one warp per item
    a.dmax = std::max(E->dmax, 1);
    a.rmax = std::max(E->rmax, 1);
    a.item_base = E->d_item_base;
    if (Lc.precompute && pass < 0) {
      int32_t rc;
      if ((rc = ensure_props(E))) return rc;
      a.prop = E->d_prop;
      a.propu = E->d_propu;
    }
    FastFn fn = fast_kernel(lmax, Lc.mode == 2);
    CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (Lc.mode == 2) {
      const int key[4] = {2, lmax, threads, (int)smem};
      if (!std::equal(key, key + 4, E->coop_key)) {
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, threads, smem));
        if (per_sm < 1) return fail(SCEMC_ERR_CUDA, "persistent fast sweep kernel cannot be resident");
        E->coop_blocks = per_sm * sm_count(E->device);
        std::copy(key, key + 4, E->coop_key);
      }
      int64_t need = ((int64_t)max_items * G + threads - 1) / threads;
      if (a.prop) need = std::max<int64_t>(need, ((int64_t)E->item_base.back() + threads - 1) / threads);
      const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(E->coop_blocks, need));
      a.bar_base = E->bar_base;
      if (Lc.flow) {
        if (!E->d_flags) {
          int32_t rc;
          if ((rc = dalloc(&E->d_flags, (size_t)std::max<int64_t>(E->n_spins, 1)))) return rc;
          CUDA_TRY(cudaMemsetAsync(E->d_flags, 0, sizeof(uint32_t) * std::max<int64_t>(E->n_spins, 1), E->stream));
        }
        a.flags = E->d_flags;
      }
      void* params[] = {&a};
      ++E->launches;
      CUDA_TRY(cudaLaunchCooperativeKernel((const void*)fn, dim3(blocks), dim3(threads), params, smem, E->stream));
      E->bar_base +=
          (unsigned long long)blocks * ((a.prop ? 1 : 0) + (Lc.flow ? 0 : std::max(E->max_colors - 1, 0)));
      return SCEMC_OK;
    }
    const int cap = sm_count(E->device) * 16;
    if (a.prop) {
      const int blocks = (int)std::min<int64_t>(cap, ((int64_t)E->item_base.back() + 255) / 256);
      ++E->launches;
      k_proposals<<<std::max(blocks, 1), 256, 0, E->stream>>>(a);
      CUDA_TRY(cudaGetLastError());
    }
    for (int c = 0; c < E->max_colors; ++c) {
      const int n = E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()];
      if (n == 0) continue;
      a.colour = c;
      const int blocks = (int)std::min<int64_t>(cap, ((int64_t)n * G + threads - 1) / threads);
      ++E->launches;
      fn<<<std::max(blocks, 1), threads, smem, E->stream>>>(a);
      CUDA_TRY(cudaGetLastError());
    }
    return SCEMC_OK;
  }
  const int threads = 256;
  const int G = Lc.G;
  if (Lc.mode == 2) {
    KFn fn = kernel_for(lmax, G, true);
    const int key[4] = {1, lmax, G, 0};
    if (!std::equal(key, key + 4, E->coop_key)) {
      int per_sm = 0;
      CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, threads, 0));
      if (per_sm < 1) return fail(SCEMC_ERR_CUDA, "persistent sweep kernel cannot be resident");
      E->coop_blocks = per_sm * sm_count(E->device);
      std::copy(key, key + 4, E->coop_key);
    }
    const int want = (int)std::min<int64_t>(E->coop_blocks, ((int64_t)max_items * G + threads - 1) / threads);
    const int blocks = std::max(1, want);
    a.bar_base = E->bar_base;
    void* params[] = {&a};
    ++E->launches;
    CUDA_TRY(cudaLaunchCooperativeKernel((const void*)fn, dim3(blocks), dim3(threads), params, 0, E->stream));
    E->bar_base += (unsigned long long)blocks * std::max(E->max_colors - 1, 0);
    return SCEMC_OK;
  }
  KFn fn = kernel_for(lmax, G, false);
  const int cap = sm_count(E->device) * 8;
  for (int c = 0; c < E->max_colors; ++c) {
    const int n = E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()];
    if (n == 0) continue;
    a.colour = c;
    const int blocks = (int)std::min<int64_t>(cap, ((int64_t)n * G + threads - 1) / threads);
    ++E->launches;
    fn<<<std::max(blocks, 1), threads, 0, E->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
  }
  return SCEMC_OK;
}

int32_t launch_tail(scemc_ensemble* E, bool add_att, bool adapt, double target, bool exchange, bool bump) {
  TailArgs t{};
  t.bump = bump;
  t.n_slots = E->n_slots;
  t.n_rungs = E->n_slots;
  t.n_lat = (int32_t)E->tabs.size();
  t.lat = E->d_lat;
  t.energy = E->d_energy;
  t.dE_fix = E->d_dEfix;
  t.cnt = E->d_cnt;
  t.win = E->d_win;
  t.add_att = add_att;
  t.adapt = adapt;
  t.adapt_target = target;
  t.step = E->d_step;
  t.exchange = exchange;
  t.slot_of_rung = E->d_slot_of_rung;
  t.rung_of_slot = E->d_rung_of_slot;
  t.beta = E->d_beta;
  t.swaps = E->d_swaps;
  t.exchange_seed = E->exchange_seed;
  t.st = E->d_st;
  ++E->launches;
  k_tail<<<1, 128, 0, E->stream>>>(t);
  CUDA_TRY(cudaGetLastError());
  return SCEMC_OK;
}

int32_t ensure_partial(scemc_ensemble* E, size_t n) {
  if (E->partial_cap >= n) return SCEMC_OK;
  if (E->d_partial) cudaFree(E->d_partial);
  E->d_partial = nullptr;
  int32_t rc;
  if ((rc = dalloc(&E->d_partial, n))) return rc;
  E->partial_cap = n;
  return SCEMC_OK;
}

// FP64 recompute for every slot. mode 0: energies into d_eout; mode 1: renormalise.
int32_t recompute(scemc_ensemble* E, int mode) {
  for (size_t li = 0; li < E->tabs.size(); ++li) {
    const scemc_tables* T = E->tabs[li];
    const int R = E->R[li];
    if (mode == 1) {
      const int64_t n = (int64_t)T->n_sites * R;
      const int blocks = (int)std::min<int64_t>(sm_count(E->device) * 4, (n + 255) / 256);
      ++E->launches;
      k_normalize<<<std::max(blocks, 1), 256, 0, E->stream>>>(E->d_lat, (int)li, E->d_spins);
      CUDA_TRY(cudaGetLastError());
    }
    const int n_chunks = (int)std::max<int64_t>(1, (T->n_inst + kChunk - 1) / kChunk);
    int32_t rc;
    if ((rc = ensure_partial(E, (size_t)n_chunks * R))) return rc;
    ++E->launches;
    k_energy_chunks<<<dim3(n_chunks, R), 256, 0, E->stream>>>(E->d_lat, (int)li, E->d_spins, E->d_partial, n_chunks);
    CUDA_TRY(cudaGetLastError());
    ++E->launches;
    k_energy_fold<<<1, 512, 0, E->stream>>>(E->d_lat, (int)li, E->d_partial, n_chunks, E->d_energy, E->d_eout,
                                            E->d_drift, E->d_max_drift, E->d_rung_of_slot, mode);
    CUDA_TRY(cudaGetLastError());
  }
  return SCEMC_OK;
}

int32_t ensure_meas(scemc_ensemble* E, int64_t rows) {
  if (E->meas_n + rows <= E->meas_cap) return SCEMC_OK;
  const int64_t cap = std::max<int64_t>(E->meas_cap * 2, E->meas_n + rows + 64);
  double* p = nullptr;
  int32_t rc;
  if ((rc = dalloc(&p, (size_t)cap * E->n_slots * E->rec_len))) return rc;
  if (E->d_meas && E->meas_n > 0)
    CUDA_TRY(cudaMemcpyAsync(p, E->d_meas, sizeof(double) * E->meas_n * E->n_slots * E->rec_len,
                             cudaMemcpyDeviceToDevice, E->stream));
  CUDA_TRY(cudaStreamSynchronize(E->stream));
  if (E->d_meas) cudaFree(E->d_meas);
  E->d_meas = p;
  E->meas_cap = cap;
  return SCEMC_OK;
}

int32_t measure(scemc_ensemble* E) {
  int32_t rc;
  if ((rc = ensure_meas(E, 1))) return rc;
  double* row = E->d_meas + (size_t)E->meas_n * E->n_slots * E->rec_len;
  for (size_t li = 0; li < E->tabs.size(); ++li) {
    const scemc_tables* T = E->tabs[li];
    const int R = E->R[li];
    const int n_chunks = (T->n_sites + kChunk - 1) / kChunk;
    const int rlen = 3 + 3 * T->n_cell_atoms;
    if ((rc = ensure_partial(E, (size_t)n_chunks * R * rlen))) return rc;
    ++E->launches;
    k_measure_chunks<<<dim3(n_chunks, R), 256, 0, E->stream>>>(E->d_lat, (int)li, E->d_spins, E->d_partial, n_chunks,
                                                               rlen);
    CUDA_TRY(cudaGetLastError());
    ++E->launches;
    k_measure_fold<<<R, 128, 0, E->stream>>>(E->d_lat, (int)li, E->d_partial, n_chunks, rlen, E->d_energy,
                                             E->d_rung_of_slot, row, E->rec_len);
    CUDA_TRY(cudaGetLastError());
  }
  E->meas_n += 1;
  return SCEMC_OK;
}

int32_t check_error(scemc_ensemble* E) {
  GridSync gs;
  CUDA_TRY(cudaMemcpyAsync(&gs, E->d_gs, sizeof(gs), cudaMemcpyDeviceToHost, E->stream));
  CUDA_TRY(cudaStreamSynchronize(E->stream));
  if (gs.error) {
    GridSync z{};
    CUDA_TRY(h2d_sync(E->d_gs, &z, sizeof(z)));
    E->bar_base = 0;
    return fail(SCEMC_ERR_TIMEOUT, "grid barrier wait gave up (bounded spin); state of this sweep is torn");
  }
  return SCEMC_OK;
}

// The chain-resident cluster kernel applies when the batch has the fast tables and
// one replica's spins plus the per-warp scratch fit in one CTA's shared memory.
int32_t cluster_fits(const scemc_ensemble* E) {
  if (!E->fast)
    return fail(SCEMC_ERR_ARG, "the cluster kernel (kernel 4) needs the fast tables (lmax 1 or 2 dense programs)");
  int optin = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, E->device));
  const int nr = fast_rows(E->lmax);
  for (const scemc_tables* T : E->tabs)
    if (cluster_smem_bytes(T->n_sites, std::max(E->dmax, 1), std::max(E->rmax, 1), nr) > (size_t)optin)
      return fail(SCEMC_ERR_ARG, "the cluster kernel (kernel 4) needs one replica's spins (" +
                                     std::to_string(T->n_sites) + " sites x 16 bytes) and its scratch in " +
                                     std::to_string(optin) + " bytes of shared memory");
  return SCEMC_OK;
}

// Cluster size of the chain-resident kernel: enough CTAs that a colour of one replica
// gives every warp about one site, at most 16 (the non-portable limit), and a size
// the device can co-schedule with this kernel's shared memory.
int cluster_size(scemc_ensemble* E, size_t smem) {
  const void* fn = E->lmax == 1 ? (const void*)k_chain_cluster<1> : (const void*)k_chain_cluster<2>;
  int items = 1;
  for (int c = 0; c < E->max_colors; ++c)
    for (size_t li = 0; li < E->tabs.size(); ++li) {
      const int32_t* sc = E->seg.data() + (size_t)c * (E->tabs.size() + 1);
      items = std::max(items, (sc[li + 1] - sc[li]) / E->R[li]);
    }
  const int warps = kClusterThreads / 32;
  int want = 1;
  while (want < 16 && want * warps < items) want <<= 1;
  for (int cs = want; cs >= 1; cs >>= 1) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)cs);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) == cudaSuccess && n > 0) return cs;
    cudaGetLastError();
  }
  return 0;
}

// One compound sweep (Metropolis + n_or overrelaxation passes) of every replica slot
// through the chain-resident cluster kernel: one cluster per slot.
// Function attributes and cluster size of the chain-resident kernel (once per batch,
// outside any stream capture).
int32_t prepare_cluster(scemc_ensemble* E) {
  if (E->cluster_cs > 0) return SCEMC_OK;
  int32_t max_ns = 1;
  for (const scemc_tables* T : E->tabs) max_ns = std::max(max_ns, T->n_sites);
  const size_t smem = cluster_smem_bytes(max_ns, std::max(E->dmax, 1), std::max(E->rmax, 1), fast_rows(E->lmax));
  const void* fn = E->lmax == 1 ? (const void*)k_chain_cluster<1> : (const void*)k_chain_cluster<2>;
  CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  const int cs = cluster_size(E, smem);
  if (cs < 1) return fail(SCEMC_ERR_CUDA, "no thread-block cluster of the chain-resident kernel fits the device");
  E->cluster_cs = cs;
  E->cluster_smem = smem;
  return SCEMC_OK;
}

int32_t run_cluster_sweep(scemc_ensemble* E, int n_or, const Launch& Lc) {
  SweepArgs a = make_args(E, -1);
  a.dmax = std::max(E->dmax, 1);
  a.rmax = std::max(E->rmax, 1);
  a.item_base = E->d_item_base;
  int32_t rc;
  if (Lc.precompute) {
    if ((rc = ensure_props(E))) return rc;
    a.prop = E->d_prop;
    a.propu = E->d_propu;
  }
  if ((rc = prepare_cluster(E))) return rc;
  const int cs = E->cluster_cs;
  const size_t smem = E->cluster_smem;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (E->profiling) {
    ev0 = take_event(E);
    ev1 = take_event(E);
    CUDA_TRY(cudaEventRecord(ev0, E->stream));
  }
  if (a.prop) {
    const int blocks = (int)std::min<int64_t>(sm_count(E->device) * 16, ((int64_t)E->item_base.back() + 255) / 256);
    ++E->launches;
    k_proposals<<<std::max(blocks, 1), 256, 0, E->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(cs * E->n_slots));
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = E->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ++E->launches;
  if (E->lmax == 1) CUDA_TRY(cudaLaunchKernelEx(&cfg, k_chain_cluster<1>, a, n_or));
  else CUDA_TRY(cudaLaunchKernelEx(&cfg, k_chain_cluster<2>, a, n_or));
  if (E->profiling) {
    CUDA_TRY(cudaEventRecord(ev1, E->stream));
    E->ev_pending.emplace_back(ev0, ev1);
    E->graph_passes_per_launch = 1 + n_or;
  }
  return SCEMC_OK;
}

int auto_lanes(const scemc_ensemble* E) {
  // Items per colour vs. ~16 resident warps per SM: give each item more lanes when
  // a colour class alone cannot fill the device.
  int64_t items = 0;
  for (int c = 0; c < E->max_colors; ++c)
    items = std::max<int64_t>(items, E->seg[(size_t)c * (E->tabs.size() + 1) + E->tabs.size()]);
  const int64_t target = (int64_t)sm_count(E->device) * 1024;
  int G = 1;
  while (G < 32 && items * G < target) G <<= 1;
  return G;
}

// kernel: 0 auto, 1 generic, 2 row-parallel fast, 3 replica-parallel, 4 chain-resident
// cluster, 5 replica-parallel with the pair records on the tensor cores; proposals: 0 auto,
// 1 precompute, 2 inline.
int32_t resolve_launch(const scemc_ensemble* E, int lanes, int mode, int kernel, int proposals, Launch* out,
                       int rep_replicas = 0, int rep_np = 0, int rep_pf = 0) {
  Launch L;
  if (rep_replicas < 0 || rep_replicas > 2) return fail(SCEMC_ERR_ARG, "rep_replicas must be 0, 1 or 2");
  if (rep_np < 0 || rep_np > 2) return fail(SCEMC_ERR_ARG, "rep_threads_per_item must be 0, 1 or 2");
  if (rep_pf < 0 || rep_pf > 2) return fail(SCEMC_ERR_ARG, "rep_prefetch must be 0, 1 or 2");
  L.rep_p = rep_replicas;
  L.rep_np = rep_np;
  L.rep_pf = rep_pf;
  if (mode == 0 && kernel == 0 && E->tuned) {
    mode = E->tuned_mode;
    kernel = E->tuned_kernel;
    if (proposals == 0) proposals = E->tuned_proposals;
    if (lanes == 0) lanes = E->tuned_lanes;
    if (proposals == 3 && (mode == 2 || mode == 4)) mode = 3;  // learned passes run per colour
    if (proposals == 3 && (kernel == 4 || kernel == 5)) kernel = 3;  // with the replica-parallel decision
  }
  if (mode < 0 || mode > 4) return fail(SCEMC_ERR_ARG, "mode must be 0..4");
  if (mode == 4 && (!E->fast || kernel == 1 || kernel == 3 || kernel == 5 || proposals == 3))
    return fail(SCEMC_ERR_ARG, "the data-flow form (mode 4) runs the row-parallel kernel with plain proposals");
  if (kernel < 0 || kernel > 5 || proposals < 0 || proposals > 3)
    return fail(SCEMC_ERR_ARG, "kernel must be 0..5 and proposals 0..3");
  if (kernel == 5) {
    if (!E->fast || E->lmax != 2)
      return fail(SCEMC_ERR_ARG, "the tensor-core replica pass (kernel 5) needs the fast tables of lmax 2");
    if (proposals == 3) return fail(SCEMC_ERR_ARG, "the tensor-core replica pass (kernel 5) runs plain proposals");
    if (mode == 2 || mode == 4) return fail(SCEMC_ERR_ARG, "the tensor-core replica pass (kernel 5) runs with mode 1 or 3");
  }
  if (kernel == 4) {
    int32_t rc;
    if ((rc = cluster_fits(E))) return rc;
    if (proposals == 3) return fail(SCEMC_ERR_ARG, "the cluster kernel (kernel 4) runs plain Metropolis proposals");
    if (mode == 2 || mode == 4) return fail(SCEMC_ERR_ARG, "the cluster kernel (kernel 4) runs with mode 1 or 3");
  }
  if (proposals == 3) {
    if (!E->mlp) return fail(SCEMC_ERR_ARG, "learned proposals need scemc_batch_set_learned first");
    if (!E->fast) return fail(SCEMC_ERR_ARG, "learned proposals need the fast tables (lmax 1 or 2 dense programs)");
    if (kernel == 1) return fail(SCEMC_ERR_ARG, "learned proposals run with kernel 2 or 3, not the generic walk");
    if (E->learned_field && kernel != 3 && kernel != 0)
      return fail(SCEMC_ERR_ARG, "a field-input learned proposal runs with kernel 3 (the fused decision)");
    if (mode == 2) return fail(SCEMC_ERR_ARG, "learned proposals run per-colour launches (mode 1 or 3)");
  }
  bool generic_ok = true;
  for (const scemc_tables* T : E->tabs) generic_ok = generic_ok && T->has_generic;
  if ((kernel == 2 || kernel == 3) && !E->fast)
    return fail(SCEMC_ERR_ARG, "the fast and replica-parallel kernels need lmax 1 or 2 and dense l in {1,2} "
                               "programs of body <= 4 (l = 1 only for body 4; l in {1, 2} for body 3 when lmax = 2), equal lmax across the batch");
  if (kernel == 1 && !generic_ok) return fail(SCEMC_ERR_ARG, "generic records were not kept for these tables");
  // untuned auto choice: threads that carry replicas once every site has at least 16
  // of them and a colour holds enough items to fill the SMs (256 per SM)
  int min_r = 1 << 30;
  for (int r : E->R) min_r = std::min(min_r, r);
  const bool rep_auto = E->fast && mode != 2 && min_r >= 16 &&
                        (int64_t)max_colour_items(E) >= (int64_t)sm_count(E->device) * 256;
  L.cluster = kernel == 4;
  L.rep = kernel == 3 || kernel == 5 || (kernel == 0 && (rep_auto || (proposals == 3 && E->learned_field)));
  L.rep_tc = kernel == 5;
  L.fast = !L.rep && (kernel == 2 || kernel == 4 || (kernel == 0 && E->fast));
  L.learned = proposals == 3;
  L.mode = mode == 0 ? ((L.rep || L.learned || L.cluster) ? 1 : 2) : mode;
  if (L.mode == 3) {
    L.graph = true;
    L.mode = 1;
  }
  if (L.mode == 4) {
    L.flow = true;
    L.mode = 2;
    L.rep = false;
    L.fast = true;
  }
  L.G = lanes ? norm_lanes(lanes) : auto_lanes(E);
  if (L.learned) {
    L.precompute = false;
  } else if (L.cluster) {  // precomputed by default: the keyed draw's FP64 trigonometry stays off the colour steps
    L.precompute = proposals != 2;
  } else if (L.fast) {
    const int64_t groups = (int64_t)max_colour_items(E) * 32;
    L.precompute = proposals == 1 || (proposals == 0 && groups < (int64_t)sm_count(E->device) * 2048);
  } else if (L.rep) {
    L.precompute = proposals == 1;
  }
  *out = L;
  return SCEMC_OK;
}

int32_t sweep_once(scemc_ensemble* E, int n_or, const Launch& L) {
  if (E->sweep_index >= 0x7ffffffell - 1)
    return fail(SCEMC_ERR_EXHAUSTED, "sweep_index exhausted the 32-bit RNG counter word");
  int32_t rc;
  if (L.cluster) return run_cluster_sweep(E, n_or, L);
  if ((rc = run_pass(E, -1, L))) return rc;
  for (int k = 0; k < n_or; ++k)
    if ((rc = run_pass(E, k, L))) return rc;
  return SCEMC_OK;
}

// The passes and tail of one compound sweep as a CUDA graph (captured once per
// configuration, replayed every sweep). Every launch reads the sweep counter from
// device memory and the tail advances it, so one capture serves all sweeps.
int32_t sweep_graph(scemc_ensemble* E, int n_or, const Launch& L, cudaGraphExec_t* out, int64_t* n_launch) {
  const int key[7] = {n_or, L.cluster ? 3 : (L.rep ? (L.rep_tc ? 4 : 2) : (L.fast ? 1 : 0)), L.learned ? 2 : (L.precompute ? 1 : 0),
                      L.fast ? 0 : (L.rep ? L.rep_p : L.G), E->recording ? 1 : 0, L.rep ? L.rep_np : 0,
                      L.rep ? L.rep_pf : 0};
  for (auto& g : E->graphs)
    if (std::equal(key, key + 7, g.key)) {
      *out = g.exec;
      *n_launch = g.launches;
      return SCEMC_OK;
    }
  int32_t rc;
  if ((L.fast || L.rep) && L.precompute)
    if ((rc = ensure_props(E))) return rc;
  if (L.learned)
    if ((rc = prepare_learned(E))) return rc;
  if (L.cluster)  // attributes and the cluster size are settled outside the capture
    if ((rc = prepare_cluster(E))) return rc;
  if (L.fast) {  // attributes are set outside the capture
    int threads;
    size_t smem;
    fast_shape(E, &threads, &smem);
    CUDA_TRY(cudaFuncSetAttribute((const void*)fast_kernel(E->lmax, false),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  if (L.rep) {
    for (int c = 0; c < E->max_colors; ++c) {
      const RepForm f = rep_form(E, c, L.rep_p, L.rep_np, L.rep_pf, L.rep_tc);
      CUDA_TRY(cudaFuncSetAttribute((const void*)f.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.smem));
    }
  }
  const bool prof = E->profiling;
  E->profiling = false;  // graph launches are timed as a whole
  const int64_t launches0 = E->launches;
  CUDA_TRY(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
  rc = sweep_once(E, n_or, L);
  if (!rc) rc = launch_tail(E, true, false, 0.5, false, true);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(E->stream, &graph);
  E->profiling = prof;
  const int64_t captured = E->launches - launches0;
  E->launches = launches0;  // captured, not yet run
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return fail(SCEMC_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return fail(SCEMC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
  scemc_ensemble::GraphEntry g;
  std::copy(key, key + 7, g.key);
  g.exec = exec;
  g.launches = captured;
  E->graphs.push_back(g);
  *out = exec;
  *n_launch = captured;
  return SCEMC_OK;
}

}  // namespace

// =============================================================================
// C ABI
// =============================================================================
namespace scemc_detail {
int32_t set_error(int32_t code, const char* msg) { return fail(code, msg); }
}  // namespace scemc_detail

extern "C" {

int32_t scemc_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return SCEMC_ERR_ARG;
  std::snprintf(buf, len, "%s", t_err.c_str());
  return SCEMC_OK;
}

int32_t scemc_version(void) { return 100; }

int32_t scemc_tables_create(const scemc_tables_desc* desc, scemc_tables** out) {
  if (!out) return fail(SCEMC_ERR_ARG, "out is NULL");
  *out = nullptr;
  auto* T = new scemc_tables();
  cudaGetDevice(&T->device);
  const int32_t rc = compile_tables(desc, T);
  if (rc != SCEMC_OK) {
    delete T;
    return rc;
  }
  *out = T;
  return SCEMC_OK;
}

int32_t scemc_tables_destroy(scemc_tables* t) {
  delete t;
  return SCEMC_OK;
}

int32_t scemc_tables_stats(const scemc_tables* t, double* d_mean, double* a_mean, int64_t* bytes) {
  if (!t) return fail(SCEMC_ERR_ARG, "tables is NULL");
  if (d_mean) *d_mean = t->d_mean;
  if (a_mean) *a_mean = t->a_mean;
  if (bytes) *bytes = t->bytes;
  return SCEMC_OK;
}

int32_t scemc_tables_records(const scemc_tables* t, double* records_mean) {
  if (!t || !records_mean) return fail(SCEMC_ERR_ARG, "NULL argument");
  *records_mean = t->n_active ? (double)t->fast_records / t->n_active : 0.0;
  return SCEMC_OK;
}

int32_t scemc_chain_create(const scemc_tables* t, const double* config, double energy, uint64_t seed, double step,
                           scemc_chain** out) {
  const int32_t one = 1;
  return create_ensemble(1, &t, &one, config, &energy, &seed, &step, out);
}

int32_t scemc_chain_destroy(scemc_chain* c) {
  delete c;
  return SCEMC_OK;
}

int32_t scemc_batch_create(int32_t n_tables, const scemc_tables* const* tables, const int32_t* replicas,
                           const double* configs, const double* energies, const uint64_t* seeds, const double* steps,
                           scemc_batch** out) {
  return create_ensemble(n_tables, tables, replicas, configs, energies, seeds, steps, out);
}

int32_t scemc_batch_destroy(scemc_batch* b) {
  delete b;
  return SCEMC_OK;
}

int32_t scemc_batch_size(const scemc_batch* b, int32_t* n_slots, int64_t* n_sites_total) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  if (n_slots) *n_slots = b->n_slots;
  if (n_sites_total) *n_sites_total = b->n_spins;
  return SCEMC_OK;
}

static int32_t check_single(const scemc_ensemble* c, const scemc_tables* t) {
  if (!c) return fail(SCEMC_ERR_ARG, "chain is NULL");
  if (c->n_slots != 1 || c->tabs.size() != 1) return fail(SCEMC_ERR_ARG, "expected a single-replica chain");
  if (t && c->tabs[0] != t) return fail(SCEMC_ERR_ARG, "chain was created on other tables");
  return SCEMC_OK;
}

static int32_t check_lanes(int32_t lanes) {
  if (lanes < 1 || (lanes & (lanes - 1)) != 0)
    return fail(SCEMC_ERR_ARG, "lanes_per_site must be a power of two (got " + std::to_string(lanes) + ")");
  return SCEMC_OK;
}

int32_t scemc_metropolis_sweep(scemc_chain* c, const scemc_tables* t, double beta, int32_t lanes_per_site,
                               int64_t* n_accepted) {
  int32_t rc;
  if ((rc = check_single(c, t)) || (rc = check_lanes(lanes_per_site))) return rc;
  if (!std::isfinite(beta)) return fail(SCEMC_ERR_ARG, "beta must be finite");
  CUDA_TRY(cudaMemcpyAsync(c->d_beta, &beta, 8, cudaMemcpyHostToDevice, c->stream));
  unsigned long long before = 0;
  CUDA_TRY(cudaMemcpyAsync(&before, c->d_cnt, 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  Launch L;
  if ((rc = resolve_launch(c, lanes_per_site, 1, 0, 0, &L))) return rc;
  if ((rc = sweep_once(c, 0, L))) return rc;
  if ((rc = launch_tail(c, true, false, 0.5, false, true))) return rc;
  unsigned long long after = 0;
  CUDA_TRY(cudaMemcpyAsync(&after, c->d_cnt, 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->sweep_index += 1;
  if (n_accepted) *n_accepted = (int64_t)(after - before);
  return SCEMC_OK;
}

int32_t scemc_overrelaxation_sweep(scemc_chain* c, const scemc_tables* t, double beta, int32_t lanes_per_site,
                                   int64_t* n_accepted, int64_t* n_attempted) {
  int32_t rc;
  if ((rc = check_single(c, t)) || (rc = check_lanes(lanes_per_site))) return rc;
  if (!std::isfinite(beta)) return fail(SCEMC_ERR_ARG, "beta must be finite");
  if (c->sweep_index >= 0x7ffffffell - 1)
    return fail(SCEMC_ERR_EXHAUSTED, "sweep_index exhausted the 32-bit RNG counter word");
  CUDA_TRY(cudaMemcpyAsync(c->d_beta, &beta, 8, cudaMemcpyHostToDevice, c->stream));
  unsigned long long before[4], after[4];
  CUDA_TRY(cudaMemcpyAsync(before, c->d_cnt, 32, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  // a stand-alone OR sweep uses pass 0 of the next sweep counter word
  Launch L;
  if ((rc = resolve_launch(c, lanes_per_site, 1, 0, 0, &L))) return rc;
  if ((rc = run_pass(c, 0, L))) return rc;
  if ((rc = launch_tail(c, false, false, 0.5, false, true))) return rc;
  CUDA_TRY(cudaMemcpyAsync(after, c->d_cnt, 32, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->sweep_index += 1;
  if (n_accepted) *n_accepted = (int64_t)(after[2] - before[2]);
  if (n_attempted) *n_attempted = (int64_t)(after[3] - before[3]);
  return SCEMC_OK;
}

int32_t scemc_run_sweeps(scemc_chain* c, const scemc_tables* t, double beta, int64_t nsweeps, int64_t renorm_interval,
                         int32_t lanes_per_site) {
  int32_t rc;
  if ((rc = check_single(c, t)) || (rc = check_lanes(lanes_per_site))) return rc;
  if (!std::isfinite(beta) || nsweeps < 0) return fail(SCEMC_ERR_ARG, "bad beta or nsweeps");
  CUDA_TRY(cudaMemcpyAsync(c->d_beta, &beta, 8, cudaMemcpyHostToDevice, c->stream));
  Launch L;
  if ((rc = resolve_launch(c, lanes_per_site, 1, 0, 0, &L))) return rc;
  for (int64_t i = 1; i <= nsweeps; ++i) {
    if ((rc = sweep_once(c, 0, L))) return rc;
    if ((rc = launch_tail(c, true, false, 0.5, false, true))) return rc;
    c->sweep_index += 1;
    if (renorm_interval > 0 && i % renorm_interval == 0)
      if ((rc = recompute(c, 1))) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_error(c);
}

int32_t scemc_download(const scemc_chain* c, double* config, double* energy, int64_t* sweep_index,
                       int64_t* counters) {
  int32_t rc;
  if ((rc = check_single(c, nullptr))) return rc;
  DownloadDst d;
  d.configs = config;
  d.energies = energy;
  d.counters = counters;
  if ((rc = payload_download(c, d))) return rc;
  if (sweep_index) *sweep_index = c->sweep_index;
  return SCEMC_OK;
}

int32_t scemc_upload(scemc_chain* c, const double* config, double energy) {
  int32_t rc;
  if ((rc = check_single(c, nullptr))) return rc;
  if (!config || !std::isfinite(energy)) return fail(SCEMC_ERR_ARG, "config NULL or energy not finite");
  return payload_upload(c, config, &energy);
}

int32_t scemc_set_step(scemc_chain* c, double step) {
  int32_t rc;
  if ((rc = check_single(c, nullptr))) return rc;
  if (!(step > 0) || !std::isfinite(step)) return fail(SCEMC_ERR_ARG, "step must be > 0");
  CUDA_TRY(h2d_sync(c->d_step, &step, 8));
  return SCEMC_OK;
}

int32_t scemc_swap_payload(scemc_chain* a, scemc_chain* b) {
  int32_t rc;
  if ((rc = check_single(a, nullptr)) || (rc = check_single(b, nullptr))) return rc;
  if (a->tabs[0] != b->tabs[0]) return fail(SCEMC_ERR_ARG, "chains live on different tables");
  if (a == b) return SCEMC_OK;
  CUDA_TRY(cudaStreamSynchronize(a->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  std::swap(a->d_spins, b->d_spins);
  double ea, eb;
  CUDA_TRY(cudaMemcpy(&ea, a->d_energy, 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(&eb, b->d_energy, 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(h2d_sync(a->d_energy, &eb, 8));
  CUDA_TRY(h2d_sync(b->d_energy, &ea, 8));
  return SCEMC_OK;
}

int32_t scemc_total_energy(const scemc_ensemble* e, int32_t replica, double* energy) {
  if (!e || !energy) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (replica < 0 || replica >= e->n_slots) return fail(SCEMC_ERR_ARG, "replica out of range");
  auto* E = const_cast<scemc_ensemble*>(e);
  int32_t rc;
  if ((rc = recompute(E, 0))) return rc;
  CUDA_TRY(cudaMemcpyAsync(energy, E->d_eout + replica, 8, cudaMemcpyDeviceToHost, E->stream));
  CUDA_TRY(cudaStreamSynchronize(E->stream));
  return SCEMC_OK;
}

int32_t scemc_renormalize(scemc_ensemble* e, double* drift) {
  if (!e) return fail(SCEMC_ERR_ARG, "NULL argument");
  int32_t rc;
  if ((rc = recompute(e, 1))) return rc;
  if (drift) CUDA_TRY(cudaMemcpyAsync(drift, e->d_drift, 8 * e->n_slots, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return SCEMC_OK;
}

int32_t scemc_batch_set_betas(scemc_batch* b, const double* betas) {
  if (!b || !betas) return fail(SCEMC_ERR_ARG, "NULL argument");
  for (int i = 0; i < b->n_slots; ++i)
    if (!std::isfinite(betas[i])) return fail(SCEMC_ERR_ARG, "beta must be finite");
  CUDA_TRY(h2d_sync(b->d_beta, betas, 8 * b->n_slots));
  return SCEMC_OK;
}

int32_t scemc_batch_set_steps(scemc_batch* b, const double* steps) {
  if (!b || !steps) return fail(SCEMC_ERR_ARG, "NULL argument");
  for (int i = 0; i < b->n_slots; ++i)
    if (!(steps[i] > 0)) return fail(SCEMC_ERR_ARG, "step must be > 0");
  CUDA_TRY(h2d_sync(b->d_step, steps, 8 * b->n_slots));
  return SCEMC_OK;
}

int32_t scemc_batch_run_async(scemc_batch* b, const scemc_run_params* p) {
  if (!b || !p) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (p->nsweeps < 0 || p->or_per_metropolis < 0 || (p->exchange && p->exchange_interval < 1))
    return fail(SCEMC_ERR_ARG, "bad run parameters");
  if (p->lanes_per_site != 0) {
    int32_t rc = check_lanes(p->lanes_per_site);
    if (rc) return rc;
  }
  if (p->phase_done < 0 || p->phase_total < 0) return fail(SCEMC_ERR_ARG, "bad phase bookkeeping");
  if (p->mode < 0 || p->mode > 4) return fail(SCEMC_ERR_ARG, "mode must be 0..4");
  const int64_t total = p->phase_total > 0 ? p->phase_total : p->phase_done + p->nsweeps;
  int32_t rc;
  Launch L;
  if ((rc = resolve_launch(b, p->lanes_per_site, p->mode, p->kernel, p->proposals, &L, p->rep_replicas, p->rep_threads_per_item,
                           p->rep_prefetch)))
    return rc;
  if (b->sweep_index + p->nsweeps >= 0x7ffffffell - 1)
    return fail(SCEMC_ERR_EXHAUSTED, "sweep_index would exhaust the 32-bit RNG counter word");
  cudaGraphExec_t exec = nullptr;
  int64_t graph_launches = 0;
  if (L.graph) {
    if ((rc = sweep_graph(b, p->or_per_metropolis, L, &exec, &graph_launches))) return rc;
  }
  for (int64_t k = 1; k <= p->nsweeps; ++k) {
    const int64_t i = p->phase_done + k;
    const bool adapt = p->adapt_interval > 0 && i % p->adapt_interval == 0;
    if (exec) {
      // passes + tail (fold, att, sweep counter) replayed as one graph
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (b->profiling) {
        e0 = take_event(b);
        e1 = take_event(b);
        CUDA_TRY(cudaEventRecord(e0, b->stream));
      }
      CUDA_TRY(cudaGraphLaunch(exec, b->stream));
      b->launches += graph_launches;
      if (b->profiling) {
        CUDA_TRY(cudaEventRecord(e1, b->stream));
        b->ev_pending.emplace_back(e0, e1);
        b->graph_passes_per_launch = 1 + p->or_per_metropolis;
      }
      if (adapt)
        if ((rc = launch_tail(b, false, true, p->adapt_target, false, false))) return rc;
    } else {
      if ((rc = sweep_once(b, p->or_per_metropolis, L))) return rc;
      if ((rc = launch_tail(b, true, adapt, p->adapt_target, false, true))) return rc;
    }
    b->sweep_index += 1;
    if (p->renorm_interval > 0 && i % p->renorm_interval == 0)
      if ((rc = recompute(b, 1))) return rc;
    if (p->measure_interval > 0 && i % p->measure_interval == 0)
      if ((rc = measure(b))) return rc;
    if (p->exchange && i % p->exchange_interval == 0 && i < total)
      if ((rc = launch_tail(b, false, false, 0.5, true, false))) return rc;
  }
  return SCEMC_OK;
}

int32_t scemc_batch_autotune(scemc_batch* b, int32_t or_per_metropolis, int32_t sweeps_per_trial, int32_t* mode,
                             int32_t* proposals, int32_t* lanes, int32_t* kernel, double* ms_per_sweep) {
  if (!b || or_per_metropolis < 0 || sweeps_per_trial < 1) return fail(SCEMC_ERR_ARG, "bad autotune arguments");
  struct Cand {
    int mode, proposals, lanes, kernel;
  };
  std::vector<Cand> cands;
  if (b->fast) {
    for (int m : {2, 3})
      for (int q : {1, 2}) cands.push_back({m, q, 0, 2});
    cands.push_back({4, 2, 0, 2});
    for (int q : {1, 2}) cands.push_back({3, q, 0, 3});
    for (int q : {1, 2}) cands.push_back({2, q, 0, 3});
    if (b->lmax == 2)
      for (int q : {1, 2}) cands.push_back({3, q, 0, 5});
    if (cluster_fits(b) == SCEMC_OK)
      for (int q : {1, 2}) cands.push_back({3, q, 0, 4});
  } else {
    for (int m : {2, 3})
      for (int g : {1, 4, 8, 32}) cands.push_back({m, 0, g, 1});
  }
  const bool prof = b->profiling;
  b->profiling = false;
  b->tuned = false;
  double best = 1e300;
  Cand bc = cands[0];
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int32_t rc = SCEMC_OK;
  for (const Cand& c : cands) {
    scemc_run_params p{};
    p.nsweeps = 1;
    p.or_per_metropolis = or_per_metropolis;
    p.mode = c.mode;
    p.proposals = c.proposals;
    p.lanes_per_site = c.lanes;
    p.kernel = c.kernel;
    if ((rc = scemc_batch_run(b, &p))) break;  // warm-up (builds graphs, sets attributes)
    p.nsweeps = sweeps_per_trial;
    cudaEventRecord(e0, b->stream);
    if ((rc = scemc_batch_run_async(b, &p))) break;
    cudaEventRecord(e1, b->stream);
    if ((rc = scemc_batch_sync(b))) break;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per = ms / sweeps_per_trial;
    if (per < best) {
      best = per;
      bc = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->profiling = prof;
  if (rc) return rc;
  b->tuned = true;
  b->tuned_mode = bc.mode;
  b->tuned_proposals = bc.proposals;
  b->tuned_lanes = bc.lanes;
  b->tuned_kernel = bc.kernel;
  if (mode) *mode = bc.mode;
  if (kernel) *kernel = bc.kernel;
  if (proposals) *proposals = bc.proposals;
  if (lanes) *lanes = bc.lanes;
  if (ms_per_sweep) *ms_per_sweep = best;
  return SCEMC_OK;
}

int32_t scemc_batch_sync(scemc_batch* b) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  harvest_events(b);
  return check_error(b);
}

int32_t scemc_batch_run(scemc_batch* b, const scemc_run_params* p) {
  const int32_t rc = scemc_batch_run_async(b, p);
  if (rc != SCEMC_OK) {
    if (b) cudaStreamSynchronize(b->stream);
    return rc;
  }
  return scemc_batch_sync(b);
}

int32_t scemc_batch_stream(const scemc_batch* b, void** stream) {
  if (!b || !stream) return fail(SCEMC_ERR_ARG, "NULL argument");
  *stream = (void*)b->stream;
  return SCEMC_OK;
}

int32_t scemc_host_register(void* ptr, int64_t bytes) {
  if (!ptr || bytes <= 0) return fail(SCEMC_ERR_ARG, "scemc_host_register: NULL pointer or non-positive size");
  CUDA_TRY(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
  return SCEMC_OK;
}

int32_t scemc_host_unregister(void* ptr) {
  if (!ptr) return fail(SCEMC_ERR_ARG, "scemc_host_unregister: NULL pointer");
  CUDA_TRY(cudaHostUnregister(ptr));
  return SCEMC_OK;
}

int32_t scemc_batch_upload(scemc_batch* b, const double* configs, const double* energies) {
  if (!b || !configs) return fail(SCEMC_ERR_ARG, "NULL argument");
  return payload_upload(b, configs, energies);
}

int32_t scemc_batch_profile(scemc_batch* b, int32_t on) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  b->profiling = on != 0;
  b->prof_ms = 0.0;
  b->prof_passes = 0;
  return SCEMC_OK;
}

int32_t scemc_batch_kernel_time(const scemc_batch* b, double* ms, int64_t* passes) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  if (ms) *ms = b->prof_ms;
  if (passes) *passes = b->prof_passes;
  return SCEMC_OK;
}

int32_t scemc_batch_launches(const scemc_batch* b, int64_t* launches) {
  if (!b || !launches) return fail(SCEMC_ERR_ARG, "NULL argument");
  *launches = b->launches;
  return SCEMC_OK;
}



int32_t scemc_batch_download(const scemc_batch* b, double* configs, double* energies, int32_t* slot_of_rung,
                             int64_t* counters, int64_t* swaps, double* steps, double* max_drift) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  DownloadDst d;
  d.configs = configs;
  d.energies = energies;
  d.slot_of_rung = slot_of_rung;
  d.counters = counters;
  d.swaps = swaps;
  d.steps = steps;
  d.max_drift = max_drift;
  return payload_download(b, d);
}

namespace {
// Saved-state blob: a header, then the device arrays in a fixed order, each padded to
// 8 bytes.
constexpr char kStateMagic[8] = {'S', 'C', 'E', 'M', 'C', 'S', 'T', '1'};
struct StateHeader {
  char magic[8];
  int32_t version, n_tables, n_slots, pad;
  int64_t n_spins, sweep_index;
  uint64_t exchange_seed;
};
struct StatePart {
  void* dev;
  size_t bytes;
};
std::vector<StatePart> state_parts(const scemc_ensemble* E) {
  const size_t n = (size_t)E->n_slots;
  return {{E->d_spins, sizeof(float4) * (size_t)E->n_spins}, {E->d_energy, 8 * n}, {E->d_dEfix, 8 * n},
          {E->d_cnt, 32 * n}, {E->d_win, 16 * n}, {E->d_swaps, 16 * n}, {E->d_beta, 8 * n}, {E->d_step, 8 * n},
          {E->d_seed, 8 * n}, {E->d_slot_of_rung, 4 * n}, {E->d_rung_of_slot, 4 * n}, {E->d_max_drift, 8 * n},
          {E->d_drift, 8 * n}, {E->d_st, sizeof(EnsState)}};
}
size_t state_bytes(const scemc_ensemble* E) {
  size_t b = sizeof(StateHeader) + 8 * E->tabs.size();
  for (const StatePart& p : state_parts(E)) b += (p.bytes + 7) & ~(size_t)7;
  return b;
}
}  // namespace

int32_t scemc_batch_state_bytes(const scemc_batch* b, int64_t* bytes) {
  if (!b || !bytes) return fail(SCEMC_ERR_ARG, "NULL argument");
  *bytes = (int64_t)state_bytes(b);
  return SCEMC_OK;
}

int32_t scemc_batch_save_state(scemc_batch* b, void* buf, int64_t bytes) {
  if (!b || !buf) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (bytes < (int64_t)state_bytes(b)) return fail(SCEMC_ERR_ARG, "state buffer too small");
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  auto* p = static_cast<unsigned char*>(buf);
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.version = 1;
  h.n_tables = (int32_t)b->tabs.size();
  h.n_slots = b->n_slots;
  h.n_spins = b->n_spins;
  h.sweep_index = b->sweep_index;
  h.exchange_seed = b->exchange_seed;
  std::memcpy(p, &h, sizeof h);
  p += sizeof h;
  for (size_t i = 0; i < b->tabs.size(); ++i) {
    const int32_t shape[2] = {b->tabs[i]->n_sites, b->R[i]};
    std::memcpy(p, shape, 8);
    p += 8;
  }
  for (const StatePart& part : state_parts(b)) {
    CUDA_TRY(cudaMemcpyAsync(p, part.dev, part.bytes, cudaMemcpyDeviceToHost, b->stream));
    p += (part.bytes + 7) & ~(size_t)7;
  }
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SCEMC_OK;
}

int32_t scemc_batch_load_state(scemc_batch* b, const void* buf, int64_t bytes) {
  if (!b || !buf) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (bytes < (int64_t)(sizeof(StateHeader) + 8 * b->tabs.size()))
    return fail(SCEMC_ERR_ARG, "state blob truncated");
  const auto* p = static_cast<const unsigned char*>(buf);
  StateHeader h;
  std::memcpy(&h, p, sizeof h);
  if (std::memcmp(h.magic, kStateMagic, 8) != 0 || h.version != 1)
    return fail(SCEMC_ERR_ARG, "not a batch state blob (magic or version)");
  if (h.n_tables != (int32_t)b->tabs.size() || h.n_slots != b->n_slots || h.n_spins != b->n_spins)
    return fail(SCEMC_ERR_ARG, "state blob was saved from a batch of another shape");
  p += sizeof h;
  for (size_t i = 0; i < b->tabs.size(); ++i) {
    int32_t shape[2];
    std::memcpy(shape, p, 8);
    if (shape[0] != b->tabs[i]->n_sites || shape[1] != b->R[i])
      return fail(SCEMC_ERR_ARG, "state blob table " + std::to_string(i + 1) + " has another size or replica count");
    p += 8;
  }
  if (bytes < (int64_t)state_bytes(b)) return fail(SCEMC_ERR_ARG, "state blob truncated");
  if (h.sweep_index < 0 || h.sweep_index >= 0x7ffffffell) return fail(SCEMC_ERR_ARG, "state blob sweep index");
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (const StatePart& part : state_parts(b)) {
    CUDA_TRY(cudaMemcpyAsync(part.dev, p, part.bytes, cudaMemcpyHostToDevice, b->stream));
    p += (part.bytes + 7) & ~(size_t)7;
  }
  if (b->d_flags)  // data-flow epochs restart from the loaded sweep
    CUDA_TRY(cudaMemsetAsync(b->d_flags, 0, sizeof(uint32_t) * std::max<int64_t>(b->n_spins, 1), b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  b->sweep_index = h.sweep_index;
  b->exchange_seed = h.exchange_seed;
  b->meas_n = 0;
  return SCEMC_OK;
}

int32_t scemc_batch_reset_counters(scemc_batch* b) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  const int n = b->n_slots;
  CUDA_TRY(cudaMemsetAsync(b->d_cnt, 0, 32 * n, b->stream));
  CUDA_TRY(cudaMemsetAsync(b->d_win, 0, 16 * n, b->stream));
  CUDA_TRY(cudaMemsetAsync(b->d_swaps, 0, 16 * n, b->stream));
  CUDA_TRY(cudaMemsetAsync(b->d_max_drift, 0, 8 * n, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return SCEMC_OK;
}

int32_t scemc_batch_fetch_measurements(scemc_batch* b, double* rec, int64_t capacity, int64_t* n_records,
                                       int32_t* record_len) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  if (record_len) *record_len = b->rec_len;
  if (n_records) *n_records = b->meas_n;
  if (!rec) return SCEMC_OK;
  if (capacity < b->meas_n) return fail(SCEMC_ERR_ARG, "capacity smaller than the number of records");
  if (b->meas_n > 0)
    CUDA_TRY(cudaMemcpy(rec, b->d_meas, sizeof(double) * b->meas_n * b->n_slots * b->rec_len, cudaMemcpyDeviceToHost));
  b->meas_n = 0;
  return SCEMC_OK;
}

int32_t scemc_batch_record(scemc_batch* b, int32_t on) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  b->recording = on != 0;
  for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
  b->graphs.clear();
  int32_t cap = 0;
  for (const scemc_tables* T : b->tabs) cap = std::max(cap, T->n_sites);
  const size_t n = (size_t)cap * kRecPasses;
  if (b->recording && !b->d_rprop) {
    int32_t rc;
    if ((rc = dalloc(&b->d_rprop, 3 * n)) || (rc = dalloc(&b->d_ru, n)) || (rc = dalloc(&b->d_rdE, n)) ||
        (rc = dalloc(&b->d_racc, n)) || (rc = dalloc(&b->d_rlqr, (size_t)cap)))
      return rc;
    b->rec_cap = cap;
  }
  // cleared on the batch's own (non-blocking) stream and waited for: a clear on the
  // legacy stream is not ordered before the batch's next kernels, which may then record
  // first and be overwritten
  if (b->recording) {
    CUDA_TRY(cudaMemsetAsync(b->d_rlqr, 0, sizeof(double) * cap, b->stream));
    CUDA_TRY(cudaMemsetAsync(b->d_racc, 3, n, b->stream));  // 3 = site not visited
    CUDA_TRY(cudaStreamSynchronize(b->stream));
  }
  return SCEMC_OK;
}

int32_t scemc_batch_record_slot(scemc_batch* b, int32_t table, int32_t replica) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  if (table < 0 || table >= (int32_t)b->tabs.size()) return fail(SCEMC_ERR_ARG, "record table out of range");
  if (replica < 0 || replica >= b->R[table]) return fail(SCEMC_ERR_ARG, "record replica out of range");
  b->rec_li = table;
  b->rec_r = replica;
  for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);  // captured launches carry the old slot
  b->graphs.clear();
  return SCEMC_OK;
}

int32_t scemc_batch_fetch_record(const scemc_batch* b, int32_t pass, float* prop, double* u, float* dE,
                                 uint8_t* acc) {
  if (!b || !b->d_rprop) return fail(SCEMC_ERR_ARG, "recording was never enabled");
  if (pass < -1 || pass + 1 >= kRecPasses) return fail(SCEMC_ERR_ARG, "pass outside -1..2");
  const size_t n = (size_t)b->tabs[b->rec_li]->n_sites, o = (size_t)(pass + 1) * (size_t)b->rec_cap;
  if (prop) CUDA_TRY(cudaMemcpy(prop, b->d_rprop + 3 * o, 12 * n, cudaMemcpyDeviceToHost));
  if (u) CUDA_TRY(cudaMemcpy(u, b->d_ru + o, 8 * n, cudaMemcpyDeviceToHost));
  if (dE) CUDA_TRY(cudaMemcpy(dE, b->d_rdE + o, 4 * n, cudaMemcpyDeviceToHost));
  if (acc) CUDA_TRY(cudaMemcpy(acc, b->d_racc + o, n, cudaMemcpyDeviceToHost));
  return SCEMC_OK;
}

int32_t scemc_batch_site_coeffs(scemc_batch* b, int32_t slot, float* c) {
  if (!b || !c) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (!b->fast) return fail(SCEMC_ERR_ARG, "site coefficients need the fast tables (lmax 1 or 2 dense programs)");
  if (slot < 0 || slot >= b->n_slots) return fail(SCEMC_ERR_ARG, "slot out of range");
  int li = 0;
  while (li + 1 < (int)b->tabs.size() && slot >= b->slot0[li + 1]) ++li;
  const int r = slot - b->slot0[li];
  const int NR = b->lmax == 1 ? 3 : 8;
  const int64_t n = (int64_t)b->tabs[li]->n_sites * NR;
  float* d_out = nullptr;
  CUDA_TRY(cudaMalloc(&d_out, sizeof(float) * std::max<int64_t>(n, 1)));
  const int blocks = (int)std::min<int64_t>(sm_count(b->device) * 8, (b->tabs[li]->n_sites + 255) / 256 + 1);
  if (b->lmax == 1) k_site_coeffs<1, false><<<blocks, 256, 0, b->stream>>>(b->d_lat, li, r, b->d_spins, d_out);
  else if (b->trip2) k_site_coeffs<2, true><<<blocks, 256, 0, b->stream>>>(b->d_lat, li, r, b->d_spins, d_out);
  else k_site_coeffs<2, false><<<blocks, 256, 0, b->stream>>>(b->d_lat, li, r, b->d_spins, d_out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(c, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(SCEMC_ERR_CUDA, std::string("site coefficients: ") + cudaGetErrorString(e));
  return SCEMC_OK;
}

int32_t scemc_batch_fetch_record_ratio(const scemc_batch* b, double* lqr) {
  if (!b || !b->d_rlqr || !lqr) return fail(SCEMC_ERR_ARG, "recording was never enabled");
  CUDA_TRY(cudaMemcpy(lqr, b->d_rlqr, sizeof(double) * b->tabs[b->rec_li]->n_sites, cudaMemcpyDeviceToHost));
  return SCEMC_OK;
}

int32_t scemc_batch_set_learned(scemc_batch* b, const scemc_mlp* m, const int32_t* env, int32_t k) {
  if (!b) return fail(SCEMC_ERR_ARG, "batch is NULL");
  std::vector<DevLattice> lats(b->tabs.size());
  CUDA_TRY(cudaMemcpy(lats.data(), b->d_lat, sizeof(DevLattice) * lats.size(), cudaMemcpyDeviceToHost));
  for (int32_t* p : b->d_env)
    if (p) cudaFree(p);
  b->d_env.assign(b->tabs.size(), nullptr);
  b->mlp = nullptr;
  b->learned_field = false;
  for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
  b->graphs.clear();
  if (m && k == 0) {  // field mode: the inputs are the site's coefficients and kT
    const int nr = b->lmax == 1 ? 3 : 8;
    if (!b->fast) return fail(SCEMC_ERR_ARG, "a field-input learned proposal needs the fast tables");
    if (m->n_in != nr + 1)
      return fail(SCEMC_ERR_ARG, "a field-input network reads n_in = NR + 1 inputs (" + std::to_string(nr + 1) + ")");
    b->mlp = m;
    b->learned_field = true;
  } else if (m) {
    if (!env) return fail(SCEMC_ERR_ARG, "env is NULL");
    if (k < 1 || k > 21 || m->n_in != 3 * k + 1)
      return fail(SCEMC_ERR_ARG, "the network reads n_in = 3 k + 1 inputs (k environment spins and kT, k <= 21)");
    int64_t off = 0;
    for (size_t i = 0; i < b->tabs.size(); ++i) {
      const scemc_tables* T = b->tabs[i];
      const int64_t n = (int64_t)T->n_sites * k;
      for (int64_t j = 0; j < n; ++j)
        if (env[off + j] < 0 || env[off + j] >= T->n_sites)
          return fail(SCEMC_ERR_ARG, "environment site outside 0..n_sites-1 of table " + std::to_string(i));
      for (int32_t s = 0; s < T->n_sites; ++s)
        for (int j = 0; j < k; ++j) {
          const int32_t t = env[off + (int64_t)s * k + j];
          if (T->site_col_of[s] > 0 && T->site_col_of[s] == T->site_col_of[t])
            return fail(SCEMC_ERR_ARG, "an environment site shares its site's colour (the proposal would not "
                                       "be reversible)");
        }
      int32_t rc;
      if ((rc = dalloc(&b->d_env[i], (size_t)n))) return rc;
      CUDA_TRY(h2d_sync(b->d_env[i], env + off, sizeof(int32_t) * n));
      off += n;
    }
    b->mlp = m;
  }
  for (size_t i = 0; i < lats.size(); ++i) {
    lats[i].env = b->d_env[i];
    lats[i].env_k = m && !b->learned_field ? k : 0;
  }
  CUDA_TRY(h2d_sync(b->d_lat, lats.data(), sizeof(DevLattice) * lats.size()));
  return SCEMC_OK;
}

int32_t scemc_color_sites(int32_t n_sites, const int32_t* site_ptr, const int32_t* site_inst, const int32_t* inst_ptr,
                          const int32_t* inst_sites, const uint8_t* site_active, int32_t* colors_out,
                          int32_t* n_colors) {
  if (n_sites < 0 || !site_ptr || !site_inst || !inst_ptr || !inst_sites || !site_active || !colors_out || !n_colors)
    return fail(SCEMC_ERR_ARG, "NULL argument");
  std::vector<int32_t> stamp;
  int32_t ncol = 0;
  for (int32_t s = 1; s <= n_sites; ++s) {
    colors_out[s - 1] = 0;
  }
  for (int32_t s = 1; s <= n_sites; ++s) {
    if (!site_active[s - 1]) continue;
    for (int32_t j = site_ptr[s - 1]; j < site_ptr[s]; ++j) {
      const int32_t i = site_inst[j - 1];
      for (int32_t q = inst_ptr[i - 1]; q < inst_ptr[i]; ++q) {
        const int32_t c = colors_out[inst_sites[q - 1] - 1];
        if (c > 0) stamp[c - 1] = s;
      }
    }
    int32_t c = 1;
    while (c <= ncol && stamp[c - 1] == s) ++c;
    if (c > ncol) {
      ncol = c;
      stamp.push_back(0);
    }
    colors_out[s - 1] = c;
  }
  *n_colors = ncol;
  return SCEMC_OK;
}

// L2 read bandwidth (GB/s) of a buffer small enough to stay in L2: every block reads
// its share of the buffer `reps` times through L2 (ld.global.cg: L1 bypassed) in one
// launch; the best of five timed launches after a warm-up. The roofline denominator
// of sweeps whose working set fits in L2.
int32_t scemc_l2_probe(int64_t bytes, int32_t reps, double* gbs) {
  if (bytes < (1 << 20) || bytes > ((int64_t)96 << 20) || reps < 1 || !gbs)
    return fail(SCEMC_ERR_ARG, "scemc_l2_probe: bytes in [1 MiB, 96 MiB], reps >= 1");
  const int64_t n4 = bytes / 16;
  float4* buf = nullptr;
  float* sink = nullptr;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  const int blocks = sm_count(dev) * 4;
  CUDA_TRY(cudaMalloc(&buf, (size_t)n4 * 16));
  CUDA_TRY(cudaMalloc(&sink, sizeof(float) * blocks));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMemset(buf, 0, (size_t)n4 * 16);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float best = 1e30f;
  for (int t = 0; t < 6 && e == cudaSuccess; ++t) {
    cudaEventRecord(e0);
    k_l2_probe<<<blocks, 256>>>(buf, n4, reps, sink);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (t > 0) best = std::min(best, ms);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  cudaFree(sink);
  if (e != cudaSuccess) return fail(SCEMC_ERR_CUDA, std::string("scemc_l2_probe: ") + cudaGetErrorString(e));
  *gbs = (double)n4 * 16.0 * reps / (best * 1e-3) / 1e9;
  return SCEMC_OK;
}

int32_t scemc_selftest_barrier_timeout(int64_t limit_ns) {
  GridSync* gs = nullptr;
  CUDA_TRY(cudaMalloc(&gs, sizeof(GridSync)));
  CUDA_TRY(cudaMemset(gs, 0, sizeof(GridSync)));
  void* params[] = {&gs, &limit_ns};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(2), dim3(32), params, 0, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  GridSync h{};
  if (e == cudaSuccess) e = cudaMemcpy(&h, gs, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(gs);
  if (e != cudaSuccess) return fail(SCEMC_ERR_CUDA, cudaGetErrorString(e));
  if (h.error) return fail(SCEMC_ERR_TIMEOUT, "grid barrier gave up after the bound, as designed");
  return SCEMC_OK;
}

}  // extern "C"

// =============================================================================
// Allocation-free FP64 energy recompute.
//
// Some callers cannot call cudaMalloc at the moment they need an energy: a host
// that owns all device memory through its own pool allocator (a Julia CUDA.jl
// program that hands the library only its arrays), or a time-critical loop that
// must not pay cudaMalloc's device-wide synchronisation. For them this variant of
// the FP64 recompute takes caller-owned device buffers and keeps its only scratch
// (the per-chunk partial sums) in a fixed file-scope device array instead of the
// buffer scemc_total_energy allocates. The array holds kStaticScratch doubles
// (512 KiB) on every GPU that loads the library, until the process exits.
// =============================================================================
namespace {

constexpr int kStaticScratch = 65536;  // doubles: n_chunks(1024 instances each) x replicas
static __device__ __align__(256) double g_energy_scratch[kStaticScratch];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Same arithmetic and chunking as k_energy_chunks, with the lattice passed by value.
__global__ void __launch_bounds__(256) k_energy_chunks_static(DevLattice L, const float4* spins, int R,
                                                              double* partial, int n_chunks) {
  const int chunk = blockIdx.x, r = blockIdx.y;
  double acc = 0.0;
  for (int k = 0; k < kChunk / 256; ++k) {
    const int64_t i = (int64_t)chunk * kChunk + k * 256 + threadIdx.x;
    if (i >= L.n_inst) break;
    const int t = L.inst_term[i];
    const int off = L.inst_ptr[i];
    double Ei = 0.0;
    for (int e = L.eprog_ptr[t]; e < L.eprog_ptr[t + 1]; ++e) {
      double p = 1.0;
      const int f0 = L.efac_ptr[e], nf = L.efac_ptr[e + 1] - f0;
      for (int m = 0; m < nf; ++m) {
        const float4 v = spins[(int64_t)L.inst_sites[off + m] * R + r];
        p *= zval_f64(L.efac_row[f0 + m], (double)v.x, (double)v.y, (double)v.z);
      }
      Ei += L.eent_w[e] * p;
    }
    acc += L.term_coef[t] * Ei;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o >= 1; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[(size_t)r * n_chunks + chunk] = red[0];
}

__global__ void k_energy_fold_static(const double* partial, int n_chunks, int R, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  double E = 0.0;
  for (int c = 0; c < n_chunks; ++c) E += partial[(size_t)r * n_chunks + c];
  out[r] = E;
}

}  // namespace

namespace {
// All-site energy gradient (gpu_gradient.jl:131-243 semantics): G lanes per (site,
// replica) walk the site's records for its leave-one-out coefficients c (FP32, the
// sweep's walk); lane 0 forms G = sum_t c_t grad Z_t(e) with FP64 tangent gradient
// rows. Read-only in the spins, one launch over every site (no colouring).
template <int LMAX, int G>
__global__ void __launch_bounds__(256) k_energy_gradient(DevLattice L, const float4* spins, int R, double* grad) {
  constexpr int NLM = (LMAX + 1) * (LMAX + 1);
  const int lane = threadIdx.x % G;
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int n_groups = (gridDim.x * blockDim.x) / G;
  const int64_t n_items = (int64_t)L.n_sites * R;
  const unsigned int gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x % 32) / G * G));
  const int64_t rounds = (n_items + n_groups - 1) / n_groups;
  for (int64_t rd = 0; rd < rounds; ++rd) {
    const int64_t item = rd * n_groups + group;
    const bool valid = item < n_items;
    const int s = valid ? (int)(item / R) : 0, r = valid ? (int)(item % R) : 0;
    float c[NLM];
#pragma unroll
    for (int k = 0; k < NLM; ++k) c[k] = 0.0f;
    if (valid) accumulate_c<LMAX, G, false>(L, spins, R, r, s, lane, c);
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1)
#pragma unroll
      for (int k = 0; k < NLM; ++k) c[k] += __shfl_xor_sync(gmask, c[k], o);
    if (!valid || lane != 0) continue;
    const float4 e = spins[(int64_t)s * R + r];
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int t = 0; t < NLM; ++t) {
      if (c[t] == 0.0f) continue;
      int l, m;
      row_lm(t, l, m);
      double g[3];
      grad_zlm_f64(l, m, e.x, e.y, e.z, g);
      gx += (double)c[t] * g[0];
      gy += (double)c[t] * g[1];
      gz += (double)c[t] * g[2];
    }
    double* out = grad + ((int64_t)r * L.n_sites + s) * 3;
    out[0] = gx;
    out[1] = gy;
    out[2] = gz;
  }
}

using GradFn = void (*)(DevLattice, const float4*, int, double*);
GradFn gradient_kernel(int lmax) {
  switch (lmax) {
    case 0: return k_energy_gradient<0, 8>;
    case 1: return k_energy_gradient<1, 8>;
    case 2: return k_energy_gradient<2, 8>;
    case 3: return k_energy_gradient<3, 8>;
    case 4: return k_energy_gradient<4, 8>;
    case 5: return k_energy_gradient<5, 8>;
    default: return k_energy_gradient<6, 8>;
  }
}

__global__ void k_config_to_spins(const double* cfg, int64_t n, float4* spins) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    spins[i] = make_float4((float)cfg[3 * i], (float)cfg[3 * i + 1], (float)cfg[3 * i + 2], 0.0f);
}
}  // namespace

// config: replicas x (3 x n_sites) FP64 host (payload order); grad the same shape.
// The spins are rounded to FP32 as in a chain.
extern "C" int32_t scemc_energy_gradient(const scemc_tables* t, const double* config, int32_t replicas,
                                         double* grad) {
  if (!t || !config || !grad) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (replicas < 1) return fail(SCEMC_ERR_ARG, "replicas must be >= 1");
  if (!t->has_generic) return fail(SCEMC_ERR_UNSUPPORTED, "generic records were not kept for these tables");
  const int64_t n = (int64_t)t->n_sites * replicas;
  for (int64_t i = 0; i < 3 * n; ++i)
    if (!std::isfinite(config[i])) return fail(SCEMC_ERR_NUMERIC, "non-finite spin component");
  // device layout spins[site * R + r]: transpose the replica-major host payload
  std::vector<double> cfg((size_t)3 * n);
  for (int32_t r = 0; r < replicas; ++r)
    for (int32_t s = 0; s < t->n_sites; ++s)
      for (int d = 0; d < 3; ++d)
        cfg[((size_t)s * replicas + r) * 3 + d] = config[((size_t)r * t->n_sites + s) * 3 + d];
  double *d_cfg = nullptr, *d_grad = nullptr;
  float4* d_spins = nullptr;
  int32_t rc = SCEMC_OK;
  if ((rc = dalloc(&d_cfg, (size_t)3 * n)) || (rc = dalloc(&d_grad, (size_t)3 * n)) ||
      (rc = dalloc(&d_spins, (size_t)n))) {
    cudaFree(d_cfg);
    cudaFree(d_grad);
    cudaFree(d_spins);
    return rc;
  }
  auto done = [&](int32_t r) {
    cudaFree(d_cfg);
    cudaFree(d_grad);
    cudaFree(d_spins);
    return r;
  };
  if (cudaMemcpy(d_cfg, cfg.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return done(fail(SCEMC_ERR_CUDA, "config upload"));
  k_config_to_spins<<<(unsigned)std::min<int64_t>(1024, (n + 255) / 256), 256>>>(d_cfg, n, d_spins);
  DevLattice L = t->dl;
  L.R = replicas;
  L.spin_off = 0;
  const int G = 8;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sm_count(t->device) * 8, (n * G + 255) / 256));
  gradient_kernel(t->lmax)<<<blocks, 256>>>(L, d_spins, replicas, d_grad);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
    return done(fail(SCEMC_ERR_CUDA, "gradient kernel"));
  if (cudaMemcpy(grad, d_grad, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return done(fail(SCEMC_ERR_CUDA, "gradient download"));
  return done(SCEMC_OK);
}

extern "C" int32_t scemc_total_energy_static(const scemc_tables* t, const void* spins, int32_t replicas,
                                             double* energies, void* stream) {
  if (!t || !spins || !energies) return fail(SCEMC_ERR_ARG, "NULL argument");
  if (replicas < 1) return fail(SCEMC_ERR_ARG, "replicas must be >= 1");
  const int64_t n_chunks = std::max<int64_t>(1, (t->n_inst + kChunk - 1) / kChunk);
  if (n_chunks * replicas > kStaticScratch)
    return fail(SCEMC_ERR_ARG, "scemc_total_energy_static: ceil(n_instances/1024) x replicas = " +
                                   std::to_string(n_chunks * replicas) + " exceeds the fixed scratch of " +
                                   std::to_string(kStaticScratch) + " partial sums");
  // one grid row per replica: the y dimension of a launch grid stops at 65535
  if (replicas > 65535) return fail(SCEMC_ERR_ARG, "scemc_total_energy_static: replicas must be <= 65535");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  // the kernels read the tables' device pointers: they must run on the tables' device
  if (dev != t->device)
    return fail(SCEMC_ERR_ARG, "scemc_total_energy_static: the current device is " + std::to_string(dev) +
                                   " but the tables live on device " + std::to_string(t->device) +
                                   "; make that device current");
  if (dev < 0 || dev >= kMaxDevices) return fail(SCEMC_ERR_ARG, "device index out of range");
  double* scratch = nullptr;
  {
    // One-time set-up per device, with that device current: the host-side name of
    // g_energy_scratch is not a device address, so its address is looked up here.
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      CUDA_TRY(cudaGetSymbolAddress(&p, g_energy_scratch));
      g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  DevLattice L = t->dl;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_energy_chunks_static<<<dim3((unsigned)n_chunks, (unsigned)replicas), 256, 0, st>>>(
      L, static_cast<const float4*>(spins), replicas, scratch, (int)n_chunks);
  CUDA_TRY(cudaGetLastError());
  k_energy_fold_static<<<(replicas + 127) / 128, 128, 0, st>>>(scratch, (int)n_chunks, replicas, energies);
  CUDA_TRY(cudaGetLastError());
  return SCEMC_OK;
}
