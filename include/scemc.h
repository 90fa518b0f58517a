/*
 * scemc.h — C ABI of libscemc_cuda.so, the B200 (sm_100a) chain-level spin Monte
 * Carlo sweep for SCEMonteCarlo.jl tiled SCE Hamiltonians.
 *
 * Conventions
 *   - Every entry point returns an int32 status (SCEMC_OK = 0); on failure the
 *     message is available from scemc_last_error(). No exception or abort ever
 *     crosses the boundary; device waits are bounded and report SCEMC_ERR_TIMEOUT.
 *   - Index arrays are passed exactly as the Julia `TiledHamiltonian` holds them
 *     (1-based); the library rebases them when it builds its device tables.
 *   - Spin configurations cross the boundary as 3 x n_sites FP64 column-major
 *     arrays (the `to_matrix` layout of the reference); the device holds them as
 *     FP32 float4. Energies are FP64.
 *   - Calls are synchronous: they return after the device work completed.
 *   - Objects are not thread-safe; one host thread per chain/batch at a time.
 *
 * Reference interfaces replaced (paths relative to the SCEMonteCarlo.jl root):
 *   scemc_tables_create        GPUTiledHamiltonian(backend, H)   src/gpu/gpu_hamiltonian.jl:66-88
 *   scemc_chain_create         GPUChainState(gH, st; seed)       src/gpu/gpu_state.jl:49-61
 *   scemc_metropolis_sweep     gpu_metropolis_sweep!             src/gpu/gpu_sweep.jl:158-190
 *   scemc_run_sweeps           gpu_run_sweeps!                   src/gpu/gpu_sweep.jl:204-218
 *   scemc_download             to_host!                          src/gpu/gpu_state.jl:71-76
 *   scemc_upload               _from_host!                       src/gpu/gpu_state.jl:81-86
 *   scemc_swap_payload         _swap_payload! (device lanes)     src/gpu/gpu_pt.jl:46-51
 *   scemc_overrelaxation_sweep overrelaxation_sweep! (CPU-only in the reference)
 *                                                                src/updates.jl:231-248
 *   scemc_total_energy         _total_energy                     src/energy.jl:55-75
 *   scemc_renormalize          _renormalize!                     src/state.jl:168-185
 *   scemc_batch_*              _gpu_lane_segment! + exchanges    src/gpu/gpu_pt.jl:82-140
 *   scemc_color_sites          _color_sites (table-build helper) src/hamiltonian.jl:456-499
 */
#ifndef SCEMC_H
#define SCEMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SCEMC_OK = 0,
  SCEMC_ERR_ARG = 1,          /* ArgumentError / DimensionMismatch equivalents */
  SCEMC_ERR_UNSUPPORTED = 2,  /* e.g. lmax > 6 (gpu_hamiltonian.jl:67-68) */
  SCEMC_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  SCEMC_ERR_TIMEOUT = 4,      /* a bounded device wait gave up (grid barrier) */
  SCEMC_ERR_EXHAUSTED = 5,    /* 32-bit sweep counter exhausted (gpu_sweep.jl:163-164) */
  SCEMC_ERR_NUMERIC = 6       /* non-finite value detected in the state */
};

typedef struct scemc_tables scemc_tables;
/* A chain and a batch are the same device object: a set of replicas over one or
 * more table sets. A chain is a batch of one replica. */
typedef struct scemc_ensemble scemc_chain;
typedef struct scemc_ensemble scemc_batch;

/* The flat arrays of one TiledHamiltonian (src/hamiltonian.jl:234-265,62-91),
 * 1-based as Julia holds them. Lengths: site_ptr n_sites+1; site_inst/site_slot/
 * site_prog/site_col/site_col2 n_adj; inst_term n_inst; inst_ptr n_inst+1;
 * inst_sites n_inst_sites; sprog_ptr n_sprog+1; sent_w/sent_tgt/sfac_ptr(+1)/
 * pent_row/pent_row2 n_sent; sfac_row/sfac_slot n_sfac; eprog_ptr n_terms+1;
 * eent_w/efac_ptr(+1) n_eent; efac_row n_efac; term_coef n_terms; color_ptr
 * n_colors+1; color_sites n_active; site_has_l1/site_active n_sites.
 * term_body/term_ls give each template's body order and per-member l (ls
 * concatenated over templates); they let the library pick its dense fast paths. */
typedef struct scemc_tables_desc {
  int32_t n_sites, nlm, lmax, n_colors, n_active, n_cell_atoms;
  int64_t n_adj, n_inst, n_inst_sites, n_sprog, n_sent, n_sfac, n_terms, n_eent, n_efac;
  const int32_t* site_ptr;
  const int32_t* site_inst;
  const int8_t* site_slot;
  const int32_t* inst_term;
  const int32_t* inst_ptr;
  const int32_t* inst_sites;
  const int32_t* site_prog;
  const int32_t* sprog_ptr;
  const double* sent_w;
  const int32_t* sent_tgt;
  const int32_t* sfac_ptr;
  const int32_t* sfac_row;
  const int8_t* sfac_slot;
  const int32_t* site_col;
  const int32_t* site_col2;
  const int32_t* pent_row;
  const int32_t* pent_row2;
  const int32_t* eprog_ptr;
  const double* eent_w;
  const int32_t* efac_ptr;
  const int32_t* efac_row;
  const double* term_coef;
  const int32_t* term_body;
  const int32_t* term_ls;
  const int32_t* color_ptr;
  const int32_t* color_sites;
  const uint8_t* site_has_l1;
  const uint8_t* site_active;
} scemc_tables_desc;

/* Copies the last error message of this host thread (NUL-terminated). */
int32_t scemc_last_error(char* buf, size_t len);
/* Library version as major*10000 + minor*100 + patch. */
int32_t scemc_version(void);

/* GPUTiledHamiltonian(backend, H): validates and uploads the tables to the current
 * CUDA device. lmax > 6 => SCEMC_ERR_UNSUPPORTED. */
int32_t scemc_tables_create(const scemc_tables_desc* desc, scemc_tables** out);
int32_t scemc_tables_destroy(scemc_tables* t);
/* Table statistics used by the roofline: mean distinct neighbours per active site
 * (d), mean adjacency entries per active site (A), and table bytes on the device. */
int32_t scemc_tables_stats(const scemc_tables* t, double* d_mean, double* a_mean, int64_t* bytes);
/* Mean merged records per active site that the row- and replica-parallel kernels
 * walk (one per distinct pair neighbour, l = 1 triplet and quad, plus the body-1
 * vector; 0 when the tables have no fast form). Each record is 8 bytes and names
 * its neighbours by local index into the site's distinct-neighbour list. */
int32_t scemc_tables_records(const scemc_tables* t, double* records_mean);

/* GPUChainState(gH, st; seed): uploads config (3 x n_sites FP64, column-major) and
 * the chain's incremental energy; step is the Metropolis rotation scale. */
int32_t scemc_chain_create(const scemc_tables* t, const double* config, double energy, uint64_t seed,
                           double step, scemc_chain** out);
int32_t scemc_chain_destroy(scemc_chain* c);

/* gpu_metropolis_sweep!: one Metropolis sweep at inverse temperature beta.
 * lanes_per_site (the reference's workgroupsize) must be a power of two; values
 * above 32 use 32. *n_accepted receives the number of accepted moves. */
int32_t scemc_metropolis_sweep(scemc_chain* c, const scemc_tables* t, double beta, int32_t lanes_per_site,
                               int64_t* n_accepted);
/* One overrelaxation sweep (reflection about the local l = 1 field + Metropolis
 * accept on the exact dE; updates.jl:66-87). *n_attempted counts sites with a
 * non-vanishing l = 1 field. */
int32_t scemc_overrelaxation_sweep(scemc_chain* c, const scemc_tables* t, double beta,
                                   int32_t lanes_per_site, int64_t* n_accepted, int64_t* n_attempted);
/* gpu_run_sweeps! without the trailing download: nsweeps Metropolis sweeps, with a
 * device renormalisation + FP64 energy recompute every renorm_interval sweeps
 * (<= 0 disables). Call scemc_download for to_host!. */
int32_t scemc_run_sweeps(scemc_chain* c, const scemc_tables* t, double beta, int64_t nsweeps,
                         int64_t renorm_interval, int32_t lanes_per_site);
/* to_host!: config (3 x n_sites FP64), incremental energy, completed sweeps and
 * counters {acc_metro, att_metro, acc_or, att_or}. Any pointer may be NULL. */
int32_t scemc_download(const scemc_chain* c, double* config, double* energy, int64_t* sweep_index,
                       int64_t* counters);
/* _from_host!: replaces config and energy; seed, sweep_index, step and counters stay. */
int32_t scemc_upload(scemc_chain* c, const double* config, double energy);
/* Step (Metropolis rotation scale) of a chain. */
int32_t scemc_set_step(scemc_chain* c, double step);
/* _swap_payload!: exchanges config and energy between two single-replica chains on
 * the same tables; seed, sweep_index, step and counters stay with each chain. */
int32_t scemc_swap_payload(scemc_chain* a, scemc_chain* b);
/* FP64 total energy of the device state (replica r of the chain or batch),
 * deterministic fixed-order reduction. */
int32_t scemc_total_energy(const scemc_ensemble* e, int32_t replica, double* energy);
/* _renormalize!: normalises active spins, recomputes the FP64 energy of every
 * replica, re-anchors the incremental energy. drift (per replica, may be NULL)
 * receives |E_incremental - E_recomputed|. */
int32_t scemc_renormalize(scemc_ensemble* e, double* drift);

/* ---- batches: many replicas (PT rungs, temperatures, chains of uneven sizes) ---- */

/* A batch over n_tables table sets with replicas[i] replicas each. Replica slots are
 * numbered table-major (all replicas of table 0, then table 1, ...). configs holds
 * 3 x n_sites(table) FP64 per slot in that order; energies, seeds and steps one per
 * slot. */
int32_t scemc_batch_create(int32_t n_tables, const scemc_tables* const* tables, const int32_t* replicas,
                           const double* configs, const double* energies, const uint64_t* seeds,
                           const double* steps, scemc_batch** out);
int32_t scemc_batch_destroy(scemc_batch* b);
int32_t scemc_batch_size(const scemc_batch* b, int32_t* n_slots, int64_t* n_sites_total);

/* Run parameters of scemc_batch_run. Rung r of a ladder owns beta, step, seed and
 * counters; the payload (spins + energy) it currently holds is slot slot_of_rung[r].
 * Ladders are the replicas of one table set (exchange only within a table). */
typedef struct scemc_run_params {
  int64_t nsweeps;           /* compound sweeps to run */
  int32_t or_per_metropolis; /* overrelaxation sweeps after each Metropolis sweep */
  int32_t exchange;          /* 1: adjacent-rung swap attempts after every exchange_interval sweeps */
  int64_t exchange_interval;
  int64_t adapt_interval;    /* > 0: step adaptation every adapt_interval sweeps (thermalisation) */
  double adapt_target;
  int64_t renorm_interval;   /* > 0: renormalise + FP64 recompute every renorm_interval sweeps */
  int64_t measure_interval;  /* > 0: record observables every measure_interval sweeps */
  int32_t lanes_per_site;    /* 0 = autotuned */
  int32_t mode;              /* 0 = auto (autotuned if scemc_batch_autotune ran, else 2), 1 = one launch per
                                colour, 2 = persistent grid kernel per pass, 3 = per-colour launches of a
                                compound sweep captured once in a CUDA graph and replayed, 4 = persistent
                                data-flow kernel per pass (row-parallel kernel; an item waits for the
                                completion flags of its earlier-colour neighbours instead of a grid barrier
                                between colours) */
  /* Phase bookkeeping (the reference's lane.phase_sweeps): sweep i of this call is
   * sweep phase_done + i of its phase; adaptation, renormalisation, measurement and
   * exchange fire on that count, and no exchange follows the phase's last sweep
   * (phase_total; 0 means phase_done + nsweeps). */
  int64_t phase_done;
  int64_t phase_total;
  int32_t kernel;     /* 0 = auto, 1 = generic record walk, 2 = row-parallel fast kernel (one warp per
                         item), 3 = replica-parallel kernel (one thread per item; per-colour launches
                         with mode 1 or 3, one persistent cooperative launch per pass with mode 2),
                         4 = chain-resident cluster kernel (one thread-block cluster per
                         replica slot holds the replica's spins in shared memory; the row-parallel
                         arithmetic, bit for bit; one launch per compound sweep, mode 1 or 3; needs
                         n_sites x 16 bytes plus scratch within one block's shared memory),
                         5 = replica-parallel kernel with the pair records on the tensor cores (lmax 2
                         fast tables; one warp per site and 32 replicas, mma.sync TF32 with both
                         operands split into a TF32 head and tail; mode 1 or 3, plain proposals; dE
                         agrees with the FMA kernels' to rounding, not bit for bit) */
  int32_t proposals;  /* 0 = auto, 1 = precompute a pass's Metropolis proposals, 2 = inline, 3 = learned
                         network (scemc_batch_set_learned; kernels 2 or 3, per-colour modes 1 or 3) */
  int32_t rep_replicas; /* kernel 3: replicas per thread, 1 or 2; 0 = per colour launch, 1 when its
                           one-replica threads fill at most two waves of the GPU, else 2 */
  int32_t rep_threads_per_item; /* kernel 3: threads sharing one item's record walk, 1 or 2; 0 = per colour
                                   launch, 2 when twice its one-replica threads fit one wave, else 1 */
  int32_t rep_prefetch; /* kernel 3: 1 = records and neighbour rows prefetched into L1 first, 2 = not;
                           0 = per colour launch, prefetch when its threads fill at most two waves.
                           Prefetching changes no arithmetic: 1 and 2 give bitwise equal chains */
} scemc_run_params;

/* Inverse temperatures per rung (n_slots values, table-major like the slots). */
int32_t scemc_batch_set_betas(scemc_batch* b, const double* betas);
int32_t scemc_batch_set_steps(scemc_batch* b, const double* steps);
int32_t scemc_batch_run(scemc_batch* b, const scemc_run_params* p);
/* Asynchronous form: enqueues the run on the batch's stream and returns; the
 * caller must call scemc_batch_sync before touching the batch again. */
int32_t scemc_batch_run_async(scemc_batch* b, const scemc_run_params* p);
int32_t scemc_batch_sync(scemc_batch* b);
/* The batch's cudaStream_t (as void*), for callers that order or time work on it. */
int32_t scemc_batch_stream(const scemc_batch* b, void** stream);
/* Replaces every slot's spins (3 x n_sites FP64 per slot, payload order) and, when
 * energies is not NULL, the running energies (with NULL they keep their old values;
 * scemc_renormalize on the batch recomputes them). The payload crosses the bus unchanged
 * in one copy; the device checks it (SCEMC_ERR_NUMERIC names the first non-finite
 * spin's replica and column, and nothing changes), rounds it to FP32 and interleaves
 * the replicas. Replaces _from_host! (src/gpu/gpu_state.jl:81-86) for every slot. */
int32_t scemc_batch_upload(scemc_batch* b, const double* configs, const double* energies);
/* Page-locks (and releases) a host buffer so that uploads and downloads through it
 * are direct DMA; a Julia caller pins the Arrays it passes to the transfer calls
 * (what CUDA.jl's Mem.pin does for the reference's to_host!/from_host! buffers). */
int32_t scemc_host_register(void* ptr, int64_t bytes);
int32_t scemc_host_unregister(void* ptr);
/* Live timing of the sweep kernels: with profiling on, each pass is bracketed by a
 * CUDA event pair on the batch stream; scemc_batch_kernel_time returns the summed
 * device time (ms) and the number of passes since profiling was switched on. */
int32_t scemc_batch_profile(scemc_batch* b, int32_t on);
/* Times the launch forms (modes 2 and 3; for fast tables the row- and
 * replica-parallel kernels with proposal precompute on/off, for the generic kernel
 * the lanes per site) for sweeps_per_trial compound sweeps each and keeps the
 * fastest for runs with mode = 0 and kernel = 0. The trial sweeps are real sweeps of
 * the batch (its chains advance). Outputs may be NULL. */
int32_t scemc_batch_autotune(scemc_batch* b, int32_t or_per_metropolis, int32_t sweeps_per_trial, int32_t* mode,
                             int32_t* proposals, int32_t* lanes, int32_t* kernel, double* ms_per_sweep);
int32_t scemc_batch_kernel_time(const scemc_batch* b, double* ms, int64_t* passes);
/* ---------------------------------------------------------------------------
 * Learned proposal network (no counterpart in the reference): a per-site MLP
 * 43 -> 128 -> 128 -> 20 (SiLU; BF16 weights on the tcgen05 tensor cores, FP32
 * accumulate) whose 20 outputs parameterise a 4-component von Mises-Fisher mixture
 * on S^2 (per component: logit, raw mean (3), raw concentration c; kappa =
 * softplus(c) / kT[meV] + 1e-3). Inputs per row (n_in = 3 k + 1 floats): the k
 * environment spins (x, y, z) in the environment table's order, then kT in meV;
 * k = 14 (bcc nearest and next-nearest shells, n_in = 43), 18 (fcc, n_in = 55), at
 * most 21 (n_in <= 64).
 * Parameters travel as one FP32 block of SCEMC_MLP_PARAMS floats: W1 [128][64]
 * (input columns n_in..63 zero), b1 [128], W2 [128][128], b2 [128], W3 [32][128]
 * (output rows 20..31 zero), b3 [32].
 * ------------------------------------------------------------------------- */
#define SCEMC_MLP_PARAMS 28960
typedef struct scemc_mlp scemc_mlp;
int32_t scemc_mlp_create(uint64_t seed, int32_t n_in, scemc_mlp** out);
int32_t scemc_mlp_destroy(scemc_mlp* m);
int32_t scemc_mlp_get_params(const scemc_mlp* m, float* params);
int32_t scemc_mlp_set_params(scemc_mlp* m, const float* params);
/* out: n x 20 network outputs for the n x n_in inputs x. */
int32_t scemc_mlp_forward(scemc_mlp* m, const float* x, int64_t n, float* out);
/* Mean negative log-likelihood of the unit targets y (n x 3) under the mixture and
 * its gradient (SCEMC_MLP_PARAMS floats); n a multiple of 128; no update. */
int32_t scemc_mlp_loss_grad(scemc_mlp* m, const float* x, const float* y, int64_t n, double* loss, float* grad);
/* Adam (beta 0.9 / 0.999) on minibatches of `batch` rows (a multiple of 128), `epochs`
 * shuffled passes over the n rows; epoch_loss (may be NULL) gets each epoch's mean
 * minibatch loss. */
int32_t scemc_mlp_train(scemc_mlp* m, const float* x, const float* y, int64_t n, int32_t batch, int32_t epochs,
                        double lr, uint64_t seed, double* epoch_loss);

/* All-site energy gradient (gpu_energy_gradient!, src/gpu/gpu_gradient.jl:193-231):
 * grad[s] = sum_t c_t(s) grad Z_t(e_s), the tangent gradient of the energy at each
 * spin (c the leave-one-out coefficients, grad Z the tangent-projected gradient rows
 * of src/gpu/grad_device.jl). config and grad: replicas x 3 x n_sites FP64 (payload
 * order); spins are rounded to FP32 as in a chain, c is accumulated in FP32 and the
 * gradient rows and the sum are FP64. No colouring: one launch over every site. */
int32_t scemc_energy_gradient(const scemc_tables* t, const double* config, int32_t replicas, double* grad);

/* Registers a learned proposal network with a batch (m = NULL unregisters). env:
 * for every table of the batch in order, n_sites x k 0-based site ids, the sites
 * whose spins (in that order) form a site's network input; 1 <= k <= 21 with the
 * network's n_in = 3 k + 1, and no
 * environment site may share its site's colour. The network is not copied: it must
 * outlive the batch's learned runs. Runs with proposals = 3 then draw every
 * Metropolis proposal from the network's vMF mixture and accept it with
 * probability min(1, exp(-beta dE) q(e | env) / q(e' | env)). */
int32_t scemc_batch_set_learned(scemc_batch* b, const scemc_mlp* m, const int32_t* env, int32_t k);
/* Leave-one-out coefficients c_t of every site of a replica slot's current spins,
 * rows 1..NR of the site's tesseral basis (NR = 3 for lmax 1, 8 for lmax 2), FP32,
 * n_sites(table) x NR values; zeros for inactive sites. They fix each site's
 * conditional distribution, exp(-beta sum_t c_t Z_t(e)), and are the inputs of a
 * learned proposal in field mode (scemc_batch_set_learned with k = 0). Needs the fast
 * tables. */
int32_t scemc_batch_site_coeffs(scemc_batch* b, int32_t slot, float* c);
/* log q(e | env) - log q(e' | env) of the recorded learned Metropolis pass (the
 * recorded replica; n_sites values, 0 where no learned proposal was recorded). */
int32_t scemc_batch_fetch_record_ratio(const scemc_batch* b, double* lqr);

/* Number of kernels the batch has enqueued on its stream since creation: sweep
 * passes, proposal precompute, tails, recomputes and measurements; a replayed
 * sweep graph adds its kernel nodes. */
int32_t scemc_batch_launches(const scemc_batch* b, int64_t* launches);
/* State readback. configs: 3 x n_sites per SLOT (payload order); energies per slot;
 * slot_of_rung per rung; counters 4 per rung {acc_metro, att_metro, acc_or, att_or};
 * swap counters 2 per rung pair {attempted, accepted} (pair r = rungs r, r+1 of one
 * table; the last rung of each table has zeros); steps per rung; max_drift per rung. */
int32_t scemc_batch_download(const scemc_batch* b, double* configs, double* energies, int32_t* slot_of_rung,
                             int64_t* counters, int64_t* swaps, double* steps, double* max_drift);
/* Resets the per-rung counters (acc/att metro, acc/att or, swaps) and max_drift. */
int32_t scemc_batch_reset_counters(scemc_batch* b);
/* Checkpoint of a batch's mutable state, for the gpu_pt lane block of a checkpoint
 * (src/checkpoint.jl:388-425, docs/specs/checkpoint-schema.md:83-100): the FP32 spins
 * bit for bit, running energies, rung maps, counters, swap counters, steps, device
 * keys, betas, adaptation windows, drift and the sweep counter with the exchange
 * parity. The keyed Philox streams have no other state, so a batch loaded with the
 * blob continues exactly as the saved one would. The tables are not included; the
 * blob records each table's size and replica count, and loading it into a batch of
 * another shape fails with SCEMC_ERR_ARG. Pending measurement records are dropped. */
int32_t scemc_batch_state_bytes(const scemc_batch* b, int64_t* bytes);
int32_t scemc_batch_save_state(scemc_batch* b, void* buf, int64_t bytes);
int32_t scemc_batch_load_state(scemc_batch* b, const void* buf, int64_t bytes);
/* Measurement records written by scemc_batch_run since the last fetch: n_records
 * rows of (n_slots x record_len) FP64, indexed by RUNG, each
 * {E, mx, my, mz, sub_x1, sub_y1, sub_z1, ...} with m over active sites and the
 * sublattice sums per cell as in src/observables.jl:104-143. Pass rec = NULL to
 * query the count and record_len; a fetch with rec clears the buffer. */
int32_t scemc_batch_fetch_measurements(scemc_batch* b, double* rec, int64_t capacity, int64_t* n_records,
                                       int32_t* record_len);

/* Parity recording for the replay gate: with recording on, every pass of a sweep
 * (pass -1 = Metropolis, 0..2 = overrelaxation passes) stores per site of the
 * recorded replica (replica 0 of table 0 unless scemc_batch_record_slot chose
 * another) the proposal (3 FP32), the accept uniform, the FP32 dE and a flag
 * (1 accepted, 0 rejected, 2 not attempted, 3 not visited). Turning it on clears
 * the record. fetch_record returns n_sites(table) values per array. */
int32_t scemc_batch_record(scemc_batch* b, int32_t on);
/* Chooses the recorded replica: replica `replica` (0-based, < replicas[table]) of
 * table `table` (0-based). */
int32_t scemc_batch_record_slot(scemc_batch* b, int32_t table, int32_t replica);
int32_t scemc_batch_fetch_record(const scemc_batch* b, int32_t pass, float* prop, double* u, float* dE,
                                 uint8_t* acc);

/* Greedy proper colouring of the site-conflict graph in site order
 * (hamiltonian.jl:456-499), host-side helper for table builders. 1-based inputs;
 * colors_out receives one colour (1-based, 0 = inactive) per site; returns the
 * number of colours in *n_colors. */
int32_t scemc_color_sites(int32_t n_sites, const int32_t* site_ptr, const int32_t* site_inst,
                          const int32_t* inst_ptr, const int32_t* inst_sites, const uint8_t* site_active,
                          int32_t* colors_out, int32_t* n_colors);

/* L2 read bandwidth (GB/s) of a `bytes`-sized device buffer (1 to 96 MiB, small
 * enough to stay in the 126 MB L2) read `reps` times in one launch through L2-only
 * loads; best of five timed launches on the current device. A measurement helper for
 * the roofline of sweeps whose working set fits in L2 (no counterpart in the
 * reference). */
int32_t scemc_l2_probe(int64_t bytes, int32_t reps, double* gbs);

/* Failure-detection self test: runs the persistent kernel's grid barrier with one
 * block that never arrives, bounded by limit_ns; returns SCEMC_ERR_TIMEOUT when the
 * wait gives up as designed (SCEMC_OK would mean the bound did not fire). */
int32_t scemc_selftest_barrier_timeout(int64_t limit_ns);

/* Allocation-free FP64 energy recompute (no counterpart in the reference; an
 * addition for callers that cannot allocate device memory when they need an
 * energy: a host whose own pool allocator owns all device memory and lends the
 * library its buffers, or a time-critical loop that must not pay cudaMalloc's
 * device-wide synchronisation).
 *   spins:    caller-owned device array of float4 (x, y, z, unused), n_sites x
 *             replicas, site-major / replica-minor (spins[site * replicas + r]);
 *   energies: caller-owned device array of replicas doubles (output);
 *   stream:   cudaStream_t to enqueue on (NULL = the legacy default stream).
 * Same arithmetic as scemc_total_energy. The call enqueues two kernels and returns;
 * the energies are ready when the stream reaches that point. The device the tables
 * were created on must be the current device (another current device returns
 * SCEMC_ERR_ARG), and spins, energies and stream must belong to it. It calls no
 * allocator: its scratch is a fixed device array of 65536 doubles (512 KiB) that
 * every GPU loading the library holds until exit, so ceil(n_instances / 1024) x
 * replicas must not exceed 65536, and replicas must not exceed 65535 (larger
 * requests return SCEMC_ERR_ARG). The first call on each device looks up that
 * array's device address (with the device current); make that first call before
 * any stream capture. All calls share the
 * array: calls whose kernels overlap on the GPU (for example on two streams) race
 * and must be serialised by the caller. The kernels write every partial sum they
 * read, so nothing in the array needs to start at zero. */
int32_t scemc_total_energy_static(const scemc_tables* t, const void* spins, int32_t replicas, double* energies,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SCEMC_H */
