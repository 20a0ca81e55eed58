/*
 * phmc.h — C ABI of the B200-native constant-pH Monte Carlo energy engine.
 *
 * The engine replaces the energy and move layer of the ph_brush MC program
 * (reference: MC/include/energy.hpp, MC/include/pme.hpp, MC/include/neighbor.hpp,
 * MC/include/mc.hpp).  Every entry point returns an int status (PHMC_OK == 0),
 * never throws, and records a message retrievable with phmc_last_error().
 * The engine owns all device memory; callers own host buffers.  One engine is
 * driven by one host thread; engines are independent of each other.
 *
 * Units follow the reference: Coulomb prefactor ke/epsilon_r with
 * ke = 138.935458 (MC/src/pme.cu:305).  Reduced units are obtained with
 * beta = 1 and epsilon_r = 138.935458 / l_B.
 *
 * An engine holds R >= 1 independent replicas (same kernels; one replica is
 * the plain engine, many replicas are the batched titration sweep).
 */
#ifndef PHMC_H
#define PHMC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHMC_ABI_VERSION 1

/* ---- status codes ---- */
enum {
    PHMC_OK = 0,
    PHMC_ERR_ARG = 1,         /* invalid argument / inconsistent input */
    PHMC_ERR_CUDA = 2,        /* CUDA runtime error (message has details) */
    PHMC_ERR_CAPACITY = 3,    /* a fixed capacity (cell, slot, pending) was exceeded */
    PHMC_ERR_BUDGET = 4,      /* a bounded device loop gave up (iteration budget) */
    PHMC_ERR_STATE = 5,       /* engine in a state that forbids the call */
    PHMC_ERR_UNSUPPORTED = 6, /* feature combination not implemented */
    PHMC_ERR_IO = 7           /* file could not be read / parsed */
};

/* ---- Coulomb kinds (reference: Params::coulombtype, MC/include/types.hpp:42) ---- */
enum { PHMC_COUL_NONE = 0, PHMC_COUL_CUT = 1, PHMC_COUL_EWALD = 2 };

/* ---- particle flags ---- */
#define PHMC_F_MOBILE     0x01 /* may be displaced */
#define PHMC_F_TITRATABLE 0x02 /* protonation site (weak base) */
#define PHMC_F_GHOST      0x04 /* empty slot: not present, interacts with nothing */
#define PHMC_F_CATION     0x08 /* mobile salt cation (reservoir swaps) */
#define PHMC_F_ANION      0x10 /* mobile anion (counterion / salt anion) */

/* ---- move kinds ---- */
enum { PHMC_MOVE_DISP = 0, PHMC_MOVE_TITR = 1, PHMC_MOVE_SWAP = 2, PHMC_MOVE_NONE = 3 };

/*
 * One replica's particle system, host arrays.  Slots [0, n_particles) hold
 * the initial particles; slots [n_particles, capacity) are empty (ghost) and
 * receive inserted ions.  Bonds are 1-2 pairs of 0-based slot indices
 * (reference: System::bonds, MC/include/types.hpp:18-28).
 */
typedef struct phmc_system {
    int n_particles;
    int capacity;
    const float* x;
    const float* y;
    const float* z;
    const float* q;
    const int* type;   /* 0-based type ids */
    const int* flags;  /* PHMC_F_* */
    int n_bonds;
    const int* bond_i;
    const int* bond_j;
    double box[3];     /* Lx, Ly, Lz (Lz already padded when the slab correction is on) */
} phmc_system;

/*
 * Interaction model, move set and engine tuning for one replica.
 * Reference-compatible energies: lj_rc = NULL and rc_lj = rc_coul (single
 * shared cutoff, MC/src/neighbor.cu:97), excl_bonded_lj = excl_bonded_coul = 1
 * (MC/src/neighbor.cu:17-19), order 4, ref_moduli = 1.
 */
typedef struct phmc_params {
    int n_types;
    const double* lj_eps;  /* n_types*n_types, row-major, symmetric */
    const double* lj_sig;  /* n_types*n_types */
    const double* lj_rc;   /* n_types*n_types per-pair cutoff, or NULL: rc_lj for all */
    double rc_lj;
    int lj_shift;          /* shift LJ to zero at its cutoff (MC/src/io.cpp:270-281) */
    int coulomb;           /* PHMC_COUL_* */
    double rc_coul;
    double epsilon_r;
    double ewald_alpha;    /* > 0 for PHMC_COUL_EWALD */
    int mesh[3];           /* SPME mesh nx, ny, nz */
    int order;             /* B-spline order p (points per dimension), 4..8 */
    int ref_moduli;        /* 1: reference moduli exactly (MC/src/pme.cu:77-113); 0: zero-modulus interpolation */
    int slab;              /* Yeh-Berkowitz + net-charge slab term (MC/src/pme.cu:434-447) */
    int excl_bonded_lj;    /* exclude 1-2 pairs from LJ */
    int excl_bonded_coul;  /* exclude 1-2 pairs from real-space Coulomb */
    double fene_k, fene_r0;  /* FENE bonds; fene_k == 0 disables */
    double wall_lo, wall_hi; /* hard walls in z; wall_hi <= wall_lo disables (z periodic) */
    double beta;
    /* titration (weak base: neutral <-> +1 with counterion insert/delete) */
    double pH, pKa;
    int type_site_neutral, type_site_charged;
    float q_site_charged;
    int type_counterion;
    float q_counterion;
    /* reservoir salt swaps (cation/anion pair insert/delete) */
    double salt_conc;      /* reservoir pair concentration, sigma^-3 (ideal activity) */
    int type_cation;
    float q_cation;
    /* move mix (probabilities; their sum must be <= 1, remainder is a no-op) */
    double p_disp, p_titr, p_swap;
    double disp_max;
    uint64_t seed;
    /* engine tuning (0 = default) */
    int cell_cap;          /* particles per cell capacity */
    int pending_max;       /* stencils buffered before the potential mesh is rebuilt */
    int threads;           /* threads per replica block in the MC kernel */
} phmc_params;

typedef struct phmc_energy_components {
    double lj;         /* LJ / WCA pair energy */
    double fene;       /* bonded FENE energy */
    double coul_real;  /* real-space Coulomb (erfc) or plain cutoff Coulomb */
    double coul_recip; /* SPME reciprocal */
    double self;       /* Ewald self term */
    double qcorr;      /* net-charge term */
    double slab;       /* Yeh-Berkowitz slab term */
    double total;
} phmc_energy_components;

/* A trial = up to two particle changes, evaluated against the current state. */
typedef struct phmc_change {
    int index;      /* slot */
    int present;    /* 1: present after the change; 0: removed */
    float x, y, z, q;
    int type;
} phmc_change;

typedef struct phmc_trial {
    int n_changes;  /* 1 or 2 */
    phmc_change c[2];
} phmc_trial;

typedef struct phmc_run_stats {
    int64_t attempted[3];  /* per move kind */
    int64_t accepted[3];
    int64_t flushes;       /* potential-mesh rebuilds */
    int n_titratable;
    int n_charged_sites;   /* currently protonated sites */
    int n_cations, n_anions;
    double energy;         /* tracked total energy (FP64) */
    double energy_drift;   /* |tracked - recomputed| at the last flush */
} phmc_run_stats;

typedef struct phmc_engine phmc_engine;

/* ---- library ---- */
int phmc_abi_version(void);
const char* phmc_last_error(void);

/* ---- lifecycle ----
 * Replaces the reference set-up: upload_atoms_to_device + copy_csr_to_device +
 * build_half_neighbors_gpu + pmeCreate (MC/src/main.cu:18-41,127-141,
 * MC/src/neighbor.cu:65-125, MC/src/pme.cu:291-335). */
int phmc_create(int n_replicas, const phmc_system* systems, const phmc_params* params,
                int device, phmc_engine** out);
int phmc_destroy(phmc_engine* e);

/* ---- energies ----
 * Full recompute on the device (replaces total_energy, MC/src/mc.cu:43-60:
 * compute_lj_sr_energy_gpu + pmeEnergy).  out has n_replicas entries. */
int phmc_energy(phmc_engine* e, phmc_energy_components* out);

/* dE of n independent trials of replica r, each against the current state.
 * No counterpart in the reference (it recomputes the total per trial). */
int phmc_delta_energy(phmc_engine* e, int replica, const phmc_trial* trials, int n, double* dE);

/* phmc_delta_energy split into the components of phmc_energy_components (total
 * = their sum); lets a caller keep the reference's separate LJ and Coulomb sums. */
int phmc_delta_energy_components(phmc_engine* e, int replica, const phmc_trial* trials, int n,
                                 phmc_energy_components* out);

/* Apply one trial to replica r (state, cell list, pending mesh changes). */
int phmc_commit(phmc_engine* e, int replica, const phmc_trial* trial);

/* Identity change of one particle (reference: set_atom_identity, MC/src/mc.cu:33-41;
 * type is 0-based as on the reference's device side). */
int phmc_set_identity(phmc_engine* e, int replica, int i, int type, float q);

/* ---- Monte Carlo ----
 * Run n_trials Metropolis trials per replica on the device (persistent
 * kernel, potential-mesh rebuilds in between).  Replaces the host trial
 * loops (MC/src/mc.cu:159-318,320-550).  stats has n_replicas entries. */
int phmc_run(phmc_engine* e, int64_t n_trials, phmc_run_stats* stats);

/* Record per-trial (move, dE, accept) of the next phmc_run into host arrays of
 * length >= n_trials (replica 0 only; NULL disables).  For replay checks. */
int phmc_set_trial_log(phmc_engine* e, int64_t capacity, int* move, double* dE, int* accepted);

/* Replay mode: the next phmc_run takes accept decisions from `decisions`
 * (replica 0, one int per trial) instead of the Metropolis test. NULL disables. */
int phmc_set_replay(phmc_engine* e, int64_t n, const int* decisions);

/* Change the move mix of replica r (-1: all) for the following runs, e.g. a
 * titration-only phase like the reference's protonation phase
 * (MC/src/mc.cu:320-550).  Same rules as phmc_params. */
int phmc_set_move_mix(phmc_engine* e, int replica, double p_disp, double p_titr, double p_swap);

/* ---- tuning (no counterpart in the reference) ----
 * pending_max: stencils buffered before the potential mesh is rebuilt (each
 * trial pays a correction per buffered stencil, each rebuild a pass over the
 * mesh); threads: threads per replica block of the MC kernel (128 or 256).
 * Both may change between runs.  phmc_autotune times `trials` trials per
 * replica for each candidate (pending_max 8..128 x threads 128/256) in two
 * interleaved passes, keeps the fastest and reports every candidate's better time; its runs are ordinary Monte Carlo
 * trials and advance the chains.  Decisions do not depend on the tuning except
 * through FP32 rounding of the reciprocal-space dE. */
typedef struct phmc_tuning {
    int pending_max;
    int threads;
    double us_per_trial;  /* autotune only: device time per trial (all replicas) of a trial-run candidate */
    /* tile shapes (phmc_set_tile_shapes) */
    int zpass;            /* z pass of the potential-mesh rebuild: 0 the shared-memory Stockham pass, k > 0 a
                             register-resident two-stage split nz = zpass_n1 x zpass_n2 (when every replica
                             has the same nz and a split for it exists) */
    int zpass_n1, zpass_n2;
    int cand_round;       /* pair pass: candidate particles per thread and round (2, 4 or 8 at order 5; 4
                             otherwise); a round's neighbour tile is cand_round x threads candidates */
    int g_rows;           /* pending-correction sum: rows of the influence kernel G in flight per thread
                             (2; 3 or 4 with cand_round 2 at order 5, one row per work item); 21 with
                             cand_round 2 or 4 at order 5: one stencil pair per warp, the lanes over its
                             (y, x) window plane, every z plane's loads in flight */
    int plane_pipe;       /* rebuild's first pass: 1 persistent blocks that bulk-copy the next band plane's
                             charges into shared memory while transforming the current one; 0 one block per
                             plane (square lateral meshes of the register passes only) */
    int energy_block;     /* full recompute: particles per block of the pair / FENE pass (64, 128, 256), or 0
                             for the cell-ordered pass (one warp per cell, partners read by broadcast) */
    double rebuild_us;    /* autotune only: device time of one rebuild of every replica's potential mesh */
    double recompute_us;  /* autotune only: device time of one full pair / FENE recompute of every replica */
    int first_stage;      /* 1: the attached surrogate judges titration / swap trials first (delayed
                             acceptance); 0: no surrogate, or bypassed because exact trials ran faster */
} phmc_tuning;
int phmc_set_tuning(phmc_engine* e, int pending_max, int threads);
/* The tile shapes above; -1 leaves a field as it is.  Decisions do not depend on them
 * except through FP32 / FP64 rounding of summation orders. */
int phmc_set_tile_shapes(phmc_engine* e, int zpass, int cand_round, int g_rows, int energy_block, int plane_pipe);
int phmc_get_tuning(phmc_engine* e, phmc_tuning* out);
/* Cost-based fallback of delayed acceptance: on = 0 bypasses the attached surrogate's
 * first stage (every trial plain Metropolis on the exact dE, as with no surrogate)
 * without detaching it; on = 1 restores it.  The autotuner sets it by timing both. */
int phmc_set_first_stage(phmc_engine* e, int on);
/* Autotuner: first the z pass (the Stockham pass and every register split of the
 * replicas' nz, timed as whole rebuilds), the first pass pipelined or not (the same
 * rebuilds), then the full recompute's block size,
 * then pending_max x threads by trial runs of `trials` trials per replica (two
 * interleaved passes, each candidate's faster time kept), then the pair pass's
 * shape (round width x G rows) at the best pending_max x threads, then, with a surrogate attached,
 * its first stage on against bypassed; keeps the fastest of each stage.
 * results[] gets one entry per candidate timed, with that stage's time set. */
int phmc_autotune(phmc_engine* e, int64_t trials, phmc_tuning* results, int max_results, int* n_results);
/* Launch quorum, 0 < quorum <= 1: an MC launch of a batched engine ends once that
 * fraction of the replicas still running at its start have filled their pending
 * buffer; the others stop with theirs partly filled, and the rebuild folds both in.
 * 1 lets every replica run until its buffer is full or its trials are done, and
 * leaves the blocks of the replicas whose buffers fill first idle until the
 * slowest fills.  Default 0.2.  Applied only when every replica's block is
 * resident at once.  Decisions do not depend on it except through FP32 rounding
 * of the reciprocal-space dE. */
int phmc_set_quorum(phmc_engine* e, double quorum);
/* Bound on the MC kernel launches one call of phmc_run (phmc_run_timed, the
 * autotuner's runs), phmc_gc_phase or phmc_phase2 may make; 0 (the default)
 * leaves only the guard against a loop that makes no progress.  A call that
 * reaches the bound with work left returns PHMC_ERR_BUDGET between launches:
 * every replica's state is consistent and a later call continues from it (a
 * device phase's results and events of that call are not written).  No
 * counterpart in the reference, whose loops are unbounded host loops. */
int phmc_set_launch_budget(phmc_engine* e, int64_t max_launches);
/* z-density profiles of the constant-pH runs (no counterpart in the reference,
 * whose driver writes configurations only): with nbins in 1..PHMC_ZHIST_MAX_BINS,
 * each replica's MC kernel adds, whenever its trial count reaches a multiple of
 * `every` during phmc_run, the histogram over z of its charged titratable sites,
 * anions and cations (nbins equal bins between the walls; [0, Lz) without walls)
 * to a device accumulator and counts the sample; nbins = 0 switches it off.  The
 * call clears the accumulators.  phmc_get_zhist gives one replica's sums,
 * counts[3 * nbins] (sites, anions, cations), and its number of samples: the mean
 * profile is counts / n_samples, the mean degree of ionisation the site counts'
 * sum / (n_samples * titratable sites). */
#define PHMC_ZHIST_MAX_BINS 64
int phmc_set_zhist(phmc_engine* e, int nbins, int64_t every);
int phmc_get_zhist(phmc_engine* e, int replica, double* counts, int64_t* n_samples);

/* ---- input files of the reference's driver (host side, no device use) ----
 * LAMMPS "full" data files: phmc_lammps_header reads the header (counts, box
 * lengths), phmc_lammps_read the Atoms and Bonds sections into caller arrays in
 * file order (bond atoms as 0-based indices; bonds naming unknown atom ids are
 * dropped; wrap != 0 wraps positions into [0, L)), with the reference reader's
 * section rules and number conversions (MC/src/io.cpp:79-146, wrap :303-316), so
 * the values are bit-identical to the reference's.  phmc_lammps_write writes a
 * file (box from 0; FP32 values with 9 significant digits) that both readers read
 * back to the same arrays (replaces write_lammps_full, MC/src/io.cpp:326-368). */
typedef struct phmc_lammps_info {
    int natoms, nbonds, nbonds_read, ntypes;
    double box[3];
} phmc_lammps_info;
int phmc_lammps_header(const char* path, phmc_lammps_info* out);
int phmc_lammps_read(const char* path, int wrap, int cap_atoms, int cap_bonds, int* id, int* mol, int* type,
                     float* q, float* x, float* y, float* z, int* bond_type, int* bond_i, int* bond_j,
                     phmc_lammps_info* info);
int phmc_lammps_write(const char* path, int natoms, const int* id, const int* mol, const int* type, const float* q,
                      const float* x, const float* y, const float* z, int nbonds, const int* bond_type,
                      const int* bond_i, const int* bond_j, int ntypes, const double* box);
/* params.in (replaces read_params, MC/src/io.cpp:171-301): the reference's keys with
 * its defaults, derived values (Ewald alpha from ewald_rtol, the LJ shift table at
 * rc) and checks, values rounded to FP32 as the reference holds them; lj_eps /
 * lj_sig / lj_shift_tbl hold ntypes x ntypes.  Superset: the native model's keys
 * pH, pKa, salt_conc, wall_lo, wall_hi, fene_k, fene_r0, p_disp, p_titr, p_swap,
 * disp_max (NaN when absent) and pme_mesh = nx ny nz (0 when absent), which the
 * reference ignores.  Unknown entries are listed comma-separated in `unknown`;
 * with strict != 0 they are an error (PHMC_ERR_IO) instead of being ignored. */
typedef struct phmc_file_params {
    double rc, epsilon_r, ewald_rtol, ewald_alpha, pme_spacing, pme_3dc_zfac, beta, target_pct, w_z_extra_nm,
        mu_eta, nacc_frac_round;
    int lj_shift, coulomb /* PHMC_COUL_CUT, PHMC_COUL_EWALD, -1 unknown */, pme_order, pme_3dc, nh_n_type,
        nh_p_type, w_type, cl_type, rng_seed, energy_interval, patience, max_attempts, direct_pct_threshold,
        gc_block_fixed, epoch_attempt_max, phase2_wc;
    double pH, pKa, salt_conc, wall_lo, wall_hi, fene_k, fene_r0, p_disp, p_titr, p_swap, disp_max;
    int mesh[3];
} phmc_file_params;
int phmc_params_read(const char* path, int ntypes, int strict, phmc_file_params* p, double* lj_eps, double* lj_sig,
                     double* lj_shift_tbl, char* unknown, int unknown_len);

/* ---- checkpoint / exact resume (no counterpart in the reference: its LAMMPS data
 * output, MC/src/io.cpp:326-368, keeps positions and identities but not the chain's
 * random-number counter, list order or tracked energies) ----
 * phmc_checkpoint_save writes every replica's particle arrays, the index lists the
 * proposals draw from and the cell lists (their order included), the per-replica
 * counters (trial index = Philox counter, accept counts, delayed-acceptance window)
 * and tracked FP64 energies and charge moments, the move mix, the tuning, the
 * launch quorum and the fixed-point charge mesh.  phmc_checkpoint_load restores
 * them into an engine created from the same systems and parameters (other
 * replicas, capacities or cells are refused with PHMC_ERR_IO) and recomputes the
 * potential; runs continue bit for bit as the saved engine's would.  An attached surrogate is
 * not part of the checkpoint (phmc_surrogate_save / _load, then attach). */
int phmc_checkpoint_save(phmc_engine* e, const char* path);
int phmc_checkpoint_load(phmc_engine* e, const char* path);

/* ---- state ----
 * replica == -1: every replica at once, arrays of sum(capacity) slots concatenated
 * in replica order (one upload and one full recompute for the whole engine). */
int phmc_get_state(phmc_engine* e, int replica, float* x, float* y, float* z, float* q,
                   int* type, int* flags);
/* Replace replica r's particle state from host arrays of capacity length (bonds
 * unchanged); rebuilds lists, cells and the potential mesh.  The reference's
 * counterpart is upload_atoms_to_device (MC/src/main.cu:18-41). */
int phmc_set_state(phmc_engine* e, int replica, const float* x, const float* y, const float* z,
                   const float* q, const int* type, const int* flags);

/* ---- measurement (no counterpart in the reference) ---- */
typedef struct phmc_profile {
    double mc_ms;            /* summed device time of Monte Carlo kernel launches */
    double flush_ms;         /* summed device time of potential-mesh rebuilds */
    int64_t mc_launches;
    int64_t flush_launches;  /* rebuild pipelines (each = spread + 3 FFT passes + reduce) */
    int64_t kernel_launches; /* every kernel the engine launched */
    double mc_alg_bytes;     /* algorithmic bytes of all trials (per-trial model in the docs) */
    double flush_alg_bytes;  /* algorithmic bytes of all rebuilds: 16 N + 32 Mcb + 12 Mb per replica (N particles,
                                Mb / Mcb real / half-spectrum mesh points of the planes between the walls) */
    int64_t trials;
    double mc_busy_ms;       /* summed over replicas: time their MC blocks ran; mc_busy_ms / (replicas * mc_ms)
                                is the share of the launches' replica slots that did work */
} phmc_profile;
/* Profiling on: per-launch CUDA events around the MC kernel and the rebuilds. */
int phmc_set_profiling(phmc_engine* e, int on);
int phmc_get_profile(phmc_engine* e, phmc_profile* out, int reset);
/* Phase clocks of the MC kernel: with `on`, each replica's block adds the SM cycles of
 * its trial phases (read with clock64 by the block's first thread at the barrier that
 * ends each phase; one extra barrier per trial separates phases 4 and 5):
 *   0 proposal (and the charge-mesh updates of the last accepted change),
 *   1 surrogate first stage, 2 cell counts + stencils + direct and bonded terms,
 *   3 candidate offsets + stencil-pair tables, 4 candidate pair terms,
 *   5 stencil . phi + pending-stencil corrections + block reduction,
 *   6 decision + commit, 7 trials that end before phase 2.
 * phmc_get_phase_cycles sums them over replicas, with the trials the replicas ran
 * since the clocks were last switched or reset in *trials (when not NULL); `reset`
 * zeroes them.  No counterpart in the reference. */
#define PHMC_PHASES 8
int phmc_set_phase_clock(phmc_engine* e, int on);
int phmc_get_phase_cycles(phmc_engine* e, int64_t cycles[PHMC_PHASES], int64_t* trials, int reset);
/* phmc_run with its device time (CUDA events on the engine stream) in *device_ms. */
int phmc_run_timed(phmc_engine* e, int64_t n_trials, double* device_ms);
/* Write `bytes` of scratch on the engine stream (evicts L2 between timed steps). */
int phmc_flush_l2(phmc_engine* e, int64_t bytes);
/* cell index of every slot (-1 for ghosts) and the cell grid dimensions */
int phmc_get_cells(phmc_engine* e, int replica, int* cell_of, int dims[3]);
int phmc_capacity(phmc_engine* e, int replica);

/* ---- allocation-free reciprocal energy ----
 * No counterpart in the reference.  SPME reciprocal-space energy of n point
 * charges (host arrays), for callers that cannot call cudaMalloc: a host
 * program whose device memory is all handed out by its own allocator (a
 * framework's caching pool, a fixed per-process budget), a plugin called back
 * from such a program, or a per-trial loop that must not stall on an
 * allocation's implicit device synchronisation.  It uses one file-scope device
 * array (about 3 MB, held by every GPU that loads the library until exit) and
 * never allocates.  Limits: n <= PHMC_STATIC_MAX_PARTICLES, nx*ny*nz <=
 * PHMC_STATIC_MAX_MESH, each side 2^a 3^b 5^c in [order, 512]; larger inputs
 * return PHMC_ERR_CAPACITY.  Works on the current device, on the legacy default
 * stream, and synchronises before it returns.  That device's first call looks
 * up the array's device address, so make it before any stream capture; after a
 * cudaDeviceReset of the device do not call it again in the process.  Calls
 * share the array (and host staging tables): a process-wide lock serialises
 * them, so calls through this function never overlap, but any other work that
 * overlaps a call on the GPU and touches the array races with it. */
#define PHMC_STATIC_MAX_PARTICLES 32768
#define PHMC_STATIC_MAX_MESH 131072
int phmc_recip_energy_static(const float* x, const float* y, const float* z, const float* q, int n,
                             const double box[3], const int mesh[3], int order, double ewald_alpha,
                             double epsilon_r, int ref_moduli, double* e_recip);

/* ---- learned surrogate and delayed acceptance (no counterpart in the reference) ----
 *
 * The surrogate is an MLP n_in -> H -> H -> H -> 1 (GELU, BF16 weights and
 * activations, FP32 accumulation on the tensor cores) trained on the GPU with
 * Adam.  A sample is one titration or swap move: PHMC_SUR_ROWS rows of n_in
 * features (the old and the new state of each changed particle; row layout in
 * the design notes) with signs -1 / +1 (0 = unused row) and a target
 * t = dE - (exact terms), where the exact terms are the direct interaction of
 * the two changed particles and the self / net-charge / slab changes.  The
 * estimate of a move is scale * sum_r sign_r y(row_r) + exact terms: minus the
 * estimate of the reverse move, so delayed acceptance with it keeps detailed
 * balance.  The engine's first stage needs n_in == PHMC_SUR_INPUTS. */
#define PHMC_SUR_INPUTS 80
#define PHMC_SUR_ROWS 4
#define PHMC_SUR_DESC_STRIDE (PHMC_SUR_ROWS * PHMC_SUR_INPUTS + 2 * PHMC_SUR_ROWS + 4)
typedef struct phmc_surrogate phmc_surrogate;
int phmc_surrogate_create(int n_in, int hidden, uint64_t seed, phmc_surrogate** out);
/* Training products (forward, input and weight gradients) on the fifth-generation
 * tensor cores (tcgen05.mma, FP32 accumulator in tensor memory) when tcgen05 != 0
 * (the default), else on the mma.sync path; process-wide, for comparisons. */
int phmc_surrogate_set_gemm(int tcgen05);
int phmc_surrogate_destroy(phmc_surrogate* s);
int phmc_surrogate_num_params(phmc_surrogate* s);
/* flat FP32 parameters: W1[n_in*H], b1[H], W2[H*H], b2[H], W3[H*H], b3[H], w4[H], b4;
 * W[k*H + j] connects input k to unit j */
int phmc_surrogate_get_params(phmc_surrogate* s, float* out, int n);
int phmc_surrogate_set_params(phmc_surrogate* s, const float* in, int n);
/* input standardisation (x - mu) / sd and the output scale (energy = scale * y) */
int phmc_surrogate_set_scaling(phmc_surrogate* s, const float* mu, const float* sd, float scale);
int phmc_surrogate_get_scaling(phmc_surrogate* s, float* mu, float* sd, float* scale);
/* per-row outputs in energy units for n_rows host rows of n_in features */
int phmc_surrogate_predict(phmc_surrogate* s, const float* x, int n_rows, float* y);
/* loss 1/2 mean((pred - clip(t)) / scale)^2 and its gradient w.r.t. the flat
 * parameters for n samples (x: n*PHMC_SUR_ROWS rows, sign: n*PHMC_SUR_ROWS) */
int phmc_surrogate_gradient(phmc_surrogate* s, const float* x, const float* sign, const float* t, int n, float clip,
                            double* loss, float* grad);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over host samples; rescale = 1 first sets the
 * standardisation and scale from the data.  *loss = mean batch loss of the last epoch. */
int phmc_surrogate_train(phmc_surrogate* s, const float* x, const float* sign, const float* t, int n, int epochs,
                         int batch, float lr, float clip, uint64_t seed, int rescale, double* loss);
int phmc_surrogate_save(phmc_surrogate* s, const char* path);
int phmc_surrogate_load(const char* path, phmc_surrogate** out);

/* Record a training sample for every titration / swap trial of the following
 * phmc_run calls (all replicas, exact dE), up to `capacity` samples; 0 stops
 * and frees.  Each call clears the samples. */
int phmc_harvest(phmc_engine* e, int capacity);
int phmc_harvest_count(phmc_engine* e, int* n);
int phmc_harvest_get(phmc_engine* e, int n, float* x, float* sign, float* t);
/* Train s on the harvested samples on the device (rescale from the data). */
int phmc_surrogate_fit(phmc_engine* e, phmc_surrogate* s, int epochs, int batch, float lr, float clip, uint64_t seed,
                       double* loss);
/* Delayed acceptance for titration and swap trials of all replicas: stage one
 * is Metropolis on the surrogate estimate, stage two on the exact dE minus the
 * estimate.  A replica returns to plain Metropolis when, over `window`
 * stage-one passes, fewer than `threshold` of them are accepted by stage two.
 * s must outlive the attachment; NULL detaches.  Resets the counters. */
int phmc_surrogate_attach(phmc_engine* e, phmc_surrogate* s, double threshold, int window);
typedef struct phmc_da_stats {
    int64_t evaluated;  /* trials judged by the surrogate */
    int64_t passed;     /* stage-one passes (exact dE computed) */
    int64_t accepted;   /* stage-two accepts */
    int fallback;       /* 1: replica went back to plain Metropolis */
    int pad;
} phmc_da_stats;
int phmc_get_da_stats(phmc_engine* e, phmc_da_stats* out); /* n_replicas entries */
/* Descriptor rows, signs, per-row outputs and exact terms of n trials of replica r
 * against the current state (PHMC_SUR_DESC_STRIDE floats per trial: rows, signs,
 * outputs, cross term, moment terms, row count, inner-cell particles); dEs gets
 * the surrogate estimate (NaN without an attached surrogate).  For checks. */
int phmc_surrogate_describe(phmc_engine* e, int replica, const phmc_trial* t, int n, float* out, double* dEs);
/* With a trial log set: also record, per trial, the stage reached (0 plain,
 * 1 rejected by the surrogate, 2 judged by the exact dE) and the estimate. */
int phmc_set_da_log(phmc_engine* e, int* stage, double* dEs);

/* ---- synthetic input (no counterpart in the reference, whose inputs are
 * LAMMPS data files, MC/src/io.cpp:79-146) ----
 * Grafted brush: chains on a square lattice at z = 0, self-avoiding random
 * walks, random initial ionisation, counterions and salt pairs in the slab.
 * Types: 0 neutral site, 1 charged site (+1), 2 anion (-1), 3 cation (+1),
 * 4 permanently charged bead (+1). */
typedef struct phmc_brush_spec {
    int chains_x, chains_y;
    double graft_spacing;
    int len_min, len_max;      /* beads per chain, drawn uniformly */
    int n_permanent;           /* inner beads with a permanent +1 charge (diblock) */
    int graft_titratable;      /* grafted (immobile) bead is a titratable site */
    double height;             /* slab height: particles in [0, height) */
    double lz;                 /* box Lz (padded for the slab correction) */
    double ion_frac;           /* initial fraction of titratable sites charged */
    double salt_conc;          /* salt pairs per sigma^3 of the slab */
    double bond_len, min_dist;
    uint64_t seed;
} phmc_brush_spec;

/* counts[0] = particles, counts[1] = bonds; box_out = {Lx, Ly, Lz}. */
int phmc_build_brush(const phmc_brush_spec* spec, int capacity, float* x, float* y, float* z, float* q, int* type,
                     int* flags, int max_bonds, int* bond_i, int* bond_j, int* counts, double* box_out);

/* ---- the reference's grand-canonical mu-control phase on the device ----
 * Replaces phase_gc_mu_control (MC/include/mc.hpp:73-82, MC/src/mc.cu:320-548):
 * pair flips NH_N + W -> NH_P(+1) + Cl(-1) and back, forward with probability
 * a c / (a c + b d) (a = |NH_N|, b = |NH_P|, c = |W|, d = |Cl| pools), accepted
 * when -beta (dE - s mu) + ln(S_before / S_after), clamped to +-40, is >= 0 or
 * its exponential beats a uniform draw; blocks of gc_block trials; at the end
 * of each epoch (accept target or attempt limit reached) mu moves by
 * kT eta (logit f - logit f*) w_info; the phase ends when the protonated count
 * reaches floor(target_pct / 100 Nh), or when no pair can flip.
 * The whole phase runs in persistent MC-kernel launches (one block per job),
 * with the reference's own random stream: the caller hands over its
 * std::mt19937 (625 words: the 624 state words and the position, in the order
 * the generator's stream output writes them) and gets it back where the
 * phase left it, so the draws, the pool order (erase + push_back) and the
 * float arithmetic of the reference's energies, mu update and acceptance are
 * the reference's.  Jobs touch distinct replicas; their pools hold distinct
 * present slots. */
#define PHMC_GC_EV_CHUNK 1     /* a block of gc_block trials ended */
#define PHMC_GC_EV_MU 2        /* an epoch ended: mu updated */
#define PHMC_GC_EV_REACHED 3   /* the protonated count reached its target: the phase ends */
#define PHMC_GC_EV_NO_PAIRS 4  /* neither direction has a pair: the phase ends */
#define PHMC_GC_EV_ALREADY 5   /* at the target before the first trial */
#define PHMC_GC_STOP_REACHED 1
#define PHMC_GC_STOP_NO_PAIRS 2
#define PHMC_GC_STOP_MAX_TRIALS 3
#define PHMC_GC_STOP_ALREADY 4
typedef struct phmc_gc_event {
    int kind;                   /* PHMC_GC_EV_* */
    int epoch;                  /* 0-based epoch */
    int step_in_block;          /* REACHED: trials of the current block so far, this one included */
    int acc_since_mu, att_since_mu;
    int block_accepted, block_attempted;
    int nprot, remaining;       /* protonated sites; max(0, target - nprot) */
    int cause_amax;             /* MU: 1 the epoch hit the attempt limit short of the accept target, else 0 */
    int64_t fwd_total, bwd_total;
    float mu_kT;                /* beta mu_eff (MU: after the update) */
    float f, w_info;            /* MU: protonated fraction, weight of the update */
    float E;                    /* REACHED, ALREADY: the phase's energy */
    float acc_rate;             /* CHUNK: block_accepted / block_attempted */
} phmc_gc_event;
typedef struct phmc_gc_job {
    int replica;
    int nh_n_type, nh_p_type, w_type, cl_type; /* engine types (0-based) */
    float q_nh_p, q_cl;                        /* charges given to NH_P and Cl (the reference: +1, -1) */
    double beta;                               /* 1 / kT */
    double target_pct;                         /* target_protonation_pct */
    double mu_eta;                             /* <= 0: 0.3 */
    double nacc_frac;                          /* sgmc_nacc_frac_round, <= 0: 0.10 */
    int gc_block;                              /* gc_block_fixed, <= 0: 2000 */
    int epoch_attempt_max;                     /* sgmc_epoch_attempt_max, <= 0: 100000 */
    int64_t max_trials;                        /* this call's trials at most (<= 0: 10^9); the reference has no bound */
    const int* nh_n; int n_nh_n;               /* pools in the reference's order (slot indices) */
    const int* nh_p; int n_nh_p;
    const int* w; int n_w;
    const int* cl; int n_cl;
    uint32_t* mt_state;                        /* in / out: the caller's generator, 625 words */
    /* Fixed-mu sampling (no counterpart in the reference, whose loop always steers mu
     * to its target): with fixed_mu != 0, mu stays at mu_kT / beta (e.g. kT ln10
     * (pKa - pH) for constant-pH sampling of a weak base), there is no mu feedback
     * and no target stop; the call ends after max_trials attempts. */
    int fixed_mu;
    double mu_kT;
} phmc_gc_job;
typedef struct phmc_gc_result {
    int attempted, accepted, accepted_forward, accepted_backward, blocks_done;
    int Nh, Nprot, target_count, reached_target;
    int stop;                                  /* PHMC_GC_STOP_* */
    float E, mu_eff;                           /* the phase's last energy and mu (the reference's real) */
    int R0, Nacc_target, epoch_attempt_max, gc_block; /* settings derived as the reference derives them */
    int n_events, events_dropped;              /* events stored for this job / beyond event_cap */
} phmc_gc_result;
/* events: n_jobs x event_cap records (job k at k * event_cap), or null. */
int phmc_gc_phase(phmc_engine* e, int n_jobs, const phmc_gc_job* jobs, phmc_gc_result* results,
                  phmc_gc_event* events, int event_cap);
/* Streaming of the phases' event records (no counterpart in the reference, whose
 * loops write their report lines as they go): after each MC launch of
 * phmc_gc_phase / phmc_phase2 (and for the records made before the first one)
 * the engine calls fn(user, job, phase, record) for every new record of every
 * job, in order, before the call returns, so a phase that runs long or never
 * reaches its target still reports as it runs.  phase 1: record is a
 * phmc_gc_event, and results[job] of the running call already holds the set-up
 * fields Nh, target_count, R0, Nacc_target, epoch_attempt_max and gc_block;
 * phase 2: a phmc_phase2_event.  Records are also stored in the call's event
 * arrays as before.  fn = NULL switches streaming off. */
typedef void (*phmc_event_fn)(void* user, int job, int phase, const void* record);
int phmc_set_event_callback(phmc_engine* e, phmc_event_fn fn, void* user);

/* ---- the reference's phase 2 (swap / jitter with patience) on the device ----
 * Replaces phase2_swap_jitter (MC/include/mc.hpp:62-71, MC/src/mc.cu:159-318):
 * four-point moves NH_P -> NH_N, NH_N -> NH_P, Cl -> W, W -> Cl (or, with no
 * NH_N left or no four-point move possible, the Cl/W pair alone), plain
 * Metropolis on the reference's float energies, a report line every
 * energy_interval attempts, and a stop after patience attempts without a new
 * best energy or after max_attempts.  A four-point move runs as two
 * two-atom evaluations (the NH half applied, the Cl/W half judged with it in
 * place; a rejection restores the NH half), so its energy change is the
 * four-atom one.  The caller's generator, pools and event records work as for
 * phmc_gc_phase; the W and Cl pools are the ones the reference keeps (below
 * z_cut), z_cut itself only enters the pools line.  Needs the engine's
 * pending_max >= 6 (PHMC_ERR_UNSUPPORTED otherwise). */
#define PHMC_P2_EV_POOLS 11         /* the pool sizes before the first attempt */
#define PHMC_P2_EV_NONE_AT_START 12 /* neither a four-point nor a Cl/W move possible: the phase ends */
#define PHMC_P2_EV_WC_EMPTY 13      /* Cl/W moves wanted, their pools empty: the phase ends */
#define PHMC_P2_EV_NONE 14          /* no valid proposal at an attempt: the phase ends */
#define PHMC_P2_EV_STEP 15          /* every energy_interval attempts */
#define PHMC_P2_EV_PATIENCE 16      /* patience reached: the phase ends */
#define PHMC_P2_STOP_PATIENCE 1
#define PHMC_P2_STOP_MAX_ATTEMPTS 2
#define PHMC_P2_STOP_NO_PROPOSALS 3
typedef struct phmc_phase2_event {
    int kind;                   /* PHMC_P2_EV_* */
    int attempted, accepted;    /* STEP */
    int since_best, patience;   /* STEP, PATIENCE */
    int mode_wc;                /* STEP: 1 the last attempt was a Cl/W move, 0 a four-point move */
    int n_nh_p, n_nh_n, n_cl, n_w;  /* POOLS */
    float E, acc;               /* STEP: the phase's energy, accepted / attempted */
    float z_cut;                /* POOLS */
    int pad;
} phmc_phase2_event;
typedef struct phmc_phase2_job {
    int replica;
    int nh_n_type, nh_p_type, w_type, cl_type; /* engine types (0-based) */
    float q_nh_p, q_cl;                        /* charges given to NH_P and Cl (the reference: +1, -1) */
    double beta;
    int max_attempts, patience, energy_interval;
    float z_cut;                               /* reported with the pools */
    const int* nh_p; int n_nh_p;               /* pools in the reference's order (slot indices) */
    const int* nh_n; int n_nh_n;
    const int* w; int n_w;                     /* W below z_cut */
    const int* cl; int n_cl;                   /* Cl below z_cut */
    uint32_t* mt_state;                        /* in / out: the caller's generator, 625 words */
} phmc_phase2_job;
typedef struct phmc_phase2_result {
    int attempted, accepted;
    float E, best_E;                           /* the reference's real */
    int stop;                                  /* PHMC_P2_STOP_* (0: ended before the first attempt) */
    int since_best;
    int n_events, events_dropped;
} phmc_phase2_result;
int phmc_phase2(phmc_engine* e, int n_jobs, const phmc_phase2_job* jobs, phmc_phase2_result* results,
                phmc_phase2_event* events, int event_cap);
/* The reference's report line of a phase-2 event (MC/src/mc.cu:191-208, 219, 296-308,
 * 310-312), fixed notation, precision 6 where the reference's stream carries no
 * precision of its own, without the newline; returns the length. */
int phmc_phase2_event_format(const phmc_phase2_event* ev, char* buf, int cap);
/* The reference's report.txt line of an event (MC/src/mc.cu:367-373, 377, 461-474,
 * 506-516, 532-545), fixed notation at its precision 6, without the newline.
 * Returns the line's length (the line is cut at cap - 1 characters). */
int phmc_gc_event_format(const phmc_gc_event* ev, const phmc_gc_result* res, char* buf, int cap);

#ifdef __cplusplus
}
#endif
#endif /* PHMC_H */
