// Shared device-side definitions of the phmc engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/phmc.h"
#include "surrogate.cuh"

#define PHMC_MAX_TYPES 8
#define PHMC_MAX_ORDER 6
#define PHMC_MAX_PEND 128
#define PHMC_FIX_SCALE 1099511627776.0   /* 2^40: fixed-point scale of the charge mesh */
#define PHMC_FIX_INV (1.0 / 1099511627776.0)

#include "mt_std.cuh"

// State of one job of the grand-canonical mu-control phase (MC/src/mc.cu:320-548),
// carried across MC-kernel launches; the reference's `real` quantities are floats.
enum { GC_NHN = 0, GC_NHP = 1, GC_W = 2, GC_CL = 3 };
struct GcDev {
    MtState mt;              // the reference's generator
    int replica;
    int type[4];             // engine types of NH_N, NH_P, W, Cl
    float q_nhp, q_cl;
    float beta, eta, f0;     // 1/kT, mu step factor, clamped target fraction
    float mu;                // mu_eff
    float E;                 // the phase's energy as the reference tracks it (R.E)
    int Nh, Nprot, target, gc_block, amax, nacc_target;
    int n[4];                // pool sizes
    int attempted, accepted, fwd, bwd;
    int epoch, block_t, block_att, block_acc, acc_mu, att_mu, blocks_done;
    int max_trials;          // bound on attempted trials of the call
    int launch_cap;          // trials per launch at most
    int stop;                // PHMC_GC_STOP_* once the phase ended
    int n_ev, ev_cap;        // events of the current launch
    // the trial in flight
    int dir;                 // +1 forward, -1 backward
    long long s_before, s_after;
    // phase 2 (MC/src/mc.cu:159-318): phase 1 = grand-canonical mu control, 2 = swaps with patience
    int phase;
    int role;                // 0 next attempt, 1 NH half of a four-point move (applied), 2 judged move, 3 NH half restored
    int four;                // the current attempt is a four-point move
    int prefer_wc;
    int max_attempts, patience, energy_interval, since_best;
    float best_E;
    int iP, iN, jCl, jW;     // the attempt's atoms
    int o_type[2];           // identities of iP, iN before the attempt
    float o_q[2];
    int stop_after_restore;  // phase ends once the NH half is restored
    int fixed;               // mu held fixed: no feedback, no target stop
};

// Per-replica constant description (the ragged descriptor table).
struct RepDesc {
    // particles
    int cap, slot_off;
    float L[3];
    double V;
    // cells
    int ncell[3], cell_off, cell_cap;
    float cell_scale[3];  // ncell / L (float), cell = (int)(x * scale)
    // mesh
    int mesh[3];
    long long mesh_off;   // offset (elements) into real / complex mesh arrays
    int oct[3];           // G octant dims (n/2+1)
    long long oct_off;
    int mod_off[3];       // offsets of the B-spline moduli per axis
    int tw_off[3];        // offsets of the twiddle tables per axis
    int tw_off_h;         // twiddle table of length nx/2 (real-to-complex path)
    int th_off[3];        // per-axis influence factors (exp(-(pi/alpha)^2 k^2) / B(k), k^2) in thtab
    float th_c;           // elf / (pi V): theta(k) = th_c tx ty tz / |k|^2
    long long meshh_off;  // offset into the half-spectrum complex mesh ((nx/2+1) x ny x nz)
    long long qb_off;     // offset of this replica's fixed-point charge mesh (nx x ny x zb_n) in qband
    int zb_lo, zb_n;      // band of planes (zb_lo + i) mod nz, i < zb_n, that the walls let hold charge (all without walls)
    int order;
    int coulomb;
    int ref_corner;
    int slab;
    float alpha, elf, rc_coul2;
    float ewald_factor;   // (pi/alpha)^2
    // walls, bonds
    int walls;
    float wall_lo, wall_hi;
    float fene_k, fene_r02;
    int excl_lj, excl_coul;
    // LJ tables (T <= 8)
    int T;
    float lj_eps[PHMC_MAX_TYPES * PHMC_MAX_TYPES];
    float lj_sig2[PHMC_MAX_TYPES * PHMC_MAX_TYPES];
    float lj_rc2[PHMC_MAX_TYPES * PHMC_MAX_TYPES];
    float lj_shift[PHMC_MAX_TYPES * PHMC_MAX_TYPES];
    // moves
    double beta, titr_log;   // titr_log = ln10 * (pKa - pH)
    double salt_c2V2;        // c_s^2 * V_slab^2
    float p_disp, p_titr, p_swap, disp_max;
    int type_site_neutral, type_site_charged, type_counterion, type_cation;
    float q_site_charged, q_counterion, q_cation;
    uint32_t key[2];
    int n_titr;
    int pend_max;
    // Ewald scalar coefficients
    double self_coef;   // -elf * alpha / sqrt(pi)
    double qcorr_coef;  // -pi * elf / (2 V alpha^2)
    double slab_coef;   // 2 pi elf / V
    double Lz2_12;      // Lz^2 / 12
    // surrogate descriptor
    float cell_w[3];      // cell widths L / ncell (float)
    int dnr[3];           // cell window of the 8-sigma descriptor sphere: offsets -dnr .. -dnr + dnk - 1,
    int dnk[3];           // dnk = min(2 r + 1, ncell) for the range r; dnr = r, or (dnk - 1) / 2 when dnk == ncell
    float sur_z0, sur_h;  // z feature = (z - sur_z0) / sur_h
    float sur_pk, sur_salt;  // pKa - pH, log10(salt) features
};

// Per-replica mutable state (device-resident between launches).
struct RepState {
    int n_mobile, n_anion, n_cation, n_free;
    int error;          // PHMC_ERR_* raised inside a kernel (0 = none)
    int stop_reason;    // 0 target reached, 1 pending full, 2 launch quorum of blocked replicas reached
    long long trial;    // next trial index (Philox counter)
    long long target;   // run until trial == target
    long long run_start; // trial index at the start of the current phmc_run (log / replay origin)
    long long att[3], acc[3];
    long long flushes;
    double E;           // tracked total energy
    double E_pair_lj, E_pair_c, E_fene, E_rec, E_self, E_qcorr, E_slab;  // tracked components
    double Q, Q2, Mz, S2;  // charge moments
    double drift;       // |tracked E_rec - recomputed| at the last flush
    double E_rec_flush; // E_rec computed at the last flush
    double alg_bytes;   // algorithmic bytes of the trials run so far
    long long trials_run;
    // delayed acceptance: trials judged by the surrogate, first-stage passes,
    // second-stage accepts; the same over the current agreement window
    long long da_eval, da_pass, da_acc, da_wpass, da_wacc;
    int da_off;         // agreement fell below the threshold: plain Metropolis from then on
    int da_pad;
    long long busy_ns;  // summed run time of this replica's MC blocks (globaltimer)
    // with phase clocks on (phmc_set_phase_clock): SM cycles of the MC kernel's phases,
    // measured by the block's thread 0 at the block barriers that end them (PHMC_PHASES)
    long long clk[8];
};

// Device pointers of the whole engine (all replicas concatenated).
struct DevPtrs {
    float4* posq;       // x, y, z, q
    int* type;
    int* flags;
    int4* bonds;        // up to 4 partners (local slot index), -1 = none
    int* cell_of;       // -1 for ghosts
    int* cell_pos;
    int* cell_count;
    int* cell_list;     // cell_off*cell_cap + c*cell_cap + k (local slot)
    int* mobile; int* mobile_pos;
    int* anions; int* anion_pos;
    int* cations; int* cation_pos;
    int* freel;
    int* titr;
    unsigned long long* qfix;  // fixed-point charge mesh
    unsigned long long* qband; // fixed-point charge mesh of the wall band, kept current by the MC kernel (even nx)
    float2* cmesh;             // complex work mesh
    float* phi;                // potential mesh (real)
    float* goct;               // influence kernel octant
    float* moduli;
    float2* twiddle;
    float2* thtab;             // per-axis influence factors of the rebuild's z pass
    RepDesc* desc;
    RepState* state;
    double* partials;          // reduction scratch
    int* dirty;                // per replica: potential mesh stale
    // trial log / replay (replica 0)
    int* log_move; double* log_dE; int* log_acc; long long log_cap;
    const int* replay; long long replay_n;
    int* log_stage; double* log_dEs;  // delayed-acceptance log (replica 0): stage reached, surrogate dE
    // per cell: present particles of each descriptor class (+1, -1, neutral titratable, permanent)
    int4* cell_cls;
    // delayed acceptance
    SurDev sur;
    int sur_late_l3;     // two-buffer staging (layer 3 copied after layer 1) to keep two MC blocks per SM
    int* quorum_ctl;     // [replicas active at the MC launch's start, of them stopped by a full pending buffer]
    float quorum;        // the launch ends once that fraction of its active replicas is blocked (>= 1: off)
    float da_threshold;  // minimum second-stage acceptance among first-stage passes
    int da_window;       // first-stage passes per agreement check
    // training-sample harvest: rows [cap][SUR_ROWS][SUR_K], signs [cap][SUR_ROWS], targets [cap]
    float* hv_rows; float* hv_sign; float* hv_target; int* hv_count; int hv_cap;
    // descriptor output of MC_DESCRIBE launches (DSC_STRIDE floats per trial)
    float* dsc_out;
    // per external trial dE components (lj, fene, coul_real, coul_recip, self, qcorr, slab), or null
    double* ext_comp;
    // grand-canonical mu-control phase: per job state, pools (4 x total slots: NH_N, NH_P, W,
    // Cl of each replica at its slot offset) and event records (ev_cap per job)
    struct GcDev* gc;
    int* gc_pool;
    int gc_pool_stride;
    unsigned char* gc_ev;  // event records of either phase (phmc_gc_event / phmc_phase2_event)
    // z-density profiles (phmc_set_zhist): after every zh_every trials each replica's MC
    // block adds its histogram over z (zh_bins bins between the walls) of charged sites,
    // anions and cations to zhist[r][3][zh_bins] and counts the sample in zh_samples[r]
    int phase_clk;      // MC kernel: accumulate RepState::clk (one extra barrier per trial)
    int zh_bins;
    long long zh_every;
    unsigned long long* zhist;
    long long* zh_samples;
};

#define DSC_STRIDE (SUR_ROWS * SUR_K + 2 * SUR_ROWS + 4)

// Descriptor class of a present particle (-1: none).
__host__ __device__ inline int desc_class(int flags, float q) {
    if (flags & PHMC_F_GHOST) return -1;
    if (flags & PHMC_F_TITRATABLE) return q != 0.0f ? 0 : 2;
    if (q < 0.0f) return 1;
    if (q > 0.0f) return (flags & PHMC_F_CATION) ? 0 : 3;  // salt cation, or a permanently charged bead
    return -1;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11), written from the paper's definition.
// ---------------------------------------------------------------------------
__host__ __device__ inline void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                                              uint32_t c2, uint32_t c3, uint32_t out[4]) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ inline float u24(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }
__host__ __device__ inline double u53(uint32_t a, uint32_t b) {
    uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
    return (double)(v & ((1ull << 53) - 1)) * (1.0 / 9007199254740992.0);
}
__host__ __device__ inline int pick_index(uint32_t v, int n) { return (int)(((uint64_t)v * (uint64_t)n) >> 32); }

// Cardinal B-spline weights of order P at fractional offset t (see the
// spreading convention: point base + j gets M_P(t + P-1-j)).
template <int P>
__device__ __forceinline__ void bspline_weights(float t, float* w) {
    float c[P];
    c[0] = t; c[1] = 1.0f - t;
#pragma unroll
    for (int n = 3; n <= P; ++n) {
        const float inv = 1.0f / (float)(n - 1);
        float nc[P];
#pragma unroll
        for (int i = 0; i < n; ++i) {
            float a = (i < n - 1) ? c[i] : 0.0f;
            float b = (i >= 1) ? c[i - 1] : 0.0f;
            nc[i] = ((t + (float)i) * a + ((float)n - t - (float)i) * b) * inv;
        }
#pragma unroll
        for (int i = 0; i < n; ++i) c[i] = nc[i];
    }
#pragma unroll
    for (int j = 0; j < P; ++j) w[j] = c[P - 1 - j];
}

// The fixed-point charge mesh: stencil of a charge and its integer value per mesh
// point, every operation rounded as written (no contraction), so that the MC
// kernel's incremental updates and the full spread give the same integers.
template <int P>
__device__ __forceinline__ void qmesh_stencil(const RepDesc& D, float4 pq, float (&w)[3][P], int (&base)[3]) {
    const float p3[3] = {pq.x, pq.y, pq.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float g = __fmul_rn(__fdiv_rn(p3[k], D.L[k]), (float)D.mesh[k]);
        const float fl = floorf(g);
        const float t = __fsub_rn(g, fl);
        float c[P];
        c[0] = t; c[1] = __fsub_rn(1.0f, t);
#pragma unroll
        for (int n = 3; n <= P; ++n) {
            const float inv = 1.0f / (float)(n - 1);
            float nc[P];
#pragma unroll
            for (int i = 0; i < n; ++i) {
                const float a = (i < n - 1) ? c[i] : 0.0f;
                const float b = (i >= 1) ? c[i - 1] : 0.0f;
                const float ta = __fmul_rn(__fadd_rn(t, (float)i), a);
                const float tb = __fmul_rn(__fsub_rn(__fsub_rn((float)n, t), (float)i), b);
                nc[i] = __fmul_rn(__fadd_rn(ta, tb), inv);
            }
#pragma unroll
            for (int i = 0; i < n; ++i) c[i] = nc[i];
        }
#pragma unroll
        for (int j = 0; j < P; ++j) w[k][j] = c[P - 1 - j];
        base[k] = (int)fl + P / 2 - P + 1;
    }
}
// q wx wy wz in units of 2^-40 (q wy wz first, as a plane's row weight)
__device__ __forceinline__ long long qmesh_value(float q, float wx, float wy, float wz) {
    return __float2ll_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(q, wy), wz), wx), 1099511627776.0f));
}

__device__ __forceinline__ float min_image(float d, float L) { return d - L * rintf(d / L); }

__device__ __forceinline__ int wrap_idx(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Pair energy between two present particles (FP32), split into LJ and Coulomb.
// `bonded` applies the 1-2 exclusion policy.
__device__ __forceinline__ void pair_energy(const RepDesc& D, float dx, float dy, float dz, int ti, int tj,
                                            float qi, float qj, bool bonded, float& elj, float& ec) {
    const float r2 = dx * dx + dy * dy + dz * dz;
    const int p = ti * D.T + tj;
    elj = 0.0f; ec = 0.0f;
    if (!(bonded && D.excl_lj) && r2 <= D.lj_rc2[p] && D.lj_eps[p] > 0.0f) {
        float s2 = D.lj_sig2[p] / r2;
        float s6 = s2 * s2 * s2;
        elj = 4.0f * D.lj_eps[p] * (s6 * s6 - s6) - D.lj_shift[p];
    }
    if (D.coulomb != PHMC_COUL_NONE && !(bonded && D.excl_coul) && r2 <= D.rc_coul2) {
        float qq = qi * qj;
        if (qq != 0.0f) {
            float r = sqrtf(r2);
            ec = (D.coulomb == PHMC_COUL_EWALD) ? D.elf * qq * erfcf(D.alpha * r) / r : D.elf * qq / r;
        }
    }
}

__device__ __forceinline__ bool in_bonds(int4 b, int j) { return b.x == j || b.y == j || b.z == j || b.w == j; }

__device__ __forceinline__ int cell_index(const RepDesc& D, float x, float y, float z) {
    int a = min(D.ncell[0] - 1, max(0, (int)(x * D.cell_scale[0])));
    int b = min(D.ncell[1] - 1, max(0, (int)(y * D.cell_scale[1])));
    int c = min(D.ncell[2] - 1, max(0, (int)(z * D.cell_scale[2])));
    return (c * D.ncell[1] + b) * D.ncell[0] + a;
}

// FENE bond energy (FP32 term); returns +inf beyond R0.
__device__ __forceinline__ float fene_energy(const RepDesc& D, float r2) {
    if (r2 >= D.fene_r02) return __int_as_float(0x7f800000);
    return -0.5f * D.fene_k * D.fene_r02 * logf(1.0f - r2 / D.fene_r02);
}

// Block-wide FP64 sum (all threads get the result).  `red` holds >= 32 doubles.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = (l < NT / 32) ? red[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (l == 0) red[32] = s;
    }
    __syncthreads();
    return red[32];
}
