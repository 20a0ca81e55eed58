// Persistent Monte Carlo kernel: one thread block per replica runs trials
// back to back until its trial target is reached or its pending-stencil
// buffer is full (the potential mesh is then rebuilt by the mesh kernels).
//
// Per trial (replaces total_energy per trial, MC/src/mc.cu:43-60,241,275,425):
//  * proposal from a counter-based Philox stream (trial index = counter), so a
//    trial is reproducible and replayable;
//  * pair dE (LJ/WCA + real-space Coulomb) over the 27 neighbour cells of
//    every changed particle's old and new state, FP32 terms, FP64 sums;
//  * FENE dE of displaced bonded beads, wall test;
//  * reciprocal dE = sum_t c_t [W_t . phi + sum_e c_e S(W_t, W_e)]
//                    + 1/2 sum_{t,t'} c_t c_t' S(W_t, W_t'),
//    phi the potential mesh of the last rebuild, W_e the stencils of changes
//    accepted since then, S(W_a, W_b) = sum_delta G[D + delta] Kx Ky Kz with
//    K the 1-D cross-correlations of the two stencils' weights and G the
//    influence kernel (octant table);
//  * self / net-charge / slab terms from FP64 charge moments;
//  * Metropolis in FP64 with the move's log factor (MC/src/mc.cu:438-440).
#include <algorithm>
#include <type_traits>
#include "common.cuh"
#include "engine.h"
#include "fft.cuh"

#define NST_MAX 4    // stencils per trial
static_assert(NST_MAX <= 4, "the pair tables count a pending pair's trial stencil by three comparisons");
#define NPROBE_MAX 4 // (old, new) states of up to two particles
#define LIST_PF 16   // leading cell-list entries of each probe cell loaded with its count
#define CAND_MAP 4096 // candidates whose probe-cell entry is tabulated in phase 3

template <int P>
struct Stencil {
    int base[3];
    int m[3][P];   // wrapped mesh coordinates
    float w[3][P];
    float coef;
};

template <int P>
struct PairK {
    float K[3][2 * P - 1];
    int f[3][2 * P - 1];  // folded octant coordinate of D + delta
    float coef;
    int pad;
    // (row offsets and coef * Ky * Kz are recomputed where they are used: 224 bytes per
    // pair at order 5 keep two MC blocks per SM up to ~100 pending stencils)
};

struct TrialS {
    int stop, skip, move, nch, accept, nprobe, nst, ext_k;
    double logf;
    uint32_t ua, ub;
    long long tnum;
    int idx[2], pres_old[2], pres_new[2], to[2], tn[2];
    float4 po[2], pn[2];
    int4 bonds[2];
    float4 probe_p[NPROBE_MAX];
    int probe_t[NPROBE_MAX], probe_owner[NPROBE_MAX], probe_cell[NPROBE_MAX];
    float probe_sign[NPROBE_MAX];
    float4 st_pos[NST_MAX];
    float st_coef[NST_MAX];
    double d_direct_lj, d_direct_c, d_fene;
    int total_cand, npairs;
    // cell bookkeeping of the old states, loaded off the critical path (phase 4)
    int cell_old[2], cpos_old[2], cnt_old[2], last_old[2];
    int fo[2];  // slot flags of the changed particles before the trial
    // surrogate first stage
    int desc, da, nrows, dtotal;
    int row_k[SUR_ROWS], row_cls[SUR_ROWS];
    float row_sign[SUR_ROWS];
    float4 dpos[2];            // descriptor centres (new position if present, else old)
    int dcx[2], dcy[2], dcz[2];
    int ccell[2], ccls[2];     // current cell / class of the changed particles (-1: absent)
    double cross, dmom, dEs;   // exact cross and charge-moment terms, surrogate dE
};

// Next trial's primary particle, loaded during the current trial's parallel
// phase.  Valid while no accepted change touched it or the lists.
struct Prefetch {
    long long t;
    int valid, move, idx, flags, type;
    float4 pq;
    int4 bonds;
};

// Fill probes and stencils from the changes in T (old -> new states).
// (The trial's fields are read once into registers and the counters kept in registers:
// one thread runs this while the block waits, so its shared-memory round trips count.)
__device__ void trial_setup(TrialS& T, const RepDesc& D) {
    const int nch = T.nch;
    const bool ewald = D.coulomb == PHMC_COUL_EWALD;
    int np = 0, ns = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (k >= nch) break;
        const bool pold = T.pres_old[k], pnew = T.pres_new[k];
        const float4 o = T.po[k], n = T.pn[k];
        const int to = T.to[k], tn = T.tn[k];
        if (pold) {
            T.probe_p[np] = o; T.probe_t[np] = to; T.probe_owner[np] = k; T.probe_sign[np] = -1.0f;
            T.probe_cell[np] = cell_index(D, o.x, o.y, o.z);
            ++np;
        }
        if (pnew) {
            T.probe_p[np] = n; T.probe_t[np] = tn; T.probe_owner[np] = k; T.probe_sign[np] = 1.0f;
            T.probe_cell[np] = cell_index(D, n.x, n.y, n.z);
            ++np;
        }
        if (ewald) {
            const bool same_pos = pold && pnew && o.x == n.x && o.y == n.y && o.z == n.z;
            if (same_pos) {
                const float c = n.w - o.w;
                if (c != 0.0f) { T.st_pos[ns] = n; T.st_coef[ns] = c; ++ns; }
            } else {
                if (pold && o.w != 0.0f) { T.st_pos[ns] = o; T.st_coef[ns] = -o.w; ++ns; }
                if (pnew && n.w != 0.0f) { T.st_pos[ns] = n; T.st_coef[ns] = n.w; ++ns; }
            }
        }
    }
    T.nprobe = np; T.nst = ns;
}

__device__ __forceinline__ float4 rand_pos(const RepDesc& D, uint32_t a, uint32_t b, uint32_t c) {
    float4 p;
    p.x = __fmul_rn(D.L[0], u24(a));
    p.y = __fmul_rn(D.L[1], u24(b));
    p.z = D.walls ? __fadd_rn(D.wall_lo, __fmul_rn(__fsub_rn(D.wall_hi, D.wall_lo), u24(c))) : __fmul_rn(D.L[2], u24(c));
    p.w = 0.0f;
    return p;
}

// The 16 Philox words of trial t: A = ctr (t, 0), B = ctr (t, 1), C = ctr (t, 2),
// and ctr (t, 3), whose first two words are the delayed-acceptance first-stage uniform.
__device__ __forceinline__ void trial_words(const RepDesc& D, long long t, uint32_t* w) {
    const uint32_t lo = (uint32_t)t, hi = (uint32_t)((unsigned long long)t >> 32);
    philox4x32_10(D.key[0], D.key[1], lo, hi, 0u, 0u, w);
    philox4x32_10(D.key[0], D.key[1], lo, hi, 1u, 0u, w + 4);
    philox4x32_10(D.key[0], D.key[1], lo, hi, 2u, 0u, w + 8);
    philox4x32_10(D.key[0], D.key[1], lo, hi, 3u, 0u, w + 12);
}

__device__ __forceinline__ int move_of(const RepDesc& D, uint32_t a0) {
    const float um = u24(a0);
    if (um < D.p_disp) return PHMC_MOVE_DISP;
    if (um < D.p_disp + D.p_titr) return PHMC_MOVE_TITR;
    if (um < D.p_disp + D.p_titr + D.p_swap) return PHMC_MOVE_SWAP;
    return PHMC_MOVE_NONE;
}

// Load the primary particle of trial t into pf (list index from the current sizes).
__device__ void prefetch_primary(Prefetch& pf, long long t, const uint32_t* rw, const RepDesc& D, const RepState& S,
                                 const DevPtrs& d) {
    pf.valid = 0;
    const int mv = move_of(D, rw[0]);
    const int so = D.slot_off;
    int i = -1;
    if (mv == PHMC_MOVE_DISP && S.n_mobile > 0) i = d.mobile[so + pick_index(rw[1], S.n_mobile)];
    else if (mv == PHMC_MOVE_TITR && D.n_titr > 0) i = d.titr[so + pick_index(rw[1], D.n_titr)];
    if (i < 0) return;
    pf.t = t; pf.move = mv; pf.idx = i;
    pf.flags = d.flags[so + i]; pf.pq = d.posq[so + i]; pf.type = d.type[so + i]; pf.bonds = d.bonds[so + i];
    pf.valid = 1;
}

// Proposal of trial T.tnum from its Philox words (same rules as the oracle's MC).
__device__ void propose(TrialS& T, const RepDesc& D, const RepState& S, const DevPtrs& d, const uint32_t* rw,
                        const Prefetch& pf) {
    const uint32_t* A = rw;
    const uint32_t* B = rw + 4;
    const uint32_t* C = rw + 8;
    T.ua = B[2]; T.ub = B[3];
    const int move = move_of(D, A[0]);
    T.move = move; T.skip = 0; T.nch = 0; T.logf = 0.0;
    const int so = D.slot_off;
    auto load_old = [&](int k, int i) {
        T.idx[k] = i;
        const int fl = d.flags[so + i];
        T.fo[k] = fl;
        T.pres_old[k] = !(fl & PHMC_F_GHOST);
        T.po[k] = d.posq[so + i]; T.to[k] = d.type[so + i]; T.bonds[k] = d.bonds[so + i];
    };
    // primary particle from the prefetch when it is still valid
    const bool use_pf = pf.valid && pf.t == T.tnum && pf.move == move;
    auto load_primary = [&](int i_from_list) {
        if (use_pf) {
            T.idx[0] = pf.idx; T.fo[0] = pf.flags; T.pres_old[0] = !(pf.flags & PHMC_F_GHOST);
            T.po[0] = pf.pq; T.to[0] = pf.type; T.bonds[0] = pf.bonds;
        } else {
            load_old(0, i_from_list);
        }
    };
    if (move == PHMC_MOVE_DISP) {
        if (S.n_mobile == 0) { T.skip = 1; return; }
        float4 po;
        int to;
        if (use_pf) {  // the prefetched particle, kept in registers for the new position
            po = pf.pq; to = pf.type;
            T.idx[0] = pf.idx; T.fo[0] = pf.flags; T.pres_old[0] = !(pf.flags & PHMC_F_GHOST);
            T.po[0] = po; T.to[0] = to; T.bonds[0] = pf.bonds;
        } else {
            load_old(0, d.mobile[so + pick_index(A[1], S.n_mobile)]);
            po = T.po[0]; to = T.to[0];
        }
        const float dm = D.disp_max;
        const float dx = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(A[2])), 1.0f));
        const float dy = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(A[3])), 1.0f));
        const float dz = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(B[0])), 1.0f));
        const float Lx = D.L[0], Ly = D.L[1], Lz = D.L[2];
        float nx = __fadd_rn(po.x, dx), ny = __fadd_rn(po.y, dy), nz = __fadd_rn(po.z, dz);
        if (nx < 0.0f) nx = __fadd_rn(nx, Lx); else if (nx >= Lx) nx = __fsub_rn(nx, Lx);
        if (ny < 0.0f) ny = __fadd_rn(ny, Ly); else if (ny >= Ly) ny = __fsub_rn(ny, Ly);
        const int walls = D.walls;
        if (!walls) { if (nz < 0.0f) nz = __fadd_rn(nz, Lz); else if (nz >= Lz) nz = __fsub_rn(nz, Lz); }
        T.pres_new[0] = 1; T.pn[0] = make_float4(nx, ny, nz, po.w); T.tn[0] = to;
        T.nch = 1;
        if (walls && (nz < D.wall_lo || nz >= D.wall_hi)) T.skip = 2;  // hard wall: infinite energy
    } else if (move == PHMC_MOVE_TITR) {
        if (D.n_titr == 0) { T.skip = 1; return; }
        load_primary(use_pf ? -1 : d.titr[so + pick_index(A[1], D.n_titr)]);
        T.pres_new[0] = 1;
        if (T.po[0].w == 0.0f) {
            if (S.n_free == 0) { T.skip = 1; return; }
            const int g = d.freel[so + S.n_free - 1];
            load_old(1, g);
            T.pn[0] = make_float4(T.po[0].x, T.po[0].y, T.po[0].z, D.q_site_charged); T.tn[0] = D.type_site_charged;
            float4 pg = rand_pos(D, A[2], A[3], B[0]); pg.w = D.q_counterion;
            T.pres_new[1] = 1; T.pn[1] = pg; T.tn[1] = D.type_counterion;
            T.logf = D.titr_log;
        } else {
            if (S.n_anion == 0) { T.skip = 1; return; }
            const int g = d.anions[so + pick_index(B[1], S.n_anion)];
            load_old(1, g);
            T.pn[0] = make_float4(T.po[0].x, T.po[0].y, T.po[0].z, 0.0f); T.tn[0] = D.type_site_neutral;
            T.pres_new[1] = 0; T.pn[1] = T.po[1]; T.tn[1] = T.to[1];
            T.logf = -D.titr_log;
        }
        T.nch = 2;
    } else if (move == PHMC_MOVE_SWAP) {
        if (u24(A[1]) < 0.5f) {
            if (S.n_free < 2) { T.skip = 1; return; }
            const int g1 = d.freel[so + S.n_free - 1], g2 = d.freel[so + S.n_free - 2];
            load_old(0, g1); load_old(1, g2);
            float4 p1 = rand_pos(D, A[2], A[3], B[0]); p1.w = D.q_cation;
            float4 p2 = rand_pos(D, C[0], C[1], C[2]); p2.w = D.q_counterion;
            T.pres_new[0] = 1; T.pn[0] = p1; T.tn[0] = D.type_cation;
            T.pres_new[1] = 1; T.pn[1] = p2; T.tn[1] = D.type_counterion;
            T.logf = log(D.salt_c2V2 / ((double)(S.n_cation + 1) * (double)(S.n_anion + 1)));
        } else {
            if (S.n_cation == 0 || S.n_anion == 0) { T.skip = 1; return; }
            const int g1 = d.cations[so + pick_index(B[1], S.n_cation)];
            const int g2 = d.anions[so + pick_index(C[3], S.n_anion)];
            load_old(0, g1); load_old(1, g2);
            T.pres_new[0] = 0; T.pn[0] = T.po[0]; T.tn[0] = T.to[0];
            T.pres_new[1] = 0; T.pn[1] = T.po[1]; T.tn[1] = T.to[1];
            T.logf = log((double)S.n_cation * (double)S.n_anion / D.salt_c2V2);
        }
        T.nch = 2;
    } else {
        T.skip = 3;  // no-op draw
    }
}

// Displacement of the prefetched particle: propose() and trial_setup() for that case,
// computed in registers from the prefetch and the trial's words and stored to the trial
// once (the general path reads back, through shared memory, fields it has just written;
// one thread runs this while the block waits).  Same values, field for field.
__device__ __forceinline__ void propose_disp_setup(TrialS& T, const RepDesc& D, const Prefetch& pf, const uint32_t* rw) {
    const uint32_t* A = rw;
    const uint32_t* B = rw + 4;
    const float4 po = pf.pq;
    const int to = pf.type, fl = pf.flags;
    const bool pold = !(fl & PHMC_F_GHOST);
    const float dm = D.disp_max;
    const float Lx = D.L[0], Ly = D.L[1], Lz = D.L[2];
    const int walls = D.walls;
    const float dx = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(A[2])), 1.0f));
    const float dy = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(A[3])), 1.0f));
    const float dz = __fmul_rn(dm, __fsub_rn(__fmul_rn(2.0f, u24(B[0])), 1.0f));
    float nx = __fadd_rn(po.x, dx), ny = __fadd_rn(po.y, dy), nz = __fadd_rn(po.z, dz);
    if (nx < 0.0f) nx = __fadd_rn(nx, Lx); else if (nx >= Lx) nx = __fsub_rn(nx, Lx);
    if (ny < 0.0f) ny = __fadd_rn(ny, Ly); else if (ny >= Ly) ny = __fsub_rn(ny, Ly);
    if (!walls) { if (nz < 0.0f) nz = __fadd_rn(nz, Lz); else if (nz >= Lz) nz = __fsub_rn(nz, Lz); }
    const float4 pn = make_float4(nx, ny, nz, po.w);
    const int skip = (walls && (nz < D.wall_lo || nz >= D.wall_hi)) ? 2 : 0;  // hard wall: infinite energy
    T.ua = B[2]; T.ub = B[3];
    T.move = PHMC_MOVE_DISP; T.skip = skip; T.nch = 1; T.logf = 0.0;
    T.idx[0] = pf.idx; T.fo[0] = fl; T.pres_old[0] = pold;
    T.po[0] = po; T.to[0] = to; T.bonds[0] = pf.bonds;
    T.pres_new[0] = 1; T.pn[0] = pn; T.tn[0] = to;
    if (skip) return;
    int np = 0, ns = 0;
    if (pold) {
        T.probe_p[np] = po; T.probe_t[np] = to; T.probe_owner[np] = 0; T.probe_sign[np] = -1.0f;
        T.probe_cell[np] = cell_index(D, po.x, po.y, po.z);
        ++np;
    }
    T.probe_p[np] = pn; T.probe_t[np] = to; T.probe_owner[np] = 0; T.probe_sign[np] = 1.0f;
    T.probe_cell[np] = cell_index(D, pn.x, pn.y, pn.z);
    ++np;
    if (D.coulomb == PHMC_COUL_EWALD) {
        if (pold && po.x == pn.x && po.y == pn.y && po.z == pn.z) {
            const float c = pn.w - po.w;
            if (c != 0.0f) { T.st_pos[ns] = pn; T.st_coef[ns] = c; ++ns; }
        } else {
            if (pold && po.w != 0.0f) { T.st_pos[ns] = po; T.st_coef[ns] = -po.w; ++ns; }
            if (pn.w != 0.0f) { T.st_pos[ns] = pn; T.st_coef[ns] = pn.w; ++ns; }
        }
    }
    T.nprobe = np; T.nst = ns;
}

// External trial (phmc_delta_energy / phmc_commit / phmc_set_identity).
__device__ void load_external(TrialS& T, const RepDesc& D, const DevPtrs& d, const phmc_trial& e) {
    const int so = D.slot_off;
    T.nch = e.n_changes; T.skip = 0; T.logf = 0.0; T.move = PHMC_MOVE_NONE;
    for (int k = 0; k < e.n_changes; ++k) {
        const int i = e.c[k].index;
        T.idx[k] = i;
        const int fl = d.flags[so + i];
        T.fo[k] = fl;
        T.pres_old[k] = !(fl & PHMC_F_GHOST);
        T.po[k] = d.posq[so + i]; T.to[k] = d.type[so + i]; T.bonds[k] = d.bonds[so + i];
        T.pres_new[k] = e.c[k].present;
        T.pn[k] = make_float4(e.c[k].x, e.c[k].y, e.c[k].z, e.c[k].q);
        T.tn[k] = e.c[k].type;
    }
    if (T.nch == 1) T.move = PHMC_MOVE_DISP;
}

// Axis k of the stencil of a charge at p (weights, base, wrapped mesh indices).
template <int P>
__device__ __forceinline__ void make_stencil_axis(Stencil<P>& s, const RepDesc& D, float4 p, int k) {
    const float pk = (k == 0) ? p.x : (k == 1 ? p.y : p.z);
    const float g = pk / D.L[k] * (float)D.mesh[k];
    const float fl = floorf(g);
    float w[P];
    bspline_weights<P>(g - fl, w);
    const int base = (int)fl + P / 2 - P + 1;
    s.base[k] = base;
#pragma unroll
    for (int j = 0; j < P; ++j) {  // base + j lies in [-P, n + P): one correction wraps it
        int m = base + j;
        m += (m < 0) ? D.mesh[k] : 0;
        m -= (m >= D.mesh[k]) ? D.mesh[k] : 0;
        s.m[k][j] = m;
        s.w[k][j] = w[j];
    }
}


__device__ __forceinline__ int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
// i mod n for |i| within a few periods (descriptor cell offsets)
__device__ __forceinline__ int wrap_small(int i, int n) {
    while (i < 0) i += n;
    while (i >= n) i -= n;
    return i;
}

__device__ __forceinline__ void list_remove(int* list, int* pos, int& n, int so, int i) {
    const int k = pos[so + i];
    const int last = list[so + n - 1];
    list[so + k] = last; pos[so + last] = k;
    --n;
    pos[so + i] = -1;
}
__device__ __forceinline__ void list_append(int* list, int* pos, int& n, int so, int i) {
    list[so + n] = i; pos[so + i] = n; ++n;
}

__device__ bool cell_remove(const DevPtrs& d, const RepDesc& D, int i) {
    const int gi = D.slot_off + i;
    const int c = d.cell_of[gi], k = d.cell_pos[gi];
    int* cnt = d.cell_count + D.cell_off + c;
    int* l = d.cell_list + ((size_t)D.cell_off + c) * D.cell_cap;
    const int n = *cnt;
    const int last = l[n - 1];
    l[k] = last; d.cell_pos[D.slot_off + last] = k;
    *cnt = n - 1;
    d.cell_of[gi] = -1; d.cell_pos[gi] = -1;
    return true;
}
__device__ bool cell_insert(const DevPtrs& d, const RepDesc& D, int i, int c) {
    const int gi = D.slot_off + i;
    int* cnt = d.cell_count + D.cell_off + c;
    const int n = *cnt;
    if (n >= D.cell_cap) return false;
    d.cell_list[((size_t)D.cell_off + c) * D.cell_cap + n] = i;
    *cnt = n + 1;
    d.cell_of[gi] = c; d.cell_pos[gi] = n;
    return true;
}

__device__ __forceinline__ double slab_energy(const RepDesc& D, double Q, double Mz, double S2) {
    if (!D.slab) return 0.0;
    double e = D.slab_coef * Mz * Mz;
    if (fabs(Q) > 1e-4) e -= D.slab_coef * Q * (S2 + Q * D.Lz2_12);
    return e;
}

// Charge-moment changes of trial T and the self / net-charge / slab energy changes.
struct Moments {
    double dQ, dQ2, dMz, dS2, dself, dqc, dslab;
};
__device__ void moment_terms(const TrialS& T, const RepDesc& D, const RepState& S, Moments& m) {
    double dQ = 0, dQ2 = 0, dMz = 0, dS2 = 0;
    for (int k = 0; k < T.nch; ++k) {
        if (T.pres_new[k]) {
            const double q = T.pn[k].w, z = T.pn[k].z;
            dQ += q; dQ2 += q * q; dMz += q * z; dS2 += q * z * z;
        }
        if (T.pres_old[k]) {
            const double q = T.po[k].w, z = T.po[k].z;
            dQ -= q; dQ2 -= q * q; dMz -= q * z; dS2 -= q * z * z;
        }
    }
    m.dQ = dQ; m.dQ2 = dQ2; m.dMz = dMz; m.dS2 = dS2;
    m.dself = 0; m.dqc = 0; m.dslab = 0;
    if (D.coulomb == PHMC_COUL_EWALD) {
        m.dself = D.self_coef * dQ2;
        const double Qn = S.Q + dQ;
        m.dqc = D.qcorr_coef * (Qn * Qn - S.Q * S.Q);
        m.dslab = slab_energy(D, Qn, S.Mz + dMz, S.S2 + dS2) - slab_energy(D, S.Q, S.Mz, S.S2);
    }
}

// ---- surrogate descriptor (every float operation rounded explicitly, so a
// host restatement reproduces the shell of every particle bit for bit) ----
__device__ __forceinline__ float min_image_rn(float d, float L) {
    return __fsub_rn(d, __fmul_rn(L, rintf(__fdiv_rn(d, L))));
}
__device__ __forceinline__ int shell_of(float dx, float dy, float dz) {
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    return (int)__fmul_rn(__fsqrt_rn(r2), 2.0f);
}
// one-hot state index of a row: charged site, neutral site, anion, cation (-1: none)
__device__ __forceinline__ int row_state(bool titr, float q) {
    if (titr) return q != 0.0f ? 0 : 1;
    return q < 0.0f ? 2 : (q > 0.0f ? 3 : -1);
}
// exact interaction of two changed particles: LJ plus bare Coulomb (Ewald) or the cutoff Coulomb
__device__ double pair_cross(const RepDesc& D, float4 a, float4 b, int ta, int tb, bool bonded) {
    const float dx = min_image(a.x - b.x, D.L[0]), dy = min_image(a.y - b.y, D.L[1]), dz = min_image(a.z - b.z, D.L[2]);
    float elj, ec;
    pair_energy(D, dx, dy, dz, ta, tb, a.w, b.w, bonded, elj, ec);
    if (D.coulomb == PHMC_COUL_EWALD) {
        const float qq = a.w * b.w;
        ec = (qq != 0.0f && !(bonded && D.excl_coul)) ? D.elf * qq / sqrtf(dx * dx + dy * dy + dz * dz) : 0.0f;
    }
    return (double)elj + (double)ec;
}

// Rows, descriptor centres, exclusions and the exact terms of the first stage (one thread).
__device__ void desc_setup(TrialS& T, const RepDesc& D) {
    int nr = 0;
    for (int k = 0; k < T.nch; ++k) {
        const float4 p = T.pres_new[k] ? T.pn[k] : T.po[k];
        T.dpos[k] = p;
        T.dcx[k] = min(D.ncell[0] - 1, max(0, (int)(p.x * D.cell_scale[0])));
        T.dcy[k] = min(D.ncell[1] - 1, max(0, (int)(p.y * D.cell_scale[1])));
        T.dcz[k] = min(D.ncell[2] - 1, max(0, (int)(p.z * D.cell_scale[2])));
        T.ccell[k] = T.pres_old[k] ? cell_index(D, T.po[k].x, T.po[k].y, T.po[k].z) : -1;
        T.ccls[k] = T.pres_old[k] ? desc_class(T.fo[k], T.po[k].w) : -1;
        const bool titr = T.pres_old[k] && (T.fo[k] & PHMC_F_TITRATABLE);
        if (T.pres_old[k]) { T.row_k[nr] = k; T.row_cls[nr] = row_state(titr, T.po[k].w); T.row_sign[nr] = -1.0f; ++nr; }
        if (T.pres_new[k]) { T.row_k[nr] = k; T.row_cls[nr] = row_state(titr, T.pn[k].w); T.row_sign[nr] = 1.0f; ++nr; }
    }
    T.nrows = nr;
}

// Exact terms of the first stage: the changed particles' direct interaction and
// the self / net-charge / slab changes (one thread, beside the descriptor work).
__device__ void desc_exact_terms(TrialS& T, const RepDesc& D, const RepState& S) {
    double cross = 0.0;
    if (T.nch == 2) {
        const bool bonded = in_bonds(T.bonds[0], T.idx[1]);
        const double a = (T.pres_new[0] && T.pres_new[1]) ? pair_cross(D, T.pn[0], T.pn[1], T.tn[0], T.tn[1], bonded) : 0.0;
        const double b = (T.pres_old[0] && T.pres_old[1]) ? pair_cross(D, T.po[0], T.po[1], T.to[0], T.to[1], bonded) : 0.0;
        cross = a - b;
    }
    T.cross = cross;
    Moments m;
    moment_terms(T, D, S, m);
    T.dmom = m.dself + m.dqc + m.dslab;
}

// ---- the reference's grand-canonical mu-control phase (MC/src/mc.cu:320-548) ----

__device__ __forceinline__ int* gc_pool(const DevPtrs& d, const RepDesc& D, int k) {
    return d.gc_pool + (size_t)k * d.gc_pool_stride + D.slot_off;
}

template <class Ev>
__device__ void gc_event(GcDev& G, const DevPtrs& d, const Ev& ev) {
    const int k = G.n_ev++;
    if (k < G.ev_cap) reinterpret_cast<Ev*>(d.gc_ev + (size_t)blockIdx.x * G.ev_cap * GC_EV_BYTES)[k] = ev;
}

__device__ __forceinline__ phmc_gc_event gc_event_base(const GcDev& G, int kind) {
    phmc_gc_event ev;
    memset(&ev, 0, sizeof ev);
    ev.kind = kind; ev.epoch = G.epoch;
    ev.acc_since_mu = G.acc_mu; ev.att_since_mu = G.att_mu;
    ev.block_accepted = G.block_acc; ev.block_attempted = G.block_att;
    ev.nprot = G.Nprot; ev.remaining = max(0, G.target - G.Nprot);
    ev.fwd_total = G.fwd; ev.bwd_total = G.bwd;
    ev.mu_kT = __fmul_rn(G.beta, G.mu);
    ev.E = G.E;
    return ev;
}

// natural log of a float as the host library's correctly rounded logf gives it
__device__ __forceinline__ float gc_logf(float x) { return (float)log((double)x); }
__device__ __forceinline__ float gc_clamp(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Proposal of the next pair flip (one thread): direction, then NH site, then W / Cl
// partner, each from the reference's generator (MC/src/mc.cu:383-417).  Sets T.stop
// when the launch or the phase ends.
__device__ void gc_propose(TrialS& T, GcDev& G, const RepDesc& D, const DevPtrs& d, int npend, int pend_max, int& launch_trials) {
    if (G.stop || npend + 2 > pend_max || launch_trials >= G.launch_cap) { T.stop = 1; return; }
    if (G.attempted >= G.max_trials) { G.stop = PHMC_GC_STOP_MAX_TRIALS; T.stop = 1; return; }
    const long long a = G.n[GC_NHN], b = G.n[GC_NHP], c = G.n[GC_W], e = G.n[GC_CL];
    const long long wf = a * c, wb = b * e;
    bool fwd;
    if (wf > 0 && wb > 0) {
        const float sum = (float)(wf + wb);
        fwd = mt_unit_float(G.mt) < __fdiv_rn((float)wf, sum);
    } else if (wf > 0) {
        fwd = true;
    } else if (wb > 0) {
        fwd = false;
    } else {
        gc_event(G, d, gc_event_base(G, PHMC_GC_EV_NO_PAIRS));
        G.stop = PHMC_GC_STOP_NO_PAIRS;
        T.stop = 1;
        return;
    }
    const int i = gc_pool(d, D, fwd ? GC_NHN : GC_NHP)[mt_index(G.mt, (uint32_t)(fwd ? a : b))];
    const int j = gc_pool(d, D, fwd ? GC_W : GC_CL)[mt_index(G.mt, (uint32_t)(fwd ? c : e))];
    G.dir = fwd ? 1 : -1;
    G.s_before = wf + wb;
    G.s_after = fwd ? (a - 1) * (c - 1) + (b + 1) * (e + 1) : (a + 1) * (c + 1) + (b - 1) * (e - 1);
    ++launch_trials;
    T.move = PHMC_MOVE_NONE; T.skip = 0; T.nch = 2; T.logf = 0.0; T.tnum = G.attempted;
    const int so = D.slot_off;
    const int idx[2] = {i, j};
    for (int k = 0; k < 2; ++k) {
        const int s = idx[k];
        T.idx[k] = s;
        T.fo[k] = d.flags[so + s];
        T.pres_old[k] = 1; T.pres_new[k] = 1;
        T.po[k] = d.posq[so + s]; T.to[k] = d.type[so + s]; T.bonds[k] = d.bonds[so + s];
        T.pn[k] = T.po[k];
    }
    T.pn[0].w = fwd ? G.q_nhp : 0.0f; T.tn[0] = G.type[fwd ? GC_NHP : GC_NHN];
    T.pn[1].w = fwd ? G.q_cl : 0.0f;  T.tn[1] = G.type[fwd ? GC_CL : GC_W];
}

// Decision and the phase's bookkeeping after the exact dE of the flip (one thread,
// MC/src/mc.cu:422-545).  The energies are the reference's: the LJ part and the
// Coulomb part of the trial state each rounded to the reference's real, summed,
// and differenced with the phase's last accepted energy.  Returns the decision.
__device__ int gc_decide(GcDev& G, const RepDesc& D, const RepState& S, const DevPtrs& d, double dlj, double dc, double drec,
                         double dself, double dqc, double dslab) {
    const double lj = S.E_pair_lj + dlj;
    const double ec = D.coulomb == PHMC_COUL_EWALD
                          ? (S.E_pair_c + dc) + (S.E_rec + drec) + (S.E_self + dself) + (S.E_qcorr + dqc) + (S.E_slab + dslab)
                          : S.E_pair_c + dc;
    const float Et = __fadd_rn(__double2float_rn(lj), __double2float_rn(ec));
    const float dEf = __fsub_rn(Et, G.E);
    const float arg = __fmul_rn(-G.beta, __fsub_rn(dEf, __fmul_rn((float)G.dir, G.mu)));
    double logH = 0.0;
    if (G.s_before > 0 && G.s_after > 0) logH = log((double)G.s_before) - log((double)G.s_after);
    double expo = (double)arg + logH;
    expo = expo < -40.0 ? -40.0 : (expo > 40.0 ? 40.0 : expo);
    const int accept = (expo >= 0.0) || (exp(expo) > (double)mt_unit_float(G.mt));
    G.attempted++; G.block_att++; G.att_mu++;
    if (accept) {
        G.accepted++; G.block_acc++; G.acc_mu++;
        if (G.dir > 0) G.fwd++; else G.bwd++;
        G.E = Et;
        G.Nprot += G.dir;
        if (!G.fixed && G.Nprot == G.target) {
            phmc_gc_event ev = gc_event_base(G, PHMC_GC_EV_REACHED);
            ev.step_in_block = G.block_t + 1;
            gc_event(G, d, ev);
            G.stop = PHMC_GC_STOP_REACHED;
            return accept;
        }
    }
    if (++G.block_t == G.gc_block) {
        phmc_gc_event ev = gc_event_base(G, PHMC_GC_EV_CHUNK);
        ev.acc_rate = __fdiv_rn((float)G.block_acc, (float)G.block_att);
        gc_event(G, d, ev);
        G.block_t = 0; G.block_att = 0; G.block_acc = 0;
        if (!G.fixed && !(G.acc_mu < G.nacc_target && G.att_mu < G.amax)) {  // the epoch ends: mu update
            const float f = G.Nh > 0 ? __fdiv_rn((float)G.Nprot, (float)G.Nh) : 0.0f;
            const float lo = (float)1e-6, hi = (float)(1.0 - 1e-6);
            const float f1 = gc_clamp(f, lo, hi);
            const float logit_diff = __fsub_rn(gc_logf(__fdiv_rn(f1, __fsub_rn(1.0f, f1))),
                                               gc_logf(__fdiv_rn(G.f0, __fsub_rn(1.0f, G.f0))));
            const bool early = (G.att_mu >= G.amax) && (G.acc_mu < G.nacc_target);
            const float w_info = G.nacc_target > 0
                                     ? gc_clamp(__fdiv_rn((float)G.acc_mu, (float)max(1, G.nacc_target)), 0.0f, 1.0f)
                                     : 1.0f;
            const float step = __fmul_rn(__fmul_rn(__fmul_rn(__fdiv_rn(1.0f, G.beta), G.eta), logit_diff), w_info);
            G.mu = __fsub_rn(G.mu, step);
            G.blocks_done = G.epoch + 1;
            phmc_gc_event mu = gc_event_base(G, PHMC_GC_EV_MU);
            mu.cause_amax = early ? 1 : 0;
            mu.f = f;
            mu.w_info = w_info;
            gc_event(G, d, mu);
            G.epoch++; G.acc_mu = 0; G.att_mu = 0;
        }
    }
    return accept;
}

// Move slot v from pool src to the end of pool dst, keeping the order of the rest
// (std::vector erase + push_back); all threads of the block.
template <int NT>
__device__ void gc_pool_move(int* src, int* dst, int& n_src, int& n_dst, int v, int* s_find) {
    if (threadIdx.x == 0) *s_find = 0x7fffffff;
    __syncthreads();
    const int n = n_src;
    for (int k = threadIdx.x; k < n; k += NT)
        if (src[k] == v) atomicMin(s_find, k);
    __syncthreads();
    const int k0 = *s_find;
    if (k0 < n) {
        for (int b = k0; b < n - 1; b += NT) {  // shift the tail down by one, NT entries per step
            const int k = b + threadIdx.x;
            const int val = (k < n - 1) ? src[k + 1] : 0;
            __syncthreads();
            if (k < n - 1) src[k] = val;
            __syncthreads();
        }
        if (threadIdx.x == 0) { dst[n_dst] = v; n_dst = n_dst + 1; n_src = n - 1; }
    }
    __syncthreads();
}

// ---- the reference's phase 2: swaps with patience (MC/src/mc.cu:159-318) ----

__device__ __forceinline__ void p2_change(TrialS& T, const DevPtrs& d, const RepDesc& D, int k, int slot, int type, float q) {
    const int so = D.slot_off;
    T.idx[k] = slot;
    T.fo[k] = d.flags[so + slot];
    T.pres_old[k] = 1; T.pres_new[k] = 1;
    T.po[k] = d.posq[so + slot]; T.to[k] = d.type[so + slot]; T.bonds[k] = d.bonds[so + slot];
    T.pn[k] = T.po[k]; T.pn[k].w = q; T.tn[k] = type;
}

// Next two-atom evaluation of phase 2 (one thread).  An attempt draws its atoms in the
// reference's order (NH_P, NH_N, Cl, W; or Cl, W) and starts with the NH half of a
// four-point move, or is a Cl/W move; the Cl/W half follows; a rejected four-point
// move ends with the NH half restored.  Attempts start only with room for all of their
// pending stencils, so a launch never ends inside one.
__device__ void p2_propose(TrialS& T, GcDev& G, const RepDesc& D, const DevPtrs& d, int npend, int pend_max, int& launch_trials) {
    T.move = PHMC_MOVE_NONE; T.skip = 0; T.nch = 2; T.logf = 0.0; T.tnum = G.attempted;
    if (G.role == 1) {  // the Cl/W half, judged with the NH half in place
        p2_change(T, d, D, 0, G.jCl, G.type[GC_W], 0.0f);
        p2_change(T, d, D, 1, G.jW, G.type[GC_CL], G.q_cl);
        G.role = 2; ++launch_trials;
        return;
    }
    if (G.role == 3) {  // restore the NH half of the rejected move
        p2_change(T, d, D, 0, G.iP, G.o_type[0], G.o_q[0]);
        p2_change(T, d, D, 1, G.iN, G.o_type[1], G.o_q[1]);
        ++launch_trials;
        return;
    }
    if (G.stop || launch_trials >= G.launch_cap) { T.stop = 1; return; }
    if (G.attempted >= G.max_attempts) { G.stop = PHMC_P2_STOP_MAX_ATTEMPTS; T.stop = 1; return; }
    const bool can_wc = G.n[GC_W] > 0 && G.n[GC_CL] > 0;
    const bool four = !G.prefer_wc && can_wc && G.n[GC_NHP] > 0 && G.n[GC_NHN] > 0;
    const bool wc = G.prefer_wc || (!four && can_wc);
    if (!four && !wc) {
        phmc_phase2_event ev;
        memset(&ev, 0, sizeof ev);
        ev.kind = PHMC_P2_EV_NONE;
        gc_event(G, d, ev);
        G.stop = PHMC_P2_STOP_NO_PROPOSALS; T.stop = 1;
        return;
    }
    if (npend + (four ? 6 : 2) > pend_max) { T.stop = 1; return; }
    G.attempted++;
    G.four = four ? 1 : 0;
    const int so = D.slot_off;
    if (four) {
        G.iP = gc_pool(d, D, GC_NHP)[mt_index(G.mt, (uint32_t)G.n[GC_NHP])];
        G.iN = gc_pool(d, D, GC_NHN)[mt_index(G.mt, (uint32_t)G.n[GC_NHN])];
        G.jCl = gc_pool(d, D, GC_CL)[mt_index(G.mt, (uint32_t)G.n[GC_CL])];
        G.jW = gc_pool(d, D, GC_W)[mt_index(G.mt, (uint32_t)G.n[GC_W])];
        G.o_type[0] = d.type[so + G.iP]; G.o_q[0] = d.posq[so + G.iP].w;
        G.o_type[1] = d.type[so + G.iN]; G.o_q[1] = d.posq[so + G.iN].w;
        p2_change(T, d, D, 0, G.iP, G.type[GC_NHN], 0.0f);
        p2_change(T, d, D, 1, G.iN, G.type[GC_NHP], G.q_nhp);
        G.role = 1;
    } else {
        G.jCl = gc_pool(d, D, GC_CL)[mt_index(G.mt, (uint32_t)G.n[GC_CL])];
        G.jW = gc_pool(d, D, GC_W)[mt_index(G.mt, (uint32_t)G.n[GC_W])];
        p2_change(T, d, D, 0, G.jCl, G.type[GC_W], 0.0f);
        p2_change(T, d, D, 1, G.jW, G.type[GC_CL], G.q_cl);
        G.role = 2;
    }
    ++launch_trials;
}

// Decision of a phase-2 evaluation (one thread).  The NH half and its restoration are
// applied unconditionally; the judged move follows the reference (MC/src/mc.cu:241-293):
// dE from the reference's float energies, accepted if dE <= 0 or exp(clamp(-beta dE))
// beats a uniform draw; then the best-energy / patience bookkeeping and the report line.
// Returns the decision; *pool_ops gets 2 (four-point pools), 3 (Cl/W pools) or 0.
__device__ int p2_decide(GcDev& G, const RepDesc& D, const RepState& S, const DevPtrs& d, double dlj, double dc, double drec,
                         double dself, double dqc, double dslab, int* pool_ops) {
    *pool_ops = 0;
    if (G.role == 1) return 1;  // the NH half: applied, judged with the Cl/W half
    if (G.role == 3) {          // restored
        G.role = 0;
        if (G.stop_after_restore) G.stop = G.stop_after_restore;
        return 1;
    }
    const double lj = S.E_pair_lj + dlj;
    const double ec = D.coulomb == PHMC_COUL_EWALD
                          ? (S.E_pair_c + dc) + (S.E_rec + drec) + (S.E_self + dself) + (S.E_qcorr + dqc) + (S.E_slab + dslab)
                          : S.E_pair_c + dc;
    const float Et = __fadd_rn(__double2float_rn(lj), __double2float_rn(ec));
    const float dEf = __fsub_rn(Et, G.E);
    float expo = __fmul_rn(-G.beta, dEf);
    expo = expo < -40.0f ? -40.0f : (expo > 40.0f ? 40.0f : expo);
    const int accept = (dEf <= 0.0f) || ((float)exp((double)expo) > mt_unit_float(G.mt));
    if (accept) {
        G.accepted++;
        G.E = Et;
        if (G.E < __fsub_rn(G.best_E, 1e-9f)) { G.best_E = G.E; G.since_best = 0; }
        else ++G.since_best;
        *pool_ops = G.four ? 2 : 3;
        G.role = 0;
    } else {
        ++G.since_best;
        G.role = G.four ? 3 : 0;
    }
    if (G.attempted % max(1, G.energy_interval) == 0) {
        phmc_phase2_event ev;
        memset(&ev, 0, sizeof ev);
        ev.kind = PHMC_P2_EV_STEP;
        ev.attempted = G.attempted; ev.accepted = G.accepted;
        ev.since_best = G.since_best; ev.patience = G.patience;
        ev.mode_wc = G.four ? 0 : 1;
        ev.E = G.E;
        ev.acc = G.attempted > 0 ? __fdiv_rn((float)G.accepted, (float)G.attempted) : 0.0f;
        gc_event(G, d, ev);
    }
    if (G.since_best >= G.patience) {
        phmc_phase2_event ev;
        memset(&ev, 0, sizeof ev);
        ev.kind = PHMC_P2_EV_PATIENCE;
        ev.since_best = G.since_best; ev.patience = G.patience;
        gc_event(G, d, ev);
        if (G.role == 3) G.stop_after_restore = PHMC_P2_STOP_PATIENCE;  // the rejected move is undone first
        else G.stop = PHMC_P2_STOP_PATIENCE;
    }
    return accept;
}

// (an atomic add whose result is unused does not wait for the line: the commit thread goes on)
__device__ __forceinline__ void cls_add(const DevPtrs& d, const RepDesc& D, int cell, int cls, int delta) {
    if (cls >= 0 && cell >= 0) atomicAdd(reinterpret_cast<int*>(d.cell_cls + D.cell_off + cell) + cls, delta);
}

template <int NT>
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[w * 3] = a; red[w * 3 + 1] = b; red[w * 3 + 2] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0, y = 0, z = 0;
        for (int k = 0; k < NT / 32; ++k) { x += red[k * 3]; y += red[k * 3 + 1]; z += red[k * 3 + 2]; }
        red[96] = x; red[97] = y; red[98] = z;
    }
    __syncthreads();
    a = red[96]; b = red[97]; c = red[98];
}

// RC: candidate particles per thread and round of the pair pass (the neighbour tile of a
// round is RC x NT candidates); RR: rows of the influence kernel G each thread has in
// flight per step of the pending-correction sum (2-4: one row per work item, strided over
// the block; 20 + w: one pair per warp, w pairs in flight, lanes over the pair's (dy, dx)
// plane); both tuning parameters
// FS: the surrogate's first stage (descriptor, network, training-sample harvest) compiled in;
// launches that use none of it (plain Monte Carlo) take the instance without its code, whose
// hot loop is then smaller in the instruction caches
template <int P, int NT, bool GC, int RC = 4, int RR = 2, bool FS = true>
__global__ void __launch_bounds__(NT, 512 / NT) k_mc(DevPtrs d, int mode, int ext_rep, const phmc_trial* __restrict__ ext, int n_ext,
                                           double* __restrict__ ext_dE, int pend_max) {
    constexpr int W = 2 * P - 1;
    constexpr int P3 = P * P * P;
    extern __shared__ __align__(16) unsigned char dsm[];
    // pending stencils [0, s_npend) followed by the current trial's stencils (a
    // commit just advances s_npend); then the stencil-pair tables
    Stencil<P>* s_pend = reinterpret_cast<Stencil<P>*>(dsm);
    PairK<P>* s_pair = reinterpret_cast<PairK<P>*>(s_pend + pend_max + NST_MAX);
    __shared__ TrialS T;
    __shared__ RepState S;
    __shared__ int s_cnt[NPROBE_MAX * 27], s_off[NPROBE_MAX * 27 + 1], s_cell[NPROBE_MAX * 27];
    __shared__ __align__(16) int s_list[NPROBE_MAX * 27 * LIST_PF];  // phase 2: leading entries of the probe cells
    __shared__ uint8_t s_cmap[CAND_MAP];  // phase 3: probe-cell entry of each candidate
    __shared__ double red[100];
    __shared__ double s_fene[4];     // FENE dE per bond slot (phase 2), summed in phase 3
    __shared__ Moments s_mo;         // the trial's charge-moment terms (phase 4)
    __shared__ int s_npend;
    __shared__ float4 s_qjob[4];     // charge-mesh updates of the last accepted change: (x, y, z, q) out / in
    __shared__ int s_qsgn[4], s_nqjob;
    __shared__ int s_qin;            // counted among the launch's active replicas
    __shared__ volatile int s_qstop; // the launch's quorum of blocked replicas was seen
    __shared__ uint32_t s_rng[32][16];  // Philox words of trials s_rng_base .. s_rng_base+31
    __shared__ long long s_rng_base;
    __shared__ Prefetch pf;
    // surrogate first stage: shell histogram per changed particle, raw rows, outputs
    __shared__ int s_hist[2 * SUR_SHELLS * SUR_CLASSES];
    __shared__ float s_rows[SUR_ROWS][SUR_K];
    __shared__ float s_F[8];
    __shared__ int s_hv_slot, s_hv_nrows;  // harvested sample whose rows are still to be stored
    __shared__ __align__(8) uint64_t s_mbar[3];  // completion of the staged weight copies
    __shared__ int s_sfail;                      // a staged copy did not arrive in time
    __shared__ float s_mu[SUR_K], s_sd[SUR_K];   // the attached network's input standardisation
    __shared__ uint16_t s_w4[SUR_HMAX];          // its output weights
    // staged first stage (aliases the pair tables, used before phase 3): activations, weights
    unsigned char* sur_base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(s_pair) + 127) & ~uintptr_t(127));
    __nv_bfloat16* act0 = reinterpret_cast<__nv_bfloat16*>(sur_base);
    __nv_bfloat16* act1 = act0 + 16 * SUR_AST;
    uint2* wa = reinterpret_cast<uint2*>(sur_base + SUR_ACT_BYTES);
    // three buffers (layer 1, 2, 3), or with sur_late_l3 two of SUR_HMAX^2 (layer 3 reuses layer 1's)
    uint2* wb = d.sur_late_l3 ? wa + SUR_WBUF_BYTES / 8 : wa + (SUR_K * SUR_HMAX * 2) / 8;
    uint2* wc = d.sur_late_l3 ? wa : wb + SUR_WBUF_BYTES / 8;
    uint32_t sur_par = 0;  // parity of the weight barriers' current phase (one phase per evaluated move)
    // grand-canonical mu-control phase: the job's state (block blockIdx.x runs job blockIdx.x)
    __shared__ __align__(16) typename std::conditional<GC, GcDev, int>::type sG;
    __shared__ int s_gc_ops, s_gc_find, s_gc_lt;
    __shared__ unsigned int s_zh[3 * PHMC_ZHIST_MAX_BINS];

    // the instance without the first stage runs Monte Carlo launches only: with the mode a
    // constant the external-trial paths drop out of its code as well
    if constexpr (!FS && !GC) mode = MC_RUN;
    const int r = GC ? d.gc[blockIdx.x].replica : ((mode == MC_RUN) ? blockIdx.x : ext_rep);
    const int tid = threadIdx.x;
    if constexpr (GC) {
        const int* src = reinterpret_cast<const int*>(d.gc + blockIdx.x);
        int* dst = reinterpret_cast<int*>(&sG);
        for (int k = tid; k < (int)(sizeof(GcDev) / sizeof(int)); k += NT) dst[k] = src[k];
        if (tid == 0) { s_gc_ops = 0; s_gc_lt = 0; }
        __syncthreads();
        if (tid == 0) sG.n_ev = 0;
    }
    // the replica's descriptor lives in shared memory for the whole launch
    __shared__ __align__(16) RepDesc sD;
    {
        const int* src = reinterpret_cast<const int*>(d.desc + r);
        int* dst = reinterpret_cast<int*>(&sD);
        for (int k = tid; k < (int)(sizeof(RepDesc) / sizeof(int)); k += NT) dst[k] = src[k];
    }
    const RepDesc& D = sD;
    if (tid == 0) {
        S = d.state[r];
        s_npend = 0;
        T.ext_k = 0;
        T.stop = 0;
        s_rng_base = -64;
        pf.valid = 0;
        s_hv_slot = -1;
        s_sfail = 0;
        s_qstop = 0;
        s_qin = 0;
        s_nqjob = 0;
        if (mode == MC_RUN && d.quorum < 1.0f && S.trial < S.target) { atomicAdd(&d.quorum_ctl[0], 1); s_qin = 1; }
        sur_mbar_init(&s_mbar[0]);
        sur_mbar_init(&s_mbar[1]);
        sur_mbar_init(&s_mbar[2]);
    }
    if (d.sur.H > 0) {
        for (int k = tid; k < SUR_K; k += NT) { s_mu[k] = d.sur.mu[k]; s_sd[k] = d.sur.sd[k]; }
        for (int k = tid; k < d.sur.H; k += NT) s_w4[k] = d.sur.w4[k];
    }
    unsigned long long t_start = 0;
    if (tid == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    // phase clocks (thread 0, after the barrier that ends each phase): 0 proposal, 1 first
    // stage, 2 cell counts + stencils + direct terms, 3 offsets + pair tables, 4 candidate pair
    // terms, 5 phi gather + pending corrections + reduction, 6 decision + commit, 7 trials
    // ended before phase 2 (first-stage rejections, invalid proposals)
    long long clk_last = clock64();
    auto mark = [&](int ph) {
        if (tid == 0 && d.phase_clk) {
            const long long now = clock64();
            S.clk[ph] += now - clk_last;
            clk_last = now;
        }
    };
    __syncthreads();

    for (;;) {
        // ---------------- proposal ----------------
        if (tid < 32) {
            if (mode == MC_RUN) {  // warp 0 refills the Philox table every 32 trials
                const long long t = S.trial;
                if (t - s_rng_base >= 32 || t < s_rng_base) {
                    trial_words(D, t + tid, s_rng[tid]);
                    __syncwarp();
                    if (tid == 0) s_rng_base = t;
                    __syncwarp();
                }
            }
            if (tid == 0) {
                bool set_up = false;
                T.stop = 0; T.desc = 0; T.da = 0;
                if (S.error) T.stop = 1;
                else if (GC) {
                    if constexpr (GC) {
                        if (sG.phase == 2) p2_propose(T, sG, D, d, s_npend, pend_max, s_gc_lt);
                        else gc_propose(T, sG, D, d, s_npend, pend_max, s_gc_lt);
                    }
                } else if (mode == MC_RUN) {
                    if (S.trial >= S.target) { T.stop = 1; S.stop_reason = 0; }
                    else if (s_npend + 2 > pend_max) {
                        T.stop = 1; S.stop_reason = 1;
                        if (s_qin) atomicAdd(&d.quorum_ctl[1], 1);
                    } else if (s_qstop) { T.stop = 1; S.stop_reason = 2; }
                    else {
                        T.tnum = S.trial;
                        const uint32_t* rw = s_rng[S.trial - s_rng_base];
                        if (pf.valid && pf.t == S.trial && pf.move == PHMC_MOVE_DISP && S.n_mobile > 0) {
                            propose_disp_setup(T, D, pf, rw);  // the common case, set up already
                            set_up = true;
                        } else propose(T, D, S, d, rw, pf);
                        S.trial++;
                    }
                } else {
                    if (T.ext_k >= n_ext) T.stop = 1;
                    else { load_external(T, D, d, ext[T.ext_k]); T.tnum = T.ext_k; }
                }
                if (!T.stop && T.skip == 0) {
                    if (!set_up) trial_setup(T, D);
                    if (!FS) {
                    } else if (mode == MC_DESCRIBE) {
                        T.desc = 1; T.da = d.sur.H > 0;
                    } else if (mode == MC_RUN && (T.move == PHMC_MOVE_TITR || T.move == PHMC_MOVE_SWAP)) {
                        // delayed acceptance (not under replay, which dictates decisions)
                        T.da = d.sur.H > 0 && !S.da_off && !(r == 0 && d.replay);
                        T.desc = T.da || d.hv_cap > 0;
                    }
                    if (FS && T.desc) desc_setup(T, D);
                }
            }
        } else {
            // warps 1..4: the last accepted change's updates of the fixed-point charge mesh
            // (integer adds of the same values a full spread computes, so the band mesh stays
            // equal to a spread of the current configuration)
            {
                const int wj = (tid >> 5) - 1;
                if (wj < s_nqjob) {
                    const float4 pq = s_qjob[wj];
                    const bool neg = s_qsgn[wj] < 0;
                    float w[3][P];
                    int base[3];
                    qmesh_stencil<P>(D, pq, w, base);
                    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
                    unsigned long long* qb = d.qband + D.qb_off;
                    const int lane = tid & 31;  // lane (bb, c) < P^2 writes the row of P points
                    const int bb = lane % P, c = lane / P;
                    int zr = base[2] + c - D.zb_lo;
                    zr %= nz;
                    zr += (zr < 0) ? nz : 0;
                    if (lane < P * P && zr < D.zb_n) {
                        float wy = 0.0f, wz = 0.0f;  // selects keep the weights in registers
#pragma unroll
                        for (int j = 0; j < P; ++j) { wy = (j == bb) ? w[1][j] : wy; wz = (j == c) ? w[2][j] : wz; }
                        int yb = base[1] + bb;
                        yb += (yb < 0) ? ny : 0;
                        yb -= (yb >= ny) ? ny : 0;
                        unsigned long long* row = qb + ((size_t)zr * ny + yb) * nx;
#pragma unroll
                        for (int a = 0; a < P; ++a) {
                            int xa = base[0] + a;
                            xa += (xa < 0) ? nx : 0;
                            xa -= (xa >= nx) ? nx : 0;
                            const long long v = qmesh_value(pq.w, w[0][a], wy, wz);
                            atomicAdd(&row[xa], (unsigned long long)(neg ? -v : v));
                        }
                    }
                }
            }
            // idle threads: store the previous trial's harvested rows, clear the shell histogram
            if (s_hv_slot >= 0) {
                float* dst = d.hv_rows + (size_t)s_hv_slot * (SUR_ROWS * SUR_K);
                for (int e = tid - 32; e < SUR_ROWS * SUR_K; e += NT - 32)
                    dst[e] = (e / SUR_K < s_hv_nrows) ? s_rows[e / SUR_K][e % SUR_K] : 0.0f;
            }
            for (int e = tid - 32; e < 2 * SUR_SHELLS * SUR_CLASSES; e += NT - 32) s_hist[e] = 0;
            for (int e = tid - 32; e < 2 * 27; e += NT - 32) { s_cnt[e] = 0; s_cell[e] = 0; }
        }
        __syncthreads();
        if (T.stop) break;
        mark(0);
        if (tid == 0) { s_hv_slot = -1; s_nqjob = 0; }
        // ---------------- surrogate first stage ----------------
        if (FS && T.desc) {
            if (T.da && tid == 0) {  // stage the three hidden layers while the descriptor is built
                sur_bulk_load(wa, d.sur.w[0], sur_layer_bytes(SUR_K, d.sur.H), &s_mbar[0]);
                sur_bulk_load(wb, d.sur.w[1], sur_layer_bytes(d.sur.H, d.sur.H), &s_mbar[1]);
                if (!d.sur_late_l3) sur_bulk_load(wc, d.sur.w[2], sur_layer_bytes(d.sur.H, d.sur.H), &s_mbar[2]);
            }
            if (tid == NT - 1) desc_exact_terms(T, D, S);
            // (a) the descriptor sphere's cells: inner 27 cells -> counts for the particle
            // pass; outer cells -> class counts binned by the distance of the cell centre
            const int nk0 = D.dnk[0], nk1 = D.dnk[1], nk2 = D.dnk[2];
            const int nc3 = nk0 * nk1 * nk2;
            constexpr int DRC = 3;
            const FastDiv f3(nc3), f2(nk0 * nk1), f1(nk0);
            for (int e0 = tid; e0 < T.nch * nc3; e0 += DRC * NT) {
                int cell_u[DRC], k_u[DRC], sl_u[DRC];
                int4 cc_u[DRC];
                int3 c3_u[DRC];
#pragma unroll
                for (int u = 0; u < DRC; ++u) {  // all loads of the batch first
                    const int e = e0 + u * NT;
                    cell_u[u] = -1;
                    if (e >= T.nch * nc3) continue;
                    int loc, lr, lx;
                    const int k = f3.div(e, loc);
                    const int lz = f2.div(loc, lr);
                    const int ly = f1.div(lr, lx);
                    const int ox = lx - D.dnr[0], oy = ly - D.dnr[1], oz = lz - D.dnr[2];
                    const int cx = wrap_small(T.dcx[k] + ox, D.ncell[0]), cy = wrap_small(T.dcy[k] + oy, D.ncell[1]),
                              cz = wrap_small(T.dcz[k] + oz, D.ncell[2]);
                    const int cell = (cz * D.ncell[1] + cy) * D.ncell[0] + cx;
                    cell_u[u] = cell; k_u[u] = k;
                    c3_u[u] = make_int3(cx, cy, cz);
                    if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1) {
                        sl_u[u] = k * 27 + (oz + 1) * 9 + (oy + 1) * 3 + (ox + 1);
                        cc_u[u].x = d.cell_count[D.cell_off + cell];
                    } else {
                        sl_u[u] = -1;
                        cc_u[u] = __ldcg(&d.cell_cls[D.cell_off + cell]);  // (updated by L2 atomics)
                    }
                }
#pragma unroll
                for (int u = 0; u < DRC; ++u) {
                    const int cell = cell_u[u];
                    if (cell < 0) continue;
                    if (sl_u[u] >= 0) {  // inner cell: count for the particle pass
                        s_cell[sl_u[u]] = cell;
                        s_cnt[sl_u[u]] = min(cc_u[u].x, D.cell_cap);
                        continue;
                    }
                    int4 cc = cc_u[u];
                    for (int j = 0; j < T.nch; ++j)
                        if (T.ccell[j] == cell) {
                            cc.x -= (T.ccls[j] == 0); cc.y -= (T.ccls[j] == 1); cc.z -= (T.ccls[j] == 2); cc.w -= (T.ccls[j] == 3);
                        }
                    if ((cc.x | cc.y | cc.z | cc.w) == 0) continue;
                    const int k = k_u[u];
                    const int cx = c3_u[u].x, cy = c3_u[u].y, cz = c3_u[u].z;
                    const float4 p = T.dpos[k];
                    const float xc = __fmul_rn(__fadd_rn((float)cx, 0.5f), D.cell_w[0]);
                    const float yc = __fmul_rn(__fadd_rn((float)cy, 0.5f), D.cell_w[1]);
                    const float zc = __fmul_rn(__fadd_rn((float)cz, 0.5f), D.cell_w[2]);
                    const int sh = shell_of(min_image_rn(__fsub_rn(xc, p.x), D.L[0]), min_image_rn(__fsub_rn(yc, p.y), D.L[1]),
                                            min_image_rn(__fsub_rn(zc, p.z), D.L[2]));
                    if (sh < SUR_SHELLS) {
                        int* hb = s_hist + k * (SUR_SHELLS * SUR_CLASSES) + sh * SUR_CLASSES;
                        if (cc.x) atomicAdd(hb, cc.x);
                        if (cc.y) atomicAdd(hb + 1, cc.y);
                        if (cc.z) atomicAdd(hb + 2, cc.z);
                        if (cc.w) atomicAdd(hb + 3, cc.w);
                    }
                }
            }
            __syncthreads();
            const int nent_d = T.nch * 27;
            if (tid < 32) {
                int carry = 0;
                for (int b0 = 0; b0 < nent_d; b0 += 32) {
                    const int e = b0 + tid;
                    const int v = (e < nent_d) ? s_cnt[e] : 0;
                    int x = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (tid >= o) x += y;
                    }
                    if (e < nent_d) s_off[e] = carry + x - v;
                    carry += __shfl_sync(0xffffffffu, x, 31);
                }
                if (tid == 0) { s_off[nent_d] = carry; T.dtotal = carry; }
            }
            __syncthreads();
            // (b) particles of the inner cells, exact distance shells (loads batched per thread)
            constexpr int RP = 4;
            for (int it0 = tid; it0 < T.dtotal; it0 += RP * NT) {
                int j_u[RP], k_u[RP];
#pragma unroll
                for (int u = 0; u < RP; ++u) {
                    const int it = it0 + u * NT;
                    j_u[u] = -1;
                    if (it >= T.dtotal) continue;
                    int lo = 0, hi = nent_d - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (s_off[mid] <= it) lo = mid; else hi = mid - 1;
                    }
                    k_u[u] = lo / 27;
                    j_u[u] = d.cell_list[((size_t)D.cell_off + s_cell[lo]) * D.cell_cap + (it - s_off[lo])];
                }
                float4 p_u[RP];
                int f_u[RP];
#pragma unroll
                for (int u = 0; u < RP; ++u) {
                    const int j = j_u[u];
                    f_u[u] = PHMC_F_GHOST;
                    if (j < 0 || j == T.idx[0] || (T.nch == 2 && j == T.idx[1])) continue;
                    p_u[u] = d.posq[D.slot_off + j];
                    f_u[u] = d.flags[D.slot_off + j];
                }
#pragma unroll
                for (int u = 0; u < RP; ++u) {
                    if (f_u[u] & PHMC_F_GHOST) continue;
                    const float4 pj = p_u[u];
                    const int c = desc_class(f_u[u], pj.w);
                    if (c < 0) continue;
                    const float4 p = T.dpos[k_u[u]];
                    const int sh = shell_of(min_image_rn(__fsub_rn(pj.x, p.x), D.L[0]), min_image_rn(__fsub_rn(pj.y, p.y), D.L[1]),
                                            min_image_rn(__fsub_rn(pj.z, p.z), D.L[2]));
                    if (sh < SUR_SHELLS) atomicAdd(&s_hist[k_u[u] * (SUR_SHELLS * SUR_CLASSES) + sh * SUR_CLASSES + c], 1);
                }
            }
            __syncthreads();
            // (c) rows: raw features, and standardised BF16 inputs when the network runs
            for (int e = tid; e < T.nrows * SUR_K; e += NT) {
                const int rr = e / SUR_K, f = e - rr * SUR_K;
                const int k = T.row_k[rr];
                float v;
                if (f < SUR_SHELLS * SUR_CLASSES) v = (float)s_hist[k * (SUR_SHELLS * SUR_CLASSES) + f];
                else if (f == 64) v = __fdiv_rn(__fsub_rn(T.dpos[k].z, D.sur_z0), D.sur_h);
                else if (f < 69) v = (f - 65 == T.row_cls[rr]) ? 1.0f : 0.0f;
                else if (f == 69) v = D.sur_pk;
                else if (f == 70) v = D.sur_salt;
                else v = 0.0f;
                s_rows[rr][f] = v;
                if (T.da) act0[rr * SUR_AST + f] = __float2bfloat16(__fdiv_rn(__fsub_rn(v, s_mu[f]), s_sd[f]));
            }
            __syncthreads();
            // (d) network on the rows (tensor cores), first-stage decision
            if (T.da) {
                sur_forward_staged<NT>(d.sur, T.nrows, act0, act1, wa, wb, wc, s_mbar, sur_par, s_F, &s_sfail,
                                       d.sur_late_l3 != 0, s_w4);
                sur_par ^= 1u;
            }
            if (tid == 0) {
                if (mode == MC_RUN) S.alg_bytes += 16.0 * T.nch * nc3 + 24.0 * T.dtotal;
                double net = 0.0;
                if (T.da) {
                    // per changed particle F(new) - F(old): the estimate is antisymmetric under reversal
                    for (int k = 0; k < T.nch; ++k) {
                        double fo = 0.0, fn = 0.0;
                        for (int rr = 0; rr < T.nrows; ++rr)
                            if (T.row_k[rr] == k) { if (T.row_sign[rr] < 0.0f) fo = s_F[rr]; else fn = s_F[rr]; }
                        net += fn - fo;
                    }
                    T.dEs = (net + T.cross) + T.dmom;
                }
                if (T.da && s_sfail) {  // a staged copy never arrived: stop this replica
                    S.error = PHMC_ERR_BUDGET;
                    T.skip = 6;
                } else if (mode == MC_DESCRIBE) {
                    float* o = d.dsc_out + (size_t)T.ext_k * DSC_STRIDE;
                    for (int e = 0; e < SUR_ROWS * SUR_K; ++e) o[e] = (e / SUR_K < T.nrows) ? s_rows[e / SUR_K][e % SUR_K] : 0.0f;
                    for (int rr = 0; rr < SUR_ROWS; ++rr) {
                        o[SUR_ROWS * SUR_K + rr] = rr < T.nrows ? T.row_sign[rr] : 0.0f;
                        o[SUR_ROWS * SUR_K + SUR_ROWS + rr] = (T.da && rr < T.nrows) ? s_F[rr] : 0.0f;
                    }
                    o[SUR_ROWS * SUR_K + 2 * SUR_ROWS] = (float)T.cross;
                    o[SUR_ROWS * SUR_K + 2 * SUR_ROWS + 1] = (float)T.dmom;
                    o[SUR_ROWS * SUR_K + 2 * SUR_ROWS + 2] = (float)T.nrows;
                    o[SUR_ROWS * SUR_K + 2 * SUR_ROWS + 3] = (float)T.dtotal;
                    T.skip = 5;
                } else if (T.da) {
                    // first stage: Metropolis on the surrogate dE with its own uniform (Philox counter (t, 3))
                    const uint32_t* w4 = s_rng[T.tnum - s_rng_base] + 12;
                    const double expo1 = -D.beta * T.dEs + T.logf;
                    const bool pass = (expo1 >= 0.0) || (u53(w4[0], w4[1]) < exp(expo1));
                    S.da_eval++;
                    if (pass) { S.da_pass++; S.da_wpass++; }
                    else T.skip = 4;
                }
            }
            __syncthreads();
        }
        mark(1);
        if (T.skip) {
            if (tid == 0) {
                if (mode == MC_RUN && T.move < 3) S.att[T.move]++;
                if (mode == MC_RUN) { S.alg_bytes += 16.0; S.trials_run++; }
                const long long li = T.tnum - S.run_start;
                if (mode == MC_RUN && r == 0 && d.log_move && li < d.log_cap) {
                    d.log_move[li] = T.move;
                    d.log_dE[li] = (T.skip == 2) ? __longlong_as_double(0x7ff0000000000000ll) : __longlong_as_double(0x7ff8000000000000ll);
                    d.log_acc[li] = 0;
                    if (d.log_stage) { d.log_stage[li] = (T.skip == 4) ? 1 : 0; d.log_dEs[li] = T.da ? T.dEs : 0.0; }
                }
                if (mode != MC_RUN) {
                    if (ext_dE) ext_dE[T.ext_k] = (T.skip == 5) ? (T.da ? T.dEs : __longlong_as_double(0x7ff8000000000000ll))
                                                                : __longlong_as_double(0x7ff0000000000000ll);
                    T.ext_k++;
                }
            }
            __syncthreads();
            mark(7);
            continue;
        }
        // ---------------- phase 2: cell counts, stencils, direct & bonded terms ----------------
        const int nent = T.nprobe * 27;
        Stencil<P>* s_tst = s_pend + s_npend;  // this trial's stencils
        if (tid < nent) {
            const int p = tid / 27, nb = tid % 27;
            // the probe's cell coordinates as cell_index computes them (no integer divisions)
            const float4 pp = T.probe_p[p];
            const int cx = min(D.ncell[0] - 1, max(0, (int)(pp.x * D.cell_scale[0])));
            const int cy = min(D.ncell[1] - 1, max(0, (int)(pp.y * D.cell_scale[1])));
            const int cz = min(D.ncell[2] - 1, max(0, (int)(pp.z * D.cell_scale[2])));
            const int nc = (wrap1(cz + nb / 9 - 1, D.ncell[2]) * D.ncell[1] + wrap1(cy + (nb / 3) % 3 - 1, D.ncell[1])) *
                               D.ncell[0] + wrap1(cx + nb % 3 - 1, D.ncell[0]);
            s_cell[tid] = nc;
            // the count and the cell's leading list entries in one round trip (entries past the
            // count are stale and never read)
            const int* row = d.cell_list + ((size_t)D.cell_off + nc) * D.cell_cap;
            int* dst = s_list + tid * LIST_PF;
            if (D.cell_cap >= LIST_PF && (D.cell_cap & 3) == 0) {
                int4 v[LIST_PF / 4];
#pragma unroll
                for (int q = 0; q < LIST_PF / 4; ++q) v[q] = reinterpret_cast<const int4*>(row)[q];
                s_cnt[tid] = min(d.cell_count[D.cell_off + nc], D.cell_cap);
#pragma unroll
                for (int q = 0; q < LIST_PF / 4; ++q) reinterpret_cast<int4*>(dst)[q] = v[q];
            } else {
                const int m = min(D.cell_cap, LIST_PF);
                for (int q = 0; q < m; ++q) dst[q] = row[q];
                s_cnt[tid] = min(d.cell_count[D.cell_off + nc], D.cell_cap);
            }
        }
        // roles after the cell counts (threads < 108): with 256 threads each in a warp of its
        // own, so that the branches run side by side rather than one after another in one warp
        constexpr int ST0 = NT >= 256 ? 128 : 108, DIR = NT >= 256 ? 160 : 120, FEN0 = NT >= 256 ? 192 : 121;
        // the trial's stencils: one thread per (stencil, axis)
        if (tid >= ST0 && tid < ST0 + 3 * T.nst) {
            const int k = (tid - ST0) / 3, ax = tid - ST0 - 3 * k;
            make_stencil_axis<P>(s_tst[k], D, T.st_pos[k], ax);
            if (ax == 0) s_tst[k].coef = T.st_coef[k];
        }
        if (tid == DIR) {
            double dl = 0.0, dc = 0.0;
            if (T.nch == 2) {
                const bool bonded = in_bonds(T.bonds[0], T.idx[1]);
                float elj, ec;
                if (T.pres_new[0] && T.pres_new[1]) {
                    pair_energy(D, min_image(T.pn[0].x - T.pn[1].x, D.L[0]), min_image(T.pn[0].y - T.pn[1].y, D.L[1]),
                                min_image(T.pn[0].z - T.pn[1].z, D.L[2]), T.tn[0], T.tn[1], T.pn[0].w, T.pn[1].w, bonded, elj, ec);
                    dl += elj; dc += ec;
                }
                if (T.pres_old[0] && T.pres_old[1]) {
                    pair_energy(D, min_image(T.po[0].x - T.po[1].x, D.L[0]), min_image(T.po[0].y - T.po[1].y, D.L[1]),
                                min_image(T.po[0].z - T.po[1].z, D.L[2]), T.to[0], T.to[1], T.po[0].w, T.po[1].w, bonded, elj, ec);
                    dl -= elj; dc -= ec;
                }
            }
            T.d_direct_lj = dl; T.d_direct_c = dc;
        }
        // FENE: one thread per bond slot b, over the changed particles; the four partial sums
        // are added in slot order in phase 3
        if (tid >= FEN0 && tid < FEN0 + 4) {
            const int b = tid - FEN0;
            double df = 0.0;
            if (D.fene_k > 0.0f) {
                const int nch = T.nch;
                int jb[2];
                float4 pjs[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {  // independent loads, issued together
                    const int4 bk = T.bonds[k];
                    const int j = (b == 0) ? bk.x : (b == 1 ? bk.y : (b == 2 ? bk.z : bk.w));
                    jb[k] = (k < nch && T.pres_old[k] && T.pres_new[k]) ? j : -1;
                    pjs[k] = (jb[k] >= 0) ? d.posq[D.slot_off + jb[k]] : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int j = jb[k];
                    if (j < 0 || (nch == 2 && (j == T.idx[0] || j == T.idx[1]))) continue;
                    const float4 pj = pjs[k];
                    const float4 pn = T.pn[k], po = T.po[k];
                    float dx = min_image(pn.x - pj.x, D.L[0]), dy = min_image(pn.y - pj.y, D.L[1]),
                          dz = min_image(pn.z - pj.z, D.L[2]);
                    const float en = fene_energy(D, dx * dx + dy * dy + dz * dz);
                    dx = min_image(po.x - pj.x, D.L[0]); dy = min_image(po.y - pj.y, D.L[1]);
                    dz = min_image(po.z - pj.z, D.L[2]);
                    const float eo = fene_energy(D, dx * dx + dy * dy + dz * dz);
                    df += (double)en - (double)eo;
                }
            }
            s_fene[b] = df;
        }
        __syncthreads();
        mark(2);
        // ---------------- phase 3: candidate offsets, stencil pair kernels ----------------
        if (tid < 32) {
            int carry = 0;
            for (int b0 = 0; b0 < nent; b0 += 32) {
                const int e = b0 + tid;
                const int v = (e < nent) ? s_cnt[e] : 0;
                int x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (tid >= o) x += y;
                }
                if (e < nent) s_off[e] = carry + x - v;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            if (tid == 0) {
                s_off[nent] = carry; T.total_cand = carry;
                T.d_fene = ((s_fene[0] + s_fene[1]) + s_fene[2]) + s_fene[3];
            }
            __syncwarp();
            // candidate -> probe-cell entry table (the pair pass reads it instead of searching)
            for (int e = tid; e < nent; e += 32) {
                const int b = s_off[e], en = min(s_off[e + 1], CAND_MAP);
                for (int c = b; c < en; ++c) s_cmap[c] = (uint8_t)e;
            }
        } else if (D.coulomb == PHMC_COUL_EWALD) {
            const int nst = T.nst, np = s_npend;
            const int npairs = nst * np + nst * (nst + 1) / 2;
            constexpr int W = 2 * P - 1;
            // one (pair, axis, offset) element per work item
            for (int e = tid - 32; e < 3 * W * npairs; e += NT - 32) {
                const int q = e / (3 * W), r3 = e - q * (3 * W);
                const int k = r3 / W, t = r3 - k * W;
                int ta, tb;
                const Stencil<P>* sb;
                float c;
                if (q < nst * np) {
                    ta = (q >= np) + (q >= 2 * np) + (q >= 3 * np);  // q / np for nst <= NST_MAX = 4
                    tb = q - ta * np;
                    sb = &s_pend[tb];
                    c = s_tst[ta].coef * s_pend[tb].coef;
                } else {
                    int rem = q - nst * np;
                    ta = 0;
                    while (rem >= nst - ta) { rem -= nst - ta; ++ta; }
                    tb = ta + rem;
                    sb = &s_tst[tb];
                    c = s_tst[ta].coef * s_tst[tb].coef * (ta == tb ? 0.5f : 1.0f);
                }
                const Stencil<P>& sa = s_tst[ta];
                const int delta = t - (P - 1);
                float s = 0.0f;
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    const int j = i - delta;
                    if (j >= 0 && j < P) s += sa.w[k][i] * sb->w[k][j];
                }
                const int n = D.mesh[k];
                int m = sa.base[k] - sb->base[k] + delta;
                m += (m < 0) ? n : 0;
                m += (m < 0) ? n : 0;
                m -= (m >= n) ? n : 0;
                m -= (m >= n) ? n : 0;
                s_pair[q].K[k][t] = s;
                s_pair[q].f[k][t] = min(m, n - m);
                if (r3 == 0) s_pair[q].coef = c;
            }
            if (tid == 32) T.npairs = npairs;
        }
        __syncthreads();
        mark(3);
        // ---------------- phase 4: all pair / mesh work items ----------------
        // helper loads off the critical path: the next trial's primary particle,
        // and the cell bookkeeping a commit of this trial would need
        if (tid == NT - 1 && mode == MC_RUN) {
            const long long tn = T.tnum + 1;
            if (tn - s_rng_base >= 0 && tn - s_rng_base < 32) prefetch_primary(pf, tn, s_rng[tn - s_rng_base], D, S, d);
            else pf.valid = 0;
        }
        // the trial's charge-moment terms (self, charged-system and slab corrections) for the
        // decision, off the decision thread's path
        if (tid == NT - 97) {  // (helpers on warps of their own: a warp runs divergent branches one after another)
            Moments mo;
            moment_terms(T, D, S, mo);
            s_mo = mo;
        }
        if (tid == NT - 33 || tid == NT - 65) {
            const int k = (tid == NT - 33) ? 0 : 1;
            if (k < T.nch && T.pres_old[k]) {
                const int gi = D.slot_off + T.idx[k];
                const int c = cell_index(D, T.po[k].x, T.po[k].y, T.po[k].z);
                const int cnt = d.cell_count[D.cell_off + c];
                T.cell_old[k] = c;
                T.cpos_old[k] = d.cell_pos[gi];
                T.cnt_old[k] = cnt;
                T.last_old[k] = (cnt > 0) ? d.cell_list[((size_t)D.cell_off + c) * D.cell_cap + cnt - 1] : -1;
            }
        }
        double acc_lj = 0.0, acc_c = 0.0, acc_rec = 0.0;
        // quorum of the launch: read here, compared after the pair work (the loads' latency
        // hides behind it), used from the next trial's proposal on
        const bool q_chk = tid == 32 && s_qin;
        int q_started = 0, q_blocked = 0;
        if (q_chk) { q_started = *(volatile int*)&d.quorum_ctl[0]; q_blocked = *(volatile int*)&d.quorum_ctl[1]; }
        {
            const int total = T.total_cand;
            const int so = D.slot_off;
            // RC candidates per thread and round: all list loads, then all particle loads, then
            // the pair terms (each thread still adds its candidates in increasing order)
            for (int it0 = tid; it0 < total; it0 += RC * NT) {
                int j_u[RC], p_u[RC];
#pragma unroll
                for (int u = 0; u < RC; ++u) {
                    const int it = it0 + u * NT;
                    j_u[u] = -1;
                    p_u[u] = 0;
                    if (it >= total) continue;
                    int lo;
                    if (it < CAND_MAP) lo = s_cmap[it];
                    else {
                        lo = 0;
                        int hi = nent - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_off[mid] <= it) lo = mid; else hi = mid - 1;
                        }
                    }
                    p_u[u] = lo / 27;
                    const int k = it - s_off[lo];
                    j_u[u] = (k < LIST_PF) ? s_list[lo * LIST_PF + k]
                                           : d.cell_list[((size_t)D.cell_off + s_cell[lo]) * D.cell_cap + k];
                }
                float4 pj_u[RC];
                int tj_u[RC];
#pragma unroll
                for (int u = 0; u < RC; ++u) {
                    const int j = j_u[u];
                    if (j < 0 || j == T.idx[0] || (T.nch == 2 && j == T.idx[1])) { j_u[u] = -1; continue; }
                    pj_u[u] = d.posq[so + j];
                    tj_u[u] = d.type[so + j];
                }
#pragma unroll
                for (int u = 0; u < RC; ++u) {
                    if (j_u[u] < 0) continue;
                    const int p = p_u[u];
                    const float4 pj = pj_u[u];
                    const float4 pp = T.probe_p[p];
                    float elj, ec;
                    pair_energy(D, min_image(pp.x - pj.x, D.L[0]), min_image(pp.y - pj.y, D.L[1]), min_image(pp.z - pj.z, D.L[2]),
                                T.probe_t[p], tj_u[u], pp.w, pj.w, in_bonds(T.bonds[T.probe_owner[p]], j_u[u]), elj, ec);
                    acc_lj += (double)(T.probe_sign[p] * elj);
                    acc_c += (double)(T.probe_sign[p] * ec);
                }
            }
        }
        if (d.phase_clk) {  // uniform over the block
            __syncthreads();
            mark(4);
        }
        if (D.coulomb == PHMC_COUL_EWALD) {
            // W_t . phi: element (stencil, c, b, a), a fastest (lanes read consecutive x)
            const float* phi = d.phi + D.mesh_off;
            const int nx = D.mesh[0], ny = D.mesh[1];
            constexpr int P3 = P * P * P;
            const int nphi = T.nst * P3;
            for (int it = tid; it < nphi; it += NT) {
                const int st = it / P3, rem = it - st * P3;
                const int c = rem / (P * P), rb = rem - c * (P * P);
                const int b = rb / P, a = rb - b * P;
                const Stencil<P>& s = s_tst[st];
                const float v = phi[((size_t)s.m[2][c] * ny + s.m[1][b]) * nx + s.m[0][a]];
                acc_rec += (double)(s.coef * s.w[0][a] * s.w[1][b] * s.w[2][c] * v);
            }
            // S(W_a, W_b) = sum over (dz, dy) rows of coef Ky Kz sum_dx Kx G[fz, fy, fx]: one
            // (pair, row) per thread and step, RR rows in flight, the row's W loads back to back;
            // row sums in FP32 (W terms of one sign pattern), the total in FP64
            const float* G = d.goct + D.oct_off;
            const int ox = D.oct[0], oy = D.oct[1];
            constexpr int WW = W * W;
            if constexpr (RR > 20) {
                // one work unit per warp and step: each lane takes EL elements (dy, dx) of the
                // unit's W x W window plane, so a load instruction reads about 32 / W consecutive
                // rows of G; the lane's loads of all W z planes are in flight together; FP32 sums
                // over the lane's EL elements, FP64 over planes.  A unit is one stencil pair, or,
                // when the trial's two stencils (a displacement's old and new charge) have the
                // same base, both of its pairs with one pending stencil: their windows are the
                // same G values (equal folded coordinates), read once and weighted twice
                static_assert(RR == 21, "one unit in flight per warp");
                constexpr int EL = (WW + 31) / 32;
                const int warp = tid >> 5, lane = tid & 31;
                const int npairs = T.npairs, np = s_npend;
                const bool merge = T.nst == 2 && np > 0 && s_tst[0].base[0] == s_tst[1].base[0] &&
                                   s_tst[0].base[1] == s_tst[1].base[1] && s_tst[0].base[2] == s_tst[1].base[2];
                const int nunit = merge ? npairs - np : npairs;
                const int oxy = oy * ox;
                for (int u = warp; u < nunit; u += NT / 32) {
                    // pairs (trial stencil 0, pending u) and (trial stencil 1, pending u) sit at u
                    // and np + u of the tables; the trial stencils' own pairs follow at 2 np
                    const int qa = (merge && u >= np) ? u + np : u;
                    const int qb = (merge && u < np) ? np + u : -1;
                    const PairK<P>& pa = s_pair[qa];
                    const PairK<P>& pb = s_pair[qb < 0 ? qa : qb];
                    int off[EL];
                    float ka[EL];
#pragma unroll
                    for (int k = 0; k < EL; ++k) {
                        const int e = min(lane + 32 * k, WW - 1);
                        const int dy = e / W, dx = e - dy * W;
                        off[k] = pa.f[1][dy] * ox + pa.f[0][dx];
                        ka[k] = (lane + 32 * k < WW) ? pa.K[1][dy] * pa.K[0][dx] : 0.0f;
                    }
                    float g[W][EL];
#pragma unroll
                    for (int dz = 0; dz < W; ++dz) {
                        const int zo = pa.f[2][dz] * oxy;
#pragma unroll
                        for (int k = 0; k < EL; ++k) g[dz][k] = __ldg(G + off[k] + zo);
                    }
#pragma unroll
                    for (int dz = 0; dz < W; ++dz) {
                        float t = 0.0f;
#pragma unroll
                        for (int k = 0; k < EL; ++k) t = fmaf(ka[k], g[dz][k], t);
                        acc_rec += (double)(pa.coef * pa.K[2][dz] * t);
                    }
                    if (qb >= 0) {
                        float kb[EL];
#pragma unroll
                        for (int k = 0; k < EL; ++k) {
                            const int e = min(lane + 32 * k, WW - 1);
                            const int dy = e / W, dx = e - dy * W;
                            kb[k] = (lane + 32 * k < WW) ? pb.K[1][dy] * pb.K[0][dx] : 0.0f;
                        }
#pragma unroll
                        for (int dz = 0; dz < W; ++dz) {
                            float t = 0.0f;
#pragma unroll
                            for (int k = 0; k < EL; ++k) t = fmaf(kb[k], g[dz][k], t);
                            acc_rec += (double)(pb.coef * pb.K[2][dz] * t);
                        }
                    }
                }
            } else {
            const int nrow = T.npairs * WW;
            for (int r0 = tid; r0 < nrow; r0 += RR * NT) {
                float gv[RR][W];
                int qv[RR], rv[RR];
#pragma unroll
                for (int u = 0; u < RR; ++u) {
                    const int rowg = min(r0 + u * NT, nrow - 1);
                    const int q = rowg / WW, rw = rowg - q * WW;
                    const int dz = rw / W, dy = rw - dz * W;
                    const PairK<P>& pk = s_pair[q];
                    const float* Grow = G + (pk.f[2][dz] * oy + pk.f[1][dy]) * ox;
#pragma unroll
                    for (int dx = 0; dx < W; ++dx) gv[u][dx] = __ldg(&Grow[pk.f[0][dx]]);
                    qv[u] = q; rv[u] = rw;
                }
#pragma unroll
                for (int u = 0; u < RR; ++u) {
                    if (r0 + u * NT >= nrow) continue;
                    const PairK<P>& pk = s_pair[qv[u]];
                    const int dz = rv[u] / W, dy = rv[u] - dz * W;
                    float s = 0.0f;
#pragma unroll
                    for (int dx = 0; dx < W; ++dx) s = fmaf(pk.K[0][dx], gv[u][dx], s);
                    acc_rec += (double)(pk.coef * pk.K[1][dy] * pk.K[2][dz] * s);
                }
            }
            }
        }
        if (q_chk && q_blocked > 0 && (float)q_blocked >= d.quorum * (float)q_started) s_qstop = 1;
        block_sum3<NT>(acc_lj, acc_c, acc_rec, red);
        mark(5);
        // ---------------- phase 5: decision and update ----------------
        if (tid == 0) {
            const Moments mo = s_mo;
            const double dQ = mo.dQ, dQ2 = mo.dQ2, dMz = mo.dMz, dS2 = mo.dS2;
            const double dself = mo.dself, dqc = mo.dqc, dslab = mo.dslab;
            const double dlj = acc_lj + T.d_direct_lj, dc = acc_c + T.d_direct_c;
            const double dE = dlj + dc + T.d_fene + acc_rec + dself + dqc + dslab;
            int accept = 0;
            if (GC) {
                if constexpr (GC) {
                    if (sG.phase == 2) {
                        int ops = 0;
                        accept = p2_decide(sG, D, S, d, dlj, dc, acc_rec, dself, dqc, dslab, &ops);
                        s_gc_ops = ops;
                    } else {
                        accept = gc_decide(sG, D, S, d, dlj, dc, acc_rec, dself, dqc, dslab);
                        s_gc_ops = accept;
                    }
                }
            } else if (mode == MC_RUN) {
                const long long li = T.tnum - S.run_start;
                if (r == 0 && d.replay && li < d.replay_n) accept = d.replay[li];
                else {
                    // delayed acceptance, second stage: the exact dE judges the surrogate's
                    // estimate (Christen & Fox 2005; the log factor cancels)
                    const double expo = T.da ? -D.beta * (dE - T.dEs) : -D.beta * dE + T.logf;
                    if (expo >= 0.0) accept = 1;
                    else {
                        // the FP64 exp only when the uniform lies within 1e-3 (relative) of a
                        // float estimate, whose error is below 1e-4 for every expo < 0: the
                        // decision is the FP64 comparison's in every case
                        const double u = u53(T.ua, T.ub);
                        const double ef = (double)__expf((float)expo);
                        if (u < ef * (1.0 - 1e-3)) accept = 1;
                        else if (u > ef * (1.0 + 1e-3)) accept = 0;
                        else accept = u < exp(expo);
                    }
                }
                if (T.da) {
                    if (accept) { S.da_acc++; S.da_wacc++; }
                    if (d.da_window > 0 && S.da_wpass >= d.da_window) {
                        if ((double)S.da_wacc < (double)d.da_threshold * (double)S.da_wpass) S.da_off = 1;
                        S.da_wpass = 0; S.da_wacc = 0;
                    }
                }
                if (T.desc && d.hv_cap > 0) {  // training sample: rows, signs, the network's target
                    const int slot = atomicAdd(d.hv_count, 1);
                    if (slot < d.hv_cap) {
                        d.hv_target[slot] = (float)(dE - T.cross - T.dmom);
                        for (int rr = 0; rr < SUR_ROWS; ++rr) d.hv_sign[(size_t)slot * SUR_ROWS + rr] = rr < T.nrows ? T.row_sign[rr] : 0.0f;
                        s_hv_slot = slot; s_hv_nrows = T.nrows;
                    }
                }
                if (r == 0 && d.log_move && li < d.log_cap) {
                    d.log_move[li] = T.move; d.log_dE[li] = dE; d.log_acc[li] = accept;
                    if (d.log_stage) { d.log_stage[li] = T.da ? 2 : 0; d.log_dEs[li] = T.da ? T.dEs : 0.0; }
                }
                S.att[T.move]++;
                // algorithmic bytes of this trial: float4+type of every candidate, the
                // moved particle, the phi stencils and the pending-correction reads
                S.alg_bytes += 20.0 * T.total_cand + 16.0 + 4.0 * P3 * T.nst + 16.0 * P3 * s_npend + (accept ? 32.0 : 0.0);
                S.trials_run++;
            } else if (mode == MC_EVAL) {
                if (ext_dE) ext_dE[T.ext_k] = dE;
            } else {
                accept = 1;
                if (ext_dE) ext_dE[T.ext_k] = dE;
            }
            if (mode != MC_RUN && d.ext_comp) {
                double* o = d.ext_comp + (size_t)T.ext_k * 7;
                o[0] = dlj; o[1] = T.d_fene; o[2] = dc; o[3] = acc_rec; o[4] = dself; o[5] = dqc; o[6] = dslab;
            }
            if (mode != MC_RUN) T.ext_k++;
            if (accept) {
                if (mode == MC_RUN) S.acc[T.move]++;
                const int so = D.slot_off;
                if (d.qband) {  // charge-mesh updates, applied by warps 1..4 in the next proposal phase
                    int nj = 0;
                    for (int k = 0; k < T.nch; ++k) {
                        const float4 o = T.po[k], nw = T.pn[k];
                        if (T.pres_old[k] && T.pres_new[k] && o.x == nw.x && o.y == nw.y && o.z == nw.z && o.w == nw.w) continue;
                        if (T.pres_old[k] && o.w != 0.0f) { s_qjob[nj] = o; s_qsgn[nj] = -1; ++nj; }
                        if (T.pres_new[k] && nw.w != 0.0f) { s_qjob[nj] = nw; s_qsgn[nj] = 1; ++nj; }
                    }
                    s_nqjob = nj;
                }
                for (int k = 0; k < T.nch; ++k) {
                    const int i = T.idx[k];
                    const int gi = so + i;
                    {  // descriptor class table: leave the old (cell, class), enter the new one
                        const int c_old = T.pres_old[k] ? cell_index(D, T.po[k].x, T.po[k].y, T.po[k].z) : -1;
                        const int k_old = T.pres_old[k] ? desc_class(T.fo[k], T.po[k].w) : -1;
                        int fl_new = T.fo[k];
                        if (!T.pres_old[k] && T.pres_new[k])
                            fl_new = PHMC_F_MOBILE | (T.pn[k].w > 0.0f ? PHMC_F_CATION : (T.pn[k].w < 0.0f ? PHMC_F_ANION : 0));
                        const int c_new = T.pres_new[k] ? cell_index(D, T.pn[k].x, T.pn[k].y, T.pn[k].z) : -1;
                        const int k_new = T.pres_new[k] ? desc_class(fl_new, T.pn[k].w) : -1;
                        if (c_old != c_new || k_old != k_new) {
                            cls_add(d, D, c_old, k_old, -1);
                            cls_add(d, D, c_new, k_new, 1);
                        }
                    }
                    if (T.pres_old[k] && T.pres_new[k]) {
                        d.posq[gi] = T.pn[k];
                        d.type[gi] = T.tn[k];
                        const int nc = cell_index(D, T.pn[k].x, T.pn[k].y, T.pn[k].z);
                        if (k == 0 && T.nch == 1 && T.nprobe == 2) {
                            // displacement: the old cell's tail and the new cell's count were
                            // loaded during the parallel phase (probe 1 = new state, entry 13 = its cell)
                            if (nc != T.cell_old[0]) {
                                const int c = T.cell_old[0], kp = T.cpos_old[0], n = T.cnt_old[0], last = T.last_old[0];
                                int* l = d.cell_list + ((size_t)D.cell_off + c) * D.cell_cap;
                                l[kp] = last;
                                d.cell_pos[so + last] = kp;
                                d.cell_count[D.cell_off + c] = n - 1;
                                const int nn = s_cnt[27 + 13];
                                if (nn >= D.cell_cap) S.error = PHMC_ERR_CAPACITY;
                                else {
                                    d.cell_list[((size_t)D.cell_off + nc) * D.cell_cap + nn] = i;
                                    d.cell_count[D.cell_off + nc] = nn + 1;
                                    d.cell_of[gi] = nc;
                                    d.cell_pos[gi] = nn;
                                }
                            }
                        } else if (nc != d.cell_of[gi]) {
                            cell_remove(d, D, i);
                            if (!cell_insert(d, D, i, nc)) S.error = PHMC_ERR_CAPACITY;
                        }
                    } else if (!T.pres_old[k] && T.pres_new[k]) {  // insertion into a free slot
                        int fk = -1;
                        for (int f = S.n_free - 1; f >= 0; --f) if (d.freel[so + f] == i) { fk = f; break; }
                        if (fk >= 0) { d.freel[so + fk] = d.freel[so + S.n_free - 1]; S.n_free--; }
                        d.posq[gi] = T.pn[k];
                        d.type[gi] = T.tn[k];
                        int fl = PHMC_F_MOBILE;
                        list_append(d.mobile, d.mobile_pos, S.n_mobile, so, i);
                        if (T.pn[k].w > 0.0f) { fl |= PHMC_F_CATION; list_append(d.cations, d.cation_pos, S.n_cation, so, i); }
                        else if (T.pn[k].w < 0.0f) { fl |= PHMC_F_ANION; list_append(d.anions, d.anion_pos, S.n_anion, so, i); }
                        d.flags[gi] = fl;
                        if (!cell_insert(d, D, i, cell_index(D, T.pn[k].x, T.pn[k].y, T.pn[k].z))) S.error = PHMC_ERR_CAPACITY;
                    } else if (T.pres_old[k] && !T.pres_new[k]) {  // deletion
                        const int fl = d.flags[gi];
                        if (fl & PHMC_F_CATION) list_remove(d.cations, d.cation_pos, S.n_cation, so, i);
                        if (fl & PHMC_F_ANION) list_remove(d.anions, d.anion_pos, S.n_anion, so, i);
                        if (fl & PHMC_F_MOBILE) list_remove(d.mobile, d.mobile_pos, S.n_mobile, so, i);
                        d.flags[gi] = PHMC_F_GHOST;
                        d.freel[so + S.n_free] = i; S.n_free++;
                        cell_remove(d, D, i);
                    }
                }
                // the trial's stencils already sit right after the pending ones
                if (s_npend + T.nst <= pend_max + NST_MAX) s_npend += T.nst;
                else S.error = PHMC_ERR_CAPACITY;
                // the next trial's prefetched particle is stale if this commit touched it or the lists
                for (int k = 0; k < T.nch; ++k)
                    if (T.idx[k] == pf.idx || T.pres_old[k] != T.pres_new[k]) pf.valid = 0;
                S.Q += dQ; S.Q2 += dQ2; S.Mz += dMz; S.S2 += dS2;
                S.E_pair_lj += dlj; S.E_pair_c += dc; S.E_fene += T.d_fene; S.E_rec += acc_rec;
                S.E_self += dself; S.E_qcorr += dqc; S.E_slab += dslab;
                S.E += dE;
            }
        }
        __syncthreads();
        if constexpr (GC) {
            const int ops = s_gc_ops;
            if (ops == 1) {  // the accepted flip's pool updates (MC/src/mc.cu:446-458)
                const bool fwd = sG.dir > 0;
                const int ka = fwd ? GC_NHN : GC_NHP, kb = fwd ? GC_NHP : GC_NHN;
                const int kc = fwd ? GC_W : GC_CL, kd = fwd ? GC_CL : GC_W;
                gc_pool_move<NT>(gc_pool(d, D, ka), gc_pool(d, D, kb), sG.n[ka], sG.n[kb], T.idx[0], &s_gc_find);
                gc_pool_move<NT>(gc_pool(d, D, kc), gc_pool(d, D, kd), sG.n[kc], sG.n[kd], T.idx[1], &s_gc_find);
            } else if (ops >= 2) {  // phase 2's accepted move (MC/src/mc.cu:252-256, 286-287)
                if (ops == 2) {
                    gc_pool_move<NT>(gc_pool(d, D, GC_NHP), gc_pool(d, D, GC_NHN), sG.n[GC_NHP], sG.n[GC_NHN], sG.iP, &s_gc_find);
                    gc_pool_move<NT>(gc_pool(d, D, GC_NHN), gc_pool(d, D, GC_NHP), sG.n[GC_NHN], sG.n[GC_NHP], sG.iN, &s_gc_find);
                }
                gc_pool_move<NT>(gc_pool(d, D, GC_CL), gc_pool(d, D, GC_W), sG.n[GC_CL], sG.n[GC_W], sG.jCl, &s_gc_find);
                gc_pool_move<NT>(gc_pool(d, D, GC_W), gc_pool(d, D, GC_CL), sG.n[GC_W], sG.n[GC_CL], sG.jW, &s_gc_find);
            }
            if (ops) {
                if (tid == 0) s_gc_ops = 0;
                __syncthreads();
            }
        }
        // z-density sample after every zh_every trials of the run (S.trial was advanced by
        // this trial's proposal before the barriers above, so every thread sees one value)
        if (!GC && mode == MC_RUN && d.zh_bins > 0 && S.trial % d.zh_every == 0) {
            const int nb = d.zh_bins;
            for (int k = tid; k < 3 * nb; k += NT) s_zh[k] = 0u;
            __syncthreads();
            const float z0 = D.walls ? D.wall_lo : 0.0f;
            const float inv = (float)nb / (D.walls ? (D.wall_hi - D.wall_lo) : D.L[2]);
            for (int i = tid; i < D.cap; i += NT) {
                const int fl = d.flags[D.slot_off + i];
                if (fl & PHMC_F_GHOST) continue;
                const float4 pq = d.posq[D.slot_off + i];
                int cls = -1;
                if (fl & PHMC_F_TITRATABLE) cls = pq.w != 0.0f ? 0 : -1;
                else if (fl & PHMC_F_ANION) cls = 1;
                else if (fl & PHMC_F_CATION) cls = 2;
                if (cls < 0) continue;
                const int b = min(max((int)((pq.z - z0) * inv), 0), nb - 1);
                atomicAdd(&s_zh[cls * nb + b], 1u);
            }
            __syncthreads();
            unsigned long long* h = d.zhist + (size_t)r * 3 * nb;  // this replica's row: one block, no race
            for (int k = tid; k < 3 * nb; k += NT) h[k] += s_zh[k];
            if (tid == 0) d.zh_samples[r] += 1;
            __syncthreads();
        }
        mark(6);
    }
    if constexpr (GC) {
        const int* src = reinterpret_cast<const int*>(&sG);
        int* dst = reinterpret_cast<int*>(d.gc + blockIdx.x);
        for (int k = tid; k < (int)(sizeof(GcDev) / sizeof(int)); k += NT) dst[k] = src[k];
    }
    if (tid == 0) {
        if (mode == MC_RUN) {
            unsigned long long t_end;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
            S.busy_ns += (long long)(t_end - t_start);
        }
        d.state[r] = S;
        if (s_npend > 0) d.dirty[r] = 1;  // potential mesh is stale: rebuild before the next MC launch
    }
}

template <int P, int NT, int RC, int RR>
static cudaError_t launch_mc_t(Engine& E, int mode, int rep, const phmc_trial* t, int n, double* dE, cudaStream_t st) {
    DevPtrs dd = E.d;
    if (E.first_stage_off) dd.sur.H = 0;  // surrogate attached but bypassed: every trial exact
    // plain Monte Carlo (no network, no harvest) takes the instance without the first stage
    const bool fs = dd.sur.H > 0 || dd.hv_cap > 0 || mode != MC_RUN;
    auto kern = fs ? k_mc<P, NT, false, RC, RR, true> : k_mc<P, NT, false, RC, RR, false>;
    size_t smem = mc_smem_bytes(P, E.pend_max, false);
    dd.sur_late_l3 = 0;
    if (dd.sur.H > 0) {
        // three staged layers when two blocks per SM still fit, else two buffers
        cudaFuncAttributes fa;
        cudaFuncGetAttributes(&fa, kern);
        int per_sm = 0;
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, E.device);
        const size_t three = mc_smem_bytes(P, E.pend_max, true);
        const bool fits2 = 2 * (three + fa.sharedSizeBytes + 1024) <= (size_t)per_sm;
        dd.sur_late_l3 = fits2 ? 0 : 1;
        smem = fits2 ? three : mc_smem_bytes(P, E.pend_max, true, true);
    }
    const int grid = (mode == MC_RUN) ? E.R : 1;
    // launch quorum only when every replica's block is resident from the start (otherwise
    // late blocks would count against a quorum the early ones already reached)
    dd.quorum = 1.0f;
    if (mode == MC_RUN && E.quorum < 1.0f) {
        int per_sm = 0, nsm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, E.device);
        if ((long long)per_sm * nsm >= E.R) {
            dd.quorum = E.quorum;
            cudaError_t e = cudaMemsetAsync(E.d.quorum_ctl, 0, 2 * sizeof(int), st);
            if (e != cudaSuccess) return e;
        }
    }
    kern<<<grid, NT, smem, st>>>(dd, mode, rep, t, n, dE, E.pend_max);
    return cudaGetLastError();
}

// One block per job of the grand-canonical phase (128 threads; no surrogate, no quorum).
template <int P>
static cudaError_t launch_mc_gc_t(Engine& E, int n_jobs, cudaStream_t st) {
    DevPtrs dd = E.d;
    dd.quorum = 1.0f;
    dd.ext_comp = nullptr;
    dd.hv_cap = 0;
    dd.log_move = nullptr;
    dd.replay = nullptr;
    dd.sur.H = 0;
    const size_t smem = mc_smem_bytes(P, E.pend_max, false);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_mc<P, 128, true, 4, 2, false>);
    if (e != cudaSuccess) return e;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, E.device);
    if (e != cudaSuccess) return e;
    if (smem + fa.sharedSizeBytes > (size_t)optin) return cudaErrorInvalidValue;
    e = cudaFuncSetAttribute(k_mc<P, 128, true, 4, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_mc<P, 128, true, 4, 2, false><<<n_jobs, 128, smem, st>>>(dd, MC_GC, 0, nullptr, 0, nullptr, E.pend_max);
    return cudaGetLastError();
}

cudaError_t launch_mc_gc(Engine& E, int n_jobs, cudaStream_t st) {
    switch (E.order) {
        case 4: return launch_mc_gc_t<4>(E, n_jobs, st);
        case 5: return launch_mc_gc_t<5>(E, n_jobs, st);
        default: return launch_mc_gc_t<6>(E, n_jobs, st);
    }
}

// Raise the dynamic shared-memory cap of the engine's MC kernel instance to the
// device maximum (minus its static shared memory), once, outside any capture.
template <int P, int NT, int RC, int RR>
static cudaError_t prepare_mc_t(Engine& E) {
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, E.device);
    if (e != cudaSuccess) return e;
    for (int fs = 0; fs < 2; ++fs) {  // with and without the first stage
        auto kern = fs ? k_mc<P, NT, false, RC, RR, true> : k_mc<P, NT, false, RC, RR, false>;
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        const int cap = optin - (int)fa.sharedSizeBytes;
        if ((size_t)cap < mc_smem_bytes(P, E.pend_max, true)) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The compiled (order, round width, G rows) variants: order 5 (the configurations' order)
// has seven pair-pass shapes, orders 4 and 6 the default one.  f gets the four template
// values as integral constants; an unsupported combination gives cudaErrorInvalidValue.
template <int V>
using IC = std::integral_constant<int, V>;
template <class F>
static cudaError_t mc_dispatch(const Engine& E, F&& f) {
    const bool t128 = E.threads == 128;
    const int rc = E.cand_round, rr = E.g_rows;
#define MC_VARIANT(p, c, g) \
    if (rc == c && rr == g) return t128 ? f(IC<p>{}, IC<128>{}, IC<c>{}, IC<g>{}) : f(IC<p>{}, IC<256>{}, IC<c>{}, IC<g>{});
    switch (E.order) {
        case 4: MC_VARIANT(4, 4, 2) break;
        case 5:
            MC_VARIANT(5, 4, 2) MC_VARIANT(5, 2, 2) MC_VARIANT(5, 8, 2) MC_VARIANT(5, 2, 3) MC_VARIANT(5, 2, 4)
            MC_VARIANT(5, 2, 21) MC_VARIANT(5, 4, 21) break;
        default: MC_VARIANT(6, 4, 2) break;
    }
#undef MC_VARIANT
    return cudaErrorInvalidValue;
}

cudaError_t prepare_mc(Engine& E) {
    return mc_dispatch(E, [&](auto p, auto nt, auto rc, auto rr) {
        return prepare_mc_t<decltype(p)::value, decltype(nt)::value, decltype(rc)::value, decltype(rr)::value>(E);
    });
}

size_t mc_smem_bytes(int order, int pend_max, bool staged_surrogate, bool two_buffers) {
    size_t st = 0, pk = 0;
    switch (order) {
        case 4: st = sizeof(Stencil<4>); pk = sizeof(PairK<4>); break;
        case 5: st = sizeof(Stencil<5>); pk = sizeof(PairK<5>); break;
        default: st = sizeof(Stencil<6>); pk = sizeof(PairK<6>); break;
    }
    // Monte Carlo trials carry <= 2 stencils against <= pend_max pending ones;
    // external trials (<= NST_MAX stencils) always start with none pending
    const size_t npairs = std::max((size_t)2 * pend_max + 3, (size_t)(NST_MAX * (NST_MAX + 1) / 2));
    // with a surrogate attached the pair tables' space also holds its activations and staged weights
    const size_t sur = staged_surrogate ? (size_t)(two_buffers ? SUR_SMEM2_BYTES : SUR_SMEM_BYTES) : (size_t)0;
    return st * (pend_max + NST_MAX) + std::max(pk * npairs, sur);
}

cudaError_t launch_mc(Engine& E, int mode, int rep, const phmc_trial* t, int n, double* dE, cudaStream_t st) {
    return mc_dispatch(E, [&](auto p, auto nt, auto rc, auto rr) {
        return launch_mc_t<decltype(p)::value, decltype(nt)::value, decltype(rc)::value, decltype(rr)::value>(
            E, mode, rep, t, n, dE, st);
    });
}
