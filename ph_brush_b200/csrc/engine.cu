// C-ABI implementation of the phmc engine (include/phmc.h): replica layout,
// uploads, influence-kernel construction, the trial/rebuild loop and state
// readback.  All entry points return a status code and never throw.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>
#include "engine.h"

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define CU(x)                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) return fail(PHMC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void phmc_set_error(int code, const std::string& msg) { (void)fail(code, msg); }

extern "C" int phmc_abi_version(void) { return PHMC_ABI_VERSION; }
extern "C" const char* phmc_last_error(void) { return g_err.c_str(); }

struct phmc_engine {
    Engine E;
    // trial log (host destinations)
    int* h_log_move = nullptr; double* h_log_dE = nullptr; int* h_log_acc = nullptr; long long log_cap = 0;
    int* d_replay = nullptr; long long replay_n = 0;
    long long replay_cap = 0;
    phmc_trial* d_trials = nullptr; double* d_dE = nullptr; int trials_cap = 0;
    std::vector<int> caps;
    // measurement
    bool profiling = false;
    int64_t clk_trials0 = 0;  // trials run by all replicas when the phase clocks were last switched or reset
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<size_t, size_t>> ev_mc, ev_flush;  // (start, end) indices into ev_pool
    phmc_profile prof{};
    void* l2_scratch = nullptr;
    int64_t l2_bytes = 0;
    std::vector<int> n_present;  // present particles per replica (for the rebuild byte model)
    // captured trial/rebuild chunks (re-captured when the launch set-up changes)
    cudaGraphExec_t graph_exec = nullptr;
    int graph_chunks = 0;
    bool graph_prof = false;
    std::vector<cudaEvent_t> gev;  // 4 per chunk when profiling
    // delayed-acceptance log destinations (host)
    int* h_da_stage = nullptr; double* h_da_dEs = nullptr;
    // device staging of state uploads / readbacks (allocated on first use, total_slots long)
    float *st_x = nullptr, *st_y = nullptr, *st_z = nullptr, *st_q = nullptr;
    int *st_t = nullptr, *st_f = nullptr, *st_err = nullptr, *st_cnt = nullptr;
    int* d_charged = nullptr;  // per replica charged-site counts of the last run
    // grand-canonical phase: job states, pools, events (allocated on first use)
    GcDev* d_gc = nullptr;
    int* d_gc_pool = nullptr;
    unsigned char* d_gc_ev = nullptr;
    // MC launches one run / phase call may make (0: only the no-progress guard)
    long long launch_budget = 0;
    // streaming of the device phases' event records
    phmc_event_fn ev_fn = nullptr;
    void* ev_user = nullptr;
};

static void drop_graph(phmc_engine* h) {
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
    h->graph_chunks = 0;
}

static int flush_dirty(phmc_engine* h);

// Make z-pass variant `id` the active one (0: the shared-memory Stockham pass; else a
// register split of the engines' common nz): job table, its per-replica offsets and the
// shared memory the kernel needs.  The caller raises the kernel's shared-memory cap.
static void select_zpass(Engine& E, int id) {
    E.zreg = id;
    if (id) { E.d_zjobs = E.d_zj_reg; E.n_zjobs = E.n_zj_reg; E.d_zjob_off = E.d_zoff_reg; E.zpass_smem = E.zpass_smem_reg; }
    else { E.d_zjobs = E.d_zj_stk; E.n_zjobs = E.n_zj_stk; E.d_zjob_off = E.d_zoff_stk; E.zpass_smem = E.zpass_smem_stk; }
}

// Capture `chunks` x (MC launch + potential-mesh rebuild) on the engine stream.
static int build_chunk_graph(phmc_engine* h, int chunks) {
    Engine& E = h->E;
    if (h->graph_exec && h->graph_chunks == chunks && h->graph_prof == h->profiling) return PHMC_OK;
    drop_graph(h);
    while ((int)h->gev.size() < 4 * chunks) {
        cudaEvent_t ev;
        CU(cudaEventCreate(&ev));
        h->gev.push_back(ev);
    }
    CU(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t err = cudaSuccess;
    int s = PHMC_OK;
    for (int k = 0; k < chunks && err == cudaSuccess && s == PHMC_OK; ++k) {
        if (h->profiling) err = cudaEventRecordWithFlags(h->gev[4 * k], E.stream, cudaEventRecordExternal);
        if (err == cudaSuccess) err = launch_mc(E, MC_RUN, 0, nullptr, 0, nullptr, E.stream);
        if (err == cudaSuccess && h->profiling) err = cudaEventRecordWithFlags(h->gev[4 * k + 1], E.stream, cudaEventRecordExternal);
        if (err == cudaSuccess && E.coulomb == PHMC_COUL_EWALD) {
            if (h->profiling) err = cudaEventRecordWithFlags(h->gev[4 * k + 2], E.stream, cudaEventRecordExternal);
            if (err == cudaSuccess) s = flush_dirty(h);
            if (err == cudaSuccess && s == PHMC_OK && h->profiling) err = cudaEventRecordWithFlags(h->gev[4 * k + 3], E.stream, cudaEventRecordExternal);
        }
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(E.stream, &g);
    if (err != cudaSuccess) { if (g) cudaGraphDestroy(g); return fail(PHMC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(err)); }
    if (s != PHMC_OK) { if (g) cudaGraphDestroy(g); return s; }
    if (e2 != cudaSuccess) return fail(PHMC_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e2));
    cudaError_t e3 = cudaGraphInstantiate(&h->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) { h->graph_exec = nullptr; return fail(PHMC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e3)); }
    h->graph_chunks = chunks;
    h->graph_prof = h->profiling;
    return PHMC_OK;
}


template <typename T>
static int dalloc(Engine& E, T** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * n);
    if (e != cudaSuccess) return fail(PHMC_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    E.allocs.push_back((void*)*p);
    return PHMC_OK;
}
#define DALLOC(p, n) do { int s_ = dalloc(E, &(p), (n)); if (s_) return s_; } while (0)

static bool smooth235(int n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5}) while (n % p == 0) n /= p;
    return n == 1;
}

// |DFT(M_p)|^2 on a length-n grid from the cardinal B-spline values at the
// integer points (de Boor recursion, restating MC/src/pme.cu:77-113).
// ref_style 1: the reference's clamp (exact zero -> 1e-30) and Nyquist patch;
// ref_style 0: a modulus below 1e-7 (odd orders at Nyquist) is replaced by the
// mean of its neighbours.
static std::vector<double> bspline_moduli(int n, int order, int ref_style) {
    const int s = order - 1;
    std::vector<double> d((size_t)s, 0.0);
    d[0] = 1.0;
    for (int k = 2; k <= s; ++k) {
        const double inv = 1.0 / k;
        for (int m = k - 1; m > 0; --m) d[m] = inv * ((k - m) * d[m - 1] + (m + 1) * d[m]);
        d[0] = inv * d[0];
    }
    std::vector<double> mod((size_t)n);
    for (int i = 0; i < n; ++i) {
        double c = 0, sn = 0;
        for (int j = 0; j < s; ++j) {
            const double a = 2.0 * M_PI * i * (j + 1) / (double)n;
            c += d[j] * std::cos(a);
            sn += d[j] * std::sin(a);
        }
        double v = c * c + sn * sn;
        if (ref_style && !(v > 0.0)) v = 1e-30;
        mod[i] = v;
    }
    if (ref_style) {
        if (n % 2 == 0 && !(mod[n / 2] > 0.0)) mod[n / 2] = mod[n / 2 - 1];
    } else {
        std::vector<double> c = mod;
        for (int i = 0; i < n; ++i)
            if (c[i] < 1e-7) mod[i] = 0.5 * (c[(i - 1 + n) % n] + c[(i + 1) % n]);
    }
    return mod;
}

static int validate(int R, const phmc_system* sys, const phmc_params* prm) {
    if (R < 1 || !sys || !prm) return fail(PHMC_ERR_ARG, "phmc_create: need n_replicas >= 1 and non-null systems/params");
    for (int r = 0; r < R; ++r) {
        const phmc_system& S = sys[r];
        const phmc_params& P = prm[r];
        char b[256];
        if (S.n_particles < 0 || S.capacity < S.n_particles || S.capacity < 1) {
            snprintf(b, sizeof b, "replica %d: invalid n_particles/capacity (%d/%d)", r, S.n_particles, S.capacity);
            return fail(PHMC_ERR_ARG, b);
        }
        if (S.n_particles > 0 && (!S.x || !S.y || !S.z || !S.q || !S.type || !S.flags)) return fail(PHMC_ERR_ARG, "null particle array");
        if (!(S.box[0] > 0 && S.box[1] > 0 && S.box[2] > 0)) return fail(PHMC_ERR_ARG, "box lengths must be > 0");
        if (P.n_types < 1 || P.n_types > PHMC_MAX_TYPES || !P.lj_eps || !P.lj_sig)
            return fail(PHMC_ERR_ARG, "n_types must be 1..8 with LJ tables");
        for (int i = 0; i < S.n_particles; ++i) {
            if (S.type[i] < 0 || S.type[i] >= P.n_types) { snprintf(b, sizeof b, "replica %d: particle %d type %d out of range", r, i, S.type[i]); return fail(PHMC_ERR_ARG, b); }
            if (!(S.flags[i] & PHMC_F_GHOST)) {
                if (!(S.x[i] >= 0 && S.x[i] < S.box[0] && S.y[i] >= 0 && S.y[i] < S.box[1] && S.z[i] >= 0 && S.z[i] < S.box[2])) {
                    snprintf(b, sizeof b, "replica %d: particle %d outside [0,L) (wrap positions first)", r, i);
                    return fail(PHMC_ERR_ARG, b);
                }
            }
        }
        for (int k = 0; k < S.n_bonds; ++k)
            if (S.bond_i[k] < 0 || S.bond_i[k] >= S.n_particles || S.bond_j[k] < 0 || S.bond_j[k] >= S.n_particles || S.bond_i[k] == S.bond_j[k])
                return fail(PHMC_ERR_ARG, "bond index out of range");
        if (P.coulomb < 0 || P.coulomb > 2) return fail(PHMC_ERR_ARG, "coulomb kind");
        if (P.coulomb != PHMC_COUL_NONE && !(P.epsilon_r > 0)) return fail(PHMC_ERR_ARG, "epsilon_r must be > 0");
        if (P.coulomb == PHMC_COUL_EWALD) {
            if (!(P.ewald_alpha > 0)) return fail(PHMC_ERR_ARG, "ewald_alpha must be > 0");
            if (P.order < 4 || P.order > 6) return fail(PHMC_ERR_UNSUPPORTED, "SPME order must be 4, 5 or 6");
            if (P.order != prm[0].order) return fail(PHMC_ERR_UNSUPPORTED, "all replicas must share the SPME order");
            for (int k = 0; k < 3; ++k)
                if (!smooth235(P.mesh[k]) || P.mesh[k] < P.order) return fail(PHMC_ERR_UNSUPPORTED, "mesh sizes must be 2^a 3^b 5^c and >= order");
            if ((size_t)P.mesh[0] * P.mesh[1] * 16 > 227 * 1024) return fail(PHMC_ERR_UNSUPPORTED, "mesh plane nx*ny too large for one block");
            if ((size_t)P.mesh[2] * ZPASS_TX * 16 > 227 * 1024) return fail(PHMC_ERR_UNSUPPORTED, "mesh nz too large for one block");
        }
        if (!(P.beta > 0)) return fail(PHMC_ERR_ARG, "beta must be > 0");
        if (P.p_disp < 0 || P.p_titr < 0 || P.p_swap < 0 || P.p_disp + P.p_titr + P.p_swap > 1.0 + 1e-12)
            return fail(PHMC_ERR_ARG, "move probabilities must be >= 0 with sum <= 1");
        if (P.p_swap > 0 && !(P.salt_conc > 0)) return fail(PHMC_ERR_ARG, "swap moves need salt_conc > 0");
    }
    return PHMC_OK;
}

static int build(phmc_engine* h, int R, const phmc_system* sys, const phmc_params* prm, int device) {
    Engine& E = h->E;
    E.R = R;
    E.device = device;
    CU(cudaSetDevice(device));
    CU(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
    E.order = prm[0].order;
    E.coulomb = prm[0].coulomb;
    E.threads = prm[0].threads == 128 ? 128 : 256;
    E.pend_max = prm[0].pending_max > 0 ? std::min(std::max(prm[0].pending_max, 4), PHMC_MAX_PEND) : 48;
    E.cell_cap = prm[0].cell_cap > 0 ? prm[0].cell_cap : 64;
    for (int r = 1; r < R; ++r)
        if (prm[r].coulomb != E.coulomb) return fail(PHMC_ERR_UNSUPPORTED, "all replicas must share the Coulomb kind");
    const bool ewald = E.coulomb == PHMC_COUL_EWALD;

    // ---- descriptors ----
    E.desc.resize(R);
    std::vector<double> h_mod;
    std::vector<float2> h_th;
    std::vector<float2> h_tw;
    std::map<int, int> tw_off;
    auto tw_table = [&](int n) {  // exp(-2 pi i j / n), j < n, one table per distinct length
        auto it = tw_off.find(n);
        if (it != tw_off.end()) return it->second;
        const int off = (int)h_tw.size();
        tw_off[n] = off;
        for (int j = 0; j < n; ++j) h_tw.push_back(make_float2((float)std::cos(-2.0 * M_PI * j / n), (float)std::sin(-2.0 * M_PI * j / n)));
        return off;
    };
    int slot_off = 0, cell_off = 0;
    long long mesh_off = 0, meshh_off = 0, oct_off = 0, qband_off = 0;
    E.use_r2c = ewald;
    for (int r = 0; r < R; ++r)
        if (prm[r].mesh[0] % 2 != 0) E.use_r2c = false;
    for (int r = 0; r < R; ++r) {
        const phmc_system& S = sys[r];
        const phmc_params& P = prm[r];
        RepDesc& D = E.desc[r];
        std::memset(&D, 0, sizeof(D));
        D.cap = S.capacity; D.slot_off = slot_off; slot_off += S.capacity;
        for (int k = 0; k < 3; ++k) D.L[k] = (float)S.box[k];
        D.V = S.box[0] * S.box[1] * S.box[2];
        D.T = P.n_types;
        double rmax = 0.0;
        for (int a = 0; a < D.T; ++a)
            for (int b = 0; b < D.T; ++b) {
                const int k = a * D.T + b;
                const double eps = P.lj_eps[k], sig = P.lj_sig[k];
                const double rc = P.lj_rc ? P.lj_rc[k] : P.rc_lj;
                D.lj_eps[k] = (eps > 0 && sig > 0) ? (float)eps : 0.0f;
                D.lj_sig2[k] = (float)(sig * sig);
                D.lj_rc2[k] = (float)(rc * rc);
                double sh = 0.0;
                if (P.lj_shift && eps > 0 && sig > 0) {
                    const double sr6 = std::pow(sig / rc, 6);
                    sh = 4.0 * eps * (sr6 * sr6 - sr6);
                }
                D.lj_shift[k] = (float)sh;
                if (eps > 0 && sig > 0) rmax = std::max(rmax, rc);
            }
        D.coulomb = P.coulomb;
        if (P.coulomb != PHMC_COUL_NONE) rmax = std::max(rmax, P.rc_coul);
        if (!(rmax > 0)) rmax = 1.0;
        for (int k = 0; k < 3; ++k) {
            D.ncell[k] = (int)std::floor(S.box[k] / rmax);
            if (D.ncell[k] < 3) return fail(PHMC_ERR_UNSUPPORTED, "box must hold at least 3 cells of the largest cutoff per axis");
            D.cell_scale[k] = (float)D.ncell[k] / D.L[k];
            // surrogate descriptor: cell widths and the cell range of the 8-sigma sphere
            D.cell_w[k] = D.L[k] / (float)D.ncell[k];
            D.dnr[k] = std::max(1, (int)std::ceil((double)SUR_RMAX * D.ncell[k] / S.box[k]));
            D.dnk[k] = std::min(2 * D.dnr[k] + 1, D.ncell[k]);
            // when the range covers the whole axis, centre the window so that it holds the
            // neighbours -1, 0, +1 (the inner cells) and every other cell once
            if (D.dnk[k] < 2 * D.dnr[k] + 1) D.dnr[k] = (D.dnk[k] - 1) / 2;
        }
        D.cell_off = cell_off; cell_off += D.ncell[0] * D.ncell[1] * D.ncell[2];
        D.cell_cap = E.cell_cap;
        const double elf = 138.935458 / (P.epsilon_r > 0 ? P.epsilon_r : 1.0);
        D.elf = (float)elf;
        D.alpha = (float)P.ewald_alpha;
        D.rc_coul2 = (float)(P.rc_coul * P.rc_coul);
        D.ewald_factor = ewald ? (float)((M_PI / P.ewald_alpha) * (M_PI / P.ewald_alpha)) : 0.0f;
        D.slab = P.slab;
        D.ref_corner = P.ref_moduli;
        D.order = E.order;
        D.walls = P.wall_hi > P.wall_lo;
        D.wall_lo = (float)P.wall_lo; D.wall_hi = (float)P.wall_hi;
        D.sur_z0 = D.walls ? D.wall_lo : 0.0f;
        D.sur_h = D.walls ? D.wall_hi - D.wall_lo : D.L[2];
        D.sur_pk = (float)(P.pKa - P.pH);
        D.sur_salt = P.salt_conc > 0 ? (float)std::log10(P.salt_conc) : -10.0f;
        D.fene_k = (float)P.fene_k; D.fene_r02 = (float)(P.fene_r0 * P.fene_r0);
        D.excl_lj = P.excl_bonded_lj; D.excl_coul = P.excl_bonded_coul;
        D.beta = P.beta;
        D.titr_log = std::log(10.0) * (P.pKa - P.pH);
        const double Vs = (double)D.L[0] * (double)D.L[1] * (D.walls ? (double)(D.wall_hi - D.wall_lo) : (double)D.L[2]);
        D.salt_c2V2 = P.salt_conc * P.salt_conc * Vs * Vs;
        D.p_disp = (float)P.p_disp; D.p_titr = (float)P.p_titr; D.p_swap = (float)P.p_swap; D.disp_max = (float)P.disp_max;
        D.type_site_neutral = P.type_site_neutral; D.type_site_charged = P.type_site_charged;
        D.type_counterion = P.type_counterion; D.type_cation = P.type_cation;
        D.q_site_charged = P.q_site_charged; D.q_counterion = P.q_counterion; D.q_cation = P.q_cation;
        D.key[0] = (uint32_t)(P.seed & 0xffffffffu); D.key[1] = (uint32_t)(P.seed >> 32);
        D.pend_max = E.pend_max;
        if (ewald) {
            D.self_coef = -elf * P.ewald_alpha / std::sqrt(M_PI);
            D.qcorr_coef = -(M_PI * elf) / (2.0 * D.V * P.ewald_alpha * P.ewald_alpha);
            D.slab_coef = (2.0 * M_PI / D.V) * elf;
            D.Lz2_12 = S.box[2] * S.box[2] / 12.0;
            for (int k = 0; k < 3; ++k) {
                D.mesh[k] = P.mesh[k];
                D.oct[k] = P.mesh[k] / 2 + 1;
                std::vector<double> m = bspline_moduli(P.mesh[k], P.order, P.ref_moduli);
                D.mod_off[k] = (int)h_mod.size();
                h_mod.insert(h_mod.end(), m.begin(), m.end());
                // the influence function factorises per axis: theta(k) = elf exp(-(pi/alpha)^2 |k|^2) /
                // (pi V |k|^2 Bx By Bz); per axis (exp(-(pi/alpha)^2 k^2) / B(k), k^2) in FP64, rounded
                // once (a zero modulus gives a zero factor, as the reference's den > 0 test does)
                D.th_off[k] = (int)h_th.size();
                const double ef = (M_PI / P.ewald_alpha) * (M_PI / P.ewald_alpha);
                for (int j = 0; j < P.mesh[k]; ++j) {
                    const int mj = (j <= P.mesh[k] / 2) ? j : j - P.mesh[k];
                    const double kk = (double)mj / (double)D.L[k];
                    const double f = (m[j] > 0.0) ? std::exp(-ef * kk * kk) / m[j] : 0.0;
                    h_th.push_back(make_float2((float)f, (float)(kk * kk)));
                }
                D.tw_off[k] = tw_table(P.mesh[k]);
            }
            D.tw_off_h = (P.mesh[0] % 2 == 0) ? tw_table(P.mesh[0] / 2) : 0;
            D.th_c = (float)(elf / (M_PI * D.V));
            // planes a charge inside the walls can reach: floor(g_z) of z in [wall_lo, wall_hi]
            // (one plane of rounding margin either side) + the stencil offsets
            // [P/2 - P + 1, P/2]; the rebuild computes and reads only these
            D.zb_lo = 0; D.zb_n = D.mesh[2];
            if (D.walls) {
                const double g = (double)D.mesh[2] / (double)D.L[2];
                const int lo = (int)std::floor(P.wall_lo * g) - 1 + E.order / 2 - E.order + 1;
                const int hi = (int)std::floor(P.wall_hi * g) + 1 + E.order / 2;
                if (hi - lo + 1 < D.mesh[2]) { D.zb_lo = ((lo % D.mesh[2]) + D.mesh[2]) % D.mesh[2]; D.zb_n = hi - lo + 1; }
            }
            D.qb_off = qband_off; qband_off += (long long)D.mesh[0] * D.mesh[1] * D.zb_n;
            D.mesh_off = mesh_off; mesh_off += (long long)D.mesh[0] * D.mesh[1] * D.mesh[2];
            D.meshh_off = meshh_off; meshh_off += (long long)(D.mesh[0] / 2 + 1) * D.mesh[1] * D.mesh[2];
            D.oct_off = oct_off; oct_off += (long long)D.oct[0] * D.oct[1] * D.oct[2];
        }
    }
    E.total_slots = slot_off;
    E.total_cells = cell_off;
    E.total_mesh = mesh_off;
    E.total_meshh = meshh_off;
    E.total_qband = qband_off;
    E.total_oct = oct_off;

    // ---- host particle arrays + lists ----
    const int N = E.total_slots;
    std::vector<float4> h_posq((size_t)N, make_float4(0, 0, 0, 0));
    std::vector<int> h_type((size_t)N, 0), h_flags((size_t)N, PHMC_F_GHOST), h_rep((size_t)N);
    std::vector<int4> h_bonds((size_t)N, make_int4(-1, -1, -1, -1));
    std::vector<int> h_mobile((size_t)N, -1), h_mpos((size_t)N, -1), h_an((size_t)N, -1), h_apos((size_t)N, -1);
    std::vector<int> h_cat((size_t)N, -1), h_cpos((size_t)N, -1), h_free((size_t)N, -1), h_titr((size_t)N, -1);
    std::vector<RepState> h_state((size_t)R);
    for (int r = 0; r < R; ++r) {
        const phmc_system& S = sys[r];
        RepDesc& D = E.desc[r];
        RepState& st = h_state[r];
        std::memset(&st, 0, sizeof(st));
        const int so = D.slot_off;
        for (int i = 0; i < D.cap; ++i) h_rep[so + i] = r;
        for (int i = 0; i < S.n_particles; ++i) {
            h_posq[so + i] = make_float4(S.x[i], S.y[i], S.z[i], S.q[i]);
            h_type[so + i] = S.type[i];
            h_flags[so + i] = S.flags[i];
        }
        for (int k = 0; k < S.n_bonds; ++k) {
            int ends[2] = {S.bond_i[k], S.bond_j[k]};
            for (int e = 0; e < 2; ++e) {
                int4& b = h_bonds[so + ends[e]];
                const int other = ends[1 - e];
                if (b.x == other || b.y == other || b.z == other || b.w == other) continue;
                if (b.x < 0) b.x = other; else if (b.y < 0) b.y = other; else if (b.z < 0) b.z = other; else if (b.w < 0) b.w = other;
                else return fail(PHMC_ERR_UNSUPPORTED, "more than 4 bonds on one particle");
            }
        }
        int nt = 0;
        for (int i = 0; i < D.cap; ++i) {
            const int f = h_flags[so + i];
            if (f & PHMC_F_GHOST) continue;
            if (f & PHMC_F_MOBILE) { h_mpos[so + i] = st.n_mobile; h_mobile[so + st.n_mobile++] = i; }
            if (f & PHMC_F_TITRATABLE) h_titr[so + nt++] = i;
            if (f & PHMC_F_ANION) { h_apos[so + i] = st.n_anion; h_an[so + st.n_anion++] = i; }
            if (f & PHMC_F_CATION) { h_cpos[so + i] = st.n_cation; h_cat[so + st.n_cation++] = i; }
        }
        D.n_titr = nt;
        for (int i = D.cap - 1; i >= 0; --i)
            if (h_flags[so + i] & PHMC_F_GHOST) h_free[so + st.n_free++] = i;
    }

    // ---- device allocations ----
    DevPtrs& d = E.d;
    DALLOC(d.posq, N); DALLOC(d.type, N); DALLOC(d.flags, N); DALLOC(d.bonds, N);
    DALLOC(d.cell_of, N); DALLOC(d.cell_pos, N);
    DALLOC(d.cell_count, E.total_cells); DALLOC(d.cell_list, (size_t)E.total_cells * E.cell_cap);
    DALLOC(d.cell_cls, E.total_cells);
    DALLOC(d.mobile, N); DALLOC(d.mobile_pos, N); DALLOC(d.anions, N); DALLOC(d.anion_pos, N);
    DALLOC(d.cations, N); DALLOC(d.cation_pos, N); DALLOC(d.freel, N); DALLOC(d.titr, N);
    DALLOC(d.desc, R); DALLOC(d.state, R); DALLOC(d.dirty, R);
    DALLOC(d.quorum_ctl, 2);
    d.quorum = 1.0f;
    DALLOC(E.d_rep_of, N);
    DALLOC(E.d_cell_rep, E.total_cells);
    int maxcap = 0;
    for (int r = 0; r < R; ++r) maxcap = std::max(maxcap, E.desc[r].cap);
    E.energy_blocks = std::max(1, std::min(PHMC_FULL_MAX_BPR, (maxcap + 127) / 128));
    E.max_cap = maxcap;
    for (const RepDesc& D : E.desc) E.max_cells = std::max(E.max_cells, D.ncell[0] * D.ncell[1] * D.ncell[2]);
    DALLOC(d.partials, (size_t)R * PHMC_FULL_MAX_BPR * 8);  // any energy_block's blocks per replica
    DALLOC(E.d_active, 1);
    CU(cudaMallocHost((void**)&E.h_active, sizeof(int)));

    CU(cudaMemcpy(d.posq, h_posq.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.type, h_type.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.flags, h_flags.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.bonds, h_bonds.data(), sizeof(int4) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.mobile, h_mobile.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.mobile_pos, h_mpos.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.anions, h_an.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.anion_pos, h_apos.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.cations, h_cat.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.cation_pos, h_cpos.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.freel, h_free.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.titr, h_titr.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(E.d_rep_of, h_rep.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.desc, E.desc.data(), sizeof(RepDesc) * R, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.state, h_state.data(), sizeof(RepState) * R, cudaMemcpyHostToDevice));
    CU(cudaMemset(d.dirty, 0, sizeof(int) * R));
    {
        std::vector<int> hc((size_t)E.total_cells);
        for (int r = 0; r < R; ++r) {
            const RepDesc& D = E.desc[r];
            for (int c = 0; c < D.ncell[0] * D.ncell[1] * D.ncell[2]; ++c) hc[(size_t)D.cell_off + c] = r;
        }
        CU(cudaMemcpy(E.d_cell_rep, hc.data(), sizeof(int) * hc.size(), cudaMemcpyHostToDevice));
    }
    h->caps.resize(R);
    for (int r = 0; r < R; ++r) h->caps[r] = E.desc[r].cap;
    h->n_present.assign(R, 0);
    for (int r = 0; r < R; ++r)
        for (int i = 0; i < E.desc[r].cap; ++i)
            if (!(h_flags[E.desc[r].slot_off + i] & PHMC_F_GHOST)) h->n_present[r]++;

    // ---- mesh ----
    if (ewald) {
        // even nx everywhere: the wall band's fixed-point charge mesh (kept by the MC kernel) +
        // half-spectrum (real-to-complex) rebuild; otherwise the scatter + full-complex path
        if (E.use_r2c) {
            DALLOC(d.cmesh, E.total_meshh);
            DALLOC(d.qband, E.total_qband);
        } else {
            DALLOC(d.qfix, E.total_mesh); DALLOC(d.cmesh, E.total_mesh);
        }
        DALLOC(d.phi, E.total_mesh);
        E.flush_kernels = E.use_r2c ? 4 : 5;
        DALLOC(d.goct, E.total_oct);
        DALLOC(d.moduli, h_mod.size()); DALLOC(d.twiddle, h_tw.size()); DALLOC(d.thtab, h_th.size());
        CU(cudaMemcpy(d.thtab, h_th.data(), sizeof(float2) * h_th.size(), cudaMemcpyHostToDevice));
        std::vector<float> hm(h_mod.begin(), h_mod.end());
        CU(cudaMemcpy(d.moduli, hm.data(), sizeof(float) * hm.size(), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(d.twiddle, h_tw.data(), sizeof(float2) * h_tw.size(), cudaMemcpyHostToDevice));
        if (!E.use_r2c) CU(cudaMemset(d.qfix, 0, sizeof(unsigned long long) * E.total_mesh));
        std::vector<int2> pj, pjb;  // all planes; the wall band's planes
        std::vector<int4> zj, zjr;  // z-pass jobs: shared-memory (Stockham) pass; register pass
        std::vector<int> zoff, zoffr;
        // register z pass possible when every replica has the same nz with a register variant
        E.zreg_default = E.use_r2c ? zreg_variant(E.desc[0].mesh[2]) : 0;
        E.plane_reg = E.use_r2c;
        for (int r = 0; r < R && E.plane_reg; ++r)
            if (!plane_reg_supported(E.desc[r].mesh[0], E.desc[r].mesh[1])) E.plane_reg = false;
        for (int r = 1; r < R && E.zreg_default; ++r)
            if (E.desc[r].mesh[2] != E.desc[0].mesh[2]) E.zreg_default = 0;
        for (int r = 0; r < R; ++r) {
            const RepDesc& D = E.desc[r];
            for (int z = 0; z < D.mesh[2]; ++z) pj.push_back(make_int2(r, z));
            for (int i = 0; i < D.zb_n; ++i) pjb.push_back(make_int2(r, (D.zb_lo + i) % D.mesh[2]));
            zoff.push_back((int)zj.size());
            zoffr.push_back((int)zjr.size());
            if (E.use_r2c) {
                // column tiles of near-equal width <= ZPASS_TX over the nx/2+1 half-spectrum columns
                const int nxh = D.mesh[0] / 2 + 1;
                if (E.zreg_default) {
                    // ZREG_TX consecutive columns of the flattened ny x nxh plane per job
                    const int ncol = nxh * D.mesh[1];
                    for (int c0 = 0; c0 < ncol; c0 += ZREG_TX) zjr.push_back(make_int4(r, c0, std::min(ZREG_TX, ncol - c0), 0));
                    E.zpass_smem_reg = std::max(E.zpass_smem_reg, zreg_smem(D.mesh[2]));
                }
                const int nt = (nxh + ZPASS_TX - 1) / ZPASS_TX;
                const int w = (nxh + nt - 1) / nt;
                for (int y = 0; y < D.mesh[1]; ++y)
                    for (int x0 = 0; x0 < nxh; x0 += w) zj.push_back(make_int4(r, y, x0, std::min(w, nxh - x0)));
                // + cell counts / ids of the cell layers a plane's stencils reach (<= order + 5 layers)
                const size_t ncell = (size_t)std::min(D.ncell[2], E.order + 5) * D.ncell[0] * D.ncell[1];
                // band spread: the 64-bit charge plane + cell counts; first pass: two complex buffers
                E.band_spread_smem = std::max(E.band_spread_smem, (size_t)D.mesh[0] * D.mesh[1] * sizeof(unsigned long long) +
                                                                      (ncell + 1) * sizeof(int));
                const size_t plane_smem = E.plane_reg ? plane_reg_smem(D.mesh[0]) : (size_t)2 * nxh * D.mesh[1] * sizeof(float2);
                E.rb_fwd_smem = std::max(E.rb_fwd_smem, plane_smem);
                E.rb_inv_smem = std::max(E.rb_inv_smem, plane_smem);
            } else {
                for (int y = 0; y < D.mesh[1]; ++y)
                    for (int x0 = 0; x0 < D.mesh[0]; x0 += ZPASS_TX) zj.push_back(make_int4(r, y, x0, 0));
                E.plane_smem = std::max(E.plane_smem, (size_t)2 * D.mesh[0] * D.mesh[1] * sizeof(float2));
            }
            E.zpass_smem_stk = std::max(E.zpass_smem_stk, (size_t)2 * ZPASS_TX * D.mesh[2] * sizeof(float2));
        }
        zoff.push_back((int)zj.size());
        zoffr.push_back((int)zjr.size());
        E.n_plane_jobs = (int)pj.size(); E.n_band_jobs = (int)pjb.size();
        E.n_zj_stk = (int)zj.size(); E.n_zj_reg = (int)zjr.size();
        DALLOC(E.d_plane_jobs, pj.size()); DALLOC(E.d_zj_stk, zj.size()); DALLOC(E.d_zoff_stk, zoff.size());
        DALLOC(E.d_band_jobs, pjb.size());
        CU(cudaMemcpy(E.d_band_jobs, pjb.data(), sizeof(int2) * pjb.size(), cudaMemcpyHostToDevice));
        DALLOC(E.d_epart, std::max(zj.size(), zjr.size()));
        CU(cudaMemcpy(E.d_plane_jobs, pj.data(), sizeof(int2) * pj.size(), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(E.d_zj_stk, zj.data(), sizeof(int4) * zj.size(), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(E.d_zoff_stk, zoff.data(), sizeof(int) * zoff.size(), cudaMemcpyHostToDevice));
        if (!zjr.empty()) {
            DALLOC(E.d_zj_reg, zjr.size()); DALLOC(E.d_zoff_reg, zoffr.size());
            CU(cudaMemcpy(E.d_zj_reg, zjr.data(), sizeof(int4) * zjr.size(), cudaMemcpyHostToDevice));
            CU(cudaMemcpy(E.d_zoff_reg, zoffr.data(), sizeof(int) * zoffr.size(), cudaMemcpyHostToDevice));
        }
        select_zpass(E, E.zreg_default);
        if (E.use_r2c) CU(rebuild_set_smem_limits(E));
        else CU(mesh_set_smem_limits(E));
    }
    CU(prepare_mc(E));
    return PHMC_OK;
}

static int check_kernel_errors(phmc_engine* h) {
    Engine& E = h->E;
    CU(cudaStreamSynchronize(E.stream));
    CU(cudaGetLastError());
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    for (int r = 0; r < E.R; ++r)
        if (st[r].error) {
            char b[160];
            snprintf(b, sizeof b, "replica %d: device error %d (%s)", r, st[r].error,
                     st[r].error == PHMC_ERR_CAPACITY ? "cell or slot capacity exceeded; raise cell_cap/capacity" : "kernel error");
            return fail(st[r].error, b);
        }
    return PHMC_OK;
}

// Rebuild the potential mesh of all replicas (mode 1) and recompute every energy component.
static int full_recompute(phmc_engine* h) {
    Engine& E = h->E;
    if (E.coulomb == PHMC_COUL_EWALD) {
        // the charge mesh from scratch (the MC kernel keeps the band mesh current between recomputes)
        if (E.use_r2c) launch_band_spread(E, E.stream);
        else launch_spread(E, nullptr, E.stream);
        launch_fft_pipeline(E, nullptr, 1, E.stream);
        CU(cudaGetLastError());
    }
    launch_full_energy(E, E.stream);
    CU(cudaGetLastError());
    return check_kernel_errors(h);
}

// Replicas with the same box, mesh, order and Ewald parameters have bit-identical influence
// kernels G: point every replica at the first copy of its octant, so that the MC kernel's G
// reads of all such replicas share one table in L2 (config 5: 256 replicas, five distinct
// boxes).  Octants are compared byte for byte on the host; the duplicates' storage is left
// allocated and unused.
static int share_octants(phmc_engine* h) {
    Engine& E = h->E;
    if (E.total_oct <= 0) return PHMC_OK;
    std::vector<float> g((size_t)E.total_oct);
    CU(cudaStreamSynchronize(E.stream));
    CU(cudaMemcpy(g.data(), E.d.goct, sizeof(float) * (size_t)E.total_oct, cudaMemcpyDeviceToHost));
    std::map<unsigned long long, std::vector<int>> by_hash;
    bool changed = false;
    for (int r = 0; r < E.R; ++r) {
        RepDesc& D = E.desc[r];
        const size_t n = (size_t)D.oct[0] * D.oct[1] * D.oct[2];
        const float* p = g.data() + D.oct_off;
        unsigned long long hs = 1469598103934665603ull ^ n;  // FNV-1a over the 32-bit words
        for (size_t i = 0; i < n; ++i) {
            uint32_t w;
            std::memcpy(&w, p + i, 4);
            hs = (hs ^ w) * 1099511628211ull;
        }
        std::vector<int>& seen = by_hash[hs];
        int same = -1;
        for (int c : seen) {
            const RepDesc& C = E.desc[c];
            if (C.oct[0] == D.oct[0] && C.oct[1] == D.oct[1] && C.oct[2] == D.oct[2] &&
                std::memcmp(g.data() + C.oct_off, p, n * sizeof(float)) == 0) { same = c; break; }
        }
        if (same >= 0) { D.oct_off = E.desc[same].oct_off; changed = true; }
        else seen.push_back(r);
    }
    if (changed) CU(cudaMemcpy(E.d.desc, E.desc.data(), sizeof(RepDesc) * E.R, cudaMemcpyHostToDevice));
    return PHMC_OK;
}

extern "C" int phmc_create(int n_replicas, const phmc_system* systems, const phmc_params* params, int device,
                           phmc_engine** out) {
    if (!out) return fail(PHMC_ERR_ARG, "out is null");
    *out = nullptr;
    int s = validate(n_replicas, systems, params);
    if (s) return s;
    phmc_engine* h = new (std::nothrow) phmc_engine;
    if (!h) return fail(PHMC_ERR_ARG, "out of host memory");
    s = build(h, n_replicas, systems, params, device);
    if (s) { phmc_destroy(h); return s; }
    Engine& E = h->E;
    launch_cell_build(E, E.stream);
    if (E.coulomb == PHMC_COUL_EWALD) {
        // influence kernel G = potential of a unit charge on mesh point 0
        launch_unit_charge(E, E.stream);
        launch_fft_pipeline(E, nullptr, 1, E.stream);
        for (int r = 0; r < E.R; ++r) launch_extract_octant(E, r, E.stream);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { phmc_destroy(h); return fail(PHMC_ERR_CUDA, std::string("G build: ") + cudaGetErrorString(e)); }
        s = share_octants(h);
        if (s) { std::string m = g_err; phmc_destroy(h); g_err = m; return s; }
    }
    s = full_recompute(h);
    if (s) { std::string m = g_err; phmc_destroy(h); g_err = m; return s; }
    *out = h;
    return PHMC_OK;
}

extern "C" int phmc_destroy(phmc_engine* h) {
    if (!h) return PHMC_OK;
    Engine& E = h->E;
    if (E.stream) cudaStreamSynchronize(E.stream);
    for (void* p : E.allocs) cudaFree(p);
    E.allocs.clear();
    if (E.h_active) cudaFreeHost(E.h_active);
    if (h->l2_scratch) cudaFree(h->l2_scratch);
    for (cudaEvent_t ev : h->ev_pool) cudaEventDestroy(ev);
    drop_graph(h);
    for (cudaEvent_t ev : h->gev) cudaEventDestroy(ev);
    if (h->d_replay) cudaFree(h->d_replay);
    if (h->d_trials) cudaFree(h->d_trials);
    if (h->d_dE) cudaFree(h->d_dE);
    if (E.d.log_move) { cudaFree(E.d.log_move); cudaFree(E.d.log_dE); cudaFree(E.d.log_acc); }
    if (E.d.log_stage) { cudaFree(E.d.log_stage); cudaFree(E.d.log_dEs); }
    if (E.d.zhist) cudaFree(E.d.zhist);
    if (E.d.zh_samples) cudaFree(E.d.zh_samples);
    if (E.d.hv_cap > 0) { cudaFree(E.d.hv_rows); cudaFree(E.d.hv_sign); cudaFree(E.d.hv_target); cudaFree(E.d.hv_count); }
    for (void* p : {(void*)h->st_x, (void*)h->st_y, (void*)h->st_z, (void*)h->st_q, (void*)h->st_t, (void*)h->st_f,
                    (void*)h->st_err, (void*)h->st_cnt, (void*)h->d_charged, (void*)h->d_gc, (void*)h->d_gc_pool,
                    (void*)h->d_gc_ev})
        if (p) cudaFree(p);
    if (E.stream) cudaStreamDestroy(E.stream);
    delete h;
    return PHMC_OK;
}

static void fill_components(const RepState& s, phmc_energy_components* c) {
    c->lj = s.E_pair_lj; c->fene = s.E_fene; c->coul_real = s.E_pair_c; c->coul_recip = s.E_rec;
    c->self = s.E_self; c->qcorr = s.E_qcorr; c->slab = s.E_slab; c->total = s.E;
}

extern "C" int phmc_energy(phmc_engine* h, phmc_energy_components* out) {
    if (!h || !out) return fail(PHMC_ERR_ARG, "null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int s = full_recompute(h);
    if (s) return s;
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    for (int r = 0; r < E.R; ++r) fill_components(st[r], &out[r]);
    return PHMC_OK;
}

static int check_trials(phmc_engine* h, int rep, const phmc_trial* t, int n) {
    if (rep < 0 || rep >= h->E.R) return fail(PHMC_ERR_ARG, "replica index out of range");
    for (int k = 0; k < n; ++k) {
        if (t[k].n_changes < 1 || t[k].n_changes > 2) return fail(PHMC_ERR_ARG, "trial must have 1 or 2 changes");
        for (int c = 0; c < t[k].n_changes; ++c) {
            const phmc_change& ch = t[k].c[c];
            if (ch.index < 0 || ch.index >= h->caps[rep]) return fail(PHMC_ERR_ARG, "change index out of range");
            if (ch.type < 0 || ch.type >= h->E.desc[rep].T) return fail(PHMC_ERR_ARG, "change type out of range");
            const RepDesc& D = h->E.desc[rep];
            if (ch.present && !(ch.x >= 0 && ch.x < D.L[0] && ch.y >= 0 && ch.y < D.L[1] && ch.z >= 0 && ch.z < D.L[2]))
                return fail(PHMC_ERR_ARG, "change position outside [0,L)");
        }
        if (t[k].n_changes == 2 && t[k].c[0].index == t[k].c[1].index) return fail(PHMC_ERR_ARG, "changes must touch distinct slots");
    }
    return PHMC_OK;
}

static int ensure_trial_buffers(phmc_engine* h, int n) {
    if (n <= h->trials_cap) return PHMC_OK;
    if (h->d_trials) { cudaFree(h->d_trials); cudaFree(h->d_dE); h->d_trials = nullptr; h->d_dE = nullptr; }
    CU(cudaMalloc((void**)&h->d_trials, sizeof(phmc_trial) * n));
    CU(cudaMalloc((void**)&h->d_dE, sizeof(double) * n));
    h->trials_cap = n;
    return PHMC_OK;
}

static int flush_dirty(phmc_engine* h) {
    Engine& E = h->E;
    if (E.coulomb != PHMC_COUL_EWALD) return PHMC_OK;
    launch_spread(E, E.d.dirty, E.stream);
    launch_fft_pipeline(E, E.d.dirty, 0, E.stream);
    CU(cudaGetLastError());
    return PHMC_OK;
}

extern "C" int phmc_delta_energy(phmc_engine* h, int rep, const phmc_trial* trials, int n, double* dE) {
    if (!h || (n > 0 && (!trials || !dE))) return fail(PHMC_ERR_ARG, "null argument");
    if (n == 0) return PHMC_OK;
    int s = check_trials(h, rep, trials, n);
    if (s) return s;
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    s = ensure_trial_buffers(h, n);
    if (s) return s;
    CU(cudaMemcpyAsync(h->d_trials, trials, sizeof(phmc_trial) * n, cudaMemcpyHostToDevice, E.stream));
    CU(launch_mc(E, MC_EVAL, rep, h->d_trials, n, h->d_dE, E.stream));
    CU(cudaMemcpyAsync(dE, h->d_dE, sizeof(double) * n, cudaMemcpyDeviceToHost, E.stream));
    return check_kernel_errors(h);
}

extern "C" int phmc_commit(phmc_engine* h, int rep, const phmc_trial* trial) {
    if (!h || !trial) return fail(PHMC_ERR_ARG, "null argument");
    int s = check_trials(h, rep, trial, 1);
    if (s) return s;
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    s = ensure_trial_buffers(h, 1);
    if (s) return s;
    CU(cudaMemcpyAsync(h->d_trials, trial, sizeof(phmc_trial), cudaMemcpyHostToDevice, E.stream));
    CU(launch_mc(E, MC_APPLY, rep, h->d_trials, 1, h->d_dE, E.stream));
    s = flush_dirty(h);
    if (s) return s;
    return check_kernel_errors(h);
}

extern "C" int phmc_set_identity(phmc_engine* h, int rep, int i, int type, float q) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    if (rep < 0 || rep >= h->E.R || i < 0 || i >= h->caps[rep]) return fail(PHMC_ERR_ARG, "index out of range");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    float4 p; int f;
    CU(cudaMemcpy(&p, E.d.posq + E.desc[rep].slot_off + i, sizeof(float4), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&f, E.d.flags + E.desc[rep].slot_off + i, sizeof(int), cudaMemcpyDeviceToHost));
    if (f & PHMC_F_GHOST) return fail(PHMC_ERR_STATE, "set_identity on an empty slot");
    phmc_trial t;
    std::memset(&t, 0, sizeof t);
    t.n_changes = 1;
    t.c[0].index = i; t.c[0].present = 1; t.c[0].x = p.x; t.c[0].y = p.y; t.c[0].z = p.z; t.c[0].q = q; t.c[0].type = type;
    return phmc_commit(h, rep, &t);
}

__global__ void k_set_target(RepState* st, int R, long long n) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    st[r].target = st[r].trial + n;
    st[r].run_start = st[r].trial;
    st[r].att[0] = st[r].att[1] = st[r].att[2] = 0;
    st[r].acc[0] = st[r].acc[1] = st[r].acc[2] = 0;
}

__global__ void k_count_active(const RepState* st, int R, int* active) {
    __shared__ int c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x)
        if (st[r].trial < st[r].target && st[r].error == 0) atomicAdd(&c, 1);
    __syncthreads();
    if (threadIdx.x == 0) *active = c;
}

extern "C" int phmc_set_trial_log(phmc_engine* h, int64_t cap, int* move, double* dE, int* acc) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    Engine& E = h->E;
    drop_graph(h);  // captured launches hold the old log pointers
    if (E.d.log_move) { cudaFree(E.d.log_move); cudaFree(E.d.log_dE); cudaFree(E.d.log_acc); }
    if (E.d.log_stage) { cudaFree(E.d.log_stage); cudaFree(E.d.log_dEs); }
    E.d.log_move = nullptr; E.d.log_dE = nullptr; E.d.log_acc = nullptr; E.d.log_cap = 0;
    E.d.log_stage = nullptr; E.d.log_dEs = nullptr;
    h->h_da_stage = nullptr; h->h_da_dEs = nullptr;
    h->h_log_move = move; h->h_log_dE = dE; h->h_log_acc = acc; h->log_cap = 0;
    if (!move || !dE || !acc || cap <= 0) return PHMC_OK;
    CU(cudaMalloc((void**)&E.d.log_move, sizeof(int) * cap));
    CU(cudaMalloc((void**)&E.d.log_dE, sizeof(double) * cap));
    CU(cudaMalloc((void**)&E.d.log_acc, sizeof(int) * cap));
    E.d.log_cap = cap; h->log_cap = cap;
    return PHMC_OK;
}

extern "C" int phmc_set_replay(phmc_engine* h, int64_t n, const int* decisions) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    Engine& E = h->E;
    drop_graph(h);  // captured launches hold the old replay pointer
    if (h->d_replay) { cudaFree(h->d_replay); h->d_replay = nullptr; }
    E.d.replay = nullptr; E.d.replay_n = 0;
    if (!decisions || n <= 0) return PHMC_OK;
    CU(cudaMalloc((void**)&h->d_replay, sizeof(int) * n));
    CU(cudaMemcpy(h->d_replay, decisions, sizeof(int) * n, cudaMemcpyHostToDevice));
    E.d.replay = h->d_replay; E.d.replay_n = n;
    return PHMC_OK;
}

// protonated (charged) titratable sites of every replica, one block per replica
__global__ void k_count_charged(DevPtrs d, int* __restrict__ out) {
    const int r = blockIdx.x;
    const RepDesc& D = d.desc[r];
    int c = 0;
    for (int k = threadIdx.x; k < D.n_titr; k += blockDim.x) c += d.posq[D.slot_off + d.titr[D.slot_off + k]].w != 0.0f;
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ int s[8];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) t += s[w];
        out[r] = t;
    }
}

static int collect_stats(phmc_engine* h, phmc_run_stats* stats) {
    Engine& E = h->E;
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    for (int r = 0; r < E.R; ++r) {
        phmc_run_stats& o = stats[r];
        std::memset(&o, 0, sizeof o);
        for (int k = 0; k < 3; ++k) { o.attempted[k] = st[r].att[k]; o.accepted[k] = st[r].acc[k]; }
        o.flushes = st[r].flushes;
        o.n_titratable = E.desc[r].n_titr;
        o.n_cations = st[r].n_cation; o.n_anions = st[r].n_anion;
        o.energy = st[r].E; o.energy_drift = st[r].drift;
    }
    // protonated sites: titratable sites with q != 0, counted on the device
    if (!h->d_charged) CU(cudaMalloc((void**)&h->d_charged, sizeof(int) * E.R));
    k_count_charged<<<E.R, 256, 0, E.stream>>>(E.d, h->d_charged);
    std::vector<int> cnt((size_t)E.R);
    CU(cudaMemcpyAsync(cnt.data(), h->d_charged, sizeof(int) * E.R, cudaMemcpyDeviceToHost, E.stream));
    CU(cudaStreamSynchronize(E.stream));
    for (int r = 0; r < E.R; ++r) stats[r].n_charged_sites = cnt[(size_t)r];
    return PHMC_OK;
}

// Run the trial/rebuild loop (internal; also used by the timed entry points).
int phmc_run_loop(phmc_engine* h, int64_t n_trials, int check_every) {
    Engine& E = h->E;
    k_set_target<<<(E.R + 127) / 128, 128, 0, E.stream>>>(E.d.state, E.R, n_trials);
    if (E.d.log_move) {
        CU(cudaMemsetAsync(E.d.log_move, 0xff, sizeof(int) * E.d.log_cap, E.stream));
    }
    h->prof.kernel_launches += 1;
    std::vector<RepState> st0;
    if (h->profiling) {
        st0.resize((size_t)E.R);
        CU(cudaMemcpyAsync(st0.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost, E.stream));
        CU(cudaStreamSynchronize(E.stream));
        h->ev_used = 0;
        h->ev_mc.clear();
        h->ev_flush.clear();
    }
    const int flush_kernels = E.flush_kernels;
    long long iter = 0;
    const long long max_iter = n_trials + 8;
    int s = build_chunk_graph(h, check_every);
    if (s) return s;
    for (;;) {
        // one graph = check_every x (MC launch + potential-mesh rebuild); chunks after
        // every replica reached its target are no-ops
        CU(cudaGraphLaunch(h->graph_exec, E.stream));
        h->prof.kernel_launches += (int64_t)check_every * (1 + flush_kernels);
        iter += check_every;
        k_count_active<<<1, 256, 0, E.stream>>>(E.d.state, E.R, E.d_active);
        h->prof.kernel_launches += 1;
        CU(cudaMemcpyAsync(E.h_active, E.d_active, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
        CU(cudaStreamSynchronize(E.stream));
        if (h->profiling) {
            for (int k = 0; k < check_every; ++k) {
                float ms = 0.f;
                CU(cudaEventElapsedTime(&ms, h->gev[4 * k], h->gev[4 * k + 1]));
                h->prof.mc_ms += ms;
                if (flush_kernels) {
                    CU(cudaEventElapsedTime(&ms, h->gev[4 * k + 2], h->gev[4 * k + 3]));
                    h->prof.flush_ms += ms;
                }
            }
            h->prof.mc_launches += check_every;
            if (flush_kernels) h->prof.flush_launches += check_every;
        }
        if (*E.h_active == 0) break;
        if (iter > max_iter) return fail(PHMC_ERR_BUDGET, "trial loop made no progress");
        if (h->launch_budget > 0 && iter >= h->launch_budget)
            return fail(PHMC_ERR_BUDGET, "launch budget reached before every replica reached its target");
    }
    if (h->profiling) {
        std::vector<RepState> st1((size_t)E.R);
        CU(cudaMemcpy(st1.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
        for (int r = 0; r < E.R; ++r) {
            const RepDesc& D = E.desc[r];
            h->prof.mc_alg_bytes += st1[r].alg_bytes - st0[r].alg_bytes;
            h->prof.trials += st1[r].trials_run - st0[r].trials_run;
            h->prof.mc_busy_ms += 1e-6 * (double)(st1[r].busy_ns - st0[r].busy_ns);
            // planes of the wall band: the first pass reads the fixed-point charge plane (8 B per
            // point) and writes the half spectrum (8 B per complex value), the z pass reads and
            // writes it, the last pass reads it and writes phi (4 B per point)
            const double Mb = (double)D.mesh[0] * D.mesh[1] * D.zb_n;
            const double Mcb = (double)(D.mesh[0] / 2 + 1) * D.mesh[1] * D.zb_n;
            h->prof.flush_alg_bytes += (double)(st1[r].flushes - st0[r].flushes) * (16.0 * h->n_present[r] + 32.0 * Mcb + 12.0 * Mb);
        }
    }
    return PHMC_OK;
}

extern "C" int phmc_set_profiling(phmc_engine* h, int on) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    h->profiling = on != 0;
    return PHMC_OK;
}

extern "C" int phmc_get_profile(phmc_engine* h, phmc_profile* out, int reset) {
    if (!h || !out) return fail(PHMC_ERR_ARG, "null argument");
    *out = h->prof;
    if (reset) std::memset(&h->prof, 0, sizeof(h->prof));
    return PHMC_OK;
}

// trials run by all replicas so far (the phase clocks' trial count is taken against it)
static int trials_run_total(Engine& E, int64_t* out) {
    std::vector<RepState> st((size_t)E.R);
    CU(cudaStreamSynchronize(E.stream));
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    int64_t t = 0;
    for (const RepState& r : st) t += r.trials_run;
    *out = t;
    return PHMC_OK;
}

extern "C" int phmc_set_phase_clock(phmc_engine* h, int on) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    CU(cudaSetDevice(h->E.device));
    const int s = trials_run_total(h->E, &h->clk_trials0);
    if (s) return s;
    h->E.d.phase_clk = on != 0;
    drop_graph(h);  // captured launches hold the old flag
    return PHMC_OK;
}

extern "C" int phmc_get_phase_cycles(phmc_engine* h, int64_t cycles[PHMC_PHASES], int64_t* trials, int reset) {
    if (!h || !cycles) return fail(PHMC_ERR_ARG, "null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    int64_t t = 0;
    for (int k = 0; k < PHMC_PHASES; ++k) cycles[k] = 0;
    for (const RepState& r : st) {
        for (int k = 0; k < PHMC_PHASES; ++k) cycles[k] += r.clk[k];
        t += r.trials_run;
    }
    if (trials) *trials = t - h->clk_trials0;  // since the clocks were last switched or reset
    if (reset) {
        for (RepState& r : st) std::memset(r.clk, 0, sizeof(r.clk));
        CU(cudaMemcpy(E.d.state, st.data(), sizeof(RepState) * E.R, cudaMemcpyHostToDevice));
        h->clk_trials0 = t;
    }
    return PHMC_OK;
}

extern "C" int phmc_run_timed(phmc_engine* h, int64_t n_trials, double* device_ms) {
    if (!h || n_trials < 0 || !device_ms) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    CU(cudaEventRecord(a, E.stream));
    int s = phmc_run_loop(h, n_trials, 4);
    if (s) { cudaEventDestroy(a); cudaEventDestroy(b); return s; }
    CU(cudaEventRecord(b, E.stream));
    CU(cudaEventSynchronize(b));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *device_ms = ms;
    return check_kernel_errors(h);
}

extern "C" int phmc_flush_l2(phmc_engine* h, int64_t bytes) {
    if (!h || bytes <= 0) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    if (bytes > h->l2_bytes) {
        if (h->l2_scratch) cudaFree(h->l2_scratch);
        h->l2_scratch = nullptr;
        CU(cudaMalloc(&h->l2_scratch, (size_t)bytes));
        h->l2_bytes = bytes;
    }
    CU(cudaMemsetAsync(h->l2_scratch, 0x5a, (size_t)bytes, E.stream));
    return PHMC_OK;
}

extern "C" int phmc_run(phmc_engine* h, int64_t n_trials, phmc_run_stats* stats) {
    if (!h || n_trials < 0) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int s = phmc_run_loop(h, n_trials, 4);
    if (s) return s;
    s = check_kernel_errors(h);
    if (s) return s;
    if (h->h_log_move && E.d.log_move) {
        const long long n = std::min<long long>(n_trials, E.d.log_cap);
        CU(cudaMemcpy(h->h_log_move, E.d.log_move, sizeof(int) * n, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(h->h_log_dE, E.d.log_dE, sizeof(double) * n, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(h->h_log_acc, E.d.log_acc, sizeof(int) * n, cudaMemcpyDeviceToHost));
        if (h->h_da_stage && E.d.log_stage) {
            CU(cudaMemcpy(h->h_da_stage, E.d.log_stage, sizeof(int) * n, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(h->h_da_dEs, E.d.log_dEs, sizeof(double) * n, cudaMemcpyDeviceToHost));
        }
    }
    if (stats) return collect_stats(h, stats);
    return PHMC_OK;
}

// ---------------------------------------------------------------------------
// state upload / readback: caller arrays <-> device staging (direct copies, DMA
// from pinned memory), interleaving, validation and list building on the device
// ---------------------------------------------------------------------------
static int ensure_state_staging(phmc_engine* h) {
    if (h->st_x) return PHMC_OK;
    const size_t n = (size_t)h->E.total_slots;
    CU(cudaMalloc((void**)&h->st_x, sizeof(float) * n));
    CU(cudaMalloc((void**)&h->st_y, sizeof(float) * n));
    CU(cudaMalloc((void**)&h->st_z, sizeof(float) * n));
    CU(cudaMalloc((void**)&h->st_q, sizeof(float) * n));
    CU(cudaMalloc((void**)&h->st_t, sizeof(int) * n));
    CU(cudaMalloc((void**)&h->st_f, sizeof(int) * n));
    CU(cudaMalloc((void**)&h->st_err, sizeof(int)));
    CU(cudaMalloc((void**)&h->st_cnt, sizeof(int) * 2 * h->E.R));
    return PHMC_OK;
}

__global__ void k_state_egress(DevPtrs d, int off, int n, float* x, float* y, float* z, float* q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = d.posq[off + i];
    x[i] = p.x; y[i] = p.y; z[i] = p.z; q[i] = p.w;
}

// staged slot arrays (index s - off) of replicas [r0, r0 + gridDim.x): 1 = type out of range,
// 2 = a present particle outside [0, L)
__global__ void k_state_check(DevPtrs d, int r0, int off, const float* __restrict__ x, const float* __restrict__ y,
                              const float* __restrict__ z, const int* __restrict__ t, const int* __restrict__ f, int* err) {
    const RepDesc& D = d.desc[r0 + blockIdx.x];
    for (int i = threadIdx.x; i < D.cap; i += blockDim.x) {
        const int s = D.slot_off + i - off;
        if (t[s] < 0 || t[s] >= D.T) atomicMax(err, 1);
        if (!(f[s] & PHMC_F_GHOST) && !(x[s] >= 0.0f && x[s] < D.L[0] && y[s] >= 0.0f && y[s] < D.L[1] && z[s] >= 0.0f && z[s] < D.L[2]))
            atomicMax(err, 2);
    }
}

// One block per replica: particle arrays, membership lists with position maps, the
// free stack (top = lowest empty slot) and the counts, in slot order as on the host.
template <int NT>
__global__ void __launch_bounds__(NT) k_state_ingest(DevPtrs d, int r0, int off, const float* __restrict__ x,
                                                     const float* __restrict__ y, const float* __restrict__ z,
                                                     const float* __restrict__ q, const int* __restrict__ t,
                                                     const int* __restrict__ f, int* __restrict__ counts) {
    const int r = r0 + blockIdx.x;
    RepDesc& D = d.desc[r];
    const int cap = D.cap, so = D.slot_off;
    __shared__ int s_ghost;
    __shared__ int s_warp[5][NT / 32];
    __shared__ int s_base[5];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // pass 1: number of empty slots (the free stack is filled from the top of the slot range)
    if (threadIdx.x == 0) s_ghost = 0;
    __syncthreads();
    int g = 0;
    for (int i = threadIdx.x; i < cap; i += NT) g += (f[so + i - off] & PHMC_F_GHOST) != 0;
    g = __reduce_add_sync(0xffffffffu, g);
    if (lane == 0) atomicAdd(&s_ghost, g);
    if (threadIdx.x < 5) s_base[threadIdx.x] = 0;
    __syncthreads();
    const int n_ghost = s_ghost;
    // pass 2: chunks of NT slots, block-wide exclusive scans of the five memberships
    for (int c0 = 0; c0 < cap; c0 += NT) {
        const int i = c0 + threadIdx.x;
        int fl = PHMC_F_GHOST;
        if (i < cap) {
            const int s = so + i - off;
            fl = f[s];
            d.posq[so + i] = make_float4(x[s], y[s], z[s], q[s]);
            d.type[so + i] = t[s];
            d.flags[so + i] = fl;
        }
        const bool pres = i < cap && !(fl & PHMC_F_GHOST);
        const int m[5] = {pres && (fl & PHMC_F_MOBILE), pres && (fl & PHMC_F_ANION), pres && (fl & PHMC_F_CATION),
                          pres && (fl & PHMC_F_TITRATABLE), i < cap && (fl & PHMC_F_GHOST)};
        int ex[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const unsigned bal = __ballot_sync(0xffffffffu, m[k]);
            ex[k] = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0) s_warp[k][warp] = __popc(bal);
        }
        __syncthreads();
        if (threadIdx.x < 5) {  // warp totals -> exclusive warp offsets, chunk total -> base
            const int k = threadIdx.x;
            int acc = s_base[k];
            for (int w = 0; w < NT / 32; ++w) { const int v = s_warp[k][w]; s_warp[k][w] = acc; acc += v; }
            s_base[k] = acc;
        }
        __syncthreads();
        if (i < cap) {
            int pos[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) pos[k] = s_warp[k][warp] + ex[k];
            d.mobile_pos[so + i] = m[0] ? pos[0] : -1;
            if (m[0]) d.mobile[so + pos[0]] = i;
            d.anion_pos[so + i] = m[1] ? pos[1] : -1;
            if (m[1]) d.anions[so + pos[1]] = i;
            d.cation_pos[so + i] = m[2] ? pos[2] : -1;
            if (m[2]) d.cations[so + pos[2]] = i;
            if (m[3]) d.titr[so + pos[3]] = i;
            if (m[4]) d.freel[so + n_ghost - 1 - pos[4]] = i;  // the highest empty slot at the bottom
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        RepState& S = d.state[r];
        S.n_mobile = s_base[0]; S.n_anion = s_base[1]; S.n_cation = s_base[2]; S.n_free = s_base[4];
        D.n_titr = s_base[3];
        counts[2 * r] = s_base[3];
        counts[2 * r + 1] = cap - s_base[4];
    }
}

extern "C" int phmc_get_state(phmc_engine* h, int rep, float* x, float* y, float* z, float* q, int* type, int* flags) {
    if (!h || rep < -1 || rep >= h->E.R) return fail(PHMC_ERR_ARG, "invalid replica");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int s = ensure_state_staging(h);
    if (s) return s;
    // one replica, or (rep == -1) all replicas concatenated in replica order, capacity slots each
    const int off = rep < 0 ? 0 : E.desc[rep].slot_off;
    const int cap = rep < 0 ? E.total_slots : E.desc[rep].cap;
    const cudaStream_t st = E.stream;
    k_state_egress<<<(cap + 255) / 256, 256, 0, st>>>(E.d, off, cap, h->st_x, h->st_y, h->st_z, h->st_q);
    CU(cudaGetLastError());
    if (x) CU(cudaMemcpyAsync(x, h->st_x, sizeof(float) * cap, cudaMemcpyDeviceToHost, st));
    if (y) CU(cudaMemcpyAsync(y, h->st_y, sizeof(float) * cap, cudaMemcpyDeviceToHost, st));
    if (z) CU(cudaMemcpyAsync(z, h->st_z, sizeof(float) * cap, cudaMemcpyDeviceToHost, st));
    if (q) CU(cudaMemcpyAsync(q, h->st_q, sizeof(float) * cap, cudaMemcpyDeviceToHost, st));
    if (type) CU(cudaMemcpyAsync(type, E.d.type + off, sizeof(int) * cap, cudaMemcpyDeviceToHost, st));
    if (flags) CU(cudaMemcpyAsync(flags, E.d.flags + off, sizeof(int) * cap, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return PHMC_OK;
}

extern "C" int phmc_set_state(phmc_engine* h, int rep, const float* x, const float* y, const float* z, const float* q,
                              const int* type, const int* flags) {
    if (!h || rep < -1 || rep >= h->E.R || !x || !y || !z || !q || !type || !flags) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int s = ensure_state_staging(h);
    if (s) return s;
    // one replica, or (rep == -1) all replicas from arrays concatenated in replica order
    const int r0 = rep < 0 ? 0 : rep, nr = rep < 0 ? E.R : 1;
    const int off = E.desc[r0].slot_off;
    const int n = E.desc[r0 + nr - 1].slot_off + E.desc[r0 + nr - 1].cap - off;
    const cudaStream_t st = E.stream;
    CU(cudaMemcpyAsync(h->st_x, x, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->st_y, y, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->st_z, z, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->st_q, q, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->st_t, type, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->st_f, flags, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(h->st_err, 0, sizeof(int), st));
    k_state_check<<<nr, 256, 0, st>>>(E.d, r0, off, h->st_x, h->st_y, h->st_z, h->st_t, h->st_f, h->st_err);
    int err = 0;
    CU(cudaMemcpyAsync(&err, h->st_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (err == 1) return fail(PHMC_ERR_ARG, "type out of range");
    if (err == 2) return fail(PHMC_ERR_ARG, "particle outside [0,L)");
    k_state_ingest<256><<<nr, 256, 0, st>>>(E.d, r0, off, h->st_x, h->st_y, h->st_z, h->st_q, h->st_t, h->st_f, h->st_cnt);
    CU(cudaGetLastError());
    std::vector<int> cnt((size_t)2 * E.R);
    CU(cudaMemcpyAsync(cnt.data() + 2 * r0, h->st_cnt + 2 * r0, sizeof(int) * 2 * nr, cudaMemcpyDeviceToHost, st));
    launch_cell_build(E, st);
    h->prof.kernel_launches += 4;
    int rc = full_recompute(h);  // synchronises the stream
    h->prof.kernel_launches += E.flush_kernels + 2;
    for (int r = r0; r < r0 + nr; ++r) {
        E.desc[(size_t)r].n_titr = cnt[(size_t)2 * r];
        h->n_present[(size_t)r] = cnt[(size_t)2 * r + 1];
    }
    return rc;
}

// ---- the reference's phases on the device: grand-canonical mu control (MC/src/mc.cu:320-548)
// and swaps with patience (MC/src/mc.cu:159-318) ----

#define GC_LAUNCH_TRIALS 2048                      // two-atom evaluations per MC launch at most
#define GC_EV_CAP (2 * GC_LAUNCH_TRIALS + 4)       // events one launch can record (two per evaluation)
static_assert(sizeof(phmc_gc_event) <= GC_EV_BYTES && sizeof(phmc_phase2_event) <= GC_EV_BYTES, "event record size");

static float gc_clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// The phase's energy as the reference tracks it: the LJ part and the Coulomb part of the
// energy components each rounded to its real, then added (MC/src/mc.cu:43-60).
static float gc_energy_real(const RepState& s, int coulomb) {
    const double ec = coulomb == PHMC_COUL_EWALD ? s.E_pair_c + s.E_rec + s.E_self + s.E_qcorr + s.E_slab : s.E_pair_c;
    return (float)s.E_pair_lj + (float)ec;
}

// Checks shared by both phases' jobs; fills the common part of the device state.
static int gc_job_common(phmc_engine* h, int replica, std::vector<int>& seen, const int types[4], const uint32_t* mt,
                         double beta, const int* const pools[4], const int npool[4], GcDev& g) {
    Engine& E = h->E;
    if (replica < 0 || replica >= E.R || seen[replica]++) return fail(PHMC_ERR_ARG, "job replicas must be distinct and in range");
    const RepDesc& D = E.desc[replica];
    for (int k = 0; k < 4; ++k)
        if (types[k] < 0 || types[k] >= D.T) return fail(PHMC_ERR_ARG, "job type out of range");
    if (!mt || mt[MT_N] > MT_N) return fail(PHMC_ERR_ARG, "job needs a generator state (624 words, position <= 624)");
    if (!(beta > 0.0)) return fail(PHMC_ERR_ARG, "beta must be positive");
    std::vector<int> flags((size_t)D.cap);
    CU(cudaMemcpy(flags.data(), E.d.flags + D.slot_off, sizeof(int) * D.cap, cudaMemcpyDeviceToHost));
    std::vector<char> used((size_t)D.cap, 0);
    for (int p = 0; p < 4; ++p) {
        if (npool[p] < 0 || (npool[p] > 0 && !pools[p])) return fail(PHMC_ERR_ARG, "job pool pointer / size invalid");
        for (int i = 0; i < npool[p]; ++i) {
            const int v = pools[p][i];
            if (v < 0 || v >= D.cap || used[(size_t)v]++) return fail(PHMC_ERR_ARG, "pool slots must be distinct and in range");
            if (flags[(size_t)v] & PHMC_F_GHOST) return fail(PHMC_ERR_ARG, "pool slot is empty");
        }
    }
    std::memset(&g, 0, sizeof g);
    for (int i = 0; i < MT_N; ++i) g.mt.x[i] = mt[i];
    g.mt.p = (int)mt[MT_N];
    g.replica = replica;
    for (int k = 0; k < 4; ++k) { g.type[k] = types[k]; g.n[k] = npool[k]; }
    g.beta = (float)beta;
    g.launch_cap = GC_LAUNCH_TRIALS;
    g.ev_cap = GC_EV_CAP;
    return PHMC_OK;
}

// Upload pools and job states, run MC launches (each followed by the potential-mesh
// rebuild of its replicas) until every job has stopped, collect the event records
// (ev_size bytes each) and return the final job states in G.
static int gc_run(phmc_engine* h, std::vector<GcDev>& G, const std::vector<const int* const*>& pools,
                  const std::vector<const int*>& npools, size_t ev_size, std::vector<std::vector<unsigned char>>& evs,
                  int phase) {
    Engine& E = h->E;
    const int n_jobs = (int)G.size();
    // records not yet handed to the caller's stream callback
    std::vector<size_t> streamed((size_t)n_jobs, 0);
    auto stream_new = [&]() {
        if (!h->ev_fn) return;
        for (int k = 0; k < n_jobs; ++k)
            for (; streamed[k] + ev_size <= evs[k].size(); streamed[k] += ev_size)
                h->ev_fn(h->ev_user, k, phase, evs[k].data() + streamed[k]);
    };
    stream_new();  // records made before the first launch
    if (!h->d_gc) {
        CU(cudaMalloc((void**)&h->d_gc, sizeof(GcDev) * E.R));
        CU(cudaMalloc((void**)&h->d_gc_pool, sizeof(int) * 4 * (size_t)E.total_slots));
        CU(cudaMalloc((void**)&h->d_gc_ev, (size_t)GC_EV_BYTES * GC_EV_CAP * E.R));
    }
    E.d.gc = h->d_gc; E.d.gc_pool = h->d_gc_pool; E.d.gc_pool_stride = E.total_slots; E.d.gc_ev = h->d_gc_ev;
    for (int k = 0; k < n_jobs; ++k)
        for (int p = 0; p < 4; ++p)
            if (npools[k][p] > 0)
                CU(cudaMemcpyAsync(h->d_gc_pool + (size_t)p * E.total_slots + E.desc[G[k].replica].slot_off, pools[k][p],
                                   sizeof(int) * npools[k][p], cudaMemcpyHostToDevice, E.stream));
    CU(cudaMemcpyAsync(h->d_gc, G.data(), sizeof(GcDev) * n_jobs, cudaMemcpyHostToDevice, E.stream));
    std::vector<unsigned char> buf;
    // every launch makes progress on each unfinished job (pending room for an attempt is
    // always there at a launch's start), so the loop ends; the bound is a guard
    const long long max_launches = 4LL * 1000000000LL + 8;
    for (long long it = 0;; ++it) {
        CU(launch_mc_gc(E, n_jobs, E.stream));
        int s = flush_dirty(h);
        if (s) return s;
        CU(cudaMemcpyAsync(G.data(), h->d_gc, sizeof(GcDev) * n_jobs, cudaMemcpyDeviceToHost, E.stream));
        s = check_kernel_errors(h);  // synchronises the stream
        if (s) return s;
        bool all = true;
        for (int k = 0; k < n_jobs; ++k) {
            if (G[k].n_ev > GC_EV_CAP) return fail(PHMC_ERR_CAPACITY, "device phase: event buffer overflow");
            if (G[k].n_ev > 0) {
                buf.resize((size_t)G[k].n_ev * ev_size);
                CU(cudaMemcpy(buf.data(), h->d_gc_ev + (size_t)k * GC_EV_CAP * GC_EV_BYTES, buf.size(), cudaMemcpyDeviceToHost));
                evs[k].insert(evs[k].end(), buf.begin(), buf.end());
            }
            all = all && G[k].stop != 0;
        }
        stream_new();
        if (all) break;
        if (it > max_launches) return fail(PHMC_ERR_BUDGET, "device phase made no progress");
        if (h->launch_budget > 0 && it + 1 >= h->launch_budget)
            return fail(PHMC_ERR_BUDGET, "launch budget reached before every job stopped");
    }
    return PHMC_OK;
}

template <class Ev>
static void gc_host_event(std::vector<unsigned char>& out, const Ev& ev) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&ev);
    out.insert(out.end(), p, p + sizeof ev);
}

// Copy a job's collected events to the caller's records; returns (kept, dropped).
template <class Ev>
static std::pair<int, int> gc_events_out(const std::vector<unsigned char>& evs, Ev* out, int cap) {
    const int n = (int)(evs.size() / sizeof(Ev));
    const int kept = out ? std::min(n, cap) : 0;
    if (kept > 0) std::memcpy(out, evs.data(), sizeof(Ev) * kept);
    return {kept, n - kept};
}

extern "C" int phmc_gc_phase(phmc_engine* h, int n_jobs, const phmc_gc_job* jobs, phmc_gc_result* results,
                             phmc_gc_event* events, int event_cap) {
    if (!h || n_jobs < 1 || !jobs || !results || event_cap < 0) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    if (n_jobs > E.R) return fail(PHMC_ERR_ARG, "more jobs than replicas");
    CU(cudaSetDevice(E.device));
    std::vector<int> seen((size_t)E.R, 0);
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    std::vector<GcDev> G((size_t)n_jobs);
    std::vector<const int* const*> pools((size_t)n_jobs);
    std::vector<const int*> npools((size_t)n_jobs);
    std::vector<std::array<const int*, 4>> pool_arr((size_t)n_jobs);
    std::vector<std::array<int, 4>> npool_arr((size_t)n_jobs);
    std::vector<std::vector<unsigned char>> evs((size_t)n_jobs);
    for (int k = 0; k < n_jobs; ++k) {
        const phmc_gc_job& J = jobs[k];
        pool_arr[k] = {J.nh_n, J.nh_p, J.w, J.cl};
        npool_arr[k] = {J.n_nh_n, J.n_nh_p, J.n_w, J.n_cl};
        pools[k] = pool_arr[k].data();
        npools[k] = npool_arr[k].data();
        const int types[4] = {J.nh_n_type, J.nh_p_type, J.w_type, J.cl_type};
        GcDev& g = G[k];
        int s = gc_job_common(h, J.replica, seen, types, J.mt_state, J.beta, pools[k], npools[k], g);
        if (s) return s;
        // settings derived as the reference derives them, in its real (MC/src/mc.cu:339-357)
        g.phase = 1;
        g.q_nhp = J.q_nh_p; g.q_cl = J.q_cl;
        g.Nh = J.n_nh_n + J.n_nh_p;
        g.Nprot = J.n_nh_p;
        const float pct = (float)J.target_pct;
        g.target = (int)std::floor(pct / 100.0 * g.Nh);
        const float lo = (float)1e-6, hi = (float)(1.0 - 1e-6);
        const float fstar = gc_clampf((float)(pct / 100.0), lo, hi);
        g.f0 = fstar;
        const float bound = 10.0f / g.beta;
        g.mu = gc_clampf((1.0f / g.beta) * std::log(fstar / (1.0f - fstar)), -bound, bound);
        g.gc_block = J.gc_block > 0 ? J.gc_block : 2000;
        g.amax = J.epoch_attempt_max > 0 ? J.epoch_attempt_max : 100000;
        const int R0 = std::max(0, g.target - g.Nprot);
        const float frac = J.nacc_frac > 0.0 ? (float)J.nacc_frac : 0.10f;
        g.nacc_target = std::max(1, (int)std::ceil((double)frac * (double)R0));
        g.eta = J.mu_eta > 0.0 ? (float)J.mu_eta : 0.3f;
        g.E = gc_energy_real(st[(size_t)J.replica], E.desc[J.replica].coulomb);
        g.max_trials = (int)std::min<int64_t>(J.max_trials > 0 ? J.max_trials : 1000000000, 1000000000);
        g.fixed = J.fixed_mu ? 1 : 0;
        if (g.fixed) g.mu = (float)(J.mu_kT / J.beta);
        if (!g.fixed && g.Nprot == g.target) {
            g.stop = PHMC_GC_STOP_ALREADY;
            phmc_gc_event ev;
            std::memset(&ev, 0, sizeof ev);
            ev.kind = PHMC_GC_EV_ALREADY; ev.nprot = g.Nprot; ev.mu_kT = g.beta * g.mu; ev.E = g.E;
            gc_host_event(evs[k], ev);
        }
        phmc_gc_result& R = results[k];
        std::memset(&R, 0, sizeof R);
        R.R0 = R0; R.Nacc_target = g.nacc_target; R.epoch_attempt_max = g.amax; R.gc_block = g.gc_block;
    }
    for (int k = 0; k < n_jobs; ++k) { results[k].Nh = G[k].Nh; results[k].target_count = G[k].target; }
    int s = gc_run(h, G, pools, npools, sizeof(phmc_gc_event), evs, 1);
    if (s) return s;
    for (int k = 0; k < n_jobs; ++k) {
        const GcDev& g = G[k];
        const phmc_gc_job& J = jobs[k];
        for (int i = 0; i < MT_N; ++i) J.mt_state[i] = g.mt.x[i];
        J.mt_state[MT_N] = (uint32_t)g.mt.p;
        phmc_gc_result& R = results[k];
        R.attempted = g.attempted; R.accepted = g.accepted;
        R.accepted_forward = g.fwd; R.accepted_backward = g.bwd; R.blocks_done = g.blocks_done;
        R.Nh = g.Nh; R.Nprot = g.Nprot; R.target_count = g.target;
        R.reached_target = (g.stop == PHMC_GC_STOP_REACHED || g.stop == PHMC_GC_STOP_ALREADY) ? 1 : 0;  // never when fixed
        R.stop = g.stop;
        R.E = g.E; R.mu_eff = g.mu;
        const auto ke = gc_events_out(evs[k], events ? events + (size_t)k * event_cap : nullptr, event_cap);
        R.n_events = ke.first; R.events_dropped = ke.second;
    }
    return PHMC_OK;
}

extern "C" int phmc_phase2(phmc_engine* h, int n_jobs, const phmc_phase2_job* jobs, phmc_phase2_result* results,
                           phmc_phase2_event* events, int event_cap) {
    if (!h || n_jobs < 1 || !jobs || !results || event_cap < 0) return fail(PHMC_ERR_ARG, "invalid argument");
    Engine& E = h->E;
    if (n_jobs > E.R) return fail(PHMC_ERR_ARG, "more jobs than replicas");
    // a four-point attempt starts only with room for six pending stencils
    if (E.pend_max < 6) return fail(PHMC_ERR_UNSUPPORTED, "phase 2 needs pending_max >= 6 (phmc_set_tuning)");
    CU(cudaSetDevice(E.device));
    std::vector<int> seen((size_t)E.R, 0);
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    std::vector<GcDev> G((size_t)n_jobs);
    std::vector<const int* const*> pools((size_t)n_jobs);
    std::vector<const int*> npools((size_t)n_jobs);
    std::vector<std::array<const int*, 4>> pool_arr((size_t)n_jobs);
    std::vector<std::array<int, 4>> npool_arr((size_t)n_jobs);
    std::vector<std::vector<unsigned char>> evs((size_t)n_jobs);
    for (int k = 0; k < n_jobs; ++k) {
        const phmc_phase2_job& J = jobs[k];
        pool_arr[k] = {J.nh_n, J.nh_p, J.w, J.cl};
        npool_arr[k] = {J.n_nh_n, J.n_nh_p, J.n_w, J.n_cl};
        pools[k] = pool_arr[k].data();
        npools[k] = npool_arr[k].data();
        const int types[4] = {J.nh_n_type, J.nh_p_type, J.w_type, J.cl_type};
        GcDev& g = G[k];
        int s = gc_job_common(h, J.replica, seen, types, J.mt_state, J.beta, pools[k], npools[k], g);
        if (s) return s;
        g.phase = 2;
        g.q_nhp = J.q_nh_p; g.q_cl = J.q_cl;
        g.max_attempts = std::max(0, J.max_attempts);
        g.patience = J.patience;
        g.energy_interval = J.energy_interval;
        g.E = gc_energy_real(st[(size_t)J.replica], E.desc[J.replica].coulomb);
        g.best_E = g.E;
        // the pools line and the checks before the first attempt (MC/src/mc.cu:185-208)
        phmc_phase2_event ev;
        std::memset(&ev, 0, sizeof ev);
        ev.kind = PHMC_P2_EV_POOLS;
        ev.n_nh_p = J.n_nh_p; ev.n_nh_n = J.n_nh_n; ev.n_cl = J.n_cl; ev.n_w = J.n_w; ev.z_cut = J.z_cut;
        gc_host_event(evs[k], ev);
        const bool can_wc = J.n_w > 0 && J.n_cl > 0;
        const bool can_four = can_wc && J.n_nh_p > 0 && J.n_nh_n > 0;
        g.prefer_wc = J.n_nh_n == 0;
        if (!g.prefer_wc && !can_four && can_wc) g.prefer_wc = 1;
        int pre = 0;
        if (!g.prefer_wc && !can_four && !can_wc) pre = PHMC_P2_EV_NONE_AT_START;
        else if (g.prefer_wc && !can_wc) pre = PHMC_P2_EV_WC_EMPTY;
        if (pre) {
            std::memset(&ev, 0, sizeof ev);
            ev.kind = pre;
            gc_host_event(evs[k], ev);
            g.stop = PHMC_P2_STOP_NO_PROPOSALS;
        }
    }
    int s = gc_run(h, G, pools, npools, sizeof(phmc_phase2_event), evs, 2);
    if (s) return s;
    for (int k = 0; k < n_jobs; ++k) {
        const GcDev& g = G[k];
        const phmc_phase2_job& J = jobs[k];
        for (int i = 0; i < MT_N; ++i) J.mt_state[i] = g.mt.x[i];
        J.mt_state[MT_N] = (uint32_t)g.mt.p;
        phmc_phase2_result& R = results[k];
        std::memset(&R, 0, sizeof R);
        R.attempted = g.attempted; R.accepted = g.accepted;
        R.E = g.E; R.best_E = g.best_E;
        R.stop = g.attempted > 0 || g.stop != PHMC_P2_STOP_NO_PROPOSALS ? g.stop : 0;
        R.since_best = g.since_best;
        const auto ke = gc_events_out(evs[k], events ? events + (size_t)k * event_cap : nullptr, event_cap);
        R.n_events = ke.first; R.events_dropped = ke.second;
    }
    return PHMC_OK;
}

extern "C" int phmc_get_cells(phmc_engine* h, int rep, int* cell_of, int dims[3]) {
    if (!h || rep < 0 || rep >= h->E.R) return fail(PHMC_ERR_ARG, "invalid replica");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    const RepDesc& D = E.desc[rep];
    if (dims) for (int k = 0; k < 3; ++k) dims[k] = D.ncell[k];
    if (cell_of) CU(cudaMemcpy(cell_of, E.d.cell_of + D.slot_off, sizeof(int) * D.cap, cudaMemcpyDeviceToHost));
    return PHMC_OK;
}

extern "C" int phmc_capacity(phmc_engine* h, int rep) {
    if (!h || rep < 0 || rep >= h->E.R) return -1;
    return h->caps[rep];
}

// ---------------------------------------------------------------------------
// learned surrogate: sample harvest, training on the harvest, attachment as the
// first stage of delayed acceptance, descriptor readback
// ---------------------------------------------------------------------------
extern "C" int phmc_harvest(phmc_engine* h, int capacity) {
    if (!h || capacity < 0) return fail(PHMC_ERR_ARG, "phmc_harvest: invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    drop_graph(h);  // captured launches hold the old buffers
    if (E.d.hv_cap > 0) { cudaFree(E.d.hv_rows); cudaFree(E.d.hv_sign); cudaFree(E.d.hv_target); cudaFree(E.d.hv_count); }
    E.d.hv_rows = nullptr; E.d.hv_sign = nullptr; E.d.hv_target = nullptr; E.d.hv_count = nullptr; E.d.hv_cap = 0;
    if (capacity == 0) return PHMC_OK;
    CU(cudaMalloc((void**)&E.d.hv_rows, sizeof(float) * (size_t)capacity * SUR_ROWS * SUR_K));
    CU(cudaMalloc((void**)&E.d.hv_sign, sizeof(float) * (size_t)capacity * SUR_ROWS));
    CU(cudaMalloc((void**)&E.d.hv_target, sizeof(float) * (size_t)capacity));
    CU(cudaMalloc((void**)&E.d.hv_count, sizeof(int)));
    CU(cudaMemset(E.d.hv_count, 0, sizeof(int)));
    E.d.hv_cap = capacity;
    return PHMC_OK;
}

static int harvest_n(phmc_engine* h, int* n) {
    Engine& E = h->E;
    int c = 0;
    if (E.d.hv_cap > 0) {
        CU(cudaStreamSynchronize(E.stream));
        CU(cudaMemcpy(&c, E.d.hv_count, sizeof(int), cudaMemcpyDeviceToHost));
    }
    *n = std::min(c, E.d.hv_cap);
    return PHMC_OK;
}

extern "C" int phmc_harvest_count(phmc_engine* h, int* n) {
    if (!h || !n) return fail(PHMC_ERR_ARG, "phmc_harvest_count: null argument");
    CU(cudaSetDevice(h->E.device));
    return harvest_n(h, n);
}

extern "C" int phmc_harvest_get(phmc_engine* h, int n, float* x, float* sign, float* t) {
    if (!h || n < 0 || (n > 0 && (!x || !sign || !t))) return fail(PHMC_ERR_ARG, "phmc_harvest_get: invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int have = 0;
    int s = harvest_n(h, &have);
    if (s) return s;
    if (n > have) return fail(PHMC_ERR_ARG, "phmc_harvest_get: fewer samples recorded than requested");
    if (n == 0) return PHMC_OK;
    CU(cudaMemcpy(x, E.d.hv_rows, sizeof(float) * (size_t)n * SUR_ROWS * SUR_K, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(sign, E.d.hv_sign, sizeof(float) * (size_t)n * SUR_ROWS, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(t, E.d.hv_target, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    return PHMC_OK;
}

extern "C" int phmc_surrogate_fit(phmc_engine* h, phmc_surrogate* sur, int epochs, int batch, float lr, float clip,
                                  uint64_t seed, double* loss) {
    if (!h || !sur) return fail(PHMC_ERR_ARG, "phmc_surrogate_fit: null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    int n = 0;
    int s = harvest_n(h, &n);
    if (s) return s;
    if (n < batch) return fail(PHMC_ERR_STATE, "phmc_surrogate_fit: fewer harvested samples than one batch");
    if (phmc_surrogate_num_params(sur) < 0) return fail(PHMC_ERR_ARG, "bad surrogate");
    s = sur_train_device(sur, E.d.hv_rows, E.d.hv_sign, E.d.hv_target, n, epochs, batch, lr, clip, seed, 1, loss);
    if (s) return s;
    // a network attached to this engine picks up the new weights
    if (E.d.sur.H > 0) {
        SurDev v;
        s = sur_device_view(sur, &v);
        if (s) return s;
        if (E.d.sur.w[0] == v.w[0]) { E.d.sur = v; drop_graph(h); }
    }
    return PHMC_OK;
}

extern "C" int phmc_surrogate_attach(phmc_engine* h, phmc_surrogate* sur, double threshold, int window) {
    if (!h || window < 0) return fail(PHMC_ERR_ARG, "phmc_surrogate_attach: invalid argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    SurDev v;
    std::memset(&v, 0, sizeof v);
    if (sur) {
        int s = sur_device_view(sur, &v);
        if (s) return s;
    }
    drop_graph(h);  // captured launches hold the old kernel parameters
    E.d.sur = v;
    E.first_stage_off = false;
    E.d.da_threshold = (float)threshold;
    E.d.da_window = window;
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    for (RepState& x : st) { x.da_eval = x.da_pass = x.da_acc = x.da_wpass = x.da_wacc = 0; x.da_off = 0; }
    CU(cudaMemcpy(E.d.state, st.data(), sizeof(RepState) * E.R, cudaMemcpyHostToDevice));
    return PHMC_OK;
}

extern "C" int phmc_get_da_stats(phmc_engine* h, phmc_da_stats* out) {
    if (!h || !out) return fail(PHMC_ERR_ARG, "phmc_get_da_stats: null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    std::vector<RepState> st((size_t)E.R);
    CU(cudaMemcpy(st.data(), E.d.state, sizeof(RepState) * E.R, cudaMemcpyDeviceToHost));
    for (int r = 0; r < E.R; ++r) {
        out[r].evaluated = st[r].da_eval; out[r].passed = st[r].da_pass; out[r].accepted = st[r].da_acc;
        out[r].fallback = st[r].da_off; out[r].pad = 0;
    }
    return PHMC_OK;
}

extern "C" int phmc_surrogate_describe(phmc_engine* h, int rep, const phmc_trial* trials, int n, float* out, double* dEs) {
    if (!h || (n > 0 && (!trials || !out || !dEs))) return fail(PHMC_ERR_ARG, "phmc_surrogate_describe: null argument");
    if (n == 0) return PHMC_OK;
    int s = check_trials(h, rep, trials, n);
    if (s) return s;
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    s = ensure_trial_buffers(h, n);
    if (s) return s;
    float* d_out = nullptr;
    CU(cudaMalloc((void**)&d_out, sizeof(float) * (size_t)n * DSC_STRIDE));
    CU(cudaMemcpyAsync(h->d_trials, trials, sizeof(phmc_trial) * n, cudaMemcpyHostToDevice, E.stream));
    E.d.dsc_out = d_out;
    cudaError_t e = launch_mc(E, MC_DESCRIBE, rep, h->d_trials, n, h->d_dE, E.stream);
    E.d.dsc_out = nullptr;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(float) * (size_t)n * DSC_STRIDE, cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dEs, h->d_dE, sizeof(double) * n, cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return fail(PHMC_ERR_CUDA, std::string("describe: ") + cudaGetErrorString(e));
    return check_kernel_errors(h);
}

extern "C" int phmc_set_da_log(phmc_engine* h, int* stage, double* dEs) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    Engine& E = h->E;
    if (!E.d.log_move) return fail(PHMC_ERR_STATE, "phmc_set_da_log needs a trial log (phmc_set_trial_log) first");
    drop_graph(h);
    if (E.d.log_stage) { cudaFree(E.d.log_stage); cudaFree(E.d.log_dEs); }
    E.d.log_stage = nullptr; E.d.log_dEs = nullptr;
    h->h_da_stage = stage; h->h_da_dEs = dEs;
    if (!stage || !dEs) return PHMC_OK;
    CU(cudaMalloc((void**)&E.d.log_stage, sizeof(int) * E.d.log_cap));
    CU(cudaMalloc((void**)&E.d.log_dEs, sizeof(double) * E.d.log_cap));
    return PHMC_OK;
}

extern "C" int phmc_set_move_mix(phmc_engine* h, int rep, double p_disp, double p_titr, double p_swap) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    Engine& E = h->E;
    if (rep < -1 || rep >= E.R) return fail(PHMC_ERR_ARG, "replica index out of range");
    if (p_disp < 0 || p_titr < 0 || p_swap < 0 || p_disp + p_titr + p_swap > 1.0 + 1e-12)
        return fail(PHMC_ERR_ARG, "move probabilities must be >= 0 with sum <= 1");
    const int r0 = rep < 0 ? 0 : rep, r1 = rep < 0 ? E.R : rep + 1;
    for (int r = r0; r < r1; ++r)
        if (p_swap > 0 && !(E.desc[r].salt_c2V2 > 0)) return fail(PHMC_ERR_ARG, "swap moves need salt_conc > 0");
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    for (int r = r0; r < r1; ++r) {
        RepDesc& D = E.desc[r];
        D.p_disp = (float)p_disp; D.p_titr = (float)p_titr; D.p_swap = (float)p_swap;
    }
    // the MC kernel reads the descriptor table at launch: captured launches stay valid
    CU(cudaMemcpy(E.d.desc, E.desc.data(), sizeof(RepDesc) * E.R, cudaMemcpyHostToDevice));
    return PHMC_OK;
}

// ---------------------------------------------------------------------------
// tuning: pending-stencil capacity (rebuild frequency against per-trial
// correction cost) and threads per replica block; both may change between runs
// ---------------------------------------------------------------------------
static int apply_tuning(phmc_engine* h, int pend, int threads) {
    Engine& E = h->E;
    const int old_p = E.pend_max, old_t = E.threads;
    E.pend_max = pend;
    E.threads = threads;
    cudaError_t e = prepare_mc(E);
    if (e != cudaSuccess) {
        E.pend_max = old_p; E.threads = old_t;
        return fail(PHMC_ERR_UNSUPPORTED, std::string("tuning does not fit the device: ") + cudaGetErrorString(e));
    }
    for (RepDesc& D : E.desc) D.pend_max = pend;
    CU(cudaMemcpy(E.d.desc, E.desc.data(), sizeof(RepDesc) * E.R, cudaMemcpyHostToDevice));
    drop_graph(h);  // captured launches hold the old launch shape
    return PHMC_OK;
}

extern "C" int phmc_set_tuning(phmc_engine* h, int pending_max, int threads) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    if (pending_max < 4 || pending_max > PHMC_MAX_PEND || (threads != 128 && threads != 256))
        return fail(PHMC_ERR_ARG, "pending_max must be in [4, 128] and threads 128 or 256");
    CU(cudaSetDevice(h->E.device));
    CU(cudaStreamSynchronize(h->E.stream));
    return apply_tuning(h, pending_max, threads);
}

extern "C" int phmc_set_quorum(phmc_engine* h, double quorum) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    if (!(quorum > 0.0 && quorum <= 1.0)) return fail(PHMC_ERR_ARG, "quorum must be in (0, 1]");
    CU(cudaSetDevice(h->E.device));
    CU(cudaStreamSynchronize(h->E.stream));
    h->E.quorum = (float)quorum;
    drop_graph(h);  // the quorum is a launch parameter of the captured MC launches
    return PHMC_OK;
}

extern "C" int phmc_set_zhist(phmc_engine* h, int nbins, int64_t every) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    if (nbins < 0 || nbins > PHMC_ZHIST_MAX_BINS) return fail(PHMC_ERR_ARG, "nbins must be in 0..PHMC_ZHIST_MAX_BINS");
    if (nbins > 0 && every < 1) return fail(PHMC_ERR_ARG, "every must be >= 1");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    if (E.d.zhist) { cudaFree(E.d.zhist); E.d.zhist = nullptr; }
    if (E.d.zh_samples) { cudaFree(E.d.zh_samples); E.d.zh_samples = nullptr; }
    E.d.zh_bins = 0;
    E.d.zh_every = 1;
    if (nbins > 0) {
        CU(cudaMalloc(&E.d.zhist, sizeof(unsigned long long) * 3 * nbins * (size_t)E.R));
        CU(cudaMalloc(&E.d.zh_samples, sizeof(long long) * (size_t)E.R));
        CU(cudaMemset(E.d.zhist, 0, sizeof(unsigned long long) * 3 * nbins * (size_t)E.R));
        CU(cudaMemset(E.d.zh_samples, 0, sizeof(long long) * (size_t)E.R));
        E.d.zh_bins = nbins;
        E.d.zh_every = every;
    }
    drop_graph(h);  // the captured MC launches hold the device pointers by value
    return PHMC_OK;
}

extern "C" int phmc_get_zhist(phmc_engine* h, int replica, double* counts, int64_t* n_samples) {
    if (!h || !counts || !n_samples) return fail(PHMC_ERR_ARG, "null argument");
    Engine& E = h->E;
    if (replica < 0 || replica >= E.R) return fail(PHMC_ERR_ARG, "replica index out of range");
    if (E.d.zh_bins <= 0) return fail(PHMC_ERR_STATE, "z-density profiles are off (phmc_set_zhist)");
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    const int nb = E.d.zh_bins;
    std::vector<unsigned long long> c((size_t)3 * nb);
    long long ns = 0;
    CU(cudaMemcpy(c.data(), E.d.zhist + (size_t)replica * 3 * nb, sizeof(unsigned long long) * 3 * nb, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&ns, E.d.zh_samples + replica, sizeof(long long), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3 * nb; ++k) counts[k] = (double)c[k];
    *n_samples = ns;
    return PHMC_OK;
}

extern "C" int phmc_set_event_callback(phmc_engine* h, phmc_event_fn fn, void* user) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    h->ev_fn = fn;
    h->ev_user = user;
    return PHMC_OK;
}

extern "C" int phmc_set_launch_budget(phmc_engine* h, int64_t max_launches) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    if (max_launches < 0) return fail(PHMC_ERR_ARG, "launch budget must be >= 0");
    h->launch_budget = max_launches;
    return PHMC_OK;
}

static void fill_tuning(const Engine& E, phmc_tuning* out) {
    std::memset(out, 0, sizeof *out);
    out->pending_max = E.pend_max;
    out->threads = E.threads;
    out->zpass = E.zreg;
    zreg_split(E.zreg, &out->zpass_n1, &out->zpass_n2);
    out->cand_round = E.cand_round;
    out->g_rows = E.g_rows;
    out->plane_pipe = E.fwd_pipe ? 1 : 0;
    out->energy_block = E.energy_block;
    out->first_stage = (E.d.sur.H > 0 && !E.first_stage_off) ? 1 : 0;
}

extern "C" int phmc_set_first_stage(phmc_engine* h, int on) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    CU(cudaSetDevice(h->E.device));
    CU(cudaStreamSynchronize(h->E.stream));
    h->E.first_stage_off = !on;
    drop_graph(h);
    return PHMC_OK;
}

extern "C" int phmc_get_tuning(phmc_engine* h, phmc_tuning* out) {
    if (!h || !out) return fail(PHMC_ERR_ARG, "null argument");
    fill_tuning(h->E, out);
    return PHMC_OK;
}

// Apply tile shapes (-1: unchanged) after checking them; the previous ones stay on failure.
static int apply_tiles(phmc_engine* h, int zpass, int cand_round, int energy_block, int g_rows = -1,
                       int plane_pipe = -1) {
    Engine& E = h->E;
    if (plane_pipe >= 0) {
        if (plane_pipe > 1) return fail(PHMC_ERR_ARG, "plane_pipe must be 0 or 1");
        E.fwd_pipe = plane_pipe == 1 && E.plane_reg;
    }
    if (zpass >= 0 && zpass != E.zreg) {
        int ids[8];
        const int n = E.zreg_default ? zreg_variants(E.desc[0].mesh[2], ids, 8) : 0;
        bool ok = zpass == 0;
        for (int k = 0; k < n; ++k) ok = ok || ids[k] == zpass;
        if (!ok || !E.use_r2c) return fail(PHMC_ERR_UNSUPPORTED, "z pass not available for these replicas' meshes");
        const int old = E.zreg;
        select_zpass(E, zpass);
        cudaError_t e = rebuild_set_smem_limits(E);
        if (e != cudaSuccess) {
            select_zpass(E, old);
            return fail(PHMC_ERR_UNSUPPORTED, std::string("z pass does not fit the device: ") + cudaGetErrorString(e));
        }
    }
    if ((cand_round >= 0 && cand_round != E.cand_round) || (g_rows >= 0 && g_rows != E.g_rows)) {
        if (cand_round >= 0 && cand_round != 2 && cand_round != 4 && cand_round != 8)
            return fail(PHMC_ERR_ARG, "cand_round must be 2, 4 or 8");
        if (g_rows >= 0 && !(g_rows >= 2 && g_rows <= 4) && g_rows != 21)
            return fail(PHMC_ERR_ARG, "g_rows must be 2, 3, 4 or 21");
        const int old_c = E.cand_round, old_g = E.g_rows;
        if (cand_round >= 0) E.cand_round = cand_round;
        if (g_rows >= 0) E.g_rows = g_rows;
        cudaError_t e = prepare_mc(E);
        if (e != cudaSuccess) {
            E.cand_round = old_c; E.g_rows = old_g;
            return fail(PHMC_ERR_UNSUPPORTED, "pair-pass shape not compiled: at order 5 (cand_round, g_rows) is one of "
                                              "(4, 2), (2, 2), (8, 2), (2, 3), (2, 4), (2, 21), (4, 21); (4, 2) at other orders");
        }
    }
    if (energy_block >= 0) {
        if (energy_block != 0 && energy_block != 64 && energy_block != 128 && energy_block != 256)
            return fail(PHMC_ERR_ARG, "energy_block must be 0 (cell order), 64, 128 or 256");
        E.energy_block = energy_block;
    }
    drop_graph(h);  // captured launches hold the old shapes
    return PHMC_OK;
}

extern "C" int phmc_set_tile_shapes(phmc_engine* h, int zpass, int cand_round, int g_rows, int energy_block,
                                    int plane_pipe) {
    if (!h) return fail(PHMC_ERR_ARG, "null engine");
    CU(cudaSetDevice(h->E.device));
    CU(cudaStreamSynchronize(h->E.stream));
    return apply_tiles(h, zpass, cand_round, energy_block, g_rows, plane_pipe);
}

// Device time (ms) of `reps` launches of f on the engine stream, after one untimed launch.
template <class F>
static int time_launches(Engine& E, int reps, F f, double* ms_out) {
    f();
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    CU(cudaEventRecord(a, E.stream));
    for (int k = 0; k < reps; ++k) f();
    CU(cudaEventRecord(b, E.stream));
    CU(cudaEventSynchronize(b));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CU(cudaGetLastError());
    *ms_out = ms / reps;
    return PHMC_OK;
}

extern "C" int phmc_autotune(phmc_engine* h, int64_t trials, phmc_tuning* results, int max_results, int* n_results) {
    if (!h || trials < 16) return fail(PHMC_ERR_ARG, "phmc_autotune: need trials >= 16");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    int n = 0;
    auto emit = [&](double us_trial, double us_rebuild, double us_recompute) {
        if (results && n < max_results) {
            fill_tuning(E, &results[n]);
            results[n].us_per_trial = us_trial; results[n].rebuild_us = us_rebuild; results[n].recompute_us = us_recompute;
        }
        ++n;
    };
    // 1. z pass: whole rebuilds of every replica's potential from its current charge mesh
    //    (the potential is a function of that mesh, so the timing leaves the state as it is)
    if (E.coulomb == PHMC_COUL_EWALD && E.use_r2c && E.zreg_default) {
        int ids[9] = {0};
        const int nv = zreg_variants(E.desc[0].mesh[2], ids + 1, 8) + 1;
        int best_id = E.zreg;
        double best = 1e300;
        for (int k = 0; k < nv; ++k) {
            if (apply_tiles(h, ids[k], -1, -1) != PHMC_OK) continue;
            double ms = 0.0;
            int s = time_launches(E, 10, [&]() { launch_rebuild_r2c(E, nullptr, 0, E.stream); }, &ms);
            if (s) return s;
            emit(0.0, ms * 1e3, 0.0);
            if (ms < best) { best = ms; best_id = ids[k]; }
        }
        int s = apply_tiles(h, best_id, -1, -1);
        if (s) return s;
    }
    // 1b. the first pass pipelined or not, with that z pass (the same whole rebuilds)
    if (E.coulomb == PHMC_COUL_EWALD && E.use_r2c && E.plane_reg) {
        double ms_pipe[2] = {1e300, 1e300};
        for (int pp = 0; pp < 2; ++pp) {
            if (apply_tiles(h, -1, -1, -1, -1, pp) != PHMC_OK) continue;
            int s = time_launches(E, 10, [&]() { launch_rebuild_r2c(E, nullptr, 0, E.stream); }, &ms_pipe[pp]);
            if (s) return s;
            int s2 = check_kernel_errors(h);
            if (s2) return s2;
            emit(0.0, ms_pipe[pp] * 1e3, 0.0);
        }
        int s = apply_tiles(h, -1, -1, -1, -1, ms_pipe[1] < ms_pipe[0] ? 1 : 0);
        if (s) return s;
    }
    // 2. full recompute's block size (pair / FENE pass and its reduction; the tracked
    //    pair energies it rewrites are those of the current state)
    {
        const int blocks[4] = {0, 64, 128, 256};
        int best_b = E.energy_block;
        double best = 1e300;
        for (int b : blocks) {
            apply_tiles(h, -1, -1, b);
            double ms = 0.0;
            int s = time_launches(E, 5, [&]() { launch_full_energy(E, E.stream); }, &ms);
            if (s) return s;
            emit(0.0, 0.0, ms * 1e3);
            if (ms < best) { best = ms; best_b = b; }
        }
        apply_tiles(h, -1, -1, best_b);
    }
    // 3. pending capacity x block size by trial runs; two passes over the candidates, each
    //    candidate's faster one kept: the chains move on while the tuner runs, and
    //    interleaving keeps that drift from favouring one candidate
    const int pends[] = {8, 16, 24, 32, 48, 64, 96, 128};
    const int ths[] = {128, 256};
    std::vector<double> best_us(16, 1e300);
    std::vector<char> fits(16, 0);
    auto time_run = [&](double* us) -> int {
        int s = phmc_run_loop(h, std::max<int64_t>(trials / 4, 4), 4);  // warm-up (captures the graph)
        if (s) return s;
        double ms = 0.0;
        s = phmc_run_timed(h, trials, &ms);
        if (s) return s;
        *us = ms * 1e3 / (double)trials;
        return PHMC_OK;
    };
    for (int pass = 0; pass < 2; ++pass) {
        int c = 0;
        for (int th : ths)
            for (int pm : pends) {
                const int k = c++;
                if (pm > PHMC_MAX_PEND || (pass == 1 && !fits[k])) continue;
                if (apply_tuning(h, pm, th) != PHMC_OK) continue;  // does not fit: skip
                fits[k] = 1;
                double us = 0.0;
                int s = time_run(&us);
                if (s) return s;
                best_us[k] = std::min(best_us[k], us);
            }
    }
    int best_p = E.pend_max, best_t = E.threads, c = 0;
    double best = 1e300;
    for (int th : ths)
        for (int pm : pends) {
            const int k = c++;
            if (!fits[k]) continue;
            if (best_us[k] < best) { best = best_us[k]; best_p = pm; best_t = th; }
        }
    c = 0;
    for (int th : ths)
        for (int pm : pends) {
            const int k = c++;
            if (!fits[k]) continue;
            if (results && n < max_results) {
                fill_tuning(E, &results[n]);
                results[n].pending_max = pm; results[n].threads = th; results[n].us_per_trial = best_us[k];
            }
            ++n;
        }
    int s = apply_tuning(h, best_p, best_t);
    if (s) return s;
    // 4. the pair pass's shape at that pending capacity and block size (order 5): round width
    //    (candidates per thread per round) x G rows in flight in the correction sum
    if (E.order == 5) {
        const int shapes[7][2] = {{4, 2}, {2, 2}, {8, 2}, {2, 3}, {2, 4}, {2, 21}, {4, 21}};
        constexpr int NSH = 7;
        double sbest[NSH] = {best, 1e300, 1e300, 1e300, 1e300, 1e300, 1e300};
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 1; k < NSH; ++k) {
                if (apply_tiles(h, -1, shapes[k][0], -1, shapes[k][1]) != PHMC_OK) continue;
                double us = 0.0;
                s = time_run(&us);
                if (s) return s;
                sbest[k] = std::min(sbest[k], us);
            }
        int bk = 0;
        for (int k = 1; k < NSH; ++k) {
            if (sbest[k] >= 1e300) continue;
            apply_tiles(h, -1, shapes[k][0], -1, shapes[k][1]);
            emit(sbest[k], 0.0, 0.0);
            if (sbest[k] < sbest[bk]) bk = k;
        }
        s = apply_tiles(h, -1, shapes[bk][0], -1, shapes[bk][1]);
        if (s) return s;
    }
    // 5. cost-based fallback of delayed acceptance: the attached surrogate's first stage
    //    against exact trials, both timed at the chosen shapes (two passes each)
    if (E.d.sur.H > 0) {
        double us_on = 1e300, us_off = 1e300;
        for (int pass = 0; pass < 2; ++pass)
            for (int off = 0; off < 2; ++off) {
                E.first_stage_off = off != 0;
                drop_graph(h);
                double us = 0.0;
                s = time_run(&us);
                if (s) { E.first_stage_off = false; return s; }
                (off ? us_off : us_on) = std::min(off ? us_off : us_on, us);
            }
        E.first_stage_off = false;
        emit(us_on, 0.0, 0.0);
        E.first_stage_off = true;
        emit(us_off, 0.0, 0.0);
        E.first_stage_off = us_off < us_on;
        drop_graph(h);
    }
    if (n_results) *n_results = n;
    return PHMC_OK;
}

extern "C" int phmc_delta_energy_components(phmc_engine* h, int rep, const phmc_trial* trials, int n,
                                            phmc_energy_components* out) {
    if (!h || (n > 0 && (!trials || !out))) return fail(PHMC_ERR_ARG, "null argument");
    if (n == 0) return PHMC_OK;
    int s = check_trials(h, rep, trials, n);
    if (s) return s;
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    s = ensure_trial_buffers(h, n);
    if (s) return s;
    double* d_c = nullptr;
    CU(cudaMalloc((void**)&d_c, sizeof(double) * 7 * (size_t)n));
    cudaError_t e = cudaMemcpyAsync(h->d_trials, trials, sizeof(phmc_trial) * n, cudaMemcpyHostToDevice, E.stream);
    E.d.ext_comp = d_c;
    if (e == cudaSuccess) e = launch_mc(E, MC_EVAL, rep, h->d_trials, n, h->d_dE, E.stream);
    E.d.ext_comp = nullptr;
    std::vector<double> hc((size_t)7 * n), dE((size_t)n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), d_c, sizeof(double) * 7 * n, cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dE.data(), h->d_dE, sizeof(double) * n, cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    cudaFree(d_c);
    if (e != cudaSuccess) return fail(PHMC_ERR_CUDA, std::string("delta_energy_components: ") + cudaGetErrorString(e));
    for (int k = 0; k < n; ++k) {
        const double* c = hc.data() + 7 * k;
        out[k].lj = c[0]; out[k].fene = c[1]; out[k].coul_real = c[2]; out[k].coul_recip = c[3];
        out[k].self = c[4]; out[k].qcorr = c[5]; out[k].slab = c[6]; out[k].total = dE[(size_t)k];
    }
    return check_kernel_errors(h);
}

// ---------------------------------------------------------------------------
// checkpoint / exact resume: everything that decides the chain's continuation
// (particle arrays, the index lists whose order the proposals draw from, the
// cell lists whose order fixes the summation order, per-replica counters and
// tracked FP64 energies and moments, move mix, tuning, and the fixed-point charge
// mesh of the wall bands); the potential is recomputed from the charge mesh
// ---------------------------------------------------------------------------
namespace {
const char kCkptMagic[8] = {'P', 'H', 'M', 'C', 'C', 'K', '0', '1'};
struct CkptRep {
    int cap, slot_off, ncell[3], mesh[3];
    float p_disp, p_titr, p_swap;
};
template <typename T>
bool ck_write_dev(FILE* f, const T* dptr, size_t n, std::vector<unsigned char>& buf) {
    buf.resize(n * sizeof(T));
    if (cudaMemcpy(buf.data(), dptr, n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    return fwrite(buf.data(), 1, buf.size(), f) == buf.size();
}
template <typename T>
bool ck_read_dev(FILE* f, T* dptr, size_t n, std::vector<unsigned char>& buf) {
    buf.resize(n * sizeof(T));
    if (fread(buf.data(), 1, buf.size(), f) != buf.size()) return false;
    return cudaMemcpy(dptr, buf.data(), n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}
}  // namespace

extern "C" int phmc_checkpoint_save(phmc_engine* h, const char* path) {
    if (!h || !path) return fail(PHMC_ERR_ARG, "phmc_checkpoint_save: null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    FILE* f = fopen(path, "wb");
    if (!f) return fail(PHMC_ERR_IO, std::string("cannot write ") + path);
    const DevPtrs& d = E.d;
    const size_t N = (size_t)E.total_slots, C = (size_t)E.total_cells;
    // version 2: the tile shapes follow the quorum (they fix summation orders, so an exact
    // resume needs them)
    const int hdr[7] = {2, E.R, E.total_slots, E.total_cells, E.cell_cap, (int)sizeof(RepState), E.pend_max};
    const int tiles[5] = {E.zreg, E.cand_round, E.energy_block, E.g_rows, E.fwd_pipe ? 1 : 0};
    bool ok = fwrite(kCkptMagic, 1, 8, f) == 8 && fwrite(hdr, sizeof(int), 7, f) == 7 &&
              fwrite(&E.threads, sizeof(int), 1, f) == 1 && fwrite(&E.quorum, sizeof(float), 1, f) == 1 &&
              fwrite(tiles, sizeof(int), 5, f) == 5;
    for (int r = 0; r < E.R && ok; ++r) {
        const RepDesc& D = E.desc[r];
        const CkptRep cr = {D.cap, D.slot_off, {D.ncell[0], D.ncell[1], D.ncell[2]}, {D.mesh[0], D.mesh[1], D.mesh[2]},
                            D.p_disp, D.p_titr, D.p_swap};
        ok = fwrite(&cr, sizeof cr, 1, f) == 1;
    }
    std::vector<unsigned char> buf;
    ok = ok && ck_write_dev(f, d.posq, N, buf) && ck_write_dev(f, d.type, N, buf) && ck_write_dev(f, d.flags, N, buf) &&
         ck_write_dev(f, d.bonds, N, buf) && ck_write_dev(f, d.cell_of, N, buf) && ck_write_dev(f, d.cell_pos, N, buf) &&
         ck_write_dev(f, d.mobile, N, buf) && ck_write_dev(f, d.mobile_pos, N, buf) && ck_write_dev(f, d.anions, N, buf) &&
         ck_write_dev(f, d.anion_pos, N, buf) && ck_write_dev(f, d.cations, N, buf) && ck_write_dev(f, d.cation_pos, N, buf) &&
         ck_write_dev(f, d.freel, N, buf) && ck_write_dev(f, d.titr, N, buf) && ck_write_dev(f, d.cell_count, C, buf) &&
         ck_write_dev(f, d.cell_list, C * E.cell_cap, buf) && ck_write_dev(f, d.cell_cls, C, buf) &&
         ck_write_dev(f, d.state, (size_t)E.R, buf);
    // the fixed-point charge mesh of the wall bands, last in the file
    if (ok && E.use_r2c) ok = ck_write_dev(f, d.qband, (size_t)E.total_qband, buf);
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(PHMC_ERR_IO, std::string("phmc_checkpoint_save: short write or device copy to ") + path);
    return PHMC_OK;
}

extern "C" int phmc_checkpoint_load(phmc_engine* h, const char* path) {
    if (!h || !path) return fail(PHMC_ERR_ARG, "phmc_checkpoint_load: null argument");
    Engine& E = h->E;
    CU(cudaSetDevice(E.device));
    CU(cudaStreamSynchronize(E.stream));
    FILE* f = fopen(path, "rb");
    if (!f) return fail(PHMC_ERR_IO, std::string("cannot read ") + path);
    auto bad = [&](const std::string& why) { fclose(f); return fail(PHMC_ERR_IO, "phmc_checkpoint_load: " + why + " (" + path + ")"); };
    char magic[8];
    int hdr[7], threads = 0;
    float quorum = 1.0f;
    if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kCkptMagic, 8) != 0) return bad("not a checkpoint");
    if (fread(hdr, sizeof(int), 7, f) != 7 || fread(&threads, sizeof(int), 1, f) != 1 || fread(&quorum, sizeof(float), 1, f) != 1)
        return bad("truncated header");
    if ((hdr[0] != 1 && hdr[0] != 2) || hdr[1] != E.R || hdr[2] != E.total_slots || hdr[3] != E.total_cells ||
        hdr[4] != E.cell_cap || hdr[5] != (int)sizeof(RepState))
        return bad("written by an engine with other replicas, capacities or cells");
    int tiles[5] = {E.zreg, E.cand_round, E.energy_block, E.g_rows, E.fwd_pipe ? 1 : 0};
    if (hdr[0] == 2 && fread(tiles, sizeof(int), 5, f) != 5) return bad("truncated header");
    std::vector<CkptRep> reps((size_t)E.R);
    for (int r = 0; r < E.R; ++r) {
        if (fread(&reps[r], sizeof(CkptRep), 1, f) != 1) return bad("truncated replica table");
        const RepDesc& D = E.desc[r];
        const CkptRep& c = reps[r];
        if (c.cap != D.cap || c.slot_off != D.slot_off || c.ncell[0] != D.ncell[0] || c.ncell[1] != D.ncell[1] ||
            c.ncell[2] != D.ncell[2] || c.mesh[0] != D.mesh[0] || c.mesh[1] != D.mesh[1] || c.mesh[2] != D.mesh[2])
            return bad("replica " + std::to_string(r) + " differs from this engine's");
    }
    const DevPtrs& d = E.d;
    const size_t N = (size_t)E.total_slots, C = (size_t)E.total_cells;
    std::vector<unsigned char> buf;
    const bool ok = ck_read_dev(f, d.posq, N, buf) && ck_read_dev(f, d.type, N, buf) && ck_read_dev(f, d.flags, N, buf) &&
                    ck_read_dev(f, d.bonds, N, buf) && ck_read_dev(f, d.cell_of, N, buf) && ck_read_dev(f, d.cell_pos, N, buf) &&
                    ck_read_dev(f, d.mobile, N, buf) && ck_read_dev(f, d.mobile_pos, N, buf) && ck_read_dev(f, d.anions, N, buf) &&
                    ck_read_dev(f, d.anion_pos, N, buf) && ck_read_dev(f, d.cations, N, buf) &&
                    ck_read_dev(f, d.cation_pos, N, buf) && ck_read_dev(f, d.freel, N, buf) && ck_read_dev(f, d.titr, N, buf) &&
                    ck_read_dev(f, d.cell_count, C, buf) && ck_read_dev(f, d.cell_list, C * E.cell_cap, buf) &&
                    ck_read_dev(f, d.cell_cls, C, buf) && ck_read_dev(f, d.state, (size_t)E.R, buf) &&
                    (!E.use_r2c || ck_read_dev(f, d.qband, (size_t)E.total_qband, buf));
    fclose(f);
    if (!ok) return fail(PHMC_ERR_IO, std::string("phmc_checkpoint_load: truncated file or device copy (") + path +
                                          "); the engine's state is undefined until the next phmc_set_state");
    // move mix and tuning as they were
    for (int r = 0; r < E.R; ++r) {
        E.desc[r].p_disp = reps[r].p_disp; E.desc[r].p_titr = reps[r].p_titr; E.desc[r].p_swap = reps[r].p_swap;
    }
    CU(cudaMemcpy(E.d.desc, E.desc.data(), sizeof(RepDesc) * E.R, cudaMemcpyHostToDevice));
    if (hdr[6] != E.pend_max || threads != E.threads) {
        const int s = apply_tuning(h, hdr[6], threads);
        if (s) return s;
    }
    {
        const int s = apply_tiles(h, tiles[0], tiles[1], tiles[2], tiles[3], tiles[4]);
        if (s) return s;
    }
    E.quorum = quorum;
    drop_graph(h);
    // potential from the restored charge mesh (the full-complex path spreads it from the
    // positions); the restored tracked energies stay
    CU(cudaMemsetAsync(E.d.dirty, 0, sizeof(int) * E.R, E.stream));
    if (E.coulomb == PHMC_COUL_EWALD) {
        if (!E.use_r2c) launch_spread(E, nullptr, E.stream);
        launch_fft_pipeline(E, nullptr, 1, E.stream);
        CU(cudaGetLastError());
    }
    return check_kernel_errors(h);
}
