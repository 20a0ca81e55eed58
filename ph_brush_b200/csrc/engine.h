// Host-side engine object and kernel launchers (internal).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "common.cuh"

#define ZPASS_TX 16
#define ZREG_TX 16  // columns per block of the register z pass

struct Engine {
    int R = 0;
    int device = 0;
    int order = 4;
    int coulomb = 0;
    int total_slots = 0;
    int total_cells = 0;
    int cell_cap = 0;
    long long total_mesh = 0;
    long long total_oct = 0;
    int threads = 256;
    int pend_max = 16;
    int cand_round = 4;          // pair pass: candidates per thread per round (2, 4, 8 at order 5)
    int g_rows = 2;              // pending-correction sum: G rows in flight per thread (2; 3, 4 with round
                                 // width 2), or 21: one unit of stencil pairs per warp (round width 2 or 4)
    int energy_block = 128;      // full recompute: particles per block of the pair / FENE pass (0: cell order)
    bool first_stage_off = false;  // the attached surrogate's first stage bypassed (cost-based fallback)
    bool fwd_pipe = false;       // the rebuild's first pass pipelined (persistent blocks, bulk-copied planes)
    int nsm = 0;                 // the device's SM count
    float quorum = 0.2f;         // MC launch quorum of blocked replicas (1: every replica runs until it stops)
    cudaStream_t stream = nullptr;
    DevPtrs d{};
    std::vector<RepDesc> desc;
    // flush job tables
    int n_plane_jobs = 0, n_zjobs = 0;
    int2* d_plane_jobs = nullptr;
    int n_band_jobs = 0;
    int2* d_band_jobs = nullptr;  // (replica, z) of the planes in each replica's wall band
    int4* d_zjobs = nullptr;     // the active z pass's jobs and per-replica job offsets
    int* d_zjob_off = nullptr;
    int4* d_zj_stk = nullptr; int* d_zoff_stk = nullptr; int n_zj_stk = 0;  // shared-memory (Stockham) z pass
    int4* d_zj_reg = nullptr; int* d_zoff_reg = nullptr; int n_zj_reg = 0;  // register z pass
    size_t zpass_smem_stk = 0, zpass_smem_reg = 0;
    double* d_epart = nullptr;
    size_t plane_smem = 0, zpass_smem = 0;
    bool use_r2c = false;        // every replica has even nx: band charge mesh + real-to-complex rebuild
    size_t rb_fwd_smem = 0, rb_inv_smem = 0, band_spread_smem = 0;
    long long total_qband = 0;   // points of the wall bands' fixed-point charge meshes
    int zreg = 0;                // active register z-pass variant for the shared nz (0: shared-memory z pass)
    int zreg_default = 0;        // the default register variant of that nz (0: none; the Stockham pass only)
    bool plane_reg = false;      // register first / last passes (every replica's lateral mesh square and supported)
    int flush_kernels = 0;       // kernels per potential-mesh rebuild
    bool unit_pending = false;   // next rebuild places a unit charge instead of the particles
    long long total_meshh = 0;
    int* d_rep_of = nullptr;
    int* d_cell_rep = nullptr;   // replica of every global cell
    int* d_dirty = nullptr;      // per replica: mesh must be rebuilt
    int* d_active = nullptr;     // device counter: replicas still running
    int* h_active = nullptr;     // pinned mirror
    // full-energy scratch
    double* d_epair = nullptr;   // per (replica, block) partial components
    int energy_blocks = 0;
    int max_cap = 0;             // largest replica capacity (slots)
    int max_cells = 0;           // largest replica's cell count
    // host copies for trial logs
    std::vector<int> bonds_host;
    std::vector<void*> allocs;
    bool has_G = false;
};

// k_umma.cu: tcgen05 GEMM for the surrogate's training (N <= 256)
cudaError_t launch_umma_gemm(int M, int N, int K, const __nv_bfloat16* A, long sai, long sak, const __nv_bfloat16* B,
                             long sbk, long sbj, int epi, float* Cf, const float* bias, const float* Zin,
                             __nv_bfloat16* Hb, int kchunk, int splits, cudaStream_t st);
int umma_take_error(cudaStream_t st);

#define PHMC_FULL_MAX_BPR 64  // blocks per replica of the full-recompute pass at most

// engine.cu: records the thread's last error message
void phmc_set_error(int code, const std::string& msg);

// k_mesh.cu
void launch_spread(Engine& E, const int* dirty, cudaStream_t st);
void launch_fft_pipeline(Engine& E, const int* dirty, int mode, cudaStream_t st);
void launch_unit_charge(Engine& E, cudaStream_t st);
void launch_extract_octant(Engine& E, int r, cudaStream_t st);
cudaError_t mesh_set_smem_limits(Engine& E);

// k_rebuild.cu
void launch_rebuild_r2c(Engine& E, const int* dirty, int unit_charge, cudaStream_t st);
cudaError_t rebuild_set_smem_limits(Engine& E);
void launch_band_spread(Engine& E, cudaStream_t st);
int zreg_variant(int nz);      // default register z-pass variant for nz, 0 if none
int zreg_variants(int nz, int* ids, int max_ids);  // every register variant for nz
void zreg_split(int id, int* n1, int* n2);         // its two stages nz = n1 x n2
size_t zreg_smem(int nz);
bool plane_reg_supported(int nx, int ny);
size_t plane_reg_smem(int n);

// k_pair.cu
void launch_cell_build(Engine& E, cudaStream_t st);
void launch_full_energy(Engine& E, cudaStream_t st);

// k_mlp.cu (surrogate network)
int sur_device_view(phmc_surrogate* h, SurDev* out);
int sur_train_device(phmc_surrogate* h, const float* d_x, const float* d_sign, const float* d_t, int ns, int epochs,
                     int batch, float lr, float clip, uint64_t seed, int rescale, double* last_loss);

// k_mc.cu
enum { MC_RUN = 0, MC_EVAL = 1, MC_APPLY = 2, MC_DESCRIBE = 3, MC_GC = 4 };
cudaError_t launch_mc(Engine& E, int mode, int rep, const phmc_trial* d_trials, int n, double* d_dE, cudaStream_t st);
cudaError_t prepare_mc(Engine& E);
#define GC_EV_BYTES 80  // bytes of one event record of either device phase
cudaError_t launch_mc_gc(Engine& E, int n_jobs, cudaStream_t st);  // grand-canonical phase: one block per job
size_t mc_smem_bytes(int order, int pend_max, bool staged_surrogate = false, bool two_buffers = false);
