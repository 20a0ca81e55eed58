// SPME mesh kernels: deterministic charge spreading, batched 3-D FFT passes
// (x/y planes resident in shared memory, z pencils in shared memory with the
// influence-function multiply fused between the forward and inverse z passes),
// potential-mesh readout.  Replaces k_spread_cubic + cuFFT R2C +
// k_recip_energy_and_apply of the reference (MC/src/pme.cu:140-249,384-422).
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include "common.cuh"
#include "engine.h"

#include "fft.cuh"

// ---------------------------------------------------------------------------
// Spreading: thread per slot; fixed-point (2^40) 64-bit atomics make the mesh
// bit-reproducible (integer addition is associative).
// ---------------------------------------------------------------------------
template <int P>
__global__ void k_spread(DevPtrs d, const int* __restrict__ rep_of, int total_slots, const int* __restrict__ dirty) {
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (gs >= total_slots) return;
    const int r = rep_of[gs];
    if (dirty && !dirty[r]) return;
    if (d.flags[gs] & PHMC_F_GHOST) return;
    const float4 pq = d.posq[gs];
    if (pq.w == 0.0f) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    float w[3][P];
    int base[3];
    const float g[3] = {pq.x / D.L[0] * (float)nx, pq.y / D.L[1] * (float)ny, pq.z / D.L[2] * (float)nz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float fl = floorf(g[k]);
        bspline_weights<P>(g[k] - fl, w[k]);
        base[k] = (int)fl + P / 2 - P + 1;
    }
    unsigned long long* q = d.qfix + D.mesh_off;
    for (int c = 0; c < P; ++c) {
        const int zc = wrap_idx(base[2] + c, nz);
        for (int b = 0; b < P; ++b) {
            const int yb = wrap_idx(base[1] + b, ny);
            const float wyz = pq.w * w[1][b] * w[2][c];
            for (int a = 0; a < P; ++a) {
                const int xa = wrap_idx(base[0] + a, nx);
                const long long v = __double2ll_rn((double)(wyz * w[0][a]) * PHMC_FIX_SCALE);
                atomicAdd(q + ((size_t)zc * ny + yb) * nx + xa, (unsigned long long)v);
            }
        }
    }
}

// Place a unit charge exactly on mesh point 0 of every replica (to obtain the
// influence kernel G as the potential of that charge).
__global__ void k_unit_charge(DevPtrs d, int R) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    d.qfix[d.desc[r].mesh_off] = (unsigned long long)(long long)PHMC_FIX_SCALE;
}

// ---------------------------------------------------------------------------
// xy plane pass.  job = (replica, z).  forward: fixed-point charges -> complex
// spectrum along x then y (the fixed-point plane is cleared for the next
// spread).  inverse: complex -> real potential, y then x.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) k_plane(DevPtrs d, const int2* __restrict__ jobs, int forward, const int* __restrict__ dirty) {
    extern __shared__ float2 sm[];
    const int2 job = jobs[blockIdx.x];
    const int r = job.x, z = job.y;
    if (dirty && !dirty[r]) return;
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1];
    const int P = nx * ny;
    float2* a = sm;
    float2* b = sm + P;
    const size_t off = (size_t)D.mesh_off + (size_t)z * P;
    if (forward) {
        unsigned long long* q = d.qfix + off;
        for (int i = threadIdx.x; i < P; i += NT) {
            const long long v = (long long)q[i];
            q[i] = 0ull;
            a[i] = make_float2((float)((double)v * PHMC_FIX_INV), 0.0f);
        }
        __syncthreads();
        float2* res = fft_lines<NT>(a, b, nx, ny, nx, 1, d.twiddle + D.tw_off[0], -1.0f, false);
        float2* oth = (res == a) ? b : a;
        res = fft_lines<NT>(res, oth, ny, nx, 1, nx, d.twiddle + D.tw_off[1], -1.0f, true);
        float2* c = d.cmesh + off;
        for (int i = threadIdx.x; i < P; i += NT) c[i] = res[i];
    } else {
        const float2* c = d.cmesh + off;
        for (int i = threadIdx.x; i < P; i += NT) a[i] = c[i];
        __syncthreads();
        float2* res = fft_lines<NT>(a, b, ny, nx, 1, nx, d.twiddle + D.tw_off[1], 1.0f, true);
        float2* oth = (res == a) ? b : a;
        res = fft_lines<NT>(res, oth, nx, ny, nx, 1, d.twiddle + D.tw_off[0], 1.0f, false);
        float* phi = d.phi + off;
        for (int i = threadIdx.x; i < P; i += NT) phi[i] = res[i].x;
    }
}

// ---------------------------------------------------------------------------
// z pencil pass with the influence multiply fused: forward FFT along z,
// E += w(kx) * theta(k) |F(k)|^2, F *= theta, inverse FFT along z.
// job = (replica, y, x0); TX columns per job.
// theta(k) = elf * exp(-(pi/alpha)^2 m^2) / (pi V m^2 Bx By Bz)   (MC/src/pme.cu:212-223)
// ---------------------------------------------------------------------------
template <int NT, int TX>
__global__ void __launch_bounds__(NT) k_zpass(DevPtrs d, const int4* __restrict__ jobs, double* __restrict__ epart,
                                              const int* __restrict__ dirty) {
    extern __shared__ float2 sm[];
    __shared__ double red[40];
    const int4 job = jobs[blockIdx.x];
    const int r = job.x, y = job.y, x0 = job.z;
    if (dirty && !dirty[r]) { if (threadIdx.x == 0) epart[blockIdx.x] = 0.0; return; }
    const RepDesc& D = d.desc[r];
    const int nx = D.mesh[0], ny = D.mesh[1], nz = D.mesh[2];
    const int tx_n = min(TX, nx - x0);
    float2* a = sm;
    float2* b = sm + TX * nz;
    float2* c = d.cmesh + D.mesh_off;
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e % TX;
        a[e] = (tx < tx_n) ? c[((size_t)z * ny + y) * nx + x0 + tx] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* res = fft_lines<NT>(a, b, nz, TX, 1, TX, d.twiddle + D.tw_off[2], -1.0f, true);
    const float* mx = d.moduli + D.mod_off[0];
    const float* my = d.moduli + D.mod_off[1];
    const float* mz = d.moduli + D.mod_off[2];
    const int myi = (y <= ny / 2) ? y : y - ny;
    const float kyv = (float)myi / D.L[1];
    const float pv = 3.14159265358979323846f * (float)D.V;
    double e_loc = 0.0;
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int kz = e / TX, tx = e % TX;
        const int kx = x0 + tx;
        float2 F = res[e];
        float th = 0.0f;
        if (tx < tx_n && !(kx == 0 && y == 0 && kz == 0)) {
            const int mxi = (kx <= nx / 2) ? kx : kx - nx;
            const int mzi = (kz <= nz / 2) ? kz : kz - nz;
            const float kxv = (float)mxi / D.L[0], kzv = (float)mzi / D.L[2];
            const float m2 = kxv * kxv + kyv * kyv + kzv * kzv;
            const float den = m2 * pv * mx[kx] * my[y] * mz[kz];
            if (den > 0.0f) th = D.elf * expf(-D.ewald_factor * m2) / den;
            float wgt = 1.0f;
            if (D.ref_corner) wgt = (kx > nx / 2) ? 0.0f : ((kx == 0 || kx == nx / 2) ? 1.0f : 2.0f);
            e_loc += (double)(wgt * th) * ((double)F.x * F.x + (double)F.y * F.y);
        }
        res[e] = make_float2(F.x * th, F.y * th);
    }
    __syncthreads();
    float2* oth = (res == a) ? b : a;
    res = fft_lines<NT>(res, oth, nz, TX, 1, TX, d.twiddle + D.tw_off[2], 1.0f, true);
    for (int e = threadIdx.x; e < nz * TX; e += NT) {
        const int z = e / TX, tx = e % TX;
        if (tx < tx_n) c[((size_t)z * ny + y) * nx + x0 + tx] = res[e];
    }
    const double s = block_sum<NT>(e_loc, red);
    if (threadIdx.x == 0) epart[blockIdx.x] = 0.5 * s;
}

// Per-replica reduction of the z-pass energy partials (fixed order) and the
// energy bookkeeping of a potential-mesh rebuild.  mode 0: rebuild after MC
// (update tracked energies, record drift); mode 1: plain recompute (set E_rec).
__global__ void k_flush_reduce(DevPtrs d, const int* __restrict__ zjob_off, const double* __restrict__ epart, int R,
                               int mode, const int* __restrict__ dirty) {
    // one block per replica; each thread sums a strided slice, then a fixed-order tree
    __shared__ double red[128];
    const int r = blockIdx.x;
    if (r >= R) return;
    if (dirty && !dirty[r]) return;
    double part = 0.0;
    for (int k = zjob_off[r] + threadIdx.x; k < zjob_off[r + 1]; k += blockDim.x) part += epart[k];
    red[threadIdx.x] = part;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double s = red[0];
    RepState& S = d.state[r];
    S.E_rec_flush = s;
    if (mode == 0) {
        S.drift = fabs(S.E_rec - s);
        S.E += s - S.E_rec;
        S.E_rec = s;
        S.flushes += 1;
        d.dirty[r] = 0;
    } else {
        S.E_rec = s;
    }
}

// Copy the non-negative octant of the potential of a unit charge (the
// influence kernel G, even in each axis) into the compact G table.
__global__ void k_extract_octant(DevPtrs d, int r) {
    const RepDesc& D = d.desc[r];
    const int ox = D.oct[0], oy = D.oct[1], oz = D.oct[2];
    const int total = ox * oy * oz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int x = i % ox, y = (i / ox) % oy, z = i / (ox * oy);
        d.goct[D.oct_off + i] = d.phi[D.mesh_off + ((size_t)z * D.mesh[1] + y) * D.mesh[0] + x];
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void launch_spread(Engine& E, const int* dirty, cudaStream_t st) {
    if (E.use_r2c) return;  // spreading is fused into the half-spectrum rebuild's first pass
    const int nt = 256, nb = (E.total_slots + nt - 1) / nt;
    switch (E.order) {
        case 4: k_spread<4><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
        case 5: k_spread<5><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
        case 6: k_spread<6><<<nb, nt, 0, st>>>(E.d, E.d_rep_of, E.total_slots, dirty); break;
    }
}

void launch_fft_pipeline(Engine& E, const int* dirty, int mode, cudaStream_t st) {
    if (E.use_r2c) {
        launch_rebuild_r2c(E, dirty, E.unit_pending ? 1 : 0, st);
        E.unit_pending = false;
    } else {
        k_plane<256><<<E.n_plane_jobs, 256, E.plane_smem, st>>>(E.d, E.d_plane_jobs, 1, dirty);
        k_zpass<256, ZPASS_TX><<<E.n_zjobs, 256, E.zpass_smem, st>>>(E.d, E.d_zjobs, E.d_epart, dirty);
        k_plane<256><<<E.n_plane_jobs, 256, E.plane_smem, st>>>(E.d, E.d_plane_jobs, 0, dirty);
    }
    k_flush_reduce<<<E.R, 128, 0, st>>>(E.d, E.d_zjob_off, E.d_epart, E.R, mode, dirty);
}

// Unit charge on mesh point 0 of every replica for the next pipeline run (the
// influence kernel G is that charge's potential).
void launch_unit_charge(Engine& E, cudaStream_t st) {
    if (E.use_r2c) { E.unit_pending = true; return; }
    k_unit_charge<<<(E.R + 127) / 128, 128, 0, st>>>(E.d, E.R);
}

void launch_extract_octant(Engine& E, int r, cudaStream_t st) { k_extract_octant<<<148, 256, 0, st>>>(E.d, r); }

// The cap is the device's opt-in maximum (not this engine's need), so that
// engines with different meshes can coexist on one device.
template <typename K>
static cudaError_t raise_dynamic_smem_cap(K kernel, int device, size_t need) {
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    const int cap = optin - (int)fa.sharedSizeBytes;  // static shared memory counts against the opt-in limit
    if (cap < (int)need) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

cudaError_t mesh_set_smem_limits(Engine& E) {
    cudaError_t e = raise_dynamic_smem_cap(k_plane<256>, E.device, E.plane_smem);
    if (e != cudaSuccess) return e;
    return raise_dynamic_smem_cap(k_zpass<256, ZPASS_TX>, E.device, E.zpass_smem);
}

// ---------------------------------------------------------------------------
// Reciprocal-space energy with no device allocation.
//
// For callers that must not allocate device memory: a host program whose
// device memory is all handed out by its own allocator (a framework's caching
// pool, a fixed per-process budget), a plugin called back from such a program,
// or a per-trial loop where an allocation's implicit device synchronisation
// would stall the pipeline.  The reference itself allocates a device scalar on
// every energy call (MC/src/energy_gpu.cu:55, MC/src/pme.cu:363).
//
// All scratch lives in one file-scope __device__ array (every GPU that loads
// the library holds it until the process exits): particle staging, the
// fixed-point charge mesh, the complex work mesh, FFT job tables, moduli,
// twiddles and the energy partials.  Limits: n <= PHMC_STATIC_MAX_PARTICLES,
// nx*ny*nz <= PHMC_STATIC_MAX_MESH, each mesh side <= 512.
// Every call shares the array and leaves its contents behind; the call clears
// what must start at zero.  The small host tables are staged in file-scope host
// arrays, shared by every host thread as well.  A process-wide lock serialises
// the calls and each call waits for its own GPU work before it returns, so
// calls made through this function never overlap; work that the caller queues
// on other streams in the same interval and that touches the array would race
// with it.  The array's device address is looked up once per device, on the
// first call made with that device current; it belongs to the device's primary
// context, so after a cudaDeviceReset of that device the entry point must not
// be called again in the process.
// ---------------------------------------------------------------------------
#define ST_MAX_N PHMC_STATIC_MAX_PARTICLES
#define ST_MAX_M PHMC_STATIC_MAX_MESH
#define ST_MAX_SIDE 512
#define ST_MAX_ZJOBS 4096
namespace {
constexpr size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t ST_OFF_QFIX = 0;
constexpr size_t ST_OFF_CMESH = ST_OFF_QFIX + al256(sizeof(unsigned long long) * ST_MAX_M);
constexpr size_t ST_OFF_POSQ = ST_OFF_CMESH + al256(sizeof(float2) * ST_MAX_M);
constexpr size_t ST_OFF_FLAGS = ST_OFF_POSQ + al256(sizeof(float4) * ST_MAX_N);
constexpr size_t ST_OFF_REP = ST_OFF_FLAGS + al256(sizeof(int) * ST_MAX_N);
constexpr size_t ST_OFF_MOD = ST_OFF_REP + al256(sizeof(int) * ST_MAX_N);
constexpr size_t ST_OFF_TW = ST_OFF_MOD + al256(sizeof(float) * 3 * ST_MAX_SIDE);
constexpr size_t ST_OFF_PJOB = ST_OFF_TW + al256(sizeof(float2) * 3 * ST_MAX_SIDE);
constexpr size_t ST_OFF_ZJOB = ST_OFF_PJOB + al256(sizeof(int2) * ST_MAX_SIDE);
constexpr size_t ST_OFF_ZOFF = ST_OFF_ZJOB + al256(sizeof(int4) * ST_MAX_ZJOBS);
constexpr size_t ST_OFF_EPART = ST_OFF_ZOFF + al256(sizeof(int) * 2);
constexpr size_t ST_OFF_DESC = ST_OFF_EPART + al256(sizeof(double) * ST_MAX_ZJOBS);
constexpr size_t ST_OFF_STATE = ST_OFF_DESC + al256(sizeof(RepDesc));
constexpr size_t ST_BYTES = ST_OFF_STATE + al256(sizeof(RepState));
}  // namespace

static __device__ __align__(256) unsigned char g_recip_scratch[ST_BYTES];

// Device address of g_recip_scratch per device, looked up on the first call made
// with that device current.
static unsigned char* g_recip_scratch_addr[64];

// Serialises the calls: the host staging tables below and the device array are
// shared by every host thread.
static std::mutex g_recip_static_lock;

// Host staging of the small tables (the same process-wide sharing rules apply).
static float4 h_st_posq[ST_MAX_N];
static int h_st_flags[ST_MAX_N];
static float h_st_mod[3 * ST_MAX_SIDE];
static float2 h_st_tw[3 * ST_MAX_SIDE];
static int2 h_st_pjob[ST_MAX_SIDE];
static int4 h_st_zjob[ST_MAX_ZJOBS];

static bool st_smooth(int n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5}) while (n % p == 0) n /= p;
    return n == 1;
}

// |DFT(M_p)|^2 on a length-n grid (same rule as the engine's moduli, written
// into a caller array).
static void st_moduli(int n, int order, int ref_style, float* out) {
    double d[16] = {0};
    const int s = order - 1;
    d[0] = 1.0;
    for (int k = 2; k <= s; ++k) {
        const double inv = 1.0 / k;
        for (int m = k - 1; m > 0; --m) d[m] = inv * ((k - m) * d[m - 1] + (m + 1) * d[m]);
        d[0] = inv * d[0];
    }
    double v[ST_MAX_SIDE];
    for (int i = 0; i < n; ++i) {
        double c = 0, sn = 0;
        for (int j = 0; j < s; ++j) {
            const double a = 2.0 * M_PI * i * (j + 1) / (double)n;
            c += d[j] * cos(a);
            sn += d[j] * sin(a);
        }
        v[i] = c * c + sn * sn;
        if (ref_style && !(v[i] > 0.0)) v[i] = 1e-30;
    }
    for (int i = 0; i < n; ++i) {
        double m = v[i];
        if (ref_style) {
            if (n % 2 == 0 && i == n / 2 && !(m > 0.0)) m = v[n / 2 - 1];
        } else if (m < 1e-7) {
            m = 0.5 * (v[(i - 1 + n) % n] + v[(i + 1) % n]);
        }
        out[i] = (float)m;
    }
}

extern "C" int phmc_recip_energy_static(const float* x, const float* y, const float* z, const float* q, int n,
                                        const double box[3], const int mesh[3], int order, double ewald_alpha,
                                        double epsilon_r, int ref_moduli, double* e_recip) {
    if (!x || !y || !z || !q || !box || !mesh || !e_recip || n < 0) {
        phmc_set_error(PHMC_ERR_ARG, "phmc_recip_energy_static: null argument or negative n");
        return PHMC_ERR_ARG;
    }
    if (n > ST_MAX_N) {
        phmc_set_error(PHMC_ERR_CAPACITY, "phmc_recip_energy_static: more particles than PHMC_STATIC_MAX_PARTICLES");
        return PHMC_ERR_CAPACITY;
    }
    if (order < 4 || order > 6 || !(ewald_alpha > 0) || !(epsilon_r > 0) || !(box[0] > 0 && box[1] > 0 && box[2] > 0)) {
        phmc_set_error(PHMC_ERR_ARG, "phmc_recip_energy_static: order must be 4..6, alpha/epsilon_r/box > 0");
        return PHMC_ERR_ARG;
    }
    const long long M = (long long)mesh[0] * mesh[1] * mesh[2];
    int zj = 0;
    for (int k = 0; k < 3; ++k)
        if (mesh[k] > ST_MAX_SIDE || !st_smooth(mesh[k]) || mesh[k] < order) {
            phmc_set_error(PHMC_ERR_CAPACITY, "phmc_recip_energy_static: each mesh side must be 2^a 3^b 5^c, >= order, <= 512");
            return PHMC_ERR_CAPACITY;
        }
    zj = mesh[1] * ((mesh[0] + ZPASS_TX - 1) / ZPASS_TX);
    const size_t plane_smem = (size_t)2 * mesh[0] * mesh[1] * sizeof(float2);
    const size_t zpass_smem = (size_t)2 * ZPASS_TX * mesh[2] * sizeof(float2);
    if (M > ST_MAX_M || zj > ST_MAX_ZJOBS || plane_smem > 227 * 1024 || zpass_smem > 227 * 1024) {
        phmc_set_error(PHMC_ERR_CAPACITY, "phmc_recip_energy_static: mesh larger than PHMC_STATIC_MAX_MESH points");
        return PHMC_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> serial(g_recip_static_lock);
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess || dev < 0 || dev >= 64) {
        phmc_set_error(PHMC_ERR_CUDA, std::string("phmc_recip_energy_static: no current device: ") + cudaGetErrorString(ce));
        return PHMC_ERR_CUDA;
    }
    if (!g_recip_scratch_addr[dev]) {  // set-up on this device's first call
        void* p = nullptr;
        ce = cudaGetSymbolAddress(&p, g_recip_scratch);
        if (ce != cudaSuccess || !p) {
            phmc_set_error(PHMC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
            return PHMC_ERR_CUDA;
        }
        g_recip_scratch_addr[dev] = (unsigned char*)p;
    }
    unsigned char* base = g_recip_scratch_addr[dev];
    // host tables
    RepDesc D;
    memset(&D, 0, sizeof D);
    D.cap = n; D.slot_off = 0;
    for (int k = 0; k < 3; ++k) { D.L[k] = (float)box[k]; D.mesh[k] = mesh[k]; D.oct[k] = mesh[k] / 2 + 1; }
    D.V = box[0] * box[1] * box[2];
    D.order = order; D.coulomb = PHMC_COUL_EWALD; D.ref_corner = ref_moduli;
    D.alpha = (float)ewald_alpha; D.elf = (float)(138.935458 / epsilon_r);
    D.ewald_factor = (float)((M_PI / ewald_alpha) * (M_PI / ewald_alpha));
    for (int k = 0; k < 3; ++k) {
        D.mod_off[k] = k * ST_MAX_SIDE;
        st_moduli(mesh[k], order, ref_moduli, h_st_mod + k * ST_MAX_SIDE);
        D.tw_off[k] = k * ST_MAX_SIDE;
        for (int j = 0; j < mesh[k]; ++j)
            h_st_tw[k * ST_MAX_SIDE + j] = make_float2((float)cos(-2.0 * M_PI * j / mesh[k]), (float)sin(-2.0 * M_PI * j / mesh[k]));
    }
    for (int i = 0; i < n; ++i) { h_st_posq[i] = make_float4(x[i], y[i], z[i], q[i]); h_st_flags[i] = 0; }
    for (int zz = 0; zz < mesh[2]; ++zz) h_st_pjob[zz] = make_int2(0, zz);
    int nzj = 0;
    for (int yy = 0; yy < mesh[1]; ++yy)
        for (int x0 = 0; x0 < mesh[0]; x0 += ZPASS_TX) h_st_zjob[nzj++] = make_int4(0, yy, x0, 0);
    const int zoff[2] = {0, nzj};
    // device pointers into the static array
    DevPtrs d;
    memset(&d, 0, sizeof d);
    d.qfix = (unsigned long long*)(base + ST_OFF_QFIX);
    d.cmesh = (float2*)(base + ST_OFF_CMESH);
    d.posq = (float4*)(base + ST_OFF_POSQ);
    d.flags = (int*)(base + ST_OFF_FLAGS);
    d.moduli = (float*)(base + ST_OFF_MOD);
    d.twiddle = (float2*)(base + ST_OFF_TW);
    d.desc = (RepDesc*)(base + ST_OFF_DESC);
    d.state = (RepState*)(base + ST_OFF_STATE);
    int* rep_of = (int*)(base + ST_OFF_REP);
    int2* pjob = (int2*)(base + ST_OFF_PJOB);
    int4* zjob = (int4*)(base + ST_OFF_ZJOB);
    int* zjob_off = (int*)(base + ST_OFF_ZOFF);
    double* epart = (double*)(base + ST_OFF_EPART);
    const cudaStream_t st = 0;
#define ST_CU(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            phmc_set_error(PHMC_ERR_CUDA, std::string("phmc_recip_energy_static: ") + #call + ": " + cudaGetErrorString(e_)); \
            return PHMC_ERR_CUDA;                                                                     \
        }                                                                                             \
    } while (0)
    // clear what must start at zero: the fixed-point mesh, replica ids, the state
    ST_CU(cudaMemsetAsync(d.qfix, 0, sizeof(unsigned long long) * (size_t)M, st));
    if (n > 0) ST_CU(cudaMemsetAsync(rep_of, 0, sizeof(int) * (size_t)n, st));
    ST_CU(cudaMemsetAsync(d.state, 0, sizeof(RepState), st));
    if (n > 0) {
        ST_CU(cudaMemcpyAsync(d.posq, h_st_posq, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
        ST_CU(cudaMemcpyAsync(d.flags, h_st_flags, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    }
    ST_CU(cudaMemcpyAsync(d.moduli, h_st_mod, sizeof(float) * 3 * ST_MAX_SIDE, cudaMemcpyHostToDevice, st));
    ST_CU(cudaMemcpyAsync(d.twiddle, h_st_tw, sizeof(float2) * 3 * ST_MAX_SIDE, cudaMemcpyHostToDevice, st));
    ST_CU(cudaMemcpyAsync(pjob, h_st_pjob, sizeof(int2) * mesh[2], cudaMemcpyHostToDevice, st));
    ST_CU(cudaMemcpyAsync(zjob, h_st_zjob, sizeof(int4) * nzj, cudaMemcpyHostToDevice, st));
    ST_CU(cudaMemcpyAsync(zjob_off, zoff, sizeof(zoff), cudaMemcpyHostToDevice, st));
    ST_CU(cudaMemcpyAsync(d.desc, &D, sizeof(RepDesc), cudaMemcpyHostToDevice, st));
    ST_CU(raise_dynamic_smem_cap(k_plane<256>, dev, plane_smem));
    ST_CU(raise_dynamic_smem_cap(k_zpass<256, ZPASS_TX>, dev, zpass_smem));
    if (n > 0) {
        const int nb = (n + 255) / 256;
        switch (order) {
            case 4: k_spread<4><<<nb, 256, 0, st>>>(d, rep_of, n, nullptr); break;
            case 5: k_spread<5><<<nb, 256, 0, st>>>(d, rep_of, n, nullptr); break;
            default: k_spread<6><<<nb, 256, 0, st>>>(d, rep_of, n, nullptr); break;
        }
    }
    k_plane<256><<<mesh[2], 256, plane_smem, st>>>(d, pjob, 1, nullptr);
    k_zpass<256, ZPASS_TX><<<nzj, 256, zpass_smem, st>>>(d, zjob, epart, nullptr);
    k_flush_reduce<<<1, 32, 0, st>>>(d, zjob_off, epart, 1, 1, nullptr);
    ST_CU(cudaGetLastError());
    RepState out;
    ST_CU(cudaMemcpyAsync(&out, d.state, sizeof(RepState), cudaMemcpyDeviceToHost, st));
    ST_CU(cudaStreamSynchronize(st));
#undef ST_CU
    *e_recip = out.E_rec;
    return PHMC_OK;
}
