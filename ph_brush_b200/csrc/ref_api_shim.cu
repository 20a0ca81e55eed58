// The reference's energy-layer API over the phmc C ABI.
//
// Implements the functions declared in the reference headers
//   MC/include/energy.hpp:7-18    compute_lj_sr_energy_gpu, compute_coul_sr_energy_gpu
//   MC/include/pme.hpp:42-49      pmeCreate, pmeDestroy, pmeEnergy
//   MC/include/neighbor.hpp:6-13  copy_csr_to_device, build_half_neighbors_gpu
// so that the reference's own driver and move loops (MC/src/main.cu, MC/src/mc.cu,
// MC/src/io.cpp, MC/src/report.cpp) link against libphmc.so in place of its
// energy sources (MC/src/energy_gpu.cu, pme.cu, neighbor.cu).  Compiled against the
// reference headers (-I<reference>/MC/include) with the reference's precision macro.
//
// The reference keeps atom positions fixed and changes identities (type, q) between
// energy calls with plain device writes (set_atom_identity, MC/src/mc.cu:33-41).
// One engine mirrors the atoms: each energy call finds the changed atoms with a
// device comparison against the engine's committed state; up to two changed atoms
// are evaluated as one trial against that state (one MC-kernel launch, no mesh
// rebuild); up to SHIM_MAX_CHANGES identity changes (the four-atom swaps of the
// reference's phase 2, a rejected swap's revert plus the next one) are committed
// pair by pair until two remain, which are then evaluated; moved atoms or more
// changes are uploaded as a new state (full recompute).  The model is the reference's: LJ cut and shifted at rc, 1-2 bonded
// pairs excluded from LJ and Coulomb, cubic-or-higher SPME with the reference's
// moduli and mesh rule, slab correction when pme_3dc is on.
#include <cuda_runtime.h>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <sstream>
#include "energy.hpp"
#include "gc_report.hpp"
#include "mc.hpp"
#include "neighbor.hpp"
#include "pme.hpp"
#include "phmc.h"
#include "report.hpp"

namespace {

void ck(int s, const char* what) {
    if (s != PHMC_OK) throw std::runtime_error(std::string(what) + ": " + phmc_last_error());
}
void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// smallest 2^a 3^b 5^c >= max(8, n) searched up to max(16, 2n + 32) (MC/src/pme.cu:46-51)
int fft_dim(int n) {
    const int nmax = std::max(16, n * 2 + 32);
    for (int m = std::max(8, n); m <= nmax; ++m) {
        int k = m;
        for (int p : {2, 3, 5})
            while (k % p == 0) k /= p;
        if (k == 1) return m;
    }
    return n;
}

// erfc(alpha rc) = rtol by bisection (used only when the caller left ewald_alpha unset)
double alpha_from_rtol(double rc, double rtol) {
    double lo = 0.0, hi = 10.0 / rc;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (std::erfc(mid * rc) > rtol) lo = mid; else hi = mid;
    }
    return 0.5 * (lo + hi);
}

template <typename T>
__global__ void k_shim_diff(int n, const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                            const T* __restrict__ q, const int* __restrict__ t, const float* __restrict__ mx,
                            const float* __restrict__ my, const float* __restrict__ mz, const float* __restrict__ mq,
                            const int* __restrict__ mt, int* __restrict__ idx, int* __restrict__ cnt, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool moved = (float)x[i] != mx[i] || (float)y[i] != my[i] || (float)z[i] != mz[i];
    const bool ident = (float)q[i] != mq[i] || t[i] != mt[i];
    if (moved) atomicOr(&cnt[1], 1);
    if (moved || ident) {
        const int k = atomicAdd(&cnt[0], 1);
        if (k < cap) idx[k] = i;
    }
}

#define SHIM_MAX_CHANGES 16
// the changed atoms' identities and positions, gathered for one copy to the host
struct ShimDiff {
    int cnt[2];
    int idx[SHIM_MAX_CHANGES];
    float q[SHIM_MAX_CHANGES], x[SHIM_MAX_CHANGES], y[SHIM_MAX_CHANGES], z[SHIM_MAX_CHANGES];
    int t[SHIM_MAX_CHANGES];
};
template <typename T>
__global__ void k_shim_gather(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                              const T* __restrict__ q, const int* __restrict__ t, ShimDiff* __restrict__ out) {
    const int k = threadIdx.x;
    if (k >= min(out->cnt[0], SHIM_MAX_CHANGES)) return;
    const int i = out->idx[k];
    out->q[k] = (float)q[i]; out->t[k] = t[i];
    out->x[k] = (float)x[i]; out->y[k] = (float)y[i]; out->z[k] = (float)z[i];
}

template <typename T>
__global__ void k_shim_mirror(int n, const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                              const T* __restrict__ q, const int* __restrict__ t, float* mx, float* my, float* mz,
                              float* mq, int* mt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    mx[i] = (float)x[i]; my[i] = (float)y[i]; mz[i] = (float)z[i]; mq[i] = (float)q[i]; mt[i] = t[i];
}

// pairs i < j with r <= rc (minimum image on all axes), 1-2 bonded pairs excluded (MC/src/neighbor.cu:74-125)
template <typename T>
__global__ void k_shim_count_pairs(int n, const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                                   T Lx, T Ly, T Lz, T rc2, const int* __restrict__ head, const int* __restrict__ list,
                                   unsigned long long* count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long c = 0;
    for (int j = i + 1; j < n; ++j) {
        T dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
        dx -= Lx * rint(dx / Lx); dy -= Ly * rint(dy / Ly); dz -= Lz * rint(dz / Lz);
        if (dx * dx + dy * dy + dz * dz > rc2) continue;
        bool bonded = false;
        if (head)
            for (int k = head[i]; k < head[i + 1]; ++k)
                if (list[k] == j) { bonded = true; break; }
        if (!bonded) ++c;
    }
    atomicAdd(count, c);
}

struct Shim {
    phmc_engine* eng = nullptr;
    int n = 0;
    // SPME settings (pmeCreate)
    bool pme = false;
    int mesh[3] = {0, 0, 0};
    int order = 4;
    double alpha = 0.0;
    bool slab = false;
    // 1-2 bonds (copy_csr_to_device)
    std::vector<int> bi, bj;
    // device mirror of the committed state
    float *mx = nullptr, *my = nullptr, *mz = nullptr, *mq = nullptr;
    int* mt = nullptr;
    ShimDiff* d_diff = nullptr;
    phmc_energy_components base{};
    // the last evaluated difference (reused by the next energy call when unchanged)
    int last_n = -1;
    int last_idx[2] = {-1, -1};
    float last_q[2] = {0, 0};
    int last_t[2] = {0, 0};
    phmc_energy_components cur{};
};
Shim g;

void release() {
    if (g.eng) phmc_destroy(g.eng);
    for (void* p : {(void*)g.mx, (void*)g.my, (void*)g.mz, (void*)g.mq, (void*)g.mt, (void*)g.d_diff})
        if (p) cudaFree(p);
    const bool pme = g.pme;
    const int mesh[3] = {g.mesh[0], g.mesh[1], g.mesh[2]};
    const int order = g.order;
    const double alpha = g.alpha;
    const bool slab = g.slab;
    std::vector<int> bi = g.bi, bj = g.bj;
    g = Shim();
    g.pme = pme; g.order = order; g.alpha = alpha; g.slab = slab;
    for (int k = 0; k < 3; ++k) g.mesh[k] = mesh[k];
    g.bi = bi; g.bj = bj;
}

template <typename V>
std::vector<double> to_host(const V& v) {
    thrust::host_vector<real> h(v.begin(), v.end());
    return std::vector<double>(h.begin(), h.end());
}

void upload_state(const DeviceAtoms& a) {
    thrust::host_vector<real> x(a.x.begin(), a.x.end()), y(a.y.begin(), a.y.end()), z(a.z.begin(), a.z.end()),
        q(a.q.begin(), a.q.end());
    thrust::host_vector<int> t(a.type.begin(), a.type.end());
    std::vector<float> fx(g.n), fy(g.n), fz(g.n), fq(g.n);
    std::vector<int> ti(t.begin(), t.end()), fl((size_t)g.n, 0);
    for (int i = 0; i < g.n; ++i) { fx[i] = (float)x[i]; fy[i] = (float)y[i]; fz[i] = (float)z[i]; fq[i] = (float)q[i]; }
    ck(phmc_set_state(g.eng, 0, fx.data(), fy.data(), fz.data(), fq.data(), ti.data(), fl.data()), "phmc_set_state");
}

void mirror(const DeviceAtoms& a) {
    k_shim_mirror<real><<<(g.n + 255) / 256, 256>>>(g.n, thrust::raw_pointer_cast(a.x.data()), thrust::raw_pointer_cast(a.y.data()),
                                                    thrust::raw_pointer_cast(a.z.data()), thrust::raw_pointer_cast(a.q.data()),
                                                    thrust::raw_pointer_cast(a.type.data()), g.mx, g.my, g.mz, g.mq, g.mt);
    cu(cudaDeviceSynchronize(), "shim mirror");
}

void ensure_engine(const DeviceAtoms& a, const DeviceParams& dp, const Box& box) {
    if (g.eng) return;
    g.n = (int)a.x.size();
    if (g.n <= 0) throw std::runtime_error("phmc shim: no atoms");
    const int T = dp.ntypes;
    std::vector<double> eps = to_host(dp.lj_eps), sig = to_host(dp.lj_sig);
    if ((int)eps.size() != T * T || (int)sig.size() != T * T) throw std::runtime_error("phmc shim: LJ tables must be ntypes^2");
    thrust::host_vector<real> x(a.x.begin(), a.x.end()), y(a.y.begin(), a.y.end()), z(a.z.begin(), a.z.end()),
        q(a.q.begin(), a.q.end());
    thrust::host_vector<int> t(a.type.begin(), a.type.end());
    std::vector<float> fx(g.n), fy(g.n), fz(g.n), fq(g.n);
    std::vector<int> ti(t.begin(), t.end()), fl((size_t)g.n, 0);
    for (int i = 0; i < g.n; ++i) { fx[i] = (float)x[i]; fy[i] = (float)y[i]; fz[i] = (float)z[i]; fq[i] = (float)q[i]; }
    phmc_system s;
    std::memset(&s, 0, sizeof s);
    s.n_particles = g.n; s.capacity = g.n;
    s.x = fx.data(); s.y = fy.data(); s.z = fz.data(); s.q = fq.data(); s.type = ti.data(); s.flags = fl.data();
    s.n_bonds = (int)g.bi.size(); s.bond_i = g.bi.data(); s.bond_j = g.bj.data();
    s.box[0] = box.Lx; s.box[1] = box.Ly; s.box[2] = box.Lz;
    phmc_params p;
    std::memset(&p, 0, sizeof p);
    p.n_types = T; p.lj_eps = eps.data(); p.lj_sig = sig.data(); p.lj_rc = nullptr; p.rc_lj = dp.rc;
    p.lj_shift = dp.lj_shift ? 1 : 0;
    if (dp.coulombtype == "pme") {
        if (!g.pme) throw std::runtime_error("phmc shim: pmeEnergy needs pmeCreate first");
        p.coulomb = PHMC_COUL_EWALD;
        for (int k = 0; k < 3; ++k) p.mesh[k] = g.mesh[k];
        p.order = g.order; p.ewald_alpha = g.alpha; p.slab = g.slab ? 1 : 0;
    } else if (dp.coulombtype == "coul_cut") {
        p.coulomb = PHMC_COUL_CUT;
    } else {
        throw std::runtime_error("phmc shim: unsupported coulombtype " + dp.coulombtype);
    }
    p.rc_coul = dp.rc; p.epsilon_r = dp.epsilon_r; p.ref_moduli = 1;
    p.excl_bonded_lj = 1; p.excl_bonded_coul = 1;
    p.beta = 1.0; p.seed = 1;
    int dev = 0;
    cu(cudaGetDevice(&dev), "cudaGetDevice");
    ck(phmc_create(1, &s, &p, dev, &g.eng), "phmc_create");
    ck(phmc_energy(g.eng, &g.base), "phmc_energy");
    cu(cudaMalloc((void**)&g.mx, sizeof(float) * g.n), "cudaMalloc");
    cu(cudaMalloc((void**)&g.my, sizeof(float) * g.n), "cudaMalloc");
    cu(cudaMalloc((void**)&g.mz, sizeof(float) * g.n), "cudaMalloc");
    cu(cudaMalloc((void**)&g.mq, sizeof(float) * g.n), "cudaMalloc");
    cu(cudaMalloc((void**)&g.mt, sizeof(int) * g.n), "cudaMalloc");
    cu(cudaMalloc((void**)&g.d_diff, sizeof(ShimDiff)), "cudaMalloc");
    mirror(a);
    g.cur = g.base;
    g.last_n = 0;
}

// Energy components of the atoms' current state.
const phmc_energy_components& evaluate(const DeviceAtoms& a, const DeviceParams& dp, const Box& box) {
    ensure_engine(a, dp, box);
    if ((int)a.x.size() != g.n) throw std::runtime_error("phmc shim: the number of atoms changed");
    cu(cudaMemset(g.d_diff, 0, sizeof(int) * 2), "cudaMemset");
    const real *ax = thrust::raw_pointer_cast(a.x.data()), *ay = thrust::raw_pointer_cast(a.y.data()),
               *az = thrust::raw_pointer_cast(a.z.data()), *aq = thrust::raw_pointer_cast(a.q.data());
    const int* at = thrust::raw_pointer_cast(a.type.data());
    char* dd = reinterpret_cast<char*>(g.d_diff);
    k_shim_diff<real><<<(g.n + 255) / 256, 256>>>(g.n, ax, ay, az, aq, at, g.mx, g.my, g.mz, g.mq, g.mt,
                                                  reinterpret_cast<int*>(dd + offsetof(ShimDiff, idx)),
                                                  reinterpret_cast<int*>(dd + offsetof(ShimDiff, cnt)), SHIM_MAX_CHANGES);
    k_shim_gather<real><<<1, SHIM_MAX_CHANGES>>>(ax, ay, az, aq, at, g.d_diff);
    ShimDiff df;
    cu(cudaMemcpy(&df, g.d_diff, sizeof df, cudaMemcpyDeviceToHost), "shim diff");
    const int nch = df.cnt[0];
    if (nch == 0) {
        g.last_n = 0;
        g.cur = g.base;
        return g.cur;
    }
    if (!df.cnt[1] && nch <= SHIM_MAX_CHANGES) {
        // changes in ascending atom order
        int ord[SHIM_MAX_CHANGES];
        for (int k = 0; k < nch; ++k) ord[k] = k;
        std::sort(ord, ord + nch, [&](int u, int v) { return df.idx[u] < df.idx[v]; });
        auto change = [&](phmc_trial& tr, int slot, int k) {
            tr.c[slot].index = df.idx[k]; tr.c[slot].present = 1;
            tr.c[slot].x = df.x[k]; tr.c[slot].y = df.y[k]; tr.c[slot].z = df.z[k];
            tr.c[slot].q = df.q[k]; tr.c[slot].type = df.t[k];
        };
        auto add = [](phmc_energy_components& e, const phmc_energy_components& d) {
            e.lj += d.lj; e.fene += d.fene; e.coul_real += d.coul_real; e.coul_recip += d.coul_recip;
            e.self += d.self; e.qcorr += d.qcorr; e.slab += d.slab; e.total += d.total;
        };
        // commit while more than two changes remain (ones or twos, so that two are left)
        int k0 = 0;
        while (nch - k0 > 2) {
            const int m = std::min(2, nch - k0 - 2);
            phmc_trial tr;
            std::memset(&tr, 0, sizeof tr);
            tr.n_changes = m;
            for (int j = 0; j < m; ++j) change(tr, j, ord[k0 + j]);
            phmc_energy_components d;
            ck(phmc_delta_energy_components(g.eng, 0, &tr, 1, &d), "phmc_delta_energy_components");
            ck(phmc_commit(g.eng, 0, &tr), "phmc_commit");
            add(g.base, d);
            for (int j = 0; j < m; ++j) {  // the mirror follows the committed state
                const int k = ord[k0 + j], i = df.idx[k];
                cu(cudaMemcpy(g.mq + i, &df.q[k], sizeof(float), cudaMemcpyHostToDevice), "shim mirror q");
                cu(cudaMemcpy(g.mt + i, &df.t[k], sizeof(int), cudaMemcpyHostToDevice), "shim mirror type");
            }
            g.last_n = -1;
            k0 += m;
        }
        const int rem = nch - k0;
        bool same = g.last_n == rem;
        for (int j = 0; j < rem && same; ++j) {
            const int k = ord[k0 + j];
            same = g.last_idx[j] == df.idx[k] && g.last_q[j] == df.q[k] && g.last_t[j] == df.t[k];
        }
        if (same) return g.cur;
        phmc_trial tr;
        std::memset(&tr, 0, sizeof tr);
        tr.n_changes = rem;
        for (int j = 0; j < rem; ++j) change(tr, j, ord[k0 + j]);
        phmc_energy_components d;
        ck(phmc_delta_energy_components(g.eng, 0, &tr, 1, &d), "phmc_delta_energy_components");
        g.cur = g.base;
        add(g.cur, d);
        g.last_n = rem;
        for (int j = 0; j < rem; ++j) {
            const int k = ord[k0 + j];
            g.last_idx[j] = df.idx[k]; g.last_q[j] = df.q[k]; g.last_t[j] = df.t[k];
        }
        return g.cur;
    }
    // more changes (or moved atoms): the current atoms become the committed state
    upload_state(a);
    ck(phmc_energy(g.eng, &g.base), "phmc_energy");
    mirror(a);
    g.cur = g.base;
    g.last_n = 0;
    return g.cur;
}

}  // namespace

// ---- MC/include/neighbor.hpp ----
DeviceCSR copy_csr_to_device(const CSR& host) {
    DeviceCSR d;
    d.rows = host.head.empty() ? 0 : (int)host.head.size() - 1;
    d.nnz = (int)host.list.size();
    d.head = thrust::device_vector<int>(host.head.begin(), host.head.end());
    d.list = thrust::device_vector<int>(host.list.begin(), host.list.end());
    // the 1-2 pairs (i < j) become the engine's bond list
    g.bi.clear(); g.bj.clear();
    for (int i = 0; i < d.rows; ++i)
        for (int k = host.head[i]; k < host.head[i + 1]; ++k)
            if (host.list[k] > i) { g.bi.push_back(i); g.bj.push_back(host.list[k]); }
    return d;
}

DeviceCSR build_half_neighbors_gpu(const DeviceAtoms& atoms, const Box& box, const DeviceCSR& bonds12_dev, real rc) {
    // The engine keeps its own cell list; the pair list itself is not needed.  Its
    // size is counted (the reference reports it) without storing it.
    DeviceCSR d;
    d.rows = (int)atoms.x.size();
    unsigned long long* cnt = nullptr;
    cu(cudaMalloc((void**)&cnt, sizeof(unsigned long long)), "cudaMalloc");
    cu(cudaMemset(cnt, 0, sizeof(unsigned long long)), "cudaMemset");
    const int* head = bonds12_dev.rows > 0 ? thrust::raw_pointer_cast(bonds12_dev.head.data()) : nullptr;
    const int* list = bonds12_dev.nnz > 0 ? thrust::raw_pointer_cast(bonds12_dev.list.data()) : nullptr;
    if (!list) head = nullptr;
    k_shim_count_pairs<real><<<(d.rows + 127) / 128, 128>>>(d.rows, thrust::raw_pointer_cast(atoms.x.data()),
                                                           thrust::raw_pointer_cast(atoms.y.data()),
                                                           thrust::raw_pointer_cast(atoms.z.data()), box.Lx, box.Ly, box.Lz,
                                                           rc * rc, head, list, cnt);
    unsigned long long h = 0;
    cudaError_t e = cudaMemcpy(&h, cnt, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(cnt);
    cu(e, "build_half_neighbors_gpu");
    d.nnz = (int)h;
    return d;
}

// ---- MC/include/energy.hpp ----
real compute_lj_sr_energy_gpu(const DeviceAtoms& atoms, const DeviceParams& dparams, const DeviceCSR&, const Box& box) {
    return (real)evaluate(atoms, dparams, box).lj;
}

real compute_coul_sr_energy_gpu(const DeviceAtoms& atoms, const DeviceParams& dparams, const DeviceCSR&, const Box& box) {
    if (dparams.coulombtype != "coul_cut") throw std::runtime_error("compute_coul_sr_energy_gpu: coulombtype must be coul_cut");
    return (real)evaluate(atoms, dparams, box).coul_real;
}

// ---- MC/include/pme.hpp ----
namespace {
// the parameters pmeCreate was given (pmeEnergy receives none); held on the heap and
// released by pmeDestroy, so no device vector outlives the CUDA runtime at exit
DeviceParams* g_pme_params = nullptr;
}

void pmeCreate(PMEPlan* plan, const DeviceParams& params, const Box& box, real rc) {
    if (!plan) throw std::runtime_error("pmeCreate: null plan");
    plan->order = params.pme_order;
    plan->use3dc = params.pme_3dc_enabled;
    plan->alpha = params.ewald_alpha > 0 ? params.ewald_alpha : (real)alpha_from_rtol(rc, params.ewald_rtol);
    plan->ewaldFactor = (real(M_PI) / plan->alpha) * (real(M_PI) / plan->alpha);
    plan->elFactor = real(138.935458) / params.epsilon_r;
    plan->vol = box.Lx * box.Ly * box.Lz;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) plan->recipBox[a][b] = 0;
    plan->recipBox[0][0] = real(1) / box.Lx; plan->recipBox[1][1] = real(1) / box.Ly; plan->recipBox[2][2] = real(1) / box.Lz;
    plan->nx = std::max(fft_dim((int)std::ceil(box.Lx / params.pme_spacing)), plan->order);
    plan->ny = std::max(fft_dim((int)std::ceil(box.Ly / params.pme_spacing)), plan->order);
    plan->nz = std::max(fft_dim((int)std::ceil(box.Lz / params.pme_spacing)), plan->order);
    plan->ngridReal = plan->nx * plan->ny * plan->nz;
    plan->ngridK = (plan->nx / 2 + 1) * plan->ny * plan->nz;
    plan->planR2C = 0;  // the engine's own FFT: no library plan
    if (g.eng) release();
    g.pme = true;
    g.mesh[0] = plan->nx; g.mesh[1] = plan->ny; g.mesh[2] = plan->nz;
    g.order = plan->order;
    g.alpha = plan->alpha;
    g.slab = plan->use3dc;
    delete g_pme_params;
    g_pme_params = new DeviceParams(params);
}

void pmeDestroy(PMEPlan* plan) {
    if (!plan) return;
    release();
    g.pme = false;
    delete g_pme_params;
    g_pme_params = nullptr;
}

real pmeEnergy(PMEPlan& plan, const DeviceAtoms& atoms, const DeviceCSR&, const Box& box, PMEEnergyComponents* components) {
    if (!g.pme || !g_pme_params) throw std::runtime_error("pmeEnergy: pmeCreate was not called");
    DeviceParams& dp = *g_pme_params;
    dp.coulombtype = "pme";
    const phmc_energy_components& c = evaluate(atoms, dp, box);
    if (components) {
        components->real_space = (real)c.coul_real;
        components->recip_space = (real)c.coul_recip;
        components->self_term = (real)c.self;
        components->qcorr_term = (real)(c.qcorr + c.slab);
    }
    (void)plan;
    return (real)(c.coul_real + c.coul_recip + c.self + c.qcorr + c.slab);
}

// ---- MC/include/mc.hpp: the grand-canonical mu-control phase on the device ----
// phase_gc_mu_control (MC/include/mc.hpp:73-82, MC/src/mc.cu:320-548) with the same
// arguments, results, report lines and generator stream, run by phmc_gc_phase in
// persistent MC-kernel launches instead of one host round trip per trial.  A driver
// calls it in place of phase_gc_mu_control (MC/src/main.cu:190).
namespace {

// The engine takes the atoms' current state (a device phase starts from it).
void adopt_atoms(const DeviceAtoms& d_atoms, const DeviceParams& d_params, const Box& box) {
    ensure_engine(d_atoms, d_params, box);
    upload_state(d_atoms);
    ck(phmc_energy(g.eng, &g.base), "phmc_energy");
    mirror(d_atoms);
    g.cur = g.base;
    g.last_n = 0;
}

// The atoms take the engine's identities after a device phase (host mirror and device arrays).
void take_identities(System& sys, DeviceAtoms& d_atoms) {
    std::vector<float> q((size_t)g.n);
    std::vector<int> t((size_t)g.n);
    ck(phmc_get_state(g.eng, 0, nullptr, nullptr, nullptr, q.data(), t.data(), nullptr), "phmc_get_state");
    thrust::host_vector<real> hq(d_atoms.q.begin(), d_atoms.q.end());
    thrust::host_vector<int> ht(d_atoms.type.begin(), d_atoms.type.end());
    for (int i = 0; i < g.n; ++i)
        if (t[(size_t)i] != ht[i] || q[(size_t)i] != (float)hq[i]) {
            ht[i] = t[(size_t)i]; hq[i] = (real)q[(size_t)i];
            sys.atoms[(size_t)i].type = t[(size_t)i] + 1;
            sys.atoms[(size_t)i].q = (real)q[(size_t)i];
        }
    d_atoms.q = hq;
    d_atoms.type = ht;
    mirror(d_atoms);
    ck(phmc_energy(g.eng, &g.base), "phmc_energy");
    g.cur = g.base;
    g.last_n = 0;
}

// std::mt19937's state words and position in its stream format, and back.
std::vector<uint32_t> rng_words(const std::mt19937& rng) {
    std::vector<uint32_t> mt(625);
    std::stringstream ss;
    ss << rng;
    for (uint32_t& v : mt) { unsigned long x = 0; ss >> x; v = (uint32_t)x; }
    return mt;
}
void rng_set(std::mt19937& rng, const std::vector<uint32_t>& mt) {
    std::stringstream ss;
    for (uint32_t v : mt) ss << v << ' ';
    ss >> rng;
}

}  // namespace

PhaseGCResult phmc_ref_phase_gc_mu_control(System& sys, DeviceAtoms& d_atoms, const DeviceParams& d_params,
                                           const DeviceCSR&, const Box& box, PMEPlan*, Params& p, const MCPlan& mcplan,
                                           std::mt19937& rng, Phase1Result* seed_out) {
    adopt_atoms(d_atoms, d_params, box);
    // pools as the reference builds them (MC/src/mc.cu:332-342)
    std::vector<int> nh_n = mcplan.idx_nh_n, nh_p = mcplan.idx_nh_p, w = mcplan.idx_w, cl;
    for (int j = 0; j < sys.natoms; ++j)
        if (sys.atoms[j].type == p.Cl_type && sys.atoms[j].z < mcplan.z_cut) cl.push_back(j);
    std::vector<uint32_t> mt = rng_words(rng);
    phmc_gc_job J;
    std::memset(&J, 0, sizeof J);
    J.replica = 0;
    J.nh_n_type = p.NH_N_type - 1; J.nh_p_type = p.NH_P_type - 1; J.w_type = p.W_type - 1; J.cl_type = p.Cl_type - 1;
    J.q_nh_p = 1.0f; J.q_cl = -1.0f;
    J.beta = p.beta; J.target_pct = p.target_protonation_pct; J.mu_eta = p.mu_eta; J.nacc_frac = p.sgmc_nacc_frac_round;
    J.gc_block = p.gc_block_fixed; J.epoch_attempt_max = p.sgmc_epoch_attempt_max;
    J.nh_n = nh_n.data(); J.n_nh_n = (int)nh_n.size();
    J.nh_p = nh_p.data(); J.n_nh_p = (int)nh_p.size();
    J.w = w.data(); J.n_w = (int)w.size();
    J.cl = cl.data(); J.n_cl = (int)cl.size();
    J.mt_state = mt.data();
    phmc_gc_result R;
    std::vector<phmc_gc_event> ev((size_t)1 << 10);
    // report lines written as the device phase runs (the reference writes them as it goes):
    // each record goes to the report stream from the engine's event callback
    struct Ctx { const phmc_gc_result* R; } ctx{&R};
    ck(phmc_set_event_callback(g.eng, [](void* u, int, int, const void* rec) {
           phmc_gc_write_event(mc_report(), *static_cast<const phmc_gc_event*>(rec), *static_cast<Ctx*>(u)->R);
       }, &ctx), "phmc_set_event_callback");
    const int rc = phmc_gc_phase(g.eng, 1, &J, &R, ev.data(), (int)ev.size());
    phmc_set_event_callback(g.eng, nullptr, nullptr);
    ck(rc, "phmc_gc_phase");
    rng_set(rng, mt);
    take_identities(sys, d_atoms);
    PhaseGCResult out;
    out.attempted = R.attempted; out.accepted = R.accepted;
    out.accepted_forward = R.accepted_forward; out.accepted_backward = R.accepted_backward;
    out.blocks_done = R.blocks_done;
    out.Nh = R.Nh; out.Nprot = R.Nprot; out.target_count = R.target_count;
    out.reached_target = R.reached_target != 0;
    out.E = (real)R.E;
    out.mu_eff = (real)R.mu_eff;
    p.mu_eff = out.mu_eff;
    if (seed_out && R.stop == PHMC_GC_STOP_REACHED) {  // pools for phase 2 (MC/src/mc.cu:475-492)
        seed_out->nh_p_mc.clear(); seed_out->nh_n_remaining.clear();
        seed_out->w_remaining.clear(); seed_out->cl_mc.clear();
        for (int idx = 0; idx < sys.natoms; ++idx) {
            const int ty = sys.atoms[(size_t)idx].type;
            const real zz = sys.atoms[(size_t)idx].z;
            if (ty == p.NH_P_type) seed_out->nh_p_mc.push_back(idx);
            else if (ty == p.NH_N_type) seed_out->nh_n_remaining.push_back(idx);
            else if (ty == p.W_type) { if (zz < mcplan.z_cut) seed_out->w_remaining.push_back(idx); }
            else if (ty == p.Cl_type) { if (zz < mcplan.z_cut) seed_out->cl_mc.push_back(idx); }
        }
        seed_out->E = out.E;
    }
    return out;
}

// phase2_swap_jitter (MC/include/mc.hpp:62-71, MC/src/mc.cu:159-318) with the same
// arguments, result, report lines and generator stream, run by phmc_phase2.  A driver
// calls it in place of phase2_swap_jitter (MC/src/main.cu:201).
Phase2Result phmc_ref_phase2_swap_jitter(System& sys, DeviceAtoms& d_atoms, const DeviceParams& d_params, const DeviceCSR&,
                                         const Box& box, PMEPlan*, const Params& p, const MCPlan& mcplan,
                                         const Phase1Result& ph1, std::mt19937& rng) {
    adopt_atoms(d_atoms, d_params, box);
    // pools as the reference keeps them (MC/src/mc.cu:173-183)
    std::vector<int> nh_p = ph1.nh_p_mc, nh_n = ph1.nh_n_remaining, w = ph1.w_remaining, cl = ph1.cl_mc;
    auto under_z = [&](std::vector<int>& pool) {
        pool.erase(std::remove_if(pool.begin(), pool.end(),
                                  [&](int i) { return i < 0 || i >= sys.natoms || sys.atoms[(size_t)i].z >= mcplan.z_cut; }),
                   pool.end());
    };
    under_z(w);
    under_z(cl);
    std::vector<uint32_t> mt = rng_words(rng);
    phmc_phase2_job J;
    std::memset(&J, 0, sizeof J);
    J.replica = 0;
    J.nh_n_type = p.NH_N_type - 1; J.nh_p_type = p.NH_P_type - 1; J.w_type = p.W_type - 1; J.cl_type = p.Cl_type - 1;
    J.q_nh_p = 1.0f; J.q_cl = -1.0f;
    J.beta = p.beta;
    J.max_attempts = p.max_attempts; J.patience = p.patience; J.energy_interval = p.energy_interval;
    J.z_cut = (float)mcplan.z_cut;
    J.nh_p = nh_p.data(); J.n_nh_p = (int)nh_p.size();
    J.nh_n = nh_n.data(); J.n_nh_n = (int)nh_n.size();
    J.w = w.data(); J.n_w = (int)w.size();
    J.cl = cl.data(); J.n_cl = (int)cl.size();
    J.mt_state = mt.data();
    phmc_phase2_result R;
    std::vector<phmc_phase2_event> ev((size_t)1 << 10);
    ck(phmc_set_event_callback(g.eng, [](void*, int, int, const void* rec) {
           phmc_p2_write_event(mc_report(), *static_cast<const phmc_phase2_event*>(rec));
       }, nullptr), "phmc_set_event_callback");
    const int rc = phmc_phase2(g.eng, 1, &J, &R, ev.data(), (int)ev.size());
    phmc_set_event_callback(g.eng, nullptr, nullptr);
    ck(rc, "phmc_phase2");
    rng_set(rng, mt);
    take_identities(sys, d_atoms);
    Phase2Result out;
    out.attempted = R.attempted;
    out.accepted = R.accepted;
    out.E = (real)R.E;
    out.best_E = (real)R.best_E;
    return out;
}
