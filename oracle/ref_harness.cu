// ORACLE — test infrastructure only.  Measuring harness around the
// reference's own, unmodified code (MC/src/{energy_gpu,pme,neighbor,mc,io,
// report}, compiled from its sources by oracle/Makefile `ref`).  Runs on a GPU.
//
//   ref_harness energy <in.data> <params.in>
//       set-up exactly as MC/src/main.cu:102-176 (read, wrap, slab padding,
//       1-2 adjacency, upload, half list, pmeCreate) and prints the
//       reference's energies as one JSON line.
//   ref_harness time <in.data> <params.in> <trials> <warmup>
//       the same set-up, then the reference's phase-2 swap loop
//       (phase2_swap_jitter, MC/src/mc.cu:159-318: identity writes +
//       total_energy per trial) run for <warmup> then <trials> attempts with
//       patience disabled, timed with CUDA events; prints one JSON line.
//   ref_harness mix <list> <steps> <warmup> <trials> <p_disp> <disp_max> <seed>
//       every replica of <list> (base paths of ref_inputs' .data / .params /
//       .extra files) set up as above, then steps of <trials> trials per
//       replica, one replica after the other (the reference has no batching),
//       in the benchmark's move mix: with probability <p_disp> a displacement
//       of a mobile atom by up to <disp_max> per axis (outside the slab:
//       rejected without an energy), else the reference's grand-canonical pair
//       flip (MC/src/mc.cu:379-440) with mu held at kT ln10 (pKa - pH).  Each
//       trial is the reference's trial: device writes of the changed values
//       (as its set_atom_identity), its total energy (LJ over the half list +
//       pmeEnergy, MC/src/mc.cu:43-60), the acceptance, writes back on
//       rejection.  The half list is the one built at set-up (the reference
//       has no displacement moves and no list update).  Timed with CUDA events
//       around each whole step; prints one JSON line.
//   ref_harness alpha <base> <mu_kT> <blocks> <block_len> <nbins> <seed>
//       the reference's grand-canonical pair flips alone with mu fixed at
//       <mu_kT> kT: no mu feedback (MC/src/mc.cu:519-530) and no target stop
//       (:468-499); at the end of each block of <block_len> attempts the
//       protonated fraction and histograms over z in [0, height) of the
//       protonated sites and of the Cl ions, then the pools are rebuilt in
//       index order (the order the reference's phase hands them on in);
//       prints one JSON line.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <fstream>
#include <random>
#include <sstream>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "device_data.hpp"
#include "energy.hpp"
#include "io.hpp"
#include "mc.hpp"
#include "neighbor.hpp"
#include "pme.hpp"
#include "report.hpp"

static DeviceAtoms upload_atoms(const System& sys) {
    DeviceAtoms d;
    d.natoms = sys.natoms;
    std::vector<real> hx(sys.natoms), hy(sys.natoms), hz(sys.natoms), hq(sys.natoms);
    std::vector<int> ht(sys.natoms);
    for (int i = 0; i < sys.natoms; ++i) {
        hx[i] = sys.atoms[i].x; hy[i] = sys.atoms[i].y; hz[i] = sys.atoms[i].z; hq[i] = sys.atoms[i].q;
        ht[i] = sys.atoms[i].type - 1;
    }
    d.x.assign(hx.begin(), hx.end()); d.y.assign(hy.begin(), hy.end()); d.z.assign(hz.begin(), hz.end());
    d.q.assign(hq.begin(), hq.end()); d.type.assign(ht.begin(), ht.end());
    return d;
}

static DeviceParams upload_params(const Params& p) {
    DeviceParams dp;
    dp.ntypes = p.ntypes; dp.rc = p.rc; dp.epsilon_r = p.epsilon_r; dp.lj_shift = p.lj_shift;
    dp.coulombtype = p.coulombtype; dp.ewald_rtol = p.ewald_rtol; dp.ewald_alpha = p.ewald_alpha;
    dp.pme_spacing = p.pme_spacing; dp.pme_order = p.pme_order; dp.pme_3dc_enabled = p.pme_3dc_enabled;
    dp.pme_3dc_zfac = p.pme_3dc_zfac;
    dp.lj_eps.assign(p.lj_eps.begin(), p.lj_eps.end());
    dp.lj_sig.assign(p.lj_sig.begin(), p.lj_sig.end());
    if (p.lj_shift) dp.lj_shift_tbl.assign(p.lj_shift_tbl.begin(), p.lj_shift_tbl.end());
    return dp;
}

// One system in the reference's set-up (MC/src/main.cu:102-139) with the state its
// move loops keep: host mirror, device arrays, half list, PME plan, energy, pools.
struct RefReplica {
    System sys;
    Params p;
    DeviceAtoms da;
    DeviceCSR db, dn;
    DeviceParams dp;
    PMEPlan plan;
    bool pme = false;
    real E = 0;
    std::vector<int> nh_n, nh_p, w, cl, mobile;
    int n_native = 0;
    double height = 0, pH = 7, pKa = 7;
    std::mt19937 rng;
    long long att[2] = {0, 0}, acc[2] = {0, 0};

    void setup(const std::string& base, unsigned seed) {
        sys = read_lammps_full(base + ".data");
        if (sys.ntypes <= 0) { int tm = 0; for (auto& a : sys.atoms) tm = std::max(tm, a.type); sys.ntypes = tm; }
        p = read_params(base + ".params", sys.ntypes);
        wrap_positions(sys);
        if (p.pme_3dc_enabled) sys.box.Lz *= (p.pme_3dc_zfac < 2.0 ? real(2.0) : p.pme_3dc_zfac);
        CSR b12 = build_bond_adjacency(sys);
        da = upload_atoms(sys);
        db = copy_csr_to_device(b12);
        dn = build_half_neighbors_gpu(da, sys.box, db, p.rc);
        dp = upload_params(p);
        pme = p.coulombtype == "pme";
        if (pme) pmeCreate(&plan, dp, sys.box, p.rc);
        std::ifstream ex(base + ".extra");
        std::string key;
        int n_mob = 0;
        while (ex >> key) {
            if (key == "n_native") ex >> n_native;
            else if (key == "height") ex >> height;
            else if (key == "pH") ex >> pH;
            else if (key == "pKa") ex >> pKa;
            else if (key == "mobile") { ex >> n_mob; mobile.resize(n_mob); for (int& m : mobile) ex >> m; }
            else { std::string v; ex >> v; }
        }
        // pools as build_plan keeps them (MC/src/mc.cu:67-110): W and Cl below z_cut
        real zmax = 0;
        for (int i = 0; i < sys.natoms; ++i)
            if (sys.atoms[i].type == p.NH_N_type || sys.atoms[i].type == p.NH_P_type) zmax = std::max(zmax, sys.atoms[i].z);
        const real z_cut = zmax + p.w_z_extra_nm;
        for (int i = 0; i < sys.natoms; ++i) {
            const int ty = sys.atoms[i].type;
            if (ty == p.NH_N_type) nh_n.push_back(i);
            else if (ty == p.NH_P_type) nh_p.push_back(i);
            else if (ty == p.W_type && sys.atoms[i].z < z_cut) w.push_back(i);
            else if (ty == p.Cl_type && sys.atoms[i].z < z_cut) cl.push_back(i);
        }
        rng.seed(seed);
        E = energy();
    }
    void release() { if (pme) pmeDestroy(&plan); pme = false; }
    real energy() {
        const real elj = compute_lj_sr_energy_gpu(da, dp, dn, sys.box);
        const real ec = pme ? pmeEnergy(plan, da, dn, sys.box) : compute_coul_sr_energy_gpu(da, dp, dn, sys.box);
        return elj + ec;
    }
    template <class T>
    static void put(thrust::device_vector<T>& v, int i, T val) {
        cudaMemcpy(thrust::raw_pointer_cast(v.data()) + i, &val, sizeof(T), cudaMemcpyHostToDevice);
    }
    void set_identity(int i, int type1, real q) {
        sys.atoms[i].type = type1; sys.atoms[i].q = q;
        put(da.q, i, q); put(da.type, i, type1 - 1);
    }
    void set_position(int i, real x, real y, real z) {
        sys.atoms[i].x = x; sys.atoms[i].y = y; sys.atoms[i].z = z;
        put(da.x, i, x); put(da.y, i, y); put(da.z, i, z);
    }
    int pick(const std::vector<int>& pool) {
        std::uniform_int_distribution<int> u(0, (int)pool.size() - 1);
        return pool[u(rng)];
    }
    // the reference's pair flip with mu fixed (MC/src/mc.cu:379-466 without the target test)
    void gc_trial(real mu) {
        std::uniform_real_distribution<real> uni(0.0, 1.0);
        const long long a = nh_n.size(), b = nh_p.size(), c = w.size(), d = cl.size();
        const long long wf = a * c, wb = b * d, s_before = wf + wb;
        bool fwd;
        if (wf > 0 && wb > 0) fwd = uni(rng) < (real)wf / (real)(wf + wb);
        else if (wf > 0) fwd = true;
        else if (wb > 0) fwd = false;
        else return;
        const int i = fwd ? pick(nh_n) : pick(nh_p);
        const int j = fwd ? pick(w) : pick(cl);
        const int ti = sys.atoms[i].type, tj = sys.atoms[j].type;
        const real qi = sys.atoms[i].q, qj = sys.atoms[j].q;
        if (fwd) { set_identity(i, p.NH_P_type, +1.0); set_identity(j, p.Cl_type, -1.0); }
        else { set_identity(i, p.NH_N_type, 0.0); set_identity(j, p.W_type, 0.0); }
        const real Et = energy();
        const real dE = Et - E;
        const int s = fwd ? 1 : -1;
        const long long s_after = fwd ? (a - 1) * (c - 1) + (b + 1) * (d + 1) : (a + 1) * (c + 1) + (b - 1) * (d - 1);
        double logH = 0.0;
        if (s_before > 0 && s_after > 0) logH = std::log((double)s_before) - std::log((double)s_after);
        double expo = (double)(-p.beta * (dE - s * mu)) + logH;
        expo = std::clamp(expo, -40.0, 40.0);
        const bool accept = (expo >= 0.0) || (std::exp(expo) > (double)uni(rng));
        ++att[1];
        if (accept) {
            ++acc[1];
            E = Et;
            auto move = [](std::vector<int>& from, std::vector<int>& to, int v) {
                from.erase(std::find(from.begin(), from.end(), v)); to.push_back(v);
            };
            if (fwd) { move(nh_n, nh_p, i); move(w, cl, j); }
            else { move(nh_p, nh_n, i); move(cl, w, j); }
        } else {
            set_identity(i, ti, qi); set_identity(j, tj, qj);
        }
    }
    // displacement of a mobile atom, Metropolis on the reference's float energies
    void disp_trial(real dmax) {
        std::uniform_real_distribution<real> uni(0.0, 1.0);
        const int i = pick(mobile);
        const real ox = sys.atoms[i].x, oy = sys.atoms[i].y, oz = sys.atoms[i].z;
        real nx = ox + dmax * (2 * uni(rng) - 1), ny = oy + dmax * (2 * uni(rng) - 1), nz = oz + dmax * (2 * uni(rng) - 1);
        const real u = uni(rng);
        ++att[0];
        if (nz < 0 || nz >= (real)height) return;
        nx -= sys.box.Lx * std::floor(nx / sys.box.Lx);
        ny -= sys.box.Ly * std::floor(ny / sys.box.Ly);
        set_position(i, nx, ny, nz);
        const real Et = energy();
        const real dE = Et - E;
        const real expo = std::clamp(-p.beta * dE, (real)-40.0, (real)40.0);
        if (dE <= 0 || std::exp(expo) > u) { ++acc[0]; E = Et; }
        else set_position(i, ox, oy, oz);
    }
};

static int run_mix(int argc, char** argv) {
    if (argc < 9) { fprintf(stderr, "usage: mix <list> <steps> <warmup> <trials> <p_disp> <disp_max> <seed>\n"); return 1; }
    std::vector<std::string> bases;
    {
        std::ifstream in(argv[2]);
        std::string b;
        while (in >> b) bases.push_back(b);
    }
    const int steps = atoi(argv[3]), warmup = atoi(argv[4]), trials = atoi(argv[5]);
    const double p_disp = atof(argv[6]);
    const real dmax = (real)atof(argv[7]);
    const unsigned seed = (unsigned)atol(argv[8]);
    std::vector<RefReplica> reps(bases.size());
    auto s0 = std::chrono::steady_clock::now();
    for (size_t r = 0; r < bases.size(); ++r) reps[r].setup(bases[r], seed + (unsigned)r);
    cudaDeviceSynchronize();
    const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
    std::mt19937 mix(seed ^ 0x5bd1e995u);
    std::uniform_real_distribution<double> um(0.0, 1.0);
    auto step = [&]() {
        for (auto& R : reps)
            for (int k = 0; k < trials; ++k) {
                if (um(mix) < p_disp) R.disp_trial(dmax);
                else R.gc_trial((real)(std::log(10.0) * (R.pKa - R.pH)) / R.p.beta);
            }
    };
    for (int s = 0; s < warmup; ++s) step();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    std::vector<float> ms(steps);
    long long att0[2] = {0, 0}, acc0[2] = {0, 0};
    for (auto& R : reps) for (int k = 0; k < 2; ++k) { att0[k] += R.att[k]; acc0[k] += R.acc[k]; }
    for (int s = 0; s < steps; ++s) {
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        step();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[s], e0, e1);
    }
    long long att[2] = {0, 0}, acc[2] = {0, 0};
    for (auto& R : reps) for (int k = 0; k < 2; ++k) { att[k] += R.att[k]; acc[k] += R.acc[k]; }
    double tot = 0;
    for (float m : ms) tot += m;
    printf("{\"replicas\": %zu, \"setup_seconds\": %.3f, \"trials_per_replica_per_step\": %d, \"seconds\": %.6f, "
           "\"attempted\": [%lld, %lld], \"accepted\": [%lld, %lld], \"n_native\": [",
           reps.size(), setup_s, trials, tot * 1e-3, att[0] - att0[0], att[1] - att0[1], acc[0] - acc0[0], acc[1] - acc0[1]);
    for (size_t r = 0; r < reps.size(); ++r) printf("%s%d", r ? ", " : "", reps[r].n_native);
    printf("], \"natoms\": [");
    for (size_t r = 0; r < reps.size(); ++r) printf("%s%d", r ? ", " : "", reps[r].sys.natoms);
    printf("], \"meshes\": [");
    for (size_t r = 0; r < reps.size(); ++r) printf("%s[%d, %d, %d]", r ? ", " : "", reps[r].plan.nx, reps[r].plan.ny, reps[r].plan.nz);
    printf("], \"step_ms\": [");
    for (int s = 0; s < steps; ++s) printf("%s%.4f", s ? ", " : "", ms[s]);
    printf("]}\n");
    for (auto& R : reps) R.release();
    return 0;
}

static int run_alpha(int argc, char** argv) {
    if (argc < 8) { fprintf(stderr, "usage: alpha <base> <mu_kT> <blocks> <block_len> <nbins> <seed>\n"); return 1; }
    RefReplica R;
    R.setup(argv[2], (unsigned)atol(argv[7]));
    const double mu_kT = atof(argv[3]);
    const int blocks = atoi(argv[4]), blen = atoi(argv[5]), nbins = atoi(argv[6]);
    const real mu = (real)mu_kT / R.p.beta;
    const int nh = (int)(R.nh_n.size() + R.nh_p.size());
    printf("{\"natoms\": %d, \"Nh\": %d, \"mu_kT\": %.10g, \"block_len\": %d, \"nbins\": %d, \"height\": %.10g, \"blocks\": [",
           R.sys.natoms, nh, mu_kT, blen, nbins, R.height);
    for (int b = 0; b < blocks; ++b) {
        for (int k = 0; k < blen; ++k) R.gc_trial(mu);
        // the state at the block's end: protonated fraction and z-histograms; then the pools
        // rebuilt in index order (as the reference's phase hands them on, MC/src/mc.cu:475-492)
        std::vector<int> hp(nbins, 0), hc(nbins, 0);
        auto bin = [&](int i) { const int z = (int)(R.sys.atoms[i].z / R.height * nbins); return std::min(std::max(z, 0), nbins - 1); };
        for (int i : R.nh_p) hp[bin(i)]++;
        for (int i : R.cl) hc[bin(i)]++;
        printf("%s{\"alpha\": %.10g, \"sites\": [", b ? ", " : "", (double)R.nh_p.size() / nh);
        for (int k = 0; k < nbins; ++k) printf("%s%d", k ? ", " : "", hp[k]);
        printf("], \"cl\": [");
        for (int k = 0; k < nbins; ++k) printf("%s%d", k ? ", " : "", hc[k]);
        printf("]}");
        fflush(stdout);
        std::sort(R.nh_n.begin(), R.nh_n.end()); std::sort(R.nh_p.begin(), R.nh_p.end());
        std::sort(R.w.begin(), R.w.end()); std::sort(R.cl.begin(), R.cl.end());
    }
    printf("], \"attempted\": %lld, \"accepted\": %lld, \"E\": %.10g}\n", R.att[1], R.acc[1], (double)R.E);
    R.release();
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 4) { fprintf(stderr, "usage: %s energy|time data params [trials warmup]\n", argv[0]); return 1; }
    const std::string mode = argv[1];
    if (mode == "mix" || mode == "alpha") {
        try {
            ReportFileGuard guard("/tmp/ref_harness_report.txt");
            return mode == "mix" ? run_mix(argc, argv) : run_alpha(argc, argv);
        } catch (const std::exception& e) {
            fprintf(stderr, "Error: %s\n", e.what());
            return 2;
        }
    }
    try {
        ReportFileGuard guard("/tmp/ref_harness_report.txt");
        System sys = read_lammps_full(argv[2]);
        if (sys.ntypes <= 0) { int t = 0; for (auto& a : sys.atoms) t = std::max(t, a.type); sys.ntypes = t; }
        Params p = read_params(argv[3], sys.ntypes);
        wrap_positions(sys);
        if (p.pme_3dc_enabled) sys.box.Lz *= (p.pme_3dc_zfac < 2.0 ? real(2.0) : p.pme_3dc_zfac);
        CSR b12 = build_bond_adjacency(sys);
        DeviceAtoms da = upload_atoms(sys);
        DeviceCSR db = copy_csr_to_device(b12);
        DeviceCSR dn = build_half_neighbors_gpu(da, sys.box, db, p.rc);
        DeviceParams dp = upload_params(p);
        PMEPlan plan;
        const bool pme = p.coulombtype == "pme";
        if (pme) pmeCreate(&plan, dp, sys.box, p.rc);
        if (mode == "energy") {
            real elj = compute_lj_sr_energy_gpu(da, dp, dn, sys.box);
            PMEEnergyComponents c{};
            real ec = pme ? pmeEnergy(plan, da, dn, sys.box, &c) : compute_coul_sr_energy_gpu(da, dp, dn, sys.box);
            printf("{\"natoms\": %d, \"nnz\": %d, \"box\": [%.9g, %.9g, %.9g], \"mesh\": [%d, %d, %d], \"alpha\": %.12g, "
                   "\"E_lj\": %.10g, \"E_coul\": %.10g, \"real\": %.10g, \"recip\": %.10g, \"self\": %.10g, \"qcorr_slab\": %.10g}\n",
                   sys.natoms, dn.nnz, (double)sys.box.Lx, (double)sys.box.Ly, (double)sys.box.Lz, plan.nx, plan.ny, plan.nz,
                   (double)plan.alpha, (double)elj, (double)ec, (double)c.real_space, (double)c.recip_space,
                   (double)c.self_term, (double)c.qcorr_term);
        } else if (mode == "time") {
            const int trials = argc > 4 ? atoi(argv[4]) : 200;
            const int warmup = argc > 5 ? atoi(argv[5]) : 10;
            std::mt19937 rng((unsigned)p.rng_seed);
            MCPlan mp = build_plan(sys, p);
            auto pools = [&]() {
                Phase1Result r;
                for (int i = 0; i < sys.natoms; ++i) {
                    const int t = sys.atoms[i].type;
                    const real zz = sys.atoms[i].z;
                    if (t == p.NH_P_type) r.nh_p_mc.push_back(i);
                    else if (t == p.NH_N_type) r.nh_n_remaining.push_back(i);
                    else if (t == p.W_type && zz < mp.z_cut) r.w_remaining.push_back(i);
                    else if (t == p.Cl_type && zz < mp.z_cut) r.cl_mc.push_back(i);
                }
                return r;
            };
            p.patience = 1 << 30;
            p.energy_interval = 1 << 30;
            p.max_attempts = warmup;
            Phase1Result ph = pools();
            phase2_swap_jitter(sys, da, dp, dn, sys.box, pme ? &plan : nullptr, p, mp, ph, rng);
            ph = pools();
            p.max_attempts = trials;
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0); cudaEventCreate(&e1);
            cudaDeviceSynchronize();
            auto w0 = std::chrono::steady_clock::now();
            cudaEventRecord(e0);
            Phase2Result r = phase2_swap_jitter(sys, da, dp, dn, sys.box, pme ? &plan : nullptr, p, mp, ph, rng);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            auto w1 = std::chrono::steady_clock::now();
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double wall = std::chrono::duration<double>(w1 - w0).count();
            printf("{\"natoms\": %d, \"mesh\": [%d, %d, %d], \"trials\": %d, \"accepted\": %d, \"seconds\": %.6f, "
                   "\"wall_seconds\": %.6f, \"trials_per_s\": %.3f, \"E\": %.10g}\n",
                   sys.natoms, plan.nx, plan.ny, plan.nz, r.attempted, r.accepted, ms * 1e-3, wall,
                   r.attempted / (ms * 1e-3), (double)r.E);
        } else {
            fprintf(stderr, "unknown mode\n");
            return 1;
        }
        if (pme) pmeDestroy(&plan);
    } catch (const std::exception& e) {
        fprintf(stderr, "Error: %s\n", e.what());
        return 2;
    }
    return 0;
}
