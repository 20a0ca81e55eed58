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
#include <cuda_runtime.h>
#include <chrono>
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

int main(int argc, char** argv) {
    if (argc < 4) { fprintf(stderr, "usage: %s energy|time data params [trials warmup]\n", argv[0]); return 1; }
    const std::string mode = argv[1];
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
