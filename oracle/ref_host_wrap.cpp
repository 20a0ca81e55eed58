// ORACLE — test infrastructure only.  C wrapper over the reference's own host
// code (MC/src/io.cpp, compiled from its sources by oracle/Makefile `ref-host`)
// so that CPU tests can pin the engine's input parsing and derived parameters
// against the reference itself.
#include "io.hpp"
#include <cstring>
#include <exception>
#include <string>

static void set_err(char* err, int n, const char* msg) {
    if (err && n > 0) { std::strncpy(err, msg, n - 1); err[n - 1] = 0; }
}

// Params read by MC/src/io.cpp:171-301.  d[] = {rc, ewald_alpha, epsilon_r, pme_spacing,
// pme_3dc_zfac, beta, ewald_rtol, target_pct, w_z_extra_nm, mu_eta, sgmc_nacc_frac_round};
// i[] = {lj_shift, coulombtype(0 cut,1 pme,2 unknown), pme_order, pme_3dc_enabled, NH_N, NH_P,
// W, Cl, rng_seed, energy_interval, patience, max_attempts, direct_pct_threshold,
// gc_block_fixed, sgmc_epoch_attempt_max, phase2_wc}; eps/sig/shift are ntypes^2.
extern "C" int refh_read_params(const char* path, int ntypes, double* d, int* i,
                                double* eps, double* sig, double* shift, char* err, int errlen) {
    try {
        Params p = read_params(path, ntypes);
        d[0] = p.rc; d[1] = p.ewald_alpha; d[2] = p.epsilon_r; d[3] = p.pme_spacing; d[4] = p.pme_3dc_zfac;
        d[5] = p.beta; d[6] = p.ewald_rtol; d[7] = p.target_protonation_pct; d[8] = p.w_z_extra_nm;
        d[9] = p.mu_eta; d[10] = p.sgmc_nacc_frac_round;
        i[0] = p.lj_shift; i[1] = p.coulombtype == "coul_cut" ? 0 : (p.coulombtype == "pme" ? 1 : 2);
        i[2] = p.pme_order; i[3] = p.pme_3dc_enabled; i[4] = p.NH_N_type; i[5] = p.NH_P_type;
        i[6] = p.W_type; i[7] = p.Cl_type; i[8] = p.rng_seed; i[9] = p.energy_interval; i[10] = p.patience;
        i[11] = p.max_attempts; i[12] = p.direct_pct_threshold; i[13] = p.gc_block_fixed;
        i[14] = p.sgmc_epoch_attempt_max; i[15] = p.phase2_wc;
        for (int k = 0; k < ntypes * ntypes; ++k) { eps[k] = p.lj_eps[k]; sig[k] = p.lj_sig[k]; shift[k] = p.lj_shift_tbl[k]; }
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

// Data file read by MC/src/io.cpp:79-146, then wrap_positions (:303-316) and the
// 1-2 adjacency (:148-169).  Arrays must hold natoms (and head natoms+1, list 2*nbonds).
extern "C" int refh_read_data(const char* path, int* counts, double* box, int* id, int* mol, int* type,
                              double* q, double* x, double* y, double* z, int* head, int* list,
                              int cap, char* err, int errlen) {
    try {
        System s = read_lammps_full(path);
        counts[0] = s.natoms; counts[1] = (int)s.bonds.size(); counts[2] = s.ntypes;
        box[0] = s.box.Lx; box[1] = s.box.Ly; box[2] = s.box.Lz;
        if (s.natoms > cap) { set_err(err, errlen, "capacity"); return 2; }
        wrap_positions(s);
        for (int k = 0; k < s.natoms; ++k) {
            id[k] = s.atoms[k].id; mol[k] = s.atoms[k].mol; type[k] = s.atoms[k].type; q[k] = s.atoms[k].q;
            x[k] = s.atoms[k].x; y[k] = s.atoms[k].y; z[k] = s.atoms[k].z;
        }
        CSR c = build_bond_adjacency(s);
        for (int k = 0; k <= s.natoms; ++k) head[k] = c.head[k];
        for (size_t k = 0; k < c.list.size(); ++k) list[k] = c.list[k];
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}
