// report.txt lines of the reference's phases run on the device, written from the
// device's event records exactly as the reference's statements write them into
// its report stream: the same text, the same stream manipulators (the precision
// the reference sets, the stream's own precision where it sets none) and the same
// line ends (std::endl or a newline).
//   grand-canonical mu control (phmc_gc_event): MC/src/mc.cu:367-373 already at
//   target, :377 no valid pairs, :461-474 reached target, :506-516 chunk, :532-545
//   mu update;
//   phase 2 (phmc_phase2_event): MC/src/mc.cu:185-189 pools, :200-206 no proposals
//   before the first attempt, :214 no proposals, :296-308 step, :310-312 patience.
// Host C++ only.
#pragma once
#include <algorithm>
#include <iomanip>
#include <ostream>
#include "../../include/phmc.h"

template <class OS>
void phmc_gc_write_event(OS& os, const phmc_gc_event& e, const phmc_gc_result& r) {
    switch (e.kind) {
        case PHMC_GC_EV_ALREADY:
            os << "[sgmc] already at target: Nprot=" << e.nprot << "/" << r.Nh << " target=" << r.target_count
               << " mu/kT=" << e.mu_kT << " E=" << e.E << " remaining=0" << std::endl;
            break;
        case PHMC_GC_EV_NO_PAIRS:
            os << "[sgmc] no valid pairs to flip; stop." << std::endl;
            break;
        case PHMC_GC_EV_REACHED:
            os << std::setprecision(6) << "[sgmc] reached target in epoch=" << e.epoch << " step_in_block=" << e.step_in_block
               << " Nprot=" << e.nprot << "/" << r.Nh << " mu/kT=" << e.mu_kT << " E=" << e.E << " fwd_acc=" << e.fwd_total
               << " bwd_acc=" << e.bwd_total << " remaining=0" << std::endl;
            break;
        case PHMC_GC_EV_CHUNK:
            os << std::setprecision(6) << "[sgmc] chunk acc=" << e.acc_since_mu << "/" << r.Nacc_target
               << " attempts=" << e.att_since_mu << " acc_rate=" << e.acc_rate << " fwd_total=" << e.fwd_total
               << " bwd_total=" << e.bwd_total << " gc_block=" << r.gc_block << " remaining=" << e.remaining << std::endl;
            break;
        case PHMC_GC_EV_MU:
            os << std::setprecision(6) << "[sgmc] mu-update#" << (e.epoch + 1) << " cause=" << (e.cause_amax ? "Amax" : "Nacc")
               << " mu/kT=" << e.mu_kT << " f=" << e.f << " acc=" << e.acc_since_mu << "/" << r.Nacc_target
               << " attempts=" << e.att_since_mu << "/" << r.epoch_attempt_max << " fwd_total=" << e.fwd_total
               << " bwd_total=" << e.bwd_total << " remaining=" << e.remaining << " R0=" << r.R0 << " w_info=" << e.w_info
               << std::endl;
            break;
        default:
            break;
    }
}

template <class OS>
void phmc_p2_write_event(OS& os, const phmc_phase2_event& e) {
    switch (e.kind) {
        case PHMC_P2_EV_POOLS:
            os << "[phase2] pools: NH_P=" << e.n_nh_p << " NH_N=" << e.n_nh_n << " Cl=" << e.n_cl << " W=" << e.n_w
               << " (z_cut=" << e.z_cut << ")\n";
            break;
        case PHMC_P2_EV_NONE_AT_START:
            os << "[phase2] no valid proposals (no 4-pt and no wc-only). Stop.\n";
            break;
        case PHMC_P2_EV_WC_EMPTY:
            os << "[phase2] wc-only requested but pools empty; Stop.\n";
            break;
        case PHMC_P2_EV_NONE:
            os << "[phase2] no valid proposals; Stop.\n";
            break;
        case PHMC_P2_EV_STEP:
            os << std::setprecision(6) << "[phase2] step=" << e.attempted << " E=" << e.E << " accepted=" << e.accepted
               << " acc=" << std::setprecision(3) << e.acc << " since_best=" << e.since_best << "/" << e.patience
               << (e.mode_wc ? " mode=wc-only\n" : " mode=4-pt\n");
            break;
        case PHMC_P2_EV_PATIENCE:
            os << "[phase2] patience reached: " << e.since_best << "/" << e.patience << ". Stop.\n";
            break;
        default:
            break;
    }
}
