// report.txt lines of the grand-canonical mu-control phase, written from the
// device's event records (phmc_gc_event) exactly as the reference's statements
// write them into its report stream (MC/src/mc.cu:367-373 already at target,
// :377 no valid pairs, :461-474 reached target, :506-516 chunk, :532-545 mu
// update): the same text, the same stream manipulators (precision 6 where the
// reference sets it, the stream's own precision where it does not), one line per
// event ended by std::endl.  Host C++ only.
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
