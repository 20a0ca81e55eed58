// C-ABI formatters of the device phases' report lines (include/phmc.h).
#include <cstring>
#include <sstream>
#include <string>
#include "gc_report.hpp"

extern "C" int phmc_gc_event_format(const phmc_gc_event* ev, const phmc_gc_result* res, char* buf, int cap) {
    if (!ev || !res) return -1;
    std::ostringstream os;
    os.setf(std::ios::fixed);  // the reference's report stream is in fixed notation from its start-up lines on
    os << std::setprecision(6);
    phmc_gc_write_event(os, *ev, *res);
    std::string line = os.str();
    if (!line.empty() && line.back() == '\n') line.pop_back();
    if (buf && cap > 0) {
        const size_t n = std::min(line.size(), (size_t)cap - 1);
        std::memcpy(buf, line.data(), n);
        buf[n] = '\0';
    }
    return (int)line.size();
}

extern "C" int phmc_phase2_event_format(const phmc_phase2_event* ev, char* buf, int cap) {
    if (!ev) return -1;
    std::ostringstream os;
    os.setf(std::ios::fixed);
    os << std::setprecision(6);
    phmc_p2_write_event(os, *ev);
    std::string line = os.str();
    if (!line.empty() && line.back() == '\n') line.pop_back();
    if (buf && cap > 0) {
        const size_t n = std::min(line.size(), (size_t)cap - 1);
        std::memcpy(buf, line.data(), n);
        buf[n] = '\0';
    }
    return (int)line.size();
}
