// Host-side input formats of the reference's driver, read and written without
// iostreams: LAMMPS "full" data files (the reference's reader
// MC/src/io.cpp:79-146, position wrap :303-316, writer :326-368) and params.in
// (MC/src/io.cpp:171-301), the latter as a superset that also carries the native
// model's keys.  The whole file is read at once and tokenised in place; numbers
// are converted by the same C library routines the reference's streams end in
// (strtod for values it reads as double, strtof for values it reads as float),
// so the parsed values are bit-identical to the reference's.
#include <cctype>
#include <charconv>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/phmc.h"

void phmc_set_error(int code, const std::string& msg);

namespace {

int fail(int code, const std::string& msg) {
    phmc_set_error(code, msg);
    return code;
}

bool slurp(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(&out[0], 1, (size_t)n, f) : 0;
    std::fclose(f);
    return got == out.size();
}

// std::isspace in the "C" locale (the locale the reference's program runs in)
inline bool is_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// One line with the surrounding white space removed (the reference's strip).
struct Line {
    const char* b;
    const char* e;
    bool empty() const { return b == e; }
    bool starts_with(const char* p) const {
        const size_t n = std::strlen(p);
        return (size_t)(e - b) >= n && std::memcmp(b, p, n) == 0;
    }
    bool contains(const char* p) const {
        const size_t n = std::strlen(p);
        if ((size_t)(e - b) < n) return false;
        for (const char* s = b; s + n <= e; ++s)
            if (std::memcmp(s, p, n) == 0) return true;
        return false;
    }
    std::string str() const { return std::string(b, e); }
};

class Lines {
  public:
    explicit Lines(const std::string& t) : p_(t.data()), end_(t.data() + t.size()) {}
    bool next(Line& l) {
        if (p_ >= end_) return false;
        const char* nl = static_cast<const char*>(std::memchr(p_, '\n', (size_t)(end_ - p_)));
        const char* le = nl ? nl : end_;
        const char* b = p_;
        const char* e = le;
        while (b < e && is_space(*b)) ++b;
        while (e > b && is_space(e[-1])) --e;
        l.b = b; l.e = e;
        p_ = nl ? nl + 1 : end_;
        return true;
    }

  private:
    const char* p_;
    const char* end_;
};

// White-space separated tokens of a line as [begin, end) ranges (<= 16 kept).
struct Spans {
    int n = 0;
    const char* b[16];
    const char* e[16];
    explicit Spans(const Line& l) {
        const char* s = l.b;
        while (s < l.e) {
            while (s < l.e && is_space(*s)) ++s;
            if (s >= l.e) break;
            const char* t = s;
            while (s < l.e && !is_space(*s)) ++s;
            if (n < 16) { b[n] = t; e[n] = s; }
            ++n;
        }
    }
};

// White-space separated tokens of a line, as NUL-terminated copies (<= 16 kept).
struct Tokens {
    int n = 0;
    char buf[16][64];
    explicit Tokens(const Line& l) {
        const char* s = l.b;
        while (s < l.e) {
            while (s < l.e && is_space(*s)) ++s;
            if (s >= l.e) break;
            const char* t = s;
            while (s < l.e && !is_space(*s)) ++s;
            if (n < 16) {
                const size_t len = std::min<size_t>((size_t)(s - t), 63);
                std::memcpy(buf[n], t, len);
                buf[n][len] = 0;
            }
            ++n;
        }
    }
};

// std::stoi: base-10 prefix with optional sign after leading white space; no digits -> error.
// std::from_chars reads the common forms (a '-' or no sign, decimal digits) the same way and
// faster; anything else goes to strtol, which std::stoi calls.
bool to_int(const char* s, int& v) {
    if (*s != '+') {
        const auto r = std::from_chars(s, s + std::strlen(s), v);
        if (r.ec == std::errc()) return true;
        if (r.ec == std::errc::result_out_of_range) return false;
    }
    errno = 0;
    char* end = nullptr;
    const long x = std::strtol(s, &end, 10);
    if (end == s || errno == ERANGE || x < -2147483648L || x > 2147483647L) return false;
    v = (int)x;
    return true;
}
// std::stod, then the reference's cast to its FP32 `real`.  std::from_chars is correctly
// rounded like strtod (which std::stod calls); signs, hexadecimal and out-of-range forms
// are left to strtod
bool to_real_via_double(const char* s, float& v) {
    if (*s != '+' && !std::strpbrk(s, "xX")) {
        double x = 0.0;
        const auto r = std::from_chars(s, s + std::strlen(s), x);
        if (r.ec == std::errc()) { v = (float)x; return true; }
    }
    errno = 0;
    char* end = nullptr;
    const double x = std::strtod(s, &end);
    if (end == s || (errno == ERANGE && std::isinf(x))) return false;
    v = (float)x;
    return true;
}
// stream extraction into the FP32 `real` (a direct correctly rounded conversion)
bool to_float(const char* s, float& v) {
    char* end = nullptr;
    const float x = std::strtof(s, &end);
    if (end == s) return false;
    v = x;
    return true;
}
// the conversions above on a token range: from_chars where it reads the same value,
// else a NUL-terminated copy through the C library routine
bool span_int(const char* b, const char* e, int& v) {
    if (*b != '+') {
        const auto r = std::from_chars(b, e, v);
        if (r.ec == std::errc()) return true;
        if (r.ec == std::errc::result_out_of_range) return false;
    }
    char t[64];
    const size_t n = std::min<size_t>((size_t)(e - b), 63);
    std::memcpy(t, b, n); t[n] = 0;
    return to_int(t, v);
}
bool span_real_via_double(const char* b, const char* e, float& v) {
    bool plain = *b != '+';
    for (const char* c = b; c < e && plain; ++c) plain = (*c != 'x' && *c != 'X');
    if (plain) {
        double x = 0.0;
        const auto r = std::from_chars(b, e, x);
        if (r.ec == std::errc()) { v = (float)x; return true; }
    }
    char t[64];
    const size_t n = std::min<size_t>((size_t)(e - b), 63);
    std::memcpy(t, b, n); t[n] = 0;
    errno = 0;
    char* end = nullptr;
    const double x = std::strtod(t, &end);
    if (end == t || (errno == ERANGE && std::isinf(x))) return false;
    v = (float)x;
    return true;
}

// `istringstream >> int` on the line's first token: 0 when it is not a number
int lead_int(const Line& l) {
    Tokens t(l);
    int v = 0;
    if (t.n == 0 || !to_int(t.buf[0], v)) return 0;
    return v;
}

struct Header {
    int natoms = 0, nbonds = 0, ntypes = 0;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// header pass of the reference's reader: counts and box bounds until "Atoms"
void read_header(const std::string& text, Header& h) {
    Lines ls(text);
    Line l;
    while (ls.next(l)) {
        if (l.empty()) continue;
        if (l.contains(" atoms") && !l.contains("atom types")) h.natoms = lead_int(l);
        else if (l.contains(" bonds") && !l.contains("bond types")) h.nbonds = lead_int(l);
        else if (l.contains(" atom types")) h.ntypes = lead_int(l);
        else {
            const char* ax[3] = {"xlo xhi", "ylo yhi", "zlo zhi"};
            bool box = false;
            for (int k = 0; k < 3 && !box; ++k)
                if (l.contains(ax[k])) {
                    Tokens t(l);
                    float a = 0.0f, b = 0.0f;
                    if (t.n >= 1 && to_float(t.buf[0], a)) {
                        h.lo[k] = a;
                        if (t.n >= 2 && to_float(t.buf[1], b)) h.hi[k] = b;
                    }
                    box = true;
                }
            if (!box && l.starts_with("Atoms")) break;
        }
    }
}

float wrap1(float r, float L) {  // MC/src/io.cpp:303-316, in FP32 as written there
    float w = r - std::floor(r / L) * L;
    if (w < 0) w += L;
    if (w >= L) w -= L;
    return w;
}

}  // namespace

extern "C" int phmc_lammps_header(const char* path, phmc_lammps_info* out) {
    if (!path || !out) return fail(PHMC_ERR_ARG, "phmc_lammps_header: null argument");
    std::string text;
    if (!slurp(path, text)) return fail(PHMC_ERR_IO, std::string("Failed to open LAMMPS data: ") + path);
    Header h;
    read_header(text, h);
    if (h.natoms <= 0) return fail(PHMC_ERR_IO, std::string("No atoms in header: ") + path);
    std::memset(out, 0, sizeof *out);
    out->natoms = h.natoms;
    out->nbonds = h.nbonds;
    out->ntypes = h.ntypes;
    for (int k = 0; k < 3; ++k) out->box[k] = (double)(h.hi[k] - h.lo[k]);
    return PHMC_OK;
}

extern "C" int phmc_lammps_read(const char* path, int wrap, int cap_atoms, int cap_bonds, int* id, int* mol, int* type,
                                float* q, float* x, float* y, float* z, int* bond_type, int* bond_i, int* bond_j,
                                phmc_lammps_info* info) {
    if (!path || !info || !id || !mol || !type || !q || !x || !y || !z || (cap_bonds > 0 && (!bond_type || !bond_i || !bond_j)))
        return fail(PHMC_ERR_ARG, "phmc_lammps_read: null argument");
    std::string text;
    if (!slurp(path, text)) return fail(PHMC_ERR_IO, std::string("Failed to open LAMMPS data: ") + path);
    Header h;
    read_header(text, h);
    if (h.natoms <= 0) return fail(PHMC_ERR_IO, std::string("No atoms in header: ") + path);
    if (h.natoms > cap_atoms) return fail(PHMC_ERR_CAPACITY, "phmc_lammps_read: more atoms than cap_atoms");
    float L[3];
    for (int k = 0; k < 3; ++k) L[k] = h.hi[k] - h.lo[k];
    // section pass: "Atoms" lines id mol type q x y z [...], "Bonds" lines id type i j.
    // Atom ids map to indices through a dense table when they are compact (the last
    // occurrence of an id wins, as in the reference's map), else through a hash map.
    std::unordered_map<int, int> id2idx;
    std::vector<int> dense;
    bool use_dense = false, index_built = false;
    auto build_index = [&](int na_) {
        int lo = 0, hi = -1;
        for (int i = 0; i < na_; ++i) { lo = (i == 0 || id[i] < lo) ? id[i] : lo; hi = (i == 0 || id[i] > hi) ? id[i] : hi; }
        use_dense = na_ > 0 && lo >= 0 && (long)hi <= 4L * na_ + 1024;
        if (use_dense) {
            dense.assign((size_t)hi + 1, -1);
            for (int i = 0; i < na_; ++i) dense[(size_t)id[i]] = i;
        } else {
            id2idx.reserve((size_t)na_ * 2);
            for (int i = 0; i < na_; ++i) id2idx[id[i]] = i;
        }
        index_built = true;
    };
    auto find_idx = [&](int key) -> int {
        if (use_dense) return (key >= 0 && (size_t)key < dense.size()) ? dense[(size_t)key] : -1;
        const auto it = id2idx.find(key);
        return it == id2idx.end() ? -1 : it->second;
    };
    int na = 0, nb = 0;
    bool in_atoms = false, in_bonds = false;
    Lines ls(text);
    Line l;
    while (ls.next(l)) {
        if (l.empty()) continue;
        if (l.starts_with("Atoms")) { in_atoms = true; in_bonds = false; continue; }
        if (l.starts_with("Bonds")) { in_atoms = false; in_bonds = true; continue; }
        if (l.starts_with("Angles") || l.starts_with("Dihedrals") || l.starts_with("Impropers") || l.starts_with("Velocities")) {
            in_atoms = in_bonds = false;
            continue;
        }
        if (in_atoms) {
            const Spans t(l);
            if (t.n < 7) continue;
            int a_id, a_mol, a_type;
            float a_q, a_x, a_y, a_z;
            if (!span_int(t.b[0], t.e[0], a_id) || !span_int(t.b[1], t.e[1], a_mol) || !span_int(t.b[2], t.e[2], a_type) ||
                !span_real_via_double(t.b[3], t.e[3], a_q) || !span_real_via_double(t.b[4], t.e[4], a_x) ||
                !span_real_via_double(t.b[5], t.e[5], a_y) || !span_real_via_double(t.b[6], t.e[6], a_z))
                return fail(PHMC_ERR_IO, "phmc_lammps_read: bad Atoms line: " + l.str());
            if (na >= cap_atoms) return fail(PHMC_ERR_CAPACITY, "phmc_lammps_read: more Atoms lines than cap_atoms");
            id[na] = a_id; mol[na] = a_mol; type[na] = a_type;
            q[na] = a_q; x[na] = a_x; y[na] = a_y; z[na] = a_z;
            ++na;
            index_built = false;
        } else if (in_bonds) {
            const Spans t(l);
            if (t.n < 4) continue;
            int b_id, b_type, ai, aj;
            if (!span_int(t.b[0], t.e[0], b_id) || !span_int(t.b[1], t.e[1], b_type) || !span_int(t.b[2], t.e[2], ai) ||
                !span_int(t.b[3], t.e[3], aj))
                return fail(PHMC_ERR_IO, "phmc_lammps_read: bad Bonds line: " + l.str());
            if (!index_built) build_index(na);
            const int ii = find_idx(ai), jj = find_idx(aj);
            if (ii < 0 || jj < 0) continue;  // bonds to unknown atoms are dropped
            if (nb >= cap_bonds) return fail(PHMC_ERR_CAPACITY, "phmc_lammps_read: more bonds than cap_bonds");
            bond_type[nb] = b_type; bond_i[nb] = ii; bond_j[nb] = jj;
            ++nb;
        }
    }
    if (na != h.natoms) return fail(PHMC_ERR_IO, "Atom count mismatch in Atoms section");
    if (wrap)
        for (int i = 0; i < na; ++i) { x[i] = wrap1(x[i], L[0]); y[i] = wrap1(y[i], L[1]); z[i] = wrap1(z[i], L[2]); }
    std::memset(info, 0, sizeof *info);
    info->natoms = na;
    info->nbonds = h.nbonds;
    info->nbonds_read = nb;
    info->ntypes = h.ntypes;
    for (int k = 0; k < 3; ++k) info->box[k] = (double)L[k];
    return PHMC_OK;
}

extern "C" int phmc_lammps_write(const char* path, int natoms, const int* id, const int* mol, const int* type, const float* q,
                                 const float* x, const float* y, const float* z, int nbonds, const int* bond_type,
                                 const int* bond_i, const int* bond_j, int ntypes, const double* box) {
    if (!path || natoms <= 0 || !id || !mol || !type || !q || !x || !y || !z || !box ||
        (nbonds > 0 && (!bond_type || !bond_i || !bond_j)))
        return fail(PHMC_ERR_ARG, "phmc_lammps_write: null argument or no atoms");
    for (int b = 0; b < nbonds; ++b)
        if (bond_i[b] < 0 || bond_i[b] >= natoms || bond_j[b] < 0 || bond_j[b] >= natoms)
            return fail(PHMC_ERR_ARG, "phmc_lammps_write: bond atom index out of range");
    int nbt = 0;
    for (int b = 0; b < nbonds; ++b) nbt = std::max(nbt, bond_type[b]);
    // the file is formatted into one buffer: integers and %.9g-equivalent values (9
    // significant digits give every FP32 value back exactly, through double, then FP32)
    std::string out;
    out.reserve((size_t)natoms * 72 + (size_t)nbonds * 32 + 256);
    char tmp[64];
    auto put_int = [&](long v) { const auto r = std::to_chars(tmp, tmp + sizeof tmp, v); out.append(tmp, r.ptr); };
    auto put_real = [&](double v) {
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v, std::chars_format::general, 9);
        out.append(tmp, r.ptr);
    };
    out += "LAMMPS data file (atom style full) written by phmc\n\n";
    put_int(natoms); out += " atoms\n";
    put_int(nbonds); out += " bonds\n\n";
    put_int(ntypes); out += " atom types\n";
    if (nbt > 0) { put_int(nbt); out += " bond types\n"; }
    const char* axes[3] = {" xlo xhi\n", " ylo yhi\n", " zlo zhi\n"};
    out += "\n";
    for (int k = 0; k < 3; ++k) { out += "0 "; put_real((double)(float)box[k]); out += axes[k]; }
    out += "\nAtoms # full\n\n";
    for (int i = 0; i < natoms; ++i) {
        put_int(id[i]); out += ' '; put_int(mol[i]); out += ' '; put_int(type[i]); out += ' ';
        put_real((double)q[i]); out += ' '; put_real((double)x[i]); out += ' '; put_real((double)y[i]); out += ' ';
        put_real((double)z[i]); out += '\n';
    }
    if (nbonds > 0) {
        out += "\nBonds\n\n";
        for (int b = 0; b < nbonds; ++b) {
            put_int(b + 1); out += ' '; put_int(bond_type[b]); out += ' '; put_int(id[bond_i[b]]); out += ' ';
            put_int(id[bond_j[b]]); out += '\n';
        }
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(PHMC_ERR_IO, std::string("Failed to open output data file: ") + path);
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    if (std::fclose(f) != 0 || !ok) return fail(PHMC_ERR_IO, std::string("short write to ") + path);
    return PHMC_OK;
}

// ---------------------------------------------------------------------------
// params.in
// ---------------------------------------------------------------------------
namespace {

// Ewald splitting parameter from the real-space tolerance: alpha = erfc^-1(rtol) / rc, with
// erf^-1 from Winitzki's approximation (a = 0.147) refined by three Newton steps on erf, as
// the reference computes it (MC/src/io.cpp:46-77), so that the derived alpha is the same
double erfinv_winitzki_newton(double x) {
    if (x <= -1.0) return -INFINITY;
    if (x >= 1.0) return INFINITY;
    const double a = 0.147;
    const double ln = std::log(1.0 - x * x);
    const double t1 = 2.0 / (M_PI * a) + ln / 2.0, t2 = ln / a;
    double v = std::sqrt(std::max(0.0, std::sqrt(t1 * t1 - t2) - t1));
    if (x < 0) v = -v;
    for (int i = 0; i < 3; ++i) v -= (std::erf(v) - x) / (2.0 / std::sqrt(M_PI) * std::exp(-v * v));
    return v;
}
double ewald_alpha_from_rtol(double rc, double rtol) {
    if (rtol <= 0.0) rtol = 1e-5;
    const double r = std::min(std::max(rtol, 1e-12), 0.5);
    const double y = r;
    const double inv = (y <= 0.0) ? INFINITY : (y >= 2.0 ? -INFINITY : erfinv_winitzki_newton(1.0 - y));
    return inv / rc;
}

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower(static_cast<unsigned char>(c));
    return s;
}
bool is_true(const std::string& v) { return v == "1" || v == "true" || v == "yes" || v == "on"; }

}  // namespace

extern "C" int phmc_params_read(const char* path, int ntypes, int strict, phmc_file_params* p, double* lj_eps,
                                double* lj_sig, double* lj_shift_tbl, char* unknown, int unknown_len) {
    if (!path || !p || ntypes < 1 || !lj_eps || !lj_sig || !lj_shift_tbl) return fail(PHMC_ERR_ARG, "phmc_params_read: null argument");
    std::string text;
    if (!slurp(path, text)) return fail(PHMC_ERR_IO, std::string("Failed to open params: ") + path);
    // the reference's defaults (its Params), FP32 values held in doubles
    std::memset(p, 0, sizeof *p);
    float rc = 0.0f, epsilon_r = 1.0f, ewald_rtol = 1e-5f, ewald_alpha = 0.0f, pme_spacing = 0.12f, zfac = 3.0f;
    float beta = (float)(1.0 / (0.008314462 * 300.0)), target_pct = 10.0f, w_z_extra = 1.0f, mu_eta = 0.3f, nacc_round = 0.10f;
    int lj_shift = 1, coulomb = PHMC_COUL_CUT, pme_order = 4, pme_3dc = 0;
    int nh_n = 4, nh_p = 5, w_t = 7, cl_t = 8, seed = 2025, energy_interval = 100, patience = 3000, max_attempts = 1000000;
    int direct_pct = 90, gc_block = 2000, epoch_max = 100000, phase2_wc = 1;
    // native keys: NaN / 0 when absent
    double nat[11];
    for (double& v : nat) v = NAN;
    const char* nat_keys[11] = {"ph", "pka", "salt_conc", "wall_lo", "wall_hi", "fene_k", "fene_r0", "p_disp", "p_titr", "p_swap", "disp_max"};
    int mesh[3] = {0, 0, 0};
    std::vector<float> eps((size_t)ntypes * ntypes, 0.0f), sig((size_t)ntypes * ntypes, 0.0f);
    std::string unk;
    auto bad = [&](const std::string& m) { return fail(PHMC_ERR_IO, "params " + std::string(path) + ": " + m); };

    Lines ls(text);
    Line l;
    while (ls.next(l)) {
        if (l.empty() || *l.b == '#') continue;
        const char* eq = static_cast<const char*>(std::memchr(l.b, '=', (size_t)(l.e - l.b)));
        if (eq) {
            Line kl{l.b, eq}, vl{eq + 1, l.e};
            while (kl.e > kl.b && is_space(kl.e[-1])) --kl.e;
            while (vl.b < vl.e && is_space(*vl.b)) ++vl.b;
            std::string key = kl.str();
            for (char& c : key) if (c == '-') c = '_';
            const std::string val = vl.str();
            if (key.empty()) continue;
            const char* v = val.c_str();
            float fv = 0.0f;
            int iv = 0;
            auto need_real = [&](float& dst) { if (!to_real_via_double(v, fv)) return false; dst = fv; return true; };
            auto need_int = [&](int& dst) { if (!to_int(v, iv)) return false; dst = iv; return true; };
            bool ok = true;
            const std::string lk = lower(key);
            if (key == "cutoff_nm") ok = need_real(rc);
            else if (key == "lj_shift") lj_shift = is_true(lower(val));
            else if (key == "epsilon_r") ok = need_real(epsilon_r);
            else if (key == "coulombtype") {
                const std::string lv = lower(val);
                coulomb = (lv == "coul_cut" || lv == "coulcut") ? PHMC_COUL_CUT : (lv == "pme" ? PHMC_COUL_EWALD : -1);
            } else if (key == "ewald_rtol") ok = need_real(ewald_rtol);
            else if (key == "ewald_alpha") ok = need_real(ewald_alpha);
            else if (key == "pme_spacing") ok = need_real(pme_spacing);
            else if (key == "pme_order") ok = need_int(pme_order);
            else if (key == "pme_3dc") {
                Tokens t(vl);
                const std::string flag = t.n >= 1 ? lower(t.buf[0]) : std::string("yes");
                float zf = zfac;
                if (t.n >= 2 && !to_float(t.buf[1], zf)) zf = 0.0f;  // a failed extraction stores 0
                pme_3dc = is_true(flag);
                zfac = zf < 2.0f ? 2.0f : zf;
            } else if (key == "nh_n_type") ok = need_int(nh_n);
            else if (key == "nh_p_type") ok = need_int(nh_p);
            else if (key == "water_type" || key == "w_type") ok = need_int(w_t);
            else if (key == "cl_type") ok = need_int(cl_t);
            else if (key == "target_pct" || key == "target_protonation_pct") ok = need_real(target_pct);
            else if (key == "rng_seed") ok = need_int(seed);
            else if (key == "energy_interval") ok = need_int(energy_interval);
            else if (key == "patience") ok = need_int(patience);
            else if (key == "max_attempts") ok = need_int(max_attempts);
            else if (key == "beta") ok = need_real(beta);
            else if (key == "w_z_extra_nm") ok = need_real(w_z_extra);
            else if (key == "direct_pct_threshold" || key == "direct_protonation_pct_threshold") ok = need_int(direct_pct);
            else if (key == "mu_eta") ok = need_real(mu_eta);
            else if (key == "gc_block_fixed") ok = need_int(gc_block);
            else if (key == "sgmc_epoch_attempt_max" || key == "epoch_attempt_max") ok = need_int(epoch_max);
            else if (key == "sgmc_nacc_frac_round" || key == "nacc_frac_round") ok = need_real(nacc_round);
            else if (key == "phase2_wc" || key == "phase2_WC") {
                const std::string lv = lower(val);
                if (lv == "1" || lv == "true" || lv == "yes" || lv == "on") phase2_wc = 1;
                else if (lv == "0" || lv == "false" || lv == "no" || lv == "off") phase2_wc = 0;
                else return bad("invalid boolean: " + val);
            } else {
                // the native model's keys (not read by the reference, which ignores unknown keys)
                int k = -1;
                for (int j = 0; j < 11; ++j) if (lk == nat_keys[j]) k = j;
                if (k >= 0) {
                    char* end = nullptr;
                    nat[k] = std::strtod(v, &end);
                    if (end == v) return bad("not a number: " + key + " = " + val);
                } else if (lk == "pme_mesh") {
                    Tokens t(vl);
                    if (t.n != 3 || !to_int(t.buf[0], mesh[0]) || !to_int(t.buf[1], mesh[1]) || !to_int(t.buf[2], mesh[2]))
                        return bad("pme_mesh takes three integers: " + val);
                } else {
                    if (!unk.empty()) unk += ",";
                    unk += key;
                }
            }
            if (!ok) return bad("bad value for " + key + ": " + val);
        } else if (l.starts_with("lj ")) {
            Tokens t(l);
            int ti = 0, tj = 0;
            float e = 0.0f, s = 0.0f;
            if (t.n < 5 || !to_int(t.buf[1], ti) || !to_int(t.buf[2], tj) || !to_float(t.buf[3], e) || !to_float(t.buf[4], s))
                return bad("bad lj line: " + l.str());
            if (ti < 1 || tj < 1 || ti > ntypes || tj > ntypes) return bad("LJ type index out of bounds");
            const size_t I = (size_t)(ti - 1) * ntypes + (tj - 1), J = (size_t)(tj - 1) * ntypes + (ti - 1);
            eps[I] = eps[J] = e;
            sig[I] = sig[J] = s;
        } else {
            if (!unk.empty()) unk += ",";
            unk += l.str();
        }
    }
    if (strict && !unk.empty()) return bad("unknown entries: " + unk);
    if (rc <= 0.0f) return bad("cutoff_nm must be > 0 in params");
    if (pme_spacing <= 0.0f) pme_spacing = 0.12f;
    if (pme_order <= 0) pme_order = 4;
    if (coulomb == PHMC_COUL_EWALD) {
        if (ewald_alpha <= 0.0f) ewald_alpha = (float)ewald_alpha_from_rtol((double)rc, (double)ewald_rtol);
    } else {
        ewald_alpha = 0.0f;
    }
    for (size_t k = 0; k < eps.size(); ++k) {
        lj_eps[k] = eps[k];
        lj_sig[k] = sig[k];
        float sh = 0.0f;
        if (lj_shift && eps[k] > 0.0f && sig[k] > 0.0f) {  // LJ at rc in FP32, as the reference tabulates it
            const float sr = sig[k] / rc, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
            sh = 4.0f * eps[k] * (sr12 - sr6);
        }
        lj_shift_tbl[k] = sh;
    }
    if (direct_pct < 10 || direct_pct > 100) return bad("direct_pct_threshold must be between 10 and 100");
    if (gc_block <= 0) gc_block = 2000;
    if (epoch_max <= 0) epoch_max = 100000;
    if (nacc_round <= 0.0f) nacc_round = 0.10f;
    if (mu_eta <= 0.0f) mu_eta = 0.3f;
    const int tcheck[4] = {nh_n, nh_p, w_t, cl_t};
    const char* tname[4] = {"nh_n_type", "nh_p_type", "w_type", "cl_type"};
    for (int k = 0; k < 4; ++k)
        if (tcheck[k] < 1 || tcheck[k] > ntypes)
            return bad(std::string(tname[k]) + " (" + std::to_string(tcheck[k]) + ") must be between 1 and " + std::to_string(ntypes));
    p->rc = rc; p->epsilon_r = epsilon_r; p->ewald_rtol = ewald_rtol; p->ewald_alpha = ewald_alpha;
    p->pme_spacing = pme_spacing; p->pme_3dc_zfac = zfac; p->beta = beta; p->target_pct = target_pct;
    p->w_z_extra_nm = w_z_extra; p->mu_eta = mu_eta; p->nacc_frac_round = nacc_round;
    p->lj_shift = lj_shift; p->coulomb = coulomb; p->pme_order = pme_order; p->pme_3dc = pme_3dc;
    p->nh_n_type = nh_n; p->nh_p_type = nh_p; p->w_type = w_t; p->cl_type = cl_t; p->rng_seed = seed;
    p->energy_interval = energy_interval; p->patience = patience; p->max_attempts = max_attempts;
    p->direct_pct_threshold = direct_pct; p->gc_block_fixed = gc_block; p->epoch_attempt_max = epoch_max; p->phase2_wc = phase2_wc;
    p->pH = nat[0]; p->pKa = nat[1]; p->salt_conc = nat[2]; p->wall_lo = nat[3]; p->wall_hi = nat[4];
    p->fene_k = nat[5]; p->fene_r0 = nat[6]; p->p_disp = nat[7]; p->p_titr = nat[8]; p->p_swap = nat[9]; p->disp_max = nat[10];
    for (int k = 0; k < 3; ++k) p->mesh[k] = mesh[k];
    if (unknown && unknown_len > 0) {
        std::strncpy(unknown, unk.c_str(), (size_t)unknown_len - 1);
        unknown[unknown_len - 1] = 0;
    }
    return PHMC_OK;
}
