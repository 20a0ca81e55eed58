// Synthetic grafted-brush systems (no counterpart in the reference, whose
// inputs are LAMMPS data files): chains grown as self-avoiding random walks
// from a square grafting lattice at z = 0, initial ionisation drawn at random,
// one counterion per positive charge and salt pairs placed uniformly in the
// slab, all without overlaps closer than min_dist.  Deterministic per seed
// (xoshiro256**, Blackman & Vigna 2018, seeded through splitmix64).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <string>

void phmc_set_error(int code, const std::string& msg);  // engine.cu

static int gen_fail(int code, const char* msg) {
    phmc_set_error(code, msg);
    return code;
}
#include "../../include/phmc.h"

namespace {
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (int i = 0; i < 4; ++i) {
            z += 0x9e3779b97f4a7c15ull;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
            s[i] = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    int below(int n) { return (int)(uni() * n); }
};

struct Grid {
    double L[3], cs;
    int n[3];
    std::vector<std::vector<int>> cells;
    std::vector<double> px, py, pz;
    Grid(double lx, double ly, double lz, double c) : cs(c) {
        L[0] = lx; L[1] = ly; L[2] = lz;
        for (int k = 0; k < 3; ++k) n[k] = std::max(1, (int)(L[k] / c));
        cells.resize((size_t)n[0] * n[1] * n[2]);
    }
    int idx(double x, double y, double z) const {
        int a = std::min(n[0] - 1, std::max(0, (int)(x / L[0] * n[0])));
        int b = std::min(n[1] - 1, std::max(0, (int)(y / L[1] * n[1])));
        int c = std::min(n[2] - 1, std::max(0, (int)(z / L[2] * n[2])));
        return (c * n[1] + b) * n[0] + a;
    }
    bool free_at(double x, double y, double z, double dmin, int skip) const {
        int a = std::min(n[0] - 1, std::max(0, (int)(x / L[0] * n[0])));
        int b = std::min(n[1] - 1, std::max(0, (int)(y / L[1] * n[1])));
        int c = std::min(n[2] - 1, std::max(0, (int)(z / L[2] * n[2])));
        const int span = (int)std::ceil(dmin / cs);
        for (int dz = -span; dz <= span; ++dz) {
            int cz = c + dz;
            if (cz < 0 || cz >= n[2]) continue;
            for (int dy = -span; dy <= span; ++dy)
                for (int dx = -span; dx <= span; ++dx) {
                    int cy = ((b + dy) % n[1] + n[1]) % n[1], cx = ((a + dx) % n[0] + n[0]) % n[0];
                    for (int j : cells[((size_t)cz * n[1] + cy) * n[0] + cx]) {
                        if (j == skip) continue;
                        double ex = x - px[j], ey = y - py[j], ez = z - pz[j];
                        ex -= L[0] * std::nearbyint(ex / L[0]);
                        ey -= L[1] * std::nearbyint(ey / L[1]);
                        if (ex * ex + ey * ey + ez * ez < dmin * dmin) return false;
                    }
                }
        }
        return true;
    }
    void add(double x, double y, double z) {
        int id = (int)px.size();
        px.push_back(x); py.push_back(y); pz.push_back(z);
        cells[idx(x, y, z)].push_back(id);
    }
    // remove the most recently added point (it is the last entry of its cell)
    void pop() {
        const int id = (int)px.size() - 1;
        cells[idx(px[id], py[id], pz[id])].pop_back();
        px.pop_back(); py.pop_back(); pz.pop_back();
    }
};
}  // namespace

extern "C" int phmc_build_brush(const phmc_brush_spec* sp, int capacity, float* x, float* y, float* z, float* q, int* type,
                                int* flags, int max_bonds, int* bond_i, int* bond_j, int* counts, double* box_out) {
    if (!sp || !x || !y || !z || !q || !type || !flags || !counts || !box_out) return gen_fail(PHMC_ERR_ARG, "phmc_build_brush: null argument");
    Rng rng(sp->seed);
    const double a = sp->graft_spacing;
    const double Lx = sp->chains_x * a, Ly = sp->chains_y * a, H = sp->height;
    box_out[0] = Lx; box_out[1] = Ly; box_out[2] = sp->lz;
    const double b = sp->bond_len, dmin = sp->min_dist;
    Grid g(Lx, Ly, H, 1.0);
    std::vector<int> ptype, pflag;
    std::vector<float> pq;
    std::vector<int> bi, bj;
    int n_pos = 0;
    const int nch = sp->chains_x * sp->chains_y;
    for (int c = 0; c < nch; ++c) {
        const int len = sp->len_min + (sp->len_max > sp->len_min ? rng.below(sp->len_max - sp->len_min + 1) : 0);
        // grow the chain's coordinates; a walk that traps itself is discarded and regrown
        const int first = (int)g.px.size();
        bool grown = false;
        for (int attempt = 0; attempt < 50 && !grown; ++attempt) {
            double cx = ((c % sp->chains_x) + 0.5) * a, cy = ((c / sp->chains_x) + 0.5) * a, cz = 0.0;
            int prev = -1;
            grown = true;
            for (int k = 0; k < len && grown; ++k) {
                if (k > 0) {
                    bool ok = false;
                    // dense grafting (>= 0.08 sigma^-2) starts from stretched chains: steps
                    // point away from the plane; regrowth of a trapped chain stretches more
                    const double dense = 1.0 / (a * a) >= 0.08 ? 1.0 : 0.0;
                    const double umin = attempt < 2 ? (dense > 0 ? 0.0 : -1.0) : (attempt < 10 ? 0.0 : 0.3);
                    for (int tries = 0; tries < 2000 && !ok; ++tries) {
                        const double dm = tries < 1000 ? dmin : 0.8 * dmin;
                        const double u = umin + (1.0 - umin) * rng.uni(), ph = 2.0 * M_PI * rng.uni();
                        const double s = std::sqrt(std::max(0.0, 1.0 - u * u));
                        double nx = cx + b * s * std::cos(ph), ny = cy + b * s * std::sin(ph), nz = cz + b * u;
                        if (nz < 0.0 || nz >= H) continue;
                        nx -= Lx * std::floor(nx / Lx);
                        ny -= Ly * std::floor(ny / Ly);
                        if (nx >= Lx) nx = 0.0;
                        if (ny >= Ly) ny = 0.0;
                        if (!g.free_at(nx, ny, nz, dm, prev)) continue;
                        cx = nx; cy = ny; cz = nz; ok = true;
                    }
                    if (!ok) { grown = false; break; }
                }
                prev = (int)g.px.size();
                g.add(cx, cy, cz);
            }
            if (!grown) while ((int)g.px.size() > first) g.pop();
        }
        if (!grown) return gen_fail(PHMC_ERR_CAPACITY, "phmc_build_brush: a chain could not be grown without overlaps (grafting too dense)");
        int prev = -1;
        for (int k = 0; k < len; ++k) {
            const int id = first + k;
            const bool perm = k < sp->n_permanent;
            const bool titr = !perm && (k > 0 || sp->graft_titratable);
            int t, f = (k == 0) ? 0 : PHMC_F_MOBILE;
            float qq;
            if (perm) { t = 4; qq = 1.0f; }
            else if (titr) {
                const bool ion = rng.uni() < sp->ion_frac;
                t = ion ? 1 : 0; qq = ion ? 1.0f : 0.0f; f |= PHMC_F_TITRATABLE;
            } else { t = 0; qq = 0.0f; }
            ptype.push_back(t); pflag.push_back(f); pq.push_back(qq);
            if (qq > 0) ++n_pos;
            if (prev >= 0) { bi.push_back(prev); bj.push_back(id); }
            prev = id;
        }
    }
    auto place = [&](int t, float qq, int f) -> bool {
        for (int tries = 0; tries < 100000; ++tries) {
            const double px = Lx * rng.uni(), py = Ly * rng.uni(), pz = H * rng.uni();
            if (!g.free_at(px, py, pz, dmin, -1)) continue;
            g.add(px, py, pz);
            ptype.push_back(t); pflag.push_back(f); pq.push_back(qq);
            return true;
        }
        return false;
    };
    for (int k = 0; k < n_pos; ++k)
        if (!place(2, -1.0f, PHMC_F_MOBILE | PHMC_F_ANION)) return gen_fail(PHMC_ERR_CAPACITY, "phmc_build_brush: no free spot for an ion (slab too dense)");
    const int n_salt = (int)std::lround(sp->salt_conc * Lx * Ly * H);
    for (int k = 0; k < n_salt; ++k) {
        if (!place(3, 1.0f, PHMC_F_MOBILE | PHMC_F_CATION)) return gen_fail(PHMC_ERR_CAPACITY, "phmc_build_brush: no free spot for an ion (slab too dense)");
        if (!place(2, -1.0f, PHMC_F_MOBILE | PHMC_F_ANION)) return gen_fail(PHMC_ERR_CAPACITY, "phmc_build_brush: no free spot for an ion (slab too dense)");
    }
    const int n = (int)g.px.size();
    counts[0] = n; counts[1] = (int)bi.size();
    if (n > capacity || (int)bi.size() > max_bonds) return gen_fail(PHMC_ERR_CAPACITY, "phmc_build_brush: output arrays too small");
    for (int i = 0; i < n; ++i) {
        x[i] = (float)g.px[i]; y[i] = (float)g.py[i]; z[i] = (float)g.pz[i];
        if (x[i] >= (float)Lx) x[i] = 0.0f;
        if (y[i] >= (float)Ly) y[i] = 0.0f;
        q[i] = pq[i]; type[i] = ptype[i]; flags[i] = pflag[i];
    }
    for (size_t k = 0; k < bi.size(); ++k) { bond_i[k] = bi[k]; bond_j[k] = bj[k]; }
    return PHMC_OK;
}
