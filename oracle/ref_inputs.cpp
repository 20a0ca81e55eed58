// ORACLE SIDE — input files for runs of the reference's own build.
//
// Writes the benchmark's synthetic brush systems in the reference's input
// format (LAMMPS "full" data file read by MC/src/io.cpp:79-146, params.in read
// by MC/src/io.cpp:171-301) so that the reference arm of the benchmark and
// the reference harness (ref_harness.cu) get the very systems the engine
// runs, without loading the engine's library.  The chains, ions and salt come
// from the engine's generator source (ph_brush_b200/csrc/brush_gen.cpp,
// compiled into this program), so a spec line gives the same particles as
// ph_brush_b200.configs; the reference's model then needs an identity pool of
// neutral W beads (one per titratable site, uniform in the slab) for its
// protonation moves, as ph_brush_b200.configs.to_reference_semantics builds.
//
//   ref_inputs <spec file> <out dir>
//
// Spec file: one replica per line, whitespace separated:
//   name chains_x chains_y graft_spacing len_min len_max n_permanent graft_titratable
//   height lz ion_frac salt_conc bond_len min_dist seed n_w w_seed pme_spacing pH pKa
// Outputs per replica: <name>.data, <name>.params and <name>.extra (the native
// particle count, slab height, pH, pKa and the mobile atoms, for the harness's
// displacement trials); one line "name natoms n_native n_sites" per replica on
// stdout.  Reference types (1-based): 3 permanent +1, 4 NH_N, 5 NH_P, 6 Na,
// 7 W, 8 Cl.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "../include/phmc.h"

void phmc_set_error(int, const std::string& msg) { fprintf(stderr, "ref_inputs: %s\n", msg.c_str()); }

namespace {
// xoshiro256** seeded through splitmix64 (Blackman & Vigna 2018): the W-bead positions
struct Xo {
    uint64_t s[4];
    explicit Xo(uint64_t seed) {
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
    double uni() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return (double)(r >> 11) * (1.0 / 9007199254740992.0);
    }
};

const int NATIVE_TO_REF[5] = {4, 5, 8, 6, 3};
const int REF_W = 7, REF_NTYPES = 8;
const double KE = 138.935458, L_BJERRUM = 1.4;

int write_replica(const std::string& line, const std::string& dir) {
    std::istringstream is(line);
    std::string name;
    phmc_brush_spec sp{};
    int n_w = 0;
    unsigned long long seed = 0, w_seed = 0;
    double pme_spacing = 0.75, pH = 7.0, pKa = 7.0;
    is >> name >> sp.chains_x >> sp.chains_y >> sp.graft_spacing >> sp.len_min >> sp.len_max >> sp.n_permanent >>
        sp.graft_titratable >> sp.height >> sp.lz >> sp.ion_frac >> sp.salt_conc >> sp.bond_len >> sp.min_dist >> seed >>
        n_w >> w_seed >> pme_spacing >> pH >> pKa;
    if (!is) { fprintf(stderr, "ref_inputs: bad spec line: %s\n", line.c_str()); return 1; }
    sp.seed = seed;
    const int nch = sp.chains_x * sp.chains_y;
    const double est_salt = sp.salt_conc * nch * sp.graft_spacing * sp.graft_spacing * sp.height * 1.1 + 16;
    const int cap = nch * sp.len_max * 2 + 2 * (int)est_salt + 64;
    std::vector<float> x(cap), y(cap), z(cap), q(cap);
    std::vector<int> t(cap), f(cap), bi(nch * sp.len_max), bj(nch * sp.len_max);
    int counts[2] = {0, 0};
    double box[3];
    if (phmc_build_brush(&sp, cap, x.data(), y.data(), z.data(), q.data(), t.data(), f.data(), (int)bi.size(), bi.data(),
                         bj.data(), counts, box) != PHMC_OK)
        return 1;
    const int n = counts[0], nb = counts[1];
    int n_sites = 0, n_charged = 0;
    for (int i = 0; i < n; ++i)
        if (f[i] & PHMC_F_TITRATABLE) { ++n_sites; n_charged += q[i] != 0.0f ? 1 : 0; }
    if (n_w < 0) n_w = n_sites;
    Xo rng(w_seed);
    std::vector<float> wx(n_w), wy(n_w), wz(n_w);
    for (int k = 0; k < n_w; ++k) {  // x, y, z of each bead in turn
        wx[k] = (float)(box[0] * rng.uni());
        wy[k] = (float)(box[1] * rng.uni());
        wz[k] = (float)(sp.height * rng.uni());
        if (wx[k] >= (float)box[0]) wx[k] = 0.0f;
        if (wy[k] >= (float)box[1]) wy[k] = 0.0f;
    }
    const int N = n + n_w;
    const double zfac = sp.lz / sp.height;
    const std::string base = dir + "/" + name;
    FILE* fh = fopen((base + ".data").c_str(), "w");
    if (!fh) { fprintf(stderr, "ref_inputs: cannot write %s.data\n", base.c_str()); return 1; }
    fprintf(fh, "# synthetic brush\n\n%d atoms\n%d bonds\n\n%d atom types\n1 bond types\n\n", N, nb, REF_NTYPES);
    fprintf(fh, "0.0 %.10f xlo xhi\n0.0 %.10f ylo yhi\n0.0 %.10f zlo zhi\n\nAtoms # full\n\n", box[0], box[1], box[2] / zfac);
    for (int i = 0; i < N; ++i) {
        const bool w = i >= n;
        const int rt = w ? REF_W : NATIVE_TO_REF[t[i]];
        const float qq = w ? 0.0f : q[i];
        fprintf(fh, "%d %d %d %.1f %.9g %.9g %.9g\n", i + 1, 1 + i / 1000, rt, (double)qq, (double)(w ? wx[i - n] : x[i]),
                (double)(w ? wy[i - n] : y[i]), (double)(w ? wz[i - n] : z[i]));
    }
    if (nb > 0) {
        fprintf(fh, "\nBonds\n\n");
        for (int k = 0; k < nb; ++k) fprintf(fh, "%d 1 %d %d\n", k + 1, bi[k] + 1, bj[k] + 1);
    }
    fclose(fh);
    // params.in in the reference's key = value format; alpha from its own rule (erfcinv(rtol) / cutoff)
    fh = fopen((base + ".params").c_str(), "w");
    if (!fh) { fprintf(stderr, "ref_inputs: cannot write %s.params\n", base.c_str()); return 1; }
    fprintf(fh, "cutoff_nm = 3\nlj_shift = yes\nepsilon_r = %.10g\ncoulombtype = pme\newald_rtol = 1e-5\n", KE / L_BJERRUM);
    fprintf(fh, "pme_spacing = %.10g\npme_order = 4\npme_3dc = yes %.10g\nbeta = 1.0\n", pme_spacing, zfac);
    fprintf(fh, "nh_n_type = 4\nnh_p_type = 5\nw_type = 7\ncl_type = 8\n");
    // target = the current protonation (floor(pct / 100 sites) == charged sites): the reference's
    // build_plan refuses a target below the current count (MC/src/mc.cu:88-91)
    fprintf(fh, "target_protonation_pct = %.10f\n", n_sites > 0 ? 100.0 * (n_charged + 0.5) / n_sites : 10.0);
    for (int i = 1; i <= REF_NTYPES; ++i)
        for (int j = i; j <= REF_NTYPES; ++j) fprintf(fh, "lj %d %d %d 1\n", i, j, (i == REF_W || j == REF_W) ? 0 : 1);
    fclose(fh);
    fh = fopen((base + ".extra").c_str(), "w");
    if (!fh) { fprintf(stderr, "ref_inputs: cannot write %s.extra\n", base.c_str()); return 1; }
    int n_mob = 0;
    for (int i = 0; i < n; ++i) n_mob += (f[i] & PHMC_F_MOBILE) ? 1 : 0;
    fprintf(fh, "n_native %d\nn_sites %d\nheight %.17g\npH %.17g\npKa %.17g\nmobile %d\n", n, n_sites, sp.height, pH, pKa, n_mob);
    for (int i = 0; i < n; ++i)
        if (f[i] & PHMC_F_MOBILE) fprintf(fh, "%d\n", i);
    fclose(fh);
    printf("%s %d %d %d\n", name.c_str(), N, n, n_sites);
    return 0;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s <spec file> <out dir>\n", argv[0]); return 1; }
    std::ifstream in(argv[1]);
    if (!in) { fprintf(stderr, "ref_inputs: cannot read %s\n", argv[1]); return 1; }
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        if (write_replica(line, argv[2])) return 2;
    }
    return 0;
}
