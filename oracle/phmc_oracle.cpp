// ORACLE — test infrastructure only.  Nothing in the product (ph_brush_b200/,
// include/) links, loads or calls this file; only tests/, the smoke check and
// bench.py's CPU-baseline leg do, and only as the checker / timed CPU baseline.
//
// FP64 CPU restatement of the ph_brush energy path (reference files cited per
// function, paths relative to the reference project root) plus the native
// model the engine adds (WCA/FENE/walls, order-p SPME, constant-pH moves) and
// an FP64 direct-Ewald sum with the Yeh-Berkowitz slab term.
//
// Parity status: the reference ships no golden vectors or tests; this oracle is
// pinned by (a) known-answer tests (Madelung constant, LJ minimum, FENE closed
// form, B-spline moduli vs a direct DFT), (b) the reference's own host code
// compiled from its sources (oracle/Makefile, target `ref-host`) and (c)
// energies printed by the reference's own CUDA routines on a B200, committed as
// fixtures under tests/golden/.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <random>
#include <sstream>
#include <stdexcept>
#include "../include/phmc.h"

typedef std::complex<double> cplx;
static const double PI = 3.14159265358979323846;
static const double KE = 138.935458;  // MC/src/pme.cu:305, MC/src/energy_gpu.cu:78

// ---------------------------------------------------------------------------
// FP64 mixed-radix FFT (forward sign -1), any length, recursive Cooley-Tukey
// for the smallest prime factor, direct DFT for prime lengths.
// ---------------------------------------------------------------------------
static void fft_rec(cplx* a, int n, int stride, cplx* out, int sign) {
    if (n == 1) { out[0] = a[0]; return; }
    int r = 0;
    for (int f : {2, 3, 5, 7}) if (n % f == 0) { r = f; break; }
    if (r == 0) {  // prime (or large prime factor): direct DFT
        for (int k = 0; k < n; ++k) {
            cplx s = 0;
            for (int j = 0; j < n; ++j) s += a[(size_t)j * stride] * std::polar(1.0, sign * 2.0 * PI * (double)((long long)j * k % n) / n);
            out[k] = s;
        }
        return;
    }
    int m = n / r;
    std::vector<cplx> sub((size_t)n);
    for (int q = 0; q < r; ++q) fft_rec(a + (size_t)q * stride, m, stride * r, sub.data() + (size_t)q * m, sign);
    for (int k = 0; k < m; ++k) {
        for (int s = 0; s < r; ++s) {
            int kk = k + s * m;
            cplx acc = 0;
            for (int q = 0; q < r; ++q) {
                cplx tw = std::polar(1.0, sign * 2.0 * PI * (double)((long long)q * kk % n) / n);
                acc += tw * sub[(size_t)q * m + k];
            }
            out[kk] = acc;
        }
    }
}

static void fft1d(cplx* line, int n, int sign) {
    std::vector<cplx> tmp(line, line + n), out((size_t)n);
    fft_rec(tmp.data(), n, 1, out.data(), sign);
    std::copy(out.begin(), out.end(), line);
}

// 3-D FFT in place, layout ((z*ny)+y)*nx+x (x fastest, MC/src/pme.cu:159).
static void fft3d(std::vector<cplx>& g, int nx, int ny, int nz, int sign) {
    #pragma omp parallel for collapse(2)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) fft1d(&g[((size_t)z * ny + y) * nx], nx, sign);
    #pragma omp parallel
    {
        std::vector<cplx> line((size_t)std::max(ny, nz));
        #pragma omp for collapse(2)
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x) {
                for (int y = 0; y < ny; ++y) line[y] = g[((size_t)z * ny + y) * nx + x];
                fft1d(line.data(), ny, sign);
                for (int y = 0; y < ny; ++y) g[((size_t)z * ny + y) * nx + x] = line[y];
            }
        #pragma omp for collapse(2)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                for (int z = 0; z < nz; ++z) line[z] = g[((size_t)z * ny + y) * nx + x];
                fft1d(line.data(), nz, sign);
                for (int z = 0; z < nz; ++z) g[((size_t)z * ny + y) * nx + x] = line[z];
            }
    }
}

extern "C" void orc_fft3d(double* re, double* im, int nx, int ny, int nz, int sign) {
    size_t M = (size_t)nx * ny * nz;
    std::vector<cplx> g(M);
    for (size_t i = 0; i < M; ++i) g[i] = cplx(re[i], im[i]);
    fft3d(g, nx, ny, nz, sign);
    for (size_t i = 0; i < M; ++i) { re[i] = g[i].real(); im[i] = g[i].imag(); }
}

// ---------------------------------------------------------------------------
// Reference host helpers, restated.
// ---------------------------------------------------------------------------

// MC/src/pme.cu:46-51 — smallest 2/3/5-smooth m >= max(8, n), searched up to max(16, 2n+32).
extern "C" int orc_ref_good_fft_dim(int n) {
    const int NMAX = std::max(16, n * 2 + 32);
    for (int m = std::max(8, n); m <= NMAX; ++m) {
        int x = m;
        for (int p : {2, 3, 5}) while (x % p == 0) x /= p;
        if (x == 1) return m;
    }
    return n;
}

// MC/src/io.cpp:46-70 — Winitzki initial guess (a = 0.147) + 3 Newton steps on erf.
static double ref_erfinv_newton(double x) {
    if (x <= -1.0) return -std::numeric_limits<double>::infinity();
    if (x >= 1.0) return std::numeric_limits<double>::infinity();
    const double a = 0.147;
    double ln = std::log(1.0 - x * x);
    double t1 = 2.0 / (PI * a) + ln / 2.0;
    double t2 = ln / a;
    double v = std::sqrt(std::max(0.0, std::sqrt(t1 * t1 - t2) - t1));
    if (x < 0) v = -v;
    for (int i = 0; i < 3; ++i) {
        double err = std::erf(v) - x;
        double d = 2.0 / std::sqrt(PI) * std::exp(-v * v);
        v -= err / d;
    }
    return v;
}

// MC/src/io.cpp:65-77 — alpha = erfcinv(clamp(rtol, 1e-12, 0.5)) / rc  (rtol <= 0 -> 1e-5).
extern "C" double orc_ref_ewald_alpha(double rc, double rtol) {
    if (rtol <= 0.0) rtol = 1e-5;
    double c = std::min(std::max(rtol, 1e-12), 0.5);
    double y = c;
    double inv;
    if (y <= 0.0) inv = std::numeric_limits<double>::infinity();
    else if (y >= 2.0) inv = -std::numeric_limits<double>::infinity();
    else inv = ref_erfinv_newton(1.0 - y);
    return inv / rc;
}

// MC/src/pme.cu:54-63 — bisection fallback used by pmeCreate when ewald_alpha <= 0.
extern "C" double orc_ref_alpha_bisect(double rc, double rtol) {
    double b = 5.0; int i = 0;
    while (std::erfc(b * rc) > rtol) { b *= 2.0; if (++i > 60) break; }
    double lo = 0.0, hi = b;
    for (int it = 0; it < 60; ++it) {
        b = 0.5 * (lo + hi);
        if (std::erfc(b * rc) > rtol) lo = b; else hi = b;
    }
    return b;
}

// Cardinal B-spline M_p at the integer points 1..p-1 by the de Boor recursion
// (MC/src/pme.cu:81-90; order p -> splineOrder p-1 coefficients).
static std::vector<double> bspline_int_values(int order) {
    const int s = order - 1;
    std::vector<double> d((size_t)s, 0.0);
    d[0] = 1.0;
    for (int k = 2; k <= s; ++k) {
        const double inv = 1.0 / k;
        for (int m = k - 1; m > 0; --m) d[m] = inv * ((k - m) * d[m - 1] + (m + 1) * d[m]);
        d[0] = inv * d[0];
    }
    return d;
}

// |DFT(M_p)|^2 on a length-n grid.
//  ref_style = 1: exactly MC/src/pme.cu:92-112 (clamp exact zeros to 1e-30, Nyquist patch).
//  ref_style = 0: native engine — entries below 1e-7 are replaced by the mean of
//                 their two neighbours (zero moduli of odd orders at Nyquist).
extern "C" void orc_moduli(int n, int order, int ref_style, double* out) {
    std::vector<double> d = bspline_int_values(order);
    const int s = order - 1;
    for (int i = 0; i < n; ++i) {
        double sc = 0, ss = 0;
        for (int j = 0; j < s; ++j) {
            double arg = (2.0 * PI * i * (j + 1)) / double(n);
            sc += d[j] * std::cos(arg);
            ss += d[j] * std::sin(arg);
        }
        double v = sc * sc + ss * ss;
        if (ref_style && !(v > 0.0)) v = 1e-30;
        out[i] = v;
    }
    if (ref_style) {
        if (n % 2 == 0) { int h = n / 2; if (!(out[h] > 0.0)) out[h] = out[h - 1]; }
    } else {
        std::vector<double> c(out, out + n);
        for (int i = 0; i < n; ++i)
            if (c[i] < 1e-7) out[i] = 0.5 * (c[(i - 1 + n) % n] + c[(i + 1) % n]);
    }
}

// B-spline weights of order p for fractional offset t in [0,1).
// Native convention: the charge at grid coordinate g = ix + t is spread to the
// p points base + j, base = ix + p/2 - p + 1, with weight w[j] = M_p(t + p-1-j).
// For p = 4 this is exactly the reference's cubic rule (MC/src/pme.cu:132-138,160-170):
// points ix-1..ix+2.
extern "C" void orc_bspline_weights(int p, double t, double* w) {
    double c[16] = {0};
    c[0] = t; c[1] = 1.0 - t;  // M_2(t), M_2(t+1)
    for (int n = 3; n <= p; ++n) {
        double nc[16] = {0};
        for (int i = 0; i < n; ++i) {
            double a = (i < n - 1) ? c[i] : 0.0;
            double b = (i >= 1) ? c[i - 1] : 0.0;
            nc[i] = ((t + i) * a + (n - t - i) * b) / (n - 1);
        }
        std::memcpy(c, nc, sizeof(c));
    }
    for (int j = 0; j < p; ++j) w[j] = c[p - 1 - j];
}

static inline int stencil_base(int ix, int p) { return ix + p / 2 - p + 1; }

// MC/src/io.cpp:148-169 — symmetric, sorted, de-duplicated 1-2 adjacency CSR.
extern "C" void orc_ref_bond_csr(int N, int nb, const int* bi, const int* bj, int* head, int* list) {
    std::vector<std::vector<int>> t((size_t)N);
    for (int k = 0; k < nb; ++k) { t[bi[k]].push_back(bj[k]); t[bj[k]].push_back(bi[k]); }
    head[0] = 0;
    for (int i = 0; i < N; ++i) {
        std::sort(t[i].begin(), t[i].end());
        t[i].erase(std::unique(t[i].begin(), t[i].end()), t[i].end());
        head[i + 1] = head[i] + (int)t[i].size();
    }
    for (int i = 0; i < N; ++i) std::copy(t[i].begin(), t[i].end(), list + head[i]);
}

static inline double min_image(double d, double L) { return d - L * std::nearbyint(d / L); }

static bool csr_has(const int* head, const int* list, int i, int j) {
    // MC/src/neighbor.cu:17-19 — binary search in the sorted 1-2 row of i.
    int lo = head[i], hi = head[i + 1] - 1;
    while (lo <= hi) { int mid = (lo + hi) >> 1; int v = list[mid]; if (v == j) return true; if (v < j) lo = mid + 1; else hi = mid - 1; }
    return false;
}

// MC/src/neighbor.cu:21-63 — half list i<j, r^2 <= rc^2 (min image, all axes),
// 1-2 pairs excluded.  Returns nnz; fills head[N+1] and list[] when list_cap >= nnz.
extern "C" int orc_ref_half_list(int N, const double* x, const double* y, const double* z,
                                 const double* box, double rc, const int* bhead, const int* blist,
                                 int* head, int* list, int list_cap) {
    std::vector<std::vector<int>> rows((size_t)N);
    const double rc2 = rc * rc;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
            if (bhead && csr_has(bhead, blist, i, j)) continue;
            double dx = min_image(x[i] - x[j], box[0]);
            double dy = min_image(y[i] - y[j], box[1]);
            double dz = min_image(z[i] - z[j], box[2]);
            if (dx * dx + dy * dy + dz * dz <= rc2) rows[i].push_back(j);
        }
    int nnz = 0;
    head[0] = 0;
    for (int i = 0; i < N; ++i) { nnz += (int)rows[i].size(); head[i + 1] = nnz; }
    if (list && list_cap >= nnz)
        for (int i = 0; i < N; ++i) std::copy(rows[i].begin(), rows[i].end(), list + head[i]);
    return nnz;
}

// MC/src/io.cpp:270-281 — LJ value at rc per type pair (0 where eps<=0 or sig<=0).
extern "C" void orc_ref_lj_shift(int T, const double* eps, const double* sig, double rc, double* out) {
    for (int k = 0; k < T * T; ++k) {
        out[k] = 0.0;
        if (eps[k] > 0.0 && sig[k] > 0.0) {
            double sr = sig[k] / rc, sr6 = std::pow(sr, 6);
            out[k] = 4.0 * eps[k] * (sr6 * sr6 - sr6);
        }
    }
}

// MC/src/energy_gpu.cu:14-46 — LJ over the half list, optional shift table.
extern "C" double orc_ref_lj(int N, const double* x, const double* y, const double* z, const int* type,
                             const int* head, const int* list, int T, const double* box,
                             const double* eps, const double* sig, const double* shift, int use_shift) {
    double E = 0.0;
    #pragma omp parallel for reduction(+ : E) schedule(dynamic, 64)
    for (int i = 0; i < N; ++i)
        for (int k = head[i]; k < head[i + 1]; ++k) {
            int j = list[k];
            double dx = min_image(x[i] - x[j], box[0]), dy = min_image(y[i] - y[j], box[1]), dz = min_image(z[i] - z[j], box[2]);
            double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            int p = type[i] * T + type[j];
            if (eps[p] <= 0.0 || sig[p] <= 0.0) continue;
            double sr6 = std::pow(sig[p] / r, 6);
            double e = 4.0 * eps[p] * (sr6 * sr6 - sr6);
            if (use_shift) e -= shift[p];
            E += e;
        }
    return E;
}

// MC/src/energy_gpu.cu:80-108 — plain cutoff Coulomb over the half list.
extern "C" double orc_ref_coul_cut(int N, const double* x, const double* y, const double* z, const double* q,
                                   const int* head, const int* list, const double* box, double epsilon_r) {
    const double elf = KE / epsilon_r;
    double E = 0.0;
    #pragma omp parallel for reduction(+ : E) schedule(dynamic, 64)
    for (int i = 0; i < N; ++i)
        for (int k = head[i]; k < head[i + 1]; ++k) {
            int j = list[k];
            double qq = q[i] * q[j];
            if (qq == 0.0) continue;
            double dx = min_image(x[i] - x[j], box[0]), dy = min_image(y[i] - y[j], box[1]), dz = min_image(z[i] - z[j], box[2]);
            E += elf * qq / std::sqrt(dx * dx + dy * dy + dz * dz);
        }
    return E;
}

// Spread charges onto a real mesh with order-p weights (native convention; p=4
// is the reference's cubic rule, MC/src/pme.cu:140-172).
static void spread(int N, const double* x, const double* y, const double* z, const double* q,
                   const int* present, const double* box, int nx, int ny, int nz, int p,
                   std::vector<double>& Q) {
    Q.assign((size_t)nx * ny * nz, 0.0);
    for (int i = 0; i < N; ++i) {
        if (present && !present[i]) continue;
        if (q[i] == 0.0) continue;
        double g[3] = {x[i] / box[0] * nx, y[i] / box[1] * ny, z[i] / box[2] * nz};
        int n3[3] = {nx, ny, nz};
        int base[3];
        double w[3][16];
        for (int d = 0; d < 3; ++d) {
            int ix = (int)std::floor(g[d]);
            orc_bspline_weights(p, g[d] - ix, w[d]);
            base[d] = stencil_base(ix, p);
        }
        for (int a = 0; a < p; ++a) {
            int xa = ((base[0] + a) % n3[0] + n3[0]) % n3[0];
            for (int b = 0; b < p; ++b) {
                int yb = ((base[1] + b) % n3[1] + n3[1]) % n3[1];
                for (int c = 0; c < p; ++c) {
                    int zc = ((base[2] + c) % n3[2] + n3[2]) % n3[2];
                    Q[((size_t)zc * ny + yb) * nx + xa] += q[i] * w[0][a] * w[1][b] * w[2][c];
                }
            }
        }
    }
}

// Reciprocal SPME energy 0.5 * sum_k theta(k) |F(k)|^2 (MC/src/pme.cu:175-249, 422).
//  ref_corner = 1: half spectrum kx in [0, nx/2] with weight 1/2 at kx==0 and kx==nx/2
//                  (exactly the reference, also for odd nx); 0: full-spectrum sum.
static double recip_energy(const std::vector<double>& Q, int nx, int ny, int nz, const double* box,
                           double alpha, double elf, const double* mx_, const double* my_, const double* mz_,
                           int ref_corner) {
    std::vector<cplx> g(Q.size());
    for (size_t i = 0; i < Q.size(); ++i) g[i] = Q[i];
    fft3d(g, nx, ny, nz, -1);
    const double V = box[0] * box[1] * box[2];
    const double ef = (PI / alpha) * (PI / alpha);
    double E = 0.0;
    #pragma omp parallel for reduction(+ : E) collapse(2)
    for (int kz = 0; kz < nz; ++kz)
        for (int ky = 0; ky < ny; ++ky) {
            int my = (ky <= ny / 2) ? ky : ky - ny;
            int mz = (kz <= nz / 2) ? kz : kz - nz;
            int kx_end = ref_corner ? nx / 2 : nx - 1;
            for (int kx = 0; kx <= kx_end; ++kx) {
                if (kx == 0 && ky == 0 && kz == 0) continue;
                int mx = ref_corner ? kx : ((kx <= nx / 2) ? kx : kx - nx);
                double kxv = mx / box[0], kyv = my / box[1], kzv = mz / box[2];
                double m2 = kxv * kxv + kyv * kyv + kzv * kzv;
                if (m2 == 0.0) continue;
                double den = m2 * PI * V * mx_[kx] * my_[ky] * mz_[kz];
                if (!(den > 0.0)) continue;
                double et = elf * std::exp(-ef * m2) / den;
                double s2 = std::norm(g[((size_t)kz * ny + ky) * nx + kx]);
                double wgt = 1.0;
                if (ref_corner) wgt = (kx == 0 || kx == nx / 2) ? 1.0 : 2.0;
                E += wgt * et * s2;
            }
        }
    return 0.5 * E;
}

static void charge_moments(int N, const double* z, const double* q, const int* present,
                           double* Q, double* Q2, double* Mz, double* Sqz2) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int i = 0; i < N; ++i) {
        if (present && !present[i]) continue;
        a += q[i]; b += q[i] * q[i]; c += q[i] * z[i]; d += q[i] * z[i] * z[i];
    }
    *Q = a; *Q2 = b; *Mz = c; *Sqz2 = d;
}

// MC/src/pme.cu:425-447 — self, net-charge and slab terms.
static void ewald_corrections(double Q, double Q2, double Mz, double Sqz2, const double* box,
                              double alpha, double elf, int slab, double* self, double* qcorr, double* eslab) {
    const double V = box[0] * box[1] * box[2];
    *self = -elf * alpha / std::sqrt(PI) * Q2;
    *qcorr = -(PI * elf) * (Q * Q) / (2.0 * V * alpha * alpha);
    *eslab = 0.0;
    if (slab) {
        const double dc = (2.0 * PI / V) * elf;
        *eslab = dc * Mz * Mz;
        if (std::fabs(Q) > 1e-4) *eslab -= dc * Q * (Sqz2 + Q * box[2] * box[2] / 12.0);
    }
}

// MC/src/pme.cu:344-457 — pmeEnergy: out = {real, recip, self, qcorr+slab}; returns the sum.
// The real-space part uses the caller's half list (1-2 pairs already excluded);
// spreading is the reference's cubic rule whatever `order` is (only the moduli
// use `order`, MC/src/pme.cu:321-323 vs :140-172).
extern "C" double orc_ref_pme(int N, const double* x, const double* y, const double* z, const double* q,
                              const int* head, const int* list, const double* box, double alpha,
                              double epsilon_r, int nx, int ny, int nz, int order, int use3dc, double* out) {
    const double elf = KE / epsilon_r;
    double Er = 0.0;
    #pragma omp parallel for reduction(+ : Er) schedule(dynamic, 64)
    for (int i = 0; i < N; ++i)
        for (int k = head[i]; k < head[i + 1]; ++k) {
            int j = list[k];
            double qq = q[i] * q[j];
            if (qq == 0.0) continue;
            double dx = min_image(x[i] - x[j], box[0]), dy = min_image(y[i] - y[j], box[1]), dz = min_image(z[i] - z[j], box[2]);
            double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            Er += elf * qq * std::erfc(alpha * r) / r;
        }
    std::vector<double> Q;
    spread(N, x, y, z, q, nullptr, box, nx, ny, nz, 4, Q);
    std::vector<double> mx((size_t)nx), my((size_t)ny), mz((size_t)nz);
    orc_moduli(nx, order, 1, mx.data());
    orc_moduli(ny, order, 1, my.data());
    orc_moduli(nz, order, 1, mz.data());
    double Ek = recip_energy(Q, nx, ny, nz, box, alpha, elf, mx.data(), my.data(), mz.data(), 1);
    double Qt, Q2, Mz, S2, self, qc, sl;
    charge_moments(N, z, q, nullptr, &Qt, &Q2, &Mz, &S2);
    ewald_corrections(Qt, Q2, Mz, S2, box, alpha, elf, use3dc, &self, &qc, &sl);
    out[0] = Er; out[1] = Ek; out[2] = self; out[3] = qc + sl;
    return Er + Ek + self + qc + sl;
}

// ---------------------------------------------------------------------------
// FP64 direct Ewald (all images) + net-charge + Yeh-Berkowitz slab term.
// Independent of the SPME mesh: the converged total does not depend on alpha.
// out = {real, recip, self, qcorr, slab, total}.
// ---------------------------------------------------------------------------
extern "C" void orc_direct_ewald(int N, const double* x, const double* y, const double* z, const double* q,
                                 const double* box, double alpha, double epsilon_r, int slab, double tol,
                                 double* out) {
    const double elf = KE / epsilon_r;
    const double V = box[0] * box[1] * box[2];
    // real space: images until erfc(alpha r)/r < tol
    double rcut = 1.0;
    while (std::erfc(alpha * rcut) / rcut > tol) rcut *= 1.05;
    int nimg[3];
    for (int d = 0; d < 3; ++d) nimg[d] = (int)std::ceil(rcut / box[d]);
    double Er = 0.0;
    #pragma omp parallel for reduction(+ : Er) schedule(dynamic, 8)
    for (int i = 0; i < N; ++i) {
        if (q[i] == 0.0) continue;
        for (int j = 0; j < N; ++j) {
            if (q[j] == 0.0) continue;
            for (int a = -nimg[0]; a <= nimg[0]; ++a)
                for (int b = -nimg[1]; b <= nimg[1]; ++b)
                    for (int c = -nimg[2]; c <= nimg[2]; ++c) {
                        if (i == j && a == 0 && b == 0 && c == 0) continue;
                        double dx = x[i] - x[j] + a * box[0], dy = y[i] - y[j] + b * box[1], dz = z[i] - z[j] + c * box[2];
                        double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                        if (r > rcut) continue;
                        Er += 0.5 * elf * q[i] * q[j] * std::erfc(alpha * r) / r;
                    }
        }
    }
    // reciprocal: |k| up to where exp(-k^2/4a^2)/k^2 * (4pi/V) < tol
    double kmax = 2.0 * alpha;
    while (std::exp(-kmax * kmax / (4 * alpha * alpha)) / (kmax * kmax) > tol) kmax *= 1.05;
    int mmax[3];
    for (int d = 0; d < 3; ++d) mmax[d] = (int)std::ceil(kmax * box[d] / (2 * PI));
    double Ek = 0.0;
    #pragma omp parallel for reduction(+ : Ek) collapse(2) schedule(dynamic, 4)
    for (int a = -mmax[0]; a <= mmax[0]; ++a)
        for (int b = -mmax[1]; b <= mmax[1]; ++b)
            for (int c = -mmax[2]; c <= mmax[2]; ++c) {
                if (a == 0 && b == 0 && c == 0) continue;
                double kx = 2 * PI * a / box[0], ky = 2 * PI * b / box[1], kz = 2 * PI * c / box[2];
                double k2 = kx * kx + ky * ky + kz * kz;
                if (k2 > kmax * kmax) continue;
                double sr = 0, si = 0;
                for (int i = 0; i < N; ++i) {
                    if (q[i] == 0.0) continue;
                    double ph = kx * x[i] + ky * y[i] + kz * z[i];
                    sr += q[i] * std::cos(ph); si += q[i] * std::sin(ph);
                }
                Ek += (2 * PI / V) * elf * std::exp(-k2 / (4 * alpha * alpha)) / k2 * (sr * sr + si * si);
            }
    double Qt, Q2, Mz, S2, self, qc, sl;
    charge_moments(N, z, q, nullptr, &Qt, &Q2, &Mz, &S2);
    ewald_corrections(Qt, Q2, Mz, S2, box, alpha, elf, slab, &self, &qc, &sl);
    out[0] = Er; out[1] = Ek; out[2] = self; out[3] = qc; out[4] = sl;
    out[5] = Er + Ek + self + qc + sl;
}

// ---------------------------------------------------------------------------
// Native model energy from scratch (FP64).
// ---------------------------------------------------------------------------
struct Model {
    int T;
    std::vector<double> eps, sig, rc2, shift;
    double rc_coul, elf, alpha;
    int coulomb, nx, ny, nz, order, ref_moduli, slab, excl_lj, excl_coul;
    double fene_k, fene_r0, wall_lo, wall_hi;
    std::vector<double> modx, mody, modz;
};

static Model make_model(const phmc_params* P) {
    Model m;
    m.T = P->n_types;
    int TT = m.T * m.T;
    m.eps.assign(P->lj_eps, P->lj_eps + TT);
    m.sig.assign(P->lj_sig, P->lj_sig + TT);
    m.rc2.resize(TT); m.shift.resize(TT);
    for (int k = 0; k < TT; ++k) {
        double rc = P->lj_rc ? P->lj_rc[k] : P->rc_lj;
        m.rc2[k] = rc * rc;
        m.shift[k] = 0.0;
        if (P->lj_shift && m.eps[k] > 0 && m.sig[k] > 0) {
            double sr6 = std::pow(m.sig[k] / rc, 6);
            m.shift[k] = 4.0 * m.eps[k] * (sr6 * sr6 - sr6);
        }
    }
    m.rc_coul = P->rc_coul; m.elf = KE / P->epsilon_r; m.alpha = P->ewald_alpha;
    m.coulomb = P->coulomb; m.nx = P->mesh[0]; m.ny = P->mesh[1]; m.nz = P->mesh[2];
    m.order = P->order; m.ref_moduli = P->ref_moduli; m.slab = P->slab;
    m.excl_lj = P->excl_bonded_lj; m.excl_coul = P->excl_bonded_coul;
    m.fene_k = P->fene_k; m.fene_r0 = P->fene_r0; m.wall_lo = P->wall_lo; m.wall_hi = P->wall_hi;
    if (m.coulomb == PHMC_COUL_EWALD) {
        m.modx.resize(m.nx); m.mody.resize(m.ny); m.modz.resize(m.nz);
        orc_moduli(m.nx, m.order, m.ref_moduli, m.modx.data());
        orc_moduli(m.ny, m.order, m.ref_moduli, m.mody.data());
        orc_moduli(m.nz, m.order, m.ref_moduli, m.modz.data());
    }
    return m;
}

struct Sys {
    int cap;
    std::vector<double> x, y, z, q;
    std::vector<int> type, flags, present;
    std::vector<std::vector<int>> bonds;  // per slot partner list
    double box[3];
};

static inline double pair_u(const Model& m, const Sys& s, int i, int j, bool bonded, double* elj, double* ec) {
    double dx = min_image(s.x[i] - s.x[j], s.box[0]);
    double dy = min_image(s.y[i] - s.y[j], s.box[1]);
    double dz = min_image(s.z[i] - s.z[j], s.box[2]);
    double r2 = dx * dx + dy * dy + dz * dz;
    int p = s.type[i] * m.T + s.type[j];
    double a = 0, b = 0;
    if (!(bonded && m.excl_lj) && r2 <= m.rc2[p] && m.eps[p] > 0 && m.sig[p] > 0) {
        double sr6 = std::pow(m.sig[p] * m.sig[p] / r2, 3);
        a = 4.0 * m.eps[p] * (sr6 * sr6 - sr6) - m.shift[p];
    }
    if (m.coulomb != PHMC_COUL_NONE && !(bonded && m.excl_coul) && r2 <= m.rc_coul * m.rc_coul) {
        double qq = s.q[i] * s.q[j];
        if (qq != 0.0) {
            double r = std::sqrt(r2);
            b = (m.coulomb == PHMC_COUL_EWALD) ? m.elf * qq * std::erfc(m.alpha * r) / r : m.elf * qq / r;
        }
    }
    *elj += a; *ec += b;
    return a + b;
}

static bool is_bonded(const Sys& s, int i, int j) {
    for (int k : s.bonds[i]) if (k == j) return true;
    return false;
}

static void energy_scratch(const Model& m, const Sys& s, phmc_energy_components* out) {
    const int N = s.cap;
    double elj = 0, ec = 0;
    #pragma omp parallel for reduction(+ : elj, ec) schedule(dynamic, 32)
    for (int i = 0; i < N; ++i) {
        if (!s.present[i]) continue;
        for (int j = i + 1; j < N; ++j) {
            if (!s.present[j]) continue;
            pair_u(m, s, i, j, is_bonded(s, i, j), &elj, &ec);
        }
    }
    double ef = 0.0;
    if (m.fene_k > 0) {
        for (int i = 0; i < N; ++i) {
            if (!s.present[i]) continue;
            for (int j : s.bonds[i]) {
                if (j <= i || !s.present[j]) continue;
                double dx = min_image(s.x[i] - s.x[j], s.box[0]), dy = min_image(s.y[i] - s.y[j], s.box[1]), dz = min_image(s.z[i] - s.z[j], s.box[2]);
                double r2 = dx * dx + dy * dy + dz * dz, R2 = m.fene_r0 * m.fene_r0;
                if (r2 >= R2) ef = std::numeric_limits<double>::infinity();
                else ef += -0.5 * m.fene_k * R2 * std::log(1.0 - r2 / R2);
            }
        }
    }
    double wall = 0.0;
    if (m.wall_hi > m.wall_lo)
        for (int i = 0; i < N; ++i)
            if (s.present[i] && (s.z[i] < m.wall_lo || s.z[i] >= m.wall_hi)) wall = std::numeric_limits<double>::infinity();
    double erec = 0, self = 0, qc = 0, sl = 0;
    if (m.coulomb == PHMC_COUL_EWALD) {
        std::vector<double> Q;
        spread(N, s.x.data(), s.y.data(), s.z.data(), s.q.data(), s.present.data(), s.box, m.nx, m.ny, m.nz, m.order, Q);
        erec = recip_energy(Q, m.nx, m.ny, m.nz, s.box, m.alpha, m.elf, m.modx.data(), m.mody.data(), m.modz.data(), m.ref_moduli);
        double Qt, Q2, Mz, S2;
        charge_moments(N, s.z.data(), s.q.data(), s.present.data(), &Qt, &Q2, &Mz, &S2);
        ewald_corrections(Qt, Q2, Mz, S2, s.box, m.alpha, m.elf, m.slab, &self, &qc, &sl);
    }
    out->lj = elj; out->fene = ef + wall; out->coul_real = ec; out->coul_recip = erec;
    out->self = self; out->qcorr = qc; out->slab = sl;
    out->total = elj + ef + wall + ec + erec + self + qc + sl;
}

static Sys make_sys(const phmc_system* S) {
    Sys s;
    s.cap = S->capacity;
    s.x.assign(s.cap, 0.0); s.y.assign(s.cap, 0.0); s.z.assign(s.cap, 0.0); s.q.assign(s.cap, 0.0);
    s.type.assign(s.cap, 0); s.flags.assign(s.cap, PHMC_F_GHOST); s.present.assign(s.cap, 0);
    s.bonds.assign(s.cap, {});
    for (int i = 0; i < S->n_particles; ++i) {
        s.x[i] = S->x[i]; s.y[i] = S->y[i]; s.z[i] = S->z[i]; s.q[i] = S->q[i];
        s.type[i] = S->type[i]; s.flags[i] = S->flags[i];
        s.present[i] = (S->flags[i] & PHMC_F_GHOST) ? 0 : 1;
    }
    for (int k = 0; k < S->n_bonds; ++k) { s.bonds[S->bond_i[k]].push_back(S->bond_j[k]); s.bonds[S->bond_j[k]].push_back(S->bond_i[k]); }
    for (int d = 0; d < 3; ++d) s.box[d] = S->box[d];
    return s;
}

extern "C" int orc_energy(const phmc_system* S, const phmc_params* P, phmc_energy_components* out) {
    Model m = make_model(P);
    Sys s = make_sys(S);
    energy_scratch(m, s, out);
    return 0;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of the 4x32 S-box with the paper's
// multipliers and Weyl key increments.
// ---------------------------------------------------------------------------
extern "C" void orc_philox(const uint32_t* key_in, const uint32_t* ctr_in, uint32_t* out) {
    uint32_t k0 = key_in[0], k1 = key_in[1];
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// ---------------------------------------------------------------------------
// CPU Monte Carlo with the engine's move set (same proposal stream; energies
// from scratch).  Used for decision replay and small statistical checks.
// ---------------------------------------------------------------------------
struct MC {
    Model m;
    Sys s;
    phmc_params P;
    uint32_t key[2];
    std::vector<int> mobile, titr, anions, cations, freel;
    std::vector<int> pos_mobile, pos_anion, pos_cation;
    double E;
    int64_t t;
    float lx, ly, lz, wlo, whi;
};

static inline float u24(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }
static inline double u53(uint32_t a, uint32_t b) {
    uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
    return (double)(v & ((1ull << 53) - 1)) * (1.0 / 9007199254740992.0);
}
static inline int pick(uint32_t v, int n) { return (int)(((uint64_t)v * (uint64_t)n) >> 32); }

static void list_add(std::vector<int>& l, std::vector<int>& pos, int i) { pos[i] = (int)l.size(); l.push_back(i); }
static void list_del(std::vector<int>& l, std::vector<int>& pos, int i) {
    int k = pos[i]; int last = l.back(); l[k] = last; pos[last] = k; l.pop_back(); pos[i] = -1;
}

extern "C" void* orc_mc_create(const phmc_system* S, const phmc_params* P) {
    MC* mc = new MC;
    mc->m = make_model(P);
    mc->s = make_sys(S);
    mc->P = *P;
    mc->key[0] = (uint32_t)(P->seed & 0xffffffffu);
    mc->key[1] = (uint32_t)(P->seed >> 32);
    int cap = mc->s.cap;
    mc->pos_mobile.assign(cap, -1); mc->pos_anion.assign(cap, -1); mc->pos_cation.assign(cap, -1);
    for (int i = 0; i < cap; ++i) {
        if (!mc->s.present[i]) continue;
        int f = mc->s.flags[i];
        if (f & PHMC_F_MOBILE) list_add(mc->mobile, mc->pos_mobile, i);
        if (f & PHMC_F_TITRATABLE) mc->titr.push_back(i);
        if (f & PHMC_F_ANION) list_add(mc->anions, mc->pos_anion, i);
        if (f & PHMC_F_CATION) list_add(mc->cations, mc->pos_cation, i);
    }
    for (int i = cap - 1; i >= 0; --i) if (!mc->s.present[i]) mc->freel.push_back(i);
    phmc_energy_components c;
    energy_scratch(mc->m, mc->s, &c);
    mc->E = c.total;
    mc->t = 0;
    mc->lx = (float)S->box[0]; mc->ly = (float)S->box[1]; mc->lz = (float)S->box[2];
    mc->wlo = (float)P->wall_lo; mc->whi = (float)P->wall_hi;
    return mc;
}

extern "C" void orc_mc_destroy(void* h) { delete (MC*)h; }

struct Change { int idx, present; double x, y, z, q; int type; };

static void apply_changes(Sys& s, const Change* c, int n) {
    for (int k = 0; k < n; ++k) {
        int i = c[k].idx;
        s.present[i] = c[k].present; s.x[i] = c[k].x; s.y[i] = c[k].y; s.z[i] = c[k].z; s.q[i] = c[k].q; s.type[i] = c[k].type;
    }
}

// One trial.  forced = -1: Metropolis; 0/1: use that decision (replay).
// Outputs the move kind, dE (FP64, from scratch; +inf for wall/FENE violations;
// NaN when the move had nothing to act on) and the decision.
extern "C" int orc_mc_step(void* h, int forced, int* move_out, double* dE_out, int* acc_out) {
    MC* mc = (MC*)h;
    Sys& s = mc->s;
    const phmc_params& P = mc->P;
    uint32_t ctr[4] = {(uint32_t)(mc->t & 0xffffffffu), (uint32_t)((uint64_t)mc->t >> 32), 0, 0};
    uint32_t A[4], B[4], C[4];
    orc_philox(mc->key, ctr, A);
    ctr[2] = 1; orc_philox(mc->key, ctr, B);
    ctr[2] = 2; orc_philox(mc->key, ctr, C);
    mc->t++;
    float um = u24(A[0]);
    float pd = (float)P.p_disp, pt = (float)P.p_titr, ps = (float)P.p_swap;
    int move = PHMC_MOVE_NONE;
    if (um < pd) move = PHMC_MOVE_DISP;
    else if (um < pd + pt) move = PHMC_MOVE_TITR;
    else if (um < pd + pt + ps) move = PHMC_MOVE_SWAP;
    *move_out = move;
    *dE_out = std::numeric_limits<double>::quiet_NaN();
    *acc_out = 0;
    Change ch[2]; int nch = 0; double logf = 0.0;
    bool walls = mc->whi > mc->wlo;
    auto rand_pos = [&](uint32_t a, uint32_t b, uint32_t c, float* px, float* py, float* pz) {
        *px = mc->lx * u24(a);
        *py = mc->ly * u24(b);
        *pz = walls ? (mc->wlo + (mc->whi - mc->wlo) * u24(c)) : mc->lz * u24(c);
    };
    const double ln10 = std::log(10.0);
    if (move == PHMC_MOVE_DISP) {
        if (mc->mobile.empty()) return 0;
        int i = mc->mobile[pick(A[1], (int)mc->mobile.size())];
        float d = (float)P.disp_max;
        float dx = d * (2.0f * u24(A[2]) - 1.0f), dy = d * (2.0f * u24(A[3]) - 1.0f), dz = d * (2.0f * u24(B[0]) - 1.0f);
        float nx = (float)s.x[i] + dx, ny = (float)s.y[i] + dy, nz = (float)s.z[i] + dz;
        if (nx < 0.0f) nx += mc->lx; else if (nx >= mc->lx) nx -= mc->lx;
        if (ny < 0.0f) ny += mc->ly; else if (ny >= mc->ly) ny -= mc->ly;
        if (!walls) { if (nz < 0.0f) nz += mc->lz; else if (nz >= mc->lz) nz -= mc->lz; }
        ch[0] = {i, 1, nx, ny, nz, s.q[i], s.type[i]}; nch = 1;
    } else if (move == PHMC_MOVE_TITR) {
        if (mc->titr.empty()) return 0;
        int site = mc->titr[pick(A[1], (int)mc->titr.size())];
        if (s.q[site] == 0.0) {
            if (mc->freel.empty()) return 0;
            int g = mc->freel.back();
            float px, py, pz; rand_pos(A[2], A[3], B[0], &px, &py, &pz);
            ch[0] = {site, 1, s.x[site], s.y[site], s.z[site], (double)P.q_site_charged, P.type_site_charged};
            ch[1] = {g, 1, px, py, pz, (double)P.q_counterion, P.type_counterion};
            nch = 2; logf = ln10 * (P.pKa - P.pH);
        } else {
            if (mc->anions.empty()) return 0;
            int g = mc->anions[pick(B[1], (int)mc->anions.size())];
            ch[0] = {site, 1, s.x[site], s.y[site], s.z[site], 0.0, P.type_site_neutral};
            ch[1] = {g, 0, s.x[g], s.y[g], s.z[g], s.q[g], s.type[g]};
            nch = 2; logf = -ln10 * (P.pKa - P.pH);
        }
    } else if (move == PHMC_MOVE_SWAP) {
        double Vs = (double)mc->lx * mc->ly * (walls ? (double)(mc->whi - mc->wlo) : (double)mc->lz);
        double cs2V2 = P.salt_conc * P.salt_conc * Vs * Vs;
        if (u24(A[1]) < 0.5f) {
            if (mc->freel.size() < 2) return 0;
            int g1 = mc->freel[mc->freel.size() - 1], g2 = mc->freel[mc->freel.size() - 2];
            float px, py, pz, qx, qy, qz;
            rand_pos(A[2], A[3], B[0], &px, &py, &pz);
            rand_pos(C[0], C[1], C[2], &qx, &qy, &qz);
            ch[0] = {g1, 1, px, py, pz, (double)P.q_cation, P.type_cation};
            ch[1] = {g2, 1, qx, qy, qz, (double)P.q_counterion, P.type_counterion};
            nch = 2;
            logf = std::log(cs2V2 / ((double)(mc->cations.size() + 1) * (double)(mc->anions.size() + 1)));
        } else {
            if (mc->cations.empty() || mc->anions.empty()) return 0;
            int g1 = mc->cations[pick(B[1], (int)mc->cations.size())];
            int g2 = mc->anions[pick(C[3], (int)mc->anions.size())];
            ch[0] = {g1, 0, s.x[g1], s.y[g1], s.z[g1], s.q[g1], s.type[g1]};
            ch[1] = {g2, 0, s.x[g2], s.y[g2], s.z[g2], s.q[g2], s.type[g2]};
            nch = 2;
            logf = std::log((double)mc->cations.size() * (double)mc->anions.size() / cs2V2);
        }
    } else {
        return 0;
    }
    // dE from scratch: apply, recompute, compare with the cached total.
    Change old[2];
    for (int k = 0; k < nch; ++k) {
        int i = ch[k].idx;
        old[k] = {i, s.present[i], s.x[i], s.y[i], s.z[i], s.q[i], s.type[i]};
    }
    apply_changes(s, ch, nch);
    phmc_energy_components c;
    energy_scratch(mc->m, s, &c);
    double dE = c.total - mc->E;
    *dE_out = dE;
    double expo = -P.beta * dE + logf;
    int acc;
    if (forced >= 0) acc = forced;
    else acc = (expo >= 0.0) || (u53(B[2], B[3]) < std::exp(expo));
    *acc_out = acc;
    if (!acc) {
        for (int k = nch - 1; k >= 0; --k) apply_changes(s, &old[k], 1);
        return 0;
    }
    mc->E = c.total;
    // list bookkeeping, in the order the engine applies it
    if (move == PHMC_MOVE_TITR) {
        int g = ch[1].idx;
        if (ch[1].present) {
            mc->freel.pop_back();
            s.flags[g] = PHMC_F_MOBILE | PHMC_F_ANION;
            list_add(mc->mobile, mc->pos_mobile, g);
            list_add(mc->anions, mc->pos_anion, g);
        } else {
            list_del(mc->anions, mc->pos_anion, g);
            list_del(mc->mobile, mc->pos_mobile, g);
            s.flags[g] = PHMC_F_GHOST;
            mc->freel.push_back(g);
        }
    } else if (move == PHMC_MOVE_SWAP) {
        int g1 = ch[0].idx, g2 = ch[1].idx;
        if (ch[0].present) {
            mc->freel.pop_back(); mc->freel.pop_back();
            s.flags[g1] = PHMC_F_MOBILE | PHMC_F_CATION;
            list_add(mc->mobile, mc->pos_mobile, g1); list_add(mc->cations, mc->pos_cation, g1);
            s.flags[g2] = PHMC_F_MOBILE | PHMC_F_ANION;
            list_add(mc->mobile, mc->pos_mobile, g2); list_add(mc->anions, mc->pos_anion, g2);
        } else {
            list_del(mc->cations, mc->pos_cation, g1); list_del(mc->mobile, mc->pos_mobile, g1);
            s.flags[g1] = PHMC_F_GHOST; mc->freel.push_back(g1);
            list_del(mc->anions, mc->pos_anion, g2); list_del(mc->mobile, mc->pos_mobile, g2);
            s.flags[g2] = PHMC_F_GHOST; mc->freel.push_back(g2);
        }
    }
    return 0;
}

extern "C" double orc_mc_energy(void* h) { return ((MC*)h)->E; }

extern "C" void orc_mc_get_state(void* h, float* x, float* y, float* z, float* q, int* type, int* flags) {
    MC* mc = (MC*)h;
    for (int i = 0; i < mc->s.cap; ++i) {
        x[i] = (float)mc->s.x[i]; y[i] = (float)mc->s.y[i]; z[i] = (float)mc->s.z[i]; q[i] = (float)mc->s.q[i];
        type[i] = mc->s.type[i]; flags[i] = mc->s.flags[i];
    }
}

// Counts of protonated titratable sites, cations and anions.
extern "C" void orc_mc_counts(void* h, int* n_charged_sites, int* n_cations, int* n_anions) {
    MC* mc = (MC*)h;
    int c = 0;
    for (int i : mc->titr) if (mc->s.q[i] != 0.0) ++c;
    *n_charged_sites = c; *n_cations = (int)mc->cations.size(); *n_anions = (int)mc->anions.size();
}

// Cell index of each slot for a grid of cx*cy*cz cells (engine rule: float
// coordinate times float(c/L), truncated, clamped), -1 for ghosts.
extern "C" void orc_cells(void* h, int cx, int cy, int cz, int* cell_of) {
    MC* mc = (MC*)h;
    float ix = (float)cx / mc->lx, iy = (float)cy / mc->ly, iz = (float)cz / mc->lz;
    for (int i = 0; i < mc->s.cap; ++i) {
        if (!mc->s.present[i]) { cell_of[i] = -1; continue; }
        int a = std::min(cx - 1, std::max(0, (int)((float)mc->s.x[i] * ix)));
        int b = std::min(cy - 1, std::max(0, (int)((float)mc->s.y[i] * iy)));
        int c = std::min(cz - 1, std::max(0, (int)((float)mc->s.z[i] * iz)));
        cell_of[i] = (c * cy + b) * cx + a;
    }
}

// ---- the reference driver's random stream, from libstdc++ itself ----
// std::mt19937 and the two distributions the reference's move loops draw with
// (MC/src/mc.cu:62-65 choose_one, uniform_real_distribution<real>(0, 1) at
// :204,353-354), for the CPU restatement of its move phases.
extern "C" void* orc_mt_create(uint32_t seed) { return new std::mt19937(seed); }
extern "C" void orc_mt_destroy(void* h) { delete (std::mt19937*)h; }
extern "C" int orc_mt_index(void* h, int n) {
    std::uniform_int_distribution<int> d(0, n - 1);
    return d(*(std::mt19937*)h);
}
extern "C" float orc_mt_unit_float(void* h) {
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    return u(*(std::mt19937*)h);
}
// the generator's 624 state words and position, in its stream format
extern "C" void orc_mt_state(void* h, uint32_t* out) {
    std::stringstream ss;
    ss << *(std::mt19937*)h;
    for (int i = 0; i < 625; ++i) { unsigned long v = 0; ss >> v; out[i] = (uint32_t)v; }
}
