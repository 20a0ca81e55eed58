// Cell list (counting sort into padded per-cell slots) and the full-energy
// kernels: LJ/WCA + real-space Coulomb over the 27 neighbour cells, FENE
// bonds, walls and charge moments, all reduced in FP64 in a fixed order.
// Replaces build_half_neighbors_gpu (O(N^2), MC/src/neighbor.cu:21-125) and
// k_lj_energy / k_coul_energy / k_real_ewald_energy plus the Thrust
// reductions of pmeEnergy (MC/src/energy_gpu.cu:14-135, MC/src/pme.cu:252-288,425-447).
#include <algorithm>
#include "common.cuh"
#include "engine.h"

__global__ void k_cell_assign(DevPtrs d, const int* __restrict__ rep_of, int total) {
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (gs >= total) return;
    const int r = rep_of[gs];
    const RepDesc& D = d.desc[r];
    if (d.flags[gs] & PHMC_F_GHOST) { d.cell_of[gs] = -1; d.cell_pos[gs] = -1; return; }
    const float4 p = d.posq[gs];
    const int c = cell_index(D, p.x, p.y, p.z);
    const int k = atomicAdd(&d.cell_count[D.cell_off + c], 1);
    if (k < D.cell_cap) d.cell_list[((size_t)D.cell_off + c) * D.cell_cap + k] = gs - D.slot_off;
    else atomicExch(&d.state[r].error, PHMC_ERR_CAPACITY);
    d.cell_of[gs] = c;
}

// Sort every cell's members by slot index (deterministic order) and record
// each member's position inside its cell.
__global__ void k_cell_sort(DevPtrs d, const int* __restrict__ cell_rep, int total_cells) {
    const int gc = blockIdx.x * blockDim.x + threadIdx.x;
    if (gc >= total_cells) return;
    const RepDesc& D = d.desc[cell_rep[gc]];
    const int n = min(d.cell_count[gc], D.cell_cap);
    int* l = d.cell_list + (size_t)gc * D.cell_cap;
    for (int a = 1; a < n; ++a) {
        int v = l[a], b = a - 1;
        while (b >= 0 && l[b] > v) { l[b + 1] = l[b]; --b; }
        l[b + 1] = v;
    }
    int4 cc = make_int4(0, 0, 0, 0);
    for (int a = 0; a < n; ++a) {
        const int gi = D.slot_off + l[a];
        d.cell_pos[gi] = a;
        const int c = desc_class(d.flags[gi], d.posq[gi].w);
        cc.x += (c == 0); cc.y += (c == 1); cc.z += (c == 2); cc.w += (c == 3);
    }
    d.cell_cls[gc] = cc;
}

void launch_cell_build(Engine& E, cudaStream_t st) {
    cudaMemsetAsync(E.d.cell_count, 0, sizeof(int) * (size_t)E.total_cells, st);
    k_cell_assign<<<(E.total_slots + 255) / 256, 256, 0, st>>>(E.d, E.d_rep_of, E.total_slots);
    k_cell_sort<<<(E.total_cells + 127) / 128, 128, 0, st>>>(E.d, E.d_cell_rep, E.total_cells);
}

#define NCOMP 7
template <int NT>
__global__ void __launch_bounds__(NT) k_full_energy(DevPtrs d, int bpr) {
    __shared__ double red[40];
    const int r = blockIdx.y;
    const RepDesc& D = d.desc[r];
    double acc[NCOMP] = {0, 0, 0, 0, 0, 0, 0};  // lj, coul, fene(+walls), Q, Q2, Mz, S2
    for (int i = blockIdx.x * NT + threadIdx.x; i < D.cap; i += bpr * NT) {
        const int gi = D.slot_off + i;
        if (d.flags[gi] & PHMC_F_GHOST) continue;
        const float4 pi = d.posq[gi];
        const int ti = d.type[gi];
        const int4 bi = d.bonds[gi];
        acc[3] += pi.w; acc[4] += (double)pi.w * pi.w;
        acc[5] += (double)pi.w * pi.z; acc[6] += (double)pi.w * pi.z * pi.z;
        if (D.walls && (pi.z < D.wall_lo || pi.z >= D.wall_hi)) acc[2] = __longlong_as_double(0x7ff0000000000000ll);
        const int c = d.cell_of[gi];
        const int cx = c % D.ncell[0], cy = (c / D.ncell[0]) % D.ncell[1], cz = c / (D.ncell[0] * D.ncell[1]);
        // each unordered pair once: the own cell with j > i, and every particle of the 13
        // neighbour cells in the forward half shell (first non-zero offset of (dz, dy, dx)
        // positive; with at least 3 cells per axis these are 13 distinct cells)
        for (int h = 0; h < 14; ++h) {
            const int dz = (h == 0) ? 0 : (h < 5 ? 0 : 1), rem = (h == 0) ? 0 : (h < 5 ? h - 1 : h - 5);
            int dy, dx;
            if (h == 0) { dy = 0; dx = 0; }
            else if (h == 1) { dy = 0; dx = 1; }
            else if (h < 5) { dy = 1; dx = rem - 2; }            // h = 2..4: (0, 1, -1..1)
            else { dy = rem / 3 - 1; dx = rem % 3 - 1; }         // h = 5..13: (1, -1..1, -1..1)
            const int nc = (wrap_idx(cz + dz, D.ncell[2]) * D.ncell[1] + wrap_idx(cy + dy, D.ncell[1])) * D.ncell[0] +
                           wrap_idx(cx + dx, D.ncell[0]);
            const int cnt = min(d.cell_count[D.cell_off + nc], D.cell_cap);
            const int* l = d.cell_list + ((size_t)D.cell_off + nc) * D.cell_cap;
            for (int k = 0; k < cnt; ++k) {
                const int j = l[k];
                if (h == 0 && j <= i) continue;
                const float4 pj = d.posq[D.slot_off + j];
                const int tj = d.type[D.slot_off + j];
                float elj, ec;
                pair_energy(D, min_image(pi.x - pj.x, D.L[0]), min_image(pi.y - pj.y, D.L[1]),
                            min_image(pi.z - pj.z, D.L[2]), ti, tj, pi.w, pj.w, in_bonds(bi, j), elj, ec);
                acc[0] += elj; acc[1] += ec;
            }
        }
        if (D.fene_k > 0.0f) {
            const int bl[4] = {bi.x, bi.y, bi.z, bi.w};
            for (int k = 0; k < 4; ++k) {
                const int j = bl[k];
                if (j <= i) continue;
                const float4 pj = d.posq[D.slot_off + j];
                const float dx = min_image(pi.x - pj.x, D.L[0]), dy = min_image(pi.y - pj.y, D.L[1]), dz = min_image(pi.z - pj.z, D.L[2]);
                acc[2] += fene_energy(D, dx * dx + dy * dy + dz * dz);
            }
        }
    }
    for (int k = 0; k < NCOMP; ++k) {
        const double s = block_sum<NT>(acc[k], red);
        if (threadIdx.x == 0) d.partials[((size_t)r * bpr + blockIdx.x) * 8 + k] = s;
    }
}

// The same sums in cell order: each warp takes whole cells of its replica (cells
// blockIdx.x * warps + w, strided by the grid), its lanes the cell's particles, and
// runs over the own cell (partners j > i) and the 13 forward neighbour cells with
// every lane reading the same partner (one broadcast load per partner instead of
// 32 divergent walks); particle terms (FENE, walls, charge moments) by the lane that
// owns the particle.  Per-block partials as k_full_energy, reduced by k_full_reduce.
template <int NT>
__global__ void __launch_bounds__(NT) k_full_energy_cells(DevPtrs d, int bpr) {
    __shared__ double red[40];
    constexpr int NW = NT / 32;
    const int r = blockIdx.y, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const RepDesc& D = d.desc[r];
    const int ncells = D.ncell[0] * D.ncell[1] * D.ncell[2];
    double acc[NCOMP] = {0, 0, 0, 0, 0, 0, 0};
    for (int c = blockIdx.x * NW + w; c < ncells; c += bpr * NW) {
        const int n = min(d.cell_count[D.cell_off + c], D.cell_cap);
        if (n == 0) continue;
        const int cx = c % D.ncell[0], cy = (c / D.ncell[0]) % D.ncell[1], cz = c / (D.ncell[0] * D.ncell[1]);
        const int* own = d.cell_list + ((size_t)D.cell_off + c) * D.cell_cap;
        for (int i0 = 0; i0 < n; i0 += 32) {
            const bool act = i0 + lane < n;
            const int i = act ? own[i0 + lane] : -1;
            const int gi = D.slot_off + (act ? i : 0);
            const float4 pi = act ? d.posq[gi] : make_float4(0.f, 0.f, 0.f, 0.f);
            const int ti = act ? d.type[gi] : 0;
            const int4 bi = act ? d.bonds[gi] : make_int4(-1, -1, -1, -1);
            if (act) {
                acc[3] += pi.w; acc[4] += (double)pi.w * pi.w;
                acc[5] += (double)pi.w * pi.z; acc[6] += (double)pi.w * pi.z * pi.z;
                if (D.walls && (pi.z < D.wall_lo || pi.z >= D.wall_hi)) acc[2] = __longlong_as_double(0x7ff0000000000000ll);
            }
            for (int h = 0; h < 14; ++h) {
                const int dz = (h == 0) ? 0 : (h < 5 ? 0 : 1), rem = (h == 0) ? 0 : (h < 5 ? h - 1 : h - 5);
                int dy, dx;
                if (h == 0) { dy = 0; dx = 0; }
                else if (h == 1) { dy = 0; dx = 1; }
                else if (h < 5) { dy = 1; dx = rem - 2; }
                else { dy = rem / 3 - 1; dx = rem % 3 - 1; }
                const int nc = (wrap_idx(cz + dz, D.ncell[2]) * D.ncell[1] + wrap_idx(cy + dy, D.ncell[1])) * D.ncell[0] +
                               wrap_idx(cx + dx, D.ncell[0]);
                const int cnt = min(d.cell_count[D.cell_off + nc], D.cell_cap);
                const int* l = d.cell_list + ((size_t)D.cell_off + nc) * D.cell_cap;
                for (int k = 0; k < cnt; ++k) {
                    const int j = l[k];
                    const float4 pj = d.posq[D.slot_off + j];
                    const int tj = d.type[D.slot_off + j];
                    if (!act || (h == 0 && j <= i)) continue;
                    float elj, ec;
                    pair_energy(D, min_image(pi.x - pj.x, D.L[0]), min_image(pi.y - pj.y, D.L[1]),
                                min_image(pi.z - pj.z, D.L[2]), ti, tj, pi.w, pj.w, in_bonds(bi, j), elj, ec);
                    acc[0] += elj; acc[1] += ec;
                }
            }
            if (act && D.fene_k > 0.0f) {
                const int bl[4] = {bi.x, bi.y, bi.z, bi.w};
                for (int k = 0; k < 4; ++k) {
                    const int j = bl[k];
                    if (j <= i) continue;
                    const float4 pj = d.posq[D.slot_off + j];
                    const float ddx = min_image(pi.x - pj.x, D.L[0]), ddy = min_image(pi.y - pj.y, D.L[1]),
                                ddz = min_image(pi.z - pj.z, D.L[2]);
                    acc[2] += fene_energy(D, ddx * ddx + ddy * ddy + ddz * ddz);
                }
            }
        }
    }
    for (int k = 0; k < NCOMP; ++k) {
        const double s = block_sum<NT>(acc[k], red);
        if (threadIdx.x == 0) d.partials[((size_t)r * bpr + blockIdx.x) * 8 + k] = s;
    }
}

__global__ void k_full_reduce(DevPtrs d, int R, int bpr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    double a[NCOMP] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < bpr; ++b)
        for (int k = 0; k < NCOMP; ++k) a[k] += d.partials[((size_t)r * bpr + b) * 8 + k];
    const RepDesc& D = d.desc[r];
    RepState& S = d.state[r];
    S.E_pair_lj = a[0]; S.E_pair_c = a[1]; S.E_fene = a[2];
    S.Q = a[3]; S.Q2 = a[4]; S.Mz = a[5]; S.S2 = a[6];
    if (D.coulomb == PHMC_COUL_EWALD) {
        S.E_self = D.self_coef * S.Q2;
        S.E_qcorr = D.qcorr_coef * S.Q * S.Q;
        double es = 0.0;
        if (D.slab) {
            es = D.slab_coef * S.Mz * S.Mz;
            if (fabs(S.Q) > 1e-4) es -= D.slab_coef * S.Q * (S.S2 + S.Q * D.Lz2_12);
        }
        S.E_slab = es;
    } else {
        S.E_self = S.E_qcorr = S.E_slab = 0.0;
        S.E_rec = 0.0;
    }
    S.E = S.E_pair_lj + S.E_pair_c + S.E_fene + S.E_rec + S.E_self + S.E_qcorr + S.E_slab;
}

// Particles per block (E.energy_block: 64, 128 or 256; 0 the cell-ordered pass) is a
// tuning parameter; blocks per replica cover the largest replica, at most
// PHMC_FULL_MAX_BPR (the partials' size).
void launch_full_energy(Engine& E, cudaStream_t st) {
    const int nt = E.energy_block;
    if (nt == 0) {  // cell order: one warp per cell, 8 warps per block
        const int bpr = std::max(1, std::min(PHMC_FULL_MAX_BPR, (E.max_cells + 7) / 8));
        k_full_energy_cells<256><<<dim3(bpr, E.R), 256, 0, st>>>(E.d, bpr);
        k_full_reduce<<<(E.R + 127) / 128, 128, 0, st>>>(E.d, E.R, bpr);
        return;
    }
    const int bpr = std::max(1, std::min(PHMC_FULL_MAX_BPR, (E.max_cap + nt - 1) / nt));
    dim3 grid(bpr, E.R);
    if (nt == 64) k_full_energy<64><<<grid, 64, 0, st>>>(E.d, bpr);
    else if (nt == 256) k_full_energy<256><<<grid, 256, 0, st>>>(E.d, bpr);
    else k_full_energy<128><<<grid, 128, 0, st>>>(E.d, bpr);
    k_full_reduce<<<(E.R + 127) / 128, 128, 0, st>>>(E.d, E.R, bpr);
}
