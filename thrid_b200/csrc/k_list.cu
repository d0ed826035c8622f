// k_list.cu -- bookkeeping pair list (mklist_cell.F90:8-352 / mklist.F90:8-234)
// and molecule wrap (transcor.F90) on the device.
//
// The device list keeps, for every atom in cell-sorted order, the FULL set of
// partners j != i with r^2 < rcut_book^2 (exact FP64 test, no FMA, Fortran
// dnint min image) minus the mkexcl exclusions.  Its i<j half is, pair for
// pair, the reference list; pgk_get_nblist() writes it back in the reference
// CSR layout and row order.  The full rows let the pair kernel accumulate the
// force of atom i without atomics on j.
//
// Cells: cellcount = INT(L/rcut_book), cell = MOD(INT((x+L)/cellsize), n)
// exactly as mklist_cell.F90:114-180.  When the reference would refuse the
// cell index (rdscript.F90:1595-1610) the same cells are scanned as distinct
// neighbour cells, which covers every pair of the all-pair mklist2a test
// because cellsize >= rcut_book.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "pgk_ctx.cuh"

#define MAX_CELL_ATOMS 4096

// transcor.F90: wrap each molecule by its first atom into [0, L)
__global__ void k_transcor(double* __restrict__ pos, const int* __restrict__ mol_idx,
                           const int* __restrict__ mol_list, int nmole, const DynState* __restrict__ dyn) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmole) return;
    int b = mol_idx[m], e = mol_idx[m + 1];
    int a0 = mol_list[b];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double L = dyn->box[d];
        double x = pos[3 * a0 + d];
        double sh = 0.0;
        if (x < 0.0) sh = L;
        else if (x > L) sh = -L;
        if (sh != 0.0)
            for (int q = b; q < e; ++q) {
                int k = mol_list[q];
                pos[3 * k + d] = __dadd_rn(pos[3 * k + d], sh);
            }
    }
}

__device__ __forceinline__ int cell_coord(double x, double L, double cs, int nc) {
    int c = (int)__ddiv_rn(__dadd_rn(x, L), cs);
    c %= nc;
    return c < 0 ? c + nc : c;
}

__global__ void k_cell_assign(const double* __restrict__ pos, int n, const DynState* __restrict__ dyn,
                              int* __restrict__ cell_of, int* __restrict__ cell_cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = cell_coord(pos[3 * i + d], dyn->box[d], dyn->cellsize[d], dyn->ncell[d]);
    int key = c[0] + dyn->ncell[0] * (c[1] + dyn->ncell[1] * c[2]);
    cell_of[i] = key;
    atomicAdd(&cell_cnt[key], 1);
}

// exclusive scan of the cell counts (one CTA; ncells <= a few 10^4)
__global__ void k_cell_scan(const int* __restrict__ cnt, int* __restrict__ start, int* __restrict__ fill,
                            int ncells, unsigned* status) {
    __shared__ int part[1024];
    int t = threadIdx.x, nt = blockDim.x;
    int per = (ncells + nt - 1) / nt;
    int b = t * per, e = min(ncells, b + per);
    int s = 0, mx = 0;
    for (int k = b; k < e; ++k) { s += cnt[k]; mx = max(mx, cnt[k]); }
    part[t] = s;
    if (mx > MAX_CELL_ATOMS) atomicOr(status, ST_CELL_OVERFLOW);
    __syncthreads();
    if (t == 0) {
        int run = 0;
        for (int k = 0; k < nt; ++k) { int v = part[k]; part[k] = run; run += v; }
        start[ncells] = run;
    }
    __syncthreads();
    int run = part[t];
    for (int k = b; k < e; ++k) { start[k] = run; fill[k] = run; run += cnt[k]; }
}

__global__ void k_cell_place(const int* __restrict__ cell_of, int n, int* __restrict__ fill, int* __restrict__ perm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = atomicAdd(&fill[cell_of[i]], 1);
    perm[p] = i;
}

// stable order inside each cell: ascending original index (bitonic sort)
__global__ void k_cell_sort(int* __restrict__ perm, const int* __restrict__ start, int ncells) {
    __shared__ int v[MAX_CELL_ATOMS];
    int cell = blockIdx.x;
    if (cell >= ncells) return;
    int b = start[cell], n = start[cell + 1] - b;
    if (n <= 1 || n > MAX_CELL_ATOMS) return;
    int np = 1;
    while (np < n) np <<= 1;
    for (int k = threadIdx.x; k < np; k += blockDim.x) v[k] = k < n ? perm[b + k] : 0x7fffffff;
    __syncthreads();
    for (int size = 2; size <= np; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < np; k += blockDim.x) {
                int p = k ^ stride;
                if (p > k) {
                    bool up = (k & size) == 0;
                    int a = v[k], c = v[p];
                    if ((a > c) == up) { v[k] = c; v[p] = a; }
                }
            }
            __syncthreads();
        }
    for (int k = threadIdx.x; k < n; k += blockDim.x) perm[b + k] = v[k];
}

__global__ void k_sorted_gather(const int* __restrict__ perm, int n, const double* __restrict__ pos,
                                const int* __restrict__ typ, int* __restrict__ iperm, double* __restrict__ pos_s,
                                int* __restrict__ typ_s) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int i = perm[s];
    iperm[i] = s;
    pos_s[3 * s + 0] = pos[3 * i + 0];
    pos_s[3 * s + 1] = pos[3 * i + 1];
    pos_s[3 * s + 2] = pos[3 * i + 2];
    typ_s[s] = typ[i];
}

__device__ __forceinline__ bool is_excluded(const int* __restrict__ exs_idx, const int* __restrict__ exs_list,
                                            int io, int jo) {
    int b = exs_idx[io], e = exs_idx[io + 1];
    for (int k = b; k < e; ++k) {
        int v = exs_list[k];
        if (v == jo) return true;
        if (v > jo) return false;
    }
    return false;
}

// one warp per sorted atom: scan the distinct neighbour cells, keep the
// exact-test pairs, drop exclusions, append to the row.
__global__ void __launch_bounds__(256) k_build_list(
        const double* __restrict__ pos_s, const int* __restrict__ perm, const int* __restrict__ cell_of,
        const int* __restrict__ cell_start, const int* __restrict__ exs_idx, const int* __restrict__ exs_list,
        int n, int cap, double sqcut, const DynState* __restrict__ dyn,
        int* __restrict__ nbr, int* __restrict__ ncnt, unsigned long long* __restrict__ counters,
        unsigned* __restrict__ status) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n) return;
    int s = warp;
    int io = perm[s];
    double xi = pos_s[3 * s], yi = pos_s[3 * s + 1], zi = pos_s[3 * s + 2];
    double L0 = dyn->box[0], L1 = dyn->box[1], L2 = dyn->box[2];
    double B0 = 1.0 / L0, B1 = 1.0 / L1, B2 = 1.0 / L2;
    int nc0 = dyn->ncell[0], nc1 = dyn->ncell[1], nc2 = dyn->ncell[2];
    int key = cell_of[io];
    int cx = key % nc0, cy = (key / nc0) % nc1, cz = key / (nc0 * nc1);
    int nz = nc2 >= 3 ? 3 : nc2, ny = nc1 >= 3 ? 3 : nc1, nx = nc0 >= 3 ? 3 : nc0;
    int count = 0, half = 0;
    int* row = nbr + (size_t)s * cap;
    for (int a = 0; a < nz; ++a) {
        int z = nc2 >= 3 ? (cz + a - 1 + nc2) % nc2 : a;
        for (int b = 0; b < ny; ++b) {
            int y = nc1 >= 3 ? (cy + b - 1 + nc1) % nc1 : b;
            for (int c = 0; c < nx; ++c) {
                int x = nc0 >= 3 ? (cx + c - 1 + nc0) % nc0 : c;
                int cell = x + nc0 * (y + nc1 * z);
                int t0 = cell_start[cell], t1 = cell_start[cell + 1];
                for (int tb = t0; tb < t1; tb += 32) {
                    int t = tb + lane;
                    bool keep = false;
                    int jo = -1;
                    if (t < t1 && t != s) {
                        double r0 = mi_exact(__dsub_rn(xi, pos_s[3 * t]), L0, B0);
                        double r1 = mi_exact(__dsub_rn(yi, pos_s[3 * t + 1]), L1, B1);
                        double r2 = mi_exact(__dsub_rn(zi, pos_s[3 * t + 2]), L2, B2);
                        double dr = __dadd_rn(__dadd_rn(__dmul_rn(r0, r0), __dmul_rn(r1, r1)), __dmul_rn(r2, r2));
                        if (dr < sqcut) {
                            jo = perm[t];
                            keep = !is_excluded(exs_idx, exs_list, io, jo);
                        }
                    }
                    unsigned m = __ballot_sync(0xffffffffu, keep);
                    unsigned mh = __ballot_sync(0xffffffffu, keep && jo > io);
                    if (keep) {
                        int off = count + __popc(m & ((1u << lane) - 1u));
                        if (off < cap) row[off] = t;
                    }
                    count += __popc(m);
                    half += __popc(mh);
                }
            }
        }
    }
    if (lane == 0) {
        ncnt[s] = min(count, cap);
        if (count > cap) atomicOr(status, ST_LIST_OVERFLOW);
        atomicMax(&counters[1], (unsigned long long)count);
        if (io < n - 1) atomicAdd(&counters[0], (unsigned long long)(half > 0 ? half : 1));
    }
}

pgk_status launch_transcor(pgk_ctx* c) {
    if (c->nmole == 0) return PGK_OK;
    k_transcor<<<(c->nmole + 255) / 256, 256, 0, c->st>>>(c->pos, c->mol_idx, c->mol_list, c->nmole, c->dyn);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// list-mode rule of rdscript.F90:1595-1610
static int list_mode_for(const pgk_ctx* c, const double* box, int* nc) {
    for (int d = 0; d < 3; ++d) nc[d] = (int)(box[d] / c->prm.rcut_book);
    if (c->prm.list_mode == PGK_LIST_CELL) return PGK_LIST_CELL;
    if (c->prm.list_mode == PGK_LIST_ALLPAIR) return PGK_LIST_ALLPAIR;
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3 || (long long)nc[0] * nc[1] * nc[2] <= 27) return PGK_LIST_ALLPAIR;
    return PGK_LIST_CELL;
}

pgk_status launch_mklist(pgk_ctx* c) {
    int n = c->natom;
    // the box may have changed on the device (MTK): read it back
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    int nc[3];
    int mode = list_mode_for(c, c->hdyn.box, nc);
    if (mode == PGK_LIST_CELL && (nc[0] < 3 || nc[1] < 3 || nc[2] < 3))
        return pgk_fail(c, PGK_E_CELL_OVERFLOW, "mklist_cell needs at least 3 cells per direction");
    for (int d = 0; d < 3; ++d) nc[d] = std::max(1, nc[d]);
    long long ncells = (long long)nc[0] * nc[1] * nc[2];
    if (ncells > c->maxcells) {
        cudaFree(c->cell_cnt); cudaFree(c->cell_start); cudaFree(c->cell_fill);
        c->maxcells = (int)ncells;
        PGK_CUDA(c, cudaMalloc(&c->cell_cnt, sizeof(int) * (ncells + 1)));
        PGK_CUDA(c, cudaMalloc(&c->cell_start, sizeof(int) * (ncells + 1)));
        PGK_CUDA(c, cudaMalloc(&c->cell_fill, sizeof(int) * (ncells + 1)));
    }
    DynState& h = c->hdyn;
    for (int d = 0; d < 3; ++d) { h.ncell[d] = nc[d]; h.cellsize[d] = h.box[d] / (double)nc[d]; }
    h.list_mode_used = mode;
    PGK_CUDA(c, cudaMemcpyAsync(c->dyn, &h, sizeof(DynState), cudaMemcpyHostToDevice, c->st));
    for (int attempt = 0; attempt < 3; ++attempt) {
        PGK_CUDA(c, cudaMemsetAsync(c->cell_cnt, 0, sizeof(int) * (ncells + 1), c->st));
        PGK_CUDA(c, cudaMemsetAsync(c->counters, 0, 2 * sizeof(unsigned long long), c->st));
        int tb = 256, nb = (n + tb - 1) / tb;
        k_cell_assign<<<nb, tb, 0, c->st>>>(c->pos, n, c->dyn, c->cell_of, c->cell_cnt);
        k_cell_scan<<<1, 1024, 0, c->st>>>(c->cell_cnt, c->cell_start, c->cell_fill, (int)ncells, c->status);
        k_cell_place<<<nb, tb, 0, c->st>>>(c->cell_of, n, c->cell_fill, c->perm);
        k_cell_sort<<<(int)ncells, 512, 0, c->st>>>(c->perm, c->cell_start, (int)ncells);
        k_sorted_gather<<<nb, tb, 0, c->st>>>(c->perm, n, c->pos, c->typ, c->iperm, c->pos_s, c->typ_s);
        double sq = c->prm.rcut_book * c->prm.rcut_book;
        long long threads = (long long)n * 32;
        k_build_list<<<(unsigned)((threads + 255) / 256), 256, 0, c->st>>>(
            c->pos_s, c->perm, c->cell_of, c->cell_start, c->exs_idx, c->exs_list, n, c->cap, sq, c->dyn,
            c->nbr, c->ncnt, c->counters, c->status);
        c->launches += 6;
        PGK_CUDA(c, cudaGetLastError());
        unsigned long long cnt[2];
        unsigned st;
        PGK_CUDA(c, cudaMemcpyAsync(cnt, c->counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaMemcpyAsync(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        if (st & ST_CELL_OVERFLOW) return pgk_fail(c, PGK_E_CELL_OVERFLOW, "number of atoms in a cell exceeds the device maximum");
        if (st & ST_LIST_OVERFLOW) {
            // grow the rows and rebuild (the reference STOPs here)
            int need = (int)((cnt[1] + 63) / 32 * 32);
            unsigned zero = 0;
            PGK_CUDA(c, cudaMemcpy(c->status, &zero, sizeof(zero), cudaMemcpyHostToDevice));
            size_t bytes = (size_t)n * need * sizeof(int);
            cudaFree(c->nbr);
            if (cudaMalloc(&c->nbr, bytes) != cudaSuccess) {
                c->nbr = nullptr;
                return pgk_fail(c, PGK_E_LIST_OVERFLOW, "pair list exceeds device memory");
            }
            c->cap = need;
            continue;
        }
        h.nlistnball = (long long)cnt[0];
        h.nmaxrow = (int)cnt[1];
        PGK_CUDA(c, cudaMemcpyAsync(&c->dyn->nlistnball, &h.nlistnball, sizeof(long long),
                                    cudaMemcpyHostToDevice, c->st));
        c->list_valid = true;
        return PGK_OK;
    }
    return pgk_fail(c, PGK_E_LIST_OVERFLOW, "pair list overflow after regrowth");
}

// Reference CSR (nb_indexall / nb_listall) from the device rows.
pgk_status export_nblist(pgk_ctx* c, int32_t* nb_index, int32_t* nb_list, int64_t cap, int64_t* nl) {
    if (!c->list_valid) return pgk_fail(c, PGK_E_INVALID, "no pair list has been built");
    int n = c->natom;
    std::vector<int> ncnt(n), perm(n), iperm(n), cell_of(n);
    std::vector<int> rows((size_t)n * c->cap);
    PGK_CUDA(c, cudaMemcpyAsync(ncnt.data(), c->ncnt, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(perm.data(), c->perm, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(iperm.data(), c->iperm, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(cell_of.data(), c->cell_of, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(rows.data(), c->nbr, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    const DynState& h = c->hdyn;
    int nc0 = h.ncell[0], nc1 = h.ncell[1], nc2 = h.ncell[2];
    bool cellmode = h.list_mode_used == PGK_LIST_CELL;
    long long pos = 0;
    std::vector<std::pair<long long, int>> tmp;
    for (int i = 0; i < n - 1; ++i) {
        int s = iperm[i];
        tmp.clear();
        int ki = cell_of[i];
        int ix = ki % nc0, iy = (ki / nc0) % nc1, iz = ki / (nc0 * nc1);
        for (int k = 0; k < ncnt[s]; ++k) {
            int j = perm[rows[(size_t)s * c->cap + k]];
            if (j <= i) continue;
            long long ord = j;
            if (cellmode) {   // 27-cell scan order z, y, x (mklist_cell.F90:218-273)
                int kj = cell_of[j];
                int jx = kj % nc0, jy = (kj / nc0) % nc1, jz = kj / (nc0 * nc1);
                int dx = ((jx - ix) % nc0 + nc0) % nc0; if (dx == nc0 - 1) dx = -1;
                int dy = ((jy - iy) % nc1 + nc1) % nc1; if (dy == nc1 - 1) dy = -1;
                int dz = ((jz - iz) % nc2 + nc2) % nc2; if (dz == nc2 - 1) dz = -1;
                long long slot = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                ord = slot * (long long)n + j;
            }
            tmp.push_back({ord, j});
        }
        std::sort(tmp.begin(), tmp.end());
        if (nb_index) nb_index[i] = (int32_t)(pos + 1);
        if (tmp.empty()) {
            if (nb_list && pos < cap) nb_list[pos] = 0;
            ++pos;
        } else {
            for (auto& p : tmp) {
                if (nb_list && pos < cap) nb_list[pos] = p.second + 1;
                ++pos;
            }
        }
    }
    if (nb_index && n >= 1) nb_index[n - 1] = (int32_t)(pos + 1);
    *nl = pos;
    if (nb_list && pos > cap) return pgk_fail(c, PGK_E_INVALID, "nb_listall capacity too small");
    return PGK_OK;
}
