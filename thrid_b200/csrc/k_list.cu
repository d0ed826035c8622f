// k_list.cu -- bookkeeping pair list (mklist_cell.F90:8-352 / mklist.F90:8-234)
// and molecule wrap (transcor.F90) on the device.
//
// Layout.  Atoms are counting-sorted into the reference's cells
// (cellcount = INT(L/rcut_book), cell = MOD(INT((x+L)/cellsize), n),
// mklist_cell.F90:114-180); inside a cell by (4x4x4 sub-cell, atom index), and
// each cell's segment is padded with dummy slots (perm = -1) to a multiple of
// 8, so every 8-slot CLUSTER lies inside one cell.
//
// List.  For every i-cluster the row holds each atom slot t that is a
// partner of at least one of the cluster's atoms s with t > s, as
// (mask << 24 | t): bit b of the mask says that (8*cluster + b, t) is a list
// pair.  Every pair is therefore stored once, in the row of its lower slot.
// Membership is the reference test pair for pair: exact FP64
// r^2 < rcut_book^2 (no FMA, Fortran dnint minimum image) minus the mkexcl
// exclusions; pgk_get_nblist() writes the pairs back in the reference CSR
// layout and row order.  When the reference would
// refuse the cell index (rdscript.F90:1595-1610) the same cells are scanned
// as distinct neighbour cells, which covers every pair of the all-pair
// mklist2a test because cellsize >= rcut_book.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "pgk_ctx.cuh"

#define MAX_CELL_ATOMS 4096
#define SUBKEY_SHIFT 25

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

// cell of each atom (reference rule) and its sort key inside the cell: the
// 4x4x4 sub-cell (Morton order) above the atom index
__global__ void k_cell_assign(const double* __restrict__ pos, int n, const DynState* __restrict__ dyn,
                              int* __restrict__ cell_of, int* __restrict__ cell_cnt, int* __restrict__ subkey) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[3], sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double L = dyn->box[d], cs = dyn->cellsize[d];
        c[d] = cell_coord(pos[3 * i + d], L, cs, dyn->ncell[d]);
        double u = __ddiv_rn(__dadd_rn(pos[3 * i + d], L), cs);
        double fr = u - floor(u);
        int q = (int)(fr * 4.0);
        sc[d] = q < 0 ? 0 : (q > 3 ? 3 : q);
    }
    int key = c[0] + dyn->ncell[0] * (c[1] + dyn->ncell[1] * c[2]);
    cell_of[i] = key;
    int morton = 0;
#pragma unroll
    for (int b = 0; b < 2; ++b)
        morton |= (((sc[0] >> b) & 1) << (3 * b)) | (((sc[1] >> b) & 1) << (3 * b + 1)) |
                  (((sc[2] >> b) & 1) << (3 * b + 2));
    subkey[i] = (morton << SUBKEY_SHIFT) | i;
    atomicAdd(&cell_cnt[key], 1);
}

// exclusive scan of the padded cell sizes (one CTA; ncells <= a few 10^4)
__global__ void k_cell_scan(const int* __restrict__ cnt, int* __restrict__ start, int* __restrict__ fill,
                            int ncells, unsigned* status) {
    __shared__ int part[1024];
    int t = threadIdx.x, nt = blockDim.x;
    int per = (ncells + nt - 1) / nt;
    int b = t * per, e = min(ncells, b + per);
    int s = 0, mx = 0;
    for (int k = b; k < e; ++k) { s += (cnt[k] + 7) & ~7; mx = max(mx, cnt[k]); }
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
    for (int k = b; k < e; ++k) { start[k] = run; fill[k] = run; run += (cnt[k] + 7) & ~7; }
}

__global__ void k_cell_place(const int* __restrict__ cell_of, int n, int* __restrict__ fill, int* __restrict__ perm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = atomicAdd(&fill[cell_of[i]], 1);
    perm[p] = i;
}

// deterministic order inside each cell: ascending (sub-cell, atom index);
// the padding slots at the end of the segment get perm = -1
__global__ void k_cell_sort(int* __restrict__ perm, const int* __restrict__ start, const int* __restrict__ cnt,
                            const int* __restrict__ subkey, int ncells) {
    __shared__ int v[MAX_CELL_ATOMS];
    int cell = blockIdx.x;
    if (cell >= ncells) return;
    int b = start[cell], n = cnt[cell], npad = start[cell + 1] - b;
    for (int k = n + threadIdx.x; k < npad; k += blockDim.x) perm[b + k] = -1;
    if (n <= 0 || n > MAX_CELL_ATOMS) return;
    int np = 1;
    while (np < n) np <<= 1;
    for (int k = threadIdx.x; k < np; k += blockDim.x) v[k] = k < n ? subkey[perm[b + k]] : 0x7fffffff;
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
    for (int k = threadIdx.x; k < n; k += blockDim.x) perm[b + k] = v[k] & ((1 << SUBKEY_SHIFT) - 1);
}

__global__ void k_sorted_gather(const int* __restrict__ perm, int npad, const double* __restrict__ pos,
                                const int* __restrict__ typ, int* __restrict__ iperm, double* __restrict__ pos_s,
                                int* __restrict__ typ_s) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npad) return;
    int i = perm[s];
    if (i < 0) {
        pos_s[3 * s + 0] = 0.0; pos_s[3 * s + 1] = 0.0; pos_s[3 * s + 2] = 0.0;
        typ_s[s] = 0;
        return;
    }
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

// one warp per i-cluster: scan the distinct neighbour cells of the cluster's
// cell, candidates t above the cluster's first slot only (each pair is stored
// in its lower slot's row).  A candidate farther than rcut_book (+ margin)
// from the bounding box of the cluster's atoms is skipped; otherwise all 8
// cluster atoms get the exact reference test (FP64, exclusions) and the entry
// (mask << 24 | t) is appended when any bit is set.
// nlistnball (the reference's row count, one sentinel per empty row) is the
// number of pairs plus the atoms i < n-1 without a partner of higher index;
// hasup[i] = 1 marks the atoms that have one.
__global__ void __launch_bounds__(256) k_build_clist(
        const double* __restrict__ pos_s, const int* __restrict__ perm, const int* __restrict__ cell_of,
        const int* __restrict__ cell_start, const int* __restrict__ cell_cnt, const int* __restrict__ exs_idx,
        const int* __restrict__ exs_list, const int2* __restrict__ exs_rng, int n, int ncl, int ccap, int sort_rows,
        double sqcut, double rbox, float sqlo, float sqhi,
        const DynState* __restrict__ dyn, int* __restrict__ clist, int* __restrict__ ccnt,
        unsigned char* __restrict__ hasup, unsigned long long* __restrict__ counters, unsigned* __restrict__ status) {
    __shared__ double spi[8][3 * 8];
    __shared__ int sio[8][8];
    __shared__ int2 srng[8][8];
    const int wib = threadIdx.x >> 5;
    const int cl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (cl >= ncl) return;
    const int s0 = 8 * cl;
    if (lane < 8) {
        int io = perm[s0 + lane];
        sio[wib][lane] = io;
        srng[wib][lane] = io >= 0 ? exs_rng[io] : make_int2(INT_MAX, -1);
        spi[wib][3 * lane] = pos_s[3 * (s0 + lane)];
        spi[wib][3 * lane + 1] = pos_s[3 * (s0 + lane) + 1];
        spi[wib][3 * lane + 2] = pos_s[3 * (s0 + lane) + 2];
    }
    __syncwarp();
    const double L[3] = {dyn->box[0], dyn->box[1], dyn->box[2]};
    const double B[3] = {1.0 / L[0], 1.0 / L[1], 1.0 / L[2]};
    const int nc0 = dyn->ncell[0], nc1 = dyn->ncell[1], nc2 = dyn->ncell[2];
    // bounding box of the real cluster atoms, minimum image relative to atom 0
    double ctr[3], hw[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double lo = 0.0, hi = 0.0;
        const double x0 = spi[wib][d];
        for (int ii = 1; ii < 8; ++ii) {
            if (sio[wib][ii] < 0) continue;
            double r = spi[wib][3 * ii + d] - x0;
            r -= L[d] * rint(r * B[d]);
            lo = fmin(lo, r); hi = fmax(hi, r);
        }
        ctr[d] = x0 + 0.5 * (lo + hi);
        hw[d] = 0.5 * (hi - lo);
    }
    const double rb2 = rbox * rbox;
    // FP32 copies for the screening tests: a pair whose FP32 squared distance
    // is below sqlo (above sqhi) is inside (outside) rcut_book whatever the
    // rounding; only pairs between the two take the exact FP64 test
    const float Lf[3] = {(float)L[0], (float)L[1], (float)L[2]};
    const float Bf[3] = {(float)B[0], (float)B[1], (float)B[2]};
    const float ctrf[3] = {(float)ctr[0], (float)ctr[1], (float)ctr[2]};
    const float hwf[3] = {(float)hw[0], (float)hw[1], (float)hw[2]};
    const float rb2f = (float)rb2 * 1.0001f + 1.0e-3f;
    const int key = cell_of[sio[wib][0]];
    const int cx = key % nc0, cy = (key / nc0) % nc1, cz = key / (nc0 * nc1);
    const int nz = nc2 >= 3 ? 3 : nc2, ny = nc1 >= 3 ? 3 : nc1, nx = nc0 >= 3 ? 3 : nc0;
    int count = 0;
    unsigned long long npair = 0;
    unsigned up = 0;                                   // bit ii: cluster atom ii has a higher-index partner
    int* row = clist + (size_t)cl * ccap;
    // Candidates that pass the bounding-box test queue up (in scan order) and
    // are tested against the 8 cluster atoms 32 at a time, so the exact tests
    // run on full warps.  Entries come out in the same order as a direct scan.
    __shared__ int squeue[8][32 + 4 * 32];
    int* queue = squeue[wib];
    int qn = 0;
    auto test_batch = [&](int t) {          // t < 0: idle lane
        unsigned mask = 0;
        if (t >= 0) {
            const double xj = pos_s[3 * t], yj = pos_s[3 * t + 1], zj = pos_s[3 * t + 2];
            const float pjf[3] = {(float)xj, (float)yj, (float)zj};
            const int jo = perm[t];
            bool jlow = false;
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
                const int io = sio[wib][ii];
                if (io < 0 || t <= s0 + ii) continue;
                float q2 = 0.f;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float r = (float)spi[wib][3 * ii + d] - pjf[d];
                    r -= Lf[d] * rintf(r * Bf[d]);
                    q2 = fmaf(r, r, q2);
                }
                if (q2 > sqhi) continue;
                bool in = q2 < sqlo;
                if (!in) {       // near rcut_book: the reference's exact FP64 test decides
                    double r0 = mi_exact(__dsub_rn(spi[wib][3 * ii], xj), L[0], B[0]);
                    double r1 = mi_exact(__dsub_rn(spi[wib][3 * ii + 1], yj), L[1], B[1]);
                    double r2 = mi_exact(__dsub_rn(spi[wib][3 * ii + 2], zj), L[2], B[2]);
                    double dr = __dadd_rn(__dadd_rn(__dmul_rn(r0, r0), __dmul_rn(r1, r1)), __dmul_rn(r2, r2));
                    in = dr < sqcut;
                }
                const int2 rg = srng[wib][ii];
                if (in && !(jo >= rg.x && jo <= rg.y && is_excluded(exs_idx, exs_list, io, jo))) {
                    mask |= 1u << ii;
                    if (jo > io) up |= 1u << ii;
                    else jlow = true;
                }
            }
            if (jlow) hasup[jo] = 1;
            npair += (unsigned long long)__popc(mask);
        }
        const unsigned m = __ballot_sync(0xffffffffu, mask != 0);
        if (mask) {
            const int off = count + __popc(m & ((1u << lane) - 1u));
            if (off < ccap) row[off] = (int)((mask << 24) | (unsigned)t);
        }
        count += __popc(m);
    };
    for (int a = 0; a < nz; ++a) {
        int z = nc2 >= 3 ? (cz + a - 1 + nc2) % nc2 : a;
        for (int b = 0; b < ny; ++b) {
            int y = nc1 >= 3 ? (cy + b - 1 + nc1) % nc1 : b;
            for (int c = 0; c < nx; ++c) {
                int x = nc0 >= 3 ? (cx + c - 1 + nc0) % nc0 : c;
                int cell = x + nc0 * (y + nc1 * z);
                int t0 = cell_start[cell], t1 = t0 + cell_cnt[cell];
                if (t1 <= s0 + 1) continue;             // every slot of the cell is below the cluster
                t0 = max(t0, s0 + 1);
                for (int tb = t0; tb < t1; tb += 128) {
                    // four candidates a lane: their positions load together
                    double px[4][3];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int t = tb + 32 * u + lane;
#pragma unroll
                        for (int d = 0; d < 3; ++d) px[u][d] = t < t1 ? pos_s[3 * t + d] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int t = tb + 32 * u + lane;
                        bool acc = false;
                        if (t < t1) {
                            float e2 = 0.f;
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                float r = (float)px[u][d] - ctrf[d];
                                r -= Lf[d] * rintf(r * Bf[d]);
                                const float ex = fmaxf(fabsf(r) - hwf[d], 0.f);
                                e2 += ex * ex;
                            }
                            acc = e2 <= rb2f;
                        }
                        const unsigned ba = __ballot_sync(0xffffffffu, acc);
                        if (acc) queue[qn + __popc(ba & ((1u << lane) - 1u))] = t;
                        qn += __popc(ba);
                    }
                    __syncwarp();
                    while (qn >= 32) {
                        const int tq = queue[lane];
                        int rest[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) rest[u] = qn - 32 > 32 * u + lane ? queue[32 + 32 * u + lane] : -1;
                        __syncwarp();
#pragma unroll
                        for (int u = 0; u < 4; ++u) if (rest[u] >= 0) queue[32 * u + lane] = rest[u];
                        qn -= 32;
                        __syncwarp();
                        test_batch(tq);
                    }
                }
            }
        }
    }
    if (qn > 0) {
        const int tq = lane < qn ? queue[lane] : -1;
        test_batch(tq);
    }
    // Group the row's entries by mask (stable counting sort in shared memory,
    // bins in inverse-Gray-code order of the masks): 32 consecutive entries
    // then mostly share their mask bits, so the pair kernel's loop over the
    // mask bits is nearly uniform across the warp.  Entries keep their
    // candidate (spatial) order inside a mask group; the result is the same on
    // every build of the same positions.
    if (sort_rows && count <= ccap) {
        extern __shared__ int srow_raw[];
        int* buf = srow_raw + (size_t)wib * (ccap + 256);
        int* bin = buf + ccap;
        for (int q = lane; q < 256; q += 32) bin[q] = 0;
        __syncwarp();
        for (int k = lane; k < count; k += 32) {
            const int e = row[k];
            buf[k] = e;
            atomicAdd(&bin[mask_bin((unsigned)e >> 24)], 1);
        }
        __syncwarp();
        warp_scan256(bin, lane);                 // exclusive scan of the 256 bins
        __syncwarp();
        for (int k0 = 0; k0 < count; k0 += 32) {
            const int k = k0 + lane;
            const bool ok = k < count;
            const int e = ok ? buf[k] : 0;
            const unsigned key = ok ? mask_bin((unsigned)e >> 24) : 256u + lane;
            const unsigned grp = __match_any_sync(0xffffffffu, key);
            const int rank = __popc(grp & ((1u << lane) - 1u));
            const int base = ok ? bin[key] : 0;
            __syncwarp();
            if (ok) {
                row[base + rank] = e;
                if (rank == 0) bin[key] = base + __popc(grp);
            }
            __syncwarp();
        }
    }
    up = __reduce_or_sync(0xffffffffu, up);
    npair = warp_sum(npair);
    if (lane < 8 && ((up >> lane) & 1u)) hasup[sio[wib][lane]] = 1;
    if (lane == 0) {
        ccnt[cl] = min(count, ccap);
        if (count > ccap) atomicOr(status, ST_LIST_OVERFLOW);
        atomicMax(&counters[1], (unsigned long long)count);
        atomicAdd(&counters[0], npair);
    }
}

// atoms i < n-1 without a partner of higher index (one sentinel row each)
__global__ void k_count_noup(const unsigned char* __restrict__ hasup, int m, unsigned long long* counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned v = (i < m && !hasup[i]) ? 1u : 0u;
    unsigned w = __popc(__ballot_sync(0xffffffffu, v));
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&counters[2], (unsigned long long)w);
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

// (re)allocate the sorted/padded arrays for up to npad_cap slots
// cluster rows (book and pruned) for npad_cap/8 clusters of ccap entries
static pgk_status alloc_rows(pgk_ctx* c) {
    pgk_dfree(c, c->clist); pgk_dfree(c, c->plist);
    c->clist = nullptr; c->plist = nullptr;
    const size_t bytes = sizeof(int) * (size_t)(c->npad_cap / 8) * c->ccap;
    if (pgk_dmalloc(c, &c->clist, bytes) != cudaSuccess) {
        c->clist = nullptr;
        return pgk_fail(c, PGK_E_NOMEM, "cluster pair list exceeds device memory");
    }
    if (c->prune_buffer > 0.f && pgk_dmalloc(c, &c->plist, bytes) != cudaSuccess) {
        c->plist = nullptr;
        return pgk_fail(c, PGK_E_NOMEM, "pruned pair list exceeds device memory");
    }
    return PGK_OK;
}

static pgk_status ensure_sorted_capacity(pgk_ctx* c, int npad_cap) {
    if (npad_cap <= c->npad_cap) return PGK_OK;
    pgk_dfree(c, c->perm); pgk_dfree(c, c->pos_s); pgk_dfree(c, c->typ_s); pgk_dfree(c, c->xq); pgk_dfree(c, c->xq64);
    pgk_dfree(c, c->ccnt); pgk_dfree(c, c->clist); pgk_dfree(c, c->fsort); pgk_dfree(c, c->plist); pgk_dfree(c, c->pcnt);
    pgk_dfree(c, c->xq_prune);
    c->perm = nullptr; c->pos_s = nullptr; c->typ_s = nullptr; c->xq = nullptr; c->xq64 = nullptr;
    c->ccnt = nullptr; c->clist = nullptr; c->fsort = nullptr; c->plist = nullptr; c->pcnt = nullptr;
    c->xq_prune = nullptr;
    int ncl = npad_cap / 8;
    PGK_CUDA(c, pgk_dmalloc(c, &c->perm, sizeof(int) * npad_cap));
    PGK_CUDA(c, pgk_dmalloc(c, &c->pos_s, sizeof(double) * 3 * npad_cap));
    PGK_CUDA(c, pgk_dmalloc(c, &c->typ_s, sizeof(int) * npad_cap));
    if (c->mixed()) {
        PGK_CUDA(c, pgk_dmalloc(c, &c->xq, sizeof(int4) * npad_cap));
        PGK_CUDA(c, pgk_dmalloc(c, &c->fsort, sizeof(long long) * 3 * (size_t)npad_cap));
        PGK_CUDA(c, cudaMemsetAsync(c->fsort, 0, sizeof(long long) * 3 * (size_t)npad_cap, c->st));
    }
    else PGK_CUDA(c, pgk_dmalloc(c, &c->xq64, sizeof(double4) * npad_cap));
    PGK_CUDA(c, pgk_dmalloc(c, &c->ccnt, sizeof(int) * ncl));
    if (c->prune_buffer > 0.f) {
        PGK_CUDA(c, pgk_dmalloc(c, &c->pcnt, sizeof(int) * ncl));
        PGK_CUDA(c, pgk_dmalloc(c, &c->xq_prune, sizeof(int4) * npad_cap));
        PGK_CUDA(c, cudaMemsetAsync(c->xq_prune, 0, sizeof(int4) * npad_cap, c->st));
    }
    c->npad_cap = npad_cap;
    return alloc_rows(c);
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
        pgk_dfree(c, c->cell_cnt); pgk_dfree(c, c->cell_start); pgk_dfree(c, c->cell_fill);
        c->maxcells = (int)ncells;
        PGK_CUDA(c, pgk_dmalloc(c, &c->cell_cnt, sizeof(int) * (ncells + 1)));
        PGK_CUDA(c, pgk_dmalloc(c, &c->cell_start, sizeof(int) * (ncells + 1)));
        PGK_CUDA(c, pgk_dmalloc(c, &c->cell_fill, sizeof(int) * (ncells + 1)));
    }
    long long npad_max = (long long)n + 7 * ncells;
    if (npad_max >= (1 << 24)) return pgk_fail(c, PGK_E_UNSUPPORTED, "more than 2^24 padded atom slots");
    pgk_status s;
    if ((npad_max + 7) / 8 * 8 > c->npad_cap) {
        if ((s = ensure_sorted_capacity(c, (int)((npad_max + 7) / 8 * 8)))) return s;
    }
    DynState& h = c->hdyn;
    for (int d = 0; d < 3; ++d) { h.ncell[d] = nc[d]; h.cellsize[d] = h.box[d] / (double)nc[d]; }
    h.list_mode_used = mode;
    PGK_CUDA(c, cudaMemcpyAsync(c->dyn, &h, sizeof(DynState), cudaMemcpyHostToDevice, c->st));
    for (int attempt = 0; attempt < 3; ++attempt) {
        PGK_CUDA(c, cudaMemsetAsync(c->cell_cnt, 0, sizeof(int) * (ncells + 1), c->st));
        PGK_CUDA(c, cudaMemsetAsync(c->counters, 0, 4 * sizeof(unsigned long long), c->st));
        int tb = 256, nb = (n + tb - 1) / tb;
        k_cell_assign<<<nb, tb, 0, c->st>>>(c->pos, n, c->dyn, c->cell_of, c->cell_cnt, c->subkey);
        k_cell_scan<<<1, 1024, 0, c->st>>>(c->cell_cnt, c->cell_start, c->cell_fill, (int)ncells, c->status);
        k_cell_place<<<nb, tb, 0, c->st>>>(c->cell_of, n, c->cell_fill, c->perm);
        k_cell_sort<<<(int)ncells, 512, 0, c->st>>>(c->perm, c->cell_start, c->cell_cnt, c->subkey, (int)ncells);
        int npad = 0;
        PGK_CUDA(c, cudaMemcpyAsync(&npad, c->cell_start + ncells, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        c->npad = npad;
        c->ncl = npad / 8;
        k_sorted_gather<<<(npad + 255) / 256, 256, 0, c->st>>>(c->perm, npad, c->pos, c->typ, c->iperm, c->pos_s,
                                                               c->typ_s);
        double sq = c->prm.rcut_book * c->prm.rcut_book;
        // screening margin on r^2: FP32 coordinates (up to twice the box) carry
        // 2^-24 relative error each, a distance component up to 4x that
        const double lmax = std::max(h.box[0], std::max(h.box[1], h.box[2]));
        const double eps_pos = 4.0 * 5.96e-8 * 2.0 * lmax;
        const double scr = std::max(0.01, 2.0 * 2.0 * c->prm.rcut_book * 1.7321 * eps_pos + 1.0e-3);
        long long threads = (long long)c->ncl * 32;
        PGK_CUDA(c, cudaMemsetAsync(c->hasup, 0, (size_t)n, c->st));
        // rows are grouped by mask in shared memory when 8 rows fit (<= 160 KB)
        const size_t sort_sm = (size_t)8 * (c->ccap + 256) * sizeof(int);
        const int sort_rows = sort_sm <= 160 * 1024 ? 1 : 0;
        if (sort_rows) PGK_CUDA(c, smem_limit(k_build_clist, sort_sm));
        k_build_clist<<<(unsigned)((threads + 255) / 256), 256, sort_rows ? sort_sm : 0, c->st>>>(
            c->pos_s, c->perm, c->cell_of, c->cell_start, c->cell_cnt, c->exs_idx, c->exs_list, c->exs_rng, n, c->ncl,
            c->ccap,
            sort_rows, sq, c->prm.rcut_book + 0.05, (float)(sq * (1.0 - 1.0e-5) - scr),
            (float)(sq * (1.0 + 1.0e-5) + scr), c->dyn, c->clist, c->ccnt, c->hasup, c->counters, c->status);
        if (n > 1) k_count_noup<<<(n - 1 + 255) / 256, 256, 0, c->st>>>(c->hasup, n - 1, c->counters);
        c->launches += 7;
        PGK_CUDA(c, cudaGetLastError());
        unsigned long long cnt[4];
        unsigned st;
        PGK_CUDA(c, cudaMemcpyAsync(cnt, c->counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaMemcpyAsync(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        if (st & ST_CELL_OVERFLOW)
            return pgk_fail(c, PGK_E_CELL_OVERFLOW, "number of atoms in a cell exceeds the device maximum");
        if (st & ST_LIST_OVERFLOW) {
            // grow the cluster rows and rebuild (the reference STOPs here)
            unsigned zero = 0;
            PGK_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(zero), c->st));
            // a quarter of headroom above the longest row, so the rows of
            // later builds (density fluctuations) rarely force another regrowth
            c->ccap = (int)(((long long)cnt[1] * 5 / 4 + 32 + 31) / 32 * 32);
            if ((s = alloc_rows(c))) return s;
            continue;
        }
        h.nlistnball = (long long)(cnt[0] + cnt[2]);
        h.nmaxrow = (int)cnt[1];
        PGK_CUDA(c, cudaMemcpyAsync(&c->dyn->nlistnball, &h.nlistnball, sizeof(long long),
                                    cudaMemcpyHostToDevice, c->st));
        c->list_valid = true;
        ++c->list_epoch;
        if (c->prune_buffer > 0.f) PGK_CUDA(c, cudaMemsetAsync(&c->prune->force, 1, 1, c->st));   // re-prune
        return pair_autotune(c);      // once per context
    }
    return pgk_fail(c, PGK_E_LIST_OVERFLOW, "pair list overflow after regrowth");
}

// Reference CSR (nb_indexall / nb_listall) from the device cluster rows:
// every stored pair goes to the row of its lower original index, then each
// row is ordered like the reference (27-cell z-y-x scan or ascending j).
pgk_status export_nblist(pgk_ctx* c, int32_t* nb_index, int32_t* nb_list, int64_t cap, int64_t* nl) {
    if (!c->list_valid) return pgk_fail(c, PGK_E_INVALID, "no pair list has been built");
    int n = c->natom, npad = c->npad, ncl = c->ncl;
    std::vector<int> ccnt(ncl), perm(npad), cell_of(n);
    std::vector<int> rows((size_t)ncl * c->ccap);
    PGK_CUDA(c, cudaMemcpyAsync(ccnt.data(), c->ccnt, sizeof(int) * ncl, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(perm.data(), c->perm, sizeof(int) * npad, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(cell_of.data(), c->cell_of, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(rows.data(), c->clist, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    const DynState& h = c->hdyn;
    int nc0 = h.ncell[0], nc1 = h.ncell[1], nc2 = h.ncell[2];
    bool cellmode = h.list_mode_used == PGK_LIST_CELL;
    std::vector<std::vector<int>> part(n);
    for (int cl = 0; cl < ncl; ++cl)
        for (int k = 0; k < ccnt[cl]; ++k) {
            unsigned e = (unsigned)rows[(size_t)cl * c->ccap + k];
            int j = perm[e & 0xFFFFFFu];
            for (int b = 0; b < 8; ++b) {
                if (!((e >> (24 + b)) & 1u)) continue;
                int i = perm[8 * cl + b];
                if (i < j) part[i].push_back(j); else part[j].push_back(i);
            }
        }
    long long pos = 0;
    std::vector<std::pair<long long, int>> tmp;
    for (int i = 0; i < n - 1; ++i) {
        tmp.clear();
        int ki = cell_of[i];
        int ix = ki % nc0, iy = (ki / nc0) % nc1, iz = ki / (nc0 * nc1);
        for (int j : part[i]) {
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
