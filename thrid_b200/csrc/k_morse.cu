// k_morse.cu -- Morse pairs on the device: the Morse pair list of
// mklist_mor_cell.F90:8-327 (27-cell scan) and mklist2a_mor
// (mklist_mor.F90:30-160, all later Morse atoms), and morsep
// (morse.F90:206-414).
//
// The reference keeps Morse pairs apart from the nonbonded list: a list of
// its own over the Morse atoms (nmorselist: atoms of a type with a Morse
// partner type), radius rcut_bookmor, its own cutoff rcutmor and MTS group
// mts_mor.  The device does the same.  Layout in HBM:
//   mor_atoms int32[nmor]            Morse atoms, ascending (0-based)
//   mor_rows  int32[nmor][mor_cap]   partners of each Morse atom in the
//                                    reference's row order, mor_cnt[nmor]
//   mor_csort int32[nmor]            Morse atoms by cell (cell mode), in
//                                    ascending index inside each cell, the
//                                    order of cell_atomid
//   mor_par   double4[ntyp*ntyp]     (D, r0, alpha, 1 = Morse pair type) at
//                                    itype + ntyp*jtype (para_welmor(it, jt))
// The list test is the reference's exactly (FP64 minimum image with dnint,
// r^2 summed left to right without FMA), so the exported list is bit-exact.
// The force kernel takes one warp per Morse atom row; FP64 throughout in the
// FP64 path, FP32 after the FP64 displacement in mixed precision (forces and
// energies into the int64 fixed-point accumulators).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "pgk_ctx.cuh"

#define MOR_MAX_CELL 1024      // Morse atoms in one cell (shared-memory sort)

__device__ __forceinline__ bool mor_pair_in(const double* __restrict__ pos, int i, int j, const double* xi,
                                            double b0, double b1, double b2, double i0, double i1, double i2,
                                            double sqcut) {
    const double r0 = mi_exact(__dsub_rn(xi[0], pos[3 * j + 0]), b0, i0);
    const double r1 = mi_exact(__dsub_rn(xi[1], pos[3 * j + 1]), b1, i1);
    const double r2 = mi_exact(__dsub_rn(xi[2], pos[3 * j + 2]), b2, i2);
    const double dr = __dadd_rn(__dadd_rn(__dmul_rn(r0, r0), __dmul_rn(r1, r1)), __dmul_rn(r2, r2));
    return dr < sqcut;
}

// cell of each Morse atom: MOD(INT((x + L) / cellsize), cellcount), wrapped
// into range for coordinates below -L (the reference would index outside
// its cell array there)
__global__ void k_mor_cell_assign(const double* __restrict__ pos, const int* __restrict__ atoms, int nm,
                                  double b0, double b1, double b2, double c0, double c1, double c2, int n0, int n1,
                                  int n2, int* __restrict__ cell, int* __restrict__ ccnt) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nm) return;
    const int i = atoms[m];
    const double L[3] = {b0, b1, b2}, cs[3] = {c0, c1, c2};
    const int nc[3] = {n0, n1, n2};
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        int v = (int)__ddiv_rn(__dadd_rn(pos[3 * i + d], L[d]), cs[d]);
        v %= nc[d];
        c[d] = v < 0 ? v + nc[d] : v;
    }
    const int key = c[0] + n0 * (c[1] + n1 * c[2]);
    cell[m] = key;
    atomicAdd(&ccnt[key], 1);
}

// exclusive scan of the cell counts (one CTA), fill pointers, overflow flag
__global__ void k_mor_cell_scan(const int* __restrict__ cnt, int* __restrict__ start, int* __restrict__ fill,
                                int ncells, unsigned* __restrict__ status) {
    __shared__ int part[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int per = (ncells + nt - 1) / nt;
    const int b = t * per, e = min(ncells, b + per);
    int s = 0, mx = 0;
    for (int k = b; k < e; ++k) { s += cnt[k]; mx = max(mx, cnt[k]); }
    part[t] = s;
    if (mx > MOR_MAX_CELL) atomicOr(status, ST_CELL_OVERFLOW);
    __syncthreads();
    if (t == 0) {
        int run = 0;
        for (int k = 0; k < nt; ++k) { const int v = part[k]; part[k] = run; run += v; }
        start[ncells] = run;
    }
    __syncthreads();
    int run = part[t];
    for (int k = b; k < e; ++k) { start[k] = run; fill[k] = run; run += cnt[k]; }
}

__global__ void k_mor_cell_place(const int* __restrict__ cell, const int* __restrict__ atoms, int nm,
                                 int* __restrict__ fill, int* __restrict__ csort) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nm) return;
    csort[atomicAdd(&fill[cell[m]], 1)] = atoms[m];
}

// ascending atom index inside each cell (cell_atomid is filled in nmorselist
// order): rank of each entry among the cell's distinct atom indices
__global__ void k_mor_cell_sort(int* __restrict__ csort, const int* __restrict__ start, const int* __restrict__ cnt,
                                int ncells) {
    __shared__ int v[MOR_MAX_CELL];
    const int cl = blockIdx.x;
    if (cl >= ncells) return;
    const int b = start[cl], n = min(cnt[cl], MOR_MAX_CELL);
    for (int k = threadIdx.x; k < n; k += blockDim.x) v[k] = csort[b + k];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int x = v[k];
        int r = 0;
        for (int q = 0; q < n; ++q) r += v[q] < x ? 1 : 0;
        csort[b + r] = x;
    }
}

// One warp per Morse atom m1 (row mor1 = m1 + 1 of the reference): candidates
// in the reference's order (cell mode: the 27 cells z, y, x from -1 to +1,
// each cell's atoms ascending; all-pair mode: the later Morse atoms), tested
// 32 at a time; the passing ones are appended in order (ballot prefix).
template <bool CELL>
__global__ void k_mor_rows(const double* __restrict__ pos, const int* __restrict__ typ,
                           const int* __restrict__ atoms, int nm, const int* __restrict__ cell,
                           const int* __restrict__ cstart, const int* __restrict__ ccnt,
                           const int* __restrict__ csort, int n0, int n1, int n2, const double4* __restrict__ par,
                           int ntyp, double b0, double b1, double b2, double i0, double i1, double i2, double sqcut,
                           int cap, int* __restrict__ rows, int* __restrict__ rcnt,
                           unsigned long long* __restrict__ ctr) {
    const int lane = threadIdx.x & 31;
    const int m1 = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (m1 >= nm) return;
    const int i = atoms[m1];
    const int ti = typ[i];
    const double xi[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int* row = rows + (size_t)m1 * cap;
    int cnt = 0;
    auto take = [&](int j, bool valid) {
        bool pass = false;
        if (valid && j > i && par[ti + ntyp * typ[j]].w != 0.0)
            pass = mor_pair_in(pos, i, j, xi, b0, b1, b2, i0, i1, i2, sqcut);
        const unsigned bal = __ballot_sync(0xffffffffu, pass);
        if (pass) {
            const int at = cnt + __popc(bal & ((1u << lane) - 1u));
            if (at < cap) row[at] = j;
        }
        cnt += __popc(bal);
    };
    if (CELL) {
        const int key = cell[m1];
        const int cx = key % n0, cy = (key / n0) % n1, cz = key / (n0 * n1);
        for (int z1 = cz - 1; z1 <= cz + 1; ++z1) {
            const int z = (z1 + n2) % n2;
            for (int y1 = cy - 1; y1 <= cy + 1; ++y1) {
                const int y = (y1 + n1) % n1;
                for (int x1 = cx - 1; x1 <= cx + 1; ++x1) {
                    const int x = (x1 + n0) % n0;
                    const int c = x + n0 * (y + n1 * z);
                    const int b = cstart[c], e = b + ccnt[c];
                    for (int q = b; q < e; q += 32) {
                        const bool valid = q + lane < e;
                        take(valid ? csort[q + lane] : -1, valid);
                    }
                }
            }
        }
    } else {
        for (int q = m1 + 1; q < nm; q += 32) {
            const bool valid = q + lane < nm;
            take(valid ? atoms[q + lane] : -1, valid);
        }
    }
    if (lane == 0) {
        rcnt[m1] = cnt;
        atomicAdd(&ctr[0], (unsigned long long)cnt);
        atomicMax(&ctr[1], (unsigned long long)cnt);
    }
}

// morsep (morse.F90:206-414): one warp per Morse row, a lane per partner.
// rij = x_i - x_j (minimum image), pairs beyond rcutmor skipped,
// F_i += 2 a D (e^-2a(r-r0) - e^-a(r-r0)) / r * rij, F_j -= the same,
// U = D (e^-2a(r-r0) - 2 e^-a(r-r0)), virial sum(F . r) and tensor F (x) r.
template <bool MIXED, bool EV>
__global__ void __launch_bounds__(256) k_morse(const double* __restrict__ pos, const int* __restrict__ typ,
                                               const int* __restrict__ atoms, int nm, const int* __restrict__ rows,
                                               const int* __restrict__ rcnt, int cap,
                                               const double4* __restrict__ par, int ntyp, double sqcut,
                                               const DynState* __restrict__ dyn, void* __restrict__ facc,
                                               long long* __restrict__ acc) {
    using T = typename std::conditional<MIXED, float, double>::type;
    const int lane = threadIdx.x & 31;
    const int m1 = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    double ev[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) ev[k] = 0.0;
    if (m1 < nm) {
        const int i = atoms[m1];
        const int ti = typ[i];
        const double xi0 = pos[3 * i], xi1 = pos[3 * i + 1], xi2 = pos[3 * i + 2];
        const double b0 = dyn->box[0], b1 = dyn->box[1], b2 = dyn->box[2];
        const double v0 = dyn->boxinv[0], v1 = dyn->boxinv[1], v2 = dyn->boxinv[2];
        const int n = min(rcnt[m1], cap);
        const int* row = rows + (size_t)m1 * cap;
        T fi0 = 0, fi1 = 0, fi2 = 0;
        T e_pot = 0, e_vir = 0, t00 = 0, t01 = 0, t02 = 0, t11 = 0, t12 = 0, t22 = 0;
        for (int q = lane; q < n; q += 32) {
            const int j = row[q];
            double r0 = xi0 - pos[3 * j], r1 = xi1 - pos[3 * j + 1], r2 = xi2 - pos[3 * j + 2];
            r0 -= b0 * round(r0 * v0);
            r1 -= b1 * round(r1 * v1);
            r2 -= b2 * round(r2 * v2);
            const double rsq = r0 * r0 + r1 * r1 + r2 * r2;
            if (rsq > sqcut) continue;
            const double4 p = par[ti + ntyp * typ[j]];
            const T x0 = (T)r0, x1 = (T)r1, x2 = (T)r2;
            const T r = sqrt((T)rsq);
            const T rinv = (T)1 / r;
            const T e1 = exp(-(r - (T)p.y) * (T)p.z);
            const T e2 = e1 * e1;
            const T ft = (T)2 * (T)p.z * (T)p.x * (e2 - e1) * rinv;
            const T f0 = ft * x0, f1 = ft * x1, f2 = ft * x2;
            fi0 += f0; fi1 += f1; fi2 += f2;
            force_add<MIXED>(facc, j, -(double)f0, -(double)f1, -(double)f2);
            if (EV) {
                e_pot += (T)p.x * (e2 - (T)2 * e1);
                e_vir += f0 * x0 + f1 * x1 + f2 * x2;
                t00 += f0 * x0; t01 += f0 * x1; t02 += f0 * x2;
                t11 += f1 * x1; t12 += f1 * x2; t22 += f2 * x2;
            }
        }
        const double s0 = warp_sum((double)fi0), s1 = warp_sum((double)fi1), s2 = warp_sum((double)fi2);
        if (lane == 0 && n > 0) force_add<MIXED>(facc, i, s0, s1, s2);
        if (EV) {
            // tensor (3,3) column-major t[a + 3 b] = sum f_a r_b; f is parallel to r
            ev[0] = e_pot; ev[1] = e_vir;
            ev[2] = t00; ev[3] = t01; ev[4] = t02;     // (0,0) (1,0) (2,0)
            ev[5] = t01; ev[6] = t11; ev[7] = t12;     // (0,1) (1,1) (2,1)
            ev[8] = t02; ev[9] = t12; ev[10] = t22;    // (0,2) (1,2) (2,2)
        }
    }
    if (EV) {
        const int idx[11] = {A_MOR, A_VMOR, A_VTMOR + 0, A_VTMOR + 1, A_VTMOR + 2, A_VTMOR + 3, A_VTMOR + 4,
                             A_VTMOR + 5, A_VTMOR + 6, A_VTMOR + 7, A_VTMOR + 8};
        block_acc<11>(ev, acc, idx, !MIXED);
    }
}

// ---------------------------------------------------------------------------
// host side

// Morse atoms and the per-type-pair table (pgk_init); nothing to do without
// a Morse pair type or with Morse switched off (mts_mor = none)
pgk_status morse_setup(pgk_ctx* c, const pgk_system* s) {
    c->nmor = 0;
    if (!s->inter_inttyp || !s->para_welmor || !s->para_radmor || !s->para_alphamor) return PGK_OK;
    if (c->prm.mts_mor != PGK_MTS_LONG && c->prm.mts_mor != PGK_MTS_SHORT) return PGK_OK;
    const int nt = s->ntyp;
    std::vector<double4> par((size_t)nt * nt);
    std::vector<char> mt(nt, 0);
    bool any = false;
    for (int a = 0; a < nt; ++a)
        for (int b = 0; b < nt; ++b) {
            const size_t k = (size_t)a + (size_t)nt * b;      // para_welmor(itype, jtype), column-major
            const bool mor = s->inter_inttyp[k] == 2;
            par[k] = make_double4(s->para_welmor[k], s->para_radmor[k], s->para_alphamor[k], mor ? 1.0 : 0.0);
            if (mor) { mt[a] = 1; any = true; }
        }
    if (!any) return PGK_OK;
    std::vector<int> atoms;
    for (int i = 0; i < s->natom; ++i)
        if (mt[s->atmindex[i] - 1]) atoms.push_back(i);
    if (atoms.empty()) return PGK_OK;
    if (c->prm.rcutmor <= 0.0) return pgk_fail(c, PGK_E_INVALID, "rcutmor must be positive with Morse pairs");
    c->nmor = (int)atoms.size();
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_par, par.size() * sizeof(double4)));
    PGK_CUDA(c, cudaMemcpy(c->mor_par, par.data(), par.size() * sizeof(double4), cudaMemcpyHostToDevice));
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_atoms, atoms.size() * sizeof(int)));
    PGK_CUDA(c, cudaMemcpy(c->mor_atoms, atoms.data(), atoms.size() * sizeof(int), cudaMemcpyHostToDevice));
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_cnt, atoms.size() * sizeof(int)));
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_cell, atoms.size() * sizeof(int)));
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_csort, atoms.size() * sizeof(int)));
    PGK_CUDA(c, pgk_dmalloc(c, &c->mor_ctr, 2 * sizeof(unsigned long long)));
    // rows: the partners of a Morse atom inside rcut_bookmor at the Morse
    // atoms' mean density, half of them stored (j > i), regrown on overflow
    const double vol = c->prm.xcel * c->prm.ycel * c->prm.zcel;
    const double rb = c->prm.rcut_bookmor > 0.0 ? c->prm.rcut_bookmor : 0.0;
    double expect = rb > 0.0 ? (double)c->nmor / vol * 4.0 / 3.0 * 3.14159265358979 * rb * rb * rb : c->nmor;
    c->mor_cap = std::max(32, std::min(c->nmor, (int)(expect * 0.75 + 64)));
    return PGK_OK;
}

// mklist_mor_cell / mklist2a_mor at the current positions (the list builds of
// moldyn*.F90 at mod(step, nstep_bookmor) == 0)
pgk_status launch_mklist_mor(pgk_ctx* c) {
    if (c->nmor == 0) return PGK_OK;
    c->mor_valid = false;         // until this build completes
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    const double* box = c->hdyn.box;
    const double binv[3] = {1.0 / box[0], 1.0 / box[1], 1.0 / box[2]};
    const double rb = c->prm.rcut_bookmor;
    // without a list radius every Morse pair within half the box diagonal
    // (mklist_mor.F90: ifbookmor off)
    const double sqcut = rb > 0.0 ? rb * rb
                                  : (box[0] / 2.0) * (box[0] / 2.0) + (box[1] / 2.0) * (box[1] / 2.0) +
                                        (box[2] / 2.0) * (box[2] / 2.0);
    int nc[3] = {1, 1, 1};
    bool cell = rb > 0.0 && c->prm.list_mode != PGK_LIST_ALLPAIR;
    if (cell) {
        for (int d = 0; d < 3; ++d) nc[d] = (int)(box[d] / rb);
        const bool small = nc[0] < 3 || nc[1] < 3 || nc[2] < 3 || (long long)nc[0] * nc[1] * nc[2] <= 27;
        if (small && c->prm.list_mode == PGK_LIST_CELL)
            return pgk_fail(c, PGK_E_CELL_OVERFLOW, "mklist_mor_cell needs at least 3 cells per direction");
        if (small) cell = false;     // the rdscript.F90:1616-1632 fallback to mklist2a_mor
    }
    const int nm = c->nmor;
    const long long ncells = (long long)nc[0] * nc[1] * nc[2];
    if (cell) {
        if (ncells > (1LL << 24)) return pgk_fail(c, PGK_E_UNSUPPORTED, "too many Morse list cells");
        if (ncells > c->mor_maxcells) {
            pgk_dfree(c, c->mor_ccnt); pgk_dfree(c, c->mor_cstart); pgk_dfree(c, c->mor_cfill);
            c->mor_ccnt = c->mor_cstart = c->mor_cfill = nullptr;
            c->mor_maxcells = (int)ncells;
            PGK_CUDA(c, pgk_dmalloc(c, &c->mor_ccnt, sizeof(int) * (ncells + 1)));
            PGK_CUDA(c, pgk_dmalloc(c, &c->mor_cstart, sizeof(int) * (ncells + 1)));
            PGK_CUDA(c, pgk_dmalloc(c, &c->mor_cfill, sizeof(int) * (ncells + 1)));
        }
        double cs[3];
        for (int d = 0; d < 3; ++d) cs[d] = box[d] / (double)nc[d];
        PGK_CUDA(c, cudaMemsetAsync(c->mor_ccnt, 0, sizeof(int) * (ncells + 1), c->st));
        const int tb = 256, nb = (nm + tb - 1) / tb;
        k_mor_cell_assign<<<nb, tb, 0, c->st>>>(c->pos, c->mor_atoms, nm, box[0], box[1], box[2], cs[0], cs[1],
                                                cs[2], nc[0], nc[1], nc[2], c->mor_cell, c->mor_ccnt);
        k_mor_cell_scan<<<1, 1024, 0, c->st>>>(c->mor_ccnt, c->mor_cstart, c->mor_cfill, (int)ncells, c->status);
        k_mor_cell_place<<<nb, tb, 0, c->st>>>(c->mor_cell, c->mor_atoms, nm, c->mor_cfill, c->mor_csort);
        k_mor_cell_sort<<<(unsigned)ncells, 256, 0, c->st>>>(c->mor_csort, c->mor_cstart, c->mor_ccnt, (int)ncells);
        c->launches += 4;
        PGK_CUDA(c, cudaGetLastError());
    }
    for (int attempt = 0; attempt < 3; ++attempt) {
        if (!c->mor_rows) {
            if (pgk_dmalloc(c, &c->mor_rows, sizeof(int) * (size_t)nm * c->mor_cap) != cudaSuccess) {
                c->mor_rows = nullptr;
                return pgk_fail(c, PGK_E_NOMEM, "Morse pair list exceeds device memory");
            }
        }
        PGK_CUDA(c, cudaMemsetAsync(c->mor_ctr, 0, 2 * sizeof(unsigned long long), c->st));
        const unsigned blocks = (unsigned)(((long long)nm * 32 + 255) / 256);
        if (cell)
            k_mor_rows<true><<<blocks, 256, 0, c->st>>>(
                c->pos, c->typ, c->mor_atoms, nm, c->mor_cell, c->mor_cstart, c->mor_ccnt, c->mor_csort, nc[0], nc[1],
                nc[2], c->mor_par, c->ntyp, box[0], box[1], box[2], binv[0], binv[1], binv[2], sqcut, c->mor_cap,
                c->mor_rows, c->mor_cnt, c->mor_ctr);
        else
            k_mor_rows<false><<<blocks, 256, 0, c->st>>>(
                c->pos, c->typ, c->mor_atoms, nm, nullptr, nullptr, nullptr, nullptr, 1, 1, 1, c->mor_par, c->ntyp,
                box[0], box[1], box[2], binv[0], binv[1], binv[2], sqcut, c->mor_cap, c->mor_rows, c->mor_cnt,
                c->mor_ctr);
        c->launches += 1;
        PGK_CUDA(c, cudaGetLastError());
        unsigned long long ctr[2];
        unsigned st = 0;
        PGK_CUDA(c, cudaMemcpyAsync(ctr, c->mor_ctr, sizeof(ctr), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaMemcpyAsync(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        if (st & ST_CELL_OVERFLOW)
            return pgk_fail(c, PGK_E_CELL_OVERFLOW, "number of atoms in a cell exceeds max (morse)");
        if ((long long)ctr[1] > c->mor_cap) {
            // grow the rows and rebuild (the reference STOPs: "nlistmorall exceed")
            pgk_dfree(c, c->mor_rows);
            c->mor_rows = nullptr;
            c->mor_cap = (int)(((long long)ctr[1] * 5 / 4 + 32 + 31) / 32 * 32);
            continue;
        }
        c->mor_mode = cell ? PGK_LIST_CELL : PGK_LIST_ALLPAIR;
        c->mor_entries = (long long)ctr[0];
        c->mor_valid = true;
        ++c->list_epoch;              // captured step graphs hold the row pointer and capacity
        return PGK_OK;
    }
    return pgk_fail(c, PGK_E_LIST_OVERFLOW, "Morse list overflow after regrowth");
}

// morsep into group g's force and energy / virial accumulators
pgk_status launch_morse(pgk_ctx* c, int group, bool ev) {
    if (c->nmor == 0) return PGK_OK;
    pgk_status s;
    if (!c->mor_valid && (s = launch_mklist_mor(c))) return s;
    const double sq = c->prm.rcutmor * c->prm.rcutmor;
    const unsigned blocks = (unsigned)(((long long)c->nmor * 32 + 255) / 256);
    long long* acc = c->acc + (size_t)group * NACC;
    void* f = c->facc[group];
#define MOR_ARGS c->pos, c->typ, c->mor_atoms, c->nmor, c->mor_rows, c->mor_cnt, c->mor_cap, c->mor_par, c->ntyp, \
                 sq, c->dyn, f, acc
    if (c->mixed()) {
        if (ev) k_morse<true, true><<<blocks, 256, 0, c->st>>>(MOR_ARGS);
        else k_morse<true, false><<<blocks, 256, 0, c->st>>>(MOR_ARGS);
    } else {
        if (ev) k_morse<false, true><<<blocks, 256, 0, c->st>>>(MOR_ARGS);
        else k_morse<false, false><<<blocks, 256, 0, c->st>>>(MOR_ARGS);
    }
#undef MOR_ARGS
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// nmorselist / mor_indexall / mor_listall of the reference (1-based, rows for
// mor1 = 1 .. nmorse-1, a 0 entry for an empty row, mor_indexall(nmorse) =
// nlistmorall + 1)
pgk_status export_morlist(pgk_ctx* c, int32_t* nmorselist, int32_t* mor_index, int32_t* mor_list, int64_t cap,
                          int64_t* nl) {
    const int nm = c->nmor;
    if (nm == 0) { if (nl) *nl = 0; return PGK_OK; }
    if (!c->mor_valid) return pgk_fail(c, PGK_E_INVALID, "no Morse list has been built");
    std::vector<int> atoms(nm), cnt(nm), rows((size_t)nm * c->mor_cap);
    PGK_CUDA(c, cudaMemcpyAsync(atoms.data(), c->mor_atoms, sizeof(int) * nm, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(cnt.data(), c->mor_cnt, sizeof(int) * nm, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(rows.data(), c->mor_rows, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost,
                                c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    long long icut = 0;
    for (int m = 0; m + 1 < nm; ++m) {
        if (mor_index) mor_index[m] = (int32_t)(icut + 1);
        if (cnt[m] == 0) {
            if (mor_list && icut < cap) mor_list[icut] = 0;
            ++icut;
            continue;
        }
        for (int k = 0; k < cnt[m]; ++k, ++icut)
            if (mor_list && icut < cap) mor_list[icut] = rows[(size_t)m * c->mor_cap + k] + 1;
    }
    if (mor_index) mor_index[nm - 1] = (int32_t)(icut + 1);
    if (nmorselist)
        for (int m = 0; m < nm; ++m) nmorselist[m] = atoms[m] + 1;
    if (nl) *nl = icut;
    return PGK_OK;
}
