// k_nonbond.cu -- real-space LJ + Ewald pair kernel (ewaldrp, ewaldr.F90:404-838)
//
// Work decomposition: one warp per atom i of the cell-sorted order, lanes
// stride over i's full neighbour row (j != i, both directions), so the force
// on i is a register sum closed by a warp shuffle reduction -- no atomics on
// j, and a fixed summation order.  Every pair is therefore evaluated twice;
// energies and virials carry a factor 1/2.
//
// Mixed precision: positions enter as 32-bit fractional fixed point per box
// axis (x/L * 2^32); the wrapped integer difference is the minimum-image
// displacement, converted to FP32 with the box scale.  The displacement error
// is ~L/2^32 (3e-8 A at L = 130 A) instead of the 8e-6 A of FP32 absolute
// coordinates.  Pair arithmetic is FP32 with the reference's natural cubic
// spline tables (spline_interp.F90) staged in shared memory; the per-atom
// force is converted once to int64 fixed point (2^32) and added to the group
// accumulator.  FP64 precision runs the same structure in double with the
// reference's dnint minimum image.
//
// Roofline: FP32 pipe (61 algorithmic flop per interacting pair) plus one
// 4-byte index and one 16-byte (32-byte FP64) gather per list entry.
#include <vector>

#include "pgk_ctx.cuh"

// ---- pack: sorted positions for the pair kernel -------------------------------
__global__ void k_pack_mixed(const double* __restrict__ pos, const double* __restrict__ chrg,
                             const int* __restrict__ perm, int n, const DynState* __restrict__ dyn,
                             int4* __restrict__ xq) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int i = perm[s];
    unsigned u[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double f = pos[3 * i + d] * dyn->boxinv[d];
        f -= floor(f);
        u[d] = (unsigned)(unsigned long long)(f * 4294967296.0);
    }
    xq[s] = make_int4((int)u[0], (int)u[1], (int)u[2], __float_as_int((float)chrg[i]));
}

__global__ void k_pack_fp64(const double* __restrict__ pos, const double* __restrict__ chrg,
                            const int* __restrict__ perm, int n, double4* __restrict__ xq) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int i = perm[s];
    xq[s] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], chrg[i]);
}

pgk_status launch_pack(pgk_ctx* c) {
    int n = c->natom;
    if (c->mixed())
        k_pack_mixed<<<(n + 255) / 256, 256, 0, c->st>>>(c->pos, c->chrg, c->perm, n, c->dyn, c->xq);
    else
        k_pack_fp64<<<(n + 255) / 256, 256, 0, c->st>>>(c->pos, c->chrg, c->perm, n, c->xq64);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// ---- pair kernel, mixed precision ------------------------------------------
struct PairArgs {
    const int* nbr; const int* ncnt; int cap; int n;
    const int* typ_s; const int* perm;
    int ntyp; int nspl; double h, inv_h;
    double rr2, rl2, rmax2, rrcut;
    void* facc; long long* acc;
};

template <bool ENE, bool VIR>
__device__ __forceinline__ void pair_term(const int4 pi, const float qi, const int ti, const int4 pj, const int tj,
                                          const float sx, const float sy, const float sz, const float rmax2,
                                          const float rr2, const float rl2, const float inv_h, const float h,
                                          const float4* __restrict__ sf, const float4* __restrict__ sp,
                                          const float2* __restrict__ slj, float& fx, float& fy, float& fz,
                                          float& ev, float& ee, float* wc, float* wl) {
    const float dx = (float)(pi.x - pj.x) * sx;
    const float dy = (float)(pi.y - pj.y) * sy;
    const float dz = (float)(pi.z - pj.z) * sz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (r2 > rmax2) return;
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    float fc = 0.f, fl = 0.f;
    if (r2 <= rr2) {
        const float r = r2 * rinv;
        const float qq = qi * __int_as_float(pj.w);
        const int idx = (int)(r * inv_h);
        const float d = fmaf(-(float)idx, h, r);
        const float4 c = sf[idx];
        fc = qq * fmaf(d, fmaf(d, fmaf(d, c.w, c.z), c.y), c.x);
        if (ENE || VIR) {
            const float4 p = sp[idx];
            ee = fmaf(qq, fmaf(d, fmaf(d, fmaf(d, p.w, p.z), p.y), p.x), ee);
        }
    }
    if (r2 <= rl2) {
        const float2 lp = slj[ti + tj];
        const float t2 = rinv2 * lp.x;
        const float t6 = t2 * t2 * t2;
        const float t12 = t6 * t6;
        fl = 12.f * lp.y * (t12 - t6) * rinv2;
        if (ENE || VIR) ev = fmaf(lp.y, t12 - 2.f * t6, ev);
    }
    const float fs = fc + fl;
    fx = fmaf(fs, dx, fx);
    fy = fmaf(fs, dy, fy);
    fz = fmaf(fs, dz, fz);
    if (VIR) {
        const float cx = fc * dx, cy = fc * dy, cz = fc * dz;
        wc[0] = fmaf(cx, dx, wc[0]); wc[1] = fmaf(cx, dy, wc[1]); wc[2] = fmaf(cx, dz, wc[2]);
        wc[3] = fmaf(cy, dy, wc[3]); wc[4] = fmaf(cy, dz, wc[4]); wc[5] = fmaf(cz, dz, wc[5]);
        const float lx = fl * dx, ly = fl * dy, lz = fl * dz;
        wl[0] = fmaf(lx, dx, wl[0]); wl[1] = fmaf(lx, dy, wl[1]); wl[2] = fmaf(lx, dz, wl[2]);
        wl[3] = fmaf(ly, dy, wl[3]); wl[4] = fmaf(ly, dz, wl[4]); wl[5] = fmaf(lz, dz, wl[5]);
    }
}

// Each lane walks entries lane, lane+32, ... of the row; the next entry's
// index, position and type are loaded before the current pair is evaluated
// (two gathers in flight per lane).  Per-lane energy/virial sums stay in
// FP32 registers across all atoms of the warp and are reduced once per block.
template <bool ENE, bool VIR>
__global__ void __launch_bounds__(256, 4) k_pair_mixed(const int4* __restrict__ xq, PairArgs a,
                                                       const float2* __restrict__ lj_g,
                                                       const float4* __restrict__ spl_g,
                                                       const DynState* __restrict__ dyn) {
    extern __shared__ float4 sm[];
    float4* sf = sm;                        // force table  (spline 0)
    float4* sp = sm + a.nspl;               // pot table    (spline 1), ENE/VIR only
    float2* slj = (float2*)(sm + (ENE || VIR ? 2 : 1) * a.nspl);
    for (int k = threadIdx.x; k < a.nspl; k += blockDim.x) {
        sf[k] = spl_g[k];
        if (ENE || VIR) sp[k] = spl_g[a.nspl + k];
    }
    for (int k = threadIdx.x; k < a.ntyp * a.ntyp; k += blockDim.x) slj[k] = lj_g[k];
    __syncthreads();

    const float sx = (float)(dyn->box[0] * (1.0 / 4294967296.0));
    const float sy = (float)(dyn->box[1] * (1.0 / 4294967296.0));
    const float sz = (float)(dyn->box[2] * (1.0 / 4294967296.0));
    const float rr2 = (float)a.rr2, rl2 = (float)a.rl2, rmax2 = (float)a.rmax2;
    const float inv_h = (float)a.inv_h, h = (float)a.h;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int* __restrict__ typ_s = a.typ_s;
    float ev = 0.f, ee = 0.f;
    float wc[6] = {0, 0, 0, 0, 0, 0}, wl[6] = {0, 0, 0, 0, 0, 0};

    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < a.n; s += nwarps) {
        const int4 pi = __ldg(xq + s);
        const float qi = __int_as_float(pi.w);
        const int ti = __ldg(typ_s + s) * a.ntyp;
        const int cnt = __ldg(a.ncnt + s);
        const int* __restrict__ row = a.nbr + (size_t)s * a.cap;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        int k = lane;
        int j = k < cnt ? __ldg(row + k) : s;
        int4 pj = __ldg(xq + j);
        int tj = __ldg(typ_s + j);
        while (k < cnt) {
            const int kn = k + 32;
            const int jn = kn < cnt ? __ldg(row + kn) : s;
            const int4 pjn = __ldg(xq + jn);
            const int tjn = __ldg(typ_s + jn);
            pair_term<ENE, VIR>(pi, qi, ti, pj, tj, sx, sy, sz, rmax2, rr2, rl2, inv_h, h, sf, sp, slj,
                                fx, fy, fz, ev, ee, wc, wl);
            k = kn; pj = pjn; tj = tjn;
        }
        fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
        if (lane == 0) force_add<true>(a.facc, a.perm[s], (double)fx, (double)fy, (double)fz);
    }
    if (ENE || VIR) {
        // pairs were counted from both sides: factor 1/2.  Tensor (a,b) -> 3*b + a.
        double v[16] = {0.5 * ev, 0.5 * ee, 0.5 * ee,
                        0.5 * wc[0], 0.5 * wc[1], 0.5 * wc[2], 0.5 * wc[3], 0.5 * wc[4], 0.5 * wc[5],
                        0.5 * wl[0], 0.5 * wl[1], 0.5 * wl[2], 0.5 * wl[3], 0.5 * wl[4], 0.5 * wl[5],
                        0.5 * ((double)wl[0] + (double)wl[3] + (double)wl[5])};
        if (VIR) {
            const int idx[16] = {A_VDW, A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8,
                                 A_VTLJ + 0, A_VTLJ + 1, A_VTLJ + 2, A_VTLJ + 4, A_VTLJ + 5, A_VTLJ + 8, A_VLJ};
            block_acc<16>(v, a.acc, idx, false);
        } else {
            double v2[2] = {v[0], v[1]};
            const int idx[2] = {A_VDW, A_ELC};
            block_acc<2>(v2, a.acc, idx, false);
        }
    }
}

// ---- pair kernel, FP64 (parity path) ---------------------------------------
template <bool ENE, bool VIR>
__global__ void __launch_bounds__(256, 2) k_pair_fp64(const double4* __restrict__ xq, PairArgs a,
                                                      const double2* __restrict__ lj_g,
                                                      const double4* __restrict__ spl_g,
                                                      const DynState* __restrict__ dyn) {
    extern __shared__ double4 smd[];
    double4* sf = smd;
    double4* sp = smd + a.nspl;
    double2* slj = (double2*)(smd + 2 * a.nspl);
    for (int k = threadIdx.x; k < a.nspl; k += blockDim.x) { sf[k] = spl_g[k]; sp[k] = spl_g[a.nspl + k]; }
    for (int k = threadIdx.x; k < a.ntyp * a.ntyp; k += blockDim.x) slj[k] = lj_g[k];
    __syncthreads();
    const double L0 = dyn->box[0], L1 = dyn->box[1], L2 = dyn->box[2];
    const double B0 = 1.0 / L0, B1 = 1.0 / L1, B2 = 1.0 / L2;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double e_vdw = 0, e_elc = 0, vc[6] = {0, 0, 0, 0, 0, 0}, vl[6] = {0, 0, 0, 0, 0, 0};
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < a.n; s += nwarps) {
        const double4 pi = xq[s];
        const int ti = a.typ_s[s] * a.ntyp;
        const int cnt = a.ncnt[s];
        const int* row = a.nbr + (size_t)s * a.cap;
        double fx = 0, fy = 0, fz = 0;
        for (int k = lane; k < cnt; k += 32) {
            const int j = __ldg(row + k);
            const double4 pj = xq[j];
            double dx = pi.x - pj.x; dx = dx - L0 * round(dx * B0);
            double dy = pi.y - pj.y; dy = dy - L1 * round(dy * B1);
            double dz = pi.z - pj.z; dz = dz - L2 * round(dz * B2);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > a.rmax2) continue;
            const double rinv2 = 1.0 / r2;
            double fc = 0, fl = 0;
            const double r = sqrt(r2);
            if (r <= a.rrcut) {
                const double qq = pi.w * pj.w;
                const int idx = (int)(r / a.h);
                const double d = r - (double)idx * a.h;
                const double4 c = sf[idx];
                fc = (c.x + d * (c.y + d * (c.z + d * c.w))) * qq;
                if (ENE || VIR) {
                    const double4 p = sp[idx];
                    e_elc += 0.5 * ((p.x + d * (p.y + d * (p.z + d * p.w))) * qq);
                }
            }
            if (r2 <= a.rl2) {
                const double2 lp = slj[ti + a.typ_s[j]];
                const double t2 = rinv2 * lp.x;
                const double t6 = t2 * t2 * t2, t12 = t6 * t6;
                fl = 12.0 * lp.y * (t12 - t6) * rinv2;
                if (ENE || VIR) e_vdw += 0.5 * (lp.y * (t12 - 2.0 * t6));
            }
            fx += fc * dx + fl * dx;
            fy += fc * dy + fl * dy;
            fz += fc * dz + fl * dz;
            if (VIR) {
                vc[0] += fc * dx * dx; vc[1] += fc * dx * dy; vc[2] += fc * dx * dz;
                vc[3] += fc * dy * dy; vc[4] += fc * dy * dz; vc[5] += fc * dz * dz;
                vl[0] += fl * dx * dx; vl[1] += fl * dx * dy; vl[2] += fl * dx * dz;
                vl[3] += fl * dy * dy; vl[4] += fl * dy * dz; vl[5] += fl * dz * dz;
            }
        }
        fx = warp_sum(fx); fy = warp_sum(fy); fz = warp_sum(fz);
        if (lane == 0) force_add<false>(a.facc, a.perm[s], fx, fy, fz);
    }
    if (ENE || VIR) {
        double v[16] = {e_vdw, e_elc, e_elc,
                        0.5 * vc[0], 0.5 * vc[1], 0.5 * vc[2], 0.5 * vc[3], 0.5 * vc[4], 0.5 * vc[5],
                        0.5 * vl[0], 0.5 * vl[1], 0.5 * vl[2], 0.5 * vl[3], 0.5 * vl[4], 0.5 * vl[5],
                        0.5 * (vl[0] + vl[3] + vl[5])};
        const int idx[16] = {A_VDW, A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8,
                             A_VTLJ + 0, A_VTLJ + 1, A_VTLJ + 2, A_VTLJ + 4, A_VTLJ + 5, A_VTLJ + 8, A_VLJ};
        block_acc<16>(v, a.acc, idx, true);
    }
}

pgk_status launch_pair(pgk_ctx* c, int group, bool ene, bool vir) {
    PairArgs a;
    a.nbr = c->nbr; a.ncnt = c->ncnt; a.cap = c->cap; a.n = c->natom;
    a.typ_s = c->typ_s; a.perm = c->perm; a.ntyp = c->ntyp; a.nspl = c->nspl;
    a.h = c->hspl; a.inv_h = 1.0 / c->hspl;
    a.rrcut = c->prm.rrcut;
    a.rr2 = c->prm.rrcut * c->prm.rrcut;
    a.rl2 = c->prm.rcut * c->prm.rcut;
    a.rmax2 = a.rr2 > a.rl2 ? a.rr2 : a.rl2;
    a.facc = c->facc[group];
    a.acc = c->acc + (size_t)group * NACC;
    int warps_per_block = 8;
    int blocks = c->nsm * 4;
    long long need = (c->natom + warps_per_block - 1) / warps_per_block;
    if (blocks > need) blocks = (int)need;
    if (blocks < 1) blocks = 1;
    if (c->mixed()) {
        size_t sm = (size_t)((ene || vir) ? 2 : 1) * c->nspl * sizeof(float4) + c->ntyp * c->ntyp * sizeof(float2);
        if (vir) {
            cudaFuncSetAttribute(k_pair_mixed<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_pair_mixed<true, true><<<blocks, 256, sm, c->st>>>(c->xq, a, c->lj32, c->spl32, c->dyn);
        } else if (ene) {
            cudaFuncSetAttribute(k_pair_mixed<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_pair_mixed<true, false><<<blocks, 256, sm, c->st>>>(c->xq, a, c->lj32, c->spl32, c->dyn);
        } else {
            cudaFuncSetAttribute(k_pair_mixed<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_pair_mixed<false, false><<<blocks, 256, sm, c->st>>>(c->xq, a, c->lj32, c->spl32, c->dyn);
        }
    } else {
        size_t sm = (size_t)2 * c->nspl * sizeof(double4) + c->ntyp * c->ntyp * sizeof(double2);
        if (vir || ene) {
            cudaFuncSetAttribute(k_pair_fp64<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_pair_fp64<true, true><<<blocks, 256, sm, c->st>>>(c->xq64, a, c->lj64, c->spl64, c->dyn);
        } else {
            cudaFuncSetAttribute(k_pair_fp64<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_pair_fp64<false, false><<<blocks, 256, sm, c->st>>>(c->xq64, a, c->lj64, c->spl64, c->dyn);
        }
    }
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// ---- excluded-pair correction (ewaldr.F90:756-826): thread per pair -------------
template <bool MIXED>
__global__ void k_excl(const double* __restrict__ pos, const double* __restrict__ chrg,
                       const int2* __restrict__ pairs, int npair, const double4* __restrict__ spl64,
                       const float4* __restrict__ spl32, int nspl, double h, const DynState* __restrict__ dyn,
                       void* facc, long long* acc, int want) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, t[6] = {0, 0, 0, 0, 0, 0};
    if (k < npair) {
        int i = pairs[k].x, j = pairs[k].y;
        double r[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v = pos[3 * i + d] - pos[3 * j + d];
            r[d] = v - dyn->box[d] * round(v * dyn->boxinv[d]);
        }
        double qq = chrg[i] * chrg[j];
        double fx, fy, fz, pot = 0.0;
        if (MIXED) {
            float rx = (float)r[0], ry = (float)r[1], rz = (float)r[2];
            float rr = sqrtf(rx * rx + ry * ry + rz * rz);
            float hf = (float)h;
            int idx = (int)(rr / hf);
            float fs = 0.f, ps = 0.f;
            if (idx < nspl - 1) {
                float d = rr - (float)idx * hf;
                float4 c = spl32[2 * nspl + idx];
                fs = -(c.x + d * (c.y + d * (c.z + d * c.w))) * (float)qq;
                float4 p = spl32[3 * nspl + idx];
                ps = (p.x + d * (p.y + d * (p.z + d * p.w))) * (float)qq;
            }
            fx = (double)(fs * rx); fy = (double)(fs * ry); fz = (double)(fs * rz);
            pot = ps;
        } else {
            double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            double fs = 0.0;
            if (rr < h * (double)(nspl - 1)) {
                int idx = (int)(rr / h);
                double d = rr - (double)idx * h;
                double4 c = spl64[2 * nspl + idx];
                fs = -(c.x + d * (c.y + d * (c.z + d * c.w))) * qq;
                double4 p = spl64[3 * nspl + idx];
                pot = (p.x + d * (p.y + d * (p.z + d * p.w))) * qq;
            }
            fx = fs * r[0]; fy = fs * r[1]; fz = fs * r[2];
        }
        force_add<MIXED>(facc, i, fx, fy, fz);
        force_add<MIXED>(facc, j, -fx, -fy, -fz);
        e = pot;
        t[0] = fx * r[0]; t[1] = fx * r[1]; t[2] = fx * r[2];
        t[3] = fy * r[1]; t[4] = fy * r[2]; t[5] = fz * r[2];
    }
    if (want) {
        double v[8] = {-e, -e, t[0], t[1], t[2], t[3], t[4], t[5]};
        const int idx[8] = {A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
        block_acc<8>(v, acc, idx, !MIXED);
    }
}

pgk_status launch_excl(pgk_ctx* c, int group, bool ene, bool vir) {
    if (c->nexpair == 0) return PGK_OK;
    int nb = (c->nexpair + 255) / 256;
    long long* acc = c->acc + (size_t)group * NACC;
    if (c->mixed())
        k_excl<true><<<nb, 256, 0, c->st>>>(c->pos, c->chrg, c->expair, c->nexpair, c->spl64, c->spl32, c->nspl,
                                            c->hspl, c->dyn, c->facc[group], acc, ene || vir);
    else
        k_excl<false><<<nb, 256, 0, c->st>>>(c->pos, c->chrg, c->expair, c->nexpair, c->spl64, c->spl32, c->nspl,
                                             c->hspl, c->dyn, c->facc[group], acc, ene || vir);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// ---- diagnostic: number of unique pairs inside the interaction cutoff --------
// (the algorithmic work unit of the pair kernel; run outside any timed region)
__global__ void k_count_pairs(const double* __restrict__ pos_s, const int* __restrict__ nbr,
                              const int* __restrict__ ncnt, int cap, int n, double rmax2,
                              const DynState* __restrict__ dyn, unsigned long long* out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    unsigned long long c = 0;
    const double L0 = dyn->box[0], L1 = dyn->box[1], L2 = dyn->box[2];
    for (int k = 0; k < ncnt[s]; ++k) {
        int t = nbr[(size_t)s * cap + k];
        if (t <= s) continue;
        double dx = pos_s[3 * s] - pos_s[3 * t]; dx -= L0 * round(dx / L0);
        double dy = pos_s[3 * s + 1] - pos_s[3 * t + 1]; dy -= L1 * round(dy / L1);
        double dz = pos_s[3 * s + 2] - pos_s[3 * t + 2]; dz -= L2 * round(dz / L2);
        if (dx * dx + dy * dy + dz * dz <= rmax2) ++c;
    }
    atomicAdd(out, c);
}

pgk_status count_pairs(pgk_ctx* c, long long* npair, long long* nentries) {
    unsigned long long* d = c->counters + 2;
    PGK_CUDA(c, cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->st));
    double rr2 = c->prm.rrcut * c->prm.rrcut, rl2 = c->prm.rcut * c->prm.rcut;
    k_count_pairs<<<(c->natom + 255) / 256, 256, 0, c->st>>>(c->pos_s, c->nbr, c->ncnt, c->cap, c->natom,
                                                              rr2 > rl2 ? rr2 : rl2, c->dyn, d);
    PGK_CUDA(c, cudaGetLastError());
    unsigned long long h = 0;
    PGK_CUDA(c, cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->st));
    std::vector<int> cnt(c->natom);
    PGK_CUDA(c, cudaMemcpyAsync(cnt.data(), c->ncnt, sizeof(int) * c->natom, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    long long e = 0;
    for (int v : cnt) e += v;
    *npair = (long long)h;
    *nentries = e;
    return PGK_OK;
}
