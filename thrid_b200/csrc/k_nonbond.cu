// k_nonbond.cu -- real-space LJ + Ewald pair kernel (ewaldrp, ewaldr.F90:404-838)
//
// Work decomposition: one warp per 8-atom i-cluster of the cell-sorted order.
// The cluster's row holds entries (mask << 24 | j); bit b of the mask says
// that (cluster atom b, j) is a list pair, and every pair is stored once (in
// the row of its lower slot).  One gather of j serves up to 8 pairs, and the
// index stream is one 4-byte entry per (cluster, j) instead of one per pair.
// Each evaluation serves both atoms (Newton's third law): the cluster atoms'
// forces are register sums closed by warp shuffles, j's force is summed over
// the entry's bits and added once per entry.  In mixed precision all force
// sums are int64 fixed point, so the integer atomics on j are exact and the
// result does not depend on their order.
//
// Mixed precision: positions enter as 32-bit fractional fixed point per box
// axis (x/L * 2^32); the wrapped integer difference is the minimum-image
// displacement, converted to FP32 with the box scale.  The displacement error
// is ~L/2^32 (3e-8 A at L = 130 A) instead of the 8e-6 A of FP32 absolute
// coordinates.  Pair arithmetic is FP32 with the reference's natural cubic
// spline tables (spline_interp.F90) staged in shared memory; each atom's
// force is converted once to int64 fixed point (2^32) and added to the group
// accumulator.  FP64 precision runs the same structure in double with the
// reference's dnint minimum image.
//
// Roofline: FP32 pipe (61 algorithmic flop per interacting pair) plus one
// 4-byte entry, one 16-byte (32-byte FP64) position and one 4-byte type
// gather per (cluster, j) entry.
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pgk_ctx.cuh"

// Mixed pair kernel launch shapes, one wave of nsm * blocks-per-SM blocks.
// Packed cluster-frame body: 128-thread blocks, five resident per SM (its ~94
// registers); smaller blocks stage the spline table more often than they
// gain, larger ones finish their fixed cluster chunks less evenly.  Scalar
// body: 256-thread blocks, three per SM (80 registers).
constexpr int pair_threads(bool frame) { return frame ? 128 : 256; }
constexpr int pair_minb(bool frame) { return frame ? 5 : 3; }
constexpr int PAIR_WARPS = 8;                      // shared-memory rows per block (the larger shape)

// ---- pack: sorted (padded) positions for the pair kernel ---------------------
__global__ void k_pack_mixed(const double* __restrict__ pos, const double* __restrict__ chrg,
                             const int* __restrict__ perm, int npad, const DynState* __restrict__ dyn,
                             int4* __restrict__ xq, const int4* __restrict__ xq_prune, PruneDev* __restrict__ P) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = s < npad ? perm[s] : -1;
    int4 v = make_int4(0, 0, 0, 0);
    if (i >= 0) {
        unsigned u[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double f = pos[3 * i + d] * dyn->boxinv[d];
            f -= floor(f);
            u[d] = (unsigned)(unsigned long long)(f * 4294967296.0);
        }
        v = make_int4((int)u[0], (int)u[1], (int)u[2], __float_as_int((float)chrg[i]));
    }
    if (s < npad) xq[s] = v;
    if (P) {
        // displacement since the last prune (minimum image, current box)
        float dd = 0.f;
        if (i >= 0) {
            const int4 o = xq_prune[s];
            const float dx = (float)(v.x - o.x) * (float)(dyn->box[0] * (1.0 / 4294967296.0));
            const float dy = (float)(v.y - o.y) * (float)(dyn->box[1] * (1.0 / 4294967296.0));
            const float dz = (float)(v.z - o.z) * (float)(dyn->box[2] * (1.0 / 4294967296.0));
            dd = sqrtf(dx * dx + dy * dy + dz * dz);
        }
        const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(dd));
        if ((threadIdx.x & 31) == 0 && m) atomicMax(&P->dmax, m);
    }
}

__global__ void k_pack_fp64(const double* __restrict__ pos, const double* __restrict__ chrg,
                            const int* __restrict__ perm, int npad, double4* __restrict__ xq) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npad) return;
    int i = perm[s];
    xq[s] = i < 0 ? make_double4(0, 0, 0, 0) : make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], chrg[i]);
}

pgk_status launch_pack(pgk_ctx* c) {
    int n = c->npad;
    if (n <= 0) return PGK_OK;
    if (c->mixed())
        k_pack_mixed<<<(n + 255) / 256, 256, 0, c->st>>>(c->pos, c->chrg, c->perm, n, c->dyn, c->xq, c->xq_prune,
                                                          c->prune_buffer > 0.f ? c->prune : nullptr);
    else
        k_pack_fp64<<<(n + 255) / 256, 256, 0, c->st>>>(c->pos, c->chrg, c->perm, n, c->xq64);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

struct PairArgs {
    const int* clist; const int* ccnt; int ccap; int ncl;
    const int* typ_s; const int* perm;
    int ntyp; int nspl; double h, inv_h;
    double rr2, rl2, rmax2, rrcut;
    // FP32 copies for the mixed kernel, read straight from the parameter
    // bank inside the pair loop (no registers held for them)
    float rr2f, rl2f, inv_hf, hf; int nsplm1;
    float ew_pa, ew_c2a, ew_mk;        // analytic real-space Ewald (EwaldF)
    void* facc; long long* acc;
    long long* fsort; int fstride;     // mixed: forces by sorted slot (SoA, stride fstride)
    // pruned rows (mixed; P null = none): on a prune step (P->do_prune) the
    // kernel reads the book rows (blist/bcnt), writes each entry's pairs inside
    // rprune (rp2) compacted into plist/pcnt and the new displacement origin
    // xq_prune; otherwise it reads plist/pcnt
    const PruneDev* P; const int* blist; const int* bcnt; int* plist; int* pcnt; int4* xq_prune; float rp2;
};

// ---- real-space Ewald force without a table (mixed precision) -----------------
// The screened Coulomb force per unit charge product, divided by r,
//   erfc(a r)/r^3 + (2a/sqrt(pi)) exp(-a^2 r^2)/r^2   (a = alpha),
// with erfc(x) = t (c1 + t (c2 + t (c3 + t (c4 + t c5)))) exp(-x^2) and
// t = 1/(1 + p x): Hastings' rational approximation as given in Abramowitz &
// Stegun, Handbook of Mathematical Functions, 7.1.26 (absolute error of erfc
// <= 1.5e-7).  Evaluated in FP32 (rcp, ex2 on the MUFU unit), the force is
// within 6e-7 of the FP64 value on the scale of the bare Coulomb force 1/r^2
// for 0.8 <= r <= 14 A and 0.28 <= a <= 0.40; where erfc(a r) is small the
// pair force is small too.  The packed cluster-frame body uses it instead of
// the spline-table fetch of the force, whose random rows cost shared-memory
// bank conflicts in every evaluation (0.358 -> 0.300 ms per evaluation on the
// 200k butane rows); the reference's spline tables (spline_interp.F90) still
// give the Coulomb energy on the steps that need energies, the force of the
// scalar body (small boxes, where the table measured faster) and the FP64
// path.
struct EwaldF { float pa, c2a, mk; };      // p a, 2a/sqrt(pi), -a^2 log2(e)
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
#define AS_P 0.3275911f
#define AS_C1 0.254829592f
#define AS_C2 -0.284496736f
#define AS_C3 1.421413741f
#define AS_C4 -1.453152027f
#define AS_C5 1.061405429f
__device__ __forceinline__ float2 ewald_force2(float2 r, float2 r2, float2 rinv, float2 rinv2, const EwaldF& ew) {
    const float2 den = __ffma2_rn(r, make_float2(ew.pa, ew.pa), make_float2(1.f, 1.f));
    const float2 t = make_float2(rcp_ftz(den.x), rcp_ftz(den.y));
    float2 poly = __ffma2_rn(t, make_float2(AS_C5, AS_C5), make_float2(AS_C4, AS_C4));
    poly = __ffma2_rn(poly, t, make_float2(AS_C3, AS_C3));
    poly = __ffma2_rn(poly, t, make_float2(AS_C2, AS_C2));
    poly = __ffma2_rn(poly, t, make_float2(AS_C1, AS_C1));
    poly = __fmul2_rn(poly, t);
    const float2 xa = __fmul2_rn(r2, make_float2(ew.mk, ew.mk));
    const float2 ex = make_float2(ex2_ftz(xa.x), ex2_ftz(xa.y));
    const float2 ec = __fmul2_rn(poly, ex);
    return __fmul2_rn(__ffma2_rn(ec, rinv, __fmul2_rn(make_float2(ew.c2a, ew.c2a), ex)), rinv2);
}

// ---- one pair, mixed precision -----------------------------------------------
// Branch-free: every pair of an entry's mask is evaluated to the end and the
// cutoffs select zero (the spline index is clamped into the table), so the
// lanes of a warp never diverge inside the pair arithmetic.  The force on
// cluster atom fi and the opposite force on j (g) accumulate directly.
// (dx, dy, dz) = x_i - x_j (minimum image), qq = q_i q_j, tij = LJ table row
// of the pair.  PAIRVIR: the tensor-only virial is summed per pair here (else
// the caller forms it from the atom forces in the cluster frame).
template <int MODE, bool PAIRVIR>
__device__ __forceinline__ void pair_term(const float dx, const float dy, const float dz, const float qq,
                                          const int tij, const float rr2, const float rl2, const float inv_h,
                                          const float h, const int nsplm1, const float4* __restrict__ sf,
                                          const float4* __restrict__ sp, const float2* __restrict__ slj,
                                          float (&fi)[3], float& gx, float& gy, float& gz, float& ev, float& ee,
                                          float* wc, float* wl, float& r2o) {
    constexpr bool ENE = MODE == PM_ENE || MODE == PM_FULL;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    r2o = r2;
    const float rinv = rsqrt_ftz(r2);
    const float rinv2 = rinv * rinv;
    const float r = r2 * rinv;
    // floor(r/h) on the FP32/ALU pipes: adding 2^23 rounded toward -inf
    // leaves floor(r/h) in the low mantissa bits (exact for r/h < 2^23)
    const float tf = r * inv_h;
    const float fb = __fadd_rd(tf, 8388608.0f);
    const float fm = fb - 8388608.0f;
    int idx = __float_as_int(fb) - 0x4B000000;
    idx = (int)min((unsigned)idx, (unsigned)nsplm1);      // into the table whatever r is (NaN included)
    const float d = fmaf(-fm, h, r);
    const float4 c = sf[idx];
    const bool inr = r2 <= rr2, inl = r2 <= rl2;
    float fc = qq * fmaf(d, fmaf(d, fmaf(d, c.w, c.z), c.y), c.x);
    fc = inr ? fc : 0.f;
    if (ENE) {
        const float4 p = sp[idx];
        const float pe = qq * fmaf(d, fmaf(d, fmaf(d, p.w, p.z), p.y), p.x);
        ee += inr ? pe : 0.f;
    }
    const float2 lp = slj[tij];
    const float t2 = rinv2 * lp.x;
    const float t6 = t2 * t2 * t2;
    const float t12 = t6 * t6;
    float fl = 12.f * lp.y * (t12 - t6) * rinv2;
    fl = inl ? fl : 0.f;
    if (ENE) ev += inl ? lp.y * (t12 - 2.f * t6) : 0.f;
    const float fs = fc + fl;
    const float cx = fs * dx, cy = fs * dy, cz = fs * dz;
    fi[0] += cx; fi[1] += cy; fi[2] += cz;
    gx -= cx; gy -= cy; gz -= cz;
    if (MODE == PM_TENS && PAIRVIR) {
        wc[0] = fmaf(cx, dx, wc[0]); wc[1] = fmaf(cx, dy, wc[1]); wc[2] = fmaf(cx, dz, wc[2]);
        wc[3] = fmaf(cy, dy, wc[3]); wc[4] = fmaf(cy, dz, wc[4]); wc[5] = fmaf(cz, dz, wc[5]);
    }
    if (MODE == PM_FULL) {
        const float ax = fc * dx, ay = fc * dy, az = fc * dz;
        wc[0] = fmaf(ax, dx, wc[0]); wc[1] = fmaf(ax, dy, wc[1]); wc[2] = fmaf(ax, dz, wc[2]);
        wc[3] = fmaf(ay, dy, wc[3]); wc[4] = fmaf(ay, dz, wc[4]); wc[5] = fmaf(az, dz, wc[5]);
        const float lx = fl * dx, ly = fl * dy, lz = fl * dz;
        wl[0] = fmaf(lx, dx, wl[0]); wl[1] = fmaf(lx, dy, wl[1]); wl[2] = fmaf(lx, dz, wl[2]);
        wl[3] = fmaf(ly, dy, wl[3]); wl[4] = fmaf(ly, dz, wl[4]); wl[5] = fmaf(lz, dz, wl[5]);
    }
}

// MODE: PM_FORCE forces only; PM_ENE + pot_vdw, pot_elc; PM_TENS + the
// combined (Coulomb + LJ) virial tensor only (what the anisotropic MTK
// barostat reads every step: diag(pintt)); PM_FULL + energies, split tensors
// and the scalar virials of ewaldrp.
//
// Each lane walks entries lane, lane+32, ... of the cluster's row; for each
// entry it evaluates the pairs with the cluster atoms whose mask bit is set
// (cluster atoms in shared memory).  Every pair is stored once, so each
// evaluation serves both atoms: the force on cluster atom ii accumulates in
// registers (closed by warp shuffles after the row), the opposite force on j
// accumulates over the entry's bits and is added once per entry to j's int64
// fixed-point accumulator -- integer atomics, so the sum is exact and
// independent of their order.  The next entry and its j record are loaded
// before the current entry's pairs are evaluated.
//
// Block b owns the contiguous cluster range [b*chunk, (b+1)*chunk); its
// warps take every 8th cluster of it, so they read overlapping j ranges at
// the same time (shared L1 lines).  Per-lane energy/virial sums stay in FP32
// registers across the block's clusters and are reduced once per block.
// PRUNE: the body of prune steps (reads the book rows, writes the pruned
// ones); the other body runs on all other steps (one launch, see k_pair_mixed).
// This body serves boxes in which a pair needs its own minimum image; wider
// boxes run the packed cluster-frame body (pair_mixed_body_x2).
template <int MODE, bool PRUNE>
__device__ __forceinline__ void pair_mixed_body(const int4* __restrict__ xq, const PairArgs& a,
                                                const float2* __restrict__ lj_g, const float4* __restrict__ spl_g,
                                                const DynState* __restrict__ dyn) {
    constexpr bool ENE = MODE == PM_ENE || MODE == PM_FULL;
    extern __shared__ float4 sm[];
    float4* sf = sm;                        // force table  (spline 0)
    float4* sp = sm + a.nspl;               // energy table (spline 1), ENE only
    float2* slj = (float2*)(sm + (ENE ? 2 : 1) * a.nspl);
    __shared__ int4 si[PAIR_WARPS][8];
    __shared__ int sti[PAIR_WARPS][8];
    for (int k = threadIdx.x; k < a.nspl; k += blockDim.x) {
        sf[k] = spl_g[k];
        if (ENE) sp[k] = spl_g[a.nspl + k];
    }
    for (int k = threadIdx.x; k < a.ntyp * a.ntyp; k += blockDim.x) slj[k] = lj_g[k];
    __syncthreads();

    const float sx = (float)(dyn->box[0] * (1.0 / 4294967296.0));
    const float sy = (float)(dyn->box[1] * (1.0 / 4294967296.0));
    const float sz = (float)(dyn->box[2] * (1.0 / 4294967296.0));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int chunk = (a.ncl + gridDim.x - 1) / gridDim.x;
    const int c_end = min(a.ncl, (blockIdx.x + 1) * chunk);
    const int* __restrict__ typ_s = a.typ_s;
    long long* __restrict__ fs0 = a.fsort;
    const int fst = a.fstride;
    float ev = 0.f, ee = 0.f;
    float wc[6] = {0, 0, 0, 0, 0, 0}, wl[6] = {0, 0, 0, 0, 0, 0};

    const bool prune = PRUNE;
    const int* __restrict__ rows = prune ? a.blist : a.clist;
    const int* __restrict__ rcnt = prune ? a.bcnt : a.ccnt;
    const float rp2 = a.rp2;

    for (int cl = blockIdx.x * chunk + warp; cl < c_end; cl += wpb) {
        __syncwarp();
        if (lane < 8) {
            const int4 v = __ldg(xq + 8 * cl + lane);
            si[warp][lane] = v;
            sti[warp][lane] = __ldg(typ_s + 8 * cl + lane) * a.ntyp;
            if (prune) a.xq_prune[8 * cl + lane] = v;
        }
        __syncwarp();
        const int cnt = __ldg(rcnt + cl);
        const int* __restrict__ row = rows + (size_t)cl * a.ccap;
        int* __restrict__ prow = a.plist + (size_t)cl * a.ccap;
        int pcount = 0;
        float f[8][3];
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) { f[ii][0] = 0.f; f[ii][1] = 0.f; f[ii][2] = 0.f; }
        // two-deep prefetch: entries two iterations ahead, their j records one
        // ahead, so no gather waits on the entry load it depends on
        unsigned e = lane < cnt ? (unsigned)__ldg(row + lane) : 0u;
        unsigned e1 = 32 + lane < cnt ? (unsigned)__ldg(row + 32 + lane) : 0u;
        int4 pj = __ldg(xq + (e & 0xFFFFFFu));
        int tj = __ldg(typ_s + (e & 0xFFFFFFu));
        for (int k0 = 0; k0 < cnt; k0 += 32) {          // warp-uniform trip count
            const int kn = k0 + 64 + lane;
            const unsigned e2 = kn < cnt ? (unsigned)__ldg(row + kn) : 0u;
            const int4 pjn = __ldg(xq + (e1 & 0xFFFFFFu));
            const int tjn = __ldg(typ_s + (e1 & 0xFFFFFFu));
            const unsigned m = e >> 24;
            const int sj = e & 0xFFFFFFu;
            float gx = 0.f, gy = 0.f, gz = 0.f;
            unsigned nm = 0;
#pragma unroll
            for (int ii = 0; ii < 8; ++ii)
                if ((m >> ii) & 1u) {
                    const int4 pi = si[warp][ii];
                    const float dx = (float)(pi.x - pj.x) * sx, dy = (float)(pi.y - pj.y) * sy;
                    const float dz = (float)(pi.z - pj.z) * sz;
                    const float qq = __int_as_float(pi.w) * __int_as_float(pj.w);
                    float r2;
                    pair_term<MODE, true>(dx, dy, dz, qq, sti[warp][ii] + tj, a.rr2f, a.rl2f, a.inv_hf, a.hf,
                                          a.nsplm1, sf, sp, slj, f[ii], gx, gy, gz, ev, ee, wc, wl, r2);
                    if (PRUNE) nm |= r2 < rp2 ? 1u << ii : 0u;
                }
            if (m) {
                unsigned long long* fj = (unsigned long long*)fs0 + sj;
                atomicAdd(fj, (unsigned long long)__float2ll_rn(gx * (float)PGK_FORCE_SCALE));
                atomicAdd(fj + fst, (unsigned long long)__float2ll_rn(gy * (float)PGK_FORCE_SCALE));
                atomicAdd(fj + 2 * fst, (unsigned long long)__float2ll_rn(gz * (float)PGK_FORCE_SCALE));
            }
            if (prune) {       // compact the entries that keep a pair inside rprune
                const unsigned b = __ballot_sync(0xffffffffu, nm != 0);
                if (nm) prow[pcount + __popc(b & ((1u << lane) - 1u))] = (int)((nm << 24) | (unsigned)sj);
                pcount += __popc(b);
            }
            e = e1; e1 = e2; pj = pjn; tj = tjn;
        }
        if (prune && lane == 0) a.pcnt[cl] = pcount;
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const float fx = warp_sum(f[ii][0]), fy = warp_sum(f[ii][1]), fz = warp_sum(f[ii][2]);
            if (lane == ii) {     // padding slots get zero sums (no mask bits)
                unsigned long long* fi = (unsigned long long*)fs0 + 8 * cl + ii;
                atomicAdd(fi, (unsigned long long)__double2ll_rn((double)fx * PGK_FORCE_SCALE));
                atomicAdd(fi + fst, (unsigned long long)__double2ll_rn((double)fy * PGK_FORCE_SCALE));
                atomicAdd(fi + 2 * fst, (unsigned long long)__double2ll_rn((double)fz * PGK_FORCE_SCALE));
            }
        }
    }
    // every pair evaluated once.  Tensor (a,b) -> 3*b + a, stored as its lower triangle.
    if (MODE == PM_FULL) {
        double v[16] = {ev, ee, ee, wc[0], wc[1], wc[2], wc[3], wc[4], wc[5],
                        wl[0], wl[1], wl[2], wl[3], wl[4], wl[5], (double)wl[0] + (double)wl[3] + (double)wl[5]};
        const int idx[16] = {A_VDW, A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8,
                             A_VTLJ + 0, A_VTLJ + 1, A_VTLJ + 2, A_VTLJ + 4, A_VTLJ + 5, A_VTLJ + 8, A_VLJ};
        block_acc<16>(v, a.acc, idx, false);
    } else if (MODE == PM_TENS) {
        double v[6] = {wc[0], wc[1], wc[2], wc[3], wc[4], wc[5]};
        const int idx[6] = {A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
        block_acc<6>(v, a.acc, idx, false);
    } else if (MODE == PM_ENE) {
        double v[2] = {ev, ee};
        const int idx[2] = {A_VDW, A_ELC};
        block_acc<2>(v, a.acc, idx, false);
    }
}

// ---- packed (FP32x2) pair arithmetic for the cluster frame -------------------
// The cluster's 8 atoms are taken as 4 pairs (2p, 2p+1); one packed operation
// (fma/add/mul.f32x2, sm_100) evaluates both atoms of a pair against the
// lane's j, so the arithmetic of two list pairs issues as one instruction.
// Only the spline and LJ table fetches, the reciprocal square root and the
// cutoff selects stay per element.  `mb` holds the entry's two mask bits for
// the pair: an element whose bit is clear, or that lies beyond its cutoff,
// contributes zero (same cutoffs and zero rules as pair_term).  SC: the LJ
// and Coulomb cutoffs are equal (one select per element).  L holds the LJ
// parameters of both atoms with j's type as (R_a^2, R_b^2, 12 eps_a,
// 12 eps_b): fl = 12 eps (R^2/r^2)^3 ((R^2/r^2)^3 - 1) / r^2, and the LJ
// energy 12 eps t6 (t6 - 2) is divided by 12 once per block.
template <int MODE, bool SC>
__device__ __forceinline__ void pair_term_x2(const float2 dx, const float2 dy, const float2 dz, const float2 qq,
                                             const float4 L, const unsigned mb, const float rr2,
                                             const float rl2, const float2 inv_h2, const float2 mh2,
                                             const int nsplm1, const EwaldF& ew,
                                             const float4* __restrict__ sp,
                                             float2 (&fi)[3], float2& gx, float2& gy, float2& gz, float2& ev,
                                             float2& ee, float2* wc, float2* wl, float2& r2o) {
    constexpr bool ENE = MODE == PM_ENE || MODE == PM_FULL;
    const float2 two23 = make_float2(8388608.0f, 8388608.0f), mtwo23 = make_float2(-8388608.0f, -8388608.0f);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    r2o = r2;
    const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    const float2 rinv2 = __fmul2_rn(rinv, rinv);
    const float2 r = __fmul2_rn(r2, rinv);
    float2 fc = __fmul2_rn(qq, ewald_force2(r, r2, rinv, rinv2, ew));
    const float2 c12 = make_float2(L.z, L.w);
    const float2 t2 = __fmul2_rn(rinv2, make_float2(L.x, L.y));
    const float2 t6 = __fmul2_rn(__fmul2_rn(t2, t2), t2);
    const float2 w = __fmul2_rn(__fmul2_rn(t6, __fadd2_rn(t6, make_float2(-1.f, -1.f))), rinv2);
    float2 fl = __fmul2_rn(c12, w);
    const bool ba = mb & 1u, bb = mb & 2u;
    const bool ra = ba && r2.x <= rr2, rb = bb && r2.y <= rr2;
    float2 fs;
    if (SC) {
        fs = __fadd2_rn(fc, fl);
        fs.x = ra ? fs.x : 0.f;
        fs.y = rb ? fs.y : 0.f;
        if (MODE == PM_FULL) {
            fc.x = ra ? fc.x : 0.f; fc.y = rb ? fc.y : 0.f;
            fl.x = ra ? fl.x : 0.f; fl.y = rb ? fl.y : 0.f;
        }
    } else {
        fc.x = ra ? fc.x : 0.f;
        fc.y = rb ? fc.y : 0.f;
        fl.x = (ba && r2.x <= rl2) ? fl.x : 0.f;
        fl.y = (bb && r2.y <= rl2) ? fl.y : 0.f;
        fs = __fadd2_rn(fc, fl);
    }
    if (ENE) {
        // Coulomb energy from the reference's spline (floor(r/h) as in pair_term)
        const float2 fb = __fadd2_rd(__fmul2_rn(r, inv_h2), two23);
        const float2 fm = __fadd2_rn(fb, mtwo23);
        const int ia = (int)min((unsigned)(__float_as_int(fb.x) - 0x4B000000), (unsigned)nsplm1);
        const int ib = (int)min((unsigned)(__float_as_int(fb.y) - 0x4B000000), (unsigned)nsplm1);
        const float2 d = __ffma2_rn(fm, mh2, r);
        const bool la_in = SC ? ra : (ba && r2.x <= rl2), lb_in = SC ? rb : (bb && r2.y <= rl2);
        const float4 pa = sp[ia], pb = sp[ib];
        float2 pe = __fmul2_rn(qq, make_float2(fmaf(d.x, fmaf(d.x, fmaf(d.x, pa.w, pa.z), pa.y), pa.x),
                                               fmaf(d.y, fmaf(d.y, fmaf(d.y, pb.w, pb.z), pb.y), pb.x)));
        pe.x = ra ? pe.x : 0.f;
        pe.y = rb ? pe.y : 0.f;
        ee = __fadd2_rn(ee, pe);
        const float2 v = __fmul2_rn(t6, __fadd2_rn(t6, make_float2(-2.f, -2.f)));
        float2 vl = __fmul2_rn(c12, v);
        vl.x = la_in ? vl.x : 0.f;
        vl.y = lb_in ? vl.y : 0.f;
        ev = __fadd2_rn(ev, vl);
    }
    const float2 cx = __fmul2_rn(fs, dx), cy = __fmul2_rn(fs, dy), cz = __fmul2_rn(fs, dz);
    fi[0] = __fadd2_rn(fi[0], cx); fi[1] = __fadd2_rn(fi[1], cy); fi[2] = __fadd2_rn(fi[2], cz);
    gx = __fadd2_rn(gx, cx); gy = __fadd2_rn(gy, cy); gz = __fadd2_rn(gz, cz);
    if (MODE == PM_FULL) {
        const float2 ax = __fmul2_rn(fc, dx), ay = __fmul2_rn(fc, dy), az = __fmul2_rn(fc, dz);
        wc[0] = __ffma2_rn(ax, dx, wc[0]); wc[1] = __ffma2_rn(ax, dy, wc[1]); wc[2] = __ffma2_rn(ax, dz, wc[2]);
        wc[3] = __ffma2_rn(ay, dy, wc[3]); wc[4] = __ffma2_rn(ay, dz, wc[4]); wc[5] = __ffma2_rn(az, dz, wc[5]);
        const float2 lx = __fmul2_rn(fl, dx), ly = __fmul2_rn(fl, dy), lz = __fmul2_rn(fl, dz);
        wl[0] = __ffma2_rn(lx, dx, wl[0]); wl[1] = __ffma2_rn(lx, dy, wl[1]); wl[2] = __ffma2_rn(lx, dz, wl[2]);
        wl[3] = __ffma2_rn(ly, dy, wl[3]); wl[4] = __ffma2_rn(ly, dz, wl[4]); wl[5] = __ffma2_rn(lz, dz, wl[5]);
    }
}

// Cluster-frame body with packed arithmetic: the same rows, entries, prune
// compaction, force sums and accumulator layout as pair_mixed_body.
// The cluster atoms are staged as 4 atom pairs (x0,x1,y0,y1 | z0,z1,q0,q1);
// each lane holds its j as (-x_j, -x_j) ... so a displacement pair is one
// packed add.  The per-lane force sums of the cluster atoms are 4 packed
// triples (the same 24 registers as 8 scalar ones); j's force is summed as a
// packed pair and its two halves added once per entry.
struct __align__(16) IPair { float4 xy; float4 zq; };

template <int MODE, bool PRUNE, bool SC>
__device__ __forceinline__ void pair_mixed_body_x2(const int4* __restrict__ xq, const PairArgs& a,
                                                   const float2* __restrict__ lj_g,
                                                   const float4* __restrict__ spl_g,
                                                   const DynState* __restrict__ dyn) {
    constexpr bool ENE = MODE == PM_ENE || MODE == PM_FULL;
    extern __shared__ float4 sm[];
    float4* sp = sm;                        // energy table (spline 1), ENE only
    float2* slj = (float2*)(sm + (ENE ? 1 : 0) * a.nspl);
    // per warp: the cluster's LJ rows, [tj][p] = (R^2, R^2, 12 eps, 12 eps) of
    // atoms 2p, 2p+1 with type tj (after the block's type table)
    float4* sljc = (float4*)(slj + ((a.ntyp * a.ntyp + 1) & ~1)) + (size_t)(threadIdx.x >> 5) * 4 * a.ntyp;
    __shared__ IPair sip[PAIR_WARPS][4];
    __shared__ int2 stp[PAIR_WARPS][4];
    if (ENE)
        for (int k = threadIdx.x; k < a.nspl; k += blockDim.x) sp[k] = spl_g[a.nspl + k];
    for (int k = threadIdx.x; k < a.ntyp * a.ntyp; k += blockDim.x) {
        const float2 l = lj_g[k];
        slj[k] = make_float2(l.x, 12.f * l.y);
    }
    const EwaldF ew{a.ew_pa, a.ew_c2a, a.ew_mk};
    __syncthreads();

    const float sx = (float)(dyn->box[0] * (1.0 / 4294967296.0));
    const float sy = (float)(dyn->box[1] * (1.0 / 4294967296.0));
    const float sz = (float)(dyn->box[2] * (1.0 / 4294967296.0));
    const float2 inv_h2 = make_float2(a.inv_hf, a.inv_hf), mh2 = make_float2(-a.hf, -a.hf);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int chunk = (a.ncl + gridDim.x - 1) / gridDim.x;
    const int c_end = min(a.ncl, (blockIdx.x + 1) * chunk);
    const int* __restrict__ typ_s = a.typ_s;
    long long* __restrict__ fs0 = a.fsort;
    const int fst = a.fstride;
    float2 ev = make_float2(0.f, 0.f), ee = make_float2(0.f, 0.f);
    float wt[6] = {0, 0, 0, 0, 0, 0};                     // TENS: sum F (x) x in the cluster frame
    float2 wc[6], wl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) { wc[k] = make_float2(0.f, 0.f); wl[k] = make_float2(0.f, 0.f); }

    const int* __restrict__ rows = PRUNE ? a.blist : a.clist;
    const int* __restrict__ rcnt = PRUNE ? a.bcnt : a.ccnt;
    const float rp2 = a.rp2;

    for (int cl = blockIdx.x * chunk + warp; cl < c_end; cl += wpb) {
        __syncwarp();
        const int4 p0 = __ldg(xq + 8 * cl);
        if (lane < 8) {
            const int4 v = __ldg(xq + 8 * cl + lane);
            float* ip = (float*)&sip[warp][lane >> 1];
            const int h = lane & 1;
            ip[h] = (float)(v.x - p0.x) * sx;
            ip[2 + h] = (float)(v.y - p0.y) * sy;
            ip[4 + h] = (float)(v.z - p0.z) * sz;
            ip[6 + h] = __int_as_float(v.w);
            ((int*)&stp[warp][lane >> 1])[h] = __ldg(typ_s + 8 * cl + lane) * a.ntyp;
            if (PRUNE) a.xq_prune[8 * cl + lane] = v;
        }
        __syncwarp();
        for (int k = lane; k < 4 * a.ntyp; k += 32) {
            const int2 T = stp[warp][k & 3];
            const float2 la = slj[T.x + (k >> 2)], lb = slj[T.y + (k >> 2)];
            sljc[k] = make_float4(la.x, lb.x, la.y, lb.y);
        }
        __syncwarp();
        const int cnt = __ldg(rcnt + cl);
        const int* __restrict__ row = rows + (size_t)cl * a.ccap;
        int* __restrict__ prow = a.plist + (size_t)cl * a.ccap;
        int pcount = 0;
        float2 f[4][3];
#pragma unroll
        for (int p = 0; p < 4; ++p) { f[p][0] = make_float2(0.f, 0.f); f[p][1] = f[p][0]; f[p][2] = f[p][0]; }
        // two-deep prefetch: entries two iterations ahead, their j records one
        // ahead, so no gather waits on the entry load it depends on
        unsigned e = lane < cnt ? (unsigned)__ldg(row + lane) : 0u;
        unsigned e1 = 32 + lane < cnt ? (unsigned)__ldg(row + 32 + lane) : 0u;
        int4 pj = __ldg(xq + (e & 0xFFFFFFu));
        int tj = __ldg(typ_s + (e & 0xFFFFFFu));
        for (int k0 = 0; k0 < cnt; k0 += 32) {          // warp-uniform trip count
            const int kn = k0 + 64 + lane;
            const unsigned e2 = kn < cnt ? (unsigned)__ldg(row + kn) : 0u;
            const int4 pjn = __ldg(xq + (e1 & 0xFFFFFFu));
            const int tjn = __ldg(typ_s + (e1 & 0xFFFFFFu));
            const unsigned m = e >> 24;
            const int sj = e & 0xFFFFFFu;
            const float jx = (float)(pj.x - p0.x) * sx;
            const float jy = (float)(pj.y - p0.y) * sy;
            const float jz = (float)(pj.z - p0.z) * sz;
            const float2 njx = make_float2(-jx, -jx), njy = make_float2(-jy, -jy), njz = make_float2(-jz, -jz);
            const float2 qj = make_float2(__int_as_float(pj.w), __int_as_float(pj.w));
            const float4* ljr = sljc + 4 * tj;
            float2 gx = make_float2(0.f, 0.f), gy = gx, gz = gx;
            unsigned nm = 0;
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const unsigned mb = (m >> (2 * p)) & 3u;
                if (mb) {
                    const IPair I = sip[warp][p];
                    const float4 L = ljr[p];
                    const float2 dx = __fadd2_rn(make_float2(I.xy.x, I.xy.y), njx);
                    const float2 dy = __fadd2_rn(make_float2(I.xy.z, I.xy.w), njy);
                    const float2 dz = __fadd2_rn(make_float2(I.zq.x, I.zq.y), njz);
                    const float2 qq = __fmul2_rn(make_float2(I.zq.z, I.zq.w), qj);
                    float2 r2;
                    pair_term_x2<MODE, SC>(dx, dy, dz, qq, L, mb, a.rr2f, a.rl2f, inv_h2, mh2, a.nsplm1, ew, sp,
                                           f[p], gx, gy, gz, ev, ee, wc, wl, r2);
                    if (PRUNE)
                        nm |= ((((mb & 1u) && r2.x < rp2) ? 1u : 0u) | (((mb & 2u) && r2.y < rp2) ? 2u : 0u))
                              << (2 * p);
                }
            }
            // force on j: minus the sum of its pairs' forces on the cluster atoms
            const float fjx = -(gx.x + gx.y), fjy = -(gy.x + gy.y), fjz = -(gz.x + gz.y);
            if (MODE == PM_TENS && m) {     // j's share of sum F (x) x (frame coordinates)
                wt[0] = fmaf(fjx, jx, wt[0]); wt[1] = fmaf(fjx, jy, wt[1]); wt[2] = fmaf(fjx, jz, wt[2]);
                wt[3] = fmaf(fjy, jy, wt[3]); wt[4] = fmaf(fjy, jz, wt[4]); wt[5] = fmaf(fjz, jz, wt[5]);
            }
            if (m) {
                unsigned long long* fj = (unsigned long long*)fs0 + sj;
                atomicAdd(fj, (unsigned long long)__float2ll_rn(fjx * (float)PGK_FORCE_SCALE));
                atomicAdd(fj + fst, (unsigned long long)__float2ll_rn(fjy * (float)PGK_FORCE_SCALE));
                atomicAdd(fj + 2 * fst, (unsigned long long)__float2ll_rn(fjz * (float)PGK_FORCE_SCALE));
            }
            if (PRUNE) {       // compact the entries that keep a pair inside rprune
                const unsigned b = __ballot_sync(0xffffffffu, nm != 0);
                if (nm) prow[pcount + __popc(b & ((1u << lane) - 1u))] = (int)((nm << 24) | (unsigned)sj);
                pcount += __popc(b);
            }
            e = e1; e1 = e2; pj = pjn; tj = tjn;
        }
        if (PRUNE && lane == 0) a.pcnt[cl] = pcount;
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const float2* fp = f[ii >> 1];
            const float fx = warp_sum((ii & 1) ? fp[0].y : fp[0].x);
            const float fy = warp_sum((ii & 1) ? fp[1].y : fp[1].x);
            const float fz = warp_sum((ii & 1) ? fp[2].y : fp[2].x);
            if (lane == ii) {     // padding slots get zero sums (no mask bits)
                if (MODE == PM_TENS) {      // cluster atom's share of sum F (x) x
                    const float* ip = (const float*)&sip[warp][ii >> 1];
                    const float px = ip[ii & 1], py = ip[2 + (ii & 1)], pz = ip[4 + (ii & 1)];
                    wt[0] = fmaf(fx, px, wt[0]); wt[1] = fmaf(fx, py, wt[1]); wt[2] = fmaf(fx, pz, wt[2]);
                    wt[3] = fmaf(fy, py, wt[3]); wt[4] = fmaf(fy, pz, wt[4]); wt[5] = fmaf(fz, pz, wt[5]);
                }
                unsigned long long* fi = (unsigned long long*)fs0 + 8 * cl + ii;
                atomicAdd(fi, (unsigned long long)__double2ll_rn((double)fx * PGK_FORCE_SCALE));
                atomicAdd(fi + fst, (unsigned long long)__double2ll_rn((double)fy * PGK_FORCE_SCALE));
                atomicAdd(fi + 2 * fst, (unsigned long long)__double2ll_rn((double)fz * PGK_FORCE_SCALE));
            }
        }
    }
    // every pair evaluated once.  Tensor (a,b) -> 3*b + a, stored as its lower triangle.
    if (MODE == PM_FULL) {
        const double evs = ((double)ev.x + (double)ev.y) * (1.0 / 12.0);
        const double ees = (double)ee.x + (double)ee.y;
        double v[16] = {evs, ees, ees};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            v[3 + k] = (double)wc[k].x + (double)wc[k].y;
            v[9 + k] = (double)wl[k].x + (double)wl[k].y;
        }
        v[15] = v[9] + v[12] + v[14];
        const int idx[16] = {A_VDW, A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8,
                             A_VTLJ + 0, A_VTLJ + 1, A_VTLJ + 2, A_VTLJ + 4, A_VTLJ + 5, A_VTLJ + 8, A_VLJ};
        block_acc<16>(v, a.acc, idx, false);
    } else if (MODE == PM_TENS) {
        double v[6] = {wt[0], wt[1], wt[2], wt[3], wt[4], wt[5]};
        const int idx[6] = {A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
        block_acc<6>(v, a.acc, idx, false);
    } else if (MODE == PM_ENE) {
        double v[2] = {((double)ev.x + (double)ev.y) * (1.0 / 12.0), (double)ee.x + (double)ee.y};
        const int idx[2] = {A_VDW, A_ELC};
        block_acc<2>(v, a.acc, idx, false);
    }
}

// One launch per evaluation: the step kind that k_prune_decide wrote on the
// device (prune step or not) selects the body, block-uniformly.  FRAME boxes
// run the packed body (SC: equal LJ and Coulomb cutoffs).
template <int MODE, bool FRAME, bool SC>
__global__ void __launch_bounds__(pair_threads(FRAME), pair_minb(FRAME)) k_pair_mixed(const int4* __restrict__ xq, PairArgs a,
                                                                        const float2* __restrict__ lj_g,
                                                                        const float4* __restrict__ spl_g,
                                                                        const DynState* __restrict__ dyn) {
    const bool prune = a.P != nullptr && a.P->do_prune;
    if (FRAME) {
        if (prune) pair_mixed_body_x2<MODE, true, SC>(xq, a, lj_g, spl_g, dyn);
        else pair_mixed_body_x2<MODE, false, SC>(xq, a, lj_g, spl_g, dyn);
    } else {
        if (prune) pair_mixed_body<MODE, true>(xq, a, lj_g, spl_g, dyn);
        else pair_mixed_body<MODE, false>(xq, a, lj_g, spl_g, dyn);
    }
}

// ---- pair kernel, FP64 (parity path) ---------------------------------------
template <bool ENE>
__global__ void __launch_bounds__(256, 2) k_pair_fp64(const double4* __restrict__ xq, PairArgs a,
                                                      const double2* __restrict__ lj_g,
                                                      const double4* __restrict__ spl_g,
                                                      const DynState* __restrict__ dyn) {
    extern __shared__ double4 smd[];
    double4* sf = smd;
    double4* sp = smd + a.nspl;
    double2* slj = (double2*)(smd + 2 * a.nspl);
    __shared__ double4 si[8][8];
    __shared__ int sti[8][8];
    for (int k = threadIdx.x; k < a.nspl; k += blockDim.x) { sf[k] = spl_g[k]; sp[k] = spl_g[a.nspl + k]; }
    for (int k = threadIdx.x; k < a.ntyp * a.ntyp; k += blockDim.x) slj[k] = lj_g[k];
    __syncthreads();
    const double L0 = dyn->box[0], L1 = dyn->box[1], L2 = dyn->box[2];
    const double B0 = 1.0 / L0, B1 = 1.0 / L1, B2 = 1.0 / L2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int chunk = (a.ncl + gridDim.x - 1) / gridDim.x;
    const int c_end = min(a.ncl, (blockIdx.x + 1) * chunk);
    double e_vdw = 0, e_elc = 0, vc[6] = {0, 0, 0, 0, 0, 0}, vl[6] = {0, 0, 0, 0, 0, 0};
    for (int cl = blockIdx.x * chunk + warp; cl < c_end; cl += wpb) {
        __syncwarp();
        if (lane < 8) {
            si[warp][lane] = xq[8 * cl + lane];
            sti[warp][lane] = a.typ_s[8 * cl + lane] * a.ntyp;
        }
        __syncwarp();
        const int cnt = a.ccnt[cl];
        const int* row = a.clist + (size_t)cl * a.ccap;
        double f[8][3];
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) { f[ii][0] = 0; f[ii][1] = 0; f[ii][2] = 0; }
        for (int k = lane; k < cnt; k += 32) {
            const unsigned e = (unsigned)__ldg(row + k);
            const int j = (int)(e & 0xFFFFFFu);
            const double4 pj = xq[j];
            const int tj = a.typ_s[j];
            const unsigned m = e >> 24;
            double gx = 0, gy = 0, gz = 0;
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
                if (!((m >> ii) & 1u)) continue;
                const double4 pi = si[warp][ii];
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
                    if (ENE) {
                        const double4 p = sp[idx];
                        e_elc += (p.x + d * (p.y + d * (p.z + d * p.w))) * qq;
                    }
                }
                if (r2 <= a.rl2) {
                    const double2 lp = slj[sti[warp][ii] + tj];
                    const double t2 = rinv2 * lp.x;
                    const double t6 = t2 * t2 * t2, t12 = t6 * t6;
                    fl = 12.0 * lp.y * (t12 - t6) * rinv2;
                    if (ENE) e_vdw += lp.y * (t12 - 2.0 * t6);
                }
                const double fx = fc * dx + fl * dx, fy = fc * dy + fl * dy, fz = fc * dz + fl * dz;
                f[ii][0] += fx; f[ii][1] += fy; f[ii][2] += fz;
                gx -= fx; gy -= fy; gz -= fz;
                if (ENE) {
                    vc[0] += fc * dx * dx; vc[1] += fc * dx * dy; vc[2] += fc * dx * dz;
                    vc[3] += fc * dy * dy; vc[4] += fc * dy * dz; vc[5] += fc * dz * dz;
                    vl[0] += fl * dx * dx; vl[1] += fl * dx * dy; vl[2] += fl * dx * dz;
                    vl[3] += fl * dy * dy; vl[4] += fl * dy * dz; vl[5] += fl * dz * dz;
                }
            }
            force_add<false>(a.facc, a.perm[j], gx, gy, gz);
        }
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const double fx = warp_sum(f[ii][0]), fy = warp_sum(f[ii][1]), fz = warp_sum(f[ii][2]);
            if (lane == ii) {
                const int io = a.perm[8 * cl + ii];
                if (io >= 0) force_add<false>(a.facc, io, fx, fy, fz);
            }
        }
    }
    if (ENE) {
        double v[16] = {e_vdw, e_elc, e_elc, vc[0], vc[1], vc[2], vc[3], vc[4], vc[5],
                        vl[0], vl[1], vl[2], vl[3], vl[4], vl[5], vl[0] + vl[3] + vl[5]};
        const int idx[16] = {A_VDW, A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8,
                             A_VTLJ + 0, A_VTLJ + 1, A_VTLJ + 2, A_VTLJ + 4, A_VTLJ + 5, A_VTLJ + 8, A_VLJ};
        block_acc<16>(v, a.acc, idx, true);
    }
}

// ---- pruned list -------------------------------------------------------------
// decision for this pair evaluation (one thread; see PruneDev)
__global__ void k_prune_decide(PruneDev* __restrict__ P, const DynState* __restrict__ dyn, float buffer,
                               float rprune) {
    if (threadIdx.x || blockIdx.x) return;
    const float dmax = __uint_as_float(P->dmax);
    double bt = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) bt = fmax(bt, fabs(dyn->box[d] / P->box[d] - 1.0));
    const bool keep = !P->force && (2.0 * (double)dmax + (double)rprune * bt < (double)buffer);   // NaN -> prune
    P->do_prune = keep ? 0 : 1;
    if (!keep) {
        P->dmax = 0u;
        P->force = 0;
        for (int d = 0; d < 3; ++d) P->box[d] = dyn->box[d];
        P->nprune += 1ull;
    }
}

// sorted-slot pair forces -> the group accumulator, leaving the slot buffer
// zero for the next call
__device__ __forceinline__ void unsort_slots(int blk, long long* __restrict__ fsort, int fst,
                                             const int* __restrict__ perm, int npad, long long* __restrict__ facc) {
    const int s = blk * blockDim.x + threadIdx.x;
    if (s >= npad) return;
    const int i = perm[s];
    const long long vx = fsort[s], vy = fsort[s + fst], vz = fsort[s + 2 * (size_t)fst];
    if (i >= 0 && (vx | vy | vz)) {     // atomic: other force kernels may run beside it
        atomicAdd((unsigned long long*)facc + 3 * (size_t)i, (unsigned long long)vx);
        atomicAdd((unsigned long long*)facc + 3 * (size_t)i + 1, (unsigned long long)vy);
        atomicAdd((unsigned long long*)facc + 3 * (size_t)i + 2, (unsigned long long)vz);
    }
    if (vx | vy | vz) { fsort[s] = 0; fsort[s + fst] = 0; fsort[s + 2 * (size_t)fst] = 0; }
}

// After a mixed pair evaluation: the sorted-slot forces into the group
// accumulator (128 threads a block).
__global__ void __launch_bounds__(128) k_pair_finish(long long* __restrict__ fsort, int fst,
                                                     const int* __restrict__ perm, int npad,
                                                     long long* __restrict__ facc) {
    unsort_slots(blockIdx.x, fsort, fst, perm, npad, facc);
}

template <int MODE, bool FRAME, bool SC>
static void pair_mixed_launch2(pgk_ctx* c, const PairArgs& a) {
    constexpr bool ENE = MODE == PM_ENE || MODE == PM_FULL;
    constexpr int nt = pair_threads(FRAME);
    // spline rows: the packed body stages the energy table only (ENE modes; its
    // force is analytic), the scalar body the force table and, in ENE modes,
    // the energy table
    size_t sm = (size_t)((FRAME ? 0 : 1) + (ENE ? 1 : 0)) * c->nspl * sizeof(float4) +
                (size_t)((c->ntyp * c->ntyp + 1) & ~1) * sizeof(float2);
    if (FRAME) sm += (size_t)(nt / 32) * 4 * c->ntyp * sizeof(float4);
    long long blocks = (long long)c->nsm * pair_minb(FRAME) * (FRAME ? std::max(c->pair_waves, 1) : 1);
    const long long need = (c->ncl + nt / 32 - 1) / (nt / 32);
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    smem_limit(k_pair_mixed<MODE, FRAME, SC>, sm);
    k_pair_mixed<MODE, FRAME, SC><<<(int)blocks, nt, sm, c->st>>>(c->xq, a, c->lj32, c->spl32, c->dyn);
    PGK_LAUNCHED(c);
}

// The cluster frame is exact when no cluster atom or listed j, taken as its
// minimum image from cluster atom 0, can lie half a box away: cluster atoms
// stay within a list cell (plus drift), listed j within rcut_book (plus drift)
// of a cluster atom.
static bool frame_ok(const pgk_ctx* c) {
    const DynState& h = c->hdyn;
    double cs = 0.0, lmin = 1e300;
    for (int d = 0; d < 3; ++d) { cs = std::max(cs, h.cellsize[d]); lmin = std::min(lmin, h.box[d]); }
    if (h.list_mode_used != PGK_LIST_CELL || c->ntyp > 64) return false;   // 64: per-warp LJ rows in smem
    return 0.5 * lmin > std::sqrt(3.0) * cs + c->prm.rcut_book + 4.0;
}

template <int MODE>
static void pair_mixed_launch(pgk_ctx* c, const PairArgs& a) {
    if (frame_ok(c) && !c->no_frame) {
        if (a.rr2f == a.rl2f) pair_mixed_launch2<MODE, true, true>(c, a);
        else pair_mixed_launch2<MODE, true, false>(c, a);
    } else {
        pair_mixed_launch2<MODE, false, false>(c, a);
    }
}

// After the mixed pair kernel: the sorted-slot forces into the group
// accumulator.  Runs on the context's current stream (the force evaluation
// may put it beside the SPME chain: the accumulator adds are atomic).  The
// pruned rows keep the order of the book rows (grouped by their book masks):
// regrouping them by their pruned masks after every prune cost more (146 us a
// prune on the 200k-atom butane rows) than it saved on the steps between
// prunes.
pgk_status launch_pair_finish(pgk_ctx* c, int group) {
    if (c->ncl <= 0 || !c->mixed()) return PGK_OK;
    const int nbu = (c->npad + 127) / 128;
    k_pair_finish<<<nbu, 128, 0, c->st>>>(c->fsort, c->npad_cap, c->perm, c->npad, (long long*)c->facc[group]);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// vmode: PM_FORCE / PM_ENE / PM_TENS / PM_FULL (see above)
// the pair kernel's arguments for one MTS group, reading the book rows
static PairArgs pair_args(pgk_ctx* c, int group) {
    PairArgs a;
    a.clist = c->clist; a.ccnt = c->ccnt; a.ccap = c->ccap; a.ncl = c->ncl;
    a.typ_s = c->typ_s; a.perm = c->perm; a.ntyp = c->ntyp; a.nspl = c->nspl;
    a.h = c->hspl; a.inv_h = 1.0 / c->hspl;
    a.rrcut = c->prm.rrcut;
    a.rr2 = c->prm.rrcut * c->prm.rrcut;
    a.rl2 = c->prm.rcut * c->prm.rcut;
    a.rmax2 = a.rr2 > a.rl2 ? a.rr2 : a.rl2;
    a.rr2f = (float)a.rr2; a.rl2f = (float)a.rl2; a.inv_hf = (float)a.inv_h; a.hf = (float)a.h;
    a.nsplm1 = c->nspl - 1;
    {
        const double al = c->prm.alpha;
        a.ew_pa = (float)(0.3275911 * al);
        a.ew_c2a = (float)(2.0 * al / std::sqrt(std::acos(-1.0)));
        a.ew_mk = (float)(-al * al * 1.4426950408889634);     // -alpha^2 log2(e)
    }
    a.facc = c->facc[group];
    a.acc = c->acc + (size_t)group * NACC;
    a.fsort = c->fsort; a.fstride = c->npad_cap;
    a.P = nullptr; a.blist = nullptr; a.bcnt = nullptr; a.plist = nullptr; a.pcnt = nullptr; a.xq_prune = nullptr;
    a.rp2 = 0.f;
    return a;
}

// ---- grid of the cluster-frame pair kernel ---------------------------------------
// The packed body's blocks take fixed chunks of cluster rows, five blocks a
// SM.  In one wave the chunks finish unevenly; several waves of smaller
// chunks balance better, at the cost of more block starts.  Timing the
// regular body (force only, on the book rows) with 1 to 4 waves on the
// 200k-atom butane rows gives 0.33, 0.30, 0.27, 0.29 ms per evaluation, and
// the step time follows: the kernel runs 3 waves.  Forces do not depend on
// the grid (each row's pair forces are summed by one warp and added as
// int64), but the energy and virial partials are FP32 sums per warp over the
// rows a warp takes, which follow the grid; so the wave count is fixed (the
// same grid, the same bits, run after run) and the per-context measurement
// runs only when PGK_PAIR_AUTOTUNE=1 (at the context's first list build; the
// choice is listed in the tuning table).
static std::mutex g_pair_tune_mu;
static std::map<int, std::string> g_pair_tune;       // cluster count -> table line

pgk_status pair_autotune(pgk_ctx* c) {
    if (c->pair_tuned) return PGK_OK;
    c->pair_tuned = true;
    c->pair_waves = 3;
    const char* env = getenv("PGK_PAIR_AUTOTUNE");
    if (!env || atoi(env) == 0 || !c->mixed() || c->ncl <= 0 || !frame_ok(c) || c->no_frame) return PGK_OK;
    pgk_status s;
    if ((s = launch_pack(c))) return s;               // current positions into the sorted slots
    const PairArgs a = pair_args(c, 0);
    const bool sc = a.rr2f == a.rl2f;
    cudaEvent_t e0, e1;
    PGK_CUDA(c, cudaEventCreate(&e0));
    PGK_CUDA(c, cudaEventCreate(&e1));
    float us[5] = {0, 0, 0, 0, 0}, best_us = 1e30f;
    int best = 3;
    const long long l0 = c->launches;
    for (int w = 1; w <= 4; ++w) {
        c->pair_waves = w;
        for (int r = 0; r < 4; ++r) {                 // one warm-up, three timed
            if (r == 1) PGK_CUDA(c, cudaEventRecord(e0, c->st));
            if (sc) pair_mixed_launch2<PM_FORCE, true, true>(c, a);
            else pair_mixed_launch2<PM_FORCE, true, false>(c, a);
        }
        PGK_CUDA(c, cudaEventRecord(e1, c->st));
        PGK_CUDA(c, cudaEventSynchronize(e1));
        float ms = 0.f;
        PGK_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
        us[w] = ms * 1e3f / 3.f;
        if (us[w] < best_us) { best_us = us[w]; best = w; }
    }
    c->launches = l0;                                 // not part of any step
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->pair_waves = best;
    // the timing launches' forces out of the slot buffer
    PGK_CUDA(c, cudaMemsetAsync(c->fsort, 0, sizeof(long long) * 3 * (size_t)c->npad_cap, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    char line[256];
    snprintf(line, sizeof(line),
             "pair %d clusters (%d atoms) fp32: waves of blocks %d (1: %.1f us, 2: %.1f us, 3: %.1f us, 4: %.1f us)\n",
             c->ncl, c->natom, best, us[1], us[2], us[3], us[4]);
    std::lock_guard<std::mutex> lk(g_pair_tune_mu);
    g_pair_tune[c->ncl] = line;
    return PGK_OK;
}

std::string pair_tuning_text() {
    std::lock_guard<std::mutex> lk(g_pair_tune_mu);
    std::string t;
    for (auto& kv : g_pair_tune) t += kv.second;
    return t;
}

pgk_status launch_pair(pgk_ctx* c, int group, int vmode, bool finish) {
    if (c->ncl <= 0) return PGK_OK;
    PairArgs a = pair_args(c, group);
    const bool pruned = c->mixed() && c->prune_buffer > 0.f;
    if (pruned) {
        const float rp = (float)std::sqrt(a.rmax2) + c->prune_buffer;
        k_prune_decide<<<1, 32, 0, c->st>>>(c->prune, c->dyn, c->prune_buffer, rp);
        c->launches += 1;
        a.P = c->prune; a.blist = c->clist; a.bcnt = c->ccnt; a.plist = c->plist; a.pcnt = c->pcnt;
        a.xq_prune = c->xq_prune; a.rp2 = rp * rp;
        a.clist = c->plist; a.ccnt = c->pcnt;
    }
    if (c->rec_pre_pair) {
        PGK_CUDA(c, cudaEventRecord(c->ev_pre_pair, c->st));
        c->rec_pre_pair_done = true;
    }
    if (c->mixed()) {
        switch (vmode) {
            case PM_FULL: pair_mixed_launch<PM_FULL>(c, a); break;
            case PM_TENS: pair_mixed_launch<PM_TENS>(c, a); break;
            case PM_ENE: pair_mixed_launch<PM_ENE>(c, a); break;
            default: pair_mixed_launch<PM_FORCE>(c, a); break;
        }
    } else {
        int blocks = c->nsm * 2;                     // 256-thread blocks, two per SM
        const long long need = (c->ncl + 7) / 8;
        if (blocks > need) blocks = (int)need;
        if (blocks < 1) blocks = 1;
        size_t sm = (size_t)2 * c->nspl * sizeof(double4) + c->ntyp * c->ntyp * sizeof(double2);
        if (vmode != PM_FORCE) {
            smem_limit(k_pair_fp64<true>, sm);
            k_pair_fp64<true><<<blocks, 256, sm, c->st>>>(c->xq64, a, c->lj64, c->spl64, c->dyn);
        } else {
            smem_limit(k_pair_fp64<false>, sm);
            k_pair_fp64<false><<<blocks, 256, sm, c->st>>>(c->xq64, a, c->lj64, c->spl64, c->dyn);
        }
        PGK_LAUNCHED(c);
    }
    PGK_CUDA(c, cudaGetLastError());
    return finish ? launch_pair_finish(c, group) : PGK_OK;
}

// ---- diagnostic: unique pairs inside the interaction cutoff, list entries ----
// (the algorithmic work units of the pair kernel; run outside any timed region)
__global__ void k_count_pairs(const double* __restrict__ pos_s, const int* __restrict__ clist,
                              const int* __restrict__ ccnt, int ccap, int ncl, double rmax2,
                              const DynState* __restrict__ dyn, unsigned long long* out) {
    int cl = blockIdx.x * blockDim.x + threadIdx.x;
    if (cl >= ncl) return;
    unsigned long long np = 0, bits = 0;
    const double L0 = dyn->box[0], L1 = dyn->box[1], L2 = dyn->box[2];
    const int cnt = ccnt[cl];
    for (int k = 0; k < cnt; ++k) {
        unsigned e = (unsigned)clist[(size_t)cl * ccap + k];
        int t = (int)(e & 0xFFFFFFu);
        for (int ii = 0; ii < 8; ++ii) {
            if (!((e >> (24 + ii)) & 1u)) continue;
            ++bits;
            int s = 8 * cl + ii;
            if (t <= s) continue;
            double dx = pos_s[3 * s] - pos_s[3 * t]; dx -= L0 * round(dx / L0);
            double dy = pos_s[3 * s + 1] - pos_s[3 * t + 1]; dy -= L1 * round(dy / L1);
            double dz = pos_s[3 * s + 2] - pos_s[3 * t + 2]; dz -= L2 * round(dz / L2);
            if (dx * dx + dy * dy + dz * dz <= rmax2) ++np;
        }
    }
    atomicAdd(out, np);
    atomicAdd(out + 1, bits);
    atomicAdd(out + 2, (unsigned long long)cnt);
}

// npair: unique pairs inside max(rrcut, rcut); nbits: list pairs, both
// directions (pair evaluations); nentries: (cluster, j) entries read
pgk_status count_pairs(pgk_ctx* c, long long* npair, long long* nentries, long long* nbits) {
    if (c->ncl <= 0) { *npair = 0; *nentries = 0; if (nbits) *nbits = 0; return PGK_OK; }
    unsigned long long* d = c->counters + 4;
    PGK_CUDA(c, cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), c->st));
    double rr2 = c->prm.rrcut * c->prm.rrcut, rl2 = c->prm.rcut * c->prm.rcut;
    k_count_pairs<<<(c->ncl + 127) / 128, 128, 0, c->st>>>(c->pos_s, c->clist, c->ccnt, c->ccap, c->ncl,
                                                            rr2 > rl2 ? rr2 : rl2, c->dyn, d);
    PGK_CUDA(c, cudaGetLastError());
    unsigned long long h[3] = {0, 0, 0};
    PGK_CUDA(c, cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    *npair = (long long)h[0];
    *nentries = (long long)h[2];
    if (nbits) *nbits = (long long)h[1];
    return PGK_OK;
}
