// k_bonded.cu -- intramolecular terms:
//   calbondp   calbond.F90:109-219      U = k (r - r0)^2
//   calanglp   calangl.F90:172-358      U = k (theta - theta0)^2
//   caltorsp   caltors.F90 (+calijkl)   U = V/div (1 + cos(n phi - phase))
//   caltorsrbp caltorsrb.F90:118-459    U = sum_n C_n (-1)^n cos^n phi
//   calnon14p  calnon14.F90:249-521     scaled 1-4 Coulomb + LJ
//   ewaldrp excluded-pair erf correction (ewaldr.F90:756-826)
//
// Layout: every term type writes the force on each of its atoms into its own
// slot of one global slot array (slot = base[type] + K*term + q, SoA x|y|z),
// one thread per term and one kernel per type, with no atomics; then
// k_slot_gather sums each atom's slots in a fixed order (a precomputed
// incidence list) and adds the total to the group's force accumulator once.
// The result is deterministic in both precisions and needs no assumption on
// molecule layout.  Energies and virials are block-reduced per type.
//
// Displacements are formed in FP64 from the master positions (Fortran anint
// minimum image); the remaining arithmetic runs in T (float for mixed).
// Angle and torsion virials use absolute coordinates exactly like the
// reference (sum f_a x_b over the term's atoms).
#include <algorithm>
#include <vector>

#include "pgk_ctx.cuh"
#include "pgk_hf.cuh"


template <typename T>
__device__ __forceinline__ void disp(const double* __restrict__ P, int a, int b, const DynState* __restrict__ dyn,
                                     T* r) {   // r = x_a - x_b, min image
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = P[3 * a + d] - P[3 * b + d];
        r[d] = (T)(v - dyn->box[d] * round(v * dyn->boxinv[d]));
    }
}
template <typename T>
__device__ __forceinline__ void crs(const T* x, const T* y, T* z) {
    z[0] = x[1] * y[2] - x[2] * y[1];
    z[1] = x[2] * y[0] - x[0] * y[2];
    z[2] = x[0] * y[1] - x[1] * y[0];
}
template <typename T>
__device__ __forceinline__ T dt3(const T* a, const T* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// pair-style virial: scalar f.r, tensor f_a r_b
__device__ __forceinline__ void vir_pair(double* v, const double* f, const double* r) {
    v[0] += f[0] * r[0] + f[1] * r[1] + f[2] * r[2];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) v[1 + a + 3 * b] += f[a] * r[b];
}
// absolute-coordinate virial of one atom
__device__ __forceinline__ void vir_abs(double* v, const double* f, const double* __restrict__ P, int at) {
    const double x[3] = {P[3 * at], P[3 * at + 1], P[3 * at + 2]};
    v[0] += f[0] * x[0] + f[1] * x[1] + f[2] * x[2];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) v[1 + a + 3 * b] += f[a] * x[b];
}

// where a term kernel puts its forces: the slot array (slot = base + K*term + q)
// or, when slot is null, the force accumulator (atomics)
struct TermOut {
    void* facc;
    void* slot;          // [3][S] of T
    long long S, base;
};
template <bool MIXED>
__device__ __forceinline__ void put_force(const TermOut& o, int term, int K, int q, int atom, const double* F,
                                          double sgn) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    if (o.slot) {
        T* sl = (T*)o.slot;
        const size_t k = (size_t)o.base + (size_t)K * term + q;
        sl[k] = (T)(sgn * F[0]);
        sl[o.S + k] = (T)(sgn * F[1]);
        sl[2 * o.S + k] = (T)(sgn * F[2]);
    } else {
        force_add<MIXED>(o.facc, atom, sgn * F[0], sgn * F[1], sgn * F[2]);
    }
}

// ---- term evaluators (P = positions, indices into P) ------------------------
template <typename T>
__device__ __forceinline__ bool eval_bond(const double* P, int i, int j, double2 p, const DynState* dyn,
                                          double (&F)[3], double (&rd)[3], double& pot) {
    if (fabs(p.x) < 1.0e-16) return false;
    T r[3];
    disp<T>(P, i, j, dyn, r);
    T rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    T dr = rr - (T)p.y;
    T fa = T(-2) * (T)p.x * dr;
#pragma unroll
    for (int d = 0; d < 3; ++d) { F[d] = (double)(fa * r[d] / rr); rd[d] = (double)r[d]; }
    pot = (double)((T)p.x * dr * dr);
    return true;
}

template <typename T>
__device__ __forceinline__ bool eval_angl(const double* P, int i, int j, int k, double2 p, const DynState* dyn,
                                          double (&F)[3][3], double& pot) {
    if (fabs(p.x) < 1.0e-32) return false;
    T rij[3], rkj[3];
    disp<T>(P, j, i, dyn, rij);
    disp<T>(P, j, k, dyn, rkj);
    T ra = sqrt(dt3(rij, rij)), rb = sqrt(dt3(rkj, rkj));
    T c = dt3(rij, rkj) / (ra * rb);
    if (c > T(1)) c = T(1); else if (c < T(-1)) c = T(-1);
    T th = acos(c), s = sin(th);
    T dth = th - (T)p.y;
    T fi[3] = {0, 0, 0}, fk[3] = {0, 0, 0};
    if (fabs((double)s) > 1.0e-14) {
        T ft = T(-2) * (T)p.x * dth / s;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            fi[d] = ft * ((rkj[d] / rb - rij[d] * c / ra) / ra);
            fk[d] = ft * ((rij[d] / ra - rkj[d] * c / rb) / rb);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        F[0][d] = (double)fi[d];
        F[1][d] = (double)(-fi[d] - fk[d]);
        F[2][d] = (double)fk[d];
    }
    pot = (double)((T)p.x * dth * dth);
    return true;
}

template <typename T>
struct TG { T c, phi, s, b[3], cc[3]; };

template <typename T>
__device__ __forceinline__ void tors_geo(const T* rij, const T* rkj, const T* rkl, TG<T>& g) {
    T ni[3], nl[3], t[3];
    crs(rij, rkj, ni);
    crs(rkj, rkl, nl);
    T ai = sqrt(dt3(ni, ni)), al = sqrt(dt3(nl, nl));
    T c = dt3(ni, nl) / (ai * al);
    if (c > T(1)) c = T(1); else if (c < T(-1)) c = T(-1);
    crs(ni, nl, t);
    T phi = acos(c);
    phi = -copysign(phi, dt3(rkj, t));
    g.c = c; g.phi = phi; g.s = sin(phi);
#pragma unroll
    for (int d = 0; d < 3; ++d) { ni[d] /= ai; nl[d] /= al; }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g.b[d] = (nl[d] - c * ni[d]) / ai;
        g.cc[d] = (ni[d] - c * nl[d]) / al;
    }
}

// periodic (RB = false, par = (barhig/divfac, phsang, period, cos(phsang)))
// or Ryckaert-Bellemans (RB = true, C = C0..C5)
template <typename T, bool RB>
__device__ __forceinline__ void eval_tors(const double* P, int i, int j, int k, int l, double4 p,
                                          const double* __restrict__ C, const DynState* dyn, double (&F)[4][3],
                                          double& pot, unsigned* status) {
    T rij[3], rkj[3], rkl[3], rik[3], rjl[3];
    disp<T>(P, j, i, dyn, rij); disp<T>(P, j, k, dyn, rkj); disp<T>(P, l, k, dyn, rkl);
    disp<T>(P, k, i, dyn, rik); disp<T>(P, l, j, dyn, rjl);
    TG<T> g;
    tors_geo(rij, rkj, rkl, g);
    T fa, e;
    if (RB) {
        T bt[6] = {(T)C[0], -(T)C[1], (T)C[2], -(T)C[3], (T)C[4], -(T)C[5]};
        T dp = bt[5];
        fa = 0;
#pragma unroll
        for (int q = 4; q >= 0; --q) { fa = fa * g.c + dp; dp = dp * g.c + bt[q]; }
        fa = -fa;
        e = dp;
    } else {
        T per = (T)p.z;
        e = (T)p.x * (T(1) + cos(per * g.phi - (T)p.y));
        int np = (int)lround(p.z);
        T c = g.c;
        if (np == 1) fa = T(1);
        else if (np == 2) fa = T(2) * c;
        else if (np == 3) fa = T(-4) * g.s * g.s + T(3);
        else if (np == 4) fa = T(4) * c * (T(2) * c * c - T(1));
        else if (np == 5) { fa = T(4) * c * c; fa = fa * (fa - T(3)) + T(1); }
        else if (np == 6) { fa = T(4) * c * c; fa = T(2) * c * (fa - T(3)) * (fa - T(1)); }
        else { fa = 0; atomicOr(status, ST_UNSUPPORTED); }
        fa = -fa * (T)p.w * (T)p.x * per;
    }
    T t1[3], t2[3];
    crs(g.b, rkj, t1);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[0][d] = (double)(fa * t1[d]);
    crs(g.cc, rkl, t1); crs(g.b, rik, t2);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[1][d] = (double)(fa * (-t1[d] + t2[d]));
    crs(g.b, rij, t1); crs(g.cc, rjl, t2);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[2][d] = (double)(fa * (-t1[d] + t2[d]));
    crs(g.cc, rkj, t1);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[3][d] = (double)(fa * t1[d]);
    pot = (double)e;
}

template <typename T>
__device__ __forceinline__ void eval_14(const double* P, int i, int j, double qq, double2 lp, double2 fc,
                                        const DynState* dyn, double (&F)[3], double (&rd)[3], double& de_out,
                                        double& dv_out) {
    T r[3];
    disp<T>(P, i, j, dyn, r);
    T r2 = dt3(r, r);
    T ri2 = T(1) / r2, ri1 = sqrt(ri2);
    T de = (T)qq * ri1;
    de = de * (T)fc.x;
    T t2 = ri2 * (T)lp.x, t6 = t2 * t2 * t2, t12 = t6 * t6;
    T E = (T)lp.y * (T)fc.y;
    T dv = E * (t12 - T(2) * t6);
    T ft = T(12) * E * (t12 - t6) * ri2;
    T fs = de * ri2 + ft;
#pragma unroll
    for (int d = 0; d < 3; ++d) { F[d] = (double)(fs * r[d]); rd[d] = (double)r[d]; }
    de_out = (double)de;
    dv_out = (double)dv;
}

// excluded-pair erf correction: spline tables 2 (force) and 3 (potential)
template <bool MIXED>
__device__ __forceinline__ void eval_excl(const double* P, int i, int j, double qq, const double4* __restrict__ spl64,
                                          const float4* __restrict__ spl32, int nspl, double h,
                                          const DynState* dyn, double (&F)[3], double (&rd)[3], double& pot) {
    double r[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = P[3 * i + d] - P[3 * j + d];
        r[d] = v - dyn->box[d] * round(v * dyn->boxinv[d]);
        rd[d] = r[d];
    }
    pot = 0.0;
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
        F[0] = (double)(fs * rx); F[1] = (double)(fs * ry); F[2] = (double)(fs * rz);
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
        F[0] = fs * r[0]; F[1] = fs * r[1]; F[2] = fs * r[2];
    }
}

// ---- per-term-type kernels (general path) -------------------------------------
template <bool MIXED>
__global__ void k_bond(const double* __restrict__ pos, const int2* __restrict__ ij, const double2* __restrict__ par,
                       int nterm, const DynState* __restrict__ dyn, TermOut out, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < nterm) {
        double F[3] = {0, 0, 0}, rd[3], e;
        int i = ij[k].x, j = ij[k].y;
        const bool on = eval_bond<T>(pos, i, j, par[k], dyn, F, rd, e);
        put_force<MIXED>(out, k, 2, 0, i, F, 1.0);
        put_force<MIXED>(out, k, 2, 1, j, F, -1.0);
        if (want && on) { v[0] = e; vir_pair(v + 1, F, rd); }
    }
    if (want) {
        const int idx[11] = {A_BOND, A_VB, A_VTB + 0, A_VTB + 1, A_VTB + 2, A_VTB + 3, A_VTB + 4, A_VTB + 5,
                             A_VTB + 6, A_VTB + 7, A_VTB + 8};
        block_acc<11>(v, acc, idx, !MIXED);
    }
}

template <bool MIXED>
__global__ void k_angl(const double* __restrict__ pos, const int4* __restrict__ ijk, const double2* __restrict__ par,
                       int nterm, const DynState* __restrict__ dyn, TermOut out, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (n < nterm) {
        double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e;
        int at[3] = {ijk[n].x, ijk[n].y, ijk[n].z};
        const bool on = eval_angl<T>(pos, at[0], at[1], at[2], par[n], dyn, F, e);
#pragma unroll
        for (int q = 0; q < 3; ++q) put_force<MIXED>(out, n, 3, q, at[q], F[q], 1.0);
        if (want && on) {
            v[0] = e;
#pragma unroll
            for (int q = 0; q < 3; ++q) vir_abs(v + 1, F[q], pos, at[q]);
        }
    }
    if (want) {
        const int idx[11] = {A_ANGL, A_VA, A_VTA + 0, A_VTA + 1, A_VTA + 2, A_VTA + 3, A_VTA + 4, A_VTA + 5,
                             A_VTA + 6, A_VTA + 7, A_VTA + 8};
        block_acc<11>(v, acc, idx, !MIXED);
    }
}

template <bool MIXED, bool RB>
__global__ void k_tors(const double* __restrict__ pos, const int4* __restrict__ ijkl, const double4* __restrict__ par,
                       const double* __restrict__ rbc, int nterm, const DynState* __restrict__ dyn, TermOut out,
                       long long* acc, int want, unsigned* status) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (n < nterm) {
        const int at[4] = {ijkl[n].x, ijkl[n].y, ijkl[n].z, ijkl[n].w};
        double F[4][3], e;
        eval_tors<T, RB>(pos, at[0], at[1], at[2], at[3], RB ? make_double4(0, 0, 0, 0) : par[n],
                         RB ? rbc + 6 * (size_t)n : nullptr, dyn, F, e, status);
#pragma unroll
        for (int q = 0; q < 4; ++q) put_force<MIXED>(out, n, 4, q, at[q], F[q], 1.0);
        if (want) {
            v[0] = e;
#pragma unroll
            for (int q = 0; q < 4; ++q) vir_abs(v + 1, F[q], pos, at[q]);
        }
    }
    if (want) {
        const int idx[11] = {RB ? A_TORSRB : A_TORS, A_VT, A_VTT + 0, A_VTT + 1, A_VTT + 2, A_VTT + 3, A_VTT + 4,
                             A_VTT + 5, A_VTT + 6, A_VTT + 7, A_VTT + 8};
        block_acc<11>(v, acc, idx, !MIXED);
    }
}

template <bool MIXED>
__global__ void k_non14(const double* __restrict__ pos, const double* __restrict__ chrg, const int* __restrict__ typ,
                        const int2* __restrict__ ij, const double2* __restrict__ fac, int nterm, int ntyp,
                        const double2* __restrict__ lj64, const DynState* __restrict__ dyn, TermOut out,
                        long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[12] = {0};
    if (n < nterm) {
        int i = ij[n].x, j = ij[n].y;
        double F[3], rd[3], de, dv;
        eval_14<T>(pos, i, j, chrg[i] * chrg[j], lj64[typ[i] * ntyp + typ[j]], fac[n], dyn, F, rd, de, dv);
        put_force<MIXED>(out, n, 2, 0, i, F, 1.0);
        put_force<MIXED>(out, n, 2, 1, j, F, -1.0);
        if (want) { v[0] = de; v[1] = dv; vir_pair(v + 2, F, rd); }
    }
    if (want) {
        const int idx[12] = {A_ELC14, A_VDW14, A_V14, A_VT14 + 0, A_VT14 + 1, A_VT14 + 2, A_VT14 + 3, A_VT14 + 4,
                             A_VT14 + 5, A_VT14 + 6, A_VT14 + 7, A_VT14 + 8};
        block_acc<12>(v, acc, idx, !MIXED);
    }
}

template <bool MIXED>
__global__ void k_excl(const double* __restrict__ pos, const double* __restrict__ chrg,
                       const int2* __restrict__ pairs, int npair, const double4* __restrict__ spl64,
                       const float4* __restrict__ spl32, int nspl, double h, const DynState* __restrict__ dyn,
                       TermOut out, long long* acc, int want) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < npair) {
        int i = pairs[k].x, j = pairs[k].y;
        double F[3], rd[3], e;
        eval_excl<MIXED>(pos, i, j, chrg[i] * chrg[j], spl64, spl32, nspl, h, dyn, F, rd, e);
        put_force<MIXED>(out, k, 2, 0, i, F, 1.0);
        put_force<MIXED>(out, k, 2, 1, j, F, -1.0);
        v[0] = -e;
        vir_pair(v + 1, F, rd);
    }
    if (want) {
        // pot_elc -= potij; pot_viri_coul -= potij; tensor (lower triangle) += f r
        double w[8] = {v[0], v[0], v[2], v[3], v[4], v[6], v[7], v[10]};
        const int idx[8] = {A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
        block_acc<8>(w, acc, idx, !MIXED);
    }
}

// ---- per-atom sum of the slot forces --------------------------------------------
// type of a slot from the type bases; only the types in `mask` were written by
// this evaluation, the others hold another MTS group's values and are skipped
struct SlotTypes { long long base[7]; };

template <bool MIXED>
__global__ void k_slot_gather(const int* __restrict__ inc_start, const int* __restrict__ inc_slot,
                              const void* __restrict__ slot, SlotTypes ty, int mask, int n, void* facc) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long S = ty.base[6];
    const T* sx = (const T*)slot;
    const T* sy = sx + S;
    const T* sz = sy + S;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int k = inc_start[i]; k < inc_start[i + 1]; ++k) {
        const int sl = inc_slot[k];
        int t = 0;
#pragma unroll
        for (int q = 1; q < 6; ++q) t += sl >= ty.base[q] ? 1 : 0;
        if (!((mask >> t) & 1)) continue;
        fx += (double)sx[sl]; fy += (double)sy[sl]; fz += (double)sz[sl];
    }
    if (fx != 0.0 || fy != 0.0 || fz != 0.0) force_add<MIXED>(facc, i, fx, fy, fz);
}

// ---- host side -------------------------------------------------------------------
template <typename V>
static void reorder(std::vector<V>& v, const std::vector<int>& order) {
    std::vector<V> out(v.size());
    for (size_t k = 0; k < order.size(); ++k) out[k] = v[order[k]];
    v.swap(out);
}

template <typename T>
static pgk_status up(pgk_ctx* c, T** dst, const std::vector<T>& v) {
    if (v.empty()) { *dst = nullptr; return PGK_OK; }
    PGK_CUDA(c, cudaMalloc(dst, v.size() * sizeof(T)));
    PGK_CUDA(c, cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PGK_OK;
}

// Term arrays ordered by their lowest atom (locality of the position gathers
// and slot writes), the global slot layout and each atom's slot incidence
// list (by type, then term), and the slot array itself.
pgk_status bonded_setup(pgk_ctx* c, HostTerms& t, const std::vector<int>&, const std::vector<int>&) {
    const int n = c->natom;
    const int K[6] = {2, 3, 4, 4, 2, 2};
    auto sort_type = [&](int count, auto first_atom, auto apply) {
        std::vector<int> order(count);
        for (int k = 0; k < count; ++k) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return first_atom(x) < first_atom(y); });
        apply(order);
    };
    auto mn = [](std::initializer_list<int> v) { return std::min(v); };
    sort_type((int)t.bij.size(), [&](int k) { return mn({t.bij[k].x, t.bij[k].y}); },
              [&](const std::vector<int>& o) { reorder(t.bij, o); reorder(t.bp, o); });
    sort_type((int)t.aijk.size(), [&](int k) { return mn({t.aijk[k].x, t.aijk[k].y, t.aijk[k].z}); },
              [&](const std::vector<int>& o) { reorder(t.aijk, o); reorder(t.ap, o); });
    sort_type((int)t.tij.size(), [&](int k) { return mn({t.tij[k].x, t.tij[k].y, t.tij[k].z, t.tij[k].w}); },
              [&](const std::vector<int>& o) { reorder(t.tij, o); reorder(t.tp, o); });
    sort_type((int)t.rij.size(), [&](int k) { return mn({t.rij[k].x, t.rij[k].y, t.rij[k].z, t.rij[k].w}); },
              [&](const std::vector<int>& o) {
                  std::vector<double> rc2(t.rc.size());
                  for (size_t k = 0; k < o.size(); ++k)
                      for (int q = 0; q < 6; ++q) rc2[6 * k + q] = t.rc[6 * o[k] + q];
                  reorder(t.rij, o);
                  t.rc.swap(rc2);
              });
    sort_type((int)t.p14.size(), [&](int k) { return mn({t.p14[k].x, t.p14[k].y}); },
              [&](const std::vector<int>& o) { reorder(t.p14, o); reorder(t.f14, o); });
    sort_type((int)t.ex.size(), [&](int k) { return mn({t.ex[k].x, t.ex[k].y}); },
              [&](const std::vector<int>& o) { reorder(t.ex, o); });
    pgk_status s;
    c->nbond = (int)t.bij.size(); c->nangl = (int)t.aijk.size(); c->ntors = (int)t.tij.size();
    c->ntorsrb = (int)t.rij.size(); c->n14 = (int)t.p14.size(); c->nexpair = (int)t.ex.size();
    if ((s = up(c, &c->bond_ij, t.bij)) || (s = up(c, &c->bond_p, t.bp)) || (s = up(c, &c->angl_ijk, t.aijk)) ||
        (s = up(c, &c->angl_p, t.ap)) || (s = up(c, &c->tors_ijkl, t.tij)) || (s = up(c, &c->tors_p, t.tp)) ||
        (s = up(c, &c->rb_ijkl, t.rij)) || (s = up(c, &c->rb_c, t.rc)) || (s = up(c, &c->p14_ij, t.p14)) ||
        (s = up(c, &c->p14_f, t.f14)) || (s = up(c, &c->expair, t.ex)))
        return s;
    const long long cnt[6] = {c->nbond, c->nangl, c->ntors, c->ntorsrb, c->n14, c->nexpair};
    c->slot_base[0] = 0;
    for (int ty = 0; ty < 6; ++ty) c->slot_base[ty + 1] = c->slot_base[ty] + K[ty] * cnt[ty];
    const long long S = c->slot_base[6];
    if (S >= (1LL << 31)) return pgk_fail(c, PGK_E_UNSUPPORTED, "more than 2^31 bonded term slots");
    std::vector<int> deg(n + 1, 0);
    auto atoms_of = [&](int ty, long long k, int* at) {
        switch (ty) {
            case 0: at[0] = t.bij[k].x; at[1] = t.bij[k].y; break;
            case 1: at[0] = t.aijk[k].x; at[1] = t.aijk[k].y; at[2] = t.aijk[k].z; break;
            case 2: at[0] = t.tij[k].x; at[1] = t.tij[k].y; at[2] = t.tij[k].z; at[3] = t.tij[k].w; break;
            case 3: at[0] = t.rij[k].x; at[1] = t.rij[k].y; at[2] = t.rij[k].z; at[3] = t.rij[k].w; break;
            case 4: at[0] = t.p14[k].x; at[1] = t.p14[k].y; break;
            default: at[0] = t.ex[k].x; at[1] = t.ex[k].y; break;
        }
    };
    int at[4];
    for (int ty = 0; ty < 6; ++ty)
        for (long long k = 0; k < cnt[ty]; ++k) {
            atoms_of(ty, k, at);
            for (int q = 0; q < K[ty]; ++q) deg[at[q] + 1]++;
        }
    for (int i = 0; i < n; ++i) deg[i + 1] += deg[i];
    std::vector<int> inc((size_t)std::max<long long>(S, 1)), fill(deg.begin(), deg.end() - 1);
    for (int ty = 0; ty < 6; ++ty)
        for (long long k = 0; k < cnt[ty]; ++k) {
            atoms_of(ty, k, at);
            for (int q = 0; q < K[ty]; ++q) inc[fill[at[q]]++] = (int)(c->slot_base[ty] + K[ty] * k + q);
        }
    if ((s = up(c, &c->inc_start, deg)) || (s = up(c, &c->inc_slot, inc))) return s;
    if (S > 0) {
        const size_t bytes = (size_t)3 * S * (c->mixed() ? sizeof(float) : sizeof(double));
        PGK_CUDA(c, cudaMalloc(&c->slot_f, bytes));
        PGK_CUDA(c, cudaMemset(c->slot_f, 0, bytes));
    }
    return PGK_OK;
}

// ---- heat-flux parts of the bonded terms (cal*_hf.F90) -----------------------
// FP64 in both precisions (heat-flux steps only); per-atom potential shares
// (1/2, 1/3, 1/4 of the term energy) and calvirihf for the pairs of atoms of
// each term, with the term forces.
__global__ void k_bond_hf(const double* __restrict__ pos, const int2* __restrict__ ij,
                          const double2* __restrict__ par, int nterm, const DynState* __restrict__ dyn, HfDev h) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nterm) return;
    double F[3], rd[3], e;
    const int i = ij[k].x, j = ij[k].y;
    if (!eval_bond<double>(pos, i, j, par[k], dyn, F, rd, e)) return;      // calbond_hf.F90:102-147
    atomicAdd(h.pot + (size_t)PGK_HF_BO * h.natom + i, 0.5 * e);
    atomicAdd(h.pot + (size_t)PGK_HF_BO * h.natom + j, 0.5 * e);
    const double Fj[3] = {-F[0], -F[1], -F[2]};
    hf_calviri(h, pos, dyn->box[2], i, j, F, Fj, 0.5, PGK_HF_BO);
}

__global__ void k_angl_hf(const double* __restrict__ pos, const int4* __restrict__ ijk,
                          const double2* __restrict__ par, int nterm, const DynState* __restrict__ dyn, HfDev h) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nterm) return;
    double F[3][3], e;
    const int at[3] = {ijk[n].x, ijk[n].y, ijk[n].z};
    if (!eval_angl<double>(pos, at[0], at[1], at[2], par[n], dyn, F, e)) return;   // calangl_hf.F90:140-230
    const double c3 = 1.0 / 3.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) atomicAdd(h.pot + (size_t)PGK_HF_AN * h.natom + at[q], c3 * e);
    const double Lz = dyn->box[2];
    hf_calviri(h, pos, Lz, at[0], at[1], F[0], F[1], c3, PGK_HF_AN);
    hf_calviri(h, pos, Lz, at[1], at[2], F[1], F[2], c3, PGK_HF_AN);
    hf_calviri(h, pos, Lz, at[2], at[0], F[2], F[0], c3, PGK_HF_AN);
}

template <bool RB>
__global__ void k_tors_hf(const double* __restrict__ pos, const int4* __restrict__ ijkl,
                          const double4* __restrict__ par, const double* __restrict__ rbc, int nterm,
                          const DynState* __restrict__ dyn, HfDev h, unsigned* status) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nterm) return;
    const int at[4] = {ijkl[n].x, ijkl[n].y, ijkl[n].z, ijkl[n].w};
    double F[4][3], e;
    eval_tors<double, RB>(pos, at[0], at[1], at[2], at[3], RB ? make_double4(0, 0, 0, 0) : par[n],
                          RB ? rbc + 6 * (size_t)n : nullptr, dyn, F, e, status);
#pragma unroll
    for (int q = 0; q < 4; ++q) atomicAdd(h.pot + (size_t)PGK_HF_TO * h.natom + at[q], 0.25 * e);
    const double Lz = dyn->box[2];          // caltors_hf.F90 / caltorsrb_hf.F90:130-200
    hf_calviri(h, pos, Lz, at[0], at[1], F[0], F[1], 0.25, PGK_HF_TO);
    hf_calviri(h, pos, Lz, at[0], at[2], F[0], F[2], 0.25, PGK_HF_TO);
    hf_calviri(h, pos, Lz, at[0], at[3], F[0], F[3], 0.25, PGK_HF_TO);
    hf_calviri(h, pos, Lz, at[1], at[2], F[1], F[2], 0.25, PGK_HF_TO);
    hf_calviri(h, pos, Lz, at[1], at[3], F[1], F[3], 0.25, PGK_HF_TO);
    hf_calviri(h, pos, Lz, at[2], at[3], F[2], F[3], 0.25, PGK_HF_TO);
}

__global__ void k_non14_hf(const double* __restrict__ pos, const double* __restrict__ chrg,
                           const int* __restrict__ typ, const int2* __restrict__ ij, const double2* __restrict__ fac,
                           int nterm, int ntyp, const double2* __restrict__ lj64, const DynState* __restrict__ dyn,
                           HfDev h) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nterm) return;
    const int i = ij[n].x, j = ij[n].y;
    double F[3], rd[3], de, dv;
    eval_14<double>(pos, i, j, chrg[i] * chrg[j], lj64[typ[i] * ntyp + typ[j]], fac[n], dyn, F, rd, de, dv);
    // calnon14_hf.F90:160-250: Coulomb and LJ shares, calvirihf of both parts
    atomicAdd(h.pot + (size_t)PGK_HF_14 * h.natom + i, 0.5 * de + 0.5 * dv);
    atomicAdd(h.pot + (size_t)PGK_HF_14 * h.natom + j, 0.5 * de + 0.5 * dv);
    const double Fj[3] = {-F[0], -F[1], -F[2]};
    hf_calviri(h, pos, dyn->box[2], i, j, F, Fj, 0.5, PGK_HF_14);
}

pgk_status launch_bonded_hf(pgk_ctx* c, const HfDev& h) {
    const int tb = 128;
    auto on = [](int mts) { return mts == PGK_MTS_LONG || mts == PGK_MTS_SHORT; };
    if (c->nbond && on(c->prm.mts_bond)) {
        k_bond_hf<<<(c->nbond + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->bond_ij, c->bond_p, c->nbond, c->dyn, h);
        PGK_LAUNCHED(c);
    }
    if (c->nangl && on(c->prm.mts_angl)) {
        k_angl_hf<<<(c->nangl + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->angl_ijk, c->angl_p, c->nangl, c->dyn, h);
        PGK_LAUNCHED(c);
    }
    if (c->ntors && on(c->prm.mts_tors)) {
        k_tors_hf<false><<<(c->ntors + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->tors_ijkl, c->tors_p, nullptr,
                                                                      c->ntors, c->dyn, h, c->status);
        PGK_LAUNCHED(c);
    }
    if (c->ntorsrb && on(c->prm.mts_torsrb)) {
        k_tors_hf<true><<<(c->ntorsrb + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->rb_ijkl, nullptr, c->rb_c,
                                                                       c->ntorsrb, c->dyn, h, c->status);
        PGK_LAUNCHED(c);
    }
    if (c->n14 && on(c->prm.mts_vdw14) && c->prm.mts_vdw14 == c->prm.mts_elc14) {
        k_non14_hf<<<(c->n14 + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij, c->p14_f, c->n14,
                                                              c->ntyp, c->lj64, c->dyn, h);
        PGK_LAUNCHED(c);
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// One MTS group's bonded terms (mask bits: 0 bond, 1 angle, 2 periodic
// torsion, 3 RB torsion, 4 1-4 pairs, 5 excluded-pair Ewald correction): one
// kernel per active type writing the slots, then the per-atom gather.
template <bool MIXED>
static void terms_impl(pgk_ctx* c, int group, int mask, bool want) {
    long long* acc = c->acc + (size_t)group * NACC;
    const int w = want ? 1 : 0;
    const int tb = 128;
    const long long S = c->slot_base[6];
    auto out = [&](int ty) { return TermOut{c->facc[group], c->slot_f, S, c->slot_base[ty]}; };
    if ((mask & 1) && c->nbond) {
        k_bond<MIXED><<<(c->nbond + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->bond_ij, c->bond_p, c->nbond, c->dyn,
                                                                   out(0), acc, w);
        PGK_LAUNCHED(c);
    }
    if ((mask & 2) && c->nangl) {
        k_angl<MIXED><<<(c->nangl + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->angl_ijk, c->angl_p, c->nangl, c->dyn,
                                                                   out(1), acc, w);
        PGK_LAUNCHED(c);
    }
    if ((mask & 4) && c->ntors) {
        k_tors<MIXED, false><<<(c->ntors + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->tors_ijkl, c->tors_p, nullptr,
                                                                          c->ntors, c->dyn, out(2), acc, w, c->status);
        PGK_LAUNCHED(c);
    }
    if ((mask & 8) && c->ntorsrb) {
        k_tors<MIXED, true><<<(c->ntorsrb + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->rb_ijkl, nullptr, c->rb_c,
                                                                           c->ntorsrb, c->dyn, out(3), acc, w,
                                                                           c->status);
        PGK_LAUNCHED(c);
    }
    if ((mask & 16) && c->n14) {
        k_non14<MIXED><<<(c->n14 + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij, c->p14_f, c->n14,
                                                                  c->ntyp, c->lj64, c->dyn, out(4), acc, w);
        PGK_LAUNCHED(c);
    }
    if ((mask & 32) && c->nexpair) {
        k_excl<MIXED><<<(c->nexpair + 255) / 256, 256, 0, c->st>>>(c->pos, c->chrg, c->expair, c->nexpair, c->spl64,
                                                                    c->spl32, c->nspl, c->hspl, c->dyn, out(5), acc,
                                                                    w);
        PGK_LAUNCHED(c);
    }
    if (S > 0) {
        SlotTypes ty;
        for (int q = 0; q < 7; ++q) ty.base[q] = c->slot_base[q];
        k_slot_gather<MIXED><<<(c->natom + 255) / 256, 256, 0, c->st>>>(c->inc_start, c->inc_slot, c->slot_f, ty,
                                                                         mask, c->natom, c->facc[group]);
        PGK_LAUNCHED(c);
    }
}

pgk_status launch_intra(pgk_ctx* c, int group, int mask, bool want) {
    const long long cnt[6] = {c->nbond, c->nangl, c->ntors, c->ntorsrb, c->n14, c->nexpair};
    int active = 0;
    for (int ty = 0; ty < 6; ++ty) if (((mask >> ty) & 1) && cnt[ty] > 0) active |= 1 << ty;
    if (!active) return PGK_OK;
    if (c->mixed()) terms_impl<true>(c, group, active, want);
    else terms_impl<false>(c, group, active, want);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// all bonded terms (the MTS assignment ignored) or only those of the group
pgk_status launch_bonded(pgk_ctx* c, int group, bool ene, bool vir, bool force_all) {
    auto on = [&](int mts) { return force_all || mts == (group == 0 ? PGK_MTS_LONG : PGK_MTS_SHORT); };
    const int mask = (on(c->prm.mts_bond) ? 1 : 0) | (on(c->prm.mts_angl) ? 2 : 0) | (on(c->prm.mts_tors) ? 4 : 0) |
                     (on(c->prm.mts_torsrb) ? 8 : 0) |
                     ((force_all || (on(c->prm.mts_vdw14) && c->prm.mts_vdw14 == c->prm.mts_elc14)) ? 16 : 0);
    return launch_intra(c, group, mask, ene || vir);
}

pgk_status launch_excl(pgk_ctx* c, int group, bool ene, bool vir) {
    return launch_intra(c, group, 32, ene || vir);
}
