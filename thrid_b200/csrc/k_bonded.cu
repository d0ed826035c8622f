// k_bonded.cu -- intramolecular terms:
//   calbondp   calbond.F90:109-219      U = k (r - r0)^2
//   calanglp   calangl.F90:172-358      U = k (theta - theta0)^2
//   caltorsp   caltors.F90 (+calijkl)   U = V/div (1 + cos(n phi - phase))
//   caltorsrbp caltorsrb.F90:118-459    U = sum_n C_n (-1)^n cos^n phi
//   calnon14p  calnon14.F90:249-521     scaled 1-4 Coulomb + LJ
//   ewaldrp excluded-pair erf correction (ewaldr.F90:756-826)
//
// Layout: bonded_setup cuts the atoms into blocks of consecutive atoms; block
// b owns the terms whose lowest atom lies in its range (terms sorted by lowest
// atom), stages the positions of its local atoms (owned range plus the
// higher atoms its terms reach) in shared memory, evaluates its terms with
// one thread per term, writes each term atom's force into a shared-memory
// slot, and then sums every local atom's slots in a fixed order (a
// precomputed per-block incidence list) and adds the total to the group's
// force accumulator once per block.  No atomics inside the block; the
// per-atom sums are deterministic.  Terms spanning BLK_FAR_SPAN atoms or more
// (rare: e.g. a disulfide bond) run in the per-type kernels with force
// atomics.  Energies and virials are block-reduced per type.
//
// Displacements are formed in FP64 from the master positions (Fortran anint
// minimum image); the remaining arithmetic runs in T (float for mixed).
// Angle and torsion virials use absolute coordinates exactly like the
// reference (sum f_a x_b over the term's atoms).
#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <vector>

#include "pgk_ctx.cuh"
#include "pgk_hf.cuh"

// block plan limits: local atoms per block, the atom span from which a term
// is "far", threads per block, slots per block (shared-memory slot planes)
#define BLK_LOC_MAX 512
#define BLK_FAR_SPAN 256
#define BLK_THREADS 256
#define BLK_SLOT_CAP_MAX 4096
static inline int blk_slot_cap(bool mixed) { return mixed ? BLK_SLOT_CAP_MAX : 2048; }


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

// the per-type kernels (far terms) add their forces with atomics
template <bool MIXED>
__device__ __forceinline__ void put_force(void* facc, int atom, const double* F, double sgn) {
    force_add<MIXED>(facc, atom, sgn * F[0], sgn * F[1], sgn * F[2]);
}

// ---- term evaluators (P = positions, indices into P) ------------------------
template <typename T>
__device__ __forceinline__ bool eval_bond(const double* P, int i, int j, double2 p, const DynState* dyn,
                                          double (&F)[3], double (&rd)[3], double& pot) {
    if (fabs(p.x) < 1.0e-16) return false;
    // the stretch r - r0 is a small difference of two ~1.5 A lengths: formed in
    // FP64 in both precisions (in FP32 its rounding alone is ~1e-5 of a
    // thermal stretch); the force arithmetic after it runs in T
    double r64[3];
    disp<double>(P, i, j, dyn, r64);
    const double rr64 = sqrt(r64[0] * r64[0] + r64[1] * r64[1] + r64[2] * r64[2]);
    const T r[3] = {(T)r64[0], (T)r64[1], (T)r64[2]};
    const T rr = (T)rr64;
    const T dr = (T)(rr64 - p.y);
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

// the same with the pair's constants formed once at setup:
// K = (q_i q_j elc fac, R^2, eps vdw fac, 0)
template <typename T>
__device__ __forceinline__ void eval_14k(const double* P, int i, int j, double4 K, const DynState* dyn,
                                         double (&F)[3], double (&rd)[3], double& de_out, double& dv_out) {
    T r[3];
    disp<T>(P, i, j, dyn, r);
    T r2 = dt3(r, r);
    T ri2 = T(1) / r2, ri1 = sqrt(ri2);
    T de = (T)K.x * ri1;
    T t2 = ri2 * (T)K.y, t6 = t2 * t2 * t2, t12 = t6 * t6;
    T E = (T)K.z;
    T dv = E * (t12 - T(2) * t6);
    T ft = T(12) * E * (t12 - t6) * ri2;
    T fs = de * ri2 + ft;
#pragma unroll
    for (int d = 0; d < 3; ++d) { F[d] = (double)(fs * r[d]); rd[d] = (double)r[d]; }
    de_out = (double)de;
    dv_out = (double)dv;
}

// ---- mixed-precision force-and-tensor forms (tensor-only steps) ---------------
// Same forces as eval_angl / eval_tors in FP32 without the energy: no inverse
// trigonometry in the torsion (the force factor is a polynomial in cos phi,
// sin^2 phi = 1 - cos^2 phi), sin(theta) = sqrt(1 - cos^2 theta) in the angle,
// reciprocals instead of divisions.  The caller forms the virial from lever
// arms relative to the term's first atom (the term forces sum to zero), so the
// FP32 tensor sums do not cancel absolute coordinates.
__device__ __forceinline__ void angl_force_f(const double* P, int i, int j, int k, double2 p,
                                             const DynState* dyn, float (&F)[3][3], float (&arm)[3][3]) {
    float rij[3], rkj[3];
    disp<float>(P, j, i, dyn, rij);
    disp<float>(P, j, k, dyn, rkj);
    const float ia = rsqrtf(dt3(rij, rij)), ib = rsqrtf(dt3(rkj, rkj));
    float c = dt3(rij, rkj) * ia * ib;
    c = fminf(fmaxf(c, -1.f), 1.f);
    const float th = acosf(c);
    const float s = sqrtf(fmaxf(1.f - c * c, 0.f));
    const float dth = th - (float)p.y;
    float fi[3] = {0, 0, 0}, fk[3] = {0, 0, 0};
    if (s > 1.0e-7f) {
        const float ft = -2.f * (float)p.x * dth / s;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            fi[d] = ft * ((rkj[d] * ib - rij[d] * c * ia) * ia);
            fk[d] = ft * ((rij[d] * ia - rkj[d] * c * ib) * ib);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        F[0][d] = fi[d]; F[1][d] = -fi[d] - fk[d]; F[2][d] = fk[d];
        arm[0][d] = 0.f; arm[1][d] = rij[d]; arm[2][d] = rij[d] - rkj[d];   // x_q - x_i
    }
}

template <bool RB>
__device__ __forceinline__ void tors_force_f(const double* P, int i, int j, int k, int l, double4 p,
                                             const double* __restrict__ C, const DynState* dyn, float (&F)[4][3],
                                             float (&arm)[4][3], unsigned* status) {
    float rij[3], rkj[3], rkl[3];
    disp<float>(P, j, i, dyn, rij); disp<float>(P, j, k, dyn, rkj); disp<float>(P, l, k, dyn, rkl);
    float rik[3], rjl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { rik[d] = rij[d] - rkj[d]; rjl[d] = rkl[d] - rkj[d]; }
    float ni[3], nl[3];
    crs(rij, rkj, ni);
    crs(rkj, rkl, nl);
    const float iai = rsqrtf(dt3(ni, ni)), ial = rsqrtf(dt3(nl, nl));
    float c = dt3(ni, nl) * iai * ial;
    c = fminf(fmaxf(c, -1.f), 1.f);
    float b[3], cc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float a = ni[d] * iai, e = nl[d] * ial;
        b[d] = (e - c * a) * iai;
        cc[d] = (a - c * e) * ial;
    }
    float fa;
    if (RB) {
        const float bt[6] = {(float)C[0], -(float)C[1], (float)C[2], -(float)C[3], (float)C[4], -(float)C[5]};
        float dp = bt[5];
        fa = 0.f;
#pragma unroll
        for (int q = 4; q >= 0; --q) { fa = fa * c + dp; dp = dp * c + bt[q]; }
        fa = -fa;
    } else {
        const int np = (int)lround(p.z);
        if (np == 1) fa = 1.f;
        else if (np == 2) fa = 2.f * c;
        else if (np == 3) fa = 4.f * c * c - 1.f;          // -4 sin^2 + 3
        else if (np == 4) fa = 4.f * c * (2.f * c * c - 1.f);
        else if (np == 5) { fa = 4.f * c * c; fa = fa * (fa - 3.f) + 1.f; }
        else if (np == 6) { fa = 4.f * c * c; fa = 2.f * c * (fa - 3.f) * (fa - 1.f); }
        else { fa = 0.f; atomicOr(status, ST_UNSUPPORTED); }
        fa = -fa * (float)p.w * (float)p.x * (float)p.z;
    }
    float t1[3], t2[3];
    crs(b, rkj, t1);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[0][d] = fa * t1[d];
    crs(cc, rkl, t1); crs(b, rik, t2);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[1][d] = fa * (-t1[d] + t2[d]);
    crs(b, rij, t1); crs(cc, rjl, t2);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[2][d] = fa * (-t1[d] + t2[d]);
    crs(cc, rkj, t1);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        F[3][d] = fa * t1[d];
        arm[0][d] = 0.f; arm[1][d] = rij[d]; arm[2][d] = rik[d]; arm[3][d] = rik[d] + rkl[d];   // x_q - x_i
    }
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
        if (rr == rr && idx >= 0 && idx < nspl - 1) {     // a non-finite distance reads no table
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
                       int nterm, const DynState* __restrict__ dyn, void* facc, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < nterm) {
        double F[3] = {0, 0, 0}, rd[3], e;
        int i = ij[k].x, j = ij[k].y;
        const bool on = eval_bond<T>(pos, i, j, par[k], dyn, F, rd, e);
        put_force<MIXED>(facc, i, F, 1.0);
        put_force<MIXED>(facc, j, F, -1.0);
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
                       int nterm, const DynState* __restrict__ dyn, void* facc, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (n < nterm) {
        double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e;
        int at[3] = {ijk[n].x, ijk[n].y, ijk[n].z};
        const bool on = eval_angl<T>(pos, at[0], at[1], at[2], par[n], dyn, F, e);
#pragma unroll
        for (int q = 0; q < 3; ++q) put_force<MIXED>(facc, at[q], F[q], 1.0);
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
                       const double* __restrict__ rbc, int nterm, const DynState* __restrict__ dyn, void* facc,
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
        for (int q = 0; q < 4; ++q) put_force<MIXED>(facc, at[q], F[q], 1.0);
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
                        const double2* __restrict__ lj64, const DynState* __restrict__ dyn, void* facc,
                        long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[12] = {0};
    if (n < nterm) {
        int i = ij[n].x, j = ij[n].y;
        double F[3], rd[3], de, dv;
        eval_14<T>(pos, i, j, chrg[i] * chrg[j], lj64[typ[i] * ntyp + typ[j]], fac[n], dyn, F, rd, de, dv);
        put_force<MIXED>(facc, i, F, 1.0);
        put_force<MIXED>(facc, j, F, -1.0);
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
                       void* facc, long long* acc, int want) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < npair) {
        int i = pairs[k].x, j = pairs[k].y;
        double F[3], rd[3], e;
        eval_excl<MIXED>(pos, i, j, chrg[i] * chrg[j], spl64, spl32, nspl, h, dyn, F, rd, e);
        put_force<MIXED>(facc, i, F, 1.0);
        put_force<MIXED>(facc, j, F, -1.0);
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

// ---- block kernel (near terms) ---------------------------------------------------
// what the block kernel reads besides positions and the block plan: the
// compact near-term records and parameter tables of each type (bonded_setup)
// and the spline tables of the excluded-pair correction
struct TermsDev {
    const double4* spl64; const float4* spl32; int nspl; double hspl;
    const uint2* rec[6]; const double* tab[6];
};
struct BlkDev {
    const int* a0; const int* nloc; const int* t; const int* soff; const int* ip; const int* incp;
    const unsigned short* inc;
    int nblk, smax;
};

// compact near-term record (bonded_setup): four 9-bit block-local atom
// indices and a 28-bit index into the type's parameter table
__device__ __forceinline__ void rec_atoms(uint2 r, int (&at)[4]) {
    at[0] = (int)(r.x & 511u);
    at[1] = (int)((r.x >> 9) & 511u);
    at[2] = (int)((r.x >> 18) & 511u);
    at[3] = (int)((r.x >> 27) | ((r.y & 15u) << 5));
}
__device__ __forceinline__ unsigned rec_par(uint2 r) { return r.y >> 4; }

// TENS: the steps that need only the total bonded virial tensor (anisotropic
// MTK steps without output): one 9-entry tensor summed over all types into
// the bond tensor slot, no energies, one block reduction.  Otherwise every
// type's energy, scalar virial and tensor, reduced per type.
template <bool MIXED, bool TENS>
__global__ void __launch_bounds__(BLK_THREADS, 2) k_intra_blk(const double* __restrict__ pos, TermsDev D, BlkDev K,
                                                              const DynState* __restrict__ dyn, void* facc,
                                                              long long* acc, int mask, int want, unsigned* status) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    extern __shared__ __align__(16) double sh[];
    __shared__ int so[8];
    const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int a0 = K.a0[b], nloc = K.nloc[b];
    double* P = sh;                                          // [BLK_LOC_MAX][3] local positions
    T* SX = (T*)(sh + 3 * BLK_LOC_MAX);                      // [3][smax] slot forces
    T* SY = SX + K.smax;
    T* SZ = SY + K.smax;
    int* IP = (int*)(SZ + K.smax);                           // [BLK_LOC_MAX+1] incidence pointers
    unsigned short* INC = (unsigned short*)(IP + BLK_LOC_MAX + 4);   // [smax] incidence (16-byte aligned)
    const int* ipg = K.incp + K.ip[b];
    // The block's terms of all enabled types as one sequence dealt round-robin
    // to the threads (term v to thread v mod nt), so every thread gets about
    // the same number of terms and no warp waits at the block's barriers for
    // another that drew the leftovers of every type.  sT[ty] = (first term,
    // end, position of the type's first term in the sequence), written by
    // warp 0 beside the staging loads.
    __shared__ int sT[6][3];
    if (tid < 32) {
        int t0 = 0, t1 = 0;
        if (tid < 6) { t0 = K.t[tid * (K.nblk + 1) + b]; t1 = K.t[tid * (K.nblk + 1) + b + 1]; }
        const int cnt = tid < 6 && ((mask >> tid) & 1) ? t1 - t0 : 0;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (tid >= o) incl += y;
        }
        if (tid < 6) { sT[tid][0] = t0; sT[tid][1] = t1; sT[tid][2] = incl - cnt; }
    }
    const int inc0 = ipg[0], ninc = ipg[nloc] - inc0;
    {
        // staging: every load of a thread is issued before its stores (the
        // sizes are bounded: 3*BLK_LOC_MAX doubles, BLK_LOC_MAX+1 pointers,
        // smax slot ids stored as 16-byte groups from a 16-byte aligned start)
        constexpr int NP = (3 * BLK_LOC_MAX + BLK_THREADS - 1) / BLK_THREADS;
        constexpr int NI = (BLK_LOC_MAX + 1 + BLK_THREADS - 1) / BLK_THREADS;
        constexpr int NV = (BLK_SLOT_CAP_MAX / 8 + BLK_THREADS - 1) / BLK_THREADS;
        double rp[NP];
        int ri[NI];
        uint4 rv[NV];
        const uint4* incv = (const uint4*)(K.inc + inc0);
        const int nv = (ninc + 7) / 8;
#pragma unroll
        for (int q = 0; q < NP; ++q) { const int l = tid + q * nt; if (l < 3 * nloc) rp[q] = pos[3 * (size_t)a0 + l]; }
#pragma unroll
        for (int q = 0; q < NI; ++q) { const int l = tid + q * nt; if (l <= nloc) ri[q] = ipg[l]; }
#pragma unroll
        for (int q = 0; q < NV; ++q) { const int l = tid + q * nt; if (l < nv) rv[q] = incv[l]; }
        if (tid < 8) so[tid] = K.soff[8 * b + tid];
#pragma unroll
        for (int q = 0; q < NP; ++q) { const int l = tid + q * nt; if (l < 3 * nloc) P[l] = rp[q]; }
#pragma unroll
        for (int q = 0; q < NI; ++q) { const int l = tid + q * nt; if (l <= nloc) IP[l] = ri[q] - inc0; }
#pragma unroll
        for (int q = 0; q < NV; ++q) { const int l = tid + q * nt; if (l < nv) ((uint4*)INC)[l] = rv[q]; }
    }
    __syncthreads();
    auto put = [&](int sl, const double* F, double sg) {
        SX[sl] = (T)(sg * F[0]); SY[sl] = (T)(sg * F[1]); SZ[sl] = (T)(sg * F[2]);
    };
    // this thread's first term of a type; the records: each type's loop loads
    // the next record one term ahead, and at its start the first record of
    // the next enabled type (carry), so no record load waits in the open
    auto kfirst = [&](int ty) { return sT[ty][0] + ((tid - sT[ty][2]) % nt + nt) % nt; };
    auto rec_at = [&](int ty, int k) {       // constant indices into D.rec (no local copy of D)
        switch (ty) {
            case 0: return __ldg(D.rec[0] + k);
            case 1: return __ldg(D.rec[1] + k);
            case 2: return __ldg(D.rec[2] + k);
            case 3: return __ldg(D.rec[3] + k);
            case 4: return __ldg(D.rec[4] + k);
            default: return __ldg(D.rec[5] + k);
        }
    };
    auto first_rec = [&](int ty) {
        const int k = kfirst(ty);
        return k < sT[ty][1] ? rec_at(ty, k) : make_uint2(0u, 0u);
    };
    auto next_rec = [&](int ty, int k) {
        return k + nt < sT[ty][1] ? __ldg(D.rec[ty] + k + nt) : make_uint2(0u, 0u);
    };
    auto carry_after = [&](int ty) {
        int u = ty + 1;
        while (u < 6 && !((mask >> u) & 1)) ++u;
        return u < 6 ? first_rec(u) : make_uint2(0u, 0u);
    };
    uint2 carry = carry_after(-1);
    double tv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};               // TENS: total tensor (a + 3b)
    float tvf[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};               // mixed TENS: FP32 sums of lever-arm terms
    constexpr bool FAST = MIXED && TENS;
    auto tens_pair = [&](const double* F, const double* r) {
#pragma unroll
        for (int bb = 0; bb < 3; ++bb)
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) {
                if (FAST) tvf[aa + 3 * bb] = fmaf((float)F[aa], (float)r[bb], tvf[aa + 3 * bb]);
                else tv[aa + 3 * bb] += F[aa] * r[bb];
            }
    };
    auto tens_arm = [&](const float* F, const float* r) {
#pragma unroll
        for (int bb = 0; bb < 3; ++bb)
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) tvf[aa + 3 * bb] = fmaf(F[aa], r[bb], tvf[aa + 3 * bb]);
    };
    auto tens_abs = [&](const double* F, int l) {
#pragma unroll
        for (int bb = 0; bb < 3; ++bb)
#pragma unroll
            for (int aa = 0; aa < 3; ++aa) tv[aa + 3 * bb] += F[aa] * P[3 * l + bb];
    };
    const bool full = want && !TENS;
    if (mask & 1) {
        const int t0 = sT[0][0], t1 = sT[0][1];
        double v[11] = {0};
        uint2 r = carry, rn;
        carry = carry_after(0);
        for (int k = kfirst(0); k < t1; k += nt, r = rn) {
            rn = next_rec(0, k);
            int at[4];
            rec_atoms(r, at);
            double F[3] = {0, 0, 0}, rd[3], e;
            const bool on = eval_bond<T>(P, at[0], at[1], __ldg((const double2*)D.tab[0] + rec_par(r)), dyn, F, rd, e);
            const int sl = so[0] + 2 * (k - t0);
            put(sl, F, 1.0); put(sl + 1, F, -1.0);
            if (TENS && on) tens_pair(F, rd);
            if (full && on) { v[0] += e; vir_pair(v + 1, F, rd); }
        }
        if (full) {
            const int idx[11] = {A_BOND, A_VB, A_VTB + 0, A_VTB + 1, A_VTB + 2, A_VTB + 3, A_VTB + 4, A_VTB + 5,
                                 A_VTB + 6, A_VTB + 7, A_VTB + 8};
            block_acc<11>(v, acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (mask & 2) {
        const int t0 = sT[1][0], t1 = sT[1][1];
        double v[11] = {0};
        uint2 r = carry, rn;
        carry = carry_after(1);
        for (int k = kfirst(1); k < t1; k += nt, r = rn) {
            rn = next_rec(1, k);
            int at[4];
            rec_atoms(r, at);
            const double2 pp = __ldg((const double2*)D.tab[1] + rec_par(r));
            const int sl = so[1] + 3 * (k - t0);
            if (FAST) {
                float Ff[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, arm[3][3];
                if (fabs(pp.x) >= 1.0e-32) {
                    angl_force_f(P, at[0], at[1], at[2], pp, dyn, Ff, arm);
#pragma unroll
                    for (int q = 0; q < 3; ++q) tens_arm(Ff[q], arm[q]);
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) { SX[sl + q] = Ff[q][0]; SY[sl + q] = Ff[q][1]; SZ[sl + q] = Ff[q][2]; }
                continue;
            }
            double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e;
            const bool on = eval_angl<T>(P, at[0], at[1], at[2], pp, dyn, F, e);
#pragma unroll
            for (int q = 0; q < 3; ++q) put(sl + q, F[q], 1.0);
            if (TENS && on) {
#pragma unroll
                for (int q = 0; q < 3; ++q) tens_abs(F[q], at[q]);
            }
            if (full && on) {
                v[0] += e;
#pragma unroll
                for (int q = 0; q < 3; ++q) vir_abs(v + 1, F[q], P, at[q]);
            }
        }
        if (full) {
            const int idx[11] = {A_ANGL, A_VA, A_VTA + 0, A_VTA + 1, A_VTA + 2, A_VTA + 3, A_VTA + 4, A_VTA + 5,
                                 A_VTA + 6, A_VTA + 7, A_VTA + 8};
            block_acc<11>(v, acc, idx, !MIXED);
            __syncthreads();
        }
    }
#pragma unroll
    for (int rb = 0; rb < 2; ++rb) {
        if (!(mask & (4 << rb))) continue;
        const int t0 = sT[2 + rb][0], t1 = sT[2 + rb][1];
        double v[11] = {0};
        uint2 r = carry, rn;
        carry = carry_after(2 + rb);
        for (int k = kfirst(2 + rb); k < t1; k += nt, r = rn) {
            rn = next_rec(2 + rb, k);
            int at[4];
            rec_atoms(r, at);
            const unsigned pi = rec_par(r);
            const double4 tp = rb ? make_double4(0, 0, 0, 0) : ((const double4*)D.tab[2])[pi];
            const double* C = rb ? D.tab[3] + 6 * (size_t)pi : nullptr;
            if (FAST) {
                float Ff[4][3], arm[4][3];
                if (rb) tors_force_f<true>(P, at[0], at[1], at[2], at[3], tp, C, dyn, Ff, arm, status);
                else tors_force_f<false>(P, at[0], at[1], at[2], at[3], tp, nullptr, dyn, Ff, arm, status);
                const int slf = so[2 + rb] + 4 * (k - t0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    tens_arm(Ff[q], arm[q]);
                    SX[slf + q] = Ff[q][0]; SY[slf + q] = Ff[q][1]; SZ[slf + q] = Ff[q][2];
                }
                continue;
            }
            double F[4][3], e;
            if (rb) eval_tors<T, true>(P, at[0], at[1], at[2], at[3], tp, C, dyn, F, e, status);
            else eval_tors<T, false>(P, at[0], at[1], at[2], at[3], tp, nullptr, dyn, F, e, status);
            const int sl = so[2 + rb] + 4 * (k - t0);
#pragma unroll
            for (int q = 0; q < 4; ++q) put(sl + q, F[q], 1.0);
            if (TENS) {
#pragma unroll
                for (int q = 0; q < 4; ++q) tens_abs(F[q], at[q]);
            }
            if (full) {
                v[0] += e;
#pragma unroll
                for (int q = 0; q < 4; ++q) vir_abs(v + 1, F[q], P, at[q]);
            }
        }
        if (full) {
            const int idx[11] = {rb ? A_TORSRB : A_TORS, A_VT, A_VTT + 0, A_VTT + 1, A_VTT + 2, A_VTT + 3,
                                 A_VTT + 4, A_VTT + 5, A_VTT + 6, A_VTT + 7, A_VTT + 8};
            block_acc<11>(v, acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (mask & 16) {
        const int t0 = sT[4][0], t1 = sT[4][1];
        double v[12] = {0};
        uint2 r = carry, rn;
        carry = carry_after(4);
        for (int k = kfirst(4); k < t1; k += nt, r = rn) {
            rn = next_rec(4, k);
            int at[4];
            rec_atoms(r, at);
            double F[3], rd[3], de, dv;
            eval_14k<T>(P, at[0], at[1], ((const double4*)D.tab[4])[rec_par(r)], dyn, F, rd, de, dv);
            const int sl = so[4] + 2 * (k - t0);
            put(sl, F, 1.0); put(sl + 1, F, -1.0);
            if (TENS) tens_pair(F, rd);
            if (full) { v[0] += de; v[1] += dv; vir_pair(v + 2, F, rd); }
        }
        if (full) {
            const int idx[12] = {A_ELC14, A_VDW14, A_V14, A_VT14 + 0, A_VT14 + 1, A_VT14 + 2, A_VT14 + 3,
                                 A_VT14 + 4, A_VT14 + 5, A_VT14 + 6, A_VT14 + 7, A_VT14 + 8};
            block_acc<12>(v, acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (mask & 32) {
        const int t0 = sT[5][0], t1 = sT[5][1];
        double v[11] = {0};
        uint2 r = carry, rn;
        carry = carry_after(5);
        for (int k = kfirst(5); k < t1; k += nt, r = rn) {
            rn = next_rec(5, k);
            int at[4];
            rec_atoms(r, at);
            double F[3], rd[3], e;
            eval_excl<MIXED>(P, at[0], at[1], __ldg(D.tab[5] + rec_par(r)), D.spl64, D.spl32, D.nspl, D.hspl, dyn, F,
                             rd, e);
            const int sl = so[5] + 2 * (k - t0);
            put(sl, F, 1.0); put(sl + 1, F, -1.0);
            if (TENS) tens_pair(F, rd);
            if (full) { v[0] -= e; vir_pair(v + 1, F, rd); }
        }
        if (full) {
            // pot_elc -= potij; pot_viri_coul -= potij; tensor (lower triangle) += f r
            double w[8] = {v[0], v[0], v[2], v[3], v[4], v[6], v[7], v[10]};
            const int idx[8] = {A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
            block_acc<8>(w, acc, idx, !MIXED);
        }
    }
    if (TENS && want) {
        const int idx[9] = {A_VTB + 0, A_VTB + 1, A_VTB + 2, A_VTB + 3, A_VTB + 4, A_VTB + 5, A_VTB + 6, A_VTB + 7,
                            A_VTB + 8};
        if (FAST) {
#pragma unroll
            for (int q = 0; q < 9; ++q) tv[q] = (double)tvf[q];
        }
        block_acc<9>(tv, acc, idx, !MIXED);
    }
    __syncthreads();
    // per local atom: its slots in incidence order (types outside mask hold
    // nothing of this evaluation and are skipped)
    for (int l = tid; l < nloc; l += nt) {
        const int p0 = IP[l], p1 = IP[l + 1];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        bool any = false;
        for (int p = p0; p < p1; ++p) {
            const int sl = INC[p];
            int ty = 0;
#pragma unroll
            for (int q = 1; q < 6; ++q) ty += sl >= so[q] ? 1 : 0;
            if (!((mask >> ty) & 1)) continue;
            fx += (double)SX[sl]; fy += (double)SY[sl]; fz += (double)SZ[sl];
            any = true;
        }
        if (any) force_add<MIXED>(facc, a0 + l, fx, fy, fz);
    }
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
    PGK_CUDA(c, pgk_dmalloc(c, dst, v.size() * sizeof(T)));
    PGK_CUDA(c, cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PGK_OK;
}

// Term arrays: per type the near terms (atom span < BLK_FAR_SPAN) first,
// ordered by their lowest atom, then the far ones.  Block plan: consecutive
// lowest atoms are gathered into blocks while the block's slots fit the
// shared-memory slot planes and its local atom range fits BLK_LOC_MAX; each
// block's incidence list gives every local atom its slots by type, term and
// position in the term.
pgk_status bonded_setup(pgk_ctx* c, HostTerms& t, const std::vector<int>&, const std::vector<int>&) {
    const int n = c->natom;
    const int K[6] = {2, 3, 4, 4, 2, 2};
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
    auto lo_hi = [&](int ty, long long k, int& lo, int& hi) {
        int at[4];
        atoms_of(ty, k, at);
        lo = hi = at[0];
        for (int q = 1; q < K[ty]; ++q) { lo = std::min(lo, at[q]); hi = std::max(hi, at[q]); }
    };
    const int count0[6] = {(int)t.bij.size(), (int)t.aijk.size(), (int)t.tij.size(), (int)t.rij.size(),
                           (int)t.p14.size(), (int)t.ex.size()};
    for (int ty = 0; ty < 6; ++ty) {
        std::vector<long long> key(count0[ty]);
        int nnear = 0;
        for (int k = 0; k < count0[ty]; ++k) {
            int lo, hi;
            lo_hi(ty, k, lo, hi);
            const bool far = hi - lo >= BLK_FAR_SPAN;
            key[k] = ((long long)(far ? 1 : 0) << 32) | (long long)lo;
            nnear += far ? 0 : 1;
        }
        std::vector<int> o(count0[ty]);
        for (int k = 0; k < count0[ty]; ++k) o[k] = k;
        std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return key[x] < key[y]; });
        switch (ty) {
            case 0: reorder(t.bij, o); reorder(t.bp, o); break;
            case 1: reorder(t.aijk, o); reorder(t.ap, o); break;
            case 2: reorder(t.tij, o); reorder(t.tp, o); break;
            case 3: {
                std::vector<double> rc2(t.rc.size());
                for (size_t k = 0; k < o.size(); ++k)
                    for (int q = 0; q < 6; ++q) rc2[6 * k + q] = t.rc[6 * o[k] + q];
                reorder(t.rij, o);
                t.rc.swap(rc2);
                break;
            }
            case 4: reorder(t.p14, o); reorder(t.f14, o); break;
            default: reorder(t.ex, o); break;
        }
        c->nnear[ty] = nnear;
    }
    pgk_status s;
    c->nbond = count0[0]; c->nangl = count0[1]; c->ntors = count0[2];
    c->ntorsrb = count0[3]; c->n14 = count0[4]; c->nexpair = count0[5];
    if ((s = up(c, &c->bond_ij, t.bij)) || (s = up(c, &c->bond_p, t.bp)) || (s = up(c, &c->angl_ijk, t.aijk)) ||
        (s = up(c, &c->angl_p, t.ap)) || (s = up(c, &c->tors_ijkl, t.tij)) || (s = up(c, &c->tors_p, t.tp)) ||
        (s = up(c, &c->rb_ijkl, t.rij)) || (s = up(c, &c->rb_c, t.rc)) || (s = up(c, &c->p14_ij, t.p14)) ||
        (s = up(c, &c->p14_f, t.f14)) || (s = up(c, &c->expair, t.ex)))
        return s;
    // per-term constants of the 1-4 and excluded pairs (charges, types and
    // LJ parameters are fixed at init), entries of the block kernel's
    // parameter tables below: one table read per term instead of the chain
    // charges -> types -> LJ row
    if (!t.q || !t.ty || !t.lj) return pgk_fail(c, PGK_E_INVALID, "bonded setup without atom data");
    std::vector<double4> k14(t.p14.size());
    for (size_t k = 0; k < t.p14.size(); ++k) {
        const int i = t.p14[k].x, j = t.p14[k].y;
        const double2 lp = t.lj[t.ty[i] * t.ntyp + t.ty[j]];
        k14[k] = make_double4(t.q[i] * t.q[j] * t.f14[k].x, lp.x, lp.y * t.f14[k].y, 0.0);
    }
    std::vector<double> qex(t.ex.size());
    for (size_t k = 0; k < t.ex.size(); ++k) qex[k] = t.q[t.ex[k].x] * t.q[t.ex[k].y];

    // ---- block plan ----
    const int cap = blk_slot_cap(c->mixed());
    std::vector<int> a0v, nlocv, soffv, ipv, incp;
    std::vector<int> tst[6];
    std::vector<unsigned short> inc;
    int ptr[6] = {0, 0, 0, 0, 0, 0};
    int cur_a0 = -1, cur_hi = -1, cur_slots = 0;
    int start[6];
    auto close_block = [&](const int* end) {
        const int b0 = cur_a0, nloc = cur_hi - cur_a0 + 1;
        int off[8];
        off[0] = 0;
        for (int ty = 0; ty < 6; ++ty) off[ty + 1] = off[ty] + K[ty] * (end[ty] - start[ty]);
        off[7] = 0;
        a0v.push_back(b0);
        nlocv.push_back(nloc);
        for (int q = 0; q < 8; ++q) soffv.push_back(off[q]);
        for (int ty = 0; ty < 6; ++ty) tst[ty].push_back(start[ty]);
        ipv.push_back((int)incp.size());
        std::vector<int> deg(nloc + 1, 0);
        int at[4];
        for (int ty = 0; ty < 6; ++ty)
            for (int k = start[ty]; k < end[ty]; ++k) {
                atoms_of(ty, k, at);
                for (int q = 0; q < K[ty]; ++q) deg[at[q] - b0 + 1]++;
            }
        for (int l = 0; l < nloc; ++l) deg[l + 1] += deg[l];
        const int base = (int)inc.size();            // a multiple of 8: 16-byte aligned groups
        for (int l = 0; l <= nloc; ++l) incp.push_back(base + deg[l]);
        inc.resize(base + ((deg[nloc] + 7) & ~7), 0);
        std::vector<int> fill(deg.begin(), deg.end() - 1);
        for (int ty = 0; ty < 6; ++ty)
            for (int k = start[ty]; k < end[ty]; ++k) {
                atoms_of(ty, k, at);
                for (int q = 0; q < K[ty]; ++q)
                    inc[base + fill[at[q] - b0]++] = (unsigned short)(off[ty] + K[ty] * (k - start[ty]) + q);
            }
    };
    for (int a = 0; a < n; ++a) {
        int end[6], slots = 0, hi = -1;
        for (int ty = 0; ty < 6; ++ty) {
            int k = ptr[ty];
            for (; k < c->nnear[ty]; ++k) {
                int lo, h;
                lo_hi(ty, k, lo, h);
                if (lo != a) break;
                slots += K[ty];
                hi = std::max(hi, h);
            }
            end[ty] = k;
        }
        if (slots == 0) continue;
        if (slots > cap)
            return pgk_fail(c, PGK_E_UNSUPPORTED, "too many bonded terms share one lowest atom");
        if (cur_a0 >= 0 && (cur_slots + slots > cap || std::max(cur_hi, hi) - cur_a0 + 1 > BLK_LOC_MAX)) {
            close_block(ptr);
            cur_a0 = -1;
        }
        if (cur_a0 < 0) {
            cur_a0 = a; cur_hi = hi; cur_slots = 0;
            for (int ty = 0; ty < 6; ++ty) start[ty] = ptr[ty];
        }
        cur_slots += slots;
        cur_hi = std::max(cur_hi, hi);
        for (int ty = 0; ty < 6; ++ty) ptr[ty] = end[ty];
    }
    if (cur_a0 >= 0) close_block(ptr);
    c->nblk = (int)a0v.size();
    if (c->nblk == 0) return PGK_OK;
    std::vector<int> tall;
    for (int ty = 0; ty < 6; ++ty) {
        tall.insert(tall.end(), tst[ty].begin(), tst[ty].end());
        tall.push_back(ptr[ty]);          // end of the last block
    }
    if ((s = up(c, &c->blk_a0, a0v)) || (s = up(c, &c->blk_nloc, nlocv)) || (s = up(c, &c->blk_t, tall)) ||
        (s = up(c, &c->blk_soff, soffv)) || (s = up(c, &c->blk_ip, ipv)) || (s = up(c, &c->blk_incp, incp)) ||
        (s = up(c, &c->blk_inc, inc)))
        return s;
    // Compact records of the near terms for the block kernel: one uint2 per
    // term (brec_pack) holding its atoms as indices local to the owning block
    // (atom - a0 < BLK_LOC_MAX = 512: 9 bits each) and the index of its
    // parameters in the type's table of distinct parameter tuples (bit-exact
    // copies of the per-term values, so results do not change).  8 bytes a
    // term instead of 24-64, so a thread can hold the first record of every
    // type in registers while the block stages its positions.
    const int npar[6] = {2, 2, 4, 6, 4, 1};
    for (int ty = 0; ty < 6; ++ty) {
        const int nn = c->nnear[ty];
        if (nn == 0) continue;
        std::vector<uint2> rec(nn);
        std::vector<double> tab;
        std::map<std::array<unsigned long long, 6>, unsigned> seen;
        for (int b = 0; b < c->nblk; ++b) {
            const int k0 = tst[ty][b], k1 = b + 1 < c->nblk ? tst[ty][b + 1] : ptr[ty];
            for (int k = k0; k < k1; ++k) {
                int at[4] = {0, 0, 0, 0};
                atoms_of(ty, k, at);
                unsigned l[4] = {0, 0, 0, 0};
                for (int q = 0; q < K[ty]; ++q) {
                    const int d = at[q] - a0v[b];
                    if (d < 0 || d >= BLK_LOC_MAX) return pgk_fail(c, PGK_E_INVALID, "bonded term outside its block");
                    l[q] = (unsigned)d;
                }
                double pv[6] = {0, 0, 0, 0, 0, 0};
                switch (ty) {
                    case 0: pv[0] = t.bp[k].x; pv[1] = t.bp[k].y; break;
                    case 1: pv[0] = t.ap[k].x; pv[1] = t.ap[k].y; break;
                    case 2: pv[0] = t.tp[k].x; pv[1] = t.tp[k].y; pv[2] = t.tp[k].z; pv[3] = t.tp[k].w; break;
                    case 3: for (int q = 0; q < 6; ++q) pv[q] = t.rc[6 * (size_t)k + q]; break;
                    case 4: pv[0] = k14[k].x; pv[1] = k14[k].y; pv[2] = k14[k].z; pv[3] = k14[k].w; break;
                    default: pv[0] = qex[k]; break;
                }
                std::array<unsigned long long, 6> key{};
                std::memcpy(key.data(), pv, sizeof(pv));
                auto it = seen.find(key);
                unsigned idx;
                if (it == seen.end()) {
                    idx = (unsigned)seen.size();
                    if (idx >= (1u << 28)) return pgk_fail(c, PGK_E_UNSUPPORTED, "too many distinct bonded parameters");
                    seen.emplace(key, idx);
                    tab.insert(tab.end(), pv, pv + npar[ty]);
                } else {
                    idx = it->second;
                }
                rec[k] = make_uint2(l[0] | (l[1] << 9) | (l[2] << 18) | ((l[3] & 31u) << 27), (l[3] >> 5) | (idx << 4));
            }
        }
        if ((s = up(c, &c->brec[ty], rec)) || (s = up(c, &c->btab[ty], tab))) return s;
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
// torsion, 3 RB torsion, 4 1-4 pairs, 5 excluded-pair Ewald correction): the
// block kernel for the near terms, the per-type kernels for the far ones.
template <bool MIXED>
static void terms_impl(pgk_ctx* c, int group, int mask, bool want, bool tens) {
    long long* acc = c->acc + (size_t)group * NACC;
    void* facc = c->facc[group];
    const int w = want ? 1 : 0;
    if (c->nblk > 0) {
        TermsDev D{c->spl64, c->spl32, c->nspl, c->hspl, {}, {}};
        for (int ty = 0; ty < 6; ++ty) { D.rec[ty] = c->brec[ty]; D.tab[ty] = c->btab[ty]; }
        const int cap = blk_slot_cap(MIXED);
        BlkDev K{c->blk_a0, c->blk_nloc, c->blk_t, c->blk_soff, c->blk_ip, c->blk_incp, c->blk_inc, c->nblk, cap};
        const size_t sm = 3 * BLK_LOC_MAX * sizeof(double) + 3 * (size_t)cap * (MIXED ? sizeof(float) : sizeof(double)) +
                          (BLK_LOC_MAX + 4) * sizeof(int) + (size_t)cap * sizeof(unsigned short);
        if (tens) {
            smem_limit(k_intra_blk<MIXED, true>, sm);
            k_intra_blk<MIXED, true><<<c->nblk, BLK_THREADS, sm, c->st>>>(c->pos, D, K, c->dyn, facc, acc, mask, w,
                                                                          c->status);
        } else {
            smem_limit(k_intra_blk<MIXED, false>, sm);
            k_intra_blk<MIXED, false><<<c->nblk, BLK_THREADS, sm, c->st>>>(c->pos, D, K, c->dyn, facc, acc, mask, w,
                                                                           c->status);
        }
        PGK_LAUNCHED(c);
    }
    const int tb = 128;
    auto nb = [&](int m) { return (m + tb - 1) / tb; };
    int f = c->nnear[0], m = c->nbond - f;
    if ((mask & 1) && m > 0) {
        k_bond<MIXED><<<nb(m), tb, 0, c->st>>>(c->pos, c->bond_ij + f, c->bond_p + f, m, c->dyn, facc, acc, w);
        PGK_LAUNCHED(c);
    }
    f = c->nnear[1]; m = c->nangl - f;
    if ((mask & 2) && m > 0) {
        k_angl<MIXED><<<nb(m), tb, 0, c->st>>>(c->pos, c->angl_ijk + f, c->angl_p + f, m, c->dyn, facc, acc, w);
        PGK_LAUNCHED(c);
    }
    f = c->nnear[2]; m = c->ntors - f;
    if ((mask & 4) && m > 0) {
        k_tors<MIXED, false><<<nb(m), tb, 0, c->st>>>(c->pos, c->tors_ijkl + f, c->tors_p + f, nullptr, m, c->dyn,
                                                      facc, acc, w, c->status);
        PGK_LAUNCHED(c);
    }
    f = c->nnear[3]; m = c->ntorsrb - f;
    if ((mask & 8) && m > 0) {
        k_tors<MIXED, true><<<nb(m), tb, 0, c->st>>>(c->pos, c->rb_ijkl + f, nullptr, c->rb_c + 6 * (size_t)f, m,
                                                     c->dyn, facc, acc, w, c->status);
        PGK_LAUNCHED(c);
    }
    f = c->nnear[4]; m = c->n14 - f;
    if ((mask & 16) && m > 0) {
        k_non14<MIXED><<<nb(m), tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij + f, c->p14_f + f, m, c->ntyp,
                                                c->lj64, c->dyn, facc, acc, w);
        PGK_LAUNCHED(c);
    }
    f = c->nnear[5]; m = c->nexpair - f;
    if ((mask & 32) && m > 0) {
        k_excl<MIXED><<<nb(m), tb, 0, c->st>>>(c->pos, c->chrg, c->expair + f, m, c->spl64, c->spl32, c->nspl,
                                               c->hspl, c->dyn, facc, acc, w);
        PGK_LAUNCHED(c);
    }
}

pgk_status launch_intra(pgk_ctx* c, int group, int mask, bool want, bool tens) {
    const long long cnt[6] = {c->nbond, c->nangl, c->ntors, c->ntorsrb, c->n14, c->nexpair};
    int active = 0;
    for (int ty = 0; ty < 6; ++ty) if (((mask >> ty) & 1) && cnt[ty] > 0) active |= 1 << ty;
    if (!active) return PGK_OK;
    if (c->mixed()) terms_impl<true>(c, group, active, want, tens && want);
    else terms_impl<false>(c, group, active, want, tens && want);
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
