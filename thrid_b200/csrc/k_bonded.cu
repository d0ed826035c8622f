// k_bonded.cu -- intramolecular terms:
//   calbondp   calbond.F90:109-219      U = k (r - r0)^2
//   calanglp   calangl.F90:172-358      U = k (theta - theta0)^2
//   caltorsp   caltors.F90 (+calijkl)   U = V/div (1 + cos(n phi - phase))
//   caltorsrbp caltorsrb.F90:118-459    U = sum_n C_n (-1)^n cos^n phi
//   calnon14p  calnon14.F90:249-521     scaled 1-4 Coulomb + LJ
//   ewaldrp excluded-pair erf correction (ewaldr.F90:756-826)
//
// Hot path: k_intra, one CTA per chunk of whole molecules (atoms contiguous):
// the chunk's positions are staged in shared memory, every term writes the
// force on each of its atoms into its own shared-memory slot, and each atom
// then sums its slots in a fixed order -- no atomics inside the chunk,
// deterministic in both precisions -- before one global add per atom
// component.  The per-term-type kernels (k_bond, k_angl, k_tors, k_non14,
// k_excl) serve systems whose molecules are not contiguous or too large.
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
                       int nterm, const DynState* __restrict__ dyn, void* facc, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < nterm) {
        double F[3], rd[3], e;
        int i = ij[k].x, j = ij[k].y;
        if (eval_bond<T>(pos, i, j, par[k], dyn, F, rd, e)) {
            force_add<MIXED>(facc, i, F[0], F[1], F[2]);
            force_add<MIXED>(facc, j, -F[0], -F[1], -F[2]);
            if (want) { v[0] = e; vir_pair(v + 1, F, rd); }
        }
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
        double F[3][3], e;
        int at[3] = {ijk[n].x, ijk[n].y, ijk[n].z};
        if (eval_angl<T>(pos, at[0], at[1], at[2], par[n], dyn, F, e)) {
#pragma unroll
            for (int q = 0; q < 3; ++q) force_add<MIXED>(facc, at[q], F[q][0], F[q][1], F[q][2]);
            if (want) {
                v[0] = e;
#pragma unroll
                for (int q = 0; q < 3; ++q) vir_abs(v + 1, F[q], pos, at[q]);
            }
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
        for (int q = 0; q < 4; ++q) force_add<MIXED>(facc, at[q], F[q][0], F[q][1], F[q][2]);
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
        force_add<MIXED>(facc, i, F[0], F[1], F[2]);
        force_add<MIXED>(facc, j, -F[0], -F[1], -F[2]);
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
        force_add<MIXED>(facc, i, F[0], F[1], F[2]);
        force_add<MIXED>(facc, j, -F[0], -F[1], -F[2]);
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

// ---- fused intramolecular kernel ----------------------------------------------
// Gather formulation, no atomics inside the chunk: every term writes the force
// on each of its atoms into its own slot (slots of a term type are laid out
// term by term, k slots per k-atom term); then each atom sums its slots in a
// fixed order (precomputed incidence list), so the result is deterministic in
// both precisions.  Chunks are whole molecules with at most INTRA_ATOMS atoms
// and INTRA_SLOTS slots.
#define INTRA_ATOMS 64
#define INTRA_SLOTS 2048

struct IntraArgs {
    const int* chunk_atom;          // [nchunk+1] first atom of each chunk
    const int* chunk_term;          // [6][nchunk+1] term ranges per type
    const int* chunk_slot;          // [6][nchunk] slot base of each type inside its chunk
    const int* inc_start;           // [natom+1] incidence CSR (chunk-local slot ids)
    const unsigned short* inc_slot;
    int nchunk;
    int mask;                       // bit t: evaluate term type t (0 bond,1 angl,2 tors,3 torsrb,4 1-4,5 excl)
    int want;
    const int2* bond_ij; const double2* bond_p;
    const int4* angl_ijk; const double2* angl_p;
    const int4* tors_ijkl; const double4* tors_p;
    const int4* rb_ijkl; const double* rb_c;
    const int2* p14_ij; const double2* p14_f;
    const int2* expair;
    const double* chrg; const int* typ; int ntyp; const double2* lj64;
    const double4* spl64; const float4* spl32; int nspl; double h;
    void* facc; long long* acc; unsigned* status;
};

template <typename T>
__device__ __forceinline__ void put(T* sx, T* sy, T* sz, int slot, const double* F, double sign) {
    sx[slot] = (T)(sign * F[0]);
    sy[slot] = (T)(sign * F[1]);
    sz[slot] = (T)(sign * F[2]);
}

template <bool MIXED>
__global__ void __launch_bounds__(256) k_intra(const double* __restrict__ pos, IntraArgs a,
                                               const DynState* __restrict__ dyn) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    __shared__ double sp[3 * INTRA_ATOMS];
    __shared__ unsigned short s_inc[INTRA_SLOTS];     // the chunk's incidence lists
    __shared__ int s_start[INTRA_ATOMS + 1];
    __shared__ double s_q[INTRA_ATOMS];                // charges and LJ types of the chunk
    __shared__ int s_t[INTRA_ATOMS];
    extern __shared__ unsigned char slot_raw[];
    T* sx = (T*)slot_raw;
    T* sy = sx + INTRA_SLOTS;
    T* sz = sy + INTRA_SLOTS;
    const int c = blockIdx.x;
    const int a0 = a.chunk_atom[c], na = a.chunk_atom[c + 1] - a0;
    const int i0 = a.inc_start[a0], ni = a.inc_start[a0 + na] - i0;
    for (int k = threadIdx.x; k < 3 * na; k += blockDim.x) sp[k] = pos[3 * (size_t)a0 + k];
    for (int k = threadIdx.x; k <= na; k += blockDim.x) s_start[k] = a.inc_start[a0 + k] - i0;
    for (int k = threadIdx.x; k < ni; k += blockDim.x) s_inc[k] = a.inc_slot[i0 + k];
    for (int k = threadIdx.x; k < na; k += blockDim.x) { s_q[k] = a.chrg[a0 + k]; s_t[k] = a.typ[a0 + k]; }
    __syncthreads();
    const int stride = a.nchunk + 1;
    const int* cs = a.chunk_slot;
    if (a.mask & 1) {   // bonds (2 slots)
        double v[11] = {0};
        const int t0 = a.chunk_term[c];
        for (int t = t0 + threadIdx.x; t < a.chunk_term[c + 1]; t += blockDim.x) {
            int i = a.bond_ij[t].x - a0, j = a.bond_ij[t].y - a0;
            double F[3] = {0, 0, 0}, rd[3], e;
            bool on = eval_bond<T>(sp, i, j, a.bond_p[t], dyn, F, rd, e);
            int sl = cs[c] + 2 * (t - t0);
            put(sx, sy, sz, sl, F, 1.0);
            put(sx, sy, sz, sl + 1, F, -1.0);
            if (a.want && on) { v[0] += e; vir_pair(v + 1, F, rd); }
        }
        if (a.want) {
            const int idx[11] = {A_BOND, A_VB, A_VTB + 0, A_VTB + 1, A_VTB + 2, A_VTB + 3, A_VTB + 4, A_VTB + 5,
                                 A_VTB + 6, A_VTB + 7, A_VTB + 8};
            block_acc<11>(v, a.acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (a.mask & 2) {   // angles (3 slots)
        double v[11] = {0};
        const int t0 = a.chunk_term[stride + c];
        for (int t = t0 + threadIdx.x; t < a.chunk_term[stride + c + 1]; t += blockDim.x) {
            const int at[3] = {a.angl_ijk[t].x - a0, a.angl_ijk[t].y - a0, a.angl_ijk[t].z - a0};
            double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e;
            bool on = eval_angl<T>(sp, at[0], at[1], at[2], a.angl_p[t], dyn, F, e);
            int sl = cs[a.nchunk + c] + 3 * (t - t0);
#pragma unroll
            for (int q = 0; q < 3; ++q) put(sx, sy, sz, sl + q, F[q], 1.0);
            if (a.want && on) {
                v[0] += e;
#pragma unroll
                for (int q = 0; q < 3; ++q) vir_abs(v + 1, F[q], sp, at[q]);
            }
        }
        if (a.want) {
            const int idx[11] = {A_ANGL, A_VA, A_VTA + 0, A_VTA + 1, A_VTA + 2, A_VTA + 3, A_VTA + 4, A_VTA + 5,
                                 A_VTA + 6, A_VTA + 7, A_VTA + 8};
            block_acc<11>(v, a.acc, idx, !MIXED);
            __syncthreads();
        }
    }
    for (int rb = 0; rb < 2; ++rb) {   // periodic (type 2) and Ryckaert-Bellemans (type 3) torsions (4 slots)
        if (!(a.mask & (4 << rb))) continue;
        double v[11] = {0};
        const int ty = 2 + rb;
        const int t0 = a.chunk_term[ty * stride + c];
        for (int t = t0 + threadIdx.x; t < a.chunk_term[ty * stride + c + 1]; t += blockDim.x) {
            const int4 q4 = rb ? a.rb_ijkl[t] : a.tors_ijkl[t];
            const int at[4] = {q4.x - a0, q4.y - a0, q4.z - a0, q4.w - a0};
            double F[4][3], e;
            if (rb) eval_tors<T, true>(sp, at[0], at[1], at[2], at[3], make_double4(0, 0, 0, 0),
                                       a.rb_c + 6 * (size_t)t, dyn, F, e, a.status);
            else eval_tors<T, false>(sp, at[0], at[1], at[2], at[3], a.tors_p[t], nullptr, dyn, F, e, a.status);
            int sl = cs[ty * a.nchunk + c] + 4 * (t - t0);
#pragma unroll
            for (int q = 0; q < 4; ++q) put(sx, sy, sz, sl + q, F[q], 1.0);
            if (a.want) {
                v[0] += e;
#pragma unroll
                for (int q = 0; q < 4; ++q) vir_abs(v + 1, F[q], sp, at[q]);
            }
        }
        if (a.want) {
            const int idx[11] = {rb ? A_TORSRB : A_TORS, A_VT, A_VTT + 0, A_VTT + 1, A_VTT + 2, A_VTT + 3,
                                 A_VTT + 4, A_VTT + 5, A_VTT + 6, A_VTT + 7, A_VTT + 8};
            block_acc<11>(v, a.acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (a.mask & 16) {  // 1-4 pairs (2 slots)
        double v[12] = {0};
        const int t0 = a.chunk_term[4 * stride + c];
        for (int t = t0 + threadIdx.x; t < a.chunk_term[4 * stride + c + 1]; t += blockDim.x) {
            int gi = a.p14_ij[t].x, gj = a.p14_ij[t].y;
            double F[3], rd[3], de, dv;
            eval_14<T>(sp, gi - a0, gj - a0, s_q[gi - a0] * s_q[gj - a0], a.lj64[s_t[gi - a0] * a.ntyp + s_t[gj - a0]],
                       a.p14_f[t], dyn, F, rd, de, dv);
            int sl = cs[4 * a.nchunk + c] + 2 * (t - t0);
            put(sx, sy, sz, sl, F, 1.0);
            put(sx, sy, sz, sl + 1, F, -1.0);
            if (a.want) { v[0] += de; v[1] += dv; vir_pair(v + 2, F, rd); }
        }
        if (a.want) {
            const int idx[12] = {A_ELC14, A_VDW14, A_V14, A_VT14 + 0, A_VT14 + 1, A_VT14 + 2, A_VT14 + 3,
                                 A_VT14 + 4, A_VT14 + 5, A_VT14 + 6, A_VT14 + 7, A_VT14 + 8};
            block_acc<12>(v, a.acc, idx, !MIXED);
            __syncthreads();
        }
    }
    if (a.mask & 32) {  // excluded-pair Ewald correction (2 slots)
        double v[11] = {0};
        const int t0 = a.chunk_term[5 * stride + c];
        for (int t = t0 + threadIdx.x; t < a.chunk_term[5 * stride + c + 1]; t += blockDim.x) {
            int gi = a.expair[t].x, gj = a.expair[t].y;
            double F[3], rd[3], e;
            eval_excl<MIXED>(sp, gi - a0, gj - a0, s_q[gi - a0] * s_q[gj - a0], a.spl64, a.spl32, a.nspl, a.h, dyn,
                             F, rd, e);
            int sl = cs[5 * a.nchunk + c] + 2 * (t - t0);
            put(sx, sy, sz, sl, F, 1.0);
            put(sx, sy, sz, sl + 1, F, -1.0);
            if (a.want) { v[0] -= e; vir_pair(v + 1, F, rd); }
        }
        if (a.want) {
            double w[8] = {v[0], v[0], v[2], v[3], v[4], v[6], v[7], v[10]};
            const int idx[8] = {A_ELC, A_VC, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
            block_acc<8>(w, a.acc, idx, !MIXED);
        }
    }
    __syncthreads();
    // each atom sums its slots in the precomputed order (slots of term types
    // that are off for this MTS group are skipped by their type ranges)
    int lo[6], hi[6];
#pragma unroll
    for (int ty = 0; ty < 6; ++ty) {
        const int k = ty == 0 ? 2 : ty == 1 ? 3 : ty <= 3 ? 4 : 2;
        lo[ty] = (a.mask >> ty) & 1 ? cs[ty * a.nchunk + c] : 0;
        hi[ty] = (a.mask >> ty) & 1 ? lo[ty] + k * (a.chunk_term[ty * stride + c + 1] - a.chunk_term[ty * stride + c]) : 0;
    }
    for (int l = threadIdx.x; l < na; l += blockDim.x) {
        double fx = 0, fy = 0, fz = 0;
        for (int k = s_start[l]; k < s_start[l + 1]; ++k) {
            const int sl = s_inc[k];
            bool on = false;
#pragma unroll
            for (int ty = 0; ty < 6; ++ty) on |= (sl >= lo[ty] && sl < hi[ty]);
            if (!on) continue;
            fx += (double)sx[sl]; fy += (double)sy[sl]; fz += (double)sz[sl];
        }
        if (fx != 0.0 || fy != 0.0 || fz != 0.0) force_add<MIXED>(a.facc, a0 + l, fx, fy, fz);
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
    PGK_CUDA(c, cudaMalloc(dst, v.size() * sizeof(T)));
    PGK_CUDA(c, cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PGK_OK;
}

// Chunks of whole molecules (contiguous atom ranges, <= INTRA_ATOMS atoms and
// <= INTRA_SLOTS term-atom slots), terms ordered by chunk, plus the per-atom
// slot incidence lists; falls back to the per-type kernels when a molecule is
// not contiguous, is too large for a chunk, or a term spans two molecules.
pgk_status bonded_setup(pgk_ctx* c, HostTerms& t, const std::vector<int>& mol_idx, const std::vector<int>& mol_list) {
    int n = c->natom;
    bool ok = !mol_idx.empty();
    const int K[6] = {2, 3, 4, 4, 2, 2};
    // slots contributed by each molecule (terms are assigned to the molecule of their first atom)
    std::vector<int> mol_of(n, -1);
    int nmol = ok ? (int)mol_idx.size() - 1 : 0;
    for (int m = 0; m < nmol && ok; ++m) {
        int b = mol_idx[m], e = mol_idx[m + 1];
        for (int q = b; q < e; ++q) {
            if (mol_list[q] != mol_list[b] + (q - b)) ok = false;
            else mol_of[mol_list[q]] = m;
        }
        if (m > 0 && mol_list[b] != mol_list[mol_idx[m - 1]] + (mol_idx[m] - mol_idx[m - 1])) ok = false;
        if (e - b > INTRA_ATOMS) ok = false;
    }
    if (ok && (nmol == 0 || mol_list[mol_idx[0]] != 0 || mol_idx[nmol] != n)) ok = false;
    std::vector<long long> mslots(nmol, 0);
    auto add_slots = [&](int first, int k) { if (ok) { int m = mol_of[first]; if (m < 0) ok = false; else mslots[m] += k; } };
    for (auto& x : t.bij) add_slots(x.x, 2);
    for (auto& x : t.aijk) add_slots(x.x, 3);
    for (auto& x : t.tij) add_slots(x.x, 4);
    for (auto& x : t.rij) add_slots(x.x, 4);
    for (auto& x : t.p14) add_slots(x.x, 2);
    for (auto& x : t.ex) add_slots(x.x, 2);
    std::vector<int> atom_chunk(n, -1), chunk_atom(1, 0);
    if (ok) {
        int natoms = 0; long long nslots = 0;
        for (int m = 0; m < nmol && ok; ++m) {
            int na = mol_idx[m + 1] - mol_idx[m];
            if (mslots[m] > INTRA_SLOTS) { ok = false; break; }
            if (natoms + na > INTRA_ATOMS || nslots + mslots[m] > INTRA_SLOTS) {
                chunk_atom.push_back(chunk_atom.back() + natoms);
                natoms = 0; nslots = 0;
            }
            natoms += na; nslots += mslots[m];
        }
        if (ok) {
            chunk_atom.push_back(n);
            int nch = (int)chunk_atom.size() - 1;
            for (int k = 0; k < nch; ++k)
                for (int a2 = chunk_atom[k]; a2 < chunk_atom[k + 1]; ++a2) atom_chunk[a2] = k;
        }
    }
    int nch = ok ? (int)chunk_atom.size() - 1 : 0;
    std::vector<int> ranges;
    auto sort_type = [&](int count, auto atoms_of, auto apply) {
        std::vector<int> order(count), ch(count);
        for (int k = 0; k < count && ok; ++k) {
            int cc = -1;
            for (int at : atoms_of(k)) {
                int x = atom_chunk[at];
                if (cc < 0) cc = x;
                else if (x != cc) ok = false;
            }
            ch[k] = cc;
        }
        if (!ok) return;
        for (int k = 0; k < count; ++k) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ch[x] < ch[y]; });
        apply(order);
        std::vector<int> r(nch + 1, 0);
        for (int k = 0; k < count; ++k) r[ch[k] + 1]++;
        for (int k = 0; k < nch; ++k) r[k + 1] += r[k];
        ranges.insert(ranges.end(), r.begin(), r.end());
    };
    if (ok) {
        sort_type((int)t.bij.size(), [&](int k) { return std::vector<int>{t.bij[k].x, t.bij[k].y}; },
                  [&](const std::vector<int>& o) { reorder(t.bij, o); reorder(t.bp, o); });
        sort_type((int)t.aijk.size(), [&](int k) { return std::vector<int>{t.aijk[k].x, t.aijk[k].y, t.aijk[k].z}; },
                  [&](const std::vector<int>& o) { reorder(t.aijk, o); reorder(t.ap, o); });
        sort_type((int)t.tij.size(),
                  [&](int k) { return std::vector<int>{t.tij[k].x, t.tij[k].y, t.tij[k].z, t.tij[k].w}; },
                  [&](const std::vector<int>& o) { reorder(t.tij, o); reorder(t.tp, o); });
        sort_type((int)t.rij.size(),
                  [&](int k) { return std::vector<int>{t.rij[k].x, t.rij[k].y, t.rij[k].z, t.rij[k].w}; },
                  [&](const std::vector<int>& o) {
                      std::vector<double> rc2(t.rc.size());
                      for (size_t k = 0; k < o.size(); ++k)
                          for (int q = 0; q < 6; ++q) rc2[6 * k + q] = t.rc[6 * o[k] + q];
                      reorder(t.rij, o);
                      t.rc.swap(rc2);
                  });
        sort_type((int)t.p14.size(), [&](int k) { return std::vector<int>{t.p14[k].x, t.p14[k].y}; },
                  [&](const std::vector<int>& o) { reorder(t.p14, o); reorder(t.f14, o); });
        sort_type((int)t.ex.size(), [&](int k) { return std::vector<int>{t.ex[k].x, t.ex[k].y}; },
                  [&](const std::vector<int>& o) { reorder(t.ex, o); });
    }
    pgk_status s;
    c->nbond = (int)t.bij.size(); c->nangl = (int)t.aijk.size(); c->ntors = (int)t.tij.size();
    c->ntorsrb = (int)t.rij.size(); c->n14 = (int)t.p14.size(); c->nexpair = (int)t.ex.size();
    if ((s = up(c, &c->bond_ij, t.bij)) || (s = up(c, &c->bond_p, t.bp)) || (s = up(c, &c->angl_ijk, t.aijk)) ||
        (s = up(c, &c->angl_p, t.ap)) || (s = up(c, &c->tors_ijkl, t.tij)) || (s = up(c, &c->tors_p, t.tp)) ||
        (s = up(c, &c->rb_ijkl, t.rij)) || (s = up(c, &c->rb_c, t.rc)) || (s = up(c, &c->p14_ij, t.p14)) ||
        (s = up(c, &c->p14_f, t.f14)) || (s = up(c, &c->expair, t.ex)))
        return s;
    c->intra_ok = ok && nch > 0;
    if (!c->intra_ok) return PGK_OK;
    c->nchunk = nch;
    // slot bases per type per chunk, and the incidence lists
    std::vector<int> slot_base(6 * (size_t)nch, 0);
    std::vector<std::vector<unsigned short>> inc(n);
    auto atom_list = [&](int ty, int k) -> std::vector<int> {
        switch (ty) {
            case 0: return {t.bij[k].x, t.bij[k].y};
            case 1: return {t.aijk[k].x, t.aijk[k].y, t.aijk[k].z};
            case 2: return {t.tij[k].x, t.tij[k].y, t.tij[k].z, t.tij[k].w};
            case 3: return {t.rij[k].x, t.rij[k].y, t.rij[k].z, t.rij[k].w};
            case 4: return {t.p14[k].x, t.p14[k].y};
            default: return {t.ex[k].x, t.ex[k].y};
        }
    };
    for (int ch = 0; ch < nch; ++ch) {
        int base = 0;
        for (int ty = 0; ty < 6; ++ty) {
            slot_base[(size_t)ty * nch + ch] = base;
            int t0 = ranges[(size_t)ty * (nch + 1) + ch], t1 = ranges[(size_t)ty * (nch + 1) + ch + 1];
            for (int k = t0; k < t1; ++k) {
                std::vector<int> at = atom_list(ty, k);
                for (int q = 0; q < K[ty]; ++q) inc[at[q]].push_back((unsigned short)(base + K[ty] * (k - t0) + q));
            }
            base += K[ty] * (t1 - t0);
        }
        if (base > INTRA_SLOTS) { c->intra_ok = false; return PGK_OK; }
    }
    std::vector<int> inc_start(n + 1, 0);
    std::vector<unsigned short> inc_slot;
    for (int i = 0; i < n; ++i) {
        inc_start[i] = (int)inc_slot.size();
        inc_slot.insert(inc_slot.end(), inc[i].begin(), inc[i].end());
    }
    inc_start[n] = (int)inc_slot.size();
    if (inc_slot.empty()) inc_slot.push_back(0);
    if ((s = up(c, &c->chunk_atom, chunk_atom)) || (s = up(c, &c->chunk_term, ranges)) ||
        (s = up(c, &c->chunk_slot, slot_base)) || (s = up(c, &c->inc_start, inc_start)) ||
        (s = up(c, &c->inc_slot, inc_slot)))
        return s;
    return PGK_OK;
}

template <bool MIXED>
static void bonded_impl(pgk_ctx* c, int group, bool want, bool all) {
    void* f = c->facc[group];
    long long* acc = c->acc + (size_t)group * NACC;
    int w = want ? 1 : 0;
    const int tb = 128;
    auto on = [&](int mts) { return all || mts == (group == 0 ? PGK_MTS_LONG : PGK_MTS_SHORT); };
    if (c->nbond && on(c->prm.mts_bond)) {
        k_bond<MIXED><<<(c->nbond + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->bond_ij, c->bond_p, c->nbond, c->dyn,
                                                                   f, acc, w);
        PGK_LAUNCHED(c);
    }
    if (c->nangl && on(c->prm.mts_angl)) {
        k_angl<MIXED><<<(c->nangl + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->angl_ijk, c->angl_p, c->nangl, c->dyn,
                                                                   f, acc, w);
        PGK_LAUNCHED(c);
    }
    if (c->ntors && on(c->prm.mts_tors)) {
        k_tors<MIXED, false><<<(c->ntors + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->tors_ijkl, c->tors_p, nullptr,
                                                                          c->ntors, c->dyn, f, acc, w, c->status);
        PGK_LAUNCHED(c);
    }
    if (c->ntorsrb && on(c->prm.mts_torsrb)) {
        k_tors<MIXED, true><<<(c->ntorsrb + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->rb_ijkl, nullptr, c->rb_c,
                                                                           c->ntorsrb, c->dyn, f, acc, w, c->status);
        PGK_LAUNCHED(c);
    }
    if (c->n14 && (all || (on(c->prm.mts_vdw14) && c->prm.mts_vdw14 == c->prm.mts_elc14))) {
        k_non14<MIXED><<<(c->n14 + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij, c->p14_f, c->n14,
                                                                  c->ntyp, c->lj64, c->dyn, f, acc, w);
        PGK_LAUNCHED(c);
    }
}

pgk_status launch_bonded(pgk_ctx* c, int group, bool ene, bool vir, bool force_all) {
    if (c->mixed()) bonded_impl<true>(c, group, ene || vir, force_all);
    else bonded_impl<false>(c, group, ene || vir, force_all);
    PGK_CUDA(c, cudaGetLastError());
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

// mask bits: 0 bond, 1 angle, 2 periodic torsion, 3 RB torsion, 4 1-4, 5 excluded pairs
pgk_status launch_intra(pgk_ctx* c, int group, int mask, bool want) {
    if (!mask) return PGK_OK;
    if (!c->intra_ok) {   // general path: one kernel per term type
        pgk_status s = PGK_OK;
        if (mask & 31) {
            int g = group;
            void* f = c->facc[g];
            long long* acc = c->acc + (size_t)g * NACC;
            int w = want ? 1 : 0;
            const int tb = 128;
            if ((mask & 1) && c->nbond) {
                if (c->mixed()) k_bond<true><<<(c->nbond + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->bond_ij, c->bond_p, c->nbond, c->dyn, f, acc, w);
                else k_bond<false><<<(c->nbond + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->bond_ij, c->bond_p, c->nbond, c->dyn, f, acc, w);
                PGK_LAUNCHED(c);
            }
            if ((mask & 2) && c->nangl) {
                if (c->mixed()) k_angl<true><<<(c->nangl + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->angl_ijk, c->angl_p, c->nangl, c->dyn, f, acc, w);
                else k_angl<false><<<(c->nangl + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->angl_ijk, c->angl_p, c->nangl, c->dyn, f, acc, w);
                PGK_LAUNCHED(c);
            }
            if ((mask & 4) && c->ntors) {
                if (c->mixed()) k_tors<true, false><<<(c->ntors + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->tors_ijkl, c->tors_p, nullptr, c->ntors, c->dyn, f, acc, w, c->status);
                else k_tors<false, false><<<(c->ntors + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->tors_ijkl, c->tors_p, nullptr, c->ntors, c->dyn, f, acc, w, c->status);
                PGK_LAUNCHED(c);
            }
            if ((mask & 8) && c->ntorsrb) {
                if (c->mixed()) k_tors<true, true><<<(c->ntorsrb + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->rb_ijkl, nullptr, c->rb_c, c->ntorsrb, c->dyn, f, acc, w, c->status);
                else k_tors<false, true><<<(c->ntorsrb + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->rb_ijkl, nullptr, c->rb_c, c->ntorsrb, c->dyn, f, acc, w, c->status);
                PGK_LAUNCHED(c);
            }
            if ((mask & 16) && c->n14) {
                if (c->mixed()) k_non14<true><<<(c->n14 + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij, c->p14_f, c->n14, c->ntyp, c->lj64, c->dyn, f, acc, w);
                else k_non14<false><<<(c->n14 + tb - 1) / tb, tb, 0, c->st>>>(c->pos, c->chrg, c->typ, c->p14_ij, c->p14_f, c->n14, c->ntyp, c->lj64, c->dyn, f, acc, w);
                PGK_LAUNCHED(c);
            }
        }
        if (mask & 32) s = launch_excl(c, group, want, want);
        if (s) return s;
        PGK_CUDA(c, cudaGetLastError());
        return PGK_OK;
    }
    IntraArgs a;
    a.chunk_atom = c->chunk_atom; a.chunk_term = c->chunk_term; a.chunk_slot = c->chunk_slot;
    a.inc_start = c->inc_start; a.inc_slot = c->inc_slot; a.nchunk = c->nchunk;
    a.mask = mask; a.want = want ? 1 : 0;
    a.bond_ij = c->bond_ij; a.bond_p = c->bond_p; a.angl_ijk = c->angl_ijk; a.angl_p = c->angl_p;
    a.tors_ijkl = c->tors_ijkl; a.tors_p = c->tors_p; a.rb_ijkl = c->rb_ijkl; a.rb_c = c->rb_c;
    a.p14_ij = c->p14_ij; a.p14_f = c->p14_f; a.expair = c->expair;
    a.chrg = c->chrg; a.typ = c->typ; a.ntyp = c->ntyp; a.lj64 = c->lj64;
    a.spl64 = c->spl64; a.spl32 = c->spl32; a.nspl = c->nspl; a.h = c->hspl;
    a.facc = c->facc[group]; a.acc = c->acc + (size_t)group * NACC; a.status = c->status;
    if (c->mixed()) {
        size_t sm = (size_t)3 * INTRA_SLOTS * sizeof(float);
        smem_limit(k_intra<true>, sm);
        k_intra<true><<<c->nchunk, 128, sm, c->st>>>(c->pos, a, c->dyn);
    } else {
        size_t sm = (size_t)3 * INTRA_SLOTS * sizeof(double);
        smem_limit(k_intra<false>, sm);
        k_intra<false><<<c->nchunk, 128, sm, c->st>>>(c->pos, a, c->dyn);
    }
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}
