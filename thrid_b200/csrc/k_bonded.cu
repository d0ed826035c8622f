// k_bonded.cu -- bonded terms, one thread per term, forces added with atomics
// (int64 fixed point in mixed precision, double in FP64):
//   calbondp   calbond.F90:109-219      U = k (r - r0)^2
//   calanglp   calangl.F90:172-358      U = k (theta - theta0)^2
//   caltorsp   caltors.F90 (+calijkl)   U = V/div (1 + cos(n phi - phase))
//   caltorsrbp caltorsrb.F90:118-459    U = sum_n C_n (-1)^n cos^n phi
//   calnon14p  calnon14.F90:249-521     scaled 1-4 Coulomb + LJ
// Displacements are formed in FP64 from the master positions (Fortran anint
// minimum image); the remaining arithmetic runs in T (float for mixed).
// Angle and torsion virials use absolute coordinates exactly like the
// reference (sum f_a x_b over the term's atoms).
#include "pgk_ctx.cuh"

template <typename T>
__device__ __forceinline__ void disp(const double* __restrict__ pos, int a, int b, const DynState* __restrict__ dyn,
                                     T* r) {   // r = x_a - x_b, min image
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = pos[3 * a + d] - pos[3 * b + d];
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
__device__ __forceinline__ void vir_abs(double* v, const double* f, const double* __restrict__ pos, int at) {
    const double x0 = pos[3 * at], x1 = pos[3 * at + 1], x2 = pos[3 * at + 2];
    v[0] += f[0] * x0 + f[1] * x1 + f[2] * x2;
    const double x[3] = {x0, x1, x2};
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) v[1 + a + 3 * b] += f[a] * x[b];
}

template <bool MIXED>
__global__ void k_bond(const double* __restrict__ pos, const int2* __restrict__ ij, const double2* __restrict__ par,
                       int nterm, const DynState* __restrict__ dyn, void* facc, long long* acc, int want) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (k < nterm) {
        double2 p = par[k];   // (k, r0)
        if (fabs(p.x) >= 1.0e-16) {
            int i = ij[k].x, j = ij[k].y;
            T r[3];
            disp<T>(pos, i, j, dyn, r);
            T rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            T dr = rr - (T)p.y;
            T fa = T(-2) * (T)p.x * dr;
            double f[3] = {(double)(fa * r[0] / rr), (double)(fa * r[1] / rr), (double)(fa * r[2] / rr)};
            force_add<MIXED>(facc, i, f[0], f[1], f[2]);
            force_add<MIXED>(facc, j, -f[0], -f[1], -f[2]);
            if (want) {
                v[0] = (double)((T)p.x * dr * dr);
                double rd[3] = {(double)r[0], (double)r[1], (double)r[2]};
                vir_pair(v + 1, f, rd);
            }
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
        double2 p = par[n];   // (k, theta0)
        if (fabs(p.x) >= 1.0e-32) {
            int i = ijk[n].x, j = ijk[n].y, k = ijk[n].z;
            T rij[3], rkj[3];
            disp<T>(pos, j, i, dyn, rij);
            disp<T>(pos, j, k, dyn, rkj);
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
            double Fi[3] = {(double)fi[0], (double)fi[1], (double)fi[2]};
            double Fk[3] = {(double)fk[0], (double)fk[1], (double)fk[2]};
            double Fj[3] = {(double)(-fi[0] - fk[0]), (double)(-fi[1] - fk[1]), (double)(-fi[2] - fk[2])};
            force_add<MIXED>(facc, i, Fi[0], Fi[1], Fi[2]);
            force_add<MIXED>(facc, j, Fj[0], Fj[1], Fj[2]);
            force_add<MIXED>(facc, k, Fk[0], Fk[1], Fk[2]);
            if (want) {
                v[0] = (double)((T)p.x * dth * dth);
                vir_abs(v + 1, Fi, pos, i);
                vir_abs(v + 1, Fj, pos, j);
                vir_abs(v + 1, Fk, pos, k);
            }
        }
    }
    if (want) {
        const int idx[11] = {A_ANGL, A_VA, A_VTA + 0, A_VTA + 1, A_VTA + 2, A_VTA + 3, A_VTA + 4, A_VTA + 5,
                             A_VTA + 6, A_VTA + 7, A_VTA + 8};
        block_acc<11>(v, acc, idx, !MIXED);
    }
}

// shared torsion geometry/forces (calijkl / calijklrb)
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

template <bool MIXED, bool RB>
__global__ void k_tors(const double* __restrict__ pos, const int4* __restrict__ ijkl, const double4* __restrict__ par,
                       const double* __restrict__ rbc, int nterm, const DynState* __restrict__ dyn, void* facc,
                       long long* acc, int want, unsigned* status) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    double v[11] = {0};
    if (n < nterm) {
        int i = ijkl[n].x, j = ijkl[n].y, k = ijkl[n].z, l = ijkl[n].w;
        T rij[3], rkj[3], rkl[3], rik[3], rjl[3];
        disp<T>(pos, j, i, dyn, rij); disp<T>(pos, j, k, dyn, rkj); disp<T>(pos, l, k, dyn, rkl);
        disp<T>(pos, k, i, dyn, rik); disp<T>(pos, l, j, dyn, rjl);
        TG<T> g;
        tors_geo(rij, rkj, rkl, g);
        T fa, pot;
        if (RB) {
            const double* C = rbc + 6 * (size_t)n;
            T bt[6] = {(T)C[0], -(T)C[1], (T)C[2], -(T)C[3], (T)C[4], -(T)C[5]};
            T dp = bt[5];
            fa = 0;
#pragma unroll
            for (int q = 4; q >= 0; --q) { fa = fa * g.c + dp; dp = dp * g.c + bt[q]; }
            fa = -fa;
            pot = dp;
        } else {
            double4 p = par[n];   // (barhig/divfac, phsang, period, cos(phsang))
            T per = (T)p.z;
            pot = (T)p.x * (T(1) + cos(per * g.phi - (T)p.y));
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
        double F[4][3];
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
        const int at[4] = {i, j, k, l};
#pragma unroll
        for (int q = 0; q < 4; ++q) force_add<MIXED>(facc, at[q], F[q][0], F[q][1], F[q][2]);
        if (want) {
            v[0] = (double)pot;
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
        T r[3];
        disp<T>(pos, i, j, dyn, r);
        T r2 = dt3(r, r);
        T ri2 = T(1) / r2, ri1 = sqrt(ri2);
        double2 fc = fac[n];   // (elc factor, vdw factor)
        T de = (T)(chrg[i] * chrg[j]) * ri1;
        de = de * (T)fc.x;
        double2 lp = lj64[typ[i] * ntyp + typ[j]];   // (R^2, E)
        T t2 = ri2 * (T)lp.x, t6 = t2 * t2 * t2, t12 = t6 * t6;
        T E = (T)lp.y * (T)fc.y;
        T dv = E * (t12 - T(2) * t6);
        T ft = T(12) * E * (t12 - t6) * ri2;
        T fs = de * ri2 + ft;
        double f[3] = {(double)(fs * r[0]), (double)(fs * r[1]), (double)(fs * r[2])};
        force_add<MIXED>(facc, i, f[0], f[1], f[2]);
        force_add<MIXED>(facc, j, -f[0], -f[1], -f[2]);
        if (want) {
            v[0] = (double)de;
            v[1] = (double)dv;
            double rd[3] = {(double)r[0], (double)r[1], (double)r[2]};
            vir_pair(v + 2, f, rd);
        }
    }
    if (want) {
        const int idx[12] = {A_ELC14, A_VDW14, A_V14, A_VT14 + 0, A_VT14 + 1, A_VT14 + 2, A_VT14 + 3, A_VT14 + 4,
                             A_VT14 + 5, A_VT14 + 6, A_VT14 + 7, A_VT14 + 8};
        block_acc<12>(v, acc, idx, !MIXED);
    }
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
