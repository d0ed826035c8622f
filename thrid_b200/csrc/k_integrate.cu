// k_integrate.cu -- FP64 integrator pieces of moldyn.F90 / moldyn_nhc.F90 /
// moldyn_mtk.F90, RATTLE (rattle.F90, rattle_mtk.F90), the NHC / MTK chain
// updates (nhcint.F90, nhcpisoint.F90, nhcpanisoint.F90), calvol/calbox and
// the atomic pressure of calpress.F90.  Everything here is FP64 in both
// precision modes (positions, velocities, constraints, chain variables).
//
// Per-atom kernels are HBM-bound (one read + one write of x/v, one read of the
// force accumulator); the chain and box kernels run on one thread and read
// the kinetic-energy / virial sums from the fixed-point accumulators, so a
// whole MD step needs no host round trip and can be captured in a CUDA graph.
#include <cmath>

#include "pgk_ctx.cuh"

// Kicks and drift of one short step in one pass over the atoms (moldyn*.F90
// array statements): long kick v = v*kl_s + (F_long/m)*kl_b, short kick
// v = v + ks_b*(F_short/m), drift x = x*dr_a + v*dr_b, in the order the KD_*
// flags give (coefficients from the chain kernels in DynState).
template <bool MIXED>
__global__ void k_kick_drift(double* __restrict__ vel, double* __restrict__ pos, double* __restrict__ old,
                             const void* __restrict__ fl, const void* __restrict__ fs,
                             const double* __restrict__ mass, int n, const DynState* __restrict__ dyn, int flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    const int d = k % 3;
    double v = vel[k];
    if ((flags & KD_SHORT) && (flags & KD_SHORT_FIRST)) v = v + dyn->ks_b * (force_get<MIXED>(fs, k) / mass[k / 3]);
    if (flags & KD_LONG) v = v * dyn->kl_s[d] + (force_get<MIXED>(fl, k) / mass[k / 3]) * dyn->kl_b[d];
    if ((flags & KD_SHORT) && !(flags & KD_SHORT_FIRST)) v = v + dyn->ks_b * (force_get<MIXED>(fs, k) / mass[k / 3]);
    vel[k] = v;
    if (flags & KD_DRIFT) {
        const double x = pos[k];
        if (flags & KD_SAVE) old[k] = x;
        pos[k] = x * dyn->dr_a[d] + v * dyn->dr_b[d];
    }
}

// rattle_c / rattle_cmtk: one thread per constraint group, Gauss-Seidel sweeps
// in the reference order, at most 300 sweeps (bounded; failure -> status bit).
// The group's atoms (a contiguous span of at most RATTLE_LOCAL atoms) are
// staged in thread-local arrays, so the sweeps run from L1 instead of
// re-reading global memory; longer spans use the global arrays directly.
#define RATTLE_LOCAL 16

struct RattleAcc {   // atom storage of one group: local copy or the global arrays
    double* x; double* v; const double* o; const double* im; int stride_lo;
};

__device__ __forceinline__ bool rattle_pos_sweeps(double* X, double* V, const double* O, const double* IM,
                                                  int lo, const int* __restrict__ glist, const int2* __restrict__ cij,
                                                  const double* __restrict__ cd, int i1, int i2, double eps,
                                                  double dt, const double* rvi) {
    bool finished = false;
    for (int it = 0; it < 300 && !finished; ++it) {
        finished = true;
        for (int ii = i1; ii < i2; ++ii) {
            int nc = glist[ii];
            int ib = cij[nc].x - lo, jb = cij[nc].y - lo;
            double dij = cd[nc];
            double R0 = X[3 * ib] - X[3 * jb], R1 = X[3 * ib + 1] - X[3 * jb + 1], R2 = X[3 * ib + 2] - X[3 * jb + 2];
            double Rsq = R0 * R0 + R1 * R1 + R2 * R2;
            double d2 = dij * dij;
            double delta = fabs(Rsq - d2) / d2;
            if (delta < eps) continue;
            finished = false;
            double O0 = O[3 * ib] - O[3 * jb], O1 = O[3 * ib + 1] - O[3 * jb + 1], O2 = O[3 * ib + 2] - O[3 * jb + 2];
            double RR = R0 * O0 + R1 * O1 + R2 * O2;
            double mi = IM[ib], mj = IM[jb];
            double gij = (Rsq - d2) / (2.0 * RR * (mi + mj) * dt);
            double G[3] = {gij * O0, gij * O1, gij * O2};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                X[3 * ib + d] = X[3 * ib + d] - mi * G[d] * dt;
                X[3 * jb + d] = X[3 * jb + d] + mj * G[d] * dt;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double Gv = G[d] * rvi[d];
                V[3 * ib + d] = V[3 * ib + d] - mi * Gv;
                V[3 * jb + d] = V[3 * jb + d] + mj * Gv;
            }
        }
    }
    return finished;
}

__global__ void k_rattle_pos(double* __restrict__ pos, double* __restrict__ vel, const double* __restrict__ old,
                             const double* __restrict__ invm, const int* __restrict__ gidx,
                             const int* __restrict__ glist, const int2* __restrict__ cij, const double* __restrict__ cd,
                             const int2* __restrict__ span, int ngroup, double eps, double dt, int use_rv,
                             const DynState* __restrict__ dyn, unsigned* status,
                             const unsigned char* __restrict__ fit) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroup || (fit && fit[g >> 5])) return;      // staged groups run in k_rattle_warp
    int i1 = gidx[g], i2 = gidx[g + 1];
    double rvi[3] = {1.0, 1.0, 1.0};
    if (use_rv) { rvi[0] = dyn->rvinv[0]; rvi[1] = dyn->rvinv[1]; rvi[2] = dyn->rvinv[2]; }
    const int lo = span[g].x, na = span[g].y;
    bool finished;
    if (na <= RATTLE_LOCAL) {
        double X[3 * RATTLE_LOCAL], V[3 * RATTLE_LOCAL], O[3 * RATTLE_LOCAL], IM[RATTLE_LOCAL];
        for (int k = 0; k < 3 * na; ++k) { X[k] = pos[3 * lo + k]; V[k] = vel[3 * lo + k]; O[k] = old[3 * lo + k]; }
        for (int k = 0; k < na; ++k) IM[k] = invm[lo + k];
        finished = rattle_pos_sweeps(X, V, O, IM, lo, glist, cij, cd, i1, i2, eps, dt, rvi);
        // write back only this group's own atoms: the spans of groups split
        // from one molecule interleave, and other threads own the rest
        for (int ii = i1; ii < i2; ++ii) {
            const int2 p2 = cij[glist[ii]];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                pos[3 * p2.x + d] = X[3 * (p2.x - lo) + d]; vel[3 * p2.x + d] = V[3 * (p2.x - lo) + d];
                pos[3 * p2.y + d] = X[3 * (p2.y - lo) + d]; vel[3 * p2.y + d] = V[3 * (p2.y - lo) + d];
            }
        }
    } else {
        finished = rattle_pos_sweeps(pos, vel, old, invm, 0, glist, cij, cd, i1, i2, eps, dt, rvi);
    }
    if (!finished) atomicOr(status, ST_RATTLE_NOCONV);
}

__device__ __forceinline__ bool rattle_vel_sweeps(const double* X, double* V, const double* IM, int lo,
                                                  const int* __restrict__ glist, const int2* __restrict__ cij,
                                                  const double* __restrict__ cd, int i1, int i2, double eps) {
    double eps2 = eps * eps;
    bool finished = false;
    for (int it = 0; it < 300 && !finished; ++it) {
        finished = true;
        for (int ii = i1; ii < i2; ++ii) {
            int nc = glist[ii];
            int ib = cij[nc].x - lo, jb = cij[nc].y - lo;
            double dij = cd[nc];
            double R[3], W[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                R[d] = X[3 * ib + d] - X[3 * jb + d];
                W[d] = V[3 * ib + d] - V[3 * jb + d];
            }
            double RV = R[0] * W[0] + R[1] * W[1] + R[2] * W[2];
            double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
            double V2 = W[0] * W[0] + W[1] * W[1] + W[2] * W[2];
            double phi = RV * RV / R2 * V2;   // precedence as in the reference
            if (phi < eps2) continue;
            finished = false;
            double mi = IM[ib], mj = IM[jb];
            double kij = RV / (dij * dij * (mi + mj));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double KR = kij * R[d];
                V[3 * ib + d] = V[3 * ib + d] - mi * KR;
                V[3 * jb + d] = V[3 * jb + d] + mj * KR;
            }
        }
    }
    return finished;
}

// rattlep_v (rattle_mtk.F90:278-542)
__global__ void k_rattle_vel(const double* __restrict__ pos, double* __restrict__ vel, const double* __restrict__ invm,
                             const int* __restrict__ gidx, const int* __restrict__ glist, const int2* __restrict__ cij,
                             const double* __restrict__ cd, const int2* __restrict__ span, int ngroup, double eps,
                             unsigned* status, const unsigned char* __restrict__ fit) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroup || (fit && fit[g >> 5])) return;      // staged groups run in k_rattle_warp
    int i1 = gidx[g], i2 = gidx[g + 1];
    const int lo = span[g].x, na = span[g].y;
    bool finished;
    if (na <= RATTLE_LOCAL) {
        double X[3 * RATTLE_LOCAL], V[3 * RATTLE_LOCAL], IM[RATTLE_LOCAL];
        for (int k = 0; k < 3 * na; ++k) { X[k] = pos[3 * lo + k]; V[k] = vel[3 * lo + k]; }
        for (int k = 0; k < na; ++k) IM[k] = invm[lo + k];
        finished = rattle_vel_sweeps(X, V, IM, lo, glist, cij, cd, i1, i2, eps);
        for (int ii = i1; ii < i2; ++ii) {
            const int2 p2 = cij[glist[ii]];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                vel[3 * p2.x + d] = V[3 * (p2.x - lo) + d];
                vel[3 * p2.y + d] = V[3 * (p2.y - lo) + d];
            }
        }
    } else {
        finished = rattle_vel_sweeps(pos, vel, invm, 0, glist, cij, cd, i1, i2, eps);
    }
    if (!finished) atomicOr(status, ST_RATTLEV_NOCONV);
}

// sum m v^2 and sum m v_a v_b (nhcint kint, calpress kinetic terms)

// ---- chain updates (single thread) -------------------------------------------
struct ChainArgs {
    pgk_mdparams md;
    int degfree;
    int dbl;
    int kind;          // 1 nhcint, 2 nhcpisoint, 3 nhcpanisoint
};

// The chain length M is a template parameter (mchain is checked to be 2..8
// before any launch), so the loops over the chain unroll and the chain's
// variables stay in registers through the serial update.
template <int M>
__device__ __forceinline__ void chain_tail(ChainDev& c, const pgk_mdparams& md, double* glogs, double w4,
                                           double w8, double gkt, bool down) {
    const double* q = md.qmass;
    if (down) {
        glogs[M - 1] = (q[M - 2] * c.vlogs[M - 2] * c.vlogs[M - 2] - gkt) / q[M - 1];
        c.vlogs[M - 1] = c.vlogs[M - 1] + glogs[M - 1] * w4;
#pragma unroll
        for (int i = M - 2; i >= 1; --i) {
            glogs[i] = (q[i - 1] * c.vlogs[i - 1] * c.vlogs[i - 1] - gkt) / q[i];
            double e8 = exp(-1.0 * w8 * c.vlogs[i + 1]);
            c.vlogs[i] = c.vlogs[i] * e8 * e8 + w4 * glogs[i] * e8;
        }
    } else {
#pragma unroll
        for (int i = 1; i <= M - 2; ++i) {
            glogs[i] = (q[i - 1] * c.vlogs[i - 1] * c.vlogs[i - 1] - gkt) / q[i];
            double e8 = exp(-1.0 * w8 * c.vlogs[i + 1]);
            c.vlogs[i] = c.vlogs[i] * e8 * e8 + w4 * glogs[i] * e8;
        }
        glogs[M - 1] = (q[M - 2] * c.vlogs[M - 2] * c.vlogs[M - 2] - gkt) / q[M - 1];
        c.vlogs[M - 1] = c.vlogs[M - 1] + glogs[M - 1] * w4;
    }
}

template <int M>
__device__ void chain_run_m(ChainDev* __restrict__ chain, const long long* __restrict__ acc, const ChainArgs& a) {
    ChainDev c = *chain;
    const pgk_mdparams& md = a.md;
    double dt = md.dt_long_cal;
    double kint = acc_get(acc, A_KE, a.dbl != 0);
    double glogs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double gkt = md.text;
    if (a.kind == 1) {   // nhcint.F90:8-140
        double gnkt = md.text * (double)a.degfree;
        glogs[0] = (kint - gnkt) / md.qmass[0];
        for (int inc = 0; inc < md.next; ++inc)
            for (int iy = 0; iy < md.nyosh; ++iy) {
                double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, true);
                double e8 = exp(-1.0 * w8 * c.vlogs[1]);
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
#pragma unroll
                for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, false);
            }
    } else if (a.kind == 2) {   // nhcpisoint.F90:6-162
        double gn1kt = md.text * (double)(a.degfree + 1);
        double dnf = 3.0 / (double)a.degfree;
        double vol = exp(3.0 * c.xlogv);
        glogs[0] = (kint + md.vmass * c.vlogv * c.vlogv - gn1kt) / md.qmass[0];
        double glogv = (dnf * kint + 3.0 * vol * (c.pint - md.pext)) / md.vmass;
        for (int inc = 0; inc < md.next; ++inc)
            for (int iy = 0; iy < md.nyosh; ++iy) {
                double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, true);
                double e8 = exp(-1.0 * w8 * c.vlogs[1]);
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
                e8 = exp(-1.0 * w8 * c.vlogs[0]);
                c.vlogv = c.vlogv * e8 * e8 + w4 * glogv * e8;
#pragma unroll
                for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
                c.vlogv = c.vlogv * e8 * e8 + w4 * glogv * e8;
                glogs[0] = (kint + md.vmass * c.vlogv * c.vlogv - gn1kt) / md.qmass[0];
                e8 = exp(-1.0 * w8 * c.vlogs[1]);
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, false);
            }
    } else {   // nhcpanisoint.F90:8-189
        int dir = md.pcont_axis == PGK_PCONT_ANISO ? 0 : md.pcont_axis - 1;
        double gndfkt = md.text * (double)(a.degfree + (dir == 0 ? 3 : 1));
        double dnf = 1.0 / (double)a.degfree;
        double vol = c.xboxh[0] * c.xboxh[1] * c.xboxh[2];
        double pv[3] = {c.pintt[0], c.pintt[4], c.pintt[8]};
        double vb2 = c.vboxg[0] * c.vboxg[0] + c.vboxg[1] * c.vboxg[1] + c.vboxg[2] * c.vboxg[2];
        glogs[0] = (kint + md.vmass * vb2 - gndfkt) / md.qmass[0];
        double gb[3];
        for (int d = 0; d < 3; ++d) gb[d] = (dnf * kint + vol * (pv[d] - md.pext)) / md.vmass;
        for (int inc = 0; inc < md.next; ++inc)
            for (int iy = 0; iy < md.nyosh; ++iy) {
                double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, true);
                double e8 = exp(-1.0 * w8 * c.vlogs[1]);
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
                e8 = exp(-1.0 * w8 * c.vlogs[0]);
                for (int d = 0; d < 3; ++d)
                    if (dir == 0 || d == dir - 1) c.vboxg[d] = c.vboxg[d] * e8 * e8 + w4 * gb[d] * e8;
#pragma unroll
                for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
                for (int d = 0; d < 3; ++d)
                    if (dir == 0 || d == dir - 1) c.vboxg[d] = c.vboxg[d] * e8 * e8 + w4 * gb[d] * e8;
                vb2 = c.vboxg[0] * c.vboxg[0] + c.vboxg[1] * c.vboxg[1] + c.vboxg[2] * c.vboxg[2];
                glogs[0] = (kint + md.vmass * vb2 - gndfkt) / md.qmass[0];
                e8 = exp(-1.0 * w8 * c.vlogs[1]);
                c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
                chain_tail<M>(c, md, glogs, w4, w8, gkt, false);
            }
    }
    *chain = c;
}

__device__ void chain_run(ChainDev* __restrict__ chain, const long long* __restrict__ acc, const ChainArgs& a) {
    switch (a.md.mchain) {
        case 2: chain_run_m<2>(chain, acc, a); break;
        case 3: chain_run_m<3>(chain, acc, a); break;
        case 4: chain_run_m<4>(chain, acc, a); break;
        case 5: chain_run_m<5>(chain, acc, a); break;
        case 6: chain_run_m<6>(chain, acc, a); break;
        case 7: chain_run_m<7>(chain, acc, a); break;
        default: chain_run_m<8>(chain, acc, a); break;
    }
}

// kick / drift coefficients of the step (moldyn_*.F90 at istep_short == 1)
// kind: 0 NVE, 1 NHC, 2 MTK
struct CoefArgs { pgk_mdparams md; int degfree; int kind; };

__device__ void coeffs_run(DynState* __restrict__ dyn, const ChainDev* __restrict__ chain, const CoefArgs& a) {
    const pgk_mdparams& md = a.md;
    const double dtl = md.dt_long_cal, dts = md.dt_long_cal / (double)md.nstep_short;
    const double e2 = 1.0 / 6.0, e4 = e2 / 20.0, e6 = e4 / 42.0, e8 = e6 / 72.0;
    const ChainDev& c = *chain;
    dyn->ks_b = 0.5 * dts;
    for (int d = 0; d < 3; ++d) { dyn->dr_a[d] = 1.0; dyn->dr_b[d] = dts; dyn->rvinv[d] = 1.0; }
    if (a.kind == 0) {
        for (int d = 0; d < 3; ++d) { dyn->kl_s[d] = 1.0; dyn->kl_b[d] = 0.5 * dtl; }
        return;
    }
    bool aniso = a.kind == 2 && md.pcont_axis != PGK_PCONT_ISO;
    if (!aniso) {
        double vext = c.vlogs[0];
        if (a.kind == 2) vext = c.vlogs[0] + (1.0 + 3.0 / (double)a.degfree) * c.vlogv;
        double ec4 = exp(-0.25 * dtl * vext);
        double a2 = (0.25 * dtl * vext) * (0.25 * dtl * vext);
        double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
        double cf = ec4 * poly;
        for (int d = 0; d < 3; ++d) { dyn->kl_s[d] = ec4 * ec4; dyn->kl_b[d] = cf * 0.5 * dtl; }
    } else {
        int dir = md.pcont_axis == PGK_PCONT_ANISO ? 0 : md.pcont_axis - 1;
        double vx[3] = {c.vlogs[0], c.vlogs[0], c.vlogs[0]};
        if (dir == 0) {
            double tr = c.vboxg[0] + c.vboxg[1] + c.vboxg[2];
            for (int d = 0; d < 3; ++d) vx[d] = c.vlogs[0] + c.vboxg[d] + 1.0 / (double)a.degfree * tr;
        } else {
            vx[dir - 1] = vx[dir - 1] + c.vboxg[dir - 1] + 1.0 / (double)a.degfree * c.vboxg[dir - 1];
        }
        for (int d = 0; d < 3; ++d) {
            double ec4 = exp(-0.25 * dtl * vx[d]);
            double a2 = (0.25 * dtl * vx[d]) * (0.25 * dtl * vx[d]);
            double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
            dyn->kl_s[d] = ec4 * ec4;
            dyn->kl_b[d] = ec4 * poly * 0.5 * dtl;
        }
    }
    if (a.kind == 2) {
        if (!aniso) {
            double aa = exp(0.5 * dts * c.vlogv), aa2 = aa * aa;
            double a2 = (0.5 * dts * c.vlogv) * (0.5 * dts * c.vlogv);
            double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
            for (int d = 0; d < 3; ++d) {
                dyn->dr_a[d] = aa2;
                dyn->dr_b[d] = aa * poly * dts;
                dyn->rvinv[d] = 1.0 / (aa * poly);
            }
        } else {
            for (int d = 0; d < 3; ++d) {
                double aa = exp(0.5 * dts * c.vboxg[d]);
                double a2 = (0.5 * dts * c.vboxg[d]) * (0.5 * dts * c.vboxg[d]);
                double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
                dyn->dr_a[d] = aa * aa;
                dyn->dr_b[d] = aa * poly * dts;
                dyn->rvinv[d] = 1.0 / (aa * poly);
            }
        }
    }
}

__global__ void k_coeffs(DynState* __restrict__ dyn, const ChainDev* __restrict__ chain, CoefArgs a) {
    if (threadIdx.x == 0 && blockIdx.x == 0) coeffs_run(dyn, chain, a);
}

// chain update followed by the step's coefficients (start of an NHC / MTK step)
__global__ void k_chain_coeffs(ChainDev* __restrict__ chain, const long long* __restrict__ acc, ChainArgs ca,
                               DynState* __restrict__ dyn, CoefArgs cf) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    chain_run(chain, acc, ca);
    coeffs_run(dyn, chain, cf);
}

// erf_corr_cutoff.F90:28-62 (the reference's min-ish rule kept)
__device__ double rkcut_of(const double* box, int n1, int n2, int n3) {
    double m1 = 0.5 * (n1 / box[0]);
    double rk = m1;
    double m2 = 0.5 * (n2 / box[1]);
    if (m2 < m1) rk = m2;
    double m3 = 0.5 * (n3 / box[2]);
    if (m3 < m2) rk = m3;
    return 0.9 * rk;
}

// volume / box update of one short step (calvol.F90, calbox.F90)
struct BoxArgs { double dts, rcut, rcut_book; int aniso, nfft1, nfft2, nfft3, update_rk; };

__global__ void k_box(DynState* __restrict__ dyn, ChainDev* __restrict__ chain, BoxArgs a, unsigned* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ChainDev& c = *chain;
    double b[3];
    if (!a.aniso) {
        c.xlogv = c.xlogv + c.vlogv * a.dts;
        double vol = exp(3.0 * c.xlogv);
        b[0] = pow(vol / dyn->yratio / dyn->zratio, 1.0 / 3.0);
        b[1] = dyn->yratio * b[0];
        b[2] = dyn->zratio * b[0];
    } else {
        for (int d = 0; d < 3; ++d) c.xboxh[d] = c.xboxh[d] * exp(c.vboxg[d] * a.dts);
        for (int d = 0; d < 3; ++d) b[d] = c.xboxh[d];
        dyn->yratio = b[1] / b[0];
        dyn->zratio = b[2] / b[0];
    }
    for (int d = 0; d < 3; ++d) { dyn->box[d] = b[d]; dyn->boxinv[d] = 1.0 / b[d]; }
    double h = fmin(b[0] * 0.5, fmin(b[1] * 0.5, b[2] * 0.5));
    if (a.rcut > h || a.rcut_book > h) atomicOr(status, ST_BOX_TOO_SMALL);
    if (a.update_rk) dyn->rkcut = rkcut_of(b, a.nfft1, a.nfft2, a.nfft3);
}

// calpress, atomic branch: pint / pintt of the current state from the kinetic
// sums and both groups' virials (+ self and net-charge terms)
struct PressArgs { double pot_ewc, netchrgsq, alpha; int ifspme, ifnetqcorrp, dbl; };

__device__ void press_run(const long long* __restrict__ acc, const DynState* __restrict__ dyn, ChainDev* chain,
                          const PressArgs& a) {
    const long long* A = acc;              // kinetic sums live in group 0
    const bool dbl = a.dbl != 0;
    double K = acc_get(A, A_KE, dbl);
    double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    double pi = 3.14159265358979323846;
    double a1 = -pi / (a.alpha * a.alpha * vol);
    double ewnq = a.ifspme ? 0.5 * a1 * a.netchrgsq : 0.0;
    double ewc = a.ifspme ? a.pot_ewc : 0.0;
    double W = ewc + ewnq, Wt[9];
    for (int k = 0; k < 9; ++k) Wt[k] = 0.0;
    for (int g = 0; g < 2; ++g) {
        const long long* G = acc + (size_t)g * NACC;
        W += acc_get(G, A_VC, dbl) + acc_get(G, A_VLJ, dbl) + acc_get(G, A_VB, dbl) + acc_get(G, A_VA, dbl) + acc_get(G, A_VT, dbl) + acc_get(G, A_V14, dbl) +
             acc_get(G, A_VMOR, dbl);   // calpress.F90:146-151 (pot_viri_mor)
        for (int k = 0; k < 9; ++k) {
            // coulomb / LJ tensors are stored as their lower triangle
            int r = k % 3, cl = k / 3;
            int ks = r >= cl ? k : cl + 3 * r;
            Wt[k] += acc_get(G, A_VTC + ks, dbl) + acc_get(G, A_VTLJ + ks, dbl) + acc_get(G, A_VTB + k, dbl) + acc_get(G, A_VTA + k, dbl) +
                     acc_get(G, A_VTT + k, dbl) + acc_get(G, A_VT14 + k, dbl) + acc_get(G, A_VTMOR + k, dbl);
        }
    }
    if (a.ifspme && !a.ifnetqcorrp) {      // calforce.F90:1018-1050 (long group)
        W += a1 * a.netchrgsq;
        for (int d = 0; d < 3; ++d) Wt[4 * d] += 0.5 * a1 * a.netchrgsq;
    } else if (a.ifspme) {
        W -= 0.5 * a1 * a.netchrgsq;
    }
    double b3 = (1.0 / dyn->box[0]) * (1.0 / dyn->box[1]) * (1.0 / dyn->box[2]);
    chain->pint = 1.0 / 3.0 * b3 * (K + W);
    for (int k = 0; k < 9; ++k) chain->pintt[k] = 1.0 * b3 * (acc_get(A, A_KET + k, dbl) + Wt[k]);
}

__global__ void k_press(const long long* __restrict__ acc, const DynState* __restrict__ dyn, ChainDev* chain,
                        PressArgs a) {
    if (threadIdx.x == 0 && blockIdx.x == 0) press_run(acc, dyn, chain, a);
}

// Kinetic sums (calkin: sum m v^2 and the tensor sum m v_a v_b) by a
// two-level reduction: every block writes its partial sums, and the last
// block to finish adds them in block order into the accumulator slots, which
// it overwrites (so nothing has to clear them first).  In mixed precision the
// partials are converted to 2^32 fixed point and added as integers (the exact
// sum per-block atomic adds would give); in FP64 the fixed order makes the
// sum deterministic.  MODE 1 then runs the chain update (nhcint, the end of an NHC
// step), MODE 2 the pressure and the chain update (calpress + nhcp*int, the
// end of an MTK step), in the last block's first thread: one launch instead of
// a clear, the reduction and a single-thread kernel.
template <int MODE>
__global__ void __launch_bounds__(256) k_kinetic_end(const double* __restrict__ vel, const double* __restrict__ mass,
                                                     int n, long long* acc, int dbl, double* part,
                                                     unsigned* done, const DynState* __restrict__ dyn,
                                                     ChainDev* chain, PressArgs pa, ChainArgs ca) {
    __shared__ double red[8][10];
    __shared__ bool last;
    double v[10] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = mass[i], x = vel[3 * i], y = vel[3 * i + 1], z = vel[3 * i + 2];
        v[0] += m * (x * x + y * y + z * z);
        const double w[3] = {x, y, z};
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) v[1 + a + 3 * b] += m * w[a] * w[b];
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 10; ++k) red[wp][k] = v[k];
    }
    __syncthreads();
    if (wp == 0) {
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            double x = lane < nw ? red[lane][k] : 0.0;
            x = warp_sum(x);
            if (lane == 0) part[10 * (size_t)blockIdx.x + k] = x;
        }
        if (lane == 0) {
            __threadfence();
            last = atomicAdd(done, 1u) == gridDim.x - 1u;
        }
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int idx[10] = {A_KE, A_KET + 0, A_KET + 1, A_KET + 2, A_KET + 3, A_KET + 4, A_KET + 5, A_KET + 6,
                         A_KET + 7, A_KET + 8};
    // every thread adds the partials of blocks t, t + 256, ... (loads in
    // flight together), then a fixed-shape block reduction: deterministic
    __shared__ long long ired[8][10];
    __shared__ double dred[8][10];
    long long is[10];
    double ds[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) { is[k] = 0; ds[k] = 0.0; }
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            const double x = __ldcg(part + 10 * (size_t)b + k);
            if (dbl) ds[k] += x;
            else is[k] += to_fix(x, PGK_FORCE_SCALE);
        }
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        if (dbl) ds[k] = warp_sum(ds[k]);
        else is[k] = warp_sum(is[k]);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 10; ++k) { ired[wp][k] = is[k]; dred[wp][k] = ds[k]; }
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        const int k = threadIdx.x;
        long long si = 0;
        double sd = 0.0;
        for (int w = 0; w < nw; ++w) { si += ired[w][k]; sd += dred[w][k]; }
        acc[idx[k]] = dbl ? __double_as_longlong(sd) : si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *done = 0u;
        if (MODE == 2) press_run(acc, dyn, chain, pa);
        if (MODE >= 1) chain_run(chain, acc, ca);
    }
}

template <bool MIXED>
__global__ void k_copy_force(const void* __restrict__ f, double* __restrict__ out, int n3) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n3) out[k] = force_get<MIXED>(f, k);
}

// ---- launchers ----------------------------------------------------------------
// one MTS group's force accumulator (3N x 8 B) and energy/virial slots
// cleared by one kernel (16-byte stores; the accumulator is 16-byte aligned)
__global__ void k_zero_group(longlong2* __restrict__ f, size_t n2, long long* __restrict__ f_tail, int tail,
                             long long* __restrict__ acc) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n2) f[k] = make_longlong2(0, 0);
    if (k < (size_t)tail) f_tail[k] = 0;
    if (k < NACC) acc[k] = 0;
}

pgk_status launch_zero_group(pgk_ctx* c, int g) {
    const size_t n3 = (size_t)3 * c->natom, n2 = n3 / 2;
    const size_t nt = std::max(n2, (size_t)NACC);
    k_zero_group<<<(unsigned)((nt + 255) / 256), 256, 0, c->st>>>((longlong2*)c->facc[g], n2,
                                                                 (long long*)c->facc[g] + 2 * n2, (int)(n3 - 2 * n2),
                                                                 c->acc + (size_t)g * NACC);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_kick_drift(pgk_ctx* c, int flags) {
    if (!flags) return PGK_OK;
    const int n3 = 3 * c->natom;
    if (c->mixed())
        k_kick_drift<true><<<(n3 + 255) / 256, 256, 0, c->st>>>(c->vel, c->pos, c->pos_old, c->facc[0], c->facc[1],
                                                               c->mass, c->natom, c->dyn, flags);
    else
        k_kick_drift<false><<<(n3 + 255) / 256, 256, 0, c->st>>>(c->vel, c->pos, c->pos_old, c->facc[0], c->facc[1],
                                                                c->mass, c->natom, c->dyn, flags);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// Warp-staged RATTLE: the 32 groups of a warp (consecutive groups cover a
// compact atom range) stage the union of their atom spans and their
// constraints in shared memory with coalesced loads; each lane then runs its
// group's sweeps (same arithmetic, same order as rattle_*_sweeps) from shared
// memory and writes back its own atoms.  Warps whose union span or
// constraint counts exceed the staging limits run the per-thread kernels.
#define RATTLE_WSPAN 192          // atoms staged per warp
#define RATTLE_WCON 8             // constraints per group
#define RATTLE_WARPS 4

struct RattleStage {
    double x[3 * RATTLE_WSPAN], v[3 * RATTLE_WSPAN], o[3 * RATTLE_WSPAN], im[RATTLE_WSPAN];
    int2 ij[32 * RATTLE_WCON];
    double d2[32 * RATTLE_WCON];
    double rc[32 * RATTLE_WCON];   // per constraint: 1/d^2 (positions), 1/(d^2 (1/m_i + 1/m_j)) (velocities)
};

template <bool POS>
__global__ void __launch_bounds__(32 * RATTLE_WARPS) k_rattle_warp(double* __restrict__ pos, double* __restrict__ vel,
                                                                  const double* __restrict__ old,
                                                                  const double* __restrict__ invm,
                                                                  const int* __restrict__ gidx,
                                                                  const int* __restrict__ glist,
                                                                  const int2* __restrict__ cij,
                                                                  const double* __restrict__ cd,
                                                                  const int2* __restrict__ span, int ngroup,
                                                                  double eps, double dt, int use_rv,
                                                                  const DynState* __restrict__ dyn,
                                                                  unsigned* status,
                                                                  const unsigned char* __restrict__ fit) {
    extern __shared__ __align__(16) unsigned char rsm_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gw = (blockIdx.x * RATTLE_WARPS + w) * 32;
    if (gw >= ngroup || !fit[gw >> 5]) return;                  // warp-uniform; others: per-thread kernel
    RattleStage& S = ((RattleStage*)rsm_raw)[w];
    const int g = gw + lane;
    const bool has = g < ngroup;
    const int i1 = has ? gidx[g] : 0, i2 = has ? gidx[g + 1] : 0;
    const int2 sp = has ? span[g] : make_int2(0x7fffffff, 0);
    const int lo = __reduce_min_sync(0xffffffffu, has ? sp.x : 0x7fffffff);
    const int hi = __reduce_max_sync(0xffffffffu, has ? sp.x + sp.y : 0);
    const int nsp = hi - lo;                                    // <= RATTLE_WSPAN (fit)
#pragma unroll 4
    for (int k = lane; k < 3 * nsp; k += 32) {
        S.x[k] = pos[3 * (size_t)lo + k];
        S.v[k] = vel[3 * (size_t)lo + k];
        if (POS) S.o[k] = old[3 * (size_t)lo + k];
    }
    for (int k = lane; k < nsp; k += 32) S.im[k] = invm[lo + k];
    const int ncon = i2 - i1;
    for (int q = 0; q < ncon; ++q) {
        const int nc = glist[i1 + q];
        const int2 p = cij[nc];
        const double dij = cd[nc];
        S.ij[lane * RATTLE_WCON + q] = make_int2(p.x - lo, p.y - lo);
        S.d2[lane * RATTLE_WCON + q] = dij * dij;
    }
    __syncwarp();
    // The sweeps' convergence tests and the velocity correction divide by
    // per-constraint constants: their reciprocals are formed once here, so
    // the serial sweep chain holds one FP64 division per correction instead
    // of two per constraint (the tests differ from the reference's quotient
    // by at most an ulp of eps)
    for (int q = 0; q < ncon; ++q) {
        const int2 p = S.ij[lane * RATTLE_WCON + q];
        const double d2 = S.d2[lane * RATTLE_WCON + q];
        S.rc[lane * RATTLE_WCON + q] = POS ? 1.0 / d2 : 1.0 / (d2 * (S.im[p.x] + S.im[p.y]));
    }
    double* X = S.x; double* V = S.v; const double* O = S.o; const double* IM = S.im;
    const int2* C = S.ij + lane * RATTLE_WCON;
    const double* D2 = S.d2 + lane * RATTLE_WCON;
    const double* RC = S.rc + lane * RATTLE_WCON;
    bool finished = false;
    if (POS) {
        double rvi[3] = {1.0, 1.0, 1.0};
        if (use_rv) { rvi[0] = dyn->rvinv[0]; rvi[1] = dyn->rvinv[1]; rvi[2] = dyn->rvinv[2]; }
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
            for (int q = 0; q < ncon; ++q) {
                const int ib = C[q].x, jb = C[q].y;
                const double d2 = D2[q];
                double R0 = X[3 * ib] - X[3 * jb], R1 = X[3 * ib + 1] - X[3 * jb + 1], R2 = X[3 * ib + 2] - X[3 * jb + 2];
                double Rsq = R0 * R0 + R1 * R1 + R2 * R2;
                double delta = fabs(Rsq - d2) * RC[q];      // |r^2 - d^2| / d^2
                if (delta < eps) continue;
                finished = false;
                double O0 = O[3 * ib] - O[3 * jb], O1 = O[3 * ib + 1] - O[3 * jb + 1], O2 = O[3 * ib + 2] - O[3 * jb + 2];
                double RR = R0 * O0 + R1 * O1 + R2 * O2;
                double mi = IM[ib], mj = IM[jb];
                double gij = (Rsq - d2) / (2.0 * RR * (mi + mj) * dt);
                double G[3] = {gij * O0, gij * O1, gij * O2};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    X[3 * ib + d] = X[3 * ib + d] - mi * G[d] * dt;
                    X[3 * jb + d] = X[3 * jb + d] + mj * G[d] * dt;
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double Gv = G[d] * rvi[d];
                    V[3 * ib + d] = V[3 * ib + d] - mi * Gv;
                    V[3 * jb + d] = V[3 * jb + d] + mj * Gv;
                }
            }
        }
    } else {
        const double eps2 = eps * eps;
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
            for (int q = 0; q < ncon; ++q) {
                const int ib = C[q].x, jb = C[q].y;
                const double dd = D2[q];          // dij * dij
                double R[3], W[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    R[d] = X[3 * ib + d] - X[3 * jb + d];
                    W[d] = V[3 * ib + d] - V[3 * jb + d];
                }
                double RV = R[0] * W[0] + R[1] * W[1] + R[2] * W[2];
                double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                double V2 = W[0] * W[0] + W[1] * W[1] + W[2] * W[2];
                if (RV * RV * V2 < eps2 * R2) continue;     // (RV^2 / R^2) V^2 < eps^2, R^2 > 0
                finished = false;
                double mi = IM[ib], mj = IM[jb];
                double kij = RV * RC[q];                    // RV / (d^2 (1/m_i + 1/m_j))
                (void)dd;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double KR = kij * R[d];
                    V[3 * ib + d] = V[3 * ib + d] - mi * KR;
                    V[3 * jb + d] = V[3 * jb + d] + mj * KR;
                }
            }
        }
    }
    if (has) {
        for (int q = 0; q < ncon; ++q) {
            const int ib = C[q].x, jb = C[q].y;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (POS) { pos[3 * ((size_t)lo + ib) + d] = X[3 * ib + d]; pos[3 * ((size_t)lo + jb) + d] = X[3 * jb + d]; }
                vel[3 * ((size_t)lo + ib) + d] = V[3 * ib + d];
                vel[3 * ((size_t)lo + jb) + d] = V[3 * jb + d];
            }
        }
        if (!finished) atomicOr(status, POS ? ST_RATTLE_NOCONV : ST_RATTLEV_NOCONV);
    }
}

// Rigid three-atom groups (rigid water): constraints q0 = (a0,a1), q1 =
// (a0,a2), q2 = (a1,a2), swept in that order.  One thread per group with its
// three atoms' positions, velocities, old positions and inverse masses in
// registers: the sweeps are the same arithmetic in the same order as
// k_rattle_warp (rattle_c / rattle_cmtk, rattle_mtk.F90:278-542 for the
// velocities), without a shared-memory round trip in the serial chain.
template <bool POS>
__global__ void __launch_bounds__(128) k_rattle_rigid3(double* __restrict__ pos, double* __restrict__ vel,
                                                       const double* __restrict__ old,
                                                       const double* __restrict__ invm,
                                                       const int4* __restrict__ atoms,
                                                       const double4* __restrict__ dl, int ngroup, double eps,
                                                       double dt, int use_rv, const DynState* __restrict__ dyn,
                                                       unsigned* status) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroup) return;
    const int4 A = atoms[g];
    const int at[3] = {A.x, A.y, A.z};
    const double4 D = dl[g];
    double X[3][3], V[3][3], O[3][3], IM[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        IM[a] = invm[at[a]];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            X[a][d] = pos[3 * (size_t)at[a] + d];
            V[a][d] = vel[3 * (size_t)at[a] + d];
            O[a][d] = POS ? old[3 * (size_t)at[a] + d] : 0.0;
        }
    }
    constexpr int CI[3] = {0, 0, 1}, CJ[3] = {1, 2, 2};
    const double dd[3] = {D.x * D.x, D.y * D.y, D.z * D.z};
    double RC[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) RC[q] = POS ? 1.0 / dd[q] : 1.0 / (dd[q] * (IM[CI[q]] + IM[CJ[q]]));
    bool finished = false;
    if (POS) {
        double rvi[3] = {1.0, 1.0, 1.0};
        if (use_rv) { rvi[0] = dyn->rvinv[0]; rvi[1] = dyn->rvinv[1]; rvi[2] = dyn->rvinv[2]; }
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int ib = CI[q], jb = CJ[q];
                const double d2 = dd[q];
                const double R0 = X[ib][0] - X[jb][0], R1 = X[ib][1] - X[jb][1], R2 = X[ib][2] - X[jb][2];
                const double Rsq = R0 * R0 + R1 * R1 + R2 * R2;
                const double delta = fabs(Rsq - d2) * RC[q];      // |r^2 - d^2| / d^2
                if (delta < eps) continue;
                finished = false;
                const double O0 = O[ib][0] - O[jb][0], O1 = O[ib][1] - O[jb][1], O2 = O[ib][2] - O[jb][2];
                const double RR = R0 * O0 + R1 * O1 + R2 * O2;
                const double mi = IM[ib], mj = IM[jb];
                const double gij = (Rsq - d2) / (2.0 * RR * (mi + mj) * dt);
                const double G[3] = {gij * O0, gij * O1, gij * O2};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    X[ib][d] = X[ib][d] - mi * G[d] * dt;
                    X[jb][d] = X[jb][d] + mj * G[d] * dt;
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double Gv = G[d] * rvi[d];
                    V[ib][d] = V[ib][d] - mi * Gv;
                    V[jb][d] = V[jb][d] + mj * Gv;
                }
            }
        }
    } else {
        const double eps2 = eps * eps;
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int ib = CI[q], jb = CJ[q];
                double R[3], W[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    R[d] = X[ib][d] - X[jb][d];
                    W[d] = V[ib][d] - V[jb][d];
                }
                const double RV = R[0] * W[0] + R[1] * W[1] + R[2] * W[2];
                const double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                const double V2 = W[0] * W[0] + W[1] * W[1] + W[2] * W[2];
                if (RV * RV * V2 < eps2 * R2) continue;     // (RV^2 / R^2) V^2 < eps^2, R^2 > 0
                finished = false;
                const double mi = IM[ib], mj = IM[jb];
                const double kij = RV * RC[q];              // RV / (d^2 (1/m_i + 1/m_j))
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double KR = kij * R[d];
                    V[ib][d] = V[ib][d] - mi * KR;
                    V[jb][d] = V[jb][d] + mj * KR;
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (POS) pos[3 * (size_t)at[a] + d] = X[a][d];
            vel[3 * (size_t)at[a] + d] = V[a][d];
        }
    if (!finished) atomicOr(status, POS ? ST_RATTLE_NOCONV : ST_RATTLEV_NOCONV);
}

// Star groups: constraints q = (c, a_{q+1}), q = 0..K-1, swept in that order
// (the X-H bonds of one heavy atom).  One thread per group, state in
// registers; same arithmetic and order as k_rattle_warp.
template <bool POS, int K>
__device__ __forceinline__ void rattle_star_group(int g, double* __restrict__ pos, double* __restrict__ vel,
                                                  const double* __restrict__ old, const double* __restrict__ invm,
                                                  const int* __restrict__ sa, const double* __restrict__ sd,
                                                  double eps, double dt, const double (&rvi)[3],
                                                  unsigned* status) {
    int at[K + 1];
    double X[K + 1][3], V[K + 1][3], O[K + 1][3], IM[K + 1], dd[K], RC[K];
#pragma unroll
    for (int a = 0; a <= K; ++a) {
        at[a] = sa[5 * (size_t)g + a];
        IM[a] = invm[at[a]];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            X[a][d] = pos[3 * (size_t)at[a] + d];
            V[a][d] = vel[3 * (size_t)at[a] + d];
            O[a][d] = POS ? old[3 * (size_t)at[a] + d] : 0.0;
        }
    }
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const double dij = sd[4 * (size_t)g + q];
        dd[q] = dij * dij;
        RC[q] = POS ? 1.0 / dd[q] : 1.0 / (dd[q] * (IM[0] + IM[q + 1]));
    }
    bool finished = false;
    if (POS) {
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
#pragma unroll
            for (int q = 0; q < K; ++q) {
                constexpr int ib = 0;
                const int jb = q + 1;
                const double d2 = dd[q];
                const double R0 = X[ib][0] - X[jb][0], R1 = X[ib][1] - X[jb][1], R2 = X[ib][2] - X[jb][2];
                const double Rsq = R0 * R0 + R1 * R1 + R2 * R2;
                const double delta = fabs(Rsq - d2) * RC[q];      // |r^2 - d^2| / d^2
                if (delta < eps) continue;
                finished = false;
                const double O0 = O[ib][0] - O[jb][0], O1 = O[ib][1] - O[jb][1], O2 = O[ib][2] - O[jb][2];
                const double RR = R0 * O0 + R1 * O1 + R2 * O2;
                const double mi = IM[ib], mj = IM[jb];
                const double gij = (Rsq - d2) / (2.0 * RR * (mi + mj) * dt);
                const double G[3] = {gij * O0, gij * O1, gij * O2};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    X[ib][d] = X[ib][d] - mi * G[d] * dt;
                    X[jb][d] = X[jb][d] + mj * G[d] * dt;
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double Gv = G[d] * rvi[d];
                    V[ib][d] = V[ib][d] - mi * Gv;
                    V[jb][d] = V[jb][d] + mj * Gv;
                }
            }
        }
    } else {
        const double eps2 = eps * eps;
        for (int it = 0; it < 300 && !finished; ++it) {
            finished = true;
#pragma unroll
            for (int q = 0; q < K; ++q) {
                constexpr int ib = 0;
                const int jb = q + 1;
                double R[3], W[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    R[d] = X[ib][d] - X[jb][d];
                    W[d] = V[ib][d] - V[jb][d];
                }
                const double RV = R[0] * W[0] + R[1] * W[1] + R[2] * W[2];
                const double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                const double V2 = W[0] * W[0] + W[1] * W[1] + W[2] * W[2];
                if (RV * RV * V2 < eps2 * R2) continue;     // (RV^2 / R^2) V^2 < eps^2, R^2 > 0
                finished = false;
                const double mi = IM[ib], mj = IM[jb];
                const double kij = RV * RC[q];              // RV / (d^2 (1/m_i + 1/m_j))
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double KR = kij * R[d];
                    V[ib][d] = V[ib][d] - mi * KR;
                    V[jb][d] = V[jb][d] + mj * KR;
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a <= K; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (POS) pos[3 * (size_t)at[a] + d] = X[a][d];
            vel[3 * (size_t)at[a] + d] = V[a][d];
        }
    if (!finished) atomicOr(status, POS ? ST_RATTLE_NOCONV : ST_RATTLEV_NOCONV);
}

// seg: first group with K = 3, 2, 1 and the group count (groups sorted by K
// from 4 down, so a warp's groups mostly share K)
template <bool POS>
__global__ void __launch_bounds__(128) k_rattle_star(double* __restrict__ pos, double* __restrict__ vel,
                                                     const double* __restrict__ old, const double* __restrict__ invm,
                                                     const int* __restrict__ sa, const double* __restrict__ sd,
                                                     int4 seg, double eps, double dt, int use_rv,
                                                     const DynState* __restrict__ dyn, unsigned* status) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= seg.w) return;
    double rvi[3] = {1.0, 1.0, 1.0};
    if (POS && use_rv) { rvi[0] = dyn->rvinv[0]; rvi[1] = dyn->rvinv[1]; rvi[2] = dyn->rvinv[2]; }
    if (g < seg.x) rattle_star_group<POS, 4>(g, pos, vel, old, invm, sa, sd, eps, dt, rvi, status);
    else if (g < seg.y) rattle_star_group<POS, 3>(g, pos, vel, old, invm, sa, sd, eps, dt, rvi, status);
    else if (g < seg.z) rattle_star_group<POS, 2>(g, pos, vel, old, invm, sa, sd, eps, dt, rvi, status);
    else rattle_star_group<POS, 1>(g, pos, vel, old, invm, sa, sd, eps, dt, rvi, status);
}

static void rattle_star_launch(pgk_ctx* c, bool pos, double eps, double dt, bool use_rv) {
    const int blocks = (c->nstar + 127) / 128;
    const int4 seg = make_int4(c->star_seg[0], c->star_seg[1], c->star_seg[2], c->star_seg[3]);
    if (pos)
        k_rattle_star<true><<<blocks, 128, 0, c->st>>>(c->pos, c->vel, c->pos_old, c->invmass, c->star_atoms,
                                                       c->star_d, seg, eps, dt, use_rv ? 1 : 0, c->dyn, c->status);
    else
        k_rattle_star<false><<<blocks, 128, 0, c->st>>>(c->pos, c->vel, nullptr, c->invmass, c->star_atoms,
                                                        c->star_d, seg, eps, 0.0, 0, c->dyn, c->status);
    PGK_LAUNCHED(c);
}

static void rattle_rigid3_launch(pgk_ctx* c, bool pos, double eps, double dt, bool use_rv) {
    const int blocks = (c->nr3 + 127) / 128;
    if (pos)
        k_rattle_rigid3<true><<<blocks, 128, 0, c->st>>>(c->pos, c->vel, c->pos_old, c->invmass, c->r3_atoms,
                                                         c->r3_d, c->nr3, eps, dt, use_rv ? 1 : 0, c->dyn, c->status);
    else
        k_rattle_rigid3<false><<<blocks, 128, 0, c->st>>>(c->pos, c->vel, nullptr, c->invmass, c->r3_atoms,
                                                          c->r3_d, c->nr3, eps, 0.0, 0, c->dyn, c->status);
    PGK_LAUNCHED(c);
}

static void rattle_warp_launch(pgk_ctx* c, bool pos, double eps, double dt, bool use_rv) {
    const int nwarp = (c->ncgroup + 31) / 32;
    const int blocks = (nwarp + RATTLE_WARPS - 1) / RATTLE_WARPS;
    const size_t sm = RATTLE_WARPS * sizeof(RattleStage);
    if (pos) {
        smem_limit(k_rattle_warp<true>, sm);
        k_rattle_warp<true><<<blocks, 32 * RATTLE_WARPS, sm, c->st>>>(c->pos, c->vel, c->pos_old, c->invmass,
                                                                     c->cg_idx, c->cg_list, c->c_ij, c->c_d,
                                                                     c->cg_span, c->ncgroup, eps, dt, use_rv ? 1 : 0,
                                                                     c->dyn, c->status, c->cg_fit);
    } else {
        smem_limit(k_rattle_warp<false>, sm);
        k_rattle_warp<false><<<blocks, 32 * RATTLE_WARPS, sm, c->st>>>(c->pos, c->vel, nullptr, c->invmass,
                                                                      c->cg_idx, c->cg_list, c->c_ij, c->c_d,
                                                                      c->cg_span, c->ncgroup, eps, 0.0, 0, c->dyn,
                                                                      c->status, c->cg_fit);
    }
    PGK_LAUNCHED(c);
}

pgk_status launch_rattle_pos(pgk_ctx* c, double eps, double dt, bool use_rv) {
    if (c->nr3 > 0) rattle_rigid3_launch(c, true, eps, dt, use_rv);
    if (c->nstar > 0) rattle_star_launch(c, true, eps, dt, use_rv);
    if (c->ncgroup == 0) { PGK_CUDA(c, cudaGetLastError()); return PGK_OK; }
    if (c->cg_nfit > 0) rattle_warp_launch(c, true, eps, dt, use_rv);
    if (c->cg_nfit < (c->ncgroup + 31) / 32) {
        k_rattle_pos<<<(c->ncgroup + 63) / 64, 64, 0, c->st>>>(c->pos, c->vel, c->pos_old, c->invmass, c->cg_idx,
                                                               c->cg_list, c->c_ij, c->c_d, c->cg_span, c->ncgroup,
                                                               eps, dt, use_rv ? 1 : 0, c->dyn, c->status,
                                                               c->cg_nfit > 0 ? c->cg_fit : nullptr);
        PGK_LAUNCHED(c);
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_rattle_vel(pgk_ctx* c, double eps) {
    if (c->nr3 > 0) rattle_rigid3_launch(c, false, eps, 0.0, false);
    if (c->nstar > 0) rattle_star_launch(c, false, eps, 0.0, false);
    if (c->ncgroup == 0) { PGK_CUDA(c, cudaGetLastError()); return PGK_OK; }
    if (c->cg_nfit > 0) rattle_warp_launch(c, false, eps, 0.0, false);
    if (c->cg_nfit < (c->ncgroup + 31) / 32) {
        k_rattle_vel<<<(c->ncgroup + 63) / 64, 64, 0, c->st>>>(c->pos, c->vel, c->invmass, c->cg_idx, c->cg_list,
                                                               c->c_ij, c->c_d, c->cg_span, c->ncgroup, eps, c->status,
                                                               c->cg_nfit > 0 ? c->cg_fit : nullptr);
        PGK_LAUNCHED(c);
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// kinetic sums into the group's accumulator (the kinetic slots of group 0
// are the ones calpress and the chains read)
pgk_status launch_kinetic(pgk_ctx* c, int group) {
    long long* acc = c->acc + (size_t)group * NACC;
    int blocks = std::min(c->nsm * 2, (c->natom + 255) / 256);
    if (blocks < 1) blocks = 1;
    k_kinetic_end<0><<<blocks, 256, 0, c->st>>>(c->vel, c->mass, c->natom, acc, c->mixed() ? 0 : 1, c->ke_part,
                                                 c->ke_done, c->dyn, c->chain, PressArgs{}, ChainArgs{});
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// mode 1: kinetic sums + chain update (end of an NHC step); 2: kinetic sums +
// pressure + chain update (end of an MTK step)
pgk_status launch_kinetic_end(pgk_ctx* c, int mode, int chain_kind, const pgk_mdparams& md) {
    PressArgs pa;
    pa.pot_ewc = c->pot_ewc;
    pa.netchrgsq = c->netchrgsq;
    pa.alpha = c->prm.alpha;
    pa.ifspme = c->prm.ifspme;
    pa.ifnetqcorrp = c->prm.ifnetqcorrp;
    pa.dbl = c->mixed() ? 0 : 1;
    ChainArgs ca;
    ca.md = md;
    ca.degfree = c->degfree;
    ca.dbl = c->mixed() ? 0 : 1;
    ca.kind = chain_kind;
    int blocks = std::min(c->nsm * 2, (c->natom + 255) / 256);
    if (blocks < 1) blocks = 1;
    if (mode == 2)
        k_kinetic_end<2><<<blocks, 256, 0, c->st>>>(c->vel, c->mass, c->natom, c->acc, pa.dbl, c->ke_part, c->ke_done,
                                                     c->dyn, c->chain, pa, ca);
    else
        k_kinetic_end<1><<<blocks, 256, 0, c->st>>>(c->vel, c->mass, c->natom, c->acc, pa.dbl, c->ke_part, c->ke_done,
                                                     c->dyn, c->chain, pa, ca);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_chain_coeffs(pgk_ctx* c, int chain_kind, int coef_kind, const pgk_mdparams& md) {
    ChainArgs ca;
    ca.md = md;
    ca.degfree = c->degfree;
    ca.dbl = c->mixed() ? 0 : 1;
    ca.kind = chain_kind;
    CoefArgs cf;
    cf.md = md;
    cf.degfree = c->degfree;
    cf.kind = coef_kind;
    k_chain_coeffs<<<1, 32, 0, c->st>>>(c->chain, c->acc, ca, c->dyn, cf);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_coeffs(pgk_ctx* c, int kind, const pgk_mdparams& md, int) {
    CoefArgs a;
    a.md = md;
    a.degfree = c->degfree;
    a.kind = kind;
    k_coeffs<<<1, 32, 0, c->st>>>(c->dyn, c->chain, a);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_box_update(pgk_ctx* c, int kind, const pgk_mdparams& md, bool with_rkcut) {
    BoxArgs a;
    a.dts = md.dt_long_cal / (double)md.nstep_short;
    a.rcut = c->prm.rcut;
    a.rcut_book = c->prm.rcut_book;
    a.aniso = (kind == 2 && md.pcont_axis != PGK_PCONT_ISO) ? 1 : 0;
    a.nfft1 = c->prm.nfft1; a.nfft2 = c->prm.nfft2; a.nfft3 = c->prm.nfft3;
    a.update_rk = (with_rkcut || c->prm.mts_ewk == PGK_MTS_SHORT) ? 1 : 0;
    k_box<<<1, 32, 0, c->st>>>(c->dyn, c->chain, a, c->status);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_press(pgk_ctx* c) {
    PressArgs a;
    a.pot_ewc = c->pot_ewc;
    a.netchrgsq = c->netchrgsq;
    a.alpha = c->prm.alpha;
    a.ifspme = c->prm.ifspme;
    a.ifnetqcorrp = c->prm.ifnetqcorrp;
    a.dbl = c->mixed() ? 0 : 1;
    k_press<<<1, 32, 0, c->st>>>(c->acc, c->dyn, c->chain, a);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_copy_force(pgk_ctx* c, int group, double* dst) {
    int n3 = 3 * c->natom;
    if (c->mixed()) k_copy_force<true><<<(n3 + 255) / 256, 256, 0, c->st>>>(c->facc[group], dst, n3);
    else k_copy_force<false><<<(n3 + 255) / 256, 256, 0, c->st>>>(c->facc[group], dst, n3);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// ---- output record (outene / outpre values) of the current step ----------------
// Sums both MTS groups' accumulators like the host read-back does, adds the
// Ewald self and net-charge constants, and stores one PGK_OUT_NCOL record.
__global__ void k_out_record(const long long* __restrict__ acc, const DynState* __restrict__ dyn,
                             const ChainDev* __restrict__ ch, int dbl, double pot_ewc, double alpha, double netchrgsq,
                             int ifspme, long long step, double* __restrict__ r) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    auto S = [&](int k) { return acc_get(acc, k, dbl != 0) + acc_get(acc + NACC, k, dbl != 0); };
    const double pi = 3.14159265358979323846;
    const double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    const double a1 = -pi / (alpha * alpha * vol);
    double e_vdw = S(A_VDW), e_elc = S(A_ELC), e_ewk = S(A_EWK), e_v14 = S(A_VDW14), e_e14 = S(A_ELC14);
    double e_b = S(A_BOND), e_a = S(A_ANGL), e_t = S(A_TORS), e_rb = S(A_TORSRB), e_mor = S(A_MOR);
    double e_ewc = ifspme ? pot_ewc : 0.0, e_nq = ifspme ? 0.5 * a1 * netchrgsq : 0.0;
    double nonbon = e_vdw + e_elc + e_ewk + e_ewc + e_nq + e_v14 + e_e14;
    double tot = e_b + e_a + e_t + e_rb + e_mor + nonbon;   // calforce.F90: pot_mor is outside pot_nonbon
    r[0] = (double)step;
    r[1] = tot; r[2] = nonbon; r[3] = e_vdw; r[4] = e_elc; r[5] = e_ewk; r[6] = e_ewc; r[7] = e_nq;
    r[8] = e_v14; r[9] = e_e14; r[10] = e_b; r[11] = e_a; r[12] = e_t; r[13] = e_rb; r[14] = e_mor;
    r[15] = acc_get(acc, A_KE, dbl != 0);
    r[16] = ch->pint;
    for (int k = 0; k < 9; ++k) r[17 + k] = ch->pintt[k];
    for (int d = 0; d < 3; ++d) r[26 + d] = dyn->box[d];
}
static_assert(PGK_OUT_NCOL == 29 && sizeof(pgk_energies) == 14 * sizeof(double), "output record layout");

pgk_status launch_out_record(pgk_ctx* c, long long step, double* dst) {
    pgk_status s;
    if ((s = launch_kinetic(c, 0))) return s;
    k_out_record<<<1, 32, 0, c->st>>>(c->acc, c->dyn, c->chain, c->mixed() ? 0 : 1, c->pot_ewc, c->prm.alpha,
                                      c->netchrgsq, c->prm.ifspme, step, dst);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}
