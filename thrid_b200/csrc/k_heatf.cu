// k_heatf.cu -- heat flux of the -DHF build and the region Langevin thermostat.
//
//   calcom.F90                  molecule centres of mass (k_calcom)
//   ewaldr_hf.F90:213-520       per-atom pair potentials and the calvirihf
//                               virial of every list pair (k_hf_pair)
//   cal*_hf.F90                 bonded parts (k_bonded.cu, launch_bonded_hf)
//   calheatf.F90:365-1466       region sums of the kinetic, potential and
//                               virial transport terms (k_heatf_part/_final)
//   langevin_regist.F90         region of each atom (k_lt_regist)
//   langevin_region.F90         half steps with random and friction terms
//                               (k_langevin)
//
// The per-atom arrays stay on the device in original atom order:
// pot[8][N] and the z column of the per-atom virial W[8][nreg][3][N]
// (category-major, so calheatf reads them coalesced).  Heat-flux steps only
// (heatfinterval); the ordinary force kernels are unchanged on those steps.
//
// k_hf_pair walks the same 8-atom cluster rows as the pair kernel: one warp
// per cluster, one lane per (cluster, j) entry, a loop over the cluster atoms
// whose mask bit is set; every list pair is stored once.  The cluster atom's
// shares collect in per-warp shared memory and are flushed once per cluster;
// j's shares go straight to the global arrays.  Both use FP64 atomics, since
// other warps add j shares to the same atoms.
// Pair arithmetic is FP32 in mixed precision and FP64 otherwise; region
// geometry and all sums are FP64 in global memory.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "pgk_ctx.cuh"
#include "pgk_hf.cuh"

// ---- calcom.F90 / molecule velocities of calheatf.F90:556-607 -------------------
__global__ void k_calcom(const double* __restrict__ x, const double* __restrict__ mass,
                         const int* __restrict__ mol_idx, const int* __restrict__ mol_list, int nmole,
                         const DynState* __restrict__ dyn, int wrap, double* __restrict__ out) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmole) return;
    int b = mol_idx[m], e = mol_idx[m + 1];
    double c[3];
    if (e - b == 1) {
        int i = mol_list[b];
        c[0] = x[3 * i]; c[1] = x[3 * i + 1]; c[2] = x[3 * i + 2];
    } else {
        double ms = 0.0;
        c[0] = c[1] = c[2] = 0.0;
        for (int q = b; q < e; ++q) {
            int i = mol_list[q];
            double mi = mass[i];
            ms = ms + mi;
            c[0] = c[0] + mi * x[3 * i]; c[1] = c[1] + mi * x[3 * i + 1]; c[2] = c[2] + mi * x[3 * i + 2];
        }
        double inv = 1.0 / ms;
        c[0] = c[0] * inv; c[1] = c[1] * inv; c[2] = c[2] * inv;
    }
    for (int d = 0; d < 3; ++d) out[3 * m + d] = wrap ? hf_wrap1(c[d], dyn->box[d]) : c[d];
}

// heat-flux z and molecule tag of every sorted slot (bit 31: molecule-based)
__global__ void k_hf_slots(const int* __restrict__ perm, int npad, const double* __restrict__ pos, HfDev h,
                           const DynState* __restrict__ dyn, double* __restrict__ zs, int* __restrict__ ms) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npad) return;
    int i = perm[s];
    if (i < 0) { zs[s] = 0.0; ms[s] = 0x7fffffff; return; }
    zs[s] = hf_z(h, pos, i, dyn->box[2]);
    ms[s] = h.mol_of[i] | (h.hftyp[i] == PGK_HFTYP_MOLE ? (int)0x80000000 : 0);
}

struct HfPairArgs {
    const int* clist; const int* ccnt; int ccap; int ncl;
    const int* typ_s; const int* perm; int ntyp;
    const double* zs; const int* ms;
    double rrcut, rr2, rl2, rmax2;
};

// calvirihf of one list pair: both atoms receive f_ij * fact (fact = sign(zi -
// zj) * frag / 2 per region); the cluster atom's share goes to its shared-
// memory accumulators wi[nreg][3], j's share to the global array (stride N).
// (pair categories ELIN, LJIN, ELC, VDW = PGK_HF_ELIN + 0..3)
template <typename T>
__device__ __forceinline__ void hf_pair_regions(T* wi, double* wj, size_t N, int nreg, const HfDev& h, double zi,
                                                double zj, double rz, double az, T fx, T fy, T fz) {
    const double zlo = fmin(zi, zj), zhi = fmax(zi, zj);
    for (int r = 0; r < nreg; ++r) {
        if (zhi < h.z1[r] || zlo > h.z2[r]) continue;
        double frag;
        if (!hf_frag(zi, zj, h.z1[r], h.z2[r], az, frag)) continue;
        const T fact = (T)(rz >= 0.0 ? frag * 0.5 : -frag * 0.5);
        const T vx = fx * fact, vy = fy * fact, vz = fz * fact;
        atomicAdd(wi + 3 * r + 0, vx);
        atomicAdd(wi + 3 * r + 1, vy);
        atomicAdd(wi + 3 * r + 2, vz);
        atomicAdd(wj + (3 * r + 0) * N, (double)vx);
        atomicAdd(wj + (3 * r + 1) * N, (double)vy);
        atomicAdd(wj + (3 * r + 2) * N, (double)vz);
    }
}

template <bool MIXED>
__global__ void __launch_bounds__(128) k_hf_pair(const int4* __restrict__ xq, const double4* __restrict__ xq64,
                                                 HfPairArgs a, const float2* __restrict__ lj32,
                                                 const double2* __restrict__ lj64, HfDev h,
                                                 const DynState* __restrict__ dyn) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    extern __shared__ __align__(16) unsigned char hf_sm[];
    const int nreg = h.nreg;
    const int per = 4 + 12 * nreg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* acc = (T*)hf_sm + (size_t)warp * 8 * per;
    for (int q = lane; q < 8 * per; q += 32) acc[q] = (T)0;
    const double Lz = dyn->box[2], invLz = 1.0 / Lz;
    const double L0 = dyn->box[0], L1 = dyn->box[1];
    const double B0 = 1.0 / L0, B1 = 1.0 / L1, B2 = 1.0 / Lz;
    const T sx = (T)(L0 * (1.0 / 4294967296.0)), sy = (T)(L1 * (1.0 / 4294967296.0)), sz = (T)(Lz * (1.0 / 4294967296.0));
    const T rr2 = (T)a.rr2, rl2 = (T)a.rl2, rmax2 = (T)a.rmax2;
    const size_t N = (size_t)h.natom;
    __syncwarp();
    for (int cl = blockIdx.x * 4 + warp; cl < a.ncl; cl += gridDim.x * 4) {
        const int cnt = a.ccnt[cl];
        const int* row = a.clist + (size_t)cl * a.ccap;
        for (int k = lane; k < cnt; k += 32) {
            const unsigned e = (unsigned)row[k];
            const int j = (int)(e & 0xFFFFFFu);
            const unsigned m = e >> 24;
            const double zj = a.zs[j];
            const int mj = a.ms[j];
            const int tj = a.typ_s[j];
            const int oj = a.perm[j];
            int4 qj = make_int4(0, 0, 0, 0);
            double4 pj = make_double4(0, 0, 0, 0);
            if (MIXED) qj = xq[j]; else pj = xq64[j];
            for (int ii = 0; ii < 8; ++ii) {
                if (!((m >> ii) & 1u)) continue;
                const int s = 8 * cl + ii;
                T dx, dy, dz, qq;
                if (MIXED) {
                    const int4 qi = xq[s];
                    dx = (T)(qi.x - qj.x) * sx; dy = (T)(qi.y - qj.y) * sy; dz = (T)(qi.z - qj.z) * sz;
                    qq = (T)(__int_as_float(qi.w) * __int_as_float(qj.w));
                } else {
                    const double4 pi = xq64[s];
                    double vx = pi.x - pj.x, vy = pi.y - pj.y, vz = pi.z - pj.z;
                    dx = (T)(vx - L0 * round(vx * B0));
                    dy = (T)(vy - L1 * round(vy * B1));
                    dz = (T)(vz - Lz * round(vz * B2));
                    qq = (T)(pi.w * pj.w);
                }
                const T r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > rmax2) continue;
                const T rinv2 = (T)1 / r2;
                const int mi = a.ms[s];
                const bool same = (mi & 0x7fffffff) == (mj & 0x7fffffff);
                const double zi = a.zs[s];
                const double rz = zi - zj, az = fabs(rz);
                const bool vir = !((mi < 0) && (mj < 0) && same) && az * invLz < 0.5;
                T* w = acc + ii * per;
                const bool coul = MIXED ? (r2 <= rr2) : (sqrt((double)r2) <= a.rrcut);
                if (coul) {                           // ewaldr_hf.F90:336-371, bare 1/r
                    const T rinv1 = (T)1 / sqrt(r2);
                    const T phi = qq * rinv1;
                    const T ft = phi * rinv2;
                    const int cat = same ? 0 : 2;
                    atomicAdd(w + cat, (T)0.5 * phi);
                    atomicAdd(h.pot + (PGK_HF_ELIN + cat) * N + oj, (double)((T)0.5 * phi));
                    if (vir) hf_pair_regions<T>(w + 4 + cat * 3 * nreg, h.W + (size_t)(PGK_HF_ELIN + cat) * nreg * 3 * N + oj,
                                                N, nreg, h, zi, zj, rz, az, ft * dx, ft * dy, ft * dz);
                }
                if (r2 <= rl2) {                      // ewaldr_hf.F90:376-470
                    T R2, E;
                    if (MIXED) { const float2 lp = lj32[a.typ_s[s] * a.ntyp + tj]; R2 = lp.x; E = lp.y; }
                    else { const double2 lp = lj64[a.typ_s[s] * a.ntyp + tj]; R2 = lp.x; E = lp.y; }
                    const T t2 = rinv2 * R2, t6 = t2 * t2 * t2, t12 = t6 * t6;
                    const T phi = E * (t12 - (T)2 * t6);
                    const T ft = (T)12 * E * (t12 - t6) * rinv2;
                    const int cat = same ? 1 : 3;
                    atomicAdd(w + cat, (T)0.5 * phi);
                    atomicAdd(h.pot + (PGK_HF_ELIN + cat) * N + oj, (double)((T)0.5 * phi));
                    if (vir) hf_pair_regions<T>(w + 4 + cat * 3 * nreg, h.W + (size_t)(PGK_HF_ELIN + cat) * nreg * 3 * N + oj,
                                                N, nreg, h, zi, zj, rz, az, ft * dx, ft * dy, ft * dz);
                }
            }
        }
        __syncwarp();
        for (int q = lane; q < 8 * per; q += 32) {
            const int ii = q / per, w = q - ii * per;
            const T v = acc[q];
            acc[q] = (T)0;
            const int io = a.perm[8 * cl + ii];
            if (io < 0 || v == (T)0) continue;
            if (w < 4) {
                atomicAdd(h.pot + (size_t)(PGK_HF_ELIN + w) * N + io, (double)v);
            } else {
                const int u = w - 4, cat = u / (3 * nreg), rem = u - cat * 3 * nreg;
                atomicAdd(h.W + ((size_t)(PGK_HF_ELIN + cat) * nreg * 3 + rem) * N + io, (double)v);
            }
        }
        __syncwarp();
    }
}

// ---- calheatf.F90, volume-based, z components --------------------------------
// per block: [nreg][17] partial sums (kinetic, 8 potential, 8 virial terms)
__global__ void __launch_bounds__(256) k_heatf_part(const double* __restrict__ pos, const double* __restrict__ vel,
                                                    const double* __restrict__ mass, const double* __restrict__ molevel,
                                                    HfDev h, const DynState* __restrict__ dyn,
                                                    double* __restrict__ part) {
    extern __shared__ double hs[];
    const int nreg = h.nreg, nv = nreg * 17;
    for (int q = threadIdx.x; q < nv; q += blockDim.x) hs[q] = 0.0;
    __syncthreads();
    const size_t N = (size_t)h.natom;
    const double Lz = dyn->box[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < h.natom; i += gridDim.x * blockDim.x) {
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        double pz, pvz;
        if (h.hftyp[i] == PGK_HFTYP_MOLE) { pz = h.molecom[3 * h.mol_of[i] + 2]; pvz = molevel[3 * h.mol_of[i] + 2]; }
        else { pz = pos[3 * i + 2]; pvz = vz; }
        pz = hf_wrap1(pz, Lz);
        const double kin = 0.5 * mass[i] * (vx * vx + vy * vy + vz * vz);
        for (int r = 0; r < nreg; ++r) {
            double* o = hs + r * 17;
            if (h.z1[r] <= pz && pz <= h.z2[r]) {
                atomicAdd(o, kin * pvz);
#pragma unroll
                for (int c = 0; c < 8; ++c) atomicAdd(o + 1 + c, h.pot[c * N + i] * pvz);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const double* w = h.W + ((size_t)c * nreg + r) * 3 * N;
                const double t = w[i] * vx + w[N + i] * vy + w[2 * N + i] * vz;
                if (t != 0.0) atomicAdd(o + 9 + c, t);
            }
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nv; q += blockDim.x) part[(size_t)blockIdx.x * nv + q] = hs[q];
}

// fixed-order sum of the block partials, volume normalisation, hftot
__global__ void k_heatf_final(const double* __restrict__ part, int nblk, int nreg, HfDev h,
                              const DynState* __restrict__ dyn, double* __restrict__ rec) {
    const int r = threadIdx.x;
    if (r >= nreg) return;
    double s[17];
    for (int c = 0; c < 17; ++c) s[c] = 0.0;
    for (int b = 0; b < nblk; ++b)
        for (int c = 0; c < 17; ++c) s[c] += part[((size_t)b * nreg + r) * 17 + c];
    const double area_inv = (1.0 / dyn->box[0]) * (1.0 / dyn->box[1]);
    const double vol_inv = area_inv / (h.z2[r] - h.z1[r]);
    double tot = 0.0;
    for (int c = 0; c < 17; ++c) { s[c] = s[c] * vol_inv; tot += s[c]; rec[r * PGK_HF_NCOL + c] = s[c]; }
    rec[r * PGK_HF_NCOL + 17] = tot;
}

// ---- region Langevin thermostat ----------------------------------------------
struct LtDev {
    int nlt;
    double x1[PGK_LT_MAX_REGIONS], x2[PGK_LT_MAX_REGIONS], y1[PGK_LT_MAX_REGIONS], y2[PGK_LT_MAX_REGIONS];
    double z1[PGK_LT_MAX_REGIONS], z2[PGK_LT_MAX_REGIONS], temp[PGK_LT_MAX_REGIONS], damp[PGK_LT_MAX_REGIONS];
    unsigned long long seed;
};

__device__ __forceinline__ bool lt_in(double lo, double hi, double x, double L) {
    return (lo <= x && x < hi) || (lo <= x - L && x - L < hi);
}
__device__ __forceinline__ int lt_region(const LtDev& l, const double* g, const double* box) {
    for (int r = 0; r < l.nlt; ++r)
        if (lt_in(l.x1[r], l.x2[r], g[0], box[0]) && lt_in(l.y1[r], l.y2[r], g[1], box[1]) &&
            lt_in(l.z1[r], l.z2[r], g[2], box[2]))
            return r;
    return -1;
}

// langevin_regist.F90:86-360 (one thread per molecule)
__global__ void k_lt_regist(const double* __restrict__ pos, const double* __restrict__ mass,
                            const int* __restrict__ mol_idx, const int* __restrict__ mol_list, int nmole,
                            const int* __restrict__ lt_mole, LtDev l, const DynState* __restrict__ dyn,
                            int* __restrict__ reg) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmole) return;
    const int b = mol_idx[m], e = mol_idx[m + 1];
    const double* box = dyn->box;
    if (lt_mole[m] && e - b > 1) {
        double ms = 0.0, g[3] = {0.0, 0.0, 0.0};
        for (int q = b; q < e; ++q) {
            int i = mol_list[q];
            ms = ms + mass[i];
            for (int d = 0; d < 3; ++d) g[d] = g[d] + mass[i] * pos[3 * i + d];
        }
        for (int d = 0; d < 3; ++d) g[d] = hf_wrap1(g[d] / ms, box[d]);
        const int r = lt_region(l, g, box);
        for (int q = b; q < e; ++q) reg[mol_list[q]] = r;
    } else {
        for (int q = b; q < e; ++q) {
            int i = mol_list[q];
            double g[3];
            for (int d = 0; d < 3; ++d) g[d] = hf_wrap1(pos[3 * i + d], box[d]);
            reg[i] = lt_region(l, g, box);
        }
    }
}

// langevin_region.F90:88-180: former half draws the random accelerations
// (Box-Muller as the reference), kick then friction; latter half friction
// then kick with the stored accelerations.  dekin (if non-null) collects
// sum m v^2 per region before (slot r) and after (slot 8 + r).
__global__ void k_langevin(double* __restrict__ vel, const double* __restrict__ mass, int n,
                           const int* __restrict__ reg, double* __restrict__ frand, LtDev l, double dt,
                           long long step, int former, double* __restrict__ dekin) {
    __shared__ double ek[2 * PGK_LT_MAX_REGIONS];
    if (dekin) {
        for (int q = threadIdx.x; q < 2 * PGK_LT_MAX_REGIONS; q += blockDim.x) ek[q] = 0.0;
        __syncthreads();
    }
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = i < n ? reg[i] : -1;
    if (i < n && former) {
        double f[3] = {0.0, 0.0, 0.0};
        if (r >= 0) {
            const double var = 2.0 * l.damp[r] * l.temp[r] / dt * mass[i];
            double u[4];
            lt_draw(l.seed, step, i, u);
            const double twopi = 2.0 * 3.14159265358979323846;
            const double a = sqrt(-2.0 * log(u[0]) * var);
            f[0] = a * cos(twopi * u[1]) / mass[i];
            f[1] = a * sin(twopi * u[1]) / mass[i];
            f[2] = sqrt(-2.0 * log(u[2]) * var) * cos(twopi * u[3]) / mass[i];
        }
        frand[3 * i] = f[0]; frand[3 * i + 1] = f[1]; frand[3 * i + 2] = f[2];
    }
    if (r >= 0) {
        double* v = vel + 3 * i;
        const double m = mass[i];
        if (dekin) atomicAdd(&ek[r], m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        const double ex = exp(-0.5 * dt * l.damp[r]);
        for (int d = 0; d < 3; ++d) {
            if (former) { v[d] = v[d] + 0.5 * dt * frand[3 * i + d]; v[d] = v[d] * ex; }
            else { v[d] = v[d] * ex; v[d] = v[d] + 0.5 * dt * frand[3 * i + d]; }
        }
        if (dekin) atomicAdd(&ek[PGK_LT_MAX_REGIONS + r], m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
    if (dekin) {
        __syncthreads();
        for (int q = threadIdx.x; q < l.nlt; q += blockDim.x)
            atomicAdd(&dekin[q], 0.5 * (ek[PGK_LT_MAX_REGIONS + q] - ek[q]));
    }
}

// ---- host side -----------------------------------------------------------------
static HfDev hf_dev(pgk_ctx* c) {
    HfDev h;
    h.nreg = c->hfp.nhfregion;
    h.natom = c->natom;
    for (int r = 0; r < PGK_HF_MAX_REGIONS; ++r) { h.z1[r] = c->hfp.hfzpos1[r]; h.z2[r] = c->hfp.hfzpos2[r]; }
    h.hftyp = c->hftyp; h.mol_of = c->mol_of; h.molecom = c->molecom;
    h.pot = c->hf_pot; h.W = c->hf_W;
    return h;
}
static LtDev lt_dev(const pgk_ctx* c) {
    LtDev l;
    const pgk_hfparams& p = c->hfp;
    l.nlt = p.nlangeregion;
    for (int r = 0; r < PGK_LT_MAX_REGIONS; ++r) {
        l.x1[r] = p.ltxpos1[r]; l.x2[r] = p.ltxpos2[r]; l.y1[r] = p.ltypos1[r]; l.y2[r] = p.ltypos2[r];
        l.z1[r] = p.ltzpos1[r]; l.z2[r] = p.ltzpos2[r]; l.temp[r] = p.r_ltemp[r]; l.damp[r] = p.r_ltdamp[r];
    }
    l.seed = p.seed;
    return l;
}

template <typename T>
static pgk_status upload_vec(pgk_ctx* c, T** dst, const std::vector<T>& v) {
    if (*dst) { pgk_dfree(c, *dst); *dst = nullptr; }
    if (v.empty()) return PGK_OK;
    PGK_CUDA(c, pgk_dmalloc(c, dst, sizeof(T) * v.size()));
    PGK_CUDA(c, cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->st));
    return PGK_OK;
}

pgk_status hf_setup(pgk_ctx* c, const pgk_hfparams* p) {
    if (p->nhfregion < 0 || p->nhfregion > PGK_HF_MAX_REGIONS || p->nlangeregion < 0 ||
        p->nlangeregion > PGK_LT_MAX_REGIONS)
        return pgk_fail(c, PGK_E_INVALID, "region count out of range");
    if (p->nhfregion > 0 && p->ifhfvol != 1)
        return pgk_fail(c, PGK_E_UNSUPPORTED, "only the local volume-based heat flux (ifhfvol) is built");
    for (int r = 0; r < p->nhfregion; ++r)
        if (!(p->hfzpos2[r] > p->hfzpos1[r])) return pgk_fail(c, PGK_E_INVALID, "hfzpos2 must exceed hfzpos1");
    pgk_status s;
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    int n = c->natom;
    c->hfp = *p;
    c->hfp.hftyp_atm = nullptr;
    c->hfp.lt_mole_based = nullptr;
    if (c->hfp.heatfinterval < 1) c->hfp.heatfinterval = 1;
    std::vector<int> molidx(c->nmole + 1), mollist, molof(n, 0), hftyp(n, PGK_HFTYP_ATOM), ltm(c->nmole, 0);
    if (c->nmole > 0) {
        PGK_CUDA(c, cudaMemcpy(molidx.data(), c->mol_idx, sizeof(int) * (c->nmole + 1), cudaMemcpyDeviceToHost));
        mollist.resize(molidx[c->nmole]);
        PGK_CUDA(c, cudaMemcpy(mollist.data(), c->mol_list, sizeof(int) * mollist.size(), cudaMemcpyDeviceToHost));
    }
    for (int m = 0; m < c->nmole; ++m)
        for (int q = molidx[m]; q < molidx[m + 1]; ++q) molof[mollist[q]] = m;
    if (p->hftyp_atm)
        for (int i = 0; i < n; ++i) {
            if (p->hftyp_atm[i] != PGK_HFTYP_ATOM && p->hftyp_atm[i] != PGK_HFTYP_MOLE)
                return pgk_fail(c, PGK_E_INVALID, "hftyp_atm must be 1 (atom) or 2 (molecule)");
            hftyp[i] = p->hftyp_atm[i];
        }
    if (p->lt_mole_based) for (int m = 0; m < c->nmole; ++m) ltm[m] = p->lt_mole_based[m] ? 1 : 0;
    if ((s = upload_vec(c, &c->mol_of, molof)) || (s = upload_vec(c, &c->hftyp, hftyp)) ||
        (s = upload_vec(c, &c->lt_mole, ltm)))
        return s;
    auto realloc = [&](double** b, size_t cnt) -> pgk_status {
        if (*b) { pgk_dfree(c, *b); *b = nullptr; }
        if (cnt == 0) return PGK_OK;
        if (pgk_dmalloc(c, b, cnt * sizeof(double)) != cudaSuccess) return pgk_fail(c, PGK_E_NOMEM, "heat-flux arrays");
        PGK_CUDA(c, cudaMemsetAsync(*b, 0, cnt * sizeof(double), c->st));
        return PGK_OK;
    };
    const int nreg = c->hfp.nhfregion;
    c->hf_nblk = 2 * c->nsm;
    if ((s = realloc(&c->molecom, (size_t)3 * std::max(1, c->nmole))) ||
        (s = realloc(&c->molevel, (size_t)3 * std::max(1, c->nmole))) ||
        (s = realloc(&c->hf_pot, (size_t)8 * n)) || (s = realloc(&c->hf_W, (size_t)8 * nreg * 3 * n)) ||
        (s = realloc(&c->hf_part, (size_t)c->hf_nblk * nreg * 17)) ||
        (s = realloc(&c->hf_rec, (size_t)std::max(1, nreg) * PGK_HF_NCOL)) ||   // one record
        (s = realloc(&c->lt_frand, (size_t)3 * n)) || (s = realloc(&c->lt_dekin, PGK_LT_MAX_REGIONS)))
        return s;
    c->hf_rec_cap = 1;
    if (c->lt_reg) pgk_dfree(c, c->lt_reg);
    c->lt_reg = nullptr;
    PGK_CUDA(c, pgk_dmalloc(c, &c->lt_reg, sizeof(int) * n));
    PGK_CUDA(c, cudaMemsetAsync(c->lt_reg, 0xff, sizeof(int) * n, c->st));
    c->hf_set = true;
    if (c->hfp.nlangeregion > 0 && (s = launch_lt_regist(c))) return s;
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return PGK_OK;
}

static pgk_status ensure_hf_slots(pgk_ctx* c) {
    if (c->hf_slots_cap >= c->npad_cap) return PGK_OK;
    pgk_dfree(c, c->hf_zs); pgk_dfree(c, c->hf_ms);
    c->hf_zs = nullptr; c->hf_ms = nullptr;
    PGK_CUDA(c, pgk_dmalloc(c, &c->hf_zs, sizeof(double) * c->npad_cap));
    PGK_CUDA(c, pgk_dmalloc(c, &c->hf_ms, sizeof(int) * c->npad_cap));
    c->hf_slots_cap = c->npad_cap;
    return PGK_OK;
}

// calforce_hf's per-atom quantities at the current positions (list and the
// pair kernel's packed coordinates must be current)
// Per-atom reciprocal terms of the bulk heat flux (pgk_set_hf_kspace) into
// the intermolecular Coulomb category: each atom's energy, and the (a, z)
// column of its tensor into region 1 -- ewaldk_hf.F90:212-230 writes
// virielct_atm(:, :, i, 1), the single region of the bulk builds.
__global__ void k_hf_kspace_add(const double* __restrict__ pot, const double* __restrict__ vir, int n, int nreg,
                                double* __restrict__ hf_pot, double* __restrict__ hf_W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    hf_pot[(size_t)PGK_HF_ELC * n + i] += pot[i];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        hf_W[((size_t)PGK_HF_ELC * nreg * 3 + a) * n + i] += vir[(size_t)9 * i + a + 6];
}

pgk_status launch_hf_kspace(pgk_ctx* c) {
    const int n = c->natom;
    const double* pot = nullptr;
    if (c->hf_kspace == PGK_HF_KSPACE_SPME) {
        pgk_status s = launch_spme_hf_atm(c);
        if (s) return s;
        pot = c->hfk_out;
    } else if (c->hf_kspace == PGK_HF_KSPACE_EWK) {
        if (!c->hf_ewk_fresh) {       // not yet evaluated at these positions by the force evaluation
            int nw = 0;
            pgk_status s = launch_ewk_hf(c, c->hf_kmax, &nw);
            if (s) return s;
        }
        pot = c->ewk_out + 3 * (size_t)n;
    }
    c->hf_ewk_fresh = false;
    if (!pot) return PGK_OK;
    k_hf_kspace_add<<<(n + 255) / 256, 256, 0, c->st>>>(pot, pot + n, n, c->hfp.nhfregion, c->hf_pot, c->hf_W);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_hf_atm(pgk_ctx* c) {
    if (!c->hf_set || c->hfp.nhfregion < 1) return pgk_fail(c, PGK_E_INVALID, "no heat-flux regions set");
    pgk_status s;
    const int n = c->natom, nreg = c->hfp.nhfregion;
    if (c->nmole > 0) {
        k_calcom<<<(c->nmole + 127) / 128, 128, 0, c->st>>>(c->pos, c->mass, c->mol_idx, c->mol_list, c->nmole,
                                                             c->dyn, 1, c->molecom);
        PGK_LAUNCHED(c);
    }
    PGK_CUDA(c, cudaMemsetAsync(c->hf_pot, 0, sizeof(double) * 8 * n, c->st));
    PGK_CUDA(c, cudaMemsetAsync(c->hf_W, 0, sizeof(double) * 8 * nreg * 3 * (size_t)n, c->st));
    HfDev h = hf_dev(c);
    const bool pair_on = c->prm.mts_vdw == PGK_MTS_LONG || c->prm.mts_vdw == PGK_MTS_SHORT;
    if (pair_on && c->ncl > 0) {
        if ((s = ensure_hf_slots(c))) return s;
        k_hf_slots<<<(c->npad + 255) / 256, 256, 0, c->st>>>(c->perm, c->npad, c->pos, h, c->dyn, c->hf_zs,
                                                              c->hf_ms);
        PGK_LAUNCHED(c);
        HfPairArgs a;
        a.clist = c->clist; a.ccnt = c->ccnt; a.ccap = c->ccap; a.ncl = c->ncl;
        a.typ_s = c->typ_s; a.perm = c->perm; a.ntyp = c->ntyp;
        a.zs = c->hf_zs; a.ms = c->hf_ms;
        a.rrcut = c->prm.rrcut;
        a.rr2 = c->prm.rrcut * c->prm.rrcut;
        a.rl2 = c->prm.rcut * c->prm.rcut;
        a.rmax2 = std::max(a.rr2, a.rl2);
        const int per = 4 + 12 * nreg;
        int blocks = std::min((c->ncl + 3) / 4, c->nsm * 8);
        if (c->mixed()) {
            size_t sm = (size_t)4 * 8 * per * sizeof(float);
            smem_limit(k_hf_pair<true>, sm);
            k_hf_pair<true><<<blocks, 128, sm, c->st>>>(c->xq, nullptr, a, c->lj32, c->lj64, h, c->dyn);
        } else {
            size_t sm = (size_t)4 * 8 * per * sizeof(double);
            smem_limit(k_hf_pair<false>, sm);
            k_hf_pair<false><<<blocks, 128, sm, c->st>>>(nullptr, c->xq64, a, c->lj32, c->lj64, h, c->dyn);
        }
        PGK_LAUNCHED(c);
        PGK_CUDA(c, cudaGetLastError());
    }
    if ((s = launch_bonded_hf(c, h))) return s;
    return launch_hf_kspace(c);
}

// calheatf with the current velocities: one record of nreg * 18 at dst (device)
pgk_status launch_heatf(pgk_ctx* c, double* dst) {
    const int nreg = c->hfp.nhfregion;
    if (c->nmole > 0) {
        k_calcom<<<(c->nmole + 127) / 128, 128, 0, c->st>>>(c->vel, c->mass, c->mol_idx, c->mol_list, c->nmole,
                                                             c->dyn, 0, c->molevel);
        PGK_LAUNCHED(c);
    }
    HfDev h = hf_dev(c);
    size_t sm = sizeof(double) * nreg * 17;
    k_heatf_part<<<c->hf_nblk, 256, sm, c->st>>>(c->pos, c->vel, c->mass, c->molevel, h, c->dyn, c->hf_part);
    k_heatf_final<<<1, 32, 0, c->st>>>(c->hf_part, c->hf_nblk, nreg, h, c->dyn, dst);
    c->launches += 2;
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_lt_regist(pgk_ctx* c) {
    if (c->nmole <= 0) return PGK_OK;
    k_lt_regist<<<(c->nmole + 127) / 128, 128, 0, c->st>>>(c->pos, c->mass, c->mol_idx, c->mol_list, c->nmole,
                                                            c->lt_mole, lt_dev(c), c->dyn, c->lt_reg);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_langevin(pgk_ctx* c, double dt, long long step, bool former) {
    const int n = c->natom;
    k_langevin<<<(n + 255) / 256, 256, 0, c->st>>>(c->vel, c->mass, n, c->lt_reg, c->lt_frand, lt_dev(c), dt, step,
                                                    former ? 1 : 0, c->hfp.ifoutthc ? c->lt_dekin : nullptr);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}
