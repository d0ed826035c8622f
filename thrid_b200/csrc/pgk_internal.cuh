// pgk_internal.cuh -- device-side data layout and helpers of libpgkgpu.so.
//
// Layout in HBM (all arrays owned by pgk_ctx, original atom order unless
// stated):
//   pos   double[3N]   AoS (x,y,z per atom), reference atmcor(3,natom)
//   vel   double[3N]   reference atmvel
//   facc  8-byte[2][3N] force accumulators of the MTS groups (0 long, 1 short):
//                       int64 fixed point (scale 2^32) in mixed precision,
//                       double in FP64 precision
//   acc   int64[2][NACC] energy / virial / kinetic accumulators (fixed 2^32)
//   sorted copies for the pair kernel (cell order, each cell padded to a
//     multiple of 8 slots): perm[npad] (slot -> original atom, -1 padding),
//     xq (int4: fractional fixed-point x,y,z + float bits of q, mixed) or
//     xq64 (double4: x,y,z,q, FP64), typ_s[npad]
//   clist int32[ncl*ccap] rows of 8-atom clusters, entries (mask << 24 | j),
//     ccnt[ncl]
//   heat flux: pot[8][N], W[8][nreg][3][N] (k_heatf.cu)
//   SPME  qacc (8-byte[K3*K2*K1]) + qc (complex[K3*K2*K1])
//   dyn   DynState      box and integrator coefficients read by every kernel,
//                       so that a whole MD step can be captured in a CUDA graph
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pgk_gpu.h"

#define PGK_FORCE_SCALE 4294967296.0          // 2^32
#define PGK_FORCE_ISCALE (1.0 / 4294967296.0)
#define PGK_GRID_SCALE 1099511627776.0         // 2^40 for the SPME charge grid
#define PGK_GRID_ISCALE (1.0 / 1099511627776.0)

// indices into one accumulator block (acc[group][..])
enum AccIdx {
    A_VDW = 0, A_ELC, A_EWK, A_BOND, A_ANGL, A_TORS, A_TORSRB, A_VDW14, A_ELC14,
    A_VC,                 // pot_viri_coul (scalar)
    A_VLJ,                // pot_viri_lj  (scalar)
    A_VTC,                // pot_virit_coul, 9
    A_VTLJ = A_VTC + 9,   // pot_virit_lj, 9
    A_VB = A_VTLJ + 9, A_VA, A_VT, A_V14,            // atm_viri_bond/angl/tors/14
    A_VTB, A_VTA = A_VTB + 9, A_VTT = A_VTA + 9, A_VT14 = A_VTT + 9,
    A_VSCA = A_VT14 + 9,  // vir_sca of scalar_sum
    A_KE,                 // sum m v^2
    A_KET,                // sum m v_a v_b, 9
    A_MOR = A_KET + 9,    // pot_mor (morsep)
    A_VMOR,               // pot_viri_mor
    A_VTMOR,              // pot_virit_mor, 9
    NACC = A_VTMOR + 9
};

// status bits (device sticky word)
#define ST_LIST_OVERFLOW   (1u << 0)
#define ST_CELL_OVERFLOW   (1u << 1)
#define ST_RATTLE_NOCONV   (1u << 2)
#define ST_BOX_TOO_SMALL   (1u << 3)
#define ST_RATTLEV_NOCONV  (1u << 4)
#define ST_UNSUPPORTED     (1u << 5)

// Pruned pair list state (mixed precision): the pair kernel reads a copy of
// the book list whose masks keep only pairs inside rprune = cutoff + buffer
// at the last prune.  dmax tracks the largest atom displacement since then
// (float bits, atomicMax); the list is re-pruned before a pair evaluation
// when 2*dmax plus the box-scaling term reaches the buffer, or when the book
// list was rebuilt (force), so no pair of the book list that comes inside
// the cutoff is ever missing from the pruned list.
struct PruneDev {
    unsigned dmax;
    int force;
    int do_prune;
    int pad;
    double box[3];                // box at the last prune
    unsigned long long nprune;    // prunes done (diagnostic)
};

struct DynState {
    double box[3], boxinv[3];
    double rkcut;
    // kick / drift coefficients (written by the chain kernels or the host)
    double kl_s[3], kl_b[3];      // long kick: v = v*kl_s + aL*kl_b
    double ks_b;                  // short kick: v += aS*ks_b
    double dr_a[3], dr_b[3];      // drift: x = x*dr_a + v*dr_b
    double rvinv[3];              // RATTLE(C) velocity divisor (rattle_cmtk rv/rvv)
    double yratio, zratio;
    int    ncell[3];              // cell counts of the current list build
    double cellsize[3];
    int    list_mode_used;
    long long nlistnball;         // reference-format count of the last build
    int    nmaxrow;               // longest cluster row of the last build (entries)
};

struct ChainDev {                 // device mirror of pgk_chain + derived
    double xlogs[8], vlogs[8];
    double xlogv, vlogv;
    double xboxh[3], vboxg[3];
    double pint, pintt[9];
};

// ---- small device helpers ------------------------------------------------
__device__ __forceinline__ long long to_fix(double v, double scale) {
    return __double2ll_rn(v * scale);
}
__device__ __forceinline__ void acc_fix(long long* p, double v, double scale = PGK_FORCE_SCALE) {
    atomicAdd((unsigned long long*)p, (unsigned long long)to_fix(v, scale));
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Energy / virial / kinetic accumulators: int64 fixed point (2^32) in mixed
// precision (order-independent, deterministic), IEEE double in FP64 precision
// (the slot's 8 bytes hold a double).
__device__ __forceinline__ void acc_add(long long* p, double x, bool dbl) {
    if (dbl) atomicAdd((double*)p, x);
    else acc_fix(p, x);
}
__device__ __forceinline__ double acc_get(const long long* acc, int k, bool dbl) {
    return dbl ? __longlong_as_double(acc[k]) : (double)acc[k] * PGK_FORCE_ISCALE;
}

// Block reduction of NV doubles; thread 0 adds the block total into
// acc[idx[k]].  blockDim.x must be a multiple of 32 (<=1024).
template <int NV>
__device__ __forceinline__ void block_acc(double (&v)[NV], long long* acc, const int (&idx)[NV], bool dbl) {
    __shared__ double red[32][NV];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) red[w][k] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? red[lane][k] : 0.0;
            x = warp_sum(x);
            if (lane == 0 && x != 0.0) acc_add(&acc[idx[k]], x, dbl);
        }
    }
}

// Force accumulation into the group buffer: fixed point (mixed) or double.
template <bool MIXED>
__device__ __forceinline__ void force_add(void* facc, int a, double fx, double fy, double fz) {
    if (MIXED) {
        long long* f = (long long*)facc + 3 * (size_t)a;
        acc_fix(f + 0, fx); acc_fix(f + 1, fy); acc_fix(f + 2, fz);
    } else {
        double* f = (double*)facc + 3 * (size_t)a;
        atomicAdd(f + 0, fx); atomicAdd(f + 1, fy); atomicAdd(f + 2, fz);
    }
}
template <bool MIXED>
__device__ __forceinline__ double force_get(const void* facc, size_t k) {
    if (MIXED) return (double)((const long long*)facc)[k] * PGK_FORCE_ISCALE;
    return ((const double*)facc)[k];
}

// Sort bin of a cluster-row entry's 8-bit mask (a dense rank 0..255).  The
// pair kernel evaluates the cluster atoms as four pairs (bits 2p, 2p+1), and a
// warp runs a pair's evaluation when any of its 32 lanes has a bit in it; so
// entries are grouped first by which of the four pairs are occupied (groups in
// inverse-Gray-code order of that 4-bit occupancy: neighbouring groups differ
// in one pair), and inside a group by the occupied pairs' states taken as a
// mixed-radix-3 number (bits 01 -> 0, 11 -> 1, 10 -> 2).  Group g starts at
// the sum of 3^popcount over the groups before it: offsets 0, 1, 4, 13, 16, 25,
// 52, 61, 64, 73, 100, 181, 208, 217, 244, 253, packed eight to a word below.
__device__ __forceinline__ unsigned mask_bin(unsigned m) {
    unsigned occ = 0, w = 0, mul = 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const unsigned b = (m >> (2 * q)) & 3u;
        if (b) {
            occ |= 1u << q;
            w += (b == 1u ? 0u : (b == 3u ? 1u : 2u)) * mul;
            mul *= 3u;
        }
    }
    occ ^= occ >> 1;
    occ ^= occ >> 2;
    occ &= 0xFu;
    const unsigned long long off = occ < 8u ? 0x3d3419100d040100ull : 0xfdf4d9d0b5644940ull;
    return (unsigned)((off >> (8u * (occ & 7u))) & 0xFFull) + w;
}

// Fortran dnint/anint (round half away from zero), exact FP64 min image
// exclusive prefix sum of 256 shared-memory bins by one warp (8 bins a lane)
__device__ __forceinline__ void warp_scan256(int* bin, int lane) {
    int v[8], t = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) { v[q] = bin[8 * lane + q]; t += v[q]; }
    int incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    int run = incl - t;
#pragma unroll
    for (int q = 0; q < 8; ++q) { bin[8 * lane + q] = run; run += v[q]; }
}

__device__ __forceinline__ double mi_exact(double r, double box, double binv) {
    return __dsub_rn(r, __dmul_rn(box, round(__dmul_rn(r, binv))));
}
