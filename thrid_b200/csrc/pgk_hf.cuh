// pgk_hf.cuh -- device helpers of the heat-flux path (calvirihf.F90) and the
// counter-based random stream of the region Langevin thermostat.
#pragma once

#include "pgk_internal.cuh"

// Pair categories of the per-atom arrays, in the order of PGK_HF_* (pgk_gpu.h).
struct HfDev {
    int nreg, natom;
    double z1[PGK_HF_MAX_REGIONS], z2[PGK_HF_MAX_REGIONS];
    const int* hftyp;        // [N] PGK_HFTYP_*
    const int* mol_of;       // [N] molecule of each atom
    const double* molecom;   // [3*nmole] calcom.F90 centres (wrapped)
    double* pot;             // [8][N] pot_*_atm
    double* W;               // [8][nreg][3][N] viri*_atm(a,3,i,r)
};

// single-shift periodic wrap used throughout the heat-flux code
__device__ __forceinline__ double hf_wrap1(double x, double L) {
    if (x < 0.0) return x + L;
    if (x >= L) return x - L;
    return x;
}

// heat-flux z of atom i: atom (wrapped) or its molecule's centre of mass
__device__ __forceinline__ double hf_z(const HfDev& h, const double* __restrict__ pos, int i, double Lz) {
    return h.hftyp[i] == PGK_HFTYP_MOLE ? h.molecom[3 * h.mol_of[i] + 2] : hf_wrap1(pos[3 * i + 2], Lz);
}

// z length of the segment (zi, zj) inside slab [z1, z2] by the plane-crossing
// cases of calvirihf.F90:214-300; false when the pair does not touch the slab
__device__ __forceinline__ bool hf_frag(double zi, double zj, double z1, double z2, double az, double& frag) {
    const double p1i = zi - z1, p1j = zj - z1, p2i = zi - z2, p2j = zj - z2;
    const bool c1 = p1i * p1j < 0.0, c2 = p2i * p2j < 0.0;
    if (!c1 && !c2) {
        if (p1i * p2i > 0.0) return false;
        frag = az;
    } else if (c1 != c2) {
        if (c1) frag = p1i > 0.0 ? p1i : p1j;
        else frag = p2i < 0.0 ? -p2i : -p2j;
    } else {
        frag = z2 - z1;
    }
    return true;
}

// calvirihf for one (i, j) pair of a bonded term: viri(:,3,i,r) += fi * f,
// viri(:,3,j,r) += -fj * f (FP64 atomics)
__device__ __forceinline__ void hf_calviri(const HfDev& h, const double* __restrict__ pos, double Lz, int i, int j,
                                           const double* fi, const double* fj, double nbc, int cat) {
    const bool mi = h.hftyp[i] == PGK_HFTYP_MOLE, mj = h.hftyp[j] == PGK_HFTYP_MOLE;
    if (mi && mj && h.mol_of[i] == h.mol_of[j]) return;
    const double zi = hf_z(h, pos, i, Lz), zj = hf_z(h, pos, j, Lz);
    const double rz = zi - zj, az = fabs(rz);
    if (az * (1.0 / Lz) >= 0.5) return;
    const double zlo = fmin(zi, zj), zhi = fmax(zi, zj);
    const size_t N = (size_t)h.natom;
    for (int r = 0; r < h.nreg; ++r) {
        if (zhi < h.z1[r] || zlo > h.z2[r]) continue;
        double frag;
        if (!hf_frag(zi, zj, h.z1[r], h.z2[r], az, frag)) continue;
        const double fact = rz >= 0.0 ? frag * nbc : -frag * nbc;
        double* w = h.W + ((size_t)cat * h.nreg + r) * 3 * N;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicAdd(w + a * N + i, fi[a] * fact);
            atomicAdd(w + a * N + j, (-fj[a]) * fact);
        }
    }
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011): counter (atom, step
// lo, step hi, draw), key = seed; two draws give four uniforms on (0, 1]
// with 53 random bits each.
__device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 1.0) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ void lt_draw(unsigned long long seed, long long step, int atom, double* u) {
#pragma unroll
    for (int call = 0; call < 2; ++call) {
        uint32_t c[4] = {(uint32_t)atom, (uint32_t)(unsigned long long)step,
                         (uint32_t)((unsigned long long)step >> 32), (uint32_t)call};
        philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        u[2 * call] = u53(c[0], c[1]);
        u[2 * call + 1] = u53(c[2], c[3]);
    }
}
