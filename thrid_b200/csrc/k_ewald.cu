// k_ewald.cu -- ewaldkp_hf (ewaldk_hf.F90:8-304): the standard-Ewald k-space
// force, energy and virial with the per-atom split that the bulk heat flux
// (-D_HF_BULK_EWK) uses, FP64 throughout.
//
// For K = (nx/Lx, ny/Ly, nz/Lz) the phase exp(2 pi i K.r) factorises over the
// axes, so no (atom, wave) needs its own sine and cosine:
//   k_ewk_tab    exp(2 pi i n r_d / L_d) per atom for n = 0..nmax_d (negative
//                n by conjugation)
//   k_ewk_sfac   partial structure factors sum_i q_i exp(2 pi i K.r_i) over
//                atom chunks: waves across threads, the chunk's table rows in
//                shared memory, two complex products per (atom, wave)
//   k_ewk_coef   chunk sums in a fixed order, the per-wave coefficients, block
//                partials of the energy and virial-tensor sums
//   k_ewk_atom   thread per atom over a segment of the waves in the
//                reference's order: one complex product per wave inside a run
//                of consecutive nz, force, energy and virial tensor of the
//                atom in registers; k_ewk_atom_sum adds the segments
//   k_ewk_final  fixed-order sum of the block partials
// Every sum runs in a fixed order: results are run-to-run identical.

#include <algorithm>
#include <cmath>
#include <vector>

#include "pgk_ctx.cuh"

#define EWK_TA 32         // atoms per shared-memory tile of k_ewk_sfac
#define EWK_KPT 4         // waves per thread of k_ewk_sfac
#define EWK_SB 128        // threads of k_ewk_sfac and k_ewk_coef
#define EWK_CT 64         // waves per shared-memory tile of k_ewk_atom
#define EWK_NCOEF 12      // K(3), A(K) bsk, A(K) bck, fac_vir3, g K_a K_b (xx yy zz xy xz yz)
#define EWK_MAX_ROWS 253  // table rows (sum of nmax_d + 1)

struct EwkArgs {
    double alpha, netchrgsq;
    int cc;                       // ifnetqcorrp
    int nmax0, nmax1;             // table row offsets: y rows start at nmax0+1, z rows at nmax0+nmax1+2
    int nrow;
};

// exp(2 pi i n r_d / L_d) as (cos, sin), row = axis block + n, [row][N]
__global__ void k_ewk_tab(const double* __restrict__ pos, int n, EwkArgs a, const DynState* __restrict__ dyn,
                          double2* __restrict__ tab) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)a.nrow * n) return;
    const int row = (int)(t / n), i = (int)(t - (long long)row * n);
    int d, m;
    if (row <= a.nmax0) { d = 0; m = row; }
    else if (row <= a.nmax0 + a.nmax1 + 1) { d = 1; m = row - a.nmax0 - 1; }
    else { d = 2; m = row - a.nmax0 - a.nmax1 - 2; }
    const double u = pos[3 * i + d] / dyn->box[d];
    double s, c;
    sincospi(2.0 * (double)m * u, &s, &c);
    tab[t] = make_double2(c, s);
}

// (x, y, z) rows of a wave and the conjugation signs of negative n
struct EwkIdx { int ix, iy, iz; double sx, sy, sz; };
__device__ __forceinline__ EwkIdx ewk_idx(int4 v, const EwkArgs& a) {
    EwkIdx r;
    r.ix = abs(v.x); r.iy = a.nmax0 + 1 + abs(v.y); r.iz = a.nmax0 + a.nmax1 + 2 + abs(v.z);
    r.sx = v.x < 0 ? -1.0 : 1.0; r.sy = v.y < 0 ? -1.0 : 1.0; r.sz = v.z < 0 ? -1.0 : 1.0;
    return r;
}
// exp(2 pi i K.r) from one atom's table rows
__device__ __forceinline__ double2 ewk_phase(const double2* __restrict__ rows, const EwkIdx& w) {
    const double2 X = rows[w.ix], Y = rows[w.iy], Z = rows[w.iz];
    const double xi = X.y * w.sx, yi = Y.y * w.sy, zi = Z.y * w.sz;
    const double pr = X.x * Y.x - xi * yi, pi = X.x * yi + xi * Y.x;
    return make_double2(pr * Z.x - pi * zi, pr * zi + pi * Z.x);
}

// part[chunk][w] = sum over the chunk's atoms of q (cos, sin)(2 pi K_w.r)
__global__ void __launch_bounds__(EWK_SB) k_ewk_sfac(const double2* __restrict__ tab, const double* __restrict__ q,
                                                     int n, int chunk, const int4* __restrict__ nv, int nwave,
                                                     EwkArgs a, double2* __restrict__ part) {
    extern __shared__ double2 ewk_sm[];
    const int nrp = a.nrow | 1;   // odd row stride: the transposed tile stores are conflict-free
    double2* rows = ewk_sm;       // [EWK_TA][nrp]
    double* sq = (double*)(ewk_sm + EWK_TA * nrp);
    const int a0 = blockIdx.y * chunk, a1 = min(n, a0 + chunk);
    EwkIdx w[EWK_KPT];
    double re[EWK_KPT], im[EWK_KPT];
#pragma unroll
    for (int j = 0; j < EWK_KPT; ++j) {
        const int k = (blockIdx.x * EWK_KPT + j) * EWK_SB + threadIdx.x;
        w[j] = ewk_idx(k < nwave ? nv[k] : make_int4(0, 0, 0, 0), a);
        re[j] = 0.0; im[j] = 0.0;
    }
    for (int t0 = a0; t0 < a1; t0 += EWK_TA) {
        const int na = min(EWK_TA, a1 - t0);
        __syncthreads();
        for (int e = threadIdx.x; e < a.nrow * EWK_TA; e += EWK_SB) {
            const int row = e / EWK_TA, at = e - row * EWK_TA;
            rows[at * nrp + row] = at < na ? tab[(size_t)row * n + t0 + at] : make_double2(0.0, 0.0);
        }
        if (threadIdx.x < EWK_TA) sq[threadIdx.x] = (int)threadIdx.x < na ? q[t0 + threadIdx.x] : 0.0;
        __syncthreads();
        for (int at = 0; at < na; ++at) {
            const double2* r = rows + at * nrp;
            const double qa = sq[at];
#pragma unroll
            for (int j = 0; j < EWK_KPT; ++j) {
                const double2 e = ewk_phase(r, w[j]);
                re[j] = fma(qa, e.x, re[j]);
                im[j] = fma(qa, e.y, im[j]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < EWK_KPT; ++j) {
        const int k = (blockIdx.x * EWK_KPT + j) * EWK_SB + threadIdx.x;
        if (k < nwave) part[(size_t)blockIdx.y * nwave + k] = make_double2(re[j], im[j]);
    }
}

// Per wave: bck, bsk summed over the chunks in order; A(K) of prepewk.F90:137-144
// at the current box; coefficient row; energy and tensor terms of
// ewaldk_hf.F90:168-272 summed over the block (fixed order) into red[block][8]
__global__ void __launch_bounds__(EWK_SB) k_ewk_coef(const double2* __restrict__ part, int nchunk,
                                                     const int4* __restrict__ nv, int nwave, EwkArgs a,
                                                     const DynState* __restrict__ dyn, double* __restrict__ coef,
                                                     double* __restrict__ red) {
    const int k = blockIdx.x * EWK_SB + threadIdx.x;
    double v[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};   // pot, cc, t xx yy zz xy xz yz
    if (k < nwave) {
        double bck = 0.0, bsk = 0.0;
        for (int c = 0; c < nchunk; ++c) {
            const double2 p = part[(size_t)c * nwave + k];
            bck += p.x; bsk += p.y;
        }
        const double pi = 3.14159265358979323846;
        const double bx = dyn->box[0], by = dyn->box[1], bz = dyn->box[2];
        const int4 m = nv[k];
        const double K[3] = {(double)m.x / bx, (double)m.y / by, (double)m.z / bz};
        const double k2 = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
        const double pot_fact = 0.5 / pi / (bx * by * bz);
        const double fac_vir = 2.0 * pi * pi / (a.alpha * a.alpha);
        const double coeff = (pi / a.alpha) * (pi / a.alpha);
        const double aw = k == 0 ? 0.0 : exp(-coeff * k2) / k2;
        const double pfa = pot_fact * aw;
        const double poti = pfa * (bsk * bsk + bck * bck);
        double* cf = coef + (size_t)k * EWK_NCOEF;
        cf[0] = K[0]; cf[1] = K[1]; cf[2] = K[2];
        cf[3] = aw * bsk; cf[4] = aw * bck;
        v[0] = poti;
        double fac3 = 0.0, g = 0.0;
        if (k > 0) {   // ewaldk_hf.F90:186: no virial term for (0,0,0)
            g = 2.0 / k2 + fac_vir;
            if (a.cc) {
                fac3 = pfa * a.netchrgsq;
                v[1] = fac3 * (-1.0 + fac_vir * k2);
            }
            const double e = poti - fac3;
            v[2] = e * (1.0 - g * K[0] * K[0]); v[3] = e * (1.0 - g * K[1] * K[1]); v[4] = e * (1.0 - g * K[2] * K[2]);
            v[5] = -e * g * K[0] * K[1]; v[6] = -e * g * K[0] * K[2]; v[7] = -e * g * K[1] * K[2];
        }
        cf[5] = fac3;
        cf[6] = g * K[0] * K[0]; cf[7] = g * K[1] * K[1]; cf[8] = g * K[2] * K[2];
        cf[9] = g * K[0] * K[1]; cf[10] = g * K[0] * K[2]; cf[11] = g * K[1] * K[2];
    }
    __shared__ double sred[EWK_SB / 32][8];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const double s = warp_sum(v[t]);
        if (lane == 0) sred[wp][t] = s;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        for (int q = 0; q < EWK_SB / 32; ++q) s += sred[q][threadIdx.x];
        red[blockIdx.x * 8 + threadIdx.x] = s;
    }
}

// Thread per atom over waves 1..nwave-1: force (ewaldk_hf.F90:178-182,
// 280-288), energy with the self term (:165-173, :295-299) and virial tensor
// (:212-230, :255-272) of the atom.  Waves come in runs of consecutive nz at
// fixed (nx, ny) (nv[w].w = 1 opens a run): the phase is taken from sincospi
// at the start of a run and advanced by exp(2 pi i z / Lz) inside it, so the
// atom's state stays in registers.  out: force [3N] | energy [N] | tensor [9N].
// The wave loop is split into nseg segments (blockIdx.y), so that small
// systems still fill the SMs; a segment starts its phase from sincospi like a
// run.  With nseg > 1 each segment writes its 11 sums to seg[(s*11+k)*N + i]
// and k_ewk_atom_sum adds them in segment order (fixed: run-to-run identical).
__device__ __forceinline__ void ewk_atom_out(int i, int n, double qi, double pq, double vol, double alpha,
                                             const double (&r)[11], double* __restrict__ out) {
    const double pi = 3.14159265358979323846;
    const double f2 = 2.0 * qi / vol;
    out[3 * (size_t)i] = f2 * r[0]; out[3 * (size_t)i + 1] = f2 * r[1]; out[3 * (size_t)i + 2] = f2 * r[2];
    out[3 * (size_t)n + i] = pq * r[3] - alpha / sqrt(pi) * (qi * qi);
    const double E = r[4], txx = r[5], tyy = r[6], tzz = r[7], txy = r[8], txz = r[9], tyz = r[10];
    double* v = out + 4 * (size_t)n + 9 * (size_t)i;
    v[0] = E - txx; v[1] = -txy; v[2] = -txz;
    v[3] = -txy; v[4] = E - tyy; v[5] = -tyz;
    v[6] = -txz; v[7] = -tyz; v[8] = E - tzz;
}

__global__ void __launch_bounds__(128) k_ewk_atom(const double* __restrict__ pos, const double* __restrict__ q,
                                                  int n, const int4* __restrict__ nv, const double* __restrict__ coef,
                                                  int nwave, EwkArgs a, const DynState* __restrict__ dyn,
                                                  double* __restrict__ out, int nseg, double* __restrict__ seg) {
    __shared__ double scf[EWK_CT * EWK_NCOEF];
    __shared__ int4 snv[EWK_CT];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const double bx = dyn->box[0], by = dyn->box[1], bz = dyn->box[2];
    const double ux = live ? pos[3 * (size_t)i] / bx : 0.0;
    const double uy = live ? pos[3 * (size_t)i + 1] / by : 0.0;
    const double uz = live ? pos[3 * (size_t)i + 2] / bz : 0.0;
    double zs, zc;
    sincospi(2.0 * uz, &zs, &zc);
    const double pi = 3.14159265358979323846;
    const double vol = bx * by * bz;
    const double pot_fact = 0.5 / pi / vol;
    const double qi = live ? q[i] : 0.0, pq = pot_fact * qi;
    double pc = 1.0, ps_ = 0.0;                                // phase (cos, sin)
    double fx = 0.0, fy = 0.0, fz = 0.0, ps = 0.0, E = 0.0;
    double txx = 0.0, tyy = 0.0, tzz = 0.0, txy = 0.0, txz = 0.0, tyz = 0.0;
    const int sgi = blockIdx.y;
    const int wb = 1 + (int)((long long)(nwave - 1) * sgi / nseg);
    const int we = 1 + (int)((long long)(nwave - 1) * (sgi + 1) / nseg);
    for (int w0 = wb; w0 < we; w0 += EWK_CT) {
        const int cnt = min(EWK_CT, we - w0);
        __syncthreads();
        for (int e = threadIdx.x; e < cnt * EWK_NCOEF; e += blockDim.x) scf[e] = coef[(size_t)w0 * EWK_NCOEF + e];
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) snv[e] = nv[w0 + e];
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            const double* cf = scf + j * EWK_NCOEF;
            const int4 v = snv[j];
            if (v.w || w0 + j == wb) {
                sincospi(2.0 * ((double)v.x * ux + (double)v.y * uy + (double)v.z * uz), &ps_, &pc);
            } else {
                const double c2 = pc * zc - ps_ * zs;
                ps_ = pc * zs + ps_ * zc;
                pc = c2;
            }
            const double t1 = ps_ * cf[3] + pc * cf[4];        // A (sin bsk + cos bck)
            const double t2 = ps_ * cf[4] - pc * cf[3];        // A (bck sin - bsk cos)
            fx = fma(t2, cf[0], fx); fy = fma(t2, cf[1], fy); fz = fma(t2, cf[2], fz);
            ps += t1;
            const double e = fma(pq, t1, -cf[5]);              // fac_vir2 - fac_vir3
            E += e;
            txx = fma(e, cf[6], txx); tyy = fma(e, cf[7], tyy); tzz = fma(e, cf[8], tzz);
            txy = fma(e, cf[9], txy); txz = fma(e, cf[10], txz); tyz = fma(e, cf[11], tyz);
        }
    }
    if (!live) return;
    const double r[11] = {fx, fy, fz, ps, E, txx, tyy, tzz, txy, txz, tyz};
    if (nseg == 1) {
        ewk_atom_out(i, n, qi, pq, vol, a.alpha, r, out);
        return;
    }
#pragma unroll
    for (int k = 0; k < 11; ++k) seg[((size_t)sgi * 11 + k) * n + i] = r[k];
}

__global__ void k_ewk_atom_sum(const double* __restrict__ q, int n, int nseg, const double* __restrict__ seg,
                               EwkArgs a, const DynState* __restrict__ dyn, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) r[k] = 0.0;
    for (int sg = 0; sg < nseg; ++sg)
#pragma unroll
        for (int k = 0; k < 11; ++k) r[k] += seg[((size_t)sg * 11 + k) * n + i];
    const double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    const double qi = q[i], pq = 0.5 / 3.14159265358979323846 / vol * qi;
    ewk_atom_out(i, n, qi, pq, vol, a.alpha, r, out);
}

// scalars: pot_ewk, pot_ewk_cc, pot_virit_coul[a + 3b]
__global__ void k_ewk_final(const double* __restrict__ red, int nblk, double* __restrict__ out) {
    __shared__ double s[8];
    if (threadIdx.x < 8) {
        double t = 0.0;
        for (int b = 0; b < nblk; ++b) t += red[b * 8 + threadIdx.x];
        s[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = s[0]; out[1] = s[1];
        double* t = out + 2;
        t[0] = s[2]; t[4] = s[3]; t[8] = s[4];
        t[1] = t[3] = s[5]; t[2] = t[6] = s[6]; t[5] = t[7] = s[7];
    }
}

// prepewk.F90:100-135: integer waves in the reference's loop order, (0,0,0) first
static int ewk_waves(int kmax, int ny0, int nz0, std::vector<int4>& nv) {
    const int yk = kmax * ny0, zk = kmax * nz0;
    nv.assign(1, make_int4(0, 0, 0, 0));
    for (int kx = -kmax; kx <= kmax; ++kx)
        for (int ky = -yk; ky <= yk; ++ky)
            for (int kz = -zk; kz <= zk; ++kz) {
                if (kx == 0 && ky == 0 && kz == 0) continue;
                const double a2 = (double)(kx * kx) + (double)(ky * ky) / (double)(ny0 * ny0) +
                                  (double)(kz * kz) / (double)(nz0 * nz0);
                if (a2 <= (double)(kmax * kmax)) nv.push_back(make_int4(kx, ky, kz, 0));
            }
    // .w = 1 where a run of consecutive nz at fixed (nx, ny) starts
    for (size_t w = 1; w < nv.size(); ++w) {
        const int4 p = nv[w - 1], v = nv[w];
        nv[w].w = (w == 1 || v.x != p.x || v.y != p.y || v.z != p.z + 1) ? 1 : 0;
    }
    return (int)nv.size();
}

static pgk_status ewk_buf(pgk_ctx* c, void** p, size_t& have, size_t want) {
    if (have >= want) return PGK_OK;
    if (*p) pgk_dfree(c, *p);
    *p = nullptr;
    have = 0;
    PGK_CUDA(c, pgk_dmalloc(c, p, want));
    have = want;
    return PGK_OK;
}

pgk_status launch_ewk_hf(pgk_ctx* c, int kmax, int* nwave_out, int only) {
    const int n = c->natom;
    if (kmax < 1 || n < 1) return pgk_fail(c, PGK_E_INVALID, "ewaldkp_hf: kmax < 1 or no atoms");
    const int ny0 = (int)std::round(c->prm.ycel / c->prm.xcel), nz0 = (int)std::round(c->prm.zcel / c->prm.xcel);
    if (ny0 < 1 || nz0 < 1) return pgk_fail(c, PGK_E_INVALID, "ewaldkp_hf: anint(ycel/xcel) or anint(zcel/xcel) is 0");
    if ((long long)kmax * (1 + ny0 + nz0) + 3 > EWK_MAX_ROWS)
        return pgk_fail(c, PGK_E_INVALID, "ewaldkp_hf: kmax too large (kmax*(1+ny0+nz0) > 250)");
    if (c->ewk_kmax != kmax) {
        std::vector<int4> nv;
        const int nw = ewk_waves(kmax, ny0, nz0, nv);
        {
            if (c->ewk_nv) pgk_dfree(c, c->ewk_nv);
            c->ewk_nv = nullptr;
            c->ewk_kmax = 0;
            PGK_CUDA(c, pgk_dmalloc(c, &c->ewk_nv, sizeof(int4) * nw));
        }
        PGK_CUDA(c, cudaMemcpyAsync(c->ewk_nv, nv.data(), sizeof(int4) * nw, cudaMemcpyHostToDevice, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        c->ewk_nwave = nw;
        c->ewk_nmax[0] = kmax; c->ewk_nmax[1] = kmax * ny0; c->ewk_nmax[2] = kmax * nz0;
        c->ewk_kmax = kmax;
    }
    const int nwave = c->ewk_nwave;
    EwkArgs a;
    a.alpha = c->prm.alpha; a.netchrgsq = c->netchrgsq; a.cc = c->prm.ifnetqcorrp != 0;
    a.nmax0 = c->ewk_nmax[0]; a.nmax1 = c->ewk_nmax[1];
    a.nrow = c->ewk_nmax[0] + c->ewk_nmax[1] + c->ewk_nmax[2] + 3;
    const int nrp = a.nrow | 1;

    // structure-factor grid: waves in blocks of EWK_SB * EWK_KPT, atoms in
    // chunks so that about four blocks run per SM
    const int nkb = (nwave + EWK_SB * EWK_KPT - 1) / (EWK_SB * EWK_KPT);
    const int ntile = (n + EWK_TA - 1) / EWK_TA;
    int nchunk = std::max(1, std::min(ntile, (4 * c->nsm + nkb - 1) / nkb));
    const int chunk = (ntile + nchunk - 1) / nchunk * EWK_TA;
    nchunk = (n + chunk - 1) / chunk;
    const int ncb = (nwave + EWK_SB - 1) / EWK_SB;

    pgk_status s;
    if ((s = ewk_buf(c, (void**)&c->ewk_tab, c->ewk_bytes[0], sizeof(double2) * a.nrow * (size_t)n)) ||
        (s = ewk_buf(c, (void**)&c->ewk_part, c->ewk_bytes[1], sizeof(double2) * nchunk * (size_t)nwave)) ||
        (s = ewk_buf(c, (void**)&c->ewk_coef, c->ewk_bytes[2], sizeof(double) * EWK_NCOEF * (size_t)nwave)) ||
        (s = ewk_buf(c, (void**)&c->ewk_red, c->ewk_bytes[3], sizeof(double) * 8 * (size_t)ncb)) ||
        (s = ewk_buf(c, (void**)&c->ewk_out, c->ewk_bytes[4], sizeof(double) * (13 * (size_t)n + 11))))
        return s;
    // wave segments of the per-atom kernel: about four blocks of 128 per SM
    const int nab = (n + 127) / 128;
    const int nseg = std::max(1, std::min(16, std::min((4 * c->nsm + nab - 1) / nab, nwave - 1)));
    if (nseg > 1 && (s = ewk_buf(c, (void**)&c->ewk_seg, c->ewk_bytes[5], sizeof(double) * 11 * (size_t)nseg * n)))
        return s;
    auto atom_kernels = [&]() {
        k_ewk_atom<<<dim3(nab, nseg), 128, 0, c->st>>>(c->pos, c->chrg, n, c->ewk_nv, c->ewk_coef, nwave, a, c->dyn,
                                                      c->ewk_out, nseg, c->ewk_seg);
        PGK_LAUNCHED(c);
        if (nseg > 1) {
            k_ewk_atom_sum<<<(n + 255) / 256, 256, 0, c->st>>>(c->chrg, n, nseg, c->ewk_seg, a, c->dyn, c->ewk_out);
            PGK_LAUNCHED(c);
        }
    };

    const size_t sm_sfac = sizeof(double2) * EWK_TA * nrp + sizeof(double) * EWK_TA;
    PGK_CUDA(c, smem_limit(k_ewk_sfac, sm_sfac));

    if (only && c->ewk_kmax == kmax && c->ewk_bytes[4] > 0) {   // one kernel on the last call's buffers
        if (only == 1)
            k_ewk_sfac<<<dim3(nkb, nchunk), EWK_SB, sm_sfac, c->st>>>(c->ewk_tab, c->chrg, n, chunk, c->ewk_nv, nwave,
                                                                        a, c->ewk_part);
        else
            atom_kernels();
        if (only == 1) PGK_LAUNCHED(c);
        PGK_CUDA(c, cudaGetLastError());
        if (nwave_out) *nwave_out = nwave;
        return PGK_OK;
    }
    const long long ntab = (long long)a.nrow * n;
    k_ewk_tab<<<(unsigned)((ntab + 255) / 256), 256, 0, c->st>>>(c->pos, n, a, c->dyn, c->ewk_tab);
    PGK_LAUNCHED(c);
    k_ewk_sfac<<<dim3(nkb, nchunk), EWK_SB, sm_sfac, c->st>>>(c->ewk_tab, c->chrg, n, chunk, c->ewk_nv, nwave, a,
                                                                c->ewk_part);
    PGK_LAUNCHED(c);
    k_ewk_coef<<<ncb, EWK_SB, 0, c->st>>>(c->ewk_part, nchunk, c->ewk_nv, nwave, a, c->dyn, c->ewk_coef, c->ewk_red);
    PGK_LAUNCHED(c);
    atom_kernels();
    k_ewk_final<<<1, 32, 0, c->st>>>(c->ewk_red, ncb, c->ewk_out + 13 * (size_t)n);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    if (nwave_out) *nwave_out = nwave;
    return PGK_OK;
}

// _HF_BULK_EWK heat-flux step (calforce_hf.F90:1046-1062): ewaldkp_hf's force
// into group g's accumulator in place of the SPME reciprocal force, pot_ewk,
// pot_viri_coul += pot_ewk + pot_ewk_cc (ewaldk_hf.F90:290) and the tensor
// (symmetric; the accumulator keeps the lower triangle)
template <bool MIXED>
__global__ void k_ewk_force_add(const double* __restrict__ out, int n, void* __restrict__ facc,
                                long long* __restrict__ acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * n) {
        if (MIXED) atomicAdd((unsigned long long*)facc + t, (unsigned long long)to_fix(out[t], PGK_FORCE_SCALE));
        else atomicAdd((double*)facc + t, out[t]);
    }
    if (t == 0) {
        const double* sc = out + 13 * (size_t)n;
        acc_add(&acc[A_EWK], sc[0], !MIXED);
        acc_add(&acc[A_VC], sc[0] + sc[1], !MIXED);
        const int lo[6] = {0, 1, 2, 4, 5, 8};
        for (int k = 0; k < 6; ++k) acc_add(&acc[A_VTC + lo[k]], sc[2 + lo[k]], !MIXED);
    }
}

pgk_status launch_ewk_force(pgk_ctx* c, int group) {
    int nw = 0;
    pgk_status s = launch_ewk_hf(c, c->hf_kmax, &nw);
    if (s) return s;
    const int n = c->natom;
    long long* acc = c->acc + (size_t)group * NACC;
    if (c->mixed()) k_ewk_force_add<true><<<(3 * n + 255) / 256, 256, 0, c->st>>>(c->ewk_out, n, c->facc[group], acc);
    else k_ewk_force_add<false><<<(3 * n + 255) / 256, 256, 0, c->st>>>(c->ewk_out, n, c->facc[group], acc);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    c->hf_ewk_fresh = true;
    return PGK_OK;
}
