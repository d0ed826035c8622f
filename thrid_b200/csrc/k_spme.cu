// k_spme.cu -- smooth particle-mesh Ewald reciprocal space (fft_pmep,
// fft_pme.F90:144-937; fft_pme_init.F90:14-289; erf_corr_cutoff.F90).
//
//  k_spread   get_scaled_fractionals + get_bspline_coeffs + fill_charge_grid:
//             one thread per atom, p^3 atomic adds into the accumulation grid
//             (int64 fixed point 2^40 in mixed precision -> order-independent,
//             deterministic; double in FP64 precision).
//  k_fft      hand-written shared-memory pencil FFT (Stockham autosort,
//             radix 4/2/3/5), one launch per axis and direction; the first
//             forward pass reads the accumulation grid directly.  Replaces the
//             FFTPACK cfftf/cfftb passes of pubz3d (fft_pme.F90:809-869).
//  k_scalar   scalar_sum: influence function, energy, virial tensor, Q *= eterm.
//  k_gather   grad_sum: force from the convolved grid, p^3 loads per atom.
// Complex grid: float2 (mixed) or double2 (FP64), x fastest, K1*K2*K3.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "pgk_ctx.cuh"

// ---- B-spline weights: fill_bspline (fft_pme_init.F90:216-260) ---------------
template <typename T, int P>
__device__ __forceinline__ void fill_bspline_d(T w, T* arr, T* darr) {
    arr[P - 1] = 0;
    arr[1] = w;
    arr[0] = T(1) - w;
#pragma unroll
    for (int k = 3; k <= P - 1; ++k) {
        T div = T(1) / T(k - 1);
        arr[k - 1] = div * w * arr[k - 2];
#pragma unroll
        for (int j = 1; j <= k - 2; ++j)
            arr[k - j - 1] = div * ((w + T(j)) * arr[k - j - 2] + (T(k - j) - w) * arr[k - j - 1]);
        arr[0] = div * (T(1) - w) * arr[0];
    }
    darr[0] = -arr[0];
#pragma unroll
    for (int j = 2; j <= P; ++j) darr[j - 1] = arr[j - 2] - arr[j - 1];
    T div = T(1) / T(P - 1);
    arr[P - 1] = div * w * arr[P - 2];
#pragma unroll
    for (int j = 1; j <= P - 2; ++j)
        arr[P - j - 1] = div * ((w + T(j)) * arr[P - j - 2] + (T(P - j) - w) * arr[P - j - 1]);
    arr[0] = div * (T(1) - w) * arr[0];
}

// scaled fractional coordinate (get_scaled_fractionals) -> base index, w
__device__ __forceinline__ void frac_coord(double x, double recip, int K, int& base, double& w) {
    double f = x * recip;
    f = f - floor(f);
    double fr = (double)K * f;
    base = min(max((int)fr, 0), K - 1);     // in range even for non-finite coordinates
    w = fr - trunc(fr);
}

// order (may be NULL): atoms in cell-sorted order, so that neighbouring
// threads touch neighbouring grid points (L2 locality of the atomics)
template <bool MIXED, int P>
__global__ void k_spread(const double* __restrict__ pos, const double* __restrict__ chrg, int n,
                         const DynState* __restrict__ dyn, int K1, int K2, int K3, void* __restrict__ qacc,
                         const int* __restrict__ order) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int a = order ? order[t] : t;
    if (a < 0) return;   // padding slot of the cell-sorted order
    double th[3][P], dth[3][P];
    int base[3];
    const int Kd[3] = {K1, K2, K3};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double w;
        frac_coord(pos[3 * a + d], dyn->boxinv[d], Kd[d], base[d], w);
        fill_bspline_d<double, P>(w, th[d], dth[d]);
    }
    double q = chrg[a];
#pragma unroll
    for (int i3 = 0; i3 < P; ++i3) {
        int k = base[2] - P + 1 + i3;
        k = k < 0 ? k + K3 : k;
        double p1 = th[2][i3] * q;
#pragma unroll
        for (int i2 = 0; i2 < P; ++i2) {
            int j = base[1] - P + 1 + i2;
            j = j < 0 ? j + K2 : j;
            double p2 = th[1][i2] * p1;
            size_t row = (size_t)K1 * (j + (size_t)K2 * k);
#pragma unroll
            for (int i1 = 0; i1 < P; ++i1) {
                int i = base[0] - P + 1 + i1;
                i = i < 0 ? i + K1 : i;
                double v = th[0][i1] * p2;
                if (MIXED) atomicAdd((unsigned long long*)qacc + row + i,
                                     (unsigned long long)__double2ll_rn(v * PGK_GRID_SCALE));
                else atomicAdd((double*)qacc + row + i, v);
            }
        }
    }
}

// Row-cooperative spread (the path the engine runs): P lanes per atom, lane
// i1 adds the points (i1, i2, i3) of all (i2, i3), so each atomic instruction
// of a warp covers 32/P atoms x P consecutive grid points -- a few L2 sectors
// per instruction instead of one sector per lane.  Each contribution is the
// same product th0 * (th1 * (th2 * q)) as in k_spread, so the mixed grid
// (integer sums) is bit-identical to k_spread's.
template <bool MIXED, int P>
__global__ void __launch_bounds__(256) k_spread_rows(const double* __restrict__ pos, const double* __restrict__ chrg,
                                                     int n, const DynState* __restrict__ dyn, int K1, int K2, int K3,
                                                     void* __restrict__ qacc, const int* __restrict__ order) {
    constexpr int G = 32 / P;
    const int lane = threadIdx.x & 31;
    const int g = lane / P, i1 = lane - g * P;
    const int t = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * G + g;
    if (g >= G || t >= n) return;
    const int a = order ? order[t] : t;
    if (a < 0) return;   // padding slot of the cell-sorted order
    double th[3][P], dth[3][P];
    int base[3];
    const int Kd[3] = {K1, K2, K3};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double w;
        frac_coord(pos[3 * a + d], dyn->boxinv[d], Kd[d], base[d], w);
        fill_bspline_d<double, P>(w, th[d], dth[d]);
    }
    double t0 = 0.0;
#pragma unroll
    for (int q = 0; q < P; ++q) t0 = q == i1 ? th[0][q] : t0;
    const double q = chrg[a];
    int i = base[0] - P + 1 + i1; i = i < 0 ? i + K1 : i;
#pragma unroll
    for (int i3 = 0; i3 < P; ++i3) {
        int k = base[2] - P + 1 + i3; k = k < 0 ? k + K3 : k;
        const double p1 = th[2][i3] * q;
#pragma unroll
        for (int i2 = 0; i2 < P; ++i2) {
            int j = base[1] - P + 1 + i2; j = j < 0 ? j + K2 : j;
            const double v = t0 * (th[1][i2] * p1);
            const size_t at = (size_t)K1 * (j + (size_t)K2 * k) + i;
            if (MIXED) atomicAdd((unsigned long long*)qacc + at, (unsigned long long)__double2ll_rn(v * PGK_GRID_SCALE));
            else atomicAdd((double*)qacc + at, v);
        }
    }
}

// ---- FFT --------------------------------------------------------------------
template <typename T> struct C2;
template <> struct C2<float> { typedef float2 t; };
template <> struct C2<double> { typedef double2 t; };

template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { a.x += b.x; a.y += b.y; return a; }
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename T2, typename T> __device__ __forceinline__ T2 cscale(T2 a, T s) { a.x *= s; a.y *= s; return a; }
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    T2 r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename T2, typename T> __device__ __forceinline__ T2 mul_i(T2 a, T s) {   // (s*i) * a
    T2 r; r.x = -s * a.y; r.y = s * a.x; return r;
}

struct FftDev {
    int n, nstage;
    int radix[PGK_MAX_RADIX_STAGES];
    const void* tw;
};

template <typename T, typename T2>
__device__ __forceinline__ void dft_r(T2* v, int R, T sg) {
    if (R == 2) {
        T2 a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if (R == 4) {
        T2 a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
        T2 s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = csub(a1, a3);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        T2 t = mul_i<T2, T>(d13, sg);
        v[1] = cadd(d02, t);
        v[3] = csub(d02, t);
    } else if (R == 3) {
        const T s60 = T(0.86602540378443864676);
        T2 a0 = v[0], a1 = v[1], a2 = v[2];
        T2 t1 = cadd(a1, a2);
        T2 t2 = csub(a0, cscale<T2, T>(t1, T(0.5)));
        T2 t3 = mul_i<T2, T>(csub(a1, a2), sg * s60);
        v[0] = cadd(a0, t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    } else if (R == 5) {
        const T c72 = T(0.30901699437494742410), s72 = T(0.95105651629515357212);
        const T c144 = T(-0.80901699437494742410), s144 = T(0.58778525229247312917);
        T2 a0 = v[0];
        T2 b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
        T2 c1 = csub(v[1], v[4]), c2 = csub(v[2], v[3]);
        T2 t1 = cadd(a0, cadd(cscale<T2, T>(b1, c72), cscale<T2, T>(b2, c144)));
        T2 t2 = cadd(a0, cadd(cscale<T2, T>(b1, c144), cscale<T2, T>(b2, c72)));
        T2 u1 = cadd(cscale<T2, T>(c1, s72), cscale<T2, T>(c2, s144));
        T2 u2 = csub(cscale<T2, T>(c1, s144), cscale<T2, T>(c2, s72));
        T2 iu1 = mul_i<T2, T>(u1, sg), iu2 = mul_i<T2, T>(u2, sg);
        v[0] = cadd(a0, cadd(b1, b2));
        v[1] = cadd(t1, iu1);
        v[4] = csub(t1, iu1);
        v[2] = cadd(t2, iu2);
        v[3] = csub(t2, iu2);
    }
}

// radix chain of a length (4s first, then 2, 3, 5), usable at compile time
__host__ __device__ constexpr int pick_radix(int m) {
    return m % 4 == 0 ? 4 : (m % 2 == 0 ? 2 : (m % 3 == 0 ? 3 : (m % 5 == 0 ? 5 : 0)));
}
__host__ __device__ constexpr int stage_radix(int n, int s) {
    int m = n;
    for (int k = 0; k < s; ++k) m /= pick_radix(m);
    return pick_radix(m);
}
__host__ __device__ constexpr int stage_ns(int n, int s) {
    int m = n, ns = 1;
    for (int k = 0; k < s; ++k) { int r = pick_radix(m); ns *= r; m /= r; }
    return ns;
}
__host__ __device__ constexpr int nstages(int n) {
    int c = 0;
    while (n > 1) { n /= pick_radix(n); ++c; }
    return c;
}

// one Stockham stage on P pencils of length n held in shared memory
// pencils are stored with pitch ld = n + 1 elements, so that the strided
// loads and stores of the y and z passes (consecutive threads on consecutive
// pencils) fall into different shared-memory banks
template <typename T, typename T2>
__device__ __forceinline__ void fft_stage(const T2* __restrict__ src, T2* __restrict__ dst, int P, int n, int R,
                                          int Ns, const T2* __restrict__ tw, T sg) {
    const int ld = n + 1;
    const int nr = n / R;
    const int twstep = n / (Ns * R);
    for (int w = threadIdx.x; w < P * nr; w += blockDim.x) {
        int p = w / nr, j = w - p * nr;
        int k = j % Ns;
        T2 v[5];
        const T2* sp = src + p * ld;
#pragma unroll
        for (int r = 0; r < 5; ++r)
            if (r < R) {
                T2 x = sp[j + r * nr];
                if (r > 0 && k > 0) {
                    T2 t = tw[r * k * twstep];
                    if (sg > 0) t.y = -t.y;
                    x = cmul(x, t);
                }
                v[r] = x;
            }
        dft_r<T, T2>(v, R, sg);
        int o = (j / Ns) * Ns * R + k;
        T2* dp = dst + p * ld;
#pragma unroll
        for (int r = 0; r < 5; ++r)
            if (r < R) dp[o + r * Ns] = v[r];
    }
}

// all stages; NC > 0 makes the length and radix chain compile-time constants
template <typename T, typename T2, int NC, int S = 0>
struct FftStages {
    static __device__ __forceinline__ void run(T2*& src, T2*& dst, int P, int n, const FftDev& plan, T sg,
                                               const T2* tw) {
        if (NC == 0) {
            int Ns = 1;
            for (int s = 0; s < plan.nstage; ++s) {
                fft_stage<T, T2>(src, dst, P, n, plan.radix[s], Ns, tw, sg);
                __syncthreads();
                T2* t = src; src = dst; dst = t;
                Ns *= plan.radix[s];
            }
        } else if (S < nstages(NC)) {
            fft_stage<T, T2>(src, dst, P, NC, stage_radix(NC, S), stage_ns(NC, S), tw, sg);
            __syncthreads();
            T2* t = src; src = dst; dst = t;
            FftStages<T, T2, NC, (S < 12 ? S + 1 : S)>::run(src, dst, P, n, plan, sg, tw);
        }
    }
};
template <typename T, typename T2, int NC>
struct FftStages<T, T2, NC, 12> {
    static __device__ __forceinline__ void run(T2*&, T2*&, int, int, const FftDev&, T, const T2*) {}
};

// influence function of one grid point (scalar_sum, fft_pme.F90:590-680)
// K1f > 0: the grid holds the k1 = 0 .. K1f/2 half of the spectrum of a real
// grid of K1f x-points (real-to-complex x transform); the energy and virial
// sums then count every point with 0 < k1 < K1f/2 twice (it stands for k and
// its mirror -k, with the same |S|^2 and the same products h_a h_b).
struct ConvArgs {
    const double* bsp; double alpha, netchrgsq; int corr; long long* acc; int want; int K1f;
};

__device__ __forceinline__ double conv_point(int k1, int k2, int k3, int K1, int K2, int K3, double s2,
                                             const ConvArgs& ca, const DynState* __restrict__ dyn, double& en,
                                             double& vs, double* vt, double w = 1.0) {
    const double pi = 3.14159265358979323846;
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    int m1 = k1 < nf1 ? k1 : k1 - K1;
    int m2 = k2 < nf2 ? k2 : k2 - K2;
    int m3 = k3 < nf3 ? k3 : k3 - K3;
    double h1 = dyn->boxinv[0] * m1, h2 = dyn->boxinv[1] * m2, h3 = dyn->boxinv[2] * m3;
    double msq = h1 * h1 + h2 * h2 + h3 * h3;
    if (msq > dyn->rkcut * dyn->rkcut) return 0.0;
    const double fac = pi * pi / (ca.alpha * ca.alpha);
    const double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    double denom = pi * vol * ca.bsp[k1] * ca.bsp[K1 + k2] * ca.bsp[K1 + K2 + k3] * msq;
    double ex = exp(-fac * msq);
    double eterm = ex / denom;
    if (ca.want) {
        double vterm = 2.0 * (fac * msq + 1.0) / msq;
        double es = eterm * s2 * w;
        en += es;
        if (ca.corr) {
            double e2 = ex * ca.netchrgsq / (pi * vol * msq) * w;
            vs += e2 * (-1.0 + 2.0 * fac * msq);
            es -= e2;
        }
        vt[0] += es * (vterm * h1 * h1 - 1.0);
        vt[1] += es * (vterm * h1 * h2);
        vt[2] += es * (vterm * h1 * h3);
        vt[3] += es * (vterm * h2 * h2 - 1.0);
        vt[4] += es * (vterm * h2 * h3);
        vt[5] += es * (vterm * h3 * h3 - 1.0);
    }
    return eterm;
}

// The same influence function in FP32 (mixed precision; the grid itself is
// FP32 there): exp and divisions on the FP32 pipes, energy and virial sums
// still accumulated in FP64.
struct ConvF { float bi[3], rk2, fac, pivol; };

__device__ __forceinline__ float conv_point_f(int k1, int k2, int k3, int K1, int K2, int K3, float s2,
                                              const ConvArgs& ca, const ConvF& cf, double& en, double& vs,
                                              double* vt, float w = 1.f) {
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    const int m1 = k1 < nf1 ? k1 : k1 - K1;
    const int m2 = k2 < nf2 ? k2 : k2 - K2;
    const int m3 = k3 < nf3 ? k3 : k3 - K3;
    const float h1 = cf.bi[0] * (float)m1, h2 = cf.bi[1] * (float)m2, h3 = cf.bi[2] * (float)m3;
    const float msq = h1 * h1 + h2 * h2 + h3 * h3;
    if (msq > cf.rk2) return 0.f;
    const float denom = cf.pivol * (float)ca.bsp[k1] * (float)ca.bsp[K1 + k2] * (float)ca.bsp[K1 + K2 + k3] * msq;
    const float ex = expf(-cf.fac * msq);
    const float eterm = ex / denom;
    if (ca.want) {
        const float vterm = 2.f * (cf.fac * msq + 1.f) / msq;
        float es = eterm * s2 * w;
        en += (double)es;
        if (ca.corr) {
            const float e2 = ex * (float)ca.netchrgsq / (cf.pivol * msq) * w;
            vs += (double)(e2 * (-1.f + 2.f * cf.fac * msq));
            es -= e2;
        }
        vt[0] += (double)(es * (vterm * h1 * h1 - 1.f));
        vt[1] += (double)(es * (vterm * h1 * h2));
        vt[2] += (double)(es * (vterm * h1 * h3));
        vt[3] += (double)(es * (vterm * h2 * h2 - 1.f));
        vt[4] += (double)(es * (vterm * h2 * h3));
        vt[5] += (double)(es * (vterm * h3 * h3 - 1.f));
    }
    return eterm;
}

// AXIS 0: pencils along x (contiguous); 1: along y; 2: along z.
// SRC: 0 = complex grid in place, 1 = int64 fixed-point accumulation grid,
//      2 = double accumulation grid (both real, first forward pass),
//      3 = complex grid in, real part out to the real grid `acc` (last
//      backward pass; the gather reads only the real part).
// CONV (AXIS 2 only): forward z transform, influence function (scalar_sum)
//      and backward z transform in one pass over the grid.
template <typename T, int AXIS, int SRC, int NC, bool CONV>
__global__ void __launch_bounds__(256) k_fft(typename C2<T>::t* __restrict__ data, const void* __restrict__ acc,
                                             int K1, int K2, int K3, FftDev plan, int P, T sg, ConvArgs ca,
                                             const DynState* __restrict__ dyn) {
    typedef typename C2<T>::t T2;
    extern __shared__ unsigned char smraw[];
    T2* bufA = (T2*)smraw;
    const int n = NC > 0 ? NC : plan.n;
    const int ld = n + 1;                 // padded pencil pitch (bank-conflict free strided access)
    T2* bufB = bufA + P * ld;
    T2* tws = bufB + P * ld;              // twiddle table (n entries) staged in shared memory
    for (int k = threadIdx.x; k < n; k += blockDim.x) tws[k] = ((const T2*)plan.tw)[k];
    size_t base;
    size_t stride;
    int yz = 0;
    if (AXIS == 0) {
        base = (size_t)blockIdx.x * P * K1;
        stride = 1;
    } else if (AXIS == 1) {
        int nxb = (K1 + P - 1) / P;
        int z = blockIdx.x / nxb, x0 = (blockIdx.x % nxb) * P;
        base = (size_t)x0 + (size_t)K1 * K2 * z;
        stride = K1;
    } else {
        int nxb = (K1 + P - 1) / P;
        int y = blockIdx.x / nxb, x0 = (blockIdx.x % nxb) * P;
        base = (size_t)x0 + (size_t)K1 * y;
        stride = (size_t)K1 * K2;
        yz = y;
    }
    const int tot = P * n;
    const int npen_total = AXIS == 0 ? K2 * K3 : K1;
    const int x0 = AXIS == 0 ? 0 : (int)(base % K1);
    // load: each thread issues its first FFT_LQ loads before any shared store
    // (one memory latency per block instead of one per element)
    auto load_one = [&](int idx, T2& v) {
        int p, m;
        if (AXIS == 0) { p = idx / n; m = idx - p * n; } else { m = idx / P; p = idx - m * P; }
        const int pg = AXIS == 0 ? blockIdx.x * P + p : x0 + p;
        v.x = 0; v.y = 0;
        if (pg < npen_total) {
            const size_t off = AXIS == 0 ? base + (size_t)p * K1 + m : base + p + stride * m;
            if (SRC == 0 || SRC == 3) v = data[off];
            else if (SRC == 1) v.x = (T)((double)((const long long*)acc)[off] * PGK_GRID_ISCALE);
            else v.x = (T)((const double*)acc)[off];
        }
        return p * ld + m;
    };
    {
        constexpr int FFT_LQ = 8;
        T2 rv[FFT_LQ];
        int ri[FFT_LQ];
#pragma unroll
        for (int q = 0; q < FFT_LQ; ++q) {
            const int idx = threadIdx.x + q * blockDim.x;
            ri[q] = idx < tot ? load_one(idx, rv[q]) : -1;
        }
#pragma unroll
        for (int q = 0; q < FFT_LQ; ++q)
            if (ri[q] >= 0) bufA[ri[q]] = rv[q];
        for (int idx = threadIdx.x + FFT_LQ * blockDim.x; idx < tot; idx += blockDim.x) {
            T2 v;
            const int si = load_one(idx, v);
            bufA[si] = v;
        }
    }
    __syncthreads();
    T2* src = bufA;
    T2* dst = bufB;
    FftStages<T, T2, NC>::run(src, dst, P, n, plan, sg, tws);
    if (CONV) {
        double en = 0, vs = 0, vt[6] = {0, 0, 0, 0, 0, 0};
        ConvF cf;
        {
            const double pi = 3.14159265358979323846;
            for (int d = 0; d < 3; ++d) cf.bi[d] = (float)dyn->boxinv[d];
            cf.rk2 = (float)(dyn->rkcut * dyn->rkcut);
            cf.fac = (float)(pi * pi / (ca.alpha * ca.alpha));
            cf.pivol = (float)(pi * dyn->box[0] * dyn->box[1] * dyn->box[2]);
        }
        const int K1f = ca.K1f > 0 ? ca.K1f : K1;       // x points of the real grid
        for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
            int p = idx / n, m = idx - p * n;
            const int sidx = p * ld + m;
            int k1 = x0 + p;
            if (k1 >= K1) continue;
            if (k1 == 0 && yz == 0 && m == 0) continue;   // m = 0 is skipped by scalar_sum
            const int w = (ca.K1f > 0 && k1 > 0 && 2 * k1 != ca.K1f) ? 2 : 1;
            T2 v = src[sidx];
            if (sizeof(T) == 4) {
                const float et = conv_point_f(k1, yz, m, K1f, K2, K3, (float)v.x * (float)v.x + (float)v.y * (float)v.y,
                                              ca, cf, en, vs, vt, (float)w);
                v.x = (T)((float)v.x * et);
                v.y = (T)((float)v.y * et);
            } else {
                double s2 = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
                double et = conv_point(k1, yz, m, K1f, K2, K3, s2, ca, dyn, en, vs, vt, (double)w);
                v.x = (T)((double)v.x * et);
                v.y = (T)((double)v.y * et);
            }
            src[sidx] = v;
        }
        __syncthreads();
        FftStages<T, T2, NC>::run(src, dst, P, n, plan, -sg, tws);
        if (ca.want) {
            double out[9] = {0.5 * en, 0.5 * en + 0.5 * vs, 0.5 * vs,
                             -0.5 * vt[0], -0.5 * vt[1], -0.5 * vt[2], -0.5 * vt[3], -0.5 * vt[4], -0.5 * vt[5]};
            const int idx9[9] = {A_EWK, A_VC, A_VSCA, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5,
                                 A_VTC + 8};
            block_acc<9>(out, ca.acc, idx9, sizeof(T) == 8);
        }
    }
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        int p, m;
        if (AXIS == 0) { p = idx / n; m = idx - p * n; } else { m = idx / P; p = idx - m * P; }
        int pg = AXIS == 0 ? blockIdx.x * P + p : x0 + p;
        if (pg < npen_total) {
            size_t off = AXIS == 0 ? base + (size_t)p * K1 + m : base + p + stride * m;
            if (SRC == 3) ((T*)acc)[off] = src[p * ld + m].x;     // real part only (what the gather reads)
            else data[off] = src[p * ld + m];
        }
    }
}

// Real-to-complex x pass (FWD) and its complex-to-real inverse, on x lines of
// a real grid of K1 = 2N points.  Forward: the line's even and odd points are
// taken as one complex sequence z_n = x_2n + i x_2n+1 (n < N), transformed by
// the length-N pencil FFT (exp(-2 pi i nk/N)), and split:
//   E_k = (Z_k + conj Z_{N-k}) / 2,  O_k = (Z_k - conj Z_{N-k}) / 2i,
//   X_k = E_k + exp(-2 pi i k / K1) O_k,  k = 0..N,
// the k1 = 0..K1/2 half of the line's spectrum (the other half is its complex
// conjugate mirror), stored with pitch N + 1.  Inverse (unnormalised,
// exp(+2 pi i)): from a Hermitian half spectrum Y_0..Y_N,
//   A_k = Y_k + conj Y_{N-k},  B_k = (Y_k - conj Y_{N-k}) exp(+2 pi i k / K1),
//   z = length-N inverse FFT of A + iB,  y_2n = Re z_n,  y_2n+1 = Im z_n,
// written to the real grid that the gather reads.  SRC (forward): 1 = int64
// fixed-point accumulation grid, 2 = double accumulation grid.
template <typename T, int SRC, int NC, bool FWD>
__global__ void __launch_bounds__(256) k_fft_rx(typename C2<T>::t* __restrict__ data, void* __restrict__ real,
                                                int K1, int nline, FftDev plan, const void* __restrict__ tw2g,
                                                int P) {
    typedef typename C2<T>::t T2;
    extern __shared__ unsigned char smraw[];
    const int N = NC > 0 ? NC : plan.n;
    const int ld = N + 1;
    const int K1h = N + 1;
    T2* bufA = (T2*)smraw;
    T2* bufB = bufA + P * ld;
    T2* tws = bufB + P * ld;              // length-N twiddles
    T2* tw2 = tws + N;                    // exp(-2 pi i k / K1), k = 0..N
    for (int k = threadIdx.x; k < N; k += blockDim.x) tws[k] = ((const T2*)plan.tw)[k];
    for (int k = threadIdx.x; k <= N; k += blockDim.x) tw2[k] = ((const T2*)tw2g)[k];
    const int line0 = blockIdx.x * P;
    if (FWD) {
        for (int idx = threadIdx.x; idx < P * N; idx += blockDim.x) {
            const int p = idx / N, m = idx - p * N;
            T2 v; v.x = 0; v.y = 0;
            if (line0 + p < nline) {
                const size_t off = (size_t)(line0 + p) * K1 + 2 * m;
                if (SRC == 1) {
                    const longlong2 q = *(const longlong2*)((const long long*)real + off);
                    v.x = (T)((double)q.x * PGK_GRID_ISCALE);
                    v.y = (T)((double)q.y * PGK_GRID_ISCALE);
                } else {
                    const double2 q = *(const double2*)((const double*)real + off);
                    v.x = (T)q.x;
                    v.y = (T)q.y;
                }
            }
            bufA[p * ld + m] = v;
        }
        __syncthreads();
        T2* src = bufA;
        T2* dst = bufB;
        FftStages<T, T2, NC>::run(src, dst, P, N, plan, T(-1), tws);
        for (int idx = threadIdx.x; idx < P * K1h; idx += blockDim.x) {
            const int p = idx / K1h, k = idx - p * K1h;
            if (line0 + p >= nline) continue;
            const T2 zk = src[p * ld + (k == N ? 0 : k)];
            T2 zc = src[p * ld + (k == 0 ? 0 : N - k)];
            zc.y = -zc.y;
            const T2 e = cscale<T2, T>(cadd(zk, zc), T(0.5));
            const T2 d = csub(zk, zc);
            T2 o; o.x = T(0.5) * d.y; o.y = T(-0.5) * d.x;        // d / 2i
            data[(size_t)(line0 + p) * K1h + k] = cadd(e, cmul(tw2[k], o));
        }
    } else {
        for (int idx = threadIdx.x; idx < P * K1h; idx += blockDim.x) {
            const int p = idx / K1h, k = idx - p * K1h;
            T2 v; v.x = 0; v.y = 0;
            if (line0 + p < nline) v = data[(size_t)(line0 + p) * K1h + k];
            bufB[p * ld + k] = v;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < P * N; idx += blockDim.x) {
            const int p = idx / N, k = idx - p * N;
            const T2 yk = bufB[p * ld + k];
            T2 yc = bufB[p * ld + N - k];
            yc.y = -yc.y;
            const T2 a = cadd(yk, yc);
            T2 t = tw2[k];
            t.y = -t.y;                                           // exp(+2 pi i k / K1)
            const T2 b = cmul(csub(yk, yc), t);
            T2 z; z.x = a.x - b.y; z.y = a.y + b.x;               // A + iB
            bufA[p * ld + k] = z;
        }
        __syncthreads();
        T2* src = bufA;
        T2* dst = bufB;
        FftStages<T, T2, NC>::run(src, dst, P, N, plan, T(1), tws);
        for (int idx = threadIdx.x; idx < P * N; idx += blockDim.x) {
            const int p = idx / N, m = idx - p * N;
            if (line0 + p >= nline) continue;
            const T2 z = src[p * ld + m];
            T* out = (T*)real + (size_t)(line0 + p) * K1 + 2 * m;
            out[0] = z.x;
            out[1] = z.y;
        }
    }
}

// ---- scalar_sum (fft_pme.F90:544-690) ----------------------------------------
template <typename T>
__global__ void k_scalar(typename C2<T>::t* __restrict__ q, int K1, int K2, int K3, const double* __restrict__ bsp,
                         const DynState* __restrict__ dyn, double alpha, double netchrgsq, int corr,
                         long long* __restrict__ acc, int want) {
    typedef typename C2<T>::t T2;
    size_t KK = (size_t)K1 * K2 * K3;
    const double pi = 3.14159265358979323846;
    const double fac = pi * pi / (alpha * alpha);
    const double r0 = dyn->boxinv[0], r1 = dyn->boxinv[1], r2 = dyn->boxinv[2];
    const double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    const double rk2 = dyn->rkcut * dyn->rkcut;
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    double en = 0, vs = 0, vt[6] = {0, 0, 0, 0, 0, 0};
    for (size_t ind = (size_t)blockIdx.x * blockDim.x + threadIdx.x; ind < KK;
         ind += (size_t)gridDim.x * blockDim.x) {
        if (ind == 0) continue;     // m = 0 is skipped by scalar_sum's loop bounds
        int k3 = (int)(ind / ((size_t)K1 * K2));
        size_t jnd = ind - (size_t)k3 * K1 * K2;
        int k2 = (int)(jnd / K1), k1 = (int)(jnd - (size_t)k2 * K1);
        int m1 = k1 < nf1 ? k1 : k1 - K1;
        int m2 = k2 < nf2 ? k2 : k2 - K2;
        int m3 = k3 < nf3 ? k3 : k3 - K3;
        double h1 = r0 * m1, h2 = r1 * m2, h3 = r2 * m3;
        double msq = h1 * h1 + h2 * h2 + h3 * h3;
        T2 v = q[ind];
        double eterm = 0.0;
        if (msq <= rk2) {
            double denom = pi * vol * bsp[k1] * bsp[K1 + k2] * bsp[K1 + K2 + k3] * msq;
            double ex = exp(-fac * msq);
            eterm = ex / denom;
            if (want) {
                double vterm = 2.0 * (fac * msq + 1.0) / msq;
                double s2 = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
                double es = eterm * s2;
                en += es;
                if (corr) {
                    double e2 = ex * netchrgsq / (pi * vol * msq);
                    vs += e2 * (-1.0 + 2.0 * fac * msq);
                    es -= e2;
                }
                vt[0] += es * (vterm * h1 * h1 - 1.0);
                vt[1] += es * (vterm * h1 * h2);
                vt[2] += es * (vterm * h1 * h3);
                vt[3] += es * (vterm * h2 * h2 - 1.0);
                vt[4] += es * (vterm * h2 * h3);
                vt[5] += es * (vterm * h3 * h3 - 1.0);
            }
        }
        v.x = (T)((double)v.x * eterm);
        v.y = (T)((double)v.y * eterm);
        q[ind] = v;
    }
    if (want) {
        // pot_ewk = en/2; pot_viri_coul += pot_ewk + vir_sca; virit -= vt/2
        double out[9] = {0.5 * en, 0.5 * en + 0.5 * vs, 0.5 * vs,
                         -0.5 * vt[0], -0.5 * vt[1], -0.5 * vt[2], -0.5 * vt[3], -0.5 * vt[4], -0.5 * vt[5]};
        const int idx[9] = {A_EWK, A_VC, A_VSCA, A_VTC + 0, A_VTC + 1, A_VTC + 2, A_VTC + 4, A_VTC + 5, A_VTC + 8};
        block_acc<9>(out, acc, idx, sizeof(T) == 8);
    }
}

// ---- grad_sum (fft_pme.F90:872-937) ------------------------------------------
template <bool MIXED, int P>
__global__ void k_gather(const double* __restrict__ pos, const double* __restrict__ chrg, int n,
                         const DynState* __restrict__ dyn, int K1, int K2, int K3, const void* __restrict__ qc,
                         void* facc, const int* __restrict__ order) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    typedef typename C2<T>::t T2;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int a = order ? order[t] : t;
    if (a < 0) return;   // padding slot of the cell-sorted order
    T th[3][P], dth[3][P];
    int base[3];
    const int Kd[3] = {K1, K2, K3};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double w;
        frac_coord(pos[3 * a + d], dyn->boxinv[d], Kd[d], base[d], w);
        fill_bspline_d<T, P>((T)w, th[d], dth[d]);
    }
    const T2* Q = (const T2*)qc;
    T f0 = 0, f1 = 0, f2 = 0;
    const T q = (T)chrg[a];
#pragma unroll
    for (int i3 = 0; i3 < P; ++i3) {
        int k = base[2] - P + 1 + i3;
        k = k < 0 ? k + K3 : k;
#pragma unroll
        for (int i2 = 0; i2 < P; ++i2) {
            int j = base[1] - P + 1 + i2;
            j = j < 0 ? j + K2 : j;
            size_t row = (size_t)K1 * (j + (size_t)K2 * k);
#pragma unroll
            for (int i1 = 0; i1 < P; ++i1) {
                int i = base[0] - P + 1 + i1;
                i = i < 0 ? i + K1 : i;
                T term = q * Q[row + i].x;
                f0 = f0 - (T)K1 * term * dth[0][i1] * th[1][i2] * th[2][i3];
                f1 = f1 - (T)K2 * term * th[0][i1] * dth[1][i2] * th[2][i3];
                f2 = f2 - (T)K3 * term * th[0][i1] * th[1][i2] * dth[2][i3];
            }
        }
    }
    force_add<MIXED>(facc, a, dyn->boxinv[0] * (double)f0, dyn->boxinv[1] * (double)f1,
                     dyn->boxinv[2] * (double)f2);
}

// Row-cooperative gather: P lanes per atom, lane i1 sums the points with
// first index i1; the P partial forces are then added in lane order by the
// group's first lane (fixed order: deterministic).
template <bool MIXED, int P>
__global__ void __launch_bounds__(256) k_gather_rows(const double* __restrict__ pos, const double* __restrict__ chrg,
                                                     int n, const DynState* __restrict__ dyn, int K1, int K2, int K3,
                                                     const void* __restrict__ qc, void* facc,
                                                     const int* __restrict__ order) {
    typedef typename std::conditional<MIXED, float, double>::type T;
    typedef typename C2<T>::t T2;
    constexpr int G = 32 / P;
    const int lane = threadIdx.x & 31;
    const int g = lane / P, i1 = lane - g * P;
    const int t = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * G + g;
    const int a = (g < G && t < n) ? (order ? order[t] : t) : -1;
    T f0 = 0, f1 = 0, f2 = 0;
    if (a >= 0) {
        T th[3][P], dth[3][P];
        int base[3];
        const int Kd[3] = {K1, K2, K3};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double w;
            frac_coord(pos[3 * a + d], dyn->boxinv[d], Kd[d], base[d], w);
            fill_bspline_d<T, P>((T)w, th[d], dth[d]);
        }
        T t0 = 0, d0 = 0;
#pragma unroll
        for (int q = 0; q < P; ++q) {
            t0 = q == i1 ? th[0][q] : t0;
            d0 = q == i1 ? dth[0][q] : d0;
        }
        const T* Q = (const T*)qc;       // real grid
        const T q = (T)chrg[a];
        int i = base[0] - P + 1 + i1; i = i < 0 ? i + K1 : i;
#pragma unroll
        for (int i3 = 0; i3 < P; ++i3) {
            int k = base[2] - P + 1 + i3; k = k < 0 ? k + K3 : k;
#pragma unroll
            for (int i2 = 0; i2 < P; ++i2) {
                int j = base[1] - P + 1 + i2; j = j < 0 ? j + K2 : j;
                const T term = q * Q[(size_t)K1 * (j + (size_t)K2 * k) + i];
                f0 = f0 - (T)K1 * term * d0 * th[1][i2] * th[2][i3];
                f1 = f1 - (T)K2 * term * t0 * dth[1][i2] * th[2][i3];
                f2 = f2 - (T)K3 * term * t0 * th[1][i2] * dth[2][i3];
            }
        }
    }
    // lane g*P collects its group's partials in lane order
    T s0 = f0, s1 = f1, s2 = f2;
#pragma unroll
    for (int q = 1; q < P; ++q) {
        const int src = (lane - i1 + q) & 31;
        const T o0 = __shfl_sync(0xffffffffu, f0, src), o1 = __shfl_sync(0xffffffffu, f1, src),
                o2 = __shfl_sync(0xffffffffu, f2, src);
        s0 += o0; s1 += o1; s2 += o2;
    }
    if (a >= 0 && i1 == 0)
        force_add<MIXED>(facc, a, dyn->boxinv[0] * (double)s0, dyn->boxinv[1] * (double)s1,
                         dyn->boxinv[2] * (double)s2);
}

// ---- host side ------------------------------------------------------------------
static void fill_bspline_h(double w, int order, double* arr, double* darr) {
    arr[order - 1] = 0.0; arr[1] = w; arr[0] = 1.0 - w;
    for (int k = 3; k <= order - 1; ++k) {
        double div = 1.0 / (double)(k - 1);
        arr[k - 1] = div * w * arr[k - 2];
        for (int j = 1; j <= k - 2; ++j) arr[k - j - 1] = div * ((w + j) * arr[k - j - 2] + (k - j - w) * arr[k - j - 1]);
        arr[0] = div * (1 - w) * arr[0];
    }
    darr[0] = -arr[0];
    for (int j = 2; j <= order; ++j) darr[j - 1] = arr[j - 2] - arr[j - 1];
    double div = 1.0 / (double)(order - 1);
    arr[order - 1] = div * w * arr[order - 2];
    for (int j = 1; j <= order - 2; ++j)
        arr[order - j - 1] = div * ((w + j) * arr[order - j - 2] + (order - j - w) * arr[order - j - 1]);
    arr[0] = div * (1 - w) * arr[0];
}

static bool factor(int n, FftPlan& pl) {
    pl.n = n; pl.nstage = 0;
    int m = n;
    while (m > 1) {
        int r = 0;
        for (int c : {4, 2, 3, 5}) if (m % c == 0) { r = c; break; }
        if (r == 0 || pl.nstage >= PGK_MAX_RADIX_STAGES) return false;
        pl.radix[pl.nstage++] = r;
        m /= r;
    }
    return true;
}

pgk_status spme_setup(pgk_ctx* c) {
    c->K[0] = c->prm.nfft1; c->K[1] = c->prm.nfft2; c->K[2] = c->prm.nfft3;
    c->order = c->prm.pme_order;
    if (c->order < 3 || c->order > 8) return pgk_fail(c, PGK_E_UNSUPPORTED, "pme_order must be 3..8");
    // spread and gather wrap a grid index once (base - order + 1 + i, plus K
    // when negative), so every axis needs at least pme_order points
    for (int d = 0; d < 3; ++d)
        if (c->K[d] < c->order) return pgk_fail(c, PGK_E_INVALID, "every nfft must be at least pme_order");
    for (int d = 0; d < 3; ++d)
        if (!factor(c->K[d], c->plan[d]))
            return pgk_fail(c, PGK_E_UNSUPPORTED, "SPME grid sizes must factor into 2, 3, 5");
    size_t KK = (size_t)c->K[0] * c->K[1] * c->K[2];
    PGK_CUDA(c, pgk_dmalloc(c, &c->qacc, KK * 8));
    PGK_CUDA(c, pgk_dmalloc(c, &c->qc, KK * (c->mixed() ? sizeof(float2) : sizeof(double2))));
    PGK_CUDA(c, pgk_dmalloc(c, &c->qr, KK * (c->mixed() ? sizeof(float) : sizeof(double))));
    PGK_CUDA(c, cudaMemset(c->qr, 0, KK * (c->mixed() ? sizeof(float) : sizeof(double))));
    // B-spline moduli (DFTMOD, fft_pme_init.F90:263-289)
    double arr[16], darr[16];
    fill_bspline_h(0.0, c->order, arr, darr);
    std::vector<double> bsp;
    for (int d = 0; d < 3; ++d) {
        int n = c->K[d];
        std::vector<double> a((size_t)n, 0.0), mod((size_t)n, 0.0);
        for (int i = 2; i <= c->order + 1 && i - 1 < n; ++i) a[i - 1] = arr[i - 2];
        const double twopi = 2.0 * 3.14159265358979323846;
        for (int k = 0; k < n; ++k) {
            double s1 = 0, s2 = 0;
            for (int j = 0; j < n; ++j) {
                double arg = twopi * (double)k * (double)j / (double)n;
                s1 += a[j] * std::cos(arg);
                s2 += a[j] * std::sin(arg);
            }
            mod[k] = s1 * s1 + s2 * s2;
        }
        for (int k = 1; k < n - 1; ++k) if (mod[k] < 1.0e-7) mod[k] = 0.5 * (mod[k - 1] + mod[k + 1]);
        bsp.insert(bsp.end(), mod.begin(), mod.end());
    }
    PGK_CUDA(c, pgk_dmalloc(c, &c->bsp, bsp.size() * sizeof(double)));
    PGK_CUDA(c, cudaMemcpy(c->bsp, bsp.data(), bsp.size() * sizeof(double), cudaMemcpyHostToDevice));
    for (int d = 0; d < 3; ++d) {
        if (!factor(c->K[d], c->plan[d]))
            return pgk_fail(c, PGK_E_UNSUPPORTED, "SPME grid sizes must factor into 2, 3, 5");
        int n = c->K[d];
        if (c->mixed()) {
            std::vector<float2> tw(n);
            for (int m = 0; m < n; ++m) {
                double ang = -2.0 * 3.14159265358979323846 * (double)m / (double)n;
                tw[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
            }
            PGK_CUDA(c, pgk_dmalloc(c, &c->plan[d].tw, n * sizeof(float2)));
            PGK_CUDA(c, cudaMemcpy(c->plan[d].tw, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
        } else {
            std::vector<double2> tw(n);
            for (int m = 0; m < n; ++m) {
                double ang = -2.0 * 3.14159265358979323846 * (double)m / (double)n;
                tw[m] = make_double2(std::cos(ang), std::sin(ang));
            }
            PGK_CUDA(c, pgk_dmalloc(c, &c->plan[d].tw, n * sizeof(double2)));
            PGK_CUDA(c, cudaMemcpy(c->plan[d].tw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
        }
    }
    // real-to-complex x transform when K1 is even and K1/2 factors into 2, 3, 5
    // (PGK_SPME_R2C=0: the complex x transform of the full grid)
    c->r2c = false;
    const char* rx = getenv("PGK_SPME_R2C");
    if (c->K[0] % 2 == 0 && factor(c->K[0] / 2, c->plan_rx) && !(rx && atoi(rx) == 0)) {
        const int nh = c->K[0] / 2;
        const double pi2 = 2.0 * 3.14159265358979323846;
        std::vector<double2> a((size_t)nh), b((size_t)nh + 1);
        for (int m = 0; m < nh; ++m) a[m] = make_double2(std::cos(-pi2 * m / nh), std::sin(-pi2 * m / nh));
        for (int k = 0; k <= nh; ++k) b[k] = make_double2(std::cos(-pi2 * k / c->K[0]), std::sin(-pi2 * k / c->K[0]));
        if (c->mixed()) {
            std::vector<float2> af(a.size()), bf(b.size());
            for (size_t k = 0; k < a.size(); ++k) af[k] = make_float2((float)a[k].x, (float)a[k].y);
            for (size_t k = 0; k < b.size(); ++k) bf[k] = make_float2((float)b[k].x, (float)b[k].y);
            PGK_CUDA(c, pgk_dmalloc(c, &c->plan_rx.tw, af.size() * sizeof(float2)));
            PGK_CUDA(c, cudaMemcpy(c->plan_rx.tw, af.data(), af.size() * sizeof(float2), cudaMemcpyHostToDevice));
            PGK_CUDA(c, pgk_dmalloc(c, &c->tw_rx, bf.size() * sizeof(float2)));
            PGK_CUDA(c, cudaMemcpy(c->tw_rx, bf.data(), bf.size() * sizeof(float2), cudaMemcpyHostToDevice));
        } else {
            PGK_CUDA(c, pgk_dmalloc(c, &c->plan_rx.tw, a.size() * sizeof(double2)));
            PGK_CUDA(c, cudaMemcpy(c->plan_rx.tw, a.data(), a.size() * sizeof(double2), cudaMemcpyHostToDevice));
            PGK_CUDA(c, pgk_dmalloc(c, &c->tw_rx, b.size() * sizeof(double2)));
            PGK_CUDA(c, cudaMemcpy(c->tw_rx, b.data(), b.size() * sizeof(double2), cudaMemcpyHostToDevice));
        }
        c->r2c = true;
    }
    return PGK_OK;
}

template <typename T, int AXIS, int SRC, int NC, bool CONV>
static void fft_launch(pgk_ctx* c, const FftDev& fd, int grid, int P, size_t sm, int sign, const ConvArgs& ca,
                       int K1) {
    typedef typename C2<T>::t T2;
    smem_limit(k_fft<T, AXIS, SRC, NC, CONV>, sm);
    k_fft<T, AXIS, SRC, NC, CONV><<<grid, 256, sm, c->st>>>((T2*)c->qc, SRC == 3 ? c->qr : c->qacc, K1, c->K[1],
                                                            c->K[2], fd, P, (T)sign, ca, c->dyn);
}

// x_ext: x points of the complex grid (0: K1; K1/2 + 1 on the half spectrum of
// the real-to-complex transform, for the y and z passes)
template <typename T, int AXIS, int SRC, bool CONV = false>
static pgk_status fft_pass(pgk_ctx* c, int sign, const ConvArgs* cap = nullptr, int x_ext = 0) {
    typedef typename C2<T>::t T2;
    const FftPlan& pl = c->plan[AXIS];
    FftDev fd;
    fd.n = pl.n; fd.nstage = pl.nstage;
    for (int s = 0; s < PGK_MAX_RADIX_STAGES; ++s) fd.radix[s] = pl.radix[s];
    fd.tw = pl.tw;
    int K1 = x_ext > 0 ? x_ext : c->K[0], K2 = c->K[1], K3 = c->K[2];
    int P = sizeof(T) == 4 ? 16 : 8;
    if (AXIS == 0) P = std::max(1, (sizeof(T) == 4 ? 2048 : 1024) / K1);
    const int tuned = CONV ? c->fft_p[3] : c->fft_p[AXIS];   // pencils per block chosen by spme_autotune
    if (tuned > 0) P = tuned;
    int grid;
    if (AXIS == 0) grid = (K2 * K3 + P - 1) / P;
    else if (AXIS == 1) grid = ((K1 + P - 1) / P) * K3;
    else grid = ((K1 + P - 1) / P) * K2;
    size_t sm = ((size_t)2 * P * (pl.n + 1) + pl.n) * sizeof(T2);   // two pencil buffers + twiddles
    ConvArgs ca{};
    if (cap) ca = *cap;
    switch (pl.n) {   // compile-time lengths of the configured grids; others run the generic stage loop
        case 32: fft_launch<T, AXIS, SRC, 32, CONV>(c, fd, grid, P, sm, sign, ca, K1); break;
        case 64: fft_launch<T, AXIS, SRC, 64, CONV>(c, fd, grid, P, sm, sign, ca, K1); break;
        case 128: fft_launch<T, AXIS, SRC, 128, CONV>(c, fd, grid, P, sm, sign, ca, K1); break;
        case 192: fft_launch<T, AXIS, SRC, 192, CONV>(c, fd, grid, P, sm, sign, ca, K1); break;
        default: fft_launch<T, AXIS, SRC, 0, CONV>(c, fd, grid, P, sm, sign, ca, K1); break;
    }
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// the real-to-complex x pass (FWD) or its inverse on the context's grids
template <typename T, int SRC, bool FWD>
static pgk_status fft_rx_pass(pgk_ctx* c) {
    typedef typename C2<T>::t T2;
    const FftPlan& pl = c->plan_rx;
    FftDev fd;
    fd.n = pl.n; fd.nstage = pl.nstage;
    for (int s = 0; s < PGK_MAX_RADIX_STAGES; ++s) fd.radix[s] = pl.radix[s];
    fd.tw = pl.tw;
    const int nline = c->K[1] * c->K[2];
    int P = c->fft_p[4] > 0 ? c->fft_p[4] : std::max(1, (sizeof(T) == 4 ? 2048 : 1024) / pl.n);
    const int grid = (nline + P - 1) / P;
    const size_t sm = ((size_t)2 * P * (pl.n + 1) + 2 * pl.n + 1) * sizeof(T2);
    void* real = FWD ? (void*)c->qacc : (void*)c->qr;
#define PGK_RX(NCV)                                                                                            \
    do {                                                                                                       \
        smem_limit(k_fft_rx<T, SRC, NCV, FWD>, sm);                                                            \
        k_fft_rx<T, SRC, NCV, FWD><<<grid, 256, sm, c->st>>>((T2*)c->qc, real, c->K[0], nline, fd, c->tw_rx, P); \
    } while (0)
    switch (pl.n) {
        case 16: PGK_RX(16); break;
        case 32: PGK_RX(32); break;
        case 64: PGK_RX(64); break;
        default: PGK_RX(0); break;
    }
#undef PGK_RX
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

template <typename T>
static pgk_status fft3(pgk_ctx* c, int sign, bool first) {
    pgk_status s;
    if (first) {
        if (sizeof(T) == 4) s = fft_pass<T, 0, 1>(c, sign);
        else s = fft_pass<T, 0, 2>(c, sign);
    } else {
        s = fft_pass<T, 0, 0>(c, sign);
    }
    if (s) return s;
    if ((s = fft_pass<T, 1, 0>(c, sign))) return s;
    return fft_pass<T, 2, 0>(c, sign);
}

// forward x, y; fused [forward z, influence function, backward z]; backward y, x
// With the real-to-complex x transform: real x, y on the half spectrum,
// [z, influence function, z backward], y backward, complex-to-real x.
template <typename T>
static pgk_status fft_convolve(pgk_ctx* c, long long* acc, int want) {
    pgk_status s;
    ConvArgs ca;
    ca.bsp = c->bsp; ca.alpha = c->prm.alpha; ca.netchrgsq = c->netchrgsq; ca.corr = c->prm.ifnetqcorrp;
    ca.acc = acc; ca.want = want; ca.K1f = 0;
    if (c->r2c) {
        const int xh = c->K[0] / 2 + 1;
        ca.K1f = c->K[0];
        if (sizeof(T) == 4) s = fft_rx_pass<T, 1, true>(c);
        else s = fft_rx_pass<T, 2, true>(c);
        if (s) return s;
        if ((s = fft_pass<T, 1, 0>(c, -1, nullptr, xh))) return s;
        if ((s = fft_pass<T, 2, 0, true>(c, -1, &ca, xh))) return s;
        if ((s = fft_pass<T, 1, 0>(c, +1, nullptr, xh))) return s;
        return fft_rx_pass<T, 0, false>(c);
    }
    if (sizeof(T) == 4) s = fft_pass<T, 0, 1>(c, -1);
    else s = fft_pass<T, 0, 2>(c, -1);
    if (s) return s;
    if ((s = fft_pass<T, 1, 0>(c, -1))) return s;
    if ((s = fft_pass<T, 2, 0, true>(c, -1, &ca))) return s;
    if ((s = fft_pass<T, 1, 0>(c, +1))) return s;
    return fft_pass<T, 0, 3>(c, +1);
}

// ---- autotuner of the FFT launch shapes ----------------------------------------
// Pencils per block of each axis pass (and of the z pass with the influence
// function) decide how many blocks a pass has: many pencils per block suit
// large grids, few suit the small grids of small replicas, whose SPME chain
// is latency-bound.  Every pencil is transformed on its own, so the results
// do not depend on the choice.  Each candidate (powers of two that fit the
// shared memory) is timed with CUDA events on the context's stream over a
// few launches on the context's grid; the fastest is kept per (grid shape,
// precision) for the whole process and listed by pgk_tuning_table.
struct TuneKey {
    int k1, k2, k3, fp32;
    bool operator<(const TuneKey& o) const {
        return std::tie(k1, k2, k3, fp32) < std::tie(o.k1, o.k2, o.k3, o.fp32);
    }
};
struct TuneVal { int p[5]; float us[5]; };
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneVal> g_tune;

// x_ext: as fft_pass (the half spectrum's width for the y and z passes of the
// real-to-complex transform)
template <typename T, int AXIS, int SRC, bool CONV>
static pgk_status tune_axis(pgk_ctx* c, int slot, int& best, float& best_us, int x_ext = 0) {
    typedef typename C2<T>::t T2;
    const int n = c->K[AXIS];
    const int npen = AXIS == 0 ? c->K[1] * c->K[2] : (x_ext > 0 ? x_ext : c->K[0]);
    cudaEvent_t e0, e1;
    PGK_CUDA(c, cudaEventCreate(&e0));
    PGK_CUDA(c, cudaEventCreate(&e1));
    ConvArgs ca{};
    ca.bsp = c->bsp; ca.alpha = c->prm.alpha; ca.netchrgsq = c->netchrgsq; ca.corr = c->prm.ifnetqcorrp;
    ca.acc = c->acc; ca.want = 0; ca.K1f = x_ext > 0 ? c->K[0] : 0;
    best = 0; best_us = 1e30f;
    for (int P = 1; P <= 64 && P <= npen; P *= 2) {
        if (((size_t)2 * P * (n + 1) + n) * sizeof(T2) > 160 * 1024) break;
        c->fft_p[slot] = P;
        pgk_status s = fft_pass<T, AXIS, SRC, CONV>(c, -1, CONV ? &ca : nullptr, x_ext);   // warm-up (and smem limit)
        if (s) return s;
        PGK_CUDA(c, cudaEventRecord(e0, c->st));
        for (int r = 0; r < 3; ++r)
            if ((s = fft_pass<T, AXIS, SRC, CONV>(c, -1, CONV ? &ca : nullptr, x_ext))) return s;
        PGK_CUDA(c, cudaEventRecord(e1, c->st));
        PGK_CUDA(c, cudaEventSynchronize(e1));
        float ms = 0.f;
        PGK_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
        const float us = ms * 1e3f / 3.f;
        if (us < best_us) { best_us = us; best = P; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->fft_p[slot] = best;
    return PGK_OK;
}

// the real-to-complex x pass (forward; the inverse uses the same shape)
template <typename T>
static pgk_status tune_rx(pgk_ctx* c, int& best, float& best_us) {
    typedef typename C2<T>::t T2;
    const int n = c->plan_rx.n, npen = c->K[1] * c->K[2];
    cudaEvent_t e0, e1;
    PGK_CUDA(c, cudaEventCreate(&e0));
    PGK_CUDA(c, cudaEventCreate(&e1));
    best = 0; best_us = 1e30f;
    for (int P = 1; P <= 64 && P <= npen; P *= 2) {
        if (((size_t)2 * P * (n + 1) + 2 * n + 1) * sizeof(T2) > 160 * 1024) break;
        c->fft_p[4] = P;
        pgk_status s = sizeof(T) == 4 ? fft_rx_pass<T, 1, true>(c) : fft_rx_pass<T, 2, true>(c);
        if (s) return s;
        PGK_CUDA(c, cudaEventRecord(e0, c->st));
        for (int r = 0; r < 3; ++r)
            if ((s = sizeof(T) == 4 ? fft_rx_pass<T, 1, true>(c) : fft_rx_pass<T, 2, true>(c))) return s;
        PGK_CUDA(c, cudaEventRecord(e1, c->st));
        PGK_CUDA(c, cudaEventSynchronize(e1));
        float ms = 0.f;
        PGK_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
        const float us = ms * 1e3f / 3.f;
        if (us < best_us) { best_us = us; best = P; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->fft_p[4] = best;
    return PGK_OK;
}

template <typename T>
static pgk_status autotune_fft(pgk_ctx* c, TuneVal& v) {
    pgk_status s;
    const int xh = c->r2c ? c->K[0] / 2 + 1 : 0;     // the y and z passes run on the half spectrum
    if ((s = tune_axis<T, 0, 0, false>(c, 0, v.p[0], v.us[0])) ||
        (s = tune_axis<T, 1, 0, false>(c, 1, v.p[1], v.us[1], xh)) ||
        (s = tune_axis<T, 2, 0, false>(c, 2, v.p[2], v.us[2], xh)) ||
        (s = tune_axis<T, 2, 0, true>(c, 3, v.p[3], v.us[3], xh)))
        return s;
    v.p[4] = 0; v.us[4] = 0.f;
    if (c->r2c && (s = tune_rx<T>(c, v.p[4], v.us[4]))) return s;
    return PGK_OK;
}

// launch shapes of this context's SPME passes: the process-wide choice for
// its grid shape, measured now if there is none yet (PGK_AUTOTUNE=0: the
// fixed defaults).  Runs at context set-up, outside any stream capture.
pgk_status spme_autotune(pgk_ctx* c) {
    for (int q = 0; q < 5; ++q) c->fft_p[q] = 0;
    const char* env = getenv("PGK_AUTOTUNE");
    if ((env && atoi(env) == 0) || !c->prm.ifspme) return PGK_OK;
    const TuneKey key{c->K[0], c->K[1], c->K[2], (c->mixed() ? 1 : 0) | (c->r2c ? 2 : 0)};
    std::lock_guard<std::mutex> lk(g_tune_mu);     // contexts of one grid shape share one measurement
    auto it = g_tune.find(key);
    if (it == g_tune.end()) {
        TuneVal v{};
        PGK_CUDA(c, cudaMemsetAsync(c->qc, 0, (size_t)c->K[0] * c->K[1] * c->K[2] * (c->mixed() ? 8 : 16), c->st));
        PGK_CUDA(c, cudaMemsetAsync(c->qacc, 0, (size_t)c->K[0] * c->K[1] * c->K[2] * 8, c->st));
        pgk_status s = c->mixed() ? autotune_fft<float>(c, v) : autotune_fft<double>(c, v);
        if (s) return s;
        PGK_CUDA(c, cudaMemsetAsync(c->acc, 0, sizeof(long long) * 2 * NACC, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        it = g_tune.emplace(key, v).first;
    }
    for (int q = 0; q < 5; ++q) c->fft_p[q] = it->second.p[q];
    return PGK_OK;
}

extern "C" int64_t pgk_tuning_table(char* buf, int64_t cap) {
    std::string t;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (auto& kv : g_tune) {
            char line[256];
            char rx[64] = "";
            if (kv.first.fp32 & 2) snprintf(rx, sizeof(rx), " real-x %d (%.1f us)", kv.second.p[4], kv.second.us[4]);
            snprintf(line, sizeof(line),
                     "spme %dx%dx%d %s: pencils per block x %d (%.1f us) y %d (%.1f us) z %d (%.1f us) "
                     "z+influence %d (%.1f us)%s\n",
                     kv.first.k1, kv.first.k2, kv.first.k3, (kv.first.fp32 & 1) ? "fp32" : "fp64", kv.second.p[0],
                     kv.second.us[0], kv.second.p[1], kv.second.us[1], kv.second.p[2], kv.second.us[2],
                     kv.second.p[3], kv.second.us[3], rx);
            t += line;
        }
    }
    t += pair_tuning_text();
    if (buf && cap > 0) {
        const size_t m = std::min((size_t)cap - 1, t.size());
        memcpy(buf, t.data(), m);
        buf[m] = 0;
    }
    return (int64_t)t.size() + 1;
}

template <bool MIXED, int P>
static void spread_gather(pgk_ctx* c, bool gather, int group) {
    const int* order = c->list_valid ? c->perm : nullptr;
    const int n = order ? c->npad : c->natom;     // sorted order runs over the padded slots
    const int warps = (n + 32 / P - 1) / (32 / P);
    if (!gather)
        k_spread_rows<MIXED, P><<<(warps + 7) / 8, 256, 0, c->st>>>(c->pos, c->chrg, n, c->dyn, c->K[0], c->K[1],
                                                                    c->K[2], c->qacc, order);
    else
        k_gather_rows<MIXED, P><<<(warps + 7) / 8, 256, 0, c->st>>>(c->pos, c->chrg, n, c->dyn, c->K[0], c->K[1],
                                                                    c->K[2], c->qr, c->facc[group], order);
    PGK_LAUNCHED(c);
}

template <bool MIXED>
static pgk_status dispatch_sg(pgk_ctx* c, bool gather, int group) {
    switch (c->order) {
        case 3: spread_gather<MIXED, 3>(c, gather, group); break;
        case 4: spread_gather<MIXED, 4>(c, gather, group); break;
        case 5: spread_gather<MIXED, 5>(c, gather, group); break;
        case 6: spread_gather<MIXED, 6>(c, gather, group); break;
        case 7: spread_gather<MIXED, 7>(c, gather, group); break;
        case 8: spread_gather<MIXED, 8>(c, gather, group); break;
        default: return pgk_fail(c, PGK_E_UNSUPPORTED, "pme_order");
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

pgk_status launch_spme(pgk_ctx* c, int group, bool ene, bool vir) {
    size_t KK = (size_t)c->K[0] * c->K[1] * c->K[2];
    PGK_CUDA(c, cudaMemsetAsync(c->qacc, 0, KK * 8, c->st));
    pgk_status s;
    long long* acc = c->acc + (size_t)group * NACC;
    int want = (ene || vir) ? 1 : 0;
    if (c->mixed()) {
        if ((s = dispatch_sg<true>(c, false, group))) return s;
        if ((s = fft_convolve<float>(c, acc, want))) return s;
        if ((s = dispatch_sg<true>(c, true, group))) return s;
    } else {
        if ((s = dispatch_sg<false>(c, false, group))) return s;
        if ((s = fft_convolve<double>(c, acc, want))) return s;
        if ((s = dispatch_sg<false>(c, true, group))) return s;
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// single stages of launch_spme for pgk_bench_kernel (1 spread, 2 gather, 3 forward FFT)
pgk_status spme_bench(pgk_ctx* c, int which) {
    if (which == 1) return c->mixed() ? dispatch_sg<true>(c, false, 0) : dispatch_sg<false>(c, false, 0);
    if (which == 2) return c->mixed() ? dispatch_sg<true>(c, true, 0) : dispatch_sg<false>(c, true, 0);
    return c->mixed() ? fft3<float>(c, -1, false) : fft3<double>(c, -1, false);
}

// ============================================================================
// Per-atom split of the SPME reciprocal energy and virial tensor (bulk heat
// flux): the SPME form of ewaldkp_hf's per-atom terms (ewaldk_hf.F90:165-230;
// the reference has them only for standard Ewald).  With S = FFT(Q) and the
// influence function eterm of scalar_sum (fft_pme.F90:544-690),
//   pot_atm(i)      = 1/2 q_i sum_g theta_i(g) IFFT(eterm S)(g) - alpha/sqrt(pi) q_i^2
//   viri_atm(a,b,i) = 1/2 q_i sum_g theta_i(g) IFFT(eterm (delta_ab - vterm h_a h_b) S)(g)
// FP64 in both precisions (the heat-flux sums are FP64): the charges go into
// a double grid, one forward transform, k_hf_sgrids writes the seven
// convolved grids (energy; tensor xx xy xz yy yz zz) as one array of 7 K^3
// points, whose x and y backward passes run as one K1 x K2 x 7K3 grid and
// whose z passes run per grid; k_hf_spme_atm gathers the seven real parts
// with each atom's B-spline weights.
// Layout: hfk_q double[K3][K2][K1]; hfk_g double2[7][K3][K2][K1];
// hfk_out double[N] energies | [9N] tensors, (3,3) column-major per atom.
// ============================================================================
__global__ void k_hf_sgrids(double2* __restrict__ g, int K1, int K2, int K3, const double* __restrict__ bsp,
                            double alpha, const DynState* __restrict__ dyn) {
    const size_t KK = (size_t)K1 * K2 * K3;
    const double pi = 3.14159265358979323846;
    const double fac = pi * pi / (alpha * alpha);
    const double vol = dyn->box[0] * dyn->box[1] * dyn->box[2];
    const double rk2 = dyn->rkcut * dyn->rkcut;
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    for (size_t ind = blockIdx.x * (size_t)blockDim.x + threadIdx.x; ind < KK; ind += (size_t)gridDim.x * blockDim.x) {
        const int k3 = (int)(ind / ((size_t)K1 * K2));
        const size_t jnd = ind - (size_t)k3 * K1 * K2;
        const int k2 = (int)(jnd / K1), k1 = (int)(jnd - (size_t)k2 * K1);
        const int m1 = k1 < nf1 ? k1 : k1 - K1;
        const int m2 = k2 < nf2 ? k2 : k2 - K2;
        const int m3 = k3 < nf3 ? k3 : k3 - K3;
        const double h[3] = {dyn->boxinv[0] * m1, dyn->boxinv[1] * m2, dyn->boxinv[2] * m3};
        const double msq = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
        double2 es = make_double2(0.0, 0.0);
        double vterm = 0.0;
        if (ind != 0 && msq <= rk2) {
            const double denom = pi * vol * bsp[k1] * bsp[K1 + k2] * bsp[K1 + K2 + k3] * msq;
            const double eterm = exp(-fac * msq) / denom;
            vterm = 2.0 * (fac * msq + 1.0) / msq;
            const double2 S = g[ind];
            es = make_double2(eterm * S.x, eterm * S.y);
        }
        g[ind] = es;
        const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double f = (ab[c][0] == ab[c][1] ? 1.0 : 0.0) - vterm * h[ab[c][0]] * h[ab[c][1]];
            g[(size_t)(1 + c) * KK + ind] = make_double2(es.x * f, es.y * f);
        }
    }
}

template <int P>
__global__ void k_hf_spme_atm(const double* __restrict__ pos, const double* __restrict__ chrg, int n,
                              const DynState* __restrict__ dyn, int K1, int K2, int K3,
                              const double2* __restrict__ g, double alpha, double* __restrict__ out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const size_t KK = (size_t)K1 * K2 * K3;
    double th[3][P], dth[3][P];
    int base[3];
    const int Kd[3] = {K1, K2, K3};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double w;
        frac_coord(pos[3 * a + d], dyn->boxinv[d], Kd[d], base[d], w);
        fill_bspline_d<double, P>(w, th[d], dth[d]);
    }
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int i3 = 0; i3 < P; ++i3) {
        int k = base[2] - P + 1 + i3;
        k = k < 0 ? k + K3 : k;
        for (int i2 = 0; i2 < P; ++i2) {
            int j = base[1] - P + 1 + i2;
            j = j < 0 ? j + K2 : j;
            const size_t row = (size_t)K1 * (j + (size_t)K2 * k);
            const double w23 = th[1][i2] * th[2][i3];
#pragma unroll
            for (int i1 = 0; i1 < P; ++i1) {
                int i = base[0] - P + 1 + i1;
                i = i < 0 ? i + K1 : i;
                const double w = th[0][i1] * w23;
#pragma unroll
                for (int c = 0; c < 7; ++c) acc[c] += w * g[(size_t)c * KK + row + i].x;
            }
        }
    }
    const double q = chrg[a], hq = 0.5 * q;
    const double self = alpha / sqrt(3.14159265358979323846);
    out[a] = hq * acc[0] - self * q * q;
    double* v = out + n + (size_t)9 * a;
    v[0] = hq * acc[1]; v[1] = hq * acc[2]; v[2] = hq * acc[3];
    v[3] = v[1];        v[4] = hq * acc[4]; v[5] = hq * acc[5];
    v[6] = v[2];        v[7] = v[5];        v[8] = hq * acc[6];
}

// one FP64 pencil pass over an explicit grid (the heat-flux grids)
template <int AXIS, int SRC>
static pgk_status hfk_fft_pass(pgk_ctx* c, double2* data, const void* src, int K3e, int sign) {
    const FftPlan& pl = c->plan[AXIS];
    FftDev fd;
    fd.n = pl.n; fd.nstage = pl.nstage;
    for (int q = 0; q < PGK_MAX_RADIX_STAGES; ++q) fd.radix[q] = pl.radix[q];
    fd.tw = c->hfk_tw[AXIS];
    const int K1 = c->K[0], K2 = c->K[1];
    int P = 8;
    if (AXIS == 0) P = std::max(1, 1024 / K1);
    int grid;
    if (AXIS == 0) grid = (K2 * K3e + P - 1) / P;
    else if (AXIS == 1) grid = ((K1 + P - 1) / P) * K3e;
    else grid = ((K1 + P - 1) / P) * K2;
    const size_t sm = ((size_t)2 * P * (pl.n + 1) + pl.n) * sizeof(double2);
    ConvArgs ca{};
    PGK_CUDA(c, smem_limit(k_fft<double, AXIS, SRC, 0, false>, sm));
    k_fft<double, AXIS, SRC, 0, false><<<grid, 256, sm, c->st>>>(data, src, K1, K2, K3e, fd, P, (double)sign, ca,
                                                                  c->dyn);
    PGK_LAUNCHED(c);
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// buffers of the heat-flux SPME split (first use; FP64 twiddles of the
// context's plans, which hold FP32 twiddles in mixed precision)
static pgk_status hfk_setup(pgk_ctx* c) {
    if (c->hfk_g) return PGK_OK;
    const size_t KK = (size_t)c->K[0] * c->K[1] * c->K[2];
    PGK_CUDA(c, pgk_dmalloc(c, &c->hfk_q, KK * sizeof(double)));
    PGK_CUDA(c, pgk_dmalloc(c, &c->hfk_g, 7 * KK * sizeof(double2)));
    PGK_CUDA(c, pgk_dmalloc(c, &c->hfk_out, (size_t)10 * c->natom * sizeof(double)));
    for (int d = 0; d < 3; ++d) {
        const int n = c->K[d];
        std::vector<double2> tw(n);
        for (int m = 0; m < n; ++m) {
            const double ang = -2.0 * 3.14159265358979323846 * (double)m / (double)n;
            tw[m] = make_double2(std::cos(ang), std::sin(ang));
        }
        PGK_CUDA(c, pgk_dmalloc(c, &c->hfk_tw[d], n * sizeof(double2)));
        PGK_CUDA(c, cudaMemcpyAsync(c->hfk_tw[d], tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice, c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
    }
    return PGK_OK;
}

template <int P>
static void hfk_spread_gather(pgk_ctx* c, bool gather) {
    const int n = c->natom;
    if (!gather)
        k_spread<false, P><<<(n + 127) / 128, 128, 0, c->st>>>(c->pos, c->chrg, n, c->dyn, c->K[0], c->K[1], c->K[2],
                                                               c->hfk_q, nullptr);
    else
        k_hf_spme_atm<P><<<(n + 127) / 128, 128, 0, c->st>>>(c->pos, c->chrg, n, c->dyn, c->K[0], c->K[1], c->K[2],
                                                             (const double2*)c->hfk_g, c->prm.alpha, c->hfk_out);
    PGK_LAUNCHED(c);
}

// the split at the current positions into c->hfk_out (device)
pgk_status launch_spme_hf_atm(pgk_ctx* c) {
    if (!c->prm.ifspme) return pgk_fail(c, PGK_E_INVALID, "ifspme is off");
    pgk_status s;
    if ((s = hfk_setup(c))) return s;
    const int K1 = c->K[0], K2 = c->K[1], K3 = c->K[2];
    const size_t KK = (size_t)K1 * K2 * K3;
    double2* g = (double2*)c->hfk_g;
    PGK_CUDA(c, cudaMemsetAsync(c->hfk_q, 0, KK * sizeof(double), c->st));
    switch (c->order) {
        case 3: hfk_spread_gather<3>(c, false); break;
        case 4: hfk_spread_gather<4>(c, false); break;
        case 5: hfk_spread_gather<5>(c, false); break;
        case 6: hfk_spread_gather<6>(c, false); break;
        case 7: hfk_spread_gather<7>(c, false); break;
        default: hfk_spread_gather<8>(c, false); break;
    }
    if ((s = hfk_fft_pass<0, 2>(c, g, c->hfk_q, K3, -1)) || (s = hfk_fft_pass<1, 0>(c, g, nullptr, K3, -1)) ||
        (s = hfk_fft_pass<2, 0>(c, g, nullptr, K3, -1)))
        return s;
    k_hf_sgrids<<<c->nsm * 4, 256, 0, c->st>>>(g, K1, K2, K3, c->bsp, c->prm.alpha, c->dyn);
    PGK_LAUNCHED(c);
    for (int q = 0; q < 7; ++q)
        if ((s = hfk_fft_pass<2, 0>(c, g + (size_t)q * KK, nullptr, K3, +1))) return s;
    if ((s = hfk_fft_pass<1, 0>(c, g, nullptr, 7 * K3, +1)) || (s = hfk_fft_pass<0, 0>(c, g, nullptr, 7 * K3, +1)))
        return s;
    switch (c->order) {
        case 3: hfk_spread_gather<3>(c, true); break;
        case 4: hfk_spread_gather<4>(c, true); break;
        case 5: hfk_spread_gather<5>(c, true); break;
        case 6: hfk_spread_gather<6>(c, true); break;
        case 7: hfk_spread_gather<7>(c, true); break;
        default: hfk_spread_gather<8>(c, true); break;
    }
    PGK_CUDA(c, cudaGetLastError());
    return PGK_OK;
}

// ============================================================================
// Allocation-free SPME reciprocal force: pgk_fft_pme_noalloc.
//
// For callers that cannot call cudaMalloc during a run: a host driver or a
// serving process that reserves all device memory up front (cudaMalloc and
// cudaFree synchronise the whole device and can fail once a pool owns the
// HBM), so per-call allocation would stall other streams or break the
// memory budget.  The caller passes device buffers for the inputs and the
// output; every temporary of the computation lives in the file-scope array
// below, of fixed size, which every GPU that loads this library holds until
// the process exits.
//
// Limits: nfft1*nfft2*nfft3 <= 64^3, each nfft <= 256, 3 <= pme_order <= 8;
// larger sizes return PGK_E_SCRATCH_LIMIT.  Every nfft must also be a
// product of 2, 3 and 5 (else PGK_E_UNSUPPORTED) and at least pme_order
// (else PGK_E_INVALID: spread and gather wrap a grid index only once).
// The first call on a device looks up the array's device address there
// (cudaGetSymbolAddress); make that first call before any stream capture.
// All calls share the one array: calls that overlap on the GPU (two streams,
// two host threads) race on it and must be serialised by the caller.
// FP64 arithmetic (the device parity path); forces are ADDED to d_force.
// ============================================================================
#define NOALLOC_MAX_GRID (64 * 64 * 64)
#define NOALLOC_MAX_N 256
#define NOALLOC_OFF_DYN 0
#define NOALLOC_OFF_ACC 1024
#define NOALLOC_OFF_BSP (NOALLOC_OFF_ACC + 2048)
#define NOALLOC_OFF_TW (NOALLOC_OFF_BSP + 3 * NOALLOC_MAX_N * 8)
#define NOALLOC_OFF_QACC (NOALLOC_OFF_TW + 3 * NOALLOC_MAX_N * 16)
#define NOALLOC_OFF_QC (NOALLOC_OFF_QACC + NOALLOC_MAX_GRID * 8)
#define NOALLOC_BYTES (NOALLOC_OFF_QC + NOALLOC_MAX_GRID * 16)
static_assert(sizeof(DynState) <= NOALLOC_OFF_ACC, "DynState slot");
static_assert(NACC * 8 <= NOALLOC_OFF_BSP - NOALLOC_OFF_ACC, "accumulator slot");
static_assert(NOALLOC_OFF_QACC % 256 == 0 && NOALLOC_OFF_QC % 256 == 0, "alignment");

static __device__ __align__(256) unsigned char g_spme_scratch[NOALLOC_BYTES];

#define NOALLOC_MAX_DEVICES 64
static unsigned char* g_scratch_ptr[NOALLOC_MAX_DEVICES];   // device address of g_spme_scratch, per device
static int g_scratch_key[NOALLOC_MAX_DEVICES][4];           // (K1, K2, K3, order) of the tables in place

// twiddles exp(-2 pi i m / n) per axis and the B-spline moduli (DFTMOD,
// fft_pme_init.F90:263-289), written into the scratch array
__global__ void k_noalloc_tables(unsigned char* base, int K1, int K2, int K3, int order) {
    double* bsp = (double*)(base + NOALLOC_OFF_BSP);
    double2* tw = (double2*)(base + NOALLOC_OFF_TW);
    const int Kd[3] = {K1, K2, K3};
    double arr[8], darr[8];
    switch (order) {
        case 3: fill_bspline_d<double, 3>(0.0, arr, darr); break;
        case 4: fill_bspline_d<double, 4>(0.0, arr, darr); break;
        case 5: fill_bspline_d<double, 5>(0.0, arr, darr); break;
        case 6: fill_bspline_d<double, 6>(0.0, arr, darr); break;
        case 7: fill_bspline_d<double, 7>(0.0, arr, darr); break;
        default: fill_bspline_d<double, 8>(0.0, arr, darr); break;
    }
    int off = 0;
    for (int d = 0; d < 3; ++d) {
        int n = Kd[d];
        for (int m = threadIdx.x; m < n; m += blockDim.x) {
            double s, c;
            sincospi(-2.0 * (double)m / (double)n, &s, &c);
            tw[d * NOALLOC_MAX_N + m] = make_double2(c, s);
            double s1 = 0.0, s2 = 0.0;
            for (int j = 1; j <= order && j < n; ++j) {   // bsp_arr(j+1) = array(j)
                double sn, cs;
                sincospi(2.0 * (double)(((long long)m * j) % n) / (double)n, &sn, &cs);
                s1 += arr[j - 1] * cs;
                s2 += arr[j - 1] * sn;
            }
            bsp[off + m] = s1 * s1 + s2 * s2;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 1; k < n - 1; ++k)
                if (bsp[off + k] < 1.0e-7) bsp[off + k] = 0.5 * (bsp[off + k - 1] + bsp[off + k + 1]);
        __syncthreads();
        off += n;
    }
}

__global__ void k_noalloc_dyn(DynState* d, double b0, double b1, double b2, double rk) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        d->box[0] = b0; d->box[1] = b1; d->box[2] = b2;
        d->boxinv[0] = 1.0 / b0; d->boxinv[1] = 1.0 / b1; d->boxinv[2] = 1.0 / b2;
        d->rkcut = rk;
    }
}

template <int AXIS, int SRC>
static cudaError_t noalloc_fft_pass(unsigned char* base, const FftPlan& pl, int K1, int K2, int K3, int sign,
                                    cudaStream_t st) {
    FftDev fd;
    fd.n = pl.n; fd.nstage = pl.nstage;
    for (int s = 0; s < PGK_MAX_RADIX_STAGES; ++s) fd.radix[s] = pl.radix[s];
    fd.tw = base + NOALLOC_OFF_TW + (size_t)AXIS * NOALLOC_MAX_N * 16;
    int P = 8;
    if (AXIS == 0) P = std::max(1, 1024 / K1);
    int grid = AXIS == 0 ? (K2 * K3 + P - 1) / P : ((K1 + P - 1) / P) * (AXIS == 1 ? K3 : K2);
    size_t sm = ((size_t)2 * P * (pl.n + 1) + pl.n) * sizeof(double2);   // two pencil buffers + twiddles
    cudaError_t e = smem_limit(k_fft<double, AXIS, SRC, 0, false>, sm);
    if (e != cudaSuccess) return e;
    ConvArgs ca{};
    k_fft<double, AXIS, SRC, 0, false><<<grid, 256, sm, st>>>((double2*)(base + NOALLOC_OFF_QC),
                                                              base + NOALLOC_OFF_QACC, K1, K2, K3, fd, P,
                                                              (double)sign, ca,
                                                              (const DynState*)(base + NOALLOC_OFF_DYN));
    return cudaGetLastError();
}

template <int P>
static void noalloc_sg(unsigned char* base, const double* pos, const double* chrg, int n, int K1, int K2, int K3,
                       double* force, bool gather, cudaStream_t st) {
    const DynState* dyn = (const DynState*)(base + NOALLOC_OFF_DYN);
    if (!gather)
        k_spread<false, P><<<(n + 127) / 128, 128, 0, st>>>(pos, chrg, n, dyn, K1, K2, K3, base + NOALLOC_OFF_QACC,
                                                            nullptr);
    else
        k_gather<false, P><<<(n + 127) / 128, 128, 0, st>>>(pos, chrg, n, dyn, K1, K2, K3, base + NOALLOC_OFF_QC,
                                                            force, nullptr);
}

static void noalloc_sg_order(int order, unsigned char* base, const double* pos, const double* chrg, int n, int K1,
                             int K2, int K3, double* force, bool gather, cudaStream_t st) {
    switch (order) {
        case 3: noalloc_sg<3>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
        case 4: noalloc_sg<4>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
        case 5: noalloc_sg<5>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
        case 6: noalloc_sg<6>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
        case 7: noalloc_sg<7>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
        default: noalloc_sg<8>(base, pos, chrg, n, K1, K2, K3, force, gather, st); break;
    }
}

extern "C" pgk_status pgk_fft_pme_noalloc(const double* d_atmcor, const double* d_atmchrg, int32_t natom,
                                          const double* box, double alpha, int32_t nfft1, int32_t nfft2,
                                          int32_t nfft3, int32_t pme_order, double* d_force, double* pot_ewk,
                                          void* stream) {
    if (!d_atmcor || !d_atmchrg || !d_force || !box || natom < 1 || alpha <= 0.0) return PGK_E_INVALID;
    if (nfft1 < 2 || nfft2 < 2 || nfft3 < 2 || pme_order < 3) return PGK_E_INVALID;
    if (nfft1 > NOALLOC_MAX_N || nfft2 > NOALLOC_MAX_N || nfft3 > NOALLOC_MAX_N ||
        (long long)nfft1 * nfft2 * nfft3 > NOALLOC_MAX_GRID || pme_order > 8)
        return PGK_E_SCRATCH_LIMIT;
    if (nfft1 < pme_order || nfft2 < pme_order || nfft3 < pme_order) return PGK_E_INVALID;
    FftPlan pl[3];
    const int Kd[3] = {nfft1, nfft2, nfft3};
    for (int d = 0; d < 3; ++d)
        if (!factor(Kd[d], pl[d])) return PGK_E_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PGK_E_CUDA;
    if (!g_scratch_ptr[dev]) {   // once per device, with that device current
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_spme_scratch) != cudaSuccess || !p) return PGK_E_CUDA;
        g_scratch_ptr[dev] = (unsigned char*)p;
        g_scratch_key[dev][0] = 0;
    }
    unsigned char* base = g_scratch_ptr[dev];
    int* key = g_scratch_key[dev];
    if (key[0] != nfft1 || key[1] != nfft2 || key[2] != nfft3 || key[3] != pme_order) {
        k_noalloc_tables<<<1, 256, 0, st>>>(base, nfft1, nfft2, nfft3, pme_order);
        if (cudaGetLastError() != cudaSuccess) return PGK_E_CUDA;
        key[0] = nfft1; key[1] = nfft2; key[2] = nfft3; key[3] = pme_order;
    }
    // erf_corr_cutoff.F90:28-62 (min-ish rule of the reference)
    double m1 = 0.5 * (nfft1 / box[0]), rk = m1, m2 = 0.5 * (nfft2 / box[1]), m3 = 0.5 * (nfft3 / box[2]);
    if (m2 < m1) rk = m2;
    if (m3 < m2) rk = m3;
    k_noalloc_dyn<<<1, 32, 0, st>>>((DynState*)(base + NOALLOC_OFF_DYN), box[0], box[1], box[2], 0.9 * rk);
    // the grid accumulates and the energy slots sum: both start at zero
    size_t KK = (size_t)nfft1 * nfft2 * nfft3;
    if (cudaMemsetAsync(base + NOALLOC_OFF_QACC, 0, KK * 8, st) != cudaSuccess) return PGK_E_CUDA;
    if (cudaMemsetAsync(base + NOALLOC_OFF_ACC, 0, NACC * 8, st) != cudaSuccess) return PGK_E_CUDA;
    noalloc_sg_order(pme_order, base, d_atmcor, d_atmchrg, natom, nfft1, nfft2, nfft3, d_force, false, st);
    if (noalloc_fft_pass<0, 2>(base, pl[0], nfft1, nfft2, nfft3, -1, st) != cudaSuccess ||
        noalloc_fft_pass<1, 0>(base, pl[1], nfft1, nfft2, nfft3, -1, st) != cudaSuccess ||
        noalloc_fft_pass<2, 0>(base, pl[2], nfft1, nfft2, nfft3, -1, st) != cudaSuccess)
        return PGK_E_CUDA;
    k_scalar<double><<<148 * 2, 256, 0, st>>>((double2*)(base + NOALLOC_OFF_QC), nfft1, nfft2, nfft3,
                                              (const double*)(base + NOALLOC_OFF_BSP),
                                              (const DynState*)(base + NOALLOC_OFF_DYN), alpha, 0.0, 0,
                                              (long long*)(base + NOALLOC_OFF_ACC), 1);
    if (noalloc_fft_pass<0, 0>(base, pl[0], nfft1, nfft2, nfft3, +1, st) != cudaSuccess ||
        noalloc_fft_pass<1, 0>(base, pl[1], nfft1, nfft2, nfft3, +1, st) != cudaSuccess ||
        noalloc_fft_pass<2, 0>(base, pl[2], nfft1, nfft2, nfft3, +1, st) != cudaSuccess)
        return PGK_E_CUDA;
    noalloc_sg_order(pme_order, base, d_atmcor, d_atmchrg, natom, nfft1, nfft2, nfft3, d_force, true, st);
    if (cudaGetLastError() != cudaSuccess) return PGK_E_CUDA;
    if (pot_ewk) {
        double e_ewk = 0.0;
        if (cudaMemcpyAsync(&e_ewk, base + NOALLOC_OFF_ACC + A_EWK * 8, sizeof(double), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PGK_E_CUDA;
        *pot_ewk = e_ewk;
    }
    return PGK_OK;
}
