// pgk_oracle.cpp -- FP64 CPU restatement of the peachgk_md force-and-
// integration path.  TEST INFRASTRUCTURE ONLY: the parity tests, smoke() and
// the CPU-baseline leg of bench.py load it as the checker; the product
// library (libpgkgpu.so) never links or calls it.
//
// Parity status: the reference is Fortran 90 and no Fortran compiler exists in
// this image, so the reference cannot be built or run here.  The restatement
// is pinned against the reference's own recorded run instead: the reference
// tree keeps the step-1 positions (out_pos.dat) and energies (out_ene.dat) of
// its Pt/Morse sample, and tests/test_golden_pt_morse.py reproduces every
// recorded energy term of calforce (LJ, real-space and SPME Coulomb, self
// term, 1-4, bond, angle, torsion, RB torsion, Morse, total) from those
// positions within the precision the recorded files carry (1e-5 .. 1e-9).
// Analytical known answers in tests/ add what a recorded energy cannot show
// (forces by finite differences, two-body LJ/Coulomb, Madelung constant,
// B-spline partition of unity, FFT vs direct DFT, spline vs erfc, constraint
// residuals, conserved NHC energy).
//
// Every routine cites the reference file:line it restates.  Arithmetic follows
// the reference order (left-to-right sums, dnint = round-half-away) and is
// compiled with -ffp-contract=off so no FMA changes the FP64 results.
// Optional OpenMP parallelism (orc_set_threads) is used for the timed CPU
// baseline; with one thread the loop order is the reference's serial order.

#include "../include/pgk_gpu.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

typedef std::complex<double> cplx;

inline double dnint(double x) { return std::round(x); }   // Fortran dnint/anint

// Static-chunk parallel loop over [0, n) on `nt` std::threads (the image has
// no OpenMP runtime).  fn(begin, end, tid) handles one contiguous chunk.
void par_chunks(int nt, long long n, const std::function<void(long long, long long, int)>& fn) {
    if (nt <= 1 || n < 2) { fn(0, n, 0); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
        long long b = n * t / nt, e = n * (t + 1) / nt;
        th.emplace_back([&fn, b, e, t]() { fn(b, e, t); });
    }
    for (auto& x : th) x.join();
}

// --------------------------------------------------------------------------
// complex FFT (own mixed radix 2/3/4/5 + generic), unnormalised.
// sign = -1: FFTPACK cfftf (exp(-2 pi i jk/n)); sign = +1: cfftb.
// Stands in for fft3-public.F CFFTF/CFFTB; checked against a direct DFT.
// --------------------------------------------------------------------------
void fft_rec(cplx* a, int n, int stride, int sign, cplx* scratch) {
    if (n == 1) return;
    int r = 0;
    for (int c : {4, 2, 3, 5}) if (n % c == 0) { r = c; break; }
    if (r == 0) {   // generic prime: direct DFT
        for (int k = 0; k < n; ++k) {
            cplx s(0, 0);
            for (int j = 0; j < n; ++j) {
                double ang = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / n;
                s += a[(long long)j * stride] * cplx(std::cos(ang), std::sin(ang));
            }
            scratch[k] = s;
        }
        for (int k = 0; k < n; ++k) a[(long long)k * stride] = scratch[k];
        return;
    }
    int m = n / r;
    // decimation in time: sub-sequences x[r*j + q], q = 0..r-1
    std::vector<cplx> sub((size_t)n);
    for (int q = 0; q < r; ++q)
        for (int j = 0; j < m; ++j) sub[(size_t)q * m + j] = a[(long long)(r * j + q) * stride];
    for (int q = 0; q < r; ++q) fft_rec(&sub[(size_t)q * m], m, 1, sign, scratch);
    for (int k = 0; k < m; ++k) {
        for (int t = 0; t < r; ++t) {
            int kk = k + t * m;
            cplx s(0, 0);
            for (int q = 0; q < r; ++q) {
                double ang = sign * 2.0 * M_PI * (double)(((long long)q * kk) % n) / n;
                s += sub[(size_t)q * m + k] * cplx(std::cos(ang), std::sin(ang));
            }
            a[(long long)kk * stride] = s;
        }
    }
}

void fft1d(cplx* a, int n, int stride, int sign) {
    std::vector<cplx> scratch((size_t)n);
    fft_rec(a, n, stride, sign, scratch.data());
}

struct Forces { std::vector<double> fl, fs; pgk_virials vl{}, vs{}; pgk_energies el{}, es{}; };

// --------------------------------------------------------------------------
struct Oracle {
    // ---- md_global mirrors (0-based) ----
    int natom = 0;
    std::vector<double> atmcor, atmvel, atmmass, atmchrg;
    std::vector<int> atmindex;  // 0-based type
    int ntyp = 0;
    std::vector<double> radij, welij;  // [i + ntyp*j]
    std::vector<int> inttyp;
    // Morse pairs (rdpara.F90:680-720), column-major (i,j) like radij
    std::vector<double> welmor, radmor, almor;
    std::vector<int> mor_atoms;            // nmorselist (linkbond.F90), 0-based
    std::vector<int> mor_idx, mor_list;    // Morse list rows: [mor_atoms+1] starts, 0-based partners
    int mor_list_mode = 0;                 // PGK_LIST_* order of the last Morse list
    std::vector<int> molidx, mollist;  // 0-based
    std::vector<int> excl_idx, excl_list;  // reference CSR kept 1-based values
    // bonded
    std::vector<int> bi, bj; std::vector<double> bk, br0;
    std::vector<int> ai, aj, ak; std::vector<double> akk, at0;
    std::vector<int> ti, tj, tk, tl, tdiv; std::vector<double> tbar, tph, tper;
    std::vector<int> rbi, rbj, rbk, rbl; std::vector<double> rbc;
    // 1-4 pairs in calnon14p order
    std::vector<int> p14i, p14j; std::vector<double> p14e, p14v;
    // constraints
    std::vector<int> cidx, clist, ci, cj; std::vector<double> cd;
    int degfree = 0;
    pgk_params prm{};
    // spline tables (spline_interp.F90)
    int nspl = 0; double hspl = 0;
    std::vector<double> xtbl;
    std::vector<double> tb[4], sb[4], sc[4], sd[4];   // 0 real, 1 realpot, 2 excs, 3 excspot
    // SPME
    std::vector<double> bsp[3];
    double rkcut = 0;
    double pot_ewc = 0, netchrgsq = 0;
    // list
    std::vector<int> nb_index;  // [natom+1] 1-based starts (reference nb_indexall)
    std::vector<int> nb_list;   // 1-based j, 0 sentinel
    long long nlistnball = 0;
    int list_used_mode = 0;
    // box
    double box[3] = {0, 0, 0};
    int nthreads = 1;
    // chain state
    pgk_chain ch{};
    double yratio = 1, zratio = 1;
    int status = 0;
    Forces F;
    // heat flux + region Langevin (moldyn_hf.F90 state)
    struct HF {
        bool set = false;
        int nreg = 0, heatfinterval = 1, nlt = 0, ifoutthc = 0;
        double z1[PGK_HF_MAX_REGIONS], z2[PGK_HF_MAX_REGIONS];
        std::vector<int> hftyp, molof, ltmole;
        std::vector<double> molecom, molevel;
        std::vector<double> pot;   // [8][natom]
        std::vector<double> W;     // [8][nreg][3][natom]: viri*_atm(a,3,i,r)
        double lx1[8], lx2[8], ly1[8], ly2[8], lz1[8], lz2[8], ltemp[8], ldamp[8];
        uint64_t seed = 0;
        std::vector<int> ltreg;    // Langevin region of each atom (-1: none)
        std::vector<double> frand; // 3N accelerations of the former half
        double dekin[8];
        // per-atom reciprocal term of the bulk heat flux (PGK_HF_KSPACE_*):
        // EWK = the -D_HF_BULK_EWK build (calforce_hf.F90:1046-1062)
        int kspace = 0, kmax = 0;
        bool ewk_now = false;      // this force evaluation is the heat-flux step's
        bool ewk_fresh = false;    // ewk_pot / ewk_vir hold ewaldkp_hf at the current positions
        std::vector<double> ewk_pot, ewk_vir;
    } hf;
};

// ---- spline_interp.F90:139-190 cal_spl_coeff ----
void cal_spl_coeff(const Oracle& o, const std::vector<double>& t, std::vector<double>& b,
                   std::vector<double>& c, std::vector<double>& d) {
    int n = o.nspl; double h = o.hspl;
    std::vector<double> al(n, 0.0), l(n, 0.0), mu(n, 0.0), z(n, 0.0);
    b.assign(n, 0.0); c.assign(n, 0.0); d.assign(n, 0.0);
    for (int i = 1; i < n - 1; ++i) al[i] = 3.0 / h * ((t[i + 1] - t[i]) - (t[i] - t[i - 1]));
    l[0] = 1.0; mu[0] = 0.0; z[0] = 0.0;
    for (int i = 1; i < n - 1; ++i) {
        l[i] = 2.0 * (o.xtbl[i + 1] - o.xtbl[i - 1]) - h * mu[i - 1];
        mu[i] = h / l[i];
        z[i] = (al[i] - h * z[i - 1]) / l[i];
    }
    l[n - 1] = 1.0; z[n - 1] = 0.0; c[n - 1] = 0.0;
    for (int i = n - 2; i >= 0; --i) {
        c[i] = z[i] - mu[i] * c[i + 1];
        b[i] = (t[i + 1] - t[i]) / h - h * (c[i + 1] + 2.0 * c[i]) / 3.0;
        d[i] = (c[i + 1] - c[i]) / (3.0 * h);
    }
}

// ---- spline_interp.F90:14-136 spline_interp_init ----
void spline_init(Oracle& o) {
    o.nspl = o.prm.nspltbl > 0 ? o.prm.nspltbl : 1100;
    double rootpi = std::sqrt(std::acos(-1.0));
    double alpha = o.prm.alpha;
    double piE = 2.0 / rootpi * alpha;
    o.hspl = (o.prm.rrcut + 2.0) / (double)o.nspl;
    o.xtbl.resize(o.nspl);
    for (int i = 0; i < o.nspl; ++i) o.xtbl[i] = (double)i * o.hspl;
    for (int k = 0; k < 4; ++k) o.tb[k].assign(o.nspl, 0.0);
    for (int k = 0; k < 4; ++k) o.tb[k][0] = 1.0;
    for (int i = 1; i < o.nspl; ++i) {
        double r = o.xtbl[i], inv = 1.0 / r, arg = alpha * r;
        double ec = std::erfc(arg), ex = std::exp(-arg * arg);
        o.tb[0][i] = inv * (piE * ex * inv + ec * inv * inv);
        o.tb[1][i] = ec * inv;
        o.tb[2][i] = inv * (-piE * ex * inv + (1.0 - ec) * inv * inv);
        o.tb[3][i] = (1.0 - ec) * inv;
    }
    for (int k = 0; k < 4; ++k) cal_spl_coeff(o, o.tb[k], o.sb[k], o.sc[k], o.sd[k]);
}

// ---- spline_interp.F90:196-242 SPLINE_INTERPFUNC ----
inline double spl(const Oracle& o, int k, double x) {
    if (x >= o.hspl * (double)(o.nspl - 1)) return 0.0;
    int idx = (int)(x / o.hspl);
    double d = x - o.xtbl[idx];
    return o.tb[k][idx] + d * (o.sb[k][idx] + d * (o.sc[k][idx] + d * o.sd[k][idx]));
}

// ---- fft_pme_init.F90:216-260 fill_bspline ----
void fill_bspline(double w, int order, double* arr, double* darr) {
    arr[order - 1] = 0.0;
    arr[1] = w;
    arr[0] = 1.0 - w;
    for (int k = 3; k <= order - 1; ++k) {
        double div = 1.0 / (double)(k - 1);
        arr[k - 1] = div * w * arr[k - 2];
        for (int j = 1; j <= k - 2; ++j)
            arr[k - j - 1] = div * ((w + j) * arr[k - j - 2] + (k - j - w) * arr[k - j - 1]);
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

// ---- fft_pme_init.F90:263-289 DFTMOD ----
void dftmod(std::vector<double>& mod, const std::vector<double>& arr, int n) {
    mod.assign(n, 0.0);
    double twopi = 2.0 * 3.14159265358979323846;
    for (int k = 0; k < n; ++k) {
        double s1 = 0, s2 = 0;
        for (int j = 0; j < n; ++j) {
            double arg = twopi * (double)k * (double)j / (double)n;
            s1 += arr[j] * std::cos(arg);
            s2 += arr[j] * std::sin(arg);
        }
        mod[k] = s1 * s1 + s2 * s2;
    }
    for (int k = 0; k < n; ++k)
        if (mod[k] < 1.0e-7 && k > 0 && k < n - 1) mod[k] = 0.5 * (mod[k - 1] + mod[k + 1]);
}

// ---- erf_corr_cutoff.F90:28-62 (the reference's min-ish rule kept) ----
double erf_corr_cutoff(const double* box, int n1, int n2, int n3) {
    double aux = 0.5;
    double m1 = aux * (n1 / box[0]);
    double rk = m1;
    double m2 = aux * (n2 / box[1]);
    if (m2 < m1) rk = m2;
    double m3 = aux * (n3 / box[2]);
    if (m3 < m2) rk = m3;
    return 0.9 * rk;
}

void spme_init(Oracle& o) {
    int order = o.prm.pme_order;
    int nmax = std::max(o.prm.nfft1, std::max(o.prm.nfft2, o.prm.nfft3));
    double arr[16], darr[16];
    fill_bspline(0.0, order, arr, darr);
    std::vector<double> bsp_arr((size_t)nmax + order + 2, 0.0);
    for (int i = 2; i <= order + 1; ++i) bsp_arr[i - 1] = arr[i - 2];
    int nf[3] = {o.prm.nfft1, o.prm.nfft2, o.prm.nfft3};
    for (int d = 0; d < 3; ++d) {
        std::vector<double> a(bsp_arr.begin(), bsp_arr.begin() + nf[d]);
        dftmod(o.bsp[d], a, nf[d]);
    }
    double pi = std::acos(-1.0), s = 0;
    for (int i = 0; i < o.natom; ++i) s += o.atmchrg[i] * o.atmchrg[i];
    o.pot_ewc = -1.0 / std::sqrt(pi) * o.prm.alpha * s;   // fft_pme_init.F90:147-156
    double q = 0;
    for (int i = 0; i < o.natom; ++i) q += o.atmchrg[i];
    o.netchrgsq = q * q;
}

// --------------------------------------------------------------------------
// mklist2a (mklist.F90:8-234) and mklist_cell (mklist_cell.F90:8-352)
// --------------------------------------------------------------------------
inline bool pair_in(const Oracle& o, int i, int j, double sqcut) {
    double rij[3];
    for (int d = 0; d < 3; ++d) {
        double r = o.atmcor[3 * i + d] - o.atmcor[3 * j + d];
        double binv = 1.0 / o.box[d];
        rij[d] = r - o.box[d] * dnint(r * binv);
    }
    double dr = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
    return dr < sqcut;
}

void finish_row(Oracle& o, int i, std::vector<int>& tmp, std::vector<int>& idx,
                std::vector<int>& lst) {
    // delete excluded atoms (mklist_cell.F90:283-293)
    int ix1 = o.excl_idx[i] - 1, ix2 = o.excl_idx[i + 1] - 2;
    int kept = (int)tmp.size();
    for (size_t a = 0; a < tmp.size(); ++a)
        for (int ix = ix1; ix <= ix2; ++ix)
            if (tmp[a] == o.excl_list[ix]) { tmp[a] = -999; --kept; break; }
    idx[i] = (int)lst.size() + 1;
    if (kept == 0) { lst.push_back(0); return; }
    for (int v : tmp) if (v > 0) lst.push_back(v);
}

// rdscript.F90:1595-1610: the cell index is refused when a cell count is < 3
// or the total number of cells is <= 27; mklist2a runs instead.
int choose_list_mode(const Oracle& o) {
    if (o.prm.list_mode == PGK_LIST_CELL) return PGK_LIST_CELL;
    if (o.prm.list_mode == PGK_LIST_ALLPAIR) return PGK_LIST_ALLPAIR;
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = (int)(o.box[d] / o.prm.rcut_book);
    if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3 || (long long)nc[0] * nc[1] * nc[2] <= 27)
        return PGK_LIST_ALLPAIR;
    return PGK_LIST_CELL;
}

// Morse list (rows per Morse atom, partners 0-based).  mklist2a_mor
// (mklist_mor.F90:30-120): for each Morse atom the later Morse atoms of a
// Morse type pair inside rcut_bookmor (minimum image), in atom order; without
// a list radius the half-box diagonal is the radius (mklist_mor.F90:30-34).
// mklist_mor_cell (mklist_mor_cell.F90:8-327): the same test over the 27-cell
// stencil (z, y, x order; cell = MOD(INT((x+L)/cs), nc); j > i by atom
// index), used when every cell count is >= 3 and there are more than 27 cells
// (rdscript.F90:1616-1632); list_mode forces either order as for the pair list.
void mklist_mor(Oracle& o) {
    double sqcut = o.prm.rcut_bookmor * o.prm.rcut_bookmor;
    if (o.prm.rcut_bookmor <= 0.0)
        sqcut = (o.box[0] / 2.0) * (o.box[0] / 2.0) + (o.box[1] / 2.0) * (o.box[1] / 2.0) +
                (o.box[2] / 2.0) * (o.box[2] / 2.0);
    const int nm = (int)o.mor_atoms.size();
    o.mor_idx.assign((size_t)nm + 1, 0);
    o.mor_list.clear();
    auto test = [&](int i, int j) {
        if (o.inttyp[o.atmindex[i] + o.ntyp * o.atmindex[j]] != 2) return false;
        double rij[3];
        for (int d = 0; d < 3; ++d) {
            double v = o.atmcor[3 * i + d] - o.atmcor[3 * j + d];
            rij[d] = v - o.box[d] * dnint(v * (1.0 / o.box[d]));
        }
        double dr = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
        return dr < sqcut;
    };
    int nc[3] = {0, 0, 0};
    bool cell = o.prm.rcut_bookmor > 0.0 && o.prm.list_mode != PGK_LIST_ALLPAIR;
    if (cell) {
        for (int d = 0; d < 3; ++d) nc[d] = (int)(o.box[d] / o.prm.rcut_bookmor);
        if (o.prm.list_mode != PGK_LIST_CELL &&
            (nc[0] < 3 || nc[1] < 3 || nc[2] < 3 || (long long)nc[0] * nc[1] * nc[2] <= 27))
            cell = false;
    }
    o.mor_list_mode = cell ? PGK_LIST_CELL : PGK_LIST_ALLPAIR;
    if (!cell) {
        for (int m1 = 0; m1 < nm; ++m1) {
            o.mor_idx[m1] = (int)o.mor_list.size();
            const int i = o.mor_atoms[m1];
            for (int m2 = m1 + 1; m2 < nm; ++m2)
                if (test(i, o.mor_atoms[m2])) o.mor_list.push_back(o.mor_atoms[m2]);
        }
        o.mor_idx[nm] = (int)o.mor_list.size();
        return;
    }
    double cs[3];
    for (int d = 0; d < 3; ++d) cs[d] = o.box[d] / (double)nc[d];
    std::vector<int> a2c((size_t)3 * nm);
    std::vector<std::vector<int>> cellv((size_t)nc[0] * nc[1] * nc[2]);
    for (int m = 0; m < nm; ++m) {
        const int i = o.mor_atoms[m];
        for (int d = 0; d < 3; ++d) a2c[3 * m + d] = ((int)((o.atmcor[3 * i + d] + o.box[d]) / cs[d])) % nc[d];
        cellv[a2c[3 * m] + (size_t)nc[0] * (a2c[3 * m + 1] + (size_t)nc[1] * a2c[3 * m + 2])].push_back(i);
    }
    for (int m1 = 0; m1 < nm; ++m1) {
        o.mor_idx[m1] = (int)o.mor_list.size();
        const int i = o.mor_atoms[m1];
        for (int z1 = a2c[3 * m1 + 2] - 1; z1 <= a2c[3 * m1 + 2] + 1; ++z1) {
            const int z = (z1 + nc[2]) % nc[2];
            for (int y1 = a2c[3 * m1 + 1] - 1; y1 <= a2c[3 * m1 + 1] + 1; ++y1) {
                const int y = (y1 + nc[1]) % nc[1];
                const size_t posyz = (size_t)y * nc[0] + (size_t)z * nc[0] * nc[1];
                for (int x1 = a2c[3 * m1] - 1; x1 <= a2c[3 * m1] + 1; ++x1) {
                    const int x = (x1 + nc[0]) % nc[0];
                    for (int j : cellv[x + posyz])
                        if (i < j && test(i, j)) o.mor_list.push_back(j);
                }
            }
        }
    }
    o.mor_idx[nm] = (int)o.mor_list.size();
}

void mklist(Oracle& o) {
    if (!o.welmor.empty()) mklist_mor(o);
    int n = o.natom;
    double sqcut = o.prm.rcut_book * o.prm.rcut_book;
    int mode = choose_list_mode(o);
    o.list_used_mode = mode;
    std::vector<std::vector<int>> rows((size_t)std::max(n - 1, 0));
    if (mode == PGK_LIST_ALLPAIR) {
        par_chunks(o.nthreads, n - 1, [&](long long b, long long e, int) {
            for (long long i = b; i < e; ++i) {
                std::vector<int>& t = rows[i];
                for (int j = (int)i + 1; j < n; ++j)
                    if (pair_in(o, (int)i, j, sqcut)) t.push_back(j + 1);
            }
        });
    } else {
        int nc[3]; double cs[3];
        for (int d = 0; d < 3; ++d) { nc[d] = (int)(o.box[d] / o.prm.rcut_book); cs[d] = o.box[d] / (double)nc[d]; }
        std::vector<int> a2c((size_t)3 * n);
        long long ncell = (long long)nc[0] * nc[1] * nc[2];
        std::vector<std::vector<int>> cell((size_t)ncell);
        for (int i = 0; i < n; ++i) {
            for (int d = 0; d < 3; ++d)
                a2c[3 * i + d] = ((int)((o.atmcor[3 * i + d] + o.box[d]) / cs[d])) % nc[d];
            long long c = a2c[3 * i] + (long long)nc[0] * (a2c[3 * i + 1] + (long long)nc[1] * a2c[3 * i + 2]);
            cell[c].push_back(i);
        }
        par_chunks(o.nthreads, n - 1, [&](long long b, long long e, int) {
        for (int i = (int)b; i < (int)e; ++i) {
            std::vector<int>& t = rows[i];
            for (int z1 = a2c[3 * i + 2] - 1; z1 <= a2c[3 * i + 2] + 1; ++z1) {
                int z = (z1 + nc[2]) % nc[2];
                for (int y1 = a2c[3 * i + 1] - 1; y1 <= a2c[3 * i + 1] + 1; ++y1) {
                    int y = (y1 + nc[1]) % nc[1];
                    long long posyz = (long long)y * nc[0] + (long long)z * nc[0] * nc[1];
                    for (int x1 = a2c[3 * i] - 1; x1 <= a2c[3 * i] + 1; ++x1) {
                        int x = (x1 + nc[0]) % nc[0];
                        for (int j : cell[x + posyz]) {
                            if (i >= j) continue;
                            if (pair_in(o, i, j, sqcut)) t.push_back(j + 1);
                        }
                    }
                }
            }
        }
        });
    }
    std::vector<int> idx((size_t)n + 1, 0), lst;
    for (int i = 0; i < n - 1; ++i) finish_row(o, i, rows[i], idx, lst);
    o.nlistnball = (long long)lst.size();
    idx[std::max(n - 1, 0)] = (int)o.nlistnball + 1;   // "non-existence last loop index i"
    o.nb_index.swap(idx);
    o.nb_list.swap(lst);
}

// --------------------------------------------------------------------------
// ewaldrp (ewaldr.F90:404-838), spline mode, no Fennell
// --------------------------------------------------------------------------
struct NBOut {
    std::vector<double> felc, fvdw;
    double pot_elc = 0, pot_vdw = 0, pvc = 0, pvlj = 0;
    double vtc[9] = {0}, vtlj[9] = {0};
};

void ewaldrp(Oracle& o, double* force, pgk_energies* e, pgk_virials* v) {
    int n = o.natom;
    double sqcut = o.prm.rrcut * o.prm.rrcut, sqcut2 = o.prm.rcut * o.prm.rcut;
    if (sqcut2 > sqcut) sqcut = sqcut2;
    double rrcut = o.prm.rrcut;
    double binv[3] = {1.0 / o.box[0], 1.0 / o.box[1], 1.0 / o.box[2]};
    int nt = std::max(1, o.nthreads);
    std::vector<NBOut> outs((size_t)nt);
    for (auto& ob : outs) { ob.felc.assign((size_t)3 * n, 0.0); ob.fvdw.assign((size_t)3 * n, 0.0); }
    int rows = n - 1;
    par_chunks(nt, rows, [&](long long b, long long e_, int tid) {
        NBOut& ob = outs[tid];
        for (int i = (int)b; i < (int)e_; ++i) {
            int j1 = o.nb_index[i] - 1, j2 = o.nb_index[i + 1] - 2;
            int it = o.atmindex[i];
            if (o.nb_list[j1] == 0) continue;
            for (int jx = j1; jx <= j2; ++jx) {
                int jj = o.nb_list[jx] - 1;
                double rij[3];
                for (int d = 0; d < 3; ++d) {
                    double r = o.atmcor[3 * i + d] - o.atmcor[3 * jj + d];
                    rij[d] = r - o.box[d] * dnint(r * binv[d]);
                }
                double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
                if (r2 > sqcut) continue;
                double rinv2 = 1.0 / r2;
                double r = std::sqrt(r2);
                if (r <= rrcut) {
                    double qq = o.atmchrg[i] * o.atmchrg[jj];
                    double ftmp = spl(o, 0, r) * qq;
                    double potij = spl(o, 1, r) * qq;
                    ob.pot_elc += potij;
                    double f[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
                    for (int d = 0; d < 3; ++d) { ob.felc[3 * i + d] += f[d]; ob.felc[3 * jj + d] -= f[d]; }
                    for (int nn = 0; nn < 3; ++nn)
                        for (int a = 0; a < 3; ++a) ob.vtc[a + 3 * nn] += f[a] * rij[nn];
                    ob.pvc += potij;
                }
                if (r2 <= sqcut2) {
                    int jt = o.atmindex[jj];
                    if (!o.inttyp.empty() && o.inttyp[it + o.ntyp * jt] != 1) continue;
                    double R = o.radij[it + o.ntyp * jt];
                    double t2 = rinv2 * (R * R);
                    double t6 = t2 * t2 * t2, t12 = t6 * t6;
                    double E = o.welij[it + o.ntyp * jt];
                    double potij = E * (t12 - 2.0 * t6);
                    ob.pot_vdw += potij;
                    double ftmp = 12.0 * E * (t12 - t6) * rinv2;
                    double f[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
                    for (int d = 0; d < 3; ++d) { ob.fvdw[3 * i + d] += f[d]; ob.fvdw[3 * jj + d] -= f[d]; }
                    for (int nn = 0; nn < 3; ++nn)
                        for (int a = 0; a < 3; ++a) ob.vtlj[a + 3 * nn] += f[a] * rij[nn];
                    ob.pvlj += f[0] * rij[0] + f[1] * rij[1] + f[2] * rij[2];
                }
            }
        }
    });
    NBOut& o0 = outs[0];
    for (int t = 1; t < nt; ++t) {
        for (size_t k = 0; k < o0.felc.size(); ++k) { o0.felc[k] += outs[t].felc[k]; o0.fvdw[k] += outs[t].fvdw[k]; }
        o0.pot_elc += outs[t].pot_elc; o0.pot_vdw += outs[t].pot_vdw;
        o0.pvc += outs[t].pvc; o0.pvlj += outs[t].pvlj;
        for (int k = 0; k < 9; ++k) { o0.vtc[k] += outs[t].vtc[k]; o0.vtlj[k] += outs[t].vtlj[k]; }
    }
    // excluded neighbours (ewaldr.F90:756-826)
    for (int i = 0; i < n - 1; ++i) {
        int j1 = o.excl_idx[i] - 1, j2 = o.excl_idx[i + 1] - 2;
        if (o.excl_list[j1] == 0) continue;
        for (int jx = j1; jx <= j2; ++jx) {
            int jj = o.excl_list[jx] - 1;
            double rij[3];
            for (int d = 0; d < 3; ++d) {
                double r = o.atmcor[3 * i + d] - o.atmcor[3 * jj + d];
                rij[d] = r - o.box[d] * dnint(r * binv[d]);
            }
            double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            double r = std::sqrt(r2);
            double qq = o.atmchrg[i] * o.atmchrg[jj];
            double ftmp = -spl(o, 2, r) * qq;
            double potij = spl(o, 3, r) * qq;
            o0.pot_elc -= potij;
            o0.pvc -= potij;
            double f[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
            for (int d = 0; d < 3; ++d) { o0.felc[3 * i + d] += f[d]; o0.felc[3 * jj + d] -= f[d]; }
            for (int nn = 0; nn < 3; ++nn)
                for (int a = 0; a < 3; ++a) o0.vtc[a + 3 * nn] += f[a] * rij[nn];
        }
    }
    for (int k = 0; k < 3 * n; ++k) force[k] = force[k] + o0.fvdw[k] + o0.felc[k];
    if (e) { e->pot_elc = o0.pot_elc; e->pot_vdw = o0.pot_vdw; }
    if (v) {
        v->pot_viri_coul += o0.pvc; v->pot_viri_lj += o0.pvlj;
        for (int k = 0; k < 9; ++k) { v->pot_virit_coul[k] += o0.vtc[k]; v->pot_virit_lj[k] += o0.vtlj[k]; }
    }
}

// --------------------------------------------------------------------------
// fft_pmep (fft_pme.F90:144-270) + helpers :273-937
// --------------------------------------------------------------------------
// get_scaled_fractionals + get_bspline_coeffs (fft_pme.F90:273-356): scaled
// fractional coordinates fr (3,N) and B-spline weights th, dth (p,3,N)
void spme_bspline(const Oracle& o, std::vector<double>& fr, std::vector<double>& th, std::vector<double>& dth) {
    int n = o.natom, p = o.prm.pme_order;
    int Kd[3] = {o.prm.nfft1, o.prm.nfft2, o.prm.nfft3};
    double recip[3] = {1.0 / o.box[0], 1.0 / o.box[1], 1.0 / o.box[2]};
    fr.assign((size_t)3 * n, 0.0); th.assign((size_t)3 * p * n, 0.0); dth.assign((size_t)3 * p * n, 0.0);
    for (int a = 0; a < n; ++a)
        for (int d = 0; d < 3; ++d) {
            double w = o.atmcor[3 * a + d] * recip[d];           // get_scaled_fractionals
            w = w - std::floor(w);
            fr[3 * a + d] = Kd[d] * w;
            double ww = fr[3 * a + d] - std::trunc(fr[3 * a + d]);  // get_bspline_coeffs (dint)
            fill_bspline(ww, p, &th[((size_t)3 * a + d) * p], &dth[((size_t)3 * a + d) * p]);
        }
}

inline int spme_wrap(int k0, int K) { return k0 >= 0 ? k0 : k0 + K; }

// fill_charge_grid (fft_pme.F90:359-422): Q(re) += q theta1 theta2 theta3
void spme_spread(const Oracle& o, const std::vector<double>& fr, const std::vector<double>& th, std::vector<cplx>& Q) {
    int n = o.natom, p = o.prm.pme_order;
    int K1 = o.prm.nfft1, K2 = o.prm.nfft2, K3 = o.prm.nfft3;
    Q.assign((size_t)K1 * K2 * K3, cplx(0, 0));
    for (int a = 0; a < n; ++a) {
        const double* t1 = &th[((size_t)3 * a + 0) * p];
        const double* t2 = &th[((size_t)3 * a + 1) * p];
        const double* t3 = &th[((size_t)3 * a + 2) * p];
        int k0 = (int)fr[3 * a + 2] - p;
        for (int i3 = 0; i3 < p; ++i3) {
            k0 += 1;
            int k = spme_wrap(k0, K3);
            double prod1 = t3[i3] * o.atmchrg[a];
            int j0 = (int)fr[3 * a + 1] - p;
            for (int i2 = 0; i2 < p; ++i2) {
                j0 += 1;
                int j = spme_wrap(j0, K2);
                double prod = t2[i2] * prod1;
                int ii0 = (int)fr[3 * a] - p;
                for (int i1 = 0; i1 < p; ++i1) {
                    ii0 += 1;
                    int i = spme_wrap(ii0, K1);
                    Q[(size_t)i + (size_t)K1 * (j + (size_t)K2 * k)] += t1[i1] * prod;
                }
            }
        }
    }
}

// pubz3d: x, y, z passes of cfftf (sign -1) or cfftb (sign +1)
void spme_fft3(const Oracle& o, std::vector<cplx>& Q, int sign) {
    int K1 = o.prm.nfft1, K2 = o.prm.nfft2, K3 = o.prm.nfft3;
    par_chunks(o.nthreads, K3, [&](long long b, long long e_, int) {
        for (long long k = b; k < e_; ++k)
            for (int j = 0; j < K2; ++j) fft1d(&Q[(size_t)K1 * (j + (size_t)K2 * k)], K1, 1, sign);
    });
    par_chunks(o.nthreads, K3, [&](long long b, long long e_, int) {
        for (long long k = b; k < e_; ++k)
            for (int i = 0; i < K1; ++i) fft1d(&Q[(size_t)i + (size_t)K1 * K2 * k], K2, K1, sign);
    });
    par_chunks(o.nthreads, K2, [&](long long b, long long e_, int) {
        for (long long j = b; j < e_; ++j)
            for (int i = 0; i < K1; ++i) fft1d(&Q[(size_t)i + (size_t)K1 * j], K3, K1 * K2, sign);
    });
}

void fft_pmep(Oracle& o, double* force, pgk_energies* e, pgk_virials* v) {
    int n = o.natom, p = o.prm.pme_order;
    int K1 = o.prm.nfft1, K2 = o.prm.nfft2, K3 = o.prm.nfft3;
    double recip[3] = {1.0 / o.box[0], 1.0 / o.box[1], 1.0 / o.box[2]};
    double vol = o.box[0] * o.box[1] * o.box[2];
    std::vector<double> fr, th, dth;
    spme_bspline(o, fr, th, dth);
    size_t KK = (size_t)K1 * K2 * K3;
    std::vector<cplx> Q;
    spme_spread(o, fr, th, Q);
    auto wrap = spme_wrap;
    auto pass3 = [&](int sign) { spme_fft3(o, Q, sign); };
    // fft_back = pubz3d(isign=-1)
    pass3(-1);
    // scalar_sum :544-690
    double pi = 3.14159265358979323846;
    double rk2 = o.rkcut * o.rkcut;
    double fac = pi * pi / (o.prm.alpha * o.prm.alpha);
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    double energy = 0, vsca = 0, vt[6] = {0, 0, 0, 0, 0, 0};
    bool corr = o.prm.ifnetqcorrp != 0;
    for (size_t ind = 1; ind < KK; ++ind) {
        int k3 = (int)(ind / ((size_t)K1 * K2));
        size_t jnd = ind - (size_t)k3 * K1 * K2;
        int k2 = (int)(jnd / K1), k1 = (int)(jnd - (size_t)k2 * K1);
        int m1 = k1 < nf1 ? k1 : k1 - K1;
        int m2 = k2 < nf2 ? k2 : k2 - K2;
        int m3 = k3 < nf3 ? k3 : k3 - K3;
        double h1 = recip[0] * m1, h2 = recip[1] * m2, h3 = recip[2] * m3;
        double msq = h1 * h1 + h2 * h2 + h3 * h3;
        double eterm;
        if (msq > rk2) {
            eterm = 0.0;
        } else {
            double denom = pi * vol * o.bsp[0][k1] * o.bsp[1][k2] * o.bsp[2][k3] * msq;
            double vterm = 2.0 * (fac * msq + 1.0) / msq;
            double s2 = std::norm(Q[ind]);
            if (!corr) {
                eterm = std::exp(-fac * msq) / denom;
                double es = eterm * s2;
                energy += es;
                vt[0] += es * (vterm * h1 * h1 - 1.0);
                vt[1] += es * (vterm * h1 * h2);
                vt[2] += es * (vterm * h1 * h3);
                vt[3] += es * (vterm * h2 * h2 - 1.0);
                vt[4] += es * (vterm * h2 * h3);
                vt[5] += es * (vterm * h3 * h3 - 1.0);
            } else {
                double e2 = std::exp(-fac * msq);
                eterm = e2 / denom;
                e2 = e2 * o.netchrgsq / (pi * vol * msq);
                double e3 = e2 * (-1.0 + 2.0 * fac * msq);
                energy += eterm * s2;
                vsca += e3;
                double es = eterm * s2 - e2;
                vt[0] += es * (vterm * h1 * h1 - 1.0);
                vt[1] += es * (vterm * h1 * h2);
                vt[2] += es * (vterm * h1 * h3);
                vt[3] += es * (vterm * h2 * h2 - 1.0);
                vt[4] += es * (vterm * h2 * h3);
                vt[5] += es * (vterm * h3 * h3 - 1.0);
            }
        }
        Q[ind] *= eterm;
    }
    double pot_ewk = 0.5 * energy;
    vsca *= 0.5;
    pass3(+1);
    // grad_sum :872-937
    std::vector<double> fadd((size_t)3 * n);
    par_chunks(o.nthreads, n, [&](long long b_, long long e_, int) {
    for (int a = (int)b_; a < (int)e_; ++a) {
        const double* t1 = &th[((size_t)3 * a + 0) * p];
        const double* t2 = &th[((size_t)3 * a + 1) * p];
        const double* t3 = &th[((size_t)3 * a + 2) * p];
        const double* d1 = &dth[((size_t)3 * a + 0) * p];
        const double* d2 = &dth[((size_t)3 * a + 1) * p];
        const double* d3 = &dth[((size_t)3 * a + 2) * p];
        double f[3] = {0, 0, 0};
        int k0 = (int)fr[3 * a + 2] - p;
        for (int i3 = 0; i3 < p; ++i3) {
            k0 += 1;
            int k = wrap(k0, K3);
            int j0 = (int)fr[3 * a + 1] - p;
            for (int i2 = 0; i2 < p; ++i2) {
                j0 += 1;
                int j = wrap(j0, K2);
                int ii0 = (int)fr[3 * a] - p;
                for (int i1 = 0; i1 < p; ++i1) {
                    ii0 += 1;
                    int i = wrap(ii0, K1);
                    double term = o.atmchrg[a] * Q[(size_t)i + (size_t)K1 * (j + (size_t)K2 * k)].real();
                    f[0] = f[0] - K1 * term * d1[i1] * t2[i2] * t3[i3];
                    f[1] = f[1] - K2 * term * t1[i1] * d2[i2] * t3[i3];
                    f[2] = f[2] - K3 * term * t1[i1] * t2[i2] * d3[i3];
                }
            }
        }
        for (int d = 0; d < 3; ++d) fadd[3 * a + d] = recip[d] * f[d];
    }
    });
    for (int k = 0; k < 3 * n; ++k) force[k] += fadd[k];
    if (e) e->pot_ewk = pot_ewk;
    if (v) {
        double vfull[9] = {vt[0], vt[1], vt[2], vt[1], vt[3], vt[4], vt[2], vt[4], vt[5]};
        for (int k = 0; k < 9; ++k) v->pot_virit_coul[k] -= 0.5 * vfull[k];
        v->pot_viri_coul += pot_ewk + vsca;
    }
}

// Per-atom split of fft_pmep's reciprocal energy and virial tensor for the
// bulk heat flux: the SPME form of ewaldkp_hf's per-atom terms
// (ewaldk_hf.F90:165-173, :212-230), which the reference has only for
// standard Ewald.  With S = FFT(Q) and the influence function eterm of
// scalar_sum (fft_pme.F90:544-690),
//   pot_atm(i)      = 1/2 q_i sum_g theta_i(g) IFFT(eterm S)(g) - alpha/sqrt(pi) q_i^2
//   viri_atm(a,b,i) = 1/2 q_i sum_g theta_i(g) IFFT(eterm (delta_ab - vterm h_a h_b) S)(g)
// so the atoms' energies (less the self term) sum to pot_ewk and their
// tensors to fft_pmep's pot_virit_coul (before the net-charge terms, which
// are global and not split).  viri_atm is (3,3,N), [a + 3b + 9i].
void spme_hf_atm(Oracle& o, double* pot_atm, double* viri_atm) {
    int n = o.natom, p = o.prm.pme_order;
    int K1 = o.prm.nfft1, K2 = o.prm.nfft2, K3 = o.prm.nfft3;
    double recip[3] = {1.0 / o.box[0], 1.0 / o.box[1], 1.0 / o.box[2]};
    double vol = o.box[0] * o.box[1] * o.box[2];
    std::vector<double> fr, th, dth;
    spme_bspline(o, fr, th, dth);
    std::vector<cplx> Q;
    spme_spread(o, fr, th, Q);
    spme_fft3(o, Q, -1);
    const size_t KK = (size_t)K1 * K2 * K3;
    // grids: 0 potential, 1..6 tensor xx xy xz yy yz zz
    std::vector<std::vector<cplx>> G(7, std::vector<cplx>(KK, cplx(0, 0)));
    const double pi = 3.14159265358979323846;
    const double rk2 = o.rkcut * o.rkcut, fac = pi * pi / (o.prm.alpha * o.prm.alpha);
    int nf1 = K1 / 2; if (2 * nf1 < K1) ++nf1;
    int nf2 = K2 / 2; if (2 * nf2 < K2) ++nf2;
    int nf3 = K3 / 2; if (2 * nf3 < K3) ++nf3;
    for (size_t ind = 1; ind < KK; ++ind) {
        int k3 = (int)(ind / ((size_t)K1 * K2));
        size_t jnd = ind - (size_t)k3 * K1 * K2;
        int k2 = (int)(jnd / K1), k1 = (int)(jnd - (size_t)k2 * K1);
        int m1 = k1 < nf1 ? k1 : k1 - K1;
        int m2 = k2 < nf2 ? k2 : k2 - K2;
        int m3 = k3 < nf3 ? k3 : k3 - K3;
        double h[3] = {recip[0] * m1, recip[1] * m2, recip[2] * m3};
        double msq = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
        if (msq > rk2) continue;
        double denom = pi * vol * o.bsp[0][k1] * o.bsp[1][k2] * o.bsp[2][k3] * msq;
        double eterm = std::exp(-fac * msq) / denom;
        double vterm = 2.0 * (fac * msq + 1.0) / msq;
        cplx es = eterm * Q[ind];
        G[0][ind] = es;
        const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
        for (int c = 0; c < 6; ++c) {
            int a = ab[c][0], b = ab[c][1];
            G[1 + c][ind] = es * ((a == b ? 1.0 : 0.0) - vterm * h[a] * h[b]);
        }
    }
    for (int c = 0; c < 7; ++c) spme_fft3(o, G[c], +1);
    const double self = o.prm.alpha / std::sqrt(pi);
    par_chunks(o.nthreads, n, [&](long long b_, long long e_, int) {
        for (int a = (int)b_; a < (int)e_; ++a) {
            const double* t1 = &th[((size_t)3 * a + 0) * p];
            const double* t2 = &th[((size_t)3 * a + 1) * p];
            const double* t3 = &th[((size_t)3 * a + 2) * p];
            double acc[7] = {0, 0, 0, 0, 0, 0, 0};
            int k0 = (int)fr[3 * a + 2] - p;
            for (int i3 = 0; i3 < p; ++i3) {
                k0 += 1;
                int k = spme_wrap(k0, K3);
                int j0 = (int)fr[3 * a + 1] - p;
                for (int i2 = 0; i2 < p; ++i2) {
                    j0 += 1;
                    int j = spme_wrap(j0, K2);
                    int ii0 = (int)fr[3 * a] - p;
                    for (int i1 = 0; i1 < p; ++i1) {
                        ii0 += 1;
                        int i = spme_wrap(ii0, K1);
                        size_t g = (size_t)i + (size_t)K1 * (j + (size_t)K2 * k);
                        double w = t1[i1] * t2[i2] * t3[i3];
                        for (int c = 0; c < 7; ++c) acc[c] += w * G[c][g].real();
                    }
                }
            }
            const double hq = 0.5 * o.atmchrg[a];
            if (pot_atm) pot_atm[a] = hq * acc[0] - self * (o.atmchrg[a] * o.atmchrg[a]);
            if (viri_atm) {
                double* v = viri_atm + (size_t)9 * a;
                v[0] = hq * acc[1]; v[1] = hq * acc[2]; v[2] = hq * acc[3];
                v[3] = v[1];        v[4] = hq * acc[4]; v[5] = hq * acc[5];
                v[6] = v[2];        v[7] = v[5];        v[8] = hq * acc[6];
            }
        }
    });
}

// --------------------------------------------------------------------------
// bonded terms
// --------------------------------------------------------------------------
inline void mi(const Oracle& o, int a, int b, double* r) {  // r = x_a - x_b, min image (anint)
    for (int d = 0; d < 3; ++d) {
        double v = o.atmcor[3 * a + d] - o.atmcor[3 * b + d];
        r[d] = v - o.box[d] * dnint(v * (1.0 / o.box[d]));
    }
}
inline void cross(const double* x, const double* y, double* z) {   // caltors.F90:478-492
    z[0] = x[1] * y[2] - x[2] * y[1];
    z[1] = x[2] * y[0] - x[0] * y[2];
    z[2] = x[0] * y[1] - x[1] * y[0];
}
inline double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// calbondp (calbond.F90:109-219)
void calbondp(Oracle& o, double* force, double& pot, double& vs, double* vt) {
    pot = 0;
    for (size_t k = 0; k < o.bi.size(); ++k) {
        if (std::fabs(o.bk[k]) < 1.0e-16) continue;
        int i = o.bi[k], j = o.bj[k];
        double rij[3]; mi(o, i, j, rij);
        double r = std::sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        pot += o.bk[k] * (r - o.br0[k]) * (r - o.br0[k]);
        double fa = -2.0 * o.bk[k] * (r - o.br0[k]);
        double f[3] = {fa * rij[0] / r, fa * rij[1] / r, fa * rij[2] / r};
        for (int d = 0; d < 3; ++d) { force[3 * i + d] += f[d]; force[3 * j + d] -= f[d]; }
        vs += f[0] * rij[0] + f[1] * rij[1] + f[2] * rij[2];
        for (int nn = 0; nn < 3; ++nn) for (int a = 0; a < 3; ++a) vt[a + 3 * nn] += f[a] * rij[nn];
    }
}

// calanglp (calangl.F90:172-358)
void calanglp(Oracle& o, double* force, double& pot, double& vs, double* vt) {
    pot = 0;
    for (size_t n = 0; n < o.ai.size(); ++n) {
        if (std::fabs(o.akk[n]) < 1.0e-32) continue;
        int i = o.ai[n], j = o.aj[n], k = o.ak[n];
        double rij[3], rkj[3];
        mi(o, j, i, rij); mi(o, j, k, rkj);
        double ra = std::sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        double rb = std::sqrt(rkj[0] * rkj[0] + rkj[1] * rkj[1] + rkj[2] * rkj[2]);
        double c = (rij[0] * rkj[0] + rij[1] * rkj[1] + rij[2] * rkj[2]) / (ra * rb);
        if (c > 1.0) c = 1.0; else if (c < -1.0) c = -1.0;
        double th = std::acos(c), s = std::sin(th);
        pot += o.akk[n] * (th - o.at0[n]) * (th - o.at0[n]);
        double fi[3] = {0, 0, 0}, fj[3] = {0, 0, 0}, fk[3] = {0, 0, 0};
        if (std::fabs(s) > 1.0e-14) {
            double ft = -2.0 * o.akk[n] * (th - o.at0[n]) / s;
            for (int d = 0; d < 3; ++d) {
                fi[d] = ft * ((rkj[d] / rb - rij[d] * c / ra) / ra);
                fk[d] = ft * ((rij[d] / ra - rkj[d] * c / rb) / rb);
                fj[d] = -fi[d] - fk[d];
            }
        }
        const int at[3] = {i, j, k};
        const double* fs[3] = {fi, fj, fk};
        for (int q = 0; q < 3; ++q)
            for (int d = 0; d < 3; ++d) force[3 * at[q] + d] += fs[q][d];
        for (int q = 0; q < 3; ++q)
            vs += fs[q][0] * o.atmcor[3 * at[q]] + fs[q][1] * o.atmcor[3 * at[q] + 1] + fs[q][2] * o.atmcor[3 * at[q] + 2];
        for (int l = 0; l < 3; ++l)
            for (int q = 0; q < 3; ++q)
                for (int a = 0; a < 3; ++a) vt[a + 3 * l] += fs[q][a] * o.atmcor[3 * at[q] + l];
    }
}

// shared geometry of calijkl / calijklrb (caltors.F90, caltorsrb.F90:260-459)
struct TorsGeo { double cphi, phi, sphi, b[3], c[3]; };
void tors_geo(const double* rij, const double* rkj, const double* rkl, TorsGeo& g) {
    double nijk[3], njkl[3], t[3];
    cross(rij, rkj, nijk);
    cross(rkj, rkl, njkl);
    double ai = std::sqrt(dot(nijk, nijk)), al = std::sqrt(dot(njkl, njkl));
    double c = dot(nijk, njkl) / (ai * al);
    if (c > 1.0) c = 1.0; else if (c < -1.0) c = -1.0;
    cross(nijk, njkl, t);
    double phi = std::acos(c);
    phi = -std::copysign(phi, dot(rkj, t));    // -sign(phi, rkj.(n1 x n2))
    g.cphi = c; g.phi = phi; g.sphi = std::sin(phi);
    for (int d = 0; d < 3; ++d) { nijk[d] /= ai; njkl[d] /= al; }
    for (int d = 0; d < 3; ++d) {
        g.b[d] = (njkl[d] - c * nijk[d]) / ai;
        g.c[d] = (nijk[d] - c * njkl[d]) / al;
    }
}
void tors_forces(double fa, const TorsGeo& g, const double* rij, const double* rkj, const double* rkl,
                 const double* rik, const double* rjl, double* fi, double* fj, double* fk, double* fl) {
    double t1[3], t2[3];
    cross(g.b, rkj, t1);
    for (int d = 0; d < 3; ++d) fi[d] = fa * t1[d];
    cross(g.c, rkl, t1); cross(g.b, rik, t2);
    for (int d = 0; d < 3; ++d) fj[d] = fa * (-t1[d] + t2[d]);
    cross(g.b, rij, t1); cross(g.c, rjl, t2);
    for (int d = 0; d < 3; ++d) fk[d] = fa * (-t1[d] + t2[d]);
    cross(g.c, rkj, t1);
    for (int d = 0; d < 3; ++d) fl[d] = fa * t1[d];
}
void add4(Oracle& o, double* force, double& vs, double* vt, int i, int j, int k, int l,
          const double* fi, const double* fj, const double* fk, const double* fl) {
    const int at[4] = {i, j, k, l};
    const double* fs[4] = {fi, fj, fk, fl};
    for (int q = 0; q < 4; ++q) for (int d = 0; d < 3; ++d) force[3 * at[q] + d] += fs[q][d];
    for (int q = 0; q < 4; ++q)
        vs += fs[q][0] * o.atmcor[3 * at[q]] + fs[q][1] * o.atmcor[3 * at[q] + 1] + fs[q][2] * o.atmcor[3 * at[q] + 2];
    for (int l2 = 0; l2 < 3; ++l2)
        for (int q = 0; q < 4; ++q)
            for (int a = 0; a < 3; ++a) vt[a + 3 * l2] += fs[q][a] * o.atmcor[3 * at[q] + l2];
}
void tors_vecs(Oracle& o, int i, int j, int k, int l, double* rij, double* rkj, double* rkl,
               double* rik, double* rjl) {
    mi(o, j, i, rij); mi(o, j, k, rkj); mi(o, l, k, rkl); mi(o, k, i, rik); mi(o, l, j, rjl);
}

// caltorsp + calijkl (caltors.F90)
void caltorsp(Oracle& o, double* force, double& pot, double& vs, double* vt) {
    pot = 0;
    for (size_t n = 0; n < o.ti.size(); ++n) {
        int i = o.ti[n], j = o.tj[n], k = o.tk[n], l = o.tl[n];
        double rij[3], rkj[3], rkl[3], rik[3], rjl[3];
        tors_vecs(o, i, j, k, l, rij, rkj, rkl, rik, rjl);
        TorsGeo g; tors_geo(rij, rkj, rkl, g);
        double period = std::fabs(o.tper[n]);
        double bar = o.tbar[n], ph = o.tph[n], div = (double)o.tdiv[n];
        pot += bar / div * (1.0 + std::cos(period * g.phi - ph));
        int np = (int)std::lround(period);
        double c = g.cphi, fa;
        if (np == 1) fa = 1.0;
        else if (np == 2) fa = 2.0 * c;
        else if (np == 3) fa = -4.0 * g.sphi * g.sphi + 3.0;
        else if (np == 4) fa = 4.0 * c * (2.0 * c * c - 1.0);
        else if (np == 5) { fa = 4.0 * c * c; fa = fa * (fa - 3.0) + 1.0; }
        else if (np == 6) { fa = 4.0 * c * c; fa = 2.0 * c * (fa - 3.0) * (fa - 1.0); }
        else { o.status = PGK_E_UNSUPPORTED; fa = 0.0; }
        fa = -fa * std::cos(ph) * bar * period / div;
        double fi[3], fj[3], fk[3], fl[3];
        tors_forces(fa, g, rij, rkj, rkl, rik, rjl, fi, fj, fk, fl);
        add4(o, force, vs, vt, i, j, k, l, fi, fj, fk, fl);
    }
}

// caltorsrbp + calijklrb (caltorsrb.F90:118-459)
void caltorsrbp(Oracle& o, double* force, double& pot, double& vs, double* vt) {
    pot = 0;
    for (size_t n = 0; n < o.rbi.size(); ++n) {
        int i = o.rbi[n], j = o.rbj[n], k = o.rbk[n], l = o.rbl[n];
        double rij[3], rkj[3], rkl[3], rik[3], rjl[3];
        tors_vecs(o, i, j, k, l, rij, rkj, rkl, rik, rjl);
        TorsGeo g; tors_geo(rij, rkj, rkl, g);
        const double* C = &o.rbc[6 * n];
        double bt[6] = {C[0], -C[1], C[2], -C[3], C[4], -C[5]};
        double dp = bt[5], fa = 0.0;
        for (int q = 4; q >= 0; --q) { fa = fa * g.cphi + dp; dp = dp * g.cphi + bt[q]; }
        fa = -fa;
        pot += dp;
        double fi[3], fj[3], fk[3], fl[3];
        tors_forces(fa, g, rij, rkj, rkl, rik, rjl, fi, fj, fk, fl);
        add4(o, force, vs, vt, i, j, k, l, fi, fj, fk, fl);
    }
}

// calnon14p (calnon14.F90:249-521)
void calnon14p(Oracle& o, double* force, double& pe, double& pv, double& vs, double* vt) {
    pe = 0; pv = 0;
    for (size_t n = 0; n < o.p14i.size(); ++n) {
        int i = o.p14i[n], j = o.p14j[n];
        int it = o.atmindex[i], jt = o.atmindex[j];
        double rij[3]; mi(o, i, j, rij);
        double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
        double ri2 = 1.0 / r2, ri1 = std::sqrt(ri2);
        double de = o.atmchrg[i] * o.atmchrg[j] * ri1;
        de = de * o.p14e[n];
        double fe[3] = {de * ri2 * rij[0], de * ri2 * rij[1], de * ri2 * rij[2]};
        double R = o.radij[it + o.ntyp * jt];
        double t2 = ri2 * (R * R), t6 = t2 * t2 * t2, t12 = t6 * t6;
        double E = o.welij[it + o.ntyp * jt] * o.p14v[n];
        double dv = E * (t12 - 2.0 * t6);
        double ft = 12.0 * E * (t12 - t6) * ri2;
        double fv[3] = {ft * rij[0], ft * rij[1], ft * rij[2]};
        for (int d = 0; d < 3; ++d) { force[3 * i + d] += fe[d]; force[3 * j + d] -= fe[d]; }
        vs += fe[0] * rij[0] + fe[1] * rij[1] + fe[2] * rij[2];
        for (int nn = 0; nn < 3; ++nn) for (int a = 0; a < 3; ++a) vt[a + 3 * nn] += fe[a] * rij[nn];
        pe += de;
        for (int d = 0; d < 3; ++d) { force[3 * i + d] += fv[d]; force[3 * j + d] -= fv[d]; }
        vs += fv[0] * rij[0] + fv[1] * rij[1] + fv[2] * rij[2];
        for (int nn = 0; nn < 3; ++nn) for (int a = 0; a < 3; ++a) vt[a + 3 * nn] += fv[a] * rij[nn];
        pv += dv;
    }
}

int ewaldkp_hf(Oracle& o, int kmax, double* force, double* pot_atm, double* viri, double* sc, int* nwave_out);

// morsep (morse.F90:206-414): Morse energy, forces and virials over the
// Morse list, pairs beyond rcutmor skipped; forces summed in fmor first
void morsep(Oracle& o, double* force, double& pot, double& vir, double* virt) {
    const int n = o.natom, nm = (int)o.mor_atoms.size();
    const double sqcut = o.prm.rcutmor * o.prm.rcutmor;
    std::vector<double> fm((size_t)3 * n, 0.0);
    for (int m1 = 0; m1 + 1 < nm; ++m1) {
        const int i = o.mor_atoms[m1], it = o.atmindex[i];
        for (int q = o.mor_idx[m1]; q < o.mor_idx[m1 + 1]; ++q) {
            const int j = o.mor_list[q], jt = o.atmindex[j];
            double rij[3]; mi(o, i, j, rij);
            double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (r2 > sqcut) continue;
            double r = std::sqrt(r2), ri1 = 1.0 / r;
            const size_t t = (size_t)it + (size_t)o.ntyp * jt;
            double rt1 = std::exp(-1.0 * (r - o.radmor[t]) * o.almor[t]);
            double rt2 = rt1 * rt1;
            double ftmp = 2.0 * o.almor[t] * o.welmor[t] * (rt2 - rt1) * ri1;
            double potij = o.welmor[t] * (rt2 - 2.0 * rt1);
            pot = pot + potij;
            double fij[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
            for (int d = 0; d < 3; ++d) { fm[3 * i + d] += fij[d]; fm[3 * j + d] -= fij[d]; }
            for (int nn = 0; nn < 3; ++nn) for (int a = 0; a < 3; ++a) virt[a + 3 * nn] += fij[a] * rij[nn];
            vir = vir + fij[0] * rij[0] + fij[1] * rij[1] + fij[2] * rij[2];
        }
    }
    for (size_t k = 0; k < fm.size(); ++k) force[k] = force[k] + fm[k];
}

// calforce (calforce.F90:8-1073) for one MTS group; force overwritten
void calforce(Oracle& o, int flag, double* force, pgk_energies* e, pgk_virials* v) {
    std::fill(force, force + 3 * o.natom, 0.0);
    pgk_energies E{}; pgk_virials V{};
    if (o.prm.mts_vdw == flag) ewaldrp(o, force, &E, &V);
    if (o.hf.ewk_now && o.prm.mts_ewk == flag) {
        // -D_HF_BULK_EWK heat-flux step (calforce_hf.F90:1046-1062): ewaldkp_hf
        // in place of fft_pmep; pot_viri_coul += pot_ewk + pot_ewk_cc (ewaldk_hf.F90:290)
        const size_t n = (size_t)o.natom;
        std::vector<double> f(3 * n, 0.0), sc(11, 0.0);
        o.hf.ewk_pot.assign(n, 0.0);
        o.hf.ewk_vir.assign(9 * n, 0.0);
        int nw = 0;
        ewaldkp_hf(o, o.hf.kmax, f.data(), o.hf.ewk_pot.data(), o.hf.ewk_vir.data(), sc.data(), &nw);
        for (size_t k = 0; k < 3 * n; ++k) force[k] += f[k];
        E.pot_ewk += sc[0];
        V.pot_viri_coul += sc[0] + sc[1];
        for (int k = 0; k < 9; ++k) V.pot_virit_coul[k] += sc[2 + k];
        o.hf.ewk_fresh = true;
    } else if (o.prm.mts_ewk == flag && o.prm.ifspme) {
        fft_pmep(o, force, &E, &V);
    }
    if (o.prm.mts_bond == flag) calbondp(o, force, E.pot_bond, V.atm_viri_bond, V.atm_virit_bond);
    if (o.prm.mts_angl == flag) calanglp(o, force, E.pot_angl, V.atm_viri_angl, V.atm_virit_angl);
    if (o.prm.mts_tors == flag) caltorsp(o, force, E.pot_tors, V.atm_viri_tors, V.atm_virit_tors);
    if (o.prm.mts_torsrb == flag) caltorsrbp(o, force, E.pot_torsrb, V.atm_viri_tors, V.atm_virit_tors);
    if (o.prm.mts_vdw14 == flag && o.prm.mts_elc14 == flag)
        calnon14p(o, force, E.pot_elc14, E.pot_vdw14, V.atm_viri_14, V.atm_virit_14);
    if (!o.welmor.empty() && o.prm.mts_mor == flag) morsep(o, force, E.pot_mor, V.pot_viri_mor, V.pot_virit_mor);
    if (flag == PGK_MTS_LONG && o.prm.ifspme) {   // :1018-1050 net charge
        double pi = std::acos(-1.0);
        double a1 = -pi / (o.prm.alpha * o.prm.alpha * o.box[0] * o.box[1] * o.box[2]);
        E.pot_ewnq = 0.5 * a1 * o.netchrgsq;
        if (!o.prm.ifnetqcorrp) {
            V.pot_viri_coul += a1 * o.netchrgsq;
            for (int d = 0; d < 3; ++d) V.pot_virit_coul[4 * d] += 0.5 * a1 * o.netchrgsq;
        } else {
            V.pot_viri_coul -= 0.5 * a1 * o.netchrgsq;
        }
        E.pot_ewc = o.pot_ewc;
    }
    E.pot_nonbon = E.pot_vdw + E.pot_elc + E.pot_ewk + E.pot_ewc + E.pot_ewnq + E.pot_vdw14 + E.pot_elc14;
    E.pot_tot = E.pot_bond + E.pot_angl + E.pot_tors + E.pot_torsrb + E.pot_mor + E.pot_nonbon;
    if (e) *e = E;
    if (v) *v = V;
}

// --------------------------------------------------------------------------
// RATTLE (rattle.F90:6-272, rattle_mtk.F90:8-542).  The mvlast/mvnow skip of
// the reference never changes results (a skipped constraint was satisfied in
// the previous sweep and none of its atoms moved since), so it is omitted.
// --------------------------------------------------------------------------
int rattle_pos(Oracle& o, const double* old, double eps, double dt, const double* rvinv) {
    for (size_t g = 0; g + 1 < o.cidx.size(); ++g) {
        int i1 = o.cidx[g], i2 = o.cidx[g + 1];
        bool finished = false;
        for (int it = 0; it < 300; ++it) {
            finished = true;
            for (int ii = i1; ii < i2; ++ii) {
                int nc = o.clist[ii];
                int ib = o.ci[nc], jb = o.cj[nc];
                double dij = o.cd[nc];
                double R[3];
                for (int d = 0; d < 3; ++d) R[d] = o.atmcor[3 * ib + d] - o.atmcor[3 * jb + d];
                double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                double d2 = dij * dij;
                double delta = std::fabs(R2 - d2) / d2;
                if (delta < eps) continue;
                finished = false;
                double Ro[3];
                for (int d = 0; d < 3; ++d) Ro[d] = old[3 * ib + d] - old[3 * jb + d];
                double RR = R[0] * Ro[0] + R[1] * Ro[1] + R[2] * Ro[2];
                double mi_ = 1.0 / o.atmmass[ib], mj_ = 1.0 / o.atmmass[jb];
                double gij = (R2 - d2) / (2.0 * RR * (mi_ + mj_) * dt);
                double G[3] = {gij * Ro[0], gij * Ro[1], gij * Ro[2]};
                for (int d = 0; d < 3; ++d) {
                    o.atmcor[3 * ib + d] = o.atmcor[3 * ib + d] - mi_ * G[d] * dt;
                    o.atmcor[3 * jb + d] = o.atmcor[3 * jb + d] + mj_ * G[d] * dt;
                }
                if (rvinv) for (int d = 0; d < 3; ++d) G[d] = G[d] * rvinv[d];
                for (int d = 0; d < 3; ++d) {
                    o.atmvel[3 * ib + d] = o.atmvel[3 * ib + d] - mi_ * G[d];
                    o.atmvel[3 * jb + d] = o.atmvel[3 * jb + d] + mj_ * G[d];
                }
            }
            if (finished) break;
        }
        if (!finished) return PGK_E_RATTLE_NOCONV;
    }
    return PGK_OK;
}

int rattlep_v(Oracle& o, double eps) {
    double eps2 = eps * eps;
    for (size_t g = 0; g + 1 < o.cidx.size(); ++g) {
        int i1 = o.cidx[g], i2 = o.cidx[g + 1];
        bool finished = false;
        for (int it = 0; it < 300; ++it) {
            finished = true;
            for (int ii = i1; ii < i2; ++ii) {
                int nc = o.clist[ii];
                int ib = o.ci[nc], jb = o.cj[nc];
                double dij = o.cd[nc];
                double R[3], V[3];
                for (int d = 0; d < 3; ++d) {
                    R[d] = o.atmcor[3 * ib + d] - o.atmcor[3 * jb + d];
                    V[d] = o.atmvel[3 * ib + d] - o.atmvel[3 * jb + d];
                }
                double RV = R[0] * V[0] + R[1] * V[1] + R[2] * V[2];
                double R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
                double V2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
                double phi = RV * RV / R2 * V2;     // reference precedence kept
                if (phi < eps2) continue;
                finished = false;
                double mi_ = 1.0 / o.atmmass[ib], mj_ = 1.0 / o.atmmass[jb];
                double kij = RV / (dij * dij * (mi_ + mj_));
                for (int d = 0; d < 3; ++d) {
                    double KR = kij * R[d];
                    o.atmvel[3 * ib + d] = o.atmvel[3 * ib + d] - mi_ * KR;
                    o.atmvel[3 * jb + d] = o.atmvel[3 * jb + d] + mj_ * KR;
                }
            }
            if (finished) break;
        }
        if (!finished) return PGK_E_RATTLEV_NOCONV;
    }
    return PGK_OK;
}

// --------------------------------------------------------------------------
// thermostat / barostat (nhcint.F90, nhcpisoint.F90, nhcpanisoint.F90)
// --------------------------------------------------------------------------
double kint_sum(const Oracle& o) {
    double k = 0;
    for (int i = 0; i < o.natom; ++i)
        k += o.atmmass[i] * (o.atmvel[3 * i] * o.atmvel[3 * i] + o.atmvel[3 * i + 1] * o.atmvel[3 * i + 1] +
                             o.atmvel[3 * i + 2] * o.atmvel[3 * i + 2]);
    return k;
}

void nhc_chain_tail(pgk_chain& c, const pgk_mdparams& md, double* glogs, double w4, double w8, double gkt,
                    bool down) {
    int M = md.mchain;
    const double* q = md.qmass;
    if (down) {
        glogs[M - 1] = (q[M - 2] * c.vlogs[M - 2] * c.vlogs[M - 2] - gkt) / q[M - 1];
        c.vlogs[M - 1] = c.vlogs[M - 1] + glogs[M - 1] * w4;
        for (int i = M - 2; i >= 1; --i) {
            glogs[i] = (q[i - 1] * c.vlogs[i - 1] * c.vlogs[i - 1] - gkt) / q[i];
            double e8 = std::exp(-1.0 * w8 * c.vlogs[i + 1]);
            c.vlogs[i] = c.vlogs[i] * e8 * e8 + w4 * glogs[i] * e8;
        }
    } else {
        for (int i = 1; i <= M - 2; ++i) {
            glogs[i] = (q[i - 1] * c.vlogs[i - 1] * c.vlogs[i - 1] - gkt) / q[i];
            double e8 = std::exp(-1.0 * w8 * c.vlogs[i + 1]);
            c.vlogs[i] = c.vlogs[i] * e8 * e8 + w4 * glogs[i] * e8;
        }
        glogs[M - 1] = (q[M - 2] * c.vlogs[M - 2] * c.vlogs[M - 2] - gkt) / q[M - 1];
        c.vlogs[M - 1] = c.vlogs[M - 1] + glogs[M - 1] * w4;
    }
}

void nhcint(Oracle& o, const pgk_mdparams& md, double dt) {   // nhcint.F90:8-140
    pgk_chain& c = o.ch;
    int M = md.mchain;
    double gnkt = md.text * (double)o.degfree, gkt = md.text;
    double kint = kint_sum(o);
    double glogs[8] = {0};
    glogs[0] = (kint - gnkt) / md.qmass[0];
    for (int inc = 0; inc < md.next; ++inc)
        for (int iy = 0; iy < md.nyosh; ++iy) {
            double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, true);
            double e8 = std::exp(-1.0 * w8 * c.vlogs[1]);
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, false);
        }
}

void nhcpisoint(Oracle& o, const pgk_mdparams& md, double dt) {  // nhcpisoint.F90:6-162
    pgk_chain& c = o.ch;
    int M = md.mchain;
    double gn1kt = md.text * (double)(o.degfree + 1), gkt = md.text;
    double dnf = 3.0 / (double)o.degfree;
    double vol = std::exp(3.0 * c.xlogv);
    double kint = kint_sum(o);
    double glogs[8] = {0};
    glogs[0] = (kint + md.vmass * c.vlogv * c.vlogv - gn1kt) / md.qmass[0];
    double glogv = (dnf * kint + 3.0 * vol * (c.pint - md.pext)) / md.vmass;
    for (int inc = 0; inc < md.next; ++inc)
        for (int iy = 0; iy < md.nyosh; ++iy) {
            double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, true);
            double e8 = std::exp(-1.0 * w8 * c.vlogs[1]);
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            e8 = std::exp(-1.0 * w8 * c.vlogs[0]);
            c.vlogv = c.vlogv * e8 * e8 + w4 * glogv * e8;
            for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
            c.vlogv = c.vlogv * e8 * e8 + w4 * glogv * e8;
            glogs[0] = (kint + md.vmass * c.vlogv * c.vlogv - gn1kt) / md.qmass[0];
            e8 = std::exp(-1.0 * w8 * c.vlogs[1]);
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, false);
        }
}

void nhcpanisoint(Oracle& o, const pgk_mdparams& md, double dt) {  // nhcpanisoint.F90:8-189
    pgk_chain& c = o.ch;
    int M = md.mchain;
    int dir = md.pcont_axis == PGK_PCONT_ANISO ? 0 : md.pcont_axis - 1;  // 1..3 uniaxial
    double gndfkt = md.text * (double)(o.degfree + (dir == 0 ? 3 : 1)), gkt = md.text;
    double dnf = 1.0 / (double)o.degfree;
    double vol = c.xboxh[0] * c.xboxh[1] * c.xboxh[2];
    double pv[3] = {c.pintt[0], c.pintt[4], c.pintt[8]};
    double kint = kint_sum(o);
    double glogs[8] = {0};
    auto vb2 = [&]() { return c.vboxg[0] * c.vboxg[0] + c.vboxg[1] * c.vboxg[1] + c.vboxg[2] * c.vboxg[2]; };
    glogs[0] = (kint + md.vmass * vb2() - gndfkt) / md.qmass[0];
    double gb[3];
    for (int d = 0; d < 3; ++d) gb[d] = (dnf * kint + vol * (pv[d] - md.pext)) / md.vmass;
    for (int inc = 0; inc < md.next; ++inc)
        for (int iy = 0; iy < md.nyosh; ++iy) {
            double w2 = md.yscoeff[iy] * dt / (double)md.next / 2.0, w4 = w2 / 2.0, w8 = w4 / 2.0;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, true);
            double e8 = std::exp(-1.0 * w8 * c.vlogs[1]);
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            e8 = std::exp(-1.0 * w8 * c.vlogs[0]);
            for (int d = 0; d < 3; ++d)
                if (dir == 0 || d == dir - 1) c.vboxg[d] = c.vboxg[d] * e8 * e8 + w4 * gb[d] * e8;
            for (int i = 0; i < M; ++i) c.xlogs[i] = c.xlogs[i] + c.vlogs[i] * w2;
            for (int d = 0; d < 3; ++d)
                if (dir == 0 || d == dir - 1) c.vboxg[d] = c.vboxg[d] * e8 * e8 + w4 * gb[d] * e8;
            glogs[0] = (kint + md.vmass * vb2() - gndfkt) / md.qmass[0];
            e8 = std::exp(-1.0 * w8 * c.vlogs[1]);
            c.vlogs[0] = c.vlogs[0] * e8 * e8 + w4 * glogs[0] * e8;
            nhc_chain_tail(c, md, glogs, w4, w8, gkt, false);
        }
}

// calpress, atomic branch (calpress.F90); vl/vs = long/short group virials
void calpress(Oracle& o, const pgk_virials& vl, const pgk_virials& vs, double* ptot, double* pt) {
    double K = 0, Kt[9] = {0};
    for (int i = 0; i < o.natom; ++i) {
        const double* v = &o.atmvel[3 * i];
        K += o.atmmass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int nn = 0; nn < 3; ++nn) for (int a = 0; a < 3; ++a) Kt[a + 3 * nn] += o.atmmass[i] * v[a] * v[nn];
    }
    double pi = std::acos(-1.0);
    double a1 = -pi / (o.prm.alpha * o.prm.alpha * o.box[0] * o.box[1] * o.box[2]);
    double ewnq = o.prm.ifspme ? 0.5 * a1 * o.netchrgsq : 0.0;
    double ewc = o.prm.ifspme ? o.pot_ewc : 0.0;
    double W = vl.pot_viri_coul + vs.pot_viri_coul + ewc + ewnq + vl.pot_viri_lj + vs.pot_viri_lj;
    W += vl.atm_viri_bond + vs.atm_viri_bond + vl.atm_viri_angl + vs.atm_viri_angl +
         vl.atm_viri_tors + vs.atm_viri_tors + vl.atm_viri_14 + vs.atm_viri_14;
    W += vl.pot_viri_mor + vs.pot_viri_mor;   // calpress.F90:146-151
    double Wt[9];
    for (int k = 0; k < 9; ++k)
        Wt[k] = vl.pot_virit_coul[k] + vs.pot_virit_coul[k] + vl.pot_virit_lj[k] + vs.pot_virit_lj[k] +
                vl.atm_virit_bond[k] + vs.atm_virit_bond[k] + vl.atm_virit_angl[k] + vs.atm_virit_angl[k] +
                vl.atm_virit_tors[k] + vs.atm_virit_tors[k] + vl.atm_virit_14[k] + vs.atm_virit_14[k] +
                vl.pot_virit_mor[k] + vs.pot_virit_mor[k];
    double binv = 1.0 / o.box[0] * (1.0 / o.box[1]) * (1.0 / o.box[2]);
    double b3 = (1.0 / o.box[0]) * (1.0 / o.box[1]) * (1.0 / o.box[2]);
    (void)binv;
    if (ptot) *ptot = 1.0 / 3.0 * b3 * (K + W);
    if (pt) for (int k = 0; k < 9; ++k) pt[k] = 1.0 * b3 * (Kt[k] + Wt[k]);
}

void transcor(Oracle& o) {   // transcor.F90 (molecule wrap by its first atom)
    for (size_t m = 0; m + 1 < o.molidx.size(); ++m) {
        int a0 = o.mollist[o.molidx[m]];
        for (int d = 0; d < 3; ++d) {
            double sh = 0.0;
            if (o.atmcor[3 * a0 + d] < 0.0) sh = o.box[d];
            else if (o.atmcor[3 * a0 + d] > o.box[d]) sh = -o.box[d];
            if (sh != 0.0)
                for (int q = o.molidx[m]; q < o.molidx[m + 1]; ++q) {
                    int k = o.mollist[q];
                    o.atmcor[3 * k + d] = o.atmcor[3 * k + d] + sh;
                }
        }
    }
}

bool box_ok(const Oracle& o) {   // calvol.F90 / calbox.F90 checks
    double h = std::min(o.box[0] * 0.5, std::min(o.box[1] * 0.5, o.box[2] * 0.5));
    return !(o.prm.rcut > h || o.prm.rcut_book > h);
}

// --------------------------------------------------------------------------
// stage drivers: moldyn.F90 (NVE), moldyn_nhc.F90 (NHC), moldyn_mtk.F90 (MTK)
// kind: 0 NVE, 1 NHC, 2 MTK
// --------------------------------------------------------------------------
int md_nbook(const Oracle& o) { return o.prm.nstep_book > 0 ? o.prm.nstep_book : 1; }

void accforce(const Oracle& o, std::vector<double>& f) {   // accforce.F90
    for (int i = 0; i < o.natom; ++i) for (int d = 0; d < 3; ++d) f[3 * i + d] = f[3 * i + d] / o.atmmass[i];
}

int moldyn(Oracle& o, int kind, long long ini, long long end, const pgk_mdparams& md, pgk_energies* eout,
           Forces& F) {
    int n = o.natom;
    double dtl = md.dt_long_cal, dts = md.dt_long_cal / (double)md.nstep_short;
    double e2 = 1.0 / 6.0, e4 = e2 / 20.0, e6 = e4 / 42.0, e8 = e6 / 72.0;
    std::vector<double> old((size_t)3 * n);
    bool aniso = kind == 2 && md.pcont_axis != PGK_PCONT_ISO;
    int dir = md.pcont_axis == PGK_PCONT_ANISO ? 0 : md.pcont_axis - 1;
    if (F.fl.size() != (size_t)3 * n) { F.fl.assign((size_t)3 * n, 0.0); F.fs.assign((size_t)3 * n, 0.0); }
    auto force_eval = [&](int flag) {
        if (flag == PGK_MTS_LONG) { calforce(o, flag, F.fl.data(), &F.el, &F.vl); accforce(o, F.fl); }
        else { calforce(o, flag, F.fs.data(), &F.es, &F.vs); accforce(o, F.fs); }
    };
    auto setpint = [&]() {
        double p, pt[9];
        calpress(o, F.vl, F.vs, &p, pt);
        o.ch.pint = p;
        for (int k = 0; k < 9; ++k) o.ch.pintt[k] = pt[k];
    };
    double expcdt2 = 1, bbv = 0.5 * dtl, ecv2[3] = {1, 1, 1}, bbvv[3] = {0, 0, 0};
    for (long long step = ini; step <= end; ++step) {
        if (step % md_nbook(o) == 1 || md_nbook(o) == 1 || step == 0) transcor(o);
        if (step % md_nbook(o) == 0 || md_nbook(o) == 1) mklist(o);
        if (step == 0) {
            force_eval(PGK_MTS_SHORT);
            force_eval(PGK_MTS_LONG);
            if (kind == 2) setpint();
        } else {
            if (kind == 1) nhcint(o, md, dtl);
            if (kind == 2) { if (!aniso) nhcpisoint(o, md, dtl); else nhcpanisoint(o, md, dtl); }
            for (int is = 1; is <= md.nstep_short; ++is) {
                if (is == 1) {
                    if (kind == 0) {
                        for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dtl * F.fl[k];
                    } else if (!aniso) {
                        double vext = o.ch.vlogs[0];
                        if (kind == 2) vext = o.ch.vlogs[0] + (1.0 + 3.0 / (double)o.degfree) * o.ch.vlogv;
                        double ec4 = std::exp(-0.25 * dtl * vext);
                        expcdt2 = ec4 * ec4;
                        double a2 = (0.25 * dtl * vext) * (0.25 * dtl * vext);
                        double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
                        double cf = ec4 * poly;
                        bbv = cf * 0.5 * dtl;
                        for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] * expcdt2 + F.fl[k] * bbv;
                    } else {
                        double vx[3];
                        for (int d = 0; d < 3; ++d) vx[d] = o.ch.vlogs[0];
                        if (dir == 0) {
                            double tr = o.ch.vboxg[0] + o.ch.vboxg[1] + o.ch.vboxg[2];
                            for (int d = 0; d < 3; ++d) vx[d] = o.ch.vlogs[0] + o.ch.vboxg[d] + 1.0 / (double)o.degfree * tr;
                        } else {
                            vx[dir - 1] = vx[dir - 1] + o.ch.vboxg[dir - 1] + 1.0 / (double)o.degfree * o.ch.vboxg[dir - 1];
                        }
                        for (int d = 0; d < 3; ++d) {
                            double ec4 = std::exp(-0.25 * dtl * vx[d]);
                            ecv2[d] = ec4 * ec4;
                            double a2 = (0.25 * dtl * vx[d]) * (0.25 * dtl * vx[d]);
                            double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
                            bbvv[d] = ec4 * poly * 0.5 * dtl;
                        }
                        for (int i = 0; i < n; ++i)
                            for (int d = 0; d < 3; ++d)
                                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] * ecv2[d] + F.fl[3 * i + d] * bbvv[d];
                    }
                }
                for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dts * F.fs[k];
                if (md.ifrattle && o.ci.size()) old = o.atmcor;
                double rvinv[3] = {1, 1, 1};
                if (kind == 2 && !aniso) {
                    double aa = std::exp(0.5 * dts * o.ch.vlogv), aa2 = aa * aa;
                    double a2 = (0.5 * dts * o.ch.vlogv) * (0.5 * dts * o.ch.vlogv);
                    double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
                    double bb = aa * poly * dts, rv = aa * poly;
                    for (int k = 0; k < 3 * n; ++k) o.atmcor[k] = o.atmcor[k] * aa2 + o.atmvel[k] * bb;
                    o.ch.xlogv = o.ch.xlogv + o.ch.vlogv * dts;
                    double vol = std::exp(3.0 * o.ch.xlogv);     // calvol.F90
                    o.box[0] = std::pow(vol / o.yratio / o.zratio, 1.0 / 3.0);
                    o.box[1] = o.yratio * o.box[0];
                    o.box[2] = o.zratio * o.box[0];
                    if (!box_ok(o)) return PGK_E_BOX_TOO_SMALL;
                    for (int d = 0; d < 3; ++d) rvinv[d] = 1.0 / rv;
                } else if (kind == 2) {
                    double aa2v[3], bbr[3];
                    for (int d = 0; d < 3; ++d) {
                        double aa = std::exp(0.5 * dts * o.ch.vboxg[d]);
                        aa2v[d] = aa * aa;
                        double a2 = (0.5 * dts * o.ch.vboxg[d]) * (0.5 * dts * o.ch.vboxg[d]);
                        double poly = 1.0 + a2 * (e2 + a2 * (e4 + a2 * (e6 + a2 * e8)));
                        bbr[d] = aa * poly * dts;
                        rvinv[d] = 1.0 / (aa * poly);
                    }
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < 3; ++d)
                            o.atmcor[3 * i + d] = o.atmcor[3 * i + d] * aa2v[d] + o.atmvel[3 * i + d] * bbr[d];
                    for (int d = 0; d < 3; ++d) o.ch.xboxh[d] = o.ch.xboxh[d] * std::exp(o.ch.vboxg[d] * dts);
                    for (int d = 0; d < 3; ++d) o.box[d] = o.ch.xboxh[d];   // calbox.F90
                    o.yratio = o.box[1] / o.box[0]; o.zratio = o.box[2] / o.box[0];
                    if (!box_ok(o)) return PGK_E_BOX_TOO_SMALL;
                } else {
                    for (int k = 0; k < 3 * n; ++k) o.atmcor[k] = o.atmcor[k] + dts * o.atmvel[k];
                }
                if (kind == 2 && o.prm.mts_ewk == PGK_MTS_SHORT)
                    o.rkcut = erf_corr_cutoff(o.box, o.prm.nfft1, o.prm.nfft2, o.prm.nfft3);
                if (md.ifrattle && o.ci.size()) {
                    int s = rattle_pos(o, old.data(), md.eps_rattle, dts, kind == 2 ? rvinv : nullptr);
                    if (s) return s;
                }
                force_eval(PGK_MTS_SHORT);
                if (is == md.nstep_short) {
                    if (kind == 2 && o.prm.mts_ewk == PGK_MTS_LONG)
                        o.rkcut = erf_corr_cutoff(o.box, o.prm.nfft1, o.prm.nfft2, o.prm.nfft3);
                    force_eval(PGK_MTS_LONG);
                }
                for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dts * F.fs[k];
                if (is == md.nstep_short) {
                    if (kind == 0) {
                        for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dtl * F.fl[k];
                    } else if (!aniso) {
                        for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] * expcdt2 + F.fl[k] * bbv;
                    } else {
                        for (int i = 0; i < n; ++i)
                            for (int d = 0; d < 3; ++d)
                                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] * ecv2[d] + F.fl[3 * i + d] * bbvv[d];
                    }
                }
                if (md.ifrattle && o.ci.size()) {
                    int s = rattlep_v(o, md.eps_rattle);
                    if (s) return s;
                }
            }
            if (kind == 1) nhcint(o, md, dtl);
            if (kind == 2) {
                setpint();
                if (!aniso) nhcpisoint(o, md, dtl); else nhcpanisoint(o, md, dtl);
            }
        }
        if (eout && (md.outinterval <= 0 ? step == end : step % md.outinterval == 0)) {
            pgk_energies e{};
            e.pot_vdw = F.el.pot_vdw + F.es.pot_vdw; e.pot_elc = F.el.pot_elc + F.es.pot_elc;
            e.pot_ewk = F.el.pot_ewk + F.es.pot_ewk; e.pot_ewc = F.el.pot_ewc + F.es.pot_ewc;
            e.pot_ewnq = F.el.pot_ewnq + F.es.pot_ewnq;
            e.pot_vdw14 = F.el.pot_vdw14 + F.es.pot_vdw14; e.pot_elc14 = F.el.pot_elc14 + F.es.pot_elc14;
            e.pot_bond = F.el.pot_bond + F.es.pot_bond; e.pot_angl = F.el.pot_angl + F.es.pot_angl;
            e.pot_tors = F.el.pot_tors + F.es.pot_tors; e.pot_torsrb = F.el.pot_torsrb + F.es.pot_torsrb;
            e.pot_mor = F.el.pot_mor + F.es.pot_mor;
            e.pot_nonbon = F.el.pot_nonbon + F.es.pot_nonbon; e.pot_tot = F.el.pot_tot + F.es.pot_tot;
            *eout = e;
        }
    }
    return PGK_OK;
}


// ============================================================================
// Heat flux of the -DHF build (volume-based IK, z direction) and the region
// Langevin thermostat.  The force routines above are unchanged; on a heat-
// flux step these restatements add the per-atom quantities that
// ewaldrp_hf / cal*p_hf compute next to the same forces.
// ============================================================================
enum { HF_BO = 0, HF_AN, HF_TO, HF_14, HF_ELIN, HF_LJIN, HF_ELC, HF_VDW };

inline double wrap1(double x, double L) {   // the single-shift P.B.C. of calcom / calvirihf / calheatf
    if (x < 0.0) return x + L;
    if (x >= L) return x - L;
    return x;
}
inline size_t widx(const Oracle& o, int cat, int r, int a, int i) {
    return (((size_t)cat * o.hf.nreg + r) * 3 + a) * o.natom + i;
}

// calcom.F90: molecule centres of mass from atmcor (monatomic molecules take
// the atom position), then wrapped once per axis
void calcom(Oracle& o, const std::vector<double>& x, std::vector<double>& out) {
    int nm = (int)o.molidx.size() - 1;
    out.assign((size_t)3 * nm, 0.0);
    for (int m = 0; m < nm; ++m) {
        int b = o.molidx[m], e = o.molidx[m + 1];
        if (e - b == 1) {
            int i = o.mollist[b];
            for (int d = 0; d < 3; ++d) out[3 * m + d] = x[3 * i + d];
        } else {
            double mass = 0.0, c[3] = {0, 0, 0};
            for (int q = b; q < e; ++q) {
                int i = o.mollist[q];
                mass = mass + o.atmmass[i];
                for (int d = 0; d < 3; ++d) c[d] = c[d] + o.atmmass[i] * x[3 * i + d];
            }
            double inv = 1.0 / mass;
            for (int d = 0; d < 3; ++d) out[3 * m + d] = c[d] * inv;
        }
        for (int d = 0; d < 3; ++d) out[3 * m + d] = wrap1(out[3 * m + d], o.box[d]);
    }
}

// calvirihf.F90:8-405, local volume-based branch without _HF_ALL_DIR/_HF_BULK:
// viri(:,3,i,r) += fi * f, viri(:,3,j,r) += -fj * f, f = +-(z length of the
// i-j segment inside slab r) * nbodycoeff
// dst: a [1][nreg][3][N] array that takes the pair instead of category cat of
// the per-atom arrays (the Morse term of morsep_hf)
void calvirihf(Oracle& o, int i, int j, const double* fi, const double* fj, double nbc, int cat,
               std::vector<double>* dst = nullptr) {
    Oracle::HF& h = o.hf;
    double* W = dst ? dst->data() : h.W.data();
    if (dst) cat = 0;
    int atomflag = 0;
    double zi, zj;
    if (h.hftyp[i] == PGK_HFTYP_MOLE) zi = h.molecom[3 * h.molof[i] + 2];
    else { ++atomflag; zi = wrap1(o.atmcor[3 * i + 2], o.box[2]); }
    if (h.hftyp[j] == PGK_HFTYP_MOLE) zj = h.molecom[3 * h.molof[j] + 2];
    else { ++atomflag; zj = wrap1(o.atmcor[3 * j + 2], o.box[2]); }
    if (atomflag == 0 && h.molof[i] == h.molof[j]) return;
    double rz = zi - zj;
    double az = std::fabs(rz);
    if (az * (1.0 / o.box[2]) >= 0.5) return;
    for (int r = 0; r < h.nreg; ++r) {
        double p1i = zi - h.z1[r], p1j = zj - h.z1[r];
        double p2i = zi - h.z2[r], p2j = zj - h.z2[r];
        int np = 0;
        bool c1 = false;
        if (p1i * p1j < 0.0) { c1 = true; ++np; }
        if (p2i * p2j < 0.0) ++np;
        double frag;
        if (np == 0) {
            if (p1i * p2i > 0.0) continue;
            frag = az;
        } else if (np == 1) {
            if (c1) frag = p1i > 0.0 ? p1i : p1j;
            else frag = p2i < 0.0 ? -p2i : -p2j;
        } else {
            frag = h.z2[r] - h.z1[r];
        }
        double fact = rz >= 0.0 ? frag * nbc : -frag * nbc;
        for (int a = 0; a < 3; ++a) {
            W[widx(o, cat, r, a, i)] += fi[a] * fact;
            W[widx(o, cat, r, a, j)] += (-fj[a]) * fact;
        }
    }
}

// ewaldr_hf.F90:213-520 heat-flux part (default: bare 1/r Coulomb)
void ewaldrp_hf(Oracle& o) {
    int n = o.natom;
    double sqcut = o.prm.rrcut * o.prm.rrcut, sqcut2 = o.prm.rcut * o.prm.rcut;
    if (sqcut2 > sqcut) sqcut = sqcut2;
    double binv[3] = {1.0 / o.box[0], 1.0 / o.box[1], 1.0 / o.box[2]};
    Oracle::HF& h = o.hf;
    for (int i = 0; i < n - 1; ++i) {
        int j1 = o.nb_index[i] - 1, j2 = o.nb_index[i + 1] - 2;
        int it = o.atmindex[i], im = h.molof[i];
        if (o.nb_list[j1] == 0) continue;
        for (int jx = j1; jx <= j2; ++jx) {
            int jj = o.nb_list[jx] - 1, jm = h.molof[jj];
            double rij[3];
            for (int d = 0; d < 3; ++d) {
                double r = o.atmcor[3 * i + d] - o.atmcor[3 * jj + d];
                rij[d] = r - o.box[d] * dnint(r * binv[d]);
            }
            double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (r2 > sqcut) continue;
            double rinv2 = 1.0 / r2;
            double r = std::sqrt(r2), rinv1 = 1.0 / r;
            if (r <= o.prm.rrcut) {
                double potij = o.atmchrg[i] * o.atmchrg[jj] * rinv1;
                double ftmp = potij * rinv2;
                double fij[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
                double fji[3] = {-fij[0], -fij[1], -fij[2]};
                int cat = im == jm ? HF_ELIN : HF_ELC;
                h.pot[(size_t)cat * n + i] += 0.5 * potij;
                h.pot[(size_t)cat * n + jj] += 0.5 * potij;
                calvirihf(o, i, jj, fij, fji, 0.5, cat);
            }
            if (r2 <= sqcut2) {
                int jt = o.atmindex[jj];
                if (!o.inttyp.empty() && o.inttyp[it + o.ntyp * jt] != 1) continue;
                double R = o.radij[it + o.ntyp * jt];
                double t2 = rinv2 * (R * R), t6 = t2 * t2 * t2, t12 = t6 * t6;
                double E = o.welij[it + o.ntyp * jt];
                double potij = E * (t12 - 2.0 * t6);
                double ftmp = 12.0 * E * (t12 - t6) * rinv2;
                double fij[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
                double fji[3] = {-fij[0], -fij[1], -fij[2]};
                int cat = im == jm ? HF_LJIN : HF_VDW;
                h.pot[(size_t)cat * n + i] += 0.5 * potij;
                h.pot[(size_t)cat * n + jj] += 0.5 * potij;
                calvirihf(o, i, jj, fij, fji, 0.5, cat);
            }
        }
    }
}

// calbond_hf.F90:95-160 (nbodycoeff 1/2)
void calbondp_hf(Oracle& o) {
    int n = o.natom;
    for (size_t k = 0; k < o.bi.size(); ++k) {
        if (std::fabs(o.bk[k]) < 1.0e-16) continue;
        int i = o.bi[k], j = o.bj[k];
        double rij[3]; mi(o, i, j, rij);
        double r = std::sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        double dp = o.bk[k] * (r - o.br0[k]) * (r - o.br0[k]);
        o.hf.pot[(size_t)HF_BO * n + i] += 0.5 * dp;
        o.hf.pot[(size_t)HF_BO * n + j] += 0.5 * dp;
        double fa = -2.0 * o.bk[k] * (r - o.br0[k]);
        double f[3] = {fa * rij[0] / r, fa * rij[1] / r, fa * rij[2] / r};
        double fji[3] = {-f[0], -f[1], -f[2]};
        calvirihf(o, i, j, f, fji, 0.5, HF_BO);
    }
}

// calangl_hf.F90:140-230 (nbodycoeff 1/3; pairs (i,j), (j,k), (k,i))
void calanglp_hf(Oracle& o) {
    int n = o.natom;
    const double c3 = 1.0 / 3.0;
    for (size_t q = 0; q < o.ai.size(); ++q) {
        if (std::fabs(o.akk[q]) < 1.0e-32) continue;
        int i = o.ai[q], j = o.aj[q], k = o.ak[q];
        double rij[3], rkj[3];
        mi(o, j, i, rij); mi(o, j, k, rkj);
        double ra = std::sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        double rb = std::sqrt(rkj[0] * rkj[0] + rkj[1] * rkj[1] + rkj[2] * rkj[2]);
        double c = (rij[0] * rkj[0] + rij[1] * rkj[1] + rij[2] * rkj[2]) / (ra * rb);
        if (c > 1.0) c = 1.0; else if (c < -1.0) c = -1.0;
        double th = std::acos(c), sn = std::sin(th);
        double dp = o.akk[q] * (th - o.at0[q]) * (th - o.at0[q]);
        o.hf.pot[(size_t)HF_AN * n + i] += c3 * dp;
        o.hf.pot[(size_t)HF_AN * n + j] += c3 * dp;
        o.hf.pot[(size_t)HF_AN * n + k] += c3 * dp;
        double fi[3] = {0, 0, 0}, fj[3] = {0, 0, 0}, fk[3] = {0, 0, 0};
        if (std::fabs(sn) > 1.0e-14) {
            double ft = -2.0 * o.akk[q] * (th - o.at0[q]) / sn;
            for (int d = 0; d < 3; ++d) {
                fi[d] = ft * ((rkj[d] / rb - rij[d] * c / ra) / ra);
                fk[d] = ft * ((rij[d] / ra - rkj[d] * c / rb) / rb);
                fj[d] = -fi[d] - fk[d];
            }
        }
        calvirihf(o, i, j, fi, fj, c3, HF_AN);
        calvirihf(o, j, k, fj, fk, c3, HF_AN);
        calvirihf(o, k, i, fk, fi, c3, HF_AN);
    }
}

// caltors_hf.F90 / caltorsrb_hf.F90:130-200 (nbodycoeff 1/4, six pairs)
void tors_hf_add(Oracle& o, int i, int j, int k, int l, double dp, const double* fi, const double* fj,
                 const double* fk, const double* fl) {
    int n = o.natom;
    const int at[4] = {i, j, k, l};
    for (int q = 0; q < 4; ++q) o.hf.pot[(size_t)HF_TO * n + at[q]] += 0.25 * dp;
    calvirihf(o, i, j, fi, fj, 0.25, HF_TO);
    calvirihf(o, i, k, fi, fk, 0.25, HF_TO);
    calvirihf(o, i, l, fi, fl, 0.25, HF_TO);
    calvirihf(o, j, k, fj, fk, 0.25, HF_TO);
    calvirihf(o, j, l, fj, fl, 0.25, HF_TO);
    calvirihf(o, k, l, fk, fl, 0.25, HF_TO);
}
void caltorsp_hf(Oracle& o) {
    for (size_t q = 0; q < o.ti.size(); ++q) {
        int i = o.ti[q], j = o.tj[q], k = o.tk[q], l = o.tl[q];
        double rij[3], rkj[3], rkl[3], rik[3], rjl[3];
        tors_vecs(o, i, j, k, l, rij, rkj, rkl, rik, rjl);
        TorsGeo g; tors_geo(rij, rkj, rkl, g);
        double period = std::fabs(o.tper[q]);
        double bar = o.tbar[q], ph = o.tph[q], div = (double)o.tdiv[q];
        double dp = bar / div * (1.0 + std::cos(period * g.phi - ph));
        int np = (int)std::lround(period);
        double c = g.cphi, fa;
        if (np == 1) fa = 1.0;
        else if (np == 2) fa = 2.0 * c;
        else if (np == 3) fa = -4.0 * g.sphi * g.sphi + 3.0;
        else if (np == 4) fa = 4.0 * c * (2.0 * c * c - 1.0);
        else if (np == 5) { fa = 4.0 * c * c; fa = fa * (fa - 3.0) + 1.0; }
        else if (np == 6) { fa = 4.0 * c * c; fa = 2.0 * c * (fa - 3.0) * (fa - 1.0); }
        else fa = 0.0;
        fa = -fa * std::cos(ph) * bar * period / div;
        double fi[3], fj[3], fk[3], fl[3];
        tors_forces(fa, g, rij, rkj, rkl, rik, rjl, fi, fj, fk, fl);
        tors_hf_add(o, i, j, k, l, dp, fi, fj, fk, fl);
    }
}
void caltorsrbp_hf(Oracle& o) {
    for (size_t q = 0; q < o.rbi.size(); ++q) {
        int i = o.rbi[q], j = o.rbj[q], k = o.rbk[q], l = o.rbl[q];
        double rij[3], rkj[3], rkl[3], rik[3], rjl[3];
        tors_vecs(o, i, j, k, l, rij, rkj, rkl, rik, rjl);
        TorsGeo g; tors_geo(rij, rkj, rkl, g);
        const double* C = &o.rbc[6 * q];
        double bt[6] = {C[0], -C[1], C[2], -C[3], C[4], -C[5]};
        double dp = bt[5], fa = 0.0;
        for (int m = 4; m >= 0; --m) { fa = fa * g.cphi + dp; dp = dp * g.cphi + bt[m]; }
        fa = -fa;
        double fi[3], fj[3], fk[3], fl[3];
        tors_forces(fa, g, rij, rkj, rkl, rik, rjl, fi, fj, fk, fl);
        tors_hf_add(o, i, j, k, l, dp, fi, fj, fk, fl);
    }
}

// calnon14_hf.F90:160-250 (nbodycoeff 1/2; Coulomb and LJ parts)
void calnon14p_hf(Oracle& o) {
    int n = o.natom;
    for (size_t q = 0; q < o.p14i.size(); ++q) {
        int i = o.p14i[q], j = o.p14j[q];
        int it = o.atmindex[i], jt = o.atmindex[j];
        double rij[3]; mi(o, i, j, rij);
        double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
        double ri2 = 1.0 / r2, ri1 = std::sqrt(ri2);
        double de = o.atmchrg[i] * o.atmchrg[j] * ri1;
        de = de * o.p14e[q];
        double fe[3] = {de * ri2 * rij[0], de * ri2 * rij[1], de * ri2 * rij[2]};
        double fe41[3] = {-fe[0], -fe[1], -fe[2]};
        o.hf.pot[(size_t)HF_14 * n + i] += 0.5 * de;
        o.hf.pot[(size_t)HF_14 * n + j] += 0.5 * de;
        calvirihf(o, i, j, fe, fe41, 0.5, HF_14);
        double R = o.radij[it + o.ntyp * jt];
        double t2 = ri2 * (R * R), t6 = t2 * t2 * t2, t12 = t6 * t6;
        double E = o.welij[it + o.ntyp * jt] * o.p14v[q];
        double dv = E * (t12 - 2.0 * t6);
        double ft = 12.0 * E * (t12 - t6) * ri2;
        double fv[3] = {ft * rij[0], ft * rij[1], ft * rij[2]};
        double fv41[3] = {-fv[0], -fv[1], -fv[2]};
        o.hf.pot[(size_t)HF_14 * n + i] += 0.5 * dv;
        o.hf.pot[(size_t)HF_14 * n + j] += 0.5 * dv;
        calvirihf(o, i, j, fv, fv41, 0.5, HF_14);
    }
}

// morsep_hf (morse_hf.F90:6-250): morsep's pair loop with half of each pair
// energy to either atom (pot_mor_atm) and calvirihf (two-body coefficient
// 1/2) into a Morse virial array [nreg][3][N] (virimort_atm); the centres of
// mass come from calcom at the current positions.
void morsep_hf(Oracle& o, double* pot_atm, std::vector<double>& W) {
    Oracle::HF& h = o.hf;
    calcom(o, o.atmcor, h.molecom);
    const int n = o.natom, nm = (int)o.mor_atoms.size();
    std::fill(pot_atm, pot_atm + n, 0.0);
    W.assign((size_t)h.nreg * 3 * n, 0.0);
    const double sqcut = o.prm.rcutmor * o.prm.rcutmor;
    for (int m1 = 0; m1 + 1 < nm; ++m1) {
        const int i = o.mor_atoms[m1], it = o.atmindex[i];
        for (int q = o.mor_idx[m1]; q < o.mor_idx[m1 + 1]; ++q) {
            const int j = o.mor_list[q], jt = o.atmindex[j];
            double rij[3]; mi(o, i, j, rij);
            double r2 = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (r2 > sqcut) continue;
            double r = std::sqrt(r2), ri1 = 1.0 / r;
            const size_t t = (size_t)it + (size_t)o.ntyp * jt;
            double rt1 = std::exp(-1.0 * (r - o.radmor[t]) * o.almor[t]);
            double rt2 = rt1 * rt1;
            double ftmp = 2.0 * o.almor[t] * o.welmor[t] * (rt2 - rt1) * ri1;
            double potij = o.welmor[t] * (rt2 - 2.0 * rt1);
            pot_atm[i] = pot_atm[i] + 0.5 * potij;
            pot_atm[j] = pot_atm[j] + 0.5 * potij;
            double fij[3] = {ftmp * rij[0], ftmp * rij[1], ftmp * rij[2]};
            double fji[3] = {-fij[0], -fij[1], -fij[2]};
            calvirihf(o, i, j, fij, fji, 0.5, 0, &W);
        }
    }
}

// calforce_hf.F90:430-460 (zeroing) + the heat-flux parts of every term;
// molecom from calcom at the current positions
void calforce_hf_atm(Oracle& o) {
    Oracle::HF& h = o.hf;
    calcom(o, o.atmcor, h.molecom);
    h.pot.assign((size_t)8 * o.natom, 0.0);
    h.W.assign((size_t)8 * h.nreg * 3 * o.natom, 0.0);
    auto on = [](int mts) { return mts == PGK_MTS_LONG || mts == PGK_MTS_SHORT; };   // term not switched off
    if (on(o.prm.mts_vdw)) ewaldrp_hf(o);
    if (on(o.prm.mts_bond)) calbondp_hf(o);
    if (on(o.prm.mts_angl)) calanglp_hf(o);
    if (on(o.prm.mts_tors)) caltorsp_hf(o);
    if (on(o.prm.mts_torsrb)) caltorsrbp_hf(o);
    if (on(o.prm.mts_vdw14) && o.prm.mts_vdw14 == o.prm.mts_elc14) calnon14p_hf(o);
    // the per-atom reciprocal term: energy to pot_elc_atm, the (a, z) column of
    // the tensor to region 1 of virielct_atm (ewaldk_hf.F90:212-230)
    const size_t n = (size_t)o.natom;
    std::vector<double> pot, vir;
    if (h.kspace == PGK_HF_KSPACE_SPME) {
        pot.assign(n, 0.0); vir.assign(9 * n, 0.0);
        spme_hf_atm(o, pot.data(), vir.data());
    } else if (h.kspace == PGK_HF_KSPACE_EWK) {
        if (!h.ewk_fresh) {
            std::vector<double> f(3 * n, 0.0), sc(11, 0.0);
            h.ewk_pot.assign(n, 0.0); h.ewk_vir.assign(9 * n, 0.0);
            int nw = 0;
            ewaldkp_hf(o, h.kmax, f.data(), h.ewk_pot.data(), h.ewk_vir.data(), sc.data(), &nw);
        }
        pot = h.ewk_pot; vir = h.ewk_vir;
    }
    h.ewk_fresh = false;
    if (!pot.empty())
        for (size_t i = 0; i < n; ++i) {
            h.pot[(size_t)PGK_HF_ELC * n + i] += pot[i];
            for (int a = 0; a < 3; ++a) h.W[((size_t)PGK_HF_ELC * h.nreg * 3 + a) * n + i] += vir[9 * i + a + 6];
        }
}

// calheatf.F90:365-1466, volume-based, z components; streaming velocity 0
void calheatf(Oracle& o, double* out) {
    Oracle::HF& h = o.hf;
    int n = o.natom, nm = (int)o.molidx.size() - 1;
    h.molevel.assign((size_t)3 * nm, 0.0);
    for (int m = 0; m < nm; ++m) {   // :556-607 (monatomic: the atom velocity)
        int b = o.molidx[m], e = o.molidx[m + 1];
        if (e - b == 1) {
            for (int d = 0; d < 3; ++d) h.molevel[3 * m + d] = o.atmvel[3 * o.mollist[b] + d];
            continue;
        }
        double mass = 0.0, v[3] = {0, 0, 0};
        for (int q = b; q < e; ++q) {
            int i = o.mollist[q];
            mass = mass + o.atmmass[i];
            for (int d = 0; d < 3; ++d) v[d] = v[d] + o.atmmass[i] * o.atmvel[3 * i + d];
        }
        double inv = 1.0 / mass;
        for (int d = 0; d < 3; ++d) h.molevel[3 * m + d] = v[d] * inv;
    }
    std::fill(out, out + (size_t)h.nreg * PGK_HF_NCOL, 0.0);
    for (int i = 0; i < n; ++i) {   // :614-760 kinetic + potential (transport) part
        double pz, vz;
        if (h.hftyp[i] == PGK_HFTYP_MOLE) {
            pz = h.molecom[3 * h.molof[i] + 2];
            vz = h.molevel[3 * h.molof[i] + 2];
        } else {
            pz = o.atmcor[3 * i + 2];
            vz = o.atmvel[3 * i + 2];
        }
        pz = wrap1(pz, o.box[2]);
        for (int r = 0; r < h.nreg; ++r) {
            if (!(h.z1[r] <= pz && pz <= h.z2[r])) continue;
            const double* v = &o.atmvel[3 * i];
            double kin = 0.5 * o.atmmass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            double* rec = out + (size_t)r * PGK_HF_NCOL;
            rec[0] += kin * vz;
            for (int c = 0; c < 8; ++c) rec[1 + c] += h.pot[(size_t)c * n + i] * vz;
        }
    }
    for (int r = 0; r < h.nreg; ++r) {   // :1020-1330 collision (virial) part
        double* rec = out + (size_t)r * PGK_HF_NCOL;
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 8; ++c)
                rec[9 + c] += h.W[widx(o, c, r, 0, i)] * o.atmvel[3 * i]
                            + h.W[widx(o, c, r, 1, i)] * o.atmvel[3 * i + 1]
                            + h.W[widx(o, c, r, 2, i)] * o.atmvel[3 * i + 2];
    }
    double area_inv = (1.0 / o.box[0]) * (1.0 / o.box[1]);
    for (int r = 0; r < h.nreg; ++r) {   // :1331-1460
        double vol_inv = area_inv / (h.z2[r] - h.z1[r]);
        double* rec = out + (size_t)r * PGK_HF_NCOL;
        double tot = 0.0;
        for (int c = 0; c < 17; ++c) { rec[c] = rec[c] * vol_inv; tot += rec[c]; }
        rec[17] = tot;
    }
}

// ---- counter-based normal deviates for langevin_region ----------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011), counter (atom, step lo, step hi, draw), key = seed.
// The reference draws from SFMT (genrand_res53); the device engine uses the
// same counter-based stream as this restatement, so the two agree draw for
// draw and the reference agrees in distribution.
void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}
// uniform on (0, 1] with 53 random bits
inline double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 1.0) * (1.0 / 9007199254740992.0);
}
void lt_draw(uint64_t seed, long long step, int atom, double* u) {
    for (int call = 0; call < 2; ++call) {
        uint32_t c[4] = {(uint32_t)atom, (uint32_t)(uint64_t)step, (uint32_t)((uint64_t)step >> 32), (uint32_t)call};
        philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        u[2 * call] = u53(c[0], c[1]);
        u[2 * call + 1] = u53(c[2], c[3]);
    }
}

// langevin_regist.F90:8-360: region of each atom (first matching region)
bool lt_inside(const Oracle::HF& h, int r, const double* g, const double* box) {
    auto in = [](double lo, double hi, double x, double L) {
        return (lo <= x && x < hi) || (lo <= x - L && x - L < hi);
    };
    return in(h.lx1[r], h.lx2[r], g[0], box[0]) && in(h.ly1[r], h.ly2[r], g[1], box[1]) &&
           in(h.lz1[r], h.lz2[r], g[2], box[2]);
}
void langevin_regist(Oracle& o) {
    Oracle::HF& h = o.hf;
    h.ltreg.assign(o.natom, -1);
    int nm = (int)o.molidx.size() - 1;
    for (int m = 0; m < nm; ++m) {
        int b = o.molidx[m], e = o.molidx[m + 1];
        if (h.ltmole[m] && e - b > 1) {
            double mass = 0.0, g[3] = {0, 0, 0};
            for (int q = b; q < e; ++q) {
                int i = o.mollist[q];
                mass = mass + o.atmmass[i];
                for (int d = 0; d < 3; ++d) g[d] = g[d] + o.atmmass[i] * o.atmcor[3 * i + d];
            }
            for (int d = 0; d < 3; ++d) g[d] = wrap1(g[d] / mass, o.box[d]);
            for (int r = 0; r < h.nlt; ++r)
                if (lt_inside(h, r, g, o.box)) {
                    for (int q = b; q < e; ++q) h.ltreg[o.mollist[q]] = r;
                    break;
                }
        } else {
            for (int q = b; q < e; ++q) {
                int i = o.mollist[q];
                double g[3];
                for (int d = 0; d < 3; ++d) g[d] = wrap1(o.atmcor[3 * i + d], o.box[d]);
                for (int r = 0; r < h.nlt; ++r)
                    if (lt_inside(h, r, g, o.box)) { h.ltreg[i] = r; break; }
            }
        }
    }
}

// langevin_region.F90:8-203 (streaming velocity zero)
void langevin_region(Oracle& o, double dt, long long step, bool former) {
    Oracle::HF& h = o.hf;
    int n = o.natom;
    double ek0[8] = {0}, ek1[8] = {0};
    if (h.ifoutthc)
        for (int i = 0; i < n; ++i) {
            int r = h.ltreg[i];
            if (r < 0) continue;
            const double* v = &o.atmvel[3 * i];
            ek0[r] += o.atmmass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
    const double pi = std::acos(-1.0);
    if (former) {
        h.frand.assign((size_t)3 * n, 0.0);
        for (int i = 0; i < n; ++i) {
            int r = h.ltreg[i];
            if (r < 0) continue;
            double var = 2.0 * h.ldamp[r] * h.ltemp[r] / dt * o.atmmass[i];
            double u[4];
            lt_draw(h.seed, step, i, u);
            double a = std::sqrt(-2.0 * std::log(u[0]) * var);
            double f0 = a * std::cos(2.0 * pi * u[1]);
            double f1 = a * std::sin(2.0 * pi * u[1]);
            double f2 = std::sqrt(-2.0 * std::log(u[2]) * var) * std::cos(2.0 * pi * u[3]);
            h.frand[3 * i] = f0 / o.atmmass[i];
            h.frand[3 * i + 1] = f1 / o.atmmass[i];
            h.frand[3 * i + 2] = f2 / o.atmmass[i];
        }
        for (int i = 0; i < n; ++i) {
            int r = h.ltreg[i];
            if (r < 0) continue;
            double ex = std::exp(-0.5 * dt * h.ldamp[r]);
            for (int d = 0; d < 3; ++d) {
                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] + 0.5 * dt * h.frand[3 * i + d];
                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] * ex;
            }
        }
    } else {
        for (int i = 0; i < n; ++i) {
            int r = h.ltreg[i];
            if (r < 0) continue;
            double ex = std::exp(-0.5 * dt * h.ldamp[r]);
            for (int d = 0; d < 3; ++d) {
                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] * ex;
                o.atmvel[3 * i + d] = o.atmvel[3 * i + d] + 0.5 * dt * h.frand[3 * i + d];
            }
        }
    }
    if (h.ifoutthc) {
        for (int i = 0; i < n; ++i) {
            int r = h.ltreg[i];
            if (r < 0) continue;
            const double* v = &o.atmvel[3 * i];
            ek1[r] += o.atmmass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
        for (int r = 0; r < h.nlt; ++r) h.dekin[r] += 0.5 * (ek1[r] - ek0[r]);
    }
}

bool hf_step(const Oracle& o, long long step) {
    return o.hf.nreg > 0 && step > 0 && (o.hf.heatfinterval == 1 || step % o.hf.heatfinterval == 1);
}

// moldyn_hf.F90:1405-2480: NVE XO-RESPA + region Langevin + heat flux
int moldyn_hf(Oracle& o, long long ini, long long end, const pgk_mdparams& md, pgk_energies* eout,
              std::vector<double>* records) {
    int n = o.natom;
    Forces& F = o.F;
    double dtl = md.dt_long_cal, dts = md.dt_long_cal / (double)md.nstep_short;
    std::vector<double> old((size_t)3 * n);
    if (F.fl.size() != (size_t)3 * n) { F.fl.assign((size_t)3 * n, 0.0); F.fs.assign((size_t)3 * n, 0.0); }
    auto force_eval = [&](int flag) {
        if (flag == PGK_MTS_LONG) { calforce(o, flag, F.fl.data(), &F.el, &F.vl); accforce(o, F.fl); }
        else { calforce(o, flag, F.fs.data(), &F.es, &F.vs); accforce(o, F.fs); }
    };
    bool lt = o.hf.nlt > 0;
    for (long long step = ini; step <= end; ++step) {
        if (step % md_nbook(o) == 1 || md_nbook(o) == 1 || step == 0) transcor(o);
        if (step % md_nbook(o) == 0 || md_nbook(o) == 1) mklist(o);
        bool hfs = hf_step(o, step);
        if (step == 0) {
            if (lt) langevin_regist(o);
            force_eval(PGK_MTS_SHORT);
            force_eval(PGK_MTS_LONG);
        } else {
            if (lt) langevin_region(o, dtl, step, true);
            for (int is = 1; is <= md.nstep_short; ++is) {
                if (is == 1) for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dtl * F.fl[k];
                for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dts * F.fs[k];
                if (md.ifrattle && o.ci.size()) old = o.atmcor;
                for (int k = 0; k < 3 * n; ++k) o.atmcor[k] = o.atmcor[k] + dts * o.atmvel[k];
                if (md.ifrattle && o.ci.size()) {
                    int s = rattle_pos(o, old.data(), md.eps_rattle, dts, nullptr);
                    if (s) return s;
                }
                o.hf.ewk_now = hfs && is == md.nstep_short && o.hf.kspace == PGK_HF_KSPACE_EWK;
                force_eval(PGK_MTS_SHORT);
                if (is == md.nstep_short) {
                    force_eval(PGK_MTS_LONG);
                    if (hfs) calforce_hf_atm(o);
                }
                o.hf.ewk_now = false;
                for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dts * F.fs[k];
                if (is == md.nstep_short)
                    for (int k = 0; k < 3 * n; ++k) o.atmvel[k] = o.atmvel[k] + 0.5 * dtl * F.fl[k];
                if (md.ifrattle && o.ci.size()) {
                    int s = rattlep_v(o, md.eps_rattle);
                    if (s) return s;
                }
            }
            if (lt) { langevin_regist(o); langevin_region(o, dtl, step, false); }
            if (hfs && records) {
                size_t b = records->size();
                records->resize(b + (size_t)o.hf.nreg * PGK_HF_NCOL);
                calheatf(o, records->data() + b);
            }
        }
        if (eout && (md.outinterval <= 0 ? step == end : step % md.outinterval == 0)) {
            pgk_energies e{};
            e.pot_vdw = F.el.pot_vdw + F.es.pot_vdw; e.pot_elc = F.el.pot_elc + F.es.pot_elc;
            e.pot_ewk = F.el.pot_ewk + F.es.pot_ewk; e.pot_ewc = F.el.pot_ewc + F.es.pot_ewc;
            e.pot_ewnq = F.el.pot_ewnq + F.es.pot_ewnq;
            e.pot_vdw14 = F.el.pot_vdw14 + F.es.pot_vdw14; e.pot_elc14 = F.el.pot_elc14 + F.es.pot_elc14;
            e.pot_bond = F.el.pot_bond + F.es.pot_bond; e.pot_angl = F.el.pot_angl + F.es.pot_angl;
            e.pot_tors = F.el.pot_tors + F.es.pot_tors; e.pot_torsrb = F.el.pot_torsrb + F.es.pot_torsrb;
            e.pot_mor = F.el.pot_mor + F.es.pot_mor;
            e.pot_nonbon = F.el.pot_nonbon + F.es.pot_nonbon; e.pot_tot = F.el.pot_tot + F.es.pot_tot;
            *eout = e;
        }
    }
    return PGK_OK;
}

// prepewk.F90:100-135: integer wave vectors in the reference's kx, ky, kz loop
// order, (0,0,0) first (nwave = 1 is reserved for it); yratio and zratio are
// the initial box ratios (rdscript.F90:1494)
int ewk_nvec(int kmax, double yratio, double zratio, std::vector<int>& nv) {
    const int ny0 = (int)std::round(yratio), nz0 = (int)std::round(zratio);   // anint, prepewk.F90:73-76
    if (kmax < 1 || ny0 < 1 || nz0 < 1) return PGK_E_INVALID;
    const int yk = kmax * ny0, zk = kmax * nz0;
    nv.assign(3, 0);
    for (int kx = -kmax; kx <= kmax; ++kx)
        for (int ky = -yk; ky <= yk; ++ky)
            for (int kz = -zk; kz <= zk; ++kz) {
                if (kx == 0 && ky == 0 && kz == 0) continue;
                double a2 = (double)(kx * kx) + (double)(ky * ky) / (double)(ny0 * ny0) +
                            (double)(kz * kz) / (double)(nz0 * nz0);
                if (a2 <= (double)(kmax * kmax)) { nv.push_back(kx); nv.push_back(ky); nv.push_back(kz); }
            }
    return PGK_OK;
}

// ewaldkp_hf (ewaldk_hf.F90:8-304) with kwave/awave of prepewk.F90:137-155 at
// the current box.  Outputs hold this term alone: force (3,N), pot_atm (N)
// with the self term, viri (3,3,N) = virielct_atm(:,:,i,1), sc = pot_ewk,
// pot_ewk_cc, pot_virit_coul(3,3).
int ewaldkp_hf(Oracle& o, int kmax, double* force, double* pot_atm, double* viri, double* sc, int* nwave_out) {
    std::vector<int> nv;
    int s = ewk_nvec(kmax, o.prm.ycel / o.prm.xcel, o.prm.zcel / o.prm.xcel, nv);
    if (s) return s;
    const int n = o.natom, nwave = (int)nv.size() / 3;
    const double pi = std::acos(-1.0), pi2 = 2.0 * pi;
    const double* box = o.box;
    const double vol = box[0] * box[1] * box[2];
    const double pot_fact = 0.5 / pi / vol, inv_vol = 1.0 / vol;
    const double alpha = o.prm.alpha, fac_vir = 2.0 * pi * pi * (1.0 / (alpha * alpha));
    const double alpha_sqrtpi = alpha / std::sqrt(pi);
    const double coeff = (pi / alpha) * (pi / alpha);
    const bool cc = o.prm.ifnetqcorrp != 0;
    std::vector<double> kw((size_t)3 * nwave), aw(nwave, 0.0);
    for (int k = 0; k < nwave; ++k) {
        for (int d = 0; d < 3; ++d) kw[3 * k + d] = (double)nv[3 * k + d] / box[d];
        if (k == 0) continue;
        double x = (double)nv[3 * k] / box[0], y = (double)nv[3 * k + 1] / box[1], z = (double)nv[3 * k + 2] / box[2];
        double a2 = x * x + y * y + z * z;
        aw[k] = std::exp(-coeff * a2) / a2;
    }
    std::vector<double> fi((size_t)3 * n, 0.0), pa(n, 0.0), va((size_t)9 * n, 0.0), sini(n), cosi(n);
    double pot_ewk = 0.0, pot_ewk_cc = 0.0, vt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double* r = o.atmcor.data();
    const double* q = o.atmchrg.data();
    for (int k = 0; k < nwave; ++k) {
        const double* K = &kw[3 * k];
        double bsk = 0.0, bck = 0.0;
        for (int i = 0; i < n; ++i) {
            double th = K[0] * r[3 * i] + K[1] * r[3 * i + 1] + K[2] * r[3 * i + 2];
            th = pi2 * th;
            sini[i] = std::sin(th);
            cosi[i] = std::cos(th);
            bsk = bsk + q[i] * sini[i];
            bck = bck + q[i] * cosi[i];
        }
        const double pfa = pot_fact * aw[k];
        const double poti = pfa * (bsk * bsk + bck * bck);
        pot_ewk = pot_ewk + poti;
        for (int i = 0; i < n; ++i) pa[i] = pa[i] + pfa * q[i] * (sini[i] * bsk + cosi[i] * bck);
        double csk[3], cck[3];
        for (int d = 0; d < 3; ++d) { csk[d] = aw[k] * bsk * K[d]; cck[d] = aw[k] * bck * K[d]; }
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) fi[3 * i + d] = fi[3 * i + d] + cck[d] * sini[i] - csk[d] * cosi[i];
        if (k == 0) continue;   // ewaldk_hf.F90:186
        const double k2 = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
        double fac3 = 0.0;
        if (cc) {   // ewaldk_hf.F90:236-240
            fac3 = pfa * o.netchrgsq;
            pot_ewk_cc = pot_ewk_cc + fac3 * (-1.0 + fac_vir * k2);
        }
        // k_fact(a,b) = (delta_ab - (2/|K|^2 + fac_vir) K_a K_b) * factor
        auto kfact = [&](double f, double* dst) {
            for (int b = 0; b < 3; ++b) {
                double col[3];
                for (int a = 0; a < 3; ++a) col[a] = -1.0 * (2.0 / k2 + fac_vir) * K[a] * K[b];
                col[b] = col[b] + 1.0;
                for (int a = 0; a < 3; ++a) dst[a + 3 * b] = dst[a + 3 * b] + col[a] * f;
            }
        };
        kfact(poti - fac3, vt);
        for (int i = 0; i < n; ++i) kfact(pfa * q[i] * (sini[i] * bsk + cosi[i] * bck) - fac3, &va[(size_t)9 * i]);
    }
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) fi[3 * i + d] = 2.0 * q[i] * inv_vol * fi[3 * i + d];
        pa[i] = pa[i] - alpha_sqrtpi * (q[i] * q[i]);
    }
    if (force) std::copy(fi.begin(), fi.end(), force);
    if (pot_atm) std::copy(pa.begin(), pa.end(), pot_atm);
    if (viri) std::copy(va.begin(), va.end(), viri);
    if (sc) {
        sc[0] = pot_ewk; sc[1] = pot_ewk_cc;
        for (int t = 0; t < 9; ++t) sc[2 + t] = vt[t];
    }
    if (nwave_out) *nwave_out = nwave;
    return PGK_OK;
}
}  // namespace

// ============================================================================
// C entry points (ctypes)
// ============================================================================
extern "C" {

void* orc_create(const pgk_system* s, const pgk_params* p) {
    Oracle* o = new Oracle();
    o->prm = *p;
    int n = s->natom;
    o->natom = n;
    o->atmmass.assign(s->atmmass, s->atmmass + n);
    o->atmchrg.assign(s->atmchrg, s->atmchrg + n);
    o->atmindex.resize(n);
    for (int i = 0; i < n; ++i) o->atmindex[i] = s->atmindex[i] - 1;
    o->ntyp = s->ntyp;
    o->radij.assign(s->vdw_radij, s->vdw_radij + s->ntyp * s->ntyp);
    o->welij.assign(s->vdw_welij, s->vdw_welij + s->ntyp * s->ntyp);
    if (s->inter_inttyp) o->inttyp.assign(s->inter_inttyp, s->inter_inttyp + s->ntyp * s->ntyp);
    if (s->inter_inttyp && s->para_welmor && s->para_radmor && s->para_alphamor) {
        const int t2 = s->ntyp * s->ntyp;
        bool any = false;
        for (int k = 0; k < t2; ++k) any = any || s->inter_inttyp[k] == 2;
        if (any) {
            o->welmor.assign(s->para_welmor, s->para_welmor + t2);
            o->radmor.assign(s->para_radmor, s->para_radmor + t2);
            o->almor.assign(s->para_alphamor, s->para_alphamor + t2);
            std::vector<char> mt(s->ntyp, 0);   // types with a Morse partner
            for (int a = 0; a < s->ntyp; ++a)
                for (int b = 0; b < s->ntyp; ++b) mt[a] = mt[a] || s->inter_inttyp[a + s->ntyp * b] == 2;
            for (int i = 0; i < n; ++i)
                if (mt[s->atmindex[i] - 1]) o->mor_atoms.push_back(i);
        }
    }
    o->molidx.resize(s->nmole + 1);
    for (int m = 0; m <= s->nmole; ++m) o->molidx[m] = s->molept_index[m] - 1;
    o->mollist.resize(o->molidx[s->nmole]);
    for (size_t q = 0; q < o->mollist.size(); ++q) o->mollist[q] = s->molept_list[q] - 1;
    o->excl_idx.assign(s->index_excl, s->index_excl + n + 1);
    o->excl_list.assign(s->list_excl, s->list_excl + (s->index_excl[n] - 1));
    for (int k = 0; k < s->nbond; ++k) {
        o->bi.push_back(s->ibond[k] - 1); o->bj.push_back(s->jbond[k] - 1);
        o->bk.push_back(s->para_cbond[k]); o->br0.push_back(s->para_eqbond[k]);
    }
    for (int k = 0; k < s->nangl; ++k) {
        o->ai.push_back(s->iangl[k] - 1); o->aj.push_back(s->jangl[k] - 1); o->ak.push_back(s->kangl[k] - 1);
        o->akk.push_back(s->para_cangl[k]); o->at0.push_back(s->para_eqangl[k]);
    }
    for (int k = 0; k < s->ntors; ++k) {
        o->ti.push_back(s->itors[k] - 1); o->tj.push_back(s->jtors[k] - 1);
        o->tk.push_back(s->ktors[k] - 1); o->tl.push_back(s->ltors[k] - 1);
        o->tdiv.push_back(s->para_divfac[k]); o->tbar.push_back(s->para_barhig[k]);
        o->tph.push_back(s->para_phsang[k]); o->tper.push_back(s->para_period[k]);
    }
    for (int k = 0; k < s->ntorsrb; ++k) {
        o->rbi.push_back(s->itorsrb[k] - 1); o->rbj.push_back(s->jtorsrb[k] - 1);
        o->rbk.push_back(s->ktorsrb[k] - 1); o->rbl.push_back(s->ltorsrb[k] - 1);
        for (int q = 0; q < 6; ++q) o->rbc.push_back(s->para_barhigrb[6 * k + q]);
    }
    // 1-4 pairs in calnon14p order: periodic torsions, then RB torsions
    if (s->ifcalnonb14)
        for (int k = 0; k < s->ntors; ++k) {
            if (!s->ifcalnonb14[k]) continue;
            int i = s->itors[k] - 1, j = s->ltors[k] - 1;
            if (i == j) continue;
            o->p14i.push_back(i); o->p14j.push_back(j);
            o->p14v.push_back(1.0 / s->para_divfac_vdw[k] * s->ring14[k]);
            o->p14e.push_back(1.0 / s->para_divfac_elc[k] * s->ring14[k]);
        }
    if (s->ifcalnonb14_rb)
        for (int k = 0; k < s->ntorsrb; ++k) {
            if (!s->ifcalnonb14_rb[k]) continue;
            int i = s->itorsrb[k] - 1, j = s->ltorsrb[k] - 1;
            if (i == j) continue;
            o->p14i.push_back(i); o->p14j.push_back(j);
            o->p14v.push_back(1.0 / s->para_divfac_vdwrb[k] * s->ring14_rb[k]);
            o->p14e.push_back(1.0 / s->para_divfac_elcrb[k] * s->ring14_rb[k]);
        }
    o->cidx.resize(s->nconst + 1);
    for (int g = 0; g <= s->nconst; ++g) o->cidx[g] = s->index_mconst[g] - 1;
    for (int q = 0; q < o->cidx[s->nconst]; ++q) o->clist.push_back(s->list_mconst[q] - 1);
    for (int c = 0; c < s->nconstraint; ++c) {
        o->ci.push_back(s->iconst[c] - 1); o->cj.push_back(s->jconst[c] - 1); o->cd.push_back(s->dconst[c]);
    }
    o->degfree = s->degfree_all;
    o->box[0] = p->xcel; o->box[1] = p->ycel; o->box[2] = p->zcel;
    o->yratio = p->ycel / p->xcel; o->zratio = p->zcel / p->xcel;
    o->atmcor.assign((size_t)3 * n, 0.0);
    o->atmvel.assign((size_t)3 * n, 0.0);
    spline_init(*o);
    spme_init(*o);
    o->rkcut = erf_corr_cutoff(o->box, p->nfft1, p->nfft2, p->nfft3);
    for (int d = 0; d < 3; ++d) o->ch.xboxh[d] = o->box[d];
    o->ch.xlogv = std::log(o->box[0] * o->box[1] * o->box[2]) / 3.0;
    return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }
void orc_set_threads(void* h, int t) { ((Oracle*)h)->nthreads = t < 1 ? 1 : t; }

void orc_set_state(void* h, const double* cor, const double* vel, const double* box) {
    Oracle* o = (Oracle*)h;
    std::copy(cor, cor + 3 * o->natom, o->atmcor.begin());
    if (vel) std::copy(vel, vel + 3 * o->natom, o->atmvel.begin());
    if (box) {
        for (int d = 0; d < 3; ++d) o->box[d] = box[d];
        o->rkcut = erf_corr_cutoff(o->box, o->prm.nfft1, o->prm.nfft2, o->prm.nfft3);
    }
}
void orc_get_state(void* h, double* cor, double* vel, double* box) {
    Oracle* o = (Oracle*)h;
    if (cor) std::copy(o->atmcor.begin(), o->atmcor.end(), cor);
    if (vel) std::copy(o->atmvel.begin(), o->atmvel.end(), vel);
    if (box) for (int d = 0; d < 3; ++d) box[d] = o->box[d];
}
void orc_set_chain(void* h, const pgk_chain* c) { ((Oracle*)h)->ch = *c; }
void orc_get_chain(void* h, pgk_chain* c) { *c = ((Oracle*)h)->ch; }

int orc_transcor(void* h) { transcor(*(Oracle*)h); return 0; }

// returns mode used (PGK_LIST_CELL / PGK_LIST_ALLPAIR); copies the CSR when cap suffices
int orc_mklist(void* h, int32_t* nb_index, int32_t* nb_list, long long cap, long long* nlist) {
    Oracle* o = (Oracle*)h;
    mklist(*o);
    *nlist = o->nlistnball;
    if (nb_index) std::copy(o->nb_index.begin(), o->nb_index.begin() + o->natom, nb_index);
    if (nb_list && cap >= o->nlistnball) std::copy(o->nb_list.begin(), o->nb_list.end(), nb_list);
    return o->list_used_mode;
}

int orc_ewaldrp(void* h, double* force, pgk_energies* e, pgk_virials* v) {
    ewaldrp(*(Oracle*)h, force, e, v); return 0;
}
int orc_fft_pmep(void* h, double* force, pgk_energies* e, pgk_virials* v) {
    fft_pmep(*(Oracle*)h, force, e, v); return 0;
}
int orc_bonded(void* h, double* force, pgk_energies* e, pgk_virials* v) {
    Oracle& o = *(Oracle*)h;
    pgk_energies E{}; pgk_virials V{};
    calbondp(o, force, E.pot_bond, V.atm_viri_bond, V.atm_virit_bond);
    calanglp(o, force, E.pot_angl, V.atm_viri_angl, V.atm_virit_angl);
    caltorsp(o, force, E.pot_tors, V.atm_viri_tors, V.atm_virit_tors);
    caltorsrbp(o, force, E.pot_torsrb, V.atm_viri_tors, V.atm_virit_tors);
    calnon14p(o, force, E.pot_elc14, E.pot_vdw14, V.atm_viri_14, V.atm_virit_14);
    if (e) { e->pot_bond = E.pot_bond; e->pot_angl = E.pot_angl; e->pot_tors = E.pot_tors;
             e->pot_torsrb = E.pot_torsrb; e->pot_elc14 = E.pot_elc14; e->pot_vdw14 = E.pot_vdw14; }
    if (v) {
        v->atm_viri_bond = V.atm_viri_bond; v->atm_viri_angl = V.atm_viri_angl;
        v->atm_viri_tors = V.atm_viri_tors; v->atm_viri_14 = V.atm_viri_14;
        for (int k = 0; k < 9; ++k) {
            v->atm_virit_bond[k] = V.atm_virit_bond[k]; v->atm_virit_angl[k] = V.atm_virit_angl[k];
            v->atm_virit_tors[k] = V.atm_virit_tors[k]; v->atm_virit_14[k] = V.atm_virit_14[k];
        }
    }
    return o.status;
}
int orc_calforce(void* h, int flag, double* force, pgk_energies* e, pgk_virials* v) {
    calforce(*(Oracle*)h, flag, force, e, v); return ((Oracle*)h)->status;
}
int orc_rattle_c(void* h, const double* old, double eps, double dt) {
    return rattle_pos(*(Oracle*)h, old, eps, dt, nullptr);
}
int orc_rattle_cmtk(void* h, const double* old, double eps, double dt, const double* rvinv) {
    return rattle_pos(*(Oracle*)h, old, eps, dt, rvinv);
}
int orc_rattlep_v(void* h, double eps) { return rattlep_v(*(Oracle*)h, eps); }
int orc_nhcint(void* h, const pgk_mdparams* md) { nhcint(*(Oracle*)h, *md, md->dt_long_cal); return 0; }
int orc_nhcpisoint(void* h, const pgk_mdparams* md) { nhcpisoint(*(Oracle*)h, *md, md->dt_long_cal); return 0; }
int orc_nhcpanisoint(void* h, const pgk_mdparams* md) { nhcpanisoint(*(Oracle*)h, *md, md->dt_long_cal); return 0; }
double orc_kint(void* h) { return kint_sum(*(Oracle*)h); }
int orc_calpress(void* h, const pgk_virials* vl, const pgk_virials* vs, double* ptot, double* pt) {
    calpress(*(Oracle*)h, *vl, *vs, ptot, pt); return 0;
}
double orc_rkcut(void* h) { return ((Oracle*)h)->rkcut; }
double orc_pot_ewc(void* h) { return ((Oracle*)h)->pot_ewc; }

// spline evaluation (table k: 0 real force, 1 real pot, 2 excl force, 3 excl pot)
double orc_spline(void* h, int k, double x) { return spl(*(Oracle*)h, k, x); }
void orc_fill_bspline(double w, int order, double* arr, double* darr) { fill_bspline(w, order, arr, darr); }
void orc_bsp_mod(void* h, int dim, double* out) {
    Oracle* o = (Oracle*)h; std::copy(o->bsp[dim].begin(), o->bsp[dim].end(), out);
}
// complex FFT of n points (interleaved re,im), sign -1 = cfftf, +1 = cfftb
void orc_fft1d(double* data, int n, int sign) { fft1d((cplx*)data, n, 1, sign); }

int orc_moldyn(void* h, int kind, long long ini, long long end, const pgk_mdparams* md, pgk_energies* e) {
    Oracle& o = *(Oracle*)h;
    return moldyn(o, kind, ini, end, *md, e, o.F);
}


int orc_set_hf(void* h, const pgk_hfparams* p) {
    Oracle* o = (Oracle*)h;
    Oracle::HF& f = o->hf;
    if (p->nhfregion < 0 || p->nhfregion > PGK_HF_MAX_REGIONS || p->nlangeregion < 0 ||
        p->nlangeregion > PGK_LT_MAX_REGIONS || (p->nhfregion > 0 && p->ifhfvol != 1))
        return PGK_E_INVALID;
    f.set = true;
    f.nreg = p->nhfregion;
    f.heatfinterval = p->heatfinterval > 0 ? p->heatfinterval : 1;
    f.nlt = p->nlangeregion;
    f.ifoutthc = p->ifoutthc;
    f.seed = p->seed;
    for (int r = 0; r < PGK_HF_MAX_REGIONS; ++r) { f.z1[r] = p->hfzpos1[r]; f.z2[r] = p->hfzpos2[r]; }
    for (int r = 0; r < PGK_LT_MAX_REGIONS; ++r) {
        f.lx1[r] = p->ltxpos1[r]; f.lx2[r] = p->ltxpos2[r]; f.ly1[r] = p->ltypos1[r]; f.ly2[r] = p->ltypos2[r];
        f.lz1[r] = p->ltzpos1[r]; f.lz2[r] = p->ltzpos2[r]; f.ltemp[r] = p->r_ltemp[r]; f.ldamp[r] = p->r_ltdamp[r];
        f.dekin[r] = 0.0;
    }
    int n = o->natom, nm = (int)o->molidx.size() - 1;
    f.hftyp.assign(n, PGK_HFTYP_ATOM);
    if (p->hftyp_atm) for (int i = 0; i < n; ++i) f.hftyp[i] = p->hftyp_atm[i];
    f.molof.assign(n, 0);
    for (int m = 0; m < nm; ++m)
        for (int q = o->molidx[m]; q < o->molidx[m + 1]; ++q) f.molof[o->mollist[q]] = m;
    f.ltmole.assign(nm, 0);
    if (p->lt_mole_based) for (int m = 0; m < nm; ++m) f.ltmole[m] = p->lt_mole_based[m];
    f.frand.assign((size_t)3 * n, 0.0);
    if (f.nlt > 0) langevin_regist(*o);
    return PGK_OK;
}
int orc_calheatf(void* h, double* out) {
    Oracle* o = (Oracle*)h;
    if (!o->hf.set || o->hf.nreg < 1) return PGK_E_INVALID;
    if (o->nb_index.empty()) mklist(*o);
    calforce_hf_atm(*o);
    calheatf(*o, out);
    return PGK_OK;
}
int orc_get_hf_atm(void* h, double* pot, double* W) {
    Oracle* o = (Oracle*)h;
    if (pot) std::copy(o->hf.pot.begin(), o->hf.pot.end(), pot);
    if (W) std::copy(o->hf.W.begin(), o->hf.W.end(), W);
    return PGK_OK;
}
int orc_moldyn_hf(void* h, long long ini, long long end, const pgk_mdparams* md, pgk_energies* e, double* rec,
                  long long cap, long long* nrec) {
    Oracle* o = (Oracle*)h;
    std::vector<double> r;
    int s = moldyn_hf(*o, ini, end, *md, e, &r);
    long long per = (long long)o->hf.nreg * PGK_HF_NCOL;
    long long nr = per > 0 ? (long long)r.size() / per : 0;
    if (rec) std::copy(r.begin(), r.begin() + (size_t)std::min(nr, cap) * per, rec);
    if (nrec) *nrec = nr;
    return s;
}
void orc_langevin_dekin(void* h, double* out) {
    Oracle* o = (Oracle*)h;
    for (int r = 0; r < o->hf.nlt; ++r) { out[r] = o->hf.dekin[r]; o->hf.dekin[r] = 0.0; }
}
void orc_lt_regions(void* h, int* out) {
    Oracle* o = (Oracle*)h;
    std::copy(o->hf.ltreg.begin(), o->hf.ltreg.end(), out);
}
void orc_philox(uint64_t seed, long long step, int atom, double* u) { lt_draw(seed, step, atom, u); }
int orc_ewk_nvec(int kmax, double yratio, double zratio, int* out, int cap, int* nwave) {
    std::vector<int> nv;
    int s = ewk_nvec(kmax, yratio, zratio, nv);
    if (s) return s;
    *nwave = (int)nv.size() / 3;
    if (out) std::copy(nv.begin(), nv.begin() + std::min((size_t)3 * cap, nv.size()), out);
    return PGK_OK;
}
// morsep_hf per-atom Morse energy (N) and virial (:,3,i,r) as W[(r*3 + a)*N + i]
int orc_morse_hf_atm(void* h, double* pot, double* W) {
    Oracle* o = (Oracle*)h;
    if (!o->hf.set || o->welmor.empty()) return PGK_E_INVALID;
    if (o->nb_index.empty()) mklist(*o);
    std::vector<double> w, p((size_t)o->natom);
    morsep_hf(*o, p.data(), w);
    if (pot) std::copy(p.begin(), p.end(), pot);
    if (W) std::copy(w.begin(), w.end(), W);
    return PGK_OK;
}
// Morse list of the last mklist: its order (PGK_LIST_*) and pair count
int orc_mor_list(void* h, long long* npair) {
    Oracle* o = (Oracle*)h;
    if (npair) *npair = (long long)o->mor_list.size();
    return o->mor_list_mode;
}
// the Morse list itself in the reference layout (mklist_mor_cell.F90:250-300):
// nmorselist (1-based atoms), mor_indexall rows 1..nmorse-1 (1-based starts,
// entry nmorse = nlistmorall + 1), mor_listall (1-based, 0 for an empty row)
int orc_get_mor_list(void* h, int* nmorselist, int* mor_index, int* mor_list, long long cap, long long* nl,
                     int* nmorse) {
    Oracle* o = (Oracle*)h;
    const int nm = (int)o->mor_atoms.size();
    if (nmorse) *nmorse = nm;
    if (nm == 0) { if (nl) *nl = 0; return PGK_OK; }
    long long icut = 0;
    for (int m = 0; m + 1 < nm; ++m) {
        if (mor_index) mor_index[m] = (int)(icut + 1);
        const int b = o->mor_idx[m], e = o->mor_idx[m + 1];
        if (b == e) {
            if (mor_list && icut < cap) mor_list[icut] = 0;
            ++icut;
            continue;
        }
        for (int q = b; q < e; ++q, ++icut)
            if (mor_list && icut < cap) mor_list[icut] = o->mor_list[q] + 1;
    }
    if (mor_index) mor_index[nm - 1] = (int)(icut + 1);
    if (nmorselist) for (int m = 0; m < nm; ++m) nmorselist[m] = o->mor_atoms[m] + 1;
    if (nl) *nl = icut;
    return PGK_OK;
}
// morsep alone at the current positions (force added, energies, virials)
int orc_morsep(void* h, double* force, pgk_energies* e, pgk_virials* v) {
    Oracle* o = (Oracle*)h;
    if (o->welmor.empty()) return PGK_E_INVALID;
    if (o->mor_idx.empty()) mklist_mor(*o);
    pgk_energies E{}; pgk_virials V{};
    morsep(*o, force, E.pot_mor, V.pot_viri_mor, V.pot_virit_mor);
    if (e) *e = E;
    if (v) *v = V;
    return PGK_OK;
}
int orc_set_hf_kspace(void* h, int mode, int kmax) {
    Oracle* o = (Oracle*)h;
    if (mode < PGK_HF_KSPACE_NONE || mode > PGK_HF_KSPACE_SPME || (mode == PGK_HF_KSPACE_EWK && kmax < 1))
        return PGK_E_INVALID;
    o->hf.kspace = mode;
    o->hf.kmax = kmax;
    o->hf.ewk_fresh = false;
    return PGK_OK;
}
int orc_spme_hf_atm(void* h, double* pot_atm, double* viri) {
    Oracle* o = (Oracle*)h;
    if (!o->prm.ifspme) return PGK_E_INVALID;
    spme_hf_atm(*o, pot_atm, viri);
    return PGK_OK;
}
int orc_ewaldkp_hf(void* h, int kmax, double* force, double* pot_atm, double* viri, double* sc, int* nwave) {
    return ewaldkp_hf(*(Oracle*)h, kmax, force, pot_atm, viri, sc, nwave);
}
void orc_philox_raw(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32(c, key[0], key[1]);
    for (int q = 0; q < 4; ++q) out[q] = c[q];
}
}  // extern "C"
