// pgk_api.cu -- C ABI of libpgkgpu.so (include/pgk_gpu.h): context set-up,
// state transfer, the fine-grained reference-named operations and the stage
// drivers that keep the whole XO-RESPA loop on the device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pgk_ctx.cuh"

// the device's memory pool of the contexts (see pgk_ctx.cuh): created on
// first use per device, release threshold at its maximum (memory stays cached)
static cudaMemPool_t device_pool() {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    pools[dev] = pool;
    return pool;
}

cudaError_t pgk_dmalloc(pgk_ctx* c, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes > 0 ? bytes : 1, c->pool, c->st);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    return cudaStreamSynchronize(c->st);
}

cudaError_t pgk_dfree(pgk_ctx* c, void* p) {
    if (!p) return cudaSuccess;
    return cudaFreeAsync(p, c->st);
}

cudaError_t smem_limit(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<const void*, size_t> limit;
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = limit[kernel];
    if (bytes <= cur) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

pgk_status spme_bench(pgk_ctx* c, int which);

pgk_status pgk_fail(pgk_ctx* c, pgk_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

namespace {

// natural cubic spline of spline_interp.F90:139-190 (cal_spl_coeff)
void spl_coeff(int n, double h, const std::vector<double>& x, const std::vector<double>& t, std::vector<double>& b,
               std::vector<double>& cc, std::vector<double>& d) {
    std::vector<double> al(n, 0.0), l(n, 0.0), mu(n, 0.0), z(n, 0.0);
    b.assign(n, 0.0); cc.assign(n, 0.0); d.assign(n, 0.0);
    for (int i = 1; i < n - 1; ++i) al[i] = 3.0 / h * ((t[i + 1] - t[i]) - (t[i] - t[i - 1]));
    l[0] = 1.0;
    for (int i = 1; i < n - 1; ++i) {
        l[i] = 2.0 * (x[i + 1] - x[i - 1]) - h * mu[i - 1];
        mu[i] = h / l[i];
        z[i] = (al[i] - h * z[i - 1]) / l[i];
    }
    for (int i = n - 2; i >= 0; --i) {
        cc[i] = z[i] - mu[i] * cc[i + 1];
        b[i] = (t[i + 1] - t[i]) / h - h * (cc[i + 1] + 2.0 * cc[i]) / 3.0;
        d[i] = (cc[i + 1] - cc[i]) / (3.0 * h);
    }
}

double rkcut_host(const double* box, int n1, int n2, int n3) {   // erf_corr_cutoff.F90
    double m1 = 0.5 * (n1 / box[0]);
    double rk = m1;
    double m2 = 0.5 * (n2 / box[1]);
    if (m2 < m1) rk = m2;
    double m3 = 0.5 * (n3 / box[2]);
    if (m3 < m2) rk = m3;
    return 0.9 * rk;
}

template <typename T>
pgk_status upload(pgk_ctx* c, T** dst, const std::vector<T>& v) {
    if (v.empty()) { *dst = nullptr; return PGK_OK; }
    PGK_CUDA(c, pgk_dmalloc(c, dst, v.size() * sizeof(T)));
    PGK_CUDA(c, cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PGK_OK;
}

pgk_status read_status(pgk_ctx* c) {
    unsigned st = 0;
    PGK_CUDA(c, cudaMemcpyAsync(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    if (!st) return PGK_OK;
    unsigned z = 0;
    PGK_CUDA(c, cudaMemsetAsync(c->status, 0, sizeof(z), c->st));
    if (st & ST_RATTLE_NOCONV) return pgk_fail(c, PGK_E_RATTLE_NOCONV, "ERROR: RATTLE(C) failed to converge within MAXITER = 300");
    if (st & ST_RATTLEV_NOCONV) return pgk_fail(c, PGK_E_RATTLEV_NOCONV, "ERROR: RATTLE(V) failed to converge within MAXITER = 300");
    if (st & ST_BOX_TOO_SMALL) return pgk_fail(c, PGK_E_BOX_TOO_SMALL, "Error: rcut is over half cell length");
    if (st & ST_LIST_OVERFLOW) return pgk_fail(c, PGK_E_LIST_OVERFLOW, "Error: nlistnball exceed number of nonbonded list");
    if (st & ST_CELL_OVERFLOW) return pgk_fail(c, PGK_E_CELL_OVERFLOW, "Error: number of atoms in cell exceeds max");
    if (st & ST_UNSUPPORTED) return pgk_fail(c, PGK_E_UNSUPPORTED, "Periodicity not supported");
    return pgk_fail(c, PGK_E_CUDA, "unknown device status");
}

// one MTS group of calforce (calforce.F90:8-1073); tensor_only selects the
// pair kernel's combined-tensor mode (anisotropic MTK steps without output)
// Three streams: the SPME chain on the second and the bonded terms on the
// third run beside the pack, the pair kernel and its finishing kernel on the
// context's stream (the pair kernel is issue-bound, the SPME and bonded
// kernels latency-bound, so they fill each other's idle issue slots).  The
// context's stream has the highest priority and the bonded terms wait for
// the prune decision, so the pair kernel's blocks are dispatched first.
// Every add into the shared force and energy accumulators is atomic (int64 in
// mixed precision: exact and independent of the interleaving).
pgk_status force_group(pgk_ctx* c, int flag, bool ene, bool vir, bool tensor_only = false) {
    int g = flag == PGK_MTS_LONG ? 0 : 1;
    pgk_status s;
    if ((s = launch_zero_group(c, g))) return s;
    const bool pairs = c->prm.mts_vdw == flag;
    if (pairs && !c->list_valid && (s = launch_mklist(c))) return s;
    const int mask = (c->prm.mts_bond == flag ? 1 : 0) | (c->prm.mts_angl == flag ? 2 : 0) |
                     (c->prm.mts_tors == flag ? 4 : 0) | (c->prm.mts_torsrb == flag ? 8 : 0) |
                     (c->prm.mts_vdw14 == flag && c->prm.mts_elc14 == flag ? 16 : 0) | (pairs ? 32 : 0);
    // _HF_BULK_EWK heat-flux step: ewaldkp_hf replaces the SPME term (calforce_hf.F90:1046-1062)
    const bool ewk_hf = c->hf_ewk_now && c->prm.mts_ewk == flag;
    const bool spme = c->prm.ifspme && c->prm.mts_ewk == flag && !ewk_hf;
    const bool fork = spme && c->st2 && (pairs || mask);
    // third stream: the bonded terms, released together with the pair kernel
    // (after the pack and the prune decision) so that the pair kernel's
    // blocks, on the higher-priority stream, take the SMs first and the
    // bonded blocks fill in beside them
    const bool third = fork && c->st3;
    if (fork) {
        PGK_CUDA(c, cudaEventRecord(c->ev_fork, c->st));
        PGK_CUDA(c, cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
        if (c->st3) PGK_CUDA(c, cudaStreamWaitEvent(c->st3, c->ev_fork, 0));
        cudaStream_t main_st = c->st;
        c->st = c->st2;
        s = launch_spme(c, g, ene, vir);
        if (!s && !third) s = launch_intra(c, g, mask, ene || vir, vir && tensor_only);
        c->st = main_st;
        if (s) return s;
        PGK_CUDA(c, cudaEventRecord(c->ev_join, c->st2));
    }
    bool bonded_after_pair = false;
    if (pairs) {
        if ((s = launch_pack(c))) return s;
        const int vmode = vir ? (tensor_only ? PM_TENS : PM_FULL) : (ene ? PM_ENE : PM_FORCE);
        c->rec_pre_pair = third;
        c->rec_pre_pair_done = false;
        s = launch_pair(c, g, vmode);
        bonded_after_pair = third && c->rec_pre_pair_done;
        c->rec_pre_pair = false;
        if (s) return s;
    }
    if (third) {
        if (bonded_after_pair) PGK_CUDA(c, cudaStreamWaitEvent(c->st3, c->ev_pre_pair, 0));
        cudaStream_t main_st = c->st;
        c->st = c->st3;
        s = launch_intra(c, g, mask, ene || vir, vir && tensor_only);
        c->st = main_st;
        if (s) return s;
        PGK_CUDA(c, cudaEventRecord(c->ev_join3, c->st3));
    }
    if (c->nmor && c->prm.mts_mor == flag && (s = launch_morse(c, g, ene || vir))) return s;   // calforce.F90:360-400
    if (fork) {
        PGK_CUDA(c, cudaStreamWaitEvent(c->st, c->ev_join, 0));
        if (c->st3) PGK_CUDA(c, cudaStreamWaitEvent(c->st, c->ev_join3, 0));
        return PGK_OK;
    }
    if (spme && (s = launch_spme(c, g, ene, vir))) return s;
    if (ewk_hf && (s = launch_ewk_force(c, g))) return s;
    return launch_intra(c, g, mask, ene || vir, vir && tensor_only);
}

double accv(const pgk_ctx* c, long long v) {
    if (c->mixed()) return (double)v * PGK_FORCE_ISCALE;
    double d;
    memcpy(&d, &v, sizeof(d));
    return d;
}

// energies / virials of the accumulators of the given groups
pgk_status read_acc(pgk_ctx* c, int gmask, pgk_energies* e, pgk_virials* v, bool add_ewald_consts) {
    std::vector<long long> a(2 * NACC);
    PGK_CUDA(c, cudaMemcpyAsync(a.data(), c->acc, sizeof(long long) * 2 * NACC, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    double S[NACC];
    for (int k = 0; k < NACC; ++k) {
        S[k] = 0;
        for (int g = 0; g < 2; ++g) if (gmask & (1 << g)) S[k] += accv(c, a[(size_t)g * NACC + k]);
    }
    for (int base : {A_VTC, A_VTLJ}) { S[base + 3] = S[base + 1]; S[base + 6] = S[base + 2]; S[base + 7] = S[base + 5]; }
    double pi = std::acos(-1.0);
    const double* b = c->hdyn.box;
    double a1 = -pi / (c->prm.alpha * c->prm.alpha * b[0] * b[1] * b[2]);
    if (add_ewald_consts && c->prm.ifspme) {
        if (!c->prm.ifnetqcorrp) {
            S[A_VC] += a1 * c->netchrgsq;
            for (int d = 0; d < 3; ++d) S[A_VTC + 4 * d] += 0.5 * a1 * c->netchrgsq;
        } else {
            S[A_VC] -= 0.5 * a1 * c->netchrgsq;
        }
    }
    if (e) {
        memset(e, 0, sizeof(*e));
        e->pot_vdw = S[A_VDW]; e->pot_elc = S[A_ELC]; e->pot_ewk = S[A_EWK];
        e->pot_vdw14 = S[A_VDW14]; e->pot_elc14 = S[A_ELC14];
        e->pot_bond = S[A_BOND]; e->pot_angl = S[A_ANGL]; e->pot_tors = S[A_TORS]; e->pot_torsrb = S[A_TORSRB];
        e->pot_mor = S[A_MOR];
        if (add_ewald_consts && c->prm.ifspme) { e->pot_ewc = c->pot_ewc; e->pot_ewnq = 0.5 * a1 * c->netchrgsq; }
        e->pot_nonbon = e->pot_vdw + e->pot_elc + e->pot_ewk + e->pot_ewc + e->pot_ewnq + e->pot_vdw14 + e->pot_elc14;
        e->pot_tot = e->pot_bond + e->pot_angl + e->pot_tors + e->pot_torsrb + e->pot_mor + e->pot_nonbon;
    }
    if (v) {
        memset(v, 0, sizeof(*v));
        v->pot_viri_coul = S[A_VC]; v->pot_viri_lj = S[A_VLJ];
        v->atm_viri_bond = S[A_VB]; v->atm_viri_angl = S[A_VA]; v->atm_viri_tors = S[A_VT]; v->atm_viri_14 = S[A_V14];
        v->pot_viri_mor = S[A_VMOR];
        for (int k = 0; k < 9; ++k) {
            v->pot_virit_coul[k] = S[A_VTC + k]; v->pot_virit_lj[k] = S[A_VTLJ + k];
            v->atm_virit_bond[k] = S[A_VTB + k]; v->atm_virit_angl[k] = S[A_VTA + k];
            v->atm_virit_tors[k] = S[A_VTT + k]; v->atm_virit_14[k] = S[A_VT14 + k];
            v->pot_virit_mor[k] = S[A_VTMOR + k];
        }
    }
    return PGK_OK;
}

pgk_status force_to_host(pgk_ctx* c, int g, double* force, bool add) {
    int n3 = 3 * c->natom;
    if (!c->fout) PGK_CUDA(c, pgk_dmalloc(c, &c->fout, sizeof(double) * n3));
    pgk_status s = launch_copy_force(c, g, c->fout);
    if (s) return s;
    c->hbuf.resize(n3);
    PGK_CUDA(c, cudaMemcpyAsync(c->hbuf.data(), c->fout, sizeof(double) * n3, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    for (int k = 0; k < n3; ++k) force[k] = add ? force[k] + c->hbuf[k] : c->hbuf[k];
    return PGK_OK;
}

pgk_status set_dyn_box(pgk_ctx* c, const double* box) {
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    for (int d = 0; d < 3; ++d) { c->hdyn.box[d] = box[d]; c->hdyn.boxinv[d] = 1.0 / box[d]; }
    c->hdyn.rkcut = rkcut_host(box, c->prm.nfft1, c->prm.nfft2, c->prm.nfft3);
    PGK_CUDA(c, cudaMemcpyAsync(c->dyn, &c->hdyn, sizeof(DynState), cudaMemcpyHostToDevice, c->st));
    return PGK_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char* pgk_version(void) { return "pgk-b200 1.0 (sm_100a)"; }

const char* pgk_status_string(pgk_status s) {
    switch (s) {
        case PGK_OK: return "ok";
        case PGK_E_LIST_OVERFLOW: return "Error: nlistnball(local) exceed number of nonbonded list";
        case PGK_E_CELL_OVERFLOW: return "Error: number of atoms in cell exceeds max (vdw and elc)";
        case PGK_E_RATTLE_NOCONV: return "ERROR: RATTLE(C) failed to converge within MAXITER";
        case PGK_E_BOX_TOO_SMALL: return "Error: rcut is over half cell length";
        case PGK_E_DEVICE_TIMEOUT: return "device wait timed out";
        case PGK_E_CUDA: return "CUDA error";
        case PGK_E_INVALID: return "invalid argument";
        case PGK_E_NOMEM: return "device memory exhausted";
        case PGK_E_UNSUPPORTED: return "unsupported option";
        case PGK_E_RATTLEV_NOCONV: return "ERROR: RATTLE(V) failed to converge within MAXITER";
        case PGK_E_SCRATCH_LIMIT: return "size exceeds the static scratch maximum of pgk_fft_pme_noalloc";
        default: return "unknown status";
    }
}

const char* pgk_last_error(const pgk_ctx* c) { return c ? c->err.c_str() : ""; }

}  // extern "C"

extern "C" {

pgk_status pgk_init(const pgk_system* s, const pgk_params* p, pgk_ctx** out) {
    if (!s || !p || !out) return PGK_E_INVALID;
    *out = nullptr;
    int n = s->natom;
    if (n >= (1 << 25)) return PGK_E_INVALID;   // sort key packs the atom index in 25 bits
    if (n < 2 || !s->atmmass || !s->atmchrg || !s->atmindex || !s->index_excl || !s->list_excl)
        return PGK_E_INVALID;
    if (p->precision != PGK_PREC_FP64 && p->precision != PGK_PREC_MIXED) return PGK_E_INVALID;
    if (p->rcut_book <= 0 || p->rcut <= 0 || p->rrcut <= 0) return PGK_E_INVALID;
    if (s->inter_inttyp)   // pair potentials other than LJ (md_global.inc:119-128) are not on the device
        for (int k = 0; k < s->ntyp * s->ntyp; ++k) {
            const int t = s->inter_inttyp[k];
            if (t < 1 || t > 10) return PGK_E_INVALID;
            if (t >= 3) return PGK_E_UNSUPPORTED;                            // SH, RFH, DOU, RP-VW, custom
            if (t == 2 && p->mts_mor != PGK_MTS_NONE && (!s->para_welmor || !s->para_radmor || !s->para_alphamor))
                return PGK_E_INVALID;                                        // Morse pair without parameters
        }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return PGK_E_CUDA;
    pgk_ctx* c = new pgk_ctx();
    if (const char* gv = getenv("PGK_GRAPHS")) c->use_graphs = atoi(gv) != 0;   // 0: launch MD steps eagerly
    c->natom = n;
    c->prec = p->precision;
    c->prm = *p;
    {
        const int S = PGK_MTS_SHORT;
        c->short_empty = p->mts_bond != S && p->mts_angl != S && p->mts_tors != S && p->mts_torsrb != S &&
                         p->mts_vdw != S && p->mts_ewk != S && p->mts_vdw14 != S && p->mts_elc14 != S;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
    // the context's stream (pack, pair kernel, integrator) at the highest
    // priority, the SPME and bonded streams at the lowest: blocks of the pair
    // kernel are dispatched before theirs when SMs free up
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio_hi) != cudaSuccess) { delete c; return PGK_E_CUDA; }
    c->pool = device_pool();
    if (!c->pool) { cudaStreamDestroy(c->st); delete c; return PGK_E_CUDA; }
    if (cudaStreamCreateWithPriority(&c->st2, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->st3, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join3, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_pre_pair, cudaEventDisableTiming) != cudaSuccess) {
        pgk_free(c);
        return PGK_E_CUDA;
    }
    if (const char* ns = getenv("PGK_STREAMS")) {       // 1: the whole force evaluation on one stream
        const int n = atoi(ns);       // 1: one stream; 2: the bonded terms after the SPME chain
        if (n <= 2) { cudaStreamDestroy(c->st3); c->st3 = nullptr; }
        if (n == 1) { cudaStreamDestroy(c->st2); c->st2 = nullptr; }
    }
    c->degfree = s->degfree_all;
    pgk_status st;
#define TRY(x) do { if ((st = (x)) != PGK_OK) { pgk_free(c); return st; } } while (0)
    // ---- atoms ----
    std::vector<double> mass(s->atmmass, s->atmmass + n), chrg(s->atmchrg, s->atmchrg + n);
    std::vector<int> typ(n);
    for (int i = 0; i < n; ++i) {
        typ[i] = s->atmindex[i] - 1;
        if (typ[i] < 0 || typ[i] >= s->ntyp) { pgk_free(c); return PGK_E_INVALID; }
    }
    TRY(upload(c, &c->mass, mass));
    {
        std::vector<double> im(n);
        for (int i = 0; i < n; ++i) im[i] = 1.0 / mass[i];   // rattle.F90: one/atmmass(ib)
        TRY(upload(c, &c->invmass, im));
    }
    TRY(upload(c, &c->chrg, chrg));
    TRY(upload(c, &c->typ, typ));
    double q = 0, q2 = 0;
    for (int i = 0; i < n; ++i) { q += chrg[i]; q2 += chrg[i] * chrg[i]; }
    c->netchrgsq = q * q;
    c->pot_ewc = -1.0 / std::sqrt(std::acos(-1.0)) * p->alpha * q2;   // fft_pme_init.F90:147-156
    size_t n3 = (size_t)3 * n;
    if (pgk_dmalloc(c, &c->pos, n3 * 8) || pgk_dmalloc(c, &c->vel, n3 * 8) || pgk_dmalloc(c, &c->pos_old, n3 * 8) ||
        pgk_dmalloc(c, &c->facc[0], n3 * 8) || pgk_dmalloc(c, &c->facc[1], n3 * 8) ||
        pgk_dmalloc(c, &c->acc, sizeof(long long) * 2 * NACC) || pgk_dmalloc(c, &c->dyn, sizeof(DynState)) ||
        pgk_dmalloc(c, &c->chain, sizeof(ChainDev)) || pgk_dmalloc(c, &c->status, sizeof(unsigned)) ||
        pgk_dmalloc(c, &c->ke_part, sizeof(double) * 20 * std::max(c->nsm, 1)) ||
        pgk_dmalloc(c, &c->ke_done, sizeof(unsigned)) || cudaMemsetAsync(c->ke_done, 0, sizeof(unsigned), c->st)) {
        pgk_free(c);
        return PGK_E_NOMEM;
    }
    cudaMemsetAsync(c->vel, 0, n3 * 8, c->st);
    cudaMemsetAsync(c->pos, 0, n3 * 8, c->st);
    cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->st);
    cudaMemsetAsync(c->acc, 0, sizeof(long long) * 2 * NACC, c->st);
    // ---- LJ tables ----
    c->ntyp = s->ntyp;
    std::vector<double2> lj64(s->ntyp * s->ntyp);
    std::vector<float2> lj32(s->ntyp * s->ntyp);
    for (int i = 0; i < s->ntyp; ++i)
        for (int j = 0; j < s->ntyp; ++j) {
            double R = s->vdw_radij[i + s->ntyp * j], E = s->vdw_welij[i + s->ntyp * j];
            if (s->inter_inttyp && s->inter_inttyp[i + s->ntyp * j] != 1) E = 0.0;
            lj64[i * s->ntyp + j] = make_double2(R * R, E);
            lj32[i * s->ntyp + j] = make_float2((float)(R * R), (float)E);
        }
    TRY(upload(c, &c->lj64, lj64));
    TRY(upload(c, &c->lj32, lj32));
    TRY(morse_setup(c, s));
    // ---- spline tables (spline_interp.F90:14-136) ----
    {
        int ns = p->nspltbl > 0 ? p->nspltbl : 1100;
        double h = (p->rrcut + 2.0) / (double)ns;
        c->nspl = ns; c->hspl = h;
        double rootpi = std::sqrt(std::acos(-1.0)), piE = 2.0 / rootpi * p->alpha;
        std::vector<double> x(ns), t[4];
        for (int i = 0; i < ns; ++i) x[i] = (double)i * h;
        for (int k = 0; k < 4; ++k) { t[k].assign(ns, 0.0); t[k][0] = 1.0; }
        for (int i = 1; i < ns; ++i) {
            double r = x[i], inv = 1.0 / r, arg = p->alpha * r;
            double ec = std::erfc(arg), ex = std::exp(-arg * arg);
            t[0][i] = inv * (piE * ex * inv + ec * inv * inv);
            t[1][i] = ec * inv;
            t[2][i] = inv * (-piE * ex * inv + (1.0 - ec) * inv * inv);
            t[3][i] = (1.0 - ec) * inv;
        }
        std::vector<double4> s64(4 * (size_t)ns);
        std::vector<float4> s32(4 * (size_t)ns);
        for (int k = 0; k < 4; ++k) {
            std::vector<double> b, cc, d;
            spl_coeff(ns, h, x, t[k], b, cc, d);
            for (int i = 0; i < ns; ++i) {
                s64[(size_t)k * ns + i] = make_double4(t[k][i], b[i], cc[i], d[i]);
                s32[(size_t)k * ns + i] = make_float4((float)t[k][i], (float)b[i], (float)cc[i], (float)d[i]);
            }
        }
        TRY(upload(c, &c->spl64, s64));
        TRY(upload(c, &c->spl32, s32));
    }
    HostTerms ht;
    std::vector<int> mol_idx_h, mol_list_h;
    // ---- exclusions ----
    {
        std::vector<std::vector<int>> part(n);
        std::vector<int2> pairs;
        for (int i = 0; i < n; ++i) {
            int b = s->index_excl[i] - 1, e = s->index_excl[i + 1] - 1;
            for (int k = b; k < e; ++k) {
                int v = s->list_excl[k];
                if (v <= 0) continue;
                int j = v - 1;
                if (j <= i || j >= n) continue;
                part[i].push_back(j);
                part[j].push_back(i);
                if (i < n - 1) pairs.push_back(make_int2(i, j));
            }
        }
        std::vector<int> idx(n + 1, 0), lst;
        for (int i = 0; i < n; ++i) {
            std::sort(part[i].begin(), part[i].end());
            part[i].erase(std::unique(part[i].begin(), part[i].end()), part[i].end());
            idx[i] = (int)lst.size();
            lst.insert(lst.end(), part[i].begin(), part[i].end());
            c->max_excl = std::max(c->max_excl, (int)part[i].size());
        }
        idx[n] = (int)lst.size();
        // (lowest, highest) partner of each atom: the list builder looks a pair
        // up only when j falls inside its atom's range
        std::vector<int2> rng(n);
        for (int i = 0; i < n; ++i)
            rng[i] = part[i].empty() ? make_int2(INT32_MAX, -1) : make_int2(part[i].front(), part[i].back());
        if (lst.empty()) lst.push_back(-1);
        TRY(upload(c, &c->exs_idx, idx));
        TRY(upload(c, &c->exs_list, lst));
        TRY(upload(c, &c->exs_rng, rng));
        ht.ex = pairs;
    }
    // ---- molecules ----
    {
        c->nmole = s->nmole;
        if (s->nmole > 0 && s->molept_index && s->molept_list) {
            std::vector<int> mi(s->nmole + 1), ml;
            for (int m = 0; m <= s->nmole; ++m) mi[m] = s->molept_index[m] - 1;
            for (int k = 0; k < mi[s->nmole]; ++k) ml.push_back(s->molept_list[k] - 1);
            TRY(upload(c, &c->mol_idx, mi));
            TRY(upload(c, &c->mol_list, ml));
            mol_idx_h = mi;
            mol_list_h = ml;
        } else {
            c->nmole = 0;
        }
    }
    // ---- bonded (uploaded in chunk order by bonded_setup) ----
    {
        for (int k = 0; k < s->nbond; ++k) {
            ht.bij.push_back(make_int2(s->ibond[k] - 1, s->jbond[k] - 1));
            ht.bp.push_back(make_double2(s->para_cbond[k], s->para_eqbond[k]));
        }
        for (int k = 0; k < s->nangl; ++k) {
            ht.aijk.push_back(make_int4(s->iangl[k] - 1, s->jangl[k] - 1, s->kangl[k] - 1, 0));
            ht.ap.push_back(make_double2(s->para_cangl[k], s->para_eqangl[k]));
        }
        for (int k = 0; k < s->ntors; ++k) {
            ht.tij.push_back(make_int4(s->itors[k] - 1, s->jtors[k] - 1, s->ktors[k] - 1, s->ltors[k] - 1));
            // caltors: barhig/divfac, phase, |period|, cos(phase) (calijkl force uses cos(phsang))
            ht.tp.push_back(make_double4(s->para_barhig[k] / (double)s->para_divfac[k], s->para_phsang[k],
                                         std::fabs(s->para_period[k]), std::cos(s->para_phsang[k])));
        }
        for (int k = 0; k < s->ntorsrb; ++k) {
            ht.rij.push_back(make_int4(s->itorsrb[k] - 1, s->jtorsrb[k] - 1, s->ktorsrb[k] - 1, s->ltorsrb[k] - 1));
            for (int qq = 0; qq < 6; ++qq) ht.rc.push_back(s->para_barhigrb[6 * k + qq]);
        }
        // 1-4 pairs in calnon14p order: periodic torsions, then RB torsions
        if (s->ifcalnonb14)
            for (int k = 0; k < s->ntors; ++k) {
                if (!s->ifcalnonb14[k]) continue;
                int i = s->itors[k] - 1, j = s->ltors[k] - 1;
                if (i == j) continue;
                ht.p14.push_back(make_int2(i, j));
                ht.f14.push_back(make_double2(1.0 / s->para_divfac_elc[k] * s->ring14[k],
                                              1.0 / s->para_divfac_vdw[k] * s->ring14[k]));
            }
        if (s->ifcalnonb14_rb)
            for (int k = 0; k < s->ntorsrb; ++k) {
                if (!s->ifcalnonb14_rb[k]) continue;
                int i = s->itorsrb[k] - 1, j = s->ltorsrb[k] - 1;
                if (i == j) continue;
                ht.p14.push_back(make_int2(i, j));
                ht.f14.push_back(make_double2(1.0 / s->para_divfac_elcrb[k] * s->ring14_rb[k],
                                              1.0 / s->para_divfac_vdwrb[k] * s->ring14_rb[k]));
            }
        ht.q = chrg.data(); ht.ty = typ.data(); ht.lj = lj64.data(); ht.ntyp = s->ntyp;
        TRY(bonded_setup(c, ht, mol_idx_h, mol_list_h));
    }
    // ---- constraints ----
    {
        c->nconstraint = s->nconstraint;
        c->ncgroup = 0;
        if (s->nconst > 0) {
            std::vector<int> gi0(s->nconst + 1), gl0;
            for (int g = 0; g <= s->nconst; ++g) gi0[g] = s->index_mconst[g] - 1;
            for (int k = 0; k < gi0[s->nconst]; ++k) gl0.push_back(s->list_mconst[k] - 1);
            std::vector<int2> cij; std::vector<double> cd;
            for (int k = 0; k < s->nconstraint; ++k) {
                cij.push_back(make_int2(s->iconst[k] - 1, s->jconst[k] - 1));
                cd.push_back(s->dconst[k]);
            }
            // Split every group into its connected components (constraints that
            // share no atom, e.g. the X-H bonds of different carbons), keeping
            // the reference order inside each.  The Gauss-Seidel sweeps of
            // rattle_c / rattlep_v give the same result either way: a component
            // only moves its own atoms, and once converged its constraints are
            // skipped by every further sweep of the group.
            std::vector<int> gi(1, 0), gl;
            std::map<int, int> parent;
            std::function<int(int)> find = [&](int a) {
                int r = a;
                while (parent[r] != r) r = parent[r];
                while (parent[a] != r) { int nx = parent[a]; parent[a] = r; a = nx; }
                return r;
            };
            for (int g = 0; g < s->nconst; ++g) {
                parent.clear();
                for (int k = gi0[g]; k < gi0[g + 1]; ++k) {
                    int2 p2 = cij[gl0[k]];
                    if (!parent.count(p2.x)) parent[p2.x] = p2.x;
                    if (!parent.count(p2.y)) parent[p2.y] = p2.y;
                    int ra = find(p2.x), rb = find(p2.y);
                    if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
                }
                std::vector<int> roots;
                std::map<int, std::vector<int>> comp;
                for (int k = gi0[g]; k < gi0[g + 1]; ++k) {
                    int r = find(cij[gl0[k]].x);
                    if (!comp.count(r)) roots.push_back(r);
                    comp[r].push_back(gl0[k]);
                }
                for (int r : roots) {
                    gl.insert(gl.end(), comp[r].begin(), comp[r].end());
                    gi.push_back((int)gl.size());
                }
            }
            // Rigid three-atom groups: the constraints (a0,a1), (a0,a2), (a1,a2)
            // in this order, each stored with its lower-listed atom first as
            // here (rigid water: O-H1, O-H2, H1-H2).  They leave the group
            // arrays for k_rattle_rigid3; the order of groups does not matter
            // (each moves only its own atoms).
            {
                std::vector<int4> r3a;
                std::vector<double4> r3d;
                std::vector<int> gi2(1, 0), gl2;
                for (int g = 0; g + 1 < (int)gi.size(); ++g) {
                    if (gi[g + 1] - gi[g] == 3) {
                        const int2 q0 = cij[gl[gi[g]]], q1 = cij[gl[gi[g] + 1]], q2 = cij[gl[gi[g] + 2]];
                        if (q1.x == q0.x && q2.x == q0.y && q2.y == q1.y && q0.x != q0.y && q1.y != q0.x &&
                            q1.y != q0.y) {
                            r3a.push_back(make_int4(q0.x, q0.y, q1.y, 0));
                            r3d.push_back(make_double4(cd[gl[gi[g]]], cd[gl[gi[g] + 1]], cd[gl[gi[g] + 2]], 0.0));
                            continue;
                        }
                    }
                    gl2.insert(gl2.end(), gl.begin() + gi[g], gl.begin() + gi[g + 1]);
                    gi2.push_back((int)gl2.size());
                }
                c->nr3 = (int)r3a.size();
                if (c->nr3) { TRY(upload(c, &c->r3_atoms, r3a)); TRY(upload(c, &c->r3_d, r3d)); }
                gi.swap(gi2);
                gl.swap(gl2);
            }
            // Star groups: K <= 4 constraints (c, a_1) ... (c, a_K) with one
            // first atom c and K distinct second atoms (the X-H bonds of one
            // heavy atom after the component split), sorted by K descending.
            {
                std::vector<int> sa[5];
                std::vector<double> sd[5];
                std::vector<int> gi2(1, 0), gl2;
                for (int g = 0; g + 1 < (int)gi.size(); ++g) {
                    const int K = gi[g + 1] - gi[g];
                    bool star = K >= 1 && K <= 4;
                    const int ctr = star ? cij[gl[gi[g]]].x : -1;
                    for (int q = 0; star && q < K; ++q) {
                        const int2 p2 = cij[gl[gi[g] + q]];
                        star = p2.x == ctr && p2.y != ctr;
                        for (int r = 0; star && r < q; ++r) star = cij[gl[gi[g] + r]].y != p2.y;
                    }
                    if (star) {
                        sa[K].push_back(ctr);
                        for (int q = 0; q < 4; ++q) {
                            sa[K].push_back(q < K ? cij[gl[gi[g] + q]].y : -1);
                            sd[K].push_back(q < K ? cd[gl[gi[g] + q]] : 0.0);
                        }
                        continue;
                    }
                    gl2.insert(gl2.end(), gl.begin() + gi[g], gl.begin() + gi[g + 1]);
                    gi2.push_back((int)gl2.size());
                }
                std::vector<int> atoms;
                std::vector<double> dls;
                for (int K = 4; K >= 1; --K) {
                    if (K < 4) c->star_seg[3 - K] = (int)(atoms.size() / 5);
                    atoms.insert(atoms.end(), sa[K].begin(), sa[K].end());
                    dls.insert(dls.end(), sd[K].begin(), sd[K].end());
                }
                c->nstar = (int)(atoms.size() / 5);
                c->star_seg[3] = c->nstar;
                if (c->nstar) { TRY(upload(c, &c->star_atoms, atoms)); TRY(upload(c, &c->star_d, dls)); }
                gi.swap(gi2);
                gl.swap(gl2);
            }
            c->ncgroup = (int)gi.size() - 1;
            std::vector<int2> span(c->ncgroup);
            for (int g = 0; g < c->ncgroup; ++g) {
                int lo = n, hi = -1;
                for (int k = gi[g]; k < gi[g + 1]; ++k) {
                    int2 p2 = cij[gl[k]];
                    lo = std::min(lo, std::min(p2.x, p2.y));
                    hi = std::max(hi, std::max(p2.x, p2.y));
                }
                span[g] = hi >= lo ? make_int2(lo, hi - lo + 1) : make_int2(0, 0);
            }
            TRY(upload(c, &c->cg_idx, gi)); TRY(upload(c, &c->cg_list, gl));
            TRY(upload(c, &c->c_ij, cij)); TRY(upload(c, &c->c_d, cd));
            TRY(upload(c, &c->cg_span, span));
            // warps of 32 consecutive groups whose atoms and constraints fit the
            // shared-memory staging of k_rattle_warp (192 atoms, 8 constraints per group)
            const int nw = (c->ncgroup + 31) / 32;
            std::vector<unsigned char> fit(nw, 0);
            c->cg_nfit = 0;
            for (int w = 0; w < nw; ++w) {
                int lo = INT32_MAX, hi = 0;
                bool ok = true;
                for (int g = 32 * w; g < std::min(c->ncgroup, 32 * w + 32); ++g) {
                    lo = std::min(lo, span[g].x);
                    hi = std::max(hi, span[g].x + span[g].y);
                    ok = ok && gi[g + 1] - gi[g] <= 8;
                }
                fit[w] = (ok && hi - lo <= 192) ? 1 : 0;
                c->cg_nfit += fit[w];
            }
            TRY(upload(c, &c->cg_fit, fit));
        }
    }
    // ---- pair list buffers (sorted slots and cluster rows grow at list time) ----
    {
        double vol = p->xcel * p->ycel * p->zcel;
        double rb = p->rcut_book;
        // partners of an 8-atom cluster: the sphere of radius rcut_book swept
        // over the cluster's extent (~ 2 A), about half of them stored (each
        // pair once, in its lower slot's row); rows regrow on overflow
        double rs = rb + 2.0;
        double expect = (double)n / vol * 4.0 / 3.0 * std::acos(-1.0) * rs * rs * rs;
        int cap = p->max_nbr > 0 ? p->max_nbr : (int)(expect + 128);
        cap = std::min(cap, ((n + 31) / 32) * 32);
        cap = ((cap + 31) / 32) * 32;
        c->ccap = std::max(cap, 32);
        // pruned list buffer (mixed): PGK_PRUNE_BUFFER overrides the 0.7 A default
        // (200k-atom butane NPT: 0.607 ms per step against 0.609 at 1 A with one
        // wave of pair blocks; 0.587 ms at 0.6, 0.7 and 0.8 A with the autotuned
        // waves); 0 disables pruning, as does a book skin too thin for the buffer
        if (c->mixed()) {
            const char* pf = getenv("PGK_PAIR_FRAME");
            c->no_frame = pf && atoi(pf) == 0;
            const char* pb = getenv("PGK_PRUNE_BUFFER");
            const double buf = pb ? atof(pb) : 0.7;
            const double rmax = std::max(p->rcut, p->rrcut);
            c->prune_buffer = (buf > 0.0 && rmax + buf < p->rcut_book) ? (float)buf : 0.f;
            if (pgk_dmalloc(c, &c->prune, sizeof(PruneDev)) ||
                cudaMemsetAsync(c->prune, 0, sizeof(PruneDev), c->st)) {
                pgk_free(c);
                return PGK_E_NOMEM;
            }
        }
        if (pgk_dmalloc(c, &c->iperm, n * sizeof(int)) || pgk_dmalloc(c, &c->cell_of, n * sizeof(int)) ||
            pgk_dmalloc(c, &c->subkey, n * sizeof(int)) || pgk_dmalloc(c, &c->counters, 8 * sizeof(unsigned long long)) ||
            pgk_dmalloc(c, &c->hasup, std::max(n, 1)) ||
            cudaMemsetAsync(c->counters, 0, 8 * sizeof(unsigned long long), c->st)) {
            pgk_free(c);
            return PGK_E_NOMEM;
        }
    }
    // ---- SPME ----
    if (p->ifspme) TRY(spme_setup(c));
    // ---- dynamic state ----
    {
        DynState& h = c->hdyn;
        memset(&h, 0, sizeof(h));
        double box[3] = {p->xcel, p->ycel, p->zcel};
        for (int d = 0; d < 3; ++d) { h.box[d] = box[d]; h.boxinv[d] = 1.0 / box[d]; }
        h.rkcut = rkcut_host(box, p->nfft1, p->nfft2, p->nfft3);
        h.yratio = p->ycel / p->xcel;
        h.zratio = p->zcel / p->xcel;
        for (int d = 0; d < 3; ++d) { h.kl_s[d] = 1.0; h.dr_a[d] = 1.0; h.rvinv[d] = 1.0; }
        if (cudaMemcpy(c->dyn, &h, sizeof(h), cudaMemcpyHostToDevice)) { pgk_free(c); return PGK_E_CUDA; }
        ChainDev ch;
        memset(&ch, 0, sizeof(ch));
        ch.xlogv = std::log(p->xcel * p->ycel * p->zcel) / 3.0;   // prepmd.F90:527
        ch.xboxh[0] = p->xcel; ch.xboxh[1] = p->ycel; ch.xboxh[2] = p->zcel;
        if (cudaMemcpy(c->chain, &ch, sizeof(ch), cudaMemcpyHostToDevice)) { pgk_free(c); return PGK_E_CUDA; }
    }
    // the set-up copies ran on the legacy stream (synchronous host arrays),
    // the memsets on the context's: both are complete after these waits
    if (cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess || cudaStreamSynchronize(c->st) != cudaSuccess) {
        pgk_free(c);
        return PGK_E_CUDA;
    }
    TRY(spme_autotune(c));
#undef TRY
    *out = c;
    return PGK_OK;
}

pgk_status pgk_free(pgk_ctx* c) {
    if (!c) return PGK_OK;
    // the context's own streams only: other contexts keep running
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->st2) cudaStreamSynchronize(c->st2);
    if (c->st3) cudaStreamSynchronize(c->st3);
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
    void* bufs[] = {c->pos, c->vel, c->pos_old, c->mass, c->invmass, c->chrg, c->typ, c->facc[0], c->facc[1], c->acc,
                    c->dyn, c->chain, c->status, c->lj64, c->lj32, c->spl64, c->spl32, c->exs_idx, c->exs_list, c->exs_rng,
                    c->expair, c->mol_idx, c->mol_list, c->bond_ij, c->bond_p, c->angl_ijk, c->angl_p, c->tors_ijkl,
                    c->tors_p, c->rb_ijkl, c->rb_c, c->p14_ij, c->p14_f, c->cg_idx, c->cg_list, c->c_ij, c->c_d,
                    c->cell_of, c->subkey, c->cell_cnt, c->cell_start, c->cell_fill, c->perm, c->iperm, c->pos_s, c->clist,
                    c->ccnt, c->xq, c->xq64, c->fsort, c->plist, c->pcnt, c->xq_prune, c->prune, c->typ_s, c->counters, c->qacc, c->qc, c->qr, c->bsp,
                    c->plan[0].tw, c->plan[1].tw, c->plan[2].tw, c->fout, c->cg_span, c->cg_fit, c->blk_a0, c->blk_nloc, c->blk_t, c->blk_soff,
                    c->blk_ip, c->blk_incp, c->blk_inc, c->brec[0], c->brec[1], c->brec[2], c->brec[3], c->brec[4],
                    c->brec[5], c->btab[0], c->btab[1], c->btab[2], c->btab[3], c->btab[4], c->btab[5],
                    c->mol_of, c->hftyp, c->molecom, c->molevel, c->hf_pot, c->hf_W, c->hf_part, c->hf_rec, c->hf_zs,
                    c->hf_ms, c->lt_mole, c->lt_reg, c->lt_frand, c->lt_dekin, c->hasup, c->out_rec,
                    c->ewk_nv, c->ewk_tab, c->ewk_part, c->ewk_coef, c->ewk_red, c->ewk_out, c->ewk_seg,
                    c->mor_atoms, c->mor_par, c->mor_rows, c->mor_cnt, c->mor_cell, c->mor_csort, c->mor_ccnt,
                    c->mor_cstart, c->mor_cfill, c->mor_ctr, c->hfk_q, c->hfk_g, c->hfk_out, c->hfk_tw[0],
                    c->hfk_tw[1], c->hfk_tw[2], c->r3_atoms, c->r3_d, c->star_atoms, c->star_d, c->plan_rx.tw,
                    c->tw_rx, c->ke_part, c->ke_done};
    for (void* b : bufs) if (b) pgk_dfree(c, b);     // stream-ordered frees on c->st
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->st2) cudaStreamDestroy(c->st2);
    if (c->st3) cudaStreamDestroy(c->st3);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->ev_join3) cudaEventDestroy(c->ev_join3);
    if (c->ev_pre_pair) cudaEventDestroy(c->ev_pre_pair);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return PGK_OK;
}

pgk_status pgk_upload_state(pgk_ctx* c, const double* cor, const double* vel, const double* box) {
    if (!c || !cor) return PGK_E_INVALID;
    size_t b = (size_t)24 * c->natom;
    PGK_CUDA(c, cudaMemcpyAsync(c->pos, cor, b, cudaMemcpyHostToDevice, c->st));
    if (vel) PGK_CUDA(c, cudaMemcpyAsync(c->vel, vel, b, cudaMemcpyHostToDevice, c->st));
    if (box) {
        pgk_status s = set_dyn_box(c, box);
        if (s) return s;
    }
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return PGK_OK;
}

pgk_status pgk_download_state(pgk_ctx* c, double* cor, double* vel, double* box) {
    if (!c) return PGK_E_INVALID;
    size_t b = (size_t)24 * c->natom;
    if (cor) PGK_CUDA(c, cudaMemcpyAsync(cor, c->pos, b, cudaMemcpyDeviceToHost, c->st));
    if (vel) PGK_CUDA(c, cudaMemcpyAsync(vel, c->vel, b, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaMemcpyAsync(&c->hdyn, c->dyn, sizeof(DynState), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    if (box) for (int d = 0; d < 3; ++d) box[d] = c->hdyn.box[d];
    return PGK_OK;
}

pgk_status pgk_set_chain(pgk_ctx* c, const pgk_chain* ch) {
    if (!c || !ch) return PGK_E_INVALID;
    ChainDev d;
    static_assert(sizeof(ChainDev) == sizeof(pgk_chain), "chain layout");
    memcpy(&d, ch, sizeof(d));
    PGK_CUDA(c, cudaMemcpyAsync(c->chain, &d, sizeof(d), cudaMemcpyHostToDevice, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return PGK_OK;
}

pgk_status pgk_get_chain(pgk_ctx* c, pgk_chain* ch) {
    if (!c || !ch) return PGK_E_INVALID;
    PGK_CUDA(c, cudaMemcpyAsync(ch, c->chain, sizeof(ChainDev), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return PGK_OK;
}

pgk_status pgk_transcor(pgk_ctx* c) {
    if (!c) return PGK_E_INVALID;
    pgk_status s = launch_transcor(c);
    if (s) return s;
    return read_status(c);
}

pgk_status pgk_mklist_cell(pgk_ctx* c, int64_t* nl) {
    if (!c) return PGK_E_INVALID;
    pgk_status s = launch_mklist(c);
    if (s) return s;
    if (nl) *nl = c->hdyn.nlistnball;
    return PGK_OK;
}

pgk_status pgk_get_nblist(pgk_ctx* c, int32_t* nb_index, int32_t* nb_list, int64_t cap, int64_t* nl) {
    if (!c || !nl) return PGK_E_INVALID;
    return export_nblist(c, nb_index, nb_list, cap, nl);
}

pgk_status pgk_calforce(pgk_ctx* c, int32_t flag, double* force, pgk_energies* e, pgk_virials* v) {
    if (!c || (flag != PGK_MTS_LONG && flag != PGK_MTS_SHORT)) return PGK_E_INVALID;
    bool want = e || v;
    pgk_status s = force_group(c, flag, want, want);
    if (s) return s;
    int g = flag == PGK_MTS_LONG ? 0 : 1;
    if (force && (s = force_to_host(c, g, force, false))) return s;
    if (want && (s = read_acc(c, 1 << g, e, v, flag == PGK_MTS_LONG))) return s;
    return read_status(c);
}

pgk_status pgk_ewaldr(pgk_ctx* c, double* force, pgk_energies* e, pgk_virials* v) {
    if (!c) return PGK_E_INVALID;
    pgk_status s;
    bool want = e || v;
    if ((s = launch_zero_group(c, 0))) return s;
    if (!c->list_valid && (s = launch_mklist(c))) return s;
    if ((s = launch_pack(c)) || (s = launch_pair(c, 0, want ? PM_FULL : PM_FORCE)) ||
        (s = launch_intra(c, 0, 32, want)))
        return s;
    if (force && (s = force_to_host(c, 0, force, true))) return s;
    if (want && (s = read_acc(c, 1, e, v, false))) return s;
    return read_status(c);
}

pgk_status pgk_fft_pme(pgk_ctx* c, double* force, pgk_energies* e, pgk_virials* v) {
    if (!c) return PGK_E_INVALID;
    if (!c->prm.ifspme) return pgk_fail(c, PGK_E_INVALID, "ifspme is off");
    pgk_status s;
    bool want = e || v;
    if ((s = launch_zero_group(c, 0)) || (s = launch_spme(c, 0, want, want))) return s;
    if (force && (s = force_to_host(c, 0, force, true))) return s;
    if (want && (s = read_acc(c, 1, e, v, false))) return s;
    return read_status(c);
}

pgk_status pgk_ewaldkp_hf(pgk_ctx* c, int32_t kmax, double* force, double* pot_atm, double* viri_atm,
                          pgk_ewk_hf* out) {
    if (!c) return PGK_E_INVALID;
    int nw = 0;
    pgk_status s = launch_ewk_hf(c, kmax, &nw);
    if (s) return s;
    const size_t n = (size_t)c->natom;
    if (force) PGK_CUDA(c, cudaMemcpyAsync(force, c->ewk_out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    if (pot_atm)
        PGK_CUDA(c, cudaMemcpyAsync(pot_atm, c->ewk_out + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    if (viri_atm)
        PGK_CUDA(c, cudaMemcpyAsync(viri_atm, c->ewk_out + 4 * n, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost,
                                    c->st));
    double sc[11];
    PGK_CUDA(c, cudaMemcpyAsync(sc, c->ewk_out + 13 * n, sizeof(sc), cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    if (out) {
        out->pot_ewk = sc[0];
        out->pot_ewk_cc = sc[1];
        for (int t = 0; t < 9; ++t) out->pot_virit_coul[t] = sc[2 + t];
        out->nwave = nw;
        out->_pad = 0;
    }
    return read_status(c);
}

pgk_status pgk_mklist_mor_cell(pgk_ctx* c, int64_t* nl) {
    if (!c) return PGK_E_INVALID;
    pgk_status s = launch_mklist_mor(c);
    if (s) return s;
    return export_morlist(c, nullptr, nullptr, nullptr, 0, nl);
}

pgk_status pgk_get_morlist(pgk_ctx* c, int32_t* nmorselist, int32_t* mor_indexall, int32_t* mor_listall,
                           int64_t cap, int64_t* nl, int32_t* nmorse) {
    if (!c) return PGK_E_INVALID;
    if (nmorse) *nmorse = c->nmor;
    return export_morlist(c, nmorselist, mor_indexall, mor_listall, cap, nl);
}

pgk_status pgk_morsep(pgk_ctx* c, double* force, pgk_energies* e, pgk_virials* v) {
    if (!c) return PGK_E_INVALID;
    pgk_status s;
    bool want = e || v;
    if ((s = launch_zero_group(c, 0)) || (s = launch_morse(c, 0, want))) return s;
    if (force && (s = force_to_host(c, 0, force, true))) return s;
    if (want && (s = read_acc(c, 1, e, v, false))) return s;
    return read_status(c);
}

pgk_status pgk_calbonded(pgk_ctx* c, double* force, pgk_energies* e, pgk_virials* v) {
    if (!c) return PGK_E_INVALID;
    pgk_status s;
    bool want = e || v;
    if ((s = launch_zero_group(c, 0)) || (s = launch_intra(c, 0, 31, want))) return s;
    if (force && (s = force_to_host(c, 0, force, true))) return s;
    if (want && (s = read_acc(c, 1, e, v, false))) return s;
    return read_status(c);
}

pgk_status pgk_rattle_c(pgk_ctx* c, const double* old, double eps, double dts) {
    if (!c || !old) return PGK_E_INVALID;
    PGK_CUDA(c, cudaMemcpyAsync(c->pos_old, old, (size_t)24 * c->natom, cudaMemcpyHostToDevice, c->st));
    pgk_status s = launch_rattle_pos(c, eps, dts, false);
    if (s) return s;
    return read_status(c);
}

pgk_status pgk_rattlep_v(pgk_ctx* c, double eps) {
    if (!c) return PGK_E_INVALID;
    pgk_status s = launch_rattle_vel(c, eps);
    if (s) return s;
    return read_status(c);
}

pgk_status pgk_calpress(pgk_ctx* c, double* kint, double* ptot, double* p9) {
    if (!c) return PGK_E_INVALID;
    pgk_status s;
    if ((s = launch_kinetic(c, 0)) || (s = launch_press(c))) return s;
    pgk_chain ch;
    if ((s = pgk_get_chain(c, &ch))) return s;
    if (kint) {
        long long k;
        PGK_CUDA(c, cudaMemcpy(&k, c->acc + A_KE, sizeof(k), cudaMemcpyDeviceToHost));
        *kint = accv(c, k);
    }
    if (ptot) *ptot = ch.pint;
    if (p9) for (int k = 0; k < 9; ++k) p9[k] = ch.pintt[k];
    return PGK_OK;
}

pgk_status pgk_sync(pgk_ctx* c) {
    if (!c) return PGK_E_INVALID;
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return read_status(c);
}

int64_t pgk_kernel_launches(const pgk_ctx* c) { return c ? c->launches : 0; }

pgk_status pgk_bench_kernel(pgk_ctx* c, int32_t which, int32_t iters, double* ms, double* units, double* entries) {
    if (!c || iters < 1 || !ms) return PGK_E_INVALID;
    pgk_status s;
    if (!c->list_valid && (s = launch_mklist(c))) return s;
    if ((s = launch_pack(c))) return s;
    if (which == 0) {
        long long np = 0, ne = 0;
        if ((s = count_pairs(c, &np, &ne))) return s;
        if (units) *units = (double)np;
        if (entries) *entries = (double)ne;
    } else if (units) {
        *units = which == 3 ? (double)c->K[0] * c->K[1] * c->K[2] : (double)c->natom;
    }
    if (which >= 256 && which < 1024) {
        int nw = 0;
        if ((s = launch_ewk_hf(c, (which - 256) & 255, &nw))) return s;
        if (units) *units = (double)c->natom * (nw - 1);
    }
    if (which >= 1 && which <= 3 && !c->prm.ifspme) return pgk_fail(c, PGK_E_INVALID, "ifspme is off");
    cudaEvent_t e0, e1;
    PGK_CUDA(c, cudaEventCreate(&e0));
    PGK_CUDA(c, cudaEventCreate(&e1));
    auto one = [&]() -> pgk_status {
        switch (which) {
            case 0: return launch_pair(c, 0, PM_TENS);
            case 1: return spme_bench(c, 1);
            case 2: return spme_bench(c, 2);
            case 3: return spme_bench(c, 3);
            case 4: return launch_mklist(c);                          // list build chain
            case 5: return launch_kick_drift(c, KD_LONG | KD_DRIFT);  // long kick + drift (moves the atoms)
            default:
                if (which >= 256 && which < 1024)
                    return launch_ewk_hf(c, (which - 256) & 255, nullptr, (which - 256) >> 8);
                if (which >= 64 && which < 128) return launch_intra(c, 0, which - 64, true);
                if (which >= 128 && which < 192) return launch_intra(c, 0, which - 128, true, true);
                return pgk_fail(c, PGK_E_INVALID, "unknown kernel id");
        }
    };
    if ((s = launch_zero_group(c, 0)) || (s = one())) return s;    // warm-up launch
    PGK_CUDA(c, cudaEventRecord(e0, c->st));
    for (int k = 0; k < iters; ++k)
        if ((s = one())) return s;
    PGK_CUDA(c, cudaEventRecord(e1, c->st));
    PGK_CUDA(c, cudaEventSynchronize(e1));
    float t = 0;
    PGK_CUDA(c, cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = (double)t / iters;
    return launch_zero_group(c, 0);
}
void* pgk_stream(const pgk_ctx* c) { return c ? (void*)c->st : nullptr; }

}  // extern "C"

// ---- stage drivers ---------------------------------------------------------------
static pgk_status md_step_body(pgk_ctx* c, int kind, int64_t step, const pgk_mdparams* md, bool ene, bool vir,
                               bool tens, bool hfs, bool lt, bool ke_ready);

// kind: 0 NVE (moldyn.F90), 1 NHC (moldyn_nhc.F90), 2 MTK (moldyn_mtk.F90),
// 3 NVE + region Langevin + heat flux (moldyn_hf.F90); hf records go to the
// device buffer c->hf_rec (kind 3), *nrec counts them
static pgk_status run_md(pgk_ctx* c, int kind, int64_t ini, int64_t end, const pgk_mdparams* md, pgk_energies* eo,
                         long long* nrec = nullptr) {
    if (!c || !md || md->nstep_short < 1 || md->dt_long_cal <= 0) return PGK_E_INVALID;
    if (kind == 3 && !c->hf_set) return pgk_fail(c, PGK_E_INVALID, "pgk_set_hf has not been called");
    if ((kind == 1 || kind == 2) && (md->mchain < 2 || md->mchain > 8 || md->nyosh < 1 || md->nyosh > 8 || md->next < 1))
        return pgk_fail(c, PGK_E_INVALID, "chain parameters");
    const int nb = c->prm.nstep_book > 0 ? c->prm.nstep_book : 1;
    // Morse list cadence (nstep_bookmor; 0 = the pair list's)
    const int nbm = c->prm.nstep_bookmor > 0 ? c->prm.nstep_bookmor : nb;
    const bool mtk = kind == 2;
    const bool hfdrv = kind == 3;
    const bool lt = hfdrv && c->hfp.nlangeregion > 0;
    const int hfi = c->hfp.heatfinterval > 0 ? c->hfp.heatfinterval : 1;
    const long long per = (long long)c->hfp.nhfregion * PGK_HF_NCOL;
    long long nr = 0;
    long long last_rec = -1;
    // ke_ready: the kinetic sums of the current velocities are in the
    // accumulators (the previous step of this run ended with them), so the
    // step's first chain half reuses them instead of summing again
    bool ke_ready = false;
    auto step_body = [&](int64_t st, bool e_, bool v_, bool t_, bool h_, bool l_) {
        return md_step_body(c, kind, st, md, e_, v_, t_, h_, l_, ke_ready);
    };
    pgk_status s;
#define RUN(x) do { if ((s = (x)) != PGK_OK) return s; } while (0)
    // the kick / drift coefficients of NVE-type steps depend on md alone
    if (kind == 0 || kind == 3) RUN(launch_coeffs(c, 0, *md, 0));
    for (int64_t step = ini; step <= end; ++step) {
        bool out = md->outinterval > 0 ? (step % md->outinterval == 0) : (step == end);
        const bool rec = out && c->out_cap > 0;         // device-side output record
        bool ene = out && (eo || rec);
        bool vir = mtk;
        bool tens = mtk && md->pcont_axis != PGK_PCONT_ISO && !ene;   // nhcpanisoint reads diag(pintt) only
        if (step % nb == 1 || nb == 1 || step == 0) RUN(launch_transcor(c));
        if (step % nb == 0 || nb == 1) RUN(launch_mklist(c));
        if (c->nmor && (step % nbm == 0 || nbm == 1 || !c->mor_valid)) RUN(launch_mklist_mor(c));
        const bool hfs = hfdrv && per > 0 && step > 0 && (hfi == 1 || step % hfi == 1);
        if (step == 0) {
            if (lt) RUN(launch_lt_regist(c));
            RUN(force_group(c, PGK_MTS_SHORT, ene || vir, vir, tens));
            RUN(force_group(c, PGK_MTS_LONG, ene || vir, vir, tens));
            if (mtk) { RUN(launch_kinetic(c, 0)); RUN(launch_press(c)); }
            ke_ready = mtk;
        } else if (c->use_graphs && c->list_valid && (c->nmor == 0 || c->mor_valid) && !hfs && !lt) {
            // the step's kernel sequence depends only on (ene, vir, tens) and the
            // list build; replay a captured CUDA graph of it
            const int key = 16 * kind + ((ene ? 1 : 0) | (vir ? 2 : 0) | (tens ? 4 : 0) | (ke_ready ? 8 : 0));
            if (memcmp(&c->graph_md, md, sizeof(pgk_mdparams)) != 0) {
                for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
                c->graphs.clear();
                c->graph_md = *md;
            }
            auto it = c->graphs.find(key);
            if (it == c->graphs.end() || it->second.epoch != c->list_epoch) {
                // capture the step; a graph of an earlier list build is updated in
                // place (same topology, new launch parameters), else instantiated
                cudaGraph_t g = nullptr;
                const long long l0 = c->launches;
                PGK_CUDA(c, cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
                pgk_status bs = step_body(step, ene, vir, tens, false, false);
                cudaError_t ce = cudaStreamEndCapture(c->st, &g);
                if (bs != PGK_OK || ce != cudaSuccess) {
                    // nothing of the step ran during the failed capture: run it
                    // eagerly and stop capturing on this context
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    c->launches = l0;
                    c->use_graphs = false;
                    c->graph_fail = std::string(cudaGetErrorString(ce)) + (bs ? " / " + c->err : "");
                    fprintf(stderr, "pgk: step capture failed (%s); this context runs its steps without graphs\n",
                            c->graph_fail.c_str());
                    RUN(step_body(step, ene, vir, tens, false, false));
                    goto step_done;
                }
                const long long nl = c->launches - l0;
                c->launches = l0;
                bool updated = false;
                if (it != c->graphs.end()) {
                    cudaGraphExecUpdateResultInfo info;
                    updated = cudaGraphExecUpdate(it->second.exec, g, &info) == cudaSuccess;
                    if (!updated) {
                        cudaGetLastError();
                        cudaGraphExecDestroy(it->second.exec);
                        c->graphs.erase(it);
                    }
                }
                if (updated) {
                    it->second.epoch = c->list_epoch;
                    it->second.launches = nl;
                    cudaGraphDestroy(g);
                } else {
                    cudaGraphExec_t ex = nullptr;
                    // node priorities: the pair kernel's stream outranks the others
                    cudaError_t ie = cudaGraphInstantiateWithFlags(&ex, g, cudaGraphInstantiateFlagUseNodePriority);
                    cudaGraphDestroy(g);
                    PGK_CUDA(c, ie);
                    it = c->graphs.emplace(key, pgk_ctx::GraphEntry{ex, nl, c->list_epoch}).first;
                }
            }
            PGK_CUDA(c, cudaGraphLaunch(it->second.exec, c->st));
            c->launches += it->second.launches;
        step_done:;
        } else {
            RUN(step_body(step, ene, vir, tens, hfs, lt));
        }
        if (step > 0) ke_ready = kind == 1 || kind == 2;
        if (step > 0) {
            if (lt) { RUN(launch_lt_regist(c)); RUN(launch_langevin(c, md->dt_long_cal, step, false)); }
            if (hfs) {
                if (nr < c->hf_rec_cap) RUN(launch_heatf(c, c->hf_rec + nr * per));
                ++nr;
            }
        }
        if (rec) {
            if (c->out_n < c->out_cap) {
                RUN(launch_out_record(c, step, c->out_rec + c->out_n * PGK_OUT_NCOL));
                last_rec = c->out_n;
            }
            ++c->out_n;
        } else if (ene) {
            RUN(read_acc(c, 3, eo, nullptr, true));
        }
    }
#undef RUN
    if (eo && last_rec >= 0) {          // energies of the last recorded output step
        double r[PGK_OUT_NCOL];
        PGK_CUDA(c, cudaMemcpyAsync(r, c->out_rec + last_rec * PGK_OUT_NCOL, sizeof(r), cudaMemcpyDeviceToHost,
                                    c->st));
        PGK_CUDA(c, cudaStreamSynchronize(c->st));
        memset(eo, 0, sizeof(pgk_energies));
        memcpy(eo, r + 1, sizeof(pgk_energies));   // record columns 1..14: the pgk_energies fields
    }
    if (nrec) *nrec = nr;
    return read_status(c);
}

// one MD step (step > 0) of run_md: the thermostat / barostat half steps and
// the XO-RESPA loop with its force evaluations
static pgk_status md_step_body(pgk_ctx* c, int kind, int64_t step, const pgk_mdparams* md, bool ene, bool vir,
                               bool tens, bool hfs, bool lt, bool ke_ready) {
    const double dts = md->dt_long_cal / (double)md->nstep_short;
    const bool rattle = md->ifrattle && (c->ncgroup > 0 || c->nr3 > 0 || c->nstar > 0);
    const bool mtk = kind == 2;
    const bool hfdrv = kind == 3;
    const int chain_kind = kind == 1 ? 1 : (md->pcont_axis == PGK_PCONT_ISO ? 2 : 3);
    pgk_status s;
#define RUN(x) do { if ((s = (x)) != PGK_OK) return s; } while (0)
    // An empty short group (every term in the long group) has zero forces: its
    // evaluation and kicks are skipped (they would add exact zeros).
    const int kshort = c->short_empty ? 0 : KD_SHORT;
    if (lt) RUN(launch_langevin(c, md->dt_long_cal, step, true));
    if (kind == 1 || kind == 2) {
        if (!ke_ready) RUN(launch_kinetic(c, 0));
        RUN(launch_chain_coeffs(c, chain_kind, hfdrv ? 0 : kind, *md));
    }
    // NVE and heat-flux steps: constant kick / drift coefficients, written
    // once per stage by run_md
    for (int is = 1; is <= md->nstep_short; ++is) {
        bool last = is == md->nstep_short;
        // the standard-Ewald heat-flux option evaluates the reciprocal term of
        // the last short step of a heat-flux step by ewaldkp_hf
        c->hf_ewk_now = hfs && last && c->hf_kspace == PGK_HF_KSPACE_EWK;
        RUN(launch_kick_drift(c, (is == 1 ? KD_LONG : 0) | kshort | KD_DRIFT | (rattle ? KD_SAVE : 0)));
        // the box update also refreshes the Ewald k cutoff for the long group's SPME
        if (mtk) RUN(launch_box_update(c, kind, *md, last));
        if (rattle) RUN(launch_rattle_pos(c, md->eps_rattle, dts, mtk));
        if (!c->short_empty) RUN(force_group(c, PGK_MTS_SHORT, ene || vir, vir, tens));
        if (last) {
            RUN(force_group(c, PGK_MTS_LONG, ene || vir, vir, tens));
            if (hfs) RUN(launch_hf_atm(c));
        }
        c->hf_ewk_now = false;
        RUN(launch_kick_drift(c, kshort | KD_SHORT_FIRST | (last ? KD_LONG : 0)));
        if (rattle) RUN(launch_rattle_vel(c, md->eps_rattle));
    }
    if (kind == 1) RUN(launch_kinetic_end(c, 1, chain_kind, *md));      // kinetic sums + nhcint
    if (mtk) RUN(launch_kinetic_end(c, 2, chain_kind, *md));            // + calpress + nhcp*int
#undef RUN
    return PGK_OK;
}

extern "C" {
pgk_status pgk_moldyn_nve(pgk_ctx* c, int64_t ini, int64_t end, const pgk_mdparams* md, pgk_energies* e) {
    return run_md(c, 0, ini, end, md, e);
}
pgk_status pgk_moldyn_nhc(pgk_ctx* c, int64_t ini, int64_t end, const pgk_mdparams* md, pgk_energies* e) {
    return run_md(c, 1, ini, end, md, e);
}
pgk_status pgk_moldyn_mtk(pgk_ctx* c, int64_t ini, int64_t end, const pgk_mdparams* md, pgk_energies* e) {
    return run_md(c, 2, ini, end, md, e);
}

pgk_status pgk_set_output(pgk_ctx* c, int64_t cap) {
    if (!c || cap < 0) return PGK_E_INVALID;
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    if (c->out_rec) { pgk_dfree(c, c->out_rec); c->out_rec = nullptr; }
    c->out_cap = 0;
    c->out_n = 0;
    if (cap > 0) {
        if (pgk_dmalloc(c, &c->out_rec, sizeof(double) * PGK_OUT_NCOL * (size_t)cap) != cudaSuccess) {
            c->out_rec = nullptr;
            return pgk_fail(c, PGK_E_NOMEM, "output record buffer");
        }
        c->out_cap = cap;
    }
    return PGK_OK;
}

pgk_status pgk_get_output(pgk_ctx* c, double* out, int64_t cap, int64_t* n) {
    if (!c || cap < 0) return PGK_E_INVALID;
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    long long have = std::min<long long>(c->out_n, c->out_cap);
    if (out && cap > 0 && have > 0)
        PGK_CUDA(c, cudaMemcpy(out, c->out_rec, sizeof(double) * PGK_OUT_NCOL * std::min<long long>(have, cap),
                               cudaMemcpyDeviceToHost));
    if (n) *n = c->out_n;
    c->out_n = 0;
    return PGK_OK;
}

pgk_status pgk_set_hf(pgk_ctx* c, const pgk_hfparams* hf) {
    if (!c || !hf) return PGK_E_INVALID;
    if (c->nmor)   // the per-atom Morse shares of morsep_hf (morse_hf.F90) are not built on the device
        return pgk_fail(c, PGK_E_UNSUPPORTED, "heat flux with Morse pairs (morsep_hf) is not built");
    pgk_status s = hf_setup(c, hf);
    if (s) return s;
    PGK_CUDA(c, cudaStreamSynchronize(cudaStreamLegacy));   // its table copies (synchronous host arrays)
    return PGK_OK;
}

pgk_status pgk_moldyn_hf(pgk_ctx* c, int64_t ini, int64_t end, const pgk_mdparams* md, pgk_energies* e,
                         double* hf_out, int64_t cap_records, int64_t* nrecords) {
    if (!c || !md || cap_records < 0) return PGK_E_INVALID;
    if (!c->hf_set) return pgk_fail(c, PGK_E_INVALID, "pgk_set_hf has not been called");
    const long long per = (long long)c->hfp.nhfregion * PGK_HF_NCOL;
    const int hfi = c->hfp.heatfinterval > 0 ? c->hfp.heatfinterval : 1;
    long long expect = 0;
    if (per > 0)
        for (int64_t st = std::max<int64_t>(ini, 1); st <= end; ++st) expect += (hfi == 1 || st % hfi == 1) ? 1 : 0;
    long long want = hf_out ? std::min<long long>(expect, cap_records) : 0;
    if (per > 0 && want > c->hf_rec_cap) {
        pgk_dfree(c, c->hf_rec);
        c->hf_rec = nullptr;
        PGK_CUDA(c, pgk_dmalloc(c, &c->hf_rec, sizeof(double) * per * want));
        c->hf_rec_cap = want;
    }
    long long cap_save = c->hf_rec_cap;
    c->hf_rec_cap = want;
    long long nr = 0;
    pgk_status s = run_md(c, 3, ini, end, md, e, &nr);
    c->hf_rec_cap = std::max(cap_save, 1LL);
    if (s) return s;
    if (hf_out && want > 0)
        PGK_CUDA(c, cudaMemcpy(hf_out, c->hf_rec, sizeof(double) * per * std::min(nr, want), cudaMemcpyDeviceToHost));
    if (nrecords) *nrecords = nr;
    return PGK_OK;
}

pgk_status pgk_set_hf_kspace(pgk_ctx* c, int32_t mode, int32_t kmax) {
    if (!c) return PGK_E_INVALID;
    if (mode == PGK_HF_KSPACE_SPME && !c->prm.ifspme) return pgk_fail(c, PGK_E_INVALID, "ifspme is off");
    if (mode == PGK_HF_KSPACE_EWK && kmax < 1) return pgk_fail(c, PGK_E_INVALID, "kmax must be at least 1");
    if (mode != PGK_HF_KSPACE_NONE && mode != PGK_HF_KSPACE_EWK && mode != PGK_HF_KSPACE_SPME)
        return pgk_fail(c, PGK_E_INVALID, "unknown k-space heat-flux mode");
    c->hf_kspace = mode;
    c->hf_kmax = mode == PGK_HF_KSPACE_EWK ? kmax : 0;
    c->hf_ewk_fresh = false;
    return PGK_OK;
}

pgk_status pgk_fft_pme_hf(pgk_ctx* c, double* pot_atm, double* viri_atm) {
    if (!c) return PGK_E_INVALID;
    pgk_status s = launch_spme_hf_atm(c);
    if (s) return s;
    const size_t n = (size_t)c->natom;
    if (pot_atm) PGK_CUDA(c, cudaMemcpyAsync(pot_atm, c->hfk_out, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    if (viri_atm)
        PGK_CUDA(c, cudaMemcpyAsync(viri_atm, c->hfk_out + n, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return read_status(c);
}

pgk_status pgk_calheatf(pgk_ctx* c, double* hf) {
    if (!c || !hf) return PGK_E_INVALID;
    if (!c->hf_set || c->hfp.nhfregion < 1) return pgk_fail(c, PGK_E_INVALID, "no heat-flux regions set");
    pgk_status s;
    if (!c->list_valid && (s = launch_mklist(c))) return s;
    if ((s = launch_pack(c)) || (s = launch_hf_atm(c)) || (s = launch_heatf(c, c->hf_rec))) return s;
    PGK_CUDA(c, cudaMemcpyAsync(hf, c->hf_rec, sizeof(double) * c->hfp.nhfregion * PGK_HF_NCOL,
                                cudaMemcpyDeviceToHost, c->st));
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    return read_status(c);
}

pgk_status pgk_get_hf_atm(pgk_ctx* c, double* pot_atm, double* viri_atm) {
    if (!c) return PGK_E_INVALID;
    if (!c->hf_set) return pgk_fail(c, PGK_E_INVALID, "pgk_set_hf has not been called");
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    size_t n = (size_t)c->natom;
    if (pot_atm) PGK_CUDA(c, cudaMemcpy(pot_atm, c->hf_pot, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost));
    if (viri_atm && c->hfp.nhfregion > 0)
        PGK_CUDA(c, cudaMemcpy(viri_atm, c->hf_W, sizeof(double) * 8 * c->hfp.nhfregion * 3 * n,
                               cudaMemcpyDeviceToHost));
    return PGK_OK;
}

pgk_status pgk_langevin_dekin(pgk_ctx* c, double* out) {
    if (!c || !out) return PGK_E_INVALID;
    if (!c->hf_set) return pgk_fail(c, PGK_E_INVALID, "pgk_set_hf has not been called");
    PGK_CUDA(c, cudaStreamSynchronize(c->st));
    double h[PGK_LT_MAX_REGIONS];
    PGK_CUDA(c, cudaMemcpy(h, c->lt_dekin, sizeof(h), cudaMemcpyDeviceToHost));
    for (int r = 0; r < c->hfp.nlangeregion; ++r) out[r] = h[r];
    PGK_CUDA(c, cudaMemsetAsync(c->lt_dekin, 0, sizeof(h), c->st));
    return PGK_OK;
}
}
