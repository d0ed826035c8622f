// pgk_serve.cu -- replica server: continuous batching of independent systems.
//
// No counterpart in the reference (peachgk_md runs one system per process).
// Requests (system, parameters, initial state, number of steps) are queued
// and admitted while earlier ones run, as worker slots and the device-memory
// budget allow (pgk_estimate_bytes).  Every admitted replica owns a full
// engine context -- coordinates, pair list, PME grids, thermostat state stay
// resident -- and its own non-blocking CUDA stream; one host worker thread
// per slot advances it in chunks of steps (each chunk replays the captured
// CUDA graph of the step, see run_md), so the kernels of different replicas
// overlap on the device.  A replica's results do not depend on what else
// runs: its kernels touch only its own buffers, and in mixed precision every
// force/energy sum is an integer sum, so the results are bit-identical to a
// run of the same replica alone.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "pgk_ctx.cuh"

namespace {

// deep copy of a pgk_system (the caller's arrays may go away after submit)
struct SystemCopy {
    pgk_system s{};
    std::vector<std::vector<double>> d;
    std::vector<std::vector<int32_t>> i;
    const double* cd(const double* p, size_t n) {
        if (!p || n == 0) return nullptr;
        d.emplace_back(p, p + n);
        return d.back().data();
    }
    const int32_t* ci(const int32_t* p, size_t n) {
        if (!p || n == 0) return nullptr;
        i.emplace_back(p, p + n);
        return i.back().data();
    }
    explicit SystemCopy(const pgk_system& x) {
        d.reserve(40); i.reserve(40);    // pointers into the vectors must stay valid
        s = x;
        const size_t n = (size_t)x.natom, t2 = (size_t)x.ntyp * x.ntyp;
        s.atmmass = cd(x.atmmass, n); s.atmchrg = cd(x.atmchrg, n); s.atmindex = ci(x.atmindex, n);
        s.vdw_radij = cd(x.vdw_radij, t2); s.vdw_welij = cd(x.vdw_welij, t2);
        s.inter_inttyp = ci(x.inter_inttyp, t2);
        s.para_welmor = cd(x.para_welmor, t2); s.para_radmor = cd(x.para_radmor, t2);
        s.para_alphamor = cd(x.para_alphamor, t2);
        s.molept_index = ci(x.molept_index, (size_t)x.nmole + 1);
        s.molept_list = ci(x.molept_list, x.molept_index ? (size_t)(x.molept_index[x.nmole] - 1) : 0);
        s.index_excl = ci(x.index_excl, n + 1);
        s.list_excl = ci(x.list_excl, x.index_excl ? (size_t)(x.index_excl[n] - 1) : 0);
        const size_t nb = x.nbond, na = x.nangl, nt = x.ntors, nr = x.ntorsrb;
        s.ibond = ci(x.ibond, nb); s.jbond = ci(x.jbond, nb);
        s.para_cbond = cd(x.para_cbond, nb); s.para_eqbond = cd(x.para_eqbond, nb);
        s.iangl = ci(x.iangl, na); s.jangl = ci(x.jangl, na); s.kangl = ci(x.kangl, na);
        s.para_cangl = cd(x.para_cangl, na); s.para_eqangl = cd(x.para_eqangl, na);
        s.itors = ci(x.itors, nt); s.jtors = ci(x.jtors, nt); s.ktors = ci(x.ktors, nt); s.ltors = ci(x.ltors, nt);
        s.para_divfac = ci(x.para_divfac, nt); s.para_barhig = cd(x.para_barhig, nt);
        s.para_phsang = cd(x.para_phsang, nt); s.para_period = cd(x.para_period, nt);
        s.ifcalnonb14 = ci(x.ifcalnonb14, nt); s.para_divfac_vdw = cd(x.para_divfac_vdw, nt);
        s.para_divfac_elc = cd(x.para_divfac_elc, nt); s.ring14 = cd(x.ring14, nt);
        s.itorsrb = ci(x.itorsrb, nr); s.jtorsrb = ci(x.jtorsrb, nr); s.ktorsrb = ci(x.ktorsrb, nr);
        s.ltorsrb = ci(x.ltorsrb, nr); s.para_barhigrb = cd(x.para_barhigrb, 6 * nr);
        s.ifcalnonb14_rb = ci(x.ifcalnonb14_rb, nr); s.para_divfac_vdwrb = cd(x.para_divfac_vdwrb, nr);
        s.para_divfac_elcrb = cd(x.para_divfac_elcrb, nr); s.ring14_rb = cd(x.ring14_rb, nr);
        s.index_mconst = ci(x.index_mconst, (size_t)x.nconst + 1);
        s.list_mconst = ci(x.list_mconst, x.index_mconst ? (size_t)(x.index_mconst[x.nconst] - 1) : 0);
        s.iconst = ci(x.iconst, x.nconstraint); s.jconst = ci(x.jconst, x.nconstraint);
        s.dconst = cd(x.dconst, x.nconstraint);
    }
};

struct Job {
    int64_t id = 0;
    std::unique_ptr<SystemCopy> sys;
    pgk_params prm{};
    pgk_mdparams md{};
    int kind = 0;
    bool has_hf = false;
    pgk_hfparams hf{};
    std::vector<int32_t> hftyp, ltmole;
    std::vector<double> x0, v0;
    double box0[3] = {0, 0, 0};
    bool has_chain = false;
    pgk_chain chain{};
    int64_t nsteps = 0;
    int64_t bytes = 0;
    // results
    std::vector<double> x, v, rec;
    double box[3] = {0, 0, 0};
    pgk_energies ene{};
    int64_t nrec = 0;
    pgk_status status = PGK_OK;
    std::string err;
    bool done = false;
    double t_submit = 0, t_start = 0, t_done = 0;
};

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct pgk_server {
    int device = 0;
    int64_t budget = 0, in_use = 0;
    int64_t next_id = 1;
    bool stop = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> queue;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    std::vector<std::thread> workers;
    int running = 0;
};

static void run_job(pgk_server* sv, Job* j) {
    cudaSetDevice(sv->device);
    pgk_ctx* c = nullptr;
    pgk_status s = pgk_init(&j->sys->s, &j->prm, &c);
    if (s == PGK_OK) s = pgk_upload_state(c, j->x0.data(), j->v0.data(), j->box0);
    if (s == PGK_OK && j->has_chain) s = pgk_set_chain(c, &j->chain);
    if (s == PGK_OK && j->has_hf) {
        pgk_hfparams h = j->hf;
        h.hftyp_atm = j->hftyp.empty() ? nullptr : j->hftyp.data();
        h.lt_mole_based = j->ltmole.empty() ? nullptr : j->ltmole.data();
        s = pgk_set_hf(c, &h);
    }
    if (s == PGK_OK) {
        const size_t per = j->has_hf ? (size_t)j->hf.nhfregion * PGK_HF_NCOL : 0;
        if (j->kind == 3) {
            int64_t cap = 0;
            if (per > 0) {
                const int hfi = j->hf.heatfinterval > 0 ? j->hf.heatfinterval : 1;
                for (int64_t st = 1; st <= j->nsteps; ++st) cap += (hfi == 1 || st % hfi == 1) ? 1 : 0;
            }
            j->rec.assign((size_t)cap * per, 0.0);
            s = pgk_moldyn_hf(c, 0, j->nsteps, &j->md, &j->ene, j->rec.empty() ? nullptr : j->rec.data(), cap,
                              &j->nrec);
        } else if (j->kind == 0) {
            s = pgk_moldyn_nve(c, 0, j->nsteps, &j->md, &j->ene);
        } else if (j->kind == 1) {
            s = pgk_moldyn_nhc(c, 0, j->nsteps, &j->md, &j->ene);
        } else {
            s = pgk_moldyn_mtk(c, 0, j->nsteps, &j->md, &j->ene);
        }
    }
    if (s == PGK_OK) {
        j->x.resize(j->x0.size());
        j->v.resize(j->v0.size());
        s = pgk_download_state(c, j->x.data(), j->v.data(), j->box);
    }
    if (s != PGK_OK) j->err = c ? pgk_last_error(c) : pgk_status_string(s);
    if (c) pgk_free(c);
    j->status = s;
}

static void worker_main(pgk_server* sv) {
    cudaSetDevice(sv->device);
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv_work.wait(lk, [&] {
                if (sv->stop) return true;
                // admit in arrival order while the memory budget allows; a job
                // larger than the whole budget runs alone
                if (sv->queue.empty()) return false;
                Job* f = sv->queue.front();
                return sv->in_use + f->bytes <= sv->budget || sv->running == 0;
            });
            if (sv->stop && sv->queue.empty()) return;
            if (sv->queue.empty()) continue;
            j = sv->queue.front();
            if (!(sv->in_use + j->bytes <= sv->budget || sv->running == 0)) continue;
            sv->queue.pop_front();
            sv->in_use += j->bytes;
            ++sv->running;
            j->t_start = now_s();
        }
        run_job(sv, j);
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            j->t_done = now_s();
            j->done = true;
            sv->in_use -= j->bytes;
            --sv->running;
            j->sys.reset();
            j->x0.clear(); j->x0.shrink_to_fit();
            j->v0.clear(); j->v0.shrink_to_fit();
        }
        sv->cv_work.notify_all();
        sv->cv_done.notify_all();
    }
}

extern "C" {

int64_t pgk_estimate_bytes(const pgk_system* s, const pgk_params* p) {
    if (!s || !p) return -1;
    const double n = s->natom;
    const bool mixed = p->precision == PGK_PREC_MIXED;
    const double vol = p->xcel * p->ycel * p->zcel;
    const double nc = std::max(1.0, std::floor(p->xcel / p->rcut_book)) *
                      std::max(1.0, std::floor(p->ycel / p->rcut_book)) *
                      std::max(1.0, std::floor(p->zcel / p->rcut_book));
    const double npad = n + 7.0 * nc;
    const double rs = p->rcut_book + 2.0;
    double cap = (n / vol * 4.0 / 3.0 * 3.14159265358979 * rs * rs * rs + 128) * 1.25;   // rows regrow with headroom
    if (p->max_nbr > 0) cap = p->max_nbr;
    const double rows = mixed ? 2.0 : 1.0;                                 // book + pruned rows (mixed)
    double bytes = n * (3 * 24 + 3 * 8 + 4 + 2 * 24 + 12 + 1 + 24)       // state, forces, list keys
                 + npad * (4 + 24 + 4 + (mixed ? 16 + 24 + 16 : 32))       // sorted copies, slot forces, prune origin
                 + rows * npad / 8.0 * (cap + 1) * 4                       // cluster rows
                 + n * 400.0;                                              // bonded terms and incidence
    if (p->ifspme) {
        const double K = (double)p->nfft1 * p->nfft2 * p->nfft3;
        bytes += K * (8 + (mixed ? 8 + 4 : 16 + 8));                       // accumulation, complex and real grids
    }
    bytes = bytes * 1.25 + 16.0 * (1 << 20);                               // regrowth margin + fixed
    return (int64_t)bytes;
}

pgk_status pgk_server_create(int32_t max_slots, int64_t hbm_budget_bytes, pgk_server** out) {
    if (!out || max_slots < 1 || max_slots > 256) return PGK_E_INVALID;
    pgk_server* sv = new pgk_server();
    cudaGetDevice(&sv->device);
    if (hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { delete sv; return PGK_E_CUDA; }
        hbm_budget_bytes = (int64_t)(0.8 * (double)fr);
    }
    sv->budget = hbm_budget_bytes;
    for (int k = 0; k < max_slots; ++k) sv->workers.emplace_back(worker_main, sv);
    *out = sv;
    return PGK_OK;
}

pgk_status pgk_server_submit(pgk_server* sv, const pgk_request* r, int64_t* id) {
    if (!sv || !r || !r->sys || !r->prm || !r->md || !r->atmcor || r->nsteps < 0) return PGK_E_INVALID;
    if (r->kind < 0 || r->kind > 3 || (r->kind == 3 && !r->hf)) return PGK_E_INVALID;
    std::unique_ptr<Job> j(new Job());
    const size_t n3 = (size_t)3 * r->sys->natom;
    j->sys.reset(new SystemCopy(*r->sys));
    j->prm = *r->prm;
    j->md = *r->md;
    j->kind = r->kind;
    j->nsteps = r->nsteps;
    j->x0.assign(r->atmcor, r->atmcor + n3);
    if (r->atmvel) j->v0.assign(r->atmvel, r->atmvel + n3); else j->v0.assign(n3, 0.0);
    if (r->box) for (int d = 0; d < 3; ++d) j->box0[d] = r->box[d];
    else { j->box0[0] = r->prm->xcel; j->box0[1] = r->prm->ycel; j->box0[2] = r->prm->zcel; }
    if (r->chain) { j->has_chain = true; j->chain = *r->chain; }
    if (r->hf) {
        j->has_hf = true;
        j->hf = *r->hf;
        if (r->hf->hftyp_atm) j->hftyp.assign(r->hf->hftyp_atm, r->hf->hftyp_atm + r->sys->natom);
        if (r->hf->lt_mole_based) j->ltmole.assign(r->hf->lt_mole_based, r->hf->lt_mole_based + r->sys->nmole);
    }
    j->bytes = pgk_estimate_bytes(r->sys, r->prm);
    if (j->has_hf) j->bytes += (int64_t)8 * r->sys->natom * (8 + 8 * 3 * j->hf.nhfregion + 4);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        j->id = sv->next_id++;
        j->t_submit = now_s();
        if (id) *id = j->id;
        sv->queue.push_back(j.get());
        sv->jobs[j->id] = std::move(j);
    }
    sv->cv_work.notify_all();
    return PGK_OK;
}

pgk_status pgk_server_poll(pgk_server* sv, int64_t id, int32_t* done) {
    if (!sv || !done) return PGK_E_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return PGK_E_INVALID;
    *done = it->second->done ? 1 : 0;
    return PGK_OK;
}

pgk_status pgk_server_wait(pgk_server* sv, int64_t id) {
    if (!sv) return PGK_E_INVALID;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return PGK_E_INVALID;
    Job* j = it->second.get();
    sv->cv_done.wait(lk, [&] { return j->done; });
    return PGK_OK;
}

pgk_status pgk_server_result(pgk_server* sv, int64_t id, double* atmcor, double* atmvel, double* box,
                             pgk_energies* ene, double* hf_out, int64_t cap_records, int64_t* nrecords,
                             double* times3) {
    if (!sv) return PGK_E_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end() || !it->second->done) return PGK_E_INVALID;
    Job* j = it->second.get();
    if (j->status != PGK_OK) return j->status;
    if (atmcor) std::memcpy(atmcor, j->x.data(), j->x.size() * sizeof(double));
    if (atmvel) std::memcpy(atmvel, j->v.data(), j->v.size() * sizeof(double));
    if (box) for (int d = 0; d < 3; ++d) box[d] = j->box[d];
    if (ene) *ene = j->ene;
    if (nrecords) *nrecords = j->nrec;
    if (hf_out && j->has_hf) {
        const size_t per = (size_t)j->hf.nhfregion * PGK_HF_NCOL;
        const size_t nr = (size_t)std::min<int64_t>(cap_records, (int64_t)(j->rec.size() / std::max<size_t>(per, 1)));
        std::memcpy(hf_out, j->rec.data(), nr * per * sizeof(double));
    }
    if (times3) { times3[0] = j->t_submit; times3[1] = j->t_start; times3[2] = j->t_done; }
    return PGK_OK;
}

const char* pgk_server_error(pgk_server* sv, int64_t id) {
    if (!sv) return "";
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return "unknown request id";
    return it->second->err.c_str();
}

pgk_status pgk_server_release(pgk_server* sv, int64_t id) {
    if (!sv) return PGK_E_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end() || !it->second->done) return PGK_E_INVALID;
    sv->jobs.erase(it);
    return PGK_OK;
}

pgk_status pgk_server_free(pgk_server* sv) {
    if (!sv) return PGK_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    for (auto& t : sv->workers) t.join();
    delete sv;
    return PGK_OK;
}

}  // extern "C"
