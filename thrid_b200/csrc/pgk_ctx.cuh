// pgk_ctx.cuh -- the engine context (host view of all device buffers) and
// the launchers each kernel file exports.
#pragma once

#include <cuda_runtime.h>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "pgk_internal.cuh"

#define PGK_MAX_RADIX_STAGES 12

struct FftPlan {              // one axis of the 3-D transform
    int n;
    int nstage;
    int radix[PGK_MAX_RADIX_STAGES];
    void* tw;                 // complex twiddles exp(-2 pi i m / n), m < n (T2)
};

// bonded-term arrays on the host before chunk ordering / upload (0-based atoms)
struct HostTerms {
    std::vector<int2> bij; std::vector<double2> bp;
    std::vector<int4> aijk; std::vector<double2> ap;
    std::vector<int4> tij; std::vector<double4> tp;
    std::vector<int4> rij; std::vector<double> rc;
    std::vector<int2> p14; std::vector<double2> f14;
    std::vector<int2> ex;
    // per-atom data the block kernel's per-term constants are formed from
    const double* q = nullptr; const int* ty = nullptr; const double2* lj = nullptr; int ntyp = 0;
};

struct pgk_ctx {
    int natom = 0;
    int prec = PGK_PREC_FP64;
    bool mixed() const { return prec == PGK_PREC_MIXED; }
    pgk_params prm{};
    cudaStream_t st = nullptr;
    // second stream of the force evaluation: the SPME chain runs on it beside
    // the pair and bonded kernels (fork and join through the two events;
    // integer or FP64 atomics on the shared force and energy accumulators)
    double* ke_part = nullptr;    // [2 nsm][10] per-block kinetic sums (k_kinetic_end)
    unsigned* ke_done = nullptr;  // blocks of k_kinetic_end finished (zero between launches)
    cudaStream_t st2 = nullptr;   // SPME chain of a force evaluation
    cudaStream_t st3 = nullptr;   // bonded terms of a force evaluation
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join3 = nullptr;
    // recorded by launch_pair just before the pair kernel when rec_pre_pair
    // is set: the bonded terms of a forked evaluation wait for it
    cudaEvent_t ev_pre_pair = nullptr;
    bool rec_pre_pair = false, rec_pre_pair_done = false;
    cudaMemPool_t pool = nullptr; // the device's memory pool (pgk_dmalloc)
    std::string err;
    long long launches = 0;
    int nsm = 148;
    int degfree = 0;
    double* fout = nullptr;       // 3N doubles of scratch for force read-back

    // ---- atoms ----
    double *pos = nullptr, *vel = nullptr, *pos_old = nullptr;
    double *mass = nullptr, *invmass = nullptr, *chrg = nullptr;
    int* typ = nullptr;           // 0-based LJ type
    void* facc[2] = {nullptr, nullptr};
    long long* acc = nullptr;     // [2][NACC]
    DynState* dyn = nullptr;      // device
    DynState hdyn{};              // host shadow (valid after sync_dyn)
    ChainDev* chain = nullptr;    // device
    unsigned* status = nullptr;   // device sticky status bits
    double pot_ewc = 0.0, netchrgsq = 0.0;
    double yratio = 1.0, zratio = 1.0;

    // ---- LJ + spline tables ----
    int ntyp = 0;
    double2* lj64 = nullptr;      // (R^2, E) per (i,j)
    float2* lj32 = nullptr;
    int nspl = 0;
    double hspl = 0.0;
    double4* spl64 = nullptr;     // [4][nspl] (a,b,c,d): 0 real, 1 realpot, 2 excs, 3 excspot
    float4* spl32 = nullptr;

    // ---- exclusions ----
    int *exs_idx = nullptr, *exs_list = nullptr;   // symmetric, 0-based, sorted
    int2* exs_rng = nullptr;                        // per atom: (lowest, highest) partner
    int2* expair = nullptr; int nexpair = 0;        // reference pairs i<j
    int max_excl = 0;

    // ---- molecules ----
    int nmole = 0;
    int *mol_idx = nullptr, *mol_list = nullptr;

    // ---- bonded ----
    int nbond = 0; int2* bond_ij = nullptr; double2* bond_p = nullptr;
    int nangl = 0; int4* angl_ijk = nullptr; double2* angl_p = nullptr;
    int ntors = 0; int4* tors_ijkl = nullptr; double4* tors_p = nullptr;   // (barhig/divfac, phsang, period, cos(phs))
    int ntorsrb = 0; int4* rb_ijkl = nullptr; double* rb_c = nullptr;       // [6*n]
    int n14 = 0; int2* p14_ij = nullptr; double2* p14_f = nullptr;          // (elc fac, vdw fac)

    // ---- bonded block plan ----
    // Per type (bond, angle, tors, RB, 1-4, excl) the terms [0, nnear) are the
    // "near" ones (atom span < BLK_FAR_SPAN), sorted by their lowest atom; the
    // rest [nnear, n) go through the per-type kernels with force atomics.
    // Block b owns the near terms whose lowest atom lies in its atom range;
    // its local atoms are [a0, a0 + nloc).
    int nnear[6] = {0, 0, 0, 0, 0, 0};
    int nblk = 0;
    int* blk_a0 = nullptr;        // [nblk]
    int* blk_nloc = nullptr;      // [nblk]
    int* blk_t = nullptr;         // [6][nblk+1] first term of each block, per type
    int* blk_soff = nullptr;      // [nblk][8] local slot offset per type, [6] = slot count
    int* blk_ip = nullptr;        // [nblk] offset of the block's nloc+1 pointers in blk_incp
    int* blk_incp = nullptr;      // per block and local atom: range in blk_inc
    unsigned short* blk_inc = nullptr;   // local slot ids, per atom by type, term, position
    uint2* brec[6] = {};          // per type: compact records of the near terms
    double* btab[6] = {};         // per type: distinct parameter tuples

    // ---- constraints ----
    bool short_empty = false;     // no term in the short MTS group
    int ncgroup = 0, nconstraint = 0;
    int *cg_idx = nullptr, *cg_list = nullptr;
    int2* c_ij = nullptr; double* c_d = nullptr;
    int2* cg_span = nullptr;      // (first atom, atom count) of each group's contiguous span
    unsigned char* cg_fit = nullptr;   // per 32 groups: 1 = staged in shared memory (k_rattle_warp)
    int cg_nfit = 0;
    // rigid three-atom groups (constraints (a0,a1), (a0,a2), (a1,a2) in that
    // order: rigid water) kept out of the group arrays above, run by
    // k_rattle_rigid3 with their state in registers
    int nr3 = 0;
    int4* r3_atoms = nullptr;     // (a0, a1, a2, -)
    double4* r3_d = nullptr;      // constraint lengths (d01, d02, d12, -)
    // star groups: constraints (c, a1), (c, a2), ... (c, aK), K <= 4 (X-H
    // bonds of one heavy atom), sorted by K from 4 down to 1, run by
    // k_rattle_star with their state in registers
    int nstar = 0;
    int star_seg[4] = {0, 0, 0, 0};   // first group with K = 3, 2, 1; [3] = nstar
    int* star_atoms = nullptr;    // [nstar][5]: c, a1..a4 (unused arms -1)
    double* star_d = nullptr;     // [nstar][4] constraint lengths

    // ---- pair list ----
    int maxcells = 0;
    int *cell_of = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
    int* subkey = nullptr;        // (sub-cell << 25) | atom, sort key inside a cell
    // Sorted order: each cell's atoms start on a multiple of 8 (8-atom
    // clusters); slots past a cell's count are padding (perm = -1).
    int npad = 0;                 // sorted slots in use (multiple of 8)
    int npad_cap = 0;             // allocated sorted slots
    int ncl = 0;                  // clusters = npad / 8
    int* perm = nullptr;          // sorted slot -> original atom, -1 = padding
    int* iperm = nullptr;         // original -> sorted slot
    double* pos_s = nullptr;      // sorted FP64 positions at list time (3*npad)
    int* clist = nullptr;         // [ncl * ccap] entries (mask << 24) | j-slot
    int* ccnt = nullptr;          // [ncl]
    // pruned copy of the rows (mixed precision, see PruneDev)
    int* plist = nullptr;         // [ncl * ccap]
    int* pcnt = nullptr;          // [ncl]
    int4* xq_prune = nullptr;     // xq at the last prune
    PruneDev* prune = nullptr;
    float prune_buffer = 0.f;     // A; 0 = no pruning (pair kernel reads the book rows)
    bool no_frame = false;        // PGK_PAIR_FRAME=0: always the per-pair minimum image
    int pair_waves = 3;           // waves of blocks of the cluster-frame pair kernel (pair_autotune)
    bool pair_tuned = false;
    int ccap = 0;
    int4* xq = nullptr;           // mixed: fixed-point fractional coords + q bits
    long long* fsort = nullptr;   // mixed: pair forces by sorted slot, [3][npad_cap] int64 fixed point (kept zero between uses)
    double4* xq64 = nullptr;      // fp64: x,y,z,q sorted
    int* typ_s = nullptr;
    unsigned long long* counters = nullptr;   // [0] list pairs, [1] longest cluster row, [2] rows without
                                              //  a higher-index partner; [4..6] count_pairs scratch
    unsigned char* hasup = nullptr;           // [N] atom has a list partner of higher index
    bool list_valid = false;
    long long list_epoch = 0;     // incremented by every list build (invalidates captured graphs)

    // ---- SPME ----
    int K[3] = {0, 0, 0};
    int order = 0;
    void* qacc = nullptr;         // accumulation grid (int64 fixed / double)
    void* qc = nullptr;           // complex grid (float2 / double2)
    void* qr = nullptr;           // real part after the backward transform (float / double), read by the gather
    double* bsp = nullptr;        // bsp_mod1|2|3
    FftPlan plan[3];
    // real-to-complex x transform (K1 even, K1/2 a product of 2, 3, 5): the
    // complex grid holds K1/2 + 1 points per x line; plan_rx is the length-
    // K1/2 complex transform, tw_rx the K1/2 + 1 factors exp(-2 pi i k / K1)
    bool r2c = false;
    FftPlan plan_rx;
    void* tw_rx = nullptr;
    int fft_p[5] = {0, 0, 0, 0, 0};  // pencils per block: x, y, z, z+influence, real x (0: default)

    // ---- Morse pairs (k_morse.cu): own list (radius rcut_bookmor) and kernel ----
    int nmor = 0;                 // Morse atoms (0: no Morse pairs or Morse switched off)
    int* mor_atoms = nullptr;     // [nmor] nmorselist, 0-based ascending
    double4* mor_par = nullptr;   // [ntyp*ntyp] (D, r0, alpha, Morse type pair) at it + ntyp*jt
    int mor_cap = 0;              // row capacity (entries)
    int* mor_rows = nullptr;      // [nmor * mor_cap] partners, reference row order
    int* mor_cnt = nullptr;       // [nmor]
    int* mor_cell = nullptr;      // [nmor] cell key (cell mode)
    int* mor_csort = nullptr;     // [nmor] Morse atoms by cell, ascending inside a cell
    int *mor_ccnt = nullptr, *mor_cstart = nullptr, *mor_cfill = nullptr;
    int mor_maxcells = 0;
    unsigned long long* mor_ctr = nullptr;   // [0] entries, [1] longest row of the last build
    int mor_mode = 0;             // PGK_LIST_* order of the last build
    long long mor_entries = 0;
    bool mor_valid = false;

    // ---- device-side output records ----
    double* out_rec = nullptr;    // [out_cap][PGK_OUT_NCOL]
    long long out_cap = 0, out_n = 0;

    // ---- heat flux and region Langevin thermostat (k_heatf.cu) ----
    bool hf_set = false;
    pgk_hfparams hfp{};           // host copy (pointer members cleared)
    int* mol_of = nullptr;        // [N] molecule of each atom
    int* hftyp = nullptr;         // [N] PGK_HFTYP_*
    double* molecom = nullptr;    // [3*nmole] calcom.F90 centres at the last heat-flux evaluation
    double* molevel = nullptr;    // [3*nmole]
    double* hf_pot = nullptr;     // [8][N]
    double* hf_W = nullptr;       // [8][nreg][3][N]
    double* hf_part = nullptr;    // [hf_nblk][nreg][17] calheatf block partials
    double* hf_rec = nullptr;     // device heat-flux records
    long long hf_rec_cap = 1;     // records hf_rec holds
    int hf_nblk = 0;
    double* hf_zs = nullptr;      // [npad_cap] heat-flux z of each sorted slot
    int* hf_ms = nullptr;         // [npad_cap] molecule tag of each sorted slot
    int hf_slots_cap = 0;
    int* lt_mole = nullptr;       // [nmole] register by centre of mass
    int* lt_reg = nullptr;        // [N] Langevin region (-1: none)
    double* lt_frand = nullptr;   // [3N] random accelerations of the former half step
    double* lt_dekin = nullptr;   // [8] det_ene_kin

    // ---- standard-Ewald k-space of the bulk heat flux (k_ewald.cu) ----
    int ewk_kmax = 0;             // wave set held in ewk_nv (0: none)
    int ewk_nwave = 0;            // waves, (0,0,0) first
    int ewk_nmax[3] = {0, 0, 0};  // largest |n| per axis
    int4* ewk_nv = nullptr;       // [nwave] (nx, ny, nz, 0)
    double2* ewk_tab = nullptr;   // [rows][N] exp(2 pi i n r_d / L_d), rows = n 0..nmax of x, y, z
    double2* ewk_part = nullptr;  // [nchunk][nwave] structure-factor partial sums (cos, sin)
    double* ewk_coef = nullptr;   // [nwave][EWK_NCOEF] per-wave coefficients
    double* ewk_red = nullptr;    // [wave blocks][8] energy / tensor partials
    double* ewk_out = nullptr;    // force 3N | energy N | tensor 9N | scalars 11
    double* ewk_seg = nullptr;    // [nseg][11][N] per-atom sums of the wave segments
    size_t ewk_bytes[6] = {0, 0, 0, 0, 0, 0};   // allocated sizes of tab, part, coef, red, out, seg

    // ---- SPME per-atom reciprocal split of the heat flux (k_spme.cu) ----
    double* hfk_q = nullptr;      // [K^3] double charge grid
    void* hfk_g = nullptr;        // [7][K^3] double2 convolved grids
    double* hfk_out = nullptr;    // energies [N] | tensors [9N]
    void* hfk_tw[3] = {nullptr, nullptr, nullptr};   // FP64 twiddles per axis
    int hf_kspace = 0;            // PGK_HF_KSPACE_* (pgk_set_hf_kspace)
    int hf_kmax = 0;              // waves of the standard-Ewald option
    bool hf_ewk_now = false;      // this force evaluation is the heat-flux step's (standard-Ewald option)
    bool hf_ewk_fresh = false;    // ewk_out holds ewaldkp_hf at the current positions

    // ---- CUDA graphs of captured MD steps (key: driver kind and step flags);
    //      valid for one list build and one set of integrator parameters ----
    struct GraphEntry { cudaGraphExec_t exec; long long launches; long long epoch; };
    std::map<int, GraphEntry> graphs;
    pgk_mdparams graph_md{};
    bool use_graphs = true;
    std::string graph_fail;       // why capture was switched off (empty: never failed)

    // ---- scratch for host transfers ----
    std::vector<double> hbuf;
};

// Device memory of a context is stream-ordered: allocations come from one
// memory pool per device (cached: nothing is returned to the driver between
// contexts) on the context's stream, followed by a wait on that stream so
// the memory is usable by any stream and by synchronous copies at once;
// frees are ordered on the context's stream.  Neither synchronises the
// device (cudaMalloc / cudaFree would), so the contexts of concurrent
// replicas start, grow their lists and end without stalling each other's
// streams or invalidating a graph capture in flight on another thread.
cudaError_t pgk_dmalloc(pgk_ctx* c, void** p, size_t bytes);
cudaError_t pgk_dfree(pgk_ctx* c, void* p);
template <typename T>
inline cudaError_t pgk_dmalloc(pgk_ctx* c, T** p, size_t bytes) { return pgk_dmalloc(c, (void**)p, bytes); }

// Raise a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit is a process-wide property of the kernel, shared by every context
// and host thread, so it only ever grows (a lower value set by one replica
// would make another replica's larger launch fail).
cudaError_t smem_limit(const void* kernel, size_t bytes);
template <typename K>
inline cudaError_t smem_limit(K* kernel, size_t bytes) { return smem_limit((const void*)kernel, bytes); }

// error helpers
pgk_status pgk_fail(pgk_ctx* c, pgk_status s, const std::string& msg);
#define PGK_CUDA(ctx, call)                                                               \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return pgk_fail(ctx, PGK_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define PGK_LAUNCHED(ctx) do { (ctx)->launches++; } while (0)

// ---- launchers (k_list.cu) ----
pgk_status launch_transcor(pgk_ctx* c);
pgk_status launch_mklist(pgk_ctx* c);
pgk_status export_nblist(pgk_ctx* c, int32_t* nb_index, int32_t* nb_list, int64_t cap, int64_t* nl);

// ---- launchers (k_nonbond.cu) ----
pgk_status launch_pack(pgk_ctx* c);
#define PM_FORCE 0
#define PM_ENE 1
#define PM_TENS 2
#define PM_FULL 3
// finish = false: the caller launches launch_pair_finish itself (mixed: the
// sorted-slot forces into the accumulator, the pruned-row regrouping)
pgk_status launch_pair(pgk_ctx* c, int group, int vmode, bool finish = true);
pgk_status pair_autotune(pgk_ctx* c);   // at the first list build (outside any capture)
std::string pair_tuning_text();
pgk_status launch_pair_finish(pgk_ctx* c, int group);
pgk_status launch_excl(pgk_ctx* c, int group, bool ene, bool vir);
pgk_status count_pairs(pgk_ctx* c, long long* npair, long long* nentries, long long* nbits = nullptr);

// ---- launchers (k_spme.cu) ----
pgk_status spme_setup(pgk_ctx* c);
pgk_status spme_autotune(pgk_ctx* c);   // FFT launch shapes (after the dynamic state is set)
pgk_status launch_spme(pgk_ctx* c, int group, bool ene, bool vir);

// per-atom split of the SPME reciprocal energy / tensor into c->hfk_out
pgk_status launch_spme_hf_atm(pgk_ctx* c);

// ---- launchers (k_bonded.cu) ----
pgk_status bonded_setup(pgk_ctx* c, HostTerms& t, const std::vector<int>& mol_idx, const std::vector<int>& mol_list);
pgk_status launch_bonded(pgk_ctx* c, int group, bool ene, bool vir, bool force_all);
// tens: only the total bonded virial tensor is wanted (it goes to the bond
// tensor slot; no energies), as in the anisotropic MTK steps without output
pgk_status launch_intra(pgk_ctx* c, int group, int mask, bool want, bool tens = false);

// ---- launchers (k_morse.cu) ----
pgk_status morse_setup(pgk_ctx* c, const pgk_system* s);
pgk_status launch_mklist_mor(pgk_ctx* c);
pgk_status launch_morse(pgk_ctx* c, int group, bool ev);
pgk_status export_morlist(pgk_ctx* c, int32_t* nmorselist, int32_t* mor_index, int32_t* mor_list, int64_t cap,
                          int64_t* nl);

// ---- launchers (k_heatf.cu, heat flux + region Langevin) ----
struct HfDev;
pgk_status hf_setup(pgk_ctx* c, const pgk_hfparams* p);
pgk_status launch_hf_atm(pgk_ctx* c);
pgk_status launch_heatf(pgk_ctx* c, double* dst);
pgk_status launch_lt_regist(pgk_ctx* c);
pgk_status launch_hf_kspace(pgk_ctx* c);           // per-atom reciprocal terms (pgk_set_hf_kspace)
pgk_status launch_ewk_force(pgk_ctx* c, int group); // ewaldkp_hf force in place of SPME (k_ewald.cu)
pgk_status launch_langevin(pgk_ctx* c, double dt, long long step, bool former);
pgk_status launch_bonded_hf(pgk_ctx* c, const HfDev& h);   // k_bonded.cu

// ---- launchers (k_ewald.cu, ewaldkp_hf) ----
// one evaluation at the current positions into c->ewk_out (device); nwave out.
// only = 1 / 2: launch k_ewk_sfac / k_ewk_atom alone on the buffers of the
// last full call with this kmax (instrumentation)
pgk_status launch_ewk_hf(pgk_ctx* c, int kmax, int* nwave, int only = 0);

// ---- launchers (k_integrate.cu) ----
pgk_status launch_zero_group(pgk_ctx* c, int group);
// k_kick_drift flags: KD_LONG long kick, KD_SHORT short kick, KD_SHORT_FIRST
// short kick before the long one (second half step), KD_DRIFT drift, KD_SAVE
// keep the positions before the drift (RATTLE)
#define KD_LONG 1
#define KD_SHORT 2
#define KD_DRIFT 4
#define KD_SAVE 8
#define KD_SHORT_FIRST 16
pgk_status launch_kick_drift(pgk_ctx* c, int flags);
pgk_status launch_chain_coeffs(pgk_ctx* c, int chain_kind, int coef_kind, const pgk_mdparams& md);
pgk_status launch_rattle_pos(pgk_ctx* c, double eps, double dt, bool use_rvinv);
pgk_status launch_rattle_vel(pgk_ctx* c, double eps);
pgk_status launch_kinetic(pgk_ctx* c, int group);
pgk_status launch_kinetic_end(pgk_ctx* c, int mode, int chain_kind, const pgk_mdparams& md);
pgk_status launch_press(pgk_ctx* c);
pgk_status launch_coeffs(pgk_ctx* c, int kind, const pgk_mdparams& md, int phase);
pgk_status launch_box_update(pgk_ctx* c, int kind, const pgk_mdparams& md, bool with_rkcut = false);
pgk_status launch_copy_force(pgk_ctx* c, int group, double* dst_dev);
pgk_status launch_out_record(pgk_ctx* c, long long step, double* dst);
