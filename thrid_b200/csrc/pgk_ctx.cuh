// pgk_ctx.cuh -- the engine context (host view of all device buffers) and
// the launchers each kernel file exports.
#pragma once

#include <cuda_runtime.h>
#include <map>
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

struct pgk_ctx {
    int natom = 0;
    int prec = PGK_PREC_FP64;
    bool mixed() const { return prec == PGK_PREC_MIXED; }
    pgk_params prm{};
    cudaStream_t st = nullptr;
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

    // ---- constraints ----
    int ncgroup = 0, nconstraint = 0;
    int *cg_idx = nullptr, *cg_list = nullptr;
    int2* c_ij = nullptr; double* c_d = nullptr;

    // ---- pair list ----
    int maxcells = 0;
    int *cell_of = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
    int* perm = nullptr;          // sorted -> original
    int* iperm = nullptr;         // original -> sorted
    double* pos_s = nullptr;      // sorted FP64 positions at list time (3N)
    int* nbr = nullptr;           // [N*cap]
    int* ncnt = nullptr;          // [N]
    int cap = 0;
    int4* xq = nullptr;           // mixed: fixed-point fractional coords + q bits
    double4* xq64 = nullptr;      // fp64: x,y,z,q sorted
    int* typ_s = nullptr;
    unsigned long long* counters = nullptr;   // [0] nlistnball, [1] max row
    bool list_valid = false;

    // ---- SPME ----
    int K[3] = {0, 0, 0};
    int order = 0;
    void* qacc = nullptr;         // accumulation grid (int64 fixed / double)
    void* qc = nullptr;           // complex grid (float2 / double2)
    double* bsp = nullptr;        // bsp_mod1|2|3
    FftPlan plan[3];

    // ---- CUDA graphs ----
    std::map<long long, cudaGraphExec_t> graphs;
    bool use_graphs = true;

    // ---- scratch for host transfers ----
    std::vector<double> hbuf;
};

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
pgk_status launch_pair(pgk_ctx* c, int group, bool ene, bool vir);
pgk_status launch_excl(pgk_ctx* c, int group, bool ene, bool vir);
pgk_status count_pairs(pgk_ctx* c, long long* npair, long long* nentries);

// ---- launchers (k_spme.cu) ----
pgk_status spme_setup(pgk_ctx* c);
pgk_status launch_spme(pgk_ctx* c, int group, bool ene, bool vir);

// ---- launchers (k_bonded.cu) ----
pgk_status launch_bonded(pgk_ctx* c, int group, bool ene, bool vir, bool force_all);

// ---- launchers (k_integrate.cu) ----
pgk_status launch_zero_group(pgk_ctx* c, int group);
pgk_status launch_kick_long(pgk_ctx* c);
pgk_status launch_kick_short(pgk_ctx* c);
pgk_status launch_drift(pgk_ctx* c, bool save_old);
pgk_status launch_rattle_pos(pgk_ctx* c, double eps, double dt, bool use_rvinv);
pgk_status launch_rattle_vel(pgk_ctx* c, double eps);
pgk_status launch_kinetic(pgk_ctx* c, int group);
pgk_status launch_chain(pgk_ctx* c, int kind, const pgk_mdparams& md);
pgk_status launch_press(pgk_ctx* c);
pgk_status launch_coeffs(pgk_ctx* c, int kind, const pgk_mdparams& md, int phase);
pgk_status launch_box_update(pgk_ctx* c, int kind, const pgk_mdparams& md);
pgk_status launch_copy_force(pgk_ctx* c, int group, double* dst_dev);
