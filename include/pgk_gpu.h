/*
 * pgk_gpu.h -- C ABI of libpgkgpu.so, the B200 (sm_100a) force-and-integration
 * engine for the peachgk_md molecular-dynamics driver.
 *
 * The reference program keeps all state in Fortran module globals
 * (md_global.inc) and calls subroutines with explicit interfaces
 * (interface_interact.F90, interface_mdtech.F90, interface_mddriver.F90).
 * This header exposes the same operations as plain C functions taking plain
 * pointers and sizes.  Every array follows the reference layout:
 *   - coordinates / velocities / forces: (3,natom) Fortran column-major, i.e.
 *     x,y,z interleaved per atom, FP64, reduced units (calbase.F90:21-40);
 *   - atom indices: 1-based, exactly as stored in the Fortran arrays;
 *   - CSR lists: 1-based start indices with the reference's 0 sentinel for an
 *     empty row (mkexcl.F90, mklist_cell.F90:297-329).
 * The library owns device mirrors of the state.  Between downloads the device
 * copy is authoritative.  Every entry point returns a pgk_status (0 = OK); the
 * reference STOPs on the same conditions.
 *
 * One context is driven from one host thread; it uses one CUDA stream.
 */
#ifndef PGK_GPU_H
#define PGK_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque engine context: device mirrors of the md_global state. */
typedef struct pgk_ctx pgk_ctx;

/* ---- status codes (each replaces a STOP of the reference) ---------------- */
typedef int32_t pgk_status;
#define PGK_OK                 0
#define PGK_E_LIST_OVERFLOW    1  /* mklist_cell.F90:342-346 "nlistnball exceed" */
#define PGK_E_CELL_OVERFLOW    2  /* mklist_cell.F90:121-145,170-176 */
#define PGK_E_RATTLE_NOCONV    3  /* rattle.F90 "RATTLE(C) failed to converge" */
#define PGK_E_BOX_TOO_SMALL    4  /* calvol.F90 / calbox.F90 "rcut is over half cell" */
#define PGK_E_DEVICE_TIMEOUT   5  /* a bounded device wait gave up */
#define PGK_E_CUDA             6  /* a CUDA runtime call failed */
#define PGK_E_INVALID          7  /* bad argument (null pointer, size, unsupported option) */
#define PGK_E_NOMEM            8  /* device allocation failed */
#define PGK_E_UNSUPPORTED      9  /* option of the reference that this engine does not build */
#define PGK_E_RATTLEV_NOCONV  10  /* rattle_mtk.F90 "RATTLE(V) failed to converge" */
#define PGK_E_SCRATCH_LIMIT   11  /* size beyond the static scratch of pgk_fft_pme_noalloc */

/* ---- option values ------------------------------------------------------- */
#define PGK_PREC_FP64   0   /* all-FP64 device path (parity path) */
#define PGK_PREC_MIXED  1   /* FP32 pair/SPME/bonded arithmetic, int64 fixed-point sums */

#define PGK_MTS_LONG    1   /* md_global.inc:130 MTS_LONG */
#define PGK_MTS_SHORT   3   /* md_global.inc:132 MTS_SHORT */
#define PGK_MTS_NONE    0   /* term switched off (commented-out mts_* keyword) */

#define PGK_PCONT_ISO    0  /* pcont_axis 'iso'   (nhcpisoint.F90)            */
#define PGK_PCONT_ANISO  1  /* pcont_axis 'aniso' (nhcpanisoint.F90, dir 0)   */
#define PGK_PCONT_X      2  /* pcont_axis 'x'     (nhcpanisoint.F90, dir 1)   */
#define PGK_PCONT_Y      3
#define PGK_PCONT_Z      4

#define PGK_LIST_AUTO    0  /* ifcellindex with the rdscript.F90:1595-1610 fallback */
#define PGK_LIST_CELL    1  /* force mklist_cell order */
#define PGK_LIST_ALLPAIR 2  /* force mklist2a order   */

/* ---- system description (topology + parameters), read once at pgk_init --
 * Per-term parameters are already expanded from the reference's type tables
 * (e.g. para_cbond(indexbondtyp(k)) -> para_cbond[k-1]).  Angles/phases are
 * in radians (prepmd.F90:230-237 converts degrees); charges are already
 * multiplied by 1/sqrt(4 pi eps0) (prepmd.F90:239-241). */
typedef struct pgk_system {
    int32_t natom;
    const double*  atmmass;       /* [natom]                                  */
    const double*  atmchrg;       /* [natom]                                  */
    const int32_t* atmindex;      /* [natom] 1-based LJ type                  */
    int32_t        ntyp;
    const double*  vdw_radij;     /* [ntyp*ntyp] column-major (i,j): R_min,ij  */
    const double*  vdw_welij;     /* [ntyp*ntyp] well depth E_ij              */
    const int32_t* inter_inttyp;  /* [ntyp*ntyp] 1 = INTTYPE_VDW (LJ), 2 = INTTYPE_MOR (no LJ;
                                     Morse when switched on); 3..10 (SH, RFH, DOU, RP-VW,
                                     custom) return PGK_E_UNSUPPORTED; NULL = all LJ */

    int32_t        nmole;         /* molecules (transcor.F90, calpress.F90)    */
    const int32_t* molept_index;  /* [nmole+1], 1-based                        */
    const int32_t* molept_list;   /* [molept_index[nmole]-1], 1-based atoms    */

    const int32_t* index_excl;    /* [natom+1] mkexcl.F90 output (j>i, 0 sentinel) */
    const int32_t* list_excl;

    int32_t nbond;                /* calbond.F90 */
    const int32_t *ibond, *jbond;
    const double  *para_cbond, *para_eqbond;

    int32_t nangl;                /* calangl.F90 */
    const int32_t *iangl, *jangl, *kangl;
    const double  *para_cangl, *para_eqangl;

    int32_t ntors;                /* caltors.F90 + 1-4 flags of calnon14.F90 */
    const int32_t *itors, *jtors, *ktors, *ltors;
    const int32_t *para_divfac;
    const double  *para_barhig, *para_phsang, *para_period;
    const int32_t *ifcalnonb14;   /* may be NULL: no 1-4 from periodic torsions */
    const double  *para_divfac_vdw, *para_divfac_elc, *ring14;

    int32_t ntorsrb;              /* caltorsrb.F90 */
    const int32_t *itorsrb, *jtorsrb, *ktorsrb, *ltorsrb;
    const double  *para_barhigrb; /* [6*ntorsrb], C0..C5 per term             */
    const int32_t *ifcalnonb14_rb;
    const double  *para_divfac_vdwrb, *para_divfac_elcrb, *ring14_rb;

    int32_t nconst;               /* constraint groups (rattle.F90 DOconstr)   */
    const int32_t* index_mconst;  /* [nconst+1], 1-based                        */
    const int32_t* list_mconst;   /* 1-based constraint ids                     */
    int32_t nconstraint;
    const int32_t *iconst, *jconst;
    const double  *dconst;

    int32_t degfree_all;          /* prepmd.F90:250-330                          */

    /* Morse pairs (morse.F90, rdpara.F90:680-720): type pairs whose
     * inter_inttyp is 2 (INTTYPE_MOR, md_global.inc:120) interact by
     * D (exp(-2a(r-r0)) - 2 exp(-a(r-r0))) instead of LJ.  [ntyp*ntyp]
     * column-major like vdw_radij; NULL = no Morse pairs.  The device engine
     * does not build Morse yet: pgk_init returns PGK_E_UNSUPPORTED when a
     * Morse pair type is present and mts_mor is not PGK_MTS_NONE (the oracle
     * restates it); with mts_mor = PGK_MTS_NONE Morse is switched off, as in
     * the reference, and those pairs carry neither Morse nor LJ. */
    const double  *para_welmor, *para_radmor, *para_alphamor;
} pgk_system;

/* ---- run-time parameters (peachgk.ini keywords after calbase) ----------- */
typedef struct pgk_params {
    double  xcel, ycel, zcel;     /* initial box                               */
    double  alpha;                /* Ewald alpha [1/length]                    */
    double  rrcut;                /* Ewald real-space cutoff                   */
    double  rcut;                 /* LJ cutoff                                 */
    double  rcut_book;            /* bookkeeping radius                        */
    int32_t nstep_book;           /* list renewal interval                     */
    int32_t list_mode;            /* PGK_LIST_*                                */
    int32_t ifspme;               /* 1: SPME reciprocal space                  */
    int32_t nfft1, nfft2, nfft3, pme_order;
    int32_t nspltbl;              /* erfc spline table points (spline_interp.F90) */
    int32_t precision;            /* PGK_PREC_*                                */
    int32_t mts_bond, mts_angl, mts_tors, mts_torsrb;
    int32_t mts_vdw;              /* gates ewaldr (LJ + real-space Ewald)      */
    int32_t mts_ewk;              /* gates fft_pme                             */
    int32_t mts_vdw14, mts_elc14; /* calnon14 runs when both equal the flag    */
    int32_t ifnetqcorrp;          /* net-charge correction for pressure        */
    int32_t max_nbr;              /* entries per 8-atom cluster row of the device pair list (0 = auto) */
    double  rcutmor;              /* Morse cutoff                              */
    double  rcut_bookmor;         /* Morse list radius (mklist_mor*.F90); <= 0: every Morse
                                     pair within half the box diagonal (ifbookmor off) */
    int32_t mts_mor;              /* gates morsep (PGK_MTS_*)                   */
    int32_t nstep_bookmor;        /* Morse list rebuild interval of the stage drivers
                                     (moldyn*.F90; 0 = nstep_book)              */
} pgk_params;

/* ---- integrator parameters (moldyn_*.F90 arguments) ---------------------- */
typedef struct pgk_mdparams {
    double  dt_long_cal;          /* reduced time step                         */
    int32_t nstep_short;          /* XO-RESPA inner steps                      */
    int32_t mchain;               /* NHC length (<= 8)                         */
    double  text;                 /* reduced target temperature                */
    double  qmass[8];             /* prepmd.F90:515-518                        */
    double  vmass;                /* prepmd.F90:521-525                        */
    int32_t next, nyosh;          /* Trotter sub-steps, Yoshida-Suzuki order   */
    double  yscoeff[8];           /* prepmd.F90:535-547                        */
    double  pext;                 /* reduced external pressure                 */
    int32_t pcont_axis;           /* PGK_PCONT_*                               */
    int32_t ifrattle;
    double  eps_rattle;
    int32_t pressinterval;        /* calpress cadence in NVT (MTK: every step) */
    int32_t outinterval;          /* energies are evaluated on these steps     */
} pgk_mdparams;

/* ---- energies (calforce.F90 OUTPUT names) ------------------------------- */
typedef struct pgk_energies {
    double pot_tot, pot_nonbon;
    double pot_vdw, pot_elc, pot_ewk, pot_ewc, pot_ewnq;
    double pot_vdw14, pot_elc14;
    double pot_bond, pot_angl, pot_tors, pot_torsrb;
    double pot_mor;               /* Morse energy (in pot_tot, not pot_nonbon; calforce.F90:1060-1070) */
} pgk_energies;

/* ---- virials (ewaldrp / fft_pmep / cal*p OUTPUT names), tensors (3,3)
 *      column-major: t[a + 3*b] = sum f_a * r_b. ---------------------------- */
typedef struct pgk_virials {
    double pot_viri_coul, pot_viri_lj;
    double pot_virit_coul[9], pot_virit_lj[9];
    double atm_viri_bond, atm_viri_angl, atm_viri_tors, atm_viri_14;
    double atm_virit_bond[9], atm_virit_angl[9], atm_virit_tors[9], atm_virit_14[9];
    double pot_viri_mor, pot_virit_mor[9];   /* morsep */
} pgk_virials;

/* ---- thermostat / barostat state (md_global.inc xlogs, vlogs, ...) ------- */
typedef struct pgk_chain {
    double xlogs[8], vlogs[8];
    double xlogv, vlogv;
    double xboxh[3], vboxg[3];
    double pint, pintt[9];
} pgk_chain;

/* ---- heat flux and region Langevin thermostat ----------------------------
 * moldyn_hf.F90 (NVE-RESPA driver of the -DHF build), calforce_hf.F90,
 * ewaldr_hf.F90, cal{bond,angl,tors,torsrb,non14}_hf.F90, calvirihf.F90,
 * calheatf.F90, calcom.F90, langevin_regist.F90, langevin_region.F90.
 * Built: the local volume-based Irving-Kirkpatrick flux (ifhfvol), z
 * direction only (the default build: no _HF_ALL_DIR / _HF_BULK), bare 1/r
 * Coulomb in the pair virial (the default of ewaldr_hf.F90:336), atom- or
 * molecule-based positions per atom (hftyp_atm), streaming velocity zero. */
#define PGK_HF_MAX_REGIONS  32
#define PGK_LT_MAX_REGIONS   8
#define PGK_HFTYP_ATOM       1   /* md_global.F90:112 HFTYP_ATOM */
#define PGK_HFTYP_MOLE       2   /* md_global.F90:113 HFTYP_MOLE */
#define PGK_HF_NCOL         18   /* values per region in a heat-flux record */
/* Per-atom categories of calheatf (pot_*_atm / viri*_atm arrays). */
#define PGK_HF_BO    0   /* bonds            pot_bo_atm,   viribot_atm   */
#define PGK_HF_AN    1   /* angles           pot_an_atm,   viriant_atm   */
#define PGK_HF_TO    2   /* torsions (+ RB)  pot_to_atm,   viritot_atm   */
#define PGK_HF_14    3   /* 1-4 pairs        pot_14_atm,   viri14t_atm   */
#define PGK_HF_ELIN  4   /* intramolecular Coulomb  pot_elin_atm, virielint_atm */
#define PGK_HF_LJIN  5   /* intramolecular LJ       pot_ljin_atm, viriljint_atm */
#define PGK_HF_ELC   6   /* intermolecular Coulomb  pot_elc_atm,  virielct_atm  */
#define PGK_HF_VDW   7   /* intermolecular LJ       pot_vdw_atm,  viriljt_atm   */
/* A heat-flux record holds, for each region r, PGK_HF_NCOL z components in
 * the order of calheatf.F90's output arrays, each divided by the region
 * volume (calheatf.F90:1330-1460):
 *   [r*18 + 0]      hfkin_atm(3,r)
 *   [r*18 + 1..8]   hfpot{bo,an,to,14,elin,ljin,elc,lj}_atm(3,r)
 *   [r*18 + 9..16]  hfviri{bo,an,to,14,elin,ljin,elc,lj}_atm(3,r)
 *   [r*18 + 17]     hftot_atm(3,r) */
typedef struct pgk_hfparams {
    int32_t nhfregion;            /* heat-flux z slabs (<= PGK_HF_MAX_REGIONS)  */
    int32_t ifhfvol;              /* must be 1: local volume-based method       */
    int32_t heatfinterval;        /* flux on steps with mod(step, n) == 1, or n == 1 */
    int32_t nlangeregion;         /* Langevin regions (<= 8); 0 = no thermostat */
    double  hfzpos1[PGK_HF_MAX_REGIONS], hfzpos2[PGK_HF_MAX_REGIONS];
    const int32_t* hftyp_atm;     /* [natom] PGK_HFTYP_*; NULL = all atom-based */
    const int32_t* lt_mole_based; /* [nmole] 1: register the molecule by its centre of
                                     mass (water, and poly without iftcratom); 0: per
                                     atom (langevin_regist.F90:86-360); NULL = all 0 */
    double  ltxpos1[PGK_LT_MAX_REGIONS], ltxpos2[PGK_LT_MAX_REGIONS];
    double  ltypos1[PGK_LT_MAX_REGIONS], ltypos2[PGK_LT_MAX_REGIONS];
    double  ltzpos1[PGK_LT_MAX_REGIONS], ltzpos2[PGK_LT_MAX_REGIONS];
    double  r_ltemp[PGK_LT_MAX_REGIONS];   /* reduced temperature (T / tempref)     */
    double  r_ltdamp[PGK_LT_MAX_REGIONS];  /* reduced damping rate (gamma * timeref) */
    uint64_t seed;                /* key of the counter-based random stream     */
    int32_t ifoutthc;             /* tally det_ene_kin per Langevin region      */
    int32_t _pad;
} pgk_hfparams;

/* ---- lifetime ------------------------------------------------------------ */
/* Library version string. */
const char* pgk_version(void);
/* Human-readable text of a status code (the reference's STOP message). */
const char* pgk_status_string(pgk_status s);

/* Build a context: copies the topology and parameters to the device, builds
 * the erfc spline tables (spline_interp_init, spline_interp.F90:14-136), the
 * B-spline moduli and self energy (fft_pme_init, fft_pme_init.F90:14-180) and
 * the Ewald k-cutoff (erf_corr_cutoff.F90:28-62).  Replaces the L3
 * pre-processing calls main_md.F90:1101-1185 for the device side. */
pgk_status pgk_init(const pgk_system* sys, const pgk_params* prm, pgk_ctx** out);
pgk_status pgk_free(pgk_ctx* ctx);
/* Last error message recorded on this context (empty if none). */
const char* pgk_last_error(const pgk_ctx* ctx);

/* ---- state transfer (host module arrays <-> device mirrors) -------------- */
/* atmcor/atmvel: (3,natom); box: xcel,ycel,zcel.  atmvel may be NULL. */
pgk_status pgk_upload_state(pgk_ctx* ctx, const double* atmcor, const double* atmvel,
                            const double* box);
pgk_status pgk_download_state(pgk_ctx* ctx, double* atmcor, double* atmvel, double* box);
pgk_status pgk_set_chain(pgk_ctx* ctx, const pgk_chain* ch);
pgk_status pgk_get_chain(pgk_ctx* ctx, pgk_chain* ch);

/* ---- fine-grained operations with the reference's names ----------------- */
/* transcor.F90: wrap each molecule by its first atom into [0,L). */
pgk_status pgk_transcor(pgk_ctx* ctx);

/* mklist_cell.F90:8-352 / mklist2a (mklist.F90:8-234) with the
 * rdscript.F90:1595-1610 fallback: builds the bookkeeping pair list on the
 * device.  *nlistnball receives the reference's nlistnball (entries incl.
 * the 0 sentinels of empty rows). */
pgk_status pgk_mklist_cell(pgk_ctx* ctx, int64_t* nlistnball);

/* Copy the last list out in the reference CSR layout: nb_indexall[natom]
 * (1-based start of row i; the entry after the last row holds
 * nlistnball+1) and nb_listall[nlistnball] (1-based j, 0 sentinel),
 * rows in the reference order (cell scan order for mklist_cell, ascending j
 * for mklist2a).  cap = capacity of nb_listall. */
pgk_status pgk_get_nblist(pgk_ctx* ctx, int32_t* nb_indexall, int32_t* nb_listall,
                          int64_t cap, int64_t* nlistnball);

/* calforce.F90:8-1073 for one MTS group (PGK_MTS_LONG / PGK_MTS_SHORT):
 * force (3,natom) is OVERWRITTEN with the group's force (not acceleration);
 * ene / vir may be NULL.  want_virial selects the *p (virial) variants. */
pgk_status pgk_calforce(pgk_ctx* ctx, int32_t mts_flag, double* force,
                        pgk_energies* ene, pgk_virials* vir);

/* Single-kernel entries used by the parity tests (force += into `force`): */
/* ewaldrp (ewaldr.F90:404-838) incl. the excluded-pair erf correction. */
pgk_status pgk_ewaldr(pgk_ctx* ctx, double* force, pgk_energies* ene, pgk_virials* vir);
/* fft_pmep (fft_pme.F90:144-270): SPME reciprocal force, pot_ewk, tensor. */
pgk_status pgk_fft_pme(pgk_ctx* ctx, double* force, pgk_energies* ene, pgk_virials* vir);
/* calbondp/calanglp/caltorsp/caltorsrbp/calnon14p (all terms, no MTS gate). */
pgk_status pgk_calbonded(pgk_ctx* ctx, double* force, pgk_energies* ene, pgk_virials* vir);
/* morsep (morse.F90:206-414): Morse force over the Morse list, pot_mor,
 * pot_viri_mor, pot_virit_mor (no MTS gate; builds the Morse list if none). */
pgk_status pgk_morsep(pgk_ctx* ctx, double* force, pgk_energies* ene, pgk_virials* vir);

/* ---- Morse pair list (its own list, as in the reference) ------------------
 * Morse atoms (nmorselist, linkbond.F90) are the atoms of a type that has a
 * Morse partner type (inter_inttyp == 2); with mts_mor = PGK_MTS_NONE the
 * engine holds no Morse list.  mklist_mor_cell (mklist_mor_cell.F90:8-327,
 * 27-cell scan) or mklist2a_mor (mklist_mor.F90: all later Morse atoms) by
 * the rule of rdscript.F90:1616-1632 (cells of rcut_bookmor, fewer than 3 per
 * direction or at most 27 in all -> mklist2a_mor; list_mode forces either).
 * *nlistmorall receives the reference's count (0 sentinels included). */
pgk_status pgk_mklist_mor_cell(pgk_ctx* ctx, int64_t* nlistmorall);
/* The last Morse list in the reference layout: nmorselist[nmorse] (1-based
 * atoms), mor_indexall[nmorse] (1-based start of row mor1 = 1..nmorse-1;
 * entry nmorse holds nlistmorall+1), mor_listall[nlistmorall] (1-based j, a 0
 * for an empty row).  Any array may be NULL; cap = capacity of mor_listall. */
pgk_status pgk_get_morlist(pgk_ctx* ctx, int32_t* nmorselist, int32_t* mor_indexall, int32_t* mor_listall,
                           int64_t cap, int64_t* nlistmorall, int32_t* nmorse);

/* rattle_c (rattle.F90:6-272) on the device state, given atmcor_old (3,natom)
 * on the host (copied in).  dt_short = time step used for the correction. */
pgk_status pgk_rattle_c(pgk_ctx* ctx, const double* atmcor_old, double eps_rattle,
                        double dt_short_cal);
/* rattlep_v (rattle_mtk.F90:278-542) on the device velocities. */
pgk_status pgk_rattlep_v(pgk_ctx* ctx, double eps_rattle);

/* ---- stage drivers: the whole XO-RESPA loop stays on the device ---------- */
/* moldyn.F90 NVE (no thermostat), moldyn_nhc.F90 NVT-NHC and moldyn_mtk.F90
 * NPT-MTK, steps inistep..endstep inclusive (step 0 = initial force only).
 * `ene` receives the energies of the last step whose index is a multiple of
 * md->outinterval (or of endstep when outinterval <= 0); may be NULL. */
pgk_status pgk_moldyn_nve(pgk_ctx* ctx, int64_t inistep, int64_t endstep,
                          const pgk_mdparams* md, pgk_energies* ene);
pgk_status pgk_moldyn_nhc(pgk_ctx* ctx, int64_t inistep, int64_t endstep,
                          const pgk_mdparams* md, pgk_energies* ene);
pgk_status pgk_moldyn_mtk(pgk_ctx* ctx, int64_t inistep, int64_t endstep,
                          const pgk_mdparams* md, pgk_energies* ene);

/* Heat-flux regions, their atom/molecule typing and the region Langevin
 * thermostat (preheatf.F90, rdlangevin.F90 settings); replaces any earlier
 * setting.  Atom registration for the thermostat happens here once
 * (langevin_regist at current_step 0 of moldyn_hf.F90:1425-1440). */
pgk_status pgk_set_hf(pgk_ctx* ctx, const pgk_hfparams* hf);

/* moldyn_hf.F90:1405-2480: NVE XO-RESPA with the region Langevin half steps
 * (langevin_region former half before the RESPA loop, re-registration and
 * latter half after it) and, on heat-flux steps (mod(step, heatfinterval) == 1
 * or heatfinterval == 1, step > 0), calforce_hf + calheatf.  Each heat-flux
 * step appends one record of nhfregion * PGK_HF_NCOL doubles to hf_out (at
 * most cap_records; *nrecords returns the count, which may exceed the
 * capacity).  hf_out may be NULL. */
pgk_status pgk_moldyn_hf(pgk_ctx* ctx, int64_t inistep, int64_t endstep, const pgk_mdparams* md,
                         pgk_energies* ene, double* hf_out, int64_t cap_records, int64_t* nrecords);

/* calcom + the per-atom heat-flux quantities of calforce_hf (ewaldrp_hf and
 * the *_hf bonded routines, calvirihf) at the current positions, then
 * calheatf with the current velocities: one record of nhfregion * 18. */
pgk_status pgk_calheatf(pgk_ctx* ctx, double* hf);

/* Per-atom arrays of the last heat-flux evaluation: pot_atm[c*natom + i]
 * (category c = PGK_HF_*, both MTS groups summed) and the z column of the
 * per-atom virial, viri_atm[((c*nhfregion + r)*3 + a)*natom + i] =
 * viri*_atm(a,3,i,r).  Either pointer may be NULL. */
pgk_status pgk_get_hf_atm(pgk_ctx* ctx, double* pot_atm, double* viri_atm);

/* ewaldkp_hf (ewaldk_hf.F90:8-304): the standard-Ewald k-space force, energy
 * and virial with their per-atom split, which the -D_HF_BULK_EWK build runs
 * in place of the reciprocal term on heat-flux steps (calforce_hf.F90:1046-1067),
 * at the context's current positions and box.  Wave vectors as prepewk /
 * upewk (prepewk.F90:100-155): integer (nx,ny,nz) != 0 with |nx| <= kmax,
 * |ny| <= kmax*ny0, |nz| <= kmax*nz0 and nx^2 + ny^2/ny0^2 + nz^2/nz0^2 <=
 * kmax^2, where ny0, nz0 = anint(ycel/xcel), anint(zcel/xcel) of the
 * context's initial box (rdscript.F90:1494); K = (nx/xcel, ny/ycel, nz/zcel)
 * at the current box.  alpha, ifnetqcorrp and (sum q)^2 come from the context.
 * The host arrays receive this term alone (the reference's in/out arrays add
 * it); each may be NULL:
 *   force        (3,natom)   2 q_i / V * sum_k A(K) (bck sin_i - bsk cos_i) K,
 *                            added by the reference to force and for_viri_coul;
 *   pot_elc_atm  (natom)     per-atom energy, with the self term
 *                            -alpha/sqrt(pi) q_i^2 (ewaldk_hf.F90:295-299);
 *   virielct_atm (3,3,natom) per-atom virial tensor, [a + 3*b + 9*i] (the
 *                            reference's region-1 slice virielct_atm(:,:,i,1)).
 * With ifnetqcorrp every atom's tensor carries -pot_fact*A(K)*netchrgsq per
 * wave (ewaldk_hf.F90:257-272), so the atom tensors then do not sum to the
 * total tensor.  kmax >= 1; ny0, nz0 >= 1; at most 253 table rows
 * (kmax*(1 + ny0 + nz0) <= 250). */
typedef struct pgk_ewk_hf {
    double  pot_ewk;              /* k-space energy                            */
    double  pot_ewk_cc;           /* net-charge correction (0 without ifnetqcorrp);
                                     pot_viri_coul += pot_ewk + pot_ewk_cc      */
    double  pot_virit_coul[9];    /* k-space virial tensor t[a + 3*b]           */
    int32_t nwave;                /* wave vectors, (0,0,0) included (nwave of prepewk) */
    int32_t _pad;
} pgk_ewk_hf;
pgk_status pgk_ewaldkp_hf(pgk_ctx* ctx, int32_t kmax, double* force, double* pot_elc_atm,
                          double* virielct_atm, pgk_ewk_hf* out);

/* Per-atom reciprocal term of the bulk heat flux.  PGK_HF_KSPACE_NONE (the
 * default, as the reference's default heat-flux build: the reciprocal term is
 * not split per atom); PGK_HF_KSPACE_EWK: the -D_HF_BULK_EWK build
 * (calforce_hf.F90:1046-1062) -- on heat-flux steps ewaldkp_hf with waves up
 * to kmax replaces the SPME term (force, pot_ewk, virial) and adds its
 * per-atom energy and virial; PGK_HF_KSPACE_SPME: the SPME force stays and
 * the per-atom split of the SPME term (pgk_fft_pme_hf) is added.  Either way
 * the energy goes to each atom's pot_elc_atm and the (a, z) column of the
 * tensor to region 1 of virielct_atm (ewaldk_hf.F90:212-230 writes region 1). */
#define PGK_HF_KSPACE_NONE 0
#define PGK_HF_KSPACE_EWK  1
#define PGK_HF_KSPACE_SPME 2
pgk_status pgk_set_hf_kspace(pgk_ctx* ctx, int32_t mode, int32_t kmax);

/* Per-atom split of fft_pmep's reciprocal energy and virial tensor: the SPME
 * form of ewaldkp_hf's per-atom terms (ewaldk_hf.F90:165-230, which the
 * reference has only for standard Ewald).  With S = FFT(Q) and scalar_sum's
 * influence function eterm: pot_atm[i] = 1/2 q_i sum_g theta_i(g)
 * IFFT(eterm S)(g) - alpha/sqrt(pi) q_i^2; viri_atm[9i + a + 3b] = 1/2 q_i
 * sum_g theta_i(g) IFFT(eterm (delta_ab - vterm h_a h_b) S)(g).  The energies
 * less the self terms sum to pot_ewk and the tensors to pot_virit_coul (the
 * net-charge terms are global and not split).  FP64 in both precisions. */
pgk_status pgk_fft_pme_hf(pgk_ctx* ctx, double* pot_atm, double* viri_atm);

/* det_ene_kin of langevin_region.F90 (kinetic energy put in (+) or taken out
 * (-) per Langevin region) summed since the last call, then reset. */
pgk_status pgk_langevin_dekin(pgk_ctx* ctx, double* det_ene_kin);

/* ---- device-side output records (outene / outpre of output_data.F90) ----
 * With a capacity set, every output step of the stage drivers (outinterval)
 * appends one record to a device buffer instead of reading the accumulators
 * back (no host synchronisation per output step); pgk_get_output copies the
 * records out and clears the buffer.  Record layout (PGK_OUT_NCOL doubles):
 *   [0] step, [1..14] the 14 pgk_energies fields in struct order (pot_tot
 *   .. pot_mor), [15] sum(m v^2), [16] pint, [17..25] pintt (column-major),
 *   [26..28] box.
 * pint/pintt are the barostat's values (moldyn_mtk); other drivers leave the
 * last ones set.  Records beyond the capacity are counted but not kept. */
#define PGK_OUT_NCOL 29
pgk_status pgk_set_output(pgk_ctx* ctx, int64_t cap_records);
pgk_status pgk_get_output(pgk_ctx* ctx, double* out, int64_t cap_records, int64_t* nrecords);

/* Kinetic energy sum(m v^2) and atomic pressure tensor (calpress.F90, atomic
 * branch) of the current device state; press9 may be NULL. */
pgk_status pgk_calpress(pgk_ctx* ctx, double* kint, double* pressatm_tot, double* press9);

/* Wait for the context's stream; returns the first sticky device error. */
pgk_status pgk_sync(pgk_ctx* ctx);

/* Number of kernels this context has launched so far (for launch accounting). */
int64_t pgk_kernel_launches(const pgk_ctx* ctx);

/* CUDA stream of the context (cudaStream_t as void*), for callers that time
 * the context's kernels with their own events.  A force evaluation also uses
 * a second, internal stream (the SPME chain and bonded terms run beside the
 * pair kernel); its work is always joined back to this stream, so events and
 * synchronisation on this stream cover everything the context launched. */
void* pgk_stream(const pgk_ctx* ctx);

/* Instrumentation (no reference counterpart): launch one kernel of the force
 * path `iters` times back to back on the context's stream, bracketed by CUDA
 * events, and return the mean device time per launch in *ms.  which:
 *   0 = real-space pair kernel (ewaldrp) with virials, 1 = SPME spread,
 *   2 = SPME gather, 3 = one forward 3-D FFT (three axis passes),
 *   4 = one pair-list build (mklist_cell / mklist2a, every kernel of it),
 *   5 = one long kick + drift pass (moves the atoms: time it last),
 *   64 + m = the bonded terms with term mask m (bit 0 bonds, 1 angles,
 *   2 torsions, 3 RB torsions, 4 1-4 pairs, 5 excluded pairs) with energies
 *   and per-type virials, 128 + m = the same with only the total virial
 *   tensor (the anisotropic MTK step without output), 256 + kmax = one
 *   ewaldkp_hf evaluation (the whole kernel chain), 512 + kmax / 768 + kmax
 *   = its structure-factor / per-atom kernel alone (kmax < 256).
 * *units receives the algorithmic work of one launch: unique pairs inside
 * the cutoff (0), atoms (1, 2, 4, 5, 64+, 128+), grid points (3), or (atom, wave)
 * pairs without (0,0,0) (256+); *entries the number
 * of (cluster, j) list entries the pair kernel reads. */
pgk_status pgk_bench_kernel(pgk_ctx* ctx, int32_t which, int32_t iters, double* ms, double* units,
                            double* entries);

/* ---- replica server (continuous batching) --------------------------------
 * No counterpart in the reference, which runs one system per process.
 * Independent replicas (different sizes and topologies) are queued with
 * pgk_server_submit and admitted while earlier ones run, in arrival order,
 * as worker slots and the device-memory budget allow (pgk_estimate_bytes;
 * a request larger than the whole budget runs alone).  Each admitted replica
 * keeps its state resident in its own context and non-blocking CUDA stream;
 * one host worker per slot runs it (captured step graphs), so the replicas'
 * kernels overlap on the device.  In mixed precision a replica's results are
 * bit-identical to a run of it alone (integer force sums, private buffers).
 * The server copies every input at submit. */
typedef struct pgk_server pgk_server;
typedef struct pgk_request {
    const pgk_system*   sys;
    const pgk_params*   prm;
    const pgk_mdparams* md;
    int32_t kind;                 /* 0 moldyn (NVE), 1 moldyn_nhc, 2 moldyn_mtk, 3 moldyn_hf */
    int32_t _pad;
    const pgk_hfparams* hf;       /* required for kind 3, else may be NULL    */
    const double* atmcor;         /* (3,natom) initial coordinates            */
    const double* atmvel;         /* (3,natom) initial velocities, NULL = 0   */
    const double* box;            /* NULL = (xcel, ycel, zcel) of prm         */
    const pgk_chain* chain;       /* NULL = zero chain                        */
    int64_t nsteps;               /* runs steps 0 .. nsteps                   */
} pgk_request;

/* Device bytes one context of this system needs (estimate with margin). */
int64_t pgk_estimate_bytes(const pgk_system* sys, const pgk_params* prm);
/* max_slots worker slots on the current device; budget <= 0 = 80 % of free memory. */
pgk_status pgk_server_create(int32_t max_slots, int64_t hbm_budget_bytes, pgk_server** out);
pgk_status pgk_server_submit(pgk_server* sv, const pgk_request* req, int64_t* id);
pgk_status pgk_server_poll(pgk_server* sv, int64_t id, int32_t* done);
pgk_status pgk_server_wait(pgk_server* sv, int64_t id);
/* Final state, last energies, heat-flux records (kind 3) and the request's
 * submit / start / finish times in seconds (steady clock) in times3. */
pgk_status pgk_server_result(pgk_server* sv, int64_t id, double* atmcor, double* atmvel, double* box,
                             pgk_energies* ene, double* hf_out, int64_t cap_records, int64_t* nrecords,
                             double* times3);
/* Error text of a failed request ("" when it succeeded). */
const char* pgk_server_error(pgk_server* sv, int64_t id);
pgk_status pgk_server_release(pgk_server* sv, int64_t id);
/* Finishes every queued request, then stops the workers. */
pgk_status pgk_server_free(pgk_server* sv);

/* Launch shapes chosen by the engine's autotuner, as text: one line per SPME
 * grid shape and precision (pencils per block of each FFT pass and its
 * measured time; every context measures the candidates for its grid shape
 * at pgk_init unless the process already holds a choice for that shape;
 * PGK_AUTOTUNE=0 in the environment keeps the fixed defaults; the choice
 * changes no result).  With PGK_PAIR_AUTOTUNE=1 also one line per
 * mixed-precision pair list in the cluster frame: the waves of blocks of the
 * pair kernel (1 to 4) timed at the context's first list build, which change
 * no force but the last bits of the kernel's FP32 energy and virial partials
 * (by default the kernel runs a fixed 3 waves).   Copies at most cap bytes (NUL-terminated)
 * and returns the length needed.  No counterpart in the reference. */
int64_t pgk_tuning_table(char* buf, int64_t cap);

/* Allocation-free SPME reciprocal force.  No counterpart in the reference.
 * For callers that must not allocate device memory during a run -- a host
 * driver or a replica server that reserves all of HBM up front, where
 * cudaMalloc/cudaFree would synchronise the device and could fail -- this
 * entry point computes fft_pmep's force on caller-owned device buffers and
 * allocates nothing: its temporaries live in one fixed static device array
 * (about 6.3 MB, held by every GPU that loads the library until exit).
 *   d_atmcor  (3,natom) device positions, d_atmchrg (natom) device charges
 *             (scaled as in prepmd.F90), box = host xcel,ycel,zcel;
 *   d_force   (3,natom) device forces, the reciprocal force is ADDED;
 *   pot_ewk   host pointer for the reciprocal energy (NULL = not needed;
 *             when given, the call waits for its stream);
 *   stream    cudaStream_t as void* (NULL = default stream).
 * Limits: nfft1*nfft2*nfft3 <= 64^3, each nfft <= 256, 3 <= pme_order <= 8;
 * larger sizes return PGK_E_SCRATCH_LIMIT.  Each nfft must also be a product
 * of 2, 3 and 5 (else PGK_E_UNSUPPORTED) and at least pme_order (else
 * PGK_E_INVALID); these checks come before any CUDA call.
 * The first call on a device looks up the array's address on that device;
 * make it before any stream capture.  All calls share the array and keep its
 * last contents: calls that overlap on the GPU race, so serialise them. */
pgk_status pgk_fft_pme_noalloc(const double* d_atmcor, const double* d_atmchrg, int32_t natom,
                               const double* box, double alpha, int32_t nfft1, int32_t nfft2,
                               int32_t nfft3, int32_t pme_order, double* d_force, double* pot_ewk,
                               void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PGK_GPU_H */
