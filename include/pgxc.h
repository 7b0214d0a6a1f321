/*
 * pgxc.h -- C ABI of libpgxc, the B200 (sm_100a) exchange-correlation grid
 * quadrature that replaces ParaGauss's per-SCF-cycle numerical XC build.
 *
 * Drop-in seam (ParaGauss source, paths relative to the project root):
 *   modules/xc_hamiltonian.f90:1124  call calc_xcks(ham_xc_arr, "orbitals")   (LDA, XC="VWN")
 *   modules/xc_hamiltonian.f90:1130  call calc_xcks_nl(ham_xc_arr)             (GGA, XC="PBE")
 * Both calls become one pgxc_build() plus a status check.  pgxc_create() is
 * called where xc_setup() runs (modules/xc_hamiltonian.f90:328-577), once per
 * geometry, and pgxc_destroy() where xc_close() runs.
 *
 * Conventions (all fixed by the reference; see the per-function comments):
 *   - lengths in bohr; arrays are the Fortran arrays passed by address, so
 *     "(n, m) column-major" means element (i, j) at [i + n*j];
 *   - basis order = unique atom -> l -> independent function -> radial
 *     function (modules/orbitalprojection_module.f90:30-45), radial functions
 *     = N_uncontracted primitives first, then contractions
 *     (modules/orbital_module.f90:1899-1930);
 *   - pgxc_build: C1 (one irrep, one partner); pgxc_build_sym: any irreps
 *     and partners; ispin 1 or 2.
 *
 * Error convention: every entry returns PGXC_OK (0) or a negative PGXC_E*
 * code; nothing aborts and no C++ exception crosses the ABI.  There is no CPU
 * fallback: without a usable CUDA device the calls fail with PGXC_ENODEV.
 */
#ifndef PGXC_H
#define PGXC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define PGXC_OK          0
#define PGXC_EINVAL     -1   /* bad argument, shape or size                 */
#define PGXC_ENOTSUP    -2   /* valid in ParaGauss but not in this library  */
#define PGXC_ENOMEM     -3   /* device allocation failed                    */
#define PGXC_ECUDA      -4   /* CUDA runtime error                          */
#define PGXC_ETIMEOUT   -5   /* a bounded device wait ran out               */
#define PGXC_ENONFINITE -6   /* NaN/Inf in an input or a result             */
#define PGXC_ENODEV     -7   /* no CUDA device / extension unusable         */

/* ---- functional ids: XC keywords of the reference ---------------------- */
/* XC="VWN": Slater exchange + VWN5 correlation (modules/xc_cntrl.f90:460-465) */
#define PGXC_XC_VWN 1
/* XC="PBE": Slater + PW92 + PBE-X enhancement + PBE-C H (xc_cntrl.f90:652-670) */
#define PGXC_XC_PBE 2
/* revPBE: Slater + PW92 + revPBE exchange (kappa 1.245) + PBE correlation
 * (keyword "revPBE", modules/xc_cntrl.f90:766-776) */
#define PGXC_XC_REVPBE 3
/* PBEsol: Slater + PW92 + PBEsol exchange (mu 10/81) + PBEsol correlation
 * (beta 0.046; keyword "PBESOL", modules/xc_cntrl.f90:788-798) */
#define PGXC_XC_PBESOL 4
/* BP86: Slater + VWN5 + Becke 88 exchange + Perdew 86 correlation
 * (keyword "BP", modules/xc_cntrl.f90:508-520) */
#define PGXC_XC_BP86 5
/* PW91: Slater + PW92 + PW91 exchange enhancement + PW91 correlation H0 + H1
 * (keyword "PW91", modules/xc_cntrl.f90:574-590) */
#define PGXC_XC_PW91 6
/* BPW91: Slater + PW92 + Becke 88 exchange + PW91 correlation
 * (keyword "BPW91", modules/xc_cntrl.f90:561-572) */
#define PGXC_XC_BPW91 7
/* BLYP: Slater + Becke 88 exchange + LYP correlation (LYP is a whole
 * correlation, no LDA part; keyword "BLYP", modules/xc_cntrl.f90:522-532) */
#define PGXC_XC_BLYP 8
/* XALPHA: Slater exchange alone, an LDA (keyword "XALPHA", modules/xc_cntrl.f90:454-458) */
#define PGXC_XC_XALPHA 9
/* B88: Slater + Becke 88 exchange, no correlation (keyword "B88", modules/xc_cntrl.f90:534-543) */
#define PGXC_XC_B88 10
/* PBEN: Slater + PW92 + PBEN exchange kappa (1 - exp(-mu s^2 / kappa)) + PBE
 * correlation (keyword "PBEN", modules/xc_cntrl.f90:714-732) */
#define PGXC_XC_PBEN 11
/* VMT, VT{8,4}, VMTsol, VT{8,4}sol: Slater + PW92 + the VMT / VT84 exchange
 * enhancements (PBE or PBEsol mu) + PBE correlation (keywords "VMT", "VT84",
 * "VMTsol", "VT84sol", modules/xc_cntrl.f90:900-950) */
#define PGXC_XC_VMT 12
#define PGXC_XC_VT84 13
#define PGXC_XC_VMTSOL 14
#define PGXC_XC_VT84SOL 15
/* HCTH/93, /120, /147, /407: Hamprecht-Cohen-Tozer-Handy exchange and
 * correlation, a whole functional with no Slater or LDA part (keywords "HCTH"
 * or "HCTHv1", "HCTH120" or "HCTHv2", "HCTH147" or "HCTHv3", "HCTH407" or
 * "HCTHv4", modules/xc_cntrl.f90:801-831; modules/hcth.f90) */
#define PGXC_XC_HCTH 16
#define PGXC_XC_HCTH120 17
#define PGXC_XC_HCTH147 18
#define PGXC_XC_HCTH407 19
/* NRECMV92: Slater + the non-relativistic Engel-Chevary-Macdonald-Vosko
 * exchange enhancement (a 2/2 Pade in s^2, g_ecmv92), no correlation
 * (keyword "NRECMV92", modules/xc_cntrl.f90:638-643) */
#define PGXC_XC_NRECMV92 20
/* PWLDA: Slater + PW92 correlation, an LDA (keywords "PWLDA", "PW-LDA",
 * "PWLSD", "PW-LSD", modules/xc_cntrl.f90:467-475) */
#define PGXC_XC_PWLDA 21
/* The grid parts of the hybrids (their exact exchange is not a grid term):
 * B3LYP = 0.80 Slater + 0.72 Becke 88 enhancement + 0.19 VWN5 + 0.81 LYP
 * (keyword "B3LYP", modules/xc_cntrl.f90:965-985); PBE0 = 0.75 Slater + PW92 +
 * 0.75 PBE exchange enhancement + PBE correlation ("PBE0", :996-1016) */
#define PGXC_XC_B3LYP 22
#define PGXC_XC_PBE0 23
/* LB94: Slater + VWN5 energy, with the van Leeuwen-Baerends correction added
 * to the potential only, -beta rho^(1/3) x^2 / (1 + 3 beta x asinh x) per
 * spin (keyword "LB94", modules/xc_cntrl.f90:500-506; baerends94_calc,
 * modules/baerends_module.f90:91-134) */
#define PGXC_XC_LB94 24
/* The relativistic keywords (exchange with X_LONGTRANS, speed of light
 * 137.03604): RVWN = relativistic Slater (x phi0(beta)) + VWN5 + the ec_RLDA
 * correction, an LDA ("RVWN", modules/xc_cntrl.f90:477-488; relxc.f90);
 * RBP = Slater + VWN5 + relativistic Becke 88 e_x (phi0 - 1 + phi2 G) +
 * Perdew 86 ("RBP", :545-558); ECMV92 = Slater + relativistic ECMV92
 * exchange ("ECMV92", :645-650) */
#define PGXC_XC_RVWN 25
#define PGXC_XC_RBP 26
#define PGXC_XC_ECMV92 27
/* RPW91 = PW92 + relativistic PW91 exchange e_x (phi0 - 1 + phi2 G_PW91)
 * (no Slater term: the keyword turns XAlpha off) + PW91 correlation H +
 * phi_c(n) times the H of pw91c_calc ("RPW91", modules/xc_cntrl.f90:626-636;
 * xc_func.f90:436-446; relxc.f90 rpw91c_calc :162-218) */
#define PGXC_XC_RPW91 28
/* RVWN_ENGEL = relativistic Slater + VWN5 + VWN5 (phic0(beta) - 1), the
 * Schmid-Engel-Dreizler-Blaha-Schwarz relativistic LDA correlation, an LDA
 * ("RVWN:Engel" / "RVWN_ENGEL", modules/xc_cntrl.f90:477-498; exchange.f90
 * correlation_lda :124-157, phic0 :159-204) */
#define PGXC_XC_RVWN_ENGEL 29
/* TPSS = TPSS exchange (tpss_X, modules/tpss.f90, TPSS_key) + TPSS
 * correlation (tpss_mgga_C, modules/tpss_mgga_module.f90), a meta-GGA: the
 * builds also form the kinetic-energy density tau = 1/2 sum occ |grad phi|^2
 * (density_calc_nl, modules/density_calc_module.f90:1540-1551) and the
 * potential's tau term 1/2 w df/dtau grad phi_i . grad phi_j
 * (modules/xc_hamiltonian.f90:1448-1454, :1534-1555); keyword "TPSS",
 * modules/xc_cntrl.f90:845-850; xc_func.f90:679-697.  Screened layout only
 * (screen_threshold >= 0). */
#define PGXC_XC_TPSS 30
/* M06L = M06-L exchange (m06_X, parameter set 1: e_x^LSDA F_PBE f(w) plus the
 * VSXC-form term) + M06-L correlation (m06_C: the VSXC-form same- and
 * opposite-spin terms plus the B97-form series), modules/m06.f90; keyword
 * "M06L", modules/xc_cntrl.f90:885-890; xc_func.f90:647-661.  A meta-GGA. */
#define PGXC_XC_M06L 31
/* M06 = the grid part of the hybrid M06 (m06_X and m06_C with parameter set
 * 2; the 0.27 exact exchange is not a grid term), keyword "M06",
 * modules/xc_cntrl.f90:892-898; xc_func.f90:663-677.  A meta-GGA. */
#define PGXC_XC_M06 32
/* VSXC = vsxc_X + vsxc_C (Van Voorhis-Scuseria, parameter set 0),
 * modules/vsxc_mgga_module.f90; keyword "VSXC" / "VS98",
 * modules/xc_cntrl.f90:952-957; xc_func.f90:776-790.  A meta-GGA.  The
 * closed-shell derivatives are the reference's: half those of the
 * open-shell form at equal spins (vsxc_X, vsxc_C). */
#define PGXC_XC_VSXC 33
/* the largest functional id */
#define PGXC_XC_LAST PGXC_XC_VSXC
/* nonzero for the meta-GGA keywords (density and potential with tau) */
#define PGXC_XC_IS_MGGA(id) ((id) >= PGXC_XC_TPSS && (id) <= PGXC_XC_VSXC)
/* nonzero for the GGA keywords (all but the five LDAs; the meta-GGAs too) */
#define PGXC_XC_IS_GGA(id) \
  ((id) != PGXC_XC_VWN && (id) != PGXC_XC_XALPHA && (id) != PGXC_XC_PWLDA && (id) != PGXC_XC_RVWN && \
   (id) != PGXC_XC_RVWN_ENGEL)

/* ---- precision modes ------------------------------------------------- */
#define PGXC_PREC_FP64        0  /* FP64 everywhere (FP64 tensor pipe): the drop-in */
/* Both contractions (X = phi P and V = Z^T phi) on the INT8 tensor cores
   with an Ozaki split: 5 balanced 7-bit digits per FP64 operand, the 15
   digit pairs of weight >= 2^-34, exact INT32 accumulation, one FP64
   combination; basis, functional, grid sums and V_xc stay FP64 */
#define PGXC_PREC_MIXED_INT8  1

/* Geometry: unique_atoms(:)%position(1:3,1) in bohr, atom-major xyz triplets. */
typedef struct pgxc_geometry {
  int32_t natoms;
  const double* coords;          /* [natoms*3] */
} pgxc_geometry;

/*
 * Orbital basis: one "shell" per (unique atom, l), in the reference order
 * (atom ascending, l ascending).  Mirrors unique_atom_basis_type
 * (modules/unique_atom_module.f90:143-168): exponents, norms (the legacy
 * norms of unique_atom_basis_norm_ob, :426-444, passed as the reference holds
 * them), N_uncontracted_fcts and contractions(N_exponents, N_contracted_fcts).
 */
typedef struct pgxc_basis {
  int32_t nshells;
  const int32_t* shell_atom;     /* [nshells] 0-based atom index            */
  const int32_t* shell_l;        /* [nshells] 0..3                          */
  const int32_t* shell_nexp;     /* [nshells] N_exponents                   */
  const int32_t* shell_nunc;     /* [nshells] N_uncontracted_fcts           */
  const int32_t* shell_ncontr;   /* [nshells] N_contracted_fcts             */
  const double* exponents;       /* [sum nexp]                              */
  const double* norms;           /* [sum nexp]                              */
  const double* contractions;    /* [sum nexp*ncontr], per shell (nexp,ncontr) column-major */
  /*
   * C1 symmetry adaptation (unique_atom_symadapt_type%m/%c of irrep 1,
   * partner 1): independent function i of angular momentum l is
   * sum_m sa_coef_l[i*(2l+1)+m] * Y_lm, m in the solid-harmonic order of
   * modules/solid_harmonics_module.f90:369-482 (p = z, x, y).  Blocks for
   * l = 0..sa_lmax are concatenated.  NULL means the identity.
   */
  const double* sa_coef;
  int32_t sa_lmax;
} pgxc_basis;

/*
 * Integration grid: grdpts(npts,4) of modules/grid_module.f90:3045-3164,
 * column-major x, y, z, w.  With weights_are_raw = 0 the weights are already
 * Becke-scaled (what mkgrid delivers).  With weights_are_raw = 1, column 4
 * holds the one-centre weights w_ang*w_rad*4*pi (grid_main_calc,
 * :425-432) and point_atom the host atom of each point; pgxc_create then
 * multiplies in the Becke partition weight on the device (becke0, :2442-2497).
 */
typedef struct pgxc_grid {
  int64_t npts;
  const double* grdpts;          /* [npts*4] column-major                   */
  int32_t weights_are_raw;
  const int32_t* point_atom;     /* [npts], required when weights_are_raw   */
} pgxc_grid;

/*
 * Atom-centred grid built by the library (grid_main_calc without pruning,
 * modules/grid_module.f90:357-504): atom a gets the Pople radial grid of
 * nrad[a] points scaled by radius[a] (RADIALGRID, :1246-1301; shells at
 * r >= 40 bohr dropped) times the Lebedev-McLaren rule with nang points
 * (INIGRD, :1359-2100; nang = 6, 8, 12, 14, 26, 38, 50, 78, 86, 110, 146,
 * 194 or 302), not rotated; points ordered atom -> shell -> angular point;
 * one-centre weights w_ang * w_rad * 4 pi (:425-432).
 */
typedef struct pgxc_grid_spec {
  const int32_t* nrad;           /* [natoms] NRADPTS of each atom            */
  const double* radius;          /* [natoms] RCUR of each atom, bohr         */
  int32_t nang;                  /* points of the angular rule               */
} pgxc_grid_spec;

typedef struct pgxc_options {
  int32_t functional;            /* PGXC_XC_VWN .. PGXC_XC_LAST             */
  int32_t ispin;                 /* 1 or 2; 2 (open shell) needs screen_threshold >= 0,
                                  * the dense layout returns PGXC_ENOTSUP */
  int32_t precision;             /* PGXC_PREC_*                             */
  int32_t batch_points;          /* points per tile, 0 -> 128 (machineparameters_veclen); only 128 */
  double  screen_threshold;      /* per-tile screening of basis functions:
                                  *   0  -> drop only functions that are exactly zero on
                                  *         the tile by the reference's alpha*r^2 < 50 rule
                                  *         (results as unscreened, up to rounding);
                                  *   >0 -> also drop functions whose |phi|, |grad phi|
                                  *         bound stays below the threshold on the tile;
                                  *   <0 -> no screening (dense layout) */
  int32_t device;                /* CUDA ordinal, -1 -> current device      */
  int32_t keep_orbitals;         /* screened layout: keep the basis values (and
                                  * their INT8 digits) of the whole grid on the
                                  * device after the first build and reuse them
                                  * in later builds of the same geometry, as the
                                  * reference's orbitals_in_memory does
                                  * (orbitalstore_module.f90); 0 -> evaluate in
                                  * every build.  Creation fails with
                                  * PGXC_ENOMEM when they do not fit. */
  int64_t max_chunk_points;      /* 0 -> sized from free HBM                */
} pgxc_options;

/* Per-phase device times of the last build, milliseconds (CUDA events). */
typedef struct pgxc_timings {
  double h2d_ms;
  double basis_ms;
  double density_ms;
  double functional_ms;
  double potential_ms;
  double d2h_ms;
  double total_ms;
  double xgemm_ms;        /* density contraction kernel (X = phi P, fused rho) */
  double vgemm_ms;        /* potential contraction kernel (V += phi^T Z)      */
  int64_t kernel_launches;
} pgxc_timings;

typedef struct pgxc_ctx pgxc_ctx;

/* Fill *opt with defaults (VWN, ispin 1, FP64, 128, exact screening 0.0, device -1). */
void pgxc_default_options(pgxc_options* opt);

/*
 * Per-geometry set-up; replaces the allocation part of xc_setup
 * (modules/xc_hamiltonian.f90:328-577) and, with weights_are_raw, the
 * Becke weighting of mkgrid (modules/grid_module.f90:3130-3137).
 * Copies geometry, basis and grid to device memory owned by *out.
 */
int pgxc_create(const pgxc_geometry* geo, const pgxc_basis* bas,
                const pgxc_grid* grid, const pgxc_options* opt,
                pgxc_ctx** out);

/*
 * pgxc_create on the grid of a spec, built on the device together with its
 * Becke weights (grid_main_calc, then mkgrid's Becke step, :3045-3164): for
 * optimiser or dynamics loops whose per-geometry grid never passes through
 * host memory.  The context behaves as one created with weights_are_raw = 1
 * (the nuclear gradient is available).
 */
int pgxc_create_on_grid(const pgxc_geometry* geo, const pgxc_basis* bas,
                        const pgxc_grid_spec* spec, const pgxc_options* opt,
                        pgxc_ctx** out);

/* Points of the grid of a spec (library extension, no reference counterpart). */
int pgxc_atomic_grid_size(const pgxc_geometry* geo, const pgxc_grid_spec* spec,
                          int64_t* npts);

/*
 * The grid of a spec written to device memory of the current device:
 * d_grdpts (npts, 4) column-major x, y, z, raw one-centre weight, and
 * d_point_atom (npts) the host atom of each point, ordered as grid_main_calc
 * orders AGRID; npts must equal pgxc_atomic_grid_size.  Enqueued on stream
 * (a cudaStream_t, NULL = legacy default) and synchronised before returning.
 */
int pgxc_atomic_grid(const pgxc_geometry* geo, const pgxc_grid_spec* spec,
                     int64_t npts, double* d_grdpts, int32_t* d_point_atom,
                     void* stream);

/* Number of orbital basis functions (irrep dimension in C1). */
int pgxc_nbas(const pgxc_ctx* ctx, int32_t* nbas);

/*
 * Screening plan of a context created with screen_threshold >= 0 (library
 * extension, no reference counterpart): 128-point tiles, padded slots, listed
 * (tile, function) pairs and sum over tiles of (listed functions)^2.
 * PGXC_EINVAL for a dense-layout context.
 */
int pgxc_screen_stats(const pgxc_ctx* ctx, int64_t* ntiles, int64_t* nslots,
                      int64_t* nlisted, double* sum_n2);

/*
 * One XC build; replaces calc_xcks (modules/xc_hamiltonian.f90:812-1036)
 * and calc_xcks_nl (:1280-1580) for n_irrep = 1, partners = 1.
 *   C   : eigvec_occ(1)%m(nbas, nocc, ispin), column-major
 *         (modules/occupied_levels_module.f90:112-117)
 *   occ : occ_num_occ(1)%m(nocc, ispin), column-major
 *   ham_xc_arr : packed upper triangle, element (k,j), k<=j, of spin s at
 *         ham_xc_arr[s + ispin*(j*(j+1)/2 + k)] (0-based), ACCUMULATED (+=)
 *         exactly like tristore (:1018-1034) and :1559-1566;
 *         xc_length must equal ispin*nbas*(nbas+1)/2.
 *   exc, nel : the build's E_xc and integrated charge are ADDED to *exc and
 *         *nel (exc_int / charge_int of :936-949, :1408-1423).
 *   timings may be NULL.
 * Synchronous: the outputs are valid on return.
 */
int pgxc_build(pgxc_ctx* ctx, const double* C, const double* occ,
               int32_t nbas, int32_t nocc, int32_t ispin,
               double* ham_xc_arr, int64_t xc_length,
               double* exc, double* nel, pgxc_timings* timings);

/*
 * Same build from the density matrix itself, for callers that form P
 * (P_s = sum_j occ_js C_js C_js^T per spin) themselves:
 *   P : nbas x nbas per spin, column-major, spin blocks of nbas*nbas,
 *       symmetric (host memory).
 * ham_xc_arr, exc and nel are accumulated into exactly as by pgxc_build.
 * Replaces the occupied-orbital products of density_calc_nl
 * (modules/density_calc_module.f90:1498-1538) by the P form of the same rho.
 */
int pgxc_build_density(pgxc_ctx* ctx, const double* P, int32_t nbas, int32_t ispin,
                       double* ham_xc_arr, int64_t xc_length,
                       double* exc, double* nel, pgxc_timings* timings);

/*
 * Same build with every operand already in device memory of the context's
 * device (for callers that keep C on the GPU).  d_exc_nel receives
 * {E_xc, N_el} (overwritten, not accumulated); d_ham_xc_arr is overwritten
 * with the packed matrix of this build.  Runs on the context's stream and
 * synchronises before returning.
 */
int pgxc_build_device(pgxc_ctx* ctx, const double* d_C, const double* d_occ,
                      int32_t nbas, int32_t nocc, int32_t ispin,
                      double* d_ham_xc_arr, int64_t xc_length,
                      double* d_exc_nel, pgxc_timings* timings);

/*
 * Post-SCF XC nuclear gradient: dE_xc/dR of every atom, ADDED into grad
 * (natoms x 3: x, y, z of atom 0, then atom 1, ...), and E_xc added into *exc
 * (may be NULL).  The grid moves with its atoms (each point with its
 * point_atom) and the Becke weights are differentiated, so this is the
 * derivative of the energy the builds integrate, as the reference's post-SCF
 * gradients with weight gradients (post_scf_calc_xc_en_and_gr(_nl),
 * modules/post_scf_module.f90:2569-3318, :3500-5193; density_calc_ph_nl,
 * modules/density_calc_module.f90:2000-3315; becke1, modules/grid_module.f90
 * :2499-2616).  Needs a context created with weights_are_raw (PGXC_ENOTSUP
 * otherwise).  FP64 in every precision mode.  A context with
 * pgxc_set_symmetry applied takes pgxc_xc_gradient_sym (PGXC_EINVAL here).
 */
int pgxc_xc_gradient(pgxc_ctx* ctx, const double* C, const double* occ,
                     int32_t nbas, int32_t nocc, int32_t ispin, double* grad, double* exc);

/*
 * E_xc of several functionals on one density, as the post-SCF XC energies
 * (post_scf_calc_xc_energy, modules/post_scf_module.f90:2204-2564, and the
 * energy table of xc_func_get_exc, modules/xc_func.f90:1011-1200): one basis
 * and density pass, then one functional pass per entry of functionals[n];
 * exc[i] is overwritten with the energy of functionals[i], *nel (may be NULL)
 * with the integrated charge.  Needs a screened context (PGXC_ENOTSUP
 * otherwise); a GGA functional needs a context created with a GGA or
 * meta-GGA functional (its density gradients).  A meta-GGA (TPSS, M06L, M06,
 * VSXC) also needs tau = 1/2 sum_i occ_i |grad psi_i|^2, which the pass forms
 * (as the reference's post-SCF pass does) in a meta-GGA context or in a GGA
 * context of the FP64 build; in an INT8 GGA context (FP32 gradient planes)
 * it returns PGXC_ENOTSUP.  No potential is built.
 */
int pgxc_xc_energies(pgxc_ctx* ctx, const double* C, const double* occ,
                     int32_t nbas, int32_t nocc, int32_t ispin,
                     int32_t n, const int32_t* functionals, double* exc, double* nel);

/*
 * Symmetry-adapted bases (n_irrep >= 1 irreps, partners >= 1 each), as the
 * reference's orbitals per irrep and partner (orbs_ob(i)%o(:,:,partner),
 * orbital_module.f90:2421-2619, from the symadapt coefficients of
 * unique_atom_module.f90).  Symmetry-adapted function fn of irrep i and
 * partner p is sum over entries e with (irrep, partner, fn) = (i, p, fn) of
 * coef[e] * chi_ao[e], chi the context's C1 basis functions (all atoms,
 * equal atoms expanded).  Indices are 0-based; repeated entries add up.
 */
typedef struct pgxc_symmetry {
  int32_t n_irrep;
  const int32_t* dims;       /* [n_irrep] functions of each irrep (per partner) */
  const int32_t* partners;   /* [n_irrep] */
  int64_t nnz;
  const int32_t* irrep;      /* [nnz] */
  const int32_t* partner;    /* [nnz] */
  const int32_t* fn;         /* [nnz] function within its irrep */
  const int32_t* ao;         /* [nnz] C1 basis function */
  const double* coef;        /* [nnz] */
} pgxc_symmetry;

/* Attach (or replace) the symmetry adaptation of a context. */
int pgxc_set_symmetry(pgxc_ctx* ctx, const pgxc_symmetry* sym);

/*
 * Pseudo-2D irreps of the attached symmetry adaptation (xc_pseudo2d_sym,
 * modules/xc_hamiltonian.f90:2637-2779, called by xc_build after the grid
 * sums): in such an irrep the functions of every (unique atom, l) block come
 * in two halves A and B (n_exponents x n_independent/2 functions each, A
 * first), and because the grid is not totally symmetric the built matrix is
 * made to satisfy H(X_A, Y_A) = H(X_B, Y_B) (their mean) and H(X_A, Y_B) =
 * -H(X_B, Y_A) (half their difference) for every pair of blocks X >= Y.
 * pgxc_build_sym applies it to its result (before accumulating into
 * ham_xc_arr) for the irreps with nblocks[i] > 0.
 *   nblocks[n_irrep] : blocks of each irrep (0: not pseudo-2D)
 *   first[sum]       : first function of each block within its irrep
 *                      (0-based, ascending: orbitalprojection_ob - 1)
 *   half[sum]        : functions in each block's first half
 * NULL nblocks removes it.  Needs pgxc_set_symmetry first.
 */
int pgxc_set_pseudo2d(pgxc_ctx* ctx, const int32_t* nblocks, const int32_t* first, const int32_t* half);

/* ispin * sum_i dims_i (dims_i + 1) / 2: the ham_xc_arr length of pgxc_build_sym. */
int pgxc_sym_xc_length(const pgxc_ctx* ctx, int64_t* xc_length);

/*
 * One XC build in the symmetry-adapted basis; replaces calc_xcks
 * (modules/xc_hamiltonian.f90:812-1036) and calc_xcks_nl (:1280-1580) for
 * any n_irrep and partners.
 *   C[i]   : eigvec_occ(i)%m(dims_i, nocc[i], ispin), column-major
 *   occ[i] : occ_num_occ(i)%m(nocc[i], ispin); the density weights each
 *            partner by occ / partners_i (density_calc_nl, :1534-1538)
 *   ham_xc_arr : per spin s, the irreps' packed triangles one after the other
 *            with spin stride ispin, element (k,j), k<=j, of irrep i at
 *            ham_xc_arr[s + ispin*(off_i + j*(j+1)/2 + k)], off_i = sum_{i'<i}
 *            dims_i'(dims_i'+1)/2; V_i = 1/partners_i sum_p phi_p^T v phi_p,
 *            ACCUMULATED (+=) as tristore and :1559-1566 do.
 *   exc, nel : added to, as by pgxc_build.
 * The grid may be the reference's symmetry-reduced one (weights times the
 * number of equal atoms): the build integrates exactly the sums it does.
 */
int pgxc_build_sym(pgxc_ctx* ctx, const double* const* C, const double* const* occ,
                   const int32_t* nocc, int32_t ispin,
                   double* ham_xc_arr, int64_t xc_length,
                   double* exc, double* nel, pgxc_timings* timings);

/*
 * The XC nuclear gradient of a symmetry-adapted context (pgxc_set_symmetry),
 * with the irreps' orbitals as pgxc_build_sym takes them.  grad (natoms x 3,
 * the context's atoms in their C1 order) and *exc are ADDED into, as
 * pgxc_xc_gradient.  The orbitals are expanded into the C1 basis and the C1
 * gradient runs on the context's grid.  On the symmetry-reduced grid of the
 * reference (the points of one equal atom per unique atom, weights times
 * n_equal_atoms, point_atom that atom) the result is the reference's grad_xc
 * before post_scf_average_gradient (modules/post_scf_module.f90:1953-1982),
 * which the caller applies as before; on the full grid it is the gradient
 * itself.  Replaces the gradient accumulation of post_scf_calc_xc_en_and_gr_nl
 * (modules/post_scf_module.f90:2940-3013) for symmetric molecules.
 */
int pgxc_xc_gradient_sym(pgxc_ctx* ctx, const double* const* C, const double* const* occ,
                         const int32_t* nocc, int32_t ispin, double* grad, double* exc);

/*
 * Batched builds of many small systems (a set of molecules, each with its own
 * context).  pgxc_batch_create captures the device build of every context
 * (as pgxc_build_device, with the device operands given here) as one parallel
 * branch of a single CUDA graph; pgxc_batch_run replays the graph, so that
 * the builds of all systems run concurrently with one launch.  Each context
 * must use the screened layout (screen_threshold >= 0) and the same device;
 * a context belongs to at most one live batch and must not be built by other
 * calls while its batch runs.  Operand pointers are fixed for the life of
 * the batch; their contents may change between runs.  nocc[i] is the
 * occupied-orbital count of context i; d_ham[i] (packed, xc_length of the
 * context) and d_exc_nel[i] ({E_xc, N_el}) are overwritten by every run.
 * pgxc_batch_run synchronises and returns the graph's device time in *ms
 * (may be NULL).  No counterpart in the reference (one system per process).
 *
 * When every context is a screened INT8 closed-shell one (no symmetry
 * adaptation, no keep_orbitals) the contexts run as one set: per chunk of
 * their concatenated 128-point tiles (all contexts' grid batches in one work
 * queue) the graph holds one launch of each kernel, whose persistent blocks
 * walk tiles of many contexts (each tile's density matrix and V_xc through a
 * per-tile context table); only the per-context density-matrix preparation
 * stays one branch per context.  pgxc_batch_create_chunked sets the set's
 * chunk in points (0: sized from free device memory, the choice of
 * pgxc_batch_create).
 */
typedef struct pgxc_batch pgxc_batch;
int pgxc_batch_create(pgxc_ctx* const* ctx, int32_t n, const double* const* d_C, const double* const* d_occ,
                      const int32_t* nocc, double* const* d_ham, double* const* d_exc_nel, pgxc_batch** out);
int pgxc_batch_create_chunked(pgxc_ctx* const* ctx, int32_t n, const double* const* d_C,
                              const double* const* d_occ, const int32_t* nocc, double* const* d_ham,
                              double* const* d_exc_nel, int64_t max_chunk_points, pgxc_batch** out);
/* Whether a batch runs as one set (1) or as per-context graph branches (0). */
int pgxc_batch_is_set(const pgxc_batch* batch, int32_t* is_set);
int pgxc_batch_run(pgxc_batch* batch, double* ms);
/* Nodes of the batch's CUDA graph: kernel launches and all nodes. */
int pgxc_batch_stats(const pgxc_batch* batch, int64_t* kernel_nodes, int64_t* nodes);
void pgxc_batch_destroy(pgxc_batch* batch);

/* Copy of the grid weights the context integrates with (Becke-scaled). */
int pgxc_grid_weights(const pgxc_ctx* ctx, double* w_out, int64_t npts);

/*
 * Basis functions and gradients on arbitrary points; replaces
 * orbital_calculate (modules/orbital_module.f90:1934-2299) with
 * calculate_orbs_and_grads_v3 (:2421-2619).
 *   pts   : (npts, 3) column-major
 *   phi   : (npts, nbas) column-major      (orbs_ob(1)%o(:,:,1))
 *   grads : (npts, 3, nbas) column-major or NULL (orbs_grads(1)%o(:,:,:,1))
 */
int pgxc_orbital_calculate(pgxc_ctx* ctx, int64_t npts, const double* pts,
                           double* phi, double* grads);

/*
 * Point-wise functional, FP64, on the device; replaces xc_functionals
 * (modules/xc_func.f90:187-899) for the two keywords.
 *   rho : (n, ispin); gam : (n, 2*ispin-1) or NULL for VWN
 *   f   : (n); fr : (n, ispin); fg : (n, 2*ispin-1) or NULL for VWN
 */
int pgxc_xc_functionals(int32_t functional, int32_t ispin, int64_t n,
                        const double* rho, const double* gam,
                        double* f, double* fr, double* fg);

/*
 * The same for a meta-GGA (PGXC_XC_IS_MGGA), which also takes the kinetic
 * energy density: xc_functionals with tau (modules/xc_func.f90:187, :679-697).
 *   tau : (n, ispin); ft : (n, ispin) = df/dtau
 * pgxc_xc_functionals rejects the meta-GGA ids (PGXC_EINVAL).
 */
int pgxc_xc_functionals_mgga(int32_t functional, int32_t ispin, int64_t n, const double* rho,
                             const double* gam, const double* tau, double* f, double* fr,
                             double* fg, double* ft);

/*
 * Becke partition weights on the device; replaces atomicweight2/becke0
 * (modules/grid_module.f90:2264-2497, autodiff/becke_step_func.f90:84-124)
 * with art = 0 (WEIGHT_GRADS default, :371-372).
 *   pts : (npts, 3) column-major; point_atom : host atom per point;
 *   w_out : partition weight of the host atom at each point.
 */
int pgxc_becke_weights(const pgxc_geometry* geo, int64_t npts,
                       const double* pts, const int32_t* point_atom,
                       double* w_out);

/*
 * Allocation-free Becke weights.  No counterpart in the reference: this is an
 * extra entry for callers that cannot let a library allocate device memory
 * (a driver whose device arrays all come from its own pool or OpenACC /
 * CUDA Fortran data regions, or a process that reserved the whole device).
 * Same result as pgxc_becke_weights, but every argument is device memory:
 *   d_coords (natoms*3), d_pts (npts,3) column-major, d_point_atom (npts),
 *   d_w_out (npts).
 * The only scratch, the natoms x natoms matrices of atom-atom distances and
 * of their reciprocals, lives in a fixed device array inside the library
 * (2 PGXC_NOALLOC_MAX_ATOMS^2 doubles, 4 MiB, present on every GPU that loads
 * the library until the process exits); natoms above PGXC_NOALLOC_MAX_ATOMS
 * is rejected with PGXC_EINVAL.  It makes no cudaMalloc/cudaFree call.  The
 * first call on a device (and again after the caller makes a different CUDA
 * context current on it) looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.  Work is queued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream) and the call returns without waiting: the
 * weights are valid once that stream is synchronised.  All calls on a device
 * share the scratch array, which keeps the last call's contents (each call
 * rewrites every entry it reads): calls that overlap on the GPU race.
 * Errors are reported through pgxc_last_error(NULL).
 */
#define PGXC_NOALLOC_MAX_ATOMS 512
int pgxc_becke_weights_noalloc(int32_t natoms, const double* d_coords,
                               int64_t npts, const double* d_pts,
                               const int32_t* d_point_atom, double* d_w_out,
                               void* stream);

const char* pgxc_last_error(const pgxc_ctx* ctx);   /* ctx may be NULL */
const char* pgxc_strerror(int status);

void pgxc_destroy(pgxc_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* PGXC_H */
