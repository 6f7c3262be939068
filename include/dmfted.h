/*
 * dmfted.h -- C-ABI of the B200 (sm_100a) exact-diagonalization impurity
 * solver for dmft-ed (normal ed_mode, normal bath).
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (DMFTED_OK == 0).  dmfted_last_error() gives the message of the last
 * failure on the calling thread.  A Fortran iso_c_binding shim maps a non-zero
 * status to `stop "<message>"`, which is what the reference does on the same
 * conditions.
 *
 * Conventions kept from the reference so that a Fortran caller passes its own
 * arrays unchanged:
 *   - sector indices are 1-based, numbered nup-major:
 *       isector = nup*(Ns+1) + ndw + 1            (ED_SETUP.f90:388-400)
 *   - a sector vector is indexed like the reference's H%map:
 *       i = rank_up + DimUp*rank_dw               (ED_SETUP.f90:880-890)
 *   - complex128 arrays are interleaved (re, im) doubles, Fortran complex(8);
 *   - multi-index arrays are Fortran column-major, e.g.
 *       impGmats(Nspin,Nspin,Norb,Norb,Lmats)     (ED_VARS_GLOBAL.f90:120-125)
 *   - the user bath array has the set_dmft_bath layout: e(ispin,iorb,k) then
 *     v(ispin,iorb,k), k fastest              (ED_BATH/dmft_aux.f90:493-512).
 *
 * One context per process and GPU.  A context queues its work on its own CUDA
 * stream; the grid-wide Green's-function chains also use a second stream of
 * the context, joined back to the first before the call returns.  Calls on a
 * context are not thread-safe (the reference's module state is not either).
 */
#ifndef DMFTED_H
#define DMFTED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DMFTED_OK 0
#define DMFTED_ERR_ARG 1         /* bad argument or size mismatch            */
#define DMFTED_ERR_CUDA 2        /* CUDA runtime failure                     */
#define DMFTED_ERR_NOMEM 3       /* device allocation failed                 */
#define DMFTED_ERR_UNSUPPORTED 4 /* configuration outside this solver        */
#define DMFTED_ERR_STATE 5       /* call out of order (no sector / no bath)  */
#define DMFTED_ERR_NOTCONV 6     /* iteration limit hit before convergence   */
#define DMFTED_ERR_NORM 7        /* state not normalised                     */

/* ---- precision of the Lanczos vectors ------------------------------- */
#define DMFTED_FP64 0  /* plain FP64: the drop-in path                       */
#define DMFTED_MIXED 1 /* FP32 vectors and H*v, compensated FP64 alpha/beta,
                          FP64 refinement of the ground state, GF chains
                          with their first 20 steps in FP64 and the rest in
                          FP32 (chains of one-CTA batches: FP64), FP64
                          continued fractions for G(iwn)                      */

/* Input variables of ED_INPUT_VARS.f90 that define the hot path, with the
 * reference's names and defaults (dmfted_default_params fills those). */
typedef struct dmfted_params {
    int32_t norb, nbath, nspin;   /* NORB, NBATH, NSPIN            :111-113 */
    int32_t hfmode, jhflag;       /* HFMODE (T), JHFLAG (F)        :143-144 */
    double uloc[3];               /* ULOC                          :114     */
    double ust, jh, jx, jp;       /* UST, JH, JX, JP               :115-118 */
    double xmu, beta;             /* XMU, BETA                     :119-120 */
    int32_t lmats, lreal;         /* LMATS, LREAL                  :133-134 */
    double wini, wfin, eps;       /* WINI, WFIN, EPS               :140-145 */
    int32_t lanc_niter;           /* LANC_NITER (512)              :154     */
    int32_t lanc_ngfiter;         /* LANC_NGFITER (200)            :155     */
    double lanc_tolerance;        /* LANC_TOLERANCE (1e-12)        :156     */
    int32_t lanc_dim_threshold;   /* LANC_DIM_THRESHOLD (256)      :157     */
    int32_t lanc_nstates_sector;  /* LANC_NSTATES_SECTOR (6)       :149     */
    int32_t lanc_nstates_total;   /* LANC_NSTATES_TOTAL (1 => T=0) :150     */
    int32_t lanc_nstates_step;    /* LANC_NSTATES_STEP (2)         :151     */
    double gs_threshold;          /* GS_THRESHOLD (1e-9)           :147     */
    double cutoff;                /* CUTOFF (1e-9)                 :146     */
    int32_t ed_twin;              /* ED_TWIN (F)                   :125     */
    int32_t lfit;                 /* LFIT (1000)                   :136     */
    int32_t cg_weight;            /* CG_WEIGHT (0)                 :164     */
    /* additions of this solver (defaults keep the reference behaviour) */
    int32_t precision;            /* DMFTED_FP64 or DMFTED_MIXED            */
    int32_t lanc_ncheck;          /* Ritz-value check interval (10)         */
    int32_t device;               /* CUDA device ordinal (0)                */
    double lanc_gf_threshold;     /* |b| that ends a GF chain (1e-13)       */
    /* the bath fit (ED_INPUT_VARS.f90:158-164) */
    int32_t cg_niter;             /* CG_NITER (500)                :158     */
    int32_t cg_scheme;            /* CG_SCHEME: DMFTED_CG_WEISS (default) or
                                     DMFTED_CG_DELTA               :159     */
    double cg_ftol;               /* CG_FTOL (1e-5)                :160     */
    int32_t cg_stop;              /* CG_STOP (0)                   :162     */
    double cg_eps;                /* CG_EPS (1e-6)                 :163     */
} dmfted_params;

/* cg_scheme: what the bath fit matches (fitgf_normal_normal.f90:72-82) */
#define DMFTED_CG_DELTA 0 /* the hybridisation Delta(iw_n)                  */
#define DMFTED_CG_WEISS 1 /* the Weiss field G0(iw_n) = 1/(iw_n+xmu-Hloc-Delta) */

typedef struct dmfted_ctx dmfted_ctx;

/* Fill *p with the reference defaults (ED_INPUT_VARS.f90:111-176). */
void dmfted_default_params(dmfted_params *p);

/* Message of the last failing call on this thread ("" if none). */
const char *dmfted_last_error(void);

/* Library version string. */
const char *dmfted_version(void);

/* ---- set-up ------------------------------------------------------------
 * dmfted_init replaces ed_init_solver_single (ED_MAIN.f90:67-107):
 * init_ed_structure (ED_SETUP.f90:135-367) and setup_pointers_normal
 * (:379-493).  It builds the Fock-space tables on the device (all popcount
 * classes of Ns-bit words, their ranks, the hopping tables) and allocates the
 * working set.  hloc: impHloc(Nspin,Nspin,Norb,Norb) complex128, may be NULL
 * (zero).  Unsupported: Norb>3, Nspin>2 (the reference stops there too,
 * ED_SETUP.f90:274-275), complex off-diagonal Hloc.                        */
int dmfted_init(const dmfted_params *p, const double *hloc, dmfted_ctx **out);
int dmfted_free(dmfted_ctx *ctx);

/* set_Hloc (ED_AUX_FUNX.f90:135-143): replace impHloc. */
int dmfted_set_hloc(dmfted_ctx *ctx, const double *hloc);

/* get_bath_dimension, normal bath (ED_BATH/user_aux.f90:11-94):
 * 2*Nspin*Norb*Nbath. */
int dmfted_get_bath_dimension(const dmfted_params *p, int32_t *nb);

/* set_dmft_bath (ED_BATH/dmft_aux.f90:474-512): load the user bath array. */
int dmfted_set_bath(dmfted_ctx *ctx, const double *bath, int32_t nb);

/* Sector tables of setup_pointers_normal (ED_SETUP.f90:379-493), all values
 * 1-based as the reference stores them.  Sizes: nsectors=(Ns+1)^2 for
 * getnup..getdimdw, 2*nsectors for getcsector/getcdgsector (index
 * (isector-1)*2+ispin-1), (Ns+1)^2 for getsector (index nup*(Ns+1)+ndw),
 * Norb*Nbath for getbathstride (index (k-1)*Norb+iorb-1), 2*Norb for
 * impindex (index (ispin-1)*Norb+iorb-1).  Any pointer may be NULL. */
int dmfted_sector_tables(dmfted_ctx *ctx, int32_t *nsectors, int32_t *getsector, int32_t *getnup,
                         int32_t *getndw, int32_t *getdim, int32_t *getdimup, int32_t *getdimdw,
                         int32_t *getcsector, int32_t *getcdgsector, int32_t *getbathstride,
                         int32_t *impindex);

/* build_sector (ED_SETUP.f90:861-891, normal): the sector -> Fock map
 * map[i] = iup + idw*2^Ns in the reference's order, computed on the device
 * by combinatorial unranking (bit-exact).  dim must equal getdim(isector);
 * needs Ns <= 15 (the reference stores the map in a default integer). */
int dmfted_build_sector(dmfted_ctx *ctx, int32_t isector, int32_t *map, int64_t dim);

/* setup_Hv_sector / delete_Hv_sector (ED_HAMILTONIAN_MATVEC.f90:99-111). */
int dmfted_setup_hv_sector(dmfted_ctx *ctx, int32_t isector);
int dmfted_delete_hv_sector(dmfted_ctx *ctx);

/* ---- H*v ----------------------------------------------------------------
 * Procedure-pointer target with the cc_sparse_HxV contract
 * (ED_VARS_GLOBAL.f90:43-49, selected at ED_MAIN.f90:269-276): Hv = H v on
 * the sector set by dmfted_setup_hv_sector, complex128 host arrays of length
 * nloc == getdim(isector).  Replaces directMatVec_cc
 * (ED_HAMILTONIAN_MATVEC.f90:289-351); copies in and out of the device on
 * every call (compatibility mode for solvers that own the vectors).     */
int dmfted_hxv_c128(dmfted_ctx *ctx, int32_t nloc, const double *v, double *hv);

/* Same product on device-resident real vectors of the current sector
 * (float64 or float32), on the context's stream; nvec vectors stored back to
 * back.  For callers that keep their vectors on the device. */
int dmfted_hxv_device_f64(dmfted_ctx *ctx, const double *d_v, double *d_hv, int32_t nvec);
int dmfted_hxv_device_f32(dmfted_ctx *ctx, const float *d_v, float *d_hv, int32_t nvec);

/* ---- device-resident solvers ----------------------------------------- */
/* Lowest eigenpair of sector isector by Lanczos on the device; stands in for
 * sp_eigh with Neigen=1 (ED_DIAG.f90:169-183).  psi (complex128, length
 * getdim) may be NULL.  *niter: H*v products used (may be NULL).  Precision
 * follows params.precision. */
int dmfted_lanczos_gs(dmfted_ctx *ctx, int32_t isector, double *e0, double *psi, int32_t *niter);

/* The eigenpairs of one sector as ed_diag_c computes them: stands in for the
 * sp_eigh call (ED_DIAG.f90:169-183) and the dense eigh branch (:184-194) with
 * the reference's choice between them -- eigh when neigen == dim or
 * dim <= lanc_dim_threshold (:136-137), Lanczos otherwise.  Returns the
 * lowest min(neigen, dim) eigenvalues in ascending order, degenerate copies
 * included (Lanczos runs are followed by probe runs orthogonal to the pairs
 * found, until a probe finds nothing new).  evals[neigen]; evecs (may be NULL)
 * complex128 eig_basis(Dim, neigen) column-major, i.e. vector i at
 * evecs + 2*i*dim, in the H%map order.  nitermax, tol: the sp_eigh arguments
 * (<= 0 takes lanc_niter / lanc_tolerance).  *nfound: pairs returned.
 * neigen == 1 follows params.precision; more pairs are FP64. */
int dmfted_gs_lanczos(dmfted_ctx *ctx, int32_t isector, int32_t neigen, int32_t nitermax,
                      double tol, double *evals, double *evecs, int32_t *nfound);

/* Three-term Lanczos tridiagonalisation from a given start vector, the
 * contract of sp_lanc_tridiag (build_gf_normal.f90:118-127): vvinit complex128
 * of length getdim(isector) (normalised here), alanc[nlanc], blanc[nlanc]
 * with blanc[0]=0 and blanc[k]=b_k coupling steps k-1 and k.  *nused: steps
 * taken before |b| fell below lanc_gf_threshold. */
int dmfted_lanc_tridiag(dmfted_ctx *ctx, int32_t isector, const double *vvinit, int32_t nlanc,
                        double *alanc, double *blanc, int32_t *nused);

/* No counterpart in the reference.  The tridiagonalisation of
 * dmfted_lanc_tridiag (FP64) for callers that cannot allocate device memory at
 * the time of the call -- a host whose device memory belongs to its own pool
 * manager, or a latency-critical loop where cudaMalloc must not run.  The
 * caller owns every buffer the call touches: d_v0 (real start vector of
 * length getdim(isector), any norm), d_work (2*getdim(isector) doubles for the
 * two rotating Lanczos vectors), d_alanc[nlanc], d_blanc[nlanc] (same
 * convention as dmfted_lanc_tridiag) and d_nused, all device pointers.  The
 * reduction scratch is a fixed array inside the library (about 90 KB per GPU,
 * held until the process exits); the call allocates and frees nothing.
 * Limit: 1 <= nlanc <= 1022, else DMFTED_ERR_ARG; a context whose model has
 * the Jhflag spin-exchange / pair-hopping terms is refused with
 * DMFTED_ERR_UNSUPPORTED (its Lanczos step needs a vector of scratch).  Calls on one device share
 * the array and must not overlap on the GPU.  The first call on a device
 * looks up the array's device address; make it before any stream capture.
 * Returns after the results are written (the context's stream is
 * synchronised). */
int dmfted_lanc_tridiag_noalloc(dmfted_ctx *ctx, int32_t isector, const double *d_v0,
                                int32_t nlanc, double *d_work, double *d_alanc, double *d_blanc,
                                int32_t *d_nused);

/* add_to_lanczos_gf_normal (build_gf_normal.f90:442-488) for one chain: adds
 * pesoBZ * sum_j Z(1,j)^2 / (z - isign (E_j - Ei)) over the Matsubara grid
 * (gmats, complex128[Lmats]) and the real axis z = w + i eps (greal,
 * complex128[Lreal], may be NULL) of the context's parameters, with
 * pesoBZ = vnorm2 exp(-beta (Ei - Egs)) / zeta at finite temperature (0 when
 * beta (Ei - Egs) >= 200) and vnorm2 / zeta at T=0 (lanc_nstates_total == 1).
 * alanc[nlanc], blanc[nlanc] in the dmfted_lanc_tridiag convention (blanc[0]
 * unused).  The pole sum is the chain's continued fraction, evaluated on the
 * device in FP64, as every solve does. */
int dmfted_add_to_lanczos_gf(dmfted_ctx *ctx, double vnorm2, double ei, double egs, double zeta,
                             int32_t nlanc, const double *alanc, const double *blanc,
                             int32_t isign, double *gmats, double *greal);

/* ---- the solve ------------------------------------------------------------
 * ed_solve_single (ED_MAIN.f90:251-289) for the normal mode:
 * set_dmft_bath, diagonalize_impurity (ED_DIAG.f90:78-398), the observables
 * of observables_impurity (ED_OBSERVABLES.f90:113-160), buildgf_impurity
 * (ED_GREENS_FUNCTIONS.f90:111-175 with build_gf_normal.f90:71-180,442-488)
 * and get_sigma_normal.  Everything stays on the device until read back with
 * the getters below.  T=0 (lanc_nstates_total==1) and finite temperature are
 * both handled.  sectors: optional list of 1-based sectors to restrict the
 * scan to (NULL / nsectors=0 scans every sector the reference scans). */
int dmfted_ed_solve(dmfted_ctx *ctx, const double *bath, int32_t nb, const int32_t *sectors,
                    int32_t nsectors);

/* Getters (ED_IO.f90:371-394).  G-like arrays are complex128 with the
 * reference's shape (Nspin,Nspin,Norb,Norb,L), column-major. */
int dmfted_get_gimp_matsubara(dmfted_ctx *ctx, double *g);
int dmfted_get_gimp_real(dmfted_ctx *ctx, double *g);
int dmfted_get_sigma_matsubara(dmfted_ctx *ctx, double *s);
int dmfted_get_sigma_real(dmfted_ctx *ctx, double *s);
int dmfted_get_g0imp_matsubara(dmfted_ctx *ctx, double *g);
/* ed_get_g0imp_real: G0and(w + i eps) = 1/G0^-1 on the real axis
 * (get_sigma_normal.f90:68 with g0and_bath_real), the same layout (Lreal). */
int dmfted_get_g0imp_real(dmfted_ctx *ctx, double *g);
/* ed_dens, ed_dens_up, ed_dens_dw, ed_docc (Norb each), ed_magz (Norb). */
int dmfted_get_observables(dmfted_ctx *ctx, double *dens, double *dens_up, double *dens_dw,
                           double *docc, double *magz);
/* The kept eigenspace: energies, 1-based sectors (state_list order,
 * ED_EIGENSPACE.f90:157-213), count, partition function Z. */
int dmfted_get_eigenspace(dmfted_ctx *ctx, int32_t cap, double *energies, int32_t *sectors,
                          int32_t *nstates, double *zeta);
/* Local energies of the last solve (local_energy_impurity,
 * ED_OBSERVABLES.f90:454-635): ed_get_eimp (ED_IO/get_eimp.f90:1-4),
 * eimp[4] = {Epot, Eint, Ehartree, Eknot}, and ed_get_doubles
 * (ED_IO/get_doubles.f90:1-4), doubles[4] = {Dust, Dund, Dse, Dph}.  As in the
 * reference: Epot includes Ehartree; Eint is never assigned there and is 0;
 * the inter-orbital Hloc hopping part of Eknot and the spin-exchange /
 * pair-hopping parts (Dse, Dph and their Jx, Jp terms in Epot, with Jhflag)
 * are summed over the kept states without the Boltzmann weight. */
int dmfted_get_eimp(dmfted_ctx *ctx, double *eimp);
int dmfted_get_doubles(dmfted_ctx *ctx, double *doubles);

/* Ground-state energy of the last solve. */
int dmfted_get_egs(dmfted_ctx *ctx, double *egs);

/* The eigenspace sizes that ed_diag/ed_analysis adapt from one solve to the
 * next: neigen_sector(1:Nsectors) and lanc_nstates_total
 * (ED_DIAG.f90:248-398).  The lattice solve keeps one copy per inequivalent
 * site and swaps it in and out of the single impurity context, as
 * ed_solve_lattice does with neigen_sectorii / neigen_totalii
 * (ED_MAIN.f90:419-423,597-611,655-656).  nsectors must equal the context's
 * sector count ((Ns+1)^2); set rejects non-positive entries. */
int dmfted_get_neigen(dmfted_ctx *ctx, int32_t *neigen, int32_t nsectors, int32_t *nstates_total);
int dmfted_set_neigen(dmfted_ctx *ctx, const int32_t *neigen, int32_t nsectors,
                      int32_t nstates_total);

/* ---- gradients -----------------------------------------------------------
 * Hellmann-Feynman gradient of the thermal energy of the last solve with
 * respect to the user bath array (same layout and length as the bath):
 *   dE/de(s,a,k) = <n_{k,s}>,  dE/dV(s,a,k) = <c+_{a s} c_{k s} + h.c.>
 * as reductions over the kept eigenvectors on the device.  For Nspin=1 the
 * two physical spins share one parameter and their terms add. */
int dmfted_hf_gradient(dmfted_ctx *ctx, double *grad, int32_t nb);

/* Batched chi^2 of the Delta fit and its gradient, the functions
 * chi2_delta_normal_normal and grad_chi2_delta_normal_normal of
 * ED_CHI2FIT/fitgf_normal_normal.f90:193-226,256-316 (the fit's gradient
 * routine, in place of grad_delta_bath), for nbatch parameter sets
 * a[b*2*nbath + j] = [e_1..e_Nbath, V_1..V_Nbath].  xdelta[L] = wm,
 * g[L] complex128 target, w[L] weights.  chi2[nbatch], grad[nbatch*2*nbath]
 * (grad may be NULL).  Host pointers; the work runs on the device of ctx. */
int dmfted_chi2_delta_batch(dmfted_ctx *ctx, int32_t nbatch, int32_t nbath, int32_t L,
                            const double *a, const double *xdelta, const double *g,
                            const double *w, double *chi2, double *grad);

/* Same on device pointers, on the context's stream (no host copies). */
int dmfted_chi2_delta_batch_device(dmfted_ctx *ctx, int32_t nbatch, int32_t nbath, int32_t L,
                                   const double *d_a, const double *d_xdelta, const double *d_g,
                                   const double *d_w, double *d_chi2, double *d_grad);

/* ---- the self-consistency around the solve --------------------------------
 * ed_chi2_fitgf (ED_CHI2FIT.f90:86-138) for the normal bath: for every
 * orbital a, the fit of the levels and hybridisations of spin ispin (1-based)
 * to fg(ispin,ispin,a,a,1:Ldelta), Ldelta = min(lfit, lmats), by
 * chi2_fitgf_normal_normal (ED_CHI2FIT/fitgf_normal_normal.f90:18-178): the
 * chi^2 of cg_scheme (delta or weiss) with the cg_weight weights, minimised by
 * the Polak-Ribiere conjugate gradient with Brent line searches (fmin_cg,
 * cg_niter, cg_ftol, cg_stop, cg_eps).  All orbitals run at once, one CTA
 * each.  fg: (Nspin,Nspin,Norb,Norb,Lmats) complex128, host; bath: the
 * set_dmft_bath layout, updated in place for spin ispin; iter[Norb] and
 * chi2[Norb] receive each fit's steps and final chi^2 (either may be NULL).
 * The solver's own bath is not changed (the next ed_solve passes it). */
int dmfted_chi2_fitgf(dmfted_ctx *ctx, const double *fg, int32_t ispin, double *bath,
                      int32_t nb, int32_t *iter, double *chi2);

/* The same minimiser on nbatch independent parameter sets at once (one CTA
 * each), all fitting one target: a[nbatch*2*nbath] start values in, minima
 * out ([e_1..e_Nbath, V_1..V_Nbath] per set); xdelta[L], g[L] complex128,
 * w[L] as dmfted_chi2_delta_batch; scheme DMFTED_CG_DELTA or
 * DMFTED_CG_WEISS with zc = xmu - Hloc_aa; the stopping controls are the
 * context's cg_* parameters.  iter[nbatch], chi2[nbatch] (may be NULL).
 * Host pointers. */
int dmfted_cg_fit_batch(dmfted_ctx *ctx, int32_t nbatch, int32_t nbath, int32_t L, double *a,
                        const double *xdelta, const double *g, const double *w, int32_t scheme,
                        double zc, int32_t *iter, double *chi2);

/* Same on device pointers, on the context's stream.  d_status[nbatch]:
 * bit 0 a line search found no bracket, bit 1 a Brent search hit its step
 * limit (the fit still returns its best point). */
int dmfted_cg_fit_batch_device(dmfted_ctx *ctx, int32_t nbatch, int32_t nbath, int32_t L,
                               double *d_a, const double *d_xdelta, const double *d_g,
                               const double *d_w, int32_t scheme, double zc, int32_t *d_iter,
                               double *d_chi2, int32_t *d_status);

/* dmft_gloc_matsubara of DMFT_Tools (drivers/ed_hm_bethe.f90:70; the legacy
 * in-tree .repo/ED_GLOC.f90:54-126,257-298) for a lattice Hamiltonian diagonal
 * in spin and orbital, on a density-of-states grid of le points:
 *   G_loc(s,s,a,a,iw_n) = sum_k wt[k] / (iw_n + xmu - Sigma(s,s,a,a,iw_n) - he[a*le+k])
 * sigma, gloc: (Nspin,Nspin,Norb,Norb,Lmats) complex128, host (off-diagonal
 * entries of gloc are zero).  For the Bethe lattice of half-bandwidth D:
 * he = linspace(-D, D, le), wt = 2 sqrt(D^2 - he^2) / (pi D^2) * de. */
int dmfted_gloc_matsubara_diag(dmfted_ctx *ctx, int32_t le, const double *he, const double *wt,
                               const double *sigma, double *gloc);

/* dmft_gloc_realaxis (drivers/ed_hm_bethe.f90:91) on the same grid: the sum
 * with w + i eps in place of i w_n, over the Lreal points linspace(wini, wfin)
 * of the context; sigma, gloc (Nspin,Nspin,Norb,Norb,Lreal) complex128. */
int dmfted_gloc_realaxis_diag(dmfted_ctx *ctx, int32_t le, const double *he, const double *wt,
                              const double *sigma, double *gloc);

/* dmft_weiss / dmft_delta (drivers/ed_hm_bethe.f90:73-77; .repo/ED_WEISS.f90:
 * 55-118) on the diagonal: scheme DMFTED_CG_WEISS gives 1/(1/G_loc + Sigma),
 * DMFTED_CG_DELTA gives iw_n + xmu - Hloc_aa - Sigma - 1/G_loc.  Same array
 * layout as dmfted_gloc_matsubara_diag; host pointers. */
int dmfted_get_weiss(dmfted_ctx *ctx, const double *gloc, const double *sigma, int32_t scheme,
                     double *out);

/* ---- files that let a run resume across the boundary (text formats) ---------
 * save_dmft_bath (ED_BATH/dmft_aux.f90:408-428 with write_dmft_bath :310-336,
 * normal bath): the bath array written as hamiltonian.restart / .used are,
 * a header of "(90(A21,1X))" labels then Nbath rows of "(90(F21.12,1X))"
 * values ((e(s,a,k), v(s,a,k), a=1..Norb), s=1..Nspin).  No device needed. */
int dmfted_save_bath(const dmfted_params *p, const char *path, const double *bath, int32_t nb);

/* The bath read of init_dmft_bath (ED_BATH/dmft_aux.f90:158-180): the header
 * skipped, then min(lines, Nbath) rows read list-directed into bath (the
 * set_dmft_bath layout).  The line count includes the header, so a file with
 * fewer than Nbath rows runs the read past its end: an error, as in the
 * reference.  No device needed. */
int dmfted_read_bath(const dmfted_params *p, const char *path, double *bath, int32_t nb);

/* print_state_list (ED_DIAG.f90:258-264,401-445): the eigenspace of the last
 * solve in the state_list.ed format, one "(i3,f18.12,2x,ES19.12,1x,2i3,3x,i3,
 * i10)" row per state (i, E_i, exp(-beta(E_i-E_min)), nup, ndw, sector, dim). */
int dmfted_print_state_list(dmfted_ctx *ctx, const char *path);

/* The state_list.restart read of setup_pointers_normal (ED_SETUP.f90:403-425):
 * lanc_nstates_total = the file's line count, neigen_sector(s) = max(1, states
 * listed in sector s), each row's nup/ndw checked against its sector (the
 * reference's stop message otherwise).  Call after dmfted_init, before the
 * first solve. */
int dmfted_read_state_list(dmfted_ctx *ctx, const char *path);

/* ---- printed outputs (ED_IO, ED_OBSERVABLES) --------------------------------
 * dir: the directory the files are written to or read from (NULL or "": the
 * working directory, as the reference); suffix: ed_file_suffix (ED_MAIN.f90:
 * 185,193,214), "" or NULL for one impurity.  All need a solve on ctx except
 * dmfted_read_impsigma.  The reference calls print_impSigma and print_impG at
 * the end of buildgf_impurity when ed_print_Sigma / ed_print_G are set
 * (ED_GREENS_FUNCTIONS.f90:161-165), write_observables at the end of
 * observables_impurity (ED_OBSERVABLES.f90:418-420) and write_energy at the
 * end of local_energy_impurity (:681-684). */

/* print_impG_normal (ED_IO/print_impG.f90:38-46): per spin s and orbital a,
 * impG_l<a><a>_s<s>_iw<suffix>.ed (Lmats lines) and impG_l<a><a>_s<s>_realw
 * <suffix>.ed (Lreal lines), each line the abscissa, Im G, Re G: the columns
 * of SciFortran's splot (not in the tree, version unpinned), written here in
 * ES24.16 so that a read gives back the same doubles. */
int dmfted_print_impg(dmfted_ctx *ctx, const char *dir, const char *suffix);
/* print_impSigma_normal (ED_IO/print_impSigma.f90:37-45): the same for the
 * self-energy, impSigma_l<a><a>_s<s>_iw / _realw<suffix>.ed. */
int dmfted_print_impsigma(dmfted_ctx *ctx, const char *dir, const char *suffix);
/* print_impG0_normal (ED_IO/print_impG0.f90:37-45): the Weiss field G0and,
 * written under the impG_... names as the reference does (so it replaces the
 * files of dmfted_print_impg). */
int dmfted_print_impg0(dmfted_ctx *ctx, const char *dir, const char *suffix);
/* read_impSigma_normal (ED_IO/read_impSigma.f90:38-46): the impSigma files
 * read back (three numbers per line, list-directed; Lmats and Lreal lines)
 * into the context's self-energies, which dmfted_get_sigma_* then return and
 * the next solve's scattering rate and Z in observables_all.ed use.  Every
 * file is read before anything changes; a missing or short file is
 * DMFTED_ERR_ARG. */
int dmfted_read_impsigma(dmfted_ctx *ctx, const char *dir, const char *suffix);
/* write_observables (ED_OBSERVABLES.f90:780-849), normal mode: one
 * "(90(F15.9,1X))" record dens(a), docc(a), dens_up(a), dens_dw(a), magz(a),
 * s2tot, egs, sz2(a,b), n2(a,b), zimp(a,s), simp(a,s) appended to
 * observables_all<suffix>.ed and written to observables_last<suffix>.ed, and
 * parameters_last<suffix>.ed ("(90F15.9)": xmu, beta, Uloc(a), Ust, Jh, Jx,
 * Jp).  zimp and simp are get_szr (:695-708) of the self-energy the solve's
 * observables saw: the reference takes them before the same solve's Green's
 * functions, i.e. from the previous solve (or a read self-energy), 0 before
 * the first.  legend != 0 also writes observables_info.ed and
 * parameters_info.ed (write_legend, :715-758), which the reference does on
 * its first call. */
int dmfted_write_observables(dmfted_ctx *ctx, const char *dir, const char *suffix,
                             int32_t legend);
/* write_energy_info and write_energy (ED_OBSERVABLES.f90:760-774,851-857):
 * energy_info.ed and energy_last<suffix>.ed ("(90F15.9)": Epot,
 * Epot-Ehartree, Eknot, Ehartree, Dust, Dund, Dse, Dph). */
int dmfted_write_energy(dmfted_ctx *ctx, const char *dir, const char *suffix);

/* ---- timing helpers (device time on the context's stream) ------------ */
/* Average device milliseconds of one H*v on the current sector over reps
 * launches after warmup launches.  flags: bit 0 = float32 vectors (else
 * float64), bit 1 = the fused Lanczos-step variant (H*v - b v_prev and the
 * alpha dot product) instead of the plain product, bit 2 = the vector order
 * used by Green's-function chains (down rank fastest when DimUp is odd and
 * DimDw even), bit 3 = the whole Lanczos step as the solver runs it (the
 * fused product, then w = u - a x and |w|).
 * The vectors are the context's own work buffers. */
int dmfted_time_hxv(dmfted_ctx *ctx, int32_t flags, int32_t warmup, int32_t reps, double *ms);

/* Live timing of the H*v launches (plain products and fused Lanczos steps)
 * of everything that runs on the context from now on: on != 0 records a CUDA
 * event pair on the context's stream around each launch.  Resets the totals.
 * No counterpart in the reference (measurement support). */
int dmfted_hxv_timing(dmfted_ctx *ctx, int32_t on);

/* The autotuner's measurements so far, one line per job-shape key of a
 * batched phase: the key, the device time of each candidate cluster size and
 * the size kept.  Written into buf (NUL-terminated, truncated to len bytes);
 * *needed (may be NULL) receives the full length + 1.  No counterpart in the
 * reference (measurement support). */
int dmfted_autotune_log(dmfted_ctx *ctx, char *buf, int32_t len, int32_t *needed);

/* Totals of the timed H*v launches since the last call (then reset): device
 * milliseconds, launch count and algorithmic bytes (read x, read v_prev for
 * the fused step, write y, at the vector precision).  Waits for the stream. */
int dmfted_get_hxv_timing(dmfted_ctx *ctx, double *ms, int64_t *launches, double *bytes);

/* Device milliseconds of the last dmfted_ed_solve, split into phases:
 * t[0]=diagonalisation, t[1]=observables, t[2]=Green's functions,
 * t[3]=total; and the H*v products each phase used in n[0..2]. */
int dmfted_get_timings(dmfted_ctx *ctx, double *t, int64_t *n);

/* Number of kernel launches the library issued since the counter was last
 * reset (*count), then reset it if reset != 0. */
int dmfted_launch_count(dmfted_ctx *ctx, int64_t *count, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif
