/*
 * ed_oracle.c -- CPU restatement of the dmft-ed exact-diagonalization hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * dmft-ed_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.  The product never links
 * or calls it.
 *
 * Parity status: UNPINNED against reference outputs.  The reference is
 * Fortran with unvendored, unpinned SciFortran / DMFT_Tools dependencies and
 * ships no tests, golden vectors or output files, and no Fortran compiler is
 * available to run it.  The restatement is instead pinned against independent
 * known answers (dense eigensolvers, the U=0 and V=0 analytic limits, sum
 * rules); see tests/test_oracle.py.
 *
 * Every routine follows the reference line by line in semantics (loop order,
 * index conventions, accumulation order), cited as file:line relative to the
 * reference project root.  Index conventions: Fortran 1-based sector indices
 * and combined-map positions are kept where they cross the API (isector,
 * binary_search result); arrays are 0-based C arrays.
 *
 * Arithmetic is complex128 where the reference's is (H*v, Lanczos vectors),
 * real64 elsewhere.  The H*v can split its rows over pthreads (the reference
 * is serial per MPI rank; the threaded form exists for the timed CPU
 * baseline, which uses every host core).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

typedef double complex zc;

/* Model parameters for the normal-mode, normal-bath Hamiltonian.
 * e, v     : bath energies / hybridisations, index [(ispin*norb+iorb)*nbath+k]
 *            (the reference's dmft_bath%e(ispin,iorb,k), ED_VARS_GLOBAL.f90:8-18)
 * hloc     : impHloc(Nspin,Nspin,Norb,Norb) in Fortran column-major order,
 *            complex128 as re/im pairs.                                      */
typedef struct {
    int32_t norb, nbath, nspin, ns;
    int32_t hfmode, jhflag;
    double uloc[3];
    double ust, jh, jx, jp, xmu, beta;
    const double *e;
    const double *v;
    const double *hloc; /* 2*Nspin*Nspin*Norb*Norb doubles */
} or_model;

static inline zc hloc_at(const or_model *M, int is, int js, int a, int b) {
    int ns = M->nspin, no = M->norb;
    long idx = is + ns * (js + ns * (a + (long)no * b));
    return M->hloc[2 * idx] + I * M->hloc[2 * idx + 1];
}
static inline double bath_e(const or_model *M, int is, int a, int k) {
    return M->e[((long)is * M->norb + a) * M->nbath + k];
}
static inline double bath_v(const or_model *M, int is, int a, int k) {
    return M->v[((long)is * M->norb + a) * M->nbath + k];
}

/* binomial: ED_SETUP.f90:1258-1275 (FP64 running product, int(x+0.5)). */
int32_t or_binomial(int32_t n1, int32_t n2) {
    double xh = 1.0;
    if (n2 < 0) return 0;
    if (n2 == 0) return 1;
    for (int i = 1; i <= n2; i++) xh = xh * (double)(n1 + 1 - i) / (double)i;
    return (int32_t)(xh + 0.5);
}

/* get_normal_sector_dimension: ED_SETUP.f90:793-805. */
int64_t or_sector_dim(int32_t ns, int32_t nup, int32_t ndw) {
    return (int64_t)or_binomial(ns, nup) * (int64_t)or_binomial(ns, ndw);
}

/* Sector tables of setup_pointers_normal, ED_SETUP.f90:379-493 (normal
 * ed_mode, normal bath).  All outputs 1-based as in the reference:
 *   getsector[(nup)*(ns+1)+ndw] ; getnup/getndw/getdim/getdimup/getdimdw[isector-1]
 *   getcsector[(isector-1)*2 + ispin-1], getcdgsector likewise (0 = none)
 *   getbathstride[(k-1)*norb + iorb-1] = Norb+(iorb-1)*Nbath+k   (:445-462)
 *   impindex[(ispin-1)*norb + iorb-1] = iorb + (ispin-1)*Ns      (:440-443)   */
void or_setup_pointers_normal(int32_t norb, int32_t nbath, int32_t *getsector,
                              int32_t *getnup, int32_t *getndw, int32_t *getdim,
                              int32_t *getdimup, int32_t *getdimdw,
                              int32_t *getcsector, int32_t *getcdgsector,
                              int32_t *getbathstride, int32_t *impindex) {
    int32_t ns = (nbath + 1) * norb;
    int32_t nsect = (ns + 1) * (ns + 1);
    int32_t isector = 0;
    for (int nup = 0; nup <= ns; nup++)
        for (int ndw = 0; ndw <= ns; ndw++) {
            isector++;
            getsector[nup * (ns + 1) + ndw] = isector;
            getnup[isector - 1] = nup;
            getndw[isector - 1] = ndw;
            getdim[isector - 1] = or_binomial(ns, nup) * or_binomial(ns, ndw);
            getdimup[isector - 1] = or_binomial(ns, nup);
            getdimdw[isector - 1] = or_binomial(ns, ndw);
        }
    for (int in = 1; in <= norb; in++) {
        impindex[in - 1] = in;
        impindex[norb + in - 1] = in + ns;
    }
    for (int i = 1; i <= nbath; i++)
        for (int iorb = 1; iorb <= norb; iorb++)
            getbathstride[(i - 1) * norb + iorb - 1] = norb + (iorb - 1) * nbath + i;
    for (int s = 0; s < nsect; s++) {
        getcsector[2 * s] = getcsector[2 * s + 1] = 0;
        getcdgsector[2 * s] = getcdgsector[2 * s + 1] = 0;
    }
    for (int s = 1; s <= nsect; s++) {
        int nup = getnup[s - 1], ndw = getndw[s - 1];
        if (nup - 1 >= 0) getcsector[2 * (s - 1) + 0] = getsector[(nup - 1) * (ns + 1) + ndw];
        if (ndw - 1 >= 0) getcsector[2 * (s - 1) + 1] = getsector[nup * (ns + 1) + ndw - 1];
        if (nup + 1 <= ns) getcdgsector[2 * (s - 1) + 0] = getsector[(nup + 1) * (ns + 1) + ndw];
        if (ndw + 1 <= ns) getcdgsector[2 * (s - 1) + 1] = getsector[nup * (ns + 1) + ndw + 1];
    }
}

/* bdecomp-based popcount of the low ntot bits (ED_SETUP.f90:1209-1219). */
static inline int bsum(int64_t i, int ntot) {
    int s = 0;
    for (int l = 0; l < ntot; l++) s += (int)((i >> l) & 1);
    return s;
}

/* build_sector, normal case: ED_SETUP.f90:874-891.  idw outer, iup inner,
 * both over 0..2^Ns-1, keep popcount matches, map(dim) = iup + idw*2^Ns.
 * Returns dim. */
int64_t or_build_sector(int32_t ns, int32_t nup, int32_t ndw, int32_t *map) {
    int64_t dim = 0;
    int64_t two_ns = (int64_t)1 << ns;
    for (int64_t idw = 0; idw < two_ns; idw++) {
        if (bsum(idw, ns) != ndw) continue;
        for (int64_t iup = 0; iup < two_ns; iup++) {
            if (bsum(iup, ns) != nup) continue;
            map[dim++] = (int32_t)(iup + idw * two_ns);
        }
    }
    return dim;
}

/* binary_search: ED_SETUP.f90:1282-1299.  Recursive bisection with
 * mid = size/2+1 (1-based); returns the 1-based position or 0. */
static int64_t bsearch_rec(const int32_t *a, int64_t n, int32_t value) {
    if (n == 0) return 0;
    int64_t mid = n / 2 + 1;
    if (a[mid - 1] > value) return bsearch_rec(a, mid - 1, value);
    if (a[mid - 1] < value) {
        int64_t r = bsearch_rec(a + mid, n - mid, value);
        return r != 0 ? mid + r : 0;
    }
    return mid;
}
int64_t or_binary_search(const int32_t *a, int64_t n, int32_t value) {
    return bsearch_rec(a, n, value);
}

/* c / cdg: ED_SETUP.f90:1055-1081.  pos is 1-based; the sign is
 * (-1)^(number of occupied levels below pos).  Return 0 on the reference's
 * stop condition ("C error: C_i|...0_i...>"), 1 otherwise. */
static inline int op_c(int pos, int32_t in, int32_t *out, double *fsgn) {
    if (!((in >> (pos - 1)) & 1)) return 0;
    double s = 1.0;
    for (int l = 1; l <= pos - 1; l++)
        if ((in >> (l - 1)) & 1) s = -s;
    *fsgn = s;
    *out = in & ~((int32_t)1 << (pos - 1));
    return 1;
}
static inline int op_cdg(int pos, int32_t in, int32_t *out, double *fsgn) {
    if ((in >> (pos - 1)) & 1) return 0;
    double s = 1.0;
    for (int l = 1; l <= pos - 1; l++)
        if ((in >> (l - 1)) & 1) s = -s;
    *fsgn = s;
    *out = in | ((int32_t)1 << (pos - 1));
    return 1;
}
int32_t or_c(int32_t pos, int32_t in, int32_t *out, double *sgn) { return op_c(pos, in, out, sgn); }
int32_t or_cdg(int32_t pos, int32_t in, int32_t *out, double *sgn) { return op_cdg(pos, in, out, sgn); }

#define IB(m, l) ((int)(((m) >> ((l) - 1)) & 1)) /* ib(l), 1-based level l */

/* Element emitter shared by the on-the-fly H*v and the explicit builder.
 * For row i (state m) every (column j, value) the reference's loop body in
 * build_hxv.f90:1-27 visits, in the same order:
 *   HxVimp.f90:1-76  (diag -xmu*n + Hloc_aa*n, same-spin Hloc hopping)
 *   HxVint.f90:1-97  (U, Ust, Ust-Jh, HFMODE shift, Jhflag S-E / P-H)
 *   HxVbath.f90:1-13 (sum_k e_k n_k, normal bath)
 *   HxVimp_bath.f90:1-38 (V_k imp<->bath hopping, both directions, per spin)
 * emit(ctx, j, val) with j the 1-based column (0 = not found). */
typedef void (*emit_fn)(void *ctx, int64_t j, zc val);

static void row_elements(const or_model *M, const int32_t *map, int64_t dim, int64_t i,
                         emit_fn emit, void *ctx) {
    const int Ns = M->ns, Norb = M->norb, Nbath = M->nbath, Nspin = M->nspin;
    int32_t m = map[i];
    double nup[3], ndw[3];
    for (int a = 1; a <= Norb; a++) {
        nup[a - 1] = (double)IB(m, a);
        ndw[a - 1] = (double)IB(m, a + Ns);
    }
    int32_t k1 = 0, k2 = 0, k3 = 0, k4 = 0;
    double sg1 = 1.0, sg2 = 1.0, sg3 = 1.0, sg4 = 1.0;
    zc htmp;
    /* HxVimp.f90:1-12: diagonal local part */
    double sn = 0.0;
    for (int a = 0; a < Norb; a++) sn += nup[a];
    double sd = 0.0;
    for (int a = 0; a < Norb; a++) sd += ndw[a];
    htmp = 0.0;
    htmp = htmp - M->xmu * (sn + sd);
    for (int a = 1; a <= Norb; a++) {
        htmp = htmp + hloc_at(M, 0, 0, a - 1, a - 1) * nup[a - 1];
        htmp = htmp + hloc_at(M, Nspin - 1, Nspin - 1, a - 1, a - 1) * ndw[a - 1];
    }
    emit(ctx, i + 1, htmp);
    /* HxVimp.f90:16-49: same-spin orbital off-diagonal Hloc */
    for (int a = 1; a <= Norb; a++)
        for (int b = 1; b <= Norb; b++) {
            zc h = hloc_at(M, 0, 0, a - 1, b - 1);
            if (h != 0.0 && IB(m, b) == 1 && IB(m, a) == 0) {
                op_c(b, m, &k1, &sg1);
                op_cdg(a, k1, &k2, &sg2);
                int64_t j = or_binary_search(map, dim, k2);
                emit(ctx, j, h * sg1 * sg2);
            }
            h = hloc_at(M, Nspin - 1, Nspin - 1, a - 1, b - 1);
            if (h != 0.0 && IB(m, b + Ns) == 1 && IB(m, a + Ns) == 0) {
                op_c(b + Ns, m, &k1, &sg1);
                op_cdg(a + Ns, k1, &k2, &sg2);
                int64_t j = or_binary_search(map, dim, k2);
                emit(ctx, j, h * sg1 * sg2);
            }
        }
    /* HxVint.f90:1-43: density-density interaction and Hartree shift */
    htmp = 0.0;
    for (int a = 0; a < Norb; a++) htmp = htmp + M->uloc[a] * nup[a] * ndw[a];
    if (Norb > 1) {
        for (int a = 0; a < Norb; a++)
            for (int b = a + 1; b < Norb; b++)
                htmp = htmp + M->ust * (nup[a] * ndw[b] + nup[b] * ndw[a]);
        for (int a = 0; a < Norb; a++)
            for (int b = a + 1; b < Norb; b++)
                htmp = htmp + (M->ust - M->jh) * (nup[a] * nup[b] + ndw[a] * ndw[b]);
    }
    if (M->hfmode) {
        for (int a = 0; a < Norb; a++)
            htmp = htmp - 0.5 * M->uloc[a] * (nup[a] + ndw[a]) + 0.25 * M->uloc[a];
        if (Norb > 1)
            for (int a = 0; a < Norb; a++)
                for (int b = a + 1; b < Norb; b++) {
                    htmp = htmp - 0.5 * M->ust * (nup[a] + ndw[a] + nup[b] + ndw[b]) + 0.25 * M->ust;
                    htmp = htmp - 0.5 * (M->ust - M->jh) * (nup[a] + ndw[a] + nup[b] + ndw[b]) +
                           0.25 * (M->ust - M->jh);
                }
    }
    emit(ctx, i + 1, htmp);
    /* HxVint.f90:45-97: spin-exchange and pair-hopping (Jhflag, Norb>1) */
    if (Norb > 1 && M->jhflag) {
        for (int a = 1; a <= Norb; a++)
            for (int b = 1; b <= Norb; b++) {
                if (a != b && IB(m, b) == 1 && IB(m, a + Ns) == 1 && IB(m, b + Ns) == 0 &&
                    IB(m, a) == 0) {
                    op_c(b, m, &k1, &sg1);
                    op_c(a + Ns, k1, &k2, &sg2);
                    op_cdg(b + Ns, k2, &k3, &sg3);
                    op_cdg(a, k3, &k4, &sg4);
                    int64_t j = or_binary_search(map, dim, k4);
                    if (j != 0) emit(ctx, j, M->jx * sg1 * sg2 * sg3 * sg4);
                }
            }
        for (int a = 1; a <= Norb; a++)
            for (int b = 1; b <= Norb; b++) {
                if (a != b && IB(m, b) == 1 && IB(m, b + Ns) == 1 && IB(m, a + Ns) == 0 &&
                    IB(m, a) == 0) {
                    op_c(b, m, &k1, &sg1);
                    op_c(b + Ns, k1, &k2, &sg2);
                    op_cdg(a + Ns, k2, &k3, &sg3);
                    op_cdg(a, k3, &k4, &sg4);
                    int64_t j = or_binary_search(map, dim, k4);
                    if (j != 0) emit(ctx, j, M->jp * sg1 * sg2 * sg3 * sg4);
                }
            }
    }
    /* HxVbath.f90:1-13: bath energies, getBathStride = Norb+(iorb-1)*Nbath+kp */
    htmp = 0.0;
    for (int a = 1; a <= Norb; a++)
        for (int kp = 1; kp <= Nbath; kp++) {
            int alfa = Norb + (a - 1) * Nbath + kp;
            htmp = htmp + bath_e(M, 0, a - 1, kp - 1) * IB(m, alfa);
            htmp = htmp + bath_e(M, Nspin - 1, a - 1, kp - 1) * IB(m, alfa + Ns);
        }
    emit(ctx, i + 1, htmp);
    /* HxVimp_bath.f90:1-38: imp <-> bath hopping, spin conserving */
    for (int a = 1; a <= Norb; a++)
        for (int kp = 1; kp <= Nbath; kp++) {
            int ms = Norb + (a - 1) * Nbath + kp;
            double vu = bath_v(M, 0, a - 1, kp - 1), vd = bath_v(M, Nspin - 1, a - 1, kp - 1);
            if (vu != 0.0 && IB(m, a) == 1 && IB(m, ms) == 0) {
                op_c(a, m, &k1, &sg1);
                op_cdg(ms, k1, &k2, &sg2);
                emit(ctx, or_binary_search(map, dim, k2), vu * sg1 * sg2);
            }
            if (vu != 0.0 && IB(m, a) == 0 && IB(m, ms) == 1) {
                op_c(ms, m, &k1, &sg1);
                op_cdg(a, k1, &k2, &sg2);
                emit(ctx, or_binary_search(map, dim, k2), vu * sg1 * sg2);
            }
            if (vd != 0.0 && IB(m, a + Ns) == 1 && IB(m, ms + Ns) == 0) {
                op_c(a + Ns, m, &k1, &sg1);
                op_cdg(ms + Ns, k1, &k2, &sg2);
                emit(ctx, or_binary_search(map, dim, k2), vd * sg1 * sg2);
            }
            if (vd != 0.0 && IB(m, a + Ns) == 0 && IB(m, ms + Ns) == 1) {
                op_c(ms + Ns, m, &k1, &sg1);
                op_cdg(a + Ns, k1, &k2, &sg2);
                emit(ctx, or_binary_search(map, dim, k2), vd * sg1 * sg2);
            }
        }
}

typedef struct {
    const zc *vin;
    zc acc;
} hxv_ctx;
static void emit_hxv(void *c, int64_t j, zc val) {
    hxv_ctx *h = (hxv_ctx *)c;
    h->acc = h->acc + val * h->vin[j - 1];
}

/* directMatVec_cc: ED_HAMILTONIAN_MATVEC.f90:289-351 + build_hxv.f90.
 * hv(i) = sum over the row's elements of htmp*vin(j).  nthreads>1 splits the
 * row range into contiguous blocks, one pthread each (rows are independent). */
typedef struct {
    const or_model *M;
    const int32_t *map;
    int64_t dim, r0, r1;
    const zc *v;
    zc *out;
} hxv_job;

static void *hxv_worker(void *arg) {
    hxv_job *J = (hxv_job *)arg;
    for (int64_t i = J->r0; i < J->r1; i++) {
        hxv_ctx c = {J->v, 0.0};
        row_elements(J->M, J->map, J->dim, i, emit_hxv, &c);
        J->out[i] = c.acc;
    }
    return NULL;
}

void or_hxv_c128(const or_model *M, const int32_t *map, int64_t dim, const double *vin,
                 double *hv, int32_t nthreads) {
    const zc *v = (const zc *)vin;
    zc *out = (zc *)hv;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (nthreads == 1 || dim < 4096) {
        hxv_job J = {M, map, dim, 0, dim, v, out};
        hxv_worker(&J);
        return;
    }
    pthread_t th[256];
    hxv_job jobs[256];
    int64_t chunk = (dim + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        int64_t r0 = t * chunk, r1 = r0 + chunk < dim ? r0 + chunk : dim;
        if (r0 > dim) r0 = dim;
        jobs[t] = (hxv_job){M, map, dim, r0, r1, v, out};
        pthread_create(&th[t], NULL, hxv_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ */
/* The "best CPU" variant of the baseline: the up/down-factored H*v that the
 * device kernels use, restated on the CPU in FP64 (real: the normal-mode
 * Hamiltonian with a real bath and Hloc is real).  It separates the gain of
 * the factored algorithm from the gain of the hardware; it is not the
 * reference's algorithm.  On the DimUp x DimDw matrix V (the H%map order):
 *   (H V)[r,c] = D[r,c] V[r,c] + sum_{r'} Hup[r,r'] V[r',c] + sum_{c'} Hdw[c,c'] V[r,c'].
 * Hup and Hdw are read off the oracle's own element emitter (row_elements):
 * the off-diagonal elements of column 0 that keep the down word are Hup, the
 * elements of row 0 that keep the up word are Hdw (a one-spin hop's sign
 * depends on that spin's word only); D is the sum of the diagonal terms.
 * Models with the Jhflag terms (which change both words) are not factored. */
typedef struct {
    int64_t dimup, dimdw, wu, wd; /* ELL widths */
    int32_t *cu, *cd;             /* [dimup*wu], [dimdw*wd] target ranks, -1 = none */
    double *vu, *vd;
    double *diag;                 /* [dim] */
} or_factored;

typedef struct {
    int64_t base, stride, self, count, cap;
    int32_t *col;
    double *val;
    double dsum;
    int modeup;
    int64_t dimup;
} fac_ctx;
static void emit_fac(void *c, int64_t j, zc val) {
    fac_ctx *f = (fac_ctx *)c;
    if (j == 0) return;
    int64_t t = j - 1;
    if (t == f->self) {
        f->dsum += creal(val);
        return;
    }
    int64_t rank;
    if (f->modeup) {
        if (t >= f->dimup) return; /* changes the down word */
        rank = t;
    } else {
        if (t % f->dimup != 0) return; /* changes the up word */
        rank = t / f->dimup;
    }
    if (f->count < f->cap) {
        f->col[f->count] = (int32_t)rank;
        f->val[f->count] = creal(val);
        f->count++;
    }
}

/* Diagonal of every element: only the diagonal terms, emitted to a sum. */
typedef struct {
    const or_model *M;
    const int32_t *map;
    int64_t dim, r0, r1;
    double *diag;
} fac_diag_job;
static void *fac_diag_worker(void *arg) {
    fac_diag_job *J = (fac_diag_job *)arg;
    or_model M1 = *J->M;
    /* the diagonal alone: no hops can reach the row itself, so an emitter that
       keeps only the self terms, with the hoppings switched off, is exact */
    double zero_v[8 * 64] = {0};
    M1.v = zero_v;
    double hl[2 * 2 * 2 * 3 * 3];
    int nh = 2 * M1.nspin * M1.nspin * M1.norb * M1.norb;
    for (int q = 0; q < nh; q++) hl[q] = J->M->hloc[q];
    for (int is = 0; is < M1.nspin; is++)
        for (int js = 0; js < M1.nspin; js++)
            for (int a = 0; a < M1.norb; a++)
                for (int b = 0; b < M1.norb; b++)
                    if (a != b || is != js) {
                        long idx = is + M1.nspin * (js + M1.nspin * (a + (long)M1.norb * b));
                        hl[2 * idx] = hl[2 * idx + 1] = 0.0;
                    }
    M1.hloc = hl;
    M1.jhflag = 0;
    for (int64_t i = J->r0; i < J->r1; i++) {
        fac_ctx f = {0};
        f.self = i;
        f.dimup = 1;
        row_elements(&M1, J->map, J->dim, i, emit_fac, &f);
        J->diag[i] = f.dsum;
    }
    return NULL;
}

or_factored *or_factored_setup(const or_model *M, const int32_t *map, int64_t dimup,
                               int64_t dimdw, int32_t nthreads) {
    if (M->jhflag && M->norb > 1) return NULL;
    if (M->norb * M->nbath > 64) return NULL;
    const int64_t dim = dimup * dimdw;
    or_factored *F = (or_factored *)calloc(1, sizeof(or_factored));
    F->dimup = dimup;
    F->dimdw = dimdw;
    F->wu = F->wd = M->norb * (M->nbath + M->norb) + 1;
    F->cu = (int32_t *)malloc(sizeof(int32_t) * dimup * F->wu);
    F->vu = (double *)calloc((size_t)(dimup * F->wu), sizeof(double));
    F->cd = (int32_t *)malloc(sizeof(int32_t) * dimdw * F->wd);
    F->vd = (double *)calloc((size_t)(dimdw * F->wd), sizeof(double));
    for (int64_t q = 0; q < dimup * F->wu; q++) F->cu[q] = -1;
    for (int64_t q = 0; q < dimdw * F->wd; q++) F->cd[q] = -1;
    for (int64_t r = 0; r < dimup; r++) {
        fac_ctx f = {0};
        f.self = r;
        f.cap = F->wu;
        f.col = F->cu + r * F->wu;
        f.val = F->vu + r * F->wu;
        f.modeup = 1;
        f.dimup = dimup;
        row_elements(M, map, dim, r, emit_fac, &f);
    }
    for (int64_t c = 0; c < dimdw; c++) {
        fac_ctx f = {0};
        f.self = c * dimup;
        f.cap = F->wd;
        f.col = F->cd + c * F->wd;
        f.val = F->vd + c * F->wd;
        f.modeup = 0;
        f.dimup = dimup;
        row_elements(M, map, dim, c * dimup, emit_fac, &f);
    }
    F->diag = (double *)malloc(sizeof(double) * dim);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    fac_diag_job jobs[256];
    int64_t chunk = (dim + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        int64_t r0 = t * chunk < dim ? t * chunk : dim;
        int64_t r1 = r0 + chunk < dim ? r0 + chunk : dim;
        jobs[t] = (fac_diag_job){M, map, dim, r0, r1, F->diag};
        pthread_create(&th[t], NULL, fac_diag_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return F;
}

void or_factored_free(or_factored *F) {
    if (!F) return;
    free(F->cu);
    free(F->vu);
    free(F->cd);
    free(F->vd);
    free(F->diag);
    free(F);
}

typedef struct {
    const or_factored *F;
    const double *x;
    double *y;
    int64_t c0, c1;
} fac_job;
static void *fac_worker(void *arg) {
    fac_job *J = (fac_job *)arg;
    const or_factored *F = J->F;
    const int64_t du = F->dimup;
    for (int64_t c = J->c0; c < J->c1; c++) {
        const double *xc = J->x + c * du;
        double *yc = J->y + c * du;
        for (int64_t r = 0; r < du; r++) yc[r] = F->diag[c * du + r] * xc[r];
        for (int64_t r = 0; r < du; r++) {
            double acc = 0.0;
            const int32_t *cl = F->cu + r * F->wu;
            const double *vl = F->vu + r * F->wu;
            for (int64_t e = 0; e < F->wu && cl[e] >= 0; e++) acc += vl[e] * xc[cl[e]];
            yc[r] += acc;
        }
        const int32_t *cl = F->cd + c * F->wd;
        const double *vl = F->vd + c * F->wd;
        for (int64_t e = 0; e < F->wd && cl[e] >= 0; e++) {
            const double v = vl[e];
            const double *xn = J->x + (int64_t)cl[e] * du;
            for (int64_t r = 0; r < du; r++) yc[r] += v * xn[r];
        }
    }
    return NULL;
}

void or_factored_hxv(const or_factored *F, const double *x, double *y, int32_t nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    fac_job jobs[256];
    int64_t chunk = (F->dimdw + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        int64_t c0 = t * chunk < F->dimdw ? t * chunk : F->dimdw;
        int64_t c1 = c0 + chunk < F->dimdw ? c0 + chunk : F->dimdw;
        jobs[t] = (fac_job){F, x, y, c0, c1};
        pthread_create(&th[t], NULL, fac_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
}

typedef struct {
    int64_t row;
    int64_t n, cap;
    int64_t *ri, *ci;
    double *re, *im;
} coo_ctx;
static void emit_coo(void *c, int64_t j, zc val) {
    coo_ctx *h = (coo_ctx *)c;
    if (j == 0 || h->n >= h->cap) return;
    h->ri[h->n] = h->row;
    h->ci[h->n] = j - 1;
    h->re[h->n] = creal(val);
    h->im[h->n] = cimag(val);
    h->n++;
}

/* The explicit sector Hamiltonian as COO triplets (row, col, value), the
 * element set ed_buildH_c inserts (ED_HAMILTONIAN_MATVEC.f90:123-198 with
 * build_h.f90, same bodies as the H*v).  Returns the number of triplets
 * written (duplicates are summed by the caller). */
int64_t or_build_coo(const or_model *M, const int32_t *map, int64_t dim, int64_t cap,
                     int64_t *ri, int64_t *ci, double *re, double *im) {
    coo_ctx c = {0, 0, cap, ri, ci, re, im};
    for (int64_t i = 0; i < dim; i++) {
        c.row = i;
        row_elements(M, map, dim, i, emit_coo, &c);
    }
    return c.n;
}

/* ------------------------------------------------------------------ */
/* Plain Lanczos: .repo/PLAIN_LANCZOS.f90:87-118 (lanczos_plain_iteration_c)
 * and :154-180 (lanczos_plain_tridiag_c), the algorithm of SciFortran's
 * sp_lanc_tridiag.  vin is normalised on the first iteration; each step:
 *   tmp = H vin - b vout ; a = <vin,tmp> ; tmp -= a vin ; b = |tmp| ;
 *   vout = vin ; vin = tmp/b
 * alanc(iter) = a, blanc(iter+1) = b (blanc(1) = 0), stop when |b|<threshold.
 * Returns the number of iterations performed. */
typedef struct {
    const or_model *M;
    const int32_t *map;
    int64_t dim;
    int nthreads;
} or_op;

static zc zdot(const zc *a, const zc *b, int64_t n) { /* Fortran dot_product: conj(a).b */
    zc s = 0.0;
    for (int64_t i = 0; i < n; i++) s += conj(a[i]) * b[i];
    return s;
}

static void lanczos_iteration(const or_op *op, int iter, zc *vin, zc *vout, zc *tmp, double *a,
                              double *b) {
    int64_t n = op->dim;
    if (iter == 1) {
        double norm = sqrt(creal(zdot(vin, vin, n)));
        for (int64_t i = 0; i < n; i++) vin[i] /= norm;
        *b = 0.0;
    }
    or_hxv_c128(op->M, op->map, n, (const double *)vin, (double *)tmp, op->nthreads);
    for (int64_t i = 0; i < n; i++) tmp[i] = tmp[i] - (*b) * vout[i];
    *a = creal(zdot(vin, tmp, n));
    for (int64_t i = 0; i < n; i++) tmp[i] = tmp[i] - (*a) * vin[i];
    *b = sqrt(creal(zdot(tmp, tmp, n)));
    for (int64_t i = 0; i < n; i++) {
        vout[i] = vin[i];
        vin[i] = tmp[i] / (*b);
    }
}

int32_t or_lanczos_tridiag(const or_model *M, const int32_t *map, int64_t dim, double *vin_,
                           int32_t nitermax, double *alanc, double *blanc, double threshold,
                           int32_t nthreads) {
    or_op op = {M, map, dim, nthreads};
    zc *vin = (zc *)vin_;
    zc *vout = (zc *)calloc((size_t)dim, sizeof(zc));
    zc *tmp = (zc *)calloc((size_t)dim, sizeof(zc));
    double a = 0.0, b = 0.0;
    int iter;
    for (int k = 0; k < nitermax; k++) alanc[k] = blanc[k] = 0.0;
    for (iter = 1; iter <= nitermax; iter++) {
        lanczos_iteration(&op, iter, vin, vout, tmp, &a, &b);
        alanc[iter - 1] = a;
        if (iter < nitermax) blanc[iter] = b;
        if (fabs(b) < threshold) break;
    }
    free(vout);
    free(tmp);
    return iter > nitermax ? nitermax : iter;
}

/* ------------------------------------------------------------------ */
/* pythag / tql2: ED_GREENS_FUNCTIONS.f90:361-539 (EISPACK QL with implicit
 * shifts; eigenvalues ascending with eigenvectors accumulated into z, which
 * is n x n column-major).  e(2:n) holds the sub-diagonal on entry. */
static double pythag(double a, double b) {
    double p = fmax(fabs(a), fabs(b));
    if (p != 0.0) {
        double r = fmin(fabs(a), fabs(b)) / p;
        r = r * r;
        for (;;) {
            double t = 4.0 + r;
            if (t == 4.0) break;
            double s = r / t;
            double u = 1.0 + 2.0 * s;
            p = u * p;
            r = (s / u) * (s / u) * r;
        }
    }
    return p;
}
static inline double fsign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }

int32_t or_tql2(int32_t n, double *d, double *e, double *z) {
#define D(i) d[(i)-1]
#define E(i) e[(i)-1]
#define Z(r, c) z[((long)(c)-1) * n + (r)-1]
    int ierr = 0;
    if (n == 1) return 0;
    for (int i = 2; i <= n; i++) E(i - 1) = E(i);
    double f = 0.0, tst1 = 0.0;
    E(n) = 0.0;
    for (int l = 1; l <= n; l++) {
        int j = 0, m;
        double h = fabs(D(l)) + fabs(E(l));
        tst1 = fmax(tst1, h);
        for (m = l; m <= n; m++) {
            double tst2 = tst1 + fabs(E(m));
            if (tst2 == tst1) break;
        }
        if (m > n) m = n; /* Fortran DO leaves m=n+1 only if no exit; E(n)=0 forces exit */
        if (m != l) {
            for (;;) {
                if (30 <= j) return l;
                j++;
                int l1 = l + 1, l2 = l1 + 1;
                double g = D(l);
                double p = (D(l1) - g) / (2.0 * E(l));
                double r = pythag(p, 1.0);
                D(l) = E(l) / (p + fsign(r, p));
                D(l1) = E(l) * (p + fsign(r, p));
                double dl1 = D(l1);
                h = g - D(l);
                for (int i = l2; i <= n; i++) D(i) = D(i) - h;
                f = f + h;
                p = D(m);
                double c = 1.0, c2 = c, c3 = c, el1 = E(l1), s = 0.0, s2 = 0.0;
                int mml = m - l;
                for (int ii = 1; ii <= mml; ii++) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    int i = m - ii;
                    g = c * E(i);
                    h = c * p;
                    r = pythag(p, E(i));
                    E(i + 1) = s * r;
                    s = E(i) / r;
                    c = p / r;
                    p = c * D(i) - s * g;
                    D(i + 1) = h + s * (c * g + s * D(i));
                    for (int k = 1; k <= n; k++) {
                        h = Z(k, i + 1);
                        Z(k, i + 1) = s * Z(k, i) + c * h;
                        Z(k, i) = c * Z(k, i) - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * E(l) / dl1;
                E(l) = s * p;
                D(l) = c * p;
                double tst2 = tst1 + fabs(E(l));
                if (!(tst2 > tst1)) break;
            }
        }
        D(l) = D(l) + f;
    }
    for (int ii = 2; ii <= n; ii++) {
        int i = ii - 1, k = i;
        double p = D(i);
        for (int j = ii; j <= n; j++)
            if (D(j) < p) {
                k = j;
                p = D(j);
            }
        if (k != i) {
            D(k) = D(i);
            D(i) = p;
            for (int j = 1; j <= n; j++) {
                double t = Z(j, i);
                Z(j, i) = Z(j, k);
                Z(j, k) = t;
            }
        }
    }
    return ierr;
#undef D
#undef E
#undef Z
}

/* ------------------------------------------------------------------ */
/* Ground state by plain Lanczos (.repo/PLAIN_LANCZOS.f90:286-385): tql2 of
 * the running tridiagonal after every step; the eigenvector is rebuilt by
 * replaying the recurrence from the same start vector and accumulating
 * v_k * Z(k,1).  (The legacy routine adds the vector AFTER the update, i.e.
 * v_{k+1}*Z(k,1), and drops the alpha of a breakdown step; this restatement
 * accumulates v_k*Z(k,1) and keeps that alpha, the Ritz pair the algorithm
 * intends.)
 * Stopping test: the one of ARPACK, the solver behind the reference's sp_eigh
 * (.repo/ARPACK_LANCZOS.f90:265-520, tol = lanc_tolerance): the Ritz estimate
 * b_{n+1} |Z(n,1)| <= threshold * max(eps^(2/3), |theta|), checked every
 * ncheck steps.  (An energy-change test stops long before the vector is
 * accurate; the Green's function is linear in the vector error.)
 * vect: complex start vector in, ground state out.  Returns nlanc;
 * *egs = lowest Ritz value. */
int32_t or_lanczos_gs(const or_model *M, const int32_t *map, int64_t dim, double *vect_,
                      int32_t nitermax, double threshold, int32_t ncheck, double *egs,
                      int32_t nthreads) {
    or_op op = {M, map, dim, nthreads};
    zc *vect = (zc *)vect_;
    zc *vin = (zc *)malloc(sizeof(zc) * dim), *vout = (zc *)calloc(dim, sizeof(zc));
    zc *tmp = (zc *)malloc(sizeof(zc) * dim);
    double *alanc = (double *)calloc(nitermax + 2, sizeof(double));
    double *blanc = (double *)calloc(nitermax + 2, sizeof(double));
    double *diag = (double *)malloc(sizeof(double) * (nitermax + 1));
    double *sub = (double *)malloc(sizeof(double) * (nitermax + 1));
    double *Z = (double *)malloc(sizeof(double) * (size_t)nitermax * nitermax);
    double *esave = (double *)calloc(nitermax + 2, sizeof(double));
    memcpy(vin, vect, sizeof(zc) * dim);
    int nlanc = 0;
    double a_ = 0.0, b_ = 0.0;
    for (int iter = 1; iter <= nitermax; iter++) {
        lanczos_iteration(&op, iter, vin, vout, tmp, &a_, &b_);
        nlanc++;
        alanc[iter] = a_;
        blanc[iter + 1] = b_;
        if (fabs(b_) < threshold) break; /* invariant subspace: keep this step's alpha */
        for (int i = 0; i < nlanc; i++) {
            diag[i] = alanc[i + 1];
            sub[i] = i == 0 ? 0.0 : blanc[i + 1];
        }
        for (long q = 0; q < (long)nlanc * nlanc; q++) Z[q] = 0.0;
        for (int i = 0; i < nlanc; i++) Z[(long)i * nlanc + i] = 1.0;
        if (fabs(b_) < threshold || nlanc % ncheck == 0 || nlanc == nitermax) {
            or_tql2(nlanc, diag, sub, Z);
            const double est = fabs(b_) * fabs(Z[(long)0 * nlanc + nlanc - 1]);
            const double eps23 = 3.666852862501036e-11; /* (2^-52)^(2/3) */
            if (est <= threshold * fmax(eps23, fabs(diag[0]))) break;
        }
    }
    for (int i = 0; i < nlanc; i++) {
        diag[i] = alanc[i + 1];
        sub[i] = i == 0 ? 0.0 : blanc[i + 1];
    }
    for (long q = 0; q < (long)nlanc * nlanc; q++) Z[q] = 0.0;
    for (int i = 0; i < nlanc; i++) Z[(long)i * nlanc + i] = 1.0;
    or_tql2(nlanc, diag, sub, Z);
    *egs = diag[0];
    /* second pass: vect = sum_k v_k Z(k,1) */
    memcpy(vin, vect, sizeof(zc) * dim);
    for (int64_t i = 0; i < dim; i++) {
        vout[i] = 0.0;
        vect[i] = 0.0;
    }
    {
        double nrm = sqrt(creal(zdot(vin, vin, dim)));
        for (int64_t i = 0; i < dim; i++) vin[i] /= nrm;
    }
    for (int iter = 1; iter <= nlanc; iter++) {
        for (int64_t i = 0; i < dim; i++) vect[i] += vin[i] * Z[iter - 1];
        if (iter == nlanc) break;
        double a = alanc[iter], b = blanc[iter];
        or_hxv_c128(M, map, dim, (const double *)vin, (double *)tmp, nthreads);
        for (int64_t i = 0; i < dim; i++) tmp[i] = tmp[i] - b * vout[i] - a * vin[i];
        double bn = blanc[iter + 1];
        for (int64_t i = 0; i < dim; i++) {
            vout[i] = vin[i];
            vin[i] = bn != 0.0 ? tmp[i] / bn : 0.0;
        }
    }
    double nrm = sqrt(creal(zdot(vect, vect, dim)));
    for (int64_t i = 0; i < dim; i++) vect[i] /= nrm;
    free(vin);
    free(vout);
    free(tmp);
    free(alanc);
    free(blanc);
    free(diag);
    free(sub);
    free(Z);
    free(esave);
    return nlanc;
}

/* ------------------------------------------------------------------ */
/* add_to_lanczos_gf_normal: build_gf_normal.f90:442-488.
 * Weight pesoBZ = vnorm2*exp(-beta(Ei-Egs))/Z (finite T, beta(Ei-Egs)<200),
 * vnorm2/Z (T=0), else 0.  tql2 of the nlanc tridiagonal (diag = alanc,
 * subdiag(2:) = blanc(2:)), then G(z) += peso Z(1,j)^2 / (z - isign*(E_j-Ei))
 * on z = i*wm (Lmats) and z = wr + i*eps (Lreal).  G arrays complex128 as
 * re/im pairs, accumulated in place. */
void or_add_to_lanczos_gf(double vnorm2, double ei, double egs, double zeta, int32_t finite_t,
                          double beta, const double *alanc, const double *blanc, int32_t nlanc,
                          int32_t isign, const double *wm, int32_t lmats, const double *wr,
                          int32_t lreal, double eps, double *gmats, double *greal) {
    double peso_bz;
    if (finite_t && beta * (ei - egs) < 200.0)
        peso_bz = vnorm2 * exp(-beta * (ei - egs)) / zeta;
    else if (!finite_t)
        peso_bz = vnorm2 / zeta;
    else
        peso_bz = 0.0;
    double *d = (double *)malloc(sizeof(double) * nlanc), *e = (double *)malloc(sizeof(double) * nlanc);
    double *Z = (double *)calloc((size_t)nlanc * nlanc, sizeof(double));
    for (int i = 0; i < nlanc; i++) {
        d[i] = alanc[i];
        e[i] = i == 0 ? 0.0 : blanc[i];
        Z[(long)i * nlanc + i] = 1.0;
    }
    or_tql2(nlanc, d, e, Z);
    zc *gm = (zc *)gmats, *gr = (zc *)greal;
    for (int j = 0; j < nlanc; j++) {
        double de = d[j] - ei;
        double z1 = Z[(long)j * nlanc + 0];
        double peso = peso_bz * z1 * z1;
        for (int i = 0; i < lmats; i++) {
            zc iw = I * wm[i];
            gm[i] = gm[i] + peso / (iw - isign * de);
        }
        for (int i = 0; i < lreal; i++) {
            zc iw = wr[i] + I * eps;
            gr[i] = gr[i] + peso / (iw - isign * de);
        }
    }
    free(d);
    free(e);
    free(Z);
}

/* vvinit of lanc_build_gf_normal_c, build_gf_normal.f90:97-116 (particle,
 * cdg) and :136-155 (hole, c): for each state m of sector I with the right
 * occupation at isite, r = cdg/c(isite, map_I(m)), j = binary_search(map_J, r),
 * vvinit(j) = sgn * psi(m).  isite is 1-based (impIndex).  vvinit zeroed
 * first.  Returns norm2 = <vvinit,vvinit> (before normalisation). */
double or_gf_vvinit(int32_t particle, int32_t isite, const int32_t *map_i, int64_t idim,
                    const int32_t *map_j, int64_t jdim, const double *psi_, double *vv_) {
    const zc *psi = (const zc *)psi_;
    zc *vv = (zc *)vv_;
    for (int64_t j = 0; j < jdim; j++) vv[j] = 0.0;
    if (isite < 1 || isite > 31) return -1.0; /* sites are 1-based levels of the word */
    for (int64_t m = 0; m < idim; m++) {
        int32_t i = map_i[m], r;
        double sgn;
        if (particle) {
            if (IB(i, isite) != 0) continue;
            op_cdg(isite, i, &r, &sgn);
        } else {
            if (IB(i, isite) != 1) continue;
            op_c(isite, i, &r, &sgn);
        }
        int64_t j = or_binary_search(map_j, jdim, r);
        if (j < 1) return -1.0; /* target state outside sector j: wrong sector pair */
        vv[j - 1] = sgn * psi[m];
    }
    return creal(zdot(vv, vv, jdim));
}

/* observables_impurity, ED_OBSERVABLES.f90:113-160 (densities and double
 * occupancy of one state, weight peso) and the diagonal bath density matrix
 * :286-305 (site = iorb + ibath*Norb + (ispin-1)*Ns, as written there).
 * out layout (accumulated): dens[norb], dens_up[norb], dens_dw[norb],
 * docc[norb], magz[norb], bath_dm[nspin][norb][nbath]. */
void or_observables_state(const or_model *M, const int32_t *map, int64_t dim, const double *psi_,
                          double peso, double *dens, double *dens_up, double *dens_dw, double *docc,
                          double *magz, double *bath_dm) {
    const zc *psi = (const zc *)psi_;
    int Ns = M->ns, Norb = M->norb, Nbath = M->nbath, Nspin = M->nspin;
    for (int64_t i = 0; i < dim; i++) {
        int32_t m = map[i];
        double w = peso * (creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]));
        for (int a = 1; a <= Norb; a++) {
            double nu = IB(m, a), nd = IB(m, a + Ns);
            dens[a - 1] += (nu + nd) * w;
            dens_up[a - 1] += nu * w;
            dens_dw[a - 1] += nd * w;
            docc[a - 1] += nu * nd * w;
            magz[a - 1] += (nu - nd) * w;
        }
    }
    for (int ib = 1; ib <= Nbath; ib++)
        for (int is = 1; is <= Nspin; is++)
            for (int a = 1; a <= Norb; a++) {
                int isite = a + ib * Norb + (is - 1) * Ns;
                double acc = 0.0;
                for (int64_t i = 0; i < dim; i++) {
                    double w = creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
                    acc += peso * IB(map[i], isite) * w;
                }
                bath_dm[((is - 1) * Norb + (a - 1)) * Nbath + ib - 1] += acc;
            }
}

/* local_energy_impurity, ED_OBSERVABLES.f90:454-633, the body for one kept
 * state (weight peso = exp(-beta(Ei-Egs))/Z or 1/Z), accumulated into
 * e[8] = {Eknot, Epot (without the Hartree part), Ehartree, Dust, Dund, Dse,
 * Dph, unused}.  As in the reference, the inter-orbital Hloc hopping terms
 * of Eknot and the spin-exchange / pair-hopping terms of Epot, Dse and Dph
 * are summed without the state's weight (ED_OBSERVABLES.f90:531,538,594-595,
 * 619-620), and only their real parts enter (the energies are real(8)). */
void or_local_energy_state(const or_model *M, const int32_t *map, int64_t dim, const double *psi_,
                           double peso, double *e) {
    const zc *psi = (const zc *)psi_;
    const int Ns = M->ns, Norb = M->norb, Nspin = M->nspin;
    const double Ust = M->ust, Jh = M->jh;
    double eloc[2][3];
    for (int is = 0; is < Nspin; is++)
        for (int a = 0; a < Norb; a++) eloc[is][a] = creal(hloc_at(M, is, is, a, a));
    for (int64_t i = 0; i < dim; i++) {
        const int32_t m = map[i];
        const double gsw = peso * (creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]));
        double nup[3], ndw[3];
        for (int a = 0; a < Norb; a++) {
            nup[a] = IB(m, a + 1);
            ndw[a] = IB(m, a + 1 + Ns);
        }
        /* LOCAL ENERGY */
        for (int a = 0; a < Norb; a++) e[0] += eloc[0][a] * nup[a] * gsw + eloc[Nspin - 1][a] * ndw[a] * gsw;
        /* HYBRIDIZATION TERMS I: same spin */
        for (int a = 1; a <= Norb; a++)
            for (int b = 1; b <= Norb; b++) {
                if (IB(m, a) == 0 && IB(m, b) == 1) {
                    int32_t k1 = 0, k2 = 0;
                    double sg1 = 1.0, sg2 = 1.0;
                    op_c(b, m, &k1, &sg1);
                    op_cdg(a, k1, &k2, &sg2);
                    const int64_t j = or_binary_search(map, dim, k2);
                    if (j > 0) e[0] += creal(hloc_at(M, 0, 0, a - 1, b - 1) * sg1 * sg2 * psi[i] * conj(psi[j - 1]));
                }
                if (IB(m, a + Ns) == 0 && IB(m, b + Ns) == 1) {
                    int32_t k1 = 0, k2 = 0;
                    double sg1 = 1.0, sg2 = 1.0;
                    op_c(b + Ns, m, &k1, &sg1);
                    op_cdg(a + Ns, k1, &k2, &sg2);
                    const int64_t j = or_binary_search(map, dim, k2);
                    if (j > 0)
                        e[0] += creal(hloc_at(M, Nspin - 1, Nspin - 1, a - 1, b - 1) * sg1 * sg2 * psi[i] *
                                      conj(psi[j - 1]));
                }
            }
        /* DENSITY-DENSITY */
        for (int a = 0; a < Norb; a++) e[1] += M->uloc[a] * nup[a] * ndw[a] * gsw;
        if (Norb > 1) {
            for (int a = 0; a < Norb; a++)
                for (int b = a + 1; b < Norb; b++) {
                    e[1] += Ust * (nup[a] * ndw[b] + nup[b] * ndw[a]) * gsw;
                    e[3] += (nup[a] * ndw[b] + nup[b] * ndw[a]) * gsw;
                }
            for (int a = 0; a < Norb; a++)
                for (int b = a + 1; b < Norb; b++) {
                    e[1] += (Ust - Jh) * (nup[a] * nup[b] + ndw[a] * ndw[b]) * gsw;
                    e[4] += (nup[a] * nup[b] + ndw[a] * ndw[b]) * gsw;
                }
        }
        /* SPIN-EXCHANGE and PAIR-HOPPING */
        if (Norb > 1 && M->jhflag) {
            for (int a = 1; a <= Norb; a++)
                for (int b = 1; b <= Norb; b++) {
                    if (a != b && IB(m, b) == 1 && IB(m, a + Ns) == 1 && IB(m, b + Ns) == 0 &&
                        IB(m, a) == 0) {
                        int32_t k1 = 0, k2 = 0, k3 = 0, k4 = 0;
                        double s1 = 1.0, s2 = 1.0, s3 = 1.0, s4 = 1.0;
                        op_c(b, m, &k1, &s1);
                        op_c(a + Ns, k1, &k2, &s2);
                        op_cdg(b + Ns, k2, &k3, &s3);
                        op_cdg(a, k3, &k4, &s4);
                        const int64_t j = or_binary_search(map, dim, k4);
                        if (j > 0) {
                            const double t = creal(s1 * s2 * s3 * s4 * psi[i] * conj(psi[j - 1]));
                            e[1] += M->jx * t;
                            e[5] += t;
                        }
                    }
                    if (a != b && IB(m, b) == 1 && IB(m, b + Ns) == 1 && IB(m, a + Ns) == 0 &&
                        IB(m, a) == 0) {
                        int32_t k1 = 0, k2 = 0, k3 = 0, k4 = 0;
                        double s1 = 1.0, s2 = 1.0, s3 = 1.0, s4 = 1.0;
                        op_c(b, m, &k1, &s1);
                        op_c(b + Ns, k1, &k2, &s2);
                        op_cdg(a + Ns, k2, &k3, &s3);
                        op_cdg(a, k3, &k4, &s4);
                        const int64_t j = or_binary_search(map, dim, k4);
                        if (j > 0) {
                            const double t = creal(s1 * s2 * s3 * s4 * psi[i] * conj(psi[j - 1]));
                            e[1] += M->jp * t;
                            e[6] += t;
                        }
                    }
                }
        }
        /* HARTREE TERMS */
        if (M->hfmode) {
            for (int a = 0; a < Norb; a++)
                e[2] += -0.5 * M->uloc[a] * (nup[a] + ndw[a]) * gsw + 0.25 * M->uloc[a] * gsw;
            if (Norb > 1)
                for (int a = 0; a < Norb; a++)
                    for (int b = a + 1; b < Norb; b++) {
                        const double nn = nup[a] + ndw[a] + nup[b] + ndw[b];
                        e[2] += -0.5 * Ust * nn * gsw + 0.25 * Ust * gsw;
                        e[2] += -0.5 * (Ust - Jh) * nn * gsw + 0.25 * (Ust - Jh) * gsw;
                    }
        }
    }
}

/* <psi| c^+_{a s} c_{k s} + h.c. |psi> and <psi|n_{k s}|psi> with the normal
 * bath stride (ED_SETUP.f90:445-462), the derivatives of the sector energy
 * with respect to V_{s,a,k} and e_{s,a,k} (Hellmann-Feynman; the operators
 * are the ones HxVimp_bath.f90 and HxVbath.f90 multiply by V and e).
 * hop[s][a][k], nk[s][a][k] accumulated with weight peso.  s runs over the
 * two physical spins (0=up, 1=down). */
void or_hf_terms_state(const or_model *M, const int32_t *map, int64_t dim, const double *psi_,
                       double peso, double *hop, double *nk) {
    const zc *psi = (const zc *)psi_;
    int Ns = M->ns, Norb = M->norb, Nbath = M->nbath;
    for (int s = 0; s < 2; s++)
        for (int a = 1; a <= Norb; a++)
            for (int kp = 1; kp <= Nbath; kp++) {
                int ms = Norb + (a - 1) * Nbath + kp + s * Ns;
                int ai = a + s * Ns;
                zc hacc = 0.0;
                double nacc = 0.0;
                for (int64_t i = 0; i < dim; i++) {
                    int32_t m = map[i], k1 = 0, k2 = 0;
                    double sg1 = 1.0, sg2 = 1.0;
                    double w = creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
                    nacc += IB(m, ms) * w;
                    if (IB(m, ai) == 1 && IB(m, ms) == 0) {
                        op_c(ai, m, &k1, &sg1);
                        op_cdg(ms, k1, &k2, &sg2);
                        int64_t j = or_binary_search(map, dim, k2);
                        hacc += conj(psi[j - 1]) * sg1 * sg2 * psi[i];
                    }
                    if (IB(m, ai) == 0 && IB(m, ms) == 1) {
                        op_c(ms, m, &k1, &sg1);
                        op_cdg(ai, k1, &k2, &sg2);
                        int64_t j = or_binary_search(map, dim, k2);
                        hacc += conj(psi[j - 1]) * sg1 * sg2 * psi[i];
                    }
                }
                long idx = ((long)s * Norb + (a - 1)) * Nbath + kp - 1;
                hop[idx] += peso * creal(hacc);
                nk[idx] += peso * nacc;
            }
}

/* ------------------------------------------------------------------ */
/* Bath functions (normal bath, normal ed_mode):
 *   delta_bath_mats  ED_BATH_FUNCTIONS.f90:247-257 : Delta = sum_k V^2/(x-e)
 *   invg0_bath_mats  ED_BATH_FUNCTIONS.f90:1800-1806: x + xmu - Hloc_aa - Delta
 *   get_sigma_normal get_sigma_normal.f90:17-39     : S = G0^-1 - 1/G
 * x complex (i*wm or wr+i*eps), arrays complex as re/im pairs. */
void or_delta_bath(const double *eps_k, const double *v_k, int32_t nbath, const double *x_,
                   int32_t L, double *delta_) {
    const zc *x = (const zc *)x_;
    zc *d = (zc *)delta_;
    for (int i = 0; i < L; i++) {
        zc s = 0.0;
        for (int k = 0; k < nbath; k++) s += v_k[k] * v_k[k] / (x[i] - eps_k[k]);
        d[i] = s;
    }
}

void or_sigma_normal(const double *eps_k, const double *v_k, int32_t nbath, double xmu,
                     double hloc_aa, const double *x_, int32_t L, const double *g_, double *s_) {
    const zc *x = (const zc *)x_, *g = (const zc *)g_;
    zc *s = (zc *)s_;
    for (int i = 0; i < L; i++) {
        zc dl = 0.0;
        for (int k = 0; k < nbath; k++) dl += v_k[k] * v_k[k] / (x[i] - eps_k[k]);
        zc invg0 = x[i] + xmu - hloc_aa - dl;
        s[i] = invg0 - 1.0 / g[i];
    }
}

/* chi2_delta_normal_normal / grad_chi2_delta_normal_normal with
 * delta_normal_normal and grad_delta_normal_normal,
 * ED_CHI2FIT/fitgf_normal_normal.f90:193-226,256-316.
 * a = [e_1..e_Nbath, V_1..V_Nbath]; xdelta = wm(1:L); g = target (re/im);
 * w = weights.  Returns chi2; grad (2*nbath) written if non-NULL. */
double or_chi2_delta(const double *a, int32_t nbath, const double *xdelta, const double *g_,
                     const double *w, int32_t L, double *grad) {
    const zc *g = (const zc *)g_;
    double chi2 = 0.0;
    zc *delta = (zc *)malloc(sizeof(zc) * L);
    for (int i = 0; i < L; i++) {
        zc s = 0.0;
        for (int k = 0; k < nbath; k++) s += a[nbath + k] * a[nbath + k] / (I * xdelta[i] - a[k]);
        delta[i] = s;
    }
    for (int i = 0; i < L; i++) {
        double re = creal(g[i] - delta[i]), im = cimag(g[i] - delta[i]);
        chi2 += (re * re + im * im) / w[i];
    }
    if (grad) {
        for (int j = 0; j < 2 * nbath; j++) {
            double s1 = 0.0, s2 = 0.0;
            for (int i = 0; i < L; i++) {
                zc dd;
                if (j < nbath) {
                    zc den = I * xdelta[i] - a[j];
                    dd = a[nbath + j] * a[nbath + j] / (den * den);
                } else {
                    int k = j - nbath;
                    dd = 2.0 * a[nbath + k] / (I * xdelta[i] - a[k]);
                }
                s1 += creal(g[i] - delta[i]) * creal(dd) / w[i];
                s2 += cimag(g[i] - delta[i]) * cimag(dd) / w[i];
            }
            grad[j] = -2.0 * (s1 + s2);
        }
    }
    free(delta);
    return chi2;
}

/* chi^2 of the bath fit for either scheme, chi2_delta_normal_normal and
 * chi2_weiss_normal_normal (ED_CHI2FIT/fitgf_normal_normal.f90:193-202,
 * 235-246) with g0and_normal_normal (:349-362): M_n = Delta_n (weiss = 0) or
 * G0_n = 1/(i x_n + zc - Delta_n), zc = xmu - Hloc_aa (weiss = 1).  The
 * gradient: the reference's grad_chi2_delta_normal_normal (:208-226) for the
 * delta scheme; for the weiss scheme the same formula with dM = G0^2 dDelta
 * (the reference differentiates this chi^2 numerically inside fmin_cg).
 * Sums run over the frequencies in order. */
double or_chi2_model(const double *a, int32_t nbath, const double *xdelta, const double *g_,
                     const double *w, int32_t L, int32_t weiss, double zcv, double *grad) {
    const zc *g = (const zc *)g_;
    double chi2 = 0.0;
    zc *m = (zc *)malloc(sizeof(zc) * L);
    zc *g02 = (zc *)malloc(sizeof(zc) * L);
    for (int i = 0; i < L; i++) {
        zc d = 0.0;
        for (int k = 0; k < nbath; k++) d += a[nbath + k] * a[nbath + k] / (I * xdelta[i] - a[k]);
        if (weiss) {
            zc g0 = 1.0 / (I * xdelta[i] + zcv - d);
            m[i] = g0;
            g02[i] = g0 * g0;
        } else {
            m[i] = d;
            g02[i] = 1.0;
        }
    }
    for (int i = 0; i < L; i++) {
        double re = creal(g[i] - m[i]), im = cimag(g[i] - m[i]);
        chi2 += (re * re + im * im) / w[i];
    }
    if (grad) {
        for (int j = 0; j < 2 * nbath; j++) {
            double s1 = 0.0, s2 = 0.0;
            for (int i = 0; i < L; i++) {
                zc dd;
                if (j < nbath) {
                    zc den = I * xdelta[i] - a[j];
                    dd = a[nbath + j] * a[nbath + j] / (den * den);
                } else {
                    int k = j - nbath;
                    dd = 2.0 * a[nbath + k] / (I * xdelta[i] - a[k]);
                }
                dd *= g02[i];
                s1 += creal(g[i] - m[i]) * creal(dd) / w[i];
                s2 += cimag(g[i] - m[i]) * cimag(dd) / w[i];
            }
            grad[j] = -2.0 * (s1 + s2);
        }
    }
    free(m);
    free(g02);
    return chi2;
}

/* fmin_cg (SciFortran SF_OPTIMIZE, absent from the tree, version unpinned),
 * called by chi2_fitgf_normal_normal (fitgf_normal_normal.f90:82-119), restated
 * from the published algorithm it implements: the Polak-Ribiere conjugate
 * gradient with line minimisation by bracketing and Brent's method with
 * derivatives (Press et al., Numerical Recipes, 2nd ed., sections 10.1, 10.3,
 * 10.6: frprmn, dlinmin, mnbrak, dbrent; the book's constants; line
 * tolerance 1e-4).  Stopping test: cg_stop 0 the book's 2|fret - fp| <= ftol
 * (|fret| + |fp| + eps); 1 |fret - fp| <= ftol; 2 fret <= ftol.
 * a (2*nbath) in/out.  Returns the final chi^2; *iter the steps taken;
 * *status bit 0 a bracket search failed, bit 1 a Brent search hit its limit. */
typedef struct {
    const double *p, *xi;
    double *q, *gr;
    int32_t na, nbath, L, weiss;
    const double *xdelta, *g, *w;
    double zc;
} cg_line;

static double cg_f1dim(const cg_line *c, double x) {
    for (int j = 0; j < c->na; j++) c->q[j] = c->p[j] + x * c->xi[j];
    return or_chi2_model(c->q, c->nbath, c->xdelta, c->g, c->w, c->L, c->weiss, c->zc, NULL);
}

static double cg_fdf1dim(const cg_line *c, double x, double *df) {
    for (int j = 0; j < c->na; j++) c->q[j] = c->p[j] + x * c->xi[j];
    double f = or_chi2_model(c->q, c->nbath, c->xdelta, c->g, c->w, c->L, c->weiss, c->zc, c->gr);
    double d = 0.0;
    for (int j = 0; j < c->na; j++) d += c->gr[j] * c->xi[j];
    *df = d;
    return f;
}

static int cg_mnbrak(const cg_line *c, double *ax, double *bx, double *cx, double *fa, double *fb,
                     double *fc) {
    const double GOLD = 1.618034, GLIMIT = 100.0, TINY = 1.0e-20;
    double t;
    *fa = cg_f1dim(c, *ax);
    *fb = cg_f1dim(c, *bx);
    if (*fb > *fa) {
        t = *ax; *ax = *bx; *bx = t;
        t = *fa; *fa = *fb; *fb = t;
    }
    *cx = *bx + GOLD * (*bx - *ax);
    *fc = cg_f1dim(c, *cx);
    for (int it = 0; *fb >= *fc; it++) {
        if (it >= 200) return 0;
        double r = (*bx - *ax) * (*fb - *fc);
        double q = (*bx - *cx) * (*fb - *fa);
        double u = *bx - ((*bx - *cx) * q - (*bx - *ax) * r) /
                             (2.0 * copysign(fmax(fabs(q - r), TINY), q - r));
        double ulim = *bx + GLIMIT * (*cx - *bx);
        double fu;
        if ((*bx - u) * (u - *cx) > 0.0) {
            fu = cg_f1dim(c, u);
            if (fu < *fc) {
                *ax = *bx; *bx = u;
                *fa = *fb; *fb = fu;
                return 1;
            } else if (fu > *fb) {
                *cx = u;
                *fc = fu;
                return 1;
            }
            u = *cx + GOLD * (*cx - *bx);
            fu = cg_f1dim(c, u);
        } else if ((*cx - u) * (u - ulim) > 0.0) {
            fu = cg_f1dim(c, u);
            if (fu < *fc) {
                *bx = *cx; *cx = u; u = *cx + GOLD * (*cx - *bx);
                *fb = *fc; *fc = fu; fu = cg_f1dim(c, u);
            }
        } else if ((u - ulim) * (ulim - *cx) >= 0.0) {
            u = ulim;
            fu = cg_f1dim(c, u);
        } else {
            u = *cx + GOLD * (*cx - *bx);
            fu = cg_f1dim(c, u);
        }
        *ax = *bx; *bx = *cx; *cx = u;
        *fa = *fb; *fb = *fc; *fc = fu;
    }
    return 1;
}

static double cg_dbrent(const cg_line *c, double ax, double bx, double cx, double tol,
                        double *xmin, int32_t *status) {
    const int ITMAX = 100;
    const double ZEPS = 1.0e-10;
    double a = fmin(ax, cx), b = fmax(ax, cx);
    double d = 0.0, e = 0.0;
    double x = bx, w = bx, v = bx;
    double dx, fx = cg_fdf1dim(c, x, &dx);
    double fw = fx, fv = fx, dw = dx, dv = dx;
    for (int iter = 0; iter < ITMAX; iter++) {
        double xm = 0.5 * (a + b);
        double tol1 = tol * fabs(x) + ZEPS, tol2 = 2.0 * tol1;
        if (fabs(x - xm) <= (tol2 - 0.5 * (b - a))) {
            *xmin = x;
            return fx;
        }
        int bisect = 1;
        if (fabs(e) > tol1) {
            double d1 = 2.0 * (b - a), d2 = d1;
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);
            double u1 = x + d1, u2 = x + d2;
            int ok1 = (a - u1) * (u1 - b) > 0.0 && dx * d1 <= 0.0;
            int ok2 = (a - u2) * (u2 - b) > 0.0 && dx * d2 <= 0.0;
            double olde = e;
            e = d;
            if (ok1 || ok2) {
                if (ok1 && ok2) d = fabs(d1) < fabs(d2) ? d1 : d2;
                else d = ok1 ? d1 : d2;
                if (fabs(d) <= fabs(0.5 * olde)) {
                    double u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = copysign(tol1, xm - x);
                    bisect = 0;
                }
            }
        }
        if (bisect) {
            e = dx >= 0.0 ? a - x : b - x;
            d = 0.5 * e;
        }
        double u, fu, du;
        if (fabs(d) >= tol1) {
            u = x + d;
            fu = cg_fdf1dim(c, u, &du);
        } else {
            u = x + copysign(tol1, d);
            fu = cg_fdf1dim(c, u, &du);
            if (fu > fx) {
                *xmin = x;
                return fx;
            }
        }
        if (fu <= fx) {
            if (u >= x) a = x;
            else b = x;
            v = w; fv = fw; dv = dw;
            w = x; fw = fx; dw = dx;
            x = u; fx = fu; dx = du;
        } else {
            if (u < x) a = u;
            else b = u;
            if (fu <= fw || w == x) {
                v = w; fv = fw; dv = dw;
                w = u; fw = fu; dw = du;
            } else if (fu <= fv || v == x || v == w) {
                v = u; fv = fu; dv = du;
            }
        }
    }
    *status |= 2;
    *xmin = x;
    return fx;
}

double or_cg_fit(double *a, int32_t nbath, const double *xdelta, const double *g, const double *w,
                 int32_t L, int32_t weiss, double zcv, int32_t itmax, double ftol, double eps,
                 int32_t istop, int32_t *iter, int32_t *status) {
    const int na = 2 * nbath;
    double *xi = (double *)malloc(sizeof(double) * na), *gv = (double *)malloc(sizeof(double) * na);
    double *h = (double *)malloc(sizeof(double) * na), *q = (double *)malloc(sizeof(double) * na);
    double *gr = (double *)malloc(sizeof(double) * na);
    cg_line c = {a, xi, q, gr, na, nbath, L, weiss, xdelta, g, w, zcv};
    *status = 0;
    *iter = 0;
    double fp = or_chi2_model(a, nbath, xdelta, g, w, L, weiss, zcv, xi);
    for (int j = 0; j < na; j++) {
        gv[j] = -xi[j];
        h[j] = gv[j];
        xi[j] = h[j];
    }
    double fret = fp;
    for (int its = 1; its <= itmax; its++) {
        *iter = its;
        double ax = 0.0, xx = 1.0, bx, fa, fx, fb, xmin = 0.0;
        if (!cg_mnbrak(&c, &ax, &xx, &bx, &fa, &fx, &fb)) *status |= 1;
        fret = cg_dbrent(&c, ax, xx, bx, 1.0e-4, &xmin, status);
        for (int j = 0; j < na; j++) {
            xi[j] *= xmin;
            a[j] += xi[j];
        }
        int done;
        if (istop == 1) done = fabs(fret - fp) <= ftol;
        else if (istop == 2) done = fret <= ftol;
        else done = 2.0 * fabs(fret - fp) <= ftol * (fabs(fret) + fabs(fp) + eps);
        if (done) break;
        fp = fret;
        or_chi2_model(a, nbath, xdelta, g, w, L, weiss, zcv, xi);
        double gg = 0.0, dgg = 0.0;
        for (int j = 0; j < na; j++) {
            gg += gv[j] * gv[j];
            dgg += (xi[j] + gv[j]) * xi[j];
        }
        if (gg == 0.0) break;
        double gam = dgg / gg;
        for (int j = 0; j < na; j++) {
            gv[j] = -xi[j];
            h[j] = gv[j] + gam * h[j];
            xi[j] = h[j];
        }
    }
    free(xi);
    free(gv);
    free(h);
    free(q);
    free(gr);
    return fret;
}

int32_t or_host_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int32_t)n : 1;
}
