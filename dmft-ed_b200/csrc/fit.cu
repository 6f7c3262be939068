// The DMFT self-consistency around the impurity solve, on the device:
//
//  * the bath fit that ed_chi2_fitgf runs once per orbital
//    (ED_CHI2FIT.f90:86-138 -> ED_CHI2FIT/fitgf_normal_normal.f90:18-178):
//    minimise chi2(a) = sum_n |G_n - M_n(a)|^2 / W_n over a = [e_1..e_Nbath,
//    V_1..V_Nbath], with M = Delta (cg_scheme "delta",
//    delta_normal_normal :256-279) or M = G0and = 1/(i w_n + xmu - Hloc_aa -
//    Delta) (cg_scheme "weiss", g0and_normal_normal :349-362), by the
//    conjugate-gradient routine fmin_cg of SciFortran (absent from the tree,
//    version unpinned; see below);
//  * the local Green's function of a lattice Hamiltonian diagonal in spin and
//    orbital on a density-of-states grid, G_loc(iw_n) = sum_k W_k / (i w_n +
//    xmu - Sigma(iw_n) - e_k) (DMFT_Tools' dmft_gloc_matsubara, called by
//    drivers/ed_hm_bethe.f90:70; the same sum as the legacy in-tree
//    .repo/ED_GLOC.f90:54-126,257-298 for 1x1 blocks);
//  * the Weiss field 1/(1/G_loc + Sigma) or the hybridisation i w_n + xmu -
//    Hloc - Sigma - 1/G_loc (dmft_weiss / dmft_delta, drivers/ed_hm_bethe.f90:
//    73-77; .repo/ED_WEISS.f90:55-118 for 1x1 blocks).
//
// The minimiser is the published Polak-Ribiere conjugate gradient with a line
// minimisation by bracketing (golden-ratio expansion with parabolic
// extrapolation) and Brent's method with first derivatives: Press, Teukolsky,
// Vetterling and Flannery, Numerical Recipes, 2nd ed., sections 10.1, 10.3
// and 10.6 (frprmn, dlinmin, mnbrak, dbrent), the family fmin_cg belongs to.
// The constants are the book's (GOLD 1.618034, GLIMIT 100, TINY 1e-20; line
// tolerance 1e-4, ZEPS 1e-10, 100 Brent steps); the stopping test with
// cg_stop = 0 is the book's 2|f_new - f_old| <= ftol (|f_new| + |f_old| +
// cg_eps).  The gradient is the analytic one in both schemes (the reference
// differentiates the weiss chi2 numerically inside fmin_cg); the minimum is
// the same, the path to it differs by the finite-difference error.
//
// One CTA per fit.  Every thread runs the same scalar control flow; each
// function value is a block-wide sum over the Matsubara points, reduced in a
// fixed order, so every thread sees the same numbers and takes the same
// branches.  A line-search evaluation returns chi2 and its derivative along
// the search direction in one pass; the full gradient is formed once per
// conjugate-gradient step.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "reduce.cuh"

namespace dmfted {

constexpr int kFitThreads = 256;
constexpr int kFitMaxBracket = 200;  // bracketing expansions before giving up
constexpr double kLineTol = 1.0e-4;  // fractional tolerance of the line minimum

struct FitArgs {
    int nbath, L;
    double *a;            // [nbatch][2 nbath]: start in, minimum out
    const double *x;      // [L] Matsubara frequencies of the fit
    const double2 *g;     // [ng][L] targets; job b fits target b % ng
    int ng;
    const double *w;      // [L] weights W_n
    const double *zc;     // [ng] xmu - Hloc_aa of the target (weiss scheme), or null:
    double zc0;           //      then zc0 for every target
    int weiss;
    int itmax, istop;
    double ftol, eps;
    int *iter;            // [nbatch] conjugate-gradient steps taken
    double *chi2;         // [nbatch] chi2 at the returned parameters
    int *status;          // [nbatch] bit 0: bracketing failed, bit 1: Brent limit
};

struct FitShared {
    double *p, *xi, *gv, *h, *q, *grad;  // [na] each
    double *acc;                         // [na][nt] gradient partial sums
    double *red;                         // [2 * nwarps] value partial sums
};

// Sum of v over the block, the same value in every thread (fixed order:
// xor butterfly inside each warp, then the warp sums in warp order).
__device__ __forceinline__ void block_sum2(double &v0, double &v1, double *red) {
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();  // earlier readers of red are done
    if ((threadIdx.x & 31) == 0) {
        red[2 * wid] = v0;
        red[2 * wid + 1] = v1;
    }
    __syncthreads();
    double s0 = 0.0, s1 = 0.0;
    for (int i = 0; i < nw; i++) {
        s0 += red[2 * i];
        s1 += red[2 * i + 1];
    }
    v0 = s0;
    v1 = s1;
}

// chi2 at parameters q and, by MODE: nothing (0); its derivative along dir
// into *dfdir (1); its gradient into grad[2 nbath] (2).  Called by every
// thread of the block with the same arguments; returns chi2 to all.
template <int MODE>
__device__ double fit_eval(const FitArgs &A, const double2 *__restrict__ g, double zc,
                           const FitShared &S, const double *q, const double *dir, double *dfdir) {
    const int tid = threadIdx.x, nt = blockDim.x, nb = A.nbath, na = 2 * nb;
    const double *pe = q, *pv = q + nb;
    if (MODE == 2)
        for (int j = 0; j < na; j++) S.acc[j * nt + tid] = 0.0;
    double f = 0.0, fd = 0.0;
    for (int n = tid; n < A.L; n += nt) {
        const double om = A.x[n];
        const double2 gn = g[n];
        const double iw = 1.0 / A.w[n];
        double dr = 0.0, di = 0.0;  // Delta = sum_k V_k^2 / (i om - e_k)
        for (int k = 0; k < nb; k++) {
            const double e = pe[k], v = pv[k];
            const double inv = 1.0 / (e * e + om * om);
            dr += v * v * (-e * inv);
            di += v * v * (-om * inv);
        }
        double mr = dr, mi = di, g2r = 1.0, g2i = 0.0;
        if (A.weiss) {  // G0 = 1/(i om + zc - Delta); dG0 = G0^2 dDelta
            const double ar = zc - dr, ai = om - di;
            const double den = 1.0 / (ar * ar + ai * ai);
            mr = ar * den;
            mi = -ai * den;
            g2r = mr * mr - mi * mi;
            g2i = 2.0 * mr * mi;
        }
        const double Rr = gn.x - mr, Ri = gn.y - mi;
        f += (Rr * Rr + Ri * Ri) * iw;
        if (MODE == 1) {
            double Dr = 0.0, Di = 0.0;  // dDelta along dir
            for (int k = 0; k < nb; k++) {
                const double e = pe[k], v = pv[k];
                const double inv = 1.0 / (e * e + om * om);
                const double re = -e * inv, im = -om * inv;
                const double r2r = re * re - im * im, r2i = 2.0 * re * im;
                const double de = dir[k], dv = dir[nb + k];
                Dr += de * v * v * r2r + dv * 2.0 * v * re;
                Di += de * v * v * r2i + dv * 2.0 * v * im;
            }
            const double tr = Dr * g2r - Di * g2i, ti = Dr * g2i + Di * g2r;
            fd += (Rr * tr + Ri * ti) * iw;
        }
        if (MODE == 2) {
            for (int k = 0; k < nb; k++) {
                const double e = pe[k], v = pv[k];
                const double inv = 1.0 / (e * e + om * om);
                const double re = -e * inv, im = -om * inv;
                const double r2r = re * re - im * im, r2i = 2.0 * re * im;
                // dDelta/de_k = V^2 r^2, dDelta/dV_k = 2 V r, each times G0^2 (weiss)
                const double er = v * v * r2r, ei = v * v * r2i;
                const double vr = 2.0 * v * re, vi = 2.0 * v * im;
                const double ter = er * g2r - ei * g2i, tei = er * g2i + ei * g2r;
                const double tvr = vr * g2r - vi * g2i, tvi = vr * g2i + vi * g2r;
                S.acc[k * nt + tid] += (Rr * ter + Ri * tei) * iw;
                S.acc[(nb + k) * nt + tid] += (Rr * tvr + Ri * tvi) * iw;
            }
        }
    }
    block_sum2(f, fd, S.red);
    if (MODE == 1) *dfdir = -2.0 * fd;
    if (MODE == 2) {
        __syncthreads();
        for (int j = tid; j < na; j += nt) {
            CSum s;
            s.zero();
            for (int t = 0; t < nt; t++) s.add(S.acc[j * nt + t]);
            S.grad[j] = -2.0 * s.value();
        }
        __syncthreads();
    }
    return f;
}

// chi2 along the line p + x xi (dlinmin's f1dim / df1dim), value and, when
// df is given, the derivative along xi.
struct LineFn {
    const FitArgs &A;
    const double2 *g;
    double zc;
    const FitShared &S;
    int na;
    __device__ double operator()(double x, double *df) const {
        __syncthreads();
        for (int j = threadIdx.x; j < na; j += blockDim.x) S.q[j] = S.p[j] + x * S.xi[j];
        __syncthreads();
        if (df) return fit_eval<1>(A, g, zc, S, S.q, S.xi, df);
        return fit_eval<0>(A, g, zc, S, S.q, nullptr, nullptr);
    }
};

// mnbrak: from ax, bx, a triple ax, bx, cx with f(bx) below f(ax) and f(cx).
// Returns false when kFitMaxBracket expansions did not bracket a minimum.
template <class Fn>
__device__ bool mnbrak(double &ax, double &bx, double &cx, double &fa, double &fb, double &fc,
                       const Fn &f) {
    const double GOLD = 1.618034, GLIMIT = 100.0, TINY = 1.0e-20;
    fa = f(ax, nullptr);
    fb = f(bx, nullptr);
    if (fb > fa) {
        double t = ax; ax = bx; bx = t;
        t = fa; fa = fb; fb = t;
    }
    cx = bx + GOLD * (bx - ax);
    fc = f(cx, nullptr);
    for (int it = 0; fb >= fc; it++) {
        if (it >= kFitMaxBracket) return false;
        const double r = (bx - ax) * (fb - fc);
        const double q = (bx - cx) * (fb - fa);
        double u = bx - ((bx - cx) * q - (bx - ax) * r) /
                            (2.0 * copysign(fmax(fabs(q - r), TINY), q - r));
        const double ulim = bx + GLIMIT * (cx - bx);
        double fu;
        if ((bx - u) * (u - cx) > 0.0) {
            fu = f(u, nullptr);
            if (fu < fc) {
                ax = bx; bx = u;
                fa = fb; fb = fu;
                return true;
            } else if (fu > fb) {
                cx = u;
                fc = fu;
                return true;
            }
            u = cx + GOLD * (cx - bx);
            fu = f(u, nullptr);
        } else if ((cx - u) * (u - ulim) > 0.0) {
            fu = f(u, nullptr);
            if (fu < fc) {
                bx = cx; cx = u; u = cx + GOLD * (cx - bx);
                fb = fc; fc = fu; fu = f(u, nullptr);
            }
        } else if ((u - ulim) * (ulim - cx) >= 0.0) {
            u = ulim;
            fu = f(u, nullptr);
        } else {
            u = cx + GOLD * (cx - bx);
            fu = f(u, nullptr);
        }
        ax = bx; bx = cx; cx = u;
        fa = fb; fb = fc; fc = fu;
    }
    return true;
}

// dbrent: the minimum of f inside the bracket (ax, bx, cx) to fractional
// tolerance tol, using the derivative; *xmin its abscissa.
template <class Fn>
__device__ double dbrent(double ax, double bx, double cx, const Fn &f, double tol, double *xmin,
                         int *status) {
    const int ITMAX = 100;
    const double ZEPS = 1.0e-10;
    double a = fmin(ax, cx), b = fmax(ax, cx);
    double d = 0.0, e = 0.0;
    double x = bx, w = bx, v = bx;
    double dx;
    double fx = f(x, &dx);
    double fw = fx, fv = fx, dw = dx, dv = dx;
    for (int iter = 0; iter < ITMAX; iter++) {
        const double xm = 0.5 * (a + b);
        const double tol1 = tol * fabs(x) + ZEPS, tol2 = 2.0 * tol1;
        if (fabs(x - xm) <= (tol2 - 0.5 * (b - a))) {
            *xmin = x;
            return fx;
        }
        bool bisect = true;
        if (fabs(e) > tol1) {
            double d1 = 2.0 * (b - a), d2 = d1;
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);  // secant with w
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);  // secant with v
            const double u1 = x + d1, u2 = x + d2;
            const bool ok1 = (a - u1) * (u1 - b) > 0.0 && dx * d1 <= 0.0;
            const bool ok2 = (a - u2) * (u2 - b) > 0.0 && dx * d2 <= 0.0;
            const double olde = e;
            e = d;
            if (ok1 || ok2) {
                if (ok1 && ok2) d = fabs(d1) < fabs(d2) ? d1 : d2;
                else d = ok1 ? d1 : d2;
                if (fabs(d) <= fabs(0.5 * olde)) {
                    const double u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = copysign(tol1, xm - x);
                    bisect = false;
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
            fu = f(u, &du);
        } else {
            u = x + copysign(tol1, d);
            fu = f(u, &du);
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

// One conjugate-gradient fit per CTA (frprmn with dlinmin).
__global__ void __launch_bounds__(kFitThreads) k_cg_fit(const FitArgs A) {
    extern __shared__ double fsm[];
    const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int nb = A.nbath, na = 2 * nb;
    FitShared S;
    S.p = fsm;
    S.xi = S.p + na;
    S.gv = S.xi + na;
    S.h = S.gv + na;
    S.q = S.h + na;
    S.grad = S.q + na;
    S.red = S.grad + na;
    S.acc = S.red + 2 * (nt >> 5);
    const int tg = b % A.ng;
    const double2 *g = A.g + (int64_t)tg * A.L;
    const double zc = A.zc ? A.zc[tg] : A.zc0;
    double *a = A.a + (int64_t)b * na;
    for (int j = tid; j < na; j += nt) S.p[j] = a[j];
    __syncthreads();
    int status = 0, iter = 0;
    double fp = fit_eval<2>(A, g, zc, S, S.p, nullptr, nullptr);
    for (int j = tid; j < na; j += nt) {
        S.gv[j] = -S.grad[j];
        S.h[j] = S.gv[j];
        S.xi[j] = S.h[j];
    }
    __syncthreads();
    double fret = fp;
    const LineFn F{A, g, zc, S, na};
    for (int its = 1; its <= A.itmax; its++) {
        iter = its;
        // dlinmin: bracket from (0, 1), Brent with derivatives, then move
        double ax = 0.0, xx = 1.0, bx, fa, fx, fb;
        if (!mnbrak(ax, xx, bx, fa, fx, fb, F)) status |= 1;
        double xmin = 0.0;
        fret = dbrent(ax, xx, bx, F, kLineTol, &xmin, &status);
        __syncthreads();
        for (int j = tid; j < na; j += nt) {
            S.xi[j] *= xmin;
            S.p[j] += S.xi[j];
        }
        __syncthreads();
        bool done;
        if (A.istop == 1) done = fabs(fret - fp) <= A.ftol;
        else if (A.istop == 2) done = fret <= A.ftol;
        else done = 2.0 * fabs(fret - fp) <= A.ftol * (fabs(fret) + fabs(fp) + A.eps);
        if (done) break;
        fp = fret;
        fit_eval<2>(A, g, zc, S, S.p, nullptr, nullptr);  // xi = gradient at p
        // Polak-Ribiere: gam = sum (xi + g) xi / sum g^2 (fixed order, thread 0)
        if (tid == 0) {
            double gg = 0.0, dgg = 0.0;
            for (int j = 0; j < na; j++) {
                const double xj = S.grad[j];
                gg += S.gv[j] * S.gv[j];
                dgg += (xj + S.gv[j]) * xj;
            }
            S.red[0] = gg;
            S.red[1] = dgg;
        }
        __syncthreads();
        const double gg = S.red[0], dgg = S.red[1];
        if (gg == 0.0) break;
        const double gam = dgg / gg;
        __syncthreads();
        for (int j = tid; j < na; j += nt) {
            S.gv[j] = -S.grad[j];
            S.h[j] = S.gv[j] + gam * S.h[j];
            S.xi[j] = S.h[j];
        }
        __syncthreads();
    }
    for (int j = tid; j < na; j += nt) a[j] = S.p[j];
    if (tid == 0) {
        A.iter[b] = iter;
        A.chi2[b] = fret;
        A.status[b] = status;
    }
}

static size_t fit_smem(int nbath, int nt) {
    const int na = 2 * nbath;
    return (size_t)(6 * na + 2 * (nt / 32) + (size_t)na * nt) * sizeof(double);
}

void cg_fit_device(dmfted_ctx *c, int nbatch, int nbath, int L, double *a, const double *x,
                   const double *g, int ng, const double *w, const double *zc, double zc0,
                   int weiss, int itmax, int istop, double ftol, double eps, int *iter,
                   double *chi2, int *status) {
    DM_REQUIRE(nbatch > 0 && nbath > 0 && L > 0 && ng > 0, DMFTED_ERR_ARG,
               "cg fit: empty batch, bath or grid");
    DM_REQUIRE(itmax >= 1, DMFTED_ERR_ARG, "cg fit: cg_niter < 1");
    int nt = kFitThreads;
    while (nt > 64 && fit_smem(nbath, nt) > 200 * 1024) nt /= 2;
    DM_REQUIRE(fit_smem(nbath, nt) <= 200 * 1024, DMFTED_ERR_UNSUPPORTED,
               "cg fit: too many bath levels for the shared-memory fit");
    static bool attr[64] = {false};
    if (!attr[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(k_cg_fit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr[c->device & 63] = true;
    }
    FitArgs A{};
    A.nbath = nbath;
    A.L = L;
    A.a = a;
    A.x = x;
    A.g = reinterpret_cast<const double2 *>(g);
    A.ng = ng;
    A.w = w;
    A.zc = zc;
    A.zc0 = zc0;
    A.weiss = weiss;
    A.itmax = itmax;
    A.istop = istop;
    A.ftol = ftol;
    A.eps = eps;
    A.iter = iter;
    A.chi2 = chi2;
    A.status = status;
    k_cg_fit<<<nbatch, nt, fit_smem(nbath, nt), c->stream>>>(A);
    DM_CHECK_LAUNCH();
    c->launches++;
}

// ---------------------------------------------------------------------------
// Lattice side of the self-consistency (Hamiltonian diagonal in spin and
// orbital).  GF arrays are (Nspin,Nspin,Norb,Norb,L) column-major complex128;
// only the diagonal (s,s,a,a) entries are read or written, the rest of the
// output is zero.
__host__ __device__ inline int64_t gf5(int nspin, int norb, int s, int a, int n) {
    return (int64_t)s + nspin * ((int64_t)s + nspin * ((int64_t)a + norb * ((int64_t)a + norb * n)));
}

// G_loc(s,s,a,a,n) = sum_k wt[k] / (z_n + xmu - Sigma(s,s,a,a,n) - he[a*le + k]),
// z_n = i w_n (Matsubara) or w_n + i eps (real axis, eps > 0); k in increasing
// order (the reference adds the k-point terms in turn).
__global__ void k_gloc_diag(int nspin, int norb, int L, int le, const double *__restrict__ he,
                            const double *__restrict__ wt, const double *__restrict__ wm,
                            double xmu, double eps, const double2 *__restrict__ sig,
                            double2 *__restrict__ gl) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nspin * norb * L) return;
    const int n = (int)(t % L);
    const int sa = (int)(t / L), s = sa % nspin, a = sa / nspin;
    const int64_t o = gf5(nspin, norb, s, a, n);
    const double2 sg = sig[o];
    const bool real_axis = eps > 0.0;
    const double zr = xmu - sg.x + (real_axis ? wm[n] : 0.0);
    const double zi = (real_axis ? eps : wm[n]) - sg.y;
    double gr = 0.0, gi = 0.0;
    for (int k = 0; k < le; k++) {
        const double dr = zr - he[(int64_t)a * le + k];
        const double den = wt[k] / (dr * dr + zi * zi);
        gr += dr * den;
        gi += -zi * den;
    }
    gl[o] = make_double2(gr, gi);
}

// scheme 1 (weiss): G0 = 1/(1/G_loc + Sigma); scheme 0 (delta):
// Delta = i w_n + xmu - Hloc_aa - Sigma - 1/G_loc.
__global__ void k_weiss_diag(int nspin, int norb, int L, int scheme, double xmu,
                             const double *__restrict__ hloc_aa, const double *__restrict__ wm,
                             const double2 *__restrict__ gl, const double2 *__restrict__ sig,
                             double2 *__restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nspin * norb * L) return;
    const int n = (int)(t % L);
    const int sa = (int)(t / L), s = sa % nspin, a = sa / nspin;
    const int64_t o = gf5(nspin, norb, s, a, n);
    const double2 G = gl[o], sg = sig[o];
    const double den = 1.0 / (G.x * G.x + G.y * G.y);
    const double ir = G.x * den, ii = -G.y * den;  // 1/G
    if (scheme == 1) {
        const double ar = ir + sg.x, ai = ii + sg.y;
        const double d2 = 1.0 / (ar * ar + ai * ai);
        out[o] = make_double2(ar * d2, -ai * d2);
    } else {
        out[o] = make_double2(xmu - hloc_aa[s * norb + a] - sg.x - ir, wm[n] - sg.y - ii);
    }
}

void gloc_diag_device(dmfted_ctx *c, int L, int le, const double *he, const double *wt,
                      const double *wm, double eps, const double *sig, double *gl) {
    const int ns = c->nspin, no = c->norb;
    DM_CUDA(cudaMemsetAsync(gl, 0, (size_t)ns * ns * no * no * L * 16, c->stream));
    const int64_t n = (int64_t)ns * no * L;
    k_gloc_diag<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        ns, no, L, le, he, wt, wm, c->p.xmu, eps, reinterpret_cast<const double2 *>(sig),
        reinterpret_cast<double2 *>(gl));
    DM_CHECK_LAUNCH();
    c->launches++;
}

void weiss_diag_device(dmfted_ctx *c, int L, int scheme, const double *hloc_aa, const double *wm,
                       const double *gl, const double *sig, double *out) {
    const int ns = c->nspin, no = c->norb;
    DM_CUDA(cudaMemsetAsync(out, 0, (size_t)ns * ns * no * no * L * 16, c->stream));
    const int64_t n = (int64_t)ns * no * L;
    k_weiss_diag<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        ns, no, L, scheme, c->p.xmu, hloc_aa, wm, reinterpret_cast<const double2 *>(gl),
        reinterpret_cast<const double2 *>(sig), reinterpret_cast<double2 *>(out));
    DM_CHECK_LAUNCH();
    c->launches++;
}

}  // namespace dmfted
