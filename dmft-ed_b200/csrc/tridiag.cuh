// Device routines on the Lanczos tridiagonal T_n (diagonal a[0..n),
// off-diagonal b[1..n)) shared by the grid-wide and the batched solvers:
// Sturm-sequence multisection for eigenvalues, inverse iteration for
// eigenvectors, the ARPACK-style Ritz test on the lowest m pairs, and the
// seeded random start vector.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace dmfted {

constexpr int kTridiagMaxThreads = 1024;  // block size limit of tridiag_eig

// (seed, i) -> uniform (0, 1]: splitmix64 of the element index, the real
// counterpart of the seeded random resid the reference hands ARPACK
// (.repo/ARPACK_LANCZOS.f90:394-403).
__device__ __forceinline__ double random_start_value(int64_t i, uint64_t seed) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return ((double)(z >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

// Sturm count: number of eigenvalues of the n x n tridiagonal (a, b[1..n-1])
// below x.  (The division-free product form of the leading minors was
// measured too: faster per count in a 256-thread block, but slower in the
// batched eigensolver's 1024-thread blocks, where the counts are bound by
// FP64 issue rather than by the latency of the division chain.)
__device__ inline int sturm_count(const double *a, const double *b, int n, double x, double pivmin) {
    int cnt = 0;
    double q = a[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0.0) cnt++;
    for (int i = 1; i < n; i++) {
        q = (a[i] - x) - b[i] * b[i] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0.0) cnt++;
    }
    return cnt;
}

// j-th lowest eigenvalue (0-based) of T_n by multisection with all threads of
// the block (at most kTridiagMaxThreads); a, b in shared memory.  Returns the
// value in every thread.
__device__ inline double tridiag_eig(const double *a, const double *b, int n, int j) {
    __shared__ int cnts[kTridiagMaxThreads];
    __shared__ double lohi[2];
    if (threadIdx.x == 0) {
        double lo = a[0], hi = a[0], amax = 0.0;
        for (int i = 0; i < n; i++) {
            const double r = (i > 0 ? fabs(b[i]) : 0.0) + (i + 1 < n ? fabs(b[i + 1]) : 0.0);
            lo = fmin(lo, a[i] - r);
            hi = fmax(hi, a[i] + r);
            amax = fmax(amax, fabs(a[i]) + r);
        }
        const double pad = 2.2e-16 * fmax(amax, 1e-300) * 4.0 + 1e-300;
        lohi[0] = lo - pad;
        lohi[1] = hi + pad;
    }
    __syncthreads();
    double amax = fmax(fabs(lohi[0]), fabs(lohi[1]));
    const double pivmin = 1e-300 + 2.2e-16 * 2.2e-16 * fmax(amax * amax, 1e-300);
    for (int round = 0; round < 40; round++) {
        const double lo = lohi[0], hi = lohi[1];
        if (hi - lo <= 2.0 * 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
        const int nt = blockDim.x;
        const double x = lo + (hi - lo) * (double)(threadIdx.x + 1) / (double)(nt + 1);
        cnts[threadIdx.x] = sturm_count(a, b, n, x, pivmin);
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            while (t < nt && cnts[t] <= j) t++;
            const double nlo = t == 0 ? lo : lo + (hi - lo) * (double)t / (double)(nt + 1);
            const double nhi = t == nt ? hi : lo + (hi - lo) * (double)(t + 1) / (double)(nt + 1);
            lohi[0] = nlo;
            lohi[1] = nhi;
        }
        __syncthreads();
    }
    const double r = 0.5 * (lohi[0] + lohi[1]);
    __syncthreads();
    return r;
}

// Eigenvector y of T_n (diag a[0..n), off-diagonal b[1..n)) for eigenvalue
// lam: three steps of inverse iteration, Gaussian elimination with partial
// pivoting on the tridiagonal.  Single thread.  ws: 5n doubles, sw: n bytes.
// nprev > 0: lam belongs to a cluster of eigenvalues (several copies of an
// eigenvalue, as a Lanczos run past rounding-level growth of a degenerate
// partner holds them) and prev[q*n..] (q < nprev) are the eigenvectors of
// the cluster's lower members.  Inverse iteration alone would return the same
// vector for every member; as in LAPACK's dstein, the iteration then starts
// from a pseudo-random vector (seed: the member's index) and is
// re-orthogonalised against the lower members after every solve, which
// converges to an orthonormal basis of the cluster's invariant subspace.
__device__ inline void tridiag_evec(const double *a, const double *b, int n, double lam, double *yv,
                             double *ws, unsigned char *sw, const double *prev = nullptr,
                             int nprev = 0) {
    double *D = ws, *U1 = ws + n, *U2 = ws + 2 * n, *M = ws + 3 * n;
    double nrm = 0.0;
    for (int i = 0; i < n; i++) nrm = fmax(nrm, fabs(a[i] - lam) + (i > 0 ? fabs(b[i]) : 0.0));
    // the replacement of a zero pivot; T - lam = 0 (a 1 x 1 sector, or lam I)
    // has no scale of its own, and 1e-15 keeps 1/tiny and the squares of the
    // solve finite
    const double tiny = (nrm > 1e-290 ? nrm : 1.0) * 1e-15;
    double d = a[0] - lam, u1 = n > 1 ? b[1] : 0.0, u2 = 0.0;
    for (int i = 0; i < n - 1; i++) {
        const double l = b[i + 1], dn = a[i + 1] - lam, un = (i + 2 < n) ? b[i + 2] : 0.0;
        if (fabs(d) >= fabs(l)) {
            if (d == 0.0) d = tiny;
            const double m = l / d;
            D[i] = d; U1[i] = u1; U2[i] = u2; M[i] = m; sw[i] = 0;
            d = dn - m * u1;
            u1 = un - m * u2;
            u2 = 0.0;
        } else {
            const double m = d / l;
            D[i] = l; U1[i] = dn; U2[i] = un; M[i] = m; sw[i] = 1;
            d = u1 - m * dn;
            u1 = u2 - m * un;
            u2 = 0.0;
        }
    }
    if (d == 0.0) d = tiny;
    D[n - 1] = d;
    // reciprocal pivots: independent divisions here, multiplications on the
    // serial back substitutions below
    for (int i = 0; i < n; i++) D[i] = 1.0 / D[i];
    if (nprev > 0)
        for (int i = 0; i < n; i++) yv[i] = random_start_value(i, 977ull + 131ull * (uint64_t)nprev) - 0.5;
    else
        for (int i = 0; i < n; i++) yv[i] = 1.0 / sqrt((double)n);
    const int iters = nprev > 0 ? 5 : 3;
    for (int it = 0; it < iters; it++) {
        for (int i = 0; i < n - 1; i++) {
            if (sw[i]) {
                const double t = yv[i];
                yv[i] = yv[i + 1];
                yv[i + 1] = t;
            }
            yv[i + 1] -= M[i] * yv[i];
        }
        yv[n - 1] *= D[n - 1];
        if (n > 1) yv[n - 2] = (yv[n - 2] - U1[n - 2] * yv[n - 1]) * D[n - 2];
        for (int i = n - 3; i >= 0; i--) yv[i] = (yv[i] - U1[i] * yv[i + 1] - U2[i] * yv[i + 2]) * D[i];
        for (int rep = 0; rep < 2 && nprev > 0; rep++)
            for (int q = 0; q < nprev; q++) {
                const double *pq = prev + (int64_t)q * n;
                double d = 0.0;
                for (int i = 0; i < n; i++) d += pq[i] * yv[i];
                for (int i = 0; i < n; i++) yv[i] -= d * pq[i];
            }
        double ss = 0.0;
        for (int i = 0; i < n; i++) ss += yv[i] * yv[i];
        ss = 1.0 / sqrt(ss);
        for (int i = 0; i < n; i++) yv[i] *= ss;
    }
    const double sg = yv[0] < 0.0 ? -1.0 : 1.0;  // deterministic sign
    for (int i = 0; i < n; i++) yv[i] *= sg;
}

// Lowest m eigenvalues of T_n, one warp per eigenvalue (warp w takes j = w,
// w + nwarps, ...), all warps at once: multisection on 32 points per round,
// the new bracket between the last lane whose Sturm count is at most j and the
// next (a ballot, no block barrier).  Sturm counts are latency-bound chains,
// so 32 points per eigenvalue in parallel cost far less than the whole block
// on one eigenvalue after another.  a, b in shared memory; lane 0 writes
// evals[j]; the caller synchronises the block before reading them.
__device__ inline void tridiag_eigs_warp(const double *a, const double *b, int n, int m,
                                         double *evals) {
    const int lane = threadIdx.x & 31, nw = (int)(blockDim.x >> 5);
    double lo = INFINITY, hi = -INFINITY, amax = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double r = (i > 0 ? fabs(b[i]) : 0.0) + (i + 1 < n ? fabs(b[i + 1]) : 0.0);
        lo = fmin(lo, a[i] - r);
        hi = fmax(hi, a[i] + r);
        amax = fmax(amax, fabs(a[i]) + r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    }
    const double pad = 2.2e-16 * fmax(amax, 1e-300) * 4.0 + 1e-300;
    lo -= pad;
    hi += pad;
    const double am = fmax(fabs(lo), fabs(hi));
    const double pivmin = 1e-300 + 2.2e-16 * 2.2e-16 * fmax(am * am, 1e-300);
    for (int j = (int)(threadIdx.x >> 5); j < m; j += nw) {
        double l = lo, h = hi;
        for (int round = 0; round < 96; round++) {
            if (h - l <= 2.0 * 2.2e-16 * fmax(fabs(l), fabs(h)) + 1e-300) break;
            const double x = l + (h - l) * (double)(lane + 1) / 33.0;
            const unsigned below = __ballot_sync(0xffffffffu, sturm_count(a, b, n, x, pivmin) <= j);
            const int t = below == 0xffffffffu ? 32 : __ffs(~below) - 1;
            const double nl = t == 0 ? l : l + (h - l) * (double)t / 33.0;
            const double nh = t == 32 ? h : l + (h - l) * (double)(t + 1) / 33.0;
            l = nl;
            h = nh;
        }
        if (lane == 0) evals[j] = 0.5 * (l + h);
    }
}

// Dynamic shared memory of the two Ritz kernels for n steps.
__host__ __device__ inline size_t ritz_smem(int n) { return (size_t)8 * n * sizeof(double) + n + 16; }

// Doubles of one eigenvector work space of ritz_multi_dev (vector, the four
// factor arrays of tridiag_evec, its pivot flags).
__host__ __device__ inline int ritz_evec_doubles(int n) { return 5 * n + (n + 7) / 8 + 1; }

// Lowest min(mwant, n) Ritz pairs of T_n with all threads of the block: a, b
// in shared memory, work = work_cap doubles of shared memory after them (at
// least ritz_evec_doubles(n)).  evals[j], Y[j*n + i] (eigenvector j, first
// component positive, re-orthogonalised against the lower ones in the small
// space) and the Ritz estimate est[j] = b_n |Y[j*n + n-1]|.  Returns, in every
// thread, whether every estimate passes ARPACK's test est <= tol *
// max(eps^(2/3), |theta|).  The eigenvalues are found one warp each; the
// inverse iterations run on lane 0 of as many warps as work spaces fit in
// work; the re-orthogonalisation, in order of j, on thread 0.
__device__ inline bool ritz_multi_dev(const double *sa, const double *sb, int n, int mwant,
                                      double tol, double bn, double *evals, double *Y, double *est,
                                      double *work, int work_cap) {
    __shared__ int okflag;
    if (threadIdx.x == 0) okflag = 1;
    const int m = min(mwant, n);
    tridiag_eigs_warp(sa, sb, n, m, evals);
    __syncthreads();
    const int per = ritz_evec_doubles(n);
    const int lanes = max(1, min(min(m, work_cap / per), (int)(blockDim.x >> 5)));
    const int w = (int)(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0 && w < lanes) {
        double *yv = work + (size_t)w * per, *ws = yv + n;
        unsigned char *sw = reinterpret_cast<unsigned char *>(ws + 4 * n);
        // clusters: consecutive eigenvalues closer than 1e-3 |T| (dstein's
        // ORTOL); lane w takes clusters w, w + lanes, ..., each member in turn
        double tn = 0.0;
        for (int i = 0; i < n; i++)
            tn = fmax(tn, fabs(sa[i]) + (i > 0 ? fabs(sb[i]) : 0.0) + (i + 1 < n ? fabs(sb[i + 1]) : 0.0));
        const double ortol = 1e-3 * tn;
        int g = -1;
        for (int j = 0, head = 0; j < m; j++) {
            if (j == 0 || evals[j] - evals[j - 1] > ortol) {
                head = j;
                g++;
            }
            if (g % lanes != w) continue;
            tridiag_evec(sa, sb, n, evals[j], yv, ws, sw, Y + (int64_t)head * n, j - head);
            for (int i = 0; i < n; i++) Y[(int64_t)j * n + i] = yv[i];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < m; j++) {
            double *yj = Y + (int64_t)j * n;
            // orthogonalise against the lower eigenvectors (close eigenvalues)
            for (int q = 0; q < j; q++) {
                double d = 0.0;
                for (int i = 0; i < n; i++) d += Y[(int64_t)q * n + i] * yj[i];
                for (int i = 0; i < n; i++) yj[i] -= d * Y[(int64_t)q * n + i];
            }
            double nr = 0.0;
            for (int i = 0; i < n; i++) nr += yj[i] * yj[i];
            nr = 1.0 / sqrt(nr);
            const double sg = yj[0] < 0.0 ? -nr : nr;
            for (int i = 0; i < n; i++) yj[i] *= sg;
            est[j] = fabs(bn) * fabs(yj[n - 1]);
            const double eps23 = 3.666852862501036e-11;
            if (!(est[j] <= tol * fmax(eps23, fabs(evals[j])))) okflag = 0;
        }
    }
    __syncthreads();
    const bool ok = okflag != 0;
    __syncthreads();
    return ok;
}

}  // namespace dmfted
