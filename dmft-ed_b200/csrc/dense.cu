// Dense eigensolve of small sectors: the branch of ed_diag_c that builds the
// sector Hamiltonian as a dense matrix and calls eigh instead of the Lanczos
// solver, taken when dim <= lanc_dim_threshold or Neigen == dim
// (ED_DIAG.f90:136-137,184-194).
//
// One CTA of kDenseThreads threads solves one sector, and the CTAs of a launch
// take sectors from an atomic queue, largest first.  The matrix is built from
// the context's factored hop tables (the elements ed_buildH_c inserts,
// build_h.f90:29-53 with Himp/Hint/Hbath/Himp_bath), then:
//   1. Householder tridiagonalisation A = Q T Q^T (the unblocked reduction of
//      LAPACK's dsytd2: per column a reflector H = I - tau v v^T, then the
//      trailing block updated by the rank-2 form A - v w^T - w v^T with
//      w = p - (tau/2)(p.v) v, p = tau A v); v overwrites the column below the
//      diagonal and tau the diagonal entry, which T has already taken;
//   2. the lowest m eigenpairs of T by Sturm multisection and inverse
//      iteration (tridiag.cuh), with clusters of equal eigenvalues -- a sector
//      holding several ground states -- given an orthonormal basis of their
//      invariant subspace;
//   3. the back-transformation x = H_0 H_1 ... H_{n-3} y of those m vectors.
// A lives in global memory (L2-resident: 0.5 MB at the default threshold of
// 256 states); the reflector and the product vectors live in shared memory.
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "jterms.cuh"
#include "sector.cuh"
#include "tridiag.cuh"

namespace dmfted {

constexpr int kDenseThreads = 1024;


// Sum over the block of one double per thread (plain FP64), returned in every
// thread.  red: 32 doubles of shared memory.
__device__ __forceinline__ double dense_block_sum(double x, double *red) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    return t;
}

__global__ void __launch_bounds__(kDenseThreads, 1)
    k_dense_eigs(const BatchTables<double> tb, const DenseJob *jobs, int njobs, unsigned *queue,
                 double *work, double *vecs, double *evals, int64_t work_cap, int64_t vec_cap,
                 int ritz_cap) {
    extern __shared__ double dyn[];  // T (a, b), then the Ritz work space
    __shared__ double s_v[kDenseMaxDim], s_p[kDenseMaxDim];
    __shared__ double s_red[32];
    __shared__ double s_ev[kDenseMaxEigen], s_est[kDenseMaxEigen];
    __shared__ double s_tau, s_k;
    __shared__ int s_job;
    const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = bd >> 5;
    const int ni = 1 << tb.norb;
    const uint32_t imask = (uint32_t)ni - 1u;
    for (;;) {
        if (tid == 0) s_job = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int jid = s_job;
        __syncthreads();
        if (jid >= njobs) break;
        const DenseJob J = jobs[jid];
        const int n = J.n;
        if (!DM_IN(J.a_off + (int64_t)n * n - 1, work_cap) ||
            !DM_IN(J.out_off + (int64_t)J.m * n - 1, vec_cap) || !DM_IN(n, kDenseMaxDim + 1) ||
            !DM_IN(J.m, kDenseMaxEigen + 1) || !DM_IN(2 * n, ritz_cap + 1))
            continue;
        double *A = work + J.a_off;
        const Sec<double> s = make_sec(tb, J.nup, J.ndw);
        for (int64_t t = tid; t < (int64_t)n * n; t += bd) A[t] = 0.0;
        __syncthreads();
        // row i = r + DimUp*q: diagonal, up hops (same column q), down hops
        // (same row r of the neighbouring columns)
        for (int i = tid; i < n; i += bd) {
            const uint32_t r = (uint32_t)i % s.dimup, q = (uint32_t)i / s.dimup;
            double *row = A + (int64_t)i * n;
            row[i] = s.du[r] + s.dd[q] + tb.dint[(s.wu[r] & imask) * ni + (s.wd[q] & imask)];
            for (int e = 0; e < s.cu[r]; e++) {
                const uint32_t en = s.eu[(int64_t)e * s.dimup + r];
                if (!DM_IN(ell_par(en), tb.P) || !DM_IN(ell_col(en), s.dimup)) continue;
                const double v = tb.sp[0].par[ell_par(en)];
                row[s.dimup * q + ell_col(en)] += ell_neg(en) ? -v : v;
            }
            for (int e = 0; e < s.cd[q]; e++) {
                const uint32_t en = s.ed[(int64_t)e * s.dimdw + q];
                if (!DM_IN(ell_par(en), tb.P) || !DM_IN(ell_col(en), s.dimdw)) continue;
                const double v = tb.sp[1].par[ell_par(en)];
                row[s.dimup * ell_col(en) + r] += ell_neg(en) ? -v : v;
            }
            if (tb.jx != 0.0 || tb.jp != 0.0)
                for_jterms(s.wu[r], s.wd[q], tb.norb, tb.jx, tb.jp,
                           [&](uint32_t tu, uint32_t td, double cf) {
                               const int64_t j = tb.rank[tu] + (int64_t)s.dimup * tb.rank[td];
                               if (DM_IN(j, n)) row[j] += cf;
                           });
        }
        __syncthreads();
        double *sa = dyn, *sb = dyn + n;
        if (tid == 0) sb[0] = 0.0;
        // ---- 1. tridiagonalisation -------------------------------------------
        for (int k = 0; k + 1 < n; k++) {
            const int m = n - k - 1;  // length of the column below the diagonal
            double part = 0.0;
            for (int i = tid; i < m; i += bd) {
                const double x = A[(int64_t)(k + 1 + i) * n + k];
                s_v[i] = x;
                if (i > 0) part += x * x;
            }
            const double tail = dense_block_sum(part, s_red);  // |x|^2 without x_0
            if (tid == 0) {
                const double x0 = s_v[0];
                sa[k] = A[(int64_t)k * n + k];
                if (m == 1 || tail == 0.0) {
                    s_tau = 0.0;  // already tridiagonal in this column
                    sb[k + 1] = x0;
                } else {
                    const double nx = sqrt(x0 * x0 + tail);
                    const double alpha = x0 >= 0.0 ? -nx : nx;
                    const double v0 = x0 - alpha;
                    s_v[0] = v0;
                    s_tau = 2.0 / (v0 * v0 + tail);
                    sb[k + 1] = alpha;
                }
                A[(int64_t)k * n + k] = s_tau;  // T holds a_k now; keep tau here
            }
            __syncthreads();
            const double tau = s_tau;
            if (tau == 0.0) continue;
            for (int i = tid; i < m; i += bd) A[(int64_t)(k + 1 + i) * n + k] = s_v[i];
            // p = tau A_sub v, one warp per row
            for (int i = warp; i < m; i += nwarp) {
                const double *row = A + (int64_t)(k + 1 + i) * n + (k + 1);
                double d = 0.0;
                for (int j = lane; j < m; j += 32) d += row[j] * s_v[j];
                for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                if (lane == 0) s_p[i] = tau * d;
            }
            __syncthreads();
            part = 0.0;
            for (int i = tid; i < m; i += bd) part += s_p[i] * s_v[i];
            const double kk = 0.5 * tau * dense_block_sum(part, s_red);
            for (int i = tid; i < m; i += bd) s_p[i] -= kk * s_v[i];  // w
            __syncthreads();
            // A_sub -= v w^T + w v^T
            for (int64_t t = tid; t < (int64_t)m * m; t += bd) {
                const int i = (int)(t / m), j = (int)(t % m);
                A[(int64_t)(k + 1 + i) * n + (k + 1 + j)] -= s_v[i] * s_p[j] + s_p[i] * s_v[j];
            }
            __syncthreads();
        }
        if (tid == 0) sa[n - 1] = A[(int64_t)(n - 1) * n + (n - 1)];
        __syncthreads();
        // ---- 2. lowest m eigenpairs of T ---------------------------------------
        double *Y = vecs + J.out_off;
        ritz_multi_dev(sa, sb, n, J.m, 1.0, 0.0, s_ev, Y, s_est, dyn + 2 * n, ritz_cap - 2 * n);
        // ---- 3. back-transformation x = H_0 ... H_{n-3} y ----------------------
        for (int k = n - 2; k >= 0; k--) {
            const double tau = A[(int64_t)k * n + k];
            if (tau == 0.0) continue;  // uniform: every thread reads the same value
            const int m = n - k - 1;
            for (int i = tid; i < m; i += bd) s_v[i] = A[(int64_t)(k + 1 + i) * n + k];
            __syncthreads();
            for (int j = warp; j < J.m; j += nwarp) {
                double *y = Y + (int64_t)j * n + (k + 1);
                double d = 0.0;
                for (int i = lane; i < m; i += 32) d += s_v[i] * y[i];
                for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                d *= tau;
                for (int i = lane; i < m; i += 32) y[i] -= d * s_v[i];
            }
            __syncthreads();
        }
        for (int j = tid; j < J.m; j += bd) evals[(int64_t)J.slot * kDenseMaxEigen + j] = s_ev[j];
        __syncthreads();
    }
}

// Dynamic shared memory of k_dense_eigs for sectors of up to n states and m
// eigenpairs: T (2n) and as many inverse-iteration work spaces (up to 8) as
// fit in 190 KB.  Returns the size in doubles.
static int dense_ritz_doubles(int n, int m) {
    const int per = ritz_evec_doubles(n);
    int lanes = std::max(1, std::min(8, m));
    while (lanes > 1 && (2 * n + lanes * per) * 8 > 190 * 1024) lanes--;
    return 2 * n + lanes * per;
}

// Host side: the lowest want[i] eigenpairs of every sector list[i] whose
// want[i] > 0, in one persistent launch.  dense_eigs_launch queues the work on
// the context's stream and returns without waiting; dense_eigs_collect waits
// for it and fills the results.
void dense_eigs_launch(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                       DensePending &pd) {
    pd = DensePending();
    pd.nlist = list.size();
    std::vector<DenseJob> &jobs = pd.jobs;
    std::vector<int> &where = pd.where;
    int64_t work = 0, vec = 0;
    for (size_t i = 0; i < list.size(); i++) {
        if (want[i] <= 0) continue;
        const SectorView s = sector_view(c, list[i]);
        DM_REQUIRE(s.dim <= kDenseMaxDim, DMFTED_ERR_UNSUPPORTED,
                   "dense sector eigensolve beyond " + std::to_string(kDenseMaxDim) + " states");
        DM_REQUIRE(want[i] <= kDenseMaxEigen, DMFTED_ERR_UNSUPPORTED,
                   "dense sector eigensolve: more than " + std::to_string(kDenseMaxEigen) +
                       " eigenpairs of one sector");
        DenseJob J;
        J.nup = s.nup;
        J.ndw = s.ndw;
        J.n = (int)s.dim;
        J.m = (int)std::min<int64_t>(want[i], s.dim);
        J.slot = (int)jobs.size();
        J.a_off = work;
        J.out_off = vec;
        work += ((int64_t)J.n * J.n + 31) / 32 * 32;
        vec += ((int64_t)J.m * J.n + 31) / 32 * 32;
        jobs.push_back(J);
        where.push_back((int)i);
    }
    if (jobs.empty()) return;
    const int nj = (int)jobs.size();
    std::vector<DenseJob> q = jobs;
    std::stable_sort(q.begin(), q.end(), [](const DenseJob &a, const DenseJob &b) {
        return a.n > b.n;
    });
    int nmax = 1, mmax = 1;
    for (auto &J : q) {
        nmax = std::max(nmax, J.n);
        mmax = std::max(mmax, J.m);
    }
    const int rcap = dense_ritz_doubles(nmax, mmax);
    c->dense_work.alloc((size_t)work);
    c->dense_vec.alloc((size_t)vec);
    c->dense_eval.alloc((size_t)nj * kDenseMaxEigen);
    c->dense_int.alloc(1);
    c->dense_jobs.alloc((size_t)nj * sizeof(DenseJob));
    DM_CUDA(cudaMemcpyAsync(c->dense_jobs.p, q.data(), nj * sizeof(DenseJob),
                            cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemsetAsync(c->dense_int.p, 0, sizeof(int), c->stream));
    const int grid = std::min(nj, num_sms(c));
    DM_CUDA(cudaFuncSetAttribute(k_dense_eigs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 rcap * (int)sizeof(double)));
    k_dense_eigs<<<grid, kDenseThreads, rcap * sizeof(double), c->stream>>>(
        batch_tables<double>(c), reinterpret_cast<const DenseJob *>(c->dense_jobs.p), nj,
        reinterpret_cast<unsigned *>(c->dense_int.p), c->dense_work.p, c->dense_vec.p,
        c->dense_eval.p, (int64_t)c->dense_work.n, (int64_t)c->dense_vec.n, rcap);
    DM_CHECK_LAUNCH();
    c->launches++;
    pd.stream = c->stream;
}

void dense_eigs_collect(dmfted_ctx *c, DensePending &pd, std::vector<DenseEig> &res) {
    res.assign(pd.nlist, DenseEig());
    const std::vector<DenseJob> &jobs = pd.jobs;
    const std::vector<int> &where = pd.where;
    const int nj = (int)jobs.size();
    if (nj == 0) return;
    std::vector<double> ev((size_t)nj * kDenseMaxEigen);
    DM_CUDA(cudaMemcpyAsync(ev.data(), c->dense_eval.p, ev.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, pd.stream));
    DM_CUDA(cudaStreamSynchronize(pd.stream));
    for (int j = 0; j < nj; j++) {
        const DenseJob &J = jobs[j];
        DenseEig &r = res[where[j]];
        r.m = J.m;
        r.evals.assign(ev.begin() + (size_t)J.slot * kDenseMaxEigen,
                       ev.begin() + (size_t)J.slot * kDenseMaxEigen + J.m);
        r.vecs = c->dense_vec.p + J.out_off;
    }
}

void dense_eigs(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                std::vector<DenseEig> &res) {
    DensePending pd;
    dense_eigs_launch(c, list, want, pd);
    dense_eigs_collect(c, pd, res);
}

}  // namespace dmfted
