// Dense eigensolve of small sectors: the branch of ed_diag_c that builds the
// sector Hamiltonian as a dense matrix and calls eigh instead of the Lanczos
// solver, taken when dim <= lanc_dim_threshold or Neigen == dim
// (ED_DIAG.f90:136-137,184-194).
//
// One CTA of kDenseThreads threads diagonalises one sector, and the CTAs of a
// launch take sectors from an atomic queue, largest first.  The matrix is
// built from the context's factored hop tables (the elements ed_buildH_c
// inserts, build_h.f90:29-53 with Himp/Hint/Hbath/Himp_bath) and diagonalised
// by the cyclic Jacobi method with the round-robin ("chess tournament")
// ordering of Brent and Luk: every round rotates npad/2 disjoint index pairs
// at once, so the two-sided update J^T A J splits into independent 2 x 2
// blocks and the eigenvector update V J into independent row pairs.  Jacobi
// returns an orthonormal eigenbasis also for exactly degenerate eigenvalues,
// which is what the reference's LAPACK eigh gives and what the ground-state
// selection needs when a sector holds several ground states.  The rotation
// is the symmetric Schur decomposition of Golub and Van Loan (Matrix
// Computations, Alg. 8.4.1).  A and V live in global memory (L2-resident for
// the default threshold, 256 states: 1 MB per sector).
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "sector.cuh"

namespace dmfted {

constexpr int kDenseThreads = 1024;
constexpr int kDenseMaxSweeps = 40;

struct DenseJob {
    int nup, ndw;
    int n, npad;      // sector dimension, padded to even
    int m;            // eigenpairs wanted (lowest m)
    int slot;         // output slot: evals[slot * kDenseMaxEigen + j], sweeps[slot]
    int64_t a_off;    // work: A (npad^2) then V (npad^2)
    int64_t out_off;  // eigenvectors: m x n FP64, vector j at out_off + j*n
};

// Player in slot j (0..npad-1) of round r of the round-robin schedule: slot 0
// keeps player 0, the others rotate.  Slots k and npad-1-k meet.
__device__ __forceinline__ int rr_player(int j, int r, int npad) {
    return j == 0 ? 0 : 1 + (j - 1 + r) % (npad - 1);
}

__global__ void __launch_bounds__(kDenseThreads, 1)
    k_dense_eigs(const BatchTables<double> tb, const DenseJob *jobs, int njobs, unsigned *queue,
                 double *work, double *vecs, double *evals, int *sweeps, int64_t work_cap,
                 int64_t vec_cap) {
    __shared__ int s_p[kDenseMaxDim / 2], s_q[kDenseMaxDim / 2];
    __shared__ double s_c[kDenseMaxDim / 2], s_s[kDenseMaxDim / 2];
    __shared__ double s_red[2 * 32];
    __shared__ double s_tot[2];
    __shared__ int s_job;
    const int tid = threadIdx.x, bd = blockDim.x;
    const int ni = 1 << tb.norb;
    const uint32_t imask = (uint32_t)ni - 1u;
    for (;;) {
        if (tid == 0) s_job = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int jid = s_job;
        __syncthreads();
        if (jid >= njobs) break;
        const DenseJob J = jobs[jid];
        const int n = J.n, np = J.npad, h = np / 2;
        if (!DM_IN(J.a_off + 2 * (int64_t)np * np - 1, work_cap) ||
            !DM_IN(J.out_off + (int64_t)J.m * n - 1, vec_cap) || !DM_IN(np, kDenseMaxDim + 1) ||
            !DM_IN(J.m, kDenseMaxEigen + 1))
            continue;
        double *A = work + J.a_off, *V = A + (int64_t)np * np;
        const Sec<double> s = make_sec(tb, J.nup, J.ndw);
        for (int64_t t = tid; t < (int64_t)np * np; t += bd) {
            const int i = (int)(t / np), j = (int)(t % np);
            A[t] = 0.0;
            V[t] = i == j ? 1.0 : 0.0;
        }
        __syncthreads();
        // row i = r + DimUp*q: diagonal, up hops (same column q), down hops
        // (same row r of the neighbouring columns)
        for (int i = tid; i < n; i += bd) {
            const uint32_t r = (uint32_t)i % s.dimup, q = (uint32_t)i / s.dimup;
            double *row = A + (int64_t)i * np;
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
        }
        __syncthreads();
        int sweep = 0;
        double prev = 0.0;
        for (; sweep < kDenseMaxSweeps; sweep++) {
            // off-diagonal and total squared norms
            double off = 0.0, tot = 0.0;
            for (int64_t t = tid; t < (int64_t)n * np; t += bd) {
                const int i = (int)(t / np), j = (int)(t % np);
                if (j >= n) continue;
                const double a = A[t], a2 = a * a;
                tot += a2;
                if (i != j) off += a2;
            }
            for (int o = 16; o > 0; o >>= 1) {
                off += __shfl_xor_sync(0xffffffffu, off, o);
                tot += __shfl_xor_sync(0xffffffffu, tot, o);
            }
            if ((tid & 31) == 0) {
                s_red[tid >> 5] = off;
                s_red[32 + (tid >> 5)] = tot;
            }
            __syncthreads();
            if (tid == 0) {
                double a = 0.0, b = 0.0;
                for (int w = 0; w < (bd >> 5); w++) {
                    a += s_red[w];
                    b += s_red[32 + w];
                }
                s_tot[0] = a;
                s_tot[1] = b;
            }
            __syncthreads();
            const double offn = s_tot[0], totn = s_tot[1];
            __syncthreads();
            // converged when the off-diagonal norm is below 1e-14 |A|_F, or
            // once it is below 1e-10 |A|_F and a sweep no longer reduces it
            // (rounding level of a large matrix)
            if (!(offn > 1e-28 * totn)) break;
            if (sweep > 0 && offn <= 1e-20 * totn && offn >= 0.25 * prev) break;
            prev = offn;
            for (int round = 0; round < np - 1; round++) {
                for (int k = tid; k < h; k += bd) {
                    int p = rr_player(k, round, np), q = rr_player(np - 1 - k, round, np);
                    if (p > q) {
                        const int t = p;
                        p = q;
                        q = t;
                    }
                    const double app = A[(int64_t)p * np + p], aqq = A[(int64_t)q * np + q];
                    const double apq = A[(int64_t)p * np + q];
                    double c = 1.0, sn = 0.0;
                    if (apq != 0.0) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                    }
                    s_p[k] = p;
                    s_q[k] = q;
                    s_c[k] = c;
                    s_s[k] = sn;
                }
                __syncthreads();
                // A <- J^T A J on the 2 x 2 blocks (rows of pair k1, columns of pair k2)
                for (int b = tid; b < h * h; b += bd) {
                    const int k1 = b / h, k2 = b % h;
                    const int p1 = s_p[k1], q1 = s_q[k1], p2 = s_p[k2], q2 = s_q[k2];
                    const double c1 = s_c[k1], s1 = s_s[k1], c2 = s_c[k2], s2 = s_s[k2];
                    double *r1 = A + (int64_t)p1 * np, *r2 = A + (int64_t)q1 * np;
                    const double x11 = r1[p2], x12 = r1[q2], x21 = r2[p2], x22 = r2[q2];
                    const double y11 = c1 * x11 - s1 * x21, y12 = c1 * x12 - s1 * x22;
                    const double y21 = s1 * x11 + c1 * x21, y22 = s1 * x12 + c1 * x22;
                    double z11 = c2 * y11 - s2 * y12, z12 = s2 * y11 + c2 * y12;
                    double z21 = c2 * y21 - s2 * y22, z22 = s2 * y21 + c2 * y22;
                    if (k1 == k2) z12 = z21 = 0.0;  // the rotated pair is annihilated
                    r1[p2] = z11;
                    r1[q2] = z12;
                    r2[p2] = z21;
                    r2[q2] = z22;
                }
                // V <- V J
                for (int b = tid; b < np * h; b += bd) {
                    const int i = b / h, k = b % h;
                    double *vr = V + (int64_t)i * np;
                    const int p = s_p[k], q = s_q[k];
                    const double c = s_c[k], sn = s_s[k];
                    const double vp = vr[p], vq = vr[q];
                    vr[p] = c * vp - sn * vq;
                    vr[q] = sn * vp + c * vq;
                }
                __syncthreads();
            }
        }
        // rank of each eigenvalue (ties by index); the lowest m are written
        for (int i = tid; i < n; i += bd) {
            const double di = A[(int64_t)i * np + i];
            int rk = 0;
            for (int j = 0; j < n; j++) {
                const double dj = A[(int64_t)j * np + j];
                rk += (dj < di || (dj == di && j < i)) ? 1 : 0;
            }
            if (rk < J.m) {
                evals[(int64_t)J.slot * kDenseMaxEigen + rk] = di;
                s_p[rk] = i;  // column of V (the pair arrays are free now)
            }
        }
        __syncthreads();
        for (int64_t t = tid; t < (int64_t)J.m * n; t += bd) {
            const int j = (int)(t / n), row = (int)(t % n);
            vecs[J.out_off + t] = V[(int64_t)row * np + s_p[j]];
        }
        if (tid == 0) sweeps[J.slot] = sweep;
        __syncthreads();
    }
}

// Host side: the lowest want[i] eigenpairs of every sector list[i] whose
// want[i] > 0, in one persistent launch.
void dense_eigs(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                std::vector<DenseEig> &res) {
    res.assign(list.size(), DenseEig());
    std::vector<DenseJob> jobs;
    std::vector<int> where;
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
        J.npad = (int)((s.dim + 1) / 2 * 2);
        if (J.npad < 2) J.npad = 2;
        J.m = (int)std::min<int64_t>(want[i], s.dim);
        J.slot = (int)jobs.size();
        J.a_off = work;
        J.out_off = vec;
        work += 2 * (int64_t)J.npad * J.npad;
        vec += ((int64_t)J.m * J.n + 31) / 32 * 32;
        jobs.push_back(J);
        where.push_back((int)i);
    }
    if (jobs.empty()) return;
    const int nj = (int)jobs.size();
    std::vector<DenseJob> q = jobs;
    std::stable_sort(q.begin(), q.end(), [](const DenseJob &a, const DenseJob &b) {
        return a.npad > b.npad;
    });
    c->dense_work.alloc((size_t)work);
    c->dense_vec.alloc((size_t)vec);
    c->dense_eval.alloc((size_t)nj * kDenseMaxEigen);
    c->dense_int.alloc((size_t)nj + 1);
    c->dense_jobs.alloc((size_t)nj * sizeof(DenseJob));
    DM_CUDA(cudaMemcpyAsync(c->dense_jobs.p, q.data(), nj * sizeof(DenseJob),
                            cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemsetAsync(c->dense_int.p + nj, 0, sizeof(int), c->stream));
    const int grid = std::min(nj, num_sms(c));
    k_dense_eigs<<<grid, kDenseThreads, 0, c->stream>>>(
        batch_tables<double>(c), reinterpret_cast<const DenseJob *>(c->dense_jobs.p), nj,
        reinterpret_cast<unsigned *>(c->dense_int.p + nj), c->dense_work.p, c->dense_vec.p,
        c->dense_eval.p, c->dense_int.p, (int64_t)c->dense_work.n, (int64_t)c->dense_vec.n);
    DM_CHECK_LAUNCH();
    c->launches++;
    std::vector<double> ev((size_t)nj * kDenseMaxEigen);
    std::vector<int> sw(nj);
    DM_CUDA(cudaMemcpyAsync(ev.data(), c->dense_eval.p, ev.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaMemcpyAsync(sw.data(), c->dense_int.p, nj * sizeof(int), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < nj; j++) {
        const DenseJob &J = jobs[j];
        DenseEig &r = res[where[j]];
        r.m = J.m;
        r.sweeps = sw[J.slot];
        r.evals.assign(ev.begin() + (size_t)J.slot * kDenseMaxEigen,
                       ev.begin() + (size_t)J.slot * kDenseMaxEigen + J.m);
        r.vecs = c->dense_vec.p + J.out_off;
        DM_REQUIRE(r.sweeps < kDenseMaxSweeps, DMFTED_ERR_NOTCONV,
                   "dense sector eigensolve: Jacobi sweeps did not converge");
    }
}

}  // namespace dmfted
