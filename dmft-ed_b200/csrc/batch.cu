// Persistent work-queue kernels for many small sectors at once.
//
// At finite temperature the solver diagonalises every (nup, ndw) sector
// (ed_diag_c, ED_DIAG.f90:93-228) and then runs the particle and hole chains
// of every kept state, spin and orbital (lanc_build_gf_normal_c,
// build_gf_normal.f90:71-180).  For a two-orbital bath (Ns = 10) the sectors
// hold at most 63,504 states: one grid-wide launch per Lanczos step leaves
// the GPU idle and costs a launch per step.  Here one CTA of kBatchThreads
// threads runs one job from start to finish -- a chain or a sector's
// eigensolve -- with block-level reductions and no host round trip, and the
// CTAs of one launch take jobs from an atomic queue in the order the host
// sorted them (largest first).  The vectors of a job stay in L1/L2.
// Large sectors are shared by a thread-block cluster of CL CTAs (one per
// SM): the elements are interleaved over the CTAs, every sum folds the CTAs'
// partials in rank order through distributed shared memory (so all CTAs
// hold identical scalars), and the cluster barrier orders each pass's vector
// writes before the next pass's gathers.
//
// The arithmetic follows the grid-wide path step for step (the same
// recurrence, unnormalised vectors with FP64 scales, compensated FP64 sums,
// the same start vectors and stopping tests); only the order in which
// partial sums are combined differs.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "internal.cuh"
#include "jterms.cuh"
#include "reduce.cuh"
#include "sector.cuh"
#include "tridiag.cuh"

namespace cg = cooperative_groups;

namespace dmfted {

constexpr int kBatchThreads = 1024;  // one CTA per SM runs one job at a time

// Couplings of both spins and the impurity diagonal, staged once per CTA.
template <typename T>
struct BatchSmem {
    T pu[kMaxParams], pd[kMaxParams], dint[64];
    double red[2 * 8 * 32];
    double bc[8];
    double cpart[2][8][2];  // block partials read by the other CTAs of the cluster
    int parity;             // which cpart buffer the next sum writes
    int job, jobl;
};

template <typename T>
__device__ void stage_tables(const BatchTables<T> &tb, BatchSmem<T> &sm) {
    for (int i = threadIdx.x; i < tb.P; i += blockDim.x) {
        sm.pu[i] = tb.sp[0].par[i];
        sm.pd[i] = tb.sp[1].par[i];
    }
    const int ni = 1 << tb.norb;
    for (int i = threadIdx.x; i < ni * ni; i += blockDim.x) sm.dint[i] = tb.dint[i];
    if (threadIdx.x == 0) sm.parity = 0;
    __syncthreads();
}

// (H x)_i for element i = r + DimUp*q: impurity and bath diagonal, then the
// up hops (rows of the same column) and the down hops (same row of the
// neighbouring columns), as the grid-wide kernel.
template <typename T>
__device__ __forceinline__ T hx_elem(const Sec<T> &s, const BatchSmem<T> &sm, int ni, int W, int P,
                                     const T *x, uint32_t r, uint32_t q) {
    const uint32_t imask = (uint32_t)ni - 1u;
    const uint32_t base = s.dimup * q;
    T h = (s.du[r] + s.dd[q] + sm.dint[(s.wu[r] & imask) * ni + (s.wd[q] & imask)]) * x[base + r];
    const int cu = s.cu[r];
    for (int e = 0; e < cu; e++) {
        if (!DM_IN(e, W)) break;
        const uint32_t en = s.eu[(int64_t)e * s.dimup + r];
        if (!DM_IN(ell_par(en), P) || !DM_IN(ell_col(en), s.dimup)) continue;
        const T v = sm.pu[ell_par(en)];
        h += (ell_neg(en) ? -v : v) * x[base + ell_col(en)];
    }
    const int cd = s.cd[q];
    for (int e = 0; e < cd; e++) {
        if (!DM_IN(e, W)) break;
        const uint32_t en = s.ed[(int64_t)e * s.dimdw + q];
        if (!DM_IN(ell_par(en), P) || !DM_IN(ell_col(en), s.dimdw)) continue;
        const T v = sm.pd[ell_par(en)];
        h += (ell_neg(en) ? -v : v) * x[s.dimup * ell_col(en) + r];
    }
    return h;
}

// The Jhflag terms of (H x)_i, i = r + DimUp*q (zero without Jhflag).
template <typename T>
__device__ __forceinline__ T hx_jterms(const BatchTables<T> &tb, const Sec<T> &s, const T *x,
                                       uint32_t r, uint32_t q) {
    double h = 0.0;
    for_jterms(s.wu[r], s.wd[q], tb.norb, tb.jx, tb.jp, [&](uint32_t tu, uint32_t td, double cf) {
        const int64_t j = tb.rank[tu] + (int64_t)s.dimup * tb.rank[td];
        if (DM_IN(j, s.dim)) h += cf * (double)x[j];
    });
    return (T)h;
}

template <int CL>
__device__ __forceinline__ int cta_rank() {
    if constexpr (CL == 1) return 0;
    else return (int)cg::this_cluster().block_rank();
}

// Sum of NS compensated partials over the job's CTAs, returned in every
// thread of every CTA.  Cluster partials are double-buffered: a buffer is
// written again only two sums later, after every CTA has passed the barrier
// of the sum in between, i.e. finished reading it.
template <int CL, int NS, typename T>
__device__ __forceinline__ void job_sum(CSum (&a)[NS], BatchSmem<T> &sm, double (&out)[NS]) {
    block_reduce<NS>(a, sm.red);
    if constexpr (CL == 1) {
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NS; k++) sm.bc[k] = a[k].value();
        }
    } else {
        cg::cluster_group cl = cg::this_cluster();
        const int buf = sm.parity;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NS; k++) {
                sm.cpart[buf][k][0] = a[k].hi;
                sm.cpart[buf][k][1] = a[k].lo;
            }
        }
        cl.sync();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < NS; k++) {
                CSum t;
                t.zero();
                for (int r = 0; r < CL; r++) {
                    const double *rp = cl.map_shared_rank(&sm.cpart[buf][k][0], r);
                    t.merge(rp[0], rp[1]);
                }
                sm.bc[k] = t.value();
            }
            sm.parity = buf ^ 1;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NS; k++) out[k] = sm.bc[k];
    __syncthreads();
}

// Next job of the queue for this CTA (CL == 1) or cluster (rank 0 takes it,
// the others read it from rank 0's shared memory).  The closing barrier
// keeps rank 0 from exiting or overwriting the slot before every CTA read it.
template <int CL, typename T>
__device__ __forceinline__ int next_job(unsigned *queue, BatchSmem<T> &sm) {
    if constexpr (CL == 1) {
        if (threadIdx.x == 0) sm.job = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int j = sm.job;
        __syncthreads();
        return j;
    } else {
        cg::cluster_group cl = cg::this_cluster();
        if (cl.block_rank() == 0 && threadIdx.x == 0) sm.job = (int)atomicAdd(queue, 1u);
        cl.sync();
        if (threadIdx.x == 0) sm.jobl = *cl.map_shared_rank(&sm.job, 0);
        cl.sync();
        return sm.jobl;
    }
}

// ---------------------------------------------------------------- chains --
struct ChainJob {
    int tnup, tndw;        // target sector
    int snup;              // source sector's nup (down-spin sign)
    int ispin, iorb, particle;
    int kmax;
    int slot;              // output slot
    int64_t psi_off;       // FP64 state vector in the eigenspace pool
    int64_t work_off;      // elements of T: three vectors of the job
};

// Chain output slot: alpha[kLzMax+2], beta[kLzMax+2], then nsteps and norm2
// in separate arrays.
constexpr int kChainStride = kLzMax + 2;

// One chain, run by CL CTAs (a cluster) or by one CTA.
// Extents of the buffers a batched launch writes or gathers from, checked
// against every job in a checked build (the checks are uniform over the CTAs
// of a cluster, so a skipped job is skipped by all of them).
struct BatchCaps {
    int64_t work, vec, aux, states, slots, lock;
};

template <typename T, int CL>
__device__ void chain_job(const BatchTables<T> &tb, BatchSmem<T> &sm, const ChainJob &J,
                          const double *states64, T *work, double *alpha, double *beta,
                          int *nsteps, double *norm2, double thr, const BatchCaps &cap) {
    const int ni = 1 << tb.norb;
    const int tid = threadIdx.x, bd = blockDim.x;
    const int rank = cta_rank<CL>();
    const bool lead = rank == 0 && tid == 0;  // writes the job's outputs
    const uint32_t i0 = (uint32_t)(rank * bd + tid), st = (uint32_t)(CL * bd);
    const Sec<T> s = make_sec(tb, J.tnup, J.tndw);
    const bool jflag = tb.jx != 0.0 || tb.jp != 0.0;
    const uint32_t dim = s.dim;
    const uint32_t ld = (dim + 31u) & ~31u;
    if (!DM_IN(J.work_off + 2 * (int64_t)ld - 1, cap.work) || !DM_IN(J.slot, cap.slots) ||
        !DM_IN(J.kmax, kChainStride - 1))
        return;
    T *P = work + J.work_off, *Q = P + ld;
    double *al = alpha + (int64_t)J.slot * kChainStride;
    double *be = beta + (int64_t)J.slot * kChainStride;
    // start vector: c^+ / c on the state, gathered through the rank
    // table (the k_apply_op rule, reference order in both sectors)
    const double *psi = states64 + J.psi_off;
    const uint32_t bit = 1u << J.iorb;
    const int64_t sdimup = tb.binom[J.snup];
    CSum n2[1];
    n2[0].zero();
    for (uint32_t i = i0; i < dim; i += st) {
        const uint32_t r = i % s.dimup, q = i / s.dimup;
        const uint32_t wj = J.ispin == 0 ? s.wu[r] : s.wd[q];
        double val = 0.0;
        const bool has = (wj & bit) != 0u;
        if (J.particle ? has : !has) {
            const uint32_t w = J.particle ? (wj ^ bit) : (wj | bit);
            const int64_t rs = DM_IN(w, tb.nrank) ? tb.rank[w] : 0;
            uint32_t par = __popc(w & (bit - 1u)) & 1u;
            int64_t src;
            if (J.ispin == 0) {
                src = rs + sdimup * q;
            } else {
                par ^= (uint32_t)J.snup & 1u;
                src = r + sdimup * rs;
            }
            if (DM_IN(J.psi_off + src, cap.states)) val = par ? -psi[src] : psi[src];
        }
        n2[0].add(val * val);
        const T vt = (T)val;
        Q[i] = vt;
        P[i] = T(0);
    }
    double tot[1];
    job_sum<CL, 1>(n2, sm, tot);
    if (lead) norm2[J.slot] = tot[0];
    // the recurrence normalises the converted vector, as k_lz_init
    CSum c0[1];
    c0[0].zero();
    for (uint32_t i = i0; i < dim; i += st) c0[0].add((double)Q[i] * (double)Q[i]);
    job_sum<CL, 1>(c0, sm, tot);
    double sc = tot[0] > 0.0 ? 1.0 / sqrt(tot[0]) : 0.0, scp = 0.0, bk = 0.0;
    int steps = 0;
    for (int k = 0; k < J.kmax; k++) {
        // u = sc H x - b_k scp v_prev (in place over v_prev), alpha = sc <x, u>
        const double cprev = k > 0 ? bk * scp : 0.0;
        CSum a[1];
        a[0].zero();
        for (uint32_t i = i0; i < dim; i += st) {
            const uint32_t r = i % s.dimup, q = i / s.dimup;
            T h = hx_elem(s, sm, ni, tb.W, tb.P, Q, r, q);
            if (jflag) h += hx_jterms(tb, s, Q, r, q);
            const T u = (T)(sc * (double)h - cprev * (double)P[i]);
            P[i] = u;
            a[0].add((double)Q[i] * (double)u);
        }
        job_sum<CL, 1>(a, sm, tot);
        const double ak = sc * tot[0];
        // w = u - alpha sc x, b_{k+1} = |w|
        const double coef = ak * sc;
        CSum b[1];
        b[0].zero();
        for (uint32_t i = i0; i < dim; i += st) {
            const T w = (T)((double)P[i] - coef * (double)Q[i]);
            P[i] = w;
            b[0].add((double)w * (double)w);
        }
        job_sum<CL, 1>(b, sm, tot);
        const double bn = sqrt(tot[0]);
        if (lead) {
            al[k] = ak;
            be[k + 1] = bn;
        }
        steps = k + 1;
        scp = sc;
        sc = bn > 0.0 ? 1.0 / bn : 0.0;
        bk = bn;
        T *t = P;
        P = Q;
        Q = t;
        if (bn < thr) break;
    }
    if (lead) {
        be[0] = 0.0;
        nsteps[J.slot] = steps;
    }
    __syncthreads();
}

// Chains [0, nbig) are shared by the CTAs of a cluster, the rest run one per
// CTA: clusters take big chains from queue[0] until none is left, then every
// CTA takes small ones from queue[1] on its own.
template <typename T, int CL>
__global__ void __launch_bounds__(kBatchThreads, 1)
    k_batch_chains(const BatchTables<T> tb, const ChainJob *jobs, int nbig, int njobs,
                   unsigned *queue, const double *states64, T *work, double *alpha, double *beta,
                   int *nsteps, double *norm2, double thr, const BatchCaps cap) {
    __shared__ BatchSmem<T> sm;
    stage_tables(tb, sm);
    if constexpr (CL > 1) {
        for (;;) {
            const int jid = next_job<CL>(queue, sm);
            if (jid >= nbig) break;
            chain_job<T, CL>(tb, sm, jobs[jid], states64, work, alpha, beta, nsteps, norm2, thr, cap);
        }
    }
    for (;;) {
        const int jid = nbig + next_job<1>(queue + 1, sm);
        if (jid >= njobs) break;
        chain_job<T, 1>(tb, sm, jobs[jid], states64, work, alpha, beta, nsteps, norm2, thr, cap);
    }
}

// ------------------------------------------------------------ eigensolve --
struct EigsJob {
    int nup, ndw;
    int neigen, kmax;
    int slot;          // output slot: evals, steps
    int64_t basis_off; // elements of T: (kmax + 1) vectors of ld elements
    int64_t vec_off;   // FP64 eigenvectors: neigen x dim
    int64_t aux_off;   // FP64 scratch: Y and coefficients (2 x neigen x kmax)
    int64_t lock_off;  // locked FP64 vectors (dim apart) in the lock pool
    int nlock;         // how many (0: plain run)
    double top;        // probe: eigenvalues above this are not wanted (early stop)
};

constexpr int kEigsChunk = 4;  // basis vectors per reorthogonalisation dot pass
constexpr int kMaxWaves = 64;  // launches of one batched eigensolve (memory budget)
constexpr double kDgks = 0.717;  // second Gram-Schmidt pass below this norm ratio

// FP64 Ritz scratch of one CTA of an eigensolve job: Y and the coefficients
// (neigen x kmax each) and the eigenvalues.
__host__ __device__ inline int64_t eigs_aux_per_cta(int neigen, int kmax) {
    return ((2 * (int64_t)neigen * kmax + kEigsMaxEigen) + 31) / 32 * 32;
}

// Dynamic shared memory of k_batch_eigs: alpha, beta, scale (kEigsMaxSteps+2
// each), the reorthogonalisation coefficients and the Ritz work space.
constexpr int kDpart = 2 * (kEigsMaxSteps + 2);  // reorthogonalisation partials (doubles)
static_assert(kDpart >= 2 * 32 * kEigsChunk, "partials of sliced groups");
__host__ __device__ inline size_t eigs_ritz_doubles() {
    return (ritz_smem(kEigsMaxSteps) + sizeof(double) - 1) / sizeof(double);
}
__host__ __device__ inline size_t eigs_smem() {
    return (size_t)4 * (kEigsMaxSteps + 2) * sizeof(double) + kDpart * sizeof(double) +
           eigs_ritz_doubles() * sizeof(double) + 3 * (size_t)(kEigsMaxSteps + 2) * sizeof(double);
}

// Partial reorthogonalisation (Simon, "The Lanczos algorithm with partial
// reorthogonalization", Math. Comp. 42 (1984)): the level of orthogonality
// w_{k+1,j} = <v_{k+1}, v_j> is estimated by the recurrence that the Lanczos
// relation implies,
//   b_{k+1} w_{k+1,j} = b_{j+1} w_{k,j+1} + (a_j - a_k) w_{k,j} + b_j w_{k,j-1}
//                       - b_k w_{k-1,j}   (+ a rounding term),
// and the new vector is reorthogonalised against the whole basis only when
// max_j |w_{k+1,j}| exceeds sqrt(eps), and then the next vector as well.
// Semi-orthogonality (|w| <= sqrt(eps)) keeps the Ritz values accurate to
// O(eps |H|) and prevents spurious copies of converged eigenvalues; the
// Ritz vectors are accurate to their residual estimates.  A full pass every
// kProEvery steps bounds any error of the estimate.
constexpr int kProEvery = 32;

// Gram-Schmidt coefficients scf[j] = <v_j, y> scale_j, v_j = scale_j B_j,
// for j < nv, over the job's elements.  The warps split into groups of
// kEigsChunk basis vectors x slices of the elements (so that short bases
// still keep every warp busy) and reduce with shuffles; the CTA's partials
// go to dpart (slot (j, slice)), and one cluster exchange folds them in
// (rank, slice) order.  The caller's next cluster barrier (the norm that
// follows) comes before any CTA rewrites dpart.  dpart: kDpart doubles.
template <typename T, int CL>
__device__ void reorth_dots(const T *B, uint32_t ld, int nv, const T *y, uint32_t dim,
                            double *dpart, double *scf, const double *ssc) {
    const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int nw = bd >> 5;
    const int rank = cta_rank<CL>();
    const int ng = (nv + kEigsChunk - 1) / kEigsChunk;
    const int nsl = ng >= nw ? 1 : nw / ng;  // element slices per group
    // this CTA's element blocks (bd elements from rank*bd, CL*bd apart) are
    // dealt to the slices round-robin
    const uint32_t st = (uint32_t)(CL * bd);
    for (int wi = warp; wi < ng * nsl; wi += nw) {
        const int g = wi / nsl, sl = wi % nsl;
        const int j0 = g * kEigsChunk;
        CSum d[kEigsChunk];
#pragma unroll
        for (int t = 0; t < kEigsChunk; t++) d[t].zero();
        for (uint32_t b0 = (uint32_t)(rank * bd) + (uint32_t)sl * st; b0 < dim;
             b0 += (uint32_t)nsl * st) {
            for (uint32_t l = lane; l < (uint32_t)bd; l += 64) {
                const uint32_t i = b0 + l, i2 = i + 32;
                if (i >= dim) break;
                const bool ok2 = l + 32 < (uint32_t)bd && i2 < dim;
                const double yi = (double)y[i];
                const double yi2 = ok2 ? (double)y[i2] : 0.0;
                double p1[kEigsChunk], p2[kEigsChunk];
#pragma unroll
                for (int t = 0; t < kEigsChunk; t++) {
                    const T *bj = B + (int64_t)(j0 + t) * ld;
                    p1[t] = j0 + t < nv ? (double)bj[i] : 0.0;
                    p2[t] = (j0 + t < nv && ok2) ? (double)bj[i2] : 0.0;
                }
#pragma unroll
                for (int t = 0; t < kEigsChunk; t++) {
                    d[t].add(p1[t] * yi);
                    d[t].add(p2[t] * yi2);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < kEigsChunk; t++) {
            warp_reduce(d[t]);
            if (lane == 0 && j0 + t < nv && DM_IN(2 * ((j0 + t) * nsl + sl) + 1, kDpart)) {
                dpart[2 * ((j0 + t) * nsl + sl)] = d[t].hi;
                dpart[2 * ((j0 + t) * nsl + sl) + 1] = d[t].lo;
            }
        }
    }
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();
    for (int j = tid; j < nv; j += bd) {
        CSum t;
        t.zero();
        for (int r = 0; r < CL; r++) {
            const double *rp = dpart;
            if constexpr (CL > 1) rp = cg::this_cluster().map_shared_rank(dpart, r);
            for (int q = 0; q < nsl; q++) t.merge(rp[2 * (j * nsl + q)], rp[2 * (j * nsl + q) + 1]);
        }
        scf[j] = t.value() * ssc[j] * ssc[j];
    }
    __syncthreads();
}

// y_i -= sum_j scf[j] B_j[i] over the job's elements, with eight independent
// partial sums (loads of eight basis vectors in flight), folded in a fixed
// order; returns this thread's share of |y|^2.
template <typename T, int CL>
__device__ __forceinline__ CSum reorth_update(const T *B, uint32_t ld, int nv, T *y, uint32_t dim,
                                              const double *scf) {
    const int rank = cta_rank<CL>();
    const uint32_t i0 = (uint32_t)(rank * blockDim.x + threadIdx.x), st = CL * blockDim.x;
    CSum nrm;
    nrm.zero();
    for (uint32_t i = i0; i < dim; i += st) {
        double acc[8];
#pragma unroll
        for (int t = 0; t < 8; t++) acc[t] = 0.0;
        int j = 0;
        for (; j + 8 <= nv; j += 8) {
#pragma unroll
            for (int t = 0; t < 8; t++)
                acc[t] = fma(scf[j + t], (double)B[(int64_t)(j + t) * ld + i], acc[t]);
        }
        for (int t = 0; j < nv; j++, t++) acc[t] = fma(scf[j], (double)B[(int64_t)j * ld + i], acc[t]);
        const double sub =
            ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
        const T w = (T)((double)y[i] - sub);
        y[i] = w;
        nrm.add((double)w * (double)w);
    }
    return nrm;
}

// y -= X X^T y over the job's elements for the nlock locked FP64 vectors X
// (dim apart, orthonormal), four at a time, twice (classical Gram-Schmidt
// with a repeat); returns this thread's share of |y|^2.
template <typename T, int CL>
__device__ CSum lock_orth(const double *X, int nlock, T *y, uint32_t dim, BatchSmem<T> &sm) {
    const int rank = cta_rank<CL>();
    const uint32_t i0 = (uint32_t)(rank * blockDim.x + threadIdx.x), st = CL * blockDim.x;
    for (int pass = 0; pass < 2; pass++)
        for (int j0 = 0; j0 < nlock; j0 += 4) {
            CSum d[4];
#pragma unroll
            for (int t = 0; t < 4; t++) d[t].zero();
            for (uint32_t i = i0; i < dim; i += st) {
                const double yi = (double)y[i];
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if (j0 + t < nlock) d[t].add(X[(int64_t)(j0 + t) * dim + i] * yi);
            }
            double tot[4];
            job_sum<CL, 4>(d, sm, tot);
            for (uint32_t i = i0; i < dim; i += st) {
                double acc = (double)y[i];
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if (j0 + t < nlock) acc -= tot[t] * X[(int64_t)(j0 + t) * dim + i];
                y[i] = (T)acc;
            }
        }
    CSum nrm;
    nrm.zero();
    for (uint32_t i = i0; i < dim; i += st) nrm.add((double)y[i] * (double)y[i]);
    return nrm;
}

// One sector's eigensolve, run by CL CTAs (a cluster) or by one CTA.
template <typename T, int CL>
__device__ void eigs_job(const BatchTables<T> &tb, BatchSmem<T> &sm, double *dyn, const EigsJob &J,
                         T *basis_pool, double *vec_pool, double *aux_pool, double *evals,
                         int *steps_out, double tol, int ncheck, const BatchCaps &cap,
                         const double *lock_pool) {
    double *sal = dyn, *sbe = sal + (kEigsMaxSteps + 2), *ssc = sbe + (kEigsMaxSteps + 2);
    double *scf = ssc + (kEigsMaxSteps + 2), *dpart = scf + (kEigsMaxSteps + 2);
    double *rwork = dpart + kDpart;
    // orthogonality estimates w_{k-1,.}, w_{k,.}, w_{k+1,.} (rotated)
    double *om0 = rwork + eigs_ritz_doubles(), *om1 = om0 + (kEigsMaxSteps + 2),
           *om2 = om1 + (kEigsMaxSteps + 2);
    const double eps = sizeof(T) == 8 ? 1.1102230246251565e-16 : 5.9604644775390625e-8;
    const double sqeps = sqrt(eps);
    __shared__ double s_omax;
    const int ni = 1 << tb.norb;
    const int tid = threadIdx.x, bd = blockDim.x;
    const int rank = cta_rank<CL>();
    const bool lead = rank == 0 && tid == 0;  // writes the job's outputs
    const uint32_t i0 = (uint32_t)(rank * bd + tid), st = (uint32_t)(CL * bd);
    const Sec<T> s = make_sec(tb, J.nup, J.ndw);
    const bool jflag = tb.jx != 0.0 || tb.jp != 0.0;
    const uint32_t dim = s.dim;
    const uint32_t ld = (dim + 31u) & ~31u;
    if (!DM_IN(J.basis_off + (int64_t)(J.kmax + 1) * ld - 1, cap.work) ||
        !DM_IN(J.vec_off + (int64_t)J.neigen * dim - 1, cap.vec) ||
        !DM_IN(J.aux_off + (rank + 1) * eigs_aux_per_cta(J.neigen, J.kmax) - 1, cap.aux) ||
        !DM_IN(J.slot, cap.slots) || !DM_IN(J.kmax, kEigsMaxSteps + 1) ||
        !DM_IN(J.neigen, kEigsMaxEigen + 1) ||
        (J.nlock > 0 && !DM_IN(J.lock_off + (int64_t)J.nlock * dim - 1, cap.lock)))
        return;
    const double *X = lock_pool + J.lock_off;
    T *B = basis_pool + J.basis_off;
    // private Ritz scratch of this CTA: Y, coefficients, eigenvalues
    const int64_t nk = (int64_t)J.neigen * J.kmax;
    double *Y = aux_pool + J.aux_off + rank * eigs_aux_per_cta(J.neigen, J.kmax);
    double *coef = Y + nk, *evp = coef + nk;
    // seeded start vector (k_random_start, converted to T), scale[0]
    CSum a1[1];
    a1[0].zero();
    for (uint32_t i = i0; i < dim; i += st) {
        const T v = (T)random_start_value(i, eigs_seed(J.nlock));
        B[i] = v;
        a1[0].add((double)v * (double)v);
    }
    if (J.nlock > 0) a1[0] = lock_orth<T, CL>(X, J.nlock, B, dim, sm);
    double tot[1];
    job_sum<CL, 1>(a1, sm, tot);
    if (tid == 0) {
        ssc[0] = tot[0] > 0.0 ? 1.0 / sqrt(tot[0]) : 0.0;
        sbe[0] = 0.0;
    }
    __syncthreads();
    if (tid == 0) {
        om1[0] = 1.0;  // w_{0,0}
        s_omax = 0.0;
    }
    double anorm = 0.0;  // running Gershgorin bound of |T|, every thread
    bool force = false;  // reorthogonalise this vector too (the one after a triggered pass)
    __syncthreads();
    int n = 0;
    bool brk = false;
    for (int k = 0; k < J.kmax; k++) {
        const T *x = B + (int64_t)k * ld;
        const T *xp = B + (int64_t)(k > 0 ? k - 1 : 0) * ld;
        T *y = B + (int64_t)(k + 1) * ld;
        const double sc = ssc[k], cprev = k > 0 ? sbe[k] * ssc[k - 1] : 0.0;
        // u = sc H x - cprev x_prev, alpha_k = sc <x, u>
        a1[0].zero();
        for (uint32_t i = i0; i < dim; i += st) {
            const uint32_t r = i % s.dimup, q = i / s.dimup;
            T h = hx_elem(s, sm, ni, tb.W, tb.P, x, r, q);
            if (jflag) h += hx_jterms(tb, s, x, r, q);
            const T u = (T)(sc * (double)h - cprev * (double)xp[i]);
            y[i] = u;
            a1[0].add((double)x[i] * (double)u);
        }
        job_sum<CL, 1>(a1, sm, tot);
        const double ak = sc * tot[0];
        // w = u - alpha sc x
        const double cf = ak * sc;
        a1[0].zero();
        for (uint32_t i = i0; i < dim; i += st) {
            const T w = (T)((double)y[i] - cf * (double)x[i]);
            y[i] = w;
            a1[0].add((double)w * (double)w);
        }
        job_sum<CL, 1>(a1, sm, tot);
        if (J.nlock > 0) {
            // H keeps the locked vectors' complement invariant only up to
            // their residuals: project the new vector every step
            a1[0] = lock_orth<T, CL>(X, J.nlock, y, dim, sm);
            job_sum<CL, 1>(a1, sm, tot);
        }
        double wn = sqrt(tot[0]), bn = wn;
        anorm = fmax(anorm, fabs(ak) + sbe[k] + wn);
        // orthogonality estimate of the new vector against v_0..v_{k-1}
        // (identical in every CTA of a cluster: same scalars, same order)
        bool reorth = force || (k % kProEvery) == kProEvery - 1 || !(wn > 0.0);
        if (!reorth && k > 0) {
            const double inv = 1.0 / wn, rnd = 2.0 * eps * anorm * inv;
            double mx = 0.0;
            for (int j = tid; j < k; j += bd) {
                double t = sbe[j + 1] * om1[j + 1] + (sal[j] - ak) * om1[j] - sbe[k] * om0[j];
                if (j > 0) t += sbe[j] * om1[j - 1];
                t = t * inv;
                t += copysign(rnd, t);
                om2[j] = t;
                mx = fmax(mx, fabs(t));
            }
            // block maximum (every thread of the CTA)
            for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if ((tid & 31) == 0) dpart[tid >> 5] = mx;
            __syncthreads();
            if (tid == 0) {
                double m = 0.0;
                for (int w = 0; w < (bd >> 5); w++) m = fmax(m, dpart[w]);
                s_omax = m;
            }
            __syncthreads();
            reorth = s_omax > sqeps;
            __syncthreads();
        }
        const bool triggered = reorth && !force && (k % kProEvery) != kProEvery - 1;
        if (reorth) {
            // full reorthogonalisation by classical Gram-Schmidt, repeated
            // once when the first pass removed much of the vector (the DGKS
            // test of ARPACK's dsaitr, |w'| < 0.717 |w|)
            for (int pass = 0; pass < 2; pass++) {
                reorth_dots<T, CL>(B, ld, k + 1, y, dim, dpart, scf, ssc);
                a1[0] = reorth_update<T, CL>(B, ld, k + 1, y, dim, scf);
                job_sum<CL, 1>(a1, sm, tot);
                bn = sqrt(tot[0]);
                if (bn >= kDgks * wn) break;
                wn = bn;
            }
            for (int j = tid; j < k; j += bd) om2[j] = eps;
        }
        force = triggered;  // the vector after a triggered pass is reorthogonalised too
        // w_{k+1,k}: local orthogonality (the alpha step), w_{k+1,k+1} = 1;
        // then rotate the estimates
        if (tid == 0) {
            om2[k] = bn > 0.0 ? 2.0 * eps * anorm / bn : 0.0;
            om2[k + 1] = 1.0;
        }
        __syncthreads();
        {
            double *t = om0;
            om0 = om1;
            om1 = om2;
            om2 = t;
        }
        // b_{k+1} = |w|
        if (tid == 0) {
            sal[k] = ak;
            sbe[k + 1] = bn;
            ssc[k + 1] = bn > 0.0 ? 1.0 / bn : 0.0;
        }
        __syncthreads();
        n = k + 1;
        if (bn < 1e-300 || bn <= kEigsBreakRel * anorm) {
            brk = true;
            break;
        }
        if (n % ncheck == 0 && n < J.kmax) {
            // Ritz test on the lowest Neigen pairs of T_n
            for (int i = tid; i < n; i += bd) rwork[i] = sal[i];
            for (int i = tid; i < n; i += bd) rwork[n + i] = i > 0 ? sbe[i] : 0.0;
            __syncthreads();
            const int m = min(J.neigen, n);
            const bool ok = ritz_multi_dev(rwork, rwork + n, n, J.neigen, tol, sbe[n], evp,
                                           Y, coef, rwork + 2 * n,
                                           (int)eigs_ritz_doubles() - 2 * n);
            if (ok && n >= m && m == J.neigen) break;
            // a probe whose lowest Ritz value stays above the acceptance
            // threshold by ten times its residual estimate found nothing new
            if (J.nlock > 0 && evp[0] > J.top && coef[0] <= 0.1 * (evp[0] - J.top)) break;
        }
    }
    (void)brk;
    // final Ritz pairs and eigenvectors v_j = sum_i Y[j,i] scale_i s_i
    for (int i = tid; i < n; i += bd) rwork[i] = sal[i];
    for (int i = tid; i < n; i += bd) rwork[n + i] = i > 0 ? sbe[i] : 0.0;
    __syncthreads();
    const int mm = min(J.neigen, n);
    ritz_multi_dev(rwork, rwork + n, n, mm, tol, sbe[n], evp, Y, coef, rwork + 2 * n,
                   (int)eigs_ritz_doubles() - 2 * n);
    if (rank == 0)
        for (int j = tid; j < mm; j += bd) evals[(int64_t)J.slot * kEigsMaxEigen + j] = evp[j];
    for (int t = tid; t < mm * n; t += bd) coef[t] = Y[t] * ssc[t % n];
    __syncthreads();
    double *V = vec_pool + J.vec_off;
    for (int j0 = 0; j0 < mm; j0 += kEigsChunk) {
        for (uint32_t i = i0; i < dim; i += st) {
            double acc[kEigsChunk];
#pragma unroll
            for (int t = 0; t < kEigsChunk; t++) acc[t] = 0.0;
            for (int l = 0; l < n; l++) {
                const double b = (double)B[(int64_t)l * ld + i];
#pragma unroll
                for (int t = 0; t < kEigsChunk; t++)
                    if (j0 + t < mm) acc[t] = fma(coef[(int64_t)(j0 + t) * n + l], b, acc[t]);
            }
#pragma unroll
            for (int t = 0; t < kEigsChunk; t++)
                if (j0 + t < mm) V[(int64_t)(j0 + t) * dim + i] = acc[t];
        }
    }
    __syncthreads();
    for (int j = 0; j < mm; j++) {
        double *v = V + (int64_t)j * dim;
        a1[0].zero();
        for (uint32_t i = i0; i < dim; i += st) a1[0].add(v[i] * v[i]);
        job_sum<CL, 1>(a1, sm, tot);
        const double inv = tot[0] > 0.0 ? 1.0 / sqrt(tot[0]) : 0.0;
        for (uint32_t i = i0; i < dim; i += st) v[i] *= inv;
    }
    if (lead) steps_out[J.slot] = n;
    __syncthreads();
}

// Sectors [0, nbig) are shared by the CTAs of a cluster, the rest run one per
// CTA (queue[0] for the clusters, then queue[1] for single CTAs).
template <typename T, int CL>
__global__ void __launch_bounds__(kBatchThreads, 1)
    k_batch_eigs(const BatchTables<T> tb, const EigsJob *jobs, int nbig, int njobs,
                 unsigned *queue, T *basis_pool, double *vec_pool, double *aux_pool,
                 double *evals, int *steps_out, double tol, int ncheck, const BatchCaps cap,
                 const double *lock_pool) {
    __shared__ BatchSmem<T> sm;
    extern __shared__ double dyn[];
    stage_tables(tb, sm);
    if constexpr (CL > 1) {
        for (;;) {
            const int jid = next_job<CL>(queue, sm);
            if (jid >= nbig) break;
            eigs_job<T, CL>(tb, sm, dyn, jobs[jid], basis_pool, vec_pool, aux_pool, evals,
                            steps_out, tol, ncheck, cap, lock_pool);
        }
    }
    for (;;) {
        const int jid = nbig + next_job<1>(queue + 1, sm);
        if (jid >= njobs) break;
        eigs_job<T, 1>(tb, sm, dyn, jobs[jid], basis_pool, vec_pool, aux_pool, evals, steps_out,
                       tol, ncheck, cap, lock_pool);
    }
}

// ------------------------------------------------------------ Green's fn --
// G(z) of every (spin, orbital) from all chains.  k_cf_terms evaluates one
// chain's continued fraction at one frequency per thread; k_cf_sum then adds,
// per (spin, orbital, z), the terms of its chains in list order (the
// reference's accumulation order over states, spins, orbitals, particle and
// hole).  The continued fraction 1/(zeta - a_0 - b_1^2/(zeta - a_1 - ...)) at
// zeta = z + E_i (particle) or E_i - z (hole) is the pole sum of
// add_to_lanczos_gf_normal (build_gf_normal.f90:442-488), evaluated bottom-up
// in FP64.
struct ChainCF {
    int slot, so, isign;
    double weight, ei;
};

__device__ __forceinline__ double2 cdiv2(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        const double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

__global__ void k_cf_terms(const ChainCF *cfs, int ncf, const double *alpha, const double *beta,
                           const int *nsteps, const double *norm2, const double *wm, int lmats,
                           const double *wr, int lreal, double eps, double2 *terms) {
    const int L = lmats + lreal;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ncf * L) return;
    const int c = (int)(t / L), f = (int)(t % L);
    const ChainCF h = cfs[c];
    const int n = nsteps[h.slot];
    double2 term = make_double2(0.0, 0.0);
    if (n > 0) {
        const double2 z = f < lmats ? make_double2(0.0, wm[f]) : make_double2(wr[f - lmats], eps);
        const double *a = alpha + (int64_t)h.slot * kChainStride;
        const double *b = beta + (int64_t)h.slot * kChainStride;
        const double2 zeta =
            h.isign > 0 ? make_double2(z.x + h.ei, z.y) : make_double2(h.ei - z.x, -z.y);
        double2 den = make_double2(zeta.x - a[n - 1], zeta.y);
        for (int k = n - 2; k >= 0; k--) {
            const double2 q = cdiv2(make_double2(b[k + 1] * b[k + 1], 0.0), den);
            den = make_double2(zeta.x - a[k] - q.x, zeta.y - q.y);
        }
        const double2 cf = cdiv2(make_double2(1.0, 0.0), den);
        const double pref = (h.isign > 0 ? 1.0 : -1.0) * h.weight * norm2[h.slot];
        term = make_double2(pref * cf.x, pref * cf.y);
    }
    terms[t] = term;
}

__global__ void k_cf_sum(const ChainCF *cfs, int ncf, int nso, const int *nsteps,
                         const double2 *terms, int lmats, int lreal, double2 *gm, double2 *gr) {
    const int L = lmats + lreal;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nso * L) return;
    const int so = (int)(t / L), f = (int)(t % L);
    double2 g = f < lmats ? gm[(int64_t)so * lmats + f] : gr[(int64_t)so * lreal + f - lmats];
    for (int c = 0; c < ncf; c++) {
        if (cfs[c].so != so || nsteps[cfs[c].slot] <= 0) continue;
        const double2 q = terms[(int64_t)c * L + f];
        g.x += q.x;
        g.y += q.y;
    }
    if (f < lmats) gm[(int64_t)so * lmats + f] = g;
    else gr[(int64_t)so * lreal + f - lmats] = g;
}

// ------------------------------------------------------------------ host --
static size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// One chain's continued fraction on the context's grids, added to host arrays
// gm[lmats], gr[lreal] (complex, gr may be null): the device evaluation every
// solve uses, for a chain given by its coefficients.
void gf_add_chain(dmfted_ctx *c, int nlanc, const double *alanc, const double *blanc,
                  double weight, double norm2, double ei, int isign, double *gm, double *gr) {
    DM_REQUIRE(nlanc >= 1 && nlanc <= kChainStride - 1, DMFTED_ERR_ARG,
               "add_to_lanczos_gf: nlanc out of range");
    const dmfted_params &p = c->p;
    const int L = p.lmats + p.lreal;
    std::vector<double> buf(2 * (size_t)kChainStride + 2, 0.0);
    std::copy(alanc, alanc + nlanc, buf.begin());
    for (int k = 1; k < nlanc; k++) buf[kChainStride + k] = blanc[k];
    buf[2 * kChainStride] = norm2;
    ChainCF cf{0, 0, isign > 0 ? 1 : -1, weight, ei};
    c->eig_aux.alloc(buf.size() + 2 * (size_t)L + 8);
    double *d = c->eig_aux.p, *d_terms = d + buf.size() + 4;
    c->bjobs.alloc(sizeof(ChainCF) + 16);
    c->bint.alloc(4);
    const int n = nlanc;
    DM_CUDA(cudaMemcpyAsync(d, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    DM_CUDA(cudaMemcpyAsync(c->bjobs.p, &cf, sizeof(cf), cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(c->bint.p, &n, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    k_cf_terms<<<div_up(L, 128), 128, 0, c->stream>>>(
        reinterpret_cast<const ChainCF *>(c->bjobs.p), 1, d, d + kChainStride, c->bint.p,
        d + 2 * kChainStride, c->d_wm.p, p.lmats, c->d_wr.p, p.lreal, p.eps,
        reinterpret_cast<double2 *>(d_terms));
    DM_CHECK_LAUNCH();
    c->launches++;
    std::vector<double> t(2 * (size_t)L);
    DM_CUDA(cudaMemcpyAsync(t.data(), d_terms, t.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    for (int f = 0; f < p.lmats; f++) {
        gm[2 * f] += t[2 * f];
        gm[2 * f + 1] += t[2 * f + 1];
    }
    if (gr)
        for (int f = 0; f < p.lreal; f++) {
            gr[2 * f] += t[2 * (p.lmats + f)];
            gr[2 * f + 1] += t[2 * (p.lmats + f) + 1];
        }
}

// Persistent launch: as many CTAs (CL == 1) or clusters as can be resident,
// at most one per job.
template <typename... KArgs, typename... Args>
static void launch_persistent(dmfted_ctx *c, void (*kern)(KArgs...), int CL, int njobs,
                              size_t smem, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = CL > 1 ? 1 : 0;
    if (CL > 8) {
        // 16 CTAs per cluster is beyond the portable size: opt in per kernel
        DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    int units = std::max(1, num_sms(c) / CL);
    if (CL > 1) {
        cfg.gridDim = dim3(units * CL);
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) == cudaSuccess && ncl > 0)
            units = ncl;
        else
            (void)cudaGetLastError();
    }
    units = std::min(units, njobs);
    cfg.gridDim = dim3(units * CL);
    DM_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
    c->launches++;
}

// CTAs per eigensolve job: from the largest sector (at least
// batch_cluster_min states per CTA, to amortise the cluster barriers; 16, the
// non-portable cluster size, from 32 per CTA: on the Ns=10 workload, whose
// largest sector holds 63,504 states, 16 took 35.9 ms of eigensolves against
// 38.6 ms for 8), or DMFTED_BATCH_CLUSTER_EIGS.  Only sectors that give every
// CTA that many states are shared; smaller ones run one per CTA.
static int eigs_cluster(const dmfted_ctx *c, int64_t dmax) {
    const int64_t per = c->batch_cluster_min;
    if (const char *e = getenv("DMFTED_BATCH_CLUSTER_EIGS")) {
        const int v = atoi(e);
        if (v == 1 || v == 2 || v == 4 || v == 8 || v == 16) return v;
    }
    return dmax >= 32 * per ? 16 : dmax >= 8 * per ? 8 : dmax >= 4 * per ? 4 : dmax >= 2 * per ? 2 : 1;
}

// CTAs per chain: two once the largest chain holds 16 x batch_cluster_min
// states (the long chains set the phase's time: 200 chains of the Ns=10
// workload took 35.0 ms with pairs against 38.9 ms one per CTA), more only
// while the chains leave SMs idle; or DMFTED_BATCH_CLUSTER_GF.
static int chain_cluster(dmfted_ctx *c, int njobs, int64_t dmax) {
    const int64_t per = c->batch_cluster_min;
    if (const char *e = getenv("DMFTED_BATCH_CLUSTER_GF")) {
        const int v = atoi(e);
        if (v == 1 || v == 2 || v == 4 || v == 8 || v == 16) return v;
    }
    int cl = dmax >= 16 * per ? 2 : 1;
    while (cl < 8 && (int64_t)njobs * cl * 2 <= 2 * (int64_t)num_sms(c) &&
           dmax / (cl * 2) >= 2 * per)
        cl *= 2;
    return cl;
}

// Autotuner of the batched phases.  The cluster size of a phase (CTAs per
// shared job) is picked per job-shape key -- precision, Fock space, hop-table
// width (the nonzeros per row), largest job dimension and the job count's
// power-of-two bucket (the state list grows over the first DMFT iterations)
// -- by measurement.  The first phase with a new key runs once at the largest
// candidate size untimed (pools reach their final size, caches warm), then
// measures the candidates -- the fixed rule's size and its neighbours, half
// and double, within 1..16 and giving every CTA of a shared job at least
// batch_cluster_min states -- in two interleaved rounds, timed with CUDA
// events on the context's stream; each candidate's faster run counts (the
// rounds cancel clock drift).  The rule's size is kept unless a candidate is
// more than 3 % faster; the choice then serves every later phase with that
// key.  The phase is left with the results of a run at the chosen size
// (re-run if another size ran last).  Enabled by DMFTED_AUTOTUNE=1; an
// environment override of the size keeps the fixed rule.
template <typename Run>
static int tuned_cluster(dmfted_ctx *c, const char *kind, const char *override_env, int rule,
                         int64_t njobs, int64_t dmax, int precision, Run run) {
    if (!c->autotune || getenv(override_env)) {
        run(rule);
        return rule;
    }
    int bucket = 0;
    while ((int64_t(1) << bucket) <= njobs) bucket++;
    char key[256];
    snprintf(key, sizeof(key), "%s prec=%d ns=%d norb=%d W=%d jobs<2^%d dmax=%lld", kind,
             precision, c->ns, c->norb, c->W, bucket, (long long)dmax);
    auto it = c->tune_choice.find(key);
    if (it != c->tune_choice.end()) {
        run(it->second);
        return it->second;
    }
    std::vector<int> cand;
    for (int cl : {rule / 2, rule, rule * 2})
        if (cl == rule || (cl >= 1 && cl <= 16 && (cl == 1 || dmax >= c->batch_cluster_min * cl)))
            cand.push_back(cl);
    run(cand.back());  // untimed: pools at their largest size, caches warm
    cudaEvent_t e0, e1;
    DM_CUDA(cudaEventCreate(&e0));
    DM_CUDA(cudaEventCreate(&e1));
    std::vector<float> t(cand.size(), 1e30f);
    for (int round = 0; round < 2; round++)
        for (size_t i = 0; i < cand.size(); i++) {
            DM_CUDA(cudaEventRecord(e0, c->stream));
            run(cand[i]);
            DM_CUDA(cudaEventRecord(e1, c->stream));
            DM_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            DM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            t[i] = std::min(t[i], ms);
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::string log = std::string(key) + " ->";
    for (size_t i = 0; i < cand.size(); i++) {
        char b[64];
        snprintf(b, sizeof(b), " CL%d=%.3fms", cand[i], t[i]);
        log += b;
    }
    int best = rule;
    float tbest = 0.97f * t[std::find(cand.begin(), cand.end(), rule) - cand.begin()];
    for (size_t i = 0; i < cand.size(); i++)
        if (t[i] < tbest) {
            tbest = t[i];
            best = cand[i];
        }
    if (best != cand.back()) run(best);
    char b[64];
    snprintf(b, sizeof(b), " chosen CL%d (rule CL%d)", best, rule);
    c->tune_log.push_back(log + b);
    c->tune_choice[key] = best;
    return best;
}

// One launch over the jobs [j0, j1) of the queue; the job table holds the
// whole queue, each wave has its own counter.
template <typename T, int CL>
static void run_batch_eigs(dmfted_ctx *c, int j0, int nbig, int j1, int wave, double tol) {
    static bool attr[64] = {false};
    if (!attr[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(k_batch_eigs<T, CL>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)eigs_smem()));
        attr[c->device & 63] = true;
    }
    launch_persistent(c, k_batch_eigs<T, CL>, CL, nbig + div_up(j1 - j0 - nbig, CL), eigs_smem(),
                      batch_tables<T>(c), reinterpret_cast<const EigsJob *>(c->bjobs.p) + j0, nbig,
                      j1 - j0, reinterpret_cast<unsigned *>(c->bint.p) + 2 * wave,
                      reinterpret_cast<T *>(c->bwork.p), c->bvec.p, c->baux.p, c->bscal.p,
                      c->bint.p + 2 * kMaxWaves, tol, std::max(1, c->p.lanc_ncheck),
                      BatchCaps{(int64_t)(c->bwork.n / sizeof(T)), (int64_t)c->bvec.n,
                                (int64_t)c->baux.n, 0, (int64_t)(c->bscal.n / kEigsMaxEigen),
                                (int64_t)c->lockpool.n},
                      (const double *)c->lockpool.p);
}

template <typename T>
static void run_batch_eigs_cl(dmfted_ctx *c, int CL, int j0, int nbig, int j1, int wave,
                              double tol) {
    switch (CL) {
        case 16: run_batch_eigs<T, 16>(c, j0, nbig, j1, wave, tol); break;
        case 8: run_batch_eigs<T, 8>(c, j0, nbig, j1, wave, tol); break;
        case 4: run_batch_eigs<T, 4>(c, j0, nbig, j1, wave, tol); break;
        case 2: run_batch_eigs<T, 2>(c, j0, nbig, j1, wave, tol); break;
        default: run_batch_eigs<T, 1>(c, j0, 0, j1, wave, tol); break;
    }
}


static void batch_eigs_cl(dmfted_ctx *c, const std::vector<int> &list,
                          const std::vector<int> &want, int precision, std::vector<BatchEig> &res,
                          int CL, const std::vector<LockSpec> *locks) {
    const dmfted_params &p = c->p;
    res.assign(list.size(), BatchEig());
    const bool fp64 = precision == DMFTED_FP64;
    const size_t es = fp64 ? sizeof(double) : sizeof(float);
    std::vector<EigsJob> jobs;
    std::vector<int> where;  // list index of each job
    std::vector<size_t> bsize;  // Krylov basis elements of each job
    size_t vec = 0, aux = 0;
    for (size_t i = 0; i < list.size(); i++) {
        const SectorView s = sector_view(c, list[i]);
        const int neigen = (int)std::min<int64_t>(s.dim, want[i]);
        if (neigen <= 0) continue;
        const int kmax = (int)std::min<int64_t>(std::min(p.lanc_niter, kLzMax - 2), s.dim);
        if (c->batch_max_dim <= 0 || s.dim > c->batch_max_dim || kmax > kEigsMaxSteps ||
            neigen > kEigsMaxEigen)
            continue;
        EigsJob J;
        J.nup = s.nup;
        J.ndw = s.ndw;
        J.neigen = neigen;
        J.kmax = kmax;
        J.slot = (int)jobs.size();
        J.basis_off = 0;
        J.vec_off = (int64_t)vec;
        J.aux_off = (int64_t)aux;
        J.lock_off = locks ? (*locks)[i].off : 0;
        J.nlock = locks ? (*locks)[i].n : 0;
        J.top = locks ? (*locks)[i].top : INFINITY;
        DM_REQUIRE(J.nlock == 0 || fp64, DMFTED_ERR_ARG, "locked eigensolve needs FP64");
        bsize.push_back((size_t)(kmax + 1) * round_up((size_t)s.dim, 32));
        vec += (size_t)neigen * s.dim;
        const bool big = CL > 1 && s.dim >= c->batch_cluster_min * CL;
        aux += (size_t)(big ? CL : 1) * eigs_aux_per_cta(neigen, kmax);
        jobs.push_back(J);
        where.push_back((int)i);
    }
    if (jobs.empty()) return;
    const int nj = (int)jobs.size();
    // queue order: longest first (full reorthogonalisation costs ~ kmax^2 dim)
    std::vector<int> order(nj);
    for (int j = 0; j < nj; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const EigsJob &x = jobs[a], &y = jobs[b];
        const double ca = (double)c->binom[x.nup] * c->binom[x.ndw] * x.kmax * x.kmax;
        const double cb = (double)c->binom[y.nup] * c->binom[y.ndw] * y.kmax * y.kmax;
        return ca > cb;
    });
    // waves of jobs whose worst-case bases fit a third of the free memory
    size_t freeb = 0, totalb = 0;
    DM_CUDA(cudaMemGetInfo(&freeb, &totalb));
    const size_t bytes = c->batch_budget > 0 ? (size_t)c->batch_budget : (freeb + c->bwork.n) / 3;
    const size_t budget = std::max<size_t>(bytes / es, 1);
    std::vector<EigsJob> q;
    std::vector<int> wave_end;
    size_t used = 0, peak = 0;
    for (int j : order) {
        if (used > 0 && used + bsize[j] > budget) {
            wave_end.push_back((int)q.size());
            used = 0;
        }
        EigsJob J = jobs[j];
        J.basis_off = (int64_t)used;
        used += bsize[j];
        peak = std::max(peak, used);
        q.push_back(J);
    }
    wave_end.push_back((int)q.size());
    DM_REQUIRE((int)wave_end.size() <= kMaxWaves, DMFTED_ERR_NOMEM,
               "batched eigensolve: Krylov bases do not fit the device memory");
    c->bwork.alloc(peak * es);
    c->bvec.alloc(vec);
    c->baux.alloc(aux);
    c->bjobs.alloc(nj * sizeof(EigsJob));
    c->bscal.alloc((size_t)nj * kEigsMaxEigen);
    c->bint.alloc(2 * kMaxWaves + nj);
    DM_CUDA(cudaMemcpyAsync(c->bjobs.p, q.data(), nj * sizeof(EigsJob), cudaMemcpyHostToDevice,
                            c->stream));
    DM_CUDA(cudaMemsetAsync(c->bint.p, 0, 2 * kMaxWaves * sizeof(int), c->stream));
    const double tol = fp64 ? p.lanc_tolerance : std::max(p.lanc_tolerance, c->mixed_tol32);
    for (size_t w = 0; w < wave_end.size(); w++) {
        const int j0 = w == 0 ? 0 : wave_end[w - 1], j1 = wave_end[w];
        int nbig = 0;  // the queue is sorted by size: big sectors lead each wave
        while (CL > 1 && j0 + nbig < j1 &&
               c->binom[q[j0 + nbig].nup] * c->binom[q[j0 + nbig].ndw] >= c->batch_cluster_min * CL)
            nbig++;
        if (fp64) run_batch_eigs_cl<double>(c, CL, j0, nbig, j1, (int)w, tol);
        else run_batch_eigs_cl<float>(c, CL, j0, nbig, j1, (int)w, tol);
    }
    std::vector<double> ev((size_t)nj * kEigsMaxEigen);
    std::vector<int> steps(nj);
    DM_CUDA(cudaMemcpyAsync(ev.data(), c->bscal.p, ev.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaMemcpyAsync(steps.data(), c->bint.p + 2 * kMaxWaves, nj * sizeof(int),
                            cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < nj; j++) {
        BatchEig &r = res[where[j]];
        r.steps = steps[j];
        r.m = std::min(jobs[j].neigen, steps[j]);
        r.evals.assign(ev.begin() + (size_t)j * kEigsMaxEigen,
                       ev.begin() + (size_t)j * kEigsMaxEigen + r.m);
        r.vecs = c->bvec.p + jobs[j].vec_off;
    }
}

void batch_eigs(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                int precision, std::vector<BatchEig> &res, const std::vector<LockSpec> *locks) {
    int64_t dmax = 0, nj = 0;
    for (size_t i = 0; i < list.size(); i++)
        if (want[i] > 0 && sector_view(c, list[i]).dim <= c->batch_max_dim) {
            dmax = std::max(dmax, sector_view(c, list[i]).dim);
            nj++;
        }
    if (nj == 0) {
        res.assign(list.size(), BatchEig());
        return;
    }
    const bool probe = locks != nullptr;
    tuned_cluster(c, probe ? "eigs-probe" : "eigs", "DMFTED_BATCH_CLUSTER_EIGS",
                  eigs_cluster(c, dmax), nj, dmax, precision,
                  [&](int cl) { batch_eigs_cl(c, list, want, precision, res, cl, locks); });
}

template <typename T, int CL>
static void run_batch_chains(dmfted_ctx *c, int nbig, int nj, double *alpha, double *beta,
                             int *nsteps, double *norm2, int64_t nslots) {
    launch_persistent(c, k_batch_chains<T, CL>, CL, nbig + div_up(nj - nbig, CL), 0,
                      batch_tables<T>(c), reinterpret_cast<const ChainJob *>(c->bjobs.p), nbig, nj,
                      reinterpret_cast<unsigned *>(c->bint.p), (const double *)c->states64.p,
                      reinterpret_cast<T *>(c->bwork.p), alpha, beta, nsteps, norm2,
                      c->p.lanc_gf_threshold,
                      BatchCaps{(int64_t)(c->bwork.n / sizeof(T)), 0, 0, (int64_t)c->states64.n,
                                nslots});
}

template <typename T>
static void run_batch_chains_cl(dmfted_ctx *c, int CL, const std::vector<ChainJob> &jobs,
                                double *alpha, double *beta, int *nsteps, double *norm2,
                                int64_t nslots) {
    const int nj = (int)jobs.size();
    DM_CUDA(cudaMemcpyAsync(c->bjobs.p, jobs.data(), nj * sizeof(ChainJob), cudaMemcpyHostToDevice,
                            c->stream));
    DM_CUDA(cudaMemsetAsync(c->bint.p, 0, 2 * sizeof(int), c->stream));
    int nbig = 0;  // sorted by size: the chains a cluster shares come first
    while (CL > 1 && nbig < nj &&
           c->binom[jobs[nbig].tnup] * c->binom[jobs[nbig].tndw] >= c->batch_cluster_min * CL)
        nbig++;
    switch (CL) {
        case 16: run_batch_chains<T, 16>(c, nbig, nj, alpha, beta, nsteps, norm2, nslots); break;
        case 8: run_batch_chains<T, 8>(c, nbig, nj, alpha, beta, nsteps, norm2, nslots); break;
        case 4: run_batch_chains<T, 4>(c, nbig, nj, alpha, beta, nsteps, norm2, nslots); break;
        case 2: run_batch_chains<T, 2>(c, nbig, nj, alpha, beta, nsteps, norm2, nslots); break;
        default: run_batch_chains<T, 1>(c, 0, nj, alpha, beta, nsteps, norm2, nslots); break;
    }
}

// The context's per-lane resources -- stream, reduction scratch, chain
// buffers -- exchanged with the second set while the guard lives, so that
// everything queued meanwhile (launches, copies, timing events) goes to the
// second stream with its own scratch.
struct SecondLane {
    dmfted_ctx *c;
    explicit SecondLane(dmfted_ctx *cc) : c(cc) { swap(); }
    ~SecondLane() { swap(); }
    SecondLane(const SecondLane &) = delete;
    SecondLane &operator=(const SecondLane &) = delete;
    void swap() {
        std::swap(c->stream, c->stream2);
        c->red_partials.swap(c->red_partials2);
        c->red_counter.swap(c->red_counter2);
        c->chainbuf.swap(c->chainbuf2);
        c->jscratch.swap(c->jscratch2);
    }
};

void batch_chains_gf(dmfted_ctx *c, const std::vector<ChainRec> &recs, int precision) {
    const dmfted_params &p = c->p;
    const int L = p.lmats + p.lreal;
    const int nrec = (int)recs.size();
    if (nrec == 0) return;
    // Batched chains (one CTA or cluster per chain) are FP64 in both forms: an
    // FP32 chain perturbs G(iwn) at the 1e-6 level and, being latency-bound
    // rather than bandwidth-bound, saves under 10 % of the chain time.
    const bool fp64 = precision == DMFTED_FP64 || !c->batch_chains_fp32;
    const size_t es = fp64 ? sizeof(double) : sizeof(float);
    c->bscal.alloc((size_t)2 * nrec * kChainStride + nrec);
    double *alpha = c->bscal.p, *beta = alpha + (size_t)nrec * kChainStride;
    double *norm2 = beta + (size_t)nrec * kChainStride;
    c->bint.alloc(2 + nrec);
    int *nsteps = c->bint.p + 2;
    std::vector<ChainJob> jobs;
    std::vector<char> batched(nrec, 0);
    size_t work = 0;
    for (int i = 0; i < nrec; i++) {
        const ChainRec &r = recs[i];
        const SectorView sj = sector_view(c, r.jsector);
        if (c->batch_max_dim <= 0 || sj.dim > c->batch_max_dim || r.nlanc > kLzMax - 2) continue;
        ChainJob J;
        J.tnup = sj.nup;
        J.tndw = sj.ndw;
        J.snup = c->getnup[r.isector - 1];
        J.ispin = r.ispin;
        J.iorb = r.iorb;
        J.particle = r.particle;
        J.kmax = r.nlanc;
        J.slot = i;
        J.psi_off = r.psi_off;
        J.work_off = (int64_t)work;
        work += 2 * round_up((size_t)sj.dim, 32);
        jobs.push_back(J);
        batched[i] = 1;
    }
    const size_t cf_off = round_up(std::max<size_t>(jobs.size(), 1) * sizeof(ChainJob), 256);
    c->bjobs.alloc(cf_off + nrec * sizeof(ChainCF));
    if (!jobs.empty()) {
        c->bwork.alloc(work * es);
        std::stable_sort(jobs.begin(), jobs.end(), [&](const ChainJob &a, const ChainJob &b) {
            const double ca = (double)c->binom[a.tnup] * c->binom[a.tndw] * a.kmax;
            const double cb = (double)c->binom[b.tnup] * c->binom[b.tndw] * b.kmax;
            return ca > cb;
        });
        int64_t dmax = 0;
        for (const ChainJob &J : jobs)
            dmax = std::max<int64_t>(dmax, c->binom[J.tnup] * c->binom[J.tndw]);
        tuned_cluster(c, "chains", "DMFTED_BATCH_CLUSTER_GF",
                      chain_cluster(c, (int)jobs.size(), dmax), (int64_t)jobs.size(), dmax,
                      fp64 ? DMFTED_FP64 : DMFTED_MIXED, [&](int cl) {
                          if (fp64) run_batch_chains_cl<double>(c, cl, jobs, alpha, beta, nsteps, norm2, nrec);
                          else run_batch_chains_cl<float>(c, cl, jobs, alpha, beta, nsteps, norm2, nrec);
                      });
    }
    // chains too large for one CTA: the grid-wide recurrence, two at a time
    // (the second on the second lane) so that each chain's kernels fill the
    // SMs the other leaves idle in its last wave, and its bandwidth-bound
    // updates overlap the other's H*v
    std::vector<int> grid_recs;
    for (int i = 0; i < nrec; i++)
        if (!batched[i]) grid_recs.push_back(i);
    auto start_vector = [&](int i, DBuf<double> &v0) {
        const ChainRec &r = recs[i];
        const SectorView si = sector_view(c, r.isector), sj = chain_view(c, r.jsector);
        v0.alloc(sj.dim);
        gf_apply_op(c, si, sj, r.iorb, r.ispin, r.particle != 0, c->states64.p + r.psi_off, v0.p,
                    norm2 + i);
    };
    auto run_chain = [&](int i, const double *v0, int slot) {
        const ChainRec &r = recs[i];
        LanczosScalars lz = lz_slot(c, slot, r.nlanc);
        lanczos_chain(c, chain_view(c, r.jsector), v0, precision, lz);
        DM_CUDA(cudaMemcpyAsync(alpha + (size_t)i * kChainStride, lz.alpha,
                                kChainStride * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        DM_CUDA(cudaMemcpyAsync(beta + (size_t)i * kChainStride, lz.beta,
                                kChainStride * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        DM_CUDA(cudaMemcpyAsync(nsteps + i, lz.status + 1, sizeof(int), cudaMemcpyDeviceToDevice,
                                c->stream));
    };
    const bool two = c->chain_lanes >= 2 && c->stream2;
    for (size_t g = 0; g < grid_recs.size(); g += two ? 2 : 1) {
        const int ia = grid_recs[g];
        const int ib = two && g + 1 < grid_recs.size() ? grid_recs[g + 1] : -1;
        start_vector(ia, c->s64b);
        if (ib >= 0) {
            start_vector(ib, c->s64d);
            DM_CUDA(cudaEventRecord(c->ev_fork, c->stream));
            DM_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
        }
        run_chain(ia, c->s64b.p, 1);
        if (ib >= 0) {
            {
                SecondLane lane(c);
                run_chain(ib, c->s64d.p, 2);  // slot 2: free during a solve
            }
            DM_CUDA(cudaEventRecord(c->ev_join, c->stream2));
            DM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        }
    }
    if (L <= 0) return;
    std::vector<ChainCF> cf(nrec);
    for (int i = 0; i < nrec; i++) {
        cf[i].slot = i;
        cf[i].so = recs[i].ispin * c->norb + recs[i].iorb;
        cf[i].isign = recs[i].particle ? 1 : -1;
        cf[i].weight = recs[i].weight;
        cf[i].ei = recs[i].e;
    }
    ChainCF *d_cf = reinterpret_cast<ChainCF *>(c->bjobs.p + cf_off);
    DM_CUDA(cudaMemcpyAsync(d_cf, cf.data(), nrec * sizeof(ChainCF), cudaMemcpyHostToDevice,
                            c->stream));
    const int nso = c->nspin * c->norb;
    c->bcf.alloc((size_t)2 * nrec * L);
    double2 *terms = reinterpret_cast<double2 *>(c->bcf.p);
    k_cf_terms<<<div_up((int64_t)nrec * L, 128), 128, 0, c->stream>>>(
        d_cf, nrec, alpha, beta, nsteps, norm2, c->d_wm.p, p.lmats, c->d_wr.p, p.lreal, p.eps,
        terms);
    k_cf_sum<<<div_up((int64_t)nso * L, 128), 128, 0, c->stream>>>(
        d_cf, nrec, nso, nsteps, terms, p.lmats, p.lreal, (double2 *)c->gm.p, (double2 *)c->gr.p);
    DM_CHECK_LAUNCH();
    c->launches += 2;
}

}  // namespace dmfted
