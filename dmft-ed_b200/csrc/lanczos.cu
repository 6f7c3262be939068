// Device-resident Lanczos: ground state (stands in for SciFortran's sp_eigh
// with Neigen=1, ED_DIAG.f90:169-183) and the three-term tridiagonalisation of
// the Green's-function chains (sp_lanc_tridiag, build_gf_normal.f90:118-127).
//
// The recurrence is the plain three-term Lanczos of
// .repo/PLAIN_LANCZOS.f90:87-118:
//     u = H v_k - b_k v_{k-1};  a_k = <v_k, u>;  w = u - a_k v_k;
//     b_{k+1} = |w|;  v_{k+1} = w / b_{k+1}
// Vectors are stored unnormalised (s_{k+1} = w) with their scales
// sc_{k+1} = 1/b_{k+1} kept on the device, so normalisation never costs a pass
// over memory: every reader multiplies by the scalar.  One step is two
// kernels: the H*v with the -b_k v_{k-1} term and the a_k dot product fused
// (k_hxv<LZ>), then the a_k axpy fused with the |w| reduction (k_lz_update).
// All scalars stay on the device; steps after convergence or breakdown are
// no-ops (status flag), so chains are queued without host round trips.
//
// The ground-state iteration stores the whole Krylov basis (B200 HBM holds
// hundreds of sector vectors) and forms the Ritz vector as one pass over it.
// Every ncheck steps a single-CTA kernel computes the lowest Ritz value by
// Sturm-sequence multisection in FP64 and compares it with the previous
// check (the energy-change test of .repo/PLAIN_LANCZOS.f90:344-351).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hxv.cuh"
#include "tridiag.cuh"

namespace dmfted {

enum { ST_DONE = 0, ST_STEPS = 1, ST_CONV = 2, ST_RITZ_VALID = 3, ST_BREAK = 4 };

// w = u - a_k sc_k s_k (in place in u), then b_{k+1} = |w|.  VW elements
// per thread per pass (16-byte accesses when n is a multiple of VW); the
// vector form issues the loads of kUpdUnroll passes before using them, so
// that each SM keeps enough bytes in flight to cover the HBM latency.
constexpr int kUpdUnroll = 4;

template <typename T, int VW>
__device__ __forceinline__ void lz_update_vec(uint4 &qu, const uint4 &qs, double coef, CSum &s) {
    T a[VW], b[VW];
    memcpy(a, &qu, 16);
    memcpy(b, &qs, 16);
#pragma unroll
    for (int q = 0; q < VW; q++) {
        a[q] = (T)((double)a[q] - coef * (double)b[q]);
        s.add((double)a[q] * (double)a[q]);
    }
    memcpy(&qu, a, 16);
}

template <typename T, int VW>
__global__ void __launch_bounds__(kRedThreads) k_lz_update(T *u, const T *scur, int64_t n,
                                                           LanczosScalars lz, int k, double thr,
                                                           double *partials, unsigned *counter) {
    if (lz.status[ST_DONE]) return;
    const double coef = lz.alpha[k] * lz.scale[k];
    CSum s;
    s.zero();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * VW;
    int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * VW;
    if constexpr (VW > 1) {
        for (; i + (kUpdUnroll - 1) * stride < n; i += kUpdUnroll * stride) {
            uint4 qu[kUpdUnroll], qs[kUpdUnroll];
#pragma unroll
            for (int q = 0; q < kUpdUnroll; q++) {
                qu[q] = *reinterpret_cast<const uint4 *>(u + i + q * stride);
                qs[q] = *reinterpret_cast<const uint4 *>(scur + i + q * stride);
            }
#pragma unroll
            for (int q = 0; q < kUpdUnroll; q++) {
                lz_update_vec<T, VW>(qu[q], qs[q], coef, s);
                *reinterpret_cast<uint4 *>(u + i + q * stride) = qu[q];
            }
        }
    }
    for (; i < n; i += stride) {
        if constexpr (VW == 1) {
            const T wt = (T)((double)u[i] - coef * (double)scur[i]);
            u[i] = wt;
            s.add((double)wt * (double)wt);
        } else {
            uint4 qu = *reinterpret_cast<const uint4 *>(u + i);
            const uint4 qs = *reinterpret_cast<const uint4 *>(scur + i);
            lz_update_vec<T, VW>(qu, qs, coef, s);
            *reinterpret_cast<uint4 *>(u + i) = qu;
        }
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot)) {
        if (threadIdx.x == 0) {
            const double b = sqrt(tot[0]);
            lz.beta[k + 1] = b;
            lz.scale[k + 1] = b > 0.0 ? 1.0 / b : 0.0;
            lz.status[ST_STEPS] = k + 1;
            if (b < thr) {
                lz.status[ST_DONE] = 1;
                lz.status[ST_BREAK] = 1;
            }
            if (k + 1 >= lz.kmax) lz.status[ST_DONE] = 1;
        }
    }
}

template <typename T>
static void launch_lz_update(dmfted_ctx *c, T *u, const T *scur, int64_t n, const LanczosScalars &lz,
                             int k, double thr);

// Start of a recurrence: scale[0] = 1/|s_0|, beta[0] = 0, status cleared.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_lz_init(const T *s0, int64_t n, LanczosScalars lz,
                                                         double *partials, unsigned *counter) {
    CSum s;
    s.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)s0[i];
        s.add(v * v);
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot)) {
        if (threadIdx.x == 0) {
            lz.scale[0] = tot[0] > 0.0 ? 1.0 / sqrt(tot[0]) : 0.0;
            lz.beta[0] = 0.0;
            for (int i = 0; i < 8; i++) lz.status[i] = 0;
            lz.ritz[0] = lz.ritz[1] = 0.0;
        }
    }
}


// Every ncheck steps: lowest Ritz value theta of T_n and the ARPACK stopping
// test on its Ritz estimate, b_n |y_n| <= tol * max(eps^(2/3), |theta|)
// (y = eigenvector of T_n, b_n = norm of the last residual).  Breakdown
// (invariant subspace) counts as converged.
__global__ void k_ritz_check(LanczosScalars lz, double tol) {
    extern __shared__ double rs[];
    const int n = lz.status[ST_STEPS];
    if (n <= 0) return;
    if (!DM_IN(n, kLzMax)) return;
    double *sa = rs, *sb = rs + n, *yv = rs + 2 * n, *ws = rs + 3 * n;
    unsigned char *sw = reinterpret_cast<unsigned char *>(rs + 8 * n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sa[i] = lz.alpha[i];
        sb[i] = i > 0 ? lz.beta[i] : 0.0;
    }
    __syncthreads();
    const double e = tridiag_eig(sa, sb, n, 0);
    if (threadIdx.x == 0) {
        tridiag_evec(sa, sb, n, e, yv, ws, sw);
        const double est = fabs(lz.beta[n]) * fabs(yv[n - 1]);
        const double eps23 = 3.666852862501036e-11;
        if (lz.status[ST_BREAK] || est <= tol * fmax(eps23, fabs(e))) {
            lz.status[ST_CONV] = 1;
            lz.status[ST_DONE] = 1;
        }
        lz.ritz[1] = est;
        lz.ritz[0] = e;
        lz.status[ST_RITZ_VALID] = 1;
    }
}

// Ritz vector coefficients coef[i] = y_i * scale_i for eigenvalue lam, so
// that the Ritz vector is sum_i coef_i s_i.
__global__ void k_ritz_vector(LanczosScalars lz, int n, double lam, double *coef) {
    extern __shared__ double rs[];
    double *sa = rs, *sb = rs + n, *yv = rs + 2 * n, *ws = rs + 3 * n;
    unsigned char *sw = reinterpret_cast<unsigned char *>(rs + 8 * n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sa[i] = lz.alpha[i];
        sb[i] = i > 0 ? lz.beta[i] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    tridiag_evec(sa, sb, n, lam, yv, ws, sw);
    for (int i = 0; i < n; i++) coef[i] = yv[i] * lz.scale[i];
}

// psi = sum_{i<n} coef_i * s_i over the stored basis (slot stride ld).  If
// v0 (float64) is given it replaces slot 0 (the refinement basis keeps its
// first vector in FP64).
template <typename T>
__global__ void k_basis_combine(const T *basis, int64_t ld, int n, const double *coef,
                                const double *v0, double *psi, int64_t dim) {
    __shared__ double sc[kLzMax + 8];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sc[i] = coef[i];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < dim;
         i += (int64_t)gridDim.x * blockDim.x) {
        double acc = v0 ? sc[0] * v0[i] : sc[0] * (double)basis[i];
        for (int k = 1; k < n; k++)
            if (DM_IN(k, kLzMax)) acc += sc[k] * (double)basis[k * ld + i];
        psi[i] = acc;
    }
}

// First step of the refinement recurrence, in FP64: w = u - a_0 sc_0 v0 with
// u = H v0 (FP64), stored rounded to FP32 in the next slot; b_1 = |w| of the
// stored values.
__global__ void __launch_bounds__(kRedThreads) k_lz_update_first(const double *u, const double *v0,
                                                                 float *out, int64_t n,
                                                                 LanczosScalars lz,
                                                                 double *partials,
                                                                 unsigned *counter) {
    if (lz.status[ST_DONE]) return;
    const double coef = lz.alpha[0] * lz.scale[0];
    CSum s;
    s.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float wt = (float)(u[i] - coef * v0[i]);
        out[i] = wt;
        s.add((double)wt * (double)wt);
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot)) {
        if (threadIdx.x == 0) {
            const double b = sqrt(tot[0]);
            lz.beta[1] = b;
            lz.scale[1] = b > 0.0 ? 1.0 / b : 0.0;
            lz.status[ST_STEPS] = 1;
            if (b < 1e-300) {
                lz.status[ST_DONE] = 1;
                lz.status[ST_BREAK] = 1;
            }
            if (1 >= lz.kmax) lz.status[ST_DONE] = 1;
        }
    }
}

// |x|^2 -> out[slot] (compensated, deterministic)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_norm2(const T *x, int64_t n, double *out,
                                                       double *partials, unsigned *counter) {
    CSum s;
    s.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)x[i];
        s.add(v * v);
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot))
        if (threadIdx.x == 0) *out = tot[0];
}

__global__ void k_scale_by_invsqrt(double *x, int64_t n, const double *n2) {
    const double s = 1.0 / sqrt(*n2);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= s;
}

template <typename TO, typename TI>
__global__ void k_convert(const TI *in, TO *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (TO)in[i];
}

// Deterministic start vector: uniform (0,1] from a splitmix64 hash of
// (seed, i) -- a real counterpart of the seeded random resid the reference
// hands ARPACK (.repo/ARPACK_LANCZOS.f90:394-403).
__global__ void k_random_start(double *x, int64_t n, uint64_t seed) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = random_start_value(i, seed);
}

// ---------------------------------------------------------------------------
static int red_grid(dmfted_ctx *c, int64_t n) {
    return (int)std::min<int64_t>(std::max<int64_t>(div_up(n, kRedThreads), 1),
                                  std::min(kMaxRedBlocks, 4 * num_sms(c)));
}

template <typename T>
static void launch_lz_update(dmfted_ctx *c, T *u, const T *scur, int64_t n, const LanczosScalars &lz,
                             int k, double thr) {
    constexpr int VW = 16 / sizeof(T);
    const bool vec = (n % VW == 0) && ((uintptr_t)u % 16 == 0) && ((uintptr_t)scur % 16 == 0);
    if (vec)
        k_lz_update<T, VW><<<red_grid(c, n / VW), kRedThreads, 0, c->stream>>>(
            u, scur, n, lz, k, thr, c->red_partials.p, c->red_counter.p);
    else
        k_lz_update<T, 1><<<red_grid(c, n), kRedThreads, 0, c->stream>>>(
            u, scur, n, lz, k, thr, c->red_partials.p, c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches++;
}

static int ew_grid(dmfted_ctx *c, int64_t n) {
    return (int)std::min<int64_t>(std::max<int64_t>(div_up(n, 256), 1), 16 * num_sms(c));
}

LanczosScalars lz_slot(dmfted_ctx *c, int slot, int kmax) {
    DM_REQUIRE(slot >= 0 && slot < kLzSlots && kmax <= kLzMax, DMFTED_ERR_ARG,
               "Lanczos scalar slot out of range");
    LanczosScalars lz;
    double *b = c->lz_d.p + (size_t)slot * kLzStride;
    lz.alpha = b;
    lz.beta = b + (kLzMax + 2);
    lz.scale = b + 2 * (kLzMax + 2);
    lz.ritz = b + 3 * (kLzMax + 2);
    lz.status = c->lz_s.p + slot * 8;
    lz.kmax = kmax;
    return lz;
}

static void norm2_device(dmfted_ctx *c, const double *x, int64_t n, double *out) {
    k_norm2<double><<<red_grid(c, n), kRedThreads, 0, c->stream>>>(x, n, out, c->red_partials.p,
                                                                      c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches++;
}

static void ritz_attr(dmfted_ctx *c) {
    static bool done[64] = {false};
    if (done[c->device & 63]) return;
    DM_CUDA(cudaFuncSetAttribute(k_ritz_check, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ritz_smem(kLzMax)));
    DM_CUDA(cudaFuncSetAttribute(k_ritz_vector, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ritz_smem(kLzMax)));
    done[c->device & 63] = true;
}

// One Lanczos step k: the fused H*v launch followed by the update kernel.
template <typename T>
void lanczos_step(dmfted_ctx *c, const SectorView &s, const T *x, const T *xp, T *y, int64_t n,
                  const LanczosScalars &lz, int k, double thr, int nstack) {
    hxv_lanczos_step<T>(c, s, x, xp, y, lz, k, nstack);
    launch_lz_update<T>(c, y, x, n, lz, k, thr);
}
template void lanczos_step<double>(dmfted_ctx *, const SectorView &, const double *,
                                   const double *, double *, int64_t, const LanczosScalars &, int,
                                   double, int);
template void lanczos_step<float>(dmfted_ctx *, const SectorView &, const float *, const float *,
                                  float *, int64_t, const LanczosScalars &, int, double, int);

// One Lanczos run on sector s storing the whole basis in T.
//  start == nullptr : random start vector (deterministic seed)
//  refine == false  : start (FP64) is rounded to T and used as s_0
//  refine == true   : T = float; s_0 = start kept in FP64, the first step
//                     (H s_0 and the residual) runs in FP64, later steps in
//                     FP32; the Ritz vector combines the FP64 s_0 with the
//                     FP32 directions.  Corrections enter the result with
//                     O(residual) coefficients, so FP32 storage of them costs
//                     only ~1e-7 of the correction.
template <typename T>
static LanczosResult gs_run(dmfted_ctx *c, const SectorView &s, double *psi, const double *start,
                            double tol, int nitermax, int ncheck, bool refine) {
    const int64_t dim = s.dim;
    int kmax = (int)std::min<int64_t>(std::min(nitermax, kLzMax - 2), dim);
    const size_t ld = (size_t)((dim + 31) / 32 * 32);
    // The stored basis takes at most 85 % of the device memory left (the
    // buffer already held counts as free), or the context's budget.  A run
    // cut below its iteration limit this way restarts from its Ritz vector
    // (lanczos_gs).
    // The memory query runs only when the basis has to grow, so that a solve
    // whose buffer is already in place makes no driver call here.
    bool capped = false;
    const size_t need = ld * sizeof(T) * (size_t)(kmax + 1);
    if (need > c->work.n || c->gs_basis_budget > 0) {
        double avail = 1e300;
        if (need > c->work.n) {
            size_t free_b = 0, total_b = 0;
            DM_CUDA(cudaMemGetInfo(&free_b, &total_b));
            avail = 0.85 * ((double)free_b + (double)c->work.n);
        }
        if (c->gs_basis_budget > 0) avail = std::min(avail, (double)c->gs_basis_budget);
        const int64_t fit = (int64_t)std::min(avail / (double)(ld * sizeof(T)), 1e9) - 1;
        DM_REQUIRE(fit >= 8 || fit >= kmax, DMFTED_ERR_NOMEM,
                   "ground-state Lanczos: the device holds fewer than 9 basis vectors");
        if (fit < kmax) {
            kmax = (int)fit;
            capped = true;
        }
    }
    c->work.alloc(ld * sizeof(T) * (size_t)(kmax + 1));
    T *basis = reinterpret_cast<T *>(c->work.p);
    LanczosScalars lz = lz_slot(c, 0, kmax);
    ritz_attr(c);
    const int eg = ew_grid(c, dim);
    const int rg = red_grid(c, dim);
    if (start) {
        k_convert<T, double><<<eg, 256, 0, c->stream>>>(start, basis, dim);
    } else {
        c->s64b.alloc(dim);
        k_random_start<<<eg, 256, 0, c->stream>>>(c->s64b.p, dim, 1234567ull);
        k_convert<T, double><<<eg, 256, 0, c->stream>>>(c->s64b.p, basis, dim);
        c->launches++;
    }
    c->launches++;
    if (refine)
        k_lz_init<double><<<rg, kRedThreads, 0, c->stream>>>(start, dim, lz, c->red_partials.p,
                                                              c->red_counter.p);
    else
        k_lz_init<T><<<rg, kRedThreads, 0, c->stream>>>(basis, dim, lz, c->red_partials.p,
                                                         c->red_counter.p);
    c->launches++;
    DM_CHECK_LAUNCH();
    int hst[8] = {0};
    int launched = 0;
    if (refine) {
        // step 0 in FP64
        c->s64c.alloc(dim);
        hxv_lanczos_step<double>(c, s, start, start, c->s64c.p, lz, 0);
        k_lz_update_first<<<rg, kRedThreads, 0, c->stream>>>(
            c->s64c.p, start, reinterpret_cast<float *>(basis + ld), dim, lz, c->red_partials.p,
            c->red_counter.p);
        DM_CHECK_LAUNCH();
        c->launches++;
        launched = 1;
    }
    // Checks fall on multiples of ncheck steps.  From the decay of the Ritz
    // estimate between two checks the loop predicts the steps still needed
    // (linear convergence) and skips checks for at most half of them, so the
    // check that sees convergence is the one the fixed schedule would run,
    // unless convergence more than doubles its pace.
    int every = ncheck;
    double est_prev = -1.0;
    int at_prev = 0;
    while (launched < kmax) {
        for (int j = 0; j < every && launched < kmax; j++, launched++) {
            const int k = launched;
            T *x = basis + (size_t)k * ld;
            const T *xp = basis + (size_t)(k > 0 ? k - 1 : k) * ld;
            T *y = basis + (size_t)(k + 1) * ld;
            lanczos_step<T>(c, s, x, xp, y, dim, lz, k, 1e-300, 1);
        }
        k_ritz_check<<<1, kRedThreads, ritz_smem(launched), c->stream>>>(lz, tol);
        DM_CHECK_LAUNCH();
        c->launches++;
        double rz[2];
        DM_CUDA(cudaMemcpyAsync(hst, lz.status, sizeof(hst), cudaMemcpyDeviceToHost, c->stream));
        DM_CUDA(cudaMemcpyAsync(rz, lz.ritz, sizeof(rz), cudaMemcpyDeviceToHost, c->stream));
        DM_CUDA(cudaStreamSynchronize(c->stream));
        if (hst[ST_DONE]) break;
        every = ncheck;
        const double target = tol * std::max(3.666852862501036e-11, std::fabs(rz[0]));
        if (est_prev > 0.0 && rz[1] > 0.0 && rz[1] < est_prev && launched > at_prev) {
            const double rate = std::log(est_prev / rz[1]) / (launched - at_prev);  // per step
            const double left = std::log(rz[1] / target) / rate;                   // steps to go
            if (left > 2.0 * ncheck) every = ncheck * std::max(1, (int)(0.5 * left / ncheck));
        }
        est_prev = rz[1];
        at_prev = launched;
    }
    if (kmax <= launched && !hst[ST_DONE] && !refine) {
        // (kmax reached inside the loop: the last check above already ran)
    }
    const int n = hst[ST_STEPS];
    double ritz[2];
    DM_CUDA(cudaMemcpy(ritz, lz.ritz, sizeof(ritz), cudaMemcpyDeviceToHost));
    const double e0 = ritz[0];
    double *coef = c->coefb.p;
    k_ritz_vector<<<1, 32, ritz_smem(n), c->stream>>>(lz, n, e0, coef);
    DM_CHECK_LAUNCH();
    k_basis_combine<T><<<eg, 256, 0, c->stream>>>(basis, (int64_t)ld, n, coef,
                                                   refine ? start : nullptr, psi, dim);
    DM_CHECK_LAUNCH();
    norm2_device(c, psi, dim, c->red_out.p);
    k_scale_by_invsqrt<<<eg, 256, 0, c->stream>>>(psi, dim, c->red_out.p);
    DM_CHECK_LAUNCH();
    c->launches += 3;
    DM_CUDA(cudaStreamSynchronize(c->stream));
    LanczosResult res{e0, n, hst[ST_CONV] != 0};
    res.capped = capped;
    return res;
}

// ||H psi - <psi|H|psi> psi|| of a unit FP64 vector: Lanczos step 0 from
// psi (the fused product and the update), read back as beta_1.
static double gs_residual(dmfted_ctx *c, const SectorView &s, const double *psi) {
    LanczosScalars lz = lz_slot(c, 0, 2);
    c->s64c.alloc(s.dim);
    k_lz_init<double><<<red_grid(c, s.dim), kRedThreads, 0, c->stream>>>(
        psi, s.dim, lz, c->red_partials.p, c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches++;
    lanczos_step<double>(c, s, psi, psi, c->s64c.p, s.dim, lz, 0, 1e-300, 1);
    double b1 = 0.0;
    DM_CUDA(cudaMemcpyAsync(&b1, lz.beta + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    return b1;
}

LanczosResult lanczos_gs(dmfted_ctx *c, const SectorView &s, double *psi, const double *start,
                         int precision, double tol, int nitermax) {
    const int ncheck = std::max(1, c->p.lanc_ncheck);
    if (precision == DMFTED_FP64) {
        // The stopping test bounds the residual through its estimate b_n |y_n|
        // from T_n.  After the lowest Ritz pair has converged and the basis
        // has lost orthogonality along it, T_n can hold a second copy of the
        // pair, and the inverse-iteration eigenvector is then some mix of
        // the two copies whose basis combination partly cancels: the energy
        // stays exact, the vector does not.  The true residual of the result
        // is therefore measured (one more H*v), and a run whose residual is
        // well above the test's bound restarts from its own vector -- a
        // short run from a near eigenvector, before any copy can form.
        LanczosResult r = gs_run<double>(c, s, psi, start, tol, nitermax, ncheck, false);
        int steps = r.steps;
        // a basis cut by device memory restarts until its steps add up to
        // about twice the iteration limit
        const int rounds = r.capped ? 3 + 2 * (nitermax + std::max(r.steps, 1) - 1) / std::max(r.steps, 1) : 3;
        for (int round = 0; round < rounds; round++) {
            const double bound = 10.0 * tol * std::max(3.666852862501036e-11, std::fabs(r.e0));
            if (!(gs_residual(c, s, psi) > bound)) break;
            c->s64b.alloc(s.dim);
            DM_CUDA(cudaMemcpyAsync(c->s64b.p, psi, s.dim * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
            r = gs_run<double>(c, s, psi, c->s64b.p, tol, nitermax, ncheck, false);
            steps += r.steps + 1;
            c->gs_restarts++;
        }
        r.steps = steps;
        return r;
    }
    // Mixed: an FP32 run to the FP32 accuracy floor, then refinement runs
    // whose first step is FP64 and whose other steps are FP32, until the
    // FP64 stopping test holds.
    const double tol32 = std::max(tol, c->mixed_tol32);
    LanczosResult r = gs_run<float>(c, s, psi, start, tol32, nitermax, ncheck, false);
    int steps = r.steps;
    const int rounds = r.capped ? 4 + 2 * (nitermax + std::max(r.steps, 1) - 1) / std::max(r.steps, 1) : 4;
    c->s64b.alloc(s.dim);
    for (int round = 0; round < rounds; round++) {
        DM_CUDA(cudaMemcpyAsync(c->s64b.p, psi, s.dim * sizeof(double), cudaMemcpyDeviceToDevice,
                                c->stream));
        r = gs_run<float>(c, s, psi, c->s64b.p, tol, nitermax, std::max(2, ncheck / 2), true);
        steps += r.steps;
        if (r.converged) break;
    }
    r.steps = steps;
    return r;
}

// ---------------------------------------------------------------------------
// Tridiagonalisation of a GF chain; two rotating buffers, no basis.  All
// steps are queued; steps after breakdown are no-ops on the device.
template <typename T>
static void chain_impl(dmfted_ctx *c, const SectorView &s, const double *v0,
                       const LanczosScalars &lz, int nstack) {
    const int64_t dim = s.dim * nstack;
    const size_t ld = (size_t)((dim + 31) / 32 * 32);
    c->chainbuf.alloc(2 * ld * sizeof(T));
    T *P = reinterpret_cast<T *>(c->chainbuf.p), *Q = P + ld;
    const int eg = ew_grid(c, dim);
    DM_CUDA(cudaMemsetAsync(P, 0, ld * sizeof(T), c->stream));
    k_convert<T, double><<<eg, 256, 0, c->stream>>>(v0, Q, dim);
    k_lz_init<T><<<red_grid(c, dim), kRedThreads, 0, c->stream>>>(Q, dim, lz, c->red_partials.p,
                                                                   c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches += 2;
    for (int k = 0; k < lz.kmax; k++) {
        lanczos_step<T>(c, s, Q, P, P, dim, lz, k, c->p.lanc_gf_threshold, nstack);
        std::swap(P, Q);
    }
}

// Mixed-precision chain: the first `head` steps in FP64, then FP32.  The
// Matsubara G(iwn) of a chain depends on its coefficients a_k, b_k with a
// weight that falls off quickly with k (the continued fraction converges
// geometrically off the real axis), and FP32 vectors perturb every
// coefficient at the 1e-7 level.  Computing the leading coefficients in FP64
// and the tail in FP32 keeps G(iwn) at FP64 accuracy (1e-12 or better for 16+
// FP64 steps on the single-orbital baths) while most H*v run in FP32.  At the
// switch the two live vectors are rounded to FP32; their scales (device
// scalars) carry over unchanged.
static void chain_mixed(dmfted_ctx *c, const SectorView &s, const double *v0,
                        const LanczosScalars &lz, int nstack, int head) {
    const int64_t dim = s.dim * nstack;
    const size_t ld = (size_t)((dim + 31) / 32 * 32);
    c->chainbuf.alloc(2 * ld * (sizeof(double) + sizeof(float)));
    double *P = reinterpret_cast<double *>(c->chainbuf.p), *Q = P + ld;
    float *Pf = reinterpret_cast<float *>(Q + ld), *Qf = Pf + ld;
    const int eg = ew_grid(c, dim);
    DM_CUDA(cudaMemsetAsync(P, 0, ld * sizeof(double), c->stream));
    k_convert<double, double><<<eg, 256, 0, c->stream>>>(v0, Q, dim);
    k_lz_init<double><<<red_grid(c, dim), kRedThreads, 0, c->stream>>>(
        Q, dim, lz, c->red_partials.p, c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches += 2;
    const int h = std::min(head, lz.kmax);
    for (int k = 0; k < h; k++) {
        lanczos_step<double>(c, s, Q, P, P, dim, lz, k, c->p.lanc_gf_threshold, nstack);
        std::swap(P, Q);
    }
    if (h >= lz.kmax) return;
    k_convert<float, double><<<eg, 256, 0, c->stream>>>(P, Pf, dim);
    k_convert<float, double><<<eg, 256, 0, c->stream>>>(Q, Qf, dim);
    DM_CHECK_LAUNCH();
    c->launches += 2;
    for (int k = h; k < lz.kmax; k++) {
        lanczos_step<float>(c, s, Qf, Pf, Pf, dim, lz, k, c->p.lanc_gf_threshold, nstack);
        std::swap(Pf, Qf);
    }
}

void lanczos_chain(dmfted_ctx *c, const SectorView &s, const double *v0, int precision,
                   const LanczosScalars &lz, int nstack) {
    if (precision == DMFTED_FP64) chain_impl<double>(c, s, v0, lz, nstack);
    else if (c->gf_head64 > 0) chain_mixed(c, s, v0, lz, nstack, c->gf_head64);
    else chain_impl<float>(c, s, v0, lz, nstack);
}

}  // namespace dmfted

namespace dmfted {

// Tridiagonalisation (FP64) on caller-owned vectors, with the reduction
// scratch and the Lanczos scalars supplied by the caller: nothing here
// allocates.  work holds the two rotating vectors (2*dim doubles).
void lanczos_chain_fixed(dmfted_ctx *c, const SectorView &s, const double *v0, double *work,
                         const LanczosScalars &lz, double *partials, unsigned *counter) {
    const int64_t dim = s.dim;
    double *P = work, *Q = work + dim;
    const int eg = ew_grid(c, dim);
    const int rg = red_grid(c, dim);
    DM_CUDA(cudaMemsetAsync(P, 0, dim * sizeof(double), c->stream));
    k_convert<double, double><<<eg, 256, 0, c->stream>>>(v0, Q, dim);
    k_lz_init<double><<<rg, kRedThreads, 0, c->stream>>>(Q, dim, lz, partials, counter);
    DM_CHECK_LAUNCH();
    c->launches += 2;
    for (int k = 0; k < lz.kmax; k++) {
        hxv_lanczos_step_scratch<double>(c, s, Q, P, P, lz, k, partials, counter);
        const bool vec = (dim % 2 == 0) && ((uintptr_t)P % 16 == 0) && ((uintptr_t)Q % 16 == 0);
        if (vec)
            k_lz_update<double, 2><<<red_grid(c, dim / 2), kRedThreads, 0, c->stream>>>(
                P, Q, dim, lz, k, c->p.lanc_gf_threshold, partials, counter);
        else
            k_lz_update<double, 1><<<rg, kRedThreads, 0, c->stream>>>(
                P, Q, dim, lz, k, c->p.lanc_gf_threshold, partials, counter);
        DM_CHECK_LAUNCH();
        c->launches++;
        std::swap(P, Q);
    }
}

}  // namespace dmfted

// ===========================================================================
// Lowest Neigen eigenpairs of a sector (the finite-temperature call of sp_eigh,
// ED_DIAG.f90:169-183, and the dense small-sector branch :184-194): Lanczos
// with full reorthogonalisation against the stored basis (classical
// Gram-Schmidt, twice), as ARPACK keeps its Krylov basis orthogonal.  Every
// ncheck steps one CTA finds the lowest Neigen Ritz values of T_n by Sturm
// multisection and their Ritz estimates by inverse iteration; all must pass
// ARPACK's test.  A single start vector sees one copy of each degenerate
// eigenvalue.
namespace dmfted {

// Partial reorthogonalisation of the grid-wide eigensolve (the batched
// solver's rule, batch.cu): after the update of step k, one CTA advances the
// orthogonality estimates w_{k+1,j} = <v_{k+1}, v_j> by Simon's recurrence
//   b_{k+1} w_{k+1,j} = b_{j+1} w_{k,j+1} + (a_j - a_k) w_{k,j} + b_j w_{k,j-1}
//                       - b_k w_{k-1,j}   (+ a rounding term)
// and sets pf[0] when max_j |w_{k+1,j}| > sqrt(eps), when the previous step
// triggered one (pf[1]) or every 32nd step; the reorthogonalisation and
// renormalisation kernels of the step do nothing while pf[0] is clear.
// om: three rotating rows of kLzMax+2 estimates; pf[2]: the running
// Gershgorin bound of |T|.
constexpr int kProRow = kLzMax + 2;
__global__ void k_pro_init(double *om, double *pf) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        om[0] = 1.0;  // w_{0,0}
        pf[0] = pf[1] = pf[2] = 0.0;
    }
}
__global__ void __launch_bounds__(kRedThreads) k_pro(LanczosScalars lz, int k, double *om,
                                                     double *pf, double eps) {
    __shared__ double red[kRedThreads / 32];
    __shared__ int s_need;
    const int tid = threadIdx.x;
    if (lz.status[ST_DONE] && lz.status[ST_STEPS] != k + 1) {
        if (tid == 0) pf[0] = 0.0;  // the recurrence has ended: nothing to reorthogonalise
        return;
    }
    const double *w0 = om + ((k + 2) % 3) * kProRow, *w1 = om + (k % 3) * kProRow;
    double *w2 = om + ((k + 1) % 3) * kProRow;
    const double ak = lz.alpha[k], bk = k > 0 ? lz.beta[k] : 0.0, bn = lz.beta[k + 1];
    const double anorm = fmax(pf[2], fabs(ak) + bk + bn);
    const bool force = pf[1] > 0.5, periodic = (k % 32) == 31;
    bool need = force || periodic || !(bn > 0.0);
    if (!need && k > 0) {
        const double inv = 1.0 / bn, rnd = 2.0 * eps * anorm * inv;
        double mx = 0.0;
        for (int j = tid; j < k; j += blockDim.x) {
            double t = lz.beta[j + 1] * w1[j + 1] + (lz.alpha[j] - ak) * w1[j] - bk * w0[j];
            if (j > 0) t += lz.beta[j] * w1[j - 1];
            t = t * inv;
            t += copysign(rnd, t);
            w2[j] = t;
            mx = fmax(mx, fabs(t));
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((tid & 31) == 0) red[tid >> 5] = mx;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
            s_need = m > sqrt(eps);
        }
        __syncthreads();
        need = s_need != 0;
    }
    if (need)
        for (int j = tid; j < k; j += blockDim.x) w2[j] = eps;
    if (tid == 0) {
        w2[k] = bn > 0.0 ? 2.0 * eps * anorm / bn : 0.0;
        w2[k + 1] = 1.0;
        pf[0] = need ? 1.0 : 0.0;
        pf[1] = (need && !force && !periodic) ? 1.0 : 0.0;
        pf[2] = anorm;
        if (bn <= kEigsBreakRel * anorm) {
            // invariant subspace: the run ends here (k_lz_renorm keeps it)
            lz.status[ST_DONE] = 1;
            lz.status[ST_BREAK] = 1;
        }
    }
}

// d_i = <s_i, w> for the nv stored vectors; one CTA per basis vector.  pf:
// the partial-reorthogonalisation flag (skip when pf[0] is clear), or null.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_reorth_dots(const T *basis, int64_t ld, int nv,
                                                             const T *w, int64_t n, double *dots,
                                                             const double *pf) {
    __shared__ double sm[64];
    const int i = blockIdx.x;
    if (i >= nv || (pf && pf[0] < 0.5)) return;
    CSum s;
    s.zero();
    const T *b = basis + (int64_t)i * ld;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) s.add((double)b[j] * (double)w[j]);
    CSum arr[1] = {s};
    block_reduce<1>(arr, sm);
    if (threadIdx.x == 0) dots[i] = arr[0].value();
}

// w -= sum_i <v_i, w> v_i with v_i = sc_i s_i, i.e. coefficient d_i sc_i^2.
template <typename T>
__global__ void k_reorth_update(const T *basis, int64_t ld, int nv, const double *dots,
                                const double *scale, T *w, int64_t n, const double *pf) {
    __shared__ double cf[kLzMax + 8];
    if (pf && pf[0] < 0.5) return;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) cf[i] = dots[i] * scale[i] * scale[i];
    __syncthreads();
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        double acc = (double)w[j];
        for (int i = 0; i < nv; i++) acc -= cf[i] * (double)basis[(int64_t)i * ld + j];
        w[j] = (T)acc;
    }
}

// b_{k+1} = |w| after reorthogonalisation; scale, step count, done flags.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_lz_renorm(const T *w, int64_t n, LanczosScalars lz,
                                                           int k, double thr, double *partials,
                                                           unsigned *counter, const double *pf) {
    if (lz.status[ST_DONE] && lz.status[ST_STEPS] != k + 1) return;
    if (pf && pf[0] < 0.5) return;  // not reorthogonalised: b_{k+1} of the update stands
    CSum s;
    s.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)w[i];
        s.add(v * v);
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot)) {
        if (threadIdx.x == 0) {
            const double b = sqrt(tot[0]);
            lz.beta[k + 1] = b;
            lz.scale[k + 1] = b > 0.0 ? 1.0 / b : 0.0;
            lz.status[ST_STEPS] = k + 1;
            lz.status[ST_DONE] = lz.status[ST_BREAK] ? 1 : 0;
            if (b < thr) {
                lz.status[ST_DONE] = 1;
                lz.status[ST_BREAK] = 1;
            }
            if (k + 1 >= lz.kmax) lz.status[ST_DONE] = 1;
        }
    }
}

// Lowest m Ritz pairs of T_n.  evals[j] (j < m), Y[j*n + i] = eigenvector j
// (inverse iteration, re-orthogonalised against the lower ones in the small
// space), est[j] = b_n |Y[j*n + n-1]|.  Converged when every estimate passes
// ARPACK's test or the recurrence broke down.  Dynamic shared memory:
// ritz_smem(n).  Y lives in global memory (m*n doubles).
__global__ void k_ritz_multi(LanczosScalars lz, double tol, int mwant, double *evals, double *Y,
                             double *est, int final_pass, int work_cap, double top) {
    extern __shared__ double rs[];
    const int n = lz.status[ST_STEPS];
    if (n <= 0) return;
    double *sa = rs, *sb = rs + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sa[i] = lz.alpha[i];
        sb[i] = i > 0 ? lz.beta[i] : 0.0;
    }
    __syncthreads();
    const bool ok = ritz_multi_dev(sa, sb, n, mwant, tol, lz.beta[n], evals, Y, est, rs + 2 * n,
                                   work_cap - 2 * n);
    if (threadIdx.x == 0 && !final_pass) {
        const int m = min(mwant, n);
        if (lz.status[ST_BREAK] || (ok && n >= m && m == mwant) || (ok && n == lz.kmax)) {
            lz.status[ST_CONV] = 1;
            lz.status[ST_DONE] = 1;
        }
        // a probe whose lowest Ritz value stays above top by ten times its
        // residual estimate found nothing it is looking for
        if (evals[0] > top && est[0] <= 0.1 * (evals[0] - top)) lz.status[ST_DONE] = 1;
    }
}

// Dynamic shared memory of k_ritz_multi for up to n steps and m pairs: a, b
// and the eigenvector work spaces of up to 8 concurrent inverse iterations,
// within 200 KB (returned in doubles through cap as well).
constexpr size_t kRitzMultiSmemMax = 200 * 1024;
static size_t ritz_multi_smem(int n, int m, int *cap) {
    int lanes = std::max(1, std::min(m, 8));
    size_t d = 2 * (size_t)n + (size_t)lanes * ritz_evec_doubles(n);
    while (lanes > 1 && d * sizeof(double) > kRitzMultiSmemMax) {
        lanes--;
        d = 2 * (size_t)n + (size_t)lanes * ritz_evec_doubles(n);
    }
    d = std::max(d, (ritz_smem(n) + sizeof(double) - 1) / sizeof(double));
    *cap = (int)d;
    return d * sizeof(double);
}

// coef[j*n + i] = Y[j*n + i] * scale_i
__global__ void k_ritz_coefs(const double *Y, const double *scale, int m, int n, double *coef) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m * n; t += gridDim.x * blockDim.x)
        coef[t] = Y[t] * scale[t % n];
}

// w -= X X^T w for the nlock FP64 locked vectors X (dim apart, orthonormal):
// two classical Gram-Schmidt passes.  dots: nlock doubles; ones: nlock ones.
static void lock_orth(dmfted_ctx *c, const double *X, int nlock, double *w, int64_t dim,
                      double *dots, const double *ones) {
    for (int pass = 0; pass < 2; pass++) {
        k_reorth_dots<double><<<nlock, kRedThreads, 0, c->stream>>>(X, dim, nlock, w, dim, dots,
                                                                    nullptr);
        k_reorth_update<double><<<ew_grid(c, dim), 256, 0, c->stream>>>(X, dim, nlock, dots, ones,
                                                                        w, dim, nullptr);
    }
    DM_CHECK_LAUNCH();
    c->launches += 4;
}

template <typename T>
static int eigs_run(dmfted_ctx *c, const SectorView &s, int neigen, double tol, int nitermax,
                    int ncheck, double *evals_h, double *vecs, const double *locked, int nlock,
                    double top) {
    const int64_t dim = s.dim;
    const int kmax = (int)std::min<int64_t>(std::min(nitermax, kLzMax - 2), dim);
    const size_t ld = (size_t)((dim + 31) / 32 * 32);
    c->work.alloc(ld * sizeof(T) * (size_t)(kmax + 1));
    T *basis = reinterpret_cast<T *>(c->work.p);
    LanczosScalars lz = lz_slot(c, 0, kmax);
    ritz_attr(c);
    static bool attr[64] = {false};
    if (!attr[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(k_ritz_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)std::max(kRitzMultiSmemMax, ritz_smem(kLzMax))));
        attr[c->device & 63] = true;
    }
    const int m = std::min<int64_t>(neigen, dim);
    DM_REQUIRE(nlock == 0 || sizeof(T) == 8, DMFTED_ERR_ARG, "locked eigensolve needs FP64");
    DM_REQUIRE(nlock <= kLzMax, DMFTED_ERR_ARG, "too many locked vectors");
    c->eig_aux.alloc((size_t)64 * 2 + (size_t)m * (kLzMax + 2) * 2 + kLzMax + 8 + 3 * kProRow + 8 +
                     2 * (size_t)(kLzMax + 8));
    double *d_evals = c->eig_aux.p, *d_est = d_evals + 64, *d_Y = d_est + 64;
    double *d_coef = d_Y + (size_t)m * (kLzMax + 2), *d_dots = d_coef + (size_t)m * (kLzMax + 2);
    double *d_om = d_dots + kLzMax + 8, *d_pf = d_om + 3 * kProRow;
    double *d_ldots = d_pf + 8, *d_ones = d_ldots + kLzMax + 8;
    if (nlock > 0) {
        std::vector<double> ones(nlock, 1.0);
        DM_CUDA(cudaMemcpyAsync(d_ones, ones.data(), nlock * sizeof(double), cudaMemcpyHostToDevice,
                                c->stream));
    }
    const double eps = sizeof(T) == 8 ? 1.1102230246251565e-16 : 5.9604644775390625e-8;
    const int eg = ew_grid(c, dim);
    const int rg = red_grid(c, dim);
    c->s64b.alloc(dim);
    k_random_start<<<eg, 256, 0, c->stream>>>(c->s64b.p, dim, eigs_seed(nlock));
    if (nlock > 0) lock_orth(c, locked, nlock, c->s64b.p, dim, d_ldots, d_ones);
    k_convert<T, double><<<eg, 256, 0, c->stream>>>(c->s64b.p, basis, dim);
    k_lz_init<T><<<rg, kRedThreads, 0, c->stream>>>(basis, dim, lz, c->red_partials.p,
                                                     c->red_counter.p);
    k_pro_init<<<1, 32, 0, c->stream>>>(d_om, d_pf);
    DM_CHECK_LAUNCH();
    c->launches += 4;
    int hst[8] = {0};
    int launched = 0;
    while (launched < kmax) {
        for (int j = 0; j < ncheck && launched < kmax; j++, launched++) {
            const int k = launched;
            T *x = basis + (size_t)k * ld;
            const T *xp = basis + (size_t)(k > 0 ? k - 1 : k) * ld;
            T *y = basis + (size_t)(k + 1) * ld;
            hxv_lanczos_step<T>(c, s, x, xp, y, lz, k);
            launch_lz_update<T>(c, y, x, dim, lz, k, 1e-300);
            // locked vectors: H keeps the space orthogonal to them only up to
            // their residuals, so the new vector is projected every step, and
            // its norm is taken again before the orthogonality estimates use it
            if (nlock > 0) {
                lock_orth(c, locked, nlock, reinterpret_cast<double *>(y), dim, d_ldots, d_ones);
                k_lz_renorm<T><<<rg, kRedThreads, 0, c->stream>>>(
                    y, dim, lz, k, 1e-300, c->red_partials.p, c->red_counter.p, nullptr);
                c->launches++;
            }
            k_pro<<<1, kRedThreads, 0, c->stream>>>(lz, k, d_om, d_pf, eps);
            for (int pass = 0; pass < 2; pass++) {
                k_reorth_dots<T><<<k + 1, kRedThreads, 0, c->stream>>>(basis, (int64_t)ld, k + 1, y,
                                                                       dim, d_dots, d_pf);
                k_reorth_update<T><<<eg, 256, 0, c->stream>>>(basis, (int64_t)ld, k + 1, d_dots,
                                                             lz.scale, y, dim, d_pf);
            }
            k_lz_renorm<T><<<rg, kRedThreads, 0, c->stream>>>(y, dim, lz, k, 1e-300,
                                                              c->red_partials.p, c->red_counter.p,
                                                              d_pf);
            DM_CHECK_LAUNCH();
            c->launches += 6;
        }
        int cap = 0;
        const size_t rsm = ritz_multi_smem(launched, m, &cap);
        k_ritz_multi<<<1, kRedThreads, rsm, c->stream>>>(lz, tol, m, d_evals, d_Y, d_est, 0, cap,
                                                         top);
        DM_CHECK_LAUNCH();
        c->launches++;
        DM_CUDA(cudaMemcpyAsync(hst, lz.status, sizeof(hst), cudaMemcpyDeviceToHost, c->stream));
        DM_CUDA(cudaStreamSynchronize(c->stream));
        if (hst[ST_DONE]) break;
    }
    const int n = hst[ST_STEPS];
    const int mm = std::min(m, n);
    int cap = 0;
    const size_t rsm = ritz_multi_smem(n, mm, &cap);
    k_ritz_multi<<<1, kRedThreads, rsm, c->stream>>>(lz, tol, mm, d_evals, d_Y, d_est, 1, cap,
                                                     top);
    k_ritz_coefs<<<div_up((int64_t)mm * n, 256), 256, 0, c->stream>>>(d_Y, lz.scale, mm, n, d_coef);
    for (int j = 0; j < mm; j++) {
        double *v = vecs + (size_t)j * dim;
        k_basis_combine<T><<<eg, 256, 0, c->stream>>>(basis, (int64_t)ld, n, d_coef + (size_t)j * n,
                                                       nullptr, v, dim);
        norm2_device(c, v, dim, c->red_out.p + 3);
        k_scale_by_invsqrt<<<eg, 256, 0, c->stream>>>(v, dim, c->red_out.p + 3);
    }
    DM_CHECK_LAUNCH();
    c->launches += 2 + 3 * mm;
    DM_CUDA(cudaMemcpyAsync(evals_h, d_evals, mm * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    return mm;
}

int lanczos_eigs(dmfted_ctx *c, const SectorView &s, int neigen, int precision, double tol,
                 int nitermax, double *evals_h, double *vecs, int *steps, const double *locked,
                 int nlock, double top) {
    const int ncheck = std::max(1, c->p.lanc_ncheck);
    int m;
    if (precision == DMFTED_FP64 || nlock > 0)
        m = eigs_run<double>(c, s, neigen, tol, nitermax, ncheck, evals_h, vecs, locked, nlock,
                             nlock > 0 ? top : 1e300);
    else
        m = eigs_run<float>(c, s, neigen, std::max(tol, c->mixed_tol32), nitermax, ncheck, evals_h,
                            vecs, nullptr, 0, 1e300);
    int st[8];
    DM_CUDA(cudaMemcpy(st, lz_slot(c, 0, 1).status, sizeof(st), cudaMemcpyDeviceToHost));
    if (steps) *steps = st[ST_STEPS];
    return m;
}

}  // namespace dmfted
