// Batched chi^2 of the Delta fit and its reverse-mode gradient, for many bath
// parameter sets at once (the reference evaluates one set per call inside
// SciFortran's fmin_cg):
//   Delta_n   = sum_k V_k^2 / (i w_n - e_k)           delta_normal_normal
//   chi2      = sum_n |G_n - Delta_n|^2 / W_n          chi2_delta_normal_normal
//   d chi2/da = -2 sum_n [Re(G-Delta) Re dDelta + Im(G-Delta) Im dDelta] / W_n
//   dDelta/de_k = V_k^2/(i w_n - e_k)^2,  dDelta/dV_k = 2 V_k/(i w_n - e_k)
// (ED_CHI2FIT/fitgf_normal_normal.f90:193-226,256-316).
//
// One CTA per parameter set, threads over Matsubara points; r_k = 1/(i w - e_k)
// is formed once per (n, k) with a single FP64 reciprocal and reused for
// Delta and both derivatives.  Per-thread accumulators sit in shared-memory
// slots and are folded in a fixed order (deterministic).  The work is FP64
// arithmetic on a few MB, so the bound is the FP64 pipe, not HBM.
#include <algorithm>

#include "internal.cuh"
#include "reduce.cuh"

namespace dmfted {

__global__ void k_chi2(int nbath, int L, const double *a, const double *x, const double2 *g,
                       const double *w, double *chi2, double *grad) {
    extern __shared__ double sm[];
    const int nt = blockDim.x, tid = threadIdx.x;
    const int b = blockIdx.x;
    const int na = 1 + 2 * nbath;
    double *pe = sm, *pv = sm + nbath;        // parameters
    double *acc = sm + 2 * nbath;              // [na][nt]
    double *rr = acc + (size_t)na * nt;        // [nbath][nt] real part of r_k
    double *ri = rr + (size_t)nbath * nt;      // imaginary part
    for (int k = tid; k < 2 * nbath; k += nt) sm[k] = a[(int64_t)b * 2 * nbath + k];
    for (int q = 0; q < na; q++) acc[q * nt + tid] = 0.0;
    __syncthreads();
    for (int n = tid; n < L; n += nt) {
        const double om = x[n];
        const double2 gn = g[n];
        const double iw = 1.0 / w[n];
        double dre = 0.0, dim = 0.0;
        for (int k = 0; k < nbath; k++) {
            const double e = pe[k], v = pv[k];
            const double inv = 1.0 / (e * e + om * om);
            const double re = -e * inv, im = -om * inv;  // 1/(i om - e)
            rr[k * nt + tid] = re;
            ri[k * nt + tid] = im;
            dre += v * v * re;
            dim += v * v * im;
        }
        const double Rr = gn.x - dre, Ri = gn.y - dim;
        acc[tid] += (Rr * Rr + Ri * Ri) * iw;
        for (int k = 0; k < nbath; k++) {
            const double v = pv[k], re = rr[k * nt + tid], im = ri[k * nt + tid];
            // dDelta/de = v^2 r^2 ; dDelta/dV = 2 v r
            const double r2r = re * re - im * im, r2i = 2.0 * re * im;
            acc[(1 + k) * nt + tid] += (Rr * v * v * r2r + Ri * v * v * r2i) * iw;
            acc[(1 + nbath + k) * nt + tid] += (Rr * 2.0 * v * re + Ri * 2.0 * v * im) * iw;
        }
    }
    __syncthreads();
    for (int q = tid; q < na; q += nt) {
        CSum s;
        s.zero();
        for (int t = 0; t < nt; t++) s.add(acc[q * nt + t]);
        const double val = s.value();
        if (q == 0) chi2[b] = val;
        else if (grad) grad[(int64_t)b * 2 * nbath + (q - 1)] = -2.0 * val;
    }
}

void chi2_batch_device(dmfted_ctx *c, int nbatch, int nbath, int L, const double *a,
                       const double *x, const double *g, const double *w, double *chi2,
                       double *grad) {
    DM_REQUIRE(nbatch > 0 && nbath > 0 && L > 0, DMFTED_ERR_ARG, "chi2: empty batch or grid");
    int nt = 128;
    auto bytes = [&](int t) { return (size_t)(2 * nbath + (1 + 2 * nbath) * t + 2 * nbath * t) * 8; };
    while (nt > 32 && bytes(nt) > 160 * 1024) nt /= 2;
    DM_REQUIRE(bytes(nt) <= 200 * 1024, DMFTED_ERR_UNSUPPORTED, "chi2: too many bath levels");
    // the attribute belongs to the device current when it is set: once per device
    static bool attr[64] = {false};
    if (!attr[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(k_chi2, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr[c->device & 63] = true;
    }
    k_chi2<<<nbatch, nt, bytes(nt), c->stream>>>(nbath, L, a, x, (const double2 *)g, w, chi2, grad);
    DM_CHECK_LAUNCH();
    c->launches++;
}

}  // namespace dmfted
