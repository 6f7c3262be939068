// Thermal-average reductions over a kept state: the density / double
// occupancy loop of observables_impurity (ED_OBSERVABLES.f90:113-160), and
// the Hellmann-Feynman operators of the bath parameters:
//   <n_{k s}>                          derivative w.r.t. e_{s,a,k} (HxVbath.f90)
//   <c^+_{a s} c_{k s} + c^+_{k s} c_{a s}>  derivative w.r.t. V_{s,a,k}
//                                       (HxVimp_bath.f90)
// with the normal bath stride Norb+(iorb-1)*Nbath+k (ED_SETUP.f90:445-462).
//
// One pass over the state vector.  Accumulators (NA of them) live in
// per-thread shared-memory slots (no atomics), are folded per CTA in a fixed
// order, and a second kernel folds the CTA partials with compensated sums,
// so the result is reproducible bit for bit.
//
// Accumulator layout: [0,norb) n_up, [norb,2norb) n_dw, [2norb,3norb) docc,
// then nk[s][a][k] (2*norb*nbath), then hop[s][a][k] (2*norb*nbath).
#include <algorithm>

#include "hxv.cuh"

namespace dmfted {

constexpr int kObsThreads = 64;

__global__ void __launch_bounds__(kObsThreads) k_obs(HxvArgs<double> a, int nbath, const double *psi,
                                                     int na, double *partials) {
    extern __shared__ double slot[];  // [na][kObsThreads]
    const int tid = threadIdx.x;
    const int norb = a.norb, pv = norb * nbath;
    for (int q = 0; q < na; q++) slot[q * kObsThreads + tid] = 0.0;
    const int off_nk = 3 * norb, off_hop = 3 * norb + 2 * pv;
    const int64_t dimup = a.dimup;
    for (int64_t cidx = blockIdx.x; cidx < a.dimdw; cidx += gridDim.x) {
        const uint32_t wd = a.wd[cidx];
        const int cd = a.cd[cidx];
        for (int64_t r = tid; r < dimup; r += kObsThreads) {
            const double x = psi[r + dimup * cidx];
            const double w = x * x;
            const uint32_t wu = a.wu[r];
            for (int o = 0; o < norb; o++) {
                const double nu = (wu >> o) & 1u, nd = (wd >> o) & 1u;
                slot[o * kObsThreads + tid] += w * nu;
                slot[(norb + o) * kObsThreads + tid] += w * nd;
                slot[(2 * norb + o) * kObsThreads + tid] += w * nu * nd;
            }
            for (int o = 0; o < norb; o++)
                for (int k = 0; k < nbath; k++) {
                    const int ms = norb + o * nbath + k;
                    const int p = o * nbath + k;
                    slot[(off_nk + p) * kObsThreads + tid] += w * (double)((wu >> ms) & 1u);
                    slot[(off_nk + pv + p) * kObsThreads + tid] += w * (double)((wd >> ms) & 1u);
                }
            const int cu = a.cu[r];
            for (int e = 0; e < cu; e++) {
                const uint32_t en = a.eu[(int64_t)e * dimup + r];
                const int p = ell_par(en);
                if (p >= pv) continue;
                const double y = psi[ell_col(en) + dimup * cidx];
                slot[(off_hop + p) * kObsThreads + tid] += ell_neg(en) ? -x * y : x * y;
            }
            for (int e = 0; e < cd; e++) {
                const uint32_t en = a.ed[(int64_t)e * a.dimdw + cidx];
                const int p = ell_par(en);
                if (p >= pv) continue;
                const double y = psi[r + dimup * (int64_t)ell_col(en)];
                slot[(off_hop + pv + p) * kObsThreads + tid] += ell_neg(en) ? -x * y : x * y;
            }
        }
    }
    __syncthreads();
    for (int q = tid; q < na; q += kObsThreads) {
        CSum s;
        s.zero();
        for (int t = 0; t < kObsThreads; t++) s.add(slot[q * kObsThreads + t]);
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 0] = s.hi;
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 1] = s.lo;
    }
}

__global__ void k_obs_fold(const double *partials, int nblocks, int na, double *out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na; q += gridDim.x * blockDim.x) {
        CSum s;
        s.zero();
        for (int b = 0; b < nblocks; b++)
            s.merge(partials[((int64_t)q * nblocks + b) * 2 + 0],
                    partials[((int64_t)q * nblocks + b) * 2 + 1]);
        out[q] = s.value();
    }
}

int obs_count(const dmfted_ctx *c) { return 3 * c->norb + 4 * c->norb * c->nbath; }

// Raw accumulators of one state (weight 1) into d_out[obs_count] (device).
void observables_raw(dmfted_ctx *c, const SectorView &s, const double *psi, double *d_out) {
    HxvArgs<double> a = make_hxv_args<double>(c, s);
    const int na = obs_count(c);
    const size_t smem = (size_t)na * kObsThreads * sizeof(double);
    DM_REQUIRE(smem <= 200 * 1024, DMFTED_ERR_UNSUPPORTED, "too many bath levels for k_obs");
    static bool attr = false;
    if (!attr) {
        DM_CUDA(cudaFuncSetAttribute(k_obs, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    const int occ = std::max(1, (int)((200 * 1024) / std::max<size_t>(smem, 1)));
    const int grid = (int)std::min<int64_t>(s.dimdw, (int64_t)num_sms(c) * std::min(occ, 8));
    DM_REQUIRE((int64_t)na * grid * 2 <= (int64_t)c->red_partials.n, DMFTED_ERR_UNSUPPORTED,
               "reduction scratch too small for the observables");
    k_obs<<<grid, kObsThreads, smem, c->stream>>>(a, c->nbath, psi, na, c->red_partials.p);
    DM_CHECK_LAUNCH();
    k_obs_fold<<<div_up(na, 128), 128, 0, c->stream>>>(c->red_partials.p, grid, na, d_out);
    DM_CHECK_LAUNCH();
    c->launches += 2;
}

}  // namespace dmfted
