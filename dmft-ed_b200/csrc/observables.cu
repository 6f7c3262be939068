// Thermal-average reductions over a kept state: the density / double
// occupancy loop of observables_impurity (ED_OBSERVABLES.f90:113-160), and
// the Hellmann-Feynman operators of the bath parameters:
//   <n_{k s}>                          derivative w.r.t. e_{s,a,k} (HxVbath.f90)
//   <c^+_{a s} c_{k s} + c^+_{k s} c_{a s}>  derivative w.r.t. V_{s,a,k}
//                                       (HxVimp_bath.f90)
// with the normal bath stride Norb+(iorb-1)*Nbath+k (ED_SETUP.f90:445-462).
//
// Accumulator layout: [0,norb) n_up, [norb,2norb) n_dw, [2norb,3norb) docc,
// then nk[s][a][k] (2*norb*nbath), then hop[s][a][k] (2*norb*nbath), then the
// impurity-configuration histogram P[iu][id] (2^norb x 2^norb: the weight of
// the states whose impurity orbitals hold the up bits iu and down bits id),
// from which local_energy_impurity's diagonal terms follow.
//
// Pair terms (k_obs_pairs, Norb > 1 only): <psi|c^+_{a s} c_{b s}|psi> for
// a != b (the inter-orbital Hloc hopping of Eknot) and the spin-exchange and
// pair-hopping expectations (Dse, Dph) of ED_OBSERVABLES.f90:504-538,585-621,
// layout hl[s][a][b] (2*norb*norb), then se, ph.
//
// Occupations (k_obs_occ, every solve): the state is the DimUp x DimDw matrix
// psi[r, c], and every occupation is diagonal in one spin, so with
// w = |psi|^2 they factor into row sums R_r = sum_c w and column sums
// C_c = sum_r w:  n_up = sum_r R_r n(r), n_dw = sum_c C_c n(c), and
// docc = sum_c n_dw(c) sum_r w n_up(r).  Per element: one square, one
// shared-memory add (the thread's own rows) and Norb FMAs; the bit weights
// are applied per row and per column.  Hop expectations (k_obs_hop) gather
// psi at the hop targets; only the Hellmann-Feynman gradient needs them, so
// they are computed when it is asked for.
//
// CTA partials are folded by a second kernel with compensated sums, in a
// fixed order: the result is reproducible bit for bit.
#include <algorithm>

#include "hxv.cuh"

namespace dmfted {

constexpr int kObsThreads = 64;
constexpr int kOccThreads = 256;

__device__ __forceinline__ double block_sum_occ(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < nw; i++) t += red[i];  // every thread, same order
    return t;
}

// Occupation accumulators [0, 3*norb + 2*norb*nbath) of one state; CTAs own
// columns, threads own rows.  Dynamic shared memory: R[dimup], then the
// CTA's accumulators.
__global__ void __launch_bounds__(kOccThreads) k_obs_occ(HxvArgs<double> a, int nbath,
                                                         const double *psi, int nocc,
                                                         double *partials) {
    extern __shared__ double occ_sm[];
    __shared__ double red[kOccThreads / 32];
    const int tid = threadIdx.x, bd = blockDim.x;
    const int norb = a.norb, pv = norb * nbath, ni = 1 << norb;
    const int nacc = nocc + ni * ni;  // occupations, then the histogram
    const int64_t dimup = a.dimup;
    double *R = occ_sm, *ca = occ_sm + dimup;
    for (int64_t r = tid; r < dimup; r += bd) R[r] = 0.0;
    for (int q = tid; q < nacc; q += bd) ca[q] = 0.0;
    __syncthreads();
    for (int64_t c = blockIdx.x; c < a.dimdw; c += gridDim.x) {
        double sw = 0.0, sd[kMaxNorb] = {0.0, 0.0, 0.0};
        double sh[1 << kMaxNorb] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t r = tid; r < dimup; r += bd) {
            const double x = psi[r + dimup * c];
            const double w = x * x;
            R[r] += w;
            sw += w;
            const uint32_t wu = a.wu[r];
#pragma unroll
            for (int o = 0; o < kMaxNorb; o++)
                if (o < norb) sd[o] += (wu >> o) & 1u ? w : 0.0;
            const uint32_t iu = wu & (uint32_t)(ni - 1);
#pragma unroll
            for (int h = 0; h < (1 << kMaxNorb); h++)
                if (h < ni) sh[h] += iu == (uint32_t)h ? w : 0.0;
        }
        const double csum = block_sum_occ(sw, red);
        double dsum[kMaxNorb];
#pragma unroll
        for (int o = 0; o < kMaxNorb; o++) dsum[o] = o < norb ? block_sum_occ(sd[o], red) : 0.0;
        double hsum[1 << kMaxNorb];
#pragma unroll
        for (int h = 0; h < (1 << kMaxNorb); h++) hsum[h] = h < ni ? block_sum_occ(sh[h], red) : 0.0;
        if (tid == 0) {
            const uint32_t wd = a.wd[c];
            const uint32_t id = wd & (uint32_t)(ni - 1);
            for (int h = 0; h < ni; h++) ca[nocc + h * ni + (int)id] += hsum[h];
            for (int o = 0; o < norb; o++) {
                const bool nd = (wd >> o) & 1u;
                if (nd) {
                    ca[norb + o] += csum;
                    ca[2 * norb + o] += dsum[o];
                }
                for (int k = 0; k < nbath; k++)
                    if ((wd >> (norb + o * nbath + k)) & 1u) ca[3 * norb + pv + o * nbath + k] += csum;
            }
        }
    }
    __syncthreads();
    // row-side occupations from the row sums
    for (int q = 0; q < norb + pv; q++) {
        const int bit = q < norb ? q : norb + (q - norb);
        double v = 0.0;
        for (int64_t r = tid; r < dimup; r += bd)
            if ((a.wu[r] >> bit) & 1u) v += R[r];
        v = block_sum_occ(v, red);
        if (tid == 0) ca[q < norb ? q : 3 * norb + (q - norb)] += v;
    }
    __syncthreads();
    for (int q = tid; q < nacc; q += bd) {
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 0] = ca[q];
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 1] = 0.0;
    }
}

// Pair terms of one state (Norb > 1): per-thread slots in shared memory,
// targets through the rank table.  Signs: a hop b -> a of one spin is
// (-1)^(occupied levels of that spin's word between a and b), the other
// spin's word contributing pairs that cancel; the spin-exchange term moves
// up b -> a and down a -> b, the pair hopping both spins b -> a, and their
// signs are the products of the two one-spin signs (ED_OBSERVABLES.f90:
// 585-621 with c/cdg of ED_SETUP.f90:1055-1081).
__device__ __forceinline__ double hop_sign(uint32_t w, int b, int a) {
    // c_b then c^+_a on word w (bit b set, bit a clear)
    const uint32_t w1 = w & ~(1u << b);
    const int p = __popc(w & ((1u << b) - 1u)) + __popc(w1 & ((1u << a) - 1u));
    return (p & 1) ? -1.0 : 1.0;
}

__global__ void __launch_bounds__(kObsThreads) k_obs_pairs(HxvArgs<double> a, const int32_t *rank,
                                                           const double *psi, int npair,
                                                           int jhflag, double *partials) {
    extern __shared__ double pslot[];  // [npair][kObsThreads]
    const int tid = threadIdx.x;
    const int norb = a.norb;
    for (int q = 0; q < npair; q++) pslot[q * kObsThreads + tid] = 0.0;
    const int64_t dimup = a.dimup;
    for (int64_t cidx = blockIdx.x; cidx < a.dimdw; cidx += gridDim.x) {
        const uint32_t wd = a.wd[cidx];
        for (int64_t r = tid; r < dimup; r += kObsThreads) {
            const double x = psi[r + dimup * cidx];
            const uint32_t wu = a.wu[r];
            for (int ai = 0; ai < norb; ai++)
                for (int bi = 0; bi < norb; bi++) {
                    if (ai == bi) continue;
                    const uint32_t ma = 1u << ai, mb = 1u << bi;
                    const bool ua = wu & ma, ub = wu & mb, da = wd & ma, db = wd & mb;
                    if (!ua && ub) {  // up hop b -> a, same column
                        const int64_t rt = rank[(wu ^ mb) | ma];
                        pslot[(ai * norb + bi) * kObsThreads + tid] +=
                            hop_sign(wu, bi, ai) * x * psi[rt + dimup * cidx];
                    }
                    if (!da && db) {  // down hop b -> a, same row
                        const int64_t qt = rank[(wd ^ mb) | ma];
                        pslot[(norb * norb + ai * norb + bi) * kObsThreads + tid] +=
                            hop_sign(wd, bi, ai) * x * psi[r + dimup * qt];
                    }
                    if (!jhflag) continue;
                    if (ub && da && !db && !ua) {  // spin exchange
                        const int64_t rt = rank[(wu ^ mb) | ma], qt = rank[(wd ^ ma) | mb];
                        pslot[(2 * norb * norb) * kObsThreads + tid] +=
                            hop_sign(wu, bi, ai) * hop_sign(wd, ai, bi) * x * psi[rt + dimup * qt];
                    }
                    if (ub && db && !da && !ua) {  // pair hopping
                        const int64_t rt = rank[(wu ^ mb) | ma], qt = rank[(wd ^ mb) | ma];
                        pslot[(2 * norb * norb + 1) * kObsThreads + tid] +=
                            hop_sign(wu, bi, ai) * hop_sign(wd, bi, ai) * x * psi[rt + dimup * qt];
                    }
                }
        }
    }
    __syncthreads();
    for (int q = tid; q < npair; q += kObsThreads) {
        CSum s;
        s.zero();
        for (int t = 0; t < kObsThreads; t++) s.add(pslot[q * kObsThreads + t]);
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 0] = s.hi;
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 1] = s.lo;
    }
}

// Hop accumulators [0, 2*norb*nbath) (the hop part of the layout) of one
// state: per-thread shared-memory slots, gathers at the hop targets.
__global__ void __launch_bounds__(kObsThreads) k_obs_hop(HxvArgs<double> a, int nbath,
                                                         const double *psi, double *partials) {
    extern __shared__ double slot[];  // [2*pv][kObsThreads]
    const int tid = threadIdx.x;
    const int norb = a.norb, pv = norb * nbath, nh = 2 * pv;
    for (int q = 0; q < nh; q++) slot[q * kObsThreads + tid] = 0.0;
    const int64_t dimup = a.dimup;
    for (int64_t cidx = blockIdx.x; cidx < a.dimdw; cidx += gridDim.x) {
        const int cd = a.cd[cidx];
        for (int64_t r = tid; r < dimup; r += kObsThreads) {
            const double x = psi[r + dimup * cidx];
            const int cu = a.cu[r];
            for (int e = 0; e < cu; e++) {
                const uint32_t en = a.eu[(int64_t)e * dimup + r];
                const int p = ell_par(en);
                if (p >= pv) continue;
                const double y = psi[ell_col(en) + dimup * cidx];
                slot[p * kObsThreads + tid] += ell_neg(en) ? -x * y : x * y;
            }
            for (int e = 0; e < cd; e++) {
                const uint32_t en = a.ed[(int64_t)e * a.dimdw + cidx];
                const int p = ell_par(en);
                if (p >= pv) continue;
                const double y = psi[r + dimup * (int64_t)ell_col(en)];
                slot[(pv + p) * kObsThreads + tid] += ell_neg(en) ? -x * y : x * y;
            }
        }
    }
    __syncthreads();
    for (int q = tid; q < nh; q += kObsThreads) {
        CSum s;
        s.zero();
        for (int t = 0; t < kObsThreads; t++) s.add(slot[q * kObsThreads + t]);
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 0] = s.hi;
        partials[((int64_t)q * gridDim.x + blockIdx.x) * 2 + 1] = s.lo;
    }
}

// One warp per accumulator: the lanes stride over the CTA partials and fold
// them with a fixed-order shuffle reduction (reproducible), so the partials'
// loads are in flight together instead of one after the other.
constexpr int kFoldWarps = 4;
__global__ void __launch_bounds__(32 * kFoldWarps) k_obs_fold(const double *partials, int nblocks,
                                                              int na, double *out) {
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * kFoldWarps + (threadIdx.x >> 5);
    if (q >= na) return;
    CSum s;
    s.zero();
    for (int b = lane; b < nblocks; b += 32)
        s.merge(partials[((int64_t)q * nblocks + b) * 2 + 0],
                partials[((int64_t)q * nblocks + b) * 2 + 1]);
    warp_reduce(s);
    if (lane == 0) out[q] = s.value();
}

int obs_count(const dmfted_ctx *c) {
    return 3 * c->norb + 4 * c->norb * c->nbath + (1 << c->norb) * (1 << c->norb);
}

int obs_pair_count(const dmfted_ctx *c) { return c->norb > 1 ? 2 * c->norb * c->norb + 2 : 0; }

// Raw accumulators of one state (weight 1) into d_out[obs_count] (device):
// the occupations and the impurity histogram, and the hop terms when hops is
// set (else zero); then the pair terms into d_out[obs_count ...
// + obs_pair_count] when Norb > 1.
void observables_raw(dmfted_ctx *c, const SectorView &s, const double *psi, double *d_out,
                     bool hops) {
    HxvArgs<double> a = make_hxv_args<double>(c, s);
    const int na = obs_count(c);
    const int pv = c->norb * c->nbath, nocc = 3 * c->norb + 2 * pv;
    const int nh = (1 << c->norb) * (1 << c->norb);
    const size_t smem = ((size_t)a.dimup + nocc + nh) * sizeof(double);
    DM_REQUIRE(smem <= 200 * 1024, DMFTED_ERR_UNSUPPORTED, "sector rows too long for k_obs_occ");
    static bool attr[64] = {false};
    if (!attr[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(k_obs_occ, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        DM_CUDA(cudaFuncSetAttribute(k_obs_hop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr[c->device & 63] = true;
    }
    const int grid = (int)std::min<int64_t>(s.dimdw, (int64_t)num_sms(c) * 2);
    DM_REQUIRE((int64_t)na * grid * 2 <= (int64_t)c->red_partials.n, DMFTED_ERR_UNSUPPORTED,
               "reduction scratch too small for the observables");
    k_obs_occ<<<grid, kOccThreads, smem, c->stream>>>(a, c->nbath, psi, nocc, c->red_partials.p);
    DM_CHECK_LAUNCH();
    k_obs_fold<<<div_up(nocc, kFoldWarps), 32 * kFoldWarps, 0, c->stream>>>(c->red_partials.p,
                                                                           grid, nocc, d_out);
    // the histogram's partials follow the occupations' (rows nocc .. nocc+nh)
    k_obs_fold<<<div_up(nh, kFoldWarps), 32 * kFoldWarps, 0, c->stream>>>(
        c->red_partials.p + (size_t)nocc * grid * 2, grid, nh, d_out + na - nh);
    DM_CHECK_LAUNCH();
    c->launches += 3;
    const int npair = obs_pair_count(c);
    if (npair > 0) {
        const size_t psmem = (size_t)npair * kObsThreads * sizeof(double);
        const int pgrid = (int)std::min<int64_t>(s.dimdw, (int64_t)num_sms(c) * 4);
        DM_REQUIRE((int64_t)npair * pgrid * 2 <= (int64_t)c->red_partials.n,
                   DMFTED_ERR_UNSUPPORTED, "reduction scratch too small for the pair terms");
        k_obs_pairs<<<pgrid, kObsThreads, psmem, c->stream>>>(a, c->rank.p + 0, psi, npair,
                                                              c->p.jhflag, c->red_partials.p);
        DM_CHECK_LAUNCH();
        k_obs_fold<<<div_up(npair, kFoldWarps), 32 * kFoldWarps, 0, c->stream>>>(
            c->red_partials.p, pgrid, npair, d_out + na);
        DM_CHECK_LAUNCH();
        c->launches += 2;
    }
    if (!hops) {
        DM_CUDA(cudaMemsetAsync(d_out + nocc, 0, (size_t)(2 * pv) * sizeof(double), c->stream));
        return;
    }
    const size_t hsmem = (size_t)2 * pv * kObsThreads * sizeof(double);
    DM_REQUIRE(hsmem <= 200 * 1024, DMFTED_ERR_UNSUPPORTED, "too many bath levels for k_obs_hop");
    const int occ = std::max(1, (int)((200 * 1024) / std::max<size_t>(hsmem, 1)));
    const int hgrid = (int)std::min<int64_t>(s.dimdw, (int64_t)num_sms(c) * std::min(occ, 8));
    DM_REQUIRE((int64_t)2 * pv * hgrid * 2 <= (int64_t)c->red_partials.n, DMFTED_ERR_UNSUPPORTED,
               "reduction scratch too small for the observables");
    k_obs_hop<<<hgrid, kObsThreads, hsmem, c->stream>>>(a, c->nbath, psi, c->red_partials.p);
    DM_CHECK_LAUNCH();
    k_obs_fold<<<div_up(2 * pv, kFoldWarps), 32 * kFoldWarps, 0, c->stream>>>(
        c->red_partials.p, hgrid, 2 * pv, d_out + nocc);
    DM_CHECK_LAUNCH();
    c->launches += 2;
}

}  // namespace dmfted
