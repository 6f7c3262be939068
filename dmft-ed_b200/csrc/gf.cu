// Green's-function kernels of lanc_build_gf_normal_c
// (ED_GREENS_FUNCTIONS/build_gf_normal.f90:71-180) and get_sigma_normal.
//
// K6 (k_apply_op): the start vector of a particle (c^+) or hole (c) chain in
// the target sector J.  The reference loops over the source states, applies
// cdg/c and finds the target with binary_search (:97-116, :136-155); here
// every target element gathers its unique source through the rank table, so
// the kernel is a coalesced write with one indexed read per element and no
// search.  Sign: (-1)^(occupied levels below the site) in the full word
// |up>|dw> (ED_SETUP.f90:1055-1081); for a down site that includes all nup
// up electrons.
//
// The chains' contributions to G (the pole sums of add_to_lanczos_gf_normal)
// are evaluated as continued fractions in batch.cu.
#include <algorithm>

#include "internal.cuh"
#include "reduce.cuh"

namespace dmfted {

__global__ void __launch_bounds__(kRedThreads) k_apply_op(int ispin, int iorb, int particle,
                                                          int nup_i, int64_t dimup_i,
                                                          int64_t dimup_j, int64_t dim_j,
                                                          int swap_j, const uint32_t *wu_j, const uint32_t *wd_j,
                                                          const int32_t *rank, const double *psi,
                                                          double *vv, double *norm2,
                                                          double *partials, unsigned *counter) {
    const uint32_t bit = 1u << iorb;
    CSum s;
    s.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < dim_j;
         i += (int64_t)gridDim.x * blockDim.x) {
        // (up rank, down rank) of target element i; a swapped target stores
        // idw + DimDw*iup
        const int64_t dimdw_j = dim_j / dimup_j;
        const int64_t rj = swap_j ? i / dimdw_j : i % dimup_j;
        const int64_t cj = swap_j ? i % dimdw_j : i / dimup_j;
        const uint32_t wj = ispin == 0 ? wu_j[rj] : wd_j[cj];
        double val = 0.0;
        // particle: the target holds the site; hole: the target lacks it
        const bool has = (wj & bit) != 0u;
        if (particle ? has : !has) {
            const uint32_t w = particle ? (wj ^ bit) : (wj | bit);
            const int64_t rs = rank[w];
            uint32_t par = __popc(w & (bit - 1u)) & 1u;
            int64_t src;
            if (ispin == 0) {
                src = rs + dimup_i * cj;
            } else {
                par ^= (uint32_t)nup_i & 1u;
                src = rj + dimup_i * rs;
            }
            val = par ? -psi[src] : psi[src];
        }
        vv[i] = val;
        s.add(val * val);
    }
    CSum arr[1] = {s};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot))
        if (threadIdx.x == 0) *norm2 = tot[0];
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    // (a.x + i a.y) / (b.x + i b.y), scaled to avoid overflow (Smith)
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        const double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

// Sigma = G0^-1 - G^-1 with G0^-1 = z + xmu - Hloc_aa - Delta(z),
// Delta(z) = sum_k V_k^2/(z - e_k) (get_sigma_normal.f90:17-39,
// ED_BATH_FUNCTIONS.f90:247-257,1800-1806), and G0and = 1/G0^-1
// (g0and_bath_mats / g0and_bath_real, :1026-1056).  One thread per (spin,
// orbital, frequency).
__global__ void k_sigma(int nspin, int norb, int nbath, const double *e, const double *v,
                        const double *hloc_aa, double xmu, const double *wm, int lmats,
                        const double *wr, int lreal, double eps, const double2 *gm,
                        const double2 *gr, double2 *sm, double2 *sr, double2 *g0m,
                        double2 *g0r) {
    const int L = lmats + lreal;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nspin * norb * L) return;
    const int f = (int)(t % L);
    const int so = (int)(t / L);  // ispin*norb + iorb
    const double2 z = f < lmats ? make_double2(0.0, wm[f]) : make_double2(wr[f - lmats], eps);
    double2 dl = make_double2(0.0, 0.0);
    for (int k = 0; k < nbath; k++) {
        const double vk = v[so * nbath + k], ek = e[so * nbath + k];
        const double2 q = cdiv(make_double2(vk * vk, 0.0), make_double2(z.x - ek, z.y));
        dl.x += q.x;
        dl.y += q.y;
    }
    const double2 ig0 = make_double2(z.x + xmu - hloc_aa[so] - dl.x, z.y - dl.y);
    const double2 g = f < lmats ? gm[(int64_t)so * lmats + f] : gr[(int64_t)so * lreal + f - lmats];
    const double2 ig = cdiv(make_double2(1.0, 0.0), g);
    const double2 sg = make_double2(ig0.x - ig.x, ig0.y - ig.y);
    if (f < lmats) {
        sm[(int64_t)so * lmats + f] = sg;
        g0m[(int64_t)so * lmats + f] = cdiv(make_double2(1.0, 0.0), ig0);
    } else {
        sr[(int64_t)so * lreal + f - lmats] = sg;
        g0r[(int64_t)so * lreal + f - lmats] = cdiv(make_double2(1.0, 0.0), ig0);
    }
}

void gf_apply_op(dmfted_ctx *c, const SectorView &si, const SectorView &sj, int iorb, int ispin,
                 bool particle, const double *psi, double *vv, double *d_norm2) {
    DM_REQUIRE(!si.swapped, DMFTED_ERR_ARG, "apply_op: the source state is in the reference order");
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(div_up(sj.dim, kRedThreads), 1),
                                            std::min(kMaxRedBlocks, 8 * num_sms(c)));
    k_apply_op<<<grid, kRedThreads, 0, c->stream>>>(
        ispin, iorb, particle ? 1 : 0, si.nup, si.dimup, sj.dimup, sj.dim, sj.swapped ? 1 : 0,
        c->words.p + sj.offup,
        c->words.p + sj.offdw, c->rank.p, psi, vv, d_norm2, c->red_partials.p, c->red_counter.p);
    DM_CHECK_LAUNCH();
    c->launches++;
}

void gf_sigma(dmfted_ctx *c) {
    const int L = c->p.lmats + c->p.lreal;
    const int64_t n = (int64_t)c->nspin * c->norb * L;
    if (n <= 0) return;
    k_sigma<<<div_up(n, 256), 256, 0, c->stream>>>(
        c->nspin, c->norb, c->nbath, c->d_bath_e.p, c->d_bath_v.p, c->d_hloc_aa.p, c->p.xmu,
        c->d_wm.p, c->p.lmats, c->d_wr.p, c->p.lreal, c->p.eps, (const double2 *)c->gm.p,
        (const double2 *)c->gr.p, (double2 *)c->sm.p, (double2 *)c->sr.p, (double2 *)c->g0m.p,
        (double2 *)c->g0r.p);
    DM_CHECK_LAUNCH();
    c->launches++;
}

}  // namespace dmfted
