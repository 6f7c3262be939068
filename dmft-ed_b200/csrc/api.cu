// C-ABI entry points (include/dmfted.h) and the host orchestration of
// ed_solve_single for the normal mode.  Every entry point converts exceptions
// into status codes; nothing here falls back to a host computation of the hot
// path.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"

namespace dmfted {

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
const char *last_error() { return g_last_error.c_str(); }

// binomial of ED_SETUP.f90:1258-1275 (FP64 running product, int(x+0.5)), used
// for the exported sector tables so they match the reference's integers.
static int32_t ref_binomial(int n1, int n2) {
    double xh = 1.0;
    if (n2 < 0) return 0;
    if (n2 == 0) return 1;
    for (int i = 1; i <= n2; i++) xh = xh * (double)(n1 + 1 - i) / (double)i;
    return (int32_t)(xh + 0.5);
}

// setup_pointers_normal, ED_SETUP.f90:379-493 (normal ed_mode, normal bath).
static void setup_pointers_normal(dmfted_ctx *c) {
    const int ns = c->ns, norb = c->norb, nbath = c->nbath;
    const int nsect = (ns + 1) * (ns + 1);
    c->nsectors = nsect;
    c->getsector.assign((ns + 1) * (ns + 1), 0);
    c->getnup.assign(nsect, 0);
    c->getndw.assign(nsect, 0);
    c->getdim.assign(nsect, 0);
    c->getdimup.assign(nsect, 0);
    c->getdimdw.assign(nsect, 0);
    c->getcsector.assign(2 * nsect, 0);
    c->getcdgsector.assign(2 * nsect, 0);
    c->getbathstride.assign(norb * nbath, 0);
    c->impindex.assign(2 * norb, 0);
    int is = 0;
    for (int nup = 0; nup <= ns; nup++)
        for (int ndw = 0; ndw <= ns; ndw++) {
            is++;
            c->getsector[nup * (ns + 1) + ndw] = is;
            c->getnup[is - 1] = nup;
            c->getndw[is - 1] = ndw;
            c->getdim[is - 1] = ref_binomial(ns, nup) * ref_binomial(ns, ndw);
            c->getdimup[is - 1] = ref_binomial(ns, nup);
            c->getdimdw[is - 1] = ref_binomial(ns, ndw);
        }
    for (int in = 1; in <= norb; in++) {
        c->impindex[in - 1] = in;
        c->impindex[norb + in - 1] = in + ns;
    }
    for (int i = 1; i <= nbath; i++)
        for (int iorb = 1; iorb <= norb; iorb++)
            c->getbathstride[(i - 1) * norb + iorb - 1] = norb + (iorb - 1) * nbath + i;
    for (int s = 1; s <= nsect; s++) {
        const int nup = c->getnup[s - 1], ndw = c->getndw[s - 1];
        if (nup - 1 >= 0) c->getcsector[2 * (s - 1) + 0] = c->getsector[(nup - 1) * (ns + 1) + ndw];
        if (ndw - 1 >= 0) c->getcsector[2 * (s - 1) + 1] = c->getsector[nup * (ns + 1) + ndw - 1];
        if (nup + 1 <= ns) c->getcdgsector[2 * (s - 1) + 0] = c->getsector[(nup + 1) * (ns + 1) + ndw];
        if (ndw + 1 <= ns) c->getcdgsector[2 * (s - 1) + 1] = c->getsector[nup * (ns + 1) + ndw + 1];
    }
    c->neigen_sector.assign(nsect, 0);
    for (int s = 0; s < nsect; s++)
        c->neigen_sector[s] = std::min(c->getdim[s], c->p.lanc_nstates_sector);
    c->twin_mask.assign(nsect, 1);
    if (c->p.ed_twin)
        for (int s = 0; s < nsect; s++)
            if (c->getnup[s] < c->getndw[s]) c->twin_mask[s] = 0;
}

static void check_hloc(const dmfted_ctx *c, const double *h) {
    const int ns = c->nspin, no = c->norb;
    for (int is = 0; is < ns; is++)
        for (int js = 0; js < ns; js++)
            for (int a = 0; a < no; a++)
                for (int b = 0; b < no; b++) {
                    const int64_t idx = is + ns * (js + ns * (a + (int64_t)no * b));
                    const double re = h[2 * idx], im = h[2 * idx + 1];
                    DM_REQUIRE(std::isfinite(re) && std::isfinite(im), DMFTED_ERR_ARG,
                               "Hloc has a non-finite entry");
                    DM_REQUIRE(im == 0.0, DMFTED_ERR_UNSUPPORTED,
                               "complex Hloc: this solver runs the real normal-bath Hamiltonian");
                    DM_REQUIRE(is == js || re == 0.0, DMFTED_ERR_UNSUPPORTED,
                               "spin off-diagonal Hloc belongs to ed_mode=nonsu2");
                }
}

static void upload_model(dmfted_ctx *c) {
    const int nso = c->nspin * c->norb;
    c->d_bath_e.alloc(std::max<size_t>(c->bath_e.size(), 1));
    c->d_bath_v.alloc(std::max<size_t>(c->bath_v.size(), 1));
    c->d_hloc_aa.alloc(nso);
    std::vector<double> haa(nso);
    for (int is = 0; is < c->nspin; is++)
        for (int a = 0; a < c->norb; a++) {
            const int64_t idx = is + c->nspin * (is + c->nspin * (a + (int64_t)c->norb * a));
            haa[is * c->norb + a] = c->hloc[2 * idx];
        }
    if (!c->bath_e.empty()) {
        DM_CUDA(cudaMemcpyAsync(c->d_bath_e.p, c->bath_e.data(), c->bath_e.size() * 8,
                                cudaMemcpyHostToDevice, c->stream));
        DM_CUDA(cudaMemcpyAsync(c->d_bath_v.p, c->bath_v.data(), c->bath_v.size() * 8,
                                cudaMemcpyHostToDevice, c->stream));
    }
    DM_CUDA(cudaMemcpyAsync(c->d_hloc_aa.p, haa.data(), nso * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
}

// Kept states of the eigenspace: a device pool of FP64 vectors.
static cudaEvent_t hv_event(dmfted_ctx *c) {
    if (!c->hv_ev_free.empty()) {
        cudaEvent_t e = c->hv_ev_free.back();
        c->hv_ev_free.pop_back();
        return e;
    }
    cudaEvent_t e;
    DM_CUDA(cudaEventCreate(&e));
    return e;
}

void hv_timer_begin(dmfted_ctx *c) {
    if (!c->hv_timing) return;
    cudaEvent_t a = hv_event(c), b = hv_event(c);
    DM_CUDA(cudaEventRecord(a, c->stream));
    c->hv_ev.emplace_back(a, b);
}

void hv_timer_end(dmfted_ctx *c, double bytes) {
    if (!c->hv_timing || c->hv_ev.size() == c->hv_ev_bytes.size()) return;
    DM_CUDA(cudaEventRecord(c->hv_ev.back().second, c->stream));
    c->hv_ev_bytes.push_back(bytes);
}

// Folds the recorded pairs into the totals (waits for both streams).  The
// time is the union of the launches' intervals, all measured from the first
// event: H*v launches of two concurrent chains overlap, and the union is the
// device time during which any H*v ran (equal to the sum when they do not).
static void hv_timer_collect(dmfted_ctx *c) {
    if (c->hv_ev.empty()) return;
    DM_CUDA(cudaStreamSynchronize(c->stream));
    if (c->stream2) DM_CUDA(cudaStreamSynchronize(c->stream2));
    std::vector<std::pair<float, float>> iv;
    const cudaEvent_t base = c->hv_ev.front().first;
    for (size_t i = 0; i < c->hv_ev_bytes.size(); i++) {
        float t0 = 0.f, t1 = 0.f;
        DM_CUDA(cudaEventElapsedTime(&t0, base, c->hv_ev[i].first));
        DM_CUDA(cudaEventElapsedTime(&t1, base, c->hv_ev[i].second));
        iv.emplace_back(t0, t1);
        c->hv_bytes += c->hv_ev_bytes[i];
        c->hv_count++;
    }
    std::sort(iv.begin(), iv.end());
    double lo = -1.0, hi = -1.0;
    for (auto &x : iv) {
        if (x.first > hi) {
            if (hi > lo) c->hv_ms += hi - lo;
            lo = x.first;
            hi = x.second;
        } else {
            hi = std::max<double>(hi, x.second);
        }
    }
    if (hi > lo) c->hv_ms += hi - lo;
    for (auto &pr : c->hv_ev) {
        c->hv_ev_free.push_back(pr.first);
        c->hv_ev_free.push_back(pr.second);
    }
    c->hv_ev.clear();
    c->hv_ev_bytes.clear();
}

__global__ void k_interleave_split(const double *z, double *re, double *im, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        re[i] = z[2 * i];
        im[i] = z[2 * i + 1];
    }
}
__global__ void k_interleave_join(const double *re, const double *im, double *z, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        z[2 * i] = re[i];
        z[2 * i + 1] = im ? im[i] : 0.0;
    }
}

static int ew(dmfted_ctx *c, int64_t n) {
    return (int)std::min<int64_t>(std::max<int64_t>(div_up(n, 256), 1), 16 * num_sms(c));
}

// Copy a device FP64 real vector to a host complex128 array (imag = 0).
static void real_to_host_c128(dmfted_ctx *c, const double *d, int64_t n, double *host) {
    c->wv64.alloc(2 * n);
    k_interleave_join<<<ew(c, n), 256, 0, c->stream>>>(d, nullptr, c->wv64.p, n);
    DM_CHECK_LAUNCH();
    c->launches++;
    DM_CUDA(cudaMemcpyAsync(host, c->wv64.p, 2 * n * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
}

// ed_analysis, finite-temperature part (ED_DIAG.f90:248-398): Z from the full
// list, then the per-sector Neigen adaptation and the cutoff trimming /
// lanc_nstates_total growth that the next solve uses.
static void ed_analysis_finite_t(dmfted_ctx *c) {
    const dmfted_params &p = c->p;
    c->egs = c->states.front().e;
    double z = 0.0;
    for (auto &st : c->states) z += std::exp(-p.beta * (st.e - c->egs));
    c->zeta = z;
    std::vector<int> count(c->nsectors, 0);
    for (auto &st : c->states) count[st.isector - 1]++;
    for (int i = 0; i < c->nsectors; i++) {
        int &ne = c->neigen_sector[i];
        if (count[i] > 0) ne++;
        else ne--;
        if (ne > count[i]) ne = count[i] + 1;
        if (ne <= 0) ne = 1;
    }
    const double ec = c->states.back().e;
    if (std::exp(-p.beta * (ec - c->egs)) > p.cutoff) {
        c->nstates_total += p.lanc_nstates_step;
    } else {
        while (c->states.size() > 1 &&
               std::exp(-p.beta * (c->states.back().e - c->egs)) <= p.cutoff)
            states_pop_last(c);
        c->nstates_total =
            std::max<int>((int)c->states.size(), p.lanc_nstates_step) + p.lanc_nstates_step;
    }
}

// ---------------------------------------------------------------------------
// The solve.  Mirrors ed_solve_single (ED_MAIN.f90:251-289):
//   diagonalize_impurity -> ed_diag_c (sector loop and state selection,
//   ED_DIAG.f90:93-228) + ed_analysis (Z, ED_DIAG.f90:248-277)
//   observables_impurity (n, docc, ED_OBSERVABLES.f90:113-160)
//   buildgf_impurity -> lanc_build_gf_normal_c per (iorb, ispin)
//   (build_gf_normal.f90:4-16,71-180) -> get_sigma_normal.

// Thermal average of the raw accumulators over the kept states, with the
// Boltzmann weights of ED_OBSERVABLES.f90:128-129 (T=0: 1/Z over the ground
// states); hops: include the hop terms of the Hellmann-Feynman gradient.
// The pair terms (obs_pair_count entries after the weighted ones) are summed
// over the states without weights, as local_energy_impurity sums them.
static std::vector<double> thermal_observables(dmfted_ctx *c, bool hops) {
    // every state's accumulators into its own slot, then one copy and one wait
    const int na = obs_count(c), np = obs_pair_count(c), nt = na + np;
    const size_t ns = c->states.size();
    c->obs_d.alloc(std::max<size_t>(ns, 1) * nt);
    for (size_t i = 0; i < ns; i++) {
        const auto &st = c->states[i];
        observables_raw(c, sector_view(c, st.isector), c->states64.p + st.off,
                        c->obs_d.p + i * nt, hops);
    }
    std::vector<double> all(ns * nt), acc(nt, 0.0);
    DM_CUDA(cudaMemcpyAsync(all.data(), c->obs_d.p, all.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < ns; i++) {
        const auto &st = c->states[i];
        const double peso =
            (c->finite_t ? std::exp(-c->p.beta * (st.e - c->egs)) : 1.0) / c->zeta;
        for (int q = 0; q < na; q++) acc[q] += peso * all[i * nt + q];
        for (int q = na; q < nt; q++) acc[q] += all[i * nt + q];
    }
    return acc;
}

// local_energy_impurity (ED_OBSERVABLES.f90:454-635) from the thermal
// accumulators: the diagonal terms from the weighted impurity-configuration
// histogram, the inter-orbital Hloc hopping of Eknot and the spin-exchange /
// pair-hopping terms from the unweighted pair sums (the reference adds those
// three without the state weight).  c->eloc = {Epot, Eint, Ehartree, Eknot,
// Dust, Dund, Dse, Dph}; Epot includes Ehartree, and Eint, which the
// reference declares but never assigns, is 0.
static void local_energies(dmfted_ctx *c, const std::vector<double> &acc) {
    const dmfted_params &p = c->p;
    const int no = c->norb, ni = 1 << no, ns = c->nspin;
    const int na = obs_count(c);
    const double *P = acc.data() + na - ni * ni;
    auto hl = [&](int is, int a, int b) {
        const int64_t idx = is + ns * (is + ns * (a + (int64_t)no * b));
        return c->hloc[2 * idx];
    };
    double eknot = 0.0, epot = 0.0, ehart = 0.0, dust = 0.0, dund = 0.0, dse = 0.0, dph = 0.0;
    for (int iu = 0; iu < ni; iu++)
        for (int id = 0; id < ni; id++) {
            const double w = P[iu * ni + id];
            double nu[kMaxNorb], nd[kMaxNorb];
            for (int a = 0; a < no; a++) {
                nu[a] = (iu >> a) & 1;
                nd[a] = (id >> a) & 1;
            }
            for (int a = 0; a < no; a++) eknot += (hl(0, a, a) * nu[a] + hl(ns - 1, a, a) * nd[a]) * w;
            for (int a = 0; a < no; a++) epot += p.uloc[a] * nu[a] * nd[a] * w;
            for (int a = 0; a < no; a++)
                for (int b = a + 1; b < no; b++) {
                    const double ud = nu[a] * nd[b] + nu[b] * nd[a];
                    const double uu = nu[a] * nu[b] + nd[a] * nd[b];
                    epot += p.ust * ud * w + (p.ust - p.jh) * uu * w;
                    dust += ud * w;
                    dund += uu * w;
                }
            if (p.hfmode) {
                for (int a = 0; a < no; a++)
                    ehart += -0.5 * p.uloc[a] * (nu[a] + nd[a]) * w + 0.25 * p.uloc[a] * w;
                for (int a = 0; a < no; a++)
                    for (int b = a + 1; b < no; b++) {
                        const double nn = nu[a] + nd[a] + nu[b] + nd[b];
                        ehart += -0.5 * p.ust * nn * w + 0.25 * p.ust * w;
                        ehart += -0.5 * (p.ust - p.jh) * nn * w + 0.25 * (p.ust - p.jh) * w;
                    }
            }
        }
    if (no > 1) {
        const double *pr = acc.data() + na;
        for (int a = 0; a < no; a++)
            for (int b = 0; b < no; b++) {
                if (a == b) continue;
                eknot += hl(0, a, b) * pr[a * no + b] + hl(ns - 1, a, b) * pr[no * no + a * no + b];
            }
        if (p.jhflag) {
            dse = pr[2 * no * no];
            dph = pr[2 * no * no + 1];
            epot += p.jx * dse + p.jp * dph;
        }
    }
    epot += ehart;
    c->eloc = {epot, 0.0, ehart, eknot, dust, dund, dse, dph};
}

// sz2, n2 and s2tot of observables_impurity (ED_OBSERVABLES.f90:131-160)
// from the weighted impurity-configuration histogram: sz_a = (n_a,up -
// n_a,dw)/2, n_a = n_a,up + n_a,dw, s2tot = <(sum_a sz_a)^2>.
static void spin_charge_moments(dmfted_ctx *c, const std::vector<double> &acc) {
    const int no = c->norb, ni = 1 << no;
    const double *P = acc.data() + obs_count(c) - ni * ni;
    c->sz2.assign((size_t)no * no, 0.0);
    c->n2.assign((size_t)no * no, 0.0);
    c->s2tot = 0.0;
    for (int iu = 0; iu < ni; iu++)
        for (int id = 0; id < ni; id++) {
            const double w = P[iu * ni + id];
            double sz[kMaxNorb], nt[kMaxNorb], stot = 0.0;
            for (int a = 0; a < no; a++) {
                const double u = (iu >> a) & 1, d = (id >> a) & 1;
                sz[a] = (u - d) / 2.0;
                nt[a] = u + d;
                stot += sz[a];
            }
            for (int a = 0; a < no; a++)
                for (int b = 0; b < no; b++) {
                    c->sz2[a * no + b] += sz[a] * sz[b] * w;
                    c->n2[a * no + b] += nt[a] * nt[b] * w;
                }
            c->s2tot += stot * stot * w;
        }
}

static void ed_solve_impl(dmfted_ctx *c, const int32_t *sectors, int nsect_list) {
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "ed_solve: bath not set");
    const dmfted_params &p = c->p;
    c->finite_t = p.lanc_nstates_total != 1;  // ED_SETUP.f90:242-246
    std::vector<int> list;
    if (sectors && nsect_list > 0) {
        for (int i = 0; i < nsect_list; i++) {
            DM_REQUIRE(sectors[i] >= 1 && sectors[i] <= c->nsectors, DMFTED_ERR_ARG,
                       "ed_solve: sector index out of range");
            list.push_back(sectors[i]);
        }
    } else {
        for (int s = 1; s <= c->nsectors; s++)
            if (c->twin_mask[s - 1]) list.push_back(s);
    }
    cudaEvent_t ev[4];
    for (auto &e : ev) DM_CUDA(cudaEventCreate(&e));
    DM_CUDA(cudaEventRecord(ev[0], c->stream));
    // ---- diagonalisation ------------------------------------------------
    const int64_t hv_diag = ed_diag(c, list);
    DM_REQUIRE(!c->states.empty(), DMFTED_ERR_NOTCONV, "ed_solve: no state kept");
    if (c->finite_t) {
        ed_analysis_finite_t(c);
    } else {
        c->egs = c->states.front().e;
        for (auto &st : c->states) c->egs = std::min(c->egs, st.e);
        c->zeta = (double)c->states.size();  // T=0: Z = number of ground states
    }
    DM_CUDA(cudaEventRecord(ev[1], c->stream));
    // ---- observables -------------------------------------------------------
    const std::vector<double> acc = thermal_observables(c, false);
    const int no = c->norb;
    c->obs.assign(5 * no, 0.0);
    for (int a = 0; a < no; a++) {
        const double nu = acc[a], nd = acc[no + a];
        c->obs[a] = nu + nd;           // dens
        c->obs[no + a] = nu;           // dens_up
        c->obs[2 * no + a] = nd;       // dens_dw
        c->obs[3 * no + a] = acc[2 * no + a];  // docc
        c->obs[4 * no + a] = nu - nd;  // magz
    }
    c->hf_terms.assign(acc.begin() + 3 * no, acc.begin() + 3 * no + 4 * no * c->nbath);
    c->hf_hops = false;  // the hop terms are computed when the gradient is asked for
    local_energies(c, acc);
    spin_charge_moments(c, acc);
    c->szr_sigma = c->sigma_now;
    DM_CUDA(cudaEventRecord(ev[2], c->stream));
    // ---- Green's functions ---------------------------------------------------
    const size_t gsz = (size_t)c->nspin * no;
    c->gm.alloc(std::max<size_t>(2 * gsz * p.lmats, 2));
    c->gr.alloc(std::max<size_t>(2 * gsz * p.lreal, 2));
    c->sm.alloc(std::max<size_t>(2 * gsz * p.lmats, 2));
    c->sr.alloc(std::max<size_t>(2 * gsz * p.lreal, 2));
    c->g0m.alloc(std::max<size_t>(2 * gsz * p.lmats, 2));
    c->g0r.alloc(std::max<size_t>(2 * gsz * p.lreal, 2));
    DM_CUDA(cudaMemsetAsync(c->gm.p, 0, c->gm.n * sizeof(double), c->stream));
    DM_CUDA(cudaMemsetAsync(c->gr.p, 0, c->gr.n * sizeof(double), c->stream));
    int64_t hv_gf = 0;
    std::vector<ChainRec> recs;
    for (auto &st : c->states) {
        double weight;
        if (c->finite_t && p.beta * (st.e - c->egs) < 200.0)
            weight = std::exp(-p.beta * (st.e - c->egs)) / c->zeta;
        else if (!c->finite_t)
            weight = 1.0 / c->zeta;
        else
            weight = 0.0;
        if (weight == 0.0) continue;  // pesoBZ = 0: the chains add nothing
        for (int ispin = 0; ispin < c->nspin; ispin++)
            for (int iorb = 0; iorb < no; iorb++)
                for (int ph = 0; ph < 2; ph++) {
                    const bool particle = ph == 0;
                    const int js = particle ? c->getcdgsector[2 * (st.isector - 1) + ispin]
                                            : c->getcsector[2 * (st.isector - 1) + ispin];
                    if (js == 0) continue;
                    ChainRec r;
                    r.psi_off = st.off;
                    r.isector = st.isector;
                    r.jsector = js;
                    r.ispin = ispin;
                    r.iorb = iorb;
                    r.particle = particle ? 1 : 0;
                    r.nlanc = (int)std::min<int64_t>(sector_view(c, js).dim, p.lanc_ngfiter);
                    r.weight = weight;
                    r.e = st.e;
                    recs.push_back(r);
                    hv_gf += r.nlanc;
                }
    }
    batch_chains_gf(c, recs, p.precision);
    gf_sigma(c);
    DM_CUDA(cudaEventRecord(ev[3], c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    // Im Sigma(iw_1), Im Sigma(iw_2) per (spin, orbital): get_szr of the
    // next solve reads them
    c->sigma_now.assign(2 * gsz, 0.0);
    for (size_t so = 0; so < gsz && p.lmats >= 2; so++) {
        double v[4];
        DM_CUDA(cudaMemcpy(v, c->sm.p + 2 * so * p.lmats, sizeof v, cudaMemcpyDeviceToHost));
        c->sigma_now[2 * so] = v[1];
        c->sigma_now[2 * so + 1] = v[3];
    }
    c->sigma_read = false;
    float ms;
    DM_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    c->stats.ms[0] = ms;
    DM_CUDA(cudaEventElapsedTime(&ms, ev[1], ev[2]));
    c->stats.ms[1] = ms;
    DM_CUDA(cudaEventElapsedTime(&ms, ev[2], ev[3]));
    c->stats.ms[2] = ms;
    DM_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[3]));
    c->stats.ms[3] = ms;
    c->stats.hv[0] = hv_diag;
    c->stats.hv[1] = 0;
    c->stats.hv[2] = hv_gf;
    for (auto &e : ev) cudaEventDestroy(e);
    c->solved = true;
}

// (Nspin,Nspin,Norb,Norb,L) Fortran layout from the device [nspin][norb][L]
// complex blocks (normal bath: diagonal in spin and orbital).
static void get_gf(dmfted_ctx *c, const dmfted::DBuf<double> &d, int L, double *out) {
    DM_REQUIRE(c->solved || (c->sigma_read && (&d == &c->sm || &d == &c->sr)), DMFTED_ERR_STATE,
               "no solve has run on this context");
    const int ns = c->nspin, no = c->norb;
    std::vector<double> h(2 * (size_t)ns * no * std::max(L, 1));
    if (L > 0)
        DM_CUDA(cudaMemcpy(h.data(), d.p, 2 * (size_t)ns * no * L * sizeof(double),
                           cudaMemcpyDeviceToHost));
    const size_t tot = (size_t)ns * ns * no * no * L;
    std::fill(out, out + 2 * tot, 0.0);
    for (int is = 0; is < ns; is++)
        for (int a = 0; a < no; a++)
            for (int l = 0; l < L; l++) {
                const size_t fi = is + ns * (is + ns * (a + (size_t)no * (a + (size_t)no * l)));
                const size_t si = ((size_t)(is * no + a) * L + l);
                out[2 * fi] = h[2 * si];
                out[2 * fi + 1] = h[2 * si + 1];
            }
}

}  // namespace dmfted

using namespace dmfted;

#define API_BEGIN try {
#define API_END                                                              \
    }                                                                        \
    catch (const StatusError &e) {                                           \
        return set_error(e.code, e.msg);                                     \
    }                                                                        \
    catch (const std::exception &e) {                                        \
        return set_error(DMFTED_ERR_ARG, e.what());                          \
    }                                                                        \
    g_last_error.clear();                                                    \
    return DMFTED_OK;

extern "C" {

void dmfted_default_params(dmfted_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->norb = 1;
    p->nbath = 6;
    p->nspin = 1;
    p->hfmode = 1;
    p->jhflag = 0;
    p->uloc[0] = 2.0;
    p->ust = p->jh = p->jx = p->jp = 0.0;
    p->xmu = 0.0;
    p->beta = 1000.0;
    p->lmats = 5000;
    p->lreal = 5000;
    p->wini = -5.0;
    p->wfin = 5.0;
    p->eps = 0.01;
    p->lanc_niter = 512;
    p->lanc_ngfiter = 200;
    p->lanc_tolerance = 1e-12;
    p->lanc_dim_threshold = 256;
    p->lanc_nstates_sector = 6;
    p->lanc_nstates_total = 1;
    p->lanc_nstates_step = 2;
    p->gs_threshold = 1e-9;
    p->cutoff = 1e-9;
    p->ed_twin = 0;
    p->lfit = 1000;
    p->cg_weight = 0;
    p->precision = DMFTED_FP64;
    p->lanc_ncheck = 10;
    p->device = 0;
    p->lanc_gf_threshold = 1e-13;
    p->cg_niter = 500;
    p->cg_scheme = DMFTED_CG_WEISS;
    p->cg_ftol = 1e-5;
    p->cg_stop = 0;
    p->cg_eps = 1e-6;
}

const char *dmfted_last_error(void) { return last_error(); }

const char *dmfted_version(void) { return "dmfted-b200 0.1 (sm_100a)"; }

int dmfted_get_bath_dimension(const dmfted_params *p, int32_t *nb) {
    API_BEGIN
    DM_REQUIRE(p && nb, DMFTED_ERR_ARG, "null argument");
    *nb = 2 * p->nspin * p->norb * p->nbath;
    API_END
}

int dmfted_init(const dmfted_params *p, const double *hloc, dmfted_ctx **out) {
    dmfted_ctx *c = nullptr;
    try {
        DM_REQUIRE(p && out, DMFTED_ERR_ARG, "null argument");
        *out = nullptr;
        DM_REQUIRE(p->norb >= 1 && p->norb <= kMaxNorb, DMFTED_ERR_UNSUPPORTED,
                   "ED ERROR: Norb > 3 is currently not supported");
        DM_REQUIRE(p->nspin == 1 || p->nspin == 2, DMFTED_ERR_UNSUPPORTED,
                   "ED ERROR: Nspin > 2 is currently not supported");
        DM_REQUIRE(p->nbath >= 0, DMFTED_ERR_ARG, "Nbath < 0");
        const int ns = (p->nbath + 1) * p->norb;
        DM_REQUIRE(ns <= kMaxNs, DMFTED_ERR_UNSUPPORTED, "Ns > 20 is outside this solver");
        DM_REQUIRE(p->lmats >= 0 && p->lreal >= 0, DMFTED_ERR_ARG, "negative frequency count");
        DM_REQUIRE(p->lanc_ngfiter >= 1 && p->lanc_ngfiter < kLzMax, DMFTED_ERR_ARG,
                   "lanc_ngfiter out of range");
        DM_REQUIRE(p->lanc_niter >= 1, DMFTED_ERR_ARG, "lanc_niter < 1");
        DM_REQUIRE(p->precision == DMFTED_FP64 || p->precision == DMFTED_MIXED, DMFTED_ERR_ARG,
                   "unknown precision mode");
        c = new dmfted_ctx();
        c->p = *p;
        if (c->p.lanc_ncheck <= 0) c->p.lanc_ncheck = 10;
        if (c->p.lanc_gf_threshold <= 0) c->p.lanc_gf_threshold = 1e-13;
        c->norb = p->norb;
        c->nbath = p->nbath;
        c->jterms = p->jhflag && p->norb > 1 && (p->jx != 0.0 || p->jp != 0.0);
        c->nspin = p->nspin;
        c->ns = ns;
        c->device = p->device;
        if (const char *e = getenv("DMFTED_HXV_NC")) c->tune_nc = atoi(e);
        if (const char *e = getenv("DMFTED_HXV_KERNEL")) c->tune_hxv = atoi(e);
        if (const char *e = getenv("DMFTED_HXV_OCC")) c->tune_occ = atoi(e);
        if (const char *e = getenv("DMFTED_ELL_GROUP")) c->tune_ell_group = std::max(1, std::min(32, atoi(e)));
        if (const char *e = getenv("DMFTED_MIXED_TOL32")) c->mixed_tol32 = atof(e);
        if (const char *e = getenv("DMFTED_GS_BASIS_MB")) c->gs_basis_budget = atoll(e) << 20;
        if (const char *e = getenv("DMFTED_AUTOTUNE")) c->autotune = atoi(e) != 0;
        if (const char *e = getenv("DMFTED_CHAIN_LANES")) c->chain_lanes = atoi(e);
        if (const char *e = getenv("DMFTED_GF_HEAD64")) c->gf_head64 = std::max(0, atoi(e));
        if (const char *e = getenv("DMFTED_BATCH_MAX_DIM")) c->batch_max_dim = atoll(e);
        if (const char *e = getenv("DMFTED_BATCH_BUDGET_MB")) c->batch_budget = atoll(e) << 20;
        if (const char *e = getenv("DMFTED_FT_EIGS_FP32")) c->ft_eigs_fp32 = atoi(e) != 0;
        if (const char *e = getenv("DMFTED_BATCH_CHAINS_FP32")) c->batch_chains_fp32 = atoi(e) != 0;
        if (const char *e = getenv("DMFTED_BATCH_CLUSTER_MIN"))
            c->batch_cluster_min = std::max<int64_t>(1, atoll(e));
        DM_CUDA(cudaSetDevice(c->device));
        DM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        const size_t nh = 2 * (size_t)c->nspin * c->nspin * c->norb * c->norb;
        c->hloc.assign(nh, 0.0);
        if (hloc) {
            check_hloc(c, hloc);
            std::copy(hloc, hloc + nh, c->hloc.begin());
        }
        // ED_SETUP.f90:242-260: T=0 iff lanc_nstates_total==1; at finite T
        // both state counts are made even (doublets are kept together)
        if (c->p.lanc_nstates_total != 1) {
            if (c->p.lanc_nstates_sector % 2 != 0) c->p.lanc_nstates_sector++;
            if (c->p.lanc_nstates_total % 2 != 0) c->p.lanc_nstates_total++;
        }
        c->nstates_total = c->p.lanc_nstates_total;
        setup_pointers_normal(c);
        fock_init(c);
        c->red_partials.alloc((size_t)2 * 64 * kMaxRedBlocks);
        c->red_counter.alloc(8);
        DM_CUDA(cudaMemsetAsync(c->red_counter.p, 0, 8 * sizeof(unsigned), c->stream));
        if (c->chain_lanes >= 2) {
            DM_CUDA(cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
            DM_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
            DM_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
            c->red_partials2.alloc((size_t)2 * 64 * kMaxRedBlocks);
            c->red_counter2.alloc(8);
            DM_CUDA(cudaMemsetAsync(c->red_counter2.p, 0, 8 * sizeof(unsigned), c->stream));
        }
        c->red_out.alloc(16);
        c->lz_d.alloc((size_t)kLzSlots * kLzStride);
        c->lz_s.alloc((size_t)kLzSlots * 8);
        DM_CUDA(cudaMemsetAsync(c->lz_s.p, 0, kLzSlots * 8 * sizeof(int), c->stream));
        c->coefb.alloc(kLzMax + 8);
        // frequency grids: wm = pi/beta (2n-1) (ED_GREENS_FUNCTIONS.f90:114),
        // wr = linspace(wini, wfin, Lreal)
        std::vector<double> wm(std::max(p->lmats, 1)), wr(std::max(p->lreal, 1));
        for (int i = 0; i < p->lmats; i++) wm[i] = M_PI / p->beta * (2.0 * (i + 1) - 1.0);
        for (int i = 0; i < p->lreal; i++)
            wr[i] = p->lreal > 1 ? p->wini + (p->wfin - p->wini) * i / (double)(p->lreal - 1)
                                 : p->wini;
        c->d_wm.alloc(wm.size());
        c->d_wr.alloc(wr.size());
        DM_CUDA(cudaMemcpyAsync(c->d_wm.p, wm.data(), wm.size() * 8, cudaMemcpyHostToDevice,
                                c->stream));
        DM_CUDA(cudaMemcpyAsync(c->d_wr.p, wr.data(), wr.size() * 8, cudaMemcpyHostToDevice,
                                c->stream));
        c->bath_e.assign((size_t)c->nspin * c->norb * c->nbath, 0.0);
        c->bath_v.assign((size_t)c->nspin * c->norb * c->nbath, 0.0);
        upload_model(c);
        DM_CUDA(cudaStreamSynchronize(c->stream));
        *out = c;
    } catch (const StatusError &e) {
        delete c;
        return set_error(e.code, e.msg);
    }
    g_last_error.clear();
    return DMFTED_OK;
}

int dmfted_free(dmfted_ctx *c) {
    API_BEGIN
    if (!c) return DMFTED_OK;
    cudaSetDevice(c->device);
    // a device error still pending from this context's last work is reported
    // here rather than left for the next context to trip over
    cudaError_t pending = c->stream ? cudaStreamSynchronize(c->stream) : cudaSuccess;
    if (c->stream2 && pending == cudaSuccess) pending = cudaStreamSynchronize(c->stream2);
    cudaStream_t st = c->stream, st2 = c->stream2;
    for (cudaEvent_t e : c->hv_ev_free) cudaEventDestroy(e);
    for (auto &pr : c->hv_ev) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    delete c;
    if (st) cudaStreamDestroy(st);
    if (st2) cudaStreamDestroy(st2);
    DM_REQUIRE(pending == cudaSuccess, DMFTED_ERR_CUDA,
               std::string("device error pending at free: ") + cudaGetErrorString(pending));
    API_END
}

int dmfted_set_hloc(dmfted_ctx *c, const double *hloc) {
    API_BEGIN
    DM_REQUIRE(c && hloc, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    check_hloc(c, hloc);
    std::copy(hloc, hloc + c->hloc.size(), c->hloc.begin());
    upload_model(c);
    if (c->bath_set) fock_set_couplings(c);
    API_END
}

int dmfted_set_bath(dmfted_ctx *c, const double *bath, int32_t nb) {
    API_BEGIN
    DM_REQUIRE(c && (bath || nb == 0), DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    const int32_t want = 2 * c->nspin * c->norb * c->nbath;
    DM_REQUIRE(nb == want, DMFTED_ERR_ARG, "set_dmft_bath error: wrong bath dimensions");
    for (int i = 0; i < nb; i++)
        DM_REQUIRE(std::isfinite(bath[i]), DMFTED_ERR_ARG, "bath has a non-finite entry");
    // set_dmft_bath, ED_BATH/dmft_aux.f90:493-512: io = k + (iorb-1)*Nbath + (ispin-1)*Nbath*Norb
    const int half = nb / 2;
    std::copy(bath, bath + half, c->bath_e.begin());
    std::copy(bath + half, bath + nb, c->bath_v.begin());
    upload_model(c);
    fock_set_couplings(c);
    c->bath_set = true;
    API_END
}

int dmfted_sector_tables(dmfted_ctx *c, int32_t *nsectors, int32_t *getsector, int32_t *getnup,
                         int32_t *getndw, int32_t *getdim, int32_t *getdimup, int32_t *getdimdw,
                         int32_t *getcsector, int32_t *getcdgsector, int32_t *getbathstride,
                         int32_t *impindex) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    auto cp = [](const std::vector<int32_t> &v, int32_t *o) {
        if (o) std::copy(v.begin(), v.end(), o);
    };
    if (nsectors) *nsectors = c->nsectors;
    cp(c->getsector, getsector);
    cp(c->getnup, getnup);
    cp(c->getndw, getndw);
    cp(c->getdim, getdim);
    cp(c->getdimup, getdimup);
    cp(c->getdimdw, getdimdw);
    cp(c->getcsector, getcsector);
    cp(c->getcdgsector, getcdgsector);
    cp(c->getbathstride, getbathstride);
    cp(c->impindex, impindex);
    API_END
}

int dmfted_build_sector(dmfted_ctx *c, int32_t isector, int32_t *map, int64_t dim) {
    API_BEGIN
    DM_REQUIRE(c && map, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    DM_REQUIRE(c->ns <= 15, DMFTED_ERR_UNSUPPORTED, "the combined map needs 2*Ns <= 31 bits");
    SectorView s = sector_view(c, isector);
    DM_REQUIRE(dim == s.dim, DMFTED_ERR_ARG, "build_sector: dim != getdim(isector)");
    DBuf<int32_t> d;
    d.alloc(std::max<int64_t>(s.dim, 1));
    fock_build_map(c, isector, d.p);
    DM_CUDA(cudaMemcpyAsync(map, d.p, s.dim * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    API_END
}

int dmfted_setup_hv_sector(dmfted_ctx *c, int32_t isector) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    sector_view(c, isector);
    c->cur_sector = isector;
    API_END
}

int dmfted_delete_hv_sector(dmfted_ctx *c) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    c->cur_sector = 0;
    API_END
}

int dmfted_hxv_c128(dmfted_ctx *c, int32_t nloc, const double *v, double *hv) {
    API_BEGIN
    DM_REQUIRE(c && v && hv, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->cur_sector != 0, DMFTED_ERR_STATE, "directMatVec_cc ERROR: Hsector NOT set");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "H*v: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    SectorView s = sector_view(c, c->cur_sector);
    DM_REQUIRE((int64_t)nloc == s.dim, DMFTED_ERR_ARG, "directMatVec_cc ERROR: Nloc != dim(isector)");
    const int64_t n = s.dim;
    c->wv64.alloc(6 * n);
    double *z = c->wv64.p, *x = z + 2 * n, *y = x + 2 * n;
    DM_CUDA(cudaMemcpyAsync(z, v, 2 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_interleave_split<<<ew(c, n), 256, 0, c->stream>>>(z, x, x + n, n);
    DM_CHECK_LAUNCH();
    hxv_f64(c, s, x, y, 2);
    k_interleave_join<<<ew(c, n), 256, 0, c->stream>>>(y, y + n, z, n);
    DM_CHECK_LAUNCH();
    c->launches += 2;
    DM_CUDA(cudaMemcpyAsync(hv, z, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    API_END
}

int dmfted_hxv_device_f64(dmfted_ctx *c, const double *d_v, double *d_hv, int32_t nvec) {
    API_BEGIN
    DM_REQUIRE(c && d_v && d_hv && nvec >= 1 && nvec <= 65535, DMFTED_ERR_ARG, "bad argument");
    DM_REQUIRE(c->cur_sector != 0, DMFTED_ERR_STATE, "directMatVec_cc ERROR: Hsector NOT set");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "H*v: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    hxv_f64(c, sector_view(c, c->cur_sector), d_v, d_hv, nvec);
    API_END
}

int dmfted_hxv_device_f32(dmfted_ctx *c, const float *d_v, float *d_hv, int32_t nvec) {
    API_BEGIN
    DM_REQUIRE(c && d_v && d_hv && nvec >= 1 && nvec <= 65535, DMFTED_ERR_ARG, "bad argument");
    DM_REQUIRE(c->cur_sector != 0, DMFTED_ERR_STATE, "directMatVec_cc ERROR: Hsector NOT set");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "H*v: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    hxv_f32(c, sector_view(c, c->cur_sector), d_v, d_hv, nvec);
    API_END
}

int dmfted_lanczos_gs(dmfted_ctx *c, int32_t isector, double *e0, double *psi, int32_t *niter) {
    API_BEGIN
    DM_REQUIRE(c && e0, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "lanczos_gs: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    SectorView s = sector_view(c, isector);
    c->s64a.alloc(s.dim);
    const int nit = (int)std::min<int64_t>(s.dim, c->p.lanc_niter);
    LanczosResult r = lanczos_gs(c, s, c->s64a.p, nullptr, c->p.precision, c->p.lanc_tolerance, nit);
    *e0 = r.e0;
    if (niter) *niter = r.steps;
    if (psi) real_to_host_c128(c, c->s64a.p, s.dim, psi);
    API_END
}

int dmfted_gs_lanczos(dmfted_ctx *c, int32_t isector, int32_t neigen, int32_t nitermax,
                      double tol, double *evals, double *evecs, int32_t *nfound) {
    API_BEGIN
    DM_REQUIRE(c && evals, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "sp_eigh: bath not set");
    DM_REQUIRE(isector >= 1 && isector <= c->nsectors, DMFTED_ERR_ARG, "sector out of range");
    DM_REQUIRE(neigen >= 1, DMFTED_ERR_ARG, "sp_eigh: Neigen < 1");
    const int64_t dim = (int64_t)c->getdimup[isector - 1] * c->getdimdw[isector - 1];
    const int ne = (int)std::min<int64_t>(neigen, dim);
    // the call's own iteration limit and tolerance, restored on every exit
    struct Restore {
        dmfted_params &p;
        int32_t niter;
        double tol;
        ~Restore() {
            p.lanc_niter = niter;
            p.lanc_tolerance = tol;
        }
    } restore{c->p, c->p.lanc_niter, c->p.lanc_tolerance};
    if (nitermax > 0) c->p.lanc_niter = nitermax;
    if (tol > 0.0) c->p.lanc_tolerance = tol;
    if (evecs) c->gsvec.alloc((size_t)ne * dim);
    int64_t steps = 0;
    const int m = sector_eigenpairs(c, isector, ne, evals, evecs ? c->gsvec.p : nullptr, &steps);
    if (evecs)
        for (int k = 0; k < m; k++)
            real_to_host_c128(c, c->gsvec.p + (int64_t)k * dim, dim, evecs + 2 * (int64_t)k * dim);
    if (nfound) *nfound = m;
    API_END
}

int dmfted_add_to_lanczos_gf(dmfted_ctx *c, double vnorm2, double ei, double egs, double zeta,
                             int32_t nlanc, const double *alanc, const double *blanc,
                             int32_t isign, double *gmats, double *greal) {
    API_BEGIN
    DM_REQUIRE(c && alanc && blanc && gmats, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(zeta > 0.0, DMFTED_ERR_ARG, "add_to_lanczos_gf: zeta <= 0");
    DM_REQUIRE(isign == 1 || isign == -1, DMFTED_ERR_ARG, "add_to_lanczos_gf: isign not +-1");
    DM_CUDA(cudaSetDevice(c->device));
    // pesoBZ of build_gf_normal.f90:457-464
    const bool finite_t = c->p.lanc_nstates_total != 1;
    double weight;
    if (finite_t && c->p.beta * (ei - egs) < 200.0) weight = std::exp(-c->p.beta * (ei - egs)) / zeta;
    else if (!finite_t) weight = 1.0 / zeta;
    else weight = 0.0;
    gf_add_chain(c, nlanc, alanc, blanc, weight, vnorm2, ei, isign, gmats, greal);
    API_END
}

int dmfted_lanc_tridiag(dmfted_ctx *c, int32_t isector, const double *vvinit, int32_t nlanc,
                        double *alanc, double *blanc, int32_t *nused) {
    API_BEGIN
    DM_REQUIRE(c && vvinit && alanc && blanc, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(nlanc >= 1 && nlanc < kLzMax, DMFTED_ERR_ARG, "nlanc out of range");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "lanc_tridiag: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    SectorView s = sector_view(c, isector);
    const int64_t n = s.dim;
    // complex start vector -> stacked (re, im) halves: the recurrence of a real
    // symmetric H on a complex vector is the real recurrence on the stack.
    c->wv64.alloc(2 * n);
    c->s64b.alloc(2 * n);
    DM_CUDA(cudaMemcpyAsync(c->wv64.p, vvinit, 2 * n * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    k_interleave_split<<<ew(c, n), 256, 0, c->stream>>>(c->wv64.p, c->s64b.p, c->s64b.p + n, n);
    DM_CHECK_LAUNCH();
    c->launches++;
    LanczosScalars lz = lz_slot(c, 2, nlanc);
    lanczos_chain(c, s, c->s64b.p, c->p.precision, lz, 2);
    std::vector<double> b(nlanc + 1);
    int st[8];
    DM_CUDA(cudaMemcpyAsync(alanc, lz.alpha, nlanc * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaMemcpyAsync(b.data(), lz.beta, (nlanc + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaMemcpyAsync(st, lz.status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    const int used = st[1];
    // steps never taken keep a = b = 0, as the zero-initialised arrays of the
    // reference's early exit do (.repo/PLAIN_LANCZOS.f90:164-179)
    for (int k = used; k < nlanc; k++) alanc[k] = 0.0;
    blanc[0] = 0.0;
    for (int k = 1; k < nlanc; k++) blanc[k] = k <= used ? b[k] : 0.0;
    if (nused) *nused = used;
    API_END
}

int dmfted_ed_solve(dmfted_ctx *c, const double *bath, int32_t nb, const int32_t *sectors,
                    int32_t nsectors) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    DM_CUDA(cudaSetDevice(c->device));
    if (bath) {
        const int rc = dmfted_set_bath(c, bath, nb);
        if (rc != DMFTED_OK) return rc;
    }
    ed_solve_impl(c, sectors, nsectors);
    API_END
}

int dmfted_get_gimp_matsubara(dmfted_ctx *c, double *g) {
    API_BEGIN
    DM_REQUIRE(c && g, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->gm, c->p.lmats, g);
    API_END
}
int dmfted_get_gimp_real(dmfted_ctx *c, double *g) {
    API_BEGIN
    DM_REQUIRE(c && g, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->gr, c->p.lreal, g);
    API_END
}
int dmfted_get_sigma_matsubara(dmfted_ctx *c, double *s) {
    API_BEGIN
    DM_REQUIRE(c && s, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->sm, c->p.lmats, s);
    API_END
}
int dmfted_get_sigma_real(dmfted_ctx *c, double *s) {
    API_BEGIN
    DM_REQUIRE(c && s, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->sr, c->p.lreal, s);
    API_END
}
int dmfted_get_g0imp_matsubara(dmfted_ctx *c, double *g) {
    API_BEGIN
    DM_REQUIRE(c && g, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->g0m, c->p.lmats, g);
    API_END
}
int dmfted_get_g0imp_real(dmfted_ctx *c, double *g) {
    API_BEGIN
    DM_REQUIRE(c && g, DMFTED_ERR_ARG, "null argument");
    get_gf(c, c->g0r, c->p.lreal, g);
    API_END
}

int dmfted_get_observables(dmfted_ctx *c, double *dens, double *dens_up, double *dens_dw,
                           double *docc, double *magz) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    const int no = c->norb;
    double *outs[5] = {dens, dens_up, dens_dw, docc, magz};
    for (int k = 0; k < 5; k++)
        if (outs[k]) std::copy(c->obs.begin() + k * no, c->obs.begin() + (k + 1) * no, outs[k]);
    API_END
}

int dmfted_get_neigen(dmfted_ctx *c, int32_t *neigen, int32_t nsectors, int32_t *nstates_total) {
    API_BEGIN
    DM_REQUIRE(c && neigen && nstates_total, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(nsectors == c->nsectors, DMFTED_ERR_ARG, "get_neigen: wrong sector count");
    for (int i = 0; i < nsectors; i++) neigen[i] = c->neigen_sector[i];
    *nstates_total = c->nstates_total;
    API_END
}

int dmfted_set_neigen(dmfted_ctx *c, const int32_t *neigen, int32_t nsectors,
                      int32_t nstates_total) {
    API_BEGIN
    DM_REQUIRE(c && neigen, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(nsectors == c->nsectors, DMFTED_ERR_ARG, "set_neigen: wrong sector count");
    DM_REQUIRE(nstates_total >= 1, DMFTED_ERR_ARG, "set_neigen: lanc_nstates_total < 1");
    for (int i = 0; i < nsectors; i++)
        DM_REQUIRE(neigen[i] >= 1, DMFTED_ERR_ARG, "set_neigen: neigen_sector entry < 1");
    for (int i = 0; i < nsectors; i++) c->neigen_sector[i] = neigen[i];
    c->nstates_total = nstates_total;
    API_END
}

int dmfted_get_eigenspace(dmfted_ctx *c, int32_t cap, double *energies, int32_t *sectors,
                          int32_t *nstates, double *zeta) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    const int n = (int)c->states.size();
    if (nstates) *nstates = n;
    if (zeta) *zeta = c->zeta;
    for (int i = 0; i < std::min(n, cap); i++) {
        if (energies) energies[i] = c->states[i].e;
        if (sectors) sectors[i] = c->states[i].isector;
    }
    API_END
}

int dmfted_get_eimp(dmfted_ctx *c, double *eimp) {
    API_BEGIN
    DM_REQUIRE(c && eimp, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    for (int k = 0; k < 4; k++) eimp[k] = c->eloc[k];
    API_END
}

int dmfted_get_doubles(dmfted_ctx *c, double *doubles) {
    API_BEGIN
    DM_REQUIRE(c && doubles, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    for (int k = 0; k < 4; k++) doubles[k] = c->eloc[4 + k];
    API_END
}

int dmfted_get_egs(dmfted_ctx *c, double *egs) {
    API_BEGIN
    DM_REQUIRE(c && egs, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    *egs = c->egs;
    API_END
}

int dmfted_hf_gradient(dmfted_ctx *c, double *grad, int32_t nb) {
    API_BEGIN
    DM_REQUIRE(c && grad, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    const int no = c->norb, nbth = c->nbath, ns = c->nspin;
    DM_REQUIRE(nb == 2 * ns * no * nbth, DMFTED_ERR_ARG, "hf_gradient: wrong bath dimensions");
    const int pv = no * nbth;
    if (!c->hf_hops) {
        DM_CUDA(cudaSetDevice(c->device));
        const std::vector<double> acc = thermal_observables(c, true);
        c->hf_terms.assign(acc.begin() + 3 * no, acc.begin() + 3 * no + 4 * no * c->nbath);
        c->hf_hops = true;
    }
    const double *nk = c->hf_terms.data();           // [2][norb][nbath]
    const double *hop = c->hf_terms.data() + 2 * pv;  // [2][norb][nbath]
    for (int is = 0; is < ns; is++)
        for (int a = 0; a < no; a++)
            for (int k = 0; k < nbth; k++) {
                const int io = k + a * nbth + is * nbth * no;
                const int p = a * nbth + k;
                double de, dv;
                if (ns == 1) {
                    de = nk[p] + nk[pv + p];
                    dv = hop[p] + hop[pv + p];
                } else {
                    de = nk[is * pv + p];
                    dv = hop[is * pv + p];
                }
                grad[io] = de;
                grad[ns * no * nbth + io] = dv;
            }
    API_END
}

int dmfted_chi2_delta_batch_device(dmfted_ctx *c, int32_t nbatch, int32_t nbath, int32_t L,
                                   const double *d_a, const double *d_xdelta, const double *d_g,
                                   const double *d_w, double *d_chi2, double *d_grad) {
    API_BEGIN
    DM_REQUIRE(c && d_a && d_xdelta && d_g && d_w && d_chi2, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    chi2_batch_device(c, nbatch, nbath, L, d_a, d_xdelta, d_g, d_w, d_chi2, d_grad);
    API_END
}

int dmfted_chi2_delta_batch(dmfted_ctx *c, int32_t nbatch, int32_t nbath, int32_t L,
                            const double *a, const double *xdelta, const double *g,
                            const double *w, double *chi2, double *grad) {
    API_BEGIN
    DM_REQUIRE(c && a && xdelta && g && w && chi2, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(nbatch > 0 && nbath > 0 && L > 0, DMFTED_ERR_ARG, "chi2: empty batch or grid");
    DM_CUDA(cudaSetDevice(c->device));
    const size_t na = (size_t)nbatch * 2 * nbath;
    DBuf<double> buf;
    buf.alloc(na + L + 2 * (size_t)L + L + nbatch + na);
    double *da = buf.p, *dx = da + na, *dg = dx + L, *dw = dg + 2 * (size_t)L, *dc = dw + L,
           *dgr = dc + nbatch;
    DM_CUDA(cudaMemcpyAsync(da, a, na * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dx, xdelta, (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dg, g, 2 * (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dw, w, (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    chi2_batch_device(c, nbatch, nbath, L, da, dx, dg, dw, dc, grad ? dgr : nullptr);
    DM_CUDA(cudaMemcpyAsync(chi2, dc, nbatch * 8, cudaMemcpyDeviceToHost, c->stream));
    if (grad) DM_CUDA(cudaMemcpyAsync(grad, dgr, na * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    API_END
}

// ---- the self-consistency around the solve (fit.cu) -------------------------

// Wdelta of chi2_fitgf_normal_normal (ED_CHI2FIT/fitgf_normal_normal.f90:44-53):
// cg_weight 0 -> Ldelta, 1 -> 1, 2 -> n, 3 -> Xdelta(n).
static std::vector<double> fit_weights(int cg_weight, const std::vector<double> &xd) {
    const int L = (int)xd.size();
    std::vector<double> w(L);
    for (int n = 0; n < L; n++) {
        switch (cg_weight) {
            case 1: w[n] = 1.0; break;
            case 2: w[n] = (double)(n + 1); break;
            case 3: w[n] = xd[n]; break;
            default: w[n] = (double)L; break;
        }
    }
    return w;
}

static void check_cg_params(const dmfted_ctx *c, int scheme) {
    DM_REQUIRE(scheme == DMFTED_CG_DELTA || scheme == DMFTED_CG_WEISS, DMFTED_ERR_ARG,
               "chi2_fitgf_normal_normal error: cg_scheme != [weiss,delta]");
    DM_REQUIRE(c->p.cg_niter >= 1, DMFTED_ERR_ARG, "cg fit: cg_niter < 1");
    DM_REQUIRE(c->p.cg_stop >= 0 && c->p.cg_stop <= 2, DMFTED_ERR_ARG, "cg fit: cg_stop not in 0..2");
}

int dmfted_chi2_fitgf(dmfted_ctx *c, const double *fg, int32_t ispin, double *bath, int32_t nb,
                      int32_t *iter, double *chi2) {
    API_BEGIN
    DM_REQUIRE(c && fg && bath, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(ispin >= 1 && ispin <= c->nspin, DMFTED_ERR_ARG, "chi2_fitgf: ispin out of range");
    DM_REQUIRE(nb == 2 * c->nspin * c->norb * c->nbath, DMFTED_ERR_ARG,
               "chi2_fitgf_normal_normal error: wrong bath dimensions");
    DM_REQUIRE(c->nbath >= 1, DMFTED_ERR_ARG, "chi2_fitgf: no bath levels to fit");
    check_cg_params(c, c->p.cg_scheme);
    DM_CUDA(cudaSetDevice(c->device));
    const int ns = c->nspin, no = c->norb, nbth = c->nbath, is = ispin - 1;
    const int L = std::min(c->p.lfit, c->p.lmats);
    DM_REQUIRE(L >= 1, DMFTED_ERR_ARG, "chi2_fitgf: Lfit < 1");
    std::vector<double> xd(L);
    for (int n = 0; n < L; n++) xd[n] = M_PI / c->p.beta * (2.0 * (n + 1) - 1.0);
    const std::vector<double> w = fit_weights(c->p.cg_weight, xd);
    // one fit per orbital: target fg(is,is,a,a,1:L), parameters of (is, a)
    std::vector<double> a((size_t)no * 2 * nbth), g((size_t)no * 2 * L), zc(no);
    const int64_t half = (int64_t)ns * no * nbth;
    for (int o = 0; o < no; o++) {
        for (int k = 0; k < nbth; k++) {
            const int64_t io = k + (int64_t)o * nbth + (int64_t)is * nbth * no;
            a[(size_t)o * 2 * nbth + k] = bath[io];
            a[(size_t)o * 2 * nbth + nbth + k] = bath[half + io];
        }
        for (int n = 0; n < L; n++) {
            const int64_t idx = is + ns * (is + ns * (o + (int64_t)no * (o + (int64_t)no * n)));
            g[((size_t)o * L + n) * 2] = fg[2 * idx];
            g[((size_t)o * L + n) * 2 + 1] = fg[2 * idx + 1];
        }
        const int64_t h = is + ns * (is + ns * (o + (int64_t)no * o));
        zc[o] = c->p.xmu - c->hloc[2 * h];
    }
    DBuf<double> buf;
    const size_t na = a.size();
    buf.alloc(na + g.size() + 2 * (size_t)L + no + no);
    double *da = buf.p, *dg = da + na, *dx = dg + g.size(), *dw = dx + L, *dz = dw + L,
           *dc = dz + no;
    DBuf<int> ibuf;
    ibuf.alloc(2 * (size_t)no);
    DM_CUDA(cudaMemcpyAsync(da, a.data(), na * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dg, g.data(), g.size() * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dx, xd.data(), (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dw, w.data(), (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dz, zc.data(), (size_t)no * 8, cudaMemcpyHostToDevice, c->stream));
    cg_fit_device(c, no, nbth, L, da, dx, dg, no, dw, dz, 0.0, c->p.cg_scheme == DMFTED_CG_WEISS,
                  c->p.cg_niter, c->p.cg_stop, c->p.cg_ftol, c->p.cg_eps, ibuf.p, dc, ibuf.p + no);
    std::vector<double> c2(no);
    std::vector<int> it(2 * (size_t)no);
    DM_CUDA(cudaMemcpyAsync(a.data(), da, na * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaMemcpyAsync(c2.data(), dc, (size_t)no * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaMemcpyAsync(it.data(), ibuf.p, 2 * (size_t)no * sizeof(int), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    for (int o = 0; o < no; o++) {
        for (int k = 0; k < nbth; k++) {
            const int64_t io = k + (int64_t)o * nbth + (int64_t)is * nbth * no;
            bath[io] = a[(size_t)o * 2 * nbth + k];
            bath[half + io] = a[(size_t)o * 2 * nbth + nbth + k];
        }
        if (iter) iter[o] = it[o];
        if (chi2) chi2[o] = c2[o];
    }
    API_END
}

int dmfted_cg_fit_batch_device(dmfted_ctx *c, int32_t nbatch, int32_t nbath, int32_t L,
                               double *d_a, const double *d_xdelta, const double *d_g,
                               const double *d_w, int32_t scheme, double zc, int32_t *d_iter,
                               double *d_chi2, int32_t *d_status) {
    API_BEGIN
    DM_REQUIRE(c && d_a && d_xdelta && d_g && d_w && d_iter && d_chi2 && d_status, DMFTED_ERR_ARG,
               "null argument");
    check_cg_params(c, scheme);
    DM_CUDA(cudaSetDevice(c->device));
    cg_fit_device(c, nbatch, nbath, L, d_a, d_xdelta, d_g, 1, d_w, nullptr, zc,
                  scheme == DMFTED_CG_WEISS, c->p.cg_niter, c->p.cg_stop, c->p.cg_ftol,
                  c->p.cg_eps, d_iter, d_chi2, d_status);
    DM_CUDA(cudaStreamSynchronize(c->stream));
    API_END
}

int dmfted_cg_fit_batch(dmfted_ctx *c, int32_t nbatch, int32_t nbath, int32_t L, double *a,
                        const double *xdelta, const double *g, const double *w, int32_t scheme,
                        double zc, int32_t *iter, double *chi2) {
    API_BEGIN
    DM_REQUIRE(c && a && xdelta && g && w, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(nbatch > 0 && nbath > 0 && L > 0, DMFTED_ERR_ARG, "cg fit: empty batch or grid");
    check_cg_params(c, scheme);
    DM_CUDA(cudaSetDevice(c->device));
    const size_t na = (size_t)nbatch * 2 * nbath;
    DBuf<double> buf;
    buf.alloc(na + 4 * (size_t)L + nbatch);
    double *da = buf.p, *dx = da + na, *dg = dx + L, *dw = dg + 2 * (size_t)L, *dc = dw + L;
    DBuf<int> ibuf;
    ibuf.alloc(2 * (size_t)nbatch);
    DM_CUDA(cudaMemcpyAsync(da, a, na * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dx, xdelta, (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dg, g, 2 * (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dw, w, (size_t)L * 8, cudaMemcpyHostToDevice, c->stream));
    cg_fit_device(c, nbatch, nbath, L, da, dx, dg, 1, dw, nullptr, zc, scheme == DMFTED_CG_WEISS,
                  c->p.cg_niter, c->p.cg_stop, c->p.cg_ftol, c->p.cg_eps, ibuf.p, dc,
                  ibuf.p + nbatch);
    std::vector<int> it(2 * (size_t)nbatch);
    DM_CUDA(cudaMemcpyAsync(a, da, na * 8, cudaMemcpyDeviceToHost, c->stream));
    if (chi2) DM_CUDA(cudaMemcpyAsync(chi2, dc, (size_t)nbatch * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaMemcpyAsync(it.data(), ibuf.p, it.size() * sizeof(int), cudaMemcpyDeviceToHost,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    if (iter) std::copy(it.begin(), it.begin() + nbatch, iter);
    API_END
}

static void gloc_diag_host(dmfted_ctx *c, int32_t le, const double *he, const double *wt,
                           const double *sigma, double *gloc, bool real_axis) {
    DM_REQUIRE(c && he && wt && sigma && gloc, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(le >= 1, DMFTED_ERR_ARG, "gloc: empty density-of-states grid");
    DM_CUDA(cudaSetDevice(c->device));
    const int L = real_axis ? c->p.lreal : c->p.lmats, no = c->norb, ns = c->nspin;
    DM_REQUIRE(L >= 1, DMFTED_ERR_ARG, "gloc: empty frequency grid");
    DM_REQUIRE(!real_axis || c->p.eps > 0.0, DMFTED_ERR_ARG, "gloc: real axis needs eps > 0");
    const size_t ng = (size_t)ns * ns * no * no * L * 2;
    DBuf<double> buf;
    buf.alloc((size_t)no * le + le + 2 * ng);
    double *dh = buf.p, *dwt = dh + (size_t)no * le, *ds = dwt + le, *dgl = ds + ng;
    DM_CUDA(cudaMemcpyAsync(dh, he, (size_t)no * le * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(dwt, wt, (size_t)le * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(ds, sigma, ng * 8, cudaMemcpyHostToDevice, c->stream));
    gloc_diag_device(c, L, le, dh, dwt, real_axis ? c->d_wr.p : c->d_wm.p,
                     real_axis ? c->p.eps : 0.0, ds, dgl);
    DM_CUDA(cudaMemcpyAsync(gloc, dgl, ng * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
}

int dmfted_gloc_matsubara_diag(dmfted_ctx *c, int32_t le, const double *he, const double *wt,
                               const double *sigma, double *gloc) {
    API_BEGIN
    gloc_diag_host(c, le, he, wt, sigma, gloc, false);
    API_END
}

int dmfted_gloc_realaxis_diag(dmfted_ctx *c, int32_t le, const double *he, const double *wt,
                              const double *sigma, double *gloc) {
    API_BEGIN
    gloc_diag_host(c, le, he, wt, sigma, gloc, true);
    API_END
}

int dmfted_get_weiss(dmfted_ctx *c, const double *gloc, const double *sigma, int32_t scheme,
                     double *out) {
    API_BEGIN
    DM_REQUIRE(c && gloc && sigma && out, DMFTED_ERR_ARG, "null argument");
    DM_REQUIRE(scheme == DMFTED_CG_DELTA || scheme == DMFTED_CG_WEISS, DMFTED_ERR_ARG,
               "get_weiss: scheme != [weiss,delta]");
    DM_CUDA(cudaSetDevice(c->device));
    const int L = c->p.lmats, no = c->norb, ns = c->nspin;
    const size_t ng = (size_t)ns * ns * no * no * L * 2;
    DBuf<double> buf;
    buf.alloc(3 * ng);
    double *dgl = buf.p, *ds = dgl + ng, *dout = ds + ng;
    DM_CUDA(cudaMemcpyAsync(dgl, gloc, ng * 8, cudaMemcpyHostToDevice, c->stream));
    DM_CUDA(cudaMemcpyAsync(ds, sigma, ng * 8, cudaMemcpyHostToDevice, c->stream));
    weiss_diag_device(c, L, scheme, c->d_hloc_aa.p, c->d_wm.p, dgl, ds, dout);
    DM_CUDA(cudaMemcpyAsync(out, dout, ng * 8, cudaMemcpyDeviceToHost, c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
    API_END
}

int dmfted_time_hxv(dmfted_ctx *c, int32_t flags, int32_t warmup, int32_t reps, double *ms) {
    API_BEGIN
    DM_REQUIRE(c && ms && reps >= 1 && warmup >= 0, DMFTED_ERR_ARG, "bad argument");
    DM_REQUIRE(c->cur_sector != 0, DMFTED_ERR_STATE, "time_hxv: Hsector NOT set");
    DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "time_hxv: bath not set");
    DM_CUDA(cudaSetDevice(c->device));
    const bool fp32 = (flags & 1) != 0, fused = (flags & 2) != 0, whole = (flags & 8) != 0;
    SectorView s = (flags & 4) ? chain_view(c, c->cur_sector) : sector_view(c, c->cur_sector);
    const size_t es = fp32 ? 4 : 8;
    const size_t ld = (size_t)((s.dim + 31) / 32 * 32);
    c->chainbuf.alloc(3 * ld * es);
    DM_CUDA(cudaMemsetAsync(c->chainbuf.p, 0, 3 * ld * es, c->stream));
    void *x = c->chainbuf.p, *y = c->chainbuf.p + ld * es, *xp = c->chainbuf.p + 2 * ld * es;
    LanczosScalars lz = lz_slot(c, 3, kLzMax);
    if (whole) lz.kmax = kLzMax - 2;  // step 1 never reaches the step limit
    if (fused || whole) {
        // step k = 1 of a recurrence with unit scales and b_1 = 0.5
        std::vector<double> init(kLzStride, 0.0);
        for (int i = 0; i < kLzMax + 2; i++) init[2 * (kLzMax + 2) + i] = 1.0;  // scale
        init[(kLzMax + 2) + 1] = 0.5;                                           // beta[1]
        DM_CUDA(cudaMemcpyAsync(lz.alpha, init.data(), kLzStride * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream));
        DM_CUDA(cudaMemsetAsync(lz.status, 0, 8 * sizeof(int), c->stream));
    }
    auto run = [&]() {
        if (whole) {
            // the whole step (update and |w| included); a negative breakdown
            // threshold keeps the zero test vectors from ending the recurrence
            if (fp32) lanczos_step<float>(c, s, (const float *)x, (const float *)xp, (float *)y, s.dim, lz, 1, -1.0, 1);
            else lanczos_step<double>(c, s, (const double *)x, (const double *)xp, (double *)y, s.dim, lz, 1, -1.0, 1);
        } else if (fused) {
            if (fp32) hxv_lanczos_step<float>(c, s, (const float *)x, (const float *)xp, (float *)y, lz, 1);
            else hxv_lanczos_step<double>(c, s, (const double *)x, (const double *)xp, (double *)y, lz, 1);
        } else {
            if (fp32) hxv_f32(c, s, (const float *)x, (float *)y, 1);
            else hxv_f64(c, s, (const double *)x, (double *)y, 1);
        }
    };
    for (int i = 0; i < warmup; i++) run();
    cudaEvent_t e0, e1;
    DM_CUDA(cudaEventCreate(&e0));
    DM_CUDA(cudaEventCreate(&e1));
    DM_CUDA(cudaEventRecord(e0, c->stream));
    for (int i = 0; i < reps; i++) run();
    DM_CUDA(cudaEventRecord(e1, c->stream));
    DM_CUDA(cudaEventSynchronize(e1));
    float t;
    DM_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    API_END
}

int dmfted_autotune_log(dmfted_ctx *c, char *buf, int32_t len, int32_t *needed) {
    API_BEGIN
    DM_REQUIRE(c && (buf || len == 0) && len >= 0, DMFTED_ERR_ARG, "bad argument");
    std::string all;
    for (const std::string &l : c->tune_log) all += l + "\n";
    if (needed) *needed = (int32_t)all.size() + 1;
    if (len > 0) {
        const size_t n = std::min<size_t>(all.size(), (size_t)len - 1);
        memcpy(buf, all.data(), n);
        buf[n] = '\0';
    }
    API_END
}

int dmfted_hxv_timing(dmfted_ctx *c, int32_t on) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    hv_timer_collect(c);
    c->hv_timing = on != 0;
    c->hv_ms = c->hv_bytes = 0.0;
    c->hv_count = 0;
    API_END
}

int dmfted_get_hxv_timing(dmfted_ctx *c, double *ms, int64_t *launches, double *bytes) {
    API_BEGIN
    DM_REQUIRE(c && ms && launches && bytes, DMFTED_ERR_ARG, "null argument");
    DM_CUDA(cudaSetDevice(c->device));
    hv_timer_collect(c);
    *ms = c->hv_ms;
    *launches = c->hv_count;
    *bytes = c->hv_bytes;
    c->hv_ms = c->hv_bytes = 0.0;
    c->hv_count = 0;
    API_END
}

int dmfted_get_timings(dmfted_ctx *c, double *t, int64_t *n) {
    API_BEGIN
    DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
    if (t)
        for (int i = 0; i < 4; i++) t[i] = c->stats.ms[i];
    if (n)
        for (int i = 0; i < 3; i++) n[i] = c->stats.hv[i];
    API_END
}

int dmfted_launch_count(dmfted_ctx *c, int64_t *count, int32_t reset) {
    API_BEGIN
    DM_REQUIRE(c && count, DMFTED_ERR_ARG, "null argument");
    *count = c->launches;
    if (reset) c->launches = 0;
    API_END
}

}  // extern "C"
