// Diagonalisation of the sectors: ed_diag_c (ED_DIAG.f90:93-228) and the
// eigenspace list it fills (ED_EIGENSPACE.f90:126-213).
//
// Every sector gets Neigen = min(dim, neigen_sector) eigenpairs, and the
// reference's branch choice (ED_DIAG.f90:136-137): the dense eigensolve
// (dense.cu) when Neigen == dim or dim <= lanc_dim_threshold, otherwise the
// Lanczos solvers -- one CTA or cluster per sector up to batch_max_dim states
// (batch.cu), grid-wide above (lanczos.cu).
//
// A Lanczos run from one start vector sees one copy of each degenerate
// eigenvalue, where the reference's ARPACK-based sp_eigh returns the
// copies.  So a run is followed by probe runs: Lanczos from a fresh start
// vector kept orthogonal to every eigenvector found so far (the found vectors
// are "locked"), which finds the lowest eigenvalue of H on their complement.
// A probe whose eigenvalue belongs to the wanted set adds it and triggers the
// next probe; the first probe that finds nothing new ends the sector.
//   - finite temperature: the first run asks for Neigen pairs; a probe
//     eigenvalue is new when fewer than Neigen pairs are known or it lies
//     below the Neigen-th lowest known one.  The lowest Neigen go to the
//     state list, es_add_state with the lanc_nstates_total cap.
//   - zero temperature: only eigenvalues within 11*gs_threshold of a sector's
//     lowest one can survive the ground-state selection (an eigenvalue e of
//     a sector whose lowest is e0 is kept only if |e - oldzero| <= gs_threshold
//     while oldzero <= e0 + 10*gs_threshold), so the first run asks for the
//     lowest pair and the probes for the degenerate copies within that
//     window, up to Neigen.  With Neigen == 1 no probe runs: the reference
//     keeps one state per sector then too.  The selection of ED_DIAG.f90:202-214
//     then runs over the sectors in order.
// The first run at T=0 on the grid path is the precision-aware ground-state
// Lanczos (FP64 or mixed); every other eigenpair is FP64 (an FP32 Krylov
// basis returns spurious copies of converged eigenvalues).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <numeric>
#include <vector>

#include "internal.cuh"

namespace dmfted {

// ---------------------------------------------------------------------------
// State list (es_add_state / es_insert_state, ED_EIGENSPACE.f90:126-213): the
// kept eigenvectors in one device pool, energy-ordered.
void states_reset(dmfted_ctx *c) { c->states.clear(); }

static int64_t state_dim(const dmfted_ctx *c, int isector) {
    return c->binom[c->getnup[isector - 1]] * c->binom[c->getndw[isector - 1]];
}

static int64_t states_used(const dmfted_ctx *c) {
    int64_t u = 0;
    for (auto &s : c->states)
        if (!s.src && s.off >= 0) u = std::max<int64_t>(u, s.off + state_dim(c, s.isector));
    return u;
}

// Grows the eigenspace store to hold `need` elements, keeping the first
// `used` ones.
static void states_reserve(dmfted_ctx *c, int64_t used, int64_t need) {
    if ((size_t)need > c->states64.n) {
        const size_t cap = std::max<size_t>((size_t)need, c->states64.n * 2);
        double *np = nullptr;
        cudaError_t err = cudaMalloc((void **)&np, cap * sizeof(double));
        DM_REQUIRE(err == cudaSuccess, DMFTED_ERR_NOMEM, "cudaMalloc for the eigenspace failed");
        if (c->states64.p && used > 0)
            DM_CUDA(cudaMemcpyAsync(np, c->states64.p, used * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
        DM_CUDA(cudaStreamSynchronize(c->stream));
        c->states64.release();
        c->states64.p = np;
        c->states64.n = cap;
    }
}

// The twin sector (ndw, nup) of a sector (get_twin_sector).
static int twin_sector(const dmfted_ctx *c, int isector) {
    const int nup = c->getnup[isector - 1], ndw = c->getndw[isector - 1];
    return c->getsector[ndw * (c->ns + 1) + nup];
}

// Energy-ordered insertion after equal energies (es_insert_state_c,
// ED_EIGENSPACE.f90:157-213: traverse until e <= next); with twin, the twin
// entry follows the state directly.
static void states_insert(dmfted_ctx *c, const dmfted_ctx::State &st, bool twin = false) {
    auto it = c->states.begin();
    while (it != c->states.end() && !(st.e <= it->e)) ++it;
    it = c->states.insert(it, st);
    if (twin) {
        dmfted_ctx::State tw{st.e, twin_sector(c, st.isector), -1, nullptr};
        tw.itwin = true;
        c->states.insert(it + 1, tw);
    }
}

// es_pop_state on the last entry (ED_EIGENSPACE.f90:219-299): a twin entry
// goes together with its state.
void states_pop_last(dmfted_ctx *c) {
    if (c->states.empty()) return;
    const bool tw = c->states.back().itwin;
    c->states.pop_back();
    if (tw && !c->states.empty()) c->states.pop_back();
}

// B[q + DimDw*r] = A[r + DimUp*q]: the twin vector of a state of sector A
// (DimUp x DimDw) in the twin sector B, whose up words are A's down words.
__global__ void k_twin_transpose(const double *A, double *B, int64_t dimup, int64_t dimdw) {
    const int64_t n = dimup * dimdw;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = k % dimup, q = k / dimup;
        B[q + dimdw * r] = A[k];
    }
}

// Copies every state whose vector is still held elsewhere into the store and
// builds the twin entries' vectors from their states'.
static void states_materialize(dmfted_ctx *c) {
    int64_t used = states_used(c), need = (used + 31) / 32 * 32;
    for (auto &s : c->states)
        if (s.src || s.itwin) need = (need + state_dim(c, s.isector) + 31) / 32 * 32;
    states_reserve(c, used, need);
    int64_t off = (used + 31) / 32 * 32;
    for (size_t i = 0; i < c->states.size(); i++) {
        auto &s = c->states[i];
        const int64_t dim = state_dim(c, s.isector);
        if (s.src) {
            DM_CUDA(cudaMemcpyAsync(c->states64.p + off, s.src, dim * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
        } else if (s.itwin && s.off < 0) {
            DM_REQUIRE(i > 0 && !c->states[i - 1].itwin, DMFTED_ERR_STATE,
                       "eigenspace: a twin entry without its state");
            const auto &a = c->states[i - 1];
            const int64_t du = c->binom[c->getnup[a.isector - 1]];
            const int64_t dd = c->binom[c->getndw[a.isector - 1]];
            k_twin_transpose<<<(int)std::min<int64_t>(div_up(dim, 256), 4 * num_sms(c)), 256, 0,
                               c->stream>>>(c->states64.p + a.off, c->states64.p + off, du, dd);
            DM_CHECK_LAUNCH();
            c->launches++;
        } else {
            continue;
        }
        s.off = off;
        s.src = nullptr;
        off = (off + dim + 31) / 32 * 32;
    }
    DM_CUDA(cudaStreamSynchronize(c->stream));
}

// es_add_state with a size limit (ED_EIGENSPACE.f90:126-151): below the
// limit insert; at the limit insert only below the highest energy, which is
// popped first (es_pop_state, :219-299).  The vector stays where it is until
// states_materialize.
static void states_add_capped(dmfted_ctx *c, double e, int isector, const double *psi, int size,
                              bool twin) {
    const bool take = (int)c->states.size() < size;
    if (!take && !(!c->states.empty() && e < c->states.back().e)) return;
    if (!take) states_pop_last(c);
    states_insert(c, dmfted_ctx::State{e, isector, -1, psi}, twin);
}

// ---------------------------------------------------------------------------
namespace {

enum Branch { kDense = 0, kBatch = 1, kGrid = 2 };

struct SectorJob {
    int isector = 0;
    SectorView s{};
    int neigen = 0;   // Neigen = min(dim, neigen_sector)
    Branch br = kDense;
    int cap = 0;      // lock-pool slots (vectors) of the sector
    int64_t base = 0; // first slot's element offset in c->lockpool
    std::vector<double> e;  // eigenvalues found, in slot order
    bool probing = false;
    int steps = 0;
    const double *dense_vecs = nullptr;  // dense branch: vectors in c->dense_vec
};

bool batch_fits(const dmfted_ctx *c, const SectorJob &j, int want) {
    const int kmax = (int)std::min<int64_t>(std::min(c->p.lanc_niter, kLzMax - 2), j.s.dim);
    return c->batch_max_dim > 0 && j.s.dim <= c->batch_max_dim && kmax <= kEigsMaxSteps &&
           want <= kEigsMaxEigen;
}

double *slot_ptr(dmfted_ctx *c, const SectorJob &j, int k) {
    return c->lockpool.p + j.base + (int64_t)k * j.s.dim;
}

// Zero temperature: the ground-state window above energy e0.
double t0_window(const dmfted_ctx *c, double e0) {
    return e0 + 11.0 * c->p.gs_threshold + 4.0 * c->p.lanc_tolerance * std::max(1.0, std::fabs(e0));
}

// The largest probe eigenvalue the sector still wants (+inf: any).  cut: an
// energy at or above which no state can enter the list any more (the T=0
// window of the lowest energy of all sectors, or the lanc_nstates_total-th
// lowest energy found at finite T; +inf when unknown).
double probe_top(const dmfted_ctx *c, const SectorJob &j, bool finite_t, double cut) {
    const int n = (int)j.e.size();
    if (!finite_t) {
        const double e0 = *std::min_element(j.e.begin(), j.e.end());
        return std::min(t0_window(c, e0), cut);
    }
    if (n < j.neigen) return cut;
    std::vector<double> srt = j.e;
    std::sort(srt.begin(), srt.end());
    const double top = srt[j.neigen - 1];
    return std::min(top - 1e-12 * std::max(1.0, std::fabs(top)), cut);
}

// Whether probe eigenvalue mu joins the sector's wanted set.
bool probe_accepts(const dmfted_ctx *c, const SectorJob &j, double mu, bool finite_t,
                   double cut) {
    const int n = (int)j.e.size();
    if (n >= j.cap || (!finite_t && n >= j.neigen)) return false;
    return finite_t ? mu < probe_top(c, j, true, cut) : mu <= probe_top(c, j, false, cut);
}

// The energy cut of the whole diagonalisation (see probe_top): at T=0 the
// window above the lowest energy found in any sector; at finite T with a list
// cap, the cap-th lowest of every sector's lowest Neigen energies (a later
// probe only adds energies, so the final list boundary can only be lower).
double list_cut(const dmfted_ctx *c, const std::vector<SectorJob> &jobs, bool finite_t,
                int list_cap) {
    if (!finite_t) {
        double emin = 1e300;
        for (auto &j : jobs)
            for (double e : j.e) emin = std::min(emin, e);
        return emin < 1e300 ? t0_window(c, emin) : 1e300;
    }
    if (list_cap <= 0) return 1e300;
    std::vector<double> all;
    for (auto &j : jobs) {
        std::vector<double> srt = j.e;
        std::sort(srt.begin(), srt.end());
        for (int k = 0; k < (int)srt.size() && k < j.neigen; k++) all.push_back(srt[k]);
    }
    if ((int)all.size() < list_cap) return 1e300;
    std::nth_element(all.begin(), all.begin() + (list_cap - 1), all.end());
    return all[list_cap - 1];
}

}  // namespace

// Eigenpairs of the sectors in `jobs` (filled: isector, neigen); mode T=0
// (cluster of the lowest eigenvalue) or finite T (lowest Neigen), or the
// single-sector contract of dmfted_gs_lanczos (finite-T rule).  On return
// every job holds its eigenvalues in j.e and its vectors in the lock pool (or
// dense_vecs), in slot order.  Returns the H*v products used.
static int64_t sector_spectra(dmfted_ctx *c, std::vector<SectorJob> &jobs, bool finite_t,
                              int list_cap) {
    const dmfted_params &p = c->p;
    const bool dbg = getenv("DMFTED_DEBUG_EIGS") != nullptr;
    double t_last = 0.0;
    auto stamp = [&](const char *what) {
        if (!dbg) return;
        DM_CUDA(cudaStreamSynchronize(c->stream));
        timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        const double t = ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
        if (t_last > 0.0) fprintf(stderr, "[eigs] %s: %.3f ms\n", what, t - t_last);
        t_last = t;
    };
    stamp("start");
    auto show = [&](const char *what, const SectorJob &j, int steps, int m, const double *ev,
                    int nlock) {
        if (!dbg) return;
        fprintf(stderr, "[eigs] %s sector %d dim %lld nlock %d steps %d m %d:", what, j.isector,
                (long long)j.s.dim, nlock, steps, m);
        for (int i = 0; i < m; i++) fprintf(stderr, " %.15g", ev[i]);
        fprintf(stderr, "\n");
    };
    const int eprec = c->ft_eigs_fp32 ? p.precision : DMFTED_FP64;
    int64_t hv = 0;
    // branch choice (ED_DIAG.f90:133-137; MPI_SIZE = 1)
    int64_t pool = 0;
    for (auto &j : jobs) {
        j.s = sector_view(c, j.isector);
        const bool dense = j.neigen == j.s.dim || j.s.dim <= std::max(p.lanc_dim_threshold, 1);
        if (dense) {
            j.br = kDense;
            continue;
        }
        const int first = finite_t ? j.neigen : 1;
        j.br = batch_fits(c, j, first) ? kBatch : kGrid;
        j.cap = (int)std::min<int64_t>(j.s.dim, finite_t ? 2 * j.neigen : j.neigen);
        j.base = pool;
        pool += (((int64_t)j.cap * j.s.dim) + 31) / 32 * 32;
    }
    if (pool > 0) c->lockpool.alloc((size_t)pool);
    // ---- dense sectors --------------------------------------------------
    // One CTA per sector (a few dozen at most): on the second stream when
    // batched Lanczos sectors follow, so that the batched kernel's CTAs start
    // on the SMs the dense ones leave free instead of after them (both take
    // their jobs from atomic queues, so neither waits for the other).
    std::vector<int> dense_l, dense_w;
    std::vector<size_t> dense_at;
    for (size_t i = 0; i < jobs.size(); i++)
        if (jobs[i].br == kDense) {
            dense_l.push_back(jobs[i].isector);
            dense_w.push_back(jobs[i].neigen);
            dense_at.push_back(i);
        }
    bool any_batch = false;
    for (auto &j : jobs) any_batch = any_batch || j.br == kBatch;
    const bool dense_aside = !dense_l.empty() && any_batch && c->stream2 && !dbg;
    DensePending dense_pd;
    if (!dense_l.empty()) {
        if (dense_aside) {
            DM_CUDA(cudaEventRecord(c->ev_fork, c->stream));
            DM_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
            std::swap(c->stream, c->stream2);
            try {
                dense_eigs_launch(c, dense_l, dense_w, dense_pd);
            } catch (...) {
                std::swap(c->stream, c->stream2);
                throw;
            }
            std::swap(c->stream, c->stream2);
        } else {
            dense_eigs_launch(c, dense_l, dense_w, dense_pd);
        }
    }
    auto dense_finish = [&]() {
        if (dense_l.empty()) return;
        std::vector<DenseEig> dr;
        dense_eigs_collect(c, dense_pd, dr);
        if (dense_aside) {
            // the vectors are read on the main stream from here on
            DM_CUDA(cudaEventRecord(c->ev_join, c->stream2));
            DM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        }
        for (size_t k = 0; k < dense_l.size(); k++) {
            SectorJob &j = jobs[dense_at[k]];
            j.e = dr[k].evals;
            j.dense_vecs = dr[k].vecs;
        }
        dense_l.clear();
    };
    if (!dense_aside) dense_finish();
    stamp("dense branch");
    // ---- first Lanczos run ---------------------------------------------------
    {
        std::vector<int> bl, bw;
        std::vector<size_t> at;
        for (size_t i = 0; i < jobs.size(); i++)
            if (jobs[i].br == kBatch) {
                bl.push_back(jobs[i].isector);
                bw.push_back(finite_t ? jobs[i].neigen : 1);
                at.push_back(i);
            }
        if (!bl.empty()) {
            std::vector<BatchEig> br;
            batch_eigs(c, bl, bw, eprec, br);
            for (size_t k = 0; k < bl.size(); k++) {
                SectorJob &j = jobs[at[k]];
                j.steps += br[k].steps;
                hv += br[k].steps;
                show("batch first", j, br[k].steps, std::max(br[k].m, 0), br[k].evals.data(), 0);
                const int m = std::min(std::max(br[k].m, 0), j.cap);
                j.e.assign(br[k].evals.begin(), br[k].evals.begin() + m);
                if (m > 0)
                    DM_CUDA(cudaMemcpyAsync(slot_ptr(c, j, 0), br[k].vecs,
                                            (size_t)m * j.s.dim * sizeof(double),
                                            cudaMemcpyDeviceToDevice, c->stream));
            }
        }
    }
    dense_finish();
    stamp("batched first runs");
    std::vector<double> ev(kLzMax + 8);
    for (auto &j : jobs) {
        if (j.br != kGrid) continue;
        const int nit = (int)std::min<int64_t>(j.s.dim, p.lanc_niter);
        if (!finite_t) {
            LanczosResult r =
                lanczos_gs(c, j.s, slot_ptr(c, j, 0), nullptr, p.precision, p.lanc_tolerance, nit);
            j.steps += r.steps;
            hv += r.steps;
            j.e.assign(1, r.e0);
            show("grid gs", j, r.steps, 1, &r.e0, 0);
        } else {
            int steps = 0;
            c->eigvecs.alloc((size_t)j.neigen * j.s.dim);
            const int m = std::min(lanczos_eigs(c, j.s, j.neigen, eprec, p.lanc_tolerance, nit,
                                                ev.data(), c->eigvecs.p, &steps),
                                   j.cap);
            j.steps += steps;
            hv += steps;
            show("grid first", j, steps, m, ev.data(), 0);
            j.e.assign(ev.begin(), ev.begin() + m);
            if (m > 0)
                DM_CUDA(cudaMemcpyAsync(slot_ptr(c, j, 0), c->eigvecs.p,
                                        (size_t)m * j.s.dim * sizeof(double),
                                        cudaMemcpyDeviceToDevice, c->stream));
        }
    }
    stamp("grid first runs");
    // ---- probes for degenerate copies -----------------------------------------
    // (FP64 only: the measurement-only FP32 eigenpairs skip them)
    const bool probes = eprec == DMFTED_FP64;
    for (auto &j : jobs)
        j.probing = probes && j.br != kDense && j.neigen > 1 && !j.e.empty() &&
                    (int)j.e.size() < j.cap;
    for (int round = 0;; round++) {
        std::vector<int> bl, bw;
        std::vector<LockSpec> locks;
        std::vector<size_t> at;
        bool any = false;
        // sectors whose lowest energy is at or above the cut cannot put a
        // state into the list, whatever copies a probe would find
        const double cut = list_cut(c, jobs, finite_t, list_cap);
        for (auto &j : jobs)
            if (j.probing && !j.e.empty() && *std::min_element(j.e.begin(), j.e.end()) >= cut)
                j.probing = false;
        for (size_t i = 0; i < jobs.size(); i++) {
            SectorJob &j = jobs[i];
            if (!j.probing) continue;
            any = true;
            if (j.br == kBatch && batch_fits(c, j, 1)) {
                bl.push_back(j.isector);
                bw.push_back(1);
                LockSpec ls;
                ls.off = j.base;
                ls.n = (int)j.e.size();
                ls.top = probe_top(c, j, finite_t, cut);
                locks.push_back(ls);
                at.push_back(i);
            }
        }
        if (!any) break;
        DM_REQUIRE(round < 4 * kDenseMaxEigen, DMFTED_ERR_NOTCONV,
                   "ed_diag: degenerate-copy probes did not end");
        if (!bl.empty()) {
            std::vector<BatchEig> br;
            batch_eigs(c, bl, bw, DMFTED_FP64, br, &locks);
            for (size_t k = 0; k < bl.size(); k++) {
                SectorJob &j = jobs[at[k]];
                j.steps += br[k].steps;
                hv += br[k].steps;
                show("batch probe", j, br[k].steps, std::max(br[k].m, 0), br[k].evals.data(),
                     (int)j.e.size());
                if (br[k].m >= 1 && probe_accepts(c, j, br[k].evals[0], finite_t, cut)) {
                    DM_CUDA(cudaMemcpyAsync(slot_ptr(c, j, (int)j.e.size()), br[k].vecs,
                                            j.s.dim * sizeof(double), cudaMemcpyDeviceToDevice,
                                            c->stream));
                    j.e.push_back(br[k].evals[0]);
                } else {
                    j.probing = false;
                }
            }
        }
        for (auto &j : jobs) {
            if (!j.probing || j.br != kGrid) continue;
            const int nit = (int)std::min<int64_t>(j.s.dim, p.lanc_niter);
            int steps = 0;
            c->eigvecs.alloc((size_t)j.s.dim);
            const int m = lanczos_eigs(c, j.s, 1, DMFTED_FP64, p.lanc_tolerance, nit, ev.data(),
                                       c->eigvecs.p, &steps, slot_ptr(c, j, 0), (int)j.e.size(),
                                       probe_top(c, j, finite_t, cut));
            j.steps += steps;
            hv += steps;
            show("grid probe", j, steps, m, ev.data(), (int)j.e.size());
            if (m >= 1 && probe_accepts(c, j, ev[0], finite_t, cut)) {
                DM_CUDA(cudaMemcpyAsync(slot_ptr(c, j, (int)j.e.size()), c->eigvecs.p,
                                        j.s.dim * sizeof(double), cudaMemcpyDeviceToDevice,
                                        c->stream));
                j.e.push_back(ev[0]);
            } else {
                j.probing = false;
            }
        }
        for (auto &j : jobs)
            if (j.probing && (int)j.e.size() >= j.cap) j.probing = false;
        stamp("probe round");
    }
    DM_CUDA(cudaStreamSynchronize(c->stream));
    return hv;
}

// Eigenpairs of job j in ascending energy (ties in slot order), at most
// `keep`: (energy, device vector).
static std::vector<std::pair<double, const double *>> ordered_pairs(dmfted_ctx *c,
                                                                    const SectorJob &j, int keep) {
    std::vector<int> idx(j.e.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return j.e[a] < j.e[b]; });
    std::vector<std::pair<double, const double *>> out;
    for (int k = 0; k < (int)idx.size() && k < keep; k++) {
        const double *v = j.br == kDense ? j.dense_vecs + (int64_t)idx[k] * j.s.dim
                                         : slot_ptr(c, j, idx[k]);
        out.emplace_back(j.e[idx[k]], v);
    }
    return out;
}

int64_t ed_diag(dmfted_ctx *c, const std::vector<int> &list) {
    const dmfted_params &p = c->p;
    states_reset(c);
    std::vector<SectorJob> jobs;
    for (int isector : list) {
        SectorJob j;
        j.isector = isector;
        j.neigen = (int)std::min<int64_t>(state_dim(c, isector), c->neigen_sector[isector - 1]);
        if (j.neigen <= 0) continue;
        jobs.push_back(j);
    }
    const int64_t hv = sector_spectra(c, jobs, c->finite_t, c->finite_t ? c->nstates_total : 0);
    // Tflag of ED_DIAG.f90:120-123: twin entries for the states of a sector
    // with nup != ndw when ed_twin is on
    auto tflag = [&](int isector) {
        return p.ed_twin && c->twin_mask[isector - 1] &&
               c->getnup[isector - 1] != c->getndw[isector - 1];
    };
    if (c->finite_t) {
        // ED_DIAG.f90:196-200: i = 1..Neigen into the capped list
        for (auto &j : jobs)
            for (auto &pr : ordered_pairs(c, j, j.neigen))
                states_add_capped(c, pr.first, j.isector, pr.second, c->nstates_total,
                                  tflag(j.isector));
    } else {
        // ED_DIAG.f90:202-214
        double oldzero = 1000.0;
        const double gsth = p.gs_threshold;
        for (auto &j : jobs)
            for (auto &pr : ordered_pairs(c, j, j.neigen)) {
                const double enemin = pr.first;
                if (enemin < oldzero - 10.0 * gsth) {
                    oldzero = enemin;
                    states_reset(c);
                    states_insert(c, dmfted_ctx::State{enemin, j.isector, -1, pr.second},
                                  tflag(j.isector));
                } else if (std::fabs(enemin - oldzero) <= gsth) {
                    oldzero = std::min(oldzero, enemin);
                    states_insert(c, dmfted_ctx::State{enemin, j.isector, -1, pr.second},
                                  tflag(j.isector));
                }
            }
    }
    states_materialize(c);
    return hv;
}

// One sector's lowest neigen eigenpairs with the branch choice of ed_diag_c
// and the degenerate copies (the finite-temperature rule).  evals_h:
// neigen doubles; vecs (device, may be null): neigen x dim FP64.  Returns
// the number found; *steps: H*v products.
int sector_eigenpairs(dmfted_ctx *c, int isector, int neigen, double *evals_h, double *vecs,
                      int64_t *steps) {
    std::vector<SectorJob> jobs(1);
    jobs[0].isector = isector;
    jobs[0].neigen = (int)std::min<int64_t>(state_dim(c, isector), neigen);
    const bool ft = neigen > 1;
    const int64_t hv = sector_spectra(c, jobs, ft, 0);
    if (steps) *steps = hv;
    const auto pr = ordered_pairs(c, jobs[0], jobs[0].neigen);
    const int64_t dim = state_dim(c, isector);
    for (size_t k = 0; k < pr.size(); k++) {
        evals_h[k] = pr[k].first;
        if (vecs)
            DM_CUDA(cudaMemcpyAsync(vecs + (int64_t)k * dim, pr[k].second, dim * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
    }
    DM_CUDA(cudaStreamSynchronize(c->stream));
    return (int)pr.size();
}

}  // namespace dmfted
