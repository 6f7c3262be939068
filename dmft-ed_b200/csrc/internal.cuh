// Internal declarations of the B200 exact-diagonalization library.
//
// Device layout (one context per process/GPU):
//   Fock tables, built once per dmfted_init, for ALL popcount classes n of
//   Ns-bit words (2^Ns words in total).  Each class starts at a storage offset
//   poff[n] padded to 32 elements, so 16-byte vector loads of any class are
//   aligned:
//     words[poff[n] + r]        r-th Ns-bit word with popcount n, increasing
//     rank[w]                   r such that words[poff[popcount w] + r] == w
//   Hopping tables per spin, rebuilt on every set_bath (they skip zero
//   couplings as the reference's `if(V/=0)` tests do):
//     cnt[poff[n] + r]          hops of word r
//     ell[W*poff[n] + e*C(Ns,n) + r]  packed hop e of word r (ELL,
//                               row-contiguous so a warp reads 32 rows at once)
//     diag[poff[n] + r]         sum_k e_k n_k of the word (bath energies)
//   A sector (nup, ndw) is a view: rows = class nup of the up tables,
//   columns = class ndw of the down tables.  A sector vector is the
//   DimUp x DimDw column-major matrix V[iup + DimUp*idw], which is exactly
//   the reference's H%map order (ED_SETUP.f90:880-890).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dmfted.h"

namespace dmfted {

constexpr int kMaxNs = 20;     // 2^20 words; rank fits the 20-bit ELL field
constexpr int kMaxNorb = 3;    // ED_SETUP.f90:275
constexpr int kMaxParams = 256;
constexpr int kMaxW = 64;      // hops per word (Norb*Nbath + Norb*(Norb-1))
constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 4096;

// Packed ELL entry: bits 0..19 target rank, 20..27 coupling index, 31 sign.
__host__ __device__ inline uint32_t ell_pack(uint32_t col, uint32_t par, uint32_t neg) {
    return col | (par << 20) | (neg << 31);
}
__host__ __device__ inline uint32_t ell_col(uint32_t e) { return e & 0xFFFFFu; }
__host__ __device__ inline uint32_t ell_par(uint32_t e) { return (e >> 20) & 0xFFu; }
__host__ __device__ inline bool ell_neg(uint32_t e) { return (e >> 31) != 0u; }

struct StatusError {
    int code;
    std::string msg;
};

// Set the thread-local last error and return code.
int set_error(int code, const std::string &msg);
const char *last_error();

#define DM_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            throw ::dmfted::StatusError{DMFTED_ERR_CUDA,                                \
                                        std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define DM_CHECK_LAUNCH() DM_CUDA(cudaGetLastError())

// Device-side index checks of a checked build (-DDMFTED_DEVICE_CHECKS): an
// out-of-range index is reported with printf and the access is skipped, so a
// bad launch shows where it went wrong instead of faulting.  Compiles to
// `true` in the normal build.
#ifdef DMFTED_DEVICE_CHECKS
__device__ __forceinline__ bool dm_in(int64_t i, int64_t n, const char *file, int line) {
    if (i >= 0 && i < n) return true;
    printf("dmfted device check failed: %s:%d block %d thread %d index %lld extent %lld\n", file,
           line, (int)blockIdx.x, (int)threadIdx.x, (long long)i, (long long)n);
    return false;
}
#define DM_IN(i, n) ::dmfted::dm_in((int64_t)(i), (int64_t)(n), __FILE__, __LINE__)
#else
#define DM_IN(i, n) true
#endif

#define DM_REQUIRE(cond, code, msg)                                  \
    do {                                                             \
        if (!(cond)) throw ::dmfted::StatusError{(code), (msg)};     \
    } while (0)

// A device buffer owned by the context (freed with it).  Grow-only: alloc()
// keeps the current allocation when it is large enough.
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void swap(DBuf &o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            n = 0;
            throw StatusError{DMFTED_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e) +
                                                    " (" + std::to_string(count * sizeof(T)) +
                                                    " bytes)"};
        }
        n = count;
    }
    void release() {
        // The context works on a non-blocking stream, so nothing orders a free
        // after that stream's queued work: wait for the device first.
        if (p) {
            cudaDeviceSynchronize();
            cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
};

// Spin-resolved hopping/diagonal tables (device).
struct SpinTables {
    DBuf<uint8_t> cnt;
    DBuf<uint32_t> ell;
    // gather table of k_hxv_lean, width WX = max(W, 8): per hop the byte offset
    // of the target row in a 16-byte-per-row tile (bits 0..23) and the signed
    // coupling index 2p + sign (bits 24..31; 255 = zero coupling, padding)
    DBuf<uint32_t> ellx;
    std::vector<int> cls_max;  // most hops of a word, per popcount class
    DBuf<double> diag;
    DBuf<float> diag_f;
    DBuf<double> par;  // [P] coupling values (V_{a,k}, then Re Hloc_{ab})
    DBuf<float> par_f;
};

// Lanczos scalar block on the device.  alpha[k], beta[k] (beta[0] = 0),
// scale[k] = 1/|s_k| of the stored (unnormalised) vector s_k, and
// status ints: [0] done, [1] steps completed, [2] converged.
struct LanczosScalars {
    double *alpha, *beta, *scale, *ritz;  // ritz[0]=last E0, ritz[1]=previous
    int *status;
    int kmax;
};

// A sector as seen by the kernels.
struct SectorView {
    int isector;  // 1-based
    int nup, ndw;
    int64_t dimup, dimdw, dim;
    int64_t offup, offdw;  // class offsets into word-indexed arrays
    // Vectors of this view are stored transposed, idw + DimDw*iup, instead of
    // the reference order iup + DimUp*idw.  Only for device-internal vectors
    // (Green's-function chains) of sectors with odd DimUp and even DimDw, so
    // that the H*v rows pair into aligned two-element vectors.
    bool swapped = false;
};

// Per-phase timing / counting of the last solve.
struct SolveStats {
    double ms[4] = {0, 0, 0, 0};
    int64_t hv[3] = {0, 0, 0};
};

}  // namespace dmfted

struct dmfted_ctx {
    dmfted_params p{};
    int ns = 0, norb = 0, nbath = 0, nspin = 0;
    int nsectors = 0;
    int W = 0;  // ELL width
    int WX = 0; // width of the lean gather table (max(W, 8))
    int P = 0;  // couplings per spin
    int64_t nwords = 0;
    std::vector<int64_t> class_off;   // compact class offsets (size kMaxNs+2)
    std::vector<int64_t> class_poff;  // storage offsets, each class padded to 32 elements
    int64_t nstore = 0;               // padded length of the word-indexed tables
    std::vector<int64_t> binom;      // C(ns, n), n = 0..ns (exact integers)
    // host sector tables (1-based, as the reference)
    std::vector<int32_t> getsector, getnup, getndw, getdim, getdimup, getdimdw, getcsector,
        getcdgsector, getbathstride, impindex;
    std::vector<uint8_t> twin_mask;
    std::vector<int32_t> neigen_sector;
    // model
    std::vector<double> bath_e, bath_v;  // [nspin][norb][nbath]
    std::vector<double> hloc;            // complex (re,im), Fortran order
    bool bath_set = false;
    bool jterms = false;  // Jhflag spin-exchange / pair-hopping terms present (Norb > 1)
    int device = 0;
    cudaStream_t stream = nullptr;
    // device Fock tables
    dmfted::DBuf<uint32_t> words;
    dmfted::DBuf<int32_t> rank;
    dmfted::DBuf<int64_t> d_class_off;
    dmfted::SpinTables spin[2];
    std::vector<uint8_t> ell_pattern[2];  // non-zero couplings the tables were built for
    bool spin_shared = true;  // Nspin == 1: down tables alias the up tables
    dmfted::DBuf<double> dint;  // [(1<<norb)^2] impurity-only diagonal
    dmfted::DBuf<float> dint_f;
    // reduction scratch and Lanczos scalars
    dmfted::DBuf<double> red_partials;  // grid-reduction (hi, lo) pairs
    dmfted::DBuf<unsigned> red_counter;  // ticket counters (left at 0)
    // second lane: a stream with its own reduction scratch, chain buffers and
    // start vector, so that two Green's-function chains run concurrently
    // (batch.cu, SecondLane)
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    dmfted::DBuf<double> red_partials2;
    dmfted::DBuf<unsigned> red_counter2;
    dmfted::DBuf<uint8_t> chainbuf2;
    dmfted::DBuf<double> s64d;
    int chain_lanes = 2;
    int64_t gs_restarts = 0;            // FP64 ground-state runs restarted on their true residual                // grid-wide chains run two at a time (1: in turn)
    dmfted::DBuf<double> red_out;        // small result slots
    dmfted::DBuf<double> lz_d;           // Lanczos scalar slots
    dmfted::DBuf<int> lz_s;              // Lanczos status slots
    dmfted::DBuf<double> coefb;          // Ritz coefficients
    // current sector of the procedure-pointer H*v
    int cur_sector = 0;
    // work vectors (grown on demand)
    dmfted::DBuf<double> wv64;            // compatibility-mode H*v vectors
    dmfted::DBuf<uint8_t> work;           // Krylov basis of the ground-state iteration
    dmfted::DBuf<uint8_t> chainbuf;       // rotating vectors of a GF chain
    dmfted::DBuf<double> s64a, s64b, s64c;  // sector-sized FP64 scratch
    double mixed_tol32 = 1e-6;            // FP32-phase stopping tolerance of the mixed form
    int64_t gs_basis_budget = 0;          // bytes the ground-state basis may take (0: 85 % of free memory)
    int gf_head64 = 20;                   // leading FP64 steps of a mixed-form GF chain
    int tune_nc = 0;                      // H*v columns per CTA override (0 = automatic)
    int tune_hxv = 0;                     // H*v kernel: 0 automatic, 1 k_hxv, 2 k_hxv_rv, 3 k_hxv_global
    int tune_occ = 3;                     // k_hxv_lean CTAs per SM (3: 80 registers; 2: 128)
    int tune_ell_group = 0;               // lanes per hop-table balance group (0: 8)
    dmfted::DBuf<double> d_wm, d_wr;      // Matsubara / real-axis grids
    dmfted::DBuf<double> d_bath_e, d_bath_v, d_hloc_aa;  // [nspin][norb][nbath], [nspin][norb]
    dmfted::DBuf<double> obs_d;           // observable accumulators of one state
    bool hf_hops = false;                 // hf_terms holds the hop expectations of the last solve
    dmfted::DBuf<double> eig_aux;         // Ritz values, vectors of T, coefficients, dots
    dmfted::DBuf<double> eigvecs;         // eigenvectors of one sector (Neigen x dim)
    // persistent work-queue path (batch.cu): sectors up to batch_max_dim
    // states run one job per CTA
    int64_t batch_max_dim = 1 << 17;
    int64_t batch_budget = 0;             // bytes of Krylov bases per launch (0: a third of free)
    int64_t batch_cluster_min = 1024;     // states per CTA for a job shared by a cluster
    // autotuner of the batched launches (batch.cu): cluster size per job-shape
    // key, measured on first use; the log keeps every measurement.  Opt-in
    // (DMFTED_AUTOTUNE=1): the job mix of a DMFT loop shifts over its first
    // iterations (adaptive Neigen), and a first-solve measurement chose a
    // size 15 % slower in steady state than the fixed rule.
    bool autotune = false;
    std::map<std::string, int> tune_choice;
    std::vector<std::string> tune_log;
    bool ft_eigs_fp32 = false;            // finite-T eigenpairs with FP32 vectors (measurement only)
    bool batch_chains_fp32 = false;       // batched GF chains in FP32 in the mixed form (measurement only)
    dmfted::DBuf<uint8_t> bwork;          // Krylov bases / chain vectors of the jobs
    dmfted::DBuf<double> bvec;            // eigenvectors of the batched sectors
    dmfted::DBuf<double> baux;            // Ritz vectors and coefficients
    dmfted::DBuf<uint8_t> bjobs;          // job tables
    dmfted::DBuf<double> bscal;           // chain alpha / beta, norm2; eigenvalues
    dmfted::DBuf<int> bint;               // queue counter, step counts
    dmfted::DBuf<double> bcf;             // continued-fraction terms (chain x frequency)
    // dense small-sector eigensolve (dense.cu)
    dmfted::DBuf<double> dense_work, dense_vec, dense_eval;
    dmfted::DBuf<int> dense_int;
    dmfted::DBuf<uint8_t> dense_jobs;
    // eigenvectors found so far per sector of a diagonalisation (diag.cu):
    // the first pass, then every probe run, which also reads them as the
    // locked vectors it keeps its Krylov space orthogonal to
    dmfted::DBuf<double> lockpool;
    dmfted::DBuf<double> gsvec;  // eigenvectors returned by dmfted_gs_lanczos
    dmfted::DBuf<uint8_t> jscratch;  // H*x of a Lanczos step computed in parts (Jhflag)
    dmfted::DBuf<uint8_t> jscratch2; // the same for the second chain lane
    int64_t launches = 0;
    // live timing of the H*v launches (dmfted_hxv_timing)
    bool hv_timing = false;
    std::vector<cudaEvent_t> hv_ev_free;              // recycled events
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> hv_ev;  // pairs not yet read
    std::vector<double> hv_ev_bytes;
    double hv_ms = 0.0, hv_bytes = 0.0;
    int64_t hv_count = 0;
    // results of the last solve (device and host)
    struct State {
        double e;
        int isector;
        int64_t off;                  // offset (elements) of the vector in states64
        const double *src = nullptr;  // not yet copied: the vector is still here
        // twin entry of ed_twin (es_insert_state_c, ED_EIGENSPACE.f90:185-195):
        // the spin-flipped copy of the state just before it in the list,
        // sector (ndw, nup); its vector is the transpose of that state's
        // DimUp x DimDw matrix (es_return_cvector with twin_sector_order,
        // ED_EIGENSPACE.f90:399-430, ED_SETUP.f90:1098-1126)
        bool itwin = false;
    };
    std::vector<State> states;  // energy-ordered eigenspace
    dmfted::DBuf<double> states64;
    double zeta = 1.0, egs = 0.0;
    bool finite_t = false;
    int nstates_total = 1;  // lanc_nstates_total, adapted by ed_analysis between solves
    dmfted::DBuf<double> gm, gr, g0m, g0r, sm, sr;  // complex (nspin,norb,L) blocks
    std::vector<double> obs;                   // dens, up, dw, docc, magz (norb each)
    std::vector<double> hf_terms;              // nk[2][norb][nbath], hop[2][norb][nbath]
    std::vector<double> eloc = std::vector<double>(8, 0.0);  // Epot Eint Ehartree Eknot Dust Dund Dse Dph
    // observables_impurity's other averages of the last solve: sz2(a,b),
    // n2(a,b) (norb x norb, b fastest), s2tot; and Im Sigma(iw_1), Im
    // Sigma(iw_2) per (spin, orbital) as they stood when its observables were
    // taken (get_szr runs before the Green's functions of the same solve:
    // the previous solve's self-energy, 0 before the first)
    std::vector<double> sz2, n2;
    double s2tot = 0.0;
    std::vector<double> szr_sigma;              // [nspin*norb][2]
    std::vector<double> sigma_now;              // the same two values after the last solve
    bool sigma_read = false;                    // Sigma loaded by dmfted_read_impsigma
    dmfted::SolveStats stats;
    bool solved = false;
};

namespace dmfted {

// ---- api.cu --------------------------------------------------------------
// Event pair around one H*v launch when live timing is on.
void hv_timer_begin(dmfted_ctx *c);
void hv_timer_end(dmfted_ctx *c, double bytes);

// ---- fock.cu -------------------------------------------------------------
void fock_init(dmfted_ctx *c);              // words, rank, class offsets
void fock_set_couplings(dmfted_ctx *c);     // cnt/ell/diag/par for both spins, dint
SectorView sector_view(const dmfted_ctx *c, int isector);
SectorView chain_view(const dmfted_ctx *c, int isector);

// ---- batch.cu ------------------------------------------------------------
constexpr int kEigsMaxSteps = 512;  // Lanczos steps of one batched eigensolve job
constexpr int kEigsMaxEigen = 64;   // eigenpairs of one batched eigensolve job
// An eigensolve ends at an invariant subspace: b_{k+1} <= kEigsBreakRel * |T|.
// Continuing from the rounding-level residual would restart the recurrence in
// a random direction and put several copies of an eigenvalue into one T,
// whose eigenvectors inverse iteration cannot separate; the copies are found
// by the probe runs instead (diag.cu).
constexpr double kEigsBreakRel = 1e-12;
// Start-vector seed of the probe run that holds nlock locked vectors (the
// first run's seed for nlock = 0): a fresh random direction each time, since
// the first run's start vector lies in the Krylov space already explored.
__host__ __device__ inline uint64_t eigs_seed(int nlock) {
    return 1234567ull + 0x9E3779B97F4A7C15ull * (uint64_t)nlock;
}
// Lowest eigenpairs of many sectors, one CTA per sector.  For every entry of
// `list`: results[i].m >= 0 when the sector ran here (m eigenpairs, values in
// evals, FP64 vectors at vecs, dim apart), -1 when it must take the grid path
// (too large, or neigen == 0 gives m = 0).
struct BatchEig {
    int m = -1, steps = 0;
    std::vector<double> evals;
    const double *vecs = nullptr;
};
// want[i]: eigenpairs wanted of sector list[i] (0: skip).  locks (may be
// null): per entry the FP64 vectors to keep the run orthogonal to, as
// (offset into c->lockpool, count); FP64 only.
struct LockSpec {
    int64_t off = 0;
    int n = 0;
    double top = 1e300;  // the run may stop once its lowest Ritz value is surely above this
};
void batch_eigs(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                int precision, std::vector<BatchEig> &results,
                const std::vector<LockSpec> *locks = nullptr);
// Green's-function chains: one record per chain, in accumulation order.
struct ChainRec {
    int64_t psi_off;  // state vector in states64
    int isector, jsector, ispin, iorb, particle, nlanc;
    double weight, e;
};
// Runs every chain (one CTA per chain up to batch_max_dim states, the grid
// path above it) and adds all of them to the Matsubara / real-axis G.
void batch_chains_gf(dmfted_ctx *c, const std::vector<ChainRec> &recs, int precision);
void fock_build_map(dmfted_ctx *c, int isector, int32_t *d_map);  // combined map
// One chain's continued fraction (coefficients on the host) added to host
// arrays gm[lmats], gr[lreal] (complex; gr may be null).
void gf_add_chain(dmfted_ctx *c, int nlanc, const double *alanc, const double *blanc,
                  double weight, double norm2, double ei, int isign, double *gm, double *gr);

// ---- dense.cu ------------------------------------------------------------
// Dense eigensolve (Householder + tridiagonal, one CTA per sector) of the sectors ed_diag_c
// hands to eigh: the lowest want[i] eigenpairs of sector list[i] (want 0:
// skipped, m = -1).  Vectors are FP64 at vecs, dim apart, owned by the
// context until the next call.
constexpr int kDenseMaxDim = 1024;
constexpr int kDenseMaxEigen = 64;
struct DenseEig {
    int m = -1;
    std::vector<double> evals;
    const double *vecs = nullptr;
};
void dense_eigs(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                std::vector<DenseEig> &res);
// The same in two halves: the launch queues the work on the context's stream
// (the one current at the call) and returns; the collect waits for it.
struct DenseJob {
    int nup, ndw;
    int n;            // sector dimension
    int m;            // eigenpairs wanted (lowest m)
    int slot;         // output slot: evals[slot * kDenseMaxEigen + j]
    int64_t a_off;    // work: A (n x n, row-major)
    int64_t out_off;  // eigenvectors: m x n FP64, vector j at out_off + j*n
};
struct DensePending {
    std::vector<DenseJob> jobs;
    std::vector<int> where;
    size_t nlist = 0;
    cudaStream_t stream = nullptr;
};
void dense_eigs_launch(dmfted_ctx *c, const std::vector<int> &list, const std::vector<int> &want,
                       DensePending &pd);
void dense_eigs_collect(dmfted_ctx *c, DensePending &pd, std::vector<DenseEig> &res);

// ---- diag.cu ---------------------------------------------------------------
// ed_diag_c (ED_DIAG.f90:93-228): every sector of `list` diagonalised with the
// reference's branch choice, then the state selection of the temperature
// regime; fills c->states.  Returns the H*v products used.
int64_t ed_diag(dmfted_ctx *c, const std::vector<int> &list);
// The lowest neigen eigenpairs of one sector, degenerate copies included, with
// ed_diag_c's branch choice (the contract of dmfted_gs_lanczos).  evals_h:
// neigen doubles; vecs (device, may be null): neigen x dim FP64.  Returns the
// number found; *steps (may be null): H*v products used.
int sector_eigenpairs(dmfted_ctx *c, int isector, int neigen, double *evals_h, double *vecs,
                      int64_t *steps);
void states_reset(dmfted_ctx *c);
// es_pop_state on the last entry: a twin entry goes together with its state.
void states_pop_last(dmfted_ctx *c);

// ---- hxv.cu --------------------------------------------------------------
// y = H x for nvec vectors of sector s (plain product).
void hxv_f64(dmfted_ctx *c, const SectorView &s, const double *x, double *y, int nvec);
void hxv_f32(dmfted_ctx *c, const SectorView &s, const float *x, float *y, int nvec);

// ---- lanczos.cu ------------------------------------------------------------
constexpr int kLzMax = 1024;                  // max steps of one recurrence
constexpr int kLzStride = 3 * (kLzMax + 2) + 4;
constexpr int kLzSlots = 4;
LanczosScalars lz_slot(dmfted_ctx *c, int slot, int kmax);
template <typename T>
void hxv_lanczos_step(dmfted_ctx *c, const SectorView &s, const T *x, const T *xprev, T *y,
                      const LanczosScalars &lz, int k, int nstack = 1);
// Lanczos step k on n = dim * nstack elements: y = w_{k+1} (unnormalised),
// a_k, b_{k+1}.
template <typename T>
void lanczos_step(dmfted_ctx *c, const SectorView &s, const T *x, const T *xp, T *y, int64_t n,
                  const LanczosScalars &lz, int k, double thr, int nstack);
struct LanczosResult {
    double e0;
    int steps;
    bool converged;
    bool capped = false;  // the stored basis was cut below the iteration limit by device memory
};
// Ground state of sector s.  psi (device, length dim, float64) receives the
// normalised Ritz vector.  start: optional device float64 start vector.
LanczosResult lanczos_gs(dmfted_ctx *c, const SectorView &s, double *psi, const double *start,
                         int precision, double tol, int nitermax);
// Queue the tridiagonalisation of a chain from device vector v0 (float64, any
// norm) into scalar slot lz (kmax = nlanc).  Asynchronous.
// nstack = 2 runs a complex vector as its stacked re/im halves (length 2*dim).
void lanczos_chain(dmfted_ctx *c, const SectorView &s, const double *v0, int precision,
                   const LanczosScalars &lz, int nstack = 1);
// The same recurrence (FP64) on caller-owned vectors and caller-supplied
// reduction scratch; allocates nothing.
template <typename T>
void hxv_lanczos_step_scratch(dmfted_ctx *c, const SectorView &s, const T *x, const T *xprev, T *y,
                              const LanczosScalars &lz, int k, double *partials,
                              unsigned *counter);
void lanczos_chain_fixed(dmfted_ctx *c, const SectorView &s, const double *v0, double *work,
                         const LanczosScalars &lz, double *partials, unsigned *counter);

// Lowest neigen eigenpairs of sector s (full reorthogonalisation).  vecs:
// device, neigen*dim FP64 (row j = eigenvector j, normalised); evals_h host.
// Returns the number of pairs found (min(neigen, dim, steps)).
// locked/nlock: FP64 vectors (dim apart, orthonormal) the run keeps its
// Krylov space orthogonal to (Lanczos on (1-XX^T) H (1-XX^T)); needs FP64.
// top: a locked run (probe) may stop once its lowest Ritz value exceeds top by
// ten times its residual estimate (nothing wanted below top is left).
int lanczos_eigs(dmfted_ctx *c, const SectorView &s, int neigen, int precision, double tol,
                 int nitermax, double *evals_h, double *vecs, int *steps,
                 const double *locked = nullptr, int nlock = 0, double top = 1e300);

// ---- gf.cu ---------------------------------------------------------------
// vv = c^+_{iorb,ispin} psi (particle) or c psi (hole) in sector sj;
// |vv|^2 -> *d_norm2 (device).  Asynchronous.
void gf_apply_op(dmfted_ctx *c, const SectorView &si, const SectorView &sj, int iorb, int ispin,
                 bool particle, const double *psi, double *vv, double *d_norm2);
void gf_sigma(dmfted_ctx *c);  // impSmats/impSreal/impG0mats from impG*

// ---- observables.cu --------------------------------------------------------
int obs_count(const dmfted_ctx *c);
int obs_pair_count(const dmfted_ctx *c);
void observables_raw(dmfted_ctx *c, const SectorView &s, const double *psi, double *d_out,
                     bool hops);

// ---- chi2.cu -------------------------------------------------------------
void chi2_batch_device(dmfted_ctx *c, int nbatch, int nbath, int L, const double *a,
                       const double *x, const double *g, const double *w, double *chi2,
                       double *grad);

// ---- fit.cu ----------------------------------------------------------------
void cg_fit_device(dmfted_ctx *c, int nbatch, int nbath, int L, double *a, const double *x,
                   const double *g, int ng, const double *w, const double *zc, double zc0,
                   int weiss, int itmax, int istop, double ftol, double eps, int *iter,
                   double *chi2, int *status);
void gloc_diag_device(dmfted_ctx *c, int L, int le, const double *he, const double *wt,
                      const double *wm, double eps, const double *sig, double *gl);
void weiss_diag_device(dmfted_ctx *c, int L, int scheme, const double *hloc_aa, const double *wm,
                       const double *gl, const double *sig, double *out);

// ---- small helpers ------------------------------------------------------------
inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
int num_sms(dmfted_ctx *c);

}  // namespace dmfted
