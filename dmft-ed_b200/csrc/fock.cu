// Fock-space tables: sector enumeration, ranks, the combined sector map and
// the spin-resolved hopping (ELL) and diagonal tables.
//
// The reference enumerates a sector by scanning all 2^Ns x 2^Ns words and
// keeping popcount matches (build_sector, ED_SETUP.f90:874-891), then finds
// every hopping target with a recursive binary search over the combined map
// (binary_search, ED_SETUP.f90:1282-1299).  Here the words of each popcount
// class are produced directly by combinatorial unranking (the r-th word of
// popcount n in increasing order), and the inverse map is a 2^Ns rank table,
// so target indices are one table load.  Both give the reference's order:
// for a fixed popcount, increasing integer order is colex order, whose rank
// is sum_i C(c_i, i) over the set-bit positions c_1 < ... < c_n.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "internal.cuh"

namespace dmfted {

// C(b, i) at b*(kMaxNs+1)+i for every b <= kMaxNs.  Constant memory is shared
// by every context of the process; this table is the same for all of them.
__constant__ int64_t c_binom[(kMaxNs + 1) * (kMaxNs + 1)];

// Class offsets of one context (they depend on Ns), passed by value.
struct ClassTab {
    int64_t off[kMaxNs + 2];   // compact offsets (enumeration)
    int64_t poff[kMaxNs + 2];  // padded storage offsets (32-element aligned)
};

static ClassTab class_tab(const dmfted_ctx *c) {
    ClassTab t{};
    for (int n = 0; n < kMaxNs + 2; n++) {
        t.off[n] = c->class_off[n];
        t.poff[n] = c->class_poff[n];
    }
    return t;
}

__device__ __forceinline__ int64_t binom_d(int b, int i) {
    return (i < 0 || b < 0 || i > b) ? 0 : c_binom[b * (kMaxNs + 1) + i];
}

// K1a: words[g] for every g in [0, 2^Ns) and the rank table.
__global__ void k_words(int ns, const ClassTab ct, uint32_t *words, int32_t *rank) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= ((int64_t)1 << ns)) return;
    int n = 0;
    while (ct.off[n + 1] <= g) n++;
    int64_t r = g - ct.off[n];
    int64_t rr = r;
    uint32_t w = 0;
    int b = ns - 1;
    for (int i = n; i >= 1; i--) {
        while (binom_d(b, i) > rr) b--;
        w |= 1u << b;
        rr -= binom_d(b, i);
        b--;
    }
    words[ct.poff[n] + r] = w;
    rank[w] = (int32_t)r;
}

// Parity of the occupied levels strictly between positions p and q.
__device__ __forceinline__ uint32_t between_parity(uint32_t w, int p, int q) {
    int lo = p < q ? p : q, hi = p < q ? q : p;
    uint32_t mask = ((1u << hi) - 1u) & ~((2u << lo) - 1u);
    return __popc(w & mask) & 1u;
}

// K2: hopping table of one spin for every word.  Entry order per word follows
// the reference's row loop: Hloc inter-orbital hopping (HxVimp.f90:16-49,
// iorb outer, jorb inner), then impurity<->bath hybridisation
// (HxVimp_bath.f90:1-38, iorb outer, kp inner; imp->bath when the impurity
// level is occupied and the bath level empty, bath->imp in the opposite
// case).  Couplings equal to zero are skipped, as the reference's
// `if(... /= 0)` conditions do.  The sign of c^+_p c_q is (-1)^(occupied
// levels strictly between p and q), the product of the two c/cdg signs of
// ED_SETUP.f90:1055-1081 (levels below the lower position cancel).
// Also writes the bath-energy part of the diagonal, sum_k e_k n_k
// (HxVbath.f90:1-13); with write_ell == 0 only the diagonal (the table depends
// on which couplings are non-zero, not on their values).
__global__ void k_ell_build(int ns, const ClassTab ct, int norb, int nbath, int W,
                            const uint32_t *words, const int32_t *rank, const double *par,
                            const double *ebath, uint8_t *cnt, uint32_t *ell, double *diag,
                            float *diag_f, int write_ell) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= ((int64_t)1 << ns)) return;
    int n = 0;
    while (ct.off[n + 1] <= g) n++;
    const int64_t r = g - ct.off[n];
    const int64_t off = ct.poff[n];
    const int64_t rows = binom_d(ns, n);
    uint32_t *erow = ell + (int64_t)W * off + r;
    const int64_t gs = off + r;  // storage index
    const uint32_t w = words[gs];
    int e = 0;
    const int pv = norb * nbath;
    if (write_ell) {
    for (int a = 0; a < norb; a++)
        for (int b = 0; b < norb; b++) {
            if (a == b) continue;
            const int p = pv + a * norb + b;
            if (par[p] == 0.0) continue;
            if (((w >> b) & 1u) && !((w >> a) & 1u)) {
                uint32_t t = (w & ~(1u << b)) | (1u << a);
                erow[(int64_t)e * rows] = ell_pack((uint32_t)rank[t], p, between_parity(w, a, b));
                e++;
            }
        }
    for (int a = 0; a < norb; a++)
        for (int k = 0; k < nbath; k++) {
            const int p = a * nbath + k;
            if (par[p] == 0.0) continue;
            const int ms = norb + a * nbath + k;
            const uint32_t ia = (w >> a) & 1u, ib = (w >> ms) & 1u;
            if (ia != ib) {
                uint32_t t = w ^ (1u << a) ^ (1u << ms);
                erow[(int64_t)e * rows] = ell_pack((uint32_t)rank[t], p, between_parity(w, a, ms));
                e++;
            }
        }
    cnt[gs] = (uint8_t)e;
    }
    double d = 0.0;
    for (int a = 0; a < norb; a++)
        for (int k = 0; k < nbath; k++) {
            const int ms = norb + a * nbath + k;
            if ((w >> ms) & 1u) d += ebath[a * nbath + k];
        }
    diag[gs] = d;
    diag_f[gs] = (float)d;
}

// Bank-quad balancing of the hopping table of one class.  In the H*v the up
// hops are gathers of 16-byte rows of the staged tile; row t sits in shared-
// memory bank quad t % 8, and one warp-wide gather serves the rows of one
// group: 64 consecutive rows split by parity when a thread owns two rows
// (vw == 2), 32 consecutive rows otherwise.  A 16-byte shared-memory access is
// served a quarter warp (8 lanes, 128 bytes) per wavefront, so the balance is
// kept within each run of `gsize` lanes (8: a quarter warp).  Which slot of a
// row's list holds which hop is free, so each group reorders its rows' entries
// greedily, slot by slot, putting on every row the hop whose target quad is
// least used so far in that slot.  Balanced quads mean fewer shared-memory
// wavefronts per gather; the set of hops of a row is unchanged.  One thread
// per group of 32 lanes.
//
// In classes whose words have at most 8 hops (those the lean H*v kernel
// serves), k_ell_climb then improves the greedy order per quarter warp by
// hill climbing: swap
// two slots of one row when that lowers the summed cost of the two slots,
// where a slot's cost is its wavefront count (the largest number of distinct
// target rows in one quad) and, below that, the sum of squared quad loads
// (which steers the search across plateaus of equal wavefront count).  On the
// 3432-row class of 14 sites at 7 particles this cuts the gather wavefronts
// of the H*v by 22 % over the greedy order (5399 -> 4184 per column tile;
// 3010 would be conflict-free).
constexpr int kClimbRows = 8, kClimbW = 16, kClimbPasses = 32;

__device__ int climb_slot_cost(const uint32_t (&t)[kClimbRows][kClimbW], const int *self, const int *c,
                               int m, int q) {
    int load[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < m; i++) {
        const uint32_t ti = q < c[i] ? t[i][q] : (uint32_t)self[i];
        bool dup = false;
        for (int j = 0; j < i; j++) dup |= (q < c[j] ? t[j][q] : (uint32_t)self[j]) == ti;
        if (!dup) load[ti & 7u]++;
    }
    int mx = 0, sq = 0;
    for (int b = 0; b < 8; b++) {
        mx = max(mx, load[b]);
        sq += load[b] * load[b];
    }
    return mx * 64 + sq;
}

__device__ void climb_quarter(uint32_t *e, int64_t rows, const int64_t *rr, const uint8_t *cnt,
                              int64_t off, int m) {
    uint32_t ent[kClimbRows][kClimbW], t[kClimbRows][kClimbW];
    int c[kClimbRows], self[kClimbRows];
    for (int i = 0; i < m; i++) {
        c[i] = min((int)cnt[off + rr[i]], kClimbW);
        self[i] = (int)rr[i];
        for (int q = 0; q < c[i]; q++) {
            ent[i][q] = e[(int64_t)q * rows + rr[i]];
            t[i][q] = ell_col(ent[i][q]);
        }
    }
    for (int pass = 0; pass < kClimbPasses; pass++) {
        bool improved = false;
        for (int i = 0; i < m; i++)
            for (int a = 0; a < c[i]; a++)
                for (int b = a + 1; b < c[i]; b++) {
                    const int before = climb_slot_cost(t, self, c, m, a) + climb_slot_cost(t, self, c, m, b);
                    uint32_t x = t[i][a];
                    t[i][a] = t[i][b];
                    t[i][b] = x;
                    const int after = climb_slot_cost(t, self, c, m, a) + climb_slot_cost(t, self, c, m, b);
                    if (after < before) {
                        improved = true;
                        x = ent[i][a];
                        ent[i][a] = ent[i][b];
                        ent[i][b] = x;
                    } else {
                        x = t[i][a];
                        t[i][a] = t[i][b];
                        t[i][b] = x;
                    }
                }
        if (!improved) break;
    }
    for (int i = 0; i < m; i++)
        for (int q = 0; q < c[i]; q++) e[(int64_t)q * rows + rr[i]] = ent[i][q];
}

__global__ void k_ell_balance(int ns, int n, int64_t off, int W, int vw, int gsize,
                              const uint8_t *cnt, uint32_t *ell) {
    const int64_t rows = binom_d(ns, n);
    const int64_t span = vw == 2 ? 64 : 32;
    const int64_t ngroups = ((rows + span - 1) / span) * vw;
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    const int64_t blk = g / vw, par = g % vw;
    uint32_t *e = ell + (int64_t)W * off;
    int load[kMaxW][8];
    const int wmax = W < kMaxW ? W : kMaxW;
    for (int q = 0; q < wmax; q++)
        for (int b = 0; b < 8; b++) load[q][b] = 0;
    for (int l = 0; l < 32; l++) {
        const int64_t r = blk * span + (int64_t)l * vw + par;
        if (r >= rows) break;
        if (l % gsize == 0)
            for (int q = 0; q < wmax; q++)
                for (int b = 0; b < 8; b++) load[q][b] = 0;
        const int c = cnt[off + r];
        // selection sort of this row's entries by current quad load, slot by slot
        for (int q = 0; q < c; q++) {
            int best = q, bl = 1 << 30;
            for (int k = q; k < c; k++) {
                const int quad = (int)(ell_col(e[(int64_t)k * rows + r]) & 7u);
                if (load[q][quad] < bl) {
                    bl = load[q][quad];
                    best = k;
                }
            }
            if (best != q) {
                const uint32_t t = e[(int64_t)q * rows + r];
                e[(int64_t)q * rows + r] = e[(int64_t)best * rows + r];
                e[(int64_t)best * rows + r] = t;
            }
            load[q][ell_col(e[(int64_t)q * rows + r]) & 7u]++;
        }
    }
}

// The hill climbing of k_ell_balance's groups, one thread per quarter warp
// (launched after the greedy pass, in classes whose words have at most 8
// hops, with gsize 8 and at most kClimbW hops per word).
__global__ void k_ell_climb(int ns, int n, int64_t off, int W, int vw, const uint8_t *cnt,
                            uint32_t *ell) {
    const int64_t rows = binom_d(ns, n);
    const int64_t span = vw == 2 ? 64 : 32;
    const int64_t nq = ((rows + span - 1) / span) * vw * 4;
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= nq) return;
    const int64_t grp = g / 4, blk = grp / vw, par = grp % vw;
    const int l0 = (int)(g % 4) * kClimbRows;
    uint32_t *e = ell + (int64_t)W * off;
    int64_t rr[kClimbRows];
    int m = 0;
    for (int i = 0; i < kClimbRows; i++) {
        const int64_t r = blk * span + (int64_t)(l0 + i) * vw + par;
        if (r < rows) rr[m++] = r;
    }
    if (m > 1) climb_quarter(e, rows, rr, cnt, off, m);
}

// Lean gather table of one class from its balanced ELL table (same slot
// order): hop e of row r becomes (target row * 16) | (2 * coupling + sign) << 24;
// slots at or beyond the row's hop count become zero-coupling entries that
// point at the row itself (conflict-free: the rows of a quarter warp sit in
// distinct bank quads).
__global__ void k_ellx_build(int64_t rows, int64_t off, int W, int WX, const uint8_t *cnt,
                             const uint32_t *ell, uint32_t *ellx) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int c = cnt[off + r];
    const uint32_t *src = ell + (int64_t)W * off + r;
    uint32_t *dst = ellx + (int64_t)WX * off + r;
    for (int e = 0; e < WX; e++) {
        uint32_t v = ((uint32_t)r << 4) | (255u << 24);
        if (e < c && e < W) {
            const uint32_t h = src[(int64_t)e * rows];
            const uint32_t sidx = ell_par(h) * 2u + (ell_neg(h) ? 1u : 0u);
            v = (ell_col(h) << 4) | ((sidx < 255u ? sidx : 255u) << 24);
        }
        dst[(int64_t)e * rows] = v;
    }
}

// Combined sector map (ED_SETUP.f90:880-890): map[i] = iup + idw*2^Ns with
// i = rank_up + DimUp*rank_dw.
__global__ void k_build_map(int ns, int64_t dimup, int64_t dim, const uint32_t *wu,
                            const uint32_t *wd, int32_t *map) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= dim) return;
    int64_t r = i % dimup, c = i / dimup;
    map[i] = (int32_t)(wu[r] | (wd[c] << ns));
}

static int64_t exact_binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; i++) r = r * (n + 1 - i) / i;
    return r;
}

void fock_init(dmfted_ctx *c) {
    const int ns = c->ns;
    std::vector<int64_t> bt((kMaxNs + 1) * (kMaxNs + 1), 0);
    for (int b = 0; b <= kMaxNs; b++)
        for (int i = 0; i <= b; i++) bt[b * (kMaxNs + 1) + i] = exact_binom(b, i);
    c->binom.assign(ns + 1, 0);
    c->class_off.assign(kMaxNs + 2, 0);
    c->class_poff.assign(kMaxNs + 2, 0);
    for (int n = 0; n <= ns; n++) c->binom[n] = exact_binom(ns, n);
    for (int n = 0; n <= kMaxNs; n++) {
        const int64_t cn = n <= ns ? c->binom[n] : 0;
        c->class_off[n + 1] = c->class_off[n] + cn;
        c->class_poff[n + 1] = c->class_poff[n] + (cn + 31) / 32 * 32;
    }
    // classes beyond ns are empty; keep offsets monotone so the class search stops
    {
        // once per device: the table is the same for every context, and other
        // contexts' kernels may be reading it
        static std::mutex mu;
        static bool loaded[64] = {false};
        std::lock_guard<std::mutex> lk(mu);
        if (!loaded[c->device & 63]) {
            DM_CUDA(cudaMemcpyToSymbol(c_binom, bt.data(), bt.size() * sizeof(int64_t)));
            loaded[c->device & 63] = true;
        }
    }
    c->nwords = (int64_t)1 << ns;
    c->nstore = c->class_poff[kMaxNs + 1];
    c->words.alloc(c->nstore);
    DM_CUDA(cudaMemsetAsync(c->words.p, 0, c->nstore * sizeof(uint32_t), c->stream));
    c->rank.alloc(c->nwords);
    k_words<<<div_up(c->nwords, 256), 256, 0, c->stream>>>(ns, class_tab(c), c->words.p,
                                                            c->rank.p);
    DM_CHECK_LAUNCH();
    c->launches++;
    c->W = c->norb * c->nbath + c->norb * (c->norb - 1);
    c->P = c->norb * c->nbath + c->norb * c->norb;
    DM_REQUIRE(c->W <= kMaxW && c->P <= kMaxParams, DMFTED_ERR_UNSUPPORTED,
               "too many couplings per level for the packed hopping table");
    c->WX = std::max(c->W, 8);
    c->spin_shared = (c->nspin == 1);
    const int nsp = c->spin_shared ? 1 : 2;
    for (int s = 0; s < nsp; s++) {
        SpinTables &t = c->spin[s];
        t.cnt.alloc(c->nstore);
        t.ell.alloc((size_t)std::max(c->W, 1) * c->nstore);
        t.ellx.alloc((size_t)c->WX * c->nstore);
        t.diag.alloc(c->nstore);
        t.diag_f.alloc(c->nstore);
        DM_CUDA(cudaMemsetAsync(t.cnt.p, 0, c->nstore, c->stream));
        t.par.alloc(c->P);
        t.par_f.alloc(c->P);
    }
    const int ni = 1 << c->norb;
    c->dint.alloc(ni * ni);
    c->dint_f.alloc(ni * ni);
}

// Impurity-only part of the diagonal as a function of the impurity occupations
// (iu, id bit sets of length Norb): HxVimp.f90:1-12 (-xmu*n + Hloc_aa*n, impurity
// levels only) and HxVint.f90:1-43 (U, Ust, Ust-Jh and the HFMODE shift).
static double impurity_diag(const dmfted_ctx *c, unsigned iu, unsigned id) {
    const int norb = c->norb, nsp = c->nspin;
    double nu[kMaxNorb], nd[kMaxNorb];
    for (int a = 0; a < norb; a++) {
        nu[a] = (iu >> a) & 1u;
        nd[a] = (id >> a) & 1u;
    }
    auto hl = [&](int is, int a) {
        int64_t idx = is + nsp * (is + nsp * (a + (int64_t)norb * a));
        return c->hloc[2 * idx];
    };
    double h = 0.0, sn = 0.0;
    for (int a = 0; a < norb; a++) sn += nu[a] + nd[a];
    h -= c->p.xmu * sn;
    for (int a = 0; a < norb; a++) {
        h += hl(0, a) * nu[a];
        h += hl(nsp - 1, a) * nd[a];
    }
    const double *U = c->p.uloc;
    const double ust = c->p.ust, jh = c->p.jh;
    for (int a = 0; a < norb; a++) h += U[a] * nu[a] * nd[a];
    if (norb > 1) {
        for (int a = 0; a < norb; a++)
            for (int b = a + 1; b < norb; b++) h += ust * (nu[a] * nd[b] + nu[b] * nd[a]);
        for (int a = 0; a < norb; a++)
            for (int b = a + 1; b < norb; b++) h += (ust - jh) * (nu[a] * nu[b] + nd[a] * nd[b]);
    }
    if (c->p.hfmode) {
        for (int a = 0; a < norb; a++) h += -0.5 * U[a] * (nu[a] + nd[a]) + 0.25 * U[a];
        if (norb > 1)
            for (int a = 0; a < norb; a++)
                for (int b = a + 1; b < norb; b++) {
                    const double nab = nu[a] + nd[a] + nu[b] + nd[b];
                    h += -0.5 * ust * nab + 0.25 * ust;
                    h += -0.5 * (ust - jh) * nab + 0.25 * (ust - jh);
                }
    }
    return h;
}

void fock_set_couplings(dmfted_ctx *c) {
    const int norb = c->norb, nbath = c->nbath, nsp = c->nspin;
    const int nsp_tab = c->spin_shared ? 1 : 2;
    for (int s = 0; s < nsp_tab; s++) {
        // spin s of the tables uses bath spin index s (0 -> ispin=1, 1 -> ispin=Nspin)
        const int bs = (s == 0) ? 0 : nsp - 1;
        std::vector<double> par(c->P, 0.0);
        std::vector<float> parf(c->P, 0.f);
        for (int a = 0; a < norb; a++)
            for (int k = 0; k < nbath; k++) {
                par[a * nbath + k] = c->bath_v[((size_t)bs * norb + a) * nbath + k];
            }
        for (int a = 0; a < norb; a++)
            for (int b = 0; b < norb; b++) {
                int64_t idx = bs + nsp * (bs + nsp * (a + (int64_t)norb * b));
                par[norb * nbath + a * norb + b] = (a == b) ? 0.0 : c->hloc[2 * idx];
            }
        for (int q = 0; q < c->P; q++) parf[q] = (float)par[q];
        SpinTables &t = c->spin[s];
        DM_CUDA(cudaMemcpyAsync(t.par.p, par.data(), c->P * sizeof(double), cudaMemcpyHostToDevice,
                                c->stream));
        DM_CUDA(cudaMemcpyAsync(t.par_f.p, parf.data(), c->P * sizeof(float), cudaMemcpyHostToDevice,
                                c->stream));
        // the table holds targets, signs and coupling indices; it changes only
        // when the set of non-zero couplings does
        std::vector<uint8_t> pattern(par.size());
        for (size_t q = 0; q < par.size(); q++) pattern[q] = par[q] != 0.0;
        const bool rebuild = pattern != c->ell_pattern[s];
        const double *d_eb = c->d_bath_e.p + (size_t)bs * norb * nbath;  // [norb][nbath] of spin bs
        k_ell_build<<<div_up(c->nwords, 256), 256, 0, c->stream>>>(
            c->ns, class_tab(c), norb, nbath, std::max(c->W, 1), c->words.p, c->rank.p, t.par.p,
            d_eb, t.cnt.p, t.ell.p, t.diag.p, t.diag_f.p, rebuild ? 1 : 0);
        DM_CHECK_LAUNCH();
        c->launches++;
        // most hops per word of each class (picks the lean H*v's hop counts,
        // and the classes whose gather order is worth the climb)
        if (rebuild) {
            std::vector<uint8_t> hc(c->nstore);
            DM_CUDA(cudaMemcpyAsync(hc.data(), t.cnt.p, c->nstore, cudaMemcpyDeviceToHost,
                                    c->stream));
            DM_CUDA(cudaStreamSynchronize(c->stream));
            t.cls_max.assign(c->ns + 1, 0);
            for (int n = 0; n <= c->ns; n++)
                for (int64_t r = 0; r < c->binom[n]; r++)
                    t.cls_max[n] = std::max<int>(t.cls_max[n], hc[c->class_poff[n] + r]);
        }
        // gather grouping of the H*v: two rows per thread for even class sizes
        for (int n = 0; rebuild && n <= c->ns; n++) {
            const int vw = (c->binom[n] % 2 == 0) ? 2 : 1;
            const int64_t ng = ((c->binom[n] + (vw == 2 ? 63 : 31)) / (vw == 2 ? 64 : 32)) * vw;
            const int gsize = c->tune_ell_group > 0 ? c->tune_ell_group : 8;
            k_ell_balance<<<div_up(ng, 64), 64, 0, c->stream>>>(
                c->ns, n, c->class_poff[n], std::max(c->W, 1), vw, gsize, t.cnt.p, t.ell.p);
            DM_CHECK_LAUNCH();
            c->launches++;
            if (t.cls_max[n] <= 8 && gsize == kClimbRows && std::max(c->W, 1) <= kClimbW) {
                k_ell_climb<<<div_up(ng * 4, 64), 64, 0, c->stream>>>(
                    c->ns, n, c->class_poff[n], std::max(c->W, 1), vw, t.cnt.p, t.ell.p);
                DM_CHECK_LAUNCH();
                c->launches++;
            }
        }
        if (rebuild) {
            for (int n = 0; n <= c->ns; n++) {
                k_ellx_build<<<div_up(c->binom[n], 256), 256, 0, c->stream>>>(
                    c->binom[n], c->class_poff[n], std::max(c->W, 1), c->WX, t.cnt.p, t.ell.p,
                    t.ellx.p);
                DM_CHECK_LAUNCH();
                c->launches++;
            }
        }
        c->ell_pattern[s] = pattern;
    }
    const int ni = 1 << norb;
    std::vector<double> di(ni * ni);
    std::vector<float> df(ni * ni);
    for (int iu = 0; iu < ni; iu++)
        for (int id = 0; id < ni; id++) {
            di[iu * ni + id] = impurity_diag(c, iu, id);
            df[iu * ni + id] = (float)di[iu * ni + id];
        }
    DM_CUDA(cudaMemcpyAsync(c->dint.p, di.data(), di.size() * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    DM_CUDA(cudaMemcpyAsync(c->dint_f.p, df.data(), df.size() * sizeof(float), cudaMemcpyHostToDevice,
                            c->stream));
    DM_CUDA(cudaStreamSynchronize(c->stream));
}

SectorView sector_view(const dmfted_ctx *c, int isector) {
    DM_REQUIRE(isector >= 1 && isector <= c->nsectors, DMFTED_ERR_ARG,
               "sector index out of range: " + std::to_string(isector));
    SectorView s;
    s.isector = isector;
    s.nup = c->getnup[isector - 1];
    s.ndw = c->getndw[isector - 1];
    s.dimup = c->binom[s.nup];
    s.dimdw = c->binom[s.ndw];
    s.dim = s.dimup * s.dimdw;
    s.offup = c->class_poff[s.nup];
    s.offdw = c->class_poff[s.ndw];
    return s;
}

SectorView chain_view(const dmfted_ctx *c, int isector) {
    SectorView s = sector_view(c, isector);
    s.swapped = s.dimup % 2 == 1 && s.dimdw % 2 == 0 && s.dimdw * 16 <= 200 * 1024;
    return s;
}

void fock_build_map(dmfted_ctx *c, int isector, int32_t *d_map) {
    SectorView s = sector_view(c, isector);
    k_build_map<<<div_up(s.dim, 256), 256, 0, c->stream>>>(c->ns, s.dimup, s.dim,
                                                            c->words.p + s.offup,
                                                            c->words.p + s.offdw, d_map);
    DM_CHECK_LAUNCH();
    c->launches++;
}

int num_sms(dmfted_ctx *c) {
    static int cached[64] = {0};
    int d = c->device;
    if (d >= 0 && d < 64 && cached[d]) return cached[d];
    int v = 0;
    DM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d));
    if (d >= 0 && d < 64) cached[d] = v;
    return v;
}

}  // namespace dmfted
