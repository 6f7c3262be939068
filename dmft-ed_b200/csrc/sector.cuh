// Sector geometry and hop tables as the one-CTA-per-job kernels see them
// (the batched Lanczos jobs in batch.cu and the dense small-sector
// eigensolve in dense.cu): the context's word-indexed tables with the class
// offsets and sizes passed by value, and a sector (nup, ndw) as views into
// them, vector order iup + DimUp*idw (the reference's H%map order).
#pragma once
#include <algorithm>

#include "internal.cuh"

namespace dmfted {

// ---------------------------------------------------------------- tables --
// Hop tables of one spin in the precision T of the vectors.
template <typename T>
struct BatchSpin {
    const uint8_t *cnt;
    const uint32_t *ell;
    const T *diag;
    const T *par;
};

template <typename T>
struct BatchTables {
    const uint32_t *words;
    const int32_t *rank;
    BatchSpin<T> sp[2];  // up, down
    const T *dint;
    int64_t poff[kMaxNs + 1];   // padded class offsets
    int64_t binom[kMaxNs + 1];  // class sizes
    int64_t nrank;              // entries of the rank table (2^Ns)
    int norb, P, W;
    double jx, jp;              // Jhflag spin-exchange / pair hopping (0: none)
};

template <typename T>
inline BatchTables<T> batch_tables(const dmfted_ctx *c) {
    BatchTables<T> b{};
    b.words = c->words.p;
    b.rank = c->rank.p;
    for (int s = 0; s < 2; s++) {
        const SpinTables &t = (s == 1 && !c->spin_shared) ? c->spin[1] : c->spin[0];
        b.sp[s].cnt = t.cnt.p;
        b.sp[s].ell = t.ell.p;
        if constexpr (sizeof(T) == 8) {
            b.sp[s].diag = (const T *)t.diag.p;
            b.sp[s].par = (const T *)t.par.p;
        } else {
            b.sp[s].diag = (const T *)t.diag_f.p;
            b.sp[s].par = (const T *)t.par_f.p;
        }
    }
    if constexpr (sizeof(T) == 8) b.dint = (const T *)c->dint.p;
    else b.dint = (const T *)c->dint_f.p;
    for (int n = 0; n <= c->ns; n++) {
        b.poff[n] = c->class_poff[n];
        b.binom[n] = c->binom[n];
    }
    b.nrank = (int64_t)1 << c->ns;
    b.norb = c->norb;
    b.P = c->P;
    b.W = std::max(c->W, 1);
    b.jx = c->jterms ? c->p.jx : 0.0;
    b.jp = c->jterms ? c->p.jp : 0.0;
    return b;
}

// Geometry of one sector inside a job (reference order iup + DimUp*idw).
template <typename T>
struct Sec {
    uint32_t dimup, dimdw, dim;
    const uint32_t *wu, *wd;
    const uint8_t *cu, *cd;
    const uint32_t *eu, *ed;
    const T *du, *dd;
};

template <typename T>
__device__ __forceinline__ Sec<T> make_sec(const BatchTables<T> &tb, int nup, int ndw) {
    Sec<T> s;
    s.dimup = (uint32_t)tb.binom[nup];
    s.dimdw = (uint32_t)tb.binom[ndw];
    s.dim = s.dimup * s.dimdw;
    const int64_t ou = tb.poff[nup], od = tb.poff[ndw];
    s.wu = tb.words + ou;
    s.wd = tb.words + od;
    s.cu = tb.sp[0].cnt + ou;
    s.cd = tb.sp[1].cnt + od;
    s.eu = tb.sp[0].ell + (int64_t)tb.W * ou;
    s.ed = tb.sp[1].ell + (int64_t)tb.W * od;
    s.du = tb.sp[0].diag + ou;
    s.dd = tb.sp[1].diag + od;
    return s;
}

}  // namespace dmfted
