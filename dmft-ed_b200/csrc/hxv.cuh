// Up/down-factored on-the-fly H*v (the product of directMatVec_cc,
// ED_HAMILTONIAN_MATVEC.f90:289-351 with build_hxv.f90 and its four includes)
// on a sector vector V stored as the DimUp x DimDw column-major matrix:
//
//   (H V)[r, c] = (Dup[r] + Ddw[c] + Dimp[imp(r), imp(c)]) V[r, c]     diagonal
//               + sum_{hops r->r'} t V[r', c]                          Hup (x) 1
//               + sum_{hops c->c'} t V[r, c']                          1 (x) Hdw
//
// Dup/Ddw: bath energies of the up/down word (HxVbath.f90), Dimp: impurity-only
// terms (HxVimp.f90 diagonal, HxVint.f90), the hops: impurity<->bath V and
// inter-orbital Hloc (HxVimp_bath.f90, HxVimp.f90:16-49).  Spin-exchange and
// pair-hopping (Jhflag) couple up and down words and are added by a separate
// gather term.
//
// One CTA owns NC consecutive columns at a time: it stages them in shared
// memory (one coalesced HBM read of V), applies the up hops as gathers from
// shared memory (random within a column), and streams the down-hop neighbour
// columns with coalesced loads (served from L2 for most of them, since every
// column is the neighbour of ~Nbath others).  Output is written once.
//
// Fused Lanczos step (LZ): with stored vectors s_k and scales sc_k (v_k =
// sc_k s_k), writes u = sc_k H s_k - beta_k sc_{k-1} s_{k-1} and the grid sum
// alpha_k = <v_k, u> (compensated FP64), so one pass over HBM produces both.
#pragma once
#include "internal.cuh"
#include "reduce.cuh"

namespace dmfted {

template <typename T>
struct HxvArgs {
    int64_t dimup, dimdw;
    int norb, P, W;
    const uint32_t *wu, *wd;   // words of the up / down class
    const T *du, *dd;          // bath-energy diagonal per word
    const uint8_t *cu, *cd;    // hop counts
    const uint32_t *eu, *ed;   // ELL (row stride dimup / dimdw)
    const T *pu, *pd;          // coupling values
    const T *dint;             // (1<<norb)^2 impurity diagonal
    const uint32_t *eux;       // lean gather table of the row class (stride dimup)
    int ku_max, kd_max;        // most hops of a row word / of a column word
    int dswap;                 // rows are down words: dint is indexed [dw][up]
    const T *x;
    T *y;
    int64_t vstride;           // batched plain products: elements between vectors
    int nstack;                // copies of the sector stacked as extra columns
                               // (a complex vector = re and im halves, since H is real)
    // fused Lanczos step
    const T *xprev;
    double *alpha, *beta, *scale;
    int *status;
    int k;
    double *partials;
    unsigned *counter;
};

template <typename T>
HxvArgs<T> make_hxv_args(const dmfted_ctx *c, const SectorView &s);

}  // namespace dmfted
