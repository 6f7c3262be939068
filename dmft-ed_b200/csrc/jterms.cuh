// The spin-exchange and pair-hopping terms of the Jhflag interaction
// (HxVint.f90:45-97), the only off-diagonal terms that change the up and the
// down word of a state together:
//   S-E: Jx c^+_{a up} c^+_{b dw} c_{a dw} c_{b up}   (a != b)
//   P-H: Jp c^+_{a up} c^+_{a dw} c_{b dw} c_{b up}   (a != b)
// On a state with up word wu and down word wd, S-E moves the up electron b -> a
// and the down electron a -> b; P-H moves both from b to a.  The sign of the
// four Jordan-Wigner operators on the combined 2Ns-bit word is the product of
// the two one-spin hop signs (the other spin's occupations enter twice and
// cancel), each (-1)^(occupied levels of that word passed by the hop).
#pragma once
#include <cstdint>

namespace dmfted {

// Sign of c^+_a c_b on a word w with bit b set and bit a clear.
__host__ __device__ inline double jw_hop_sign(uint32_t w, int b, int a) {
    const uint32_t w1 = w & ~(1u << b);
#ifdef __CUDA_ARCH__
    const int p = __popc(w & ((1u << b) - 1u)) + __popc(w1 & ((1u << a) - 1u));
#else
    const int p = __builtin_popcount(w & ((1u << b) - 1u)) + __builtin_popcount(w1 & ((1u << a) - 1u));
#endif
    return (p & 1) ? -1.0 : 1.0;
}

// Calls f(tu, td, coef) for every S-E / P-H term of the state (wu, wd): the
// target words and the matrix element <target|H|state> = coef.
template <typename F>
__host__ __device__ inline void for_jterms(uint32_t wu, uint32_t wd, int norb, double jx, double jp,
                                           F f) {
    for (int a = 0; a < norb; a++)
        for (int b = 0; b < norb; b++) {
            if (a == b) continue;
            const uint32_t ma = 1u << a, mb = 1u << b;
            if (!(wu & mb) || (wu & ma)) continue;  // up: b occupied, a empty
            const uint32_t tu = (wu & ~mb) | ma;
            const double su = jw_hop_sign(wu, b, a);
            if (jx != 0.0 && (wd & ma) && !(wd & mb))
                f(tu, (wd & ~ma) | mb, jx * su * jw_hop_sign(wd, a, b));
            if (jp != 0.0 && (wd & mb) && !(wd & ma))
                f(tu, (wd & ~mb) | ma, jp * su * jw_hop_sign(wd, b, a));
        }
}

}  // namespace dmfted
