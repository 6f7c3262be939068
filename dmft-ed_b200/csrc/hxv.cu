// Kernels and launchers of the factored H*v; see hxv.cuh for the formulation.
#include <algorithm>
#include <cstring>

#include "hxv.cuh"
#include "jterms.cuh"

namespace dmfted {

// Vector helpers: VW consecutive elements, 16-byte aligned when VW > 1.
template <typename E, int VW>
__device__ __forceinline__ void vld(const E *p, E (&v)[VW]) {
    if constexpr (VW == 1) {
        v[0] = p[0];
    } else if constexpr (sizeof(E) * VW == 16) {
        const uint4 q = *reinterpret_cast<const uint4 *>(p);
        memcpy(v, &q, 16);
    } else if constexpr (sizeof(E) * VW == 8) {
        const uint2 q = *reinterpret_cast<const uint2 *>(p);
        memcpy(v, &q, 8);
    } else if constexpr (sizeof(E) * VW == 4) {
        const unsigned q = *reinterpret_cast<const unsigned *>(p);
        memcpy(v, &q, 4);
    } else {
        const unsigned short q = *reinterpret_cast<const unsigned short *>(p);
        memcpy(v, &q, 2);
    }
}
template <typename E, int VW>
__device__ __forceinline__ void vst(E *p, const E (&v)[VW]) {
    if constexpr (VW == 1) {
        p[0] = v[0];
    } else if constexpr (sizeof(E) * VW == 16) {
        uint4 q;
        memcpy(&q, v, 16);
        *reinterpret_cast<uint4 *>(p) = q;
    } else {
        uint2 q;
        memcpy(&q, v, 8);
        *reinterpret_cast<uint2 *>(p) = q;
    }
}

// Occupancy: 3 CTAs of 256 threads per SM (register cap 85) measured best on
// B200 for the Ns=14 sectors; the down-hop load batch is 8 columns for FP32
// and 4 for FP64 (register pressure).
constexpr int kHxvMinBlocks = 3;
template <typename T>
constexpr int dw_batch() { return sizeof(T) == 8 ? 4 : 8; }
constexpr int kUpBatch = 8;  // hopping-table entries prefetched per row vector

// Loads of neighbour columns: cached in L2 only (no reuse inside the CTA, and
// L1 is kept for the hopping tables).  Output stores: evict-first, so the
// input vector stays resident in L2 for the neighbour reads of other CTAs.
template <typename E, int VW>
__device__ __forceinline__ void vld_cg(const E *p, E (&v)[VW]) {
    if constexpr (sizeof(E) * VW == 16) {
        const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(p));
        memcpy(v, &q, 16);
    } else if constexpr (sizeof(E) * VW == 8) {
        const uint2 q = __ldcg(reinterpret_cast<const uint2 *>(p));
        memcpy(v, &q, 8);
    } else if constexpr (sizeof(E) * VW == 4) {
        const unsigned q = __ldcg(reinterpret_cast<const unsigned *>(p));
        memcpy(v, &q, 4);
    } else {
        v[0] = __ldcg(p);
    }
}
template <typename E, int VW>
__device__ __forceinline__ void vst_cs(E *p, const E (&v)[VW]) {
    if constexpr (sizeof(E) * VW == 16) {
        uint4 q;
        memcpy(&q, v, 16);
        __stcs(reinterpret_cast<uint4 *>(p), q);
    } else if constexpr (sizeof(E) * VW == 8) {
        uint2 q;
        memcpy(&q, v, 8);
        __stcs(reinterpret_cast<uint2 *>(p), q);
    } else if constexpr (sizeof(E) * VW == 4) {
        unsigned q;
        memcpy(&q, v, 4);
        __stcs(reinterpret_cast<unsigned *>(p), q);
    } else {
        __stcs(p, v[0]);
    }
}

// Streaming load (last use: evict first) and an L2-resident store.
template <typename E, int VW>
__device__ __forceinline__ void vld_cs(const E *p, E (&v)[VW]) {
    static_assert(sizeof(E) * VW == 8 || sizeof(E) * VW == 16, "8- or 16-byte vectors");
    if constexpr (sizeof(E) * VW == 16) {
        const uint4 q = __ldcs(reinterpret_cast<const uint4 *>(p));
        memcpy(v, &q, 16);
    } else {
        const uint2 q = __ldcs(reinterpret_cast<const uint2 *>(p));
        memcpy(v, &q, 8);
    }
}
template <typename E, int VW>
__device__ __forceinline__ void vst_cg(E *p, const E (&v)[VW]) {
    static_assert(sizeof(E) * VW == 8 || sizeof(E) * VW == 16, "8- or 16-byte vectors");
    if constexpr (sizeof(E) * VW == 16) {
        uint4 q;
        memcpy(&q, v, 16);
        __stcg(reinterpret_cast<uint4 *>(p), q);
    } else {
        uint2 q;
        memcpy(&q, v, 8);
        __stcg(reinterpret_cast<uint2 *>(p), q);
    }
}

// Factored H*v.  A CTA owns a tile of NC consecutive columns, staged in
// shared memory row-interleaved (xs[row*NC + j]) so that one up-hop gather is
// a single NC-wide load serving all NC columns.  Each thread owns VW
// consecutive rows per pass (16-byte global loads and stores).  The down hops
// stream whole neighbour columns from L2/HBM with kDwBatch loads in flight.
template <typename T, int NC, int VW, bool LZ>
__global__ void __launch_bounds__(256, kHxvMinBlocks) k_hxv(const HxvArgs<T> a) {
    constexpr int kDwBatch = dw_batch<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T spu[kMaxParams];
    __shared__ T sdint[64];
    __shared__ T sdd[NC];
    __shared__ unsigned simp[NC];
    __shared__ int scnt[NC];
    __shared__ T sval[NC][kMaxW];
    __shared__ int64_t soff[NC][kMaxW];

    if (LZ) {
        if (a.status[0]) return;  // chain finished: every later step is a no-op
    }
    const int tid = threadIdx.x, bd = blockDim.x;
    const int64_t dimup = a.dimup, dimdw = a.dimdw, ncols = dimdw * a.nstack;
    for (int i = tid; i < a.P; i += bd) spu[i] = a.pu[i];
    const int ni = 1 << a.norb;
    for (int i = tid; i < ni * ni; i += bd) sdint[i] = a.dint[a.dswap ? (i % ni) * ni + i / ni : i];
    const unsigned imask = (unsigned)ni - 1u;

    double sc = 1.0, cprev = 0.0;
    if (LZ) {
        sc = a.scale[a.k];
        cprev = a.k > 0 ? a.beta[a.k] * a.scale[a.k - 1] : 0.0;
    }
    // u = sc*acc - cprev*xprev in the vector precision; for FP32 vectors both
    // scalars are split into a float pair (hi + lo) so that they enter with
    // full FP64 accuracy and only the final fused multiply-add rounds.
    const T sch = (T)sc, scl = (T)(sc - (double)sch);
    const T cph = (T)cprev, cpl = (T)(cprev - (double)cph);
    const T *x = a.x + (int64_t)blockIdx.y * a.vstride;
    T *y = a.y + (int64_t)blockIdx.y * a.vstride;
    T *xs = reinterpret_cast<T *>(smem_raw);  // [dimup][NC]
    CSum dot;
    dot.zero();

    for (int64_t c0 = (int64_t)blockIdx.x * NC; c0 < ncols; c0 += (int64_t)gridDim.x * NC) {
        const int nc = (int)min((int64_t)NC, ncols - c0);
        __syncthreads();
        // stage the tile: NC column loads per row vector, transposed in registers
        for (int64_t r = (int64_t)tid * VW; r < dimup; r += (int64_t)bd * VW) {
            T v[NC][VW];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                if (j < nc && DM_IN((c0 + j) * dimup + r + VW - 1, ncols * dimup)) {
                    vld<T, VW>(x + (c0 + j) * dimup + r, v[j]);
                } else {
#pragma unroll
                    for (int i = 0; i < VW; i++) v[j][i] = T(0);
                }
            }
#pragma unroll
            for (int i = 0; i < VW; i++) {
                T row[NC];
#pragma unroll
                for (int j = 0; j < NC; j++) row[j] = v[j][i];
                if (DM_IN((r + i) * NC + NC - 1, dimup * NC)) vst<T, NC>(xs + (r + i) * NC, row);
            }
        }
        // column data and decoded down hops (value, element offset of the
        // neighbour column)
        if (tid < nc) {
            const int64_t cg = c0 + tid, q = cg / dimdw;
            const int64_t cc = DM_IN(cg - q * dimdw, dimdw) ? cg - q * dimdw : 0;
            scnt[tid] = a.cd[cc];
            simp[tid] = a.wd[cc] & imask;
            sdd[tid] = a.dd[cc];
        } else if (tid < NC) {
            // unused columns of a partial tile: defined values, never stored
            scnt[tid] = 0;
            simp[tid] = 0;
            sdd[tid] = T(0);
        }
        for (int t = tid; t < nc * a.W; t += bd) {
            const int j = t / a.W, e = t % a.W;
            const int64_t cg = c0 + j, q = cg / dimdw, cc = cg - q * dimdw;
            if (e < (int)a.cd[cc] && DM_IN(e, kMaxW) && DM_IN(e, a.W)) {
                const uint32_t en = a.ed[(int64_t)e * dimdw + cc];
                const bool ok = DM_IN(ell_par(en), a.P) && DM_IN(ell_col(en), dimdw);
                T v = ok ? a.pd[ell_par(en)] : T(0);
                sval[j][e] = ell_neg(en) ? -v : v;
                soff[j][e] = ok ? (q * dimdw + (int64_t)ell_col(en)) * dimup : 0;
            }
        }
        __syncthreads();
        for (int64_t r = (int64_t)tid * VW; r < dimup; r += (int64_t)bd * VW) {
            uint32_t wu[VW];
            T du[VW];
            uint8_t cu[VW];
            if (!DM_IN(r + VW - 1, dimup)) break;
            vld<uint32_t, VW>(a.wu + r, wu);
            vld<T, VW>(a.du + r, du);
            vld<uint8_t, VW>(a.cu + r, cu);
            T acc[NC][VW];
            int cmax = 0;
#pragma unroll
            for (int i = 0; i < VW; i++) {
                cmax = max(cmax, (int)cu[i]);
                T xr[NC];
                vld<T, NC>(xs + (r + i) * NC, xr);
#pragma unroll
                for (int j = 0; j < NC; j++)
                    acc[j][i] = (du[i] + sdd[j] + sdint[(wu[i] & imask) * ni + (simp[j] & imask)]) * xr[j];
            }
            // up hops: table entries prefetched, then NC-wide gathers
            for (int e0 = 0; e0 < cmax; e0 += kUpBatch) {
                uint32_t en[kUpBatch][VW];
#pragma unroll
                for (int q = 0; q < kUpBatch; q++)
                    if (e0 + q < cmax && DM_IN(e0 + q, a.W))
                        vld<uint32_t, VW>(a.eu + (int64_t)(e0 + q) * dimup + r, en[q]);
#pragma unroll
                for (int q = 0; q < kUpBatch; q++) {
#pragma unroll
                    for (int i = 0; i < VW; i++) {
                        if (e0 + q < (int)cu[i] && DM_IN(ell_col(en[q][i]), dimup) &&
                            DM_IN(ell_par(en[q][i]), a.P)) {
                            T v = spu[ell_par(en[q][i])];
                            if (ell_neg(en[q][i])) v = -v;
                            T xg[NC];
                            vld<T, NC>(xs + (int64_t)ell_col(en[q][i]) * NC, xg);
#pragma unroll
                            for (int j = 0; j < NC; j++) acc[j][i] += v * xg[j];
                        }
                    }
                }
            }
            // down hops: whole neighbour columns, loads batched for MLP
#pragma unroll
            for (int j = 0; j < NC; j++) {
                if (j < nc) {
                    const int ce = scnt[j];
                    const int64_t idx = (c0 + j) * dimup + r;
                    // v_{k-1} is loaded ahead of the down hops so that its
                    // latency overlaps theirs (except FP64 two-row vectors,
                    // where the extra live registers spill)
                    constexpr bool kEarly = !(sizeof(T) == 8 && VW == 2);
                    T xp[VW];
                    if (LZ && kEarly) {
                        if (DM_IN(idx + VW - 1, ncols * dimup)) vld<T, VW>(a.xprev + idx, xp);
                    }
                    for (int e0 = 0; e0 < ce; e0 += kDwBatch) {
                        T xv[kDwBatch][VW];
#pragma unroll
                        for (int q = 0; q < kDwBatch; q++)
                            if (e0 + q < ce && DM_IN(soff[j][e0 + q] + r + VW - 1, ncols * dimup))
                                vld_cg<T, VW>(x + soff[j][e0 + q] + r, xv[q]);
#pragma unroll
                        for (int q = 0; q < kDwBatch; q++)
                            if (e0 + q < ce) {
                                const T v = sval[j][e0 + q];
#pragma unroll
                                for (int i = 0; i < VW; i++) acc[j][i] += v * xv[q][i];
                            }
                    }
                    if (!DM_IN(idx + VW - 1, ncols * dimup)) continue;
                    if (LZ) {
                        if (!kEarly) vld<T, VW>(a.xprev + idx, xp);
#pragma unroll
                        for (int i = 0; i < VW; i++) {
                            if constexpr (sizeof(T) == 8) {
                                acc[j][i] = sc * acc[j][i] - cprev * xp[i];
                            } else {
                                T t = -cpl * xp[i];
                                t = fmaf(-cph, xp[i], t);
                                t = fmaf(scl, acc[j][i], t);
                                acc[j][i] = fmaf(sch, acc[j][i], t);
                            }
                        }
                    }
                    vst_cs<T, VW>(y + idx, acc[j]);
                }
            }
            if (LZ) {
                // <x, u> over this row vector: the staged rows are re-read
                // as NC-wide vectors; products of two floats are exact in
                // FP64, and one compensated add per row vector
                double part = 0.0;
#pragma unroll
                for (int i = 0; i < VW; i++) {
                    T xr[NC];
                    vld<T, NC>(xs + (r + i) * NC, xr);
#pragma unroll
                    for (int j = 0; j < NC; j++)
                        if (j < nc) part = fma((double)xr[j], (double)acc[j][i], part);
                }
                dot.add(part);
            }
        }
    }
    if (LZ) {
        CSum arr[1] = {dot};
        double tot[1];
        if (grid_reduce<1>(arr, a.partials, a.counter, tot)) {
            if (tid == 0) a.alpha[a.k] = sc * tot[0];
        }
    }
}

// ---------------------------------------------------------------------------
// k_hxv_rv: the same product with the global loads of a row vector issued
// together.  Each thread owns two consecutive rows (r, r+1) of the NC-column
// tile per pass.  Before any shared-memory work it issues, at once, the
// down-hop neighbour loads of all NC columns (up to kRvDw per column, held in
// registers), the v_{k-1} rows and the hopping-table entries of its rows; the
// diagonal and the up-hop gathers from shared memory then run while those
// loads are in flight, and the neighbour values are consumed last.  One L2
// round trip per row vector instead of one per column (the v_{k-1} rows are
// issued after the up hops, where the hop-table registers are free).
//
// Shared-memory traffic per row vector is cut to what the gathers need:
//  * the down-hop offsets and couplings of the tile are read as 16-byte
//    broadcasts (uint4 / T4), four or two hops per read;
//  * the column part of the diagonal (bath energies of the down word plus
//    the impurity term for each impurity up-state) is one table per column,
//    cdg[j][iu];
//  * the two rows' 16-byte accesses to the staged tile are ordered per lane
//    (lanes 4..7 of each quarter warp take row r+1 first), so each quarter
//    warp touches eight distinct bank quads.
constexpr int kRvDw = 8;      // down-hop neighbour loads per column held in registers
constexpr int kRvUp = 8;      // hopping-table entries per row loaded ahead
constexpr int kRvBlocks = 2;  // CTAs of 256 threads per SM (register budget 128)

template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};

template <typename T, bool LZ>
__global__ void __launch_bounds__(256, kRvBlocks) k_hxv_rv(const HxvArgs<T> a) {
    constexpr int NC = 16 / sizeof(T);
    constexpr int KD = kRvDw, KU = kRvUp;
    using T2 = typename Pair<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T spu[kMaxParams];
    __shared__ __align__(16) T cdg[NC][1 << kMaxNorb];
    __shared__ __align__(16) uint32_t noff[NC][kMaxW];
    __shared__ __align__(16) T nval[NC][kMaxW];
    __shared__ int scnt[NC];

    if (LZ) {
        if (a.status[0]) return;  // chain finished: every later step is a no-op
    }
    const int tid = threadIdx.x, bd = blockDim.x;
    const int sw = (tid >> 2) & 1;  // this lane's row order for 16-byte tile accesses
    const int64_t dimup = a.dimup, dimdw = a.dimdw, ncols = dimdw * a.nstack;
    const int64_t total = ncols * dimup;
    (void)total;  // bounds of the checked build
    for (int i = tid; i < a.P; i += bd) spu[i] = a.pu[i];
    const int ni = 1 << a.norb;
    const unsigned imask = (unsigned)ni - 1u;
    const int W = a.W, WW = W > KD ? W : KD;

    double sc = 1.0, cprev = 0.0;
    if (LZ) {
        sc = a.scale[a.k];
        cprev = a.k > 0 ? a.beta[a.k] * a.scale[a.k - 1] : 0.0;
    }
    const T sch = (T)sc, scl = (T)(sc - (double)sch);
    const T cph = (T)cprev, cpl = (T)(cprev - (double)cph);
    const T *x = a.x + (int64_t)blockIdx.y * a.vstride;
    T *y = a.y + (int64_t)blockIdx.y * a.vstride;
    const T *xprev = LZ ? a.xprev + (int64_t)blockIdx.y * a.vstride : nullptr;
    T *xs = reinterpret_cast<T *>(smem_raw);  // [dimup][NC]
    CSum dot;
    dot.zero();

    for (int64_t c0 = (int64_t)blockIdx.x * NC; c0 < ncols; c0 += (int64_t)gridDim.x * NC) {
        const int nc = (int)min((int64_t)NC, ncols - c0);
        __syncthreads();
        // stage the tile (rows r and r+1 of NC columns), transposed in registers
        for (int64_t r = (int64_t)tid * 2; r < dimup; r += (int64_t)bd * 2) {
            T2 v[NC];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                const int64_t idx = (c0 + j) * dimup + r;
                if (j < nc && DM_IN(idx + 1, total))
                    v[j] = *reinterpret_cast<const T2 *>(x + idx);
                else
                    v[j].x = v[j].y = T(0);
            }
            T ra[NC], rb[NC];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                ra[j] = sw ? v[j].y : v[j].x;
                rb[j] = sw ? v[j].x : v[j].y;
            }
            if (DM_IN((r + 1) * NC + NC - 1, dimup * NC)) {
                vst<T, NC>(xs + (r + sw) * NC, ra);
                vst<T, NC>(xs + (r + 1 - sw) * NC, rb);
            }
        }
        // column tables: diagonal per impurity up-state, down-hop offsets and
        // couplings (zero for the unused slots and the columns of a partial tile)
        if (tid < NC) {
            int cnt = 0;
            if (tid < nc) {
                const int64_t cg = c0 + tid, q = cg / dimdw;
                const int64_t cc = DM_IN(cg - q * dimdw, dimdw) ? cg - q * dimdw : 0;
                cnt = a.cd[cc];
                const unsigned id = a.wd[cc] & imask;
                const T dd = a.dd[cc];
                for (int iu = 0; iu < ni; iu++)
                    cdg[tid][iu] = dd + a.dint[a.dswap ? id * ni + iu : iu * ni + id];
            } else {
                for (int iu = 0; iu < ni; iu++) cdg[tid][iu] = T(0);
            }
            scnt[tid] = cnt;
        }
        for (int t = tid; t < NC * WW; t += bd) {
            const int j = t / WW, e = t % WW;
            uint32_t off = 0;
            T v = T(0);
            if (j < nc && e < W) {
                const int64_t cg = c0 + j, q = cg / dimdw, cc = cg - q * dimdw;
                if (e < (int)a.cd[cc] && DM_IN(e, kMaxW)) {
                    const uint32_t en = a.ed[(int64_t)e * dimdw + cc];
                    const bool ok = DM_IN(ell_par(en), a.P) && DM_IN(ell_col(en), dimdw);
                    v = ok ? a.pd[ell_par(en)] : T(0);
                    if (ell_neg(en)) v = -v;
                    off = ok ? (uint32_t)((q * dimdw + (int64_t)ell_col(en)) * dimup) : 0u;
                }
            }
            if (DM_IN(e, kMaxW)) {
                noff[j][e] = off;
                nval[j][e] = v;
            }
        }
        __syncthreads();
        for (int64_t r = (int64_t)tid * 2; r < dimup; r += (int64_t)bd * 2) {
            // 1. global loads: neighbour rows of every column, v_{k-1}, hop tables
            int cnts[NC];
            T2 nb[NC][KD];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                cnts[j] = scnt[j];
                uint32_t o[KD];
#pragma unroll
                for (int e = 0; e < KD; e += 4) {
                    const uint4 q4 = *reinterpret_cast<const uint4 *>(&noff[j][e]);
                    o[e] = q4.x;
                    o[e + 1] = q4.y;
                    o[e + 2] = q4.z;
                    o[e + 3] = q4.w;
                }
#pragma unroll
                for (int e = 0; e < KD; e++) {
                    if (e < cnts[j] && DM_IN(o[e] + r + 1, total)) {
                        T t2[2];
                        vld_cg<T, 2>(x + o[e] + r, t2);
                        nb[j][e].x = t2[0];
                        nb[j][e].y = t2[1];
                    } else {
                        nb[j][e].x = nb[j][e].y = T(0);
                    }
                }
            }
            const unsigned short cu2 = *reinterpret_cast<const unsigned short *>(a.cu + r);
            const int cu0 = cu2 & 0xff, cu1 = cu2 >> 8;
            const int cmax = max(cu0, cu1);
            uint2 en[KU];
#pragma unroll
            for (int q = 0; q < KU; q++) {
                if (q < cmax && DM_IN(q, W))
                    en[q] = *reinterpret_cast<const uint2 *>(a.eu + (int64_t)q * dimup + r);
                else
                    en[q] = make_uint2(0u, 0u);
            }
            const uint2 wu2 = *reinterpret_cast<const uint2 *>(a.wu + r);
            const T2 du2 = *reinterpret_cast<const T2 *>(a.du + r);

            // 2. diagonal from the staged tile
            T acc[NC][2];
            {
                T x0[NC], x1[NC];
                T xa[NC], xb[NC];
                vld<T, NC>(xs + (r + sw) * NC, xa);
                vld<T, NC>(xs + (r + 1 - sw) * NC, xb);
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    x0[j] = sw ? xb[j] : xa[j];
                    x1[j] = sw ? xa[j] : xb[j];
                }
                const unsigned iu0 = wu2.x & imask, iu1 = wu2.y & imask;
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    acc[j][0] = (du2.x + cdg[j][iu0]) * x0[j];
                    acc[j][1] = (du2.y + cdg[j][iu1]) * x1[j];
                }
            }
            // 3. up hops: NC-wide gathers from the tile
#pragma unroll
            for (int q = 0; q < KU; q++) {
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    const uint32_t e = i ? en[q].y : en[q].x;
                    if (q < (i ? cu1 : cu0) && DM_IN(ell_col(e), dimup) && DM_IN(ell_par(e), a.P)) {
                        T v = spu[ell_par(e)];
                        if (ell_neg(e)) v = -v;
                        T xg[NC];
                        vld<T, NC>(xs + (int64_t)ell_col(e) * NC, xg);
#pragma unroll
                        for (int j = 0; j < NC; j++) acc[j][i] += v * xg[j];
                    }
                }
            }
            for (int q = KU; q < cmax && q < W; q++) {
                const uint2 e2 = *reinterpret_cast<const uint2 *>(a.eu + (int64_t)q * dimup + r);
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    const uint32_t e = i ? e2.y : e2.x;
                    if (q < (i ? cu1 : cu0) && DM_IN(ell_col(e), dimup) && DM_IN(ell_par(e), a.P)) {
                        T v = spu[ell_par(e)];
                        if (ell_neg(e)) v = -v;
                        T xg[NC];
                        vld<T, NC>(xs + (int64_t)ell_col(e) * NC, xg);
#pragma unroll
                        for (int j = 0; j < NC; j++) acc[j][i] += v * xg[j];
                    }
                }
            }
            // v_{k-1} rows: issued here, where the hop-table registers are free
            T2 xp[NC];
            if (LZ) {
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    const int64_t idx = (c0 + j) * dimup + r;
                    if (j < nc && DM_IN(idx + 1, total))
                        xp[j] = *reinterpret_cast<const T2 *>(xprev + idx);
                    else
                        xp[j].x = xp[j].y = T(0);
                }
            }
            // 4. down hops: consume the neighbour rows, stream any beyond KD
#pragma unroll
            for (int j = 0; j < NC; j++) {
                constexpr int NV = 16 / sizeof(T);
                T vv[KD];
#pragma unroll
                for (int e = 0; e < KD; e += NV) {
                    T t4[NV];
                    vld<T, NV>(&nval[j][e], t4);
#pragma unroll
                    for (int i = 0; i < NV; i++) vv[e + i] = t4[i];
                }
#pragma unroll
                for (int e = 0; e < KD; e++) {
                    acc[j][0] += vv[e] * nb[j][e].x;
                    acc[j][1] += vv[e] * nb[j][e].y;
                }
                for (int e = KD; e < cnts[j] && e < W; e++) {
                    const uint32_t o = noff[j][e];
                    if (!DM_IN(o + r + 1, total)) continue;
                    T xv[2];
                    vld_cg<T, 2>(x + o + r, xv);
                    const T v = nval[j][e];
                    acc[j][0] += v * xv[0];
                    acc[j][1] += v * xv[1];
                }
            }
            // 5. Lanczos combination, store, alpha partial (the rows' own
            // values re-read from the tile)
            double part = 0.0;
            T x0[NC], x1[NC];
            if (LZ) {
                T xa[NC], xb[NC];
                vld<T, NC>(xs + (r + sw) * NC, xa);
                vld<T, NC>(xs + (r + 1 - sw) * NC, xb);
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    x0[j] = sw ? xb[j] : xa[j];
                    x1[j] = sw ? xa[j] : xb[j];
                }
            }
#pragma unroll
            for (int j = 0; j < NC; j++) {
                if (j >= nc) continue;
                const int64_t idx = (c0 + j) * dimup + r;
                if (!DM_IN(idx + 1, total)) continue;
                if (LZ) {
                    const T xpv[2] = {xp[j].x, xp[j].y};
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        if constexpr (sizeof(T) == 8) {
                            acc[j][i] = sc * acc[j][i] - cprev * xpv[i];
                        } else {
                            T t = -cpl * xpv[i];
                            t = fmaf(-cph, xpv[i], t);
                            t = fmaf(scl, acc[j][i], t);
                            acc[j][i] = fmaf(sch, acc[j][i], t);
                        }
                    }
                    part = fma((double)x0[j], (double)acc[j][0], part);
                    part = fma((double)x1[j], (double)acc[j][1], part);
                }
                vst_cs<T, 2>(y + idx, acc[j]);
            }
            if (LZ) dot.add(part);
        }
    }
    if (LZ) {
        CSum arr[1] = {dot};
        double tot[1];
        if (grid_reduce<1>(arr, a.partials, a.counter, tot)) {
            if (tid == 0) a.alpha[a.k] = sc * tot[0];
        }
    }
}

// ---------------------------------------------------------------------------
// k_hxv_lean: k_hxv_rv with the per-element instruction count cut down, for
// sectors whose words have at most 8 hops per spin (every sector of the
// single-orbital baths up to Nbath = 15 at and near half filling).
//  * Row hops come from the gather table `ellx` (built from the balanced ELL
//    table): each entry is the shared-memory byte offset of the target row
//    (bits 0..23) and an index into a signed-coupling table (bits 24..31,
//    2p for +V_p, 2p+1 for -V_p, kLeanZero for 0).  A row with fewer than KU
//    hops is padded with zero-coupling entries that point at the row itself,
//    so the hop loop has a fixed length and no predicates.
//  * Column hops are padded the same way to KD per column (padding points at
//    the column's own data with a zero coupling).
//  * Row and element indices are 32-bit (the stacked vector has fewer than
//    2^32 elements).
// KU, KD: hops per row / per column after padding (7 or 8).
constexpr uint32_t kLeanZero = 255u;

// MODE 0: plain product; 1: fused Lanczos step (u and its alpha).  MB: CTAs
// of 256 threads per SM the register budget is set for.
template <typename T, int KU, int KD, int MODE, int MB = kRvBlocks>
__global__ void __launch_bounds__(256, MB) k_hxv_lean(const HxvArgs<T> a,
                                                    const uint32_t *__restrict__ eux) {
    constexpr bool LZ = MODE >= 1;
    constexpr int NC = 16 / sizeof(T);
    constexpr int NV = 16 / sizeof(T);
    using T2 = typename Pair<T>::type;
    static_assert(KU <= 8 && KD <= 8, "hop counts above 8 use k_hxv_rv");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T spv[256];
    __shared__ __align__(16) T cdg[NC][1 << kMaxNorb];
    __shared__ __align__(16) uint32_t noff[NC][8];
    __shared__ __align__(16) T nval[NC][8];

    if (LZ) {
        if (a.status[0]) return;  // chain finished: every later step is a no-op
    }
    const int tid = threadIdx.x, bd = blockDim.x;
    const int sw = (tid >> 2) & 1;  // this lane's row order for 16-byte tile accesses
    const uint32_t dimup = (uint32_t)a.dimup, dimdw = (uint32_t)a.dimdw;
    const uint32_t ncols = dimdw * (uint32_t)a.nstack;
    const uint32_t total = ncols * dimup;
    (void)total;  // bounds of the checked build
    for (int i = tid; i < 256; i += bd) {
        T v = T(0);
        if (i < 2 * a.P && i != (int)kLeanZero) {
            v = a.pu[i >> 1];
            if (i & 1) v = -v;
        }
        spv[i] = v;
    }
    const int ni = 1 << a.norb;
    const unsigned imask = (unsigned)ni - 1u;

    double sc = 1.0, cprev = 0.0;
    if (LZ) {
        sc = a.scale[a.k];
        cprev = a.k > 0 ? a.beta[a.k] * a.scale[a.k - 1] : 0.0;
    }
    const T sch = (T)sc, scl = (T)(sc - (double)sch);
    const T cph = (T)cprev, cpl = (T)(cprev - (double)cph);
    const T *x = a.x + (int64_t)blockIdx.y * a.vstride;
    T *y = a.y + (int64_t)blockIdx.y * a.vstride;
    const T *xprev = LZ ? a.xprev + (int64_t)blockIdx.y * a.vstride : nullptr;
    T *xs = reinterpret_cast<T *>(smem_raw);  // [dimup][NC]
    const unsigned char *xsb = smem_raw;
    CSum dot;
    dot.zero();

    for (uint32_t c0 = blockIdx.x * NC; c0 < ncols; c0 += gridDim.x * NC) {
        const int nc = (int)min((uint32_t)NC, ncols - c0);
        __syncthreads();
        // stage the tile (rows r and r+1 of NC columns), transposed in registers
        for (uint32_t r = tid * 2; r < dimup; r += bd * 2) {
            T2 v[NC];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                const uint32_t idx = (c0 + j) * dimup + r;
                if (j < nc && DM_IN(idx + 1, total))
                    v[j] = *reinterpret_cast<const T2 *>(x + idx);
                else
                    v[j].x = v[j].y = T(0);
            }
            T ra[NC], rb[NC];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                ra[j] = sw ? v[j].y : v[j].x;
                rb[j] = sw ? v[j].x : v[j].y;
            }
            if (DM_IN((r + 1) * NC + NC - 1, dimup * NC)) {
                vst<T, NC>(xs + (r + sw) * NC, ra);
                vst<T, NC>(xs + (r + 1 - sw) * NC, rb);
            }
        }
        // column tables; padding and the columns of a partial tile read the
        // last real column of the tile with a zero coupling
        if (tid < NC) {
            if (tid < nc) {
                const uint32_t cg = c0 + tid, q = cg / dimdw;
                const uint32_t cc = DM_IN(cg - q * dimdw, dimdw) ? cg - q * dimdw : 0u;
                const unsigned id = a.wd[cc] & imask;
                const T dd = a.dd[cc];
                for (int iu = 0; iu < ni; iu++)
                    cdg[tid][iu] = dd + a.dint[a.dswap ? id * ni + iu : iu * ni + id];
            } else {
                for (int iu = 0; iu < ni; iu++) cdg[tid][iu] = T(0);
            }
        }
        for (int t = tid; t < NC * 8; t += bd) {
            const int j = t >> 3, e = t & 7;
            const uint32_t jl = (uint32_t)min(j, nc - 1);
            uint32_t off = (c0 + jl) * dimup;
            T v = T(0);
            if (j < nc && e < KD) {
                const uint32_t cg = c0 + j, q = cg / dimdw, cc = cg - q * dimdw;
                if (e < (int)a.cd[cc] && DM_IN(e, a.W)) {
                    const uint32_t en = a.ed[(int64_t)e * dimdw + cc];
                    const bool ok = DM_IN(ell_par(en), a.P) && DM_IN(ell_col(en), dimdw);
                    if (ok) {
                        v = a.pd[ell_par(en)];
                        if (ell_neg(en)) v = -v;
                        off = (q * dimdw + ell_col(en)) * dimup;
                    }
                }
            }
            noff[j][e] = off;
            nval[j][e] = v;
        }
        __syncthreads();
        for (uint32_t r = tid * 2; r < dimup; r += bd * 2) {
            // 1. global loads: neighbour rows of every column, hop tables
            T2 nb[NC][KD];
#pragma unroll
            for (int j = 0; j < NC; j++) {
                uint32_t o[8];
                const uint4 q0 = *reinterpret_cast<const uint4 *>(&noff[j][0]);
                const uint4 q1 = *reinterpret_cast<const uint4 *>(&noff[j][4]);
                o[0] = q0.x; o[1] = q0.y; o[2] = q0.z; o[3] = q0.w;
                o[4] = q1.x; o[5] = q1.y; o[6] = q1.z; o[7] = q1.w;
#pragma unroll
                for (int e = 0; e < KD; e++) {
                    T t2[2];
                    if (DM_IN(o[e] + r + 1, total)) {
                        vld_cg<T, 2>(x + (o[e] + r), t2);
                    } else {
                        t2[0] = t2[1] = T(0);
                    }
                    nb[j][e].x = t2[0];
                    nb[j][e].y = t2[1];
                }
            }
            uint2 en[KU];
#pragma unroll
            for (int q = 0; q < KU; q++)
                en[q] = *reinterpret_cast<const uint2 *>(eux + (q * dimup + r));
            const uint2 wu2 = *reinterpret_cast<const uint2 *>(a.wu + r);
            const T2 du2 = *reinterpret_cast<const T2 *>(a.du + r);

            // 2. diagonal from the staged tile; the rows' own values stay in
            // registers for the alpha partial of step 5
            T acc[NC][2];
            T x0[NC], x1[NC];
            {
                T xa[NC], xb[NC];
                vld<T, NC>(xs + (r + sw) * NC, xa);
                vld<T, NC>(xs + (r + 1 - sw) * NC, xb);
                const unsigned iu0 = wu2.x & imask, iu1 = wu2.y & imask;
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    x0[j] = sw ? xb[j] : xa[j];
                    x1[j] = sw ? xa[j] : xb[j];
                    acc[j][0] = (du2.x + cdg[j][iu0]) * x0[j];
                    acc[j][1] = (du2.y + cdg[j][iu1]) * x1[j];
                }
            }
            // 3. row hops: NC-wide gathers from the tile, fixed count
#pragma unroll
            for (int q = 0; q < KU; q++) {
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    const uint32_t e = i ? en[q].y : en[q].x;
                    const T v = spv[e >> 24];
                    const uint32_t bo = e & 0xFFFFFFu;
                    T xg[NC];
                    if (DM_IN(bo / 16, dimup)) {
                        vld<T, NC>(reinterpret_cast<const T *>(xsb + bo), xg);
                    } else {
#pragma unroll
                        for (int j = 0; j < NC; j++) xg[j] = T(0);
                    }
#pragma unroll
                    for (int j = 0; j < NC; j++) acc[j][i] += v * xg[j];
                }
            }
            // v_{k-1} rows: issued here, where the hop-table registers are free
            T2 xp[NC];
            if (LZ) {
#pragma unroll
                for (int j = 0; j < NC; j++) {
                    const uint32_t idx = (c0 + (uint32_t)min(j, nc - 1)) * dimup + r;
                    if (DM_IN(idx + 1, total)) {
                        T t2[2];
                        vld_cs<T, 2>(xprev + idx, t2);  // last use of v_{k-1} in the step
                        xp[j].x = t2[0];
                        xp[j].y = t2[1];
                    } else {
                        xp[j].x = xp[j].y = T(0);
                    }
                }
            }
            // 4. column hops: consume the neighbour rows
#pragma unroll
            for (int j = 0; j < NC; j++) {
                T vv[8];
#pragma unroll
                for (int e = 0; e < 8; e += NV) {
                    T t4[NV];
                    vld<T, NV>(&nval[j][e], t4);
#pragma unroll
                    for (int i = 0; i < NV; i++) vv[e + i] = t4[i];
                }
#pragma unroll
                for (int e = 0; e < KD; e++) {
                    acc[j][0] += vv[e] * nb[j][e].x;
                    acc[j][1] += vv[e] * nb[j][e].y;
                }
            }
            // 5. Lanczos combination, store, alpha partial
            double part = 0.0;
#pragma unroll
            for (int j = 0; j < NC; j++) {
                if (j >= nc) continue;
                const uint32_t idx = (c0 + j) * dimup + r;
                if (!DM_IN(idx + 1, total)) continue;
                if (LZ) {
                    const T xpv[2] = {xp[j].x, xp[j].y};
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        if constexpr (sizeof(T) == 8) {
                            acc[j][i] = sc * acc[j][i] - cprev * xpv[i];
                        } else {
                            T t = -cpl * xpv[i];
                            t = fmaf(-cph, xpv[i], t);
                            t = fmaf(scl, acc[j][i], t);
                            acc[j][i] = fmaf(sch, acc[j][i], t);
                        }
                    }
                    part = fma((double)x0[j], (double)acc[j][0], part);
                    part = fma((double)x1[j], (double)acc[j][1], part);
                }
                vst_cs<T, 2>(y + idx, acc[j]);
            }
            if (LZ) dot.add(part);
        }
    }
    if (MODE == 1) {
        CSum arr[1] = {dot};
        double tot[1];
        if (grid_reduce<1>(arr, a.partials, a.counter, tot)) {
            if (tid == 0) a.alpha[a.k] = sc * tot[0];
        }
    }
}

// ---------------------------------------------------------------------------
// k_hxv_global: the same product for sectors whose columns do not fit in
// shared memory (DimUp x 16 bytes above the 200 KB a tile may take: Ns >= 16
// near half filling).  One thread per element, in index order (a warp holds
// consecutive rows of one column): the up hops gather from the element's own
// column in global memory (a column is at most a few hundred KB, served from
// L1/L2), the down hops read whole neighbour columns (coalesced), the tables
// are the ELL ones of the other kernels.
template <typename T, bool LZ>
__global__ void __launch_bounds__(256) k_hxv_global(const HxvArgs<T> a) {
    if (LZ) {
        if (a.status[0]) return;  // chain finished: every later step is a no-op
    }
    __shared__ T spu[kMaxParams];
    __shared__ T sdint[64];
    const int tid = threadIdx.x;
    for (int i = tid; i < a.P && i < kMaxParams; i += blockDim.x) spu[i] = a.pu[i];
    const int ni = 1 << a.norb;
    for (int i = tid; i < ni * ni; i += blockDim.x)
        sdint[i] = a.dint[a.dswap ? (i % ni) * ni + i / ni : i];
    __syncthreads();
    const unsigned imask = (unsigned)ni - 1u;
    const int64_t dimup = a.dimup, dimdw = a.dimdw, ncols = dimdw * a.nstack;
    const int64_t total = ncols * dimup;
    double sc = 1.0, cprev = 0.0;
    if (LZ) {
        sc = a.scale[a.k];
        cprev = a.k > 0 ? a.beta[a.k] * a.scale[a.k - 1] : 0.0;
    }
    const T sch = (T)sc, scl = (T)(sc - (double)sch);
    const T cph = (T)cprev, cpl = (T)(cprev - (double)cph);
    const T *x = a.x + (int64_t)blockIdx.y * a.vstride;
    T *y = a.y + (int64_t)blockIdx.y * a.vstride;
    const T *xprev = LZ ? a.xprev + (int64_t)blockIdx.y * a.vstride : nullptr;
    CSum dot;
    dot.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + tid; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cg = i / dimup, r = i - cg * dimup;
        const int64_t q = cg / dimdw, cc = cg - q * dimdw;
        const T xi = x[i];
        T acc = (a.du[r] + a.dd[cc] + sdint[(a.wu[r] & imask) * ni + (a.wd[cc] & imask)]) * xi;
        const int nu = a.cu[r], nd = a.cd[cc];
        const T *col = x + cg * dimup;
        for (int e = 0; e < nu && e < a.W; e++) {
            const uint32_t en = a.eu[(int64_t)e * dimup + r];
            if (!DM_IN(ell_col(en), dimup) || !DM_IN(ell_par(en), a.P)) continue;
            const T v = ell_neg(en) ? -spu[ell_par(en)] : spu[ell_par(en)];
            acc += v * col[ell_col(en)];
        }
        for (int e = 0; e < nd && e < a.W; e++) {
            const uint32_t en = a.ed[(int64_t)e * dimdw + cc];
            if (!DM_IN(ell_col(en), dimdw) || !DM_IN(ell_par(en), a.P)) continue;
            const T v = ell_neg(en) ? -a.pd[ell_par(en)] : a.pd[ell_par(en)];
            acc += v * x[(q * dimdw + (int64_t)ell_col(en)) * dimup + r];
        }
        if (LZ) {
            const T xp = xprev[i];
            if constexpr (sizeof(T) == 8) {
                acc = sc * acc - cprev * xp;
            } else {
                T t = -cpl * xp;
                t = fmaf(-cph, xp, t);
                t = fmaf(scl, acc, t);
                acc = fmaf(sch, acc, t);
            }
            dot.add((double)xi * (double)acc);
        }
        y[i] = acc;
    }
    if (LZ) {
        CSum arr[1] = {dot};
        double tot[1];
        if (grid_reduce<1>(arr, a.partials, a.counter, tot)) {
            if (tid == 0) a.alpha[a.k] = sc * tot[0];
        }
    }
}

template <typename T>
HxvArgs<T> make_hxv_args(const dmfted_ctx *c, const SectorView &s) {
    HxvArgs<T> a{};
    // rows (r) and columns (q) of the stored vector: up and down spin in the
    // reference order, exchanged for a swapped view (H = H_up + H_dw + D is
    // symmetric in the two factors; the hop signs depend on one spin only)
    const bool sw = s.swapped;
    const SpinTables &tu = c->spin[0];
    const SpinTables &td = c->spin_shared ? c->spin[0] : c->spin[1];
    const SpinTables &tr = sw ? td : tu, &tq = sw ? tu : td;
    const int64_t offr = sw ? s.offdw : s.offup, offq = sw ? s.offup : s.offdw;
    a.dimup = sw ? s.dimdw : s.dimup;
    a.dimdw = sw ? s.dimup : s.dimdw;
    a.norb = c->norb;
    a.P = c->P;
    a.W = std::max(c->W, 1);
    a.wu = c->words.p + offr;
    a.wd = c->words.p + offq;
    a.cu = tr.cnt.p + offr;
    a.cd = tq.cnt.p + offq;
    a.eu = tr.ell.p + (int64_t)a.W * offr;
    a.ed = tq.ell.p + (int64_t)a.W * offq;
    a.eux = tr.ellx.p ? tr.ellx.p + (int64_t)c->WX * offr : nullptr;
    const int nr = sw ? s.ndw : s.nup, nq = sw ? s.nup : s.ndw;
    a.ku_max = (int)tr.cls_max.size() > nr ? tr.cls_max[nr] : kMaxW;
    a.kd_max = (int)tq.cls_max.size() > nq ? tq.cls_max[nq] : kMaxW;
    a.dswap = sw ? 1 : 0;
    if constexpr (sizeof(T) == 8) {
        a.du = (const T *)tr.diag.p + offr;
        a.dd = (const T *)tq.diag.p + offq;
        a.pu = (const T *)tr.par.p;
        a.pd = (const T *)tq.par.p;
        a.dint = (const T *)c->dint.p;
    } else {
        a.du = (const T *)tr.diag_f.p + offr;
        a.dd = (const T *)tq.diag_f.p + offq;
        a.pu = (const T *)tr.par_f.p;
        a.pd = (const T *)tq.par_f.p;
        a.dint = (const T *)c->dint_f.p;
    }
    a.vstride = s.dim;
    a.nstack = 1;
    return a;
}
template HxvArgs<double> make_hxv_args<double>(const dmfted_ctx *, const SectorView &);
template HxvArgs<float> make_hxv_args<float>(const dmfted_ctx *, const SectorView &);

// Launch configuration.  VW: 16-byte vectors when the column stride keeps
// them aligned (DimUp*sizeof(T) a multiple of 16).  NC: two columns per CTA
// when there are enough columns to fill the GPU, else one.  The staged
// columns must fit in shared memory (DimUp*sizeof(T)*NC <= 200 KB).
struct HxvCfg {
    int nc, vw, threads;
    size_t smem;
    int grid;
    bool global;  // the columns do not fit in shared memory: k_hxv_global
};


static bool aligned_to(const void *p, size_t b) { return ((uintptr_t)p % b) == 0; }

template <typename T>
static HxvCfg hxv_config(dmfted_ctx *c, const SectorView &s, const HxvArgs<T> &a, int nstack = 1) {
    HxvCfg g;
    // two rows per thread-vector: 8-byte (FP32) or 16-byte (FP64) accesses;
    // needs an even row count and every base pointer aligned to the vector size
    const size_t vb = 2 * sizeof(T);
    const bool aligned = aligned_to(a.x, vb) && aligned_to(a.y, vb) &&
                         (!a.xprev || aligned_to(a.xprev, vb)) && aligned_to(a.wu, 8) &&
                         aligned_to(a.du, vb) && aligned_to(a.eu, 8) && aligned_to(a.cu, 2) &&
                         ((a.vstride * (int64_t)sizeof(T)) % vb == 0);
    g.vw = (a.dimup % 2 == 0 && aligned) ? 2 : 1;
    const int64_t ncols = a.dimdw * nstack;
    g.nc = 16 / (int)sizeof(T);  // one 16-byte gather serves the whole tile
    const size_t tile = (size_t)a.dimup * sizeof(T) * g.nc;
    g.global = tile > (size_t)200 * 1024 || c->tune_hxv == 3;
    if (g.global) {
        // one thread per element
        g.threads = 256;
        g.smem = 0;
        g.grid = (int)std::min<int64_t>(std::max<int64_t>(div_up(ncols * a.dimup, 256), 1),
                                        std::min<int64_t>(kMaxRedBlocks, 8 * num_sms(c)));
        return g;
    }
    g.threads = (a.dimup <= (int64_t)128 * g.vw * 2) ? 128 : 256;
    g.smem = tile;
    g.grid = (int)std::min<int64_t>((ncols + g.nc - 1) / g.nc, kMaxRedBlocks);
    return g;
}

template <typename T, int NC, int VW, bool LZ>
static void launch_nc(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    auto kern = k_hxv<T, NC, VW, LZ>;
    static bool attr_set[64] = {false};
    if (!attr_set[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr_set[c->device & 63] = true;
    }
    dim3 grid(g.grid, nvec);
    kern<<<grid, g.threads, g.smem, c->stream>>>(a);
    DM_CHECK_LAUNCH();
    c->launches++;
}

template <typename T, bool LZ>
static void launch_rv(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    auto kern = k_hxv_rv<T, LZ>;
    static bool attr_set[64] = {false};
    if (!attr_set[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr_set[c->device & 63] = true;
    }
    dim3 grid(g.grid, nvec);
    kern<<<grid, g.threads, g.smem, c->stream>>>(a);
    DM_CHECK_LAUNCH();
    c->launches++;
}

template <typename T, int KU, int KD, int MODE, int MB>
static void launch_lean_mb(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    auto kern = k_hxv_lean<T, KU, KD, MODE, MB>;
    static bool attr_set[64] = {false};
    if (!attr_set[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr_set[c->device & 63] = true;
    }
    dim3 grid(g.grid, nvec);
    kern<<<grid, g.threads, g.smem, c->stream>>>(a, a.eux);
    DM_CHECK_LAUNCH();
    c->launches++;
}

// Three CTAs per SM (register cap 80, a few bytes of spills) measured 5-9 %
// faster than two (128 registers) on the Ns=14 sectors in both precisions:
// latency hiding pays more than the registers.  DMFTED_HXV_OCC=2 keeps two.
template <typename T, int KU, int KD, int MODE>
static void launch_lean_k(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    if (c->tune_occ == 2) launch_lean_mb<T, KU, KD, MODE, kRvBlocks>(c, a, g, nvec);
    else launch_lean_mb<T, KU, KD, MODE, 3>(c, a, g, nvec);
}

// Hop counts padded to 7 or 8 (rows and columns independently).
template <typename T, int MODE>
static void launch_lean(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    const bool u8 = a.ku_max > 7, d8 = a.kd_max > 7;
    if (u8 && d8) launch_lean_k<T, 8, 8, MODE>(c, a, g, nvec);
    else if (u8) launch_lean_k<T, 8, 7, MODE>(c, a, g, nvec);
    else if (d8) launch_lean_k<T, 7, 8, MODE>(c, a, g, nvec);
    else launch_lean_k<T, 7, 7, MODE>(c, a, g, nvec);
}

// Whether the lean kernel serves this sector view: at most 8 hops per word
// on either side, signed coupling indices within 8 bits, row offsets within
// 24 bits, two-row vectors, fewer than 2^32 stacked elements.
template <typename T>
static bool lean_ok(const dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g) {
    return g.vw == 2 && c->tune_hxv != 1 && c->tune_hxv != 2 && a.eux && a.ku_max <= 8 &&
           a.kd_max <= 8 && 2 * a.P <= (int)kLeanZero && a.dimup * 16 < (1 << 24) &&
           (double)a.dimup * a.dimdw * a.nstack < 4.0e9;
}

template <typename T, bool LZ>
static void launch_hxv(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    constexpr int NCT = 16 / sizeof(T);
    // algorithmic bytes: read x (and v_prev for the Lanczos step), write y
    const double bytes = (LZ ? 3.0 : 2.0) * (double)a.dimup * a.dimdw * a.nstack * nvec * sizeof(T);
    // the register-batched kernel needs two-row vectors and 32-bit element
    // offsets within the stacked vector
    const bool rv = g.vw == 2 && c->tune_hxv != 1 &&
                    (double)a.dimup * a.dimdw * a.nstack < 4.0e9;
    const bool lean = !g.global && lean_ok<T>(c, a, g);
    hv_timer_begin(c);
    if (g.global) {
        k_hxv_global<T, LZ><<<dim3(g.grid, nvec), g.threads, 0, c->stream>>>(a);
        DM_CHECK_LAUNCH();
        c->launches++;
    } else if (lean) launch_lean<T, LZ ? 1 : 0>(c, a, g, nvec);
    else if (rv) launch_rv<T, LZ>(c, a, g, nvec);
    else if (g.vw == 2) launch_nc<T, NCT, 2, LZ>(c, a, g, nvec);
    else launch_nc<T, NCT, 1, LZ>(c, a, g, nvec);
    hv_timer_end(c, bytes);
}

// y += H_J x for the Jhflag spin-exchange / pair-hopping terms (jterms.cuh),
// on nvec vectors vstride apart, each nstack stacked halves of the sector
// (dim apart), in the view's storage order.  One thread per element gathers
// the targets through the rank table.
template <typename T>
__global__ void k_hxv_jadd(const uint32_t *__restrict__ wup, const uint32_t *__restrict__ wdw,
                           const int32_t *__restrict__ rank, uint32_t dimup, uint32_t dimdw,
                           int swapped, int norb, double jx, double jp, const T *x, T *y,
                           int nstack, int nvec, int64_t vstride) {
    const int64_t dim = (int64_t)dimup * dimdw;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < dim;
         e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = swapped ? (uint32_t)(e / dimdw) : (uint32_t)(e % dimup);
        const uint32_t q = swapped ? (uint32_t)(e % dimdw) : (uint32_t)(e / dimup);
        for (int v = 0; v < nvec; v++)
            for (int h = 0; h < nstack; h++) {
                const int64_t base = v * vstride + h * dim;
                double acc = 0.0;
                for_jterms(wup[r], wdw[q], norb, jx, jp, [&](uint32_t tu, uint32_t td, double cf) {
                    const int64_t rt = rank[tu], qt = rank[td];
                    const int64_t j = swapped ? qt + (int64_t)dimdw * rt : rt + (int64_t)dimup * qt;
                    if (DM_IN(j, dim)) acc += cf * (double)x[base + j];
                });
                if (acc != 0.0) y[base + e] = (T)((double)y[base + e] + acc);
            }
    }
}

template <typename T>
static void hxv_jadd(dmfted_ctx *c, const SectorView &s, const T *x, T *y, int nstack, int nvec,
                     int64_t vstride) {
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(div_up(s.dim, 256), 1),
                                            (int64_t)num_sms(c) * 8);
    k_hxv_jadd<T><<<grid, 256, 0, c->stream>>>(c->words.p + s.offup, c->words.p + s.offdw,
                                                c->rank.p, (uint32_t)s.dimup, (uint32_t)s.dimdw,
                                                s.swapped ? 1 : 0, c->norb, c->p.jx, c->p.jp, x, y,
                                                nstack, nvec, vstride);
    DM_CHECK_LAUNCH();
    c->launches++;
}

// The Lanczos combination of the fused step, for products computed in parts
// (Jhflag): u = sc hx - cprev x_prev into y (y may be x_prev: each element is
// read before it is written, by the same thread), alpha_k = sc <x, u>.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_lz_combine(T *y, const T *hx, const T *x,
                                                            const T *xprev, int64_t n,
                                                            LanczosScalars lz, int k,
                                                            double *partials, unsigned *counter) {
    if (lz.status[0]) return;  // the recurrence has ended
    const double sc = lz.scale[k], cprev = k > 0 ? lz.beta[k] * lz.scale[k - 1] : 0.0;
    CSum d;
    d.zero();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T u = (T)(sc * (double)hx[i] - cprev * (double)xprev[i]);
        y[i] = u;
        d.add((double)x[i] * (double)u);
    }
    CSum arr[1] = {d};
    double tot[1];
    if (grid_reduce<1>(arr, partials, counter, tot)) {
        if (threadIdx.x == 0) lz.alpha[k] = sc * tot[0];
    }
}

// Lanczos step k in parts: the plain product into the context's scratch, the
// Jhflag terms, then the combination and alpha (the fused kernels hold no
// Jhflag terms; y may alias x_prev, as the in-place chains have it).
template <typename T>
static void lanczos_step_parts(dmfted_ctx *c, const SectorView &s, const T *x, const T *xprev,
                               T *y, const LanczosScalars &lz, int k, int nstack,
                               double *partials, unsigned *counter) {
    const int64_t n = s.dim * nstack;
    c->jscratch.alloc((size_t)n * sizeof(T) + 256);
    T *hx = reinterpret_cast<T *>(c->jscratch.p);
    HxvArgs<T> a = make_hxv_args<T>(c, s);
    a.nstack = nstack;
    a.x = x;
    a.y = hx;
    HxvCfg g = hxv_config<T>(c, s, a, nstack);
    launch_hxv<T, false>(c, a, g, 1);
    hxv_jadd<T>(c, s, x, hx, nstack, 1, 0);
    const int grid = (int)std::min<int64_t>(std::max<int64_t>(div_up(n, kRedThreads), 1),
                                            std::min<int64_t>(kMaxRedBlocks, (int64_t)num_sms(c) * 8));
    k_lz_combine<T><<<grid, kRedThreads, 0, c->stream>>>(y, hx, x, xprev, n, lz, k, partials,
                                                        counter);
    DM_CHECK_LAUNCH();
    c->launches++;
}

template <typename T>
static void hxv_plain(dmfted_ctx *c, const SectorView &s, const T *x, T *y, int nvec) {
    HxvArgs<T> a = make_hxv_args<T>(c, s);
    a.x = x;
    a.y = y;
    HxvCfg g = hxv_config<T>(c, s, a);
    launch_hxv<T, false>(c, a, g, nvec);
    if (c->jterms) hxv_jadd<T>(c, s, x, y, 1, nvec, a.vstride);
}

void hxv_f64(dmfted_ctx *c, const SectorView &s, const double *x, double *y, int nvec) {
    hxv_plain<double>(c, s, x, y, nvec);
}
void hxv_f32(dmfted_ctx *c, const SectorView &s, const float *x, float *y, int nvec) {
    hxv_plain<float>(c, s, x, y, nvec);
}

// Fused Lanczos step k on the stored vectors (see hxv.cuh).
template <typename T>
void hxv_lanczos_step(dmfted_ctx *c, const SectorView &s, const T *x, const T *xprev, T *y,
                      const LanczosScalars &lz, int k, int nstack) {
    if (c->jterms) {
        lanczos_step_parts<T>(c, s, x, xprev, y, lz, k, nstack, c->red_partials.p,
                              c->red_counter.p);
        return;
    }
    HxvArgs<T> a = make_hxv_args<T>(c, s);
    a.nstack = nstack;
    a.x = x;
    a.y = y;
    a.xprev = xprev;
    a.alpha = lz.alpha;
    a.beta = lz.beta;
    a.scale = lz.scale;
    a.status = lz.status;
    a.k = k;
    a.partials = c->red_partials.p;
    a.counter = c->red_counter.p;
    HxvCfg g = hxv_config<T>(c, s, a, nstack);
    launch_hxv<T, true>(c, a, g, 1);
}
template void hxv_lanczos_step<double>(dmfted_ctx *, const SectorView &, const double *,
                                       const double *, double *, const LanczosScalars &, int, int);
template void hxv_lanczos_step<float>(dmfted_ctx *, const SectorView &, const float *,
                                      const float *, float *, const LanczosScalars &, int, int);

}  // namespace dmfted

namespace dmfted {

// Fused Lanczos step whose reduction scratch is supplied by the caller (the
// context's own scratch is not touched).
template <typename T>
void hxv_lanczos_step_scratch(dmfted_ctx *c, const SectorView &s, const T *x, const T *xprev, T *y,
                              const LanczosScalars &lz, int k, double *partials,
                              unsigned *counter) {
    DM_REQUIRE(!c->jterms, DMFTED_ERR_UNSUPPORTED,
               "the Jhflag terms need scratch memory of the size of a vector: "
               "use dmfted_lanc_tridiag for this model");
    HxvArgs<T> a = make_hxv_args<T>(c, s);
    a.x = x;
    a.y = y;
    a.xprev = xprev;
    a.alpha = lz.alpha;
    a.beta = lz.beta;
    a.scale = lz.scale;
    a.status = lz.status;
    a.k = k;
    a.partials = partials;
    a.counter = counter;
    HxvCfg g = hxv_config<T>(c, s, a, 1);
    launch_hxv<T, true>(c, a, g, 1);
}
template void hxv_lanczos_step_scratch<double>(dmfted_ctx *, const SectorView &, const double *,
                                               const double *, double *, const LanczosScalars &,
                                               int, double *, unsigned *);

}  // namespace dmfted
