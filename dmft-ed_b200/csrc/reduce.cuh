// Deterministic compensated FP64 reductions.
//
// Every partial is a (hi, lo) pair carried with two-sum error-free
// transformations (Knuth TwoSum), merged by warp shuffles, then across warps
// through shared memory.  Grid-level sums use a fixed-order "last block
// finishes" pattern: each block stores its pair in partials[blockIdx], takes a
// ticket, and the block holding the last ticket folds all pairs in blockIdx
// order.  The result is bit-reproducible for a given grid shape.
#pragma once
#include <cuda_runtime.h>

namespace dmfted {

__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

struct CSum {
    double hi, lo;
    __device__ __forceinline__ void zero() { hi = 0.0; lo = 0.0; }
    __device__ __forceinline__ void add(double x) {
        double s, e;
        two_sum(hi, x, s, e);
        hi = s;
        lo += e;
    }
    __device__ __forceinline__ void merge(double h2, double l2) {
        double s, e;
        two_sum(hi, h2, s, e);
        hi = s;
        lo += l2 + e;
    }
    __device__ __forceinline__ double value() const { return hi + lo; }
};

__device__ __forceinline__ void warp_reduce(CSum &a) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double h = __shfl_down_sync(0xffffffffu, a.hi, off);
        double l = __shfl_down_sync(0xffffffffu, a.lo, off);
        a.merge(h, l);
    }
}

// Block reduction of NS sums; result valid in thread 0.  Needs blockDim.x a
// multiple of 32 and <= 1024.  sm: 2*NS*32 doubles of shared memory.
template <int NS>
__device__ __forceinline__ void block_reduce(CSum (&a)[NS], double *sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NS; k++) warp_reduce(a[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NS; k++) {
            sm[(k * 32 + wid) * 2 + 0] = a[k].hi;
            sm[(k * 32 + wid) * 2 + 1] = a[k].lo;
        }
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NS; k++) {
            CSum t;
            t.zero();
            if (lane < nw) {
                t.hi = sm[(k * 32 + lane) * 2 + 0];
                t.lo = sm[(k * 32 + lane) * 2 + 1];
            }
            warp_reduce(t);
            a[k] = t;
        }
    }
    __syncthreads();
}

// Grid reduction of NS sums.  partials: 2*NS*gridDim.x doubles, counter: one
// unsigned that is 0 on entry and is left 0.  Returns true in every thread of
// the single block that finished last; tot[] then holds the grid sums (valid
// in all threads of that block).
template <int NS>
__device__ __forceinline__ bool grid_reduce(CSum (&a)[NS], double *partials, unsigned *counter,
                                            double (&tot)[NS]) {
    __shared__ double sm[2 * NS * 32];
    __shared__ bool last;
    block_reduce<NS>(a, sm);
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NS; k++) {
            partials[(k * nb + bid) * 2 + 0] = a[k].hi;
            partials[(k * nb + bid) * 2 + 1] = a[k].lo;
        }
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == (unsigned)(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    CSum b[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) b[k].zero();
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NS; k++)
            b[k].merge(__ldcg(&partials[(k * nb + j) * 2 + 0]),
                       __ldcg(&partials[(k * nb + j) * 2 + 1]));
    }
    block_reduce<NS>(b, sm);
    __shared__ double res[NS];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NS; k++) res[k] = b[k].value();
        *counter = 0u;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NS; k++) tot[k] = res[k];
    return true;
}

}  // namespace dmfted
