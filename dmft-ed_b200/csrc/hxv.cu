// Kernels and launchers of the factored H*v; see hxv.cuh for the formulation.
#include <algorithm>

#include "hxv.cuh"

namespace dmfted {

template <typename T, int NC, bool STAGE, bool LZ>
__global__ void __launch_bounds__(256) k_hxv(const HxvArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T spu[kMaxParams], spd[kMaxParams];
    __shared__ T sdint[64];
    __shared__ T sdd[NC];
    __shared__ unsigned simp[NC];
    __shared__ int scnt[NC];
    __shared__ int64_t sbase[NC];
    __shared__ uint32_t sent[NC * kMaxW];

    if (LZ) {
        if (a.status[0]) return;  // chain finished: every later step is a no-op
    }
    const int tid = threadIdx.x, bd = blockDim.x;
    const int64_t dimup = a.dimup, dimdw = a.dimdw, ncols = dimdw * a.nstack;
    for (int i = tid; i < a.P; i += bd) {
        spu[i] = a.pu[i];
        spd[i] = a.pd[i];
    }
    const int ni = 1 << a.norb;
    for (int i = tid; i < ni * ni; i += bd) sdint[i] = a.dint[i];
    const unsigned imask = (unsigned)ni - 1u;

    double sc = 1.0, cprev = 0.0;
    if (LZ) {
        sc = a.scale[a.k];
        cprev = a.k > 0 ? a.beta[a.k] * a.scale[a.k - 1] : 0.0;
    }
    const T *x = a.x + (int64_t)blockIdx.y * a.vstride;
    T *y = a.y + (int64_t)blockIdx.y * a.vstride;
    T *xs = reinterpret_cast<T *>(smem_raw);
    CSum dot;
    dot.zero();

    for (int64_t c0 = (int64_t)blockIdx.x * NC; c0 < ncols; c0 += (int64_t)gridDim.x * NC) {
        const int nc = (int)min((int64_t)NC, ncols - c0);
        __syncthreads();
        const T *xc;
        if (STAGE) {
            for (int j = 0; j < nc; j++) {
                const T *src = x + (c0 + j) * dimup;
                T *dst = xs + (int64_t)j * dimup;
                for (int64_t r = tid; r < dimup; r += bd) dst[r] = src[r];
            }
            xc = xs;
        } else {
            xc = x + c0 * dimup;
        }
        if (tid < nc) {
            const int64_t cg = c0 + tid, q = cg / dimdw, cc = cg - q * dimdw;
            scnt[tid] = a.cd[cc];
            simp[tid] = a.wd[cc] & imask;
            sdd[tid] = a.dd[cc];
            sbase[tid] = q * dimdw;
        }
        for (int t = tid; t < nc * a.W; t += bd) {
            const int j = t / a.W, e = t % a.W;
            const int64_t cc = (c0 + j) % dimdw;
            if (e < (int)a.cd[cc]) sent[j * kMaxW + e] = a.ed[(int64_t)e * dimdw + cc];
        }
        __syncthreads();
        for (int64_t r = tid; r < dimup; r += bd) {
            const unsigned iu = a.wu[r] & imask;
            const T dur = a.du[r];
            T acc[NC];
#pragma unroll
            for (int j = 0; j < NC; j++)
                if (j < nc) acc[j] = (dur + sdd[j] + sdint[iu * ni + simp[j]]) * xc[(int64_t)j * dimup + r];
            const int cnt = a.cu[r];
            for (int e = 0; e < cnt; e++) {
                const uint32_t en = a.eu[(int64_t)e * dimup + r];
                T v = spu[ell_par(en)];
                if (ell_neg(en)) v = -v;
                const int64_t col = ell_col(en);
#pragma unroll
                for (int j = 0; j < NC; j++)
                    if (j < nc) acc[j] += v * xc[(int64_t)j * dimup + col];
            }
#pragma unroll
            for (int j = 0; j < NC; j++) {
                if (j >= nc) break;
                const int ce = scnt[j];
                const int64_t base = sbase[j];
                for (int e = 0; e < ce; e++) {
                    const uint32_t en = sent[j * kMaxW + e];
                    T v = spd[ell_par(en)];
                    if (ell_neg(en)) v = -v;
                    acc[j] += v * x[(base + ell_col(en)) * dimup + r];
                }
                const int64_t idx = (c0 + j) * dimup + r;
                if (LZ) {
                    const double u = sc * (double)acc[j] - cprev * (double)a.xprev[idx];
                    const T ut = (T)u;
                    y[idx] = ut;
                    dot.add((double)xc[(int64_t)j * dimup + r] * (double)ut);
                } else {
                    y[idx] = acc[j];
                }
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

template <typename T>
HxvArgs<T> make_hxv_args(const dmfted_ctx *c, const SectorView &s) {
    HxvArgs<T> a{};
    const SpinTables &tu = c->spin[0];
    const SpinTables &td = c->spin_shared ? c->spin[0] : c->spin[1];
    a.dimup = s.dimup;
    a.dimdw = s.dimdw;
    a.norb = c->norb;
    a.P = c->P;
    a.W = std::max(c->W, 1);
    a.wu = c->words.p + s.offup;
    a.wd = c->words.p + s.offdw;
    a.cu = tu.cnt.p + s.offup;
    a.cd = td.cnt.p + s.offdw;
    a.eu = tu.ell.p + (int64_t)a.W * s.offup;
    a.ed = td.ell.p + (int64_t)a.W * s.offdw;
    if constexpr (sizeof(T) == 8) {
        a.du = (const T *)tu.diag.p + s.offup;
        a.dd = (const T *)td.diag.p + s.offdw;
        a.pu = (const T *)tu.par.p;
        a.pd = (const T *)td.par.p;
        a.dint = (const T *)c->dint.p;
    } else {
        a.du = (const T *)tu.diag_f.p + s.offup;
        a.dd = (const T *)td.diag_f.p + s.offdw;
        a.pu = (const T *)tu.par_f.p;
        a.pd = (const T *)td.par_f.p;
        a.dint = (const T *)c->dint_f.p;
    }
    a.vstride = s.dim;
    a.nstack = 1;
    return a;
}
template HxvArgs<double> make_hxv_args<double>(const dmfted_ctx *, const SectorView &);
template HxvArgs<float> make_hxv_args<float>(const dmfted_ctx *, const SectorView &);

// Launch configuration: columns per CTA and whether the columns fit in
// shared memory.  Picked from the column size; a column block of up to
// ~56 KB keeps 3-4 CTAs resident per SM.
struct HxvCfg {
    int nc;
    bool stage;
    size_t smem;
    int grid;
};

template <typename T>
static HxvCfg hxv_config(dmfted_ctx *c, const SectorView &s, int nstack = 1) {
    HxvCfg g;
    const size_t col = (size_t)s.dimup * sizeof(T);
    const size_t budget = 56 * 1024;
    if (col * 4 <= budget) g.nc = 4;
    else if (col * 2 <= budget) g.nc = 2;
    else g.nc = 1;
    g.stage = col * g.nc <= 200 * 1024;
    g.smem = g.stage ? col * g.nc : 0;
    int64_t blocks = (s.dimdw * nstack + g.nc - 1) / g.nc;
    g.grid = (int)std::min<int64_t>(blocks, kMaxRedBlocks);
    return g;
}

template <typename T, int NC, bool STAGE, bool LZ>
static void launch_nc(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    auto kern = k_hxv<T, NC, STAGE, LZ>;
    static bool attr_set[64] = {false};
    if (g.smem > 48 * 1024 && !attr_set[c->device & 63]) {
        DM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
        attr_set[c->device & 63] = true;
    }
    dim3 grid(g.grid, nvec);
    kern<<<grid, 256, g.smem, c->stream>>>(a);
    DM_CHECK_LAUNCH();
    c->launches++;
}

template <typename T, bool LZ>
static void launch_hxv(dmfted_ctx *c, const HxvArgs<T> &a, const HxvCfg &g, int nvec) {
    if (g.stage) {
        if (g.nc == 4) launch_nc<T, 4, true, LZ>(c, a, g, nvec);
        else if (g.nc == 2) launch_nc<T, 2, true, LZ>(c, a, g, nvec);
        else launch_nc<T, 1, true, LZ>(c, a, g, nvec);
    } else {
        launch_nc<T, 1, false, LZ>(c, a, g, nvec);
    }
}

template <typename T>
static void hxv_plain(dmfted_ctx *c, const SectorView &s, const T *x, T *y, int nvec) {
    HxvArgs<T> a = make_hxv_args<T>(c, s);
    a.x = x;
    a.y = y;
    HxvCfg g = hxv_config<T>(c, s);
    launch_hxv<T, false>(c, a, g, nvec);
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
    HxvCfg g = hxv_config<T>(c, s, nstack);
    launch_hxv<T, true>(c, a, g, 1);
}
template void hxv_lanczos_step<double>(dmfted_ctx *, const SectorView &, const double *,
                                       const double *, double *, const LanczosScalars &, int, int);
template void hxv_lanczos_step<float>(dmfted_ctx *, const SectorView &, const float *,
                                      const float *, float *, const LanczosScalars &, int, int);

}  // namespace dmfted
