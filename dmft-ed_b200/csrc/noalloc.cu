// dmfted_lanc_tridiag_noalloc: the Green's-function chain tridiagonalisation
// for callers that cannot allocate device memory when they call it.
//
// Who cannot allocate: a Fortran or C host whose device memory is owned by its
// own pool manager, code running inside a region where cudaMalloc is
// forbidden or would synchronise a latency-critical loop, or a caller that
// prepared all buffers up front.  Such a caller owns the start vector, the two
// work vectors and the outputs; the only other device memory the recurrence
// needs (grid-reduction partial sums, the ticket counter, the Lanczos scalars)
// lives in the fixed array below, inside the library image.
//
// Limits and sharing: the array holds kNoAllocBlocks partial-sum pairs and
// the scalars of one recurrence of up to kNoAllocMaxSteps steps (about 90 KB
// per GPU, held by every GPU that loads the library until the process exits).
// Every call on a device uses the same array and leaves its contents behind;
// the counter and status words are cleared at the start of each call.  Calls
// that overlap on the GPU (different streams, threads or contexts on the same
// device) race on the array and must be serialised by the caller.
//
// Set-up: the first call on a device looks up the device address of the array
// (cudaGetSymbolAddress, with that device current) and caches it; make that
// first call before any stream capture that the call could belong to.
#include <mutex>

#include "internal.cuh"

namespace dmfted {

constexpr int kNoAllocBlocks = kMaxRedBlocks;      // grid-reduction blocks covered
constexpr int kNoAllocMaxSteps = kLzMax - 2;       // longest chain accepted
constexpr int kNoAllocPartials = 2 * kNoAllocBlocks;           // (hi, lo) pairs
constexpr int kNoAllocWords = 8;                                // counter / status slots
constexpr int kNoAllocScalars = 3 * (kLzMax + 2) + 4;          // alpha, beta, scale, ritz
constexpr int kNoAllocDoubles = kNoAllocPartials + 2 * kNoAllocWords + kNoAllocScalars;

// The scratch of every call of dmfted_lanc_tridiag_noalloc on this device.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[64] = {nullptr};

// Device address of the array on `device` (looked up once per device, with
// that device current).
static double *noalloc_scratch(int device) {
    DM_REQUIRE(device >= 0 && device < 64, DMFTED_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        DM_CUDA(cudaSetDevice(device));
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        DM_REQUIRE(e == cudaSuccess && p != nullptr, DMFTED_ERR_CUDA,
                   std::string("cudaGetSymbolAddress of the fixed scratch failed: ") +
                       cudaGetErrorString(e));
        g_noalloc_addr[device] = static_cast<double *>(p);
    }
    return g_noalloc_addr[device];
}

// alanc/blanc in the dmfted_lanc_tridiag convention: steps never taken keep
// a = b = 0, blanc[0] = 0.
__global__ void k_noalloc_outputs(LanczosScalars lz, int nlanc, double *a, double *b, int *nused) {
    const int used = lz.status[1];
    for (int i = threadIdx.x; i < nlanc; i += blockDim.x) {
        a[i] = i < used ? lz.alpha[i] : 0.0;
        b[i] = (i == 0 || i > used) ? 0.0 : lz.beta[i];
    }
    if (threadIdx.x == 0) *nused = used;
}

}  // namespace dmfted

using namespace dmfted;

extern "C" int dmfted_lanc_tridiag_noalloc(dmfted_ctx *c, int32_t isector, const double *d_v0,
                                           int32_t nlanc, double *d_work, double *d_alanc,
                                           double *d_blanc, int32_t *d_nused) {
    try {
        DM_REQUIRE(c && d_v0 && d_work && d_alanc && d_blanc && d_nused, DMFTED_ERR_ARG,
                   "null argument");
        DM_REQUIRE(nlanc >= 1 && nlanc <= kNoAllocMaxSteps, DMFTED_ERR_ARG,
                   "lanc_tridiag_noalloc: nlanc must be in [1, " +
                       std::to_string(kNoAllocMaxSteps) +
                       "], the capacity of the fixed scratch (got " + std::to_string(nlanc) + ")");
        DM_REQUIRE(c->bath_set, DMFTED_ERR_STATE, "lanc_tridiag_noalloc: bath not set");
        double *base = noalloc_scratch(c->device);
        DM_CUDA(cudaSetDevice(c->device));
        const SectorView s = sector_view(c, isector);
        double *partials = base;
        unsigned *counter = reinterpret_cast<unsigned *>(base + kNoAllocPartials);
        int *status = reinterpret_cast<int *>(base + kNoAllocPartials + kNoAllocWords);
        double *scal = base + kNoAllocPartials + 2 * kNoAllocWords;
        LanczosScalars lz;
        lz.alpha = scal;
        lz.beta = scal + (kLzMax + 2);
        lz.scale = scal + 2 * (kLzMax + 2);
        lz.ritz = scal + 3 * (kLzMax + 2);
        lz.status = status;
        lz.kmax = nlanc;
        // the ticket counter must start at zero; the status words too
        DM_CUDA(cudaMemsetAsync(counter, 0, kNoAllocWords * sizeof(double), c->stream));
        DM_CUDA(cudaMemsetAsync(status, 0, kNoAllocWords * sizeof(double), c->stream));
        lanczos_chain_fixed(c, s, d_v0, d_work, lz, partials, counter);
        k_noalloc_outputs<<<1, 256, 0, c->stream>>>(lz, nlanc, d_alanc, d_blanc, d_nused);
        DM_CHECK_LAUNCH();
        c->launches++;
        DM_CUDA(cudaStreamSynchronize(c->stream));
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    set_error(DMFTED_OK, "");
    return DMFTED_OK;
}
