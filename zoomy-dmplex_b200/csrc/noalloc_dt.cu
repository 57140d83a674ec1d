// CFL time step without any device allocation (zsme_compute_dt_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a
// time step: a host code that reserves all device memory up front and forbids
// allocation afterwards (a PETSc or MPI application driving its own memory
// pools), a process that runs under a fixed device-memory budget, or code
// that must not hit the allocator's implicit device synchronisation inside a
// timing-critical loop.  This entry point computes the same CFL step as
// zsme_compute_dt, but on state arrays the caller already owns, and keeps its
// only scratch -- the per-block partial minima -- in a file-scope device
// array that is part of the loaded library image.
//
// Limits and sharing:
//  * at most ZSME_NOALLOC_MAX_CELLS cells (512 KB of scratch, held by every
//    GPU that loads the library until the process exits); larger inputs are
//    rejected with ZSME_ERR_LIMIT;
//  * all calls share the one array: calls whose kernels overlap on the GPU
//    (different streams, or different host threads on one device) race and
//    must be serialised by the caller;
//  * the array keeps the last call's contents; every entry a call reads is
//    written earlier in the same call, so nothing needs clearing;
//  * the first call on each device (and in each CUDA context on it) looks up
//    the array's device address (cudaGetSymbolAddress) with that device
//    current; make that first call before any stream capture begins on the
//    device, and again after cudaDeviceReset or a context switch of its own;
//  * cells whose d_rc is >= DBL_MAX (or +inf) are left out of the minimum,
//    which is how a partitioned caller keeps its halo cells out of the CFL dt.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <mutex>
#include <string>

#include "model_prelude.h"
#include "prepared_mesh.h"
#include "zsme.h"

namespace sme1d_l0_malpasset {
#include "sme1d_l0_malpasset/Model.H"
#include "sme1d_l0_malpasset/Numerics.H"
}
namespace sme2d_l0 {
#include "sme2d_l0/Model.H"
#include "sme2d_l0/Numerics.H"
}
namespace sme2d_l1 {
#include "sme2d_l1/Model.H"
#include "sme2d_l1/Numerics.H"
}
namespace sme2d_l2 {
#include "sme2d_l2/Model.H"
#include "sme2d_l2/Numerics.H"
}
namespace sme2d_l4 {
#include "sme2d_l4/Model.H"
#include "sme2d_l4/Numerics.H"
}

namespace {

constexpr int kBlock = 256;
constexpr int kMaxBlocks = (ZSME_NOALLOC_MAX_CELLS + kBlock - 1) / kBlock;

// The scratch: one partial minimum per block of the first kernel.
static __device__ __align__(256) double g_dt_partial[kMaxBlocks];

// Per-block minimum of r_c / lambda_c (VirtualSolver.hpp:318-345) over a state
// in caller memory (cell-major, any cell order, rc in the same order).
template <class M, class N>
__global__ void __launch_bounds__(kBlock) dt_partial_kernel(int C, const double* __restrict__ q,
                                                            const double* __restrict__ aux,
                                                            const double* __restrict__ rc,
                                                            const double* __restrict__ p, double* partial) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, DIM = M::dimension;
    const int c = blockIdx.x * kBlock + threadIdx.x;
    double ratio = DBL_MAX;
    if (c < C) {
        double qc[NQ], ac[NA];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qc[i] = q[(size_t)c * NQ + i];
#pragma unroll
        for (int i = 0; i < NA; ++i) ac[i] = aux[(size_t)c * NA + i];
        double eig = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double n[3] = {0.0, 0.0, 0.0};
            n[d] = 1.0;
            auto r = N::local_max_abs_eigenvalue(qc, ac, p, n);
            if (r[0] > eig) eig = r[0];
        }
        // a cell without wave speed, or with rc >= DBL_MAX (a halo cell left out
        // of the minimum), does not constrain dt; a ratio enters the minimum
        // only by winning a "<" comparison, so a NaN never masks another cell
        // (VirtualSolver.hpp:326, 341-344)
        if (!(eig < 1e-14)) {
            const double rcv = rc[c];
            if (rcv < DBL_MAX) {
                const double v = rcv / eig;
                if (v < ratio) ratio = v;
            }
        }
    }
    __shared__ double red[kBlock / 32];
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, ratio, off);
        if (o < ratio) ratio = o;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ratio;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = red[0];
        for (int w = 1; w < kBlock / 32; ++w)
            if (red[w] < r) r = red[w];
        partial[blockIdx.x] = r;
    }
}

// Minimum of the partials -> dt = cfl * min, or dt_max if no cell constrains.
__global__ void __launch_bounds__(kBlock) dt_final_kernel(const double* partial, int nblocks, double cfl,
                                                          double dt_max, double* out) {
    double r = DBL_MAX;
    for (int i = threadIdx.x; i < nblocks; i += kBlock)
        if (partial[i] < r) r = partial[i];
    __shared__ double red[kBlock / 32];
    for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, r, off);
        if (o < r) r = o;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBlock / 32; ++w)
            if (red[w] < r) r = red[w];
        *out = (!isfinite(r) || r >= 0.5 * DBL_MAX) ? dt_max : cfl * r;
    }
}

// Device address of g_dt_partial, looked up once per (device, CUDA context).
// The context is part of the key because the array's address belongs to the
// module loaded in one context: after cudaDeviceReset, or under a driver-API
// context that the host code made current itself (PETSc can create one), the
// same ordinal needs a fresh lookup.  The current context is read through the
// runtime's driver entry point, so the library still links the runtime only;
// where that entry point is unavailable the key is the ordinal alone.  A new
// context that happens to reuse a destroyed one's handle value is not told
// apart from it.
using CtxGetCurrent = int (*)(void**);
constexpr int kMaxEntries = 64;
std::mutex g_mu;
struct ScratchEntry {
    int dev;
    void* ctx;
    double* addr;
};
ScratchEntry g_entries[kMaxEntries];
int g_n_entries = 0;
CtxGetCurrent g_ctx_fn = nullptr;
bool g_ctx_fn_looked_up = false;

void* current_context() {
    if (!g_ctx_fn_looked_up) {
        g_ctx_fn_looked_up = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_fn = reinterpret_cast<CtxGetCurrent>(fn);
        else
            cudaGetLastError();
    }
    void* ctx = nullptr;
    if (g_ctx_fn && g_ctx_fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

int scratch_address(int dev, double** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    void* ctx = current_context();
    for (int i = 0; i < g_n_entries; ++i)
        if (g_entries[i].dev == dev && g_entries[i].ctx == ctx) {
            *out = g_entries[i].addr;
            return ZSME_OK;
        }
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_dt_partial);
    if (e != cudaSuccess)
        return zsme::set_error(ZSME_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    // the lookup makes the device's primary context current on a thread that had none
    if (!ctx) ctx = current_context();
    // keep the newest entries when the table is full (contexts that came and went)
    if (g_n_entries == kMaxEntries) {
        for (int i = 1; i < kMaxEntries; ++i) g_entries[i - 1] = g_entries[i];
        g_n_entries--;
    }
    g_entries[g_n_entries++] = ScratchEntry{dev, ctx, p};
    *out = p;
    return ZSME_OK;
}

template <class M, class N>
int run(int C, const double* q, const double* aux, const double* rc, const double* p, double cfl, double* out,
        cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return zsme::set_error(ZSME_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    double* scratch = nullptr;
    const int rcode = scratch_address(dev, &scratch);
    if (rcode) return rcode;
    const int nb = (C + kBlock - 1) / kBlock;
    dt_partial_kernel<M, N><<<nb, kBlock, 0, s>>>(C, q, aux, rc, p, scratch);
    dt_final_kernel<<<1, kBlock, 0, s>>>(scratch, nb, cfl, M::dt_max, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return zsme::set_error(ZSME_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ZSME_OK;
}

}  // namespace

extern "C" int zsme_compute_dt_noalloc(const char* model, int32_t n_cells, const double* d_q_aos,
                                       const double* d_aux_aos, const double* d_rc, const double* d_params,
                                       double cfl, double* d_dt, void* stream) {
    if (!model || !d_q_aos || !d_aux_aos || !d_rc || !d_params || !d_dt)
        return zsme::set_error(ZSME_ERR_ARG, "null argument");
    if (n_cells <= 0) return zsme::set_error(ZSME_ERR_ARG, "n_cells must be > 0");
    if (n_cells > ZSME_NOALLOC_MAX_CELLS)
        return zsme::set_error(ZSME_ERR_LIMIT, "zsme_compute_dt_noalloc: " + std::to_string(n_cells) +
                                                   " cells exceed the compiled maximum of " +
                                                   std::to_string(ZSME_NOALLOC_MAX_CELLS));
    cudaStream_t s = (cudaStream_t)stream;
#define ZSME_NOALLOC_CASE(NS)                                                                   \
    if (!std::strcmp(model, #NS))                                                               \
        return run<NS::Model<double>, NS::Numerics<double>>(n_cells, d_q_aos, d_aux_aos, d_rc,  \
                                                            d_params, cfl, d_dt, s);
    ZSME_NOALLOC_CASE(sme1d_l0_malpasset)
    ZSME_NOALLOC_CASE(sme2d_l0)
    ZSME_NOALLOC_CASE(sme2d_l1)
    ZSME_NOALLOC_CASE(sme2d_l2)
    ZSME_NOALLOC_CASE(sme2d_l4)
#undef ZSME_NOALLOC_CASE
    return zsme::set_error(ZSME_ERR_MODEL, std::string("unknown model: ") + model);
}
