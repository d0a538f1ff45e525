// Allocation-free PSD projection of one symmetric block.
//
// Some hosts of this solver cannot call cudaMalloc at the point where they
// need a projection: a plugin running inside an application that owns all
// device memory through its own pool and forbids allocations after start-up,
// or a latency-bound loop where an allocation (which can synchronise the
// device) is not acceptable.  v2b_project_block_noalloc serves them: it runs
// the same kernels as the library's projection (symmetrize_kernel,
// jacobi_warm_kernel from V = I with the library's 30-sweep limit, the
// batched GEMM tiles) but takes every scratch buffer from one file-scope
// __device__ array instead of cudaMalloc.
//
// The array holds up to kNoAllocMaxDim = 128 rows: its size is fixed at
// build time (about 4.4 MB) and every GPU that loads the library keeps it
// until the process exits.  All calls in a process share it and it keeps the
// contents of the last call; the entry point clears what must start at zero
// on every call.  Calls that overlap on the GPU (different streams or host
// threads) race on the array and must be serialised by the caller.  The
// first call on a device, with that device current, looks up the array's
// device address with cudaGetSymbolAddress (the host-side name of the array
// is only a stand-in, never a device address) and caches it with the
// context's id; a call in a new context (after cudaDeviceReset) looks it up
// again.  Make the first call on each device before any stream capture.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <mutex>
#include <string>

#include "v2b_eig.cuh"
#include "v2b_kernels.cuh"
#include "v2rdm_b200.h"

namespace v2b {

constexpr int kNoAllocMaxDim = 128;
constexpr int kNoAllocSweeps = 30;   // the library projection's Jacobi sweep limit
constexpr int kNoAllocPairs = kNoAllocMaxDim / 2;
constexpr int64_t kNoAllocMat = (int64_t)kNoAllocMaxDim * kNoAllocMaxDim;   // doubles per matrix
// rotation record + per-step counts (in double2 units), as jacobi_warm_kernel lays them out
constexpr int64_t kNoAllocRot = (int64_t)kNoAllocSweeps * (kNoAllocMaxDim - 1) * kNoAllocPairs +
                                ((int64_t)kNoAllocSweeps * (kNoAllocMaxDim - 1) + 3) / 4 + 1;
constexpr int kNoAllocTiles = (kNoAllocMaxDim / kGemmTile) * (kNoAllocMaxDim / kGemmTile);

// layout of the scratch array, in 256-byte aligned sections
struct NoAllocLayout {
    double Us[kNoAllocMat];
    double W[kNoAllocMat];
    double P[kNoAllocMat];
    double Vt[kNoAllocMat];
    double2 rot[kNoAllocRot];
    int4 tiles[kNoAllocTiles];
    int64_t boff[1];
    int64_t rot_off[1];
    int bdim[1];
    int counters[2];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocLayout)];

// descriptors, counters and V = I for one n x n block, written on the device
__global__ void noalloc_setup_kernel(NoAllocLayout *L, int n) {
    const int nt = (n + kGemmTile - 1) / kGemmTile;
    if (threadIdx.x == 0) {
        L->boff[0] = 0;
        L->rot_off[0] = 0;
        L->bdim[0] = n;
        L->counters[0] = 0;
        L->counters[1] = 0;
    }
    for (int t = threadIdx.x; t < nt * nt; t += blockDim.x) L->tiles[t] = make_int4(0, t / nt, t % nt, 0);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) L->Vt[e] = (e / n == e % n) ? 1.0 : 0.0;
}

}  // namespace v2b

namespace {

std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
unsigned char *g_noalloc_base[kMaxDevices] = {};
unsigned long long g_noalloc_ctx[kMaxDevices] = {};   // context the address belongs to

int fail(int code, const std::string &msg) {
    v2b::set_last_error(msg);   // read back through v2b_last_error()
    return code;
}

template <class T>
T *section(unsigned char *base, size_t offset) {
    return reinterpret_cast<T *>(base + offset);
}

}  // namespace

extern "C" int v2b_project_block_noalloc(const double *d_U, int n, double mu, double *d_x,
                                         double *d_z, void *stream) {
    using namespace v2b;
    if (!d_U || !d_x || !d_z) return fail(V2B_BAD_ARG, "project_block_noalloc: NULL pointer");
    if (n < 1 || n > kNoAllocMaxDim)
        return fail(V2B_BAD_ARG, "project_block_noalloc: block dimension " + std::to_string(n) +
                                     " outside 1.." + std::to_string(kNoAllocMaxDim));
    if (!(mu > 0.0)) return fail(V2B_BAD_ARG, "project_block_noalloc: mu must be positive");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(V2B_NO_DEVICE, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(V2B_BAD_ARG, "device ordinal out of range");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        const unsigned long long ctx = current_context_id();
        if (!g_noalloc_base[dev] || g_noalloc_ctx[dev] != ctx) {
            // host code sees only a stand-in for the array: ask the runtime for
            // its address on this device
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(V2B_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_noalloc_base[dev] = (unsigned char *)p;
            g_noalloc_ctx[dev] = current_context_id();   // the lookup created the context if needed
        }
        base = g_noalloc_base[dev];
    }
    // the Jacobi kernel's shared-memory limit is shared with the rest of the
    // library: raise it when this block needs more, never lower it
    e = raise_dynamic_smem((const void *)jacobi_warm_kernel, (int)jacobi_smem_bytes(n));
    if (e != cudaSuccess)
        return fail(V2B_CUDA_ERROR, std::string("shared-memory attribute: ") + cudaGetErrorString(e));
    NoAllocLayout *L = section<NoAllocLayout>(base, 0);
    double *Us = section<double>(base, offsetof(NoAllocLayout, Us));
    double *W = section<double>(base, offsetof(NoAllocLayout, W));
    double *P = section<double>(base, offsetof(NoAllocLayout, P));
    double *Vt = section<double>(base, offsetof(NoAllocLayout, Vt));
    double2 *rot = section<double2>(base, offsetof(NoAllocLayout, rot));
    int4 *tiles = section<int4>(base, offsetof(NoAllocLayout, tiles));
    int64_t *boff = section<int64_t>(base, offsetof(NoAllocLayout, boff));
    int64_t *rot_off = section<int64_t>(base, offsetof(NoAllocLayout, rot_off));
    int *bdim = section<int>(base, offsetof(NoAllocLayout, bdim));
    int *counters = section<int>(base, offsetof(NoAllocLayout, counters));

    cudaStream_t s = (cudaStream_t)stream;
    const int nt = (n + kGemmTile - 1) / kGemmTile;
    noalloc_setup_kernel<<<1, 256, 0, s>>>(L, n);
    // Us = sym(U); with V = I the rotated block T0 = V^T Us V is Us itself
    symmetrize_kernel<<<nt * nt, 256, 0, s>>>(d_U, Us, tiles, boff, bdim);
    jacobi_warm_kernel<<<1, kJacobiThreads, jacobi_smem_bytes(n), s>>>(
        Us, P, Vt, boff, bdim, rot, rot_off, kNoAllocSweeps, 1e-14, 1e-13, counters, counters + 1);
    e = launch_gemm_tiles(kGemmTNStore, nt * nt, s, Vt, P, W, tiles, boff, bdim, nullptr, Us, 0.0,
                          nullptr, nullptr, nullptr, nullptr);
    if (e == cudaSuccess)
        e = launch_gemm_tiles(kGemmNNProject, nt * nt, s, W, Vt, nullptr, tiles, boff, bdim, nullptr,
                              Us, 1.0 / mu, d_x, d_z, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(V2B_CUDA_ERROR, cudaGetErrorString(e));
    return V2B_OK;
}
