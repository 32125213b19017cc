// updateVariablesSA on caller-owned device arrays, with no allocation.
//
// Who needs this: a caller whose device memory is owned by its own
// allocator and who must not have a library allocate behind its back --
// Julia's CUDA.jl pool, a framework's caching allocator, or an application
// that keeps allocation out of its step loop because cudaMalloc/cudaFree
// synchronise the device and are not allowed while a stream is being
// captured.  Such a caller hands in device pointers for every input and
// output; the only extra memory this entry point uses is the fixed
// file-scope scratch array below, which exists once per GPU for as long as
// the library stays loaded.
//
// The kernel is the no-allocation variant of the update-and-reduce stage of
// the fused cell kernel: per cell the primitives from the new conservative
// state (evaluate2d.jl:87-93), Delta = Unew - Uold and Uold <- Unew
// (:95-104), and the per-variable residual sum of Delta^2 with the largest
// VMAX (updateResidualSA, evaluate2d.jl:17-20) through a two-level
// reduction: one record per 256-cell tile in the scratch array, then the
// block that finishes last (elected by a ticket counter in the same array)
// reduces the records in a fixed order.  Built with -fmad=false like the
// other FP64 kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/godunov2d.h"
#include "gd2d_internal.h"

namespace {

constexpr int64_t kNoAllocMaxCells = int64_t(1) << 24;  // 16,777,216 cells
constexpr int kNoAllocTile = 256;
constexpr int64_t kNoAllocMaxTiles = kNoAllocMaxCells / kNoAllocTile;  // 65,536
constexpr int kRec = 8;  // res[4], vmax, bad, 2 spare
// Records, then 256 bytes holding the ticket counter (first 4 bytes).
constexpr int64_t kScratchDoubles = kNoAllocMaxTiles * kRec + 32;

}  // namespace

// 4 MiB + 256 B per GPU: the whole scratch of this entry point.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

namespace {

struct Red {
    double r0, r1, r2, r3, vmax, bad;
};

__device__ __forceinline__ void red_combine(Red &a, const Red &b) {
    a.r0 += b.r0; a.r1 += b.r1; a.r2 += b.r2; a.r3 += b.r3;
    a.vmax = fmax(a.vmax, b.vmax);
    a.bad = fmax(a.bad, b.bad);
}

__device__ __forceinline__ void red_shfl(Red &a, int off) {
    Red b;
    b.r0 = __shfl_down_sync(0xffffffffu, a.r0, off);
    b.r1 = __shfl_down_sync(0xffffffffu, a.r1, off);
    b.r2 = __shfl_down_sync(0xffffffffu, a.r2, off);
    b.r3 = __shfl_down_sync(0xffffffffu, a.r3, off);
    b.vmax = __shfl_down_sync(0xffffffffu, a.vmax, off);
    b.bad = __shfl_down_sync(0xffffffffu, a.bad, off);
    red_combine(a, b);
}

// Fixed-tree block reduction; the result is valid in thread 0.
__device__ __forceinline__ void red_block(Red &a, Red *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int off = 16; off > 0; off >>= 1) red_shfl(a, off);
    if (lane == 0) sh[warp] = a;
    __syncthreads();
    if (warp == 0) {
        if (lane < nw) a = sh[lane];
        else a = Red{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int off = 16; off > 0; off >>= 1) red_shfl(a, off);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kNoAllocTile)
k_update_variables_noalloc(const double *__restrict__ unew, double *__restrict__ uold, double *__restrict__ prims,
                           int64_t n, double G, double *scratch, int64_t ntiles, double *stats_out) {
    __shared__ Red sh[kNoAllocTile / 32];
    __shared__ int s_last;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch + kNoAllocMaxTiles * kRec);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Red a{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < n) {
        const double U1 = unew[i], U2 = unew[n + i], U3 = unew[2 * n + i], U4 = unew[3 * n + i];
        const double rho = U1;
        const double ux = U2 / U1;
        const double uy = U3 / U1;
        const double p = (G - 1.0) * (U4 - 0.5 * (U2 * U2 + U3 * U3) / U1);
        const double as = sqrt(G * p / rho);
        const double vmax = sqrt(ux * ux + uy * uy) + as;
        prims[i] = rho; prims[n + i] = ux; prims[2 * n + i] = uy; prims[3 * n + i] = p;
        const double d0 = U1 - uold[i], d1 = U2 - uold[n + i], d2 = U3 - uold[2 * n + i], d3 = U4 - uold[3 * n + i];
        uold[i] = U1; uold[n + i] = U2; uold[2 * n + i] = U3; uold[3 * n + i] = U4;
        a.r0 = d0 * d0; a.r1 = d1 * d1; a.r2 = d2 * d2; a.r3 = d3 * d3;
        a.vmax = vmax;
        const bool ok = isfinite(U1) && isfinite(U2) && isfinite(U3) && isfinite(U4) && rho > 0.0 && p > 0.0;
        a.bad = ok ? 0.0 : 1.0;
    }
    red_block(a, sh);
    if (threadIdx.x == 0) {
        double *rec = scratch + (int64_t)blockIdx.x * kRec;
        rec[0] = a.r0; rec[1] = a.r1; rec[2] = a.r2; rec[3] = a.r3; rec[4] = a.vmax; rec[5] = a.bad;
        __threadfence();
        const unsigned int prev = atomicAdd(ticket, 1u);
        s_last = (prev == (unsigned int)(ntiles - 1)) ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    Red acc{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t t = threadIdx.x; t < ntiles; t += blockDim.x) {
        const double *rec = scratch + t * kRec;
        Red b{__ldcg(rec), __ldcg(rec + 1), __ldcg(rec + 2), __ldcg(rec + 3), __ldcg(rec + 4), __ldcg(rec + 5)};
        red_combine(acc, b);
    }
    red_block(acc, sh);
    if (threadIdx.x == 0) {
        stats_out[0] = acc.r0; stats_out[1] = acc.r1; stats_out[2] = acc.r2; stats_out[3] = acc.r3;
        stats_out[4] = acc.vmax;
        stats_out[5] = acc.bad;
        *ticket = 0u;  // leave the counter at zero for the next call
    }
}

std::mutex g_addr_mutex;
// Device address of the scratch array per device ordinal, with the id of the
// context it was looked up in: the address is only valid in that context.
// After cudaDeviceReset (or any other teardown of the primary context) the
// module is loaded again into a new context, whose id differs, so the
// address is looked up again rather than reused.
struct ScratchAddr {
    void *addr;
    unsigned long long ctx_id;
};
ScratchAddr g_scratch_addr[256] = {};

// The driver's cuCtxGetCurrent / cuCtxGetId, fetched through the runtime (the
// library links no driver library).  Context ids are unique for the life of
// the process, unlike context handles, which a new context may reuse.
typedef int (*PfnCtxGetCurrent)(void **ctx);
typedef int (*PfnCtxGetId)(void *ctx, unsigned long long *id);

// Id of the calling thread's current context, or 0 when none is current or
// the driver does not offer context ids.  Called with g_addr_mutex held.
unsigned long long current_context_id() {
    static bool looked_up = false;
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    if (!looked_up) {
        looked_up = true;
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
            get_id = reinterpret_cast<PfnCtxGetId>(f2);
        }
        (void)cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx) return 0;
    if (get_id(ctx, &id) != 0) return 0;
    return id;
}

int noalloc_fail(int code, const char *msg) {
    gd2d::set_handleless_error(msg);
    return code;
}

}  // namespace

extern "C" int gd2d_update_variables_noalloc(const double *d_unew, double *d_uold, double *d_prims, int64_t n_cells,
                                             double gamma, double *d_stats, void *stream) {
    if (!d_unew || !d_uold || !d_prims || !d_stats)
        return noalloc_fail(GD2D_ERR_ARG, "gd2d_update_variables_noalloc: NULL device pointer");
    if (n_cells <= 0 || n_cells > kNoAllocMaxCells) {
        char buf[256];
        snprintf(buf, sizeof buf,
                 "gd2d_update_variables_noalloc: n_cells=%lld outside 1..%lld (fixed scratch of this entry point)",
                 (long long)n_cells, (long long)kNoAllocMaxCells);
        return noalloc_fail(GD2D_ERR_ARG, buf);
    }
    if (!(gamma > 1.0)) return noalloc_fail(GD2D_ERR_ARG, "gd2d_update_variables_noalloc: gamma must be > 1");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256)
        return noalloc_fail(GD2D_ERR_CUDA, "gd2d_update_variables_noalloc: no current CUDA device");
    double *scratch = nullptr;
    {
        // Once per device (per context of that device), with that device
        // current: the device address of the scratch symbol (the host-side
        // name is only a stand-in, never a device address).
        std::lock_guard<std::mutex> lock(g_addr_mutex);
        ScratchAddr &sa = g_scratch_addr[dev];
        const unsigned long long ctx = current_context_id();
        if (!sa.addr || ctx == 0 || ctx != sa.ctx_id) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                char buf[256];
                snprintf(buf, sizeof buf, "gd2d_update_variables_noalloc: cudaGetSymbolAddress: %s",
                         cudaGetErrorString(e));
                return noalloc_fail(GD2D_ERR_CUDA, buf);
            }
            sa.addr = p;
            // the lookup made the device's context current if it was not yet
            sa.ctx_id = current_context_id();
        }
        scratch = static_cast<double *>(sa.addr);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ntiles = (n_cells + kNoAllocTile - 1) / kNoAllocTile;
    // the ticket counter must start at zero (a previous call may have failed)
    e = cudaMemsetAsync(scratch + kNoAllocMaxTiles * kRec, 0, 256, st);
    if (e != cudaSuccess) return noalloc_fail(GD2D_ERR_CUDA, cudaGetErrorString(e));
    k_update_variables_noalloc<<<(unsigned int)ntiles, kNoAllocTile, 0, st>>>(d_unew, d_uold, d_prims, n_cells, gamma,
                                                                            scratch, ntiles, d_stats);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(GD2D_ERR_CUDA, cudaGetErrorString(e));
    return GD2D_OK;
}
