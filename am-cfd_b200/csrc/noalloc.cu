// Energy residual for callers that cannot let the library allocate device memory.
//
// Who needs it: an application that owns all device memory through its own pool
// (for example a larger multiphysics code that embeds this solver and hands out
// every byte itself), or one that runs under a fixed device-memory budget where a
// cudaMalloc inside a library call may fail or stall.  Such a caller keeps its own
// coefficient and enthalpy buffers and wants the residual of the energy equation
// (the reference's calculateResiduals(5)) without the library touching the
// allocator.
//
// How: the per-plane partial sums live in g_resid_scratch, a file-scope device
// array that exists on every GPU from the moment the library is loaded until the
// process exits (64 KiB per GPU).  Host code cannot use the array's name as a
// device address, so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it together with the
// device's current CUDA context; make that first call before any stream capture.
// A later call under a different context (after cudaDeviceReset, say) looks the
// address up again.  The function allocates nothing and calls no allocating
// library routine.
//
// Errors: a CUDA error already pending on the calling thread when the call starts
// (left by the caller's own earlier work) is neither reported as this call's nor
// cleared: the call returns AMCFD_E_CUDA at once and leaves it for the caller.
//
// Limits and sharing: at most kMaxPlanes = 4096 interior k-planes (nk - 2); larger
// grids are rejected with AMCFD_E_CAPACITY before anything is launched.  All calls
// on one GPU share the array: every entry a call reads is written by the same call
// first, so nothing has to start at zero, but two calls that overlap on the GPU
// (different streams without ordering) race on it and must not be issued.
#include <cstdio>
#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "amcfd.h"

namespace {

constexpr int kMaxPlanes = 4096;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_resid_scratch[2 * kMaxPlanes];

std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};  // the context each address belongs to

// The calling thread's current driver context (cuCtxGetCurrent through the
// runtime's entry-point query, so the library needs no -lcuda); null if unknown.
CUcontext current_context()
{
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &ptr, cudaEnableDefault, &qr) != cudaSuccess ||
            qr != cudaDriverEntryPointSuccess || !ptr)
            return nullptr;
        fn = reinterpret_cast<Fn>(ptr);
    }
    CUcontext c = nullptr;
    return fn(&c) == CUDA_SUCCESS ? c : nullptr;
}

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Two sums of one interior plane k: sum |(sum_nb a_nb h_nb + su)/ap - h| and sum |h|.
__global__ void __launch_bounds__(256) resid_plane_kernel(
    const double *an, const double *as, const double *ae, const double *aw, const double *at,
    const double *ab, const double *ap, const double *su, const double *h, int ni, int nj,
    int pitch, double *part)
{
    const int k = blockIdx.x + 1;
    const size_t sj = (size_t)pitch, sk = (size_t)nj * pitch;
    double sd = 0.0, sh = 0.0;
    const int nin = ni - 2, ncell = nin * (nj - 2);
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
        const int j = 1 + q / nin, i = 1 + q % nin;
        const size_t c = (size_t)k * sk + (size_t)j * sj + i;
        const double hc = h[c];
        double r = (an[c] * h[c + sj] + as[c] * h[c - sj] + ae[c] * h[c + 1] + aw[c] * h[c - 1] +
                    at[c] * h[c + sk] + ab[c] * h[c - sk] + su[c]) / ap[c] - hc;
        sd += fabs(r);
        sh += fabs(hc);
    }
    __shared__ double red[2][8];
    sd = wsum(sd);
    sh = wsum(sh);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = sd;
        red[1][warp] = sh;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// resorh = sum_d / (sum_h + 1e-6) over the planes, in plane order (CFDSolverManager.cpp:2099).
__global__ void resid_final_kernel(const double *part, int nplanes, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int p = 0; p < nplanes; ++p) {
        a += part[2 * p];
        b += part[2 * p + 1];
    }
    out[0] = a / (b + 1.0e-6);
}

}  // namespace

extern "C" int amcfd_energy_residual_noalloc(const double *an, const double *as, const double *ae,
                                             const double *aw, const double *at, const double *ab,
                                             const double *ap, const double *su, const double *h,
                                             int ni, int nj, int nk, int pitch,
                                             double *resorh_dev, void *stream)
{
    if (!an || !as || !ae || !aw || !at || !ab || !ap || !su || !h || !resorh_dev)
        return AMCFD_E_ARG;
    if (ni < 3 || nj < 3 || nk < 3 || pitch < ni) return AMCFD_E_ARG;
    if (nk - 2 > kMaxPlanes) {
        fprintf(stderr,
                "amcfd_energy_residual_noalloc: %d interior k-planes exceed the fixed scratch "
                "capacity of %d planes\n", nk - 2, kMaxPlanes);
        return AMCFD_E_CAPACITY;
    }
    // an error the caller's own earlier work left pending stays the caller's
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        fprintf(stderr, "amcfd_energy_residual_noalloc: a CUDA error was already pending (%s); nothing launched\n",
                cudaGetErrorString(pending));
        return AMCFD_E_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return AMCFD_E_CUDA;
    double *part;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        // the first call, or the device's context changed since the address was taken
        // (a thread with no current context yet looks it up again, which makes the
        // device's primary context current)
        const CUcontext cur = current_context();
        if (!g_scratch_ptr[dev] || !cur || cur != g_scratch_ctx[dev]) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_resid_scratch);
            if (e != cudaSuccess || !ptr) {
                fprintf(stderr, "amcfd_energy_residual_noalloc: cudaGetSymbolAddress: %s\n",
                        cudaGetErrorString(e));
                return AMCFD_E_CUDA;
            }
            g_scratch_ptr[dev] = (double *)ptr;
            g_scratch_ctx[dev] = current_context();
        }
        part = g_scratch_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    resid_plane_kernel<<<nk - 2, 256, 0, s>>>(an, as, ae, aw, at, ab, ap, su, h, ni, nj, pitch, part);
    resid_final_kernel<<<1, 32, 0, s>>>(part, nk - 2, resorh_dev);
    if (cudaGetLastError() != cudaSuccess) return AMCFD_E_CUDA;
    return AMCFD_OK;
}
