// fpsg_noalloc.cu — ensemble observable sums without any device allocation.
//
// fpsg_run reduces the per-trajectory diagonals into ensemble sums with
// k_reduce_part / k_reduce_fin, whose chunk partials live in a buffer the context
// allocates with cudaMalloc.  Some callers cannot allocate at all: code that runs
// while a CUDA graph is being captured, hosts whose device memory belongs to
// another runtime's pool allocator, and integrators that bring their own
// trajectories and only want this library's fixed-order ensemble sums.  For them
// fpsg_ensemble_sums_noalloc keeps its chunk partials in the file-scope array
// g_partials below.
//
// Order of the sums: trajectories in chunks of 64 (ascending within a chunk),
// then a Kahan-compensated combine of the chunk partials in chunk order — the
// reduction of fpsg_run's stream path (FPSG_PATH_STREAM), so for the same FP64
// states the sums are equal to that path's bit for bit.  fpsg_run's resident path
// sums per CTA instead and agrees to rounding.
//
// Limits and sharing:
//   - g_partials holds FPSG_NOALLOC_SCRATCH_DOUBLES doubles (2 MiB); every GPU that
//     loads this library keeps that much device memory until the process exits;
//   - the call needs 5 n ceil(B / 64) partials; larger requests are rejected with
//     FPSG_ERR_INVALID (e.g. n = 100 allows B <= 33536, n = 512 allows B <= 6528);
//   - every call shares g_partials: calls that overlap on the GPU (other streams,
//     other host threads) race on it and must be serialised by the caller;
//   - the call works on the calling thread's current device; rho, sums and the
//     stream must belong to it;
//   - the device address of g_partials is looked up with cudaGetSymbolAddress on
//     every call made outside a stream capture, and cached per device for calls
//     made during one; the first call on a device must therefore come before any
//     capture, and after a cudaDeviceReset the first call must again be made
//     outside a capture.
// The partial pass overwrites every slot it uses, so nothing needs clearing
// between calls.
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/fpsg.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kChunk = 64;   // trajectories per partial sum (fpsg_run's stream path uses the same)

static __device__ __align__(256) double g_partials[FPSG_NOALLOC_SCRATCH_DOUBLES];

// the host-side name g_partials is not a device address; these are, per device
double* g_partials_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// partial sums over trajectories [c*chunk, min(B, (c+1)*chunk)) in ascending order:
// part[c][o*n + i] for o = 0..4: Re rho_up_ii, Re rho_dn_ii, their squares, product
__global__ void k_noalloc_part(const double* __restrict__ rho, int B, int n, int chunk, double* __restrict__ part)
{
    const int c = blockIdx.x;
    const int b0 = c * chunk, b1 = min(B, b0 + chunk);
    const size_t nn2 = 2 * (size_t)n * n;   // doubles per spin matrix
    for (int w = threadIdx.x; w < 5 * n; w += blockDim.x) {
        const int o = w / n, i = w - o * n;
        double acc = 0.0;
        for (int b = b0; b < b1; ++b) {
            const double du = rho[((size_t)b * 2) * nn2 + 2 * ((size_t)i * n + i)];
            const double dd = rho[((size_t)b * 2 + 1) * nn2 + 2 * ((size_t)i * n + i)];
            acc += o == 0 ? du : o == 1 ? dd : o == 2 ? du * du : o == 3 ? dd * dd : du * dd;
        }
        part[(size_t)c * 5 * n + w] = acc;
    }
}

// Kahan sum of the chunk partials in chunk order
__global__ void k_noalloc_fin(const double* __restrict__ part, int nchunks, int W, double* __restrict__ out)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        double s = 0.0, comp = 0.0;
        for (int c = 0; c < nchunks; ++c) {
            const double y = part[(size_t)c * W + w] - comp;
            const double t = s + y;
            comp = (t - s) - y;
            s = t;
        }
        out[w] = s;
    }
}

// Device address of g_partials on device `dev`: looked up afresh outside a stream
// capture (so a cudaDeviceReset in between is harmless), the cached one during a
// capture.  Returns nullptr with *rc set on failure.
double* partials_on(int dev, cudaStream_t s, int* rc)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    if (capturing) cudaGetLastError();   // a refused query (legacy stream during a capture) is not this call's error
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!capturing) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            *rc = FPSG_ERR_CUDA;
            return nullptr;
        }
        g_partials_addr[dev] = static_cast<double*>(p);
    } else if (!g_partials_addr[dev]) {
        *rc = FPSG_ERR_STATE;   // the set-up call has to come before the capture
        return nullptr;
    }
    return g_partials_addr[dev];
}

}  // namespace

extern "C" int fpsg_ensemble_sums_noalloc(const double* rho, int B, int n, double* sums, void* stream)
{
    if (!rho || !sums || B < 1 || n < 1) return FPSG_ERR_INVALID;
    const long nchunks = ((long)B + kChunk - 1) / kChunk;
    if ((long)n > FPSG_NOALLOC_SCRATCH_DOUBLES / 5 || nchunks * 5 * (long)n > FPSG_NOALLOC_SCRATCH_DOUBLES)
        return FPSG_ERR_INVALID;   // the partials would not fit g_partials
    // an error left pending by earlier work on this thread is not consumed or
    // reported as this call's: refuse to launch and leave it for its owner
    if (cudaPeekAtLastError() != cudaSuccess) return FPSG_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return FPSG_ERR_NO_DEVICE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = FPSG_OK;
    double* part = partials_on(dev, s, &rc);
    if (!part) return rc;
    const int W = 5 * n;
    k_noalloc_part<<<(int)nchunks, 256, 0, s>>>(rho, B, n, kChunk, part);
    if (cudaGetLastError() != cudaSuccess) return FPSG_ERR_CUDA;
    k_noalloc_fin<<<(W + 255) / 256, 256, 0, s>>>(part, (int)nchunks, W, sums);
    if (cudaGetLastError() != cudaSuccess) return FPSG_ERR_CUDA;
    return FPSG_OK;
}
