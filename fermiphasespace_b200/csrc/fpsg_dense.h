// fpsg_dense.h — host interface of the dense tensor-core path (fpsg_dense.cu).
//
// State layout of the path: full matrices, FP32, two planes per spin matrix
// (plane 0 = real part, plane 1 = imaginary part), padded to NP x NP with
// zeros, m = 2 b + spin.  Within a plane, 32-row x 4-column blocks of 512 bytes
// (element (i, j) at plane_off(i, j)): a warp whose lanes hold 32 consecutive
// rows reads 4 consecutive columns as one contiguous 512-byte segment.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstddef>
#include <cstdint>

#include "fpsg_device.cuh"

namespace fpsg {
namespace dense {

constexpr int NP = 256;                    // padded matrix size (n <= NP)
// Operand modes: split BF16x3 (chunks of 32 bf16 columns) or split TF32x3 (16
// tf32 columns); a chunk tile is 256 rows x 64 bytes either way.
template <bool TF32> struct Mode;
template <> struct Mode<false> { using T = __nv_bfloat16; static constexpr int KCE = 32, EPC = 8; };
template <> struct Mode<true> { using T = float; static constexpr int KCE = 16, EPC = 4; };
constexpr int TILE_BYTES = NP * 64;        // one chunk tile
constexpr size_t TC_BYTES = 2 * (size_t)NP * NP * 4;   // T big/small (or hi/lo) tiles, enough for either mode

__host__ __device__ __forceinline__ int plane_off(int i, int j)
{
    return ((((i >> 5) * (NP >> 2)) + (j >> 2)) << 7) + ((i & 31) << 2) + (j & 3);
}

// Arguments of one RK stage over all matrices:
//     out = a0 P0 + a1 P1 + ax X + hk k(X),   k(X) = -i [X, Delta(X)]
struct DenseArgs {
    int n, M;                    // sites, spin matrices (2 B)
    const float* X;              // stage input
    const float* P0;             // extra RK inputs (null = unused)
    const float* P1;
    float a0, a1, ax, hk;
    float* out;
    const void* Tc;              // tM without its diagonal, split in two terms, [2][chunks][tile] canonical
    DevSys<float> sys;           // diagonal terms (tM_jj, Hartree rows, potential, pulse projection)
    const float* Ud;             // dense U, V ([NP][NP], zero-padded) for long-range Coulomb, else null
    const float* Vd;
    float pulse;                 // pulse amplitude x envelope at the stage time
    unsigned* err;
    // test hook (FPSG_FLAG_TEST_EXPIRE_WAIT): > 0 makes one thread wait, with this
    // poll limit, on a barrier nothing arrives at, before any tensor memory or copy;
    // the wait runs out, the error flag is set and every CTA returns
    uint32_t probe_polls = 0;
};

size_t stage_smem_bytes();
int stage_threads();
cudaError_t configure();                                        // opt-in shared memory
cudaError_t launch_stage(const DenseArgs& a, int grid, bool tf32, cudaStream_t st);
// T ([NP][NP] FP32 device, diagonal dropped) -> canonical two-term tiles of the mode
cudaError_t prep_T(const float* T_full, void* Tc, bool tf32, cudaStream_t st);
// packed FP64 state [M][ne] complex -> full FP32 planes
cudaError_t unpack(const cplx<double>* rho, int n, int M, float* X, cudaStream_t st);
// full FP32 planes -> packed state [M][ne] complex (upper triangle)
cudaError_t pack_f64(const float* X, int n, int M, cplx<double>* rho, cudaStream_t st);
cudaError_t pack_f32(const float* X, int n, int M, cplx<float>* rho, cudaStream_t st);

}  // namespace dense
}  // namespace fpsg
