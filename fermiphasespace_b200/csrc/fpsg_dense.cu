// fpsg_dense.cu — the dense tensor-core path (sm_100a, tcgen05).
//
// For long-range hopping (moire lattices: tens of hopping partners per site)
// the commutator is GEMM-shaped.  Delta = T + diag(d) with T = tM off its
// diagonal, real symmetric and the same for every trajectory, and d the
// per-matrix diagonal (tM_jj, Hartree, potential, pulse).  With X = Xr + i Xi
// (Xr symmetric, Xi antisymmetric):
//     k = -i (X Delta - Delta X) = (Di + Xi o delta) - i (Dr + Xr o delta),
//     Dc = Xc T - T Xc,  delta_ij = d_j - d_i.
// Both products of Dc read their operands straight from the row-major planes:
// as the B operand of an MMA a stored row-major tile is its transpose, which is
// T itself for T, Xr for Xr and -Xi for Xi; the sign of -T Xr is the
// instruction's A-negate bit.  So one 256 x 256 accumulator per plane holds Dc
// with no transposed access in the epilogue.
//
// Precision: each operand is split into two terms, bf16 hi + lo (16 significant
// bits, kind::f16, K = 16 per instruction) or tf32 big + small (~21 bits,
// kind::tf32, K = 8), and a product uses the three terms big*big + big*small +
// small*big, accumulated in FP32 in tensor memory.  Diagonal terms, the RK combination and
// the state are FP32.
//
// One launch = one RK stage of every spin matrix.  Persistent CTAs (one per SM),
// warp-specialised:
//   warps 0-15  epilogue: Hartree diagonal d of the matrix, then per plane read
//               the accumulator from tensor memory and write
//               out = a0 P0 + a1 P1 + ax X + hk k (the 3/8 RK rule in terms of
//               stored stage inputs)
//   warps 16-23 producers: stage X chunks (256 rows x 32 columns) into shared
//               memory as bf16 hi/lo in the no-swizzle K-major core-matrix
//               layout, once per accumulator tile; one thread also bulk-copies
//               the matching T chunks
//   warp 24     allocates tensor memory; one thread issues tcgen05.mma
// Three shared-memory stages of 64 KB; tensor memory holds the 256 x 256 FP32
// accumulator of one plane as two 128-row tiles of 256 columns, filled one after
// the other (one pass over K per tile), so that the epilogue of one tile runs
// while the MMAs of the other accumulate.
#include "fpsg_dense.h"
#include "fpsg_tc.cuh"

namespace fpsg {
namespace dense {

constexpr int STAGES = 3;
constexpr int STAGE_BYTES = 4 * TILE_BYTES;         // X hi, X lo, T hi, T lo (16 KB each)
constexpr int N_EPI_WARPS = 16;                     // 4 lane quarters x 4 column groups of 64
constexpr int EPI_COLS = NP / (N_EPI_WARPS / 4);    // columns per epilogue warp
constexpr int EPI_BLK = 8;                          // columns per tensor-memory read
constexpr int N_PROD_WARPS = 8;
constexpr int PROD_WARP0 = N_EPI_WARPS;
constexpr int MMA_WARP = PROD_WARP0 + N_PROD_WARPS;
constexpr int NTHREADS = (MMA_WARP + 1) * 32;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t LBO = 128;                       // K-adjacent core matrices
constexpr uint32_t SBO = 4 * 128;                   // next 8-row group (64-byte chunk rows)
constexpr size_t PLANE = (size_t)NP * NP;

// error bits (unsigned flag shared with the other kernels)
constexpr unsigned ERR_WAIT = 1u << 4;

// element (r, k) of a chunk tile, k in [0, KCE): core matrices of 8 rows x 16
// bytes (EPC elements per core row), row groups SBO apart, K-cores LBO apart
template <int EPC>
__host__ __device__ __forceinline__ int canon(int r, int k)
{
    return ((((r >> 3) * 4) + k / EPC) * (8 * EPC)) + ((r & 7) * EPC) + (k % EPC);
}

struct Shared {
    // after the stage buffers
    float d[2][NP];          // Delta_jj of the matrix (double-buffered by matrix)
    float nd[2][NP];         // diagonals: other spin, same spin
    uint64_t fullX[STAGES];  // producers' conversions done (128 arrivals)
    uint64_t fullT[STAGES];  // T bulk copies landed (1 arrival + bytes)
    uint64_t empty[STAGES];  // MMAs reading the stage are done
    uint64_t tfull[2];       // accumulator tile mt complete
    uint64_t tempty[2];      // epilogue done with accumulator tile mt (16 warps)
    uint64_t drain;
    uint64_t probe;          // test hook: a barrier nothing arrives at
    uint32_t tmem_base;
    int abort;
    int epi_ok[2];           // the accumulator wait's outcome (per tile), shared by all epilogue threads
};

size_t stage_smem_bytes() { return (size_t)STAGES * STAGE_BYTES + sizeof(Shared) + 1024; }
int stage_threads() { return NTHREADS; }

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity, Shared* sh, unsigned* err)
{
    for (uint32_t i = 0; i < (1u << 24); ++i) {
        if (tc::mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && *(volatile int*)&sh->abort) return false;
    }
    *(volatile int*)&sh->abort = 1;
    atomicOr(err, ERR_WAIT);
    return false;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);   // .x = a (low half), .y = b
    return *reinterpret_cast<const uint32_t*>(&v);
}

// hi = bf16(x), lo = bf16(x - hi) for 8 values
__device__ __forceinline__ void split8(const float4& u, const float4& v, uint4& hi, uint4& lo)
{
    const float x[8] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w};
    float h[8], l[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        h[t] = __bfloat162float(__float2bfloat16_rn(x[t]));
        l[t] = x[t] - h[t];
    }
    hi = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
    lo = make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]), pack_bf16(l[6], l[7]));
}

// tf32 split of 4 values: big = tf32(x), small = tf32(x - big)
__device__ __forceinline__ void split4_tf32(const float4& u, uint4& big, uint4& small)
{
    const float x[4] = {u.x, u.y, u.z, u.w};
    uint32_t b[4], l[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const float hb = tc::round_tf32(x[t]);
        b[t] = __float_as_uint(hb);
        l[t] = __float_as_uint(tc::round_tf32(x[t] - hb));
    }
    big = make_uint4(b[0], b[1], b[2], b[3]);
    small = make_uint4(l[0], l[1], l[2], l[3]);
}

template <bool TF32>
__global__ void __launch_bounds__(NTHREADS, 1) k_dense_stage(DenseArgs a)
{
    using MD = Mode<TF32>;
    using T = typename MD::T;
    constexpr int KCE = MD::KCE, EPC = MD::EPC, NCHE = NP / KCE, TILE_E = NP * KCE;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* stages = smem;
    Shared* sh = reinterpret_cast<Shared*>(smem + (size_t)STAGES * STAGE_BYTES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t mstride = 2 * PLANE;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tc::mbar_init(&sh->fullX[s], N_PROD_WARPS * 32);
            tc::mbar_init(&sh->fullT[s], 1);
            tc::mbar_init(&sh->empty[s], 1);
        }
        for (int t = 0; t < 2; ++t) {
            tc::mbar_init(&sh->tfull[t], 1);
            tc::mbar_init(&sh->tempty[t], N_EPI_WARPS);
        }
        tc::mbar_init(&sh->drain, 1);
        tc::mbar_init(&sh->probe, 1);
        sh->abort = 0;
        tc::mbar_fence_init();
    }
    if (a.probe_polls > 0) {
        // the bounded-wait test: nothing has been allocated or issued yet, so the
        // CTA can leave as soon as the wait has run out and flagged the error
        __syncthreads();
        if (threadIdx.x == 0 && !tc::mbar_wait(&sh->probe, 0, a.err, ERR_WAIT, a.probe_polls))
            sh->abort = 1;
        __syncthreads();
        if (sh->abort) return;
    }
    if (warp == MMA_WARP) {
        tc::tmem_alloc(&sh->tmem_base, TMEM_COLS);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tbase = sh->tmem_base;

    if (warp >= PROD_WARP0 && warp < MMA_WARP) {
        // ------------------------------------------------------------ producers
        const int pt = threadIdx.x - PROD_WARP0 * 32;
        const int pw = pt >> 5;
        const int r8 = lane & 7, kq = lane >> 3;
        int it = 0;
        long t_issued[STAGES] = {-1, -1, -1};
        bool ok = true;
        for (int m = blockIdx.x; m < a.M && ok; m += gridDim.x) {
            for (int pm = 0; pm < 4 && ok; ++pm) {          // plane p = pm >> 1, tile pm & 1
                const float* Xp = a.X + (size_t)m * mstride + (size_t)(pm >> 1) * PLANE;
                for (int kc = 0; kc < NCHE; ++kc, ++it) {
                    const int s = it % STAGES;
                    if (!wait_bar(&sh->empty[s], ((it / STAGES) & 1) ^ 1, sh, a.err)) { ok = false; break; }
                    unsigned char* st = stages + (size_t)s * STAGE_BYTES;
                    if (pt == 0) {
                        const char* tcb = reinterpret_cast<const char*>(a.Tc);
                        tc::mbar_arrive_expect_tx(&sh->fullT[s], 2 * TILE_BYTES);
                        tc::bulk_g2s(st + 2 * TILE_BYTES, tcb + (size_t)kc * TILE_BYTES, TILE_BYTES, &sh->fullT[s]);
                        tc::bulk_g2s(st + 3 * TILE_BYTES, tcb + (size_t)(NCHE + kc) * TILE_BYTES, TILE_BYTES,
                                     &sh->fullT[s]);
                        t_issued[s] = it;
                    }
                    T* xh = reinterpret_cast<T*>(st);
                    T* xl = xh + TILE_E;
                    // lane (r8, kq): one 16-byte core row of row r, K-core kq
                    float4 v[NP / 8 / N_PROD_WARPS][TF32 ? 1 : 2];
#pragma unroll
                    for (int q = 0; q < NP / 8 / N_PROD_WARPS; ++q) {
                        const int r = (pw + q * N_PROD_WARPS) * 8 + r8;
                        const int k = kc * KCE + kq * EPC;
                        v[q][0] = __ldg(reinterpret_cast<const float4*>(Xp + plane_off(r, k)));
                        if constexpr (!TF32) v[q][TF32 ? 0 : 1] = __ldg(reinterpret_cast<const float4*>(Xp + plane_off(r, k + 4)));
                    }
#pragma unroll
                    for (int q = 0; q < NP / 8 / N_PROD_WARPS; ++q) {
                        const int r = (pw + q * N_PROD_WARPS) * 8 + r8;
                        uint4 hi, lo;
                        if constexpr (TF32) split4_tf32(v[q][0], hi, lo);
                        else split8(v[q][0], v[q][TF32 ? 0 : 1], hi, lo);
                        *reinterpret_cast<uint4*>(xh + canon<EPC>(r, kq * EPC)) = hi;
                        *reinterpret_cast<uint4*>(xl + canon<EPC>(r, kq * EPC)) = lo;
                    }
                    tc::fence_async_smem();
                    tc::mbar_arrive(&sh->fullX[s]);
                }
            }
        }
        // bulk copies still in flight must land before the CTA exits
        if (pt == 0)
            for (int s = 0; s < STAGES; ++s)
                if (t_issued[s] >= 0) {
                    const uint32_t par = (uint32_t)((t_issued[s] / STAGES) & 1);
                    for (uint32_t i = 0; i < (1u << 24); ++i)
                        if (tc::mbar_try_wait(&sh->fullT[s], par)) break;
                }
    } else if (warp == MMA_WARP) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t id_xt = TF32 ? tc::idesc_tf32_f32(128, NP, false) : tc::idesc_bf16_f32(128, NP, false);
            int it = 0;
            int uu[2] = {0, 0};                 // uses of each accumulator tile
            bool ok = true;
            for (int m = blockIdx.x; m < a.M && ok; m += gridDim.x) {
                for (int p = 0; p < 2 && ok; ++p) {
                    // p = 0: D = Xr T - T Xr (negate A of the second product);
                    // p = 1: D = Xi T + T (-Xi) (the B tile of Xi reads as -Xi)
                    const uint32_t id_tx = TF32 ? tc::idesc_tf32_f32(128, NP, p == 0) : tc::idesc_bf16_f32(128, NP, p == 0);
                    // one pass over K per 128-row accumulator tile, so that the epilogue
                    // of one tile runs while the MMAs of the other accumulate
                    for (int mt = 0; mt < 2 && ok; ++mt) {
                        if (!wait_bar(&sh->tempty[mt], (uu[mt] & 1) ^ 1, sh, a.err)) { ok = false; break; }
                        tc::tc_fence_after();
                        const uint32_t moff = mt * 16 * SBO;
                        const uint32_t d = tbase + mt * NP;
                        for (int kc = 0; kc < NCHE; ++kc, ++it) {
                            const int s = it % STAGES;
                            const uint32_t par = (it / STAGES) & 1;
                            if (!wait_bar(&sh->fullX[s], par, sh, a.err) || !wait_bar(&sh->fullT[s], par, sh, a.err)) {
                                ok = false;
                                break;
                            }
                            tc::tc_fence_after();
                            const uint32_t base = tc::smem_u32(stages + (size_t)s * STAGE_BYTES);
                            const uint32_t xh = base, xl = base + TILE_BYTES, th = base + 2 * TILE_BYTES,
                                           tl = base + 3 * TILE_BYTES;
#pragma unroll
                            for (int ks = 0; ks < 2; ++ks) {          // two 32-byte K steps per 64-byte chunk row
                                const uint32_t koff = ks * 2 * LBO;
                                const uint32_t acc0 = (kc > 0 || ks > 0) ? 1u : 0u;
                                auto mma = [](uint32_t dd, uint64_t ad, uint64_t bd, uint32_t id, uint32_t acc) {
                                    if constexpr (TF32) tc::mma_tf32(dd, ad, bd, id, acc);
                                    else tc::mma_bf16(dd, ad, bd, id, acc);
                                };
                                mma(d, tc::smem_desc(xh + moff + koff, LBO, SBO), tc::smem_desc(th + koff, LBO, SBO), id_xt, acc0);
                                mma(d, tc::smem_desc(xh + moff + koff, LBO, SBO), tc::smem_desc(tl + koff, LBO, SBO), id_xt, 1u);
                                mma(d, tc::smem_desc(xl + moff + koff, LBO, SBO), tc::smem_desc(th + koff, LBO, SBO), id_xt, 1u);
                                mma(d, tc::smem_desc(th + moff + koff, LBO, SBO), tc::smem_desc(xh + koff, LBO, SBO), id_tx, 1u);
                                mma(d, tc::smem_desc(th + moff + koff, LBO, SBO), tc::smem_desc(xl + koff, LBO, SBO), id_tx, 1u);
                                mma(d, tc::smem_desc(tl + moff + koff, LBO, SBO), tc::smem_desc(xh + koff, LBO, SBO), id_tx, 1u);
                            }
                            tc::mma_commit(&sh->empty[s]);
                        }
                        if (ok) tc::mma_commit(&sh->tfull[mt]);
                        ++uu[mt];
                    }
                }
            }
            // every MMA issued must be complete before tensor memory is freed
            tc::mma_commit(&sh->drain);
            for (uint32_t i = 0; i < (1u << 24); ++i)
                if (tc::mbar_try_wait(&sh->drain, 0)) break;
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue
        const int et = threadIdx.x;                 // 0 .. 32 N_EPI_WARPS - 1
        const int q4 = warp & 3, hh = warp >> 2;
        const DevSys<float>& sy = a.sys;
        int ue[2] = {0, 0}, mi = 0;              // uses of each accumulator tile
        bool ok = true;
        for (int m = blockIdx.x; m < a.M && ok; m += gridDim.x, ++mi) {
            const float* Xm = a.X + (size_t)m * mstride;
            const float* Xo = a.X + (size_t)(m ^ 1) * mstride;
            // Delta_jj = ((tM_jj + sum U (n_other + s)) + sum V (n_same + s)) + ext_jj + pulse proj_j
            for (int j = et; j < NP; j += N_EPI_WARPS * 32) {
                sh->nd[0][j] = j < a.n ? Xo[plane_off(j, j)] : 0.f;
                sh->nd[1][j] = j < a.n ? Xm[plane_off(j, j)] : 0.f;
            }
            tc::named_sync(1, N_EPI_WARPS * 32);
            for (int j = et; j < NP; j += N_EPI_WARPS * 32) {
                float dj = 0.f;
                if (j < a.n) {
                    dj = sy.tdiag[j];
                    if (a.Ud) {
                        // long-range Coulomb: U and V are symmetric, so thread j walks
                        // column j and the warp reads each row k contiguously
                        float uacc = 0.f, vacc = 0.f;
                        for (int k = 0; k < a.n; ++k) uacc += a.Ud[(size_t)k * NP + j] * (sh->nd[0][k] + sy.shift);
                        dj += uacc;
                        if (sy.coul == 2) {
                            for (int k = 0; k < a.n; ++k) vacc += a.Vd[(size_t)k * NP + j] * (sh->nd[1][k] + sy.shift);
                            dj += vacc;
                        }
                    } else if (sy.coul != 0) {
                        float uacc = 0.f;
                        for (int q = sy.up[j]; q < sy.up[j + 1]; ++q) uacc += sy.uv[q] * (sh->nd[0][sy.uk[q]] + sy.shift);
                        dj += uacc;
                        if (sy.coul == 2) {
                            float vacc = 0.f;
                            for (int q = sy.vp[j]; q < sy.vp[j + 1]; ++q) vacc += sy.vv[q] * (sh->nd[1][sy.vk[q]] + sy.shift);
                            dj += vacc;
                        }
                    }
                    if (sy.has_ext) dj += sy.ediag[j];
                    if (sy.n_bins > 0) dj += a.pulse * sy.proj[j];
                }
                sh->d[mi & 1][j] = dj;
            }
            tc::named_sync(1, N_EPI_WARPS * 32);
            const float* dd = sh->d[mi & 1];
            for (int p = 0; p < 2 && ok; ++p) {
                const int qp = 1 - p;                           // plane this pass updates
                const float* xp = Xm + (size_t)p * PLANE;
                const float* xq = Xm + (size_t)qp * PLANE;
                const float* p0 = a.P0 ? a.P0 + (size_t)m * mstride + (size_t)qp * PLANE : nullptr;
                const float* p1 = a.P1 ? a.P1 + (size_t)m * mstride + (size_t)qp * PLANE : nullptr;
                float* oq = a.out + (size_t)m * mstride + (size_t)qp * PLANE;
                const float sgn = p == 0 ? -1.f : 1.f;          // k_im = -(Dr + ...), k_re = Di + ...
#pragma unroll 1
                for (int mt = 0; mt < 2; ++mt) {
                    // one thread waits; the outcome is made uniform so that every
                    // epilogue thread takes the same named barriers
                    if (et == 0) sh->epi_ok[mt] = wait_bar(&sh->tfull[mt], ue[mt] & 1, sh, a.err) ? 1 : 0;
                    tc::named_sync(2, N_EPI_WARPS * 32);
                    if (!sh->epi_ok[mt]) { ok = false; break; }
                    ++ue[mt];
                    tc::tc_fence_after();
                    const int i = mt * 128 + q4 * 32 + lane;
                    const float di = dd[i];
#pragma unroll 1
                    for (int jb = 0; jb < EPI_COLS / EPI_BLK; ++jb) {
                        const int j0 = hh * EPI_COLS + jb * EPI_BLK;
                        // global loads first: their latency overlaps the tensor-memory read
                        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
                        float4 vp[EPI_BLK / 4], vq[EPI_BLK / 4], v0[EPI_BLK / 4], v1[EPI_BLK / 4];
#pragma unroll
                        for (int c = 0; c < EPI_BLK / 4; ++c) {
                            const int off = plane_off(i, j0 + 4 * c);
                            vp[c] = __ldcs(reinterpret_cast<const float4*>(xp + off));
                            vq[c] = __ldcs(reinterpret_cast<const float4*>(xq + off));
                            v0[c] = p0 ? __ldcs(reinterpret_cast<const float4*>(p0 + off)) : z4;
                            v1[c] = p1 ? __ldcs(reinterpret_cast<const float4*>(p1 + off)) : z4;
                        }
                        float acc[EPI_BLK];
                        tc::tmem_ld8(tbase + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(mt * NP + j0), acc);
                        const float* fp = reinterpret_cast<const float*>(vp);
                        const float* fq = reinterpret_cast<const float*>(vq);
                        const float* f0 = reinterpret_cast<const float*>(v0);
                        const float* f1 = reinterpret_cast<const float*>(v1);
                        float o[EPI_BLK];
#pragma unroll
                        for (int t = 0; t < EPI_BLK; ++t) {
                            const int j = j0 + t;
                            float v = acc[t] + fp[t] * (dd[j] - di);
                            if (p == 0 && i == j) v = 0.f;       // the imaginary diagonal stays zero
                            const float k = sgn * v;
                            o[t] = ((a.a0 * f0[t] + a.a1 * f1[t]) + a.ax * fq[t]) + a.hk * k;
                        }
#pragma unroll
                        for (int c = 0; c < EPI_BLK / 4; ++c)
                            *reinterpret_cast<float4*>(oq + plane_off(i, j0 + 4 * c)) =
                                make_float4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
                    }
                    tc::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&sh->tempty[mt]);
                }
            }
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == MMA_WARP) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tbase, TMEM_COLS);
    }
}

// canonical two-term tiles of T (zero diagonal) from a dense [NP][NP] FP32 matrix:
// bf16 hi/lo or tf32 big/small
template <bool TF32>
__global__ void k_dense_prep_T(const float* __restrict__ Tm, void* __restrict__ Tc)
{
    using MD = Mode<TF32>;
    using T = typename MD::T;
    constexpr int KCE = MD::KCE, EPC = MD::EPC, NCHE = NP / KCE, TILE_E = NP * KCE;
    T* out = reinterpret_cast<T*>(Tc);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < NP * NP; x += gridDim.x * blockDim.x) {
        const int r = x / NP, k = x - r * NP;
        const float v = (r == k) ? 0.f : Tm[x];
        const int kc = k / KCE, o = canon<EPC>(r, k - kc * KCE);
        if constexpr (TF32) {
            const float big = tc::round_tf32(v);
            out[(size_t)kc * TILE_E + o] = big;
            out[(size_t)(NCHE + kc) * TILE_E + o] = tc::round_tf32(v - big);
        } else {
            const __nv_bfloat16 hi = __float2bfloat16_rn(v);
            out[(size_t)kc * TILE_E + o] = hi;
            out[(size_t)(NCHE + kc) * TILE_E + o] = __float2bfloat16_rn(v - __bfloat162float(hi));
        }
    }
}

__global__ void k_dense_unpack(const cplx<double>* __restrict__ rho, int n, int M, float* __restrict__ X)
{
    const int ne = n * (n + 1) / 2;
    const long total = (long)M * NP * NP;
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total; x += (long)gridDim.x * blockDim.x) {
        const int m = (int)(x / (NP * NP));
        const int rem = (int)(x - (long)m * NP * NP);
        const int i = rem / NP, j = rem - i * NP;
        float re = 0.f, im = 0.f;
        if (i < n && j < n) {
            if (i <= j) {
                const cplx<double> v = rho[(size_t)m * ne + cs(j) + i];
                re = (float)v.re; im = (float)v.im;
            } else {
                const cplx<double> v = rho[(size_t)m * ne + cs(i) + j];
                re = (float)v.re; im = -(float)v.im;
            }
        }
        X[(size_t)m * 2 * PLANE + plane_off(i, j)] = re;
        X[(size_t)m * 2 * PLANE + PLANE + plane_off(i, j)] = im;
    }
}

template <typename R>
__global__ void k_dense_pack(const float* __restrict__ X, int n, int M, cplx<R>* __restrict__ rho)
{
    const int ne = n * (n + 1) / 2;
    const long total = (long)M * ne;
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total; x += (long)gridDim.x * blockDim.x) {
        const int m = (int)(x / ne), p = (int)(x - (long)m * ne);
        int j = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
        while (cs(j) > p) --j;
        while (cs(j + 1) <= p) ++j;
        const int i = p - cs(j);
        const size_t o = (size_t)m * 2 * PLANE + plane_off(i, j);
        rho[x] = cplx<R>{(R)X[o], (i == j) ? R(0) : (R)X[o + PLANE]};
    }
}

cudaError_t configure()
{
    cudaError_t e = cudaFuncSetAttribute(k_dense_stage<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stage_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_dense_stage<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_smem_bytes());
}

cudaError_t launch_stage(const DenseArgs& a, int grid, bool tf32, cudaStream_t st)
{
    if (tf32) k_dense_stage<true><<<grid, NTHREADS, stage_smem_bytes(), st>>>(a);
    else k_dense_stage<false><<<grid, NTHREADS, stage_smem_bytes(), st>>>(a);
    return cudaGetLastError();
}

cudaError_t prep_T(const float* T_full, void* Tc, bool tf32, cudaStream_t st)
{
    if (tf32) k_dense_prep_T<true><<<64, 256, 0, st>>>(T_full, Tc);
    else k_dense_prep_T<false><<<64, 256, 0, st>>>(T_full, Tc);
    return cudaGetLastError();
}

static int grid_for(long total) { return (int)std::max(1L, std::min(total / 256 + 1, 148L * 16)); }

cudaError_t unpack(const cplx<double>* rho, int n, int M, float* X, cudaStream_t st)
{
    k_dense_unpack<<<grid_for((long)M * NP * NP), 256, 0, st>>>(rho, n, M, X);
    return cudaGetLastError();
}

cudaError_t pack_f64(const float* X, int n, int M, cplx<double>* rho, cudaStream_t st)
{
    k_dense_pack<double><<<grid_for((long)M * n * (n + 1) / 2), 256, 0, st>>>(X, n, M, rho);
    return cudaGetLastError();
}

cudaError_t pack_f32(const float* X, int n, int M, cplx<float>* rho, cudaStream_t st)
{
    k_dense_pack<float><<<grid_for((long)M * n * (n + 1) / 2), 256, 0, st>>>(X, n, M, rho);
    return cudaGetLastError();
}

}  // namespace dense
}  // namespace fpsg
