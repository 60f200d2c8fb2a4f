// fpsg_kernels.cuh — the trajectory kernels (sm_100a).
//
//  k_stream_stage   one RK stage of all trajectories per launch; each CTA stages
//                   one spin matrix of one trajectory (packed, ne complex) in
//                   shared memory and runs the CSR commutator stencil on it.
//                   State lives in HBM.  Used for any n, and as the plain FP64 path.
//  k_resident       the whole time window per launch; each CTA (or 2-CTA cluster,
//                   one spin per CTA exchanging diagonals through distributed
//                   shared memory) keeps its trajectories in shared memory and
//                   registers for every step; HBM sees the state once per launch.
//  k_sample         product-state fTWA samples (src/FHfTWASolver.cpp:342-362).
//  reductions       deterministic fixed-order FP64 ensemble sums (Kahan).
#pragma once
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include "fpsg_device.cuh"

namespace fpsg {

namespace cg = cooperative_groups;

// observable record layout per snapshot: [du n][dd n][d2u n][d2d n][dud n][E 4]
__host__ __device__ __forceinline__ int rec_width(int n) { return 5 * n + 4; }

// ------------------------------------------------------------------ energies
// Per-matrix energy partials (fTWA: src/FHfTWASolver.cpp:399-411; HF onsite:
// src/FHHFSolver.cpp:375-391) for the spin matrix X; other = other spin (packed).
// e[0] += sum_ij N_ij tM_ij, e[1] += half of the opposite-spin term (spin-up
// matrices count both halves), e[2] += same-spin V term, e[3] += potential.
template <typename R>
__device__ __forceinline__ void energy_partials(const DevSys<R>& s, const cplx<R>* X, const cplx<R>* other,
                                                int spin, int do_e1, int do_e2, int lane, int nlanes,
                                                double e[4])
{
    const double shift = (double)s.shift;
    for (int j = lane; j < s.n; j += nlanes) {
        const double nj = (double)X[cs(j) + j].re + shift;
        double t0 = nj * (double)s.tdiag[j], t3 = 0.0;
        for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
            const int k = s.hk[q];
            if (k == j) continue;
            const double x = (double)getH<R>(X, k, j).re;
            t0 += x * (double)s.tv[q];
            if (s.has_ext) t3 += x * (double)s.xv[q];
        }
        e[0] += t0;
        if (s.has_ext) e[3] += nj * (double)s.ediag[j] + t3;
        if (do_e2) {
            double v = 0.0, fx = 0.0;
            for (int q = s.vp[j]; q < s.vp[j + 1]; ++q) {
                const int k = s.vk[q];
                v += (double)s.vv[q] * ((double)X[cs(k) + k].re + shift);
                if (s.fock) {   // exchange: V_jk N_jk N_kj = V_jk |N_jk|^2 (src/FHHFSolver.cpp:271-272)
                    const cplx<R> x = getH<R>(X, j, k);
                    fx += (double)s.vv[q] * ((double)x.re * (double)x.re + (double)x.im * (double)x.im);
                }
            }
            e[2] += 0.5 * (nj * v - fx);
        }
        if (do_e1 && spin == 0) {
            const double oj = (double)other[cs(j) + j].re + shift;
            double uo = 0.0, us = 0.0;
            for (int q = s.up[j]; q < s.up[j + 1]; ++q) {
                const int k = s.uk[q];
                uo += (double)s.uv[q] * ((double)other[cs(k) + k].re + shift);
                us += (double)s.uv[q] * ((double)X[cs(k) + k].re + shift);
            }
            e[1] += 0.5 * (nj * uo + oj * us);
        }
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ streaming stage
template <typename R>
struct StreamArgs {
    DevSys<R> sys;
    cplx<R>* rho; cplx<R>* A; cplx<R>* Bc;
    const cplx<R>* Xc; cplx<R>* Xn;
    int B, stage;
    R h, pulse;
    int record, do_e1, do_e2;
    double* diagbuf;   // [B][2][n]  per-trajectory diagonal at the snapshot
    double* ebuf;      // [B][2][4]  per-trajectory energy partials
    double2* whole;    // [2][ne] running sums of rho (or null)
    unsigned* err;
};

// One RK stage of spin matrix m (the body of the stream kernels).  GX = false
// stages the matrix in shared memory; GX = true reads it from global memory
// (through L1/L2) for n whose packed matrix exceeds shared memory.  Both do the
// same arithmetic in the same order.  Every thread of the CTA takes part.
template <typename R, bool GX>
__device__ __forceinline__ void stream_matrix(const StreamArgs<R>& a, int m, unsigned char* smem)
{
    const int n = a.sys.n, ne = a.sys.ne;
    cplx<R>* Xs = reinterpret_cast<cplx<R>*>(smem);
    const size_t xbytes = GX ? 0 : sizeof(cplx<R>) * ne;
    R* Dd = reinterpret_cast<R*>(smem + xbytes);
    double* red = reinterpret_cast<double*>(smem + ((xbytes + sizeof(R) * n + 15) & ~size_t(15)));
    const int s = m & 1;
    const cplx<R>* xg = a.Xc + (size_t)m * ne;
    const cplx<R>* xo = a.Xc + (size_t)(m ^ 1) * ne;
    const cplx<R>* X = GX ? xg : Xs;
    if (!GX)
        for (int p = threadIdx.x; p < ne; p += blockDim.x) Xs[p] = xg[p];
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) Dd[j] = delta_diag<R>(a.sys, j, X, xo, a.pulse);
    if (a.record) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double d = (double)X[cs(j) + j].re;
            if (!isfinite(d)) atomicOr(a.err, 1u);
            a.diagbuf[(size_t)m * n + j] = d;
        }
        double e[4] = {0.0, 0.0, 0.0, 0.0};
        energy_partials<R>(a.sys, X, xo, s, a.do_e1, a.do_e2, threadIdx.x, blockDim.x, e);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double v = warp_sum(e[c]);
            if (l == 0) red[w * 4 + c] = v;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double v = 0.0;
            for (int q = 0; q < nw; ++q) v += red[q * 4 + threadIdx.x];
            a.ebuf[(size_t)m * 4 + threadIdx.x] = v;
        }
        if (a.whole)
            for (int p = threadIdx.x; p < ne; p += blockDim.x) {
                atomicAdd(&a.whole[(size_t)s * ne + p].x, (double)X[p].re);
                atomicAdd(&a.whole[(size_t)s * ne + p].y, (double)X[p].im);
            }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < ne; p += blockDim.x) {
        const uint32_t ij = a.sys.pij[p];
        const int i = ij & 0xffff, j = ij >> 16;
        const cplx<R> k = commutator_elem<R>(a.sys, X, Dd, i, j);
        const size_t g = (size_t)m * ne + p;
        const cplx<R> z = {R(0), R(0)};
        cplx<R> rho = (a.stage == 0) ? X[p] : a.rho[g];
        cplx<R> A = (a.stage == 1 || a.stage == 2) ? a.A[g] : z;
        cplx<R> Bc = (a.stage >= 2) ? a.Bc[g] : z;
        cplx<R> Xn;
        rk_update<R>(a.stage, k, a.h, rho, A, Bc, Xn);
        if (a.stage == 0) { a.A[g] = A; a.Xn[g] = Xn; }
        else if (a.stage == 1) { a.A[g] = A; a.Bc[g] = Bc; a.Xn[g] = Xn; }
        else if (a.stage == 2) { a.Bc[g] = Bc; a.Xn[g] = Xn; }
        else { a.rho[g] = rho; }
    }
    __syncthreads();
}

template <typename R, bool GX = false>
__global__ void __launch_bounds__(256) k_stream_stage(StreamArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int M = a.B * 2;
    for (int m = blockIdx.x; m < M; m += gridDim.x) stream_matrix<R, GX>(a, m, smem);
}

// The stream stage over several systems at once: items[q] = (system, matrix),
// args[system] = that system's stage arguments.  One persistent launch walks the
// item list (ordered by the scheduler) with a grid stride.
template <typename R, bool GX = false>
__global__ void __launch_bounds__(512) k_batch_stage(const StreamArgs<R>* __restrict__ args,
                                                    const int2* __restrict__ items, int n_items)
{
    extern __shared__ __align__(16) unsigned char smem[];
    for (int q = blockIdx.x; q < n_items; q += gridDim.x) {
        const int2 it = items[q];
        stream_matrix<R, GX>(args[it.x], it.y, smem);
    }
}

// HF with distance Coulomb (src/FHHFSolver.cpp:575-608): Delta = tM + diag(U n_other
// + V n_same) - N o V (+ potential, pulse) is dense and complex.  Each CTA builds
// Delta of its matrix column-major in global scratch, with the additions in the
// oracle's order, then every packed element sums X_ik Delta_kj and X_kj Delta_ik
// over all k in ascending order (complex multiply-adds as four fma).
template <typename R>
struct FockArgs {
    StreamArgs<R> s;
    const R* tMf; const R* Uf; const R* Vf; const R* extf;   // dense real parts, col-major
    cplx<R>* D;                                               // [2B][n][n] scratch
};

template <typename R>
__device__ __forceinline__ void cmaddR(R& re, R& im, cplx<R> x, cplx<R> d)
{
    re = fmaR<R>(x.re, d.re, re);
    re = fmaR<R>(-x.im, d.im, re);
    im = fmaR<R>(x.re, d.im, im);
    im = fmaR<R>(x.im, d.re, im);
}

template <typename R>
__global__ void __launch_bounds__(256) k_fock_stage(FockArgs<R> f)
{
    const StreamArgs<R>& a = f.s;
    const int n = a.sys.n, ne = a.sys.ne;
    const int M = a.B * 2;
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const cplx<R>* X = a.Xc + (size_t)m * ne;
        const cplx<R>* xo = a.Xc + (size_t)(m ^ 1) * ne;
        cplx<R>* D = f.D + (size_t)m * n * n;
        if (a.record) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const double d = (double)X[cs(j) + j].re;
                if (!isfinite(d)) atomicOr(a.err, 1u);
                a.diagbuf[(size_t)m * n + j] = d;
            }
        }
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            R u = R(0), v = R(0);
            for (int k = 0; k < n; ++k) u = fmaR<R>(f.Uf[(size_t)k * n + j], addR<R>(xo[cs(k) + k].re, a.sys.shift), u);
            for (int k = 0; k < n; ++k) v = fmaR<R>(f.Vf[(size_t)k * n + j], X[cs(k) + k].re, v);
            const R pj = a.sys.n_bins > 0 ? mulR<R>(a.pulse, a.sys.proj[j]) : R(0);
            for (int i = 0; i < n; ++i) {
                cplx<R> d = {f.tMf[(size_t)j * n + i], R(0)};
                if (i == j && a.sys.coul != 0) d.re = addR<R>(d.re, u);
                const R vij = f.Vf[(size_t)j * n + i];
                const cplx<R> x = getH<R>(X, i, j);
                const R nvr = mulR<R>(x.re, vij), nvi = mulR<R>(x.im, vij);
                const R mre = (i == j) ? subR<R>(v, nvr) : subR<R>(R(0), nvr);
                const R mim = subR<R>(R(0), nvi);
                d.re = addR<R>(d.re, mre);
                d.im = addR<R>(d.im, mim);
                if (a.sys.has_ext) { d.re = addR<R>(d.re, f.extf[(size_t)j * n + i]); d.im = addR<R>(d.im, R(0)); }
                if (i == j && a.sys.n_bins > 0) d.re = addR<R>(d.re, pj);
                D[(size_t)j * n + i] = d;
            }
        }
        __syncthreads();
        if (a.record) {
            double e[4] = {0.0, 0.0, 0.0, 0.0};
            energy_partials<R>(a.sys, X, xo, m & 1, a.do_e1, a.do_e2, threadIdx.x, blockDim.x, e);
            __shared__ double red[32 * 4];
            const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double vv = warp_sum(e[c]);
                if (l == 0) red[w * 4 + c] = vv;
            }
            __syncthreads();
            if (threadIdx.x < 4) {
                double vv = 0.0;
                for (int q = 0; q < nw; ++q) vv += red[q * 4 + threadIdx.x];
                a.ebuf[(size_t)m * 4 + threadIdx.x] = vv;
            }
            if (a.whole)
                for (int p = threadIdx.x; p < ne; p += blockDim.x) {
                    atomicAdd(&a.whole[(size_t)(m & 1) * ne + p].x, (double)X[p].re);
                    atomicAdd(&a.whole[(size_t)(m & 1) * ne + p].y, (double)X[p].im);
                }
        }
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            R are = R(0), aim = R(0), bre = R(0), bim = R(0);
            for (int k = 0; k < n; ++k) cmaddR<R>(are, aim, getH<R>(X, i, k), D[(size_t)j * n + k]);
            for (int k = 0; k < n; ++k) cmaddR<R>(bre, bim, getH<R>(X, k, j), D[(size_t)k * n + i]);
            cplx<R> kk;
            kk.re = subR<R>(aim, bim);
            kk.im = -subR<R>(are, bre);
            const size_t g = (size_t)m * ne + p;
            const cplx<R> z = {R(0), R(0)};
            cplx<R> rho = (a.stage == 0) ? X[p] : a.rho[g];
            cplx<R> A = (a.stage == 1 || a.stage == 2) ? a.A[g] : z;
            cplx<R> Bc = (a.stage >= 2) ? a.Bc[g] : z;
            cplx<R> Xn;
            rk_update<R>(a.stage, kk, a.h, rho, A, Bc, Xn);
            if (a.stage == 0) { a.A[g] = A; a.Xn[g] = Xn; }
            else if (a.stage == 1) { a.A[g] = A; a.Bc[g] = Bc; a.Xn[g] = Xn; }
            else if (a.stage == 2) { a.Bc[g] = Bc; a.Xn[g] = Xn; }
            else { a.rho[g] = rho; }
        }
        __syncthreads();
    }
}

// record-only pass for the stream path (the last fTWA snapshot of a window is
// recorded by stage 0 anyway; HF's final snapshot has no step after it)
template <typename R>
__global__ void __launch_bounds__(256) k_stream_record(StreamArgs<R> a)
{
    __shared__ double red[32 * 4];
    const int n = a.sys.n, ne = a.sys.ne;
    const int M = a.B * 2;
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const int s = m & 1;
        const cplx<R>* X = a.Xc + (size_t)m * ne;
        const cplx<R>* xo = a.Xc + (size_t)(m ^ 1) * ne;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double d = (double)X[cs(j) + j].re;
            if (!isfinite(d)) atomicOr(a.err, 1u);
            a.diagbuf[(size_t)m * n + j] = d;
        }
        double e[4] = {0.0, 0.0, 0.0, 0.0};
        energy_partials<R>(a.sys, X, xo, s, a.do_e1, a.do_e2, threadIdx.x, blockDim.x, e);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double v = warp_sum(e[c]);
            if (l == 0) red[w * 4 + c] = v;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double v = 0.0;
            for (int q = 0; q < nw; ++q) v += red[q * 4 + threadIdx.x];
            a.ebuf[(size_t)m * 4 + threadIdx.x] = v;
        }
        if (a.whole)
            for (int p = threadIdx.x; p < ne; p += blockDim.x) {
                atomicAdd(&a.whole[(size_t)s * ne + p].x, (double)X[p].re);
                atomicAdd(&a.whole[(size_t)s * ne + p].y, (double)X[p].im);
            }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ resident
// One CTA holds M spin matrices for the whole launch (M = G trajectories of one
// spin in split mode — the other spin lives in the peer CTA of a 2-CTA cluster —
// or M = 2G, matrix m = 2g + s, otherwise).  Shared memory (32-bit offsets):
//   X   [2][n][RP] complex (+1 spare each)  double-buffered stacked columns:
//                                   X(m; i, k) at k*RP + m*n + i
//   rho [NT*EPT] complex            the state at the start of the step, by element
//   Dd  [M][n]                      Delta_jj of each matrix for the current stage
//   dg  [2][M n + 1]                diagonal of X, double-buffered like X; the
//                                   other spin (possibly in the peer CTA) reads it
//                                   for its Hartree term
//   es  [M][4] double               energy partials
//   ell [2P+1][n]                   Delta's column j as fixed-width entries, slot-major
//                                   (lanes reading column i of consecutive i hit
//                                   consecutive entries)
//                                   {k*RP, Delta_kj}: P below the diagonal
//                                   (zero-padded in front), the diagonal, P above
//                                   (zero-padded at the end)
// RP = M n rounded up to an odd number, so reads with stride RP (the transposed
// element X(m; j, i) of consecutive i) fall in distinct banks; the spare slot at
// n*RP absorbs the writes of threads that have no element, so the hot loop has no
// branches.
template <typename R>
struct ResArgs {
    DevSys<R> sys;
    cplx<R>* state;       // [B][2][ne]
    int B, G;             // trajectories, trajectories per CTA (per cluster when split)
    R h;
    const R* ptab;        // pulse value per (step, stage), from the launch's first step
    long step_base;
    int t_begin, t_end, S, Tp, hf;
    int record, do_en, do_e1, do_e2;
    const int* ell_k;     // [n][2P+1] row index k of each entry, -1 for padding
    const R* ell_v;       // [n][2P+1] Delta_kj (0 for padding; diagonal slot unused)
    const int* ell_pad;   // [2P+1] dominant offset k - j of each slot
    double* slots;        // [gridDim.x][Tp][W]
    double2* whole;       // [Tp][2][ne] or null
    unsigned* err;
    // optional: every step's four stage inputs, [step][4][B][2][ne] packed (the
    // adjoint's segment recompute); null = not kept
    cplx<R>* dump;
    size_t dump_count;    // B * 2 * ne
    // Delta_jj of the next stage written by the pass itself (on-site or no Coulomb
    // term): U_jj per site, 0 where U has no entry in row j; null = not used
    const R* udiag;
    // element (i | j << 16) of each of a matrix's ne slots: full 32-row column
    // segments first, so that most warps read one column of X (no bank conflicts),
    // then the 32 x 32 diagonal blocks
    const uint32_t* order;
    // FP32 stages only: when set, the launch reads and writes the state here, in
    // FP64 ([B][2][ne], the context's master copy), instead of `state`, and
    // compensates the state update: each element is kept as its FP32 value plus
    // the rounding residual of the last update (a bf16 pair in shared memory), and
    // hi + lo goes back to FP64 at the end of the launch
    cplx<double>* state64 = nullptr;
};

// bf16 pair <-> float pair (low half = first value); bf16 -> float is exact
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16x2(uint32_t u)
{
    return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}

// The last RK stage with a compensated state update (FP32):
//     d = (Bc + k4) h/8 + lo,   rho' = fl(rho + d),   lo' = (rho + d) - rho'
// (the residual by Knuth's TwoSum, exact in FP32, then kept as bf16).  Without
// it the update loses the low bits of d every step, about 2^-25 |rho|, which at
// h = 0.005 is some 50 times the rounding the stage arithmetic itself commits.
__device__ __forceinline__ void rk_final_comp(cplx<float> k, float h, cplx<float>& rho, uint32_t& lo2,
                                              const cplx<float>& Bc)
{
    const float2 lo = unpack_bf16x2(lo2);
    const float hs = h * 0.125f;
    const float dre = __fmaf_rn(__fadd_rn(Bc.re, k.re), hs, lo.x);
    const float dim = __fmaf_rn(__fadd_rn(Bc.im, k.im), hs, lo.y);
    const float sre = __fadd_rn(rho.re, dre), sim = __fadd_rn(rho.im, dim);
    const float bre = __fsub_rn(sre, rho.re), bim = __fsub_rn(sim, rho.im);
    const float rre = __fadd_rn(__fsub_rn(rho.re, __fsub_rn(sre, bre)), __fsub_rn(dre, bre));
    const float rim = __fadd_rn(__fsub_rn(rho.im, __fsub_rn(sim, bim)), __fsub_rn(dim, bim));
    rho.re = sre;
    rho.im = sim;
    lo2 = pack_bf16x2(rre, rim);
}

// where a resident element's value goes in a packed [B][2][ne] buffer
struct DumpMap {
    int gbase, rank, B, ne, split;
};

// packed upper-triangle index cs(j) + i of a resident element code i | j << 10 | m << 20
__device__ __forceinline__ int res_packed(uint32_t code)
{
    const int i = (int)(code & 1023u), j = (int)((code >> 10) & 1023u);
    return ((j * (j + 1)) >> 1) + i;
}

template <typename R> struct Ent;
template <> struct __align__(8) Ent<float> { int off; float v; };
template <> struct __align__(16) Ent<double> { int off; int pad; double v; };

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template <typename R>
struct ResLayout {
    size_t x, rho, dd, dg, es, ell, lo, xs, sd, total;
};

// Delta_jj from diagonal arrays (same spin, other spin), order as delta_diag.
template <typename R>
__device__ __forceinline__ R delta_diag_v(const DevSys<R>& s, int j, const R* same, const R* other, R pulse)
{
    R d = s.tdiag[j];
    if (s.coul != 0) {
        R u = R(0);
        for (int q = s.up[j]; q < s.up[j + 1]; ++q)
            u = fmaR<R>(s.uv[q], addR<R>(other[s.uk[q]], s.shift), u);
        d = addR<R>(d, u);
        if (s.coul == 2) {
            R v = R(0);
            for (int q = s.vp[j]; q < s.vp[j + 1]; ++q)
                v = fmaR<R>(s.vv[q], addR<R>(same[s.vk[q]], s.shift), v);
            d = addR<R>(d, v);
        }
    }
    if (s.has_ext) d = addR<R>(d, s.ediag[j]);
    if (s.n_bins > 0) d = addR<R>(d, mulR<R>(pulse, s.proj[j]));
    return d;
}

// energy partials of one matrix in the stacked layout (see energy_partials)
template <typename R>
__device__ __forceinline__ void energy_partials_full(const DevSys<R>& s, const cplx<R>* X, int RP, int row0,
                                                     const R* dsame, const R* dother, int spin, int do_e1,
                                                     int do_e2, int lane, int nlanes, double e[4])
{
    const double shift = (double)s.shift;
    for (int j = lane; j < s.n; j += nlanes) {
        const double nj = (double)dsame[j] + shift;
        double t0 = nj * (double)s.tdiag[j], t3 = 0.0;
        for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
            const int k = s.hk[q];
            if (k == j) continue;
            const double x = (double)X[j * RP + row0 + k].re;
            t0 += x * (double)s.tv[q];
            if (s.has_ext) t3 += x * (double)s.xv[q];
        }
        e[0] += t0;
        if (s.has_ext) e[3] += nj * (double)s.ediag[j] + t3;
        if (do_e2) {
            double v = 0.0;
            for (int q = s.vp[j]; q < s.vp[j + 1]; ++q) v += (double)s.vv[q] * ((double)dsame[s.vk[q]] + shift);
            e[2] += 0.5 * nj * v;
        }
        if (do_e1 && spin == 0) {
            const double oj = (double)dother[j] + shift;
            double uo = 0.0, us = 0.0;
            for (int q = s.up[j]; q < s.up[j + 1]; ++q) {
                uo += (double)s.uv[q] * ((double)dother[s.uk[q]] + shift);
                us += (double)s.uv[q] * ((double)dsame[s.uk[q]] + shift);
            }
            e[1] += 0.5 * (nj * uo + oj * us);
        }
    }
}

// Each thread
// evaluates, for its own upper-triangle element (i, j),
//     C_ij = sum_{k in col(j)} X_ik Delta_kj   (column j's fixed-width entries:
//            warp-uniform broadcasts, X(k, rows) contiguous across the warp)
//     C_ji = sum_{k in col(i)} X_jk Delta_ki   (column i's entries per lane; the
//            reads X(k, j) are strided by the odd RP, so they hit distinct banks)
// both in ascending k (oracle order), then dX_ij = -i (C_ij - conj(C_ji)).  X is
// double-buffered: the pass reads X[cur] and writes X[cur ^ 1].
template <typename R>
__host__ __device__ __forceinline__ ResLayout<R> res_layout_direct(int n, int M, int P, int nt_ept, bool comp = false)
{
    ResLayout<R> L;
    const size_t RP = (size_t)((M * n) | 1);
    size_t o = 0;
    L.x = o;    o = align16(o + sizeof(cplx<R>) * 2 * ((size_t)n * RP + 1));
    L.rho = o;  o = align16(o + sizeof(cplx<R>) * (size_t)nt_ept);
    L.dd = o;   o = align16(o + sizeof(R) * 2 * (size_t)M * n);   // double-buffered
    L.dg = o;   o = align16(o + sizeof(R) * 2 * ((size_t)M * n + 1));
    L.es = o;   o = align16(o + sizeof(double) * 4 * ((size_t)M + 32));   // per matrix, then per warp
    L.ell = o;  o = align16(o + sizeof(Ent<R>) * (size_t)n * (2 * P + 1));
    L.lo = o;   if (comp) o = align16(o + sizeof(uint32_t) * (size_t)nt_ept);   // bf16 residual pairs
    L.total = o;
    return L;
}

// Next-stage diagonal written by the pass: the thread that owns (j, j) of one spin
// matrix forms Delta_jj of the partner spin's matrix for the next stage, in the
// order of delta_diag_v with only an on-site U term (one entry U_jj, or none):
//     ((tM_jj + U_jj (n_jj + shift)) + extPot_jj) + pulse * proj_j
struct DdNext {
    void* dst;      // partner's Delta_jj buffer of the next stage (null: not written)
    int pxor;       // partner matrix = m ^ pxor within dst (0: the peer CTA, same m)
};

template <typename R, int NT, int EPT, int STAGE, int P, bool DUMP>
__device__ __forceinline__ void res_direct_pass(const cplx<R>* __restrict__ X, cplx<R>* __restrict__ Xn,
                                                const Ent<R>* __restrict__ ell, const R* __restrict__ Dd,
                                                cplx<R>* __restrict__ rhoS, R* __restrict__ dgn,
                                                const uint32_t (&ix)[EPT], cplx<R> (&Ar)[EPT], cplx<R> (&Br)[EPT],
                                                R h, int tid, int n, int RP, int spare, int dgspare,
                                                cplx<R>* __restrict__ dump_in, cplx<R>* __restrict__ dump_out,
                                                const DumpMap dm, const DdNext dnx, const DevSys<R>& sys,
                                                const R* __restrict__ udiag, R pvn, uint32_t* __restrict__ loS)
{
    constexpr int NE = 2 * P + 1;
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        const bool valid = ix[q] != ~0u;
        const int i = valid ? (int)(ix[q] & 1023u) : 0;
        const int j = valid ? (int)((ix[q] >> 10) & 1023u) : 0;
        const int row0 = valid ? (int)(ix[q] >> 20) * n : 0;
        const int bi = row0 + i, bj = row0 + j;
        // C_ij over column j
        const Ent<R>* ej = ell + j;          // entry s of column j at ej[s * n]
        const Ent<R>* ei = ell + i;
        R are = R(0), aim = R(0), bre = R(0), bim = R(0);
#pragma unroll
        for (int s = 0; s < P; ++s) {
            const Ent<R> e = ej[s * n];
            const cplx<R> x = X[e.off + bi];
            are = fmaR<R>(x.re, e.v, are);
            aim = fmaR<R>(x.im, e.v, aim);
        }
        // the diagonal terms: FP64 sums them in place (the oracle's order); FP32 forms
        // X_ij (Delta_jj - Delta_ii) once after the off-diagonal sums, so the two large
        // diagonal products no longer cancel in the difference C_ij - conj(C_ji)
        constexpr bool kDiagApart = std::is_same<R, float>::value;
        if constexpr (!kDiagApart) {
            const R d = Dd[bj];
            const cplx<R> x = X[j * RP + bi];
            are = fmaR<R>(x.re, d, are);
            aim = fmaR<R>(x.im, d, aim);
        }
#pragma unroll
        for (int s = P + 1; s < NE; ++s) {
            const Ent<R> e = ej[s * n];
            const cplx<R> x = X[e.off + bi];
            are = fmaR<R>(x.re, e.v, are);
            aim = fmaR<R>(x.im, e.v, aim);
        }
        // C_ji over column i
#pragma unroll
        for (int s = 0; s < P; ++s) {
            const Ent<R> e = ei[s * n];
            const cplx<R> x = X[e.off + bj];
            bre = fmaR<R>(x.re, e.v, bre);
            bim = fmaR<R>(x.im, e.v, bim);
        }
        if constexpr (!kDiagApart) {
            const R d = Dd[bi];
            const cplx<R> x = X[i * RP + bj];
            bre = fmaR<R>(x.re, d, bre);
            bim = fmaR<R>(x.im, d, bim);
        }
#pragma unroll
        for (int s = P + 1; s < NE; ++s) {
            const Ent<R> e = ei[s * n];
            const cplx<R> x = X[e.off + bj];
            bre = fmaR<R>(x.re, e.v, bre);
            bim = fmaR<R>(x.im, e.v, bim);
        }
        if constexpr (kDiagApart) {
            const cplx<R> x = X[j * RP + bi];             // this element, X_ij
            const R dd = Dd[bj] - Dd[bi];
            are = fmaR<R>(x.re, dd, are);
            aim = fmaR<R>(x.im, dd, aim);
        }
        cplx<R> k;
        k.re = subR<R>(aim, -bim);
        k.im = -subR<R>(are, bre);
        cplx<R> rho = rhoS[f];
        cplx<R> xn;
        size_t gidx = ~size_t(0);
        if constexpr (DUMP) {
            if (valid) {
                const int m = (int)(ix[q] >> 20);
                const int g = dm.split ? m : (m >> 1), s = dm.split ? dm.rank : (m & 1);
                const int b = dm.gbase + g;
                if (b < dm.B) gidx = ((size_t)b * 2 + s) * dm.ne + (size_t)res_packed(ix[q]);
            }
            if (STAGE == 0 && gidx != ~size_t(0)) dump_in[gidx] = rho;      // stage input X1 = rho
        }
        if constexpr (STAGE == 3 && std::is_same<R, float>::value) {
            if (loS != nullptr) {
                rk_final_comp(k, h, rho, loS[f], Br[q]);
                xn = rho;
            } else {
                rk_update<R>(STAGE, k, h, rho, Ar[q], Br[q], xn);
            }
        } else {
            rk_update<R>(STAGE, k, h, rho, Ar[q], Br[q], xn);
        }
        if constexpr (DUMP)
            if (STAGE < 3 && gidx != ~size_t(0)) dump_out[gidx] = xn;       // next stage input
        if (STAGE == 3) rhoS[f] = rho;
        const int oij = valid ? j * RP + bi : spare;
        const int oji = valid ? i * RP + bj : spare;
        Xn[oji] = cplx<R>{xn.re, -xn.im};
        Xn[oij] = xn;                         // on the diagonal this second store wins
        if (valid && i == j) {
            dgn[bi] = xn.re;
            if (dnx.dst != nullptr) {
                R d = sys.tdiag[i];
                if (sys.coul != 0) {
                    R u = R(0);
                    const R uu = udiag[i];
                    if (uu != R(0)) u = fmaR<R>(uu, addR<R>(xn.re, sys.shift), u);
                    d = addR<R>(d, u);
                }
                if (sys.has_ext) d = addR<R>(d, sys.ediag[i]);
                if (sys.n_bins > 0) d = addR<R>(d, mulR<R>(pvn, sys.proj[i]));
                const int m = (int)(ix[q] >> 20);
                static_cast<R*>(dnx.dst)[(m ^ dnx.pxor) * n + i] = d;
            }
        }
        (void)dgspare;
    }
}

// DUMP = true: the adjoint's recompute variant, which also writes every stage
// input to a.dump
template <typename R, int NT, int EPT, bool SPLIT, int P, bool DUMP = false>
__global__ void __launch_bounds__(NT, 1) k_resident(ResArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    const int M = SPLIT ? a.G : 2 * a.G;
    const int RR = M * n;
    const int RP = RR | 1;
    const int E = M * ne;
    const int DGS = RR + 1;
    const int XS = n * RP + 1;               // X buffer stride (spare slot at n*RP)
    const int SPARE = n * RP;
    constexpr int NE = 2 * P + 1;
    const bool comp = std::is_same<R, float>::value && a.state64 != nullptr;
    const ResLayout<R> L = res_layout_direct<R>(n, M, P, NT * EPT, comp);
    uint32_t* loS = comp ? reinterpret_cast<uint32_t*>(smem + L.lo) : nullptr;
    cplx<R>* Xb = reinterpret_cast<cplx<R>*>(smem + L.x);
    cplx<R>* rhoS = reinterpret_cast<cplx<R>*>(smem + L.rho);
    R* Dd = reinterpret_cast<R*>(smem + L.dd);
    R* dg = reinterpret_cast<R*>(smem + L.dg);
    double* es = reinterpret_cast<double*>(smem + L.es);
    Ent<R>* ell = reinterpret_cast<Ent<R>*>(smem + L.ell);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    static_assert(NW <= 32, "the per-warp energy partials (es) have room for 32 warps");
    const int W = rec_width(n);

    // Padding entries (value 0) read an in-buffer address congruent mod 16 to the
    // slot's dominant neighbour column, so neighbouring lanes keep distinct banks.
    const bool pad_room = n * RP >= RR + 16;
    for (int q = tid; q < n * NE; q += NT) {
        Ent<R> e;
        const int k = a.ell_k[q], col = q / NE, slot = q - col * NE;
        if (k >= 0) e.off = k * RP;
        else if (pad_room) e.off = ((((col + a.ell_pad[slot]) * RP) % 16) + 16) % 16;
        else e.off = col * RP;
        e.v = a.ell_v[q];
        if constexpr (sizeof(Ent<R>) == 16) reinterpret_cast<int*>(&e)[1] = 0;
        ell[slot * n + col] = e;
    }

    int rank = 0, cid = blockIdx.x, ncl = gridDim.x;
    R* peer_dg = nullptr;
    R* peer_dd = Dd;
    if constexpr (SPLIT) {
        cg::cluster_group cl = cg::this_cluster();
        rank = (int)cl.block_rank();
        cid = blockIdx.x >> 1;
        ncl = gridDim.x >> 1;
        peer_dg = cl.map_shared_rank(dg, rank ^ 1);
        peer_dd = cl.map_shared_rank(Dd, rank ^ 1);
    }
    auto bar = [&]() {
        if constexpr (SPLIT) cg::this_cluster().sync(); else __syncthreads();
    };
    auto other_dg = [&](int p, int m) -> const R* {
        if constexpr (SPLIT) return peer_dg + p * DGS + m * n;
        else return dg + p * DGS + (m ^ 1) * n;
    };

    cplx<R> Ar[EPT], Br[EPT];
    uint32_t ix[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        uint32_t v = ~0u;
        if (f < E) {
            const int m = f / ne;
            const uint32_t p = a.order[f - m * ne];
            v = (p & 0xffffu) | ((p >> 16) << 10) | ((uint32_t)m << 20);
        }
        ix[q] = v;
    }
    double* myslot = a.slots ? a.slots + (size_t)blockIdx.x * a.Tp * W : nullptr;
    // rows past M*n (the odd-stride padding row) are never written by the passes but
    // may be read by zero-weight padding entries: start them at zero
    for (int q = tid; q < 2 * XS; q += NT) Xb[q] = cplx<R>{R(0), R(0)};

    const int ngroups = (a.B + a.G - 1) / a.G;
    __syncthreads();
    for (int gid = cid; gid < ngroups; gid += ncl) {
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            cplx<R> v = {R(0), R(0)};
            uint32_t lo = 0;
            if (ix[q] != ~0u) {
                const int i = ix[q] & 1023u, j = (ix[q] >> 10) & 1023u, m = ix[q] >> 20;
                const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
                const int b = gid * a.G + g;
                if (b < a.B) {
                    const size_t gi = ((size_t)b * 2 + s) * ne + res_packed(ix[q]);
                    if (comp) {
                        const cplx<double> x = a.state64[gi];
                        v.re = (R)x.re;
                        v.im = (R)x.im;
                        lo = pack_bf16x2((float)(x.re - (double)v.re), (float)(x.im - (double)v.im));
                    } else {
                        v = a.state[gi];
                    }
                }
                Xb[j * RP + m * n + i] = v;
                Xb[i * RP + m * n + j] = cplx<R>{v.re, -v.im};
                Xb[j * RP + m * n + i] = v;
                if (i == j) dg[m * n + i] = v.re;
            }
            rhoS[f] = v;
            if (comp) loS[f] = lo;
            Ar[q] = v; Br[q] = v;
        }
        int cur = 0, dcur = 0;
        bool dd_ok = false;                  // Dd[dcur] already holds this stage's diagonal
        long gstep = a.step_base;
        bar();
        for (int t = a.t_begin; t < a.t_end; ++t) {
            if (a.record) {
                const cplx<R>* X = Xb + cur * XS;
                const R* d0 = dg + cur * DGS;
                const int nvec = SPLIT ? (rank == 0 ? 3 : 2) : 5;
                for (int w = tid; w < nvec * n; w += NT) {
                    const int oo = w / n, j = w - oo * n;
                    int o;
                    if (SPLIT) o = rank == 0 ? (oo == 0 ? 0 : oo == 1 ? 2 : 4) : (oo == 0 ? 1 : 3);
                    else o = oo;
                    double acc = 0.0;
                    for (int g = 0; g < a.G; ++g) {
                        if (gid * a.G + g >= a.B) break;
                        double du, dd;
                        if (SPLIT) {
                            const double mine = (double)d0[g * n + j], oth = (double)other_dg(cur, g)[j];
                            du = rank == 0 ? mine : oth;
                            dd = rank == 0 ? oth : mine;
                        } else {
                            du = (double)d0[(2 * g) * n + j];
                            dd = (double)d0[(2 * g + 1) * n + j];
                        }
                        if (!isfinite(du) || !isfinite(dd)) atomicOr(a.err, 1u);
                        acc += o == 0 ? du : o == 1 ? dd : o == 2 ? du * du : o == 3 ? dd * dd : du * dd;
                    }
                    atomicAdd(myslot + (size_t)t * W + o * n + j, acc);
                }
                if (a.do_en) {
                    // every thread of the CTA works on each matrix in turn
                    double* ew = es + 4 * M;              // per-warp partials
                    for (int m = 0; m < M; ++m) {
                        const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
                        double e[4] = {0.0, 0.0, 0.0, 0.0};
                        energy_partials_full<R>(a.sys, X, RP, m * n, d0 + m * n, other_dg(cur, m), s, a.do_e1,
                                                a.do_e2, tid, NT, e);
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const double v = warp_sum(e[c]);
                            if (lane == 0) ew[warp * 4 + c] = v;
                        }
                        __syncthreads();
                        if (tid < 4) {
                            double v = 0.0;
                            for (int q = 0; q < NW; ++q) v += ew[q * 4 + tid];
                            es[m * 4 + tid] = (gid * a.G + g < a.B) ? v : 0.0;
                        }
                        __syncthreads();
                    }
                    if (tid < 4) {
                        double acc = 0.0;
                        for (int m = 0; m < M; ++m) acc += es[m * 4 + tid];
                        atomicAdd(myslot + (size_t)t * W + 5 * n + tid, acc);
                    }
                }
                if (a.whole) {
#pragma unroll
                    for (int q = 0; q < EPT; ++q) {
                        const int f = tid + q * NT;
                        if (f >= E) continue;
                        const int m = f / ne;
                        const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
                        if (gid * a.G + g >= a.B) continue;
                        const int p = res_packed(ix[q]);
                        atomicAdd(&a.whole[((size_t)t * 2 + s) * ne + p].x, (double)rhoS[f].re);
                        atomicAdd(&a.whole[((size_t)t * 2 + s) * ne + p].y, (double)rhoS[f].im);
                    }
                }
            }
            const int nsteps = (a.hf && t == a.Tp - 1) ? 0 : a.S;
            for (int st = 0; st < nsteps; ++st, ++gstep) {
#pragma unroll
                for (int stage = 0; stage < 4; ++stage) {
                    R* Dc = Dd + dcur * RR;
                    if (!dd_ok) {
                        const R pv = a.sys.n_bins > 0 ? a.ptab[(gstep - a.step_base) * 4 + stage] : R(0);
                        for (int w = tid; w < RR; w += NT) {
                            const int m = w / n, j = w - m * n;
                            Dc[w] = delta_diag_v<R>(a.sys, j, dg + cur * DGS + m * n, other_dg(cur, m), pv);
                        }
                        __syncthreads();
                    }
                    // does another stage follow in this launch (possibly after a record)?
                    const bool more = stage < 3 || st + 1 < nsteps ||
                                      (t + 1 < a.t_end && a.S > 0 && !(a.hf && t + 1 == a.Tp - 1));
                    DdNext dnx = {nullptr, SPLIT ? 0 : 1};
                    R pvn = R(0);
                    if (a.udiag != nullptr && more) {
                        dnx.dst = (SPLIT ? peer_dd : Dd) + (dcur ^ 1) * RR;
                        if (a.sys.n_bins > 0) pvn = a.ptab[(gstep - a.step_base) * 4 + stage + 1];
                    }
                    const cplx<R>* X = Xb + cur * XS;
                    cplx<R>* Xn = Xb + (cur ^ 1) * XS;
                    R* dgn = dg + (cur ^ 1) * DGS;
                    cplx<R>* din = nullptr;
                    cplx<R>* dout = nullptr;
                    if (DUMP && a.dump) {
                        din = a.dump + (size_t)(gstep - a.step_base) * 4 * a.dump_count;
                        dout = din + (size_t)(stage + 1) * a.dump_count;
                    }
                    const DumpMap dm = {gid * a.G, rank, a.B, ne, SPLIT ? 1 : 0};
                    if (stage == 0) res_direct_pass<R, NT, EPT, 0, P, DUMP>(X, Xn, ell, Dc, rhoS, dgn, ix, Ar, Br, a.h, tid, n, RP, SPARE, RR, din, dout, dm, dnx, a.sys, a.udiag, pvn, loS);
                    else if (stage == 1) res_direct_pass<R, NT, EPT, 1, P, DUMP>(X, Xn, ell, Dc, rhoS, dgn, ix, Ar, Br, a.h, tid, n, RP, SPARE, RR, din, dout, dm, dnx, a.sys, a.udiag, pvn, loS);
                    else if (stage == 2) res_direct_pass<R, NT, EPT, 2, P, DUMP>(X, Xn, ell, Dc, rhoS, dgn, ix, Ar, Br, a.h, tid, n, RP, SPARE, RR, din, dout, dm, dnx, a.sys, a.udiag, pvn, loS);
                    else res_direct_pass<R, NT, EPT, 3, P, DUMP>(X, Xn, ell, Dc, rhoS, dgn, ix, Ar, Br, a.h, tid, n, RP, SPARE, RR, din, dout, dm, dnx, a.sys, a.udiag, pvn, loS);
                    bar();
                    cur ^= 1;
                    dcur ^= 1;
                    dd_ok = dnx.dst != nullptr;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            if (f >= E) continue;
            const int m = f / ne;
            const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
            const int b = gid * a.G + g;
            if (b < a.B) {
                const size_t gi = ((size_t)b * 2 + s) * ne + res_packed(ix[q]);
                if (comp) {
                    const float2 lo = unpack_bf16x2(loS[f]);
                    a.state64[gi] = cplx<double>{(double)rhoS[f].re + (double)lo.x, (double)rhoS[f].im + (double)lo.y};
                } else {
                    a.state[gi] = rhoS[f];
                }
            }
        }
        bar();
    }
}

}  // namespace fpsg
