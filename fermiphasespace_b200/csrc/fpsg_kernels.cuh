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
        double t0 = nj * (double)s.tdiag[j];
        for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
            const int k = s.hk[q];
            if (k == j) continue;
            t0 += (double)getH<R>(X, k, j).re * (double)s.hv[q];
        }
        e[0] += t0;
        if (s.has_ext) e[3] += nj * (double)s.ediag[j];
        if (do_e2) {
            double v = 0.0;
            for (int q = s.vp[j]; q < s.vp[j + 1]; ++q) {
                const int k = s.vk[q];
                v += (double)s.vv[q] * ((double)X[cs(k) + k].re + shift);
            }
            e[2] += 0.5 * nj * v;
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

template <typename R>
__global__ void __launch_bounds__(256) k_stream_stage(StreamArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    cplx<R>* X = reinterpret_cast<cplx<R>*>(smem);
    R* Dd = reinterpret_cast<R*>(X + ne);
    double* red = reinterpret_cast<double*>(smem + ((sizeof(cplx<R>) * ne + sizeof(R) * n + 15) & ~size_t(15)));
    const int M = a.B * 2;
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const int b = m >> 1, s = m & 1;
        const cplx<R>* xg = a.Xc + (size_t)m * ne;
        const cplx<R>* xo = a.Xc + (size_t)(m ^ 1) * ne;
        for (int p = threadIdx.x; p < ne; p += blockDim.x) X[p] = xg[p];
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
        (void)b;
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

// ---- per-snapshot fixed-order reduction of the per-trajectory buffers
// part[c][w] = sum over trajectories of chunk c (ascending) of the record values.
__global__ void k_reduce_part(const double* __restrict__ diagbuf, const double* __restrict__ ebuf,
                              int B, int n, int chunk, double* __restrict__ part)
{
    const int W = rec_width(n);
    const int c = blockIdx.x;
    const int b0 = c * chunk, b1 = min(B, b0 + chunk);
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        double acc = 0.0;
        if (w < 5 * n) {
            const int o = w / n, j = w - o * n;
            for (int b = b0; b < b1; ++b) {
                const double du = diagbuf[((size_t)b * 2) * n + j];
                const double dd = diagbuf[((size_t)b * 2 + 1) * n + j];
                acc += o == 0 ? du : o == 1 ? dd : o == 2 ? du * du : o == 3 ? dd * dd : du * dd;
            }
        } else {
            const int e = w - 5 * n;
            for (int b = b0; b < b1; ++b) acc += ebuf[((size_t)b * 2) * 4 + e] + ebuf[((size_t)b * 2 + 1) * 4 + e];
        }
        part[(size_t)c * W + w] = acc;
    }
}

// out[w] = Kahan sum over c of part[c][w] (c ascending)
__global__ void k_reduce_fin(const double* __restrict__ part, int nchunks, int W, double* __restrict__ out)
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

// ------------------------------------------------------------------ resident
// One CTA holds M spin matrices for the whole launch (M = G trajectories of one
// spin in split mode — the other spin lives in the peer CTA of a 2-CTA cluster —
// or M = 2G, matrix m = 2g + s, otherwise).  Shared memory (32-bit offsets):
//   X   [n][RP] complex (+1 spare)  column k of all M matrices stacked:
//                                   X(m; i, k) at k*RP + m*n + i
//   C   [n][RP] complex (+1 spare)  C = X Delta, same layout
//   rho [NT*EPT] complex            the state at the start of the step, by element
//   Dd  [M][n]                      Delta_jj of each matrix for the current stage
//   dg  [2][M n + 1]                diagonal of X, double-buffered by stage parity;
//                                   the other spin (possibly in the peer CTA)
//                                   reads it for its Hartree term
//   es  [M][4] double               energy partials
//   ell [n][2P+1]                   Delta's column j as fixed-width entries
//                                   {k*RP, Delta_kj}: P below the diagonal
//                                   (zero-padded in front), the diagonal, P above
//                                   (zero-padded at the end)
// RP = M n rounded up to an odd number so that the transposed reads C(m; j, i)
// of the element pass fall in distinct banks; the spare slot at n*RP absorbs the
// writes of lanes and elements that have no work, so the hot loops have no
// branches.
//
// A stage is three passes:
//   (1) Dd from dg;
//   (2) C = X Delta, a sparse-times-dense product: a warp owns 32 stacked rows
//       and one column j, so the 2P+1 terms of col(j) are warp-uniform shared
//       memory broadcasts and the reads X(k, rows) are contiguous; terms are
//       summed in ascending k (the oracle's order; zero padding adds exact zeros);
//   (3) per upper-triangle element (A and Bc of the RK combination in registers):
//       dX_ij = -i (C_ij - conj(C_ji))  [= -i (X Delta - Delta X)_ij for Hermitian
//       X and real symmetric Delta], RK update, X_ij and its mirror written back.
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
    const int* ell_k;     // [n][2P+1] row index k of each entry (j itself for padding)
    const R* ell_v;       // [n][2P+1] Delta_kj (0 for padding; diagonal slot unused)
    double* slots;        // [gridDim.x][Tp][W]
    double2* whole;       // [Tp][2][ne] or null
    unsigned* err;
};

template <typename R> struct Ent;
template <> struct __align__(8) Ent<float> { int off; float v; };
template <> struct __align__(16) Ent<double> { int off; int pad; double v; };

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template <typename R>
struct ResLayout {
    size_t x, c, rho, dd, dg, es, ell, total;
};

template <typename R>
__host__ __device__ __forceinline__ ResLayout<R> res_layout(int n, int M, int P, int nt_ept)
{
    ResLayout<R> L;
    const size_t RP = (size_t)((M * n) | 1);
    size_t o = 0;
    L.x = o;    o = align16(o + sizeof(cplx<R>) * ((size_t)n * RP + 1));
    L.c = o;    o = align16(o + sizeof(cplx<R>) * ((size_t)n * RP + 1));
    L.rho = o;  o = align16(o + sizeof(cplx<R>) * (size_t)nt_ept);
    L.dd = o;   o = align16(o + sizeof(R) * (size_t)M * n);
    L.dg = o;   o = align16(o + sizeof(R) * 2 * ((size_t)M * n + 1));
    L.es = o;   o = align16(o + sizeof(double) * 4 * (size_t)M);
    L.ell = o;  o = align16(o + sizeof(Ent<R>) * (size_t)n * (2 * P + 1));
    L.total = o;
    return L;
}

template <typename R>
__host__ __device__ __forceinline__ size_t res_smem_bytes(int n, int M, int P, int nt_ept)
{
    return res_layout<R>(n, M, P, nt_ept).total;
}

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
        double t0 = nj * (double)s.tdiag[j];
        for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
            const int k = s.hk[q];
            if (k == j) continue;
            t0 += (double)X[j * RP + row0 + k].re * (double)s.hv[q];
        }
        e[0] += t0;
        if (s.has_ext) e[3] += nj * (double)s.ediag[j];
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

// pass (3) for one compile-time RK stage.  Elements without work point at the
// spare slots, so every thread runs the same straight-line code.
template <typename R, int NT, int EPT, int STAGE>
__device__ __forceinline__ void res_element_pass(const cplx<R>* __restrict__ C, cplx<R>* __restrict__ X,
                                                 cplx<R>* __restrict__ rhoS, R* __restrict__ dgn,
                                                 const int (&oij)[EPT], const int (&oji)[EPT], const int (&odg)[EPT],
                                                 cplx<R> (&Ar)[EPT], cplx<R> (&Br)[EPT], R h, int tid)
{
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        const cplx<R> cij = C[oij[q]];
        const cplx<R> cji = C[oji[q]];
        cplx<R> k;
        k.re = subR<R>(cij.im, -cji.im);
        k.im = -subR<R>(cij.re, cji.re);
        cplx<R> rho = rhoS[f];
        cplx<R> xn;
        rk_update<R>(STAGE, k, h, rho, Ar[q], Br[q], xn);
        if (STAGE == 3) rhoS[f] = rho;
        X[oij[q]] = xn;
        X[oji[q]] = cplx<R>{xn.re, -xn.im};   // the diagonal writes itself twice
        dgn[odg[q]] = xn.re;
    }
}

template <typename R, int NT, int EPT, bool SPLIT, int P>
__global__ void __launch_bounds__(NT, 1) k_resident(ResArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    const int M = SPLIT ? a.G : 2 * a.G;
    const int RR = M * n;
    const int RP = RR | 1;
    const int E = M * ne;
    const int DGS = RR + 1;                  // dg parity stride (spare at RR)
    const int SPARE = n * RP;                // spare X / C slot
    constexpr int NE = 2 * P + 1;            // entries per column
    const ResLayout<R> L = res_layout<R>(n, M, P, NT * EPT);
    cplx<R>* X = reinterpret_cast<cplx<R>*>(smem + L.x);
    cplx<R>* C = reinterpret_cast<cplx<R>*>(smem + L.c);
    cplx<R>* rhoS = reinterpret_cast<cplx<R>*>(smem + L.rho);
    R* Dd = reinterpret_cast<R*>(smem + L.dd);
    R* dg = reinterpret_cast<R*>(smem + L.dg);
    double* es = reinterpret_cast<double*>(smem + L.es);
    Ent<R>* ell = reinterpret_cast<Ent<R>*>(smem + L.ell);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    const int W = rec_width(n);

    for (int q = tid; q < n * NE; q += NT) {
        Ent<R> e;
        e.off = a.ell_k[q] * RP;
        e.v = a.ell_v[q];
        if constexpr (sizeof(Ent<R>) == 16) reinterpret_cast<int*>(&e)[1] = 0;
        ell[q] = e;
    }

    int rank = 0, cid = blockIdx.x, ncl = gridDim.x;
    R* peer_dg = nullptr;
    if constexpr (SPLIT) {
        cg::cluster_group cl = cg::this_cluster();
        rank = (int)cl.block_rank();
        cid = blockIdx.x >> 1;
        ncl = gridDim.x >> 1;
        peer_dg = cl.map_shared_rank(dg, rank ^ 1);
    }
    auto bar = [&]() {
        if constexpr (SPLIT) cg::this_cluster().sync(); else __syncthreads();
    };
    // diagonal array of the other spin of matrix m at parity p
    auto other_dg = [&](int p, int m) -> const R* {
        if constexpr (SPLIT) return peer_dg + p * DGS + m * n;
        else return dg + p * DGS + (m ^ 1) * n;
    };

    // per element: shared-memory offsets of X_ij, X_ji and of its dg slot
    cplx<R> Ar[EPT], Br[EPT];
    int oij[EPT], oji[EPT], odg[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        oij[q] = SPARE; oji[q] = SPARE; odg[q] = RR;
        if (f < E) {
            const int m = f / ne;
            const uint32_t p = a.sys.pij[f - m * ne];
            const int i = p & 0xffffu, j = p >> 16;
            oij[q] = j * RP + m * n + i;
            oji[q] = i * RP + m * n + j;
            if (i == j) odg[q] = m * n + i;
        }
    }
    double* myslot = a.slots ? a.slots + (size_t)blockIdx.x * a.Tp * W : nullptr;

    // pass (2) work split: warp -> (row block, column), advanced without divisions
    const int nrb = (RR + 31) >> 5;
    const int dq = NW / nrb, dr = NW % nrb;
    const int rb0 = warp % nrb, j0 = warp / nrb;
    const bool fixed_rb = (dr == 0);
    int rd_fixed = 0;
    {
        const int r = rb0 * 32 + lane;
        rd_fixed = (min(r, RR - 1) / n) * n;
    }

    const int ngroups = (a.B + a.G - 1) / a.G;
    __syncthreads();
    for (int gid = cid; gid < ngroups; gid += ncl) {
        // ---- load the packed state into the stacked full layout
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            cplx<R> v = {R(0), R(0)};
            if (f < E) {
                const int m = f / ne;
                const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
                const int b = gid * a.G + g;
                if (b < a.B) v = a.state[((size_t)b * 2 + s) * ne + (f - m * ne)];
                X[oij[q]] = v;
                X[oji[q]] = cplx<R>{v.re, -v.im};
                X[oij[q]] = v;
                dg[odg[q]] = v.re;
            }
            rhoS[f] = v;
            Ar[q] = v; Br[q] = v;
        }
        int par = 0;
        long gstep = a.step_base;
        bar();
        for (int t = a.t_begin; t < a.t_end; ++t) {
            if (a.record) {
                const R* d0 = dg + par * DGS;
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
                            const double mine = (double)d0[g * n + j], oth = (double)other_dg(par, g)[j];
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
                    for (int m = warp; m < M; m += NW) {
                        const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
                        double e[4] = {0.0, 0.0, 0.0, 0.0};
                        energy_partials_full<R>(a.sys, X, RP, m * n, d0 + m * n, other_dg(par, m), s, a.do_e1,
                                                a.do_e2, lane, 32, e);
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const double v = warp_sum(e[c]);
                            if (lane == 0) es[m * 4 + c] = (gid * a.G + g < a.B) ? v : 0.0;
                        }
                    }
                    __syncthreads();
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
                        const int p = f - m * ne;
                        atomicAdd(&a.whole[((size_t)t * 2 + s) * ne + p].x, (double)rhoS[f].re);
                        atomicAdd(&a.whole[((size_t)t * 2 + s) * ne + p].y, (double)rhoS[f].im);
                    }
                }
            }
            const int nsteps = (a.hf && t == a.Tp - 1) ? 0 : a.S;
            for (int st = 0; st < nsteps; ++st, ++gstep) {
#pragma unroll
                for (int stage = 0; stage < 4; ++stage) {
                    const R pv = a.sys.n_bins > 0 ? a.ptab[(gstep - a.step_base) * 4 + stage] : R(0);
                    // (1) Delta diagonal
                    for (int w = tid; w < RR; w += NT) {
                        const int m = w / n, j = w - m * n;
                        Dd[w] = delta_diag_v<R>(a.sys, j, dg + par * DGS + m * n, other_dg(par, m), pv);
                    }
                    __syncthreads();
                    // (2) C = X Delta
                    {
                        int rb = rb0, j = j0;
                        while (j < n) {
                            const int r = rb * 32 + lane;
                            const int rr = min(r, RR - 1);
                            const int rd = fixed_rb ? rd_fixed : (rr / n) * n;
                            const Ent<R>* e = ell + j * NE;
                            R are = R(0), aim = R(0);
#pragma unroll
                            for (int q = 0; q < P; ++q) {
                                const Ent<R> en = e[q];
                                const cplx<R> x = X[en.off + rr];
                                are = fmaR<R>(x.re, en.v, are);
                                aim = fmaR<R>(x.im, en.v, aim);
                            }
                            {
                                const R ddj = Dd[rd + j];
                                const cplx<R> x = X[j * RP + rr];
                                are = fmaR<R>(x.re, ddj, are);
                                aim = fmaR<R>(x.im, ddj, aim);
                            }
#pragma unroll
                            for (int q = P + 1; q < NE; ++q) {
                                const Ent<R> en = e[q];
                                const cplx<R> x = X[en.off + rr];
                                are = fmaR<R>(x.re, en.v, are);
                                aim = fmaR<R>(x.im, en.v, aim);
                            }
                            C[r < RR ? j * RP + r : SPARE] = cplx<R>{are, aim};
                            rb += dr; j += dq;
                            if (rb >= nrb) { rb -= nrb; j += 1; }
                        }
                    }
                    __syncthreads();
                    // (3) commutator element, RK update, write back X and its mirror
                    R* dgn = dg + (par ^ 1) * DGS;
                    if (stage == 0) res_element_pass<R, NT, EPT, 0>(C, X, rhoS, dgn, oij, oji, odg, Ar, Br, a.h, tid);
                    else if (stage == 1) res_element_pass<R, NT, EPT, 1>(C, X, rhoS, dgn, oij, oji, odg, Ar, Br, a.h, tid);
                    else if (stage == 2) res_element_pass<R, NT, EPT, 2>(C, X, rhoS, dgn, oij, oji, odg, Ar, Br, a.h, tid);
                    else res_element_pass<R, NT, EPT, 3>(C, X, rhoS, dgn, oij, oji, odg, Ar, Br, a.h, tid);
                    bar();
                    par ^= 1;
                }
            }
        }
        // store
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            if (f >= E) continue;
            const int m = f / ne;
            const int g = SPLIT ? m : (m >> 1), s = SPLIT ? rank : (m & 1);
            const int b = gid * a.G + g;
            if (b < a.B) a.state[((size_t)b * 2 + s) * ne + (f - m * ne)] = rhoS[f];
        }
        bar();
    }
}

// Kahan sum over CTA slots: out[t][w] = sum_c slots[c][t][w] (c ascending)
__global__ void k_slot_reduce(const double* __restrict__ slots, int nslots, long TW, double* __restrict__ out)
{
    for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < TW; w += (long)gridDim.x * blockDim.x) {
        double s = 0.0, comp = 0.0;
        for (int c = 0; c < nslots; ++c) {
            const double y = slots[(size_t)c * TW + w] - comp;
            const double t = s + y;
            comp = (t - s) - y;
            s = t;
        }
        out[w] = s;
    }
}

// ------------------------------------------------------------------ sampler
// Product-state samples, packed FP64 (rotation handled separately).
// Spin up uses the upper triangle of W (symmatu), spin down the lower (symmatl).
__global__ void k_sample(int n, int ne, int B, uint64_t seed, const double* __restrict__ occ_u,
                         const double* __restrict__ occ_d, cplx<double>* __restrict__ out)
{
    const long total = (long)B * ne;
    const double rs2 = sqrt(2.0);
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total; x += (long)gridDim.x * blockDim.x) {
        const int b = (int)(x / ne), p = (int)(x - (long)b * ne);
        int j = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
        while (cs(j) > p) --j;
        while (cs(j + 1) <= p) ++j;
        const int i = p - cs(j);
        cplx<double> vu, vd;
        if (i == j) {
            vu.re = occ_u[i] - 0.5; vu.im = 0.0;
            vd.re = occ_d[i] - 0.5; vd.im = 0.0;
        } else {
            double g1, g2;
            // spin up: element (i, j), i < j, linear index j*n + i
            gauss_pair(seed, (uint64_t)b, (uint32_t)(j * n + i), g1, g2);
            double su = sqrt(__ddiv_rn(__dsub_rn(__dadd_rn(occ_u[i], occ_u[j]), __dmul_rn(__dmul_rn(2.0, occ_u[i]), occ_u[j])), 2.0));
            vu.re = __dmul_rn(__ddiv_rn(g1, rs2), su);
            vu.im = __dmul_rn(__ddiv_rn(g2, rs2), su);
            // spin down: lower element (j, i), linear index i*n + j; upper = its conjugate
            gauss_pair(seed, (uint64_t)b, (uint32_t)(i * n + j), g1, g2);
            double sd = sqrt(__ddiv_rn(__dsub_rn(__dadd_rn(occ_d[j], occ_d[i]), __dmul_rn(__dmul_rn(2.0, occ_d[j]), occ_d[i])), 2.0));
            vd.re = __dmul_rn(__ddiv_rn(g1, rs2), sd);
            vd.im = -__dmul_rn(__ddiv_rn(g2, rs2), sd);
        }
        out[((size_t)b * 2) * ne + p] = vu;
        out[((size_t)b * 2 + 1) * ne + p] = vd;
    }
}

// rho <- R rho R^H per trajectory and spin (rotated ground-state initial
// conditions, src/FHfTWASolver.cpp:359,362).  Dense FP64; one CTA per matrix.
__global__ void k_rotate(int n, int ne, int B, const cplx<double>* __restrict__ Ru, const cplx<double>* __restrict__ Rd,
                         cplx<double>* __restrict__ state, cplx<double>* __restrict__ scratch)
{
    // scratch: [gridDim.x][2][n*n] (M full, then T = R M)
    for (int m = blockIdx.x; m < 2 * B; m += gridDim.x) {
        const int s = m & 1;
        const cplx<double>* R = s ? Rd : Ru;
        if (!R) continue;
        cplx<double>* M = scratch + (size_t)blockIdx.x * 2 * n * n;
        cplx<double>* T = M + (size_t)n * n;
        cplx<double>* P = state + (size_t)m * ne;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q % n, j = q / n;
            M[q] = getH<double>(P, i, j);
        }
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {   // T = R M
            const int i = q % n, j = q / n;
            double re = 0.0, im = 0.0;
            for (int k = 0; k < n; ++k) {
                const cplx<double> r = R[(size_t)k * n + i], x = M[(size_t)j * n + k];
                re = __fma_rn(r.re, x.re, re); re = __fma_rn(-r.im, x.im, re);
                im = __fma_rn(r.re, x.im, im); im = __fma_rn(r.im, x.re, im);
            }
            T[q].re = re; T[q].im = im;
        }
        __syncthreads();
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {  // (T R^H)_ij, i <= j
            int j = 0;
            while (cs(j + 1) <= p) ++j;
            const int i = p - cs(j);
            double re = 0.0, im = 0.0;
            for (int k = 0; k < n; ++k) {
                const cplx<double> t = T[(size_t)k * n + i], r = R[(size_t)k * n + j];  // conj(R_jk)
                re = __fma_rn(t.re, r.re, re); re = __fma_rn(t.im, r.im, re);
                im = __fma_rn(-t.re, r.im, im); im = __fma_rn(t.im, r.re, im);
            }
            if (i == j) im = 0.0;
            P[p].re = re; P[p].im = im;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ conversions
__global__ void k_f64_to_f32(const cplx<double>* __restrict__ in, cplx<float>* __restrict__ out, long count)
{
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < count; x += (long)gridDim.x * blockDim.x) {
        out[x].re = (float)in[x].re;
        out[x].im = (float)in[x].im;
    }
}
__global__ void k_f32_to_f64(const cplx<float>* __restrict__ in, cplx<double>* __restrict__ out, long count)
{
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < count; x += (long)gridDim.x * blockDim.x) {
        out[x].re = (double)in[x].re;
        out[x].im = (double)in[x].im;
    }
}

}  // namespace fpsg
