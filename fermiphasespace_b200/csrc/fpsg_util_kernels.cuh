// fpsg_util_kernels.cuh — the non-template kernels: ensemble reductions, the
// initial-state sampler and rotation, precision conversions.  Included by one
// translation unit only (fpsg_abi.cu).
#pragma once
#include "fpsg_kernels.cuh"

namespace fpsg {

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

// k_reduce_fin with the snapshot index read from device memory, so that a
// captured graph replays unchanged from snapshot to snapshot
__global__ void k_reduce_fin_at(const double* __restrict__ part, int nchunks, int W, double* __restrict__ sums,
                                const int* __restrict__ t_ctr)
{
    double* out = sums + (size_t)(*t_ctr) * W;
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

__global__ void k_tick(int* t_ctr)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *t_ctr += 1;
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
__global__ void k_sample(int n, int ne, int B, long b0, uint64_t seed, const double* __restrict__ occ_u,
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
            gauss_pair(seed, (uint64_t)(b0 + b), (uint32_t)(j * n + i), g1, g2);
            double su = sqrt(__ddiv_rn(__dsub_rn(__dadd_rn(occ_u[i], occ_u[j]), __dmul_rn(__dmul_rn(2.0, occ_u[i]), occ_u[j])), 2.0));
            vu.re = __dmul_rn(__ddiv_rn(g1, rs2), su);
            vu.im = __dmul_rn(__ddiv_rn(g2, rs2), su);
            // spin down: lower element (j, i), linear index i*n + j; upper = its conjugate
            gauss_pair(seed, (uint64_t)(b0 + b), (uint32_t)(i * n + j), g1, g2);
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
