// fpsg_adjoint.cuh — kernels of the discrete adjoint of the 3/8-rule RK4 step.
//
// The forward map per spin is k = f(X) = -i (X Delta - Delta X), Delta = T +
// diag(d), d_j = tM_jj + sum_k U_jk (n_other,k + s) [+ sum_k V_jk (n_same,k + s)]
// + ext_jj + a_bin(t) env(t) proj_j.  With the real inner product
// <A, B> = Re tr(A^H B) over full matrices, the vector-Jacobian product of f at X
// for an output adjoint Kb is
//     Xb = i (Kb Delta - Delta Kb)                         (Delta held fixed)
//     db_j = 2 Im (Kb^H X)_jj                              (adjoint of d_j)
//     Xb_other,kk += sum_j U_jk db_j,  Xb_same,kk += sum_j V_jk db_j
//     U scale:  sum_j db_j sum_k U_jk (n_other,k + s)
//     t scale:  <Kb, -i [X, T]>
//     pulse:    a_bin(t) receives env(t) sum_j proj_j db_j
// Every map keeps Hermiticity, so the adjoint state is stored packed like the
// state (upper triangle, column by column).  Offdiagonal packed entries stand for
// two entries of the full matrix in inner products (weight 2).
#pragma once
#include "fpsg_kernels.cuh"

namespace fpsg {

template <typename R>
struct VjpArgs {
    DevSys<R> sys;
    int B;
    const cplx<R>* X;          // stage input, [B][2][ne]
    const cplx<R>* lam;        // adjoint of the step output
    const cplx<R>* xb4;        // adjoints of later stage inputs (may be null)
    const cplx<R>* xb3;
    const cplx<R>* xb2;
    R c_lam, c4, c3, c2;       // Kb = c_lam lam + c4 xb4 + c3 xb3 + c2 xb2
    R pulse;                   // pulse value at the stage time (a_bin env)
    double env;                // env(t) at the stage time
    int bin;                   // pulse bin of the stage time (or -1)
    cplx<R>* xb_out;           // adjoint of this stage input (linear part)
    R* dbar;                   // [B][2][n]
    double* pacc;              // [B][2][2 + n_bins]: U scale, t scale, pulse bins
    int n_bins;
};

template <typename R>
__global__ void __launch_bounds__(256) k_vjp_stage(VjpArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    cplx<R>* Kb = reinterpret_cast<cplx<R>*>(smem);
    cplx<R>* Xs = Kb + ne;
    R* Dd = reinterpret_cast<R*>(Xs + ne);
    R* Tdg = Dd + n;
    double* red = reinterpret_cast<double*>(smem + ((2 * sizeof(cplx<R>) * ne + 2 * sizeof(R) * n + 15) & ~size_t(15)));
    const int M = a.B * 2;
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const size_t base = (size_t)m * ne;
        const cplx<R>* xo = a.X + (size_t)(m ^ 1) * ne;
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {
            cplx<R> k = {R(0), R(0)};
            const cplx<R> lv = a.lam[base + p];
            k.re = a.c_lam * lv.re; k.im = a.c_lam * lv.im;
            if (a.xb4) { const cplx<R> v = a.xb4[base + p]; k.re += a.c4 * v.re; k.im += a.c4 * v.im; }
            if (a.xb3) { const cplx<R> v = a.xb3[base + p]; k.re += a.c3 * v.re; k.im += a.c3 * v.im; }
            if (a.xb2) { const cplx<R> v = a.xb2[base + p]; k.re += a.c2 * v.re; k.im += a.c2 * v.im; }
            Kb[p] = k;
            Xs[p] = a.X[base + p];
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            Dd[j] = delta_diag<R>(a.sys, j, Xs, xo, a.pulse);
            Tdg[j] = a.sys.tdiag[j];
        }
        __syncthreads();
        // Linear part Xb = i [Kb, Delta].  The t-scale term <Kb, -i [X, tM]> equals
        // <X, i [Kb, tM]> = <X, Xb> - sum_j (Delta_jj - tM_jj) db_j (Delta = tM +
        // diag(Delta_jj - tM_jj)), so no second commutator is needed.
        double tsc = 0.0;
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            const cplx<R> c = commutator_elem<R>(a.sys, Kb, Dd, i, j);
            const cplx<R> xb = {-c.re, -c.im};
            a.xb_out[base + p] = xb;
            const double wgt = (i == j) ? 1.0 : 2.0;
            tsc += wgt * ((double)Xs[p].re * (double)xb.re + (double)Xs[p].im * (double)xb.im);
        }
        // db_j = 2 Im sum_r conj(Kb_rj) X_rj: one warp per column, lanes over rows
        double usc = 0.0, psc = 0.0;
        const double shift = (double)a.sys.shift;
        for (int j = w; j < n; j += nw) {
            double im = 0.0;
            for (int r = l; r < n; r += 32) {
                const cplx<R> kb = getH<R>(Kb, r, j), x = getH<R>(Xs, r, j);
                im += (double)kb.re * (double)x.im - (double)kb.im * (double)x.re;
            }
            im = warp_sum(im);
            if (l == 0) {
                const double db = 2.0 * im;
                a.dbar[(size_t)m * n + j] = (R)db;
                tsc -= ((double)Dd[j] - (double)Tdg[j]) * db;
                if (a.sys.coul != 0) {
                    double uo = 0.0;
                    for (int q = a.sys.up[j]; q < a.sys.up[j + 1]; ++q)
                        uo += (double)a.sys.uv[q] * ((double)xo[cs(a.sys.uk[q]) + a.sys.uk[q]].re + shift);
                    if (a.sys.coul == 2)
                        for (int q = a.sys.vp[j]; q < a.sys.vp[j + 1]; ++q)
                            uo += (double)a.sys.vv[q] * ((double)Xs[cs(a.sys.vk[q]) + a.sys.vk[q]].re + shift);
                    usc += db * uo;
                }
                if (a.bin >= 0) psc += db * a.env * (double)a.sys.proj[j];
            }
        }
        double vals[3] = {usc, tsc, psc};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = warp_sum(vals[c]);
            if (l == 0) red[w * 3 + c] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.0;
            for (int q = 0; q < nw; ++q) v += red[q * 3 + threadIdx.x];
            const int slot = threadIdx.x < 2 ? threadIdx.x : 2 + a.bin;
            if (threadIdx.x < 2 || a.bin >= 0) a.pacc[(size_t)m * (2 + a.n_bins) + slot] += v;
        }
        __syncthreads();
    }
}

// k_vjp_stage in the direct form of the resident kernel, for lattices whose
// Delta columns fit a fixed width (P entries on each side of the diagonal): Kb is
// staged as a full matrix (column pitch RPc = n | 1, both triangles), so every
// term of the commutator is a branch-free shared load, and the column entries
// come from slot-major tables.  The nonzero terms are summed in ascending k
// exactly as the CSR form sums them (padding adds exact zeros), so the result is
// the same to the bit.
template <typename R>
size_t vjp_ell_smem(int n, int ne, int P)
{
    const int RPc = n | 1, NE = 2 * P + 1;
    size_t o = sizeof(cplx<R>) * (size_t)n * RPc;
    o += sizeof(R) * (size_t)ne + sizeof(R) * (size_t)n;
    o = (o + 15) & ~size_t(15);
    o += sizeof(int) * (size_t)NE * n;
    o = (o + 15) & ~size_t(15);
    o += sizeof(R) * (size_t)NE * n;
    o = (o + 15) & ~size_t(15);
    return o + sizeof(double) * 32 * 3;
}

template <typename R, int P>
__global__ void __launch_bounds__(256) k_vjp_stage_ell(VjpArgs<R> a, const int* __restrict__ ell_k,
                                                       const R* __restrict__ ell_v)
{
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NE = 2 * P + 1;
    const int n = a.sys.n, ne = a.sys.ne, RPc = n | 1;
    cplx<R>* K = reinterpret_cast<cplx<R>*>(smem);                 // K(r, c) at c * RPc + r
    R* EP = reinterpret_cast<R*>(K + (size_t)n * RPc);               // Im(conj(Kb_p) X_p), packed
    R* Dd = EP + ne;
    size_t o = ((sizeof(cplx<R>) * (size_t)n * RPc + sizeof(R) * (size_t)(ne + n)) + 15) & ~size_t(15);
    int* EK = reinterpret_cast<int*>(smem + o);                      // [NE][n] row index of slot s of column c
    o = (o + sizeof(int) * (size_t)NE * n + 15) & ~size_t(15);
    R* EV = reinterpret_cast<R*>(smem + o);                          // [NE][n] Delta entry (0 for padding)
    o = (o + sizeof(R) * (size_t)NE * n + 15) & ~size_t(15);
    double* red = reinterpret_cast<double*>(smem + o);
    const int M = a.B * 2;
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int q = threadIdx.x; q < n * NE; q += blockDim.x) {
        const int col = q / NE, sl = q - col * NE;
        const int k = ell_k[q];
        EK[sl * n + col] = k >= 0 ? k : col;
        EV[sl * n + col] = k >= 0 ? ell_v[q] : R(0);
    }
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const size_t base = (size_t)m * ne;
        const cplx<R>* X = a.X + base;
        const cplx<R>* xo = a.X + (size_t)(m ^ 1) * ne;
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {
            cplx<R> k = {R(0), R(0)};
            const cplx<R> lv = a.lam[base + p];
            k.re = a.c_lam * lv.re; k.im = a.c_lam * lv.im;
            if (a.xb4) { const cplx<R> v = a.xb4[base + p]; k.re += a.c4 * v.re; k.im += a.c4 * v.im; }
            if (a.xb3) { const cplx<R> v = a.xb3[base + p]; k.re += a.c3 * v.re; k.im += a.c3 * v.im; }
            if (a.xb2) { const cplx<R> v = a.xb2[base + p]; k.re += a.c2 * v.re; k.im += a.c2 * v.im; }
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            K[(size_t)j * RPc + i] = k;
            if (i != j) K[(size_t)i * RPc + j] = cplx<R>{k.re, -k.im};
        }
        for (int j = threadIdx.x; j < n; j += blockDim.x) Dd[j] = delta_diag<R>(a.sys, j, X, xo, a.pulse);
        __syncthreads();
        double tsc = 0.0;
        for (int p = threadIdx.x; p < ne; p += blockDim.x) {
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            R are = R(0), aim = R(0), bre = R(0), bim = R(0);
#pragma unroll
            for (int sl = 0; sl < NE; ++sl) {         // sum_k Kb_ik Delta_kj over column j
                const int k = EK[sl * n + j];
                const R d = sl == P ? Dd[j] : EV[sl * n + j];
                const cplx<R> x = K[(size_t)k * RPc + i];
                are = fmaR<R>(x.re, d, are);
                aim = fmaR<R>(x.im, d, aim);
            }
#pragma unroll
            for (int sl = 0; sl < NE; ++sl) {         // sum_k Kb_kj Delta_ki over column i
                const int k = EK[sl * n + i];
                const R d = sl == P ? Dd[i] : EV[sl * n + i];
                const cplx<R> x = K[(size_t)j * RPc + k];
                bre = fmaR<R>(x.re, d, bre);
                bim = fmaR<R>(x.im, d, bim);
            }
            // i [Kb, Delta] = -(-i [Kb, Delta])
            const cplx<R> xb = {-subR<R>(aim, bim), subR<R>(are, bre)};
            a.xb_out[base + p] = xb;
            const cplx<R> x = X[p], kb = K[(size_t)j * RPc + i];
            const double wgt = (i == j) ? 1.0 : 2.0;
            tsc += wgt * ((double)x.re * (double)xb.re + (double)x.im * (double)xb.im);
            EP[p] = (R)((double)kb.re * (double)x.im - (double)kb.im * (double)x.re);
        }
        __syncthreads();
        // db_j = 2 Im sum_r conj(Kb_rj) X_rj: upper elements of column j as they are,
        // the mirrored lower part (upper row j) with the opposite sign
        double usc = 0.0, psc = 0.0;
        const double shift = (double)a.sys.shift;
        for (int j = w; j < n; j += nw) {
            double im = 0.0;
            for (int r = l; r < n; r += 32) im += r <= j ? (double)EP[cs(j) + r] : -(double)EP[cs(r) + j];
            im = warp_sum(im);
            if (l == 0) {
                const double db = 2.0 * im;
                a.dbar[(size_t)m * n + j] = (R)db;
                tsc -= ((double)Dd[j] - (double)a.sys.tdiag[j]) * db;
                if (a.sys.coul != 0) {
                    double uo = 0.0;
                    for (int q = a.sys.up[j]; q < a.sys.up[j + 1]; ++q)
                        uo += (double)a.sys.uv[q] * ((double)xo[cs(a.sys.uk[q]) + a.sys.uk[q]].re + shift);
                    if (a.sys.coul == 2)
                        for (int q = a.sys.vp[j]; q < a.sys.vp[j + 1]; ++q)
                            uo += (double)a.sys.vv[q] * ((double)X[cs(a.sys.vk[q]) + a.sys.vk[q]].re + shift);
                    usc += db * uo;
                }
                if (a.bin >= 0) psc += db * a.env * (double)a.sys.proj[j];
            }
        }
        double vals[3] = {usc, tsc, psc};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = warp_sum(vals[c]);
            if (l == 0) red[w * 3 + c] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.0;
            for (int q = 0; q < nw; ++q) v += red[q * 3 + threadIdx.x];
            const int slot = threadIdx.x < 2 ? threadIdx.x : 2 + a.bin;
            if (threadIdx.x < 2 || a.bin >= 0) a.pacc[(size_t)m * (2 + a.n_bins) + slot] += v;
        }
        __syncthreads();
    }
}

// Hartree coupling of the stage adjoint: Xb_other,kk += sum_j U_jk db_j and
// (distance Coulomb) Xb_same,kk += sum_j V_jk db_j.  U and V are symmetric, so
// their row lists serve as column lists.
template <typename R>
__global__ void k_vjp_cross(DevSys<R> sys, int B, const R* __restrict__ dbar, cplx<R>* __restrict__ xb)
{
    const int n = sys.n, ne = sys.ne;
    const long total = (long)B * 2 * n;
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total; x += (long)gridDim.x * blockDim.x) {
        const int m = (int)(x / n), k = (int)(x - (long)m * n);
        const R* dother = dbar + (size_t)(m ^ 1) * n;
        const R* dsame = dbar + (size_t)m * n;
        R add = R(0);
        if (sys.coul != 0) {
            for (int q = sys.up[k]; q < sys.up[k + 1]; ++q) add += sys.uv[q] * dother[sys.uk[q]];
            if (sys.coul == 2)
                for (int q = sys.vp[k]; q < sys.vp[k + 1]; ++q) add += sys.vv[q] * dsame[sys.vk[q]];
        }
        xb[(size_t)m * ne + cs(k) + k].re += add;
    }
}

// lam += xb1 + xb2 + xb3 + xb4
template <typename R>
__global__ void k_lam_update(long count, cplx<R>* __restrict__ lam, const cplx<R>* __restrict__ a,
                             const cplx<R>* __restrict__ b, const cplx<R>* __restrict__ c, const cplx<R>* __restrict__ d)
{
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < count; x += (long)gridDim.x * blockDim.x) {
        cplx<R> v = lam[x];
        v.re += ((a[x].re + b[x].re) + c[x].re) + d[x].re;
        v.im += ((a[x].im + b[x].im) + c[x].im) + d[x].im;
        lam[x] = v;
    }
}

// snapshot loss: lam_s,ii += w (n_other,ii + s) for the doublon term
// w * sum_i (rho_up,ii rho_dn,ii + (rho_up,ii + rho_dn,ii)/2)
template <typename R>
__global__ void k_loss_grad(int n, int ne, int B, const cplx<R>* __restrict__ y, cplx<R>* __restrict__ lam, double w)
{
    const long total = (long)B * 2 * n;
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < total; x += (long)gridDim.x * blockDim.x) {
        const int m = (int)(x / n), i = (int)(x - (long)m * n);
        const double other = (double)y[(size_t)(m ^ 1) * ne + cs(i) + i].re;
        lam[(size_t)m * ne + cs(i) + i].re += (R)(w * (other + 0.5));
    }
}

// parameter totals: out[c] = sum over trajectories and spins of pacc[.][c] (fixed order)
__global__ void k_pacc_reduce(const double* __restrict__ pacc, int M, int W, double* __restrict__ out)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < W; c += gridDim.x * blockDim.x) {
        double s = 0.0, comp = 0.0;
        for (int m = 0; m < M; ++m) {
            const double y = pacc[(size_t)m * W + c] - comp;
            const double t = s + y;
            comp = (t - s) - y;
            s = t;
        }
        out[c] = s;
    }
}

}  // namespace fpsg
