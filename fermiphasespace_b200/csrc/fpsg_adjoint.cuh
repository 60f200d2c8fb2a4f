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

namespace fpsg {

// ------------------------------------------------------------------------------
// Reverse sweep of one checkpoint segment with the trajectories resident.
//
// A 2-CTA cluster takes one trajectory at a time (CTA rank = spin) and runs all
// steps of the segment backwards: per stage g = 4 .. 1 it builds the output
// adjoint Kb = c_lam lam + sum c_g' xb_g' (registers) into a full shared matrix,
// forms xb_g = i [Kb, Delta] and the element products Im(conj(Kb) X) in the direct
// form of the resident forward kernel, sums them per column to db_j, hands db to
// the partner spin over DSMEM for the Hartree cross term, and accumulates the
// parameter partials; after the four stages lam += xb1 + xb2 + xb3 + xb4 and, at a
// snapshot, the loss term.  Only the stage inputs are read from global memory
// (prefetched a stage ahead); lam stays in registers for the whole segment.  It
// takes the place of k_vjp_stage_ell + k_vjp_cross per stage and k_lam_update +
// k_loss_grad per step, with the same formulas and the same order of additions
// inside each term (the per-matrix partial sums of the t scale follow the thread
// layout, so the parameter gradients agree to rounding, not to the bit).
// Requirements: on-site or no Coulomb term (Delta_jj from U_jj alone), fixed-width
// columns (P), and n (n + 1) / 2 <= NT * EPT.
template <typename R>
struct VjpSegArgs {
    DevSys<R> sys;
    int B;
    const cplx<R>* seg;        // [step][4][B][2][ne] stage inputs of the segment
    size_t count;              // B * 2 * ne
    int nsteps;                // steps in the segment
    long s0;                   // global index of its first step
    cplx<R>* lam;              // [B][2][ne]: adjoint after the segment in, before it out
    const R* ptab;             // [step][4] pulse value a_bin env (global step), null: no pulse
    const double* envtab;      // [step][4] env(t) at the stage time
    const int* bintab;         // [step][4] pulse bin of the stage time
    double* pacc;              // [B][2][2 + n_bins]: U scale, t scale, pulse bins
    int n_bins;
    R h;
    int S, Tp;                 // steps per snapshot, snapshots (loss weights)
    double dt, lscale;
    const int* ell_k;          // [n][2P+1] row index of each column entry, -1 = padding
    const R* ell_v;
    const uint32_t* order;     // element (i | j << 16) of each slot
    const R* udiag;            // U_jj
    unsigned* err;
};

template <typename R>
struct __align__(8) VEnt { int k; R v; };
template <>
struct __align__(16) VEnt<double> { int k; int pad; double v; };

template <typename R, int P, bool XS = false>
__host__ __device__ __forceinline__ size_t vjp_seg_smem(int n, int ne, int n_bins)
{
    const int RPc = n | 1, NE = 2 * P + 1;
    size_t o = sizeof(cplx<R>) * (size_t)n * RPc;          // K
    o = align16(o + sizeof(R) * (size_t)n * RPc);           // EP (full, signed)
    o = align16(o + sizeof(R) * (size_t)n * 3);             // Dd, xod, xo0
    o = align16(o + sizeof(R) * (size_t)n * 2);             // dbo[2]
    o = align16(o + sizeof(R) * (size_t)n * 4);             // site constants tdiag, udiag, ediag, proj
    o = align16(o + sizeof(VEnt<R>) * (size_t)NE * n);      // column entries
    o += sizeof(double) * 32 * 3;                           // per-warp partials
    o = align16(o + sizeof(cplx<R>) * (size_t)n);           // stage-1 adjoint of the diagonal
    o = align16(o + sizeof(double) * (size_t)(2 + n_bins)); // parameter partials of the trajectory
    o = align16(o + sizeof(double) * (size_t)(512 + 64 * 3)); // running partials per thread / column group
    if (XS) o += sizeof(cplx<R>) * 3 * (size_t)ne;          // stage adjoints 4, 3, 2 by slot
    return o;
}

// XS = true keeps the stage adjoints 4, 3, 2 in shared memory (one slot per element,
// thread-private) instead of registers, so that two clusters fit on an SM pair.
template <typename R, int NT, int EPT, int P, bool XS = false>
__global__ void __launch_bounds__(NT, XS ? 2 : 1) k_vjp_segment(VjpSegArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NE = 2 * P + 1, NW = NT / 32;
    const int n = a.sys.n, ne = a.sys.ne, RPc = n | 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    size_t o = sizeof(cplx<R>) * (size_t)n * RPc;
    cplx<R>* K = reinterpret_cast<cplx<R>*>(smem);                  // Kb(r, c) at c * RPc + r
    // Im(conj(Kb_rj) X_rj) for every (r, j) at j * RPc + r: the upper element's
    // product, and its negative at the mirrored position
    R* EP = reinterpret_cast<R*>(smem + o);
    o = align16(o + sizeof(R) * (size_t)n * RPc);
    R* Dd = reinterpret_cast<R*>(smem + o);                          // Delta_jj of the stage
    R* xod = Dd + n;                                                 // partner's stage-input diagonal
    R* xo0 = xod + n;                                                // the same for stage 1 (loss term)
    o = align16(o + sizeof(R) * (size_t)n * 3);
    R* dbo = reinterpret_cast<R*>(smem + o);                         // [2][n] partner's db, by stage parity
    o = align16(o + sizeof(R) * (size_t)n * 2);
    R* c_t = reinterpret_cast<R*>(smem + o);                         // tM_jj
    R* c_u = c_t + n;                                                // U_jj
    R* c_e = c_u + n;                                                // extPot_jj
    R* c_p = c_e + n;                                                // pulse projection
    o = align16(o + sizeof(R) * (size_t)n * 4);
    VEnt<R>* ell = reinterpret_cast<VEnt<R>*>(smem + o);             // [NE][n]
    o = align16(o + sizeof(VEnt<R>) * (size_t)NE * n);
    double* red = reinterpret_cast<double*>(smem + o);               // [NW][3]
    cplx<R>* x1d = reinterpret_cast<cplx<R>*>(red + 32 * 3);         // [n] stage-1 adjoint of the diagonal
    o = align16(o + sizeof(double) * 32 * 3 + sizeof(cplx<R>) * (size_t)n);
    double* pac = reinterpret_cast<double*>(smem + o);               // [2 + n_bins] this trajectory's partials
    o = align16(o + sizeof(double) * (size_t)(2 + a.n_bins));
    // running parameter partials over the segment, summed over the CTA once per
    // trajectory (and, for a pulse bin, when the bin changes): the t scale per
    // thread; the U scale, the open pulse bin and a finished bin per column group
    static_assert(NT <= 512 && NW * 4 <= 64, "running partials sized for 512 threads");
    double* acct = reinterpret_cast<double*>(smem + o);              // [NT]
    double* accu = acct + 512;                                       // [64]
    double* accp = accu + 64;                                        // [64]
    double* accf = accp + 64;                                        // [64]
    o = align16(o + sizeof(double) * (size_t)(512 + 64 * 3));
    cplx<R>* x4s = reinterpret_cast<cplx<R>*>(smem + o);             // [3][ne] (XS only)
    cplx<R>* x3s = x4s + ne;
    cplx<R>* x2s = x3s + ne;

    cg::cluster_group cl = cg::this_cluster();
    const int s = (int)cl.block_rank();
    const int cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;
    R* peer_dbo = cl.map_shared_rank(dbo, s ^ 1);

    for (int q = tid; q < n * NE; q += NT) {
        const int col = q / NE, sl = q - col * NE;
        const int k = a.ell_k[q];
        VEnt<R> e;
        e.k = (sl == P || k < 0) ? col : k;
        e.v = (sl == P || k < 0) ? R(0) : a.ell_v[q];
        if constexpr (sizeof(VEnt<R>) == 16) reinterpret_cast<int*>(&e)[1] = 0;
        ell[sl * n + col] = e;
    }
    for (int j = tid; j < n; j += NT) {
        c_t[j] = a.sys.tdiag[j];
        c_u[j] = a.udiag[j];
        c_e[j] = a.sys.has_ext ? a.sys.ediag[j] : R(0);
        c_p[j] = a.sys.n_bins > 0 ? a.sys.proj[j] : R(0);
    }
    // slot -> element (i | j << 16), ~0 for an empty slot
    uint32_t ij[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        ij[q] = f < ne ? a.order[f] : ~0u;
    }
    auto I_ = [&](int q) { return (int)(ij[q] & 0xffffu); };
    auto J_ = [&](int q) { return (int)(ij[q] >> 16); };
    auto P_ = [&](int q) { return cs(J_(q)) + I_(q); };
    const R hR = a.h;
    const double shift = (double)a.sys.shift;
    const int PW = 2 + a.n_bins;
    __syncthreads();

    for (int b = cid; b < a.B; b += ncl) {
        const int m = 2 * b + s;
        const size_t base = (size_t)m * ne, obase = (size_t)(m ^ 1) * ne;
        cplx<R> lam[EPT], x4r[XS ? 1 : EPT], x3r[XS ? 1 : EPT], x2r[XS ? 1 : EPT], xg[EPT];
        auto X4 = [&](int q) -> cplx<R>& { if constexpr (XS) return x4s[tid + q * NT]; else return x4r[q]; };
        auto X3 = [&](int q) -> cplx<R>& { if constexpr (XS) return x3s[tid + q * NT]; else return x3r[q]; };
        auto X2 = [&](int q) -> cplx<R>& { if constexpr (XS) return x2s[tid + q * NT]; else return x2r[q]; };
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            lam[q] = ij[q] != ~0u ? a.lam[base + P_(q)] : cplx<R>{R(0), R(0)};
            if (!XS || ij[q] != ~0u) X4(q) = X3(q) = X2(q) = cplx<R>{R(0), R(0)};
        }
        for (int c = tid; c < PW; c += NT) pac[c] = 0.0;
        acct[tid] = 0.0;
        if (tid < 64) { accu[tid] = 0.0; accp[tid] = 0.0; }
        int bin_acc = -1;                    // the pulse bin accp holds
        // the input of the first stage handled (last step, stage 4) and its pulse data
        R dgo = R(0);
        R pv_n = R(0);
        double env_n = 0.0;
        int bin_n = -1;
        {
            const long gl = (a.s0 + a.nsteps - 1) * 4 + 3;
            if (a.ptab) pv_n = a.ptab[gl];
            if (a.envtab) env_n = a.envtab[gl];
            if (a.bintab) bin_n = a.bintab[gl];
            const cplx<R>* X = a.seg + (size_t)(a.nsteps - 1) * 4 * a.count + 3 * a.count;
#pragma unroll
            for (int q = 0; q < EPT; ++q) xg[q] = ij[q] != ~0u ? X[base + P_(q)] : cplx<R>{R(0), R(0)};
            if (tid < n) dgo = X[obase + cs(tid) + tid].re;
        }
        int par = 0;
        for (int qs = a.nsteps - 1; qs >= 0; --qs) {
            const long gq = a.s0 + qs;
            // one RK stage backwards; G = 3 .. 0 is stage 4 .. 1
            auto stage = [&](auto Gc) {
                constexpr int G = decltype(Gc)::value;
                auto XG = [&](int q) -> cplx<R>& {                  // where this stage's adjoint goes (G > 0)
                    if constexpr (G == 3) return X4(q);
                    else if constexpr (G == 2) return X3(q);
                    else return X2(q);
                };
                const R pv = pv_n;
                const double env = env_n;
                const int bin = bin_n;
                // (a) Kb into shared memory; Delta_jj of the stage input
                const R c_l = (G == 0 || G == 3) ? hR / R(8) : R(3) * hR / R(8);
#pragma unroll
                for (int q = 0; q < EPT; ++q) {
                    if (ij[q] == ~0u) continue;
                    cplx<R> k;
                    k.re = mulR<R>(c_l, lam[q].re);
                    k.im = mulR<R>(c_l, lam[q].im);
                    if constexpr (G == 2) {
                        const cplx<R> v4 = X4(q);
                        k.re = fmaR<R>(hR, v4.re, k.re); k.im = fmaR<R>(hR, v4.im, k.im);
                    }
                    if constexpr (G == 1) {
                        const cplx<R> v4 = X4(q), v3 = X3(q);
                        k.re = fmaR<R>(-hR, v4.re, k.re); k.im = fmaR<R>(-hR, v4.im, k.im);
                        k.re = fmaR<R>(hR, v3.re, k.re); k.im = fmaR<R>(hR, v3.im, k.im);
                    }
                    if constexpr (G == 0) {
                        const cplx<R> v4 = X4(q), v3 = X3(q), v2 = X2(q);
                        k.re = fmaR<R>(hR, v4.re, k.re); k.im = fmaR<R>(hR, v4.im, k.im);
                        k.re = fmaR<R>(-hR / R(3), v3.re, k.re); k.im = fmaR<R>(-hR / R(3), v3.im, k.im);
                        k.re = fmaR<R>(hR / R(3), v2.re, k.re); k.im = fmaR<R>(hR / R(3), v2.im, k.im);
                    }
                    const int i = I_(q), j = J_(q);
                    K[(size_t)j * RPc + i] = k;
                    if (i != j) K[(size_t)i * RPc + j] = cplx<R>{k.re, -k.im};
                }
                if (tid < n) {
                    R d = c_t[tid];
                    if (a.sys.coul != 0) {
                        R u = R(0);
                        if (c_u[tid] != R(0)) u = fmaR<R>(c_u[tid], addR<R>(dgo, a.sys.shift), u);
                        d = addR<R>(d, u);
                    }
                    if (a.sys.has_ext) d = addR<R>(d, c_e[tid]);
                    if (a.sys.n_bins > 0) d = addR<R>(d, mulR<R>(pv, c_p[tid]));
                    Dd[tid] = d;
                    xod[tid] = dgo;
                    if (G == 0) xo0[tid] = dgo;
                }
                __syncthreads();
                // (b) xb = i [Kb, Delta], element products, t-scale partial
                double tsc = 0.0;
#pragma unroll
                for (int q = 0; q < EPT; ++q) {
                    if (ij[q] == ~0u) continue;
                    const int i = I_(q), j = J_(q);
                    const cplx<R> kb = K[(size_t)j * RPc + i];
                    // both diagonal slots read Kb_ij: FP64 sums them in place (the order of the
                    // per-stage kernels), FP32 adds Kb_ij (Delta_jj - Delta_ii) once afterwards
                    constexpr bool kDiagApart = std::is_same<R, float>::value;
                    R are = R(0), aim = R(0), bre = R(0), bim = R(0);
#pragma unroll
                    for (int sl = 0; sl < NE; ++sl) {          // sum_k Kb_ik Delta_kj over column j
                        if (kDiagApart && sl == P) continue;
                        const VEnt<R> e = ell[sl * n + j];
                        const R d = sl == P ? Dd[j] : e.v;
                        const cplx<R> x = K[(size_t)e.k * RPc + i];
                        are = fmaR<R>(x.re, d, are);
                        aim = fmaR<R>(x.im, d, aim);
                    }
#pragma unroll
                    for (int sl = 0; sl < NE; ++sl) {          // sum_k Kb_kj Delta_ki over column i
                        if (kDiagApart && sl == P) continue;
                        const VEnt<R> e = ell[sl * n + i];
                        const R d = sl == P ? Dd[i] : e.v;
                        const cplx<R> x = K[(size_t)j * RPc + e.k];
                        bre = fmaR<R>(x.re, d, bre);
                        bim = fmaR<R>(x.im, d, bim);
                    }
                    if constexpr (kDiagApart) {
                        const R dd = Dd[j] - Dd[i];
                        are = fmaR<R>(kb.re, dd, are);
                        aim = fmaR<R>(kb.im, dd, aim);
                    }
                    const cplx<R> xb = {-subR<R>(aim, bim), subR<R>(are, bre)};
                    const cplx<R> x = xg[q];
                    R ep;
                    if constexpr (std::is_same<R, float>::value) {
                        // one rounding per product term, no double conversions per element
                        const float d = fmaf(x.re, xb.re, x.im * xb.im);
                        tsc += (double)((i == j) ? d : 2.0f * d);
                        ep = fmaf(kb.re, x.im, -(kb.im * x.re));
                    } else {
                        const double wgt = (i == j) ? 1.0 : 2.0;
                        tsc += wgt * ((double)x.re * (double)xb.re + (double)x.im * (double)xb.im);
                        ep = (R)((double)kb.re * (double)x.im - (double)kb.im * (double)x.re);
                    }
                    EP[(size_t)j * RPc + i] = ep;
                    if (i != j) EP[(size_t)i * RPc + j] = -ep;
                    if constexpr (G > 0) {
                        XG(q) = xb;
                    } else {
                        if (i == j) {
                            x1d[i] = xb;                        // finished after the cross term
                        } else {
                            const cplx<R> v4 = X4(q), v3 = X3(q), v2 = X2(q);
                            lam[q].re = addR<R>(lam[q].re, addR<R>(addR<R>(addR<R>(xb.re, v2.re), v3.re), v4.re));
                            lam[q].im = addR<R>(lam[q].im, addR<R>(addR<R>(addR<R>(xb.im, v2.im), v3.im), v4.im));
                        }
                    }
                }
                // prefetch the next stage input (the stage before, or stage 4 of the step before)
                if (G > 0 || qs > 0) {
                    const int ng = G > 0 ? G - 1 : 3, nq = G > 0 ? qs : qs - 1;
                    const cplx<R>* X = a.seg + (size_t)nq * 4 * a.count + (size_t)ng * a.count;
#pragma unroll
                    for (int q = 0; q < EPT; ++q) xg[q] = ij[q] != ~0u ? X[base + P_(q)] : cplx<R>{R(0), R(0)};
                    if (tid < n) dgo = X[obase + cs(tid) + tid].re;
                    const long gl = (a.s0 + nq) * 4 + ng;
                    if (a.ptab) pv_n = a.ptab[gl];
                    if (a.envtab) env_n = a.envtab[gl];
                    if (a.bintab) bin_n = a.bintab[gl];
                }
                __syncthreads();
                // (c) db_j = 2 Im sum_r conj(Kb_rj) X_rj: eight lanes per column, four
                // columns per warp at a time
                double usc = 0.0, psc = 0.0;
                // a new pulse bin: each column group hands its finished bin's partial
                // to accf, summed after the cluster barrier
                int flush_bin = -1;
                if (bin >= 0 && bin != bin_acc) flush_bin = bin_acc;
                // (the four groups start 7 rows apart, so with a pitch of 1 mod 32 their
                // eight consecutive rows fall in four disjoint groups of banks)
                const int sub = lane & 7, grp = lane >> 3;
                for (int j0 = warp * 4; j0 < n; j0 += NW * 4) {
                    const int j = j0 + grp;
                    double im = 0.0;
                    if (j < n) {
                        const R* col = EP + (size_t)j * RPc;
                        int r = (7 * grp + sub) % n;
                        for (int u = sub; u < n; u += 8) {
                            im += (double)col[r];
                            r += 8;
                            if (r >= n) r -= n;
                        }
                    }
                    im += __shfl_xor_sync(0xffffffffu, im, 4);
                    im += __shfl_xor_sync(0xffffffffu, im, 2);
                    im += __shfl_xor_sync(0xffffffffu, im, 1);
                    if (sub == 0 && j < n) {
                        const double db = 2.0 * im;
                        peer_dbo[par * n + j] = (R)db;
                        tsc -= ((double)Dd[j] - (double)c_t[j]) * db;
                        if (a.sys.coul != 0) usc += db * ((double)c_u[j] * ((double)xod[j] + shift));
                        if (bin >= 0) psc += db * env * (double)c_p[j];
                    }
                }
                acct[tid] += tsc;
                if (sub == 0) {
                    const int gi = warp * 4 + grp;
                    accu[gi] += usc;
                    if (bin >= 0) {
                        if (bin != bin_acc) {
                            accf[gi] = accp[gi];
                            accp[gi] = 0.0;
                        }
                        accp[gi] += psc;
                    }
                }
                if (bin >= 0) bin_acc = bin;
                cl.sync();
                if (tid == 2 && flush_bin >= 0) {
                    double v = 0.0;
                    for (int g = 0; g < NW * 4; ++g) v += accf[g];
                    pac[2 + flush_bin] += v;
                }
                // (d) Hartree cross term from the partner's db on the diagonal
#pragma unroll
                for (int q = 0; q < EPT; ++q) {
                    if (ij[q] == ~0u) continue;
                    const int i = I_(q);
                    if (i != J_(q)) continue;
                    R add = R(0);
                    if (a.sys.coul != 0 && c_u[i] != R(0)) add = fmaR<R>(c_u[i], dbo[par * n + i], add);
                    if constexpr (G > 0) {
                        if (a.sys.coul != 0) XG(q).re = addR<R>(XG(q).re, add);
                    } else {
                        cplx<R> xb = x1d[i];
                        if (a.sys.coul != 0) xb.re = addR<R>(xb.re, add);
                        const cplx<R> v4 = X4(q), v3 = X3(q), v2 = X2(q);
                        lam[q].re = addR<R>(lam[q].re, addR<R>(addR<R>(addR<R>(xb.re, v2.re), v3.re), v4.re));
                        lam[q].im = addR<R>(lam[q].im, addR<R>(addR<R>(addR<R>(xb.im, v2.im), v3.im), v4.im));
                    }
                }
                par ^= 1;
            };
            stage(std::integral_constant<int, 3>());
            stage(std::integral_constant<int, 2>());
            stage(std::integral_constant<int, 1>());
            stage(std::integral_constant<int, 0>());
            // snapshot loss term at the step's input: lam_ii += w (n_other,ii + 1/2)
            if (gq % a.S == 0 && gq > 0) {
                const int t = (int)(gq / a.S);
                const double w = ((t == 0 || t == a.Tp - 1) ? 0.5 * a.dt : a.dt) * a.lscale;
#pragma unroll
                for (int q = 0; q < EPT; ++q) {
                    if (ij[q] == ~0u) continue;
                    const int i = I_(q);
                    if (i == J_(q)) lam[q].re += (R)(w * ((double)xo0[i] + 0.5));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q)
            if (ij[q] != ~0u) a.lam[base + P_(q)] = lam[q];
        // the segment's partials: one CTA sum each
        __syncthreads();
        {
            const double vt = warp_sum(acct[tid]);
            const double vu = warp_sum(lane < 4 ? accu[warp * 4 + lane] : 0.0);
            const double vp = warp_sum(lane < 4 ? accp[warp * 4 + lane] : 0.0);
            if (lane == 0) { red[warp * 3 + 0] = vu; red[warp * 3 + 1] = vt; red[warp * 3 + 2] = vp; }
        }
        __syncthreads();
        if (tid < 3) {
            double v = 0.0;
            for (int w = 0; w < NW; ++w) v += red[w * 3 + tid];
            if (tid < 2) pac[tid] += v;
            else if (bin_acc >= 0) pac[2 + bin_acc] += v;
        }
        __syncthreads();
        for (int c = tid; c < PW; c += NT) a.pacc[(size_t)m * PW + c] += pac[c];
        cl.sync();
    }
}

}  // namespace fpsg
