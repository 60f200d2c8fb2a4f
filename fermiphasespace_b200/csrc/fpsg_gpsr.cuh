// fpsg_gpsr.cuh — the GPSR drift (gaussian phase-space representation solver).
//
// FHGPSRSolver integrates a general complex density matrix per spin (the
// stochastic diffusion term makes it non-Hermitian) with a drift and a diffusion
// part per step (src/FHGPSRSolver.cpp:632-661).  The drift is the 3/8-rule RK4
// increment (step_Drift_RK4_38, src/FHGPSRSolver.cpp:168-206) of
//     f(rho) = -i (rho Delta - Delta rho),
//     Delta_up = tM + diagmat(U * diag(rho_dn)) [+ extPot],  Delta_dn likewise
// (src/FHGPSRSolver.cpp:111-134): no 1/2 shift, no V term, and a complex diagonal,
// because diag(rho) is complex.  This file computes that increment for a batch of
// trajectories, one RK stage per launch (each stage needs the other spin's
// diagonal of the same stage input):
//   stage 0: A = k1,            X1 = rho + k1 h / 3
//   stage 1: X2 = rho + (-A/3 + k2) h,  Bc = A + 3 k2,  A = A - k2
//   stage 2: X3 = rho + (A + k3) h,     Bc = Bc + 3 k3
//   stage 3: drift = (Bc + k4) h / 8
// in the reference's expression order, FP64, with the oracle's arithmetic contract
// (complex multiply-accumulates as fused multiply-adds, k ascending; the real
// off-diagonal entries of Delta as two of them), so the result is the oracle's to
// the bit.  One CTA per matrix at a time: the stage input staged in shared memory
// with an odd column pitch when it fits, read from global memory otherwise; Delta's
// static part from the column tables of the other paths, its diagonal formed per
// matrix in shared memory.
#pragma once
#include "fpsg_device.cuh"

namespace fpsg {

struct GpsrArgs {
    DevSys<double> sys;
    int M;                                   // matrices: 2 per trajectory (spin up, down)
    const cplx<double>* rho;                 // [M][n][n] column-major: the step's start
    const cplx<double>* X;                   // this stage's input (rho for stage 0)
    cplx<double>* Xn;                        // the next stage's input (stages 0-2)
    cplx<double>* A;                         // RK accumulators, [M][n][n]
    cplx<double>* Bc;
    cplx<double>* drift;                     // stage 3: the drift increment
    double h;                                // the step d_t
    int stage_x_in_smem;                     // 1: stage the input matrix in shared memory
};

__host__ __device__ inline size_t gpsr_smem_bytes(int n, bool x_in_smem)
{
    const size_t P = (size_t)(n | 1);
    return sizeof(cplx<double>) * ((x_in_smem ? (size_t)n * P : 0) + (size_t)n);
}

// acc += x * d (complex d), the oracle's four fused multiply-adds
__device__ __forceinline__ void gpsr_cmadd(cplx<double>& acc, cplx<double> x, cplx<double> d)
{
    acc.re = __fma_rn(x.re, d.re, acc.re);
    acc.re = __fma_rn(-x.im, d.im, acc.re);
    acc.im = __fma_rn(x.re, d.im, acc.im);
    acc.im = __fma_rn(x.im, d.re, acc.im);
}

template <int STAGE>
__global__ void __launch_bounds__(256) k_gpsr_stage(GpsrArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n;
    const size_t nn = (size_t)n * n;
    const int P = a.stage_x_in_smem ? (n | 1) : n;
    cplx<double>* xs = reinterpret_cast<cplx<double>*>(smem);
    cplx<double>* dsh = xs + (a.stage_x_in_smem ? (size_t)n * (n | 1) : 0);   // Delta_jj of this matrix
    const DevSys<double>& s = a.sys;
    for (int m = blockIdx.x; m < a.M; m += gridDim.x) {
        const cplx<double>* Xg = a.X + (size_t)m * nn;
        const cplx<double>* Xo = a.X + (size_t)(m ^ 1) * nn;      // the other spin's stage input
        const cplx<double>* Xr = Xg;
        if (a.stage_x_in_smem) {
            for (size_t q = threadIdx.x; q < nn; q += blockDim.x) {
                const int j = (int)(q / n), i = (int)(q - (size_t)j * n);
                xs[(size_t)j * P + i] = Xg[q];
            }
            Xr = xs;
        }
        // Delta_jj = ((tM_jj + sum_k U_kj rho_other,kk) + extPot_jj), complex
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            cplx<double> u = {0.0, 0.0};
            if (s.coul != 0)
                for (int q = s.up[j]; q < s.up[j + 1]; ++q) {
                    const cplx<double> o = Xo[(size_t)s.uk[q] * n + s.uk[q]];
                    u.re = __fma_rn(o.re, s.uv[q], u.re);
                    u.im = __fma_rn(o.im, s.uv[q], u.im);
                }
            cplx<double> d = {s.tdiag[j], 0.0};
            if (s.coul != 0) {
                d.re = __dadd_rn(d.re, u.re);
                d.im = __dadd_rn(d.im, u.im);
            }
            if (s.has_ext) {
                d.re = __dadd_rn(d.re, s.ediag[j]);
                d.im = __dadd_rn(d.im, 0.0);
            }
            dsh[j] = d;
        }
        __syncthreads();
        for (size_t q = threadIdx.x; q < nn; q += blockDim.x) {
            const int j = (int)(q / n), i = (int)(q - (size_t)j * n);
            // C1 = sum_k X_ik Delta_kj over column j; C2 = sum_k X_kj Delta_ik over column i
            cplx<double> c1 = {0.0, 0.0}, c2 = {0.0, 0.0};
            for (int e = s.hp[j]; e < s.hp[j + 1]; ++e) {
                const int k = s.hk[e];
                const cplx<double> x = Xr[(size_t)k * P + i];
                if (k == j) {
                    gpsr_cmadd(c1, x, dsh[j]);
                } else {
                    c1.re = __fma_rn(x.re, s.hv[e], c1.re);
                    c1.im = __fma_rn(x.im, s.hv[e], c1.im);
                }
            }
            for (int e = s.hp[i]; e < s.hp[i + 1]; ++e) {
                const int k = s.hk[e];
                const cplx<double> x = Xr[(size_t)j * P + k];
                if (k == i) {
                    gpsr_cmadd(c2, x, dsh[i]);
                } else {
                    c2.re = __fma_rn(x.re, s.hv[e], c2.re);
                    c2.im = __fma_rn(x.im, s.hv[e], c2.im);
                }
            }
            cplx<double> k;
            k.re = __dsub_rn(c1.im, c2.im);
            k.im = -__dsub_rn(c1.re, c2.re);
            const size_t g = (size_t)m * nn + q;
            const cplx<double> r = a.rho[g];
            const double h = a.h;
            if (STAGE == 0) {
                a.A[g] = k;
                a.Xn[g] = cplx<double>{__dadd_rn(r.re, div3_rn(__dmul_rn(k.re, h))),
                                       __dadd_rn(r.im, div3_rn(__dmul_rn(k.im, h)))};
            } else if (STAGE == 1) {
                const cplx<double> A = a.A[g];
                a.Xn[g] = cplx<double>{__dadd_rn(r.re, __dmul_rn(__dadd_rn(div3_rn(-A.re), k.re), h)),
                                       __dadd_rn(r.im, __dmul_rn(__dadd_rn(div3_rn(-A.im), k.im), h))};
                a.Bc[g] = cplx<double>{__dadd_rn(A.re, __dmul_rn(k.re, 3.0)), __dadd_rn(A.im, __dmul_rn(k.im, 3.0))};
                a.A[g] = cplx<double>{__dsub_rn(A.re, k.re), __dsub_rn(A.im, k.im)};
            } else if (STAGE == 2) {
                const cplx<double> A = a.A[g], Bc = a.Bc[g];
                a.Xn[g] = cplx<double>{__dadd_rn(r.re, __dmul_rn(__dadd_rn(A.re, k.re), h)),
                                       __dadd_rn(r.im, __dmul_rn(__dadd_rn(A.im, k.im), h))};
                a.Bc[g] = cplx<double>{__dadd_rn(Bc.re, __dmul_rn(k.re, 3.0)), __dadd_rn(Bc.im, __dmul_rn(k.im, 3.0))};
            } else {
                const cplx<double> Bc = a.Bc[g];
                // x / 8 == x * 0.125 exactly
                a.drift[g] = cplx<double>{__dmul_rn(__dmul_rn(__dadd_rn(Bc.re, k.re), h), 0.125),
                                          __dmul_rn(__dmul_rn(__dadd_rn(Bc.im, k.im), h), 0.125)};
            }
        }
        __syncthreads();     // the next matrix overwrites the staged input and Delta_jj
    }
}

}  // namespace fpsg
