// fpsg_device.cuh — device-side types and helpers shared by the trajectory kernels.
//
// State layout in HBM and shared memory: every spin density matrix rho (n x n,
// Hermitian) is stored as its packed upper triangle, column by column:
//     element (i, j), i <= j, lives at  cs(j) + i,   cs(j) = j (j + 1) / 2,
// so one matrix takes ne = n (n + 1) / 2 complex numbers (half of the dense
// col-major arma::cx_dmat the reference keeps, src/FHfTWASolver.cpp:331-334).
// A trajectory is [2][ne] (spin up, spin down); B trajectories are [B][2][ne].
//
// Arithmetic contract with the FP64 oracle (oracle/fps_oracle.c): the commutator
// of src/FHfTWASolver.cpp:598-599 is evaluated element by element as
//     a = sum_k X_ik Delta_kj,  b = sum_k Delta_ik X_kj   (k ascending)
//     dX_ij = -i (a - b)
// with one fused multiply-add per real component and term; Delta is real
// symmetric, so zero entries are skipped without changing a bit.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace fpsg {

// Aligned to its size, so that one complex element moves as one 8- or 16-byte access
// (every buffer of them starts at an allocation or a 16-byte aligned offset).
template <typename R> struct __align__(2 * sizeof(R)) cplx { R re, im; };

template <typename R> __device__ __forceinline__ R fmaR(R a, R b, R c);
template <> __device__ __forceinline__ double fmaR<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <> __device__ __forceinline__ float  fmaR<float>(float a, float b, float c)     { return __fmaf_rn(a, b, c); }
template <typename R> __device__ __forceinline__ R addR(R a, R b);
template <> __device__ __forceinline__ double addR<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float  addR<float>(float a, float b)    { return __fadd_rn(a, b); }
template <typename R> __device__ __forceinline__ R subR(R a, R b);
template <> __device__ __forceinline__ double subR<double>(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float  subR<float>(float a, float b)    { return __fsub_rn(a, b); }
template <typename R> __device__ __forceinline__ R mulR(R a, R b);
template <> __device__ __forceinline__ double mulR<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float  mulR<float>(float a, float b)    { return __fmul_rn(a, b); }
template <typename R> __device__ __forceinline__ R divR(R a, R b);
template <> __device__ __forceinline__ double divR<double>(double a, double b) { return __ddiv_rn(a, b); }
template <> __device__ __forceinline__ float  divR<float>(float a, float b)    { return __fdiv_rn(a, b); }

// x / 3 correctly rounded, in three operations instead of a general division, by
// Markstein's correction (P. Markstein, IBM J. Res. Develop. 34(1), 1990): with
// y = RN(1/3) (= 1/3 (1 - 2^-54)), q = RN(x y) lies within one ulp of x/3, the
// remainder r = x - 3q is exact as one fma, and RN(q + r y) is the correctly rounded
// quotient.  r = 0 means q is exact (and keeps the sign of a zero x).  Valid while
// x/3 is a normal number, as the RK stage values are.
__device__ __forceinline__ double div3_rn(double x)
{
    const double y = 0x1.5555555555555p-2;
    const double q = __dmul_rn(x, y);
    const double r = __fma_rn(-q, 3.0, x);
    return r == 0.0 ? q : __fma_rn(r, y, q);
}
template <typename R> __device__ __forceinline__ R div3R(R a);
template <> __device__ __forceinline__ double div3R<double>(double a) { return div3_rn(a); }
template <> __device__ __forceinline__ float  div3R<float>(float a)   { return __fdiv_rn(a, 3.0f); }

__host__ __device__ __forceinline__ int cs(int j) { return (j * (j + 1)) >> 1; }

// X(r, c) of a packed Hermitian matrix
template <typename R>
__device__ __forceinline__ cplx<R> getH(const cplx<R>* __restrict__ P, int r, int c)
{
    if (r <= c) return P[cs(c) + r];
    cplx<R> v = P[cs(r) + c];
    v.im = -v.im;
    return v;
}

// Static description of the system on the device (all arrays in global memory;
// small and read-only, they stay in L1/L2).
template <typename R>
struct DevSys {
    int n, ne;
    // Delta's static pattern by column j: entries k ascending, including k == j
    // (whose value is the dynamic diagonal); val = tM_kj + extPot_kj for k != j.
    const int* hp; const int* hk; const R* hv;
    // the two parts of hv's off-diagonal values, tM_kj and extPot_kj (0 at k == j),
    // for the energy rows tH and pe, which the reference keeps apart
    const R* tv; const R* xv;
    const R* tdiag;    // tM_jj
    const R* ediag;    // extPot_jj (static potential), 0 when absent
    const int* up; const int* uk; const R* uv;   // U by rows (nonzeros)
    const int* vp; const int* vk; const R* vv;   // V by rows (nonzeros), coulomb == DISTANCE
    const uint32_t* pij;  // packed index -> i | (j << 16)
    int coul;       // 0 null, 1 onSite, 2 distance
    int fock;       // HF with distance Coulomb: Delta has the exchange term -N o V
    int has_ext;
    R shift;        // 1/2 for fTWA (rho = N - 1/2), 0 for HF
    // time-dependent site pulse (0 bins: none)
    int n_bins; const double* amp; double bin_width, t0, td; const R* proj;
};

// Pulse value at time t (double, as the host defines the time grid).
template <typename R>
__device__ __forceinline__ double pulse_at(const DevSys<R>& s, double t)
{
    if (s.n_bins <= 0) return 0.0;
    double bf = floor(t / s.bin_width);
    long b = (long)bf;
    if (b < 0) b = 0;
    if (b > s.n_bins - 1) b = s.n_bins - 1;
    double x = (t - s.t0) / s.td;
    return s.amp[b] * exp(-0.5 * (x * x));
}

// Delta_jj = ((tM_jj + (U n_other)_j) + (V n_same)_j) + extPot_jj [+ pulse]
// (order of src/FHfTWASolver.cpp:571-594).  diag_same/diag_other: packed matrices.
template <typename R>
__device__ __forceinline__ R delta_diag(const DevSys<R>& s, int j, const cplx<R>* __restrict__ same,
                                        const cplx<R>* __restrict__ other, R pulse)
{
    R d = s.tdiag[j];
    if (s.coul != 0) {
        R u = R(0);
        for (int q = s.up[j]; q < s.up[j + 1]; ++q) {
            const int k = s.uk[q];
            u = fmaR<R>(s.uv[q], addR<R>(other[cs(k) + k].re, s.shift), u);
        }
        d = addR<R>(d, u);
        if (s.coul == 2) {
            R v = R(0);
            for (int q = s.vp[j]; q < s.vp[j + 1]; ++q) {
                const int k = s.vk[q];
                v = fmaR<R>(s.vv[q], addR<R>(same[cs(k) + k].re, s.shift), v);
            }
            d = addR<R>(d, v);
        }
    }
    if (s.has_ext) d = addR<R>(d, s.ediag[j]);
    if (s.n_bins > 0) d = addR<R>(d, mulR<R>(pulse, s.proj[j]));
    return d;
}

// k = -i (X Delta - Delta X) at (i, j), X packed, Delta diagonal in Dd.
template <typename R>
__device__ __forceinline__ cplx<R> commutator_elem(const DevSys<R>& s, const cplx<R>* __restrict__ X,
                                                   const R* __restrict__ Dd, int i, int j)
{
    R are = R(0), aim = R(0), bre = R(0), bim = R(0);
    for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
        const int k = s.hk[q];
        const R d = (k == j) ? Dd[j] : s.hv[q];
        const cplx<R> x = getH<R>(X, i, k);
        are = fmaR<R>(x.re, d, are);
        aim = fmaR<R>(x.im, d, aim);
    }
    for (int q = s.hp[i]; q < s.hp[i + 1]; ++q) {
        const int k = s.hk[q];
        const R d = (k == i) ? Dd[i] : s.hv[q];
        const cplx<R> x = getH<R>(X, k, j);
        bre = fmaR<R>(x.re, d, bre);
        bim = fmaR<R>(x.im, d, bim);
    }
    cplx<R> r;
    r.re = subR<R>(aim, bim);
    r.im = -subR<R>(are, bre);
    return r;
}

// ---------------------------------------------------------------- RK 3/8 stages
// Expression order of src/FHfTWASolver.cpp:647-660.  Per element the private
// state is rho, A and Bc:
//   stage 0: A = k1;                 X = rho + (k1*h)/3
//   stage 1: X = rho + ((-k1)/3 + k2)*h;  A = k1 - k2;  Bc = k1 + k2*3
//   stage 2: X = rho + (A + k3)*h;   Bc = Bc + k3*3
//   stage 3: rho = rho + ((Bc + k4)*h)/8
template <typename R>
__device__ __forceinline__ void rk_update(int stage, cplx<R> k, R h, cplx<R>& rho, cplx<R>& A,
                                          cplx<R>& Bc, cplx<R>& Xn)
{
    const R three = R(3);
    if constexpr (std::is_same<R, float>::value) {
        // FP32 stages: same combinations with reciprocal multiplies instead of
        // correctly rounded divisions (no bit-parity requirement in FP32)
        const float r3 = 1.0f / 3.0f, r8 = 0.125f;
        if (stage == 0) {
            A = k;
            Xn.re = rho.re + k.re * h * r3;
            Xn.im = rho.im + k.im * h * r3;
        } else if (stage == 1) {
            Xn.re = rho.re + (k.re - A.re * r3) * h;
            Xn.im = rho.im + (k.im - A.im * r3) * h;
            Bc.re = A.re + k.re * three;
            Bc.im = A.im + k.im * three;
            A.re = A.re - k.re;
            A.im = A.im - k.im;
        } else if (stage == 2) {
            Xn.re = rho.re + (A.re + k.re) * h;
            Xn.im = rho.im + (A.im + k.im) * h;
            Bc.re = Bc.re + k.re * three;
            Bc.im = Bc.im + k.im * three;
        } else {
            rho.re = rho.re + (Bc.re + k.re) * (h * r8);
            rho.im = rho.im + (Bc.im + k.im) * (h * r8);
            Xn = rho;
        }
        return;
    }
    if (stage == 0) {
        A = k;
        Xn.re = addR<R>(rho.re, div3R<R>(mulR<R>(k.re, h)));
        Xn.im = addR<R>(rho.im, div3R<R>(mulR<R>(k.im, h)));
    } else if (stage == 1) {
        Xn.re = addR<R>(rho.re, mulR<R>(addR<R>(div3R<R>(-A.re), k.re), h));
        Xn.im = addR<R>(rho.im, mulR<R>(addR<R>(div3R<R>(-A.im), k.im), h));
        Bc.re = addR<R>(A.re, mulR<R>(k.re, three));
        Bc.im = addR<R>(A.im, mulR<R>(k.im, three));
        A.re = subR<R>(A.re, k.re);
        A.im = subR<R>(A.im, k.im);
    } else if (stage == 2) {
        Xn.re = addR<R>(rho.re, mulR<R>(addR<R>(A.re, k.re), h));
        Xn.im = addR<R>(rho.im, mulR<R>(addR<R>(A.im, k.im), h));
        Bc.re = addR<R>(Bc.re, mulR<R>(k.re, three));
        Bc.im = addR<R>(Bc.im, mulR<R>(k.im, three));
    } else {
        // x / 8 == x * 0.125 exactly (a power of two): the same correctly rounded value
        rho.re = addR<R>(rho.re, mulR<R>(mulR<R>(addR<R>(Bc.re, k.re), h), R(0.125)));
        rho.im = addR<R>(rho.im, mulR<R>(mulR<R>(addR<R>(Bc.im, k.im), h), R(0.125)));
        Xn = rho;
    }
}

// stage times t, t + h/3, t + 2 dt/3 (snapshot interval: src/FHfTWASolver.cpp:653), t + h
__host__ __device__ __forceinline__ double stage_time(int stage, double t, double h, double dt)
{
    return stage == 0 ? t : stage == 1 ? t + h / 3.0 : stage == 2 ? t + 2.0 * dt / 3.0 : t + h;
}

// Philox4x32-10 (Salmon et al., SC'11) and the engine's Gaussian draw; identical
// to oracle_gauss_pair in the oracle so that samples can be compared.
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ void gauss_pair(uint64_t seed, uint64_t b, uint32_t e, double& g1, double& g2)
{
    uint32_t c[4] = { e, (uint32_t)b, (uint32_t)(b >> 32), 0x46505347u };
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((((uint64_t)c[0]) << 32) | c[1]) >> 11;
    const uint64_t d = ((((uint64_t)c[2]) << 32) | c[3]) >> 11;
    const double ua = __dmul_rn(__dadd_rn((double)a, 0.5), 0x1.0p-53);
    const double ub = __dmul_rn(__dadd_rn((double)d, 0.5), 0x1.0p-53);
    const double r = sqrt(-2.0 * log(ua));
    const double th = __dmul_rn(6.283185307179586476925286766559, ub);
    double sn, cn;
    sincos(th, &sn, &cn);
    g1 = __dmul_rn(r, cn);
    g2 = __dmul_rn(r, sn);
}

}  // namespace fpsg
