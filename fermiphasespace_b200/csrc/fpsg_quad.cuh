// fpsg_quad.cuh — the resident kernel for matrices too large for one CTA per spin.
//
// k_resident keeps a spin matrix in one CTA: the full Hermitian matrix twice
// (double-buffered) plus the state of every element.  That fits 227 KB of shared
// memory up to n = 100 in FP32, and not at all for FP64 at n = 100 (323 KB for the
// two matrix buffers alone).  k_resident_quad runs one trajectory on a cluster of
// four CTAs: rank r holds spin s = r >> 1 and owns half h = r & 1 of that spin's
// packed elements.  Each CTA keeps
//   X     the full matrix of its spin, single-buffered (n x RP complex, RP = n | 1,
//         column-major: X(i, k) at k*RP + i, plus a spare slot at n*RP),
//   rho   the state of its own elements (registers hold the RK accumulators),
//   Dd    Delta_jj of its spin for the current stage, dg the diagonal of X,
//   ell   Delta's columns in a compact fixed width W: every entry of column j in
//         ascending row order, the diagonal among them (recognised by its row),
//         zero-weight padding at the end — so a column with all its neighbours on
//         one side (periodic lattices) costs no more than any other,
// so FP64 fits up to n = 100 and FP32 up to n = 144.  One RK stage:
//   1. every CTA computes k for its elements from its local X and Dd (the column
//      sums of k_resident, in the same ascending order) and the RK
//      update, holding the new stage input in registers;
//   2. cluster barrier (every CTA is done reading X and Dd);
//   3. every CTA writes its new elements into its own X and, through distributed
//      shared memory, into its sibling's (rank ^ 1), both triangle positions; the
//      owners of diagonal elements write dg to both CTAs of the spin and, for an
//      on-site (or absent) Coulomb term, the partner spin's next-stage Delta_jj into
//      both of its CTAs;
//   4. cluster barrier; for a general Coulomb term each CTA then forms its Dd from
//      its dg and the partner spin's dg (read remotely).
// The arithmetic of every element is that of k_resident (and so of the FP64
// oracle), so the FP64 variant is bit-identical to the oracle.
#pragma once
#include "fpsg_kernels.cuh"

namespace fpsg {

// new stage inputs of the first QUAD_XS elements of every thread wait for the
// write phase in shared memory rather than registers (the accumulators of the
// others fill the register budget)
constexpr int QUAD_XS = 2;

// shared-memory layout of k_resident_quad (byte offsets); `xs` holds QUAD_XS x NT
// complex (NT = nt_ept / EPT is not needed here: callers pass nt)
template <typename R>
__host__ __device__ __forceinline__ ResLayout<R> quad_layout(int n, int W, int nt_ept, bool comp, int nt)
{
    ResLayout<R> L;
    const size_t RP = (size_t)(n | 1);
    size_t o = 0;
    L.x = o;    o = align16(o + sizeof(cplx<R>) * ((size_t)n * RP + 1));
    L.rho = o;  o = align16(o + sizeof(cplx<R>) * (size_t)nt_ept);
    L.dd = o;   o = align16(o + sizeof(R) * (size_t)n);
    L.dg = o;   o = align16(o + sizeof(R) * ((size_t)n + 1));
    L.es = o;   o = align16(o + sizeof(double) * 4 * 17);
    L.ell = o;  o = align16(o + sizeof(Ent<R>) * (size_t)n * W);
    L.lo = o;   if (comp) o = align16(o + sizeof(uint32_t) * (size_t)nt_ept);
    L.xs = o;   o = align16(o + sizeof(cplx<R>) * (size_t)QUAD_XS * nt);
    L.sd = o;   o = align16(o + sizeof(R) * 4 * (size_t)n);      // tM_jj, U_jj, extPot_jj, pulse projection
    L.total = o;
    return L;
}

// Distributed shared memory through 32-bit shared::cluster addresses (fewer
// registers than generic 64-bit pointers): the address of this CTA's `p` in the
// shared memory of cluster rank `rank`, and stores there.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r) : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster(uint32_t a, cplx<double> v)
{
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.re), "d"(v.im) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, cplx<float> v)
{
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.re), "f"(v.im) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, float v)
{
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

// The two halves take alternate 32-slot chunks of the matrix's slot order (full
// 32-row column segments first, then the 32 x 32 diagonal blocks), so both get the
// same mix of cheap and expensive chunks and every warp keeps 32 consecutive slots
// of one chunk.  Slot of a half's local element f, and the slots a half needs.
__host__ __device__ __forceinline__ int quad_slot(int f, int half)
{
    return ((((f >> 5) << 1) | half) << 5) | (f & 31);
}
__host__ __device__ __forceinline__ int quad_need(int ne)
{
    return ((ne + 63) / 64) * 32;
}

// One RK stage of this CTA's elements: k from the local X and Dd, the RK update,
// the new stage input left in xs[] (the first QUAD_XS elements) or xn[] (registers).
template <typename R, int NT, int EPT, int STAGE, int W>
__device__ __forceinline__ void quad_pass(const cplx<R>* __restrict__ X, const Ent<R>* __restrict__ ell,
                                          const R* __restrict__ Dd, cplx<R>* __restrict__ rhoS,
                                          const uint32_t (&ix)[EPT], cplx<R> (&Ar)[EPT], cplx<R> (&Br)[EPT],
                                          cplx<R> (&xn)[EPT], cplx<R>* __restrict__ xs, R h, int tid, int n,
                                          int RP, uint32_t* __restrict__ loS)
{
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        const bool valid = ix[q] != ~0u;
        const int i = valid ? (int)(ix[q] & 1023u) : 0;
        const int j = valid ? (int)((ix[q] >> 10) & 1023u) : 0;
        const Ent<R>* ej = ell + j;
        const Ent<R>* ei = ell + i;
        const int jo = j * RP, io = i * RP;
        // FP64 sums the diagonal terms in place (the oracle's order); FP32 drops them from
        // the sums and adds X_ij (Delta_jj - Delta_ii) afterwards (no cancellation)
        constexpr bool kDiagApart = std::is_same<R, float>::value;
        const R dj = kDiagApart ? R(0) : Dd[j], di = kDiagApart ? R(0) : Dd[i];
        R are = R(0), aim = R(0), bre = R(0), bim = R(0);
        // C_ij = sum over column j of X(i, k) Delta_kj, k ascending
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const Ent<R> e = ej[s * n];
            const cplx<R> x = X[e.off + i];
            const R w = e.off == jo ? dj : e.v;
            are = fmaR<R>(x.re, w, are);
            aim = fmaR<R>(x.im, w, aim);
        }
        // C_ji = sum over column i of X(j, k) Delta_ki, k ascending
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const Ent<R> e = ei[s * n];
            const cplx<R> x = X[e.off + j];
            const R w = e.off == io ? di : e.v;
            bre = fmaR<R>(x.re, w, bre);
            bim = fmaR<R>(x.im, w, bim);
        }
        if constexpr (kDiagApart) {
            const cplx<R> x = X[jo + i];                   // this element, X_ij
            const R dd = Dd[j] - Dd[i];
            are = fmaR<R>(x.re, dd, are);
            aim = fmaR<R>(x.im, dd, aim);
        }
        cplx<R> k;
        k.re = subR<R>(aim, -bim);
        k.im = -subR<R>(are, bre);
        cplx<R> rho = rhoS[f];
        cplx<R> out;
        if constexpr (STAGE == 3 && std::is_same<R, float>::value) {
            if (loS != nullptr) {
                rk_final_comp(k, h, rho, loS[f], Br[q]);
                out = rho;
            } else {
                rk_update<R>(STAGE, k, h, rho, Ar[q], Br[q], out);
            }
        } else {
            rk_update<R>(STAGE, k, h, rho, Ar[q], Br[q], out);
        }
        if (q < QUAD_XS) xs[q * NT + tid] = out;
        else xn[q] = out;
        if (STAGE == 3) rhoS[f] = rho;
    }
}

// ResArgs::ell_k / ell_v hold the compact columns here ([n][W], rows ascending, the
// diagonal among them, padding rows != the column with weight 0).
template <typename R, int NT, int EPT, int W>
__global__ void __launch_bounds__(NT, 1) k_resident_quad(ResArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    const int RP = n | 1;
    const int SPARE = n * RP;
    const bool comp = std::is_same<R, float>::value && a.state64 != nullptr;
    const ResLayout<R> L = quad_layout<R>(n, W, NT * EPT, comp, NT);
    cplx<R>* X = reinterpret_cast<cplx<R>*>(smem + L.x);
    cplx<R>* rhoS = reinterpret_cast<cplx<R>*>(smem + L.rho);
    R* Dd = reinterpret_cast<R*>(smem + L.dd);
    R* dg = reinterpret_cast<R*>(smem + L.dg);
    double* es = reinterpret_cast<double*>(smem + L.es);
    Ent<R>* ell = reinterpret_cast<Ent<R>*>(smem + L.ell);
    uint32_t* loS = comp ? reinterpret_cast<uint32_t*>(smem + L.lo) : nullptr;
    cplx<R>* xs = reinterpret_cast<cplx<R>*>(smem + L.xs);
    R* sd = reinterpret_cast<R*>(smem + L.sd);      // [4][n] static diagonal terms
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    static_assert(NW <= 16, "the per-warp energy partials (es) have room for 16 warps");
    const int RW = rec_width(n);     // doubles per snapshot record

    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int spin = rank >> 1, half = rank & 1;
    const int cid = blockIdx.x >> 2, ncl = gridDim.x >> 2;
    // remote shared memory: the sibling's X and dg, the partner spin's dg and Dd
    const uint32_t sibX = cluster_addr(X, rank ^ 1);
    const uint32_t sib_dg = cluster_addr(dg, rank ^ 1);
    const R* other_dg = cl.map_shared_rank(dg, rank ^ 2);        // read in records and Dd only
    const uint32_t pDd0 = cluster_addr(Dd, (rank ^ 2) & ~1);
    const uint32_t pDd1 = cluster_addr(Dd, (rank ^ 2) | 1);

    // compact column entries, slot-major (lanes reading consecutive columns hit
    // consecutive entries)
    for (int q = tid; q < n * W; q += NT) {
        Ent<R> e;
        const int col = q / W, slot = q - col * W;
        e.off = a.ell_k[q] * RP;
        e.v = a.ell_v[q];
        if constexpr (sizeof(Ent<R>) == 16) reinterpret_cast<int*>(&e)[1] = 0;
        ell[slot * n + col] = e;
    }
    // this CTA's elements: its half's alternate 32-slot chunks of the slot order
    uint32_t ix[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int p = quad_slot(tid + q * NT, half);
        uint32_t v = ~0u;
        if (p < ne) {
            const uint32_t o = a.order[p];
            v = (o & 0xffffu) | ((o >> 16) << 10);
        }
        ix[q] = v;
    }
    for (int j = tid; j < n; j += NT) {
        sd[j] = a.sys.tdiag[j];
        sd[n + j] = a.udiag ? a.udiag[j] : R(0);
        sd[2 * n + j] = a.sys.ediag[j];
        sd[3 * n + j] = a.sys.proj[j];
    }
    double* myslot = a.slots ? a.slots + (size_t)blockIdx.x * a.Tp * RW : nullptr;
    // rows past n (the odd-pitch padding row) are read only by zero-weight entries
    for (int q = tid; q < n * RP + 1; q += NT) X[q] = cplx<R>{R(0), R(0)};

    cplx<R> Ar[EPT], Br[EPT], xn[EPT];
    __syncthreads();
    for (int b = cid; b < a.B; b += ncl) {
        // the whole matrix of this spin into X; this CTA's elements into rho
        const size_t base = ((size_t)b * 2 + spin) * ne;
        for (int p = tid; p < ne; p += NT) {
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            cplx<R> v;
            if (comp) {
                const cplx<double> x = a.state64[base + p];
                v.re = (R)x.re;
                v.im = (R)x.im;
            } else {
                v = a.state[base + p];
            }
            X[i * RP + j] = cplx<R>{v.re, -v.im};
            X[j * RP + i] = v;
            if (i == j) dg[i] = v.re;
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            cplx<R> v = {R(0), R(0)};
            uint32_t lo = 0;
            if (ix[q] != ~0u) {
                const int p = res_packed(ix[q]);
                if (comp) {
                    const cplx<double> x = a.state64[base + p];
                    v.re = (R)x.re;
                    v.im = (R)x.im;
                    lo = pack_bf16x2((float)(x.re - (double)v.re), (float)(x.im - (double)v.im));
                } else {
                    v = a.state[base + p];
                }
            }
            rhoS[f] = v;
            if (comp) loS[f] = lo;
            Ar[q] = v; Br[q] = v;
        }
        bool dd_ok = false;                  // Dd already holds this stage's diagonal
        long gstep = a.step_base;
        cl.sync();
        for (int t = a.t_begin; t < a.t_end; ++t) {
            if (a.record) {
                // half 0 of each spin records: spin 0 du, du^2, du dd; spin 1 dd, dd^2
                if (half == 0) {
                    const int nvec = spin == 0 ? 3 : 2;
                    for (int w = tid; w < nvec * n; w += NT) {
                        const int oo = w / n, j = w - oo * n;
                        const int o = spin == 0 ? (oo == 0 ? 0 : oo == 1 ? 2 : 4) : (oo == 0 ? 1 : 3);
                        const double mine = (double)dg[j], oth = (double)other_dg[j];
                        const double du = spin == 0 ? mine : oth, dd = spin == 0 ? oth : mine;
                        if (!isfinite(du) || !isfinite(dd)) atomicOr(a.err, 1u);
                        const double acc = o == 0 ? du : o == 1 ? dd : o == 2 ? du * du : o == 3 ? dd * dd : du * dd;
                        atomicAdd(myslot + (size_t)t * RW + o * n + j, acc);
                    }
                    if (a.do_en) {
                        double e[4] = {0.0, 0.0, 0.0, 0.0};
                        energy_partials_full<R>(a.sys, X, RP, 0, dg, other_dg, spin, a.do_e1, a.do_e2, tid, NT, e);
                        double* ew = es + 4;
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const double v = warp_sum(e[c]);
                            if (lane == 0) ew[warp * 4 + c] = v;
                        }
                        __syncthreads();
                        if (tid < 4) {
                            double v = 0.0;
                            for (int q = 0; q < NW; ++q) v += ew[q * 4 + tid];
                            atomicAdd(myslot + (size_t)t * RW + 5 * n + tid, v);
                        }
                    }
                }
                if (a.whole) {
#pragma unroll
                    for (int q = 0; q < EPT; ++q) {
                        if (ix[q] == ~0u) continue;
                        const int f = tid + q * NT;
                        const int p = res_packed(ix[q]);
                        atomicAdd(&a.whole[((size_t)t * 2 + spin) * ne + p].x, (double)rhoS[f].re);
                        atomicAdd(&a.whole[((size_t)t * 2 + spin) * ne + p].y, (double)rhoS[f].im);
                    }
                }
            }
            const int nsteps = (a.hf && t == a.Tp - 1) ? 0 : a.S;
            for (int st = 0; st < nsteps; ++st, ++gstep) {
#pragma unroll
                for (int stage = 0; stage < 4; ++stage) {
                    if (!dd_ok) {
                        const R pv = a.sys.n_bins > 0 ? a.ptab[(gstep - a.step_base) * 4 + stage] : R(0);
                        for (int j = tid; j < n; j += NT) Dd[j] = delta_diag_v<R>(a.sys, j, dg, other_dg, pv);
                        __syncthreads();
                    }
                    // does another stage follow in this launch (possibly after a record)?
                    const bool more = stage < 3 || st + 1 < nsteps ||
                                      (t + 1 < a.t_end && a.S > 0 && !(a.hf && t + 1 == a.Tp - 1));
                    const bool fuse = a.udiag != nullptr && more;
                    R pvn = R(0);
                    if (fuse && a.sys.n_bins > 0) pvn = a.ptab[(gstep - a.step_base) * 4 + stage + 1];
                    if (stage == 0) quad_pass<R, NT, EPT, 0, W>(X, ell, Dd, rhoS, ix, Ar, Br, xn, xs, a.h, tid, n, RP, loS);
                    else if (stage == 1) quad_pass<R, NT, EPT, 1, W>(X, ell, Dd, rhoS, ix, Ar, Br, xn, xs, a.h, tid, n, RP, loS);
                    else if (stage == 2) quad_pass<R, NT, EPT, 2, W>(X, ell, Dd, rhoS, ix, Ar, Br, xn, xs, a.h, tid, n, RP, loS);
                    else quad_pass<R, NT, EPT, 3, W>(X, ell, Dd, rhoS, ix, Ar, Br, xn, xs, a.h, tid, n, RP, loS);
                    cl.sync();        // every CTA is done reading X, dg and Dd of this stage
#pragma unroll
                    for (int q = 0; q < EPT; ++q) {
                        const bool valid = ix[q] != ~0u;
                        const int i = valid ? (int)(ix[q] & 1023u) : 0;
                        const int j = valid ? (int)((ix[q] >> 10) & 1023u) : 0;
                        const int oij = valid ? j * RP + i : SPARE;
                        const int oji = valid ? i * RP + j : SPARE;
                        const cplx<R> v = q < QUAD_XS ? xs[q * NT + tid] : xn[q];
                        const cplx<R> vc = {v.re, -v.im};
                        X[oji] = vc;
                        X[oij] = v;                    // on the diagonal this second store wins
                        st_cluster(sibX + (uint32_t)oji * (uint32_t)sizeof(cplx<R>), vc);
                        st_cluster(sibX + (uint32_t)oij * (uint32_t)sizeof(cplx<R>), v);
                        if (valid && i == j) {
                            dg[i] = v.re;
                            st_cluster(sib_dg + (uint32_t)i * (uint32_t)sizeof(R), v.re);
                            if (fuse) {
                                // Delta_ii of the partner spin for the next stage (on-site U only)
                                R d = sd[i];
                                if (a.sys.coul != 0) {
                                    R u = R(0);
                                    const R uu = sd[n + i];
                                    if (uu != R(0)) u = fmaR<R>(uu, addR<R>(v.re, a.sys.shift), u);
                                    d = addR<R>(d, u);
                                }
                                if (a.sys.has_ext) d = addR<R>(d, sd[2 * n + i]);
                                if (a.sys.n_bins > 0) d = addR<R>(d, mulR<R>(pvn, sd[3 * n + i]));
                                st_cluster(pDd0 + (uint32_t)i * (uint32_t)sizeof(R), d);
                                st_cluster(pDd1 + (uint32_t)i * (uint32_t)sizeof(R), d);
                            }
                        }
                    }
                    cl.sync();        // X, dg (and the fused Dd) of the next stage are in place
                    dd_ok = fuse;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            if (ix[q] == ~0u) continue;
            const int f = tid + q * NT;
            const size_t gi = base + res_packed(ix[q]);
            if (comp) {
                const float2 lo = unpack_bf16x2(loS[f]);
                a.state64[gi] = cplx<double>{(double)rhoS[f].re + (double)lo.x, (double)rhoS[f].im + (double)lo.y};
            } else {
                a.state[gi] = rhoS[f];
            }
        }
        cl.sync();            // nobody reads this trajectory's X or dg any more
    }
}

}  // namespace fpsg

namespace fpsg {

// ------------------------------------------------------------------------------
// k_resident_quad_hp — the 4-CTA kernel with the spin matrix stored once per CTA as
// one real n x P array (P = n | 1, column-major, element (r, c) at c*P + r):
//     r < c:  Re X(r, c)        r > c:  Im X(c, r)        r == c:  X(r, r) (real)
// Half the bytes of the complex matrix, so it fits twice: the pass reads buffer
// `cur` and writes its new elements straight into buffer `cur ^ 1`, its own and
// (through distributed shared memory) its sibling's, and one cluster barrier per
// stage replaces k_resident_quad's two (no stage outputs held across a barrier, so
// no staging of them in registers or shared memory either).  A read of X(r, c)
// takes the two words a = M[c*P + r], b = M[r*P + c]:
//     r < c: (a, b)      r > c: (b, -a)      r == c: (a, 0)
// — the diagonal's imaginary part is taken as zero, as it is in every Hermitian
// state (the equations of motion keep it zero).  For 32 consecutive rows r and one
// column c, the a words are consecutive and the b words are P (odd) apart, so both
// reads are free of bank conflicts.  Every product and sum is the one of
// k_resident_quad in the same order, so the FP64 result is the oracle's to the bit.
// A column entry carries its row k and k * P: 16-byte Ent<double> as (off = k P,
// pad = k); 8-byte Ent<float> as off = k P | k << 20 (n P < 2^20) and an FP32 weight.
// FP64 takes the 8-byte entries (E8) when every weight is exactly an FP32 number
// (nearest-neighbour lattices with t = 1, say), which halves the per-lane column
// loads and changes no product.  FP32 keeps the compensated state update's residuals
// in registers (one word per element).
template <typename R, bool E8>
using HpEnt = typename std::conditional<E8, Ent<float>, Ent<R>>::type;

template <typename E>
__device__ __forceinline__ int hp_kP(const E& e)
{
    if constexpr (sizeof(E) == 16) return e.off;
    else return e.off & 0xfffff;
}
template <typename E>
__device__ __forceinline__ int hp_k(const E& e)
{
    if constexpr (sizeof(E) == 16) return reinterpret_cast<const int*>(&e)[1];
    else return (int)((uint32_t)e.off >> 20);
}

template <typename R>
__host__ __device__ __forceinline__ ResLayout<R> quad_hp_layout(int n, int W, int nt_ept, bool e8)
{
    ResLayout<R> L;
    const size_t P = (size_t)(n | 1);
    const size_t mw = (size_t)n * P + 2;          // + two spare words for empty slots
    size_t o = 0;
    L.x = o;    o = align16(o + sizeof(R) * 2 * mw);
    L.rho = o;  o = align16(o + sizeof(cplx<R>) * (size_t)nt_ept);
    L.dd = o;   o = align16(o + sizeof(R) * 2 * (size_t)n);
    L.dg = o;   o = align16(o + sizeof(R) * 2 * ((size_t)n + 1));
    L.es = o;   o = align16(o + sizeof(double) * 4 * 33);
    L.ell = o;  o = align16(o + (e8 ? sizeof(Ent<float>) : sizeof(Ent<R>)) * (size_t)n * W);
    L.lo = o;
    L.xs = o;
    L.sd = o;   o = align16(o + sizeof(R) * 4 * (size_t)n);
    L.total = o;
    return L;
}

// energy partials of one spin from the packed real matrix (Re X(k, j) at
// M[max(k, j) * P + min(k, j)]), in the order of energy_partials_full
template <typename R>
__device__ __forceinline__ void energy_partials_hp(const DevSys<R>& s, const R* M, int P, const R* dsame,
                                                   const R* dother, int spin, int do_e1, int do_e2, int lane,
                                                   int nlanes, double e[4])
{
    const double shift = (double)s.shift;
    for (int j = lane; j < s.n; j += nlanes) {
        const double nj = (double)dsame[j] + shift;
        double t0 = nj * (double)s.tdiag[j], t3 = 0.0;
        for (int q = s.hp[j]; q < s.hp[j + 1]; ++q) {
            const int k = s.hk[q];
            if (k == j) continue;
            const double x = (double)(k < j ? M[j * P + k] : M[k * P + j]);
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

// X(r, c) from the packed matrix (see k_resident_quad_hp)
template <typename R>
__device__ __forceinline__ cplx<R> hp_load(const R* __restrict__ M, int cP_r, int rP_c, int r, int c)
{
    const R a = M[cP_r], b = M[rP_c];
    cplx<R> x;
    x.re = r <= c ? a : b;
    x.im = r < c ? b : (r > c ? -a : R(0));
    return x;
}

// One RK stage of this CTA's elements from M (buffer cur): k, the RK update, and the
// new stage input written into Mn (this CTA's next buffer) and the sibling's.
// STAGE >= 0 fixes the stage at compile time; STAGE = -1 takes it from `stage`.  The
// kernel uses the run-time stage in FP64 (one copy of the unrolled element loop
// instead of four, and no spills: 310 -> 276 ms per 16384 x 20 steps at n = 100) and
// four specialised copies in FP32 (the run-time stage spills there: 28.5 -> 34.2 ms per
// 2048 x 20 steps at n = 108).
template <typename R, int NT, int EPT, int STAGE, int W, bool E8, int NH>
__device__ __forceinline__ void quad_hp_pass(int stage, const R* __restrict__ M, R* __restrict__ Mn, uint32_t sibMn,
                                             const HpEnt<R, E8>* __restrict__ ell, const R* __restrict__ Dd,
                                             cplx<R>* __restrict__ rhoS, const uint32_t (&ix)[EPT],
                                             cplx<R> (&Ar)[EPT], cplx<R> (&Br)[EPT], uint32_t (&lo)[EPT], bool comp,
                                             R h, int tid, int n, int P, R* __restrict__ dgn, uint32_t sib_dgn,
                                             bool fuse, uint32_t pDd0, uint32_t pDd1, const R* __restrict__ sd,
                                             const DevSys<R>& sys, R pvn)
{
    // FP64 sums the diagonal terms in place (the oracle's order); FP32 drops them from
    // the sums and adds X_ij (Delta_jj - Delta_ii) afterwards (no cancellation)
    constexpr bool kDiagApart = std::is_same<R, float>::value;
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int f = tid + q * NT;
        const bool valid = ix[q] != ~0u;
        const int i = valid ? (int)(ix[q] & 1023u) : 0;
        const int j = valid ? (int)((ix[q] >> 10) & 1023u) : 0;
        using E = HpEnt<R, E8>;
        const E* ej = ell + j;
        const E* ei = ell + i;
        const int jP = j * P, iP = i * P;
        const R dj = kDiagApart ? R(0) : Dd[j], di = kDiagApart ? R(0) : Dd[i];
        R are = R(0), aim = R(0), bre = R(0), bim = R(0);
        // FP64 warps whose every element has all its column-j rows k above i and all its
        // column-i rows k below j (bit 30, set at kernel start) read X without the
        // selection: X(i, k) = (a, b) and X(j, k) = (b, -a), the same products
        if (sizeof(R) == 8 && ((ix[q] >> 30) & 1u)) {
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const E e = ej[s * n];
                const int k = hp_k(e);
                const R ra = M[hp_kP(e) + i], rb = M[iP + k];
                const R w = k == j ? dj : (R)e.v;
                are = fmaR<R>(ra, w, are);
                aim = fmaR<R>(rb, w, aim);
            }
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const E e = ei[s * n];
                const int k = hp_k(e);
                const R ra = M[hp_kP(e) + j], rb = M[jP + k];
                const R w = k == i ? di : (R)e.v;
                bre = fmaR<R>(rb, w, bre);
                bim = fmaR<R>(-ra, w, bim);
            }
        } else {
            // C_ij = sum over column j of X(i, k) Delta_kj, k ascending
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const E e = ej[s * n];
                const int k = hp_k(e);
                const cplx<R> x = hp_load<R>(M, hp_kP(e) + i, iP + k, i, k);
                const R w = k == j ? dj : (R)e.v;
                are = fmaR<R>(x.re, w, are);
                aim = fmaR<R>(x.im, w, aim);
            }
            // C_ji = sum over column i of X(j, k) Delta_ki, k ascending
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const E e = ei[s * n];
                const int k = hp_k(e);
                const cplx<R> x = hp_load<R>(M, hp_kP(e) + j, jP + k, j, k);
                const R w = k == i ? di : (R)e.v;
                bre = fmaR<R>(x.re, w, bre);
                bim = fmaR<R>(x.im, w, bim);
            }
        }
        if constexpr (kDiagApart) {
            const cplx<R> x = hp_load<R>(M, jP + i, iP + j, i, j);      // this element, X_ij
            const R dd = Dd[j] - Dd[i];
            are = fmaR<R>(x.re, dd, are);
            aim = fmaR<R>(x.im, dd, aim);
        }
        cplx<R> k;
        k.re = subR<R>(aim, -bim);
        k.im = -subR<R>(are, bre);
        const int sg = STAGE >= 0 ? STAGE : stage;      // STAGE -1: any stage; -2: stages 0-2
        cplx<R> rho = rhoS[f];
        cplx<R> out;
        if constexpr (STAGE == 3 && std::is_same<R, float>::value) {
            if (comp) {
                rk_final_comp(k, h, rho, lo[q], Br[q]);
                out = rho;
            } else {
                rk_update<R>(3, k, h, rho, Ar[q], Br[q], out);
            }
        } else {
            static_assert(STAGE != -1 || std::is_same<R, double>::value, "FP32 takes stage 3 at compile time");
            rk_update<R>(sg, k, h, rho, Ar[q], Br[q], out);
        }
        if (sg == 3) rhoS[f] = rho;
        if (!valid) continue;
        // the new element into both copies of the next buffer
        const int ore = jP + i, oim = iP + j;
        Mn[ore] = out.re;
        if constexpr (NH == 2) st_cluster(sibMn + (uint32_t)ore * (uint32_t)sizeof(R), out.re);
        if (i != j) {
            Mn[oim] = out.im;
            if constexpr (NH == 2) st_cluster(sibMn + (uint32_t)oim * (uint32_t)sizeof(R), out.im);
        } else {
            dgn[i] = out.re;
            if constexpr (NH == 2) st_cluster(sib_dgn + (uint32_t)i * (uint32_t)sizeof(R), out.re);
            if (fuse) {
                // Delta_ii of the partner spin for the next stage (on-site U only)
                R d = sd[i];
                if (sys.coul != 0) {
                    R u = R(0);
                    const R uu = sd[n + i];
                    if (uu != R(0)) u = fmaR<R>(uu, addR<R>(out.re, sys.shift), u);
                    d = addR<R>(d, u);
                }
                if (sys.has_ext) d = addR<R>(d, sd[2 * n + i]);
                if (sys.n_bins > 0) d = addR<R>(d, mulR<R>(pvn, sd[3 * n + i]));
                st_cluster(pDd0 + (uint32_t)i * (uint32_t)sizeof(R), d);
                if constexpr (NH == 2) st_cluster(pDd1 + (uint32_t)i * (uint32_t)sizeof(R), d);
            }
        }
    }
}

// ResArgs::ell_k / ell_v hold the compact columns ([n][W], rows ascending, the
// diagonal among them, padding rows != the column with weight 0), as for
// k_resident_quad.  FP32 with ResArgs::state64 set: the compensated state update,
// the state read and written as FP64.  E8: 8-byte column entries (FP32 weights).
// NH: CTAs per spin — 2 (a 4-CTA cluster per trajectory, each CTA half of its spin's
// elements, the new elements written to the sibling too) or 1 (a 2-CTA cluster per
// trajectory, one CTA per spin holding all of its elements: no sibling, and every SM
// usable, where the spin's state fits beside the two matrix buffers).
template <typename R, int NT, int EPT, int W, bool E8, int NH>
__global__ void __launch_bounds__(NT, 1) k_resident_quad_hp(ResArgs<R> a)
{
    static_assert(NH == 1 || NH == 2, "one or two CTAs per spin");
    static_assert(E8 || sizeof(Ent<R>) == 16, "FP32 column entries are the 8-byte kind");
    using E = HpEnt<R, E8>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = a.sys.n, ne = a.sys.ne;
    const int P = n | 1;
    const int MW = n * P + 2;                       // words per buffer
    const bool comp = std::is_same<R, float>::value && a.state64 != nullptr;
    const ResLayout<R> L = quad_hp_layout<R>(n, W, NT * EPT, E8);
    R* M = reinterpret_cast<R*>(smem + L.x);        // [2][MW]
    cplx<R>* rhoS = reinterpret_cast<cplx<R>*>(smem + L.rho);
    R* Dd = reinterpret_cast<R*>(smem + L.dd);      // [2][n]
    R* dg = reinterpret_cast<R*>(smem + L.dg);      // [2][n + 1]
    double* es = reinterpret_cast<double*>(smem + L.es);
    E* ell = reinterpret_cast<E*>(smem + L.ell);
    R* sd = reinterpret_cast<R*>(smem + L.sd);      // [4][n] static diagonal terms
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    static_assert(NW <= 32, "the per-warp energy partials (es) have room for 32 warps");
    const int RW = rec_width(n);

    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int spin = NH == 2 ? rank >> 1 : rank, half = NH == 2 ? rank & 1 : 0;
    const int cid = blockIdx.x / (2 * NH), ncl = gridDim.x / (2 * NH);
    const int prank = NH == 2 ? rank ^ 2 : rank ^ 1;             // a CTA of the partner spin
    const uint32_t sibM = NH == 2 ? cluster_addr(M, rank ^ 1) : 0u;
    const uint32_t sib_dg = NH == 2 ? cluster_addr(dg, rank ^ 1) : 0u;
    const R* other_dg = cl.map_shared_rank(dg, prank);           // read in records and Dd only
    const uint32_t pDd0 = cluster_addr(Dd, NH == 2 ? (prank & ~1) : prank);
    const uint32_t pDd1 = NH == 2 ? cluster_addr(Dd, prank | 1) : pDd0;

    for (int q = tid; q < n * W; q += NT) {
        E e;
        const int col = q / W, slot = q - col * W;
        const int k = a.ell_k[q];
        if constexpr (sizeof(E) == 16) {
            e.off = k * P;
            reinterpret_cast<int*>(&e)[1] = k;
        } else {
            e.off = (k * P) | (k << 20);
        }
        e.v = (decltype(e.v))a.ell_v[q];
        ell[slot * n + col] = e;
    }
    uint32_t ix[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int p = NH == 2 ? quad_slot(tid + q * NT, half) : tid + q * NT;
        uint32_t v = ~0u;
        if (p < ne) {
            const uint32_t o = a.order[p];
            v = (o & 0xffffu) | ((o >> 16) << 10);
        }
        ix[q] = v;
    }
    for (int j = tid; j < n; j += NT) {
        sd[j] = a.sys.tdiag[j];
        sd[n + j] = a.udiag ? a.udiag[j] : R(0);
        sd[2 * n + j] = a.sys.ediag[j];
        sd[3 * n + j] = a.sys.proj[j];
    }
    double* myslot = a.slots ? a.slots + (size_t)blockIdx.x * a.Tp * RW : nullptr;
    // padding entries (weight 0) read rows < n only; the spare words take no reads
    for (int q = tid; q < 2 * MW; q += NT) M[q] = R(0);

    cplx<R> Ar[EPT], Br[EPT];
    uint32_t lo[EPT];
    __syncthreads();
    if constexpr (sizeof(R) == 8) {
        // mark (bit 30 of ix) the warps whose elements all read X(i, k) with i < k over
        // column j and X(j, k) with j > k over column i (the fast form of the pass)
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            bool ok = true;
            if (ix[q] != ~0u) {
                const int i = (int)(ix[q] & 1023u), j = (int)((ix[q] >> 10) & 1023u);
                for (int s = 0; s < W; ++s) ok = ok && hp_k(ell[s * n + j]) > i && hp_k(ell[s * n + i]) < j;
            }
            const bool all = __all_sync(0xffffffffu, ok);
            if (all && ix[q] != ~0u) ix[q] |= 1u << 30;
        }
    }
    for (int b = cid; b < a.B; b += ncl) {
        int cur = 0;
        const size_t base = ((size_t)b * 2 + spin) * ne;
        for (int p = tid; p < ne; p += NT) {
            const uint32_t ij = a.sys.pij[p];
            const int i = ij & 0xffff, j = ij >> 16;
            cplx<R> v;
            if (comp) {
                const cplx<double> x = a.state64[base + p];
                v.re = (R)x.re;
                v.im = (R)x.im;
            } else {
                v = a.state[base + p];
            }
            M[j * P + i] = v.re;
            if (i != j) M[i * P + j] = v.im;
            else dg[i] = v.re;
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int f = tid + q * NT;
            cplx<R> v = {R(0), R(0)};
            lo[q] = 0;
            if (ix[q] != ~0u) {
                const int p = res_packed(ix[q]);
                if (comp) {
                    const cplx<double> x = a.state64[base + p];
                    v.re = (R)x.re;
                    v.im = (R)x.im;
                    lo[q] = pack_bf16x2((float)(x.re - (double)v.re), (float)(x.im - (double)v.im));
                } else {
                    v = a.state[base + p];
                }
            }
            rhoS[f] = v;
            Ar[q] = v; Br[q] = v;
        }
        bool dd_ok = false;                  // Dd[cur] already holds this stage's diagonal
        long gstep = a.step_base;
        cl.sync();
        for (int t = a.t_begin; t < a.t_end; ++t) {
            const R* Mc = M + cur * MW;
            const R* dgc = dg + cur * (n + 1);
            const R* odgc = other_dg + cur * (n + 1);
            if (a.record) {
                // half 0 of each spin records: spin 0 du, du^2, du dd; spin 1 dd, dd^2.
                // dg[cur] and the partner's are not overwritten before the next stage's
                // barrier, which every CTA reaches after this.
                if (half == 0) {
                    const int nvec = spin == 0 ? 3 : 2;
                    for (int w = tid; w < nvec * n; w += NT) {
                        const int oo = w / n, j = w - oo * n;
                        const int o = spin == 0 ? (oo == 0 ? 0 : oo == 1 ? 2 : 4) : (oo == 0 ? 1 : 3);
                        const double mine = (double)dgc[j], oth = (double)odgc[j];
                        const double du = spin == 0 ? mine : oth, dd = spin == 0 ? oth : mine;
                        if (!isfinite(du) || !isfinite(dd)) atomicOr(a.err, 1u);
                        const double acc = o == 0 ? du : o == 1 ? dd : o == 2 ? du * du : o == 3 ? dd * dd : du * dd;
                        atomicAdd(myslot + (size_t)t * RW + o * n + j, acc);
                    }
                    if (a.do_en) {
                        double e[4] = {0.0, 0.0, 0.0, 0.0};
                        energy_partials_hp<R>(a.sys, Mc, P, dgc, odgc, spin, a.do_e1, a.do_e2, tid, NT, e);
                        double* ew = es + 4;
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const double v = warp_sum(e[c]);
                            if (lane == 0) ew[warp * 4 + c] = v;
                        }
                        __syncthreads();
                        if (tid < 4) {
                            double v = 0.0;
                            for (int q = 0; q < NW; ++q) v += ew[q * 4 + tid];
                            atomicAdd(myslot + (size_t)t * RW + 5 * n + tid, v);
                        }
                    }
                }
                if (a.whole) {
#pragma unroll
                    for (int q = 0; q < EPT; ++q) {
                        if (ix[q] == ~0u) continue;
                        const int f = tid + q * NT;
                        const int p = res_packed(ix[q]);
                        atomicAdd(&a.whole[((size_t)t * 2 + spin) * ne + p].x, (double)rhoS[f].re);
                        atomicAdd(&a.whole[((size_t)t * 2 + spin) * ne + p].y, (double)rhoS[f].im);
                    }
                }
            }
            const int nsteps = (a.hf && t == a.Tp - 1) ? 0 : a.S;
            for (int st = 0; st < nsteps; ++st, ++gstep) {
#define FPSG_HP_PASS(S_)                                                                                   \
    quad_hp_pass<R, NT, EPT, S_, W, E8, NH>(stage, Mr, Mw, sMw, ell, Ddc, rhoS, ix, Ar, Br, lo, comp, a.h, tid, n, P, \
                                        dgw, sdgw, fuse, pd0, pd1, sd, a.sys, pvn)
#define FPSG_HP_STAGE_BODY                                                                                     \
                    const int nxt = cur ^ 1;                                                                          \
                    R* Ddc = Dd + cur * n;                                                                            \
                    if (!dd_ok) {                                                                                     \
                        const R pv = a.sys.n_bins > 0 ? a.ptab[(gstep - a.step_base) * 4 + stage] : R(0);             \
                        const R* dgs = dg + cur * (n + 1);                                                            \
                        const R* dgo = other_dg + cur * (n + 1);                                                      \
                        for (int j = tid; j < n; j += NT) Ddc[j] = delta_diag_v<R>(a.sys, j, dgs, dgo, pv);           \
                        __syncthreads();                                                                              \
                    }                                                                                                 \
                    const bool more = stage < 3 || st + 1 < nsteps ||                                                 \
                                      (t + 1 < a.t_end && a.S > 0 && !(a.hf && t + 1 == a.Tp - 1));                   \
                    const bool fuse = a.udiag != nullptr && more;                                                     \
                    R pvn = R(0);                                                                                     \
                    if (fuse && a.sys.n_bins > 0) pvn = a.ptab[(gstep - a.step_base) * 4 + stage + 1];                \
                    const R* Mr = M + cur * MW;                                                                       \
                    R* Mw = M + nxt * MW;                                                                             \
                    const uint32_t sMw = sibM + (uint32_t)(nxt * MW) * (uint32_t)sizeof(R);                           \
                    R* dgw = dg + nxt * (n + 1);                                                                      \
                    const uint32_t sdgw = sib_dg + (uint32_t)(nxt * (n + 1)) * (uint32_t)sizeof(R);                   \
                    const uint32_t pd0 = pDd0 + (uint32_t)(nxt * n) * (uint32_t)sizeof(R);                            \
                    const uint32_t pd1 = pDd1 + (uint32_t)(nxt * n) * (uint32_t)sizeof(R);                            \
                    if constexpr (std::is_same<R, double>::value) {                                                   \
                        FPSG_HP_PASS(-1);                                                                             \
                    } else {                                                                                          \
                        if constexpr (EPT >= 9) {                                                                     \
                            if (stage < 3) FPSG_HP_PASS(-2);                                                          \
                            else FPSG_HP_PASS(3);                                                                     \
                        } else {                                                                                      \
                            if (stage == 0) FPSG_HP_PASS(0);                                                          \
                            else if (stage == 1) FPSG_HP_PASS(1);                                                     \
                            else if (stage == 2) FPSG_HP_PASS(2);                                                     \
                            else FPSG_HP_PASS(3);                                                                     \
                        }                                                                                             \
                    }                                                                                                 \
                    cl.sync(); /* buffer nxt (and its dg, fused Dd) complete in every CTA */                          \
                    cur = nxt;                                                                                        \
                    dd_ok = fuse;
                // FP64: the stage loop rolled, one copy of the pass for all stages.  FP32
                // with many elements per thread: rolled, one copy for stages 1-3 and one
                // for the last stage's compensated update (four copies overflow the
                // instruction cache: 12x12 grid 54.9 -> 48.1 ms per 2048 x 20 steps);
                // with few: unrolled, four specialised copies (kagome 108: 32.3 -> 28.5 ms)
                if constexpr (std::is_same<R, double>::value || EPT >= 9) {
#pragma unroll 1
                    for (int stage = 0; stage < 4; ++stage) {
                        FPSG_HP_STAGE_BODY
                    }
                } else {
#pragma unroll
                    for (int stage = 0; stage < 4; ++stage) {
                        FPSG_HP_STAGE_BODY
                    }
                }
#undef FPSG_HP_STAGE_BODY
#undef FPSG_HP_PASS
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            if (ix[q] == ~0u) continue;
            const int f = tid + q * NT;
            const size_t gi = base + res_packed(ix[q]);
            if (comp) {
                const float2 l = unpack_bf16x2(lo[q]);
                a.state64[gi] = cplx<double>{(double)rhoS[f].re + (double)l.x, (double)rhoS[f].im + (double)l.y};
            } else {
                a.state[gi] = rhoS[f];
            }
        }
        cl.sync();            // nobody reads this trajectory's matrices or dg any more
    }
}

}  // namespace fpsg
