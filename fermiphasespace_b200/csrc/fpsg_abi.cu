// fpsg_abi.cu — the C ABI declared in include/fpsg.h: context, device tables,
// path selection and launch sequencing.  No exception crosses the boundary.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/fpsg.h"
#include "fpsg_kernels.cuh"
#include "fpsg_resident.h"
#include "fpsg_util_kernels.cuh"
#include "fpsg_adjoint.cuh"
#include "fpsg_gpsr.cuh"
#include "fpsg_dense.h"

using namespace fpsg;

namespace {

struct DevAlloc {
    void* p = nullptr;
    size_t bytes = 0;
};

template <typename R>
struct DevTables {
    int *hp = nullptr, *hk = nullptr, *up = nullptr, *uk = nullptr, *vp = nullptr, *vk = nullptr;
    R *tv = nullptr, *xv = nullptr;   // tM_kj and extPot_kj at the entries of hv (energies)
    R *hv = nullptr, *tdiag = nullptr, *ediag = nullptr, *uv = nullptr, *vv = nullptr, *proj = nullptr;
    int* ell_k = nullptr;   // [n][2P+1] fixed-width columns of Delta (resident path), -1 = padding
    R* ell_v = nullptr;
    int* ell_pad = nullptr; // [2P+1] dominant neighbour offset k - j of each slot
    std::vector<int> ell_dpad;
    int ell_p = 0;          // P, or 0 when a column has more than 8 entries on one side
    // compact columns (two-CTAs-per-spin kernel): [n][cell_w] rows ascending with the
    // diagonal among them, padding rows (!= the column) with weight 0 at the end
    int* cell_k = nullptr;
    R* cell_v = nullptr;
    int cell_w = 0;         // 5, 9, 13 or 17; 0 when a column has more than 17 entries
    bool cell_f32 = false;  // every compact weight is exactly an FP32 number
    R* udiag = nullptr;     // U_jj (0 where row j of U has no entry)
    bool dd_fusable = false;  // no Coulomb term, or on-site only (U diagonal): the resident
                              // pass can form the next stage's Delta_jj itself
};

struct Status {
    int code;
    std::string msg;
};

}  // namespace

struct fpsg_ctx {
    int device = 0;
    uint64_t flags = 0;                    // FPSG_FLAG_*
    int sm_count = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    uint64_t mem_cap = 0, mem_used = 0;
    std::vector<DevAlloc> allocs;
    std::vector<DevAlloc> pool;            // per-call scratch kept for the next call (counted in mem_used)
    int64_t grad_keep = -1;                // fpsg_set_grad_memory: -1 automatic
    fpsg_grad_info grad_info = {0, 0, 0, 0};   // the last fpsg_grad call's plan

    // system
    bool sys_set = false;
    int n = 0, ne = 0, coul = 0, ext_null = 1;
    bool ext_offdiag = false;              // the static potential has an off-diagonal entry
    std::vector<double> tM, U, V, ext;     // dense real parts, col-major
    uint32_t* pij = nullptr;
    uint32_t* res_order = nullptr;         // resident kernel's slot order (see res_slot_order)
    DevTables<double> t64;
    DevTables<float> t32;
    int nnz_h = 0;

    // pulse
    int n_bins = 0;
    std::vector<double> amp, proj;
    double bin_width = 1.0, p_t0 = 0.0, p_td = 1.0;
    double* d_amp = nullptr;

    // state (canonical FP64 packed)
    int B = 0;
    cplx<double>* rho64 = nullptr;

    // batch autotuner: batch shape -> (threads per CTA, schedule)
    std::map<std::string, std::pair<int, int>> batch_tune;
};

namespace {

int fail(fpsg_ctx* c, int code, const std::string& m)
{
    if (c) c->err = m;
    return code;
}

int cuda_fail(fpsg_ctx* c, cudaError_t e, const char* where)
{
    return fail(c, FPSG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);  \
    } while (0)

int dalloc(fpsg_ctx* ctx, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (ctx->mem_cap && ctx->mem_used + bytes > ctx->mem_cap)
        return fail(ctx, FPSG_ERR_OOM, "device memory cap reached (" + std::to_string(ctx->mem_used + bytes) +
                                           " > " + std::to_string(ctx->mem_cap) + " bytes)");
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(ctx, FPSG_ERR_OOM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    ctx->allocs.push_back({*p, bytes});
    ctx->mem_used += bytes;
    return FPSG_OK;
}

void dfree(fpsg_ctx* ctx, void* p)
{
    if (!p) return;
    for (size_t i = 0; i < ctx->allocs.size(); ++i)
        if (ctx->allocs[i].p == p) {
            ctx->mem_used -= ctx->allocs[i].bytes;
            ctx->allocs.erase(ctx->allocs.begin() + i);
            break;
        }
    cudaFree(p);
}

// Per-call scratch.  A run allocates its stage buffers, FP32 state copies and
// record buffers for the call only; cudaMalloc/cudaFree of a GB-sized buffer per
// call costs far more host time than a short run takes on the device, so released
// scratch stays allocated in the context's pool and the next call of a similar size
// takes it back.  Pooled blocks count towards the memory cap; a cap, an allocation
// failure or fpsg_destroy frees them.
void trim_pool(fpsg_ctx* ctx)
{
    std::vector<DevAlloc> blocks;
    blocks.swap(ctx->pool);
    for (auto& a : blocks) dfree(ctx, a.p);
}

int talloc(fpsg_ctx* ctx, void** p, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    int best = -1;
    for (int i = 0; i < (int)ctx->pool.size(); ++i) {
        const size_t b = ctx->pool[i].bytes;
        if (b >= bytes && b <= 2 * bytes + (1u << 20) && (best < 0 || b < ctx->pool[best].bytes)) best = i;
    }
    if (best >= 0) {
        *p = ctx->pool[best].p;
        ctx->pool.erase(ctx->pool.begin() + best);
        return FPSG_OK;
    }
    int rc = dalloc(ctx, p, bytes);
    if (rc == FPSG_ERR_OOM && !ctx->pool.empty()) {
        trim_pool(ctx);
        rc = dalloc(ctx, p, bytes);
    }
    return rc;
}

void trelease(fpsg_ctx* ctx, void* p)
{
    if (!p) return;
    for (auto& a : ctx->pool)
        if (a.p == p) return;
    for (auto& a : ctx->allocs)
        if (a.p == p) {
            ctx->pool.push_back(a);
            return;
        }
}

// Slot order of the resident kernel's elements (i | j << 16, i <= j).  A warp
// takes 32 consecutive slots; its loads of X(k, i) for one column k are
// conflict-free when the 32 elements share the column j and have consecutive
// rows.  So the full 32-row segments (rows 32r .. 32r+31 of a column j >= 32r+32)
// come first.  Each 32 x 32 diagonal block follows as 16 warps of two columns:
// column c (rows 0..c of the block) with column 31 - c without its diagonal
// element (rows 0..30-c), 32 slots in all; the 16 diagonal elements left over from
// all blocks close the order, after a trailing partial block in packed order.
// Every slot computes the same value in any order; only the bank pattern changes.
std::vector<uint32_t> res_slot_order(int n)
{
    std::vector<uint32_t> o, left;
    o.reserve((size_t)n * (n + 1) / 2);
    auto put = [&](std::vector<uint32_t>& v, int i, int j) { v.push_back((uint32_t)i | ((uint32_t)j << 16)); };
    for (int r = 0; r + 32 < n; r += 32)
        for (int j = r + 32; j < n; ++j)
            for (int i = r; i < r + 32; ++i) put(o, i, j);
    for (int r = 0; r < n; r += 32) {
        if (r + 32 <= n) {
            for (int c = 0; c < 16; ++c) {
                for (int i = r; i <= r + c; ++i) put(o, i, r + c);
                const int cc = 31 - c;
                for (int i = r; i < r + cc; ++i) put(o, i, r + cc);
                put(left, r + cc, r + cc);
            }
        } else {
            for (int j = r; j < n; ++j)
                for (int i = r; i <= j; ++i) put(o, i, j);
        }
    }
    o.insert(o.end(), left.begin(), left.end());
    return o;
}

// Small host tables (system tables, occupations, rotations) go into pooled blocks,
// so that a new fpsg_set_system or fpsg_sample reuses the previous call's blocks
// instead of a cudaFree / cudaMalloc pair per table.
template <typename T>
int upload(fpsg_ctx* ctx, T** dst, const std::vector<T>& v)
{
    int rc = talloc(ctx, (void**)dst, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (rc) return rc;
    if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return FPSG_OK;
}

template <typename R>
void free_tables(fpsg_ctx* ctx, DevTables<R>& t)
{
    trelease(ctx, t.hp); trelease(ctx, t.hk); trelease(ctx, t.up); trelease(ctx, t.uk); trelease(ctx, t.vp);
    trelease(ctx, t.tv); trelease(ctx, t.xv);
    trelease(ctx, t.vk); trelease(ctx, t.hv); trelease(ctx, t.tdiag); trelease(ctx, t.ediag); trelease(ctx, t.uv);
    trelease(ctx, t.vv); trelease(ctx, t.proj); trelease(ctx, t.ell_k); trelease(ctx, t.ell_v);
    trelease(ctx, t.ell_pad); trelease(ctx, t.udiag); trelease(ctx, t.cell_k); trelease(ctx, t.cell_v);
    t = DevTables<R>();
}

template <typename R>
int build_tables(fpsg_ctx* ctx, DevTables<R>& t)
{
    const int n = ctx->n;
    std::vector<int> hp(1, 0), hk, up(1, 0), uk, vp(1, 0), vk;
    std::vector<R> hv, tvv, xvv, tdiag(n), ediag(n, R(0)), uv, vv, proj(n, R(0));
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < n; ++k) {
            const double tv = ctx->tM[(size_t)j * n + k];
            const double ev = ctx->ext_null ? 0.0 : ctx->ext[(size_t)j * n + k];
            if (k == j || tv != 0.0 || ev != 0.0) {
                hk.push_back(k);
                hv.push_back(ctx->ext_null ? (R)tv : (R)(tv + ev));
                tvv.push_back(k == j ? R(0) : (R)tv);
                xvv.push_back(k == j ? R(0) : (R)ev);
            }
        }
        hp.push_back((int)hk.size());
        tdiag[j] = (R)ctx->tM[(size_t)j * n + j];
        if (!ctx->ext_null) ediag[j] = (R)ctx->ext[(size_t)j * n + j];
        for (int k = 0; k < n; ++k) {
            const double u = ctx->U[(size_t)k * n + j];   // U(j, k)
            if (u != 0.0) { uk.push_back(k); uv.push_back((R)u); }
            const double v = ctx->V[(size_t)k * n + j];
            if (v != 0.0) { vk.push_back(k); vv.push_back((R)v); }
        }
        up.push_back((int)uk.size());
        vp.push_back((int)vk.size());
    }
    if (ctx->n_bins > 0)
        for (int j = 0; j < n; ++j) proj[j] = (R)ctx->proj[j];
    ctx->nnz_h = (int)hk.size();
    std::vector<R> udiag(n, R(0));
    bool u_diag_only = true;
    for (int j = 0; j < n; ++j)
        for (int q = up[j]; q < up[j + 1]; ++q) {
            if (uk[q] == j) udiag[j] = uv[q];
            else u_diag_only = false;
        }
    t.dd_fusable = ctx->coul == FPSG_COULOMB_NULL || (ctx->coul == FPSG_COULOMB_ONSITE && u_diag_only);
    // fixed-width columns: P entries below the diagonal (zero padding in front),
    // the diagonal, P above (zero padding at the end); the padding reads column j
    // and adds an exact zero, so the sums keep the oracle's order and bits.
    int maxside = 0;
    for (int j = 0; j < n; ++j) {
        int lo = 0, hi = 0;
        for (int q = hp[j]; q < hp[j + 1]; ++q) (hk[q] < j ? lo : hk[q] > j ? hi : lo) += (hk[q] == j) ? 0 : 1;
        maxside = std::max(maxside, std::max(lo, hi));
    }
    t.ell_p = maxside <= 2 ? 2 : maxside <= 4 ? 4 : maxside <= 8 ? 8 : 0;
    std::vector<int> ek;
    std::vector<R> ev;
    if (t.ell_p) {
        const int P = t.ell_p, NE = 2 * P + 1;
        ek.assign((size_t)n * NE, 0);
        ev.assign((size_t)n * NE, R(0));
        for (int j = 0; j < n; ++j) {
            std::vector<int> lk, uk2;
            std::vector<R> lv, uv2;
            for (int q = hp[j]; q < hp[j + 1]; ++q) {
                if (hk[q] < j) { lk.push_back(hk[q]); lv.push_back(hv[q]); }
                else if (hk[q] > j) { uk2.push_back(hk[q]); uv2.push_back(hv[q]); }
            }
            int* K = ek.data() + (size_t)j * NE;
            R* Vv = ev.data() + (size_t)j * NE;
            for (int q = 0; q < NE; ++q) { K[q] = -1; Vv[q] = R(0); }
            K[P] = j;
            const int pad = P - (int)lk.size();
            for (size_t q = 0; q < lk.size(); ++q) { K[pad + q] = lk[q]; Vv[pad + q] = lv[q]; }
            for (size_t q = 0; q < uk2.size(); ++q) { K[P + 1 + q] = uk2[q]; Vv[P + 1 + q] = uv2[q]; }
        }
        // padding entries (K = -1) get the slot's dominant neighbour offset, so that
        // the shared-memory reads of neighbouring lanes keep their bank pattern
        t.ell_dpad.assign(NE, 0);
        for (int q = 0; q < NE; ++q) {
            std::map<int, int> cnt;
            for (int j = 0; j < n; ++j)
                if (ek[(size_t)j * NE + q] >= 0) cnt[ek[(size_t)j * NE + q] - j]++;
            int best = 0, bc = -1;
            for (auto& kv : cnt) if (kv.second > bc) { bc = kv.second; best = kv.first; }
            t.ell_dpad[q] = best;
        }
    }
    // compact columns: the entries of column j in ascending row order with zero-weight
    // padding.  Lanes reading the same slot of neighbouring columns keep their bank
    // pattern when the slot means the same offset k - j in every column, so the slots
    // follow the most common offset pattern (for a grid: -nx, -1, 0, +1, +nx) and a
    // column whose offsets are a subset of it puts each entry at its offset's slot;
    // other columns are packed in ascending order.  Either way the real entries keep
    // their ascending order (the oracle's summation order).  A padding entry reads a
    // row at the slot's offset when one exists (else a neighbouring row), never row j
    // itself, which marks the diagonal.
    int maxcol = 0;
    for (int j = 0; j < n; ++j) maxcol = std::max(maxcol, hp[j + 1] - hp[j]);
    std::vector<int> pattern;
    {
        std::map<std::vector<int>, int> freq;
        for (int j = 0; j < n; ++j) {
            std::vector<int> offs;
            for (int q = hp[j]; q < hp[j + 1]; ++q) offs.push_back(hk[q] - j);
            freq[offs]++;
        }
        int bestc = -1;
        for (auto& kv : freq)
            if ((int)kv.first.size() >= maxcol - 0 && kv.second > bestc) { bestc = kv.second; pattern = kv.first; }
        // a column of maximal size defines the pattern; fall back to the most common one
        if (pattern.empty())
            for (auto& kv : freq)
                if (kv.second > bestc) { bestc = kv.second; pattern = kv.first; }
    }
    const int wneed = std::max(maxcol, (int)pattern.size());
    t.cell_w = wneed <= 5 ? 5 : wneed <= 9 ? 9 : wneed <= 13 ? 13 : wneed <= 17 ? 17 : 0;
    std::vector<int> ck;
    std::vector<R> cv;
    if (t.cell_w && n > 1) {
        const int Wc = t.cell_w;
        ck.assign((size_t)n * Wc, 0);
        cv.assign((size_t)n * Wc, R(0));
        for (int j = 0; j < n; ++j) {
            int* K = ck.data() + (size_t)j * Wc;
            R* Vv = cv.data() + (size_t)j * Wc;
            const int nb = j > 0 ? j - 1 : j + 1;
            for (int s2 = 0; s2 < Wc; ++s2) { K[s2] = -1; Vv[s2] = R(0); }
            bool aligned = true;
            std::vector<int> slot_of;
            for (int q = hp[j]; q < hp[j + 1]; ++q) {
                const auto it = std::find(pattern.begin(), pattern.end(), hk[q] - j);
                if (it == pattern.end()) { aligned = false; break; }
                slot_of.push_back((int)(it - pattern.begin()));
            }
            if (aligned) {
                for (int q = hp[j], e = 0; q < hp[j + 1]; ++q, ++e) {
                    K[slot_of[e]] = hk[q];
                    Vv[slot_of[e]] = hk[q] == j ? R(0) : hv[q];
                }
                for (int s2 = 0; s2 < Wc; ++s2)
                    if (K[s2] < 0) {
                        const int kk = s2 < (int)pattern.size() ? j + pattern[s2] : -1;
                        K[s2] = (kk >= 0 && kk < n && kk != j) ? kk : nb;
                    }
            } else {
                int s2 = 0;
                for (int q = hp[j]; q < hp[j + 1]; ++q, ++s2) {
                    K[s2] = hk[q];
                    Vv[s2] = hk[q] == j ? R(0) : hv[q];
                }
                for (; s2 < Wc; ++s2) K[s2] = nb;
            }
        }
    } else {
        t.cell_w = 0;
    }
    t.cell_f32 = true;
    for (const R v : cv)
        if ((R)(float)v != v) t.cell_f32 = false;
    int rc;
    if ((rc = upload(ctx, &t.cell_k, ck)) || (rc = upload(ctx, &t.cell_v, cv))) return rc;
    if ((rc = upload(ctx, &t.hp, hp)) || (rc = upload(ctx, &t.hk, hk)) || (rc = upload(ctx, &t.hv, hv)) ||
        (rc = upload(ctx, &t.tv, tvv)) || (rc = upload(ctx, &t.xv, xvv)) ||
        (rc = upload(ctx, &t.tdiag, tdiag)) || (rc = upload(ctx, &t.ediag, ediag)) ||
        (rc = upload(ctx, &t.up, up)) || (rc = upload(ctx, &t.uk, uk)) || (rc = upload(ctx, &t.uv, uv)) ||
        (rc = upload(ctx, &t.vp, vp)) || (rc = upload(ctx, &t.vk, vk)) || (rc = upload(ctx, &t.vv, vv)) ||
        (rc = upload(ctx, &t.proj, proj)) || (rc = upload(ctx, &t.ell_k, ek)) || (rc = upload(ctx, &t.ell_v, ev)) ||
        (rc = upload(ctx, &t.ell_pad, t.ell_dpad)) || (rc = upload(ctx, &t.udiag, udiag)))
        return rc;
    return FPSG_OK;
}

template <typename R>
DevSys<R> make_sys(fpsg_ctx* ctx, const DevTables<R>& t, int method)
{
    DevSys<R> s;
    s.n = ctx->n; s.ne = ctx->ne;
    s.hp = t.hp; s.hk = t.hk; s.hv = t.hv; s.tv = t.tv; s.xv = t.xv; s.tdiag = t.tdiag; s.ediag = t.ediag;
    s.up = t.up; s.uk = t.uk; s.uv = t.uv; s.vp = t.vp; s.vk = t.vk; s.vv = t.vv;
    s.pij = ctx->pij;
    s.coul = ctx->coul;
    s.fock = (method == FPSG_METHOD_HF && ctx->coul == FPSG_COULOMB_DISTANCE) ? 1 : 0;
    s.has_ext = ctx->ext_null ? 0 : 1;
    s.shift = method == FPSG_METHOD_FTWA ? R(0.5) : R(0);
    s.n_bins = ctx->n_bins; s.amp = ctx->d_amp; s.bin_width = ctx->bin_width; s.t0 = ctx->p_t0; s.td = ctx->p_td;
    s.proj = t.proj;
    return s;
}

template <typename R> DevTables<R>& tables(fpsg_ctx* c);
template <> DevTables<double>& tables<double>(fpsg_ctx* c) { return c->t64; }
template <> DevTables<float>& tables<float>(fpsg_ctx* c) { return c->t32; }

double host_pulse(const fpsg_ctx* c, double t)
{
    if (c->n_bins <= 0) return 0.0;
    long b = (long)std::floor(t / c->bin_width);
    if (b < 0) b = 0;
    if (b > c->n_bins - 1) b = c->n_bins - 1;
    const double x = (t - c->p_t0) / c->p_td;
    return c->amp[b] * std::exp(-0.5 * (x * x));
}

// ------------------------------------------------------------------ resident configs
static int p_index(int P) { return P == 2 ? 0 : P == 4 ? 1 : 2; }

struct ResPlan {
    int idx = -1, G = 0;
    size_t smem = 0;
    bool comp = false;   // FP32 compensated state update (state read and written in FP64)
    bool quad = false;   // k_resident_quad (4-CTA clusters, idx into quad_cfgs), G = 1
    bool hp = false;     // with quad: k_resident_quad_hp (idx into quad_hp_cfgs)
    bool e8 = false;     // with hp: 8-byte column entries (FP32 weights)
    int nh = 2;          // with hp: CTAs per spin (1: 2-CTA clusters)
};

template <typename R>
size_t res_bytes(int n, int M, int P, int cap, bool comp = false)
{
    return res_layout_direct<R>(n, M, P, cap, comp).total;
}

// Picks a resident configuration and the trajectories per CTA: the stacked rows
// (M n) fill whole warps, the elements fit the thread x register budget, the
// shared memory fits, and there are enough CTAs to cover the SMs.
template <typename R>
ResPlan plan_resident(fpsg_ctx* ctx, int B, bool comp = false)
{
    ResPlan best;
    const auto& cf = res_cfgs<R>();
    const int n = ctx->n, ne = ctx->ne;
    const int P = tables<R>(ctx).ell_p;
    double best_score = -1e300;
    if (P == 0) return best;      // a column too wide for the fixed-width stencil
    for (int c = 0; c < (int)cf.size(); ++c) {
        const int per = cf[c].split ? 1 : 2;
        const int cap = cf[c].nt * cf[c].ept;
        int Gmax = cap / (per * ne);
        while (Gmax > 0 && res_bytes<R>(n, per * Gmax, P, cap, comp) > ctx->smem_optin) --Gmax;
        if (Gmax < 1) continue;
        const int ctas_per_group = cf[c].split ? 2 : 1;
        const int want_groups = std::max(1, ctx->sm_count * 2 / ctas_per_group);
        int G = std::max(1, std::min(Gmax, (B + want_groups - 1) / want_groups));
        const int M = per * G;
        const double elem_fill = (double)(M * ne) / cap;                          // thread utilisation
        const double row_fill = (double)(M * n) / (32.0 * ((M * n + 31) / 32));     // lane utilisation
        const double split_pen = cf[c].split ? 0.9 : 1.0;
        const double score = elem_fill * row_fill * split_pen - 0.002 * cf[c].ept;
        if (score > best_score) {
            best_score = score;
            best.idx = c; best.G = G;
            best.smem = res_bytes<R>(n, M, P, cap, comp);
            best.comp = comp;
        }
    }
    return best;
}

// The 4-CTA-cluster kernel for matrices too large for k_resident: the smallest
// elements-per-thread whose half-matrix slots cover both halves and whose shared
// memory (the full matrix once, half the element states) fits.
template <typename R>
ResPlan plan_quad(fpsg_ctx* ctx, bool comp)
{
    ResPlan best;
    const int n = ctx->n, ne = ctx->ne;
    const int Wc = tables<R>(ctx).cell_w;
    if (Wc == 0 || n > 1024) return best;
    const int need = quad_need(ne);
    // the packed, double-buffered matrix (one cluster barrier per stage) where it
    // fits, the first fitting configuration in the table's order of preference: one CTA
    // per spin (2-CTA clusters) where the spin's whole state fits beside the matrix
    // buffers, else two.  With two CTAs per spin FP32 takes it only for columns of at
    // most 5 entries: each entry costs two 4-byte loads and a selection instead of one
    // 8-byte load, which the saved barrier and staging outweigh there (kagome 108:
    // 35.6 -> 28.5 ms per 2048 x 20 steps; 12x12 grid equal) but not for 13 entries
    // (fcc 108: 53.1 -> 57.8 ms)
    if (quad_w_index(Wc) >= 0) {
        const auto& hf = quad_hp_cfgs<R>();
        const bool e8 = !std::is_same<R, double>::value || tables<R>(ctx).cell_f32;
        for (int c = 0; c < (int)hf.size(); ++c) {
            const int nh = hf[c].nh;
            if (nh == 2 && !(std::is_same<R, double>::value || Wc <= 5)) continue;
            const int cap = hf[c].nt * hf[c].ept;
            if (cap < (nh == 2 ? need : ne)) continue;
            const size_t sm = quad_hp_layout<R>(n, Wc, cap, e8).total;
            if (sm > ctx->smem_optin) continue;
            best.idx = c; best.G = 1; best.smem = sm; best.quad = true; best.hp = true; best.e8 = e8;
            best.nh = nh; best.comp = comp;
            return best;
        }
    }
    const auto& cf = quad_cfgs<R>();
    for (int c = 0; c < (int)cf.size(); ++c) {
        const int cap = cf[c].nt * cf[c].ept;
        if (cap < need) continue;
        const size_t sm = quad_layout<R>(n, Wc, cap, comp, cf[c].nt).total;
        if (sm > ctx->smem_optin) continue;
        best.idx = c; best.G = 1; best.smem = sm; best.quad = true; best.comp = comp;
        break;
    }
    return best;
}

// The resident configuration of a run: one CTA (or 2-CTA cluster) per matrix group
// when it fits, else two CTAs per spin; FP32 with the compensated state update when
// its residuals fit too (and the context does not ask for the plain update).
template <typename R>
ResPlan choose_resident(fpsg_ctx* ctx, int B)
{
    const bool comp_ok = !std::is_same<R, double>::value && !(ctx->flags & FPSG_FLAG_FP32_PLAIN_STATE);
    ResPlan plan;
    if (comp_ok) plan = plan_resident<R>(ctx, B, true);
    if (plan.idx < 0) plan = plan_resident<R>(ctx, B);
    if (plan.idx < 0 && comp_ok) plan = plan_quad<R>(ctx, true);
    if (plan.idx < 0) plan = plan_quad<R>(ctx, false);
    return plan;
}

int set_error_from_flag(fpsg_ctx* ctx, unsigned flag)
{
    if (flag & 1u) return fail(ctx, FPSG_ERR_DIVERGED, "a trajectory became non-finite");
    if (flag & (1u << 4)) return fail(ctx, FPSG_ERR_TIMEOUT, "a device-side wait of the dense path gave up");
    return FPSG_OK;
}

// ------------------------------------------------------------------ the runner
struct RunReq {
    int method, precision, path;
    double dt;
    int S, Tp;
    int record;          // 0: advance only
    uint32_t obs;
    double t_start;      // advance only
    int n_steps;         // advance only
};

struct RunOut {
    std::vector<double> sums;    // [Tp][W]
    std::vector<double> whole;   // [Tp][2][ne][2]
    double device_ms = 0.0;
    int64_t launches = 0;
    int path_used = 0;
};

// One resident configuration, ready to launch: the kernel, its block size and
// shared memory, and the persistent grid (cluster pairs in split mode).
template <typename R>
struct ResLauncher {
    ResKernel<R> fn = nullptr;
    int nt = 0, grid = 0;
    bool split = false;
    int cdim = 1;           // CTAs per cluster: 1, 2 (split) or 4 (quad)
    size_t smem = 0;

    int setup(fpsg_ctx* ctx, const ResPlan& plan, int B, bool dump = false)
    {
        if (plan.quad) {
            if (dump) return fail(ctx, FPSG_ERR_UNSUPPORTED, "the 4-CTA resident kernel keeps no stage inputs");
            const QuadCfg<R>& qc = plan.hp ? quad_hp_cfgs<R>()[plan.idx] : quad_cfgs<R>()[plan.idx];
            fn = (plan.hp && plan.e8 ? qc.fn8 : qc.fn)[quad_w_index(tables<R>(ctx).cell_w)];
            nt = qc.nt; split = false; cdim = plan.hp ? 2 * plan.nh : 4; smem = plan.smem;
            CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            cudaLaunchConfig_t lc = config(ctx, cdim * B);
            cudaLaunchAttribute at[1];
            cluster_attr(at, lc);
            int ncl = 0;
            CK(cudaOccupancyMaxActiveClusters(&ncl, (void*)fn, &lc));
            if (ncl < 1) return fail(ctx, FPSG_ERR_UNSUPPORTED, "no cluster fits for the two-CTAs-per-spin resident path");
            grid = cdim * std::min(B, ncl);
            return FPSG_OK;
        }
        const ResCfg<R>& cfg = res_cfgs<R>()[plan.idx];
        fn = dump ? cfg.fn_dump[p_index(tables<R>(ctx).ell_p)] : cfg.fn[p_index(tables<R>(ctx).ell_p)];
        nt = cfg.nt; split = cfg.split; cdim = split ? 2 : 1; smem = plan.smem;
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int ngroups = (B + plan.G - 1) / plan.G;
        if (split) {
            cudaLaunchConfig_t lc = config(ctx, 2 * ngroups);
            cudaLaunchAttribute at[1];
            cluster_attr(at, lc);
            int ncl = 0;
            CK(cudaOccupancyMaxActiveClusters(&ncl, (void*)fn, &lc));
            if (ncl < 1) return fail(ctx, FPSG_ERR_UNSUPPORTED, "no cluster fits for the resident split path");
            grid = 2 * std::min(ngroups, ncl);
        } else {
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, smem));
            if (per_sm < 1) return fail(ctx, FPSG_ERR_UNSUPPORTED, "resident kernel does not fit");
            grid = std::min(ngroups, per_sm * ctx->sm_count);
        }
        return FPSG_OK;
    }
    cudaLaunchConfig_t config(fpsg_ctx* ctx, int g) const
    {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(g); lc.blockDim = dim3(nt); lc.dynamicSmemBytes = smem; lc.stream = ctx->stream;
        return lc;
    }
    void cluster_attr(cudaLaunchAttribute* at, cudaLaunchConfig_t& lc) const
    {
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cdim > 1 ? cdim : 2; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        lc.attrs = at; lc.numAttrs = 1;
    }
    int launch(fpsg_ctx* ctx, const ResArgs<R>& ra) const
    {
        if (cdim > 1) {
            cudaLaunchConfig_t lc = config(ctx, grid);
            cudaLaunchAttribute at[1];
            cluster_attr(at, lc);
            CK(cudaLaunchKernelEx(&lc, fn, ra));
        } else {
            fn<<<grid, nt, smem, ctx->stream>>>(ra);
        }
        CK(cudaGetLastError());
        return FPSG_OK;
    }
};

template <typename R>
int run_impl(fpsg_ctx* ctx, const RunReq& q, RunOut& out)
{
    const int n = ctx->n, ne = ctx->ne, B = ctx->B;
    const int W = rec_width(n);
    const bool hf = q.method == FPSG_METHOD_HF;
    const double h = q.dt / (double)q.S;
    DevSys<R> sys = make_sys<R>(ctx, tables<R>(ctx), q.method);
    const size_t count = (size_t)B * 2 * ne;
    int rc = FPSG_OK;
    std::vector<void*> temps;
    auto tmp = [&](void** p, size_t bytes) -> int {
        int r = talloc(ctx, p, bytes);
        if (!r) temps.push_back(*p);
        return r;
    };
    auto cleanup = [&]() { for (void* p : temps) trelease(ctx, p); };

    const int do_e1 = hf ? (ctx->coul != FPSG_COULOMB_NULL) : 1;
    const int do_e2 = hf ? (ctx->coul == FPSG_COULOMB_DISTANCE) : 1;
    const int rec_e = (q.obs & FPSG_OBS_ENERGIES) ? 1 : 0;
    // HF with a same-spin V: dense complex Delta (Fock term), stream stages only
    const bool fock = hf && ctx->coul == FPSG_COULOMB_DISTANCE;

    int path = q.path;
    ResPlan plan;
    if (fock) {
        if (path == FPSG_PATH_RESIDENT) { cleanup(); return fail(ctx, FPSG_ERR_UNSUPPORTED, "HF with the Fock term runs on the stream path"); }
        path = FPSG_PATH_STREAM;
    }
    if (path == FPSG_PATH_AUTO || path == FPSG_PATH_RESIDENT) {
        plan = choose_resident<R>(ctx, B);
        if (plan.idx < 0) {
            if (path == FPSG_PATH_RESIDENT) { cleanup(); return fail(ctx, FPSG_ERR_UNSUPPORTED, "system too large for the resident path"); }
            path = FPSG_PATH_STREAM;
        } else path = FPSG_PATH_RESIDENT;
    }
    if (path == FPSG_PATH_DENSE) { cleanup(); return fail(ctx, FPSG_ERR_UNSUPPORTED, "dense tensor-core path not available for this precision"); }
    out.path_used = path;

    // state in the run precision (the compensated FP32 resident path reads and
    // writes the FP64 master copy itself)
    cplx<R>* st = nullptr;
    if (std::is_same<R, double>::value) st = (cplx<R>*)ctx->rho64;
    else if (!plan.comp) {
        if ((rc = tmp((void**)&st, sizeof(cplx<R>) * count))) { cleanup(); return rc; }
        k_f64_to_f32<<<std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
            ctx->rho64, (cplx<float>*)st, (long)count);
        out.launches++;
    }
    unsigned* d_err = nullptr;
    if ((rc = tmp((void**)&d_err, sizeof(unsigned)))) { cleanup(); return rc; }
    CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), ctx->stream));

    // total steps and per-step pulse table
    long total_steps;
    int t_first = 0, t_last = q.Tp;
    if (q.record) total_steps = hf ? (long)(q.Tp - 1) * q.S : (long)q.Tp * q.S;
    else total_steps = q.n_steps;
    std::vector<R> ptab_h;
    R* ptab = nullptr;
    if (ctx->n_bins > 0 && total_steps > 0) {
        ptab_h.resize((size_t)total_steps * 4);
        double tc = q.record ? 0.0 : q.t_start;
        for (long s = 0; s < total_steps; ++s) {
            for (int g = 0; g < 4; ++g) ptab_h[(size_t)s * 4 + g] = (R)host_pulse(ctx, stage_time(g, tc, h, q.dt));
            tc += h;
        }
        if ((rc = tmp((void**)&ptab, sizeof(R) * ptab_h.size()))) { cleanup(); return rc; }
        CK(cudaMemcpyAsync(ptab, ptab_h.data(), sizeof(R) * ptab_h.size(), cudaMemcpyHostToDevice, ctx->stream));
    }

    double* sums = nullptr;
    double2* whole = nullptr;
    if (q.record) {
        if ((rc = tmp((void**)&sums, sizeof(double) * (size_t)q.Tp * W))) { cleanup(); return rc; }
        CK(cudaMemsetAsync(sums, 0, sizeof(double) * (size_t)q.Tp * W, ctx->stream));
        if (q.obs & FPSG_OBS_WHOLE) {
            if ((rc = tmp((void**)&whole, sizeof(double2) * (size_t)q.Tp * 2 * ne))) { cleanup(); return rc; }
            CK(cudaMemsetAsync(whole, 0, sizeof(double2) * (size_t)q.Tp * 2 * ne, ctx->stream));
        }
    }


    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (path == FPSG_PATH_RESIDENT) {
        ResLauncher<R> rl;
        if ((rc = rl.setup(ctx, plan, B))) { cleanup(); return rc; }
        const int grid = rl.grid;
        double* slots = nullptr;
        if (q.record) {
            const size_t sb = sizeof(double) * (size_t)grid * q.Tp * W;
            if ((rc = tmp((void**)&slots, sb))) { cleanup(); return rc; }
            CK(cudaMemsetAsync(slots, 0, sb, ctx->stream));
        }
        ResArgs<R> ra;
        ra.sys = sys; ra.state = st; ra.B = B; ra.G = plan.G; ra.h = (R)h; ra.ptab = ptab;
        ra.S = q.S; ra.Tp = q.record ? q.Tp : 1 << 30; ra.hf = hf ? 1 : 0;
        ra.record = q.record; ra.do_en = rec_e; ra.do_e1 = do_e1 && rec_e; ra.do_e2 = do_e2 && rec_e;
        ra.ell_k = plan.quad ? tables<R>(ctx).cell_k : tables<R>(ctx).ell_k;
        ra.ell_v = plan.quad ? tables<R>(ctx).cell_v : tables<R>(ctx).ell_v;
        ra.ell_pad = tables<R>(ctx).ell_pad;
        ra.slots = slots; ra.whole = whole; ra.err = d_err;
        ra.dump = nullptr; ra.dump_count = 0;
        ra.udiag = tables<R>(ctx).dd_fusable ? tables<R>(ctx).udiag : nullptr;
        ra.order = ctx->res_order;
        ra.state64 = plan.comp ? ctx->rho64 : nullptr;
        // chunk the time axis so one launch stays in the tens of milliseconds
        const long per_launch_steps = std::max<long>(1, 4096L * 1024 / std::max<long>(1, (long)B));
        if (q.record) {
            const int chunk = (int)std::max<long>(1, std::min<long>(q.Tp, per_launch_steps / q.S + 1));
            long step_base = 0;
            for (int t0 = t_first; t0 < t_last; t0 += chunk) {
                const int t1 = std::min(t_last, t0 + chunk);
                ra.t_begin = t0; ra.t_end = t1; ra.step_base = step_base;
                ra.ptab = ptab ? ptab + step_base * 4 : nullptr;
                ra.step_base = 0;
                if ((rc = rl.launch(ctx, ra))) { cleanup(); return rc; }
                out.launches++;
                for (int t = t0; t < t1; ++t) step_base += (hf && t == q.Tp - 1) ? 0 : q.S;
            }
            const long TW = (long)q.Tp * W;
            k_slot_reduce<<<std::max(1, std::min<int>((int)((TW + 255) / 256), ctx->sm_count * 4)), 256, 0, ctx->stream>>>(slots, grid, TW, sums);
            CK(cudaGetLastError());
            out.launches++;
        } else {
            long done = 0;
            while (done < q.n_steps) {
                const long m = std::min<long>(q.n_steps - done, per_launch_steps);
                ra.t_begin = 0; ra.t_end = (int)m; ra.S = 1; ra.step_base = 0;
                ra.ptab = ptab ? ptab + done * 4 : nullptr;
                if ((rc = rl.launch(ctx, ra))) { cleanup(); return rc; }
                out.launches++;
                done += m;
            }
        }
    } else {
        // ---------------- stream path: one launch per RK stage
        cplx<R> *A = nullptr, *Bc = nullptr, *X0 = nullptr, *X1 = nullptr;
        if ((rc = tmp((void**)&A, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&Bc, sizeof(cplx<R>) * count)) ||
            (rc = tmp((void**)&X0, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&X1, sizeof(cplx<R>) * count))) {
            cleanup(); return rc;
        }
        double *diagbuf = nullptr, *ebuf = nullptr, *part = nullptr;
        const int chunk = 64;
        const int nch = (B + chunk - 1) / chunk;
        if (q.record) {
            if ((rc = tmp((void**)&diagbuf, sizeof(double) * (size_t)B * 2 * n)) ||
                (rc = tmp((void**)&ebuf, sizeof(double) * (size_t)B * 2 * 4)) ||
                (rc = tmp((void**)&part, sizeof(double) * (size_t)nch * W))) {
                cleanup(); return rc;
            }
        }
        // stage the matrix in shared memory when it fits, else read it from global memory
        size_t smem = ((sizeof(cplx<R>) * ne + sizeof(R) * n + 15) & ~size_t(15)) + sizeof(double) * 32 * 4;
        const bool gx = smem > ctx->smem_optin;
        if (gx) smem = ((sizeof(R) * n + 15) & ~size_t(15)) + sizeof(double) * 32 * 4;
        auto stage_fn = gx ? k_stream_stage<R, true> : k_stream_stage<R, false>;
        CK(cudaFuncSetAttribute(stage_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_fn, 256, smem));
        const int grid = std::max(1, std::min(2 * B, std::max(1, per_sm) * ctx->sm_count));
        StreamArgs<R> sa;
        sa.sys = sys; sa.rho = st; sa.A = A; sa.Bc = Bc; sa.B = B; sa.h = (R)h;
        sa.do_e1 = do_e1 && rec_e; sa.do_e2 = do_e2 && rec_e;
        sa.diagbuf = diagbuf; sa.ebuf = ebuf; sa.err = d_err;
        FockArgs<R> fa;
        if (fock) {
            const size_t nn = (size_t)n * n;
            std::vector<R> tm(nn), uu(nn), vv(nn), ee(nn, R(0));
            for (size_t x = 0; x < nn; ++x) {
                tm[x] = (R)ctx->tM[x]; uu[x] = (R)ctx->U[x]; vv[x] = (R)ctx->V[x];
                if (!ctx->ext_null) ee[x] = (R)ctx->ext[x];
            }
            R *dt_ = nullptr, *du_ = nullptr, *dv_ = nullptr, *de_ = nullptr;
            cplx<R>* dd_ = nullptr;
            if ((rc = tmp((void**)&dt_, sizeof(R) * nn)) || (rc = tmp((void**)&du_, sizeof(R) * nn)) ||
                (rc = tmp((void**)&dv_, sizeof(R) * nn)) || (rc = tmp((void**)&de_, sizeof(R) * nn)) ||
                (rc = tmp((void**)&dd_, sizeof(cplx<R>) * nn * 2 * B))) {
                cleanup(); return rc;
            }
            CK(cudaMemcpyAsync(dt_, tm.data(), sizeof(R) * nn, cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(du_, uu.data(), sizeof(R) * nn, cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(dv_, vv.data(), sizeof(R) * nn, cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(de_, ee.data(), sizeof(R) * nn, cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            fa.tMf = dt_; fa.Uf = du_; fa.Vf = dv_; fa.extf = de_; fa.D = dd_;
        }
        const int fgrid = std::max(1, std::min(2 * B, 4 * ctx->sm_count));
        long gstep = 0;
        auto do_step = [&](bool record_now, double2* wslot) -> int {
            const cplx<R>* xc[4] = { st, X0, X1, X0 };
            cplx<R>* xn[4] = { X0, X1, X0, nullptr };
            for (int g = 0; g < 4; ++g) {
                sa.stage = g; sa.Xc = xc[g]; sa.Xn = xn[g];
                sa.pulse = ptab ? (R)ptab_h[(size_t)gstep * 4 + g] : R(0);
                sa.record = (g == 0 && record_now) ? 1 : 0;
                sa.whole = sa.record ? wslot : nullptr;
                if (fock) {
                    fa.s = sa;
                    k_fock_stage<R><<<fgrid, 256, 0, ctx->stream>>>(fa);
                } else {
                    stage_fn<<<grid, 256, smem, ctx->stream>>>(sa);
                }
                CK(cudaGetLastError());
                out.launches++;
            }
            ++gstep;
            return FPSG_OK;
        };
        auto reduce_snapshot = [&](int t) -> int {
            k_reduce_part<<<nch, 256, 0, ctx->stream>>>(diagbuf, ebuf, B, n, chunk, part);
            k_reduce_fin<<<std::max(1, (W + 255) / 256), 256, 0, ctx->stream>>>(part, nch, W, sums + (size_t)t * W);
            CK(cudaGetLastError());
            out.launches += 2;
            return FPSG_OK;
        };
        if (q.record) {
            for (int t = 0; t < q.Tp; ++t) {
                double2* wslot = whole ? whole + (size_t)t * 2 * ne : nullptr;
                const int nsteps = (hf && t == q.Tp - 1) ? 0 : q.S;
                if (nsteps == 0) {
                    sa.Xc = st; sa.record = 1; sa.whole = wslot;
                    k_stream_record<R><<<grid, 256, 0, ctx->stream>>>(sa);
                    CK(cudaGetLastError());
                    out.launches++;
                }
                for (int s = 0; s < nsteps; ++s)
                    if ((rc = do_step(s == 0, wslot))) { cleanup(); return rc; }
                if ((rc = reduce_snapshot(t))) { cleanup(); return rc; }
            }
        } else {
            for (long s = 0; s < q.n_steps; ++s)
                if ((rc = do_step(false, nullptr))) { cleanup(); return rc; }
        }
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));

    if (!std::is_same<R, double>::value && !plan.comp) {
        k_f32_to_f64<<<std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
            (const cplx<float>*)st, ctx->rho64, (long)count);
        out.launches++;
    }
    unsigned flag = 0;
    CK(cudaMemcpyAsync(&flag, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    if (q.record) {
        out.sums.resize((size_t)q.Tp * W);
        CK(cudaMemcpyAsync(out.sums.data(), sums, sizeof(double) * out.sums.size(), cudaMemcpyDeviceToHost, ctx->stream));
        if (whole) {
            out.whole.resize((size_t)q.Tp * 2 * ne * 2);
            CK(cudaMemcpyAsync(out.whole.data(), whole, sizeof(double) * out.whole.size(), cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    out.device_ms = ms;
    cleanup();
    return set_error_from_flag(ctx, flag);
}


// ------------------------------------------------------------------ dense path
// The tensor-core path (fpsg_dense.cu) for the split precisions: full FP32
// matrices, one launch per RK stage.  The 3/8 rule in terms of stored stage
// inputs (X1 = rho):
//     X2 = X1 + h/3 k1,  X3 = 2 rho - X2 + h k2,  X4 = 2 X2 - X3 + h k3,
//     rho' = -rho/8 + 3/4 X3 + 3/8 X4 + h/8 k4,
// the same polynomial as src/FHfTWASolver.cpp:629-661 with the k's eliminated.
int dense_impl(fpsg_ctx* ctx, const RunReq& q, RunOut& out)
{
    using namespace fpsg::dense;
    const int n = ctx->n, ne = ctx->ne, B = ctx->B, M = 2 * B, W = rec_width(n);
    const bool hf = q.method == FPSG_METHOD_HF;
    const double h = q.dt / (double)q.S;
    if (n > NP) return fail(ctx, FPSG_ERR_UNSUPPORTED, "the dense path handles n <= 256");
    if (ctx->smem_optin < stage_smem_bytes()) return fail(ctx, FPSG_ERR_UNSUPPORTED, "not enough shared memory for the dense path");
    DevSys<float> sys = make_sys<float>(ctx, tables<float>(ctx), q.method);
    std::vector<void*> temps;
    int rc = FPSG_OK;
    auto tmp = [&](void** p, size_t bytes) -> int {
        int r = talloc(ctx, p, bytes);
        if (!r) temps.push_back(*p);
        return r;
    };
    auto cleanup = [&]() { for (void* p : temps) trelease(ctx, p); };
    const size_t mat = (size_t)M * 2 * NP * NP;
    float *R = nullptr, *Xa = nullptr, *Xb = nullptr, *Xc = nullptr, *Tf = nullptr, *Ud = nullptr, *Vd = nullptr;
    void* Tc = nullptr;
    const bool tf32 = q.precision == FPSG_PREC_SPLIT_TF32X3;
    unsigned* d_err = nullptr;
    if ((rc = tmp((void**)&R, sizeof(float) * mat)) || (rc = tmp((void**)&Xa, sizeof(float) * mat)) ||
        (rc = tmp((void**)&Xb, sizeof(float) * mat)) || (rc = tmp((void**)&Xc, sizeof(float) * mat)) ||
        (rc = tmp((void**)&Tf, sizeof(float) * NP * NP)) ||
        (rc = tmp(&Tc, TC_BYTES)) ||
        (rc = tmp((void**)&d_err, sizeof(unsigned)))) {
        cleanup();
        return rc;
    }
    CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), ctx->stream));
    {
        // the shared operand is Delta off its diagonal: tM plus the static potential's
        // off-diagonal part (src/FHfTWASolver.cpp:586-596 adds the whole extPot to Delta),
        // row-major; both are real symmetric.  prep_T zeroes the diagonal, which the
        // epilogue adds per matrix (tM_jj + Hartree + extPot_jj + pulse).
        std::vector<float> th((size_t)NP * NP, 0.f);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v = ctx->tM[(size_t)j * n + i];
                if (!ctx->ext_null) v += ctx->ext[(size_t)j * n + i];
                th[(size_t)i * NP + j] = (float)v;
            }
        CK(cudaMemcpyAsync(Tf, th.data(), sizeof(float) * th.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(prep_T(Tf, Tc, tf32, ctx->stream));
        if (ctx->coul == FPSG_COULOMB_DISTANCE) {
            // dense Hartree rows for long-range Coulomb (coalesced in the kernel)
            std::vector<float> uh((size_t)NP * NP, 0.f), vh((size_t)NP * NP, 0.f);
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    uh[(size_t)i * NP + j] = (float)ctx->U[(size_t)j * n + i];
                    vh[(size_t)i * NP + j] = (float)ctx->V[(size_t)j * n + i];
                }
            if ((rc = tmp((void**)&Ud, sizeof(float) * uh.size())) || (rc = tmp((void**)&Vd, sizeof(float) * vh.size()))) {
                cleanup();
                return rc;
            }
            CK(cudaMemcpyAsync(Ud, uh.data(), sizeof(float) * uh.size(), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(Vd, vh.data(), sizeof(float) * vh.size(), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        CK(unpack(ctx->rho64, n, M, R, ctx->stream));
        CK(configure());
        out.launches += 2;
    }
    double *sums = nullptr, *diagbuf = nullptr, *ebuf = nullptr, *part = nullptr;
    double2* whole = nullptr;
    cplx<float>* packed = nullptr;
    const int chunk = 64, nch = (B + chunk - 1) / chunk;
    const int do_e1 = hf ? (ctx->coul != FPSG_COULOMB_NULL) : 1;
    const int rec_e = (q.obs & FPSG_OBS_ENERGIES) ? 1 : 0;
    if (q.record) {
        if ((rc = tmp((void**)&sums, sizeof(double) * (size_t)q.Tp * W)) ||
            (rc = tmp((void**)&diagbuf, sizeof(double) * (size_t)B * 2 * n)) ||
            (rc = tmp((void**)&ebuf, sizeof(double) * (size_t)B * 2 * 4)) ||
            (rc = tmp((void**)&part, sizeof(double) * (size_t)nch * W)) ||
            (rc = tmp((void**)&packed, sizeof(cplx<float>) * (size_t)M * ne))) {
            cleanup();
            return rc;
        }
        CK(cudaMemsetAsync(ebuf, 0, sizeof(double) * (size_t)B * 2 * 4, ctx->stream));
        if (q.obs & FPSG_OBS_WHOLE) {
            if ((rc = tmp((void**)&whole, sizeof(double2) * (size_t)q.Tp * 2 * ne))) { cleanup(); return rc; }
            CK(cudaMemsetAsync(whole, 0, sizeof(double2) * (size_t)q.Tp * 2 * ne, ctx->stream));
        }
    }
    StreamArgs<float> sa;
    sa.sys = sys; sa.rho = packed; sa.A = nullptr; sa.Bc = nullptr; sa.B = B; sa.h = (float)h;
    sa.do_e1 = do_e1 && rec_e; sa.do_e2 = (hf ? 0 : 1) && rec_e;
    sa.diagbuf = diagbuf; sa.ebuf = ebuf; sa.err = d_err; sa.stage = 0; sa.Xn = nullptr; sa.pulse = 0.f;
    const int rgrid = std::max(1, std::min(2 * B, 4 * ctx->sm_count));
    const int grid = std::max(1, std::min(M, ctx->sm_count));

    DenseArgs da;
    da.n = n; da.M = M; da.Tc = Tc; da.sys = sys; da.err = d_err; da.Ud = Ud; da.Vd = Vd;
    // test hook: the call's first launch waits on a barrier nothing arrives at
    da.probe_polls = (ctx->flags & FPSG_FLAG_TEST_EXPIRE_WAIT) ? 4096u : 0u;
    double tc = q.record ? 0.0 : q.t_start;
    auto step = [&]() -> int {
        const float hf32 = (float)h;
        for (int g = 0; g < 4; ++g) {
            da.pulse = ctx->n_bins > 0 ? (float)host_pulse(ctx, stage_time(g, tc, h, q.dt)) : 0.f;
            switch (g) {
            case 0: da.X = R;  da.P0 = nullptr; da.P1 = nullptr; da.a0 = 0.f;  da.a1 = 0.f;   da.ax = 1.f;    da.hk = hf32 / 3.f; da.out = Xa; break;
            case 1: da.X = Xa; da.P0 = R;       da.P1 = nullptr; da.a0 = 2.f;  da.a1 = 0.f;   da.ax = -1.f;   da.hk = hf32;       da.out = Xb; break;
            case 2: da.X = Xb; da.P0 = Xa;      da.P1 = nullptr; da.a0 = 2.f;  da.a1 = 0.f;   da.ax = -1.f;   da.hk = hf32;       da.out = Xc; break;
            default: da.X = Xc; da.P0 = R;      da.P1 = Xb;      da.a0 = -0.125f; da.a1 = 0.75f; da.ax = 0.375f; da.hk = hf32 / 8.f; da.out = R; break;
            }
            CK(launch_stage(da, grid, tf32, ctx->stream));
            da.probe_polls = 0;
            out.launches++;
        }
        tc += h;
        return FPSG_OK;
    };
    auto record = [&](int t) -> int {
        CK(pack_f32(R, n, M, packed, ctx->stream));
        sa.Xc = packed; sa.record = 1;
        sa.whole = whole ? whole + (size_t)t * 2 * ne : nullptr;
        k_stream_record<float><<<rgrid, 256, 0, ctx->stream>>>(sa);
        k_reduce_part<<<nch, 256, 0, ctx->stream>>>(diagbuf, ebuf, B, n, chunk, part);
        k_reduce_fin<<<std::max(1, (W + 255) / 256), 256, 0, ctx->stream>>>(part, nch, W, sums + (size_t)t * W);
        CK(cudaGetLastError());
        out.launches += 4;
        return FPSG_OK;
    };
    out.path_used = FPSG_PATH_DENSE;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (q.record) {
        for (int t = 0; t < q.Tp; ++t) {
            if ((rc = record(t))) { cleanup(); return rc; }
            const int nsteps = (hf && t == q.Tp - 1) ? 0 : q.S;
            for (int s = 0; s < nsteps; ++s)
                if ((rc = step())) { cleanup(); return rc; }
        }
    } else {
        for (long s = 0; s < q.n_steps; ++s)
            if ((rc = step())) { cleanup(); return rc; }
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(pack_f64(R, n, M, ctx->rho64, ctx->stream));
    out.launches++;
    unsigned flag = 0;
    CK(cudaMemcpyAsync(&flag, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    if (q.record) {
        out.sums.resize((size_t)q.Tp * W);
        CK(cudaMemcpyAsync(out.sums.data(), sums, sizeof(double) * out.sums.size(), cudaMemcpyDeviceToHost, ctx->stream));
        if (whole) {
            out.whole.resize((size_t)q.Tp * 2 * ne * 2);
            CK(cudaMemcpyAsync(out.whole.data(), whole, sizeof(double) * out.whole.size(), cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    out.device_ms = ms;
    cleanup();
    return set_error_from_flag(ctx, flag);
}

// ------------------------------------------------------------------ adjoint
template <typename R>
using ResKernelVjp = void (*)(VjpSegArgs<R>);

template <typename R>
int grad_impl(fpsg_ctx* ctx, double dt, int S, int Tp, int C, double* loss_out, double* gU, double* gT,
              double* gP, double* dev_ms, double* fwd_ms)
{
    C = S * ((C + S - 1) / S);   // checkpoint segments hold whole snapshots
    const int n = ctx->n, ne = ctx->ne, Ball = ctx->B, W = rec_width(n), nb = ctx->n_bins;
    const long Nsteps = (long)(Tp - 1) * S;
    const double h = dt / (double)S;
    DevSys<R> sys = make_sys<R>(ctx, tables<R>(ctx), FPSG_METHOD_FTWA);
    std::vector<void*> temps;
    std::vector<cudaEvent_t> evs;   // per chunk: start, end of its forward sweep
    int rc = FPSG_OK;
    auto tmp = [&](void** p, size_t bytes) -> int {
        int r = talloc(ctx, p, bytes);
        if (!r) temps.push_back(*p);
        return r;
    };
    cplx<R>* keep = nullptr;     // stage inputs of the last segments, written by the forward sweep
    auto cleanup = [&]() {
        for (void* p : temps) trelease(ctx, p);
        trelease(ctx, keep);
        keep = nullptr;
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
        evs.clear();
    };
    const int nck = (int)(Nsteps / C) + 1;
    const long nseg = Nsteps > 0 ? (Nsteps - 1) / C + 1 : 0;   // checkpoint segments
    const int PW = 2 + nb;

    // ---- trajectory chunks.  A segment whose stage inputs the forward sweep keeps
    // needs no recompute in the reverse sweep (one forward pass over the segment
    // saved).  When the stage inputs of every segment of the whole ensemble do not fit
    // the memory the kept segments may take, the trajectories run in chunks, each a
    // full forward and reverse sweep of its own, sized so that every segment of a
    // chunk is kept.  A chunk holds a multiple of one trajectory per SM (the
    // concurrency of the resident forward and reverse kernels; a smaller chunk would
    // leave clusters idle, which costs more than a recompute).  Trajectories are
    // independent: the per-trajectory parameter partials, and so the gradients, do not
    // depend on the chunking, and the loss sums change only in rounding.
    ResPlan plan = plan_resident<R>(ctx, Ball);
    int B = Ball;                  // trajectories per chunk (the last one may hold fewer)
    if (plan.idx >= 0 && Nsteps > 0 && ctx->grad_keep != 0 && Ball >= 2 * ctx->sm_count) {
        const size_t traj = sizeof(cplx<R>) * 2 * (size_t)ne;
        const size_t per_keep = traj * 4 * (size_t)C * (size_t)nseg;          // every segment kept
        const size_t per_tmp = traj * (size_t)(10 + nck + 4 * C);              // the chunk's scratch
        size_t fre = 0, tot = 0, pooled = 0;
        if (cudaMemGetInfo(&fre, &tot) != cudaSuccess) { cudaGetLastError(); fre = 0; }
        for (const auto& a : ctx->pool) pooled += a.bytes;
        size_t avail = fre + pooled;       // pooled scratch is reused or released
        if (ctx->mem_cap) {
            const size_t held = ctx->mem_used > pooled ? ctx->mem_used - pooled : 0;
            avail = std::min<size_t>(avail, ctx->mem_cap > held ? ctx->mem_cap - held : 0);
        }
        const size_t budget = avail / 4 * 3;
        long nchunk = 1;
        const size_t need = (size_t)Ball * (per_keep + per_tmp);
        if (budget > 0 && need > budget) nchunk = (long)((need + budget - 1) / budget);
        if (ctx->grad_keep > 0)
            nchunk = std::max<long>(nchunk, (long)(((size_t)Ball * per_keep + (size_t)ctx->grad_keep - 1) / (size_t)ctx->grad_keep));
        nchunk = std::min<long>(nchunk, Ball / ctx->sm_count);
        if (nchunk > 1) {
            const int q = ctx->sm_count;
            B = (int)((Ball + nchunk - 1) / nchunk);
            B = ((B + q - 1) / q) * q;
            if (B >= Ball) B = Ball;
            else plan = plan_resident<R>(ctx, B);
        }
    }
    const size_t count = (size_t)B * 2 * ne;
    int n_keep = 0;                                            // segments kept from the sweep
    cplx<R> *st, *A, *Bc, *X0, *X1, *ck, *seg, *lam, *xb;
    R* dbar;
    double *pacc, *diagbuf, *ebuf, *part, *sums, *pout;
    unsigned* d_err;
    const int chunk = 64, nch = (B + chunk - 1) / chunk;
    if ((rc = tmp((void**)&st, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&A, sizeof(cplx<R>) * count)) ||
        (rc = tmp((void**)&Bc, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&X0, sizeof(cplx<R>) * count)) ||
        (rc = tmp((void**)&X1, sizeof(cplx<R>) * count)) ||
        (rc = tmp((void**)&ck, sizeof(cplx<R>) * count * nck)) ||
        (rc = tmp((void**)&seg, sizeof(cplx<R>) * count * 4 * C)) ||
        (rc = tmp((void**)&lam, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&xb, sizeof(cplx<R>) * count * 4)) ||
        (rc = tmp((void**)&dbar, sizeof(R) * (size_t)B * 2 * n)) ||
        (rc = tmp((void**)&pacc, sizeof(double) * (size_t)Ball * 2 * PW)) ||
        (rc = tmp((void**)&diagbuf, sizeof(double) * (size_t)B * 2 * n)) ||
        (rc = tmp((void**)&ebuf, sizeof(double) * (size_t)B * 2 * 4)) ||
        (rc = tmp((void**)&part, sizeof(double) * (size_t)nch * W)) ||
        (rc = tmp((void**)&sums, sizeof(double) * (size_t)Tp * W)) || (rc = tmp((void**)&pout, sizeof(double) * PW)) ||
        (rc = tmp((void**)&d_err, sizeof(unsigned)))) {
        cleanup();
        return rc;
    }
    const int cgrid = std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8));
    CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(pacc, 0, sizeof(double) * (size_t)Ball * 2 * PW, ctx->stream));
    CK(cudaMemsetAsync(ebuf, 0, sizeof(double) * (size_t)B * 2 * 4, ctx->stream));

    // time grid: t_n accumulated as the oracle does; pulse value, envelope and bin per stage
    std::vector<double> tn(Nsteps + 1, 0.0);
    for (long q = 1; q <= Nsteps; ++q) tn[q] = tn[q - 1] + h;
    auto stage_info = [&](long step, int g, R& pv, double& env, int& bin) {
        pv = R(0); env = 0.0; bin = -1;
        if (nb <= 0) return;
        const double t = stage_time(g, tn[step], h, dt);
        long b = (long)std::floor(t / ctx->bin_width);
        if (b < 0) b = 0;
        if (b > nb - 1) b = nb - 1;
        const double x = (t - ctx->p_t0) / ctx->p_td;
        env = std::exp(-0.5 * (x * x));
        bin = (int)b;
        pv = (R)(ctx->amp[b] * env);
    };

    const size_t smem = ((sizeof(cplx<R>) * ne + sizeof(R) * n + 15) & ~size_t(15)) + sizeof(double) * 32 * 4;
    const size_t vsmem = ((2 * sizeof(cplx<R>) * ne + 2 * sizeof(R) * n + 15) & ~size_t(15)) + sizeof(double) * 32 * 3;
    if (smem > ctx->smem_optin || vsmem > ctx->smem_optin) { cleanup(); return fail(ctx, FPSG_ERR_UNSUPPORTED, "system too large for the adjoint kernels"); }
    CK(cudaFuncSetAttribute(k_stream_stage<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaFuncSetAttribute(k_vjp_stage<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsmem));
    int per_sm = 0, vper_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stream_stage<R>, 256, smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&vper_sm, k_vjp_stage<R>, 256, vsmem));
    const int grid = std::max(1, std::min(2 * B, std::max(1, per_sm) * ctx->sm_count));
    const int vgrid = std::max(1, std::min(2 * B, std::max(1, vper_sm) * ctx->sm_count));
    StreamArgs<R> sa;
    sa.sys = sys; sa.A = A; sa.Bc = Bc; sa.B = B; sa.h = (R)h;
    sa.do_e1 = 0; sa.do_e2 = 0; sa.diagbuf = diagbuf; sa.ebuf = ebuf; sa.whole = nullptr; sa.err = d_err;
    auto fwd_step = [&](cplx<R>* rho, long step, cplx<R>* const xin[4], bool record) -> int {
        // xin[0] = stage 1 input (rho), xin[1..3] = where the stage 2..4 inputs go
        sa.rho = rho;
        for (int g = 0; g < 4; ++g) {
            R pv; double env; int bin;
            stage_info(step, g, pv, env, bin);
            sa.stage = g;
            sa.Xc = xin[g];
            sa.Xn = g < 3 ? xin[g + 1] : nullptr;
            sa.pulse = pv;
            sa.record = (g == 0 && record) ? 1 : 0;
            k_stream_stage<R><<<grid, 256, smem, ctx->stream>>>(sa);
        }
        return cudaGetLastError() == cudaSuccess ? FPSG_OK : fail(ctx, FPSG_ERR_CUDA, "adjoint forward stage launch failed");
    };
    auto reduce_snapshot = [&](int t) {
        k_reduce_part<<<nch, 256, 0, ctx->stream>>>(diagbuf, ebuf, B, n, chunk, part);
        k_reduce_fin<<<std::max(1, (W + 255) / 256), 256, 0, ctx->stream>>>(part, nch, W, sums + (size_t)t * W);
    };

    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    // ---- set-up of the forward sweep.  The resident kernel runs one launch per
    // checkpoint segment (C is a multiple of S, so segments hold whole snapshots);
    // the last snapshot takes no steps.  Without a resident configuration the stream
    // stages do the same (in one chunk).
    ResLauncher<R> rl, rld;   // forward sweep; segment recompute (writes the stage inputs)
    R* ptab = nullptr;
    double* slots = nullptr;
    ResArgs<R> ra;
    if (plan.idx >= 0) {
        if ((rc = rl.setup(ctx, plan, B)) || (rc = rld.setup(ctx, plan, B, true))) { cleanup(); return rc; }
        if (nb > 0 && Nsteps > 0) {
            std::vector<R> ph((size_t)Nsteps * 4);
            for (long q = 0; q < Nsteps; ++q)
                for (int g = 0; g < 4; ++g) { R pv; double env; int bin; stage_info(q, g, pv, env, bin); ph[(size_t)q * 4 + g] = pv; }
            if ((rc = tmp((void**)&ptab, sizeof(R) * ph.size()))) { cleanup(); return rc; }
            CK(cudaMemcpyAsync(ptab, ph.data(), sizeof(R) * ph.size(), cudaMemcpyHostToDevice, ctx->stream));
        }
        // the snapshot records of every chunk accumulate in the same per-CTA slots
        const size_t sb = sizeof(double) * (size_t)rl.grid * Tp * W;
        if ((rc = tmp((void**)&slots, sb))) { cleanup(); return rc; }
        CK(cudaMemsetAsync(slots, 0, sb, ctx->stream));
        ra.sys = sys; ra.state = st; ra.B = B; ra.G = plan.G; ra.h = (R)h;
        ra.S = S; ra.Tp = Tp; ra.hf = 1; ra.record = 1; ra.do_en = 0; ra.do_e1 = 0; ra.do_e2 = 0;
        ra.ell_k = tables<R>(ctx).ell_k; ra.ell_v = tables<R>(ctx).ell_v; ra.ell_pad = tables<R>(ctx).ell_pad;
        ra.slots = slots; ra.whole = nullptr; ra.err = d_err; ra.step_base = 0;
        ra.dump = nullptr; ra.dump_count = 0;
        ra.udiag = tables<R>(ctx).dd_fusable ? tables<R>(ctx).udiag : nullptr;
        ra.order = ctx->res_order;
        // The last n_keep segments of a chunk keep their stage inputs from its sweep
        // (the recompute variant of the kernel, records on), so the backward pass needs
        // no recompute for them: in whole segments, up to three quarters of the free
        // device memory and of what the memory cap leaves, and within the budget of
        // fpsg_set_grad_memory.  One buffer serves every chunk.
        // The buffer goes back to the context's pool; a later call takes the largest
        // pooled block when it holds at least as many segments as a new buffer could,
        // since memory written before is much faster to fill than a fresh allocation
        // of tens of GB.
        if (Nsteps > 0 && ctx->grad_keep != 0) {
            const size_t segbytes = sizeof(cplx<R>) * count * 4 * (size_t)C;
            const long want = ctx->grad_keep > 0 ? std::min<long>(nseg, (long)((size_t)ctx->grad_keep / segbytes)) : nseg;
            int bi = -1;
            for (int i = 0; i < (int)ctx->pool.size(); ++i)
                if (ctx->pool[i].bytes >= segbytes && (bi < 0 || ctx->pool[i].bytes > ctx->pool[bi].bytes)) bi = i;
            auto fresh_segments = [&]() -> long {   // segments a new buffer could hold
                if (want <= 0) return 0;
                size_t fre = 0, tot = 0;
                if (cudaMemGetInfo(&fre, &tot) != cudaSuccess) { cudaGetLastError(); fre = 0; }
                size_t budget = fre / 4 * 3;
                if (ctx->mem_cap)
                    budget = std::min<size_t>(budget, ctx->mem_cap > ctx->mem_used ? (ctx->mem_cap - ctx->mem_used) / 4 * 3 : 0);
                return std::min<long>(want, (long)(budget / segbytes));
            };
            long fresh = fresh_segments();
            const long pooled = bi >= 0 ? std::min<long>(want, (long)(ctx->pool[bi].bytes / segbytes)) : 0;
            if (pooled > 0 && pooled >= fresh) {
                keep = (cplx<R>*)ctx->pool[bi].p;
                n_keep = (int)pooled;
                ctx->pool.erase(ctx->pool.begin() + bi);
            } else if (fresh > 0) {
                if (bi >= 0) {
                    // the pooled block holds fewer segments than a new buffer: release it
                    // first, so that it neither stays allocated beside the new buffer nor
                    // is left out of the memory the new buffer may take
                    void* old = ctx->pool[bi].p;
                    ctx->pool.erase(ctx->pool.begin() + bi);
                    dfree(ctx, old);
                    fresh = fresh_segments();
                }
                n_keep = (int)fresh;
                if (n_keep > 0 && talloc(ctx, (void**)&keep, segbytes * (size_t)n_keep) != FPSG_OK) {
                    keep = nullptr;
                    n_keep = 0;
                    ctx->err.clear();
                }
            }
        }
    }

    // ---- set-up of the backward pass
    auto wt = [&](int t) { return (t == 0 || t == Tp - 1) ? 0.5 * dt : dt; };
    const double lscale = 1.0 / ((double)n * (double)Ball);
    cplx<R>* xbs[4] = {xb, xb + count, xb + 2 * count, xb + 3 * count};
    // the direct-form VJP kernel when Delta's columns have a fixed width and it fits
    const int ellP = tables<R>(ctx).ell_p;
    const size_t esmem = ellP ? vjp_ell_smem<R>(n, ne, ellP) : 0;
    const bool use_ell = ellP != 0 && esmem <= ctx->smem_optin;
    auto ell_fn = ellP == 2 ? k_vjp_stage_ell<R, 2> : ellP == 4 ? k_vjp_stage_ell<R, 4> : k_vjp_stage_ell<R, 8>;
    int egrid = 1;
    if (use_ell) {
        CK(cudaFuncSetAttribute(ell_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ell_fn, 256, esmem));
        egrid = std::max(1, std::min(2 * B, std::max(1, per_sm) * ctx->sm_count));
    }
    const R hR = (R)h;
    // the segment-resident reverse kernel: on-site (or no) Coulomb term, fixed-width
    // columns with P <= 4, the packed matrix within 512 x 5 slots
    constexpr int SEG_NT = 512, SEG_EPT = 5;
    const bool use_seg = plan.idx >= 0 && tables<R>(ctx).dd_fusable && (ellP == 2 || ellP == 4) &&
                         ne <= SEG_NT * SEG_EPT &&
                         (ellP == 2 ? vjp_seg_smem<R, 2>(n, ne, nb) : vjp_seg_smem<R, 4>(n, ne, nb)) <= ctx->smem_optin;
    auto seg_fn = ellP == 2 ? k_vjp_segment<R, SEG_NT, SEG_EPT, 2> : k_vjp_segment<R, SEG_NT, SEG_EPT, 4>;
    VjpSegArgs<R> vs;
    int seg_grid = 0;
    size_t seg_smem = 0;
    if (use_seg) {
        // two variants: stage adjoints in registers (one cluster per SM pair) or in
        // shared memory (64 registers, two clusters per SM pair when they fit)
        auto seg_fn_xs = ellP == 2 ? k_vjp_segment<R, SEG_NT, SEG_EPT, 2, true> : k_vjp_segment<R, SEG_NT, SEG_EPT, 4, true>;
        const size_t smem_xs = ellP == 2 ? vjp_seg_smem<R, 2, true>(n, ne, nb) : vjp_seg_smem<R, 4, true>(n, ne, nb);
        seg_smem = ellP == 2 ? vjp_seg_smem<R, 2>(n, ne, nb) : vjp_seg_smem<R, 4>(n, ne, nb);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        auto clusters = [&](ResKernelVjp<R> fn, size_t sm, int& ncl) -> int {
            ncl = 0;
            if (sm > ctx->smem_optin) return FPSG_OK;
            CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            cudaLaunchConfig_t lc = {};
            lc.gridDim = dim3(2 * B); lc.blockDim = dim3(SEG_NT); lc.dynamicSmemBytes = sm; lc.stream = ctx->stream;
            lc.attrs = at; lc.numAttrs = 1;
            CK(cudaOccupancyMaxActiveClusters(&ncl, (void*)fn, &lc));
            return FPSG_OK;
        };
        int ncl = 0, ncl_xs = 0;
        if ((rc = clusters(seg_fn, seg_smem, ncl)) || (rc = clusters(seg_fn_xs, smem_xs, ncl_xs))) { cleanup(); return rc; }
        if (ncl_xs > ncl) { seg_fn = seg_fn_xs; seg_smem = smem_xs; ncl = ncl_xs; }
        seg_grid = 2 * std::max(1, std::min(B, ncl));
        double* envtab = nullptr;
        int* bintab = nullptr;
        if (nb > 0 && Nsteps > 0) {
            std::vector<double> eh((size_t)Nsteps * 4);
            std::vector<int> bh((size_t)Nsteps * 4);
            for (long q = 0; q < Nsteps; ++q)
                for (int g = 0; g < 4; ++g) {
                    R pv; double env; int bin;
                    stage_info(q, g, pv, env, bin);
                    eh[(size_t)q * 4 + g] = env; bh[(size_t)q * 4 + g] = bin;
                }
            if ((rc = tmp((void**)&envtab, sizeof(double) * eh.size())) || (rc = tmp((void**)&bintab, sizeof(int) * bh.size()))) {
                cleanup(); return rc;
            }
            CK(cudaMemcpyAsync(envtab, eh.data(), sizeof(double) * eh.size(), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(bintab, bh.data(), sizeof(int) * bh.size(), cudaMemcpyHostToDevice, ctx->stream));
        }
        vs.sys = sys; vs.seg = seg; vs.count = count; vs.lam = lam;
        vs.ptab = ptab; vs.envtab = envtab; vs.bintab = bintab; vs.n_bins = nb;
        vs.h = hR; vs.S = S; vs.Tp = Tp; vs.dt = dt; vs.lscale = lscale;
        vs.ell_k = tables<R>(ctx).ell_k; vs.ell_v = tables<R>(ctx).ell_v; vs.order = ctx->res_order;
        vs.udiag = tables<R>(ctx).udiag; vs.err = d_err;
    }

    for (int b0 = 0; b0 < Ball; b0 += B) {
        const int Bk = std::min(B, Ball - b0);               // this chunk's trajectories
        const size_t ck_count = (size_t)Bk * 2 * ne;
        const int lgrid = std::max(1, std::min<int>((int)(((long)Bk * 2 * n + 255) / 256), ctx->sm_count * 8));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        evs.push_back(e0);
        CK(cudaEventCreate(&e1));
        evs.push_back(e1);
        CK(cudaEventRecord(e0, ctx->stream));
        if (std::is_same<R, double>::value)
            CK(cudaMemcpyAsync(st, ctx->rho64 + (size_t)b0 * 2 * ne, sizeof(cplx<R>) * ck_count, cudaMemcpyDeviceToDevice, ctx->stream));
        else
            k_f64_to_f32<<<cgrid, 256, 0, ctx->stream>>>(ctx->rho64 + (size_t)b0 * 2 * ne, (cplx<float>*)st, (long)ck_count);
        CK(cudaMemsetAsync(lam, 0, sizeof(cplx<R>) * count, ctx->stream));

        // ---- forward pass of the chunk: checkpoints and the loss records
        if (plan.idx >= 0) {
            ra.B = Bk;
            const int k = C / S;
            long step = 0;
            for (int t0 = 0; t0 < Tp; t0 += k) {
                const int t1 = std::min(Tp, t0 + k);
                if (step < Nsteps)
                    CK(cudaMemcpyAsync(ck + (size_t)(step / C) * count, st, sizeof(cplx<R>) * ck_count, cudaMemcpyDeviceToDevice, ctx->stream));
                ra.t_begin = t0; ra.t_end = t1;
                ra.ptab = ptab ? ptab + std::min<long>(step, Nsteps - 1) * 4 : nullptr;
                const long c = step / C;
                if (step < Nsteps && c >= nseg - n_keep) {
                    ResArgs<R> rk = ra;
                    rk.dump = keep + (size_t)(c - (nseg - n_keep)) * 4 * (size_t)C * count;
                    rk.dump_count = count;
                    if ((rc = rld.launch(ctx, rk))) { cleanup(); return rc; }
                } else if ((rc = rl.launch(ctx, ra))) {
                    cleanup();
                    return rc;
                }
                step += (long)(t1 - t0) * S - (t1 == Tp ? S : 0);
            }
        } else {
            for (long q = 0; q < Nsteps; ++q) {
                if (q % C == 0)
                    CK(cudaMemcpyAsync(ck + (size_t)(q / C) * count, st, sizeof(cplx<R>) * count, cudaMemcpyDeviceToDevice, ctx->stream));
                const bool rec = (q % S == 0);
                cplx<R>* const xin[4] = {st, X0, X1, X0};
                if ((rc = fwd_step(st, q, xin, rec))) { cleanup(); return rc; }
                if (rec) reduce_snapshot((int)(q / S));
            }
            sa.Xc = st; sa.record = 1;
            k_stream_record<R><<<grid, 256, 0, ctx->stream>>>(sa);
            reduce_snapshot(Tp - 1);
        }
        CK(cudaEventRecord(e1, ctx->stream));

        // ---- backward pass of the chunk
        k_loss_grad<R><<<lgrid, 256, 0, ctx->stream>>>(n, ne, Bk, st, lam, wt(Tp - 1) * lscale);
        double* pacc_c = pacc + (size_t)b0 * 2 * PW;
        for (long c = (Nsteps - 1) / C; c >= 0 && Nsteps > 0; --c) {
            const long s0 = c * C, s1 = std::min<long>(Nsteps, s0 + C);
            // the segment's stage inputs: kept from the sweep, or recomputed from its
            // checkpoint by one resident launch that writes each step's four stage inputs
            // into seg (or by stream stages)
            const bool kept = c >= nseg - n_keep;
            cplx<R>* segp = kept ? keep + (size_t)(c - (nseg - n_keep)) * 4 * (size_t)C * count : seg;
            if (!kept) {
                CK(cudaMemcpyAsync(X0, ck + (size_t)c * count, sizeof(cplx<R>) * ck_count, cudaMemcpyDeviceToDevice, ctx->stream));
                if (plan.idx >= 0) {
                    ResArgs<R> rr = ra;
                    rr.state = X0; rr.record = 0; rr.S = 1; rr.hf = 0; rr.Tp = 1 << 30;
                    rr.t_begin = 0; rr.t_end = (int)(s1 - s0); rr.step_base = 0;
                    rr.ptab = ptab ? ptab + s0 * 4 : nullptr;
                    rr.slots = nullptr; rr.whole = nullptr;
                    rr.dump = seg; rr.dump_count = count;
                    if ((rc = rld.launch(ctx, rr))) { cleanup(); return rc; }
                } else {
                    for (long q = s0; q < s1; ++q) {
                        cplx<R>* sq = seg + (size_t)(q - s0) * 4 * count;
                        CK(cudaMemcpyAsync(sq, X0, sizeof(cplx<R>) * count, cudaMemcpyDeviceToDevice, ctx->stream));
                        cplx<R>* const xin[4] = {X0, sq + count, sq + 2 * count, sq + 3 * count};
                        if ((rc = fwd_step(X0, q, xin, false))) { cleanup(); return rc; }
                    }
                }
            }
            if (use_seg) {
                vs.B = Bk; vs.pacc = pacc_c;
                vs.nsteps = (int)(s1 - s0); vs.s0 = s0; vs.seg = segp;
                cudaLaunchConfig_t lc = {};
                lc.gridDim = dim3(seg_grid); lc.blockDim = dim3(SEG_NT); lc.dynamicSmemBytes = seg_smem; lc.stream = ctx->stream;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = 2; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
                lc.attrs = at; lc.numAttrs = 1;
                CK(cudaLaunchKernelEx(&lc, seg_fn, vs));
                continue;
            }
            for (long q = s1 - 1; q >= s0; --q) {
                cplx<R>* sq = segp + (size_t)(q - s0) * 4 * count;
                const R c_lam[4] = {hR / R(8), R(3) * hR / R(8), R(3) * hR / R(8), hR / R(8)};
                for (int g = 3; g >= 0; --g) {
                    VjpArgs<R> va;
                    va.sys = sys; va.B = Bk; va.X = sq + (size_t)g * count; va.lam = lam;
                    va.c_lam = c_lam[g]; va.xb4 = va.xb3 = va.xb2 = nullptr; va.c4 = va.c3 = va.c2 = R(0);
                    if (g == 2) { va.xb4 = xbs[3]; va.c4 = hR; }
                    if (g == 1) { va.xb4 = xbs[3]; va.c4 = -hR; va.xb3 = xbs[2]; va.c3 = hR; }
                    if (g == 0) { va.xb4 = xbs[3]; va.c4 = hR; va.xb3 = xbs[2]; va.c3 = -hR / R(3); va.xb2 = xbs[1]; va.c2 = hR / R(3); }
                    stage_info(q, g, va.pulse, va.env, va.bin);
                    va.xb_out = xbs[g]; va.dbar = dbar; va.pacc = pacc_c; va.n_bins = nb;
                    if (use_ell)
                        ell_fn<<<egrid, 256, esmem, ctx->stream>>>(va, tables<R>(ctx).ell_k, tables<R>(ctx).ell_v);
                    else
                        k_vjp_stage<R><<<vgrid, 256, vsmem, ctx->stream>>>(va);
                    k_vjp_cross<R><<<lgrid, 256, 0, ctx->stream>>>(sys, Bk, dbar, xbs[g]);
                }
                k_lam_update<R><<<cgrid, 256, 0, ctx->stream>>>((long)ck_count, lam, xbs[0], xbs[1], xbs[2], xbs[3]);
                if (q % S == 0 && q > 0)
                    k_loss_grad<R><<<lgrid, 256, 0, ctx->stream>>>(n, ne, Bk, sq, lam, wt((int)(q / S)) * lscale);
                CK(cudaGetLastError());
            }
        }
    }
    if (plan.idx >= 0) {
        const long TW = (long)Tp * W;
        k_slot_reduce<<<std::max(1, std::min<int>((int)((TW + 255) / 256), ctx->sm_count * 4)), 256, 0, ctx->stream>>>(slots, rl.grid, TW, sums);
        CK(cudaGetLastError());
    }
    k_pacc_reduce<<<1, 64, 0, ctx->stream>>>(pacc, Ball * 2, PW, pout);
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    std::vector<double> hs((size_t)Tp * W), hp(PW);
    unsigned flag = 0;
    CK(cudaMemcpyAsync(hs.data(), sums, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hp.data(), pout, sizeof(double) * PW, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&flag, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f, fms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    for (size_t q = 0; q + 1 < evs.size(); q += 2) {
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, evs[q], evs[q + 1]));
        fms += f;
    }
    cleanup();
    if (flag) return set_error_from_flag(ctx, flag);
    double L = 0.0;
    const double Bd = (double)Ball;
    for (int t = 0; t < Tp; ++t) {
        const double* sm = hs.data() + (size_t)t * W;
        double acc = 0.0;
        for (int i = 0; i < n; ++i) acc += (sm[4 * n + i] / Bd + (sm[i] + sm[n + i]) / (2.0 * Bd)) + 0.25;
        L += wt(t) * acc / n;
    }
    if (loss_out) *loss_out = L;
    if (gU) *gU = hp[0];
    if (gT) *gT = hp[1];
    if (gP) for (int b = 0; b < nb; ++b) gP[b] = hp[2 + b];
    if (dev_ms) *dev_ms = ms;
    if (fwd_ms) *fwd_ms = fms;
    ctx->grad_info.chunk_traj = B;
    ctx->grad_info.chunks = (Ball + B - 1) / B;
    ctx->grad_info.segments = (int)nseg;
    ctx->grad_info.kept_segments = n_keep;
    return FPSG_OK;
}

int check_real_symmetric(const double* M, int n, const char* name, std::string& why)
{
    if (!M) return 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const double re = M[2 * ((size_t)j * n + i)], im = M[2 * ((size_t)j * n + i) + 1];
            const double ret = M[2 * ((size_t)i * n + j)];
            if (!std::isfinite(re) || !std::isfinite(im)) { why = std::string(name) + " has a non-finite entry"; return 1; }
            if (im != 0.0) { why = std::string(name) + " has a non-zero imaginary part"; return 1; }
            if (re != ret) { why = std::string(name) + " is not symmetric"; return 1; }
        }
    return 0;
}

// Normalised observables from the ensemble sums (src/FHfTWASolver.cpp:489-551;
// HF: src/FHHFSolver.cpp:404-419) into the caller's buffers.
void fill_outputs(int n, int ne, int B, int method, double dt, int S, int Tp, uint32_t obs_mask, const RunOut& ro,
                  fpsg_outputs* out)
{
    const int W = rec_width(n);
    const double Bd = (double)B;
    const bool ftwa = method == FPSG_METHOD_FTWA;
    for (int t = 0; t < Tp; ++t) {
        const double* s = ro.sums.data() + (size_t)t * W;
        if (out->time) out->time[t] = t * dt;
        for (int i = 0; i < n; ++i) {
            const double du = s[i], dd = s[n + i], d2u = s[2 * n + i], d2d = s[3 * n + i], dud = s[4 * n + i];
            const size_t o = (size_t)i * Tp + t;
            if (ftwa) {
                if (out->niiu) out->niiu[o] = du / Bd + 0.5;
                if (out->niid) out->niid[o] = dd / Bd + 0.5;
                if (out->n2iiu) out->n2iiu[o] = (d2u / Bd + (du + du) / (2.0 * Bd)) + 0.25;
                if (out->n2iid) out->n2iid[o] = (d2d / Bd + (dd + dd) / (2.0 * Bd)) + 0.25;
                if (out->nund) out->nund[o] = (dud / Bd + (du + dd) / (2.0 * Bd)) + 0.25;
            } else {
                if (out->niiu) out->niiu[o] = du / Bd;
                if (out->niid) out->niid[o] = dd / Bd;
                if (out->n2iiu) out->n2iiu[o] = d2u / Bd;
                if (out->n2iid) out->n2iid[o] = d2d / Bd;
                if (out->nund) out->nund[o] = dud / Bd;
            }
        }
        if (out->energies) {
            double tot = 0.0;
            for (int e = 0; e < 4; ++e) {
                double v = (obs_mask & FPSG_OBS_ENERGIES) ? s[5 * n + e] / Bd : 0.0;
                out->energies[(size_t)e * Tp + t] = v;
                tot += v;
            }
            out->energies[(size_t)4 * Tp + t] = tot;
        }
        if (!ro.whole.empty())
            for (int sp = 0; sp < 2; ++sp) {
                double* dst = sp == 0 ? out->whole_u : out->whole_d;
                if (!dst) continue;
                const double* src = ro.whole.data() + ((size_t)t * 2 + sp) * ne * 2;
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i) {
                        double re, im;
                        if (i <= j) { re = src[2 * (cs(j) + i)]; im = src[2 * (cs(j) + i) + 1]; }
                        else { re = src[2 * (cs(i) + j)]; im = -src[2 * (cs(i) + j) + 1]; }
                        re = re / Bd + ((ftwa && i == j) ? 0.5 : 0.0);
                        im = im / Bd;
                        dst[2 * ((size_t)t * n * n + (size_t)j * n + i)] = re;
                        dst[2 * ((size_t)t * n * n + (size_t)j * n + i) + 1] = im;
                    }
            }
    }
    out->device_ms = ro.device_ms;
    out->kernel_launches = ro.launches;
    out->traj_steps = (int64_t)B * (ftwa ? (int64_t)Tp * S : (int64_t)(Tp - 1) * S);
    out->path_used = ro.path_used;
}

// ------------------------------------------------------------------ batch
// Releases the device memory of a context made for one system of a batch (its
// stream and events belong to the parent).
void release_sub(fpsg_ctx* c)
{
    for (auto& a : c->allocs) cudaFree(a.p);
    c->allocs.clear();
    c->pool.clear();
}

template <typename R>
int batch_impl(fpsg_ctx* ctx, const fpsg_system_desc* sd, int ns, int method, double dt, int S, int Tp,
               uint32_t obs, fpsg_batch_info* info)
{
    const bool hf = method == FPSG_METHOD_HF;
    const double h = dt / (double)S;
    std::vector<std::unique_ptr<fpsg_ctx>> subs;
    std::vector<void*> temps;
    cudaGraph_t graph = nullptr, rgraph = nullptr;
    cudaGraphExec_t gexec = nullptr, rgexec = nullptr;
    auto tmp = [&](void** p, size_t bytes) -> int {
        int r = talloc(ctx, p, bytes);
        if (!r) temps.push_back(*p);
        return r;
    };
    auto cleanup = [&]() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (rgexec) cudaGraphExecDestroy(rgexec);
        if (rgraph) cudaGraphDestroy(rgraph);
        for (void* p : temps) trelease(ctx, p);
        for (auto& c : subs) release_sub(c.get());
    };
    // systems and their samples, each in a context of its own
    for (int k = 0; k < ns; ++k) {
        subs.emplace_back(new fpsg_ctx());
        fpsg_ctx* c = subs.back().get();
        c->device = ctx->device; c->sm_count = ctx->sm_count; c->smem_optin = ctx->smem_optin;
        c->stream = ctx->stream; c->ev0 = ctx->ev0; c->ev1 = ctx->ev1; c->flags = ctx->flags;
        c->mem_cap = ctx->mem_cap ? (ctx->mem_cap > ctx->mem_used ? ctx->mem_cap - ctx->mem_used : 1) : 0;
        int rc = fpsg_set_system(c, sd[k].n, sd[k].tM, sd[k].U, sd[k].V, sd[k].extpot, sd[k].coulomb_kind,
                                 sd[k].extpot_is_null);
        if (!rc) rc = fpsg_sample(c, sd[k].n_traj, sd[k].seed, sd[k].occ_up, sd[k].occ_dn, nullptr, nullptr);
        if (rc) {
            const std::string why = c->err;
            cleanup();
            return fail(ctx, rc, "system " + std::to_string(k) + ": " + why);
        }
    }
    unsigned* d_err = nullptr;
    int* t_ctr = nullptr;
    int rc = FPSG_OK;
    if ((rc = tmp((void**)&d_err, sizeof(unsigned))) || (rc = tmp((void**)&t_ctr, sizeof(int)))) { cleanup(); return rc; }
    CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(t_ctr, 0, sizeof(int), ctx->stream));
    const int rec_e = (obs & FPSG_OBS_ENERGIES) ? 1 : 0;
    std::vector<RunOut> ro(ns);
    std::vector<int> path_of(ns, FPSG_PATH_STREAM);

    // ---- systems that fit a resident kernel: every launch of every such system in
    // one captured graph (state in shared memory for whole windows of snapshots)
    struct ResSys {
        int k;
        ResPlan plan;
        ResLauncher<R> rl;
        cplx<R>* st;
        double *slots, *sums;
        ResArgs<R> ra;
    };
    std::vector<ResSys> rs;
    std::vector<int> sidx;                 // the others, on the stream stage
    for (int k = 0; k < ns; ++k) {
        fpsg_ctx* c = subs[k].get();
        const ResPlan plan = choose_resident<R>(c, c->B);
        if (plan.idx < 0) { sidx.push_back(k); continue; }
        ResSys r;
        r.k = k; r.plan = plan;
        if ((rc = r.rl.setup(c, plan, c->B))) { const std::string why = c->err; cleanup(); return fail(ctx, rc, why); }
        const int W = rec_width(c->n);
        const size_t count = (size_t)c->B * 2 * c->ne;
        r.st = nullptr;
        if (std::is_same<R, double>::value) r.st = (cplx<R>*)c->rho64;
        else if (!plan.comp) {
            if ((rc = tmp((void**)&r.st, sizeof(cplx<R>) * count))) { cleanup(); return rc; }
            k_f64_to_f32<<<std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
                c->rho64, (cplx<float>*)r.st, (long)count);
        }
        const size_t sbytes = sizeof(double) * (size_t)r.rl.grid * Tp * W;
        if ((rc = tmp((void**)&r.slots, sbytes)) || (rc = tmp((void**)&r.sums, sizeof(double) * (size_t)Tp * W))) {
            cleanup();
            return rc;
        }
        CK(cudaMemsetAsync(r.slots, 0, sbytes, ctx->stream));
        ResArgs<R>& ra = r.ra;
        ra.sys = make_sys<R>(c, tables<R>(c), method); ra.state = r.st; ra.B = c->B; ra.G = plan.G; ra.h = (R)h;
        ra.ptab = nullptr; ra.step_base = 0; ra.S = S; ra.Tp = Tp; ra.hf = hf ? 1 : 0;
        ra.record = 1; ra.do_en = rec_e;
        ra.do_e1 = (hf ? (c->coul != FPSG_COULOMB_NULL) : 1) && rec_e;
        ra.do_e2 = (hf ? (c->coul == FPSG_COULOMB_DISTANCE) : 1) && rec_e;
        ra.ell_k = plan.quad ? tables<R>(c).cell_k : tables<R>(c).ell_k;
        ra.ell_v = plan.quad ? tables<R>(c).cell_v : tables<R>(c).ell_v;
        ra.ell_pad = tables<R>(c).ell_pad;
        ra.slots = r.slots; ra.whole = nullptr; ra.err = d_err; ra.dump = nullptr; ra.dump_count = 0;
        ra.udiag = tables<R>(c).dd_fusable ? tables<R>(c).udiag : nullptr;
        ra.order = c->res_order;
        ra.state64 = plan.comp ? c->rho64 : nullptr;
        path_of[k] = FPSG_PATH_RESIDENT;
        rs.push_back(r);
    }
    int res_nodes = 0;
    int64_t res_launches = 0;
    if (!rs.empty()) {
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        for (ResSys& r : rs) {
            fpsg_ctx* c = subs[r.k].get();
            // time chunks as in fpsg_run, so one launch stays in the tens of milliseconds
            const long per_launch_steps = std::max<long>(1, 4096L * 1024 / std::max<long>(1, (long)c->B));
            const int chunk = (int)std::max<long>(1, std::min<long>(Tp, per_launch_steps / S + 1));
            for (int t0 = 0; t0 < Tp; t0 += chunk) {
                r.ra.t_begin = t0; r.ra.t_end = std::min(Tp, t0 + chunk);
                if (r.rl.launch(c, r.ra) != FPSG_OK) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(ctx->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    const std::string why = c->err;
                    cleanup();
                    return fail(ctx, FPSG_ERR_CUDA, why);
                }
                ++res_nodes;
            }
            const long TW = (long)Tp * rec_width(c->n);
            k_slot_reduce<<<std::max(1, std::min<int>((int)((TW + 255) / 256), ctx->sm_count * 4)), 256, 0, ctx->stream>>>(
                r.slots, r.rl.grid, TW, r.sums);
            ++res_nodes;
        }
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &rgraph);
        if (e != cudaSuccess) { cleanup(); return cuda_fail(ctx, e, "graph capture of the resident batch"); }
        e = cudaGraphInstantiate(&rgexec, rgraph, 0);
        if (e != cudaSuccess) { cleanup(); return cuda_fail(ctx, e, "graph instantiation"); }
        res_launches = res_nodes;
    }

    // ---- the rest: the stream stage over all their matrices, one persistent launch
    // per RK stage over a cost-ordered work list, one snapshot interval per graph replay
    const int chunk = 64;
    struct SysBuf {
        int k, n, ne, B, W, nch;
        cplx<R> *st, *A, *Bc, *X0, *X1;
        double *diagbuf, *ebuf, *part, *sums;
        double cost;
    };
    const int nss = (int)sidx.size();
    std::vector<SysBuf> sb(nss);
    size_t smem_full = 0, smem_gx = 0;
    int n_items = 0;
    for (int l = 0; l < nss; ++l) {
        fpsg_ctx* c = subs[sidx[l]].get();
        SysBuf& b = sb[l];
        b.k = sidx[l];
        b.n = c->n; b.ne = c->ne; b.B = c->B; b.W = rec_width(b.n); b.nch = (b.B + chunk - 1) / chunk;
        const size_t count = (size_t)b.B * 2 * b.ne;
        if (std::is_same<R, double>::value) b.st = (cplx<R>*)c->rho64;
        else if ((rc = tmp((void**)&b.st, sizeof(cplx<R>) * count))) { cleanup(); return rc; }
        if ((rc = tmp((void**)&b.A, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&b.Bc, sizeof(cplx<R>) * count)) ||
            (rc = tmp((void**)&b.X0, sizeof(cplx<R>) * count)) || (rc = tmp((void**)&b.X1, sizeof(cplx<R>) * count)) ||
            (rc = tmp((void**)&b.diagbuf, sizeof(double) * (size_t)b.B * 2 * b.n)) ||
            (rc = tmp((void**)&b.ebuf, sizeof(double) * (size_t)b.B * 2 * 4)) ||
            (rc = tmp((void**)&b.part, sizeof(double) * (size_t)b.nch * b.W)) ||
            (rc = tmp((void**)&b.sums, sizeof(double) * (size_t)Tp * b.W))) {
            cleanup();
            return rc;
        }
        CK(cudaMemsetAsync(b.ebuf, 0, sizeof(double) * (size_t)b.B * 2 * 4, ctx->stream));
        if (!std::is_same<R, double>::value)
            k_f64_to_f32<<<std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
                c->rho64, (cplx<float>*)b.st, (long)count);
        // work of one matrix-stage: every packed element walks its Delta column(s)
        b.cost = (double)b.ne * (2.0 + (double)c->nnz_h / b.n);
        smem_full = std::max(smem_full, ((sizeof(cplx<R>) * b.ne + sizeof(R) * b.n + 15) & ~size_t(15)) + sizeof(double) * 64);
        smem_gx = std::max(smem_gx, ((sizeof(R) * b.n + 15) & ~size_t(15)) + sizeof(double) * 64);
        n_items += 2 * b.B;
    }
    const bool gx = smem_full > ctx->smem_optin;
    const size_t smem = gx ? smem_gx : smem_full;
    auto kfn = gx ? k_batch_stage<R, true> : k_batch_stage<R, false>;
    int best_nt = 0, best_order = 0, grid = 0, nodes = 0;
    double tune_ms = 0.0;
    std::vector<StreamArgs<R>> ha;
    if (nss > 0) {
        CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // stage arguments: variant 0 = stage 0 recording a snapshot, 1..4 = stages 0..3
        ha.resize((size_t)5 * nss);
        for (int v = 0; v < 5; ++v)
            for (int l = 0; l < nss; ++l) {
                fpsg_ctx* c = subs[sidx[l]].get();
                SysBuf& b = sb[l];
                StreamArgs<R>& a = ha[(size_t)v * nss + l];
                const int g = v == 0 ? 0 : v - 1;
                const cplx<R>* xc[4] = {b.st, b.X0, b.X1, b.X0};
                cplx<R>* xn[4] = {b.X0, b.X1, b.X0, nullptr};
                a.sys = make_sys<R>(c, tables<R>(c), method);
                a.rho = b.st; a.A = b.A; a.Bc = b.Bc; a.Xc = xc[g]; a.Xn = xn[g];
                a.B = b.B; a.stage = g; a.h = (R)h; a.pulse = R(0);
                a.record = v == 0 ? 1 : 0;
                a.do_e1 = (hf ? (c->coul != FPSG_COULOMB_NULL) : 1) && rec_e;
                a.do_e2 = (hf ? 0 : 1) && rec_e;
                a.diagbuf = b.diagbuf; a.ebuf = b.ebuf; a.whole = nullptr; a.err = d_err;
            }
        StreamArgs<R>* args = nullptr;
        if ((rc = tmp((void**)&args, sizeof(StreamArgs<R>) * ha.size()))) { cleanup(); return rc; }
        CK(cudaMemcpyAsync(args, ha.data(), sizeof(StreamArgs<R>) * ha.size(), cudaMemcpyHostToDevice, ctx->stream));

        // schedules: 0 = systems by cost per matrix, descending, each system's matrices
        // contiguous (large matrices first, small ones fill the tail); 1 = round robin
        std::vector<int> by_cost(nss);
        for (int l = 0; l < nss; ++l) by_cost[l] = l;
        std::stable_sort(by_cost.begin(), by_cost.end(), [&](int x, int y) { return sb[x].cost > sb[y].cost; });
        std::vector<int2> hitems((size_t)2 * n_items);
        {
            size_t q = 0;
            for (int l : by_cost)
                for (int m = 0; m < 2 * sb[l].B; ++m) hitems[q++] = make_int2(l, m);
            int maxm = 0;
            for (int l = 0; l < nss; ++l) maxm = std::max(maxm, 2 * sb[l].B);
            for (int m = 0; m < maxm; ++m)
                for (int l : by_cost)
                    if (m < 2 * sb[l].B) hitems[q++] = make_int2(l, m);
        }
        int2* items = nullptr;
        if ((rc = tmp((void**)&items, sizeof(int2) * hitems.size()))) { cleanup(); return rc; }
        CK(cudaMemcpyAsync(items, hitems.data(), sizeof(int2) * hitems.size(), cudaMemcpyHostToDevice, ctx->stream));

        // autotuner: threads per CTA x schedule, timed on the side-effect-free stage 0
        std::string sig = std::string(std::is_same<R, double>::value ? "f64" : "f32") + (gx ? "g" : "s");
        for (int l = 0; l < nss; ++l)
            sig += ":" + std::to_string(sb[l].n) + "x" + std::to_string(sb[l].B) + "x" + std::to_string(subs[sidx[l]]->nnz_h);
        best_nt = 256;
        auto grid_for = [&](int nt) -> int {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nt, smem) != cudaSuccess) { cudaGetLastError(); per_sm = 1; }
            return std::max(1, std::min(n_items, std::max(1, per_sm) * ctx->sm_count));
        };
        auto it = ctx->batch_tune.find(sig);
        if (it != ctx->batch_tune.end()) {
            best_nt = it->second.first; best_order = it->second.second;
        } else {
            const auto w0 = std::chrono::steady_clock::now();
            float best = 1e30f;
            const int nts[3] = {128, 256, 512};
            for (int nt : nts)
                for (int order = 0; order < 2; ++order) {
                    const int g = grid_for(nt);
                    const int2* itp = items + (size_t)order * n_items;
                    kfn<<<g, nt, smem, ctx->stream>>>(args + nss, itp, n_items);
                    CK(cudaEventRecord(ctx->ev0, ctx->stream));
                    for (int r = 0; r < 2; ++r) kfn<<<g, nt, smem, ctx->stream>>>(args + nss, itp, n_items);
                    CK(cudaEventRecord(ctx->ev1, ctx->stream));
                    CK(cudaEventSynchronize(ctx->ev1));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
                    if (ms < best) { best = ms; best_nt = nt; best_order = order; }
                }
            ctx->batch_tune[sig] = std::make_pair(best_nt, best_order);
            tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        }
        grid = grid_for(best_nt);
        const int2* itp = items + (size_t)best_order * n_items;

        // one snapshot interval as a graph: record + S steps + per-system reductions + tick
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        for (int st = 0; st < S; ++st)
            for (int g = 0; g < 4; ++g) {
                const int v = g == 0 ? (st == 0 ? 0 : 1) : g + 1;
                kfn<<<grid, best_nt, smem, ctx->stream>>>(args + (size_t)v * nss, itp, n_items);
                ++nodes;
            }
        for (int l = 0; l < nss; ++l) {
            SysBuf& b = sb[l];
            k_reduce_part<<<b.nch, 256, 0, ctx->stream>>>(b.diagbuf, b.ebuf, b.B, b.n, chunk, b.part);
            k_reduce_fin_at<<<std::max(1, (b.W + 255) / 256), 256, 0, ctx->stream>>>(b.part, b.nch, b.W, b.sums, t_ctr);
            nodes += 2;
        }
        k_tick<<<1, 32, 0, ctx->stream>>>(t_ctr);
        ++nodes;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (e != cudaSuccess) { cleanup(); return cuda_fail(ctx, e, "graph capture of the batch interval"); }
        e = cudaGraphInstantiate(&gexec, graph, 0);
        if (e != cudaSuccess) { cleanup(); return cuda_fail(ctx, e, "graph instantiation"); }
    }

    int64_t launches = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (rgexec) {
        CK(cudaGraphLaunch(rgexec, ctx->stream));
        launches += res_launches;
    }
    if (gexec) {
        const int replays = hf ? Tp - 1 : Tp;
        for (int t = 0; t < replays; ++t) {
            CK(cudaGraphLaunch(gexec, ctx->stream));
            launches += nodes;
        }
        if (hf) {   // the last HF snapshot takes no step after it
            for (int l = 0; l < nss; ++l) {
                SysBuf& b = sb[l];
                k_stream_record<R><<<std::max(1, std::min(2 * b.B, 4 * ctx->sm_count)), 256, 0, ctx->stream>>>(ha[l]);
                k_reduce_part<<<b.nch, 256, 0, ctx->stream>>>(b.diagbuf, b.ebuf, b.B, b.n, chunk, b.part);
                k_reduce_fin_at<<<std::max(1, (b.W + 255) / 256), 256, 0, ctx->stream>>>(b.part, b.nch, b.W, b.sums, t_ctr);
                launches += 3;
            }
            CK(cudaGetLastError());
        }
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    // FP32 states back into each system's FP64 copy (not read by the caller; kept consistent)
    for (ResSys& r : rs)
        if (!std::is_same<R, double>::value && !r.plan.comp) {
            fpsg_ctx* c = subs[r.k].get();
            const size_t count = (size_t)c->B * 2 * c->ne;
            k_f32_to_f64<<<std::max(1, std::min<int>((int)((count + 255) / 256), ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
                (const cplx<float>*)r.st, c->rho64, (long)count);
        }
    unsigned flag = 0;
    CK(cudaMemcpyAsync(&flag, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    for (ResSys& r : rs) {
        ro[r.k].sums.resize((size_t)Tp * rec_width(subs[r.k]->n));
        CK(cudaMemcpyAsync(ro[r.k].sums.data(), r.sums, sizeof(double) * ro[r.k].sums.size(), cudaMemcpyDeviceToHost,
                           ctx->stream));
    }
    for (int l = 0; l < nss; ++l) {
        ro[sb[l].k].sums.resize((size_t)Tp * sb[l].W);
        CK(cudaMemcpyAsync(ro[sb[l].k].sums.data(), sb[l].sums, sizeof(double) * ro[sb[l].k].sums.size(),
                           cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    int64_t traj_steps = 0;
    for (int k = 0; k < ns; ++k) {
        fpsg_ctx* c = subs[k].get();
        ro[k].device_ms = ms;
        ro[k].launches = launches;
        ro[k].path_used = path_of[k];
        if (sd[k].out) fill_outputs(c->n, c->ne, c->B, method, dt, S, Tp, obs, ro[k], sd[k].out);
        traj_steps += (int64_t)c->B * (hf ? (int64_t)(Tp - 1) * S : (int64_t)Tp * S);
    }
    if (info) {
        info->block_threads = best_nt; info->schedule = best_order; info->grid = grid;
        info->graph_nodes = nodes + res_nodes;
        info->tune_ms = tune_ms; info->device_ms = ms; info->traj_steps = traj_steps; info->kernel_launches = launches;
    }
    cleanup();
    return set_error_from_flag(ctx, flag);
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

const char* fpsg_version(void) { return "fpsg 0.1 sm_100a"; }

int fpsg_create(fpsg_ctx** out, int device, uint64_t flags)
{
    if (!out) return FPSG_ERR_INVALID;
    if (flags & ~(uint64_t)(FPSG_FLAG_TEST_EXPIRE_WAIT | FPSG_FLAG_FP32_PLAIN_STATE)) return FPSG_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return FPSG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return FPSG_ERR_INVALID;
    fpsg_ctx* ctx = new (std::nothrow) fpsg_ctx();
    if (!ctx) return FPSG_ERR_OOM;
    ctx->device = device;
    ctx->flags = flags;
    if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return FPSG_ERR_CUDA; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete ctx; return FPSG_ERR_CUDA; }
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        delete ctx;
        return FPSG_ERR_CUDA;
    }
    *out = ctx;
    return FPSG_OK;
}

void fpsg_destroy(fpsg_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& a : ctx->allocs) cudaFree(a.p);
    ctx->allocs.clear();
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* fpsg_last_error(const fpsg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fpsg_set_grad_memory(fpsg_ctx* ctx, int64_t bytes)
{
    if (!ctx) return FPSG_ERR_INVALID;
    ctx->grad_keep = bytes < 0 ? -1 : bytes;
    return FPSG_OK;
}

int fpsg_last_grad_info(const fpsg_ctx* ctx, fpsg_grad_info* info)
{
    if (!ctx || !info) return FPSG_ERR_INVALID;
    *info = ctx->grad_info;
    return FPSG_OK;
}

int fpsg_set_memory_cap(fpsg_ctx* ctx, uint64_t bytes)
{
    if (!ctx) return FPSG_ERR_INVALID;
    ctx->mem_cap = bytes;
    if (bytes) trim_pool(ctx);
    return FPSG_OK;
}

int fpsg_set_system(fpsg_ctx* ctx, int n, const double* tM, const double* U, const double* V,
                    const double* extpot, int coulomb_kind, int extpot_is_null)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (n < 1 || n > 4096) return fail(ctx, FPSG_ERR_INVALID, "n must be in [1, 4096]");
    if (!tM || !U) return fail(ctx, FPSG_ERR_INVALID, "tM and U are required");
    if (coulomb_kind < 0 || coulomb_kind > 2) return fail(ctx, FPSG_ERR_INVALID, "bad coulomb kind");
    std::string why;
    if (check_real_symmetric(tM, n, "tM", why) || check_real_symmetric(U, n, "U", why) ||
        check_real_symmetric(V, n, "V", why) || (!extpot_is_null && check_real_symmetric(extpot, n, "extpot", why)))
        return fail(ctx, FPSG_ERR_UNSUPPORTED, why + " (the engine needs real symmetric inputs)");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    free_tables(ctx, ctx->t64);
    free_tables(ctx, ctx->t32);
    trelease(ctx, ctx->pij); ctx->pij = nullptr;
    trelease(ctx, ctx->res_order); ctx->res_order = nullptr;
    if (ctx->B > 0 && ctx->n != n) { dfree(ctx, ctx->rho64); ctx->rho64 = nullptr; ctx->B = 0; }
    ctx->n = n;
    ctx->ne = n * (n + 1) / 2;
    ctx->coul = coulomb_kind;
    ctx->ext_null = extpot_is_null ? 1 : 0;
    const size_t nn = (size_t)n * n;
    ctx->tM.assign(nn, 0.0); ctx->U.assign(nn, 0.0); ctx->V.assign(nn, 0.0); ctx->ext.assign(nn, 0.0);
    for (size_t q = 0; q < nn; ++q) {
        ctx->tM[q] = tM[2 * q];
        ctx->U[q] = U[2 * q];
        if (V) ctx->V[q] = V[2 * q];
        if (extpot && !extpot_is_null) ctx->ext[q] = extpot[2 * q];
    }
    ctx->ext_offdiag = false;
    for (int j = 0; j < n && !ctx->ext_null; ++j)
        for (int i = 0; i < n; ++i)
            if (i != j && ctx->ext[(size_t)j * n + i] != 0.0) ctx->ext_offdiag = true;
    if (ctx->n_bins > 0 && (int)ctx->proj.size() != n) ctx->n_bins = 0;
    std::vector<uint32_t> pij((size_t)ctx->ne);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) pij[(size_t)cs(j) + i] = (uint32_t)i | ((uint32_t)j << 16);
    int rc;
    if ((rc = upload(ctx, &ctx->pij, pij)) || (rc = upload(ctx, &ctx->res_order, res_slot_order(n)))) return rc;
    if ((rc = build_tables<double>(ctx, ctx->t64))) return rc;
    if ((rc = build_tables<float>(ctx, ctx->t32))) return rc;
    ctx->sys_set = true;
    return FPSG_OK;
}

int fpsg_set_pulse(fpsg_ctx* ctx, int n_bins, const double* amp, double bin_width, double t0, double td,
                   const double* proj)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (!ctx->sys_set) return fail(ctx, FPSG_ERR_STATE, "fpsg_set_system must come first");
    if (n_bins < 0) return fail(ctx, FPSG_ERR_INVALID, "n_bins < 0");
    trelease(ctx, ctx->d_amp); ctx->d_amp = nullptr;
    if (n_bins == 0) {
        ctx->n_bins = 0;
    } else {
        if (!amp || !proj || !(bin_width > 0.0) || !(td != 0.0)) return fail(ctx, FPSG_ERR_INVALID, "bad pulse parameters");
        ctx->n_bins = n_bins;
        ctx->amp.assign(amp, amp + n_bins);
        ctx->proj.assign(proj, proj + ctx->n);
        ctx->bin_width = bin_width; ctx->p_t0 = t0; ctx->p_td = td;
        int rc;
        if ((rc = upload(ctx, &ctx->d_amp, ctx->amp))) return rc;
    }
    free_tables(ctx, ctx->t64);
    free_tables(ctx, ctx->t32);
    int rc;
    if ((rc = build_tables<double>(ctx, ctx->t64))) return rc;
    if ((rc = build_tables<float>(ctx, ctx->t32))) return rc;
    return FPSG_OK;
}

static int alloc_state(fpsg_ctx* ctx, int B)
{
    if (ctx->rho64 && ctx->B == B) return FPSG_OK;
    dfree(ctx, ctx->rho64); ctx->rho64 = nullptr; ctx->B = 0;
    int rc = dalloc(ctx, (void**)&ctx->rho64, sizeof(cplx<double>) * (size_t)B * 2 * ctx->ne);
    if (rc) return rc;
    ctx->B = B;
    return FPSG_OK;
}

int fpsg_set_initial_samples(fpsg_ctx* ctx, int B, const double* rho0)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (!ctx->sys_set) return fail(ctx, FPSG_ERR_STATE, "fpsg_set_system must come first");
    if (B < 1 || !rho0) return fail(ctx, FPSG_ERR_INVALID, "B >= 1 and rho0 required");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    const int n = ctx->n, ne = ctx->ne;
    std::vector<cplx<double>> pk((size_t)B * 2 * ne);
    for (size_t m = 0; m < (size_t)B * 2; ++m) {
        const double* M = rho0 + m * 2 * (size_t)n * n;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i <= j; ++i) {
                cplx<double> v = { M[2 * ((size_t)j * n + i)], M[2 * ((size_t)j * n + i) + 1] };
                if (!std::isfinite(v.re) || !std::isfinite(v.im)) return fail(ctx, FPSG_ERR_INVALID, "non-finite initial sample");
                if (i == j) v.im = 0.0;
                pk[m * ne + cs(j) + i] = v;
            }
    }
    int rc = alloc_state(ctx, B);
    if (rc) return rc;
    if (cudaMemcpy(ctx->rho64, pk.data(), sizeof(cplx<double>) * pk.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ctx, FPSG_ERR_CUDA, "upload of initial samples failed");
    return FPSG_OK;
}

int fpsg_sample(fpsg_ctx* ctx, int B, uint64_t seed, const double* occ_up, const double* occ_dn,
                const double* rot_up, const double* rot_dn)
{
    return fpsg_sample_range(ctx, 0, B, seed, occ_up, occ_dn, rot_up, rot_dn);
}

int fpsg_sample_range(fpsg_ctx* ctx, int64_t first, int B, uint64_t seed, const double* occ_up,
                      const double* occ_dn, const double* rot_up, const double* rot_dn)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (first < 0) return fail(ctx, FPSG_ERR_INVALID, "first trajectory index must be >= 0");
    if (!ctx->sys_set) return fail(ctx, FPSG_ERR_STATE, "fpsg_set_system must come first");
    if (B < 1 || !occ_up || !occ_dn) return fail(ctx, FPSG_ERR_INVALID, "B >= 1 and occupations required");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    const int n = ctx->n, ne = ctx->ne;
    int rc = alloc_state(ctx, B);
    if (rc) return rc;
    double *ou = nullptr, *od = nullptr;
    cplx<double> *Ru = nullptr, *Rd = nullptr, *scr = nullptr;
    std::vector<double> vu(occ_up, occ_up + n), vd(occ_dn, occ_dn + n);
    if ((rc = upload(ctx, &ou, vu)) || (rc = upload(ctx, &od, vd))) { trelease(ctx, ou); trelease(ctx, od); return rc; }
    k_sample<<<std::max(1, std::min<int>((int)(((long)B * ne + 255) / 256), ctx->sm_count * 16)), 256, 0, ctx->stream>>>(
        n, ne, B, (long)first, seed, ou, od, ctx->rho64);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && (rot_up || rot_dn)) {
        const int grid = std::min(2 * B, ctx->sm_count * 4);
        std::vector<cplx<double>> hu, hd;
        // the caller's buffers need only double alignment: copy bytes, not elements
        if (rot_up) { hu.resize((size_t)n * n); std::memcpy(hu.data(), rot_up, sizeof(cplx<double>) * hu.size()); }
        if (rot_dn) { hd.resize((size_t)n * n); std::memcpy(hd.data(), rot_dn, sizeof(cplx<double>) * hd.size()); }
        if ((rot_up && (rc = upload(ctx, &Ru, hu))) || (rot_dn && (rc = upload(ctx, &Rd, hd))) ||
            (rc = talloc(ctx, (void**)&scr, sizeof(cplx<double>) * (size_t)grid * 2 * n * n))) {
            trelease(ctx, ou); trelease(ctx, od); trelease(ctx, Ru); trelease(ctx, Rd); trelease(ctx, scr);
            return rc;
        }
        k_rotate<<<grid, 256, 0, ctx->stream>>>(n, ne, B, Ru, Rd, ctx->rho64, scr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    trelease(ctx, ou); trelease(ctx, od); trelease(ctx, Ru); trelease(ctx, Rd); trelease(ctx, scr);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fpsg_sample");
    return FPSG_OK;
}

static int validate_run(fpsg_ctx* ctx, int method, int precision, int path, double dt, int S)
{
    if (!ctx->sys_set) return fail(ctx, FPSG_ERR_STATE, "fpsg_set_system must come first");
    if (ctx->B < 1) return fail(ctx, FPSG_ERR_STATE, "no initial samples (fpsg_sample or fpsg_set_initial_samples)");
    if (method != FPSG_METHOD_FTWA && method != FPSG_METHOD_HF) return fail(ctx, FPSG_ERR_INVALID, "unknown method");
    if (precision < 0 || precision > 3) return fail(ctx, FPSG_ERR_INVALID, "unknown precision");
    if (path < 0 || path > 3) return fail(ctx, FPSG_ERR_INVALID, "unknown path");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(ctx, FPSG_ERR_INVALID, "dt must be positive");
    if (S < 1) return fail(ctx, FPSG_ERR_INVALID, "steps_per_snapshot must be >= 1");
    const bool split = precision == FPSG_PREC_SPLIT_BF16X3 || precision == FPSG_PREC_SPLIT_TF32X3;
    if (method == FPSG_METHOD_HF && ctx->coul == FPSG_COULOMB_DISTANCE && split)
        return fail(ctx, FPSG_ERR_UNSUPPORTED, "HF with the Fock term runs on the stream path (FP64 or FP32)");
    if (split && path != FPSG_PATH_AUTO && path != FPSG_PATH_DENSE)
        return fail(ctx, FPSG_ERR_INVALID, "the split precisions run on the dense path only");
    if (path == FPSG_PATH_DENSE && !split)
        return fail(ctx, FPSG_ERR_INVALID, "the dense path computes in split BF16x3 or TF32x3");
    return FPSG_OK;
}

int fpsg_run(fpsg_ctx* ctx, int method, int precision, int path, double dt, int steps_per_snapshot,
             int n_snapshots, uint32_t obs_mask, fpsg_outputs* out)
{
    if (!ctx) return FPSG_ERR_INVALID;
    const auto w0 = std::chrono::steady_clock::now();
    int rc = validate_run(ctx, method, precision, path, dt, steps_per_snapshot);
    if (rc) return rc;
    if (n_snapshots < 1) return fail(ctx, FPSG_ERR_INVALID, "n_snapshots must be >= 1");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    RunReq q;
    q.method = method; q.precision = precision; q.path = path; q.dt = dt; q.S = steps_per_snapshot;
    q.Tp = n_snapshots; q.record = 1; q.obs = obs_mask; q.t_start = 0.0; q.n_steps = 0;
    RunOut ro;
    rc = precision == FPSG_PREC_FP64          ? run_impl<double>(ctx, q, ro)
         : (precision == FPSG_PREC_SPLIT_BF16X3 || precision == FPSG_PREC_SPLIT_TF32X3) ? dense_impl(ctx, q, ro)
                                               : run_impl<float>(ctx, q, ro);
    if (rc) return rc;
    if (!out) return FPSG_OK;
    fill_outputs(ctx->n, ctx->ne, ctx->B, method, dt, steps_per_snapshot, n_snapshots, obs_mask, ro, out);
    out->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    return FPSG_OK;
}

int fpsg_advance(fpsg_ctx* ctx, int method, int precision, int path, double dt, int steps_per_snapshot,
                 double t_start, int n_steps, double* device_ms, int64_t* launches)
{
    if (!ctx) return FPSG_ERR_INVALID;
    int rc = validate_run(ctx, method, precision, path, dt, steps_per_snapshot);
    if (rc) return rc;
    if (n_steps < 0) return fail(ctx, FPSG_ERR_INVALID, "n_steps must be >= 0");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    RunReq q;
    q.method = method; q.precision = precision; q.path = path; q.dt = dt; q.S = steps_per_snapshot;
    q.Tp = 1; q.record = 0; q.obs = 0; q.t_start = t_start; q.n_steps = n_steps;
    RunOut ro;
    rc = precision == FPSG_PREC_FP64          ? run_impl<double>(ctx, q, ro)
         : (precision == FPSG_PREC_SPLIT_BF16X3 || precision == FPSG_PREC_SPLIT_TF32X3) ? dense_impl(ctx, q, ro)
                                               : run_impl<float>(ctx, q, ro);
    if (device_ms) *device_ms = ro.device_ms;
    if (launches) *launches = ro.launches;
    return rc;
}

int fpsg_run_batch(fpsg_ctx* ctx, const fpsg_system_desc* systems, int n_systems, int method, int precision,
                   double dt, int steps_per_snapshot, int n_snapshots, uint32_t obs_mask, fpsg_batch_info* info)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (!systems || n_systems < 1) return fail(ctx, FPSG_ERR_INVALID, "at least one system is required");
    if (method != FPSG_METHOD_FTWA && method != FPSG_METHOD_HF) return fail(ctx, FPSG_ERR_INVALID, "unknown method");
    if (precision != FPSG_PREC_FP64 && precision != FPSG_PREC_FP32)
        return fail(ctx, FPSG_ERR_UNSUPPORTED, "batches run in FP64 or FP32");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(ctx, FPSG_ERR_INVALID, "dt must be positive");
    if (steps_per_snapshot < 1 || n_snapshots < 1) return fail(ctx, FPSG_ERR_INVALID, "steps_per_snapshot and n_snapshots must be >= 1");
    if (obs_mask & FPSG_OBS_WHOLE) return fail(ctx, FPSG_ERR_UNSUPPORTED, "whole-matrix observables are not recorded in batches");
    for (int k = 0; k < n_systems; ++k) {
        const fpsg_system_desc& d = systems[k];
        if (d.n < 1 || d.n_traj < 1 || !d.tM || !d.U || !d.occ_up || !d.occ_dn)
            return fail(ctx, FPSG_ERR_INVALID, "system " + std::to_string(k) + ": n, n_traj, tM, U and occupations are required");
        if (method == FPSG_METHOD_HF && d.coulomb_kind == FPSG_COULOMB_DISTANCE)
            return fail(ctx, FPSG_ERR_UNSUPPORTED, "HF with a same-spin V is not batched");
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    return precision == FPSG_PREC_FP64
               ? batch_impl<double>(ctx, systems, n_systems, method, dt, steps_per_snapshot, n_snapshots, obs_mask, info)
               : batch_impl<float>(ctx, systems, n_systems, method, dt, steps_per_snapshot, n_snapshots, obs_mask, info);
}

int fpsg_grad(fpsg_ctx* ctx, int precision, double dt, int steps_per_snapshot, int n_snapshots,
              int checkpoint_every, double* loss, double* dL_dUscale, double* dL_dtscale, double* dL_dpulse,
              double* device_ms, double* forward_ms)
{
    if (!ctx) return FPSG_ERR_INVALID;
    int rc = validate_run(ctx, FPSG_METHOD_FTWA, precision, FPSG_PATH_STREAM, dt, steps_per_snapshot);
    if (rc) return rc;
    if (n_snapshots < 2) return fail(ctx, FPSG_ERR_INVALID, "n_snapshots must be >= 2");
    if (checkpoint_every < 1) return fail(ctx, FPSG_ERR_INVALID, "checkpoint_every must be >= 1");
    // the tM-scale term uses <K, -i[X, tM]> = <X, i[K, Delta]> - sum_j (Delta_jj - tM_jj) dbar_j,
    // which holds only when Delta equals tM off its diagonal
    if (ctx->ext_offdiag)
        return fail(ctx, FPSG_ERR_UNSUPPORTED, "fpsg_grad needs a diagonal static potential (extpot has off-diagonal entries)");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    return precision == FPSG_PREC_FP64
               ? grad_impl<double>(ctx, dt, steps_per_snapshot, n_snapshots, checkpoint_every, loss, dL_dUscale,
                                   dL_dtscale, dL_dpulse, device_ms, forward_ms)
               : grad_impl<float>(ctx, dt, steps_per_snapshot, n_snapshots, checkpoint_every, loss, dL_dUscale,
                                  dL_dtscale, dL_dpulse, device_ms, forward_ms);
}

// GPSR drift of B trajectories given as full complex matrices (host buffers in and
// out); four stage launches over all matrices, FP64 (src/FHGPSRSolver.cpp:168-206).
int fpsg_gpsr_drift(fpsg_ctx* ctx, int B, const double* rho, double t, double d_t, double* drift)
{
    if (!ctx) return FPSG_ERR_INVALID;
    (void)t;
    if (!ctx->sys_set) return fail(ctx, FPSG_ERR_STATE, "fpsg_set_system must come first");
    if (B < 1 || !rho || !drift) return fail(ctx, FPSG_ERR_INVALID, "B >= 1 and non-null rho, drift needed");
    if (!std::isfinite(d_t)) return fail(ctx, FPSG_ERR_INVALID, "d_t must be finite");
    if (ctx->n_bins > 0)
        return fail(ctx, FPSG_ERR_UNSUPPORTED, "the GPSR drift takes static potentials only (a pulse is set)");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    const int n = ctx->n;
    const size_t nn = (size_t)n * n, count = (size_t)B * 2 * nn;
    const size_t bytes = sizeof(cplx<double>) * count;
    std::vector<void*> temps;
    auto cleanup = [&]() { for (void* p : temps) trelease(ctx, p); };
    cplx<double> *r, *x0, *x1, *A, *Bc, *dr;
    cplx<double>** bufs[6] = {&r, &x0, &x1, &A, &Bc, &dr};
    for (auto b : bufs) {
        int rc = talloc(ctx, (void**)b, bytes);
        if (rc) { cleanup(); return rc; }
        temps.push_back(*b);
    }
    CK(cudaMemcpyAsync(r, rho, bytes, cudaMemcpyHostToDevice, ctx->stream));
    GpsrArgs a;
    a.sys = make_sys<double>(ctx, tables<double>(ctx), FPSG_METHOD_HF);   // shift 0
    a.sys.fock = 0;                                                       // no exchange term
    a.M = 2 * B; a.rho = r; a.A = A; a.Bc = Bc; a.drift = dr; a.h = d_t;
    a.stage_x_in_smem = gpsr_smem_bytes(n, true) <= ctx->smem_optin ? 1 : 0;
    const size_t smem = gpsr_smem_bytes(n, a.stage_x_in_smem != 0);
    void (*fns[4])(GpsrArgs) = {k_gpsr_stage<0>, k_gpsr_stage<1>, k_gpsr_stage<2>, k_gpsr_stage<3>};
    int per_sm = 1;
    for (auto fn : fns) CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fns[0], 256, smem));
    const int grid = std::max(1, std::min(2 * B, std::max(1, per_sm) * ctx->sm_count));
    const cplx<double>* in[4] = {r, x0, x1, x0};
    cplx<double>* out[4] = {x0, x1, x0, nullptr};
    for (int g = 0; g < 4; ++g) {
        a.X = in[g];
        a.Xn = out[g];
        fns[g]<<<grid, 256, smem, ctx->stream>>>(a);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(drift, dr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cleanup();
    return FPSG_OK;
}

int fpsg_get_state(fpsg_ctx* ctx, double* rho)
{
    if (!ctx) return FPSG_ERR_INVALID;
    if (ctx->B < 1) return fail(ctx, FPSG_ERR_STATE, "no state");
    if (!rho) return fail(ctx, FPSG_ERR_INVALID, "null output");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, FPSG_ERR_CUDA, "cudaSetDevice");
    const int n = ctx->n, ne = ctx->ne;
    std::vector<cplx<double>> pk((size_t)ctx->B * 2 * ne);
    if (cudaMemcpy(pk.data(), ctx->rho64, sizeof(cplx<double>) * pk.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ctx, FPSG_ERR_CUDA, "state download failed");
    for (size_t m = 0; m < (size_t)ctx->B * 2; ++m) {
        double* M = rho + m * 2 * (size_t)n * n;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                cplx<double> v = (i <= j) ? pk[m * ne + cs(j) + i] : pk[m * ne + cs(i) + j];
                if (i > j) v.im = -v.im;
                M[2 * ((size_t)j * n + i)] = v.re;
                M[2 * ((size_t)j * n + i) + 1] = v.im;
            }
    }
    return FPSG_OK;
}

int fpsg_num_trajectories(const fpsg_ctx* ctx) { return ctx ? ctx->B : 0; }

}  // extern "C"
