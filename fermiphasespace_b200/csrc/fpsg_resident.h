// fpsg_resident.h — the instantiated configurations of the resident kernel.
// Each precision's table lives in its own translation unit (fpsg_res_f32.cu,
// fpsg_res_f64.cu) so that the kernel variants compile in parallel.
#pragma once
#include <vector>

#include "fpsg_kernels.cuh"
#include "fpsg_quad.cuh"

namespace fpsg {

template <typename R>
using ResKernel = void (*)(ResArgs<R>);

template <typename R>
struct ResCfg {
    int nt, ept;            // threads per CTA, elements per thread
    bool split;             // one spin per CTA in a 2-CTA cluster
    ResKernel<R> fn[3];     // P = 2, 4, 8 entries per side of the diagonal
    ResKernel<R> fn_dump[3];  // the same, writing every stage input (adjoint recompute)
};

template <typename R>
const std::vector<ResCfg<R>>& res_cfgs();

template <>
const std::vector<ResCfg<float>>& res_cfgs<float>();
template <>
const std::vector<ResCfg<double>>& res_cfgs<double>();

// 4-CTA-cluster configurations (k_resident_quad): two CTAs per spin matrix
template <typename R>
struct QuadCfg {
    int nt, ept;            // threads per CTA, elements per thread (of half a matrix)
    ResKernel<R> fn[4];     // compact column width W = 5, 9, 13, 17
    ResKernel<R> fn8[4];    // k_resident_quad_hp: the same with 8-byte column entries
    int nh = 2;             // k_resident_quad_hp: CTAs per spin (1: 2-CTA clusters)
};

// index of a compact column width in QuadCfg::fn (-1: wider than supported)
inline int quad_w_index(int W) { return W <= 5 ? 0 : W <= 9 ? 1 : W <= 13 ? 2 : W <= 17 ? 3 : -1; }

template <typename R>
const std::vector<QuadCfg<R>>& quad_cfgs();

template <>
const std::vector<QuadCfg<float>>& quad_cfgs<float>();
template <>
const std::vector<QuadCfg<double>>& quad_cfgs<double>();

// 4-CTA configurations with the packed, double-buffered matrix (k_resident_quad_hp)
template <typename R>
const std::vector<QuadCfg<R>>& quad_hp_cfgs();

template <>
const std::vector<QuadCfg<float>>& quad_hp_cfgs<float>();
template <>
const std::vector<QuadCfg<double>>& quad_hp_cfgs<double>();

}  // namespace fpsg

#define FPSG_RES(R, NT, EPT, SPLIT)                                                                           \
    {NT, EPT, SPLIT,                                                                                      \
     {k_resident<R, NT, EPT, SPLIT, 2>, k_resident<R, NT, EPT, SPLIT, 4>, k_resident<R, NT, EPT, SPLIT, 8>}, \
     {k_resident<R, NT, EPT, SPLIT, 2, true>, k_resident<R, NT, EPT, SPLIT, 4, true>,                     \
      k_resident<R, NT, EPT, SPLIT, 8, true>}}

#define FPSG_QUAD(R, NT, EPT)                                                                     \
    {NT, EPT, {k_resident_quad<R, NT, EPT, 5>, k_resident_quad<R, NT, EPT, 9>, k_resident_quad<R, NT, EPT, 13>, \
               k_resident_quad<R, NT, EPT, 17>}, {}}

// FP64: 16-byte (FP64 weights) and 8-byte (FP32-exact weights) column entries
#define FPSG_QUAD_HP64(NT, EPT)                                                                         \
    {NT, EPT, {k_resident_quad_hp<double, NT, EPT, 5, false, 2>, k_resident_quad_hp<double, NT, EPT, 9, false, 2>, \
               k_resident_quad_hp<double, NT, EPT, 13, false, 2>, k_resident_quad_hp<double, NT, EPT, 17, false, 2>}, \
              {k_resident_quad_hp<double, NT, EPT, 5, true, 2>, k_resident_quad_hp<double, NT, EPT, 9, true, 2>,     \
               k_resident_quad_hp<double, NT, EPT, 13, true, 2>, k_resident_quad_hp<double, NT, EPT, 17, true, 2>}}
// FP32: 8-byte entries only; NH_ CTAs per spin (2: 4-CTA clusters, 1: 2-CTA clusters)
#define FPSG_QUAD_HP32(NT, EPT, NH_)                                                                    \
    {NT, EPT, {k_resident_quad_hp<float, NT, EPT, 5, true, NH_>, k_resident_quad_hp<float, NT, EPT, 9, true, NH_>,   \
               k_resident_quad_hp<float, NT, EPT, 13, true, NH_>, k_resident_quad_hp<float, NT, EPT, 17, true, NH_>}, \
              {k_resident_quad_hp<float, NT, EPT, 5, true, NH_>, k_resident_quad_hp<float, NT, EPT, 9, true, NH_>,   \
               k_resident_quad_hp<float, NT, EPT, 13, true, NH_>, k_resident_quad_hp<float, NT, EPT, 17, true, NH_>}, NH_}
