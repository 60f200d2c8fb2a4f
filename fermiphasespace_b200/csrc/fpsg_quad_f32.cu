// fpsg_quad_f32.cu — FP32 configurations of the 4-CTA-cluster resident kernels.
#include "fpsg_resident.h"

namespace fpsg {

template <>
const std::vector<QuadCfg<float>>& quad_cfgs<float>()
{
    static const std::vector<QuadCfg<float>> v = {
        FPSG_QUAD(float, 512, 6), FPSG_QUAD(float, 512, 8), FPSG_QUAD(float, 384, 14),
    };
    return v;
}

template <>
const std::vector<QuadCfg<float>>& quad_hp_cfgs<float>()
{
    static const std::vector<QuadCfg<float>> v = {
        FPSG_QUAD_HP32(512, 12, 1), FPSG_QUAD_HP32(512, 6, 2), FPSG_QUAD_HP32(512, 11, 2),
    };
    return v;
}

}  // namespace fpsg
