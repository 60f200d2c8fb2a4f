// fpsg_quad_f64.cu — FP64 configurations of the 4-CTA-cluster resident kernels.
#include "fpsg_resident.h"

namespace fpsg {

template <>
const std::vector<QuadCfg<double>>& quad_cfgs<double>()
{
    static const std::vector<QuadCfg<double>> v = {
        FPSG_QUAD(double, 512, 3), FPSG_QUAD(double, 512, 5),
    };
    return v;
}

template <>
const std::vector<QuadCfg<double>>& quad_hp_cfgs<double>()
{
    static const std::vector<QuadCfg<double>> v = {
        FPSG_QUAD_HP64(512, 5), FPSG_QUAD_HP64(640, 4), FPSG_QUAD_HP64(384, 7),
    };
    return v;
}

}  // namespace fpsg
