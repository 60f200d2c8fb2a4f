// fpsg_res_f32.cu — FP32 resident-kernel configurations.
#include "fpsg_resident.h"

namespace fpsg {

template <>
const std::vector<ResCfg<float>>& res_cfgs<float>()
{
    static const std::vector<ResCfg<float>> v = {
        FPSG_RES(float, 128, 1, false), FPSG_RES(float, 128, 2, false), FPSG_RES(float, 128, 4, false),
        FPSG_RES(float, 256, 4, false), FPSG_RES(float, 256, 8, false), FPSG_RES(float, 512, 8, false),
        FPSG_RES(float, 512, 8, true), FPSG_RES(float, 512, 10, true),
    };
    return v;
}

}  // namespace fpsg
