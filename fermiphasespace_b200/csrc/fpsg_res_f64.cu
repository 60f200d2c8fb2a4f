// fpsg_res_f64.cu — FP64 resident-kernel configurations.
#include "fpsg_resident.h"

namespace fpsg {

template <>
const std::vector<ResCfg<double>>& res_cfgs<double>()
{
    static const std::vector<ResCfg<double>> v = {
        FPSG_RES(double, 128, 1, false), FPSG_RES(double, 128, 2, false), FPSG_RES(double, 128, 4, false),
        FPSG_RES(double, 256, 4, false), FPSG_RES(double, 256, 8, false),
        FPSG_RES(double, 256, 9, true), FPSG_RES(double, 512, 8, true),
    };
    return v;
}

}  // namespace fpsg
