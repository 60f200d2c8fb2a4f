// makeSitesSystem — writes <folder>/<name>.json and <name>.xyz for a generated
// lattice (makeSitesSystem.cpp:49-221).  Usage:
//   makeSitesSystem <name> <geometry> <param1> <param2> ... [ic_sw|ic_cw|ic_tbgs|ic_mfgs] [--folder DIR]
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "fps_host.h"

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cout << "To make a new system :" << std::endl;
        std::cout << "./makeSitesSystem <nameOfTheSystem> <geometryOfTheSites> <param1> <param2> ..." << std::endl;
        return 0;
    }
    std::string name = argv[1], geometry = argc > 2 ? argv[2] : "grid", ic = "ic_sw", folder = "systemsFolder";
    std::vector<double> params;
    bool numeric = true;   // a non-numeric argument ends the parameter list, as in the reference
    for (int a = 3; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "ic_sw" || s == "ic_cw" || s == "ic_tbgs" || s == "ic_mfgs") { ic = s; continue; }
        if (s == "--folder" && a + 1 < argc) { folder = argv[++a]; continue; }
        char* end = nullptr;
        const double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str()) numeric = false;
        else if (numeric) params.push_back(v);
    }
    std::cout << "== Writing a new FH system." << std::endl;
    const int rc = fpsh_make_sites_system(name.c_str(), folder.c_str(), geometry.c_str(), params.data(),
                                          (int)params.size(), ic.c_str());
    if (rc) std::cerr << "makeSitesSystem: " << fpsh_last_error() << std::endl;
    return rc ? 1 : 0;
}
