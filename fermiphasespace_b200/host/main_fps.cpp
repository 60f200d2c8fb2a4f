// fps — runs one simulation file (fps.cpp:26-282) with method "fTWA" or "HF" on the GPU engine.
#include <iostream>
#include <string>

#include "fps_host.h"

int main(int argc, char** argv)
{
    std::cout << "== FermiPhaseSpace simulation (B200 trajectory engine)" << std::endl;
    if (argc < 2) {
        std::cout << "Need a json file. " << std::endl;
        return 1;
    }
    const int rc = fpsh_run_fps(argv[1]);
    if (rc) std::cerr << "fps: " << fpsh_last_error() << std::endl;
    std::cout << "== Program closing." << std::endl;
    return rc;
}
