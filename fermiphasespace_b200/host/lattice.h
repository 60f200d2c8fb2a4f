// lattice.h — site geometry (FermiPhaseSpace's FHLattice, include/FHLattice.h:54-159).
#pragma once

#include <array>
#include <string>
#include <vector>

#include "json.h"

namespace fps {

using Vec3 = std::array<double, 3>;

class FHLattice {
public:
    // JSON lattice block (src/FHLattice.cpp:101-167): positionsFile (xyz, relative
    // to folder), latticeType, periodic, latticeMatrix[3][3], latticeZero[3].
    static bool fromJson(const Json& root, const std::string& folder, FHLattice& out, std::string& err);
    // Generator (src/FHLattice.cpp:169-325): type name and parameters, missing
    // parameters count as 1 (makeSitesSystem.cpp:128-131).  Types: grid, bcc,
    // fcc, honeyCombs, triangular, graphene, moireHC, moire, plus kagome and
    // fccPeriodic (conventional cubic cells with periodic boundaries), which the
    // reference names but does not generate.
    static bool generate(const std::string& type, std::vector<double> params, FHLattice& out, std::string& err);

    int nSites() const { return (int)pos.size(); }
    double distance(int i, int j) const { return dist[(size_t)i * pos.size() + j]; }
    void setPositions(const std::vector<Vec3>& p, const std::string& siteName = "C");
    void computeMatrices();                 // distances (minimum image when periodic)
    bool readPositions(const std::string& path, std::string& err);
    bool writePositions(const std::string& baseName, const std::string& folder, std::string& err) const;
    Json toJson() const;                    // writeFHLatticeJson, src/FHLattice.cpp:741-770

    std::vector<Vec3> pos;
    std::vector<std::string> siteNames;
    std::vector<double> dist;               // n x n
    std::string type = "none";
    std::string name;
    bool periodic = false;
    double latticeMatrix[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // columns are the lattice vectors
    double latticeZero[3] = {0, 0, 0};
    double neighbourDistance = 1.0;
    double samePointDistance = 1e-4;        // JSON-lattice default, include/FHLattice.h:77
};

}  // namespace fps
