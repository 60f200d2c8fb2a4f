// system.h — the Fermi-Hubbard system the solvers integrate (FermiPhaseSpace's
// FHSystem with its FHTunnelingInteraction, FHCoulombInteraction,
// FHExternalPotential and FHCoreHole members).  Matrices are dense n x n real,
// column-major (element (i, j) at j*n + i); the reference keeps them as
// arma::cx_dmat with zero imaginary parts.
#pragma once

#include <string>
#include <vector>

#include "json.h"
#include "lattice.h"

namespace fps {

// Real symmetric eigen-decomposition (cyclic Jacobi, Golub & Van Loan,
// Matrix Computations, 4th ed., §8.5): eigenvalues ascending, eigenvectors as
// the columns of V (col-major).  Replaces arma::eig_sym for the real symmetric
// matrices of the TB / MF ground states (src/FHSystem.cpp:917-921, 982-988).
void eig_sym(int n, const std::vector<double>& A, std::vector<double>& w, std::vector<double>& V);

enum CoulombKind { COUL_NULL = 0, COUL_ONSITE = 1, COUL_DISTANCE = 2 };

struct CoreHole {                       // FHCoreHole, src/FHCoreHole.cpp:7-21
    unsigned site = 0;
    double eps = -2, X = -1, Uc = 1, G = 1;
    double occUp = 1, occDn = 0;
};

class FHSystem {
public:
    // FHSystem(Json, folder), src/FHSystem.cpp:123-326
    static bool fromJson(const Json& sys, const std::string& folder, FHSystem& out, std::string& err);
    // FHSystem(FHLattice) + setBasisInteractions, src/FHSystem.cpp:329-338, 599-603
    static FHSystem basis(const FHLattice& lat);

    int nSites() const { return n; }            // orbitals per spin (lattice + core hole)
    int nLatticeSites() const { return lattice.nSites(); }

    void setInitialConditions(const std::string& kind);   // spinWave / chargeWave / tbGroundState / mfGroundState
    void computeTBGroundState();                // src/FHSystem.cpp:911-940
    void computeMFGroundState();                // src/FHSystem.cpp:943-1019
    Json toJson() const;                        // writeFHSystemJson, src/FHSystem.cpp:1025-1140
    Json tbGroundStateJson();
    Json mfGroundStateJson();

    FHLattice lattice;
    int n = 0;
    std::vector<double> tM, U, V, ext;          // n x n
    int coulomb = COUL_NULL;
    bool extNull = true;
    bool hasCoreHole = false;
    CoreHole coreHole;

    // initial condition: "givenDiagonal" family (with occupations), tbGroundState, mfGroundState
    std::string icType = "none", icSubtype;
    std::vector<double> occUp, occDn;           // lattice sites
    unsigned nPartUp = 0, nPartDn = 0;

    // parameters kept for the JSON writers
    std::string tunnType = "null";
    std::vector<double> tunnDistances, tunnEnergies;
    std::string coulType = "null";
    double onSiteU = 1.0;
    std::vector<double> coulDistances, coulEnergies;
    std::string extType = "null";

    // ground states (lattice sites only)
    bool tbComputed = false, mfComputed = false;
    std::vector<double> tbE, tbV, tbNu, tbNd;
    std::vector<double> mfEu, mfEd, mfVu, mfVd, mfNu, mfNd;
    int mfIterations = 0;
    double mfResidue = 0.0;
};

}  // namespace fps
