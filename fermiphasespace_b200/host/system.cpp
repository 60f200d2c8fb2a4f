// system.cpp — FHSystem: Hamiltonian matrices, initial conditions, core hole and
// the tight-binding / mean-field ground states.
#include "system.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace fps {

// ------------------------------------------------------------------ eigensolver
void eig_sym(int n, const std::vector<double>& Ain, std::vector<double>& w, std::vector<double>& V)
{
    std::vector<double> A = Ain;
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    auto a = [&](int i, int j) -> double& { return A[(size_t)j * n + i]; };
    auto v = [&](int i, int j) -> double& { return V[(size_t)j * n + i]; };
    double fro = 0.0;
    for (double x : A) fro += x * x;
    fro = std::sqrt(fro);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < j; ++i) off += a(i, j) * a(i, j);
        if (std::sqrt(2.0 * off) <= 1e-15 * std::max(fro, 1e-300)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a(p, q);
                if (apq == 0.0) continue;
                // symmetric Schur decomposition of the 2x2 block (p, q)
                const double tau = (a(q, q) - a(p, p)) / (2.0 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::abs(tau) + std::sqrt(1.0 + tau * tau));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {   // A <- A J (columns p, q)
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {   // A <- J^T A (rows p, q)
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {   // V <- V J
                    const double vkp = v(k, p), vkq = v(k, q);
                    v(k, p) = c * vkp - s * vkq;
                    v(k, q) = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return a(x, x) < a(y, y); });
    w.assign(n, 0.0);
    std::vector<double> Vs((size_t)n * n);
    for (int c = 0; c < n; ++c) {
        w[c] = a(order[c], order[c]);
        // sign convention: largest-magnitude component positive
        int im = 0;
        for (int k = 1; k < n; ++k)
            if (std::abs(v(k, order[c])) > std::abs(v(im, order[c]))) im = k;
        const double sg = v(im, order[c]) < 0 ? -1.0 : 1.0;
        for (int k = 0; k < n; ++k) Vs[(size_t)c * n + k] = sg * v(k, order[c]);
    }
    V.swap(Vs);
}

namespace {

void projector(int n, const std::vector<double>& V, unsigned nocc, std::vector<double>& N)
{
    N.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (unsigned k = 0; k < nocc && (int)k < n; ++k) s += V[(size_t)k * n + i] * V[(size_t)k * n + j];
            N[(size_t)j * n + i] = s;
        }
}

Json jarray(const std::vector<double>& v)
{
    Json a = Json::array();
    for (double x : v) a.append(x);
    return a;
}

}  // namespace

// FHTunnelingInteraction::addTunneling, src/FHTunnelingInteraction.cpp:293-312
static void add_tunneling(const FHLattice& lat, std::vector<double>& T, double d, double E)
{
    const int n = lat.nSites();
    const double ths = lat.samePointDistance;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            const double x = lat.distance(i, j) - d;
            if (x * x < ths) {
                T[(size_t)j * n + i] += E;
                T[(size_t)i * n + j] += E;
            }
        }
}

// FHCoulombInteraction::addCoulombinU / addCoulombinV, src/FHCoulombInteraction.cpp:246-288
static void add_coulomb(const FHLattice& lat, std::vector<double>& U, std::vector<double>& V, double d, double E)
{
    const int n = lat.nSites();
    const double ths = lat.samePointDistance;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const double x = lat.distance(i, j) - d;
            if (x * x < ths) {
                U[(size_t)j * n + i] += E;
                if (i != j) V[(size_t)j * n + i] += E;
            }
        }
}

// FHSystem::setInitialConditions(type, nPart), src/FHSystem.cpp:536-595
static void diagonal_ic(const std::string& sub, unsigned nu, unsigned nd, int N, std::vector<double>& up,
                        std::vector<double>& dn)
{
    up.assign(N, 0.0);
    dn.assign(N, 0.0);
    if (sub == "spinWave") {
        for (unsigned s = 0; s < std::min((unsigned)N, 2 * nu); s += 2) up[s] = 1.0;
        for (unsigned s = 1; s < std::min((unsigned)N, 2 * nd); s += 2) dn[s] = 1.0;
    } else if (sub == "chargeWave") {
        for (unsigned s = 0; s < std::min((unsigned)N, 2 * nu); s += 2) up[s] = 1.0;
        for (unsigned s = 0; s < std::min((unsigned)N, 2 * nd); s += 2) dn[s] = 1.0;
    }
}

bool FHSystem::fromJson(const Json& sys, const std::string& folder, FHSystem& out, std::string& err)
{
    out = FHSystem();
    if (!FHLattice::fromJson(sys.get("lattice", Json()), folder, out.lattice, err)) return false;
    const FHLattice& lat = out.lattice;
    const int N = lat.nSites();
    out.n = N;
    const size_t nn = (size_t)N * N;
    out.tM.assign(nn, 0.0); out.U.assign(nn, 0.0); out.V.assign(nn, 0.0); out.ext.assign(nn, 0.0);

    // tunneling, src/FHTunnelingInteraction.cpp:16-125
    const Json& tj = sys["tunnelingInteraction"];
    const std::string tt = tj.get("type", "null").asString();
    if (tt == "nearestNeighbors") {
        const double d = tj.get("neighborDistance", 1.0).asDouble(), E = tj.get("neighborInteraction", -1.0).asDouble();
        add_tunneling(lat, out.tM, d, E);
        out.tunnType = tt; out.tunnDistances = {d}; out.tunnEnergies = {E};
    } else if (tt == "distanceInteraction") {
        const Json& ds = tj["distances"];
        const Json& es = tj["energies"];
        out.tunnType = tt;
        if (!ds.isNull()) {
            if (ds.size() != es.size()) { err = "tunnelingInteraction: distances and energies differ in length"; return false; }
            for (size_t q = 0; q < ds.size(); ++q) {
                add_tunneling(lat, out.tM, ds[q].asDouble(), es[q].asDouble());
                out.tunnDistances.push_back(ds[q].asDouble());
                out.tunnEnergies.push_back(es[q].asDouble());
            }
        }
    } else if (tt == "distanceInteraction1" || tt == "distanceInteraction2" || tt == "given") {
        out.tunnType = tt;   // parsed by the reference, no matrix entries
    }

    // Coulomb, src/FHCoulombInteraction.cpp:13-33 (+ distanceInteraction, :57-76)
    const Json& cj = sys["coulombInteraction"];
    const std::string ct = cj.get("type", "null").asString();
    if (ct == "onSite") {
        out.onSiteU = cj.get("onSiteInteraction", 1.0).asDouble();
        add_coulomb(lat, out.U, out.V, 0.0, out.onSiteU);
        out.coulomb = COUL_ONSITE;
        out.coulType = ct;
    } else if (ct == "distanceInteraction") {
        const Json& ds = cj["distances"];
        const Json& es = cj["energies"];
        if (ds.size() != es.size()) { err = "coulombInteraction: distances and energies differ in length"; return false; }
        for (size_t q = 0; q < ds.size(); ++q) {
            add_coulomb(lat, out.U, out.V, ds[q].asDouble(), es[q].asDouble());
            out.coulDistances.push_back(ds[q].asDouble());
            out.coulEnergies.push_back(es[q].asDouble());
        }
        out.coulomb = COUL_DISTANCE;
        out.coulType = ct;
    }

    // external potential, src/FHSystem.cpp:146-169
    const Json& ej = sys["externalPotential"];
    if (!ej.isNull()) {
        const std::string et = ej.get("type", "null").asString();
        if (et == "constant") {
            const Json& dg = ej["diagonal"];
            for (int i = 0; i < N && i < (int)dg.size(); ++i) out.ext[(size_t)i * N + i] = dg[i].asDouble();
            out.extNull = false;
            out.extType = et;
        } else if (et == "coreHole") {
            const unsigned site = ej.get("site", 0).asUInt();
            const double pot = ej.get("holePotential", -1.0).asDouble();
            if ((int)site < N) out.ext[(size_t)site * N + site] = pot;
            out.extNull = false;
            out.extType = "constant";
        }
    }

    // initial condition, src/FHSystem.cpp:173-289
    const Json& ic = sys["IC"];
    if (!ic.isNull()) {
        const std::string type = ic.get("type", "givenDiagonal").asString();
        const unsigned nu = (unsigned)ic.get("nPartUp", (long long)std::ceil(N / 2.0)).asUInt();
        const unsigned nd = (unsigned)ic.get("nPartDown", (long long)std::floor(N / 2.0)).asUInt();
        out.nPartUp = nu; out.nPartDn = nd;
        if (type == "givenDiagonal") {
            out.icType = "givenDiagonal";
            const std::string sub = ic.get("subtype", "spinWave").asString();
            out.icSubtype = sub;
            out.occUp.assign(N, 0.0);
            out.occDn.assign(N, 0.0);
            if (sub == "spinWave" || sub == "chargeWave") {
                diagonal_ic(sub, nu, nd, N, out.occUp, out.occDn);
            } else if (sub == "spinWave3" || sub == "chargeWave3") {
                const int mid = N / 2;   // std::ceil of an integer division
                for (int s = 0; s < mid; ++s) out.occUp[s] = 1.0;
                if (sub == "spinWave3") for (int s = mid; s < N; ++s) out.occDn[s] = 1.0;
                else for (int s = 0; s < mid; ++s) out.occDn[s] = 1.0;
            } else if (sub == "givenInJson") {
                const Json& a = ic["IC_NuDiag"];
                const Json& b = ic["IC_NdDiag"];
                if (a.isArray()) for (int s = 0; s < std::min((int)a.size(), N); ++s) out.occUp[s] = a[s].asBool() ? 1.0 : 0.0;
                if (b.isArray()) for (int s = 0; s < std::min((int)b.size(), N); ++s) out.occDn[s] = b[s].asBool() ? 1.0 : 0.0;
            }
        } else if (type == "tbGroundState") {
            out.icType = type;
            out.computeTBGroundState();
        } else if (type == "mfGroundState") {
            out.icType = type;
            out.computeMFGroundState();
        } else if (type == "groundState") {
            err = "IC type groundState has no solver initialisation in FermiPhaseSpace (use mfGroundState)";
            return false;
        }
    }

    // core hole, src/FHSystem.cpp:296-324: one extra orbital coupled to `site`
    const Json& ch = sys["coreHole"];
    if (!ch.isNull() && ch.get("presence", false).asBool()) {
        CoreHole h;
        h.site = ch.get("site", 0).asUInt();
        h.eps = ch.get("eps", -2.0).asDouble();
        h.X = ch.get("X", -1.0).asDouble();
        h.Uc = ch.get("Uc", 1.0).asDouble();
        h.G = ch.get("G", 1.0).asDouble();
        const Json& occ = ch["IC"];
        if (occ.size() > 0) h.occUp = occ[0].asDouble();
        if (occ.size() > 1) h.occDn = occ[1].asDouble();
        if ((int)h.site >= N) { err = "coreHole site outside the lattice"; return false; }
        if (out.coulomb == COUL_DISTANCE) { err = "coreHole with a distance Coulomb interaction is not supported"; return false; }
        const int M = N + 1;
        auto grow = [&](const std::vector<double>& A) {
            std::vector<double> B((size_t)M * M, 0.0);
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) B[(size_t)j * M + i] = A[(size_t)j * N + i];
            return B;
        };
        std::vector<double> T2 = grow(out.tM), U2 = grow(out.U), V2((size_t)M * M, 0.0), E2((size_t)M * M, 0.0);
        T2[(size_t)N * M + h.site] = h.X;            // FHTunnelingInteraction::addSite
        T2[(size_t)h.site * M + N] = h.X;
        std::vector<double> cou(M, 0.0);             // FHCoulombInteraction::addSite (U, V += c/2 on row/col N)
        cou[h.site] = h.G;
        cou[N] = h.Uc;
        for (int i = 0; i < M; ++i) {
            U2[(size_t)N * M + i] += cou[i] / 2.0;
            U2[(size_t)i * M + N] += cou[i] / 2.0;
            V2[(size_t)N * M + i] += cou[i] / 2.0;
            V2[(size_t)i * M + N] += cou[i] / 2.0;
        }
        V2[(size_t)N * M + N] = 0.0;
        // the system's potential is replaced by the hole potential alone (src/FHSystem.cpp:311-312)
        out.extNull = (h.eps == 0.0);
        E2[(size_t)N * M + N] = h.eps;
        out.tM.swap(T2); out.U.swap(U2); out.V.swap(V2); out.ext.swap(E2);
        out.coulomb = COUL_DISTANCE;                 // type "given": U and same-spin V both act
        out.hasCoreHole = true;
        out.coreHole = h;
        out.n = M;
    }
    return true;
}

FHSystem FHSystem::basis(const FHLattice& lat)
{
    FHSystem s;
    s.lattice = lat;
    const int N = lat.nSites();
    s.n = N;
    s.tM.assign((size_t)N * N, 0.0); s.U.assign((size_t)N * N, 0.0); s.V.assign((size_t)N * N, 0.0);
    s.ext.assign((size_t)N * N, 0.0);
    add_tunneling(lat, s.tM, 1.0, -1.0);
    s.tunnType = "nearestNeighbors"; s.tunnDistances = {1.0}; s.tunnEnergies = {-1.0};
    std::vector<double> vdummy((size_t)N * N, 0.0);
    add_coulomb(lat, s.U, vdummy, 0.0, 1.0);     // addCoulombinU only (src/FHCoulombInteraction.cpp:35-54)
    s.coulomb = COUL_ONSITE; s.coulType = "onSite"; s.onSiteU = 1.0;
    return s;
}

// FHSystem::setInitialConditions(type), src/FHSystem.cpp:453-530
void FHSystem::setInitialConditions(const std::string& kind)
{
    const int N = lattice.nSites();
    occUp.assign(N, 0.0);
    occDn.assign(N, 0.0);
    if (kind == "spinWave" || kind == "chargeWave") {
        icType = "givenDiagonal";
        icSubtype = kind;
        for (int s = 0; s < N; ++s) {
            if (s % 2 == 0) { occUp[s] = 1.0; if (kind == "chargeWave") occDn[s] = 1.0; }
            else if (kind == "spinWave") occDn[s] = 1.0;
        }
        nPartUp = (unsigned)std::count(occUp.begin(), occUp.end(), 1.0);
        nPartDn = (unsigned)std::count(occDn.begin(), occDn.end(), 1.0);
    } else {
        icType = kind;
        nPartUp = (unsigned)std::ceil(N / 2.0);
        nPartDn = (unsigned)std::floor(N / 2.0);
        if (kind == "tbGroundState") computeTBGroundState();
        else if (kind == "mfGroundState") computeMFGroundState();
    }
}

void FHSystem::computeTBGroundState()
{
    const int N = lattice.nSites();
    std::vector<double> T((size_t)N * N);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) T[(size_t)j * N + i] = tM[(size_t)j * n + i];
    eig_sym(N, T, tbE, tbV);
    projector(N, tbV, nPartUp, tbNu);
    projector(N, tbV, nPartDn, tbNd);
    tbComputed = true;
}

void FHSystem::computeMFGroundState()
{
    const int N = lattice.nSites();
    std::vector<double> du(N, 0.0), dd(N, 0.0);   // starting densities: zero (Hartree-free first pass)
    const double thr = 0.0001 * N;
    mfIterations = 0;
    bool conv = false;
    std::vector<double> Hu((size_t)N * N), Hd((size_t)N * N);
    while (mfIterations < 100 && !conv) {
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                Hu[(size_t)j * N + i] = tM[(size_t)j * n + i];
                Hd[(size_t)j * N + i] = tM[(size_t)j * n + i];
            }
        for (int i = 0; i < N; ++i) {
            double su = 0.0, sd = 0.0;
            for (int k = 0; k < N; ++k) {
                su += U[(size_t)k * n + i] * dd[k];
                sd += U[(size_t)k * n + i] * du[k];
            }
            Hu[(size_t)i * N + i] += su;
            Hd[(size_t)i * N + i] += sd;
        }
        eig_sym(N, Hu, mfEu, mfVu);
        eig_sym(N, Hd, mfEd, mfVd);
        projector(N, mfVu, nPartUp, mfNu);
        projector(N, mfVd, nPartDn, mfNd);
        ++mfIterations;
        double ru = 0.0, rd = 0.0;
        for (int i = 0; i < N; ++i) {
            const double a = mfNu[(size_t)i * N + i] - du[i], b = mfNd[(size_t)i * N + i] - dd[i];
            ru += a * a; rd += b * b;
        }
        mfResidue = std::sqrt(ru) + std::sqrt(rd);
        if (mfResidue < thr) conv = true;
        else
            for (int i = 0; i < N; ++i) { du[i] = mfNu[(size_t)i * N + i]; dd[i] = mfNd[(size_t)i * N + i]; }
    }
    mfComputed = true;
}

static Json matrix_rows(int N, const std::vector<double>& M)
{
    Json rows = Json::array();
    for (int i = 0; i < N; ++i) {
        Json r = Json::array();
        for (int j = 0; j < N; ++j) r.append(M[(size_t)j * N + i]);
        rows.append(r);
    }
    return rows;
}

Json FHSystem::tbGroundStateJson()
{
    if (!tbComputed) computeTBGroundState();
    Json j = Json::object();
    j["energyVector"] = jarray(tbE);
    j["rotationMatrix"] = matrix_rows(lattice.nSites(), tbV);
    return j;
}

Json FHSystem::mfGroundStateJson()
{
    if (!mfComputed) computeMFGroundState();
    Json j = Json::object();
    j["energyVectorUp"] = jarray(mfEu);
    j["energyVectorDown"] = jarray(mfEd);
    j["rotationMatrixUp"] = matrix_rows(lattice.nSites(), mfVu);
    j["rotationMatrixDown"] = matrix_rows(lattice.nSites(), mfVd);
    j["iterationsNeeded"] = mfIterations;
    j["residueComputation"] = mfResidue;
    return j;
}

Json FHSystem::toJson() const
{
    Json root = Json::object();
    root["lattice"] = lattice.toJson();
    Json ic = Json::object();
    if (icType == "givenDiagonal") {
        ic["type"] = "givenDiagonal";
        if (icSubtype == "spinWave" || icSubtype == "chargeWave") ic["subtype"] = icSubtype;
    } else if (icType != "none") {
        ic["type"] = icType;
    }
    root["IC"] = ic;
    Json t = Json::object();
    if (tunnType == "nearestNeighbors") {
        t["type"] = tunnType;
        t["neighborDistance"] = tunnDistances.empty() ? 1.0 : tunnDistances[0];
        t["neighborInteraction"] = tunnEnergies.empty() ? -1.0 : tunnEnergies[0];
    } else if (tunnType == "distanceInteraction") {
        t["type"] = tunnType;
        t["distances"] = jarray(tunnDistances);
        t["energies"] = jarray(tunnEnergies);
    } else {
        t["type"] = "null";
    }
    root["tunnelingInteraction"] = t;
    Json c = Json::object();
    if (coulType == "onSite") {
        c["type"] = "onSite";
        c["onSiteInteraction"] = onSiteU;
    } else if (coulType == "distanceInteraction") {
        c["type"] = coulType;
        c["distances"] = jarray(coulDistances);
        c["energies"] = jarray(coulEnergies);
    } else {
        c["type"] = "null";
    }
    root["coulombInteraction"] = c;
    Json e = Json::object();
    if (!extNull) {
        e["type"] = "constant";
        std::vector<double> d;
        for (int i = 0; i < n; ++i) d.push_back(ext[(size_t)i * n + i]);
        e["diagonal"] = jarray(d);
    } else {
        e["type"] = "null";
    }
    root["externalPotential"] = e;
    return root;
}

}  // namespace fps
