// lattice.cpp — FHLattice: xyz I/O, minimum-image distances and the site
// generators.  Generators keep the reference's site order and floating-point
// construction so that generated systems match FermiPhaseSpace's site by site.
#include "lattice.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>

namespace fps {

namespace {

const double kPi = 3.14159265358979323846;

// makeBCGrid, src/FHLattice.cpp:872-895 (x fastest)
std::vector<Vec3> make_grid(unsigned nx, unsigned ny, unsigned nz, double a)
{
    std::vector<Vec3> p;
    for (unsigned z = 0; z < nz; ++z)
        for (unsigned y = 0; y < ny; ++y)
            for (unsigned x = 0; x < nx; ++x) p.push_back({a * x, a * y, a * z});
    return p;
}

// makeBCCGrid, src/FHLattice.cpp:909-939
std::vector<Vec3> make_bcc(unsigned nx, unsigned ny, unsigned nz, double a)
{
    std::vector<Vec3> p;
    for (unsigned z = 0; z <= nz; ++z)
        for (unsigned y = 0; y <= ny; ++y)
            for (unsigned x = 0; x <= nx; ++x) {
                p.push_back({a * x, a * y, a * z});
                if (x != nx && y != ny && z != nz) p.push_back({a * (x + 0.5), a * (y + 0.5), a * (z + 0.5)});
            }
    return p;
}

// makeFCCGrid, src/FHLattice.cpp:948-989
std::vector<Vec3> make_fcc(unsigned nx, unsigned ny, unsigned nz, double a)
{
    std::vector<Vec3> p;
    for (unsigned z = 0; z <= nz; ++z)
        for (unsigned y = 0; y <= ny; ++y)
            for (unsigned x = 0; x <= nx; ++x) {
                p.push_back({a * x, a * y, a * z});
                if (y != ny && z != nz) p.push_back({a * x, a * (y + 0.5), a * (z + 0.5)});
                if (x != nx && z != nz) p.push_back({a * (x + 0.5), a * y, a * (z + 0.5)});
                if (x != nx && y != ny) p.push_back({a * (x + 0.5), a * (y + 0.5), a * z});
            }
    return p;
}

// conventional fcc cells with periodic boundaries: 4 sites per cell
std::vector<Vec3> make_fcc_periodic(unsigned nx, unsigned ny, unsigned nz, double a)
{
    std::vector<Vec3> p;
    for (unsigned z = 0; z < nz; ++z)
        for (unsigned y = 0; y < ny; ++y)
            for (unsigned x = 0; x < nx; ++x) {
                p.push_back({a * x, a * y, a * z});
                p.push_back({a * x, a * (y + 0.5), a * (z + 0.5)});
                p.push_back({a * (x + 0.5), a * y, a * (z + 0.5)});
                p.push_back({a * (x + 0.5), a * (y + 0.5), a * z});
            }
    return p;
}

// kagome: cells a1 = (2a, 0), a2 = (a, sqrt3 a), basis (0,0), (a,0), (a/2, sqrt3 a/2);
// nearest-neighbour distance a; cells x fastest
std::vector<Vec3> make_kagome(unsigned nx, unsigned ny, double a)
{
    const double s3 = std::sqrt(3.0);
    std::vector<Vec3> p;
    for (unsigned y = 0; y < ny; ++y)
        for (unsigned x = 0; x < nx; ++x) {
            const double ox = 2.0 * a * x + a * y, oy = s3 * a * y;
            p.push_back({ox, oy, 0.0});
            p.push_back({ox + a, oy, 0.0});
            p.push_back({ox + 0.5 * a, oy + 0.5 * s3 * a, 0.0});
        }
    return p;
}

// getNextIndex, src/FHLattice.cpp:1329-1350
void next_index(unsigned& i, unsigned& j)
{
    if (i == j) { i = i + 1; j = 0; }
    else if (i == j + 1) { j = i; i = 0; }
    else if (i > j) { j = j + 1; }
    else { i = i + 1; }
}

// makeHoneyCombs, src/FHLattice.cpp:998-1066
std::vector<Vec3> make_honeycombs(unsigned nCombs, double a)
{
    const double s3 = std::sqrt(3.0);
    const std::vector<Vec3> pos0 = {{-s3 / 2 * a, -0.5 * a, 0}, {-s3 / 2 * a, 0.5 * a, 0}, {0 * a, 1 * a, 0},
                                    {0 * a, -1 * a, 0},         {s3 / 2 * a, -0.5 * a, 0}, {s3 / 2 * a, 0.5 * a, 0}};
    const double iv[2] = {s3 * a, 0 * a}, jv[2] = {s3 / 2 * a, 1.5 * a};
    unsigned bi[2] = {0, 0};
    std::vector<Vec3> pos;
    for (unsigned c = 0; c < nCombs; ++c) {
        std::vector<Vec3> pn = pos0;
        for (int q = 0; q < 6; ++q) {
            pn[q][0] = pos0[q][0] + iv[0] * bi[0] + jv[0] * bi[1];
            pn[q][1] = pos0[q][1] + iv[1] * bi[0] + jv[1] * bi[1];
        }
        pos.insert(pos.end(), pn.begin(), pn.end());
        next_index(bi[0], bi[1]);
    }
    const double thr = 0.0001 * a;
    for (size_t i1 = 0; i1 < pos.size(); ++i1) {
        unsigned found = 0;
        size_t i2 = i1 + 1;
        while (i2 < pos.size() && found < 2) {
            double d = 0;
            for (int k = 0; k < 3; ++k) d += std::abs(pos[i1][k] - pos[i2][k]);
            if (std::abs(d) < thr) { pos.erase(pos.begin() + i2); ++found; }
            else ++i2;
        }
    }
    return pos;
}

// makeGraphene, src/FHLattice.cpp:1093-1130
std::vector<Vec3> make_graphene(int nx, int ny, double a)
{
    const double s3 = std::sqrt(3.0);
    const double iv[2] = {s3 * a, 0 * a}, jv[2] = {s3 / 2 * a, 1.5 * a};
    std::vector<Vec3> pos;
    for (int j = 0; j < ny; ++j) {
        Vec3 y0 = {0, -0.5 * a, 0}, y1 = {0, 0.5 * a, 0};
        y0[0] += jv[0] * j; y0[1] += jv[1] * j;
        y1[0] += jv[0] * j; y1[1] += jv[1] * j;
        for (int i = 0; i < nx; ++i) {
            Vec3 p0 = y0, p1 = y1;
            p0[0] += iv[0] * i; p0[1] += iv[1] * i;
            p1[0] += iv[0] * i; p1[1] += iv[1] * i;
            pos.push_back(p0);
            pos.push_back(p1);
        }
    }
    return pos;
}

// makeTetragones, src/FHLattice.cpp:1142-1166
std::vector<Vec3> make_tetragones(int nx, int ny, int nz, double a)
{
    const double s3 = std::sqrt(3.0);
    const double iv[3] = {a, 0, 0}, jv[3] = {1. / 2. * a, s3 / 2. * a, 0};
    const double kv[3] = {1. / 2. * a, 1. / (2 * s3) * a, std::sqrt(2.0) / s3 * a};
    std::vector<Vec3> pos;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                pos.push_back({i * iv[0] + j * jv[0] + k * kv[0], i * iv[1] + j * jv[1] + k * kv[1],
                               i * iv[2] + j * jv[2] + k * kv[2]});
    return pos;
}

void set_box(double L[3][3], const double m[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) L[i][j] = m[i][j];
}

// makeMoireGraphene, src/FHLattice.cpp:1272-1307 (theta in degrees)
std::vector<Vec3> make_moire(int nx, int ny, double a, double b, double theta)
{
    const double s3 = std::sqrt(3.0);
    const double th = theta * kPi / 180;
    std::vector<Vec3> pos;
    const double c0[3] = {s3 * a * nx, 0, 0}, c1[3] = {s3 / 2 * a * ny, 1.5 * a * ny, 0};
    const double mid[3] = {(c0[0] + c1[0]) / 2., (c0[1] + c1[1]) / 2., (c0[2] + c1[2]) / 2.};
    for (unsigned layer = 0; layer < 2; ++layer) {
        const double ct = std::cos(layer * th), st = std::sin(layer * th);
        std::vector<Vec3> pl = make_graphene(nx, ny, a);
        for (auto& p : pl) {
            const double x = p[0] - mid[0], y = p[1] - mid[1], z = p[2] - mid[2];
            const double rx = ct * x + -st * y + 0 * z;
            const double ry = st * x + ct * y + 0 * z;
            p = {rx, ry, layer * b};
        }
        pos.insert(pos.end(), pl.begin(), pl.end());
    }
    return pos;
}

}  // namespace

void FHLattice::setPositions(const std::vector<Vec3>& p, const std::string& siteName)
{
    pos = p;
    siteNames.assign(p.size(), siteName);
    computeMatrices();
}

// computeDistance / computeMatrices, src/FHLattice.cpp:516-539, 777-825
void FHLattice::computeMatrices()
{
    const size_t n = pos.size();
    dist.assign(n * n, 0.0);
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
            const double dx = pos[i][0] - pos[j][0], dy = pos[i][1] - pos[j][1], dz = pos[i][2] - pos[j][2];
            double d = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (periodic) {
                for (int zs = -1; zs < 2; ++zs)
                    for (int ys = -1; ys < 2; ++ys)
                        for (int xs = -1; xs < 2; ++xs) {
                            const double ex = dx + xs * latticeMatrix[0][0] + ys * latticeMatrix[0][1] + zs * latticeMatrix[0][2];
                            const double ey = dy + xs * latticeMatrix[1][0] + ys * latticeMatrix[1][1] + zs * latticeMatrix[1][2];
                            const double ez = dz + xs * latticeMatrix[2][0] + ys * latticeMatrix[2][1] + zs * latticeMatrix[2][2];
                            d = std::min(d, std::sqrt(ex * ex + ey * ey + ez * ez));
                        }
            }
            dist[i * n + j] = d;
        }
}

bool FHLattice::readPositions(const std::string& path, std::string& err)
{
    std::ifstream f(path);
    if (!f.is_open()) { err = "problem with the site position file " + path; return false; }
    std::string line;
    if (!std::getline(f, line)) { err = "empty xyz file " + path; return false; }
    long announced = -1;
    try { announced = std::stol(line); } catch (...) { err = "bad site count in " + path; return false; }
    std::getline(f, line);   // comment
    std::vector<Vec3> p;
    std::vector<std::string> names;
    while (std::getline(f, line)) {
        std::stringstream ss(line);
        std::string nm;
        if (!(ss >> nm)) continue;    // blank line
        std::vector<double> c;
        std::string tok;
        while (ss >> tok) {
            try { c.push_back(std::stod(tok)); } catch (...) { err = "bad coordinate in " + path; return false; }
        }
        c.resize(3, 0.0);
        p.push_back({c[0], c[1], c[2]});
        names.push_back(nm);
    }
    if ((long)p.size() != announced) {
        err = "problem in the xyz file: " + std::to_string(announced) + " sites announced, " + std::to_string(p.size()) + " found";
        return false;
    }
    pos = p;
    siteNames = names;
    computeMatrices();
    return true;
}

// writePositions, src/FHLattice.cpp:715-737
bool FHLattice::writePositions(const std::string& baseName, const std::string& folder, std::string& err) const
{
    std::string path = baseName + ".xyz";
    if (!folder.empty()) path = folder + "/" + path;
    std::ofstream f(path);
    if (!f.is_open()) { err = "cannot write " + path; return false; }
    f << pos.size() << std::endl;
    f.precision(6);
    for (size_t i = 0; i < pos.size(); ++i)
        f << std::endl << siteNames[i] << "\t" << pos[i][0] << "\t" << pos[i][1] << "\t" << pos[i][2];
    return true;
}

Json FHLattice::toJson() const
{
    Json j = Json::object();
    j["latticeType"] = type;
    j["positionsFile"] = name + ".xyz";
    j["periodic"] = periodic;
    Json m = Json::array();
    for (int r = 0; r < 3; ++r) {
        Json row = Json::array();
        for (int c = 0; c < 3; ++c) row.append(latticeMatrix[r][c]);
        m.append(row);
    }
    j["latticeMatrix"] = m;
    Json z = Json::array();
    for (int c = 0; c < 3; ++c) z.append(latticeZero[c]);
    j["latticeZero"] = z;
    return j;
}

bool FHLattice::fromJson(const Json& root, const std::string& folder, FHLattice& out, std::string& err)
{
    out = FHLattice();
    std::string file = root.get("positionsFile", "").asString();
    if (!folder.empty()) file = folder + "/" + file;
    out.type = root.get("latticeType", "none").asString();
    out.periodic = root.get("periodic", false).asBool();
    const Json& m = root["latticeMatrix"];
    if (!m.isNull())
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) out.latticeMatrix[i][j] = m[i][j].asDouble();
    const Json& z = root["latticeZero"];
    if (!z.isNull())
        for (int j = 0; j < 3; ++j) out.latticeZero[j] = z[j].asDouble();
    const bool per = out.periodic;
    out.periodic = false;            // the xyz read computes open distances first
    if (!out.readPositions(file, err)) return false;
    out.periodic = per;
    if (per) out.computeMatrices();
    return true;
}

bool FHLattice::generate(const std::string& type, std::vector<double> prm, FHLattice& out, std::string& err)
{
    out = FHLattice();
    while (prm.size() < 5) prm.push_back(1.0);
    out.type = type;
    std::vector<Vec3> p;
    const double s3 = std::sqrt(3.0);
    if (type == "grid") {
        const unsigned nx = (unsigned)prm[0], ny = (unsigned)prm[1], nz = (unsigned)prm[2];
        const double a = prm[3];
        p = make_grid(nx, ny, nz, a);
        const double b[3][3] = {{nx * a, 0, 0}, {0, ny * a, 0}, {0, 0, nz * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "bcc") {
        const unsigned nx = (unsigned)prm[0], ny = (unsigned)prm[1], nz = (unsigned)prm[2];
        const double a = prm[3];
        p = make_bcc(nx, ny, nz, a);
        const double b[3][3] = {{nx * a, 0, 0}, {0, ny * a, 0}, {0, 0, nz * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a / s3;
    } else if (type == "fcc") {
        const unsigned nx = (unsigned)prm[0], ny = (unsigned)prm[1], nz = (unsigned)prm[2];
        const double a = prm[3];
        p = make_fcc(nx, ny, nz, a);
        const double b[3][3] = {{nx * a, 0, 0}, {0, ny * a, 0}, {0, 0, nz * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a / std::sqrt(2.0);
    } else if (type == "fccPeriodic") {
        const unsigned nx = (unsigned)prm[0], ny = (unsigned)prm[1], nz = (unsigned)prm[2];
        const double a = prm[3];
        p = make_fcc_periodic(nx, ny, nz, a);
        const double b[3][3] = {{nx * a, 0, 0}, {0, ny * a, 0}, {0, 0, nz * a}};
        set_box(out.latticeMatrix, b);
        out.periodic = true;
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a / std::sqrt(2.0);
    } else if (type == "honeyCombs") {
        const unsigned nc = (unsigned)prm[0];
        const double a = prm[1];
        p = make_honeycombs(nc, a);
        const double sq = std::sqrt((double)nc);
        const unsigned fs = (unsigned)std::floor(sq), csq = (unsigned)std::ceil(sq);
        const unsigned nx = csq, ny = fs + (unsigned)((nc - fs * fs) > fs);
        const double b[3][3] = {{s3 * a * nx, s3 / 2 * a * ny, 0}, {0, 1.5 * a * ny, 0}, {0, 0, 10 * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "triangular") {
        const int nx = (int)prm[0], ny = (int)prm[1], nz = (int)prm[2];
        const double a = prm[3];
        p = make_tetragones(nx, ny, nz, a);
        const double b[3][3] = {{a * nx, a / 2 * ny, a / 2 * nz},
                                {0, s3 * a / 2 * ny, a / (2 * s3) * nz},
                                {0, 0, std::sqrt(2.0) * a / s3 * nz}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "graphene") {
        const int nx = (int)prm[0], ny = (int)prm[1];
        const double a = prm[2];
        p = make_graphene(nx, ny, a);
        const double b[3][3] = {{s3 * a * nx, s3 / 2 * a * ny, 0}, {0, 1.5 * a * ny, 0}, {0, 0, 10 * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "moire") {
        const int nx = (int)prm[0], ny = (int)prm[1];
        const double a = prm[2], bb = prm[3], th = prm[4];
        p = make_moire(nx, ny, a, bb, th);
        const double b[3][3] = {{s3 * a * nx, s3 / 2 * a * ny, 0}, {0, 1.5 * a * ny, 0}, {0, 0, 10 * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "kagome") {
        const unsigned nx = (unsigned)prm[0], ny = (unsigned)prm[1];
        const double a = prm[2];
        p = make_kagome(nx, ny, a);
        const double b[3][3] = {{2 * a * nx, a * ny, 0}, {0, s3 * a * ny, 0}, {0, 0, 10 * a}};
        set_box(out.latticeMatrix, b);
        out.samePointDistance = 1e-6 * a; out.neighbourDistance = a;
    } else if (type == "none") {
        p = make_grid(2, 1, 1, 1);
    } else {
        err = "unknown lattice type " + type;
        return false;
    }
    out.setPositions(p, "C");
    return true;
}

}  // namespace fps
