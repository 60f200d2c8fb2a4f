// host_api.cpp — the C ABI of include/fps_host.h over the host classes.
#include <cstring>
#include <iostream>
#include <string>

#include "fps_host.h"
#include "json.h"
#include "shard.h"
#include "solver.h"
#include "system.h"

struct fpsh_system {
    fps::FHSystem sys;
};

namespace {
thread_local std::string g_err;

int set_err(const std::string& e)
{
    g_err = e;
    return -1;
}
}  // namespace

extern "C" {

const char* fpsh_last_error(void) { return g_err.c_str(); }

int fpsh_system_load(const char* json_path, fpsh_system** out)
{
    if (!json_path || !out) return set_err("null argument");
    *out = nullptr;
    try {
        const std::string path(json_path);
        const size_t slash = path.find_last_of('/');
        const std::string folder = (slash == std::string::npos) ? "" : path.substr(0, slash + 1);
        fps::Json root;
        std::string err;
        if (!fps::Json::parseFile(path, root, err)) return set_err(err);
        auto* s = new fpsh_system();
        if (!fps::FHSystem::fromJson(root.get("system", fps::Json()), folder, s->sys, err)) {
            delete s;
            return set_err(err);
        }
        *out = s;
        return 0;
    } catch (const std::exception& e) {
        return set_err(e.what());
    }
}

void fpsh_system_free(fpsh_system* s) { delete s; }

int fpsh_system_n(const fpsh_system* s) { return s ? s->sys.n : 0; }

int fpsh_system_matrices(const fpsh_system* s, double* tM, double* U, double* V, double* ext, int* flags)
{
    if (!s) return set_err("null system");
    const size_t nn = (size_t)s->sys.n * s->sys.n;
    if (tM) std::memcpy(tM, s->sys.tM.data(), nn * sizeof(double));
    if (U) std::memcpy(U, s->sys.U.data(), nn * sizeof(double));
    if (V) std::memcpy(V, s->sys.V.data(), nn * sizeof(double));
    if (ext) std::memcpy(ext, s->sys.ext.data(), nn * sizeof(double));
    if (flags) {
        flags[0] = s->sys.coulomb;
        flags[1] = s->sys.extNull ? 1 : 0;
        flags[2] = s->sys.hasCoreHole ? 1 : 0;
    }
    return 0;
}

int fpsh_system_occupations(const fpsh_system* s, double* up, double* dn)
{
    if (!s) return set_err("null system");
    const int N = s->sys.nLatticeSites();
    for (int i = 0; i < N; ++i) {
        if (up) up[i] = i < (int)s->sys.occUp.size() ? s->sys.occUp[i] : 0.0;
        if (dn) dn[i] = i < (int)s->sys.occDn.size() ? s->sys.occDn[i] : 0.0;
    }
    return 0;
}

int fpsh_system_ground_state(fpsh_system* s, int which, double* nu, double* nd, double* eu, double* ed)
{
    if (!s) return set_err("null system");
    fps::FHSystem& y = s->sys;
    if (y.nPartUp == 0 && y.nPartDn == 0) {
        const int N = y.nLatticeSites();
        y.nPartUp = (unsigned)((N + 1) / 2);
        y.nPartDn = (unsigned)(N / 2);
    }
    const int N = y.nLatticeSites();
    const size_t nn = (size_t)N * N;
    if (which == 0) {
        y.computeTBGroundState();
        if (nu) std::memcpy(nu, y.tbNu.data(), nn * sizeof(double));
        if (nd) std::memcpy(nd, y.tbNd.data(), nn * sizeof(double));
        if (eu) std::memcpy(eu, y.tbE.data(), N * sizeof(double));
        if (ed) std::memcpy(ed, y.tbE.data(), N * sizeof(double));
    } else {
        y.computeMFGroundState();
        if (nu) std::memcpy(nu, y.mfNu.data(), nn * sizeof(double));
        if (nd) std::memcpy(nd, y.mfNd.data(), nn * sizeof(double));
        if (eu) std::memcpy(eu, y.mfEu.data(), N * sizeof(double));
        if (ed) std::memcpy(ed, y.mfEd.data(), N * sizeof(double));
    }
    return 0;
}

int fpsh_system_positions(const fpsh_system* s, double* xyz)
{
    if (!s || !xyz) return set_err("null argument");
    for (int i = 0; i < s->sys.nLatticeSites(); ++i)
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = s->sys.lattice.pos[i][k];
    return 0;
}

int fpsh_run_fps(const char* json_path)
{
    if (!json_path) return set_err("null path");
    try {
        std::string err;
        const int rc = fps::run_fps(json_path, err);
        if (rc) set_err(err);
        return rc;
    } catch (const std::exception& e) {
        return set_err(e.what());
    }
}

// makeSitesSystem.cpp:49-221
int fpsh_make_sites_system(const char* name, const char* folder, const char* geometry, const double* params,
                           int n_params, const char* ic)
{
    if (!name || !geometry) return set_err("null argument");
    try {
        std::vector<double> prm(params ? params : nullptr, params ? params + n_params : nullptr);
        fps::FHLattice lat;
        std::string err;
        if (!fps::FHLattice::generate(geometry, prm, lat, err)) return set_err(err);
        lat.name = name;
        fps::FHSystem sys = fps::FHSystem::basis(lat);
        const std::string icn = ic ? ic : "ic_sw";
        sys.setInitialConditions(icn == "ic_cw" ? "chargeWave" : icn == "ic_tbgs" ? "tbGroundState"
                                 : icn == "ic_mfgs" ? "mfGroundState" : "spinWave");
        fps::Json root = fps::Json::object();
        root["sim_name"] = name;
        root["method"] = "HF";
        fps::Json p = fps::Json::object();
        p["t_max"] = 2.0;
        p["dt"] = 0.01;
        p["stepsPerTimePoints"] = 1;     // the key the reference generator writes (the solvers read stepsParTimePoints)
        p["n_traj"] = 1000;
        p["int_order"] = 4;
        root["parameters"] = p;
        fps::Json sj = sys.toJson();
        if (sys.tbComputed) sj["tbGroundState"] = sys.tbGroundStateJson();
        if (sys.mfComputed) sj["mfGroundState"] = sys.mfGroundStateJson();
        root["system"] = sj;
        fps::Json r = fps::Json::object();
        r["diagDMatrix"] = true;
        r["diag2DMatrix"] = false;
        r["onSiteDoublons"] = false;
        r["wholeDMatrix"] = false;
        r["tbStates"] = false;
        r["mfStates"] = false;
        r["energies"] = true;
        root["results"] = r;
        const std::string dir = folder ? folder : "systemsFolder";
        const std::string path = dir + "/" + name + ".json";
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) return set_err("cannot write " + path);
        const std::string doc = root.styled();
        std::fwrite(doc.data(), 1, doc.size(), f);
        std::fclose(f);
        if (!lat.writePositions(name, dir, err)) return set_err(err);
        std::cout << "== " << name << " system created with " << lat.nSites() << " sites and "
                  << sys.nPartUp + sys.nPartDn << " particles." << std::endl;
        return 0;
    } catch (const std::exception& e) {
        return set_err(e.what());
    }
}

int fpsh_shard_range(long long n_traj, int rank, int world, long long* first, long long* end)
{
    if (!first || !end || world < 1 || rank < 0 || rank >= world || n_traj < 0) return set_err("bad shard arguments");
    fps::shardRange(n_traj, rank, world, *first, *end);
    return 0;
}

int fpsh_shard_sum(const char* addr, int port, int rank, int world, double* data, long long count, double timeout_s)
{
    if ((!data && count > 0) || count < 0 || world < 1) return set_err("bad shard arguments");
    try {
        fps::ShardEnv e;
        e.rank = rank; e.world = world; e.port = port; e.timeout_s = timeout_s;
        if (addr) e.addr = addr;
        std::vector<double> v(data, data + count);
        std::string err;
        const int rc = fps::shardSum(e, v, err);
        if (rc) return set_err(err);
        std::copy(v.begin(), v.end(), data);
        return 0;
    } catch (const std::exception& ex) {
        return set_err(ex.what());
    }
}

}  // extern "C"
