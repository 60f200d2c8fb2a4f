// solver.cpp — FHSolver / FHfTWASolver / FHHFSolver over libfpsg, the result
// writer and the `fps` driver.
#include "solver.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>

#include "fpsg.h"

namespace fps {

static const char* kFpsVersion = "0.5.0";   // FPS_VERSION, include/FHSystem.h:21-23

EngineOptions EngineOptions::fromJson(const Json& g)
{
    EngineOptions o;
    if (!g.isObject()) return o;
    const std::string p = g.get("precision", "fp64").asString();
    o.precision = p == "fp32" ? FPSG_PREC_FP32
                : p == "bf16x3" ? FPSG_PREC_SPLIT_BF16X3
                : p == "tf32x3" ? FPSG_PREC_SPLIT_TF32X3 : FPSG_PREC_FP64;
    const std::string path = g.get("path", "auto").asString();
    o.path = path == "stream" ? FPSG_PATH_STREAM
           : path == "resident" ? FPSG_PATH_RESIDENT
           : path == "dense" ? FPSG_PATH_DENSE : FPSG_PATH_AUTO;
    o.device = (int)g.get("device", 0).asInt();
    o.seed = (unsigned long long)g.get("seed", 0).asInt();
    o.computedEnergies = g.get("fTWAEnergies", "reference").asString() == "computed";
    return o;
}

FHSolver::~FHSolver()
{
    if (ctx) fpsg_destroy(ctx);
}

void FHSolver::setResultFile(const std::string& w, const std::string& f)
{
    workName = w;
    folderName = f;
    talkative = false;
}

void FHSolver::setResultsWriter(const std::string& how, bool yn)
{
    if (how == "txt") writeResultsTxt = yn;
    if (how == "json") writeResultsJson = yn;
}

// src/FHSolver.cpp:34-45
void FHSolver::setResultsToSave(const Json& res)
{
    saveDiagDMatrix = res.get("diagDMatrix", true).asBool();
    saveDiag2DMatrix = res.get("diag2DMatrix", false).asBool();
    saveNiuNid = res.get("onSiteDoublons", false).asBool();
    saveWholeDMatrix = res.get("wholeDMatrix", false).asBool();
    saveEnergies = res.get("energies", true).asBool();
    saveTBStates = res.get("tbStates", false).asBool();
    saveMFStates = res.get("mfStates", false).asBool();
}

void FHSolver::setSaveTBStates(bool yn)
{
    saveTBStates = yn;
    if (yn && !sys->tbComputed) sys->computeTBGroundState();
}

void FHSolver::setSaveMFStates(bool yn)
{
    saveMFStates = yn;
    if (yn && !sys->mfComputed) sys->computeMFGroundState();
}

// src/FHSolver.cpp:95-101
void FHSolver::setTimeParameters(double t_max, double d_t, unsigned nPerTS)
{
    tMax = t_max;
    dt = d_t;
    nStepsPerTimePoint = nPerTS;
    nTimePoints = (unsigned)std::floor(tMax / dt + 1);
}

int FHSolver::fail(int code, const std::string& msg)
{
    status_ = code;
    error_ = msg;
    std::cerr << "fps: " << msg << std::endl;
    return code;
}

int FHSolver::openEngine()
{
    if (ctx) return FPSG_OK;
    int rc = fpsg_create(&ctx, engine.device, 0);
    if (rc != FPSG_OK) return fail(rc, "no CUDA device for the trajectory engine (fpsg_create: " + std::to_string(rc) + ")");
    const int n = sys->n;
    std::vector<double> T(2 * (size_t)n * n, 0.0), U(T.size(), 0.0), V(T.size(), 0.0), E(T.size(), 0.0);
    for (size_t q = 0; q < (size_t)n * n; ++q) {
        T[2 * q] = sys->tM[q];
        U[2 * q] = sys->U[q];
        V[2 * q] = sys->V[q];
        E[2 * q] = sys->ext[q];
    }
    rc = fpsg_set_system(ctx, n, T.data(), U.data(), V.data(), sys->extNull ? nullptr : E.data(), sys->coulomb,
                         sys->extNull ? 1 : 0);
    if (rc != FPSG_OK) return fail(rc, std::string("fpsg_set_system: ") + fpsg_last_error(ctx));
    return FPSG_OK;
}

std::complex<double> FHSolver::wholeAt(int spin, int t, int i, int j) const
{
    const int n = sys->n;
    const std::vector<double>& w = spin ? wholeD : wholeU;
    const size_t q = (size_t)t * n * n + (size_t)j * n + i;
    return {w[2 * q], w[2 * q + 1]};
}

// diag(V^T N(t) V) for every snapshot; V real (lattice sites), extended by the
// identity on a core-hole orbital
void FHSolver::statesFromWhole(const std::vector<double>& Vr, int nr, int spin, std::vector<double>& out) const
{
    const int n = sys->n, Tp = (int)nTimePoints;
    auto Vx = [&](int i, int k) -> double {
        if (i < nr && k < nr) return Vr[(size_t)k * nr + i];
        return i == k ? 1.0 : 0.0;
    };
    out.assign((size_t)n * Tp, 0.0);
    for (int t = 0; t < Tp; ++t)
        for (int k = 0; k < n; ++k) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) {
                const double vjk = Vx(j, k);
                if (vjk == 0.0) continue;
                double c = 0.0;
                for (int i = 0; i < n; ++i) c += Vx(i, k) * wholeAt(spin, t, i, j).real();
                s += c * vjk;
            }
            out[(size_t)k * Tp + t] = s;
        }
}

static Json line_real(const std::vector<double>& a, int row, int Tp)
{
    Json r = Json::array();
    for (int t = 0; t < Tp; ++t) r.append(a[(size_t)row * Tp + t]);
    return r;
}

static Json line_complex(const std::vector<std::complex<double>>& v)
{
    Json c = Json::object(), re = Json::array(), im = Json::array();
    for (const auto& z : v) { re.append(z.real()); im.append(z.imag()); }
    c["r"] = re;
    c["i"] = im;
    return c;
}

// FHSolver::writeResults, src/FHSolver.cpp:171-307
bool FHSolver::writeResults()
{
    if (!writeResultsJson) return true;
    const int n = sys->n, Tp = (int)nTimePoints;
    Json res = jsonFile;
    if (!res.isObject()) res = Json::object();
    res["fpsVersion"] = kFpsVersion;
    if (sys->tbComputed) res["tbGroundState"] = sys->tbGroundStateJson();
    if (sys->mfComputed) res["mfGroundState"] = sys->mfGroundStateJson();
    Json sim = Json::object();
    Json tl = Json::array();
    for (double t : timeLine) tl.append(t);
    sim["t"] = tl;
    auto site_block = [&](const std::vector<double>& a) {
        Json arr = Json::array();
        for (int i = 0; i < n; ++i) arr.append(line_real(a, i, Tp));
        return arr;
    };
    if (saveWholeDMatrix && !wholeU.empty()) {
        std::vector<std::complex<double>> u, d;
        for (int t = 0; t < Tp; ++t) { u.push_back(wholeAt(0, t, 0, n - 1)); d.push_back(wholeAt(1, t, 0, n - 1)); }
        sim["N1hu"] = line_complex(u);
        sim["N1hd"] = line_complex(d);
    }
    if (saveDiagDMatrix) { sim["Niiu"] = site_block(Niiu); sim["Niid"] = site_block(Niid); }
    if (saveDiag2DMatrix) { sim["N2iiu"] = site_block(N2iiu); sim["N2iid"] = site_block(N2iid); }
    if (saveNiuNid) sim["NuNd"] = site_block(NiuNid);
    if (saveTBStates && !Mkku.empty()) { sim["Mkku"] = site_block(Mkku); sim["Mkkd"] = site_block(Mkkd); }
    if (saveMFStates && !Mukku.empty()) { sim["Mukku"] = site_block(Mukku); sim["Mukkd"] = site_block(Mukkd); }
    if (saveEnergies) {
        Json E = Json::object();
        E["tH"] = line_real(Energies, 0, Tp);
        E["U"] = line_real(Energies, 1, Tp);
        E["V"] = line_real(Energies, 2, Tp);
        E["pe"] = line_real(Energies, 3, Tp);
        E["tot"] = line_real(Energies, 4, Tp);
        sim["E"] = E;
    }
    if (sys->hasCoreHole) {
        Json c = Json::object();
        c["u"] = line_complex(NiCHu);
        c["d"] = line_complex(NiCHd);
        sim["NiCh"] = c;
    }
    res["simulation"] = sim;
    resultPath_ = folderName + workName + ".json";
    std::ofstream f(resultPath_);
    if (!f.is_open()) { fail(FPSG_ERR_INVALID, "cannot write " + resultPath_); return false; }
    f << res.styled();
    std::cout << "   -- Results written in " << resultPath_ << std::endl;
    return true;
}

// ------------------------------------------------------------------ fTWA
void FHfTWASolver::setIntegratorOrder(int order)
{
    integratorOrder = (order == 4) ? 4 : 2;
}

void FHfTWASolver::setMethodParameters(const Json& p)
{
    const double d = p.get("dt", 0.01).asDouble();
    const double tm = p.get("t_max", 2).asDouble();
    const int s = (int)p.get("stepsParTimePoints", 1).asInt();   // this exact key (src/FHfTWASolver.cpp:53)
    const int nt = (int)p.get("n_traj", 10).asInt();
    const int io = (int)p.get("int_order", 2).asInt();
    setTimeParameters(tm, d, (unsigned)std::max(1, s));
    setIntegratorOrder(io);
    setfTWAParameters((unsigned)std::max(0, nt));
}

int FHfTWASolver::initiateSolver()
{
    status_ = 0;
    if (saveTBStates && !sys->tbComputed) sys->computeTBGroundState();
    if (saveMFStates && !sys->mfComputed) sys->computeMFGroundState();
    const int N = sys->nLatticeSites(), n = sys->n;
    initialDiagU.assign(n, 0.0);
    initialDiagD.assign(n, 0.0);
    rotU.clear();
    rotD.clear();
    auto complexRot = [&](const std::vector<double>& Vr) {
        std::vector<double> R(2 * (size_t)n * n, 0.0);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double v = (i < N && j < N) ? Vr[(size_t)j * N + i] : (i == j ? 1.0 : 0.0);
                R[2 * ((size_t)j * n + i)] = v;
            }
        return R;
    };
    if (sys->icType == "givenDiagonal") {
        for (int i = 0; i < N; ++i) { initialDiagU[i] = sys->occUp[i]; initialDiagD[i] = sys->occDn[i]; }
    } else if (sys->icType == "tbGroundState" || sys->icType == "mfGroundState") {
        const bool tb = sys->icType == "tbGroundState";
        if (tb && !sys->tbComputed) sys->computeTBGroundState();
        if (!tb && !sys->mfComputed) sys->computeMFGroundState();
        for (unsigned i = 0; i < sys->nPartUp && (int)i < N; ++i) initialDiagU[i] = 1.0;
        for (unsigned i = 0; i < sys->nPartDn && (int)i < N; ++i) initialDiagD[i] = 1.0;
        rotU = complexRot(tb ? sys->tbV : sys->mfVu);
        rotD = complexRot(tb ? sys->tbV : sys->mfVd);
    } else {
        return fail(FPSG_ERR_INVALID, "fTWA needs an initial condition (system.IC)");
    }
    if (sys->hasCoreHole) {
        initialDiagU[n - 1] = sys->coreHole.occUp;
        initialDiagD[n - 1] = sys->coreHole.occDn;
    }
    return FPSG_OK;
}

int FHfTWASolver::runSimulation()
{
    std::cout << "   -- Start simulation." << std::endl;
    if (nTraj < 1) return fail(FPSG_ERR_INVALID, "n_traj must be at least 1");
    const bool sharded = shard.world > 1;
    long long first = 0, end = nTraj;
    if (sharded) {
        shardRange((long long)nTraj, shard.rank, shard.world, first, end);
        engine.device = shard.local;                     // one GPU per rank
        std::cout << "   -- Shard " << shard.rank << " of " << shard.world << " will compute trajectories from "
                  << first << " to " << end - 1 << std::endl;
    }
    const int Bloc = (int)(end - first);
    int rc = FPSG_OK;
    if (Bloc > 0 && (rc = openEngine())) return rc;
    const int n = sys->n, Tp = (int)nTimePoints;
    if (Bloc > 0) {
        rc = fpsg_sample_range(ctx, first, Bloc, engine.seed, initialDiagU.data(), initialDiagD.data(),
                               rotU.empty() ? nullptr : rotU.data(), rotD.empty() ? nullptr : rotD.data());
        if (rc) return fail(rc, std::string("fpsg_sample_range: ") + fpsg_last_error(ctx));
    }
    const bool needWhole = saveWholeDMatrix || saveTBStates || saveMFStates || sys->hasCoreHole;
    uint32_t mask = FPSG_OBS_DIAG | FPSG_OBS_DIAG2 | FPSG_OBS_DOUBLONS | FPSG_OBS_ENERGIES;
    if (needWhole) mask |= FPSG_OBS_WHOLE;
    Niiu.assign((size_t)n * Tp, 0.0); Niid = Niiu; N2iiu = Niiu; N2iid = Niiu; NiuNid = Niiu;
    Energies.assign((size_t)5 * Tp, 0.0);
    timeLine.assign(Tp, 0.0);
    if (needWhole) { wholeU.assign(2 * (size_t)Tp * n * n, 0.0); wholeD = wholeU; }
    fpsg_outputs o = {};
    o.time = timeLine.data();
    o.niiu = Niiu.data(); o.niid = Niid.data(); o.n2iiu = N2iiu.data(); o.n2iid = N2iid.data(); o.nund = NiuNid.data();
    o.energies = Energies.data();
    o.whole_u = needWhole ? wholeU.data() : nullptr;
    o.whole_d = needWhole ? wholeD.data() : nullptr;
    if (Bloc > 0) {
        rc = fpsg_run(ctx, FPSG_METHOD_FTWA, engine.precision, engine.path, dt, (int)nStepsPerTimePoint, Tp, mask, &o);
        if (rc) return fail(rc, std::string("fpsg_run: ") + fpsg_last_error(ctx));
    } else {
        for (int t = 0; t < Tp; ++t) timeLine[t] = t * dt;
    }
    deviceMs_ = o.device_ms;
    trajSteps_ = o.traj_steps;
    if (sharded) {
        // the one exchange of the sharded run: each rank's normalised observables are
        // affine in its trajectory sums with the same constant (Niiu = S/B + 1/2, ...),
        // so the ensemble value is the trajectory-weighted mean sum_r B_r x_r / nTraj
        std::vector<std::vector<double>*> parts = {&Niiu, &Niid, &N2iiu, &N2iid, &NiuNid, &Energies};
        if (needWhole) { parts.push_back(&wholeU); parts.push_back(&wholeD); }
        std::vector<double> buf;
        for (auto* v : parts)
            for (double x : *v) buf.push_back(x * (double)Bloc);
        std::string why;
        if (shardSum(shard, buf, why) != 0) return fail(FPSG_ERR_INVALID, "trajectory shards: " + why);
        size_t q = 0;
        for (auto* v : parts)
            for (double& x : *v) x = buf[q++] / (double)nTraj;
        std::cout << "   -- Observables summed over " << shard.world << " shards" << std::endl;
    }
    // the reference merges the energy sums only for core-hole systems
    if (!sys->hasCoreHole && !engine.computedEnergies) std::fill(Energies.begin(), Energies.end(), 0.0);
    if (saveTBStates) {
        statesFromWhole(sys->tbV, sys->nLatticeSites(), 0, Mkku);
        statesFromWhole(sys->tbV, sys->nLatticeSites(), 1, Mkkd);
    }
    if (saveMFStates) {
        statesFromWhole(sys->mfVu, sys->nLatticeSites(), 0, Mukku);
        statesFromWhole(sys->mfVd, sys->nLatticeSites(), 1, Mukkd);
    }
    if (sys->hasCoreHole) {
        NiCHu.assign(Tp, 0.0); NiCHd.assign(Tp, 0.0);
        for (int t = 0; t < Tp; ++t) {
            NiCHu[t] = wholeAt(0, t, (int)sys->coreHole.site, n - 1);
            NiCHd[t] = wholeAt(1, t, (int)sys->coreHole.site, n - 1);
        }
    }
    if (!sharded || shard.rank == 0) writeResults();
    return status_;
}

// ------------------------------------------------------------------ HF
void FHHFSolver::setIntegratorOrder(int order)
{
    integratorOrder = (order == 1 || order == 4) ? order : 2;
}

void FHHFSolver::setMethodParameters(const Json& p)
{
    const double d = p.get("dt", 0.01).asDouble();
    const double tm = p.get("t_max", 2).asDouble();
    const int s = (int)p.get("stepsParTimePoints", 1).asInt();
    setTimeParameters(tm, d, (unsigned)std::max(1, s));
    setIntegratorOrder((int)p.get("int_order", 2).asInt());
}

int FHHFSolver::initiateSolver()
{
    status_ = 0;
    const int N = sys->nLatticeSites(), n = sys->n;
    N0u.assign(2 * (size_t)n * n, 0.0);
    N0d = N0u;
    auto put = [&](std::vector<double>& M, const std::vector<double>& src) {
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) M[2 * ((size_t)j * n + i)] = src[(size_t)j * N + i];
    };
    if (sys->icType == "givenDiagonal") {
        for (int i = 0; i < N; ++i) {
            N0u[2 * ((size_t)i * n + i)] = sys->occUp[i];
            N0d[2 * ((size_t)i * n + i)] = sys->occDn[i];
        }
    } else if (sys->icType == "tbGroundState") {
        if (!sys->tbComputed) sys->computeTBGroundState();
        put(N0u, sys->tbNu);
        put(N0d, sys->tbNd);
    } else if (sys->icType == "mfGroundState") {
        if (!sys->mfComputed) sys->computeMFGroundState();
        put(N0u, sys->mfNu);
        put(N0d, sys->mfNd);
    } else {
        return fail(FPSG_ERR_INVALID, "No initial condition found.");
    }
    if (saveTBStates && !sys->tbComputed) sys->computeTBGroundState();
    if (saveMFStates && !sys->mfComputed) sys->computeMFGroundState();
    if (sys->hasCoreHole) {
        N0u[2 * ((size_t)(n - 1) * n + (n - 1))] = sys->coreHole.occUp;
        N0d[2 * ((size_t)(n - 1) * n + (n - 1))] = sys->coreHole.occDn;
    }
    return FPSG_OK;
}

int FHHFSolver::runSimulation()
{
    std::cout << "   -- Start simulation." << std::endl;
    int rc = openEngine();
    if (rc) return rc;
    const int n = sys->n, Tp = (int)nTimePoints;
    std::vector<double> rho0(N0u);
    rho0.insert(rho0.end(), N0d.begin(), N0d.end());
    rc = fpsg_set_initial_samples(ctx, 1, rho0.data());
    if (rc) return fail(rc, std::string("fpsg_set_initial_samples: ") + fpsg_last_error(ctx));
    const bool needWhole = saveWholeDMatrix || saveTBStates || saveMFStates || sys->hasCoreHole;
    uint32_t mask = FPSG_OBS_DIAG | FPSG_OBS_DIAG2 | FPSG_OBS_DOUBLONS | FPSG_OBS_ENERGIES;
    if (needWhole) mask |= FPSG_OBS_WHOLE;
    Niiu.assign((size_t)n * Tp, 0.0); Niid = Niiu; N2iiu = Niiu; N2iid = Niiu; NiuNid = Niiu;
    Energies.assign((size_t)5 * Tp, 0.0);
    timeLine.assign(Tp, 0.0);
    if (needWhole) { wholeU.assign(2 * (size_t)Tp * n * n, 0.0); wholeD = wholeU; }
    fpsg_outputs o = {};
    o.time = timeLine.data();
    o.niiu = Niiu.data(); o.niid = Niid.data(); o.n2iiu = N2iiu.data(); o.n2iid = N2iid.data(); o.nund = NiuNid.data();
    o.energies = Energies.data();
    o.whole_u = needWhole ? wholeU.data() : nullptr;
    o.whole_d = needWhole ? wholeD.data() : nullptr;
    rc = fpsg_run(ctx, FPSG_METHOD_HF, FPSG_PREC_FP64, engine.path, dt, (int)nStepsPerTimePoint, Tp, mask, &o);
    if (rc) return fail(rc, std::string("fpsg_run: ") + fpsg_last_error(ctx));
    deviceMs_ = o.device_ms;
    trajSteps_ = o.traj_steps;
    if (saveTBStates) {
        statesFromWhole(sys->tbV, sys->nLatticeSites(), 0, Mkku);
        statesFromWhole(sys->tbV, sys->nLatticeSites(), 1, Mkkd);
    }
    if (saveMFStates) {
        statesFromWhole(sys->mfVu, sys->nLatticeSites(), 0, Mukku);
        statesFromWhole(sys->mfVd, sys->nLatticeSites(), 1, Mukkd);
    }
    if (sys->hasCoreHole) {            // recorded from t = 1 on (src/FHHFSolver.cpp:393-398)
        NiCHu.assign(Tp, 0.0); NiCHd.assign(Tp, 0.0);
        for (int t = 1; t < Tp; ++t) {
            NiCHu[t] = wholeAt(0, t, (int)sys->coreHole.site, n - 1);
            NiCHd[t] = wholeAt(1, t, (int)sys->coreHole.site, n - 1);
        }
    }
    writeResults();
    return status_;
}

// ------------------------------------------------------------------ fps
int run_fps(const std::string& path, std::string& err, bool quiet)
{
    (void)quiet;
    const size_t slash = path.find_last_of('/');
    std::string folder = (slash == std::string::npos) ? "" : path.substr(0, slash + 1);
    std::cout << "== Loading data : " << std::endl;
    std::cout << "   -- Work file : " << path.substr(slash == std::string::npos ? 0 : slash + 1) << std::endl;
    std::cout << "   -- Work folder : " << folder << std::endl;
    Json root;
    if (!Json::parseFile(path, root, err)) return 1;
    const std::string simName = root.get("sim_name", "defaultSimName").asString();
    const std::string method = root.get("method", "HF").asString();
    FHSystem sys;
    if (!FHSystem::fromJson(root.get("system", Json()), folder, sys, err)) return 1;
    std::cout << "   -- System loaded" << std::endl;
    const EngineOptions eo = EngineOptions::fromJson(root["gpu"]);
    const auto t0 = std::chrono::steady_clock::now();
    int rc = 0;
    if (method == "GPSR" || method == "ED" || method == "fTWA_GS") {
        err = "method " + method + " is not part of this engine (fTWA and HF only)";
        return 2;
    }
    if (method == "fTWA") {
        std::cout << "== Computation of fTWA dynamic " << std::endl;
        FHfTWASolver s(&sys);
        s.setEngineOptions(eo);
        s.setShard(ShardEnv::fromEnvironment());
        s.setResultFile(simName + "_fTWA_res", folder);
        s.setJsonFile(root);
        s.setResultsWriter("json");
        s.setResultsToSave(root["results"]);
        s.setMethodParameters(root["parameters"]);
        rc = s.initiateSolver();
        if (!rc) rc = s.runSimulation();
        if (rc) err = s.error();
    } else {
        // fps.cpp:155-162: any other name runs HF; HF is one deterministic density
        // matrix, so under several ranks rank 0 alone computes it
        const ShardEnv se = ShardEnv::fromEnvironment();
        if (se.world > 1 && se.rank != 0) {
            std::cout << "== HF runs on rank 0 only (rank " << se.rank << " has nothing to do)" << std::endl;
            return 0;
        }
        std::cout << "== Computation of HF dynamic " << std::endl;
        FHHFSolver s(&sys);
        s.setEngineOptions(eo);
        s.setResultFile(simName + "_HF_res", folder);
        s.setJsonFile(root);
        s.setResultsWriter("json");
        s.setResultsToSave(root["results"]);
        s.setMethodParameters(root["parameters"]);
        rc = s.initiateSolver();
        if (!rc) rc = s.runSimulation();
        if (rc) err = s.error();
    }
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "== Computation time : " << el << " s." << std::endl;
    return rc ? 1 : 0;
}

}  // namespace fps
