// solver.h — FermiPhaseSpace's solver interface on top of the GPU engine.
//
// FHSolver / FHfTWASolver / FHHFSolver keep the public methods the reference's
// `fps` calls (include/FHSolver.h:23-47, include/FHfTWASolver.h:28-44,
// include/FHHFSolver.h:31-47): setResultFile, setJsonFile, setResultsWriter,
// setResultsToSave, setMethodParameters, initiateSolver, runSimulation.  The
// trajectory loop itself runs in libfpsg.so through the C ABI of include/fpsg.h.
//
// Extension (ignored by the reference, so input files stay interchangeable): a
// top-level "gpu" object with "precision" ("fp64" | "fp32" | "bf16x3" | "tf32x3",
// the last two on the tensor-core path), "path" ("auto" | "stream" | "resident" |
// "dense"), "device", "seed" and "fTWAEnergies" ("reference": the
// reference's output, energies all zero except for core-hole systems,
// src/FHfTWASolver.cpp:470-476; "computed": the energies it accumulates).
#pragma once

#include <complex>
#include <string>
#include <vector>

#include "json.h"
#include "shard.h"
#include "system.h"

struct fpsg_ctx;

namespace fps {

struct EngineOptions {
    int precision = 0;       // FPSG_PREC_FP64
    int path = 0;            // FPSG_PATH_AUTO
    int device = 0;
    unsigned long long seed = 0;
    bool computedEnergies = false;
    static EngineOptions fromJson(const Json& gpu);
};

class FHSolver {
public:
    explicit FHSolver(FHSystem* s) : sys(s) {}
    virtual ~FHSolver();

    void setResultFile(const std::string& workName, const std::string& folderName);
    void setResultsWriter(const std::string& how, bool yn = true);
    void setTimeParameters(double t_max, double dt, unsigned nPerTS = 1);
    void setTalkative(bool yn) { talkative = yn; }
    void setJsonFile(const Json& file) { jsonFile = file; }
    void setResultsToSave(const Json& res);
    void setSaveWholeDMatrix(bool yn) { saveWholeDMatrix = yn; }
    void setSaveDiagDMatrix(bool yn) { saveDiagDMatrix = yn; }
    void setSaveDiag2DMatrix(bool yn) { saveDiag2DMatrix = yn; }
    void setSaveEnergies(bool yn) { saveEnergies = yn; }
    void setSaveTBStates(bool yn);
    void setSaveMFStates(bool yn);
    void setEngineOptions(const EngineOptions& o) { engine = o; }

    // status of the last initiateSolver / runSimulation (0 = OK, else an FPSG_ERR_* code)
    int status() const { return status_; }
    const std::string& error() const { return error_; }
    double deviceMs() const { return deviceMs_; }
    long long trajSteps() const { return trajSteps_; }
    const std::string& resultPath() const { return resultPath_; }

protected:
    bool writeResults();
    int fail(int code, const std::string& msg);
    int openEngine();
    // ensemble-mean N(t) (n x n complex, col-major) from the engine's whole-matrix output
    std::complex<double> wholeAt(int spin, int t, int i, int j) const;
    void statesFromWhole(const std::vector<double>& Vrot, int nrot, int spin, std::vector<double>& out) const;

    FHSystem* sys;
    Json jsonFile = Json::object();
    bool writeResultsJson = false, writeResultsTxt = false;
    bool saveWholeDMatrix = false, saveDiagDMatrix = true, saveDiag2DMatrix = true, saveNiuNid = false;
    bool saveTBStates = false, saveMFStates = false, saveEnergies = true;
    std::string workName, folderName;
    bool talkative = false;
    double tMax = 1.0, dt = 0.01;
    unsigned nStepsPerTimePoint = 1, nTimePoints = 100;
    EngineOptions engine;

    // results, [site][time] unless noted
    std::vector<double> timeLine;
    std::vector<double> Niiu, Niid, N2iiu, N2iid, NiuNid, Mkku, Mkkd, Mukku, Mukkd;
    std::vector<double> Energies;               // [5][time]: tH, U, V, pe, tot
    std::vector<double> wholeU, wholeD;         // [time][n][n] complex interleaved
    std::vector<std::complex<double>> NiCHu, NiCHd;

    fpsg_ctx* ctx = nullptr;
    int status_ = 0;
    std::string error_;
    double deviceMs_ = 0.0;
    long long trajSteps_ = 0;
    std::string resultPath_;
};

class FHfTWASolver : public FHSolver {
public:
    explicit FHfTWASolver(FHSystem* s) : FHSolver(s) {}
    // Trajectory shards (the reference's MPI solver, src/FHfTWAMPISolver.cpp): with
    // world > 1 this process integrates its contiguous range of the seeded ensemble
    // on its own GPU, the ranks sum their observables, and rank 0 alone writes the
    // results.  world = 1 (the default) is the single-process solver.
    void setShard(const ShardEnv& e) { shard = e; }
    void setMethodParameters(const Json& param);     // src/FHfTWASolver.cpp:49-60
    void setIntegratorOrder(int order);              // accepted; RK4 3/8 is always used (:90)
    void setfTWAParameters(unsigned nT) { nTraj = nT; }
    int initiateSolver();                            // src/FHfTWASolver.cpp:74-213
    int runSimulation();                             // src/FHfTWASolver.cpp:222-556

protected:
    unsigned nTraj = 1;
    int integratorOrder = 2;
    ShardEnv shard;
    std::vector<double> initialDiagU, initialDiagD;
    std::vector<double> rotU, rotD;                  // complex interleaved n x n, empty = identity
};

class FHHFSolver : public FHSolver {
public:
    explicit FHHFSolver(FHSystem* s) : FHSolver(s) {}
    void setMethodParameters(const Json& param);     // src/FHHFSolver.cpp:50-58
    void setIntegratorOrder(int order);
    int initiateSolver();                            // src/FHHFSolver.cpp:61-174
    int runSimulation();                             // src/FHHFSolver.cpp:181-434

protected:
    int integratorOrder = 2;
    std::vector<double> N0u, N0d;                    // complex interleaved n x n
};

// the `fps` program (fps.cpp:26-282): returns 0 on success
int run_fps(const std::string& jsonPath, std::string& err, bool quiet = false);

}  // namespace fps
