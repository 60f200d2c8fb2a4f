// shard.h — trajectory shards across processes (one per GPU) for the fTWA solver.
//
// The reference's MPI solver (src/FHfTWAMPISolver.cpp) splits the nTraj trajectories
// into contiguous ranges, one per rank (:89-100: nTraj / world each, the last
// nTraj % world ranks one more), and gathers the observables to rank 0 with one
// MPI_Send / MPI_Recv per array (:368-558).  Here each rank draws its range of the
// seeded ensemble (fpsg_sample_range), integrates it on its own GPU, and the ranks
// sum their trajectory-weighted observables in one exchange over TCP (the data is
// a few MB at most): rank 0 receives every other rank's buffer, sums the buffers in
// rank order (a fixed order, so the result does not depend on arrival order) and
// sends the sum back.  Every wait is bounded by a deadline, so a rank that never
// arrives ends the job with an error instead of a hang.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace fps {

struct ShardEnv {
    int rank = 0, world = 1, local = 0;
    std::string addr = "127.0.0.1";
    int port = 29517;
    double timeout_s = 600.0;

    // RANK / WORLD_SIZE / LOCAL_RANK / MASTER_ADDR (torchrun) or OMPI_COMM_WORLD_*
    // (mpirun); the exchange port is FPS_SHARD_PORT, else MASTER_PORT + 1 (torchrun's
    // own store holds MASTER_PORT), else 29517; FPS_SHARD_TIMEOUT (seconds) bounds it.
    static ShardEnv fromEnvironment();
};

// [first, end) of rank's trajectories (src/FHfTWAMPISolver.cpp:89-100)
void shardRange(long long nTraj, int rank, int world, long long& first, long long& end);

// Element-wise sum of `data` over all ranks, in rank order, left in `data` on every
// rank.  0 on success; otherwise an error code with the reason in `err`.
int shardSum(const ShardEnv& env, std::vector<double>& data, std::string& err);

}  // namespace fps
