/*
 * fps_host.h — C ABI of the host layer (libfpshost.so): the FermiPhaseSpace system
 * loader, the `fps` driver and the system generator, for callers outside C++
 * (Python tests and scripts).  The C++ classes themselves (FHSystem, FHLattice,
 * FHfTWASolver, FHHFSolver in fermiphasespace_b200/host) are the interface C++
 * callers use, as the reference's fps.cpp uses its own.
 */
#ifndef FPS_HOST_H
#define FPS_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fpsh_system fpsh_system;

/* Loads the "system" block of a simulation JSON file the way FHSystem(Json, folder)
 * does (src/FHSystem.cpp:123-326); the xyz file is resolved relative to the JSON
 * file's folder as fps.cpp does. 0 on success. */
int  fpsh_system_load(const char* json_path, fpsh_system** out);
void fpsh_system_free(fpsh_system* s);
/* orbitals per spin (lattice sites, plus one for a core hole) */
int  fpsh_system_n(const fpsh_system* s);
/* dense real n x n col-major matrices (any pointer may be NULL); flags[0] = Coulomb
 * kind (0 null, 1 onSite, 2 distance/given), flags[1] = external potential null,
 * flags[2] = core hole present */
int  fpsh_system_matrices(const fpsh_system* s, double* tM, double* U, double* V, double* ext, int* flags);
/* initial diagonal occupations of the lattice sites (givenDiagonal initial conditions) */
int  fpsh_system_occupations(const fpsh_system* s, double* occ_up, double* occ_dn);
/* which = 0: tight-binding ground state of tM (src/FHSystem.cpp:911-940);
 * which = 1: Hartree mean-field ground state (src/FHSystem.cpp:943-1019).
 * Densities (lattice x lattice, col-major) and single-particle energies; NULL skips. */
int  fpsh_system_ground_state(fpsh_system* s, int which, double* n_up, double* n_dn, double* e_up, double* e_dn);
/* site positions [n][3] */
int  fpsh_system_positions(const fpsh_system* s, double* xyz);

/* The fps program (fps.cpp:26-282) on one JSON file: 0 on success. */
int  fpsh_run_fps(const char* json_path);
/* makeSitesSystem (makeSitesSystem.cpp:49-221): writes <folder>/<name>.json and .xyz */
int  fpsh_make_sites_system(const char* name, const char* folder, const char* geometry, const double* params,
                            int n_params, const char* ic);
const char* fpsh_last_error(void);

/* Trajectory shards across processes (the reference's MPI solver,
 * src/FHfTWAMPISolver.cpp:89-100 and :368-558).  fpsh_shard_range gives
 * [first, end) of rank's trajectories (n_traj / world each, the last n_traj % world
 * ranks one more).  fpsh_shard_sum sums `count` doubles element-wise over `world`
 * processes through a TCP exchange at addr:port (rank 0 listens, receives every
 * other rank's buffer, sums in rank order and sends the sum back), leaving the sum
 * in `data` on every rank; every wait ends after timeout_s seconds with an error.
 * `fps` launched with WORLD_SIZE / RANK / LOCAL_RANK (torchrun) or OMPI_COMM_WORLD_*
 * (mpirun) in its environment shards an fTWA run this way (port FPS_SHARD_PORT,
 * else MASTER_PORT + 1) and rank 0 writes the results.  0 on success. */
int  fpsh_shard_range(long long n_traj, int rank, int world, long long* first, long long* end);
int  fpsh_shard_sum(const char* addr, int port, int rank, int world, double* data, long long count, double timeout_s);

#ifdef __cplusplus
}
#endif
#endif
