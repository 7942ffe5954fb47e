/*
 * rumd_b200.h -- C ABI of the B200-native RUMD time-step engine.
 *
 * One engine holds any number of independent MD systems ("replicas": a plain
 * Sample is an engine with one replica) resident in HBM on one GPU, and
 * advances all of them with the same fused kernels:
 *   neighbour-list rebuild (cell-key stable sort + sorted 5x5x5 cell scan),
 *   shifted-force / shifted-potential Lennard-Jones forces, energy and virial,
 *   Nose-Hoover leap-frog NVT update, FP64 reductions.
 *
 * Conventions
 *   - Every function returns B2MD_OK (0) or a B2MD_ERR_* code; the message of
 *     the last failure on the calling thread is b2md_last_error().  No C++
 *     exception crosses this boundary.
 *   - Particle arrays passed in or out are HOST arrays in the ORIGINAL
 *     particle order (RUMD's convention: host data is never sorted,
 *     src/ParticleData.cu:333-393), float32 with 4 components per particle:
 *       positions  [x, y, z, type bit-cast to float]  (ParticleData.h:41)
 *       velocities [vx, vy, vz, 1/m]                 (ParticleData.h:42)
 *       forces     [fx, fy, fz, u_i]  u_i already halved (PairPotential.cu:371)
 *       virials    [w_mol, s_xz, s_xy, w_i]  w_i = sum_j d^2 s (ParticleData.h:44)
 *       stresses   [s_xx, s_yy, s_zz, s_yz]           (ParticleData.h:46)
 *     Images are int32 [imx, imy, imz] per particle.
 *   - Parameter tables use RUMD's layout: float params[T][T][12] with
 *     p0 = Rcut (absolute), p1 = A12, p2 = A6, p10 = s(Rcut)*Rcut,
 *     p11 = u(Rcut) (PairPotential.cu:82-125, PairPotential.h:149-207).
 */
#ifndef RUMD_B200_H
#define RUMD_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define B2MD_API __attribute__((visibility("default")))
#else
#define B2MD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define B2MD_OK 0
#define B2MD_ERR_ARG 1       /* invalid argument */
#define B2MD_ERR_CUDA 2      /* CUDA runtime error (message has the detail) */
#define B2MD_ERR_NOMEM 3     /* device memory or engine capacity exhausted */
#define B2MD_ERR_STATE 4     /* call not valid in the current state */
#define B2MD_ERR_OVERFLOW 5  /* neighbour list could not be made large enough */

#define B2MD_CUTOFF_NS 0
#define B2MD_CUTOFF_SP 1
#define B2MD_CUTOFF_SF 2

/* pair functions: which RUMD class the parameter table rows belong to */
#define B2MD_POT_LJ_12_6 0            /* Pot_LJ_12_6 / Pot_IPL_12_6: p0 rc, p1 A12, p2 A6 */
#define B2MD_POT_LJ_12_6_SMOOTH_2_4 1 /* Pot_LJ_12_6_smooth_2_4 (PairPotential.h:218-256):
                                         p0 rc, p1 1/sigma^2, p2 4 eps, p3 c2, p4 c4 */
#define B2MD_POT_IPL_N 2              /* Pot_IPL_n (PairPotential.h:603-637):
                                         p0 rc, p1 1/sigma^2, p2 eps, p3 n */

/* fields for b2md_replica_get / b2md_replica_set */
#define B2MD_FIELD_POS 0
#define B2MD_FIELD_VEL 1
#define B2MD_FIELD_FORCE 2
#define B2MD_FIELD_VIRIAL 3
#define B2MD_FIELD_IMAGES 4
#define B2MD_FIELD_STRESS 5

/* indices of b2md_replica_stats output (doubles) */
#define B2MD_STAT_PE 0          /* sum_i u_i of the last force evaluation      */
#define B2MD_STAT_VIRIAL 1      /* sum_i w_i / 6                               */
#define B2MD_STAT_KE 2          /* leap-frog KE(t) of the last integrated step */
#define B2MD_STAT_XI 3          /* Nose-Hoover thermostat state                 */
#define B2MD_STAT_KE2 4         /* sum m v^2 (t + h/2) of the last step         */
#define B2MD_STAT_STEPS 5       /* steps integrated since the replica was added */
#define B2MD_STAT_REBUILDS 6    /* neighbour-list rebuilds                      */
#define B2MD_STAT_STEPS_LEFT 7  /* steps still queued for b2md_run_queued       */
#define B2MD_STAT_OVERFLOW 8    /* 1 if the list overflowed and is waiting      */
#define B2MD_STAT_TARGET_T 9    /* current target temperature                   */
#define B2MD_STAT_MAX_NBRS 10   /* list capacity per particle                   */
#define B2MD_STAT_ACTUAL_MAX_NBRS 11 /* largest neighbour count of the last build */
#define B2MD_STAT_MEAN_NBRS 12  /* mean neighbour-list length of the last build  */
#define B2MD_STAT_WINDOW_TILES 13 /* tiles with a position window (force mode 2)  */
#define B2MD_STAT_TILES 14      /* tiles (blocks) of the replica                 */
#define B2MD_NSTAT 15

typedef struct b2md_engine b2md_engine;

/* One MD system.  Mirrors the state a RUMD Sample + Pot_LJ_12_6 +
 * IntegratorNVT hold (Sample.h:33-90, PairPotential.h:33-128,
 * IntegratorNVT.h:14-92). */
typedef struct {
  int n;                    /* number of particles (>= 2)                          */
  int ntypes;               /* number of particle types (1..8)                     */
  float box[3];             /* rectangular periodic box lengths                    */
  const float* params;      /* ntypes*ntypes*12 floats, RUMD layout                */
  int cutoff_method;        /* B2MD_CUTOFF_*                                       */
  float skin;               /* neighbour-list skin (NeighborList::SetSkin)         */
  float dt;                 /* time step                                           */
  double target_T;          /* thermostat target temperature                       */
  double tau;               /* thermostat relaxation time (omega^2 = 4 pi^2/tau^2) */
  double dT_per_step;       /* SetTemperatureChangePerTimeStep                     */
  double xi;                /* initial thermostat state                            */
  unsigned thermostat_mask; /* bit t set: type t is thermostatted (0 = NVE)        */
  int reset_interval;       /* zero total momentum every k steps (0 = never)       */
  int max_nbrs;             /* list capacity per particle (0 = density estimate)   */
  int energy_interval;      /* log (pe, W, KE, xi) every k steps (0 = off)         */
  int energy_capacity;      /* number of log entries kept                          */
  int potential;            /* B2MD_POT_* (0: LJ 12-6)                             */
} b2md_replica_desc;

/* Engine lifetime.  Replaces the allocation that RUMD spreads over
 * Sample::SetNumberOfParticles (Sample.cu:208-249),
 * NeighborList::AllocateNeighborList (NeighborList.cu:275-295) and
 * IntegratorNVT::AllocateIntegratorState (IntegratorNVT.cu:106-126).
 * Capacities bound what b2md_replica_add may admit (0 = grow on demand).
 * pb = particles per block, tp = threads per particle (Sample(pb, tp)). */
B2MD_API int b2md_engine_create(int device, long long max_particles, int max_replicas,
                       long long max_list_entries, int pb, int tp, b2md_engine** out);
B2MD_API int b2md_engine_destroy(b2md_engine* e);
/* Sample::SetPB_TP (Sample.h:96).  Accepts RUMD's shapes (pb 1..1024, tp
 * 1..64; Autotune.py:156-158 tries pb 16..192 and tp up to 64) and maps them
 * onto the engine's: pb rounded up to a multiple of 32 (at most 512), tp the
 * largest of 1, 2, 4, 8 not above the request, halved until pb*tp <= 512.
 * The same mapping applies to b2md_engine_create. */
B2MD_API int b2md_engine_set_launch(b2md_engine* e, int pb, int tp);
/* The launch shape in effect after that mapping (Sample::GetKernelPlan,
 * Sample.h:160-163). */
B2MD_API int b2md_engine_get_launch(b2md_engine* e, int* pb, int* tp);
/* Device bytes currently allocated by the engine. */
B2MD_API int b2md_engine_memory(b2md_engine* e, long long* bytes);
/* Device bytes held by the active replicas in the engine's pools (used) and
 * allocated by the engine in all (reserved, as b2md_engine_memory).  With
 * b2md_replica_footprint this is the admission budget of a server: RUMD has
 * one system per process and sizes its buffers per Sample
 * (Sample.cu:208-249, NeighborList.cu:275-295). */
B2MD_API int b2md_engine_usage(b2md_engine* e, long long* used, long long* reserved);
/* Counters of the engine's host-side events since its creation (the first
 * n of B2MD_COUNTERS): step-graph instantiations; valid graphs dropped by a
 * re-layout, by a pool growth (pools moved), by a list repair, by another
 * setting change; neighbour lists enlarged after an overflow; tile layouts
 * applied; b2md_run_queued_async chunks launched. */
#define B2MD_COUNTER_GRAPH_BUILDS 0
#define B2MD_COUNTER_INVAL_LAYOUT 1
#define B2MD_COUNTER_INVAL_POOL 2
#define B2MD_COUNTER_INVAL_REPAIR 3
#define B2MD_COUNTER_INVAL_OTHER 4
#define B2MD_COUNTER_LIST_REPAIRS 5
#define B2MD_COUNTER_LAYOUTS 6
#define B2MD_COUNTER_CHUNKS 7
#define B2MD_COUNTERS 8
B2MD_API int b2md_engine_counters(b2md_engine* e, long long* out, int n);
/* Chooses CUDA-graph conditional rebuild nodes (1, default) or unconditional
 * early-exit rebuild kernels (0) for b2md_run. */
B2MD_API int b2md_engine_set_graph_mode(b2md_engine* e, int conditional);
/* Kernel variants, picked by the autotuner next to pb and tp (the analogue of
 * the kernel plan that Autotune.py tunes).  Every variant gives the same
 * neighbour lists and forces bit for bit.
 *   B2MD_VARIANT_FORCE_MODE    how the force kernel reads neighbours:
 *                              0 list entries and positions from global
 *                                memory inside the loop (streamed);
 *                              1 the tile's list rows first copied to shared
 *                                memory (TMA bulk copies);
 *                              2 the tile's position window -- every slot
 *                                segment holding a listed neighbour of the
 *                                tile, made with the list -- copied to shared
 *                                memory (one TMA bulk copy per segment), with
 *                                a 16-bit list of window offsets.
 *   B2MD_VARIANT_BUILD_LANES   the list build: 0 (default) one warp per
 *                              cell, each lane testing a contiguous run of
 *                              the cell's candidates against up to four of
 *                              its particles at once; 1,2,4,8 lanes per
 *                              particle; 32: one warp per cell, 32
 *                              candidates per round staged in shared memory
 *                              (with force mode 2 the lane build runs for 0
 *                              and 32, with min(8, 512/pb) lanes).
 *   B2MD_VARIANT_BUILD_SMEM    1: the list build assembles a tile's list in
 *                              shared memory and writes it with bulk stores;
 *                              0: it stores entries straight to the list.
 *   B2MD_VARIANT_WINDOW_CAP    mode 2: window capacity in particles (shared
 *                              memory of the force kernel, 16 bytes each);
 *                              tiles with larger windows stream.
 *   B2MD_VARIANT_WINDOW_LIST_ROWS  mode 2: rows (multiple of 8) of the 16-bit
 *                              window list copied to shared memory with the
 *                              window; a tile whose longest list is longer
 *                              reads its list from global memory.  0: never.
 *   B2MD_VARIANT_SM_TILES      mode 0: 1 = the force kernel runs as many
 *                              blocks as fit on the GPU, and each block claims
 *                              tiles from its SM's share of the tile range,
 *                              so each SM works on neighbouring tiles whose
 *                              neighbours share its L1; 0 = one block per tile.
 *   B2MD_VARIANT_PERSISTENT    1 (default): b2md_run drives streamed-mode
 *                              engines whose tiles all fit on the GPU at once
 *                              with one cooperative kernel (k_steps) that
 *                              runs steps back to back, with a grid barrier
 *                              between them, until a list rebuild is due;
 *                              engines with more tiles than resident blocks
 *                              (batches) with k_flow: whole steps, list
 *                              rebuilds included, each replica stepping on
 *                              its own through a queue of ready work items;
 *                              (k_batch and k_flow apply to at most 1024
 *                              replicas of at most 65536 particles);
 *                              3: k_flow whenever it applies (the limits
 *                              of k_batch);  2: k_batch, the same items
 *                              with one grid barrier per step for all
 *                              replicas;
 *                              0: one kernel launch per step.
 *   B2MD_VARIANT_PERSISTENT_ACTIVE  read-only: the persistent kernel of the
 *                              current step graph (1 k_steps, 2 k_batch,
 *                              3 k_flow, 0 none).
 *   B2MD_VARIANT_GRAPH_BUILDS  read-only: step graphs instantiated so far
 *                              (admissions and removals do not rebuild a
 *                              k_batch graph).
 *   B2MD_VARIANT_SPLIT_SORT_TILES  k_batch: replicas of at least this many
 *                              tiles (default 16) sort their particles as
 *                              phase items spread over many blocks; smaller
 *                              ones are sorted by one block each.  Same
 *                              permutation either way.
 * No reference counterpart beyond Sample::SetPB_TP (Sample.h:96). */
enum {
  B2MD_VARIANT_FORCE_MODE = 0,
  B2MD_VARIANT_BUILD_LANES = 1,
  B2MD_VARIANT_BUILD_SMEM = 2,
  B2MD_VARIANT_WINDOW_CAP = 3,
  B2MD_VARIANT_SM_TILES = 4,
  B2MD_VARIANT_WINDOW_LIST_ROWS = 5,
  B2MD_VARIANT_PERSISTENT = 6,
  B2MD_VARIANT_PERSISTENT_ACTIVE = 7,
  B2MD_VARIANT_GRAPH_BUILDS = 8,
  B2MD_VARIANT_SPLIT_SORT_TILES = 9
};
B2MD_API int b2md_engine_set_variant(b2md_engine* e, int which, int value);
B2MD_API int b2md_engine_get_variant(b2md_engine* e, int which, int* value);

/* Admission of one system (Sample::ReadConf + SetPotential + SetIntegrator,
 * Simulation.py:29-31,157-214).  vel4/im3 may be NULL (zero).
 * Admission does not wait for running work: the particle data is copied into
 * the engine's pinned staging and uploaded in stream order after what is
 * already queued (a running b2md_run_queued_async chunk), and the tile
 * layout is applied before the next launch.  When pos4 and vel4 are both in
 * page-locked memory (cudaMallocHost / cudaHostRegister) they are copied from
 * directly and the call returns once those copies are done. */
B2MD_API int b2md_replica_add(b2md_engine* e, const b2md_replica_desc* d, const float* pos4,
                     const float* vel4, const int* im3, int* id_out);
/* Removal (a finished job leaving).  Returns at once: its memory goes back to
 * the pools for later admissions, whose uploads are queued behind any work
 * still using it. */
B2MD_API int b2md_replica_remove(b2md_engine* e, int id);
/* Device bytes that b2md_replica_add(d) would hold in the pools (its share
 * of b2md_engine_usage's used bytes), without admitting anything. */
B2MD_API int b2md_replica_footprint(b2md_engine* e, const b2md_replica_desc* d, long long* bytes);
/* Copies a field out in original order (ParticleData::Copy*FromDevice,
 * ParticleData.cu:383-470).  out: n*4 floats, or n*3 ints for images. */
B2MD_API int b2md_replica_get(b2md_engine* e, int id, int field, void* out);
/* Positions, velocities and images together, in original order, with one
 * read of the sort permutation (ParticleData::CopyPosFromDevice +
 * CopyVelFromDevice, ParticleData.cu:383-420).  Any output may be NULL:
 * pos4 and vel4 n*4 floats, im3 n*3 ints. */
B2MD_API int b2md_replica_read(b2md_engine* e, int id, float* pos4, float* vel4, int* im3);
/* Replaces positions, velocities or images (ParticleData::CopyPosToDevice
 * with reset_sorting, ParticleData.cu:333-355).  Setting positions forces a
 * neighbour-list rebuild before the next force evaluation. */
B2MD_API int b2md_replica_set(b2md_engine* e, int id, int field, const void* in);
/* Pair parameter table / cut-off method / skin / pair function
 * (PairPotential::SetParams + CopyParamsToGPU, PairPotential.cu:82-125;
 * SetNbListSkin; Sample::SetPotential with another Pot_* class).  The
 * replica's potential list becomes this one potential (Sample.cu:251-259). */
B2MD_API int b2md_replica_set_potential(b2md_engine* e, int id, int ntypes, const float* params,
                               int cutoff_method, float skin, int potential);
/* Sample::AddPotential (Sample.cu:261-278): a second pair potential (same
 * number of types; its own parameter table, cut-off method and pair
 * function).  Sample::CalcF evaluates both (Sample.cu:335-336): the forces,
 * energies, virials and stresses of the second are added to the first's
 * once both per-particle sums are complete (PairPotential.cu:370-388).  One
 * neighbour list serves both, built with the larger cut-off per type pair
 * and the first potential's skin.  At most two potentials per replica; an
 * engine holding such a replica runs its steps with the per-step graphs
 * (the persistent kernels evaluate one potential). */
B2MD_API int b2md_replica_add_potential(b2md_engine* e, int id, int ntypes, const float* params,
                                        int cutoff_method, int potential);
/* Integrator settings (IntegratorNVT::SetTimeStep, SetTargetTemperature,
 * SetRelaxationTime, SetThermostatState, SetThermostatOn*,
 * SetTemperatureChangePerTimeStep; IntegratorNVT.cu:132-190). */
B2MD_API int b2md_replica_set_integrator(b2md_engine* e, int id, float dt, double target_T,
                                double tau, double dT_per_step, unsigned thermostat_mask);
B2MD_API int b2md_replica_set_xi(b2md_engine* e, int id, double xi);
B2MD_API int b2md_replica_set_reset_interval(b2md_engine* e, int id, int reset_interval);
/* NeighborList::SetNB_Method (NeighborList.cu:226-245): -1 "default" (cell
 * sort when the 5x5x5 scan covers rc+skin, else all pairs), 0 "sort", 1 "n2". */
B2MD_API int b2md_replica_set_nb_method(b2md_engine* e, int id, int method);
/* FP64 scalars of the replica, B2MD_NSTAT doubles (Sample::GetPotentialEnergy,
 * GetVirial, IntegratorNVT::GetKineticEnergy/GetThermostatState). */
B2MD_API int b2md_replica_stats(b2md_engine* e, int id, double* out);
/* (Re)configures the energy log: one entry every interval steps of a run,
 * the last capacity entries kept; clears the log. */
B2MD_API int b2md_replica_set_energy_log(b2md_engine* e, int id, int interval, int capacity);
/* Energy log: up to cap entries of (run step, pe, W, KE, xi); returns count. */
B2MD_API int b2md_replica_energy_log(b2md_engine* e, int id, double* out, int cap, int* count);
/* Stress tensor sum (Sample::GetStress, Sample.cu:393-444): 6 doubles
 * (xx, yy, zz, yz, xz, xy), requires a force evaluation with stress. */
B2MD_API int b2md_replica_stress(b2md_engine* e, int id, int include_kinetic, double* out6);

/* Sample::CalcF (Sample.cu:329-351) for every replica: neighbour-list update
 * (NeighborList::UpdateNBlist, NeighborList.cu:583-690) then pair forces
 * (Calcf_NBL_tp*, PairPotential.cu:330-515). */
B2MD_API int b2md_calc_f(b2md_engine* e, int stress);
/* IntegratorNVT::Integrate (IntegratorNVT.cu:64-92) for every replica. */
B2MD_API int b2md_integrate(b2md_engine* e);
/* IntegratorNVT::SetMomentumToZero (IntegratorNVT.cu:176-183). */
B2MD_API int b2md_zero_momentum(b2md_engine* e);
/* Simulation.Run(nsteps) (Simulation.py:538-622) for every replica, in
 * lock step: momentum reset every reset_interval steps, CalcF, Integrate,
 * then a final CalcF.  Runs as CUDA graphs of fused kernels with the rebuild
 * decided on the device; list overflow is repaired on the host (capacity
 * doubled, NeighborList.cu:657-676) and the run resumed. */
B2MD_API int b2md_run(b2md_engine* e, long long nsteps);
/* b2md_run with eager launches instead of graphs, for measurement (a
 * profiler can follow eager launches, not conditional graph nodes).  With the
 * persistent step kernel in effect, the loop of the persistent graph runs
 * from the host: the rebuild kernels, then one cooperative k_steps launch
 * that runs steps until a rebuild is due; CUDA events bracket each k_steps
 * launch.  Otherwise events bracket every fused step kernel and the host
 * reads the rebuild decision before each step (one small kernel and a 4-byte
 * copy), launching the rebuild kernels only when a list is due, as the step
 * graph's conditional node does.  Returns the summed step-kernel time and the
 * number of kernel launches in the run. */
B2MD_API int b2md_run_timed(b2md_engine* e, long long nsteps, double* step_kernel_ms,
                            long long* launches);
/* Batched/served form: each replica advances its own queued step count
 * (b2md_replica_queue_steps) in the same launches; returns when all queues
 * are empty or after max_steps launches-worth of steps (0 = until empty).
 * Queueing steps is itself asynchronous (in stream order). */
B2MD_API int b2md_replica_queue_steps(b2md_engine* e, int id, long long nsteps);
B2MD_API int b2md_run_queued(b2md_engine* e, long long max_steps, long long* steps_run);

/* The served form's chunks, for a host that admits and retires jobs while the
 * GPU runs.  b2md_run_queued_async applies pending admissions/removals,
 * launches up to max_steps steps of the queued work (0 = until empty) and
 * returns at once with a ticket; a snapshot of every replica's state at the
 * end of the chunk is copied to pinned host memory behind it.  At most two
 * chunks are in flight: a third call first waits for the oldest.  A batched
 * persistent graph (k_batch) is not rebuilt by admissions or removals.
 * b2md_run_queued_poll sets *done without blocking.  b2md_run_queued_wait
 * waits for the chunk (one of the two most recent), reports a device wait
 * that gave up, enlarges overflowed lists (their replicas continue in the
 * next chunk), and returns the steps the chunk ran and, for replica ids
 * 0..cap-1, B2MD_CHUNK_FIELDS doubles each from the snapshot (replicas not
 * active when the chunk was launched have ACTIVE 0 and STEPS_LEFT -1).
 * The analogue of RUMD's Simulation.Run loop (Simulation.py:538-622) for many
 * systems at once, without the per-block host round trips. */
#define B2MD_CHUNK_ACTIVE 0
#define B2MD_CHUNK_STEPS 1
#define B2MD_CHUNK_STEPS_LEFT 2
#define B2MD_CHUNK_PE 3
#define B2MD_CHUNK_VIRIAL 4
#define B2MD_CHUNK_KE 5
#define B2MD_CHUNK_XI 6
#define B2MD_CHUNK_REBUILDS 7
#define B2MD_CHUNK_OVERFLOW 8
#define B2MD_CHUNK_FIELDS 9
B2MD_API int b2md_run_queued_async(b2md_engine* e, long long max_steps, long long* ticket);
B2MD_API int b2md_run_queued_poll(b2md_engine* e, long long ticket, int* done);
B2MD_API int b2md_run_queued_wait(b2md_engine* e, long long ticket, long long* steps_run, double* states,
                                  int cap);

/* Parity hooks.  Neighbour list of replica id in ORIGINAL particle ids:
 * counts[n], nbl[n][max_nbrs] row-major (entries in list order). */
B2MD_API int b2md_nbl_export(b2md_engine* e, int id, unsigned* counts, unsigned* nbl, int max_nbrs);
/* d_unsorted_index (ParticleData.h:56): original id of each sorted slot. */
B2MD_API int b2md_sort_export(b2md_engine* e, int id, unsigned* unsorted_index);
/* Cell key grid used by the rebuild: nc[3]. */
B2MD_API int b2md_cell_grid(b2md_engine* e, int id, int* nc3);

B2MD_API int b2md_sync(b2md_engine* e);
/* The engine's CUDA stream (cudaStream_t) for callers that interleave work. */
B2MD_API void* b2md_stream(b2md_engine* e);
B2MD_API const char* b2md_last_error(void);
B2MD_API const char* b2md_version(void);

/* Evaluates, on the device, the squared minimum-image distance of npairs
 * pairs both as the reference source expression (compiled with nvcc's default
 * multiply-add contraction) and as this engine's explicit form; used by the
 * parity tests to pin the neighbour-list arithmetic.  Inputs and outputs are
 * host arrays: a4/b4 npairs*4 floats, box 3 floats, out 2*npairs floats. */
B2MD_API int b2md_probe_dist2(const float* a4, const float* b4, const float* box, int npairs, float* out);
/* Same for the cell coordinate (int)(nc * (x / L + 0.5f)) of n coordinates:
 * out 2*n ints (reference expression, explicit form). */
B2MD_API int b2md_probe_cell(const float* x, int n, float box, int nc, int* out);
/* integrateNVTAlgorithm's velocity/position update and wrap as the reference
 * source writes them (IntegratorNVT.cu:385-399, SimulationBox.h:140-155),
 * compiled with default nvcc flags, next to the engine's explicit forms:
 * ref9 / eng9 receive (v, r, image) per particle. */
/* Measured peaks of the current device for the roofline fractions: L2 read
 * bandwidth (GB/s, a 48 MiB buffer read past L1) and FP32 FMA throughput
 * (TFLOP/s, independent FMA chains), best of `trials`, CUDA-event timed.
 * No counterpart in the reference (measurement only). */
B2MD_API int b2md_measure_peaks(int trials, double* l2_gbs, double* fma_tflops);
B2MD_API int b2md_probe_nvt(const float* r4, const float* v4, const float* f4, const float* xi, float dt,
                            const float* box, int n, float* ref9, float* eng9);

/* LJ forces, per-particle energies, total potential energy and virial of one
 * configuration, for callers that cannot allocate device memory during the
 * call: for example a host program that owns every device buffer and lends
 * this library only pointers, or a real-time loop that must not call
 * cudaMalloc/cudaFree (they may synchronise the device and take unbounded
 * time).  No counterpart in the reference; it allocates nothing.
 *   pos4    DEVICE pointer, n*4 floats (x, y, z, type bits), caller-owned
 *   box     host, 3 floats;  params host, ntypes*ntypes*12 floats (RUMD layout)
 *   force4  DEVICE pointer, n*4 floats out (fx, fy, fz, u_i)
 *   sums    DEVICE pointer, 2 doubles out (sum u_i, virial W)
 *   stream  cudaStream_t to run on (NULL = default stream); returns at launch
 * All pairs within the cut-off are summed (no neighbour list).  n is at most
 * 65536: the only scratch is a fixed array of that capacity in the library's
 * device image, one per GPU, kept until the process exits and shared by every
 * call, so calls that overlap on the GPU race; order them on one stream.  The
 * first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  A later call in another CUDA context of the
 * device (after cudaDeviceReset, say) looks it up again.  Every cut-off must
 * be at most half of every box length (the minimum-image sum counts one
 * image per pair); larger ones return B2MD_ERR_ARG. */
B2MD_API int b2md_forces_noalloc(const float* pos4, int n, const float* box, int ntypes, const float* params,
                                 int cutoff_method, float* force4, double* sums, void* stream);

/* ---- FP64 engine: the accuracy oracle on the GPU ----
 * The same step (neighbour list, LJ pair forces, Nose-Hoover leap-frog,
 * energy/virial/kinetic sums) in double precision throughout: what RUMD
 * becomes after changeToDouble.sh (changeToDouble.sh:1-189).  One system per
 * engine, particles in the caller's order.  Pair constants: rc, A12, A6 from
 * the RUMD table (params[k*12 + 0..2]); s(rc) rc and u(rc) recomputed in FP64.
 *   pos4: x, y, z, type (as a whole number);  vel4: vx, vy, vz, 1/m;  im3 may
 *   be NULL.  max_nbrs 0 = 1.6 x the ideal-gas estimate + 32.
 *   b2md_f64_run: energies (NULL or nsteps*4 doubles) = pe, W, KE(t), xi per
 *   step, as Simulation.Run's energies file rows.
 *   b2md_f64_stats: out[7] = pe, W, KE(t), KE2, xi, rebuilds, steps. */
typedef struct b2md_f64 b2md_f64;
#define B2MD_F64_POS 0    /* double4 per particle */
#define B2MD_F64_VEL 1    /* double4 per particle */
#define B2MD_F64_FORCE 2  /* double4: fx, fy, fz, u_i */
#define B2MD_F64_IMAGES 3 /* 3 ints per particle */
B2MD_API int b2md_f64_create(int device, int n, int ntypes, const double* box3, const float* params,
                             int cutoff_method, double skin, int max_nbrs, b2md_f64** out);
B2MD_API int b2md_f64_destroy(b2md_f64* h);
B2MD_API int b2md_f64_set_state(b2md_f64* h, const double* pos4, const double* vel4, const int* im3);
B2MD_API int b2md_f64_set_integrator(b2md_f64* h, double dt, double target_T, double tau, int thermostat_on,
                                     int reset_interval);
B2MD_API int b2md_f64_set_xi(b2md_f64* h, double xi);
B2MD_API int b2md_f64_calc_f(b2md_f64* h);
B2MD_API int b2md_f64_run(b2md_f64* h, long long nsteps, double* energies);
B2MD_API int b2md_f64_get(b2md_f64* h, int field, void* out);
B2MD_API int b2md_f64_stats(b2md_f64* h, double* out);

#ifdef __cplusplus
}
#endif
#endif /* RUMD_B200_H */
