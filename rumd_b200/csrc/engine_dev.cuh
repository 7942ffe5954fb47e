// Device-side data layout and kernels of the B200 RUMD engine.
//
// Layout in HBM (one engine = many replicas; a plain Sample is one replica):
//   particle pools, indexed p0 + local slot (slot = position in cell-sorted order)
//     r[2]    float4  x, y, z, type bits   (ping-pong: step k reads r[rbuf], writes r[rbuf^1])
//     v[2]    float4  vx, vy, vz, 1/m      (ping-pong with abuf: swapped only by the sort)
//     im[2]   int4    images               (abuf)
//     uidx[2] uint    original particle id (abuf)  == d_unsorted_index (ParticleData.h:56)
//     f, w, sts float4 as RUMD (ParticleData.h:41-46); last_r float4; nn uint
//   list pool: entry k of slot i at nbl[nbl0 + lpos(k, i, stride)]: blocks of
//     8 entries, block b of all slots one run (RUMD's nbl[k*nvp + i],
//     NeighborList.cu:1293, with 8 consecutive entries of a slot packed into
//     one 32-byte sector: the list build writes a sector per 8 entries and a
//     thread of the force kernel reads 4 entries with one 16-byte load, while
//     a warp's loads of one block still cover consecutive sectors)
//   window list: wl[nbl0 + lpos(k, i, stride)] (uint16), the same entries as
//     nbl written as offsets into the tile's position window (see below)
//   cell pools: cnt[cell0 + c], start[cell0 + c] (chunk-local exclusive prefix)
//   per-tile position window: wseg[tile*kWinSeg + s] = (first slot, length,
//     window offset, 0) for the slot segments that hold every listed
//     neighbour of the tile's particles, sorted by slot; wmeta[tile] =
//     (segments, window particles), or (-1, -1) when the tile has none.
//   per-tile / per-group FP64 partial sums for deterministic two-level reductions.
//
// A "tile" is pb consecutive slots of one replica; one CUDA block processes one
// tile (pb particles x tp threads per particle).  Tiles never straddle replicas,
// so a replica's arithmetic is the same alone and in any batch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace b2md {

constexpr int kMaxTypes = 8;
constexpr int kParStride = 12;  // packed floats per type pair
constexpr int kNumParam = 12;   // RUMD NumParam (rumd_base.h)
constexpr int kNPart = 8;       // FP64 partial sums per tile
constexpr int kGroup = 32;      // tiles per reduction group
constexpr int kMaxBlock = 512;  // pb*tp limit (launch bounds)
constexpr int kWinSeg = 128;    // slot segments per tile position window
constexpr int kWinBase = 4;     // cell rows (y, z) a tile may span for a window

// Place of list entry k of slot i in a replica's list (stride = its slots).
__host__ __device__ __forceinline__ size_t lpos(unsigned k, unsigned i, size_t stride) {
  return (size_t)(k >> 3) * (stride << 3) + ((size_t)i << 3) + (k & 7u);
}
// List rows allocated for a capacity of max_nbrs entries (whole blocks of 8).
__host__ __device__ __forceinline__ int list_rows(int max_nbrs) { return (max_nbrs + 7) & ~7; }

enum { P_PE = 0, P_W, P_KE2, P_KET, P_PX, P_PY, P_PZ, P_M };
enum { CUT_NS = 0, CUT_SP = 1, CUT_SF = 2 };
enum { NB_CELLS = 0, NB_N2 = 1 };
// pair functions (the RUMD classes whose rows the parameter table holds)
enum { POT_LJ_12_6 = 0, POT_LJ_12_6_SMOOTH_2_4 = 1, POT_IPL_N = 2 };

// Packed pair row (kParStride floats; slot 6 is (rc+skin)^2 for every pair
// function, read by the list build).  The cut-off method is folded into c_s,
// c_u0 (and c_ur):
//   LJ 12-6:          rc^2, A12, A6, c_s, c_u0, c_ur, (rc+skin)^2, 0, ...
//   LJ 12-6 smooth:   rc^2, sigma^2, 4 eps, b, c, e, (rc+skin)^2, g, c_s, c_u0
//                     (b = -2 c2 4eps/sigma^2, c = -4 c4 4eps/sigma^4,
//                      e = c2 4eps/sigma^2, g = c4 4eps/sigma^4)
//   IPL n:            rc^2, sigma^2, eps, n/2, n eps, 0, (rc+skin)^2, 0, c_s, c_u0
// (see lj_pair).
struct RepDev {
  int n, p0, tile0, ntiles;
  int group0, ngroups;
  int ntypes, par0;
  int cell0, ncell;
  int nc[3];
  int nb_method;
  int max_nbrs, nbl_stride;
  long long nbl0;
  float L[3], invL[3];
  float ilim[3];  // |x| below L/2 - (rc_max + 2 skin): no minimum image needed (k_force)
  float skin2_4;
  float dt, omega2;
  int cutoff;
  unsigned thermo_mask;
  int reset_interval;
  int energy_interval, energy_cap;
  long long elog0;
  double dof;
  int active;
  int potential;  // POT_*
  // Sample::AddPotential: a second pair function evaluated over the same list
  // (built with the larger cut-off of the two), its sums added to the
  // first's; npot = 1 or 2
  int npot, par1, potential1;
};

struct RepState {
  double xi, T, dT;
  double ke2, ke_t, pe, vir;
  double P[3], M;
  long long steps;       // total integrated steps
  long long steps_left;  // queued steps
  long long run_step;    // step index inside the current run (momentum-reset schedule)
  int rbuf, abuf;
  int rebuild, exceed;
  int overflow, nrebuilds;
  int actual_max_nbrs, nlog;
  int err;               // a bounded device wait gave up (reported to the host)
  unsigned sort_done;    // k_batch: epoch of the replica's last in-launch sort
  unsigned sort_items;   // k_batch: phase items of the replica's split sort completed (reset by the last)
  int flow_left;         // k_flow: items of the replica's current phase not yet finished
  int launch_steps;      // k_flow: steps the replica ran in the current launch
  int build_next;        // k_rb_build_runs: the replica's next unclaimed cell (0 between builds)
};

// Control block of the persistent step kernel (k_steps), one per engine.
struct PersistCtl {
  unsigned long long arrive;  // setup barrier: blocks arrived
  unsigned long long word[2];  // step barriers (alternating): arrivals and the finalizers' tallies
  unsigned gen;     // grid-barrier generation
  int budget;       // steps this graph launch may still run (set by the host)
  int err;          // a grid-barrier wait gave up (reported to the host)
  unsigned ticket;  // k_batch: work-item tickets claimed in this launch
  unsigned readers; // k_batch: blocks that have read the step's rebuild list
  int fcnt[2];      // k_batch: replicas on the rebuild list of steps of each parity
  int ftiles[2];    // k_batch: their tiles
  // the tile layout in effect (written by the host with every re-layout, in
  // stream order): graphs of k_batch read these instead of capturing them,
  // so admissions and removals need no new graph
  int lay_ntiles;
  int lay_nrep;
  // k_flow's item queue: tickets taken by consumers (head) and producers
  // (tail), monotone across launches; replicas still stepping; the most
  // steps a replica ran in the launch; blocks that left the launch
  unsigned long long qhead, qtail;
  int active;
  int ran;
  unsigned exited;
};

struct EngArgs {
  float4* r[2];
  float4* v[2];
  int4* im[2];
  unsigned* uidx[2];
  float4* f;
  float4* w;
  float4* sts;
  float4* last_r;
  unsigned* nn;
  unsigned* nbl;
  int* key;
  int* slot;
  unsigned* order;
  int* cnt;
  int* cstart;
  int* ctot;    // per tile: cell-chunk total (scan)
  int* cpref;   // per tile: exclusive prefix of chunk totals within the replica
  const float* par;
  const RepDev* rep;
  RepState* st;
  const int* tile_rep;
  const int* tile_first;
  double* tpart;
  double* gpart;
  unsigned* gctr;
  unsigned* rctr;
  unsigned* fctr;
  int* any_rebuild;
  double* elog;
  int ntiles;
  int nrep;
  int idx_pitch;  // k_force: slots per staged list block (pb)
  int idx_rows;   // k_force: rows of the staged list tile (max list capacity over replicas)
  int max_types;  // largest type count over the active replicas (pair-table rows in shared memory)
  PersistCtl* pctl;  // k_steps control block
  // tpart, gpart, gctr and rctr hold two halves each: k_steps alternates
  // them by step parity (the other kernels use the first)
  long long gpart_half, tpart_half;
  int gctr_half, rctr_half;
  unsigned short* wl;  // window list (force mode 2)
  int4* wseg;          // per-tile window segments
  int2* wmeta;         // per-tile (segments, particles)
  int win_on;          // list builds also build the windows
  int win_cap;         // window capacity in particles (shared memory of k_force)
  int wl_rows;         // window-list rows k_force stages in shared memory (multiple of 8; 0 = none)
  int nreg;            // SM regions for k_force tile claiming (0 = one tile per block)
  unsigned* smctr;     // per-region claim counters [nreg] + tiles claimed [nreg]
  int* flist;          // k_batch: rebuild lists, two halves by step parity (replica ids)
  int bshared_off;     // k_batch: offset of its per-block tables in dynamic shared memory
  int split_tiles;     // k_batch: replicas of at least this many tiles sort as phase items over many blocks
  int2* fq;            // k_flow: item queue slots (replica, item code)
  unsigned long long* fseq;  // k_flow: ticket + 1 of the item in each slot (release-published)
  unsigned qcap;       // k_flow: queue slots
  int rb_steps_only;   // rebuild kernels of a run: only replicas with queued steps (CalcF: every flagged one)
};

}  // namespace b2md
