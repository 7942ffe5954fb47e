// Host side of the B200 RUMD engine: pools in HBM, replica admission, CUDA
// graphs with device-decided neighbour-list rebuilds, and the C ABI declared
// in include/rumd_b200.h.
#include "../../include/rumd_b200.h"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using namespace b2md;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

struct CudaErr {
  cudaError_t e;
  const char* what;
  int line;
};

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) throw CudaErr{e_, #call, __LINE__};     \
  } while (0)

struct ApiErr {
  int code;
  std::string msg;
};

[[noreturn]] void api_fail(int code, const std::string& m) { throw ApiErr{code, m}; }

// First-fit allocator of [0, cap) ranges, alignment in units.
struct RangeAlloc {
  long long cap = 0;
  std::map<long long, long long> free_;  // offset -> size
  void init(long long c) { cap = c; free_.clear(); if (c > 0) free_[0] = c; }
  void grow(long long c) {
    if (c <= cap) return;
    long long old = cap;
    cap = c;
    auto it = free_.end();
    if (!free_.empty()) {
      --it;
      if (it->first + it->second == old) { it->second += c - old; return; }
    }
    free_[old] = c - old;
  }
  long long alloc(long long n, long long align) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      long long off = (it->first + align - 1) / align * align;
      long long pad = off - it->first;
      if (pad + n <= it->second) {
        long long start = it->first, size = it->second;
        free_.erase(it);
        if (pad > 0) free_[start] = pad;
        if (size - pad - n > 0) free_[off + n] = size - pad - n;
        return off;
      }
    }
    return -1;
  }
  void release(long long off, long long n) {
    if (n <= 0) return;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
    }
  }
  long long used_end() const {
    if (free_.empty()) return cap;
    auto it = std::prev(free_.end());
    return it->first + it->second == cap ? it->first : cap;
  }
};

struct HostRep {
  bool active = false;
  int n = 0, np = 0;           // particles, padded
  long long p0 = -1;
  long long nbl0 = -1, nbl_len = 0;
  long long cell0 = -1;
  int ncell = 0;
  long long par0 = -1;
  int npar = 0;
  long long elog0 = -1;
  int ecap = 0;
  RepDev d{};
  float rcmax = 0.f, skin = 0.f;
  std::vector<float> params;   // RUMD layout
  int nb_method_req = -1;      // -1 default
  long long bytes = 0;         // device bytes held in the engine's pools (b2md_engine_usage)
  long long admit_seq = 0;     // chunks launched before this replica was admitted
  long long repair_seq = -1;   // chunks launched when its list was last enlarged
  // a second pair potential (b2md_replica_add_potential): RUMD layout table,
  // pair function, cut-off method, its packed table's place
  std::vector<float> params1;
  int potential1 = -1, cutoff1 = 0;
  long long par1 = -1;
  int npar1 = 0;
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  long long n = 0;
};

// A region of the pinned staging ring whose host-to-device copies may still
// be queued behind earlier work on the stream; reusable once `ev` completed.
struct StageBlk {
  size_t lo, hi;
  cudaEvent_t ev;
};

// One chunk of queued steps launched by b2md_run_queued_async, with pinned
// snapshots of the control block and the replica states copied right after
// it in stream order.
struct ChunkRec {
  long long ticket = 0;        // 0: never used
  bool waited = true;
  bool persistent = false;     // budgeted persistent graph (else per-step graphs)
  long long budget = 0, ran = 0;
  cudaEvent_t done = nullptr;
  int* h_in = nullptr;         // pinned: the step budget copied to the device
  PersistCtl* h_ctl = nullptr; // pinned: control block after the chunk
  RepState* h_st = nullptr;    // pinned: replica states after the chunk
  int st_cap = 0;
  std::vector<char> active;    // replicas active when the chunk was launched
};

}  // namespace

struct b2md_engine {
  int device = 0;
  cudaStream_t stream = nullptr, cap_stream = nullptr;
  int pb = 64, tp = 4;
  int cond_mode = 1;
  // pools
  long long pcap = 0, ecap = 0, ccap = 0, qcap = 0, zcap = 0;
  int rcap = 0;
  // kernel variants (b2md_engine_set_variant)
  int force_mode = 0;          // force kernel: FM_STREAMED, FM_STAGED or FM_WINDOW
  bool sm_tiles = false;       // FM_STREAMED: blocks claim tiles from their SM's region
  int nsm = 0;                 // streaming multiprocessors of the device
  unsigned* smctr = nullptr;   // SM-region claim counters (nsm + 1)
  int win_cap = 2560;          // FM_WINDOW: window capacity in particles
  int wl_rows_cap = 128;       // FM_WINDOW: window-list rows staged in shared memory (0 = stream)
  int build_lanes = 0;         // list build: 0 contiguous candidate runs per lane, else lanes per particle (32: one warp per cell)
  bool build_smem = false;     // list build: tile assembled in shared memory
  int persist = 1;             // runs: 0 one launch per step; 1 persistent (k_steps when every tile has a
                               // resident block, else k_flow); 2 k_batch, 3 k_flow whenever they apply
  bool persist_on = false;     // the current graphs are persistent ones (kind below)
  int persist_kind = 0;        // 1 k_steps, 2 k_batch, 3 k_flow
  int* flist = nullptr;        // k_batch rebuild lists (2 x rcap)
  int split_tiles = 16;        // k_batch: replicas of at least this many tiles sort in phases over many blocks
  int2* fq = nullptr;          // k_flow: item queue slots
  unsigned long long* fseq = nullptr;  // k_flow: published ticket of each slot
  unsigned fqcap = 0;          // k_flow: queue slots
  PersistCtl* pctl = nullptr;  // k_steps control block
  int* h_budget = nullptr;     // pinned: the step budget written before each persistent launch
  void* h_stage = nullptr;     // pinned staging for particle uploads and read-backs (grown on demand)
  size_t h_stage_bytes = 0;
  // pinned ring for host-to-device copies that may wait behind running work
  // (admissions, layout uploads): a call fills a region and returns at once
  char* ring = nullptr;
  size_t ring_cap = 0, ring_head = 0;
  std::vector<StageBlk> ring_pending;                  // regions with copies possibly in flight
  std::vector<std::pair<size_t, size_t>> ring_open;    // regions of the current call (no event yet)
  bool layout_dirty = false;     // admissions/removals since the last tile layout upload
  std::vector<int> momentum_due; // replicas whose momentum is computed after the next upload
  int graph_types = 0;           // pair-table rows in the current persistent graph's shared memory
  bool wl_on = false;            // window-list pool allocated (force mode 2 used)
  int graph_builds = 0;          // step-graph instantiations so far (B2MD_VARIANT_GRAPH_BUILDS)
  long long invalidations[4] = {0, 0, 0, 0};  // valid graphs dropped, by reason (INV_*)
  long long list_repairs = 0;    // lists enlarged after an overflow
  long long layout_uploads = 0;  // tile layouts applied
  ChunkRec chunk[2];             // b2md_run_queued_async chunks (by ticket parity)
  long long chunk_seq = 0;
  RangeAlloc palloc, ealloc, calloc, qalloc, zalloc;
  float4* r[2] = {nullptr, nullptr};
  float4* v[2] = {nullptr, nullptr};
  int4* im[2] = {nullptr, nullptr};
  unsigned* uidx[2] = {nullptr, nullptr};
  float4 *f = nullptr, *w = nullptr, *sts = nullptr, *last_r = nullptr;
  unsigned *nn = nullptr, *order = nullptr;
  int *key = nullptr, *slot = nullptr;
  unsigned* nbl = nullptr;
  unsigned short* wl = nullptr;  // window list (same layout as nbl)
  int *cnt = nullptr, *cstart = nullptr;
  float* par = nullptr;
  double* elog = nullptr;
  RepDev* rep = nullptr;
  RepState* st = nullptr;
  unsigned* rctr = nullptr;
  // tiles
  int ntiles = 0, tcap = 0, ngroups = 0, gcap = 0;
  int *tile_rep = nullptr, *tile_first = nullptr, *ctot = nullptr, *cpref = nullptr;
  int4* wseg = nullptr;  // per-tile window segments
  int2* wmeta = nullptr;  // per-tile (segments, particles)
  double *tpart = nullptr, *gpart = nullptr;
  unsigned* gctr = nullptr;
  unsigned* fctr = nullptr;
  int* any_rebuild = nullptr;
  std::vector<HostRep> reps;
  // graphs
  bool graphs_valid = false;
  cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};  // [0]: 1 step, [1]: kChunk steps, [2]: persistent
  cudaGraph_t graph[3] = {nullptr, nullptr, nullptr};
  long long bytes = 0;
};

namespace {

constexpr int kChunk = 32;
constexpr int kMaxDynSmemBytes = 220 * 1024;  // dynamic shared memory a list-tile kernel may use
// largest position window: fits the shared memory, and 16-bit window offsets
constexpr int kMaxWindow = (kMaxDynSmemBytes - (int)(kParSmemFloats * sizeof(float))) / (int)sizeof(float4);

template <class T>
void dev_grow(b2md_engine* e, T*& p, long long old_n, long long new_n, bool zero_new) {
  T* np = nullptr;
  CK(cudaMalloc(&np, (size_t)std::max<long long>(new_n, 1) * sizeof(T)));
  e->bytes += (new_n - old_n) * (long long)sizeof(T);
  if (p && old_n > 0) CK(cudaMemcpyAsync(np, p, (size_t)old_n * sizeof(T), cudaMemcpyDeviceToDevice, e->stream));
  if (zero_new && new_n > old_n)
    CK(cudaMemsetAsync(np + old_n, 0, (size_t)(new_n - old_n) * sizeof(T), e->stream));
  if (p) {
    CK(cudaStreamSynchronize(e->stream));
    CK(cudaFree(p));
  }
  p = np;
}

// Pinned host staging of at least `bytes` (kept for the engine's life), so
// that particle uploads and read-backs are DMA copies.  Sized per particle
// for the largest use (read-back: id + r + v + images, plus alignment).
constexpr size_t kStagePerParticle = 64;
void* host_stage(b2md_engine* e, size_t bytes) {
  if (bytes > e->h_stage_bytes) {
    if (e->h_stage) {
      CK(cudaStreamSynchronize(e->stream));
      CK(cudaFreeHost(e->h_stage));
      e->h_stage = nullptr;
      e->h_stage_bytes = 0;
    }
    const size_t b = std::max(bytes, (size_t)1 << 20);
    CK(cudaMallocHost(&e->h_stage, b));
    e->h_stage_bytes = b;
  }
  return e->h_stage;
}

// Page-locked host memory (cudaMallocHost / cudaHostRegister): DMA-able as is.
bool is_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// ---- pinned staging ring ----
// Host-to-device copies from pageable memory may make the driver wait for the
// stream, so copies that should not wait for running work (admissions, tile
// layouts) go through this ring: the call copies its data into a region,
// queues the copies and records an event behind them; a later call reuses the
// region once that event has completed.  Only when the ring is full does a
// call wait, for the oldest copies in its way.
void ring_reset(b2md_engine* e) {
  for (auto& b : e->ring_pending) cudaEventDestroy(b.ev);
  e->ring_pending.clear();
  e->ring_open.clear();
  e->ring_head = 0;
}

// Records an event behind the copies queued from this call's regions.
void stage_commit(b2md_engine* e) {
  for (const auto& o : e->ring_open) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, e->stream));
    e->ring_pending.push_back({o.first, o.second, ev});
  }
  e->ring_open.clear();
}

// A ring of at least `cap` bytes (grown while nothing may still read it).
void ring_reserve(b2md_engine* e, size_t cap) {
  if (cap <= e->ring_cap) return;
  CK(cudaStreamSynchronize(e->stream));
  ring_reset(e);
  if (e->ring) CK(cudaFreeHost(e->ring));
  e->ring = nullptr;
  e->ring_cap = 0;
  CK(cudaMallocHost(&e->ring, cap));
  e->ring_cap = cap;
}

char* stage_alloc(b2md_engine* e, size_t bytes) {
  const size_t n = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
  if (2 * n > e->ring_cap) ring_reserve(e, std::max<size_t>(4 * n, (size_t)4 << 20));
  size_t lo = e->ring_head;
  if (lo + n > e->ring_cap) lo = 0;
  const size_t hi = lo + n;
  for (const auto& o : e->ring_open)
    if (o.first < hi && lo < o.second) {  // this call's own earlier region: commit it first
      stage_commit(e);
      break;
    }
  for (size_t k = 0; k < e->ring_pending.size();) {
    StageBlk& b = e->ring_pending[k];
    bool done;
    if (b.lo < hi && lo < b.hi) {
      CK(cudaEventSynchronize(b.ev));
      done = true;
    } else {
      const cudaError_t q = cudaEventQuery(b.ev);
      if (q != cudaSuccess && q != cudaErrorNotReady) throw CudaErr{q, "cudaEventQuery(stage)", __LINE__};
      done = q == cudaSuccess;
    }
    if (done) {
      cudaEventDestroy(b.ev);
      b = e->ring_pending.back();
      e->ring_pending.pop_back();
    } else {
      ++k;
    }
  }
  e->ring_head = hi;
  e->ring_open.push_back({lo, hi});
  return e->ring + lo;
}

// Why valid step graphs were dropped (b2md_engine_counters).
enum { INV_OTHER = 0, INV_LAYOUT = 1, INV_POOL = 2, INV_REPAIR = 3, INV_REASONS = 4 };

void invalidate_graphs(b2md_engine* e, int why = INV_OTHER) {
  if (e->graphs_valid) ++e->invalidations[why];
  for (int k = 0; k < 3; ++k) {
    if (e->gexec[k]) cudaGraphExecDestroy(e->gexec[k]);
    if (e->graph[k]) cudaGraphDestroy(e->graph[k]);
    e->gexec[k] = nullptr;
    e->graph[k] = nullptr;
  }
  e->graphs_valid = false;
}

void grow_particles(b2md_engine* e, long long need) {
  if (need <= e->pcap) return;
  long long nc = std::max(need, e->pcap * 2);
  nc = (nc + 31) / 32 * 32;
  for (int k = 0; k < 2; ++k) {
    dev_grow(e, e->r[k], e->pcap, nc, true);
    dev_grow(e, e->v[k], e->pcap, nc, true);
    dev_grow(e, e->im[k], e->pcap, nc, true);
    dev_grow(e, e->uidx[k], e->pcap, nc, true);
  }
  dev_grow(e, e->f, e->pcap, nc, true);
  dev_grow(e, e->w, e->pcap, nc, true);
  dev_grow(e, e->sts, e->pcap, nc, true);
  dev_grow(e, e->last_r, e->pcap, nc, true);
  dev_grow(e, e->nn, e->pcap, nc, true);
  dev_grow(e, e->order, e->pcap, nc, true);
  dev_grow(e, e->key, e->pcap, nc, true);
  dev_grow(e, e->slot, e->pcap, nc, true);
  e->palloc.grow(nc);
  e->pcap = nc;
  invalidate_graphs(e, INV_POOL);
}

// The list pool; the 16-bit window list beside it only once force mode 2
// has been chosen (enable_window_list).
void grow_list(b2md_engine* e, long long need) {
  if (need <= e->ecap) return;
  long long nc = std::max(need, e->ecap + e->ecap / 2);
  dev_grow(e, e->nbl, e->ecap, nc, false);
  if (e->wl_on) dev_grow(e, e->wl, e->ecap, nc, false);
  e->ealloc.grow(nc);
  e->ecap = nc;
  invalidate_graphs(e, INV_POOL);
}

void enable_window_list(b2md_engine* e) {
  if (e->wl_on) return;
  dev_grow(e, e->wl, 0, e->ecap, false);
  e->wl_on = true;
  invalidate_graphs(e, INV_POOL);
}

void grow_cells(b2md_engine* e, long long need) {
  if (need <= e->ccap) return;
  long long nc = std::max(need, e->ccap * 2);
  dev_grow(e, e->cnt, e->ccap, nc, true);
  dev_grow(e, e->cstart, e->ccap, nc, true);
  e->calloc.grow(nc);
  e->ccap = nc;
  invalidate_graphs(e, INV_POOL);
}

void grow_params(b2md_engine* e, long long need) {
  if (need <= e->qcap) return;
  long long nc = std::max(need, std::max<long long>(e->qcap * 2, 1024));
  dev_grow(e, e->par, e->qcap, nc, true);
  e->qalloc.grow(nc);
  e->qcap = nc;
  invalidate_graphs(e, INV_POOL);
}

void grow_elog(b2md_engine* e, long long need) {
  if (need <= e->zcap) return;
  long long nc = std::max(need, e->zcap * 2);
  dev_grow(e, e->elog, e->zcap * 5, nc * 5, true);
  e->zalloc.grow(nc);
  e->zcap = nc;
  invalidate_graphs(e, INV_POOL);
}

void grow_reps(b2md_engine* e, int need) {
  if (need <= e->rcap) return;
  int nc = std::max(need, std::max(e->rcap * 2, 8));
  dev_grow(e, e->rep, e->rcap, nc, true);
  dev_grow(e, e->st, e->rcap, nc, true);
  dev_grow(e, e->rctr, 2LL * e->rcap, 2LL * nc, true);  // two halves (k_steps: by step parity)
  dev_grow(e, e->flist, 2LL * e->rcap, 2LL * nc, true);  // two halves (k_batch: by step parity)
  e->rcap = nc;
  invalidate_graphs(e, INV_POOL);
}

// Largest type count over the active replicas.
int max_types_active(const b2md_engine* e) {
  int m = 1;
  for (const auto& h : e->reps)
    if (h.active) m = std::max(m, h.d.ntypes);
  return m;
}

EngArgs make_args(b2md_engine* e) {
  EngArgs a;
  for (int k = 0; k < 2; ++k) { a.r[k] = e->r[k]; a.v[k] = e->v[k]; a.im[k] = e->im[k]; a.uidx[k] = e->uidx[k]; }
  a.f = e->f; a.w = e->w; a.sts = e->sts; a.last_r = e->last_r; a.nn = e->nn; a.nbl = e->nbl;
  a.key = e->key; a.slot = e->slot; a.order = e->order; a.cnt = e->cnt; a.cstart = e->cstart;
  a.ctot = e->ctot; a.cpref = e->cpref; a.par = e->par; a.rep = e->rep; a.st = e->st;
  a.tile_rep = e->tile_rep; a.tile_first = e->tile_first; a.tpart = e->tpart; a.gpart = e->gpart;
  a.gctr = e->gctr; a.rctr = e->rctr; a.fctr = e->fctr; a.any_rebuild = e->any_rebuild; a.elog = e->elog;
  a.ntiles = e->ntiles;
  a.nrep = (int)e->reps.size();
  a.pctl = e->pctl;
  a.gpart_half = (long long)e->gcap * kNPart;
  a.tpart_half = (long long)e->tcap * kNPart;
  a.gctr_half = e->gcap;
  a.rctr_half = e->rcap;

  // staged list tile (force mode 1): pb slots per block of 8 entries
  a.idx_pitch = e->pb;
  a.idx_rows = 0;
  a.max_types = 1;
  for (auto& h : e->reps)
    if (h.active) {
      a.idx_rows = std::max(a.idx_rows, h.d.max_nbrs);
      a.max_types = std::max(a.max_types, h.d.ntypes);
    }
  a.wl = e->wl;
  a.wseg = e->wseg;
  a.wmeta = e->wmeta;
  a.win_on = e->force_mode == FM_WINDOW ? 1 : 0;
  a.nreg = (e->sm_tiles && e->force_mode == FM_STREAMED) ? e->nsm : 0;
  a.smctr = e->smctr;
  a.win_cap = e->win_cap;
  a.wl_rows = e->force_mode == FM_WINDOW ? std::min(list_rows(a.idx_rows), e->wl_rows_cap & ~7) : 0;
  a.flist = e->flist;
  a.bshared_off = 0;
  a.split_tiles = e->split_tiles;
  a.fq = e->fq;
  a.fseq = e->fseq;
  a.qcap = e->fqcap;
  a.rb_steps_only = 0;
  return a;
}

// Dynamic shared memory of k_force: pair table [+ staged list tile | position
// window], at least the block reduction's scratch that overlays it at the end.
// Streamed blocks hold only the rows of the engine's largest type count, which
// leaves the rest of the SM's unified memory to L1.
size_t force_smem(const b2md_engine* e, const EngArgs& a) {
  const int mode = e->force_mode;
  size_t extra = 0;
  if (mode == FM_STAGED) extra = (size_t)list_rows(a.idx_rows) * a.idx_pitch * sizeof(unsigned);
  if (mode == FM_WINDOW)
    extra = (size_t)a.win_cap * sizeof(float4) + (size_t)a.wl_rows * a.idx_pitch * sizeof(unsigned short);
  const size_t table = mode == FM_STREAMED ? (size_t)a.max_types * a.max_types * kParStride * sizeof(float)
                                           : (size_t)kParSmemFloats * sizeof(float);
  const size_t need = std::max(table + extra, (size_t)force_red_bytes(e->pb * e->tp));
  return (need + 15) & ~(size_t)15;
}

// Dynamic shared memory of k_steps: the pair table, which stays loaded for
// the launch, then the reduction scratch.
size_t persist_smem(const b2md_engine* e, const EngArgs& a) {
  return (size_t)persist_table_bytes(a) + (size_t)force_red_bytes(e->pb * e->tp);
}

// Dynamic shared memory of k_rb_build: cut-off table [+ list tile] [+ window scratch].
size_t build_smem(const b2md_engine* e, const EngArgs& a) {
  const int pb = e->pb;
  return (size_t)kCs2Floats * sizeof(float) + (e->build_smem ? (size_t)list_rows(a.idx_rows) * pb * sizeof(unsigned) : 0) +
         (a.win_on ? sizeof(WinTable) : 0);
}

// Marks every tile as having no position window (k_force then streams its
// neighbours) until the next list build makes them.
void drop_windows(b2md_engine* e) {
  if (e->wmeta && e->tcap > 0) CK(cudaMemsetAsync(e->wmeta, 0xff, (size_t)e->tcap * sizeof(int2), e->stream));
}

// Tile and reduction-group tables of at least T tiles and G groups.
bool grow_tiles(b2md_engine* e, int T, int G) {
  bool grew = false;
  if (T > e->tcap) {
    int nc = std::max(T, e->tcap * 2);
    dev_grow(e, e->tile_rep, e->tcap, nc, true);
    dev_grow(e, e->tile_first, e->tcap, nc, true);
    dev_grow(e, e->ctot, e->tcap, nc, true);
    dev_grow(e, e->cpref, e->tcap, nc, true);
    dev_grow(e, e->tpart, 2LL * e->tcap * kNPart, 2LL * nc * kNPart, false);  // two halves
    dev_grow(e, e->wseg, (long long)e->tcap * kWinSeg, (long long)nc * kWinSeg, false);
    dev_grow(e, e->wmeta, e->tcap, nc, false);
    e->tcap = nc;
    grew = true;
  }
  if (G > e->gcap) {
    int nc = std::max(G, e->gcap * 2);
    dev_grow(e, e->gpart, 2LL * e->gcap * kNPart, 2LL * nc * kNPart, false);  // two halves
    dev_grow(e, e->gctr, 2LL * e->gcap, 2LL * nc, true);  // two halves
    e->gcap = nc;
    grew = true;
  }
  if (grew) invalidate_graphs(e, INV_POOL);
  return grew;
}

int persist_kind_for(b2md_engine* e);
int max_types_active(const b2md_engine* e);

// Re-lays out tiles and reduction groups over the active replicas and queues
// the upload of the tile tables, the replica table and the layout words that
// k_batch reads, through the staging ring: nothing waits for running work.
// A batched persistent graph stays valid (it reads the layout from the
// device) unless the pools moved or a replica brings more particle types
// than its shared-memory pair table holds; the other graphs capture the
// layout and are rebuilt.
void apply_layout(b2md_engine* e) {
  int T = 0, G = 0;
  for (auto& h : e->reps) {
    if (!h.active) { h.d.tile0 = T; h.d.ntiles = 0; h.d.group0 = G; h.d.ngroups = 0; h.d.active = 0; continue; }
    h.d.tile0 = T;
    h.d.ntiles = (h.n + e->pb - 1) / e->pb;
    h.d.group0 = G;
    h.d.ngroups = (h.d.ntiles + kGroup - 1) / kGroup;
    T += h.d.ntiles;
    G += h.d.ngroups;
  }
  grow_tiles(e, T, G);
  const int R = (int)e->reps.size();
  const size_t tb = ((size_t)T * sizeof(int) + 15) & ~(size_t)15;
  const size_t rb = (size_t)R * sizeof(RepDev);
  char* stage = stage_alloc(e, 2 * tb + rb + 16);
  int* trep = reinterpret_cast<int*>(stage);
  int* tfirst = reinterpret_cast<int*>(stage + tb);
  RepDev* table = reinterpret_cast<RepDev*>(stage + 2 * tb);
  int* lay = reinterpret_cast<int*>(stage + 2 * tb + rb);
  for (int r = 0; r < R; ++r) {
    const HostRep& h = e->reps[r];
    table[r] = h.d;
    for (int t = 0; t < h.d.ntiles; ++t) {
      trep[h.d.tile0 + t] = r;
      tfirst[h.d.tile0 + t] = t * e->pb;
    }
  }
  lay[0] = T;
  lay[1] = R;
  if (T > 0) {
    CK(cudaMemcpyAsync(e->tile_rep, trep, T * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->tile_first, tfirst, T * sizeof(int), cudaMemcpyHostToDevice, e->stream));
  }
  if (R > 0) CK(cudaMemcpyAsync(e->rep, table, rb, cudaMemcpyHostToDevice, e->stream));
  static_assert(offsetof(PersistCtl, lay_nrep) == offsetof(PersistCtl, lay_ntiles) + sizeof(int), "layout words");
  CK(cudaMemcpyAsync(&e->pctl->lay_ntiles, lay, 2 * sizeof(int), cudaMemcpyHostToDevice, e->stream));
  stage_commit(e);
  e->ntiles = T;
  e->ngroups = G;
  e->layout_dirty = false;
  drop_windows(e);  // tiles changed: no window until the next list build
  const bool keep = e->graphs_valid && (e->persist_kind == 2 || e->persist_kind == 3) &&
                    persist_kind_for(e) == e->persist_kind && max_types_active(e) <= e->graph_types;
  if (!keep) invalidate_graphs(e, INV_LAYOUT);
  ++e->layout_uploads;
}

// Applies admissions and removals made since the last launch, then computes
// the momentum of the replicas admitted since (before any kernel uses them).
void launch_momentum_of(b2md_engine* e, int id);
void ensure_layout(b2md_engine* e) {
  if (e->layout_dirty) apply_layout(e);
  if (!e->momentum_due.empty()) {
    std::vector<int> due;
    due.swap(e->momentum_due);
    for (int id : due)
      if (id < (int)e->reps.size() && e->reps[id].active) launch_momentum_of(e, id);
  }
}

// Re-layout now (a launch shape change).
void relayout(b2md_engine* e) {
  e->layout_dirty = true;
  ensure_layout(e);
}

void upload_rep(b2md_engine* e, int id) {
  const HostRep& h = e->reps[id];
  CK(cudaMemcpyAsync(e->rep + id, &h.d, sizeof(RepDev), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
}

HostRep& get_rep(b2md_engine* e, int id) {
  if (!e) api_fail(B2MD_ERR_ARG, "null engine");
  if (id < 0 || id >= (int)e->reps.size() || !e->reps[id].active) api_fail(B2MD_ERR_ARG, "no replica with this id");
  return e->reps[id];
}

RepState read_state(b2md_engine* e, int id) {
  RepState s;
  CK(cudaMemcpyAsync(&s, e->st + id, sizeof(RepState), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return s;
}

std::vector<RepState> read_states(b2md_engine* e) {
  std::vector<RepState> s(e->reps.size());
  if (!s.empty()) {
    CK(cudaMemcpyAsync(s.data(), e->st, s.size() * sizeof(RepState), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
  }
  return s;
}

template <class T>
void write_field(b2md_engine* e, int id, size_t off, const T& val) {
  CK(cudaMemcpyAsync(reinterpret_cast<char*>(e->st + id) + off, &val, sizeof(T), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
}
#define WRITE_STATE(e, id, field, val) write_field(e, id, offsetof(RepState, field), (decltype(RepState::field))(val))

// A RUMD parameter table's pair function, cut-off method and parameters.
void check_potential(int ntypes, const float* params, int cutoff, int potential) {
  if (ntypes < 1 || ntypes > kMaxTypes) api_fail(B2MD_ERR_ARG, "ntypes must be 1..8");
  if (cutoff < 0 || cutoff > 2) api_fail(B2MD_ERR_ARG, "cutoff method must be NS, SP or SF");
  if (potential < POT_LJ_12_6 || potential > POT_IPL_N)
    api_fail(B2MD_ERR_ARG, "pair function must be LJ 12-6, LJ 12-6 smooth 2-4 or IPL n");
  if (potential != POT_LJ_12_6)
    for (int k = 0; k < ntypes * ntypes; ++k)
      if (params[k * kNumParam] > 0.f && !(params[k * kNumParam + 1] > 0.f))
        api_fail(B2MD_ERR_ARG, "pair parameter 1 (1/sigma^2) must be positive");
}

// Cell grid (NeighborList.cu:717-732), method and minimum-image limits from
// the largest cut-off of the replica's potentials.
void derive_grid(HostRep& h);

// Sample::SetPotential (Sample.cu:251-259): the replica's potential list
// becomes this one potential (a second one added earlier is dropped).
void set_potential(HostRep& h, int ntypes, const float* params, int cutoff, float skin, int potential) {
  check_potential(ntypes, params, cutoff, potential);
  if (!(skin >= 0.f)) api_fail(B2MD_ERR_ARG, "skin must be >= 0");
  float rc = 0.f;
  for (int k = 0; k < ntypes * ntypes; ++k) rc = std::max(rc, params[k * kNumParam]);
  if (!(rc > 0.f)) api_fail(B2MD_ERR_ARG, "all cut-offs are zero");
  h.d.potential = potential;
  h.params.assign(params, params + ntypes * ntypes * kNumParam);
  h.d.ntypes = ntypes;
  h.d.cutoff = cutoff;
  h.skin = skin;
  h.params1.clear();
  h.potential1 = -1;
  h.d.npot = 1;
  h.d.potential1 = 0;
  derive_grid(h);
}

void derive_grid(HostRep& h) {
  const int ntypes = h.d.ntypes;
  const float skin = h.skin;
  h.rcmax = 0.f;
  for (int k = 0; k < ntypes * ntypes; ++k) h.rcmax = std::max(h.rcmax, h.params[k * kNumParam]);
  for (size_t k = 0; k < h.params1.size() / kNumParam; ++k) h.rcmax = std::max(h.rcmax, h.params1[k * kNumParam]);
  h.d.skin2_4 = (float)(0.25 * skin * skin);
  for (int d = 0; d < 3; ++d) h.d.ilim[d] = 0.5f * h.d.L[d] - (h.rcmax + 2.f * skin) - 0.01f;
  int ncheck[3];
  for (int d = 0; d < 3; ++d) {
    float q = 2 * h.d.L[d] / (h.rcmax + skin);
    ncheck[d] = (int)floor(q);
    h.d.nc[d] = ncheck[d] < 5 ? 5 : ncheck[d];
  }
  bool grid_complete = ncheck[0] >= 5 && ncheck[1] >= 5 && ncheck[2] >= 5;
  if (h.nb_method_req == NB_CELLS) h.d.nb_method = NB_CELLS;
  else if (h.nb_method_req == NB_N2) h.d.nb_method = NB_N2;
  else h.d.nb_method = grid_complete ? NB_CELLS : NB_N2;
}

// The engine's per-pair rows of one potential (RUMD table `params`, pair
// function `pot`, cut-off method `cutoff`).  q[6], the list build's
// (rc + skin)^2, is the larger over the replica's potentials in the first
// table (the list serves both).
std::vector<float> pack_table(const HostRep& h, const std::vector<float>& params, int pot, int cutoff) {
  int T = h.d.ntypes;
  std::vector<float> out(T * T * kParStride, 0.f);
  for (int k = 0; k < T * T; ++k) {
    const float* p = &params[k * kNumParam];
    float* q = &out[k * kParStride];
    float rc = p[0];
    const float sc = p[kNumParam - 2], uc = p[kNumParam - 1];  // s(rc)*rc, u(rc)
    // fij's cut-off terms (PairPotential.h:1208-1221) as s -= c_s/r, u += c_s r + c_u0
    const bool sf = cutoff == CUT_SF, sp = cutoff == CUT_SP;
    const float c_s = sf ? sc : 0.f;
    const float c_u0 = sf ? -(sc * rc + uc) : (sp ? -uc : 0.f);
    float cs = rc + h.skin;  // calculateNBL_*: (params + skin)^2 in float
    q[0] = rc * rc;
    q[6] = cs * cs;
    if (&params == &h.params && !h.params1.empty()) {
      const float cs1 = h.params1[k * kNumParam] + h.skin;
      q[6] = std::max(q[6], cs1 * cs1);
    }
    if (pot == POT_LJ_12_6) {
      q[1] = p[1];
      q[2] = p[2];
      q[3] = c_s;
      q[4] = c_u0;
      q[5] = c_s;
    } else if (pot == POT_LJ_12_6_SMOOTH_2_4) {
      // u = 4eps [(s/r)^12 - (s/r)^6 + c2 (r/s)^2 + c4 (r/s)^4]: the r^2 and
      // r^4 terms folded into b, c (force) and e, g (energy) per unit of d^2
      const float is2 = p[1], a = p[2], c2 = p[3], c4 = p[4];
      q[1] = rc > 0.f ? 1.f / is2 : 0.f;
      q[2] = a;
      q[3] = -2.f * c2 * a * is2;
      q[4] = -4.f * c4 * a * is2 * is2;
      q[5] = c2 * a * is2;
      q[7] = c4 * a * is2 * is2;
      q[8] = c_s;
      q[9] = c_u0;
    } else {  // POT_IPL_N: u = eps (sigma/r)^n
      q[1] = rc > 0.f ? 1.f / p[1] : 0.f;
      q[2] = p[2];
      q[3] = 0.5f * p[3];
      q[4] = p[3] * p[2];
      q[8] = c_s;
      q[9] = c_u0;
    }
  }
  return out;
}

int estimate_max_nbrs(const HostRep& h) {
  double V = (double)h.d.L[0] * h.d.L[1] * h.d.L[2];
  double rs = (double)h.rcmax + h.skin;
  double est = 1.5 * (4.0 / 3.0) * M_PI * rs * rs * rs * h.n / V;
  int m = (int)std::ceil(est);
  m = std::max(m, 32);
  m = std::min(m, std::max(h.n - 1, 1));
  return m;
}

void place_cells(b2md_engine* e, HostRep& h) {
  int ncell = h.d.nc[0] * h.d.nc[1] * h.d.nc[2];
  if (h.cell0 >= 0 && h.ncell == ncell) return;
  if (h.cell0 >= 0) e->calloc.release(h.cell0, h.ncell);
  long long off = e->calloc.alloc(ncell, 1);
  if (off < 0) {
    grow_cells(e, e->ccap + ncell);
    off = e->calloc.alloc(ncell, 1);
  }
  h.cell0 = off;
  h.ncell = ncell;
  h.d.cell0 = (int)off;
  h.d.ncell = ncell;
}

// One packed table into the parameter pool at *off (placed, or moved when
// its size changed), uploaded through the staging ring.
void place_table(b2md_engine* e, const std::vector<float>& packed, long long* off, int* len) {
  const int np = (int)packed.size();
  if (*off < 0 || *len != np) {
    if (*off >= 0) e->qalloc.release(*off, *len);
    long long o = e->qalloc.alloc(np, 8);
    if (o < 0) {
      grow_params(e, e->qcap + np + 8);
      o = e->qalloc.alloc(np, 8);
    }
    *off = o;
    *len = np;
  }
  float* stage = reinterpret_cast<float*>(stage_alloc(e, np * sizeof(float)));
  std::memcpy(stage, packed.data(), np * sizeof(float));
  CK(cudaMemcpyAsync(e->par + *off, stage, np * sizeof(float), cudaMemcpyHostToDevice, e->stream));
  stage_commit(e);
}

// The replica's packed tables: its potential's, and a second potential's.
void place_params(b2md_engine* e, HostRep& h) {
  place_table(e, pack_table(h, h.params, h.d.potential, h.d.cutoff), &h.par0, &h.npar);
  h.d.par0 = (int)h.par0;
  if (h.potential1 >= 0) {
    place_table(e, pack_table(h, h.params1, h.potential1, h.cutoff1), &h.par1, &h.npar1);
    h.d.par1 = (int)h.par1;
    h.d.npot = 2;
    h.d.potential1 = h.potential1;
  } else {
    if (h.par1 >= 0) e->qalloc.release(h.par1, h.npar1);
    h.par1 = -1;
    h.npar1 = 0;
    h.d.par1 = 0;
    h.d.npot = 1;
  }
}

void place_list(b2md_engine* e, HostRep& h, int max_nbrs) {
  long long len = (long long)list_rows(max_nbrs) * h.np;
  if (h.nbl0 >= 0) e->ealloc.release(h.nbl0, h.nbl_len);
  long long off = e->ealloc.alloc(len, 32);
  if (off < 0) {
    grow_list(e, e->ealloc.used_end() + len + 32);
    off = e->ealloc.alloc(len, 32);
    if (off < 0) api_fail(B2MD_ERR_NOMEM, "neighbour-list pool exhausted");
  }
  h.nbl0 = off;
  h.nbl_len = len;
  h.d.nbl0 = off;
  h.d.max_nbrs = max_nbrs;
  h.d.nbl_stride = h.np;
  drop_windows(e);  // window list entries live at the old place
}

// ---- launches ----
// Kernels in one rebuild sequence (launch_rebuild).
int rebuild_launches(const b2md_engine* e) { return e->force_mode == FM_WINDOW ? 9 : 8; }

void launch_rebuild(b2md_engine* e, cudaStream_t s, const EngArgs& a) {
  const int T = e->ntiles;
  const int R = (int)e->reps.size();
  if (T == 0) return;
  k_rb_clear<<<T, e->pb, 0, s>>>(a);
  k_rb_count<<<T, e->pb, 0, s>>>(a);
  k_rb_scan_local<<<T, e->pb, 0, s>>>(a);
  k_rb_scan_tiles<<<R, 256, 0, s>>>(a);
  k_rb_scatter<<<T, e->pb, 0, s>>>(a);
  k_rb_fix<<<T, e->pb, 0, s>>>(a);
  k_rb_permute<<<T, e->pb, 0, s>>>(a);
  if (a.win_on) k_rb_window<<<T, e->pb, sizeof(WinScratch), s>>>(a);
  // list build: build_lanes lanes per particle (fewer when pb*lanes would
  // exceed a block), the list either assembled in shared memory or stored
  // straight to global memory
  if (e->build_lanes == 0 && !a.win_on) {
    // one warp per cell, contiguous candidate runs per lane
    k_rb_build_runs<<<T, kRunWarps * 32, 0, s>>>(a);
    return;
  }
  if (e->build_lanes == 32 && !a.win_on) {
    // one warp per cell, candidates staged in shared memory
    const size_t cw = (size_t)kCs2Floats * sizeof(float) + (size_t)kCwWarps * kCwCand * (sizeof(float4) + sizeof(int));
    k_rb_build_cw<<<T, kCwWarps * 32, cw, s>>>(a);
    return;
  }
  const size_t smem = build_smem(e, a);
  if (smem > kMaxDynSmemBytes)
    api_fail(B2MD_ERR_NOMEM, "neighbour-list tile does not fit in shared memory: use a smaller pb");
  // (position windows need the lane build: the warp builds run it with 8 lanes)
  const int lanes = std::min(e->build_lanes == 0 || e->build_lanes == 32 ? 8 : e->build_lanes, kMaxBlock / e->pb);
#define LB(LPV)                                                                    \
  if (lanes >= LPV) {                                                              \
    if (a.win_on) {                                                                \
      if (e->build_smem) k_rb_build<LPV, true, true><<<T, e->pb * LPV, smem, s>>>(a); \
      else k_rb_build<LPV, false, true><<<T, e->pb * LPV, smem, s>>>(a);             \
    } else {                                                                       \
      if (e->build_smem) k_rb_build<LPV, true, false><<<T, e->pb * LPV, smem, s>>>(a); \
      else k_rb_build<LPV, false, false><<<T, e->pb * LPV, smem, s>>>(a);             \
    }                                                                              \
    return;                                                                        \
  }
  LB(8) LB(4) LB(2) LB(1)
#undef LB
}

typedef void (*ForceFn)(EngArgs, int, cudaGraphConditionalHandle);

template <int MODE>
ForceFn force_fn_var(int tp, bool fused, bool stress) {
#define SEL(TPV)                                                                      \
  if (tp == TPV) {                                                                    \
    if (fused) return k_force<TPV, true, false, MODE>;                                \
    return stress ? k_force<TPV, false, true, MODE> : k_force<TPV, false, false, MODE>; \
  }
  SEL(1) SEL(2) SEL(4) SEL(8)
#undef SEL
  return nullptr;
}

ForceFn force_fn_raw(int tp, bool fused, bool stress, int mode) {
  if (mode == FM_STAGED) return force_fn_var<FM_STAGED>(tp, fused, stress);
  if (mode == FM_WINDOW) return force_fn_var<FM_WINDOW>(tp, fused, stress);
  return force_fn_var<FM_STREAMED>(tp, fused, stress);
}

// The force kernel for (tp, fused, stress), allowed to use the dynamic
// shared memory the staged list tile `a` needs.
ForceFn force_fn(const b2md_engine* e, bool fused, bool stress, const EngArgs& a) {
  ForceFn fn = force_fn_raw(e->tp, fused, stress, e->force_mode);
  if (force_smem(e, a) > kMaxDynSmemBytes)
    api_fail(B2MD_ERR_NOMEM, "neighbour-list tile does not fit in shared memory: use a smaller pb");
  return fn;
}

// Lets every kernel that stages list tiles use up to kMaxDynSmemBytes of
// dynamic shared memory (set once, before any stream capture).
void init_func_attrs(int device) {
  static unsigned long long done_mask = 0ull;  // one bit per device
  const unsigned long long bit = 1ull << (device & 63);
  if (done_mask & bit) return;
  const void* builds[] = {
      (const void*)k_rb_build<1, true, false>,  (const void*)k_rb_build<2, true, false>,
      (const void*)k_rb_build<4, true, false>,  (const void*)k_rb_build<8, true, false>,
      (const void*)k_rb_build<1, false, false>, (const void*)k_rb_build<2, false, false>,
      (const void*)k_rb_build<4, false, false>, (const void*)k_rb_build<8, false, false>,
      (const void*)k_rb_build<1, true, true>,   (const void*)k_rb_build<2, true, true>,
      (const void*)k_rb_build<4, true, true>,   (const void*)k_rb_build<8, true, true>,
      (const void*)k_rb_build<1, false, true>,  (const void*)k_rb_build<2, false, true>,
      (const void*)k_rb_build<4, false, true>,  (const void*)k_rb_build<8, false, true>};
  for (const void* f : builds)
    CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemBytes));
  CK(cudaFuncSetAttribute((const void*)k_rb_build_cw, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemBytes));
  for (int mode : {FM_STAGED, FM_WINDOW})
    for (int tp : {1, 2, 4, 8})
      for (int v = 0; v < 3; ++v)
        CK(cudaFuncSetAttribute((const void*)force_fn_raw(tp, v == 0, v == 2, mode),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemBytes));
  done_mask |= bit;
}

// Grid of k_force: one block per tile, or with SM tiles as many blocks as
// fit on the GPU at once -- all SMs then hold the same number of blocks, so
// each SM's region of tiles is worked by its own blocks (blocks that find no
// tile left exit at once).
int force_grid(const b2md_engine* e, const EngArgs& a, ForceFn fn, size_t smem) {
  if (a.nreg <= 0) return e->ntiles;
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, e->pb * e->tp, smem));
  return std::max(1, std::max(per_sm, 1) * e->nsm);
}

void launch_force(b2md_engine* e, cudaStream_t s, const EngArgs& a, bool fused, bool stress) {
  if (e->ntiles == 0) return;
  ForceFn fn = force_fn(e, fused, stress, a);
  const size_t smem = force_smem(e, a);
  fn<<<force_grid(e, a, fn, smem), e->pb * e->tp, smem, s>>>(a, 0, cudaGraphConditionalHandle{});
}

void check_launch() { CK(cudaGetLastError()); }

// Builds the step graphs: [gate] -> K x { IF(rebuild) {rebuild kernels} ; fused step }.
void build_graph(b2md_engine* e, int which, int K) {
  EngArgs a = make_args(e);
  a.rb_steps_only = 1;
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  const size_t smem = force_smem(e, a);
  ForceFn fstep = force_fn(e, true, false, a);
  if (e->cond_mode) {
    std::vector<cudaGraphConditionalHandle> hs(K);
    for (int k = 0; k < K; ++k) CK(cudaGraphConditionalHandleCreate(&hs[k], g, 0, cudaGraphCondAssignDefault));
    cudaGraphNode_t prev;
    {
      cudaKernelNodeParams kp = {};
      void* args[] = {&a, &hs[0]};
      kp.func = (void*)k_gate;
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(256);
      kp.kernelParams = args;
      CK(cudaGraphAddKernelNode(&prev, g, nullptr, 0, &kp));
    }
    for (int k = 0; k < K; ++k) {
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = hs[k];
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t cnode;
      CK(cudaGraphAddNode(&cnode, g, &prev, 1, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      CK(cudaStreamBeginCaptureToGraph(e->cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      launch_rebuild(e, e->cap_stream, a);
      cudaGraph_t captured;
      CK(cudaStreamEndCapture(e->cap_stream, &captured));
      int has_next = (k + 1 < K) ? 1 : 0;
      cudaGraphConditionalHandle hn = has_next ? hs[k + 1] : cudaGraphConditionalHandle{};
      cudaKernelNodeParams kp = {};
      void* args[] = {&a, &has_next, &hn};
      kp.func = (void*)fstep;
      kp.gridDim = dim3(force_grid(e, a, fstep, smem));
      kp.blockDim = dim3(e->pb * e->tp);
      kp.sharedMemBytes = (unsigned)smem;
      kp.kernelParams = args;
      cudaGraphNode_t knode;
      CK(cudaGraphAddKernelNode(&knode, g, &cnode, 1, &kp));
      prev = knode;
    }
  } else {
    cudaGraph_t captured;
    CK(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K; ++k) {
      launch_rebuild(e, e->cap_stream, a);
      fstep<<<force_grid(e, a, fstep, smem), e->pb * e->tp, smem, e->cap_stream>>>(a, 0, cudaGraphConditionalHandle{});
    }
    CK(cudaStreamEndCapture(e->cap_stream, &captured));
    CK(cudaGraphDestroy(g));
    g = captured;
  }
  cudaGraphExec_t ex;
  CK(cudaGraphInstantiate(&ex, g, 0));
  e->graph[which] = g;
  e->gexec[which] = ex;
}

typedef void (*StepsFn)(EngArgs, cudaGraphConditionalHandle);

StepsFn steps_fn(int tp) {
  switch (tp) {
    case 1: return k_steps<1>;
    case 2: return k_steps<2>;
    case 4: return k_steps<4>;
    default: return k_steps<8>;
  }
}

// Runs may use a persistent step graph: streamed force mode, no SM-region
// tile claiming, conditional graph nodes.
bool persist_mode(const b2md_engine* e) {
  return e->persist != 0 && e->cond_mode && e->force_mode == FM_STREAMED && !e->sm_tiles;
}

typedef void (*BatchFn)(EngArgs, cudaGraphConditionalHandle);

BatchFn batch_fn(int tp) {
  switch (tp) {
    case 1: return k_batch<1>;
    case 2: return k_batch<2>;
    case 4: return k_batch<4>;
    default: return k_batch<8>;
  }
}

BatchFn flow_fn(int tp) {
  switch (tp) {
    case 1: return k_flow<1>;
    case 2: return k_flow<2>;
    case 4: return k_flow<4>;
    default: return k_flow<8>;
  }
}

// k_flow's item queue: more slots than items can be outstanding (at most one
// phase of every replica, no more than the tiles, plus a ticket per block),
// twice over.  Slots start unpublished (zero); tickets never repeat.
void ensure_flow_queue(b2md_engine* e) {
  const long long need = 2LL * ((long long)e->tcap + 32LL * std::max(e->nsm, 1)) + 1024;
  if (need <= (long long)e->fqcap) return;
  dev_grow(e, e->fq, e->fqcap, need, true);
  dev_grow(e, e->fseq, e->fqcap, need, true);
  e->fqcap = (unsigned)need;
  invalidate_graphs(e, INV_POOL);
}

// k_batch applies when one block can hold a replica's sort and the step's
// rebuild list: at most kBatchMaxRep replicas of at most kBatchMaxN
// particles each.
bool batch_eligible(const b2md_engine* e) {
  if ((int)e->reps.size() > kBatchMaxRep) return false;
  for (const auto& h : e->reps)
    if (h.active && h.n > kBatchMaxN) return false;
  return true;
}

// The persistent kernels evaluate one potential per replica; a replica with
// a second one runs on the per-step graphs (k_force adds its sums).
bool single_potential(const b2md_engine* e) {
  for (const auto& h : e->reps)
    if (h.active && h.d.npot > 1) return false;
  return true;
}

// Dynamic shared memory of k_batch: the larger of the force tile's region and
// the list build's, then the per-block rebuild-list tables.
size_t batch_smem(const b2md_engine* e, EngArgs& a) {
  const size_t build = (size_t)kCs2Floats * sizeof(float) + (size_t)(e->pb * e->tp / 32) * 32 * kRunStride * sizeof(int);
  const size_t tile = std::max(force_smem(e, a), build);
  a.bshared_off = (int)((tile + 15) & ~(size_t)15);
  return (size_t)a.bshared_off + sizeof(BatchShared);
}

// Dynamic shared memory of k_flow: the larger of the force tile's region and
// the list build's.
size_t flow_smem(const b2md_engine* e, const EngArgs& a) {
  const size_t build = (size_t)kCs2Floats * sizeof(float) + (size_t)(e->pb * e->tp / 32) * 32 * kRunStride * sizeof(int);
  return (std::max(force_smem(e, a), build) + 15) & ~(size_t)15;
}

// Grid of k_steps: every block resident at once (the launch is cooperative),
// at most one block per tile.
int steps_grid(const b2md_engine* e, StepsFn fn, size_t smem) {
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, e->pb * e->tp, smem));
  if (per_sm < 1) api_fail(B2MD_ERR_NOMEM, "the persistent step kernel does not fit on an SM: use a smaller pb*tp");
  return std::max(1, std::min(e->ntiles, per_sm * e->nsm));
}

// The persistent step graph:
//   gate_loop -> WHILE(loop) { rebuild kernels -> k_steps }
// k_steps runs fused steps with a grid barrier between them until a list
// rebuild is due, the step budget (pctl->budget, written by the host before
// each launch) is spent or no replica has steps left, and sets the loop
// condition.  The rebuild kernels act on the replicas whose rebuild flag is
// set and exit at once otherwise.  Between rebuilds the steps cost one grid
// barrier each instead of a conditional node and a kernel launch.
void build_persist_graph(b2md_engine* e) {
  EngArgs a = make_args(e);
  a.rb_steps_only = 1;
  const size_t smem = persist_smem(e, a);
  force_fn(e, true, false, a);  // checks the shared-memory need
  StepsFn fs = steps_fn(e->tp);
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hl;
  CK(cudaGraphConditionalHandleCreate(&hl, g, 0, cudaGraphCondAssignDefault));
  cudaGraphNode_t gate;
  {
    cudaKernelNodeParams kp = {};
    void* args[] = {&a, &hl};
    kp.func = (void*)k_gate_loop;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(256);
    kp.kernelParams = args;
    CK(cudaGraphAddKernelNode(&gate, g, nullptr, 0, &kp));
  }
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hl;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, g, &gate, 1, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  // the loop body: the rebuild kernels (each exits at once for replicas
  // whose rebuild flag is clear: k_steps stops only when one is due, or at
  // the budget, or at the start of the run), then k_steps
  CK(cudaStreamBeginCaptureToGraph(e->cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_rebuild(e, e->cap_stream, a);
  cudaStreamCaptureStatus cst;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  CK(cudaStreamGetCaptureInfo(e->cap_stream, &cst, nullptr, nullptr, &deps, &ndeps));
  std::vector<cudaGraphNode_t> leaf(deps, deps + ndeps);
  cudaGraph_t captured;
  CK(cudaStreamEndCapture(e->cap_stream, &captured));
  {
    cudaKernelNodeParams kp = {};
    void* args[] = {&a, &hl};
    kp.func = (void*)fs;
    kp.gridDim = dim3(steps_grid(e, fs, smem));
    kp.blockDim = dim3(e->pb * e->tp);
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = args;
    cudaGraphNode_t knode;
    CK(cudaGraphAddKernelNode(&knode, body, leaf.data(), leaf.size(), &kp));
    cudaKernelNodeAttrValue av = {};
    av.cooperative = 1;
    CK(cudaGraphKernelNodeSetAttribute(knode, cudaKernelNodeAttributeCooperative, &av));
  }
  cudaGraphExec_t ex;
  CK(cudaGraphInstantiate(&ex, g, 0));
  e->graph[2] = g;
  e->gexec[2] = ex;
}

// The batched persistent graph:
//   gate_loop -> WHILE(loop) { k_batch }
// k_batch runs whole steps -- the list rebuilds of the replicas whose lists
// are due included -- with one grid barrier per step, until the budget is
// spent, no replica has steps left or a list overflows (the host repairs it
// and launches again).
void build_batch_graph(b2md_engine* e, bool flow) {
  if (flow) ensure_flow_queue(e);
  EngArgs a = make_args(e);
  e->graph_types = a.max_types;
  const size_t smem = flow ? flow_smem(e, a) : batch_smem(e, a);
  force_fn(e, true, false, a);  // checks the shared-memory need
  BatchFn fb = flow ? flow_fn(e->tp) : batch_fn(e->tp);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fb, e->pb * e->tp, smem));
  if (per_sm < 1) api_fail(B2MD_ERR_NOMEM, "the batched step kernel does not fit on an SM: use a smaller pb*tp");
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hl;
  CK(cudaGraphConditionalHandleCreate(&hl, g, 0, cudaGraphCondAssignDefault));
  cudaGraphNode_t gate;
  {
    cudaKernelNodeParams kp = {};
    void* args[] = {&a, &hl};
    kp.func = (void*)k_gate_loop;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(256);
    kp.kernelParams = args;
    CK(cudaGraphAddKernelNode(&gate, g, nullptr, 0, &kp));
  }
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hl;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, g, &gate, 1, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  {
    cudaKernelNodeParams kp = {};
    void* args[] = {&a, &hl};
    kp.func = (void*)fb;
    kp.gridDim = dim3(std::max(1, per_sm * e->nsm));
    kp.blockDim = dim3(e->pb * e->tp);
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = args;
    cudaGraphNode_t knode;
    CK(cudaGraphAddKernelNode(&knode, body, nullptr, 0, &kp));
    cudaKernelNodeAttrValue av = {};
    av.cooperative = 1;
    CK(cudaGraphKernelNodeSetAttribute(knode, cudaKernelNodeAttributeCooperative, &av));
  }
  cudaGraphExec_t ex;
  CK(cudaGraphInstantiate(&ex, g, 0));
  e->graph[2] = g;
  e->gexec[2] = ex;
}

// Which persistent kernel runs the steps: 1 k_steps (every tile has a
// resident block), 3 k_flow (more tiles than resident blocks, or asked for
// with persistent = 3), 2 k_batch (asked for with persistent = 2), 0 none
// (one launch per step).  k_flow, whose replicas step on their own, measured
// 1.7-2.7x faster than k_batch's one step barrier for all replicas (4 x 32768
// KA: 87 vs 148 us per step; 16 x 8192: 74 vs 179; 64 x 2048: 72 vs 192).
int persist_kind_for(b2md_engine* e) {
  if (!persist_mode(e) || e->ntiles == 0 || e->reps.size() >= (1u << 20)) return 0;  // the barrier tally fields
  if (!single_potential(e)) return 0;
  if (e->persist == 3) return batch_eligible(e) ? 3 : 0;
  if (e->persist == 1) {
    EngArgs a = make_args(e);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)steps_fn(e->tp), e->pb * e->tp,
                                                     persist_smem(e, a)));
    if ((long long)per_sm * e->nsm >= e->ntiles) return 1;
    return batch_eligible(e) ? 3 : 0;
  }
  return batch_eligible(e) ? 2 : 0;
}

// The persistent graph is used when the whole tile set is resident at once
// (one tile per block): with several tiles per block its fixed tile order
// balances worse than the hardware's block scheduling (2.12e9 vs 2.26e9
// particle-steps/s for LJ at N = 1M), while with one tile per block it saves
// the per-step launch (1.2455e9 vs 1.2335e9 for KA at N = 65536).
void ensure_graphs(b2md_engine* e) {
  if (e->graphs_valid) return;
  invalidate_graphs(e);
  e->persist_kind = persist_kind_for(e);
  e->persist_on = e->persist_kind != 0;
  if (e->persist_kind == 1) {
    build_persist_graph(e);
  } else if (e->persist_kind == 2 || e->persist_kind == 3) {
    build_batch_graph(e, e->persist_kind == 3);
  } else {
    build_graph(e, 0, 1);
    build_graph(e, 1, kChunk);
  }
  e->graphs_valid = true;
  ++e->graph_builds;
}

// A step-barrier wait of k_steps that gave up (reported, then cleared).
void check_persist(b2md_engine* e) {
  int err = 0;
  CK(cudaMemcpy(&err, &e->pctl->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    CK(cudaMemset(&e->pctl->err, 0, sizeof(int)));
    api_fail(B2MD_ERR_CUDA, "a step-barrier wait of the persistent step kernel gave up");
  }
}

// Overflowed lists: double the capacity (NeighborList.cu:657-676) and flag a rebuild.
bool repair_overflow(b2md_engine* e) {
  std::vector<RepState> s = read_states(e);
  bool any = false;
  for (size_t r = 0; r < e->reps.size(); ++r)
    if (e->reps[r].active && s[r].err)
      api_fail(B2MD_ERR_CUDA, "a bounded device wait for the neighbour-list copy gave up (replica " +
                                  std::to_string(r) + ")");
  for (size_t r = 0; r < e->reps.size(); ++r) {
    HostRep& h = e->reps[r];
    if (!h.active || !s[r].overflow) continue;
    int want = std::max(h.d.max_nbrs * 2, s[r].actual_max_nbrs + 8);
    want = std::min(want, std::max(h.n - 1, 1));
    if (want <= h.d.max_nbrs) api_fail(B2MD_ERR_OVERFLOW, "neighbour list cannot grow further");
    place_list(e, h, want);
    upload_rep(e, (int)r);
    WRITE_STATE(e, (int)r, overflow, 0);
    WRITE_STATE(e, (int)r, rebuild, 1);
    any = true;
    ++e->list_repairs;
  }
  // The graphs read each replica's list place and capacity from the replica
  // table, and a pool growth has dropped them already; only the variants that
  // size shared memory by the longest list (staged list tiles, position
  // windows, a build assembling its tile in shared memory) must be rebuilt.
  if (any && (e->force_mode != FM_STREAMED || e->build_smem)) invalidate_graphs(e, INV_REPAIR);
  return any;
}

void calc_f(b2md_engine* e, bool stress) {
  ensure_layout(e);
  for (int attempt = 0; attempt < 8; ++attempt) {
    EngArgs a = make_args(e);
    launch_rebuild(e, e->stream, a);
    launch_force(e, e->stream, a, false, stress);
    check_launch();
    if (!repair_overflow(e)) return;
  }
  api_fail(B2MD_ERR_OVERFLOW, "neighbour list overflow persists");
}

long long max_steps_left(b2md_engine* e) {
  std::vector<RepState> s = read_states(e);
  long long m = 0;
  for (size_t r = 0; r < e->reps.size(); ++r)
    if (e->reps[r].active && !s[r].overflow) m = std::max(m, s[r].steps_left);
  return m;
}

// Runs up to `limit` steps of the queued work with the step graphs.
long long run_steps(b2md_engine* e, long long limit) {
  ensure_layout(e);
  long long done = 0;
  for (int guard = 0; guard < 64; ++guard) {
    long long todo = std::min(max_steps_left(e), limit - done);
    if (todo <= 0) break;
    ensure_graphs(e);
    if (e->persist_on) {
      todo = std::min<long long>(todo, 1 << 30);
      *e->h_budget = (int)todo;
      CK(cudaMemcpyAsync(&e->pctl->budget, e->h_budget, sizeof(int), cudaMemcpyHostToDevice, e->stream));
      CK(cudaGraphLaunch(e->gexec[2], e->stream));
      CK(cudaStreamSynchronize(e->stream));
      check_persist(e);
    } else {
      long long big = todo / kChunk, small = todo % kChunk;
      for (long long k = 0; k < big; ++k) CK(cudaGraphLaunch(e->gexec[1], e->stream));
      for (long long k = 0; k < small; ++k) CK(cudaGraphLaunch(e->gexec[0], e->stream));
      CK(cudaStreamSynchronize(e->stream));
    }
    done += todo;
    if (!repair_overflow(e)) {
      // replicas that were frozen by an overflow keep their queue; others are done
      if (max_steps_left(e) == 0) break;
    }
    done = std::min(done, limit);
  }
  return done;
}

template <class F>
int guarded(F&& fn) {
  try {
    fn();
    return B2MD_OK;
  } catch (const ApiErr& x) {
    g_err = x.msg;
    return x.code;
  } catch (const CudaErr& x) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %s (%s) at engine.cu:%d: %s", cudaGetErrorName(x.e),
             cudaGetErrorString(x.e), x.line, x.what);
    g_err = buf;
    cudaGetLastError();
    return x.e == cudaErrorMemoryAllocation ? B2MD_ERR_NOMEM : B2MD_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return B2MD_ERR_NOMEM;
  }
}

// Waits for a chunk of b2md_run_queued_async and checks what it left: a
// step-barrier wait that gave up is reported; overflowed lists are enlarged
// and flagged for a rebuild (their replicas continue in the next chunk).
long long replica_bytes(const b2md_engine* e, const HostRep& h);
void finish_chunk(b2md_engine* e, ChunkRec& c) {
  CK(cudaEventSynchronize(c.done));
  c.waited = true;
  if (c.h_ctl->err) {
    CK(cudaStreamSynchronize(e->stream));
    check_persist(e);  // clears the flag and reports
  }
  c.ran = c.persistent ? c.budget - c.h_ctl->budget : c.budget;
  // overflowed lists, from the snapshot and without waiting for the chunk
  // in flight (it skips replicas flagged as overflowed): the list is placed
  // anew, the replica's descriptor uploaded through the staging ring and its
  // flags reset in stream order; a later snapshot still showing the flag
  // (taken before the reset) is not repaired twice
  bool any = false;
  for (size_t r = 0; r < c.active.size() && r < e->reps.size(); ++r) {
    HostRep& h = e->reps[r];
    if (!c.active[r] || !h.active || h.admit_seq >= c.ticket) continue;  // not the replica the chunk ran
    const RepState& st = c.h_st[r];
    if (st.err)
      api_fail(B2MD_ERR_CUDA, "a bounded device wait for the neighbour-list copy gave up (replica " +
                                  std::to_string(r) + ")");
    if (!st.overflow || h.repair_seq >= c.ticket) continue;
    int want = std::max(h.d.max_nbrs * 2, st.actual_max_nbrs + 8);
    want = std::min(want, std::max(h.n - 1, 1));
    if (want <= h.d.max_nbrs) api_fail(B2MD_ERR_OVERFLOW, "neighbour list cannot grow further");
    place_list(e, h, want);
    h.bytes = replica_bytes(e, h);
    RepDev* d = reinterpret_cast<RepDev*>(stage_alloc(e, sizeof(RepDev)));
    *d = h.d;
    CK(cudaMemcpyAsync(e->rep + r, d, sizeof(RepDev), cudaMemcpyHostToDevice, e->stream));
    stage_commit(e);
    k_clear_overflow<<<1, 1, 0, e->stream>>>(e->st + r);
    check_launch();
    h.repair_seq = e->chunk_seq;
    ++e->list_repairs;
    any = true;
  }
  if (any && (e->force_mode != FM_STREAMED || e->build_smem)) invalidate_graphs(e, INV_REPAIR);
}

ChunkRec* find_chunk(b2md_engine* e, long long ticket) {
  for (auto& c : e->chunk)
    if (c.ticket == ticket && ticket > 0) return &c;
  api_fail(B2MD_ERR_ARG, "no chunk with this ticket (only the two most recent are kept)");
}

// A replica's host record from its description: validated, potential
// packed and cell grid derived, nothing placed yet.
HostRep describe(const b2md_replica_desc* d) {
  if (d->n < 2) api_fail(B2MD_ERR_ARG, "need at least 2 particles");
  for (int k = 0; k < 3; ++k)
    if (!(d->box[k] > 0.f)) api_fail(B2MD_ERR_ARG, "box lengths must be positive");
  if (!d->params) api_fail(B2MD_ERR_ARG, "params is null");
  if (!(d->dt > 0.f)) api_fail(B2MD_ERR_ARG, "dt must be positive");
  HostRep h;
  h.n = d->n;
  h.np = (d->n + 31) / 32 * 32;
  h.d.n = d->n;
  for (int k = 0; k < 3; ++k) {
    h.d.L[k] = d->box[k];
    h.d.invL[k] = 1.f / d->box[k];
  }
  set_potential(h, d->ntypes, d->params, d->cutoff_method, d->skin, d->potential);
  h.d.dt = d->dt;
  h.d.omega2 = (float)(4. * M_PI * M_PI / (d->tau * d->tau));
  h.d.thermo_mask = d->thermostat_mask;
  h.d.reset_interval = d->reset_interval;
  h.d.dof = 3.0 * d->n - 3.0;
  h.d.energy_interval = d->energy_interval;
  h.d.active = 1;
  return h;
}

int list_capacity(const HostRep& h, const b2md_replica_desc* d) {
  return d->max_nbrs > 0 ? d->max_nbrs : estimate_max_nbrs(h);
}

// Device bytes per particle slot: r, v, images and ids double-buffered,
// forces, virials, stresses, last-build positions, list length, sort order,
// cell keys and slots.
constexpr long long kSlotBytes = 2 * (3 * sizeof(float4) + sizeof(unsigned)) + 4 * sizeof(float4) + 4 * sizeof(int);

// Device bytes replica h holds in the engine's pools (its slots, its list
// -- and window list once force mode 2 is in use --, cells, pair table,
// energy log, tile and group tables and its replica-table entries).
long long replica_bytes(const b2md_engine* e, const HostRep& h) {
  const long long nt = (h.n + e->pb - 1) / e->pb, ng = (nt + kGroup - 1) / kGroup;
  long long b = (long long)h.np * kSlotBytes;
  b += (long long)list_rows(h.d.max_nbrs) * h.np * (long long)(sizeof(unsigned) + (e->wl_on ? sizeof(unsigned short) : 0));
  b += (long long)h.ncell * 2 * sizeof(int);
  b += (long long)h.d.npot * h.d.ntypes * h.d.ntypes * kParStride * sizeof(float);
  b += (long long)h.ecap * 5 * sizeof(double);
  b += nt * (long long)(4 * sizeof(int) + 2 * kNPart * sizeof(double) + kWinSeg * sizeof(int4) + sizeof(int2));
  b += ng * (long long)(2 * kNPart * sizeof(double) + 2 * sizeof(unsigned));
  b += (long long)(sizeof(RepDev) + sizeof(RepState) + 4 * sizeof(int));
  return b;
}

// RUMD's launch shapes mapped onto the engine's: tiles are whole warps (pb
// rounded up to a multiple of 32, at most 512) and tp is a power of two up
// to 8 (the largest one <= the request), halved until pb * tp <= 512.  RUMD's
// autotuner tries pb in {16, 32, 48, 64, 96, 128, 192} and tp up to 64
// (Autotune.py:156-158); e.g. (16, 4) -> (32, 4), (48, 1) -> (64, 1),
// (192, 8) -> (192, 2), (64, 64) -> (64, 8).  False for pb < 1 or tp < 1 or
// sizes far outside those ranges.
bool map_launch(int pb, int tp, int* pb_out, int* tp_out) {
  if (pb < 1 || pb > 1024 || tp < 1 || tp > 64) return false;
  int p = std::min((pb + 31) / 32 * 32, kMaxBlock);
  int t = 8;
  while (t > tp) t >>= 1;
  while (t > 1 && p * t > kMaxBlock) t >>= 1;
  *pb_out = p;
  *tp_out = t;
  return true;
}

void launch_momentum(b2md_engine* e) {
  ensure_layout(e);
  if (e->ntiles == 0) return;
  EngArgs a = make_args(e);
  k_momentum<<<e->ntiles, e->pb * e->tp, 0, e->stream>>>(a, e->tp, 0);
  check_launch();
}

// The momentum of one replica's velocities (after its admission).
void launch_momentum_of(b2md_engine* e, int id) {
  const HostRep& h = e->reps[id];
  if (h.d.ntiles == 0) return;
  EngArgs a = make_args(e);
  k_momentum<<<h.d.ntiles, e->pb * e->tp, 0, e->stream>>>(a, e->tp, h.d.tile0);
  check_launch();
}

}  // namespace

// Lets other translation units of the library report a message through
// b2md_last_error (not exported).
namespace b2md_internal {
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace b2md_internal

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* b2md_last_error(void) { return g_err.c_str(); }
const char* b2md_version(void) { return "rumd_b200 0.1 (sm_100a)"; }

int b2md_engine_create(int device, long long max_particles, int max_replicas, long long max_list_entries,
                       int pb, int tp, b2md_engine** out) {
  if (!out) return fail(B2MD_ERR_ARG, "out is null");
  *out = nullptr;
  if (!map_launch(pb, tp, &pb, &tp)) return fail(B2MD_ERR_ARG, "pb must be 1..1024 and tp 1..64 (got %d, %d)", pb, tp);
  b2md_engine* e = new b2md_engine();
  int rc = guarded([&] {
    CK(cudaSetDevice(device));
    e->device = device;
    CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));
    e->pb = pb;
    e->tp = tp;
    e->palloc.init(0);
    e->ealloc.init(0);
    e->calloc.init(0);
    e->qalloc.init(0);
    e->zalloc.init(0);
    grow_particles(e, std::max<long long>(max_particles, 32));
    grow_list(e, std::max<long long>(max_list_entries, 1024));
    // cells, pair tables and tile tables for the expected particles and
    // replicas, so that admissions up to them do not grow (and move) a pool
    const long long R = std::max(max_replicas, 1);
    grow_cells(e, std::max<long long>(1024, max_particles / 2 + 128 * R));
    grow_params(e, std::max<long long>(1024, 64 * R));
    grow_elog(e, 16);
    grow_reps(e, (int)R);
    if (max_particles > 0) {
      const long long T = std::min<long long>(max_particles / pb + R, 1 << 30);
      grow_tiles(e, (int)T, (int)(T / kGroup + R));
    }
    // pinned staging for the expected particles, so that admissions and
    // read-backs do not allocate it later
    if (max_particles > 0) {
      host_stage(e, (size_t)max_particles * kStagePerParticle);
      ring_reserve(e, std::min<size_t>(std::max<size_t>((size_t)max_particles * 64, (size_t)4 << 20),
                                       (size_t)64 << 20));
    }
    init_func_attrs(device);
    CK(cudaMalloc(&e->fctr, sizeof(unsigned)));
    CK(cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, device));
    CK(cudaMalloc(&e->smctr, (e->nsm + 1) * sizeof(unsigned)));
    CK(cudaMemsetAsync(e->smctr, 0, (e->nsm + 1) * sizeof(unsigned), e->stream));
    // [0]: "a replica needs a rebuild" raised by the step kernel;
    // [1]: the same decision read by the host in b2md_run_timed
    CK(cudaMalloc(&e->any_rebuild, 2 * sizeof(int)));
    CK(cudaMalloc(&e->pctl, sizeof(PersistCtl)));
    CK(cudaMemsetAsync(e->pctl, 0, sizeof(PersistCtl), e->stream));
    CK(cudaMallocHost(&e->h_budget, sizeof(int)));
    CK(cudaMemsetAsync(e->fctr, 0, sizeof(unsigned), e->stream));
    CK(cudaMemsetAsync(e->any_rebuild, 0, 2 * sizeof(int), e->stream));
    CK(cudaStreamSynchronize(e->stream));
  });
  if (rc != B2MD_OK) {
    b2md_engine_destroy(e);
    return rc;
  }
  *out = e;
  return B2MD_OK;
}

int b2md_engine_destroy(b2md_engine* e) {
  if (!e) return B2MD_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  invalidate_graphs(e);
  void* ptrs[] = {e->r[0], e->r[1], e->v[0], e->v[1], e->im[0], e->im[1], e->uidx[0], e->uidx[1], e->f, e->w,
                  e->sts, e->last_r, e->nn, e->order, e->key, e->slot, e->nbl, e->cnt, e->cstart, e->par, e->elog,
                  e->rep, e->st, e->rctr, e->tile_rep, e->tile_first, e->ctot, e->cpref, e->tpart, e->gpart,
                  e->gctr, e->fctr, e->any_rebuild, e->wl, e->wseg, e->wmeta, e->smctr, e->pctl, e->flist,
                  e->fq, e->fseq};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (e->h_budget) cudaFreeHost(e->h_budget);
  if (e->h_stage) cudaFreeHost(e->h_stage);
  ring_reset(e);
  if (e->ring) cudaFreeHost(e->ring);
  for (auto& c : e->chunk) {
    if (c.done) cudaEventDestroy(c.done);
    if (c.h_in) cudaFreeHost(c.h_in);
    if (c.h_ctl) cudaFreeHost(c.h_ctl);
    if (c.h_st) cudaFreeHost(c.h_st);
  }
  if (e->stream) cudaStreamDestroy(e->stream);
  if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
  delete e;
  return B2MD_OK;
}

int b2md_engine_set_launch(b2md_engine* e, int pb, int tp) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  if (!map_launch(pb, tp, &pb, &tp)) return fail(B2MD_ERR_ARG, "pb must be 1..1024 and tp 1..64 (got %d, %d)", pb, tp);
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    e->pb = pb;
    e->tp = tp;
    invalidate_graphs(e);
    for (auto& h : e->reps)
      if (h.active) h.bytes = replica_bytes(e, h);
    relayout(e);
  });
}

int b2md_engine_get_launch(b2md_engine* e, int* pb, int* tp) {
  if (!e || !pb || !tp) return fail(B2MD_ERR_ARG, "null argument");
  *pb = e->pb;
  *tp = e->tp;
  return B2MD_OK;
}

int b2md_engine_memory(b2md_engine* e, long long* bytes) {
  if (!e || !bytes) return fail(B2MD_ERR_ARG, "null argument");
  *bytes = e->bytes;
  return B2MD_OK;
}

int b2md_engine_set_graph_mode(b2md_engine* e, int conditional) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  e->cond_mode = conditional ? 1 : 0;
  invalidate_graphs(e);
  return B2MD_OK;
}

int b2md_engine_set_variant(b2md_engine* e, int which, int value) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  switch (which) {
    case B2MD_VARIANT_FORCE_MODE:
      if (value < FM_STREAMED || value > FM_WINDOW) return fail(B2MD_ERR_ARG, "force mode must be 0, 1 or 2");
      if (value == FM_WINDOW && e->force_mode != FM_WINDOW) {
        // windows of earlier builds may be stale: none until the next list
        // build, which also makes the window list (allocated now)
        int rc = guarded([&] {
          CK(cudaSetDevice(e->device));
          enable_window_list(e);
          drop_windows(e);
        });
        if (rc) return rc;
      }
      e->force_mode = value;
      break;
    case B2MD_VARIANT_WINDOW_LIST_ROWS:
      if (value < 0 || value > 1024 || value % 8 != 0)
        return fail(B2MD_ERR_ARG, "window-list rows must be a multiple of 8 in 0..1024 (got %d)", value);
      e->wl_rows_cap = value;
      break;
    case B2MD_VARIANT_SM_TILES:
      if (value != 0 && value != 1) return fail(B2MD_ERR_ARG, "sm_tiles must be 0 or 1");
      e->sm_tiles = value != 0;
      break;
    case B2MD_VARIANT_WINDOW_CAP:
      if (value < 256 || value > kMaxWindow)
        return fail(B2MD_ERR_ARG, "window capacity must be 256..%d particles (got %d)", kMaxWindow, value);
      if (value != e->win_cap) {
        int rc = guarded([&] { drop_windows(e); });
        if (rc) return rc;
      }
      e->win_cap = value;
      break;
    case B2MD_VARIANT_BUILD_LANES:
      if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 32)
        return fail(B2MD_ERR_ARG,
                    "build lanes must be 0 (row scan, one thread per particle), 1, 2, 4, 8 or 32 (one warp per "
                    "cell) (got %d)", value);
      e->build_lanes = value;
      break;
    case B2MD_VARIANT_BUILD_SMEM:
      if (value != 0 && value != 1) return fail(B2MD_ERR_ARG, "build_smem must be 0 or 1");
      e->build_smem = value != 0;
      break;
    case B2MD_VARIANT_PERSISTENT:
      if (value < 0 || value > 3) return fail(B2MD_ERR_ARG, "persistent must be 0, 1, 2 or 3");
      e->persist = value;
      break;
    case B2MD_VARIANT_PERSISTENT_ACTIVE:
      return fail(B2MD_ERR_ARG, "persistent_active is read-only");
    case B2MD_VARIANT_GRAPH_BUILDS:
      return fail(B2MD_ERR_ARG, "graph_builds is read-only");
    case B2MD_VARIANT_SPLIT_SORT_TILES:
      if (value < 1) return fail(B2MD_ERR_ARG, "split_sort_tiles must be >= 1 (got %d)", value);
      e->split_tiles = value;
      break;
    default:
      return fail(B2MD_ERR_ARG, "unknown variant %d", which);
  }
  invalidate_graphs(e);
  return B2MD_OK;
}

int b2md_engine_get_variant(b2md_engine* e, int which, int* value) {
  if (!e || !value) return fail(B2MD_ERR_ARG, "null argument");
  switch (which) {
    case B2MD_VARIANT_FORCE_MODE: *value = e->force_mode; break;
    case B2MD_VARIANT_SM_TILES: *value = e->sm_tiles ? 1 : 0; break;
    case B2MD_VARIANT_WINDOW_LIST_ROWS: *value = e->wl_rows_cap; break;
    case B2MD_VARIANT_WINDOW_CAP: *value = e->win_cap; break;
    case B2MD_VARIANT_BUILD_LANES: *value = e->build_lanes; break;
    case B2MD_VARIANT_BUILD_SMEM: *value = e->build_smem ? 1 : 0; break;
    case B2MD_VARIANT_PERSISTENT: *value = e->persist; break;
    case B2MD_VARIANT_PERSISTENT_ACTIVE: *value = (e->graphs_valid && e->persist_on) ? e->persist_kind : 0; break;
    case B2MD_VARIANT_GRAPH_BUILDS: *value = e->graph_builds; break;
    case B2MD_VARIANT_SPLIT_SORT_TILES: *value = e->split_tiles; break;
    default: return fail(B2MD_ERR_ARG, "unknown variant %d", which);
  }
  return B2MD_OK;
}

int b2md_replica_add(b2md_engine* e, const b2md_replica_desc* d, const float* pos4, const float* vel4,
                     const int* im3, int* id_out) {
  if (!e || !d || !pos4 || !id_out) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    HostRep h = describe(d);
    // types must be in range, inverse masses positive
    for (int i = 0; i < d->n; ++i) {
      int t;
      std::memcpy(&t, &pos4[4 * i + 3], 4);
      if (t < 0 || t >= d->ntypes) api_fail(B2MD_ERR_ARG, "particle type out of range");
    }
    if (vel4)
      for (int i = 0; i < h.n; ++i)
        if (!(vel4[4 * i + 3] > 0.f)) api_fail(B2MD_ERR_ARG, "inverse mass (vel4[.,3]) must be positive");
    int id = -1;
    for (size_t r = 0; r < e->reps.size(); ++r)
      if (!e->reps[r].active) { id = (int)r; break; }
    if (id < 0) {
      id = (int)e->reps.size();
      grow_reps(e, id + 1);
      e->reps.emplace_back();
    }
    // particle segment
    long long p0 = e->palloc.alloc(h.np, 32);
    if (p0 < 0) {
      grow_particles(e, e->palloc.used_end() + h.np + 32);
      p0 = e->palloc.alloc(h.np, 32);
      if (p0 < 0) api_fail(B2MD_ERR_NOMEM, "particle pool exhausted");
    }
    h.p0 = p0;
    h.d.p0 = (int)p0;
    place_cells(e, h);
    place_params(e, h);
    place_list(e, h, list_capacity(h, d));
    if (d->energy_interval > 0 && d->energy_capacity > 0) {
      long long z = e->zalloc.alloc(d->energy_capacity, 1);
      if (z < 0) {
        grow_elog(e, e->zalloc.used_end() + d->energy_capacity);
        z = e->zalloc.alloc(d->energy_capacity, 1);
      }
      h.elog0 = z;
      h.ecap = d->energy_capacity;
      h.d.elog0 = z;
      h.d.energy_cap = d->energy_capacity;
    } else {
      h.d.energy_interval = 0;
      h.d.energy_cap = 0;
    }
    h.active = true;
    h.bytes = replica_bytes(e, h);
    // particle data (slot order = original order until the first sort).
    // Arrays the caller already pinned are copied from directly, and the
    // call then returns when the copies are done; otherwise r, v and the
    // images are packed into the staging ring, as the device stores them,
    // and the call returns at once -- the copies run after the work already
    // queued (a running chunk), before the next launch.  last_r and the ids
    // are made on the device.
    const size_t nb = (size_t)h.n * sizeof(float4);
    const bool direct = is_pinned(pos4) && vel4 && is_pinned(vel4);
    const float4* sr = reinterpret_cast<const float4*>(pos4);
    const float4* sv = reinterpret_cast<const float4*>(vel4);
    if (!direct) {
      char* stage = stage_alloc(e, 2 * nb);
      float4* r = reinterpret_cast<float4*>(stage);
      float4* v = reinterpret_cast<float4*>(stage + nb);
      std::memcpy(r, pos4, nb);
      if (vel4) std::memcpy(v, vel4, nb);
      else
        for (int i = 0; i < h.n; ++i) v[i] = make_float4(0.f, 0.f, 0.f, 1.f);
      sr = r;
      sv = v;
    }
    CK(cudaMemcpyAsync(e->r[0] + p0, sr, nb, cudaMemcpyHostToDevice, e->stream));
    CK(cudaMemcpyAsync(e->v[0] + p0, sv, nb, cudaMemcpyHostToDevice, e->stream));
    if (im3) {
      int4* si = reinterpret_cast<int4*>(stage_alloc(e, nb));
      for (int i = 0; i < h.n; ++i) si[i] = make_int4(im3[3 * i], im3[3 * i + 1], im3[3 * i + 2], 0);
      CK(cudaMemcpyAsync(e->im[0] + p0, si, nb, cudaMemcpyHostToDevice, e->stream));
    } else {
      CK(cudaMemsetAsync(e->im[0] + p0, 0, nb, e->stream));
    }
    CK(cudaMemcpyAsync(e->last_r + p0, e->r[0] + p0, nb, cudaMemcpyDeviceToDevice, e->stream));
    k_iota<<<(h.n + 255) / 256, 256, 0, e->stream>>>(e->uidx[0] + p0, h.n);
    check_launch();
    CK(cudaMemsetAsync(e->f + p0, 0, h.np * sizeof(float4), e->stream));
    CK(cudaMemsetAsync(e->w + p0, 0, h.np * sizeof(float4), e->stream));
    CK(cudaMemsetAsync(e->sts + p0, 0, h.np * sizeof(float4), e->stream));
    CK(cudaMemsetAsync(e->nn + p0, 0, h.np * sizeof(unsigned), e->stream));
    RepState* s = reinterpret_cast<RepState*>(stage_alloc(e, sizeof(RepState)));
    std::memset(s, 0, sizeof(RepState));
    s->xi = d->xi;
    s->T = d->target_T;
    s->dT = d->dT_per_step;
    s->rebuild = 1;
    CK(cudaMemcpyAsync(e->st + id, s, sizeof(RepState), cudaMemcpyHostToDevice, e->stream));
    stage_commit(e);
    h.admit_seq = e->chunk_seq;
    e->reps[id] = h;
    // tiles, the replica table and the momentum follow before the next launch
    e->layout_dirty = true;
    e->momentum_due.push_back(id);
    if (direct) CK(cudaStreamSynchronize(e->stream));
    *id_out = id;
  });
}

int b2md_replica_remove(b2md_engine* e, int id) {
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    // The ranges go back to the pools at once: whatever is queued on the
    // stream (a running chunk) still finishes with them before any later
    // admission's copies, which are queued behind it, overwrite them.
    e->palloc.release(h.p0, h.np);
    e->ealloc.release(h.nbl0, h.nbl_len);
    e->calloc.release(h.cell0, h.ncell);
    e->qalloc.release(h.par0, h.npar);
    if (h.par1 >= 0) e->qalloc.release(h.par1, h.npar1);
    if (h.elog0 >= 0) e->zalloc.release(h.elog0, h.ecap);
    h = HostRep();
    e->layout_dirty = true;  // the tile layout without it is uploaded before the next launch
  });
}

int b2md_replica_footprint(b2md_engine* e, const b2md_replica_desc* d, long long* bytes) {
  if (!e || !d || !bytes) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    HostRep h = describe(d);
    const int ncell = h.d.nc[0] * h.d.nc[1] * h.d.nc[2];
    h.ncell = ncell;
    h.d.max_nbrs = list_capacity(h, d);
    h.ecap = (d->energy_interval > 0 && d->energy_capacity > 0) ? d->energy_capacity : 0;
    *bytes = replica_bytes(e, h);
  });
}

int b2md_engine_counters(b2md_engine* e, long long* out, int n) {
  if (!e || (n > 0 && !out)) return fail(B2MD_ERR_ARG, "null argument");
  const long long v[B2MD_COUNTERS] = {e->graph_builds, e->invalidations[INV_LAYOUT], e->invalidations[INV_POOL],
                                      e->invalidations[INV_REPAIR], e->invalidations[INV_OTHER], e->list_repairs,
                                      e->layout_uploads, e->chunk_seq};
  for (int k = 0; k < n && k < B2MD_COUNTERS; ++k) out[k] = v[k];
  return B2MD_OK;
}

int b2md_engine_usage(b2md_engine* e, long long* used, long long* reserved) {
  if (!e || !used || !reserved) return fail(B2MD_ERR_ARG, "null argument");
  long long u = 0;
  for (const auto& h : e->reps)
    if (h.active) u += h.bytes;
  *used = u;
  *reserved = e->bytes;
  return B2MD_OK;
}

int b2md_replica_get(b2md_engine* e, int id, int field, void* out) {
  if (!out) return fail(B2MD_ERR_ARG, "out is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    std::vector<unsigned> ids(h.n);
    CK(cudaMemcpyAsync(ids.data(), e->uidx[s.abuf] + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    if (field == B2MD_FIELD_IMAGES) {
      std::vector<int4> tmp(h.n);
      CK(cudaMemcpyAsync(tmp.data(), e->im[s.abuf] + h.p0, h.n * sizeof(int4), cudaMemcpyDeviceToHost, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      int* o = static_cast<int*>(out);
      for (int k = 0; k < h.n; ++k) {
        unsigned i = ids[k];
        o[3 * i] = tmp[k].x; o[3 * i + 1] = tmp[k].y; o[3 * i + 2] = tmp[k].z;
      }
      return;
    }
    const float4* src = nullptr;
    switch (field) {
      case B2MD_FIELD_POS: src = e->r[s.rbuf]; break;
      case B2MD_FIELD_VEL: src = e->v[s.abuf]; break;
      case B2MD_FIELD_FORCE: src = e->f; break;
      case B2MD_FIELD_VIRIAL: src = e->w; break;
      case B2MD_FIELD_STRESS: src = e->sts; break;
      default: api_fail(B2MD_ERR_ARG, "unknown field");
    }
    std::vector<float4> tmp(h.n);
    CK(cudaMemcpyAsync(tmp.data(), src + h.p0, h.n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    float4* o = static_cast<float4*>(out);
    for (int k = 0; k < h.n; ++k) o[ids[k]] = tmp[k];
  });
}

int b2md_replica_read(b2md_engine* e, int id, float* pos4, float* vel4, int* im3) {
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    const size_t n = (size_t)h.n;
    char* stage = static_cast<char*>(host_stage(e, n * kStagePerParticle));
    unsigned* ids = reinterpret_cast<unsigned*>(stage);
    float4* sr = reinterpret_cast<float4*>(stage + ((n * sizeof(unsigned) + 15) & ~(size_t)15));
    float4* sv = sr + n;
    int4* si = reinterpret_cast<int4*>(sv + n);
    CK(cudaMemcpyAsync(ids, e->uidx[s.abuf] + h.p0, n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    if (pos4) CK(cudaMemcpyAsync(sr, e->r[s.rbuf] + h.p0, n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    if (vel4) CK(cudaMemcpyAsync(sv, e->v[s.abuf] + h.p0, n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    if (im3) CK(cudaMemcpyAsync(si, e->im[s.abuf] + h.p0, n * sizeof(int4), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    float4* po = reinterpret_cast<float4*>(pos4);
    float4* vo = reinterpret_cast<float4*>(vel4);
    for (size_t k = 0; k < n; ++k) {
      const unsigned i = ids[k];
      if (pos4) po[i] = sr[k];
      if (vel4) vo[i] = sv[k];
      if (im3) {
        im3[3 * (size_t)i] = si[k].x;
        im3[3 * (size_t)i + 1] = si[k].y;
        im3[3 * (size_t)i + 2] = si[k].z;
      }
    }
  });
}

int b2md_replica_set(b2md_engine* e, int id, int field, const void* in) {
  if (!in) return fail(B2MD_ERR_ARG, "in is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    std::vector<unsigned> ids(h.n);
    CK(cudaMemcpyAsync(ids.data(), e->uidx[s.abuf] + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    if (field == B2MD_FIELD_IMAGES) {
      const int* src = static_cast<const int*>(in);
      std::vector<int4> tmp(h.n);
      for (int k = 0; k < h.n; ++k) {
        unsigned i = ids[k];
        tmp[k] = make_int4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0);
      }
      CK(cudaMemcpyAsync(e->im[s.abuf] + h.p0, tmp.data(), h.n * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      return;
    }
    const float4* src = static_cast<const float4*>(in);
    std::vector<float4> tmp(h.n);
    for (int k = 0; k < h.n; ++k) tmp[k] = src[ids[k]];
    if (field == B2MD_FIELD_POS) {
      for (int k = 0; k < h.n; ++k) {
        int t;
        std::memcpy(&t, &tmp[k].w, 4);
        if (t < 0 || t >= h.d.ntypes) api_fail(B2MD_ERR_ARG, "particle type out of range");
      }
      CK(cudaMemcpyAsync(e->r[s.rbuf] + h.p0, tmp.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      WRITE_STATE(e, id, rebuild, 1);
    } else if (field == B2MD_FIELD_VEL) {
      for (int k = 0; k < h.n; ++k)
        if (!(tmp[k].w > 0.f)) api_fail(B2MD_ERR_ARG, "inverse mass must be positive");
      CK(cudaMemcpyAsync(e->v[s.abuf] + h.p0, tmp.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice, e->stream));
      launch_momentum(e);
      CK(cudaStreamSynchronize(e->stream));
    } else {
      api_fail(B2MD_ERR_ARG, "field cannot be set");
    }
  });
}

int b2md_replica_set_potential(b2md_engine* e, int id, int ntypes, const float* params, int cutoff_method,
                               float skin, int potential) {
  if (!params) return fail(B2MD_ERR_ARG, "params is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    if (ntypes != h.d.ntypes) api_fail(B2MD_ERR_ARG, "number of types cannot change");
    set_potential(h, ntypes, params, cutoff_method, skin, potential);
    place_cells(e, h);
    place_params(e, h);
    int want = estimate_max_nbrs(h);
    if (want > h.d.max_nbrs) place_list(e, h, want);
    h.bytes = replica_bytes(e, h);
    upload_rep(e, id);
    WRITE_STATE(e, id, rebuild, 1);
    invalidate_graphs(e);
  });
}

int b2md_replica_add_potential(b2md_engine* e, int id, int ntypes, const float* params, int cutoff_method,
                               int potential) {
  if (!params) return fail(B2MD_ERR_ARG, "params is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    if (ntypes != h.d.ntypes) api_fail(B2MD_ERR_ARG, "the added potential must have the replica's number of types");
    if (h.potential1 >= 0) api_fail(B2MD_ERR_ARG, "a replica holds at most two potentials");
    check_potential(ntypes, params, cutoff_method, potential);
    h.params1.assign(params, params + ntypes * ntypes * kNumParam);
    h.potential1 = potential;
    h.cutoff1 = cutoff_method;
    derive_grid(h);  // the list reaches the larger cut-off
    place_cells(e, h);
    place_params(e, h);
    int want = estimate_max_nbrs(h);
    if (want > h.d.max_nbrs) place_list(e, h, want);
    h.bytes = replica_bytes(e, h);
    upload_rep(e, id);
    WRITE_STATE(e, id, rebuild, 1);
    invalidate_graphs(e);
  });
}

int b2md_replica_set_integrator(b2md_engine* e, int id, float dt, double target_T, double tau, double dT_per_step,
                                unsigned thermostat_mask) {
  if (!(dt > 0.f)) return fail(B2MD_ERR_ARG, "dt must be positive");
  if (!(tau > 0.0)) return fail(B2MD_ERR_ARG, "tau must be positive");
  if (target_T < 0.0) return fail(B2MD_ERR_ARG, "targetTemperature is negative");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    h.d.dt = dt;
    h.d.omega2 = (float)(4. * M_PI * M_PI / (tau * tau));
    h.d.thermo_mask = thermostat_mask;
    upload_rep(e, id);
    WRITE_STATE(e, id, T, target_T);
    WRITE_STATE(e, id, dT, dT_per_step);
  });
}

int b2md_replica_set_xi(b2md_engine* e, int id, double xi) {
  return guarded([&] {
    get_rep(e, id);
    CK(cudaSetDevice(e->device));
    WRITE_STATE(e, id, xi, xi);
  });
}

int b2md_replica_set_reset_interval(b2md_engine* e, int id, int reset_interval) {
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    h.d.reset_interval = std::max(reset_interval, 0);
    upload_rep(e, id);
  });
}

int b2md_replica_set_nb_method(b2md_engine* e, int id, int method) {
  if (method < -1 || method > 1) return fail(B2MD_ERR_ARG, "method must be -1 (default), 0 (sort) or 1 (n2)");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    h.nb_method_req = method;
    derive_grid(h);
    upload_rep(e, id);
    WRITE_STATE(e, id, rebuild, 1);
    invalidate_graphs(e);
  });
}

int b2md_replica_stats(b2md_engine* e, int id, double* out) {
  if (!out) return fail(B2MD_ERR_ARG, "out is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    ensure_layout(e);
    RepState s = read_state(e, id);
    out[B2MD_STAT_PE] = s.pe;
    out[B2MD_STAT_VIRIAL] = s.vir;
    out[B2MD_STAT_KE] = s.ke_t;
    out[B2MD_STAT_XI] = s.xi;
    out[B2MD_STAT_KE2] = s.ke2;
    out[B2MD_STAT_STEPS] = (double)s.steps;
    out[B2MD_STAT_REBUILDS] = s.nrebuilds;
    out[B2MD_STAT_STEPS_LEFT] = (double)s.steps_left;
    out[B2MD_STAT_OVERFLOW] = s.overflow;
    out[B2MD_STAT_TARGET_T] = s.T;
    out[B2MD_STAT_MAX_NBRS] = h.d.max_nbrs;
    out[B2MD_STAT_ACTUAL_MAX_NBRS] = s.actual_max_nbrs;
    std::vector<unsigned> nn(h.n);
    CK(cudaMemcpyAsync(nn.data(), e->nn + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    double tot = 0;
    for (unsigned c : nn) tot += c;
    out[B2MD_STAT_MEAN_NBRS] = tot / h.n;
    // tiles whose neighbours k_force reads from a position window
    int wt = 0;
    if (e->force_mode == FM_WINDOW && h.d.ntiles > 0) {
      std::vector<int2> wm(h.d.ntiles);
      CK(cudaMemcpyAsync(wm.data(), e->wmeta + h.d.tile0, h.d.ntiles * sizeof(int2), cudaMemcpyDeviceToHost,
                         e->stream));
      CK(cudaStreamSynchronize(e->stream));
      for (const int2& m : wm) wt += m.x >= 0;
    }
    out[B2MD_STAT_WINDOW_TILES] = wt;
    out[B2MD_STAT_TILES] = h.d.ntiles;
  });
}

int b2md_replica_set_energy_log(b2md_engine* e, int id, int interval, int capacity) {
  if (interval < 0 || capacity < 0) return fail(B2MD_ERR_ARG, "interval and capacity must be >= 0");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
    if (h.elog0 >= 0) e->zalloc.release(h.elog0, h.ecap);
    h.elog0 = -1;
    h.ecap = 0;
    h.d.energy_interval = 0;
    h.d.energy_cap = 0;
    h.d.elog0 = 0;
    if (interval > 0 && capacity > 0) {
      long long z = e->zalloc.alloc(capacity, 1);
      if (z < 0) {
        grow_elog(e, e->zalloc.used_end() + capacity);
        z = e->zalloc.alloc(capacity, 1);
      }
      h.elog0 = z;
      h.ecap = capacity;
      h.d.elog0 = z;
      h.d.energy_cap = capacity;
      h.d.energy_interval = interval;
    }
    upload_rep(e, id);
    WRITE_STATE(e, id, nlog, 0);
    invalidate_graphs(e);
  });
}

int b2md_replica_energy_log(b2md_engine* e, int id, double* out, int cap, int* count) {
  if (!out || !count) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    int have = std::min(s.nlog, h.ecap);
    int first = s.nlog - have;
    std::vector<double> buf((size_t)h.ecap * 5);
    if (h.ecap > 0) {
      CK(cudaMemcpyAsync(buf.data(), e->elog + h.elog0 * 5, buf.size() * sizeof(double), cudaMemcpyDeviceToHost,
                         e->stream));
      CK(cudaStreamSynchronize(e->stream));
    }
    int nout = std::min(have, cap);
    for (int k = 0; k < nout; ++k) {
      int slot = (first + k) % std::max(h.ecap, 1);
      for (int c = 0; c < 5; ++c) out[5 * k + c] = buf[(size_t)slot * 5 + c];
    }
    *count = nout;
  });
}

int b2md_replica_stress(b2md_engine* e, int id, int include_kinetic, double* out6) {
  if (!out6) return fail(B2MD_ERR_ARG, "out is null");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    std::vector<float4> sts(h.n), w(h.n), v(h.n);
    RepState s = read_state(e, id);
    CK(cudaMemcpyAsync(sts.data(), e->sts + h.p0, h.n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(w.data(), e->w + h.p0, h.n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(v.data(), e->v[s.abuf] + h.p0, h.n * sizeof(float4), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    // Sample::GetStress (Sample.cu:393-444)
    double st[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < h.n; ++i) {
      st[0] += sts[i].x; st[1] += sts[i].y; st[2] += sts[i].z; st[3] += sts[i].w;
      st[4] += w[i].y; st[5] += w[i].z;
      if (include_kinetic) {
        float mass2 = 2.f / v[i].w;
        st[0] -= mass2 * v[i].x * v[i].x; st[1] -= mass2 * v[i].y * v[i].y; st[2] -= mass2 * v[i].z * v[i].z;
        st[3] -= mass2 * v[i].y * v[i].z; st[4] -= mass2 * v[i].x * v[i].z; st[5] -= mass2 * v[i].x * v[i].y;
      }
    }
    double V = (double)h.d.L[0] * h.d.L[1] * h.d.L[2];
    for (int k = 0; k < 6; ++k) out6[k] = 0.5 * st[k] / V;
  });
}

int b2md_calc_f(b2md_engine* e, int stress) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    calc_f(e, stress != 0);
    CK(cudaStreamSynchronize(e->stream));
  });
}

int b2md_integrate(b2md_engine* e) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ensure_layout(e);
    if (e->ntiles == 0) return;
    EngArgs a = make_args(e);
    k_integrate<<<e->ntiles, e->pb * e->tp, 0, e->stream>>>(a, e->tp);
    check_launch();
  });
}

int b2md_zero_momentum(b2md_engine* e) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ensure_layout(e);
    if (e->ntiles == 0) return;
    EngArgs a = make_args(e);
    k_momentum<<<e->ntiles, e->pb * e->tp, 0, e->stream>>>(a, e->tp, 0);
    k_apply_zero_momentum<<<e->ntiles, e->pb, 0, e->stream>>>(a);
    k_momentum<<<e->ntiles, e->pb * e->tp, 0, e->stream>>>(a, e->tp, 0);
    check_launch();
  });
}

int b2md_run(b2md_engine* e, long long nsteps) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  if (nsteps < 0) return fail(B2MD_ERR_ARG, "nsteps must be >= 0");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ensure_layout(e);
    if (e->ntiles == 0) return;
    EngArgs a = make_args(e);
    int R = (int)e->reps.size();
    k_set_steps<<<(R + 127) / 128, 128, 0, e->stream>>>(a, nsteps, 1);
    launch_momentum(e);
    check_launch();
    // every queue holds exactly nsteps; run until all are empty (a replica
    // frozen by a list overflow catches up after its repair)
    if (nsteps > 0) run_steps(e, 1LL << 62);
    calc_f(e, false);
    CK(cudaStreamSynchronize(e->stream));
  });
}

int b2md_run_timed(b2md_engine* e, long long nsteps, double* step_kernel_ms, long long* launches) {
  if (!e || !step_kernel_ms || !launches) return fail(B2MD_ERR_ARG, "null argument");
  if (nsteps < 0) return fail(B2MD_ERR_ARG, "nsteps must be >= 0");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    *step_kernel_ms = 0.0;
    *launches = 0;
    ensure_layout(e);
    if (e->ntiles == 0) return;
    EngArgs a = make_args(e);
    a.rb_steps_only = 1;
    int R = (int)e->reps.size();
    k_set_steps<<<(R + 127) / 128, 128, 0, e->stream>>>(a, nsteps, 1);
    launch_momentum(e);
    long long nl = 2;
    const int kind = persist_kind_for(e);
    if (kind == 2 || kind == 3) {
      // the batched graph's loop from the host: k_batch (or k_flow) launches
      // (each runs whole steps, rebuilds included) until the budget is spent
      const bool flow = kind == 3;
      if (flow) {
        ensure_flow_queue(e);
        a = make_args(e);
      }
      const BatchFn fb = flow ? flow_fn(e->tp) : batch_fn(e->tp);
      size_t bsmem = flow ? flow_smem(e, a) : batch_smem(e, a);
      force_fn(e, true, false, a);
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fb, e->pb * e->tp, bsmem));
      if (per_sm < 1) api_fail(B2MD_ERR_NOMEM, "the batched step kernel does not fit on an SM: use a smaller pb*tp");
      cudaEvent_t e0, e1;
      CK(cudaEventCreate(&e0));
      CK(cudaEventCreate(&e1));
      int* h_left = nullptr;
      CK(cudaMallocHost(&h_left, sizeof(int)));
      int budget = (int)std::min<long long>(nsteps, 1 << 30);
      double tot = 0.0;
      cudaGraphConditionalHandle none = 0;
      for (int guard = 0; budget > 0 && guard < 1 << 20; ++guard) {
        *e->h_budget = budget;
        CK(cudaMemcpyAsync(&e->pctl->budget, e->h_budget, sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CK(cudaMemsetAsync(&e->pctl->arrive, 0, sizeof(unsigned long long), e->stream));
        CK(cudaEventRecord(e0, e->stream));
        void* args[] = {&a, &none};
        CK(cudaLaunchCooperativeKernel((const void*)fb, dim3(per_sm * e->nsm), dim3(e->pb * e->tp), args, bsmem,
                                       e->stream));
        CK(cudaEventRecord(e1, e->stream));
        CK(cudaMemcpyAsync(h_left, &e->pctl->budget, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
        CK(cudaStreamSynchronize(e->stream));
        check_persist(e);
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        tot += ms;
        nl += 1;
        budget = *h_left;
        if (repair_overflow(e)) {
          a = make_args(e);  // the repaired list moved
          bsmem = flow ? flow_smem(e, a) : batch_smem(e, a);
          continue;
        }
        if (max_steps_left(e) == 0) break;
      }
      cudaFreeHost(h_left);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      calc_f(e, false);
      CK(cudaStreamSynchronize(e->stream));
      *step_kernel_ms = tot;
      *launches = nl + rebuild_launches(e) + 1;
      return;
    }
    if (kind == 1) {
      // the persistent graph's launch sequence with the host taking the loop
      // decision: rebuild kernels (they exit at once when no rebuild is due),
      // then one cooperative k_steps launch that runs steps until a rebuild is
      // due or the budget is spent; each launch is timed with its steps
      const StepsFn fs = steps_fn(e->tp);
      const size_t psmem = persist_smem(e, a);
      force_fn(e, true, false, a);  // checks the shared-memory need
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fs, e->pb * e->tp, psmem));
      if ((long long)per_sm * e->nsm >= e->ntiles) {
        const int grid = steps_grid(e, fs, psmem);
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        int* h_left = nullptr;
        CK(cudaMallocHost(&h_left, sizeof(int)));
        int budget = (int)std::min<long long>(nsteps, 1 << 30);
        *e->h_budget = budget;
        CK(cudaMemcpyAsync(&e->pctl->budget, e->h_budget, sizeof(int), cudaMemcpyHostToDevice, e->stream));
        double tot = 0.0;
        cudaGraphConditionalHandle none = 0;
        while (budget > 0) {
          launch_rebuild(e, e->stream, a);
          nl += rebuild_launches(e);
          CK(cudaMemsetAsync(&e->pctl->arrive, 0, sizeof(unsigned long long), e->stream));
          CK(cudaEventRecord(e0, e->stream));
          void* args[] = {&a, &none};
          CK(cudaLaunchCooperativeKernel((const void*)fs, dim3(grid), dim3(e->pb * e->tp), args, psmem, e->stream));
          CK(cudaEventRecord(e1, e->stream));
          CK(cudaMemcpyAsync(h_left, &e->pctl->budget, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
          CK(cudaStreamSynchronize(e->stream));
          check_persist(e);
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          tot += ms;
          nl += 1;
          const int ran = budget - *h_left;
          budget = *h_left;
          if (ran <= 0 || max_steps_left(e) == 0) break;  // no replica has steps left
        }
        cudaFreeHost(h_left);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (repair_overflow(e)) run_steps(e, nsteps);
        calc_f(e, false);
        CK(cudaStreamSynchronize(e->stream));
        *step_kernel_ms = tot;
        *launches = nl + rebuild_launches(e) + 1;
        return;
      }
    }
    const size_t smem = force_smem(e, a);
    ForceFn fstep = force_fn(e, true, false, a);
    std::vector<cudaEvent_t> ev(2 * nsteps);
    for (auto& x : ev) CK(cudaEventCreate(&x));
    int* h_any = nullptr;
    CK(cudaMallocHost(&h_any, sizeof(int)));
    // the launch sequence of the step graph, with the host taking the
    // conditional node's decision: rebuild kernels only when a replica is due
    for (long long k = 0; k < nsteps; ++k) {
      k_gate_flag<<<1, 128, 0, e->stream>>>(a, e->any_rebuild + 1);
      CK(cudaMemcpyAsync(h_any, e->any_rebuild + 1, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      if (*h_any) {
        launch_rebuild(e, e->stream, a);
        nl += rebuild_launches(e);
      }
      CK(cudaEventRecord(ev[2 * k], e->stream));
      fstep<<<force_grid(e, a, fstep, smem), e->pb * e->tp, smem, e->stream>>>(a, 0, cudaGraphConditionalHandle{});
      CK(cudaEventRecord(ev[2 * k + 1], e->stream));
      nl += 2;
    }
    check_launch();
    CK(cudaStreamSynchronize(e->stream));
    cudaFreeHost(h_any);
    double tot = 0.0;
    for (long long k = 0; k < nsteps; ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]));
      tot += ms;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    if (repair_overflow(e)) run_steps(e, nsteps);
    calc_f(e, false);
    CK(cudaStreamSynchronize(e->stream));
    *step_kernel_ms = tot;
    *launches = nl + rebuild_launches(e) + 1;
  });
}

int b2md_replica_queue_steps(b2md_engine* e, int id, long long nsteps) {
  if (nsteps < 0) return fail(B2MD_ERR_ARG, "nsteps must be >= 0");
  return guarded([&] {
    get_rep(e, id);
    CK(cudaSetDevice(e->device));
    // in stream order: after the work already queued, before the next launch
    k_queue_steps<<<1, 1, 0, e->stream>>>(e->st + id, nsteps);
    check_launch();
  });
}

int b2md_run_queued(b2md_engine* e, long long max_steps, long long* steps_run) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ensure_layout(e);
    long long lim = max_steps > 0 ? max_steps : (1LL << 62);
    long long n = e->ntiles ? run_steps(e, lim) : 0;
    if (steps_run) *steps_run = n;
  });
}

int b2md_run_queued_async(b2md_engine* e, long long max_steps, long long* ticket) {
  if (!e || !ticket) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ChunkRec& c = e->chunk[(e->chunk_seq + 1) & 1];
    if (c.ticket && !c.waited) finish_chunk(e, c);  // a third chunk waits for the oldest
    if (!c.done) {
      CK(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
      CK(cudaMallocHost(&c.h_in, sizeof(int)));
      CK(cudaMallocHost(&c.h_ctl, sizeof(PersistCtl)));
    }
    ensure_layout(e);
    const int R = (int)e->reps.size();
    if (R > c.st_cap) {
      if (c.h_st) CK(cudaFreeHost(c.h_st));  // its last copy completed (the chunk was waited)
      c.h_st = nullptr;
      c.st_cap = 0;
      CK(cudaMallocHost(&c.h_st, (size_t)std::max(R, e->rcap) * sizeof(RepState)));
      c.st_cap = std::max(R, e->rcap);
    }
    c.active.assign(R, 0);
    for (int r = 0; r < R; ++r) c.active[r] = e->reps[r].active ? 1 : 0;
    c.persistent = false;
    c.budget = 0;
    c.ran = 0;
    if (e->ntiles > 0) {
      ensure_graphs(e);
      const long long lim = max_steps > 0 ? std::min<long long>(max_steps, 1 << 30) : (1 << 30);
      if (e->persist_on) {
        // the persistent graph runs until the budget is spent, no replica
        // has steps left or a list overflows; it leaves the unspent budget
        c.persistent = true;
        c.budget = lim;
        *c.h_in = (int)lim;
        CK(cudaMemcpyAsync(&e->pctl->budget, c.h_in, sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CK(cudaGraphLaunch(e->gexec[2], e->stream));
      } else {
        // per-step graphs: the queue lengths decide how many (read first)
        const long long todo = std::min(max_steps_left(e), lim);
        for (long long k = 0; k < todo / kChunk; ++k) CK(cudaGraphLaunch(e->gexec[1], e->stream));
        for (long long k = 0; k < todo % kChunk; ++k) CK(cudaGraphLaunch(e->gexec[0], e->stream));
        c.budget = todo;
      }
    }
    CK(cudaMemcpyAsync(c.h_ctl, e->pctl, sizeof(PersistCtl), cudaMemcpyDeviceToHost, e->stream));
    if (R > 0) CK(cudaMemcpyAsync(c.h_st, e->st, (size_t)R * sizeof(RepState), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaEventRecord(c.done, e->stream));
    c.ticket = ++e->chunk_seq;
    c.waited = false;
    *ticket = c.ticket;
  });
}

int b2md_run_queued_poll(b2md_engine* e, long long ticket, int* done) {
  if (!e || !done) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    ChunkRec* c = find_chunk(e, ticket);
    if (c->waited) {
      *done = 1;
      return;
    }
    CK(cudaSetDevice(e->device));
    const cudaError_t q = cudaEventQuery(c->done);
    if (q != cudaSuccess && q != cudaErrorNotReady) throw CudaErr{q, "cudaEventQuery(chunk)", __LINE__};
    *done = q == cudaSuccess;
  });
}

int b2md_run_queued_wait(b2md_engine* e, long long ticket, long long* steps_run, double* states, int cap) {
  if (!e) return fail(B2MD_ERR_ARG, "null argument");
  if (cap < 0 || (cap > 0 && !states)) return fail(B2MD_ERR_ARG, "states must hold cap rows");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    ChunkRec* c = find_chunk(e, ticket);
    if (!c->waited) finish_chunk(e, *c);
    if (steps_run) *steps_run = c->ran;
    const int R = (int)c->active.size();
    for (int r = 0; r < cap; ++r) {
      double* o = states + (size_t)r * B2MD_CHUNK_FIELDS;
      for (int k = 0; k < B2MD_CHUNK_FIELDS; ++k) o[k] = 0.0;
      if (r >= R || !c->active[r]) {
        o[B2MD_CHUNK_STEPS_LEFT] = -1.0;
        continue;
      }
      const RepState& s = c->h_st[r];
      o[B2MD_CHUNK_ACTIVE] = 1.0;
      o[B2MD_CHUNK_STEPS] = (double)s.steps;
      o[B2MD_CHUNK_STEPS_LEFT] = (double)s.steps_left;
      o[B2MD_CHUNK_PE] = s.pe;
      o[B2MD_CHUNK_VIRIAL] = s.vir;
      o[B2MD_CHUNK_KE] = s.ke_t;
      o[B2MD_CHUNK_XI] = s.xi;
      o[B2MD_CHUNK_REBUILDS] = s.nrebuilds;
      o[B2MD_CHUNK_OVERFLOW] = s.overflow;
    }
  });
}

int b2md_nbl_export(b2md_engine* e, int id, unsigned* counts, unsigned* nbl, int max_nbrs) {
  if (!counts || !nbl) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    std::vector<unsigned> ids(h.n), nn(h.n), lst((size_t)list_rows(h.d.max_nbrs) * h.np);
    CK(cudaMemcpyAsync(ids.data(), e->uidx[s.abuf] + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(nn.data(), e->nn + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(lst.data(), e->nbl + h.nbl0, lst.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    for (int sl = 0; sl < h.n; ++sl) {
      unsigned i = ids[sl];
      unsigned c = std::min<unsigned>(nn[sl], (unsigned)max_nbrs);
      counts[i] = nn[sl];
      for (unsigned k = 0; k < c; ++k) nbl[(size_t)i * max_nbrs + k] = ids[lst[lpos(k, (unsigned)sl, h.np)]];
    }
  });
}

int b2md_sort_export(b2md_engine* e, int id, unsigned* unsorted_index) {
  if (!unsorted_index) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    CK(cudaSetDevice(e->device));
    RepState s = read_state(e, id);
    CK(cudaMemcpyAsync(unsorted_index, e->uidx[s.abuf] + h.p0, h.n * sizeof(unsigned), cudaMemcpyDeviceToHost,
                       e->stream));
    CK(cudaStreamSynchronize(e->stream));
  });
}

int b2md_cell_grid(b2md_engine* e, int id, int* nc3) {
  if (!nc3) return fail(B2MD_ERR_ARG, "null argument");
  return guarded([&] {
    HostRep& h = get_rep(e, id);
    for (int k = 0; k < 3; ++k) nc3[k] = h.d.nc[k];
    if (h.d.nb_method != NB_CELLS) nc3[0] = nc3[1] = nc3[2] = 0;
  });
}

int b2md_sync(b2md_engine* e) {
  if (!e) return fail(B2MD_ERR_ARG, "null engine");
  return guarded([&] {
    CK(cudaSetDevice(e->device));
    CK(cudaStreamSynchronize(e->stream));
  });
}

void* b2md_stream(b2md_engine* e) { return e ? (void*)e->stream : nullptr; }

}  // extern "C"
