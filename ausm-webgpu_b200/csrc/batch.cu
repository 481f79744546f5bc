// ausm_batch_*: many independent solves advanced by one kernel launch per RK stage and
// scheme group (kernels_batch.cu), the n-step sequence captured as a CUDA graph in which
// the scheme groups are independent branches (their stage chains overlap on the GPU).
//
// Device data: one BatchSolve descriptor per member (its buffers, constants, scheme,
// first work item and current-buffer index), the members' tensor maps (kBatchMaps
// each) and the item table (one BatchItem per tile: solve, rotation at upload, tile
// coordinates, M).  The host keeps a mirror of the descriptors and re-uploads them,
// the item table with the members' current rotations and a zeroed step counter, when a
// member's constants, scheme or state buffer index changed since the last upload (a
// parameter change, a new state, a ramp step); the graph reads these at replay time,
// so it stays valid until the membership changes.  The buffer rotation (cur) advances
// on the device at the end of each step sequence (descriptors and step counter) and in
// the mirror on the host, identically.
//
// Ordering: a member's own calls run on the batch stream while it is a member, so batch
// steps and member calls (state read-back, forces, set_params) are ordered by the
// stream alone.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ausm.h"
#include "ausm_internal.h"
#include "solver_internal.h"

using ausm::BatchSolve;

struct ausm_batch {
  int dev = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<ausm_solver*> members;
  // Work-list order: descriptor k describes members[order[k]].  Members are grouped by
  // scheme (so CTAs resident at the same time mostly run one scheme's code), larger
  // grids first within a scheme.
  std::vector<int> order;
  std::vector<BatchSolve> mirror;  // what the device descriptors hold, in work-list order
  struct Group {
    int scheme, s_lo, s_hi, t_lo, t_hi;  // group key (group_key), descriptors [s_lo, s_hi), items [t_lo, t_hi)
  };
  std::vector<Group> groups;
  cudaStream_t aux[2] = {nullptr, nullptr};  // branches of the second and third group
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
  bool uploaded = false;
  int total_tiles = 0;
  int total_chunks = 0;  // residual-norm chunks of all members
  BatchSolve* d_solves = nullptr;
  std::vector<ausm::BatchItem> items;  // the work items (the device's d_items)
  ausm::BatchItem* d_items = nullptr;
  int item_cap = 0;
  int* d_steps = nullptr;  // steps taken since the item table was uploaded (d_err + 1)
  CUtensorMap* d_maps = nullptr;  // kBatchMaps per descriptor when tma
  bool tma = false;               // every member has tensor maps: stages load tiles by TMA
  int rows = 16;                  // tile height of the work list
  int tuned_rows = 0;             // height chosen by the last tuning run (0: none yet)
  double tuned_cells = 0.0;       // the batch's cell count at that run
  int* d_err = nullptr;           // set by a TMA tile whose bounded wait gave up
  int* h_err = nullptr;           // pinned copy of *d_err
  bool err_read_queued = false;   // a copy of *d_err to *h_err is queued on st
  int cap = 0;  // descriptor capacity of d_solves / d_maps / d_out / d_l2
  float* d_out = nullptr;
  double* d_l2 = nullptr;
  double* d_part = nullptr;
  int part_cap = 0;
  float* h_out = nullptr;
  double* h_l2 = nullptr;
  bool graphs = true;
  std::map<int, cudaGraphExec_t> graph;  // per n, for the current membership
  std::string err;
};

namespace {

constexpr int kTX = 32;  // tile width of the batched stage kernels (height: ausm_batch::rows)
constexpr int kNormChunk = 512;  // cells per residual-norm chunk (kernels_batch.cu)

int bfail(ausm_batch* b, int code, const std::string& msg) {
  ausm::set_thread_error(msg);
  if (b) b->err = msg;
  return code;
}
#define BCU(b, call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? AUSM_ERR_OOM : AUSM_ERR_CUDA,  \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)
#define BNEED(b, cond, code, msg)            \
  do {                                       \
    if (!(cond)) return bfail(b, code, msg); \
  } while (0)

int use_dev(ausm_batch* b) {
  int d = -1;
  BCU(b, cudaGetDevice(&d));
  if (d != b->dev) BCU(b, cudaSetDevice(b->dev));
  return AUSM_OK;
}

void drop_graphs(ausm_batch* b) {
  for (auto& kv : b->graph) cudaGraphExecDestroy(kv.second);
  b->graph.clear();
}

// Work-list group of a member: its scheme, plus 4 when MUSCL is on (the group's
// kernels are then instantiated with MUSCL known on, without a per-face branch).
int group_key(const ausm_solver* h) { return h->p.scheme + (h->p.muscl > 0 ? 4 : 0); }

BatchSolve describe(const ausm_solver* h, int tile0, int chunk0, const CUtensorMap* maps) {
  BatchSolve d{};
  d.chunk0 = chunk0;
  d.maps = maps;
  for (int k = 0; k < 3; k++) d.Q[k] = h->Q[k];
  d.Mi = h->Mi;
  d.Mj = h->Mj;
  d.dt = h->dt;
  d.wave = h->wave;
  d.c = h->c;
  d.M = h->M;
  d.N = h->N;
  d.scheme = group_key(h);
  d.tiles_x = (h->M + kTX - 1) / kTX;
  d.tile0 = tile0;
  d.cur = h->cur;
  return d;
}

const CUtensorMap* maps_of(const ausm_batch* b, int k) {
  return b->tma ? b->d_maps + ausm::kBatchMaps * (size_t)k : nullptr;
}

// Grows the per-member and per-tile device arrays (dropping graphs that point at them).
int ensure_capacity(ausm_batch* b) {
  const int n = (int)b->members.size();
  if (n > b->cap) {
    int cap = std::max(n, 2 * b->cap);
    if (b->cap) drop_graphs(b);
    BCU(b, cudaStreamSynchronize(b->st));
    cudaFree(b->d_solves);
    cudaFree(b->d_maps);
    cudaFree(b->d_out);
    cudaFree(b->d_l2);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_l2);
    b->d_solves = nullptr; b->d_maps = nullptr; b->d_out = nullptr; b->d_l2 = nullptr; b->h_out = nullptr; b->h_l2 = nullptr;
    b->cap = 0;
    BCU(b, cudaMalloc((void**)&b->d_solves, cap * sizeof(BatchSolve)));
    BCU(b, cudaMalloc((void**)&b->d_maps, cap * ausm::kBatchMaps * sizeof(CUtensorMap)));
    BCU(b, cudaMalloc((void**)&b->d_out, cap * 2 * sizeof(float)));
    BCU(b, cudaMalloc((void**)&b->d_l2, cap * sizeof(double)));
    BCU(b, cudaMallocHost((void**)&b->h_out, cap * 2 * sizeof(float)));
    BCU(b, cudaMallocHost((void**)&b->h_l2, cap * sizeof(double)));
    b->cap = cap;
    b->uploaded = false;
  }
  if (b->total_tiles > b->item_cap) {
    int cap = std::max(b->total_tiles, 2 * b->item_cap);
    drop_graphs(b);
    BCU(b, cudaStreamSynchronize(b->st));
    cudaFree(b->d_items);
    b->d_items = nullptr;
    b->item_cap = 0;
    BCU(b, cudaMalloc((void**)&b->d_items, cap * sizeof(ausm::BatchItem)));
    b->item_cap = cap;
    b->uploaded = false;
  }
  if (b->total_chunks > b->part_cap) {
    int cap = std::max(b->total_chunks, 2 * b->part_cap);
    BCU(b, cudaStreamSynchronize(b->st));
    cudaFree(b->d_part);
    b->d_part = nullptr;
    b->part_cap = 0;
    BCU(b, cudaMalloc((void**)&b->d_part, cap * sizeof(double)));
    b->part_cap = cap;
  }
  return AUSM_OK;
}

// Rebuilds the work list after a membership change.
void relayout(ausm_batch* b) {
  drop_graphs(b);
  b->mirror.clear();
  const int n = (int)b->members.size();
  b->order.resize(n);
  for (int k = 0; k < n; k++) b->order[k] = k;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    const ausm_solver *p = b->members[x], *q = b->members[y];
    if (group_key(p) != group_key(q)) return group_key(p) < group_key(q);
    return (size_t)p->M * p->N > (size_t)q->M * q->N;
  });
  int t = 0;
  b->groups.clear();
  b->items.clear();
  b->tma = !b->members.empty();
  for (ausm_solver* h : b->members) b->tma = b->tma && h->tma[0].ok && h->tma[1].ok && h->tma[2].ok;
  if (!b->tma) b->rows = 16;
  const int rows = b->rows;
  int chunks = 0;
  for (int k : b->order) {
    const ausm_solver* h = b->members[k];
    const int s = (int)b->mirror.size();
    if (b->groups.empty() || b->groups.back().scheme != group_key(h)) b->groups.push_back({group_key(h), s, s, t, t});
    b->mirror.push_back(describe(h, t, chunks, maps_of(b, s)));
    const int tx = (h->M + kTX - 1) / kTX, tiles = tx * ((h->N + rows - 1) / rows);
    for (int k = 0; k < tiles; k++) b->items.push_back({s, 0, (k % tx) | (k / tx) << 16, h->M});
    t += tiles;
    chunks += (int)(((size_t)h->M * h->N + kNormChunk - 1) / kNormChunk);
    b->groups.back().s_hi = s + 1;
    b->groups.back().t_hi = t;
  }
  b->total_tiles = t;
  b->total_chunks = chunks;
  b->uploaded = false;
}

// Brings the device descriptors up to date with the members' host state.
int sync_descriptors(ausm_batch* b) {
  for (size_t k = 0; k < b->members.size(); k++)
    if (group_key(b->members[b->order[k]]) != b->mirror[k].scheme) {  // regroup
      relayout(b);
      break;
    }
  bool changed = !b->uploaded;
  for (size_t k = 0; k < b->members.size(); k++) {
    BatchSolve d = describe(b->members[b->order[k]], b->mirror[k].tile0, b->mirror[k].chunk0, maps_of(b, (int)k));
    if (std::memcmp(&d, &b->mirror[k], sizeof d) != 0) {
      b->mirror[k] = d;
      changed = true;
    }
  }
  if (changed && !b->members.empty()) {
    // pageable source: the call returns once the source has been staged
    BCU(b, cudaMemcpyAsync(b->d_solves, b->mirror.data(), b->mirror.size() * sizeof(BatchSolve),
                           cudaMemcpyHostToDevice, b->st));
    if (b->tma) {  // each member's maps, in work-list order
      std::vector<CUtensorMap> maps;
      maps.reserve(ausm::kBatchMaps * b->members.size());
      for (int k : b->order) {
        const ausm::TmaMaps& t = b->members[k]->tma[ausm::tile_index(b->rows)];
        for (int q = 0; q < 3; q++) maps.push_back(t.halo[q]);
        for (int q = 0; q < 3; q++) maps.push_back(t.plain[q]);
        maps.push_back(t.mi);
        maps.push_back(t.mj);
        for (int q = 0; q < 3; q++) maps.push_back(t.wrap[q]);
      }
      BCU(b, cudaMemcpyAsync(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                             b->st));
    }
    // the item table with each solve's current rotation, and the step count restarted
    for (ausm::BatchItem& it : b->items) it.cur = b->mirror[it.solve].cur;
    BCU(b, cudaMemcpyAsync(b->d_items, b->items.data(), b->items.size() * sizeof(ausm::BatchItem),
                           cudaMemcpyHostToDevice, b->st));
    BCU(b, cudaMemsetAsync(b->d_steps, 0, sizeof(int), b->st));
    b->uploaded = true;
  }
  return AUSM_OK;
}

// dt per member; per scheme group (own branch) 3n stages; then the rotation advance and
// the dt / wave gather
void enqueue_steps(ausm_batch* b, int n) {
  const int ns = (int)b->members.size();
  int* err = b->tma ? b->d_err : nullptr;
  ausm::launch_batch_dt(b->d_solves, ns, b->st);
  const int G = (int)b->groups.size();
  for (int g = 1; g < G; g++) {
    cudaEventRecord(b->fork, b->st);
    cudaStreamWaitEvent(b->aux[g - 1], b->fork, 0);
  }
  for (int g = 0; g < G; g++) {
    const ausm_batch::Group& q = b->groups[g];
    cudaStream_t s = g == 0 ? b->st : b->aux[g - 1];
    for (int k = 0; k < n; k++) {
      ausm::launch_batch_stage(q.scheme, 1, false, b->d_solves, b->d_items, b->d_steps, b->d_maps, q.t_lo, q.t_hi, k, b->rows, err, s);
      ausm::launch_batch_stage(q.scheme, 2, false, b->d_solves, b->d_items, b->d_steps, b->d_maps, q.t_lo, q.t_hi, k, b->rows, err, s);
      ausm::launch_batch_stage(q.scheme, 3, k == n - 1, b->d_solves, b->d_items, b->d_steps, b->d_maps, q.t_lo, q.t_hi, k, b->rows, err,
                               s);
    }
  }
  for (int g = 1; g < G; g++) {
    cudaEventRecord(b->join[g - 1], b->aux[g - 1]);
    cudaStreamWaitEvent(b->st, b->join[g - 1], 0);
  }
  ausm::launch_batch_advance(b->d_solves, ns, n, b->d_steps, b->st);
  ausm::launch_batch_gather(b->d_solves, ns, b->d_out, b->st);
}

// Tile-height autotuning of the batch (as tuned_tile_rows for one solve): for each
// candidate height the work list is laid out again and the stage-1 launches of every
// scheme group are timed on the members' own data (stage 1 writes only each member's
// scratch buffer).  Runs on the first step and again when the batch's cell count has
// changed by more than a factor of two; AUSM_TILE_ROWS fixes the height.
int tune_rows(ausm_batch* b) {
  double cells = 0.0;
  for (ausm_solver* h : b->members) cells += (double)h->M * h->N;
  if (!b->tma) return AUSM_OK;
  int fixed = 0;
  if (const char* e = std::getenv("AUSM_TILE_ROWS")) fixed = std::atoi(e);
  if (const char* e = std::getenv("AUSM_AUTOTUNE"))
    if (e[0] == '0') fixed = 16;
  if (fixed == 8 || fixed == 16 || fixed == 32) {
    if (b->rows != fixed) {
      b->rows = fixed;
      relayout(b);
      int rc = ensure_capacity(b);
      if (rc) return rc;
    }
    return AUSM_OK;
  }
  if (b->tuned_rows && cells <= 2.0 * b->tuned_cells && 2.0 * cells >= b->tuned_cells) return AUSM_OK;
  const int reps = (int)std::max(5.0, std::min(100.0, 1.0e8 / std::max(cells, 1.0)));
  float best_ms[3] = {INFINITY, INFINITY, INFINITY};
  const int cand[3] = {8, 16, 32};
  for (int round = 0; round < 2; round++)  // each candidate's best of two rounds counts
    for (int k = 0; k < 3; k++) {
      const int r = cand[k];
      b->rows = r;
      relayout(b);
      int rc = ensure_capacity(b);
      if (!rc) rc = sync_descriptors(b);
      if (rc) return rc;
      auto launch = [&] {
        for (const ausm_batch::Group& q : b->groups)
          ausm::launch_batch_stage(q.scheme, 1, false, b->d_solves, b->d_items, b->d_steps, b->d_maps, q.t_lo, q.t_hi, 0, r, b->d_err,
                                   b->st);
      };
      launch();
      BCU(b, cudaEventRecord(b->e0, b->st));
      for (int k2 = 0; k2 < reps; k2++) launch();
      BCU(b, cudaEventRecord(b->e1, b->st));
      BCU(b, cudaEventSynchronize(b->e1));
      BCU(b, cudaGetLastError());
      float ms = 0.0f;
      BCU(b, cudaEventElapsedTime(&ms, b->e0, b->e1));
      best_ms[k] = std::min(best_ms[k], ms);
    }
  int best_rows = 16;
  float best = INFINITY;
  for (int k = 0; k < 3; k++)
    if (best_ms[k] < best) {
      best = best_ms[k];
      best_rows = cand[k];
    }
  b->rows = best_rows;
  relayout(b);
  int rc = ensure_capacity(b);
  if (rc) return rc;
  b->tuned_rows = best_rows;
  b->tuned_cells = cells;
  return AUSM_OK;
}

// Timeout reporting, as for one solver (api.cu): every step sequence queues a copy of
// the batch's error flag; the next call that waits for the batch stream reads it,
// clears the flag and returns AUSM_ERR_TIMEOUT.
int queue_err_read(ausm_batch* b) {
  BCU(b, cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->st));
  b->err_read_queued = true;
  return AUSM_OK;
}
int sync_and_check(ausm_batch* b) {
  BCU(b, cudaStreamSynchronize(b->st));
  if (!b->err_read_queued) return AUSM_OK;
  b->err_read_queued = false;
  if (*b->h_err == 0) return AUSM_OK;
  *b->h_err = 0;
  BCU(b, cudaMemsetAsync(b->d_err, 0, sizeof(int), b->st));
  return bfail(b, AUSM_ERR_TIMEOUT, "a tile load did not arrive within the bounded wait");
}

int run_steps(ausm_batch* b, int n) {
  if (!b->graphs) {
    enqueue_steps(b, n);
    BCU(b, cudaGetLastError());
    return AUSM_OK;
  }
  auto it = b->graph.find(n);
  if (it == b->graph.end()) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    BCU(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    enqueue_steps(b, n);
    cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(b, AUSM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    it = b->graph.emplace(n, ge).first;
  }
  BCU(b, cudaGraphLaunch(it->second, b->st));
  return AUSM_OK;
}

}  // namespace

namespace ausm {
// Called by ausm_destroy and ausm_batch_remove: detaches h, back on its own stream.
int batch_detach(ausm_batch* b, ausm_solver* h);
}

extern "C" {

int ausm_batch_create(ausm_batch** out) {
  if (!out) return bfail(nullptr, AUSM_ERR_INVALID, "null output handle");
  *out = nullptr;
  ausm_batch* b = new ausm_batch();
  auto bail = [&](cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    ausm_batch_destroy(b);
    return bfail(nullptr, e == cudaErrorMemoryAllocation ? AUSM_ERR_OOM : AUSM_ERR_CUDA, msg);
  };
  cudaError_t e = cudaGetDevice(&b->dev);
  if (e != cudaSuccess) return bail(e, "cudaGetDevice");
  e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(e, "cudaStreamCreateWithFlags");
  if ((e = cudaEventCreate(&b->e0)) != cudaSuccess || (e = cudaEventCreate(&b->e1)) != cudaSuccess)
    return bail(e, "cudaEventCreate");
  for (int g = 0; g < 2; g++) {
    e = cudaStreamCreateWithFlags(&b->aux[g], cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "cudaStreamCreateWithFlags");
    e = cudaEventCreateWithFlags(&b->join[g], cudaEventDisableTiming);
    if (e != cudaSuccess) return bail(e, "cudaEventCreate");
  }
  e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (e != cudaSuccess) return bail(e, "cudaEventCreate");
  if ((e = cudaMalloc((void**)&b->d_err, 2 * sizeof(int))) != cudaSuccess) return bail(e, "cudaMalloc");
  if ((e = cudaMallocHost((void**)&b->h_err, sizeof(int))) != cudaSuccess) return bail(e, "cudaMallocHost");
  *b->h_err = 0;
  if ((e = cudaMemsetAsync(b->d_err, 0, 2 * sizeof(int), b->st)) != cudaSuccess) return bail(e, "cudaMemsetAsync");
  b->d_steps = b->d_err + 1;
  *out = b;
  return AUSM_OK;
}

int ausm_batch_destroy(ausm_batch* b) {
  if (!b) return AUSM_OK;
  cudaSetDevice(b->dev);
  while (!b->members.empty()) ausm::batch_detach(b, b->members.back());
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graphs(b);
  cudaFree(b->d_solves);
  cudaFree(b->d_items);
  cudaFree(b->d_maps);
  cudaFree(b->d_err);
  cudaFree(b->d_out);
  cudaFree(b->d_l2);
  cudaFree(b->d_part);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->h_l2) cudaFreeHost(b->h_l2);
  if (b->h_err) cudaFreeHost(b->h_err);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  if (b->fork) cudaEventDestroy(b->fork);
  for (int g = 0; g < 2; g++) {
    if (b->aux[g]) {
      cudaStreamSynchronize(b->aux[g]);
      cudaStreamDestroy(b->aux[g]);
    }
    if (b->join[g]) cudaEventDestroy(b->join[g]);
  }
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return AUSM_OK;
}

const char* ausm_batch_last_error(const ausm_batch* b) { return b ? b->err.c_str() : ausm_last_error(nullptr); }

int ausm_batch_add(ausm_batch* b, ausm_solver* h) {
  BNEED(b, b && h, AUSM_ERR_INVALID, "null handle");
  BNEED(b, !h->batch, AUSM_ERR_STATE, h->batch == b ? "solver is already a member" : "solver belongs to another batch");
  BNEED(b, h->dev == b->dev, AUSM_ERR_INVALID, "solver and batch are on different devices");
  BNEED(b, h->engine == AUSM_ENGINE_FUSED, AUSM_ERR_STATE, "batch members use the fused engine");
  BNEED(b, h->has_grid && h->has_state, AUSM_ERR_STATE, "a member needs a grid and a state");
  int rc = use_dev(b);
  if (rc) return rc;
  // the member's queued work completes before anything on the batch stream that follows
  BCU(b, cudaEventRecord(h->e0, h->st));
  BCU(b, cudaStreamWaitEvent(b->st, h->e0, 0));
  b->members.push_back(h);
  h->batch = b;
  h->st = b->st;
  relayout(b);
  return ensure_capacity(b);
}

int ausm_batch_remove(ausm_batch* b, ausm_solver* h) {
  BNEED(b, b && h, AUSM_ERR_INVALID, "null handle");
  BNEED(b, h->batch == b, AUSM_ERR_NOT_FOUND, "solver is not a member of this batch");
  return ausm::batch_detach(b, h);
}

int ausm_batch_size(const ausm_batch* b, int* n) {
  if (!b || !n) return bfail(nullptr, AUSM_ERR_INVALID, "null argument");
  *n = (int)b->members.size();
  return AUSM_OK;
}

int ausm_batch_member(const ausm_batch* b, int k, ausm_solver** h) {
  if (!b || !h) return bfail(nullptr, AUSM_ERR_INVALID, "null argument");
  if (k < 0 || k >= (int)b->members.size()) return bfail(nullptr, AUSM_ERR_INVALID, "member index out of range");
  *h = b->members[k];
  return AUSM_OK;
}

int ausm_batch_set_graphs(ausm_batch* b, int enable) {
  BNEED(b, b, AUSM_ERR_INVALID, "null handle");
  b->graphs = enable != 0;
  return AUSM_OK;
}

}  // extern "C"

namespace {
// ausm_batch_step; read_err as in api.cu's step_impl
int batch_step_impl(ausm_batch* b, int n, float* dt_wave, bool read_err) {
  BNEED(b, b, AUSM_ERR_INVALID, "null handle");
  BNEED(b, n >= 0, AUSM_ERR_INVALID, "n must be >= 0");
  int rc = use_dev(b);
  if (rc) return rc;
  const int ns = (int)b->members.size();
  if (ns == 0 || n == 0) return AUSM_OK;
  for (ausm_solver* h : b->members)
    BNEED(b, h->has_grid && h->has_state, AUSM_ERR_STATE, "a member lost its grid or state");
  rc = tune_rows(b);
  if (rc) return rc;
  rc = sync_descriptors(b);
  if (rc) return rc;
  rc = run_steps(b, n);
  if (rc) return rc;
  for (size_t k = 0; k < b->members.size(); k++) {
    ausm_solver* h = b->members[b->order[k]];
    h->cur = (h->cur + n) % 3;
    b->mirror[k].cur = h->cur;  // the device advanced its copy
    ausm::ramp_after_steps(h, n);
  }
  if (b->tma && (read_err || dt_wave) && (rc = queue_err_read(b))) return rc;
  if (!dt_wave) return AUSM_OK;
  BCU(b, cudaMemcpyAsync(b->h_out, b->d_out, ns * 2 * sizeof(float), cudaMemcpyDeviceToHost, b->st));
  if ((rc = sync_and_check(b))) return rc;
  for (int k = 0; k < ns; k++) {
    dt_wave[2 * b->order[k]] = b->h_out[2 * k];
    dt_wave[2 * b->order[k] + 1] = b->h_out[2 * k + 1];
  }
  for (int k = 0; k < ns; k++)
    if (!std::isfinite(dt_wave[2 * k + 1]) || !std::isfinite(dt_wave[2 * k]))
      return bfail(b, AUSM_ERR_DIVERGED, "member " + std::to_string(k) + ": max wave speed is not finite");
  return AUSM_OK;
}
}  // namespace

extern "C" {

int ausm_batch_step(ausm_batch* b, int n, float* dt_wave) { return batch_step_impl(b, n, dt_wave, true); }

int ausm_batch_residual_l2(ausm_batch* b, double* l2) {
  BNEED(b, b && l2, AUSM_ERR_INVALID, "null argument");
  int rc = use_dev(b);
  if (rc) return rc;
  const int ns = (int)b->members.size();
  if (ns == 0) return AUSM_OK;
  rc = sync_descriptors(b);
  if (rc) return rc;
  for (const ausm_batch::Group& q : b->groups)
    ausm::launch_batch_stage(q.scheme, 0, false, b->d_solves, b->d_items, b->d_steps, b->d_maps, q.t_lo, q.t_hi, 0, b->rows, nullptr,
                             b->st);
  ausm::launch_batch_residual_norm(b->d_solves, ns, b->total_chunks, b->d_part, b->d_l2, b->st);
  BCU(b, cudaGetLastError());
  BCU(b, cudaMemcpyAsync(b->h_l2, b->d_l2, ns * sizeof(double), cudaMemcpyDeviceToHost, b->st));
  if ((rc = sync_and_check(b))) return rc;
  for (int k = 0; k < ns; k++) l2[b->order[k]] = b->h_l2[k];
  return AUSM_OK;
}

int ausm_batch_synchronize(ausm_batch* b) {
  BNEED(b, b, AUSM_ERR_INVALID, "null handle");
  return sync_and_check(b);
}

int ausm_batch_time_steps(ausm_batch* b, int n, int reps, float* ms_out) {
  BNEED(b, b && ms_out && n > 0 && reps > 0, AUSM_ERR_INVALID, "need n > 0, reps > 0 and an output");
  int rc = use_dev(b);
  if (rc) return rc;
  BCU(b, cudaEventRecord(b->e0, b->st));
  for (int r = 0; r < reps; r++) {
    rc = batch_step_impl(b, n, nullptr, false);
    if (rc) return rc;
  }
  BCU(b, cudaEventRecord(b->e1, b->st));
  if (b->tma && (rc = queue_err_read(b))) return rc;
  BCU(b, cudaEventSynchronize(b->e1));
  BCU(b, cudaEventElapsedTime(ms_out, b->e0, b->e1));
  return sync_and_check(b);
}

}  // extern "C"

namespace ausm {
int batch_detach(ausm_batch* b, ausm_solver* h) {
  cudaSetDevice(b->dev);
  // the member's own stream continues after everything the batch queued so far
  cudaEventRecord(h->e0, b->st);
  cudaStreamWaitEvent(h->own_st, h->e0, 0);
  h->st = h->own_st;
  h->batch = nullptr;
  for (size_t k = 0; k < b->members.size(); k++)
    if (b->members[k] == h) {
      b->members.erase(b->members.begin() + k);
      break;
    }
  relayout(b);
  return AUSM_OK;
}
}  // namespace ausm
