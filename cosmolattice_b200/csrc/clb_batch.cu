// clb_batch.cu - batched lphi4 ensemble behind the C ABI (clb_batch_*).
//
// Many independent one-field lphi4 lattices advance together: each fused VV stage is one
// k_batch_sweep launch over all members plus one k_batch_tail (one block per member), the
// schedule of the single-lattice fused path (clb_api.cu, EvolveVV).  clb_batch_evolve captures the
// launches of a whole call in a CUDA graph and replays it, so a 2000-step ensemble run is one
// graph launch with no host work between steps.

#include "../../include/clb200.h"
#include "clb_batch.cuh"
#include "clb_vv.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

using namespace clb;

namespace {
thread_local std::string g_berr;
constexpr int kPackBlocks = 148 * 8;
constexpr int kMeasBlocks = 148 * 4;

// Sweep configurations the autotuner chooses from: block shapes compiled for (threads along z and
// y, z sites per thread), and the x-run lengths (planes per block, capped at the member's N).
struct TileShape {
  int bz, by, vz;
};
constexpr TileShape kTiles[] = {{32, 4, 1}, {32, 8, 1},  {32, 16, 1}, {64, 4, 1}, {16, 8, 2}, {16, 16, 2},
                                {32, 8, 2}, {8, 16, 4},  {8, 32, 4},  {16, 8, 4}, {16, 16, 4}};
constexpr int kNTiles = sizeof(kTiles) / sizeof(kTiles[0]);
constexpr int kRuns[] = {8, 16, 32, 64, 1024};
constexpr int kDefaultTile = 1, kDefaultRun = 32; // 32 x 8 tiles, 32-plane runs

// Shapes compiled for the persistent form (block z and y threads, z sites per thread); x-runs as
// kRuns.  Clusters of kClusterCTAs blocks (the portable maximum).
constexpr TileShape kPersist[] = {{32, 8, 1}, {16, 8, 2}, {16, 8, 4}, {32, 4, 1}};
constexpr int kNPersist = sizeof(kPersist) / sizeof(kPersist[0]);
constexpr int kClusterCTAs = 8;

// Tuned configurations by ensemble (precision, device and sorted member sizes), for the process:
// graph-form tile and run, then whether the persistent form won, with its shape and run.
struct Tuned {
  int tile, run;
  bool persist;
  int ptile, prun;
};
std::map<std::string, Tuned> g_tuned;

} // namespace

struct clb_batch {
  int n = 0;
  clb_config cfg{};                // shared dt, evolver, expansion, precision, device
  std::vector<clb_model_desc> md;
  std::vector<BatchLat> lat;       // host copy of the member descriptors
  std::vector<int> blk_lat;
  int total_blocks = 0;
  int tile = kDefaultTile, run = kDefaultRun; // sweep configuration (kTiles index, x-run)
  bool tuned = false;                         // set by the autotuner or the caller
  clb_batch_tuning tuning{};
  size_t blk_cap = 0, part_cap = 0;           // d_blk, d_part capacities (elements)
  long long total_elems = 0;
  bool fp32 = false;
  size_t esz = 8;
  void *f[2] = {nullptr, nullptr}, *p[2] = {nullptr, nullptr};
  int cf = 0, rs = 0;
  BatchLat *d_lat = nullptr;
  int *d_blk = nullptr;
  DevState *d_st = nullptr;
  double *d_part = nullptr, *d_sums = nullptr, *d_stage = nullptr;
  size_t stage_n = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::vector<double> ws;
  std::vector<char> has_state;
  bool initialized = false;
  double last_ms = 0;
  int64_t launches = 0;
  struct Graph {
    cudaGraphExec_t exec;
    int64_t launches; // kernels in the graph
  };
  std::map<std::tuple<int64_t, int, int>, Graph> graphs; // (steps, cf, rs) -> graph
  // the persistent form (k_batch_persist): shape index into kPersist, x-run, cluster count
  bool persist = false;
  int ptile = 0, prun = 8, pclusters = 0;
  BatchLat *d_plat = nullptr; // member descriptors with the persistent tile grid
  int *d_members = nullptr, *d_offsets = nullptr;
  clb_batch_form form{};
  std::string err;
  int fail(int code, const std::string &m)
  {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char *where)
  {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return CLB_ECUDA;
  }
};

namespace {

template <int BZ, int BY, int VZ, class R>
void sweep_tile(clb_batch *b, bool drift, bool kick, int red, double dtw, double h1, double h2)
{
  const R *fin = static_cast<const R *>(b->f[b->cf]), *pin = static_cast<const R *>(b->p[b->cf]);
  R *fout = static_cast<R *>(b->f[drift ? b->cf ^ 1 : b->cf]), *pout = static_cast<R *>(b->p[drift ? b->cf ^ 1 : b->cf]);
  const dim3 grid(b->total_blocks), block(BZ, BY);
  constexpr int SM = Ring<BZ, BY, VZ, R>::BYTES;
#define CLB_BS(D, K, RD)                                                                                               \
  k_batch_sweep<BZ, BY, VZ, R, D, K, RD><<<grid, block, SM, b->stream>>>(fin, pin, fout, pout, b->d_lat, b->d_blk,   \
                                                                           b->d_st, b->rs, dtw, h1, h2, b->d_part)
  if (drift && kick && red)
    CLB_BS(true, true, 3);
  else if (drift && kick)
    CLB_BS(true, true, 0);
  else if (kick)
    CLB_BS(false, true, 0);
  else
    CLB_BS(false, false, 3);
#undef CLB_BS
}

// Rings above the default 48 KB of dynamic shared memory need the kernel's opt-in (set once per
// kernel, outside any stream capture: at layout time).
template <int BZ, int BY, int VZ, class R> cudaError_t ring_attr()
{
  constexpr int SM = Ring<BZ, BY, VZ, R>::BYTES;
  if (SM <= 48 * 1024) return cudaSuccess;
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_batch_sweep<BZ, BY, VZ, R, true, true, 3>, a, SM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_sweep<BZ, BY, VZ, R, true, true, 0>, a, SM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_sweep<BZ, BY, VZ, R, false, true, 0>, a, SM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_sweep<BZ, BY, VZ, R, false, false, 3>, a, SM);
  return e;
}

template <class R> cudaError_t ring_attr_tile(int t)
{
  switch (t) {
  case 0: return ring_attr<32, 4, 1, R>();
  case 1: return ring_attr<32, 8, 1, R>();
  case 2: return ring_attr<32, 16, 1, R>();
  case 3: return ring_attr<64, 4, 1, R>();
  case 4: return ring_attr<16, 8, 2, R>();
  case 5: return ring_attr<16, 16, 2, R>();
  case 6: return ring_attr<32, 8, 2, R>();
  case 7: return ring_attr<8, 16, 4, R>();
  case 8: return ring_attr<8, 32, 4, R>();
  case 9: return ring_attr<16, 8, 4, R>();
  default: return ring_attr<16, 16, 4, R>();
  }
}

// One sweep with the current configuration; advance = false leaves the buffer parity and the
// reference slot as they are (the autotuner's timing sweeps write only the idle buffers).
template <class R>
void sweep_launch(clb_batch *b, bool drift, bool kick, int red, double dtw, double h1, double h2, bool advance = true)
{
  switch (b->tile) {
  case 0: sweep_tile<32, 4, 1, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 1: sweep_tile<32, 8, 1, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 2: sweep_tile<32, 16, 1, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 3: sweep_tile<64, 4, 1, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 4: sweep_tile<16, 8, 2, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 5: sweep_tile<16, 16, 2, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 6: sweep_tile<32, 8, 2, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 7: sweep_tile<8, 16, 4, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 8: sweep_tile<8, 32, 4, R>(b, drift, kick, red, dtw, h1, h2); break;
  case 9: sweep_tile<16, 8, 4, R>(b, drift, kick, red, dtw, h1, h2); break;
  default: sweep_tile<16, 16, 4, R>(b, drift, kick, red, dtw, h1, h2); break;
  }
  ++b->launches;
  if (!advance) return;
  if (drift) b->cf ^= 1;
  if (sizeof(R) == 4 && (drift || kick)) b->rs ^= 1;
}

// Member sweep grids for (tile, run): per-member tile counts, block ranges and the block ->
// member table, uploaded to the device (buffers grown when needed).
cudaError_t layout(clb_batch *b, int tile, int run)
{
  const TileShape t = kTiles[tile];
  const cudaError_t ea = b->fp32 ? ring_attr_tile<float>(tile) : ring_attr_tile<double>(tile);
  if (ea != cudaSuccess) return ea;
  int blocks = 0;
  b->blk_lat.clear();
  for (int i = 0; i < b->n; ++i) {
    BatchLat &L = b->lat[(size_t)i];
    L.gx = (L.N + t.bz * t.vz - 1) / (t.bz * t.vz);
    L.gy = (L.N + t.by - 1) / t.by;
    L.LX = std::min(L.N, run);
    L.gz = (L.N + L.LX - 1) / L.LX;
    L.first_block = blocks;
    L.nblocks = L.gx * L.gy * L.gz;
    blocks += L.nblocks;
    for (int k = 0; k < L.nblocks; ++k) b->blk_lat.push_back(i);
  }
  cudaError_t e = cudaSuccess;
  if ((size_t)blocks > b->blk_cap) {
    if (b->d_blk) cudaFree(b->d_blk);
    b->d_blk = nullptr;
    e = cudaMalloc(&b->d_blk, (size_t)blocks * sizeof(int));
    if (e != cudaSuccess) return e;
    b->blk_cap = (size_t)blocks;
  }
  const size_t part = (size_t)std::max(blocks * kRedSlots, kMeasBlocks * 7);
  if (part > b->part_cap) {
    if (b->d_part) cudaFree(b->d_part);
    b->d_part = nullptr;
    e = cudaMalloc(&b->d_part, part * sizeof(double));
    if (e != cudaSuccess) return e;
    b->part_cap = part;
  }
  e = cudaMemcpyAsync(b->d_lat, b->lat.data(), (size_t)b->n * sizeof(BatchLat), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_blk, b->blk_lat.data(), (size_t)blocks * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return e;
  b->total_blocks = blocks;
  b->tile = tile;
  b->run = run;
  return cudaSuccess;
}

// Drops the captured graphs (they hold the old grid).
void drop_graphs(clb_batch *b)
{
  for (auto &g : b->graphs) cudaGraphExecDestroy(g.second.exec);
  b->graphs.clear();
}

// VZ sites per thread need every member's N to be a multiple of VZ (aligned vector loads).
bool tile_fits(const clb_batch *b, int t)
{
  for (const BatchLat &L : b->lat)
    if (L.N % kTiles[t].vz) return false;
  return true;
}

clb_batch_tuning tuning_of(int t, int run, int candidates, double ms, double ms_def)
{
  return clb_batch_tuning{kTiles[t].bz * kTiles[t].vz, kTiles[t].by, kTiles[t].vz, run, candidates, ms, ms_def};
}

std::string tune_key(const clb_batch *b)
{
  std::vector<int> ns;
  for (const BatchLat &L : b->lat) ns.push_back(L.N);
  std::sort(ns.begin(), ns.end());
  std::string k = std::to_string(b->cfg.device) + (b->fp32 ? "/fp32/" : "/fp64/");
  for (int n : ns) k += std::to_string(n) + ",";
  return k;
}

void sweep(clb_batch *b, bool drift, bool kick, int red, double dtw, double h1, double h2, bool advance = true)
{
  if (b->fp32)
    sweep_launch<float>(b, drift, kick, red, dtw, h1, h2, advance);
  else
    sweep_launch<double>(b, drift, kick, red, dtw, h1, h2, advance);
}

// Autotuner: times the fused drift + two-kick + reduction sweep (the one every stage runs) of the
// whole ensemble for every (tile, run) candidate, `reps` launches each after a warm-up launch, on
// the handle's stream with CUDA events, and keeps the fastest.  The timing sweeps read the current
// state and write only the idle state buffers, the next reference slot and the partials, so the
// state is unchanged.
int autotune_graph(clb_batch *b, int reps)
{
  const double dt = b->cfg.dt, w = b->ws[0];
  cudaError_t e = cudaSuccess;
  double best = 1e300, def = 0;
  int bt = kDefaultTile, br = kDefaultRun, count = 0;
  int maxN = 0;
  for (const BatchLat &L : b->lat) maxN = std::max(maxN, L.N);
  for (int t = 0; t < kNTiles && e == cudaSuccess; ++t) {
    if (!tile_fits(b, t)) continue;
    for (int run : kRuns) {
      if (run != kRuns[0] && run / 2 >= maxN) continue; // the same grids as run / 2
      if ((e = layout(b, t, run)) != cudaSuccess) break;
      sweep(b, true, true, 3, dt * w, w * dt / 2, w * dt / 2, false);
      cudaEventRecord(b->ev[0], b->stream);
      for (int r = 0; r < reps; ++r) sweep(b, true, true, 3, dt * w, w * dt / 2, w * dt / 2, false);
      cudaEventRecord(b->ev[1], b->stream);
      if ((e = cudaEventSynchronize(b->ev[1])) != cudaSuccess) break;
      float ms = 0;
      cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
      const double per = ms / reps;
      ++count;
      if (t == kDefaultTile && run == kDefaultRun) def = per;
      if (per < best) {
        best = per;
        bt = t;
        br = run;
      }
    }
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = layout(b, bt, br);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_autotune");
  drop_graphs(b);
  b->tuned = true;
  b->tuning = tuning_of(bt, br, count, best, def);
  return CLB_OK;
}

void btail(clb_batch *b, uint32_t flags, bool reduced, double w = 0, double w2 = 0)
{
  TailOp op{flags, 0, w, w2, nullptr, -1};
  k_batch_tail<<<b->n, 256, 0, b->stream>>>(b->d_part, b->d_lat, b->d_st, op, reduced ? 1 : 0);
  ++b->launches;
}

cudaError_t persist_run(clb_batch *b, int64_t nsteps);

// The fused VV schedule of EvolveVV (clb_api.cu) over all members: one launch of the persistent
// form, or a sweep and a tail launch per stage.
void evolve_launches(clb_batch *b, int64_t nsteps)
{
  if (b->persist) {
    persist_run(b, nsteps);
    return;
  }
  const double dt = b->cfg.dt;
  const bool ex = b->cfg.expansion != 0;
  const std::vector<double> &ws = b->ws;
  const size_t P = ws.size(), S = 2 * P - 1;
  auto wof = [&](size_t i) { return ws[i < P ? i : S - i - 1]; };
  const int64_t total = nsteps * (int64_t)S;
  const double w0 = wof(0);
  if (ex) btail(b, T_VV_KICK_HALF, false, 0, w0);
  sweep(b, false, true, 0, 0.0, w0 * dt / 2, 0.0);
  if (ex) btail(b, T_VV_DRIFT, false, 0, w0);
  for (int64_t k = 0; k < total; ++k) {
    const size_t i = (size_t)(k % (int64_t)S);
    const double w = wof(i);
    const bool more = k + 1 < total;
    const double wn = more ? wof((size_t)((k + 1) % (int64_t)S)) : 0.0;
    sweep(b, true, true, ex ? 3 : 0, dt * w, w * dt / 2, more ? wn * dt / 2 : 0.0);
    if (ex) {
      uint32_t fl = T_STORE_PI2_I | T_STORE_FIELDS | T_VV_KICK_ONE;
      if (more) fl |= T_VV_KICK_HALF | T_VV_DRIFT;
      btail(b, fl, true, w, wn);
    }
  }
}

// ---- persistent form ----------------------------------------------------------------------------
template <class R, int BZ, int BY, int VZ> struct Persist {
  static_assert(Ring<BZ, BY, VZ, R>::BYTES <= 48 * 1024, "persistent shapes keep the default shared-memory limit");
  static cudaLaunchConfig_t config(clb_batch *b, int clusters, cudaLaunchAttribute *at)
  {
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kClusterCTAs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t c{};
    c.gridDim = dim3((unsigned)(clusters * kClusterCTAs));
    c.blockDim = dim3(BZ, BY);
    c.dynamicSmemBytes = Ring<BZ, BY, VZ, R>::BYTES; // at most 48 KB for the persistent shapes
    c.stream = b->stream;
    c.attrs = at;
    c.numAttrs = 1;
    return c;
  }
  static int max_clusters(clb_batch *b)
  {
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t c = config(b, 148, at);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_batch_persist<BZ, BY, VZ, R>, &c) != cudaSuccess) return 0;
    return n;
  }
  static cudaError_t launch(clb_batch *b, const PersistArgs &a)
  {
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t c = config(b, b->pclusters, at);
    R *f0 = static_cast<R *>(b->f[0]), *f1 = static_cast<R *>(b->f[1]);
    R *p0 = static_cast<R *>(b->p[0]), *p1 = static_cast<R *>(b->p[1]);
    return cudaLaunchKernelEx(&c, k_batch_persist<BZ, BY, VZ, R>, f0, p0, f1, p1, (const BatchLat *)b->d_plat,
                              b->d_st, (const int *)b->d_members, (const int *)b->d_offsets, a);
  }
};

// Calls F with the Persist instantiation of shape t for the ensemble's precision.
template <class F> auto with_persist(const clb_batch *b, int t, F &&f)
{
#define CLB_PS(R)                                                                                                        switch (t) {                                                                                                           case 0: return f(Persist<R, 32, 8, 1>{});                                                                             case 1: return f(Persist<R, 16, 8, 2>{});                                                                             case 2: return f(Persist<R, 16, 8, 4>{});                                                                             default: return f(Persist<R, 32, 4, 1>{});                                                                            }
  if (b->fp32) {
    CLB_PS(float)
  } else {
    CLB_PS(double)
  }
#undef CLB_PS
}

bool persist_fits(const clb_batch *b, int t)
{
  for (const BatchLat &L : b->lat)
    if (L.N % kPersist[t].vz) return false;
  return true;
}

// The persistent form's member table for shape t and x-run `run`: each member's tile grid, and the
// members dealt to as many clusters as the device holds at once (at most one per member), longest
// first to the least-loaded cluster.  A member's cost is its CTA's share of tiles per stage (the
// sites of ceil(tiles / 8) tiles) plus a fixed per-stage cost of the cluster barriers and tail.
cudaError_t persist_layout(clb_batch *b, int t, int run)
{
  const TileShape sh = kPersist[t];
  int nc = with_persist(b, t, [&](auto P) { return decltype(P)::max_clusters(b); });
  if (nc < 1) return cudaErrorInvalidConfiguration;
  nc = std::min(nc, b->n);
  std::vector<BatchLat> L = b->lat;
  std::vector<std::pair<double, int>> cost;
  for (int i = 0; i < b->n; ++i) {
    BatchLat &l = L[(size_t)i];
    l.gx = (l.N + sh.bz * sh.vz - 1) / (sh.bz * sh.vz);
    l.gy = (l.N + sh.by - 1) / sh.by;
    l.LX = std::min(l.N, run);
    l.gz = (l.N + l.LX - 1) / l.LX;
    l.first_block = 0;
    l.nblocks = l.gx * l.gy * l.gz;
    const double per_cta = (double)((l.nblocks + kClusterCTAs - 1) / kClusterCTAs) * sh.bz * sh.vz * sh.by * l.LX;
    cost.push_back({per_cta + 4096.0, i});
  }
  std::stable_sort(cost.begin(), cost.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
  std::vector<double> load((size_t)nc, 0.0);
  std::vector<std::vector<int>> lists((size_t)nc);
  for (const auto &c : cost) {
    const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
    load[k] += c.first;
    lists[k].push_back(c.second);
  }
  std::vector<int> members, offsets{0};
  for (const auto &l : lists) {
    members.insert(members.end(), l.begin(), l.end());
    offsets.push_back((int)members.size());
  }
  cudaError_t e = cudaMemcpyAsync(b->d_plat, L.data(), L.size() * sizeof(BatchLat), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_members, members.data(), members.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_offsets, offsets.data(), offsets.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return e;
  b->ptile = t;
  b->prun = run;
  b->pclusters = nc;
  return cudaSuccess;
}

// One k_batch_persist launch for nsteps steps; the buffer parity and reference slot advance as the
// per-stage launches would (a first kick sweep, then one drift sweep per stage).
cudaError_t persist_run(clb_batch *b, int64_t nsteps)
{
  PersistArgs a{};
  const std::vector<double> &ws = b->ws;
  const size_t P = ws.size(), S = 2 * P - 1;
  for (size_t i = 0; i < S; ++i) a.w[i] = ws[i < P ? i : S - i - 1];
  a.dt = b->cfg.dt;
  a.expansion = b->cfg.expansion != 0;
  a.stages = (int)S;
  a.nsteps = nsteps;
  a.cf0 = b->cf;
  a.rs0 = b->rs;
  const cudaError_t e = with_persist(b, b->ptile, [&](auto Q) { return decltype(Q)::launch(b, a); });
  ++b->launches;
  const int64_t sweeps = nsteps * (int64_t)S;
  if (sweeps % 2) b->cf ^= 1;
  if (b->fp32 && (sweeps + 1) % 2) b->rs ^= 1;
  return e;
}

// The state a timing launch starts from: the live buffers, the members' DevStates, the parity.
struct Snapshot {
  void *f = nullptr, *p = nullptr;
  DevState *st = nullptr;
  int cf = 0, rs = 0;
  ~Snapshot()
  {
    for (void *q : {f, p, (void *)st})
      if (q) cudaFree(q);
  }
};

cudaError_t snap_take(clb_batch *b, Snapshot &s)
{
  const size_t bytes = (size_t)b->total_elems * b->esz;
  cudaError_t e = cudaMalloc(&s.f, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s.p, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s.st, (size_t)b->n * sizeof(DevState));
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.f, b->f[b->cf], bytes, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s.p, b->p[b->cf], bytes, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.st, b->d_st, (size_t)b->n * sizeof(DevState), cudaMemcpyDeviceToDevice, b->stream);
  s.cf = b->cf;
  s.rs = b->rs;
  return e;
}

cudaError_t snap_put(clb_batch *b, const Snapshot &s)
{
  const size_t bytes = (size_t)b->total_elems * b->esz;
  b->cf = s.cf;
  b->rs = s.rs;
  cudaError_t e = cudaMemcpyAsync(b->f[b->cf], s.f, bytes, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->p[b->cf], s.p, bytes, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_st, s.st, (size_t)b->n * sizeof(DevState), cudaMemcpyDeviceToDevice, b->stream);
  return e;
}

// Milliseconds per step of a `steps`-step evolve call in the current form: captured as a graph,
// launched once to warm up and once timed (CUDA events on the handle's stream), each launch from
// the snapshot.
cudaError_t time_form(clb_batch *b, const Snapshot &sn, int64_t steps, double &ms)
{
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  cudaError_t e = snap_put(b, sn);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  const int64_t l0 = b->launches;
  evolve_launches(b, steps);
  const int64_t nl = b->launches - l0;
  b->launches = l0;
  e = cudaStreamEndCapture(b->stream, &g);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  for (int r = 0; r < 2 && e == cudaSuccess; ++r) {
    if ((e = snap_put(b, sn)) != cudaSuccess) break;
    cudaEventRecord(b->ev[0], b->stream);
    e = cudaGraphLaunch(x, b->stream);
    b->launches += nl;
    cudaEventRecord(b->ev[1], b->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b->ev[1]);
  }
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, b->ev[0], b->ev[1]);
  ms = t / (double)steps;
  if (x) cudaGraphExecDestroy(x);
  const cudaError_t e2 = snap_put(b, sn);
  return e != cudaSuccess ? e : e2;
}

// CLB_BATCH_PERSISTENT: "0" keeps the per-stage graph form, "1" the persistent form, unset lets
// the autotuner choose.
int persistent_choice()
{
  const char *env = std::getenv("CLB_BATCH_PERSISTENT");
  if (env && env[0] == '0') return 0;
  if (env && env[0] == '1') return 1;
  return -1;
}

bool persist_allowed(const clb_batch *b) { return 2 * b->ws.size() - 1 <= (size_t)kMaxStages; }

// The full autotuner: the graph form's sweep configuration (autotune_graph), then whole evolve
// calls of kFormSteps steps in that form and in the persistent form for every compiled shape and
// x-run, each from a snapshot of the state (restored afterwards), keeping the fastest form.
constexpr int64_t kFormSteps = 8;
int autotune(clb_batch *b, int reps)
{
  int r = autotune_graph(b, reps);
  if (r != CLB_OK) return r;
  const int choice = persist_allowed(b) ? persistent_choice() : 0;
  b->form = clb_batch_form{};
  b->persist = false;
  if (choice != 0) {
    Snapshot sn;
    cudaError_t e = snap_take(b, sn);
    double best = 1e300, ms = 0;
    int bt = -1, br = 0;
    if (e == cudaSuccess && choice < 0) {
      e = time_form(b, sn, kFormSteps, ms);
      b->form.ms_graph = ms;
    }
    int maxN = 0;
    for (const BatchLat &L : b->lat) maxN = std::max(maxN, L.N);
    for (int t = 0; t < kNPersist && e == cudaSuccess; ++t) {
      if (!persist_fits(b, t)) continue;
      for (int run : {8, 16, 32}) {
        if (run != 8 && run / 2 >= maxN) continue;
        if ((e = persist_layout(b, t, run)) != cudaSuccess) break;
        b->persist = true;
        e = time_form(b, sn, kFormSteps, ms);
        b->persist = false;
        if (e != cudaSuccess) break;
        ++b->form.candidates;
        if (ms < best) {
          best = ms;
          bt = t;
          br = run;
        }
      }
    }
    if (e == cudaSuccess && bt >= 0) {
      e = persist_layout(b, bt, br);
      b->form.ms_persistent = best;
      b->persist = choice == 1 || best < b->form.ms_graph;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_autotune: forms");
  }
  g_tuned[tune_key(b)] = Tuned{b->tile, b->run, b->persist, b->ptile, b->prun};
  return CLB_OK;
}

int check(clb_batch *b, const char *where)
{
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, where);
  std::vector<DevState> s((size_t)b->n);
  e = cudaMemcpy(s.data(), b->d_st, s.size() * sizeof(DevState), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return b->cuda_fail(e, where);
  for (int i = 0; i < b->n; ++i)
    if (s[(size_t)i].status != 0)
      return b->fail(CLB_ENONFINITE, std::string(where) + ": member " + std::to_string(i) + " has a non-finite average or a(t)");
  return CLB_OK;
}

} // namespace

extern "C" {

const char *clb_batch_last_error(const clb_batch *b) { return b ? b->err.c_str() : g_berr.c_str(); }

void clb_batch_destroy(clb_batch *b)
{
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &g : b->graphs) cudaGraphExecDestroy(g.second.exec);
  for (int i = 0; i < 2; ++i) {
    if (b->f[i]) cudaFree(b->f[i]);
    if (b->p[i]) cudaFree(b->p[i]);
  }
  for (void *q : {(void *)b->d_lat, (void *)b->d_blk, (void *)b->d_st, (void *)b->d_part, (void *)b->d_sums,
                  (void *)b->d_stage, (void *)b->d_plat, (void *)b->d_members, (void *)b->d_offsets})
    if (q) cudaFree(q);
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int clb_batch_create(const clb_config *cfgs, const clb_model_desc *mds, int32_t n, clb_batch **out)
{
  if (!cfgs || !mds || !out || n < 1) {
    g_berr = "clb_batch_create: null argument or empty batch";
    return CLB_EINVAL;
  }
  *out = nullptr;
  const clb_config &c0 = cfgs[0];
  if (c0.expansion && c0.fixed_background) {
    g_berr = "clb_batch_create: the batched ensemble runs the self-consistent expansion";
    return CLB_EUNSUPPORTED;
  }
  std::vector<double> ws = vv_coefficients(c0.evolver);
  if (ws.empty()) {
    g_berr = "clb_batch_create: the batched ensemble runs the VV evolvers";
    return CLB_EUNSUPPORTED;
  }
  if (c0.precision != CLB_PREC_FP64 && c0.precision != CLB_PREC_FP32_SPLIT) {
    g_berr = "clb_batch_create: unknown precision";
    return CLB_EINVAL;
  }
  if (c0.dt == 0 || !std::isfinite(c0.dt)) {
    g_berr = "clb_batch_create: dt cannot be zero, abort.";
    return CLB_EINVAL;
  }
  for (int i = 0; i < n; ++i) {
    const clb_config &c = cfgs[i];
    const clb_model_desc &m = mds[i];
    if (c.dt != c0.dt || c.evolver != c0.evolver || c.expansion != c0.expansion || c.precision != c0.precision ||
        c.device != c0.device) {
      g_berr = "clb_batch_create: members must share dt, evolver, expansion, precision and device";
      return CLB_EINVAL;
    }
    if (m.kind != CLB_MODEL_LPHI4 || m.n_scalars != 1) {
      g_berr = "clb_batch_create: members are one-field lphi4 lattices";
      return CLB_EUNSUPPORTED;
    }
    if (c.N < 2 || c.N > 1024 || !(c.dx > 0) || !(m.fStar > 0) || !(m.MPl > 0) || !(m.omegaStar > 0)) {
      g_berr = "clb_batch_create: member " + std::to_string(i) + ": N in [2, 1024], positive dx, fStar, omegaStar, MPl";
      return CLB_EINVAL;
    }
  }
  cudaError_t e = cudaSetDevice(c0.device);
  if (e != cudaSuccess) {
    g_berr = std::string("clb_batch_create: cudaSetDevice: ") + cudaGetErrorString(e);
    return CLB_ECUDA;
  }
  clb_batch *b = new clb_batch();
  b->n = n;
  b->cfg = c0;
  b->md.assign(mds, mds + n);
  b->ws = ws;
  b->fp32 = c0.precision == CLB_PREC_FP32_SPLIT;
  b->esz = b->fp32 ? 4 : 8;
  b->has_state.assign((size_t)n, 0);
  long long off = 0;
  for (int i = 0; i < n; ++i) {
    BatchLat L{};
    const int N = cfgs[i].N;
    L.N = N;
    L.off = off;
    L.inv_dx2 = 1.0 / (cfgs[i].dx * cfgs[i].dx);
    L.mc = ScalarModel::couplings(mds[i].couplings);
    const double fm = mds[i].fStar / mds[i].MPl;
    L.sp = SFParams{mds[i].alpha, fm * fm, c0.dt, 1.0 / ((double)N * N * N)};
    const long long n3 = (long long)N * N * N;
    off += (n3 + 31) / 32 * 32; // 128-byte aligned members
    b->lat.push_back(L);
  }
  b->total_elems = off;
  long long max_n3 = 0;
  for (auto &L : b->lat) max_n3 = std::max(max_n3, (long long)L.N * L.N * L.N);
  b->stage_n = (size_t)max_n3;
  const size_t bytes = (size_t)off * b->esz;
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
  for (int i = 0; ok && i < 2; ++i)
    ok = cudaMalloc(&b->f[i], bytes) == cudaSuccess && cudaMalloc(&b->p[i], bytes) == cudaSuccess &&
         cudaMemset(b->f[i], 0, bytes) == cudaSuccess && cudaMemset(b->p[i], 0, bytes) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_lat, (size_t)n * sizeof(BatchLat)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_st, (size_t)n * sizeof(DevState)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_plat, (size_t)n * sizeof(BatchLat)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_members, (size_t)n * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_offsets, (size_t)(n + 1) * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_sums, 8 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_stage, b->stage_n * sizeof(double)) == cudaSuccess;
  ok = ok && cudaEventCreate(&b->ev[0]) == cudaSuccess && cudaEventCreate(&b->ev[1]) == cudaSuccess;
  if (ok) {
    // a configuration tuned earlier in this process for the same ensemble, else the default
    auto it = g_tuned.find(tune_key(b));
    const bool cached = it != g_tuned.end();
    ok = layout(b, cached ? it->second.tile : kDefaultTile, cached ? it->second.run : kDefaultRun) == cudaSuccess;
    if (ok && cached) {
      b->tuned = true;
      b->tuning = tuning_of(b->tile, b->run, 0, 0.0, 0.0);
      if (it->second.persist) {
        ok = persist_layout(b, it->second.ptile, it->second.prun) == cudaSuccess;
        b->persist = true;
      }
    }
  }
  if (ok) {
    std::vector<DevState> s((size_t)n);
    for (auto &x : s) {
      x = DevState{};
      x.aI = x.aSI = x.aIM = 1.0;
      x.drift_p = x.kick_A = x.kick_B = 1.0;
    }
    ok = cudaMemcpy(b->d_st, s.data(), s.size() * sizeof(DevState), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  if (!ok) {
    g_berr = std::string("clb_batch_create: device allocation failed: ") + cudaGetErrorString(cudaGetLastError());
    clb_batch_destroy(b);
    return CLB_ENOMEM;
  }
  *out = b;
  return CLB_OK;
}

// Member i's state from host arrays (N^3 doubles each).  The FP32 split form stores deviations
// from the FP64 volume means, which become the member's references.
int clb_batch_set_state(clb_batch *b, int32_t i, const double *fields, const double *momenta, const clb_scalefactor *sf)
{
  if (!b || !fields || !momenta) return b ? b->fail(CLB_EINVAL, "clb_batch_set_state: null argument") : CLB_EINVAL;
  if (i < 0 || i >= b->n) return b->fail(CLB_EINVAL, "clb_batch_set_state: member index out of range");
  const BatchLat &L = b->lat[(size_t)i];
  const size_t n3 = (size_t)L.N * L.N * L.N;
  double fo = 0, po = 0;
  if (b->fp32) {
    for (size_t k = 0; k < n3; ++k) {
      fo += fields[k];
      po += momenta[k];
    }
    fo /= (double)n3;
    po /= (double)n3;
  }
  DevState s{};
  s.aI = s.aSI = s.aIM = 1.0;
  if (sf) {
    s.aI = sf->aI;
    s.aSI = sf->aSI;
    s.aIM = sf->aIM;
    s.aDotI = sf->aDotI;
    s.aDotSI = sf->aDotSI;
    s.aDotSIM = sf->aDotSIM;
  }
  const double al = b->md[(size_t)i].alpha;
  s.drift_p = std::pow(s.aSI, al - 3);
  s.kick_A = std::pow(s.aI, 1 + al);
  s.kick_B = std::pow(s.aI, 3 + al);
  s.ref_phi[0][0] = s.ref_phi[1][0] = fo;
  s.ref_pi[0][0] = s.ref_pi[1][0] = po;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  for (int w = 0; w < 2 && e == cudaSuccess; ++w) {
    const double *src = w == 0 ? fields : momenta;
    void *dst = w == 0 ? b->f[b->cf] : b->p[b->cf];
    e = cudaMemcpyAsync(b->d_stage, src, n3 * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) break;
    if (b->fp32)
      k_batch_pack<float><<<kPackBlocks, 256, 0, b->stream>>>(b->d_stage, static_cast<float *>(dst) + L.off, n3, w == 0 ? fo : po);
    else
      k_batch_pack<double><<<kPackBlocks, 256, 0, b->stream>>>(b->d_stage, static_cast<double *>(dst) + L.off, n3, 0.0);
    e = cudaStreamSynchronize(b->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpy(b->d_st + i, &s, sizeof(s), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_set_state");
  b->has_state[(size_t)i] = 1;
  b->initialized = false;
  return CLB_OK;
}

int clb_batch_get_state(clb_batch *b, int32_t i, double *fields, double *momenta, clb_scalefactor *sf)
{
  if (!b) return CLB_EINVAL;
  if (i < 0 || i >= b->n) return b->fail(CLB_EINVAL, "clb_batch_get_state: member index out of range");
  const BatchLat &L = b->lat[(size_t)i];
  const size_t n3 = (size_t)L.N * L.N * L.N;
  DevState s;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, b->d_st + i, sizeof(s), cudaMemcpyDeviceToHost);
  for (int w = 0; w < 2 && e == cudaSuccess; ++w) {
    double *dst = w == 0 ? fields : momenta;
    if (!dst) continue;
    const void *src = w == 0 ? b->f[b->cf] : b->p[b->cf];
    if (b->fp32)
      k_batch_unpack<float><<<kPackBlocks, 256, 0, b->stream>>>(static_cast<const float *>(src) + L.off, b->d_stage, n3,
                                                                w == 0 ? s.ref_phi[b->rs][0] : s.ref_pi[b->rs][0]);
    else
      k_batch_unpack<double><<<kPackBlocks, 256, 0, b->stream>>>(static_cast<const double *>(src) + L.off, b->d_stage, n3, 0.0);
    e = cudaMemcpyAsync(dst, b->d_stage, n3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  }
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_get_state");
  if (sf) {
    sf->aI = s.aI;
    sf->aSI = s.aSI;
    sf->aIM = s.aIM;
    sf->aDotI = s.aDotI;
    sf->aDotSI = s.aDotSI;
    sf->aDotSIM = s.aDotSIM;
  }
  return CLB_OK;
}

// Averages::setAllAverages and aDot = sqrt(RHS) for every member (modelinitializer.h:74-80).
int clb_batch_initialize(clb_batch *b, int32_t correct_adot)
{
  if (!b) return CLB_EINVAL;
  for (int i = 0; i < b->n; ++i)
    if (!b->has_state[(size_t)i]) return b->fail(CLB_ESTATE, "clb_batch_initialize: member " + std::to_string(i) + " has no state");
  sweep(b, false, false, 3, 0.0, 0.0, 0.0);
  uint32_t fl = T_STORE_ALL;
  if (b->cfg.expansion && correct_adot) fl |= T_CORRECT_ADOT;
  btail(b, fl, true);
  const int r = check(b, "clb_batch_initialize");
  if (r == CLB_OK) b->initialized = true;
  return r;
}

// nsteps VV steps of every member, as one CUDA graph (captured once per (nsteps, buffer parity)).
int clb_batch_evolve(clb_batch *b, int64_t nsteps)
{
  if (!b) return CLB_EINVAL;
  if (!b->initialized) return b->fail(CLB_ESTATE, "clb_batch_evolve: call clb_batch_initialize first");
  if (nsteps < 0) return b->fail(CLB_EINVAL, "clb_batch_evolve: negative step count");
  if (nsteps == 0) return CLB_OK;
  if (!b->tuned) {
    // first evolve: choose the sweep configuration (CLB_BATCH_AUTOTUNE=0 keeps the default)
    const char *env = std::getenv("CLB_BATCH_AUTOTUNE");
    if (!(env && env[0] == '0')) {
      const int r = autotune(b, 5);
      if (r != CLB_OK) return r;
    } else {
      b->tuned = true;
      b->tuning = tuning_of(b->tile, b->run, 0, 0.0, 0.0);
      if (persist_allowed(b) && persistent_choice() == 1) {
        const int t = persist_fits(b, 0) ? 0 : 3;
        const cudaError_t e = persist_layout(b, t, 8);
        if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_evolve: persistent layout");
        b->persist = true;
      }
    }
  }
  const auto key = std::make_tuple(nsteps, b->cf, b->rs);
  auto it = b->graphs.find(key);
  const int cf0 = b->cf, rs0 = b->rs;
  if (it == b->graphs.end()) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_evolve: capture");
    const int64_t l0 = b->launches;
    evolve_launches(b, nsteps);
    const int64_t nl = b->launches - l0;
    e = cudaStreamEndCapture(b->stream, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->cf = cf0;
      b->rs = rs0;
      return b->cuda_fail(e, "clb_batch_evolve: graph");
    }
    it = b->graphs.emplace(key, clb_batch::Graph{x, nl}).first;
  } else {
    b->launches += it->second.launches;
    // replay: the buffer parity and reference slot advance as the captured launches did
    const int64_t sweeps = nsteps * (int64_t)(2 * b->ws.size() - 1);
    if (sweeps % 2) b->cf ^= 1;
    if (b->fp32 && (sweeps + 1) % 2) b->rs ^= 1;
  }
  cudaEventRecord(b->ev[0], b->stream);
  cudaError_t e = cudaGraphLaunch(it->second.exec, b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_evolve: launch");
  cudaEventRecord(b->ev[1], b->stream);
  const int r = check(b, "clb_batch_evolve");
  float ms = 0;
  if (cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]) == cudaSuccess) b->last_ms = ms;
  return r;
}

int clb_batch_last_evolve_ms(clb_batch *b, double *ms)
{
  if (!b || !ms) return CLB_EINVAL;
  *ms = b->last_ms;
  return CLB_OK;
}

int clb_batch_kernel_launches(clb_batch *b, int64_t *n)
{
  if (!b || !n) return CLB_EINVAL;
  *n = b->launches;
  return CLB_OK;
}

// Frequent measurement of member i: energies, Friedmann check and means (energiesmeasurer.h:45-122,
// meansmeasurer.h:28-48), with the setAllAverages side effect of Energies::rho (energies.h:219).
int clb_batch_measure(clb_batch *b, int32_t i, double e0, clb_measurement *m)
{
  if (!b || !m) return b ? b->fail(CLB_EINVAL, "clb_batch_measure: null argument") : CLB_EINVAL;
  if (i < 0 || i >= b->n) return b->fail(CLB_EINVAL, "clb_batch_measure: member index out of range");
  if (!b->initialized) return b->fail(CLB_ESTATE, "clb_batch_measure: call clb_batch_initialize first");
  const BatchLat &L = b->lat[(size_t)i];
  DevState s;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&s, b->d_st + i, sizeof(s), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_measure");
  const double al = b->md[(size_t)i].alpha;
  const double am = std::pow(s.aI, al - 3);
  if (b->fp32)
    k_batch_measure<float><<<kMeasBlocks, 256, 0, b->stream>>>(static_cast<const float *>(b->f[b->cf]),
                                                              static_cast<const float *>(b->p[b->cf]), L, b->d_st + i,
                                                              b->rs, am, b->d_part);
  else
    k_batch_measure<double><<<kMeasBlocks, 256, 0, b->stream>>>(static_cast<const double *>(b->f[b->cf]),
                                                               static_cast<const double *>(b->p[b->cf]), L, b->d_st + i,
                                                               b->rs, am, b->d_part);
  k_sum_partials<7><<<1, 256, 0, b->stream>>>(b->d_part, kMeasBlocks, b->d_sums);
  double v[7];
  e = cudaMemcpyAsync(v, b->d_sums, sizeof(v), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_measure");
  const double inv = L.sp.inv_n3;
  for (double &x : v) x *= inv;
  std::memset(m, 0, sizeof(*m));
  auto ipow = [](double x, int n) {
    double r = x;
    for (int k = 1; k < n; ++k) r = r * x;
    return r;
  };
  const double am6 = 1.0 / ipow(s.aI, 6), am2 = 1.0 / ipow(s.aI, 2);
  const double Ekin = 0.5 * v[0] * am6, Egrad = 0.5 * v[1] * am2, V = v[6];
  const double Etot = (Ekin + Egrad) + V;
  m->energies[0] = Ekin;
  m->energies[1] = Egrad;
  m->energies[2] = V;
  m->energies[3] = Etot;
  m->n_energies = 4;
  if (b->cfg.expansion) {
    s.potAvI = s.potAvSI = V;
    s.pi2AvI = s.pi2AvSI = v[0];
    s.grad2AvI = v[1];
    const double rho = (0.5 * s.pi2AvI * am6 + 0.5 * s.grad2AvI * am2) + s.potAvI;
    const double LHS = s.aDotI * s.aDotI;
    const double RHS = std::pow(s.aI, 2 * al + 2) / 3. * L.sp.fm2 * rho;
    m->friedmann[0] = (LHS - RHS) / (LHS + RHS);
    m->friedmann[1] = LHS;
    m->friedmann[2] = RHS;
    e = cudaMemcpy(b->d_st + i, &s, sizeof(s), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_measure");
  } else {
    m->friedmann[0] = std::fabs(1.0 - Etot / e0);
  }
  const double r1 = v[3] - v[2] * v[2], r2 = v[5] - v[4] * v[4];
  m->means[0][0] = v[2];
  m->means[0][1] = v[4];
  m->means[0][2] = v[3];
  m->means[0][3] = v[5];
  m->means[0][4] = r1 > 0 ? std::sqrt(r1) : 0;
  m->means[0][5] = r2 > 0 ? std::sqrt(r2) : 0;
  m->n_means = 1;
  m->aI = s.aI;
  m->aDotI = s.aDotI;
  m->hubble = s.aDotI / s.aI;
  return CLB_OK;
}


int clb_batch_autotune(clb_batch *b, int32_t reps, clb_batch_tuning *out)
{
  if (!b) return CLB_EINVAL;
  if (reps < 1 || reps > 1000) return b->fail(CLB_EINVAL, "clb_batch_autotune: reps in [1, 1000]");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_autotune");
  const int r = autotune(b, reps);
  if (r == CLB_OK && out) *out = b->tuning;
  return r;
}

int clb_batch_set_tuning(clb_batch *b, int32_t tile_z, int32_t tile_y, int32_t sites_per_thread, int32_t planes_x)
{
  if (!b) return CLB_EINVAL;
  int t = -1;
  for (int k = 0; k < kNTiles; ++k)
    if (kTiles[k].bz * kTiles[k].vz == tile_z && kTiles[k].by == tile_y && kTiles[k].vz == sites_per_thread) t = k;
  if (t < 0) return b->fail(CLB_EINVAL, "clb_batch_set_tuning: not a compiled tile (see clb_batch_tuning)");
  if (!tile_fits(b, t))
    return b->fail(CLB_EINVAL, "clb_batch_set_tuning: every member's N must be a multiple of sites_per_thread");
  if (planes_x < 1) return b->fail(CLB_EINVAL, "clb_batch_set_tuning: planes_x must be >= 1");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = layout(b, t, planes_x);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_set_tuning");
  drop_graphs(b);
  b->tuned = true;
  b->tuning = tuning_of(t, planes_x, 0, 0.0, 0.0);
  b->persist = false;
  return CLB_OK;
}

int clb_batch_set_persistent(clb_batch *b, int32_t tile_z, int32_t tile_y, int32_t sites_per_thread, int32_t planes_x)
{
  if (!b) return CLB_EINVAL;
  if (!persist_allowed(b)) return b->fail(CLB_EUNSUPPORTED, "clb_batch_set_persistent: too many stages per step");
  int t = -1;
  for (int k = 0; k < kNPersist; ++k)
    if (kPersist[k].bz * kPersist[k].vz == tile_z && kPersist[k].by == tile_y && kPersist[k].vz == sites_per_thread)
      t = k;
  if (t < 0) return b->fail(CLB_EINVAL, "clb_batch_set_persistent: not a compiled tile (see clb_batch_form)");
  if (!persist_fits(b, t))
    return b->fail(CLB_EINVAL, "clb_batch_set_persistent: every member's N must be a multiple of sites_per_thread");
  if (planes_x < 1) return b->fail(CLB_EINVAL, "clb_batch_set_persistent: planes_x must be >= 1");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = persist_layout(b, t, planes_x);
  if (e != cudaSuccess) return b->cuda_fail(e, "clb_batch_set_persistent");
  drop_graphs(b);
  if (!b->tuned) {
    b->tuned = true;
    b->tuning = tuning_of(b->tile, b->run, 0, 0.0, 0.0);
  }
  b->persist = true;
  return CLB_OK;
}

int clb_batch_get_form(clb_batch *b, clb_batch_form *out)
{
  if (!b || !out) return CLB_EINVAL;
  clb_batch_form f = b->form;
  f.persistent = b->persist ? 1 : 0;
  if (b->persist) {
    const TileShape sh = kPersist[b->ptile];
    f.tile_z = sh.bz * sh.vz;
    f.tile_y = sh.by;
    f.sites_per_thread = sh.vz;
    f.planes_x = b->prun;
    f.clusters = b->pclusters;
    f.cluster_blocks = kClusterCTAs;
  } else {
    f.tile_z = f.tile_y = f.sites_per_thread = f.planes_x = f.clusters = f.cluster_blocks = 0;
  }
  *out = f;
  return CLB_OK;
}

int clb_batch_get_tuning(clb_batch *b, clb_batch_tuning *out)
{
  if (!b || !out) return CLB_EINVAL;
  *out = b->tuned ? b->tuning : tuning_of(b->tile, b->run, 0, 0.0, 0.0);
  return CLB_OK;
}

} // extern "C"
