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

// Tuned configurations by ensemble (precision, device and sorted member sizes), for the process.
std::map<std::string, std::pair<int, int>> g_tuned;

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
#define CLB_BS(D, K, RD)                                                                                               \
  k_batch_sweep<BZ, BY, VZ, R, D, K, RD><<<grid, block, 0, b->stream>>>(fin, pin, fout, pout, b->d_lat, b->d_blk,    \
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
int autotune(clb_batch *b, int reps)
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
  g_tuned[tune_key(b)] = {bt, br};
  return CLB_OK;
}

void btail(clb_batch *b, uint32_t flags, bool reduced, double w = 0, double w2 = 0)
{
  TailOp op{flags, 0, w, w2, nullptr, -1};
  k_batch_tail<<<b->n, 256, 0, b->stream>>>(b->d_part, b->d_lat, b->d_st, op, reduced ? 1 : 0);
  ++b->launches;
}

// The fused VV schedule of EvolveVV (clb_api.cu) over all members.
void evolve_launches(clb_batch *b, int64_t nsteps)
{
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
                  (void *)b->d_stage})
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
  ok = ok && cudaMalloc(&b->d_sums, 8 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&b->d_stage, b->stage_n * sizeof(double)) == cudaSuccess;
  ok = ok && cudaEventCreate(&b->ev[0]) == cudaSuccess && cudaEventCreate(&b->ev[1]) == cudaSuccess;
  if (ok) {
    // a configuration tuned earlier in this process for the same ensemble, else the default
    auto it = g_tuned.find(tune_key(b));
    const bool cached = it != g_tuned.end();
    ok = layout(b, cached ? it->second.first : kDefaultTile, cached ? it->second.second : kDefaultRun) == cudaSuccess;
    if (cached) {
      b->tuned = true;
      b->tuning = tuning_of(b->tile, b->run, 0, 0.0, 0.0);
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
  return CLB_OK;
}

int clb_batch_get_tuning(clb_batch *b, clb_batch_tuning *out)
{
  if (!b || !out) return CLB_EINVAL;
  *out = b->tuned ? b->tuning : tuning_of(b->tile, b->run, 0, 0.0, 0.0);
  return CLB_OK;
}

} // extern "C"
