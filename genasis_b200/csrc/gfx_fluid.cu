// gfx_fluid.cu -- host side of the C ABI in include/gfx_fluid.h.
//
// One gfx_fluid handle = one single-brick chart with its Fluid_P_I current,
// the RK2 step and the integrator's time-step logic.  The handle owns the
// per-axis geometry tables, the stage scratch (primitives of the intermediate
// state Y and the partial solution U + K1/2, both without ghosts), the shock
// feature bits and a device-side clock for the evolve loop.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "adjoint_kernels.cuh"
#include "aux_kernels.cuh"
#include "chart_kernels.cuh"
#include "gfx_fluid.h"

using namespace gfx;

namespace {

thread_local std::string g_last_error;

// A named range of the calling thread for profilers (NVTX, header-only;
// without a tool attached a push is a call to a no-op).  The names are the
// reference's routines, so a profile of the library's launches reads by the
// reference's phases.
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(expr)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(GFX_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                  \
  } while (0)

// Per-axis geometry of the reference chart, Chart_Template.f90:478-560 (edges
// by repeated addition; the ghost widths pass through real(KDL), i.e. default
// single precision, as declared at :476-478), :827-841 (centres), :973-990
// (half widths); GeometryFlat_Kernel.f90:22-24 (widths); Difference_Kernel on
// the centres; the limiter's denominators of Gradient_Kernel.f90:176-180.
struct HostAxis {
  std::vector<double> X, WL, WR, W, dXI, SQ, CDEN, RDXI, RCDEN, RW;
  std::vector<double> PAR;  // PG_N tables of m + 1 (parabolic reconstruction)
};

HostAxis build_axis(int n, double mn, double mx, int g) {
  const int m = n + 2 * g;
  std::vector<double> edge(m + 1);
  double* E1 = edge.data() + g - 1;  // E1[i] = Edge(i), i in [1-g, n+g+1]
  const double width = (mx - mn) / (double)n;
  E1[1] = mn;
  for (int i = 2; i <= n + 1; ++i) E1[i] = E1[i - 1] + width;
  for (int iC = 1; iC <= g; ++iC) {
    const float w_ig = (float)(E1[iC + 1] - E1[iC]);
    const float w_og = (float)(E1[n - iC + 2] - E1[n - iC + 1]);
    E1[1 - iC] = E1[2 - iC] - (double)w_ig;
    E1[n + 1 + iC] = E1[n + iC] + (double)w_og;
  }
  HostAxis a;
  a.X.resize(m);
  a.WL.resize(m);
  a.WR.resize(m);
  a.W.resize(m);
  a.dXI.assign(m + 1, 0.0);
  a.SQ.assign(m + 1, 0.0);
  a.CDEN.assign(m + 1, 0.0);
  for (int t = 0; t < m; ++t) {
    const double c = 0.5 * (edge[t] + edge[t + 1]);
    a.X[t] = c;
    a.WL[t] = c - edge[t];
    a.WR[t] = edge[t + 1] - c;
    a.W[t] = a.WL[t] + a.WR[t];
  }
  for (int t = 1; t < m; ++t) {
    a.dXI[t] = a.X[t] - a.X[t - 1];
    a.SQ[t] = a.dXI[t] * a.dXI[t];
  }
  for (int t = 1; t + 1 < m; ++t)
    a.CDEN[t] = a.dXI[t] * a.dXI[t + 1] * (a.dXI[t] + a.dXI[t + 1]);
  // correctly rounded reciprocals for the exact divisions of the kernels
  a.RDXI.assign(m + 1, 0.0);
  a.RCDEN.assign(m + 1, 0.0);
  a.RW.assign(m + 1, 0.0);
  for (int t = 1; t < m; ++t) a.RDXI[t] = 1.0 / a.dXI[t];
  for (int t = 1; t + 1 < m; ++t) a.RCDEN[t] = 1.0 / a.CDEN[t];
  for (int t = 0; t < m; ++t) a.RW[t] = 1.0 / a.W[t];
  // PARABOLIC: centre, its square, inner and outer edges, and the geometry
  // denominators of IncrementDivergence_FV__Kernel.f90:382-575 for the cells
  // that have both neighbours, with their rounded reciprocals
  const int L = m + 1;
  a.PAR.assign((size_t)PG_N * L, 0.0);
  auto P = [&](int q, int t) -> double& { return a.PAR[(size_t)q * L + t]; };
  for (int t = 0; t < m; ++t) {
    P(PG_XC, t) = a.X[t];
    P(PG_X2, t) = a.X[t] * a.X[t];
    P(PG_XI, t) = a.X[t] - a.WL[t];
    P(PG_XO, t) = a.X[t] + a.WR[t];
  }
  for (int t = 1; t + 1 < m; ++t) {
    const double xAM = a.X[t - 1], xAC = a.X[t], xAP = a.X[t + 1];
    const double x2AM = xAM * xAM, x2AC = xAC * xAC, x2AP = xAP * xAP;
    const double xI = P(PG_XI, t), xO = P(PG_XO, t);
    const double D[6] = {
        (x2AM - x2AP) * xAC + (x2AP - x2AC) * xAM + (x2AC - x2AM) * xAP,
        (x2AC - x2AM) + 2.0 * (xAM - xAC) * xAM,
        (x2AC - x2AP) + 2.0 * (xAP - xAC) * xAP,
        (xI - xO) * (x2AC + xI * xO - xAC * (xI + xO)),
        (x2AC - xO * xO) + 2.0 * xI * (xO - xAC),
        (x2AC - xI * xI) + 2.0 * xO * (xI - xAC)};
    const int qd[6] = {PG_D1, PG_DA, PG_DB, PG_D3, PG_D4A, PG_D4B};
    for (int e = 0; e < 6; ++e) {
      P(qd[e], t) = D[e];
      P(qd[e] + 1, t) = 1.0 / D[e];
    }
  }
  return a;
}

enum FeatureState { FEAT_ZERO = 0, FEAT_VALID = 1, FEAT_PENDING = 2 };

// Launch attributes and the SM count belong to each device's context, so
// they are set up and cached per device (the current one at the call).
constexpr int kMaxDevices = 64;

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
  return dev;
}

int g_num_sms[kMaxDevices] = {};
std::once_flag g_sm_once[kMaxDevices];

int num_sms() {
  const int dev = current_device();
  if (dev < 0) return 148;
  std::call_once(g_sm_once[dev], [dev] {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_num_sms[dev] = n > 0 ? n : 148;
  });
  return g_num_sms[dev];
}

// gfx_fluid_debug_fail_allocation: the allocations of this thread still to
// pass before the one that fails (-1: none fails)
thread_local int g_fail_alloc = -1;

// cudaMalloc that leaves *p null when it fails (and clears the error it
// records), so that a handle whose lazy allocation failed allocates again on
// its next call instead of keeping a pointer it does not own.
template <class T>
bool dev_alloc(T** p, size_t bytes) {
  if (g_fail_alloc >= 0 && g_fail_alloc-- == 0) {
    *p = nullptr;
    return false;
  }
  if (cudaMalloc(p, bytes) == cudaSuccess) return true;
  *p = nullptr;
  cudaGetLastError();
  return false;
}

// The cycles of an evolve after its first, replayed from the cycle's graph
// in chunks of kChunkCycles with up to kChunksInFlight chunks ahead of the
// host.  After enqueuing chunk j the host waits for the clock copied after
// chunk j - (kChunksInFlight - 1), so the device keeps the chunks between
// queued: a host thread that is off its core for less than their device time
// (a CPU quota, a busy host) leaves no gap on the device.  The events block
// instead of spinning, leaving the host's cores to others while the host
// waits.  Chunks enqueued after the finish run as no-ops (the kernels test
// the clock's done flag).
constexpr int kChunksInFlight = 4;
constexpr int kChunkCycles = 8;

struct ChunkRing {
  Clock* host = nullptr;                  // [kChunksInFlight] pinned copies of the clock
  cudaEvent_t ev[kChunksInFlight] = {};   // after each copy
};

int ring_init(ChunkRing& R) {
  if (R.host) return GFX_OK;
  for (int j = 0; j < kChunksInFlight; ++j) {
    if (R.ev[j]) continue;
    const cudaError_t e =
        cudaEventCreateWithFlags(&R.ev[j], cudaEventDisableTiming | cudaEventBlockingSync);
    if (e != cudaSuccess) {
      R.ev[j] = nullptr;
      return fail(GFX_ERR_CUDA, "event of the evolve clock: %s", cudaGetErrorString(e));
    }
  }
  if (cudaMallocHost(&R.host, kChunksInFlight * sizeof(Clock)) != cudaSuccess) {
    R.host = nullptr;
    return fail(GFX_ERR_NO_MEMORY, "cudaMallocHost of the evolve clock");
  }
  return GFX_OK;
}

void ring_free(ChunkRing& R) {
  for (int j = 0; j < kChunksInFlight; ++j)
    if (R.ev[j]) cudaEventDestroy(R.ev[j]);
  if (R.host) cudaFreeHost(R.host);
  R = ChunkRing{};
}

// Replays `graph` on s from cycle done_cycles to n_cycles_max (the evolve's
// first cycle ran eagerly), reading the device clock dc between chunks, and
// adds the kernels it launches to *launches.
int ring_run(ChunkRing& R, cudaGraphExec_t graph, long long graph_kernels, long long* launches,
             const Clock* dc, int done_cycles, int n_cycles_max, cudaStream_t s) {
  long long j = 0;  // chunks enqueued
  while (done_cycles < n_cycles_max) {
    const int slot = (int)(j % kChunksInFlight);
    const int nrep = std::min(kChunkCycles, n_cycles_max - done_cycles);
    for (int r = 0; r < nrep; ++r) CUDA_TRY(cudaGraphLaunch(graph, s));
    *launches += (long long)nrep * graph_kernels;
    done_cycles += nrep;
    CUDA_TRY(cudaMemcpyAsync(R.host + slot, dc, sizeof(Clock), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaEventRecord(R.ev[slot], s));
    const long long w = j - (kChunksInFlight - 1);  // the chunk the host waits for
    ++j;
    if (w >= 0) {
      const int ws = (int)(w % kChunksInFlight);
      CUDA_TRY(cudaEventSynchronize(R.ev[ws]));
      if (R.host[ws].done) break;
    }
  }
  return GFX_OK;
}

}  // namespace

// z slabs of the pipelined gfx_fluid_step_host
constexpr int kMaxSlabs = 32;

struct gfx_fluid {
  gfx_fluid_config cfg;
  const gfx_fluid_chart* chart = nullptr;  // the chart this brick belongs to, if any
  Phys ph;
  Box box;
  HostAxis axis[3];
  double* geo = nullptr;  // device tables
  AxisGeo dgeo[3];
  double* Yp = nullptr;
  double* H = nullptr;
  double* Pst = nullptr;
  uint8_t* df = nullptr;
  unsigned long long* tsi_bits = nullptr;  // [1]
  int* counters = nullptr;                 // [4]
  Clock* clock = nullptr;                  // evolve clock
  ChunkRing ring;                          // the evolve's clock copies between chunks
  cudaEvent_t evolve_ev[2] = {};           // gfx_fluid_evolve_timed: around its work
  double* dt_slot = nullptr;               // dt of gfx_fluid_step
  WorkItem* items = nullptr;
  int n_items = 0;
  double* U_stage = nullptr;  // device copy for gfx_fluid_step_host
  cudaStream_t host_stream = nullptr;
  int features = FEAT_ZERO;
  const double* features_src = nullptr;
  bool prims_pending = false;
  size_t face_size = 0;
  // evolve graph cache
  cudaGraphExec_t graph = nullptr;
  double* graph_U = nullptr;
  long long graph_kernels = 0;  // kernel nodes per replay
  long long launches = 0;       // kernels launched so far
  // adjoint workspace (allocated by the first gfx_fluid_step_adjoint):
  // W0, lamZ, lamW, lamK1 (compact, 5 fields each), flags of U^n, and a
  // recomputed U^n+1 when the caller passes none
  double* adj = nullptr;
  uint8_t* adj_flags = nullptr;
  unsigned long long* branch_buf = nullptr;  // gfx_fluid_step_branches: [2 + kinds]
  double* adj_U = nullptr;
  // tuning (gfx_fluid_set_tuning; 0 = built-in default)
  int z_chunk = 0;
  int adjoint_segment = 0;
  int tile_y = kTileY;  // tile rows of the work list (8 or 16)
  unsigned long long* state_counts = nullptr;  // [2] for gfx_fluid_check_state
  double* partials = nullptr;                  // per-block sums of gfx_fluid_totals
  double* Ksrc = nullptr;  // [6][nV]: a stage's divergence for gfx_fluid_step_sources
  double* wn = nullptr;  // [5][nP]: the primitives of the state the last stage 2 wrote
  const double* wn_of = nullptr;  // that state (null when unknown or since rewritten)
  // pipelined gfx_fluid_step_host: copy streams, per-slab events and counters
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_in[kMaxSlabs] = {}, ev_out[kMaxSlabs] = {}, ev_end = nullptr;
  int* slab_counters = nullptr;  // [2 * kMaxSlabs]
  WorkItem* host_items = nullptr;  // the work list of the slabs, z chunks of host_chunk
  int host_n_items = 0, host_chunk = 0, host_tile_y = 0;
};

namespace {

template <int MODE, bool IN_PRIM, bool HLLC, bool GRAV, int NF, int BAT,
          bool PARAB = false, int TYt = kTileY>
cudaError_t launch_stage_t(const BrickDesc& d, const BrickDesc* many, const WorkItem* items,
                           int n_items, int* counter, const Phys& ph, cudaStream_t s) {
  using SM = StageLayout<NF, TYt, PARAB>;
  // the shared-memory attribute and the occupancy, once per device
  static std::once_flag once[kMaxDevices];
  static cudaError_t attr_err[kMaxDevices];
  static int per_sm[kMaxDevices];
  auto kern = stage_kernel<MODE, IN_PRIM, HLLC, GRAV, NF, BAT, PARAB, TYt>;
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  std::call_once(once[dev], [&] {
    int n = 1;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)SM::kBytes);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, SM::NT, SM::kBytes);
    attr_err[dev] = e;
    per_sm[dev] = n < 1 ? 1 : n;
  });
  if (attr_err[dev] != cudaSuccess) return attr_err[dev];
  // persistent grid: every resident CTA slot pulls work items
  const int grid = std::max(1, std::min(n_items, num_sms() * per_sm[dev]));
  kern<<<grid, SM::NT, SM::kBytes, s>>>(d, many, items, n_items, counter, ph);
  return cudaGetLastError();
}

// The PARABOLIC variants (single bricks only).
cudaError_t launch_stage_parabolic(int mode, bool in_prim, bool hllc, bool grav,
                                   const BrickDesc& d, const WorkItem* items, int n_items,
                                   int* counter, const Phys& ph, cudaStream_t s) {
#define GFX_PSTAGE(M, IP, HC, GR, NF)                                                     \
  if (mode == M && in_prim == IP && hllc == HC && grav == GR)                            \
    return launch_stage_t<M, IP, HC, GR, NF, BAT_SINGLE, true>(d, nullptr, items, n_items, \
                                                               counter, ph, s);
  GFX_PSTAGE(MODE_INCREMENT, false, false, false, 6)
  GFX_PSTAGE(MODE_INCREMENT, false, true, false, 6)
  GFX_PSTAGE(MODE_INCREMENT, true, false, false, 6)
  GFX_PSTAGE(MODE_INCREMENT, true, true, false, 6)
  GFX_PSTAGE(MODE_STAGE1, false, false, false, 5)
  GFX_PSTAGE(MODE_STAGE1, false, true, false, 5)
  GFX_PSTAGE(MODE_STAGE1, false, false, true, 5)
  GFX_PSTAGE(MODE_STAGE1, false, true, true, 5)
  GFX_PSTAGE(MODE_STAGE1, true, false, false, 5)
  GFX_PSTAGE(MODE_STAGE1, true, true, false, 5)
  GFX_PSTAGE(MODE_STAGE1, true, false, true, 5)
  GFX_PSTAGE(MODE_STAGE1, true, true, true, 5)
  GFX_PSTAGE(MODE_STAGE2, true, false, false, 5)
  GFX_PSTAGE(MODE_STAGE2, true, true, false, 5)
  GFX_PSTAGE(MODE_STAGE2, true, false, true, 5)
  GFX_PSTAGE(MODE_STAGE2, true, true, true, 5)
#undef GFX_PSTAGE
  return cudaErrorInvalidValue;
}

// The LINEAR variants for tile height TYt.  bat: BAT_SINGLE (d describes
// the brick), BAT_BRICKS or BAT_CHART (many holds a descriptor per brick).
template <int TYt>
cudaError_t launch_stage_linear(int mode, bool in_prim, bool hllc, bool grav, int bat,
                                const BrickDesc& d, const BrickDesc* many,
                                const WorkItem* items, int n_items, int* counter,
                                const Phys& ph, cudaStream_t s) {
#define GFX_STAGE(M, IP, HC, GR, NF, BA)                                                  \
  if (mode == M && in_prim == IP && hllc == HC && grav == GR && bat == BA)              \
    return launch_stage_t<M, IP, HC, GR, NF, BA, false, TYt>(d, many, items, n_items,     \
                                                             counter, ph, s);
#define GFX_STAGE_B(M, IP, HC, GR, NF)  \
  GFX_STAGE(M, IP, HC, GR, NF, BAT_SINGLE) \
  GFX_STAGE(M, IP, HC, GR, NF, BAT_BRICKS)
  GFX_STAGE(MODE_INCREMENT, false, false, false, 6, BAT_SINGLE)
  GFX_STAGE(MODE_INCREMENT, false, true, false, 6, BAT_SINGLE)
  GFX_STAGE(MODE_INCREMENT, true, false, false, 6, BAT_SINGLE)
  GFX_STAGE(MODE_INCREMENT, true, true, false, 6, BAT_SINGLE)
  GFX_STAGE_B(MODE_STAGE1, false, false, false, 5)
  GFX_STAGE_B(MODE_STAGE1, false, true, false, 5)
  GFX_STAGE(MODE_STAGE1, false, false, true, 5, BAT_SINGLE)
  GFX_STAGE(MODE_STAGE1, false, true, true, 5, BAT_SINGLE)
  GFX_STAGE_B(MODE_STAGE1, true, false, false, 5)
  GFX_STAGE_B(MODE_STAGE1, true, true, false, 5)
  GFX_STAGE(MODE_STAGE1, true, false, true, 5, BAT_SINGLE)
  GFX_STAGE(MODE_STAGE1, true, true, true, 5, BAT_SINGLE)
  GFX_STAGE_B(MODE_STAGE2, true, false, false, 5)
  GFX_STAGE_B(MODE_STAGE2, true, true, false, 5)
  GFX_STAGE(MODE_STAGE2, true, false, true, 5, BAT_SINGLE)
  GFX_STAGE(MODE_STAGE2, true, true, true, 5, BAT_SINGLE)
#undef GFX_STAGE_B
#undef GFX_STAGE
  return cudaErrorInvalidValue;
}

// The chart variants (16-row tiles): stage 1 from conserved values or kept
// primitives, stage 2, with or without HLLC and gravity.
// Tile rows of a chart's work items: the height each build's autotuned
// single bricks choose (8-row tiles, two CTAs per SM, in the fast build)
#if GFX_FAST_MATH
constexpr int kChartTileY = 8;
#else
constexpr int kChartTileY = kTileY;
#endif

cudaError_t launch_stage_chart(int mode, bool in_prim, bool hllc, bool grav,
                               const BrickDesc* many, const WorkItem* items, int n_items,
                               int* counter, const Phys& ph, cudaStream_t s) {
  BrickDesc none;
  memset(&none, 0, sizeof(none));
#define GFX_CSTAGE(M, IP, HC, GR)                                                          \
  if (mode == M && in_prim == IP && hllc == HC && grav == GR)                            \
    return launch_stage_t<M, IP, HC, GR, 5, BAT_CHART, false, kChartTileY>(               \
        none, many, items, n_items, counter, ph, s);
  GFX_CSTAGE(MODE_STAGE1, false, false, false)
  GFX_CSTAGE(MODE_STAGE1, false, true, false)
  GFX_CSTAGE(MODE_STAGE1, false, false, true)
  GFX_CSTAGE(MODE_STAGE1, false, true, true)
  GFX_CSTAGE(MODE_STAGE1, true, false, false)
  GFX_CSTAGE(MODE_STAGE1, true, true, false)
  GFX_CSTAGE(MODE_STAGE1, true, false, true)
  GFX_CSTAGE(MODE_STAGE1, true, true, true)
  GFX_CSTAGE(MODE_STAGE2, true, false, false)
  GFX_CSTAGE(MODE_STAGE2, true, true, false)
  GFX_CSTAGE(MODE_STAGE2, true, false, true)
  GFX_CSTAGE(MODE_STAGE2, true, true, true)
#undef GFX_CSTAGE
  return cudaErrorInvalidValue;
}

// The stage launch of a brick (or, with many, of a batch): PARABOLIC single
// bricks at the default tile height, LINEAR at the tile height of the work
// list (d.tile_y).
cudaError_t launch_stage(int mode, bool in_prim, bool hllc, bool grav, const BrickDesc& d,
                         const BrickDesc* many, const WorkItem* items, int n_items,
                         int* counter, const Phys& ph, cudaStream_t s) {
  const bool bat = many != nullptr;
  const int ty = d.tile_y ? d.tile_y : kTileY;
  if (!bat && d.geo[0].PAR != nullptr && ph.parabolic)
    return ty == kTileY ? launch_stage_parabolic(mode, in_prim, hllc, grav, d, items, n_items,
                                                 counter, ph, s)
                        : cudaErrorInvalidValue;
  const int bat_kind = bat ? BAT_BRICKS : BAT_SINGLE;
  if (ty == 8)
    return launch_stage_linear<8>(mode, in_prim, hllc, grav, bat_kind, d, many, items, n_items,
                                  counter, ph, s);
  if (ty == kTileY)
    return launch_stage_linear<kTileY>(mode, in_prim, hllc, grav, bat_kind, d, many, items,
                                       n_items, counter, ph, s);
  return cudaErrorInvalidValue;
}

int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  const long long cap = (long long)num_sms() * 16;
  return (int)std::max(1LL, std::min(g, cap));
}

int validate(const gfx_fluid_config* c) {
  if (!c) return fail(GFX_ERR_ARGUMENT, "config is NULL");
  for (int d = 0; d < 3; ++d) {
    if (c->n_cells[d] < 4)
      return fail(GFX_ERR_ARGUMENT, "n_cells[%d] = %d: need at least 4 proper cells", d,
                  c->n_cells[d]);
    if (!(c->max_coordinate[d] > c->min_coordinate[d]))
      return fail(GFX_ERR_ARGUMENT, "max_coordinate[%d] must exceed min_coordinate[%d]", d, d);
    // the exact divisions by geometry values assume widths in [2^-98, 2^98]
    const double w = (c->max_coordinate[d] - c->min_coordinate[d]) / c->n_cells[d];
    if (!(w >= 0x1p-98 && w <= 0x1p98))
      return fail(GFX_ERR_UNSUPPORTED, "axis %d: cell width %g outside [2^-98, 2^98]", d, w);
    for (int s = 0; s < 2; ++s)
      if (c->boundary[d][s] < GFX_BC_OUTFLOW || c->boundary[d][s] > GFX_BC_PERIODIC)
        return fail(GFX_ERR_ARGUMENT, "boundary[%d][%d] = %d is not a boundary condition", d,
                    s, c->boundary[d][s]);
    if ((c->boundary[d][0] == GFX_BC_PERIODIC) != (c->boundary[d][1] == GFX_BC_PERIODIC))
      return fail(GFX_ERR_ARGUMENT, "axis %d: PERIODIC must be set on both faces", d);
  }
  if ((long long)(c->n_cells[0] + 4) * (c->n_cells[1] + 4) * (c->n_cells[2] + 4) >= (1LL << 31))
    return fail(GFX_ERR_UNSUPPORTED, "a brick of 2^31 or more values (with ghosts)");
  if (c->n_ghost_layers != 2)
    return fail(GFX_ERR_UNSUPPORTED, "n_ghost_layers = %d: only 2 (the reference default)",
                c->n_ghost_layers);
  if (c->riemann_solver != GFX_RIEMANN_HLL && c->riemann_solver != GFX_RIEMANN_HLLC)
    return fail(GFX_ERR_ARGUMENT, "riemann_solver = %d", c->riemann_solver);
  if (!(c->adiabatic_index > 1.0)) return fail(GFX_ERR_ARGUMENT, "adiabatic_index must be > 1");
  if (c->n_ramp_cycles < 1) return fail(GFX_ERR_ARGUMENT, "n_ramp_cycles must be >= 1");
  if (c->reconstruction != GFX_RECONSTRUCTION_LINEAR &&
      c->reconstruction != GFX_RECONSTRUCTION_PARABOLIC)
    return fail(GFX_ERR_ARGUMENT, "reconstruction = %d", c->reconstruction);
#if GFX_FAST_MATH
  // the parabola's extremum tests switch its face values on quantities that
  // a unit in the last place moves; only the exact build reproduces them
  if (c->reconstruction == GFX_RECONSTRUCTION_PARABOLIC)
    return fail(GFX_ERR_UNSUPPORTED,
                "PARABOLIC reconstruction: the exact build (libgfx_fluid.so) only");
#endif
  if (!(c->courant_factor > 0.0)) return fail(GFX_ERR_ARGUMENT, "courant_factor must be > 0");
  return GFX_OK;
}

// The step entry points of a single brick apply its boundary conditions on
// every face; a brick of a chart has faces whose ghosts live in its
// neighbours, so those calls go through the chart.
int refuse_chart_brick(const gfx_fluid* h, const char* fn) {
  if (h && h->chart)
    return fail(GFX_ERR_ARGUMENT, "%s: a brick of a chart steps through gfx_fluid_chart_*", fn);
  return GFX_OK;
}

// Work list of one brick: TX x ty columns, cut along z into chunks so that the
// persistent grid has several items per SM.
// z_chunk > 0 fixes the pencil length instead (the autotuner's knob).
std::vector<WorkItem> make_items(const int n[3], int brick, int z_chunk = 0,
                                 int ty = kTileY) {
  const int cx = (n[0] + TX - 1) / TX, cy = (n[1] + ty - 1) / ty;
  const long long cols = (long long)cx * cy;
  const long long want = 16LL * num_sms();
  int chunks = (int)std::max(1LL, std::min<long long>(n[2] / 16, (want + cols - 1) / cols));
  if (chunks < 1) chunks = 1;
  int len = (n[2] + chunks - 1) / chunks;
  if (z_chunk > 0) len = std::min(n[2], z_chunk);
  std::vector<WorkItem> v;
  for (int z = 0; z < n[2]; z += len)
    for (int y = 0; y < cy; ++y)
      for (int x = 0; x < cx; ++x) v.push_back({brick, x * TX, y * ty, z, std::min(n[2], z + len)});
  return v;
}

BrickDesc make_desc(gfx_fluid* h, const double* U_in, double* U_out, double* K,
                    const double* P_in, const uint8_t* df, double* fluence,
                    const double* dt_ptr, double weight, const int* skip) {
  BrickDesc d;
  memset(&d, 0, sizeof(d));
  for (int a = 0; a < 3; ++a) {
    d.nb[a][0] = d.nb[a][1] = -1;
    d.n[a] = h->box.n[a];
    d.m[a] = h->box.m[a];
    d.bc[a][0] = h->box.bc[a][0];
    d.bc[a][1] = h->box.bc[a][1];
    d.geo[a] = h->dgeo[a];
  }
  d.nV = h->box.nV;
  d.nP = h->box.nP;
  d.U_in = U_in;
  d.U_out = U_out;
  d.K = K;
  d.P_in = P_in;
  d.Yp = h->Yp;
  d.H = h->H;
  d.df = df;
  d.fluence = fluence;
  d.face_size = (long long)h->face_size;
  d.dt = dt_ptr;
  d.weight = weight;
  d.tsi_bits = h->tsi_bits;
  d.skip = skip;
  d.tile_y = h->tile_y;
  return d;
}

__global__ void set_scalar_kernel(double* p, double v) { *p = v; }

// Compact proper-cell flag bytes into the ghost layout (ghosts get 0).
__global__ void scatter_flags_kernel(Box b, const uint8_t* __restrict__ df,
                                     uint8_t* __restrict__ out) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < b.nV;
       v += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(v, b.m[0], b.m[1], i, j, k);
    i -= 2;
    j -= 2;
    k -= 2;
    uint8_t f = 0;
    if (i >= 0 && j >= 0 && k >= 0 && i < b.n[0] && j < b.n[1] && k < b.n[2])
      f = df[i + (long long)b.n[0] * (j + (long long)b.n[1] * k)];
    out[v] = f;
  }
}

// DIFFUSIVE_FLUX_I flags of the planes [k0, k1), from U or from the compact
// primitives Pst when given (reads the state of planes k0 - 1 to k1).
cudaError_t launch_features(const Box& b, const Phys& ph, const double* U, const double* Pst,
                            uint8_t* df, int k0, int k1, cudaStream_t s) {
  if (k1 <= k0) return cudaSuccess;
  if (Pst)
    detect_features_kernel<true>
        <<<detect_grid(b, k0, k1), kDetThreads, 0, s>>>(b, ph, U, Pst, df, k0, k1);
  else
    detect_features_kernel<false>
        <<<detect_grid(b, k0, k1), kDetThreads, 0, s>>>(b, ph, U, Pst, df, k0, k1);
  return cudaGetLastError();
}

int run_features(gfx_fluid* h, const double* U, const double* Pst, cudaStream_t s) {
  CUDA_TRY(launch_features(h->box, h->ph, U, Pst, h->df, 0, h->box.n[2], s));
  h->launches += 1;
  return GFX_OK;
}

// Shock flags of the state the previous step's stage 2 wrote, from the
// primitives it stored (valid only between the steps of one evolve, where
// nothing else touches the state; the same values the recovery from the
// stored, floored state gives).
int run_features_wn(gfx_fluid* h, const double* U, cudaStream_t s) {
  return run_features(h, U, h->wn, s);
}

// The Sources records of RK2 stage `stage` (0, 1) into S [10][nV]: the
// stage's divergence increment once more, from the input the fused stage
// reads (U, or the compact primitives P when in_prim), by the increment
// kernel into the scratch Ksrc (the same arithmetic, so the same K as the
// stage's before its gravity term), then the records.  counter: a work
// counter zeroed for this launch.
int enqueue_sources(gfx_fluid* h, const double* U, const double* P, bool in_prim,
                    const uint8_t* df, const double* dt_ptr, int stage, double* S, int* counter,
                    cudaStream_t s) {
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  const size_t bytes = 6 * (size_t)h->box.nV * sizeof(double);
  CUDA_TRY(cudaMemsetAsync(h->Ksrc, 0, bytes, s));
  BrickDesc d = make_desc(h, U, nullptr, h->Ksrc, in_prim ? P : nullptr, df, nullptr, dt_ptr,
                          0.5, nullptr);
  CUDA_TRY(launch_stage(MODE_INCREMENT, in_prim, hllc, false, d, nullptr, h->items, h->n_items,
                        counter, h->ph, s));
  const int blk = 256;
  if (stage == 0)
    record_sources_kernel<true><<<grid_for(h->box.nV, blk), blk, 0, s>>>(
        h->box, h->ph, h->Ksrc, dt_ptr, 0.5, U, in_prim ? P : nullptr, S);
  else
    record_sources_kernel<false><<<grid_for(h->box.nV, blk), blk, 0, s>>>(
        h->box, h->ph, h->Ksrc, dt_ptr, 0.5, U, in_prim ? P : nullptr, S);
  CUDA_TRY(cudaGetLastError());
  h->launches += 2;
  return GFX_OK;
}

// The launches of one RK2 step on U (in place).  dt_ptr, skip: device scalars.
// detect: whether the shock flags must be recomputed from U first.  ev (may
// be null): 5 events recorded between the phases for gfx_fluid_step_timed.
// from_wn: the step follows a step of the same evolve, whose stage 2 stored
// the primitives of U: shock detection and stage 1 read them instead of
// recovering them from U.  sources (may be null): [10][nV], the step's
// Sources records (gfx_fluid_step_sources; needs h->Ksrc).
int enqueue_step(gfx_fluid* h, double* U, const double* dt_ptr, const int* skip,
                 double* fluence, bool detect, cudaStream_t s, cudaEvent_t* ev = nullptr,
                 bool from_wn = false, double* sources = nullptr) {
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  const bool grav = h->cfg.uniform_acceleration != 0.0;
  reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 4);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  if (fluence)
    CUDA_TRY(cudaMemsetAsync(fluence, 0, sizeof(double) * 36 * h->face_size, s));
  if (ev) CUDA_TRY(cudaEventRecord(ev[0], s));
  if (hllc && detect) {
    Range r("FluidFeatures_P % Detect");
    int rc = from_wn ? run_features_wn(h, U, s) : run_features(h, U, nullptr, s);
    if (rc) return rc;
  }
  if (ev) CUDA_TRY(cudaEventRecord(ev[1], s));
  const uint8_t* df = hllc ? h->df : nullptr;
  const bool in_prim = from_wn || h->prims_pending;
  const double* P1 = from_wn ? h->wn : (h->prims_pending ? h->Pst : nullptr);
  if (sources) {
    int rc = enqueue_sources(h, U, P1, in_prim, df, dt_ptr, 0, sources, h->counters + 2, s);
    if (rc) return rc;
  }
  BrickDesc d1 = make_desc(h, U, nullptr, nullptr, P1, df, fluence, dt_ptr, 0.5, skip);
  {
    Range r("Step_RK_C_ASC % ComputeStage 1");
    CUDA_TRY(launch_stage(MODE_STAGE1, in_prim, hllc, grav, d1, nullptr, h->items, h->n_items,
                          h->counters, h->ph, s));
  }
  if (ev) CUDA_TRY(cudaEventRecord(ev[2], s));
  if (sources) {
    int rc = enqueue_sources(h, U, h->Yp, true, df, dt_ptr, 1, sources, h->counters + 3, s);
    if (rc) return rc;
  }
  BrickDesc d2 = make_desc(h, U, U, nullptr, h->Yp, df, fluence, dt_ptr, 0.5, skip);
  d2.wn = h->wn;
  {
    Range r("Step_RK_C_ASC % ComputeStage 2");
    CUDA_TRY(launch_stage(MODE_STAGE2, true, hllc, grav, d2, nullptr, h->items, h->n_items,
                          h->counters + 1, h->ph, s));
  }
  if (ev) CUDA_TRY(cudaEventRecord(ev[3], s));
  const int blk = 256;
  const Box& bx = h->box;
  const long long shell = bx.nV - bx.nP;
  ghost_refresh_shell_kernel<<<grid_for(shell, blk), blk, 0, s>>>(bx, h->ph, U);
  CUDA_TRY(cudaGetLastError());
  if (ev) CUDA_TRY(cudaEventRecord(ev[4], s));
  h->launches += 3;
  return GFX_OK;
}

}  // namespace

struct gfx_fluid_batch {
  int n = 0;
  std::vector<gfx_fluid*> h;
  std::vector<double*> U;
  Phys ph;
  bool hllc = false, grav = false;
  BrickDesc* d1 = nullptr;   // stage 1 from conserved input, per brick
  BrickDesc* d1p = nullptr;  // stage 1 from kept primitives, per brick
  BrickDesc* d1w = nullptr;  // stage 1 from the primitives the last stage 2 stored
  BrickDesc* d2 = nullptr;   // stage 2, per brick
  WorkItem* items = nullptr;
  int n_items = 0;
  DetItem* det_items = nullptr;  // tiles of the features (HLLC)
  int n_det_items = 0;
  BatchBrick* bb = nullptr;
  long long total_v = 0, total_c = 0;
  unsigned long long* tsi_bits = nullptr;  // [n]
  Clock* clocks = nullptr;                 // [n]
  int* counters = nullptr;                 // [4]
  cudaGraphExec_t graph = nullptr;
  long long graph_kernels = 0;
  long long launches = 0;
  int tile_y = kTileY;
};

namespace {

// The launches of one batched cycle: shock flags (HLLC), the two stages for
// every brick, ghosts, then each brick's clock and next time step.  d1: the
// stage-1 descriptors (input from primitives when in_prim).
int enqueue_batch_cycle(gfx_fluid_batch* B, bool detect, const BrickDesc* d1, bool in_prim,
                        cudaStream_t s) {
  const int blk = 256;
  reset_bits_kernel<<<grid_for(std::max(B->n, 4), blk), blk, 0, s>>>(B->tsi_bits, B->n,
                                                                      B->counters, 4);
  CUDA_TRY(cudaGetLastError());
  B->launches += 1;
  if (B->hllc && detect) {
    batch_detect_features_kernel<<<B->n_det_items, kDetThreads, 0, s>>>(B->bb, B->det_items,
                                                                        B->ph);
    CUDA_TRY(cudaGetLastError());
    B->launches += 1;
  }
  BrickDesc none;
  memset(&none, 0, sizeof(none));
  none.tile_y = B->tile_y;
  CUDA_TRY(launch_stage(MODE_STAGE1, in_prim, B->hllc, false, none, d1, B->items, B->n_items,
                        B->counters, B->ph, s));
  CUDA_TRY(launch_stage(MODE_STAGE2, true, B->hllc, false, none, B->d2, B->items, B->n_items,
                        B->counters + 1, B->ph, s));
  const long long shells = B->total_v - B->total_c;
  batch_ghost_refresh_kernel<<<grid_for(shells, blk), blk, 0, s>>>(B->bb, B->n, shells,
                                                                   B->ph);
  advance_clock_kernel<<<grid_for(B->n, blk), blk, 0, s>>>(B->clocks, B->n);
  finalize_dt_kernel<<<grid_for(B->n, blk), blk, 0, s>>>(B->ph, B->tsi_bits, B->clocks, B->n, 1);
  CUDA_TRY(cudaGetLastError());
  B->launches += 5;
  return GFX_OK;
}

}  // namespace

namespace {

// gfx_fluid_step with U in host memory, pipelined over z slabs (whole
// z chunks of the work list) on three streams: the copy of the inputs (the
// five fields D, S1, S2, S3, G of every plane: DS is rewritten by the step and
// never read), the compute, and the copy of the result (all six fields).
// Shock detection and stage 1 of a slab start as soon as its planes and the
// two above it have arrived; stage 2 of a slab as soon as stage 1 of the slab
// above it is done, and every slab is copied back as soon as its stage 2 and
// the x / y ghosts of its planes are done, so that the copies back overlap
// the copies in of later slabs; the z ghost planes, which reach across the
// brick, come last.  The
// launches and their inputs are those of gfx_fluid_step, so the result is
// the same bit for bit.  Returns GFX_ERR_UNSUPPORTED when the work list is too
// short to pipeline (the caller then takes the unpipelined path).
int step_host_pipelined(gfx_fluid* h, double* U_host, double dt, double* fluence_host) {
  const Box& b = h->box;
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  if (h->prims_pending) return GFX_ERR_UNSUPPORTED;
  // the slabs' own work list, cut along z into chunks of at least 2 planes:
  // kThin chunks of half length first (the copies back begin once the first
  // slabs are computed, so these arrive and finish early), then chunks of
  // the tuned length, shortened so that the brick has up to kMaxSlabs slabs
  constexpr int kThin = 4;
  const int n2 = b.n[2];
  const WorkItem first = make_items(b.n, 0, h->z_chunk, h->tile_y)[0];
  const int len0 = first.z1 - first.z0;
  const int len = std::min(len0, std::max(2, (n2 + kMaxSlabs - 1) / kMaxSlabs));
  const int thin = std::max(2, len / 2);
  const int n_thin = (n2 >= kThin * thin + 2 * len) ? kThin : 0;
  std::vector<int> cz(1, 0);
  for (int c = 0; c < n_thin; ++c) cz.push_back(cz.back() + thin);
  {
    const int rest = n2 - cz.back();
    int l = len;
    while (rest % l == 1 && l < rest) ++l;  // no one-plane chunk at the end
    for (int z = cz.back() + l; z < n2; z += l) cz.push_back(z);
    cz.push_back(n2);
  }
  const int nchunks = (int)cz.size() - 1;
  if (nchunks < 2 || cz[nchunks] - cz[nchunks - 1] < 2) return GFX_ERR_UNSUPPORTED;
  const int ty = h->tile_y;
  const int cx = (b.n[0] + TX - 1) / TX, cy = (b.n[1] + ty - 1) / ty, cols = cx * cy;
  if (h->host_chunk != len || h->host_tile_y != ty) {
    std::vector<WorkItem> items;
    for (int c = 0; c < nchunks; ++c)
      for (int y = 0; y < cy; ++y)
        for (int x = 0; x < cx; ++x) items.push_back({0, x * TX, y * ty, cz[c], cz[c + 1]});
    cudaFree(h->host_items);
    h->host_items = nullptr;
    h->host_chunk = 0;
    if (!dev_alloc(&h->host_items, items.size() * sizeof(WorkItem)))
      return fail(GFX_ERR_NO_MEMORY, "cudaMalloc slab work items");
    CUDA_TRY(cudaMemcpy(h->host_items, items.data(), items.size() * sizeof(WorkItem),
                        cudaMemcpyHostToDevice));
    h->host_n_items = (int)items.size();
    h->host_chunk = len;
    h->host_tile_y = ty;
  }
  // slabs: the thin chunks one by one, the others in even groups
  const int S = std::min(kMaxSlabs, nchunks);
  const int S_thin = std::min(n_thin, S - 1);
  int it[kMaxSlabs + 1], zs[kMaxSlabs + 1];
  for (int j = 0; j <= S; ++j) {
    const int c = (j <= S_thin) ? j
                                : S_thin + (int)((long long)(j - S_thin) * (nchunks - S_thin) /
                                                 (S - S_thin));
    it[j] = c * cols;
    zs[j] = cz[c];
  }
  if (!h->copy_in) CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_in, cudaStreamNonBlocking));
  if (!h->copy_out) CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_out, cudaStreamNonBlocking));
  for (int j = 0; j < kMaxSlabs; ++j) {
    if (!h->ev_in[j]) CUDA_TRY(cudaEventCreateWithFlags(&h->ev_in[j], cudaEventDisableTiming));
    if (!h->ev_out[j]) CUDA_TRY(cudaEventCreateWithFlags(&h->ev_out[j], cudaEventDisableTiming));
  }
  if (!h->ev_end) CUDA_TRY(cudaEventCreateWithFlags(&h->ev_end, cudaEventDisableTiming));
  if (!h->slab_counters && !dev_alloc(&h->slab_counters, 2 * kMaxSlabs * sizeof(int)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc slab counters");
  cudaStream_t sc = h->host_stream, si = h->copy_in, so = h->copy_out;
  double* U = h->U_stage;
  const size_t nV = (size_t)b.nV, plane = (size_t)b.m[0] * b.m[1];
  // planes [p0, p1) of the first nf fields: one 2-D copy whose rows are the
  // fields (pitch nV values on both sides), so that a slab is one transfer
  auto copy = [&](cudaStream_t st, int nf, int p0, int p1, cudaMemcpyKind kind) -> cudaError_t {
    if (p1 <= p0) return cudaSuccess;
    const size_t off = (size_t)p0 * plane;
    double* dst = (kind == cudaMemcpyHostToDevice) ? U + off : U_host + off;
    const double* src = (kind == cudaMemcpyHostToDevice) ? U_host + off : U + off;
    return cudaMemcpy2DAsync(dst, nV * sizeof(double), src, nV * sizeof(double),
                             (size_t)(p1 - p0) * plane * sizeof(double), nf, kind, st);
  };
  // inputs: the top planes first (a periodic z axis reads them from slab 0),
  // then the slabs; plane index P = z + 2 of the ghost layout
  CUDA_TRY(copy(si, 5, n2, n2 + 4, cudaMemcpyHostToDevice));
  for (int j = 0; j < S; ++j) {
    const int p0 = (j == 0) ? 0 : zs[j] + 2, p1 = std::min(zs[j + 1] + 2, n2);
    CUDA_TRY(copy(si, 5, p0, p1, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaEventRecord(h->ev_in[j], si));
  }
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  const bool grav = h->cfg.uniform_acceleration != 0.0;
  const bool detect = hllc && h->features == FEAT_PENDING;
  const int blk = 256;
  double* fl = fluence_host ? U + 6 * nV : nullptr;
  reset_bits_kernel<<<1, 32, 0, sc>>>(h->tsi_bits, 1, h->slab_counters, 2 * S);
  set_scalar_kernel<<<1, 1, 0, sc>>>(h->dt_slot, dt);
  CUDA_TRY(cudaGetLastError());
  if (fl) CUDA_TRY(cudaMemsetAsync(fl, 0, sizeof(double) * 36 * h->face_size, sc));
  long long launches = 2;
  const uint8_t* df = hllc ? h->df : nullptr;
  BrickDesc d1 = make_desc(h, U, nullptr, nullptr, nullptr, df, fl, h->dt_slot, 0.5, nullptr);
  BrickDesc d2 = make_desc(h, U, U, nullptr, h->Yp, df, fl, h->dt_slot, 0.5, nullptr);
  d2.wn = h->wn;
  auto stage = [&](int mode, int j) -> cudaError_t {
    ++launches;
    return launch_stage(mode, mode == MODE_STAGE2, hllc, grav, mode == MODE_STAGE1 ? d1 : d2,
                        nullptr, h->host_items + it[j], it[j + 1] - it[j],
                        h->slab_counters + (mode == MODE_STAGE1 ? 0 : S) + j, h->ph, sc);
  };
  // the flags of planes [g(j), g(j+1)) with g(j) = zs[j] + 1 inside the
  // brick: those of slab j shifted up one plane, so that they include the
  // first plane of slab j+1 (whose flags stage 1 of slab j reads) and need the
  // state up to the second plane of slab j+1 only
  auto g = [&](int j) { return (j == 0) ? 0 : (j == S) ? n2 : zs[j] + 1; };
  auto flags = [&](int j) -> cudaError_t {
    ++launches;
    return launch_features(b, h->ph, U, nullptr, h->df, g(j), g(j + 1), sc);
  };
  // stage 2 of slab j, the x / y ghosts of its planes, then its copy back
  auto finish = [&](int j) -> cudaError_t {
    cudaError_t e = stage(MODE_STAGE2, j);
    if (e != cudaSuccess) return e;
    const long long v0 = (long long)(zs[j] + 2) * plane, v1 = (long long)(zs[j + 1] + 2) * plane;
    ghost_refresh_range_kernel<<<grid_for(v1 - v0, blk), blk, 0, sc>>>(b, h->ph, U, v0, v1);
    ++launches;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(h->ev_out[j], sc)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(so, h->ev_out[j], 0)) != cudaSuccess) return e;
    return copy(so, 6, zs[j] + 2, zs[j + 1] + 2, cudaMemcpyDeviceToHost);
  };
  // Once slab j is in: the flags of range j-1 and stage 1 of slab j-1 (which
  // reads two planes into slab j); then stage 2 of slab j-2, whose state no
  // later detection or stage 1 reads, so that its copy back overlaps the
  // copy in of the slabs still to come.  On a periodic z axis stage 1 of the
  // last slab reads the first planes of slab 0, which is therefore finished
  // last.
  const bool zper = b.bc[2][0] == BC_PERIODIC;
  int fin = zper ? 1 : 0;  // the next slab to finish
  for (int j = 0; j < S; ++j) {
    CUDA_TRY(cudaStreamWaitEvent(sc, h->ev_in[j], 0));
    if (j >= 1) {
      if (detect) CUDA_TRY(flags(j - 1));
      CUDA_TRY(stage(MODE_STAGE1, j - 1));
    }
    while (fin <= j - 2) CUDA_TRY(finish(fin++));
  }
  if (detect) CUDA_TRY(flags(S - 1));
  CUDA_TRY(stage(MODE_STAGE1, S - 1));
  while (fin < S) CUDA_TRY(finish(fin++));
  if (zper) CUDA_TRY(finish(0));
  // the z ghost planes, then their copy back and the fluence
  ghost_refresh_range_kernel<<<grid_for(2 * (long long)plane, blk), blk, 0, sc>>>(
      b, h->ph, U, 0, 2 * (long long)plane);
  ghost_refresh_range_kernel<<<grid_for(2 * (long long)plane, blk), blk, 0, sc>>>(
      b, h->ph, U, (long long)(n2 + 2) * plane, (long long)(n2 + 4) * plane);
  CUDA_TRY(cudaGetLastError());
  launches += 2;
  CUDA_TRY(cudaEventRecord(h->ev_end, sc));
  CUDA_TRY(cudaStreamWaitEvent(so, h->ev_end, 0));
  CUDA_TRY(copy(so, 6, 0, 2, cudaMemcpyDeviceToHost));
  CUDA_TRY(copy(so, 6, n2 + 2, n2 + 4, cudaMemcpyDeviceToHost));
  if (fluence_host)
    CUDA_TRY(cudaMemcpyAsync(fluence_host, fl, 36 * h->face_size * sizeof(double),
                             cudaMemcpyDeviceToHost, so));
  CUDA_TRY(cudaStreamSynchronize(so));
  CUDA_TRY(cudaStreamSynchronize(sc));
  h->launches += launches;
  h->prims_pending = false;
  h->features = FEAT_PENDING;
  h->features_src = U;
  h->wn_of = nullptr;  // the staging copy is overwritten by the next call
  return GFX_OK;
}

int create_handle(const gfx_fluid_config* cfg, const HostAxis* axes, gfx_fluid** out);

}  // namespace

extern "C" {

int gfx_fluid_config_default(gfx_fluid_config* c) {
  if (!c) return fail(GFX_ERR_ARGUMENT, "config is NULL");
  memset(c, 0, sizeof(*c));
  for (int d = 0; d < 3; ++d) {
    c->n_cells[d] = 32;
    c->min_coordinate[d] = 0.0;
    c->max_coordinate[d] = 1.0;
    c->boundary[d][0] = c->boundary[d][1] = GFX_BC_OUTFLOW;
  }
  c->n_ghost_layers = 2;
  c->riemann_solver = GFX_RIEMANN_HLLC;
  c->use_limiter = 1;
  c->limiter_parameter = 1.4;
  c->adiabatic_index = 1.4;
  c->shock_threshold = 0.1;
  c->courant_factor = 0.7;
  c->baryon_density_min = 0.0;
  c->uniform_acceleration = 0.0;
  c->n_ramp_cycles = 100;
  c->reconstruction = GFX_RECONSTRUCTION_LINEAR;
  return GFX_OK;
}

int gfx_fluid_create(const gfx_fluid_config* cfg, gfx_fluid** out) {
  if (!out) return fail(GFX_ERR_ARGUMENT, "out is NULL");
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) return rc;
  return create_handle(cfg, nullptr, out);
}

}  // extern "C"

namespace {

// The handle of one brick: its own chart geometry (axes == null), or the
// given per-axis tables (a brick of a chart, whose tables are a slice of the
// chart's).  cfg has been validated by the caller.
int create_handle(const gfx_fluid_config* cfg, const HostAxis* axes, gfx_fluid** out) {
  gfx_fluid* h = new (std::nothrow) gfx_fluid();
  if (!h) return fail(GFX_ERR_NO_MEMORY, "host allocation failed");
  h->cfg = *cfg;
  Phys& ph = h->ph;
  ph.gamma = cfg->adiabatic_index;
  ph.gm1 = cfg->adiabatic_index - 1.0;
  ph.c_v = 1.0 / (1.0 * (cfg->adiabatic_index - 1.0));
  ph.theta = cfg->limiter_parameter;
  ph.nmin = cfg->baryon_density_min;
  ph.accel = cfg->uniform_acceleration;
  ph.shock_threshold = cfg->shock_threshold;
  ph.courant = cfg->courant_factor;
  ph.use_limiter = cfg->use_limiter ? 1 : 0;
  ph.n_ramp = cfg->n_ramp_cycles;
  ph.parabolic = cfg->reconstruction == GFX_RECONSTRUCTION_PARABOLIC ? 1 : 0;
  Box& b = h->box;
  for (int d = 0; d < 3; ++d) {
    b.n[d] = cfg->n_cells[d];
    b.m[d] = cfg->n_cells[d] + 4;
    b.bc[d][0] = cfg->boundary[d][0];
    b.bc[d][1] = cfg->boundary[d][1];
    h->axis[d] = axes ? axes[d]
                      : build_axis(b.n[d], cfg->min_coordinate[d], cfg->max_coordinate[d], 2);
  }
  b.nV = (long long)b.m[0] * b.m[1] * b.m[2];
  b.nP = (long long)b.n[0] * b.n[1] * b.n[2];
  h->face_size = (size_t)std::max({(long long)b.n[1] * b.n[2], (long long)b.n[0] * b.n[2],
                                   (long long)b.n[0] * b.n[1]});
  auto cleanup = [&](int code) {
    gfx_fluid_destroy(h);
    return code;
  };
  // geometry arena: 9 tables per axis, then the PG_N parabolic ones, each m + 1 long
  size_t geo_len = 0;
  for (int d = 0; d < 3; ++d) geo_len += (9 + PG_N) * (size_t)(b.m[d] + 1);
  if (!dev_alloc(&h->geo, geo_len * sizeof(double)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc geometry"));
  {
    std::vector<double> host(geo_len, 0.0);
    size_t off = 0;
    for (int d = 0; d < 3; ++d) {
      const HostAxis& a = h->axis[d];
      const int L = b.m[d] + 1;
      const std::vector<double>* tabs[9] = {&a.W,   &a.WL,   &a.WR,    &a.dXI, &a.SQ,
                                            &a.CDEN, &a.RDXI, &a.RCDEN, &a.RW};
      const double** dst[9] = {&h->dgeo[d].W,    &h->dgeo[d].WL,   &h->dgeo[d].WR,
                               &h->dgeo[d].dXI,  &h->dgeo[d].SQ,   &h->dgeo[d].CDEN,
                               &h->dgeo[d].RDXI, &h->dgeo[d].RCDEN, &h->dgeo[d].RW};
      for (int q = 0; q < 9; ++q) {
        std::copy(tabs[q]->begin(), tabs[q]->end(), host.begin() + off);
        // tables are m long except the difference-based ones (m + 1)
        *dst[q] = h->geo + off;
        off += L;
      }
      std::copy(a.PAR.begin(), a.PAR.end(), host.begin() + off);
      h->dgeo[d].PAR = h->geo + off;
      off += (size_t)PG_N * L;
    }
    if (cudaMemcpy(h->geo, host.data(), geo_len * sizeof(double), cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return cleanup(fail(GFX_ERR_CUDA, "copy geometry tables"));
  }
  const size_t nP = (size_t)b.nP;
  if (!dev_alloc(&h->Yp, 5 * nP * sizeof(double)) ||
      !dev_alloc(&h->H, 5 * nP * sizeof(double)) ||
      !dev_alloc(&h->Pst, 5 * nP * sizeof(double)) ||
      !dev_alloc(&h->df, nP) ||
      !dev_alloc(&h->tsi_bits, 2 * sizeof(unsigned long long)) ||
      !dev_alloc(&h->counters, 4 * sizeof(int)) ||
      !dev_alloc(&h->clock, 2 * sizeof(Clock)) ||
      !dev_alloc(&h->dt_slot, sizeof(double)) ||
      !dev_alloc(&h->wn, 5 * nP * sizeof(double)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc of the stage scratch (%zu cells)", nP));
  if (cudaMemset(h->df, 0, nP) != cudaSuccess)
    return cleanup(fail(GFX_ERR_CUDA, "clear features"));
  std::vector<WorkItem> items = make_items(b.n, 0);
  h->n_items = (int)items.size();
  if (!dev_alloc(&h->items, items.size() * sizeof(WorkItem)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc work items"));
  if (cudaMemcpy(h->items, items.data(), items.size() * sizeof(WorkItem),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(GFX_ERR_CUDA, "copy work items"));
  h->features = FEAT_ZERO;
  *out = h;
  return GFX_OK;
}

}  // namespace

extern "C" {

int gfx_fluid_destroy(gfx_fluid* h) {
  if (!h) return GFX_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  cudaFree(h->geo);
  cudaFree(h->Yp);
  cudaFree(h->H);
  cudaFree(h->Pst);
  cudaFree(h->df);
  cudaFree(h->tsi_bits);
  cudaFree(h->counters);
  cudaFree(h->clock);
  cudaFree(h->dt_slot);
  cudaFree(h->items);
  cudaFree(h->U_stage);
  cudaFree(h->adj);
  cudaFree(h->adj_flags);
  cudaFree(h->branch_buf);
  cudaFree(h->adj_U);
  cudaFree(h->state_counts);
  cudaFree(h->partials);
  cudaFree(h->wn);
  cudaFree(h->slab_counters);
  cudaFree(h->Ksrc);
  cudaFree(h->host_items);
  for (int j = 0; j < kMaxSlabs; ++j) {
    if (h->ev_in[j]) cudaEventDestroy(h->ev_in[j]);
    if (h->ev_out[j]) cudaEventDestroy(h->ev_out[j]);
  }
  if (h->ev_end) cudaEventDestroy(h->ev_end);
  for (int j = 0; j < 2; ++j)
    if (h->evolve_ev[j]) cudaEventDestroy(h->evolve_ev[j]);
  ring_free(h->ring);
  if (h->copy_in) cudaStreamDestroy(h->copy_in);
  if (h->copy_out) cudaStreamDestroy(h->copy_out);
  if (h->host_stream) cudaStreamDestroy(h->host_stream);
  delete h;
  return GFX_OK;
}

int gfx_fluid_n_values(const gfx_fluid* h, size_t* n) {
  if (!h || !n) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *n = (size_t)h->box.nV;
  return GFX_OK;
}

int gfx_fluid_fluence_face_size(const gfx_fluid* h, size_t* face_size) {
  if (!h || !face_size) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *face_size = h->face_size;
  return GFX_OK;
}

int gfx_fluid_geometry(const gfx_fluid* h, int axis, double* c, double* wl, double* wr) {
  if (!h || axis < 0 || axis > 2) return fail(GFX_ERR_ARGUMENT, "bad handle or axis");
  const HostAxis& a = h->axis[axis];
  if (c) std::copy(a.X.begin(), a.X.end(), c);
  if (wl) std::copy(a.WL.begin(), a.WL.end(), wl);
  if (wr) std::copy(a.WR.begin(), a.WR.end(), wr);
  return GFX_OK;
}

int gfx_fluid_from_primitive(gfx_fluid* h, const double* prim, double* U, void* stream) {
  Range range_("Fluid_P_I % ComputeFromPrimitive");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_from_primitive")) return rc0;
  if (!h || !prim || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  from_primitive_kernel<<<grid_for(h->box.nV, 256), 256, 0, s>>>(h->box, h->ph, prim, U,
                                                                  h->Pst);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  h->prims_pending = true;
  h->wn_of = nullptr;
  return GFX_OK;
}

int gfx_fluid_to_primitive(gfx_fluid* h, double* U, double* prim, double* aux, void* stream) {
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  to_primitive_kernel<<<grid_for(h->box.nV, 256), 256, 0, s>>>(h->box, h->ph, U, prim, aux);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  h->prims_pending = false;
  h->wn_of = nullptr;
  return GFX_OK;
}

int gfx_fluid_detect_features(gfx_fluid* h, const double* U, void* stream) {
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_detect_features")) return rc0;
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  int rc = run_features(h, U, h->prims_pending ? h->Pst : nullptr, (cudaStream_t)stream);
  if (rc) return rc;
  h->features = FEAT_VALID;
  return GFX_OK;
}

int gfx_fluid_clear_features(gfx_fluid* h, void* stream) {
  if (!h) return fail(GFX_ERR_ARGUMENT, "NULL handle");
  CUDA_TRY(cudaMemsetAsync(h->df, 0, (size_t)h->box.nP, (cudaStream_t)stream));
  h->features = FEAT_ZERO;
  return GFX_OK;
}

int gfx_fluid_get_features(gfx_fluid* h, uint8_t* flags, void* stream) {
  if (!h || !flags) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->features == FEAT_PENDING) {
    int rc = run_features(h, h->features_src, nullptr, s);
    if (rc) return rc;
    h->features = FEAT_VALID;
  }
  scatter_flags_kernel<<<grid_for(h->box.nV, 256), 256, 0, s>>>(h->box, h->df, flags);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  return GFX_OK;
}

int gfx_fluid_increment(gfx_fluid* h, const double* U, double* K, double dt, double weight,
                        double* fluence, void* stream) {
  Range range_("IncrementDivergence_FV % Compute");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_increment")) return rc0;
  if (!h || !U || !K) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  if (hllc && h->features == FEAT_PENDING) {
    int rc = run_features(h, h->features_src, nullptr, s);
    if (rc) return rc;
    h->features = FEAT_VALID;
  }
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 4);
  CUDA_TRY(cudaGetLastError());
  const bool in_prim = h->prims_pending;
  BrickDesc d = make_desc(h, U, nullptr, K, in_prim ? h->Pst : nullptr, hllc ? h->df : nullptr,
                          fluence, h->dt_slot, weight, nullptr);
  CUDA_TRY(launch_stage(MODE_INCREMENT, in_prim, hllc, false, d, nullptr, h->items,
                        h->n_items, h->counters, h->ph, s));
  h->launches += 3;
  return GFX_OK;
}

int gfx_fluid_step(gfx_fluid* h, double* U, double dt, double* fluence, void* stream) {
  Range range_("Step_RK_C_ASC % Compute");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step")) return rc0;
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  cudaStream_t s = (cudaStream_t)stream;
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  const bool detect = (h->features == FEAT_PENDING);
  int rc = enqueue_step(h, U, h->dt_slot, nullptr, fluence, detect, s);
  if (rc) return rc;
  h->prims_pending = false;
  h->features = FEAT_PENDING;
  h->features_src = U;
  h->wn_of = U;
  return GFX_OK;
}

int gfx_fluid_step_sources(gfx_fluid* h, double* U, double dt, double* fluence,
                           double* sources, void* stream) {
  Range range_("Step_RK_C_ASC % Compute (Sources records)");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step_sources")) return rc0;
  if (!h || !U || !sources) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  if (!h->Ksrc && !dev_alloc(&h->Ksrc, 6 * (size_t)h->box.nV * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc sources scratch");
  cudaStream_t s = (cudaStream_t)stream;
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  const bool detect = (h->features == FEAT_PENDING);
  int rc = enqueue_step(h, U, h->dt_slot, nullptr, fluence, detect, s, nullptr, false, sources);
  if (rc) return rc;
  h->prims_pending = false;
  h->features = FEAT_PENDING;
  h->features_src = U;
  h->wn_of = U;
  return GFX_OK;
}

int gfx_fluid_step_host(gfx_fluid* h, double* U_host, double dt, double* fluence_host) {
  Range range_("Step_RK_C_ASC % Compute (host state)");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step_host")) return rc0;
  if (!h || !U_host) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  const size_t bytes = 6 * (size_t)h->box.nV * sizeof(double);
  if (!h->host_stream) CUDA_TRY(cudaStreamCreateWithFlags(&h->host_stream, cudaStreamNonBlocking));
  if (!h->U_stage && !dev_alloc(&h->U_stage, bytes + 36 * h->face_size * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc host-step staging");
  int prc = step_host_pipelined(h, U_host, dt, fluence_host);
  if (prc != GFX_ERR_UNSUPPORTED) return prc;
  cudaStream_t s = h->host_stream;
  double* fl = fluence_host ? h->U_stage + 6 * (size_t)h->box.nV : nullptr;
  CUDA_TRY(cudaMemcpyAsync(h->U_stage, U_host, bytes, cudaMemcpyHostToDevice, s));
  int rc = gfx_fluid_step(h, h->U_stage, dt, fl, s);
  if (rc) return rc;
  h->features_src = h->U_stage;
  h->wn_of = nullptr;  // the staging copy is overwritten by the next call
  CUDA_TRY(cudaMemcpyAsync(U_host, h->U_stage, bytes, cudaMemcpyDeviceToHost, s));
  if (fluence_host)
    CUDA_TRY(cudaMemcpyAsync(fluence_host, fl, 36 * h->face_size * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return GFX_OK;
}

int gfx_fluid_timestep(gfx_fluid* h, const double* U, int i_cycle, double* dt_host,
                       void* stream) {
  Range range_("Integrator_C_PS % ComputeTimeStepLocal");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_timestep")) return rc0;
  if (!h || !U || !dt_host) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 0);
  CUDA_TRY(cudaGetLastError());
  inverse_timestep_kernel<<<grid_for(h->box.nP, 256), 256, 0, s>>>(
      h->box, h->ph, U, h->prims_pending ? h->Pst : nullptr, h->dgeo[0], h->dgeo[1],
      h->dgeo[2], h->tsi_bits);
  CUDA_TRY(cudaGetLastError());
  Clock c;
  memset(&c, 0, sizeof(c));
  c.cycle = i_cycle;
  c.time = 0.0;
  c.finish = DBL_MAX;
  c.max_cycle = 0x7fffffff;
  Clock* dc = h->clock + 1;
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  finalize_dt_kernel<<<1, 1, 0, s>>>(h->ph, h->tsi_bits, dc, 1, 0);
  CUDA_TRY(cudaGetLastError());
  h->launches += 3;
  CUDA_TRY(cudaMemcpyAsync(&c, dc, sizeof(c), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  *dt_host = c.dt;
  return GFX_OK;
}

}  // extern "C"

namespace {

// The evolve loop of gfx_fluid_evolve; ev (may be null): two events, recorded
// on the stream before the first of its device work and after the last.
int evolve_impl(gfx_fluid* h, double* U, double time, int i_cycle, double finish_time,
                int n_cycles_max, double* time_out, int* i_cycle_out, cudaStream_t s,
                cudaEvent_t* ev) {
  Range range_("Integrator % Evolve");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_evolve")) return rc0;
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (n_cycles_max < 0) return fail(GFX_ERR_ARGUMENT, "n_cycles_max < 0");
  Clock c;
  memset(&c, 0, sizeof(c));
  c.time = time;
  c.finish = finish_time;
  c.cycle = i_cycle;
  c.max_cycle = (int)std::min<long long>(0x7fffffffLL, (long long)i_cycle + n_cycles_max);
  c.done = !(c.time < c.finish && c.cycle < c.max_cycle);
  Clock* dc = h->clock;
  if (ev) CUDA_TRY(cudaEventRecord(ev[0], s));
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  if (!c.done) {
    // initial dt from the state (ComputeNewTime before the first cycle)
    reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 0);
    inverse_timestep_kernel<<<grid_for(h->box.nP, 256), 256, 0, s>>>(
        h->box, h->ph, U, h->prims_pending ? h->Pst : nullptr, h->dgeo[0], h->dgeo[1],
        h->dgeo[2], h->tsi_bits);
    finalize_dt_kernel<<<1, 1, 0, s>>>(h->ph, h->tsi_bits, dc, 1, 1);
    CUDA_TRY(cudaGetLastError());
    h->launches += 3;
    // first cycle eagerly (its features follow the handle's state)
    int rc = enqueue_step(h, U, &dc->dt, &dc->done, nullptr, h->features == FEAT_PENDING, s);
    if (rc) return rc;
    advance_clock_kernel<<<1, 1, 0, s>>>(dc, 1);
    finalize_dt_kernel<<<1, 1, 0, s>>>(h->ph, h->tsi_bits, dc, 1, 1);
    CUDA_TRY(cudaGetLastError());
    h->launches += 2;
    h->prims_pending = false;
    h->features = FEAT_PENDING;
    h->features_src = U;
    h->wn_of = U;
    // remaining cycles: one graph per cycle, replayed
    if (h->graph && (h->graph_U != U)) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    if (!h->graph) {
      cudaStream_t cs;
      CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g;
      const long long before = h->launches;
      CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      // every captured cycle follows a step of this evolve: its flags and its
      // stage 1 read the primitives that step's stage 2 stored
      int rc2 = enqueue_step(h, U, &dc->dt, &dc->done, nullptr, true, cs, nullptr, true);
      advance_clock_kernel<<<1, 1, 0, cs>>>(dc, 1);
      finalize_dt_kernel<<<1, 1, 0, cs>>>(h->ph, h->tsi_bits, dc, 1, 1);
      cudaError_t ce = cudaStreamEndCapture(cs, &g);
      cudaStreamDestroy(cs);
      h->graph_kernels = h->launches - before + 2;
      h->launches = before;
      if (rc2) return rc2;
      if (ce != cudaSuccess) return fail(GFX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&h->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess)
        return fail(GFX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      h->graph_U = U;
    }
    // the remaining cycles in chunks, several in flight (ChunkRing)
    if (int rc3 = ring_init(h->ring)) return rc3;
    if (int rc3 = ring_run(h->ring, h->graph, h->graph_kernels, &h->launches, dc, 1,
                           n_cycles_max, s))
      return rc3;
  }
  if (ev) CUDA_TRY(cudaEventRecord(ev[1], s));
  CUDA_TRY(cudaMemcpyAsync(&c, dc, sizeof(c), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (time_out) *time_out = c.time;
  if (i_cycle_out) *i_cycle_out = c.cycle;
  return GFX_OK;
}

}  // namespace

extern "C" {

int gfx_fluid_evolve(gfx_fluid* h, double* U, double time, int i_cycle, double finish_time,
                     int n_cycles_max, double* time_out, int* i_cycle_out, void* stream) {
  return evolve_impl(h, U, time, i_cycle, finish_time, n_cycles_max, time_out, i_cycle_out,
                     (cudaStream_t)stream, nullptr);
}

int gfx_fluid_evolve_timed(gfx_fluid* h, double* U, double time, int i_cycle,
                           double finish_time, int n_cycles_max, double* time_out,
                           int* i_cycle_out, double* ms_out, void* stream) {
  if (!h || !ms_out) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (!h->evolve_ev[0]) {
    for (int j = 0; j < 2; ++j) CUDA_TRY(cudaEventCreate(&h->evolve_ev[j]));
  }
  int rc = evolve_impl(h, U, time, i_cycle, finish_time, n_cycles_max, time_out, i_cycle_out,
                       (cudaStream_t)stream, h->evolve_ev);
  if (rc) return rc;
  float ms = 0.0f;
  CUDA_TRY(cudaEventElapsedTime(&ms, h->evolve_ev[0], h->evolve_ev[1]));
  *ms_out = ms;
  return GFX_OK;
}

int gfx_fluid_step_timed(gfx_fluid* h, double* U, double dt, double* fluence, double* ms_out,
                         void* stream) {
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step_timed")) return rc0;
  if (!h || !U || !ms_out) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t ev[5];
  for (int i = 0; i < 5; ++i) CUDA_TRY(cudaEventCreate(&ev[i]));
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  const bool detect = (h->features == FEAT_PENDING);
  // the kernels of an evolve cycle when U is the state this handle's last
  // stage 2 produced: features and stage 1 from the primitives it stored
  const bool from_wn = (U == h->wn_of) && !h->prims_pending;
  int rc = enqueue_step(h, U, h->dt_slot, nullptr, fluence, detect, s, ev, from_wn);
  if (rc == GFX_OK) {
    h->prims_pending = false;
    h->features = FEAT_PENDING;
    h->features_src = U;
    h->wn_of = U;
    cudaError_t e = cudaEventSynchronize(ev[4]);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
      float ms = 0.f;
      e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      ms_out[i] = ms;
    }
    if (e != cudaSuccess) rc = fail(GFX_ERR_CUDA, "event timing: %s", cudaGetErrorString(e));
  }
  for (int i = 0; i < 5; ++i) cudaEventDestroy(ev[i]);
  return rc;
}

int gfx_fluid_kernel_launches(const gfx_fluid* h, long long* count) {
  if (!h || !count) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *count = h->launches;
  return GFX_OK;
}

int gfx_fluid_batch_create(int n, gfx_fluid* const* handles, double* const* U,
                           gfx_fluid_batch** out) {
  if (!out || n < 1 || !handles || !U) return fail(GFX_ERR_ARGUMENT, "bad batch arguments");
  *out = nullptr;
  for (int b = 0; b < n; ++b) {
    if (!handles[b] || !U[b]) return fail(GFX_ERR_ARGUMENT, "brick %d: NULL handle or state", b);
    if (int rc0 = refuse_chart_brick(handles[b], "gfx_fluid_batch_create")) return rc0;
  }
  const gfx_fluid_config& c0 = handles[0]->cfg;
  for (int b = 1; b < n; ++b) {
    const gfx_fluid_config& c = handles[b]->cfg;
    if (c.riemann_solver != c0.riemann_solver || c.uniform_acceleration != 0.0 ||
        c.adiabatic_index != c0.adiabatic_index || c.limiter_parameter != c0.limiter_parameter ||
        c.use_limiter != c0.use_limiter || c.shock_threshold != c0.shock_threshold ||
        c.courant_factor != c0.courant_factor || c.baryon_density_min != c0.baryon_density_min ||
        c.n_ramp_cycles != c0.n_ramp_cycles)
      return fail(GFX_ERR_ARGUMENT, "brick %d: parameters differ from brick 0", b);
  }
  if (c0.uniform_acceleration != 0.0)
    return fail(GFX_ERR_UNSUPPORTED, "batched bricks with gravity are not built");
  for (int b = 0; b < n; ++b)
    if (handles[b]->cfg.reconstruction != GFX_RECONSTRUCTION_LINEAR)
      return fail(GFX_ERR_UNSUPPORTED, "batched bricks: LINEAR reconstruction only");
  gfx_fluid_batch* B = new (std::nothrow) gfx_fluid_batch();
  if (!B) return fail(GFX_ERR_NO_MEMORY, "host allocation failed");
  auto cleanup = [&](int code) {
    gfx_fluid_batch_destroy(B);
    return code;
  };
  B->n = n;
  B->tile_y = handles[0]->tile_y;
  for (int b = 1; b < n; ++b)
    if (handles[b]->tile_y != B->tile_y)
      return cleanup(fail(GFX_ERR_ARGUMENT, "brick %d: tile rows differ from brick 0", b));
  B->h.assign(handles, handles + n);
  B->U.assign(U, U + n);
  B->ph = handles[0]->ph;
  B->hllc = c0.riemann_solver == GFX_RIEMANN_HLLC;
  if (!dev_alloc(&B->tsi_bits, n * sizeof(unsigned long long)) ||
      !dev_alloc(&B->clocks, n * sizeof(Clock)) ||
      !dev_alloc(&B->counters, 4 * sizeof(int)) ||
      !dev_alloc(&B->d1, n * sizeof(BrickDesc)) ||
      !dev_alloc(&B->d1p, n * sizeof(BrickDesc)) ||
      !dev_alloc(&B->d1w, n * sizeof(BrickDesc)) ||
      !dev_alloc(&B->d2, n * sizeof(BrickDesc)) ||
      !dev_alloc(&B->bb, n * sizeof(BatchBrick)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc batch tables"));
  std::vector<BrickDesc> d1(n), d1p(n), d1w(n), d2(n);
  std::vector<BatchBrick> bb(n);
  std::vector<WorkItem> items;
  std::vector<long long> work;
  std::vector<DetItem> det;
  for (int b = 0; b < n; ++b) {
    gfx_fluid* h = handles[b];
    const uint8_t* df = B->hllc ? h->df : nullptr;
    for (int z = 0; z < h->box.n[2]; z += kDetKZ)
      for (int y = 0; y < h->box.n[1]; y += kDetTY)
        for (int x = 0; x < h->box.n[0]; x += kDetTX) det.push_back({b, x, y, z});
    const double* dt = &B->clocks[b].dt;
    const int* skip = &B->clocks[b].done;
    d1[b] = make_desc(h, U[b], nullptr, nullptr, nullptr, df, nullptr, dt, 0.5, skip);
    d1p[b] = make_desc(h, U[b], nullptr, nullptr, h->Pst, df, nullptr, dt, 0.5, skip);
    d1w[b] = make_desc(h, U[b], nullptr, nullptr, h->wn, df, nullptr, dt, 0.5, skip);
    d2[b] = make_desc(h, U[b], U[b], nullptr, h->Yp, df, nullptr, dt, 0.5, skip);
    d2[b].wn = h->wn;
    d1[b].tsi_bits = d1p[b].tsi_bits = d1w[b].tsi_bits = d2[b].tsi_bits = B->tsi_bits + b;
    bb[b].box = h->box;
    bb[b].U = U[b];
    bb[b].df = h->df;
    bb[b].skip = skip;
    bb[b].v_off = B->total_v;
    bb[b].c_off = B->total_c;
    B->total_v += h->box.nV;
    B->total_c += h->box.nP;
    // z chunks of 32 planes (few prologues, many items to balance), or the
    // brick's tuned pencil length
    const int* nn = h->box.n;
    const int len = std::min(nn[2], h->z_chunk > 0 ? h->z_chunk : 32);
    const int ty = B->tile_y;
    for (int z = 0; z < nn[2]; z += len)
      for (int y = 0; y < nn[1]; y += ty)
        for (int x = 0; x < nn[0]; x += TX) {
          items.push_back({b, x, y, z, std::min(nn[2], z + len)});
          work.push_back((long long)std::min(TX, nn[0] - x) * std::min(ty, nn[1] - y) *
                         (std::min(nn[2], z + len) - z));
        }
  }
  // longest items first (LPT order for the persistent CTAs' work counter)
  std::vector<int> order(items.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  std::vector<WorkItem> sorted(items.size());
  for (size_t i = 0; i < order.size(); ++i) sorted[i] = items[order[i]];
  B->n_items = (int)sorted.size();
  if (!dev_alloc(&B->items, sorted.size() * sizeof(WorkItem)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc batch work items"));
  if (B->hllc) {
    B->n_det_items = (int)det.size();
    if (!dev_alloc(&B->det_items, det.size() * sizeof(DetItem)))
      return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc batch feature tiles"));
    if (cudaMemcpy(B->det_items, det.data(), det.size() * sizeof(DetItem),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return cleanup(fail(GFX_ERR_CUDA, "copy batch feature tiles"));
  }
  if (cudaMemcpy(B->d1, d1.data(), n * sizeof(BrickDesc), cudaMemcpyHostToDevice) ||
      cudaMemcpy(B->d1p, d1p.data(), n * sizeof(BrickDesc), cudaMemcpyHostToDevice) ||
      cudaMemcpy(B->d1w, d1w.data(), n * sizeof(BrickDesc), cudaMemcpyHostToDevice) ||
      cudaMemcpy(B->d2, d2.data(), n * sizeof(BrickDesc), cudaMemcpyHostToDevice) ||
      cudaMemcpy(B->bb, bb.data(), n * sizeof(BatchBrick), cudaMemcpyHostToDevice) ||
      cudaMemcpy(B->items, sorted.data(), sorted.size() * sizeof(WorkItem),
                 cudaMemcpyHostToDevice))
    return cleanup(fail(GFX_ERR_CUDA, "copy batch tables"));
  std::vector<Clock> clk(n);
  for (auto& c : clk) {
    memset(&c, 0, sizeof(c));
    c.finish = DBL_MAX;
    c.max_cycle = 0x7fffffff;
  }
  if (cudaMemcpy(B->clocks, clk.data(), n * sizeof(Clock), cudaMemcpyHostToDevice))
    return cleanup(fail(GFX_ERR_CUDA, "init batch clocks"));
  *out = B;
  return GFX_OK;
}

int gfx_fluid_batch_destroy(gfx_fluid_batch* B) {
  if (!B) return GFX_OK;
  if (B->graph) cudaGraphExecDestroy(B->graph);
  cudaFree(B->tsi_bits);
  cudaFree(B->clocks);
  cudaFree(B->counters);
  cudaFree(B->d1);
  cudaFree(B->d1p);
  cudaFree(B->d1w);
  cudaFree(B->d2);
  cudaFree(B->bb);
  cudaFree(B->items);
  cudaFree(B->det_items);
  delete B;
  return GFX_OK;
}

int gfx_fluid_batch_set_clocks(gfx_fluid_batch* B, double time, int i_cycle) {
  if (!B) return fail(GFX_ERR_ARGUMENT, "NULL batch");
  std::vector<Clock> clk(B->n);
  for (auto& c : clk) {
    memset(&c, 0, sizeof(c));
    c.time = time;
    c.cycle = i_cycle;
    c.finish = DBL_MAX;
    c.max_cycle = 0x7fffffff;
  }
  CUDA_TRY(cudaMemcpy(B->clocks, clk.data(), B->n * sizeof(Clock), cudaMemcpyHostToDevice));
  return GFX_OK;
}

// per brick: finish time and cycle limit for this call, done flags
__global__ void batch_arm_clocks_kernel(Clock* clk, int n, double finish, int n_cycles) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  Clock& c = clk[b];
  c.finish = finish;
  const long long mc = (long long)c.cycle + n_cycles;
  c.max_cycle = (int)(mc > 0x7fffffffLL ? 0x7fffffffLL : mc);
  c.done = !(c.time < c.finish && c.cycle < c.max_cycle);
}

int gfx_fluid_batch_evolve(gfx_fluid_batch* B, double finish_time, int n_cycles, void* stream) {
  Range range_("Integrator % Evolve (batched bricks)");
  if (!B || n_cycles < 0) return fail(GFX_ERR_ARGUMENT, "bad batch evolve arguments");
  if (n_cycles == 0) return GFX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  // one state for the first cycle: every brick's primitives kept, or none
  int pend = 0, feat_pending = 0, feat_zero = 0;
  for (gfx_fluid* h : B->h) {
    pend += h->prims_pending;
    feat_pending += (h->features == FEAT_PENDING);
    feat_zero += (h->features == FEAT_ZERO);
  }
  if (pend != 0 && pend != B->n)
    return fail(GFX_ERR_STATE, "batch: bricks mix kept primitives and conserved states");
  if (B->hllc && feat_pending != 0 && feat_pending != B->n)
    return fail(GFX_ERR_STATE, "batch: bricks mix pending and current features");
  const bool in_prim = pend == B->n;
  const int blk = 256;
  batch_arm_clocks_kernel<<<grid_for(B->n, blk), blk, 0, s>>>(B->clocks, B->n, finish_time,
                                                              n_cycles);
  reset_bits_kernel<<<grid_for(std::max(B->n, 4), blk), blk, 0, s>>>(B->tsi_bits, B->n,
                                                                      B->counters, 0);
  CUDA_TRY(cudaGetLastError());
  B->launches += 2;
  for (int b = 0; b < B->n; ++b) {
    gfx_fluid* h = B->h[b];
    inverse_timestep_kernel<<<grid_for(h->box.nP, 256), 256, 0, s>>>(
        h->box, h->ph, B->U[b], in_prim ? h->Pst : nullptr, h->dgeo[0], h->dgeo[1],
        h->dgeo[2], B->tsi_bits + b);
  }
  finalize_dt_kernel<<<grid_for(B->n, blk), blk, 0, s>>>(B->ph, B->tsi_bits, B->clocks, B->n, 1);
  CUDA_TRY(cudaGetLastError());
  B->launches += B->n + 1;
  // first cycle eagerly (its primitives and features follow the handles' state)
  int rc = enqueue_batch_cycle(B, B->hllc && feat_pending == B->n, in_prim ? B->d1p : B->d1,
                               in_prim, s);
  if (rc) return rc;
  for (gfx_fluid* h : B->h) {
    h->prims_pending = false;
    h->features = FEAT_PENDING;
    h->wn_of = nullptr;
  }
  for (int b = 0; b < B->n; ++b) B->h[b]->features_src = B->U[b];
  if (n_cycles > 1) {
    if (!B->graph) {
      cudaStream_t cs;
      CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g;
      const long long before = B->launches;
      CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      // the replayed cycles follow a stage 2 of this evolve: stage 1 reads
      // the primitives it stored
      int rc2 = enqueue_batch_cycle(B, true, B->d1w, true, cs);
      cudaError_t ce = cudaStreamEndCapture(cs, &g);
      cudaStreamDestroy(cs);
      B->graph_kernels = B->launches - before;
      B->launches = before;
      if (rc2) return rc2;
      if (ce != cudaSuccess)
        return fail(GFX_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&B->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess)
        return fail(GFX_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ce));
    }
    for (int r = 1; r < n_cycles; ++r) CUDA_TRY(cudaGraphLaunch(B->graph, s));
    B->launches += (long long)(n_cycles - 1) * B->graph_kernels;
  }
  return GFX_OK;
}

int gfx_fluid_batch_clocks(gfx_fluid_batch* B, double* time, int* cycle, void* stream) {
  if (!B) return fail(GFX_ERR_ARGUMENT, "NULL batch");
  std::vector<Clock> clk(B->n);
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(clk.data(), B->clocks, B->n * sizeof(Clock), cudaMemcpyDeviceToHost,
                           s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int b = 0; b < B->n; ++b) {
    if (time) time[b] = clk[b].time;
    if (cycle) cycle[b] = clk[b].cycle;
  }
  return GFX_OK;
}

int gfx_fluid_batch_kernel_launches(const gfx_fluid_batch* B, long long* count) {
  if (!B || !count) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *count = B->launches;
  return GFX_OK;
}

int gfx_fluid_check_state(gfx_fluid* h, const double* U, void* stream) {
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (!h->state_counts && !dev_alloc(&h->state_counts, 2 * sizeof(unsigned long long)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc state counters");
  CUDA_TRY(cudaMemsetAsync(h->state_counts, 0, 2 * sizeof(unsigned long long), s));
  check_state_kernel<<<grid_for(h->box.nP, 256), 256, 0, s>>>(h->box, h->ph, U,
                                                               h->state_counts);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  unsigned long long c[2] = {0, 0};
  CUDA_TRY(cudaMemcpyAsync(c, h->state_counts, sizeof(c), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (c[0] != 0)
    return fail(GFX_ERR_STATE, "%llu proper cells hold non-finite values (%llu at the density "
                "floor)", c[0], c[1]);
  return GFX_OK;
}

int gfx_fluid_resume(gfx_fluid* h, double* U) {
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_resume")) return rc0;
  if (!h || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  h->prims_pending = false;
  h->features = FEAT_PENDING;
  h->features_src = U;
  h->wn_of = nullptr;
  return GFX_OK;
}

int gfx_fluid_totals(gfx_fluid* h, const double* U, double* totals, void* stream) {
  if (!h || !U || !totals) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = 4 * num_sms();
  const long long chunk = (h->box.nP + blocks - 1) / blocks;
  if (!h->partials && !dev_alloc(&h->partials, 6 * blocks * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc tally partials");
  totals_kernel<<<blocks, 256, 0, s>>>(h->box, U, h->dgeo[0], h->dgeo[1], h->dgeo[2], chunk,
                                       h->partials);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  std::vector<double> part(6 * (size_t)blocks);
  CUDA_TRY(cudaMemcpyAsync(part.data(), h->partials, part.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int q = 0; q < 6; ++q) {
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += part[6 * (size_t)b + q];
    totals[q] = t;
  }
  return GFX_OK;
}

int gfx_fluid_set_tuning(gfx_fluid* h, int z_chunk, int adjoint_segment, int tile_rows) {
  if (!h) return fail(GFX_ERR_ARGUMENT, "NULL handle");
  if (z_chunk < 0 || adjoint_segment < 0 || adjoint_segment > 4096)
    return fail(GFX_ERR_ARGUMENT, "z_chunk = %d, adjoint_segment = %d", z_chunk,
                adjoint_segment);
  if (tile_rows == 0) tile_rows = kTileY;
  if (tile_rows != 8 && tile_rows != kTileY)
    return fail(GFX_ERR_ARGUMENT, "tile_rows = %d: 8 or %d", tile_rows, kTileY);
  if (tile_rows != kTileY && h->cfg.reconstruction != GFX_RECONSTRUCTION_LINEAR)
    return fail(GFX_ERR_UNSUPPORTED, "PARABOLIC runs on %d-row tiles only", kTileY);
  if (z_chunk != h->z_chunk || tile_rows != h->tile_y) {
    std::vector<WorkItem> items = make_items(h->box.n, 0, z_chunk, tile_rows);
    WorkItem* d = nullptr;
    if (cudaMalloc(&d, items.size() * sizeof(WorkItem)) != cudaSuccess)
      return fail(GFX_ERR_NO_MEMORY, "cudaMalloc work items");
    if (cudaMemcpy(d, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice) !=
        cudaSuccess) {
      cudaFree(d);
      return fail(GFX_ERR_CUDA, "copy work items");
    }
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(h->items);
    h->items = d;
    h->n_items = (int)items.size();
    // the cycle graph holds the old list
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    h->z_chunk = z_chunk;
    h->tile_y = tile_rows;
  }
  h->adjoint_segment = adjoint_segment;
  return GFX_OK;
}

int gfx_fluid_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return GFX_ERR_ARGUMENT;
  snprintf(buf, len, "%s", g_last_error.c_str());
  return GFX_OK;
}

int gfx_fluid_debug_fail_allocation(int nth) {
  g_fail_alloc = nth < 0 ? -1 : nth;
  return GFX_OK;
}

}  // extern "C"

// ---- One RK2 step that allocates nothing ----------------------------------
// Some callers cannot call cudaMalloc: a host program whose memory manager
// claims the device memory up front into a pool of its own (cudaMalloc then
// fails, or is not theirs to call), or a code path that cannot afford the
// device-wide synchronisation that cudaMalloc and cudaFree imply.  For them
// gfx_fluid_step_noalloc runs the step of gfx_fluid_step without a handle:
// every table and buffer that the step needs besides the caller's state lives
// in one fixed array of device memory, compiled into this library.  Every GPU
// that loads the library holds the array until the process exits.
namespace {

constexpr size_t kNoAllocScratchBytes = GFX_FLUID_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The array's device address on the current device.  In host code the array's
// name is only a host-side stand-in, so the address is asked of the runtime,
// with that device current.  It is asked on every call rather than cached:
// after a cudaDeviceReset the module is loaded again, possibly elsewhere, and
// the lookup costs little next to a step.  The first call on a device is the
// one that loads the module there.
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(GFX_ERR_UNSUPPORTED, "device %d: the no-allocation step serves devices 0..%d",
                dev, kMaxDevices - 1);
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(GFX_ERR_CUDA, "cudaGetSymbolAddress of the no-allocation scratch: %s",
                cudaGetErrorString(e));
  *out = (unsigned char*)p;
  return GFX_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Byte offsets of the step's buffers inside the scratch array.
struct NoAllocLayout {
  size_t geo[3], edge[3], yp, h, df, bits, counters, dt, items, total;
};

// Parameters of the set-up kernel: the chart of the brick, the work list's
// shape (the same cut of columns and z chunks as the handle's list) and the
// step's time step.
struct NoAllocSetup {
  int n[3], m[3];
  double mn[3], mx[3];
  double* geo[3];   // 9 tables of m + 1 values per axis
  double* edge[3];  // m + 1 cell edges per axis
  WorkItem* items;
  int cx, cy, len, n_items;
  unsigned long long* bits;
  int* counters;
  double* dt_slot;
  double dt;
};

// Geometry tables, work list, CFL word, work counters and time step of one
// step, written into the scratch by one CTA.  The tables are the values of
// build_axis (the same operations in the same order, IEEE divisions), so the
// step reads the numbers that a handle's tables hold.
__global__ void noalloc_setup_kernel(NoAllocSetup p) {
  if (threadIdx.x < 3) {
    // cell edges by repeated addition, ghost widths through single precision
    // (Chart_Template.f90:478-560): a sequential chain, one thread per axis
    const int d = threadIdx.x, n = p.n[d], g = 2;
    double* E1 = p.edge[d] + g - 1;
    const double width = (p.mx[d] - p.mn[d]) / (double)n;
    E1[1] = p.mn[d];
    for (int i = 2; i <= n + 1; ++i) E1[i] = E1[i - 1] + width;
    for (int iC = 1; iC <= g; ++iC) {
      const float w_ig = (float)(E1[iC + 1] - E1[iC]);
      const float w_og = (float)(E1[n - iC + 2] - E1[n - iC + 1]);
      E1[1 - iC] = E1[2 - iC] - (double)w_ig;
      E1[n + 1 + iC] = E1[n + iC] + (double)w_og;
    }
  }
  for (int i = threadIdx.x; i < p.n_items; i += blockDim.x) {
    const int x = i % p.cx, y = (i / p.cx) % p.cy, zc = i / (p.cx * p.cy);
    const int z0 = zc * p.len;
    p.items[i] = {0, x * TX, y * kTileY, z0, min(p.n[2], z0 + p.len)};
  }
  if (threadIdx.x == 0) {
    p.bits[0] = 0x0010000000000000ull;  // ordered_bits(-DBL_MAX), as reset_bits_kernel
    p.bits[1] = 0x0010000000000000ull;
    for (int c = 0; c < 4; ++c) p.counters[c] = 0;
    *p.dt_slot = p.dt;
  }
  __syncthreads();
  for (int d = 0; d < 3; ++d) {
    const int m = p.m[d], L = m + 1;
    const double* e = p.edge[d];
    double* G = p.geo[d];
    for (int t = threadIdx.x; t <= m; t += blockDim.x) {
      double W = 0.0, WL = 0.0, WR = 0.0, RW = 0.0;
      if (t < m) {
        const double c = 0.5 * (e[t] + e[t + 1]);
        WL = c - e[t];
        WR = e[t + 1] - c;
        W = WL + WR;
        RW = 1.0 / W;
      }
      double dxi = 0.0, sq = 0.0, rdxi = 0.0, cden = 0.0, rcden = 0.0;
      if (t >= 1 && t < m) {
        const double c0 = 0.5 * (e[t - 1] + e[t]);
        const double c1 = 0.5 * (e[t] + e[t + 1]);
        dxi = c1 - c0;
        sq = dxi * dxi;
        rdxi = 1.0 / dxi;
        if (t + 1 < m) {
          const double c2 = 0.5 * (e[t + 1] + e[t + 2]);
          const double dxn = c2 - c1;
          cden = dxi * dxn * (dxi + dxn);
          rcden = 1.0 / cden;
        }
      }
      // table order of the handle's arena: W, WL, WR, dXI, SQ, CDEN, RDXI, RCDEN, RW
      G[0 * L + t] = W;
      G[1 * L + t] = WL;
      G[2 * L + t] = WR;
      G[3 * L + t] = dxi;
      G[4 * L + t] = sq;
      G[5 * L + t] = cden;
      G[6 * L + t] = rdxi;
      G[7 * L + t] = rcden;
      G[8 * L + t] = RW;
    }
  }
}

}  // namespace

extern "C" {

// The step of gfx_fluid_step on a handle whose state was set from conserved
// values (no pending primitives): features detected from U_dev first when
// detect_features is nonzero, zero features otherwise (the first step after
// initialisation).  Every buffer besides U_dev and fluence_dev is carved from
// the fixed scratch array; nothing is allocated.
int gfx_fluid_step_noalloc(const gfx_fluid_config* cfg, double* U, double dt,
                           int detect_features, double* fluence, void* stream) {
  int rc = validate(cfg);
  if (rc) return rc;
  if (!U) return fail(GFX_ERR_ARGUMENT, "U_dev is NULL");
  if (cfg->reconstruction != GFX_RECONSTRUCTION_LINEAR)
    return fail(GFX_ERR_UNSUPPORTED, "the no-allocation step: LINEAR reconstruction only");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  // the parameters and chart of gfx_fluid_create, without the handle
  Phys ph;
  memset(&ph, 0, sizeof(ph));
  ph.gamma = cfg->adiabatic_index;
  ph.gm1 = cfg->adiabatic_index - 1.0;
  ph.c_v = 1.0 / (1.0 * (cfg->adiabatic_index - 1.0));
  ph.theta = cfg->limiter_parameter;
  ph.nmin = cfg->baryon_density_min;
  ph.accel = cfg->uniform_acceleration;
  ph.shock_threshold = cfg->shock_threshold;
  ph.courant = cfg->courant_factor;
  ph.use_limiter = cfg->use_limiter ? 1 : 0;
  ph.n_ramp = cfg->n_ramp_cycles;
  Box b;
  memset(&b, 0, sizeof(b));
  for (int d = 0; d < 3; ++d) {
    b.n[d] = cfg->n_cells[d];
    b.m[d] = cfg->n_cells[d] + 4;
    b.bc[d][0] = cfg->boundary[d][0];
    b.bc[d][1] = cfg->boundary[d][1];
  }
  b.nV = (long long)b.m[0] * b.m[1] * b.m[2];
  b.nP = (long long)b.n[0] * b.n[1] * b.n[2];
  const long long face_size = std::max({(long long)b.n[1] * b.n[2],
                                        (long long)b.n[0] * b.n[2],
                                        (long long)b.n[0] * b.n[1]});
  // work list shape: the cut of make_items
  const int cx = (b.n[0] + TX - 1) / TX, cy = (b.n[1] + kTileY - 1) / kTileY;
  const long long cols = (long long)cx * cy;
  const long long want = 16LL * num_sms();
  const int chunks =
      (int)std::max(1LL, std::min<long long>(b.n[2] / 16, (want + cols - 1) / cols));
  const int len = (b.n[2] + chunks - 1) / chunks;
  const long long n_items = cols * ((b.n[2] + len - 1) / len);
  // scratch layout, every buffer on a 256-byte boundary
  NoAllocLayout L;
  size_t off = 0;
  for (int d = 0; d < 3; ++d) {
    L.geo[d] = off;
    off = align256(off + 9 * (size_t)(b.m[d] + 1) * sizeof(double));
    L.edge[d] = off;
    off = align256(off + (size_t)(b.m[d] + 1) * sizeof(double));
  }
  const size_t nP = (size_t)b.nP;
  L.yp = off;
  off = align256(off + 5 * nP * sizeof(double));
  L.h = off;
  off = align256(off + 5 * nP * sizeof(double));
  L.df = off;
  off = align256(off + nP);
  L.bits = off;
  off = align256(off + 2 * sizeof(unsigned long long));
  L.counters = off;
  off = align256(off + 4 * sizeof(int));
  L.dt = off;
  off = align256(off + sizeof(double));
  L.items = off;
  off = align256(off + (size_t)n_items * sizeof(WorkItem));
  L.total = off;
  if (L.total > kNoAllocScratchBytes)
    return fail(GFX_ERR_ARGUMENT,
                "brick %d x %d x %d needs %zu bytes of scratch; the no-allocation step has "
                "%zu: about 81 bytes per proper cell plus the chart tables, so up to about 50000 "
                "proper cells (37^3 fits, 38^3 does not)",
                b.n[0], b.n[1], b.n[2], L.total, kNoAllocScratchBytes);
  unsigned char* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;

  NoAllocSetup p;
  memset(&p, 0, sizeof(p));
  AxisGeo geo[3];
  for (int d = 0; d < 3; ++d) {
    p.n[d] = b.n[d];
    p.m[d] = b.m[d];
    p.mn[d] = cfg->min_coordinate[d];
    p.mx[d] = cfg->max_coordinate[d];
    p.geo[d] = (double*)(base + L.geo[d]);
    p.edge[d] = (double*)(base + L.edge[d]);
    const int Lt = b.m[d] + 1;
    const double* G = p.geo[d];
    geo[d] = {G, G + Lt, G + 2 * Lt, G + 3 * Lt, G + 4 * Lt,
              G + 5 * Lt, G + 6 * Lt, G + 7 * Lt, G + 8 * Lt};
  }
  p.items = (WorkItem*)(base + L.items);
  p.cx = cx;
  p.cy = cy;
  p.len = len;
  p.n_items = (int)n_items;
  p.bits = (unsigned long long*)(base + L.bits);
  p.counters = (int*)(base + L.counters);
  p.dt_slot = (double*)(base + L.dt);
  p.dt = dt;
  // the scratch keeps the previous call's contents: the set-up rewrites the
  // tables and the work list and zeroes the CFL word and the work counters
  // (the two things that must start at zero) before the stages run
  noalloc_setup_kernel<<<1, 256, 0, s>>>(p);
  CUDA_TRY(cudaGetLastError());
  if (fluence) CUDA_TRY(cudaMemsetAsync(fluence, 0, sizeof(double) * 36 * face_size, s));
  const bool hllc = cfg->riemann_solver == GFX_RIEMANN_HLLC;
  const bool grav = cfg->uniform_acceleration != 0.0;
  uint8_t* df = (uint8_t*)(base + L.df);
  if (hllc && detect_features) CUDA_TRY(launch_features(b, ph, U, nullptr, df, 0, b.n[2], s));
  const uint8_t* feat = (hllc && detect_features) ? df : nullptr;
  BrickDesc d;
  memset(&d, 0, sizeof(d));
  for (int a = 0; a < 3; ++a) {
    d.n[a] = b.n[a];
    d.m[a] = b.m[a];
    d.bc[a][0] = b.bc[a][0];
    d.bc[a][1] = b.bc[a][1];
    d.geo[a] = geo[a];
  }
  d.nV = b.nV;
  d.nP = b.nP;
  d.Yp = (double*)(base + L.yp);
  d.H = (double*)(base + L.h);
  d.df = feat;
  d.fluence = fluence;
  d.face_size = face_size;
  d.dt = p.dt_slot;
  d.weight = 0.5;
  d.tsi_bits = p.bits;
  d.skip = nullptr;
  BrickDesc d1 = d;
  d1.U_in = U;
  CUDA_TRY(launch_stage(MODE_STAGE1, false, hllc, grav, d1, nullptr, p.items, p.n_items,
                        p.counters, ph, s));
  BrickDesc d2 = d;
  d2.U_in = U;
  d2.U_out = U;
  d2.P_in = d.Yp;
  CUDA_TRY(launch_stage(MODE_STAGE2, true, hllc, grav, d2, nullptr, p.items, p.n_items,
                        p.counters + 1, ph, s));
  ghost_refresh_kernel<<<grid_for(b.nV, 256), 256, 0, s>>>(b, ph, U);
  CUDA_TRY(cudaGetLastError());
  return GFX_OK;
}

}  // extern "C"

// ---- Discrete adjoint of one RK2 step --------------------------------------
namespace {

template <int D>
cudaError_t launch_adj_face(const AdjDesc& A, bool hllc, const Phys& ph, cudaStream_t s) {
  constexpr int T1 = (D == 0) ? 1 : 0;
  constexpr int T2 = (D == 2) ? 1 : 2;
  const long long total = (long long)A.nseg * A.n[T1] * A.n[T2];
  const int blk = 128;
  if constexpr (D == 0) {  // one lane per face, a warp per kAdjXFaces faces of a pencil
    const long long lanes =
        32LL * ((A.n[0] + 1 + kAdjXFaces - 1) / kAdjXFaces) * A.n[1] * A.n[2];
    if (hllc)
      adj_face_x_kernel<true><<<grid_for(lanes, blk), blk, 0, s>>>(A, ph);
    else
      adj_face_x_kernel<false><<<grid_for(lanes, blk), blk, 0, s>>>(A, ph);
  } else if (hllc)
    adj_face_kernel<D, true><<<grid_for(total, blk), blk, 0, s>>>(A, ph);
  else
    adj_face_kernel<D, false><<<grid_for(total, blk), blk, 0, s>>>(A, ph);
  return cudaGetLastError();
}

// L^T of one stage: lamW += (dK/dW)^T (kscale lamK), one launch per direction.
int enqueue_adj_stage(gfx_fluid* h, const double* W, const double* lamK, double kscale,
                      double* lamW, const uint8_t* df, double dt, cudaStream_t s) {
  AdjDesc A;
  memset(&A, 0, sizeof(A));
  for (int a = 0; a < 3; ++a) {
    A.n[a] = h->box.n[a];
    A.bc[a][0] = h->box.bc[a][0];
    A.bc[a][1] = h->box.bc[a][1];
    A.geo[a] = h->dgeo[a];
  }
  A.nP = h->box.nP;
  A.W = W;
  A.lamK = lamK;
  A.lamW = lamW;
  A.df = df;
  A.dt = dt;
  A.kscale = kscale;
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  A.seg = h->adjoint_segment > 0 ? h->adjoint_segment : 8;
  A.nseg = (h->box.n[0] + 1 + A.seg - 1) / A.seg;
  CUDA_TRY(launch_adj_face<0>(A, hllc, h->ph, s));
  A.nseg = (h->box.n[1] + 1 + A.seg - 1) / A.seg;
  CUDA_TRY(launch_adj_face<1>(A, hllc, h->ph, s));
  A.nseg = (h->box.n[2] + 1 + A.seg - 1) / A.seg;
  CUDA_TRY(launch_adj_face<2>(A, hllc, h->ph, s));
  h->launches += 3;
  return GFX_OK;
}

}  // namespace

extern "C" {

int gfx_fluid_step_adjoint(gfx_fluid* h, const double* U_n, double dt, const double* lam_np1,
                           double* lam_n, const double* U_np1, int detect_features,
                           void* stream) {
  Range range_("Step_RK_C_ASC % Compute (adjoint)");
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step_adjoint")) return rc0;
  if (!h || !U_n || !lam_np1 || !lam_n) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (lam_n == lam_np1) return fail(GFX_ERR_ARGUMENT, "lam_n must not alias lam_np1");
  if (h->cfg.reconstruction != GFX_RECONSTRUCTION_LINEAR)
    return fail(GFX_ERR_UNSUPPORTED, "adjoint: LINEAR reconstruction only");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  cudaStream_t s = (cudaStream_t)stream;
  const Box& b = h->box;
  if (b.nP >= (1LL << 31))
    return fail(GFX_ERR_UNSUPPORTED, "adjoint: %lld proper cells (at most 2^31 - 1)", b.nP);
  const size_t nP = (size_t)b.nP, nV = (size_t)b.nV;
  // each buffer on its own: a failed allocation leaves its pointer null and
  // the next call tries it again
  if (!h->adj && !dev_alloc(&h->adj, 20 * nP * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc adjoint workspace (%zu cells)", nP);
  if (!h->adj_flags && !dev_alloc(&h->adj_flags, nP))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc adjoint flags");
  if (!U_np1 && !h->adj_U && !dev_alloc(&h->adj_U, 6 * nV * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc adjoint state");
  double* W0 = h->adj;
  double* lamZ = W0 + 5 * nP;
  double* lamW = lamZ + 5 * nP;
  double* lamK1 = lamW + 5 * nP;
  uint8_t* df = h->adj_flags;
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  const bool grav = h->cfg.uniform_acceleration != 0.0;
  const int blk = 256;
  // features of U^n (zero for the first step after initialisation)
  const uint8_t* feat = nullptr;
  if (hllc && detect_features) {
    CUDA_TRY(launch_features(b, h->ph, U_n, nullptr, df, 0, b.n[2], s));
    h->launches += 1;
    feat = df;
  }
  // forward recomputation from the checkpoint: stage 1 (which also stores the
  // primitives W0 of U^n it recovers, and W1 into Yp) and, without U^n+1
  // from the caller, stage 2
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 4);
  CUDA_TRY(cudaGetLastError());
  h->launches += 2;
  BrickDesc d1 = make_desc(h, U_n, nullptr, nullptr, nullptr, feat, nullptr, h->dt_slot, 0.5,
                           nullptr);
  d1.wn = W0;
  CUDA_TRY(launch_stage(MODE_STAGE1, false, hllc, grav, d1, nullptr, h->items, h->n_items,
                        h->counters, h->ph, s));
  h->launches += 1;
  const double* Unew = U_np1;
  if (!Unew) {
    BrickDesc d2 = make_desc(h, U_n, h->adj_U, nullptr, h->Yp, feat, nullptr, h->dt_slot, 0.5,
                             nullptr);
    CUDA_TRY(launch_stage(MODE_STAGE2, true, hllc, grav, d2, nullptr, h->items, h->n_items,
                          h->counters + 1, h->ph, s));
    h->launches += 1;
    Unew = h->adj_U;
  }
  // reverse sweep
  adj_final_kernel<<<grid_for(b.nP, blk), blk, 0, s>>>(b, h->ph, lam_np1, Unew, lamZ);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemsetAsync(lamW, 0, 5 * nP * sizeof(double), s));
  h->launches += 1;
  int rc = enqueue_adj_stage(h, h->Yp, lamZ, 0.5, lamW, feat, dt, s);
  if (rc) return rc;
  adj_mid_kernel<<<grid_for(b.nP, blk), blk, 0, s>>>(b, h->ph, dt, h->Yp, lamZ, lamW, lamK1);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  CUDA_TRY(cudaMemsetAsync(lamW, 0, 5 * nP * sizeof(double), s));
  CUDA_TRY(cudaMemsetAsync(lam_n, 0, 6 * nV * sizeof(double), s));
  rc = enqueue_adj_stage(h, W0, lamK1, 1.0, lamW, feat, dt, s);
  if (rc) return rc;
  adj_last_kernel<<<grid_for(b.nP, blk), blk, 0, s>>>(b, h->ph, dt, W0, lamK1, lamZ, lamW,
                                                       lam_n);
  CUDA_TRY(cudaGetLastError());
  h->launches += 1;
  return GFX_OK;
}

static_assert(BR_KINDS == GFX_BRANCH_KINDS, "branch kinds of the header");

int gfx_fluid_step_branches(gfx_fluid* h, const double* U_n, double dt, int detect_features,
                            unsigned long long* out, void* stream) {
  if (int rc0 = refuse_chart_brick(h, "gfx_fluid_step_branches")) return rc0;
  if (!h || !U_n || !out) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (h->cfg.reconstruction != GFX_RECONSTRUCTION_LINEAR)
    return fail(GFX_ERR_UNSUPPORTED, "branch signature: LINEAR reconstruction only");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  cudaStream_t s = (cudaStream_t)stream;
  const Box& b = h->box;
  if (b.nP >= (1LL << 31))
    return fail(GFX_ERR_UNSUPPORTED, "branch signature: %lld proper cells", b.nP);
  const size_t nP = (size_t)b.nP;
  // each buffer on its own (as in gfx_fluid_step_adjoint)
  if (!h->adj && !dev_alloc(&h->adj, 20 * nP * sizeof(double)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc adjoint workspace (%zu cells)", nP);
  if (!h->adj_flags && !dev_alloc(&h->adj_flags, nP))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc adjoint flags");
  if (!h->branch_buf &&
      !dev_alloc(&h->branch_buf, (2 + BR_KINDS) * sizeof(unsigned long long)))
    return fail(GFX_ERR_NO_MEMORY, "cudaMalloc branch signature");
  double* W0 = h->adj;
  uint8_t* df = h->adj_flags;
  const bool hllc = h->cfg.riemann_solver == GFX_RIEMANN_HLLC;
  const bool grav = h->cfg.uniform_acceleration != 0.0;
  const int blk = 256;
  const uint8_t* feat = nullptr;
  if (hllc && detect_features) {
    CUDA_TRY(launch_features(b, h->ph, U_n, nullptr, df, 0, b.n[2], s));
    h->launches += 1;
    feat = df;
  }
  // the forward of the step from U^n, as the adjoint recomputes it: W0, and
  // stage 1 for W1 (into Yp)
  adj_prims_kernel<<<grid_for(b.nP, blk), blk, 0, s>>>(b, h->ph, U_n, W0);
  set_scalar_kernel<<<1, 1, 0, s>>>(h->dt_slot, dt);
  reset_bits_kernel<<<1, 32, 0, s>>>(h->tsi_bits, 1, h->counters, 4);
  CUDA_TRY(cudaGetLastError());
  h->launches += 3;
  BrickDesc d1 = make_desc(h, U_n, nullptr, nullptr, nullptr, feat, nullptr, h->dt_slot, 0.5,
                           nullptr);
  CUDA_TRY(launch_stage(MODE_STAGE1, false, hllc, grav, d1, nullptr, h->items, h->n_items,
                        h->counters, h->ph, s));
  h->launches += 1;
  CUDA_TRY(cudaMemsetAsync(h->branch_buf, 0, (2 + BR_KINDS) * sizeof(unsigned long long), s));
  AdjDesc A;
  memset(&A, 0, sizeof(A));
  for (int a = 0; a < 3; ++a) {
    A.n[a] = b.n[a];
    A.bc[a][0] = b.bc[a][0];
    A.bc[a][1] = b.bc[a][1];
    A.geo[a] = h->dgeo[a];
  }
  A.nP = b.nP;
  A.df = feat;
  for (int stage = 0; stage < 2; ++stage) {
    A.W = stage == 0 ? W0 : h->Yp;
    if (hllc)
      branch_signature_kernel<true><<<grid_for(b.nP, blk), blk, 0, s>>>(A, h->ph, stage,
                                                                        h->branch_buf);
    else
      branch_signature_kernel<false><<<grid_for(b.nP, blk), blk, 0, s>>>(A, h->ph, stage,
                                                                         h->branch_buf);
    CUDA_TRY(cudaGetLastError());
    h->launches += 1;
  }
  CUDA_TRY(cudaMemcpyAsync(out, h->branch_buf, (2 + BR_KINDS) * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return GFX_OK;
}

}  // extern "C"

// ---- A chart of several bricks on one device --------------------------------
// Chart_SLD (Chart_SLD__Form.f90) splits one domain into equal bricks, one
// per MPI rank, and exchanges the ghost layers of faces and edges between
// them every stage (ExchangeGhostData, :131-201, called for the increment
// from Step_RK_C_ASC__Template.f90:1237-1246).  On one device every brick's
// cells are in the same memory: the chart's stage launches are batched
// launches whose work items span all bricks, and a halo cell across a face
// is read from the neighbouring brick's arrays of the same stage (the
// descriptors of a stage link each brick to the bricks across its faces).
// The chart has one clock and one time step (the MIN all-reduce of the
// time step, Integrator_Template.f90:919, is the one CFL word every brick's
// stage 2 reduces into).
struct gfx_fluid_chart {
  gfx_fluid_config cfg;      // the whole chart
  int nbk[3] = {1, 1, 1};    // bricks per axis
  int n = 0;                 // bricks
  std::vector<gfx_fluid*> h;  // brick b = ix + nbk[0] (iy + nbk[1] iz)
  std::vector<double*> U;     // the bound states
  std::vector<int> links;     // [b][3][2] brick across each face, or -1
  Phys ph;
  bool hllc = false, grav = false;
  BrickDesc *d1 = nullptr, *d1p = nullptr, *d1w = nullptr, *d2 = nullptr;  // device, [n]
  std::vector<BrickDesc> hd1, hd1p, hd1w, hd2;                             // host copies
  ChartBrick* cb = nullptr;
  std::vector<ChartBrick> hcb;
  WorkItem* items = nullptr;
  int n_items = 0;
  long long total_v = 0, total_c = 0;
  unsigned long long* tsi_bits = nullptr;  // [1]
  Clock* clock = nullptr;                  // [2]: the chart's clock, a scratch clock
  int* counters = nullptr;                 // [4]
  ChunkRing ring;                          // the evolve's clock copies between chunks
  int features = FEAT_ZERO;
  bool prims_pending = false;  // the kept primitives are the state (after from_primitive)
  bool wn_valid = false;       // the primitives the last stage 2 stored are the state's
  cudaGraphExec_t graph = nullptr;
  long long graph_kernels = 0, launches = 0;
};

namespace {

__global__ void chart_set_clock_kernel(Clock* c, double dt) {
  c->dt = dt;
  c->done = 0;
}

int chart_upload_descs(gfx_fluid_chart* C, cudaStream_t s) {
  const size_t bytes = C->n * sizeof(BrickDesc);
  CUDA_TRY(cudaMemcpyAsync(C->d1, C->hd1.data(), bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(C->d1p, C->hd1p.data(), bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(C->d1w, C->hd1w.data(), bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(C->d2, C->hd2.data(), bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(C->cb, C->hcb.data(), C->n * sizeof(ChartBrick),
                           cudaMemcpyHostToDevice, s));
  // the host copies may change on the next call: the copies above are staged
  // from pageable memory, finish them before returning
  CUDA_TRY(cudaStreamSynchronize(s));
  return GFX_OK;
}

// The inverse CFL time of every brick's state into the chart's word, and
// the time step of clock dc from it.
int chart_initial_dt(gfx_fluid_chart* C, Clock* dc, int clip, cudaStream_t s) {
  reset_bits_kernel<<<1, 32, 0, s>>>(C->tsi_bits, 1, C->counters, 0);
  for (int b = 0; b < C->n; ++b) {
    gfx_fluid* h = C->h[b];
    inverse_timestep_kernel<<<grid_for(h->box.nP, 256), 256, 0, s>>>(
        h->box, h->ph, C->U[b], C->prims_pending ? h->Pst : nullptr, h->dgeo[0], h->dgeo[1],
        h->dgeo[2], C->tsi_bits);
  }
  finalize_dt_kernel<<<1, 1, 0, s>>>(C->ph, C->tsi_bits, dc, 1, clip);
  CUDA_TRY(cudaGetLastError());
  C->launches += C->n + 2;
  return GFX_OK;
}

// The shock features of the whole chart in one tiled launch, from the
// primitives the last stage 2 stored (from_wn) or from the conserved states.
cudaError_t launch_chart_features(const gfx_fluid_chart* C, bool from_wn, const int* skip,
                                  cudaStream_t s) {
  const Box& b0 = C->h[0]->box;
  Box chart = b0;
  for (int a = 0; a < 3; ++a) chart.n[a] = b0.n[a] * C->nbk[a];
  const dim3 grid = detect_grid(chart, 0, chart.n[2]);
  if (from_wn)
    chart_detect_features_kernel<true><<<grid, kDetThreads, 0, s>>>(C->cb, C->nbk[0], C->nbk[1],
                                                                    C->nbk[2], C->ph, skip);
  else
    chart_detect_features_kernel<false><<<grid, kDetThreads, 0, s>>>(
        C->cb, C->nbk[0], C->nbk[1], C->nbk[2], C->ph, skip);
  return cudaGetLastError();
}

// The launches of one RK2 step of every brick (dt and the skip flag in the
// chart's clock): features (across brick faces), stage 1, stage 2, ghosts.
int enqueue_chart_step(gfx_fluid_chart* C, bool detect, bool from_wn, cudaStream_t s) {
  const int blk = 256;
  const int* skip = &C->clock[0].done;
  reset_bits_kernel<<<1, 32, 0, s>>>(C->tsi_bits, 1, C->counters, 4);
  CUDA_TRY(cudaGetLastError());
  C->launches += 1;
  if (C->hllc && detect) {
    CUDA_TRY(launch_chart_features(C, from_wn, skip, s));
    C->launches += 1;
  }
  const bool in_prim = C->prims_pending || from_wn;
  const BrickDesc* d1 = C->prims_pending ? C->d1p : (from_wn ? C->d1w : C->d1);
  CUDA_TRY(launch_stage_chart(MODE_STAGE1, in_prim, C->hllc, C->grav, d1, C->items, C->n_items,
                              C->counters, C->ph, s));
  CUDA_TRY(launch_stage_chart(MODE_STAGE2, true, C->hllc, C->grav, C->d2, C->items,
                              C->n_items, C->counters + 1, C->ph, s));
  const long long shell = C->total_v - C->total_c;
  chart_ghost_refresh_kernel<<<grid_for(shell, blk), blk, 0, s>>>(C->cb, C->n, shell, C->ph,
                                                                  skip);
  CUDA_TRY(cudaGetLastError());
  C->launches += 3;
  return GFX_OK;
}

HostAxis slice_axis(const HostAxis& g, int o, int m) {
  // entries o .. o + m of the chart's tables: the brick's ghost-inclusive
  // index t is the chart's o + t
  HostAxis a;
  auto cut = [&](const std::vector<double>& v, int len) {
    std::vector<double> r(len, 0.0);
    for (int t = 0; t < len; ++t)
      if (o + t < (int)v.size()) r[t] = v[o + t];
    return r;
  };
  a.X = cut(g.X, m);
  a.WL = cut(g.WL, m);
  a.WR = cut(g.WR, m);
  a.W = cut(g.W, m);
  a.dXI = cut(g.dXI, m + 1);
  a.SQ = cut(g.SQ, m + 1);
  a.CDEN = cut(g.CDEN, m + 1);
  a.RDXI = cut(g.RDXI, m + 1);
  a.RCDEN = cut(g.RCDEN, m + 1);
  a.RW = cut(g.RW, m + 1);
  const int Lg = (int)(g.PAR.size() / PG_N), L = m + 1;
  a.PAR.assign((size_t)PG_N * L, 0.0);
  for (int q = 0; q < PG_N; ++q)
    for (int t = 0; t < L; ++t)
      if (o + t < Lg) a.PAR[(size_t)q * L + t] = g.PAR[(size_t)q * Lg + o + t];
  return a;
}

}  // namespace

extern "C" {

int gfx_fluid_chart_create(const gfx_fluid_config* cfg, const int n_bricks[3],
                           gfx_fluid_chart** out) {
  if (!out || !n_bricks) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) return rc;
  if (cfg->reconstruction != GFX_RECONSTRUCTION_LINEAR)
    return fail(GFX_ERR_UNSUPPORTED, "a chart of bricks: LINEAR reconstruction only");
  int nb[3];
  for (int a = 0; a < 3; ++a) {
    if (n_bricks[a] < 1) return fail(GFX_ERR_ARGUMENT, "n_bricks[%d] = %d", a, n_bricks[a]);
    if (cfg->n_cells[a] % n_bricks[a] != 0)
      return fail(GFX_ERR_ARGUMENT, "axis %d: %d cells do not split into %d equal bricks", a,
                  cfg->n_cells[a], n_bricks[a]);
    nb[a] = cfg->n_cells[a] / n_bricks[a];
    if (nb[a] < 4)
      return fail(GFX_ERR_ARGUMENT, "axis %d: bricks of %d cells; at least 4 per axis", a,
                  nb[a]);
  }
  gfx_fluid_chart* C = new (std::nothrow) gfx_fluid_chart();
  if (!C) return fail(GFX_ERR_NO_MEMORY, "host allocation failed");
  auto cleanup = [&](int code) {
    gfx_fluid_chart_destroy(C);
    return code;
  };
  C->cfg = *cfg;
  for (int a = 0; a < 3; ++a) C->nbk[a] = n_bricks[a];
  C->n = n_bricks[0] * n_bricks[1] * n_bricks[2];
  C->hllc = cfg->riemann_solver == GFX_RIEMANN_HLLC;
  C->grav = cfg->uniform_acceleration != 0.0;
  // the chart's geometry, of which every brick takes its slice
  HostAxis G[3];
  for (int a = 0; a < 3; ++a)
    G[a] = build_axis(cfg->n_cells[a], cfg->min_coordinate[a], cfg->max_coordinate[a], 2);
  C->links.assign((size_t)C->n * 6, -1);
  std::vector<WorkItem> items;
  std::vector<long long> work;
  for (int b = 0; b < C->n; ++b) {
    const int ib[3] = {b % n_bricks[0], (b / n_bricks[0]) % n_bricks[1],
                       b / (n_bricks[0] * n_bricks[1])};
    gfx_fluid_config bc = *cfg;
    HostAxis A[3];
    for (int a = 0; a < 3; ++a) {
      bc.n_cells[a] = nb[a];
      const int o = ib[a] * nb[a];  // the brick's first proper cell in the chart
      A[a] = slice_axis(G[a], o, nb[a] + 4);
      // the brick's extent, for the record (the geometry is the slice)
      bc.min_coordinate[a] = G[a].X[o + 2] - G[a].WL[o + 2];
      bc.max_coordinate[a] = G[a].X[o + nb[a] + 1] + G[a].WR[o + nb[a] + 1];
      const bool first = ib[a] == 0, last = ib[a] == n_bricks[a] - 1;
      const bool per = cfg->boundary[a][0] == GFX_BC_PERIODIC;
      bc.boundary[a][0] = first ? cfg->boundary[a][0] : BC_NEIGHBOR;
      bc.boundary[a][1] = last ? cfg->boundary[a][1] : BC_NEIGHBOR;
      int lo[3] = {ib[0], ib[1], ib[2]}, hi[3] = {ib[0], ib[1], ib[2]};
      lo[a] = first ? n_bricks[a] - 1 : ib[a] - 1;
      hi[a] = last ? 0 : ib[a] + 1;
      auto idx = [&](const int* q) { return q[0] + n_bricks[0] * (q[1] + n_bricks[1] * q[2]); };
      C->links[b * 6 + a * 2 + 0] = (!first || per) ? idx(lo) : -1;
      C->links[b * 6 + a * 2 + 1] = (!last || per) ? idx(hi) : -1;
    }
    gfx_fluid* h = nullptr;
    rc = create_handle(&bc, A, &h);
    if (rc) return cleanup(rc);
    h->chart = C;
    C->h.push_back(h);
    if (b == 0) C->ph = h->ph;
    // work items of 32 x kChartTileY columns, z chunks of 32 planes, longest first
    const int len = std::min(nb[2], 32);
    for (int z = 0; z < nb[2]; z += len)
      for (int y = 0; y < nb[1]; y += kChartTileY)
        for (int x = 0; x < nb[0]; x += TX) {
          items.push_back({b, x, y, z, std::min(nb[2], z + len)});
          work.push_back((long long)std::min(TX, nb[0] - x) * std::min(kChartTileY, nb[1] - y) *
                         (std::min(nb[2], z + len) - z));
        }
  }
  std::vector<int> order(items.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  std::vector<WorkItem> sorted(items.size());
  for (size_t i = 0; i < order.size(); ++i) sorted[i] = items[order[i]];
  C->n_items = (int)sorted.size();
  const size_t n = (size_t)C->n;
  if (!dev_alloc(&C->d1, n * sizeof(BrickDesc)) ||
      !dev_alloc(&C->d1p, n * sizeof(BrickDesc)) ||
      !dev_alloc(&C->d1w, n * sizeof(BrickDesc)) ||
      !dev_alloc(&C->d2, n * sizeof(BrickDesc)) ||
      !dev_alloc(&C->cb, n * sizeof(ChartBrick)) ||
      !dev_alloc(&C->items, sorted.size() * sizeof(WorkItem)) ||
      !dev_alloc(&C->tsi_bits, sizeof(unsigned long long)) ||
      !dev_alloc(&C->clock, 2 * sizeof(Clock)) ||
      !dev_alloc(&C->counters, 4 * sizeof(int)))
    return cleanup(fail(GFX_ERR_NO_MEMORY, "cudaMalloc chart tables"));
  if (cudaMemcpy(C->items, sorted.data(), sorted.size() * sizeof(WorkItem),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(C->clock, 0, 2 * sizeof(Clock)) != cudaSuccess)
    return cleanup(fail(GFX_ERR_CUDA, "copy chart work items"));
  *out = C;
  return GFX_OK;
}

int gfx_fluid_chart_destroy(gfx_fluid_chart* C) {
  if (!C) return GFX_OK;
  if (C->graph) cudaGraphExecDestroy(C->graph);
  for (gfx_fluid* h : C->h) gfx_fluid_destroy(h);
  cudaFree(C->d1);
  cudaFree(C->d1p);
  cudaFree(C->d1w);
  cudaFree(C->d2);
  cudaFree(C->cb);
  cudaFree(C->items);
  cudaFree(C->tsi_bits);
  cudaFree(C->clock);
  cudaFree(C->counters);
  ring_free(C->ring);
  delete C;
  return GFX_OK;
}

int gfx_fluid_chart_n_bricks(const gfx_fluid_chart* C, int* n) {
  if (!C || !n) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *n = C->n;
  return GFX_OK;
}

int gfx_fluid_chart_brick(gfx_fluid_chart* C, int b, gfx_fluid** handle, int* brick_index) {
  if (!C || b < 0 || b >= C->n) return fail(GFX_ERR_ARGUMENT, "brick %d of a chart", b);
  if (handle) *handle = C->h[b];
  if (brick_index) {
    brick_index[0] = b % C->nbk[0];
    brick_index[1] = (b / C->nbk[0]) % C->nbk[1];
    brick_index[2] = b / (C->nbk[0] * C->nbk[1]);
  }
  return GFX_OK;
}

int gfx_fluid_chart_bind(gfx_fluid_chart* C, double* const* U) {
  if (!C || !U) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  for (int b = 0; b < C->n; ++b)
    if (!U[b]) return fail(GFX_ERR_ARGUMENT, "brick %d: NULL state", b);
  C->U.assign(U, U + C->n);
  C->hd1.assign(C->n, BrickDesc());
  C->hd1p.assign(C->n, BrickDesc());
  C->hd1w.assign(C->n, BrickDesc());
  C->hd2.assign(C->n, BrickDesc());
  C->hcb.assign(C->n, ChartBrick());
  C->total_v = C->total_c = 0;
  const double* dt = &C->clock[0].dt;
  const int* skip = &C->clock[0].done;
  for (int b = 0; b < C->n; ++b) {
    gfx_fluid* h = C->h[b];
    const uint8_t* df = C->hllc ? h->df : nullptr;
    BrickDesc* ds[4] = {&C->hd1[b], &C->hd1p[b], &C->hd1w[b], &C->hd2[b]};
    const BrickDesc* dev[4] = {C->d1, C->d1p, C->d1w, C->d2};
    *ds[0] = make_desc(h, U[b], nullptr, nullptr, nullptr, df, nullptr, dt, 0.5, skip);
    *ds[1] = make_desc(h, U[b], nullptr, nullptr, h->Pst, df, nullptr, dt, 0.5, skip);
    *ds[2] = make_desc(h, U[b], nullptr, nullptr, h->wn, df, nullptr, dt, 0.5, skip);
    *ds[3] = make_desc(h, U[b], U[b], nullptr, h->Yp, df, nullptr, dt, 0.5, skip);
    ds[3]->wn = h->wn;
    for (int k = 0; k < 4; ++k) {
      ds[k]->tsi_bits = C->tsi_bits;
      ds[k]->links = dev[k];
      for (int a = 0; a < 3; ++a)
        for (int side = 0; side < 2; ++side) ds[k]->nb[a][side] = C->links[b * 6 + a * 2 + side];
    }
    ChartBrick& c = C->hcb[b];
    memset(&c, 0, sizeof(c));
    c.box = h->box;
    for (int a = 0; a < 3; ++a)
      for (int side = 0; side < 2; ++side) c.nb[a][side] = C->links[b * 6 + a * 2 + side];
    c.U = U[b];
    c.Pst = h->Pst;
    c.wn = h->wn;
    c.df = h->df;
    c.v_off = C->total_v;
    c.c_off = C->total_c;
    C->total_v += h->box.nV;
    C->total_c += h->box.nP;
  }
  if (C->graph) {
    cudaGraphExecDestroy(C->graph);
    C->graph = nullptr;
  }
  C->wn_valid = false;
  return chart_upload_descs(C, nullptr);
}

int gfx_fluid_chart_from_primitive(gfx_fluid_chart* C, const double* const* prim, void* stream) {
  if (!C || !prim) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (C->U.empty()) return fail(GFX_ERR_ARGUMENT, "chart: bind the bricks' states first");
  cudaStream_t s = (cudaStream_t)stream;
  for (int b = 0; b < C->n; ++b) {
    if (!prim[b]) return fail(GFX_ERR_ARGUMENT, "brick %d: NULL primitives", b);
    C->hcb[b].prim = prim[b];
  }
  int rc = chart_upload_descs(C, s);
  if (rc) return rc;
  chart_from_primitive_kernel<<<grid_for(C->total_v, 256), 256, 0, s>>>(C->cb, C->n,
                                                                         C->total_v, C->ph);
  CUDA_TRY(cudaGetLastError());
  C->launches += 1;
  for (int b = 0; b < C->n; ++b) C->hcb[b].prim = nullptr;
  C->prims_pending = true;
  C->wn_valid = false;
  C->features = FEAT_ZERO;
  for (gfx_fluid* h : C->h) CUDA_TRY(cudaMemsetAsync(h->df, 0, (size_t)h->box.nP, s));
  return GFX_OK;
}

int gfx_fluid_chart_set_conserved(gfx_fluid_chart* C, void* stream) {
  if (!C) return fail(GFX_ERR_ARGUMENT, "NULL chart");
  if (C->U.empty()) return fail(GFX_ERR_ARGUMENT, "chart: bind the bricks' states first");
  cudaStream_t s = (cudaStream_t)stream;
  for (int b = 0; b < C->n; ++b) {
    gfx_fluid* h = C->h[b];
    to_primitive_kernel<<<grid_for(h->box.nV, 256), 256, 0, s>>>(h->box, h->ph, C->U[b],
                                                                  nullptr, nullptr);
  }
  CUDA_TRY(cudaGetLastError());
  C->launches += C->n;
  C->prims_pending = false;
  C->wn_valid = false;
  CUDA_TRY(cudaMemsetAsync(&C->clock[0].done, 0, sizeof(int), s));
  if (C->hllc) {
    CUDA_TRY(launch_chart_features(C, false, nullptr, s));
    C->launches += 1;
  }
  C->features = FEAT_VALID;
  return GFX_OK;
}

int gfx_fluid_chart_timestep(gfx_fluid_chart* C, int i_cycle, double* dt_host, void* stream) {
  if (!C || !dt_host) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  if (C->U.empty()) return fail(GFX_ERR_ARGUMENT, "chart: bind the bricks' states first");
  cudaStream_t s = (cudaStream_t)stream;
  Clock c;
  memset(&c, 0, sizeof(c));
  c.cycle = i_cycle;
  c.finish = DBL_MAX;
  c.max_cycle = 0x7fffffff;
  Clock* dc = C->clock + 1;
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  int rc = chart_initial_dt(C, dc, 0, s);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(&c, dc, sizeof(c), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  *dt_host = c.dt;
  return GFX_OK;
}

int gfx_fluid_chart_step(gfx_fluid_chart* C, double dt, double* const* fluence, void* stream) {
  Range range_("Step_RK_C_ASC % Compute (chart)");
  if (!C) return fail(GFX_ERR_ARGUMENT, "NULL chart");
  if (C->U.empty()) return fail(GFX_ERR_ARGUMENT, "chart: bind the bricks' states first");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(GFX_ERR_ARGUMENT, "dt = %g", dt);
  cudaStream_t s = (cudaStream_t)stream;
  if (fluence) {
    for (int b = 0; b < C->n; ++b) {
      C->hd1[b].fluence = C->hd1p[b].fluence = C->hd1w[b].fluence = C->hd2[b].fluence =
          fluence[b];
      if (fluence[b])
        CUDA_TRY(cudaMemsetAsync(fluence[b], 0, sizeof(double) * 36 * C->h[b]->face_size, s));
    }
    int rc = chart_upload_descs(C, s);
    if (rc) return rc;
  }
  chart_set_clock_kernel<<<1, 1, 0, s>>>(C->clock, dt);
  CUDA_TRY(cudaGetLastError());
  C->launches += 1;
  const bool from_wn = C->wn_valid && !C->prims_pending;
  int rc = enqueue_chart_step(C, C->features == FEAT_PENDING, from_wn, s);
  if (fluence) {
    for (int b = 0; b < C->n; ++b)
      C->hd1[b].fluence = C->hd1p[b].fluence = C->hd1w[b].fluence = C->hd2[b].fluence = nullptr;
    int rc2 = chart_upload_descs(C, s);
    if (!rc) rc = rc2;
  }
  if (rc) return rc;
  C->prims_pending = false;
  C->features = FEAT_PENDING;
  C->wn_valid = true;
  return GFX_OK;
}

int gfx_fluid_chart_evolve(gfx_fluid_chart* C, double time, int i_cycle, double finish_time,
                           int n_cycles_max, double* time_out, int* i_cycle_out, void* stream) {
  Range range_("Integrator % Evolve (chart)");
  if (!C) return fail(GFX_ERR_ARGUMENT, "NULL chart");
  if (C->U.empty()) return fail(GFX_ERR_ARGUMENT, "chart: bind the bricks' states first");
  if (n_cycles_max < 0) return fail(GFX_ERR_ARGUMENT, "n_cycles_max < 0");
  cudaStream_t s = (cudaStream_t)stream;
  Clock c;
  memset(&c, 0, sizeof(c));
  c.time = time;
  c.finish = finish_time;
  c.cycle = i_cycle;
  c.max_cycle = (int)std::min<long long>(0x7fffffffLL, (long long)i_cycle + n_cycles_max);
  c.done = !(c.time < c.finish && c.cycle < c.max_cycle);
  Clock* dc = C->clock;
  CUDA_TRY(cudaMemcpyAsync(dc, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  if (!c.done) {
    int rc = chart_initial_dt(C, dc, 1, s);
    if (rc) return rc;
    // the first cycle eagerly (its features and primitives follow the state)
    rc = enqueue_chart_step(C, C->features == FEAT_PENDING, C->wn_valid && !C->prims_pending, s);
    if (rc) return rc;
    advance_clock_kernel<<<1, 1, 0, s>>>(dc, 1);
    finalize_dt_kernel<<<1, 1, 0, s>>>(C->ph, C->tsi_bits, dc, 1, 1);
    CUDA_TRY(cudaGetLastError());
    C->launches += 2;
    C->prims_pending = false;
    C->features = FEAT_PENDING;
    C->wn_valid = true;
    if (!C->graph) {
      cudaStream_t cs;
      CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g;
      const long long before = C->launches;
      CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      int rc2 = enqueue_chart_step(C, true, true, cs);
      advance_clock_kernel<<<1, 1, 0, cs>>>(dc, 1);
      finalize_dt_kernel<<<1, 1, 0, cs>>>(C->ph, C->tsi_bits, dc, 1, 1);
      cudaError_t ce = cudaStreamEndCapture(cs, &g);
      cudaStreamDestroy(cs);
      C->graph_kernels = C->launches - before + 2;
      C->launches = before;
      if (rc2) return rc2;
      if (ce != cudaSuccess) return fail(GFX_ERR_CUDA, "chart graph capture: %s",
                                         cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&C->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess)
        return fail(GFX_ERR_CUDA, "chart graph instantiate: %s", cudaGetErrorString(ce));
    }
    // the remaining cycles in chunks, several in flight (ChunkRing)
    if (int rc3 = ring_init(C->ring)) return rc3;
    if (int rc3 = ring_run(C->ring, C->graph, C->graph_kernels, &C->launches, dc, 1,
                           n_cycles_max, s))
      return rc3;
  }
  CUDA_TRY(cudaMemcpyAsync(&c, dc, sizeof(c), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (time_out) *time_out = c.time;
  if (i_cycle_out) *i_cycle_out = c.cycle;
  return GFX_OK;
}

int gfx_fluid_chart_kernel_launches(const gfx_fluid_chart* C, long long* count) {
  if (!C || !count) return fail(GFX_ERR_ARGUMENT, "NULL argument");
  *count = C->launches;
  return GFX_OK;
}

}  // extern "C"
