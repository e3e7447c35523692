// C ABI and runtime of the B200 FDTD engine (declarations in include/fdtd.h).
//
// Replaces SolverFDTD::solver_run_cu (rfnetwork/core/src/solver.cu:546-1143):
// instead of 48 device arrays and four kernel launches per step on the
// default stream, each simulation keeps its fields double-buffered in an
// x-fastest layout, its coefficients as a 16-bit material index plus a row
// table, and the whole time loop is one kernel launch per step (plus a DFT
// pass every kDftChunk steps), captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/fdtd.h"
#include "fdtd_compile.h"
#include "fdtd_kernels.cuh"
#include "fdtd_adjoint.cuh"
#include "fdtd_nf2ff.cuh"
#include "fdtd_step_stream.cuh"
#include "fdtd_adjoint_stream.cuh"
#include <cudaTypedefs.h>

using namespace rfn;

namespace {

constexpr int kDftChunk = 256;  // steps between DFT accumulation passes
constexpr int kMaxProbes = 1 << 20;
constexpr int kMaxMonitors = 50;  // MAX_MONITORS, rfnetwork/core/inc/solver.h:15

// error text of the calls without a handle, kept per calling thread
thread_local std::string g_error;

struct CudaError {
  cudaError_t code;
  std::string where;
};

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) throw CudaError{e_, #call};             \
  } while (0)

struct ArgError {
  int code;
  std::string msg;
};

// The engine's device memory comes from a stream-ordered pool of its own per
// device that keeps freed blocks (release threshold: never), so the ~1 GB of
// one solve is reused by the next instead of being unmapped and mapped again
// (which otherwise adds a few hundred ms to some solves).
cudaMemPool_t engine_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw ArgError{FDTD_ERR_CUDA, "device index out of range"};
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    CK(cudaMemPoolCreate(&pools[dev], &props));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
  }
  return pools[dev];
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  void alloc(size_t count) {
    free();
    if (count) {
      CK(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), engine_pool(), 0));
      CK(cudaStreamSynchronize(0));  // usable on every stream from here
    }
    n = cap = count;
  }
  // Like alloc, but keeps the allocation when it already holds `count`.
  void reserve(size_t count) {
    if (count > cap) alloc(count);
    n = count;
  }
  void free() {
    if (p) {
      cudaDeviceSynchronize();  // no stream may still use it (cudaFree would wait the same way)
      cudaFreeAsync(p, 0);
      cudaStreamSynchronize(0);
    }
    p = nullptr;
    n = cap = 0;
  }
  ~DevBuf() { free(); }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

struct Monitor {
  int field, axis, position, n_step, n_freq;
  std::vector<float> phase;  // interleaved complex64 rows
  int n_phase_rows;
  int n1, n2;
  size_t out_bytes(int nt) const {
    const size_t plane = size_t(n1) * n2;
    return n_freq ? plane * n_freq * 8 : plane * size_t(nt / n_step + 1) * 4;
  }
};

int threads_for_host() {
  unsigned h = std::thread::hardware_concurrency();
  return int(std::max(1u, std::min(h, 32u)));
}

}  // namespace

// Kernel selection of an engine: the plain-load kernel (one cell per thread)
// or the TMA-pipelined streaming kernel (tile height, plane slots), and the z chunk.
struct KernelConfig {
  int variant = 1;  // 0 plain loads, 1 TMA streaming
  int ty = 0;       // tile height; 0 (with variant 1): autotuned (ty, stages, zchunk)
  int stages = 6;   // streaming: shared-memory plane slots
  int zchunk = 0;   // 0: pick from the grid size
  int one_list = 0; // streaming: every tile through the general instantiation (no plain-tile kernel beside it)
};

// Step-kernel shapes the autotuner times, (variant, tile height, plane slots,
// z chunk, one tile list), and its choices per set of grid sizes
// (process-wide). With one list the plain tiles run in the general kernel's
// interior path: one launch per step instead of two side by side, which can
// pay on grids whose step time is mostly launch and pipeline latency.
constexpr int kTuneCandidates[][5] = {{1, 8, 6, 0, 0}, {1, 8, 8, 0, 0},  {1, 8, 4, 0, 0}, {1, 8, 6, 32, 0},
                                      {1, 12, 4, 0, 0}, {1, 6, 6, 0, 0}, {1, 4, 6, 0, 0}, {1, 4, 6, 16, 0},
                                      {1, 8, 6, 4, 0}, {1, 4, 6, 4, 0},  {1, 8, 6, 0, 1}, {1, 8, 6, 4, 1},
                                      {1, 4, 6, 4, 1}};
using TuneChoice = std::array<int, 5>;
std::mutex g_tune_mutex;
std::map<std::vector<int>, TuneChoice> g_tune_cache;

// RFN_FDTD_ONE_LIST=1: explicit streaming shapes run every tile through the
// general kernel (the autotuner decides this by itself).
int one_list_env() {
  const char* v = std::getenv("RFN_FDTD_ONE_LIST");
  return v && std::atoi(v) != 0 ? 1 : 0;
}

KernelConfig default_config() {
  KernelConfig c;
  if (const char* v = std::getenv("RFN_FDTD_KERNEL"))
    c.variant = std::string(v) == "plain" ? 0 : 1;
  if (const char* v = std::getenv("RFN_FDTD_TY")) c.ty = std::atoi(v);
  if (const char* v = std::getenv("RFN_FDTD_STAGES")) c.stages = std::atoi(v);
  if (const char* v = std::getenv("RFN_FDTD_ZCHUNK")) c.zchunk = std::atoi(v);
  c.one_list = one_list_env();
  return c;
}

struct Engine;

struct fdtd_sim {
  int nx, ny, nz;
  std::vector<float> coef[kNumCoef];
  // borrowed caller arrays (fdtd_set_coefficient_view); null: coef[i] holds a copy
  const float* coef_view[kNumCoef] = {};
  bool have_coef[kNumCoef] = {};
  std::vector<ProbeSpec> probes;
  std::vector<std::vector<float>> probe_values;
  std::vector<Monitor> monitors;
  // DFT specification
  int n_series = 0, n_freq = 0;
  std::vector<int> series_start, term_probe;
  std::vector<double> term_weight, omega;

  // device state (valid when prepared)
  bool compiled = false;
  bool prepared = false;
  int prepared_nt = -1;
  int pitch = 0;
  size_t cells_padded = 0;
  CompiledGrid grid;
  SplitPlan split_plan;         // slab thicknesses and sparse slots of the split cells
  SplitDev split_geo{};         // store geometry (base pointers set when prepared)
  size_t split_buf_pairs = 0;   // split pairs per time buffer (all stores)
  DevBuf<float> fields;        // 2 x 6 field arrays
  DevBuf<float> splits;        // 2 x 12 split arrays (only when split cells exist)
  DevBuf<uint16_t> mat;
  DevBuf<float4> rows;
  DevBuf<int2> cell_probes;
  DevBuf<float> src, rec;
  DevBuf<int> is_src;
  DevBuf<int> d_series_start, d_term_probe;
  DevBuf<double> d_term_weight, d_omega;
  DevBuf<double2> dft_X;
  DevBuf<MonDev> d_mons;
  std::vector<std::unique_ptr<DevBuf<char>>> mon_out;
  std::vector<std::unique_ptr<DevBuf<float2>>> mon_phase;
  SimDev dev{};
  DevBuf<SimDev> d_dev;  // this simulation's descriptor alone (monitor kernel)

  std::unique_ptr<Engine> engine;  // batch of one for fdtd_run
  KernelConfig cfg = default_config();
  cudaStream_t ext_stream = nullptr;
  uint32_t dbg_wait_limit = kStreamWaitLimit;  // fdtd_set_debug
  int dbg_withhold = -1;
  std::string err;
  fdtd_stats stats{};
  int64_t h2d_bytes = 0, d2h_bytes = 0;  // bytes copied over PCIe/C2C by this simulation
  // What the last run kept for a gradient (fdtd_adjoint): adj_mode 1 = state
  // snapshots (fdtd_run_checkpointed), one per segment of ckpt_every steps:
  // the 6 field arrays of the time buffer the segment starts from, then (when
  // allocated) its 12 split arrays; adj_mode 2 = the forward history of the
  // gradient box at every step (fdtd_run_recorded), [nt][9][box cells].
  int adj_mode = 0;
  int ckpt_every = 0;
  int ckpt_nt = -1;
  DevBuf<float> ckpt;
  int adj_box[6] = {0, 0, 0, 0, 0, 0};
  DevBuf<float> hist;
  bool adj_in_batch = false;  // the recorded run was a batch run
  bool use_graph = true;      // fdtd_set_graph
  // table rows given to the cells of one box by fdtd_set_box_coefficients
  // (one per cell, after the compiled rows)
  int base_rows = 0;
  int box_rows_from = -1;
  int box_rows_box[6] = {0, 0, 0, 0, 0, 0};
  int generation = 0;  // bumped whenever device buffers are reallocated
};

int64_t box_cells(const int* b) { return int64_t(b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]); }

// dJ/d(record of probe p at step n), [P][nt], from dJ/dX of the device DFT
// (X_sf = sum over the series' terms (p, w) of w sum_n rec_p[n] e^{-i w_f n};
// with the gradient convention G = dJ/dRe X + i dJ/dIm X this is
// sum over the terms (series, p, w) of w sum_f (Re G_sf cos(w_f n) - Im G_sf sin(w_f n))).
std::vector<float> record_adjoints(const fdtd_sim* s, const double* dJdX, int nt) {
  const int P = int(s->probes.size());
  std::vector<float> radj(size_t(std::max(P, 1)) * nt, 0.f);
  std::vector<double> acc(static_cast<size_t>(nt));
  for (int se = 0; se < s->n_series; ++se) {
    std::fill(acc.begin(), acc.end(), 0.0);
    for (int f = 0; f < s->n_freq; ++f) {
      const double gr = dJdX[(size_t(se) * s->n_freq + f) * 2], gi = dJdX[(size_t(se) * s->n_freq + f) * 2 + 1];
      if (gr == 0.0 && gi == 0.0) continue;
      const double om = s->omega[size_t(f)];
      for (int n = 0; n < nt; ++n) acc[size_t(n)] += gr * std::cos(om * n) - gi * std::sin(om * n);
    }
    for (int t = s->series_start[size_t(se)]; t < s->series_start[size_t(se) + 1]; ++t) {
      const int p = s->term_probe[size_t(t)];
      const double w = s->term_weight[size_t(t)];
      for (int n = 0; n < nt; ++n) radj[size_t(p) * nt + n] += float(w * acc[size_t(n)]);
    }
  }
  return radj;
}

// Host-to-device copy that counts its bytes on the simulation.
void h2d(fdtd_sim* s, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  s->h2d_bytes += int64_t(bytes);
}

void d2h(fdtd_sim* s, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
  s->d2h_bytes += int64_t(bytes);
}

using StreamKernelFn = void (*)(const SimDev*, const StreamTile*, int, int, unsigned*, unsigned, int*, int, int,
                                uint32_t, int);

// One tile height of the streaming step kernel: the general and the
// plain-tile instantiation, and the bytes of its exchange buffers, plane
// slots and split regions.
struct StreamVariant {
  int ty, threads, min_blocks;
  uint32_t xch_bytes, main_bytes, split_bytes;
  StreamKernelFn fn, fn_plain;
};

template <int TY>
StreamVariant stream_variant() {
  using G = StreamGeom<TY>;
  return StreamVariant{TY, G::THREADS, G::MIN_BLOCKS, uint32_t(2 * G::XCH), G::MAIN, G::REGION,
                       &fdtd_step_stream_kernel<TY, false>, &fdtd_step_stream_kernel<TY, true>};
}

const std::vector<StreamVariant>& stream_variants() {
  static const std::vector<StreamVariant> v = {stream_variant<4>(), stream_variant<6>(), stream_variant<8>(),
                                               stream_variant<12>()};
  return v;
}

// The streaming kernel with tile height ty and `stages` plane slots (3..8).
const StreamVariant* find_stream_variant(int ty, int stages) {
  if (stages < 3 || stages > kSlotsMax) return nullptr;
  for (auto& v : stream_variants())
    if (v.ty == ty) return &v;
  return nullptr;
}

// Dynamic shared bytes of a streaming block with (at most) `want` plane
// slots and, when a simulation has split cells, four to six split regions,
// sized for the kernel's resident blocks per SM (or fewer blocks, when three
// plane slots and four regions do not fit beside that many); the slot and
// region counts it fits go to n_main / n_reg.
uint32_t stream_slots(const StreamVariant& v, int want, bool splits, int* n_main, int* n_reg) {
  constexpr uint32_t kSmemPerSm = 233472, kPerBlockReserve = 1024 + 512, kMaxPerBlock = 232448 - 512;
  const uint32_t split_min = splits ? kRegionsMin * v.split_bytes : 0;
  uint32_t budget = 0;
  for (int blocks = v.min_blocks; blocks >= 1; --blocks) {
    budget = std::min(kSmemPerSm / blocks - kPerBlockReserve, kMaxPerBlock) - v.xch_bytes;
    if (budget >= 3 * v.main_bytes + split_min) break;
  }
  if (budget < 3 * v.main_bytes + split_min)
    throw ArgError{FDTD_ERR_LIMIT, "Streaming kernel's plane slots do not fit in shared memory."};
  const uint32_t m = std::min<uint32_t>(uint32_t(std::min(want, kSlotsMax)), (budget - split_min) / v.main_bytes);
  const uint32_t rg = splits ? std::min<uint32_t>(kRegionsMax, (budget - m * v.main_bytes) / v.split_bytes) : 0;
  *n_main = int(std::max<uint32_t>(m, 3));
  *n_reg = int(rg);
  return v.xch_bytes + uint32_t(*n_main) * v.main_bytes + rg * v.split_bytes;
}

// Whether a (variant, tile height, stages) triple names an instantiated kernel.
bool kernel_exists(int variant, int ty, int stages) {
  if (variant == 0) return true;
  if (variant == 1) return ty == 0 || find_stream_variant(ty, stages) != nullptr;
  return false;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) throw ArgError{FDTD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable"};
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tiled tensor map over a field group of simulation s: dims (x, y, z) and,
// for rank 5, (component, buffer) with the given element strides.
// xmul = 2 for the split pairs, whose x rows hold 2 floats per cell.
void encode_map(CUtensorMap* m, const void* base, CUtensorMapDataType type, int elem, const fdtd_sim* s, int rank,
                int box_x, int box_y, int ncomp, size_t comp_stride, size_t buf_stride, int xmul = 1) {
  const cuuint64_t row = cuuint64_t(s->pitch) * xmul;
  const cuuint64_t dims[5] = {row, cuuint64_t(s->ny), cuuint64_t(s->nz), cuuint64_t(ncomp), 2};
  const cuuint64_t strides[4] = {row * elem, row * s->ny * elem,
                                 cuuint64_t(comp_stride) * elem, cuuint64_t(buf_stride) * elem};
  const cuuint32_t box[5] = {cuuint32_t(box_x), cuuint32_t(box_y), 1, cuuint32_t(ncomp), 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = get_encode_fn()(m, type, cuuint32_t(rank), const_cast<void*>(base), dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw ArgError{FDTD_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(int(r))};
}

// Tensor maps of the streaming kernel (box widths of StreamGeom).
void encode_stream_maps(StreamMaps& m, const fdtd_sim* s, int ty) {
  std::memset(&m, 0, sizeof(m));
  const auto F = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const size_t N = s->cells_padded;
  encode_map(&m.E, s->fields.p, F, 4, s, 5, 36, ty + 1, 3, N, 6 * N);
  encode_map(&m.H, s->fields.p + 3 * N, F, 4, s, 5, 40, ty + 2, 3, N, 6 * N);
  if (s->splits.n) {
    // each slab store: x rows of 2 w floats (pairs interleaved), h rows, its
    // depth in planes, 6 pair components, 2 time buffers; boxes of 36 pairs
    // and the E (ty + 1) or H (ty) rows, 3 components
    const SplitDev& g = s->split_geo;
    for (int st = 0; st < 6; ++st) {
      if (!g.comp[st]) continue;
      const cuuint64_t w2 = cuuint64_t(2 * g.w[st]);
      const cuuint64_t dims[5] = {w2, cuuint64_t(g.h[st]), cuuint64_t(g.comp[st] / (int64_t(g.w[st]) * g.h[st])), 6,
                                  2};
      const cuuint64_t strides[4] = {w2 * 4, w2 * g.h[st] * 4, cuuint64_t(g.comp[st]) * 8,
                                     cuuint64_t(s->split_buf_pairs) * 8};
      const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
      for (int k = 0; k < 2; ++k) {
        const cuuint32_t box[5] = {72, cuuint32_t(k == 0 ? ty + 1 : ty), 1, 3, 1};
        CUresult r = get_encode_fn()(k == 0 ? &m.Es[st] : &m.Hs[st], F, 5,
                                     reinterpret_cast<float2*>(s->splits.p) + g.off[st], dims, strides, box, estr,
                                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
          throw ArgError{FDTD_ERR_CUDA, "cuTensorMapEncodeTiled failed for a split store: " + std::to_string(int(r))};
      }
    }
  }
  encode_map(&m.ids, s->mat.p, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, s, 3, 40, ty + 1, 1, 0, 0);
}

// Everything one launch of the streaming kernel needs.
struct StreamClass {
  const StreamVariant* v = nullptr;
  uint32_t ring = 0;                 // dynamic shared bytes: exchange buffers, plane slots, split slots
  int n_main = 0, n_reg = 0;
  std::vector<StreamTile> host_tiles;     // tiles with split-field or probe cells (general kernel)
  std::vector<StreamTile> host_tiles_p;   // plain tiles (plain-tile kernel, beside the general one)
  std::vector<StreamMaps> host_maps;
  DevBuf<StreamMaps> d_maps;
  DevBuf<SimDev> d_sims;
  DevBuf<StreamTile> d_tiles, d_tiles_p;
  DevBuf<unsigned> d_counter;        // tile counters: general list, plain list
  int n_tiles = 0, grid = 0;
  int n_tiles_p = 0, grid_p = 0, n_main_p = 0;
  uint32_t ring_p = 0;
  void reset() {
    v = nullptr;
    ring = ring_p = 0;
    host_tiles.clear();
    host_tiles_p.clear();
    d_tiles_p.free();
    n_tiles_p = grid_p = n_main_p = 0;
    host_maps.clear();
    d_maps.free();
    d_sims.free();
    d_tiles.free();
    d_counter.free();
    n_tiles = grid = 0;
  }
};

struct Engine {
  std::vector<fdtd_sim*> sims;
  KernelConfig cfg;
  StreamClass scls;        // streaming kernel
  DevBuf<SimDev> d_sims;   // plain kernel
  DevBuf<int4> d_tiles;    // plain kernel
  DevBuf<int> d_err;
  int n_tiles = 0;
  int grid = 0;
  int zchunk_used = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t ext_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_nt = -1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t cap_stream = nullptr;                   // box-history captures beside the steps
  cudaEvent_t cap_fork = nullptr, cap_join = nullptr;
  cudaStream_t step_side = nullptr;                    // the plain-tile kernel beside the general one
  cudaEvent_t step_fork = nullptr, step_join = nullptr;
  cudaStream_t rep_stream = nullptr;                   // checkpointed adjoint: segment replays
  cudaEvent_t seg_done[2] = {nullptr, nullptr};        // replay of a segment into history half k & 1 done
  cudaEvent_t seg_free[2] = {nullptr, nullptr};        // its reversal done: the half may be refilled
  int64_t step_launches = 0, dft_launches = 0, adj_launches = 0;
  double adj_ms = 0;
  uint32_t wait_limit = kStreamWaitLimit;  // polls per mbarrier wait of the streaming kernel
  int withhold = -1;                       // test hook: plane the TMA kernels' producers never issue
  bool use_graph = true;  // replay the time loop as a captured CUDA graph
  double last_ms = 0;
  double tune_ms = 0;      // host time of the autotuner's trial runs in the last tiling (0: cached choice)
  int tune_trials = 0;     // candidate shapes it timed
  bool timing_pending = false;

  cudaStream_t stream() const { return ext_stream ? ext_stream : own_stream; }

  void init() {
    if (!own_stream) CK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    if (!ev0) CK(cudaEventCreate(&ev0));
    if (!ev1) CK(cudaEventCreate(&ev1));
    if (!cap_stream) CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    if (!cap_fork) CK(cudaEventCreateWithFlags(&cap_fork, cudaEventDisableTiming));
    if (!cap_join) CK(cudaEventCreateWithFlags(&cap_join, cudaEventDisableTiming));
    if (!rep_stream) {
      // the replays take SMs first as blocks retire; the reversal fills the rest
      int lo = 0, hi = 0;
      CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      CK(cudaStreamCreateWithPriority(&rep_stream, cudaStreamNonBlocking, hi));
    }
    if (!step_side) CK(cudaStreamCreateWithFlags(&step_side, cudaStreamNonBlocking));
    if (!step_fork) CK(cudaEventCreateWithFlags(&step_fork, cudaEventDisableTiming));
    if (!step_join) CK(cudaEventCreateWithFlags(&step_join, cudaEventDisableTiming));
    for (int h = 0; h < 2; ++h) {
      if (!seg_done[h]) CK(cudaEventCreateWithFlags(&seg_done[h], cudaEventDisableTiming));
      if (!seg_free[h]) CK(cudaEventCreateWithFlags(&seg_free[h], cudaEventDisableTiming));
    }
  }
  ~Engine() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (cap_fork) cudaEventDestroy(cap_fork);
    if (cap_join) cudaEventDestroy(cap_join);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    for (int h = 0; h < 2; ++h) {
      if (seg_done[h]) cudaEventDestroy(seg_done[h]);
      if (seg_free[h]) cudaEventDestroy(seg_free[h]);
    }
    if (rep_stream) cudaStreamDestroy(rep_stream);
    if (step_fork) cudaEventDestroy(step_fork);
    if (step_join) cudaEventDestroy(step_join);
    if (step_side) cudaStreamDestroy(step_side);
    if (own_stream) cudaStreamDestroy(own_stream);
  }

  void reset_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_nt = -1;
  }

  void build_tiles() {
    reset_graph();
    int dev = 0, n_sm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    if (!d_err.n) {
      d_err.alloc(1);
      CK(cudaMemset(d_err.p, 0, sizeof(int)));
    }
    if (cfg.variant == 1) {
      if (cfg.ty == 0)
        autotune(n_sm);
      else
        build_stream_tiles(n_sm);
      return;
    }
    // plain kernel: 31 x 7 tiles, z cut into chunks
    std::vector<SimDev> devs;
    for (auto* s : sims) devs.push_back(s->dev);
    const std::vector<int4> tiles = plain_tiles(n_sm, cfg.zchunk, &zchunk_used);
    grid = int(tiles.size());
    d_sims.alloc(devs.size());
    CK(cudaMemcpy(d_sims.p, devs.data(), devs.size() * sizeof(SimDev), cudaMemcpyHostToDevice));
    d_tiles.alloc(tiles.size());
    CK(cudaMemcpy(d_tiles.p, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice));
    n_tiles = int(tiles.size());
  }

  // Tiles of the plain kernel and of the adjoint step kernel: 31 x kTileY
  // columns cut in z chunks, (simulation, x0 | y0 << 16, z0 | z1 << 16, 0),
  // about eight per SM over the whole set of simulations.
  std::vector<int4> plain_tiles(int n_sm, int zchunk, int* zlen_out = nullptr, int tx = kTileX, int ty = kTileY,
                                int per_sm = 8) {
    std::vector<int4> tiles;
    int64_t xy_tiles = 0;
    for (auto* s : sims) xy_tiles += int64_t((s->nx + tx - 1) / tx) * ((s->ny + ty - 1) / ty);
    const int64_t want = int64_t(n_sm) * per_sm;
    for (size_t i = 0; i < sims.size(); ++i) {
      fdtd_sim* s = sims[i];
      int chunks = int(std::max<int64_t>(1, (want + xy_tiles - 1) / std::max<int64_t>(xy_tiles, 1)));
      chunks = std::min(chunks, std::max(1, s->nz / 8));
      const int zlen = zchunk > 0 ? zchunk : (s->nz + chunks - 1) / chunks;
      if (zlen_out) *zlen_out = zlen;
      for (int z0 = 0; z0 < s->nz; z0 += zlen)
        for (int y0 = 0; y0 < s->ny; y0 += ty)
          for (int x0 = 0; x0 < s->nx; x0 += tx) {
            const int z1 = std::min(s->nz, z0 + zlen);
            tiles.push_back(make_int4(int(i), x0 | (y0 << 16), z0 | (z1 << 16), 0));
          }
    }
    return tiles;
  }

  // Picks the streaming kernel's (tile height, plane slots, z chunk) for this
  // set of grids: each candidate runs a few time steps on the simulations
  // themselves (their fields are cleared again by the next run), the fastest
  // is kept and remembered for the same grid sizes.
  void autotune(int n_sm) {
    tune_ms = 0;
    tune_trials = 0;
    std::vector<int> key;
    int nt_min = 1 << 30;
    for (auto* s : sims) {
      key.insert(key.end(), {s->nx, s->ny, s->nz});
      nt_min = std::min(nt_min, s->prepared_nt);
    }
    auto apply = [&](const TuneChoice& c) {
      cfg.variant = c[0];
      cfg.ty = c[1];
      cfg.stages = c[2];
      cfg.zchunk = c[3];
      cfg.one_list = c[4];
    };
    {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        apply(it->second);
        build_stream_tiles(n_sm);
        return;
      }
    }
    const int warm = 2, timed = std::min(8, nt_min - warm);
    TuneChoice best = {kTuneCandidates[0][0], kTuneCandidates[0][1], kTuneCandidates[0][2],
                       kTuneCandidates[0][3], kTuneCandidates[0][4]};
    if (timed >= 2) {
      const auto t0 = std::chrono::steady_clock::now();
      init();
      cudaStream_t st = stream();
      float best_ms = 1e30f;
      for (const auto& cand : kTuneCandidates) {
        apply({cand[0], cand[1], cand[2], cand[3], cand[4]});
        try {
          build_stream_tiles(n_sm);
        } catch (const ArgError& e) {
          if (e.code != FDTD_ERR_LIMIT) throw;
          continue;  // this shape's slots do not fit next to these grids' split slots
        }
        CK(cudaMemsetAsync(scls.d_counter.p, 0, scls.d_counter.n * sizeof(unsigned), st));
        for (int n = 0; n < warm; ++n) launch_step(st, n);
        CK(cudaEventRecord(ev0, st));
        for (int n = warm; n < warm + timed; ++n) launch_step(st, n);
        CK(cudaEventRecord(ev1, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        ++tune_trials;
        if (ms < best_ms) {
          best_ms = ms;
          best = {cand[0], cand[1], cand[2], cand[3], cand[4]};
        }
      }
      check_error();
      tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      g_tune_cache[key] = best;
    }
    apply(best);
    build_stream_tiles(n_sm);
  }

  // Streaming kernel: 31 x TY column tiles cut in z chunks of at most 62
  // planes (cut at the z slabs' inner faces), each with the mask of its
  // planes that hold split-field cells.
  void build_stream_tiles(int n_sm) {
    StreamClass& c = scls;
    c.reset();
    const void* fn = nullptr;
    int threads = 0, smem = 0, ty = 0;
    {
      c.v = find_stream_variant(cfg.ty, cfg.stages);
      if (!c.v) throw ArgError{FDTD_ERR_ARG, "No streaming kernel instantiated for this tile height / stage count."};
      fn = reinterpret_cast<const void*>(c.v->fn);
      threads = c.v->threads;
      bool splits = false;
      for (auto* s : sims) splits = splits || s->splits.n > 0;
      c.ring = stream_slots(*c.v, cfg.stages, splits, &c.n_main, &c.n_reg);
      smem = int(c.ring);
      ty = c.v->ty;
    }
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) throw ArgError{FDTD_ERR_LIMIT, "Step kernel does not fit on an SM."};
    // the plain-tile instantiation: plane slots only
    int per_sm_p = 0;
    {
      int no_regions = 0;
      c.ring_p = stream_slots(*c.v, cfg.stages, false, &c.n_main_p, &no_regions);
      const void* fp = reinterpret_cast<const void*>(c.v->fn_plain);
      CK(cudaFuncSetAttribute(fp, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c.ring_p)));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_p, fp, threads, int(c.ring_p)));
      if (per_sm_p < 1) throw ArgError{FDTD_ERR_LIMIT, "Step kernel does not fit on an SM."};
    }
    int64_t cols = 0;
    for (auto* s : sims) cols += int64_t((s->nx + kStreamOwnX - 1) / kStreamOwnX) * ((s->ny + ty - 1) / ty);
    const int64_t slots = int64_t(per_sm) * n_sm;
    zchunk_used = 1 << 30;
    for (size_t i = 0; i < sims.size(); ++i) {
      fdtd_sim* s = sims[i];
      int zc = cfg.zchunk;
      if (zc <= 0) {
        // about four tiles per resident block
        const int64_t chunks = std::max<int64_t>(1, (slots * 4 + cols - 1) / std::max<int64_t>(cols, 1));
        zc = int((s->nz + chunks - 1) / chunks);
      }
      zc = std::max(1, std::min(zc, 62));
      zchunk_used = std::min(zchunk_used, zc);
      c.host_maps.emplace_back();
      encode_stream_maps(c.host_maps.back(), s, ty);
      const GradedIndex split_idx(s->grid, kFlagESplit | kFlagHSplit);
      // z chunks of at most zc planes that do not straddle a z slab's inner
      // face: the first core chunk starts one plane past the low slab (its
      // halo plane is then a core plane), so interior columns of core chunks
      // are plain tiles
      std::vector<std::pair<int, int>> zr;
      std::vector<int> chunk_of(size_t(s->nz), 0);
      {
        const int* pt = s->split_plan.t;
        const int zlo = pt[4] > 0 ? std::min(s->nz, pt[4] + 1) : 0;
        const int zhi = pt[5] > 0 ? std::max(zlo, s->nz - pt[5]) : s->nz;
        auto cut = [&](int a, int b) {
          for (int z = a; z < b; z += zc) zr.push_back({z, std::min(b, z + zc)});
        };
        cut(0, zlo);
        cut(zlo, zhi);
        cut(zhi, s->nz);
        for (size_t k = 0; k < zr.size(); ++k)
          for (int z = zr[k].first; z < zr[k].second; ++z) chunk_of[size_t(z)] = int(k);
      }
      // tiles (x / 31, y / TY, z chunk) that own a probe cell
      std::unordered_set<int64_t> probe_tiles;
      const int ntx = (s->nx + kStreamOwnX - 1) / kStreamOwnX, nty = (s->ny + ty - 1) / ty;
      for (const int64_t cell : s->grid.probe_cell) {
        const int z = int(cell % s->nz), y = int((cell / s->nz) % s->ny), x = int(cell / (int64_t(s->nz) * s->ny));
        probe_tiles.insert((int64_t(chunk_of[size_t(z)]) * nty + y / ty) * ntx + x / kStreamOwnX);
      }
      for (size_t zk = 0; zk < zr.size(); ++zk)
        for (int y0 = 0; y0 < s->ny; y0 += ty)
          for (int x0 = 0; x0 < s->nx; x0 += kStreamOwnX) {
            const int z0 = zr[zk].first, z1 = zr[zk].second;
            // planes holding split cells in the E region (columns x0-1 .. x0+30, rows y0-1 .. y0+ty-1)
            uint64_t mask = 0;
            for (int j = 0; j < z1 - z0 + 1; ++j) {
              const int z = z0 - 1 + j;
              if (z >= 0 && split_idx.count(x0 - 1, x0 + kStreamOwnX, y0 - 1, y0 + ty, z, z + 1) > 0)
                mask |= uint64_t(1) << j;
            }
            // slab stores the tile's rows and columns reach on planes outside the z slabs
            const int* pt = s->split_plan.t;
            const int zc0 = pt[4], zc1 = s->nz - pt[5];
            int ys = -1, xs = -1;
            if (zc1 > zc0) {
              if (pt[2] > 0 && y0 - 1 < pt[2]) ys = kStYlo;
              else if (pt[3] > 0 && y0 + ty - 1 >= s->ny - pt[3]) ys = kStYhi;
              if (pt[0] > 0 && x0 - 1 < pt[0]) xs = kStXlo;
              else if (pt[1] > 0 && x0 + kStreamOwnX - 1 >= s->nx - pt[1]) xs = kStXhi;
            }
            StreamTile t{};
            t.sim = int(i);
            t.x0 = x0;
            t.y0 = y0;
            t.z0 = z0;
            t.z1 = z1;
            t.ys = ys;
            t.xs = xs;
            t.plain = mask == 0 && !probe_tiles.count((int64_t(zk) * nty + y0 / ty) * ntx + x0 / kStreamOwnX);
            t.split_lo = uint32_t(mask);
            t.split_hi = uint32_t(mask >> 32);
            c.host_tiles.push_back(t);
          }
    }
    // Plain tiles go to the plain-tile kernel, the others to the general one.
    // Persistent blocks take tiles in list order, so the costliest go first
    // and the last tiles taken are short ones: a plane with split-field cells
    // costs about three ordinary planes. Stable, so tiles of equal cost keep
    // their z-chunk-major order and neighbours still share halos in L2.
    {
      std::vector<StreamTile> all;
      all.swap(c.host_tiles);
      for (const auto& t : all) (t.plain && !cfg.one_list ? c.host_tiles_p : c.host_tiles).push_back(t);
    }
    auto cost = [](const StreamTile& t) {
      return (t.z1 - t.z0 + 1) + 2 * (__builtin_popcount(t.split_lo) + __builtin_popcount(t.split_hi));
    };
    for (auto* list : {&c.host_tiles, &c.host_tiles_p})
      std::stable_sort(list->begin(), list->end(),
                       [&](const StreamTile& a, const StreamTile& b) { return cost(a) > cost(b); });
    c.n_tiles = int(c.host_tiles.size());
    c.n_tiles_p = int(c.host_tiles_p.size());
    c.d_maps.alloc(c.host_maps.size());
    CK(cudaMemcpy(c.d_maps.p, c.host_maps.data(), c.host_maps.size() * sizeof(StreamMaps), cudaMemcpyHostToDevice));
    std::vector<SimDev> devs;
    for (size_t i = 0; i < sims.size(); ++i) {
      devs.push_back(sims[i]->dev);
      devs.back().maps = c.d_maps.p + i;
    }
    c.d_sims.alloc(devs.size());
    CK(cudaMemcpy(c.d_sims.p, devs.data(), devs.size() * sizeof(SimDev), cudaMemcpyHostToDevice));
    c.d_tiles.alloc(std::max<size_t>(1, c.host_tiles.size()));
    if (c.n_tiles)
      CK(cudaMemcpy(c.d_tiles.p, c.host_tiles.data(), c.host_tiles.size() * sizeof(StreamTile), cudaMemcpyHostToDevice));
    c.d_tiles_p.alloc(std::max<size_t>(1, c.host_tiles_p.size()));
    if (c.n_tiles_p)
      CK(cudaMemcpy(c.d_tiles_p.p, c.host_tiles_p.data(), c.host_tiles_p.size() * sizeof(StreamTile),
                    cudaMemcpyHostToDevice));
    c.d_counter.alloc(2);
    c.grid = int(std::min<int64_t>(c.n_tiles, slots));
    c.grid_p = int(std::min<int64_t>(c.n_tiles_p, int64_t(per_sm_p) * n_sm));
    n_tiles = c.n_tiles + c.n_tiles_p;
    grid = c.grid + c.grid_p;
  }

  // The streaming kernels of step n (counters counted from step n0, with at
  // most `cap` blocks each): the general kernel on st and the plain-tile
  // kernel beside it on a forked stream, or on st after it when `side` is
  // false.
  int launch_stream_step(cudaStream_t st, int n, int n0, int cap, bool side) {
    StreamClass& c = scls;
    const int g = std::min(c.grid, cap), gp = std::min(c.grid_p, cap);
    const bool fork = side && c.n_tiles > 0 && c.n_tiles_p > 0;
    if (fork) {
      CK(cudaEventRecord(step_fork, st));
      CK(cudaStreamWaitEvent(step_side, step_fork, 0));
    }
    if (c.n_tiles > 0) {
      const unsigned base = unsigned(n - n0) * unsigned(c.n_tiles + g);
      c.v->fn<<<g, c.v->threads, c.ring, st>>>(c.d_sims.p, c.d_tiles.p, c.n_tiles, n, c.d_counter.p, base, d_err.p,
                                                  c.n_main, c.n_reg, wait_limit, withhold);
      CK(cudaGetLastError());
    }
    if (c.n_tiles_p > 0) {
      const unsigned base = unsigned(n - n0) * unsigned(c.n_tiles_p + gp);
      c.v->fn_plain<<<gp, c.v->threads, c.ring_p, fork ? step_side : st>>>(
          c.d_sims.p, c.d_tiles_p.p, c.n_tiles_p, n, c.d_counter.p + 1, base, d_err.p, c.n_main_p, 0, wait_limit,
          withhold);
      CK(cudaGetLastError());
    }
    if (fork) {
      CK(cudaEventRecord(step_join, step_side));
      CK(cudaStreamWaitEvent(st, step_join, 0));
    }
    return int(c.n_tiles > 0) + int(c.n_tiles_p > 0);
  }

  // The kernels of time step n on st; returns how many were launched.
  int launch_step(cudaStream_t st, int n) {
    if (cfg.variant == 1) {
      return launch_stream_step(st, n, 0, 1 << 30, true);
    } else {
      fdtd_step_kernel<kTileY><<<n_tiles, dim3(32, kBlockY), 0, st>>>(d_sims.p, d_tiles.p, n);
      CK(cudaGetLastError());
      return 1;
    }
  }

  // Step n of a checkpointed adjoint's segment replay (segment from step n0),
  // with the streaming kernels on at most `per_sm` blocks per SM each, one
  // after the other, so that the reversal of the next segment, running at the
  // same time on another stream, finds room on every SM. The tile counters
  // were cleared before n0.
  void launch_replay_step(cudaStream_t st, int n, int n0, int n_sm, int per_sm) {
    if (cfg.variant == 1) {
      launch_stream_step(st, n, n0, n_sm * per_sm, false);
    } else {
      launch_step(st, n);
    }
  }

  // Orders the streaming kernels' tile lists for segment replays by the
  // Chebyshev distance (cells) of each tile's owned cells from the gradient
  // box of its simulation (boxes[i] for sims[i]; null: never needed).
  void build_replay_tiles(const std::vector<const int*>& boxes) {
    StreamClass& c = scls;
    auto order = [&](const std::vector<StreamTile>& src, DevBuf<StreamTile>& dst, std::vector<int>& dist) {
      std::vector<std::pair<int, StreamTile>> v;
      v.reserve(src.size());
      for (const auto& t : src) {
        const fdtd_sim* s = sims[size_t(t.sim)];
        const int* b = boxes[size_t(t.sim)];
        if (!b) continue;
        auto gap = [](int a0, int a1, int b0, int b1) { return std::max(0, std::max(a0 - (b1 - 1), b0 - (a1 - 1))); };
        const int x1 = std::min(s->nx, t.x0 + kStreamOwnX), y1 = std::min(s->ny, t.y0 + c.v->ty);
        const int d = std::max(gap(t.x0, x1, b[0], b[1]), std::max(gap(t.y0, y1, b[2], b[3]), gap(t.z0, t.z1, b[4], b[5])));
        v.emplace_back(d, t);
      }
      std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      dist.resize(v.size());
      std::vector<StreamTile> h(v.size());
      for (size_t i = 0; i < v.size(); ++i) {
        dist[i] = v[i].first;
        h[i] = v[i].second;
      }
      dst.reserve(std::max<size_t>(1, h.size()));
      if (!h.empty()) CK(cudaMemcpy(dst.p, h.data(), h.size() * sizeof(StreamTile), cudaMemcpyHostToDevice));
    };
    order(c.host_tiles, rep_tiles, rep_dist);
    order(c.host_tiles_p, rep_tiles_p, rep_dist_p);
  }

  // Step n of a segment replay restricted to the tiles within `reach` cells of
  // the gradient boxes (lists from build_replay_tiles), the general kernel
  // then the plain-tile kernel on st, at most `cap` blocks each; base_g /
  // base_p carry the tile counters' bases from step to step of the segment.
  void launch_replay_subset(cudaStream_t st, int n, int reach, int cap, unsigned& base_g, unsigned& base_p) {
    StreamClass& c = scls;
    const int ng = int(std::upper_bound(rep_dist.begin(), rep_dist.end(), reach) - rep_dist.begin());
    const int np = int(std::upper_bound(rep_dist_p.begin(), rep_dist_p.end(), reach) - rep_dist_p.begin());
    if (ng > 0) {
      const int g = std::min(std::min(c.grid, cap), ng);
      c.v->fn<<<g, c.v->threads, c.ring, st>>>(c.d_sims.p, rep_tiles.p, ng, n, c.d_counter.p, base_g, d_err.p,
                                                  c.n_main, c.n_reg, wait_limit, withhold);
      CK(cudaGetLastError());
      base_g += unsigned(ng + g);
    }
    if (np > 0) {
      const int g = std::min(std::min(c.grid_p, cap), np);
      c.v->fn_plain<<<g, c.v->threads, c.ring_p, st>>>(c.d_sims.p, rep_tiles_p.p, np, n, c.d_counter.p + 1, base_p,
                                                        d_err.p, c.n_main_p, 0, wait_limit, withhold);
      CK(cudaGetLastError());
      base_p += unsigned(np + g);
    }
  }

  // Box-history capture of the simulations in recorded mode (adj_mode 2):
  // one adj_capture_kernel launch per time step, before the step, inside the
  // captured time loop.
  DevBuf<CapSim> d_caps;
  int n_caps = 0, cap_blocks = 1;

  void build_caps() {
    std::vector<CapSim> v;
    int64_t nb_max = 0;
    for (auto* s : sims)
      if (s->adj_mode == 2) {
        CapSim c{};
        c.s = s->dev;
        c.bx0 = s->adj_box[0]; c.bx1 = s->adj_box[1]; c.by0 = s->adj_box[2];
        c.by1 = s->adj_box[3]; c.bz0 = s->adj_box[4]; c.bz1 = s->adj_box[5];
        c.nb = box_cells(s->adj_box);
        c.hist = s->hist.p;
        nb_max = std::max(nb_max, c.nb);
        v.push_back(c);
      }
    n_caps = int(v.size());
    d_caps.alloc(v.size());
    if (!v.empty()) CK(cudaMemcpy(d_caps.p, v.data(), v.size() * sizeof(CapSim), cudaMemcpyHostToDevice));
    cap_blocks = int(std::min<int64_t>(1024, std::max<int64_t>(1, (nb_max + 255) / 256)));
  }

  // Adjoint work buffers of each request slot, kept between sweeps.
  struct AdjBufs {
    DevBuf<float> lam, lams, radj, seg;
    DevBuf<float> rec_save;  // the forward's probe records, kept while segment replays rewrite them
    DevBuf<int> pidx, pfld;
    DevBuf<double> grad;
  };
  // Segment replays of a checkpointed adjoint (streaming kernels): the general
  // and plain tile lists ordered by each tile's distance from its simulation's
  // gradient box, nearest first, with those distances (cells).
  DevBuf<StreamTile> rep_tiles, rep_tiles_p;
  std::vector<int> rep_dist, rep_dist_p;
  std::vector<std::unique_ptr<AdjBufs>> adj_bufs;
  DevBuf<AdjSim> adj_d_as;
  DevBuf<int4> adj_d_t;
  DevBuf<CapSim> adj_d_c;
  DevBuf<AdjMaps> adj_d_maps;     // streaming reverse step: tensor maps of each simulation's adjoint state
  DevBuf<int4> adj_d_ts;          // its tiles (w: the tile's boxes hold split cells)
  DevBuf<unsigned> adj_counter;   // its tile counter
  static int adj_tiles_per_sm() {
    const char* v = std::getenv("RFN_ADJ_TILES_PER_SM");
    return v ? std::max(1, std::atoi(v)) : 4;
  }
  // planes per tile along z (0: picked by adj_pick_zchunk)
  static int adj_zchunk() {
    const char* v = std::getenv("RFN_ADJ_ZCHUNK");
    return v ? std::max(0, std::atoi(v)) : 0;
  }
  // Planes per reverse-step tile along z when `slots` blocks of tx x ty tiles
  // are resident at once: the tiles should fill whole waves of blocks (a short
  // last wave leaves SMs idle) and load few halo planes (two per tile). Picks
  // the largest (tiles / (waves * slots)) * (owned planes / loaded planes)
  // over chunks of 4 planes or more that give at least two waves; 4 planes
  // when even those give fewer.
  // Planes per tile for the persistent reverse step on `slots` blocks: the
  // longest even chunks (nz_max / c planes, c = 1, 2, ...) that still give
  // at least 15/16 of the blocks a tile; 4 planes when none do.
  int adj_pick_zchunk_persistent(int64_t slots, int tx, int ty) const {
    int nz_max = 0;
    for (auto* s : sims) nz_max = std::max(nz_max, s->nz);
    for (int c = 1; c <= nz_max / 4; ++c) {
      const int zl = (nz_max + c - 1) / c;
      int64_t tiles = 0;
      for (auto* s : sims) tiles += int64_t((s->nx + tx - 1) / tx) * ((s->ny + ty - 1) / ty) * ((s->nz + zl - 1) / zl);
      if (16 * tiles >= 15 * slots) return zl;
    }
    return 4;
  }
  int adj_pick_zchunk(int64_t slots, int tx, int ty) const {
    int nz_max = 0;
    int64_t owned = 0;  // tile columns x planes
    for (auto* s : sims) {
      nz_max = std::max(nz_max, s->nz);
      owned += int64_t((s->nx + tx - 1) / tx) * ((s->ny + ty - 1) / ty) * s->nz;
    }
    double best = -1.0;
    int pick = 4;
    for (int zl = 4; zl <= nz_max; ++zl) {
      int64_t tiles = 0;
      for (auto* s : sims) tiles += int64_t((s->nx + tx - 1) / tx) * ((s->ny + ty - 1) / ty) * ((s->nz + zl - 1) / zl);
      const int64_t waves = (tiles + slots - 1) / slots;
      if (waves < 2) break;  // the tile count only falls as the chunks grow
      const double score = double(tiles) / double(waves * slots) * double(owned) / double(owned + 2 * tiles);
      if (score > best + 1e-12) {
        best = score;
        pick = zl;
      }
    }
    return pick;
  }

  // One simulation's part of an adjoint sweep: dJ/dX of its device DFT, the
  // gradient box, and where the [9][box cells] gradient goes.
  struct AdjRequest {
    fdtd_sim* s;
    const double* dJdX;
    const int* box;
    double* grad_out;
  };

  // Discrete adjoint of the last run of the simulations of this engine, all
  // made for a gradient in the same mode (adj_mode of the first): gradient of
  // J with respect to (Ca, Cb1, Cb2) of each E component on each box. The
  // adjoint state runs backwards from step nt-1 with one adj_step_kernel
  // launch per step over the tiles of all simulations. In recorded mode the
  // box history of every step is already on the device. With checkpoints the
  // run is replayed segment by segment, last segment first, capturing each
  // segment's box history into one half of a two-segment buffer; the replay
  // of segment k-1 (its own stream) runs while segment k is reversed.
  void adjoint(const std::vector<AdjRequest>& req) {
    init();
    cudaStream_t st = stream();
    const int mode = req[0].s->adj_mode;
    const int nt = req[0].s->ckpt_nt, K = mode == 1 ? req[0].s->ckpt_every : nt;
    int dev = 0, n_sm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    // work buffers are kept on the engine between sweeps (allocation and
    // release of ~36 floats per cell would otherwise come with every gradient)
    if (adj_bufs.size() < req.size()) adj_bufs.resize(req.size());
    std::vector<AdjSim> as(req.size());
    std::vector<CapSim> caps;
    int64_t nb_max = 0;
    int p_max = 0;
    for (size_t i = 0; i < req.size(); ++i) {
      fdtd_sim* s = req[i].s;
      const int* box = req[i].box;
      if (!adj_bufs[i]) adj_bufs[i] = std::make_unique<AdjBufs>();
      AdjBufs* B = adj_bufs[i].get();
      const size_t N = s->cells_padded;
      const int64_t nb = box_cells(box);
      nb_max = std::max(nb_max, nb);
      const int P = int(s->probes.size());
      p_max = std::max(p_max, P);
      const std::vector<float> radj = record_adjoints(s, req[i].dJdX, nt);
      std::vector<int> pidx(size_t(std::max(P, 1)), 0), pfld(size_t(std::max(P, 1)), 0);
      for (int pr = 0; pr < P; ++pr) {
        const int64_t cell = s->grid.probe_cell[size_t(pr)];
        const int z = int(cell % s->nz), y = int((cell / s->nz) % s->ny), x = int(cell / (int64_t(s->nz) * s->ny));
        pidx[size_t(pr)] = z * s->ny * s->pitch + y * s->pitch + x;
        pfld[size_t(pr)] = s->probes[size_t(pr)].field;
      }
      B->lam.reserve(12 * N);
      CK(cudaMemsetAsync(B->lam.p, 0, 12 * N * sizeof(float), st));
      if (s->splits.n) {
        B->lams.reserve(24 * N);
        CK(cudaMemsetAsync(B->lams.p, 0, 24 * N * sizeof(float), st));
      }
      B->radj.reserve(radj.size());
      CK(cudaMemcpy(B->radj.p, radj.data(), radj.size() * sizeof(float), cudaMemcpyHostToDevice));
      B->pidx.reserve(pidx.size());
      CK(cudaMemcpy(B->pidx.p, pidx.data(), pidx.size() * sizeof(int), cudaMemcpyHostToDevice));
      B->pfld.reserve(pfld.size());
      CK(cudaMemcpy(B->pfld.p, pfld.data(), pfld.size() * sizeof(int), cudaMemcpyHostToDevice));
      B->grad.reserve(9 * size_t(nb));
      CK(cudaMemsetAsync(B->grad.p, 0, 9 * size_t(nb) * sizeof(double), st));
      AdjSim& a = as[i];
      a = AdjSim{};
      a.nx = s->nx; a.ny = s->ny; a.nz = s->nz; a.pitch = s->pitch; a.plane = s->ny * s->pitch; a.nt = nt;
      a.mat = s->mat.p;
      a.rows = s->rows.p;
      a.cell_probes = s->cell_probes.p;
      a.N = int64_t(N);
      a.lam = B->lam.p;
      a.lams = B->lams.p;
      a.radj = B->radj.p;
      a.probe_idx = B->pidx.p;
      a.probe_field = B->pfld.p;
      a.n_probes = P;
      a.bx0 = box[0]; a.bx1 = box[1]; a.by0 = box[2]; a.by1 = box[3]; a.bz0 = box[4]; a.bz1 = box[5];
      a.nb = nb;
      a.grad = B->grad.p;
      if (mode == 2) {
        a.hist = s->hist.p;
      } else {
        B->seg.reserve(2 * size_t(K) * 9 * size_t(nb));
        a.hist = B->seg.p;
        CapSim c{};
        c.s = s->dev;
        c.bx0 = box[0]; c.bx1 = box[1]; c.by0 = box[2]; c.by1 = box[3]; c.bz0 = box[4]; c.bz1 = box[5];
        c.nb = nb;
        c.hist = B->seg.p;
        caps.push_back(c);
      }
    }
    int plain_per_sm = 2;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&plain_per_sm, &adj_step_kernel<kAdjTileY, 2>,
                                                     32 * (kAdjTileY + 2), 0));
    const int zc = adj_zchunk() ? adj_zchunk()
                   : std::getenv("RFN_ADJ_TILES_PER_SM")
                       ? 0
                       : adj_pick_zchunk(int64_t(std::max(plain_per_sm, 1)) * n_sm, kAdjTileX, kAdjTileY);
    const std::vector<int4> tiles = plain_tiles(n_sm, zc, nullptr, kAdjTileX, kAdjTileY, adj_tiles_per_sm());
    // The streaming reverse step, on request (RFN_ADJ_STREAM=1; the plain one
    // is the default): tiles (split tiles first), tensor maps of each
    // simulation's adjoint state and material index, plane slots sized for
    // two blocks per SM.
    using AG = AdjGeom<kAdjStreamTileY>;
    const char* sv = std::getenv("RFN_ADJ_STREAM");
    const bool stream_adj = sv && std::atoi(sv) != 0;
    int n_ts = 0, adj_grid = 0, adj_slots = 0;
    uint32_t adj_smem = 0;
    unsigned adj_base = 0;
    if (stream_adj) {
      constexpr uint32_t kBudget = 233472 / 2 - 1024 - 512 - 9600;  // two blocks per SM, beside the static arrays
      adj_slots = int(std::min<uint32_t>(kAdjStreamSlotsMax, kBudget / AG::SLOT));
      if (adj_slots < 3) throw ArgError{FDTD_ERR_LIMIT, "Streaming reverse step's plane slots do not fit."};
      adj_smem = uint32_t(adj_slots) * AG::SLOT;
      const void* fn = reinterpret_cast<const void*>(&adj_stream_kernel<kAdjStreamTileY>);
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(adj_smem)));
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, AG::THREADS, int(adj_smem)));
      if (per_sm < 1) throw ArgError{FDTD_ERR_LIMIT, "Streaming reverse step does not fit on an SM."};
      const int zcs = adj_zchunk() ? adj_zchunk()
                      : std::getenv("RFN_ADJ_TILES_PER_SM")
                          ? 0
                          : adj_pick_zchunk_persistent(int64_t(per_sm) * n_sm, kAdjTileX, kAdjStreamTileY);
      std::vector<int4> ts = plain_tiles(n_sm, zcs, nullptr, kAdjTileX, kAdjStreamTileY, adj_tiles_per_sm());
      std::vector<GradedIndex> gis;
      for (const auto& rq : req) gis.emplace_back(rq.s->grid, kFlagESplit | kFlagHSplit);
      for (auto& t : ts) {
        // the boxes of every plane of the tile: columns x0-1 .. x0+30, rows y0-1 .. y0+TY, planes z0-1 .. z1
        const int x0 = t.y & 0xffff, y0 = int(unsigned(t.y) >> 16), z0 = t.z & 0xffff, z1 = int(unsigned(t.z) >> 16);
        t.w = gis[size_t(t.x)].count(x0 - 1, x0 + kAdjTileX + 1, y0 - 1, y0 + kAdjStreamTileY + 1, z0 - 1, z1 + 1) > 0;
      }
      std::stable_sort(ts.begin(), ts.end(), [](const int4& a, const int4& b) { return a.w > b.w; });
      n_ts = int(ts.size());
      std::vector<AdjMaps> hm(req.size());
      for (size_t i = 0; i < req.size(); ++i) {
        fdtd_sim* s = req[i].s;
        const size_t N = s->cells_padded;
        std::memset(&hm[i], 0, sizeof(AdjMaps));
        const auto F = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        float* lam = adj_bufs[i]->lam.p;
        encode_map(&hm[i].lam_e, lam, F, 4, s, 5, AG::EW, AG::ER, 3, N, 6 * N);
        encode_map(&hm[i].lam_h, lam + 3 * N, F, 4, s, 5, AG::HW, AG::HR, 3, N, 6 * N);
        if (s->splits.n) encode_map(&hm[i].halves, adj_bufs[i]->lams.p, F, 4, s, 5, AG::SW, AG::HR, 12, N, 12 * N);
        encode_map(&hm[i].ids, s->mat.p, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, s, 3, AG::IW, AG::HR, 1, 0, 0);
      }
      adj_d_maps.reserve(hm.size());
      CK(cudaMemcpy(adj_d_maps.p, hm.data(), hm.size() * sizeof(AdjMaps), cudaMemcpyHostToDevice));
      adj_d_ts.reserve(ts.size());
      CK(cudaMemcpy(adj_d_ts.p, ts.data(), ts.size() * sizeof(int4), cudaMemcpyHostToDevice));
      adj_grid = int(std::min<int64_t>(n_ts, int64_t(per_sm) * n_sm));
      adj_counter.reserve(1);
      CK(cudaMemsetAsync(adj_counter.p, 0, sizeof(unsigned), st));
    }
    auto reverse_step = [&](int n, int hist_n0) {
      if (stream_adj) {
        adj_stream_kernel<kAdjStreamTileY><<<adj_grid, AG::THREADS, adj_smem, st>>>(
            adj_d_as.p, adj_d_maps.p, adj_d_ts.p, n_ts, n, hist_n0, adj_counter.p, adj_base, d_err.p, adj_slots,
            wait_limit);
        adj_base += unsigned(n_ts + adj_grid);
      } else {
        // register cap: two resident blocks per SM (default) or three
        const char* mb = std::getenv("RFN_ADJ_MINB");
        auto adj_fn = (mb && std::atoi(mb) == 3) ? &adj_step_kernel<kAdjTileY, 3> : &adj_step_kernel<kAdjTileY, 2>;
        adj_fn<<<int(tiles.size()), dim3(32, kAdjTileY + 2), 0, st>>>(adj_d_as.p, adj_d_t.p, n, hist_n0);
      }
      CK(cudaGetLastError());
      ++adj_launches;
    };
    DevBuf<AdjSim>& d_as = adj_d_as;
    DevBuf<int4>& d_t = adj_d_t;
    DevBuf<CapSim>& d_c = adj_d_c;
    d_as.reserve(as.size());
    CK(cudaMemcpy(d_as.p, as.data(), as.size() * sizeof(AdjSim), cudaMemcpyHostToDevice));
    d_t.reserve(tiles.size());
    CK(cudaMemcpy(d_t.p, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice));
    if (!caps.empty()) {
      d_c.reserve(caps.size());
      CK(cudaMemcpy(d_c.p, caps.data(), caps.size() * sizeof(CapSim), cudaMemcpyHostToDevice));
    }
    const int cap_grid = int(std::min<int64_t>(1024, std::max<int64_t>(1, (nb_max + 255) / 256)));
    if (p_max > 0) {
      adj_inject_kernel<<<dim3((p_max + 127) / 128, unsigned(as.size())), 128, 0, st>>>(d_as.p, nt - 1,
                                                                                        (nt - 1) & 1);
      CK(cudaGetLastError());
    }
    adj_launches = 0;
    CK(cudaEventRecord(ev0, st));
    if (mode == 2) {
      for (int n = nt - 1; n >= 0; --n) reverse_step(n, 0);
    } else {
      const int nseg = (nt + K - 1) / K;
      const char* rb = std::getenv("RFN_REPLAY_BLOCKS_PER_SM");
      const int per_sm = rb ? std::max(1, std::atoi(rb)) : 1;
      cudaStream_t rs = rep_stream;
      // The history of step n is the state before step n, so a segment
      // [n0, n1) replays steps n0 .. n1-2 only. The history reads the box and
      // the H values one cell beyond it (the +1 neighbours of the E update's
      // differences), and a step moves information by at most one cell along
      // each axis, so step n needs to be right only within n1-1-n cells of the
      // box: with the streaming kernels each replay step runs the tiles within
      // that reach (nearest first). Tiles outside it keep stale values, which
      // never reach what the history reads before the segment ends.
      const bool cone = cfg.variant == 1 && !std::getenv("RFN_REPLAY_FULL");
      if (cone) {
        std::vector<const int*> boxes(sims.size(), nullptr);
        for (const auto& r : req)
          for (size_t i = 0; i < sims.size(); ++i)
            if (sims[i] == r.s) boxes[i] = r.box;
        build_replay_tiles(boxes);
      }
      // the replays rewrite probe records (outside the reach, with stale
      // values): the forward's records are kept aside and put back at the end
      for (size_t i = 0; i < req.size(); ++i) {
        fdtd_sim* s = req[i].s;
        adj_bufs[i]->rec_save.reserve(s->rec.n);
        CK(cudaMemcpyAsync(adj_bufs[i]->rec_save.p, s->rec.p, s->rec.n * sizeof(float), cudaMemcpyDeviceToDevice, st));
      }
      // segment k replayed on rs from its snapshot into history half k & 1,
      // each step's box capture beside it (as in a recorded run)
      auto replay = [&](int k) {
        const int n0 = k * K, n1 = std::min(nt, n0 + K), h0 = n0 - (k & 1) * K;
        const size_t b = size_t(n0 & 1);
        for (const auto& r : req) {
          fdtd_sim* s = r.s;
          const size_t N = s->cells_padded;
          const size_t sb = s->splits.n ? 2 * s->split_buf_pairs : 0;  // split floats per time buffer
          const size_t stride = 6 * N + sb;
          const float* src = s->ckpt.p + size_t(k) * stride;
          CK(cudaMemcpyAsync(s->fields.p + b * 6 * N, src, 6 * N * sizeof(float), cudaMemcpyDeviceToDevice, rs));
          if (sb)
            CK(cudaMemcpyAsync(s->splits.p + b * sb, src + 6 * N, sb * sizeof(float), cudaMemcpyDeviceToDevice, rs));
        }
        if (cfg.variant == 1) CK(cudaMemsetAsync(scls.d_counter.p, 0, scls.d_counter.n * sizeof(unsigned), rs));
        unsigned base_g = 0, base_p = 0;
        for (int n = n0; n < n1; ++n) {
          CK(cudaEventRecord(cap_fork, rs));
          CK(cudaStreamWaitEvent(cap_stream, cap_fork, 0));
          adj_capture_kernel<<<dim3(cap_grid, unsigned(caps.size())), 256, 0, cap_stream>>>(d_c.p, n, h0);
          CK(cudaGetLastError());
          CK(cudaEventRecord(cap_join, cap_stream));
          if (n + 1 < n1) {
            if (cone)
              launch_replay_subset(rs, n, n1 - 1 - n, n_sm * per_sm, base_g, base_p);
            else
              launch_replay_step(rs, n, n0, n_sm, per_sm);
          }
          CK(cudaStreamWaitEvent(rs, cap_join, 0));
        }
        CK(cudaEventRecord(seg_done[k & 1], rs));
      };
      CK(cudaEventRecord(cap_fork, st));  // the replays start after this sweep's set-up on st
      CK(cudaStreamWaitEvent(rs, cap_fork, 0));
      replay(nseg - 1);
      for (int k = nseg - 1; k >= 0; --k) {
        if (k >= 1) {
          // history half (k-1) & 1 was last read by the reversal of segment k+1
          if (k + 1 < nseg) CK(cudaStreamWaitEvent(rs, seg_free[(k + 1) & 1], 0));
          replay(k - 1);
        }
        const int n0 = k * K, n1 = std::min(nt, n0 + K);
        CK(cudaStreamWaitEvent(st, seg_done[k & 1], 0));
        for (int n = n1 - 1; n >= n0; --n) reverse_step(n, n0 - (k & 1) * K);
        CK(cudaEventRecord(seg_free[k & 1], st));
      }
      for (size_t i = 0; i < req.size(); ++i) {
        fdtd_sim* s = req[i].s;
        CK(cudaMemcpyAsync(s->rec.p, adj_bufs[i]->rec_save.p, s->rec.n * sizeof(float), cudaMemcpyDeviceToDevice, st));
      }
    }
    CK(cudaEventRecord(ev1, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    adj_ms = ms;
    check_error();
    for (size_t i = 0; i < req.size(); ++i)
      CK(cudaMemcpy(req[i].grad_out, adj_bufs[i]->grad.p, adj_bufs[i]->grad.n * sizeof(double),
                    cudaMemcpyDeviceToHost));
  }

  // Enqueue one full run of nt steps on stream st (used for capture and for
  // direct launches alike).
  void enqueue(cudaStream_t st, int nt) {
    step_launches = dft_launches = 0;
    for (auto* s : sims) {
      CK(cudaMemsetAsync(s->fields.p, 0, s->fields.n * sizeof(float), st));
      if (s->splits.n) CK(cudaMemsetAsync(s->splits.p, 0, s->splits.n * sizeof(float), st));
      if (s->dft_X.n) CK(cudaMemsetAsync(s->dft_X.p, 0, s->dft_X.n * sizeof(double2), st));
      for (size_t m = 0; m < s->monitors.size(); ++m)
        CK(cudaMemsetAsync(s->mon_out[m]->p, 0, s->mon_out[m]->n, st));
    }
    if (scls.d_counter.n) CK(cudaMemsetAsync(scls.d_counter.p, 0, scls.d_counter.n * sizeof(unsigned), st));
    int dft_from = 0;
    for (int n = 0; n < nt; ++n) {
      for (auto* s : sims)
        if (s->ckpt_every > 0 && n % s->ckpt_every == 0 && s->ckpt.n) {
          const size_t N = s->cells_padded, b = size_t(n & 1);
          const size_t sb = s->splits.n ? 2 * s->split_buf_pairs : 0;  // split floats per time buffer
          const size_t stride = 6 * N + sb;
          float* dst = s->ckpt.p + size_t(n / s->ckpt_every) * stride;
          CK(cudaMemcpyAsync(dst, s->fields.p + b * 6 * N, 6 * N * sizeof(float), cudaMemcpyDeviceToDevice, st));
          if (sb)
            CK(cudaMemcpyAsync(dst + 6 * N, s->splits.p + b * sb, sb * sizeof(float), cudaMemcpyDeviceToDevice, st));
        }
      if (n_caps) {
        // the box history of step n reads buffer n & 1, which step n only
        // reads and step n+1 overwrites: it runs on a side stream beside step n
        CK(cudaEventRecord(cap_fork, st));
        CK(cudaStreamWaitEvent(cap_stream, cap_fork, 0));
        adj_capture_kernel<<<dim3(cap_blocks, unsigned(n_caps)), 256, 0, cap_stream>>>(d_caps.p, n, 0);
        CK(cudaGetLastError());
        CK(cudaEventRecord(cap_join, cap_stream));
      }
      step_launches += launch_step(st, n);
      if (n_caps) CK(cudaStreamWaitEvent(st, cap_join, 0));
      for (auto* s : sims)
        if (!s->monitors.empty()) {
          monitor_kernel<<<64, 256, 0, st>>>(s->d_dev.p, s->d_mons.p, int(s->monitors.size()), n, (n + 1) & 1);
          CK(cudaGetLastError());
        }
      if ((n + 1) % kDftChunk == 0 || n + 1 == nt) {
        for (auto* s : sims)
          if (s->n_series > 0 && s->n_freq > 0) {
            DftDev d{s->n_series, s->n_freq, nt, s->d_series_start.p, s->d_term_probe.p, s->d_term_weight.p,
                     s->d_omega.p, s->rec.p, s->dft_X.p};
            dft_accumulate_kernel<<<dim3(s->n_freq, s->n_series), 256, 0, st>>>(d, dft_from, n + 1);
            CK(cudaGetLastError());
            ++dft_launches;
          }
        dft_from = n + 1;
      }
    }
    // sentinel: a diverged run ends with non-finite records or fields
    for (auto* s : sims) {
      const int64_t nrec = int64_t(s->probes.size()) * nt;
      if (nrec > 0) {
        nonfinite_check_kernel<<<int(std::min<int64_t>(256, (nrec + 255) / 256)), 256, 0, st>>>(s->rec.p, nrec,
                                                                                              d_err.p);
        CK(cudaGetLastError());
      }
      const size_t b = size_t(nt & 1) * 6 * s->cells_padded;  // buffer the last step wrote
      nonfinite_check_kernel<<<296, 256, 0, st>>>(s->fields.p + b, int64_t(6 * s->cells_padded), d_err.p);
      CK(cudaGetLastError());
    }
  }

  void run_async(int nt) {
    init();
    cudaStream_t st = stream();
    if (!use_graph) {  // every launch issued from the host, step by step
      reset_graph();
      build_caps();
      CK(cudaEventRecord(ev0, st));
      enqueue(st, nt);
      CK(cudaEventRecord(ev1, st));
      timing_pending = true;
      return;
    }
    if (graph_nt != nt) {
      reset_graph();
      build_caps();
      cudaStream_t cap;
      CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cudaGraph_t g = nullptr;
      try {
        CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        enqueue(cap, nt);
        CK(cudaStreamEndCapture(cap, &g));
        CK(cudaGraphInstantiate(&graph, g, 0));
      } catch (...) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(cap, &dummy);
        if (dummy) cudaGraphDestroy(dummy);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        throw;
      }
      cudaGraphDestroy(g);
      cudaStreamDestroy(cap);
      graph_nt = nt;
    }
    CK(cudaEventRecord(ev0, st));
    CK(cudaGraphLaunch(graph, st));
    CK(cudaEventRecord(ev1, st));
    timing_pending = true;
  }

  void sync() {
    CK(cudaStreamSynchronize(stream()));
    if (timing_pending) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      last_ms = ms;
      timing_pending = false;
    }
    check_error();
  }

  // Reads (and clears) the error code the kernels record: a bounded wait that
  // expired, or the end-of-run sentinel's non-finite value.
  void check_error() {
    if (!d_err.n) return;
    int e = 0;
    CK(cudaMemcpy(&e, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      CK(cudaMemset(d_err.p, 0, sizeof(int)));
      if (e == kErrNonFinite)
        throw ArgError{FDTD_ERR_NONFINITE, "the run diverged: a probe record or a field value is not finite"};
      throw ArgError{FDTD_ERR_DEVICE, "step kernel gave up waiting for a TMA plane load (code " +
                                          std::to_string(e) + ")"};
    }
  }
};

namespace {

// Geometry of the split stores of a plan (SplitDev without base pointers);
// returns the pairs one time buffer holds. z and y stores span whole x rows
// (pitch); x stores span the core y rows and an even number of pairs from an
// even origin, so their rows and TMA boxes start on 16 bytes.
size_t split_layout(const SplitPlan& plan, int nx, int ny, int nz, int pitch, SplitDev& g) {
  g = SplitDev{};
  const int* t = plan.t;
  for (int k = 0; k < 6; ++k) g.t[k] = t[k];
  const int zc0 = t[4], zc = std::max(0, nz - t[4] - t[5]);
  auto set = [&](int st, int ox, int oy, int oz, int w, int h, int d) {
    g.ox[st] = ox; g.oy[st] = oy; g.oz[st] = oz; g.w[st] = w; g.h[st] = h;
    g.comp[st] = int64_t(w) * h * d;
  };
  set(kStZlo, 0, 0, 0, pitch, ny, t[4]);
  set(kStZhi, 0, 0, nz - t[5], pitch, ny, t[5]);
  set(kStYlo, 0, 0, zc0, pitch, t[2], zc);
  set(kStYhi, 0, ny - t[3], zc0, pitch, t[3], zc);
  const int yc = std::max(0, ny - t[2] - t[3]);
  const int wxl = t[0] ? (t[0] + 1) & ~1 : 0;
  const int oxh = (nx - t[1]) & ~1;
  const int wxh = t[1] ? (nx - oxh + 1) & ~1 : 0;
  set(kStXlo, 0, t[2], zc0, wxl, yc, zc);
  set(kStXhi, oxh, t[2], zc0, wxh, yc, zc);
  int64_t off = 0;
  for (int st = 0; st < 6; ++st) {
    g.off[st] = off;
    off += 6 * g.comp[st];
  }
  g.off[kStSparse] = off;
  off += 6 * plan.n_sparse;
  return size_t(off);
}

void compile_host(fdtd_sim* s) {
  if (s->compiled) return;
  for (int i = 0; i < kNumCoef; ++i)
    if (!s->have_coef[i]) throw ArgError{FDTD_ERR_STATE, std::string("Coefficient not set: ") + kCoefNames[i]};
  const float* cp[kNumCoef];
  for (int i = 0; i < kNumCoef; ++i) cp[i] = s->coef_view[i] ? s->coef_view[i] : s->coef[i].data();
  std::string err;
  if (!compile_grid(s->nx, s->ny, s->nz, cp, s->probes, threads_for_host(), s->grid, err))
    throw ArgError{FDTD_ERR_LIMIT, err};
  if (!plan_split_storage(s->grid, s->split_plan, err)) throw ArgError{FDTD_ERR_LIMIT, err};
  s->compiled = true;
  s->base_rows = int(s->grid.rows.size());
  s->box_rows_from = -1;
}

void prepare(fdtd_sim* s, int nt) {
  if (s->prepared && s->prepared_nt == nt) return;
  for (size_t p = 0; p < s->probe_values.size(); ++p)
    if (s->probes[p].is_source && int(s->probe_values[p].size()) < nt)
      throw ArgError{FDTD_ERR_ARG, "Invalid data source array shape. Expected shape greater or equal to " +
                                       std::to_string(nt)};
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  if (!s->prepared) {
    compile_host(s);
    ++s->generation;
    s->pitch = ((nx + 31) / 32) * 32;
    s->cells_padded = size_t(nz) * ny * s->pitch;
    if (s->cells_padded >= (size_t(1) << 31) - size_t(2) * ny * s->pitch)
      throw ArgError{FDTD_ERR_LIMIT, "Grid too large for 32-bit cell offsets."};
    const size_t N = s->cells_padded;
    s->fields.alloc(12 * N);
    // split pairs only in the slab stores and the sparse store
    s->split_buf_pairs = split_layout(s->split_plan, nx, ny, nz, s->pitch, s->split_geo);
    for (int st = 0; st < 6; ++st)  // the kernels step between a store's components with 32-bit strides
      if (6 * s->split_geo.comp[st] >= (int64_t(1) << 31))
        throw ArgError{FDTD_ERR_LIMIT, "PML slab too large for 32-bit split-pair offsets."};
    const bool any_split = s->grid.e_split_cells > 0 || s->grid.h_split_cells > 0;
    s->splits.alloc(any_split ? 2 * 2 * s->split_buf_pairs : 0);
    // material index: upload in reference order, transpose on the device
    {
      DevBuf<uint16_t> tmp;
      tmp.alloc(s->grid.ids.size());
      h2d(s, tmp.p, s->grid.ids.data(), s->grid.ids.size() * 2);
      s->mat.alloc(N);
      CK(cudaMemset(s->mat.p, 0, N * 2));
      transpose_ids_kernel<<<1024, 256>>>(tmp.p, s->mat.p, nx, ny, nz, s->pitch);
      CK(cudaGetLastError());
      CK(cudaDeviceSynchronize());
    }
    s->rows.alloc(s->grid.rows.size() * 8);
    h2d(s, s->rows.p, s->grid.rows.data(), s->grid.rows.size() * sizeof(Row));
    s->cell_probes.alloc(std::max<size_t>(1, s->grid.cell_probes.size()));
    if (!s->grid.cell_probes.empty())
      h2d(s, s->cell_probes.p, s->grid.cell_probes.data(), s->grid.cell_probes.size() * sizeof(int2));
    std::vector<int> srcflag(std::max<size_t>(1, s->probes.size()), 0);
    for (size_t p = 0; p < s->probes.size(); ++p) srcflag[p] = s->probes[p].is_source;
    s->is_src.alloc(srcflag.size());
    h2d(s, s->is_src.p, srcflag.data(), srcflag.size() * sizeof(int));
    s->prepared = true;
  }
  // per-nt buffers: source amplitudes, records, DFT, monitors
  const size_t P = s->probes.size();
  s->src.alloc(std::max<size_t>(1, P * size_t(nt)));
  s->rec.alloc(std::max<size_t>(1, P * size_t(nt)));
  {
    std::vector<float> host(std::max<size_t>(1, P * size_t(nt)), 0.f);
    for (size_t p = 0; p < P; ++p)
      if (s->probes[p].is_source)
        std::memcpy(&host[p * nt], s->probe_values[p].data(), size_t(nt) * sizeof(float));
    h2d(s, s->src.p, host.data(), host.size() * sizeof(float));
  }
  if (s->n_series > 0) {
    s->d_series_start.alloc(s->series_start.size());
    h2d(s, s->d_series_start.p, s->series_start.data(), s->series_start.size() * 4);
    s->d_term_probe.alloc(std::max<size_t>(1, s->term_probe.size()));
    if (!s->term_probe.empty())
      h2d(s, s->d_term_probe.p, s->term_probe.data(), s->term_probe.size() * 4);
    s->d_term_weight.alloc(std::max<size_t>(1, s->term_weight.size()));
    if (!s->term_weight.empty())
      h2d(s, s->d_term_weight.p, s->term_weight.data(), s->term_weight.size() * 8);
    s->d_omega.alloc(s->omega.size());
    h2d(s, s->d_omega.p, s->omega.data(), s->omega.size() * 8);
    s->dft_X.alloc(size_t(s->n_series) * s->n_freq);
  }
  std::vector<MonDev> mdev;
  s->mon_out.clear();
  s->mon_phase.clear();
  for (auto& m : s->monitors) {
    if (m.n_freq && m.n_phase_rows < nt / m.n_step + 1)
      throw ArgError{FDTD_ERR_ARG, "Monitor phase table has fewer rows than nt/n_step + 1."};
    auto out = std::make_unique<DevBuf<char>>();
    out->alloc(m.out_bytes(nt));
    auto ph = std::make_unique<DevBuf<float2>>();
    if (m.n_freq) {
      ph->alloc(m.phase.size() / 2);
      h2d(s, ph->p, m.phase.data(), m.phase.size() * 4);
    }
    mdev.push_back(MonDev{m.field, m.axis, m.position, m.n_step, m.n_freq, m.n1, m.n2, out->p, ph->p});
    s->mon_out.push_back(std::move(out));
    s->mon_phase.push_back(std::move(ph));
  }
  s->d_mons.alloc(mdev.size());
  if (!mdev.empty())
    h2d(s, s->d_mons.p, mdev.data(), mdev.size() * sizeof(MonDev));

  // descriptor
  SimDev& d = s->dev;
  const size_t N = s->cells_padded;
  d.nx = nx; d.ny = ny; d.nz = nz; d.pitch = s->pitch; d.plane = ny * s->pitch; d.nt = nt;
  for (int b = 0; b < 2; ++b) {
    for (int c = 0; c < 3; ++c) {
      d.E[b][c] = s->fields.p + (size_t(b) * 6 + c) * N;
      d.H[b][c] = s->fields.p + (size_t(b) * 6 + 3 + c) * N;
    }
    // split pairs of time buffer b: the stores back to back
    d.sp = s->split_geo;
    for (int bb = 0; bb < 2; ++bb)
      d.sp.base[bb] = s->splits.n ? reinterpret_cast<float2*>(s->splits.p) + size_t(bb) * s->split_buf_pairs : nullptr;
  }
  d.mat = s->mat.p;
  d.rows = s->rows.p;
  d.cell_probes = s->cell_probes.p;
  d.src = s->src.p;
  d.rec = s->rec.p;
  d.is_src = s->is_src.p;
  d.cells = int64_t(N);
  s->d_dev.alloc(1);
  h2d(s, s->d_dev.p, &d, sizeof(SimDev));
  s->prepared_nt = nt;
}

void fill_stats(fdtd_sim* s, const Engine* e) {
  fdtd_stats& st = s->stats;
  st.nx = s->nx; st.ny = s->ny; st.nz = s->nz; st.nt = s->prepared_nt;
  st.n_rows = int(s->grid.rows.size());
  st.id_bytes = 2;
  st.e_split_cells = s->grid.e_split_cells;
  st.h_split_cells = s->grid.h_split_cells;
  st.compile_ms = s->grid.compile_ms;
  st.h2d_bytes = s->h2d_bytes;
  st.d2h_bytes = s->d2h_bytes;
  if (e) {
    st.variant = e->cfg.variant;
    st.tile_y = e->cfg.variant != 0 ? e->cfg.ty : kTileY;
    st.stages = e->cfg.variant != 0 ? e->cfg.stages : 0;
    st.zchunk = e->zchunk_used;
    st.grid = e->grid;
    st.n_tiles = e->n_tiles;
    st.step_launches = e->step_launches;
    st.dft_launches = e->dft_launches;
    st.last_run_ms = e->last_ms;
    st.tune_ms = e->tune_ms;
    st.tune_trials = e->tune_trials;
  }
}

template <typename F>
int guarded(std::string* err, F&& f) {
  try {
    f();
    return FDTD_OK;
  } catch (const ArgError& a) {
    if (err) *err = a.msg;
    return a.code;
  } catch (const CudaError& c) {
    if (err) *err = c.where + ": " + cudaGetErrorString(c.code);
    return FDTD_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    if (err) *err = "host allocation failed";
    return FDTD_ERR_LIMIT;
  } catch (const std::exception& e) {
    if (err) *err = e.what();
    return FDTD_ERR_ARG;
  }
}

int coef_index(const char* name) {
  for (int i = 0; i < kNumCoef; ++i)
    if (std::strcmp(name, kCoefNames[i]) == 0) return i;
  return -1;
}

}  // namespace

// Drops what the last run kept for a gradient (snapshots or box history).
void leave_adjoint_mode(fdtd_sim* s) {
  s->adj_mode = 0;
  s->adj_in_batch = false;
  s->ckpt_every = 0;
  s->ckpt_nt = -1;
  s->ckpt.free();
  s->hist.free();
  std::fill(s->adj_box, s->adj_box + 6, 0);
}

// A fresh single-simulation engine for s (descriptors, tiles, graph).
void new_engine(fdtd_sim* s) {
  s->engine.reset();
  s->engine = std::make_unique<Engine>();
  s->engine->sims = {s};
  s->engine->cfg = s->cfg;
  s->engine->ext_stream = s->ext_stream;
  s->engine->use_graph = s->use_graph;
  s->engine->wait_limit = s->dbg_wait_limit;
  s->engine->withhold = s->dbg_withhold;
  s->engine->build_tiles();
}

// A gradient box must be non-empty, inside the grid and free of cells with
// split E storage (PML slabs, source cells): the gradient treats the box
// cells' E pairs as one total with one Ca.
void check_gradient_box(const fdtd_sim* s, const int* box) {
  if (box[0] < 0 || box[2] < 0 || box[4] < 0 || box[1] > s->nx || box[3] > s->ny || box[5] > s->nz ||
      box[0] >= box[1] || box[2] >= box[3] || box[4] >= box[5])
    throw ArgError{FDTD_ERR_ARG, "gradient box must be a non-empty box inside the grid."};
  for (int x = box[0]; x < box[1]; ++x)
    for (int y = box[2]; y < box[3]; ++y)
      for (int z = box[4]; z < box[5]; ++z) {
        const uint32_t f = s->grid.rows[s->grid.ids[(size_t(x) * s->ny + y) * s->nz + z]].w[R_FLAGS];
        if (f & kFlagESplit) throw ArgError{FDTD_ERR_ARG, "gradient box holds split-field (PML or source) cells."};
      }
}

struct fdtd_batch {
  std::vector<fdtd_sim*> sims;
  Engine engine;
  bool dirty = true;
  std::vector<int> gens;  // members' device-buffer generations the engine was built on
  std::string err;
  fdtd_stats stats{};
};

// Whether a member's device buffers moved since the batch engine was built.
bool batch_moved(const fdtd_batch* b) {
  if (b->gens.size() != b->sims.size()) return true;
  for (size_t i = 0; i < b->sims.size(); ++i)
    if (b->gens[i] != b->sims[i]->generation) return true;
  return false;
}

void note_generations(fdtd_batch* b) {
  b->gens.clear();
  for (auto* s : b->sims) b->gens.push_back(s->generation);
}

// Material index of the box cells on the device: ids [x][y][z] of the box.
__global__ void set_box_ids_kernel(uint16_t* mat, int ny, int pitch, int x0, int y0, int z0, int bnx, int bny,
                                   int bnz, const uint16_t* ids) {
  const int64_t nb = int64_t(bnx) * bny * bnz;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nb; i += int64_t(gridDim.x) * blockDim.x) {
    const int zz = int(i % bnz), yy = int((i / bnz) % bny), xx = int(i / (int64_t(bnz) * bny));
    mat[size_t(z0 + zz) * ny * pitch + size_t(y0 + yy) * pitch + (x0 + xx)] = ids[i];
  }
}

// E-update coefficients of a box: host arrays, and the compiled table when
// there is one (one dedicated row per box cell after the compiled rows).
void set_box_coefficients(fdtd_sim* s, const int* box, const float* coefs) {
  static const char* const names[3][4] = {{"Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z"},
                                           {"Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x"},
                                           {"Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y"}};
  if (box[0] < 0 || box[2] < 0 || box[4] < 0 || box[1] > s->nx || box[3] > s->ny || box[5] > s->nz ||
      box[0] >= box[1] || box[2] >= box[3] || box[4] >= box[5])
    throw ArgError{FDTD_ERR_ARG, "box must be a non-empty box inside the grid."};
  int ci[3][4];
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < 4; ++k) {
      ci[c][k] = coef_index(names[c][k]);
      if (!s->have_coef[ci[c][k]])
        throw ArgError{FDTD_ERR_STATE, std::string("Coefficient not set: ") + names[c][k]};
    }
  if (s->compiled) check_gradient_box(s, box);
  for (int c = 0; c < 3; ++c)  // the patch writes the host arrays: copy borrowed ones first
    for (int k = 0; k < 4; ++k) {
      const int i = ci[c][k];
      if (s->coef_view[i]) {
        s->coef[i].assign(s->coef_view[i], s->coef_view[i] + size_t(s->nx) * s->ny * s->nz);
        s->coef_view[i] = nullptr;
      }
    }
  const int bny = box[3] - box[2], bnz = box[5] - box[4];
  const int64_t nb = box_cells(box);
  auto cell_of = [&](int64_t bi) {
    const int zz = int(bi % bnz), yy = int((bi / bnz) % bny), xx = int(bi / (int64_t(bnz) * bny));
    return (size_t(box[0] + xx) * s->ny + (box[2] + yy)) * s->nz + (box[4] + zz);
  };
  for (int64_t bi = 0; bi < nb; ++bi) {
    const size_t cell = cell_of(bi);
    for (int c = 0; c < 3; ++c) {
      const float ca = coefs[(3 * c + 0) * nb + bi], cb1 = coefs[(3 * c + 1) * nb + bi],
                  cb2 = coefs[(3 * c + 2) * nb + bi];
      s->coef[ci[c][0]][cell] = ca;
      s->coef[ci[c][1]][cell] = ca;
      s->coef[ci[c][2]][cell] = cb1;
      s->coef[ci[c][3]][cell] = cb2;
    }
  }
  if (!s->compiled) return;  // the next run compiles the arrays
  if (s->engine) CK(cudaStreamSynchronize(s->engine->stream()));
  std::vector<uint16_t>& ids = s->grid.ids;
  std::vector<Row>& rows = s->grid.rows;
  bool new_ids = false;
  if (s->box_rows_from >= 0 && !std::equal(box, box + 6, s->box_rows_box)) {
    // another box: the next run compiles the patched arrays afresh
    s->compiled = false;
    s->prepared = false;
    return;
  }
  if (s->box_rows_from < 0) {
    if (int64_t(s->base_rows) + nb > 65536)
      throw ArgError{FDTD_ERR_LIMIT, "box needs more rows than the 16-bit material index can address."};
    s->box_rows_from = s->base_rows;
    std::copy(box, box + 6, s->box_rows_box);
    rows.resize(size_t(s->base_rows) + size_t(nb));
    for (int64_t bi = 0; bi < nb; ++bi) {
      const size_t cell = cell_of(bi);
      rows[size_t(s->base_rows + bi)] = rows[ids[cell]];
      ids[cell] = uint16_t(s->base_rows + bi);
    }
    new_ids = true;
  }
  for (int64_t bi = 0; bi < nb; ++bi) {
    Row& r = rows[size_t(s->box_rows_from + bi)];
    for (int c = 0; c < 3; ++c) {
      const float ca = coefs[(3 * c + 0) * nb + bi], cb1 = coefs[(3 * c + 1) * nb + bi],
                  cb2 = coefs[(3 * c + 2) * nb + bi];
      std::memcpy(&r.w[4 * c + 0], &ca, 4);
      std::memcpy(&r.w[4 * c + 1], &cb1, 4);
      std::memcpy(&r.w[4 * c + 2], &ca, 4);
      std::memcpy(&r.w[4 * c + 3], &cb2, 4);
    }
  }
  if (!s->prepared) return;  // the next run uploads the table
  if (s->rows.n < rows.size() * 8) {
    // a larger table: every descriptor holding the old pointer is rebuilt
    s->rows.alloc(rows.size() * 8);
    h2d(s, s->rows.p, rows.data(), rows.size() * sizeof(Row));
    s->dev.rows = s->rows.p;
    h2d(s, s->d_dev.p, &s->dev, sizeof(SimDev));
    ++s->generation;
    s->engine.reset();
  } else {
    h2d(s, s->rows.p + size_t(s->box_rows_from) * 8, rows.data() + s->box_rows_from, size_t(nb) * sizeof(Row));
  }
  if (new_ids) {
    std::vector<uint16_t> bids(static_cast<size_t>(nb));
    for (int64_t bi = 0; bi < nb; ++bi) bids[size_t(bi)] = uint16_t(s->box_rows_from + bi);
    DevBuf<uint16_t> tmp;
    tmp.alloc(bids.size());
    h2d(s, tmp.p, bids.data(), bids.size() * 2);
    set_box_ids_kernel<<<256, 256>>>(s->mat.p, s->ny, s->pitch, box[0], box[2], box[4], box[1] - box[0], bny, bnz,
                                     tmp.p);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
}

extern "C" {

int fdtd_set_box_coefficients(fdtd_sim* s, const int* box, const float* coefs) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (!box || !coefs) throw ArgError{FDTD_ERR_ARG, "null argument"};
    set_box_coefficients(s, box, coefs);
  });
}

int fdtd_create(int nx, int ny, int nz, fdtd_sim** out) {
  if (!out) {
    g_error = "fdtd_create: null output pointer";
    return FDTD_ERR_ARG;
  }
  *out = nullptr;
  if (nx < 2 || ny < 2 || nz < 2 || nx > 65535 || ny > 65535 || nz > 65535) {
    g_error = "Grid dimensions must be between 2 and 65535 cells.";
    return FDTD_ERR_ARG;
  }
  auto* s = new (std::nothrow) fdtd_sim();
  if (!s) {
    g_error = "host allocation failed";
    return FDTD_ERR_LIMIT;
  }
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  *out = s;
  return FDTD_OK;
}

int fdtd_set_coefficient(fdtd_sim* s, const char* name, const float* data, int nx, int ny, int nz) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    const int i = name ? coef_index(name) : -1;
    if (i < 0) throw ArgError{FDTD_ERR_ARG, std::string("Unknown coefficient array ") + (name ? name : "(null)")};
    const int expect[3] = {s->nx, s->ny, s->nz}, got[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a)
      if (expect[a] != got[a])
        throw ArgError{FDTD_ERR_ARG, std::string("Invalid data array ") + name + ". Expected shape on axis " +
                                         std::to_string(a) + " of " + std::to_string(expect[a])};
    if (!data) throw ArgError{FDTD_ERR_ARG, "null coefficient data"};
    s->coef[i].assign(data, data + size_t(nx) * ny * nz);
    s->coef_view[i] = nullptr;
    s->have_coef[i] = true;
    s->prepared = false;
    s->compiled = false;
  });
}

int fdtd_set_coefficient_view(fdtd_sim* s, const char* name, const float* data, int nx, int ny, int nz) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    const int i = name ? coef_index(name) : -1;
    if (i < 0) throw ArgError{FDTD_ERR_ARG, std::string("Unknown coefficient array ") + (name ? name : "(null)")};
    const int expect[3] = {s->nx, s->ny, s->nz}, got[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a)
      if (expect[a] != got[a])
        throw ArgError{FDTD_ERR_ARG, std::string("Invalid data array ") + name + ". Expected shape on axis " +
                                         std::to_string(a) + " of " + std::to_string(expect[a])};
    if (!data) throw ArgError{FDTD_ERR_ARG, "null coefficient data"};
    std::vector<float>().swap(s->coef[i]);
    s->coef_view[i] = data;
    s->have_coef[i] = true;
    s->prepared = false;
    s->compiled = false;
  });
}

int fdtd_add_probe(fdtd_sim* s, int field, int i, int j, int k, int is_source, const float* values, int n_values,
                   int* index) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (field < 0 || field > 5) throw ArgError{FDTD_ERR_ARG, "Invalid probe field type."};
    if (int(s->probes.size()) >= kMaxProbes) throw ArgError{FDTD_ERR_LIMIT, "Exceeded maximum number of probes."};
    if (is_source && (!values || n_values < 0)) throw ArgError{FDTD_ERR_ARG, "Source probe needs values."};
    s->probes.push_back(ProbeSpec{field, i, j, k, is_source ? 1 : 0});
    s->probe_values.emplace_back();
    if (values && n_values > 0) s->probe_values.back().assign(values, values + n_values);
    if (index) *index = int(s->probes.size()) - 1;
    s->prepared = false;
    s->compiled = false;
  });
}

int fdtd_add_monitor(fdtd_sim* s, int field, int axis, int position, int n_step, int n_freq, const float* phase,
                     int n_phase_rows, int* index) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (int(s->monitors.size()) >= kMaxMonitors)
      throw ArgError{FDTD_ERR_LIMIT, "Exceeded maximum number of monitors."};
    if (field < 0 || field > 5 || axis < 0 || axis > 2 || n_step < 1 || n_freq < 0)
      throw ArgError{FDTD_ERR_ARG, "Invalid monitor field, axis, n_step or n_frequencies."};
    Monitor m{};
    m.field = field;
    m.axis = axis;
    m.n_step = n_step;
    m.n_freq = n_freq;
    // GPU-layout position shift of solver_init_monitors (solver.cpp:394-441, gpu = 1)
    int pos = position;
    if (axis == 0 && (field == 3 || field == 1 || field == 2)) pos -= 1;
    if (axis == 1 && (field == 4 || field == 0 || field == 2)) pos -= 1;
    if (axis == 2 && (field == 5 || field == 0 || field == 1)) pos -= 1;
    m.position = pos;
    m.n1 = axis == 0 ? s->ny : s->nx;
    m.n2 = axis == 2 ? s->ny : s->nz;
    if (n_freq) {
      if (!phase || n_phase_rows < 1) throw ArgError{FDTD_ERR_ARG, "Phasor monitor needs a dtft_phase table."};
      m.phase.assign(phase, phase + size_t(n_phase_rows) * n_freq * 2);
      m.n_phase_rows = n_phase_rows;
    }
    s->monitors.push_back(std::move(m));
    if (index) *index = int(s->monitors.size()) - 1;
    s->prepared_nt = -1;
  });
}

int fdtd_set_dft(fdtd_sim* s, int n_series, int n_terms, const int* term_series, const int* term_probe,
                 const double* term_weight, int n_freq, const double* omega) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (n_series < 0 || n_terms < 0 || n_freq < 0) throw ArgError{FDTD_ERR_ARG, "Negative DFT size."};
    if (n_series > 0 && n_freq > 0 && (!omega || (n_terms > 0 && (!term_series || !term_probe || !term_weight))))
      throw ArgError{FDTD_ERR_ARG, "null DFT array"};
    std::vector<std::vector<std::pair<int, double>>> per(n_series);
    for (int t = 0; t < n_terms; ++t) {
      if (term_series[t] < 0 || term_series[t] >= n_series)
        throw ArgError{FDTD_ERR_ARG, "DFT term refers to a series out of range."};
      if (term_probe[t] < 0 || term_probe[t] >= int(s->probes.size()))
        throw ArgError{FDTD_ERR_ARG, "DFT term refers to a probe out of range (add probes first)."};
      per[term_series[t]].emplace_back(term_probe[t], term_weight[t]);
    }
    s->n_series = n_series;
    s->n_freq = n_freq;
    s->series_start.assign(1, 0);
    s->term_probe.clear();
    s->term_weight.clear();
    for (auto& v : per) {
      for (auto& pw : v) {
        s->term_probe.push_back(pw.first);
        s->term_weight.push_back(pw.second);
      }
      s->series_start.push_back(int(s->term_probe.size()));
    }
    s->omega.assign(omega, omega + n_freq);
    s->prepared_nt = -1;
  });
}

int fdtd_compile(fdtd_sim* s, int* n_rows, int64_t* e_split_cells, int64_t* h_split_cells) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    compile_host(s);
    if (n_rows) *n_rows = int(s->grid.rows.size());
    if (e_split_cells) *e_split_cells = s->grid.e_split_cells;
    if (h_split_cells) *h_split_cells = s->grid.h_split_cells;
  });
}

int fdtd_get_material_table(fdtd_sim* s, uint16_t* ids, int64_t n_ids, uint32_t* rows, int n_rows) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (!s->compiled) throw ArgError{FDTD_ERR_STATE, "Material table not compiled."};
    if (ids) {
      if (size_t(n_ids) != s->grid.ids.size()) throw ArgError{FDTD_ERR_ARG, "ids size mismatch."};
      std::memcpy(ids, s->grid.ids.data(), s->grid.ids.size() * 2);
    }
    if (rows) {
      if (size_t(n_rows) != s->grid.rows.size()) throw ArgError{FDTD_ERR_ARG, "rows size mismatch."};
      std::memcpy(rows, s->grid.rows.data(), s->grid.rows.size() * sizeof(Row));
    }
  });
}

int fdtd_set_kernel(fdtd_sim* s, int variant, int tile_y, int stages, int zchunk) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (variant < 0 || variant > 1)
      throw ArgError{FDTD_ERR_ARG, "variant must be 0 (plain) or 1 (stream)"};
    if (!kernel_exists(variant, tile_y, stages))
      throw ArgError{FDTD_ERR_ARG, "No kernel instantiated for this variant / tile height / stage count."};
    KernelConfig c;
    c.variant = variant;
    c.ty = tile_y;
    c.stages = stages;
    c.zchunk = zchunk;
    c.one_list = one_list_env();
    s->cfg = c;
    s->engine.reset();
  });
}

int fdtd_set_graph(fdtd_sim* s, int enabled) {
  if (!s) return FDTD_ERR_ARG;
  s->use_graph = enabled != 0;
  if (s->engine) {
    s->engine->use_graph = s->use_graph;
    s->engine->reset_graph();
  }
  return FDTD_OK;
}

int fdtd_set_debug(fdtd_sim* s, unsigned wait_limit, int withhold_plane) {
  if (!s) return FDTD_ERR_ARG;
  s->dbg_wait_limit = wait_limit ? wait_limit : kStreamWaitLimit;
  s->dbg_withhold = withhold_plane < 0 ? -1 : withhold_plane;
  if (s->engine) {
    s->engine->wait_limit = s->dbg_wait_limit;
    s->engine->withhold = s->dbg_withhold;
    s->engine->reset_graph();
  }
  return FDTD_OK;
}

int fdtd_set_stream(fdtd_sim* s, void* stream) {
  if (!s) return FDTD_ERR_ARG;
  s->ext_stream = static_cast<cudaStream_t>(stream);
  if (s->engine) s->engine->ext_stream = s->ext_stream;
  return FDTD_OK;
}

int fdtd_run_async(fdtd_sim* s, int nt) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (nt < 1) throw ArgError{FDTD_ERR_ARG, "nt must be positive."};
    if (s->adj_mode) {  // the time loop is captured without snapshots or history again
      leave_adjoint_mode(s);
      s->engine.reset();
    }
    const bool rebuild = !s->prepared || s->prepared_nt != nt || !s->engine;
    prepare(s, nt);
    if (rebuild) new_engine(s);
    s->engine->run_async(nt);
    fill_stats(s, s->engine.get());
  });
}

int fdtd_run_checkpointed(fdtd_sim* s, int nt, int every) {
  if (!s) return FDTD_ERR_ARG;
  const int rc = guarded(&s->err, [&] {
    if (nt < 1 || every < 1) throw ArgError{FDTD_ERR_ARG, "nt and the checkpoint interval must be positive."};
    // a re-prepared simulation has new device buffers: the engine (descriptors,
    // tensor maps, graph) must be rebuilt with it
    const bool rebuild = !s->prepared || s->prepared_nt != nt || !s->engine || s->adj_mode != 1 ||
                         s->ckpt_every != every || s->ckpt_nt != nt;
    prepare(s, nt);
    const size_t N = s->cells_padded;
    const size_t stride = 6 * N + (s->splits.n ? 2 * s->split_buf_pairs : 0);
    const size_t nseg = size_t((nt + every - 1) / every);
    if (rebuild) {
      leave_adjoint_mode(s);
      s->adj_mode = 1;
      s->ckpt_every = every;
      s->ckpt_nt = nt;
      s->ckpt.alloc(nseg * stride);
      new_engine(s);
    }
    s->engine->run_async(nt);
    fill_stats(s, s->engine.get());
  });
  if (rc) return rc;
  return fdtd_synchronize(s);
}

int fdtd_run_recorded(fdtd_sim* s, int nt, const int* box) {
  if (!s) return FDTD_ERR_ARG;
  const int rc = guarded(&s->err, [&] {
    if (nt < 1 || !box) throw ArgError{FDTD_ERR_ARG, "nt must be positive and the box given."};
    const bool rebuild = !s->prepared || s->prepared_nt != nt || !s->engine || s->adj_mode != 2 ||
                         s->ckpt_nt != nt || !std::equal(box, box + 6, s->adj_box);
    prepare(s, nt);
    check_gradient_box(s, box);
    if (rebuild) {
      leave_adjoint_mode(s);
      s->hist.alloc(size_t(nt) * 9 * size_t(box_cells(box)));
      s->adj_mode = 2;
      s->ckpt_nt = nt;
      std::copy(box, box + 6, s->adj_box);
      new_engine(s);
    }
    s->engine->run_async(nt);
    fill_stats(s, s->engine.get());
  });
  if (rc) return rc;
  return fdtd_synchronize(s);
}

int fdtd_adjoint(fdtd_sim* s, const double* dJ_dX, int n_series, int n_freq, const int* box, double* grad) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (!dJ_dX || !box || !grad) throw ArgError{FDTD_ERR_ARG, "null argument"};
    if (!s->engine || s->adj_mode == 0 || s->ckpt_nt < 1)
      throw ArgError{FDTD_ERR_STATE, "fdtd_adjoint needs a preceding fdtd_run_checkpointed or fdtd_run_recorded."};
    if (n_series != s->n_series || n_freq != s->n_freq || n_series < 1 || n_freq < 1)
      throw ArgError{FDTD_ERR_ARG, "dJ/dX size does not match the DFT of the run."};
    if (s->engine->sims.size() != 1) throw ArgError{FDTD_ERR_STATE, "adjoint runs need a single simulation."};
    check_gradient_box(s, box);
    if (s->adj_mode == 2 && !std::equal(box, box + 6, s->adj_box))
      throw ArgError{FDTD_ERR_ARG, "gradient box differs from the box recorded by fdtd_run_recorded."};
    if (s->adj_in_batch) throw ArgError{FDTD_ERR_STATE, "the recorded run was a batch run: use fdtd_batch_adjoint."};
    s->engine->adjoint({Engine::AdjRequest{s, dJ_dX, box, grad}});
    s->stats.adjoint_launches = s->engine->adj_launches;
    s->stats.adjoint_ms = s->engine->adj_ms;
  });
}

int fdtd_synchronize(fdtd_sim* s) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (!s->engine) throw ArgError{FDTD_ERR_STATE, "No run in flight."};
    s->engine->sync();
    fill_stats(s, s->engine.get());
  });
}

int fdtd_run(fdtd_sim* s, int nt) {
  int rc = fdtd_run_async(s, nt);
  if (rc) return rc;
  return fdtd_synchronize(s);
}

int fdtd_get_probe_values(fdtd_sim* s, float* out, int n_probes, int nt) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (!s->prepared || s->prepared_nt < 0) throw ArgError{FDTD_ERR_STATE, "No completed run."};
    if (n_probes != int(s->probes.size()) || nt != s->prepared_nt)
      throw ArgError{FDTD_ERR_ARG, "Probe output size does not match the last run."};
    if (n_probes == 0) return;
    d2h(s, out, s->rec.p, size_t(n_probes) * nt * sizeof(float));
  });
}

int fdtd_get_dft(fdtd_sim* s, double* out, int n_series, int n_freq) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (n_series != s->n_series || n_freq != s->n_freq) throw ArgError{FDTD_ERR_ARG, "DFT size mismatch."};
    if (!s->dft_X.n) throw ArgError{FDTD_ERR_STATE, "No DFT configured."};
    d2h(s, out, s->dft_X.p, s->dft_X.n * sizeof(double2));
  });
}

int fdtd_get_monitor(fdtd_sim* s, int m, void* out, int64_t n_bytes) {
  if (!s) return FDTD_ERR_ARG;
  return guarded(&s->err, [&] {
    if (m < 0 || m >= int(s->mon_out.size())) throw ArgError{FDTD_ERR_ARG, "Monitor index out of range."};
    if (size_t(n_bytes) != s->mon_out[m]->n) throw ArgError{FDTD_ERR_ARG, "Monitor output size mismatch."};
    d2h(s, out, s->mon_out[m]->p, size_t(n_bytes));
  });
}

int fdtd_get_stats(const fdtd_sim* s, fdtd_stats* out) {
  if (!s || !out) return FDTD_ERR_ARG;
  *out = s->stats;
  out->h2d_bytes = s->h2d_bytes;
  out->d2h_bytes = s->d2h_bytes;
  if (s->compiled) {
    for (int k = 0; k < 6; ++k) out->split_slab[k] = s->split_plan.t[k];
    out->slab_cells = s->split_plan.slab_cells;
    out->sparse_split_cells = s->split_plan.sparse_cells;
    out->split_bytes = int64_t(s->splits.n * sizeof(float));
  }
  return FDTD_OK;
}

const char* fdtd_last_error(const fdtd_sim* s) { return s ? s->err.c_str() : g_error.c_str(); }

void fdtd_destroy(fdtd_sim* s) {
  if (!s) return;
  if (s->engine) {
    cudaStreamSynchronize(s->engine->stream());
    s->engine.reset();
  }
  delete s;
}

int fdtd_batch_create(fdtd_sim* const* sims, int n_sims, fdtd_batch** out) {
  if (!out || !sims || n_sims < 1) {
    g_error = "fdtd_batch_create: invalid arguments";
    return FDTD_ERR_ARG;
  }
  *out = nullptr;
  auto* b = new (std::nothrow) fdtd_batch();
  if (!b) {
    g_error = "host allocation failed";
    return FDTD_ERR_LIMIT;
  }
  for (int i = 0; i < n_sims; ++i) {
    if (!sims[i]) {
      delete b;
      g_error = "fdtd_batch_create: null simulation";
      return FDTD_ERR_ARG;
    }
    b->sims.push_back(sims[i]);
  }
  b->engine.sims = b->sims;
  b->engine.cfg = default_config();
  *out = b;
  return FDTD_OK;
}

int fdtd_batch_set_kernel(fdtd_batch* b, int variant, int tile_y, int stages, int zchunk) {
  if (!b) return FDTD_ERR_ARG;
  return guarded(&b->err, [&] {
    if (variant < 0 || variant > 1)
      throw ArgError{FDTD_ERR_ARG, "variant must be 0 (plain) or 1 (stream)"};
    if (!kernel_exists(variant, tile_y, stages))
      throw ArgError{FDTD_ERR_ARG, "No kernel instantiated for this variant / tile height / stage count."};
    b->engine.cfg.variant = variant;
    b->engine.cfg.ty = tile_y;
    b->engine.cfg.stages = stages;
    b->engine.cfg.zchunk = zchunk;
    b->engine.cfg.one_list = one_list_env();
    b->dirty = true;
  });
}

int fdtd_batch_set_stream(fdtd_batch* b, void* stream) {
  if (!b) return FDTD_ERR_ARG;
  b->engine.ext_stream = static_cast<cudaStream_t>(stream);
  return FDTD_OK;
}

int fdtd_batch_run(fdtd_batch* b, int nt) {
  if (!b) return FDTD_ERR_ARG;
  return guarded(&b->err, [&] {
    if (nt < 1) throw ArgError{FDTD_ERR_ARG, "nt must be positive."};
    bool rebuild = b->engine.graph_nt != nt || b->engine.n_tiles == 0 || b->dirty;
    b->dirty = false;
    for (auto* s : b->sims) {
      if (!s->prepared || s->prepared_nt != nt) rebuild = true;
      if (s->adj_mode) {
        leave_adjoint_mode(s);
        rebuild = true;
      }
      try {
        prepare(s, nt);
      } catch (ArgError& a) {
        a.msg = "batch member: " + a.msg;
        throw;
      }
    }
    if (batch_moved(b)) rebuild = true;
    if (rebuild) {
      b->engine.graph_nt = -1;
      b->engine.build_tiles();
      note_generations(b);
    }
    b->engine.run_async(nt);
    b->engine.sync();
    for (auto* s : b->sims) fill_stats(s, &b->engine);
    fdtd_stats& st = b->stats;
    st = fdtd_stats{};
    st.nt = nt;
    st.variant = b->engine.cfg.variant;
    st.tile_y = b->engine.cfg.variant != 0 ? b->engine.cfg.ty : kTileY;
    st.stages = b->engine.cfg.variant != 0 ? b->engine.cfg.stages : 0;
    st.zchunk = b->engine.zchunk_used;
    st.grid = b->engine.grid;
    st.n_tiles = b->engine.n_tiles;
    st.step_launches = b->engine.step_launches;
    st.dft_launches = b->engine.dft_launches;
    st.last_run_ms = b->engine.last_ms;
    st.tune_ms = b->engine.tune_ms;
    st.tune_trials = b->engine.tune_trials;
    for (auto* s : b->sims) {
      st.e_split_cells += s->grid.e_split_cells;
      st.h_split_cells += s->grid.h_split_cells;
      st.n_rows += int(s->grid.rows.size());
      st.compile_ms += s->grid.compile_ms;
    }
    st.id_bytes = 2;
  });
}

int fdtd_batch_run_recorded(fdtd_batch* b, int nt, const int* boxes) {
  if (!b) return FDTD_ERR_ARG;
  return guarded(&b->err, [&] {
    if (nt < 1 || !boxes) throw ArgError{FDTD_ERR_ARG, "nt must be positive and the boxes given."};
    bool rebuild = b->engine.graph_nt != nt || b->engine.n_tiles == 0 || b->dirty;
    b->dirty = false;
    for (size_t i = 0; i < b->sims.size(); ++i) {
      fdtd_sim* s = b->sims[i];
      const int* box = boxes + 6 * i;
      if (!s->prepared || s->prepared_nt != nt) rebuild = true;
      try {
        prepare(s, nt);
        check_gradient_box(s, box);
      } catch (ArgError& a) {
        a.msg = "batch member " + std::to_string(i) + ": " + a.msg;
        throw;
      }
      if (s->adj_mode != 2 || !s->adj_in_batch || s->ckpt_nt != nt || !std::equal(box, box + 6, s->adj_box)) {
        leave_adjoint_mode(s);
        s->hist.alloc(size_t(nt) * 9 * size_t(box_cells(box)));
        s->adj_mode = 2;
        s->adj_in_batch = true;
        s->ckpt_nt = nt;
        std::copy(box, box + 6, s->adj_box);
        rebuild = true;
      }
    }
    if (batch_moved(b)) rebuild = true;
    if (rebuild) {
      b->engine.graph_nt = -1;
      b->engine.build_tiles();
      note_generations(b);
    }
    b->engine.run_async(nt);
    b->engine.sync();
    for (auto* s : b->sims) fill_stats(s, &b->engine);
    b->stats.nt = nt;
    b->stats.last_run_ms = b->engine.last_ms;
    b->stats.step_launches = b->engine.step_launches;
    b->stats.tune_ms = b->engine.tune_ms;
    b->stats.tune_trials = b->engine.tune_trials;
  });
}

int fdtd_batch_run_checkpointed(fdtd_batch* b, int nt, int every, const int* boxes) {
  if (!b) return FDTD_ERR_ARG;
  return guarded(&b->err, [&] {
    if (nt < 1 || every < 1 || !boxes)
      throw ArgError{FDTD_ERR_ARG, "nt and the checkpoint interval must be positive and the boxes given."};
    bool rebuild = b->engine.graph_nt != nt || b->engine.n_tiles == 0 || b->dirty;
    b->dirty = false;
    const size_t nseg = size_t((nt + every - 1) / every);
    for (size_t i = 0; i < b->sims.size(); ++i) {
      fdtd_sim* s = b->sims[i];
      const int* box = boxes + 6 * i;
      if (!s->prepared || s->prepared_nt != nt) rebuild = true;
      try {
        prepare(s, nt);
        check_gradient_box(s, box);
      } catch (ArgError& a) {
        a.msg = "batch member " + std::to_string(i) + ": " + a.msg;
        throw;
      }
      if (s->adj_mode != 1 || !s->adj_in_batch || s->ckpt_nt != nt || s->ckpt_every != every ||
          !std::equal(box, box + 6, s->adj_box)) {
        leave_adjoint_mode(s);
        const size_t stride = 6 * s->cells_padded + (s->splits.n ? 2 * s->split_buf_pairs : 0);
        s->ckpt.alloc(nseg * stride);
        s->adj_mode = 1;
        s->adj_in_batch = true;
        s->ckpt_every = every;
        s->ckpt_nt = nt;
        std::copy(box, box + 6, s->adj_box);
        rebuild = true;
      }
    }
    if (batch_moved(b)) rebuild = true;
    if (rebuild) {
      b->engine.graph_nt = -1;
      b->engine.build_tiles();
      note_generations(b);
    }
    b->engine.run_async(nt);
    b->engine.sync();
    for (auto* s : b->sims) fill_stats(s, &b->engine);
    b->stats.nt = nt;
    b->stats.last_run_ms = b->engine.last_ms;
    b->stats.step_launches = b->engine.step_launches;
    b->stats.tune_ms = b->engine.tune_ms;
    b->stats.tune_trials = b->engine.tune_trials;
  });
}

int fdtd_batch_adjoint(fdtd_batch* b, const double* const* dJ_dX, double* const* grad) {
  if (!b) return FDTD_ERR_ARG;
  return guarded(&b->err, [&] {
    if (!dJ_dX || !grad) throw ArgError{FDTD_ERR_ARG, "null argument"};
    std::vector<Engine::AdjRequest> req;
    const int mode = b->sims.empty() ? 0 : b->sims[0]->adj_mode;
    for (size_t i = 0; i < b->sims.size(); ++i) {
      fdtd_sim* s = b->sims[i];
      if (s->adj_mode == 0 || s->adj_mode != mode || !s->adj_in_batch || b->engine.graph_nt != s->ckpt_nt)
        throw ArgError{FDTD_ERR_STATE,
                       "fdtd_batch_adjoint needs a preceding fdtd_batch_run_recorded or fdtd_batch_run_checkpointed."};
      if (s->n_series < 1 || s->n_freq < 1) throw ArgError{FDTD_ERR_STATE, "batch member without a DFT."};
      if (!dJ_dX[i] || !grad[i]) throw ArgError{FDTD_ERR_ARG, "null member array"};
      req.push_back(Engine::AdjRequest{s, dJ_dX[i], s->adj_box, grad[i]});
    }
    b->engine.adjoint(req);
    b->stats.adjoint_launches = b->engine.adj_launches;
    b->stats.adjoint_ms = b->engine.adj_ms;
  });
}

int fdtd_batch_get_stats(const fdtd_batch* b, fdtd_stats* out) {
  if (!b || !out) return FDTD_ERR_ARG;
  *out = b->stats;
  return FDTD_OK;
}

const char* fdtd_batch_last_error(const fdtd_batch* b) { return b ? b->err.c_str() : g_error.c_str(); }

void fdtd_batch_destroy(fdtd_batch* b) {
  if (!b) return;
  cudaStreamSynchronize(b->engine.stream());
  delete b;
}

const char* fdtd_global_error(void) { return g_error.c_str(); }

int fdtd_trim_memory(int64_t keep_bytes, int64_t* reserved, int64_t* used) {
  return guarded(&g_error, [&] {
    if (keep_bytes < 0) throw ArgError{FDTD_ERR_ARG, "fdtd_trim_memory: keep_bytes must be >= 0"};
    cudaMemPool_t pool = engine_pool();
    // blocks freed by destroyed simulations are returned once every stream is past their last use
    CK(cudaDeviceSynchronize());
    CK(cudaMemPoolTrimTo(pool, size_t(keep_bytes)));
    uint64_t r = 0, u = 0;
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved) *reserved = int64_t(r);
    if (used) *used = int64_t(u);
  });
}

int fdtd_nf2ff(const fdtd_nf2ff_face* faces, int n_faces, int n_freq, const float* beta, int n_theta,
               const float* theta, int n_phi, const float* phi, float* out) {
  return guarded(&g_error, [&] {
    if (!faces || n_faces < 0 || n_freq < 1 || n_theta < 1 || n_phi < 1 || !beta || !theta || !phi || !out)
      throw ArgError{FDTD_ERR_ARG, "fdtd_nf2ff: invalid arguments"};
    if (int64_t(n_theta) * n_phi > (int64_t(1) << 30) || n_freq > 65535)
      throw ArgError{FDTD_ERR_LIMIT, "fdtd_nf2ff: too many directions or frequencies"};
    int64_t n_cells = 0;
    for (int i = 0; i < n_faces; ++i) {
      const fdtd_nf2ff_face& fc = faces[i];
      if (fc.axis < 0 || fc.axis > 2 || fc.n0 < 0 || fc.n1 < 0)
        throw ArgError{FDTD_ERR_ARG, "fdtd_nf2ff: invalid face"};
      if (int64_t(fc.n0) * fc.n1 > 0 && (!fc.r0 || !fc.r1 || !fc.ds || !fc.J || !fc.M))
        throw ArgError{FDTD_ERR_ARG, "fdtd_nf2ff: null face array"};
      n_cells += int64_t(fc.n0) * fc.n1;
    }
    if (n_cells * n_freq > (int64_t(1) << 31)) throw ArgError{FDTD_ERR_LIMIT, "fdtd_nf2ff: surface too large"};
    // cells of all faces, one block per frequency: position and ds J, ds M
    std::vector<Nf2ffCell> host(size_t(std::max<int64_t>(1, n_cells * n_freq)));
    int64_t c0 = 0;
    for (int i = 0; i < n_faces; ++i) {
      const fdtd_nf2ff_face& fc = faces[i];
      const int64_t nc = int64_t(fc.n0) * fc.n1;
      for (int64_t c = 0; c < nc; ++c) {
        float xyz[3];
        const int o0 = fc.axis == 0 ? 1 : 0, o1 = fc.axis == 2 ? 1 : 2;
        xyz[fc.axis] = fc.pos;
        xyz[o0] = fc.r0[c];
        xyz[o1] = fc.r1[c];
        const float ds = fc.ds[c];
        for (int f = 0; f < n_freq; ++f) {
          float v[12];
          for (int q = 0; q < 3; ++q)
            for (int k = 0; k < 2; ++k) {
              v[2 * q + k] = ds * fc.J[((size_t(q) * n_freq + f) * nc + c) * 2 + k];
              v[6 + 2 * q + k] = ds * fc.M[((size_t(q) * n_freq + f) * nc + c) * 2 + k];
            }
          Nf2ffCell& cell = host[size_t(f) * n_cells + c0 + c];
          cell.pos = make_float4(xyz[0], xyz[1], xyz[2], 0.f);
          cell.j01 = make_float4(v[0], v[1], v[2], v[3]);
          cell.j2m0 = make_float4(v[4], v[5], v[6], v[7]);
          cell.m12 = make_float4(v[8], v[9], v[10], v[11]);
        }
      }
      c0 += nc;
    }
    DevBuf<Nf2ffCell> d_cells;
    DevBuf<float> d_beta, d_theta, d_phi;
    DevBuf<float2> d_out;
    d_cells.alloc(host.size());
    CK(cudaMemcpy(d_cells.p, host.data(), host.size() * sizeof(Nf2ffCell), cudaMemcpyHostToDevice));
    d_beta.alloc(size_t(n_freq));
    CK(cudaMemcpy(d_beta.p, beta, size_t(n_freq) * 4, cudaMemcpyHostToDevice));
    d_theta.alloc(size_t(n_theta));
    CK(cudaMemcpy(d_theta.p, theta, size_t(n_theta) * 4, cudaMemcpyHostToDevice));
    d_phi.alloc(size_t(n_phi));
    CK(cudaMemcpy(d_phi.p, phi, size_t(n_phi) * 4, cudaMemcpyHostToDevice));
    const size_t n_out = size_t(2) * n_freq * n_theta * n_phi;
    d_out.alloc(n_out);
    const dim3 grid(unsigned((int64_t(n_theta) * n_phi + kNf2ffThreads - 1) / kNf2ffThreads), unsigned(n_freq));
    nf2ff_kernel<<<grid, kNf2ffThreads>>>(d_cells.p, int(n_cells), d_beta.p, d_theta.p, n_theta, d_phi.p, n_phi,
                                          d_out.p);
    CK(cudaGetLastError());
    CK(cudaMemcpy(out, d_out.p, n_out * sizeof(float2), cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"

// ------------------------------------------------ stepping without allocation
//
// fdtd_step_noalloc advances a grid whose device buffers the caller owns, with
// the plain step kernel (fdtd_step_kernel). That kernel reads two small
// engine-built arrays besides the caller's data: the grid descriptor (SimDev)
// and the tile list. The other entry points cudaMalloc them per simulation;
// here they live in one file-scope device array of fixed size, so the call
// allocates nothing on the device. A set-up kernel writes both into the array
// on the caller's stream from its launch parameters (the descriptor by value,
// the tiles from the grid sizes), so the call leaves no host memory behind
// that the GPU still has to read after it returns.
namespace {

constexpr int kNoallocMaxTiles = 65536;          // tile-list capacity (16 B per tile)
constexpr size_t kNoallocDescBytes = 1024;       // room for the SimDev descriptor
constexpr size_t kNoallocScratchBytes = kNoallocDescBytes + size_t(kNoallocMaxTiles) * sizeof(int4);  // 1 MiB + 1 KiB
static_assert(sizeof(SimDev) <= kNoallocDescBytes, "descriptor does not fit its scratch slot");

// Shared by every call on a device, for the life of the process.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoallocMaxDevices] = {};   // device address of the array, per device

// Writes the descriptor and the tile list of one call into the scratch array:
// tiles of 31 x 7 columns in z chunks of zlen planes, x fastest, then y, then
// the chunk (the plain kernel's tile order), as (0, x0 | y0 << 16, z0 | z1 << 16, 0).
__global__ void noalloc_setup_kernel(SimDev d, int zlen, int n_tiles, unsigned char* scratch) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *reinterpret_cast<SimDev*>(scratch) = d;
  int4* tiles = reinterpret_cast<int4*>(scratch + kNoallocDescBytes);
  const int ntx = (d.nx + kTileX - 1) / kTileX, nty = (d.ny + kTileY - 1) / kTileY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_tiles; i += gridDim.x * blockDim.x) {
    const int xt = i % ntx, yt = (i / ntx) % nty, zc = i / (ntx * nty);
    const int x0 = xt * kTileX, y0 = yt * kTileY, z0 = zc * zlen, z1 = min(d.nz, z0 + zlen);
    tiles[i] = make_int4(0, x0 | (y0 << 16), z0 | (z1 << 16), 0);
  }
}

}  // namespace

extern "C" int fdtd_step_noalloc(const fdtd_device_grid* g, int n0, int n_steps, void* stream) {
  if (!g) {
    g_error = "fdtd_step_noalloc: null grid";
    return FDTD_ERR_ARG;
  }
  const int nx = g->nx, ny = g->ny, nz = g->nz, pitch = g->pitch;
  if (nx < 2 || ny < 2 || nz < 2 || nx > 65535 || ny > 65535 || nz > 65535 || pitch < nx) {
    g_error = "fdtd_step_noalloc: dimensions must be 2..65535 cells with pitch >= nx";
    return FDTD_ERR_ARG;
  }
  if (g->nt < 1 || n0 < 0 || n_steps < 0 || int64_t(n0) + n_steps > g->nt) {
    g_error = "fdtd_step_noalloc: steps n0 .. n0+n_steps-1 must lie in [0, nt)";
    return FDTD_ERR_ARG;
  }
  if (g->n_rows < 1 || g->n_rows > 65536 || g->n_probes < 0) {
    g_error = "fdtd_step_noalloc: n_rows must be 1..65536 (a 16-bit index) and n_probes >= 0";
    return FDTD_ERR_ARG;
  }
  const size_t N = size_t(nz) * ny * pitch;
  if (N >= (size_t(1) << 31) - size_t(2) * ny * pitch) {
    g_error = "fdtd_step_noalloc: grid too large for 32-bit cell offsets";
    return FDTD_ERR_LIMIT;
  }
  // the engine's tiling of the plain kernel: 31 x 7 columns, z cut so that
  // about 8 blocks per SM exist (at least 8 planes per chunk)
  const int64_t xy_tiles = int64_t((nx + kTileX - 1) / kTileX) * ((ny + kTileY - 1) / kTileY);
  if (xy_tiles > kNoallocMaxTiles) {
    g_error = "fdtd_step_noalloc: the grid needs " + std::to_string(xy_tiles) +
              " tiles per z chunk; the static tile list holds " + std::to_string(kNoallocMaxTiles);
    return FDTD_ERR_LIMIT;
  }
  if (!g->fields || !g->splits || !g->mat || !g->rows || !g->cell_probes || !g->src || !g->rec || !g->is_src) {
    g_error = "fdtd_step_noalloc: every buffer pointer must be a device address";
    return FDTD_ERR_ARG;
  }
  if (reinterpret_cast<uintptr_t>(g->splits) % 8 != 0 || reinterpret_cast<uintptr_t>(g->rows) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(g->cell_probes) % 8 != 0) {
    g_error = "fdtd_step_noalloc: splits and cell_probes must be 8-byte aligned, rows 16-byte aligned";
    return FDTD_ERR_ARG;
  }
  if (n_steps == 0) return FDTD_OK;
  try {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) throw ArgError{FDTD_ERR_LIMIT, "device ordinal out of range"};
    unsigned char* scratch = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mutex);
      if (!g_noalloc_ptr[dev]) {
        // once per device: host code cannot name the array's device address directly
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
      }
      scratch = g_noalloc_ptr[dev];
    }
    int n_sm = 148;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t want = int64_t(n_sm) * 8;
    int chunks = int(std::max<int64_t>(1, (want + xy_tiles - 1) / xy_tiles));
    chunks = std::min(chunks, std::max(1, nz / 8));
    chunks = int(std::min<int64_t>(chunks, kNoallocMaxTiles / xy_tiles));
    const int zlen = (nz + chunks - 1) / chunks;
    const int n_tiles = int(xy_tiles) * ((nz + zlen - 1) / zlen);
    SimDev d{};
    d.nx = nx; d.ny = ny; d.nz = nz; d.pitch = pitch; d.plane = ny * pitch; d.nt = g->nt;
    for (int b = 0; b < 2; ++b) {
      for (int c = 0; c < 3; ++c) {
        d.E[b][c] = g->fields + (size_t(b) * 6 + c) * N;
        d.H[b][c] = g->fields + (size_t(b) * 6 + 3 + c) * N;
      }
    }
    // the caller's splits cover the whole grid: one z-face store holding every
    // cell, component m of time buffer b at pairs (6 b + m) N
    d.sp.t[4] = nz;
    d.sp.w[kStZlo] = pitch;
    d.sp.h[kStZlo] = ny;
    d.sp.comp[kStZlo] = int64_t(N);
    for (int b = 0; b < 2; ++b) d.sp.base[b] = reinterpret_cast<float2*>(g->splits) + size_t(b) * 6 * N;
    d.mat = g->mat;
    d.rows = reinterpret_cast<const float4*>(g->rows);
    d.cell_probes = reinterpret_cast<const int2*>(g->cell_probes);
    d.src = g->src;
    d.rec = g->rec;
    d.is_src = g->is_src;
    d.cells = int64_t(N);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    noalloc_setup_kernel<<<std::min(1024, (n_tiles + 255) / 256), 256, 0, st>>>(d, zlen, n_tiles, scratch);
    CK(cudaGetLastError());
    const SimDev* d_desc = reinterpret_cast<const SimDev*>(scratch);
    const int4* d_tiles = reinterpret_cast<const int4*>(scratch + kNoallocDescBytes);
    for (int n = n0; n < n0 + n_steps; ++n) {
      fdtd_step_kernel<kTileY><<<n_tiles, dim3(32, kBlockY), 0, st>>>(d_desc, d_tiles, n);
      CK(cudaGetLastError());
    }
    return FDTD_OK;
  } catch (const ArgError& a) {
    g_error = "fdtd_step_noalloc: " + a.msg;
    return a.code;
  } catch (const CudaError& c) {
    g_error = "fdtd_step_noalloc: " + c.where + ": " + cudaGetErrorString(c.code);
    return FDTD_ERR_CUDA;
  }
}
