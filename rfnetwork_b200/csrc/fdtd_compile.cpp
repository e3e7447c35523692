// Host-side compilation of per-component coefficient arrays into a material
// index + coefficient-row table (see fdtd_compile.h).
//
// The reference CUDA engine reads 30 float arrays per cell and step
// (rfnetwork/core/src/solver.cu:116-437). Almost all cells share a handful of
// distinct coefficient tuples, so the engine stores one 16-bit row index per
// cell instead, and the kernels fetch the row from a table. Compilation folds
// three reference behaviours into the rows so the kernels need no special
// cases:
//  1. the x-max PEC wall: solver_init_fields zeroes the last x plane of the
//     Cy, Cz and Dx arrays (rfnetwork/core/src/solver.cpp:294-328);
//  2. the update guards of efield_update_kernel (solver.cu:152-185): a split
//     on the y-max / z-max / x-max boundary is not updated, i.e. keeps its
//     value. A split that is never updated and never receives a source stays
//     exactly zero, so it can take its partner split's Ca with Cb = 0 without
//     changing any result; only a guarded split carrying a source keeps the
//     literal (Ca = 1, Cb = 0) "keep" row;
//  3. split-field storage: a component whose two splits have different Ca
//     (E) or Da (H) -- in the PML slabs -- or that carries a soft source is
//     stored as its two splits, and its cell is flagged for split storage.
//     Every other component is advanced in unsplit form,
//     f' = Ca f + Cb1 d1 + Cb2 d2, which is the same algebra. Inside a
//     single-axis slab only two of the three components of E and of H need
//     their splits (in a z slab, ez and hz decay alike along x and y).
#include "fdtd_compile.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>

namespace rfn {

const char* const kCoefNames[kNumCoef] = {
    "Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z", "Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x",
    "Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y", "Da_hx_y", "Da_hx_z", "Db_hx_y1", "Db_hx_y2",
    "Db_hx_z1", "Db_hx_z2", "Da_hy_z", "Da_hy_x", "Db_hy_z1", "Db_hy_z2", "Db_hy_x1", "Db_hy_x2",
    "Da_hz_x", "Da_hz_y", "Db_hz_x1", "Db_hz_x2", "Db_hz_y1", "Db_hz_y2"};

namespace {

// kCoefNames index -> row slot.
constexpr int kSlotOf[kNumCoef] = {
    R_CA_EX_Y, R_CA_EX_Z, R_CB_EX_Y, R_CB_EX_Z, R_CA_EY_Z, R_CA_EY_X, R_CB_EY_Z, R_CB_EY_X,
    R_CA_EZ_X, R_CA_EZ_Y, R_CB_EZ_X, R_CB_EZ_Y, R_DA_HX_Y, R_DA_HX_Z, R_DB1_HX_Y, R_DB2_HX_Y,
    R_DB1_HX_Z, R_DB2_HX_Z, R_DA_HY_Z, R_DA_HY_X, R_DB1_HY_Z, R_DB2_HY_Z, R_DB1_HY_X, R_DB2_HY_X,
    R_DA_HZ_X, R_DA_HZ_Y, R_DB1_HZ_X, R_DB2_HZ_X, R_DB1_HZ_Y, R_DB2_HZ_Y};

inline uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

struct RowHash {
  size_t operator()(const Row& r) const {
    uint64_t h = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < kRowWords; ++i) {
      h ^= r.w[i] + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
      h *= 0xBF58476D1CE4E5B9ull;
    }
    return size_t(h ^ (h >> 31));
  }
};
struct RowEq {
  bool operator()(const Row& a, const Row& b) const { return std::memcmp(a.w, b.w, sizeof(a.w)) == 0; }
};
using RowMap = std::unordered_map<Row, uint32_t, RowHash, RowEq>;

}  // namespace

GradedIndex::GradedIndex(const CompiledGrid& g, uint32_t mask) : nx(g.nx), ny(g.ny), nz(g.nz) {
  // summed-volume table of flagged cells, indexed [x][y][z] with a zero border:
  // the 2D sums over (y, z) of every x plane (planes in parallel, each thread
  // writing its planes' borders too, so the table needs no serial zero fill),
  // then the running sum along x (plane positions in parallel)
  sy_ = nz + 1;
  sx_ = int64_t(ny + 1) * sy_;
  sv_.reset(new int32_t[size_t(nx + 1) * size_t(sx_)]);
  const int n_threads = int(std::max(1u, std::min(std::thread::hardware_concurrency(), 32u)));
  auto parallel = [n_threads](int64_t n, auto&& body) {  // body(a, b) over [a, b) slices of [0, n)
    const int k = int(std::max<int64_t>(1, std::min<int64_t>(n_threads, n)));
    std::vector<std::thread> pool;
    for (int t = 0; t < k; ++t) pool.emplace_back(body, n * t / k, n * (t + 1) / k);
    for (auto& th : pool) th.join();
  };
  int32_t* const sv = sv_.get();
  parallel(nx, [&](int64_t xa, int64_t xb) {
    if (xa == 0) std::fill(sv, sv + sx_, 0);  // the x = -1 plane
    for (int64_t x = xa; x < xb; ++x) {
      int32_t* P = sv + (x + 1) * sx_;
      std::fill(P, P + sy_, 0);  // the y = -1 row
      for (int y = 0; y < ny; ++y) {
        const uint16_t* id = g.ids.data() + (size_t(x) * ny + y) * nz;
        P[(y + 1) * sy_] = 0;  // the z = -1 entry
        int32_t run = 0;
        for (int z = 0; z < nz; ++z) {
          run += (g.rows[id[z]].w[R_FLAGS] & mask) ? 1 : 0;
          P[(y + 1) * sy_ + z + 1] = run + P[y * sy_ + z + 1];
        }
      }
    }
  });
  parallel(sx_, [&](int64_t ja, int64_t jb) {
    for (int x = 1; x <= nx; ++x) {
      int32_t* cur = sv + x * sx_;
      const int32_t* prev = cur - sx_;
      for (int64_t j = ja; j < jb; ++j) cur[j] += prev[j];
    }
  });
}

int64_t GradedIndex::count(int x0, int x1, int y0, int y1, int z0, int z1) const {
  x0 = std::max(x0, 0); y0 = std::max(y0, 0); z0 = std::max(z0, 0);
  x1 = std::min(x1, nx); y1 = std::min(y1, ny); z1 = std::min(z1, nz);
  if (x1 <= x0 || y1 <= y0 || z1 <= z0) return 0;
  auto at = [&](int x, int y, int z) { return int64_t(sv_[size_t(x * sx_ + y * sy_ + z)]); };
  return at(x1, y1, z1) - at(x0, y1, z1) - at(x1, y0, z1) - at(x1, y1, z0) + at(x0, y0, z1) + at(x0, y1, z0) +
         at(x1, y0, z0) - at(x0, y0, z0);
}

Box3 core_box(const GradedIndex& gi, int halo_x, int align) {
  const int nx = gi.nx, ny = gi.ny, nz = gi.nz;
  auto count = [&](int x0, int x1, int y0, int y1, int z0, int z1) { return gi.count(x0, x1, y0, y1, z0, z1); };
  Box3 b{0, nx, 0, ny, 0, nz};
  for (;;) {
    const int ex0 = b.x0 - halo_x, ey0 = b.y0 - 1, ez0 = b.z0 - 1;
    if (b.empty()) return Box3{};
    if (count(ex0, b.x1, ey0, b.y1, ez0, b.z1) == 0) break;
    // shrink the face whose outermost layer of the extended box holds most
    // graded cells (layers clipped to the grid)
    const int lx = std::max(ex0, 0), ly = std::max(ey0, 0), lz = std::max(ez0, 0);
    const int64_t c[6] = {
        count(lx, lx + 1, ey0, b.y1, ez0, b.z1), count(b.x1 - 1, b.x1, ey0, b.y1, ez0, b.z1),
        count(ex0, b.x1, ly, ly + 1, ez0, b.z1), count(ex0, b.x1, b.y1 - 1, b.y1, ez0, b.z1),
        count(ex0, b.x1, ey0, b.y1, lz, lz + 1), count(ex0, b.x1, ey0, b.y1, b.z1 - 1, b.z1)};
    int best = 0;
    for (int k = 1; k < 6; ++k)
      if (c[k] > c[best]) best = k;
    switch (best) {
      case 0: b.x0 += 1; break;
      case 1: b.x1 -= 1; break;
      case 2: b.y0 += 1; break;
      case 3: b.y1 -= 1; break;
      case 4: b.z0 += 1; break;
      default: b.z1 -= 1; break;
    }
  }
  b.x0 = (b.x0 + align - 1) / align * align;
  if (b.x1 != nx) b.x1 = b.x1 / align * align;
  if (b.empty()) return Box3{};
  return b;
}

bool plan_split_storage(CompiledGrid& g, SplitPlan& plan, std::string& err) {
  plan = SplitPlan();
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const GradedIndex split(g, kFlagESplit | kFlagHSplit);
  // a slab grows while its next layer is more than half split
  auto mostly = [&](int x0, int x1, int y0, int y1, int z0, int z1) {
    const int64_t n = int64_t(x1 - x0) * (y1 - y0) * (z1 - z0);
    return n > 0 && 2 * split.count(x0, x1, y0, y1, z0, z1) > n;
  };
  int* t = plan.t;
  while (t[4] < nz && mostly(0, nx, 0, ny, t[4], t[4] + 1)) ++t[4];
  while (t[4] + t[5] < nz && mostly(0, nx, 0, ny, nz - 1 - t[5], nz - t[5])) ++t[5];
  const int z0 = t[4], z1 = nz - t[5];
  if (z1 > z0) {
    while (t[2] < ny && mostly(0, nx, t[2], t[2] + 1, z0, z1)) ++t[2];
    while (t[2] + t[3] < ny && mostly(0, nx, ny - 1 - t[3], ny - t[3], z0, z1)) ++t[3];
    const int y0 = t[2], y1 = ny - t[3];
    if (y1 > y0) {
      while (t[0] < nx && mostly(t[0], t[0] + 1, y0, y1, z0, z1)) ++t[0];
      while (t[0] + t[1] < nx && mostly(nx - 1 - t[1], nx - t[1], y0, y1, z0, z1)) ++t[1];
    }
  }
  const int64_t ncell = int64_t(nx) * ny * nz;
  const int64_t core = int64_t(std::max(0, nx - t[0] - t[1])) * std::max(0, ny - t[2] - t[3]) *
                       std::max(0, nz - t[4] - t[5]);
  plan.slab_cells = ncell - core;
  // sparse split cells: probe cells keep their (unique) probe-list offset as
  // slot; the others get fresh slots after the probe entries, on rows of their
  // own. They lie in the core box that no slab covers (split_store_of gives
  // the sparse store there), visited in cell order; x planes and (x, y) rows
  // of the core box without split cells are skipped through the summed-volume
  // counts.
  int64_t next = int64_t(g.cell_probes.size());
  const int cx0 = t[0], cx1 = nx - t[1], cy0 = t[2], cy1 = ny - t[3], cz0 = t[4], cz1 = nz - t[5];
  const bool any_sparse = cx1 > cx0 && cy1 > cy0 && cz1 > cz0 && split.count(cx0, cx1, cy0, cy1, cz0, cz1) > 0;
  for (int x = any_sparse ? cx0 : cx1; x < cx1; ++x) {
    if (split.count(x, x + 1, cy0, cy1, cz0, cz1) == 0) continue;
    for (int y = cy0; y < cy1; ++y) {
      if (split.count(x, x + 1, y, y + 1, cz0, cz1) == 0) continue;
      for (int z = cz0; z < cz1; ++z) {
        uint16_t& id = g.ids[(size_t(x) * ny + y) * nz + z];
        const Row& r = g.rows[id];
        if (!(r.w[R_FLAGS] & (kFlagESplit | kFlagHSplit))) continue;
        ++plan.sparse_cells;
        if ((r.w[R_FLAGS] >> 16) != 0) continue;  // a probe cell: its row is its own
        if (g.rows.size() >= 65536) {
          err = "The sparse split cells need more rows than the 16-bit material index addresses.";
          return false;
        }
        Row u = r;
        u.w[R_PROBE] = uint32_t(next++);
        id = uint16_t(g.rows.size());
        g.rows.push_back(u);
      }
    }
  }
  plan.n_sparse = next;
  return true;
}

float row_coefficient(const Row& r, int c) {
  float f;
  std::memcpy(&f, &r.w[kSlotOf[c]], 4);
  return f;
}

bool compile_grid(int nx, int ny, int nz, const float* const* coef, const std::vector<ProbeSpec>& probes,
                  int n_threads, CompiledGrid& out, std::string& err) {
  auto t0 = std::chrono::steady_clock::now();
  if (nx < 2 || ny < 2 || nz < 2) {
    err = "Grid must have at least 2 cells along each axis.";
    return false;
  }
  for (int i = 0; i < kNumCoef; ++i)
    if (!coef[i]) {
      err = std::string("Missing coefficient array ") + kCoefNames[i];
      return false;
    }
  const int64_t ncell = int64_t(nx) * ny * nz;
  out = CompiledGrid();
  out.nx = nx;
  out.ny = ny;
  out.nz = nz;

  // ---- probes: Yee shift and per-cell grouping (solver.cpp:503-525)
  std::vector<std::pair<int64_t, int>> by_cell;  // (cell, probe)
  out.probe_cell.resize(probes.size());
  for (size_t p = 0; p < probes.size(); ++p) {
    const ProbeSpec& q = probes[p];
    if (q.field < 0 || q.field > 5) {
      err = "Invalid probe field type.";
      return false;
    }
    int x = q.i, y = q.j, z = q.k;
    if (q.field == 1 || q.field == 2 || q.field == 3) x -= 1;
    if (q.field == 0 || q.field == 2 || q.field == 4) y -= 1;
    if (q.field == 0 || q.field == 1 || q.field == 5) z -= 1;
    if (x < 0 || y < 0 || z < 0) {
      err = "Source cannot be placed on grid edge";
      return false;
    }
    if (x >= nx || y >= ny || z >= nz) {
      err = "Probe index outside the solver grid";
      return false;
    }
    const int64_t cell = (int64_t(x) * ny + y) * nz + z;
    out.probe_cell[p] = cell;
    by_cell.emplace_back(cell, int(p));
  }
  std::stable_sort(by_cell.begin(), by_cell.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  // cell -> (first entry, count, source-field mask)
  struct CellInfo {
    int first, count;
    unsigned src_mask;
  };
  std::unordered_map<int64_t, CellInfo> cell_info;
  for (size_t e = 0; e < by_cell.size(); ++e) {
    const int p = by_cell[e].second;
    out.cell_probes.push_back({p, probes[p].field});
    auto it = cell_info.find(by_cell[e].first);
    if (it == cell_info.end()) it = cell_info.emplace(by_cell[e].first, CellInfo{int(e), 0, 0u}).first;
    it->second.count += 1;
    if (probes[p].is_source) it->second.src_mask |= 1u << probes[p].field;
  }
  for (auto& kv : cell_info)
    if (kv.second.count > 0xFFFF) {
      err = "Too many probes on one cell.";
      return false;
    }
  // the probe cells in increasing cell order, walked alongside the cells below
  std::vector<std::pair<int64_t, CellInfo>> probe_cells(cell_info.begin(), cell_info.end());
  std::sort(probe_cells.begin(), probe_cells.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });

  // ---- rows, built per x slab in parallel with thread-local dedup
  n_threads = std::max(1, std::min(n_threads, nx));
  std::vector<RowMap> local_maps(n_threads);
  std::vector<std::vector<Row>> local_rows(n_threads);
  // every cell's entry is written by the worker of its x slab (no serial zero fill)
  std::unique_ptr<uint32_t[]> local_ids(new uint32_t[size_t(ncell)]);
  std::vector<int64_t> e_split(n_threads, 0), h_split(n_threads, 0);
  auto work = [&](int t, int xa, int xb) {
    RowMap& map = local_maps[t];
    std::vector<Row>& rows = local_rows[t];
    Row prev;
    uint32_t prev_id = UINT32_MAX;
    std::vector<uint32_t> prev_col(static_cast<size_t>(nz), UINT32_MAX);  // ids of the previous (x, y) column
    int64_t n_esplit = 0, n_hsplit = 0;
    // next probe cell at or after this slab's first cell
    size_t pc = size_t(std::lower_bound(probe_cells.begin(), probe_cells.end(), int64_t(xa) * ny * nz,
                                        [](const auto& a, int64_t c) { return a.first < c; }) -
                       probe_cells.begin());
    for (int x = xa; x < xb; ++x)
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
          const int64_t cell = (int64_t(x) * ny + y) * nz + z;
          Row r;
          for (int c = 0; c < kNumCoef; ++c) r.w[kSlotOf[c]] = fbits(coef[c][cell]);
          if (x == nx - 1)  // solver_init_fields zeroes the last x plane of Cy, Cz, Dx
            for (int s = R_CA_EY_Z; s <= R_DB2_HX_Z; ++s) r.w[s] = 0u;
          unsigned src_mask = 0;
          int probe_first = -1, probe_count = 0;
          if (pc < probe_cells.size() && probe_cells[pc].first == cell) {
            src_mask = probe_cells[pc].second.src_mask;
            probe_first = probe_cells[pc].second.first;
            probe_count = probe_cells[pc].second.count;
            ++pc;
          }
          // guarded (never updated) E splits: ex_y, ez_y at y max; ex_z, ey_z at
          // z max; ey_x, ez_x at x max (solver.cu:152-185)
          const bool frozen[6] = {y == ny - 1, z == nz - 1, z == nz - 1, x == nx - 1, x == nx - 1, y == ny - 1};
          for (int s = 0; s < 6; ++s) {
            if (!frozen[s]) continue;
            const int comp = s / 2, partner = s ^ 1;
            if (src_mask & (1u << comp)) {
              r.w[2 * s] = fbits(1.0f);
              r.w[2 * s + 1] = 0u;
            } else {
              r.w[2 * s] = frozen[partner] ? 0u : r.w[2 * partner];
              r.w[2 * s + 1] = 0u;
            }
          }
          uint32_t flags = 0;
          // a component is stored split when its two splits decay differently
          // (Ca or Da differ: PML) or when it carries a soft source
          const bool comp_diff[6] = {
              r.w[R_CA_EX_Y] != r.w[R_CA_EX_Z], r.w[R_CA_EY_Z] != r.w[R_CA_EY_X],
              r.w[R_CA_EZ_X] != r.w[R_CA_EZ_Y], r.w[R_DA_HX_Y] != r.w[R_DA_HX_Z],
              r.w[R_DA_HY_Z] != r.w[R_DA_HY_X], r.w[R_DA_HZ_X] != r.w[R_DA_HZ_Y]};
          for (int c = 0; c < 6; ++c)
            if (comp_diff[c] || (src_mask & (1u << c))) flags |= kFlagCompSplit0 << c;
          const bool e_diff = comp_diff[0] || comp_diff[1] || comp_diff[2];
          const bool h_diff = comp_diff[3] || comp_diff[4] || comp_diff[5];
          if (flags & (7u * kFlagCompSplit0)) flags |= kFlagESplit;
          if (flags & (0x38u * kFlagCompSplit0)) flags |= kFlagHSplit;
          if (e_diff || h_diff) flags |= kFlagGraded;
          flags |= uint32_t(probe_count) << 16;
          n_esplit += (flags & kFlagESplit) ? 1 : 0;  // thread-local: the shared counters sit in one cache line
          n_hsplit += (flags & kFlagHSplit) ? 1 : 0;
          r.w[R_FLAGS] = flags;
          r.w[R_PROBE] = uint32_t(probe_first);
          // the row is usually that of the cell below (z - 1) or of the cell
          // at the same z one column back (y - 1; e.g. a z-PML slab, whose
          // rows change with z only); the hash table is the last resort
          uint32_t id;
          const uint32_t back = prev_col[size_t(z)];
          if (prev_id != UINT32_MAX && RowEq()(r, prev)) {
            id = prev_id;
          } else if (back != UINT32_MAX && RowEq()(r, rows[back])) {
            id = back;
            prev = r;
            prev_id = id;
          } else {
            auto it = map.find(r);
            if (it == map.end()) {
              it = map.emplace(r, uint32_t(rows.size())).first;
              rows.push_back(r);
            }
            id = it->second;
            prev = r;
            prev_id = id;
          }
          prev_col[size_t(z)] = id;
          local_ids[size_t(cell)] = id;
        }
    e_split[t] = n_esplit;
    h_split[t] = n_hsplit;
  };
  {
    std::vector<std::thread> pool;
    const int base = nx / n_threads, rem = nx % n_threads;
    int xa = 0;
    for (int t = 0; t < n_threads; ++t) {
      const int xb = xa + base + (t < rem ? 1 : 0);
      pool.emplace_back(work, t, xa, xb);
      xa = xb;
    }
    for (auto& th : pool) th.join();
  }

  // ---- merge the thread-local tables; row 0 is the all-zero row
  RowMap global;
  Row zero;
  std::memset(zero.w, 0, sizeof(zero.w));
  zero.w[R_PROBE] = uint32_t(-1);
  global.emplace(zero, 0u);
  out.rows.push_back(zero);
  std::vector<std::vector<uint32_t>> remap(n_threads);
  for (int t = 0; t < n_threads; ++t) {
    remap[t].resize(local_rows[t].size());
    for (size_t i = 0; i < local_rows[t].size(); ++i) {
      auto ins = global.emplace(local_rows[t][i], uint32_t(out.rows.size()));
      if (ins.second) out.rows.push_back(local_rows[t][i]);
      remap[t][i] = ins.first->second;
    }
  }
  if (out.rows.size() > 65536) {
    err = "The coefficient arrays hold " + std::to_string(out.rows.size()) +
          " distinct cell rows; the material table holds at most 65536.";
    return false;
  }
  out.ids.resize(size_t(ncell));
  {
    std::vector<std::thread> pool;
    const int base = nx / n_threads, rem = nx % n_threads;
    int xa = 0;
    for (int t = 0; t < n_threads; ++t) {
      const int xb = xa + base + (t < rem ? 1 : 0);
      pool.emplace_back([&, t, xa, xb] {
        const size_t a = size_t(xa) * ny * nz, b = size_t(xb) * ny * nz;
        for (size_t c = a; c < b; ++c) out.ids[c] = uint16_t(remap[t][local_ids[c]]);
      });
      xa = xb;
    }
    for (auto& th : pool) th.join();
  }
  for (int t = 0; t < n_threads; ++t) {
    out.e_split_cells += e_split[t];
    out.h_split_cells += h_split[t];
  }
  out.compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

}  // namespace rfn
