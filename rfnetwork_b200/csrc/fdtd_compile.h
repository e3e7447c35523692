// Host-side compilation of the reference's 30 per-component coefficient
// arrays into a per-cell material index plus a table of distinct coefficient
// rows, the form the B200 kernels read.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace rfn {

constexpr int kNumCoef = 30;

// Coefficient names in the key order of the dict built at
// rfnetwork/solver.py:1473-1518.
extern const char* const kCoefNames[kNumCoef];

// Position of each coefficient inside a table row (the kernel's order).
enum RowSlot : int {
  // E: (Ca, Cb) per split, splits ordered as in solver.h:20-39
  R_CA_EX_Y = 0, R_CB_EX_Y, R_CA_EX_Z, R_CB_EX_Z,
  R_CA_EY_Z, R_CB_EY_Z, R_CA_EY_X, R_CB_EY_X,
  R_CA_EZ_X, R_CB_EZ_X, R_CA_EZ_Y, R_CB_EZ_Y,
  // H: (Da, Db1, Db2) per split, solver.h:41-79
  R_DA_HX_Y = 12, R_DB1_HX_Y, R_DB2_HX_Y, R_DA_HX_Z, R_DB1_HX_Z, R_DB2_HX_Z,
  R_DA_HY_Z, R_DB1_HY_Z, R_DB2_HY_Z, R_DA_HY_X, R_DB1_HY_X, R_DB2_HY_X,
  R_DA_HZ_X, R_DB1_HZ_X, R_DB2_HZ_X, R_DA_HZ_Y, R_DB1_HZ_Y, R_DB2_HZ_Y,
  R_FLAGS = 30,  // bit 0: E split storage, bit 1: H split storage, bits 8..13: which component
                 // (ex ey ez hx hy hz) is stored split, bits 16..31: probe entries
  R_PROBE = 31,  // first entry of this cell in the per-cell probe list (-1 if none)
  kRowWords = 32
};
constexpr uint32_t kFlagESplit = 1u;
constexpr uint32_t kFlagHSplit = 2u;
// the cell's split coefficients differ (a PML cell), as opposed to a cell that
// is split only because it carries a soft source
constexpr uint32_t kFlagGraded = 4u;
// component c (0..5 = ex ey ez hx hy hz) of the cell is stored as its two
// splits; the other components of a split cell are advanced unsplit
constexpr uint32_t kFlagCompSplit0 = 1u << 8;

struct Row {
  uint32_t w[kRowWords];
};

struct ProbeSpec {
  int field;          // 0..5
  int i, j, k;        // full-grid component index
  int is_source;
};

// One entry of the per-cell probe list: probe index and its field code.
struct CellProbe {
  int probe;
  int field;
};

struct CompiledGrid {
  int nx = 0, ny = 0, nz = 0;
  std::vector<Row> rows;                 // distinct rows; row 0 is all zero
  std::vector<uint16_t> ids;             // per cell, reference order [x][y][z]
  std::vector<CellProbe> cell_probes;    // grouped per probe cell
  std::vector<int64_t> probe_cell;       // per probe: cell index (x*ny + y)*nz + z
  int64_t e_split_cells = 0, h_split_cells = 0;
  double compile_ms = 0;
};

// Where the split pairs of a grid live. The PML slabs (runs of planes, rows
// or columns at a face in which most cells are split) each get a store of
// their own, in the priority z faces, then y faces, then x faces: a cell
// belongs to the first slab that contains it. A split cell outside every slab
// (a soft-source cell, or a split cell of a model without slabs) is "sparse":
// its pairs sit at the slot its row's word 31 names in a sparse store, and its
// row is unique to it.
enum SplitStore : int { kStoreXlo = 0, kStoreXhi, kStoreYlo, kStoreYhi, kStoreZlo, kStoreZhi, kStoreSparse };

struct SplitPlan {
  int t[6] = {0, 0, 0, 0, 0, 0};  // slab thickness in cells: x-lo, x-hi, y-lo, y-hi, z-lo, z-hi
  int64_t n_sparse = 0;           // sparse slots (word-31 values 0 .. n_sparse-1)
  int64_t slab_cells = 0;         // cells inside the slabs
  int64_t sparse_cells = 0;       // split cells outside them
};

// Store of cell (x, y, z) under plan t (kStoreSparse: outside every slab).
inline int split_store_of(const int* t, int nx, int ny, int nz, int x, int y, int z) {
  if (z < t[4]) return kStoreZlo;
  if (z >= nz - t[5]) return kStoreZhi;
  if (y < t[2]) return kStoreYlo;
  if (y >= ny - t[3]) return kStoreYhi;
  if (x < t[0]) return kStoreXlo;
  if (x >= nx - t[1]) return kStoreXhi;
  return kStoreSparse;
}

// Finds the slabs of a compiled grid and gives every sparse split cell a
// unique row whose word 31 is its sparse slot (a probe cell keeps its
// probe-list offset, already unique). Returns false with `err` when the
// table would exceed 65536 rows.
bool plan_split_storage(CompiledGrid& g, SplitPlan& plan, std::string& err);

// Builds the table. coef[i] points to kCoefNames[i]'s (nx, ny, nz) array.
// Returns false with `err` set on invalid input or when more than 65535
// distinct rows are needed.
bool compile_grid(int nx, int ny, int nz, const float* const* coef, const std::vector<ProbeSpec>& probes,
                  int n_threads, CompiledGrid& out, std::string& err);

// Expands a row back to the coefficient the reference kernel would apply to
// split `c` (coefficient index into kCoefNames) -- used by tests.
float row_coefficient(const Row& r, int c);

struct Box3 {
  int x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
  bool empty() const { return x1 <= x0 || y1 <= y0 || z1 <= z0; }
};

// Counts the cells of a compiled grid whose row flags intersect `mask`
// (default: graded PML cells) in boxes, in O(1) through a summed-volume table.
class GradedIndex {
 public:
  explicit GradedIndex(const CompiledGrid& g, uint32_t mask = kFlagGraded);
  // flagged cells in [x0,x1) x [y0,y1) x [z0,z1), clipped to the grid
  int64_t count(int x0, int x1, int y0, int y1, int z0, int z1) const;
  int nx, ny, nz;

 private:
  std::unique_ptr<int32_t[]> sv_;  // every entry written by the constructor's parallel passes
  int64_t sx_, sy_;
};

// The "core" of a grid: a box whose cells, together with the halo the fused
// kernel recomputes (x0-halo_x .. x0-1, y0-1, z0-1), hold no graded (PML)
// split cell. x0 is a multiple of `align`, x1 one too unless it is nx.
// Everything outside it is the PML shell. Empty when no such box exists.
Box3 core_box(const GradedIndex& gi, int halo_x, int align);

}  // namespace rfn
