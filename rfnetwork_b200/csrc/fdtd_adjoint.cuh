// Discrete adjoint of the FDTD time step, for gradients of objectives of the
// probe series with respect to the E-update coefficients of a box of cells.
//
// The forward step n (fdtd_step_kernel / fdtd_step_stream_kernel) is linear
// in the state. Writing every E and H component as a pair of split halves,
//   E  s_{2c}' = Ca_{2c} s_{2c} + Cb_{2c} dA_c(H),
//      s_{2c+1}' = Ca_{2c+1} s_{2c+1} + Cb_{2c+1} dB_c(H),    E_c' = s_{2c}' + s_{2c+1}'
//   H  h_s' = Da_s h_s + Db2_s e(own) - Db1_s e(-1 neighbour),  H_c' = h_{2c}' + h_{2c+1}'
// (sources add constants; probes record the totals after the step). An
// unsplit cell is the case of equal decays, whose stored total is the sum.
//
// The adjoint state mirrors the forward storage: for an unsplit cell both
// halves of a pair carry the same adjoint (d/ds_k of E = s_0 + s_1 is the
// same for both halves, and equal decays keep them equal), so one total per
// component is kept, in a [2 buffers][3] array like the fields; split cells
// (PML slabs, source cells) keep both halves in [2][6] arrays like the split
// fields. One reverse step is one launch, adj_step_kernel, which walks z
// upwards through a 30 x TY tile much as the forward kernel does:
//   E part   mu = lamE + (own Db2 lamH) - (Db1 lamH of the +1 neighbours),
//            lamE' = Ca mu, and the adjoints of the H differences ad = Cb mu,
//            computed on the tile and its -1 halo row / column;
//   H part   lamH' = Da lamH + (ad of the -1 neighbours - own ad), the
//            transposed differences, with the -1 neighbours' ad taken by warp
//            shuffle (x), shared memory (y) and registers (z);
//   records  the adjoints dJ/d(record of step n-1) of this cell's probes are
//            added to lamE' / lamH' as they are stored;
//   gradient mu times the forward history of the box cells, accumulated in
//            FP64: dJ/dCa = sum mu E^n, dJ/dCb1 = sum mu dA(H^n), dJ/dCb2 =
//            sum mu dB(H^n).
// Reverse step n reads buffer n & 1 and writes the other; the history of step
// n sits at slot n - hist_n0 of each simulation's hist.
#pragma once

#include <cstdint>

#include "fdtd_kernels.cuh"

namespace rfn {

struct AdjSim {
  int nx, ny, nz, pitch, plane, nt;
  const uint16_t* mat;       // material index [z][y][pitch]
  const float4* rows;        // 8 float4 per table row
  const int2* cell_probes;   // (probe, field) grouped per probe cell
  int64_t N;                 // floats per component array
  // adjoint state, [2 buffers][6][N]: E totals ex ey ez, then H totals hx hy hz
  // (unsplit cells); halves [2][12][N]: ex_y ex_z ey_z ey_x ez_x ez_y, then
  // hx_y hx_z hy_z hy_x hz_x hz_y (split cells; null without split cells)
  float* lam;
  float* lams;
  const float* radj;         // [P][nt] dJ/d(record of probe p at step n)
  const int* probe_idx;      // [P] cell offset of each probe
  const int* probe_field;    // [P] 0..5 = ex ey ez hx hy hz
  int n_probes;
  int bx0, bx1, by0, by1, bz0, bz1;  // gradient box (cells)
  int64_t nb;                // cells in the box
  double* grad;              // [3 components][Ca, Cb1, Cb2][box cells]
  const float* hist;         // forward history: [9][nb] per step = E_x E_y E_z, dA_x dB_x .. dB_z
};

// Box history of one simulation at one step: E^n and the six H differences
// the E update of step n uses.
struct CapSim {
  SimDev s;
  int bx0, bx1, by0, by1, bz0, bz1;
  int64_t nb;
  float* hist;               // [steps][9][nb]
};

__device__ __forceinline__ float adj_ld(const float* p, int i) { return __ldg(p + i); }

// The adjoint halves of the H pairs of one cell (totals duplicated for an
// unsplit cell); tot / half point at component 0 of the H totals / halves.
__device__ __forceinline__ void adj_load_h(const float* tot, const float* half, int64_t N, int idx, uint32_t fl,
                                           float (&h)[6]) {
  if (fl & kHSplit) {
#pragma unroll
    for (int k = 0; k < 6; ++k) h[k] = adj_ld(half + k * N, idx);
  } else {
    const float hx = adj_ld(tot, idx), hy = adj_ld(tot + N, idx), hz = adj_ld(tot + 2 * N, idx);
    h[0] = hx; h[1] = hx; h[2] = hy; h[3] = hy; h[4] = hz; h[5] = hz;
  }
}

__device__ __forceinline__ uint32_t adj_flags(const float4* row) { return __float_as_uint(__ldg(row + 7).z); }

// Per-cell arithmetic of one reverse step, with the rounding fixed by
// intrinsics so that every kernel that uses it gives the same bits.
//
// E part: from the cell's E adjoint lE (totals in 0..2, or six halves), its
// own H adjoint h (six halves; an unsplit cell's halves repeat its totals),
// the Db1-weighted H adjoints of its +1 neighbours (z: qz_hx, qz_hy; x:
// qx_hy, qx_hz; y: qy_hx, qy_hz) and its table row: mu, lamE' (into lE) and
// the adjoints ad of the six H differences.
__device__ __forceinline__ void adj_e_part(const float4& ra, const float4& rb, const float4& rd, const float4& p,
                                           const float4& q, const float4& u, const float4& v, const float4& r7,
                                           uint32_t fl, const float (&h)[6], float qz_hx, float qz_hy, float qx_hy,
                                           float qx_hz, float qy_hx, float qy_hz, float (&lE)[6], float (&mu)[6],
                                           float (&ad)[6]) {
  // Db2 slots: hx_y p.z, hx_z q.y, hy_z u.x, hy_x u.w, hz_x v.z, hz_y r7.y
  const float aEx = __fadd_rn(__fmaf_rn(u.x, h[2], -qz_hy), __fmaf_rn(r7.y, h[5], -qy_hz));
  const float aEy = __fadd_rn(__fmaf_rn(q.y, h[1], -qz_hx), __fmaf_rn(v.z, h[4], -qx_hz));
  const float aEz = __fadd_rn(__fmaf_rn(p.z, h[0], -qy_hx), __fmaf_rn(u.w, h[3], -qx_hy));
  if (!(fl & kESplit)) {
    const float mx = __fadd_rn(lE[0], aEx), my = __fadd_rn(lE[1], aEy), mz = __fadd_rn(lE[2], aEz);
    mu[0] = mx; mu[1] = mx; mu[2] = my; mu[3] = my; mu[4] = mz; mu[5] = mz;
    lE[0] = __fmul_rn(ra.x, mx); lE[1] = __fmul_rn(rb.x, my); lE[2] = __fmul_rn(rd.x, mz);
  } else {
    const float aE[3] = {aEx, aEy, aEz};
    const float ca[6] = {ra.x, ra.z, rb.x, rb.z, rd.x, rd.z};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      mu[k] = __fadd_rn(lE[k], aE[k / 2]);
      lE[k] = __fmul_rn(ca[k], mu[k]);
    }
  }
  const float cb[6] = {ra.y, ra.w, rb.y, rb.w, rd.y, rd.w};
#pragma unroll
  for (int k = 0; k < 6; ++k) ad[k] = __fmul_rn(cb[k], mu[k]);
}

// H part: lamH' of a cell from its H adjoint h, its ad and the ad of its -1
// neighbours (y: a0_m, a5_m; x: a3_m, a4_m; z: a1_p, a2_p).
__device__ __forceinline__ void adj_h_part(const float4& p, const float4& q, const float4& u, const float4& v,
                                           uint32_t fl, const float (&h)[6], const float (&ad)[6], float a0_m,
                                           float a5_m, float a3_m, float a4_m, float a1_p, float a2_p,
                                           float (&lh)[6]) {
  const float aH[3] = {__fadd_rn(__fsub_rn(a2_p, ad[2]), __fsub_rn(a5_m, ad[5])),
                       __fadd_rn(__fsub_rn(a1_p, ad[1]), __fsub_rn(a4_m, ad[4])),
                       __fadd_rn(__fsub_rn(a0_m, ad[0]), __fsub_rn(a3_m, ad[3]))};
  if (!(fl & kHSplit)) {
    lh[0] = __fmaf_rn(p.x, h[0], aH[0]);
    lh[1] = __fmaf_rn(q.z, h[2], aH[1]);
    lh[2] = __fmaf_rn(v.x, h[4], aH[2]);
  } else {
    const float da[6] = {p.x, p.w, q.z, u.y, v.x, v.w};
#pragma unroll
    for (int k = 0; k < 6; ++k) lh[k] = __fmaf_rn(da[k], h[k], aH[k / 2]);
  }
}

// dJ/d(Ca, Cb1, Cb2) of one box cell accumulated for one step (FP64).
__device__ __forceinline__ void adj_grad_cell(double* grad, int64_t nb, int64_t bi, const float* hs,
                                              const float (&mu)[6]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double* g = grad + 3 * k * nb + bi;
    g[0] = __fma_rn(double(mu[2 * k]), double(__ldg(hs + k * nb + bi)), g[0]);
    g[nb] = __fma_rn(double(mu[2 * k]), double(__ldg(hs + (3 + 2 * k) * nb + bi)), g[nb]);
    g[2 * nb] = __fma_rn(double(mu[2 * k + 1]), double(__ldg(hs + (4 + 2 * k) * nb + bi)), g[2 * nb]);
  }
}

// Tile of the adjoint step kernel: lane 0 is the -1 halo column, lanes 1..30
// the owned columns and lane 31 only provides Db1 lamH of the column above
// the tile (x0 + 30) to lane 30; warp 0 is the -1 halo row, warps 1..TY the
// owned rows and warp TY+1 only provides Db1 lamH of the row above the tile.
constexpr int kAdjTileX = 30;
constexpr int kAdjTileY = 7;

template <int TY, int MINB>
__global__ void __launch_bounds__(32 * (TY + 2), MINB)
adj_step_kernel(const AdjSim* __restrict__ sims, const int4* __restrict__ tiles, int n, int hist_n0) {
  const int4 t = tiles[blockIdx.x];
  const AdjSim& A = sims[t.x];
  const int x0 = t.y & 0xffff, y0 = int(unsigned(t.y) >> 16), z0 = t.z & 0xffff, z1 = int(unsigned(t.z) >> 16);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int c = x0 - 1 + lane;  // this lane's column
  const int r = y0 - 1 + w;     // this warp's row
  const int nx = A.nx, ny = A.ny, nz = A.nz, pitch = A.pitch, plane = A.plane;
  const bool in_xy = c >= 0 && c < nx && r >= 0 && r < ny;
  const bool worker = lane < 31 && w <= TY;  // computes E (tile and -1 halo)
  const bool own = in_xy && lane >= 1 && lane <= 30 && w >= 1 && w <= TY;
  const int cur = n & 1, nxt = cur ^ 1;
  const int col = r * pitch + c;
  const int64_t N = A.N;
  const float* __restrict__ rE = A.lam + cur * 6 * N;    // read: E totals, then H totals
  const float* __restrict__ rH = rE + 3 * N;
  float* __restrict__ wE = A.lam + nxt * 6 * N;          // write
  float* __restrict__ wH = wE + 3 * N;
  const float* __restrict__ rEs = A.lams + cur * 12 * N;  // halves (split cells only)
  const float* __restrict__ rHs = rEs + 6 * N;
  float* __restrict__ wEs = A.lams + nxt * 12 * N;
  float* __restrict__ wHs = wEs + 6 * N;
  const uint16_t* __restrict__ mat = A.mat;
  const float4* __restrict__ rows = A.rows;

  __shared__ float s_qhx[2][TY + 2][32];  // Db1 lamH of hx_y, read by the row below
  __shared__ float s_qhz[2][TY + 2][32];  // Db1 lamH of hz_y
  __shared__ float s_a0[2][TY + 2][32];   // ad of dA_x (= dhz_y), read by the row above
  __shared__ float s_a5[2][TY + 2][32];   // ad of dB_z (= dhx_y)

  auto mat_at = [&](int z) -> int { return (in_xy && z >= 0 && z < nz) ? int(__ldg(mat + z * plane + col)) : 0; };
  auto flags_of = [&](int id) -> uint32_t { return adj_flags(rows + 8 * id); };

  // register pipeline along z: material ids four planes ahead, flags three,
  // H adjoints two and E adjoints one, so every load of a plane depends on
  // registers only and is consumed one plane after it was issued
  auto load_e = [&](int z, uint32_t fl, float (&e)[6]) {
    if (!(worker && in_xy && z >= 0 && z < nz)) return;
    const int i = z * plane + col;
    if (fl & kESplit) {
#pragma unroll
      for (int k = 0; k < 6; ++k) e[k] = adj_ld(rEs + k * N, i);
    } else {
      e[0] = adj_ld(rE, i); e[1] = adj_ld(rE + N, i); e[2] = adj_ld(rE + 2 * N, i);
    }
  };
  auto load_h = [&](int z, uint32_t fl, float (&h)[6]) {
    if (in_xy && z >= 0 && z < nz) adj_load_h(rH, rHs, N, z * plane + col, fl, h);
  };
  int id_c = mat_at(z0 - 1);
  int id_n1 = mat_at(z0);
  int id_n2 = mat_at(z0 + 1);
  int id_n3 = mat_at(z0 + 2);
  uint32_t fl_c = flags_of(id_c);
  uint32_t fl_n1 = flags_of(id_n1);
  uint32_t fl_n2 = flags_of(id_n2);
  float h_c[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, h_n[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float e_c[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  load_h(z0 - 1, fl_c, h_c);
  load_h(z0, fl_n1, h_n);
  load_e(z0 - 1, fl_c, e_c);
  {
    const float4* rc = rows + 8 * id_c;
    s_qhx[(z0 - 1) & 1][w][lane] = __fmul_rn(__ldg(rc + 3).y, h_c[0]);
    s_qhz[(z0 - 1) & 1][w][lane] = __fmul_rn(__ldg(rc + 7).x, h_c[5]);
  }
  float a1_p = 0.f, a2_p = 0.f;
  __syncthreads();

  for (int z = z0 - 1; z < z1; ++z) {
    const bool zin = z >= 0 && z < nz;
    const bool live = in_xy && zin;
    const int idx = z * plane + col;
    const int buf = z & 1;

    // ---- loads for the planes ahead (addresses from registers only)
    const int id_n4 = mat_at(z + 4);
    const uint32_t fl_n3 = flags_of(id_n3);
    // the table row two planes ahead into L1 where the index changes (z-graded PML rows)
    if (id_n2 != id_n1) prefetch_l1(rows + 8 * id_n2);
    float h_n2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, e_n[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    load_h(z + 2, fl_n2, h_n2);
    load_e(z + 1, fl_n1, e_n);
    // ---- table rows of this plane and of the look-ahead (the Db1 words of
    // hx_y, hx_z, hy_z and hz_y: this plane's own where the index is the same)
    const float4* row = rows + 8 * id_c;
    const float4 ra = __ldg(row + 0), rb = __ldg(row + 1), rd = __ldg(row + 2);
    const float4 p = __ldg(row + 3), q = __ldg(row + 4), u = __ldg(row + 5), v = __ldg(row + 6), r7 = __ldg(row + 7);
    float pn_y = p.y, qn_x = q.x, qn_w = q.w, r7n_x = r7.x;
    if (id_n1 != id_c) {
      const float4* rn = rows + 8 * id_n1;
      pn_y = __ldg(&rn[3].y); qn_x = __ldg(&rn[4].x); qn_w = __ldg(&rn[4].w); r7n_x = __ldg(&rn[7].x);
    }
    float lE[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) lE[k] = e_c[k];

    // ---- Db1 lamH of the +1 neighbours: z+1 from the look-ahead, x+1 from
    // the lane on the right, y+1 from the row above (written last plane)
    const float qz_hx = __fmul_rn(qn_x, h_n[1]), qz_hy = __fmul_rn(qn_w, h_n[2]);
    const float qx_hy = __shfl_down_sync(0xffffffffu, __fmul_rn(u.z, h_c[3]), 1);
    const float qx_hz = __shfl_down_sync(0xffffffffu, __fmul_rn(v.y, h_c[4]), 1);
    const float qy_hx = s_qhx[buf][w + (w <= TY ? 1 : 0)][lane];
    const float qy_hz = s_qhz[buf][w + (w <= TY ? 1 : 0)][lane];
    // and this column's own values at z+1 for the row below, next plane
    s_qhx[buf ^ 1][w][lane] = __fmul_rn(pn_y, h_n[0]);
    s_qhz[buf ^ 1][w][lane] = __fmul_rn(r7n_x, h_n[5]);

    // ---- E part: mu, lamE', ad
    float mu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, ad[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (live && worker)
      adj_e_part(ra, rb, rd, p, q, u, v, r7, fl_c, h_c, qz_hx, qz_hy, qx_hy, qx_hz, qy_hx, qy_hz, lE, mu, ad);

    // ---- -1 neighbours' ad
    s_a0[buf][w][lane] = ad[0];
    s_a5[buf][w][lane] = ad[5];
    const float a3_m = __shfl_up_sync(0xffffffffu, ad[3], 1);
    const float a4_m = __shfl_up_sync(0xffffffffu, ad[4], 1);
    __syncthreads();

    if (own && z >= z0 && zin) {
      const float a0_m = s_a0[buf][w - 1][lane];
      const float a5_m = s_a5[buf][w - 1][lane];
      float lh[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      adj_h_part(p, q, u, v, fl_c, h_c, ad, a0_m, a5_m, a3_m, a4_m, a1_p, a2_p, lh);
      // adjoints of this cell's records of step n-1 (E^n, H^n)
      const int np = int(fl_c >> 16);
      if (np && n >= 1) {
        const int first = __float_as_int(r7.w);
        for (int e = 0; e < np; ++e) {
          const int2 pe = __ldg(A.cell_probes + first + e);
          const float rv = __ldg(A.radj + size_t(pe.x) * A.nt + (n - 1));
          // both halves of a split pair, or the total (slots 0..2) of an unsplit cell
          const bool is_e = pe.y < 3;
          const int cc = is_e ? pe.y : pe.y - 3;
          const bool sp = (fl_c & (is_e ? kESplit : kHSplit)) != 0;
#pragma unroll
          for (int k = 0; k < 6; ++k)
            if (sp ? (k / 2 == cc) : (k == cc)) {
              if (is_e) lE[k] = __fadd_rn(lE[k], rv);
              else lh[k] = __fadd_rn(lh[k], rv);
            }
        }
      }
      if (fl_c & kESplit) {
#pragma unroll
        for (int k = 0; k < 6; ++k) wEs[k * N + idx] = lE[k];
      } else {
        wE[idx] = lE[0]; wE[N + idx] = lE[1]; wE[2 * N + idx] = lE[2];
      }
      if (fl_c & kHSplit) {
#pragma unroll
        for (int k = 0; k < 6; ++k) wHs[k * N + idx] = lh[k];
      } else {
        wH[idx] = lh[0]; wH[N + idx] = lh[1]; wH[2 * N + idx] = lh[2];
      }
      if (A.hist && c >= A.bx0 && c < A.bx1 && r >= A.by0 && r < A.by1 && z >= A.bz0 && z < A.bz1) {
        const int bny = A.by1 - A.by0, bnz = A.bz1 - A.bz0;
        const int64_t nb = A.nb;
        const int64_t bi = (int64_t(c - A.bx0) * bny + (r - A.by0)) * bnz + (z - A.bz0);
        const float* hs = A.hist + int64_t(n - hist_n0) * 9 * nb;
        adj_grad_cell(A.grad, nb, bi, hs, mu);
      }
    }
    a1_p = ad[1];
    a2_p = ad[2];
    id_c = id_n1;
    fl_c = fl_n1;
    id_n1 = id_n2;
    fl_n1 = fl_n2;
    id_n2 = id_n3;
    fl_n2 = fl_n3;
    id_n3 = id_n4;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      h_c[k] = h_n[k];
      h_n[k] = h_n2[k];
      e_c[k] = e_n[k];
    }
  }
}

// Adjoints of the records of step `step` into buffer `buf` (the start of the
// reverse sweep; later steps add theirs inside adj_step_kernel). One block
// row per simulation.
__global__ void adj_inject_kernel(const AdjSim* __restrict__ sims, int step, int buf) {
  const AdjSim& A = sims[blockIdx.y];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.n_probes) return;
  const float rv = A.radj[size_t(p) * A.nt + step];
  if (rv == 0.f) return;
  const int idx = A.probe_idx[p], f = A.probe_field[p];
  const uint32_t fl = adj_flags(A.rows + 8 * A.mat[idx]);
  const int64_t N = A.N;
  // field f: total f of [E totals, H totals], or halves 2f, 2f+1 of the 12 halves
  if (fl & (f < 3 ? kESplit : kHSplit)) {
    float* h = A.lams + buf * 12 * N;
    atomicAdd(h + (2 * f) * N + idx, rv);
    atomicAdd(h + (2 * f + 1) * N + idx, rv);
  } else {
    atomicAdd(A.lam + (buf * 6 + f) * N + idx, rv);
  }
}

// Forward history of the boxes at the start of step n (fields of buffer
// n & 1), written at step slot n - n0. One block row per simulation.
__global__ void adj_capture_kernel(const CapSim* __restrict__ caps, int n, int n0) {
  const CapSim& C = caps[blockIdx.y];
  const SimDev& s = C.s;
  const int bnx = C.bx1 - C.bx0, bny = C.by1 - C.by0, bnz = C.bz1 - C.bz0;
  (void)bnx;
  const int64_t nb = C.nb;
  float* hist = C.hist + int64_t(n - n0) * 9 * nb;
  const int b = n & 1;
  const float* const* E = s.E[b];
  const float* const* H = s.H[b];
  for (int64_t bi = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; bi < nb; bi += int64_t(gridDim.x) * blockDim.x) {
    const int zz = int(bi % bnz), yy = int((bi / bnz) % bny), xx = int(bi / (int64_t(bnz) * bny));
    const int x = C.bx0 + xx, y = C.by0 + yy, z = C.bz0 + zz;
    const int idx = z * s.plane + y * s.pitch + x;
    auto h = [&](int c, bool ok, int off) { return ok ? H[c][idx + off] : 0.f; };
    const bool xn = x + 1 < s.nx, yn = y + 1 < s.ny, zn = z + 1 < s.nz;
    const float hx = H[0][idx], hy = H[1][idx], hz = H[2][idx];
    hist[0 * nb + bi] = E[0][idx];
    hist[1 * nb + bi] = E[1][idx];
    hist[2 * nb + bi] = E[2][idx];
    hist[3 * nb + bi] = h(2, yn, s.pitch) - hz;  // dA_x = dhz_y
    hist[4 * nb + bi] = h(1, zn, s.plane) - hy;  // dB_x = dhy_z
    hist[5 * nb + bi] = h(0, zn, s.plane) - hx;  // dA_y = dhx_z
    hist[6 * nb + bi] = h(2, xn, 1) - hz;        // dB_y = dhz_x
    hist[7 * nb + bi] = h(1, xn, 1) - hy;        // dA_z = dhy_x
    hist[8 * nb + bi] = h(0, yn, s.pitch) - hx;  // dB_z = dhx_y
  }
}

}  // namespace rfn
