// sm_100a kernels of the FDTD time loop.
//
// One launch of `fdtd_step_kernel` advances every cell of every simulation in
// a batch by one full Yee step: E^{n} -> E^{n+1} (efield_update_kernel,
// rfnetwork/core/src/solver.cu:116-191), soft sources / E probes
// (e_probe_update_kernel, solver.cu:439-490), H^{n} -> H^{n+1}
// (hfield_update_kernel, solver.cu:278-356) and H sources / probes
// (h_probe_update_kernel, solver.cu:492-543) -- four launches per step in the
// reference, one here.
//
// Layout in HBM (per simulation, GPU index space of the reference):
//   fields   float32 [z][y][x], x fastest, row pitch a multiple of 32 floats;
//            two buffers per field (step n reads buffer n&1, writes the other),
//            so a block can recompute its halo from consistent step-n data
//            while neighbours already write step n+1.
//   splits   the two split components of E (ex_y, ex_z, ...) and H, stored
//            as pairs: float2 [component][z][y][x] = (first, second split),
//            read and written only for the components the material table
//            flags as split (PML slabs, source cells); the other components
//            of every cell are stored as totals in the field arrays.
//   material uint16 [z][y][x] row index into a table of 32-word rows: the
//            cell's 30 update coefficients + flags + probe-list offset.
//
// Work decomposition: a block owns a tile of 31 (x) by TY (y) cells and a
// z range, with one warp per y row plus one halo row below (y0-1) and lane 0
// on the halo column (x0-1). It streams up through z: at plane z every lane
// computes E^{n+1}(z) for its column, trades x neighbours by warp shuffle and
// y neighbours through shared memory, then the owned cells compute
// H^{n+1}(z) from E^{n+1}(z) and E^{n+1}(z-1) (kept in registers). The halo
// row / column recompute E so no second sweep over memory is needed.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rfn {

constexpr int kTileX = 31;        // cells owned per tile along x (lane 0 is the halo column)
constexpr int kTileY = 7;         // rows owned per tile along y (warp 0 is the halo row)
constexpr int kBlockY = kTileY + 1;

constexpr uint32_t kESplit = 1u, kHSplit = 2u;
// bit of component c (0..5 = ex ey ez hx hy hz) stored as its split pair
constexpr uint32_t kCompSplit0 = 1u << 8;


// Split-pair storage of one simulation. The cells of the PML slabs keep their
// six split pairs ((ex_y ex_z) (ey_z ey_x) (ez_x ez_y) (hx_y hx_z) (hy_z hy_x)
// (hz_x hz_y)) in six slab stores, one per face, each a box [6][depth][h][w]
// of pairs at origin (ox, oy, oz); a cell belongs to the first of the z
// faces, the y faces, the x faces whose slab (thickness t) holds it. A split
// cell in no slab (a soft-source cell) is "sparse": its six pairs sit at the
// slot named by its table row's word 31 in the sparse store [slot][6]. Per
// time buffer the stores lie back to back from base[b].
constexpr int kStXlo = 0, kStXhi = 1, kStYlo = 2, kStYhi = 3, kStZlo = 4, kStZhi = 5, kStSparse = 6;

struct SplitDev {
  float2* base[2];
  int t[6];                            // slab thickness: x-lo, x-hi, y-lo, y-hi, z-lo, z-hi
  int ox[6], oy[6], oz[6], w[6], h[6];  // slab stores: origin, row pitch (pairs), rows per plane
  int64_t off[7];                      // pair offset of each store inside a time buffer
  int64_t comp[6];                     // pairs per component of each slab store
};

// Store holding the split pairs of cell (x, y, z).
__host__ __device__ __forceinline__ int split_store(const SplitDev& S, int nx, int ny, int nz, int x, int y,
                                                    int z) {
  if (z < S.t[4]) return kStZlo;
  if (z >= nz - S.t[5]) return kStZhi;
  if (y < S.t[2]) return kStYlo;
  if (y >= ny - S.t[3]) return kStYhi;
  if (x < S.t[0]) return kStXlo;
  if (x >= nx - S.t[1]) return kStXhi;
  return kStSparse;
}

// Pair of component 0 of cell (x, y, z) in store st of time buffer b (slot:
// the cell's row word 31, used by the sparse store); component m lies m *
// stride pairs further. split_off is its offset from the buffer's base.
__device__ __forceinline__ int64_t split_off(const SplitDev& S, int st, int x, int y, int z, int slot,
                                             int& stride) {
  if (st == kStSparse) {
    stride = 1;
    return S.off[kStSparse] + int64_t(slot) * 6;
  }
  stride = int(S.comp[st]);
  return S.off[st] + (int64_t(z - S.oz[st]) * S.h[st] + (y - S.oy[st])) * S.w[st] + (x - S.ox[st]);
}

__device__ __forceinline__ float2* split_ptr(const SplitDev& S, int b, int st, int x, int y, int z, int slot,
                                             int& stride) {
  return S.base[b] + split_off(S, st, x, y, z, slot, stride);
}

struct SimDev {
  const void* maps;       // tensor maps of the streaming kernel (set per engine)
  int nx, ny, nz, pitch;  // cells; pitch = floats per x row
  int plane;              // ny * pitch
  int nt;
  float* E[2][3];         // [buffer][ex, ey, ez]
  float* H[2][3];         // [buffer][hx, hy, hz]
  SplitDev sp;            // split pairs of the split cells
  const uint16_t* mat;    // [z][y][pitch]
  const float4* rows;     // 8 float4 per row
  const int2* cell_probes;  // (probe, field) grouped per probe cell
  const float* src;       // [P][nt] soft-source amplitudes
  float* rec;             // [P][nt] recorded field values
  const int* is_src;      // [P]
  int64_t cells;          // floats per component array (E[b][c+1] - E[b][c], also for splits)
};

__device__ __forceinline__ float ldf(const float* p, int i, bool ok) { return ok ? __ldg(p + i) : 0.0f; }

// The update arithmetic with its rounding order fixed by intrinsics, so every
// kernel variant produces the same bits (the compiler may otherwise contract
// a*b + c*d either way).
//   E split      s' = Ca s + Cb d                    (solver.cu:154-184)
//   E unsplit    f' = (Ca f + Cb1 d1) + Cb2 d2        (sum of the two splits)
//   H term       g  = Db2 e2 - Db1 e1                  (solver.cu:329-350)
//   H split      s' = Da s + g
//   H unsplit    f' = (Da f + g1) + g2
__device__ __forceinline__ float upd_e_split(float ca, float s, float cb, float d) {
  return __fmaf_rn(cb, d, __fmul_rn(ca, s));
}
__device__ __forceinline__ float upd_e(float ca, float f, float cb1, float d1, float cb2, float d2) {
  return __fmaf_rn(cb2, d2, __fmaf_rn(cb1, d1, __fmul_rn(ca, f)));
}
__device__ __forceinline__ float h_term(float b2, float e2, float b1, float e1) {
  return __fmaf_rn(b2, e2, -__fmul_rn(b1, e1));
}
__device__ __forceinline__ float upd_h_split(float da, float s, float g) { return __fmaf_rn(da, s, g); }
__device__ __forceinline__ float upd_h(float da, float f, float g1, float g2) {
  return __fadd_rn(__fmaf_rn(da, f, g1), g2);
}

template <int TY>
__global__ void __launch_bounds__(32 * (TY + 1))
fdtd_step_kernel(const SimDev* __restrict__ sims, const int4* __restrict__ tiles, int n) {
  const int4 t = tiles[blockIdx.x];
  const SimDev& S = sims[t.x];
  const int x0 = t.y & 0xffff, y0 = int(unsigned(t.y) >> 16), z0 = t.z & 0xffff, z1 = int(unsigned(t.z) >> 16);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int c = x0 - 1 + lane;  // this lane's column
  const int r = y0 - 1 + w;     // this warp's row
  const int nx = S.nx, ny = S.ny, nz = S.nz, pitch = S.pitch, plane = S.plane;
  const bool in_xy = c >= 0 && c < nx && r >= 0 && r < ny;
  const bool own = in_xy && lane >= 1 && w >= 1;  // tile cells this thread stores
  const bool has_yn = in_xy && r + 1 < ny;
  const bool has_xn = (c + 1) >= 0 && (c + 1) < nx && r >= 0 && r < ny;
  const int cur = n & 1, nxt = cur ^ 1;

  const float* __restrict__ Ex = S.E[cur][0];
  const float* __restrict__ Ey = S.E[cur][1];
  const float* __restrict__ Ez = S.E[cur][2];
  const float* __restrict__ Hx = S.H[cur][0];
  const float* __restrict__ Hy = S.H[cur][1];
  const float* __restrict__ Hz = S.H[cur][2];

  __shared__ float s_ex[2][TY + 1][32];
  __shared__ float s_ez[2][TY + 1][32];

  const int col = r * pitch + c;  // offset inside a z plane (valid when in_xy)
  float hx_c = 0.f, hy_c = 0.f;   // H^n at (c, r, z), carried from the look-ahead
  float ex_p = 0.f, ey_p = 0.f;   // E^{n+1} at (c, r, z-1)
  {
    const int zp = z0 - 1;
    const bool ok = in_xy && zp >= 0;
    hx_c = ldf(Hx, zp * plane + col, ok);
    hy_c = ldf(Hy, zp * plane + col, ok);
  }

  for (int z = z0 - 1; z < z1; ++z) {
    const bool zin = z >= 0 && z < nz;
    const bool live = in_xy && zin;
    const int idx = z * plane + col;
    const int buf = z & 1;

    // ---- H^n around (c, r, z)
    const float hz_c = ldf(Hz, idx, live);
    const bool zn_ok = in_xy && z + 1 < nz && z + 1 >= 0;
    const float hx_n = ldf(Hx, idx + plane, zn_ok);
    const float hy_n = ldf(Hy, idx + plane, zn_ok);
    const float hz_yn = ldf(Hz, idx + pitch, has_yn && zin);
    const float hx_yn = ldf(Hx, idx + pitch, has_yn && zin);
    float hz_xn = __shfl_down_sync(0xffffffffu, hz_c, 1);
    float hy_xn = __shfl_down_sync(0xffffffffu, hy_c, 1);
    if (lane == 31) {
      hz_xn = ldf(Hz, idx + 1, has_xn && zin);
      hy_xn = ldf(Hy, idx + 1, has_xn && zin);
    }

    // ---- E^{n+1}(c, r, z)
    float ex = 0.f, ey = 0.f, ez = 0.f;
    float4 rw7 = make_float4(0.f, 0.f, 0.f, 0.f);
    int id = 0;
    uint32_t flags = 0;
    if (live) {
      id = __ldg(S.mat + idx);
      const float4* row = S.rows + 8 * id;
      const float4 a = __ldg(row + 0), b = __ldg(row + 1), d = __ldg(row + 2);
      rw7 = __ldg(row + 7);
      flags = __float_as_uint(rw7.z);
      const float dhz_y = hz_yn - hz_c, dhy_z = hy_n - hy_c;
      const float dhx_z = hx_n - hx_c, dhz_x = hz_xn - hz_c;
      const float dhy_x = hy_xn - hy_c, dhx_y = hx_yn - hx_c;
      if (!(flags & kESplit)) {
        // interior: both splits share Ca, so f' = Ca f + Cb1 d1 + Cb2 d2
        ex = upd_e(a.x, __ldg(Ex + idx), a.y, dhz_y, a.w, dhy_z);
        ey = upd_e(b.x, __ldg(Ey + idx), b.y, dhx_z, b.w, dhz_x);
        ez = upd_e(d.x, __ldg(Ez + idx), d.y, dhy_x, d.w, dhx_y);
      } else {
        // per component: split pair (ex_y, ex_z), ... or unsplit total
        const int st = split_store(S.sp, nx, ny, nz, c, r, z);
        int cs;
        const float2* Es = split_ptr(S.sp, cur, st, c, r, z, __float_as_int(rw7.w), cs);
        float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0;
        if (flags & (kCompSplit0 << 0)) {
          p0 = __ldg(Es);
          p0.x = upd_e_split(a.x, p0.x, a.y, dhz_y);  // ex_y
          p0.y = upd_e_split(a.z, p0.y, a.w, dhy_z);  // ex_z
        } else {
          ex = upd_e(a.x, __ldg(Ex + idx), a.y, dhz_y, a.w, dhy_z);
        }
        if (flags & (kCompSplit0 << 1)) {
          p1 = __ldg(Es + cs);
          p1.x = upd_e_split(b.x, p1.x, b.y, dhx_z);  // ey_z
          p1.y = upd_e_split(b.z, p1.y, b.w, dhz_x);  // ey_x
        } else {
          ey = upd_e(b.x, __ldg(Ey + idx), b.y, dhx_z, b.w, dhz_x);
        }
        if (flags & (kCompSplit0 << 2)) {
          p2 = __ldg(Es + 2 * cs);
          p2.x = upd_e_split(d.x, p2.x, d.y, dhy_x);  // ez_x
          p2.y = upd_e_split(d.z, p2.y, d.w, dhx_y);  // ez_y
        } else {
          ez = upd_e(d.x, __ldg(Ez + idx), d.y, dhy_x, d.w, dhx_y);
        }
        const int np = int(flags >> 16);
        if (np) {
          // soft sources: s1 += v; s2 += v; f = s1 + s2 (solver.cu:459-488);
          // a sourced component is always stored split
          const int first = __float_as_int(rw7.w);
          for (int e = 0; e < np; ++e) {
            const int2 pe = __ldg(S.cell_probes + first + e);
            if (pe.y < 3 && __ldg(S.is_src + pe.x)) {
              const float v = __ldg(S.src + (size_t)pe.x * S.nt + n);
              if (pe.y == 0) { p0.x = __fadd_rn(p0.x, v); p0.y = __fadd_rn(p0.y, v); }
              if (pe.y == 1) { p1.x = __fadd_rn(p1.x, v); p1.y = __fadd_rn(p1.y, v); }
              if (pe.y == 2) { p2.x = __fadd_rn(p2.x, v); p2.y = __fadd_rn(p2.y, v); }
            }
          }
        }
        const bool stor = own && z >= z0;
        float2* Eo = split_ptr(S.sp, nxt, st, c, r, z, __float_as_int(rw7.w), cs);
        if (flags & (kCompSplit0 << 0)) {
          ex = __fadd_rn(p0.x, p0.y);
          if (stor) Eo[0] = p0;
        }
        if (flags & (kCompSplit0 << 1)) {
          ey = __fadd_rn(p1.x, p1.y);
          if (stor) Eo[cs] = p1;
        }
        if (flags & (kCompSplit0 << 2)) {
          ez = __fadd_rn(p2.x, p2.y);
          if (stor) Eo[2 * cs] = p2;
        }
      }
    }

    // ---- neighbour exchange of E^{n+1}
    s_ex[buf][w][lane] = ex;
    s_ez[buf][w][lane] = ez;
    const float ey_xm = __shfl_up_sync(0xffffffffu, ey, 1);
    const float ez_xm = __shfl_up_sync(0xffffffffu, ez, 1);
    __syncthreads();

    if (own && z >= z0 && zin) {
      const float ex_ym = s_ex[buf][w - 1][lane];
      const float ez_ym = s_ez[buf][w - 1][lane];
      // totals of the components not stored split
      if (!(flags & (kCompSplit0 << 0))) S.E[nxt][0][idx] = ex;
      if (!(flags & (kCompSplit0 << 1))) S.E[nxt][1][idx] = ey;
      if (!(flags & (kCompSplit0 << 2))) S.E[nxt][2][idx] = ez;
      const float4* row = S.rows + 8 * id;
      const float4 p = __ldg(row + 3), q = __ldg(row + 4), u = __ldg(row + 5), v6 = __ldg(row + 6);
      // slots 12..29: (Da, Db1, Db2) for hx_y, hx_z, hy_z, hy_x, hz_x, hz_y
      const float da_xy = p.x, b1_xy = p.y, b2_xy = p.z, da_xz = p.w;
      const float b1_xz = q.x, b2_xz = q.y, da_yz = q.z, b1_yz = q.w;
      const float b2_yz = u.x, da_yx = u.y, b1_yx = u.z, b2_yx = u.w;
      const float da_zx = v6.x, b1_zx = v6.y, b2_zx = v6.z, da_zy = v6.w;
      const float b1_zy = rw7.x, b2_zy = rw7.y;
      const float gxy = h_term(b2_xy, ez, b1_xy, ez_ym);
      const float gxz = h_term(b2_xz, ey, b1_xz, ey_p);
      const float gyz = h_term(b2_yz, ex, b1_yz, ex_p);
      const float gyx = h_term(b2_yx, ez, b1_yx, ez_xm);
      const float gzx = h_term(b2_zx, ey, b1_zx, ey_xm);
      const float gzy = h_term(b2_zy, ex, b1_zy, ex_ym);
      float hx, hy, hz;
      if (!(flags & kHSplit)) {
        hx = upd_h(da_xy, hx_c, gxy, gxz);
        hy = upd_h(da_yz, hy_c, gyz, gyx);
        hz = upd_h(da_zx, hz_c, gzx, gzy);
      } else {
        const int st = split_store(S.sp, nx, ny, nz, c, r, z);
        int cs;
        const float2* Hs = split_ptr(S.sp, cur, st, c, r, z, __float_as_int(rw7.w), cs);
        Hs += 3 * cs;
        float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0;
        if (flags & (kCompSplit0 << 3)) {
          p0 = __ldg(Hs);
          p0.x = upd_h_split(da_xy, p0.x, gxy);
          p0.y = upd_h_split(da_xz, p0.y, gxz);
        } else {
          hx = upd_h(da_xy, hx_c, gxy, gxz);
        }
        if (flags & (kCompSplit0 << 4)) {
          p1 = __ldg(Hs + cs);
          p1.x = upd_h_split(da_yz, p1.x, gyz);
          p1.y = upd_h_split(da_yx, p1.y, gyx);
        } else {
          hy = upd_h(da_yz, hy_c, gyz, gyx);
        }
        if (flags & (kCompSplit0 << 5)) {
          p2 = __ldg(Hs + 2 * cs);
          p2.x = upd_h_split(da_zx, p2.x, gzx);
          p2.y = upd_h_split(da_zy, p2.y, gzy);
        } else {
          hz = upd_h(da_zx, hz_c, gzx, gzy);
        }
        const int np = int(flags >> 16);
        if (np) {
          const int first = __float_as_int(rw7.w);
          for (int e = 0; e < np; ++e) {
            const int2 pe = __ldg(S.cell_probes + first + e);
            if (pe.y >= 3 && __ldg(S.is_src + pe.x)) {
              const float v = __ldg(S.src + (size_t)pe.x * S.nt + n);
              if (pe.y == 3) { p0.x = __fadd_rn(p0.x, v); p0.y = __fadd_rn(p0.y, v); }
              if (pe.y == 4) { p1.x = __fadd_rn(p1.x, v); p1.y = __fadd_rn(p1.y, v); }
              if (pe.y == 5) { p2.x = __fadd_rn(p2.x, v); p2.y = __fadd_rn(p2.y, v); }
            }
          }
        }
        float2* Ho = split_ptr(S.sp, nxt, st, c, r, z, __float_as_int(rw7.w), cs);
        Ho += 3 * cs;
        if (flags & (kCompSplit0 << 3)) {
          hx = __fadd_rn(p0.x, p0.y);
          Ho[0] = p0;
        }
        if (flags & (kCompSplit0 << 4)) {
          hy = __fadd_rn(p1.x, p1.y);
          Ho[cs] = p1;
        }
        if (flags & (kCompSplit0 << 5)) {
          hz = __fadd_rn(p2.x, p2.y);
          Ho[2 * cs] = p2;
        }
      }
      S.H[nxt][0][idx] = hx;
      S.H[nxt][1][idx] = hy;
      S.H[nxt][2][idx] = hz;
      const int np = int(flags >> 16);
      if (np) {  // record probes of this cell (solver.cu:467, 521)
        const int first = __float_as_int(rw7.w);
        for (int e = 0; e < np; ++e) {
          const int2 pe = __ldg(S.cell_probes + first + e);
          const float val = pe.y == 0 ? ex : pe.y == 1 ? ey : pe.y == 2 ? ez : pe.y == 3 ? hx : pe.y == 4 ? hy : hz;
          S.rec[(size_t)pe.x * S.nt + n] = val;
        }
      }
    }
    ex_p = ex;
    ey_p = ey;
    hx_c = hx_n;
    hy_c = hy_n;
  }
}

// Brings the cache line holding p into L1 ahead of its use.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Error codes the kernels record in the engine's error word.
constexpr int kErrWaitExpired = 1;  // a bounded pipeline wait gave up
constexpr int kErrNonFinite = 2;    // a probe record or a final field value is NaN or infinite

// Run sentinel: records kErrNonFinite when any of n floats is NaN or
// infinite (a diverged run), checked once after the last step.
__global__ void nonfinite_check_kernel(const float* __restrict__ v, int64_t n, int* __restrict__ err) {
  bool bad = false;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    bad |= !isfinite(__ldg(v + i));
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(err, 0, kErrNonFinite);
}

// Ids arrive in the reference order [x][y][z]; the kernels read [z][y][pitch].
__global__ void transpose_ids_kernel(const uint16_t* __restrict__ in, uint16_t* __restrict__ out, int nx, int ny,
                                     int nz, int pitch) {
  const int64_t total = int64_t(nx) * ny * nz;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int z = int(i % nz);
    const int64_t xy = i / nz;
    const int y = int(xy % ny), x = int(xy / ny);
    out[(int64_t(z) * ny + y) * pitch + x] = in[i];
  }
}

// ------------------------------------------------------------------ DFT
struct DftDev {
  int n_series, n_freq, nt;
  const int* series_start;   // n_series + 1
  const int* term_probe;
  const double* term_weight;
  const double* omega;       // radians per step
  const float* rec;          // [P][nt]
  double2* X;                // [n_series][n_freq]
};

// X[s][f] += sum_{n0 <= n < n1} series_s[n] e^{-j omega_f n}. One block per
// (f, s); fixed-order block reduction, so results are deterministic.
__global__ void __launch_bounds__(256) dft_accumulate_kernel(DftDev d, int n0, int n1) {
  const int f = blockIdx.x, s = blockIdx.y;
  const double om = d.omega[f];
  const int t0 = d.series_start[s], t1 = d.series_start[s + 1];
  double re = 0.0, im = 0.0;
  for (int n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
    double v = 0.0;
    for (int t = t0; t < t1; ++t) v += d.term_weight[t] * double(d.rec[size_t(d.term_probe[t]) * d.nt + n]);
    double sn, cs;
    sincos(om * double(n), &sn, &cs);
    re += v * cs;
    im -= v * sn;
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  __shared__ double sre[8], sim[8];
  const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) {
    sre[wid] = re;
    sim[wid] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < int(blockDim.x >> 5); ++i) {
      a += sre[i];
      b += sim[i];
    }
    double2 x = d.X[s * d.n_freq + f];
    x.x += a;
    x.y += b;
    d.X[s * d.n_freq + f] = x;
  }
}

// -------------------------------------------------------------- monitors
struct MonDev {
  int field, axis, position, n_step, n_freq, n1, n2;
  void* out;                 // float [Nm][n1][n2] or float2 [n_freq][n1][n2]
  const float2* phase;       // [Nm][n_freq]
};

// Samples the fields after step n (E and H of the new buffer), i.e. after the
// sources of the step are applied, as the CPU engine does (solver.cpp:1129-1161).
__global__ void monitor_kernel(const SimDev* __restrict__ sim, const MonDev* __restrict__ mons, int n_mon, int n,
                               int buf) {
  const SimDev& S = *sim;
  for (int m = 0; m < n_mon; ++m) {
    const MonDev M = mons[m];
    if (n > 0 && (n % M.n_step) != 0) continue;
    const int mn = n / M.n_step;
    const int total = M.n1 * M.n2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
      const int a = e / M.n2, b = e % M.n2;
      int x, y, z;
      if (M.axis == 0) { x = M.position; y = a; z = b; }
      else if (M.axis == 1) { x = a; y = M.position; z = b; }
      else { x = a; y = b; z = M.position; }
      if (x < 0 || y < 0 || z < 0 || x >= S.nx || y >= S.ny || z >= S.nz) continue;
      const int idx = z * S.plane + y * S.pitch + x;
      const float4 r7 = S.rows[8 * S.mat[idx] + 7];
      const uint32_t flags = __float_as_uint(r7.z);
      float v;
      if (M.field < 3) {
        if (flags & (kCompSplit0 << M.field)) {
          int cs;
          const float2* pp = split_ptr(S.sp, buf, split_store(S.sp, S.nx, S.ny, S.nz, x, y, z), x, y, z,
                                       __float_as_int(r7.w), cs);
          const float2 p = pp[M.field * cs];
          v = p.x + p.y;
        } else {
          v = S.E[buf][M.field][idx];
        }
      } else {
        v = S.H[buf][M.field - 3][idx];
      }
      if (M.n_freq == 0) {
        static_cast<float*>(M.out)[size_t(mn) * total + e] = v;
      } else {
        float2* o = static_cast<float2*>(M.out);
        for (int f = 0; f < M.n_freq; ++f) {
          const float2 ph = M.phase[size_t(mn) * M.n_freq + f];
          float2 acc = o[size_t(f) * total + e];
          acc.x += v * ph.x;
          acc.y += v * ph.y;
          o[size_t(f) * total + e] = acc;
        }
      }
    }
  }
}

}  // namespace rfn
