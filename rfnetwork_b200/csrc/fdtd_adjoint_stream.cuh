// Streaming reverse step of the discrete adjoint for sm_100a: the adjoint
// state of each z plane staged in shared memory by the tensor-memory
// accelerator, as the streaming forward kernel stages the fields.
//
// Same recursion, same per-cell arithmetic (adj_e_part / adj_h_part /
// adj_grad_cell of fdtd_adjoint.cuh) and the same tile geometry as
// adj_step_kernel, so the two give the same bits:
//   tile      30 (x) by TY (y) owned cells and a z range [z0, z1). Consumer
//             warp w (0 .. TY+1) sits on row y0-1+w, lane l on column
//             x0-1+l: row y0-1 and column x0-1 are the -1 halo whose ad the
//             owned cells need, row y0+TY and column x0+30 only provide the
//             Db1-weighted H adjoints of the +1 neighbours.
//   producer  one more warp (lane 0) takes tiles from a global counter and,
//             per z plane z0-1 .. z1, issues into a free plane slot:
//               lamH  3 totals, rows y0-1 .. y0+TY, 40 columns
//               lamE  3 totals, rows y0-1 .. y0+TY-1, 36 columns
//               index 16-bit material rows, rows y0-1 .. y0+TY, 40 columns
//               halves the 12 adjoint halves of split cells (E then H), rows
//                      y0-1 .. y0+TY, 40 columns, for tiles the host flagged
//                      as holding split cells
//             Boxes start at an x that is a multiple of 16 bytes at or below
//             x0-1; boxes reaching outside the grid fill with zeros, and a
//             zero index selects the all-zero row.
//   consumers per plane z: E part for the tile and its -1 halo (mu, lamE',
//             ad) from plane z and the look-ahead plane z+1; one barrier;
//             then H part, adjoint record sources, stores and the FP64
//             gradient of box cells for the owned cells.
//   waits     bounded, as in the forward kernel: an expired wait is voted at
//             the next barrier, recorded in the error word, and the block
//             returns.
#pragma once

#include "fdtd_adjoint.cuh"
#include "fdtd_step_stream.cuh"

namespace rfn {

// Tensor maps of one simulation for the streaming reverse step.
struct AdjMaps {
  CUtensorMap lam_e, lam_h, halves, ids;
};

template <int TY>
struct AdjGeom {
  static constexpr int HW = 40, EW = 36, IW = 40, SW = 40;  // box widths along x
  static constexpr int HR = TY + 2, ER = TY + 1;            // box heights along y
  static constexpr int HC = HR * HW;                        // floats per lamH component
  static constexpr int EC = ER * EW;                        // floats per lamE component
  static constexpr int SC = HR * SW;                        // floats per half
  static constexpr int HB = 3 * HC * 4, EB = 3 * EC * 4, IB = HR * IW * 2, SB = 12 * SC * 4;
  static constexpr int A(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_E = A(HB);
  static constexpr int OFF_I = OFF_E + A(EB);
  static constexpr int OFF_S = OFF_I + A(IB);
  static constexpr uint32_t SLOT = OFF_S + A(SB);           // one plane: lamH, lamE, index, halves
  static constexpr uint32_t MAIN_BYTES = HB + EB + IB;
  static constexpr int NCW = TY + 2;                        // consumer warps
  static constexpr int CONSUMERS = 32 * NCW;
  static constexpr int THREADS = CONSUMERS + 32;            // + the producer warp
};

// The four H-adjoint halves of a cell that its +z neighbour's terms use:
// hx_y, hx_z, hy_z and hz_y (halves 0, 1, 2 and 5).
template <int TY>
__device__ __forceinline__ void adj_stream_h4(const float* sH, const float* sS, int hb, uint32_t fl, float& h0,
                                              float& h1, float& h2, float& h5) {
  using G = AdjGeom<TY>;
  if (fl & kHSplit) {
    h0 = sS[6 * G::SC + hb]; h1 = sS[7 * G::SC + hb]; h2 = sS[8 * G::SC + hb]; h5 = sS[11 * G::SC + hb];
  } else {
    h0 = sH[hb]; h1 = h0; h2 = sH[G::HC + hb]; h5 = sH[2 * G::HC + hb];
  }
}

constexpr int kAdjStreamTileY = 7;
constexpr int kAdjStreamSlotsMax = 6;

// The cell's H adjoint as six halves, from the staged plane (totals
// repeated for an unsplit cell).
template <int TY>
__device__ __forceinline__ void adj_stream_h(const float* sH, const float* sS, int hb, int sbi, uint32_t fl,
                                             float (&h)[6]) {
  using G = AdjGeom<TY>;
  if (fl & kHSplit) {
#pragma unroll
    for (int k = 0; k < 6; ++k) h[k] = sS[(6 + k) * G::SC + sbi];
  } else {
    const float hx = sH[hb], hy = sH[G::HC + hb], hz = sH[2 * G::HC + hb];
    h[0] = hx; h[1] = hx; h[2] = hy; h[3] = hy; h[4] = hz; h[5] = hz;
  }
}

// One reverse step (time step n: reads adjoint buffer n & 1, writes the
// other) over a tile list, persistent blocks taking tiles from `counter`.
template <int TY>
__global__ void __launch_bounds__(AdjGeom<TY>::THREADS, 2)
adj_stream_kernel(const AdjSim* __restrict__ sims, const AdjMaps* __restrict__ maps,
                  const int4* __restrict__ tiles, int n_tiles, int n, int hist_n0, unsigned* __restrict__ counter,
                  unsigned base, int* __restrict__ err, int n_slots, uint32_t wait_limit) {
  using G = AdjGeom<TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* const ring = smem;  // n_slots plane slots
  __shared__ __align__(8) uint64_t full[kAdjStreamSlotsMax], empty[kAdjStreamSlotsMax];
  __shared__ float s_qhx[2][TY + 2][32];  // Db1 lamH of hx_y, read by the row below
  __shared__ float s_qhz[2][TY + 2][32];  // Db1 lamH of hz_y
  __shared__ float s_a0[2][TY + 2][32];   // ad of dA_x (= dhz_y), read by the row above
  __shared__ float s_a5[2][TY + 2][32];   // ad of dB_z (= dhx_y)
  __shared__ int s_tq[4];
  const int tid = threadIdx.x;
  const int cur = n & 1, nxt = cur ^ 1;
  constexpr int NC = G::CONSUMERS;
  const int P = n_slots;

  if (tid == 0) {
    for (int s = 0; s < P; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], G::NCW);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // =================================================================== producer
  if (tid >= NC) {
    if (tid != NC) return;
    uint32_t q = 0, rel = 0;  // planes issued; planes below rel released by every consumer warp
    SlotPos qp{0u, 0u}, rp{0u, 0u};
    int k = 0;
    const AdjMaps* cur_maps = nullptr;
    bool failed = false;
    auto release_upto = [&](uint32_t u) -> bool {
      while (rel <= u) {
        if (!mbar_wait_bounded(&empty[rp.slot], rp.par, wait_limit)) return false;
        ++rel;
        rp = rp.next(P);
      }
      return true;
    };
    for (;;) {
      const unsigned v = atomicAdd(counter, 1u) - base;
      const int t = v < unsigned(n_tiles) ? int(v) : -1;
      int4 td = make_int4(0, 0, 0, 0);
      int nload = 1;
      const AdjMaps* m = nullptr;
      if (t >= 0) {
        td = __ldg(tiles + t);
        nload = int(unsigned(td.z) >> 16) - (td.z & 0xffff) + 2;  // planes z0-1 .. z1
        m = maps + td.x;
        if (m != cur_maps) {
          tensormap_acquire(&m->lam_e);
          tensormap_acquire(&m->lam_h);
          tensormap_acquire(&m->halves);
          tensormap_acquire(&m->ids);
          cur_maps = m;
        }
      }
      const int x0 = td.y & 0xffff, y0 = int(unsigned(td.y) >> 16), z0 = td.z & 0xffff;
      const int xs = (x0 - 1) & ~3, xi = (x0 - 1) & ~7;
      const bool halves = t >= 0 && td.w != 0;
      for (int j = 0; j < nload; ++j) {
        if (q >= uint32_t(P) && !release_upto(q - P)) {
          failed = true;
          break;
        }
        const int slot = int(qp.slot);
        if (j == 0) s_tq[k & 3] = t;
        if (t < 0) {  // end of the stream: complete the phase without data
          mbar_arrive(&full[slot]);
          ++q;
          qp = qp.next(P);
          break;
        }
        unsigned char* b = ring + uint32_t(slot) * G::SLOT;
        uint64_t* fb = &full[slot];
        const int zp = z0 - 1 + j;
        fence_proxy_async();
        mbar_arrive_expect_tx(fb, G::MAIN_BYTES + (halves ? uint32_t(G::SB) : 0u));
        tma_load_5d(b, &m->lam_h, xs, y0 - 1, zp, 0, cur, fb);  // (lam_h's map starts at the H totals)
        tma_load_5d(b + G::OFF_E, &m->lam_e, xs, y0 - 1, zp, 0, cur, fb);
        tma_load_3d(b + G::OFF_I, &m->ids, xi, y0 - 1, zp, fb);
        if (halves) tma_load_5d(b + G::OFF_S, &m->halves, xs, y0 - 1, zp, 0, cur, fb);
        ++q;
        qp = qp.next(P);
      }
      if (failed || t < 0) break;
      ++k;
    }
    if (failed) {
      atomicExch(err, kErrWaitExpired);
      for (uint32_t r = rel; r < q; ++r, rp = rp.next(P)) mbar_wait_bounded(&full[rp.slot], rp.par, wait_limit);
    }
    return;
  }

  // ================================================================== consumers
  const int lane = tid & 31, w = tid >> 5;
  SlotPos cp{0u, 0u};  // ring position of the plane being computed
  for (int k = 0;; ++k) {
    bool ok = mbar_wait_bounded(&full[cp.slot], cp.par, wait_limit);
    if (named_bar_or(kStreamBar, NC, !ok)) {
      if (tid == 0) atomicExch(err, kErrWaitExpired);
      return;
    }
    const int ti = s_tq[k & 3];
    if (ti < 0) break;
    const int4 td = __ldg(tiles + ti);
    const AdjSim& A = sims[td.x];
    const int x0 = td.y & 0xffff, y0 = int(unsigned(td.y) >> 16), z0 = td.z & 0xffff;
    const int z1 = int(unsigned(td.z) >> 16);
    const int c = x0 - 1 + lane, r = y0 - 1 + w;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const bool in_xy = c >= 0 && c < nx && r >= 0 && r < ny;
    const bool worker = lane < 31 && w <= TY;  // computes E (tile and -1 halo)
    const bool own = in_xy && lane >= 1 && lane <= 30 && w >= 1 && w <= TY;
    const int oh = (x0 - 1) - ((x0 - 1) & ~3), oi = (x0 - 1) - ((x0 - 1) & ~7);
    const int hb = w * G::HW + oh + lane;  // lamH and halves (same width)
    const int eb = w * G::EW + oh + lane;  // lamE (workers)
    const int ib = w * G::IW + oi + lane;
    const float4* __restrict__ rows = A.rows;
    const int npl = z1 - z0 + 1;           // planes z0-1 .. z1-1 computed

    // plane z0-1: this column's Db1 lamH for the row below
    {
      const unsigned char* st = ring + cp.slot * G::SLOT;
      const int id = ok ? int(reinterpret_cast<const uint16_t*>(st + G::OFF_I)[ib]) : 0;
      const float4* rc = rows + 8 * id;
      float h[6];
      adj_stream_h<TY>(reinterpret_cast<const float*>(st), reinterpret_cast<const float*>(st + G::OFF_S), hb, hb,
                       adj_flags(rc), h);
      s_qhx[(z0 - 1) & 1][w][lane] = __fmul_rn(__ldg(rc + 3).y, h[0]);
      s_qhz[(z0 - 1) & 1][w][lane] = __fmul_rn(__ldg(rc + 7).x, h[5]);
    }
    named_bar_sync(kStreamBar, NC);

    float a1_p = 0.f, a2_p = 0.f;  // ad[1], ad[2] of this column one plane below
    for (int i = 0; i < npl; ++i) {
      const SlotPos np = cp.next(P);
      // the look-ahead plane z+1 (H adjoints and rows of the +z neighbour)
      ok = ok && mbar_wait_bounded(&full[np.slot], np.par, wait_limit);
      const int z = z0 - 1 + i;
      const bool zin = z >= 0 && z < nz;
      const bool live = in_xy && zin;
      const int buf = z & 1;
      const unsigned char* st = ring + cp.slot * G::SLOT;
      const unsigned char* sn = ring + np.slot * G::SLOT;
      const float* sS = reinterpret_cast<const float*>(st + G::OFF_S);
      // (after an expired wait the values are stale but in bounds; the vote
      // below then ends the block before anything is stored)
      const int id_c = ok ? int(reinterpret_cast<const uint16_t*>(st + G::OFF_I)[ib]) : 0;
      const int id_n = ok ? int(reinterpret_cast<const uint16_t*>(sn + G::OFF_I)[ib]) : 0;
      // this cell's table row (read through L1; most cells keep their row along z)
      const float4* row = rows + 8 * id_c;
      const float4 ra = __ldg(row), rb = __ldg(row + 1), rd = __ldg(row + 2), p = __ldg(row + 3);
      const float4 q = __ldg(row + 4), u = __ldg(row + 5), v = __ldg(row + 6), r7 = __ldg(row + 7);
      const uint32_t fl_c = __float_as_uint(r7.z);
      // the look-ahead row's Db1 words of hx_y, hx_z, hy_z and hz_y, and flags
      float pn_y = p.y, qn_x = q.x, qn_w = q.w, r7n_x = r7.x;
      uint32_t fl_n = fl_c;
      if (id_n != id_c) {
        const float4* rn = rows + 8 * id_n;
        pn_y = __ldg(&rn[3].y); qn_x = __ldg(&rn[4].x); qn_w = __ldg(&rn[4].w);
        const float4 w7 = __ldg(rn + 7);
        r7n_x = w7.x;
        fl_n = __float_as_uint(w7.z);
      }
      float h_c[6], hn0, hn1, hn2, hn5;
      adj_stream_h<TY>(reinterpret_cast<const float*>(st), sS, hb, hb, fl_c, h_c);
      adj_stream_h4<TY>(reinterpret_cast<const float*>(sn), reinterpret_cast<const float*>(sn + G::OFF_S), hb, fl_n,
                        hn0, hn1, hn2, hn5);
      float lE[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (worker && live) {
        if (fl_c & kESplit) {
#pragma unroll
          for (int m = 0; m < 6; ++m) lE[m] = sS[m * G::SC + hb];
        } else {
          const float* sE = reinterpret_cast<const float*>(st + G::OFF_E);
          lE[0] = sE[eb]; lE[1] = sE[G::EC + eb]; lE[2] = sE[2 * G::EC + eb];
        }
      }

      // Db1 lamH of the +1 neighbours: z+1 from the look-ahead, x+1 from the
      // lane on the right, y+1 from the row above (written last plane)
      const float qz_hx = __fmul_rn(qn_x, hn1), qz_hy = __fmul_rn(qn_w, hn2);
      const float qx_hy = __shfl_down_sync(0xffffffffu, __fmul_rn(u.z, h_c[3]), 1);
      const float qx_hz = __shfl_down_sync(0xffffffffu, __fmul_rn(v.y, h_c[4]), 1);
      const float qy_hx = s_qhx[buf][w + (w <= TY ? 1 : 0)][lane];
      const float qy_hz = s_qhz[buf][w + (w <= TY ? 1 : 0)][lane];
      // and this column's own values at z+1 for the row below, next plane
      s_qhx[buf ^ 1][w][lane] = __fmul_rn(pn_y, hn0);
      s_qhz[buf ^ 1][w][lane] = __fmul_rn(r7n_x, hn5);

      // E part: mu, lamE', ad
      float mu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, ad[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (live && worker)
        adj_e_part(ra, rb, rd, p, q, u, v, r7, fl_c, h_c, qz_hx, qz_hy, qx_hy, qx_hz, qy_hx, qy_hz, lE, mu, ad);

      // -1 neighbours' ad
      s_a0[buf][w][lane] = ad[0];
      s_a5[buf][w][lane] = ad[5];
      const float a3_m = __shfl_up_sync(0xffffffffu, ad[3], 1);
      const float a4_m = __shfl_up_sync(0xffffffffu, ad[4], 1);
      if (named_bar_or(kStreamBar, NC, !ok)) {
        if (tid == 0) atomicExch(err, kErrWaitExpired);
        return;
      }

      if (own && z >= z0 && zin) {
        const int64_t N = A.N;
        const int idx = z * A.plane + r * A.pitch + c;
        const float a0_m = s_a0[buf][w - 1][lane];
        const float a5_m = s_a5[buf][w - 1][lane];
        float lh[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        adj_h_part(p, q, u, v, fl_c, h_c, ad, a0_m, a5_m, a3_m, a4_m, a1_p, a2_p, lh);
        // adjoints of this cell's records of step n-1 (E^n, H^n)
        const int npr = int(fl_c >> 16);
        if (npr && n >= 1) {
          const int first = __float_as_int(r7.w);
          for (int e = 0; e < npr; ++e) {
            const int2 pe = __ldg(A.cell_probes + first + e);
            const float rv = __ldg(A.radj + size_t(pe.x) * A.nt + (n - 1));
            // both halves of a split pair, or the total (slots 0..2) of an unsplit cell
            const bool is_e = pe.y < 3;
            const int cc = is_e ? pe.y : pe.y - 3;
            const bool sp = (fl_c & (is_e ? kESplit : kHSplit)) != 0;
#pragma unroll
            for (int m = 0; m < 6; ++m)
              if (sp ? (m / 2 == cc) : (m == cc)) {
                if (is_e) lE[m] = __fadd_rn(lE[m], rv);
                else lh[m] = __fadd_rn(lh[m], rv);
              }
          }
        }
        float* __restrict__ wE = A.lam + nxt * 6 * N;
        if (fl_c & kESplit) {
          float* wEs = A.lams + nxt * 12 * N;
#pragma unroll
          for (int m = 0; m < 6; ++m) wEs[m * N + idx] = lE[m];
        } else {
          wE[idx] = lE[0]; wE[N + idx] = lE[1]; wE[2 * N + idx] = lE[2];
        }
        if (fl_c & kHSplit) {
          float* wHs = A.lams + nxt * 12 * N + 6 * N;
#pragma unroll
          for (int m = 0; m < 6; ++m) wHs[m * N + idx] = lh[m];
        } else {
          float* wH = wE + 3 * N;
          wH[idx] = lh[0]; wH[N + idx] = lh[1]; wH[2 * N + idx] = lh[2];
        }
        if (A.hist && c >= A.bx0 && c < A.bx1 && r >= A.by0 && r < A.by1 && z >= A.bz0 && z < A.bz1) {
          const int bny = A.by1 - A.by0, bnz = A.bz1 - A.bz0;
          const int64_t bi = (int64_t(c - A.bx0) * bny + (r - A.by0)) * bnz + (z - A.bz0);
          adj_grad_cell(A.grad, A.nb, bi, A.hist + int64_t(n - hist_n0) * 9 * A.nb, mu);
        }
      }
      a1_p = ad[1];
      a2_p = ad[2];
      // plane z is no longer read by this warp
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[cp.slot]);
      cp = np;
    }
    // the look-ahead plane z1 was read only by the last iteration
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[cp.slot]);
    cp = cp.next(P);
  }
}

}  // namespace rfn
