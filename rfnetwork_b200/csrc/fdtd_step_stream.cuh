// Streaming step kernel for sm_100a: one thread per Yee cell, z planes staged
// in shared memory by the tensor-memory accelerator (cp.async.bulk.tensor)
// through a ring of S mbarrier-guarded stages.
//
// Same update as fdtd_step_kernel (fdtd_kernels.cuh) through the same
// rounding-fixed helpers, so the two kernels produce the same bits.
//
//   tile      31 (x) by TY (y) owned cells and a z range [z0, z1). The block
//             has TY + 1 consumer warps, one per row y0-1 .. y0+TY-1; lane l
//             of a warp sits on column x0-1+l. Row y0-1 and column x0-1 are
//             the halo whose E^{n+1} the H update needs; they are recomputed
//             here rather than read back, so one sweep over memory advances
//             the whole step.
//   producer  one more warp (lane 0) takes tiles from a global atomic counter
//             and, per z plane, waits for a free stage ("empty" mbarrier) and
//             issues the plane's loads onto the stage's "full" mbarrier:
//               H^n     3 components, rows y0-1 .. y0+TY, 40 columns
//               E^n     3 components, rows y0-1 .. y0+TY-1, 36 columns
//               index   16-bit material rows, 40 columns
//               splits  the 3 E and 3 H split pairs (float2 per cell) over
//                       36 columns, only for planes the host flagged as holding
//                       split-field cells (a 64-bit mask per tile), from at
//                       most two slab stores (SplitDev): the plane's z-face
//                       store, or the tile's y-face store and x-face store.
//                       Split cells of other stores (soft-source cells, the
//                       rare corner of a small grid) are read from global
//                       memory directly
//             Every box starts at an x that is a multiple of 16 bytes at or
//             below x0-1; the consumers index from that offset. Boxes reaching
//             outside the grid fill with zeros and a zero material index
//             selects the all-zero coefficient row, so halo and grid edges
//             need no bounds checks in the arithmetic. The last plane of a
//             tile (z1) is only the look-ahead of H for dH/dz: H alone.
//   consumers per plane z: E^{n+1}(z) for every thread's cell from H^n(z),
//             H^n(z+1) and E^n(z) in shared memory; E x/y neighbours are traded
//             by warp shuffle and a small double-buffered shared array; one
//             barrier; then H^{n+1}(z) of the owned cells from E^{n+1}(z) and
//             E^{n+1}(z-1), which each thread kept from its previous plane.
//   waits     every mbarrier wait is bounded. A consumer whose wait expires
//             votes at the next barrier; then all consumers record an error
//             code and return; the producer gives up on the stage it waits
//             for, drains its own loads (bounded) and returns.
#pragma once

#include "fdtd_kernels.cuh"
#include "tma.cuh"

#include <climits>
#include <type_traits>

namespace rfn {

constexpr int kStreamOwnX = 31;           // owned columns per tile (lane 0 is the halo column)
constexpr uint32_t kStreamWaitLimit = 1u << 20;  // sleeping polls (each <= 2 us) per wait
constexpr int kStreamBar = 1;             // named barrier of the consumer warps

// Tensor maps of one simulation for the streaming kernel: the fields, the
// material index, and the E and H split pairs of each slab store.
struct StreamMaps {
  CUtensorMap E, H, ids, Es[6], Hs[6];
};

// One tile: owned [x0, x0+31) x [y0, y0+TY) x [z0, z1). Bit j of `split` is
// set when plane z0-1+j holds split-field cells inside the tile's E region.
// On planes outside the z slabs the tile's split pairs come from slab store
// ys (a y face, or -1) and xs (an x face, or -1). `plain` marks a tile with no
// split-field cells and no probe cells, which takes the consumers' interior
// path (no per-cell flag tests).
struct StreamTile {
  int sim, x0, y0, z0, z1, ys, plain, xs;
  uint32_t split_lo, split_hi, pad2, pad3;
};

template <int TY>
struct StreamGeom {
  static constexpr int HW = 40, EW = 36, IW = 40;  // box widths along x
  static constexpr int HR = TY + 2, ER = TY + 1;   // box heights along y
  static constexpr int HC = HR * HW;               // floats per H component
  static constexpr int EC = ER * EW;               // floats per E component (float2 pairs per E split pair)
  static constexpr int SHC = TY * EW;              // float2 pairs per H split pair
  static constexpr int HB = 3 * HC * 4;
  static constexpr int EB = 3 * EC * 4;
  static constexpr int IB = ER * IW * 2;
  static constexpr int SEB = 6 * EC * 4;           // 3 E split pairs of 8 bytes per cell
  static constexpr int SHB = 6 * SHC * 4;          // 3 H split pairs
  static constexpr int A(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_E = A(HB);
  static constexpr int OFF_I = OFF_E + A(EB);
  static constexpr uint32_t MAIN = OFF_I + A(IB);  // plane slot: H, E, index
  static constexpr uint32_t SPLIT_HS = A(SEB);     // H pairs inside a split region
  static constexpr uint32_t REGION = A(SEB) + A(SHB); // split region: one store's E pairs, then H pairs
  static constexpr uint32_t MAIN_BYTES = HB + EB + IB;
  static constexpr uint32_t SPLIT_BYTES = SEB + SHB;
  static constexpr int NCW = TY + 1;               // consumer warps
  static constexpr int CONSUMERS = 32 * NCW;
  static constexpr int THREADS = CONSUMERS + 32;   // + the producer warp
  static constexpr int XCH = 2 * ER * 32 * 4;      // one E neighbour-exchange buffer (ex, ez), bytes
  // resident blocks per SM the register budget is sized for (shared memory allows as many)
  static constexpr int MIN_BLOCKS = TY <= 4 ? 4 : TY <= 6 ? 3 : 2;
};

// Plane slots and split regions of the streaming kernel (at most). A plane
// with split cells takes one region per slab store it stages (one or two),
// so four regions let the plane being computed and its look-ahead hold two
// each.
constexpr int kSlotsMax = 8;
constexpr int kRegionsMax = 6;
constexpr int kRegionsMin = 4;

// A plane's place in the ring of P plane slots: slot index and the parity of
// the slot's current use, advanced without a division.
struct SlotPos {
  uint32_t slot, par;
  __device__ __forceinline__ SlotPos next(uint32_t P) const {
    return slot + 1 == P ? SlotPos{0u, par ^ 1u} : SlotPos{slot + 1, par};
  }
};

// A staged split region of one plane, as the producer describes it to the
// consumers: its shared-memory offset, and where the step writes the pairs of
// its store's cells: cell (x, y) at pn + y w + x, components comp pairs apart.
// `kind` (of region A) says which cells the staged stores hold: 0 every cell
// of the plane (its z store), 1 the cells of the tile's y-face store (A) and
// x-face store (B), -1 none (nothing staged).
struct RegionRec {
  int smem, w, comp, kind;
  float2* pn;
  long long pad;
};

__device__ __forceinline__ StreamTile load_stream_tile(const StreamTile* tiles, int i) {
  const int4* p = reinterpret_cast<const int4*>(tiles + i);
  const int4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  return StreamTile{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, uint32_t(c.x), uint32_t(c.y), uint32_t(c.z), uint32_t(c.w)};
}

// Soft sources of one field group of a cell (solver.cu:459-488, 515-541):
// s1 += v; s2 += v for every source probe on a component of that group (a
// sourced component is always stored as its split pair).
__device__ __forceinline__ void stream_inject(const SimDev& Sd, const float4& r7, uint32_t flags, int n, bool e_side,
                                              float2 (&p)[3]) {
  const int np = int(flags >> 16);
  const int first = __float_as_int(r7.w);
  for (int e = 0; e < np; ++e) {
    const int2 pe = __ldg(Sd.cell_probes + first + e);
    const bool mine = e_side ? pe.y < 3 : pe.y >= 3;
    if (mine && __ldg(Sd.is_src + pe.x)) {
      const float v = __ldg(Sd.src + (size_t)pe.x * Sd.nt + n);
      const int c = e_side ? pe.y : pe.y - 3;
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (c == k) {
          p[k].x = __fadd_rn(p[k].x, v);
          p[k].y = __fadd_rn(p[k].y, v);
        }
    }
  }
}

// PLAIN_ONLY: an instantiation for lists of plain tiles only, compiled
// with the interior plane loop alone (fewer live registers, no split
// regions); it runs beside the general instantiation, which takes the tiles
// with split-field or probe cells.
template <int TY, bool PLAIN_ONLY>
__global__ void __launch_bounds__(StreamGeom<TY>::THREADS, StreamGeom<TY>::MIN_BLOCKS)
fdtd_step_stream_kernel(const SimDev* __restrict__ sims, const StreamTile* __restrict__ tiles, int n_tiles, int n,
                        unsigned* __restrict__ counter, unsigned base, int* __restrict__ err, int n_main,
                        int n_reg, uint32_t wait_limit, int withhold) {
  using G = StreamGeom<TY>;
  // dynamic shared memory: the E exchange buffers, n_main plane slots (H, E,
  // index), n_reg split regions (E and H pairs of one slab store). A warp
  // holds two plane slots (the plane and its look-ahead) and their regions at
  // a time; a plane's regions are free again once that plane is released.
  extern __shared__ __align__(128) unsigned char smem[];
  float* xch = reinterpret_cast<float*>(smem);  // [2][ex, ez][ER][32]
  unsigned char* ring = smem + 2 * G::XCH;
  __shared__ __align__(8) uint64_t full[kSlotsMax], empty[kSlotsMax];
  __shared__ RegionRec s_rec[kSlotsMax][2];    // each plane's regions A and B
  __shared__ signed char s_memb[G::CONSUMERS];  // each consumer cell's region on core planes (own thread only)
  __shared__ uint32_t s_ruser[kRegionsMax];    // last plane that used each region (producer only)
  __shared__ int s_tq[4];
  const int tid = threadIdx.x;
  const int cur = n & 1, nxt = cur ^ 1;
  constexpr int NC = G::CONSUMERS;
  const int P = n_main;

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
    uint32_t q = 0;    // planes issued
    uint32_t rel = 0;  // planes below rel are known to be released by every consumer warp
    uint32_t nr = 0;   // regions taken
    SlotPos qp{0u, 0u}, rp{0u, 0u};  // ring positions of planes q and rel
    int k = 0;
    const StreamMaps* cur_maps = nullptr;
    bool failed = false;
    // waits until plane u has been released (planes are released in order)
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
      StreamTile td{};
      int nload = 1;
      uint64_t mask = 0;
      const StreamMaps* maps = nullptr;
      const SplitDev* sp = nullptr;
      int snz = 0;
      if (t >= 0) {
        td = load_stream_tile(tiles, t);
        nload = td.z1 - td.z0 + 2;  // planes z0-1 .. z1
        mask = uint64_t(td.split_lo) | (uint64_t(td.split_hi) << 32);
        maps = reinterpret_cast<const StreamMaps*>(sims[td.sim].maps);
        sp = &sims[td.sim].sp;
        snz = sims[td.sim].nz;
        if (maps != cur_maps) {
          tensormap_acquire(&maps->E);
          tensormap_acquire(&maps->H);
          tensormap_acquire(&maps->ids);
          for (int st = 0; st < 6; ++st) {
            tensormap_acquire(&maps->Es[st]);
            tensormap_acquire(&maps->Hs[st]);
          }
          cur_maps = maps;
        }
      }
      const int xs = (td.x0 - 1) & ~3, xi = (td.x0 - 1) & ~7;
      for (int j = 0; j < nload; ++j) {
        const bool last = t >= 0 && j == nload - 1;
        const bool split = t >= 0 && !last && n_reg > 0 && ((mask >> j) & 1u);
        // slab stores staged for this plane: regions A and B of its split slot
        int sa = -1, sbs = -1;
        const int zp = td.z0 - 1 + j;
        if (split) {
          if (zp < sp->t[4]) sa = kStZlo;
          else if (zp >= snz - sp->t[5]) sa = kStZhi;
          else {
            sa = td.ys;
            sbs = td.xs;
          }
        }
        // the plane slot's previous plane, and the split slot's last user, must be released
        if (q >= uint32_t(P) && !release_upto(q - P)) {
          failed = true;
          break;
        }
        const int slot = int(qp.slot);
        // a region for each staged store; a region's last plane must be released
        uint32_t soff[2] = {0u, 0u};
        for (int rgn = 0; rgn < 2; ++rgn) {
          if ((rgn == 0 ? sa : sbs) < 0) continue;
          const uint32_t rs = nr % uint32_t(n_reg);
          if (nr >= uint32_t(n_reg) && !release_upto(s_ruser[rs])) {
            failed = true;
            break;
          }
          s_ruser[rs] = q;
          ++nr;
          soff[rgn] = uint32_t(P) * G::MAIN + rs * G::REGION;
        }
        if (failed) break;
        for (int rgn = 0; rgn < 2; ++rgn) {
          const int st = rgn == 0 ? sa : sbs;
          RegionRec rr{int(soff[rgn]), 0, 0, -1, nullptr, 0};
          if (rgn == 0) rr.kind = sa == kStZlo || sa == kStZhi ? 0 : (sa >= 0 || sbs >= 0) ? 1 : -1;
          if (st >= 0) {
            const int64_t o = sp->off[st] + (int64_t(zp - sp->oz[st]) * sp->h[st] - sp->oy[st]) * sp->w[st] - sp->ox[st];
            rr.w = sp->w[st];
            rr.comp = int(sp->comp[st]);
            rr.pn = sp->base[cur ^ 1] + o;
          }
          s_rec[slot][rgn] = rr;
        }
        if (j == 0) s_tq[k & 3] = t;
        if (t < 0) {  // end of the stream: complete the phase without data
          mbar_arrive(&full[slot]);
          ++q;
          qp = qp.next(P);
          break;
        }
        if (int(q) == withhold) {  // test hook: this plane is never issued, so the waits for it expire
          ++q;
          qp = qp.next(P);
          continue;
        }
        unsigned char* b = ring + uint32_t(slot) * G::MAIN;
        uint64_t* fb = &full[slot];
        fence_proxy_async();
        mbar_arrive_expect_tx(fb, last ? uint32_t(G::HB)
                                       : G::MAIN_BYTES + (sa >= 0 ? G::SPLIT_BYTES : 0u) +
                                             (sbs >= 0 ? G::SPLIT_BYTES : 0u));
        tma_load_5d(b, &maps->H, xs, td.y0 - 1, zp, 0, cur, fb);
        if (!last) {
          tma_load_5d(b + G::OFF_E, &maps->E, xs, td.y0 - 1, zp, 0, cur, fb);
          tma_load_3d(b + G::OFF_I, &maps->ids, xi, td.y0 - 1, zp, fb);
          // split pairs are interleaved along x (float column 2x holds cell
          // x), in each store's own coordinates (origin ox, oy, oz)
          for (int rgn = 0; rgn < 2; ++rgn) {
            const int st = rgn == 0 ? sa : sbs;
            if (st < 0) continue;
            unsigned char* d = ring + soff[rgn];
            const int sx = 2 * (xs - sp->ox[st]), sz = zp - sp->oz[st];
            tma_load_5d(d, &maps->Es[st], sx, td.y0 - 1 - sp->oy[st], sz, 0, cur, fb);
            // H pairs: components 3..5 of the store
            tma_load_5d(d + G::SPLIT_HS, &maps->Hs[st], sx, td.y0 - sp->oy[st], sz, 3, cur, fb);
          }
        }
        ++q;
        qp = qp.next(P);
      }
      if (failed || t < 0) break;
      ++k;
    }
    if (failed) {
      atomicExch(err, kErrWaitExpired);
      // drain the loads still in flight (bounded)
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
    const StreamTile td = load_stream_tile(tiles, ti);
    const SimDev& Sd = sims[td.sim];
    const int x0 = td.x0, y0 = td.y0, z0 = td.z0;
    const int c = x0 - 1 + lane, r = y0 - 1 + w;
    const int oh = (x0 - 1) - ((x0 - 1) & ~3), oi = (x0 - 1) - ((x0 - 1) & ~7);
    const bool own_xy = lane >= 1 && w >= 1 && c < Sd.nx && r < Sd.ny;
    const int plane = Sd.plane;
    float* __restrict__ const fo = Sd.E[nxt][0];   // E then H components of step n+1, N apart
    const int npl = td.z1 - z0 + 1;                // planes z0-1 .. z1-1 computed
    const int hb = w * G::HW + oh + lane;
    const int eb = w * G::EW + oh + lane;
    const int ib = w * G::IW + oi + lane;
    const int sb = (w - 1) * G::EW + oh + lane;    // H split box (owned rows)
    int idx = (z0 - 1) * plane + r * Sd.pitch + c; // cell offset of plane z (owned cells, z >= z0)
    // this thread's cell on the tile's core planes: held by the tile's y-face
    // store (staged as region A: 0), its x-face store (region B: 1) or neither
    // (kept in shared memory: no register across the plane loop)
    if (!PLAIN_ONLY && !td.plain) {
      const int t0 = Sd.sp.t[0], t1 = Sd.sp.t[1], t2 = Sd.sp.t[2], y3 = Sd.ny - Sd.sp.t[3];
      int memb = -1;
      if ((td.ys == kStYlo && r < t2) || (td.ys == kStYhi && r >= y3)) memb = 0;
      else if (r >= t2 && r < y3 && ((td.xs == kStXlo && c < t0) || (td.xs == kStXhi && c >= Sd.nx - t1))) memb = 1;
      s_memb[tid] = (signed char)memb;
    }

    // The plane loop, instantiated for plain tiles (FAST: every cell unsplit,
    // no probes, so no per-cell flag tests) and for the general case.
    auto planes = [&](auto fast_tag) -> bool {
      constexpr bool FAST = decltype(fast_tag)::value;
      float ex_p = 0.f, ey_p = 0.f;  // E^{n+1} of this cell one plane below
      // this cell's table row, reloaded when its material index changes along
      // z (declared per path: the interior path keeps only the words it reads)
      const float4* __restrict__ const rows = Sd.rows;
      int row_id = -1;
      float4 ra = {}, rb = {}, rd = {}, rp = {}, rq = {}, ru = {}, rv = {}, r7 = {};
      for (int i = 0; i < npl; ++i) {
        const SlotPos np = cp.next(P);
        // plane z was waited for as the look-ahead of the previous iteration
        ok = ok && mbar_wait_bounded(&full[np.slot], np.par, wait_limit);
        const unsigned char* st = ring + cp.slot * G::MAIN;
        const float* sH = reinterpret_cast<const float*>(st);
        const float* sE = reinterpret_cast<const float*>(st + G::OFF_E);
        const uint16_t* sI = reinterpret_cast<const uint16_t*>(st + G::OFF_I);
        const float* nH = reinterpret_cast<const float*>(ring + np.slot * G::MAIN);
        float* xb = xch + (i & 1) * (G::XCH / 4);
        constexpr int HC = G::HC, EC = G::EC;
        const bool store = own_xy && i > 0;
        const int z = z0 - 1 + i;
        // split pairs of this plane: the slab stores the producer staged in
        // regions A and B (region 0 / 1 of a cell that one of them holds),
        // other stores and sparse cells from global memory (region -1)
        const RegionRec* const rr = s_rec[cp.slot];
        // the E (m < 3) or H pair of component m of this cell, from its
        // staged region or the store
        auto pair_in = [&](int rgn, int m, const float2* gp, int cs) -> float2 {
          if (rgn < 0) return __ldg(gp + m * cs);
          const unsigned char* rg = ring + rr[rgn].smem;
          return m < 3 ? reinterpret_cast<const float2*>(rg)[m * EC + eb]
                       : reinterpret_cast<const float2*>(rg + G::SPLIT_HS)[(m - 3) * G::SHC + sb];
        };

        // ------------------------------------------------------------ E phase
        // (after an expired wait the values are stale but in bounds; the vote
        // below then ends the block before anything is stored)
        const float hx_c = sH[hb], hy_c = sH[HC + hb], hz_c = sH[2 * HC + hb];
        const float dhz_y = sH[2 * HC + hb + G::HW] - hz_c, dhy_z = nH[HC + hb] - hy_c;
        const float dhx_z = nH[hb] - hx_c, dhz_x = sH[2 * HC + hb + 1] - hz_c;
        const float dhy_x = sH[HC + hb + 1] - hy_c, dhx_y = sH[hb + G::HW] - hx_c;
        const int id = ok ? int(sI[ib]) : 0;  // a stage that never arrived may hold any bits
        if (i + 1 < npl) {
          // the next plane's row into L1 while this plane computes
          const int idn = reinterpret_cast<const uint16_t*>(ring + np.slot * G::MAIN + G::OFF_I)[ib];
          if (ok && idn != id) prefetch_l1(rows + 8 * idn);
        }
        if (id != row_id) {
          const float4* row = rows + 8 * id;
          ra = __ldg(row); rb = __ldg(row + 1); rd = __ldg(row + 2); rp = __ldg(row + 3);
          rq = __ldg(row + 4); ru = __ldg(row + 5); rv = __ldg(row + 6); r7 = __ldg(row + 7);
          row_id = id;
        }
        const uint32_t flags = __float_as_uint(r7.z);
        // a split cell's store, staged region (-1: none) and pair offset,
        // found once per plane for both phases
        // (so: from the staged region's pointers, or from the store base for region -1)
        int rgn = -1, cs = 0;
        int64_t so = 0;
        if (!FAST && (flags & (kESplit | kHSplit))) {
          const int kind = rr[0].kind;
          rgn = kind == 0 ? 0 : kind == 1 ? int(s_memb[tid]) : -1;
          if (rgn >= 0) {
            so = int64_t(r) * rr[rgn].w + c;
            cs = rr[rgn].comp;
          } else {
            so = split_off(Sd.sp, split_store(Sd.sp, Sd.nx, Sd.ny, Sd.nz, c, r, z), c, r, z,
                           __float_as_int(r7.w), cs);
          }
        }
        float ex, ey, ez;
        if (FAST || !(flags & kESplit)) {
          // both splits share Ca: f' = Ca f + Cb1 d1 + Cb2 d2
          ex = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
          ey = upd_e(rb.x, sE[EC + eb], rb.y, dhx_z, rb.w, dhz_x);
          ez = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
        } else {
          // per component: the split pair (one 8-byte load) or the unsplit total
          float2 sp[3];
          const float2* gp = rgn >= 0 ? nullptr : Sd.sp.base[cur] + so;  // read only for region -1
  #pragma unroll
          for (int m = 0; m < 3; ++m) sp[m] = make_float2(0.f, 0.f);
          if (flags & (kCompSplit0 << 0)) {
            sp[0] = pair_in(rgn, 0, gp, cs);
            sp[0].x = upd_e_split(ra.x, sp[0].x, ra.y, dhz_y);  // ex_y
            sp[0].y = upd_e_split(ra.z, sp[0].y, ra.w, dhy_z);  // ex_z
          } else {
            ex = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
          }
          if (flags & (kCompSplit0 << 1)) {
            sp[1] = pair_in(rgn, 1, gp, cs);
            sp[1].x = upd_e_split(rb.x, sp[1].x, rb.y, dhx_z);  // ey_z
            sp[1].y = upd_e_split(rb.z, sp[1].y, rb.w, dhz_x);  // ey_x
          } else {
            ey = upd_e(rb.x, sE[EC + eb], rb.y, dhx_z, rb.w, dhz_x);
          }
          if (flags & (kCompSplit0 << 2)) {
            sp[2] = pair_in(rgn, 2, gp, cs);
            sp[2].x = upd_e_split(rd.x, sp[2].x, rd.y, dhy_x);  // ez_x
            sp[2].y = upd_e_split(rd.z, sp[2].y, rd.w, dhx_y);  // ez_y
          } else {
            ez = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
          }
          if (flags >> 16) stream_inject(Sd, r7, flags, n, true, sp);
          if (flags & (kCompSplit0 << 0)) ex = __fadd_rn(sp[0].x, sp[0].y);
          if (flags & (kCompSplit0 << 1)) ey = __fadd_rn(sp[1].x, sp[1].y);
          if (flags & (kCompSplit0 << 2)) ez = __fadd_rn(sp[2].x, sp[2].y);
          if (store) {
            float2* po = rgn >= 0 ? rr[rgn].pn + so : Sd.sp.base[nxt] + so;
  #pragma unroll
            for (int m = 0; m < 3; ++m)
              if (flags & (kCompSplit0 << m)) po[m * cs] = sp[m];
          }
        }
        xb[w * 32 + lane] = ex;
        xb[G::ER * 32 + w * 32 + lane] = ez;
        const float ey_xm = __shfl_up_sync(0xffffffffu, ey, 1);
        const float ez_xm = __shfl_up_sync(0xffffffffu, ez, 1);
        // E^{n+1}(z) of the block complete; a consumer whose wait expired votes here
        if (named_bar_or(kStreamBar, NC, !ok)) {
          if (tid == 0) atomicExch(err, kErrWaitExpired);
          return false;
        }

        // ------------------------------------------------------------ H phase
        if (store) {
          const float ex_ym = xb[(w - 1) * 32 + lane];
          const float ez_ym = xb[G::ER * 32 + (w - 1) * 32 + lane];
          // totals of the components not stored split
          if (FAST || !(flags & (kCompSplit0 << 0))) fo[idx] = ex;
          const int64_t N = Sd.cells;  // floats per component, read where used: no register across the plane loop
          if (FAST || !(flags & (kCompSplit0 << 1))) fo[N + idx] = ey;
          if (FAST || !(flags & (kCompSplit0 << 2))) fo[2 * N + idx] = ez;
          // slots 12..29: (Da, Db1, Db2) of hx_y, hx_z, hy_z, hy_x, hz_x, hz_y
          const float gxy = h_term(rp.z, ez, rp.y, ez_ym);
          const float gxz = h_term(rq.y, ey, rq.x, ey_p);
          const float gyz = h_term(ru.x, ex, rq.w, ex_p);
          const float gyx = h_term(ru.w, ez, ru.z, ez_xm);
          const float gzx = h_term(rv.z, ey, rv.y, ey_xm);
          const float gzy = h_term(r7.y, ex, r7.x, ex_ym);
          float hx, hy, hz;
          if (FAST || !(flags & kHSplit)) {
            hx = upd_h(rp.x, hx_c, gxy, gxz);
            hy = upd_h(rq.z, hy_c, gyz, gyx);
            hz = upd_h(rv.x, hz_c, gzx, gzy);
          } else {
            float2 sp[3];
            const float2* gp = rgn >= 0 ? nullptr : Sd.sp.base[cur] + so;  // read only for region -1
  #pragma unroll
            for (int m = 0; m < 3; ++m) sp[m] = make_float2(0.f, 0.f);
            if (flags & (kCompSplit0 << 3)) {
              sp[0] = pair_in(rgn, 3, gp, cs);
              sp[0].x = upd_h_split(rp.x, sp[0].x, gxy);
              sp[0].y = upd_h_split(rp.w, sp[0].y, gxz);
            } else {
              hx = upd_h(rp.x, hx_c, gxy, gxz);
            }
            if (flags & (kCompSplit0 << 4)) {
              sp[1] = pair_in(rgn, 4, gp, cs);
              sp[1].x = upd_h_split(rq.z, sp[1].x, gyz);
              sp[1].y = upd_h_split(ru.y, sp[1].y, gyx);
            } else {
              hy = upd_h(rq.z, hy_c, gyz, gyx);
            }
            if (flags & (kCompSplit0 << 5)) {
              sp[2] = pair_in(rgn, 5, gp, cs);
              sp[2].x = upd_h_split(rv.x, sp[2].x, gzx);
              sp[2].y = upd_h_split(rv.w, sp[2].y, gzy);
            } else {
              hz = upd_h(rv.x, hz_c, gzx, gzy);
            }
            if (flags >> 16) stream_inject(Sd, r7, flags, n, false, sp);
            if (flags & (kCompSplit0 << 3)) hx = __fadd_rn(sp[0].x, sp[0].y);
            if (flags & (kCompSplit0 << 4)) hy = __fadd_rn(sp[1].x, sp[1].y);
            if (flags & (kCompSplit0 << 5)) hz = __fadd_rn(sp[2].x, sp[2].y);
            float2* po = rgn >= 0 ? rr[rgn].pn + so : Sd.sp.base[nxt] + so;
  #pragma unroll
            for (int m = 0; m < 3; ++m)
              if (flags & (kCompSplit0 << (3 + m))) po[(3 + m) * cs] = sp[m];
          }
          fo[3 * N + idx] = hx;
          fo[4 * N + idx] = hy;
          fo[5 * N + idx] = hz;
          const int np = FAST ? 0 : int(flags >> 16);
          if (np) {  // record the probes of this cell (solver.cu:467, 521)
            const int first = __float_as_int(r7.w);
            for (int e = 0; e < np; ++e) {
              const int2 pe = __ldg(Sd.cell_probes + first + e);
              const float val = pe.y == 0 ? ex : pe.y == 1 ? ey : pe.y == 2 ? ez : pe.y == 3 ? hx : pe.y == 4 ? hy : hz;
              Sd.rec[(size_t)pe.x * Sd.nt + n] = val;
            }
          }
        }
        ex_p = ex;
        ey_p = ey;
        // plane z is no longer read by this warp
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[cp.slot]);
        cp = np;
        idx += plane;
      }
      return true;
    };
    if constexpr (PLAIN_ONLY) {
      if (!planes(std::true_type{})) return;
    } else {
      if (!(td.plain ? planes(std::true_type{}) : planes(std::false_type{}))) return;
    }
    // the look-ahead plane z1 was read only by the last iteration
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[cp.slot]);
    cp = cp.next(P);
  }
}

}  // namespace rfn
