// Row-marching step kernel for sm_100a: the streaming kernel's tiles and TMA
// boxes, with each consumer warp walking TY rows of its tile per z plane.
//
// Same update as fdtd_step_kernel (fdtd_kernels.cuh) through the same
// rounding-fixed helpers, so all step kernels produce the same bits.
//
//   tile      31 (x) by XW*TY (y) owned cells and a z range [z0, z1), the
//             streaming kernel's tile list and tensor maps (StreamTile,
//             StreamMaps) with tile height XW*TY. Consumer warp w owns rows
//             y0 + w*TY .. y0 + w*TY + TY-1; lane l sits on column x0-1+l.
//   per plane a warp first recomputes E^{n+1} (ex, ez) of the row below its
//             rows (its own halo row), then for each of its rows computes
//             E^{n+1} and, from it, H^{n+1}: the row below's E^{n+1} is still
//             in registers, the x neighbour comes by warp shuffle and the
//             plane below's E^{n+1} was kept per row. H^n of row r+1, read
//             for the E update of row r, is row r+1's own H^n. The warps of
//             a block never wait for each other: no block barrier, no
//             shared-memory exchange.
//   planes    the producer warp (lane 0) streams planes z0-1 .. z1 of each
//             tile into shared memory: H, E and the material index into one of
//             n_main plane slots ("full" and "empty" mbarrier each), and, for
//             the planes the host flagged as holding split-field cells, the
//             six split pairs (over the tile width or a 16-column window) into
//             one of n_split split slots, free again once the plane that used
//             it is released. The last plane of a tile is only the look-ahead
//             of dH/dz (H). A warp holds at most two plane slots (the plane
//             and its look-ahead) and one split slot, so two of each suffice
//             for progress; the rest are loads in flight.
//   waits     every mbarrier wait is bounded; a warp whose wait expires
//             records an error code and returns, the producer gives up and
//             drains its own loads (bounded) before it returns.
#pragma once

#include "fdtd_step_stream.cuh"

namespace rfn {

constexpr int kMarchSlots = 8;  // plane slots at most (a tile streams >= 3 planes: s_tq holds 4 tiles)
constexpr int kMarchSplitSlots = 4;

template <int XW, int TY>
struct MarchGeom {
  static constexpr int ROWS = XW * TY;                  // owned rows per tile
  static constexpr int HW = 40, EW = 36, IW = 40;       // box widths along x (as the streaming kernel)
  static constexpr int HR = ROWS + 2, ER = ROWS + 1;    // box heights: rows y0-1 .. y0+ROWS (H), .. y0+ROWS-1
  static constexpr int HC = HR * HW;                    // floats per H component
  static constexpr int EC = ER * EW;                    // floats per E component
  static constexpr int HB = 3 * HC * 4, EB = 3 * EC * 4, IB = ER * IW * 2;
  static constexpr int A(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_E = A(HB), OFF_I = OFF_E + A(EB), OFF_S = OFF_I + A(IB);
  // split pairs over the tile width: E [3][ER][36], H [3][ROWS][36]; narrow window: 16 columns
  static constexpr int SEF = 3 * ER * EW * 8, SHF = 3 * ROWS * EW * 8;
  static constexpr int SEN = 3 * ER * kStreamWin * 8, SHN = 3 * ROWS * kStreamWin * 8;
  static constexpr uint32_t MAIN = OFF_S;                          // plane slot bytes (H, E, index)
  static constexpr uint32_t SPLIT = A(SEF) + A(SHF);                // split slot bytes (36 columns)
  static constexpr uint32_t SPLIT_HS_F = A(SEF), SPLIT_HS_N = A(SEN); // H pairs inside a split slot
  static constexpr int THREADS = 32 * (XW + 1);
};

template <int XW, int TY>
__global__ void __launch_bounds__(MarchGeom<XW, TY>::THREADS, 1)
fdtd_step_march_kernel(const SimDev* __restrict__ sims, const StreamTile* __restrict__ tiles, int n_tiles, int n,
                       unsigned* __restrict__ counter, unsigned base, int* __restrict__ err, int n_main,
                       int n_split, uint32_t wait_limit, int withhold) {
  using G = MarchGeom<XW, TY>;
  constexpr int NC = 32 * XW;
  const int P = n_main;  // plane slots (2 .. kMarchSlots), then n_split split slots (2 .. kMarchSplitSlots)
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) uint64_t full[kMarchSlots], empty[kMarchSlots];
  __shared__ uint32_t s_soff[kMarchSlots];       // byte offset of the plane's split slot (read by the consumers)
  __shared__ uint32_t s_suser[kMarchSplitSlots]; // last plane that used each split slot (producer only)
  __shared__ int s_tq[4];
  const int tid = threadIdx.x;
  const int cur = n & 1, nxt = cur ^ 1;

  if (tid == 0) {
    for (int s = 0; s < P; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], XW);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // =================================================================== producer
  if (tid >= NC) {
    if (tid != NC) return;
    uint32_t q = 0;    // planes issued
    uint32_t rel = 0;  // planes below rel are known to be released by every consumer warp
    uint32_t ns = 0;   // split slots taken
    int k = 0;
    const StreamMaps* cur_maps = nullptr;
    bool failed = false;
    // waits until plane u has been released (planes are released in order)
    auto release_upto = [&](uint32_t u) -> bool {
      while (rel <= u) {
        if (!mbar_wait_bounded(&empty[rel % P], (rel / P) & 1u, wait_limit)) return false;
        ++rel;
      }
      return true;
    };
    for (;;) {
      const unsigned v = atomicAdd(counter, 1u) - base;
      const int t = v < unsigned(n_tiles) ? int(v) : -1;
      StreamTile td{};
      int nload = 1;
      uint64_t mask = 0, narrow = 0;
      const StreamMaps* maps = nullptr;
      if (t >= 0) {
        td = load_stream_tile(tiles, t);
        nload = td.z1 - td.z0 + 2;  // planes z0-1 .. z1
        mask = uint64_t(td.split_lo) | (uint64_t(td.split_hi) << 32);
        narrow = uint64_t(td.narrow_lo) | (uint64_t(td.narrow_hi) << 32);
        maps = reinterpret_cast<const StreamMaps*>(sims[td.sim].maps);
        if (maps != cur_maps) {
          tensormap_acquire(&maps->E);
          tensormap_acquire(&maps->H);
          tensormap_acquire(&maps->ids);
          tensormap_acquire(&maps->Es);
          tensormap_acquire(&maps->Hs);
          tensormap_acquire(&maps->Es16);
          tensormap_acquire(&maps->Hs16);
          cur_maps = maps;
        }
      }
      const int xs = (td.x0 - 1) & ~3, xi = (td.x0 - 1) & ~7;
      for (int j = 0; j < nload; ++j) {
        const bool last = t >= 0 && j == nload - 1;
        const bool split = t >= 0 && !last && ((mask >> j) & 1u);
        const bool win = (narrow >> j) & 1u;
        // the plane slot's previous plane, and the split slot's last user, must be released
        if (q >= uint32_t(P) && !release_upto(q - P)) {
          failed = true;
          break;
        }
        const int slot = int(q % P);
        uint32_t soff = 0;
        if (split) {
          const uint32_t ss = ns % uint32_t(n_split);
          if (ns >= uint32_t(n_split) && !release_upto(s_suser[ss])) {
            failed = true;
            break;
          }
          s_suser[ss] = q;
          ++ns;
          soff = uint32_t(P) * G::MAIN + ss * G::SPLIT;
        }
        s_soff[slot] = soff;
        if (j == 0) s_tq[k & 3] = t;
        if (t < 0) {  // end of the stream: complete the phase without data
          mbar_arrive(&full[slot]);
          ++q;
          break;
        }
        if (int(q) == withhold) {  // test hook: this plane is never issued (its waits expire)
          ++q;
          continue;
        }
        unsigned char* b = ring + uint32_t(slot) * G::MAIN;
        unsigned char* sb = ring + soff;
        uint64_t* fb = &full[slot];
        const int zp = td.z0 - 1 + j;
        fence_proxy_async();
        mbar_arrive_expect_tx(fb, last ? uint32_t(G::HB)
                                  : uint32_t(G::HB + G::EB + G::IB) +
                                        (!split ? 0u : win ? uint32_t(G::SEN + G::SHN) : uint32_t(G::SEF + G::SHF)));
        tma_load_5d(b, &maps->H, xs, td.y0 - 1, zp, 0, cur, fb);
        if (!last) {
          tma_load_5d(b + G::OFF_E, &maps->E, xs, td.y0 - 1, zp, 0, cur, fb);
          tma_load_3d(b + G::OFF_I, &maps->ids, xi, td.y0 - 1, zp, fb);
          // split pairs are interleaved along x: float column 2x holds cell x
          if (split && win) {
            tma_load_5d(sb, &maps->Es16, 2 * td.wx0, td.y0 - 1, zp, 0, cur, fb);
            tma_load_5d(sb + G::SPLIT_HS_N, &maps->Hs16, 2 * td.wx0, td.y0, zp, 0, cur, fb);
          } else if (split) {
            tma_load_5d(sb, &maps->Es, 2 * xs, td.y0 - 1, zp, 0, cur, fb);
            tma_load_5d(sb + G::SPLIT_HS_F, &maps->Hs, 2 * xs, td.y0, zp, 0, cur, fb);
          }
        }
        ++q;
      }
      if (failed || t < 0) break;
      ++k;
    }
    if (failed) {
      atomicExch(err, kErrWaitExpired);
      // drain the loads still in flight (bounded)
      for (uint32_t r = rel; r < q; ++r) mbar_wait_bounded(&full[r % P], (r / P) & 1u, wait_limit);
    }
    return;
  }

  // ================================================================== consumers
  const int lane = tid & 31, w = tid >> 5;
  // coefficient rows kept while the material index does not change: the E
  // part (slots 0..11, flags, probe entry) and the H part (slots 12..29)
  const float4* __restrict__ rows = nullptr;
  int rid_e = -1, rid_h = -1;
  float4 ra = {}, rb = {}, rd = {}, rp = {}, rq = {}, ru = {}, rv = {};
  float hb1 = 0.f, hb2 = 0.f;  // Db1, Db2 of hz_y (slots 28, 29)
  uint32_t fl_e = 0, fl_h = 0;
  int pr_e = 0, pr_h = 0;
  uint32_t q = 0;  // plane sequence number: slot q % n_main, phase parity (q / n_main) & 1
  for (int k = 0;; ++k) {
    if (!mbar_wait_bounded(&full[q % P], (q / P) & 1u, wait_limit)) {
      if (lane == 0) atomicExch(err, kErrWaitExpired);
      return;
    }
    const int ti = s_tq[k & 3];
    if (ti < 0) break;
    const StreamTile td = load_stream_tile(tiles, ti);
    const SimDev& Sd = sims[td.sim];
    if (Sd.rows != rows) {
      rows = Sd.rows;
      rid_e = rid_h = -1;
    }
    const int x0 = td.x0, y0 = td.y0, z0 = td.z0;
    const int c = x0 - 1 + lane;
    const int oh = (x0 - 1) - ((x0 - 1) & ~3), oi = (x0 - 1) - ((x0 - 1) & ~7);
    const bool own_x = lane >= 1 && c < Sd.nx;
    const int ny = Sd.ny;
    const int plane = Sd.plane, pitch = Sd.pitch;
    const int64_t N = Sd.cells;
    float* __restrict__ const fo = Sd.E[nxt][0];   // E then H components of step n+1, N apart
    float2* __restrict__ const spo = Sd.Es[nxt][0]; // split pairs of step n+1: E comp m at m N, H comp m at (3+m) N
    const int npl = td.z1 - z0 + 1;                 // planes z0-1 .. z1-1 computed
    const int wc = c - td.wx0;                      // column inside the narrow window
    const uint64_t narrow = uint64_t(td.narrow_lo) | (uint64_t(td.narrow_hi) << 32);
    const uint64_t smask = uint64_t(td.split_lo) | (uint64_t(td.split_hi) << 32);
    const int br0 = w * TY;                         // box row of this warp's halo row (grid row y0-1+br0)
    // cell offset of (c, y0-1+br0, z0-1); rows of this warp follow at +pitch
    int idx0 = (z0 - 1) * plane + (y0 - 1 + br0) * pitch + c;
    float exp_[TY], eyp_[TY];                       // E^{n+1} of the plane below, per owned row

    auto planes = [&](auto fast_tag) -> bool {
      constexpr bool FAST = decltype(fast_tag)::value;
#pragma unroll
      for (int j = 0; j < TY; ++j) exp_[j] = eyp_[j] = 0.f;
      for (int i = 0; i < npl; ++i) {
        const uint32_t qn = q + 1;
        // plane z+1 (the look-ahead of dH/dz)
        if (!mbar_wait_bounded(&full[qn % P], (qn / P) & 1u, wait_limit)) {
          if (lane == 0) atomicExch(err, kErrWaitExpired);
          return false;
        }
        const unsigned char* st = ring + (q % P) * G::MAIN;
        const float* sH = reinterpret_cast<const float*>(st);
        const float* sE = reinterpret_cast<const float*>(st + G::OFF_E);
        const uint16_t* sI = reinterpret_cast<const uint16_t*>(st + G::OFF_I);
        const bool win = (narrow >> i) & 1u;
        const unsigned char* ss = ring + s_soff[q % P];
        const float2* sEs = reinterpret_cast<const float2*>(ss);
        const float2* sHs = reinterpret_cast<const float2*>(ss + (win ? G::SPLIT_HS_N : G::SPLIT_HS_F));
        const float* nH = reinterpret_cast<const float*>(ring + (qn % P) * G::MAIN);
        const bool hphase = i > 0;                   // plane z0-1 only seeds E^{n+1}(z-1)
        const bool splitp = !FAST && ((smask >> i) & 1u);
        const int sw = win ? kStreamWin : G::EW;     // split box width
        const int scol = win ? wc : oh + lane;       // this cell's column in the split box
        constexpr int HC = G::HC, EC = G::EC, HW = G::HW, EW = G::EW, IW = G::IW;

        // row loaders: the E part and the H part of the coefficient row of material id
        auto load_e = [&](int id) {
          if (id != rid_e) {
            const float4* row = rows + 8 * id;
            ra = __ldg(row); rb = __ldg(row + 1); rd = __ldg(row + 2);
            const float4 r7 = __ldg(row + 7);
            fl_e = __float_as_uint(r7.z);
            pr_e = __float_as_int(r7.w);
            rid_e = id;
          }
        };
        auto load_h = [&](int id) {
          if (id != rid_h) {
            const float4* row = rows + 8 * id;
            rp = __ldg(row + 3); rq = __ldg(row + 4); ru = __ldg(row + 5); rv = __ldg(row + 6);
            const float4 r7 = __ldg(row + 7);
            hb1 = r7.x; hb2 = r7.y;
            fl_h = __float_as_uint(r7.z);
            pr_h = __float_as_int(r7.w);
            rid_h = id;
          }
        };

        // ---------------------------------------------------- halo row (j = 0)
        // H^n of the current row, carried down the rows
        const int hb0 = br0 * HW + oh + lane;
        float hx0 = sH[hb0], hy0 = sH[HC + hb0], hz0 = sH[2 * HC + hb0];
        float ex_ym = 0.f, ez_ym = 0.f;  // E^{n+1} of the row below
        if (hphase) {
          const float hx1 = sH[hb0 + HW], hz1 = sH[2 * HC + hb0 + HW];
          const float dhz_y = hz1 - hz0, dhy_z = nH[HC + hb0] - hy0;
          const float dhy_x = sH[HC + hb0 + 1] - hy0, dhx_y = hx1 - hx0;
          const int eb = br0 * EW + oh + lane;
          load_e(int(sI[br0 * IW + oi + lane]));
          if (FAST || !(fl_e & kESplit)) {
            ex_ym = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
            ez_ym = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
          } else {
            float2 sp[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) sp[m] = make_float2(0.f, 0.f);
            const float2* sP = sEs + br0 * sw + scol;
            if (fl_e & (kCompSplit0 << 0)) {
              sp[0] = sP[0];
              sp[0].x = upd_e_split(ra.x, sp[0].x, ra.y, dhz_y);
              sp[0].y = upd_e_split(ra.z, sp[0].y, ra.w, dhy_z);
            } else {
              ex_ym = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
            }
            if (fl_e & (kCompSplit0 << 2)) {
              sp[2] = sP[2 * G::ER * sw];
              sp[2].x = upd_e_split(rd.x, sp[2].x, rd.y, dhy_x);
              sp[2].y = upd_e_split(rd.z, sp[2].y, rd.w, dhx_y);
            } else {
              ez_ym = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
            }
            if (fl_e >> 16) stream_inject(Sd, make_float4(0.f, 0.f, 0.f, __int_as_float(pr_e)), fl_e, n, true, sp);
            if (fl_e & (kCompSplit0 << 0)) ex_ym = __fadd_rn(sp[0].x, sp[0].y);
            if (fl_e & (kCompSplit0 << 2)) ez_ym = __fadd_rn(sp[2].x, sp[2].y);
          }
        }

        // ---------------------------------------------------- owned rows
        // H^n of the first owned row (the row above the halo row)
        hx0 = sH[hb0 + HW];
        hy0 = sH[HC + hb0 + HW];
        hz0 = sH[2 * HC + hb0 + HW];
#pragma unroll
        for (int j = 1; j <= TY; ++j) {
          const int br = br0 + j;                  // box row (grid row y0-1+br)
          const int hb = br * HW + oh + lane;
          const float hx1 = sH[hb + HW], hy1 = sH[HC + hb + HW], hz1 = sH[2 * HC + hb + HW];
          const float dhz_y = hz1 - hz0, dhx_y = hx1 - hx0;
          const float dhz_x = sH[2 * HC + hb + 1] - hz0, dhy_x = sH[HC + hb + 1] - hy0;
          const float dhy_z = nH[HC + hb] - hy0, dhx_z = nH[hb] - hx0;
          const int eb = br * EW + oh + lane;
          const int id = int(sI[br * IW + oi + lane]);
          load_e(id);
          float ex, ey, ez;
          float2 sp[3];
          if (FAST || !(fl_e & kESplit)) {
            // both splits share Ca: f' = Ca f + Cb1 d1 + Cb2 d2
            ex = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
            ey = upd_e(rb.x, sE[EC + eb], rb.y, dhx_z, rb.w, dhz_x);
            ez = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
          } else {
#pragma unroll
            for (int m = 0; m < 3; ++m) sp[m] = make_float2(0.f, 0.f);
            const float2* sP = sEs + br * sw + scol;
            if (fl_e & (kCompSplit0 << 0)) {
              sp[0] = sP[0];
              sp[0].x = upd_e_split(ra.x, sp[0].x, ra.y, dhz_y);  // ex_y
              sp[0].y = upd_e_split(ra.z, sp[0].y, ra.w, dhy_z);  // ex_z
            } else {
              ex = upd_e(ra.x, sE[eb], ra.y, dhz_y, ra.w, dhy_z);
            }
            if (fl_e & (kCompSplit0 << 1)) {
              sp[1] = sP[G::ER * sw];
              sp[1].x = upd_e_split(rb.x, sp[1].x, rb.y, dhx_z);  // ey_z
              sp[1].y = upd_e_split(rb.z, sp[1].y, rb.w, dhz_x);  // ey_x
            } else {
              ey = upd_e(rb.x, sE[EC + eb], rb.y, dhx_z, rb.w, dhz_x);
            }
            if (fl_e & (kCompSplit0 << 2)) {
              sp[2] = sP[2 * G::ER * sw];
              sp[2].x = upd_e_split(rd.x, sp[2].x, rd.y, dhy_x);  // ez_x
              sp[2].y = upd_e_split(rd.z, sp[2].y, rd.w, dhx_y);  // ez_y
            } else {
              ez = upd_e(rd.x, sE[2 * EC + eb], rd.y, dhy_x, rd.w, dhx_y);
            }
            if (fl_e >> 16) stream_inject(Sd, make_float4(0.f, 0.f, 0.f, __int_as_float(pr_e)), fl_e, n, true, sp);
            if (fl_e & (kCompSplit0 << 0)) ex = __fadd_rn(sp[0].x, sp[0].y);
            if (fl_e & (kCompSplit0 << 1)) ey = __fadd_rn(sp[1].x, sp[1].y);
            if (fl_e & (kCompSplit0 << 2)) ez = __fadd_rn(sp[2].x, sp[2].y);
          }
          const float ey_xm = __shfl_up_sync(0xffffffffu, ey, 1);
          const float ez_xm = __shfl_up_sync(0xffffffffu, ez, 1);
          const int idx = idx0 + j * pitch;
          if (hphase && own_x && y0 - 1 + br < ny) {
            if (!FAST && (fl_e & kESplit)) {
#pragma unroll
              for (int m = 0; m < 3; ++m)
                if (fl_e & (kCompSplit0 << m)) spo[m * N + idx] = sp[m];
            }
            // totals of the components not stored split
            if (FAST || !(fl_e & (kCompSplit0 << 0))) fo[idx] = ex;
            if (FAST || !(fl_e & (kCompSplit0 << 1))) fo[N + idx] = ey;
            if (FAST || !(fl_e & (kCompSplit0 << 2))) fo[2 * N + idx] = ez;
            load_h(id);
            // slots 12..29: (Da, Db1, Db2) of hx_y, hx_z, hy_z, hy_x, hz_x, hz_y
            const float gxy = h_term(rp.z, ez, rp.y, ez_ym);
            const float gxz = h_term(rq.y, ey, rq.x, eyp_[j - 1]);
            const float gyz = h_term(ru.x, ex, rq.w, exp_[j - 1]);
            const float gyx = h_term(ru.w, ez, ru.z, ez_xm);
            const float gzx = h_term(rv.z, ey, rv.y, ey_xm);
            const float gzy = h_term(hb2, ex, hb1, ex_ym);
            float hx, hy, hz;
            if (FAST || !(fl_h & kHSplit)) {
              hx = upd_h(rp.x, hx0, gxy, gxz);
              hy = upd_h(rq.z, hy0, gyz, gyx);
              hz = upd_h(rv.x, hz0, gzx, gzy);
            } else {
              float2 hp[3];
#pragma unroll
              for (int m = 0; m < 3; ++m) hp[m] = make_float2(0.f, 0.f);
              const float2* sP = sHs + (br - 1) * sw + scol;
              if (fl_h & (kCompSplit0 << 3)) {
                hp[0] = sP[0];
                hp[0].x = upd_h_split(rp.x, hp[0].x, gxy);
                hp[0].y = upd_h_split(rp.w, hp[0].y, gxz);
              } else {
                hx = upd_h(rp.x, hx0, gxy, gxz);
              }
              if (fl_h & (kCompSplit0 << 4)) {
                hp[1] = sP[G::ROWS * sw];
                hp[1].x = upd_h_split(rq.z, hp[1].x, gyz);
                hp[1].y = upd_h_split(ru.y, hp[1].y, gyx);
              } else {
                hy = upd_h(rq.z, hy0, gyz, gyx);
              }
              if (fl_h & (kCompSplit0 << 5)) {
                hp[2] = sP[2 * G::ROWS * sw];
                hp[2].x = upd_h_split(rv.x, hp[2].x, gzx);
                hp[2].y = upd_h_split(rv.w, hp[2].y, gzy);
              } else {
                hz = upd_h(rv.x, hz0, gzx, gzy);
              }
              if (fl_h >> 16) stream_inject(Sd, make_float4(0.f, 0.f, 0.f, __int_as_float(pr_h)), fl_h, n, false, hp);
              if (fl_h & (kCompSplit0 << 3)) hx = __fadd_rn(hp[0].x, hp[0].y);
              if (fl_h & (kCompSplit0 << 4)) hy = __fadd_rn(hp[1].x, hp[1].y);
              if (fl_h & (kCompSplit0 << 5)) hz = __fadd_rn(hp[2].x, hp[2].y);
#pragma unroll
              for (int m = 0; m < 3; ++m)
                if (fl_h & (kCompSplit0 << (3 + m))) spo[(3 + m) * N + idx] = hp[m];
            }
            fo[3 * N + idx] = hx;
            fo[4 * N + idx] = hy;
            fo[5 * N + idx] = hz;
            const int np = FAST ? 0 : int(fl_h >> 16);
            if (np) {  // record the probes of this cell (solver.cu:467, 521)
              for (int e = 0; e < np; ++e) {
                const int2 pe = __ldg(Sd.cell_probes + pr_h + e);
                const float val = pe.y == 0 ? ex : pe.y == 1 ? ey : pe.y == 2 ? ez : pe.y == 3 ? hx : pe.y == 4 ? hy : hz;
                Sd.rec[(size_t)pe.x * Sd.nt + n] = val;
              }
            }
          }
          (void)splitp;
          ex_ym = ex;
          ez_ym = ez;
          exp_[j - 1] = ex;
          eyp_[j - 1] = ey;
          hx0 = hx1;
          hy0 = hy1;
          hz0 = hz1;
        }
        // plane z is no longer read by this warp
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[q % P]);
        ++q;
        idx0 += plane;
      }
      return true;
    };
    if (!(td.plain ? planes(std::true_type{}) : planes(std::false_type{}))) return;
    // the look-ahead plane z1 was read only by the last iteration
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q % P]);
    ++q;
  }
}

}  // namespace rfn
