// TMA-pipelined, warp-specialized FDTD step kernels for sm_100a.
//
// Same update as fdtd_step_kernel (fdtd_kernels.cuh) through the same
// rounding-fixed helpers, so every variant produces the same bits; the planes
// are staged in shared memory by the tensor-memory accelerator instead of
// per-thread loads.
//
//   tile      TX (x) by TY (y) owned cells and a z range [z0, z1), clipped to
//             [x0, x1) x [y0, y1). E is also recomputed on the halo row y0-1,
//             the halo float4 column x0-4..x0-1 and the plane z0-1, so H needs
//             no second sweep over memory.
//   stream    a persistent block consumes one continuous stream of z planes:
//             the planes z0-1 .. z1 of its first tile, then of the next tile
//             taken from a global atomic counter, and so on.
//   producer  one warp (lane 0) owns the stream: it takes tiles, waits until
//             the consumers release a stage ("empty" mbarrier), and issues that
//             plane's loads onto the stage's "full" mbarrier -- five
//             cp.async.bulk.tensor loads, because each tensor map covers all
//             components and both time buffers of a field group (5D maps:
//             x, y, z, component, buffer). Tile changes, counter atomics and
//             tensor-map fences never stall the consumers.
//   stage     one z plane of: the H^n box [x0-4, x0+TX+4) x [y0-1, y0+TY+1)
//             (3 components), the E^n box [x0-4, x0+TX) x [y0-1, y0+TY), the
//             16-bit material-index box [x0-8, x0+TX) x [y0-1, y0+TY), and the
//             split fields of PML cells: MODE_WINDOW stages the six E and six
//             H split components over a 16-column window [wx0, wx0+16) (the
//             x-PML slab inside an ordinary tile), MODE_FULL over the whole E
//             box / owned box (the y- and z-PML slabs). Every x start is a
//             multiple of 16 bytes; boxes reaching outside the grid fill with
//             zeros, and a zero material index selects the all-zero coefficient
//             row, so the halo and the grid edges need no bounds checks in the
//             update. Split cells outside any staged window (soft-source cells)
//             read their splits with global loads.
//   consumers E phase: one float4 group (4 cells along x) per thread over the
//             halo-extended tile; named barrier; H phase: one group per owned
//             float4. Both read neighbours from shared memory only. A thread
//             keeps the coefficient row of its group while the material index
//             does not change from plane to plane.
//   waits     every mbarrier wait is bounded; on expiry the block records an
//             error code, the producer drains its loads (bounded), and all
//             warps return.
#pragma once

#include "fdtd_kernels.cuh"
#include "tma.cuh"

namespace rfn {

constexpr uint32_t kWaitLimit = 1u << 20;  // sleeping polls of one mbarrier (each <= 2 us) before giving up
constexpr int kErrTmaTimeout = 1;
constexpr int kSplitWin = 16;              // split window width (MODE_WINDOW)
constexpr int MODE_WINDOW = 0, MODE_FULL = 1;
constexpr int kBarCompute = 1;             // named barrier of the consumer warps

// Tensor maps of one simulation for one tile shape (5D: x, y, z, component, buffer).
struct TmaMaps {
  CUtensorMap E, H, ids, Es, Hs;
};

// One tile. wx0 < 0: no split window.
struct TileDesc {
  int sim, x0, y0, z0, z1, x1, y1, wx0;
};

template <int TX, int TY, int MODE>
struct TmaGeom {
  static constexpr int HBX = TX + 8, EBX = TX + 4, IBX = TX + 8;
  static constexpr int GX = TX / 4 + 1;                            // E-phase groups per row
  static constexpr int SEW = MODE == MODE_FULL ? EBX : kSplitWin;  // E split box width
  static constexpr int SHW = MODE == MODE_FULL ? TX : kSplitWin;   // H split box width
  static constexpr int HC = (TY + 2) * HBX;                        // floats per H component
  static constexpr int EC = (TY + 1) * EBX;
  static constexpr int SEC = (TY + 1) * SEW;
  static constexpr int SHC = TY * SHW;
  static constexpr int HB = 3 * HC * 4;
  static constexpr int EB = 3 * EC * 4;
  static constexpr int IB = (TY + 1) * IBX * 2;
  static constexpr int SEB = 6 * SEC * 4;
  static constexpr int SHB = 6 * SHC * 4;
  static constexpr int A(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_E = A(HB);
  static constexpr int OFF_I = OFF_E + A(EB);
  static constexpr int OFF_ES = OFF_I + A(IB);
  static constexpr int OFF_HS = OFF_ES + A(SEB);
  static constexpr int STAGE = OFF_HS + A(SHB);
  static constexpr uint32_t MAIN_BYTES = HB + EB + IB;
  static constexpr uint32_t SPLIT_BYTES = SEB + SHB;
  static constexpr int ENEW_PLANE = 3 * EC;  // floats
  static constexpr int ENEW = 2 * ENEW_PLANE * 4;
  static constexpr int EGROUPS = (TY + 1) * GX;
  static constexpr int HGROUPS = TY * (TX / 4);
  static constexpr int CONSUMERS = (EGROUPS + 31) / 32 * 32;
  static constexpr int THREADS = CONSUMERS + 32;  // + the producer warp
};

template <int TX, int TY, int S, int MODE>
constexpr int tma_smem_bytes() {
  using G = TmaGeom<TX, TY, MODE>;
  return S * G::STAGE + G::ENEW + 16 * S;
}

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
// next-cell difference along x: (v[j+1] - v[j]), the last one against `after`
__device__ __forceinline__ float4 dnext4(float4 v, float after) {
  return make_float4(v.y - v.x, v.z - v.y, v.w - v.z, after - v.w);
}
__device__ __forceinline__ float4 upd_e4(float ca, float4 f, float cb1, float4 d1, float cb2, float4 d2) {
  return make_float4(upd_e(ca, f.x, cb1, d1.x, cb2, d2.x), upd_e(ca, f.y, cb1, d1.y, cb2, d2.y),
                     upd_e(ca, f.z, cb1, d1.z, cb2, d2.z), upd_e(ca, f.w, cb1, d1.w, cb2, d2.w));
}
__device__ __forceinline__ float4 h_term4(float b2, float4 e2, float b1, float4 e1) {
  return make_float4(h_term(b2, e2.x, b1, e1.x), h_term(b2, e2.y, b1, e1.y), h_term(b2, e2.z, b1, e1.z),
                     h_term(b2, e2.w, b1, e1.w));
}
__device__ __forceinline__ float4 upd_h4(float da, float4 f, float4 g1, float4 g2) {
  return make_float4(upd_h(da, f.x, g1.x, g2.x), upd_h(da, f.y, g1.y, g2.y), upd_h(da, f.z, g1.z, g2.z),
                     upd_h(da, f.w, g1.w, g2.w));
}
// previous-cell value along x: (v[j-1]), the first one is `before`
__device__ __forceinline__ float4 prev4(float before, float4 v) { return make_float4(before, v.x, v.y, v.z); }
__device__ __forceinline__ float f4(const float4& v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }
__device__ __forceinline__ void set4(float4& v, int j, float a) {
  if (j == 0) v.x = a; else if (j == 1) v.y = a; else if (j == 2) v.z = a; else v.w = a;
}

// Soft sources of a cell (solver.cu:459-488, 515-541): s1 += v; s2 += v.
__device__ __forceinline__ void inject(const SimDev& Sd, const float4& r7, uint32_t flags, int n, bool e_side,
                                       float (&s)[6]) {
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
          s[2 * k] = __fadd_rn(s[2 * k], v);
          s[2 * k + 1] = __fadd_rn(s[2 * k + 1], v);
        }
    }
  }
}

__device__ __forceinline__ TileDesc load_tile(const TileDesc* tiles, int i) {
  const int4* p = reinterpret_cast<const int4*>(tiles + i);
  const int4 a = __ldg(p), b = __ldg(p + 1);
  return TileDesc{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

template <int TX, int TY, int S, int MODE>
__global__ void __launch_bounds__(TmaGeom<TX, TY, MODE>::THREADS)
fdtd_step_tma_kernel(const SimDev* __restrict__ sims, const TileDesc* __restrict__ tiles, int n_tiles, int n,
                     unsigned* __restrict__ counter, unsigned base, int* __restrict__ err) {
  using G = TmaGeom<TX, TY, MODE>;
  // S <= 7 keeps the producer at most three tiles ahead (s_tq ring of 4);
  // S >= 3: the current plane, the next one and one in flight.
  static_assert(S >= 3 && S <= 7, "stage count out of range");
  extern __shared__ __align__(128) unsigned char smem[];
  float* enew = reinterpret_cast<float*>(smem + S * G::STAGE);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + G::ENEW);
  uint64_t* empty = full + S;
  __shared__ int s_tq[4];  // tile indices handed from the producer to the consumers
  const int tid = threadIdx.x;
  const int cur = n & 1, nxt = cur ^ 1;
  constexpr int NC = G::CONSUMERS;
  constexpr int NCW = NC / 32;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // =================================================================== producer
  if (tid >= NC) {
    if (tid != NC) return;
    uint32_t q = 0;
    int k = 0;
    const TmaMaps* cur_maps = nullptr;
    bool failed = false;
    for (;;) {
      const unsigned v = atomicAdd(counter, 1u) - base;
      const int t = v < unsigned(n_tiles) ? int(v) : -1;
      TileDesc td{};
      int npl = 1;
      bool split = false;
      const TmaMaps* maps = nullptr;
      if (t >= 0) {
        td = load_tile(tiles, t);
        npl = td.z1 - td.z0 + 2;
        maps = sims[td.sim].maps;
        split = MODE == MODE_FULL || td.wx0 >= 0;
        if (maps != cur_maps) {
          tensormap_acquire(&maps->E);
          tensormap_acquire(&maps->H);
          tensormap_acquire(&maps->ids);
          tensormap_acquire(&maps->Es);
          tensormap_acquire(&maps->Hs);
          cur_maps = maps;
        }
      }
      for (int j = 0; j < npl; ++j, ++q) {
        const int s = int(q % S);
        if (q >= uint32_t(S) && !mbar_wait_bounded(&empty[s], ((q / S) + 1) & 1u, kWaitLimit)) {
          failed = true;
          break;
        }
        if (j == 0) s_tq[k & 3] = t;
        if (t < 0) {  // end of the stream: complete the phase without data
          mbar_arrive(&full[s]);
          ++q;
          break;
        }
        unsigned char* b = smem + s * G::STAGE;
        const int zp = td.z0 - 1 + j;
        fence_proxy_async();
        mbar_arrive_expect_tx(&full[s], G::MAIN_BYTES + (split ? G::SPLIT_BYTES : 0u));
        tma_load_5d(b, &maps->H, td.x0 - 4, td.y0 - 1, zp, 0, cur, &full[s]);
        tma_load_5d(b + G::OFF_E, &maps->E, td.x0 - 4, td.y0 - 1, zp, 0, cur, &full[s]);
        tma_load_3d(b + G::OFF_I, &maps->ids, td.x0 - 8, td.y0 - 1, zp, &full[s]);
        if (split) {
          const int ex = MODE == MODE_FULL ? td.x0 - 4 : td.wx0;
          const int hx = MODE == MODE_FULL ? td.x0 : td.wx0;
          tma_load_5d(b + G::OFF_ES, &maps->Es, ex, td.y0 - 1, zp, 0, cur, &full[s]);
          tma_load_5d(b + G::OFF_HS, &maps->Hs, hx, td.y0, zp, 0, cur, &full[s]);
        }
      }
      if (failed || t < 0) break;
      ++k;
    }
    if (failed) {
      atomicExch(err, kErrTmaTimeout);
      // drain the loads still in flight (bounded)
      for (uint32_t r = q > uint32_t(S) ? q - S : 0; r < q; ++r)
        mbar_wait_bounded(&full[r % S], (r / S) & 1u, kWaitLimit);
    }
    return;
  }

  // ================================================================== consumers
  const int lane = tid & 31;
  uint32_t q0 = 0;  // sequence number of the current tile's first plane
  for (int k = 0;; ++k) {
    bool ok = mbar_wait_bounded(&full[q0 % S], (q0 / S) & 1u, kWaitLimit);
    if (named_bar_or(kBarCompute, NC, !ok)) {
      if (tid == 0) atomicExch(err, kErrTmaTimeout);
      return;
    }
    const int ti = s_tq[k & 3];
    if (ti < 0) break;
    const TileDesc td = load_tile(tiles, ti);
    const SimDev& Sd = sims[td.sim];
    const int x0 = td.x0, y0 = td.y0, z0 = td.z0, tx1 = td.x1, ty1 = td.y1, wx0 = td.wx0;
    const int plane = Sd.plane, pitch = Sd.pitch;
    const float4* __restrict__ rows = Sd.rows;
    float* const eo0 = Sd.E[nxt][0];
    float* const eo1 = Sd.E[nxt][1];
    float* const eo2 = Sd.E[nxt][2];
    float* const ho0 = Sd.H[nxt][0];
    float* const ho1 = Sd.H[nxt][1];
    float* const ho2 = Sd.H[nxt][2];
    const int npl = td.z1 - z0 + 2;

    // coefficient rows kept across planes (E part for the E phase, H part for the H phase)
    int e_id = -1, h_id = -1;
    float4 ra = {}, rb = {}, rd = {}, re7 = {};
    float4 hp = {}, hq = {}, hu = {}, hv = {}, h7 = {};

    for (int i = 0; i + 1 < npl; ++i) {
      const int z = z0 - 1 + i;
      const uint32_t q = q0 + i;
      if (i > 0) {
        ok = mbar_wait_bounded(&full[q % S], (q / S) & 1u, kWaitLimit);
      }
      ok = ok && mbar_wait_bounded(&full[(q + 1) % S], ((q + 1) / S) & 1u, kWaitLimit);
      // the barrier also separates the previous H phase from this E phase (enew reuse)
      if (named_bar_or(kBarCompute, NC, !ok)) {
        if (tid == 0) atomicExch(err, kErrTmaTimeout);
        return;
      }
      const unsigned char* st = smem + int(q % S) * G::STAGE;
      const unsigned char* st1 = smem + int((q + 1) % S) * G::STAGE;
      const float* sH = reinterpret_cast<const float*>(st);
      const float* sE = reinterpret_cast<const float*>(st + G::OFF_E);
      const uint16_t* sId = reinterpret_cast<const uint16_t*>(st + G::OFF_I);
      const float* sEs = reinterpret_cast<const float*>(st + G::OFF_ES);
      const float* sHs = reinterpret_cast<const float*>(st + G::OFF_HS);
      const float* nH = reinterpret_cast<const float*>(st1);
      float* en = enew + (i & 1) * G::ENEW_PLANE;
      const float* ep = enew + ((i - 1) & 1) * G::ENEW_PLANE;
      constexpr int HC = G::HC, EC = G::EC;

      // ------------------------------------------------------------ E phase
      if (tid < G::EGROUPS) {
        const int er = tid / G::GX, cg = tid % G::GX;
        const int hb = er * G::HBX + 4 * cg;
        const float4 hx_c = lds4(sH + hb), hy_c = lds4(sH + HC + hb), hz_c = lds4(sH + 2 * HC + hb);
        const float hy_x4 = sH[HC + hb + 4], hz_x4 = sH[2 * HC + hb + 4];
        const float4 hz_yn = lds4(sH + 2 * HC + hb + G::HBX), hx_yn = lds4(sH + hb + G::HBX);
        const float4 hx_zn = lds4(nH + hb), hy_zn = lds4(nH + HC + hb);
        const int eb = er * G::EBX + 4 * cg;
        const float4 ex_o = lds4(sE + eb), ey_o = lds4(sE + EC + eb), ez_o = lds4(sE + 2 * EC + eb);
        const uint2 idw = *reinterpret_cast<const uint2*>(sId + er * G::IBX + 4 * cg + 4);
        const int id4[4] = {int(idw.x & 0xffffu), int(idw.x >> 16), int(idw.y & 0xffffu), int(idw.y >> 16)};
        const int xg = x0 - 4 + 4 * cg, r = y0 - 1 + er;
        const bool own_row = er >= 1 && cg >= 1 && r < ty1 && z >= z0;
        const bool uniform = id4[0] == id4[1] && id4[0] == id4[2] && id4[0] == id4[3];
        if (uniform) {
          if (id4[0] != e_id) {
            const float4* row = rows + 8 * id4[0];
            ra = __ldg(row); rb = __ldg(row + 1); rd = __ldg(row + 2); re7 = __ldg(row + 7);
            e_id = id4[0];
          }
        } else {
          e_id = -1;
        }
        float4 exn, eyn, ezn;
        if (uniform && !(__float_as_uint(re7.z) & kESplit)) {
          // common case: one coefficient row, no split storage -- branch-free float4 update
          exn = upd_e4(ra.x, ex_o, ra.y, sub4(hz_yn, hz_c), ra.w, sub4(hy_zn, hy_c));
          eyn = upd_e4(rb.x, ey_o, rb.y, sub4(hx_zn, hx_c), rb.w, dnext4(hz_c, hz_x4));
          ezn = upd_e4(rd.x, ez_o, rd.y, dnext4(hy_c, hy_x4), rd.w, sub4(hx_yn, hx_c));
        } else
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
          float4 a = ra, b = rb, d = rd, r7 = re7;
          if (!uniform) {
            const float4* row = rows + 8 * id4[j];
            a = __ldg(row); b = __ldg(row + 1); d = __ldg(row + 2); r7 = __ldg(row + 7);
          }
          const uint32_t flags = __float_as_uint(r7.z);
          const float hzj = f4(hz_c, j), hyj = f4(hy_c, j), hxj = f4(hx_c, j);
          const float dhz_y = f4(hz_yn, j) - hzj, dhy_z = f4(hy_zn, j) - hyj;
          const float dhx_z = f4(hx_zn, j) - hxj, dhz_x = (j < 3 ? f4(hz_c, j + 1) : hz_x4) - hzj;
          const float dhy_x = (j < 3 ? f4(hy_c, j + 1) : hy_x4) - hyj, dhx_y = f4(hx_yn, j) - hxj;
          float ex, ey, ez;
          if (!(flags & kESplit)) {
            ex = upd_e(a.x, f4(ex_o, j), a.y, dhz_y, a.w, dhy_z);
            ey = upd_e(b.x, f4(ey_o, j), b.y, dhx_z, b.w, dhz_x);
            ez = upd_e(d.x, f4(ez_o, j), d.y, dhy_x, d.w, dhx_y);
          } else {
            const int xc = xg + j;
            const int idx = z * plane + r * pitch + xc;
            float sp[6];
            int so = -1;
            if (MODE == MODE_FULL) {
              so = eb + j;
            } else if (wx0 >= 0 && xc >= wx0 && xc < wx0 + kSplitWin) {
              so = er * kSplitWin + (xc - wx0);
            }
            if (so >= 0) {
#pragma unroll
              for (int c = 0; c < 6; ++c) sp[c] = sEs[c * G::SEC + so];
            } else {
#pragma unroll
              for (int c = 0; c < 6; ++c) sp[c] = __ldg(Sd.Es[cur][c] + idx);
            }
            sp[0] = upd_e_split(a.x, sp[0], a.y, dhz_y);
            sp[1] = upd_e_split(a.z, sp[1], a.w, dhy_z);
            sp[2] = upd_e_split(b.x, sp[2], b.y, dhx_z);
            sp[3] = upd_e_split(b.z, sp[3], b.w, dhz_x);
            sp[4] = upd_e_split(d.x, sp[4], d.y, dhy_x);
            sp[5] = upd_e_split(d.z, sp[5], d.w, dhx_y);
            if (flags >> 16) inject(Sd, r7, flags, n, true, sp);
            ex = __fadd_rn(sp[0], sp[1]);
            ey = __fadd_rn(sp[2], sp[3]);
            ez = __fadd_rn(sp[4], sp[5]);
            if (own_row && xc < tx1) {
              float* const* Eo = Sd.Es[nxt];
#pragma unroll
              for (int c = 0; c < 6; ++c) Eo[c][idx] = sp[c];
            }
          }
          set4(exn, j, ex);
          set4(eyn, j, ey);
          set4(ezn, j, ez);
        }
        *reinterpret_cast<float4*>(en + eb) = exn;
        *reinterpret_cast<float4*>(en + EC + eb) = eyn;
        *reinterpret_cast<float4*>(en + 2 * EC + eb) = ezn;
      }
      named_bar_sync(kBarCompute, NC);

      // ------------------------------------------------------------ H phase
      if (z >= z0 && tid < G::HGROUPS) {
        const int hr = tid / (TX / 4), hc = tid % (TX / 4);
        const int r = y0 + hr, xg = x0 + 4 * hc;
        if (r < ty1 && xg < tx1) {
          const int eo = (hr + 1) * G::EBX + 4 + 4 * hc;
          const float4 ex = lds4(en + eo), ey = lds4(en + EC + eo), ez = lds4(en + 2 * EC + eo);
          const float ey_xm0 = en[EC + eo - 1], ez_xm0 = en[2 * EC + eo - 1];
          const float4 ex_ym = lds4(en + eo - G::EBX), ez_ym = lds4(en + 2 * EC + eo - G::EBX);
          const float4 ex_zm = lds4(ep + eo), ey_zm = lds4(ep + EC + eo);
          const int ho = (hr + 1) * G::HBX + 4 + 4 * hc;
          const float4 hx_o = lds4(sH + ho), hy_o = lds4(sH + HC + ho), hz_o = lds4(sH + 2 * HC + ho);
          const uint2 idw = *reinterpret_cast<const uint2*>(sId + (hr + 1) * G::IBX + 8 + 4 * hc);
          const int id4[4] = {int(idw.x & 0xffffu), int(idw.x >> 16), int(idw.y & 0xffffu), int(idw.y >> 16)};
          const bool uniform = id4[0] == id4[1] && id4[0] == id4[2] && id4[0] == id4[3];
          const int idx0 = z * plane + r * pitch + xg;
          if (uniform) {
            if (id4[0] != h_id) {
              const float4* row = rows + 8 * id4[0];
              hp = __ldg(row + 3); hq = __ldg(row + 4); hu = __ldg(row + 5); hv = __ldg(row + 6); h7 = __ldg(row + 7);
              h_id = id4[0];
            }
          } else {
            h_id = -1;
          }
          const uint32_t uflags = __float_as_uint(h7.z);
          if (uniform && xg + 3 < tx1 && !(uflags & (kESplit | kHSplit)) && (uflags >> 16) == 0) {
            // common case: one coefficient row, no split storage, no probe -- float4 update and stores
            const float4 gxy = h_term4(hp.z, ez, hp.y, ez_ym);
            const float4 gxz = h_term4(hq.y, ey, hq.x, ey_zm);
            const float4 gyz = h_term4(hu.x, ex, hq.w, ex_zm);
            const float4 gyx = h_term4(hu.w, ez, hu.z, prev4(ez_xm0, ez));
            const float4 gzx = h_term4(hv.z, ey, hv.y, prev4(ey_xm0, ey));
            const float4 gzy = h_term4(h7.y, ex, h7.x, ex_ym);
            *reinterpret_cast<float4*>(eo0 + idx0) = ex;
            *reinterpret_cast<float4*>(eo1 + idx0) = ey;
            *reinterpret_cast<float4*>(eo2 + idx0) = ez;
            *reinterpret_cast<float4*>(ho0 + idx0) = upd_h4(hp.x, hx_o, gxy, gxz);
            *reinterpret_cast<float4*>(ho1 + idx0) = upd_h4(hq.z, hy_o, gyz, gyx);
            *reinterpret_cast<float4*>(ho2 + idx0) = upd_h4(hv.x, hz_o, gzx, gzy);
          } else {
          float4 hxn, hyn, hzn;
          uint32_t esplit_mask = 0;
#pragma unroll 1
          for (int j = 0; j < 4; ++j) {
            float4 p = hp, qv = hq, u = hu, v6 = hv, r7 = h7;
            if (!uniform) {
              const float4* row = rows + 8 * id4[j];
              p = __ldg(row + 3); qv = __ldg(row + 4); u = __ldg(row + 5); v6 = __ldg(row + 6); r7 = __ldg(row + 7);
            }
            const uint32_t flags = __float_as_uint(r7.z);
            if (flags & kESplit) esplit_mask |= 1u << j;
            const float exj = f4(ex, j), eyj = f4(ey, j), ezj = f4(ez, j);
            const float ey_xm = j == 0 ? ey_xm0 : f4(ey, j - 1);
            const float ez_xm = j == 0 ? ez_xm0 : f4(ez, j - 1);
            const float gxy = h_term(p.z, ezj, p.y, f4(ez_ym, j));
            const float gxz = h_term(qv.y, eyj, qv.x, f4(ey_zm, j));
            const float gyz = h_term(u.x, exj, qv.w, f4(ex_zm, j));
            const float gyx = h_term(u.w, ezj, u.z, ez_xm);
            const float gzx = h_term(v6.z, eyj, v6.y, ey_xm);
            const float gzy = h_term(r7.y, exj, r7.x, f4(ex_ym, j));
            float hx, hy, hz;
            if (!(flags & kHSplit)) {
              hx = upd_h(p.x, f4(hx_o, j), gxy, gxz);
              hy = upd_h(qv.z, f4(hy_o, j), gyz, gyx);
              hz = upd_h(v6.x, f4(hz_o, j), gzx, gzy);
            } else {
              const int xc = xg + j;
              const int idx = idx0 + j;
              float sp[6];
              int so = -1;
              if (MODE == MODE_FULL) {
                so = hr * TX + 4 * hc + j;
              } else if (wx0 >= 0 && xc >= wx0 && xc < wx0 + kSplitWin) {
                so = hr * kSplitWin + (xc - wx0);
              }
              if (so >= 0) {
#pragma unroll
                for (int c = 0; c < 6; ++c) sp[c] = sHs[c * G::SHC + so];
              } else {
#pragma unroll
                for (int c = 0; c < 6; ++c) sp[c] = __ldg(Sd.Hs[cur][c] + idx);
              }
              sp[0] = upd_h_split(p.x, sp[0], gxy);
              sp[1] = upd_h_split(p.w, sp[1], gxz);
              sp[2] = upd_h_split(qv.z, sp[2], gyz);
              sp[3] = upd_h_split(u.y, sp[3], gyx);
              sp[4] = upd_h_split(v6.x, sp[4], gzx);
              sp[5] = upd_h_split(v6.w, sp[5], gzy);
              if (flags >> 16) inject(Sd, r7, flags, n, false, sp);
              hx = __fadd_rn(sp[0], sp[1]);
              hy = __fadd_rn(sp[2], sp[3]);
              hz = __fadd_rn(sp[4], sp[5]);
              if (xc < tx1) {
                float* const* Ho = Sd.Hs[nxt];
#pragma unroll
                for (int c = 0; c < 6; ++c) Ho[c][idx] = sp[c];
              }
            }
            set4(hxn, j, hx);
            set4(hyn, j, hy);
            set4(hzn, j, hz);
            const int np = int(flags >> 16);
            if (np && xg + j < tx1) {  // record probes (solver.cu:467, 521)
              const int first = __float_as_int(r7.w);
              for (int e = 0; e < np; ++e) {
                const int2 pe = __ldg(Sd.cell_probes + first + e);
                const float val = pe.y == 0 ? exj : pe.y == 1 ? eyj : pe.y == 2 ? ezj
                                : pe.y == 3 ? hx : pe.y == 4 ? hy : hz;
                Sd.rec[(size_t)pe.x * Sd.nt + n] = val;
              }
            }
          }
          if (xg + 3 < tx1 && esplit_mask == 0) {
            *reinterpret_cast<float4*>(eo0 + idx0) = ex;
            *reinterpret_cast<float4*>(eo1 + idx0) = ey;
            *reinterpret_cast<float4*>(eo2 + idx0) = ez;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (xg + j < tx1 && !(esplit_mask & (1u << j))) {
                eo0[idx0 + j] = f4(ex, j);
                eo1[idx0 + j] = f4(ey, j);
                eo2[idx0 + j] = f4(ez, j);
              }
          }
          if (xg + 3 < tx1) {
            *reinterpret_cast<float4*>(ho0 + idx0) = hxn;
            *reinterpret_cast<float4*>(ho1 + idx0) = hyn;
            *reinterpret_cast<float4*>(ho2 + idx0) = hzn;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (xg + j < tx1) {
                ho0[idx0 + j] = f4(hxn, j);
                ho1[idx0 + j] = f4(hyn, j);
                ho2[idx0 + j] = f4(hzn, j);
              }
          }
          }
        }
      }
      // plane q is no longer read by anyone
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[q % S]);
    }
    // the tile's last plane was read only as the look-ahead of its last iteration
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[(q0 + npl - 1) % S]);
    q0 += uint32_t(npl);
  }
}

}  // namespace rfn
