// Reverse step of the discrete adjoint in the marching kernel's form: the
// adjoint state of every z plane is staged in shared memory by TMA, persistent
// blocks take tiles from an atomic counter, each consumer warp walks TY rows
// of its tile per plane.
//
// The arithmetic is adj_step_kernel's (fdtd_adjoint.cuh), term for term:
//   E part   mu = lamE + (own Db2 lamH) - (Db1 lamH of the +1 neighbours),
//            lamE' = Ca mu, ad = Cb mu (the adjoints of the H differences);
//   H part   lamH' = Da lamH + (ad of the -1 neighbours - own ad);
//   records  the adjoints of this cell's records of step n-1 are added to
//            lamE' / lamH' as they are stored;
//   gradient mu times the forward history of the box cells, in FP64.
// The +1 neighbours' Db1 lamH products need the neighbours' coefficient rows:
// x+1 comes from the lane on the right (which computes its own products; lane
// 31 is only that provider, so a tile owns 30 columns), y+1 from the next row
// of the index box and z+1 from the next plane's, each a two-value lookup of
// the neighbour's row (skipped when it is the cell's own row). The -1
// neighbours' ad come by warp shuffle (x), from the row below in registers (y)
// and from the plane below, kept per row (z). Lane 0 and each warp's first row
// are the -1 halo whose ad the H part needs.
//
// Shared memory per plane: lamH (3 totals, rows y0-1 .. y0+ROWS), lamE (rows
// y0-1 .. y0+ROWS-1), the material index (rows y0-1 .. y0+ROWS), and, for the
// planes the host flagged as holding split cells, the six E and six H halves
// of the same boxes. The last plane of a tile (z1) is the look-ahead of the
// z+1 products: lamH, index and H halves only. Plane and split slots are
// pooled as in the forward marching kernel.
#pragma once

#include "fdtd_adjoint.cuh"
#include "fdtd_step_march.cuh"

namespace rfn {

// Tensor maps of one simulation's adjoint buffers.
struct AdjMaps {
  CUtensorMap lamE, lamH, ids, lamEs, lamHs;
};

constexpr int kAdjMarchOwnX = 30;  // owned columns: lane 0 is the -1 halo, lane 31 the +1 provider

template <int XW, int TY>
struct AdjMarchGeom {
  static constexpr int ROWS = XW * TY;
  static constexpr int W = 36, IW = 40;                 // box widths: columns x0-1 .. x0+30 from a 16-byte start
  static constexpr int HR = ROWS + 2, ER = ROWS + 1, IR = ROWS + 2;
  static constexpr int HC = HR * W, EC = ER * W;        // floats per component / half
  static constexpr int HB = 3 * HC * 4, EB = 3 * EC * 4, IB = IR * IW * 2;
  static constexpr int SEB = 6 * EC * 4, SHB = 6 * HC * 4;
  static constexpr int A(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OFF_E = A(HB), OFF_I = OFF_E + A(EB);
  static constexpr uint32_t MAIN = OFF_I + A(IB);
  static constexpr uint32_t SPLIT = A(SHB) + A(SEB);    // H halves first (the look-ahead plane has only those)
  static constexpr uint32_t SPLIT_E = A(SHB);
  static constexpr int THREADS = 32 * (XW + 1);
};

template <int XW, int TY>
__global__ void __launch_bounds__(AdjMarchGeom<XW, TY>::THREADS, 1)
adj_march_kernel(const AdjSim* __restrict__ sims, const StreamTile* __restrict__ tiles, int n_tiles, int n,
                 int hist_n0, unsigned* __restrict__ counter, unsigned base, int* __restrict__ err, int n_main,
                 int n_split, uint32_t wait_limit) {
  using G = AdjMarchGeom<XW, TY>;
  constexpr int NC = 32 * XW;
  const int P = n_main;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) uint64_t full[kMarchSlots], empty[kMarchSlots];
  __shared__ uint32_t s_soff[kMarchSlots];
  __shared__ uint32_t s_suser[kMarchSplitSlots];
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
    uint32_t q = 0, rel = 0, ns = 0;
    int k = 0;
    const AdjMaps* cur_maps = nullptr;
    bool failed = false;
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
      uint64_t mask = 0;
      const AdjMaps* maps = nullptr;
      if (t >= 0) {
        td = load_stream_tile(tiles, t);
        nload = td.z1 - td.z0 + 2;  // planes z0-1 .. z1
        mask = uint64_t(td.split_lo) | (uint64_t(td.split_hi) << 32);
        maps = reinterpret_cast<const AdjMaps*>(sims[td.sim].maps);
        if (maps != cur_maps) {
          tensormap_acquire(&maps->lamE);
          tensormap_acquire(&maps->lamH);
          tensormap_acquire(&maps->ids);
          tensormap_acquire(&maps->lamEs);
          tensormap_acquire(&maps->lamHs);
          cur_maps = maps;
        }
      }
      const int xs = (td.x0 - 1) & ~3, xi = (td.x0 - 1) & ~7;
      for (int j = 0; j < nload; ++j) {
        const bool last = t >= 0 && j == nload - 1;
        const bool split = t >= 0 && ((mask >> j) & 1u);
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
        if (t < 0) {
          mbar_arrive(&full[slot]);
          ++q;
          break;
        }
        unsigned char* b = ring + uint32_t(slot) * G::MAIN;
        unsigned char* sb = ring + soff;
        uint64_t* fb = &full[slot];
        const int zp = td.z0 - 1 + j;
        fence_proxy_async();
        mbar_arrive_expect_tx(fb, uint32_t(G::HB + G::IB) + (last ? 0u : uint32_t(G::EB)) +
                                      (split ? uint32_t(G::SHB) + (last ? 0u : uint32_t(G::SEB)) : 0u));
        // the maps' fourth coordinate is 6 * buffer + component (totals) or 12 * buffer + half
        tma_load_4d(b, &maps->lamH, xs, td.y0 - 1, zp, 6 * cur + 3, fb);
        tma_load_3d(b + G::OFF_I, &maps->ids, xi, td.y0 - 1, zp, fb);
        if (!last) tma_load_4d(b + G::OFF_E, &maps->lamE, xs, td.y0 - 1, zp, 6 * cur, fb);
        if (split) {
          tma_load_4d(sb, &maps->lamHs, xs, td.y0 - 1, zp, 12 * cur + 6, fb);
          if (!last) tma_load_4d(sb + G::SPLIT_E, &maps->lamEs, xs, td.y0 - 1, zp, 12 * cur, fb);
        }
        ++q;
      }
      if (failed || t < 0) break;
      ++k;
    }
    if (failed) {
      atomicExch(err, kErrWaitExpired);
      for (uint32_t r = rel; r < q; ++r) mbar_wait_bounded(&full[r % P], (r / P) & 1u, wait_limit);
    }
    return;
  }

  // ================================================================== consumers
  const int lane = tid & 31, w = tid >> 5;
  const float4* __restrict__ rows = nullptr;
  int rid = -1;
  float4 ra = {}, rb = {}, rd = {}, rp = {}, rq = {}, ru = {}, rv = {}, r7 = {};
  uint32_t fl = 0;
  uint32_t q = 0;
  for (int k = 0;; ++k) {
    if (!mbar_wait_bounded(&full[q % P], (q / P) & 1u, wait_limit)) {
      if (lane == 0) atomicExch(err, kErrWaitExpired);
      return;
    }
    const int ti = s_tq[k & 3];
    if (ti < 0) break;
    const StreamTile td = load_stream_tile(tiles, ti);
    const AdjSim& A = sims[td.sim];
    if (A.rows != rows) {
      rows = A.rows;
      rid = -1;
    }
    const int x0 = td.x0, y0 = td.y0, z0 = td.z0;
    const int c = x0 - 1 + lane;
    const int oh = (x0 - 1) - ((x0 - 1) & ~3), oi = (x0 - 1) - ((x0 - 1) & ~7);
    const bool own_x = lane >= 1 && lane <= kAdjMarchOwnX && c < A.nx;
    const int ny = A.ny, plane = A.plane, pitch = A.pitch;
    const int64_t N = A.N;
    float* __restrict__ wE = A.lam + nxt * 6 * N;   // E totals, then H totals (3 N further)
    float* __restrict__ wEs = A.lams + nxt * 12 * N; // E halves, then H halves (6 N further)
    const int npl = td.z1 - z0 + 1;
    const uint64_t smask = uint64_t(td.split_lo) | (uint64_t(td.split_hi) << 32);
    const int br0 = w * TY;
    int idx0 = (z0 - 1) * plane + (y0 - 1 + br0) * pitch + c;
    const int col = oh + lane, icol = oi + lane;
    float a1p[TY], a2p[TY];  // ad[1], ad[2] of the plane below, per owned row

    auto load_row = [&](int id) {
      if (id != rid) {
        const float4* row = rows + 8 * id;
        ra = __ldg(row); rb = __ldg(row + 1); rd = __ldg(row + 2); rp = __ldg(row + 3);
        rq = __ldg(row + 4); ru = __ldg(row + 5); rv = __ldg(row + 6); r7 = __ldg(row + 7);
        fl = __float_as_uint(r7.z);
        rid = id;
      }
    };

#pragma unroll
    for (int j = 0; j < TY; ++j) a1p[j] = a2p[j] = 0.f;
    bool ok = true;
    for (int i = 0; i < npl && ok; ++i) {
      const uint32_t qn = q + 1;
      if (!mbar_wait_bounded(&full[qn % P], (qn / P) & 1u, wait_limit)) {
        if (lane == 0) atomicExch(err, kErrWaitExpired);
        return;
      }
      const unsigned char* st = ring + (q % P) * G::MAIN;
      const float* sH = reinterpret_cast<const float*>(st);
      const float* sE = reinterpret_cast<const float*>(st + G::OFF_E);
      const uint16_t* sI = reinterpret_cast<const uint16_t*>(st + G::OFF_I);
      const unsigned char* ss = ring + s_soff[q % P];
      const float* sHs = reinterpret_cast<const float*>(ss);
      const float* sEs = reinterpret_cast<const float*>(ss + G::SPLIT_E);
      const unsigned char* nst = ring + (qn % P) * G::MAIN;
      const float* nH = reinterpret_cast<const float*>(nst);
      const uint16_t* nI = reinterpret_cast<const uint16_t*>(nst + G::OFF_I);
      const float* nHs = reinterpret_cast<const float*>(ring + s_soff[qn % P]);
      const bool split_here = (smask >> i) & 1u, split_next = (smask >> (i + 1)) & 1u;
      const bool hphase = i > 0;
      const int z = z0 - 1 + i;
      constexpr int HC = G::HC, EC = G::EC, W = G::W, IW = G::IW;

      // lamH halves of the cell at box row br of a plane (totals duplicated when unsplit)
      auto halves = [&](const float* tH, const float* tHs, bool sp_plane, int br, uint32_t f, float (&h)[6]) {
        const int b = br * W + col;
        if (sp_plane && (f & kHSplit)) {
#pragma unroll
          for (int s = 0; s < 6; ++s) h[s] = tHs[s * HC + b];
        } else {
          const float hx = tH[b], hy = tH[HC + b], hz = tH[2 * HC + b];
          h[0] = hx; h[1] = hx; h[2] = hy; h[3] = hy; h[4] = hz; h[5] = hz;
        }
      };

      float a0m = 0.f, a5m = 0.f;  // ad[0], ad[5] of the row below
#pragma unroll
      for (int j = 0; j <= TY; ++j) {
        const int br = br0 + j;
        const int id = int(sI[br * IW + icol]);
        load_row(id);
        float h[6];
        halves(sH, sHs, split_here, br, fl, h);
        // Db1 lamH of the +1 neighbours. y+1: the next row of this plane
        float qy_hx, qy_hz;
        {
          const int idy = int(sI[(br + 1) * IW + icol]);
          float b1x = rp.y, b1z = r7.x;
          uint32_t fy = fl;
          if (idy != id) {
            const float4* ry = rows + 8 * idy;
            b1x = __ldg(ry + 3).y;
            const float4 y7 = __ldg(ry + 7);
            b1z = y7.x;
            fy = __float_as_uint(y7.z);
          }
          const int b = (br + 1) * W + col;
          const bool sp = split_here && (fy & kHSplit);
          qy_hx = b1x * (sp ? sHs[0 * HC + b] : sH[b]);           // hx_y half
          qy_hz = b1z * (sp ? sHs[5 * HC + b] : sH[2 * HC + b]);  // hz_y half
        }
        // z+1: the same row of the next plane
        float qz_hx, qz_hy;
        {
          const int idz = int(nI[br * IW + icol]);
          float b1x = rq.x, b1y = rq.w;
          uint32_t fz = fl;
          if (idz != id) {
            const float4* rz = rows + 8 * idz;
            const float4 z4 = __ldg(rz + 4);
            b1x = z4.x;
            b1y = z4.w;
            fz = __float_as_uint(__ldg(rz + 7).z);
          }
          const int b = br * W + col;
          const bool sp = split_next && (fz & kHSplit);
          qz_hx = b1x * (sp ? nHs[1 * HC + b] : nH[b]);           // hx_z half
          qz_hy = b1y * (sp ? nHs[2 * HC + b] : nH[HC + b]);      // hy_z half
        }
        // x+1: the lane on the right
        const float qx_hy = __shfl_down_sync(0xffffffffu, ru.z * h[3], 1);
        const float qx_hz = __shfl_down_sync(0xffffffffu, rv.y * h[4], 1);

        // ---- E part
        const float aEx = (ru.x * h[2] - qz_hy) + (r7.y * h[5] - qy_hz);
        const float aEy = (rq.y * h[1] - qz_hx) + (rv.z * h[4] - qx_hz);
        const float aEz = (rp.z * h[0] - qy_hx) + (ru.w * h[3] - qx_hy);
        float mu[6], lE[6], ad[6];
        const bool esplit = fl & kESplit;
        {
          const int b = br * W + col;
          if (!esplit || !split_here) {
            const float mx = sE[b] + aEx, my = sE[EC + b] + aEy, mz = sE[2 * EC + b] + aEz;
            mu[0] = mx; mu[1] = mx; mu[2] = my; mu[3] = my; mu[4] = mz; mu[5] = mz;
            lE[0] = ra.x * mx; lE[1] = rb.x * my; lE[2] = rd.x * mz;
            lE[3] = lE[4] = lE[5] = 0.f;
          } else {
            const float aE[3] = {aEx, aEy, aEz};
            const float ca[6] = {ra.x, ra.z, rb.x, rb.z, rd.x, rd.z};
#pragma unroll
            for (int s = 0; s < 6; ++s) {
              mu[s] = sEs[s * EC + b] + aE[s / 2];
              lE[s] = ca[s] * mu[s];
            }
          }
          const float cb[6] = {ra.y, ra.w, rb.y, rb.w, rd.y, rd.w};
#pragma unroll
          for (int s = 0; s < 6; ++s) ad[s] = cb[s] * mu[s];
        }
        // -1 neighbours' ad along x
        const float a3m = __shfl_up_sync(0xffffffffu, ad[3], 1);
        const float a4m = __shfl_up_sync(0xffffffffu, ad[4], 1);

        // ---- H part, records, stores, gradient (owned cells)
        if (j >= 1 && hphase && own_x && y0 - 1 + br < ny) {
          const int idx = idx0 + j * pitch;
          const float aH[3] = {(a2p[j - 1] - ad[2]) + (a5m - ad[5]), (a1p[j - 1] - ad[1]) + (a4m - ad[4]),
                               (a0m - ad[0]) + (a3m - ad[3])};
          float lh[6];
          const bool hsplit = fl & kHSplit;
          if (!hsplit) {
            lh[0] = rp.x * h[0] + aH[0];
            lh[1] = rq.z * h[2] + aH[1];
            lh[2] = rv.x * h[4] + aH[2];
            lh[3] = lh[4] = lh[5] = 0.f;
          } else {
            const float da[6] = {rp.x, rp.w, rq.z, ru.y, rv.x, rv.w};
#pragma unroll
            for (int s = 0; s < 6; ++s) lh[s] = da[s] * h[s] + aH[s / 2];
          }
          const int np = int(fl >> 16);
          if (np && n >= 1) {
            const int first = __float_as_int(r7.w);
            for (int e = 0; e < np; ++e) {
              const int2 pe = __ldg(A.cell_probes + first + e);
              const float rvv = __ldg(A.radj + size_t(pe.x) * A.nt + (n - 1));
              const bool is_e = pe.y < 3;
              const int cc = is_e ? pe.y : pe.y - 3;
              const bool sp = is_e ? esplit : hsplit;
#pragma unroll
              for (int s = 0; s < 6; ++s)
                if (sp ? (s / 2 == cc) : (s == cc)) {
                  if (is_e) lE[s] += rvv;
                  else lh[s] += rvv;
                }
            }
          }
          if (esplit) {
#pragma unroll
            for (int s = 0; s < 6; ++s) wEs[s * N + idx] = lE[s];
          } else {
            wE[idx] = lE[0]; wE[N + idx] = lE[1]; wE[2 * N + idx] = lE[2];
          }
          if (hsplit) {
#pragma unroll
            for (int s = 0; s < 6; ++s) wEs[(6 + s) * N + idx] = lh[s];
          } else {
            wE[3 * N + idx] = lh[0]; wE[4 * N + idx] = lh[1]; wE[5 * N + idx] = lh[2];
          }
          const int r = y0 - 1 + br;
          if (A.hist && c >= A.bx0 && c < A.bx1 && r >= A.by0 && r < A.by1 && z >= A.bz0 && z < A.bz1) {
            const int bny = A.by1 - A.by0, bnz = A.bz1 - A.bz0;
            const int64_t nb = A.nb;
            const int64_t bi = (int64_t(c - A.bx0) * bny + (r - A.by0)) * bnz + (z - A.bz0);
            const float* hs = A.hist + int64_t(n - hist_n0) * 9 * nb;
#pragma unroll
            for (int s = 0; s < 3; ++s) {
              A.grad[(3 * s + 0) * nb + bi] += double(mu[2 * s]) * double(__ldg(hs + s * nb + bi));
              A.grad[(3 * s + 1) * nb + bi] += double(mu[2 * s]) * double(__ldg(hs + (3 + 2 * s) * nb + bi));
              A.grad[(3 * s + 2) * nb + bi] += double(mu[2 * s + 1]) * double(__ldg(hs + (4 + 2 * s) * nb + bi));
            }
          }
        }
        if (j >= 1) {
          a1p[j - 1] = ad[1];
          a2p[j - 1] = ad[2];
        }
        a0m = ad[0];
        a5m = ad[5];
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[q % P]);
      ++q;
      idx0 += plane;
    }
    (void)ok;
    // the look-ahead plane z1
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q % P]);
    ++q;
  }
}

}  // namespace rfn
