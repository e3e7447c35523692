// Discrete adjoint of the FDTD time step, for gradients of objectives of the
// probe series with respect to the E-update coefficients of a box of cells.
//
// The forward step n (fdtd_step_kernel / fdtd_step_stream_kernel) is linear
// in the state (E, H and the split fields):
//   E split pair  s_{2c}' = C[4c] s_{2c} + C[4c+1] dA_c(H),
//                 s_{2c+1}' = C[4c+2] s_{2c+1} + C[4c+3] dB_c(H)   (+ sources)
//   H split pair  h_s' = Da_s h_s + g_s(E')                        (+ sources)
// with an unsplit cell the special case of equal decays (both halves of the
// pair share Ca / Da and the total is what is stored). The adjoint keeps one
// value per half of every pair for every cell -- for an unsplit cell the two
// halves stay equal, so one formula serves all cells -- and runs the
// transposed recursion backwards in time, one reverse step as three launches:
//   adj_probe_kernel  dJ/d(recorded value) into the pair halves of the probed
//                     component (the records read E^{n+1} and H^{n+1})
//   adj_e_kernel      lamE: add the transposed g terms (own Db2 lamH, the
//                     neighbours' Q), decay by Ca, emit dA / dB adjoints, and
//                     accumulate the gradient of the box cells in FP64
//   adj_h_kernel      lamH: decay by Da and add the transposed differences of
//                     the neighbouring dA / dB adjoints; and Q_s = Db1_s lamH_s,
//                     the part of the next reverse step's H-update transpose
//                     that lands on the neighbouring E cell (the probe kernel
//                     keeps Q in step with what it adds to lamH)
// Index conventions follow the forward kernels: arrays [z][y][pitch].
#pragma once

#include <cstdint>

#include "fdtd_kernels.cuh"

namespace rfn {

struct AdjDev {
  SimDev s;             // geometry, material table, probe list
  float* lamE;          // [6][N] E pair halves (ex_y ex_z ey_z ey_x ez_x ez_y)
  float* lamH;          // [6][N] H pair halves (hx_y hx_z hy_z hy_x hz_x hz_y)
  float* q;             // [6][N] Db1_s lamH_s
  float* ad;            // [6][N] adjoints of dA_x dB_x dA_y dB_y dA_z dB_z
  int64_t N;            // floats per component array
  int bx0, bx1, by0, by1, bz0, bz1;  // gradient box (cells)
  double* grad;         // [3 components][Ca, Cb1, Cb2][box cells]
  const float* hist;    // forward history of this step: [9][box cells] = E_x E_y E_z, dA_x dB_x .. dB_z
};

__device__ __forceinline__ const float4* adj_row(const SimDev& s, int idx) { return s.rows + 8 * s.mat[idx]; }

// The Db1 coefficient of each H split s (slots 13, 16, 19, 22, 25, 28).
__device__ __forceinline__ void adj_db1(const float4* row, float (&b1)[6]) {
  const float4 p = __ldg(row + 3), q = __ldg(row + 4), u = __ldg(row + 5), v = __ldg(row + 6), r7 = __ldg(row + 7);
  b1[0] = p.y; b1[1] = q.x; b1[2] = q.w; b1[3] = u.z; b1[4] = v.y; b1[5] = r7.x;
}

// Field values recorded by probes at step n are E^{n+1} / H^{n+1}: their
// adjoints enter both halves of the probed component's pair.
__global__ void adj_probe_kernel(AdjDev a, const int* __restrict__ probe_idx, const int* __restrict__ probe_field,
                                 const float* __restrict__ radj, int n_probes, int nt, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_probes) return;
  const float r = radj[size_t(p) * nt + n];
  if (r == 0.f) return;
  const int f = probe_field[p];
  const int64_t idx = probe_idx[p];
  float* base = f < 3 ? a.lamE : a.lamH;
  const int c = f < 3 ? f : f - 3;
  atomicAdd(base + (2 * c) * a.N + idx, r);
  atomicAdd(base + (2 * c + 1) * a.N + idx, r);
  if (f >= 3) {
    float b1[6];
    adj_db1(adj_row(a.s, int(idx)), b1);
    atomicAdd(a.q + (2 * c) * a.N + idx, b1[2 * c] * r);
    atomicAdd(a.q + (2 * c + 1) * a.N + idx, b1[2 * c + 1] * r);
  }
}

__global__ void adj_e_kernel(AdjDev a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  const SimDev& s = a.s;
  if (x >= s.nx || y >= s.ny) return;
  const int idx = z * s.plane + y * s.pitch + x;
  const int64_t N = a.N;
  const float4* row = adj_row(s, idx);
  const float4 ra = __ldg(row), rb = __ldg(row + 1), rd = __ldg(row + 2);
  const float4 p = __ldg(row + 3), q = __ldg(row + 4), u = __ldg(row + 5), v = __ldg(row + 6), r7 = __ldg(row + 7);
  // Db2 of the six H splits at this cell (slots 14, 17, 20, 23, 26, 29)
  const float b2[6] = {p.z, q.y, u.x, u.w, v.z, r7.y};
  float ag[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) ag[k] = a.lamH[k * N + idx];
  const bool xn = x + 1 < s.nx, yn = y + 1 < s.ny, zn = z + 1 < s.nz;
  auto qn = [&](int k, bool ok, int off) { return ok ? a.q[k * N + idx + off] : 0.f; };
  // transposed g terms: own Db2 lamH, minus the neighbour's Db1 lamH
  const float aEx = (b2[2] * ag[2] - qn(2, zn, s.plane)) + (b2[5] * ag[5] - qn(5, yn, s.pitch));
  const float aEy = (b2[1] * ag[1] - qn(1, zn, s.plane)) + (b2[4] * ag[4] - qn(4, xn, 1));
  const float aEz = (b2[0] * ag[0] - qn(0, yn, s.pitch)) + (b2[3] * ag[3] - qn(3, xn, 1));
  const float aET[3] = {aEx, aEy, aEz};
  const float ca[6] = {ra.x, ra.z, rb.x, rb.z, rd.x, rd.z};  // decay of each E split
  const float cb[6] = {ra.y, ra.w, rb.y, rb.w, rd.y, rd.w};  // difference coefficient of each E split
  float mu[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    mu[k] = a.lamE[k * N + idx] + aET[k / 2];
    a.lamE[k * N + idx] = ca[k] * mu[k];
    a.ad[k * N + idx] = cb[k] * mu[k];
  }
  if (x >= a.bx0 && x < a.bx1 && y >= a.by0 && y < a.by1 && z >= a.bz0 && z < a.bz1) {
    const int bnx = a.bx1 - a.bx0, bny = a.by1 - a.by0, bnz = a.bz1 - a.bz0;
    const int64_t nb = int64_t(bnx) * bny * bnz;
    const int64_t bi = (int64_t(x - a.bx0) * bny + (y - a.by0)) * bnz + (z - a.bz0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // unsplit design cells: both halves of the pair hold the same adjoint
      const double m = double(mu[2 * c]);
      a.grad[(3 * c + 0) * nb + bi] += m * double(a.hist[c * nb + bi]);
      a.grad[(3 * c + 1) * nb + bi] += m * double(a.hist[(3 + 2 * c) * nb + bi]);
      a.grad[(3 * c + 2) * nb + bi] += double(mu[2 * c + 1]) * double(a.hist[(4 + 2 * c) * nb + bi]);
    }
  }
}

__global__ void adj_h_kernel(AdjDev a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  const SimDev& s = a.s;
  if (x >= s.nx || y >= s.ny) return;
  const int idx = z * s.plane + y * s.pitch + x;
  const int64_t N = a.N;
  auto ad = [&](int k) { return a.ad[k * N + idx]; };
  auto adm = [&](int k, bool ok, int off) { return ok ? a.ad[k * N + idx - off] : 0.f; };
  const bool xm = x > 0, ym = y > 0, zm = z > 0;
  // transposed differences (dA_x = dhz_y, dB_x = dhy_z, dA_y = dhx_z, dB_y = dhz_x, dA_z = dhy_x, dB_z = dhx_y)
  const float aHx = (adm(2, zm, s.plane) - ad(2)) + (adm(5, ym, s.pitch) - ad(5));
  const float aHy = (adm(1, zm, s.plane) - ad(1)) + (adm(4, xm, 1) - ad(4));
  const float aHz = (adm(0, ym, s.pitch) - ad(0)) + (adm(3, xm, 1) - ad(3));
  const float aH[3] = {aHx, aHy, aHz};
  const float4* row = adj_row(s, idx);
  const float4 p = __ldg(row + 3), q = __ldg(row + 4), u = __ldg(row + 5), v = __ldg(row + 6), r7 = __ldg(row + 7);
  const float da[6] = {p.x, p.w, q.z, u.y, v.x, v.w};
  const float b1[6] = {p.y, q.x, q.w, u.z, v.y, r7.x};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float l = da[k] * a.lamH[k * N + idx] + aH[k / 2];
    a.lamH[k * N + idx] = l;
    a.q[k * N + idx] = b1[k] * l;
  }
}

// Forward history of the box at the start of step n: E^n and the H
// differences the E update of step n uses.
__global__ void adj_capture_kernel(AdjDev a, int buf, float* __restrict__ hist) {
  const int bnx = a.bx1 - a.bx0, bny = a.by1 - a.by0, bnz = a.bz1 - a.bz0;
  const int64_t nb = int64_t(bnx) * bny * bnz;
  const SimDev& s = a.s;
  for (int64_t bi = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; bi < nb; bi += int64_t(gridDim.x) * blockDim.x) {
    const int zz = int(bi % bnz), yy = int((bi / bnz) % bny), xx = int(bi / (int64_t(bnz) * bny));
    const int x = a.bx0 + xx, y = a.by0 + yy, z = a.bz0 + zz;
    const int idx = z * s.plane + y * s.pitch + x;
    const float* const* E = s.E[buf];
    const float* const* H = s.H[buf];
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
