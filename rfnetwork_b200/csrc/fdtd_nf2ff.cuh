// Near-field to far-field transform of equivalent surface currents
// (rfnetwork/core/src/postprocess.cpp:130-505, postprocess_nf2ff).
//
// For every frequency f and direction (theta, phi), with r^ = (u, v, w) =
// (sin th cos ph, sin th sin ph, cos th):
//   S_J = sum over the surface cells c of ds_c J_c exp(j beta r^ . r_c), S_M alike
//   N_theta = S_Jx cos th cos ph + S_Jy cos th sin ph - S_Jz sin th,  N_phi = -S_Jx sin ph + S_Jy cos ph
//   L_theta, L_phi from S_M the same way
//   E_theta = (-j beta / 4 pi) (L_phi + eta0 N_theta),  E_phi = (j beta / 4 pi) (L_theta - eta0 N_phi)
// The reference loops frequency x theta x phi x faces on one CPU thread and
// forms the four sums per face; here one thread owns one direction of one
// frequency and the six current moments S_J, S_M are accumulated over all
// cells of all faces at once, the cells streamed through shared memory in
// chunks shared by the block. Phases and products are FP32 (as the
// reference), the running sums FP64 across chunks.
#pragma once

#include <cstdint>

namespace rfn {

constexpr double kEta0 = 376.730313;  // free-space impedance used by the reference (postprocess.cpp:39)
constexpr int kNf2ffThreads = 128;

// One surface cell at one frequency: position (m) and ds J, ds M (complex).
struct Nf2ffCell {
  float4 pos;  // x, y, z, unused
  float4 j01;  // Jx re, im, Jy re, im
  float4 j2m0; // Jz re, im, Mx re, im
  float4 m12;  // My re, im, Mz re, im
};

__global__ void __launch_bounds__(kNf2ffThreads)
nf2ff_kernel(const Nf2ffCell* __restrict__ cells, int n_cells, const float* __restrict__ beta,
             const float* __restrict__ theta, int n_theta, const float* __restrict__ phi, int n_phi,
             float2* __restrict__ out) {
  __shared__ Nf2ffCell s_cells[kNf2ffThreads];
  const int f = blockIdx.y, n_freq = gridDim.y;
  const int a = blockIdx.x * kNf2ffThreads + threadIdx.x;
  const bool live = a < n_theta * n_phi;
  const int th = live ? a / n_phi : 0, ph = live ? a % n_phi : 0;
  float sin_th, cos_th, sin_ph, cos_ph;
  sincosf(theta[th], &sin_th, &cos_th);
  sincosf(phi[ph], &sin_ph, &cos_ph);
  const float u = sin_th * cos_ph, v = sin_th * sin_ph, w = cos_th;
  const float b = beta[f];
  const Nf2ffCell* cf = cells + size_t(f) * n_cells;
  double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // Jx Jy Jz Mx My Mz, (re, im)
  for (int c0 = 0; c0 < n_cells; c0 += kNf2ffThreads) {
    const int nc = min(kNf2ffThreads, n_cells - c0);
    __syncthreads();
    if (threadIdx.x < nc) s_cells[threadIdx.x] = cf[c0 + threadIdx.x];
    __syncthreads();
    float part[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < nc; ++k) {
      const Nf2ffCell& c = s_cells[k];
      float s, co;
      sincosf(b * (u * c.pos.x + v * c.pos.y + w * c.pos.z), &s, &co);
      const float cur[12] = {c.j01.x, c.j01.y, c.j01.z, c.j01.w, c.j2m0.x, c.j2m0.y,
                             c.j2m0.z, c.j2m0.w, c.m12.x, c.m12.y, c.m12.z, c.m12.w};
#pragma unroll
      for (int q = 0; q < 6; ++q) {  // (re + j im) (co + j s)
        part[2 * q] += cur[2 * q] * co - cur[2 * q + 1] * s;
        part[2 * q + 1] += cur[2 * q] * s + cur[2 * q + 1] * co;
      }
    }
#pragma unroll
    for (int q = 0; q < 12; ++q) acc[q] += double(part[q]);
  }
  if (!live) return;
  const double ct = cos_th, st = sin_th, cp = cos_ph, sp = sin_ph;
  // N and L: (re, im)
  const double nt_r = acc[0] * ct * cp + acc[2] * ct * sp - acc[4] * st, nt_i = acc[1] * ct * cp + acc[3] * ct * sp - acc[5] * st;
  const double np_r = -acc[0] * sp + acc[2] * cp, np_i = -acc[1] * sp + acc[3] * cp;
  const double lt_r = acc[6] * ct * cp + acc[8] * ct * sp - acc[10] * st, lt_i = acc[7] * ct * cp + acc[9] * ct * sp - acc[11] * st;
  const double lp_r = -acc[6] * sp + acc[8] * cp, lp_i = -acc[7] * sp + acc[9] * cp;
  const double k = double(b) / (4.0 * 3.14159265358979323846);
  // E_theta = -j k (L_phi + eta0 N_theta); E_phi = j k (L_theta - eta0 N_phi)
  const double et_r = lp_r + kEta0 * nt_r, et_i = lp_i + kEta0 * nt_i;
  const double ep_r = lt_r - kEta0 * np_r, ep_i = lt_i - kEta0 * np_i;
  const size_t o = (size_t(f) * n_theta + th) * n_phi + ph;
  out[o] = make_float2(float(k * et_i), float(-k * et_r));
  out[size_t(n_freq) * n_theta * n_phi + o] = make_float2(float(-k * ep_i), float(k * ep_r));
}

}  // namespace rfn
