// CPU oracle for the FDTD time-stepping path -- TEST INFRASTRUCTURE ONLY.
//
// A plain-loop restatement of the reference's threaded CPU engine
//   rfnetwork/core/src/solver.cpp  (SolverFDTD::solver_init_* 239-532,
//   solver_run 534-599, solver_controller 604-674, solver_thread 676-1165,
//   update_monitor 1168-1191, update_phasor_monitor 1194-1225)
// written without Eigen (the reference's Eigen submodule is not vendored).
// Eigen is only used there for element-wise Map expressions, so every
// expression below is the same element-wise arithmetic in the same order:
//   E split:  s = Ca*s + Cb*(h1 - h0)               (solver.cpp:909-949)
//   H split:  s = Da*s + (Db2*e2 - Db1*e1)          (solver.cpp:1055-1094)
//   totals:   f = s1 + s2                            (solver.cpp:957-959, 1097-1099)
// Compile with -ffp-contract=off so no multiply-add is fused: the reference
// is built without -march flags (setup.py), so it has no FMA either.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg may load this
// library; it is the checker, never the product path.

#include <algorithm>
#include <barrier>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

enum { EX = 0, EY = 1, EZ = 2, HX = 3, HY = 4, HZ = 5 };
constexpr int kMaxMonitors = 50;    // solver.h:15
constexpr int kMaxProbes = 5000;    // solver.h:16
constexpr int kMaxThreads = 20;     // solver.h:17

// Index of each coefficient in the 30-entry pointer table passed across the
// C ABI (the key order of the dict built at solver.py:1473-1518).
enum Coef {
  Ca_ex_y, Ca_ex_z, Cb_ex_y, Cb_ex_z,
  Ca_ey_z, Ca_ey_x, Cb_ey_z, Cb_ey_x,
  Ca_ez_x, Ca_ez_y, Cb_ez_x, Cb_ez_y,
  Da_hx_y, Da_hx_z, Db_hx_y1, Db_hx_y2, Db_hx_z1, Db_hx_z2,
  Da_hy_z, Da_hy_x, Db_hy_z1, Db_hy_z2, Db_hy_x1, Db_hy_x2,
  Da_hz_x, Da_hz_y, Db_hz_x1, Db_hz_x2, Db_hz_y1, Db_hz_y2,
  kNumCoef
};

template <typename T>
struct Probe {
  T* values;
  int field;
  int x, y, z;          // solver-grid cell after the Yee shift
  bool is_source;
  size_t off;           // offset into the field arrays of `field`
};

template <typename T>
struct Monitor {
  void* values;
  const std::complex<T>* phase;
  int n_freq, field, axis, position, n_step, n1, n2;
  int row_stride, col_stride, yz_offset;
};

template <typename T>
class OracleSolver {
 public:
  OracleSolver(int nx, int ny, int nz) : Nx(nx), Ny(ny), Nz(nz) {
    // Per-slice shapes of the thread grid (solver.cpp:707-721).
    fs_y[EX] = Ny + 1; fs_z[EX] = Nz + 1;
    fs_y[EY] = Ny;     fs_z[EY] = Nz + 1;
    fs_y[EZ] = Ny + 1; fs_z[EZ] = Nz;
    fs_y[HX] = Ny;     fs_z[HX] = Nz;
    fs_y[HY] = Ny + 1; fs_z[HY] = Nz;
    fs_y[HZ] = Ny;     fs_z[HZ] = Nz + 1;
    for (int f = 0; f < 6; ++f) {
      size_t n = size_t(Nx) * fs_y[f] * fs_z[f];
      tot[f].assign(n, T(0));
      s1[f].assign(n, T(0));
      s2[f].assign(n, T(0));
    }
    zero_h.assign(size_t(Ny + 1) * (Nz + 1), T(0));
    zero_e.assign(size_t(Ny + 1) * (Nz + 1), T(0));
  }

  // solver_init_fields (solver.cpp:239-349): borrow the CPU-shaped arrays and
  // zero the last x plane of Cy, Cz and Dx so the x-max wall stays PEC. The
  // reference does this in place on the caller's arrays; the oracle keeps a
  // private copy instead.
  void set_coefficients(const T* const* c) {
    const size_t cx = size_t(Ny - 1) * (Nz - 1), cy = size_t(Ny) * (Nz - 1),
                 cz = size_t(Ny - 1) * Nz, dx = size_t(Ny) * Nz,
                 dy = size_t(Ny + 1) * Nz, dz = size_t(Ny) * (Nz + 1);
    const size_t plane[kNumCoef] = {cx, cx, cx, cx, cy, cy, cy, cy, cz, cz, cz, cz,
                                    dx, dx, dx, dx, dx, dx, dy, dy, dy, dy, dy, dy,
                                    dz, dz, dz, dz, dz, dz};
    for (int i = 0; i < kNumCoef; ++i) {
      coef_plane[i] = plane[i];
      coef[i].assign(c[i], c[i] + plane[i] * Nx);
    }
    auto zero_last = [&](int i) {
      std::fill(coef[i].begin() + (Nx - 1) * coef_plane[i], coef[i].end(), T(0));
    };
    for (int i : {Cb_ey_z, Cb_ey_x, Ca_ey_z, Ca_ey_x, Cb_ez_x, Cb_ez_y, Ca_ez_x, Ca_ez_y,
                  Db_hx_y1, Db_hx_y2, Db_hx_z1, Db_hx_z2, Da_hx_y, Da_hx_z})
      zero_last(i);
  }

  // solver_init_probes (solver.cpp:465-532) plus the offset computation of
  // solver_thread (solver.cpp:774-828).
  void add_probe(int field, int i, int j, int k, int is_source, T* values) {
    if (field < 0 || field > 5) throw std::runtime_error("Invalid probe field type.");
    Probe<T> p{values, field, i, j, k, is_source != 0, 0};
    if (field == EY || field == EZ || field == HX) p.x -= 1;
    if (field == EX || field == EZ || field == HY) p.y -= 1;
    if (field == EX || field == EY || field == HZ) p.z -= 1;
    if (p.x < 0 || p.y < 0 || p.z < 0)
      throw std::runtime_error("Source cannot be placed on grid edge");
    int oy = p.y, oz = p.z;
    if (field == EX) { oy += 1; oz += 1; }
    if (field == EY) { oz += 1; }
    if (field == EZ) { oy += 1; }
    if (field == HY) { oy += 1; }
    if (field == HZ) { oz += 1; }
    // The reference has no upper-bound check here and would write outside the
    // thread slab; the oracle rejects such probes instead.
    if (p.x >= Nx || oy >= fs_y[field] || oz >= fs_z[field])
      throw std::runtime_error("Probe index outside the solver grid");
    p.off = (size_t(p.x) * fs_y[field] + oy) * fs_z[field] + oz;
    probes.push_back(p);
  }

  // solver_init_monitors (solver.cpp:351-463), CPU branch (gpu = 0).
  void add_monitor(int field, int axis, int position, int n_step, int n_freq, void* values,
                   const std::complex<T>* phase) {
    if (field < 0 || field > 5) throw std::runtime_error("Invalid monitor field type.");
    if (n_step < 1) throw std::runtime_error("Invalid monitor step.");
    Monitor<T> m{values, phase, n_freq, field, axis, position, n_step, 0, 0, 0, 0, 0};
    if (axis == 0) {
      if (field == HX || field == EY || field == EZ) m.position -= 1;
      m.row_stride = fs_z[field];
      m.col_stride = 1;
      m.yz_offset = 0;
      m.n1 = fs_y[field];
      m.n2 = fs_z[field];
    } else if (axis == 1) {
      m.row_stride = fs_y[field] * fs_z[field];
      m.col_stride = 1;
      m.yz_offset = m.position * fs_z[field];
      m.n1 = Nx;
      m.n2 = fs_z[field];
      if (m.position < 0 || m.position >= fs_y[field])
        throw std::runtime_error("Monitor position outside the solver grid");
    } else if (axis == 2) {
      m.row_stride = fs_y[field] * fs_z[field];
      m.col_stride = fs_z[field];
      m.yz_offset = m.position;
      m.n1 = Nx;
      m.n2 = fs_y[field];
      if (m.position < 0 || m.position >= fs_z[field])
        throw std::runtime_error("Monitor position outside the solver grid");
    } else {
      throw std::runtime_error("Invalid monitor axis.");
    }
    monitors.push_back(m);
  }

  // solver_run + solver_controller + solver_thread (solver.cpp:534-1165). The
  // x slabs are split exactly as the reference splits them; the two barriers
  // per step stand in for the controller's condition variables.
  void run(int Nt, int n_threads) {
    if (n_threads < 1 || n_threads > kMaxThreads)
      throw std::runtime_error("Invalid number of threads.");
    n_threads = std::min(n_threads, Nx);
    std::vector<int> xs(n_threads + 1, 0);
    int base = Nx / n_threads, rem = Nx % n_threads;
    for (int t = 0; t < n_threads; ++t) xs[t + 1] = xs[t] + base + (t < rem ? 1 : 0);

    std::barrier sync(n_threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t)
      pool.emplace_back([&, t] { worker(xs[t], xs[t + 1], Nt, sync); });
    for (auto& th : pool) th.join();
  }

 private:
  int Nx, Ny, Nz;
  int fs_y[6], fs_z[6];
  std::vector<T> tot[6], s1[6], s2[6];
  std::vector<T> zero_h, zero_e;
  std::vector<T> coef[kNumCoef];
  size_t coef_plane[kNumCoef];
  std::vector<Probe<T>> probes;
  std::vector<Monitor<T>> monitors;

  size_t slice(int f) const { return size_t(fs_y[f]) * fs_z[f]; }
  const T* C(int i, int x) const { return coef[i].data() + size_t(x) * coef_plane[i]; }

  void update_e(int x) {
    const int ny = Ny, nz = Nz;
    T* exy = s1[EX].data() + x * slice(EX);  T* exz = s2[EX].data() + x * slice(EX);
    T* eyz = s1[EY].data() + x * slice(EY);  T* eyx = s2[EY].data() + x * slice(EY);
    T* ezx = s1[EZ].data() + x * slice(EZ);  T* ezy = s2[EZ].data() + x * slice(EZ);
    const T* hx = tot[HX].data() + x * slice(HX);
    const T* hy = tot[HY].data() + x * slice(HY);
    const T* hz = tot[HZ].data() + x * slice(HZ);
    const T* hy1 = (x < Nx - 1) ? tot[HY].data() + (x + 1) * slice(HY) : zero_h.data();
    const T* hz1 = (x < Nx - 1) ? tot[HZ].data() + (x + 1) * slice(HZ) : zero_h.data();
    const T *caxy = C(Ca_ex_y, x), *cbxy = C(Cb_ex_y, x), *caxz = C(Ca_ex_z, x), *cbxz = C(Cb_ex_z, x);
    const T *cayz = C(Ca_ey_z, x), *cbyz = C(Cb_ey_z, x), *cayx = C(Ca_ey_x, x), *cbyx = C(Cb_ey_x, x);
    const T *cazx = C(Ca_ez_x, x), *cbzx = C(Cb_ez_x, x), *cazy = C(Ca_ez_y, x), *cbzy = C(Cb_ez_y, x);
    const int ex_r = nz + 1, ey_r = nz + 1, ez_r = nz, hx_r = nz, hy_r = nz, hz_r = nz + 1;

    // ex: rows 1..Ny-1, cols 1..Nz-1 (solver.cpp:909-918)
    for (int j = 1; j < ny; ++j) {
      const int c = (j - 1) * (nz - 1) - 1;
      for (int k = 1; k < nz; ++k) {
        const int e = j * ex_r + k;
        exy[e] = caxy[c + k] * exy[e] + cbxy[c + k] * (hz[j * hz_r + k] - hz[(j - 1) * hz_r + k]);
        exz[e] = caxz[c + k] * exz[e] + cbxz[c + k] * (hy[j * hy_r + k] - hy[j * hy_r + k - 1]);
      }
    }
    // ey: rows 0..Ny-1, cols 1..Nz-1 (solver.cpp:924-933)
    for (int j = 0; j < ny; ++j) {
      const int c = j * (nz - 1) - 1;
      for (int k = 1; k < nz; ++k) {
        const int e = j * ey_r + k;
        eyz[e] = cayz[c + k] * eyz[e] + cbyz[c + k] * (hx[j * hx_r + k] - hx[j * hx_r + k - 1]);
        eyx[e] = cayx[c + k] * eyx[e] + cbyx[c + k] * (hz1[j * hz_r + k] - hz[j * hz_r + k]);
      }
    }
    // ez: rows 1..Ny-1, cols 0..Nz-1 (solver.cpp:940-949)
    for (int j = 1; j < ny; ++j) {
      const int c = (j - 1) * nz;
      for (int k = 0; k < nz; ++k) {
        const int e = j * ez_r + k;
        ezx[e] = cazx[c + k] * ezx[e] + cbzx[c + k] * (hy1[j * hy_r + k] - hy[j * hy_r + k]);
        ezy[e] = cazy[c + k] * ezy[e] + cbzy[c + k] * (hx[j * hx_r + k] - hx[(j - 1) * hx_r + k]);
      }
    }
    sum_slice(EX, x);
    sum_slice(EY, x);
    sum_slice(EZ, x);
  }

  void update_h(int x) {
    const int ny = Ny, nz = Nz;
    T* hxy = s1[HX].data() + x * slice(HX);  T* hxz = s2[HX].data() + x * slice(HX);
    T* hyz = s1[HY].data() + x * slice(HY);  T* hyx = s2[HY].data() + x * slice(HY);
    T* hzx = s1[HZ].data() + x * slice(HZ);  T* hzy = s2[HZ].data() + x * slice(HZ);
    const T* ex = tot[EX].data() + x * slice(EX);
    const T* ey = tot[EY].data() + x * slice(EY);
    const T* ez = tot[EZ].data() + x * slice(EZ);
    const T* ey0 = (x > 0) ? tot[EY].data() + (x - 1) * slice(EY) : zero_e.data();
    const T* ez0 = (x > 0) ? tot[EZ].data() + (x - 1) * slice(EZ) : zero_e.data();
    const T *dxy = C(Da_hx_y, x), *dxz = C(Da_hx_z, x);
    const T *bxy1 = C(Db_hx_y1, x), *bxy2 = C(Db_hx_y2, x), *bxz1 = C(Db_hx_z1, x), *bxz2 = C(Db_hx_z2, x);
    const T *dyz = C(Da_hy_z, x), *dyx = C(Da_hy_x, x);
    const T *byz1 = C(Db_hy_z1, x), *byz2 = C(Db_hy_z2, x), *byx1 = C(Db_hy_x1, x), *byx2 = C(Db_hy_x2, x);
    const T *dzx = C(Da_hz_x, x), *dzy = C(Da_hz_y, x);
    const T *bzx1 = C(Db_hz_x1, x), *bzx2 = C(Db_hz_x2, x), *bzy1 = C(Db_hz_y1, x), *bzy2 = C(Db_hz_y2, x);
    const int ex_r = nz + 1, ey_r = nz + 1, ez_r = nz;

    // hx: Ny x Nz (solver.cpp:1055-1064)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int h = j * nz + k;
        hxy[h] = dxy[h] * hxy[h] + (bxy2[h] * ez[(j + 1) * ez_r + k] - bxy1[h] * ez[j * ez_r + k]);
        hxz[h] = dxz[h] * hxz[h] + (bxz2[h] * ey[j * ey_r + k + 1] - bxz1[h] * ey[j * ey_r + k]);
      }
    // hy: (Ny+1) x Nz (solver.cpp:1070-1079)
    for (int j = 0; j <= ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int h = j * nz + k;
        hyz[h] = dyz[h] * hyz[h] + (byz2[h] * ex[j * ex_r + k + 1] - byz1[h] * ex[j * ex_r + k]);
        hyx[h] = dyx[h] * hyx[h] + (byx2[h] * ez[j * ez_r + k] - byx1[h] * ez0[j * ez_r + k]);
      }
    // hz: Ny x (Nz+1) (solver.cpp:1085-1094)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k <= nz; ++k) {
        const int h = j * (nz + 1) + k;
        hzx[h] = dzx[h] * hzx[h] + (bzx2[h] * ey[j * ey_r + k] - bzx1[h] * ey0[j * ey_r + k]);
        hzy[h] = dzy[h] * hzy[h] + (bzy2[h] * ex[(j + 1) * ex_r + k] - bzy1[h] * ex[j * ex_r + k]);
      }
    sum_slice(HX, x);
    sum_slice(HY, x);
    sum_slice(HZ, x);
  }

  void sum_slice(int f, int x) {
    const size_t n = slice(f), o = size_t(x) * n;
    T* t = tot[f].data() + o;
    const T* a = s1[f].data() + o;
    const T* b = s2[f].data() + o;
    for (size_t i = 0; i < n; ++i) t[i] = a[i] + b[i];
  }

  // Probe block (solver.cpp:962-976 and 1103-1116).
  void apply_probe(const Probe<T>& p, int n) {
    if (p.is_source) {
      s1[p.field][p.off] = s1[p.field][p.off] + p.values[n];
      s2[p.field][p.off] = s2[p.field][p.off] + p.values[n];
      tot[p.field][p.off] = s1[p.field][p.off] + s2[p.field][p.off];
    }
    p.values[n] = tot[p.field][p.off];
  }

  // update_monitor / update_phasor_monitor (solver.cpp:1168-1225).
  void sample_monitor(const Monitor<T>& m, int n, int x0, int x1) {
    if (n > 0 && (n % m.n_step) != 0) return;
    if (m.axis == 0 && (m.position < x0 || m.position >= x1)) return;
    const int mn = n / m.n_step;
    const T* fld = tot[m.field].data();
    const size_t n1n2 = size_t(m.n1) * m.n2;
    auto value_at = [&](int a, int b) -> T {   // (a, b) in monitor-plane coordinates
      if (m.axis == 0) return fld[size_t(m.position) * n1n2 + size_t(a) * m.n2 + b];
      return fld[size_t(a) * m.row_stride + m.yz_offset + size_t(b) * m.col_stride];
    };
    const int a0 = (m.axis == 0) ? 0 : x0, a1 = (m.axis == 0) ? m.n1 : x1;
    if (m.n_freq == 0) {
      T* out = static_cast<T*>(m.values) + size_t(mn) * n1n2;
      for (int a = a0; a < a1; ++a)
        for (int b = 0; b < m.n2; ++b) out[size_t(a) * m.n2 + b] = value_at(a, b);
    } else {
      for (int f = 0; f < m.n_freq; ++f) {
        std::complex<T>* out = static_cast<std::complex<T>*>(m.values) + size_t(f) * n1n2;
        const std::complex<T> ph = m.phase[size_t(mn) * m.n_freq + f];
        for (int a = a0; a < a1; ++a)
          for (int b = 0; b < m.n2; ++b)
            out[size_t(a) * m.n2 + b] += std::complex<T>(value_at(a, b)) * ph;
      }
    }
  }

  void worker(int x0, int x1, int Nt, std::barrier<>& sync) {
    std::vector<const Probe<T>*> ep, hp;
    for (const auto& p : probes)
      if (p.x >= x0 && p.x < x1) (p.field < 3 ? ep : hp).push_back(&p);
    for (int n = 0; n < Nt; ++n) {
      for (int x = x0; x < x1; ++x) update_e(x);
      for (auto* p : ep) apply_probe(*p, n);
      sync.arrive_and_wait();
      for (int x = x0; x < x1; ++x) update_h(x);
      for (auto* p : hp) apply_probe(*p, n);
      sync.arrive_and_wait();
      for (const auto& m : monitors) sample_monitor(m, n, x0, x1);
    }
  }
};

template <typename T>
int run_oracle(int nx, int ny, int nz, int nt, int n_threads, const void* const* coeff,
               int n_probes, const int* probe_field, const int* probe_ijk,
               const int* probe_is_source, void* const* probe_values, int n_monitors,
               const int* mon_field, const int* mon_axis, const int* mon_position,
               const int* mon_n_step, const int* mon_n_freq, void* const* mon_values,
               const void* const* mon_phase, char* err, int err_len) {
  try {
    if (nx < 1 || ny < 2 || nz < 2 || nt < 0) throw std::runtime_error("Invalid grid size.");
    if (n_probes > kMaxProbes) throw std::runtime_error("Exceeded maximum number of probes.");
    if (n_monitors > kMaxMonitors) throw std::runtime_error("Exceeded maximum number of monitors.");
    OracleSolver<T> s(nx, ny, nz);
    s.set_coefficients(reinterpret_cast<const T* const*>(coeff));
    for (int m = 0; m < n_monitors; ++m)
      s.add_monitor(mon_field[m], mon_axis[m], mon_position[m], mon_n_step[m], mon_n_freq[m],
                    mon_values[m], static_cast<const std::complex<T>*>(mon_phase[m]));
    for (int p = 0; p < n_probes; ++p)
      s.add_probe(probe_field[p], probe_ijk[3 * p], probe_ijk[3 * p + 1], probe_ijk[3 * p + 2],
                  probe_is_source[p], static_cast<T*>(probe_values[p]));
    s.run(nt, n_threads);
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::snprintf(err, size_t(err_len), "%s", e.what());
    }
    return 1;
  }
}

}  // namespace

extern "C" {

int oracle_run_f32(int nx, int ny, int nz, int nt, int n_threads, const void* const* coeff,
                   int n_probes, const int* probe_field, const int* probe_ijk,
                   const int* probe_is_source, void* const* probe_values, int n_monitors,
                   const int* mon_field, const int* mon_axis, const int* mon_position,
                   const int* mon_n_step, const int* mon_n_freq, void* const* mon_values,
                   const void* const* mon_phase, char* err, int err_len) {
  return run_oracle<float>(nx, ny, nz, nt, n_threads, coeff, n_probes, probe_field, probe_ijk,
                           probe_is_source, probe_values, n_monitors, mon_field, mon_axis,
                           mon_position, mon_n_step, mon_n_freq, mon_values, mon_phase, err,
                           err_len);
}

int oracle_run_f64(int nx, int ny, int nz, int nt, int n_threads, const void* const* coeff,
                   int n_probes, const int* probe_field, const int* probe_ijk,
                   const int* probe_is_source, void* const* probe_values, int n_monitors,
                   const int* mon_field, const int* mon_axis, const int* mon_position,
                   const int* mon_n_step, const int* mon_n_freq, void* const* mon_values,
                   const void* const* mon_phase, char* err, int err_len) {
  return run_oracle<double>(nx, ny, nz, nt, n_threads, coeff, n_probes, probe_field, probe_ijk,
                            probe_is_source, probe_values, n_monitors, mon_field, mon_axis,
                            mon_position, mon_n_step, mon_n_freq, mon_values, mon_phase, err,
                            err_len);
}

}  // extern "C"
