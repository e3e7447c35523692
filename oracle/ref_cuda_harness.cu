// Harness that runs the reference's own CUDA engine -- TEST INFRASTRUCTURE ONLY.
//
// rfnetwork/core/src/solver.cu (SolverFDTD::solver_run_cu, solver.cu:546-1143)
// is compiled unmodified from the reference checkout next to this file. The
// reference fills SolverFDTD's members in solver_init_fields / _monitors /
// _probes (rfnetwork/core/src/solver.cpp:239-532), which live in the
// Eigen-dependent translation unit and cannot be built here; this harness sets
// the same members the same way for the GPU case (gpu = 1):
//   * coefficient pointers, with the last x plane of Cy, Cz and Dx zeroed
//     (solver.cpp:294-328) on a private copy;
//   * probes with the Yee index shift (solver.cpp:503-520) and is_source set
//     for every probe, as solver.cpp:528 does (it stores the dict lookup, which
//     is non-null whenever the key exists);
//   * monitors with the GPU position shifts and strides (solver.cpp:377-460).
// Both this file and solver.cu are compiled with -Dprivate=public so the
// harness can reach the members.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "solver.h"

SolverFDTD::SolverFDTD() {
  n_monitors = 0;
  n_probes = 0;
  n_threads = 0;
}

namespace {
enum { EX = 0, EY = 1, EZ = 2, HX = 3, HY = 4, HZ = 5 };
}

extern "C" int ref_cuda_run(int Nx, int Ny, int Nz, int Nt, const float* const* coef, int n_probes,
                            const int* probe_field, const int* probe_ijk, float* const* probe_values,
                            int n_monitors, const int* mon_field, const int* mon_axis, const int* mon_position,
                            const int* mon_n_step, const int* mon_n_freq, void* const* mon_values,
                            void* const* mon_phase, char* err, int err_len) {
  try {
    if (n_probes > MAX_PROBES || n_monitors > MAX_MONITORS) throw std::runtime_error("too many probes/monitors");
    auto* s = new SolverFDTD();
    std::vector<std::vector<float>> copies(30);
    const size_t N = size_t(Nx) * Ny * Nz, plane = size_t(Ny) * Nz;
    for (int i = 0; i < 30; ++i) copies[i].assign(coef[i], coef[i] + N);
    // order of `coef`: the dict key order of rfnetwork/solver.py:1473-1518
    float** c = nullptr;
    std::vector<float*> p(30);
    for (int i = 0; i < 30; ++i) p[i] = copies[i].data();
    c = p.data();
    s->Nx = Nx;
    s->Ny = Ny;
    s->Nz = Nz;
    s->Cx.Ca_ex_y = c[0]; s->Cx.Ca_ex_z = c[1]; s->Cx.Cb_ex_y = c[2]; s->Cx.Cb_ex_z = c[3];
    s->Cy.Ca_ey_z = c[4]; s->Cy.Ca_ey_x = c[5]; s->Cy.Cb_ey_z = c[6]; s->Cy.Cb_ey_x = c[7];
    s->Cz.Ca_ez_x = c[8]; s->Cz.Ca_ez_y = c[9]; s->Cz.Cb_ez_x = c[10]; s->Cz.Cb_ez_y = c[11];
    s->Dx.Da_hx_y = c[12]; s->Dx.Da_hx_z = c[13]; s->Dx.Db_hx_y1 = c[14]; s->Dx.Db_hx_y2 = c[15];
    s->Dx.Db_hx_z1 = c[16]; s->Dx.Db_hx_z2 = c[17];
    s->Dy.Da_hy_z = c[18]; s->Dy.Da_hy_x = c[19]; s->Dy.Db_hy_z1 = c[20]; s->Dy.Db_hy_z2 = c[21];
    s->Dy.Db_hy_x1 = c[22]; s->Dy.Db_hy_x2 = c[23];
    s->Dz.Da_hz_x = c[24]; s->Dz.Da_hz_y = c[25]; s->Dz.Db_hz_x1 = c[26]; s->Dz.Db_hz_x2 = c[27];
    s->Dz.Db_hz_y1 = c[28]; s->Dz.Db_hz_y2 = c[29];
    for (int i = 4; i < 18; ++i) std::memset(c[i] + (Nx - 1) * plane, 0, plane * sizeof(float));

    s->n_probes = n_probes;
    for (int q = 0; q < n_probes; ++q) {
      Probe& pr = s->probes[q];
      pr.values = probe_values[q];
      pr.field_type = probe_field[q];
      pr.x_cell = probe_ijk[3 * q];
      pr.y_cell = probe_ijk[3 * q + 1];
      pr.z_cell = probe_ijk[3 * q + 2];
      const int f = pr.field_type;
      if (f == EY || f == EZ || f == HX) pr.x_cell -= 1;
      if (f == EX || f == EZ || f == HY) pr.y_cell -= 1;
      if (f == EX || f == EY || f == HZ) pr.z_cell -= 1;
      if (pr.x_cell < 0 || pr.y_cell < 0 || pr.z_cell < 0)
        throw std::runtime_error("Source cannot be placed on grid edge");
      if (pr.x_cell >= Nx || pr.y_cell >= Ny || pr.z_cell >= Nz)
        throw std::runtime_error("Probe index outside the solver grid");
      pr.is_source = true;
    }

    s->n_monitors = n_monitors;
    for (int m = 0; m < n_monitors; ++m) {
      Monitor& M = s->monitors[m];
      const int field = mon_field[m], axis = mon_axis[m];
      M.field_type = field;
      M.position = mon_position[m];
      M.n_step = mon_n_step[m];
      M.axis = axis;
      if (axis == 0) {
        if (field == HX || field == EY || field == EZ) M.position -= 1;
        M.N1 = Ny;
        M.N2 = Nz;
      } else if (axis == 1) {
        if (field == HY || field == EX || field == EZ) M.position -= 1;
        M.N1 = Nx;
        M.N2 = Nz;
      } else {
        if (field == HZ || field == EX || field == EY) M.position -= 1;
        M.N1 = Nx;
        M.N2 = Ny;
      }
      M.N1N2 = M.N1 * M.N2;
      M.n_phasors = mon_n_freq[m];
      M.values = static_cast<char*>(mon_values[m]);
      M.dtft_phase = static_cast<std::complex<float>*>(mon_phase[m]);
    }
    s->solver_run_cu(Nt);
    delete s;
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), size_t(err_len) - 1);
      err[err_len - 1] = 0;
    }
    return 1;
  }
}
