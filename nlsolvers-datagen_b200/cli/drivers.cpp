// Drop-in replacements for the ten executables of device/drivers
// (device/drivers/CMakeLists.txt:15-31). Same names, same positional argv,
// same .npy inputs and outputs, same derived constants:
//   real 2-D (kg_driver_dev_2d.cpp:19-49):  nx ny Lx Ly u0 v0 traj vel T nt ns m c
//   real 3-D (kg_driver_dev_3d.cpp:19-49):  nx ny nz Lx Ly Lz u0 v0 traj vel T nt ns m c
//   NLSE 2-D (nlse_cubic_driver_2d.cpp:19-41): nx ny Lx Ly u0 traj T nt ns m c
//   NLSE 3-D (nlse_cubic_driver_3d.cpp:19-44): nx ny nz Lx Ly Lz u0 traj T nt ns m c
// Compiled once per executable with NLS_DRIVER_ID (0..9, table below).
// Optional environment knobs (the launchers need none of them):
//   NLS_PRECISION=fp32|fp64   (default fp64, the reference's arithmetic; fp32: compensated
//                              FP32 fields and FP32 Krylov basis, within 1e-5 rel-L2 of it)
//   NLS_KRYLOV_K=<k>          (default: the reference binary's k)
//   NLS_SEED=<uint64>         (phi^4 noise key; default: wall clock, as stochastic_phi4.cuh:25)
//   NLS_SEWI_VARIANT=reference|corrected
//   NLS_NONLINEARITY=sine|dsine|sinh (KG / phi^4 executables) or cq|sat (NLSE):
//                              the solvers the reference's build names without sources
//                              (sine-Gordon, double / hyperbolic sine-Gordon, cubic-quintic,
//                              saturable NLSE; forms in include/nlsb200.h); default: the
//                              executable's own nonlinearity
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nlsb200.h"
#include "../csrc/npy.hpp"

#ifndef NLS_DRIVER_ID
#error "NLS_DRIVER_ID must be defined"
#endif

namespace {

struct Driver {
  const char *name;
  int method, dim, k;
};
// reference k per binary: kg_driver_dev_2d.cpp:138, nlse_cubic_driver_2d.cpp:104,
// nlse_cubic_sewi_driver_2d.cpp:104, nlse_cubic_driver_3d.cpp:112, nlse_cubic_sewi_driver_3d.cpp:112
const Driver kDrivers[10] = {
    {"kg_gautschi_2d_dev", NLS_KG_GAUTSCHI, 2, 10}, {"kg_sv_2d_dev", NLS_KG_SV, 2, 10},
    {"kg_gautschi_3d_dev", NLS_KG_GAUTSCHI, 3, 10}, {"kg_sv_3d_dev", NLS_KG_SV, 3, 10},
    {"sp4_sv_2d_dev", NLS_SP4_SV, 2, 10},           {"sp4_sv_3d_dev", NLS_SP4_SV, 3, 10},
    {"nlse_2d_dev", NLS_NLSE_SS2, 2, 20},           {"nlse_3d_dev", NLS_NLSE_SS2, 3, 25},
    {"nlse_sewi_2d_dev", NLS_NLSE_SEWI, 2, 10},     {"nlse_sewi_3d_dev", NLS_NLSE_SEWI, 3, 15},
};

const Driver &D = kDrivers[NLS_DRIVER_ID];
bool nlse() { return D.method == NLS_NLSE_SS2 || D.method == NLS_NLSE_SEWI; }

std::vector<uint64_t> expect_shape(uint32_t nx, uint32_t ny, uint32_t nz) {
  if (D.dim == 2) return {ny, nx};
  return {nz, ny, nx};
}

std::string shape_str(const std::vector<uint64_t> &s) {
  std::string r;
  for (size_t i = 0; i < s.size(); ++i) r += (i ? "x" : "") + std::to_string(s[i]);
  return r;
}

npy::Array load_checked(const std::string &path, const std::string &descr,
                        const std::vector<uint64_t> &shape, const char *what) {
  npy::Array a = npy::load(path);
  if (a.descr != descr) throw std::runtime_error(std::string(what) + ": expected dtype " + descr + ", got " + a.descr);
  if (a.shape != shape)
    throw std::runtime_error(std::string("Error: ") + what + " array dimensions mismatch. Expected: " +
                             shape_str(shape) + " Got: " + shape_str(a.shape));
  return a;
}

void usage(const char *argv0) {
  if (D.dim == 2 && !nlse())
    std::cerr << "Usage: " << argv0
              << " nx ny Lx Ly input_u0.npy input_v0.npy output_traj.npy output_vel.npy T nt "
                 "num_snapshots input_m.npy input_c.npy\n";
  else if (D.dim == 3 && !nlse())
    std::cerr << "Usage: " << argv0
              << " nx ny nz Lx Ly Lz input_u0.npy input_v0.npy output_traj.npy output_vel.npy T nt "
                 "num_snapshots input_m.npy input_c.npy\n";
  else if (D.dim == 2)
    std::cerr << "Usage: " << argv0
              << " nx ny Lx Ly input_u0.npy output_traj.npy T nt num_snapshots input_m.npy input_c.npy\n";
  else
    std::cerr << "Usage: " << argv0
              << " nx ny nz Lx Ly Lz input_u0.npy output_traj.npy T nt num_snapshots input_m.npy "
                 "input_c.npy\n";
}

int lib_error(int rc, const char *what) {
  char buf[512];
  nls_last_error(buf, sizeof(buf));
  std::cerr << what << " failed: " << nls_strerror(rc) << ": " << buf << "\n";
  return 1;
}

int run(int argc, char **argv) {
  const int want = (D.dim == 2 ? 14 : 16) - (nlse() ? 2 : 0);
  if (argc != want) {
    usage(argv[0]);
    return 1;
  }
  int a = 1;
  const uint32_t nx = std::stoul(argv[a++]);
  const uint32_t ny = std::stoul(argv[a++]);
  const uint32_t nz = D.dim == 3 ? (uint32_t)std::stoul(argv[a++]) : 1u;
  const double Lx = std::stod(argv[a++]);
  const double Ly = std::stod(argv[a++]);
  const double Lz = D.dim == 3 ? std::stod(argv[a++]) : 0.0;
  const std::string f_u0 = argv[a++];
  const std::string f_v0 = nlse() ? "" : argv[a++];
  const std::string f_traj = argv[a++];
  const std::string f_vel = nlse() ? "" : argv[a++];
  const double T = std::stod(argv[a++]);
  const uint32_t nt = std::stoul(argv[a++]);
  const uint32_t ns = std::stoul(argv[a++]);
  const std::string f_m = argv[a++];
  const std::string f_c = argv[a++];
  if (ns == 0 || nt / ns == 0) {
    std::cerr << "Error: need nt >= num_snapshots > 0\n";
    return 1;
  }
  const std::vector<uint64_t> shape = expect_shape(nx, ny, nz);
  npy::Array u0 = load_checked(f_u0, nlse() ? "<c16" : "<f8", shape, "Input");
  npy::Array v0;
  if (!nlse()) v0 = load_checked(f_v0, "<f8", shape, "Velocity");
  npy::Array m = load_checked(f_m, "<f8", shape, "Coupling m");
  npy::Array c = load_checked(f_c, "<f8", shape, "Anisotropy c");

  nls_problem p;
  nls_problem_defaults(&p, D.method, D.dim);
  p.nx = (int32_t)nx;
  p.ny = (int32_t)ny;
  p.nz = (int32_t)nz;
  p.Lx = Lx;
  p.Ly = Ly;
  p.Lz = Lz;
  p.T = T;
  p.nt = (int32_t)nt;
  p.ns = (int32_t)ns;
  p.k = D.k;
  if (const char *e = std::getenv("NLS_KRYLOV_K")) p.k = std::atoi(e);
  p.precision = NLS_FP64;
  if (const char *e = std::getenv("NLS_PRECISION")) p.precision = std::strcmp(e, "fp32") == 0 ? NLS_FP32 : NLS_FP64;
  if (const char *e = std::getenv("NLS_SEWI_VARIANT")) p.sewi_variant = std::strcmp(e, "corrected") == 0 ? 1 : 0;
  if (const char *e = std::getenv("NLS_NONLINEARITY")) {
    const char *names[] = {"poly", "sine", "dsine", "sinh", "cq", "sat"};
    int kind = -1;
    for (int i = 0; i < 6; ++i)
      if (std::strcmp(e, names[i]) == 0) kind = i;
    if (kind < 0) {
      std::cerr << "NLS_NONLINEARITY must be one of poly, sine, dsine, sinh, cq, sat\n";
      return 1;
    }
    p.nonlinearity = kind;
  }
  const double *cd = reinterpret_cast<const double *>(c.data.data());
  const uint64_t n = u0.count();
  bool c_is_one = true;
  for (uint64_t i = 0; i < n && c_is_one; ++i) c_is_one = cd[i] == 1.0;
  p.has_c = c_is_one ? 0 : 1;  // c == 1: identical arithmetic, no c traffic
  if (D.method == NLS_SP4_SV || D.method == NLS_SP4_GAUTSCHI) {
    // noise scale alpha sqrt(kBT dx)/dt with dx = 2L/(nx-1) (stochastic_phi4_dev.hpp:47-51)
    const double dt = T / nt, dx = 2 * Lx / (nx - 1);
    p.rm = -(0.01 * std::sqrt(2.0 * dx) / dt);
    p.seed = (uint64_t)std::time(nullptr);
    if (const char *e = std::getenv("NLS_SEED")) p.seed = std::strtoull(e, nullptr, 10);
  }
  nls_handle *h = nullptr;
  int rc = nls_create(&p, reinterpret_cast<const double *>(u0.data.data()),
                      nlse() ? nullptr : reinterpret_cast<const double *>(v0.data.data()),
                      reinterpret_cast<const double *>(m.data.data()), p.has_c ? cd : nullptr, &h);
  if (rc) return lib_error(rc, "nls_create");
  rc = nls_run(h);
  if (rc) {
    nls_destroy(h);
    return lib_error(rc, "nls_run");
  }
  const uint64_t comps = nlse() ? 2 : 1;
  std::vector<double> traj(ns * n * comps), vel(nlse() ? 0 : ns * n);
  rc = nls_snapshot(h, traj.data(), nlse() ? nullptr : vel.data());
  nls_destroy(h);
  if (rc) return lib_error(rc, "nls_snapshot");
  // outputs (ns, ny, nx) / (ns, nz, ny, nx); kg_driver_dev_3d.cpp:161 writes a
  // 3-entry header for 4-D data, here the header matches the data.
  std::vector<uint64_t> oshape = {ns};
  for (auto d : shape) oshape.push_back(d);
  npy::save(f_traj, nlse() ? "<c16" : "<f8", oshape, traj.data(), traj.size() * sizeof(double));
  if (!nlse()) npy::save(f_vel, "<f8", oshape, vel.data(), vel.size() * sizeof(double));
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception &e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
}
