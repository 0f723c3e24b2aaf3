// quasi_run: C++ host driver over the C ABI of libquasi_gpu.so, with the
// reference's command line and output files (quasi/quasi.cpp main()).
//
//   quasi_run <nu> <ep*1000> <fc_size> <load> [--grid NX NY NZ] [--variant quasi|stb]
//             [--precision fp64|fp32] [--ranks P] [--ic planar|undulated|interface|droplet|stb|focal_conic]
//             [--seed S] [--steps K] [--until-l1 X] [--step-l1 N] [--step-save M] [--digits D] [--out DIR]
//
// load == 1 reads DIR/save/psi<rank>.dat (one value per line, (i_local, j, k)
// order, quasi.cpp:692-717); otherwise the IC is built by the library
// (the reference's own is focal_conic, quasi.cpp:543-589).  Every --step-l1
// steps L1.dat, mass.dat, energy.dat are appended (quasi.cpp:1969-2033) and
// every --step-save diagnostics psi<rank>.dat is rewritten and the j = Ny/2
// mid-slices psiMid/vx/vy/vz/divv/p/rho.dat are appended (quasi.cpp:2037-2280).
// Values are written with --digits significant digits (the reference's
// ostream default is 6; the default here is 17 so that dumps round-trip).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/quasi_gpu.h"

namespace {

[[noreturn]] void die(const std::string& what) {
  std::cerr << "quasi_run: " << what << "\n";
  std::exit(1);
}

void check(int rc, const char* what) {
  if (rc != QUASI_OK) die(std::string(what) + ": " + quasi_last_error());
}

struct Args {
  double nu = 1, ep_arg = 675, fc = 6;
  int load = 0;
  int nx = 64, ny = 64, nz = 128;
  int variant = QUASI_VARIANT_QUASI, precision = QUASI_PREC_FP64, ranks = 1;
  int ic = QUASI_IC_FOCAL_CONIC;
  unsigned long long seed = 1234;
  long steps = 500;
  double until_l1 = -1;
  int step_l1 = 50, step_save = 10, digits = 17;
  std::string out = "quasi_out";
};

int ic_kind(const std::string& s) {
  const char* names[] = {"planar", "undulated", "interface", "droplet", "stb", "focal_conic"};
  for (int i = 0; i < 6; ++i)
    if (s == names[i]) return i;
  die("unknown --ic " + s);
}

Args parse(int argc, char** argv) {
  if (argc < 5) die("usage: quasi_run <nu> <ep*1000> <fc_size> <load> [options]");
  Args a;
  a.nu = std::atof(argv[1]);
  a.ep_arg = std::atof(argv[2]);
  a.fc = std::atof(argv[3]);
  a.load = std::atoi(argv[4]);
  for (int i = 5; i < argc; ++i) {
    std::string k = argv[i];
    auto need = [&](int n) {
      if (i + n >= argc) die("missing value for " + k);
    };
    if (k == "--grid") { need(3); a.nx = std::atoi(argv[++i]); a.ny = std::atoi(argv[++i]); a.nz = std::atoi(argv[++i]); }
    else if (k == "--variant") { need(1); std::string v = argv[++i]; a.variant = v == "stb" ? QUASI_VARIANT_STB : QUASI_VARIANT_QUASI; }
    else if (k == "--precision") { need(1); std::string v = argv[++i]; a.precision = v == "fp32" ? QUASI_PREC_FP32 : QUASI_PREC_FP64; }
    else if (k == "--ranks") { need(1); a.ranks = std::atoi(argv[++i]); }
    else if (k == "--ic") { need(1); a.ic = ic_kind(argv[++i]); }
    else if (k == "--seed") { need(1); a.seed = std::strtoull(argv[++i], nullptr, 10); }
    else if (k == "--steps") { need(1); a.steps = std::atol(argv[++i]); }
    else if (k == "--until-l1") { need(1); a.until_l1 = std::atof(argv[++i]); }
    else if (k == "--step-l1") { need(1); a.step_l1 = std::atoi(argv[++i]); }
    else if (k == "--step-save") { need(1); a.step_save = std::atoi(argv[++i]); }
    else if (k == "--digits") { need(1); a.digits = std::atoi(argv[++i]); }
    else if (k == "--out") { need(1); a.out = argv[++i]; }
    else die("unknown option " + k);
  }
  return a;
}

void append(const std::string& path, const double* v, size_t n, int digits, bool truncate = false) {
  std::ofstream f(path, truncate ? std::ios::trunc : std::ios::app);
  if (!f) die("cannot open " + path);
  f << std::setprecision(digits);
  for (size_t i = 0; i < n; ++i) f << v[i] << "\n";
}

// x-z slice at j = ny/2 in the reference's gathered order (i major, k minor)
std::vector<double> mid_slice(const std::vector<double>& a, int nx, int ny, int nz) {
  std::vector<double> s(size_t(nx) * nz);
  const int j = ny / 2;
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k) s[size_t(i) * nz + k] = a[(size_t(i) * ny + j) * nz + k];
  return s;
}

}  // namespace

int main(int argc, char** argv) {
  Args a = parse(argc, argv);
  quasi_config cfg;
  check(quasi_config_default(&cfg, a.variant, a.nx, a.ny, a.nz), "config");
  cfg.nu_arg = a.nu;
  cfg.ep_arg = a.ep_arg;
  cfg.precision = a.precision;
  cfg.emulate_ranks = a.ranks;
  mkdir(a.out.c_str(), 0755);
  const size_t n = size_t(a.nx) * a.ny * a.nz;
  const size_t n0 = size_t(a.nx / a.ranks) * a.ny * a.nz;
  std::vector<double> psi(n);
  if (a.load == 1) {
    for (int r = 0; r < a.ranks; ++r) {
      std::ifstream f(a.out + "/save/psi" + std::to_string(r) + ".dat");
      if (!f) die("cannot read " + a.out + "/save/psi" + std::to_string(r) + ".dat");
      for (size_t i = 0; i < n0; ++i)
        if (!(f >> psi[r * n0 + i])) die("short restart file for rank " + std::to_string(r));
    }
  } else {
    quasi_ic ic;
    check(quasi_ic_default(&ic, a.ic), "ic");
    ic.seed = a.seed;
    ic.fc_size = a.fc;
    check(quasi_initial_condition(&cfg, &ic, psi.data()), "initial condition");
  }
  {
    std::ofstream info(a.out + "/info");   // quasi.cpp:609-629
    info << "Nx: " << a.nx << "\nNy: " << a.ny << "\nNz: " << a.nz << "\nPoints per wavelength (nw): " << cfg.nw
         << "\nq0 (z direction): " << cfg.q0 << "\nepsilon: " << -0.001 * a.ep_arg << "\nbeta: " << cfg.beta
         << "\ngamma: " << cfg.gamma << "\nViscosity (nu): " << a.nu << "\ndt: " << cfg.dt
         << "\nstepL1: " << a.step_l1 << "\nstepSave: " << a.step_save << "\ndivv switch: " << cfg.divv_switch
         << "\nInitial amp: " << cfg.amp << "\nkp: " << cfg.kp << "\nrho_0: " << cfg.rho_0
         << "\nFocal conic initial size (fc): " << a.fc << "\n";
  }
  const char* series[] = {"L1", "mass", "energy", "psiMid", "vx", "vy", "vz", "divv", "p", "rho"};
  for (const char* s : series) std::ofstream(a.out + "/" + s + ".dat", std::ios::trunc);

  quasi_handle* h = nullptr;
  check(quasi_create(&cfg, &h), "create");
  check(quasi_set_psi(h, psi.data()), "set_psi");
  check(quasi_init(h), "init");
  auto t0 = std::chrono::steady_clock::now();
  long nloop = 0;
  int count_l1 = 0, count_save = 0;
  double l1 = 1.0;
  std::vector<double> field(n);
  while (a.until_l1 > 0 ? l1 > a.until_l1 : nloop < a.steps) {
    check(quasi_step(h, 1), "step");
    ++nloop;
    if (++count_l1 == a.step_l1) {
      double d[3];
      check(quasi_diagnostics(h, d), "diagnostics");
      l1 = d[0];
      append(a.out + "/L1.dat", &d[0], 1, a.digits);
      append(a.out + "/mass.dat", &d[1], 1, a.digits);
      if (a.variant == QUASI_VARIANT_QUASI) append(a.out + "/energy.dat", &d[2], 1, a.digits);
      count_l1 = 0;
      if (++count_save == a.step_save) {
        count_save = 0;
        check(quasi_get_field(h, QUASI_FIELD_PSI, field.data()), "psi");
        for (int r = 0; r < a.ranks; ++r)
          append(a.out + "/psi" + std::to_string(r) + ".dat", field.data() + r * n0, n0, a.digits, true);
        std::vector<double> s = mid_slice(field, a.nx, a.ny, a.nz);
        append(a.out + "/psiMid.dat", s.data(), s.size(), a.digits);
        const struct { int f; const char* name; } mids[] = {{QUASI_FIELD_VX, "vx"}, {QUASI_FIELD_VY, "vy"},
                                                              {QUASI_FIELD_VZ, "vz"}, {QUASI_FIELD_DIVV, "divv"},
                                                              {QUASI_FIELD_P, "p"}, {QUASI_FIELD_RHO, "rho"}};
        if (a.variant == QUASI_VARIANT_QUASI)
          for (const auto& m : mids) {
            check(quasi_get_field(h, m.f, field.data()), m.name);
            s = mid_slice(field, a.nx, a.ny, a.nz);
            append(a.out + "/" + m.name + ".dat", s.data(), s.size(), a.digits);
          }
      }
    }
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "Finished " << nloop << " steps in " << wall << " seconds [Wall Clock]\n";
  quasi_destroy(h);
  return 0;
}
