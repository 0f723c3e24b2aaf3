// Seeded initial conditions on the host (reference layout, doubles).
//   planar      psi = A(z) cos(q0 z),  A(z) = A0/2 (1 - tanh((z - Lz/2)/w))
//   undulated   psi = A(z) cos(q0 z + delta sin(2 pi x/Lx) sin(2 pi y/Ly))
//   interface   psi = A(z - h) cos(q0 (z - h)),  h(x) = eps_h cos(q_h x)
//   droplet     psi = A(r) cos(q0 z),  A(r) = A0/2 (1 - tanh((r - R)/w)),  R = radius_frac L
//   stb         quasi-stb.cpp:549-550: A cos(q0 z) + (A phi/2)(cos(q0 z + Q x) - cos(q0 z - Q x)), phi = 0.1
//   focal_conic quasi.cpp:543-589 (the reference's own "new" IC, size aE = bE = fc_size)
// w = width_wavelengths * 2 pi / q0; A0 = sqrt(9 beta / (10 gamma)) unless amp0 > 0
// (the one-mode coexistence amplitude: 1.8 = 1.34164^2 for the quasi defaults).
// Uniform noise in [-noise, noise) from a splitmix64 stream:
//   u_idx = (splitmix64(seed + (idx+1) * 0x9E3779B97F4A7C15) >> 11) * 2^-53.
#include <cmath>
#include <cstdint>

#include "../../include/quasi_gpu.h"

namespace {

uint64_t splitmix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

double env(double a0, double s, double w) { return a0 * 0.5 * (1.0 - std::tanh(s / w)); }

}  // namespace

extern "C" {

QUASI_API int quasi_ic_default(quasi_ic* ic, int kind) {
  if (!ic || kind < 0 || kind > QUASI_IC_FOCAL_CONIC) return QUASI_ERR_INVALID;
  *ic = quasi_ic{};
  ic->kind = kind;
  ic->seed = 1234;
  ic->noise = kind == QUASI_IC_FOCAL_CONIC ? 0.0 : 1e-3;
  ic->delta = 0.5;
  ic->eps_h = 0.0;
  ic->q_h = 0.0;
  ic->radius_frac = 0.3;
  ic->width_wavelengths = 4.0;
  ic->amp0 = 0.0;
  ic->fc_size = 6.0;
  return QUASI_OK;
}

QUASI_API int quasi_initial_condition(const quasi_config* c, const quasi_ic* ic, double* out) {
  if (!c || !ic || !out || c->nx <= 0 || c->ny <= 0 || c->nz <= 0 || c->nw <= 0 || !(c->q0 > 0))
    return QUASI_ERR_INVALID;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const double dx = (nx * 2.0 * M_PI / (c->q0 * c->nw)) / nx;
  const double dy = (ny * 2.0 * M_PI / (c->q0 * c->nw)) / ny;
  const double dz = (nz * 2.0 * M_PI / (c->q0 * c->nw)) / nz;
  const double lx = nx * dx, ly = ny * dy, lz = nz * dz;
  const double a0 = ic->amp0 > 0 ? ic->amp0 : std::sqrt(9.0 * c->beta / (10.0 * c->gamma));
  const double w = ic->width_wavelengths * 2.0 * M_PI / c->q0;
  const double q0 = c->q0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const double x = i * dx, y = j * dy, z = k * dz;
        double v = 0.0;
        switch (ic->kind) {
          case QUASI_IC_PLANAR:
            v = env(a0, z - lz / 2, w) * std::cos(q0 * z);
            break;
          case QUASI_IC_UNDULATED:
            v = env(a0, z - lz / 2, w) *
                std::cos(q0 * z + ic->delta * std::sin(2 * M_PI * x / lx) * std::sin(2 * M_PI * y / ly));
            break;
          case QUASI_IC_INTERFACE: {
            const double zz = z - ic->eps_h * std::cos(ic->q_h * x);
            v = env(a0, zz - lz / 2, w) * std::cos(q0 * zz);
            break;
          }
          case QUASI_IC_DROPLET: {
            const double rx = x - lx / 2, ry = y - ly / 2, rz = z - lz / 2;
            const double r = std::sqrt(rx * rx + ry * ry + rz * rz);
            const double lmin = std::fmin(lx, std::fmin(ly, lz));
            v = env(a0, r - ic->radius_frac * lmin, w) * std::cos(q0 * z);
            break;
          }
          case QUASI_IC_STB: {
            const double phi = 0.1, amp = c->amp;
            v = amp * std::cos(q0 * k * dz) + (amp * phi / 2) * std::cos(q0 * k * dz + c->q_pert * x) -
                (amp * phi / 2) * std::cos(q0 * k * dz - c->q_pert * x);
            break;
          }
          case QUASI_IC_FOCAL_CONIC: {
            const double mid = double(nx / 2);
            const double ae = ic->fc_size, be = ic->fc_size;
            const double xs = i - mid, ys = j - mid, zs = k;
            const double ds = std::sqrt(xs * xs + ys * ys);
            if (zs < be + 1) {
              if (ds < mid) {
                if (std::sqrt(std::pow((ds - mid) / ae, 2) + std::pow(zs / be, 2)) > 1) v = 0.0;
                else v = c->amp * std::cos(q0 * dz * std::sqrt(std::pow((be / ae) * (ds - mid), 2) + zs * zs));
              } else {
                v = std::fabs(zs) < be ? c->amp * std::cos(q0 * zs * dz) : 0.0;
              }
            }
            break;
          }
          default:
            return QUASI_ERR_INVALID;
        }
        out[(size_t(i) * ny + j) * nz + k] = v;
      }
  if (ic->noise != 0.0) {
    const size_t n = size_t(nx) * ny * nz;
    for (size_t idx = 0; idx < n; ++idx) {
      const uint64_t z = splitmix(ic->seed + (idx + 1) * 0x9E3779B97F4A7C15ULL);
      const double u = double(z >> 11) * (1.0 / 9007199254740992.0);
      out[idx] += (2.0 * u - 1.0) * ic->noise;
    }
  }
  return QUASI_OK;
}

}  // extern "C"
