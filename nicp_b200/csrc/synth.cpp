// synth.cpp -- seeded procedural-room depth renderer (see include/nicp_synth.h).
#include "nicp_synth.h"

#include <cmath>
#include <cstring>

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// uniform in [0, 1) from a 64-bit hash
inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(splitmix64(seed ^ 0xA0761D6478BD642Full)) {}
  double next() { s = splitmix64(s); return u01(s); }
  double range(double a, double b) { return a + (b - a) * next(); }
};

inline double ray_exit_box(const double o[3], const double d[3], const double lo[3], const double hi[3]) {
  double t = 1e300;
  for (int i = 0; i < 3; i++) {
    if (d[i] > 1e-15) t = std::fmin(t, (hi[i] - o[i]) / d[i]);
    else if (d[i] < -1e-15) t = std::fmin(t, (lo[i] - o[i]) / d[i]);
  }
  return t;
}

inline double ray_enter_box(const double o[3], const double d[3], const double lo[3], const double hi[3]) {
  double tn = -1e300, tf = 1e300;
  for (int i = 0; i < 3; i++) {
    if (std::fabs(d[i]) < 1e-15) {
      if (o[i] < lo[i] || o[i] > hi[i]) return -1;
      continue;
    }
    double t1 = (lo[i] - o[i]) / d[i], t2 = (hi[i] - o[i]) / d[i];
    if (t1 > t2) { double x = t1; t1 = t2; t2 = x; }
    tn = std::fmax(tn, t1);
    tf = std::fmin(tf, t2);
  }
  if (tn > tf || tf <= 0) return -1;
  return tn > 0 ? tn : -1;
}

inline double ray_sphere(const double o[3], const double d[3], const double s[4]) {
  double oc[3] = {o[0] - s[0], o[1] - s[1], o[2] - s[2]};
  double a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double b = 2 * (d[0] * oc[0] + d[1] * oc[1] + d[2] * oc[2]);
  double c = oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2] - s[3] * s[3];
  double disc = b * b - 4 * a * c;
  if (disc < 0) return -1;
  double t = (-b - std::sqrt(disc)) / (2 * a);
  return t > 1e-9 ? t : -1;
}

}  // namespace

extern "C" int nicp_synth_scene_make(uint64_t seed, int kind, nicp_synth_scene *out) {
  if (!out) return -1;
  std::memset(out, 0, sizeof(*out));
  Rng rng(seed * 0x100000001B3ull + (uint64_t)kind);
  double zlo, zhi, xy;
  if (kind == NICP_SYNTH_FAR_ROOM) {
    double lo[3] = {-4.0, -2.0, -0.5}, hi[3] = {4.0, 2.0, 8.0};
    std::memcpy(out->room_min, lo, sizeof(lo));
    std::memcpy(out->room_max, hi, sizeof(hi));
    zlo = 0.9; zhi = 7.0; xy = 3.0;
  } else {
    double lo[3] = {-1.5, -1.5, -2.0}, hi[3] = {1.5, 1.5, 2.0};
    std::memcpy(out->room_min, lo, sizeof(lo));
    std::memcpy(out->room_max, hi, sizeof(hi));
    zlo = -0.9; zhi = 1.6; xy = 1.1;
  }
  out->num_spheres = 6;
  for (int i = 0; i < 6; i++) {
    double r = rng.range(0.1, 0.4);
    out->spheres[i][0] = rng.range(-xy, xy);
    out->spheres[i][1] = rng.range(-1.1, 1.1);
    out->spheres[i][2] = rng.range(zlo, zhi);
    out->spheres[i][3] = r;
  }
  out->num_boxes = 4;
  for (int i = 0; i < 4; i++) {
    double c[3] = {rng.range(-xy, xy), rng.range(-1.1, 1.1), rng.range(zlo, zhi)};
    for (int k = 0; k < 3; k++) {
      double h = rng.range(0.1, 0.35);
      out->boxes[i][k] = c[k] - h;
      out->boxes[i][3 + k] = c[k] + h;
    }
  }
  return 0;
}

extern "C" int nicp_synth_render(const nicp_synth_scene *sc, const double *P, float fx, float fy, float cx,
                                 float cy, int rows, int cols, uint64_t noise_seed, double sigma_coef,
                                 double drop_prob, uint16_t *out) {
  if (!sc || !P || !out || rows <= 0 || cols <= 0) return -1;
  const double o[3] = {P[3], P[7], P[11]};
  long long valid = 0;
#pragma omp parallel for schedule(static) reduction(+ : valid)
  for (int r = 0; r < rows; r++) {
    for (int c = 0; c < cols; c++) {
      double dc[3] = {(c - (double)cx) / fx, (r - (double)cy) / fy, 1.0};
      double d[3];
      for (int i = 0; i < 3; i++) d[i] = P[i * 4 + 0] * dc[0] + P[i * 4 + 1] * dc[1] + P[i * 4 + 2] * dc[2];
      double t = ray_exit_box(o, d, sc->room_min, sc->room_max);
      for (int k = 0; k < sc->num_spheres; k++) {
        double ts = ray_sphere(o, d, sc->spheres[k]);
        if (ts > 0 && ts < t) t = ts;
      }
      for (int k = 0; k < sc->num_boxes; k++) {
        double tb = ray_enter_box(o, d, sc->boxes[k], sc->boxes[k] + 3);
        if (tb > 0 && tb < t) t = tb;
      }
      // z-depth along the optical axis (dc has unit z)
      double z = t;
      uint64_t pix = (uint64_t)r * (uint64_t)cols + (uint64_t)c;
      uint64_t h0 = splitmix64(noise_seed ^ splitmix64(pix * 3 + 1));
      uint64_t h1 = splitmix64(h0 + 0x632BE59BD9B4E019ull);
      uint64_t h2 = splitmix64(h1 + 0x8CB92BA72F3D8DD7ull);
      double u1 = u01(h0), u2 = u01(h1);
      if (u1 < 1e-300) u1 = 1e-300;
      double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      z += sigma_coef * z * z * g;
      uint16_t v = 0;
      if (!(u01(h2) < drop_prob) && z > 0 && std::isfinite(z)) {
        double mm = std::floor(z * 1000.0 + 0.5);
        if (mm > 65535.0) mm = 65535.0;
        v = (uint16_t)mm;
      }
      out[(size_t)r * cols + c] = v;
      valid += (v != 0);
    }
  }
  return (int)valid;
}
