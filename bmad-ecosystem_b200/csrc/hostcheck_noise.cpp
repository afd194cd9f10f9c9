// hostcheck_noise.cpp -- TEST-ONLY: the host check build with every transcendental result moved
// by one ulp (up or down, chosen by a hash of the argument, for about half of the calls).
// Tracking with it measures how far 1-ulp libm differences alone carry a particle from the
// reference over many turns: the envelope the GPU (whose libm differs from the host's by about
// one ulp) is checked against.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace bmadgpu {
namespace noise {
inline uint64_t bits(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }
inline double nudge(double r, double a, double b) {
  uint64_t h = bits(a) * 0x9E3779B97F4A7C15ull ^ (bits(b) + 0x632BE59BD9B4E019ull);
  h ^= h >> 29;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 32;
  switch (h & 3) {
    case 0: return std::nextafter(r, INFINITY);
    case 1: return std::nextafter(r, -INFINITY);
    default: return r;
  }
}
}  // namespace noise
inline double sin(double x) { return noise::nudge(std::sin(x), x, 1.0); }
inline double cos(double x) { return noise::nudge(std::cos(x), x, 2.0); }
inline double asin(double x) { return noise::nudge(std::asin(x), x, 3.0); }
inline double atan2(double y, double x) { return noise::nudge(std::atan2(y, x), y, x); }
inline double sinh(double x) { return noise::nudge(std::sinh(x), x, 4.0); }
inline double cosh(double x) { return noise::nudge(std::cosh(x), x, 5.0); }
}  // namespace bmadgpu

#define bmadgpu_hostcheck_track bmadgpu_hostcheck_noise_track
#define bmadgpu_hostcheck_last_error bmadgpu_hostcheck_noise_last_error
#include "hostcheck.cpp"
