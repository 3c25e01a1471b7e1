// Seeded synthetic Gaussian-mixture data (host). Stands in for the public
// datasets the reference's scripts name (algorithms/vamana/scripts/*), which
// are not available offline.
//
// Every value is a pure function of (seed, stream, row, dim) through a
// splitmix64 hash, so the data does not depend on thread count or order:
//   centre[c][t]  uint8: lo + (hi - lo) * U(seed, 1, c, t)
//                 float: N(0,1) from U(seed, 1, c, 2t), U(seed, 1, c, 2t+1)
//   comp(row)     U64(seed, 2 + 2*stream, row, 0) mod components
//   noise         N(0,1) from U(seed, 3 + 2*stream, row, 2t) and (.., 2t+1)
//   value         centre + sigma * noise (double); uint8: rounded half away
//                 from zero and clipped to [0,255]; float: the row is
//                 L2-normalised in double then rounded to float.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/parlayann_b200.h"

namespace {

inline uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
inline uint64_t hkey(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b) {
  return mix64(mix64(mix64(seed ^ (stream << 56)) + a) + b);
}
inline double unif(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
inline double normal(uint64_t h1, uint64_t h2) {
  double u1 = unif(h1), u2 = unif(h2);
  return std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586476925286766559 * u2);
}

}  // namespace

extern "C" int pann_synth_mixture(int dtype, uint64_t n, uint32_t d, uint32_t components, uint64_t seed,
                                  uint32_t stream, double lo, double hi, double sigma, int normalize, void* out) {
  if (!out || d == 0 || components == 0 || (dtype != PANN_U8 && dtype != PANN_F32)) return PANN_EINVAL;
  std::vector<double> centres((size_t)components * d);
  for (uint32_t c = 0; c < components; c++)
    for (uint32_t t = 0; t < d; t++) {
      double v;
      if (dtype == PANN_U8) v = lo + (hi - lo) * unif(hkey(seed, 1, c, t));
      else v = normal(hkey(seed, 1, c, 2ull * t), hkey(seed, 1, c, 2ull * t + 1));
      centres[(size_t)c * d + t] = v;
    }
  const uint64_t s_comp = 2 + 2ull * stream, s_noise = 3 + 2ull * stream;
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > 64) nt = 64;
  auto work = [&](unsigned tid) {
    std::vector<double> buf(d);
    for (uint64_t i = tid; i < n; i += nt) {
      uint32_t comp = (uint32_t)(hkey(seed, s_comp, i, 0) % components);
      const double* cen = &centres[(size_t)comp * d];
      for (uint32_t t = 0; t < d; t++)
        buf[t] = cen[t] + sigma * normal(hkey(seed, s_noise, i, 2ull * t), hkey(seed, s_noise, i, 2ull * t + 1));
      if (dtype == PANN_U8) {
        uint8_t* o = static_cast<uint8_t*>(out) + i * d;
        for (uint32_t t = 0; t < d; t++) {
          double r = std::round(buf[t]);
          o[t] = (uint8_t)(r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r));
        }
      } else {
        float* o = static_cast<float*>(out) + i * d;
        double nrm = 1.0;
        if (normalize) {
          double s = 0.0;
          for (uint32_t t = 0; t < d; t++) s += buf[t] * buf[t];
          nrm = std::sqrt(s);
          if (nrm == 0.0) nrm = 1.0;
        }
        for (uint32_t t = 0; t < d; t++) o[t] = (float)(buf[t] / nrm);
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  return PANN_OK;
}
