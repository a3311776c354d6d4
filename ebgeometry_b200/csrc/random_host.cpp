// Random::samplePoints (RandomImplem.hpp:27-44): n points uniform in [0,1)^3 from a 64-bit Mersenne
// twister seeded with `seed`, each coordinate a std::uniform_real_distribution<double>(0, 1) draw.
// The reference builds each point with emplace_back(dist(rng), dist(rng), dist(rng)), whose
// argument order C++ leaves to the compiler; GCC, the reference's compiler here, evaluates it right
// to left, so a point's z is the first of its three draws and x the last.  Host only: the point
// sets are inputs that a caller makes once.
#include <cstdint>
#include <random>

#include "capi_common.h"
#include "ebgeometry_b200.h"

extern "C" ebg_status ebg_sample_points(int64_t n, uint64_t seed, double* out_host)
{
  if (n < 0 || (n > 0 && out_host == nullptr)) {
    return ebg::setError(EBG_ERR_INVALID, "null output or negative count");
  }
  std::mt19937_64                        rng(seed);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (int64_t i = 0; i < n; i++) {
    const double first = dist(rng), second = dist(rng), third = dist(rng);
    out_host[3 * i]     = third;
    out_host[3 * i + 1] = second;
    out_host[3 * i + 2] = first;
  }
  return EBG_OK;
}
