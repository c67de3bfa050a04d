// Project-written stand-in for the one Boost.Math facility that the
// reference's analytic FPR code uses (blocked_bloomfilter/math.hpp:8,40-55):
// the Poisson probability mass function.  TEST INFRASTRUCTURE ONLY: it lets
// the oracle build compile the reference's own FPR loops unchanged.
//
// pdf(k; mean) = exp(k ln(mean) - mean - ln(k!)), evaluated in log space with
// std::lgamma.  Boost rejects a non-positive mean with a domain error; so does
// this stand-in.
#pragma once
#include <cmath>
#include <stdexcept>

namespace boost {
namespace math {

template <class RealType = double, class Policy = void>
class poisson_distribution {
 public:
  explicit poisson_distribution(RealType mean = 1) : mean_(mean) {
    if (!(mean > 0)) throw std::domain_error("poisson_distribution: mean must be > 0");
  }
  RealType mean() const { return mean_; }

 private:
  RealType mean_;
};

template <class RealType, class Policy, class K>
inline RealType pdf(const poisson_distribution<RealType, Policy>& d, const K& k_in) {
  const double k = static_cast<double>(k_in);
  const double m = static_cast<double>(d.mean());
  return static_cast<RealType>(std::exp(k * std::log(m) - m - std::lgamma(k + 1.0)));
}

}  // namespace math
}  // namespace boost
