// Minimal stand-in for boost/math/special_functions/binomial.hpp (Boost is not
// installed here).  Only the two functions the reference's solid-harmonic
// code calls are provided; both are exact for the small arguments it uses.
// Test infrastructure only.
#ifndef HFORACLE_BOOST_BINOMIAL_SHIM
#define HFORACLE_BOOST_BINOMIAL_SHIM
namespace boost { namespace math {
template <typename T> T factorial(unsigned n) {
  T r = 1;
  for (unsigned i = 2; i <= n; ++i) r *= static_cast<T>(i);
  return r;
}
template <typename T> T binomial_coefficient(unsigned n, unsigned k) {
  if (k > n) return 0;
  unsigned long long r = 1;
  if (k > n - k) k = n - k;
  for (unsigned i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return static_cast<T>(r);
}
}}  // namespace boost::math
#endif
