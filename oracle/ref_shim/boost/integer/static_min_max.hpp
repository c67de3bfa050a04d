// Project-written stand-in for boost/integer/static_min_max.hpp (compile-time
// min/max of two unsigned values), used by the reference's dispatch headers.
#pragma once
namespace boost {
template <unsigned long A, unsigned long B> struct static_unsigned_min { static const unsigned long value = A < B ? A : B; };
template <unsigned long A, unsigned long B> struct static_unsigned_max { static const unsigned long value = A > B ? A : B; };
}
