// TEST INFRASTRUCTURE. A declaration-only stand-in for the Boost header that the
// reference's include/global.hpp includes, so that header parses without Boost.
// global.hpp only names boost::multi_array<double, 3> in an alias; the
// reference's Normalizer, the only code compiled against this stand-in, never
// uses it.
#pragma once
#include <cstddef>
namespace boost {
template <typename T, std::size_t N>
class multi_array;
}
