// TEST INFRASTRUCTURE. A declaration-only stand-in for the Boost header that the
// reference's include/global.hpp includes, so that header parses without Boost.
// global.hpp only names boost::format in a using-declaration; the reference's
// Normalizer (include/normalizer.hpp, src/Misc/Normalizer.cpp), the only code
// compiled against this stand-in, never uses it.
#pragma once
namespace boost {
class format;
}
