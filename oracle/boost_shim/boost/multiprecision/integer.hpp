// Project-written stand-in: msb/lsb/bit_test live in cpp_int.hpp of this shim.
#pragma once
#include <boost/multiprecision/cpp_int.hpp>
