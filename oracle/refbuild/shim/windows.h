// Stand-in for <windows.h> when compiling the reference's sources with GCC.
// TEST INFRASTRUCTURE (reference cross-check build only).
// The reference relies on the min/max function-like macros that windows.h
// defines.  Every standard header the reference uses is included first so
// that the macros cannot break them, then the macros are defined.
#pragma once
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>
#include <omp.h>
#include <Eigen/Core>
#include <nlohmann/json.hpp>

#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif
