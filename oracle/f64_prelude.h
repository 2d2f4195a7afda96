/* Force-included first by the float64 oracle variant (test infrastructure).
 * Standard headers are pulled in before `float` is redefined so library
 * declarations keep their real types; oracle_true_float keeps the 32-bit
 * type for frame I/O in the harness. */
#pragma once
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>
typedef float oracle_true_float;
#define float double
