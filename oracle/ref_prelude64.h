// Force-included after ref_prelude.h in the FP64 build of the oracle
// (oracle/_ref/liboracle64.so).  TEST INFRASTRUCTURE ONLY.
//
// The reference's physics is written in float (Eigen::Vector3f, Matrix6f,
// float scalars).  Long runs are judged against the same code carried out in
// double: every standard header the reference, the Eigen-API shim and the
// harness use is included first, then `float` is defined as `double`, so the
// unmodified sources that follow (and the shim's fixed-size types, whose
// names keep their `f` suffix) compute in double.  Float literals (1e-6f,
// 0.5f) keep their float values and are widened where they meet a double, so
// the FP64 run uses the FP32 run's constants.  std::clamp/min/max calls that
// mix a double variable with such a literal get the overloads below, which
// have the standard's semantics.  Static assertions are switched off: the
// only one that fails is the renderer's check that its GPU matrix struct of
// floats is 48 bytes (geometry.hpp:45), which the physics never uses.
#pragma once
#include "ref_prelude.h"

#include <atomic>
#include <chrono>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>

namespace std {
inline double clamp(double v, float lo, float hi) { return v < (double)lo ? (double)lo : ((double)hi < v ? (double)hi : v); }
inline double clamp(double v, double lo, float hi) { return v < lo ? lo : ((double)hi < v ? (double)hi : v); }
inline double clamp(double v, float lo, double hi) { return v < (double)lo ? (double)lo : (hi < v ? hi : v); }
inline double max(float a, double b) { return (double)a < b ? b : (double)a; }
inline double max(double a, float b) { return a < (double)b ? (double)b : a; }
inline double min(float a, double b) { return b < (double)a ? b : (double)a; }
inline double min(double a, float b) { return (double)b < a ? (double)b : a; }
}  // namespace std

#define float double
#define static_assert(...) static_assert(true, "")
