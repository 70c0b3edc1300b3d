// Test infrastructure only (the checker). Included by ref_driver.cpp when it is built
// as cmpmc_ref_crlibm: the reference's calls of std::log, sin, cos, acos, exp, pow, hypot and
// cbrt are routed to correctly rounded values -- the function evaluated in IEEE
// binary128 by libquadmath (error below one binary128 ulp) and rounded once to double.
// While g_crlibm is false (the default; the driver clears it around the generator and
// the lattice build) the platform libm is used, as in the plain reference.
//
// This is the reference with a correctly rounded libm: it differs from the glibc build
// only where glibc 2.39's result is not the double nearest to the exact value.
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <fstream>
#include <functional>
#include <limits>
#include <math.h>
#include <mutex>
#include <numbers>
#include <optional>
#include <quadmath.h>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace cmpmc_oracle {
inline thread_local bool g_crlibm = false;
}

namespace std {
inline double cr_log_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(logq(x)) : ::log(x); }
inline double cr_sin_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(sinq(x)) : ::sin(x); }
inline double cr_cos_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(cosq(x)) : ::cos(x); }
inline double cr_exp_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(expq(x)) : ::exp(x); }
inline double cr_pow_q(double x, double y) {
    return cmpmc_oracle::g_crlibm ? static_cast<double>(powq(x, y)) : ::pow(x, y);
}
inline double cr_hypot_q(double x, double y) {
    return cmpmc_oracle::g_crlibm ? static_cast<double>(hypotq(x, y)) : ::hypot(x, y);
}
inline double cr_cbrt_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(cbrtq(x)) : ::cbrt(x); }
inline double cr_acos_q(double x) { return cmpmc_oracle::g_crlibm ? static_cast<double>(acosq(x)) : ::acos(x); }
inline double cr_atan2_q(double y, double x) {
    return cmpmc_oracle::g_crlibm ? static_cast<double>(atan2q(y, x)) : ::atan2(y, x);
}
}  // namespace std
using std::cr_acos_q;
using std::cr_atan2_q;
using std::cr_cbrt_q;
using std::cr_cos_q;
using std::cr_exp_q;
using std::cr_hypot_q;
using std::cr_log_q;
using std::cr_pow_q;
using std::cr_sin_q;

#define log cr_log_q
#define sin cr_sin_q
#define cos cr_cos_q
#define exp cr_exp_q
#define pow cr_pow_q
#define hypot cr_hypot_q
#define cbrt cr_cbrt_q
#define acos cr_acos_q
#define atan2 cr_atan2_q
