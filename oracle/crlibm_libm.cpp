// Test infrastructure only (the checker). A correctly rounded libm for the oracle programs:
// linked into cmpmc_ref_crlibm and shim_example, these definitions of log, sin, cos,
// sincos, exp, pow, hypot, cbrt, acos and atan2 take the place of the platform's (glibc's)
// for every call in the program, including those the compiler emits for the reference's
// own code. The reference's headers are compiled exactly as in the unmodified build; only
// the libm they are linked against differs.
//
// While the calling thread's flag is on (cmpmc_oracle_set_crlibm(1)), each function is
// evaluated in IEEE binary128 by libquadmath (error below one binary128 ulp) and rounded
// once to double: the correctly rounded result except where the exact value lies within a
// binary128 ulp of a rounding boundary. While it is off (the default; the drivers turn it
// off around the host generators and the lattice build, which run on the host in the
// device path too) the platform's function is called.
#include <dlfcn.h>
#include <quadmath.h>

#include <cstdlib>

namespace {

thread_local int g_on = 0;

template <class F>
F platform(const char* name) {
    void* f = dlsym(RTLD_NEXT, name);
    if (!f) std::abort();
    return reinterpret_cast<F>(f);
}

using F1 = double (*)(double);
using F2 = double (*)(double, double);
using FSC = void (*)(double, double*, double*);

}  // namespace

extern "C" {

void cmpmc_oracle_set_crlibm(int on) { g_on = on; }

double log(double x) {
    static const F1 f = platform<F1>("log");
    return g_on ? static_cast<double>(logq(x)) : f(x);
}
double sin(double x) {
    static const F1 f = platform<F1>("sin");
    return g_on ? static_cast<double>(sinq(x)) : f(x);
}
double cos(double x) {
    static const F1 f = platform<F1>("cos");
    return g_on ? static_cast<double>(cosq(x)) : f(x);
}
void sincos(double x, double* s, double* c) {
    static const FSC f = platform<FSC>("sincos");
    if (g_on) {
        *s = static_cast<double>(sinq(x));
        *c = static_cast<double>(cosq(x));
    } else {
        f(x, s, c);
    }
}
double exp(double x) {
    static const F1 f = platform<F1>("exp");
    return g_on ? static_cast<double>(expq(x)) : f(x);
}
double pow(double x, double y) {
    static const F2 f = platform<F2>("pow");
    return g_on ? static_cast<double>(powq(x, y)) : f(x, y);
}
double hypot(double x, double y) {
    static const F2 f = platform<F2>("hypot");
    return g_on ? static_cast<double>(hypotq(x, y)) : f(x, y);
}
double cbrt(double x) {
    static const F1 f = platform<F1>("cbrt");
    return g_on ? static_cast<double>(cbrtq(x)) : f(x);
}
double acos(double x) {
    static const F1 f = platform<F1>("acos");
    return g_on ? static_cast<double>(acosq(x)) : f(x);
}
double atan2(double y, double x) {
    static const F2 f = platform<F2>("atan2");
    return g_on ? static_cast<double>(atan2q(y, x)) : f(y, x);
}

}  // extern "C"
