// Host build of cleo_b200/csrc/ddmath.h for tests/test_ddmath.py.
#include "../cleo_b200/csrc/ddmath.h"
extern "C" double dd_pow(double x, double y) { return cleo::dpow(x, y); }
extern "C" double dd_exp(double x) { return cleo::dexp(x); }
