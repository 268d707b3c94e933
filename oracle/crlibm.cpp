// crlibm.cpp — correctly rounded pow and exp for the oracle's second build (TEST INFRASTRUCTURE).
//
// liboracle_cr.so is the oracle compiled with ORACLE_CR_LIBM: its pow and exp calls come here
// instead of the host libm. These are the double-double evaluations of cleo_b200/csrc/ddmath.h
// built for the host, whose correct rounding tests/test_ddmath.py checks against 60-digit
// decimal arithmetic. With them the oracle computes the arithmetic that the CUDA path documents
// (every pow and exp correctly rounded), so the two can be compared bit for bit; the host-libm
// build, liboracle.so, pins the restatement to CLEO's own sources.
#include <cstdint>

#include "../cleo_b200/csrc/ddmath.h"

extern "C" double oc_cr_pow(double x, double y) { return cleo::dpow(x, y); }
extern "C" double oc_cr_exp(double x) { return cleo::dexp(x); }
