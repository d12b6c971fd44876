// TEST INFRASTRUCTURE ONLY: the host build of the device's correctly rounded
// exp (bb_pd_b200/csrc/crexp.cuh, pinned against an 80-digit evaluation by
// tests/test_crexp.py), for the oracle's restated exponential law when a
// test selects it (orc_use_cr_exp).
#include "crexp.cuh"

extern "C" double orc_cr_exp(double x) { return bbpd::cr_exp(x); }
