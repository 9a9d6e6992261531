// Kernel instantiation lists (X-macros).  Generated to match
// template_degree() in dr_types.h; tests/test_native_host.py checks that
// every (class, m, D) the planner can pick appears here.
#pragma once

#define DR_COMPANION_INSTANCES(X) \
    X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 6) X(2, 8) X(2, 12) X(2, 16) \
    X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 6) X(3, 8) X(3, 12) X(3, 16) \
    X(4, 1) X(4, 2) X(4, 3) X(4, 4) X(4, 6) X(4, 8) X(4, 12) X(4, 16) \
    X(5, 1) X(5, 2) X(5, 3) X(5, 4) X(5, 6) X(5, 8) X(5, 12) X(6, 1) \
    X(6, 2) X(6, 3) X(6, 4) X(6, 6) X(6, 8)

#define DR_RATIONAL_INSTANCES(X) \
    X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 6) X(2, 8) X(2, 12) X(2, 16) \
    X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 6) X(3, 8) X(3, 12) X(3, 16) \
    X(4, 1) X(4, 2) X(4, 3) X(4, 4) X(4, 6) X(4, 8) X(4, 12)

#define DR_DENSE_INSTANCES(X) \
    X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 6) X(2, 8) X(2, 12) X(2, 16) \
    X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 6)

// split shadow (integer-difference head + interpreted tail): companion PCFs and
// CMFs of m <= 3 with difference depths up to 8
#define DR_SPLIT_INSTANCES(X) \
    X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 6) X(2, 8) \
    X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 6) X(3, 8)

#define DR_INTERP_INSTANCES(X) X(1, 0) X(2, 0) X(3, 0) X(4, 0) X(5, 0) X(6, 0) X(7, 0) X(8, 0)
