// Stand-in for the reference's hccs scheme.  TEST INFRASTRUCTURE ONLY.
// The reference's hccs.cpp does not compile (it uses ibeg/iend before
// declaring them, hccs.cpp:61-64), yet fieldOperator.cpp instantiates the
// class by name.  This file gives the class its vtable so the facade links;
// selecting "hccs" in Method.in stops the checker loudly.
#include "hccs.hpp"

#include <cstdio>
#include <cstdlib>

namespace {
[[noreturn]] void no_hccs() {
    std::fprintf(stderr, "reference checker: the reference's hccs scheme does not compile\n");
    std::exit(95);
}
}  // namespace

nuc3d::hccs::hccs() : ss(1.0e-6), p(2) {}
nuc3d::hccs::~hccs() {}
void nuc3d::hccs::interpolationInner(const Field &, const int, Field &, const int) { no_hccs(); }
void nuc3d::hccs::interpolationBoundaryL(const Field &, const Field &, const int, Field &,
                                         const int) {
    no_hccs();
}
void nuc3d::hccs::interpolationBoundaryR(const Field &, const Field &, const int, Field &,
                                         const int) {
    no_hccs();
}
