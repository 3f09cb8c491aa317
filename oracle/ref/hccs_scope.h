/* Force-included (g++ -include) when the checker compiles the reference's
 * hccs.cpp where it lies.  TEST INFRASTRUCTURE ONLY.
 *
 * hccs.cpp sizes its Thomas work arrays with ibeg/iend before it declares them
 * (hccs.cpp:61-64 and :277-282), which is why the reference does not compile.
 * These namespace-scope names satisfy that first use: the arrays get 65536
 * entries (lines up to 65532 cells), and the function's own ibeg/iend, declared
 * a few lines later, shadow these for everything else.  No line of the
 * reference is changed. */
#ifndef NUC3D_REF_HCCS_SCOPE_H
#define NUC3D_REF_HCCS_SCOPE_H
namespace nuc3d {
static const int ibeg = 0;
static const int iend = 1 << 16;
}  // namespace nuc3d
#endif
