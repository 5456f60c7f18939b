// Strongly connected components + condensation DAG (buildSCC_DAG, gir.cpp:798-839).
#include "common.cuh"

namespace gir {
int scc_build(gir_dev* g) { return fail(g, GIR_ERR_STATE, "buildSCC_DAG: not available in this build"); }
}  // namespace gir
