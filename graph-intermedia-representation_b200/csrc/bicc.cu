// Per-SCC biconnected blocks (buildBCT, gir.cpp:2063-2089).
#include "common.cuh"

namespace gir {
int bct_build(gir_dev* g) { return fail(g, GIR_ERR_STATE, "buildBCT: not available in this build"); }
}  // namespace gir
