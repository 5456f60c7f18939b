// C++ GIR class over the gir_dev C ABI (placeholder until the class lands).
#include "gir_b200.hpp"
