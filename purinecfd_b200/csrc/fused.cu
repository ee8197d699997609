// Fused tiled stage kernels (placeholder until the tiled path lands).
#include "engine.h"
namespace jst {
Engine* make_fused_engine(SolverCore*, std::string& err) {
    err = "fused path not built yet";
    return nullptr;
}
}  // namespace jst
