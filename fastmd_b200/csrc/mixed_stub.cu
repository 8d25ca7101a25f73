#include "engine.h"
namespace fmd {
std::unique_ptr<SimEngine> make_mixed_engine(const RunConfig&, Topology, const fmd_melt_spec*) {
  throw Error(FMD_ERR_STATE, "mixed form not built yet");
}
}
