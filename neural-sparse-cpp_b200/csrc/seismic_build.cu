// SEISMIC index build on the device.
#include <stdexcept>

#include "index_state.h"

namespace nsparse {
namespace detail {

void seismic_build(SeismicState&, int, const SeismicClusterParameters&) {
    throw std::runtime_error("SEISMIC device build is not available in this build");
}

}  // namespace detail
}  // namespace nsparse
