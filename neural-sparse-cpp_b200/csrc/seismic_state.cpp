// Host/device synchronisation of the SEISMIC lists held by an index.
#include <mutex>

#include "index_state.h"

namespace nsparse {
namespace detail {

void SeismicState::ensure_lists() {
    std::lock_guard<std::mutex> g(mu);
    if (!dev_valid && host_valid) {
        lists_dev.upload(lists, vectors.host.dim);
        dev_valid = true;
    }
    if (dev_valid) lists_dev.bind_rows(vectors.dev, nsp::Workspace::get().stream());
}

const nsp::SeismicHost& SeismicState::host_lists() {
    std::lock_guard<std::mutex> g(mu);
    if (!host_valid && dev_valid) {
        lists_dev.download(lists);
        host_valid = true;
    }
    return lists;
}

}  // namespace detail
}  // namespace nsparse
