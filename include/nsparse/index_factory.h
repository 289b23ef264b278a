// index_factory (reference: nsparse/index_factory.h:16, index_factory.cpp:63-153).
// Descriptions: "brutal", "inverted", "seismic,lambda=..|beta=..|alpha=..|seed=..",
// "seismic_sq,quantizer=8bit|vmin=..|vmax=..|lambda=..|...", "idmap,<delegate>".
#ifndef NSPARSE_B200_INDEX_FACTORY_H
#define NSPARSE_B200_INDEX_FACTORY_H

#include "nsparse/index.h"

namespace nsparse {
Index* index_factory(int dimension, const char* description);
}

#endif
