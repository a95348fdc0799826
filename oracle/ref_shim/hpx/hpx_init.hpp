// Stand-in for <hpx/hpx_init.hpp> (test infrastructure).
#pragma once
#include <hpx/hpx.hpp>

namespace hpx {
inline int init(int, char **) { return 0; }
}  // namespace hpx
