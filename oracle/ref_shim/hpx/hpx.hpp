// Stand-in for <hpx/hpx.hpp> (test infrastructure).
#pragma once
#include <hpx/async.hpp>
#include <string>
#include <vector>

namespace hpx {
inline int finalize() { return 0; }
}  // namespace hpx
