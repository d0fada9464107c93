// Two-cells-per-thread corrective pass (fast arithmetic only), its own
// translation unit so the large kernel compiles in parallel with the rest.
#include "launch.h"
#include "tma.cuh"

#include <type_traits>

namespace mpd {
namespace fast {
#include "kernels_pair.cuh"
}  // namespace fast
}  // namespace mpd
