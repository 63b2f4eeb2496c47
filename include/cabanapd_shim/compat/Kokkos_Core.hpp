// Stand-in for <Kokkos_Core.hpp> so CabanaPD programs build unchanged against
// the cabanapd_b200 front end: add -I include/cabanapd_shim/compat.
#pragma once
#include "../kokkos.hpp"
