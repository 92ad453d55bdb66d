// Kokkos-API shim — TEST INFRASTRUCTURE ONLY (oracle).  The reference's
// include/matrix.h:15 includes this header and then uses the core Kokkos
// names, so it forwards to the shim's core header.
#pragma once
#include "Kokkos_Core.hpp"
