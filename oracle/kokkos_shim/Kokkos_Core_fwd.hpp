// Kokkos-compatible host shim (oracle test infrastructure): forward header.
#pragma once
#include <Kokkos_Core.hpp>
