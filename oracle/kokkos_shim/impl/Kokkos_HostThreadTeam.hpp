// Kokkos-compatible host shim (oracle test infrastructure): intentionally empty.
#pragma once
