/* Part of the project-written Kokkos-API shim (test infrastructure): forwards to Kokkos_Core.hpp. */
#pragma once
#include "Kokkos_Core.hpp"
