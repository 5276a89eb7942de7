/* Kokkos configuration for the CPU checker build: Serial + OpenMP host backends, C++20.
 * Written by hand in place of the header Kokkos's CMake would generate; only the
 * settings this build uses are defined. */
#if !defined(KOKKOS_MACROS_HPP) || defined(KOKKOS_CORE_CONFIG_H)
#error "Do not include KokkosCore_config.h directly; include Kokkos_Macros.hpp instead."
#else
#define KOKKOS_CORE_CONFIG_H
#endif
#define KOKKOS_VERSION 40601
#define KOKKOS_VERSION_MAJOR 4
#define KOKKOS_VERSION_MINOR 6
#define KOKKOS_VERSION_PATCH 1
#define KOKKOS_ENABLE_SERIAL
#define KOKKOS_ENABLE_OPENMP
#define KOKKOS_ENABLE_CXX20
#define KOKKOS_ENABLE_LIBDL
