#include "Kokkos_Version_Info.hpp"
namespace Kokkos {
namespace Impl {
std::string GIT_BRANCH             = "vendored";
std::string GIT_COMMIT_HASH        = "4.6.01";
std::string GIT_CLEAN_STATUS       = "CLEAN";
std::string GIT_COMMIT_DESCRIPTION = "vendored Kokkos 4.6.01";
std::string GIT_COMMIT_DATE        = "";
}  // namespace Impl
}  // namespace Kokkos
