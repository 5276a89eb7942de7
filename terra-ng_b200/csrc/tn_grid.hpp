// Host-side thick spherical shell mesh: icosahedral diamonds, radii, boundary
// flags, node ownership and the duplicate-node classes of diamond interfaces.
//
// Layout (identical to the reference's Grid4DDataScalar / Grid4DDataVec with
// Kokkos::LayoutRight, grid/grid_types.hpp:12-113):
//   nodal scalar  (diamond, x, y, r)    r fastest, one array per vector component
//   lateral coords (diamond, x, y, 3)   unit-sphere coordinates
//   radii         (r)                   identical for all ten diamonds
//
// Only the one-subdomain-per-diamond distribution is supported (ten subdomains,
// local subdomain id == diamond id), which is what a single GPU runs.
#pragma once

#include <cstdint>
#include <vector>

namespace tn {

// ShellBoundaryFlag values (grid/shell/bit_masks.hpp:8-16).
enum : uint8_t {
    kFlagInner    = 1u << 0,
    kFlagBoundary = 1u << 1,
    kFlagCMB      = (1u << 1) | (1u << 2),
    kFlagSurface  = (1u << 1) | (1u << 3),
};

// BoundaryConditionFlag values (grid/shell/bit_masks.hpp:20-25).
enum BoundaryCondition : int { kNeumann = 0, kDirichlet = 1, kFreeslip = 2 };

struct ShellLevel {
    int lat_level = 0;   // lateral refinement level of a diamond
    int rad_level = 0;   // radial refinement level (layers = 2^rad_level)
    int nl        = 0;   // nodes per diamond side = 2^lat_level + 1
    int nr        = 0;   // radial nodes = 2^rad_level + 1

    std::vector<double>  coords;     // (10, nl, nl, 3) unit sphere
    std::vector<double>  radii;      // (nr)
    std::vector<uint8_t> owned_lat;  // (10, nl, nl) 1 where this copy owns the node

    // Duplicate-node classes: nodes shared by 2..5 diamonds. For class c the
    // members are dup_members[dup_offset[c] .. dup_offset[c+1]) given as
    // lateral linear indices (d * nl + x) * nl + y. Non-duplicated nodes are
    // not listed.
    std::vector<int32_t> dup_offset;
    std::vector<int32_t> dup_members;

    int64_t num_stored_nodes() const { return 10ll * nl * nl * nr; }
    int64_t num_unique_nodes() const { return (10ll * (nl - 1) * (nl - 1) + 2) * nr; }
};

// Unit-sphere node coordinates of all ten diamonds at lateral level `lat_level`,
// written to out[(d * n + x) * n + y) * 3 + c] with n = 2^lat_level + 1.
void unit_sphere_coords(int lat_level, double* out);

// Uniform shell radii (grid/shell/spherical_shell.hpp:27-52).
void uniform_radii(double r_min, double r_max, int num_shells, double* out);

// Build one level. Throws std::invalid_argument on bad sizes.
ShellLevel make_shell_level(int lat_level, int rad_level, double r_min, double r_max);

// Boundary flag of node (x, y, r): CMB on r == 0, SURFACE on r == nr - 1,
// INNER elsewhere (grid/shell/bit_masks.hpp:99-133).
inline uint8_t boundary_flag(int r, int nr)
{
    if (r == 0) return kFlagCMB;
    if (r == nr - 1) return kFlagSurface;
    return kFlagInner;
}

}  // namespace tn
