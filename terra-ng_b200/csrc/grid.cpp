// Host mesh generation for the thick spherical shell.
//
// Coordinates follow the reference's recursive midpoint refinement of the ten
// icosahedral diamonds (grid/shell/spherical_shell.hpp:276-392, base nodes and
// diamond map :465-604). Here the refinement is evaluated level by level
// instead of by memoised recursion; every node is still the normalised sum of
// the same two parents, so the values are identical. This file must be
// compiled without floating-point contraction (-ffp-contract=off) so that
// `a + b`, `x * x + y * y` etc. are rounded exactly as written, like the
// reference's default (non -march) host build.
#include "tn_grid.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>

namespace tn {
namespace {

struct V3 {
    double v[3];
};

// Vec::normalized (dense/vec.hpp:76-107): divide by sqrt of the left-to-right
// sum of squares, skip when the magnitude is <= 1e-15.
V3 normalized_sum(const V3& a, const V3& b)
{
    V3 m;
    for (int c = 0; c < 3; ++c) m.v[c] = a.v[c] + b.v[c];
    double s = 0.0;
    for (int c = 0; c < 3; ++c) s += m.v[c] * m.v[c];
    const double mag = std::sqrt(s);
    if (mag > 1e-15)
        for (int c = 0; c < 3; ++c) m.v[c] /= mag;
    return m;
}

// Twelve icosahedral base nodes (spherical_shell.hpp:471-515).
std::array<V3, 12> icosahedral_nodes()
{
    std::array<V3, 12> n{};
    const double fifthpi = 0.4 * std::asin(1.0);
    const double w       = 2.0 * std::acos(1.0 / (2.0 * std::sin(fifthpi)));
    const double cosw    = std::cos(w);
    const double sinw    = std::sin(w);
    n[0]                 = {{0.0, 0.0, 1.0}};
    n[11]                = {{0.0, 0.0, -1.0}};
    for (int k = 1; k <= 5; ++k) {
        const double phi = 2.0 * (static_cast<double>(k) - 0.5) * fifthpi;
        n[k]             = {{sinw * std::cos(phi), sinw * std::sin(phi), cosw}};
    }
    for (int k = 1; k <= 5; ++k) {
        const double phi = 2.0 * (static_cast<double>(k) - 1) * fifthpi;
        n[k + 5]         = {{sinw * std::cos(phi), sinw * std::sin(phi), -cosw}};
    }
    return n;
}

// Diamond-to-base-node map, pole first, counter-clockwise (spherical_shell.hpp:521-566).
constexpr int kDiamondNodes[10][4] = {
    {0, 5, 6, 1},   {0, 1, 7, 2},   {0, 2, 8, 3},   {0, 3, 9, 4},  {0, 4, 10, 5},
    {11, 7, 1, 6},  {11, 8, 2, 7},  {11, 9, 3, 8},  {11, 10, 4, 9}, {11, 6, 5, 10},
};

// Corner base nodes of diamond d in the (x, y) frame: {p00, pN0, pNN, p0N}.
// "Left"/"right" swap between hemispheres (spherical_shell.hpp:574-601).
std::array<int, 4> diamond_corners(int d)
{
    const int L = d < 5 ? 1 : 3;
    const int R = d < 5 ? 3 : 1;
    return {kDiamondNodes[d][0], kDiamondNodes[d][L], kDiamondNodes[d][2], kDiamondNodes[d][R]};
}

}  // namespace

void unit_sphere_coords(int lat_level, double* out)
{
    if (lat_level < 0 || lat_level > 12) throw std::invalid_argument("lateral level out of range");
    const int E = 1 << lat_level;  // intervals per side
    const int n = E + 1;
    const auto base = icosahedral_nodes();

    std::vector<V3> g(static_cast<size_t>(n) * n);
    auto at = [&](int i, int j) -> V3& { return g[static_cast<size_t>(i) * n + j]; };

    for (int d = 0; d < 10; ++d) {
        const auto c = diamond_corners(d);
        at(0, 0) = base[c[0]];
        at(E, 0) = base[c[1]];
        at(E, E) = base[c[2]];
        at(0, E) = base[c[3]];
        // Stride l grid -> stride l/2 grid. A node first present on the stride-h
        // grid (h = l/2) is the normalised sum of two stride-l parents:
        //   i%l==0, j%l==h : (i, j-h) + (i, j+h)      horizontal midpoint
        //   i%l==h, j%l==0 : (i-h, j) + (i+h, j)      vertical midpoint
        //   i%l==h, j%l==h : (i-h, j+h) + (i+h, j-h)  anti-diagonal midpoint
        for (int l = E; l >= 2; l /= 2) {
            const int h = l / 2;
            for (int i = 0; i <= E; i += h) {
                for (int j = 0; j <= E; j += h) {
                    const bool ii = (i % l) == 0, jj = (j % l) == 0;
                    if (ii && jj) continue;
                    if (ii)
                        at(i, j) = normalized_sum(at(i, j - h), at(i, j + h));
                    else if (jj)
                        at(i, j) = normalized_sum(at(i - h, j), at(i + h, j));
                    else
                        at(i, j) = normalized_sum(at(i - h, j + h), at(i + h, j - h));
                }
            }
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < 3; ++k)
                    out[((static_cast<size_t>(d) * n + i) * n + j) * 3 + k] = at(i, j).v[k];
    }
}

void uniform_radii(double r_min, double r_max, int num_shells, double* out)
{
    if (num_shells < 2) throw std::invalid_argument("Number of shells must be at least 2.");
    if (r_min >= r_max) throw std::invalid_argument("r_min must be strictly less than r_max.");
    const double r_step = (r_max - r_min) / (num_shells - 1);
    for (int i = 0; i < num_shells; ++i) out[i] = r_min + i * r_step;
    out[num_shells - 1] = r_max;
}

ShellLevel make_shell_level(int lat_level, int rad_level, double r_min, double r_max)
{
    if (lat_level < 0 || lat_level > 10) throw std::invalid_argument("lateral level must be in [0, 10]");
    if (rad_level < 0 || rad_level > 12) throw std::invalid_argument("radial level must be in [0, 12]");
    ShellLevel s;
    s.lat_level = lat_level;
    s.rad_level = rad_level;
    s.nl        = (1 << lat_level) + 1;
    s.nr        = (1 << rad_level) + 1;
    const int n = s.nl;

    s.coords.resize(static_cast<size_t>(10) * n * n * 3);
    unit_sphere_coords(lat_level, s.coords.data());
    s.radii.resize(s.nr);
    uniform_radii(r_min, r_max, s.nr, s.radii.data());

    // Duplicate classes from the diamond-edge topology: every diamond edge
    // joins two base nodes; the node at parameter t along the edge from the
    // lower-numbered base node is the same point in every diamond sharing the
    // edge. Corner nodes are keyed by their base node.
    const int E = n - 1;
    std::map<std::pair<int, int>, std::vector<std::vector<int32_t>>> edge_nodes;
    std::vector<std::vector<int32_t>> vertex_nodes(12);
    auto lat_index = [&](int d, int x, int y) { return static_cast<int32_t>((d * n + x) * n + y); };

    for (int d = 0; d < 10; ++d) {
        const auto c = diamond_corners(d);  // p00, pN0, pNN, p0N
        struct EdgeDef {
            int a, b;   // base nodes at t = 0 and t = E
            int x0, y0; // lattice point at t = 0
            int dx, dy; // lattice step per t
        };
        const EdgeDef edges[4] = {
            {c[0], c[1], 0, 0, 1, 0},   // y = 0:  p00 -> pN0
            {c[3], c[2], 0, E, 1, 0},   // y = E:  p0N -> pNN
            {c[0], c[3], 0, 0, 0, 1},   // x = 0:  p00 -> p0N
            {c[1], c[2], E, 0, 0, 1},   // x = E:  pN0 -> pNN
        };
        for (const auto& e : edges) {
            const auto key = std::make_pair(std::min(e.a, e.b), std::max(e.a, e.b));
            auto& list     = edge_nodes[key];
            if (list.empty()) list.resize(std::max(0, E - 1));
            for (int t = 1; t < E; ++t) {
                const int tp = (e.a < e.b) ? t : E - t;
                list[tp - 1].push_back(lat_index(d, e.x0 + t * e.dx, e.y0 + t * e.dy));
            }
        }
        vertex_nodes[c[0]].push_back(lat_index(d, 0, 0));
        vertex_nodes[c[1]].push_back(lat_index(d, E, 0));
        vertex_nodes[c[2]].push_back(lat_index(d, E, E));
        vertex_nodes[c[3]].push_back(lat_index(d, 0, E));
    }

    s.owned_lat.assign(static_cast<size_t>(10) * n * n, 1);
    s.dup_offset.clear();
    s.dup_members.clear();
    s.dup_offset.push_back(0);
    auto add_class = [&](std::vector<int32_t> m) {
        if (m.size() < 2) return;
        std::sort(m.begin(), m.end());  // ascending lateral index == ascending diamond id
        for (size_t i = 1; i < m.size(); ++i) s.owned_lat[m[i]] = 0;  // owner: lowest diamond
        s.dup_members.insert(s.dup_members.end(), m.begin(), m.end());
        s.dup_offset.push_back(static_cast<int32_t>(s.dup_members.size()));
    };
    for (auto& v : vertex_nodes) add_class(v);
    for (auto& kv : edge_nodes)
        for (auto& m : kv.second) add_class(m);

    // Sanity: the number of owned lateral nodes must equal the number of unique
    // lateral nodes, 10 * E^2 + 2.
    int64_t owned = 0;
    for (auto o : s.owned_lat) owned += o;
    if (owned != 10ll * E * E + 2) throw std::logic_error("ownership count mismatch");
    return s;
}

}  // namespace tn
