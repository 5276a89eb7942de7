// C entry points around the reference's own FP64 Stokes path, compiled from the reference sources
// (test infrastructure only: the checker and the CPU baseline, never the product).
//
// Every function builds the reference's objects exactly as its application or tests do
// (apps/mantlecirculation/src/stokes_solver.hpp:169-610, tests/test_epsilon_divdiv_stokes.cpp:240-520),
// copies plain host arrays in, runs the reference code, and copies the result out. Array layouts are the
// reference's: nodal fields (10, nl, nl, nr) with r fastest, one block per vector component; coordinates
// (10, nl, nl, 3); radii (10, nr); per-cell fields (10, nl-1, nl-1, nr-1); element matrices
// (10, nl-1, nl-1, nr-1, 2, 18, 18). Boundary-condition codes: 0 Neumann, 1 Dirichlet, 2 free-slip
// (grid/shell/bit_masks.hpp:24-29). Every function returns 0, or -1 with a message (tnr_last_error).
//
// Single process, one rank: the MPI stand-in in mpi_stub/ turns reductions into copies; the interface sum
// over diamond duplicates is the reference's own same-rank communication path.

#include <Kokkos_Core.hpp>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "terra/linalg/vector_q1.hpp"

// ---------------------------------------------------------------------------------------------------------
// Start vectors for the Chebyshev power iteration. The reference draws them from Kokkos's XorShift64 pool
// (power_iteration.hpp:26, grid_operations.hpp:748-773), whose stream depends on backend and thread
// count. A checker that must reproduce another implementation's iterates supplies them instead: this
// overload of terra::linalg::randomize is found by argument-dependent lookup and, as an exact
// non-template match, is preferred over the generic template. It fills the vector from the buffer
// registered for its mesh size, or leaves the reference's own randomize in charge when none is registered.
// ---------------------------------------------------------------------------------------------------------
namespace tnr {
struct StartVectors
{
    std::map< long, const double* > by_size; // key: nodes per component
};
inline StartVectors& start_vectors()
{
    static StartVectors s;
    return s;
}
} // namespace tnr

namespace terra::linalg {
void randomize( VectorQ1Vec< double, 3 >& v );
}

#include "terra/fe/strong_algebraic_dirichlet_enforcement.hpp"
#include "terra/fe/strong_algebraic_freeslip_enforcement.hpp"
#include "terra/fe/wedge/operators/shell/divergence_kerngen.hpp"
#include "terra/fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp"
#include "terra/fe/wedge/operators/shell/epsilon_divdiv_stokes.hpp"
#include "terra/fe/wedge/operators/shell/gradient_kerngen.hpp"
#include "terra/fe/wedge/operators/shell/kmass.hpp"
#include "terra/fe/wedge/operators/shell/prolongation_constant.hpp"
#include "terra/fe/wedge/operators/shell/prolongation_linear.hpp"
#include "terra/fe/wedge/operators/shell/restriction_linear.hpp"
#include "terra/fe/wedge/operators/shell/restriction_constant.hpp"
#include "terra/fe/wedge/operators/shell/vector_mass.hpp"
#include "terra/grid/bit_masks.hpp"
#include "terra/io/xdmf.hpp"
#include "terra/grid/grid_types.hpp"
#include "terra/grid/shell/bit_masks.hpp"
#include "terra/grid/shell/spherical_shell.hpp"
#include "terra/kernels/common/grid_operations.hpp"
#include "terra/linalg/solvers/block_preconditioner_2x2.hpp"
#include "terra/linalg/solvers/chebyshev.hpp"
#include "terra/linalg/solvers/diagonal_solver.hpp"
#include "terra/linalg/solvers/fgmres.hpp"
#include "terra/linalg/solvers/gca/gca.hpp"
#include "terra/linalg/solvers/gca/gca_elements_collector.hpp"
#include "terra/linalg/solvers/multigrid.hpp"
#include "terra/linalg/solvers/pcg.hpp"
#include "terra/linalg/vector_q1isoq2_q1.hpp"
#include "terra/util/table.hpp"

namespace terra::linalg {
void randomize( VectorQ1Vec< double, 3 >& v )
{
    auto&      g = v.grid_data();
    const long n = static_cast< long >( g.comp_[0].size() );
    const auto it = tnr::start_vectors().by_size.find( n );
    if ( it == tnr::start_vectors().by_size.end() )
    {
        v.randomize_impl();
        return;
    }
    for ( int d = 0; d < 3; ++d )
        std::memcpy( g.comp_[d].data(), it->second + d * n, sizeof( double ) * n );
}
} // namespace terra::linalg

using namespace terra;
using grid::Grid2DDataScalar;
using grid::Grid3DDataVec;
using grid::Grid4DDataScalar;
using grid::Grid4DDataVec;
using grid::NodeOwnershipFlag;
using grid::shell::BoundaryConditionFlag;
using grid::shell::BoundaryConditions;
using grid::shell::DistributedDomain;
using grid::shell::ShellBoundaryFlag;
using linalg::VectorQ1IsoQ2Q1;
using linalg::VectorQ1Scalar;
using linalg::VectorQ1Vec;

namespace {

thread_local std::string g_error;

struct Level
{
    std::shared_ptr< DistributedDomain >  domain;
    Grid3DDataVec< double, 3 >            coords;
    Grid2DDataScalar< double >            radii;
    Grid4DDataScalar< NodeOwnershipFlag > owned;
    Grid4DDataScalar< ShellBoundaryFlag > boundary;
    int                                   nl = 0, nr = 0;
    long nodes() const { return 10L * nl * nl * nr; }
    long cells() const { return 10L * ( nl - 1 ) * ( nl - 1 ) * ( nr - 1 ); }
};

// Levels are cached: building a DistributedDomain and its neighbourhoods is set-up work.
Level& level( int lat, int rad, double r_min, double r_max )
{
    static std::map< std::tuple< int, int, double, double >, Level > cache;
    const auto key = std::make_tuple( lat, rad, r_min, r_max );
    auto       it  = cache.find( key );
    if ( it != cache.end() )
        return it->second;
    Level L;
    // one subdomain per diamond, one rank (stokes_solver.hpp: lat_sdr = rad_sdr = 0)
    L.domain   = std::make_shared< DistributedDomain >( DistributedDomain::create_uniform( lat, rad, r_min, r_max, 0, 0 ) );
    L.coords   = grid::shell::subdomain_unit_sphere_single_shell_coords< double >( *L.domain );
    L.radii    = grid::shell::subdomain_shell_radii< double >( *L.domain );
    L.owned    = grid::setup_node_ownership_mask_data( *L.domain );
    L.boundary = grid::shell::setup_boundary_mask_data( *L.domain );
    L.nl       = static_cast< int >( L.owned.extent( 1 ) );
    L.nr       = static_cast< int >( L.owned.extent( 3 ) );
    if ( L.owned.extent( 0 ) != 10 )
        throw std::runtime_error( "expected one subdomain per diamond" );
    return cache.emplace( key, std::move( L ) ).first->second;
}

BoundaryConditionFlag bc_flag( int c )
{
    switch ( c )
    {
    case 0:
        return BoundaryConditionFlag::NEUMANN;
    case 1:
        return BoundaryConditionFlag::DIRICHLET;
    case 2:
        return BoundaryConditionFlag::FREESLIP;
    default:
        throw std::runtime_error( "boundary condition code must be 0, 1 or 2" );
    }
}

void set_bcs( BoundaryConditions& bcs, int bc_cmb, int bc_surface )
{
    bcs[0] = { ShellBoundaryFlag::CMB, bc_flag( bc_cmb ) };
    bcs[1] = { ShellBoundaryFlag::SURFACE, bc_flag( bc_surface ) };
}

void load( const Grid4DDataScalar< double >& v, const double* h )
{
    std::memcpy( v.data(), h, sizeof( double ) * v.size() );
}
void store( const Grid4DDataScalar< double >& v, double* h )
{
    std::memcpy( h, v.data(), sizeof( double ) * v.size() );
}
void load( const Grid4DDataVec< double, 3 >& v, const double* h )
{
    const long n = static_cast< long >( v.comp_[0].size() );
    for ( int d = 0; d < 3; ++d )
        std::memcpy( v.comp_[d].data(), h + d * n, sizeof( double ) * n );
}
void store( const Grid4DDataVec< double, 3 >& v, double* h )
{
    const long n = static_cast< long >( v.comp_[0].size() );
    for ( int d = 0; d < 3; ++d )
        std::memcpy( h + d * n, v.comp_[d].data(), sizeof( double ) * n );
}

Grid4DDataScalar< double > scalar_field( const Level& L, const double* h, const char* name )
{
    Grid4DDataScalar< double > v( std::string( name ), size_t( 10 ), size_t( L.nl ), size_t( L.nl ), size_t( L.nr ) );
    if ( h )
        load( v, h );
    return v;
}

Grid4DDataScalar< double > cell_field( const Level& L, const double* h )
{
    Grid4DDataScalar< double > v( std::string( "k_q0" ), size_t( 10 ), size_t( L.nl - 1 ), size_t( L.nl - 1 ), size_t( L.nr - 1 ) );
    load( v, h );
    return v;
}

// With fewer than 16 OpenMP threads the reference's GradientKerngen picks 1x1x1 team tiles
// (gradient_kerngen.hpp:154-166) and its fast path then reads a one-node coarse-pressure tile where a fine cell
// needs two, giving wrong results. Below that thread count the checker runs the gradient's own slow path
// (force_slow_path), which the reference's tests hold equal to the fast one (test_gradient_fast_vs_slow.cpp).
template < typename G >
void guard_small_teams( G& gradient )
{
    if ( Kokkos::DefaultExecutionSpace().concurrency() < 16 )
        gradient.force_slow_path();
}

// The reference logs its set-up to std::cout (util/logging.hpp); inside a call the stream is pointed at a
// sink so that a host process printing machine-readable lines keeps a clean stdout.
struct NullBuf : std::streambuf
{
    int overflow( int c ) override { return c == EOF ? 0 : c; }
};

template < typename F >
int guarded( F&& f )
{
    static NullBuf  sink;
    std::streambuf* saved = std::cout.rdbuf( &sink );
    int             rc    = 0;
    try
    {
        f();
        Kokkos::fence();
    }
    catch ( const std::exception& e )
    {
        g_error = e.what();
        rc      = -1;
    }
    std::cout.rdbuf( saved );
    return rc;
}

using Viscous  = fe::wedge::operators::shell::EpsilonDivDivKerngen< double >;
using Stokes   = fe::wedge::operators::shell::EpsDivDivStokes< double >;
using Div      = fe::wedge::operators::shell::DivergenceKerngen< double >;
using Grad     = fe::wedge::operators::shell::GradientKerngen< double >;
using PMass    = fe::wedge::operators::shell::KMass< double >;
using VMass    = fe::wedge::operators::shell::VectorMass< double >;
using Prolong  = fe::wedge::operators::shell::ProlongationVecConstant< double >;
using Restrict = fe::wedge::operators::shell::RestrictionVecConstant< double >;

} // namespace

extern "C" {

const char* tnr_last_error()
{
    return g_error.c_str();
}

int tnr_init( int num_threads )
{
    return guarded( [&] {
        if ( !Kokkos::is_initialized() )
        {
            Kokkos::InitializationSettings s;
            if ( num_threads > 0 )
                s.set_num_threads( num_threads );
            s.set_disable_warnings( true );
            Kokkos::initialize( s );
        }
    } );
}

int tnr_num_threads()
{
    return Kokkos::DefaultHostExecutionSpace().concurrency();
}

/// Mesh of one level (spherical_shell.hpp:2599-2640, 2826-2887; bit_masks.hpp). class_rep receives, per node,
/// the smallest global node index among its interface duplicates: the MIN-reduced global-id field with which
/// the reference itself derives ownership (grid/bit_masks.hpp:29-79), taken per node instead of per subdomain.
int tnr_mesh( int lat, int rad, double r_min, double r_max, double* coords, double* radii, uint8_t* boundary,
              uint8_t* owned, int64_t* class_rep )
{
    return guarded( [&] {
        Level& L = level( lat, rad, r_min, r_max );
        if ( coords )
            std::memcpy( coords, L.coords.data(), sizeof( double ) * L.coords.size() );
        if ( radii )
            std::memcpy( radii, L.radii.data(), sizeof( double ) * L.radii.size() );
        if ( boundary )
            std::memcpy( boundary, L.boundary.data(), L.boundary.size() );
        if ( owned )
            std::memcpy( owned, L.owned.data(), L.owned.size() );
        if ( class_rep )
        {
            auto ids = grid::shell::allocate_scalar_grid< int64_t >( "global_node_id", *L.domain );
            for ( const auto& [info, value] : L.domain->subdomains() )
            {
                const int  sd   = std::get< 0 >( value );
                const long base = static_cast< long >( info.diamond_id() ) * L.nl * L.nl * L.nr;
                for ( int x = 0; x < L.nl; ++x )
                    for ( int y = 0; y < L.nl; ++y )
                        for ( int r = 0; r < L.nr; ++r )
                            ids( sd, x, y, r ) = base + ( static_cast< long >( x ) * L.nl + y ) * L.nr + r;
            }
            communication::shell::SubdomainNeighborhoodSendRecvBuffer< int64_t > sb( *L.domain ), rb( *L.domain );
            communication::shell::pack_send_and_recv_local_subdomain_boundaries( *L.domain, ids, sb, rb );
            communication::shell::unpack_and_reduce_local_subdomain_boundaries(
                *L.domain, ids, rb, communication::CommunicationReduction::MIN );
            Kokkos::fence();
            std::memcpy( class_rep, ids.data(), sizeof( int64_t ) * ids.size() );
        }
    } );
}

/// EpsilonDivDivKerngen<double>::apply_impl (epsilon_divdiv_kerngen.hpp:577-792). path 0 lets the operator pick
/// its fast path from the boundary conditions, path 1 forces KernelPath::Slow. k_q0 (per cell) replaces the
/// nodal k when given (set_q0_coefficient_field). add != 0 selects OperatorApplyMode::Add (dst is read),
/// comm == 0 SkipCommunication.
int tnr_epsdivdiv( int lat, double r_min, double r_max, const double* k, const double* k_q0, int bc_cmb,
                   int bc_surface, int diagonal, int path, int add, int comm, const double* src, double* dst )
{
    return guarded( [&] {
        Level&             L  = level( lat, lat, r_min, r_max );
        auto               kk = scalar_field( L, k, "k" );
        BoundaryConditions bcs;
        set_bcs( bcs, bc_cmb, bc_surface );
        Viscous A( *L.domain, L.coords, L.radii, L.boundary, kk, bcs, diagonal != 0 );
        if ( k_q0 )
            A.set_q0_coefficient_field( cell_field( L, k_q0 ) );
        if ( path == 1 )
            A.set_kernel_path( Viscous::KernelPath::Slow );
        A.set_operator_apply_and_communication_modes(
            add ? linalg::OperatorApplyMode::Add : linalg::OperatorApplyMode::Replace,
            comm ? linalg::OperatorCommunicationMode::CommunicateAdditively
                 : linalg::OperatorCommunicationMode::SkipCommunication );
        VectorQ1Vec< double > s( "src", *L.domain, L.owned ), d( "dst", *L.domain, L.owned );
        load( s.grid_data(), src );
        if ( add )
            load( d.grid_data(), dst );
        linalg::apply( A, s, d );
        store( d.grid_data(), dst );
    } );
}

/// DivergenceKerngen<double> (divergence_kerngen.hpp:206-257): u on level lat, p on level lat-1.
int tnr_divergence( int lat, double r_min, double r_max, int bc_cmb, int bc_surface, const double* u, double* p )
{
    return guarded( [&] {
        Level&             F = level( lat, lat, r_min, r_max );
        Level&             C = level( lat - 1, lat - 1, r_min, r_max );
        BoundaryConditions bcs;
        set_bcs( bcs, bc_cmb, bc_surface );
        Div                   B( *F.domain, *C.domain, F.coords, F.radii, F.boundary, bcs );
        VectorQ1Vec< double > s( "u", *F.domain, F.owned );
        VectorQ1Scalar< double > d( "p", *C.domain, C.owned );
        load( s.grid_data(), u );
        linalg::apply( B, s, d );
        store( d.grid_data(), p );
    } );
}

/// GradientKerngen<double> (gradient_kerngen.hpp:207-...): p on level lat-1, u on level lat.
int tnr_gradient( int lat, double r_min, double r_max, int bc_cmb, int bc_surface, const double* p, double* u )
{
    return guarded( [&] {
        Level&             F = level( lat, lat, r_min, r_max );
        Level&             C = level( lat - 1, lat - 1, r_min, r_max );
        BoundaryConditions bcs;
        set_bcs( bcs, bc_cmb, bc_surface );
        Grad                     G( *F.domain, *C.domain, F.coords, F.radii, F.boundary, bcs );
        guard_small_teams( G );
        VectorQ1Scalar< double > s( "p", *C.domain, C.owned );
        VectorQ1Vec< double >    d( "u", *F.domain, F.owned );
        load( s.grid_data(), p );
        linalg::apply( G, s, d );
        store( d.grid_data(), u );
    } );
}

/// Lumped KMass diagonal (kmass.hpp:98-181 with set_lumped_diagonal, applied to ones as stokes_solver.hpp:569-582).
int tnr_kmass_lumped( int lat, double r_min, double r_max, const double* k, double* diag )
{
    return guarded( [&] {
        Level& L = level( lat, lat, r_min, r_max );
        PMass  M( *L.domain, L.coords, L.radii, scalar_field( L, k, "k" ), false );
        M.set_lumped_diagonal( true );
        VectorQ1Scalar< double > ones( "ones", *L.domain, L.owned ), d( "d", *L.domain, L.owned );
        linalg::assign( ones, 1.0 );
        linalg::apply( M, ones, d );
        store( d.grid_data(), diag );
    } );
}

/// VectorMass<double> apply (vector_mass.hpp), as used for the right-hand side (stokes_solver.hpp:660).
int tnr_vector_mass( int lat, double r_min, double r_max, const double* src, double* dst )
{
    return guarded( [&] {
        Level&                L = level( lat, lat, r_min, r_max );
        VMass                 M( *L.domain, L.coords, L.radii, false );
        VectorQ1Vec< double > s( "s", *L.domain, L.owned ), d( "d", *L.domain, L.owned );
        load( s.grid_data(), src );
        linalg::apply( M, s, d );
        store( d.grid_data(), dst );
    } );
}

/// fine += P coarse (ProlongationVecConstant in Add mode, prolongation_constant.hpp:102-192).
int tnr_prolongate_add( int fine_lat, double r_min, double r_max, const double* coarse, double* fine )
{
    return guarded( [&] {
        Level&                F = level( fine_lat, fine_lat, r_min, r_max );
        Level&                C = level( fine_lat - 1, fine_lat - 1, r_min, r_max );
        Prolong               P( linalg::OperatorApplyMode::Add );
        VectorQ1Vec< double > c( "c", *C.domain, C.owned ), f( "f", *F.domain, F.owned );
        load( c.grid_data(), coarse );
        load( f.grid_data(), fine );
        linalg::apply( P, c, f );
        store( f.grid_data(), fine );
    } );
}

/// coarse = R fine (RestrictionVecConstant, restriction_constant.hpp:133-250).
int tnr_restrict( int fine_lat, double r_min, double r_max, const double* fine, double* coarse )
{
    return guarded( [&] {
        Level&                F = level( fine_lat, fine_lat, r_min, r_max );
        Level&                C = level( fine_lat - 1, fine_lat - 1, r_min, r_max );
        Restrict              R( *C.domain );
        VectorQ1Vec< double > f( "f", *F.domain, F.owned ), c( "c", *C.domain, C.owned );
        load( f.grid_data(), fine );
        linalg::apply( R, f, c );
        store( c.grid_data(), coarse );
    } );
}

/// Linear transfers per component (ProlongationLinear in Add mode, prolongation_linear.hpp:14-194;
/// RestrictionLinear with its interface sum, restriction_linear.hpp:16-215); ncomp components, each a
/// contiguous nodal field.
int tnr_prolongate_linear_add( int fine_lat, double r_min, double r_max, int ncomp, const double* coarse, double* fine )
{
    return guarded( [&] {
        Level& F = level( fine_lat, fine_lat, r_min, r_max );
        Level& C = level( fine_lat - 1, fine_lat - 1, r_min, r_max );
        fe::wedge::operators::shell::ProlongationLinear< double > P( F.coords, F.radii, linalg::OperatorApplyMode::Add );
        for ( int c = 0; c < ncomp; ++c )
        {
            VectorQ1Scalar< double > cv( "c", *C.domain, C.owned ), fv( "f", *F.domain, F.owned );
            load( cv.grid_data(), coarse + c * C.nodes() );
            load( fv.grid_data(), fine + c * F.nodes() );
            linalg::apply( P, cv, fv );
            store( fv.grid_data(), fine + c * F.nodes() );
        }
    } );
}

int tnr_restrict_linear( int fine_lat, double r_min, double r_max, int ncomp, const double* fine, double* coarse )
{
    return guarded( [&] {
        Level& F = level( fine_lat, fine_lat, r_min, r_max );
        Level& C = level( fine_lat - 1, fine_lat - 1, r_min, r_max );
        fe::wedge::operators::shell::RestrictionLinear< double > R( *C.domain, F.coords, F.radii );
        for ( int c = 0; c < ncomp; ++c )
        {
            VectorQ1Scalar< double > fv( "f", *F.domain, F.owned ), cv( "c", *C.domain, C.owned );
            load( fv.grid_data(), fine + c * F.nodes() );
            linalg::apply( R, fv, cv );
            store( cv.grid_data(), coarse + c * C.nodes() );
        }
    } );
}

/// Galerkin coarse operators built top-down as the application does (stokes_solver.hpp:375-389): the Neumann
/// operator of level fine_lat with nodal coefficient k, coarsened by TwoGridGCA level by level down to
/// coarse_lat, with InterpolationMode::Linear when linear != 0 (else Constant, the application's default). out
/// receives the element matrices of level coarse_lat.
int tnr_gca( int fine_lat, int coarse_lat, double r_min, double r_max, const double* k, int linear, double* out )
{
    return guarded( [&] {
        if ( coarse_lat >= fine_lat || coarse_lat < 0 )
            throw std::runtime_error( "need 0 <= coarse_lat < fine_lat" );
        const int          n = fine_lat - coarse_lat + 1; // levels coarse_lat .. fine_lat
        BoundaryConditions neumann;
        set_bcs( neumann, 0, 0 );
        Level& F  = level( fine_lat, fine_lat, r_min, r_max );
        auto   kf = scalar_field( F, k, "k" );
        Viscous A_fine( *F.domain, F.coords, F.radii, F.boundary, kf, neumann, false );
        std::vector< Viscous > A_c;
        Level&                 L0 = level( coarse_lat, coarse_lat, r_min, r_max );
        VectorQ1Scalar< double > elements( "GCAElements", *L0.domain, L0.owned );
        linalg::assign( elements, 1.0 );
        for ( int i = 0; i < n - 1; ++i )
        {
            Level& L = level( coarse_lat + i, coarse_lat + i, r_min, r_max );
            A_c.emplace_back( *L.domain, L.coords, L.radii, L.boundary, scalar_field( L, nullptr, "k_c" ), neumann,
                              false );
            A_c.back().set_stored_matrix_mode( linalg::OperatorStoredMatrixMode::Full, i, elements.grid_data() );
        }
        for ( int i = n - 2; i >= 0; --i )
        {
            linalg::solvers::TwoGridGCA< double, Viscous >(
                i == n - 2 ? A_fine : A_c[i + 1], A_c[i], i, elements.grid_data(), true,
                linear ? linalg::solvers::InterpolationMode::Linear : linalg::solvers::InterpolationMode::Constant );
        }
        const int nc = L0.nl - 1, rc = L0.nr - 1;
        long      o  = 0;
        for ( int sd = 0; sd < 10; ++sd )
            for ( int x = 0; x < nc; ++x )
                for ( int y = 0; y < nc; ++y )
                    for ( int r = 0; r < rc; ++r )
                        for ( int w = 0; w < 2; ++w )
                        {
                            const auto m = A_c[0].get_local_matrix( sd, x, y, r, w );
                            for ( int i = 0; i < 18; ++i )
                                for ( int j = 0; j < 18; ++j )
                                    out[o++] = m( i, j );
                        }
    } );
}

/// GCAElementsCollector (gca_elements_collector.hpp:49-103) on level lat with nodal coefficient k: out (one
/// value per cell of level lat - level_range, (10, n-1, n-1, nr-1)) receives the GCAElements entries of those
/// cells (1 where marked, else 0).
int tnr_gca_marks( int lat, int level_range, double r_min, double r_max, const double* k, double* out )
{
    return guarded( [&] {
        if ( level_range < 0 || lat - level_range < 0 )
            throw std::runtime_error( "bad level range" );
        Level& F = level( lat, lat, r_min, r_max );
        Level& C = level( lat - level_range, lat - level_range, r_min, r_max );
        VectorQ1Scalar< double > elements( "GCAElements", *C.domain, C.owned );
        linalg::assign( elements, 0.0 );
        auto kf = scalar_field( F, k, "k" );
        linalg::solvers::GCAElementsCollector< double >( *F.domain, kf, level_range, elements.grid_data() );
        Kokkos::fence();
        const auto& e = elements.grid_data();
        long        o = 0;
        for ( int sd = 0; sd < 10; ++sd )
            for ( int x = 0; x < C.nl - 1; ++x )
                for ( int y = 0; y < C.nl - 1; ++y )
                    for ( int r = 0; r < C.nr - 1; ++r )
                        out[o++] = e( sd, x, y, r );
    } );
}

/// The Stokes solve of the application (stokes_solver.hpp:169-610 set-up, :644-691 solve without the pressure
/// normalisation): FGMRES(restart) with the block-triangular preconditioner; velocity block = Multigrid V-cycles
/// with Chebyshev(order, iterations, power_iterations) smoothing on levels lat-num_levels+1 .. lat, GCA coarse
/// operators when gca != 0 (else the coarse operators take k_levels), PCG(50, 1e-6, 1e-16) on the coarsest
/// level; Schur block = inverse lumped KMass with coefficient k_schur (pressure level). start[l] (optional,
/// coarsest first) are the power-iteration start vectors, 3 components each; the smoothers estimate their
/// spectra on the first solve. tnr_stokes_create builds everything (*setup_seconds: its wall time);
/// tnr_stokes_solve runs FGMRES on b from the initial guess in x (b and x: 3 velocity components on level lat,
/// then pressure on level lat-1), fills history with the relative residual per iteration (history[0] = 1) and
/// *seconds with the wall time of the solve alone.
struct StokesRef
{
    using Smoother   = linalg::solvers::Chebyshev< Viscous >;
    using Coarse     = linalg::solvers::PCG< Viscous >;
    using MG         = linalg::solvers::Multigrid< Viscous, Prolong, Restrict, Smoother, Coarse >;
    using Schur      = linalg::solvers::DiagonalSolver< PMass >;
    using PrecStokes = linalg::solvers::BlockTriangularPreconditioner2x2< Stokes, Viscous, PMass, Grad, MG, Schur >;

    std::vector< Level* >                         lv;
    std::map< long, std::vector< double > >       starts;
    std::shared_ptr< util::Table >                table;
    std::unique_ptr< Stokes >                     K, K_neumann;
    std::vector< Viscous >                        A_c;
    std::vector< Prolong >                        Pv;
    std::vector< Restrict >                       Rv;
    std::vector< VectorQ1Vec< double > >          inv_diag, tmp, tmp2, tmp_r, tmp_e, coarse_tmps;
    std::unique_ptr< Coarse >                     coarse;
    std::unique_ptr< MG >                         mg;
    std::unique_ptr< PMass >                      pmass;
    VectorQ1Scalar< double >                      lumped;
    std::unique_ptr< Schur >                      schur;
    VectorQ1IsoQ2Q1< double >                     prec_tmp;
    std::unique_ptr< PrecStokes >                 prec;
    std::vector< VectorQ1IsoQ2Q1< double > >      ftmp;
    VectorQ1IsoQ2Q1< double >                     xv, bv;
    int                                           restart = 30;
};

int tnr_stokes_create( int lat, int num_levels, double r_min, double r_max, int bc_cmb, int bc_surface,
                       const double* k, const double* const* k_levels, const double* k_schur,
                       const double* const* start, int gca, int restart, int cheb_order, int cheb_iterations,
                       int power_iterations, int vcycles, void** out, double* setup_seconds )
{
    return guarded( [&] {
        const auto t0       = std::chrono::steady_clock::now();
        const int  coarsest = lat - num_levels + 1;
        if ( coarsest < 0 || num_levels < 2 )
            throw std::runtime_error( "bad level range" );
        auto S = std::make_unique< StokesRef >();
        for ( int l = coarsest; l <= lat; ++l )
            S->lv.push_back( &level( l, l, r_min, r_max ) );
        Level&             F = *S->lv.back();
        Level&             P = *S->lv[num_levels - 2];
        BoundaryConditions bcs, neumann;
        set_bcs( bcs, bc_cmb, bc_surface );
        set_bcs( neumann, 0, 0 );
        if ( start )
            for ( int l = 0; l < num_levels; ++l )
                if ( start[l] )
                {
                    const long n = 10L * S->lv[l]->nl * S->lv[l]->nl * S->lv[l]->nr;
                    S->starts[n].assign( start[l], start[l] + 3 * n );
                }

        S->table     = std::make_shared< util::Table >();
        auto kf      = scalar_field( F, k, "eta" );
        S->K         = std::make_unique< Stokes >( *F.domain, *P.domain, F.coords, F.radii, F.boundary, kf, bcs, false );
        S->K_neumann = std::make_unique< Stokes >( *F.domain, *P.domain, F.coords, F.radii, F.boundary, kf, neumann,
                                                   false );
        guard_small_teams( S->K->block_12() );

        Level&                   L0 = *S->lv[0];
        VectorQ1Scalar< double > elements( "GCAElements", *L0.domain, L0.owned );
        linalg::assign( elements, gca == 1 ? 1.0 : 0.0 );
        if ( gca == 2 ) // adaptive GCA (stokes_solver.hpp:278-287)
            linalg::solvers::GCAElementsCollector< double >( *F.domain, kf, num_levels - 1, elements.grid_data() );
        for ( int l = 0; l < num_levels - 1; ++l )
        {
            Level& L = *S->lv[l];
            S->A_c.emplace_back( *L.domain, L.coords, L.radii, L.boundary,
                                 scalar_field( L, k_levels ? k_levels[l] : nullptr, "k_c" ), bcs, false );
            if ( gca )
                S->A_c.back().set_stored_matrix_mode( gca == 2 ? linalg::OperatorStoredMatrixMode::Selective :
                                                                 linalg::OperatorStoredMatrixMode::Full,
                                                      l, elements.grid_data() );
            S->Pv.emplace_back( linalg::OperatorApplyMode::Add );
            S->Rv.emplace_back( *L.domain );
        }
        if ( gca )
            for ( int l = num_levels - 2; l >= 0; --l )
                linalg::solvers::TwoGridGCA< double, Viscous >(
                    l == num_levels - 2 ? S->K_neumann->block_11() : S->A_c[l + 1], S->A_c[l], l,
                    elements.grid_data() );

        for ( int l = 0; l < num_levels; ++l )
        {
            Level& L = *S->lv[l];
            S->tmp.emplace_back( "tmp_mg", *L.domain, L.owned );
            S->tmp2.emplace_back( "tmp_mg_2", *L.domain, L.owned );
            if ( l < num_levels - 1 )
            {
                S->tmp_r.emplace_back( "tmp_mg_r", *L.domain, L.owned );
                S->tmp_e.emplace_back( "tmp_mg_e", *L.domain, L.owned );
            }
            S->inv_diag.emplace_back( "inverse_diagonal", *L.domain, L.owned );
            VectorQ1Vec< double > ones( "ones", *L.domain, L.owned );
            linalg::assign( ones, 1.0 );
            auto& A = ( l == num_levels - 1 ) ? S->K->block_11() : S->A_c[l];
            A.set_diagonal( true );
            linalg::apply( A, ones, S->inv_diag.back() );
            A.set_diagonal( false );
            linalg::invert_entries( S->inv_diag.back() );
        }

        std::vector< StokesRef::Smoother > smoothers;
        for ( int l = 0; l < num_levels; ++l )
            smoothers.emplace_back( cheb_order, S->inv_diag[l],
                                    std::vector< VectorQ1Vec< double > >{ S->tmp[l], S->tmp2[l] }, cheb_iterations,
                                    power_iterations );
        for ( int i = 0; i < 4; ++i )
            S->coarse_tmps.emplace_back( "tmp_coarse_grid", *L0.domain, L0.owned );
        S->coarse = std::make_unique< StokesRef::Coarse >(
            linalg::solvers::IterativeSolverParameters{ 50, 1e-6, 1e-16 }, S->table, S->coarse_tmps );
        S->coarse->set_tag( "coarse_grid_pcg" );
        S->mg = std::make_unique< StokesRef::MG >( S->Pv, S->Rv, S->A_c, S->tmp_r, S->tmp_e, S->tmp, smoothers,
                                                   smoothers, *S->coarse, vcycles, 1e-6 );

        VectorQ1Scalar< double > kp( "k_pm", *P.domain, P.owned );
        load( kp.grid_data(), k_schur );
        S->pmass = std::make_unique< PMass >( *P.domain, P.coords, P.radii, kp.grid_data(), false );
        S->pmass->set_lumped_diagonal( true );
        S->lumped = VectorQ1Scalar< double >( "lumped_diagonal_pmass", *P.domain, P.owned );
        {
            VectorQ1Scalar< double > ones( "ones", *P.domain, P.owned );
            linalg::assign( ones, 1.0 );
            linalg::apply( *S->pmass, ones, S->lumped );
        }
        S->schur    = std::make_unique< StokesRef::Schur >( S->lumped );
        S->prec_tmp = VectorQ1IsoQ2Q1< double >( "triangular_prec_tmp", *F.domain, *P.domain, F.owned, P.owned );
        S->prec     = std::make_unique< StokesRef::PrecStokes >( S->K->block_11(), *S->pmass, S->K->block_12(),
                                                             S->prec_tmp, *S->mg, *S->schur );
        for ( int i = 0; i < 2 * restart + 4; ++i )
            S->ftmp.emplace_back( "stokes_tmp_fgmres", *F.domain, *P.domain, F.owned, P.owned );
        S->xv      = VectorQ1IsoQ2Q1< double >( "u", *F.domain, *P.domain, F.owned, P.owned );
        S->bv      = VectorQ1IsoQ2Q1< double >( "f", *F.domain, *P.domain, F.owned, P.owned );
        S->restart = restart;
        Kokkos::fence();
        *setup_seconds = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
        *out           = S.release();
    } );
}

int tnr_stokes_solve( void* h, double rtol, double atol, int max_it, const double* b, double* x, double* history,
                      int max_hist, int* n_hist, double* seconds )
{
    return guarded( [&] {
        auto*      S  = static_cast< StokesRef* >( h );
        const long nu = S->lv.back()->nodes();
        tnr::start_vectors().by_size.clear();
        for ( const auto& [n, v] : S->starts )
            tnr::start_vectors().by_size[n] = v.data();
        linalg::solvers::FGMRES< Stokes, StokesRef::PrecStokes > fgmres(
            S->ftmp,
            linalg::solvers::FGMRESOptions< double >{ .restart                     = S->restart,
                                                      .relative_residual_tolerance = rtol,
                                                      .absolute_residual_tolerance = atol,
                                                      .max_iterations              = max_it },
            S->table, *S->prec );
        fgmres.set_tag( "stokes_fgmres" );
        S->table->clear();
        load( S->xv.block_1().grid_data(), x );
        load( S->xv.block_2().grid_data(), x + 3 * nu );
        load( S->bv.block_1().grid_data(), b );
        load( S->bv.block_2().grid_data(), b + 3 * nu );
        Kokkos::fence();
        const auto t0 = std::chrono::steady_clock::now();
        linalg::solvers::solve( fgmres, *S->K, S->xv, S->bv );
        Kokkos::fence();
        *seconds = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
        store( S->xv.block_1().grid_data(), x );
        store( S->xv.block_2().grid_data(), x + 3 * nu );
        int n = 0;
        for ( const auto& row : S->table->rows() )
        {
            const auto tag = row.find( "tag" );
            if ( tag == row.end() || util::Table::value_to_string( tag->second ) != "stokes_fgmres" )
                continue;
            const auto rr = row.find( "relative_residual" );
            if ( rr != row.end() && n < max_hist )
                history[n++] = std::get< double >( rr->second );
        }
        *n_hist = n;
        tnr::start_vectors().by_size.clear();
    } );
}

void tnr_stokes_destroy( void* h )
{
    delete static_cast< StokesRef* >( h );
}

/// dst = A_l src with operator l (0 = coarsest) of the velocity hierarchy of a StokesRef (A_c[l], the fine
/// block for l = num_levels - 1), Replace + CommunicateAdditively, in diagonal mode when diagonal != 0.
/// src, dst: 3 components of the level's nodes.
int tnr_stokes_level_apply( void* h, int l, int diagonal, const double* src, double* dst )
{
    return guarded( [&] {
        auto*     S = static_cast< StokesRef* >( h );
        const int n = static_cast< int >( S->lv.size() );
        if ( l < 0 || l >= n )
            throw std::runtime_error( "level out of range" );
        Level&                L = *S->lv[l];
        auto&                 A = ( l == n - 1 ) ? S->K->block_11() : S->A_c[l];
        VectorQ1Vec< double > u( "u", *L.domain, L.owned ), v( "v", *L.domain, L.owned );
        load( u.grid_data(), src );
        A.set_diagonal( diagonal != 0 );
        linalg::apply( A, u, v );
        A.set_diagonal( false );
        Kokkos::fence();
        store( v.grid_data(), dst );
    } );
}

/// Wall time of `reps` consecutive EpsilonDivDivKerngen<double> applies (Replace + CommunicateAdditively, fast
/// path chosen by the boundary conditions) after one warm-up apply, as the reference's operator benchmark
/// times them (apps/benchmarks/performance/benchmark_operators.cpp): seconds[i] per apply.
int tnr_epsdivdiv_time( int lat, double r_min, double r_max, const double* k, int bc_cmb, int bc_surface,
                        const double* src, int reps, double* seconds )
{
    return guarded( [&] {
        Level&             L  = level( lat, lat, r_min, r_max );
        auto               kk = scalar_field( L, k, "k" );
        BoundaryConditions bcs;
        set_bcs( bcs, bc_cmb, bc_surface );
        Viscous               A( *L.domain, L.coords, L.radii, L.boundary, kk, bcs, false );
        VectorQ1Vec< double > s( "src", *L.domain, L.owned ), d( "dst", *L.domain, L.owned );
        load( s.grid_data(), src );
        linalg::apply( A, s, d );
        Kokkos::fence();
        for ( int i = 0; i < reps; ++i )
        {
            const auto t0 = std::chrono::steady_clock::now();
            linalg::apply( A, s, d );
            Kokkos::fence();
            seconds[i] = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
        }
    } );
}

/// Right-hand-side boundary treatment of the application (stokes_solver.hpp:662-671): zero the velocity on the
/// Dirichlet boundary (strong_algebraic_dirichlet_enforcement.hpp:114-123), then remove the normal component on
/// the free-slip boundary (strong_algebraic_freeslip_enforcement.hpp:22-38). f is a Stokes vector (3 velocity
/// components on level lat, pressure on level lat-1), changed in place.
int tnr_rhs_enforce( int lat, double r_min, double r_max, int bc_cmb, int bc_surface, double* f )
{
    return guarded( [&] {
        Level&             F = level( lat, lat, r_min, r_max );
        Level&             P = level( lat - 1, lat - 1, r_min, r_max );
        BoundaryConditions bcs;
        set_bcs( bcs, bc_cmb, bc_surface );
        VectorQ1IsoQ2Q1< double > fv( "f", *F.domain, *P.domain, F.owned, P.owned );
        const long                nu = F.nodes();
        load( fv.block_1().grid_data(), f );
        load( fv.block_2().grid_data(), f + 3 * nu );
        fe::strong_algebraic_homogeneous_velocity_dirichlet_enforcement_stokes_like(
            fv, F.boundary, grid::shell::get_shell_boundary_flag( bcs, BoundaryConditionFlag::DIRICHLET ) );
        fe::strong_algebraic_freeslip_enforcement_in_place(
            fv, F.coords, F.boundary, grid::shell::get_shell_boundary_flag( bcs, BoundaryConditionFlag::FREESLIP ) );
        Kokkos::fence();
        store( fv.block_1().grid_data(), f );
        store( fv.block_2().grid_data(), f + 3 * nu );
    } );
}

/// The reference's XDMFOutput (io/xdmf.hpp) on level lat: one write() of a scalar field and a 3-vector field (FP64
/// data written with out_bytes 4 or 8), geometry in geometry_bytes, into `directory`.
int tnr_xdmf_write( int lat, double r_min, double r_max, const char* directory, int geometry_bytes, const double* scalar,
                    const double* vec, int out_bytes )
{
    return guarded( [&] {
        Level& L = level( lat, lat, r_min, r_max );
        using X  = io::XDMFOutput< double >;
        X xdmf( directory, *L.domain, L.coords, L.radii,
                geometry_bytes == 8 ? X::OutputTypeFloat::Float64 : X::OutputTypeFloat::Float32 );
        const auto ot = out_bytes == 8 ? X::OutputTypeFloat::Float64 : X::OutputTypeFloat::Float32;
        Grid4DDataScalar< double > s( std::string( "temperature" ), size_t( 10 ), size_t( L.nl ), size_t( L.nl ),
                                      size_t( L.nr ) );
        load( s, scalar );
        Grid4DDataVec< double, 3 > v( "velocity", 10, L.nl, L.nl, L.nr );
        load( v, vec );
        xdmf.add( s, ot );
        xdmf.add( v, ot );
        xdmf.write();
    } );
}

} // extern "C"
