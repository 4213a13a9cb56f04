//------------------------------------------------------------------------------------------------------------
// Test-infrastructure driver around the reference solver (crockatt/idc-transport-solver, 2-D build).
//
// Linked only into oracle/_ref/libidcref.so by oracle/Makefile.ref.  It is the CHECKER: the tests, the
// golden-fixture generator and the CPU-baseline leg of bench.py call it; nothing in the product does.
//
// It constructs the reference's own objects (DomainDecomposition, OrdinateFlux, CrossSection,
// SweepOperator, SISolver) from plain arrays and calls their public routines:
//   * SweepOperator<RKDG::OrdinateFlux>::Apply   linear_solvers/Abstract/SweepOperator.cpp:118-135
//   * TransportOperator::Pmv / Smv / Lmv         operators/RKDG/TransportOperator.cpp:37, 203, 1215
//   * SISolver<RKDG::OrdinateFlux>::Solve        linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190
//   * IDCIntegrator::Step (non-hybrid)           time_integrators/RKDG/idc.cpp:521, 846-955
//
// Ordinate injection.  The reference has no level-symmetric set (utils/Quadrule/OrdinateSet.cpp:37-59),
// so the driver places the caller's (xi, eta, w) into OrdinateSet's static cache under a private order
// key before any object is built; every object constructed with that key then shares the injected data
// (OrdinateSet::Reconfigure looks the key up first, OrdinateSet.cpp:183-204).  This translation unit is
// compiled with -fno-access-control for that purpose.  Ordinates must already be sorted into the four
// quadrant ranges the reference expects (xi>0,eta>0 | xi>0,eta<0 | xi<0,eta>0 | xi<0,eta<0).
//------------------------------------------------------------------------------------------------------------

# include <chrono>
# include <cmath>
# include <cstring>
# include <limits>
# include <memory>
# include <string>

# include "linear_solvers/Abstract/SweepOperator.hpp"
# include "linear_solvers/Abstract/ImplicitSolver/SISolver.hpp"
# include "objects/DomainDecomposition.hpp"
# include "objects/RKDG/CrossSection.hpp"
# include "objects/RKDG/DensityFunction.hpp"
# include "objects/RKDG/OrdinateFlux.hpp"
# include "operators/RKDG/TransportOperator.hpp"
# include "time_integrators/RKDG/idc.hpp"
# include "utils/ParameterList.hpp"
# include "utils/Quadrule/OrdinateSet.hpp"
# include "utils/global.hpp"

using Quadrule::OrdinateSet;

namespace {

int64_t next_order_key = 1000000;

struct RefProblem {
    int reflect = 0;   // BoundaryEdge bits of the reflecting edges (Global::reflecting_boundaries while in use)
    int sigma_degree = 0;   // DG degree of the cross sections: 0 (piecewise constant) or p
    bool periodic = false;  // Global::periodic while in use
    int64_t nx, ny, p, N, nq;
    int64_t order_key;
    ParameterList plist;
    std::unique_ptr<DomainDecomposition> dd;
    std::unique_ptr<RKDG::CrossSection> sigma_t, sigma_s;
    std::unique_ptr<RKDG::OrdinateFlux> psi, aux;
    std::unique_ptr<RKDG::ScalarFlux> phi;
    std::unique_ptr<SweepOperator<RKDG::OrdinateFlux>> sweep;
    std::unique_ptr<SISolver<RKDG::OrdinateFlux>> si;
    double dt;

    size_t psi_len() const { return (size_t)(nx + 2) * (ny + 2) * nq * N; }
    size_t phi_len() const { return (size_t)(nx + 2) * (ny + 2) * N; }
    size_t sig_len() const {   // values per cross section: one per cell, or (p+1)^2 Legendre moments
        return (size_t)(nx + 2) * (ny + 2) * (sigma_degree ? N : 1);
    }
};

// Installs (xi, eta, w) in the reference's ordinate cache under a fresh key and returns that key.
int64_t InjectOrdinates ( int64_t nq, const double * xi, const double * eta, const double * w ) {

    OrdinateSet::OrdinateData data {};
    data.type = OrdinateSet::OrdinateType::SphericalTriangle;
    data.order = next_order_key++;
    data.num_nodes = nq;
    data.symmetric_reduce = true;
    data.xi_ptr  = new double[nq];
    data.eta_ptr = new double[nq];
    data.mu_ptr  = new double[nq];
    data.phi_ptr = new double[nq];
    data.weights = new double[nq];
    data.reflect_map = nullptr;

    for ( int64_t q = 0; q < nq; ++q ) {
        data.xi_ptr[q]  = xi[q];
        data.eta_ptr[q] = eta[q];
        data.mu_ptr[q]  = std::sqrt( std::max( 0.0, 1.0 - xi[q]*xi[q] - eta[q]*eta[q] ) );
        data.phi_ptr[q] = std::atan2( eta[q], xi[q] );
        data.weights[q] = w[q];
    }
    data.LocateOctants();
    try {   // reflection partners, for reflecting boundaries (level-symmetric sets have them)
        data.ComputeReflectMap();
    } catch ( std::exception & ) {
        data.reflect_map = nullptr;
    }

    OrdinateSet::ordinate_cache.insert(
        std::make_pair( std::make_tuple( data.type, data.order, true ), data ) );

    return data.order;
}

void CopyIn ( Abstract::DensityFunction & f, const double * src, size_t n ) {
    std::memcpy( f.density, src, n * sizeof(double) );
}

void CopyOut ( const Abstract::DensityFunction & f, double * dst, size_t n ) {
    std::memcpy( dst, f.density, n * sizeof(double) );
}

// Global::reflecting_boundaries and Global::periodic of a problem for the duration of a call into the
// reference (it reads the globals in its sweeps, halo operations and solvers), reset afterwards so that other
// problems see neither.
struct ReflectScope {
    explicit ReflectScope ( int mask, bool periodic = false ) {
        Global::reflecting_boundaries = static_cast<BoundaryEdge>( mask );
        Global::periodic = periodic;
    }
    ~ReflectScope () {
        Global::reflecting_boundaries = BoundaryEdge::None;
        Global::periodic = false;
    }
};

} // namespace


extern "C" {

//------------------------------------------------------------------------------------------------------------
// Builds a problem: uniform nx x ny grid on [ax,bx]x[ay,by], DG degree p (tensor Q_p), nq injected
// ordinates, piecewise-constant sigma_t / sigma_s given on the halo-padded (nx+2)(ny+2) cell grid
// (index j + (ny+2)*i), time step dt (+inf for steady state).  sweep_pattern is the reference's key
// ("wavefront" or "sequential").  Returns an opaque handle, or nullptr on error.
//------------------------------------------------------------------------------------------------------------
// reflect: BoundaryEdge bits of reflecting edges; periodic: Global::periodic (deck key `periodic`);
// sigma_degree: 0, or p for high-order cross sections given as
// (p+1)^2 Legendre moments per cell ([cell][u][v], the DensityFunction layout), as Init configures them when the
// deck does not ask for piecewise-constant cross sections (utils/init.cpp:740-745).
void * ref_create_ex ( int64_t nx, int64_t ny, double ax, double bx, double ay, double by, int64_t p,
                       int64_t nq, const double * xi, const double * eta, const double * w,
                       const double * sigma_t, const double * sigma_s, double dt,
                       const char * sweep_pattern, double si_abs_tol, int64_t si_max_its, int reflect,
                       int sigma_degree, int periodic ) {
    try {
        if ( sigma_degree != 0 && sigma_degree != p ) throw std::runtime_error( "sigma_degree must be 0 or p" );
        ReflectScope scope( reflect, periodic != 0 );   // SweepPatternUniCart decides on sequential quadrants when built
        auto * P = new RefProblem();
        P->reflect = reflect;
        P->periodic = periodic != 0;
        P->sigma_degree = sigma_degree;
        P->nx = nx; P->ny = ny; P->p = p; P->N = (p + 1) * (p + 1); P->nq = nq; P->dt = dt;

        Global::DG_degree = p;
        ComputeTPI();

        P->plist.SetValue( "nx", std::to_string(nx) );
        P->plist.SetValue( "ny", std::to_string(ny) );
        P->plist.SetValue( "dg_degree", std::to_string(p) );
        char buf[64];
        std::snprintf( buf, sizeof buf, "%.17g", ax ); P->plist.SetValue( "ax", buf );
        std::snprintf( buf, sizeof buf, "%.17g", bx ); P->plist.SetValue( "bx", buf );
        std::snprintf( buf, sizeof buf, "%.17g", ay ); P->plist.SetValue( "ay", buf );
        std::snprintf( buf, sizeof buf, "%.17g", by ); P->plist.SetValue( "by", buf );
        P->plist.SetValue( "sweep_pattern", sweep_pattern ? sweep_pattern : "wavefront" );
        P->plist.SetValue( "sweep_solve", "gaussian-elimination" );
        P->plist.SetValue( "solve_type", "source-iteration" );
        std::snprintf( buf, sizeof buf, "%.17g", si_abs_tol ); P->plist.SetValue( "abs_tol", buf );
        P->plist.SetValue( "max_its", std::to_string(si_max_its) );

        P->dd.reset( new DomainDecomposition( P->plist ) );

        P->order_key = InjectOrdinates( nq, xi, eta, w );
        OrdinateSet oset( P->order_key, true, OrdinateSet::OrdinateType::SphericalTriangle );

        // default-construct + Reconfigure, the way Init builds them (utils/init.cpp:741-750)
        P->sigma_t.reset( new RKDG::CrossSection() );
        P->sigma_s.reset( new RKDG::CrossSection() );
        P->sigma_t->Reconfigure( *P->dd, sigma_degree );
        P->sigma_s->Reconfigure( *P->dd, sigma_degree );
        CopyIn( *P->sigma_t, sigma_t, P->sig_len() );
        CopyIn( *P->sigma_s, sigma_s, P->sig_len() );
        P->sigma_t->ComputeTensor();
        P->sigma_s->ComputeTensor();

        P->psi.reset( new RKDG::OrdinateFlux() );
        P->aux.reset( new RKDG::OrdinateFlux() );
        P->phi.reset( new RKDG::ScalarFlux() );
        P->psi->Reconfigure( *P->dd, oset, p );
        P->aux->Reconfigure( *P->dd, oset, p );
        P->phi->Reconfigure( *P->dd, p );
        P->psi->ZeroDensity();
        P->aux->ZeroDensity();
        P->phi->ZeroDensity();

        P->sweep.reset( new SweepOperator<RKDG::OrdinateFlux>( *P->dd, oset, P->plist, dt ) );
        P->si.reset( new SISolver<RKDG::OrdinateFlux>( *P->dd, oset, P->plist, dt ) );
        return P;

    } catch ( std::exception & e ) {
        std::fprintf( stderr, "ref_create: %s\n", e.what() );
        return nullptr;
    }
}

// Piecewise-constant cross sections.
void * ref_create_reflecting ( int64_t nx, int64_t ny, double ax, double bx, double ay, double by, int64_t p,
                               int64_t nq, const double * xi, const double * eta, const double * w,
                               const double * sigma_t, const double * sigma_s, double dt,
                               const char * sweep_pattern, double si_abs_tol, int64_t si_max_its, int reflect ) {
    return ref_create_ex( nx, ny, ax, bx, ay, by, p, nq, xi, eta, w, sigma_t, sigma_s, dt, sweep_pattern,
                          si_abs_tol, si_max_its, reflect, 0, 0 );
}

// The same without reflecting boundaries (vacuum or given inflow on every edge).
void * ref_create ( int64_t nx, int64_t ny, double ax, double bx, double ay, double by, int64_t p,
                    int64_t nq, const double * xi, const double * eta, const double * w,
                    const double * sigma_t, const double * sigma_s, double dt,
                    const char * sweep_pattern, double si_abs_tol, int64_t si_max_its ) {
    return ref_create_reflecting( nx, ny, ax, bx, ay, by, p, nq, xi, eta, w, sigma_t, sigma_s, dt, sweep_pattern,
                                  si_abs_tol, si_max_its, 0 );
}

void ref_destroy ( void * h ) { delete static_cast<RefProblem *>(h); }

// SweepOperator::Apply on psi_inout (halo layout, source in / psi out).  *seconds = wall time of Apply.
int ref_apply ( void * h, double * psi_inout, double dt, double * seconds ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->psi, psi_inout, P->psi_len() );
        auto t0 = std::chrono::steady_clock::now();
        P->sweep->Apply( *P->psi, *P->sigma_t, dt );
        auto t1 = std::chrono::steady_clock::now();
        if ( seconds ) *seconds = std::chrono::duration<double>( t1 - t0 ).count();
        CopyOut( *P->psi, psi_inout, P->psi_len() );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_apply: %s\n", e.what() ); return 1; }
}

// Times `reps` back-to-back applications of SweepOperator::Apply to the array already loaded by a
// previous ref_apply (the data is re-loaded before each one so every sweep sees the same source).
int ref_apply_timed ( void * h, const double * source, double dt, int64_t reps, double * seconds ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        double total = 0.0;
        for ( int64_t r = 0; r < reps; ++r ) {
            CopyIn( *P->psi, source, P->psi_len() );
            auto t0 = std::chrono::steady_clock::now();
            P->sweep->Apply( *P->psi, *P->sigma_t, dt );
            auto t1 = std::chrono::steady_clock::now();
            total += std::chrono::duration<double>( t1 - t0 ).count();
        }
        if ( seconds ) *seconds = total;
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_apply_timed: %s\n", e.what() ); return 1; }
}

// phi <- beta*phi + alpha*P psi over interior cells (TransportOperator::Pmv with OpDomain::Interior).
int ref_pmv ( void * h, double alpha, double beta, const double * psi, double * phi ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->psi, psi, P->psi_len() );
        CopyIn( *P->phi, phi, P->phi_len() );
        TransportOperator::Pmv( alpha, beta, *P->psi, *P->phi, OpDomain::Interior );
        CopyOut( *P->phi, phi, P->phi_len() );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_pmv: %s\n", e.what() ); return 1; }
}

// psi <- beta*psi + alpha*S phi over interior cells with sigma_s (TransportOperator::Smv).
int ref_smv ( void * h, double alpha, double beta, const double * phi, double * psi ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->psi, psi, P->psi_len() );
        CopyIn( *P->phi, phi, P->phi_len() );
        TransportOperator::Smv( alpha, beta, *P->sigma_s, *P->phi, *P->psi, OpDomain::Interior );
        CopyOut( *P->psi, psi, P->psi_len() );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_smv: %s\n", e.what() ); return 1; }
}

// y <- beta*y + alpha*L x with sigma_t (TransportOperator::Lmv, out-of-place form).
int ref_lmv ( void * h, double alpha, double beta, const double * x, double * y ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->psi, x, P->psi_len() );
        CopyIn( *P->aux, y, P->psi_len() );
        TransportOperator::Lmv( alpha, beta, *P->sigma_t, *P->psi, *P->aux );
        CopyOut( *P->aux, y, P->psi_len() );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_lmv: %s\n", e.what() ); return 1; }
}

// Source iteration from a zero initial guess (SISolver::Solve); source_inout holds Q on entry and psi on
// return.  *iters and *err report the iteration count and the final absolute l2 change of phi.
int ref_si_solve ( void * h, double * source_inout, double dt, int64_t * iters, double * seconds ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->aux, source_inout, P->psi_len() );
        P->si->SetInitialGuess( nullptr );
        auto t0 = std::chrono::steady_clock::now();
        P->si->Solve( *P->aux, *P->sigma_t, *P->sigma_s, dt, nullptr );
        auto t1 = std::chrono::steady_clock::now();
        if ( seconds ) *seconds = std::chrono::duration<double>( t1 - t0 ).count();
        CopyOut( *P->aux, source_inout, P->psi_len() );
        if ( iters ) *iters = -1;
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_si_solve: %s\n", e.what() ); return 1; }
}

// `steps` time steps of size dt with the reference's own IDC integrator: IDCIntegrator::Create
// (time_integrators/RKDG/idc.cpp:94-102) in the non-hybrid update form (idc_type "update") on
// num_nodes Gauss-Lobatto nodes (SetNodes reads them from Global::input_list, :2305-2381) with
// num_corr corrections; every substep is SISolver::Solve to si_abs_tol (solve_type "source-iteration",
// started from the integrator's initial guess), each step IDCIntegrator::Step (:521-560 ->
// Step_Nonhybrid :846-955).  psi_inout holds psi^0 on entry and psi^steps on return (halo layout; the
// integrator returns the last stage with its ghost cells zeroed); source is q, constant in time, its ghost
// cells the inflow values.
int ref_idc_steps ( void * h, double * psi_inout, const double * source, double dt, int64_t steps,
                    int64_t num_nodes, int64_t num_corr, double si_abs_tol, int64_t si_max_its ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        ParameterList pl = P->plist;
        char buf[64];
        pl.SetValue( "cfl", "1" );   // read by TimeIntegrator's constructor; Step takes the step size itself
        pl.SetValue( "ang_order", std::to_string( P->order_key ) );
        pl.SetValue( "ordinate_type", "spherical-triangle" );   // the type the injected set is cached under
        pl.SetValue( "ordinate_sym_reduce", "true" );
        pl.SetValue( "idc_type", "update" );
        pl.SetValue( "idc_num_corr", std::to_string( num_corr ) );
        pl.SetValue( "hybrid_method", "none" );
        pl.SetValue( "solve_type", "source-iteration" );
        std::snprintf( buf, sizeof buf, "%.17g", si_abs_tol ); pl.SetValue( "abs_tol", buf );
        pl.SetValue( "max_its", std::to_string( si_max_its ) );
        Global::input_list.SetValue( "idc_nodes_type", "gauss-lobatto" );
        Global::input_list.SetValue( "idc_num_nodes", std::to_string( num_nodes ) );

        std::unique_ptr<IDCIntegrator> idc( IDCIntegrator::Create( pl ) );
        OrdinateSet oset( P->order_key, true, OrdinateSet::OrdinateType::SphericalTriangle );
        RKDG::OrdinateFlux psi, src;
        psi.Reconfigure( *P->dd, oset, P->p );
        src.Reconfigure( *P->dd, oset, P->p );
        CopyIn( psi, psi_inout, P->psi_len() );
        CopyIn( src, source, P->psi_len() );
        for ( int64_t n = 0; n < steps; ++n )
            idc->Step( psi, src, *P->sigma_t, *P->sigma_s, dt );
        CopyOut( psi, psi_inout, P->psi_len() );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_idc_steps: %s\n", e.what() ); return 1; }
}

// DensityFunction::WriteToDisk (objects/RKDG/DensityFunction.cpp:2228-2400) of a scalar flux given on the
// halo layout: the reference's .sd2 file.
int ref_write_sd ( void * h, const double * phi, const char * path ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->phi, phi, P->phi_len() );
        P->phi->WriteToDisk( std::string( path ) );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_write_sd: %s\n", e.what() ); return 1; }
}

// OrdinateFlux::WriteToDisk (objects/RKDG/OrdinateFlux.cpp:2720-2930) of an angular flux given on the halo
// layout: the reference's .af2 file.
int ref_write_af ( void * h, const double * psi, const char * path ) {
    auto * P = static_cast<RefProblem *>(h);
    ReflectScope scope( P->reflect, P->periodic );
    try {
        CopyIn( *P->psi, psi, P->psi_len() );
        P->psi->WriteToDisk( std::string( path ) );
        return 0;
    } catch ( std::exception & e ) { std::fprintf( stderr, "ref_write_af: %s\n", e.what() ); return 1; }
}

} // extern "C"
