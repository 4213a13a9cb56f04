//------------------------------------------------------------------------------------------------------------
// SweepPatternGPU: the reference-side binding of the B200 sweep, as a maintainer of the reference adds it.
//
// A new sweep pattern, registered under the deck key `sweep_pattern gpu-wavefront` through the reference's
// own factory (SweepPatternDerivedFactory, linear_solvers/Abstract/SweepPattern/SweepPattern.cpp:274-306),
// whose Sweep (the virtual of SweepPattern.hpp:117-122) hands the reference's arrays to the C ABI of
// libidcsweep.so (include/idcsweep.h).  SweepOperator::Apply (SweepOperator.cpp:118-135) and everything
// above it -- SISolver, the Peierls solvers, the DIRK and IDC integrators -- call it unchanged.
//
// It needs three one-line additions to the reference's headers, which oracle/plugin_headers.py makes in
// copies under oracle/_ref/plugin_include (the reference tree is not touched):
//   * `class SweepPatternGPU;` among the nested pattern declarations of SweepOperator
//     (linear_solvers/Abstract/SweepOperator.hpp:44-46), as every pattern is a nested class;
//   * `double GetDt() const` in SweepCellSolveBase (Abstract/SweepCellSolve/SweepCellSolveBase.hpp:118)
//     and in SweepCellSolveManager (Abstract/SweepCellSolve/SweepCellSolveManager.hpp:97): Apply hands dt
//     to the cell solvers (SetDt), not to the pattern, and the GPU sweep needs it.
//
// Built by oracle/Makefile.ref into oracle/_ref/libidcref_gpu.so (the reference objects, the test driver
// oracle/ref_driver.cpp and this file, linked against libidcsweep.so).  Test infrastructure: the tests run
// the reference's own solvers through it and compare with the reference's CPU patterns.
//------------------------------------------------------------------------------------------------------------

# include <cstring>
# include <stdexcept>
# include <string>
# include <vector>

# include "idcsweep.h"
# include "linear_solvers/Abstract/SweepOperator.hpp"
# include "linear_solvers/Abstract/SweepPattern/SweepPattern.hpp"
# include "linear_solvers/Abstract/SweepPattern/SweepPatternDerivedFactory.hpp"
# include "linear_solvers/Abstract/SweepPattern/SweepPatternUniCart.hpp"
# include "linear_solvers/Abstract/SweepCellSolve/SweepCellSolveManager.hpp"
# include "objects/RKDG/CrossSection.hpp"
# include "objects/RKDG/OrdinateFlux.hpp"
# include "utils/global.hpp"

namespace {

// The reference reports errors as exceptions; the ABI returns status codes.
void idc_check ( int rc, const char * what ) {
    if ( rc != IDC_OK )
        throw std::runtime_error( std::string( "gpu-wavefront: " ) + what + ": " + idc_strerror( rc ) + ": "
                                  + idc_last_error_message() );
}

} // namespace


template< class OrdinateFlux >
class SweepOperator<OrdinateFlux>::SweepPatternGPU : public SweepOperator<OrdinateFlux>::SweepPatternUniCart {

    friend typename SweepPattern::template SweepPatternDerivedFactory<SweepPatternGPU>;

protected:

    // The grid and the ordinate set are fixed for the SweepOperator's life.  The context is made here for
    // piecewise-constant cross sections (so a missing GPU fails the pattern's construction, as the reference
    // reports errors) and made again at a sweep whose cross sections have the flux's DG degree.
    SweepPatternGPU ( const SweepOperator<OrdinateFlux> & op, const ParameterList & input_list )
        : SweepPatternUniCart( op, input_list ) {

        make_context( 0 );
    }

    void make_context ( int64_t sigma_degree ) const {

        if ( this->ctx ) idc_ctx_destroy( this->ctx );
        this->ctx = nullptr;
        const SweepOperator<OrdinateFlux> & op = this->sw_op;
        idc_problem_desc d {};
        d.nx = op.nx(0);
        d.ny = op.nx(1);
        d.ax = op.ax(0);
        d.bx = op.bx(0);
        d.ay = op.ax(1);
        d.by = op.bx(1);
        d.dg_degree = Global::DG_degree;
        d.sigma_degree = sigma_degree;
        d.device = 0;
        d.flags = 0;
        idc_check( idc_ctx_create( &d, &this->ctx ), "idc_ctx_create" );
        this->ctx_sigma_degree = sigma_degree;

        const int64_t nq = op.nq();
        std::vector<double> xi( nq ), eta( nq ), w( nq );
        for ( int64_t q = 0; q < nq; ++q ) {
            xi[q] = op.xi(q);
            eta[q] = op.eta(q);
            w[q] = op.w(q);
        }
        const int64_t qb[5] = { op.Quadrants(0), op.Quadrants(1), op.Quadrants(2), op.Quadrants(3),
                                op.Quadrants(4) };
        idc_check( idc_set_ordinates( this->ctx, nq, xi.data(), eta.data(), w.data(), qb ), "idc_set_ordinates" );
    }

public:

    ~SweepPatternGPU ( void ) override {  if ( this->ctx ) idc_ctx_destroy( this->ctx );  }

    static const std::string Descriptor ( void ) {  return "gpu-wavefront";  }
    const std::string GetDescriptor ( void ) const override {  return Descriptor();  }

    // SweepPattern::Sweep: result <- L^{-1} source with the inflow values in the ghost cells of `source`.
    void Sweep ( const OrdinateFlux & source, OrdinateFlux & result, const RKDG::CrossSection & sigma,
                 const RKDG::OrdinateFlux * const /* initial_condition: not used by a direct sweep */ ) const override {

        if ( !this->ctx || this->ctx_sigma_degree != sigma.DG_degree ) make_context( sigma.DG_degree );

        // reflecting boundaries (SweepPatternUniCart.cpp:46-88): the library sweeps the quadrants in the same
        // sequence and reflects between them; the BoundaryEdge bits are the ABI's IDC_EDGE_* bits
        idc_check( idc_set_reflecting( this->ctx, static_cast<int32_t>( Global::reflecting_boundaries ) & 15 ),
                   "idc_set_reflecting" );
        idc_check( idc_set_periodic( this->ctx, Global::periodic ? 1 : 0 ), "idc_set_periodic" );
        idc_check( idc_set_sigma( this->ctx, sigma.PointerAtCell( 0, 0 ), nullptr, IDC_LOC_HOST ), "idc_set_sigma" );
        const double dt = this->sw_op.sweep_cell_solve->GetDt();   // set by SweepOperator::Apply
        if ( &source == &result ) {
            idc_check( idc_sweep( this->ctx, result.PointerAtCell( 0, 0 ), dt, nullptr, IDC_PREC_FP64, IDC_LOC_HOST ),
                       "idc_sweep" );
        } else {
            idc_check( idc_sweep_out( this->ctx, source.PointerAtCell( 0, 0 ), result.PointerAtCell( 0, 0 ), dt,
                                      nullptr, IDC_PREC_FP64, IDC_LOC_HOST ), "idc_sweep_out" );
        }
        // the reference's patterns leave the halos dirty on a periodic grid (SweepPatternUniCartWavefront.cpp:324-331),
        // so the next reader synchronises them
        if ( Global::periodic ) result.MarkAllHalosDirty();
    }

private:

    mutable idc_ctx * ctx = nullptr;
    mutable int64_t ctx_sigma_degree = -1;
};


// Registration under "gpu-wavefront", as the reference's own patterns register (SweepPatternUniCartWavefront.cpp,
// end of file).
template class SweepOperator<RKDG::OrdinateFlux>::SweepPatternGPU;
template class SweepOperator<RKDG::OrdinateFlux>::SweepPattern::SweepPatternDerivedFactory<
    SweepOperator<RKDG::OrdinateFlux>::SweepPatternGPU >;
