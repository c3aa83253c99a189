// Weibel instability (the set-up of the reference's test driver,
// openmp/em2d/main.cpp:179-259) written against the drop-in C++ headers:
// 128x128 cells in 8x8 tiles, box 12.8 x 12.8, dt 0.07, electrons and
// positrons at 4x4 ppc with ThermalCorr uth 0.1 and counter-streaming
// uz = +-0.6.  Prints the energy report and the "[benchmark] <x> GPart/s"
// line the reference's benchmark script reads, and writes Bx/By/Bz, the
// electron particles, the electron charge and two electron phase spaces
// (ux; x-uz) as ZDF files.
//
//   weibel [nsteps] [literal]    nsteps < 0 (default) runs to t = 35;
//                                "literal" makes both species electrons
#include "simulation.h"

#include <cstdlib>
#include <cstring>

int main( int argc, char ** argv ) {
    const int nsteps = argc > 1 ? std::atoi( argv[1] ) : -1;
    const bool literal = argc > 2 && std::strcmp( argv[2], "literal" ) == 0;

    const uint2 ntiles = make_uint2( 8, 8 ), nx = make_uint2( 16, 16 );
    const float2 box = make_float2( 12.8f, 12.8f );
    Simulation sim( ntiles, nx, box, 0.07f );
    std::cout << "Weibel: " << ntiles << " tiles of " << nx << " cells, box " << box << '\n';

    const float3 uth = make_float3( 0.1f, 0.1f, 0.1f );
    Species electrons( "electrons", -1.0f, make_uint2( 4, 4 ) );
    electrons.set_udist( UDistribution::ThermalCorr( uth, make_float3( 0, 0, 0.6f ) ) );
    Species positrons( "positrons", literal ? -1.0f : 1.0f, make_uint2( 4, 4 ) );
    positrons.set_udist( UDistribution::ThermalCorr( uth, make_float3( 0, 0, -0.6f ) ) );
    sim.add_species( electrons );
    sim.add_species( positrons );

    Timer timer;
    timer.start();
    if ( nsteps < 0 )
        while ( sim.get_t() <= 35.0 ) sim.advance();
    else
        for ( int n = 0; n < nsteps; n++ ) sim.advance();
    sim.energy_info();        // waits for the GPU
    timer.stop();

    for ( auto c : { fcomp::x, fcomp::y, fcomp::z } ) sim.emf.save( emf::b, c );
    electrons.save();
    electrons.save_charge();
    electrons.save_phasespace( phasespace::ux, make_float2( -1.0f, 1.0f ), 128 );
    electrons.save_phasespace( phasespace::x, make_float2( 0.0f, 12.8f ), 128, phasespace::uz, make_float2( -1.5f, 1.5f ), 96 );

    const double gpart = sim.get_nmove() / timer.elapsed( timer::s ) / 1.e9;
    std::cout << "[benchmark] " << gpart << " GPart/s\n"
              << "steps: " << sim.get_iter() << ", wall time " << timer.elapsed( timer::s ) << " s\n";
    return 0;
}
