// Laser wakefield acceleration (the set-up of the reference's test driver,
// openmp/em2d/main.cpp:540-607) written against the drop-in C++ headers:
// 1024x128 cells in 32x32 tiles, box 20.48 x 25.6, dt at 0.9 of the Courant
// limit; electrons at 4x4 ppc behind a density step at x = 20.48; a Gaussian
// pulse (a0 1, omega0 10, W0 4, fwhm 2, start 17, focus 20, on axis 12.8,
// Ez polarisation); moving window; compensated 4-pass current filter along x.
// Prints the energy report and the "[benchmark] <x> GPart/s" line, and
// writes Ex/Ey/Ez and the electron charge as ZDF files.
//
//   lwfa [tmax]        tmax defaults to 22
#include "simulation.h"

#include <cstdlib>

int main( int argc, char ** argv ) {
    const float tmax = argc > 1 ? std::atof( argv[1] ) : 22.0f;

    const uint2 cells = make_uint2( 1024, 128 ), nx = make_uint2( 32, 32 );
    const float2 box = make_float2( 20.48f, 25.6f );
    Simulation sim( make_uint2( cells.x / nx.x, cells.y / nx.y ), nx, box, zpic::courant( cells, box ) * 0.9f );

    Species electrons( "electrons", -1.0f, make_uint2( 4, 4 ) );
    electrons.set_density( Density::Step( coord::x, 1.0f, 20.48f ) );
    sim.add_species( electrons );

    Laser::Gaussian pulse;
    pulse.a0 = 1.0f;       pulse.omega0 = 10.0f;
    pulse.W0 = 4.0f;       pulse.fwhm = 2.0f;
    pulse.start = 17.0f;   pulse.focus = 20.0f;
    pulse.axis = 12.8f;    pulse.sin_pol = 1;
    pulse.add( sim.emf );

    sim.set_moving_window();
    sim.current.set_filter( Filter::Compensated( coord::x, 4 ) );

    Timer timer;
    timer.start();
    while ( sim.get_t() < tmax ) sim.advance_mov_window();
    sim.energy_info();        // waits for the GPU
    timer.stop();

    for ( auto c : { fcomp::x, fcomp::y, fcomp::z } ) sim.emf.save( emf::e, c );
    electrons.save_charge();

    std::cout << "[benchmark] " << sim.get_nmove() / timer.elapsed( timer::s ) / 1.e9 << " GPart/s\n"
              << "t = " << sim.get_t() << " after " << sim.get_iter() << " steps, wall time "
              << timer.elapsed( timer::s ) << " s\n";
    return 0;
}
