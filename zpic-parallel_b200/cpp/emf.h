// emf.h -- EMF (emf.h:24-197 of the reference) over libzpic_b200.so
#ifndef ZPIC_B200_EMF_H_
#define ZPIC_B200_EMF_H_

#include "zpic.h"
#include "vec3grid.h"
#include "current.h"
#include "moving_window.h"

namespace emf {
enum field { e = 0, b };
namespace bc { enum type { none = 0, periodic, pec, pmc }; }
typedef bnd<bc::type> bc_type;
}

class EMF {
    zpic_sim * h_;
    emf::bc_type bc;
    const float2 dx;
    const double dt;
    int iter;
    MovingWindow moving_window;
public:
    vec3grid<float3> * E;
    vec3grid<float3> * B;
    const float2 box;

    EMF( zpic_sim * h, uint2 const ntiles, uint2 const nx, float2 const box, double const dt ) :
        h_( h ), bc( emf::bc::periodic ), dx( make_float2( box.x / ( nx.x * ntiles.x ), box.y / ( nx.y * ntiles.y ) ) ),
        dt( dt ), iter( 0 ), box( box ) {
        E = new vec3grid<float3>( h, ZPIC_GRID_E, ntiles, nx );
        E->name = "Electric field";
        B = new vec3grid<float3>( h, ZPIC_GRID_B, ntiles, nx );
        B->name = "Magnetic field";
    }
    ~EMF() { delete E; delete B; }

    zpic_sim * handle() const { return h_; }
    auto get_iter() { return iter; }
    auto get_dt() { return dt; }
    emf::bc_type get_bc() { return bc; }

    void set_bc( emf::bc_type new_bc ) {
        const int32_t b[4] = { new_bc.x.lower, new_bc.x.upper, new_bc.y.lower, new_bc.y.upper };
        zpic::check( zpic_b200_emf_set_bc( h_, b ) );
        bc = new_bc;
        std::string bc_name[] = { "none", "periodic", "pec", "pmc" };
        std::cout << "(*info*) EMF boundary conditions\n";
        std::cout << "(*info*) x : [ " << bc_name[bc.x.lower] << ", " << bc_name[bc.x.upper] << " ]\n";
        std::cout << "(*info*) y : [ " << bc_name[bc.y.lower] << ", " << bc_name[bc.y.upper] << " ]\n";
    }

    int set_moving_window() {
        if ( iter != 0 ) { std::cerr << "(*error*) set_moving_window() called with iter != 0\n"; return -1; }
        moving_window.init( dx.x );
        bc.x.lower = bc.x.upper = emf::bc::none;
        return 0;
    }

    void advance() { zpic::check( zpic_b200_emf_advance( h_, 0 ) ); step_bookkeeping(); }
    void advance( Current & ) { zpic::check( zpic_b200_emf_advance( h_, 1 ) ); step_bookkeeping(); }

    void step_bookkeeping() {
        iter += 1;
        if ( moving_window.active() && moving_window.needs_move( iter * dt ) ) moving_window.advance();
    }

    // EMF::save (emf.cpp:593-655)
    void save( emf::field const field, fcomp::cart const fc ) {
        const char comp[] = { 'x', 'y', 'z' };
        zdf::grid_info info;
        info.name = std::string( field == emf::e ? "E" : "B" ) + comp[fc];
        info.label = std::string( field == emf::e ? "E_" : "B_" ) + comp[fc];
        info.units = "m_e c \\omega_n e^{-1}";
        info.axis = { { "x", 0, 0.0 + moving_window.motion(), box.x + moving_window.motion(), "x", "c/\\omega_n" },
                      { "y", 0, 0.0, box.y, "y", "c/\\omega_n" } };
        zdf::iteration it; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        ( field == emf::e ? E : B )->save( fc, info, it, "EMF" );
    }

    // EMF::get_energy (emf.cpp:662-713)
    void get_energy( double3 & ene_E, double3 & ene_B ) {
        double e[3], b[3];
        zpic::check( zpic_b200_emf_energy( h_, e, b ) );
        ene_E = make_double3( e[0], e[1], e[2] );
        ene_B = make_double3( b[0], b[1], b[2] );
    }
};

#endif
