// Writes one grid file with the drop-in ZDF writer (zpic-parallel_b200/cpp/zdf.h)
// from a raw float32 dense array, for the byte-compatibility test.
//   zdf_write_grid <data.bin> <nx> <ny> <name> <label> <units> <xmin> <xmax> <ymin> <ymax> <iter> <t> <path> [iter_name]
#include "zdf.h"
#include <cstdio>
#include <cstdlib>
#include <vector>

int main( int argc, char ** argv ) {
    if ( argc < 14 ) return 2;
    const unsigned nx = atoi( argv[2] ), ny = atoi( argv[3] );
    std::vector<float> d( (size_t) nx * ny );
    FILE * f = fopen( argv[1], "rb" );
    if ( !f || fread( d.data(), 4, d.size(), f ) != d.size() ) return 3;
    fclose( f );
    zdf::grid_info info;
    info.name = argv[4]; info.label = argv[5]; info.units = argv[6];
    info.ndims = 2; info.count[0] = nx; info.count[1] = ny;
    info.axis = { { "x", 0, atof( argv[7] ), atof( argv[8] ), "x", "c/\\omega_n" },
                  { "y", 0, atof( argv[9] ), atof( argv[10] ), "y", "c/\\omega_n" } };
    zdf::iteration it; it.n = atoi( argv[11] ); it.t = atof( argv[12] ); it.time_units = "1/\\omega_n";
    if ( argc > 14 ) it.name = argv[14];
    return zdf::save_grid( d.data(), info, it, argv[13] ) ? 0 : 1;
}
