// zdf.h -- writer for ZDF diagnostic files (the reference's zdf.c / zdf-cpp.h
// format): grid files "<path>/<name>-<iter:06>.zdf" and particle files
// "<path>/particles-<name>-<iter:06>.zdf", readable by the reference's zdf.py.
//
// Record layout (kept alike for compatibility): "ZDF1" magic; records of
// {uint32 id, string name, uint64 length, payload}; strings are uint32 length
// + bytes padded to 4; little-endian.
#ifndef ZPIC_B200_ZDF_H_
#define ZPIC_B200_ZDF_H_

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <sys/stat.h>

namespace zdf {

enum data_type { null_t = 0, int8, uint8, int16, uint16, int32, uint32, int64, uint64, float32, float64 };

struct grid_axis {
    std::string name; int type = 0; double min = 0, max = 0; std::string label, units;
};
struct grid_info {
    std::string name; uint32_t ndims = 2; uint64_t count[3] = { 0, 0, 0 };
    std::string label, units; std::vector<grid_axis> axis;
};
struct iteration {
    std::string name; int32_t n = 0; double t = 0; std::string time_units;
};
struct part_info {
    std::string name, label; uint64_t np = 0;
    std::vector<std::string> quants, qlabels, qunits;
};

constexpr uint32_t INT32_ID = 0x00010000, DOUBLE_ID = 0x00020000, STRING_ID = 0x00030000;
constexpr uint32_t DATASET_ID = 0x00100002, ITERATION_ID = 0x00200001, GRID_INFO_ID = 0x00210001;
constexpr uint32_t PART_INFO_ID = 0x00220002;

inline size_t rndup4( size_t n ) { return ( n + 3 ) / 4 * 4; }
inline size_t str_size( const std::string & s ) { return 4 + ( s.empty() ? 0 : rndup4( s.size() ) ); }

// mkdir -p
inline int create_path( const std::string & path ) {
    if ( path.empty() ) return 0;
    std::string cur;
    size_t p = 0;
    while ( p != std::string::npos ) {
        p = path.find( '/', p + 1 );
        cur = path.substr( 0, p );
        if ( mkdir( cur.c_str(), S_IRWXU | S_IRGRP | S_IXGRP | S_IROTH | S_IXOTH ) && errno != EEXIST ) return errno;
    }
    return 0;
}

class file {
    FILE * fp = nullptr;
    uint32_t ndatasets = 0;
    void put( const void * p, size_t n ) { if ( n ) fwrite( p, 1, n, fp ); }
    void u32( uint32_t v ) { put( &v, 4 ); }
    void i32( int32_t v ) { put( &v, 4 ); }
    void u64( uint64_t v ) { put( &v, 8 ); }
    void f64( double v ) { put( &v, 8 ); }
    void str( const std::string & s ) {
        u32( (uint32_t) s.size() );
        put( s.data(), s.size() );
        static const char pad[4] = { 0, 0, 0, 0 };
        put( pad, rndup4( s.size() ) - s.size() );
    }
    void record( uint32_t id, const std::string & name, uint64_t len ) { u32( id ); str( name ); u64( len ); }
public:
    bool open( const std::string & filename ) {
        fp = fopen( filename.c_str(), "w+b" );
        if ( !fp ) { perror( "(*error*) Unable to open ZDF file for writing" ); return false; }
        put( "ZDF1", 4 );
        return true;
    }
    void close() { if ( fp ) fclose( fp ); fp = nullptr; }
    ~file() { close(); }
    void add_string( const std::string & name, const std::string & s ) { record( STRING_ID, name, str_size( s ) ); str( s ); }
    void add_iteration( const iteration & it ) {
        record( ITERATION_ID, it.name.empty() ? "Iteration" : it.name, 4 + 8 + str_size( it.time_units ) );
        i32( it.n ); f64( it.t ); str( it.time_units );
    }
    void add_grid_info( const grid_info & g ) {
        size_t len = 4 + g.ndims * 8 + str_size( g.label ) + str_size( g.units ) + 4;
        for ( unsigned i = 0; i < g.ndims && !g.axis.empty(); i++ )
            len += str_size( g.axis[i].name ) + 4 + 16 + str_size( g.axis[i].label ) + str_size( g.axis[i].units );
        record( GRID_INFO_ID, g.name, len );
        u32( g.ndims );
        for ( unsigned i = 0; i < g.ndims; i++ ) u64( g.count[i] );
        str( g.label ); str( g.units );
        i32( g.axis.empty() ? 0 : 1 );
        for ( unsigned i = 0; i < g.ndims && !g.axis.empty(); i++ ) {
            str( g.axis[i].name ); i32( g.axis[i].type ); f64( g.axis[i].min ); f64( g.axis[i].max );
            str( g.axis[i].label ); str( g.axis[i].units );
        }
    }
    void add_part_info( const part_info & p ) {
        size_t len = str_size( p.label ) + 8 + 4;
        for ( size_t i = 0; i < p.quants.size(); i++ )
            len += str_size( p.quants[i] ) + str_size( p.qlabels[i] ) + str_size( p.qunits[i] );
        record( PART_INFO_ID, p.name, len );
        str( p.label ); u64( p.np ); u32( (uint32_t) p.quants.size() );
        for ( auto & q : p.quants ) str( q );
        for ( auto & q : p.qlabels ) str( q );
        for ( auto & q : p.qunits ) str( q );
    }
    // float32 dataset of ndims dimensions
    void add_dataset( const std::string & name, const float * data, unsigned ndims, const uint64_t * count ) {
        uint64_t n = 1;
        for ( unsigned i = 0; i < ndims; i++ ) n *= count[i];
        record( DATASET_ID, name, 4 * n + 4 + 4 + 4 + 8 * ndims );
        u32( ++ndatasets ); i32( float32 ); u32( ndims );
        for ( unsigned i = 0; i < ndims; i++ ) u64( count[i] );
        put( data, 4 * n );
    }
};

// zdf_save_grid (grid file with one float32 dataset)
inline int save_grid( const float * data, const grid_info & info, const iteration & it, const std::string & path ) {
    create_path( path );
    char fn[1024];
    snprintf( fn, sizeof fn, "%s/%s-%06u.zdf", path.c_str(), info.name.c_str(), (unsigned) it.n );
    file f;
    if ( !f.open( fn ) ) return 0;
    f.add_string( "TYPE", "grid" );
    f.add_grid_info( info );
    f.add_iteration( it );
    f.add_dataset( info.name, data, info.ndims, info.count );
    return 1;
}

// zdf_open_part_file + zdf_add_quant_part_file for every quantity
inline int save_particles( const part_info & info, const iteration & it, const std::string & path,
                           const std::vector<std::vector<float>> & quants ) {
    create_path( path );
    char fn[1024];
    snprintf( fn, sizeof fn, "%s/particles-%s-%06u.zdf", path.c_str(), info.name.c_str(), (unsigned) it.n );
    file f;
    if ( !f.open( fn ) ) return 0;
    f.add_string( "TYPE", "particles" );
    f.add_part_info( info );
    f.add_iteration( it );
    for ( size_t q = 0; q < info.quants.size(); q++ ) {
        const uint64_t n = info.np;
        f.add_dataset( info.quants[q], quants[q].data(), 1, &n );
    }
    return 1;
}

}  // namespace zdf

#endif
