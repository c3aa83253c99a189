// vec_types.h -- host vector types of the drop-in C++ API (the reference's
// openmp/em2d/vec_types.h names: int2, uint2, float2, float3, double3 and
// their make_* constructors and stream output).
#ifndef ZPIC_B200_VEC_TYPES_H_
#define ZPIC_B200_VEC_TYPES_H_

#include <iostream>

#if defined( __CUDACC__ )
#include <vector_types.h>
#include <vector_functions.h>
#else
struct alignas( 8 ) int2 { int x, y; };
struct alignas( 8 ) uint2 { unsigned int x, y; };
struct alignas( 8 ) float2 { float x, y; };
struct alignas( 16 ) double2 { double x, y; };
struct float3 { float x, y, z; };
struct double3 { double x, y, z; };
struct int3 { int x, y, z; };
static inline int2 make_int2( int x, int y ) { return { x, y }; }
static inline uint2 make_uint2( unsigned x, unsigned y ) { return { x, y }; }
static inline float2 make_float2( float x, float y ) { return { x, y }; }
static inline double2 make_double2( double x, double y ) { return { x, y }; }
static inline float3 make_float3( float x, float y, float z ) { return { x, y, z }; }
static inline double3 make_double3( double x, double y, double z ) { return { x, y, z }; }
static inline int3 make_int3( int x, int y, int z ) { return { x, y, z }; }
#endif

static inline std::ostream & operator<<( std::ostream & os, const uint2 & v ) { return os << "(" << v.x << ", " << v.y << ")"; }
static inline std::ostream & operator<<( std::ostream & os, const int2 & v ) { return os << "(" << v.x << ", " << v.y << ")"; }
static inline std::ostream & operator<<( std::ostream & os, const float2 & v ) { return os << "(" << v.x << ", " << v.y << ")"; }
static inline std::ostream & operator<<( std::ostream & os, const float3 & v ) { return os << "(" << v.x << ", " << v.y << ", " << v.z << ")"; }
static inline std::ostream & operator<<( std::ostream & os, const double3 & v ) { return os << "(" << v.x << ", " << v.y << ", " << v.z << ")"; }
static inline double3 & operator+=( double3 & a, const double3 & b ) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }

#endif
