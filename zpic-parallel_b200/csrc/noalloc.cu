// noalloc.cu -- charge deposition for callers that cannot allocate device memory.
//
// zpic_b200_species_charge() allocates its per-tile scratch grid with
// cudaMalloc on every call.  Some callers cannot do that: a host framework
// that owns all device memory through its own pool and forbids foreign
// allocations, a real-time or in-situ analysis loop that must not stall on
// the allocator (cudaMalloc may synchronise the device), or code that records
// its work into a CUDA graph, where cudaMalloc is not a capturable operation.
// zpic_b200_charge_deposit_noalloc() gives them the same charge density with
// the scratch held in a fixed-size device array that belongs to the library.
//
// The scratch array is a file-scope __device__ array: every GPU that loads
// this library holds it (32 MiB) until the process exits.  All calls share it
// and it keeps the last call's contents; each call clears the part it uses
// before depositing.  Calls that overlap on the GPU (e.g. issued on two
// streams at once) race on the array and give wrong results: serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "zpic_b200.h"

namespace zb {
cudaError_t launch_charge_finish( cudaStream_t, const float *, float *, int, int, int, int, int, int, int, int );
void set_last_error( const std::string & msg );   // message returned by zpic_b200_last_error()
}

// Maximum scratch size: ntiles * roundup4((nx.x+1)*(nx.y+1)) floats, i.e. the
// tiled charge grid with guard cells {0,1} (species.cpp:2486-2491).  8 Mi
// floats cover, e.g., a 2048x2048 grid in 16x16 tiles (4,784,128 floats).
constexpr size_t kChargeScratchFloats = size_t( 8 ) << 20;

static __device__ __align__( 256 ) float g_charge_scratch[ kChargeScratchFloats ];

namespace {

std::mutex g_setup_mu;
float * g_scratch_addr[ 128 ] = {};   // device address of g_charge_scratch, per device

int err( int code, const std::string & msg ) { zb::set_last_error( msg ); return code; }

// Once per device, with that device current: resolve the device address of
// the scratch array.  The symbol's name in host code is only a host-side
// stand-in and must never be handed to a kernel.
int scratch_address( int device, float ** out ) {
    std::lock_guard<std::mutex> lock( g_setup_mu );
    if ( device < 0 || device >= 128 ) return err( ZPIC_E_INVALID, "device index out of range" );
    if ( !g_scratch_addr[ device ] ) {
        void * p = nullptr;
        cudaError_t e = cudaGetSymbolAddress( &p, g_charge_scratch );
        if ( e != cudaSuccess || !p ) return err( ZPIC_E_CUDA, std::string( "cudaGetSymbolAddress: " ) + cudaGetErrorString( e ) );
        g_scratch_addr[ device ] = static_cast<float *>( p );
    }
    *out = g_scratch_addr[ device ];
    return ZPIC_OK;
}

__global__ void k_clear( float * __restrict__ p, size_t n ) {
    for ( size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x )
        p[i] = 0.0f;
}

// dep_charge_kernel (species.cpp:2348-2399) on particles in the reference's
// packed layout: per-tile shared-memory sums added to the tile's block of the
// scratch grid (guard cells {0,1}, ext = nx + 1).
__global__ void k_dep_charge_packed( const int32_t * __restrict__ np, const int32_t * __restrict__ offset,
                                     const int2 * __restrict__ ix, const float2 * __restrict__ x, float q,
                                     float * __restrict__ scratch, int cextx, int cvol ) {
    extern __shared__ float sc[];
    const int t = blockIdx.x;
    for ( int i = threadIdx.x; i < cvol; i += blockDim.x ) sc[i] = 0.f;
    __syncthreads();
    const int n = np[t], off = offset[t];
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) {
        const int2 c = ix[ off + i ];
        const float2 p = x[ off + i ];
        const int idx = c.y * cextx + c.x;
        const float s0x = 0.5f - p.x, s1x = 0.5f + p.x, s0y = 0.5f - p.y, s1y = 0.5f + p.y;
        atomicAdd( sc + idx, s0y * s0x * q );
        atomicAdd( sc + idx + 1, s0y * s1x * q );
        atomicAdd( sc + idx + cextx, s1y * s0x * q );
        atomicAdd( sc + idx + 1 + cextx, s1y * s1x * q );
    }
    __syncthreads();
    for ( int i = threadIdx.x; i < cvol; i += blockDim.x ) scratch[ (size_t) t * cvol + i ] += sc[i];
}

}  // namespace

extern "C" int zpic_b200_charge_deposit_noalloc( uint32_t ntiles_x, uint32_t ntiles_y, uint32_t nx_x, uint32_t nx_y,
                                                 float q, const int32_t * d_np, const int32_t * d_offset,
                                                 const int32_t * d_ix, const float * d_x, float * d_charge,
                                                 void * stream ) {
    if ( ntiles_x == 0 || ntiles_y == 0 || nx_x == 0 || nx_y == 0 || !d_np || !d_offset || !d_ix || !d_x || !d_charge )
        return err( ZPIC_E_INVALID, "invalid argument" );
    const int cextx = nx_x + 1, cexty = nx_y + 1;
    const int cvol = ( cextx * cexty + 3 ) & ~3;
    const size_t ntiles = (size_t) ntiles_x * ntiles_y;
    const size_t need = ntiles * (size_t) cvol;
    if ( need > kChargeScratchFloats || (size_t) cvol * sizeof( float ) > 48 * 1024 )
        return err( ZPIC_E_INVALID, "grid too large for the fixed scratch: needs " + std::to_string( need ) +
                                    " floats, the maximum is " + std::to_string( kChargeScratchFloats ) +
                                    " (and at most 12288 cells per tile block)" );
    int dev = 0;
    cudaError_t e = cudaGetDevice( &dev );
    if ( e != cudaSuccess ) return err( ZPIC_E_CUDA, cudaGetErrorString( e ) );
    float * scratch = nullptr;
    int rc = scratch_address( dev, &scratch );
    if ( rc != ZPIC_OK ) return rc;
    cudaStream_t st = static_cast<cudaStream_t>( stream );
    k_clear<<< 592, 256, 0, st >>>( scratch, need );
    k_dep_charge_packed<<< (unsigned) ntiles, 256, cvol * sizeof( float ), st >>>(
        d_np, d_offset, reinterpret_cast<const int2 *>( d_ix ), reinterpret_cast<const float2 *>( d_x ), q,
        scratch, cextx, cvol );
    // add_from_gc + gather into the dense [ny][nx] output; the charge grid is
    // a new grid object in the reference, hence periodic (grid.h:79)
    e = zb::launch_charge_finish( st, scratch, d_charge, ntiles_x, ntiles_y, nx_x, nx_y, cextx, cvol, 1, 1 );
    if ( e == cudaSuccess ) e = cudaGetLastError();
    if ( e != cudaSuccess ) return err( ZPIC_E_CUDA, cudaGetErrorString( e ) );
    return ZPIC_OK;
}
