// noalloc.cu -- charge deposition for callers that cannot allocate device memory.
//
// zpic_b200_species_charge() allocates its per-tile scratch grid with
// cudaMalloc on every call.  Some callers cannot do that: a host framework
// that owns all device memory through its own pool and forbids foreign
// allocations, or a real-time or in-situ analysis loop that runs inside
// another code's time step and must not stall on the allocator (cudaMalloc
// may synchronise the device).  zpic_b200_charge_deposit_noalloc() gives them
// the same charge density with the scratch held in a fixed-size device array
// that belongs to the library.
//
// The scratch array is a file-scope __device__ array: every GPU that loads
// this library holds it (32 MiB) until the process exits.  All calls share it
// and it keeps the last call's contents; each call clears the part it uses
// before depositing.  Calls that overlap on the GPU (e.g. issued on two
// streams at once) race on the array and give wrong results: serialise them.
#include <cuda.h>
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
// Largest tile block (guard cells included): its shared-memory copy takes
// at most 48 KiB.
constexpr uint32_t kMaxTileCells = 12288;

static __device__ __align__( 256 ) float g_charge_scratch[ kChargeScratchFloats ];

namespace {

std::mutex g_setup_mu;

// Device address of g_charge_scratch per device, tagged with the unique ID of
// the context it was resolved in (a context created after cudaDeviceReset()
// gets a new ID, and may load the array at another address).
struct ScratchAddr { unsigned long long ctx_id; float * addr; };
ScratchAddr g_scratch[ 128 ] = {};

int err( int code, const std::string & msg ) { zb::set_last_error( msg ); return code; }

// Unique ID of the current context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points so the library needs no libcuda
// link); 0 when the driver does not provide them.
unsigned long long current_context_id() {
    using get_current_t = CUresult ( * )( CUcontext * );
    using get_id_t = CUresult ( * )( CUcontext, unsigned long long * );
    static get_current_t get_current = nullptr;
    static get_id_t get_id = nullptr;
    static bool looked_up = false;
    if ( !looked_up ) {
        void * f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if ( cudaGetDriverEntryPoint( "cuCtxGetCurrent", &f, cudaEnableDefault, &q ) == cudaSuccess &&
             q == cudaDriverEntryPointSuccess )
            get_current = reinterpret_cast<get_current_t>( f );
        f = nullptr;
        if ( cudaGetDriverEntryPoint( "cuCtxGetId", &f, cudaEnableDefault, &q ) == cudaSuccess &&
             q == cudaDriverEntryPointSuccess )
            get_id = reinterpret_cast<get_id_t>( f );
        cudaGetLastError();
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if ( get_current && get_id && get_current( &ctx ) == CUDA_SUCCESS && ctx && get_id( ctx, &id ) == CUDA_SUCCESS )
        return id;
    return 0;
}

// Set-up, once per device (and again only if the device's context was
// replaced), with that device current: the device address of the scratch
// array.  The array's name in host code is a host-side stand-in, never a
// device address: handing it to a kernel would fault or, where the GPU can
// reach host memory, silently use the wrong memory.
int scratch_address( int device, float ** out ) {
    std::lock_guard<std::mutex> lock( g_setup_mu );
    if ( device < 0 || device >= 128 ) return err( ZPIC_E_INVALID, "device index out of range" );
    const unsigned long long id = current_context_id();
    ScratchAddr & c = g_scratch[ device ];
    if ( !c.addr || c.ctx_id != id ) {
        void * p = nullptr;
        cudaError_t e = cudaGetSymbolAddress( &p, g_charge_scratch );
        if ( e != cudaSuccess || !p ) return err( ZPIC_E_CUDA, std::string( "cudaGetSymbolAddress: " ) + cudaGetErrorString( e ) );
        c.addr = static_cast<float *>( p );
        c.ctx_id = id;
    }
    *out = c.addr;
    return ZPIC_OK;
}

__global__ void k_clear( float * __restrict__ p, size_t n ) {
    for ( size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x )
        p[i] = 0.0f;
}

// dep_charge_kernel (species.cpp:2348-2399) on particles in the reference's
// packed layout: per-tile shared-memory sums added to the tile's block of the
// scratch grid (guard cells {0,1}, ext = nx + 1).  A particle whose cell lies
// outside [0, nx) of its tile (an unsorted set, e.g. after a move without the
// tile sort) would address outside the tile's block: it is skipped.
__global__ void k_dep_charge_packed( const int32_t * __restrict__ np, const int32_t * __restrict__ offset,
                                     const int2 * __restrict__ ix, const float2 * __restrict__ x, float q,
                                     float * __restrict__ scratch, int nxx, int nxy, int cextx, int cvol ) {
    extern __shared__ float sc[];
    const int t = blockIdx.x;
    for ( int i = threadIdx.x; i < cvol; i += blockDim.x ) sc[i] = 0.f;
    __syncthreads();
    const int n = np[t], off = offset[t];
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) {
        const int2 c = ix[ off + i ];
        if ( c.x < 0 || c.x >= nxx || c.y < 0 || c.y >= nxy ) continue;
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
    // Tile block: (nx_x+1)*(nx_y+1) cells, at most kMaxTileCells (48 KiB of
    // shared memory).  Each side is bounded first, so the products below
    // cannot overflow.
    if ( nx_x >= kMaxTileCells || nx_y >= kMaxTileCells ||
         (uint64_t) ( nx_x + 1 ) * ( nx_y + 1 ) > kMaxTileCells )
        return err( ZPIC_E_INVALID, "tile too large for the fixed scratch: (nx.x+1)*(nx.y+1) = " +
                                    std::to_string( (uint64_t) ( nx_x + 1ull ) * ( nx_y + 1ull ) ) +
                                    " cells, the maximum is " + std::to_string( kMaxTileCells ) );
    const int cextx = (int) nx_x + 1, cexty = (int) nx_y + 1;
    const int cvol = ( cextx * cexty + 3 ) & ~3;
    const uint64_t ntiles = (uint64_t) ntiles_x * ntiles_y;
    if ( ntiles > kChargeScratchFloats || ntiles * (uint64_t) cvol > kChargeScratchFloats )
        return err( ZPIC_E_INVALID, "grid too large for the fixed scratch: needs " +
                                    std::to_string( ntiles ) + " tiles x " + std::to_string( cvol ) +
                                    " floats, the maximum is " + std::to_string( kChargeScratchFloats ) + " floats" );
    const size_t need = (size_t) ntiles * cvol;
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
        scratch, (int) nx_x, (int) nx_y, cextx, cvol );
    // add_from_gc + gather into the dense [ny][nx] output; the charge grid is
    // a new grid object in the reference, hence periodic (grid.h:79)
    e = zb::launch_charge_finish( st, scratch, d_charge, (int) ntiles_x, (int) ntiles_y, (int) nx_x, (int) nx_y,
                                  cextx, cvol, 1, 1 );
    if ( e == cudaSuccess ) e = cudaGetLastError();
    if ( e != cudaSuccess ) return err( ZPIC_E_CUDA, cudaGetErrorString( e ) );
    return ZPIC_OK;
}
