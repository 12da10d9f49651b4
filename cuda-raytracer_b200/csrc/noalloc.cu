// cr_render_device_noalloc: the render entry point for callers that cannot
// allocate device memory while they render.
//
// cr_render_device allocates its per-path wave state (about 140 bytes per
// path in flight) on first use and whenever a larger wave is requested.  Some
// callers cannot let that happen: a frame callback or real-time loop in which
// a cudaMalloc or cudaFree would synchronise the device and stall the frame,
// or an application that budgets all device memory at start-up and forbids
// allocation afterwards.  For them this entry point keeps the wave state in
// the fixed device array below, which every GPU that loads the library holds
// until the process exits (CR_NOALLOC_MAX_WAVE_PATHS paths, about 37 MB).
//
// The array lives in this file.  In host code its name is only a host-side
// stand-in, not a device address, so the first call on each device looks up
// the real address with cudaGetSymbolAddress, with that device current, and
// caches it; later calls reuse it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cr.h"
#include "internal.h"
#include "render.h"

namespace cr
{
namespace
{
constexpr size_t align256( size_t x ) { return ( x + 255 ) & ~size_t( 255 ); }

constexpr size_t NA_PATHS = CR_NOALLOC_MAX_WAVE_PATHS;
constexpr size_t NA_COUNTERS = n_counters_for( CR_NOALLOC_MAX_BOUNCE );
// Byte offsets of the wave arrays inside the scratch array.
constexpr size_t OFF_RAY_O = 0;
constexpr size_t OFF_RAY_D = OFF_RAY_O + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_HIT = OFF_RAY_D + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_BETA = OFF_HIT + align256( NA_PATHS * sizeof( HitRec ) );
constexpr size_t OFF_L = OFF_BETA + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_Q0 = OFF_L + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_Q1 = OFF_Q0 + align256( NA_PATHS * sizeof( uint32_t ) );
constexpr size_t OFF_SQ = OFF_Q1 + align256( NA_PATHS * sizeof( uint32_t ) );
constexpr size_t OFF_SH_O = OFF_SQ + align256( NA_PATHS * sizeof( uint32_t ) );
constexpr size_t OFF_SH_D = OFF_SH_O + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_SH_C = OFF_SH_D + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_COUNTERS = OFF_SH_C + align256( NA_PATHS * sizeof( float4 ) );
constexpr size_t OFF_ERR = OFF_COUNTERS + align256( NA_COUNTERS * sizeof( uint32_t ) );
constexpr size_t OFF_WORK = OFF_ERR + align256( sizeof( uint32_t ) );
constexpr size_t NA_BYTES = OFF_WORK + align256( 4 * sizeof( unsigned long long ) );

// The wave state of every cr_render_device_noalloc call on this device.
static __device__ __align__( 256 ) unsigned char g_noalloc_scratch[ NA_BYTES ];

constexpr int NA_MAX_DEVICES = 256;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[ NA_MAX_DEVICES ] = {};

// Device address of g_noalloc_scratch on the current device (set-up on the
// first call per device, with that device current).
int scratch_address( unsigned char **out, std::string &err )
{
	int dev = 0;
	cudaError_t e = cudaGetDevice( &dev );
	if ( e != cudaSuccess )
	{
		err = std::string( "cudaGetDevice: " ) + cudaGetErrorString( e );
		return CR_ERR_CUDA;
	}
	if ( dev < 0 || dev >= NA_MAX_DEVICES )
	{
		err = "device index out of range for the no-allocation scratch table";
		return CR_ERR_INVALID;
	}
	std::lock_guard<std::mutex> lock( g_setup_mutex );
	if ( !g_scratch_ptr[ dev ] )
	{
		void *ptr = nullptr;
		e = cudaGetSymbolAddress( &ptr, g_noalloc_scratch );
		if ( e != cudaSuccess || !ptr )
		{
			err = std::string( "cudaGetSymbolAddress of the no-allocation scratch: " ) + cudaGetErrorString( e );
			return CR_ERR_CUDA;
		}
		g_scratch_ptr[ dev ] = static_cast<unsigned char *>( ptr );
	}
	*out = g_scratch_ptr[ dev ];
	return CR_OK;
}

}  // namespace
}  // namespace cr

using namespace cr;

extern "C" int cr_render_device_noalloc( cr_scene *s, const cr_render_desc *desc, double *d_sum, double *d_sumsq,
										 uint32_t *d_count, void *stream )
{
	std::string err;
	if ( !s || !desc || !d_sum || !d_sumsq || !d_count )
	{
		set_last_error( "null argument" );
		return CR_ERR_INVALID;
	}
	if ( desc->wave_paths > CR_NOALLOC_MAX_WAVE_PATHS )
	{
		set_last_error( "wave_paths " + std::to_string( desc->wave_paths ) + " exceeds the no-allocation maximum of " +
						std::to_string( CR_NOALLOC_MAX_WAVE_PATHS ) + " paths" );
		return CR_ERR_INVALID;
	}
	// Requests this entry point cannot serve are refused before the request is
	// resolved: resolving a guided request would set up the scene's guide and
	// its training records, which allocates.
	if ( desc->guiding )
	{
		set_last_error( "cr_render_device_noalloc does not take guided renders (the guide's training records are "
						"allocated per scene); use cr_render_device" );
		return CR_ERR_UNSUPPORTED;
	}
	const uint32_t max_bounce = effective_max_bounce( s, desc );
	if ( max_bounce > CR_NOALLOC_MAX_BOUNCE )
	{
		set_last_error( "max_bounce " + std::to_string( max_bounce ) + " exceeds the no-allocation maximum of " +
						std::to_string( CR_NOALLOC_MAX_BOUNCE ) );
		return CR_ERR_INVALID;
	}
	DevScene sc;
	RenderConfig cfg;
	int rc = prepare_render( s, desc, sc, cfg, err );
	if ( rc != CR_OK )
	{
		set_last_error( err );
		return rc;
	}
	unsigned char *base = nullptr;
	rc = scratch_address( &base, err );
	if ( rc != CR_OK )
	{
		set_last_error( err );
		return rc;
	}
	uint64_t samples = uint64_t( cfg.ww ) * cfg.wh * cfg.spp;
	uint64_t wave = desc->wave_paths ? desc->wave_paths : CR_NOALLOC_MAX_WAVE_PATHS;
	cfg.wave_paths = uint32_t( wave < samples ? wave : samples );
	cfg.count_work = false;
	WaveBuffers wb;
	wb.capacity = cfg.wave_paths;
	wb.ray_o = reinterpret_cast<float4 *>( base + OFF_RAY_O );
	wb.ray_d = reinterpret_cast<float4 *>( base + OFF_RAY_D );
	wb.hit = reinterpret_cast<HitRec *>( base + OFF_HIT );
	wb.beta = reinterpret_cast<float4 *>( base + OFF_BETA );
	wb.L = reinterpret_cast<float4 *>( base + OFF_L );
	wb.queue[ 0 ] = reinterpret_cast<uint32_t *>( base + OFF_Q0 );
	wb.queue[ 1 ] = reinterpret_cast<uint32_t *>( base + OFF_Q1 );
	wb.shadow_queue = reinterpret_cast<uint32_t *>( base + OFF_SQ );
	wb.sh_o = reinterpret_cast<float4 *>( base + OFF_SH_O );
	wb.sh_d = reinterpret_cast<float4 *>( base + OFF_SH_D );
	wb.sh_c = reinterpret_cast<float4 *>( base + OFF_SH_C );
	wb.counters = reinterpret_cast<uint32_t *>( base + OFF_COUNTERS );
	wb.n_counters = n_counters_for( cfg.max_bounce );
	wb.err = reinterpret_cast<uint32_t *>( base + OFF_ERR );
	wb.work = reinterpret_cast<unsigned long long *>( base + OFF_WORK );
	cudaStream_t st = static_cast<cudaStream_t>( stream );
	// The array keeps the previous call's contents: the error word must start
	// at zero (queue counters are cleared per wave by render_waves).
	cudaError_t e = cudaMemsetAsync( wb.err, 0, sizeof( uint32_t ), st );
	if ( e != cudaSuccess )
	{
		set_last_error( std::string( "cudaMemsetAsync: " ) + cudaGetErrorString( e ) );
		return CR_ERR_CUDA;
	}
	try
	{
		render_waves( sc, cfg, wb, d_sum, d_sumsq, d_count, st, nullptr );
	}
	catch ( const std::exception &ex )
	{
		set_last_error( ex.what() );
		return CR_ERR_CUDA;
	}
	return CR_OK;
}
