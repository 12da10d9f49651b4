// Microbenchmarks for the rooflines that the measured HBM copy and BF16 GEMM
// peaks (MEASURED_PEAKS.json) do not give:
// L2-resident read bandwidth, random record gathers from L2 (the access
// pattern of BVH traversal) and FP32 FMA throughput, measured in the same
// process as the kernels they are compared with.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "../../include/cr.h"

namespace
{
void check( cudaError_t e, const char *what )
{
	if ( e != cudaSuccess ) throw std::runtime_error( std::string( what ) + ": " + cudaGetErrorString( e ) );
}

// Every thread reads float4s of a buffer that fits in L2, `passes` times over;
// the sum is written only when it matches an impossible value, so the loads
// are kept without a store per load.
__global__ void k_l2_read( const float4 *__restrict__ buf, uint32_t n4, uint32_t passes, float *sink )
{
	float4 acc = make_float4( 0.f, 0.f, 0.f, 0.f );
	const uint32_t stride = gridDim.x * blockDim.x;
	for ( uint32_t p = 0; p < passes; ++p )
		for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride )
		{
			float4 v = __ldcg( buf + i );  // L2, not L1
			acc.x += v.x, acc.y += v.y, acc.z += v.z, acc.w += v.w;
		}
	if ( acc.x + acc.y + acc.z + acc.w == -1.2345f ) *sink = acc.x;
}

// 8 independent FMA chains per thread, `iters` rounds.
__global__ void k_fma( uint32_t iters, float *sink )
{
	float a[ 8 ];
	for ( int k = 0; k < 8; ++k ) a[ k ] = float( threadIdx.x + k );
	const float m = 1.0000001f, c = 1e-7f;
	for ( uint32_t i = 0; i < iters; ++i )
#pragma unroll
		for ( int k = 0; k < 8; ++k ) a[ k ] = fmaf( a[ k ], m, c );
	float s = 0.f;
	for ( int k = 0; k < 8; ++k ) s += a[ k ];
	if ( s == -1.2345f ) *sink = s;
}
// Random whole-record gathers: every thread fetches `iters` records of R
// 16-byte words at independent pseudo-random indices (xorshift32), through the
// L1/texture path as the traversal kernels read BVH nodes and triangles.
template <int R>
__global__ void __launch_bounds__( 128 ) k_gather( const uint4 *__restrict__ buf, uint32_t n_rec, uint32_t iters,
												   uint32_t *sink )
{
	uint32_t x = 0x9E3779B9u ^ ( blockIdx.x * blockDim.x + threadIdx.x ) * 0x85EBCA6Bu;
	uint32_t acc = 0;
	for ( uint32_t i = 0; i < iters; ++i )
	{
		x ^= x << 13, x ^= x >> 17, x ^= x << 5;
		const uint4 *p = buf + size_t( x % n_rec ) * R;
#pragma unroll
		for ( int k = 0; k < R; ++k )
		{
			const uint4 v = __ldg( p + k );
			acc ^= v.x ^ v.y ^ v.z ^ v.w;
		}
	}
	if ( acc == 0x12345678u ) *sink = acc;
}
}  // namespace

// Achievable rate of random record gathers from an L2-resident array:
// records of `record_bytes` (80: a wide BVH node, 48: a triangle) from an
// array of `array_bytes`; returns the gathered bytes per second.
extern "C" int cr_measure_gather_impl( void *stream, uint32_t record_bytes, uint64_t array_bytes, double *gbs,
									   const char **err )
{
	cudaStream_t st = (cudaStream_t)stream;
	uint4 *buf = nullptr;
	uint32_t *sink = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	try
	{
		if ( record_bytes != 48 && record_bytes != 80 ) throw std::runtime_error( "record_bytes must be 48 or 80" );
		if ( array_bytes < ( 1u << 20 ) || array_bytes > ( 1ull << 30 ) ) throw std::runtime_error( "array_bytes out of range" );
		int dev = 0, sms = 0;
		check( cudaGetDevice( &dev ), "device" );
		check( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ), "device" );
		const uint32_t n_rec = uint32_t( array_bytes / record_bytes );
		check( cudaMalloc( &buf, size_t( n_rec ) * record_bytes ), "cudaMalloc" );
		check( cudaMalloc( &sink, 4 ), "cudaMalloc" );
		check( cudaMemsetAsync( buf, 0, size_t( n_rec ) * record_bytes, st ), "memset" );
		check( cudaEventCreate( &e0 ), "event" );
		check( cudaEventCreate( &e1 ), "event" );
		const uint32_t blocks = sms * 8, iters = 2048;
		auto launch = [&]( uint32_t it ) {
			if ( record_bytes == 80 )
				k_gather<5><<<blocks, 128, 0, st>>>( buf, n_rec, it, sink );
			else
				k_gather<3><<<blocks, 128, 0, st>>>( buf, n_rec, it, sink );
		};
		launch( 256 );  // warm-up: the array into L2
		check( cudaEventRecord( e0, st ), "event" );
		launch( iters );
		check( cudaEventRecord( e1, st ), "event" );
		check( cudaEventSynchronize( e1 ), "event" );
		float ms = 0.f;
		check( cudaEventElapsedTime( &ms, e0, e1 ), "event" );
		if ( gbs ) *gbs = double( blocks ) * 128.0 * iters * record_bytes / ( ms * 1e-3 ) / 1e9;
		check( cudaGetLastError(), "gather" );
	}
	catch ( const std::exception &ex )
	{
		static thread_local std::string msg;
		msg = ex.what();
		*err = msg.c_str();
	}
	if ( buf ) cudaFree( buf );
	if ( sink ) cudaFree( sink );
	if ( e0 ) cudaEventDestroy( e0 );
	if ( e1 ) cudaEventDestroy( e1 );
	return *err ? -1 : 0;
}

extern "C" int cr_measure_peaks_impl( void *stream, double *l2_gbs, double *fp32_tflops, const char **err )
{
	cudaStream_t st = (cudaStream_t)stream;
	float4 *buf = nullptr;
	float *sink = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	try
	{
		int dev = 0, sms = 0;
		check( cudaGetDevice( &dev ), "device" );
		check( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ), "device" );
		const uint32_t bytes = 32u << 20;  // 32 MB: resident in the 126 MB L2
		const uint32_t n4 = bytes / 16;
		check( cudaMalloc( &buf, bytes ), "cudaMalloc" );
		check( cudaMalloc( &sink, 4 ), "cudaMalloc" );
		check( cudaMemsetAsync( buf, 0, bytes, st ), "memset" );
		check( cudaEventCreate( &e0 ), "event" );
		check( cudaEventCreate( &e1 ), "event" );
		float ms = 0.f;
		const uint32_t passes = 64;
		k_l2_read<<<sms * 8, 256, 0, st>>>( buf, n4, 2, sink );  // warm-up: the buffer into L2
		check( cudaEventRecord( e0, st ), "event" );
		k_l2_read<<<sms * 8, 256, 0, st>>>( buf, n4, passes, sink );
		check( cudaEventRecord( e1, st ), "event" );
		check( cudaEventSynchronize( e1 ), "event" );
		check( cudaEventElapsedTime( &ms, e0, e1 ), "event" );
		if ( l2_gbs ) *l2_gbs = double( bytes ) * passes / ( ms * 1e-3 ) / 1e9;
		const uint32_t iters = 1u << 14, blocks = sms * 16, threads = 256;
		k_fma<<<blocks, threads, 0, st>>>( 64, sink );
		check( cudaEventRecord( e0, st ), "event" );
		k_fma<<<blocks, threads, 0, st>>>( iters, sink );
		check( cudaEventRecord( e1, st ), "event" );
		check( cudaEventSynchronize( e1 ), "event" );
		check( cudaEventElapsedTime( &ms, e0, e1 ), "event" );
		if ( fp32_tflops ) *fp32_tflops = 2.0 * 8.0 * iters * double( blocks ) * threads / ( ms * 1e-3 ) / 1e12;
		check( cudaGetLastError(), "peaks" );
	}
	catch ( const std::exception &ex )
	{
		static thread_local std::string msg;
		msg = ex.what();
		*err = msg.c_str();
	}
	if ( buf ) cudaFree( buf );
	if ( sink ) cudaFree( sink );
	if ( e0 ) cudaEventDestroy( e0 );
	if ( e1 ) cudaEventDestroy( e1 );
	return *err ? -1 : 0;
}
