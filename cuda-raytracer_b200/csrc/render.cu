// Wavefront Radiance integrator and batched ray queries.
//
// The reference runs one RadianceKernel::execute per (pixel, sample) on a CPU
// thread (src/core/kernel/radiance.cu:14-81, src/core/tracer/cpuMulticore.cu:53-64).
// Here a wave of paths advances one bounce at a time through separate
// kernels so every stage runs with coherent control flow:
//
//   k_generate   camera rays (PinholeLens::sample, src/core/misc/lens.hpp:62-66)
//   per bounce:
//     k_extend   closest hit for the live queue            (Scene::intersect(Ray))
//     k_shade    emission, NEE set-up, BSDF continuation, Russian roulette;
//                appends to the shadow queue and the next live queue with one
//                warp ballot + one atomic per warp
//     k_shadow   any hit for the shadow queue; unoccluded contributions added
//   k_accumulate per-pixel FP64 sums of the finite samples (cpuMulticore.cu:58-64)
//
// Queue lengths live in device memory, so a wave needs no host round trip.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cr.h"
#include "cr_device.cuh"
#include "render.h"
#include "traverse.cuh"
#include "guide.cuh"
#include "guide_tc.cuh"

namespace cr
{
namespace
{
constexpr float KOISHI_EPS = 4e-3f;  // LocalVaryings::emitRay/emitSeg offset (varyings.hpp:19-37)

constexpr uint32_t BIN_AXIS_BITS = 3;                           // ray binning: 8 cells per axis
constexpr uint32_t N_BINS = 8u << ( 3 * BIN_AXIS_BITS );        // x 8 octants = 4096 bins

struct WaveArgs
{
	uint64_t first;  // first global sample of the wave
	uint32_t n;      // samples in the wave
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated append: every lane of the warp calls this with its flag.
__device__ __forceinline__ uint32_t warp_append( bool want, uint32_t *counter )
{
	uint32_t mask = __ballot_sync( ~0u, want );
	if ( !mask ) return 0;
	uint32_t leader = __ffs( mask ) - 1;
	uint32_t base = 0;
	if ( lane_id() == leader ) base = atomicAdd( counter, __popc( mask ) );
	base = __shfl_sync( ~0u, base, leader );
	return base + __popc( mask & ( ( 1u << lane_id() ) - 1u ) );
}

// Lens::sample of sub-pixel sample k of pixel (x, y) (src/core/misc/lens.hpp):
// PinholeLens (:56-66) shoots from the camera through the stratified point on
// the image plane; OrthographicLens (:40-53) moves the origin by that plane
// offset times 4 / width and shoots along the view direction.
// The products and sums are written as explicit fused multiply-adds so that
// every kernel that generates camera rays (single and batched renders) forms
// bit-identical rays, whatever the compiler would contract in each context.
__device__ __forceinline__ float3 fma3( float3 a, float s, float3 b )
{
	return f3( fmaf( a.x, s, b.x ), fmaf( a.y, s, b.y ), fmaf( a.z, s, b.z ) );
}

__device__ __forceinline__ float3 normalize_fma( float3 a )
{
	const float l2 = fmaf( a.x, a.x, fmaf( a.y, a.y, __fmul_rn( a.z, a.z ) ) );
	return a * ( 1.0f / sqrtf( l2 ) );
}

__device__ __forceinline__ void camera_ray( const DevCamera &c, uint32_t x, uint32_t y, uint32_t k, float3 &o, float3 &d )
{
	const float fx = float( x ) - float( c.width ) * 0.5f, fy = float( y ) - float( c.height ) * 0.5f;
	const float kx = float( k % c.pw ), ky = float( k / c.pw );
	if ( c.lens == 1 )
	{
		const float3 p = fma3( f3( c.v ), fy, fma3( f3( c.u ), fx, fma3( f3( c.dv ), ky, fma3( f3( c.du ), kx, f3( 0.f, 0.f, 0.f ) ) ) ) );
		const float s = 4.f / float( c.width );
		o = fma3( p, s, f3( c.o ) );
		d = normalize_fma( f3( c.n ) );
		return;
	}
	const float3 t = fma3( f3( c.v ), fy, fma3( f3( c.u ), fx, f3( c.n ) ) );
	o = f3( c.o );
	d = normalize_fma( fma3( f3( c.dv ), ky, fma3( f3( c.du ), kx, t ) ) );
}

__global__ void k_generate( DevScene sc, RenderConfig cfg, WaveBuffers wb, WaveArgs wa )
{
	if ( blockIdx.x == 0 && threadIdx.x == 0 ) wb.counters[ CNT_EXT ] = wa.n;
	for ( uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < wa.n; s += gridDim.x * blockDim.x )
	{
		uint64_t g = wa.first + s;
		uint32_t pix = uint32_t( g / cfg.spp ), k = uint32_t( g % cfg.spp );
		uint32_t x = cfg.x0 + pix % cfg.ww, y = cfg.y0 + pix / cfg.ww;
		float3 o, d;
		camera_ray( sc.cam, x, y, k, o, d );
		wb.ray_o[ s ] = make_float4( o.x, o.y, o.z, 0.f );
		wb.ray_d[ s ] = make_float4( d.x, d.y, d.z, INFINITY );
		wb.beta[ s ] = make_float4( 1.f, 1.f, 1.f, 0.f );
		wb.L[ s ] = make_float4( 0.f, 0.f, 0.f, 0.f );
		wb.queue[ 0 ][ s ] = s;
	}
}

// Closest-hit queue of one bounce: rays from the path state, hit records out.
struct ExtendIO
{
	static constexpr bool MULTI = false;
	const uint32_t *queue;
	const float4 *ray_o, *ray_d;
	HitRec *hit;
	__device__ void load( uint32_t i, uint32_t &item, float3 &o, float3 &d, float &tmin, float &tmax ) const
	{
		item = queue[ i ];
		float4 a = ray_o[ item ], b = ray_d[ item ];
		o = f3( a ), d = f3( b ), tmin = a.w, tmax = b.w;
	}
	__device__ void finish( uint32_t item, const HitRec &h, bool ) const { hit[ item ] = h; }
};

// Ray binning: a counting sort of a traversal queue by (direction octant,
// Morton code of the origin's cell in an 8^3 grid over the root node's box).
// The persistent traversal kernel hands consecutive queue entries to the lanes
// of a warp, so after the sort a warp traces rays that start close together
// and head the same way: they fetch the same nodes and take the same branches.
// Only the traversal reads the sorted queue; shading keeps path order, whose
// per-path state accesses stay coalesced (shading in sorted order doubled the
// shading time on the 1.31M-triangle scene).
// A memset and three launches: count (per-block shared-memory histograms added
// to the global one), scan (counts to offsets), scatter (each block reserves
// its range of every bin it holds with one atomic, then places its rays).
// Each block takes the same contiguous slice of the queue in both passes, and
// a warp adds each run of equal keys among its lanes with one atomic.  The
// order inside a bin is whatever the atomics give, which changes no result
// (every ray's hit is its own).
__device__ __forceinline__ uint32_t ray_bin( const float3 lo, const float3 scale, const float4 o, const float4 d )
{
	const uint32_t oct = ( d.x < 0.f ? 1u : 0u ) | ( d.y < 0.f ? 2u : 0u ) | ( d.z < 0.f ? 4u : 0u );
	const float lim = float( ( 1u << BIN_AXIS_BITS ) - 1u );
	// fmaxf first: a NaN coordinate lands in cell 0
	const uint32_t cx = uint32_t( fminf( fmaxf( ( o.x - lo.x ) * scale.x, 0.f ), lim ) );
	const uint32_t cy = uint32_t( fminf( fmaxf( ( o.y - lo.y ) * scale.y, 0.f ), lim ) );
	const uint32_t cz = uint32_t( fminf( fmaxf( ( o.z - lo.z ) * scale.z, 0.f ), lim ) );
	uint32_t m = 0;
#pragma unroll
	for ( uint32_t k = 0; k < BIN_AXIS_BITS; ++k )
		m |= ( ( ( cx >> k ) & 1u ) << ( 3 * k ) ) | ( ( ( cy >> k ) & 1u ) << ( 3 * k + 1 ) ) |
			 ( ( ( cz >> k ) & 1u ) << ( 3 * k + 2 ) );
	return ( oct << ( 3 * BIN_AXIS_BITS ) ) | m;
}

// The binning grid: the root node's box (its children's planes span
// p .. p + 255 * 2^e per axis), cut into 2^BIN_AXIS_BITS cells per axis.
__device__ __forceinline__ void bin_frame( const WNode *nodes, float3 &lo, float3 &scale )
{
	const uint4 n0 = __ldg( reinterpret_cast<const uint4 *>( nodes ) );
	lo = f3( __uint_as_float( n0.x ), __uint_as_float( n0.y ), __uint_as_float( n0.z ) );
	const float cells = float( 1u << BIN_AXIS_BITS );
	scale = f3( cells / ( 255.f * __uint_as_float( ( n0.w & 0xFFu ) << 23 ) ),
				cells / ( 255.f * __uint_as_float( ( ( n0.w >> 8 ) & 0xFFu ) << 23 ) ),
				cells / ( 255.f * __uint_as_float( ( ( n0.w >> 16 ) & 0xFFu ) << 23 ) ) );
}

constexpr int BIN_THREADS = 512;

// This block's slice [lo, hi) of a queue of n entries.
__device__ __forceinline__ void bin_slice( uint32_t n, uint32_t &lo, uint32_t &hi )
{
	const uint32_t per = ( n + gridDim.x - 1 ) / gridDim.x;
	lo = min( n, blockIdx.x * per );
	hi = min( n, lo + per );
}

// Runs of equal keys among a warp's lanes: whether this lane starts one, the
// run's first lane, and its length (from its first lane).  Lanes with key ~0u
// (no ray) form runs of their own, which the callers skip.
struct KeyRun
{
	uint32_t first, len;
};
__device__ __forceinline__ KeyRun key_run( uint32_t key, uint32_t lane )
{
	const uint32_t prev = __shfl_up_sync( ~0u, key, 1 );
	const uint32_t heads = __ballot_sync( ~0u, lane == 0 || key != prev );
	const uint32_t first = 31u - __clz( heads & ( 0xFFFFFFFFu >> ( 31u - lane ) ) );  // last head at or below lane
	const uint32_t after = lane == 31 ? 0u : heads & ( 0xFFFFFFFFu << ( lane + 1 ) );
	const uint32_t end = after ? uint32_t( __ffs( after ) - 1 ) : 32u;
	return KeyRun{ first, end - lane };  // len is meaningful on the run's first lane
}

__global__ void __launch_bounds__( BIN_THREADS ) k_bin_count( const uint32_t *__restrict__ queue, const uint32_t *n_ptr,
															   const float4 *__restrict__ ray_o,
															   const float4 *__restrict__ ray_d, const WNode *nodes,
															   uint32_t *__restrict__ bins )
{
	__shared__ uint32_t h[ N_BINS ];
	for ( uint32_t b = threadIdx.x; b < N_BINS; b += blockDim.x ) h[ b ] = 0;
	__syncthreads();
	uint32_t lo, hi;
	bin_slice( *n_ptr, lo, hi );
	float3 blo, scale;
	bin_frame( nodes, blo, scale );
	const uint32_t lane = lane_id();
	// the block strides together, so every lane of a warp takes part in the vote
	for ( uint32_t base = lo; base < hi; base += blockDim.x )
	{
		const uint32_t i = base + threadIdx.x;
		uint32_t key = ~0u;
		if ( i < hi )
		{
			const uint32_t item = queue[ i ];
			key = ray_bin( blo, scale, ray_o[ item ], ray_d[ item ] );
		}
		const KeyRun run = key_run( key, lane );
		if ( key != ~0u && run.first == lane ) atomicAdd( h + key, run.len );
	}
	__syncthreads();
	for ( uint32_t b = threadIdx.x; b < N_BINS; b += blockDim.x )
		if ( h[ b ] ) atomicAdd( bins + b, h[ b ] );
}

// Counts -> exclusive offsets, in place: one block of 1024 threads, each
// scanning N_BINS / 1024 consecutive bins staged through shared memory.
__global__ void __launch_bounds__( 1024 ) k_bin_scan( uint32_t *bins )
{
	constexpr uint32_t PER = N_BINS / 1024;
	__shared__ uint32_t v[ N_BINS ];
	__shared__ uint32_t warp_sum[ 32 ];
	const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
	for ( uint32_t b = t; b < N_BINS; b += 1024 ) v[ b ] = bins[ b ];
	__syncthreads();
	uint32_t s = 0;
#pragma unroll
	for ( uint32_t k = 0; k < PER; ++k ) s += v[ t * PER + k ];
	uint32_t x = s;  // inclusive scan of the threads' sums within the warp
#pragma unroll
	for ( int o = 1; o < 32; o <<= 1 )
	{
		const uint32_t y = __shfl_up_sync( ~0u, x, o );
		if ( lane >= uint32_t( o ) ) x += y;
	}
	if ( lane == 31 ) warp_sum[ warp ] = x;
	__syncthreads();
	if ( warp == 0 )
	{
		uint32_t w = warp_sum[ lane ];
#pragma unroll
		for ( int o = 1; o < 32; o <<= 1 )
		{
			const uint32_t y = __shfl_up_sync( ~0u, w, o );
			if ( lane >= uint32_t( o ) ) w += y;
		}
		warp_sum[ lane ] = w;
	}
	__syncthreads();
	uint32_t run = x - s + ( warp ? warp_sum[ warp - 1 ] : 0u );
#pragma unroll
	for ( uint32_t k = 0; k < PER; ++k )
	{
		const uint32_t c = v[ t * PER + k ];
		v[ t * PER + k ] = run;
		run += c;
	}
	__syncthreads();
	for ( uint32_t b = t; b < N_BINS; b += 1024 ) bins[ b ] = v[ b ];
}

__global__ void __launch_bounds__( BIN_THREADS ) k_bin_scatter( const uint32_t *__restrict__ queue, const uint32_t *n_ptr,
																 const float4 *__restrict__ ray_o,
																 const float4 *__restrict__ ray_d, const WNode *nodes,
																 uint32_t *__restrict__ bins, uint32_t *__restrict__ out,
																 uint32_t *err )
{
	__shared__ uint32_t h[ N_BINS ];
	for ( uint32_t b = threadIdx.x; b < N_BINS; b += blockDim.x ) h[ b ] = 0;
	__syncthreads();
	const uint32_t n = *n_ptr;
	uint32_t lo, hi;
	bin_slice( n, lo, hi );
	float3 blo, scale;
	bin_frame( nodes, blo, scale );
	const uint32_t lane = lane_id();
	// pass 1: this block's count per bin (as k_bin_count)
	for ( uint32_t base = lo; base < hi; base += blockDim.x )
	{
		const uint32_t i = base + threadIdx.x;
		uint32_t key = ~0u;
		if ( i < hi )
		{
			const uint32_t item = queue[ i ];
			key = ray_bin( blo, scale, ray_o[ item ], ray_d[ item ] );
		}
		const KeyRun run = key_run( key, lane );
		if ( key != ~0u && run.first == lane ) atomicAdd( h + key, run.len );
	}
	__syncthreads();
	// reserve this block's range of each bin it holds
	for ( uint32_t b = threadIdx.x; b < N_BINS; b += blockDim.x )
		if ( h[ b ] ) h[ b ] = atomicAdd( bins + b, h[ b ] );
	__syncthreads();
	// pass 2: place the rays
	for ( uint32_t base = lo; base < hi; base += blockDim.x )
	{
		const uint32_t i = base + threadIdx.x;
		uint32_t key = ~0u, item = 0;
		if ( i < hi )
		{
			item = queue[ i ];
			key = ray_bin( blo, scale, ray_o[ item ], ray_d[ item ] );
		}
		const KeyRun run = key_run( key, lane );
		uint32_t pos = 0;
		if ( key != ~0u && run.first == lane ) pos = atomicAdd( h + key, run.len );
		pos = __shfl_sync( ~0u, pos, run.first ) + ( lane - run.first );
		if ( key != ~0u )
		{
			if ( pos < n )
				out[ pos ] = item;
			else
				atomicOr( err, 16u );
		}
	}
}

// Shadow queue of one bounce: an unoccluded ray adds its contribution.
struct ShadowIO
{
	static constexpr bool MULTI = false;
	const uint32_t *queue;
	const float4 *ray_o, *ray_d, *contrib;
	float4 *L;
	__device__ void load( uint32_t i, uint32_t &item, float3 &o, float3 &d, float &tmin, float &tmax ) const
	{
		item = queue[ i ];
		float4 a = ray_o[ item ], b = ray_d[ item ];
		o = f3( a ), d = f3( b ), tmin = a.w, tmax = b.w;
	}
	__device__ void finish( uint32_t item, const HitRec &, bool occluded ) const
	{
		if ( occluded ) return;
		float4 c = contrib[ item ], l = L[ item ];
		L[ item ] = make_float4( l.x + c.x, l.y + c.y, l.z + c.z, l.w );
	}
};

// The same queues in a batched render: each path's scene is its job's.
struct BatchExtendIO : ExtendIO
{
	static constexpr bool MULTI = true;
	const DevScene *scenes;
	const uint32_t *path_job;
	__device__ const DevScene *scene( uint32_t item ) const { return scenes + path_job[ item ]; }
};

struct BatchShadowIO : ShadowIO
{
	static constexpr bool MULTI = true;
	const DevScene *scenes;
	const uint32_t *path_job;
	__device__ const DevScene *scene( uint32_t item ) const { return scenes + path_job[ item ]; }
};

// Batched ray queries of the C ABI: n x {o, d, tmax} in, cr_hit out.
struct QueryIO
{
	static constexpr bool MULTI = false;
	const float *rays;
	cr_hit *out;
	const float4 *tris, *attrs;
	const DevSphere *spheres;
	const uint32_t *prim_first;
	__device__ void load( uint32_t i, uint32_t &item, float3 &o, float3 &d, float &tmin, float &tmax ) const
	{
		item = i;
		const float *r = rays + 7 * size_t( i );
		o = f3( r[ 0 ], r[ 1 ], r[ 2 ] ), d = f3( r[ 3 ], r[ 4 ], r[ 5 ] );
		tmin = 0.f;
		tmax = r[ 6 ] > 0.f ? r[ 6 ] : INFINITY;
	}
	__device__ void finish( uint32_t item, const HitRec &h, bool found ) const
	{
		cr_hit res;
		res.prim = -1, res.tri = -1, res.t = INFINITY, res.u = res.v = 0.f;
		if ( found )
		{
			res.t = h.t, res.u = h.u, res.v = h.v;
			if ( h.id & HIT_SPHERE )
				res.prim = spheres[ h.id & ~HIT_SPHERE ].prim;
			else
			{
				uint32_t gid = __float_as_uint( tris[ 3 * size_t( h.id ) ].w );
				int prim = __float_as_int( attrs[ 3 * size_t( gid ) + 1 ].w );
				res.prim = prim;
				res.tri = int( gid - prim_first[ prim ] );
			}
		}
		out[ item ] = res;
	}
};

// Idle lanes per warp that trigger a refill in batched ray queries.
constexpr uint32_t QUERY_REFILL_MIN = 16;
// Closest-hit traversal: a triangle step once a quarter of the active lanes want one.
constexpr uint32_t EXT_TRI_VOTE = 4;
// Any-hit traversal: the shadow queue's own refill threshold (0: the closest-hit one).
inline uint32_t shadow_refill( const RenderConfig &cfg ) { return cfg.shadow_refill_min ? cfg.shadow_refill_min : cfg.refill_min; }

struct Surface
{
	float3 p, ns, ng;
	int32_t shader, light;
};

__device__ __forceinline__ Surface surface_at( const DevScene &sc, float3 o, float3 d, const HitRec &h, bool need_ng )
{
	Surface s;
	s.p = o + d * h.t;
	if ( h.id & HIT_SPHERE )
	{
		const DevSphere &sp = sc.spheres[ h.id & ~HIT_SPHERE ];
		s.ns = normalize( s.p - f3( sp.c ) );  // Sphere::normal (sphere.hpp:18-21, 52)
		s.ng = s.ns;
		s.shader = sp.shader;
		s.light = sp.light;
		return s;
	}
	const float4 *tp = sc.tris + 3 * size_t( h.id );
	float4 a = __ldg( tp );
	uint32_t gid = __float_as_uint( a.w );
	const float4 *ap = sc.attrs + 3 * size_t( gid );
	float4 n0 = __ldg( ap ), n1 = __ldg( ap + 1 ), n2 = __ldg( ap + 2 );
	// Mesh::normal (mesh.hpp:85-91) with interplot (ray.hpp:93-98).
	s.ns = normalize( f3( n0 ) * ( 1.f - h.u - h.v ) + f3( n1 ) * h.u + f3( n2 ) * h.v );
	s.shader = __float_as_int( n0.w );
	s.light = __float_as_int( n2.w );
	if ( need_ng )
	{
		float4 b = __ldg( tp + 1 ), c = __ldg( tp + 2 );
		s.ng = normalize( cross( f3( b ) - f3( a ), f3( c ) - f3( a ) ) );
	}
	else
		s.ng = s.ns;
	return s;
}

// Light point for the reference estimator: AreaLight::sample via
// Mesh::sample (mesh.hpp:92-98, 1024-point table) or Sphere::sample
// (sphere.hpp:22-30, theta uniform in [0, pi]); area pdf.
__device__ __forceinline__ void koishi_light_point( const DevScene &sc, const DevLight &lt, float ux, float uy,
													float3 &lp, float3 &ln, float &pdf )
{
	if ( lt.kind == LIGHT_MESH )
	{
		uint32_t k = min( uint32_t( floorf( ux * 1024.f ) ), 1023u );
		lp = f3( sc.light_tables[ 2 * ( lt.table + k ) ] );
		ln = f3( sc.light_tables[ 2 * ( lt.table + k ) + 1 ] );
		pdf = lt.koishi_pdf;
		return;
	}
	const DevSphere &sp = sc.spheres[ lt.index ];
	float th = ux * PI_F, ph = uy * PI_F * 2.f;
	float st, ct, sph, cph;
	sincosf( th, &st, &ct );
	sincosf( ph, &sph, &cph );
	float3 w = f3( st * sph, st * cph, ct );
	lp = f3( sp.c ) + w * sp.r;
	ln = w;
	pdf = 1.f / ( 4.f * PI_F * sp.r2 );
}

// Light point for the MIS estimator: area-proportional triangle, uniform point.
__device__ __forceinline__ void mis_light_point( const DevScene &sc, const DevLight &lt, float u0, float u1, float u2,
												 float3 &lp, float3 &ln, float &pdfA )
{
	if ( lt.kind == LIGHT_SPHERE )
	{
		const DevSphere &sp = sc.spheres[ lt.index ];
		float z = 1.f - 2.f * u1, r = sqrtf( fmaxf( 0.f, 1.f - z * z ) ), s, c;
		sincosf( 2.f * PI_F * u2, &s, &c );
		float3 w = f3( r * c, r * s, z );
		lp = f3( sp.c ) + w * sp.r;
		ln = w;
		pdfA = 1.f / lt.area;
		return;
	}
	const float *cdf = sc.light_cdf + lt.cdf;
	float target = u0 * cdf[ lt.n_tris - 1 ];
	int lo = 0, hi = lt.n_tris - 1;
	while ( lo < hi )
	{
		int mid = ( lo + hi ) >> 1;
		if ( cdf[ mid ] > target )
			hi = mid;
		else
			lo = mid + 1;
	}
	const float4 *tv = sc.light_tris + 3 * size_t( lt.index + lo );
	float3 v0 = f3( tv[ 0 ] ), v1 = f3( tv[ 1 ] ), v2 = f3( tv[ 2 ] );
	float su = sqrtf( u1 ), b0 = 1.f - su, b1 = u2 * su;
	lp = v0 * b0 + v1 * b1 + v2 * ( 1.f - b0 - b1 );
	ln = normalize( cross( v1 - v0, v2 - v0 ) );
	pdfA = 1.f / lt.area;
}

struct PathOut
{
	bool alive = false, shadow = false;
	float4 ro, rd, so, sd, sc;
};

// Light::sample of the reference estimator for a point p: the light point lp
// and the unoccluded radiance li it delivers.  Area lights
// (areaLight.hpp:19-31, Primitive::sample primitive.hpp:25-33) divide the
// emission by the solid-angle pdf; a point light (pointLight.hpp:21-29)
// delivers its emission as it is.
__device__ __forceinline__ void koishi_light_sample( const DevScene &sc, const DevLight &lt, float3 p, float ux, float uy,
													 float3 &lp, float3 &li )
{
	if ( lt.kind == LIGHT_POINT )
	{
		lp = f3( lt.pos );
		li = f3( lt.emission );
		return;
	}
	float3 ln;
	float pdf;
	koishi_light_point( sc, lt, ux, uy, lp, ln, pdf );
	const float3 wiw = p - lp;
	pdf *= dot( wiw, wiw ) / fabsf( dot( ln, normalize( wiw ) ) );
	li = f3( lt.emission ) / pdf;
}

// One vertex of RadianceKernel::execute (radiance.cu:22-71), reference
// semantics.  The vertex's numbers come in the reference's order: light
// choice and light point (draws 0-2, also reserved when the scene has no
// light), then the shaders' draws and the Russian roulette draw.  A shader
// without selection draws (all but Mixed and GlassBSDF) takes a fixed layout:
// sample3 = draws 3-5, roulette = draw 6.
// What a profiled vertex adds to its RadianceKernel::Slice record
// (radiance.cu:41-53): f for the light sample's direction, theta, the shader,
// and whether Russian roulette ended the path here.
struct ProfOut
{
	float3 f = { 0.f, 0.f, 0.f };
	float theta = 0.f;
	uint32_t shader = 0;
	bool rr_killed = false;
};

// PROF: a profiled render, whose paths follow the reference's loop exactly:
// a path whose throughput is zero (or whose radiance is not finite) goes on
// bouncing, as it does in radiance.cu, so that the Slice's bounce counter and
// records match.
template <bool PROF = false>
__device__ __forceinline__ void shade_koishi( const DevScene &sc, const RenderConfig &cfg, uint2 key, uint64_t g,
											  uint32_t bounce, float4 ro, float4 rd, const HitRec &h, float4 &beta4,
											  float4 &L4, PathOut &out, ProfOut *prof = nullptr )
{
	float3 o = f3( ro ), d = f3( rd );
	Surface s = surface_at( sc, o, d, h, false );
	Frame fr = koishi_frame( s.ns );
	float3 wo = fr.local( -d );
	float3 beta = f3( beta4 ), L = f3( L4 );
	const DevShader sh = sc.shaders[ s.shader ];
	const bool simple = sh.type != SH_MIXED && sh.type != SH_GLASS;
	const float4 r0 = rand4( key, g, bounce, 0 );
	VertexRng rng( key, g, bounce, r0, 3 );
	float3 wi = f3( 0.f, 0.f, 0.f );
	if ( sc.n_lights )
	{
		uint32_t nl = sc.n_lights;
		uint32_t idx = min( uint32_t( floorf( r0.x * float( nl ) ) ), nl - 1 );
		float lpdf = 1.f / float( nl );
		const DevLight lt = sc.lights[ idx ];
		const float ux = r0.y, uy = r0.z;
		float3 lp, li;
		koishi_light_sample( sc, lt, s.p, ux, uy, lp, li );
		float3 dd = lp - s.p;   // LocalVaryings::emitSeg (varyings.hpp:27-37)
		float3 sd = normalize( dd );
		float3 diff = normalize( sd ) * KOISHI_EPS;
		float3 so = s.p + diff;
		float st = length( dd - 2.f * diff );
		wi = fr.local( normalize( lp - s.p ) );
		float3 emission;
		float3 f = simple ? leaf_eval( sh, wo, wi, emission ) : koishi_eval( sc.shaders, s.shader, wo, wi, rng, emission );
		if constexpr ( PROF ) prof->f = f;
		float3 c = beta * f * li * ( fabsf( wi.z ) / lpdf );
		if ( !finite3( c ) )
			L = f3( NAN, NAN, NAN );
		else if ( !is_zero( c ) )
		{
			out.shadow = true;
			out.so = make_float4( so.x, so.y, so.z, 0.f );
			out.sd = make_float4( sd.x, sd.y, sd.z, st );
			out.sc = make_float4( c.x, c.y, c.z, 0.f );
		}
		L = L + beta * emission;  // radiance.cu:39
	}
	if constexpr ( PROF )
	{
		// theta = acos(wo . reflect(wi, +z)), reflect(v, n) = 2 n (n.v) - v (vmath.hpp)
		prof->theta = acosf( dot( wo, f3( -wi.x, -wi.y, wi.z ) ) );
		prof->shader = uint32_t( s.shader );
	}
	float3 emission_s, f;
	float u_rr;
	if ( simple )
	{
		const float4 r1 = rand4( key, g, bounce, 1 );
		f = leaf_sample( sh, wo, r0.w, r1.x, wi, emission_s );  // radiance.cu:55-60
		u_rr = r1.z;
	}
	else
	{
		f = koishi_sample( sc.shaders, s.shader, wo, rng, wi, emission_s );
		u_rr = rng.next();
	}
	beta = beta * f * fabsf( wi.z );
	float3 nd = fr.global( wi );
	float3 no = s.p + nd * KOISHI_EPS;
	bool alive = true;
	float rr = maxc( beta );  // radiance.cu:62-68
	if ( rr < 1.f && bounce > 3 )
	{
		float q = fmaxf( .05f, 1.f - rr );
		if ( u_rr < q )
		{
			alive = false;
			if constexpr ( PROF ) prof->rr_killed = true;
		}
		else
			beta = beta / ( 1.f - q );
	}
	if constexpr ( PROF )
	{
		if ( bounce + 1 > cfg.max_bounce ) alive = false;
	}
	else if ( bounce + 1 > cfg.max_bounce || is_zero( beta ) || !finite3( L ) || !finite3( beta ) )
		alive = false;
	if ( !finite3( L ) ) out.shadow = false;
	beta4 = make_float4( beta.x, beta.y, beta.z, 0.f );
	L4 = make_float4( L.x, L.y, L.z, 0.f );
	out.alive = alive;
	out.ro = make_float4( no.x, no.y, no.z, 0.f );
	out.rd = make_float4( nd.x, nd.y, nd.z, INFINITY );
}

// One vertex of the MIS estimator (power heuristic over BSDF sampling and
// area-light NEE; see cr_device.cuh for the BSDFs).
// The guide's proposal for one path vertex, written by the inference kernel
// already prepared for evaluation (9 x 16 bytes):
//   slot k < 8, lobe k: mean xyz and weight as FP16, then kappa log2(e) and
//                       log2(P_k * vMF normaliser) as FP32, P_k = weight /
//                       (sum of the 8 stored weights)
//   slot 8:             the probability of sampling the guide (FP32)
// Sampling (lobe k with probability P_k, then the vMF of mean mu_k and
// concentration kappa_k) and density evaluation (sum_k 2^(k2 (mu.w - 1) + c))
// read the same stored values, the means renormalised after FP16 decoding, so
// the density is the sampled one to FP32 rounding.  Shading reads the lobes
// from memory as it evaluates them and keeps none in registers.
constexpr uint32_t LOBE_SLOTS = 9;  // 16-byte slots per path

__device__ __forceinline__ void store_lobes( uint4 *dst, const Lobe *lb, float sel )
{
	__half wh[ G_LOBES ];
	float sum = 0.f;
#pragma unroll
	for ( int k = 0; k < G_LOBES; ++k )
	{
		wh[ k ] = __float2half_rn( lb[ k ].weight );
		sum += __half2float( wh[ k ] );
	}
	const float inv = sum > 0.f ? 1.f / sum : 0.f;
#pragma unroll
	for ( int k = 0; k < G_LOBES; ++k )
	{
		const float kap = lb[ k ].kappa;
		const float norm = kap / ( 2.f * PI_F * ( -expm1f( -2.f * kap ) ) );
		const float P = sum > 0.f ? __half2float( wh[ k ] ) * inv : 1.f / G_LOBES;
		const __half2 m01 = __floats2half2_rn( lb[ k ].mu.x, lb[ k ].mu.y );
		__half2 m2w = __floats2half2_rn( lb[ k ].mu.z, 0.f );
		m2w.y = sum > 0.f ? wh[ k ] : __float2half_rn( 1.f );
		dst[ k ] = make_uint4( *reinterpret_cast<const uint32_t *>( &m01 ), *reinterpret_cast<const uint32_t *>( &m2w ),
							   __float_as_uint( kap * 1.4426950408889634f ), __float_as_uint( log2f( P * norm ) ) );
	}
	dst[ 8 ] = make_uint4( __float_as_uint( sel ), 0u, 0u, 0u );
}

struct StoredLobe
{
	float3 mu;
	float weight, k2, c;
};

__device__ __forceinline__ StoredLobe load_lobe( const uint4 *rec, int k )
{
	const uint4 q = rec[ k ];
	const float2 m01 = __half22float2( *reinterpret_cast<const __half2 *>( &q.x ) );
	const float2 m2w = __half22float2( *reinterpret_cast<const __half2 *>( &q.y ) );
	StoredLobe l;
	const float3 m = f3( m01.x, m01.y, m2w.x );
	const float l2 = dot( m, m );
	l.mu = l2 > 1e-20f ? m * rsqrtf( l2 ) : f3( 0.f, 0.f, 1.f );
	l.weight = m2w.y;
	l.k2 = __uint_as_float( q.z );
	l.c = __uint_as_float( q.w );
	return l;
}

// The stored mixture's density at direction w.  The loop stays rolled: unrolled,
// the guided shading kernel held all 8 lobes of both of its calls in registers
// (170 of them) and ran 1.4x slower.
__device__ __forceinline__ float stored_pdf( const uint4 *rec, float3 w )
{
	float p = 0.f;
#pragma unroll 1
	for ( int k = 0; k < G_LOBES; ++k )
	{
		const StoredLobe l = load_lobe( rec, k );
		p += exp2f( fmaf( l.k2, dot( l.mu, w ) - 1.f, l.c ) );
	}
	return p;
}

// A direction from the stored mixture: lobe k with probability P_k (u0), then
// its vMF by the numerically stable inversion of Jakob ("Numerically stable
// sampling of the von Mises Fisher distribution on S2", 2012).
__device__ __forceinline__ float3 stored_sample( const uint4 *rec, float u0, float u1, float u2 )
{
	float sum = 0.f;
#pragma unroll
	for ( int k = 0; k < G_LOBES; ++k ) sum += __half2float( __ushort_as_half( uint16_t( rec[ k ].y >> 16 ) ) );
	const float target = u0 * sum;
	int k = 0;
	float acc = 0.f;
	for ( ; k < G_LOBES - 1; ++k )
	{
		acc += __half2float( __ushort_as_half( uint16_t( rec[ k ].y >> 16 ) ) );
		if ( target < acc ) break;
	}
	const StoredLobe l = load_lobe( rec, k );
	const float kappa = l.k2 * 0.6931471805599453f;
	float w = 1.f + logf( u1 + ( 1.f - u1 ) * expf( -2.f * kappa ) ) / kappa;
	w = fminf( fmaxf( w, -1.f ), 1.f );
	float r = sqrtf( fmaxf( 0.f, 1.f - w * w ) ), s, c;
	sincosf( 2.f * PI_F * u2, &s, &c );
	Frame f = onb_frame( l.mu );
	return normalize( f.u * ( r * c ) + f.v * ( r * s ) + f.n * w );
}

__device__ __forceinline__ void shade_mis( const DevScene &sc, const RenderConfig &cfg, uint2 key, uint64_t g,
										   uint32_t bounce, float4 ro, float4 rd, const HitRec &h, float4 &beta4,
										   float4 &L4, PathOut &out, const uint4 *lobes, uint32_t rec_i )
{
	float3 o = f3( ro ), d = f3( rd );
	Surface s = surface_at( sc, o, d, h, true );
	const DevShader sh = sc.shaders[ s.shader ];
	float3 beta = f3( beta4 ), L = f3( L4 );
	float nl = float( sc.n_lights );
	if ( sh.type == SH_EMISSION )
	{
		float w = 1.f;
		// beta4.w: the previous continuation's density, negative after a delta
		// (pass-through) continuation, which next-event estimation cannot sample
		if ( bounce > 0 && s.light >= 0 && beta4.w >= 0.f )
		{
			float cosl = fabsf( dot( s.ng, d ) );
			float pb = beta4.w;
			float pl = cosl > 0.f ? h.t * h.t / cosl / sc.lights[ s.light ].area / nl : INFINITY;
			w = pb * pb / ( pb * pb + pl * pl );
		}
		L = L + beta * f3( sh.emission ) * w;
	}
	// Training target of the previous vertex: the radiance gathered so far,
	// taken after this vertex's emission, so the target holds the light that
	// reached the previous vertex through this surface (indirect light) and
	// leaves the lights themselves to next-event estimation.
	if ( rec_i != 0xFFFFFFFFu && bounce > 0 ) cfg.rec.L[ rec_i - 1 ] = make_float4( L.x, L.y, L.z, 0.f );
	// Two-sided shading: the geometric normal faces the incoming ray and the
	// shading normal is put on the same side.  `entering`: the ray arrives from
	// outside the surface as built (the dielectrics' side).
	const bool entering = dot( s.ng, d ) < 0.f;
	if ( dot( s.ng, d ) > 0.f ) s.ng = -s.ng;
	if ( dot( s.ns, s.ng ) < 0.f ) s.ns = -s.ns;
	Frame fr = onb_frame( s.ns );
	float3 wo = fr.local( -d );
	float4 r0 = rand4( key, g, bounce, 0 ), r1 = rand4( key, g, bounce, 1 );
	// Lambert, Glossy and Emission take the reflection-only fast path; the
	// other shaders (dielectrics, pass-through, black, mixtures) the general one
	const bool simple = sh.type == SH_LAMBERT || sh.type == SH_GLOSSY || sh.type == SH_EMISSION;
	const bool transmits = !simple && ( mis_transmits( sh.type ) ||
										( sh.type == SH_MIXED && ( mis_transmits( sc.shaders[ sh.child[ 0 ] ].type ) ||
																   mis_transmits( sc.shaders[ sh.child[ 1 ] ].type ) ) ) );
	const bool guided = simple && cfg.guide_sample && guided_vertex( cfg.guide, bounce, cfg.max_bounce );
	// the probability of sampling the guide: fixed, or learned per vertex
	float sel = 0.f;
	if ( guided ) sel = cfg.guide.learn_select ? __uint_as_float( lobes[ 8 ].x ) : cfg.guide.select_prob;
	if ( sc.n_lights )
	{
		uint32_t nli = sc.n_lights;
		uint32_t idx = min( uint32_t( floorf( r0.x * nl ) ), nli - 1 );
		float ur = r0.x * nl - float( idx );
		const DevLight lt = sc.lights[ idx ];
		const bool point = lt.kind == LIGHT_POINT;
		float3 lp, ln = f3( 0.f, 0.f, 1.f );
		float pdfA = 1.f;
		if ( point )
			lp = f3( lt.pos );
		else
			mis_light_point( sc, lt, ur, r0.y, r0.z, lp, ln, pdfA );
		float3 dw = lp - s.p;
		float dist2 = dot( dw, dw ), dist = sqrtf( dist2 );
		float3 wiw = dw / dist;
		// a point light of intensity I = color * strength gives I cos / r^2 and
		// is reached by next-event estimation alone (weight 1)
		float cosl = point ? 1.f : fabsf( dot( ln, wiw ) );
		if ( cosl > 0.f && dist > 0.f && ( transmits || dot( wiw, s.ng ) > 0.f ) )
		{
			float pl = point ? dist2 / nl : pdfA * dist2 / cosl / nl;
			float3 wi = fr.local( wiw );
			float pb;
			float3 f = simple ? mis_eval( sh, wo, wi, pb ) : mis_eval_tab( sc.shaders, s.shader, wo, wi, entering, pb );
			// one-sample MIS of guide and BSDF: the continuation density
			if ( guided ) pb = sel * stored_pdf( lobes, wiw ) + ( 1.f - sel ) * pb;
			if ( !is_zero( f ) )
			{
				// the last vertex has no continuation that could reach the light:
				// its light sample takes the whole weight
				float w = bounce == cfg.max_bounce || point ? 1.f : pl * pl / ( pl * pl + pb * pb );
				float3 c = beta * f * f3( lt.emission ) * ( fabsf( wi.z ) * w / pl );
				if ( finite3( c ) && !is_zero( c ) )
				{
					// Both ends leave their surfaces: the shading point along its
					// geometric normal (on the light's side), the light point along
					// the light's normal towards the shading point; the ray runs
					// between the two.  A point light is its own end.
					float3 so = offset_ray( s.p, dot( wiw, s.ng ) > 0.f ? s.ng : -s.ng );
					float3 to = point ? lp : offset_ray( lp, dot( ln, wiw ) < 0.f ? ln : -ln );
					float3 sd = to - so;
					float len = length( sd );
					sd = sd / len;
					out.shadow = true;
					out.so = make_float4( so.x, so.y, so.z, 0.f );
					out.sd = make_float4( sd.x, sd.y, sd.z, len );
					out.sc = make_float4( c.x, c.y, c.z, 0.f );
				}
			}
		}
	}
	float3 wi;
	float pdf;
	float pb_s = 0.f;  // the BSDF density of the sampled direction (training records)
	float3 wt, nd;
	bool delta = false;
	if ( !simple )
	{
		// a selection number for Mixed and the dielectrics
		const float us = rand4( key, g, bounce, 2 ).x;
		wt = mis_sample_tab( sc.shaders, s.shader, wo, entering, us, r1.x, r1.y, wi, pdf, delta );
		nd = fr.global( wi );
		pb_s = pdf;
	}
	else if ( guided )
	{
		// one-sample MIS: the guide with probability sel, else the BSDF; the
		// weight uses the combined density of both strategies
		if ( r1.z < sel )
		{
			nd = stored_sample( lobes, r1.w, r1.x, r1.y );
			wi = fr.local( nd );
		}
		else
		{
			mis_sample( sh, wo, r1.x, r1.y, wi, pdf );
			nd = fr.global( wi );
		}
		float pb;
		float3 f = mis_eval( sh, wo, wi, pb );
		pdf = sel * stored_pdf( lobes, nd ) + ( 1.f - sel ) * pb;
		wt = pdf > 0.f ? f * ( wi.z / pdf ) : f3( 0.f, 0.f, 0.f );
		pb_s = pb;
	}
	else
	{
		wt = mis_sample( sh, wo, r1.x, r1.y, wi, pdf );
		nd = fr.global( wi );
		pb_s = pdf;
	}
	beta = beta * wt;
	// a continuation through the surface leaves from its far side
	const bool through = wi.z < 0.f;
	bool alive = !is_zero( beta ) && ( through ? dot( nd, s.ng ) < 0.f : dot( nd, s.ng ) > 0.f );
	float rr = maxc( beta );
	if ( alive && rr < 1.f && bounce >= cfg.rr_start )
	{
		float q = fmaxf( .05f, 1.f - rr );
		if ( r0.w < q )
			alive = false;
		else
			beta = beta / ( 1.f - q );
	}
	if ( bounce + 1 > cfg.max_bounce || !finite3( beta ) ) alive = false;
	float3 no = offset_ray( s.p, through ? -s.ng : s.ng );
	if ( delta ) pdf = 0.f;  // no density: not a training sample
	if ( rec_i != 0xFFFFFFFFu )
	{
		// training record of this vertex (its radiance target follows once the
		// rest of the path is known)
		cfg.rec.x[ rec_i ] = make_float4( s.p.x, s.p.y, s.p.z, alive ? 1.f : 0.f );
		// w: luminance of f * cos for the sampled direction (wt = f cos / pdf)
		cfg.rec.wo[ rec_i ] = make_float4( -d.x, -d.y, -d.z, lum( wt ) * pdf );
		cfg.rec.n[ rec_i ] = make_float4( s.ns.x, s.ns.y, s.ns.z, delta ? 0.f : pb_s );
		cfg.rec.om[ rec_i ] = make_float4( nd.x, nd.y, nd.z, pdf );
		cfg.rec.T[ rec_i ] = make_float4( beta.x, beta.y, beta.z, 0.f );
	}
	beta4 = make_float4( beta.x, beta.y, beta.z, delta ? -1.f : pdf );
	L4 = make_float4( L.x, L.y, L.z, 0.f );
	out.alive = alive;
	out.ro = make_float4( no.x, no.y, no.z, 0.f );
	out.rd = make_float4( nd.x, nd.y, nd.z, INFINITY );
}

__device__ __forceinline__ uint2 philox_key( uint64_t seed )
{
	return make_uint2( uint32_t( seed ), uint32_t( seed >> 32 ) ^ 0x5EED5EEDu );
}

// Last job whose first global sample (pixel) is <= g: binary search.
template <bool PIXELS>
__device__ __forceinline__ uint32_t find_job( const BatchJobDev *jobs, uint32_t n, uint64_t g )
{
	uint32_t lo = 0, hi = n;
	while ( hi - lo > 1 )
	{
		uint32_t mid = ( lo + hi ) >> 1;
		if ( ( PIXELS ? jobs[ mid ].first_pixel : jobs[ mid ].first_sample ) <= g )
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

// Camera rays of a batched wave: global sample -> job -> pixel and sample index.
__global__ void k_generate_batch( BatchDev bd, WaveBuffers wb )
{
	const WaveArgs wa{ wb.bwave->first, wb.bwave->n };
	if ( blockIdx.x == 0 && threadIdx.x == 0 ) wb.counters[ CNT_EXT ] = wa.n;
	for ( uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < wa.n; s += gridDim.x * blockDim.x )
	{
		const uint64_t g = wa.first + s;
		const uint32_t j = find_job<false>( bd.jobs, bd.n_jobs, g );
		const BatchJobDev &job = bd.jobs[ j ];
		const uint64_t local = g - job.first_sample;
		const uint32_t pix = uint32_t( local / job.spp ), k = uint32_t( local % job.spp );
		const uint32_t x = pix % job.width, y = pix / job.width;
		float3 o, d;
		camera_ray( bd.scenes[ j ].cam, x, y, k, o, d );
		wb.ray_o[ s ] = make_float4( o.x, o.y, o.z, 0.f );
		wb.ray_d[ s ] = make_float4( d.x, d.y, d.z, INFINITY );
		wb.beta[ s ] = make_float4( 1.f, 1.f, 1.f, 0.f );
		wb.L[ s ] = make_float4( 0.f, 0.f, 0.f, 0.f );
		wb.queue[ 0 ][ s ] = s;
		wb.path_job[ s ] = j;
	}
}

// BATCH: the wave mixes several jobs; each path shades in its job's scene with
// its job's random key, and `sc` and `key` are unused.
// One instantiation per estimator, so that the reference estimator's shading
// is not held to the registers of the guided MIS shading.
// PROF: a profiled render (reference estimator, one scene): each shaded vertex
// writes its bounce record and each ending path its slice's bounce counter.
// GUIDED: a guided MIS render (lobes and training records); plain MIS renders
// take the instantiation without the guide's code, and its registers.
template <bool BATCH, int EST, bool PROF = false, bool GUIDED = false>
__global__ void __launch_bounds__( 256 ) k_shade( DevScene sc, RenderConfig cfg, WaveBuffers wb, WaveArgs wa,
												  uint32_t bounce, uint2 key, BatchDev bd )
{
	if constexpr ( BATCH ) wa = WaveArgs{ wb.bwave->first, wb.bwave->n };  // the wave runs from device memory
	const uint32_t n = wb.counters[ CPB * bounce + CNT_EXT ];
	const uint32_t *q = wb.queue[ bounce & 1 ];
	uint32_t *nq = wb.queue[ ( bounce + 1 ) & 1 ];
	uint32_t *next_count = wb.counters + CPB * ( bounce + 1 ) + CNT_EXT;
	uint32_t *shadow_count = wb.counters + CPB * bounce + CNT_SHADOW;
	const uint32_t stride = gridDim.x * blockDim.x;
	// The next iteration's queue entry and hit record are fetched one iteration
	// ahead, so their latency overlaps this iteration's shading (5 % off the
	// shading of the 1.31M-triangle scene).  Guided shading, at the register
	// limit already, fetches in place.
	constexpr bool PREFETCH = !GUIDED;
	uint32_t pf_path = 0;
	HitRec pf_h{};
	if constexpr ( PREFETCH )
	{
		const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
		if ( i0 < n ) pf_path = q[ i0 ], pf_h = wb.hit[ pf_path ];
	}
	for ( uint32_t base = blockIdx.x * blockDim.x + threadIdx.x - lane_id(); base < n; base += stride )
	{
		uint32_t i = base + lane_id();
		PathOut out;
		uint32_t path = 0;
		uint32_t cur_path = 0;
		HitRec cur_h{};
		if constexpr ( PREFETCH )
		{
			cur_path = pf_path, cur_h = pf_h;
			if ( i + stride < n ) pf_path = q[ i + stride ], pf_h = wb.hit[ pf_path ];
		}
		if ( i < n )
		{
			if constexpr ( PREFETCH )
				path = cur_path;
			else
				path = q[ i ];
			HitRec h = PREFETCH ? cur_h : wb.hit[ path ];
			const uint32_t stride = cfg.max_bounce + 1;
			uint32_t rec_j = 0xFFFFFFFFu;
			if ( GUIDED && cfg.guiding && path >= cfg.rec_offset )
			{
				uint32_t off = path - cfg.rec_offset, j = off / cfg.rec_stride;
				if ( j * cfg.rec_stride == off && j < cfg.rec_paths ) rec_j = j;
			}
			const bool recorded = rec_j != 0xFFFFFFFFu;
			if constexpr ( PROF )
			{
				// the loop's intersect failed here: the slice counts `bounce` vertices
				if ( h.id == HIT_MISS ) cfg.prof.slices[ wa.first + path ].bounce = bounce;
			}
			if ( recorded && bounce > 0 && h.id == HIT_MISS )
			{
				// the previous vertex's continuation left the scene: no indirect light
				float4 Lp = wb.L[ path ];
				cfg.rec.L[ rec_j * stride + bounce - 1 ] = make_float4( Lp.x, Lp.y, Lp.z, 0.f );
			}
			if ( h.id != HIT_MISS )
			{
				float4 beta = wb.beta[ path ], L = wb.L[ path ];
				float4 ro = wb.ray_o[ path ], rd = wb.ray_d[ path ];
				// Random streams are keyed by the absolute (pixel, sample), so a
				// film does not depend on the window or the wave size.
				uint64_t gw = wa.first + path;
				if constexpr ( BATCH )
				{
					// a job renders its whole image: its local sample index is the key
					const uint32_t j = wb.path_job[ path ];
					const BatchJobDev &job = bd.jobs[ j ];
					const uint2 jkey = philox_key( job.seed + *bd.seed_offset );
					const uint64_t g = gw - job.first_sample;
					if constexpr ( EST == EST_MIS )
						shade_mis( bd.scenes[ j ], cfg, jkey, g, bounce, ro, rd, h, beta, L, out, nullptr, 0xFFFFFFFFu );
					else
						shade_koishi( bd.scenes[ j ], cfg, jkey, g, bounce, ro, rd, h, beta, L, out );
				}
				else
				{
					uint32_t pix = uint32_t( gw / cfg.spp ), k = uint32_t( gw % cfg.spp );
					uint64_t g = ( uint64_t( cfg.y0 + pix / cfg.ww ) * sc.cam.width + cfg.x0 + pix % cfg.ww ) * cfg.spp + k;
					if constexpr ( EST == EST_MIS && GUIDED )
						shade_mis( sc, cfg, key, g, bounce, ro, rd, h, beta, L, out,
								   cfg.guide_sample ? wb.lobes + size_t( path ) * LOBE_SLOTS : nullptr,
								   recorded ? rec_j * stride + bounce : 0xFFFFFFFFu );
					else if constexpr ( EST == EST_MIS )
						shade_mis( sc, cfg, key, g, bounce, ro, rd, h, beta, L, out, nullptr, 0xFFFFFFFFu );
					else if constexpr ( PROF )
					{
						ProfOut po;
						shade_koishi<true>( sc, cfg, key, g, bounce, ro, rd, h, beta, L, out, &po );
						// the window is the profiler's area: a path's sample index in the
						// window is its slice (Profiler::at, kernel.hpp:62-68)
						const uint64_t si = wa.first + path;
						if ( bounce < cfg.prof.depth )
						{
							cr_profile_bounce &r = cfg.prof.bounces[ si * cfg.prof.depth + bounce ];
							r.ray_o[ 0 ] = ro.x, r.ray_o[ 1 ] = ro.y, r.ray_o[ 2 ] = ro.z;
							r.ray_d[ 0 ] = rd.x, r.ray_d[ 1 ] = rd.y, r.ray_d[ 2 ] = rd.z;
							r.f[ 0 ] = po.f.x, r.f[ 1 ] = po.f.y, r.f[ 2 ] = po.f.z;
							r.theta = po.theta;
							r.L[ 0 ] = L.x, r.L[ 1 ] = L.y, r.L[ 2 ] = L.z;  // the light sample's share follows
							r.shader = po.shader;
						}
						// Russian roulette breaks before ++bounce; otherwise the loop
						// counts this vertex
						if ( !out.alive ) cfg.prof.slices[ si ].bounce = po.rr_killed ? bounce : bounce + 1;
					}
					else
						shade_koishi( sc, cfg, key, g, bounce, ro, rd, h, beta, L, out );
				}
				wb.beta[ path ] = beta;
				wb.L[ path ] = L;
				if ( out.alive )
				{
					wb.ray_o[ path ] = out.ro;
					wb.ray_d[ path ] = out.rd;
				}
				if ( out.shadow )
				{
					wb.sh_o[ path ] = out.so;
					wb.sh_d[ path ] = out.sd;
					wb.sh_c[ path ] = out.sc;
				}
			}
		}
		uint32_t si = warp_append( out.shadow, shadow_count );
		if ( out.shadow ) wb.shadow_queue[ si ] = path;
		uint32_t ni = warp_append( out.alive, next_count );
		if ( out.alive ) nq[ ni ] = path;
	}
}

// Guide inference for the paths of one bounce that hit a surface: inputs as
// the MIS shading sees them (position, outgoing direction, two-sided shading
// normal), BF16 tensor-core forward pass (guide_tc.cuh), mixture parameters
// per path.
__global__ void __launch_bounds__( tc::THREADS, 2 ) k_guide_infer( DevScene sc, RenderConfig cfg, WaveBuffers wb,
																	uint32_t bounce, const uint8_t *Wp )
{
	const uint32_t n = wb.counters[ CPB * bounce + CNT_EXT ];
	const uint32_t *q = wb.queue[ bounce & 1 ];
	auto src = [&]( uint32_t i, float3 &x, float3 &wo, float3 &nrm ) -> bool {
		const uint32_t path = q[ i ];
		const HitRec h = wb.hit[ path ];
		if ( h.id == HIT_MISS ) return false;
		const float3 o = f3( wb.ray_o[ path ] ), d = f3( wb.ray_d[ path ] );
		Surface s = surface_at( sc, o, d, h, true );
		if ( dot( s.ng, d ) > 0.f ) s.ng = -s.ng;
		if ( dot( s.ns, s.ng ) < 0.f ) s.ns = -s.ns;
		x = s.p, wo = -d, nrm = s.ns;
		return true;
	};
	auto sink = [&]( uint32_t i, const float *out ) {
		Lobe lb[ G_LOBES ];
		lobes_from_output( out, lb );
		store_lobes( wb.lobes + size_t( q[ i ] ) * LOBE_SLOTS, lb,
					 cfg.guide.learn_select ? guide_selection( out ) : cfg.guide.select_prob );
	};
	tc::mlp_forward_tc<48>( cfg.guide, Wp, n, src, sink, wb.err );
}

// Profiled renders: after the any-hit pass of `bounce`, each shaded vertex's
// record takes the path's radiance with its light sample's share (the
// reference adds the occlusion-tested light sample before it records L).
__global__ void k_profile_fix( RenderConfig cfg, WaveBuffers wb, WaveArgs wa, uint32_t bounce )
{
	const uint32_t n = wb.counters[ CPB * bounce + CNT_EXT ];
	const uint32_t *q = wb.queue[ bounce & 1 ];
	if ( bounce >= cfg.prof.depth ) return;
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		const uint32_t path = q[ i ];
		if ( wb.hit[ path ].id == HIT_MISS ) continue;
		const float4 l = wb.L[ path ];
		float *L = cfg.prof.bounces[ ( wa.first + path ) * cfg.prof.depth + bounce ].L;
		L[ 0 ] = l.x, L[ 1 ] = l.y, L[ 2 ] = l.z;
	}
}

// Profiled renders, end of a wave: each slice takes its sample's radiance.
__global__ void k_profile_final( RenderConfig cfg, WaveBuffers wb, WaveArgs wa )
{
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wa.n; i += gridDim.x * blockDim.x )
	{
		const float4 l = wb.L[ i ];
		float *L = cfg.prof.slices[ wa.first + i ].L;
		L[ 0 ] = l.x, L[ 1 ] = l.y, L[ 2 ] = l.z;
	}
}

__global__ void k_accumulate( RenderConfig cfg, WaveBuffers wb, WaveArgs wa, double *sum, double *sumsq,
							  uint32_t *count )
{
	uint64_t p0 = wa.first / cfg.spp, p1 = ( wa.first + wa.n - 1 ) / cfg.spp;
	for ( uint64_t p = p0 + blockIdx.x * blockDim.x + threadIdx.x; p <= p1; p += gridDim.x * blockDim.x )
	{
		uint64_t s0 = max( p * cfg.spp, wa.first ), s1 = min( ( p + 1 ) * cfg.spp, wa.first + wa.n );
		double a0 = 0, a1 = 0, a2 = 0, q0 = 0, q1 = 0, q2 = 0;
		uint32_t c = 0;
		for ( uint64_t s = s0; s < s1; ++s )
		{
			float4 l = wb.L[ s - wa.first ];
			if ( !isfinite( l.x ) || !isfinite( l.y ) || !isfinite( l.z ) ) continue;  // cpuMulticore.cu:58-64
			++c;
			a0 += l.x, a1 += l.y, a2 += l.z;
			q0 += double( l.x ) * l.x, q1 += double( l.y ) * l.y, q2 += double( l.z ) * l.z;
		}
		sum[ 3 * p ] += a0, sum[ 3 * p + 1 ] += a1, sum[ 3 * p + 2 ] += a2;
		sumsq[ 3 * p ] += q0, sumsq[ 3 * p + 1 ] += q1, sumsq[ 3 * p + 2 ] += q2;
		count[ p ] += c;
	}
}

// The reference's debug kernels on the bounce-0 hits (L was zeroed by
// k_generate): NormalKernel (normal.hpp:17-31) writes n * 0.5 + 0.5;
// HalfVectorKernel (halfVector.hpp:17-43) the angle between the normal and the
// half vector of the view direction and a light-0 sample, * 2 / pi;
// VisibilityKernel (visibility.hpp:17-41) queues the light-0 sample's segment,
// whose any-hit pass adds (1, 1, 1) when it is unoccluded and its radiance
// E / pdf is not zero.  Light sampling is AreaLight::sample as in
// shade_koishi, with the reference's 4e-3 segment offsets.
__global__ void __launch_bounds__( 128 ) k_aov( DevScene sc, RenderConfig cfg, WaveBuffers wb, WaveArgs wa, uint2 key )
{
	const uint32_t n = wb.counters[ CNT_EXT ];
	const uint32_t *q = wb.queue[ 0 ];
	uint32_t *shadow_count = wb.counters + CNT_SHADOW;
	const uint32_t stride = gridDim.x * blockDim.x;
	for ( uint32_t base = blockIdx.x * blockDim.x + threadIdx.x - lane_id(); base < n; base += stride )
	{
		const uint32_t i = base + lane_id();
		bool shadow = false;
		uint32_t path = 0;
		if ( i < n )
		{
			path = q[ i ];
			const HitRec h = wb.hit[ path ];
			if ( h.id != HIT_MISS )
			{
				const float3 o = f3( wb.ray_o[ path ] ), d = f3( wb.ray_d[ path ] );
				const Surface s = surface_at( sc, o, d, h, false );
				float3 L = f3( 0.f, 0.f, 0.f );
				if ( cfg.kernel == KERNEL_NORMAL )
					L = s.ns * 0.5f + f3( 0.5f, 0.5f, 0.5f );
				else
				{
					const uint64_t gw = wa.first + path;
					const uint32_t pix = uint32_t( gw / cfg.spp ), k = uint32_t( gw % cfg.spp );
					const uint64_t g =
						( uint64_t( cfg.y0 + pix / cfg.ww ) * sc.cam.width + cfg.x0 + pix % cfg.ww ) * cfg.spp + k;
					const float4 r0 = rand4( key, g, 0, 0 );
					const DevLight lt = sc.lights[ 0 ];
					float3 lp, li;
					koishi_light_sample( sc, lt, s.p, r0.x, r0.y, lp, li );
					if ( cfg.kernel == KERNEL_HALFVECTOR )
					{
						const Frame fr = koishi_frame( s.ns );
						const float3 wo = fr.local( -d ), wi = fr.local( normalize( lp - s.p ) );
						const float a = acosf( normalize( wi + wo ).z ) * ( 2.f / PI_F );
						L = f3( a, a, a );
					}
					else
					{
						if ( !( li.x == 0.f && li.y == 0.f && li.z == 0.f ) )
						{
							const float3 dd = lp - s.p;
							const float3 sd = normalize( dd );
							const float3 diff = sd * KOISHI_EPS;
							const float3 so = s.p + diff;
							wb.sh_o[ path ] = make_float4( so.x, so.y, so.z, 0.f );
							wb.sh_d[ path ] = make_float4( sd.x, sd.y, sd.z, length( dd - 2.f * diff ) );
							wb.sh_c[ path ] = make_float4( 1.f, 1.f, 1.f, 0.f );
							shadow = true;
						}
					}
				}
				wb.L[ path ] = make_float4( L.x, L.y, L.z, 0.f );
			}
		}
		const uint32_t si = warp_append( shadow, shadow_count );
		if ( shadow ) wb.shadow_queue[ si ] = path;
	}
}

// Film accumulation of a batched wave: global pixels p0..p1 (those whose
// samples meet the wave), each into its job's film.
__global__ void k_accumulate_batch( BatchDev bd, WaveBuffers wb )
{
	const BatchWave w = *wb.bwave;
	const WaveArgs wa{ w.first, w.n };
	for ( uint64_t p = w.p0 + blockIdx.x * blockDim.x + threadIdx.x; p <= w.p1 && w.n; p += gridDim.x * blockDim.x )
	{
		const uint32_t j = find_job<true>( bd.jobs, bd.n_jobs, p );
		const BatchJobDev &job = bd.jobs[ j ];
		const uint64_t lp = p - job.first_pixel;
		const uint64_t f0 = job.first_sample + lp * job.spp;
		uint64_t s0 = max( f0, wa.first ), s1 = min( f0 + job.spp, wa.first + wa.n );
		double a0 = 0, a1 = 0, a2 = 0, q0 = 0, q1 = 0, q2 = 0;
		uint32_t c = 0;
		for ( uint64_t s = s0; s < s1; ++s )
		{
			float4 l = wb.L[ s - wa.first ];
			if ( !isfinite( l.x ) || !isfinite( l.y ) || !isfinite( l.z ) ) continue;  // cpuMulticore.cu:58-64
			++c;
			a0 += l.x, a1 += l.y, a2 += l.z;
			q0 += double( l.x ) * l.x, q1 += double( l.y ) * l.y, q2 += double( l.z ) * l.z;
		}
		job.sum[ 3 * lp ] += a0, job.sum[ 3 * lp + 1 ] += a1, job.sum[ 3 * lp + 2 ] += a2;
		job.sumsq[ 3 * lp ] += q0, job.sumsq[ 3 * lp + 1 ] += q1, job.sumsq[ 3 * lp + 2 ] += q2;
		job.count[ lp ] += c;
	}
}

// Global pixel of global sample g of a batch.
__device__ __forceinline__ uint64_t batch_pixel( const BatchDev &bd, uint64_t g )
{
	const BatchJobDev &job = bd.jobs[ find_job<false>( bd.jobs, bd.n_jobs, g ) ];
	return job.first_pixel + ( g - job.first_sample ) / job.spp;
}

// Before the first wave of a batched render: wave 0, ray tally cleared.
__global__ void k_batch_init( WaveBuffers wb )
{
	if ( threadIdx.x || blockIdx.x ) return;
	wb.bwave->index = 0;
	wb.tally[ 0 ] = wb.tally[ 1 ] = 0;
}

// Start of a batched wave: its samples and pixel range from its index, and
// cleared queue counters.  One block.
__global__ void k_batch_wave_begin( BatchDev bd, WaveBuffers wb, uint64_t total, uint32_t wave_paths )
{
	for ( uint32_t i = threadIdx.x; i < wb.n_counters; i += blockDim.x ) wb.counters[ i ] = 0;
	if ( threadIdx.x ) return;
	BatchWave &w = *wb.bwave;
	const uint64_t first = uint64_t( w.index ) * wave_paths;
	w.first = first;
	if ( first >= total )  // no wave this far (the loop stops before it)
	{
		w.n = 0, w.p0 = 1, w.p1 = 0;
		return;
	}
	w.n = total - first < wave_paths ? uint32_t( total - first ) : wave_paths;
	w.p0 = batch_pixel( bd, first );
	w.p1 = batch_pixel( bd, first + w.n - 1 );
}

// End of a batched wave: adds its queue lengths to the running ray tally,
// advances the wave index and, in the graph, runs the loop again while waves
// remain.
__global__ void k_batch_wave_end( WaveBuffers wb, uint32_t max_bounce, uint64_t total, uint32_t wave_paths,
								  cudaGraphConditionalHandle loop, int looped )
{
	if ( threadIdx.x || blockIdx.x ) return;
	unsigned long long e = 0, sh = 0;
	for ( uint32_t b = 0; b <= max_bounce; ++b )
		e += wb.counters[ CPB * b + CNT_EXT ], sh += wb.counters[ CPB * b + CNT_SHADOW ];
	wb.tally[ 0 ] += e, wb.tally[ 1 ] += sh;
	const uint32_t next = wb.bwave->index + 1;
	wb.bwave->index = next;
	if ( looped ) cudaGraphSetConditional( loop, uint64_t( next ) * wave_paths < total ? 1u : 0u );
}

// Single-node shader kernels behind cr_bsdf_eval / cr_bsdf_sample (the host
// refuses shaders that draw selection numbers there).
__global__ void k_bsdf_eval( int est, DevShader sh, const float *wo, const float *wi, uint64_t n, float *f, float *pdf )
{
	const DevShader tab[ 1 ] = { sh };
	for ( uint64_t i = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; i < n; i += uint64_t( gridDim.x ) * blockDim.x )
	{
		float3 o = f3( wo + 3 * i ), w = f3( wi + 3 * i ), r, e;
		float p = 0.f;
		if ( est == EST_MIS )
			r = mis_eval( sh, o, w, p );
		else
		{
			ArrayRng rng{ nullptr, 0, 0 };
			r = koishi_eval( tab, 0, o, w, rng, e );
		}
		f[ 3 * i ] = r.x, f[ 3 * i + 1 ] = r.y, f[ 3 * i + 2 ] = r.z;
		pdf[ i ] = p;
	}
}

__global__ void k_bsdf_sample( int est, DevShader sh, const float *wo, const float *u, uint64_t n, float *wi, float *wt,
							   float *pdf )
{
	const DevShader tab[ 1 ] = { sh };
	for ( uint64_t i = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; i < n; i += uint64_t( gridDim.x ) * blockDim.x )
	{
		float3 o = f3( wo + 3 * i ), w = f3( 0.f, 0.f, 0.f ), r, e;
		float p = 0.f;
		if ( est == EST_MIS )
			r = mis_sample( sh, o, u[ 2 * i ], u[ 2 * i + 1 ], w, p );
		else
		{
			ArrayRng rng{ u + 2 * i, 2, 0 };
			r = koishi_sample( tab, 0, o, rng, w, e );
			r = r * fabsf( w.z );
		}
		wi[ 3 * i ] = w.x, wi[ 3 * i + 1 ] = w.y, wi[ 3 * i + 2 ] = w.z;
		wt[ 3 * i ] = r.x, wt[ 3 * i + 1 ] = r.y, wt[ 3 * i + 2 ] = r.z;
		pdf[ i ] = p;
	}
}

// Shader::execute of table entry 0 (nested Mixed entries follow it) over n
// samples with scripted uniforms, k per sample (cr_shader_execute).
__global__ void k_shader_execute( const DevShader *tab, int target, const float *wo, float *wi, const float *u,
								  uint32_t k, uint64_t n, float *f, float *em, uint32_t *used )
{
	for ( uint64_t i = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; i < n; i += uint64_t( gridDim.x ) * blockDim.x )
	{
		float3 o = f3( wo + 3 * i ), w = f3( wi + 3 * i ), r, e;
		ArrayRng rng{ u + uint64_t( k ) * i, k, 0 };
		if ( target == 0 )
			r = koishi_eval( tab, 0, o, w, rng, e );
		else
			r = koishi_sample( tab, 0, o, rng, w, e );
		wi[ 3 * i ] = w.x, wi[ 3 * i + 1 ] = w.y, wi[ 3 * i + 2 ] = w.z;
		f[ 3 * i ] = r.x, f[ 3 * i + 1 ] = r.y, f[ 3 * i + 2 ] = r.z;
		em[ 3 * i ] = e.x, em[ 3 * i + 1 ] = e.y, em[ 3 * i + 2 ] = e.z;
		used[ i ] = rng.used;
	}
}

// The render's generator on scripted (counter, key) pairs (cr_philox4x32_10).
__global__ void k_philox( const uint32_t *ck, uint64_t n, uint32_t *out )
{
	for ( uint64_t i = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; i < n; i += uint64_t( gridDim.x ) * blockDim.x )
	{
		const uint32_t *q = ck + 6 * i;
		const uint4 r = philox4x32_10( make_uint4( q[ 0 ], q[ 1 ], q[ 2 ], q[ 3 ] ), make_uint2( q[ 4 ], q[ 5 ] ) );
		out[ 4 * i ] = r.x, out[ 4 * i + 1 ] = r.y, out[ 4 * i + 2 ] = r.z, out[ 4 * i + 3 ] = r.w;
	}
}

void check( cudaError_t e, const char *what )
{
	if ( e != cudaSuccess ) throw std::runtime_error( std::string( what ) + ": " + cudaGetErrorString( e ) );
}

// Wave state comes from the library's own memory pool of the current device.
template <typename T>
void alloc( T *&p, size_t n, cudaStream_t st )
{
	check( cudaMallocFromPoolAsync( (void **)&p, sizeof( T ) * std::max<size_t>( n, 1 ), device_pool(), st ), "wave alloc" );
}

struct EventPool
{
	std::vector<cudaEvent_t> ev;
	size_t used = 0;
	cudaEvent_t get()
	{
		if ( used == ev.size() )
		{
			cudaEvent_t e;
			check( cudaEventCreate( &e ), "event" );
			ev.push_back( e );
		}
		return ev[ used++ ];
	}
	~EventPool()
	{
		for ( auto e : ev ) cudaEventDestroy( e );
	}
};

}  // namespace

namespace
{
constexpr int MAX_DEVICES = 64;
std::mutex g_dev_mutex;
int g_sms[ MAX_DEVICES ] = {};
std::set<std::pair<int, const void *>> g_smem_set;

int current_device()
{
	int dev = 0;
	check( cudaGetDevice( &dev ), "cudaGetDevice" );
	return dev;
}
}  // namespace

// One memory pool per device for the library's stream-ordered allocations (wave
// state, the BVH build's scratch and output, scene upload staging, the films of
// host-array calls), whose release threshold keeps freed memory mapped: the
// next scene's or render's buffers then reuse it instead of mapping hundreds of
// MB to gigabytes of device memory again.  trim_device_pools (cr_trim_memory)
// hands the cached memory back.
namespace
{
cudaMemPool_t g_pools[ MAX_DEVICES ] = {};
}

cudaMemPool_t device_pool()
{
	const int dev = current_device();
	if ( dev < 0 || dev >= MAX_DEVICES ) throw std::runtime_error( "device index out of range" );
	std::lock_guard<std::mutex> lock( g_dev_mutex );
	if ( !g_pools[ dev ] )
	{
		cudaMemPoolProps props{};
		props.allocType = cudaMemAllocationTypePinned;
		props.handleTypes = cudaMemHandleTypeNone;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id = dev;
		cudaMemPool_t pool = nullptr;
		check( cudaMemPoolCreate( &pool, &props ), "memory pool" );
		uint64_t keep = UINT64_MAX;
		check( cudaMemPoolSetAttribute( pool, cudaMemPoolAttrReleaseThreshold, &keep ), "memory pool" );
		g_pools[ dev ] = pool;
	}
	return g_pools[ dev ];
}

void trim_device_pools()
{
	std::lock_guard<std::mutex> lock( g_dev_mutex );
	for ( cudaMemPool_t pool : g_pools )
		if ( pool ) check( cudaMemPoolTrimTo( pool, 0 ), "memory pool trim" );
}

int sm_count()
{
	const int dev = current_device();
	if ( dev < 0 || dev >= MAX_DEVICES ) throw std::runtime_error( "device index out of range" );
	std::lock_guard<std::mutex> lock( g_dev_mutex );
	if ( !g_sms[ dev ] )
	{
		int n = 0;
		check( cudaDeviceGetAttribute( &n, cudaDevAttrMultiProcessorCount, dev ), "SM count" );
		g_sms[ dev ] = n > 0 ? n : 148;
	}
	return g_sms[ dev ];
}

void ensure_smem_limit( const void *fn, int bytes, const char *what )
{
	const int dev = current_device();
	std::lock_guard<std::mutex> lock( g_dev_mutex );
	if ( g_smem_set.count( { dev, fn } ) ) return;
	check( cudaFuncSetAttribute( fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes ), what );
	g_smem_set.insert( { dev, fn } );
}

void alloc_wave( WaveBuffers &wb, uint32_t capacity, uint32_t max_bounce, cudaStream_t st )
{
	wb.capacity = capacity;
	alloc( wb.ray_o, capacity, st );
	alloc( wb.ray_d, capacity, st );
	alloc( wb.hit, capacity, st );
	alloc( wb.beta, capacity, st );
	alloc( wb.L, capacity, st );
	alloc( wb.queue[ 0 ], capacity, st );
	alloc( wb.queue[ 1 ], capacity, st );
	alloc( wb.shadow_queue, capacity, st );
	alloc( wb.sh_o, capacity, st );
	alloc( wb.sh_d, capacity, st );
	alloc( wb.sh_c, capacity, st );
	wb.n_counters = n_counters_for( max_bounce );
	alloc( wb.counters, wb.n_counters, st );
	alloc( wb.err, 1, st );
	alloc( wb.work, 4, st );
	check( cudaMemsetAsync( wb.err, 0, sizeof( uint32_t ), st ), "wave init" );
}

void free_wave( WaveBuffers &wb, cudaStream_t st )
{
	void *ps[] = { wb.ray_o, wb.ray_d, wb.hit, wb.beta, wb.L, wb.queue[ 0 ], wb.queue[ 1 ], wb.shadow_queue,
				   wb.sh_o, wb.sh_d, wb.sh_c, wb.counters, wb.err, wb.work, wb.lobes, wb.path_job, wb.tally,
				   wb.binned, wb.bins, wb.bwave };
	for ( void *p : ps )
		if ( p ) cudaFreeAsync( p, st );
	wb = WaveBuffers();
}

// Sort queue[0 .. *n) into wb.binned (the launches of one traversal stage).
void bin_queue( const DevScene &sc, const WaveBuffers &wb, const uint32_t *queue, const uint32_t *n,
				const float4 *ray_o, const float4 *ray_d, int grid, cudaStream_t st )
{
	check( cudaMemsetAsync( wb.bins, 0, sizeof( uint32_t ) * N_BINS, st ), "memset" );
	k_bin_count<<<grid, BIN_THREADS, 0, st>>>( queue, n, ray_o, ray_d, sc.nodes, wb.bins );
	k_bin_scan<<<1, 1024, 0, st>>>( wb.bins );
	k_bin_scatter<<<grid, BIN_THREADS, 0, st>>>( queue, n, ray_o, ray_d, sc.nodes, wb.bins, wb.binned, wb.err );
}

void alloc_bins( WaveBuffers &wb, cudaStream_t st )
{
	if ( !wb.binned ) alloc( wb.binned, wb.capacity, st );
	if ( !wb.bins ) alloc( wb.bins, N_BINS, st );
}

void alloc_lobes( WaveBuffers &wb, cudaStream_t st )
{
	if ( wb.lobes ) return;
	alloc( wb.lobes, size_t( wb.capacity ) * LOBE_SLOTS, st );
}

void alloc_batch_state( WaveBuffers &wb, cudaStream_t st )
{
	if ( !wb.path_job ) alloc( wb.path_job, wb.capacity, st );
	if ( !wb.tally ) alloc( wb.tally, 2, st );
	if ( !wb.bwave ) alloc( wb.bwave, 1, st );
}

namespace
{
// Samples of a batch: the last job's end.
uint64_t batch_total( const BatchJobDev *jobs, uint32_t n_jobs )
{
	const BatchJobDev &last = jobs[ n_jobs - 1 ];
	return last.first_sample + uint64_t( last.width ) * last.height * last.spp;
}

void check_batch_state( uint32_t n_jobs, const RenderConfig &cfg, const WaveBuffers &wb )
{
	if ( n_jobs == 0 ) throw std::runtime_error( "batched render without jobs" );
	if ( !wb.path_job || !wb.tally || !wb.bwave ) throw std::runtime_error( "batched render without its wave state" );
	if ( cfg.wave_paths == 0 || cfg.wave_paths > wb.capacity )
		throw std::runtime_error( "wave size exceeds the allocated wave buffers" );
}

// One wave of a batched render, every kernel reading the wave from
// wb.bwave: begin (wave bounds, counters), generation, max_bounce + 1 x
// (closest hit, shading, shadow rays), accumulation, end (tally, next wave
// and, when `looped`, the graph loop's condition).  timed(kind, launch) wraps
// each stage.
template <class Timed>
void batch_wave_kernels( const BatchDev &bd, const RenderConfig &cfg, WaveBuffers &wb, uint64_t total, cudaStream_t st,
						 Timed &&timed, cudaGraphConditionalHandle loop, bool looped )
{
	const int sms = sm_count();
	const int g_ext = sms * std::max( 1, std::min( 8, cfg.traverse_blocks_per_sm ) );
	const uint32_t shade_t = cfg.shade_threads == 64 || cfg.shade_threads == 256 ? cfg.shade_threads : 128u;
	const int g_shade_k = int( uint32_t( sms ) * 1024u / shade_t );  // k_shade: SMs x 1024 threads
	const int g_wide = sms * 16;                                      // generation and accumulation
	const uint32_t P = cfg.wave_paths;
	timed( 3, [&] {
		k_batch_wave_begin<<<1, 256, 0, st>>>( bd, wb, total, P );
		k_generate_batch<<<g_wide, 256, 0, st>>>( bd, wb );
	} );
	for ( uint32_t b = 0; b <= cfg.max_bounce; ++b )
	{
		timed( 0, [&] {
			BatchExtendIO io;
			io.queue = wb.queue[ b & 1 ], io.ray_o = wb.ray_o, io.ray_d = wb.ray_d, io.hit = wb.hit;
			io.scenes = bd.scenes, io.path_job = wb.path_job;
			const uint32_t *n = wb.counters + CPB * b + CNT_EXT;
			uint32_t *cur = wb.counters + CPB * b + CNT_EXT_CURSOR;
			k_traverse<BatchExtendIO, false, false><<<g_ext, TRAVERSE_THREADS, 0, st>>>( DevScene{}, io, n, 0, cur, wb.err,
																						  wb.work, cfg.refill_min, EXT_TRI_VOTE );
		} );
		timed( 2, [&] {
			if ( cfg.estimator == EST_MIS )
				k_shade<true, EST_MIS><<<g_shade_k, shade_t, 0, st>>>( DevScene{}, cfg, wb, WaveArgs{}, b, uint2{}, bd );
			else
				k_shade<true, EST_KOISHI><<<g_shade_k, shade_t, 0, st>>>( DevScene{}, cfg, wb, WaveArgs{}, b, uint2{}, bd );
		} );
		timed( 1, [&] {
			BatchShadowIO io;
			io.queue = wb.shadow_queue, io.ray_o = wb.sh_o, io.ray_d = wb.sh_d, io.contrib = wb.sh_c, io.L = wb.L;
			io.scenes = bd.scenes, io.path_job = wb.path_job;
			const uint32_t *n = wb.counters + CPB * b + CNT_SHADOW;
			uint32_t *cur = wb.counters + CPB * b + CNT_SHADOW_CURSOR;
			k_traverse<BatchShadowIO, true, false><<<g_ext, TRAVERSE_THREADS, 0, st>>>( DevScene{}, io, n, 0, cur, wb.err,
																						 wb.work + 2, shadow_refill( cfg ), cfg.shadow_vote );
		} );
	}
	timed( 3, [&] {
		k_accumulate_batch<<<g_wide, 256, 0, st>>>( bd, wb );
		k_batch_wave_end<<<1, 32, 0, st>>>( wb, cfg.max_bounce, total, P, loop, looped ? 1 : 0 );
	} );
	check( cudaGetLastError(), "batched render launch" );
}
}  // namespace

void render_batch_waves( const BatchDev &bd, const BatchJobDev *jobs, uint32_t n_jobs, const RenderConfig &cfg,
						 WaveBuffers &wb, cudaStream_t st, StageTimes *times )
{
	check_batch_state( n_jobs, cfg, wb );
	const uint64_t total = batch_total( jobs, n_jobs );
	EventPool pool;
	struct Mark
	{
		cudaEvent_t a, b;
		int kind;
	};
	std::vector<Mark> marks;
	cudaEvent_t t0 = nullptr, t1 = nullptr;
	if ( times )
	{
		t0 = pool.get(), t1 = pool.get();
		check( cudaEventRecord( t0, st ), "event" );
	}
	auto timed = [&]( int kind, auto &&launch ) {
		if ( !times )
		{
			launch();
			return;
		}
		Mark m{ pool.get(), pool.get(), kind };
		check( cudaEventRecord( m.a, st ), "event" );
		launch();
		check( cudaEventRecord( m.b, st ), "event" );
		marks.push_back( m );
		times->launches++;
		if ( kind == 0 ) times->extend_launches++;
		if ( kind == 1 ) times->shadow_launches++;
	};
	k_batch_init<<<1, 32, 0, st>>>( wb );
	for ( uint64_t first = 0; first < total; first += cfg.wave_paths )
	{
		batch_wave_kernels( bd, cfg, wb, total, st, timed, cudaGraphConditionalHandle{}, false );
		if ( times ) times->waves++;
	}
	if ( times )
	{
		check( cudaEventRecord( t1, st ), "event" );
		check( cudaEventSynchronize( t1 ), "event" );
		float ms;
		check( cudaEventElapsedTime( &ms, t0, t1 ), "event" );
		times->total += ms;
		for ( auto &m : marks )
		{
			check( cudaEventElapsedTime( &ms, m.a, m.b ), "event" );
			( m.kind == 0 ? times->extend : m.kind == 1 ? times->shadow : m.kind == 2 ? times->shade : times->other ) += ms;
		}
		unsigned long long t[ 2 ];
		check( cudaMemcpy( t, wb.tally, sizeof t, cudaMemcpyDeviceToHost ), "tally" );
		times->rays_extend += t[ 0 ], times->rays_shadow += t[ 1 ];
	}
}


uint32_t build_batch_graph( const BatchDev &bd, const BatchJobDev *jobs, uint32_t n_jobs, const RenderConfig &cfg,
							WaveBuffers &wb, cudaStream_t st, cudaGraph_t *out )
{
	check_batch_state( n_jobs, cfg, wb );
	const uint64_t total = batch_total( jobs, n_jobs );
	cudaGraph_t g = nullptr;
	check( cudaGraphCreate( &g, 0 ), "graph" );
	// a capture that fails part-way is ended before the error propagates
	auto captured = [&]( cudaGraph_t into, auto &&launch ) {
		check( cudaStreamBeginCaptureToGraph( st, into, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal ),
			   "graph capture" );
		try
		{
			launch();
		}
		catch ( ... )
		{
			cudaStreamEndCapture( st, &into );
			throw;
		}
		check( cudaStreamEndCapture( st, &into ), "graph capture" );
	};
	try
	{
		captured( g, [&] {
			k_batch_init<<<1, 32, 0, st>>>( wb );
			check( cudaGetLastError(), "batched render launch" );
		} );
		cudaGraphNode_t init = nullptr;
		size_t n_init = 1;
		check( cudaGraphGetNodes( g, &init, &n_init ), "graph" );
		if ( n_init != 1 ) throw std::runtime_error( "batch graph: unexpected initial nodes" );
		// the loop runs at least once (a batch has samples); its body decides whether to go on
		cudaGraphConditionalHandle loop{};
		check( cudaGraphConditionalHandleCreate( &loop, g, 1u, cudaGraphCondAssignDefault ), "graph conditional" );
		cudaGraphNodeParams cp{};
		cp.type = cudaGraphNodeTypeConditional;
		cp.conditional.handle = loop;
		cp.conditional.type = cudaGraphCondTypeWhile;
		cp.conditional.size = 1;
		cudaGraphNode_t cond = nullptr;
		check( cudaGraphAddNode( &cond, g, &init, 1, &cp ), "graph conditional" );
		cudaGraph_t body = cp.conditional.phGraph_out[ 0 ];
		auto direct = []( int, auto &&launch ) { launch(); };
		captured( body, [&] { batch_wave_kernels( bd, cfg, wb, total, st, direct, loop, true ); } );
		size_t n_body = 0;
		check( cudaGraphGetNodes( body, nullptr, &n_body ), "graph" );
		*out = g;
		return uint32_t( 1 + n_body );
	}
	catch ( ... )
	{
		cudaGraphDestroy( g );
		throw;
	}
}

void render_waves( const DevScene &sc, const RenderConfig &cfg, WaveBuffers &wb, double *film_sum, double *film_sumsq,
				   uint32_t *film_count, cudaStream_t st, StageTimes *times, GuideState *guide )
{
	if ( cfg.guiding && ( !guide || !wb.lobes || cfg.estimator != EST_MIS ) )
		throw std::runtime_error( "guided render without a guide, lobe buffer or MIS estimator" );
	const bool profiled = cfg.prof.slices != nullptr;
	if ( profiled && ( cfg.estimator != EST_KOISHI || cfg.kernel != KERNEL_RADIANCE || cfg.guiding || !cfg.prof.bounces ) )
		throw std::runtime_error( "a profiled render takes the Radiance kernel with the reference estimator" );
	const uint64_t total = uint64_t( cfg.ww ) * cfg.wh * cfg.spp;
	if ( cfg.wave_paths == 0 || cfg.wave_paths > wb.capacity )
		throw std::runtime_error( "wave size exceeds the allocated wave buffers" );
	const uint32_t P = cfg.wave_paths;
	const int sms = sm_count();
	const int g_ext = sms * std::max( 1, std::min( 8, cfg.traverse_blocks_per_sm ) );
	const int g_shade = sms * 8;
	const uint32_t shade_t = cfg.shade_threads == 64 || cfg.shade_threads == 256 ? cfg.shade_threads : 128u;
	const int g_shade_k = int( uint32_t( sms ) * 1024u / shade_t );  // k_shade: SMs x 1024 threads
	const uint2 key = make_uint2( uint32_t( cfg.seed ), uint32_t( cfg.seed >> 32 ) ^ 0x5EED5EEDu );
	const bool binning = cfg.bin_rays && wb.binned && wb.bins && sc.n_nodes > 0;
	EventPool pool;
	struct Mark
	{
		cudaEvent_t a, b;
		int kind;  // 0 extend 1 shadow 2 shade 3 other 4 guide inference 5 guide training
	};
	std::vector<Mark> marks;
	cudaEvent_t t0 = nullptr, t1 = nullptr;
	if ( times )
	{
		t0 = pool.get();
		t1 = pool.get();
		check( cudaEventRecord( t0, st ), "event" );
		if ( cfg.count_work ) check( cudaMemsetAsync( wb.work, 0, 4 * sizeof( unsigned long long ), st ), "memset" );
	}
	auto timed = [&]( int kind, auto &&launch ) {
		if ( !times )
		{
			launch();
			return;
		}
		Mark m{ pool.get(), pool.get(), kind };
		check( cudaEventRecord( m.a, st ), "event" );
		launch();
		check( cudaEventRecord( m.b, st ), "event" );
		marks.push_back( m );
		times->launches++;
		if ( kind == 0 ) times->extend_launches++;
		if ( kind == 1 ) times->shadow_launches++;
		if ( kind == 4 ) times->guide_launches++;
	};
	std::vector<uint32_t> host_counts;
	for ( uint64_t first = 0; first < total; first += P )
	{
		WaveArgs wa{ first, uint32_t( std::min<uint64_t>( P, total - first ) ) };
		check( cudaMemsetAsync( wb.counters, 0, sizeof( uint32_t ) * wb.n_counters, st ), "memset" );
		// per-wave copy: which paths are recorded, and whether the guide is sampled
		RenderConfig wc = cfg;
		uint32_t steps = 0, batch = 0;
		// record and train only while the training budget lasts; sample the guide after warm-up
		const bool training = cfg.guiding && ( guide->max_steps == 0 || guide->step < guide->max_steps );
		if ( cfg.guiding && !training ) wc.guiding = false;
		if ( cfg.guiding && guide->step >= guide->warmup_steps )
		{
			wc.guide_sample = true;
			ensure_smem_limit( reinterpret_cast<const void *>( k_guide_infer ), int( tc::SMEM_BYTES ), "guide inference smem" );
			if ( guide->packed_step != guide->step )  // BF16 copy of the weights this wave samples with
			{
				guide->pack_weights( st );
				guide->packed_step = guide->step;
			}
		}
		if ( training )
		{
			batch = std::min( guide->train_paths, wa.n );
			// steps this wave: steps_per_wave, or what is left of the budget
			uint32_t take = guide->steps_per_wave;
			if ( guide->max_steps ) take = std::min( take, guide->max_steps - guide->step );
			wc.rec_paths = uint32_t( std::min<uint64_t>( uint64_t( batch ) * take, wa.n ) );
			steps = ( wc.rec_paths + batch - 1 ) / batch;
			wc.rec_stride = wa.n / wc.rec_paths;
			wc.rec_offset = uint32_t( ( guide->waves++ * 2654435761ull ) % wc.rec_stride );
			check( cudaMemsetAsync( cfg.rec.x, 0, sizeof( float4 ) * size_t( wc.rec_paths ) * ( cfg.max_bounce + 1 ), st ),
				   "memset" );
		}
		timed( 3, [&] {
			int gg = int( std::min<uint64_t>( ( wa.n + 255 ) / 256, uint64_t( sms ) * 16 ) );
			k_generate<<<gg, 256, 0, st>>>( sc, wc, wb, wa );
		} );
		for ( uint32_t b = 0; b <= ( cfg.kernel == KERNEL_RADIANCE ? cfg.max_bounce : 0u ); ++b )
		{
			timed( 0, [&] {
				ExtendIO io{ wb.queue[ b & 1 ], wb.ray_o, wb.ray_d, wb.hit };
				const uint32_t *n = wb.counters + CPB * b + CNT_EXT;
				uint32_t *cur = wb.counters + CPB * b + CNT_EXT_CURSOR;
				// camera rays are coherent in pixel order already
				if ( binning && b > 0 )
				{
					bin_queue( sc, wb, io.queue, n, wb.ray_o, wb.ray_d, sms * 4, st );
					io.queue = wb.binned;
				}
				if ( cfg.count_work )
					k_traverse<ExtendIO, false, true><<<g_ext, TRAVERSE_THREADS, 0, st>>>( sc, io, n, 0, cur, wb.err, wb.work, cfg.refill_min,
																						  EXT_TRI_VOTE );
				else
					k_traverse<ExtendIO, false, false><<<g_ext, TRAVERSE_THREADS, 0, st>>>( sc, io, n, 0, cur, wb.err, wb.work, cfg.refill_min,
																						   EXT_TRI_VOTE );
			} );
			if ( wc.guide_sample && guided_vertex( wc.guide, b, cfg.max_bounce ) )
				timed( 4, [&] {
					k_guide_infer<<<sms * 2, tc::THREADS, tc::SMEM_BYTES, st>>>( sc, wc, wb, b, guide->Wp );
				} );
			if ( cfg.kernel != KERNEL_RADIANCE )
				timed( 2, [&] { k_aov<<<g_shade, 128, 0, st>>>( sc, wc, wb, wa, key ); } );
			else
				timed( 2, [&] {
					if ( cfg.estimator == EST_MIS && ( wc.guiding || wc.guide_sample ) )
						k_shade<false, EST_MIS, false, true><<<g_shade_k, shade_t, 0, st>>>( sc, wc, wb, wa, b, key, BatchDev{} );
					else if ( cfg.estimator == EST_MIS )
						k_shade<false, EST_MIS><<<g_shade_k, shade_t, 0, st>>>( sc, wc, wb, wa, b, key, BatchDev{} );
					else if ( profiled )
						k_shade<false, EST_KOISHI, true><<<g_shade_k, shade_t, 0, st>>>( sc, wc, wb, wa, b, key, BatchDev{} );
					else
						k_shade<false, EST_KOISHI><<<g_shade_k, shade_t, 0, st>>>( sc, wc, wb, wa, b, key, BatchDev{} );
				} );
			if ( sc.n_lights && cfg.kernel != KERNEL_NORMAL && cfg.kernel != KERNEL_HALFVECTOR )
				timed( 1, [&] {
					ShadowIO io{ wb.shadow_queue, wb.sh_o, wb.sh_d, wb.sh_c, wb.L };
					const uint32_t *n = wb.counters + CPB * b + CNT_SHADOW;
					uint32_t *cur = wb.counters + CPB * b + CNT_SHADOW_CURSOR;
					if ( binning )
					{
						bin_queue( sc, wb, io.queue, n, wb.sh_o, wb.sh_d, sms * 4, st );
						io.queue = wb.binned;
					}
					if ( cfg.count_work )
						k_traverse<ShadowIO, true, true><<<g_ext, TRAVERSE_THREADS, 0, st>>>( sc, io, n, 0, cur, wb.err, wb.work + 2,
																							 shadow_refill( cfg ), cfg.shadow_vote );
					else
						k_traverse<ShadowIO, true, false><<<g_ext, TRAVERSE_THREADS, 0, st>>>( sc, io, n, 0, cur, wb.err, wb.work + 2,
																							  shadow_refill( cfg ), cfg.shadow_vote );
				} );
			if ( profiled ) timed( 3, [&] { k_profile_fix<<<g_shade, 128, 0, st>>>( wc, wb, wa, b ); } );
		}
		if ( profiled ) timed( 3, [&] { k_profile_final<<<g_shade, 128, 0, st>>>( wc, wb, wa ); } );
		if ( steps )
			timed( 5, [&] {
				// online training on this wave's recorded vertices, one Adam step per batch
				for ( uint32_t k = 0; k < steps; ++k )
				{
					uint32_t j0 = k * batch;
					guide->train_step( wb.L, j0, std::min( batch, wc.rec_paths - j0 ), cfg.max_bounce + 1, wc.rec_offset,
									   wc.rec_stride, st );
				}
			} );
		timed( 3, [&] {
			uint64_t npx = ( first + wa.n - 1 ) / cfg.spp - first / cfg.spp + 1;
			int gg = int( std::min<uint64_t>( ( npx + 255 ) / 256, uint64_t( sms ) * 16 ) );
			k_accumulate<<<gg, 256, 0, st>>>( wc, wb, wa, film_sum, film_sumsq, film_count );
		} );
		check( cudaGetLastError(), "render launch" );
		if ( times )
		{
			times->waves++;
			host_counts.resize( wb.n_counters );
			check( cudaMemcpyAsync( host_counts.data(), wb.counters, sizeof( uint32_t ) * wb.n_counters,
									cudaMemcpyDeviceToHost, st ),
				   "counts" );
			check( cudaStreamSynchronize( st ), "counts" );
			for ( uint32_t b = 0; b <= cfg.max_bounce; ++b )
			{
				times->rays_extend += host_counts[ CPB * b + CNT_EXT ];
				times->rays_shadow += host_counts[ CPB * b + CNT_SHADOW ];
				// the guide's inference runs on the bounce's whole extension queue
				if ( wc.guide_sample && guided_vertex( wc.guide, b, cfg.max_bounce ) )
					times->guide_rows += host_counts[ CPB * b + CNT_EXT ];
			}
		}
	}
	if ( times )
	{
		check( cudaEventRecord( t1, st ), "event" );
		check( cudaEventSynchronize( t1 ), "event" );
		float ms;
		check( cudaEventElapsedTime( &ms, t0, t1 ), "event" );
		times->total += ms;
		for ( auto &m : marks )
		{
			check( cudaEventElapsedTime( &ms, m.a, m.b ), "event" );
			( m.kind == 0 ? times->extend : m.kind == 1 ? times->shadow : m.kind == 2 ? times->shade
																  : m.kind >= 4 ? times->guide : times->other ) += ms;
			if ( m.kind == 5 ) times->guide_train += ms;
		}
		if ( cfg.count_work )
		{
			unsigned long long w[ 4 ];
			check( cudaMemcpy( w, wb.work, sizeof w, cudaMemcpyDeviceToHost ), "work" );
			times->nodes += w[ 0 ];
			times->tris += w[ 1 ];
			times->shadow_nodes += w[ 2 ];
			times->shadow_tris += w[ 3 ];
		}
	}
}

void launch_trace( const DevScene &sc, const float *rays, uint64_t n, int any_hit, cr_hit *out, uint32_t *err,
				   cudaStream_t st, unsigned long long *work )
{
	if ( !n ) return;
	if ( n >= ( 1ull << 32 ) - 64 ) throw std::runtime_error( "too many rays in one query" );
	// err[0] is the error word, err[1] the work cursor of this query.
	check( cudaMemsetAsync( err + 1, 0, sizeof( uint32_t ), st ), "trace cursor" );
	int g = int( std::min<uint64_t>( ( n + 127 ) / 128, uint64_t( sm_count() ) * 8 ) );
	QueryIO io{ rays, out, sc.tris, sc.attrs, sc.spheres, sc.prim_first };
	// with `work` (2 counters, added to): the counting build, nodes and primitives tested
	if ( any_hit && work )
		k_traverse<QueryIO, true, true><<<g, TRAVERSE_THREADS, 0, st>>>( sc, io, nullptr, uint32_t( n ), err + 1, err, work,
																QUERY_REFILL_MIN, EXT_TRI_VOTE );
	else if ( any_hit )
		k_traverse<QueryIO, true, false><<<g, TRAVERSE_THREADS, 0, st>>>( sc, io, nullptr, uint32_t( n ), err + 1, err, nullptr,
																 QUERY_REFILL_MIN, EXT_TRI_VOTE );
	else if ( work )
		k_traverse<QueryIO, false, true><<<g, TRAVERSE_THREADS, 0, st>>>( sc, io, nullptr, uint32_t( n ), err + 1, err, work,
																 QUERY_REFILL_MIN, EXT_TRI_VOTE );
	else
		k_traverse<QueryIO, false, false><<<g, TRAVERSE_THREADS, 0, st>>>( sc, io, nullptr, uint32_t( n ), err + 1, err, nullptr,
																  QUERY_REFILL_MIN, EXT_TRI_VOTE );
	check( cudaGetLastError(), "trace launch" );
}

void launch_philox( const uint32_t *ctr_key, uint64_t n, uint32_t *out, cudaStream_t st )
{
	if ( !n ) return;
	int g = int( std::min<uint64_t>( ( n + 255 ) / 256, 4096 ) );
	k_philox<<<g, 256, 0, st>>>( ctr_key, n, out );
	check( cudaGetLastError(), "philox launch" );
}

void launch_bsdf_eval( int est, const DevShader &sh, const float *wo, const float *wi, uint64_t n, float *f, float *pdf,
					   cudaStream_t st )
{
	if ( !n ) return;
	int g = int( std::min<uint64_t>( ( n + 255 ) / 256, 4096 ) );
	k_bsdf_eval<<<g, 256, 0, st>>>( est, sh, wo, wi, n, f, pdf );
	check( cudaGetLastError(), "bsdf launch" );
}

void launch_bsdf_sample( int est, const DevShader &sh, const float *wo, const float *u, uint64_t n, float *wi,
						 float *wt, float *pdf, cudaStream_t st )
{
	if ( !n ) return;
	int g = int( std::min<uint64_t>( ( n + 255 ) / 256, 4096 ) );
	k_bsdf_sample<<<g, 256, 0, st>>>( est, sh, wo, u, n, wi, wt, pdf );
	check( cudaGetLastError(), "bsdf launch" );
}

void launch_shader_execute( const DevShader *tab, int target, const float *wo, float *wi, const float *u, uint32_t k,
							uint64_t n, float *f, float *emission, uint32_t *used, cudaStream_t st )
{
	if ( !n ) return;
	int g = int( std::min<uint64_t>( ( n + 255 ) / 256, 4096 ) );
	k_shader_execute<<<g, 256, 0, st>>>( tab, target, wo, wi, u, k, n, f, emission, used );
	check( cudaGetLastError(), "shader launch" );
}

}  // namespace cr
