// Persistent wide-BVH traversal kernel shared by the closest-hit queue
// (k_extend), the shadow queue (k_shadow) and the batched ray queries of the
// C ABI.
//
// Each warp owns 32 traversal states.  A lane that finishes its ray is refilled
// from the queue (one atomic per warp) once enough lanes are idle, so a warp no
// longer waits for its slowest ray.  Every iteration the warp votes between a
// node step (each lane with no pending triangles visits one wide node, popping
// the stack first when its current group is exhausted, or finishes) and a
// triangle step (each lane with pending triangles tests one), taking the
// triangle step once a quarter of the active lanes want it; the other lanes
// wait, so lanes in one iteration run the same code.
#pragma once
#include "cr_device.cuh"

namespace cr
{
constexpr uint32_t FULL_MASK = 0xFFFFFFFFu;

// A quantised plane byte q as the float 32768 + q, exactly: the byte goes to
// bits 8..15 of a float whose exponent makes bit 8 worth 1 (0x47000000 is
// 2^15).  One byte permute, no integer-to-float conversion.
__device__ __forceinline__ float q8_biased( uint32_t w, uint32_t i )
{
	return __uint_as_float( __byte_perm( w, 0x47000000u, 0x7404u | ( i << 4 ) ) );
}
constexpr float Q8_BIAS = 32768.f;

// Three-operand max / min (PTX max.f32 / min.f32 with three sources, sm_100).
__device__ __forceinline__ float fmax3( float a, float b, float c )
{
	float d;
	asm( "max.f32 %0, %1, %2, %3;" : "=f"( d ) : "f"( a ), "f"( b ), "f"( c ) );
	return d;
}
__device__ __forceinline__ float fmin3( float a, float b, float c )
{
	float d;
	asm( "min.f32 %0, %1, %2, %3;" : "=f"( d ) : "f"( a ), "f"( b ), "f"( c ) );
	return d;
}

// Intersects the ray with the 8 children of `node`; returns the node-group
// hits (bits at slot ^ octant) and the triangle-group hits (24-bit mask).
//
// Child plane k of an axis lies at p + 2^e q_k, so its ray distance is
// (p - o) / d + q_k 2^e / d = fma(32768 + q_k, S, B) with S = 2^e / d (exact:
// a power of two times 1/d) and B = (p - o) / d - 32768 S (one rounding).
// The extra rounding of B is 2^-9 of one quantisation step S, below the
// rounding of (p - o) / d for any node further away than a few node widths.
__device__ __forceinline__ void visit_node( const WNode *nodes, const RayPre &r, uint32_t node, float tmin,
											float tlim, uint2 &ng, uint2 &tg )
{
	const uint4 *np = reinterpret_cast<const uint4 *>( nodes ) + 5 * size_t( node );
	uint4 n0 = __ldg( np ), n1 = __ldg( np + 1 ), n2 = __ldg( np + 2 ), n3 = __ldg( np + 3 ), n4 = __ldg( np + 4 );
	float3 p = f3( __uint_as_float( n0.x ), __uint_as_float( n0.y ), __uint_as_float( n0.z ) );
	uint32_t ex = n0.w & 0xFFu, ey = ( n0.w >> 8 ) & 0xFFu, ez = ( n0.w >> 16 ) & 0xFFu, imask = n0.w >> 24;
	float3 adj_s = f3( __uint_as_float( ex << 23 ) * r.invd.x, __uint_as_float( ey << 23 ) * r.invd.y,
					   __uint_as_float( ez << 23 ) * r.invd.z );
	float3 adj_o = ( p - r.o ) * r.invd;
	adj_o = f3( fmaf( -Q8_BIAS, adj_s.x, adj_o.x ), fmaf( -Q8_BIAS, adj_s.y, adj_o.y ), fmaf( -Q8_BIAS, adj_s.z, adj_o.z ) );
	uint32_t nx0 = n2.x, nx1 = n2.y, fx0 = n3.z, fx1 = n3.w;
	uint32_t ny0 = n2.z, ny1 = n2.w, fy0 = n4.x, fy1 = n4.y;
	uint32_t nz0 = n3.x, nz1 = n3.y, fz0 = n4.z, fz1 = n4.w;
	if ( r.oct & 1u ) { uint32_t t0 = nx0, t1 = nx1; nx0 = fx0, nx1 = fx1, fx0 = t0, fx1 = t1; }
	if ( r.oct & 2u ) { uint32_t t0 = ny0, t1 = ny1; ny0 = fy0, ny1 = fy1, fy0 = t0, fy1 = t1; }
	if ( r.oct & 4u ) { uint32_t t0 = nz0, t1 = nz1; nz0 = fz0, nz1 = fz1, fz0 = t0, fz1 = t1; }
	uint32_t node_hits = 0, tri_hits = 0;
#pragma unroll
	for ( int i = 0; i < 8; ++i )
	{
		const int sh = 8 * ( i & 3 );
		const uint32_t bi = uint32_t( i & 3 );
		uint32_t wnx = i < 4 ? nx0 : nx1, wny = i < 4 ? ny0 : ny1, wnz = i < 4 ? nz0 : nz1;
		uint32_t wfx = i < 4 ? fx0 : fx1, wfy = i < 4 ? fy0 : fy1, wfz = i < 4 ? fz0 : fz1;
		float tnx = fmaf( q8_biased( wnx, bi ), adj_s.x, adj_o.x ), tfx = fmaf( q8_biased( wfx, bi ), adj_s.x, adj_o.x );
		float tny = fmaf( q8_biased( wny, bi ), adj_s.y, adj_o.y ), tfy = fmaf( q8_biased( wfy, bi ), adj_s.y, adj_o.y );
		float tnz = fmaf( q8_biased( wnz, bi ), adj_s.z, adj_o.z ), tfz = fmaf( q8_biased( wfz, bi ), adj_s.z, adj_o.z );
		const float tn = fmax3( tnx, tny, fmaxf( tnz, tmin ) );
		const float tf = fmin3( tfx, tfy, fminf( tfz, tlim ) );
		// meta: the leaf's unary triangle count in bits 5..7 above its offset
		// (0 for internal and empty slots), so its triangles' bits are the
		// count bits shifted by the offset
		const uint32_t meta = ( ( i < 4 ? n1.z : n1.w ) >> sh ) & 0xFFu;
		const bool internal = ( imask >> i ) & 1u;
		if ( tn <= tf )
		{
			if ( internal )
				node_hits |= 1u << ( i ^ r.oct );
			else
				tri_hits |= __funnelshift_l( 0u, meta >> 5, meta );
		}
	}
	ng = node_hits ? make_uint2( n1.x, ( node_hits << 24 ) | imask ) : make_uint2( 0u, 0u );
	tg = make_uint2( n1.y, tri_hits );
}

// Ray source and result sink of the persistent kernel.  refill_min: idle lanes
// (1..32) that trigger a refill from the queue.  tri_vote: the warp takes a
// triangle step once tri_vote x (lanes with triangles pending) >= active lanes
// (4: a quarter; 32: any lane).
//   load(i, item, o, d, tmin, tmax): the i-th queued ray
//   finish(item, hit, found): store the result
//   MULTI: the queue mixes the rays of several scenes (a batched render);
//          scene(item) is the ray's scene, otherwise every ray uses `sc`
constexpr int TRAVERSE_THREADS = 128;  // threads per block of k_traverse (every launch uses this)
constexpr int SHARED_STACK = 8;        // stack entries per thread kept in shared memory

template <class IO, bool ANY, bool COUNT>
__global__ void __launch_bounds__( TRAVERSE_THREADS, 8 ) k_traverse( DevScene sc, IO io, const uint32_t *n_ptr, uint32_t n_host,
														uint32_t *cursor, uint32_t *err, unsigned long long *work,
														uint32_t refill_min, uint32_t tri_vote )
{
	const uint32_t n = n_ptr ? *n_ptr : n_host;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t lt_mask = ( 1u << lane ) - 1u;
	const float grow = 1.0f + 4.0f * 5.96e-8f;
	uint32_t wnodes = 0, wtris = 0;
	bool active = false, exhausted = false;
	uint32_t item = 0, budget = 0;
	RayPre r;
	float tmin = 0.f;
	HitRec hit;
	bool found = false;
	uint2 ng = make_uint2( 0u, 0u ), tg = make_uint2( 0u, 0u );
	// Traversal stack of (node base, hit mask) groups: the first SHARED_STACK
	// entries in shared memory (entry k of thread t at [k][t]: a warp's 32
	// entries are 256 contiguous bytes, no bank conflicts), deeper ones in
	// local memory, which shallow 8-wide trees rarely reach.
	__shared__ uint2 sstack[ SHARED_STACK ][ TRAVERSE_THREADS ];
	uint2 *const my_stack = &sstack[ 0 ][ threadIdx.x ];
	int sp = 0;
	uint2 stack[ TRAVERSAL_STACK - SHARED_STACK ];
	// this lane's geometry: the kernel's scene, or the current ray's in a batch
	const WNode *nodes = sc.nodes;
	const float4 *tris = sc.tris;
	uint32_t n_nodes = sc.n_nodes, n_tris = sc.n_tris, sph_base = sc.sph_base;
	for ( ;; )
	{
		if ( !exhausted )
		{
			uint32_t idle = __ballot_sync( FULL_MASK, !active );
			if ( uint32_t( __popc( idle ) ) >= refill_min )
			{
				uint32_t leader = __ffs( idle ) - 1, base = 0;
				if ( lane == leader ) base = atomicAdd( cursor, uint32_t( __popc( idle ) ) );
				base = __shfl_sync( FULL_MASK, base, leader );
				if ( base + __popc( idle ) >= n ) exhausted = true;
				if ( !active )
				{
					uint32_t i = base + __popc( idle & lt_mask );
					if ( i < n )
					{
						float3 o, d;
						float tmax;
						io.load( i, item, o, d, tmin, tmax );
						if constexpr ( IO::MULTI )
						{
							const DevScene *ps = io.scene( item );
							nodes = ps->nodes, tris = ps->tris;
							n_nodes = ps->n_nodes, n_tris = ps->n_tris, sph_base = ps->sph_base;
						}
						hit.t = tmax;
						hit.id = HIT_MISS;
						hit.u = hit.v = 0.f;
						found = false;
						// A NaN ray would pass every slab test; it hits nothing.
						if ( n_nodes == 0 || !finite3( o ) || !finite3( d ) )
							io.finish( item, hit, found );
						else
						{
							r = make_ray( o, d );
							ng = make_uint2( 0u, ( 1u << ( 24 + r.oct ) ) | 1u );
							tg = make_uint2( 0u, 0u );
							sp = 0;
							budget = n_nodes;
							active = true;
						}
					}
				}
			}
		}
		const uint32_t act = __ballot_sync( FULL_MASK, active );
		if ( !act )
		{
			if ( exhausted ) break;
			continue;
		}
		const uint32_t want_tri = __ballot_sync( FULL_MASK, active && tg.y != 0u );
		// triangle step once tri_vote x the lanes with triangles pending cover
		// the active lanes (closest hit: a quarter; a sweep of 1/32 .. 24/32 on
		// the 1.31M-triangle workload peaked at 8/32)
		const bool tri_step = tri_vote * __popc( want_tri ) >= __popc( act );
		if ( !active ) continue;
		bool done = false;
		if ( tri_step )
		{
			if ( tg.y )
			{
				uint32_t k = __ffs( tg.y ) - 1;
				tg.y &= tg.y - 1u;
				uint32_t ti = tg.x + k;
				if ( ti >= n_tris )
				{
					atomicOr( err, 4u );
					tg.y = 0u;
				}
				else
				{
					const float4 *tp = tris + 3 * size_t( ti );
					float4 a = __ldg( tp ), b = __ldg( tp + 1 ), c = __ldg( tp + 2 );
					if ( COUNT ) ++wtris;
					float t, u = 0.f, v = 0.f;
					const uint32_t gid = __float_as_uint( a.w );
					// a sphere record: (box lo, id), (box hi, -), (centre, r^2)
					const bool sphere = gid >= sph_base;
					if ( sphere ? sphere_test( f3( c ), c.w, r.o, r.d, tmin, hit.t, t )
								: tri_test( r, f3( a ), f3( b ), f3( c ), tmin, hit.t, t, u, v ) )
					{
						hit.t = t, hit.id = sphere ? ( HIT_SPHERE | ( gid - sph_base ) ) : ti, hit.u = u, hit.v = v;
						found = true;
						if ( ANY ) done = true;
					}
				}
			}
		}
		else if ( !tg.y )
		{
			// an exhausted group: pop the next one and visit its next child in
			// this same step (a pushed group always has a child left)
			if ( ng.y <= 0x00FFFFFFu && sp > 0 )
			{
				--sp;
				ng = sp < SHARED_STACK ? my_stack[ TRAVERSE_THREADS * sp ] : stack[ sp - SHARED_STACK ];
			}
			if ( ng.y > 0x00FFFFFFu )
			{
				uint32_t b = __ffs( ng.y >> 24 ) - 1;
				ng.y &= ~( 1u << ( 24 + b ) );
				uint32_t slot = b ^ r.oct;
				uint32_t node = ng.x + __popc( ng.y & 0xFFu & ( ( 1u << slot ) - 1u ) );
				if ( node >= n_nodes || budget-- == 0 )
				{
					atomicOr( err, 2u );
					done = true;
				}
				else
				{
					if ( ng.y > 0x00FFFFFFu )
					{
						if ( sp < SHARED_STACK )
							my_stack[ TRAVERSE_THREADS * sp++ ] = ng;
						else if ( sp < TRAVERSAL_STACK )
							stack[ sp++ - SHARED_STACK ] = ng;
						else
							atomicOr( err, 1u );
					}
					if ( COUNT ) ++wnodes;
					visit_node( nodes, r, node, tmin, hit.t * grow, ng, tg );
				}
			}
			else
				done = true;
		}
		if ( done )
		{
			io.finish( item, hit, found );
			active = false;
		}
	}
	if ( COUNT )
	{
		for ( int o = 16; o; o >>= 1 )
		{
			wnodes += __shfl_xor_sync( FULL_MASK, wnodes, o );
			wtris += __shfl_xor_sync( FULL_MASK, wtris, o );
		}
		if ( lane == 0 )
		{
			atomicAdd( work, (unsigned long long)wnodes );
			atomicAdd( work + 1, (unsigned long long)wtris );
		}
	}
}

}  // namespace cr
