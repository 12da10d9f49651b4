// GPU BVH builder: replaces the reference's recursive host builder
// (createBVH / doCreateBVH / plainlizeBVH, src/core/primitive/mesh.cu:35-143).
//
//  1. per-triangle boxes, centroid bounds            k_tri_boxes
//  2. 63-bit Morton codes of the centroids           k_morton
//  3. radix sort (CUB) of (code, triangle)
//  4. binary tree: locally-ordered clustering (PLOC, the default:
//     k_ploc_*), or the radix tree of Karras (HPG 2012, k_karras) with
//  5. bottom-up boxes and SAH leaf/split costs       k_bottom_up
//     (leaves of up to 3 triangles where the SAH says a leaf is cheaper;
//     PLOC takes the same decision as it merges)
//  6. top-down collapse into quantised 8-wide nodes  k_collapse (one level
//     per launch): each wide node opens its binary subtree greedily by the
//     largest child surface area until 8 children, assigns children to slots
//     in ray-octant order, quantises child boxes to 8 bits per plane and
//     writes its leaf triangles contiguously in traversal order.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "cr_device.cuh"

namespace cr
{
namespace
{

struct BNode
{
	float4 lo, hi;       // lo.w = SAH cost, hi.w unused
	int left, right;     // unified ids: internal i -> i, leaf k -> n_int + k
	int parent;
	int first, count;    // sorted primitive range
	int leaf;            // 1 if this node becomes a wide-BVH leaf
};

__device__ __forceinline__ void atomic_min_f( float *a, float v )
{
	if ( v >= 0.f )
		atomicMin( reinterpret_cast<int *>( a ), __float_as_int( v ) );
	else
		atomicMax( reinterpret_cast<unsigned *>( a ), __float_as_uint( v ) );
}
__device__ __forceinline__ void atomic_max_f( float *a, float v )
{
	if ( v >= 0.f )
		atomicMax( reinterpret_cast<int *>( a ), __float_as_int( v ) );
	else
		atomicMin( reinterpret_cast<unsigned *>( a ), __float_as_uint( v ) );
}

__device__ __forceinline__ float area( float3 lo, float3 hi )
{
	float3 e = f3( fmaxf( hi.x - lo.x, 0.f ), fmaxf( hi.y - lo.y, 0.f ), fmaxf( hi.z - lo.z, 0.f ) );
	return 2.f * ( e.x * e.y + e.y * e.z + e.z * e.x );
}

// src: 3 float4 per triangle (v0, v1, v2) in global order.
__global__ void k_tri_boxes( const float4 *src, uint32_t n, float4 *blo, float4 *bhi, float *cbounds )
{
	float3 lo = f3( INFINITY, INFINITY, INFINITY ), hi = f3( -INFINITY, -INFINITY, -INFINITY );
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		float3 a = f3( src[ 3 * i ] ), b = f3( src[ 3 * i + 1 ] ), c = f3( src[ 3 * i + 2 ] );
		float3 l = f3( fminf( a.x, fminf( b.x, c.x ) ), fminf( a.y, fminf( b.y, c.y ) ), fminf( a.z, fminf( b.z, c.z ) ) );
		float3 h = f3( fmaxf( a.x, fmaxf( b.x, c.x ) ), fmaxf( a.y, fmaxf( b.y, c.y ) ), fmaxf( a.z, fmaxf( b.z, c.z ) ) );
		blo[ i ] = make_float4( l.x, l.y, l.z, 0.f );
		bhi[ i ] = make_float4( h.x, h.y, h.z, 0.f );
		float3 c3 = ( l + h ) * 0.5f;
		lo = f3( fminf( lo.x, c3.x ), fminf( lo.y, c3.y ), fminf( lo.z, c3.z ) );
		hi = f3( fmaxf( hi.x, c3.x ), fmaxf( hi.y, c3.y ), fmaxf( hi.z, c3.z ) );
	}
	for ( int o = 16; o; o >>= 1 )
	{
		lo.x = fminf( lo.x, __shfl_xor_sync( ~0u, lo.x, o ) );
		lo.y = fminf( lo.y, __shfl_xor_sync( ~0u, lo.y, o ) );
		lo.z = fminf( lo.z, __shfl_xor_sync( ~0u, lo.z, o ) );
		hi.x = fmaxf( hi.x, __shfl_xor_sync( ~0u, hi.x, o ) );
		hi.y = fmaxf( hi.y, __shfl_xor_sync( ~0u, hi.y, o ) );
		hi.z = fmaxf( hi.z, __shfl_xor_sync( ~0u, hi.z, o ) );
	}
	if ( ( threadIdx.x & 31 ) == 0 )
	{
		atomic_min_f( cbounds + 0, lo.x ), atomic_min_f( cbounds + 1, lo.y ), atomic_min_f( cbounds + 2, lo.z );
		atomic_max_f( cbounds + 3, hi.x ), atomic_max_f( cbounds + 4, hi.y ), atomic_max_f( cbounds + 5, hi.z );
	}
}

__device__ __forceinline__ uint64_t spread21( uint64_t x )
{
	x &= 0x1FFFFFull;
	x = ( x | x << 32 ) & 0x1F00000000FFFFull;
	x = ( x | x << 16 ) & 0x1F0000FF0000FFull;
	x = ( x | x << 8 ) & 0x100F00F00F00F00Full;
	x = ( x | x << 4 ) & 0x10C30C30C30C30C3ull;
	x = ( x | x << 2 ) & 0x1249249249249249ull;
	return x;
}

__global__ void k_morton( const float4 *blo, const float4 *bhi, uint32_t n, const float *cb, uint64_t *keys,
						  uint32_t *vals )
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if ( i >= n ) return;
	float3 lo = f3( cb[ 0 ], cb[ 1 ], cb[ 2 ] ), hi = f3( cb[ 3 ], cb[ 4 ], cb[ 5 ] );
	float3 c = ( f3( blo[ i ] ) + f3( bhi[ i ] ) ) * 0.5f;
	const float S = 2097151.f;
	float ex = hi.x - lo.x, ey = hi.y - lo.y, ez = hi.z - lo.z;
	uint64_t x = uint64_t( ex > 0 ? fminf( fmaxf( ( c.x - lo.x ) / ex, 0.f ), 1.f ) * S : 0.f );
	uint64_t y = uint64_t( ey > 0 ? fminf( fmaxf( ( c.y - lo.y ) / ey, 0.f ), 1.f ) * S : 0.f );
	uint64_t z = uint64_t( ez > 0 ? fminf( fmaxf( ( c.z - lo.z ) / ez, 0.f ), 1.f ) * S : 0.f );
	keys[ i ] = ( spread21( x ) << 2 ) | ( spread21( y ) << 1 ) | spread21( z );
	vals[ i ] = i;
}

// Common prefix length of keys i and j (ties broken by index), -1 outside.
__device__ __forceinline__ int delta( const uint64_t *k, int n, int i, int j )
{
	if ( j < 0 || j >= n ) return -1;
	uint64_t a = k[ i ], b = k[ j ];
	if ( a == b ) return 64 + __clz( uint32_t( i ^ j ) );
	return __clzll( a ^ b );
}

__global__ void k_karras( const uint64_t *k, int n, BNode *nodes )
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	int n_int = n - 1;
	if ( i >= n_int ) return;
	int d = ( delta( k, n, i, i + 1 ) - delta( k, n, i, i - 1 ) ) >= 0 ? 1 : -1;
	int dmin = delta( k, n, i, i - d );
	int lmax = 2;
	while ( delta( k, n, i, i + lmax * d ) > dmin ) lmax <<= 1;
	int l = 0;
	for ( int t = lmax >> 1; t >= 1; t >>= 1 )
		if ( delta( k, n, i, i + ( l + t ) * d ) > dmin ) l += t;
	int j = i + l * d;
	int dnode = delta( k, n, i, j );
	int s = 0;
	int t = l;
	do
	{
		t = ( t + 1 ) >> 1;
		if ( delta( k, n, i, i + ( s + t ) * d ) > dnode ) s += t;
	} while ( t > 1 );
	int g = i + s * d + min( d, 0 );
	int lo = min( i, j ), hi = max( i, j );
	int left = ( lo == g ) ? n_int + g : g;
	int right = ( hi == g + 1 ) ? n_int + g + 1 : g + 1;
	nodes[ i ].left = left;
	nodes[ i ].right = right;
	nodes[ i ].first = lo;
	nodes[ i ].count = hi - lo + 1;
	nodes[ left ].parent = i;
	nodes[ right ].parent = i;
}

__global__ void k_bottom_up( int n, const uint32_t *order, const float4 *blo, const float4 *bhi, BNode *nodes,
							 int *flags, BuildParams bp )
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if ( k >= n ) return;
	int n_int = n - 1;
	int id = n_int + k;
	uint32_t prim = order[ k ];
	float4 lo = blo[ prim ], hi = bhi[ prim ];
	float a = area( f3( lo ), f3( hi ) );
	lo.w = bp.cost_tri * a;
	nodes[ id ].lo = lo;
	nodes[ id ].hi = hi;
	nodes[ id ].first = k;
	nodes[ id ].count = 1;
	nodes[ id ].leaf = 1;
	nodes[ id ].left = nodes[ id ].right = -1;
	if ( n == 1 ) return;
	int p = nodes[ id ].parent;
	while ( p >= 0 )
	{
		__threadfence();
		if ( atomicAdd( flags + p, 1 ) == 0 ) return;  // the sibling finishes this node
		__threadfence();
		BNode &nd = nodes[ p ];
		const BNode &L = nodes[ nd.left ];
		const BNode &R = nodes[ nd.right ];
		float4 l0 = __ldcg( &L.lo ), l1 = __ldcg( &L.hi );
		float4 r0 = __ldcg( &R.lo ), r1 = __ldcg( &R.hi );
		float3 mlo = f3( fminf( l0.x, r0.x ), fminf( l0.y, r0.y ), fminf( l0.z, r0.z ) );
		float3 mhi = f3( fmaxf( l1.x, r1.x ), fmaxf( l1.y, r1.y ), fmaxf( l1.z, r1.z ) );
		float A = area( mlo, mhi );
		float split = bp.cost_node * A + l0.w + r0.w;
		float leafc = bp.cost_tri * A * float( nd.count );
		bool as_leaf = nd.count <= bp.max_leaf && leafc <= split;
		nd.lo = make_float4( mlo.x, mlo.y, mlo.z, as_leaf ? leafc : split );
		nd.hi = make_float4( mhi.x, mhi.y, mhi.z, 0.f );
		nd.leaf = as_leaf ? 1 : 0;
		p = nd.parent;
	}
}

// ----------------------------------------------------------------------------
// Locally-ordered clustering (PLOC; Meister and Bittner, "Parallel Locally-
// Ordered Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG
// 2018), in our own code.  The clusters start as the Morton-sorted leaves; each
// round every cluster finds the cluster within `radius` positions whose merged
// box has the smallest surface area, mutual nearest neighbours merge into a new
// internal node (kept at the lower position, bottom-up SAH leaf decision as in
// k_bottom_up), and the survivors are compacted in order.
__global__ void k_ploc_leaves( int n, const uint32_t *order, const float4 *blo, const float4 *bhi, BNode *nodes,
							   int *clusters, BuildParams bp )
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if ( k >= n ) return;
	int id = ( n - 1 ) + k;
	uint32_t prim = order[ k ];
	float4 lo = blo[ prim ], hi = bhi[ prim ];
	lo.w = bp.cost_tri * area( f3( lo ), f3( hi ) );
	BNode &b = nodes[ id ];
	b.lo = lo, b.hi = hi;
	b.left = b.right = -1, b.parent = -1;
	b.first = k, b.count = 1, b.leaf = 1;
	clusters[ k ] = id;
}

__device__ __forceinline__ float merged_area( const BNode &a, const BNode &b )
{
	return area( f3( fminf( a.lo.x, b.lo.x ), fminf( a.lo.y, b.lo.y ), fminf( a.lo.z, b.lo.z ) ),
				 f3( fmaxf( a.hi.x, b.hi.x ), fmaxf( a.hi.y, b.hi.y ), fmaxf( a.hi.z, b.hi.z ) ) );
}

// Nearest neighbour of every cluster within `radius` positions (ties: lower position).
__global__ void k_ploc_nn( const int *clusters, int m, const BNode *nodes, int *nn, int radius )
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if ( i >= m ) return;
	const BNode &a = nodes[ clusters[ i ] ];
	float best = INFINITY;
	int bj = -1;
	int j0 = max( 0, i - radius ), j1 = min( m - 1, i + radius );
	for ( int j = j0; j <= j1; ++j )
	{
		if ( j == i ) continue;
		float d = merged_area( a, nodes[ clusters[ j ] ] );
		if ( d < best ) best = d, bj = j;
	}
	nn[ i ] = bj;
}

// Mutual nearest neighbours merge; `keep` flags the surviving positions.
__global__ void k_ploc_merge( int *clusters, const int *nn, int m, BNode *nodes, int *node_counter, int *keep,
							  BuildParams bp )
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if ( i >= m ) return;
	int j = nn[ i ];
	bool mutual = j >= 0 && nn[ j ] == i;
	if ( !mutual )
	{
		keep[ i ] = 1;
		return;
	}
	if ( i > j )
	{
		keep[ i ] = 0;  // merged into position j
		return;
	}
	int l = clusters[ i ], r = clusters[ j ];
	int id = atomicAdd( node_counter, 1 );
	const BNode &L = nodes[ l ];
	const BNode &R = nodes[ r ];
	float3 mlo = f3( fminf( L.lo.x, R.lo.x ), fminf( L.lo.y, R.lo.y ), fminf( L.lo.z, R.lo.z ) );
	float3 mhi = f3( fmaxf( L.hi.x, R.hi.x ), fmaxf( L.hi.y, R.hi.y ), fmaxf( L.hi.z, R.hi.z ) );
	float A = area( mlo, mhi );
	int count = L.count + R.count;
	float split = bp.cost_node * A + L.lo.w + R.lo.w;
	float leafc = bp.cost_tri * A * float( count );
	bool as_leaf = count <= bp.max_leaf && leafc <= split;
	BNode &nd = nodes[ id ];
	nd.lo = make_float4( mlo.x, mlo.y, mlo.z, as_leaf ? leafc : split );
	nd.hi = make_float4( mhi.x, mhi.y, mhi.z, 0.f );
	nd.left = l, nd.right = r, nd.parent = -1;
	nd.first = 0, nd.count = count, nd.leaf = as_leaf ? 1 : 0;
	nodes[ l ].parent = id, nodes[ r ].parent = id;
	clusters[ i ] = id;
	keep[ i ] = 1;
}

__global__ void k_ploc_compact( const int *clusters, const int *keep, const int *pos, int m, int *out )
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if ( i < m && keep[ i ] ) out[ pos[ i ] ] = clusters[ i ];
}

// Depth-first leaf ranges, top-down over the internal nodes created in one
// merge round (ids id0 .. id1-1; their parents were created later).
__global__ void k_ploc_ranges( BNode *nodes, int id0, int id1 )
{
	int id = id0 + blockIdx.x * blockDim.x + threadIdx.x;
	if ( id >= id1 ) return;
	const BNode &nd = nodes[ id ];
	nodes[ nd.left ].first = nd.first;
	nodes[ nd.right ].first = nd.first + nodes[ nd.left ].count;
}

// Leaf k (Morton position) -> its depth-first position: the primitive order
// the collapse writes triangles in.
__global__ void k_ploc_order( int n, const BNode *nodes, const uint32_t *sorted, uint32_t *order )
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if ( k >= n ) return;
	order[ nodes[ n - 1 + k ].first ] = sorted[ k ];
}

// ----------------------------------------------------------------------------
// Collapse planning by dynamic programming over the binary tree (after Ylitie,
// Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs", HPG 2017, section 4.1), in our own code.  For every
// binary node m and slot budget i = 1..8, C(m, i) is the least SAH cost of
// representing m's subtree by at most i wide-node children:
//   C(m, 1)  = min(leaf: A(m) count c_tri  if count <= max_leaf,
//                  wide node: A(m) c_node + D(m, 8))
//   C(m, i)  = min(C(m, i-1), D(m, i))                          (i >= 2)
//   D(m, i)  = min over k of C(left, k) + C(right, i - k)
// One decision byte per (m, i): bit 7 = "C(m, i) is C(m, i-1)", low bits = the
// best k of D(m, i); byte 0 = "m is a leaf" for i = 1.  Byte 0 of a node that
// becomes a wide node also keeps, in bits 1-3, the best k of D(m, 8) - 1.
constexpr float DP_INF = 3.0e38f;

__global__ void k_dp_leaves( int n, const BNode *nodes, float *cost, uint8_t *dec, BuildParams bp )
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if ( k >= n ) return;
	int id = ( n - 1 ) + k;
	const BNode &b = nodes[ id ];
	float c = bp.dp_cost_tri * area( f3( b.lo ), f3( b.hi ) );
	for ( int i = 0; i < 8; ++i ) cost[ 8 * size_t( id ) + i ] = c;
	dec[ 8 * size_t( id ) ] = 1;
	for ( int i = 1; i < 8; ++i ) dec[ 8 * size_t( id ) + i ] = 0x80;
}

// The internal nodes created in one clustering round (their children exist).
__global__ void k_dp_round( BNode *nodes, int id0, int id1, float *cost, uint8_t *dec, BuildParams bp )
{
	int id = id0 + blockIdx.x * blockDim.x + threadIdx.x;
	if ( id >= id1 ) return;
	BNode &nd = nodes[ id ];
	const float *cl = cost + 8 * size_t( nd.left ), *cr = cost + 8 * size_t( nd.right );
	float A = area( f3( nd.lo ), f3( nd.hi ) );
	float D[ 9 ];
	uint8_t K[ 9 ];
	for ( int i = 2; i <= 8; ++i )
	{
		float best = DP_INF;
		uint8_t bk = 1;
		for ( int k = 1; k < i; ++k )
		{
			float c = cl[ k - 1 ] + cr[ i - k - 1 ];
			if ( c < best ) best = c, bk = uint8_t( k );
		}
		D[ i ] = best, K[ i ] = bk;
	}
	float leafc = nd.count <= bp.max_leaf ? bp.dp_cost_tri * A * float( nd.count ) : DP_INF;
	float internal = bp.dp_cost_node * A + D[ 8 ];
	bool leaf = leafc <= internal;
	float C[ 8 ];
	C[ 0 ] = leaf ? leafc : internal;
	uint8_t *d = dec + 8 * size_t( id );
	d[ 0 ] = uint8_t( ( leaf ? 1 : 0 ) | ( ( K[ 8 ] - 1 ) << 1 ) );
	for ( int i = 2; i <= 8; ++i )
	{
		bool prev = C[ i - 2 ] <= D[ i ];
		C[ i - 1 ] = prev ? C[ i - 2 ] : D[ i ];
		d[ i - 1 ] = uint8_t( ( prev ? 0x80 : 0 ) | K[ i ] );
	}
	for ( int i = 0; i < 8; ++i ) cost[ 8 * size_t( id ) + i ] = C[ i ];
	nd.leaf = leaf ? 1 : 0;
}

// The children of a wide node built from binary node m: the roots of the best
// representation of m's two subtrees with 8 slots.  Returns their count (0 on
// a stack overflow, which the caller reports).
__device__ __forceinline__ int dp_children( const BNode *bn, const uint8_t *dec, int m, int *ch )
{
	int sn[ 16 ], si[ 16 ], sp = 0, nc = 0;
	const int k8 = ( ( dec[ 8 * size_t( m ) ] >> 1 ) & 7 ) + 1;
	sn[ sp ] = bn[ m ].right, si[ sp++ ] = 8 - k8;
	sn[ sp ] = bn[ m ].left, si[ sp++ ] = k8;
	while ( sp > 0 )
	{
		--sp;
		int x = sn[ sp ], i = si[ sp ];
		const uint8_t *d = dec + 8 * size_t( x );
		while ( i > 1 && ( d[ i - 1 ] & 0x80 ) ) --i;
		if ( i == 1 )
		{
			if ( nc == 8 ) return 0;
			ch[ nc++ ] = x;
		}
		else
		{
			if ( sp + 2 > 16 ) return 0;
			int k = d[ i - 1 ] & 0x7F;
			sn[ sp ] = bn[ x ].right, si[ sp++ ] = i - k;
			sn[ sp ] = bn[ x ].left, si[ sp++ ] = k;
		}
	}
	return nc;
}

struct WorkItem
{
	int bnode;
	uint32_t wnode;
};

__device__ __forceinline__ uint8_t quant_lo( float c, float p, float s, float inv )
{
	float q = floorf( ( c - p ) * inv );
	q = fminf( fmaxf( q, 0.f ), 255.f );
	while ( q > 0.f && p + q * s > c ) q -= 1.f;
	return uint8_t( q );
}
__device__ __forceinline__ uint8_t quant_hi( float c, float p, float s, float inv )
{
	float q = ceilf( ( c - p ) * inv );
	q = fminf( fmaxf( q, 0.f ), 255.f );
	while ( q < 255.f && p + q * s < c ) q += 1.f;
	return uint8_t( q );
}

// Smallest biased exponent e with 2^(e-127) * 255 >= extent.
__device__ __forceinline__ uint32_t quant_exp( float extent )
{
	if ( !( extent > 0.f ) ) return 1u;
	int e = int( ceilf( log2f( extent / 255.f ) ) );
	e = max( e, -126 );
	while ( ldexpf( 255.f, e ) < extent ) ++e;
	return uint32_t( e + 127 );
}

__global__ void k_collapse( const WorkItem *work, const uint32_t *n_work, WorkItem *next, uint32_t *n_next,
							const BNode *bn, int n_int, const uint32_t *order, const float4 *src, WNode *wn,
							float4 *tris, uint32_t *counters /* [0] nodes, [1] tris, [2] max depth, [7] errors */,
							uint32_t depth, const uint8_t *dec )
{
	uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
	if ( w >= *n_work ) return;
	WorkItem it = work[ w ];
	int ch[ 8 ];
	int nc = 0;
	const BNode &root = bn[ it.bnode ];
	if ( root.leaf )
		ch[ nc++ ] = it.bnode;
	else if ( dec )
	{
		nc = dp_children( bn, dec, it.bnode, ch );
		if ( nc == 0 )
		{
			// cannot happen for a consistent plan; fall back to the two children
			atomicAdd( counters + 7, 1u );
			ch[ 0 ] = root.left, ch[ 1 ] = root.right, nc = 2;
		}
	}
	else
	{
		ch[ nc++ ] = root.left;
		ch[ nc++ ] = root.right;
		while ( nc < 8 )
		{
			int best = -1;
			float ba = -1.f;
			for ( int c = 0; c < nc; ++c )
			{
				const BNode &b = bn[ ch[ c ] ];
				if ( b.leaf ) continue;
				float a = area( f3( b.lo ), f3( b.hi ) );
				if ( a > ba ) ba = a, best = c;
			}
			if ( best < 0 ) break;
			int id = ch[ best ];
			ch[ best ] = bn[ id ].left;
			ch[ nc++ ] = bn[ id ].right;
		}
	}
	// Octant slot assignment: slot s receives the child nearest along
	// direction signs s (bit0: -x, bit1: -y, bit2: -z), greedily.
	float3 plo = f3( root.lo ), phi = f3( root.hi );
	float3 pc = ( plo + phi ) * 0.5f;
	int child_in[ 8 ];
	for ( int s = 0; s < 8; ++s ) child_in[ s ] = -1;
	uint32_t used_c = 0, used_s = 0;
	for ( int round = 0; round < nc; ++round )
	{
		float best = INFINITY;
		int bc = 0, bs = 0;
		for ( int c = 0; c < nc; ++c )
		{
			if ( used_c >> c & 1u ) continue;
			const BNode &b = bn[ ch[ c ] ];
			float3 cc = ( f3( b.lo ) + f3( b.hi ) ) * 0.5f - pc;
			for ( int s = 0; s < 8; ++s )
			{
				if ( used_s >> s & 1u ) continue;
				float3 dir = f3( ( s & 1 ) ? -1.f : 1.f, ( s & 2 ) ? -1.f : 1.f, ( s & 4 ) ? -1.f : 1.f );
				float cost = dot( cc, dir );
				if ( cost < best ) best = cost, bc = c, bs = s;
			}
		}
		used_c |= 1u << bc;
		used_s |= 1u << bs;
		child_in[ bs ] = bc;
	}
	// Allocate children and triangles.
	uint32_t n_internal = 0, n_tri = 0;
	for ( int c = 0; c < nc; ++c )
	{
		const BNode &b = bn[ ch[ c ] ];
		if ( b.leaf )
			n_tri += b.count;
		else
			++n_internal;
	}
	uint32_t child_base = n_internal ? atomicAdd( counters + 0, n_internal ) : 0;
	uint32_t tri_base = atomicAdd( counters + 1, n_tri );
	WNode nd;
	float3 ext = phi - plo;
	uint32_t ex = quant_exp( ext.x ), ey = quant_exp( ext.y ), ez = quant_exp( ext.z );
	float sx = __uint_as_float( ex << 23 ), sy = __uint_as_float( ey << 23 ), sz = __uint_as_float( ez << 23 );
	float ix = 1.f / sx, iy = 1.f / sy, iz = 1.f / sz;
	nd.px = plo.x, nd.py = plo.y, nd.pz = plo.z;
	nd.ex = uint8_t( ex ), nd.ey = uint8_t( ey ), nd.ez = uint8_t( ez );
	nd.imask = 0;
	nd.child_base = child_base;
	nd.tri_base = tri_base;
	uint32_t rank = 0, toff = 0;
	for ( int s = 0; s < 8; ++s )
	{
		int c = child_in[ s ];
		if ( c < 0 )
		{
			nd.meta[ s ] = 0;
			nd.qlo_x[ s ] = nd.qlo_y[ s ] = nd.qlo_z[ s ] = 255;
			nd.qhi_x[ s ] = nd.qhi_y[ s ] = nd.qhi_z[ s ] = 0;
			continue;
		}
		const BNode &b = bn[ ch[ c ] ];
		nd.qlo_x[ s ] = quant_lo( b.lo.x, plo.x, sx, ix );
		nd.qlo_y[ s ] = quant_lo( b.lo.y, plo.y, sy, iy );
		nd.qlo_z[ s ] = quant_lo( b.lo.z, plo.z, sz, iz );
		nd.qhi_x[ s ] = quant_hi( b.hi.x, plo.x, sx, ix );
		nd.qhi_y[ s ] = quant_hi( b.hi.y, plo.y, sy, iy );
		nd.qhi_z[ s ] = quant_hi( b.hi.z, plo.z, sz, iz );
		if ( b.leaf )
		{
			// the leaf's triangle count in unary (1, 3 or 7) above its offset
			nd.meta[ s ] = uint8_t( ( ( ( 1u << b.count ) - 1u ) << 5 ) | toff );
			for ( int k = 0; k < b.count; ++k )
			{
				uint32_t prim = order[ b.first + k ];
				float4 *dst = tris + 3 * size_t( tri_base + toff + k );
				float4 a = src[ 3 * size_t( prim ) ], bb = src[ 3 * size_t( prim ) + 1 ], cc = src[ 3 * size_t( prim ) + 2 ];
				dst[ 0 ] = make_float4( a.x, a.y, a.z, __uint_as_float( prim ) );
				dst[ 1 ] = make_float4( bb.x, bb.y, bb.z, 0.f );
				dst[ 2 ] = cc;  // w: 0 for a triangle, r^2 for a sphere
			}
			toff += b.count;
		}
		else
		{
			nd.meta[ s ] = 0;
			nd.imask |= uint8_t( 1u << s );
			uint32_t q = atomicAdd( n_next, 1u );
			next[ q ] = WorkItem{ ch[ c ], child_base + rank };
			++rank;
		}
	}
	wn[ it.wnode ] = nd;
	atomicMax( counters + 2, depth );
}

void check( cudaError_t e, const char *what )
{
	if ( e != cudaSuccess ) throw std::runtime_error( std::string( what ) + ": " + cudaGetErrorString( e ) );
}

}  // namespace

void build_wide_bvh( const float4 *d_src, uint32_t n, WideBvh &out, cudaStream_t st, const BuildParams &bp )
{
	// leaves of at most 3 primitives: a node's meta byte holds the count in unary (3 bits)
	if ( bp.max_leaf < 1 || bp.max_leaf > 3 || bp.radius < 1 || bp.radius > 256 || !( bp.cost_node > 0.f ) ||
		 !( bp.cost_tri > 0.f ) )
		throw std::runtime_error( "bvh: build parameters out of range" );
	out.n_nodes = 0;
	out.n_tris = n;
	out.depth = 0;
	if ( n == 0 ) return;
	float4 *blo, *bhi;
	float *cb;
	uint64_t *keys, *keys2;
	uint32_t *vals, *vals2;
	BNode *bn;
	int *flags;
	WorkItem *wa, *wb;
	uint32_t *cnt;  // [0] nodes [1] tris [2] depth [3] n_work a [4] n_work b
	size_t n_b = 2 * size_t( n ) - 1;
	check( cudaMallocAsync( &blo, sizeof( float4 ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &bhi, sizeof( float4 ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &cb, sizeof( float ) * 6, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &keys, sizeof( uint64_t ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &keys2, sizeof( uint64_t ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &vals, sizeof( uint32_t ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &vals2, sizeof( uint32_t ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &bn, sizeof( BNode ) * n_b, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &flags, sizeof( int ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &wa, sizeof( WorkItem ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &wb, sizeof( WorkItem ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &cnt, sizeof( uint32_t ) * 8, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &out.nodes, sizeof( WNode ) * n, device_pool(), st ), "bvh alloc" );
	check( cudaMallocAsync( &out.tris, sizeof( float4 ) * 3 * n, device_pool(), st ), "bvh alloc" );

	float init[ 6 ] = { INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY };
	check( cudaMemcpyAsync( cb, init, sizeof init, cudaMemcpyHostToDevice, st ), "bvh init" );
	check( cudaMemsetAsync( flags, 0, sizeof( int ) * n, st ), "bvh init" );
	check( cudaMemsetAsync( bn, 0xFF, sizeof( BNode ) * n_b, st ), "bvh init" );
	int tb = 256;
	int gb = int( std::min<uint32_t>( ( n + tb - 1 ) / tb, 148u * 8u ) );
	k_tri_boxes<<<gb, tb, 0, st>>>( d_src, n, blo, bhi, cb );
	k_morton<<<( n + tb - 1 ) / tb, tb, 0, st>>>( blo, bhi, n, cb, keys, vals );
	size_t temp = 0;
	check( cub::DeviceRadixSort::SortPairs( nullptr, temp, keys, keys2, vals, vals2, int( n ), 0, 63, st ), "sort" );
	void *dtemp;
	check( cudaMallocAsync( &dtemp, temp, device_pool(), st ), "bvh alloc" );
	check( cub::DeviceRadixSort::SortPairs( dtemp, temp, keys, keys2, vals, vals2, int( n ), 0, 63, st ), "sort" );
	int root_id = 0;
	const uint32_t *order = vals2;
	float *dp_cost = nullptr;
	uint8_t *dp_dec = nullptr;
	if ( !bp.ploc || n < 2 )
	{
		if ( n > 1 ) k_karras<<<( n - 1 + tb - 1 ) / tb, tb, 0, st>>>( keys2, int( n ), bn );
		k_bottom_up<<<( n + tb - 1 ) / tb, tb, 0, st>>>( int( n ), vals2, blo, bhi, bn, flags, bp );
		check( cudaGetLastError(), "bvh kernels" );
	}
	else
	{
		// clusters, neighbours, flags, positions and the depth-first order reuse
		// the Morton buffers: keys (as two int arrays), keys2's second half, vals
		int *cl = reinterpret_cast<int *>( keys ), *cl2 = cl + n;
		int *nn = reinterpret_cast<int *>( keys2 ) + n, *keep = flags, *pos = reinterpret_cast<int *>( wa );
		int *counter = reinterpret_cast<int *>( cnt ) + 6;
		check( cudaMemsetAsync( counter, 0, sizeof( int ), st ), "bvh init" );
		k_ploc_leaves<<<( n + tb - 1 ) / tb, tb, 0, st>>>( int( n ), vals2, blo, bhi, bn, cl, bp );
		size_t scan_temp = 0;
		check( cub::DeviceScan::ExclusiveSum( nullptr, scan_temp, keep, pos, int( n ), st ), "scan" );
		void *stemp;
		check( cudaMallocAsync( &stemp, scan_temp, device_pool(), st ), "bvh alloc" );
		std::vector<int> round_base;  // first internal id of each merge round
		int m = int( n ), created = 0;
		while ( m > 1 )
		{
			int gm = ( m + tb - 1 ) / tb;
			k_ploc_nn<<<gm, tb, 0, st>>>( cl, m, bn, nn, bp.radius );
			k_ploc_merge<<<gm, tb, 0, st>>>( cl, nn, m, bn, counter, keep, bp );
			check( cub::DeviceScan::ExclusiveSum( stemp, scan_temp, keep, pos, m, st ), "scan" );
			k_ploc_compact<<<gm, tb, 0, st>>>( cl, keep, pos, m, cl2 );
			check( cudaGetLastError(), "bvh ploc" );
			int last[ 2 ], made = 0;
			check( cudaMemcpyAsync( last, pos + m - 1, sizeof( int ), cudaMemcpyDeviceToHost, st ), "bvh ploc" );
			check( cudaMemcpyAsync( last + 1, keep + m - 1, sizeof( int ), cudaMemcpyDeviceToHost, st ), "bvh ploc" );
			check( cudaMemcpyAsync( &made, counter, sizeof( int ), cudaMemcpyDeviceToHost, st ), "bvh ploc" );
			check( cudaStreamSynchronize( st ), "bvh ploc" );
			int m2 = last[ 0 ] + last[ 1 ];
			if ( m2 >= m || made <= created ) throw std::runtime_error( "bvh: clustering made no progress" );
			round_base.push_back( created );
			created = made;
			std::swap( cl, cl2 );
			m = m2;
		}
		if ( created != int( n ) - 1 ) throw std::runtime_error( "bvh: clustering left unmerged clusters" );
		check( cudaMemcpyAsync( &root_id, cl, sizeof( int ), cudaMemcpyDeviceToHost, st ), "bvh ploc" );
		check( cudaStreamSynchronize( st ), "bvh ploc" );
		// depth-first ranges: the root starts at 0; rounds top-down
		int zero = 0;
		check( cudaMemcpyAsync( &bn[ root_id ].first, &zero, sizeof( int ), cudaMemcpyHostToDevice, st ), "bvh ploc" );
		round_base.push_back( created );
		for ( int r = int( round_base.size() ) - 2; r >= 0; --r )
		{
			int id0 = round_base[ r ], id1 = round_base[ r + 1 ];
			k_ploc_ranges<<<( id1 - id0 + tb - 1 ) / tb, tb, 0, st>>>( bn, id0, id1 );
		}
		if ( bp.dp_collapse )
		{
			// collapse plan, bottom-up in creation order (children come from earlier rounds)
			check( cudaMallocAsync( &dp_cost, sizeof( float ) * 8 * n_b, device_pool(), st ), "bvh alloc" );
			check( cudaMallocAsync( &dp_dec, 8 * n_b, device_pool(), st ), "bvh alloc" );
			k_dp_leaves<<<( n + tb - 1 ) / tb, tb, 0, st>>>( int( n ), bn, dp_cost, dp_dec, bp );
			for ( size_t r = 0; r + 1 < round_base.size(); ++r )
			{
				int id0 = round_base[ r ], id1 = round_base[ r + 1 ];
				k_dp_round<<<( id1 - id0 + tb - 1 ) / tb, tb, 0, st>>>( bn, id0, id1, dp_cost, dp_dec, bp );
			}
			check( cudaGetLastError(), "bvh plan" );
		}
		// the depth-first primitive order replaces the Morton order (vals)
		k_ploc_order<<<( n + tb - 1 ) / tb, tb, 0, st>>>( int( n ), bn, vals2, vals );
		check( cudaGetLastError(), "bvh ploc" );
		check( cudaStreamSynchronize( st ), "bvh ploc" );
		cudaFreeAsync( stemp, st );
		order = vals;
	}

	// Root work item: binary root -> wide node 0.
	WorkItem root{ root_id, 0 };
	uint32_t c0[ 8 ] = { 1, 0, 0, 1, 0, 0, 0, 0 };
	check( cudaMemcpyAsync( wa, &root, sizeof root, cudaMemcpyHostToDevice, st ), "bvh root" );
	check( cudaMemcpyAsync( cnt, c0, sizeof c0, cudaMemcpyHostToDevice, st ), "bvh root" );
	uint32_t n_work = 1, depth = 0;
	WorkItem *cur = wa, *nxt = wb;
	uint32_t *ncur = cnt + 3, *nnext = cnt + 4;
	while ( n_work )
	{
		check( cudaMemsetAsync( nnext, 0, sizeof( uint32_t ), st ), "bvh level" );
		k_collapse<<<( n_work + 127 ) / 128, 128, 0, st>>>( cur, ncur, nxt, nnext, bn, int( n ) - 1, order, d_src,
															out.nodes, out.tris, cnt, depth + 1, dp_dec );
		check( cudaGetLastError(), "bvh collapse" );
		check( cudaMemcpyAsync( &n_work, nnext, sizeof( uint32_t ), cudaMemcpyDeviceToHost, st ), "bvh level" );
		check( cudaStreamSynchronize( st ), "bvh level" );
		std::swap( cur, nxt );
		std::swap( ncur, nnext );
		++depth;
		if ( depth > 4096 ) throw std::runtime_error( "bvh: collapse did not terminate" );
	}
	uint32_t res[ 8 ];
	check( cudaMemcpyAsync( res, cnt, sizeof res, cudaMemcpyDeviceToHost, st ), "bvh result" );
	check( cudaStreamSynchronize( st ), "bvh result" );
	out.n_nodes = res[ 0 ];
	out.depth = res[ 2 ];
	if ( res[ 1 ] != n ) throw std::runtime_error( "bvh: triangle count mismatch after collapse" );
	if ( res[ 7 ] ) throw std::runtime_error( "bvh: inconsistent collapse plan" );
	if ( dp_cost ) cudaFreeAsync( dp_cost, st );
	if ( dp_dec ) cudaFreeAsync( dp_dec, st );
	for ( void *p : { (void *)blo, (void *)bhi, (void *)cb, (void *)keys, (void *)keys2, (void *)vals, (void *)vals2,
					  (void *)bn, (void *)flags, (void *)wa, (void *)wb, (void *)cnt, dtemp } )
		cudaFreeAsync( p, st );
}

// Float min / max through the integer order of the IEEE bits (non-negative
// values order as signed ints, negative ones reversed as unsigned).
__device__ __forceinline__ void atomic_min_float( float *a, float v )
{
	if ( v >= 0.f )
		atomicMin( reinterpret_cast<int *>( a ), __float_as_int( v ) );
	else
		atomicMax( reinterpret_cast<unsigned int *>( a ), __float_as_uint( v ) );
}
__device__ __forceinline__ void atomic_max_float( float *a, float v )
{
	if ( v >= 0.f )
		atomicMax( reinterpret_cast<int *>( a ), __float_as_int( v ) );
	else
		atomicMin( reinterpret_cast<unsigned int *>( a ), __float_as_uint( v ) );
}

__global__ void k_flatten_mesh( FlatMesh m, float4 *__restrict__ src, float4 *__restrict__ attrs, float *bounds )
{
	float lo[ 3 ] = { INFINITY, INFINITY, INFINITY }, hi[ 3 ] = { -INFINITY, -INFINITY, -INFINITY };
	for ( uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m.nt; t += gridDim.x * blockDim.x )
	{
		const size_t g = m.g0 + t;
#pragma unroll
		for ( int k = 0; k < 3; ++k )
		{
			const uint32_t vi = m.idx[ 3 * size_t( t ) + k ];
			const float x = m.v[ 3 * size_t( vi ) ], y = m.v[ 3 * size_t( vi ) + 1 ], z = m.v[ 3 * size_t( vi ) + 2 ];
			const int w = k == 0 ? m.shader : k == 1 ? m.prim : m.light;
			src[ 3 * g + k ] = make_float4( x, y, z, 0.f );
			attrs[ 3 * g + k ] = make_float4( m.n[ 3 * size_t( vi ) ], m.n[ 3 * size_t( vi ) + 1 ], m.n[ 3 * size_t( vi ) + 2 ],
											  __int_as_float( w ) );
			// fminf / fmaxf skip a NaN operand, as the host's std::min did
			lo[ 0 ] = fminf( lo[ 0 ], x ), lo[ 1 ] = fminf( lo[ 1 ], y ), lo[ 2 ] = fminf( lo[ 2 ], z );
			hi[ 0 ] = fmaxf( hi[ 0 ], x ), hi[ 1 ] = fmaxf( hi[ 1 ], y ), hi[ 2 ] = fmaxf( hi[ 2 ], z );
		}
	}
#pragma unroll
	for ( int a = 0; a < 3; ++a )
		for ( int o = 16; o; o >>= 1 )
		{
			lo[ a ] = fminf( lo[ a ], __shfl_xor_sync( 0xFFFFFFFFu, lo[ a ], o ) );
			hi[ a ] = fmaxf( hi[ a ], __shfl_xor_sync( 0xFFFFFFFFu, hi[ a ], o ) );
		}
	if ( ( threadIdx.x & 31u ) == 0 )
		for ( int a = 0; a < 3; ++a )
		{
			// NaN coordinates never enter the bounds (fminf / fmaxf drop them);
			// a warp that saw no vertex holds +inf / -inf, which change nothing
			if ( !isnan( lo[ a ] ) ) atomic_min_float( bounds + a, lo[ a ] );
			if ( !isnan( hi[ a ] ) ) atomic_max_float( bounds + 3 + a, hi[ a ] );
		}
}

void flatten_mesh( const FlatMesh &m, float4 *src, float4 *attrs, float *bounds, cudaStream_t st )
{
	if ( m.nt == 0 ) return;
	int dev = 0, sms = 0;
	check( cudaGetDevice( &dev ), "device" );
	check( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ), "device" );
	const int grid = int( std::min<uint64_t>( ( m.nt + 255 ) / 256, uint64_t( sms ) * 8 ) );
	k_flatten_mesh<<<grid, 256, 0, st>>>( m, src, attrs, bounds );
	check( cudaGetLastError(), "flatten launch" );
}

}  // namespace cr
