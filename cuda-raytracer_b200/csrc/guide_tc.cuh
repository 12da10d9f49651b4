// Tensor-core forward pass of the guide MLP on sm_100a (tcgen05 + TMEM).
//
// One CTA of 256 threads holds the weights once and runs two independent
// groups of 128 threads, one per tile of 128 rows (queries).  Every thread
// owns one row: it gathers the row's encoding (hash grid, SH, normal) in
// FP32, rounds it to BF16 and stores it into its tile's shared-memory
// operand.  For each of the 5 layers the group's first thread issues
// tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M = 128, N = 64, K = 16; four
// K steps per layer) with the activations as A and the layer's BF16 weights
// as B, both in shared memory; the accumulators live in tensor memory (64
// columns per tile).  tcgen05.commit signals the group's mbarrier; the
// threads then read their row back with tcgen05.ld, add the bias, apply the
// ReLU, round to BF16 and overwrite their A row for the next layer.  The last
// layer's row is handed to the caller's sink in FP32.  The groups synchronise
// on named barriers of their own, so one group's hash-grid gathers overlap
// the other's MMA round trips.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8 x 16-byte core matrices, element (r, k) at
//     (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
// with LBO = 128 bytes (next 8 columns of K) and SBO = 1024 bytes (next 8
// rows), so one 64-wide block of 8 rows is 1 KB and a K step of 16 advances
// the descriptor start by 256 bytes.
//
// Every wait on the mbarrier is bounded; on a timeout the kernel records
// error bit 8 in the device error word, waits (bounded) for the MMAs it has
// in flight, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "guide.cuh"

namespace cr
{
namespace tc
{
constexpr uint32_t ROWS = 128;                      // MMA tile rows (M)
constexpr uint32_t TILES = 2;                       // tiles per CTA iteration
constexpr uint32_t THREADS = ROWS * TILES;          // one thread per row
constexpr uint32_t LBO = 128, SBO = 1024;           // canonical K-major strides (bytes)
constexpr uint32_t TILE_BYTES = ROWS * G_IN * 2;    // 16 KB of BF16 activations
constexpr uint32_t W_BYTES = G_HID * G_IN * 2;      // 8 KB of BF16 weights per layer
constexpr uint32_t TMEM_COLS = 64 * TILES;          // FP32 accumulators: 64 columns per tile

// Shared-memory map, from a 128-byte aligned base.
constexpr uint32_t OFF_W = 0;
constexpr uint32_t OFF_A = OFF_W + G_LAYERS * W_BYTES;          // 40960
constexpr uint32_t OFF_BIAS = OFF_A + TILES * TILE_BYTES;       // 73728
constexpr uint32_t OFF_BAR = OFF_BIAS + G_LAYERS * G_HID * 4;   // 75008: one mbarrier per tile
constexpr uint32_t OFF_TMEM = OFF_BAR + 8 * TILES;              // 75024
constexpr uint32_t SMEM_USED = OFF_TMEM + 8;                    // 75032
constexpr uint32_t SMEM_BYTES = SMEM_USED + 128;                // slack for the alignment

// Weight images in device memory: the forward image (layer l: N = out, K = in)
// followed by the transposed image the backward pass uses (N = in, K = out).
constexpr uint32_t WIMG_BYTES = G_LAYERS * W_BYTES;   // 40960
constexpr uint32_t WP_BYTES = 2 * WIMG_BYTES;

constexpr uint32_t WAIT_LIMIT = 1u << 22;  // try_wait rounds before an MMA wait gives up
constexpr uint32_t ERR_MMA_TIMEOUT = 8u;   // device error word bit

// Instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = ( 1u << 4 ) | ( 1u << 7 ) | ( 1u << 10 ) | ( ( 64u >> 3 ) << 17 ) | ( ( ROWS >> 4 ) << 24 );

__host__ __device__ constexpr uint32_t canon( uint32_t r, uint32_t k )
{
	return ( r >> 3 ) * SBO + ( k >> 3 ) * LBO + ( r & 7u ) * 16u + ( k & 7u ) * 2u;
}

// Shared-memory matrix descriptor (sm_100 format): start address >> 4 at bits
// 0-13, LBO >> 4 at 16-29, SBO >> 4 at 32-45, version 1 at 46-47, base offset
// 0, layout type 0 (no swizzle) at 61-63.
__device__ __forceinline__ uint64_t sdesc( uint32_t saddr, uint32_t sbo = SBO )
{
	return uint64_t( ( saddr >> 4 ) & 0x3FFFu ) | ( uint64_t( LBO >> 4 ) << 16 ) | ( uint64_t( sbo >> 4 ) << 32 ) |
		   ( 1ull << 46 );
}

// Canonical K-major offset for a tile whose K extent is 128 (SBO = 16 * LBO).
__host__ __device__ constexpr uint32_t canon128( uint32_t r, uint32_t k )
{
	return ( r >> 3 ) * ( 16u * LBO ) + ( k >> 3 ) * LBO + ( r & 7u ) * 16u + ( k & 7u ) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32( const void *p ) { return uint32_t( __cvta_generic_to_shared( p ) ); }

__device__ __forceinline__ void fence_async_smem() { asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" ); }
__device__ __forceinline__ void tc_before_sync() { asm volatile( "tcgen05.fence::before_thread_sync;" ::: "memory" ); }
__device__ __forceinline__ void tc_after_sync() { asm volatile( "tcgen05.fence::after_thread_sync;" ::: "memory" ); }

__device__ __forceinline__ void mma_bf16( uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate )
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
		:
		: "r"( d_tmem ), "l"( a ), "l"( b ), "r"( IDESC ), "r"( accumulate )
		: "memory" );
}

// Named barrier of tile group t (ids 1 and 2; 0 is __syncthreads), and the
// same barrier as an OR-reduction of a predicate over the group.
// (Immediate barrier ids: a register id makes the compiler reserve all 16.)
static_assert( TILES == 2 && ROWS == 128, "two tile groups of 128 threads" );
__device__ __forceinline__ void group_sync( uint32_t t )
{
	if ( t == 0 )
		asm volatile( "bar.sync 1, 128;" ::: "memory" );
	else
		asm volatile( "bar.sync 2, 128;" ::: "memory" );
}
__device__ __forceinline__ bool group_or( uint32_t t, bool pred )
{
	uint32_t r;
	if ( t == 0 )
		asm volatile(
			"{\n\t.reg .pred p, q;\n\t"
			"setp.ne.u32 p, %1, 0;\n\t"
			"bar.red.or.pred q, 1, 128, p;\n\t"
			"selp.u32 %0, 1, 0, q;\n\t}"
			: "=r"( r )
			: "r"( uint32_t( pred ) )
			: "memory" );
	else
		asm volatile(
			"{\n\t.reg .pred p, q;\n\t"
			"setp.ne.u32 p, %1, 0;\n\t"
			"bar.red.or.pred q, 2, 128, p;\n\t"
			"selp.u32 %0, 1, 0, q;\n\t}"
			: "=r"( r )
			: "r"( uint32_t( pred ) )
			: "memory" );
	return r != 0;
}

__device__ __forceinline__ void mma_commit( uint32_t bar )
{
	asm volatile( "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"( bar ) : "memory" );
}

__device__ __forceinline__ bool mbar_wait( uint32_t bar, uint32_t parity )
{
	for ( uint32_t i = 0; i < WAIT_LIMIT; ++i )
	{
		uint32_t done;
		asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}"
			: "=r"( done )
			: "r"( bar ), "r"( parity )
			: "memory" );
		if ( done ) return true;
	}
	return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16( uint32_t taddr, float *v )
{
	uint32_t r[ 16 ];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 "
		"{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
		: "=r"( r[ 0 ] ), "=r"( r[ 1 ] ), "=r"( r[ 2 ] ), "=r"( r[ 3 ] ), "=r"( r[ 4 ] ), "=r"( r[ 5 ] ), "=r"( r[ 6 ] ),
		  "=r"( r[ 7 ] ), "=r"( r[ 8 ] ), "=r"( r[ 9 ] ), "=r"( r[ 10 ] ), "=r"( r[ 11 ] ), "=r"( r[ 12 ] ),
		  "=r"( r[ 13 ] ), "=r"( r[ 14 ] ), "=r"( r[ 15 ] )
		: "r"( taddr ) );
#pragma unroll
	for ( int i = 0; i < 16; ++i ) v[ i ] = __uint_as_float( r[ i ] );
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile( "tcgen05.wait::ld.sync.aligned;" ::: "memory" ); }

__device__ __forceinline__ uint32_t pack_bf16x2( float a, float b )
{
	__nv_bfloat162 h = __floats2bfloat162_rn( a, b );
	return *reinterpret_cast<uint32_t *>( &h );
}

// Stores 64 values of row r as BF16 into a canonical K-major tile.
__device__ __forceinline__ void store_row( uint8_t *tile, uint32_t r, const float *v )
{
#pragma unroll
	for ( int j = 0; j < 8; ++j )
	{
		uint4 q = make_uint4( pack_bf16x2( v[ 8 * j ], v[ 8 * j + 1 ] ), pack_bf16x2( v[ 8 * j + 2 ], v[ 8 * j + 3 ] ),
							  pack_bf16x2( v[ 8 * j + 4 ], v[ 8 * j + 5 ] ), pack_bf16x2( v[ 8 * j + 6 ], v[ 8 * j + 7 ] ) );
		*reinterpret_cast<uint4 *>( tile + canon( r, 8 * j ) ) = q;
	}
}

// Row r's network input for (x, wo, n), as guide_encode lays it out (the hash
// features from the paired FP16 table), written straight into a canonical
// K-major tile as BF16, 8 values at a time.
__device__ __forceinline__ void encode_store_row( const GuideDev &g, float3 x, float3 wo, float3 n, uint8_t *tile,
												  uint32_t r )
{
	const float3 u = ( x - g.bmin ) * g.binv;
	// Each level's two trilinear features come from the paired FP16 table:
	// each of the cell's four (y, z) edges is one 8-byte load that holds both
	// of its x-corners (a slot and its +x neighbour's, the next slot).  All 48
	// loads of the row are issued before any is used, so the row waits for one
	// L2 round trip rather than one per level (4 % off the inference kernel).
	uint2 pr[ G_LEVELS ][ 4 ];
	float tt[ G_LEVELS ][ 3 ];
#pragma unroll
	for ( int l = 0; l < G_LEVELS; ++l )
	{
		const float res = grid_res( l );
		const float px = fminf( fmaxf( u.x, 0.f ), 1.f ) * res, py = fminf( fmaxf( u.y, 0.f ), 1.f ) * res,
					pz = fminf( fmaxf( u.z, 0.f ), 1.f ) * res;
		const float fx = floorf( px ), fy = floorf( py ), fz = floorf( pz );
		const uint32_t ix = uint32_t( fx ), iy = uint32_t( fy ), iz = uint32_t( fz );
		tt[ l ][ 0 ] = px - fx, tt[ l ][ 1 ] = py - fy, tt[ l ][ 2 ] = pz - fz;
		const uint2 *tab = g.grid_pairs + size_t( l ) * G_T;
#pragma unroll
		for ( int k = 0; k < 4; ++k )
			pr[ l ][ k ] = __ldg( tab + grid_index( l, ix, iy + ( k & 1 ), iz + ( k >> 1 ) ) );
	}
	uint32_t w[ 4 ];
#pragma unroll
	for ( int l = 0; l < G_LEVELS; ++l )
	{
		const float tx = tt[ l ][ 0 ], ty = tt[ l ][ 1 ], tz = tt[ l ][ 2 ];
		float f0 = 0.f, f1 = 0.f;
#pragma unroll
		for ( int k = 0; k < 4; ++k )
		{
			const uint32_t dy = k & 1, dz = k >> 1;
			const float2 a = __half22float2( *reinterpret_cast<const __half2 *>( &pr[ l ][ k ].x ) );
			const float2 b = __half22float2( *reinterpret_cast<const __half2 *>( &pr[ l ][ k ].y ) );
			const float wyz = ( dy ? ty : 1.f - ty ) * ( dz ? tz : 1.f - tz );
			const float w0 = wyz * ( 1.f - tx ), w1 = wyz * tx;
			f0 += w0 * a.x + w1 * b.x;
			f1 += w0 * a.y + w1 * b.y;
		}
		w[ l & 3 ] = pack_bf16x2( f0, f1 );
		if ( ( l & 3 ) == 3 )
			*reinterpret_cast<uint4 *>( tile + canon( r, 8 * ( l >> 2 ) ) ) = make_uint4( w[ 0 ], w[ 1 ], w[ 2 ], w[ 3 ] );
	}
	float sh[ G_SH ];
	sh16( wo.x, wo.y, wo.z, sh );
#pragma unroll
	for ( int j = 0; j < 2; ++j )
		*reinterpret_cast<uint4 *>( tile + canon( r, G_ENC + 8 * j ) ) =
			make_uint4( pack_bf16x2( sh[ 8 * j ], sh[ 8 * j + 1 ] ), pack_bf16x2( sh[ 8 * j + 2 ], sh[ 8 * j + 3 ] ),
						pack_bf16x2( sh[ 8 * j + 4 ], sh[ 8 * j + 5 ] ), pack_bf16x2( sh[ 8 * j + 6 ], sh[ 8 * j + 7 ] ) );
	*reinterpret_cast<uint4 *>( tile + canon( r, G_ENC + G_SH ) ) =
		make_uint4( pack_bf16x2( n.x, n.y ), pack_bf16x2( n.z, 0.f ), 0u, 0u );
	*reinterpret_cast<uint4 *>( tile + canon( r, 48 ) ) = make_uint4( 0u, 0u, 0u, 0u );
	*reinterpret_cast<uint4 *>( tile + canon( r, 56 ) ) = make_uint4( 0u, 0u, 0u, 0u );
}

// Runs the network over rows 0..n-1.  src(i, x, wo, nrm) -> bool fetches row
// i's inputs (false: the row is skipped); sink(i, out) receives the 64 FP32
// outputs of a fetched row (the first OUT_COLS of them: 48 covers the 40 the
// lobes use, 64 gives all).  Wp: the BF16 weights in the shared-memory image
// (G_LAYERS x W_BYTES, canonical layout, 16-byte aligned).  Called by every
// thread of a THREADS-wide CTA with SMEM_BYTES of dynamic shared memory.
template <int OUT_COLS, class Src, class Sink>
__device__ __forceinline__ void mlp_forward_tc( const GuideDev &g, const uint8_t *__restrict__ Wp, uint32_t n,
												Src &&src, Sink &&sink, uint32_t *err )
{
	extern __shared__ uint8_t smem_raw[];
	uint8_t *sm = reinterpret_cast<uint8_t *>( ( reinterpret_cast<uintptr_t>( smem_raw ) + 127 ) & ~uintptr_t( 127 ) );
	const uint32_t tid = threadIdx.x, warp = tid >> 5;
	const uint32_t tile = tid / ROWS, row = tid % ROWS;
	const uint32_t bar = smem_u32( sm + OFF_BAR ) + 8u * tile;  // this group's mbarrier
	uint32_t *tmem_slot = reinterpret_cast<uint32_t *>( sm + OFF_TMEM );
	float *bias = reinterpret_cast<float *>( sm + OFF_BIAS );

	// weights and biases into shared memory (16-byte copies)
	{
		const uint4 *src4 = reinterpret_cast<const uint4 *>( Wp );
		uint4 *dst4 = reinterpret_cast<uint4 *>( sm + OFF_W );
		for ( uint32_t i = tid; i < G_LAYERS * W_BYTES / 16; i += THREADS ) dst4[ i ] = __ldg( src4 + i );
		for ( uint32_t i = tid; i < G_LAYERS * G_HID; i += THREADS ) bias[ i ] = g.b[ i ];
	}
	if ( row == 0 )
	{
		asm volatile( "mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"( bar ) : "memory" );
		asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
	}
	if ( warp == 0 )
	{
		asm volatile( "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"( smem_u32( tmem_slot ) ),
					  "r"( TMEM_COLS )
					  : "memory" );
		asm volatile( "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory" );
	}
	fence_async_smem();
	tc_before_sync();
	__syncthreads();
	tc_after_sync();
	const uint32_t tmem = *tmem_slot;
	// this thread's TMEM lane (row) and its tile's 64 accumulator columns
	const uint32_t my_tmem = tmem + ( ( ( warp & 3u ) * 32u ) << 16 ) + tile * 64u;
	uint8_t *my_tile = sm + OFF_A + tile * TILE_BYTES;
	uint32_t phase = 0;
	bool failed = false;

	for ( uint32_t base = blockIdx.x * THREADS; base < n; base += gridDim.x * THREADS )
	{
		const uint32_t i = base + tid;
		float3 x = f3( 0.f, 0.f, 0.f ), wo = f3( 0.f, 0.f, 1.f ), nrm = f3( 0.f, 0.f, 1.f );
		const bool valid = i < n && src( i, x, wo, nrm );
		if ( valid )
			encode_store_row( g, x, wo, nrm, my_tile, row );
		else
#pragma unroll
			for ( int j = 0; j < 8; ++j ) *reinterpret_cast<uint4 *>( my_tile + canon( row, 8 * j ) ) = make_uint4( 0u, 0u, 0u, 0u );
		for ( int l = 0; l < G_LAYERS; ++l )
		{
			// make this thread's A row visible to the tensor core, then the
			// group's first thread issues the layer for its tile
			fence_async_smem();
			tc_before_sync();
			group_sync( tile );
			if ( row == 0 )
			{
				tc_after_sync();
				for ( uint32_t k = 0; k < G_IN / 16; ++k )
					mma_bf16( tmem + tile * 64u, sdesc( smem_u32( my_tile ) + k * 2u * LBO ),
							  sdesc( smem_u32( sm + OFF_W + l * W_BYTES ) + k * 2u * LBO ), k > 0 );
				mma_commit( bar );
			}
			const bool ok = mbar_wait( bar, phase );
			phase ^= 1u;
			if ( group_or( tile, !ok ) )
			{
				failed = true;
				break;
			}
			tc_after_sync();
			const float *bl = bias + l * G_HID;
			if ( l < G_LAYERS - 1 )
			{
				// 16 columns at a time: bias, ReLU, BF16, back into this row
#pragma unroll
				for ( int c = 0; c < 4; ++c )
				{
					float a[ 16 ];
					tmem_ld16( my_tmem + 16u * c, a );
					tmem_wait_ld();
					uint32_t q[ 8 ];
#pragma unroll
					for ( int k = 0; k < 8; ++k )
						q[ k ] = pack_bf16x2( fmaxf( a[ 2 * k ] + bl[ 16 * c + 2 * k ], 0.f ),
											  fmaxf( a[ 2 * k + 1 ] + bl[ 16 * c + 2 * k + 1 ], 0.f ) );
					*reinterpret_cast<uint4 *>( my_tile + canon( row, 16 * c ) ) = make_uint4( q[ 0 ], q[ 1 ], q[ 2 ], q[ 3 ] );
					*reinterpret_cast<uint4 *>( my_tile + canon( row, 16 * c + 8 ) ) = make_uint4( q[ 4 ], q[ 5 ], q[ 6 ], q[ 7 ] );
				}
			}
			else
			{
				float out[ OUT_COLS ];
#pragma unroll
				for ( int c = 0; c < OUT_COLS / 16; ++c ) tmem_ld16( my_tmem + 16u * c, out + 16 * c );
				tmem_wait_ld();
#pragma unroll
				for ( int k = 0; k < OUT_COLS; ++k ) out[ k ] += bl[ k ];
				if ( valid ) sink( i, out );
			}
			// the next MMA overwrites the accumulators: finish this thread's reads first
			tc_before_sync();
		}
		if ( failed ) break;
	}
	if ( failed )
	{
		if ( row == 0 ) atomicOr( err, ERR_MMA_TIMEOUT );
		// the timed-out phase once more (bounded): no MMA may still write TMEM below
		mbar_wait( bar, phase ^ 1u );
	}
	// both groups done before the tensor memory goes
	tc_before_sync();
	__syncthreads();
	if ( warp == 0 )
	{
		tc_after_sync();
		asm volatile( "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"( tmem ), "r"( TMEM_COLS ) : "memory" );
	}
}

}  // namespace tc
}  // namespace cr
