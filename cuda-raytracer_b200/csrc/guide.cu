// Learned path guiding: parameters, online training and the FP32 kernels.
//
// Training data are the tracer's own path vertices.  For a vertex with inputs
// (x, wo, n) that continued along direction w sampled with density p, the
// incident radiance estimate is Li = (L_path - L_next) / T, where T is the
// path throughput after the vertex and L_next the radiance the path had
// gathered once it reached the next vertex, that vertex's emission included.
// Li is thus the light arriving through other surfaces (indirect light); the
// lights themselves are left to next-event estimation, so the guide does not
// take their share away from it.  The network is fitted by
// minimising the weighted negative log-likelihood
//     sum_r w_r * -log q(w_r | x_r, wo_r, n_r) / sum_r w_r,   w_r = lum(Li_r) / p_r,
// a Monte Carlo estimate of the KL divergence from the normalised incident
// radiance to the mixture q (the neural importance sampling objective of
// Mueller et al., 2019), with Adam.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "guide.cuh"
#include "guide.h"
#include "guide_tc.cuh"
#include "render.h"

namespace cr
{
namespace
{
void check( cudaError_t e, const char *what )
{
	if ( e != cudaSuccess ) throw std::runtime_error( std::string( what ) + ": " + cudaGetErrorString( e ) );
}

constexpr int ROW = G_HID + 1;  // padded shared-memory row (floats): conflict-free row access
constexpr int TRAIN_ROWS = 128;


// Radiance targets of the recorded vertices and the total weight.
__global__ void k_guide_targets( GuideRecords rec, const float4 *L, uint32_t n_paths, uint32_t stride, uint32_t j0,
								 uint32_t rec_offset, uint32_t rec_stride, bool product, float *wsum )
{
	float local = 0.f;
	uint32_t n = n_paths * stride;
	for ( uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x )
	{
		float4 x = rec.x[ r ];
		if ( x.w <= 0.f ) continue;  // not a valid record
		const uint32_t path = rec_offset + ( j0 + r / stride ) * rec_stride;
		float4 Lf = L[ path ], La = rec.L[ r ], T = rec.T[ r ], om = rec.om[ r ];
		float3 li = f3( ( Lf.x - La.x ) / T.x, ( Lf.y - La.y ) / T.y, ( Lf.z - La.z ) / T.z );
		// incident radiance Li, or the product Li f cos (the integrand), per unit density
		float w = fmaxf( lum( li ), 0.f ) / om.w * ( product ? rec.wo[ r ].w : 1.f );
		if ( !isfinite( w ) || !finite3( f3( Lf ) ) ) w = 0.f;
		rec.x[ r ].w = w > 0.f ? 1.f : 0.f;
		rec.T[ r ].w = w;
		local += w;
	}
	for ( int o = 16; o; o >>= 1 ) local += __shfl_xor_sync( 0xFFFFFFFFu, local, o );
	if ( ( threadIdx.x & 31 ) == 0 && local > 0.f ) atomicAdd( wsum, local );
}

// One training pass over the valid records: forward, mixture NLL gradient,
// backward, gradients accumulated into gW / gb / ggrid.  128 records per
// block; activations live in shared memory (rows padded to 65 floats).
__global__ void __launch_bounds__( TRAIN_ROWS ) k_guide_train_fp32( GuideRecords rec, uint32_t n, GuideDev g,
																	const float *wsum, float *gW, float *gb,
																	float *ggrid, float *loss )
{
	extern __shared__ float sm[];
	float *H0 = sm;                               // inputs          [128][65]
	float *Z = H0 + TRAIN_ROWS * ROW;             // z_1..z_4       4 x [128][65]
	float *DZ = Z + 4 * TRAIN_ROWS * ROW;         // current grad    [128][65]
	const int m = threadIdx.x;
	const float norm = *wsum > 0.f ? 1.f / *wsum : 0.f;
	for ( uint32_t base = blockIdx.x * TRAIN_ROWS; base < n; base += gridDim.x * TRAIN_ROWS )
	{
		uint32_t r = base + m;
		float w = 0.f, pb = 0.f;
		float3 x = f3( 0.f, 0.f, 0.f ), wo = x, nn = x, om = x;
		if ( r < n && rec.x[ r ].w > 0.f )
		{
			const float4 n4 = rec.n[ r ];
			x = f3( rec.x[ r ] ), wo = f3( rec.wo[ r ] ), nn = f3( n4 ), om = f3( rec.om[ r ] );
			pb = n4.w;
			w = rec.T[ r ].w * norm;
		}
		float in[ G_IN ], out[ G_OUT ], acts[ 4 * G_HID ];
		guide_encode( g, x, wo, nn, in );
		guide_forward_fp32( g.W, g.b, in, out, acts );
		for ( int i = 0; i < G_IN; ++i ) H0[ m * ROW + i ] = in[ i ];
		for ( int l = 0; l < 4; ++l )
			for ( int i = 0; i < G_HID; ++i ) Z[ ( l * TRAIN_ROWS + m ) * ROW + i ] = acts[ l * G_HID + i ];
		float g_out[ G_OUT ];
		float nll = 0.f;
		if ( w > 0.f )
			nll = -w * ( g.learn_select ? mixture_nll_grad_select( out, om, pb, w, g_out )
										: mixture_nll_grad( out, om, w, g_out ) );
		else
			for ( int i = 0; i < G_OUT; ++i ) g_out[ i ] = 0.f;
		for ( int o = 16; o; o >>= 1 ) nll += __shfl_xor_sync( 0xFFFFFFFFu, nll, o );
		if ( ( m & 31 ) == 0 && nll != 0.f ) atomicAdd( loss, nll );
		for ( int i = 0; i < G_OUT; ++i ) DZ[ m * ROW + i ] = g_out[ i ];
		__syncthreads();
		for ( int l = G_LAYERS - 1; l >= 0; --l )
		{
			// input of layer l: h_l = relu(z_l) (l >= 1) or the encoding (l = 0)
			const float *Hl = l == 0 ? H0 : Z + ( l - 1 ) * TRAIN_ROWS * ROW;
			const bool relu = l > 0;
			// gW_l[o][i] += sum_m dz[m][o] h[m][i]: thread -> (o = m/2, i in half m%2)
			{
				int o = m >> 1, i0 = ( m & 1 ) * 32;
				float acc[ 32 ];
				for ( int j = 0; j < 32; ++j ) acc[ j ] = 0.f;
				for ( int mm = 0; mm < TRAIN_ROWS; ++mm )
				{
					float dz = DZ[ mm * ROW + o ];
					if ( dz == 0.f ) continue;
					const float *hr = Hl + mm * ROW + i0;
					for ( int j = 0; j < 32; ++j ) acc[ j ] = fmaf( dz, relu ? fmaxf( hr[ j ], 0.f ) : hr[ j ], acc[ j ] );
				}
				float *dst = gW + size_t( l ) * G_W + o * G_IN + i0;
				for ( int j = 0; j < 32; ++j )
					if ( acc[ j ] != 0.f ) atomicAdd( dst + j, acc[ j ] );
			}
			if ( m < G_HID )
			{
				float s = 0.f;
				for ( int mm = 0; mm < TRAIN_ROWS; ++mm ) s += DZ[ mm * ROW + m ];
				if ( s != 0.f ) atomicAdd( gb + l * G_HID + m, s );
			}
			// dh = W_l^T dz (row m), then through the ReLU of z_l
			float dh[ G_IN ];
			const float *Wl = g.W + size_t( l ) * G_W;
			for ( int i = 0; i < G_IN; ++i ) dh[ i ] = 0.f;
			for ( int o = 0; o < G_HID; ++o )
			{
				float dz = DZ[ m * ROW + o ];
				if ( dz == 0.f ) continue;
				for ( int i = 0; i < G_IN; ++i ) dh[ i ] = fmaf( Wl[ o * G_IN + i ], dz, dh[ i ] );
			}
			__syncthreads();
			if ( l > 0 )
			{
				const float *Zl = Z + ( l - 1 ) * TRAIN_ROWS * ROW + m * ROW;
				for ( int i = 0; i < G_HID; ++i ) DZ[ m * ROW + i ] = Zl[ i ] > 0.f ? dh[ i ] : 0.f;
			}
			else if ( w > 0.f )
			{
				// hash-grid features: scatter the gradient to the 8 corners per level
				float3 u = ( x - g.bmin ) * g.binv;
				for ( int lv = 0; lv < G_LEVELS; ++lv )
				{
					float d0 = dh[ 2 * lv ], d1 = dh[ 2 * lv + 1 ];
					if ( d0 == 0.f && d1 == 0.f ) continue;
					GridCorners c;
					grid_corners( lv, u, c );
					float *tab = ggrid + size_t( lv ) * G_T * G_FEAT;
					for ( int k = 0; k < 8; ++k )
					{
						atomicAdd( tab + 2 * c.idx[ k ], c.w[ k ] * d0 );
						atomicAdd( tab + 2 * c.idx[ k ] + 1, c.w[ k ] * d1 );
					}
				}
			}
			__syncthreads();
		}
	}
}

// ---------------------------------------------------------------------------
// Tensor-core training pass (tcgen05): the same gradients as k_guide_train_fp32
// with BF16 operands and FP32 accumulation.  One CTA of 128 threads takes a
// tile of 128 records at a time, one record per thread.
//   forward   z_l = W_l h_l + b_l:      A = h_l (rows x in), B = W_l (out x in)
//   backward  dh_l = W_l^T delta_l:     A = delta_l (rows x out), B = W_l^T (in x out)
//             gW_l += delta_l^T h_l:    A = delta_l^T (out x rows, padded to 128
//                                       rows of zeros), B = h_l^T (in x rows)
// gW accumulates in tensor memory over all tiles of the CTA and is added to
// global memory once at the end; bias gradients are reduced across each warp
// (lane L ends with columns 2L and 2L+1) and hash-grid gradients are scattered
// with FP32 atomics, as in the FP32 pass.
namespace tt
{
constexpr uint32_t THREADS = 128;
constexpr uint32_t H_BYTES = tc::TILE_BYTES;                // one 128 x 64 BF16 tile
constexpr uint32_t SBO128 = 16 * tc::LBO;                   // row-group stride of K = 128 tiles
constexpr uint32_t OFF_W = 0;                               // forward weight image
constexpr uint32_t OFF_WT = OFF_W + tc::WIMG_BYTES;         // transposed weight image
constexpr uint32_t OFF_H = OFF_WT + tc::WIMG_BYTES;         // h_0 .. h_4
constexpr uint32_t OFF_DZ = OFF_H + G_LAYERS * H_BYTES;     // delta (rows x out)
constexpr uint32_t OFF_DZT = OFF_DZ + H_BYTES;              // delta^T (128 x 128, rows 64.. zero)
constexpr uint32_t OFF_HT = OFF_DZT + 2 * H_BYTES;          // h^T (64 x 128)
constexpr uint32_t OFF_BIAS = OFF_HT + H_BYTES;             // 5 x 64 floats
constexpr uint32_t OFF_BAR = OFF_BIAS + G_LAYERS * G_HID * 4;
constexpr uint32_t OFF_TMEM = OFF_BAR + 8;
constexpr uint32_t SMEM_BYTES = OFF_TMEM + 8 + 128;
constexpr uint32_t TMEM_COLS = 512;                         // D (64) + gW of 5 layers (5 x 64)
constexpr uint32_t COL_DW = 64;
static_assert( SMEM_BYTES <= 232448, "training tile exceeds the shared memory of one CTA" );
static_assert( OFF_WT == OFF_W + tc::WIMG_BYTES, "weight images must be contiguous" );
}  // namespace tt

// One layer's MMAs for the whole tile, issued by thread 0 and committed to
// `bar`; every thread then waits (bounded) for the commit.  Returns false on a
// timeout (the same on every thread).
template <class Issue>
__device__ __forceinline__ bool tc_step( uint32_t tid, uint32_t bar, uint32_t &phase, Issue &&issue )
{
	tc::fence_async_smem();
	tc::tc_before_sync();
	__syncthreads();
	if ( tid == 0 )
	{
		tc::tc_after_sync();
		issue();
		tc::mma_commit( bar );
	}
	const bool ok = tc::mbar_wait( bar, phase );
	phase ^= 1u;
	if ( __syncthreads_or( !ok ) ) return false;
	tc::tc_after_sync();
	return true;
}

__device__ __forceinline__ void tmem_ld64( uint32_t taddr, float *v )
{
#pragma unroll
	for ( int c = 0; c < 4; ++c ) tc::tmem_ld16( taddr + 16u * c, v + 16 * c );
	tc::tmem_wait_ld();
}

__device__ __forceinline__ void st_bf16( uint8_t *p, float v )
{
	*reinterpret_cast<__nv_bfloat16 *>( p ) = __float2bfloat16_rn( v );
}

__global__ void __launch_bounds__( tt::THREADS, 1 ) k_guide_train_tc( GuideRecords rec, uint32_t n, GuideDev g,
																	   const uint8_t *Wp, const float *wsum, float *gW,
																	   float *gb, float *ggrid, float *loss,
																	   uint32_t *err )
{
	using namespace tt;
	extern __shared__ uint8_t smem_raw[];
	uint8_t *sm = reinterpret_cast<uint8_t *>( ( reinterpret_cast<uintptr_t>( smem_raw ) + 127 ) & ~uintptr_t( 127 ) );
	const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
	const uint32_t bar = tc::smem_u32( sm + OFF_BAR );
	uint32_t *tmem_slot = reinterpret_cast<uint32_t *>( sm + OFF_TMEM );
	float *bias = reinterpret_cast<float *>( sm + OFF_BIAS );
	{
		const uint4 *s4 = reinterpret_cast<const uint4 *>( Wp );
		uint4 *d4 = reinterpret_cast<uint4 *>( sm + OFF_W );
		for ( uint32_t i = tid; i < tc::WP_BYTES / 16; i += THREADS ) d4[ i ] = __ldg( s4 + i );
		for ( uint32_t i = tid; i < G_LAYERS * G_HID; i += THREADS ) bias[ i ] = g.b[ i ];
		// rows 64..127 of delta^T stay zero: the gW product is padded to M = 128
		uint4 *z = reinterpret_cast<uint4 *>( sm + OFF_DZT + 8 * SBO128 );
		for ( uint32_t i = tid; i < 8 * SBO128 / 16; i += THREADS ) z[ i ] = make_uint4( 0u, 0u, 0u, 0u );
	}
	if ( tid == 0 )
	{
		asm volatile( "mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"( bar ) : "memory" );
		asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
	}
	if ( warp == 0 )
	{
		asm volatile( "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"( tc::smem_u32( tmem_slot ) ),
					  "r"( TMEM_COLS )
					  : "memory" );
		asm volatile( "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory" );
	}
	tc::fence_async_smem();
	tc::tc_before_sync();
	__syncthreads();
	tc::tc_after_sync();
	const uint32_t tmem = *tmem_slot;
	const uint32_t my_lane = tmem + ( ( warp * 32u ) << 16 );  // this thread's TMEM lane (row), column 0
	const float norm = *wsum > 0.f ? 1.f / *wsum : 0.f;
	const uint32_t a_dz = tc::smem_u32( sm + OFF_DZ ), a_dzt = tc::smem_u32( sm + OFF_DZT ), a_ht = tc::smem_u32( sm + OFF_HT );
	uint32_t phase = 0;
	bool failed = false, any = false;
	float gbacc[ G_LAYERS ][ 2 ];
#pragma unroll
	for ( int l = 0; l < G_LAYERS; ++l ) gbacc[ l ][ 0 ] = gbacc[ l ][ 1 ] = 0.f;

	for ( uint32_t base = blockIdx.x * THREADS; base < n; base += gridDim.x * THREADS )
	{
		const uint32_t r = base + tid;
		float w = 0.f, pb = 0.f;
		float3 x = f3( 0.f, 0.f, 0.f ), wo = f3( 0.f, 0.f, 1.f ), nn = f3( 0.f, 0.f, 1.f ), om = f3( 0.f, 0.f, 1.f );
		if ( r < n && rec.x[ r ].w > 0.f )
		{
			const float4 n4 = rec.n[ r ];
			x = f3( rec.x[ r ] ), wo = f3( rec.wo[ r ] ), nn = f3( n4 ), om = f3( rec.om[ r ] );
			pb = n4.w;
			w = rec.T[ r ].w * norm;
		}
		float v[ G_IN ];
		if ( w > 0.f )
			guide_encode( g, x, wo, nn, v );
		else
#pragma unroll
			for ( int k = 0; k < G_IN; ++k ) v[ k ] = 0.f;
		tc::store_row( sm + OFF_H, tid, v );
		// ---- forward
		for ( int l = 0; l < G_LAYERS && !failed; ++l )
		{
			const uint32_t a_h = tc::smem_u32( sm + OFF_H + l * H_BYTES ), a_w = tc::smem_u32( sm + OFF_W + l * tc::W_BYTES );
			if ( !tc_step( tid, bar, phase, [&] {
					 for ( uint32_t k = 0; k < 4; ++k )
						 tc::mma_bf16( tmem, tc::sdesc( a_h + 256u * k ), tc::sdesc( a_w + 256u * k ), k > 0 );
				 } ) )
			{
				failed = true;
				break;
			}
			tmem_ld64( my_lane, v );
			const float *bl = bias + l * G_HID;
			if ( l < G_LAYERS - 1 )
			{
#pragma unroll
				for ( int k = 0; k < G_HID; ++k ) v[ k ] = fmaxf( v[ k ] + bl[ k ], 0.f );
				tc::store_row( sm + OFF_H + ( l + 1 ) * H_BYTES, tid, v );
			}
			else
#pragma unroll
				for ( int k = 0; k < G_OUT; ++k ) v[ k ] += bl[ k ];
			tc::tc_before_sync();
		}
		if ( failed ) break;
		// ---- loss gradient at the output
		float dz[ G_OUT ];
		float nll = 0.f;
		if ( w > 0.f )
			nll = -w * ( g.learn_select ? mixture_nll_grad_select( v, om, pb, w, dz ) : mixture_nll_grad( v, om, w, dz ) );
		else
#pragma unroll
			for ( int k = 0; k < G_OUT; ++k ) dz[ k ] = 0.f;
		for ( int o = 16; o; o >>= 1 ) nll += __shfl_xor_sync( 0xFFFFFFFFu, nll, o );
		if ( lane == 0 && nll != 0.f ) atomicAdd( loss, nll );
		// ---- backward
		for ( int l = G_LAYERS - 1; l >= 0; --l )
		{
			uint8_t *hl = sm + OFF_H + l * H_BYTES;
			// this row of h_l (BF16) for h_l^T and the ReLU mask
			uint4 hrow[ 8 ];
#pragma unroll
			for ( int j = 0; j < 8; ++j ) hrow[ j ] = *reinterpret_cast<const uint4 *>( hl + tc::canon( tid, 8 * j ) );
			const __nv_bfloat16 *hb = reinterpret_cast<const __nv_bfloat16 *>( hrow );
			tc::store_row( sm + OFF_DZ, tid, dz );
#pragma unroll
			for ( int k = 0; k < 64; ++k )
			{
				st_bf16( sm + OFF_DZT + tc::canon128( k, tid ), dz[ k ] );
				*reinterpret_cast<__nv_bfloat16 *>( sm + OFF_HT + tc::canon128( k, tid ) ) = hb[ k ];
			}
			// bias gradient: reduce-scatter of dz over the warp's 32 rows
			{
				float t[ 64 ];
#pragma unroll
				for ( int k = 0; k < 64; ++k ) t[ k ] = dz[ k ];
#pragma unroll
				for ( int h = 32, o = 16; o; h >>= 1, o >>= 1 )
				{
					const bool hi = lane & uint32_t( o );
#pragma unroll
					for ( int j = 0; j < h; ++j )
					{
						float send = hi ? t[ j ] : t[ j + h ];
						float keep = hi ? t[ j + h ] : t[ j ];
						t[ j ] = keep + __shfl_xor_sync( 0xFFFFFFFFu, send, o );
					}
				}
				gbacc[ l ][ 0 ] += t[ 0 ], gbacc[ l ][ 1 ] += t[ 1 ];
			}
			const uint32_t a_wt = tc::smem_u32( sm + OFF_WT + l * tc::W_BYTES );
			const uint32_t first = any ? 1u : 0u;
			if ( !tc_step( tid, bar, phase, [&] {
					 for ( uint32_t k = 0; k < 8; ++k )
						 tc::mma_bf16( tmem + COL_DW + 64u * l, tc::sdesc( a_dzt + 256u * k, SBO128 ),
									   tc::sdesc( a_ht + 256u * k, SBO128 ), ( k > 0 ) | first );
					 for ( uint32_t k = 0; k < 4; ++k )
						 tc::mma_bf16( tmem, tc::sdesc( a_dz + 256u * k ), tc::sdesc( a_wt + 256u * k ), k > 0 );
				 } ) )
			{
				failed = true;
				break;
			}
			float dh[ G_IN ];
			tmem_ld64( my_lane, dh );
			tc::tc_before_sync();
			if ( l > 0 )
			{
#pragma unroll
				for ( int k = 0; k < G_HID; ++k ) dz[ k ] = __bfloat162float( hb[ k ] ) > 0.f ? dh[ k ] : 0.f;
			}
			else if ( w > 0.f )
			{
				// hash-grid features: scatter the gradient to the 8 corners per level
				float3 u = ( x - g.bmin ) * g.binv;
				for ( int lv = 0; lv < G_LEVELS; ++lv )
				{
					float d0 = dh[ 2 * lv ], d1 = dh[ 2 * lv + 1 ];
					if ( d0 == 0.f && d1 == 0.f ) continue;
					GridCorners c;
					grid_corners( lv, u, c );
					float *tab = ggrid + size_t( lv ) * G_T * G_FEAT;
					for ( int k = 0; k < 8; ++k )
					{
						atomicAdd( tab + 2 * c.idx[ k ], c.w[ k ] * d0 );
						atomicAdd( tab + 2 * c.idx[ k ] + 1, c.w[ k ] * d1 );
					}
				}
			}
		}
		if ( failed ) break;
		any = true;
	}
	if ( failed )
	{
		if ( tid == 0 ) atomicOr( err, tc::ERR_MMA_TIMEOUT );
		tc::mbar_wait( bar, phase ^ 1u );  // the timed-out commit, once more (bounded)
	}
	else if ( any )
	{
		// gW rows (output units) live in TMEM lanes 0..63: warps 0 and 1
		if ( warp < 2 )
			for ( int l = 0; l < G_LAYERS; ++l )
			{
				float dw[ G_IN ];
				tmem_ld64( my_lane + COL_DW + 64u * l, dw );
				float *dst = gW + size_t( l ) * G_W + size_t( tid ) * G_IN;
				for ( int k = 0; k < G_IN; ++k )
					if ( dw[ k ] != 0.f ) atomicAdd( dst + k, dw[ k ] );
			}
#pragma unroll
		for ( int l = 0; l < G_LAYERS; ++l )
		{
			if ( gbacc[ l ][ 0 ] != 0.f ) atomicAdd( gb + l * G_HID + 2 * lane, gbacc[ l ][ 0 ] );
			if ( gbacc[ l ][ 1 ] != 0.f ) atomicAdd( gb + l * G_HID + 2 * lane + 1, gbacc[ l ][ 1 ] );
		}
	}
	tc::tc_before_sync();
	__syncthreads();
	if ( warp == 0 )
	{
		tc::tc_after_sync();
		asm volatile( "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"( tmem ), "r"( TMEM_COLS ) : "memory" );
	}
}

// Adam (Kingma and Ba 2015) on a flat parameter array; clears the gradient.
__global__ void k_adam( float *p, float *grad, float *m, float *v, uint32_t n, float lr, float b1, float b2, float eps,
						float c1, float c2 )
{
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		float gi = grad[ i ];
		if ( !isfinite( gi ) ) gi = 0.f;
		float mi = b1 * m[ i ] + ( 1.f - b1 ) * gi;
		float vi = b2 * v[ i ] + ( 1.f - b2 ) * gi * gi;
		m[ i ] = mi, v[ i ] = vi;
		p[ i ] -= lr * ( mi / c1 ) / ( sqrtf( vi / c2 ) + eps );
		grad[ i ] = 0.f;
	}
}

__global__ void k_guide_forward_batch( GuideDev g, const float *inp, uint32_t n, float *out )
{
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		const float *q = inp + 9 * size_t( i );
		float in[ G_IN ];
		guide_encode( g, f3( q[ 0 ], q[ 1 ], q[ 2 ] ), f3( q[ 3 ], q[ 4 ], q[ 5 ] ), f3( q[ 6 ], q[ 7 ], q[ 8 ] ), in );
		guide_forward_fp32( g.W, g.b, in, out + G_OUT * size_t( i ), nullptr );
	}
}

// FP32 master grid -> the inference's paired FP16 table: slot e of level l
// holds the features of slots e and e + 1 (mod G_T).
__global__ void k_pack_grid_pairs( const float *__restrict__ grid, uint2 *__restrict__ pairs )
{
	const uint32_t n = uint32_t( G_LEVELS ) * G_T;
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		const uint32_t l = i / G_T, e = i % G_T, e1 = ( e + 1 ) & uint32_t( G_T - 1 );
		const float2 a = reinterpret_cast<const float2 *>( grid )[ size_t( l ) * G_T + e ];
		const float2 b = reinterpret_cast<const float2 *>( grid )[ size_t( l ) * G_T + e1 ];
		__half2 ha = __floats2half2_rn( a.x, a.y ), hb = __floats2half2_rn( b.x, b.y );
		pairs[ i ] = make_uint2( *reinterpret_cast<uint32_t *>( &ha ), *reinterpret_cast<uint32_t *>( &hb ) );
	}
}

// FP32 master weights [G_LAYERS][64 out][64 in] -> the BF16 shared-memory
// images of the tensor-core passes: forward (layer l at l * W_BYTES, element
// (out, in) at canon(out, in)) and, after it, transposed (element (out, in) at
// canon(in, out)).
__global__ void k_pack_weights_bf16( const float *__restrict__ W, uint8_t *__restrict__ Wp )
{
	for ( uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < uint32_t( G_LAYERS * G_W ); e += gridDim.x * blockDim.x )
	{
		uint32_t l = e / G_W, o = ( e % G_W ) / G_IN, in = e % G_IN;
		const __nv_bfloat16 v = __float2bfloat16_rn( W[ e ] );
		*reinterpret_cast<__nv_bfloat16 *>( Wp + l * tc::W_BYTES + tc::canon( o, in ) ) = v;
		*reinterpret_cast<__nv_bfloat16 *>( Wp + tc::WIMG_BYTES + l * tc::W_BYTES + tc::canon( in, o ) ) = v;
	}
}

__global__ void __launch_bounds__( tc::THREADS, 2 ) k_guide_forward_batch_tc( GuideDev g, const uint8_t *Wp,
																			   const float *inp, uint32_t n,
																			   float *out, uint32_t *err )
{
	auto src = [&]( uint32_t i, float3 &x, float3 &wo, float3 &nrm ) -> bool {
		const float *q = inp + 9 * size_t( i );
		x = f3( q[ 0 ], q[ 1 ], q[ 2 ] ), wo = f3( q[ 3 ], q[ 4 ], q[ 5 ] ), nrm = f3( q[ 6 ], q[ 7 ], q[ 8 ] );
		return true;
	};
	auto sink = [&]( uint32_t i, const float *o ) {
		// out is 16-byte aligned (checked by the host) and rows are 256 bytes
		float4 *dst = reinterpret_cast<float4 *>( out + G_OUT * size_t( i ) );
		for ( int j = 0; j < G_OUT / 4; ++j ) dst[ j ] = make_float4( o[ 4 * j ], o[ 4 * j + 1 ], o[ 4 * j + 2 ], o[ 4 * j + 3 ] );
	};
	tc::mlp_forward_tc<G_OUT>( g, Wp, n, src, sink, err );
}

// Records of `stride` floats: {x, wo, n, w, weight} and, when stride is 14,
// the BSDF density of w (learned selection).
__global__ void k_records_from_host( GuideRecords rec, const float *src, uint32_t n, uint32_t stride )
{
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		const float *q = src + stride * size_t( i );
		rec.x[ i ] = make_float4( q[ 0 ], q[ 1 ], q[ 2 ], q[ 12 ] > 0.f ? 1.f : 0.f );
		rec.wo[ i ] = make_float4( q[ 3 ], q[ 4 ], q[ 5 ], 0.f );
		rec.n[ i ] = make_float4( q[ 6 ], q[ 7 ], q[ 8 ], stride > 13 ? q[ 13 ] : 0.f );
		rec.om[ i ] = make_float4( q[ 9 ], q[ 10 ], q[ 11 ], 1.f );
		rec.T[ i ] = make_float4( 1.f, 1.f, 1.f, q[ 12 ] );
		rec.L[ i ] = make_float4( 0.f, 0.f, 0.f, 0.f );
	}
}

__global__ void k_sum_weights( GuideRecords rec, uint32_t n, float *wsum )
{
	float s = 0.f;
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
		if ( rec.x[ i ].w > 0.f ) s += rec.T[ i ].w;
	for ( int o = 16; o; o >>= 1 ) s += __shfl_xor_sync( 0xFFFFFFFFu, s, o );
	if ( ( threadIdx.x & 31 ) == 0 && s != 0.f ) atomicAdd( wsum, s );
}

template <typename T>
void dalloc( T *&p, size_t n )
{
	check( cudaMalloc( (void **)&p, sizeof( T ) * std::max<size_t>( n, 1 ) ), "guide alloc" );
}

constexpr size_t TRAIN_SMEM = size_t( 6 ) * TRAIN_ROWS * ROW * sizeof( float );

}  // namespace

size_t GuideState::grid_size() { return size_t( G_LEVELS ) * G_T * G_FEAT; }
size_t GuideState::w_size() { return size_t( G_LAYERS ) * G_W; }
size_t GuideState::b_size() { return size_t( G_LAYERS ) * G_HID; }

void GuideState::init( float3 lo, float3 hi, uint64_t seed )
{
	release();
	float3 ext = make_float3( hi.x - lo.x, hi.y - lo.y, hi.z - lo.z );
	float pad = 1e-3f * std::max( ext.x, std::max( ext.y, ext.z ) ) + 1e-6f;
	bmin = make_float3( lo.x - pad, lo.y - pad, lo.z - pad );
	float e = std::max( ext.x, std::max( ext.y, ext.z ) ) + 2 * pad;  // one cube: isotropic cells
	binv = make_float3( 1.f / e, 1.f / e, 1.f / e );
	dalloc( grid, grid_size() ), dalloc( grid_m, grid_size() ), dalloc( grid_v, grid_size() ), dalloc( ggrid, grid_size() );
	dalloc( W, w_size() ), dalloc( W_m, w_size() ), dalloc( W_v, w_size() ), dalloc( gW, w_size() );
	dalloc( b, b_size() ), dalloc( b_m, b_size() ), dalloc( b_v, b_size() ), dalloc( gb, b_size() );
	dalloc( wsum, 1 ), dalloc( loss, 1 ), dalloc( err, 1 ), dalloc( err_train, 1 ), dalloc( Wp, size_t( tc::WP_BYTES ) );
	dalloc( grid_pairs, size_t( G_LEVELS ) * G_T );
	check( cudaMemset( loss, 0, 4 ), "guide init" );
	check( cudaMemset( err_train, 0, 4 ), "guide init" );
	std::mt19937_64 rng( seed );
	std::uniform_real_distribution<float> ug( -1e-4f, 1e-4f );
	std::vector<float> h( grid_size() );
	for ( auto &x : h ) x = ug( rng );
	check( cudaMemcpy( grid, h.data(), h.size() * 4, cudaMemcpyHostToDevice ), "guide init" );
	std::vector<float> w( w_size() );
	for ( int l = 0; l < G_LAYERS; ++l )
	{
		int fan_in = l == 0 ? G_USED_IN : G_HID;
		float a = std::sqrt( 6.f / float( fan_in + G_HID ) );
		std::uniform_real_distribution<float> uw( -a, a );
		for ( int o = 0; o < G_HID; ++o )
			for ( int i = 0; i < G_IN; ++i )
				w[ size_t( l ) * G_W + o * G_IN + i ] = ( l == 0 && i >= G_USED_IN ) ? 0.f : uw( rng ) * ( l == G_LAYERS - 1 ? 0.1f : 1.f );
	}
	check( cudaMemcpy( W, w.data(), w.size() * 4, cudaMemcpyHostToDevice ), "guide init" );
	for ( float *p : { grid_m, grid_v, ggrid } ) check( cudaMemset( p, 0, grid_size() * 4 ), "guide init" );
	for ( float *p : { W_m, W_v, gW } ) check( cudaMemset( p, 0, w_size() * 4 ), "guide init" );
	for ( float *p : { b, b_m, b_v, gb } ) check( cudaMemset( p, 0, b_size() * 4 ), "guide init" );
	step = 0;
	waves = 0;
	packed_step = ~0u;
	ready = true;
}

void GuideState::release()
{
	for ( float *p : { grid, grid_m, grid_v, ggrid, W, W_m, W_v, gW, b, b_m, b_v, gb, wsum, loss } )
		if ( p ) cudaFree( p );
	grid = grid_m = grid_v = ggrid = W = W_m = W_v = gW = b = b_m = b_v = gb = wsum = loss = nullptr;
	if ( Wp ) cudaFree( Wp );
	if ( grid_pairs ) cudaFree( grid_pairs );
	grid_pairs = nullptr;
	if ( err ) cudaFree( err );
	if ( err_train ) cudaFree( err_train );
	Wp = nullptr, err = nullptr, err_train = nullptr;
	if ( rec.x ) free_records();
	ready = false;
}

GuideDev GuideState::dev() const
{
	GuideDev g;
	g.grid = grid, g.grid_pairs = grid_pairs, g.W = W, g.b = b, g.bmin = bmin, g.binv = binv, g.select_prob = select_prob;
	g.guided_bounces = guided_bounces;
	g.learn_select = learn_select ? 1u : 0u;
	return g;
}

void GuideState::ensure_records( uint32_t n )
{
	if ( rec_capacity >= n ) return;
	if ( rec.x ) free_records();
	for ( float4 **p : { &rec.x, &rec.wo, &rec.n, &rec.om, &rec.T, &rec.L } ) dalloc( *p, n );
	rec_capacity = n;
}

void GuideState::free_records()
{
	for ( float4 *p : { rec.x, rec.wo, rec.n, rec.om, rec.T, rec.L } )
		if ( p ) cudaFree( p );
	rec = GuideRecords();
	rec_capacity = 0;
}

void GuideState::train_step( const float4 *L, uint32_t j0, uint32_t n_paths, uint32_t stride, uint32_t rec_offset,
							 uint32_t rec_stride, cudaStream_t st )
{
	GuideRecords r = rec;
	const size_t first = size_t( j0 ) * stride;
	for ( float4 **p : { &r.x, &r.wo, &r.n, &r.om, &r.T, &r.L } ) *p += first;
	check( cudaMemsetAsync( wsum, 0, 4, st ), "guide targets" );
	uint32_t n = n_paths * stride;
	k_guide_targets<<<std::min<uint32_t>( ( n + 255 ) / 256, 2048 ), 256, 0, st>>>( r, L, n_paths, stride, j0, rec_offset,
																				 rec_stride, product_target, wsum );
	check( cudaGetLastError(), "guide targets" );
	gradients( r, n, st, tc_train );
	adam( st );
}

void GuideState::gradients( const GuideRecords &r, uint32_t n, cudaStream_t st, bool tensor_cores )
{
	if ( tensor_cores )
	{
		ensure_smem_limit( reinterpret_cast<const void *>( k_guide_train_tc ), int( tt::SMEM_BYTES ), "guide tc train smem" );
		uint32_t blocks = std::min<uint32_t>( ( n + tt::THREADS - 1 ) / tt::THREADS, uint32_t( sm_count() ) );
		if ( blocks == 0 ) return;
		pack_weights( st );
		check( cudaMemsetAsync( loss, 0, 4, st ), "guide train" );
		k_guide_train_tc<<<blocks, tt::THREADS, tt::SMEM_BYTES, st>>>( r, n, dev(), Wp, wsum, gW, gb, ggrid, loss, err_train );
		check( cudaGetLastError(), "guide train" );
		return;
	}
	ensure_smem_limit( reinterpret_cast<const void *>( k_guide_train_fp32 ), int( TRAIN_SMEM ), "guide smem" );
	uint32_t blocks = std::min<uint32_t>( ( n + TRAIN_ROWS - 1 ) / TRAIN_ROWS, uint32_t( sm_count() ) * 2 );
	if ( blocks == 0 ) return;
	check( cudaMemsetAsync( loss, 0, 4, st ), "guide train" );
	k_guide_train_fp32<<<blocks, TRAIN_ROWS, TRAIN_SMEM, st>>>( r, n, dev(), wsum, gW, gb, ggrid, loss );
	check( cudaGetLastError(), "guide train" );
}

void GuideState::adam( cudaStream_t st )
{
	++step;
	const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
	float c1 = 1.f - std::pow( b1, float( step ) ), c2 = 1.f - std::pow( b2, float( step ) );
	auto run = [&]( float *p, float *g, float *m, float *v, size_t n, float e ) {
		k_adam<<<std::min<size_t>( ( n + 255 ) / 256, 4096 ), 256, 0, st>>>( p, g, m, v, uint32_t( n ), lr, b1, b2, e, c1, c2 );
	};
	run( W, gW, W_m, W_v, w_size(), eps );
	run( b, gb, b_m, b_v, b_size(), eps );
	run( grid, ggrid, grid_m, grid_v, grid_size(), 1e-15f );
	check( cudaGetLastError(), "guide adam" );
}

void GuideState::forward_batch( const float *d_in, uint32_t n, float *d_out, cudaStream_t st )
{
	k_guide_forward_batch<<<std::min<uint32_t>( ( n + 127 ) / 128, 4096 ), 128, 0, st>>>( dev(), d_in, n, d_out );
	check( cudaGetLastError(), "guide forward" );
}

void GuideState::pack_weights( cudaStream_t st )
{
	k_pack_weights_bf16<<<( G_LAYERS * G_W + 255 ) / 256, 256, 0, st>>>( W, Wp );
	k_pack_grid_pairs<<<1024, 256, 0, st>>>( grid, grid_pairs );
	check( cudaGetLastError(), "guide weight packing" );
}

uint32_t GuideState::forward_batch_tc( const float *d_in, uint32_t n, float *d_out, cudaStream_t st )
{
	if ( reinterpret_cast<uintptr_t>( d_out ) % 16 ) throw std::runtime_error( "guide forward: output not 16-byte aligned" );
	ensure_smem_limit( reinterpret_cast<const void *>( k_guide_forward_batch_tc ), int( tc::SMEM_BYTES ), "guide tc smem" );
	check( cudaMemsetAsync( err, 0, 4, st ), "guide forward" );
	pack_weights( st );
	uint32_t blocks = std::min<uint32_t>( ( n + tc::THREADS - 1 ) / tc::THREADS, uint32_t( sm_count() ) * 2 );
	if ( blocks )
		k_guide_forward_batch_tc<<<blocks, tc::THREADS, tc::SMEM_BYTES, st>>>( dev(), Wp, d_in, n, d_out, err );
	check( cudaGetLastError(), "guide forward" );
	uint32_t e = 0;
	check( cudaMemcpyAsync( &e, err, 4, cudaMemcpyDeviceToHost, st ), "guide forward" );
	check( cudaStreamSynchronize( st ), "guide forward" );
	return e;
}

void GuideState::load_records( const float *d_src, uint32_t n, uint32_t stride, cudaStream_t st )
{
	ensure_records( n );
	k_records_from_host<<<std::min<uint32_t>( ( n + 255 ) / 256, 4096 ), 256, 0, st>>>( rec, d_src, n, stride );
	check( cudaMemsetAsync( wsum, 0, 4, st ), "guide records" );
	k_sum_weights<<<std::min<uint32_t>( ( n + 255 ) / 256, 1024 ), 256, 0, st>>>( rec, n, wsum );
	check( cudaGetLastError(), "guide records" );
}

}  // namespace cr
