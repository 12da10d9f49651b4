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
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "guide.cuh"
#include "guide.h"
#include "guide_tc.cuh"

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
		float w = 0.f;
		float3 x = f3( 0.f, 0.f, 0.f ), wo = x, nn = x, om = x;
		if ( r < n && rec.x[ r ].w > 0.f )
		{
			x = f3( rec.x[ r ] ), wo = f3( rec.wo[ r ] ), nn = f3( rec.n[ r ] ), om = f3( rec.om[ r ] );
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
			nll = -w * logf( mixture_nll_grad( out, om, w, g_out ) );
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

// FP32 master weights [G_LAYERS][64 out][64 in] -> the BF16 shared-memory image
// of the tensor-core forward (layer l at l * W_BYTES, element (out, in) at
// canon(out, in)).
__global__ void k_pack_weights_bf16( const float *__restrict__ W, uint8_t *__restrict__ Wp )
{
	for ( uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < uint32_t( G_LAYERS * G_W ); e += gridDim.x * blockDim.x )
	{
		uint32_t l = e / G_W, o = ( e % G_W ) / G_IN, in = e % G_IN;
		*reinterpret_cast<__nv_bfloat16 *>( Wp + l * tc::W_BYTES + tc::canon( o, in ) ) = __float2bfloat16_rn( W[ e ] );
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
	tc::mlp_forward_tc( g, Wp, n, src, sink, err );
}

__global__ void k_records_from_host( GuideRecords rec, const float *src, uint32_t n )
{
	for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
	{
		const float *q = src + 13 * size_t( i );
		rec.x[ i ] = make_float4( q[ 0 ], q[ 1 ], q[ 2 ], q[ 12 ] > 0.f ? 1.f : 0.f );
		rec.wo[ i ] = make_float4( q[ 3 ], q[ 4 ], q[ 5 ], 0.f );
		rec.n[ i ] = make_float4( q[ 6 ], q[ 7 ], q[ 8 ], 0.f );
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
	dalloc( wsum, 1 ), dalloc( loss, 1 ), dalloc( err, 1 ), dalloc( Wp, size_t( tc::W_BYTES ) * G_LAYERS );
	check( cudaMemset( loss, 0, 4 ), "guide init" );
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
	ready = true;
}

void GuideState::release()
{
	for ( float *p : { grid, grid_m, grid_v, ggrid, W, W_m, W_v, gW, b, b_m, b_v, gb, wsum, loss } )
		if ( p ) cudaFree( p );
	grid = grid_m = grid_v = ggrid = W = W_m = W_v = gW = b = b_m = b_v = gb = wsum = loss = nullptr;
	if ( Wp ) cudaFree( Wp );
	if ( err ) cudaFree( err );
	Wp = nullptr, err = nullptr;
	if ( rec.x ) free_records();
	ready = false;
}

GuideDev GuideState::dev() const
{
	GuideDev g;
	g.grid = grid, g.W = W, g.b = b, g.bmin = bmin, g.binv = binv, g.select_prob = select_prob;
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
	gradients( r, n, st );
	adam( st );
}

void GuideState::gradients( const GuideRecords &r, uint32_t n, cudaStream_t st )
{
	static bool attr = false;
	if ( !attr )
	{
		check( cudaFuncSetAttribute( k_guide_train_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, int( TRAIN_SMEM ) ),
			   "guide smem" );
		attr = true;
	}
	uint32_t blocks = std::min<uint32_t>( ( n + TRAIN_ROWS - 1 ) / TRAIN_ROWS, 148 * 2 );
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
	check( cudaGetLastError(), "guide weight packing" );
}

uint32_t GuideState::forward_batch_tc( const float *d_in, uint32_t n, float *d_out, cudaStream_t st )
{
	if ( reinterpret_cast<uintptr_t>( d_out ) % 16 ) throw std::runtime_error( "guide forward: output not 16-byte aligned" );
	static bool attr = false;
	if ( !attr )
	{
		check( cudaFuncSetAttribute( k_guide_forward_batch_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
									 int( tc::SMEM_BYTES ) ),
			   "guide tc smem" );
		attr = true;
	}
	check( cudaMemsetAsync( err, 0, 4, st ), "guide forward" );
	pack_weights( st );
	int device = 0, sms = 0;
	check( cudaGetDevice( &device ), "device" );
	check( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, device ), "device" );
	uint32_t blocks = std::min<uint32_t>( ( n + tc::THREADS - 1 ) / tc::THREADS, uint32_t( sms ) * 2 );
	if ( blocks )
		k_guide_forward_batch_tc<<<blocks, tc::THREADS, tc::SMEM_BYTES, st>>>( dev(), Wp, d_in, n, d_out, err );
	check( cudaGetLastError(), "guide forward" );
	uint32_t e = 0;
	check( cudaMemcpyAsync( &e, err, 4, cudaMemcpyDeviceToHost, st ), "guide forward" );
	check( cudaStreamSynchronize( st ), "guide forward" );
	return e;
}

void GuideState::load_records( const float *d_src, uint32_t n, cudaStream_t st )
{
	ensure_records( n );
	k_records_from_host<<<std::min<uint32_t>( ( n + 255 ) / 256, 4096 ), 256, 0, st>>>( rec, d_src, n );
	check( cudaMemsetAsync( wsum, 0, 4, st ), "guide records" );
	k_sum_weights<<<std::min<uint32_t>( ( n + 255 ) / 256, 1024 ), 256, 0, st>>>( rec, n, wsum );
	check( cudaGetLastError(), "guide records" );
}

}  // namespace cr
