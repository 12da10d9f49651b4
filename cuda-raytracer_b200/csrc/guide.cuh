// Learned path guiding: device math shared by the inference, training and
// shading kernels.
//
// Network: position x (12-level multiresolution hash grid, 2 features per
// level, trilinear), outgoing direction wo (real spherical harmonics up to
// degree 3, 16 terms) and the shading normal n go in; four hidden layers of
// width 64 (ReLU); the output holds 8 von Mises-Fisher lobes (mean direction,
// concentration, weight).  The distribution proposes incident directions at
// a path vertex and is mixed with BSDF sampling by one-sample MIS.
#pragma once
#include "cr_device.cuh"

namespace cr
{
constexpr int G_LEVELS = 12, G_FEAT = 2, G_LOG2T = 16, G_T = 1 << G_LOG2T;
constexpr int G_IN = 64, G_HID = 64, G_OUT = 64, G_LAYERS = 5, G_LOBES = 8;
constexpr int G_ENC = G_LEVELS * G_FEAT;           // 24 hash features
constexpr int G_SH = 16;                           // SH terms (l = 0..3)
constexpr int G_USED_IN = G_ENC + G_SH + 3;        // 43 (the rest of the 64 inputs are zero)
constexpr int G_W = G_HID * G_IN;                  // weights per layer (all 64 x 64)
constexpr float G_KAPPA_MIN = 0.05f, G_KAPPA_MAX = 5000.f;
// Learned selection: output G_SEL_OUT is the logit of the probability of
// sampling the guide rather than the BSDF at a vertex, clamped to
// [G_SEL_MIN, G_SEL_MAX] so that both strategies keep some samples.
constexpr int G_SEL_OUT = 40;
constexpr float G_SEL_MIN = 0.02f, G_SEL_MAX = 0.98f;

struct GuideDev
{
	const float *grid;   // [G_LEVELS][G_T][G_FEAT], FP32 master
	// [G_LEVELS][G_T]: FP16 features of slot e and of slot e + 1 (mod G_T; its
	// +x neighbour), 8 bytes, for the inference's paired gathers
	const uint2 *grid_pairs;
	const float *W;      // [G_LAYERS][64 out][64 in], FP32 master weights
	const float *b;      // [G_LAYERS][64] biases
	float3 bmin, binv;   // scene box: x -> (x - bmin) * binv in [0,1]^3
	float select_prob;   // probability of sampling the guide at a vertex (fixed selection)
	uint32_t guided_bounces;  // vertices 0 .. guided_bounces-1 sample the guide (0: all)
	uint32_t learn_select;    // 1: the network's output G_SEL_OUT gives the probability per vertex
};

// Whether vertex `bounce` of a path of at most max_bounce + 1 vertices
// samples the guide: the guide shapes continuations only, so never the last
// vertex, and only the first guided_bounces vertices when that is set.
__host__ __device__ __forceinline__ bool guided_vertex( const GuideDev &g, uint32_t bounce, uint32_t max_bounce )
{
	return bounce < max_bounce && ( g.guided_bounces == 0 || bounce < g.guided_bounces );
}

// Luminance (Rec. 709 weights): the scalar the guide's training weights use.
__host__ __device__ __forceinline__ float lum( float3 c ) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// Resolution of level l: 4 * 1.5^l cells per axis (4 .. 346).
__host__ __device__ __forceinline__ float grid_res( int l )
{
	float r = 4.f;
	for ( int i = 0; i < l; ++i ) r *= 1.5f;
	return floorf( r );
}

// Table slot of an integer lattice point: coarse levels whose lattice fits the
// table are indexed directly; finer ones hash y and z with the xor-of-primes
// hash of Teschner et al. (2003) and add x, so that on every level the +x
// neighbour of a point lives in the next slot (mod the table size).  The
// inference gathers both x-corners of a cell with one load from a table
// whose entries are stored paired with their next slot's (guide_tc.cuh).
__host__ __device__ __forceinline__ uint32_t grid_index( int l, uint32_t ix, uint32_t iy, uint32_t iz )
{
	uint32_t res = uint32_t( grid_res( l ) ) + 1u;
	uint64_t dense = uint64_t( res ) * res * res;
	if ( dense <= uint64_t( G_T ) ) return ix + res * ( iy + res * iz );
	return ( ix + ( iy * 2654435761u ^ iz * 805459861u ) ) & uint32_t( G_T - 1 );
}

// Real spherical harmonics of bands l = 0..3 of a unit vector (16 terms,
// "degree 4" when counting bands), orthonormal basis.
__host__ __device__ __forceinline__ void sh16( float x, float y, float z, float *o )
{
	const float c0 = 0.28209479177387814f, c1 = 0.4886025119029199f;
	const float c2a = 1.0925484305920792f, c2b = 0.31539156525252005f, c2c = 0.5462742152960396f;
	const float c3a = 0.5900435899266435f, c3b = 2.890611442640554f, c3c = 0.4570457994644658f;
	const float c3d = 0.3731763325901154f, c3e = 1.445305721320277f;
	float xx = x * x, yy = y * y, zz = z * z;
	o[ 0 ] = c0;
	o[ 1 ] = -c1 * y, o[ 2 ] = c1 * z, o[ 3 ] = -c1 * x;
	o[ 4 ] = c2a * x * y, o[ 5 ] = -c2a * y * z, o[ 6 ] = c2b * ( 3.f * zz - 1.f ), o[ 7 ] = -c2a * x * z;
	o[ 8 ] = c2c * ( xx - yy );
	o[ 9 ] = -c3a * y * ( 3.f * xx - yy ), o[ 10 ] = c3b * x * y * z, o[ 11 ] = -c3c * y * ( 5.f * zz - 1.f );
	o[ 12 ] = c3d * z * ( 5.f * zz - 3.f ), o[ 13 ] = -c3c * x * ( 5.f * zz - 1.f );
	o[ 14 ] = c3e * z * ( xx - yy ), o[ 15 ] = -c3a * x * ( xx - 3.f * yy );
}

// Trilinear corners of level l at normalised position u in [0,1]^3.
struct GridCorners
{
	uint32_t idx[ 8 ];
	float w[ 8 ];
};

__device__ __forceinline__ void grid_corners( int l, float3 u, GridCorners &c )
{
	float res = grid_res( l );
	float px = fminf( fmaxf( u.x, 0.f ), 1.f ) * res, py = fminf( fmaxf( u.y, 0.f ), 1.f ) * res,
		  pz = fminf( fmaxf( u.z, 0.f ), 1.f ) * res;
	float fx = floorf( px ), fy = floorf( py ), fz = floorf( pz );
	uint32_t ix = uint32_t( fx ), iy = uint32_t( fy ), iz = uint32_t( fz );
	float tx = px - fx, ty = py - fy, tz = pz - fz;
#pragma unroll
	for ( int k = 0; k < 8; ++k )
	{
		uint32_t dx = k & 1, dy = ( k >> 1 ) & 1, dz = ( k >> 2 ) & 1;
		c.idx[ k ] = grid_index( l, ix + dx, iy + dy, iz + dz );
		c.w[ k ] = ( dx ? tx : 1.f - tx ) * ( dy ? ty : 1.f - ty ) * ( dz ? tz : 1.f - tz );
	}
}

// Network input for (x, wo, n): 24 hash features, 16 SH terms of wo, n, zeros.
__device__ __forceinline__ void guide_encode( const GuideDev &g, float3 x, float3 wo, float3 n, float *in )
{
	float3 u = ( x - g.bmin ) * g.binv;
#pragma unroll
	for ( int l = 0; l < G_LEVELS; ++l )
	{
		GridCorners c;
		grid_corners( l, u, c );
		float f0 = 0.f, f1 = 0.f;
		const float *tab = g.grid + size_t( l ) * G_T * G_FEAT;
#pragma unroll
		for ( int k = 0; k < 8; ++k )
		{
			float2 v = *reinterpret_cast<const float2 *>( tab + 2 * c.idx[ k ] );
			f0 += c.w[ k ] * v.x;
			f1 += c.w[ k ] * v.y;
		}
		in[ 2 * l ] = f0, in[ 2 * l + 1 ] = f1;
	}
	sh16( wo.x, wo.y, wo.z, in + G_ENC );
	in[ G_ENC + G_SH ] = n.x, in[ G_ENC + G_SH + 1 ] = n.y, in[ G_ENC + G_SH + 2 ] = n.z;
	for ( int i = G_USED_IN; i < G_IN; ++i ) in[ i ] = 0.f;
}

// ------------------------------------------------------------------ vMF mixture
struct Lobe
{
	float3 mu;
	float kappa, weight;
};

__host__ __device__ __forceinline__ float softplusf( float x ) { return x > 20.f ? x : log1pf( expf( x ) ); }

// Output layer (first 40 of 64) to lobes: mean = normalize(o[0..2]),
// kappa = softplus(o[3]) clamped, weight = softmax over o[4] of all lobes.
__device__ __forceinline__ void lobes_from_output( const float *o, Lobe *lb )
{
	float mx = -INFINITY;
	for ( int k = 0; k < G_LOBES; ++k ) mx = fmaxf( mx, o[ 5 * k + 4 ] );
	float sum = 0.f;
	for ( int k = 0; k < G_LOBES; ++k )
	{
		float3 m = f3( o[ 5 * k ], o[ 5 * k + 1 ], o[ 5 * k + 2 ] );
		float l2 = dot( m, m );
		lb[ k ].mu = l2 > 1e-20f ? m * rsqrtf( l2 ) : f3( 0.f, 0.f, 1.f );
		lb[ k ].kappa = fminf( fmaxf( softplusf( o[ 5 * k + 3 ] ), G_KAPPA_MIN ), G_KAPPA_MAX );
		lb[ k ].weight = expf( o[ 5 * k + 4 ] - mx );
		sum += lb[ k ].weight;
	}
	for ( int k = 0; k < G_LOBES; ++k ) lb[ k ].weight /= sum;
}

// The learned probability of sampling the guide: sigmoid of the selection
// logit, clamped; `free` reports whether the clamp left it alone.
__host__ __device__ __forceinline__ float guide_selection( const float *o, bool *free = nullptr )
{
	const float raw = 1.f / ( 1.f + expf( -o[ G_SEL_OUT ] ) );
	if ( free ) *free = raw > G_SEL_MIN && raw < G_SEL_MAX;
	return fminf( fmaxf( raw, G_SEL_MIN ), G_SEL_MAX );
}

// vMF density on the sphere: kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu.w - 1)).
__device__ __forceinline__ float vmf_pdf( const Lobe &l, float3 w )
{
	float norm = l.kappa / ( 2.f * PI_F * ( -expm1f( -2.f * l.kappa ) ) );
	return norm * expf( l.kappa * ( dot( l.mu, w ) - 1.f ) );
}

__device__ __forceinline__ float mixture_pdf( const Lobe *lb, float3 w )
{
	float p = 0.f;
	for ( int k = 0; k < G_LOBES; ++k ) p += lb[ k ].weight * vmf_pdf( lb[ k ], w );
	return p;
}

// A mixture prepared for repeated evaluation at one vertex: per lobe the mean,
// the weight, kappa log2(e) and log2(weight * vMF normaliser), so that the
// density costs one exp2 per lobe.
struct PreparedLobe
{
	float3 mu;
	float weight, k2, c;
};

__device__ __forceinline__ void prepare_lobe( const Lobe &l, PreparedLobe &p )
{
	const float norm = l.kappa / ( 2.f * PI_F * ( -expm1f( -2.f * l.kappa ) ) );
	p.mu = l.mu, p.weight = l.weight;
	p.k2 = l.kappa * 1.4426950408889634f;
	p.c = log2f( l.weight * norm );  // -inf for a lobe of weight 0
}

// mixture_pdf of the prepared lobes.
__device__ __forceinline__ float prepared_pdf( const PreparedLobe *lb, float3 w )
{
	float p = 0.f;
#pragma unroll
	for ( int k = 0; k < G_LOBES; ++k ) p += exp2f( fmaf( lb[ k ].k2, dot( lb[ k ].mu, w ) - 1.f, lb[ k ].c ) );
	return p;
}

// Sample the mixture: lobe by weight (u0), then a vMF direction with the
// numerically stable inversion of Jakob ("Numerically stable sampling of the
// von Mises Fisher distribution on S2", 2012).
__device__ __forceinline__ float3 mixture_sample( const PreparedLobe *lb, float u0, float u1, float u2 )
{
	int k = 0;
	float acc = 0.f;
	for ( ; k < G_LOBES - 1; ++k )
	{
		acc += lb[ k ].weight;
		if ( u0 < acc ) break;
	}
	const PreparedLobe &l = lb[ k ];
	const float kappa = l.k2 * 0.6931471805599453f;
	float w = 1.f + logf( u1 + ( 1.f - u1 ) * expf( -2.f * kappa ) ) / kappa;
	w = fminf( fmaxf( w, -1.f ), 1.f );
	float r = sqrtf( fmaxf( 0.f, 1.f - w * w ) ), s, c;
	sincosf( 2.f * PI_F * u2, &s, &c );
	Frame f = onb_frame( l.mu );
	return normalize( f.u * ( r * c ) + f.v * ( r * s ) + f.n * w );
}

}  // namespace cr

namespace cr
{
// FP32 forward pass of one sample: h0 = in, h_{l+1} = relu(W_l h_l + b_l) for
// l < 4, out = W_4 h_4 + b_4.  `acts` (optional) receives h_1..h_4 pre-ReLU
// values z_1..z_4 (4 x 64) for the backward pass.
__device__ __forceinline__ void guide_forward_fp32( const float *__restrict__ W, const float *__restrict__ b,
													const float *in, float *out, float *acts )
{
	float h[ G_HID ], z[ G_HID ];
	for ( int i = 0; i < G_IN; ++i ) h[ i ] = in[ i ];
	for ( int l = 0; l < G_LAYERS; ++l )
	{
		const float *Wl = W + size_t( l ) * G_W;
		for ( int o = 0; o < G_HID; ++o )
		{
			float acc = b[ l * G_HID + o ];
			for ( int i = 0; i < G_IN; ++i ) acc = fmaf( Wl[ o * G_IN + i ], h[ i ], acc );
			z[ o ] = acc;
		}
		if ( l == G_LAYERS - 1 )
			for ( int o = 0; o < G_OUT; ++o ) out[ o ] = z[ o ];
		else
		{
			if ( acts )
				for ( int o = 0; o < G_HID; ++o ) acts[ l * G_HID + o ] = z[ o ];
			for ( int o = 0; o < G_HID; ++o ) h[ o ] = fmaxf( z[ o ], 0.f );
		}
	}
}

// Gradient of -log q(w) with respect to the 40 used outputs, times `scale`;
// returns log q(w).  The lobes' log densities and their responsibilities are
// formed in log space (log-sum-exp), so a direction far from every lobe, whose
// vMF densities all underflow in FP32 at large kappa, still gets its gradient.
__device__ __forceinline__ float mixture_nll_grad( const float *o, float3 w, float scale, float *g )
{
	Lobe lb[ G_LOBES ];
	lobes_from_output( o, lb );
	float lv[ G_LOBES ], mx = -INFINITY;
	for ( int k = 0; k < G_LOBES; ++k )
	{
		const float kap = lb[ k ].kappa;
		// log(weight * kappa / (2 pi (1 - exp(-2 kappa)))) + kappa (mu.w - 1)
		lv[ k ] = logf( lb[ k ].weight ) + logf( kap / ( 2.f * PI_F ) ) - log1pf( -expf( -2.f * kap ) ) +
				  kap * ( dot( lb[ k ].mu, w ) - 1.f );
		mx = fmaxf( mx, lv[ k ] );
	}
	float sum = 0.f;
	for ( int k = 0; k < G_LOBES; ++k ) sum += expf( lv[ k ] - mx );
	const float logq = mx + logf( sum );
	for ( int i = 0; i < G_OUT; ++i ) g[ i ] = 0.f;
	for ( int k = 0; k < G_LOBES; ++k )
	{
		float gam = expf( lv[ k ] - logq );  // responsibility
		// weight logits: pi_k - gamma_k
		g[ 5 * k + 4 ] = scale * ( lb[ k ].weight - gam );
		// concentration: d log v / d kappa = 1/kappa - 2/(e^{2 kappa} - 1) + mu.w - 1
		float kap = lb[ k ].kappa, raw = o[ 5 * k + 3 ];
		float sp = softplusf( raw );
		bool clamped = sp < G_KAPPA_MIN || sp > G_KAPPA_MAX;
		float dlogv = 1.f / kap - 2.f / expm1f( 2.f * kap ) + dot( lb[ k ].mu, w ) - 1.f;
		float sig = 1.f / ( 1.f + expf( -raw ) );
		g[ 5 * k + 3 ] = clamped ? 0.f : -scale * gam * dlogv * sig;
		// mean: d v / d m = v kappa (w - mu (mu.w)) / |m|
		float3 m = f3( o[ 5 * k ], o[ 5 * k + 1 ], o[ 5 * k + 2 ] );
		float len = sqrtf( fmaxf( dot( m, m ), 1e-20f ) );
		float3 dm = ( w - lb[ k ].mu * dot( lb[ k ].mu, w ) ) * ( -scale * gam * kap / len );
		g[ 5 * k ] = dm.x, g[ 5 * k + 1 ] = dm.y, g[ 5 * k + 2 ] = dm.z;
	}
	return logq;
}

// Learned selection: gradient of -log m, m = s q(w) + (1 - s) pb, the density
// of the one-sample MIS of guide (probability s) and BSDF (density pb) that
// the renderer samples with, times `scale`; returns log m (in log space too).
// The lobe outputs get the plain NLL gradient times the guide's share
// s q / m; the selection logit gets -(q - pb) / m s (1 - s).
__device__ __forceinline__ float mixture_nll_grad_select( const float *o, float3 w, float pb, float scale, float *g )
{
	const float logq = mixture_nll_grad( o, w, scale, g );
	bool free;
	const float s = guide_selection( o, &free );
	const float a = logf( s ) + logq;                                   // log(s q)
	const float c = pb > 0.f ? logf( 1.f - s ) + logf( pb ) : -INFINITY;  // log((1 - s) pb)
	const float mx = fmaxf( a, c );
	const float logm = mx + logf( expf( a - mx ) + expf( c - mx ) );
	const float r = expf( a - logm );  // the guide's share s q / m
	for ( int i = 0; i < 5 * G_LOBES; ++i ) g[ i ] *= r;
	// -(q - pb) / m * s (1 - s) = -((1 - s) r - s (1 - r)) with (1 - s) pb / m = 1 - r
	g[ G_SEL_OUT ] = free ? -scale * ( ( 1.f - s ) * r - s * ( 1.f - r ) ) : 0.f;
	return logm;
}
}  // namespace cr
