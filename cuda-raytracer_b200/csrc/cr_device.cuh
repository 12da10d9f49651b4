// Device code shared by the traversal, shading and parity kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_common.h"

namespace cr
{
// ------------------------------------------------------------------ float3 math
__device__ __forceinline__ float3 f3( float x, float y, float z ) { return make_float3( x, y, z ); }
__device__ __forceinline__ float3 f3( const float *p ) { return make_float3( p[ 0 ], p[ 1 ], p[ 2 ] ); }
__device__ __forceinline__ float3 f3( float4 a ) { return make_float3( a.x, a.y, a.z ); }
__device__ __forceinline__ float3 operator+( float3 a, float3 b ) { return f3( a.x + b.x, a.y + b.y, a.z + b.z ); }
__device__ __forceinline__ float3 operator-( float3 a, float3 b ) { return f3( a.x - b.x, a.y - b.y, a.z - b.z ); }
__device__ __forceinline__ float3 operator-( float3 a ) { return f3( -a.x, -a.y, -a.z ); }
__device__ __forceinline__ float3 operator*( float3 a, float3 b ) { return f3( a.x * b.x, a.y * b.y, a.z * b.z ); }
__device__ __forceinline__ float3 operator*( float3 a, float s ) { return f3( a.x * s, a.y * s, a.z * s ); }
__device__ __forceinline__ float3 operator*( float s, float3 a ) { return f3( a.x * s, a.y * s, a.z * s ); }
__device__ __forceinline__ float3 operator/( float3 a, float s ) { return f3( a.x / s, a.y / s, a.z / s ); }
__device__ __forceinline__ float dot( float3 a, float3 b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross( float3 a, float3 b )
{
	return f3( a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y );
}
__device__ __forceinline__ float length( float3 a ) { return sqrtf( dot( a, a ) ); }
__device__ __forceinline__ float3 normalize( float3 a ) { return a * ( 1.0f / sqrtf( dot( a, a ) ) ); }
__device__ __forceinline__ float maxc( float3 a ) { return fmaxf( a.x, fmaxf( a.y, a.z ) ); }
__device__ __forceinline__ bool finite3( float3 a ) { return isfinite( a.x ) && isfinite( a.y ) && isfinite( a.z ); }
__device__ __forceinline__ bool is_zero( float3 a ) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
__device__ __forceinline__ float comp( float3 a, int k ) { return k == 0 ? a.x : ( k == 1 ? a.y : a.z ); }

constexpr float PI_F = 3.14159265358979323846f;

// ------------------------------------------------------------------ Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64 multiplies
// with the published round multipliers and Weyl key increments.
__device__ __forceinline__ uint4 philox4x32_10( uint4 c, uint2 k )
{
	const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
	for ( int r = 0; r < 10; ++r )
	{
		uint32_t hi0 = __umulhi( M0, c.x ), lo0 = M0 * c.x;
		uint32_t hi1 = __umulhi( M1, c.z ), lo1 = M1 * c.z;
		c = make_uint4( hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0 );
		k.x += W0;
		k.y += W1;
	}
	return c;
}

// Uniform in (0, 1): 24 random bits, centred in their interval so that 0 and 1
// never occur (the Beckmann sampler takes log(u)).
__device__ __forceinline__ float u01( uint32_t x ) { return ( float( x >> 8 ) + 0.5f ) * ( 1.0f / 16777216.0f ); }

// Four uniforms for (sample id, bounce, stream) under the render's key.
__device__ __forceinline__ float4 rand4( uint2 key, uint64_t sample, uint32_t bounce, uint32_t stream )
{
	uint4 r = philox4x32_10( make_uint4( uint32_t( sample ), uint32_t( sample >> 32 ), bounce, stream ), key );
	return make_float4( u01( r.x ), u01( r.y ), u01( r.z ), u01( r.w ) );
}

// ------------------------------------------------------------------ traversal
struct RayPre
{
	float3 o, d, invd;
	uint32_t oct;
	int kx, ky, kz;
	float sx, sy, sz;
};

__device__ __forceinline__ RayPre make_ray( float3 o, float3 d )
{
	RayPre r;
	r.o = o;
	r.d = d;
	const float tiny = 1e-30f;
	float dx = fabsf( d.x ) < tiny ? copysignf( tiny, d.x ) : d.x;
	float dy = fabsf( d.y ) < tiny ? copysignf( tiny, d.y ) : d.y;
	float dz = fabsf( d.z ) < tiny ? copysignf( tiny, d.z ) : d.z;
	r.invd = f3( 1.0f / dx, 1.0f / dy, 1.0f / dz );
	r.oct = ( d.x < 0.f ? 1u : 0u ) | ( d.y < 0.f ? 2u : 0u ) | ( d.z < 0.f ? 4u : 0u );
	// Watertight ray/triangle set-up (Woop, Benthin and Wald, JCGT 2013):
	// kz = dominant axis, winding preserved by swapping kx/ky when d[kz] < 0.
	float ax = fabsf( d.x ), ay = fabsf( d.y ), az = fabsf( d.z );
	int kz = ( ax >= ay && ax >= az ) ? 0 : ( ay >= az ? 1 : 2 );
	int kx = kz == 2 ? 0 : kz + 1;
	int ky = kx == 2 ? 0 : kx + 1;
	if ( comp( d, kz ) < 0.f )
	{
		int t = kx;
		kx = ky;
		ky = t;
	}
	r.kx = kx, r.ky = ky, r.kz = kz;
	float dkz = comp( d, kz );
	r.sx = comp( d, kx ) / dkz;
	r.sy = comp( d, ky ) / dkz;
	r.sz = 1.0f / dkz;
	return r;
}

// Watertight ray/triangle test; accepts tmin < t < tmax, edges inclusive,
// no back-face culling.  Returns u, v = weights of v1 and v2.
__device__ __forceinline__ bool tri_test( const RayPre &r, float3 v0, float3 v1, float3 v2, float tmin, float tmax,
										  float &t, float &u, float &v )
{
	float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
	float Akz = comp( A, r.kz ), Bkz = comp( B, r.kz ), Ckz = comp( C, r.kz );
	float Ax = fmaf( -r.sx, Akz, comp( A, r.kx ) ), Ay = fmaf( -r.sy, Akz, comp( A, r.ky ) );
	float Bx = fmaf( -r.sx, Bkz, comp( B, r.kx ) ), By = fmaf( -r.sy, Bkz, comp( B, r.ky ) );
	float Cx = fmaf( -r.sx, Ckz, comp( C, r.kx ) ), Cy = fmaf( -r.sy, Ckz, comp( C, r.ky ) );
	float U = Cx * By - Cy * Bx;
	float V = Ax * Cy - Ay * Cx;
	float W = Bx * Ay - By * Ax;
	if ( U == 0.f || V == 0.f || W == 0.f )
	{
		// Exact fallback on an edge, as the watertight method prescribes.
		U = float( double( Cx ) * double( By ) - double( Cy ) * double( Bx ) );
		V = float( double( Ax ) * double( Cy ) - double( Ay ) * double( Cx ) );
		W = float( double( Bx ) * double( Ay ) - double( By ) * double( Ax ) );
	}
	if ( ( U < 0.f || V < 0.f || W < 0.f ) && ( U > 0.f || V > 0.f || W > 0.f ) ) return false;
	float det = U + V + W;
	if ( det == 0.f ) return false;
	float T = U * ( r.sz * Akz ) + V * ( r.sz * Bkz ) + W * ( r.sz * Ckz );
	float sdet = fabsf( det );
	float sT = det < 0.f ? -T : T;
	if ( !( sT > tmin * sdet ) || !( sT < tmax * sdet ) ) return false;
	float rcp = 1.0f / det;
	t = T * rcp;
	u = V * rcp;
	v = W * rcp;
	return true;
}

// Sphere::intersect (reference src/core/primitive/sphere.hpp:31-54): near
// root, else far root, accepted when t >= 0 and within (tmin, tmax).
// The roots are formed without the reference's cancellation-prone
// |oc|^2 - (d.oc)^2: the squared distance of the centre from the ray line is
// taken from the perpendicular vector itself, and the smaller-magnitude root
// comes from the product of the roots (c / q), as in Haines et al.,
// "Precision Improvements for Ray/Sphere Intersection" (Ray Tracing Gems, 2019).
__device__ __forceinline__ bool sphere_test( float3 centre, float r2, float3 o, float3 d, float tmin, float tmax,
											 float &t )
{
	float3 oc = centre - o;
	float poc = dot( d, oc );
	float3 perp = oc - d * poc;
	float det = r2 - dot( perp, perp );
	if ( det < 0.f ) return false;
	float q = poc + copysignf( sqrtf( det ), poc );  // root of larger magnitude
	float c = dot( oc, oc ) - r2;
	float r0 = q != 0.f ? c / q : 0.f, r1 = q;
	float t_near = fminf( r0, r1 ), t_far = fmaxf( r0, r1 );
	t = t_near < 0.f ? t_far : t_near;
	return t >= 0.f && t > tmin && t < tmax;
}


// ------------------------------------------------------------------ shading helpers
// Reference frame (src/core/meta/scene.hpp:48-53): u = n x (0,1,0), v = n x u,
// both normalised (NaN when n is parallel to +-y, as in the reference).
struct Frame
{
	float3 u, v, n;
	__device__ float3 local( float3 w ) const { return normalize( f3( dot( w, u ), dot( w, v ), dot( w, n ) ) ); }
	__device__ float3 global( float3 w ) const { return normalize( u * w.x + v * w.y + n * w.z ); }
};

__device__ __forceinline__ Frame koishi_frame( float3 n )
{
	Frame f;
	f.n = n;
	f.u = normalize( f3( -n.z, 0.f, n.x ) );
	f.v = normalize( cross( n, f.u ) );
	return f;
}

// Orthonormal basis of Duff et al., "Building an Orthonormal Basis, Revisited"
// (JCGT 2017).
__device__ __forceinline__ Frame onb_frame( float3 n )
{
	Frame f;
	f.n = n;
	float sign = copysignf( 1.0f, n.z );
	float a = -1.0f / ( sign + n.z );
	float b = n.x * n.y * a;
	f.u = f3( 1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x );
	f.v = f3( b, sign + n.y * n.y * a, -n.y );
	return f;
}

// H::sampleCos (src/util/hemisphere.hpp:76-95): concentric disk mapping.
__device__ __forceinline__ float3 sample_cos( float r1, float r2 )
{
	float ux = 2.f * r1 - 1.f, uy = 2.f * r2 - 1.f;
	if ( ux == 0.f && uy == 0.f ) return f3( 0.f, 0.f, 1.f );
	float r, phi;
	if ( ux * ux > uy * uy )
		r = ux, phi = ( PI_F / 4.f ) * ( uy / ux );
	else
		r = uy, phi = ( PI_F / 2.f ) - ( PI_F / 4.f ) * ( ux / uy );
	float s, c;
	sincosf( phi, &s, &c );
	return f3( r * c, r * s, sqrtf( fmaxf( 0.f, 1.f - r * r ) ) );
}

// BeckmannDistribution::f (src/ext/distribution/beckmann.hpp:19-24): D(h)|cos|.
__device__ __forceinline__ float beckmann_f( float alpha2, float3 w )
{
	float c2 = w.z * w.z;
	float s2 = fmaxf( 0.f, 1.f - c2 );
	float tg2 = s2 / c2;
	return expf( -tg2 / alpha2 ) / ( PI_F * alpha2 * c2 * c2 ) * fabsf( w.z );
}

// BeckmannDistribution::sample (src/ext/distribution/beckmann.hpp:26-38).
__device__ __forceinline__ float3 beckmann_sample( float alpha2, float u1, float u2 )
{
	float tg2 = -alpha2 * logf( u1 );
	float phi = u2 * 2.f * PI_F;
	float costh = 1.f / sqrtf( 1.f + tg2 );
	float sinth = sqrtf( fmaxf( 0.f, 1.f - costh * costh ) );
	float s, c;
	sincosf( phi, &s, &c );
	return f3( sinth * s, sinth * c, costh );
}

__device__ __forceinline__ float3 reflect( float3 I, float3 N ) { return N * ( dot( N, I ) * 2.f ) - I; }

// Uniform stream of one path vertex, served in the order the reference's
// Sampler serves RadianceKernel::execute (radiance.cu:29-68) and the shaders
// it runs: Philox blocks (sample, bounce, 0), (sample, bounce, 1), ... drawn
// four at a time as they are consumed.
struct VertexRng
{
	uint2 key;
	uint64_t g;
	uint32_t bounce, blk;
	float4 b;
	int i;
	// b0: block 0, already drawn; start: draws of it already taken
	__device__ __forceinline__ VertexRng( uint2 k, uint64_t s, uint32_t bn, float4 b0, int start )
		: key( k ), g( s ), bounce( bn ), blk( 1 ), b( b0 ), i( start )
	{
	}
	__device__ __forceinline__ float next()
	{
		if ( i == 4 ) b = rand4( key, g, bounce, blk++ ), i = 0;
		const float v = i == 0 ? b.x : i == 1 ? b.y : i == 2 ? b.z : b.w;
		++i;
		return v;
	}
};

// Uniforms read from an array (n per sample) in the order they are drawn;
// draws past the end read 0.5 and are still counted.
struct ArrayRng
{
	const float *u;
	uint32_t n, used;
	__device__ __forceinline__ float next()
	{
		const float v = used < n ? u[ used ] : 0.5f;
		++used;
		return v;
	}
};

// SphericalDistribution::f of a shader's distribution: Beckmann D(h)|cos|
// (beckmann.hpp:19-24) or the cosine lobe (cosine.hpp:14-17).
__device__ __forceinline__ float dist_f( const DevShader &sh, float3 w )
{
	if ( sh.dist == DIST_COSINE ) return w.z >= 0.f ? 1.0f / PI_F : 0.f;
	return beckmann_f( sh.alpha2, w );
}

// distribution->sample( sampler.sample3() ): three draws, the first two used
// (beckmann.hpp:26-38, cosine.hpp:18-23).
template <class Rng>
__device__ __forceinline__ float3 dist_sample( const DevShader &sh, Rng &rng )
{
	const float u1 = rng.next(), u2 = rng.next();
	rng.next();
	return sh.dist == DIST_COSINE ? sample_cos( u1, u2 ) : beckmann_sample( sh.alpha2, u1, u2 );
}

// The Fresnel scala (src/ext/scala/fresnel.hpp:17-31): unpolarised dielectric
// reflectance for the outgoing direction, 1 past the critical angle.
__device__ __forceinline__ float fresnel_fac( float ior, float3 wo )
{
	const float eta = wo.z > 0.f ? 1.f / ior : ior;
	const float ci = fabsf( wo.z );
	const float st = eta * sqrtf( fmaxf( 0.f, 1.f - ci * ci ) );
	if ( st >= 1.f ) return 1.f;
	const float q = ci / sqrtf( fmaxf( 0.f, 1.f - st * st ) );
	const float a = ( q - eta ) / ( q + eta ), b = ( eta * q - 1.f ) / ( eta * q + 1.f );
	return .5f * ( a * a + b * b );
}

// refract (src/vec/vmath.hpp:517-526): I refracted about N with relative
// index eta; false (R untouched) past the critical angle.
__device__ __forceinline__ bool refract_dir( float3 I, float3 N, float eta, float3 &R )
{
	const float c = dot( N, I );
	const float s2 = fmaxf( 0.f, 1.f - c * c ) * eta * eta;
	if ( s2 >= 1.f ) return false;
	R = normalize( -I * eta + N * ( eta * c - sqrtf( 1.f - s2 ) ) );
	return true;
}

// Walks the Mixed shaders from table entry idx to the leaf that executes:
// each Mixed draws one number and runs shaders[1] below its fac, else
// shaders[0] (mixed.hpp:24-29).  The host bounds the depth.
template <class Rng>
__device__ __forceinline__ int koishi_leaf( const DevShader *tab, int idx, float3 wo, Rng &rng )
{
	for ( int d = 0; d < MAX_SHADER_DEPTH && tab[ idx ].type == SH_MIXED; ++d )
	{
		const DevShader &m = tab[ idx ];
		const float f = m.fac_kind == FAC_FRESNEL ? fresnel_fac( m.ior, wo ) : m.fac;
		idx = m.child[ rng.next() < f ? 1 : 0 ];
	}
	return idx;
}

// compute_f_by_wi_wo of a shader that draws no selection number (all but
// Mixed and GlassBSDF): Lambert (lambert.hpp:31-33), GlossyBSDF
// (glossy.hpp:27-29), Emission as white Lambert that also sets the varyings'
// emission (emission.hpp:22-27), and zero for Transparent
// (transparent.hpp:24-26), Blackhole (blackhole.hpp:17-20) and
// RefractionBSDF (refraction.hpp:35-38).
__device__ __forceinline__ float3 leaf_eval( const DevShader &sh, float3 wo, float3 wi, float3 &emission )
{
	emission = sh.type == SH_EMISSION ? f3( sh.emission ) : f3( 0.f, 0.f, 0.f );
	switch ( sh.type )
	{
	case SH_LAMBERT:
	case SH_EMISSION:
		return wi.z >= 0.f ? f3( sh.albedo ) * ( 1.0f / PI_F ) : f3( 0.f, 0.f, 0.f );
	case SH_GLOSSY:
		return f3( sh.color ) * dist_f( sh, normalize( wo + wi ) );
	default:
		return f3( 0.f, 0.f, 0.f );
	}
}

// The transmission half of RefractionBSDF and GlassBSDF (refraction.hpp:24-33,
// glass.hpp:40-49) for a half-vector h from the distribution: flipped to wo's
// side, it refracts wo; f = color scaled by 1/eta^2 when entering.  wi is
// left as it was when the refraction fails (f = 0).
__device__ __forceinline__ float3 koishi_refract( const DevShader &sh, float3 wo, float3 h, float3 &wi )
{
	const float eta = wo.z > 0.f ? 1.f / sh.ior : sh.ior;
	if ( wo.z < 0.f ) h = -h;
	if ( !refract_dir( wo, h, eta, wi ) ) return f3( 0.f, 0.f, 0.f );
	return f3( sh.color ) / ( eta < 1.f ? eta * eta : 1.f );
}

// sample_wi_f_by_wo of a shader that draws no selection number, given the
// first two numbers (u1, u2) of its sampler.sample3() (Transparent and
// Blackhole draw none): Lambert (lambert.hpp:26-30 with cosine.hpp:18-23:
// f = color * R), GlossyBSDF (glossy.hpp:22-26), Transparent (wi = -wo,
// f = color), Blackhole (wi = +z, f = 0), RefractionBSDF.  Returns f; the
// caller multiplies by |cos|.  wi is in/out (see koishi_refract); emission is
// what the shader writes to the varyings (Emission only).
__device__ __forceinline__ float3 leaf_sample( const DevShader &sh, float3 wo, float u1, float u2, float3 &wi,
											   float3 &emission )
{
	emission = sh.type == SH_EMISSION ? f3( sh.emission ) : f3( 0.f, 0.f, 0.f );
	switch ( sh.type )
	{
	case SH_LAMBERT:
	case SH_EMISSION:
		wi = sample_cos( u1, u2 );
		return wi.z >= 0.f ? f3( sh.albedo ) : f3( 0.f, 0.f, 0.f );
	case SH_GLOSSY:
		wi = reflect( wo, sh.dist == DIST_COSINE ? sample_cos( u1, u2 ) : beckmann_sample( sh.alpha2, u1, u2 ) );
		return wo.z * wi.z > 0.f ? f3( sh.color ) : f3( 0.f, 0.f, 0.f );
	case SH_TRANSPARENT:
		wi = -wo;
		return f3( sh.color );
	case SH_REFRACTION:
		return koishi_refract( sh, wo, sh.dist == DIST_COSINE ? sample_cos( u1, u2 ) : beckmann_sample( sh.alpha2, u1, u2 ),
							   wi );
	default:  // Blackhole
		wi = f3( 0.f, 0.f, 1.f );
		return f3( 0.f, 0.f, 0.f );
	}
}

// Whether a shader draws numbers in its sample_wi_f_by_wo (sampler.sample3()).
__device__ __forceinline__ bool samples_draw( int type ) { return type != SH_TRANSPARENT && type != SH_BLACKHOLE; }

// Koishi estimator, compute_f_by_wi_wo of table entry idx with the draws the
// reference makes: one per Mixed on the way to the leaf, and GlassBSDF's
// Fresnel draw picking the reflection or the transmission half-vector
// (glass.hpp:25-53).
template <class Rng>
__device__ __forceinline__ float3 koishi_eval( const DevShader *tab, int idx, float3 wo, float3 wi, Rng &rng,
											   float3 &emission )
{
	const DevShader &sh = tab[ koishi_leaf( tab, idx, wo, rng ) ];
	if ( sh.type != SH_GLASS ) return leaf_eval( sh, wo, wi, emission );
	emission = f3( 0.f, 0.f, 0.f );
	if ( rng.next() < fresnel_fac( sh.ior, wo ) ) return f3( sh.color ) * dist_f( sh, normalize( wo + wi ) );
	return f3( sh.color ) * dist_f( sh, normalize( wo + wi * sh.ior ) );
}

// Koishi estimator, sample_wi_f_by_wo of table entry idx with the draws the
// reference makes (Mixed selections, GlassBSDF's Fresnel draw, then the
// shader's sampler.sample3()).
template <class Rng>
__device__ __forceinline__ float3 koishi_sample( const DevShader *tab, int idx, float3 wo, Rng &rng, float3 &wi,
												 float3 &emission )
{
	const DevShader &sh = tab[ koishi_leaf( tab, idx, wo, rng ) ];
	if ( sh.type == SH_GLASS )
	{
		emission = f3( 0.f, 0.f, 0.f );
		const bool refl = rng.next() < fresnel_fac( sh.ior, wo );
		const float3 h = dist_sample( sh, rng );
		if ( !refl ) return koishi_refract( sh, wo, h, wi );
		wi = reflect( wo, h );
		return wo.z * wi.z > 0.f ? f3( sh.color ) : f3( 0.f, 0.f, 0.f );
	}
	float u1 = 0.5f, u2 = 0.5f;
	if ( samples_draw( sh.type ) )
	{
		u1 = rng.next(), u2 = rng.next();
		rng.next();
	}
	return leaf_sample( sh, wo, u1, u2, wi, emission );
}

// MIS estimator BSDFs: Lambert albedo/pi with cosine pdf; Beckmann microfacet
// reflection color*D*G/(4 cos_o cos_i) with the Smith G1 rational fit of
// Walter et al. (EGSR 2007) and pdf D cos_h / (4 |wo.h|).
__device__ __forceinline__ float smith_g1( float alpha, float3 w )
{
	float c = w.z;
	if ( c <= 0.f ) return 0.f;
	float s = sqrtf( fmaxf( 0.f, 1.f - c * c ) );
	if ( s == 0.f ) return 1.f;
	float a = c / ( alpha * s );
	if ( a >= 1.6f ) return 1.f;
	return ( 3.535f * a + 2.181f * a * a ) / ( 1.f + 2.276f * a + 2.577f * a * a );
}

// Beckmann D(h) with tan^2 from the tangential components, which keeps FP32
// accuracy for half-vectors near the normal (1 - cos^2 cancels there).
__device__ __forceinline__ float beckmann_d( float alpha2, float3 h )
{
	float c2 = h.z * h.z;
	float tg2 = ( h.x * h.x + h.y * h.y ) / c2;
	return expf( -tg2 / alpha2 ) / ( PI_F * alpha2 * c2 * c2 );
}

__device__ __forceinline__ float3 mis_eval( const DevShader &sh, float3 wo, float3 wi, float &pdf )
{
	pdf = 0.f;
	if ( wo.z <= 0.f || wi.z <= 0.f ) return f3( 0.f, 0.f, 0.f );
	if ( sh.type == SH_GLOSSY )
	{
		float3 h = normalize( wo + wi );
		float dh = beckmann_d( sh.alpha2, h );
		float G = smith_g1( sh.alpha, wo ) * smith_g1( sh.alpha, wi );
		pdf = dh * h.z / ( 4.f * fabsf( dot( wo, h ) ) );
		return f3( sh.color ) * ( dh * G / ( 4.f * wo.z * wi.z ) );
	}
	pdf = wi.z * ( 1.0f / PI_F );
	return f3( sh.albedo ) * ( 1.0f / PI_F );
}

// Returns the sample weight f*cos/pdf (zero when the sample is rejected).
// For the Beckmann lobe D cancels: weight = color * G * |wo.h| / (cos_o cos_h).
__device__ __forceinline__ float3 mis_sample( const DevShader &sh, float3 wo, float u1, float u2, float3 &wi, float &pdf )
{
	pdf = 0.f;
	if ( sh.type == SH_GLOSSY )
	{
		float3 h = beckmann_sample( sh.alpha2, u1, u2 );
		wi = reflect( wo, h );
		float woh = dot( wo, h );
		if ( wo.z <= 0.f || wi.z <= 0.f || woh <= 0.f ) return f3( 0.f, 0.f, 0.f );
		float G = smith_g1( sh.alpha, wo ) * smith_g1( sh.alpha, wi );
		pdf = beckmann_d( sh.alpha2, h ) * h.z / ( 4.f * woh );
		return f3( sh.color ) * ( G * woh / ( wo.z * h.z ) );
	}
	wi = sample_cos( u1, u2 );
	if ( wo.z <= 0.f || wi.z <= 0.f ) return f3( 0.f, 0.f, 0.f );
	pdf = wi.z * ( 1.0f / PI_F );
	return f3( sh.albedo );
}

// The MIS estimator's remaining shaders, physically restated (the reference's
// versions are the koishi_* functions): RefractionBSDF and GlassBSDF as the
// rough dielectric of Walter et al. ("Microfacet Models for Refraction through
// Rough Surfaces", EGSR 2007) with a Beckmann distribution (Refraction: its
// transmission alone), Transparent as a delta pass-through, Blackhole black,
// Mixed as the fac-weighted mixture of two such leaves.  wo.z > 0 (the frame
// faces the incoming ray); `entering`: wo lies outside the surface as built,
// which sets the dielectric's index on either side.

// Smith G1 of direction v for microfacet normal h, either side of the surface.
__device__ __forceinline__ float smith_g1h( float alpha, float3 v, float3 h )
{
	if ( dot( v, h ) * v.z <= 0.f ) return 0.f;
	return smith_g1( alpha, f3( v.x, v.y, fabsf( v.z ) ) );
}

// Unpolarised Fresnel reflectance of a dielectric interface for cos_o > 0 on
// the side of index 1 and relative index eta of the other side.
__device__ __forceinline__ float fresnel_dielectric( float cos_o, float eta )
{
	const float s2 = ( 1.f - cos_o * cos_o ) / ( eta * eta );
	if ( s2 >= 1.f ) return 1.f;
	const float ct = sqrtf( 1.f - s2 );
	const float rs = ( cos_o - eta * ct ) / ( cos_o + eta * ct ), rp = ( eta * cos_o - ct ) / ( eta * cos_o + ct );
	return .5f * ( rs * rs + rp * rp );
}

__device__ __forceinline__ bool mis_transmits( int type )
{
	return type == SH_GLASS || type == SH_REFRACTION || type == SH_TRANSPARENT;
}

// f and pdf of a rough dielectric leaf for wi on either side.
__device__ __forceinline__ float3 dielectric_eval( const DevShader &sh, float3 wo, float3 wi, bool entering, float &pdf )
{
	pdf = 0.f;
	const float eo = entering ? 1.f : sh.ior, et = entering ? sh.ior : 1.f;
	if ( wi.z > 0.f )
	{
		if ( sh.type == SH_REFRACTION ) return f3( 0.f, 0.f, 0.f );
		const float3 h = normalize( wo + wi );
		const float F = fresnel_dielectric( dot( wo, h ), et / eo );
		const float D = beckmann_d( sh.alpha2, h );
		const float G = smith_g1h( sh.alpha, wo, h ) * smith_g1h( sh.alpha, wi, h );
		pdf = F * D * h.z / ( 4.f * fabsf( dot( wo, h ) ) );
		return f3( sh.color ) * ( F * D * G / ( 4.f * wo.z * wi.z ) );
	}
	if ( !( wi.z < 0.f ) ) return f3( 0.f, 0.f, 0.f );
	float3 h = normalize( -( wo * eo + wi * et ) );
	if ( h.z < 0.f ) h = -h;
	const float co = dot( wo, h ), ci = dot( wi, h );
	if ( co <= 0.f || ci >= 0.f ) return f3( 0.f, 0.f, 0.f );
	const float F = sh.type == SH_GLASS ? fresnel_dielectric( co, et / eo ) : 0.f;
	const float D = beckmann_d( sh.alpha2, h );
	const float G = smith_g1h( sh.alpha, wo, h ) * smith_g1h( sh.alpha, wi, h );
	const float den = et * ci + eo * co;
	pdf = ( 1.f - F ) * D * h.z * et * et * fabsf( ci ) / ( den * den );
	return f3( sh.color ) * ( ( 1.f - F ) * D * G * fabsf( ci ) * co * eo * eo / ( fabsf( wi.z ) * wo.z * den * den ) );
}

// f and pdf of any leaf (not Mixed) for the MIS estimator.
__device__ __forceinline__ float3 mis_eval_leaf( const DevShader &sh, float3 wo, float3 wi, bool entering, float &pdf )
{
	pdf = 0.f;
	if ( wo.z <= 0.f ) return f3( 0.f, 0.f, 0.f );
	switch ( sh.type )
	{
	case SH_LAMBERT:
	case SH_EMISSION:
	case SH_GLOSSY:
		return mis_eval( sh, wo, wi, pdf );
	case SH_GLASS:
	case SH_REFRACTION:
		return dielectric_eval( sh, wo, wi, entering, pdf );
	default:  // Transparent (delta), Blackhole
		return f3( 0.f, 0.f, 0.f );
	}
}

// Mixed's fac: the Constant, or the Fresnel scala with the reference's side
// convention (fresnel.hpp:17-31: the cosine of wo against the surface as built).
__device__ __forceinline__ float mis_fac( const DevShader &m, float3 wo, bool entering )
{
	if ( m.fac_kind != FAC_FRESNEL ) return fminf( 1.f, fmaxf( 0.f, m.fac ) );
	return fresnel_fac( m.ior, f3( wo.x, wo.y, entering ? wo.z : -wo.z ) );
}

// f and pdf of table entry idx: a leaf, or a Mixed of two leaves.
__device__ __forceinline__ float3 mis_eval_tab( const DevShader *tab, int idx, float3 wo, float3 wi, bool entering,
												float &pdf )
{
	const DevShader &sh = tab[ idx ];
	if ( sh.type != SH_MIXED ) return mis_eval_leaf( sh, wo, wi, entering, pdf );
	const float F = mis_fac( sh, wo, entering );
	float pa, pb;
	const float3 fa = mis_eval_leaf( tab[ sh.child[ 0 ] ], wo, wi, entering, pa );
	const float3 fb = mis_eval_leaf( tab[ sh.child[ 1 ] ], wo, wi, entering, pb );
	pdf = ( 1.f - F ) * pa + F * pb;
	return fa * ( 1.f - F ) + fb * F;
}

// Sampled direction of a leaf (u_sel picks a dielectric's reflection); false
// when it yields none.  Transparent's is the delta direction -wo.
__device__ __forceinline__ bool mis_sample_dir_leaf( const DevShader &sh, float3 wo, bool entering, float u_sel, float u1,
													 float u2, float3 &wi )
{
	if ( wo.z <= 0.f ) return false;
	switch ( sh.type )
	{
	case SH_TRANSPARENT:
		wi = -wo;
		return true;
	case SH_GLOSSY:
	{
		const float3 h = beckmann_sample( sh.alpha2, u1, u2 );
		wi = reflect( wo, h );
		return wi.z > 0.f && dot( wo, h ) > 0.f;
	}
	case SH_GLASS:
	case SH_REFRACTION:
	{
		const float eo = entering ? 1.f : sh.ior, et = entering ? sh.ior : 1.f;
		const float3 h = beckmann_sample( sh.alpha2, u1, u2 );
		const float co = dot( wo, h );
		if ( co <= 0.f ) return false;
		const float F = sh.type == SH_GLASS ? fresnel_dielectric( co, et / eo ) : 0.f;
		if ( u_sel < F )
		{
			wi = reflect( wo, h );
			return wi.z > 0.f;
		}
		if ( !refract_dir( wo, h, eo / et, wi ) ) return false;
		return wi.z < 0.f;
	}
	case SH_LAMBERT:
	case SH_EMISSION:
		wi = sample_cos( u1, u2 );
		return wi.z > 0.f;
	default:  // Blackhole
		return false;
	}
}

// Sample of table entry idx: returns the weight f|cos|/pdf with wi and pdf;
// `delta` for Transparent's pass-through (weight = color, no density).
__device__ __forceinline__ float3 mis_sample_tab( const DevShader *tab, int idx, float3 wo, bool entering, float u_sel,
												  float u1, float u2, float3 &wi, float &pdf, bool &delta )
{
	pdf = 0.f, delta = false;
	const DevShader *leaf = &tab[ idx ];
	if ( leaf->type == SH_MIXED )
	{
		const float F = mis_fac( *leaf, wo, entering );
		const bool b = u_sel < F;
		u_sel = b ? u_sel / F : ( u_sel - F ) / ( 1.f - F );
		leaf = &tab[ leaf->child[ b ? 1 : 0 ] ];
	}
	if ( !mis_sample_dir_leaf( *leaf, wo, entering, u_sel, u1, u2, wi ) ) return f3( 0.f, 0.f, 0.f );
	if ( leaf->type == SH_TRANSPARENT )
	{
		delta = true;
		return f3( leaf->color );
	}
	const float3 f = mis_eval_tab( tab, idx, wo, wi, entering, pdf );
	return pdf > 0.f ? f * ( fabsf( wi.z ) / pdf ) : f3( 0.f, 0.f, 0.f );
}

// Spawn point offset off a surface along its geometric normal by an amount
// that scales with the point's magnitude (Waechter and Binder, "A Fast and
// Robust Method for Avoiding Self-Intersection", Ray Tracing Gems 2019).
__device__ __forceinline__ float3 offset_ray( float3 p, float3 n )
{
	const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
	int3 of_i = make_int3( int( int_scale * n.x ), int( int_scale * n.y ), int( int_scale * n.z ) );
	float3 p_i = f3( __int_as_float( __float_as_int( p.x ) + ( p.x < 0 ? -of_i.x : of_i.x ) ),
					 __int_as_float( __float_as_int( p.y ) + ( p.y < 0 ? -of_i.y : of_i.y ) ),
					 __int_as_float( __float_as_int( p.z ) + ( p.z < 0 ? -of_i.z : of_i.z ) ) );
	return f3( fabsf( p.x ) < origin ? p.x + float_scale * n.x : p_i.x,
			   fabsf( p.y ) < origin ? p.y + float_scale * n.y : p_i.y,
			   fabsf( p.z ) < origin ? p.z + float_scale * n.z : p_i.z );
}

}  // namespace cr
