// FP64 CPU oracle for the Radiance path of xlnx/cuda-raytracer.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h): the checker the CUDA path is
// compared with.  Every function cites the reference file:line it restates;
// ORC_MIS functions restate the corrected estimator documented in oracle.h.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace
{
constexpr double PI = 3.14159265358979323846;
constexpr double INF = std::numeric_limits<double>::infinity();

struct V3
{
	double x = 0, y = 0, z = 0;
	V3() = default;
	V3( double a, double b, double c ) : x( a ), y( b ), z( c ) {}
	double operator[]( int i ) const { return i == 0 ? x : i == 1 ? y : z; }
	double &operator[]( int i ) { return i == 0 ? x : i == 1 ? y : z; }
};
inline V3 operator+( V3 a, V3 b ) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline V3 operator-( V3 a, V3 b ) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline V3 operator-( V3 a ) { return { -a.x, -a.y, -a.z }; }
inline V3 operator*( V3 a, V3 b ) { return { a.x * b.x, a.y * b.y, a.z * b.z }; }
inline V3 operator*( V3 a, double s ) { return { a.x * s, a.y * s, a.z * s }; }
inline V3 operator*( double s, V3 a ) { return a * s; }
inline V3 operator/( V3 a, double s ) { return { a.x / s, a.y / s, a.z / s }; }
inline double dot( V3 a, V3 b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross( V3 a, V3 b ) { return { a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y }; }
inline double length( V3 a ) { return std::sqrt( dot( a, a ) ); }
inline V3 normalize( V3 a ) { return a * ( 1.0 / std::sqrt( dot( a, a ) ) ); }
inline V3 vmin( V3 a, V3 b ) { return { std::min( a.x, b.x ), std::min( a.y, b.y ), std::min( a.z, b.z ) }; }
inline V3 vmax( V3 a, V3 b ) { return { std::max( a.x, b.x ), std::max( a.y, b.y ), std::max( a.z, b.z ) }; }
inline double maxc( V3 a ) { return std::max( a.x, std::max( a.y, a.z ) ); }
inline bool finite3( V3 a ) { return std::isfinite( a.x ) && std::isfinite( a.y ) && std::isfinite( a.z ); }

// float3 helpers used where the reference computes a stored table in float.
struct F3
{
	float x, y, z;
};
inline F3 fadd( F3 a, F3 b ) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
inline F3 fsub( F3 a, F3 b ) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
inline F3 fmul( F3 a, float s ) { return { a.x * s, a.y * s, a.z * s }; }
inline F3 fcross( F3 a, F3 b ) { return { a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y }; }
inline F3 fnormalize( F3 a )
{
	float r = 1.0f / std::sqrt( a.x * a.x + a.y * a.y + a.z * a.z );
	return fmul( a, r );
}

struct Shader
{
	int type;
	V3 R{ 1, 1, 1 }, color{ 1, 1, 1 };
	double alpha = 0.5;  // Beckmann roughness (alpha2 = roughness^2, beckmann.hpp:11-17)
	V3 emission;         // color * strength (emission.hpp:12-20)
	int dist = ORC_DIST_BECKMANN;       // Glossy, Refraction, Glass distribution
	double ior = 1;                     // Refraction, Glass, Mixed with a Fresnel fac
	int fac_kind = ORC_FAC_CONSTANT;    // Mixed
	double fac = 0;                     // Mixed with a Constant fac
	int child[ 2 ] = { -1, -1 };        // Mixed: shaders[0], shaders[1]
};

struct Tri
{
	V3 v0, v1, v2, n0, n1, n2;
	F3 fv0, fv1, fv2, fn0, fn1, fn2;
	int prim, index;
};

struct Prim
{
	int kind;  // 0 mesh, 1 sphere
	int shader;
	int first_tri = 0, n_tri = 0;
	V3 c;
	double r = 0;
	float fc[ 3 ] = { 0, 0, 0 }, fr = 0;
	int light = -1;
};

struct Light
{
	int prim = -1;
	int kind;  // 0 mesh, 1 sphere, 2 point (pointLight.hpp)
	V3 pos, emission;  // point lights
	// ORC_KOISHI mesh table (mesh.hpp:61-84)
	std::vector<F3> tp, tn;
	float kpdf = 0;
	// ORC_MIS area sampling
	std::vector<double> cdf;
	double area = 0;
};

struct Node
{
	V3 lo, hi;
	int left = -1, right = -1, first = 0, count = 0;
};

struct Camera
{
	V3 pos{ 1, 0, 0 }, target{ -1, 0, 0 }, up{ 0, 0, 1 };
	float fpos[ 3 ] = { 1, 0, 0 }, ftarget[ 3 ] = { -1, 0, 0 }, fup[ 3 ] = { 0, 0, 1 };
	double fovx = 90;
	int lens = 0;  // CameraConfig::lens: 0 pinhole, 1 orthographic
};

struct Hit
{
	double t = INF, u = 0, v = 0;
	int tri = -1;   // global triangle (tris[]) or -1
	int prim = -1;  // prim index
	V3 sphere_n;
};

// Splitmix64-based per-sample stream (oracle-only randomness).
struct Rng
{
	uint64_t s;
	static uint64_t mix( uint64_t z )
	{
		z += 0x9E3779B97F4A7C15ull;
		z = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
		z = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
		return z ^ ( z >> 31 );
	}
	Rng( uint64_t seed, uint64_t a, uint64_t b ) : s( mix( seed ^ mix( a * 0x100000001B3ull + b ) ) ) {}
	double next()
	{
		s = mix( s );
		return double( s >> 11 ) * ( 1.0 / 9007199254740992.0 );
	}
};

}  // namespace

struct orc_scene
{
	std::vector<Shader> shaders;
	std::vector<Prim> prims;
	std::vector<Tri> tris;
	std::vector<int> bvh_tris;
	std::vector<Node> nodes;
	std::vector<Light> lights;
	std::vector<Light> point_lights;  // pointLight assets, in asset order
	Camera cam;
	double scale = 1;
};

namespace
{
// ---------------------------------------------------------------- BVH (speed only)
void build_bvh( orc_scene *s )
{
	s->bvh_tris.resize( s->tris.size() );
	for ( size_t i = 0; i < s->tris.size(); ++i ) s->bvh_tris[ i ] = int( i );
	s->nodes.clear();
	if ( s->tris.empty() ) return;
	std::vector<V3> cen( s->tris.size() );
	for ( size_t i = 0; i < s->tris.size(); ++i )
		cen[ i ] = ( s->tris[ i ].v0 + s->tris[ i ].v1 + s->tris[ i ].v2 ) / 3.0;
	struct Task
	{
		int node, first, count;
	};
	std::vector<Task> stack;
	s->nodes.push_back( Node() );
	stack.push_back( { 0, 0, int( s->tris.size() ) } );
	while ( !stack.empty() )
	{
		Task t = stack.back();
		stack.pop_back();
		V3 lo( INF, INF, INF ), hi( -INF, -INF, -INF ), clo = lo, chi = hi;
		for ( int i = t.first; i < t.first + t.count; ++i )
		{
			const Tri &tr = s->tris[ s->bvh_tris[ i ] ];
			lo = vmin( lo, vmin( tr.v0, vmin( tr.v1, tr.v2 ) ) );
			hi = vmax( hi, vmax( tr.v0, vmax( tr.v1, tr.v2 ) ) );
			clo = vmin( clo, cen[ s->bvh_tris[ i ] ] );
			chi = vmax( chi, cen[ s->bvh_tris[ i ] ] );
		}
		s->nodes[ t.node ].lo = lo;
		s->nodes[ t.node ].hi = hi;
		V3 e = chi - clo;
		int axis = e.x >= e.y && e.x >= e.z ? 0 : e.y >= e.z ? 1 : 2;
		if ( t.count <= 4 || e[ axis ] <= 0 )
		{
			s->nodes[ t.node ].first = t.first;
			s->nodes[ t.node ].count = t.count;
			continue;
		}
		int mid = t.first + t.count / 2;
		std::nth_element( s->bvh_tris.begin() + t.first, s->bvh_tris.begin() + mid,
						  s->bvh_tris.begin() + t.first + t.count,
						  [&]( int a, int b ) { return cen[ a ][ axis ] < cen[ b ][ axis ]; } );
		int l = int( s->nodes.size() );
		s->nodes.push_back( Node() );
		s->nodes.push_back( Node() );
		s->nodes[ t.node ].left = l;
		s->nodes[ t.node ].right = l + 1;
		stack.push_back( { l, t.first, mid - t.first } );
		stack.push_back( { l + 1, mid, t.first + t.count - mid } );
	}
}

inline bool box_hit( const Node &n, V3 o, V3 inv, double tmax )
{
	double t0 = 0, t1 = tmax;
	for ( int a = 0; a < 3; ++a )
	{
		double ta = ( n.lo[ a ] - o[ a ] ) * inv[ a ], tb = ( n.hi[ a ] - o[ a ] ) * inv[ a ];
		if ( ta > tb ) std::swap( ta, tb );
		if ( std::isnan( ta ) || std::isnan( tb ) ) continue;
		t0 = std::max( t0, ta );
		t1 = std::min( t1, tb );
	}
	return t0 <= t1 * ( 1 + 1e-9 ) + 1e-12;
}

// Moller-Trumbore as in Ray::intersect_triangle (src/core/basic/ray.hpp:37-52):
// t > 0, u >= 0, v >= 0, u + v <= 1, no epsilon.
inline bool mt( V3 o, V3 d, V3 v0, V3 e1, V3 e2, double &t, double &u, double &v )
{
	V3 T = o - v0, P = cross( d, e2 ), Q = cross( T, e1 );
	double det = dot( e1, P );
	double inv = 1.0 / det;
	u = dot( T, P ) * inv;
	v = dot( d, Q ) * inv;
	t = dot( e2, Q ) * inv;
	return t > 0. && u >= 0. && v >= 0. && u + v <= 1.;
}

// Sphere::intersect (src/core/primitive/sphere.hpp:31-54): near root, else far
// root, accepted when t >= 0.
inline bool sphere_hit( V3 c, double r, V3 o, V3 d, double &t )
{
	V3 oc = c - o;
	double poc = dot( d, oc );
	double d2 = dot( oc, oc ) - poc * poc;
	double det = r * r - d2;
	if ( det < 0 ) return false;
	det = std::sqrt( det );
	t = poc - det;
	if ( t < 0 ) t = poc + det;
	return t >= 0;
}

// Closest hit over all primitives (src/core/meta/scene.hpp:35-55), FP64.
bool intersect( const orc_scene *s, V3 o, V3 d, double tmax, Hit &h )
{
	h = Hit();
	h.t = tmax;
	bool any = false;
	if ( !s->nodes.empty() )
	{
		V3 inv( 1.0 / d.x, 1.0 / d.y, 1.0 / d.z );
		int stack[ 128 ];
		int sp = 0;
		stack[ sp++ ] = 0;
		while ( sp )
		{
			const Node &n = s->nodes[ stack[ --sp ] ];
			if ( !box_hit( n, o, inv, h.t ) ) continue;
			if ( n.left < 0 )
			{
				for ( int i = n.first; i < n.first + n.count; ++i )
				{
					const Tri &tr = s->tris[ s->bvh_tris[ i ] ];
					double t, u, v;
					if ( mt( o, d, tr.v0, tr.v1 - tr.v0, tr.v2 - tr.v0, t, u, v ) && t < h.t )
					{
						h.t = t, h.u = u, h.v = v, h.tri = s->bvh_tris[ i ], h.prim = tr.prim;
						any = true;
					}
				}
			}
			else
			{
				stack[ sp++ ] = n.left;
				stack[ sp++ ] = n.right;
			}
		}
	}
	for ( size_t p = 0; p < s->prims.size(); ++p )
	{
		const Prim &pr = s->prims[ p ];
		if ( pr.kind != 1 ) continue;
		double t;
		if ( sphere_hit( pr.c, pr.r, o, d, t ) && t < h.t )
		{
			h.t = t, h.tri = -1, h.prim = int( p );
			h.sphere_n = normalize( o + d * t - pr.c );
			any = true;
		}
	}
	return any;
}

// Any hit on (tmin, tmax) used by ORC_MIS shadow rays.
bool occluded_ray( const orc_scene *s, V3 o, V3 d, double tmin, double tmax )
{
	if ( !s->nodes.empty() )
	{
		V3 inv( 1.0 / d.x, 1.0 / d.y, 1.0 / d.z );
		int stack[ 128 ];
		int sp = 0;
		stack[ sp++ ] = 0;
		while ( sp )
		{
			const Node &n = s->nodes[ stack[ --sp ] ];
			if ( !box_hit( n, o, inv, tmax ) ) continue;
			if ( n.left < 0 )
			{
				for ( int i = n.first; i < n.first + n.count; ++i )
				{
					const Tri &tr = s->tris[ s->bvh_tris[ i ] ];
					double t, u, v;
					if ( mt( o, d, tr.v0, tr.v1 - tr.v0, tr.v2 - tr.v0, t, u, v ) && t > tmin && t < tmax )
						return true;
				}
			}
			else
			{
				stack[ sp++ ] = n.left;
				stack[ sp++ ] = n.right;
			}
		}
	}
	for ( auto &pr : s->prims )
	{
		if ( pr.kind != 1 ) continue;
		V3 oc = pr.c - o;
		double poc = dot( d, oc ), det = pr.r * pr.r - ( dot( oc, oc ) - poc * poc );
		if ( det < 0 ) continue;
		det = std::sqrt( det );
		double t0 = poc - det, t1 = poc + det;
		if ( ( t0 > tmin && t0 < tmax ) || ( t1 > tmin && t1 < tmax ) ) return true;
	}
	return false;
}

// Scene::intersect(Seg) (src/core/meta/scene.hpp:57-67): meshes use
// Seg::intersect_triangle (src/core/basic/ray.hpp:81-90), a plane-side
// rejection followed by the ray test; spheres use Primitive::intersect(Seg)
// (src/core/primitive/primitive.hpp:15-20): ray hit with t <= seg.t.
bool occluded_seg( const orc_scene *s, V3 o, V3 d, double len )
{
	V3 e = o + d * len;
	if ( !s->nodes.empty() )
	{
		V3 lo = vmin( o, e ), hi = vmax( o, e );
		int stack[ 128 ];
		int sp = 0;
		stack[ sp++ ] = 0;
		while ( sp )
		{
			const Node &n = s->nodes[ stack[ --sp ] ];
			if ( n.hi.x < lo.x || n.hi.y < lo.y || n.hi.z < lo.z || n.lo.x > hi.x || n.lo.y > hi.y ||
				 n.lo.z > hi.z )
				continue;
			if ( n.left < 0 )
			{
				for ( int i = n.first; i < n.first + n.count; ++i )
				{
					const Tri &tr = s->tris[ s->bvh_tris[ i ] ];
					V3 d1 = tr.v1 - tr.v0, d2 = tr.v2 - tr.v0;
					V3 nn = cross( d1, d2 );
					if ( dot( o - tr.v0, nn ) * dot( e - tr.v0, nn ) > 0 ) continue;
					double t, u, v;
					if ( mt( o, d, tr.v0, d1, d2, t, u, v ) ) return true;
				}
			}
			else
			{
				stack[ sp++ ] = n.left;
				stack[ sp++ ] = n.right;
			}
		}
	}
	for ( auto &pr : s->prims )
	{
		if ( pr.kind != 1 ) continue;
		double t;
		if ( sphere_hit( pr.c, pr.r, o, d, t ) && t <= len ) return true;
	}
	return false;
}

// ---------------------------------------------------------------- camera
// PinholeLens::sample and OrthographicLens::sample (src/core/misc/lens.hpp:15-66)
// in FP64.
struct Lens
{
	V3 o, n, u, v, du, dv;
	double w, h;
	uint32_t pw;
	int kind;
	Lens( const Camera &c, uint32_t W, uint32_t H, uint32_t spp )
	{
		w = W, h = H, kind = c.lens;
		pw = uint32_t( std::ceil( std::sqrt( double( spp ) ) ) );
		o = c.pos;
		n = normalize( c.target ) * ( double( W ) / ( 2 * std::tan( c.fovx * PI / 180.0 * 0.5 ) ) );
		u = normalize( cross( n, c.up ) );
		v = normalize( cross( n, u ) );
		du = u / double( pw );
		dv = v / double( pw );
	}
	void ray( uint32_t x, uint32_t y, uint32_t k, V3 &ro, V3 &rd ) const
	{
		V3 p = u * ( double( x ) - w * .5 ) + v * ( double( y ) - h * .5 ) + du * double( k % pw ) + dv * double( k / pw );
		if ( kind == 1 )  // lens.hpp:47-52: origin moved by the plane offset * 4 / w
			ro = o + p * ( 4.0 / w ), rd = normalize( n );
		else
			ro = o, rd = normalize( n + p );
	}
};

// ---------------------------------------------------------------- BSDFs
// H::sampleCos (src/util/hemisphere.hpp:76-95): concentric disk to cosine lobe.
V3 sample_cos( double r1, double r2 )
{
	double ux = 2. * r1 - 1, uy = 2. * r2 - 1;
	if ( ux == 0 && uy == 0 ) return { 0, 0, 1 };
	double r, phi;
	if ( ux * ux > uy * uy )
		r = ux, phi = ( PI / 4 ) * ( uy / ux );
	else
		r = uy, phi = ( PI / 2 ) - ( ( PI / 4 ) * ( ux / uy ) );
	return { r * std::cos( phi ), r * std::sin( phi ), std::sqrt( std::max( 0., 1. - r * r ) ) };
}

// BeckmannDistribution::f (src/ext/distribution/beckmann.hpp:19-24): D(h)|cos th|.
double beckmann_f( double alpha2, V3 w )
{
	double c2 = w.z * w.z;
	double s2 = std::max( 0., 1 - c2 );
	double tg2 = s2 / c2;
	return std::exp( -tg2 / alpha2 ) / ( PI * alpha2 * c2 * c2 ) * std::fabs( w.z );
}

// BeckmannDistribution::sample (src/ext/distribution/beckmann.hpp:26-38).
V3 beckmann_sample( double alpha2, double u1, double u2 )
{
	double tg2 = -alpha2 * std::log( u1 );
	double phi = u2 * 2 * PI;
	double costh = 1. / std::sqrt( 1 + tg2 );
	double sinth = std::sqrt( std::max( 0., 1. - costh * costh ) );
	return { sinth * std::sin( phi ), sinth * std::cos( phi ), costh };
}

inline V3 reflect( V3 I, V3 N ) { return N * ( dot( N, I ) * 2. ) - I; }  // vmath.hpp:470-489

// A Sampler as a shader sees it: one draw at a time, in order.
struct Draws
{
	virtual double next() = 0;
};
struct RngDraws : Draws
{
	Rng &r;
	explicit RngDraws( Rng &x ) : r( x ) {}
	double next() override { return r.next(); }
};
// Scripted draws; past the end 0.5, still counted.
struct ArrayDraws : Draws
{
	const double *u;
	int n, used = 0;
	ArrayDraws( const double *a, int k ) : u( a ), n( k ) {}
	double next() override
	{
		double v = used < n ? u[ used ] : 0.5;
		++used;
		return v;
	}
};

// SphericalDistribution::f and ::sample( sampler.sample3() ): Beckmann
// (beckmann.hpp:19-38) or the cosine lobe (cosine.hpp:14-23); sampling draws
// three numbers and uses two.
double dist_f( const Shader &sh, V3 w )
{
	if ( sh.dist == ORC_DIST_COSINE ) return w.z >= 0 ? 1.0 / PI : 0.0;
	return beckmann_f( sh.alpha * sh.alpha, w );
}
V3 dist_sample( const Shader &sh, Draws &u )
{
	double u1 = u.next(), u2 = u.next();
	u.next();
	return sh.dist == ORC_DIST_COSINE ? sample_cos( u1, u2 ) : beckmann_sample( sh.alpha * sh.alpha, u1, u2 );
}

// Fresnel::compute (src/ext/scala/fresnel.hpp:17-31): dielectric reflectance
// for wo, 1 past the critical angle.
double fresnel( double ior, V3 wo )
{
	double e = wo.z > 0 ? 1 / ior : ior;
	double ci = std::fabs( wo.z );
	double sr = e * std::sqrt( std::max( 0., 1 - ci * ci ) );
	if ( sr >= 1 ) return 1;
	double cr = std::sqrt( std::max( 0., 1 - sr * sr ) );
	double par = ( ci - e * cr ) / ( ci + e * cr ), perp = ( e * ci - cr ) / ( e * ci + cr );
	return .5 * ( par * par + perp * perp );
}

// refract (src/vec/vmath.hpp:517-526).
bool refract( V3 I, V3 N, double eta, V3 &R )
{
	double c = dot( N, I );
	double s2 = std::max( 0., 1 - c * c ) * eta * eta;
	if ( s2 >= 1 ) return false;
	R = normalize( -I * eta + N * ( eta * c - std::sqrt( 1 - s2 ) ) );
	return true;
}

// Mixed::execute (mixed.hpp:24-29): one draw per Mixed, shaders[1] below fac.
int leaf( const std::vector<Shader> &tab, int idx, V3 wo, Draws &u )
{
	while ( tab[ idx ].type == ORC_MIXED )
	{
		const Shader &m = tab[ idx ];
		double f = m.fac_kind == ORC_FAC_FRESNEL ? fresnel( m.ior, wo ) : m.fac;
		idx = m.child[ u.next() < f ? 1 : 0 ];
	}
	return idx;
}

// ORC_KOISHI compute_f_by_wi_wo: Lambert (lambert.hpp:31-33), Glossy
// (glossy.hpp:27-29), Emission as white Lambert that sets the emission
// (emission.hpp:22-27), Glass (glass.hpp:25-53), zero for Transparent,
// Blackhole and Refraction (transparent.hpp:24-26, blackhole.hpp:17-20,
// refraction.hpp:35-38).
V3 k_eval( const std::vector<Shader> &tab, int idx, V3 wo, V3 wi, Draws &u, V3 &emission )
{
	const Shader &sh = tab[ leaf( tab, idx, wo, u ) ];
	emission = sh.type == ORC_EMISSION ? sh.emission : V3();
	switch ( sh.type )
	{
	case ORC_LAMBERT:
		return wi.z >= 0 ? sh.color * sh.R * ( 1.0 / PI ) : V3();
	case ORC_EMISSION:
		return wi.z >= 0 ? V3( 1, 1, 1 ) * ( 1.0 / PI ) : V3();
	case ORC_GLOSSY:
		return sh.color * dist_f( sh, normalize( wo + wi ) );
	case ORC_GLASS:
		if ( u.next() < fresnel( sh.ior, wo ) ) return sh.color * dist_f( sh, normalize( wo + wi ) );
		return sh.color * dist_f( sh, normalize( wo + wi * sh.ior ) );
	default:
		return V3();
	}
}

// Refraction through a sampled half-vector (refraction.hpp:24-33,
// glass.hpp:40-49); wi unchanged and f = 0 past the critical angle.
V3 k_refract( const Shader &sh, V3 wo, Draws &u, V3 &wi )
{
	V3 h = dist_sample( sh, u );
	double e = wo.z > 0 ? 1 / sh.ior : sh.ior;
	if ( wo.z < 0 ) h = -h;
	if ( !refract( wo, h, e, wi ) ) return V3();
	return sh.color / ( e < 1 ? e * e : 1 );
}

// ORC_KOISHI sample_wi_f_by_wo: Lambert (lambert.hpp:26-30, cosine.hpp:18-23:
// pdf 1/pi so f = color*R), Glossy (glossy.hpp:22-26), Transparent
// (transparent.hpp:20-23), Blackhole (blackhole.hpp:14-16), Refraction,
// Glass (glass.hpp:25-49).  wi is in/out.
V3 k_sample( const std::vector<Shader> &tab, int idx, V3 wo, Draws &u, V3 &wi, V3 &emission )
{
	const Shader &sh = tab[ leaf( tab, idx, wo, u ) ];
	emission = sh.type == ORC_EMISSION ? sh.emission : V3();
	switch ( sh.type )
	{
	case ORC_LAMBERT:
	case ORC_EMISSION:
	{
		double u1 = u.next(), u2 = u.next();
		u.next();
		wi = sample_cos( u1, u2 );
		V3 c = sh.type == ORC_LAMBERT ? sh.color * sh.R : V3( 1, 1, 1 );
		return wi.z >= 0 ? c : V3();
	}
	case ORC_GLOSSY:
		wi = reflect( wo, dist_sample( sh, u ) );
		return wo.z * wi.z > 0. ? sh.color : V3();
	case ORC_TRANSPARENT:
		wi = -wo;
		return sh.color;
	case ORC_REFRACTION:
		return k_refract( sh, wo, u, wi );
	case ORC_GLASS:
		if ( u.next() < fresnel( sh.ior, wo ) )
		{
			wi = reflect( wo, dist_sample( sh, u ) );
			return wo.z * wi.z > 0. ? sh.color : V3();
		}
		return k_refract( sh, wo, u, wi );
	default:
		wi = V3( 0, 0, 1 );
		return V3();
	}
}

// ORC_MIS BSDFs: Lambert color*R/pi with cosine pdf; Beckmann microfacet
// reflection color*D*G/(4 cos_o cos_i) with Walter et al.'s Smith G1 and the
// half-vector pdf D cos_h / (4 |wo.h|); Emission reflects as white Lambert.
// The remaining shaders, physically restated (the reference's own versions
// are the ORC_KOISHI ones above): RefractionBSDF and GlassBSDF as the rough
// dielectric of Walter et al. ("Microfacet Models for Refraction through
// Rough Surfaces", EGSR 2007) with a Beckmann distribution (Refraction: its
// transmission alone), Transparent as a delta pass-through, Blackhole black,
// Mixed as the fac-weighted mixture of two such leaves.  wo.z > 0 always (the
// frame faces the incoming ray); `entering` says whether wo lies outside the
// surface (against the geometric normal as built), which sets the dielectric's
// index on either side.
double smith_g1( double alpha, V3 w )
{
	double c = w.z;
	if ( c <= 0 ) return 0;
	double s = std::sqrt( std::max( 0., 1 - c * c ) );
	if ( s == 0 ) return 1;
	double a = c / ( alpha * s );
	if ( a >= 1.6 ) return 1;
	return ( 3.535 * a + 2.181 * a * a ) / ( 1 + 2.276 * a + 2.577 * a * a );
}

// Smith G1 of direction v for microfacet normal h, either side of the surface.
double smith_g1h( double alpha, V3 v, V3 h )
{
	if ( dot( v, h ) * v.z <= 0 ) return 0;
	return smith_g1( alpha, V3( v.x, v.y, std::fabs( v.z ) ) );
}

// Unpolarised Fresnel reflectance of a dielectric interface for cos_o > 0 on
// the side of index 1 and relative index eta of the other side.
double fresnel_dielectric( double cos_o, double eta )
{
	double s2 = ( 1 - cos_o * cos_o ) / ( eta * eta );
	if ( s2 >= 1 ) return 1;
	double ct = std::sqrt( 1 - s2 );
	double rs = ( cos_o - eta * ct ) / ( cos_o + eta * ct ), rp = ( eta * cos_o - ct ) / ( eta * cos_o + ct );
	return .5 * ( rs * rs + rp * rp );
}

bool m_delta( const Shader &sh ) { return sh.type == ORC_TRANSPARENT; }
bool m_transmits( const Shader &sh ) { return sh.type == ORC_GLASS || sh.type == ORC_REFRACTION || sh.type == ORC_TRANSPARENT; }

// f and pdf of a leaf (not Mixed); a delta or black leaf has none.
void m_eval_leaf( const Shader &sh, V3 wo, V3 wi, bool entering, V3 &f, double &pdf )
{
	f = V3(), pdf = 0;
	if ( wo.z <= 0 ) return;
	if ( sh.type == ORC_GLASS || sh.type == ORC_REFRACTION )
	{
		const double eo = entering ? 1 : sh.ior, et = entering ? sh.ior : 1;
		const double a = sh.alpha, a2 = a * a;
		if ( wi.z > 0 )
		{
			if ( sh.type == ORC_REFRACTION ) return;
			V3 h = normalize( wo + wi );
			double F = fresnel_dielectric( dot( wo, h ), et / eo );
			double D = beckmann_f( a2, h ) / std::fabs( h.z );
			double G = smith_g1h( a, wo, h ) * smith_g1h( a, wi, h );
			f = sh.color * ( F * D * G / ( 4 * wo.z * wi.z ) );
			pdf = F * D * h.z / ( 4 * std::fabs( dot( wo, h ) ) );
		}
		else if ( wi.z < 0 )
		{
			V3 h = normalize( -( wo * eo + wi * et ) );
			if ( h.z < 0 ) h = -h;
			double co = dot( wo, h ), ci = dot( wi, h );
			if ( co <= 0 || ci >= 0 ) return;
			double F = sh.type == ORC_GLASS ? fresnel_dielectric( co, et / eo ) : 0;
			double D = beckmann_f( a2, h ) / std::fabs( h.z );
			double G = smith_g1h( a, wo, h ) * smith_g1h( a, wi, h );
			double den = et * ci + eo * co;
			f = sh.color * ( ( 1 - F ) * D * G * std::fabs( ci ) * co * eo * eo / ( std::fabs( wi.z ) * wo.z * den * den ) );
			pdf = ( 1 - F ) * D * h.z * et * et * std::fabs( ci ) / ( den * den );
		}
		return;
	}
	if ( sh.type == ORC_TRANSPARENT || sh.type == ORC_BLACKHOLE || sh.type == ORC_MIXED || wi.z <= 0 ) return;
	if ( sh.type == ORC_GLOSSY )
	{
		V3 h = normalize( wo + wi );
		double a2 = sh.alpha * sh.alpha;
		double dh = beckmann_f( a2, h ) / std::fabs( h.z );
		double G = smith_g1( sh.alpha, wo ) * smith_g1( sh.alpha, wi );
		f = sh.color * ( dh * G / ( 4 * wo.z * wi.z ) );
		pdf = dh * h.z / ( 4 * std::fabs( dot( wo, h ) ) );
		return;
	}
	V3 c = sh.type == ORC_LAMBERT ? sh.color * sh.R : V3( 1, 1, 1 );
	f = c * ( 1.0 / PI );
	pdf = wi.z / PI;
}

// Mixed's fac for the MIS estimator: the Constant, or the Fresnel scala with
// the reference's side convention (fresnel.hpp:17-31, cos of wo against the
// surface as built).
double m_fac( const Shader &m, V3 wo, bool entering )
{
	if ( m.fac_kind != ORC_FAC_FRESNEL ) return std::min( 1.0, std::max( 0.0, m.fac ) );
	double cosi = entering ? wo.z : -wo.z;
	double e = cosi > 0 ? 1 / m.ior : m.ior;
	cosi = std::fabs( cosi );
	double sr = e * std::sqrt( std::max( 0., 1 - cosi * cosi ) );
	if ( sr >= 1 ) return 1;
	double cr = std::sqrt( std::max( 0., 1 - sr * sr ) );
	double par = ( cosi - e * cr ) / ( cosi + e * cr ), perp = ( e * cosi - cr ) / ( e * cosi + cr );
	return .5 * ( par * par + perp * perp );
}

// f and pdf of table entry idx (a leaf, or a Mixed of two leaves).
void m_eval( const std::vector<Shader> &tab, int idx, V3 wo, V3 wi, bool entering, V3 &f, double &pdf )
{
	const Shader &sh = tab[ idx ];
	if ( sh.type != ORC_MIXED ) return m_eval_leaf( sh, wo, wi, entering, f, pdf );
	double F = m_fac( sh, wo, entering );
	V3 fa, fb;
	double pa, pb;
	m_eval_leaf( tab[ sh.child[ 0 ] ], wo, wi, entering, fa, pa );
	m_eval_leaf( tab[ sh.child[ 1 ] ], wo, wi, entering, fb, pb );
	f = fa * ( 1 - F ) + fb * F;
	pdf = ( 1 - F ) * pa + F * pb;
}

// Direction of a leaf's sampling (u_sel picks a dielectric's reflection);
// false when it yields none.  Transparent is the delta direction -wo.
bool m_sample_dir_leaf( const Shader &sh, V3 wo, bool entering, double u_sel, double u1, double u2, V3 &wi )
{
	if ( wo.z <= 0 ) return false;
	switch ( sh.type )
	{
	case ORC_TRANSPARENT:
		wi = -wo;
		return true;
	case ORC_BLACKHOLE:
	case ORC_MIXED:
		return false;
	case ORC_GLOSSY:
	{
		V3 h = beckmann_sample( sh.alpha * sh.alpha, u1, u2 );
		wi = reflect( wo, h );
		return wi.z > 0 && dot( wo, h ) > 0;
	}
	case ORC_GLASS:
	case ORC_REFRACTION:
	{
		const double eo = entering ? 1 : sh.ior, et = entering ? sh.ior : 1;
		V3 h = beckmann_sample( sh.alpha * sh.alpha, u1, u2 );
		double co = dot( wo, h );
		if ( co <= 0 ) return false;
		double F = sh.type == ORC_GLASS ? fresnel_dielectric( co, et / eo ) : 0;
		if ( u_sel < F )
		{
			wi = reflect( wo, h );
			return wi.z > 0;
		}
		if ( !refract( wo, h, eo / et, wi ) ) return false;
		return wi.z < 0;
	}
	default:
		wi = sample_cos( u1, u2 );
		return wi.z > 0;
	}
}

// Sample of table entry idx: wi, weight f|cos|/pdf and pdf; delta for a
// Transparent pass-through (weight = color, no density).
void m_sample( const std::vector<Shader> &tab, int idx, V3 wo, bool entering, double u_sel, double u1, double u2,
			   V3 &wi, V3 &weight, double &pdf, bool &delta )
{
	weight = V3(), pdf = 0, delta = false;
	const Shader *leaf = &tab[ idx ];
	if ( leaf->type == ORC_MIXED )
	{
		double F = m_fac( *leaf, wo, entering );
		bool b = u_sel < F;
		u_sel = b ? u_sel / F : ( u_sel - F ) / ( 1 - F );
		leaf = &tab[ leaf->child[ b ? 1 : 0 ] ];
	}
	if ( !m_sample_dir_leaf( *leaf, wo, entering, u_sel, u1, u2, wi ) ) return;
	if ( m_delta( *leaf ) )
	{
		weight = leaf->color, delta = true;
		return;
	}
	V3 f;
	m_eval( tab, idx, wo, wi, entering, f, pdf );
	if ( pdf > 0 ) weight = f * ( std::fabs( wi.z ) / pdf );
}

// Building an orthonormal basis, revisited (Duff et al., JCGT 2017).
void onb( V3 n, V3 &b1, V3 &b2 )
{
	double sign = std::copysign( 1.0, n.z );
	double a = -1.0 / ( sign + n.z );
	double b = n.x * n.y * a;
	b1 = V3( 1.0 + sign * n.x * n.x * a, sign * b, -sign * n.x );
	b2 = V3( b, sign + n.y * n.y * a, -n.y );
}

// ---------------------------------------------------------------- integrators
struct Frame
{
	V3 u, v, n;
	V3 local( V3 w ) const { return normalize( V3( dot( w, u ), dot( w, v ), dot( w, n ) ) ); }
	V3 global( V3 w ) const { return normalize( u * w.x + v * w.y + n * w.z ); }
};

// Light::sample for a point p of the reference estimator, before the
// occlusion test: AreaLight::sample (areaLight.hpp:19-31) through the mesh
// table (mesh.hpp:92-98) or Sphere::sample (sphere.hpp:22-30, theta uniform
// in [0, pi]) with Primitive::sample's solid-angle pdf (primitive.hpp:25-33);
// PointLight::sample (pointLight.hpp:21-29) delivers its emission unscaled.
void koishi_light( const orc_scene *s, const Light &lt, V3 p, double ux, double uy, V3 &lpos, V3 &li )
{
	if ( lt.kind == 2 )
	{
		lpos = lt.pos, li = lt.emission;
		return;
	}
	const Prim &lp = s->prims[ lt.prim ];
	V3 lnrm;
	double pdf;
	if ( lt.kind == 0 )
	{
		size_t k = std::min( size_t( std::floor( ux * 1024 ) ), size_t( 1023 ) );
		lpos = V3( lt.tp[ k ].x, lt.tp[ k ].y, lt.tp[ k ].z );
		lnrm = V3( lt.tn[ k ].x, lt.tn[ k ].y, lt.tn[ k ].z );
		pdf = lt.kpdf;
	}
	else
	{
		double th = ux * PI, ph = uy * PI * 2;
		V3 w( std::sin( th ) * std::sin( ph ), std::sin( th ) * std::cos( ph ), std::cos( th ) );
		lpos = lp.c + w * lp.r;
		lnrm = w;
		pdf = 1. / ( 4 * PI * lp.r * lp.r );
	}
	V3 wiw = p - lpos;
	pdf *= dot( wiw, wiw ) / std::fabs( dot( lnrm, normalize( wiw ) ) );
	li = s->shaders[ lp.shader ].emission / pdf;
}

// RadianceKernel::execute (src/core/kernel/radiance.cu:14-81), reference semantics.
V3 radiance_koishi( const orc_scene *s, V3 o, V3 d, uint32_t max_bounce, Rng &rng )
{
	V3 L, beta( 1, 1, 1 );
	const double eps = 4e-3;  // varyings.hpp:19-37
	size_t nl = s->lights.size();
	for ( uint32_t bounce = 0;; ++bounce )
	{
		Hit h;
		if ( !intersect( s, o, d, INF, h ) ) break;
		if ( bounce > max_bounce ) break;
		const Prim &pr = s->prims[ h.prim ];
		V3 n;
		if ( h.tri >= 0 )
		{
			const Tri &t = s->tris[ h.tri ];
			n = normalize( t.n0 * ( 1 - h.u - h.v ) + t.n1 * h.u + t.n2 * h.v );  // mesh.hpp:85-91
		}
		else
			n = h.sphere_n;
		Frame fr;  // scene.hpp:48-53
		fr.n = n;
		fr.u = normalize( cross( n, V3( 0, 1, 0 ) ) );
		fr.v = normalize( cross( n, fr.u ) );
		V3 p = o + d * h.t;
		V3 wo = fr.local( -d );
		RngDraws u( rng );
		V3 emission, wi;
		if ( nl )
		{
			// radiance.cu:29-38: light choice, Light::sample with sample2()
			size_t idx = std::min( size_t( std::floor( u.next() * double( nl ) ) ), nl - 1 );
			double lpdf = 1.0 / double( nl );
			double ux = u.next(), uy = u.next();
			V3 lpos, li;
			koishi_light( s, s->lights[ idx ], p, ux, uy, lpos, li );
			V3 dd = lpos - p;  // LocalVaryings::emitSeg (varyings.hpp:27-37)
			V3 sd = normalize( dd );
			V3 diff = normalize( sd ) * eps;
			V3 so = p + diff;
			double st = length( dd - 2.0 * diff );
			if ( occluded_seg( s, so, sd, st ) ) li = V3();
			wi = fr.local( normalize( lpos - p ) );
			V3 f = k_eval( s->shaders, pr.shader, wo, wi, u, emission );
			L = L + beta * f * li * ( std::fabs( wi.z ) / lpdf );
		}
		L = L + beta * emission;  // radiance.cu:39
		// radiance.cu:55-60
		V3 es;
		V3 f = k_sample( s->shaders, pr.shader, wo, u, wi, es );
		beta = beta * f * std::fabs( wi.z );
		d = fr.global( wi );
		o = p + d * eps;
		// radiance.cu:62-68
		double rr = maxc( beta );
		if ( rr < 1. && bounce > 3 )
		{
			double q = std::max( .05, 1 - rr );
			if ( u.next() < q ) break;
			beta = beta / ( 1 - q );
		}
		if ( beta.x == 0 && beta.y == 0 && beta.z == 0 ) break;
	}
	return L;
}

// The reference's debug kernels: NormalKernel (normal.hpp:17-31),
// VisibilityKernel (visibility.hpp:17-41) and HalfVectorKernel
// (halfVector.hpp:17-43).  Visibility and HalfVector draw one sample of light 0
// through AreaLight::sample (areaLight.hpp:19-31), as the Radiance kernel's
// light sampling above does for the chosen light.
V3 aov_koishi( const orc_scene *s, V3 o, V3 d, int kind, Rng &rng )
{
	const double eps = 4e-3;  // varyings.hpp:19-37
	Hit h;
	if ( !intersect( s, o, d, INF, h ) ) return V3();
	const Prim &pr = s->prims[ h.prim ];
	V3 n;
	if ( h.tri >= 0 )
	{
		const Tri &t = s->tris[ h.tri ];
		n = normalize( t.n0 * ( 1 - h.u - h.v ) + t.n1 * h.u + t.n2 * h.v );
	}
	else
		n = h.sphere_n;
	(void)pr;
	if ( kind == ORC_AOV_NORMAL ) return n * 0.5 + V3( 0.5, 0.5, 0.5 );
	if ( s->lights.empty() ) return V3();
	Frame fr;
	fr.n = n;
	fr.u = normalize( cross( n, V3( 0, 1, 0 ) ) );
	fr.v = normalize( cross( n, fr.u ) );
	V3 p = o + d * h.t;
	V3 wo = fr.local( -d );
	double ux = rng.next(), uy = rng.next();
	V3 lpos, li;
	koishi_light( s, s->lights[ 0 ], p, ux, uy, lpos, li );
	if ( kind == ORC_AOV_HALFVECTOR )
	{
		V3 wi = fr.local( normalize( lpos - p ) );
		V3 hv = normalize( wi + wo );
		double a = std::acos( hv.z ) * 2 / PI;
		return V3( a, a, a );
	}
	V3 dd = lpos - p;
	V3 sd = normalize( dd );
	V3 diff = normalize( sd ) * eps;
	V3 so = p + diff;
	double st = length( dd - 2.0 * diff );
	if ( occluded_seg( s, so, sd, st ) ) li = V3();
	bool zero = li.x == 0 && li.y == 0 && li.z == 0;
	return zero ? V3() : V3( 1, 1, 1 );
}

// Light sampling for ORC_MIS: uniform light choice, area-proportional
// triangle choice, uniform point on the triangle / sphere.
void mis_light_sample( const orc_scene *s, const Light &lt, double u0, double u1, double u2, V3 &lp,
					   V3 &ln, double &pdfA )
{
	const Prim &pr = s->prims[ lt.prim ];
	if ( lt.kind == 1 )
	{
		double z = 1 - 2 * u1, r = std::sqrt( std::max( 0., 1 - z * z ) ), ph = 2 * PI * u2;
		V3 w( r * std::cos( ph ), r * std::sin( ph ), z );
		lp = pr.c + w * pr.r;
		ln = w;
		pdfA = 1.0 / ( 4 * PI * pr.r * pr.r );
		return;
	}
	size_t k = std::upper_bound( lt.cdf.begin(), lt.cdf.end(), u0 * lt.cdf.back() ) - lt.cdf.begin();
	k = std::min( k, lt.cdf.size() - 1 );
	const Tri &t = s->tris[ pr.first_tri + k ];
	double su = std::sqrt( u1 ), b0 = 1 - su, b1 = u2 * su;
	lp = t.v0 * b0 + t.v1 * b1 + t.v2 * ( 1 - b0 - b1 );
	ln = normalize( cross( t.v1 - t.v0, t.v2 - t.v0 ) );
	pdfA = 1.0 / lt.area;
}

V3 radiance_mis( const orc_scene *s, V3 o, V3 d, uint32_t max_bounce, Rng &rng, int variant = 0 )
{
	V3 L, beta( 1, 1, 1 );
	size_t nl = s->lights.size();
	double prev_pdf = 0;
	bool prev_delta = false;
	for ( uint32_t bounce = 0;; ++bounce )
	{
		Hit h;
		if ( !intersect( s, o, d, INF, h ) ) break;
		if ( bounce > max_bounce ) break;
		const Prim &pr = s->prims[ h.prim ];
		const Shader &sh = s->shaders[ pr.shader ];
		V3 ns, ng;
		if ( h.tri >= 0 )
		{
			const Tri &t = s->tris[ h.tri ];
			ns = normalize( t.n0 * ( 1 - h.u - h.v ) + t.n1 * h.u + t.n2 * h.v );
			ng = normalize( cross( t.v1 - t.v0, t.v2 - t.v0 ) );
		}
		else
			ns = ng = h.sphere_n;
		V3 p = o + d * h.t;
		if ( sh.type == ORC_EMISSION )
		{
			double w = 1;
			if ( bounce > 0 && variant == 3 && !prev_delta ) w = 0;
			if ( bounce > 0 && variant == 0 && !prev_delta )
			{
				const Light &lt = s->lights[ pr.light ];
				double cosl = std::fabs( dot( ng, d ) );
				double pl = cosl > 0 ? ( h.t * h.t / cosl ) / ( lt.kind == 1 ? 4 * PI * pr.r * pr.r : lt.area ) /
										 double( nl )
									 : INF;
				w = prev_pdf * prev_pdf / ( prev_pdf * prev_pdf + pl * pl );
			}
			L = L + beta * sh.emission * w;
		}
		// wo outside the surface as built: the dielectrics' index on either side
		const bool entering = dot( ng, d ) < 0;
		if ( dot( ng, d ) > 0 ) ng = -ng;
		if ( dot( ns, ng ) < 0 ) ns = -ns;
		Frame fr;
		fr.n = ns;
		onb( ns, fr.u, fr.v );
		V3 wo = fr.local( -d );
		const bool transmits = m_transmits( sh ) ||
							   ( sh.type == ORC_MIXED && ( m_transmits( s->shaders[ sh.child[ 0 ] ] ) ||
														   m_transmits( s->shaders[ sh.child[ 1 ] ] ) ) );
		if ( nl && variant != 2 )
		{
			double u0 = rng.next(), u1 = rng.next(), u2 = rng.next();
			size_t idx = std::min( size_t( std::floor( u0 * double( nl ) ) ), nl - 1 );
			double ur = u0 * double( nl ) - double( idx );
			const Light &lt = s->lights[ idx ];
			if ( lt.kind == 2 )
			{
				// a point light of intensity color * strength: irradiance I cos / r^2,
				// sampled only by NEE (weight 1)
				V3 dw = lt.pos - p;
				double dist2 = dot( dw, dw ), dist = std::sqrt( dist2 );
				V3 wiw = dw / dist;
				if ( dist > 0 && ( dot( wiw, ng ) > 0 || transmits ) )
				{
					V3 wi = fr.local( wiw ), f;
					double pb;
					m_eval( s->shaders, pr.shader, wo, wi, entering, f, pb );
					if ( ( f.x > 0 || f.y > 0 || f.z > 0 ) && !occluded_ray( s, p, wiw, 1e-7 * s->scale, dist * ( 1 - 1e-4 ) ) )
						L = L + beta * f * lt.emission * ( std::fabs( wi.z ) * double( nl ) / dist2 );
				}
			}
			else
			{
				V3 lp, ln;
				double pdfA;
				mis_light_sample( s, lt, ur, u1, u2, lp, ln, pdfA );
				V3 dw = lp - p;
				double dist2 = dot( dw, dw ), dist = std::sqrt( dist2 );
				V3 wiw = dw / dist;
				double cosl = std::fabs( dot( ln, wiw ) );
				if ( cosl > 0 && dist > 0 )
				{
					double pl = pdfA * dist2 / cosl / double( nl );
					V3 wi = fr.local( wiw );
					V3 f;
					double pb;
					m_eval( s->shaders, pr.shader, wo, wi, entering, f, pb );
					if ( ( f.x > 0 || f.y > 0 || f.z > 0 ) && ( dot( wiw, ng ) > 0 || transmits ) &&
						 !occluded_ray( s, p, wiw, 1e-7 * s->scale, dist * ( 1 - 1e-4 ) ) )
					{
						// The last vertex has no continuation that could reach the light,
						// so its light sample takes the whole weight: the estimate is then
						// the light of all paths of at most max_bounce + 1 segments, for
						// whatever continuation density the other vertices use.
						double w = variant == 3 || bounce == max_bounce ? 1.0 : pl * pl / ( pl * pl + pb * pb );
						L = L + beta * f * s->shaders[ s->prims[ lt.prim ].shader ].emission * ( std::fabs( wi.z ) * w / pl );
					}
				}
			}
		}
		double u1 = rng.next(), u2 = rng.next(), us = rng.next();
		V3 wi, wt;
		double pdf;
		bool delta;
		m_sample( s->shaders, pr.shader, wo, entering, us, u1, u2, wi, wt, pdf, delta );
		beta = beta * wt;
		if ( beta.x == 0 && beta.y == 0 && beta.z == 0 ) break;
		prev_pdf = pdf, prev_delta = delta;
		d = fr.global( wi );
		// a continuation on the far side of the surface leaves from that side
		const bool through = wi.z < 0;
		if ( through ? dot( d, ng ) >= 0 : dot( d, ng ) <= 0 ) break;
		o = p + ng * ( ( through ? -1e-7 : 1e-7 ) * s->scale );
		double rr = maxc( beta );
		if ( rr < 1. && bounce > 3 )
		{
			double q = std::max( .05, 1 - rr );
			if ( rng.next() < q ) break;
			beta = beta / ( 1 - q );
		}
	}
	return L;
}

// ---------------------------------------------------------------- koishi light tables
// Face order of a mesh as the reference stores it: the triangle list padded to
// a multiple of 4 with copies of its last triangle (createBVH, mesh.cu:135-143)
// then permuted by the recursive build (doCreateBVH, mesh.cu:35-111).
struct TInfo
{
	uint32_t idx;
	F3 vmax, vmin;
};

static float vol( F3 lo, F3 hi ) { return ( hi.x - lo.x ) * ( hi.y - lo.y ) * ( hi.z - lo.z ); }

void koishi_order( std::vector<TInfo> &info, size_t b, size_t e )
{
	F3 lo = info[ b ].vmin, hi = info[ b ].vmax;
	for ( size_t i = b; i < e; ++i )
	{
		lo = { std::min( lo.x, info[ i ].vmin.x ), std::min( lo.y, info[ i ].vmin.y ), std::min( lo.z, info[ i ].vmin.z ) };
		hi = { std::max( hi.x, info[ i ].vmax.x ), std::max( hi.y, info[ i ].vmax.y ), std::max( hi.z, info[ i ].vmax.z ) };
	}
	size_t len = e - b;
	if ( len <= 16 ) return;
	F3 w = fsub( hi, lo );
	auto first = info.begin() + b, last = info.begin() + e;
	if ( w.x >= w.y && w.x >= w.z )
		std::sort( first, last, []( const TInfo &a, const TInfo &c ) { return a.vmin.x < c.vmin.x; } );
	else if ( w.y >= w.x && w.y >= w.z )
		std::sort( first, last, []( const TInfo &a, const TInfo &c ) { return a.vmin.y < c.vmin.y; } );
	else
		std::sort( first, last, []( const TInfo &a, const TInfo &c ) { return a.vmin.z < c.vmin.z; } );
	std::vector<float> low( len ), high( len );
	const float inf = std::numeric_limits<float>::infinity();
	F3 a{ inf, inf, inf }, c{ -inf, -inf, -inf };
	for ( size_t i = 0; i < len; ++i )
	{
		auto &t = info[ b + i ];
		a = { std::min( t.vmin.x, a.x ), std::min( t.vmin.y, a.y ), std::min( t.vmin.z, a.z ) };
		c = { std::max( t.vmax.x, c.x ), std::max( t.vmax.y, c.y ), std::max( t.vmax.z, c.z ) };
		low[ i ] = vol( a, c );
	}
	a = { inf, inf, inf }, c = { -inf, -inf, -inf };
	for ( size_t i = len; i-- > 0; )
	{
		auto &t = info[ b + i ];
		a = { std::min( t.vmin.x, a.x ), std::min( t.vmin.y, a.y ), std::min( t.vmin.z, a.z ) };
		c = { std::max( t.vmax.x, c.x ), std::max( t.vmax.y, c.y ), std::max( t.vmax.z, c.z ) };
		high[ i ] = vol( a, c );
	}
	for ( size_t i = 4; i < len; i += 4 )
		if ( low[ i - 1 ] - high[ i ] >= 0.f )
		{
			koishi_order( info, b, b + i );
			koishi_order( info, b + i, e );
			return;
		}
	koishi_order( info, b, b + len / 2 );
	koishi_order( info, b + len / 2, e );
}

// Mesh::generateSamples (src/core/primitive/mesh.hpp:61-84), drawing from the
// reference's 48-bit generator (src/core/misc/sampler.hpp:22-36).
struct Drand48
{
	uint64_t x;
	float next()
	{
		x = ( 0x5DEECE66Dull * x + 0xB16ull ) & 0xFFFFFFFFFFFFull;
		return float( uint32_t( x >> 16 ) ) / float( 0x100000000LL );
	}
};

void koishi_table( const orc_scene *s, Light &lt, Drand48 &rng )
{
	const Prim &pr = s->prims[ lt.prim ];
	std::vector<TInfo> info;
	for ( int i = 0; i < pr.n_tri; ++i )
	{
		const Tri &t = s->tris[ pr.first_tri + i ];
		TInfo ti;
		ti.idx = uint32_t( i );
		ti.vmax = { std::max( t.fv0.x, std::max( t.fv1.x, t.fv2.x ) ), std::max( t.fv0.y, std::max( t.fv1.y, t.fv2.y ) ),
					std::max( t.fv0.z, std::max( t.fv1.z, t.fv2.z ) ) };
		ti.vmin = { std::min( t.fv0.x, std::min( t.fv1.x, t.fv2.x ) ), std::min( t.fv0.y, std::min( t.fv1.y, t.fv2.y ) ),
					std::min( t.fv0.z, std::min( t.fv1.z, t.fv2.z ) ) };
		info.push_back( ti );
	}
	TInfo lastInfo = info.back();
	while ( info.size() % 4 ) info.push_back( lastInfo );
	koishi_order( info, 0, info.size() );
	size_t nf = info.size();
	lt.tp.resize( 1024 );
	lt.tn.resize( 1024 );
	for ( int i = 0; i < 1024; ++i )
	{
		float r = rng.next();
		uint32_t idx = std::min( uint32_t( std::floor( r * float( nf ) ) ), uint32_t( nf - 1 ) );
		float a = rng.next(), b = rng.next();
		float uu = std::min( a, b ), vv = std::max( a, b );
		const Tri &t = s->tris[ pr.first_tri + info[ idx ].idx ];
		F3 d1 = fsub( t.fv1, t.fv0 ), d2 = fsub( t.fv2, t.fv0 );
		lt.tp[ i ] = fadd( fadd( t.fv0, fmul( d1, uu ) ), fmul( d2, vv ) );
		float w0 = 1 - uu - vv;
		lt.tn[ i ] = fnormalize( fadd( fadd( fmul( t.fn0, w0 ), fmul( t.fn1, uu ) ), fmul( t.fn2, vv ) ) );
	}
	float area = 0;
	for ( auto &ti : info )
	{
		const Tri &t = s->tris[ pr.first_tri + ti.idx ];
		F3 c = fcross( fsub( t.fv1, t.fv0 ), fsub( t.fv2, t.fv0 ) );
		float len = std::sqrt( c.x * c.x + c.y * c.y + c.z * c.z );
		area = float( double( area ) + double( len ) * .5 );
	}
	lt.kpdf = 1.f / area;
}

V3 fv( const float *p ) { return V3( p[ 0 ], p[ 1 ], p[ 2 ] ); }
F3 ff( const float *p ) { return F3{ p[ 0 ], p[ 1 ], p[ 2 ] }; }

}  // namespace

extern "C" {

orc_scene *orc_scene_new( void ) { return new orc_scene(); }
void orc_scene_free( orc_scene *s ) { delete s; }

int orc_add_shader( orc_scene *s, int type, const double *p )
{
	Shader sh;
	sh.type = type;
	switch ( type )
	{
	case ORC_LAMBERT:
		sh.R = V3( p[ 0 ], p[ 1 ], p[ 2 ] ), sh.color = V3( p[ 3 ], p[ 4 ], p[ 5 ] );
		break;
	case ORC_GLOSSY:
		sh.color = V3( p[ 0 ], p[ 1 ], p[ 2 ] ), sh.alpha = p[ 3 ], sh.dist = int( p[ 4 ] );
		break;
	case ORC_EMISSION:
	{
		// Emission stores color * strength computed in float (emission.hpp:12-20).
		float c[ 3 ] = { float( p[ 0 ] ), float( p[ 1 ] ), float( p[ 2 ] ) }, st = float( p[ 3 ] );
		sh.emission = V3( c[ 0 ] * st, c[ 1 ] * st, c[ 2 ] * st );
		break;
	}
	case ORC_TRANSPARENT:
		sh.color = V3( p[ 0 ], p[ 1 ], p[ 2 ] );
		break;
	case ORC_BLACKHOLE:
		break;
	case ORC_REFRACTION:
	case ORC_GLASS:
		sh.color = V3( p[ 0 ], p[ 1 ], p[ 2 ] ), sh.ior = float( p[ 3 ] ), sh.alpha = p[ 4 ], sh.dist = int( p[ 5 ] );
		break;
	case ORC_MIXED:
		sh.fac_kind = int( p[ 0 ] );
		if ( sh.fac_kind == ORC_FAC_FRESNEL )
			sh.ior = float( p[ 1 ] );
		else
			sh.fac = float( p[ 1 ] );
		sh.child[ 0 ] = int( p[ 2 ] ), sh.child[ 1 ] = int( p[ 3 ] );
		for ( int k = 0; k < 2; ++k )  // children first: the table stays acyclic
			if ( sh.child[ k ] < 0 || sh.child[ k ] >= int( s->shaders.size() ) ) return -1;
		break;
	default:
		return -1;
	}
	s->shaders.push_back( sh );
	return int( s->shaders.size() - 1 );
}

void orc_mis_eval( const orc_scene *s, int shader, const double *wo, const double *wi, int entering, double *f,
				   double *pdf )
{
	V3 ff;
	m_eval( s->shaders, shader, V3( wo[ 0 ], wo[ 1 ], wo[ 2 ] ), V3( wi[ 0 ], wi[ 1 ], wi[ 2 ] ), entering != 0, ff, *pdf );
	f[ 0 ] = ff.x, f[ 1 ] = ff.y, f[ 2 ] = ff.z;
}

int orc_mis_sample( const orc_scene *s, int shader, const double *wo, int entering, const double *u, double *wi,
					double *weight, double *pdf )
{
	V3 w, i;
	bool delta;
	m_sample( s->shaders, shader, V3( wo[ 0 ], wo[ 1 ], wo[ 2 ] ), entering != 0, u[ 2 ], u[ 0 ], u[ 1 ], i, w, *pdf, delta );
	wi[ 0 ] = i.x, wi[ 1 ] = i.y, wi[ 2 ] = i.z;
	weight[ 0 ] = w.x, weight[ 1 ] = w.y, weight[ 2 ] = w.z;
	return delta ? 1 : 0;
}

int orc_add_point_light( orc_scene *s, const float *pos, const double *color, double strength )
{
	// PointLight (pointLight.hpp:13-18): emission = color * strength in float
	Light lt;
	lt.kind = 2;
	lt.pos = fv( pos );
	float st = float( strength );
	lt.emission = V3( float( color[ 0 ] ) * st, float( color[ 1 ] ) * st, float( color[ 2 ] ) * st );
	s->point_lights.push_back( lt );
	return int( s->point_lights.size() - 1 );
}

int orc_shade( const orc_scene *s, int shader, int target, const double *wo, double *wi, const double *u, int k,
			   double *f, double *emission )
{
	if ( shader < 0 || shader >= int( s->shaders.size() ) ) return -1;
	ArrayDraws d( u, k );
	V3 o( wo[ 0 ], wo[ 1 ], wo[ 2 ] ), i( wi[ 0 ], wi[ 1 ], wi[ 2 ] ), e, r;
	if ( target == 0 )
		r = k_eval( s->shaders, shader, o, i, d, e );
	else
		r = k_sample( s->shaders, shader, o, d, i, e );
	for ( int c = 0; c < 3; ++c ) f[ c ] = r[ c ], emission[ c ] = e[ c ], wi[ c ] = i[ c ];
	return d.used;
}

int orc_add_mesh( orc_scene *s, const float *v, uint32_t nv, const float *n, const uint32_t *idx, uint32_t nt,
				  int shader )
{
	Prim pr;
	pr.kind = 0;
	pr.shader = shader;
	pr.first_tri = int( s->tris.size() );
	pr.n_tri = int( nt );
	int pid = int( s->prims.size() );
	for ( uint32_t t = 0; t < nt; ++t )
	{
		uint32_t a = idx[ 3 * t ], b = idx[ 3 * t + 1 ], c = idx[ 3 * t + 2 ];
		if ( a >= nv || b >= nv || c >= nv ) return -1;
		Tri tr;
		tr.fv0 = ff( v + 3 * a ), tr.fv1 = ff( v + 3 * b ), tr.fv2 = ff( v + 3 * c );
		tr.fn0 = ff( n + 3 * a ), tr.fn1 = ff( n + 3 * b ), tr.fn2 = ff( n + 3 * c );
		tr.v0 = fv( v + 3 * a ), tr.v1 = fv( v + 3 * b ), tr.v2 = fv( v + 3 * c );
		tr.n0 = fv( n + 3 * a ), tr.n1 = fv( n + 3 * b ), tr.n2 = fv( n + 3 * c );
		tr.prim = pid;
		tr.index = int( t );
		s->tris.push_back( tr );
	}
	s->prims.push_back( pr );
	return pid;
}

int orc_add_sphere( orc_scene *s, const float *c, float r, int shader )
{
	Prim pr;
	pr.kind = 1;
	pr.shader = shader;
	pr.c = fv( c );
	// The reference keeps r^2 in float and recovers r with sqrt (sphere.hpp:11-16,26).
	float r2 = r * r;
	pr.r = std::sqrt( double( r2 ) );
	pr.fr = r;
	std::memcpy( pr.fc, c, sizeof pr.fc );
	s->prims.push_back( pr );
	return int( s->prims.size() - 1 );
}

void orc_set_camera( orc_scene *s, const float *pos, const float *target, const float *up, float fovx )
{
	s->cam.pos = fv( pos ), s->cam.target = fv( target ), s->cam.up = fv( up );
	s->cam.fovx = fovx;
}

void orc_set_lens( orc_scene *s, int lens ) { s->cam.lens = lens; }

int orc_finalize( orc_scene *s, uint64_t light_seed )
{
	build_bvh( s );
	V3 lo( INF, INF, INF ), hi( -INF, -INF, -INF );
	for ( auto &t : s->tris ) lo = vmin( lo, vmin( t.v0, vmin( t.v1, t.v2 ) ) ), hi = vmax( hi, vmax( t.v0, vmax( t.v1, t.v2 ) ) );
	for ( auto &p : s->prims )
		if ( p.kind == 1 ) lo = vmin( lo, p.c - V3( p.r, p.r, p.r ) ), hi = vmax( hi, p.c + V3( p.r, p.r, p.r ) );
	s->scale = std::isfinite( lo.x ) ? std::max( 1.0, maxc( vmax( vmax( -lo, hi ), V3() ) ) ) : 1.0;
	// point lights first, in asset order (scene.cu:156-163), then area lights
	s->lights = s->point_lights;
	Drand48 rng{ light_seed & 0xFFFFFFFFFFFFull };
	for ( size_t p = 0; p < s->prims.size(); ++p )
	{
		Prim &pr = s->prims[ p ];
		if ( s->shaders[ pr.shader ].type != ORC_EMISSION ) continue;
		if ( pr.kind == 0 && pr.n_tri == 0 ) continue;
		Light lt;
		lt.prim = int( p );
		lt.kind = pr.kind;
		if ( pr.kind == 0 )
		{
			koishi_table( s, lt, rng );
			double acc = 0;
			for ( int i = 0; i < pr.n_tri; ++i )
			{
				const Tri &t = s->tris[ pr.first_tri + i ];
				acc += 0.5 * length( cross( t.v1 - t.v0, t.v2 - t.v0 ) );
				lt.cdf.push_back( acc );
			}
			lt.area = acc;
		}
		else
			lt.area = 4 * PI * pr.r * pr.r;
		pr.light = int( s->lights.size() );
		s->lights.push_back( std::move( lt ) );
	}
	return 0;
}

int orc_num_lights( const orc_scene *s ) { return int( s->lights.size() ); }

double orc_light_table( const orc_scene *s, int l, float *pts )
{
	const Light &lt = s->lights[ l ];
	if ( lt.kind != 0 ) return -1;
	for ( int i = 0; i < 1024; ++i )
	{
		pts[ 6 * i + 0 ] = lt.tp[ i ].x, pts[ 6 * i + 1 ] = lt.tp[ i ].y, pts[ 6 * i + 2 ] = lt.tp[ i ].z;
		pts[ 6 * i + 3 ] = lt.tn[ i ].x, pts[ 6 * i + 4 ] = lt.tn[ i ].y, pts[ 6 * i + 5 ] = lt.tn[ i ].z;
	}
	return lt.kpdf;
}

void orc_trace( const orc_scene *s, const float *rays, uint64_t n, int32_t *prim, int32_t *tri, double *t,
				double *u, double *v )
{
	for ( uint64_t i = 0; i < n; ++i )
	{
		const float *r = rays + 7 * i;
		Hit h;
		double tmax = std::isfinite( r[ 6 ] ) && r[ 6 ] > 0 ? double( r[ 6 ] ) : INF;
		bool hit = intersect( s, fv( r ), fv( r + 3 ), tmax, h );
		prim[ i ] = hit ? h.prim : -1;
		tri[ i ] = hit && h.tri >= 0 ? s->tris[ h.tri ].index : -1;
		t[ i ] = hit ? h.t : INF;
		u[ i ] = h.u, v[ i ] = h.v;
	}
}

void orc_ray_triangle( const orc_scene *s, const float *ray, int prim, int tri, double *t, double *u, double *v )
{
	const Tri &tr = s->tris[ s->prims[ prim ].first_tri + tri ];
	mt( fv( ray ), fv( ray + 3 ), tr.v0, tr.v1 - tr.v0, tr.v2 - tr.v0, *t, *u, *v );
}

void orc_occluded( const orc_scene *s, const float *segs, uint64_t n, uint8_t *out )
{
	for ( uint64_t i = 0; i < n; ++i )
	{
		const float *r = segs + 7 * i;
		out[ i ] = occluded_seg( s, fv( r ), fv( r + 3 ), r[ 6 ] ) ? 1 : 0;
	}
}

int orc_render( const orc_scene *s, uint32_t W, uint32_t H, uint32_t spp, uint32_t max_bounce, int estimator,
				uint64_t seed, uint32_t threads, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, double *sum,
				double *sumsq, uint32_t *count )
{
	if ( x1 > W || y1 > H || x0 >= x1 || y0 >= y1 || spp == 0 ) return -1;
	if ( estimator != ORC_KOISHI && estimator < ORC_AOV_NORMAL )
	{
		// the corrected estimator: microfacet shaders with the Beckmann
		// distribution, and Mixed of two leaves
		auto leaf_ok = [&]( const Shader &sh ) {
			if ( sh.type == ORC_MIXED ) return false;
			if ( sh.type == ORC_GLOSSY || sh.type == ORC_GLASS || sh.type == ORC_REFRACTION )
				return sh.dist == ORC_DIST_BECKMANN;
			return true;
		};
		for ( const Prim &p : s->prims )
		{
			const Shader &sh = s->shaders[ p.shader ];
			bool ok = sh.type == ORC_MIXED ? leaf_ok( s->shaders[ sh.child[ 0 ] ] ) && leaf_ok( s->shaders[ sh.child[ 1 ] ] )
										   : leaf_ok( sh );
			if ( !ok ) return -2;
		}
	}
	Lens lens( s->cam, W, H, spp );
	uint32_t ww = x1 - x0;
	std::atomic<uint32_t> next{ y0 };
	auto work = [&]() {
		for ( ;; )
		{
			uint32_t y = next.fetch_add( 1 );
			if ( y >= y1 ) break;
			for ( uint32_t x = x0; x < x1; ++x )
			{
				double a[ 3 ] = { 0, 0, 0 }, q[ 3 ] = { 0, 0, 0 };
				uint32_t c = 0;
				for ( uint32_t k = 0; k < spp; ++k )
				{
					Rng rng( seed, uint64_t( y ) * W + x, k );
					V3 ro, d;
					lens.ray( x, y, k, ro, d );
					V3 L = estimator == ORC_KOISHI ? radiance_koishi( s, ro, d, max_bounce, rng )
						   : estimator >= ORC_AOV_NORMAL
							   ? aov_koishi( s, ro, d, estimator, rng )
							   : radiance_mis( s, ro, d, max_bounce, rng, estimator == ORC_MIS ? 0 : estimator );
					if ( !finite3( L ) ) continue;  // cpuMulticore.cu:58-64
					++c;
					for ( int ch = 0; ch < 3; ++ch ) a[ ch ] += L[ ch ], q[ ch ] += L[ ch ] * L[ ch ];
				}
				size_t px = size_t( y - y0 ) * ww + ( x - x0 );
				for ( int ch = 0; ch < 3; ++ch ) sum[ 3 * px + ch ] = a[ ch ], sumsq[ 3 * px + ch ] = q[ ch ];
				count[ px ] = c;
			}
		}
	};
	if ( threads == 0 ) threads = std::max( 1u, std::thread::hardware_concurrency() );
	std::vector<std::thread> ts;
	for ( uint32_t i = 0; i < threads; ++i ) ts.emplace_back( work );
	for ( auto &t : ts ) t.join();
	return 0;
}

static Shader make_shader( int type, const double *p )
{
	orc_scene tmp;
	orc_add_shader( &tmp, type, p );
	return tmp.shaders[ 0 ];
}

void orc_bsdf_eval( int estimator, int type, const double *params, const double *wo, const double *wi, double *f,
					double *pdf )
{
	Shader sh = make_shader( type, params );
	V3 o( wo[ 0 ], wo[ 1 ], wo[ 2 ] ), i( wi[ 0 ], wi[ 1 ], wi[ 2 ] ), ff3, e;
	double pp = 0;
	if ( estimator == ORC_MIS )
		m_eval_leaf( sh, o, i, true, ff3, pp );
	else
	{
		ArrayDraws d( nullptr, 0 );
		ff3 = k_eval( std::vector<Shader>{ sh }, 0, o, i, d, e );
	}
	f[ 0 ] = ff3.x, f[ 1 ] = ff3.y, f[ 2 ] = ff3.z;
	*pdf = pp;
}

void orc_bsdf_sample( int estimator, int type, const double *params, const double *wo, const double *u, double *wi,
					  double *weight, double *pdf )
{
	Shader sh = make_shader( type, params );
	V3 o( wo[ 0 ], wo[ 1 ], wo[ 2 ] ), i, w;
	double pp = 0;
	if ( estimator == ORC_MIS )
	{
		bool delta;
		m_sample( std::vector<Shader>{ sh }, 0, o, true, 0.5, u[ 0 ], u[ 1 ], i, w, pp, delta );
	}
	else
	{
		ArrayDraws d( u, 2 );
		V3 e, f = k_sample( std::vector<Shader>{ sh }, 0, o, d, i, e );
		w = f * std::fabs( i.z );
	}
	wi[ 0 ] = i.x, wi[ 1 ] = i.y, wi[ 2 ] = i.z;
	weight[ 0 ] = w.x, weight[ 1 ] = w.y, weight[ 2 ] = w.z;
	*pdf = pp;
}

// Seg::intersect_bbox (src/core/basic/ray.hpp:59-79): separating-axis test of a
// segment against a box, restated in float as the reference evaluates it.
int orc_seg_box( const float *seg, const float *bmin, const float *bmax )
{
	float o[ 3 ] = { seg[ 0 ], seg[ 1 ], seg[ 2 ] }, d[ 3 ] = { seg[ 3 ], seg[ 4 ], seg[ 5 ] }, t = seg[ 6 ];
	float c[ 3 ], l[ 3 ], p0[ 3 ], p1[ 3 ], m[ 3 ], w[ 3 ], W[ 3 ];
	for ( int a = 0; a < 3; ++a )
	{
		c[ a ] = ( bmin[ a ] + bmax[ a ] ) * .5f;
		l[ a ] = bmax[ a ] - c[ a ];
		p0[ a ] = o[ a ] - c[ a ];
		p1[ a ] = p0[ a ] + d[ a ] * t;
		m[ a ] = ( p0[ a ] + p1[ a ] ) * .5f;
		w[ a ] = m[ a ] - p0[ a ];
		W[ a ] = std::fabs( w[ a ] );
		if ( std::fabs( m[ a ] ) - W[ a ] - l[ a ] > 0 ) return 0;
	}
	if ( std::fabs( -w[ 2 ] * m[ 1 ] + w[ 1 ] * m[ 2 ] ) > l[ 1 ] * W[ 2 ] + l[ 2 ] * W[ 1 ] ||
		 std::fabs( -w[ 2 ] * m[ 0 ] + w[ 0 ] * m[ 2 ] ) > l[ 0 ] * W[ 2 ] + l[ 2 ] * W[ 0 ] ||
		 std::fabs( -w[ 1 ] * m[ 0 ] + w[ 0 ] * m[ 1 ] ) > l[ 0 ] * W[ 1 ] + l[ 1 ] * W[ 0 ] )
		return 0;
	return 1;
}

int orc_sphere_hit( const float *c, float r, const float *ray, double *t )
{
	double tt = INF;
	bool h = sphere_hit( fv( c ), std::sqrt( double( r * r ) ), fv( ray ), fv( ray + 3 ), tt );
	*t = tt;
	return h ? 1 : 0;
}

}  // extern "C"
