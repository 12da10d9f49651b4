// Host runtime behind include/cr.h: scene model, reference JSON schema,
// mesh importers, reference-compatible light tables, device upload, render
// driver, PNG/PFM output.  No CPU fallback exists: every ray query and every
// radiance sample is computed by the CUDA kernels in render.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/cr.h"
#include "bvh_build.h"
#include "guide.h"
#include "internal.h"
#include "json.h"
#include "render.h"

using namespace cr;

namespace
{
thread_local std::string g_last_error;

struct CrError : std::runtime_error
{
	int code;
	CrError( int c, const std::string &m ) : std::runtime_error( m ), code( c ) {}
};

[[noreturn]] void fail( int code, const std::string &msg ) { throw CrError( code, msg ); }

void cuda_check( cudaError_t e, const char *what )
{
	if ( e != cudaSuccess ) fail( CR_ERR_CUDA, std::string( what ) + ": " + cudaGetErrorString( e ) );
}

template <typename F>
int guarded( F &&f )
{
	try
	{
		f();
		return CR_OK;
	}
	catch ( const CrError &e )
	{
		g_last_error = e.what();
		return e.code;
	}
	catch ( const std::exception &e )
	{
		g_last_error = e.what();
		std::string m = e.what();
		if ( m.find( "json" ) != std::string::npos ) return CR_ERR_PARSE;
		return CR_ERR_CUDA;
	}
	catch ( ... )
	{
		g_last_error = "unknown error";
		return CR_ERR_INVALID;
	}
}

// ------------------------------------------------------------------ host scene model
struct HostMesh
{
	std::vector<float> v, n;
	std::vector<uint32_t> idx;
	int shader = -1;
};

struct HostSphere
{
	float c[ 3 ];
	float r;
	int shader = -1;
};

struct HostPrim
{
	int kind;   // 0 mesh, 1 sphere
	int index;  // into meshes / spheres
};

struct HostCamera
{
	float pos[ 3 ] = { 1, 0, 0 }, target[ 3 ] = { -1, 0, 0 }, up[ 3 ] = { 0, 0, 1 };
	float fovx = 90;
	int lens = 0;  // 0 pinhole, 1 orthographic
};

// A scene's device array: stream-ordered from the library's memory pool and
// freed on the same stream (a synchronous cudaFree of a scene's arrays stalled
// scene destruction for up to 0.6 s).
template <typename T>
struct DevBuf
{
	T *p = nullptr;
	size_t n = 0;
	void upload( const std::vector<T> &h, cudaStream_t st )
	{
		alloc( h.size(), st );
		if ( n ) cuda_check( cudaMemcpyAsync( p, h.data(), sizeof( T ) * n, cudaMemcpyHostToDevice, st ), "upload" );
	}
	void alloc( size_t count, cudaStream_t st )
	{
		release( st );
		n = count;
		if ( n ) cuda_check( cudaMallocAsync( (void **)&p, sizeof( T ) * n, device_pool(), st ), "cudaMalloc" );
	}
	// freed in the order of `st`, after the work queued there
	void release( cudaStream_t st )
	{
		if ( p ) cudaFreeAsync( p, st );
		p = nullptr;
		n = 0;
	}
};

}  // namespace

struct cr_scene
{
	std::vector<std::pair<std::string, DevShader>> shaders;
	std::map<std::string, int> shader_ids;
	Json shader_cfg;  // the scene's "shaders" object, instantiated on first use
	std::vector<HostMesh> meshes;
	std::vector<HostSphere> spheres;
	std::vector<HostPrim> prims;
	std::vector<DevLight> point_lights;  // pointLight assets, in asset order
	HostCamera cam;
	bool has_camera = false;
	uint32_t max_bounce = 16;  // RadianceKernel::Configuration (radiance.hpp:12-15)
	int estimator = EST_KOISHI;
	std::string kernel = "Radiance", tracer = "CPUMulticore";

	// committed state
	bool committed = false;
	cudaStream_t stream = nullptr;
	WideBvh bvh;
	DevBuf<float4> attrs, light_tables, light_tris;
	DevBuf<float> light_cdf;
	DevBuf<DevSphere> dspheres;
	DevBuf<DevShader> dshaders;
	DevBuf<DevLight> dlights;
	DevBuf<uint32_t> prim_first;
	DevBuf<uint32_t> err;
	std::vector<DevLight> lights;
	std::vector<float4> tables_host;
	std::vector<int> prim_light;  // light id of each primitive, -1 for none (set at commit)
	std::string mis_blocker;  // why the MIS estimator cannot render this scene (empty: it can)
	uint64_t n_tris = 0;
	float scale = 1;
	WaveBuffers wave;
	uint32_t wave_bounces = 0;
	GuideState guide;
	float3 box_lo{ 0, 0, 0 }, box_hi{ 1, 1, 1 };
	// launch configuration (defaults, or the choice of cr_autotune)
	uint32_t tune_wave = 1u << 22, tune_refill = 16;
	int tune_blocks = 8;
	uint32_t tune_shade = 128;
	bool tune_bin = false;
	uint32_t tune_svote = 4, tune_srefill = 0;
	BuildParams build;  // BVH build options (cr_scene_set_build)

	~cr_scene() { release(); }
	void release_device()
	{
		if ( wave.capacity ) free_wave( wave, stream );
		if ( bvh.nodes ) cudaFreeAsync( bvh.nodes, stream );
		if ( bvh.tris ) cudaFreeAsync( bvh.tris, stream );
		bvh = WideBvh();
		attrs.release( stream ), light_tables.release( stream ), light_tris.release( stream ), light_cdf.release( stream );
		dspheres.release( stream ), dshaders.release( stream ), dlights.release( stream ), prim_first.release( stream );
		err.release( stream );
		if ( stream ) cudaStreamSynchronize( stream );
		committed = false;
	}
	void release()
	{
		release_device();
		if ( stream ) cudaStreamDestroy( stream );
		stream = nullptr;
	}
};

namespace
{
// ------------------------------------------------------------------ shaders
// Factory<Shader>::create over the shader registry (src/ext/shader/shader.impl.cu:15-24).
using ShaderTable = std::vector<std::pair<std::string, DevShader>>;

// A [Type, {props}] config (util/config.hpp:39-49) or the error the reference
// would raise for a malformed one.
const Json &config_props( const Json &cfg, const char *what )
{
	if ( !cfg.is_array() || cfg.size() < 1 || !cfg.at( 0 ).is_string() )
		fail( CR_ERR_PARSE, std::string( what ) + " config must be [Type, {props}]" );
	static const Json empty = [] {
		Json j;
		j.type = Json::Object;
		return j;
	}();
	return cfg.size() > 1 ? cfg.at( 1 ) : empty;
}

// A required number property (the reference's get<float>( props, key ) throws
// when it is absent).
float required_number( const Json &p, const char *key, const std::string &owner )
{
	const Json *v = p.find( key );
	if ( !v || !v->is_number() ) fail( CR_ERR_PARSE, owner + " needs a number \"" + key + "\"" );
	return float( v->num );
}

// The SphericalDistribution of a GlossyBSDF, RefractionBSDF or GlassBSDF
// (distribution.impl.cu: "Cosine", "Beckmann" with roughness, beckmann.hpp:11-17).
void parse_distribution( const Json &p, const std::string &owner, DevShader &s )
{
	const Json *d = p.find( "distribution" );
	if ( !d ) fail( CR_ERR_PARSE, owner + " needs a distribution" );
	const Json &dp = config_props( *d, "distribution" );
	const std::string &kind = d->at( 0 ).str;
	if ( kind == "Beckmann" )
	{
		float rough = float( dp.number_or( "roughness", 0.5 ) );
		s.dist = DIST_BECKMANN, s.alpha = rough, s.alpha2 = rough * rough;
	}
	else if ( kind == "Cosine" )
		s.dist = DIST_COSINE;
	else
		fail( CR_ERR_PARSE, "no such type: " + kind );
}

// Factory<Shader>::create (shader.impl.cu:16-23) into a flat table: returns
// the entry for cfg; the shaders a Mixed nests are appended to tab first and
// referenced by index.
DevShader make_shader( const Json &cfg, ShaderTable &tab, const std::string &name, int depth = 0 )
{
	if ( depth >= MAX_SHADER_DEPTH ) fail( CR_ERR_UNSUPPORTED, "shader " + name + " nests Mixed shaders too deeply" );
	const Json &p = config_props( cfg, "shader" );
	const std::string &type = cfg.at( 0 ).str;
	DevShader s;
	std::memset( &s, 0, sizeof s );
	float one[ 3 ] = { 1, 1, 1 };
	auto tint = [&]( DevShader &x ) {
		float c[ 3 ] = { 1, 1, 1 };
		p.vec3( "color", c );
		for ( int i = 0; i < 3; ++i ) x.color[ i ] = c[ i ], x.albedo[ i ] = c[ i ];
	};
	if ( type == "Lambert" )  // lambert.hpp:12-19
	{
		float R[ 3 ] = { 1, 1, 1 }, c[ 3 ] = { 1, 1, 1 };
		p.vec3( "R", R ), p.vec3( "color", c );
		s.type = SH_LAMBERT;
		for ( int i = 0; i < 3; ++i ) s.albedo[ i ] = c[ i ] * R[ i ], s.color[ i ] = c[ i ];
	}
	else if ( type == "GlossyBSDF" )  // glossy.hpp:11-17
	{
		tint( s );
		parse_distribution( p, "GlossyBSDF", s );
		s.type = SH_GLOSSY;
	}
	else if ( type == "Emission" )  // emission.hpp:12-20
	{
		float c[ 3 ] = { 1, 1, 1 };
		p.vec3( "color", c );
		float strength = float( p.number_or( "strength", 2.0 ) );
		s.type = SH_EMISSION;
		for ( int i = 0; i < 3; ++i ) s.emission[ i ] = c[ i ] * strength, s.albedo[ i ] = one[ i ], s.color[ i ] = one[ i ];
	}
	else if ( type == "Transparent" )  // transparent.hpp:11-15
	{
		tint( s );
		s.type = SH_TRANSPARENT;
	}
	else if ( type == "Blackhole" )  // blackhole.hpp:11
		s.type = SH_BLACKHOLE;
	else if ( type == "RefractionBSDF" || type == "GlassBSDF" )  // refraction.hpp:11-19, glass.hpp:11-21
	{
		tint( s );
		s.ior = required_number( p, "ior", type );
		parse_distribution( p, type, s );
		s.type = type == "GlassBSDF" ? SH_GLASS : SH_REFRACTION;
	}
	else if ( type == "Mixed" )  // mixed.hpp:11-20
	{
		const Json *fac = p.find( "fac" );
		if ( !fac ) fail( CR_ERR_PARSE, "Mixed needs a fac" );
		const Json &fp = config_props( *fac, "fac" );
		const std::string &fk = fac->at( 0 ).str;
		if ( fk == "Constant" )  // constant.hpp:11-20
			s.fac_kind = FAC_CONSTANT, s.fac = required_number( fp, "value", "Constant" );
		else if ( fk == "Fresnel" )  // fresnel.hpp:11-16
			s.fac_kind = FAC_FRESNEL, s.ior = required_number( fp, "ior", "Fresnel" );
		else
			fail( CR_ERR_PARSE, "no such type: " + fk );
		const Json *shs = p.find( "shaders" );
		if ( !shs || !shs->is_array() || shs->size() < 2 ) fail( CR_ERR_PARSE, "Mixed needs two \"shaders\"" );
		for ( int k = 0; k < 2; ++k )
		{
			std::string child = name + ".shaders[" + std::to_string( k ) + "]";
			DevShader c = make_shader( shs->at( k ), tab, child, depth + 1 );
			tab.emplace_back( child, c );
			s.child[ k ] = int( tab.size() - 1 );
		}
		s.type = SH_MIXED;
	}
	else
		fail( CR_ERR_PARSE, "no such type: " + type );
	return s;
}

// Whether the MIS estimator's BSDFs leave out a shader: the microfacet ones
// need the Beckmann distribution, and a Mixed two such leaves (no nesting).
bool mis_leaf_ok( const DevShader &s )
{
	if ( s.type == SH_MIXED ) return false;
	if ( s.type == SH_GLOSSY || s.type == SH_GLASS || s.type == SH_REFRACTION ) return s.dist == DIST_BECKMANN;
	return true;
}

bool koishi_only( const ShaderTable &tab, const DevShader &s )
{
	if ( s.type == SH_MIXED ) return !mis_leaf_ok( tab[ s.child[ 0 ] ].second ) || !mis_leaf_ok( tab[ s.child[ 1 ] ].second );
	return !mis_leaf_ok( s );
}

// The single-shader MIS helpers (cr_bsdf_eval / cr_bsdf_sample) cover the
// reflection-only BSDFs; renders cover the rest.
bool mis_helper_ok( const DevShader &s ) { return s.type == SH_LAMBERT || s.type == SH_EMISSION || ( s.type == SH_GLOSSY && s.dist == DIST_BECKMANN ); }

int shader_id( cr_scene *s, const std::string &name )
{
	auto it = s->shader_ids.find( name );
	if ( it != s->shader_ids.end() ) return it->second;
	const Json *cfg = s->shader_cfg.find( name );
	if ( !cfg ) fail( CR_ERR_INVALID, "Configuration for shader {" + name + "} not found." );
	DevShader sh = make_shader( *cfg, s->shaders, name );
	s->shaders.emplace_back( name, sh );
	int id = int( s->shaders.size() - 1 );
	s->shader_ids[ name ] = id;
	return id;
}

// ------------------------------------------------------------------ meshes
void smooth_normals( const std::vector<float> &v, const std::vector<uint32_t> &idx, std::vector<float> &n )
{
	n.assign( v.size(), 0.f );
	for ( size_t t = 0; t + 2 < idx.size(); t += 3 )
	{
		const float *a = &v[ 3 * idx[ t ] ], *b = &v[ 3 * idx[ t + 1 ] ], *c = &v[ 3 * idx[ t + 2 ] ];
		float e1[ 3 ] = { b[ 0 ] - a[ 0 ], b[ 1 ] - a[ 1 ], b[ 2 ] - a[ 2 ] };
		float e2[ 3 ] = { c[ 0 ] - a[ 0 ], c[ 1 ] - a[ 1 ], c[ 2 ] - a[ 2 ] };
		float fn[ 3 ] = { e1[ 1 ] * e2[ 2 ] - e1[ 2 ] * e2[ 1 ], e1[ 2 ] * e2[ 0 ] - e1[ 0 ] * e2[ 2 ],
						  e1[ 0 ] * e2[ 1 ] - e1[ 1 ] * e2[ 0 ] };
		for ( int k = 0; k < 3; ++k )
			for ( int c3 = 0; c3 < 3; ++c3 ) n[ 3 * idx[ t + k ] + c3 ] += fn[ c3 ];
	}
	for ( size_t i = 0; i + 2 < n.size(); i += 3 )
	{
		float l = std::sqrt( n[ i ] * n[ i ] + n[ i + 1 ] * n[ i + 1 ] + n[ i + 2 ] * n[ i + 2 ] );
		if ( l > 0 )
			n[ i ] /= l, n[ i + 1 ] /= l, n[ i + 2 ] /= l;
		else
			n[ i ] = 0, n[ i + 1 ] = 0, n[ i + 2 ] = 1;
	}
}

int add_mesh( cr_scene *s, const float *v, uint32_t nv, const float *n, const uint32_t *idx, uint32_t nt, int shader )
{
	if ( s->committed ) fail( CR_ERR_STATE, "scene already committed" );
	if ( ( nv && !v ) || ( nt && !idx ) ) fail( CR_ERR_INVALID, "null mesh array" );
	HostMesh m;
	m.v.assign( v, v + size_t( nv ) * 3 );
	m.idx.assign( idx, idx + size_t( nt ) * 3 );
	for ( float x : m.v )
		if ( !std::isfinite( x ) ) fail( CR_ERR_INVALID, "non-finite vertex coordinate" );
	for ( uint32_t i : m.idx )
		if ( i >= nv ) fail( CR_ERR_INVALID, "triangle index out of range" );
	if ( n )
		m.n.assign( n, n + size_t( nv ) * 3 );
	else
		smooth_normals( m.v, m.idx, m.n );
	m.shader = shader;
	s->meshes.push_back( std::move( m ) );
	s->prims.push_back( HostPrim{ 0, int( s->meshes.size() - 1 ) } );
	return int( s->prims.size() - 1 );
}

struct Group
{
	std::string name;
	std::vector<float> v, n;
	std::vector<uint32_t> idx;
};

std::string read_file( const std::string &path )
{
	std::ifstream f( path, std::ios::binary );
	if ( !f ) fail( CR_ERR_PARSE, "cannot open " + path );
	std::stringstream ss;
	ss << f.rdbuf();
	return ss.str();
}

// CRM1 binary mesh groups (written by the package's scene generator).
std::vector<Group> load_crm( const std::string &path )
{
	std::string d = read_file( path );
	size_t off = 0;
	auto take = [&]( void *dst, size_t n ) {
		if ( off + n > d.size() ) fail( CR_ERR_PARSE, "truncated mesh file " + path );
		std::memcpy( dst, d.data() + off, n );
		off += n;
	};
	char magic[ 4 ];
	take( magic, 4 );
	if ( std::memcmp( magic, "CRM1", 4 ) ) fail( CR_ERR_PARSE, "not a CRM1 mesh file: " + path );
	uint32_t ng;
	take( &ng, 4 );
	std::vector<Group> out( ng );
	for ( auto &g : out )
	{
		uint32_t len, nv, nt;
		take( &len, 4 );
		g.name.resize( len );
		if ( len ) take( &g.name[ 0 ], len );
		take( &nv, 4 );
		take( &nt, 4 );
		g.v.resize( size_t( nv ) * 3 );
		g.n.resize( size_t( nv ) * 3 );
		g.idx.resize( size_t( nt ) * 3 );
		take( g.v.data(), g.v.size() * 4 );
		take( g.n.data(), g.n.size() * 4 );
		take( g.idx.data(), g.idx.size() * 4 );
	}
	return out;
}

// Wavefront OBJ: v / vn / f (polygons fanned into triangles, negative indices
// allowed), split into one group per `usemtl` material as the reference's
// importer splits an imported scene per material (mesh.cu:332-402).  Groups
// without vertex normals get area-weighted smooth normals, as assimp's
// aiProcess_GenSmoothNormals does for the reference (scene.cu:40-44).
std::vector<Group> load_obj( const std::string &path )
{
	std::istringstream in( read_file( path ) );
	std::vector<float> P, N;
	struct Corner
	{
		long v, n;
	};
	std::vector<std::string> order;
	std::map<std::string, std::vector<std::array<Corner, 3>>> faces;
	// faces before any usemtl: the material assimp gives a mesh without one
	std::string mat = "DefaultMaterial";
	std::string line;
	size_t lineno = 0;
	auto fix = []( long i, size_t count ) -> long { return i < 0 ? long( count ) + i : i - 1; };
	while ( std::getline( in, line ) )
	{
		++lineno;
		std::istringstream ls( line );
		std::string tag;
		if ( !( ls >> tag ) || tag[ 0 ] == '#' ) continue;
		if ( tag == "v" || tag == "vn" )
		{
			float a, b, c;
			if ( !( ls >> a >> b >> c ) ) fail( CR_ERR_PARSE, path + ":" + std::to_string( lineno ) + ": bad vector" );
			auto &dst = tag == "v" ? P : N;
			dst.push_back( a ), dst.push_back( b ), dst.push_back( c );
		}
		else if ( tag == "usemtl" )
			ls >> mat;
		else if ( tag == "f" )
		{
			std::vector<Corner> poly;
			std::string tok;
			while ( ls >> tok )
			{
				Corner c{ 0, -1 };
				size_t s1 = tok.find( '/' );
				c.v = std::stol( tok.substr( 0, s1 ) );
				c.v = fix( c.v, P.size() / 3 );
				if ( s1 != std::string::npos )
				{
					size_t s2 = tok.find( '/', s1 + 1 );
					if ( s2 != std::string::npos && s2 + 1 < tok.size() ) c.n = fix( std::stol( tok.substr( s2 + 1 ) ), N.size() / 3 );
				}
				if ( c.v < 0 || size_t( c.v ) >= P.size() / 3 || ( c.n >= 0 && size_t( c.n ) >= N.size() / 3 ) )
					fail( CR_ERR_PARSE, path + ":" + std::to_string( lineno ) + ": index out of range" );
				poly.push_back( c );
			}
			if ( poly.size() < 3 ) continue;
			if ( !faces.count( mat ) ) order.push_back( mat );
			for ( size_t k = 1; k + 1 < poly.size(); ++k ) faces[ mat ].push_back( { poly[ 0 ], poly[ k ], poly[ k + 1 ] } );
		}
	}
	std::vector<Group> out;
	for ( auto &name : order )
	{
		Group g;
		g.name = name;
		std::map<std::pair<long, long>, uint32_t> remap;
		bool all_n = true;
		for ( auto &f : faces[ name ] )
			for ( auto &c : f )
			{
				auto key = std::make_pair( c.v, c.n );
				auto it = remap.find( key );
				uint32_t id;
				if ( it == remap.end() )
				{
					id = uint32_t( g.v.size() / 3 );
					remap[ key ] = id;
					g.v.insert( g.v.end(), &P[ 3 * c.v ], &P[ 3 * c.v ] + 3 );
					if ( c.n >= 0 )
						g.n.insert( g.n.end(), &N[ 3 * c.n ], &N[ 3 * c.n ] + 3 );
					else
						all_n = false, g.n.insert( g.n.end(), { 0.f, 0.f, 0.f } );
				}
				else
					id = it->second;
				g.idx.push_back( id );
			}
		if ( !all_n ) smooth_normals( g.v, g.idx, g.n );
		out.push_back( std::move( g ) );
	}
	return out;
}

bool ends_with( const std::string &s, const std::string &e );

// Stanford PLY: ascii, binary_little_endian or binary_big_endian, any
// elements and properties (scalars and lists of every PLY type).  The vertex
// element gives x, y, z and, when all three are present, nx, ny, nz; the face
// element's vertex_indices (or vertex_index) list gives polygons, fanned into
// triangles.  A PLY file carries no materials, so its mesh is one group named
// "DefaultMaterial", the name assimp gives an imported mesh without one (the
// reference binds imported meshes to shaders by material name,
// scene.cu:180-198).  Missing normals are generated as for OBJ.
std::vector<Group> load_ply( const std::string &path )
{
	const std::string d = read_file( path );
	size_t pos = 0;
	auto line = [&]() {
		size_t e = d.find( '\n', pos );
		if ( e == std::string::npos ) fail( CR_ERR_PARSE, path + ": truncated PLY header" );
		std::string l = d.substr( pos, e - pos );
		pos = e + 1;
		if ( !l.empty() && l.back() == '\r' ) l.pop_back();
		return l;
	};
	if ( line() != "ply" ) fail( CR_ERR_PARSE, path + ": not a PLY file" );
	enum Fmt { ASCII, LE, BE } fmt = ASCII;
	struct Prop
	{
		std::string name;
		int type = 0, count_type = 0;  // bytes of the value / of the list count (0: scalar)
		bool is_float = false, is_signed = false, list = false;
		bool count_signed = false;
	};
	struct Elem
	{
		std::string name;
		uint64_t count = 0;
		std::vector<Prop> props;
	};
	std::vector<Elem> elems;
	auto type_of = [&]( const std::string &t, int &bytes, bool &fl, bool &sg ) {
		static const std::map<std::string, std::array<int, 3>> T = {
			{ "char", { 1, 0, 1 } },    { "int8", { 1, 0, 1 } },   { "uchar", { 1, 0, 0 } },   { "uint8", { 1, 0, 0 } },
			{ "short", { 2, 0, 1 } },   { "int16", { 2, 0, 1 } },  { "ushort", { 2, 0, 0 } },  { "uint16", { 2, 0, 0 } },
			{ "int", { 4, 0, 1 } },     { "int32", { 4, 0, 1 } },  { "uint", { 4, 0, 0 } },    { "uint32", { 4, 0, 0 } },
			{ "float", { 4, 1, 1 } },   { "float32", { 4, 1, 1 } }, { "double", { 8, 1, 1 } }, { "float64", { 8, 1, 1 } } };
		auto it = T.find( t );
		if ( it == T.end() ) fail( CR_ERR_PARSE, path + ": unknown PLY type '" + t + "'" );
		bytes = it->second[ 0 ], fl = it->second[ 1 ] != 0, sg = it->second[ 2 ] != 0;
	};
	for ( ;; )
	{
		std::istringstream ls( line() );
		std::string tag;
		ls >> tag;
		if ( tag == "end_header" ) break;
		if ( tag == "format" )
		{
			std::string f;
			ls >> f;
			fmt = f == "ascii" ? ASCII : f == "binary_little_endian" ? LE : f == "binary_big_endian" ? BE : ( fail( CR_ERR_PARSE, path + ": unknown PLY format '" + f + "'" ), ASCII );
		}
		else if ( tag == "element" )
		{
			Elem e;
			ls >> e.name >> e.count;
			elems.push_back( e );
		}
		else if ( tag == "property" )
		{
			if ( elems.empty() ) fail( CR_ERR_PARSE, path + ": PLY property before any element" );
			Prop p;
			std::string t;
			ls >> t;
			if ( t == "list" )
			{
				std::string ct, vt;
				ls >> ct >> vt >> p.name;
				bool fl;
				type_of( ct, p.count_type, fl, p.count_signed );
				if ( fl ) fail( CR_ERR_PARSE, path + ": PLY list count of a floating type" );
				type_of( vt, p.type, p.is_float, p.is_signed );
				p.list = true;
			}
			else
			{
				ls >> p.name;
				type_of( t, p.type, p.is_float, p.is_signed );
			}
			elems.back().props.push_back( p );
		}
		// comment / obj_info lines are skipped
	}
	// value readers
	std::istringstream ascii( fmt == ASCII ? d.substr( pos ) : std::string() );
	auto read_bin = [&]( int bytes, bool fl, bool sg ) -> double {
		if ( pos + size_t( bytes ) > d.size() ) fail( CR_ERR_PARSE, path + ": truncated PLY data" );
		unsigned char b[ 8 ];
		std::memcpy( b, d.data() + pos, bytes );
		pos += bytes;
		if ( fmt == BE ) std::reverse( b, b + bytes );
		if ( fl )
		{
			if ( bytes == 4 )
			{
				float f;
				std::memcpy( &f, b, 4 );
				return f;
			}
			double v;
			std::memcpy( &v, b, 8 );
			return v;
		}
		uint64_t u = 0;
		std::memcpy( &u, b, bytes );
		if ( sg && bytes < 8 && ( u >> ( 8 * bytes - 1 ) ) & 1 ) u |= ~uint64_t( 0 ) << ( 8 * bytes );
		return sg ? double( int64_t( u ) ) : double( u );
	};
	auto read_val = [&]( int bytes, bool fl, bool sg ) -> double {
		if ( fmt != ASCII ) return read_bin( bytes, fl, sg );
		double v;
		if ( !( ascii >> v ) ) fail( CR_ERR_PARSE, path + ": truncated PLY data" );
		return v;
	};
	std::vector<float> P, N;
	std::vector<uint32_t> F;
	uint64_t nv = 0;
	bool has_n = false;
	for ( const Elem &e : elems )
	{
		int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, iface = -1;
		for ( size_t k = 0; k < e.props.size(); ++k )
		{
			const std::string &n = e.props[ k ].name;
			if ( e.name == "vertex" )
			{
				if ( n == "x" ) ix = int( k );
				if ( n == "y" ) iy = int( k );
				if ( n == "z" ) iz = int( k );
				if ( n == "nx" ) inx = int( k );
				if ( n == "ny" ) iny = int( k );
				if ( n == "nz" ) inz = int( k );
			}
			if ( e.name == "face" && e.props[ k ].list && ( n == "vertex_indices" || n == "vertex_index" ) ) iface = int( k );
		}
		if ( e.name == "vertex" )
		{
			if ( ix < 0 || iy < 0 || iz < 0 ) fail( CR_ERR_PARSE, path + ": PLY vertices without x, y, z" );
			has_n = inx >= 0 && iny >= 0 && inz >= 0;
			nv = e.count;
			if ( nv > ( 1ull << 31 ) ) fail( CR_ERR_PARSE, path + ": too many PLY vertices" );
			P.reserve( 3 * nv ), N.reserve( has_n ? 3 * nv : 0 );
		}
		for ( uint64_t i = 0; i < e.count; ++i )
		{
			double vals[ 6 ] = { 0, 0, 0, 0, 0, 0 };
			for ( size_t k = 0; k < e.props.size(); ++k )
			{
				const Prop &p = e.props[ k ];
				if ( !p.list )
				{
					double v = read_val( p.type, p.is_float, p.is_signed );
					int slot = int( k ) == ix ? 0 : int( k ) == iy ? 1 : int( k ) == iz ? 2 : int( k ) == inx ? 3 : int( k ) == iny ? 4 : int( k ) == inz ? 5 : -1;
					if ( e.name == "vertex" && slot >= 0 ) vals[ slot ] = v;
					continue;
				}
				double cnt = read_val( p.count_type, false, p.count_signed );
				if ( !( cnt >= 0 && cnt < 1e6 ) ) fail( CR_ERR_PARSE, path + ": bad PLY list length" );
				std::vector<uint32_t> poly;
				for ( uint32_t j = 0; j < uint32_t( cnt ); ++j )
				{
					double v = read_val( p.type, p.is_float, p.is_signed );
					if ( int( k ) == iface )
					{
						if ( !( v >= 0 && v < double( nv ) ) ) fail( CR_ERR_PARSE, path + ": PLY face index out of range" );
						poly.push_back( uint32_t( v ) );
					}
				}
				for ( size_t j = 1; j + 1 < poly.size(); ++j ) F.insert( F.end(), { poly[ 0 ], poly[ j ], poly[ j + 1 ] } );
			}
			if ( e.name == "vertex" )
			{
				P.insert( P.end(), { float( vals[ 0 ] ), float( vals[ 1 ] ), float( vals[ 2 ] ) } );
				if ( has_n ) N.insert( N.end(), { float( vals[ 3 ] ), float( vals[ 4 ] ), float( vals[ 5 ] ) } );
			}
		}
	}
	Group g;
	g.name = "DefaultMaterial";
	g.v = std::move( P );
	g.idx = std::move( F );
	if ( has_n )
		g.n = std::move( N );
	else
		smooth_normals( g.v, g.idx, g.n );
	std::vector<Group> out;
	out.push_back( std::move( g ) );
	return out;
}

std::vector<Group> load_mesh_file( const std::string &path )
{
	if ( ends_with( path, ".crm" ) ) return load_crm( path );
	if ( ends_with( path, ".ply" ) ) return load_ply( path );
	return load_obj( path );
}

std::string join_path( const std::string &base, const std::string &p )
{
	if ( p.empty() || p[ 0 ] == '/' || base.empty() ) return p;
	return base + "/" + p;
}

bool ends_with( const std::string &s, const std::string &e )
{
	return s.size() >= e.size() && std::equal( e.rbegin(), e.rend(), s.rbegin(), []( char a, char b ) {
			   return std::tolower( (unsigned char)a ) == std::tolower( (unsigned char)b );
		   } );
}

// Kernel configuration from the "tracer" entry (tracer.hpp:14-17, radiance.hpp:12-15).
void read_tracer( cr_scene *s, const Json &doc )
{
	const Json *tr = doc.find( "tracer" );
	if ( !tr ) return;
	if ( !tr->is_array() || tr->size() < 1 || !tr->at( 0 ).is_string() ) fail( CR_ERR_PARSE, "tracer must be [Name, {props}]" );
	s->tracer = tr->at( 0 ).str;
	if ( tr->size() < 2 ) return;
	const Json *k = tr->at( 1 ).find( "kernel" );
	if ( !k ) return;
	if ( !k->is_array() || k->size() < 1 || !k->at( 0 ).is_string() ) fail( CR_ERR_PARSE, "kernel must be [Name, {props}]" );
	s->kernel = k->at( 0 ).str;
	if ( k->size() > 1 )
	{
		double mb = k->at( 1 ).number_or( "maxBounce", 16 );
		if ( mb < 0 || mb > 1024 ) fail( CR_ERR_INVALID, "maxBounce out of range" );
		s->max_bounce = uint32_t( mb );
		std::string est = k->at( 1 ).string_or( "estimator", "koishi" );
		if ( est == "koishi" )
			s->estimator = EST_KOISHI;
		else if ( est == "mis" )
			s->estimator = EST_MIS;
		else
			fail( CR_ERR_INVALID, "unknown estimator '" + est + "' (koishi or mis)" );
	}
}

// Scene::Scene (src/core/meta/scene.cu:18-219).
void load_scene( cr_scene *s, const std::string &text, const std::string &base )
{
	Json doc = parse_json( text );
	const Json *sc = doc.find( "scene" );
	if ( !sc || !sc->is_object() ) fail( CR_ERR_PARSE, "missing \"scene\" object" );
	read_tracer( s, doc );
	if ( const Json *sh = sc->find( "shaders" ) )
	{
		if ( !sh->is_object() ) fail( CR_ERR_PARSE, "\"shaders\" must be an object" );
		s->shader_cfg = *sh;
	}
	else
		s->shader_cfg.type = Json::Object;
	if ( const Json *cams = sc->find( "camera" ) )
	{
		if ( !cams->is_array() ) fail( CR_ERR_PARSE, "\"camera\" must be an array" );
		if ( cams->size() )
		{
			const Json &c = cams->at( 0 );  // Renderer uses scene.camera[0] (renderer.cu:21-25)
			HostCamera hc;
			std::string lens = c.string_or( "lens", "pinhole" );
			if ( lens == "orthographic" )
				hc.lens = 1;
			else if ( lens != "pinhole" )
				fail( CR_ERR_PARSE, "unknown lens type: " + lens );
			hc.fovx = float( c.number_or( "fovx", 90 ) );
			c.vec3( "position", hc.pos ), c.vec3( "target", hc.target ), c.vec3( "upaxis", hc.up );
			s->cam = hc;
			s->has_camera = true;
		}
	}
	bool imported = false;
	if ( const Json *assets = sc->find( "assets" ) )
	{
		if ( !assets->is_array() ) fail( CR_ERR_PARSE, "\"assets\" must be an array" );
		for ( auto &a : assets->arr )
		{
			if ( !a.is_array() || a.size() < 1 || !a.at( 0 ).is_string() ) fail( CR_ERR_PARSE, "asset must be [name, {props}]" );
			const std::string &name = a.at( 0 ).str;
			Json none;
			none.type = Json::Object;
			const Json &p = a.size() > 1 ? a.at( 1 ) : none;
			if ( name == "import" )
			{
				if ( imported ) fail( CR_ERR_INVALID, "importing multiple scenes is not allowed" );
				imported = true;
				std::string path = join_path( base, p.string_or( "path", "" ) );
				std::vector<Group> groups = load_mesh_file( path );
				for ( auto &g : groups )
				{
					if ( g.idx.empty() ) continue;
					int sid = shader_id( s, g.name );
					add_mesh( s, g.v.data(), uint32_t( g.v.size() / 3 ), g.n.data(), g.idx.data(),
							  uint32_t( g.idx.size() / 3 ), sid );
				}
			}
			else if ( name == "sphere" )
			{
				HostSphere hs;
				if ( !p.vec3( "o", hs.c ) ) fail( CR_ERR_PARSE, "sphere needs \"o\"" );
				hs.r = float( p.number_or( "r", 1.0 ) );
				hs.shader = shader_id( s, p.string_or( "shader", "" ) );
				s->spheres.push_back( hs );
				s->prims.push_back( HostPrim{ 1, int( s->spheres.size() - 1 ) } );
			}
			else if ( name.find( "light" ) != std::string::npos || name.find( "Light" ) != std::string::npos )
			{
				if ( name != "pointLight" ) fail( CR_ERR_PARSE, "unknown light type: " + name );
				// PointLight (pointLight.hpp:13-18): position required, color * strength
				DevLight L;
				std::memset( &L, 0, sizeof L );
				L.kind = LIGHT_POINT;
				if ( !p.vec3( "position", L.pos ) ) fail( CR_ERR_PARSE, "pointLight needs \"position\"" );
				float c[ 3 ] = { 1, 1, 1 };
				p.vec3( "color", c );
				float strength = float( p.number_or( "strength", 2.0 ) );
				for ( int k = 0; k < 3; ++k ) L.emission[ k ] = c[ k ] * strength;
				s->point_lights.push_back( L );
			}
			else
				fail( CR_ERR_PARSE, "unknown asset type: " + name );
		}
	}
}

// ------------------------------------------------------------------ light tables
// Face order of a mesh as the reference stores it: the list padded to a
// multiple of 4 with copies of its last triangle (createBVH, mesh.cu:135-143),
// then permuted by the reference's recursive builder (doCreateBVH, mesh.cu:35-111),
// whose comparator sorts are reproduced with the same std::sort.
struct TriBox
{
	uint32_t idx;
	float vmax[ 3 ], vmin[ 3 ];
};

float box_volume( const float lo[ 3 ], const float hi[ 3 ] )
{
	return ( hi[ 0 ] - lo[ 0 ] ) * ( hi[ 1 ] - lo[ 1 ] ) * ( hi[ 2 ] - lo[ 2 ] );
}

void reference_face_order( std::vector<TriBox> &t, size_t b, size_t e )
{
	size_t len = e - b;
	if ( len <= 16 ) return;
	float lo[ 3 ], hi[ 3 ];
	for ( int a = 0; a < 3; ++a ) lo[ a ] = t[ b ].vmin[ a ], hi[ a ] = t[ b ].vmax[ a ];
	for ( size_t i = b; i < e; ++i )
		for ( int a = 0; a < 3; ++a ) lo[ a ] = std::min( lo[ a ], t[ i ].vmin[ a ] ), hi[ a ] = std::max( hi[ a ], t[ i ].vmax[ a ] );
	float w[ 3 ] = { hi[ 0 ] - lo[ 0 ], hi[ 1 ] - lo[ 1 ], hi[ 2 ] - lo[ 2 ] };
	int ax = ( w[ 0 ] >= w[ 1 ] && w[ 0 ] >= w[ 2 ] ) ? 0 : ( w[ 1 ] >= w[ 0 ] && w[ 1 ] >= w[ 2 ] ) ? 1 : 2;
	std::sort( t.begin() + b, t.begin() + e, [ax]( const TriBox &x, const TriBox &y ) { return x.vmin[ ax ] < y.vmin[ ax ]; } );
	const float inf = std::numeric_limits<float>::infinity();
	std::vector<float> low( len ), high( len );
	float a0[ 3 ] = { inf, inf, inf }, a1[ 3 ] = { -inf, -inf, -inf };
	for ( size_t i = 0; i < len; ++i )
	{
		for ( int a = 0; a < 3; ++a ) a0[ a ] = std::min( t[ b + i ].vmin[ a ], a0[ a ] ), a1[ a ] = std::max( t[ b + i ].vmax[ a ], a1[ a ] );
		low[ i ] = box_volume( a0, a1 );
	}
	for ( int a = 0; a < 3; ++a ) a0[ a ] = inf, a1[ a ] = -inf;
	for ( size_t i = len; i-- > 0; )
	{
		for ( int a = 0; a < 3; ++a ) a0[ a ] = std::min( t[ b + i ].vmin[ a ], a0[ a ] ), a1[ a ] = std::max( t[ b + i ].vmax[ a ], a1[ a ] );
		high[ i ] = box_volume( a0, a1 );
	}
	for ( size_t i = 4; i < len; i += 4 )
		if ( low[ i - 1 ] - high[ i ] >= 0.f )
		{
			reference_face_order( t, b, b + i );
			reference_face_order( t, b + i, e );
			return;
		}
	reference_face_order( t, b, b + len / 2 );
	reference_face_order( t, b + len / 2, e );
}

// The reference's 48-bit generator (src/core/misc/sampler.hpp:22-36).
struct Lcg48
{
	uint64_t x;
	float next()
	{
		x = ( 0x5DEECE66Dull * x + 0xB16ull ) & 0xFFFFFFFFFFFFull;
		return float( uint32_t( x >> 16 ) ) / float( 0x100000000LL );
	}
};

// Mesh::generateSamples (src/core/primitive/mesh.hpp:61-84): 1024 points,
// face picked uniformly by index, barycentrics (min, max) of two uniforms;
// pdf = 1 / total area over the padded face list.
float reference_light_table( const HostMesh &m, Lcg48 &rng, float4 *out )
{
	size_t nt = m.idx.size() / 3;
	std::vector<TriBox> t( nt );
	for ( size_t i = 0; i < nt; ++i )
	{
		t[ i ].idx = uint32_t( i );
		for ( int a = 0; a < 3; ++a )
		{
			float x0 = m.v[ 3 * m.idx[ 3 * i ] + a ], x1 = m.v[ 3 * m.idx[ 3 * i + 1 ] + a ], x2 = m.v[ 3 * m.idx[ 3 * i + 2 ] + a ];
			t[ i ].vmax[ a ] = std::max( x0, std::max( x1, x2 ) );
			t[ i ].vmin[ a ] = std::min( x0, std::min( x1, x2 ) );
		}
	}
	TriBox last = t.back();
	while ( t.size() % 4 ) t.push_back( last );
	reference_face_order( t, 0, t.size() );
	size_t nf = t.size();
	auto vert = [&]( uint32_t tri, int k, int a ) { return m.v[ 3 * m.idx[ 3 * tri + k ] + a ]; };
	auto nrm = [&]( uint32_t tri, int k, int a ) { return m.n[ 3 * m.idx[ 3 * tri + k ] + a ]; };
	for ( int i = 0; i < 1024; ++i )
	{
		float r = rng.next();
		uint32_t f = std::min( uint32_t( std::floor( r * float( nf ) ) ), uint32_t( nf - 1 ) );
		float a = rng.next(), b = rng.next();
		float u = std::min( a, b ), v = std::max( a, b );
		uint32_t tri = t[ f ].idx;
		float p[ 3 ], n[ 3 ];
		float w0 = 1 - u - v;
		for ( int c = 0; c < 3; ++c )
		{
			float o = vert( tri, 0, c ), d1 = vert( tri, 1, c ) - o, d2 = vert( tri, 2, c ) - o;
			p[ c ] = o + d1 * u + d2 * v;
			n[ c ] = nrm( tri, 0, c ) * w0 + nrm( tri, 1, c ) * u + nrm( tri, 2, c ) * v;
		}
		float inv = 1.0f / std::sqrt( n[ 0 ] * n[ 0 ] + n[ 1 ] * n[ 1 ] + n[ 2 ] * n[ 2 ] );
		out[ 2 * i ] = make_float4( p[ 0 ], p[ 1 ], p[ 2 ], 0.f );
		out[ 2 * i + 1 ] = make_float4( n[ 0 ] * inv, n[ 1 ] * inv, n[ 2 ] * inv, 0.f );
	}
	float area = 0;
	for ( auto &tb : t )
	{
		float d1[ 3 ], d2[ 3 ];
		for ( int c = 0; c < 3; ++c ) d1[ c ] = vert( tb.idx, 1, c ) - vert( tb.idx, 0, c ), d2[ c ] = vert( tb.idx, 2, c ) - vert( tb.idx, 0, c );
		float cx = d1[ 1 ] * d2[ 2 ] - d2[ 1 ] * d1[ 2 ], cy = d1[ 2 ] * d2[ 0 ] - d2[ 2 ] * d1[ 0 ], cz = d1[ 0 ] * d2[ 1 ] - d2[ 0 ] * d1[ 1 ];
		area = float( double( area ) + double( std::sqrt( cx * cx + cy * cy + cz * cz ) ) * .5 );
	}
	return 1.f / area;
}

// ------------------------------------------------------------------ commit
void commit( cr_scene *s, uint64_t light_seed, cudaStream_t user_stream )
{
	if ( s->committed ) return;
	if ( !s->stream ) cuda_check( cudaStreamCreateWithFlags( &s->stream, cudaStreamNonBlocking ), "stream" );
	cudaStream_t st = user_stream ? user_stream : s->stream;
	uint64_t nt = 0;
	for ( auto &m : s->meshes ) nt += m.idx.size() / 3;
	if ( nt >= ( 1ull << 31 ) ) fail( CR_ERR_INVALID, "too many triangles" );
	s->n_tris = nt;
	std::vector<uint32_t> prim_first( s->prims.size(), 0 );
	std::vector<int> prim_light( s->prims.size(), -1 );
	// Lights: the pointLight assets in asset order (scene.cu:156-163), then
	// every Emission-shaded primitive in primitive order (scene.cu:200-216).
	std::vector<DevLight> lights( s->point_lights );
	s->mis_blocker.clear();
	for ( const HostPrim &hp : s->prims )
	{
		int shader = hp.kind == 0 ? s->meshes[ hp.index ].shader : s->spheres[ hp.index ].shader;
		if ( s->mis_blocker.empty() && koishi_only( s->shaders, s->shaders[ shader ].second ) )
			s->mis_blocker = "shader " + s->shaders[ shader ].first;
	}
	std::vector<float4> tables, ltris;
	std::vector<float> cdf;
	Lcg48 rng{ light_seed & 0xFFFFFFFFFFFFull };
	for ( size_t p = 0; p < s->prims.size(); ++p )
	{
		const HostPrim &hp = s->prims[ p ];
		int shader = hp.kind == 0 ? s->meshes[ hp.index ].shader : s->spheres[ hp.index ].shader;
		const DevShader &sh = s->shaders[ shader ].second;
		if ( sh.type != SH_EMISSION ) continue;
		DevLight L;
		std::memset( &L, 0, sizeof L );
		for ( int c = 0; c < 3; ++c ) L.emission[ c ] = sh.emission[ c ];
		if ( hp.kind == 1 )
		{
			const HostSphere &hs = s->spheres[ hp.index ];
			L.kind = LIGHT_SPHERE;
			L.index = hp.index;
			float r2 = hs.r * hs.r;
			L.area = float( 4.0 * M_PI * double( r2 ) );
			L.koishi_pdf = 1.f / ( 4.f * float( M_PI ) * r2 );
		}
		else
		{
			const HostMesh &m = s->meshes[ hp.index ];
			if ( m.idx.empty() ) continue;
			L.kind = LIGHT_MESH;
			L.index = int( ltris.size() / 3 );
			L.n_tris = int( m.idx.size() / 3 );
			L.table = int( tables.size() / 2 );
			tables.resize( tables.size() + 2048 );
			L.koishi_pdf = reference_light_table( m, rng, &tables[ tables.size() - 2048 ] );
			L.cdf = int( cdf.size() );
			double acc = 0;
			for ( int t = 0; t < L.n_tris; ++t )
			{
				const float *a = &m.v[ 3 * m.idx[ 3 * t ] ], *b = &m.v[ 3 * m.idx[ 3 * t + 1 ] ], *c = &m.v[ 3 * m.idx[ 3 * t + 2 ] ];
				double e1[ 3 ] = { double( b[ 0 ] ) - a[ 0 ], double( b[ 1 ] ) - a[ 1 ], double( b[ 2 ] ) - a[ 2 ] };
				double e2[ 3 ] = { double( c[ 0 ] ) - a[ 0 ], double( c[ 1 ] ) - a[ 1 ], double( c[ 2 ] ) - a[ 2 ] };
				double cx = e1[ 1 ] * e2[ 2 ] - e1[ 2 ] * e2[ 1 ], cy = e1[ 2 ] * e2[ 0 ] - e1[ 0 ] * e2[ 2 ], cz = e1[ 0 ] * e2[ 1 ] - e1[ 1 ] * e2[ 0 ];
				acc += 0.5 * std::sqrt( cx * cx + cy * cy + cz * cz );  // FP64 prefix sum
				cdf.push_back( float( acc ) );
				ltris.push_back( make_float4( a[ 0 ], a[ 1 ], a[ 2 ], 0 ) );
				ltris.push_back( make_float4( b[ 0 ], b[ 1 ], b[ 2 ], 0 ) );
				ltris.push_back( make_float4( c[ 0 ], c[ 1 ], c[ 2 ], 0 ) );
			}
			L.area = float( acc );
			if ( !( acc > 0 ) ) continue;  // a degenerate emitter contributes nothing
		}
		prim_light[ p ] = int( lights.size() );
		lights.push_back( L );
	}
	// Flatten triangles in primitive order, on the device: the indexed meshes
	// go up as they are (12 bytes per vertex and normal, 12 per triangle), and
	// k_flatten_mesh writes the builder's vertex records and the attribute
	// records, and the bounds of the referenced vertices.
	uint64_t g = 0;
	size_t n_sph = 0;
	for ( size_t p = 0; p < s->prims.size(); ++p )
	{
		prim_first[ p ] = uint32_t( g );
		if ( s->prims[ p ].kind == 0 )
			g += s->meshes[ s->prims[ p ].index ].idx.size() / 3;
		else
			++n_sph;
	}
	const uint64_t n_prims = nt + n_sph;
	if ( n_prims >= ( 1ull << 31 ) ) fail( CR_ERR_INVALID, "too many primitives" );
	float4 *d_src = nullptr;
	if ( n_prims ) cuda_check( cudaMallocAsync( (void **)&d_src, sizeof( float4 ) * 3 * n_prims, device_pool(), st ), "cudaMalloc" );
	// the builder's input lives until the end of the commit, whichever way it ends
	struct StreamFree
	{
		void *p;
		cudaStream_t st;
		~StreamFree()
		{
			if ( p ) cudaFreeAsync( p, st );
		}
	} src_guard{ d_src, st };
	s->attrs.alloc( 3 * nt, st );
	float lo[ 3 ] = { INFINITY, INFINITY, INFINITY }, hi[ 3 ] = { -INFINITY, -INFINITY, -INFINITY };
	if ( nt )
	{
		size_t nv_all = 0;
		for ( const HostMesh &m : s->meshes ) nv_all += m.v.size() / 3;
		float *d_v = nullptr, *d_n = nullptr, *d_b = nullptr;
		uint32_t *d_idx = nullptr;
		cuda_check( cudaMallocAsync( (void **)&d_v, sizeof( float ) * 3 * std::max<size_t>( nv_all, 1 ), device_pool(), st ), "cudaMalloc" );
		StreamFree v_guard{ d_v, st };
		cuda_check( cudaMallocAsync( (void **)&d_n, sizeof( float ) * 3 * std::max<size_t>( nv_all, 1 ), device_pool(), st ), "cudaMalloc" );
		StreamFree n_guard{ d_n, st };
		cuda_check( cudaMallocAsync( (void **)&d_idx, sizeof( uint32_t ) * 3 * nt, device_pool(), st ), "cudaMalloc" );
		StreamFree idx_guard{ d_idx, st };
		cuda_check( cudaMallocAsync( (void **)&d_b, sizeof( float ) * 6, device_pool(), st ), "cudaMalloc" );
		StreamFree b_guard{ d_b, st };
		const float b0[ 6 ] = { INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY };
		cuda_check( cudaMemcpyAsync( d_b, b0, sizeof b0, cudaMemcpyHostToDevice, st ), "upload" );
		size_t vo = 0, io = 0;
		for ( size_t p = 0; p < s->prims.size(); ++p )
		{
			const HostPrim &hp = s->prims[ p ];
			if ( hp.kind != 0 ) continue;
			const HostMesh &m = s->meshes[ hp.index ];
			const size_t nv = m.v.size() / 3, nm = m.idx.size() / 3;
			if ( !nm ) continue;
			cuda_check( cudaMemcpyAsync( d_v + 3 * vo, m.v.data(), sizeof( float ) * 3 * nv, cudaMemcpyHostToDevice, st ), "upload" );
			cuda_check( cudaMemcpyAsync( d_n + 3 * vo, m.n.data(), sizeof( float ) * 3 * nv, cudaMemcpyHostToDevice, st ), "upload" );
			cuda_check( cudaMemcpyAsync( d_idx + 3 * io, m.idx.data(), sizeof( uint32_t ) * 3 * nm, cudaMemcpyHostToDevice, st ),
						"upload" );
			FlatMesh fm{ d_v + 3 * vo, d_n + 3 * vo, d_idx + 3 * io, uint32_t( nm ), prim_first[ p ], m.shader, int( p ),
						 prim_light[ p ] };
			flatten_mesh( fm, d_src, s->attrs.p, d_b, st );
			vo += nv, io += nm;
		}
		float b[ 6 ];
		cuda_check( cudaMemcpyAsync( b, d_b, sizeof b, cudaMemcpyDeviceToHost, st ), "bounds" );
		cuda_check( cudaStreamSynchronize( st ), "flatten" );
		for ( int a = 0; a < 3; ++a ) lo[ a ] = b[ a ], hi[ a ] = b[ 3 + a ];
	}
	std::vector<DevSphere> ds;
	std::vector<float4> sph_src;
	for ( size_t p = 0; p < s->prims.size(); ++p )
	{
		const HostPrim &hp = s->prims[ p ];
		if ( hp.kind != 1 ) continue;
		const HostSphere &hs = s->spheres[ hp.index ];
		DevSphere d;
		for ( int a = 0; a < 3; ++a )
			d.c[ a ] = hs.c[ a ], lo[ a ] = std::min( lo[ a ], hs.c[ a ] - hs.r ), hi[ a ] = std::max( hi[ a ], hs.c[ a ] + hs.r );
		d.r2 = hs.r * hs.r;  // the reference keeps r^2 (sphere.hpp:11-16)
		d.r = std::sqrt( d.r2 );
		d.shader = hs.shader;
		d.prim = int( p );
		d.light = prim_light[ p ];
		ds.push_back( d );
		// the sphere as a BVH primitive: its box (the builder's bounds of the
		// three points) and, in the third record, centre and r^2
		sph_src.push_back( make_float4( hs.c[ 0 ] - d.r, hs.c[ 1 ] - d.r, hs.c[ 2 ] - d.r, 0.f ) );
		sph_src.push_back( make_float4( hs.c[ 0 ] + d.r, hs.c[ 1 ] + d.r, hs.c[ 2 ] + d.r, 0.f ) );
		sph_src.push_back( make_float4( hs.c[ 0 ], hs.c[ 1 ], hs.c[ 2 ], d.r2 ) );
	}
	if ( !sph_src.empty() )
		cuda_check( cudaMemcpyAsync( d_src + 3 * nt, sph_src.data(), sizeof( float4 ) * sph_src.size(), cudaMemcpyHostToDevice, st ),
					"upload" );
	float sc = 1;
	for ( int a = 0; a < 3; ++a )
		if ( std::isfinite( lo[ a ] ) ) sc = std::max( sc, std::max( std::fabs( lo[ a ] ), std::fabs( hi[ a ] ) ) );
	s->scale = sc;
	if ( std::isfinite( lo[ 0 ] ) )
		s->box_lo = make_float3( lo[ 0 ], lo[ 1 ], lo[ 2 ] ), s->box_hi = make_float3( hi[ 0 ], hi[ 1 ], hi[ 2 ] );
	std::vector<DevShader> dsh;
	for ( auto &x : s->shaders ) dsh.push_back( x.second );

	s->dspheres.upload( ds, st );
	s->dshaders.upload( dsh, st );
	s->dlights.upload( lights, st );
	s->light_tables.upload( tables, st );
	s->light_tris.upload( ltris, st );
	s->light_cdf.upload( cdf, st );
	s->prim_first.upload( prim_first, st );
	s->err.upload( std::vector<uint32_t>( 2, 0 ), st );  // [0] error word, [1] query work cursor
	s->lights = lights;
	s->tables_host = tables;
	s->prim_light = prim_light;
	// BVH over the triangles (ids 0 .. nt-1) and the spheres (ids nt ..)
	if ( n_prims )
	{
		try
		{
			build_wide_bvh( d_src, uint32_t( n_prims ), s->bvh, st, s->build );
		}
		catch ( const std::exception &e )
		{
			fail( CR_ERR_CUDA, e.what() );
		}
		if ( s->bvh.depth > uint32_t( TRAVERSAL_STACK ) )
			fail( CR_ERR_INVALID, "BVH depth " + std::to_string( s->bvh.depth ) + " exceeds the traversal stack" );
	}
	cuda_check( cudaStreamSynchronize( st ), "commit" );
	s->committed = true;
}

DevScene dev_scene( const cr_scene *s )
{
	DevScene d;
	std::memset( &d, 0, sizeof d );
	d.nodes = s->bvh.nodes;
	d.tris = s->bvh.tris;
	d.attrs = s->attrs.p;
	d.spheres = s->dspheres.p;
	d.shaders = s->dshaders.p;
	d.lights = s->dlights.p;
	d.light_tables = s->light_tables.p;
	d.light_tris = s->light_tris.p;
	d.light_cdf = s->light_cdf.p;
	d.prim_first = s->prim_first.p;
	d.n_nodes = s->bvh.n_nodes;
	d.n_tris = s->bvh.n_tris;  // BVH primitives: the triangles, then the spheres
	d.sph_base = uint32_t( s->n_tris );
	d.n_spheres = uint32_t( s->dspheres.n );
	d.n_lights = uint32_t( s->dlights.n );
	d.n_shaders = uint32_t( s->dshaders.n );
	d.scene_scale = s->scale;
	return d;
}

// The Lens base (src/core/misc/lens.hpp:15-27) for a W x H image at spp; the
// lens kind selects PinholeLens or OrthographicLens (renderer.cu:30-38).
DevCamera make_camera( const HostCamera &c, uint32_t w, uint32_t h, uint32_t spp )
{
	auto norm = []( const float a[ 3 ], float o[ 3 ] ) {
		float r = 1.0f / std::sqrt( a[ 0 ] * a[ 0 ] + a[ 1 ] * a[ 1 ] + a[ 2 ] * a[ 2 ] );
		for ( int i = 0; i < 3; ++i ) o[ i ] = a[ i ] * r;
	};
	auto crs = []( const float a[ 3 ], const float b[ 3 ], float o[ 3 ] ) {
		o[ 0 ] = a[ 1 ] * b[ 2 ] - b[ 1 ] * a[ 2 ];
		o[ 1 ] = a[ 2 ] * b[ 0 ] - b[ 2 ] * a[ 0 ];
		o[ 2 ] = a[ 0 ] * b[ 1 ] - b[ 0 ] * a[ 1 ];
	};
	DevCamera d;
	d.width = w, d.height = h;
	d.lens = uint32_t( c.lens );
	d.pw = uint32_t( std::ceil( std::sqrt( double( spp ) ) ) );
	float t[ 3 ], tmp[ 3 ];
	norm( c.target, t );
	float scale = float( double( w ) / ( 2 * std::tan( double( c.fovx ) * .5 * M_PI / 180.0 ) ) );
	for ( int i = 0; i < 3; ++i ) d.n[ i ] = t[ i ] * scale, d.o[ i ] = c.pos[ i ];
	crs( d.n, c.up, tmp );
	norm( tmp, d.u );
	crs( d.n, d.u, tmp );
	norm( tmp, d.v );
	for ( int i = 0; i < 3; ++i ) d.du[ i ] = d.u[ i ] / float( d.pw ), d.dv[ i ] = d.v[ i ] / float( d.pw );
	return d;
}

struct Resolved
{
	RenderConfig cfg;
	DevScene sc;
	uint64_t samples;
};

// Factory<Kernel> names (src/core/kernel/kernel.impl.cu:10-15) -> KERNEL_*; -1 if unknown.
int kernel_id( const std::string &name )
{
	if ( name == "Radiance" ) return KERNEL_RADIANCE;
	if ( name == "Normal" ) return KERNEL_NORMAL;
	if ( name == "Visibility" ) return KERNEL_VISIBILITY;
	if ( name == "HalfVector" ) return KERNEL_HALFVECTOR;
	return -1;
}

Resolved resolve( cr_scene *s, const cr_render_desc *desc )
{
	if ( !s || !desc ) fail( CR_ERR_INVALID, "null argument" );
	if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
	if ( !desc->width || !desc->height || !desc->spp ) fail( CR_ERR_INVALID, "width, height and spp must be positive" );
	if ( !s->has_camera ) fail( CR_ERR_INVALID, "no camera in the scene" );
	const int kernel = kernel_id( s->kernel );
	if ( kernel < 0 )
		fail( CR_ERR_UNSUPPORTED, "kernel '" + s->kernel + "' is not registered (Radiance, Normal, Visibility, HalfVector)" );

	Resolved r;
	RenderConfig &c = r.cfg;
	uint32_t x0 = desc->x0, y0 = desc->y0, x1 = desc->x1, y1 = desc->y1;
	if ( !x0 && !y0 && !x1 && !y1 ) x1 = desc->width, y1 = desc->height;
	if ( x1 > desc->width || y1 > desc->height || x0 >= x1 || y0 >= y1 ) fail( CR_ERR_INVALID, "bad pixel window" );
	c.spp = desc->spp;
	c.max_bounce = desc->max_bounce == UINT32_MAX ? s->max_bounce : desc->max_bounce;
	if ( c.max_bounce > 1024 ) fail( CR_ERR_INVALID, "max_bounce out of range" );
	c.estimator = desc->estimator < 0 ? s->estimator : desc->estimator;
	if ( c.estimator != EST_KOISHI && c.estimator != EST_MIS ) fail( CR_ERR_INVALID, "unknown estimator" );
	if ( c.estimator == EST_MIS && !s->mis_blocker.empty() )
		fail( CR_ERR_UNSUPPORTED, "the MIS estimator takes microfacet shaders with the Beckmann distribution and "
								  "Mixed of two leaves; " + s->mis_blocker + " has the reference estimator only" );
	c.x0 = x0, c.y0 = y0, c.ww = x1 - x0, c.wh = y1 - y0;
	c.seed = desc->seed;
	r.samples = uint64_t( c.ww ) * c.wh * c.spp;
	uint64_t cap = desc->wave_paths ? desc->wave_paths : s->tune_wave;
	cap = std::min<uint64_t>( cap, r.samples );
	cap = std::min<uint64_t>( cap, 1ull << 30 );
	c.wave_paths = uint32_t( cap );
	c.count_work = desc->count_work != 0;
	c.refill_min = desc->refill_min ? std::min<uint32_t>( desc->refill_min, 32 ) : s->tune_refill;
	c.traverse_blocks_per_sm =
		desc->traverse_blocks_per_sm ? int( std::min<uint32_t>( desc->traverse_blocks_per_sm, 8 ) ) : s->tune_blocks;
	if ( desc->shade_threads && desc->shade_threads != 64 && desc->shade_threads != 128 && desc->shade_threads != 256 )
		fail( CR_ERR_INVALID, "shade_threads must be 64, 128 or 256" );
	c.shade_threads = desc->shade_threads ? desc->shade_threads : s->tune_shade;
	c.bin_rays = desc->bin_rays ? desc->bin_rays > 0 : s->tune_bin;
	if ( desc->shadow_vote > 32 || desc->shadow_refill_min > 32 )
		fail( CR_ERR_INVALID, "shadow_vote and shadow_refill_min must be 1..32" );
	c.shadow_vote = desc->shadow_vote ? desc->shadow_vote : s->tune_svote;
	c.shadow_refill_min = desc->shadow_refill_min ? desc->shadow_refill_min : s->tune_srefill;
	// plain renders: the reference's roulette after bounce 3; guided renders:
	// none (on the occluded-light scene roulette's variance is most of what
	// the guide leaves, and removing it makes guiding 2.7x as efficient as
	// plain MIS without roulette, against 1.3x with it)
	c.rr_start = desc->rr_start ? desc->rr_start : ( desc->guiding ? UINT32_MAX : 4u );
	r.sc = dev_scene( s );
	r.sc.cam = make_camera( s->cam, desc->width, desc->height, desc->spp );
	c.kernel = kernel;
	if ( ( kernel == KERNEL_VISIBILITY || kernel == KERNEL_HALFVECTOR ) && s->lights.empty() )
		fail( CR_ERR_INVALID, "kernel '" + s->kernel + "' samples light 0, and the scene has no light" );
	if ( kernel != KERNEL_RADIANCE && desc->guiding )
		fail( CR_ERR_INVALID, "learned path guiding needs the Radiance kernel" );
	if ( desc->guiding )
	{
		if ( c.estimator != EST_MIS ) fail( CR_ERR_INVALID, "learned path guiding needs the MIS estimator" );
		if ( !s->guide.ready ) s->guide.init( s->box_lo, s->box_hi, 0x9E3779B9ull );
		c.guiding = true;
		c.guide = s->guide.dev();
		const uint64_t rec_paths =
			std::min<uint64_t>( uint64_t( s->guide.train_paths ) * s->guide.steps_per_wave, c.wave_paths );
		const uint64_t slots = rec_paths * ( uint64_t( c.max_bounce ) + 1 );
		if ( slots > ( 1ull << 28 ) ) fail( CR_ERR_INVALID, "guide training records exceed 2^28 vertices per wave" );
		s->guide.ensure_records( uint32_t( slots ) );
		c.rec = s->guide.rec;
	}
	return r;
}

// Whether the wave state of `paths` paths (WaveBuffers: about 140 bytes per
// path plus the queue counters) fits in half of the device's free memory.
bool wave_fits( uint64_t paths, uint32_t max_bounce )
{
	size_t free_b = 0, total_b = 0;
	if ( cudaMemGetInfo( &free_b, &total_b ) != cudaSuccess ) return false;
	const uint64_t need = paths * ( 6 * sizeof( float4 ) + 3 * sizeof( float4 ) + sizeof( HitRec ) + 4 * sizeof( uint32_t ) ) +
						  uint64_t( n_counters_for( max_bounce ) ) * 4;
	return need * 2 <= free_b;
}

void ensure_wave( cr_scene *s, uint32_t cap, uint32_t max_bounce, cudaStream_t st, bool lobes = false,
				  bool bins = false )
{
	if ( !( s->wave.capacity >= cap && s->wave_bounces >= max_bounce ) )
	{
		if ( s->wave.capacity ) free_wave( s->wave, st );
		alloc_wave( s->wave, cap, max_bounce, st );
		s->wave_bounces = max_bounce;
	}
	if ( lobes ) alloc_lobes( s->wave, st );
	if ( bins ) alloc_bins( s->wave, st );
}

void check_device_error( cr_scene *s, cudaStream_t st )
{
	uint32_t e = 0;
	cuda_check( cudaMemcpyAsync( &e, s->wave.capacity ? s->wave.err : s->err.p, 4, cudaMemcpyDeviceToHost, st ), "error word" );
	cuda_check( cudaStreamSynchronize( st ), "error word" );
	if ( e ) fail( CR_ERR_DEVICE, "a traversal kernel reported error flags " + std::to_string( e ) +
								  " (1: stack overflow, 2: node index or budget, 4: triangle index, 8: guide MMA wait timed out, "
								  "16: ray binning overflow)" );
}

void fill_stats( cr_stats *out, const StageTimes &t, uint64_t samples )
{
	if ( !out ) return;
	std::memset( out, 0, sizeof *out );
	out->ms_total = t.total, out->ms_extend = t.extend, out->ms_shadow = t.shadow, out->ms_shade = t.shade;
	out->ms_other = t.other + t.guide;
	out->ms_guide = t.guide;
	out->ms_guide_train = t.guide_train;
	out->samples = samples;
	out->rays_extend = t.rays_extend, out->rays_shadow = t.rays_shadow;
	out->nodes = t.nodes, out->tris = t.tris, out->shadow_nodes = t.shadow_nodes, out->shadow_tris = t.shadow_tris;
	out->launches = t.launches, out->waves = t.waves;
	out->extend_launches = t.extend_launches, out->shadow_launches = t.shadow_launches;
	out->guide_launches = t.guide_launches, out->guide_rows = t.guide_rows;
}

void render_device( cr_scene *s, const cr_render_desc *desc, double *sum, double *sq, uint32_t *cnt, cudaStream_t st,
					cr_stats *stats )
{
	Resolved r = resolve( s, desc );
	ensure_wave( s, r.cfg.wave_paths, r.cfg.max_bounce, st, r.cfg.guiding, r.cfg.bin_rays );
	StageTimes t;
	render_waves( r.sc, r.cfg, s->wave, sum, sq, cnt, st, stats ? &t : nullptr, &s->guide );
	if ( stats )
	{
		fill_stats( stats, t, r.samples );
		check_device_error( s, st );
	}
}

// ------------------------------------------------------------------ PNG
uint32_t crc32( const unsigned char *p, size_t n, uint32_t c = 0xFFFFFFFFu )
{
	// built once, thread-safely (a function-local static)
	static const std::array<uint32_t, 256> table = [] {
		std::array<uint32_t, 256> t{};
		for ( uint32_t i = 0; i < 256; ++i )
		{
			uint32_t x = i;
			for ( int k = 0; k < 8; ++k ) x = ( x & 1 ) ? 0xEDB88320u ^ ( x >> 1 ) : x >> 1;
			t[ i ] = x;
		}
		return t;
	}();
	for ( size_t i = 0; i < n; ++i ) c = table[ ( c ^ p[ i ] ) & 0xFF ] ^ ( c >> 8 );
	return c;
}

void put_be32( std::string &s, uint32_t v )
{
	s += char( v >> 24 ), s += char( v >> 16 ), s += char( v >> 8 ), s += char( v );
}

void png_chunk( std::string &out, const char *type, const std::string &data )
{
	put_be32( out, uint32_t( data.size() ) );
	std::string td = std::string( type, 4 ) + data;
	out += td;
	put_be32( out, crc32( (const unsigned char *)td.data(), td.size() ) ^ 0xFFFFFFFFu );
}

// 8-bit RGB PNG with stored (uncompressed) deflate blocks.
void write_png( const std::string &path, uint32_t w, uint32_t h, const double *rgb )
{
	std::string raw;
	raw.reserve( size_t( h ) * ( 1 + 3 * size_t( w ) ) );
	for ( uint32_t y = 0; y < h; ++y )
	{
		raw += char( 0 );
		for ( uint32_t x = 0; x < 3 * w; ++x )
		{
			double c = rgb[ size_t( y ) * 3 * w + x ];
			c = std::min( std::max( c, 0.0 ), 1.0 );  // util::Image<3> Component (image.hpp:29-40)
			raw += char( (unsigned char)( float( c ) * 255 ) );
		}
	}
	std::string z;
	z += char( 0x78 ), z += char( 0x01 );
	size_t off = 0;
	do
	{
		size_t n = std::min<size_t>( 65535, raw.size() - off );
		bool last = off + n == raw.size();
		z += char( last ? 1 : 0 );
		z += char( n & 0xFF ), z += char( n >> 8 ), z += char( ~n & 0xFF ), z += char( ( ~n >> 8 ) & 0xFF );
		z.append( raw, off, n );
		off += n;
	} while ( off < raw.size() );
	uint32_t a = 1, b = 0;
	for ( unsigned char c : raw ) a = ( a + c ) % 65521, b = ( b + a ) % 65521;
	put_be32( z, ( b << 16 ) | a );
	std::string out = "\x89PNG\r\n\x1a\n";
	std::string ihdr;
	put_be32( ihdr, w ), put_be32( ihdr, h );
	ihdr += char( 8 ), ihdr += char( 2 ), ihdr += char( 0 ), ihdr += char( 0 ), ihdr += char( 0 );
	png_chunk( out, "IHDR", ihdr );
	png_chunk( out, "IDAT", z );
	png_chunk( out, "IEND", "" );
	std::ofstream f( path, std::ios::binary );
	if ( !f ) fail( CR_ERR_INVALID, "cannot write " + path );
	f.write( out.data(), std::streamsize( out.size() ) );
}

void write_pfm( const std::string &path, uint32_t w, uint32_t h, const double *rgb )
{
	std::ofstream f( path, std::ios::binary );
	if ( !f ) fail( CR_ERR_INVALID, "cannot write " + path );
	f << "PF\n" << w << " " << h << "\n-1.0\n";
	std::vector<float> row( 3 * size_t( w ) );
	for ( uint32_t y = h; y-- > 0; )  // PFM rows run bottom to top
	{
		for ( size_t x = 0; x < 3 * size_t( w ); ++x ) row[ x ] = float( rgb[ size_t( y ) * 3 * w + x ] );
		f.write( (const char *)row.data(), std::streamsize( row.size() * 4 ) );
	}
}

std::string dir_of( const std::string &p )
{
	size_t k = p.find_last_of( '/' );
	return k == std::string::npos ? std::string( "." ) : p.substr( 0, k );
}

}  // namespace

// ====================================================================== internal helpers
int cr::prepare_render( cr_scene *s, const cr_render_desc *desc, DevScene &sc, RenderConfig &cfg, std::string &err )
{
	int rc = guarded( [&] {
		Resolved r = resolve( s, desc );
		sc = r.sc;
		cfg = r.cfg;
	} );
	if ( rc != CR_OK ) err = g_last_error;
	return rc;
}

void cr::set_last_error( const std::string &msg ) { g_last_error = msg; }

uint32_t cr::effective_max_bounce( const cr_scene *s, const cr_render_desc *desc )
{
	return desc->max_bounce == UINT32_MAX ? s->max_bounce : desc->max_bounce;
}

// ====================================================================== C ABI
extern "C" {

const char *cr_last_error( void ) { return g_last_error.c_str(); }
const char *cr_version( void ) { return "cr_b200 1.0 (sm_100a)"; }

int cr_trim_memory( void )
{
	return guarded( [&] { trim_device_pools(); } );
}

int cr_scene_create_empty( cr_scene **out )
{
	return guarded( [&] {
		if ( !out ) fail( CR_ERR_INVALID, "null output" );
		auto *s = new cr_scene();
		s->shader_cfg.type = Json::Object;
		*out = s;
	} );
}

int cr_scene_create( const char *json_text, const char *base_dir, cr_scene **out )
{
	return guarded( [&] {
		if ( !json_text || !out ) fail( CR_ERR_INVALID, "null argument" );
		*out = nullptr;
		std::unique_ptr<cr_scene> s( new cr_scene() );
		load_scene( s.get(), json_text, base_dir ? base_dir : "" );
		commit( s.get(), 0x330E, nullptr );
		*out = s.release();
	} );
}

int cr_scene_add_shader( cr_scene *s, const char *name, const char *config_json )
{
	int id = -1;
	int rc = guarded( [&] {
		if ( !s || !name || !config_json ) fail( CR_ERR_INVALID, "null argument" );
		if ( s->committed ) fail( CR_ERR_STATE, "scene already committed" );
		Json cfg = parse_json( config_json );
		DevShader sh = make_shader( cfg, s->shaders, name );
		auto it = s->shader_ids.find( name );
		if ( it != s->shader_ids.end() )
			s->shaders[ it->second ].second = sh, id = it->second;
		else
		{
			s->shaders.emplace_back( name, sh );
			id = int( s->shaders.size() - 1 );
			s->shader_ids[ name ] = id;
		}
	} );
	return rc == CR_OK ? id : rc;
}

int cr_scene_add_mesh( cr_scene *s, const float *v, uint32_t nv, const float *n, const uint32_t *idx, uint32_t nt,
					   const char *shader )
{
	int id = -1;
	int rc = guarded( [&] {
		if ( !s || !shader ) fail( CR_ERR_INVALID, "null argument" );
		id = add_mesh( s, v, nv, n, idx, nt, shader_id( s, shader ) );
	} );
	return rc == CR_OK ? id : rc;
}

int cr_scene_add_sphere( cr_scene *s, const float *c, float r, const char *shader )
{
	int id = -1;
	int rc = guarded( [&] {
		if ( !s || !c || !shader ) fail( CR_ERR_INVALID, "null argument" );
		if ( s->committed ) fail( CR_ERR_STATE, "scene already committed" );
		if ( !( r > 0 ) || !std::isfinite( r ) ) fail( CR_ERR_INVALID, "sphere radius must be positive" );
		HostSphere hs;
		std::memcpy( hs.c, c, sizeof hs.c );
		hs.r = r;
		hs.shader = shader_id( s, shader );
		s->spheres.push_back( hs );
		s->prims.push_back( HostPrim{ 1, int( s->spheres.size() - 1 ) } );
		id = int( s->prims.size() - 1 );
	} );
	return rc == CR_OK ? id : rc;
}

int cr_scene_add_point_light( cr_scene *s, const float *position, const float *color, float strength )
{
	int id = -1;
	int rc = guarded( [&] {
		if ( !s || !position ) fail( CR_ERR_INVALID, "null argument" );
		if ( s->committed ) fail( CR_ERR_STATE, "scene already committed" );
		DevLight L;
		std::memset( &L, 0, sizeof L );
		L.kind = LIGHT_POINT;
		std::memcpy( L.pos, position, sizeof L.pos );
		for ( int k = 0; k < 3; ++k ) L.emission[ k ] = ( color ? color[ k ] : 1.f ) * strength;
		s->point_lights.push_back( L );
		id = int( s->point_lights.size() - 1 );
	} );
	return rc == CR_OK ? id : rc;
}

int cr_scene_set_camera( cr_scene *s, const float *pos, const float *target, const float *up, float fovx )
{
	return guarded( [&] {
		if ( !s || !pos || !target || !up ) fail( CR_ERR_INVALID, "null argument" );
		std::memcpy( s->cam.pos, pos, 12 );
		std::memcpy( s->cam.target, target, 12 );
		std::memcpy( s->cam.up, up, 12 );
		s->cam.fovx = fovx;
		s->cam.lens = 0;
		s->has_camera = true;
	} );
}

int cr_scene_set_lens( cr_scene *s, int lens )
{
	return guarded( [&] {
		if ( !s ) fail( CR_ERR_INVALID, "null scene" );
		if ( lens != CR_LENS_PINHOLE && lens != CR_LENS_ORTHOGRAPHIC ) fail( CR_ERR_INVALID, "unknown lens type" );
		s->cam.lens = lens;
	} );
}

int cr_scene_commit( cr_scene *s, uint64_t light_seed, void *stream )
{
	return guarded( [&] {
		if ( !s ) fail( CR_ERR_INVALID, "null scene" );
		commit( s, light_seed, (cudaStream_t)stream );
	} );
}

int cr_bvh_build( cr_scene *s ) { return cr_scene_commit( s, 0x330E, nullptr ); }

int cr_scene_info( const cr_scene *s, uint64_t *nt, uint32_t *np, uint32_t *nl, uint32_t *nn )
{
	return guarded( [&] {
		if ( !s ) fail( CR_ERR_INVALID, "null scene" );
		if ( nt ) *nt = s->n_tris;
		if ( np ) *np = uint32_t( s->prims.size() );
		if ( nl ) *nl = uint32_t( s->lights.size() );
		if ( nn ) *nn = s->bvh.n_nodes;
	} );
}

void cr_scene_destroy( cr_scene *s ) { delete s; }

int cr_light_table( const cr_scene *s, uint32_t light, float *out, float *pdf )
{
	return guarded( [&] {
		if ( !s || !out ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		if ( light >= s->lights.size() ) fail( CR_ERR_INVALID, "no such light" );
		const DevLight &L = s->lights[ light ];
		if ( L.kind != LIGHT_MESH ) fail( CR_ERR_INVALID, "light is not a mesh light" );
		for ( int i = 0; i < 1024; ++i )
		{
			const float4 &p = s->tables_host[ 2 * ( L.table + i ) ], &n = s->tables_host[ 2 * ( L.table + i ) + 1 ];
			float v[ 6 ] = { p.x, p.y, p.z, n.x, n.y, n.z };
			std::memcpy( out + 6 * i, v, sizeof v );
		}
		if ( pdf ) *pdf = L.koishi_pdf;
	} );
}

int cr_scene_set_light_table( cr_scene *s, uint32_t primitive, const float *points, float pdf )
{
	return guarded( [&] {
		if ( !s || !points ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		if ( primitive >= s->prim_light.size() || s->prim_light[ primitive ] < 0 )
			fail( CR_ERR_INVALID, "primitive is not an emissive mesh" );
		const uint32_t light = uint32_t( s->prim_light[ primitive ] );
		DevLight &L = s->lights[ light ];
		if ( L.kind != LIGHT_MESH ) fail( CR_ERR_INVALID, "primitive is not an emissive mesh" );
		if ( !( pdf > 0.f ) || !std::isfinite( pdf ) ) fail( CR_ERR_INVALID, "light table pdf must be positive" );
		for ( int i = 0; i < 1024; ++i )
		{
			const float *q = points + 6 * i;
			for ( int k = 0; k < 6; ++k )
				if ( !std::isfinite( q[ k ] ) ) fail( CR_ERR_INVALID, "light table point is not finite" );
			s->tables_host[ 2 * ( L.table + i ) ] = make_float4( q[ 0 ], q[ 1 ], q[ 2 ], 0.f );
			s->tables_host[ 2 * ( L.table + i ) + 1 ] = make_float4( q[ 3 ], q[ 4 ], q[ 5 ], 0.f );
		}
		L.koishi_pdf = pdf;
		cuda_check( cudaMemcpy( s->light_tables.p + 2 * size_t( L.table ), &s->tables_host[ 2 * size_t( L.table ) ],
								sizeof( float4 ) * 2048, cudaMemcpyHostToDevice ),
					"light table upload" );
		cuda_check( cudaMemcpy( s->dlights.p + light, &L, sizeof( DevLight ), cudaMemcpyHostToDevice ), "light upload" );
	} );
}

int cr_trace_rays_device( cr_scene *s, const float *d_rays, uint64_t n, cr_hit *d_hits, int any_hit, void *stream )
{
	return guarded( [&] {
		if ( !s || ( n && ( !d_rays || !d_hits ) ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		launch_trace( dev_scene( s ), d_rays, n, any_hit, d_hits, s->err.p, (cudaStream_t)stream );
	} );
}

int cr_trace_rays( cr_scene *s, const float *rays, uint64_t n, cr_hit *hits, int any_hit )
{
	return guarded( [&] {
		if ( !s || ( n && ( !rays || !hits ) ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		if ( !n ) return;
		cudaStream_t st = s->stream;
		float *dr = nullptr;
		cr_hit *dh = nullptr;
		cuda_check( cudaMallocAsync( (void **)&dr, sizeof( float ) * 7 * n, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&dh, sizeof( cr_hit ) * n, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMemcpyAsync( dr, rays, sizeof( float ) * 7 * n, cudaMemcpyHostToDevice, st ), "upload" );
		launch_trace( dev_scene( s ), dr, n, any_hit, dh, s->err.p, st );
		cuda_check( cudaMemcpyAsync( hits, dh, sizeof( cr_hit ) * n, cudaMemcpyDeviceToHost, st ), "download" );
		cudaFreeAsync( dr, st );
		cudaFreeAsync( dh, st );
		cuda_check( cudaStreamSynchronize( st ), "trace" );
		uint32_t e = 0;
		cuda_check( cudaMemcpy( &e, s->err.p, 4, cudaMemcpyDeviceToHost ), "error word" );
		if ( e ) fail( CR_ERR_DEVICE, "a traversal kernel reported error flags " + std::to_string( e ) );
	} );
}

int cr_trace_work( cr_scene *s, const float *rays, uint64_t n, int any_hit, uint64_t work[ 2 ] )
{
	return guarded( [&] {
		if ( !s || !work || ( n && !rays ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		work[ 0 ] = work[ 1 ] = 0;
		if ( !n ) return;
		cudaStream_t st = s->stream;
		float *dr = nullptr;
		cr_hit *dh = nullptr;
		unsigned long long *dw = nullptr;
		cuda_check( cudaMallocAsync( (void **)&dr, sizeof( float ) * 7 * n, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&dh, sizeof( cr_hit ) * n, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&dw, sizeof( unsigned long long ) * 2, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMemsetAsync( dw, 0, sizeof( unsigned long long ) * 2, st ), "memset" );
		cuda_check( cudaMemcpyAsync( dr, rays, sizeof( float ) * 7 * n, cudaMemcpyHostToDevice, st ), "upload" );
		launch_trace( dev_scene( s ), dr, n, any_hit, dh, s->err.p, st, dw );
		unsigned long long w[ 2 ];
		cuda_check( cudaMemcpyAsync( w, dw, sizeof w, cudaMemcpyDeviceToHost, st ), "download" );
		cudaFreeAsync( dr, st );
		cudaFreeAsync( dh, st );
		cudaFreeAsync( dw, st );
		cuda_check( cudaStreamSynchronize( st ), "trace" );
		uint32_t e = 0;
		cuda_check( cudaMemcpy( &e, s->err.p, 4, cudaMemcpyDeviceToHost ), "error word" );
		if ( e ) fail( CR_ERR_DEVICE, "a traversal kernel reported error flags " + std::to_string( e ) );
		work[ 0 ] = w[ 0 ], work[ 1 ] = w[ 1 ];
	} );
}

int cr_guide_train( cr_scene *s, const cr_render_desc *desc, void *stream, uint32_t *passes )
{
	return guarded( [&] {
		if ( !s || !desc ) fail( CR_ERR_INVALID, "null argument" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		GuideState &g = s->guide;
		if ( g.max_steps == 0 ) fail( CR_ERR_INVALID, "the guide has no training budget (max_steps 0)" );
		cr_render_desc d = *desc;
		d.guiding = 1;
		d.estimator = CR_ESTIMATOR_MIS;
		uint32_t x0 = d.x0, y0 = d.y0, x1 = d.x1, y1 = d.y1;
		if ( !x0 && !y0 && !x1 && !y1 ) x1 = d.width, y1 = d.height;
		if ( x1 > d.width || y1 > d.height || x0 >= x1 || y0 >= y1 ) fail( CR_ERR_INVALID, "bad pixel window" );
		const uint64_t npx = uint64_t( x1 - x0 ) * ( y1 - y0 );
		// a pass of about one wave's recorded paths, recorded whole
		const uint64_t want = uint64_t( g.steps_per_wave ) * g.train_paths;
		d.spp = uint32_t( std::max<uint64_t>( 1, std::min<uint64_t>( ( want + npx - 1 ) / npx, 1u << 16 ) ) );
		cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
		double *sum = nullptr, *sq = nullptr;
		uint32_t *cnt = nullptr;
		cuda_check( cudaMallocAsync( (void **)&sum, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&sq, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&cnt, npx * 4, device_pool(), st ), "cudaMalloc" );
		uint32_t k = 0;
		try
		{
			// the first pass sets the guide up if it has none; every pass takes at
			// least one step, so the loop ends within the budget's count
			for ( uint32_t guard = 0; g.step < g.max_steps && guard < g.max_steps; ++guard, ++k )
			{
				render_device( s, &d, sum, sq, cnt, st, nullptr );
				d.seed += 0x9E3779B97F4A7C15ull;
			}
		}
		catch ( ... )
		{
			cudaFreeAsync( sum, st ), cudaFreeAsync( sq, st ), cudaFreeAsync( cnt, st );
			throw;
		}
		cudaFreeAsync( sum, st ), cudaFreeAsync( sq, st ), cudaFreeAsync( cnt, st );
		check_device_error( s, st );
		if ( passes ) *passes = k;
	} );
}

int cr_render_device( cr_scene *s, const cr_render_desc *desc, double *d_sum, double *d_sq, uint32_t *d_cnt,
					  void *stream, cr_stats *stats )
{
	return guarded( [&] {
		if ( !d_sum || !d_sq || !d_cnt ) fail( CR_ERR_INVALID, "null film" );
		render_device( s, desc, d_sum, d_sq, d_cnt, (cudaStream_t)stream, stats );
	} );
}

int cr_render( cr_scene *s, const cr_render_desc *desc, double *film, cr_stats *stats )
{
	return guarded( [&] {
		if ( !film ) fail( CR_ERR_INVALID, "null film" );
		Resolved r = resolve( s, desc );
		cudaStream_t st = s->stream;
		size_t npx = size_t( r.cfg.ww ) * r.cfg.wh;
		double *sum, *sq;
		uint32_t *cnt;
		cuda_check( cudaMallocAsync( (void **)&sum, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&sq, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&cnt, npx * 4, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMemsetAsync( sum, 0, npx * 24, st ), "memset" );
		cuda_check( cudaMemsetAsync( sq, 0, npx * 24, st ), "memset" );
		cuda_check( cudaMemsetAsync( cnt, 0, npx * 4, st ), "memset" );
		std::vector<uint32_t> hc( npx );
		try
		{
			render_device( s, desc, sum, sq, cnt, st, stats );
			cuda_check( cudaMemcpyAsync( film, sum, npx * 24, cudaMemcpyDeviceToHost, st ), "download" );
			cuda_check( cudaMemcpyAsync( hc.data(), cnt, npx * 4, cudaMemcpyDeviceToHost, st ), "download" );
			cuda_check( cudaStreamSynchronize( st ), "render" );
		}
		catch ( ... )
		{
			cudaFreeAsync( sum, st ), cudaFreeAsync( sq, st ), cudaFreeAsync( cnt, st );
			throw;
		}
		cudaFreeAsync( sum, st ), cudaFreeAsync( sq, st ), cudaFreeAsync( cnt, st );
		check_device_error( s, st );
		for ( size_t p = 0; p < npx; ++p )
			for ( int c = 0; c < 3; ++c ) film[ 3 * p + c ] = hc[ p ] ? film[ 3 * p + c ] / hc[ p ] : 0.0;
	} );
}

int cr_render_profile( cr_scene *s, const cr_render_desc *desc, uint32_t depth, cr_profile_slice *slices,
					   cr_profile_bounce *bounces, double *film )
{
	return guarded( [&] {
		if ( !slices || ( depth && !bounces ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( depth > 64 ) fail( CR_ERR_INVALID, "profile depth must be at most 64" );
		Resolved r = resolve( s, desc );
		if ( r.cfg.estimator != EST_KOISHI || r.cfg.kernel != KERNEL_RADIANCE || r.cfg.guiding )
			fail( CR_ERR_UNSUPPORTED, "the profile is RadianceKernel's: the Radiance kernel with the reference estimator" );
		const uint64_t n = r.samples;
		if ( n * std::max<uint64_t>( depth, 1 ) > ( 1ull << 28 ) )
			fail( CR_ERR_INVALID, "profile too large: at most 2^28 bounce records" );
		cudaStream_t st = s->stream;
		const size_t npx = size_t( r.cfg.ww ) * r.cfg.wh;
		ProfileDev pd;
		pd.depth = depth;
		double *sum = nullptr, *sq = nullptr;
		uint32_t *cnt = nullptr;
		auto release = [&] {  // once: the pointers are cleared
			for ( void *p : { (void *)pd.slices, (void *)pd.bounces, (void *)sum, (void *)sq, (void *)cnt } )
				if ( p ) cudaFreeAsync( p, st );
			pd.slices = nullptr, pd.bounces = nullptr, sum = nullptr, sq = nullptr, cnt = nullptr;
		};
		try
		{
			cuda_check( cudaMallocAsync( (void **)&pd.slices, sizeof( cr_profile_slice ) * n, device_pool(), st ), "cudaMalloc" );
			cuda_check( cudaMemsetAsync( pd.slices, 0, sizeof( cr_profile_slice ) * n, st ), "memset" );
			// at depth 0 no record is written; one keeps the buffer valid
			const size_t nb = std::max<size_t>( n * depth, 1 );
			cuda_check( cudaMallocAsync( (void **)&pd.bounces, sizeof( cr_profile_bounce ) * nb, device_pool(), st ), "cudaMalloc" );
			cuda_check( cudaMemsetAsync( pd.bounces, 0, sizeof( cr_profile_bounce ) * nb, st ), "memset" );
			cuda_check( cudaMallocAsync( (void **)&sum, npx * 24, device_pool(), st ), "cudaMalloc" );
			cuda_check( cudaMallocAsync( (void **)&sq, npx * 24, device_pool(), st ), "cudaMalloc" );
			cuda_check( cudaMallocAsync( (void **)&cnt, npx * 4, device_pool(), st ), "cudaMalloc" );
			cuda_check( cudaMemsetAsync( sum, 0, npx * 24, st ), "memset" );
			cuda_check( cudaMemsetAsync( sq, 0, npx * 24, st ), "memset" );
			cuda_check( cudaMemsetAsync( cnt, 0, npx * 4, st ), "memset" );
			r.cfg.prof = pd;
			ensure_wave( s, r.cfg.wave_paths, r.cfg.max_bounce, st, false, r.cfg.bin_rays );
			render_waves( r.sc, r.cfg, s->wave, sum, sq, cnt, st, nullptr, &s->guide );
			cuda_check( cudaMemcpyAsync( slices, pd.slices, sizeof( cr_profile_slice ) * n, cudaMemcpyDeviceToHost, st ),
						"download" );
			if ( depth )
				cuda_check( cudaMemcpyAsync( bounces, pd.bounces, sizeof( cr_profile_bounce ) * n * depth,
											 cudaMemcpyDeviceToHost, st ),
							"download" );
			std::vector<uint32_t> hc( npx );
			std::vector<double> hs( film ? npx * 3 : 0 );
			if ( film )
			{
				cuda_check( cudaMemcpyAsync( hs.data(), sum, npx * 24, cudaMemcpyDeviceToHost, st ), "download" );
				cuda_check( cudaMemcpyAsync( hc.data(), cnt, npx * 4, cudaMemcpyDeviceToHost, st ), "download" );
			}
			cuda_check( cudaStreamSynchronize( st ), "profile" );
			release();
			check_device_error( s, st );
			if ( film )
				for ( size_t p = 0; p < npx; ++p )
					for ( int c = 0; c < 3; ++c ) film[ 3 * p + c ] = hc[ p ] ? hs[ 3 * p + c ] / hc[ p ] : 0.0;
		}
		catch ( ... )
		{
			release();
			throw;
		}
	} );
}

// Profiler::~Profiler (src/core/kernel/kernel.cu) and
// RadianceKernel::Slice::writeSlice (src/core/kernel/radiance.hpp:31-47): the
// reference's text, with its vectors printed as "[ x, y, z ]" (vec.hpp:220-251)
// and numbers in the stream's default format.
static void write_profile( std::ostream &os, const uint32_t area[ 4 ], uint32_t spp, uint32_t depth,
						   const cr_profile_slice *slices, const cr_profile_bounce *bounces )
{
	auto v3 = [&]( const float *v ) { os << "[ " << v[ 0 ] << ", " << v[ 1 ] << ", " << v[ 2 ] << " ]"; };
	const uint32_t aw = area[ 2 ] - area[ 0 ], ah = area[ 3 ] - area[ 1 ];
	for ( uint32_t y = 0; y != ah; ++y )
		for ( uint32_t x = 0; x != aw; ++x )
			for ( uint32_t k = 0; k != spp; ++k )
			{
				os << "at [ " << x + area[ 0 ] << ", " << y + area[ 1 ] << ", " << k << " ]: " << std::endl;
				const size_t si = ( size_t( aw ) * y + x ) * spp + k;
				const cr_profile_slice &sl = slices[ si ];
				if ( sl.L[ 0 ] >= 1e2f && sl.L[ 1 ] >= 1e2f && sl.L[ 2 ] >= 1e2f )
				{
					os << "bounce: " << size_t( sl.bounce ) << " / " << size_t( depth ) << std::endl;
					for ( uint32_t i = 0; i != std::min( sl.bounce, depth ); ++i )
					{
						const cr_profile_bounce &b = bounces[ si * depth + i ];
						os << "ray: ";
						v3( b.ray_o );
						v3( b.ray_d );
						os << std::endl << "f: ";
						v3( b.f );
						os << std::endl << "theta: " << b.theta << std::endl << "L: ";
						v3( b.L );
						os << std::endl << "shader: " << b.shader << std::endl;
					}
				}
			}
}

int cr_profile_write( const char *path, const uint32_t area[ 4 ], uint32_t spp, uint32_t depth,
					  const cr_profile_slice *slices, const cr_profile_bounce *bounces )
{
	return guarded( [&] {
		if ( !path || !area || !slices || ( depth && !bounces ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( area[ 2 ] < area[ 0 ] || area[ 3 ] < area[ 1 ] ) fail( CR_ERR_INVALID, "bad profile area" );
		std::ofstream of( path );
		if ( !of ) fail( CR_ERR_INVALID, std::string( "cannot write " ) + path );
		write_profile( of, area, spp, depth, slices, bounces );
		if ( !of ) fail( CR_ERR_INVALID, std::string( "write failed: " ) + path );
	} );
}

int cr_autotune( cr_scene *s, const cr_render_desc *desc, void *stream, cr_tuning *out )
{
	return guarded( [&] {
		if ( !out ) fail( CR_ERR_INVALID, "null output" );
		Resolved base = resolve( s, desc );
		cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
		// Sample render: a band of 1/8 of the window's rows around its middle,
		// at the request's spp capped at 64.
		RenderConfig cfg = base.cfg;
		uint32_t band = std::max<uint32_t>( 1, cfg.wh / 8 );
		cfg.y0 = cfg.y0 + ( cfg.wh - band ) / 2;
		cfg.wh = band;
		uint32_t spp = std::min<uint32_t>( cfg.spp, 64 );
		DevScene sc = base.sc;
		if ( spp != cfg.spp ) sc.cam = make_camera( s->cam, sc.cam.width, sc.cam.height, spp );
		cfg.spp = spp;
		cfg.count_work = false;
		cfg.guiding = false;
		uint64_t samples = uint64_t( cfg.ww ) * cfg.wh * cfg.spp;
		size_t npx = size_t( cfg.ww ) * cfg.wh;
		double *sum, *sq;
		uint32_t *cnt;
		cuda_check( cudaMallocAsync( (void **)&sum, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&sq, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&cnt, npx * 4, device_pool(), st ), "cudaMalloc" );
		uint32_t tried = 0, shade = 128, svote = 4, srefill = 0;
		bool bin = false;
		auto rate = [&]( uint32_t wave, uint32_t refill, int blocks ) {
			RenderConfig c = cfg;
			c.wave_paths = uint32_t( std::min<uint64_t>( wave, samples ) );
			c.refill_min = refill;
			c.traverse_blocks_per_sm = blocks;
			c.shade_threads = shade;
			c.bin_rays = bin;
			c.shadow_vote = svote, c.shadow_refill_min = srefill;
			ensure_wave( s, c.wave_paths, c.max_bounce, st, false, bin );
			StageTimes warm, t;
			render_waves( sc, c, s->wave, sum, sq, cnt, st, &warm );
			render_waves( sc, c, s->wave, sum, sq, cnt, st, &t );
			++tried;
			return double( samples ) / ( t.total * 1e3 );
		};
		uint32_t wave = 1u << 22, refill = 16;
		int blocks = 8;
		double best = rate( wave, refill, blocks );
		double dflt = best;
		for ( uint32_t r : { 4u, 8u, 12u, 24u, 32u } )
		{
			double v = rate( wave, r, blocks );
			if ( v > best ) best = v, refill = r;
		}
		for ( int b : { 4, 6 } )
		{
			double v = rate( wave, refill, b );
			if ( v > best ) best = v, blocks = b;
		}
		// the shading kernel's block size (its grid keeps 1024 threads per SM)
		for ( uint32_t t : { 64u, 256u } )
		{
			const uint32_t keep = shade;
			shade = t;
			double v = rate( wave, refill, blocks );
			if ( v > best )
				best = v;
			else
				shade = keep;
		}
		// the any-hit traversal's own triangle vote and refill threshold
		for ( uint32_t v : { 2u, 8u, 32u } )
		{
			const uint32_t keep = svote;
			svote = v;
			double r = rate( wave, refill, blocks );
			if ( r > best )
				best = r;
			else
				svote = keep;
		}
		for ( uint32_t f : { 4u, 8u, 16u, 24u } )
		{
			if ( f == refill ) continue;
			const uint32_t keep = srefill;
			srefill = f;
			double r = rate( wave, refill, blocks );
			if ( r > best )
				best = r;
			else
				srefill = keep;
		}
		// ray binning before the secondary and shadow traversals
		{
			bin = true;
			double v = rate( wave, refill, blocks );
			if ( v > best )
				best = v;
			else
				bin = false;
		}
		for ( uint32_t w : { 1u << 20, 1u << 21, 1u << 23 } )
		{
			if ( w > samples && wave >= samples ) continue;
			double v = rate( w, refill, blocks );
			if ( v > best ) best = v, wave = w;
		}
		// HBM-sized waves (about 140 bytes of state per path): keep doubling
		// while the sample holds that many paths, memory allows, and it pays
		for ( uint32_t w = 1u << 24; w <= ( 1u << 26 ) && wave == w / 2 && w <= samples && wave_fits( w, cfg.max_bounce ); w *= 2 )
		{
			double v = rate( w, refill, blocks );
			if ( v > best ) best = v, wave = w;
		}
		cudaFreeAsync( sum, st ), cudaFreeAsync( sq, st ), cudaFreeAsync( cnt, st );
		cuda_check( cudaStreamSynchronize( st ), "autotune" );
		s->tune_wave = wave, s->tune_refill = refill, s->tune_blocks = blocks, s->tune_shade = shade;
		s->tune_bin = bin;
		s->tune_svote = svote, s->tune_srefill = srefill;
		out->wave_paths = wave, out->refill_min = refill, out->traverse_blocks_per_sm = uint32_t( blocks );
		out->shade_threads = shade;
		out->bin_rays = bin ? 1 : -1;
		out->shadow_vote = svote, out->shadow_refill_min = srefill ? srefill : refill;
		out->candidates_tried = tried;
		out->msamples_per_s = best;
		out->default_msamples_per_s = dflt;
	} );
}

// ------------------------------------------------------------------ batches
struct cr_batch
{
	std::vector<cr_batch_job> req;   // the caller's job table
	std::vector<BatchJobDev> jobs;   // host copy of the device table
	DevScene *d_scenes = nullptr;
	BatchJobDev *d_jobs = nullptr;
	uint64_t *d_seed = nullptr;
	uint64_t total = 0;              // samples per render
	uint32_t max_bounce = 7;
	int estimator = EST_KOISHI;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	WaveBuffers wave;
	uint32_t wave_bounces = 0;
	uint32_t tune_wave = 1u << 22, tune_refill = 16;
	int tune_blocks = 8;
	uint32_t tune_shade = 128;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	uint32_t graph_nodes = 0;  // kernel nodes of the graph, its loop body counted once

	void drop_graph()
	{
		if ( exec ) cudaGraphExecDestroy( exec );
		if ( graph ) cudaGraphDestroy( graph );
		exec = nullptr, graph = nullptr;
	}
	~cr_batch()
	{
		drop_graph();
		if ( wave.capacity ) free_wave( wave, stream );
		if ( stream ) cudaStreamSynchronize( stream );
		for ( void *p : { (void *)d_scenes, (void *)d_jobs, (void *)d_seed } )
			if ( p ) cudaFree( p );
		if ( own_stream && stream ) cudaStreamDestroy( stream );
	}
};

namespace
{
// Device scene and job tables of a batch, every job at spp / spp_div (>= 1);
// films: the caller's, or `films` (sum, sumsq, count base pointers laid out job
// after job) when not null.
void batch_tables( const cr_batch *b, uint32_t spp_div, double *films_sum, double *films_sq, uint32_t *films_cnt,
				   std::vector<BatchJobDev> &jobs, std::vector<DevScene> &scenes )
{
	jobs.clear(), scenes.clear();
	uint64_t fs = 0, fp = 0;
	for ( const cr_batch_job &r : b->req )
	{
		BatchJobDev j{};
		j.width = r.width, j.height = r.height, j.spp = std::max<uint32_t>( 1, r.spp / spp_div );
		j.first_sample = fs, j.first_pixel = fp, j.seed = r.seed;
		if ( films_sum )
			j.sum = films_sum + 3 * fp, j.sumsq = films_sq + 3 * fp, j.count = films_cnt + fp;
		else
			j.sum = r.d_sum, j.sumsq = r.d_sumsq, j.count = r.d_count;
		DevScene sc = dev_scene( r.scene );
		sc.cam = make_camera( r.scene->cam, r.width, r.height, j.spp );
		jobs.push_back( j ), scenes.push_back( sc );
		fs += uint64_t( r.width ) * r.height * j.spp;
		fp += uint64_t( r.width ) * r.height;
	}
}

void upload( void *dst, const void *src, size_t bytes, cudaStream_t st )
{
	cuda_check( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyHostToDevice, st ), "batch upload" );
}

void batch_ensure_wave( cr_batch *b, uint32_t cap )
{
	if ( !( b->wave.capacity >= cap && b->wave_bounces >= b->max_bounce ) )
	{
		if ( b->wave.capacity ) free_wave( b->wave, b->stream );
		alloc_wave( b->wave, cap, b->max_bounce, b->stream );
		b->wave_bounces = b->max_bounce;
	}
	alloc_batch_state( b->wave, b->stream );
}

RenderConfig batch_config( const cr_batch *b, uint32_t wave, uint32_t refill, int blocks, uint64_t total,
						   uint32_t shade = 128 )
{
	RenderConfig c{};
	c.spp = 1, c.max_bounce = b->max_bounce, c.estimator = b->estimator;
	c.x0 = c.y0 = 0, c.ww = c.wh = 1, c.seed = 0;
	c.wave_paths = uint32_t( std::min<uint64_t>( wave, total ) );
	c.count_work = false;
	c.refill_min = refill, c.traverse_blocks_per_sm = blocks;
	c.shade_threads = shade;
	return c;
}

void batch_check_error( cr_batch *b )
{
	uint32_t e = 0;
	cuda_check( cudaMemcpyAsync( &e, b->wave.err, 4, cudaMemcpyDeviceToHost, b->stream ), "error word" );
	cuda_check( cudaStreamSynchronize( b->stream ), "error word" );
	if ( e ) fail( CR_ERR_DEVICE, "a batched render kernel reported error flags " + std::to_string( e ) );
}
}  // namespace

extern "C" int cr_measure_peaks_impl( void *stream, double *l2_gbs, double *fp32_tflops, const char **err );

int cr_measure_peaks( void *stream, double *l2_read_gbs, double *fp32_tflops )
{
	return guarded( [&] {
		const char *err = nullptr;
		if ( cr_measure_peaks_impl( stream, l2_read_gbs, fp32_tflops, &err ) != 0 )
			fail( CR_ERR_CUDA, err ? err : "peak measurement failed" );
	} );
}

extern "C" int cr_measure_gather_impl( void *stream, uint32_t record_bytes, uint64_t array_bytes, double *gbs,
									   const char **err );

int cr_measure_gather( void *stream, uint32_t record_bytes, uint64_t array_bytes, double *gbs )
{
	return guarded( [&] {
		const char *err = nullptr;
		if ( cr_measure_gather_impl( stream, record_bytes, array_bytes, gbs, &err ) != 0 )
			fail( CR_ERR_INVALID, err ? err : "gather measurement failed" );
	} );
}

int cr_mesh_file_info( const char *path, uint32_t *n_groups, uint64_t *n_vertices, uint64_t *n_triangles,
					   double *checksum )
{
	return guarded( [&] {
		if ( !path ) fail( CR_ERR_INVALID, "null path" );
		std::vector<Group> groups = load_mesh_file( path );
		uint64_t nv = 0, nt = 0, corner = 0;
		double cs = 0;
		for ( const Group &g : groups )
		{
			nv += g.v.size() / 3, nt += g.idx.size() / 3;
			// positions of the triangle corners, weighted by the corner's rank in
			// the whole file: sensitive to order, not to the grouping
			for ( size_t t = 0; t < g.idx.size(); ++t, ++corner )
				for ( int c = 0; c < 3; ++c ) cs += double( g.v[ 3 * size_t( g.idx[ t ] ) + c ] ) * double( ( corner % 7 ) + 1 );
		}
		if ( n_groups ) *n_groups = uint32_t( groups.size() );
		if ( n_vertices ) *n_vertices = nv;
		if ( n_triangles ) *n_triangles = nt;
		if ( checksum ) *checksum = cs;
	} );
}

int cr_scene_set_kernel( cr_scene *s, const char *name )
{
	return guarded( [&] {
		if ( !s || !name ) fail( CR_ERR_INVALID, "null argument" );
		if ( kernel_id( name ) < 0 )
			fail( CR_ERR_UNSUPPORTED, std::string( "kernel '" ) + name + "' is not registered (Radiance, Normal, Visibility, HalfVector)" );
		s->kernel = name;
	} );
}

int cr_scene_set_build( cr_scene *s, const cr_build_config *cfg )
{
	return guarded( [&] {
		if ( !s || !cfg ) fail( CR_ERR_INVALID, "null argument" );
		if ( s->committed ) fail( CR_ERR_STATE, "the BVH options must be set before cr_scene_commit" );
		if ( cfg->builder != CR_BUILD_PLOC && cfg->builder != CR_BUILD_LBVH ) fail( CR_ERR_INVALID, "unknown builder" );
		if ( cfg->max_leaf < 1 || cfg->max_leaf > 3 ) fail( CR_ERR_INVALID, "max_leaf must be in [1, 3]" );
		if ( cfg->ploc_radius < 1 || cfg->ploc_radius > 256 ) fail( CR_ERR_INVALID, "ploc_radius must be in [1, 256]" );
		if ( !( cfg->cost_node > 0.f ) || !( cfg->cost_tri > 0.f ) || !( cfg->wide_cost_node > 0.f ) ||
			 !( cfg->wide_cost_tri > 0.f ) )
			fail( CR_ERR_INVALID, "SAH costs must be positive" );
		if ( cfg->collapse != CR_COLLAPSE_SAH && cfg->collapse != CR_COLLAPSE_GREEDY ) fail( CR_ERR_INVALID, "unknown collapse" );
		s->build.ploc = cfg->builder == CR_BUILD_PLOC;
		s->build.radius = int( cfg->ploc_radius );
		s->build.max_leaf = int( cfg->max_leaf );
		s->build.cost_node = cfg->cost_node, s->build.cost_tri = cfg->cost_tri;
		s->build.dp_collapse = cfg->collapse == CR_COLLAPSE_SAH;
		s->build.dp_cost_node = cfg->wide_cost_node, s->build.dp_cost_tri = cfg->wide_cost_tri;
	} );
}

int cr_batch_create( const cr_batch_job *jobs, uint32_t n_jobs, uint32_t max_bounce, int32_t estimator, void *stream,
					 cr_batch **out )
{
	return guarded( [&] {
		if ( !out ) fail( CR_ERR_INVALID, "null output" );
		*out = nullptr;
		if ( !jobs || n_jobs == 0 ) fail( CR_ERR_INVALID, "empty batch" );
		if ( n_jobs > 65536 ) fail( CR_ERR_INVALID, "more than 65536 jobs in a batch" );
		if ( max_bounce > 1024 ) fail( CR_ERR_INVALID, "max_bounce out of range" );
		if ( estimator != EST_KOISHI && estimator != EST_MIS ) fail( CR_ERR_INVALID, "unknown estimator" );
		for ( uint32_t i = 0; i < n_jobs; ++i )
		{
			const cr_batch_job &j = jobs[ i ];
			const std::string at = "batch job " + std::to_string( i ) + ": ";
			if ( !j.scene || !j.scene->committed ) fail( CR_ERR_STATE, at + "scene missing or not committed" );
			if ( !j.scene->has_camera ) fail( CR_ERR_INVALID, at + "no camera in the scene" );
			if ( !j.width || !j.height || !j.spp ) fail( CR_ERR_INVALID, at + "width, height and spp must be positive" );
			if ( !j.d_sum || !j.d_sumsq || !j.d_count ) fail( CR_ERR_INVALID, at + "null film" );
			if ( estimator == EST_MIS && !j.scene->mis_blocker.empty() )
				fail( CR_ERR_UNSUPPORTED, at + "the MIS estimator does not cover " + j.scene->mis_blocker );
		}
		std::unique_ptr<cr_batch> b( new cr_batch );
		b->req.assign( jobs, jobs + n_jobs );
		b->max_bounce = max_bounce, b->estimator = estimator;
		if ( stream )
			b->stream = (cudaStream_t)stream;
		else
		{
			cuda_check( cudaStreamCreateWithFlags( &b->stream, cudaStreamNonBlocking ), "batch stream" );
			b->own_stream = true;
		}
		std::vector<DevScene> scenes;
		batch_tables( b.get(), 1, nullptr, nullptr, nullptr, b->jobs, scenes );
		const BatchJobDev &last = b->jobs.back();
		b->total = last.first_sample + uint64_t( last.width ) * last.height * last.spp;
		cuda_check( cudaMalloc( (void **)&b->d_scenes, sizeof( DevScene ) * n_jobs ), "cudaMalloc" );
		cuda_check( cudaMalloc( (void **)&b->d_jobs, sizeof( BatchJobDev ) * n_jobs ), "cudaMalloc" );
		cuda_check( cudaMalloc( (void **)&b->d_seed, sizeof( uint64_t ) ), "cudaMalloc" );
		upload( b->d_scenes, scenes.data(), sizeof( DevScene ) * n_jobs, b->stream );
		upload( b->d_jobs, b->jobs.data(), sizeof( BatchJobDev ) * n_jobs, b->stream );
		cuda_check( cudaMemsetAsync( b->d_seed, 0, sizeof( uint64_t ), b->stream ), "batch" );
		cuda_check( cudaStreamSynchronize( b->stream ), "batch" );
		*out = b.release();
	} );
}

int cr_batch_autotune( cr_batch *b, cr_tuning *out )
{
	return guarded( [&] {
		if ( !b || !out ) fail( CR_ERR_INVALID, "null argument" );
		cudaStream_t st = b->stream;
		uint64_t npx = b->jobs.back().first_pixel + uint64_t( b->jobs.back().width ) * b->jobs.back().height;
		double *sum = nullptr, *sq = nullptr;
		uint32_t *cnt = nullptr;
		cuda_check( cudaMallocAsync( (void **)&sum, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&sq, npx * 24, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&cnt, npx * 4, device_pool(), st ), "cudaMalloc" );
		std::vector<BatchJobDev> jobs;
		std::vector<DevScene> scenes;
		batch_tables( b, 16, sum, sq, cnt, jobs, scenes );
		const uint32_t n = uint32_t( jobs.size() );
		const uint64_t total = jobs.back().first_sample + uint64_t( jobs.back().width ) * jobs.back().height * jobs.back().spp;
		DevScene *d_scenes = nullptr;
		BatchJobDev *d_jobs = nullptr;
		cuda_check( cudaMallocAsync( (void **)&d_scenes, sizeof( DevScene ) * n, device_pool(), st ), "cudaMalloc" );
		cuda_check( cudaMallocAsync( (void **)&d_jobs, sizeof( BatchJobDev ) * n, device_pool(), st ), "cudaMalloc" );
		upload( d_scenes, scenes.data(), sizeof( DevScene ) * n, st );
		upload( d_jobs, jobs.data(), sizeof( BatchJobDev ) * n, st );
		BatchDev bd{ d_scenes, d_jobs, b->d_seed, n };
		uint32_t tried = 0;
		uint32_t shade = 128;
		auto rate = [&]( uint32_t wave, uint32_t refill, int blocks ) {
			RenderConfig c = batch_config( b, wave, refill, blocks, total, shade );
			batch_ensure_wave( b, c.wave_paths );
			StageTimes warm, t;
			render_batch_waves( bd, jobs.data(), n, c, b->wave, st, &warm );
			render_batch_waves( bd, jobs.data(), n, c, b->wave, st, &t );
			++tried;
			return double( total ) / ( t.total * 1e3 );
		};
		uint32_t wave = 1u << 22, refill = 16;
		int blocks = 8;
		double best = rate( wave, refill, blocks ), dflt = best;
		for ( uint32_t r : { 8u, 12u, 24u } )
		{
			double v = rate( wave, r, blocks );
			if ( v > best ) best = v, refill = r;
		}
		for ( int bl : { 4, 6 } )
		{
			double v = rate( wave, refill, bl );
			if ( v > best ) best = v, blocks = bl;
		}
		// the shading kernel's block size (its grid keeps 1024 threads per SM)
		for ( uint32_t t : { 64u, 256u } )
		{
			const uint32_t keep = shade;
			shade = t;
			double v = rate( wave, refill, blocks );
			if ( v > best )
				best = v;
			else
				shade = keep;
		}
		for ( uint32_t w : { 1u << 21, 1u << 23 } )
		{
			if ( w > total && wave >= total ) continue;
			double v = rate( w, refill, blocks );
			if ( v > best ) best = v, wave = w;
		}
		// HBM-sized waves: fewer waves, so fewer launches per render (and graph
		// nodes per replay); keep doubling while it pays and memory allows
		for ( uint32_t w = 1u << 24; w <= ( 1u << 26 ) && wave == w / 2 && w <= total && wave_fits( w, b->max_bounce ); w *= 2 )
		{
			double v = rate( w, refill, blocks );
			if ( v > best ) best = v, wave = w;
		}
		for ( void *p : { (void *)sum, (void *)sq, (void *)cnt, (void *)d_scenes, (void *)d_jobs } ) cudaFreeAsync( p, st );
		cuda_check( cudaStreamSynchronize( st ), "batch autotune" );
		batch_check_error( b );
		b->tune_wave = wave, b->tune_refill = refill, b->tune_blocks = blocks, b->tune_shade = shade;
		out->shade_threads = shade;
		out->bin_rays = -1;  // batches trace in queue order
		out->shadow_vote = 4, out->shadow_refill_min = refill;
		b->drop_graph();
		out->wave_paths = wave, out->refill_min = refill, out->traverse_blocks_per_sm = uint32_t( blocks );
		out->candidates_tried = tried;
		out->msamples_per_s = best;
		out->default_msamples_per_s = dflt;
	} );
}

int cr_batch_set_tuning( cr_batch *b, const cr_tuning *t )
{
	return guarded( [&] {
		if ( !b || !t ) fail( CR_ERR_INVALID, "null argument" );
		if ( t->refill_min > 32 ) fail( CR_ERR_INVALID, "refill_min must be 1..32" );
		if ( t->traverse_blocks_per_sm > 8 ) fail( CR_ERR_INVALID, "traverse_blocks_per_sm must be 1..8" );
		if ( t->shade_threads && t->shade_threads != 64 && t->shade_threads != 128 && t->shade_threads != 256 )
			fail( CR_ERR_INVALID, "shade_threads must be 64, 128 or 256" );
		if ( t->wave_paths > ( 1u << 30 ) ) fail( CR_ERR_INVALID, "wave_paths above 2^30" );
		if ( t->wave_paths ) b->tune_wave = t->wave_paths;
		if ( t->refill_min ) b->tune_refill = t->refill_min;
		if ( t->traverse_blocks_per_sm ) b->tune_blocks = int( t->traverse_blocks_per_sm );
		if ( t->shade_threads ) b->tune_shade = t->shade_threads;
		b->drop_graph();
	} );
}

int cr_batch_render( cr_batch *b, uint64_t seed_offset, cr_stats *stats )
{
	return guarded( [&] {
		if ( !b ) fail( CR_ERR_INVALID, "null batch" );
		cudaStream_t st = b->stream;
		const uint32_t n = uint32_t( b->jobs.size() );
		RenderConfig c = batch_config( b, b->tune_wave, b->tune_refill, b->tune_blocks, b->total, b->tune_shade );
		if ( !b->exec )
		{
			// one graph for the whole batch: a device-side loop over its waves
			batch_ensure_wave( b, c.wave_paths );
			cuda_check( cudaStreamSynchronize( st ), "batch" );
			BatchDev bd{ b->d_scenes, b->d_jobs, b->d_seed, n };
			b->drop_graph();  // a graph left by a failed instantiation
			b->graph_nodes = build_batch_graph( bd, b->jobs.data(), n, c, b->wave, st, &b->graph );
			cuda_check( cudaGraphInstantiate( &b->exec, b->graph, 0 ), "graph instantiate" );
		}
		upload( b->d_seed, &seed_offset, sizeof( uint64_t ), st );
		cudaEvent_t e0 = nullptr, e1 = nullptr;
		if ( stats )
		{
			cuda_check( cudaEventCreate( &e0 ), "event" ), cuda_check( cudaEventCreate( &e1 ), "event" );
			cuda_check( cudaEventRecord( e0, st ), "event" );
		}
		cudaError_t le = cudaGraphLaunch( b->exec, st );
		if ( stats )
		{
			cudaEventRecord( e1, st );
			cudaError_t se = cudaEventSynchronize( e1 );
			float ms = 0.f;
			if ( le == cudaSuccess && se == cudaSuccess ) cudaEventElapsedTime( &ms, e0, e1 );
			cudaEventDestroy( e0 ), cudaEventDestroy( e1 );
			cuda_check( le, "graph launch" );
			cuda_check( se, "batched render" );
			batch_check_error( b );
			unsigned long long t[ 2 ] = { 0, 0 };
			cuda_check( cudaMemcpy( t, b->wave.tally, sizeof t, cudaMemcpyDeviceToHost ), "tally" );
			StageTimes tm;
			tm.total = ms, tm.rays_extend = t[ 0 ], tm.rays_shadow = t[ 1 ];
			tm.waves = uint32_t( ( b->total + c.wave_paths - 1 ) / c.wave_paths );
			// the body's kernels run once per wave, after the initialising one
			tm.launches = 1 + tm.waves * ( b->graph_nodes - 1 );
			fill_stats( stats, tm, b->total );
			stats->graph_nodes = b->graph_nodes;
		}
		else
			cuda_check( le, "graph launch" );
	} );
}

void cr_batch_destroy( cr_batch *b ) { delete b; }

int cr_guide_reset( cr_scene *s, uint64_t seed )
{
	return guarded( [&] {
		if ( !s ) fail( CR_ERR_INVALID, "null scene" );
		if ( !s->committed ) fail( CR_ERR_STATE, "scene not committed" );
		s->guide.init( s->box_lo, s->box_hi, seed );
	} );
}

int cr_guide_info( const cr_scene *s, float *bmin, float *binv, uint32_t *step, uint32_t *sizes )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		if ( bmin ) bmin[ 0 ] = s->guide.bmin.x, bmin[ 1 ] = s->guide.bmin.y, bmin[ 2 ] = s->guide.bmin.z;
		if ( binv ) binv[ 0 ] = s->guide.binv.x, binv[ 1 ] = s->guide.binv.y, binv[ 2 ] = s->guide.binv.z;
		if ( step ) *step = s->guide.step;
		if ( sizes )
			sizes[ 0 ] = uint32_t( GuideState::grid_size() ), sizes[ 1 ] = uint32_t( GuideState::w_size() ),
			sizes[ 2 ] = uint32_t( GuideState::b_size() );
	} );
}

int cr_guide_configure( cr_scene *s, const cr_guide_config *in, cr_guide_config *out )
{
	return guarded( [&] {
		if ( !s ) fail( CR_ERR_INVALID, "null scene" );
		GuideState &g = s->guide;
		if ( in )
		{
			if ( !( in->lr > 0.f && in->lr < 1.f ) ) fail( CR_ERR_INVALID, "guide lr must be in (0, 1)" );
			if ( !( in->select_prob >= 0.f && in->select_prob < 1.f ) )
				fail( CR_ERR_INVALID, "guide select_prob must be in [0, 1)" );
			if ( in->train_paths < 1 || in->train_paths > ( 1u << 20 ) )
				fail( CR_ERR_INVALID, "guide train_paths must be in [1, 2^20]" );
			if ( in->steps_per_wave < 1 || in->steps_per_wave > 64 )
				fail( CR_ERR_INVALID, "guide steps_per_wave must be in [1, 64]" );
			g.lr = in->lr, g.select_prob = in->select_prob, g.train_paths = in->train_paths;
			g.steps_per_wave = in->steps_per_wave, g.warmup_steps = in->warmup_steps;
			g.product_target = in->product_target != 0;
			g.max_steps = in->max_steps;
			g.guided_bounces = in->guided_bounces;
			g.learn_select = in->learn_select != 0;
		}
		if ( out )
		{
			out->lr = g.lr, out->select_prob = g.select_prob, out->train_paths = g.train_paths;
			out->steps_per_wave = g.steps_per_wave, out->warmup_steps = g.warmup_steps;
			out->product_target = g.product_target ? 1u : 0u;
			out->max_steps = g.max_steps;
			out->guided_bounces = g.guided_bounces;
			out->learn_select = g.learn_select ? 1u : 0u;
		}
	} );
}

int cr_guide_loss( const cr_scene *s, float *loss )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		if ( !loss ) fail( CR_ERR_INVALID, "null argument" );
		cuda_check( cudaMemcpy( loss, s->guide.loss, 4, cudaMemcpyDeviceToHost ), "guide loss" );
	} );
}

int cr_guide_params( cr_scene *s, float *grid, float *W, float *b, int set )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		auto io = [&]( float *host, float *dev, size_t n ) {
			if ( !host ) return;
			cuda_check( set ? cudaMemcpy( dev, host, n * 4, cudaMemcpyHostToDevice )
							: cudaMemcpy( host, dev, n * 4, cudaMemcpyDeviceToHost ),
						"guide params" );
		};
		io( grid, s->guide.grid, GuideState::grid_size() );
		io( W, s->guide.W, GuideState::w_size() );
		io( b, s->guide.b, GuideState::b_size() );
		if ( set ) s->guide.packed_step = ~0u;  // the tensor-core weight image is stale
	} );
}

int cr_guide_forward( cr_scene *s, const float *inputs, uint64_t n, float *out )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		if ( !n ) return;
		if ( !inputs || !out ) fail( CR_ERR_INVALID, "null argument" );
		float *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( float ) * ( 9 + G_OUT ) * n ), "cudaMalloc" );
		cudaMemcpy( d, inputs, sizeof( float ) * 9 * n, cudaMemcpyHostToDevice );
		s->guide.forward_batch( d, uint32_t( n ), d + 9 * n, nullptr );
		cudaError_t e = cudaMemcpy( out, d + 9 * n, sizeof( float ) * G_OUT * n, cudaMemcpyDeviceToHost );
		cudaFree( d );
		cuda_check( e, "guide forward" );
	} );
}

int cr_guide_forward_tc( cr_scene *s, const float *inputs, uint64_t n, float *out )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		if ( !n ) return;
		if ( !inputs || !out ) fail( CR_ERR_INVALID, "null argument" );
		if ( n > ( 1ull << 31 ) ) fail( CR_ERR_INVALID, "too many inputs" );
		// outputs after the inputs, at a 256-byte boundary: the kernel stores them as float4
		const size_t out_off = ( 9 * n + 63 ) / 64 * 64;
		float *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( float ) * ( out_off + G_OUT * n ) ), "cudaMalloc" );
		uint32_t e = 0;
		try
		{
			cuda_check( cudaMemcpy( d, inputs, sizeof( float ) * 9 * n, cudaMemcpyHostToDevice ), "guide forward" );
			e = s->guide.forward_batch_tc( d, uint32_t( n ), d + out_off, nullptr );
			cuda_check( cudaMemcpy( out, d + out_off, sizeof( float ) * G_OUT * n, cudaMemcpyDeviceToHost ), "guide forward" );
		}
		catch ( ... )
		{
			cudaFree( d );
			throw;
		}
		cudaFree( d );
		if ( e ) fail( CR_ERR_DEVICE, "guide tensor-core forward: an MMA wait timed out (error word " + std::to_string( e ) + ")" );
	} );
}

namespace
{
int guide_gradients( cr_scene *s, const float *records, uint64_t n, float *gW, float *gb, float *ggrid, bool tc )
{
	return guarded( [&] {
		if ( !s || !s->guide.ready ) fail( CR_ERR_STATE, "no guide on this scene (cr_guide_reset first)" );
		if ( !n || !records ) fail( CR_ERR_INVALID, "no records" );
		GuideState &g = s->guide;
		const uint32_t stride = g.learn_select ? 14u : 13u;
		float *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( float ) * stride * n ), "cudaMalloc" );
		cudaMemcpy( d, records, sizeof( float ) * stride * n, cudaMemcpyHostToDevice );
		g.load_records( d, uint32_t( n ), stride, nullptr );
		cuda_check( cudaMemset( g.err_train, 0, 4 ), "guide gradients" );
		g.gradients( g.rec, uint32_t( n ), nullptr, tc );
		cuda_check( cudaDeviceSynchronize(), "guide gradients" );
		uint32_t ew = 0;
		cudaMemcpy( &ew, g.err_train, 4, cudaMemcpyDeviceToHost );
		if ( ew )
		{
			cudaFree( d );
			fail( CR_ERR_DEVICE, "guide tensor-core training pass: an MMA wait timed out" );
		}
		if ( gW ) cudaMemcpy( gW, g.gW, GuideState::w_size() * 4, cudaMemcpyDeviceToHost );
		if ( gb ) cudaMemcpy( gb, g.gb, GuideState::b_size() * 4, cudaMemcpyDeviceToHost );
		if ( ggrid ) cudaMemcpy( ggrid, g.ggrid, GuideState::grid_size() * 4, cudaMemcpyDeviceToHost );
		cudaMemset( g.gW, 0, GuideState::w_size() * 4 );
		cudaMemset( g.gb, 0, GuideState::b_size() * 4 );
		cudaError_t e = cudaMemset( g.ggrid, 0, GuideState::grid_size() * 4 );
		cudaFree( d );
		cuda_check( e, "guide gradients" );
	} );
}
}  // namespace

int cr_guide_gradients( cr_scene *s, const float *records, uint64_t n, float *gW, float *gb, float *ggrid )
{
	return guide_gradients( s, records, n, gW, gb, ggrid, false );
}

int cr_guide_gradients_tc( cr_scene *s, const float *records, uint64_t n, float *gW, float *gb, float *ggrid )
{
	return guide_gradients( s, records, n, gW, gb, ggrid, true );
}

int cr_write_png( const char *path, uint32_t w, uint32_t h, const double *rgb )
{
	return guarded( [&] {
		if ( !path || !rgb ) fail( CR_ERR_INVALID, "null argument" );
		write_png( path, w, h, rgb );
	} );
}

int cr_render_file( const char *json_path, const char *png_path, const char *pfm_path, uint32_t spp, uint32_t w,
					uint32_t h, const char *kernel, const char *tracer )
{
	return guarded( [&] {
		if ( !json_path || !png_path ) fail( CR_ERR_INVALID, "null argument" );
		std::string text = read_file( json_path );
		std::unique_ptr<cr_scene> s( new cr_scene() );
		load_scene( s.get(), text, dir_of( json_path ) );
		if ( kernel && *kernel ) s->kernel = kernel;
		if ( tracer && *tracer ) s->tracer = tracer;
		static const char *tracers[] = { "CudaWavefront", "CPUMulticore", "CPUMultiCoreTracer", "CudaSingleGPU" };
		if ( std::find_if( std::begin( tracers ), std::end( tracers ), [&]( const char *t ) { return s->tracer == t; } ) ==
			 std::end( tracers ) )
			fail( CR_ERR_UNSUPPORTED, "no such tracer: " + s->tracer );
		commit( s.get(), 0x330E, nullptr );
		cr_render_desc d;
		std::memset( &d, 0, sizeof d );
		d.width = w, d.height = h, d.spp = spp, d.max_bounce = UINT32_MAX, d.estimator = -1, d.seed = 1;
		std::vector<double> film( size_t( w ) * h * 3 );
		// The Renderer's profiler (renderer.hpp:17-23, kernel.cu): when enabled,
		// the tracer renders its area only (cpuMulticore.cu:17; the rest of the
		// image stays black) and the slices go to its output file.
		const Json doc = parse_json( text );
		const Json *pj = doc.find( "profiler" );
		// a "profiler" block is enabled unless it says otherwise (Profiler::Configuration, kernel.hpp:37-43)
		const bool profile = pj && pj->number_or( "enable", 1 ) != 0;
		if ( profile )
		{
			uint32_t area[ 4 ] = { 0, 0, w, h };
			if ( const Json *a = pj->find( "area" ) )
			{
				if ( !a->is_array() || a->size() != 4 ) fail( CR_ERR_PARSE, "profiler area must be [x0, y0, x1, y1]" );
				for ( int i = 0; i < 4; ++i )
				{
					const double v = a->at( i ).num;
					area[ i ] = v < 0 ? 0u : uint32_t( std::min<double>( v, i % 2 ? h : w ) );
				}
			}
			uint32_t depth = 8;  // RadianceKernel::Slice's default (radiance.hpp:27-31)
			if ( const Json *pp = pj->find( "props" ) ) depth = uint32_t( pp->number_or( "depth", 8 ) );
			const std::string out = pj->string_or( "output", "a.prof" );
			if ( area[ 2 ] > area[ 0 ] && area[ 3 ] > area[ 1 ] )
			{
				cr_render_desc pdsc = d;
				pdsc.x0 = area[ 0 ], pdsc.y0 = area[ 1 ], pdsc.x1 = area[ 2 ], pdsc.y1 = area[ 3 ];
				const size_t aw = area[ 2 ] - area[ 0 ], ah = area[ 3 ] - area[ 1 ], n = aw * ah * spp;
				std::vector<cr_profile_slice> sl( n );
				std::vector<cr_profile_bounce> bo( n * depth );
				std::vector<double> win( aw * ah * 3 );
				int rc = cr_render_profile( s.get(), &pdsc, depth, sl.data(), bo.data(), win.data() );
				if ( rc != CR_OK ) fail( rc, g_last_error );
				for ( size_t y = 0; y < ah; ++y )
					std::memcpy( &film[ 3 * ( ( area[ 1 ] + y ) * size_t( w ) + area[ 0 ] ) ], &win[ 3 * y * aw ], 24 * aw );
				rc = cr_profile_write( out.c_str(), area, spp, depth, sl.data(), bo.data() );
				if ( rc != CR_OK ) fail( rc, g_last_error );
			}
		}
		else
		{
			int rc = cr_render( s.get(), &d, film.data(), nullptr );
			if ( rc != CR_OK ) fail( rc, g_last_error );
		}
		write_png( png_path, w, h, film.data() );
		if ( pfm_path && *pfm_path ) write_pfm( pfm_path, w, h, film.data() );
	} );
}

// A single-node shader for cr_bsdf_eval / cr_bsdf_sample: those take two
// uniforms per sample and no selection numbers.
static DevShader shader_from_json( int est, const char *js )
{
	if ( !js ) fail( CR_ERR_INVALID, "null shader" );
	ShaderTable tab;
	DevShader sh = make_shader( parse_json( js ), tab, "shader" );
	if ( sh.type == SH_MIXED || sh.type == SH_GLASS )
		fail( CR_ERR_INVALID, "Mixed and GlassBSDF draw selection numbers: use cr_shader_execute" );
	if ( est == EST_MIS && !mis_helper_ok( sh ) )
		fail( CR_ERR_UNSUPPORTED, "the MIS helpers cover Lambert, Beckmann GlossyBSDF and Emission; render to test the others" );
	return sh;
}

int cr_philox4x32_10( const uint32_t *ctr_key, uint64_t n, uint32_t *out )
{
	return guarded( [&] {
		if ( !n ) return;
		if ( !ctr_key || !out ) fail( CR_ERR_INVALID, "null argument" );
		if ( n > ( 1ull << 28 ) ) fail( CR_ERR_INVALID, "at most 2^28 pairs per call" );
		uint32_t *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( uint32_t ) * 10 * n ), "cudaMalloc" );
		cudaError_t e = cudaMemcpy( d, ctr_key, 24 * n, cudaMemcpyHostToDevice );
		if ( e == cudaSuccess )
		{
			launch_philox( d, n, d + 6 * n, nullptr );
			e = cudaMemcpy( out, d + 6 * n, 16 * n, cudaMemcpyDeviceToHost );
		}
		cudaFree( d );
		cuda_check( e, "philox" );
	} );
}

int cr_bsdf_eval( int est, const char *shader_json, const float *wo, const float *wi, uint64_t n, float *f, float *pdf )
{
	return guarded( [&] {
		DevShader sh = shader_from_json( est, shader_json );
		if ( !n ) return;
		if ( !wo || !wi || !f || !pdf ) fail( CR_ERR_INVALID, "null argument" );
		float *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( float ) * 10 * n ), "cudaMalloc" );
		float *dwo = d, *dwi = d + 3 * n, *df = d + 6 * n, *dp = d + 9 * n;
		cudaMemcpy( dwo, wo, 12 * n, cudaMemcpyHostToDevice );
		cudaMemcpy( dwi, wi, 12 * n, cudaMemcpyHostToDevice );
		launch_bsdf_eval( est, sh, dwo, dwi, n, df, dp, nullptr );
		cudaMemcpy( f, df, 12 * n, cudaMemcpyDeviceToHost );
		cudaError_t e = cudaMemcpy( pdf, dp, 4 * n, cudaMemcpyDeviceToHost );
		cudaFree( d );
		cuda_check( e, "bsdf eval" );
	} );
}

int cr_bsdf_sample( int est, const char *shader_json, const float *wo, const float *u, uint64_t n, float *wi,
					float *weight, float *pdf )
{
	return guarded( [&] {
		DevShader sh = shader_from_json( est, shader_json );
		if ( !n ) return;
		if ( !wo || !u || !wi || !weight || !pdf ) fail( CR_ERR_INVALID, "null argument" );
		float *d;
		cuda_check( cudaMalloc( (void **)&d, sizeof( float ) * 12 * n ), "cudaMalloc" );
		float *dwo = d, *du = d + 3 * n, *dwi = d + 5 * n, *dw = d + 8 * n, *dp = d + 11 * n;
		cudaMemcpy( dwo, wo, 12 * n, cudaMemcpyHostToDevice );
		cudaMemcpy( du, u, 8 * n, cudaMemcpyHostToDevice );
		launch_bsdf_sample( est, sh, dwo, du, n, dwi, dw, dp, nullptr );
		cudaMemcpy( wi, dwi, 12 * n, cudaMemcpyDeviceToHost );
		cudaMemcpy( weight, dw, 12 * n, cudaMemcpyDeviceToHost );
		cudaError_t e = cudaMemcpy( pdf, dp, 4 * n, cudaMemcpyDeviceToHost );
		cudaFree( d );
		cuda_check( e, "bsdf sample" );
	} );
}

int cr_shader_execute( const char *shader_json, int target, const float *wo, float *wi, const float *u, uint32_t k,
					   uint64_t n, float *f, float *emission, uint32_t *used )
{
	return guarded( [&] {
		if ( !shader_json ) fail( CR_ERR_INVALID, "null shader" );
		if ( target != CR_SHADE_EVAL && target != CR_SHADE_SAMPLE ) fail( CR_ERR_INVALID, "unknown shader target" );
		ShaderTable tab;
		DevShader root = make_shader( parse_json( shader_json ), tab, "shader" );
		if ( !n ) return;
		if ( !wo || !wi || !f || !emission || !used || ( k && !u ) ) fail( CR_ERR_INVALID, "null argument" );
		if ( n > ( 1ull << 28 ) || uint64_t( k ) > 64 ) fail( CR_ERR_INVALID, "at most 2^28 samples of 64 uniforms" );
		// entry 0 is the root; nested entries keep their order, one slot later
		std::vector<DevShader> dt( 1, root );
		for ( auto &x : tab ) dt.push_back( x.second );
		for ( auto &x : dt )
			if ( x.type == SH_MIXED ) ++x.child[ 0 ], ++x.child[ 1 ];
		const size_t tb = ( sizeof( DevShader ) * dt.size() + 255 ) / 256 * 256;
		const size_t bytes = tb + 4 * ( 12 * n + size_t( k ) * n + n );
		char *d;
		cuda_check( cudaMalloc( (void **)&d, bytes ), "cudaMalloc" );
		DevShader *dtab = (DevShader *)d;
		float *dwo = (float *)( d + tb ), *dwi = dwo + 3 * n, *df = dwi + 3 * n, *de = df + 3 * n, *du = de + 3 * n;
		uint32_t *dused = (uint32_t *)( du + size_t( k ) * n );
		cudaMemcpy( dtab, dt.data(), sizeof( DevShader ) * dt.size(), cudaMemcpyHostToDevice );
		cudaMemcpy( dwo, wo, 12 * n, cudaMemcpyHostToDevice );
		cudaMemcpy( dwi, wi, 12 * n, cudaMemcpyHostToDevice );
		if ( k ) cudaMemcpy( du, u, 4 * size_t( k ) * n, cudaMemcpyHostToDevice );
		launch_shader_execute( dtab, target == CR_SHADE_EVAL ? 0 : 1, dwo, dwi, du, k, n, df, de, dused, nullptr );
		cudaMemcpy( wi, dwi, 12 * n, cudaMemcpyDeviceToHost );
		cudaMemcpy( f, df, 12 * n, cudaMemcpyDeviceToHost );
		cudaMemcpy( emission, de, 12 * n, cudaMemcpyDeviceToHost );
		cudaError_t e = cudaMemcpy( used, dused, 4 * n, cudaMemcpyDeviceToHost );
		cudaFree( d );
		cuda_check( e, "shader execute" );
	} );
}

}  // extern "C"
