// Reference harness: drives the reference's own CPU Radiance path
// (xlnx/cuda-raytracer, compiled from its sources by oracle/Makefile) so its
// outputs can pin the oracle and the CUDA path.  This file is test
// infrastructure; nothing in the product links it.
//
// Meshes reach the reference the way its own scene loader hands them over
// after assimp (src/core/meta/scene.cu:47-51): one PolyMesh per material group
// (src/core/primitive/mesh.cu:404-433) appended to Scene::primitives, then an
// AreaLight plus Mesh::generateSamples for every Emission-shaded mesh, exactly
// as src/core/meta/scene.cu:200-216 does for imported meshes.
//
// Sub-commands (all binary files are little-endian):
//   render <scene.json> <W> <H> <spp> <threads> <out.crf> [maxBounce] [seed] [kernel]
//       per-pixel float film through RadianceKernel::execute
//       (src/core/kernel/radiance.cu:14-81), driven pixel by pixel like
//       CPUMulticoreTracer::execute (src/core/tracer/cpuMulticore.cu:53-64):
//       NaN/Inf samples dropped, sums kept in double with sums of squares.
//   trace  <scene.json> <rays.f32> <out.hits>
//       closest hit per ray over Scene::primitives with the reference's
//       per-primitive intersect (src/core/meta/scene.hpp:35-55).
//   work   <scene.json> <rays.f32>
//       the reference's traversal work on the rays (as for trace), printed as
//       one JSON line: for every ray, Scene::intersect(Ray) (scene.hpp:35-55)
//       asks every primitive; a mesh walks its own BVH as Mesh::intersect(Ray)
//       does (src/core/primitive/mesh.cu:200-267: depth first, both children's
//       boxes tested with the reference's Ray::intersect_bbox at every step,
//       every face of a reached leaf tested, no pruning by distance).  The
//       walk is restated here over the mesh's own BVHNode and Face arrays to
//       count what it reads: node records (36 bytes), faces (36 bytes) and
//       sphere tests.
//   occlude <scene.json> <segs.f32> <out.u8>
//       Scene::intersect(Seg) (src/core/meta/scene.hpp:57-67) per segment.
//   lights <scene.json> <out.lights>
//       the 1024-point tables of every emissive mesh (src/core/primitive/mesh.hpp:61-84).
//   bench  <scene.json> <W> <H> <spp> <threads> [maxBounce] [repeats] [x0 y0 x1 y1]
//       wall time of the reference's own CPUMulticoreTracer::execute, once per repeat;
//       with an area, the tracer renders that pixel window only, through an
//       enabled Profiler (src/core/tracer/cpuMulticore.cu:17), whose dump is discarded.
//   plugin <scene.json> <W> <H> <spp> <out.u8> [seed]      (cr_ref_plugin only)
//       the CudaWavefront Tracer plugin (cuda-raytracer_b200/plugin/cudaWavefront.hpp)
//       registered in Factory<Tracer> as src/core/tracer/tracer.impl.cu:8-11
//       registers the CPU tracer, created by name and run through
//       Tracer::execute (src/core/tracer/tracer.hpp:20-21) as the Renderer
//       does; out: the 8-bit W x H x 3 image it wrote.
//   profile <scene.json> <W> <H> <spp> <x0> <y0> <x1> <y1> <depth> <out.prof> [threads]
//       CPUMulticoreTracer::execute with an enabled Profiler over the area
//       (src/core/kernel/kernel.hpp:35-81, src/core/tracer/cpuMulticore.cu:17):
//       the reference's own per-bounce dump, written by Profiler::~Profiler.
//   shade  <shader.json> <records.f32> <k> <out.f32>
//       Shader::execute (src/core/nodes/shader.hpp:17-23) of the [Type, {props}]
//       shader in shader.json, built by Factory<Shader>::create, for records
//       {wo.xyz, wi.xyz, u[k]}: once with compute_f_by_wi_wo on (wo, wi) and
//       once with sample_wi_f_by_wo on wo (wi preset), each with the sampler
//       scripted to hand out u from its start.  Out per record (float):
//       eval f.xyz, eval emission.xyz, eval draws, sample wi.xyz, sample f.xyz,
//       sample emission.xyz, sample draws.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <core/kernel/radiance.hpp>
#include <core/light/areaLight.hpp>
#include <core/meta/scene.hpp>
#include <core/misc/lens.hpp>
#include <core/primitive/mesh.hpp>
#include <core/primitive/sphere.hpp>
#include <core/tracer/cpuMulticore.hpp>
#include <core/tracer/tracer.hpp>
#include <ext/shader/emission.hpp>
#include <util/image.hpp>

#ifdef CR_HARNESS_PLUGIN
#include <cudaWavefront.hpp>
#endif

using namespace koishi;
using namespace koishi::core;

#ifdef CR_HARNESS_PLUGIN
// The registration line a maintainer adds to src/core/tracer/tracer.impl.cu.
static volatile int cr_plugin_registry[] = { Factory<Tracer>::reg<CudaWavefrontTracer>( "CudaWavefront" ) };
#endif

namespace
{
struct Group
{
	std::string name;
	std::vector<float> v, n;
	std::vector<uint32_t> idx;
};

bool read_crm( const std::string &path, std::vector<Group> &out )
{
	std::ifstream f( path, std::ios::binary );
	if ( !f ) return false;
	char magic[ 4 ];
	f.read( magic, 4 );
	if ( std::memcmp( magic, "CRM1", 4 ) ) return false;
	uint32_t ng;
	f.read( (char *)&ng, 4 );
	for ( uint32_t g = 0; g < ng; ++g )
	{
		Group gr;
		uint32_t len, nv, nt;
		f.read( (char *)&len, 4 );
		gr.name.resize( len );
		f.read( &gr.name[ 0 ], len );
		f.read( (char *)&nv, 4 );
		f.read( (char *)&nt, 4 );
		gr.v.resize( size_t( nv ) * 3 );
		gr.n.resize( size_t( nv ) * 3 );
		gr.idx.resize( size_t( nt ) * 3 );
		f.read( (char *)gr.v.data(), gr.v.size() * 4 );
		f.read( (char *)gr.n.data(), gr.n.size() * 4 );
		f.read( (char *)gr.idx.data(), gr.idx.size() * 4 );
		out.push_back( std::move( gr ) );
	}
	return bool( f );
}

std::string dir_of( const std::string &p )
{
	auto k = p.find_last_of( '/' );
	return k == std::string::npos ? std::string( "." ) : p.substr( 0, k );
}

// Identity of a primitive independent of insertion order: kind 0 = mesh group
// (index in the imported file), kind 1 = sphere (index among sphere assets).
struct PrimId
{
	int kind, index;
};

struct FaceKey
{
	uint32_t b[ 9 ];
	bool operator==( const FaceKey &o ) const { return !std::memcmp( b, o.b, sizeof b ); }
};
struct FaceKeyHash
{
	size_t operator()( const FaceKey &k ) const
	{
		uint64_t h = 1469598103934665603ull;
		for ( auto x : k.b ) h = ( h ^ x ) * 1099511628211ull;
		return h;
	}
};

FaceKey key_of( const float3 &o, const float3 &d1, const float3 &d2 )
{
	FaceKey k;
	float a[ 9 ] = { o.x, o.y, o.z, d1.x, d1.y, d1.z, d2.x, d2.y, d2.z };
	std::memcpy( k.b, a, sizeof a );
	return k;
}

struct Loaded
{
	json doc;
	Scene *scene = nullptr;
	std::vector<PrimId> prim_ids;                                       // per scene.primitives entry
	std::vector<std::unordered_map<FaceKey, uint32_t, FaceKeyHash>> face_maps;  // per mesh group
	std::vector<Mesh *> emissive_meshes;
	std::vector<int> emissive_groups;
	uint32_t max_bounce = 16;
};

// Build the reference Scene from the JSON document; mesh groups come from a
// CRM file named by an ["import", {"path": ...}] asset.
void load( const std::string &path, Loaded &L, uint64_t light_seed )
{
	std::ifstream f( path );
	f >> L.doc;
	Properties sceneProps = L.doc[ "scene" ].get<Properties>();
	if ( L.doc.count( "tracer" ) )
	{
		auto &tr = L.doc[ "tracer" ];
		if ( tr.is_array() && tr.size() > 1 && tr[ 1 ].count( "kernel" ) )
		{
			auto &k = tr[ 1 ][ "kernel" ];
			if ( k.is_array() && k.size() > 1 && k[ 1 ].count( "maxBounce" ) )
				L.max_bounce = k[ 1 ][ "maxBounce" ].get<uint32_t>();
		}
	}
	// The light tables are drawn while the scene is assembled; seed first.
	harness_rng::seed_this_thread( light_seed );
	L.scene = new Scene( sceneProps );
	Scene &scene = *L.scene;

	// Reproduce the shader-name list the Scene constructor built from sphere
	// assets (src/core/meta/scene.cu:136-156) so injected meshes share ids.
	std::vector<std::string> names;
	std::vector<std::string> importPaths;
	int sphereCount = 0;
	for ( auto &asset : L.doc[ "scene" ][ "assets" ] )
	{
		std::string kind = asset[ 0 ].get<std::string>();
		if ( kind == "sphere" )
		{
			auto nm = asset[ 1 ][ "shader" ].get<std::string>();
			bool found = false;
			for ( auto &x : names ) found |= ( x == nm );
			if ( !found ) names.push_back( nm );
			L.prim_ids.push_back( PrimId{ 1, sphereCount++ } );
		}
		else if ( kind == "import" )
		{
			importPaths.push_back( asset[ 1 ][ "path" ].get<std::string>() );
		}
	}
	std::vector<Group> groups;
	for ( auto &p : importPaths )
	{
		std::string full = p[ 0 ] == '/' ? p : dir_of( path ) + "/" + p;
		if ( !read_crm( full, groups ) )
		{
			std::cerr << "cannot read mesh file " << full << std::endl;
			std::exit( 2 );
		}
	}
	auto shaderCfg = L.doc[ "scene" ][ "shaders" ];
	size_t firstMesh = scene.primitives.size();
	for ( size_t g = 0; g < groups.size(); ++g )
	{
		auto &gr = groups[ g ];
		poly::vector<float3> verts( gr.v.size() / 3 ), norms( gr.n.size() / 3 );
		for ( size_t i = 0; i < verts.size(); ++i )
		{
			verts[ i ] = float3{ gr.v[ 3 * i ], gr.v[ 3 * i + 1 ], gr.v[ 3 * i + 2 ] };
			norms[ i ] = float3{ gr.n[ 3 * i ], gr.n[ 3 * i + 1 ], gr.n[ 3 * i + 2 ] };
		}
		std::vector<uint3> tris( gr.idx.size() / 3 );
		std::unordered_map<FaceKey, uint32_t, FaceKeyHash> fmap;
		for ( size_t t = 0; t < tris.size(); ++t )
		{
			tris[ t ] = uint3{ gr.idx[ 3 * t ], gr.idx[ 3 * t + 1 ], gr.idx[ 3 * t + 2 ] };
			float3 o = verts[ tris[ t ].x ];
			fmap[ key_of( o, verts[ tris[ t ].y ] - o, verts[ tris[ t ].z ] - o ) ] = uint32_t( t );
		}
		L.face_maps.push_back( std::move( fmap ) );
		uint32_t sid = uint32_t( -1 );
		for ( size_t i = 0; i < names.size(); ++i )
			if ( names[ i ] == gr.name ) sid = uint32_t( i );
		if ( sid == uint32_t( -1 ) )
		{
			if ( !shaderCfg.count( gr.name ) )
			{
				std::cerr << "no shader named " << gr.name << std::endl;
				std::exit( 2 );
			}
			Config c = shaderCfg[ gr.name ].get<Config>();
			scene.shaders.emplace_back( Factory<Shader>::create( c ) );
			names.push_back( gr.name );
			sid = uint32_t( names.size() - 1 );
		}
		PolyMesh pm( std::move( verts ), std::move( norms ), tris );
		for ( auto &m : pm.mesh )
		{
			m.shaderId = sid;
			scene.primitives.emplace_back( poly::make_object<Mesh>( std::move( m ) ) );
			L.prim_ids.push_back( PrimId{ 0, int( g ) } );
		}
	}
	// Area lights for emissive meshes, in primitive order (src/core/meta/scene.cu:200-216).
	// Sphere lights were already made by the Scene constructor.
	for ( size_t i = firstMesh; i < scene.primitives.size(); ++i )
	{
		auto &m = scene.primitives[ i ];
		auto *em = dynamic_cast<const ext::Emission *>( &*scene.shaders[ m->shaderId ] );
		if ( em )
		{
			scene.lights.emplace_back( poly::make_object<AreaLight>( em->emission, m ) );
			auto *mesh = dynamic_cast<Mesh *>( &*m );
			mesh->generateSamples();
			L.emissive_meshes.push_back( mesh );
			L.emissive_groups.push_back( L.prim_ids[ i ].index );
		}
	}
}

Config kernel_config( uint32_t maxBounce, const std::string &name = "Radiance" )
{
	Properties kp;
	kp[ "maxBounce" ] = maxBounce;
	return Config( name, kp );
}

int cmd_render( int argc, char **argv )
{
	if ( argc < 8 ) return 1;
	std::string path = argv[ 2 ];
	uint32_t W = std::stoul( argv[ 3 ] ), H = std::stoul( argv[ 4 ] ), spp = std::stoul( argv[ 5 ] );
	uint32_t nth = std::stoul( argv[ 6 ] );
	std::string out = argv[ 7 ];
	uint64_t seed = argc > 9 ? std::stoull( argv[ 9 ] ) : 7;
	std::string kname = argc > 10 ? argv[ 10 ] : "Radiance";  // any Factory<Kernel> name
	Loaded L;
	load( path, L, 0x330E );
	uint32_t mb = argc > 8 ? std::stoul( argv[ 8 ] ) : L.max_bounce;
	harness_rng::base_seed() = seed;
	auto kern = Factory<Kernel>::create( kernel_config( mb, kname ) );
	// the Renderer's lens choice (src/core/renderer/renderer.cu:30-38)
	PinholeLens pinhole( L.scene->camera[ 0 ], W, H, spp );
	OrthographicLens ortho( L.scene->camera[ 0 ], W, H, spp );
	const Lens &lens = L.scene->camera[ 0 ].lens == 1 ? static_cast<const Lens &>( ortho ) : pinhole;
	std::vector<double> sum( size_t( W ) * H * 3 ), sq( size_t( W ) * H * 3 );
	std::vector<uint32_t> cnt( size_t( W ) * H );
	std::atomic<uint32_t> nextRow{ 0 };
	auto worker = [&]() {
		static constexpr uint32_t block_size = 1 << 16;
		std::vector<char> block( block_size );
		HybridAllocator pool( block.data(), block_size );
		Sampler rng;
		for ( ;; )
		{
			uint32_t j = nextRow.fetch_add( 1 );
			if ( j >= H ) break;
			for ( uint32_t i = 0; i < W; ++i )
			{
				double s[ 3 ] = { 0, 0, 0 }, q[ 3 ] = { 0, 0, 0 };
				uint32_t valid = 0;
				for ( uint32_t k = 0; k < spp; ++k )
				{
					float3 r = kern->execute( lens.sample( i, j, k ), *L.scene, pool, rng, nullptr );
					pool.clear();
					if ( !hasnan( r ) && !hasinf( r ) )
					{
						++valid;
						double c[ 3 ] = { r.x, r.y, r.z };
						for ( int ch = 0; ch < 3; ++ch ) s[ ch ] += c[ ch ], q[ ch ] += c[ ch ] * c[ ch ];
					}
				}
				size_t p = size_t( j ) * W + i;
				for ( int ch = 0; ch < 3; ++ch ) sum[ 3 * p + ch ] = s[ ch ], sq[ 3 * p + ch ] = q[ ch ];
				cnt[ p ] = valid;
			}
		}
	};
	auto t0 = std::chrono::steady_clock::now();
	std::vector<std::thread> ts;
	for ( uint32_t t = 0; t < nth; ++t ) ts.emplace_back( worker );
	for ( auto &t : ts ) t.join();
	double sec = std::chrono::duration<double>( std::chrono::steady_clock::now() - t0 ).count();
	std::ofstream f( out, std::ios::binary );
	f.write( "CRF1", 4 );
	f.write( (char *)&W, 4 );
	f.write( (char *)&H, 4 );
	f.write( (char *)&spp, 4 );
	f.write( (char *)sum.data(), sum.size() * 8 );
	f.write( (char *)sq.data(), sq.size() * 8 );
	f.write( (char *)cnt.data(), cnt.size() * 4 );
	std::printf( "{\"seconds\": %.6f, \"samples\": %llu, \"threads\": %u}\n", sec,
				 (unsigned long long)W * H * spp, nth );
	return 0;
}

std::vector<float> read_f32( const std::string &p )
{
	std::ifstream f( p, std::ios::binary | std::ios::ate );
	size_t n = size_t( f.tellg() ) / 4;
	f.seekg( 0 );
	std::vector<float> v( n );
	f.read( (char *)v.data(), n * 4 );
	return v;
}

int cmd_trace( int argc, char **argv )
{
	if ( argc < 5 ) return 1;
	Loaded L;
	load( argv[ 2 ], L, 0x330E );
	auto rays = read_f32( argv[ 3 ] );
	size_t n = rays.size() / 7;
	std::vector<char> block( 1 << 16 );
	HybridAllocator pool( block.data(), block.size() );
	std::ofstream f( argv[ 4 ], std::ios::binary );
	for ( size_t r = 0; r < n; ++r )
	{
		const float *x = &rays[ 7 * r ];
		Ray ray;
		ray.o = float3{ x[ 0 ], x[ 1 ], x[ 2 ] };
		ray.d = normalized_float3( float3{ x[ 3 ], x[ 4 ], x[ 5 ] } );
		Hit best;
		int bestPrim = -1;
		for ( size_t p = 0; p < L.scene->primitives.size(); ++p )
		{
			Hit h;
			if ( L.scene->primitives[ p ]->intersect( ray, h, pool ) && h.t < best.t ) best = h, bestPrim = int( p );
			pool.clear();
		}
		int32_t kind = -1, index = -1, tri = -1;
		float t = INFINITY;
		if ( bestPrim >= 0 )
		{
			kind = L.prim_ids[ bestPrim ].kind;
			index = L.prim_ids[ bestPrim ].index;
			t = best.t;
			if ( kind == 0 )
			{
				auto *mesh = dynamic_cast<const Mesh *>( &*L.scene->primitives[ bestPrim ] );
				auto &face = mesh->faces[ best.id ];
				auto it = L.face_maps[ index ].find( key_of( face.o, face.d1, face.d2 ) );
				tri = it == L.face_maps[ index ].end() ? -2 : int32_t( it->second );
			}
		}
		f.write( (char *)&kind, 4 );
		f.write( (char *)&index, 4 );
		f.write( (char *)&tri, 4 );
		f.write( (char *)&t, 4 );
	}
	return 0;
}

// Mesh::intersect(Ray)'s walk (mesh.cu:200-267), counting the node records
// and faces it reads; the box test is the reference's own.
void mesh_work( const Mesh &m, const Ray &ray, uint64_t &nodes, uint64_t &faces )
{
	if ( !m.bvh.size() ) return;
	std::vector<uint32_t> stack{ 0 };
	++nodes;  // the root's record (its offset)
	while ( !stack.empty() )
	{
		uint32_t i = stack.back();
		stack.pop_back();
		bool reached = true;
		while ( uint32_t offset = m.bvh[ i ].offset )
		{
			nodes += 2;  // both children's boxes
			const bool left = ray.intersect_bbox( m.bvh[ i + 1 ].vmin, m.bvh[ i + 1 ].vmax );
			const bool right = ray.intersect_bbox( m.bvh[ i + offset ].vmin, m.bvh[ i + offset ].vmax );
			if ( !left && !right )
			{
				reached = false;
				break;
			}
			if ( left && right ) stack.push_back( i + offset );
			i = left ? i + 1 : i + offset;
		}
		if ( reached ) faces += m.bvh[ i ].end - m.bvh[ i ].begin;
	}
}

int cmd_work( int argc, char **argv )
{
	if ( argc < 4 ) return 1;
	Loaded L;
	load( argv[ 2 ], L, 0x330E );
	auto rays = read_f32( argv[ 3 ] );
	const size_t n = rays.size() / 7;
	uint64_t nodes = 0, faces = 0, spheres = 0;
	for ( size_t r = 0; r < n; ++r )
	{
		const float *x = &rays[ 7 * r ];
		Ray ray;
		ray.o = float3{ x[ 0 ], x[ 1 ], x[ 2 ] };
		ray.d = normalized_float3( float3{ x[ 3 ], x[ 4 ], x[ 5 ] } );
		for ( size_t p = 0; p < L.scene->primitives.size(); ++p )
		{
			if ( auto *mesh = dynamic_cast<const Mesh *>( &*L.scene->primitives[ p ] ) )
				mesh_work( *mesh, ray, nodes, faces );
			else
				++spheres;
		}
	}
	std::printf( "{\"rays\": %zu, \"nodes\": %llu, \"faces\": %llu, \"spheres\": %llu}\n", n,
				 (unsigned long long)nodes, (unsigned long long)faces, (unsigned long long)spheres );
	return 0;
}

int cmd_occlude( int argc, char **argv )
{
	if ( argc < 5 ) return 1;
	Loaded L;
	load( argv[ 2 ], L, 0x330E );
	auto segs = read_f32( argv[ 3 ] );
	size_t n = segs.size() / 7;
	std::vector<char> block( 1 << 16 );
	HybridAllocator pool( block.data(), block.size() );
	std::vector<uint8_t> out( n );
	for ( size_t r = 0; r < n; ++r )
	{
		const float *x = &segs[ 7 * r ];
		Seg s;
		s.o = float3{ x[ 0 ], x[ 1 ], x[ 2 ] };
		s.d = normalized_float3( float3{ x[ 3 ], x[ 4 ], x[ 5 ] } );
		s.t = x[ 6 ];
		out[ r ] = L.scene->intersect( s, pool ) ? 1 : 0;
		pool.clear();
	}
	std::ofstream f( argv[ 4 ], std::ios::binary );
	f.write( (char *)out.data(), n );
	return 0;
}

int cmd_lights( int argc, char **argv )
{
	if ( argc < 4 ) return 1;
	uint64_t seed = argc > 4 ? std::stoull( argv[ 4 ] ) : 0x330E;
	Loaded L;
	load( argv[ 2 ], L, seed );
	std::ofstream f( argv[ 3 ], std::ios::binary );
	uint32_t n = uint32_t( L.emissive_meshes.size() );
	f.write( (char *)&n, 4 );
	for ( size_t i = 0; i < L.emissive_meshes.size(); ++i )
	{
		auto *m = L.emissive_meshes[ i ];
		int32_t g = L.emissive_groups[ i ];
		uint32_t nf = uint32_t( m->faces.size() );
		f.write( (char *)&g, 4 );
		f.write( (char *)&m->pdf, 4 );
		f.write( (char *)&nf, 4 );
		for ( uint32_t k = 0; k < 1024; ++k )
		{
			float a[ 6 ] = { m->samples[ k ].p.x, m->samples[ k ].p.y, m->samples[ k ].p.z,
							 m->samples[ k ].n.x, m->samples[ k ].n.y, m->samples[ k ].n.z };
			f.write( (char *)a, sizeof a );
		}
	}
	return 0;
}

int cmd_bench( int argc, char **argv )
{
	if ( argc < 7 ) return 1;
	std::string path = argv[ 2 ];
	uint32_t W = std::stoul( argv[ 3 ] ), H = std::stoul( argv[ 4 ] ), spp = std::stoul( argv[ 5 ] );
	uint32_t nth = std::stoul( argv[ 6 ] );
	Loaded L;
	load( path, L, 0x330E );
	uint32_t mb = argc > 7 ? std::stoul( argv[ 7 ] ) : L.max_bounce;
	Properties tp;
	tp[ "maxThreads" ] = nth;
	Properties kp;
	kp[ "maxBounce" ] = mb;
	tp[ "kernel" ] = json::array( { "Radiance", kp } );
	auto tracer = Factory<Tracer>::create( Config( "CPUMulticore", tp ) );
	util::Image<3> image( W, H );
	poly::object<Lens> lens;
	if ( L.scene->camera[ 0 ].lens == 1 )
		lens = poly::make_object<OrthographicLens>( L.scene->camera[ 0 ], W, H, spp );
	else
		lens = poly::make_object<PinholeLens>( L.scene->camera[ 0 ], W, H, spp );
	SamplerGenerator gen;
	Properties pp;
	uint64_t px = uint64_t( W ) * H;
	if ( argc > 12 )
	{
		uint32_t a[ 4 ] = { uint32_t( std::stoul( argv[ 9 ] ) ), uint32_t( std::stoul( argv[ 10 ] ) ),
							uint32_t( std::stoul( argv[ 11 ] ) ), uint32_t( std::stoul( argv[ 12 ] ) ) };
		pp[ "enable" ] = true;
		pp[ "output" ] = "/dev/null";
		pp[ "area" ] = json::array( { a[ 0 ], a[ 1 ], a[ 2 ], a[ 3 ] } );
		px = uint64_t( a[ 2 ] - a[ 0 ] ) * ( a[ 3 ] - a[ 1 ] );
	}
	else
		pp[ "enable" ] = false;
	Profiler profiler( pp, tracer->getKernel(), W, H, spp );
	int repeats = argc > 8 ? std::stoi( argv[ 8 ] ) : 1;
	for ( int r = 0; r < repeats; ++r )
	{
		auto t0 = std::chrono::steady_clock::now();
		tracer->execute( image, lens, gen, *L.scene, spp, profiler );
		double sec = std::chrono::duration<double>( std::chrono::steady_clock::now() - t0 ).count();
		std::fprintf( stderr, "{\"seconds\": %.6f, \"samples\": %llu, \"threads\": %u}\n", sec,
					  (unsigned long long)( px * spp ), nth );
	}
	return 0;
}

}  // namespace

int cmd_profile( int argc, char **argv )
{
	if ( argc < 12 ) return 1;
	std::string path = argv[ 2 ];
	uint32_t W = std::stoul( argv[ 3 ] ), H = std::stoul( argv[ 4 ] ), spp = std::stoul( argv[ 5 ] );
	uint32_t area[ 4 ] = { uint32_t( std::stoul( argv[ 6 ] ) ), uint32_t( std::stoul( argv[ 7 ] ) ),
						   uint32_t( std::stoul( argv[ 8 ] ) ), uint32_t( std::stoul( argv[ 9 ] ) ) };
	uint32_t depth = std::stoul( argv[ 10 ] );
	std::string out = argv[ 11 ];
	uint32_t nth = argc > 12 ? std::stoul( argv[ 12 ] ) : std::max( 1u, std::thread::hardware_concurrency() - 1 );
	Loaded L;
	load( path, L, 0x330E );
	Properties tp;
	tp[ "maxThreads" ] = nth;
	Properties kp;
	kp[ "maxBounce" ] = L.max_bounce;
	tp[ "kernel" ] = json::array( { "Radiance", kp } );
	auto tracer = Factory<Tracer>::create( Config( "CPUMulticore", tp ) );
	util::Image<3> image( W, H );
	poly::object<Lens> lens;
	if ( L.scene->camera[ 0 ].lens == 1 )
		lens = poly::make_object<OrthographicLens>( L.scene->camera[ 0 ], W, H, spp );
	else
		lens = poly::make_object<PinholeLens>( L.scene->camera[ 0 ], W, H, spp );
	SamplerGenerator gen;
	Properties pp;
	pp[ "enable" ] = true;
	pp[ "output" ] = out;
	pp[ "area" ] = json::array( { area[ 0 ], area[ 1 ], area[ 2 ], area[ 3 ] } );
	Properties sp;
	sp[ "depth" ] = depth;
	pp[ "props" ] = sp;
	{
		Profiler profiler( pp, tracer->getKernel(), W, H, spp );
		tracer->execute( image, lens, gen, *L.scene, spp, profiler );
	}  // ~Profiler writes `out`
	return 0;
}

#ifdef CR_HARNESS_PLUGIN
int cmd_plugin( int argc, char **argv )
{
	if ( argc < 7 ) return 1;
	std::string path = argv[ 2 ];
	uint32_t W = std::stoul( argv[ 3 ] ), H = std::stoul( argv[ 4 ] ), spp = std::stoul( argv[ 5 ] );
	std::string out = argv[ 6 ];
	uint32_t seed = argc > 7 ? std::stoul( argv[ 7 ] ) : 1u;
	Loaded L;
	load( path, L, 0x330E );
	Properties tp;
	Properties kp;
	kp[ "maxBounce" ] = L.max_bounce;
	tp[ "kernel" ] = json::array( { "Radiance", kp } );
	tp[ "seed" ] = seed;
	auto tracer = Factory<Tracer>::create( Config( "CudaWavefront", tp ) );
	util::Image<3> image( W, H );
	poly::object<Lens> lens;
	if ( L.scene->camera[ 0 ].lens == 1 )
		lens = poly::make_object<OrthographicLens>( L.scene->camera[ 0 ], W, H, spp );
	else
		lens = poly::make_object<PinholeLens>( L.scene->camera[ 0 ], W, H, spp );
	SamplerGenerator gen;
	Properties pp;
	pp[ "enable" ] = false;
	Profiler profiler( pp, tracer->getKernel(), W, H, spp );
	tracer->execute( image, lens, gen, *L.scene, spp, profiler );
	std::ofstream f( out, std::ios::binary );
	f.write( (const char *)image.data(), std::streamsize( size_t( W ) * H * 3 ) );
	return f ? 0 : 2;
}
#endif

int cmd_shade( int argc, char **argv )
{
	if ( argc < 6 ) return 1;
	std::ifstream jf( argv[ 2 ] );
	json j;
	jf >> j;
	auto shader = Factory<Shader>::create( j.get<Config>() );
	const uint32_t k = std::stoul( argv[ 4 ] );
	auto rec = read_f32( argv[ 3 ] );
	const size_t stride = 6 + k, n = rec.size() / stride;
	static constexpr uint32_t block_size = 1 << 16;
	std::vector<char> block( block_size );
	HybridAllocator pool( block.data(), block_size );
	Sampler rng;
	auto &sc = harness_rng::script();
	std::vector<float> out;
	out.reserve( n * 17 );
	for ( size_t i = 0; i < n; ++i )
	{
		const float *r = &rec[ i * stride ];
		for ( int target = 0; target < 2; ++target )
		{
			Varyings v;
			static_cast<float3 &>( v.wo ) = float3{ r[ 0 ], r[ 1 ], r[ 2 ] };
			static_cast<float3 &>( v.wi ) = float3{ r[ 3 ], r[ 4 ], r[ 5 ] };
			sc.u = r + 6, sc.n = k, sc.used = 0;
			shader->execute( v, rng, pool, target == 0 ? compute_f_by_wi_wo : sample_wi_f_by_wo );
			pool.clear();
			if ( target == 1 ) out.insert( out.end(), { v.wi.x, v.wi.y, v.wi.z } );
			out.insert( out.end(), { v.f.x, v.f.y, v.f.z, v.emission.x, v.emission.y, v.emission.z, float( sc.used ) } );
		}
	}
	sc.u = nullptr;
	std::ofstream f( argv[ 5 ], std::ios::binary );
	f.write( (const char *)out.data(), out.size() * 4 );
	return 0;
}

int main( int argc, char **argv )
{
	if ( argc < 2 )
	{
		std::fprintf( stderr, "usage: cr_ref render|trace|occlude|lights|bench ...\n" );
		return 1;
	}
	std::string cmd = argv[ 1 ];
	int rc = 1;
	try
	{
		if ( cmd == "render" ) rc = cmd_render( argc, argv );
		else if ( cmd == "trace" ) rc = cmd_trace( argc, argv );
		else if ( cmd == "work" ) rc = cmd_work( argc, argv );
		else if ( cmd == "occlude" ) rc = cmd_occlude( argc, argv );
		else if ( cmd == "lights" ) rc = cmd_lights( argc, argv );
		else if ( cmd == "bench" ) rc = cmd_bench( argc, argv );
		else if ( cmd == "shade" ) rc = cmd_shade( argc, argv );
		else if ( cmd == "profile" ) rc = cmd_profile( argc, argv );
#ifdef CR_HARNESS_PLUGIN
		else if ( cmd == "plugin" ) rc = cmd_plugin( argc, argv );
#endif
	}
	catch ( const std::exception &e )
	{
		std::fprintf( stderr, "error: %s\n", e.what() );
		return 3;
	}
	if ( rc == 1 ) std::fprintf( stderr, "bad arguments for %s\n", cmd.c_str() );
	return rc;
}
