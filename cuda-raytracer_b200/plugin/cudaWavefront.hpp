// CudaWavefrontTracer: the Tracer plugin that puts this library behind the
// reference renderer's own tracer registry.
//
// A maintainer of xlnx/cuda-raytracer adds this header as
// src/core/tracer/cudaWavefront.hpp, one registration line to
// src/core/tracer/tracer.impl.cu:8-11
//     Factory<Tracer>::reg<CudaWavefrontTracer>( "CudaWavefront" )
// and links -L<this repository>/cuda-raytracer_b200/lib -lcr_b200.  A scene
// file whose tracer is ["CudaWavefront", {"kernel": ["Radiance", {...}]}]
// then renders on the GPU through Tracer::execute
// (src/core/tracer/tracer.hpp:20-21), the call CPUMulticoreTracer::execute
// (src/core/tracer/cpuMulticore.cu:14-122) answers on the CPU.
//
// execute() hands the reference's in-memory Scene (scene.hpp:27-31) to the C
// ABI of include/cr.h as it is: shaders through their own writeNode, meshes
// as their faces and normals (mesh.hpp:54-55), spheres, point lights, camera 0
// (the one Renderer::render uses, renderer.cu:25), and each emissive mesh's own
// 1024-point light table and pdf (Mesh::samples, Mesh::pdf, mesh.hpp:58-84),
// so the GPU samples the very light points the CPU tracer would.  It renders
// with the reference estimator (CR_ESTIMATOR_KOISHI) and writes the per-pixel
// mean of the finite samples into the 8-bit image, as the CPU tracer does.
#pragma once
#include <cr.h>  // include/ of this repository

#include <map>
#include <string>
#include <vector>

#include <core/light/pointLight.hpp>
#include <core/primitive/mesh.hpp>
#include <core/primitive/sphere.hpp>
#include <ext/shader/emission.hpp>
#include "tracer.hpp"

namespace koishi
{
namespace core
{
// Sphere keeps its centre and squared radius private (sphere.hpp:57-59), and
// PointLight its position and emission (pointLight.hpp:31-33).  Inside the
// reference a maintainer may add accessors instead; against the unmodified
// reference the plugin reads them through explicit template instantiation,
// where C++ allows naming private members ([temp.spec.general]).
namespace cr_access
{
template <class Tag, typename Tag::type M>
struct grant
{
	friend typename Tag::type get( Tag ) { return M; }
};
struct sphere_o { using type = float3 Sphere::*; friend type get( sphere_o ); };
struct sphere_r2 { using type = float Sphere::*; friend type get( sphere_r2 ); };
struct point_p { using type = float3 PointLight::*; friend type get( point_p ); };
struct point_e { using type = float3 PointLight::*; friend type get( point_e ); };
template struct grant<sphere_o, &Sphere::o>;
template struct grant<sphere_r2, &Sphere::r2>;
template struct grant<point_p, &PointLight::p>;
template struct grant<point_e, &PointLight::emission>;
}  // namespace cr_access

// writeNode (src/core/nodes/node.hpp) prints some nodes with short names and
// bare values (glass.hpp:55-60, mixed.hpp:31-36, fresnel.hpp:32-35,
// constant.hpp:22-25, beckmann.hpp, cosine.hpp:27-30, blackhole.hpp:24-27);
// this maps one shader node back to the [Type, {props}] array that
// Factory<Shader>::create (and cr_scene_add_shader) reads.
inline json cr_shader_config( const json &j )
{
	if ( j.is_string() ) return json::array( { j, json::object() } );  // "Blackhole"
	auto it = j.begin();
	static const std::map<std::string, std::string> reg = {
		{ "Glass", "GlassBSDF" }, { "Refraction", "RefractionBSDF" }, { "Glossy", "GlossyBSDF" } };
	std::string name = reg.count( it.key() ) ? reg.at( it.key() ) : it.key();
	json props = it.value();
	if ( props.count( "distribution" ) )  // {"Beckmann": roughness} or "Cosine"
	{
		auto &d = props[ "distribution" ];
		props[ "distribution" ] = d.is_string() ? json::array( { "Cosine", json::object() } )
												: json::array( { "Beckmann", { { "roughness", d.begin().value() } } } );
	}
	if ( name == "Mixed" )  // fac: a number or {"Fresnel": ior}
	{
		auto &f = props[ "fac" ];
		props[ "fac" ] = f.is_number() ? json::array( { "Constant", { { "value", f } } } )
									   : json::array( { "Fresnel", { { "ior", f.begin().value() } } } );
		for ( auto &c : props[ "shaders" ] ) c = cr_shader_config( c );
	}
	return json::array( { name, props } );
}

struct CudaWavefrontTracer : Tracer
{
	struct Configuration : serializable<Configuration>
	{
		Property( uint, maxBounce, 16u );  // RadianceKernel::Configuration (radiance.hpp:12-15)
	};

	CudaWavefrontTracer( const Properties &props ) :
	  Tracer( props )
	{
		Configuration c = json( get( props, "kernel", Config( "Radiance", {} ) ).props );
		maxBounce = c.maxBounce;
		seed = get( props, "seed", 1u );
	}

	void execute( util::Image<3> &image, poly::object<Lens> &, SamplerGenerator &, Scene &scene, uint spp,
				  Profiler & ) override
	{
		cr_scene *s = nullptr;
		check( cr_scene_create_empty( &s ), s );
		std::vector<std::string> names( scene.shaders.size() );
		for ( uint i = 0; i != scene.shaders.size(); ++i )
		{
			json j;
			scene.shaders[ i ]->writeNode( j );
			names[ i ] = std::to_string( i );
			check( cr_scene_add_shader( s, names[ i ].c_str(), cr_shader_config( j ).dump().c_str() ), s );
		}
		// point lights come first in the light list, then the area lights in
		// primitive order, as the reference builds it (scene.cu:156-163, 200-216)
		for ( auto &l : scene.lights )
			if ( auto *pl = dynamic_cast<const PointLight *>( &*l ) )
			{
				const float3 &p = pl->*get( cr_access::point_p{} ), &e = pl->*get( cr_access::point_e{} );
				check( cr_scene_add_point_light( s, &p.x, &e.x, 1.f ), s );  // emission = color * strength
			}
		std::vector<std::pair<uint32_t, const Mesh *>> emissive;  // (primitive id, mesh) of each emissive mesh
		for ( auto &p : scene.primitives )
		{
			const std::string &sid = names.at( p->shaderId );
			const bool emits = dynamic_cast<const ext::Emission *>( &*scene.shaders[ p->shaderId ] ) != nullptr;
			if ( auto *m = dynamic_cast<const Mesh *>( &*p ) )
			{
				std::vector<float> v, n;
				std::vector<uint32_t> idx;
				v.reserve( 9 * m->faces.size() ), n.reserve( 9 * m->faces.size() ), idx.reserve( 3 * m->faces.size() );
				for ( uint f = 0; f != m->faces.size(); ++f )
				{
					const auto &F = m->faces[ f ];
					const auto &N = m->normals[ f ];
					const float3 vs[ 3 ] = { F.o, F.o + F.d1, F.o + F.d2 }, ns[ 3 ] = { N.n0, N.n1, N.n2 };
					for ( int k = 0; k < 3; ++k )
					{
						v.insert( v.end(), { vs[ k ].x, vs[ k ].y, vs[ k ].z } );
						n.insert( n.end(), { ns[ k ].x, ns[ k ].y, ns[ k ].z } );
						idx.push_back( 3 * f + k );
					}
				}
				const int prim = cr_scene_add_mesh( s, v.data(), uint32_t( v.size() / 3 ), n.data(), idx.data(),
												   uint32_t( idx.size() / 3 ), sid.c_str() );
				check( prim, s );
				if ( emits ) emissive.emplace_back( uint32_t( prim ), m );
			}
			else if ( auto *sp = dynamic_cast<const Sphere *>( &*p ) )
			{
				const float3 &o = sp->*get( cr_access::sphere_o{} );
				check( cr_scene_add_sphere( s, &o.x, std::sqrt( sp->*get( cr_access::sphere_r2{} ) ), sid.c_str() ), s );
			}
		}
		auto &cam = scene.camera[ 0 ];
		check( cr_scene_set_camera( s, &cam.position.x, &cam.target.x, &cam.upaxis.x, cam.fovx ), s );
		check( cr_scene_set_lens( s, int( cam.lens ) ), s );
		check( cr_scene_commit( s, 0x330E, nullptr ), s );
		for ( auto &e : emissive )
		{
			const Mesh &m = *e.second;
			if ( m.samples.size() != 1024 ) continue;  // generateSamples not run: keep the library's table
			std::vector<float> pts( 6 * 1024 );
			for ( uint k = 0; k != 1024; ++k )
			{
				const float3 p = m.samples[ k ].p, nn = m.samples[ k ].n;
				const float q[ 6 ] = { p.x, p.y, p.z, nn.x, nn.y, nn.z };
				std::copy( q, q + 6, pts.begin() + 6 * k );
			}
			check( cr_scene_set_light_table( s, e.first, pts.data(), m.pdf ), s );
		}
		cr_render_desc d{};
		d.width = image.width(), d.height = image.height(), d.spp = spp;
		d.max_bounce = maxBounce, d.estimator = CR_ESTIMATOR_KOISHI, d.seed = seed;
		std::vector<double> film( 3 * size_t( d.width ) * d.height );
		check( cr_render( s, &d, film.data(), nullptr ), s );
		for ( uint y = 0; y != d.height; ++y )
			for ( uint x = 0; x != d.width; ++x )
			{
				const double *c = &film[ 3 * ( size_t( y ) * d.width + x ) ];
				image.at( x, y ) = float3{ float( c[ 0 ] ), float( c[ 1 ] ), float( c[ 2 ] ) };
			}
		cr_scene_destroy( s );
	}

	uint maxBounce;
	uint seed;

private:
	static void check( int rc, cr_scene *s )
	{
		if ( rc >= 0 ) return;
		std::string msg = std::string( "CudaWavefront: " ) + cr_last_error();
		if ( s ) cr_scene_destroy( s );
		KTHROW( msg );
	}
};

}  // namespace core
}  // namespace koishi
