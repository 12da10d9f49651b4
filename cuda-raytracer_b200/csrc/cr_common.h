// Data layouts shared by the host runtime and the CUDA kernels.
//
// HBM layout of one committed scene (all arrays 16-byte aligned):
//   nodes    WNode[n_nodes]        80 B  quantised 8-wide BVH, root = node 0
//   tris     float4[3*n_tris]      48 B  per BVH primitive in leaf order; a triangle:
//                                        (v0.xyz, global id), (v1.xyz, -), (v2.xyz, -);
//                                        a sphere (id sph_base + sphere index):
//                                        (box lo.xyz, id), (box hi.xyz, -), (centre.xyz, r^2)
//   attrs    float4[3*n_tris]      48 B  per triangle in global order:
//                                        (n0.xyz, shader), (n1.xyz, prim), (n2.xyz, light)
//   spheres  DevSphere[n_spheres]
//   shaders  DevShader[n_shaders]
//   lights   DevLight[n_lights] + koishi tables float4[2*1024] per mesh light
//            + area CDFs / light triangles for the MIS estimator
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define CR_HD __host__ __device__
#else
#define CR_HD
#endif

namespace cr
{
enum ShaderType : int32_t
{
	SH_LAMBERT = 0,
	SH_GLOSSY = 1,
	SH_EMISSION = 2,
	SH_TRANSPARENT = 3,  // transparent.hpp
	SH_BLACKHOLE = 4,    // blackhole.hpp
	SH_REFRACTION = 5,   // refraction.hpp ("RefractionBSDF")
	SH_GLASS = 6,        // glass.hpp ("GlassBSDF")
	SH_MIXED = 7         // mixed.hpp
};

// SphericalDistribution of a GlossyBSDF, RefractionBSDF or GlassBSDF
// (src/ext/distribution/distribution.impl.cu).
enum DistKind : int32_t
{
	DIST_BECKMANN = 0,
	DIST_COSINE = 1
};

// Scala<float> of a Mixed shader's "fac" (src/ext/scala/scala.impl.cu).
enum FacKind : int32_t
{
	FAC_CONSTANT = 0,
	FAC_FRESNEL = 1
};

// Deepest chain of Mixed shaders a shader table may hold (the device walks
// it with a bounded loop).
constexpr int MAX_SHADER_DEPTH = 16;

enum Estimator : int32_t
{
	EST_KOISHI = 0,
	EST_MIS = 1
};

// One 8-wide BVH node, 80 bytes = 5 x 16-byte loads.
//  * child box i = p + 2^e * [q_lo[i], q_hi[i]] per axis (conservatively rounded)
//  * imask bit i: slot i is an internal node; its index is
//    child_base + popc(imask & ((1<<i)-1))
//  * meta[i] for a leaf slot: (unary n_tris << 5) | offset (unary: 1, 3, 7), triangles
//    tri_base + offset .. + n_tris - 1 (n_tris 1..3, offset 0..23); 0 if empty
//  * slots are assigned so that visiting slot (k ^ oct) for k = 0..7 is
//    roughly front to back for rays whose direction-sign octant is oct.
struct alignas( 16 ) WNode
{
	float px, py, pz;
	uint8_t ex, ey, ez, imask;
	uint32_t child_base;
	uint32_t tri_base;
	uint8_t meta[ 8 ];
	uint8_t qlo_x[ 8 ], qlo_y[ 8 ], qlo_z[ 8 ];
	uint8_t qhi_x[ 8 ], qhi_y[ 8 ], qhi_z[ 8 ];
};
static_assert( sizeof( WNode ) == 80, "WNode must be 80 bytes" );

// One node of a scene's shader table.  Named shaders come first (their index
// is the shader id primitives carry); the shaders nested in a Mixed follow.
struct DevShader
{
	int32_t type;
	float albedo[ 3 ];    // Lambert: color * R; Emission: 1
	float color[ 3 ];     // Glossy, Transparent, Refraction, Glass tint
	float alpha, alpha2;  // Beckmann roughness and its square
	float emission[ 3 ];  // Emission: color * strength
	float ior;            // Refraction, Glass; Mixed with a Fresnel fac
	float fac;            // Mixed with a Constant fac: its value
	int32_t fac_kind;     // Mixed: FacKind
	int32_t dist;         // Glossy, Refraction, Glass: DistKind
	int32_t child[ 2 ];   // Mixed: table indices of shaders[0] and shaders[1]
};

struct DevSphere
{
	float c[ 3 ];
	float r2;       // radius squared, as the reference stores it
	float r;        // sqrt(r2)
	int32_t shader;
	int32_t prim;   // primitive id in scene order
	int32_t light;  // light id or -1
};

enum LightKind : int32_t
{
	LIGHT_MESH = 0,
	LIGHT_SPHERE = 1,
	LIGHT_POINT = 2  // pointLight asset (src/core/light/pointLight.hpp)
};

struct DevLight
{
	int32_t kind;
	int32_t index;        // sphere index, or first entry in light_tris
	int32_t n_tris;       // mesh lights: number of triangles
	int32_t table;        // mesh lights: offset (in float4) of the 1024-point table
	float emission[ 3 ];
	float koishi_pdf;     // area pdf of the reference's table (incl. padding copies)
	float area;           // true area (MIS)
	int32_t cdf;          // offset of the area CDF in light_cdf
	float pos[ 3 ];       // point lights: position
};

struct DevCamera
{
	float o[ 3 ], n[ 3 ], u[ 3 ], v[ 3 ], du[ 3 ], dv[ 3 ];
	uint32_t width, height, pw;
	uint32_t lens;  // CameraConfig::lens: 0 pinhole, 1 orthographic
};

// Everything a kernel needs to know about one committed scene.
struct DevScene
{
	const WNode *nodes;
	const float4 *tris;       // 3 per triangle, BVH leaf order
	const float4 *attrs;      // 3 per triangle, global order
	const DevSphere *spheres;
	const DevShader *shaders;
	const DevLight *lights;
	const float4 *light_tables;  // 2 float4 per point: (p, -), (n, -)
	const float4 *light_tris;    // 3 float4 per emissive triangle (v0, v1, v2), MIS sampling
	const float *light_cdf;
	const uint32_t *prim_first;  // first global triangle of each primitive
	uint32_t n_nodes, n_tris, n_spheres, n_lights, n_shaders;
	uint32_t sph_base;  // BVH primitive ids from here on are spheres (n_tris counts both)
	float scene_scale;
	DevCamera cam;
};

// Hit record written by the closest-hit kernels: 16 bytes.
//   t, slot (BVH-order triangle index, or 0x80000000 | sphere, or ~0u miss), u, v
struct HitRec
{
	float t;
	uint32_t id;
	float u, v;
};

constexpr uint32_t HIT_MISS = 0xFFFFFFFFu;
constexpr uint32_t HIT_SPHERE = 0x80000000u;
constexpr int TRAVERSAL_STACK = 32;

}  // namespace cr
