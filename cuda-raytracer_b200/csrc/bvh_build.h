// GPU builder of the quantised 8-wide BVH (see bvh_build.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "cr_common.h"

namespace cr
{
struct WideBvh
{
	WNode *nodes = nullptr;   // device, n_nodes entries (allocation holds n_tris)
	float4 *tris = nullptr;   // device, 3 float4 per triangle in leaf order
	uint32_t n_nodes = 0, n_tris = 0, depth = 0;
};

// The library's memory pool of the current device (render.cu), which keeps
// freed memory mapped: the builder's scratch and output come from it.
cudaMemPool_t device_pool();

// d_src: 3 float4 (v0, v1, v2) per triangle in global order, on the device.
// Allocates out.nodes / out.tris with cudaMallocAsync on `st`; throws
// std::runtime_error on failure.  Synchronises `st` once per tree level.
// Build options.  ploc: binary tree by locally-ordered clustering (higher
// quality) within `radius` positions of the Morton order; otherwise the
// Karras radix tree (faster build).  max_leaf (1..3) triangles per leaf;
// cost_node / cost_tri: SAH costs of a node visit and a triangle test.
struct BuildParams
{
	bool ploc = true;
	int radius = 10;
	int max_leaf = 3;
	float cost_node = 1.2f, cost_tri = 1.0f;
	// 8-wide collapse: plan by dynamic programming over the SAH (PLOC trees),
	// with the costs of a wide-node visit and a triangle test; false: greedy
	// (open the largest child first)
	bool dp_collapse = true;
	float dp_cost_node = 1.0f, dp_cost_tri = 0.6f;
};
void build_wide_bvh( const float4 *d_src, uint32_t n, WideBvh &out, cudaStream_t st,
					 const BuildParams &bp = BuildParams() );

// One indexed mesh, on the device, flattened into triangles g0 .. g0 + nt - 1:
// src[3 g + k] = (vertex k, 0) for the builder, attrs[3 g + k] = (normal k,
// w) with w the int bits of the shader (k = 0), primitive (k = 1) and light
// (k = 2) ids.  bounds (6 floats: lo xyz, hi xyz, +inf / -inf before the
// first call) grows over the coordinates (NaN skipped) of the referenced vertices.
// Indices must be below the vertex count (checked when meshes are added).
struct FlatMesh
{
	const float *v, *n;     // 3 floats per vertex
	const uint32_t *idx;    // 3 per triangle
	uint32_t nt;
	uint64_t g0;
	int shader, prim, light;
};
void flatten_mesh( const FlatMesh &m, float4 *src, float4 *attrs, float *bounds, cudaStream_t st );
}  // namespace cr
