// Host side of the learned path guide (see guide.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "guide.cuh"

namespace cr
{
// Training records, SoA (one entry per recorded path vertex):
//   x  = (position, valid)       wo = (outgoing direction, -)
//   n  = (shading normal, -)     om = (sampled direction, sampling pdf)
//   T  = (throughput after the vertex, training weight)
//   L  = (radiance gathered up to and including the vertex, -)
struct GuideRecords
{
	float4 *x = nullptr, *wo = nullptr, *n = nullptr, *om = nullptr, *T = nullptr, *L = nullptr;
};

struct GuideState
{
	bool ready = false;
	float *grid = nullptr, *grid_m = nullptr, *grid_v = nullptr, *ggrid = nullptr;
	float *W = nullptr, *W_m = nullptr, *W_v = nullptr, *gW = nullptr;
	float *b = nullptr, *b_m = nullptr, *b_v = nullptr, *gb = nullptr;
	float *wsum = nullptr;
	float3 bmin{ 0, 0, 0 }, binv{ 1, 1, 1 };
	float lr = 1e-2f;
	float select_prob = 0.5f;
	uint32_t step = 0;
	uint32_t train_paths = 32768;  // paths per wave whose vertices are recorded
	GuideRecords rec;
	uint32_t rec_capacity = 0;

	static size_t grid_size();
	static size_t w_size();
	static size_t b_size();

	void init( float3 lo, float3 hi, uint64_t seed );
	void release();
	~GuideState() { release(); }
	GuideDev dev() const;
	void ensure_records( uint32_t n );
	void free_records();
	// radiance targets of the recorded vertices of one wave (paths 0..n_paths-1)
	void compute_targets( const float4 *L, uint32_t n_paths, uint32_t stride, cudaStream_t st );
	void gradients( uint32_t n, cudaStream_t st );  // accumulate into gW, gb, ggrid
	void adam( cudaStream_t st );                   // update and clear the gradients
	void train_from_records( uint32_t n, cudaStream_t st );
	void forward_batch( const float *d_in, uint32_t n, float *d_out, cudaStream_t st );
	// records from n x 13 floats {x, wo, n, w, weight} (device), for tests
	void load_records( const float *d_src, uint32_t n, cudaStream_t st );
};
}  // namespace cr
