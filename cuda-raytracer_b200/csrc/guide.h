// Host side of the learned path guide (see guide.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "guide.cuh"

namespace cr
{
// Training records, SoA (one entry per recorded path vertex):
//   x  = (position, valid)       wo = (outgoing direction, -)
//   n  = (shading normal, BSDF density of the sampled direction)
//   om = (sampled direction, sampling pdf)
//   wo.w = luminance of f * cos for the sampled direction
//   T  = (throughput after the vertex, training weight)
//   L  = (radiance the path had gathered once it reached the next vertex,
//         that vertex's emission included, -)
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
	uint8_t *Wp = nullptr;    // device: BF16 weights in the tensor-core operand layout (guide_tc.cuh)
	uint2 *grid_pairs = nullptr;  // device: the inference's paired FP16 copy of the grid (guide.cuh GuideDev)
	uint32_t *err = nullptr;  // device: error word of the batch forward calls
	uint32_t *err_train = nullptr;  // device: error word of the tensor-core training pass
	bool tc_train = true;     // train with the tensor-core pass (false: the FP32 pass)
	float *wsum = nullptr;    // device: total weight of the current batch
	float *loss = nullptr;    // device: weighted NLL of the last batch trained on
	float3 bmin{ 0, 0, 0 }, binv{ 1, 1, 1 };
	float lr = 1e-2f;
	float select_prob = 0.5f;
	uint32_t step = 0;              // Adam steps taken
	uint64_t waves = 0;             // waves trained on (moves the record offset)
	uint32_t train_paths = 32768;   // paths per batch: up to 32768 x 8 = 2^18 vertices at max_bounce 7
	uint32_t steps_per_wave = 64;   // batches (Adam steps) recorded and trained per wave: front-loaded
	uint32_t warmup_steps = 8;      // steps before the guide is first sampled
	bool product_target = true;     // fit Li * f * cos (the integrand) instead of Li
	uint32_t max_steps = 600;       // training budget in Adam steps (0: train every wave)
	uint32_t guided_bounces = 0;    // leading vertices that sample the guide (0: all but the last)
	bool learn_select = false;      // the network also outputs the per-vertex probability of sampling the guide
	uint32_t packed_step = ~0u;     // step whose weights Wp holds (~0: none)
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
	// One training step on recorded paths j0 .. j0+n_paths-1 of a wave (slots
	// j * stride + bounce; path j of the record is wave path rec_offset + j *
	// rec_stride, whose final radiance is L[path]): radiance targets, gradients
	// of the weighted NLL, Adam.
	void train_step( const float4 *L, uint32_t j0, uint32_t n_paths, uint32_t stride, uint32_t rec_offset,
					 uint32_t rec_stride, cudaStream_t st );
	// accumulate into gW, gb, ggrid over n record slots of r (weights in T.w, total
	// in wsum), with the tensor-core pass or the FP32 pass
	void gradients( const GuideRecords &r, uint32_t n, cudaStream_t st, bool tensor_cores );
	void adam( cudaStream_t st );  // update and clear the gradients
	void forward_batch( const float *d_in, uint32_t n, float *d_out, cudaStream_t st );
	void pack_weights( cudaStream_t st );  // W -> Wp and grid -> grid_pairs
	// BF16 tensor-core forward of n inputs {x, wo, n} (9 floats) to 64 outputs
	// each (d_out 16-byte aligned: stored as float4); returns the device error
	// word (0: no MMA timed out)
	uint32_t forward_batch_tc( const float *d_in, uint32_t n, float *d_out, cudaStream_t st );
	// records from n x stride floats {x, wo, n, w, weight[, bsdf pdf]} (device,
	// stride 13 or 14), for tests
	void load_records( const float *d_src, uint32_t n, uint32_t stride, cudaStream_t st );
};
}  // namespace cr
