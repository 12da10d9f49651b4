// Host-side launch interface of the CUDA kernels (render.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/cr.h"
#include "cr_common.h"
#include "guide.h"

namespace cr
{
// Per-path SoA state of one wave, sized for `capacity` paths.
struct BatchWave;

struct WaveBuffers
{
	uint32_t capacity = 0;
	float4 *ray_o = nullptr, *ray_d = nullptr;  // (o, tmin), (d, tmax)
	HitRec *hit = nullptr;
	float4 *beta = nullptr;                     // (throughput, previous BSDF pdf)
	float4 *L = nullptr;                        // (radiance, -)
	uint32_t *queue[ 2 ] = { nullptr, nullptr };
	uint32_t *shadow_queue = nullptr;
	float4 *sh_o = nullptr, *sh_d = nullptr, *sh_c = nullptr;
	uint32_t *counters = nullptr;               // per bounce b, CPB entries: see CNT_* below
	uint32_t n_counters = 0;
	uint32_t *err = nullptr;                    // device error word
	unsigned long long *work = nullptr;         // extension [0] nodes [1] triangles, shadow [2] [3]
	uint4 *lobes = nullptr;                     // guided renders: 8 lobes x (mean, kappa, weight) per path,
	                                            // FP16, and the guide's selection probability: 6 x 16 bytes per path
	uint32_t *path_job = nullptr;               // batched renders: the job (scene render) of each path
	unsigned long long *tally = nullptr;        // batched renders: closest-hit and shadow rays traced
	uint32_t *binned = nullptr;                 // ray binning: the sorted queue of one traversal launch
	uint32_t *bins = nullptr;                   // ray binning: per-bin counts, then offsets (N_BINS)
	BatchWave *bwave = nullptr;                 // batched renders: the current wave
};

// One scene's render inside a batch (device copy).  A job renders its whole
// image; its samples are global samples first_sample .. + width*height*spp,
// pixel-major, and its pixels global pixels first_pixel .. + width*height.
struct BatchJobDev
{
	uint64_t first_sample, first_pixel;
	uint32_t width, height, spp, pad;
	uint64_t seed;
	double *sum, *sumsq;
	uint32_t *count;
};

// The current wave of a batched render, in device memory: the kernels of a
// wave read it, so that one captured wave body serves every wave.
struct BatchWave
{
	uint64_t first;   // first global sample of the wave
	uint64_t p0, p1;  // first and last global pixel of the wave's samples (p0 > p1: none)
	uint32_t n;       // samples in the wave
	uint32_t index;   // wave number
};

struct BatchDev
{
	const DevScene *scenes;        // one per job, with the job's camera
	const BatchJobDev *jobs;
	const uint64_t *seed_offset;   // added to every job's seed (changes between graph replays)
	uint32_t n_jobs;
};

// Device counters per bounce: queue lengths and the traversal kernels' work cursors.
constexpr uint32_t CPB = 4;
constexpr uint32_t CNT_EXT = 0, CNT_SHADOW = 1, CNT_EXT_CURSOR = 2, CNT_SHADOW_CURSOR = 3;
inline constexpr uint32_t n_counters_for( uint32_t max_bounce ) { return CPB * ( max_bounce + 3 ); }

// The reference's kernel registry (src/core/kernel/kernel.impl.cu:10-15).
enum : int32_t
{
	KERNEL_RADIANCE = 0,
	KERNEL_NORMAL = 1,      // NormalKernel (normal.hpp:17-31)
	KERNEL_VISIBILITY = 2,  // VisibilityKernel (visibility.hpp:17-41)
	KERNEL_HALFVECTOR = 3   // HalfVectorKernel (halfVector.hpp:17-43)
};

// Per-bounce profile of a profiled render (cr_render_profile), device arrays:
// one slice per sample of the window, `depth` bounce records per sample.
struct ProfileDev
{
	cr_profile_slice *slices = nullptr;
	cr_profile_bounce *bounces = nullptr;
	uint32_t depth = 0;
};

struct RenderConfig
{
	uint32_t spp, max_bounce;
	int32_t estimator;
	int32_t kernel = KERNEL_RADIANCE;
	uint32_t x0, y0, ww, wh;  // window origin and size
	uint64_t seed;
	uint32_t wave_paths;
	bool count_work;
	bool guiding = false;            // learned guide: records and training (MIS estimator)
	bool guide_sample = false;       // guided renders: sample the guide (off while it warms up)
	GuideDev guide{};
	// Training records of one wave: the vertices of paths rec_offset + j * rec_stride,
	// j < rec_paths, at slots j * (max_bounce + 1) + bounce.  The paths are spread over
	// the whole wave (a wave is pixel-major) and the offset moves from wave to wave.
	GuideRecords rec{};
	uint32_t rec_paths = 0, rec_stride = 1, rec_offset = 0;
	uint32_t refill_min = 16;        // traversal: idle lanes per warp that trigger a refill (1..32)
	int traverse_blocks_per_sm = 8;  // traversal grid = SMs x this (1..8; 128-thread blocks)
	uint32_t shade_threads = 128;    // shading block size (64, 128 or 256); grid of SMs x 1024 threads
	uint32_t rr_start = 4;           // MIS estimator: first bounce at which Russian roulette may end a path
	bool bin_rays = false;           // sort secondary and shadow queues by (octant, origin cell) before tracing
	uint32_t shadow_vote = 4;        // any-hit traversal: triangle step once this x (lanes wanting one) >= active lanes
	uint32_t shadow_refill_min = 0;  // any-hit traversal: idle lanes that trigger a refill (0: refill_min)
	ProfileDev prof{};               // profiled renders (reference estimator, Radiance kernel)
};

struct StageTimes
{
	double extend = 0, shadow = 0, shade = 0, other = 0, total = 0, guide = 0, guide_train = 0;
	uint32_t launches = 0, waves = 0, extend_launches = 0, shadow_launches = 0, guide_launches = 0;
	uint64_t rays_extend = 0, rays_shadow = 0, nodes = 0, tris = 0, shadow_nodes = 0, shadow_tris = 0, guide_rows = 0;
};

void alloc_wave( WaveBuffers &wb, uint32_t capacity, uint32_t max_bounce, cudaStream_t st );
// The current device's memory pool for wave state, and a hand-back of the
// memory that the pools keep mapped.
cudaMemPool_t device_pool();
void trim_device_pools();
void free_wave( WaveBuffers &wb, cudaStream_t st );

// Render the window into the film (device buffers, accumulated).  When
// `times` is not null, stage times are measured with CUDA events and the
// call synchronises `st` at the end.
void render_waves( const DevScene &sc, const RenderConfig &cfg, WaveBuffers &wb, double *film_sum,
				   double *film_sumsq, uint32_t *film_count, cudaStream_t st, StageTimes *times,
				   GuideState *guide = nullptr );
void alloc_lobes( WaveBuffers &wb, cudaStream_t st );
void alloc_bins( WaveBuffers &wb, cudaStream_t st );  // ray binning buffers (RenderConfig::bin_rays)
void alloc_batch_state( WaveBuffers &wb, cudaStream_t st );

// Batched render of many scenes: the waves run over the concatenated samples
// of all jobs, so one launch per stage serves every scene.  `jobs` is the host
// copy of the device table.  cfg carries the launch configuration, the
// estimator and max_bounce (window and spp fields are unused).  The host
// issues every wave's kernels; `times` (when not null) gets the stage times.
void render_batch_waves( const BatchDev &bd, const BatchJobDev *jobs, uint32_t n_jobs, const RenderConfig &cfg,
						 WaveBuffers &wb, cudaStream_t st, StageTimes *times );

// The same render as one CUDA graph: an initialising kernel, then a
// conditional WHILE node whose body is one wave's kernels (the wave's index
// lives in device memory; the body's last kernel advances it and ends the loop
// after the last wave).  The graph is built with stream captures on `st`
// (which must not be capturing).  Returns the kernel nodes of the graph, the
// body counted once.
uint32_t build_batch_graph( const BatchDev &bd, const BatchJobDev *jobs, uint32_t n_jobs, const RenderConfig &cfg,
							WaveBuffers &wb, cudaStream_t st, cudaGraph_t *out );

void launch_trace( const DevScene &sc, const float *rays, uint64_t n, int any_hit,
				   cr_hit *out, uint32_t *err, cudaStream_t st, unsigned long long *work = nullptr );

void launch_bsdf_eval( int estimator, const DevShader &sh, const float *wo, const float *wi, uint64_t n, float *f,
					   float *pdf, cudaStream_t st );
void launch_bsdf_sample( int estimator, const DevShader &sh, const float *wo, const float *u, uint64_t n, float *wi,
						 float *weight, float *pdf, cudaStream_t st );
// Shader::execute of tab[0] (target 0 compute_f_by_wi_wo, 1 sample_wi_f_by_wo),
// k scripted uniforms per sample; device arrays.
void launch_shader_execute( const DevShader *tab, int target, const float *wo, float *wi, const float *u, uint32_t k,
							uint64_t n, float *f, float *emission, uint32_t *used, cudaStream_t st );

// Philox4x32-10 of the render (cr_device.cuh) on n (c0..c3, k0, k1) device
// words; out n x 4 device words.
void launch_philox( const uint32_t *ctr_key, uint64_t n, uint32_t *out, cudaStream_t st );

// SMs of the current device (cached per device).
int sm_count();

// Raises the dynamic shared-memory limit of kernel `fn` to `bytes` on the
// current device.  The attribute belongs to a device's context, so it is set
// once per (device, kernel); thread-safe.
void ensure_smem_limit( const void *fn, int bytes, const char *what );
}  // namespace cr
