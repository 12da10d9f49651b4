// Harness replacement for the reference's host Sampler
// (src/core/misc/sampler.hpp:22-36 and :95-130 in xlnx/cuda-raytracer).
//
// This file sits earlier on the include path than the reference's `src/`, so
// every `#include <core/misc/sampler.hpp>` in the reference resolves here.
// The public interface (sample/sample2/sample3/sample4, SamplerGenerator::create)
// matches the reference; the generator arithmetic is the same 48-bit linear
// congruential step (multiplier 0x5DEECE66D, increment 0xB,16 = 0xB16, output
// bits 47..16 scaled by 2^-32).  The one deliberate deviation: the reference
// keeps a single process-wide static state seeded from time() and shared by all
// tracer threads (a data race, and no two runs alike).  Here each thread owns its
// state, seeded deterministically from harness_seed() and a per-thread index, so
// light-point tables and parity runs are reproducible.  A thread may also
// script its draws (harness_rng::script()), which the harness's `shade`
// command uses to run one Shader::execute on known numbers.
#pragma once

#include <atomic>
#include <cstdint>
#include <vec/vmath.hpp>
#include <core/basic/basic.hpp>

namespace koishi
{
namespace core
{
namespace harness_rng
{
inline std::atomic<uint64_t> &base_seed()
{
	static std::atomic<uint64_t> s{ 0x1234ABCDull };
	return s;
}
inline std::atomic<uint64_t> &thread_counter()
{
	static std::atomic<uint64_t> c{ 0 };
	return c;
}
inline uint64_t mix64( uint64_t z )
{
	z += 0x9E3779B97F4A7C15ull;
	z = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
	z = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
	return z ^ ( z >> 31 );
}
struct State
{
	uint64_t x;
	bool init = false;
};
inline State &state()
{
	thread_local State st;
	if ( !st.init )
	{
		uint64_t k = thread_counter().fetch_add( 1 );
		st.x = mix64( base_seed().load() ^ mix64( k + 1 ) ) & 0xFFFFFFFFFFFFull;
		st.init = true;
	}
	return st;
}
// Scripted draws of the calling thread: while u is set, sample() hands out
// u[0..n) in order (0.5 past the end) and counts them in used.
struct Script
{
	const float *u = nullptr;
	uint32_t n = 0, used = 0;
};
inline Script &script()
{
	thread_local Script sc;
	return sc;
}
// Set the calling thread's 48-bit state exactly (used before the scene is
// built so that Mesh::generateSamples draws a known sequence).
inline void seed_this_thread( uint64_t x48 )
{
	state().x = x48 & 0xFFFFFFFFFFFFull;
}
}  // namespace harness_rng

struct SamplerGenerator;

struct Sampler
{
	friend struct SamplerGenerator;

	float sample()
	{
		auto &sc = harness_rng::script();
		if ( sc.u )
		{
			float v = sc.used < sc.n ? sc.u[ sc.used ] : 0.5f;
			++sc.used;
			return v;
		}
		auto &st = harness_rng::state();
		st.x = ( 0x5DEECE66Dull * st.x + 0xB16ull ) & 0xFFFFFFFFFFFFull;
		unsigned int x = unsigned( st.x >> 16 );
		return (float)x / (float)0x100000000LL;
	}
	float2 sample2()
	{
		float a = sample();
		float b = sample();
		return float2{ a, b };
	}
	float3 sample3()
	{
		float a = sample();
		float b = sample();
		float c = sample();
		return float3{ a, b, c };
	}
	float4 sample4()
	{
		float a = sample();
		float b = sample();
		float c = sample();
		float d = sample();
		return float4{ a, b, c, d };
	}

	Sampler() = default;
};

struct SamplerGenerator : emittable
{
	SamplerGenerator() = default;
	Sampler create() const { return Sampler(); }
};

}  // namespace core

}  // namespace koishi
