// TEST INFRASTRUCTURE ONLY -- used when compiling the reference's own cpu::snn from its
// sources into oracle/_ref/ (see oracle/Makefile). Placed ahead of the reference's include
// path, this header stands in for spice/cpu/backend.h (spice/cpu/backend.h:8-53) with the
// same member set and behaviour, except for rand():
//
//   The reference draws its Poisson input from one sequential xoroshiro128p stream per net
//   (spice/cpu/backend.h:24). cpu::snn calls rand() exactly once per Poisson neuron per step,
//   in ascending neuron order (spice/models/brunel.h:40-45, spice/cpu/snn.h.cpp:145-153), so
//   the k-th call is (step = k / npoisson, neuron = k % npoisson). This backend answers that
//   call with the counter-based Philox draw the GPU path uses for the same (step, neuron),
//   which makes the two sides draw the very same numbers.
#pragma once

#include <spice/util/random.h>

#include "../../../philox.h"

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace oracle
{
// One net per library at a time: the harness sets these before constructing a net. Hidden,
// so that the two builds (parity and fast) loaded into one process keep separate counters
// (default-visibility inline variables would be merged across the libraries).
struct __attribute__( ( visibility( "hidden" ) ) ) counter_rng
{
	static inline uint64_t seed = 1;
	static inline uint64_t npoisson = 1;
	static inline uint64_t calls = 0;
};
} // namespace oracle

namespace spice
{
struct backend
{
	explicit backend( ulong_ seed ) { spice_assert( seed > 0 ); }

	template <typename T>
	static void atomic_add( T & var, T val )
	{
		var += val;
	}

	float rand()
	{
		uint64_t const k = oracle::counter_rng::calls++;
		uint32_t const neuron = static_cast<uint32_t>( k % oracle::counter_rng::npoisson );
		uint32_t const step = static_cast<uint32_t>( k / oracle::counter_rng::npoisson );
		return oracle::uniform_left_inc( oracle::neuron_u32( oracle::counter_rng::seed, neuron, step, 0 ) );
	}

	template <typename T>
	static T min( T x, T hi )
	{
		return std::min( x, hi );
	}

	template <typename T>
	static T max( T lo, T x )
	{
		return std::max( lo, x );
	}

	template <typename T>
	static T clamp( T x, T lo, T hi )
	{
		return min( hi, max( lo, x ) );
	}

	template <typename T>
	static T exp( T x )
	{
		return std::exp( x );
	}

	static float pow( float x, float y ) { return std::pow( x, y ); }
};
} // namespace spice
