// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle (the checker), never the product.
//
// Philox-4x32-10 counter-based generator, restated from the published algorithm:
//   J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random numbers:
//   as easy as 1, 2, 3", SC'11 (section 3.2, the Philox S-box with 10 rounds).
// The GPU build carries its own independent copy (spice_b200/csrc/philox.cuh);
// the two are checked against each other and against the published known-answer
// vectors by the tests.
//
// Streams used by the simulator (both sides must agree):
//   key  = (seed & 0xffffffff, seed >> 32)
//   neuron draws : ctr = (neuron, step, call, 0x4E455552)   ('NEUR')
//   graph draws  : ctr = (src,    chunk, conn, 0x47524150)   ('GRAP')
// uniform_left_inc(x) = (x >> 8) / 2^24 exactly as the reference
// (spice/util/random.h:117-121).
#pragma once

#include <cstdint>

namespace oracle
{
struct philox_out
{
	uint32_t v[4];
};

inline void philox_mulhilo( uint32_t a, uint32_t b, uint32_t & hi, uint32_t & lo )
{
	uint64_t const p = static_cast<uint64_t>( a ) * b;
	hi = static_cast<uint32_t>( p >> 32 );
	lo = static_cast<uint32_t>( p );
}

inline philox_out philox4x32_10( uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1 )
{
	for( int r = 0; r < 10; r++ )
	{
		uint32_t hi0, lo0, hi1, lo1;
		philox_mulhilo( 0xD2511F53u, c0, hi0, lo0 );
		philox_mulhilo( 0xCD9E8D57u, c2, hi1, lo1 );
		uint32_t const n0 = hi1 ^ c1 ^ k0;
		uint32_t const n2 = hi0 ^ c3 ^ k1;
		c0 = n0;
		c1 = lo1;
		c2 = n2;
		c3 = lo0;
		k0 += 0x9E3779B9u;
		k1 += 0xBB67AE85u;
	}
	return { { c0, c1, c2, c3 } };
}

constexpr uint32_t TAG_NEURON = 0x4E455552u;
constexpr uint32_t TAG_GRAPH = 0x47524150u;

inline uint32_t neuron_u32( uint64_t seed, uint32_t neuron, uint32_t step, uint32_t call )
{
	return philox4x32_10(
	           neuron, step, call, TAG_NEURON, static_cast<uint32_t>( seed ), static_cast<uint32_t>( seed >> 32 ) )
	    .v[0];
}

// spice/util/random.h:117-121
inline float uniform_left_inc( uint32_t x ) { return ( x >> 8 ) / 16777216.0f; }
} // namespace oracle
