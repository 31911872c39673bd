// Device-side building blocks shared by the kernels:
//  * Philox-4x32-10 (Salmon et al., SC'11) -- the counter-based generator behind the
//    Poisson draws and the graph generator. Streams:
//        key = (seed lo, seed hi)
//        neuron draw  ctr = (neuron, step, call, 'NEUR')
//        graph draw   ctr = (src, candidate / 4, connection, 'GRAP')
//  * reg_tuple: a neuron's attributes held in registers, with get<I>()
//  * device_backend: the Backend a model sees inside the kernels
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace spk
{
constexpr uint32_t TAG_NEURON = 0x4E455552u;
constexpr uint32_t TAG_GRAPH = 0x47524150u;

struct u32x4
{
	uint32_t x, y, z, w;
};

__device__ __forceinline__ u32x4 philox4x32_10( u32x4 c, uint32_t k0, uint32_t k1 )
{
#pragma unroll
	for( int r = 0; r < 10; r++ )
	{
		uint32_t const lo0 = 0xD2511F53u * c.x;
		uint32_t const hi0 = __umulhi( 0xD2511F53u, c.x );
		uint32_t const lo1 = 0xCD9E8D57u * c.z;
		uint32_t const hi1 = __umulhi( 0xCD9E8D57u, c.z );
		c = { hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
		k0 += 0x9E3779B9u;
		k1 += 0xBB67AE85u;
	}
	return c;
}

// uniform in [0, 1) with 24 random bits (spice/util/random.h:117-121)
__device__ __forceinline__ float uniform_left_inc( uint32_t x ) { return ( x >> 8 ) / 16777216.0f; }

// A fixed-size heterogeneous tuple held in registers.
template <typename... Ts>
struct reg_tuple;
template <>
struct reg_tuple<>
{
};
template <typename T, typename... Ts>
struct reg_tuple<T, Ts...>
{
	T head;
	reg_tuple<Ts...> tail;
};

template <int I>
struct tuple_at
{
	template <typename T, typename... Ts>
	__device__ __forceinline__ static auto & get( reg_tuple<T, Ts...> & t )
	{
		return tuple_at<I - 1>::get( t.tail );
	}
};
template <>
struct tuple_at<0>
{
	template <typename T, typename... Ts>
	__device__ __forceinline__ static T & get( reg_tuple<T, Ts...> & t )
	{
		return t.head;
	}
};

template <typename List>
struct reg_tuple_of;
template <template <typename...> class L, typename... Ts>
struct reg_tuple_of<L<Ts...>>
{
	using type = reg_tuple<Ts...>;
};

// Iterator over one neuron whose attributes live in a reg_tuple.
template <typename Tuple>
struct reg_iter
{
	Tuple & t;
	uint32_t i;
	template <int I>
	__device__ __forceinline__ auto & get() const
	{
		return tuple_at<I>::get( t );
	}
	__device__ __forceinline__ uint32_t id() const { return i; }
};

// Iterator over one synapse weight held in a register (plastic receive).
struct weight_iter
{
	float w;
	template <int I>
	__device__ __forceinline__ float const & get() const
	{
		return w;
	}
};

// Iterator over one synapse weight, writable (synapse::init).
struct weight_iter_rw
{
	float & w;
	template <int I>
	__device__ __forceinline__ float & get() const
	{
		return w;
	}
};

struct null_syn_iter
{
};

// The Backend models see on the device. rand() is the counter-based draw for
// (seed, neuron, step, call); atomic_add is a plain add because every neuron's state is
// owned by exactly one thread; min/max/clamp follow std::min/std::max argument semantics
// (spice/cpu/backend.h:28-44) so signed zeros and ties resolve like the reference's CPU.
struct device_backend
{
	uint32_t k0, k1, neuron, step, calls;

	__device__ __forceinline__ device_backend( uint64_t seed, uint32_t neuron_, uint32_t step_ )
	    : k0( static_cast<uint32_t>( seed ) )
	    , k1( static_cast<uint32_t>( seed >> 32 ) )
	    , neuron( neuron_ )
	    , step( step_ )
	    , calls( 0 )
	{
	}

	__device__ __forceinline__ float rand()
	{
		u32x4 const r = philox4x32_10( { neuron, step, calls++, TAG_NEURON }, k0, k1 );
		return uniform_left_inc( r.x );
	}

	template <typename T>
	__device__ __forceinline__ static void atomic_add( T & var, T val )
	{
		var += val;
	}

	template <typename T>
	__device__ __forceinline__ static T min( T x, T hi )
	{
		return ( hi < x ) ? hi : x;
	}
	template <typename T>
	__device__ __forceinline__ static T max( T lo, T x )
	{
		return ( lo < x ) ? x : lo;
	}
	template <typename T>
	__device__ __forceinline__ static T clamp( T x, T lo, T hi )
	{
		return min( hi, max( lo, x ) );
	}
	__device__ __forceinline__ static float exp( float x ) { return expf( x ); }
	__device__ __forceinline__ static float pow( float x, float y ) { return powf( x, y ); }
};

// Backend for replaying `times` identical arrivals through one receive() call: its
// atomic_add performs the `times` additions one after another -- the same sequence of
// roundings as `times` separate calls -- while the rest of receive() (conditions,
// constants) runs once. Valid for receive() functions that change state only through
// one atomic_add whose value does not depend on the attribute it adds to (the input-class
// contract of include/spice/models/model.h).
struct repeat_backend : device_backend
{
	unsigned times;
	__device__ __forceinline__ repeat_backend( uint64_t seed, uint32_t neuron_, uint32_t step_, unsigned times_ )
	    : device_backend( seed, neuron_, step_ )
	    , times( times_ )
	{
	}
	template <typename T>
	__device__ __forceinline__ void atomic_add( T & var, T val ) const
	{
		T v = var;
		for( unsigned r = 0; r < times; r++ ) v += val;
		var = v;
	}
};

// Kahan-compensated clock (spice/snn.cpp:38-44, spice/util/numeric.h:9-33): the dt a step
// hands to the models is the compensated delta.
struct clock_state
{
	long long step;
	float c;
	float sum;
	unsigned int done; // CTAs that finished the current launch
	unsigned int pad;
};

__device__ __forceinline__ float kahan_add( float & c, float & sum, float d )
{
	float const y = __fsub_rn( d, c );
	float const t = __fadd_rn( sum, y );
	c = __fsub_rn( __fsub_rn( t, sum ), y );
	sum = t;
	return y;
}

__device__ __forceinline__ int warp_inclusive_scan( int x )
{
	int const lane = threadIdx.x & 31;
#pragma unroll
	for( int o = 1; o < 32; o <<= 1 )
	{
		int const y = __shfl_up_sync( 0xffffffffu, x, o );
		if( lane >= o ) x += y;
	}
	return x;
}

// Exclusive scan of one int per thread over the block; returns the prefix, *total gets the
// sum. `scratch` holds >= 33 ints of shared memory. Ends with a __syncthreads.
__device__ __forceinline__ int block_exclusive_scan( int x, int * scratch, int * total )
{
	int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = ( blockDim.x + 31 ) >> 5;
	int const incl = warp_inclusive_scan( x );
	if( lane == 31 ) scratch[warp] = incl;
	__syncthreads();
	if( warp == 0 )
	{
		int v = lane < nwarps ? scratch[lane] : 0;
		int const vi = warp_inclusive_scan( v );
		scratch[lane] = vi - v;
		if( lane == 31 ) scratch[32] = vi;
	}
	__syncthreads();
	int const r = scratch[warp] + incl - x;
	*total = scratch[32];
	__syncthreads();
	return r;
}
} // namespace spk
