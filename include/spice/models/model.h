// The neuron / synapse model concept: plain C++ structs whose static member functions the
// simulator inlines into its kernels. Same shape as the reference's concept
// (spice/models/model.h:10-58): a model declares its per-neuron and per-synapse attributes
// as type lists and provides static init / update / receive functions templated on an
// iterator (get<I>(it) yields attribute I of one neuron or synapse) and a backend
// (rand, atomic_add, min, max, clamp, exp, pow).
//
// Two optional additions let the B200 kernels keep results identical to the reference
// CPU simulator while avoiding floating-point atomics:
//
//  * input classes (non-plastic models). If a neuron's receive() adds one of a few
//    constants chosen only by which class the source neuron falls in, and the classes are
//    contiguous ascending source-id ranges, the model declares
//        static constexpr int input_classes = K;
//        static int input_class( int src, snn_info );    // 0..K-1, non-decreasing in src
//        static int class_source( int cls, snn_info );   // any source id of class cls
//    The kernels then count arrivals per (destination, class) with integer shared-memory
//    atomics and replay them as class_source(0) x count0, class_source(1) x count1, ...
//    through the model's own receive(): the same floating-point additions, in the same
//    order, as the reference's ascending-source delivery. The replay calls receive() once
//    per class with a backend whose atomic_add(attr, value) adds `value` count times in
//    sequence, so a model with input classes must change state in receive() only through
//    one atomic_add whose value does not depend on the attribute it adds to.
//
//  * pair STDP with per-neuron traces (plastic models). See brunel_with_plasticity.h.
#pragma once

#include <spice/snn_info.h>

#include <cstddef>
#include <cstdint>
#include <tuple>

#if defined( __CUDACC__ )
#define SPICE_HD __host__ __device__
#else
#define SPICE_HD
#endif

namespace spice
{
namespace util
{
template <std::size_t I, typename... Ts>
struct nth_type;
template <typename T, typename... Ts>
struct nth_type<0, T, Ts...>
{
	using type = T;
};
template <std::size_t I, typename T, typename... Ts>
struct nth_type<I, T, Ts...>
{
	using type = typename nth_type<I - 1, Ts...>::type;
};

template <typename... Ts>
struct type_list
{
	using tuple_t = std::tuple<Ts...>;
	static constexpr std::size_t size = sizeof...( Ts );
	static constexpr std::size_t size_in_bytes = ( sizeof( Ts ) + ... + 0 );
	template <std::size_t I>
	using type = typename nth_type<I, Ts...>::type;
	// F<Ts...>, e.g. a register tuple of the attribute types
	template <template <typename...> class F>
	using apply = F<Ts...>;
};

// get<I>(iter): attribute I of the neuron/synapse the iterator points at.
template <int I, typename Iter>
SPICE_HD auto & get( Iter && it )
{
	return it.template get<I>();
}
} // namespace util

template <typename... Ts>
struct neuron : util::type_list<Ts...>
{
	static constexpr int input_classes = 0;

	template <typename Iter, typename Backend>
	SPICE_HD static void init( Iter, snn_info, Backend & )
	{
	}

	template <typename Iter, typename Backend>
	SPICE_HD static bool update( Iter, float, snn_info, Backend & )
	{
		return false;
	}

	template <typename Iter, typename SynIter, typename Backend>
	SPICE_HD static void receive( int, Iter, SynIter &&, snn_info, Backend & )
	{
	}
};

template <typename... Ts>
struct synapse : util::type_list<Ts...>
{
	static constexpr bool has_stdp = false;
	// the tuple synapses() exports (the reference's synapse tuple)
	using export_tuple_t = std::tuple<Ts...>;

	template <typename Iter, typename Backend>
	SPICE_HD static void init( Iter, int, int, snn_info, Backend & )
	{
	}

	SPICE_HD static bool plastic( int, int, snn_info ) { return false; }
};

struct model
{
	struct neuron : ::spice::neuron<>
	{
	};
	struct synapse : ::spice::synapse<>
	{
	};
};
} // namespace spice
