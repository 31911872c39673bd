// The models compiled into the library, by their C-ABI id (spk_model in spice_b200.h), and
// what the host needs to know about each. The reference selects its models the same way:
// every model is a compile-time template argument instantiated in the library
// (spice/cuda/snn.d.cpp:247-250).
#pragma once

#include <spice/models/brunel.h>
#include <spice/models/brunel_fixed.h>
#include <spice/models/brunel_with_plasticity.h>
#include <spice/models/brunel_with_plasticity_a012.h>
#include <spice/models/synth.h>
#include <spice/models/vogels_abbott.h>
#include <spice/models/vogels_abbott_ns.h>
#include <spice_b200.h>

// a model compiled in beside the library's own (a user build, the tests' model): the
// header that defines it (SPK_USER_MODEL_HEADER) and its type (SPK_USER_MODEL), C-ABI id
// SPK_USER_MODEL_ID
#if defined( SPK_USER_MODEL_HEADER ) && defined( SPK_USER_MODEL )
#include SPK_USER_MODEL_HEADER
#define SPK_HAS_USER_MODEL 1
#endif

#include <type_traits>

namespace spk
{
template <typename M>
struct model_tag
{
	using type = M;
};

#if defined( SPK_HAS_USER_MODEL )
constexpr int MODEL_COUNT = SPK_USER_MODEL_ID + 1;
#else
constexpr int MODEL_COUNT = SPK_USER_MODEL_ID;
#endif

// f(model_tag<Model>{}) for the model with C-ABI id `model`; false if there is none
template <typename F>
bool with_model( int model, F && f )
{
	switch( model )
	{
	case SPK_VOGELS_ABBOTT: f( model_tag<spice::vogels_abbott>{} ); return true;
	case SPK_BRUNEL: f( model_tag<spice::brunel>{} ); return true;
	case SPK_BRUNEL_PLUS: f( model_tag<spice::brunel_with_plasticity>{} ); return true;
	case SPK_SYNTH: f( model_tag<spice::synth>{} ); return true;
	case SPK_VOGELS_ABBOTT_NS: f( model_tag<spice::vogels_abbott_ns>{} ); return true;
	case SPK_BRUNEL_FIXED: f( model_tag<spice::brunel_fixed>{} ); return true;
	case SPK_BRUNEL_PLUS_A012: f( model_tag<spice::brunel_with_plasticity_a012>{} ); return true;
#if defined( SPK_HAS_USER_MODEL )
	case SPK_USER_MODEL_ID: f( model_tag<SPK_USER_MODEL>{} ); return true;
#endif
	default: return false;
	}
}

template <typename Model>
constexpr bool is_plastic_model = Model::synapse::has_stdp;
// models the counting kernels (window_flat, window_slots, window_counts) run: input classes,
// no plasticity, no synapse attributes (the counts replay knows only the source's class)
template <typename Model>
constexpr bool is_flat_model = Model::neuron::input_classes > 0 && !Model::synapse::has_stdp && Model::synapse::size == 0;
// models that only the generic kernel (window_ordered) runs: the other non-plastic ones
template <typename Model>
constexpr bool needs_ordered = !Model::synapse::has_stdp && !is_flat_model<Model>;

struct model_traits
{
	bool plastic;
	bool ordered;      // runs on window_ordered only (needs_ordered)
	int classes;       // input classes (0 for plastic models and the models window_ordered runs)
	int neuron_attrs;
	int synapse_attrs; // as exported (the reference's synapse tuple)
	char types[16];    // 'f' / 'i' per neuron attribute, then per exported synapse attribute
};

template <typename T>
constexpr char type_char()
{
	return std::is_floating_point<T>::value ? 'f' : 'i';
}
template <typename Tuple, std::size_t... I>
void tuple_chars( char * out, std::index_sequence<I...> )
{
	( ( out[I] = type_char<std::tuple_element_t<I, Tuple>>() ), ... );
}

template <typename Model>
model_traits traits_of()
{
	using N = typename Model::neuron;
	using E = typename Model::synapse::export_tuple_t;
	model_traits t{};
	t.plastic = is_plastic_model<Model>;
	t.ordered = needs_ordered<Model>;
	t.classes = is_flat_model<Model> ? N::input_classes : 0;
	t.neuron_attrs = (int)N::size;
	t.synapse_attrs = (int)std::tuple_size<E>::value;
	static_assert( N::size + std::tuple_size<E>::value < sizeof( model_traits::types ), "too many attributes" );
	tuple_chars<typename N::tuple_t>( t.types, std::make_index_sequence<N::size>() );
	tuple_chars<E>( t.types + t.neuron_attrs, std::make_index_sequence<std::tuple_size<E>::value>() );
	return t;
}
} // namespace spk
