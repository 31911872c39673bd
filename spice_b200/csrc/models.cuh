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

#include <type_traits>

namespace spk
{
template <typename M>
struct model_tag
{
	using type = M;
};

constexpr int MODEL_COUNT = 7;

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
	default: return false;
	}
}

template <typename Model>
constexpr bool is_plastic_model = Model::synapse::has_stdp;
// models the window_flat kernels run: input classes, no plasticity
template <typename Model>
constexpr bool is_flat_model = Model::neuron::input_classes > 0 && !Model::synapse::has_stdp;

struct model_traits
{
	bool plastic;
	int classes;       // input classes (0 for plastic models)
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
	t.classes = t.plastic ? 0 : N::input_classes;
	t.neuron_attrs = (int)N::size;
	t.synapse_attrs = t.plastic ? (int)std::tuple_size<E>::value : 0;
	tuple_chars<typename N::tuple_t>( t.types, std::make_index_sequence<N::size>() );
	if( t.plastic ) tuple_chars<E>( t.types + t.neuron_attrs, std::make_index_sequence<std::tuple_size<E>::value>() );
	return t;
}
} // namespace spk
