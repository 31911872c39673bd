// Brunel network with pair STDP on excitatory->excitatory synapses
// (spice/models/brunel_with_plasticity.h:9-138).
//
// The reference stores three attributes per synapse (W, Zpre, Zpost) and updates every
// plastic synapse every step on the CPU (spice/cpu/snn.h.cpp:161-179). Zpre only ever sees
// the source's delayed spikes and Zpost only the target's spikes, both start at 1.0 and
// both decay by the same factor, so every plastic synapse leaving neuron s carries the
// same Zpre and every plastic synapse entering d the same Zpost: they are per-neuron
// traces. This model therefore stores W per synapse and the two traces per neuron; the
// simulator updates the traces every step (bit-identical to the reference's per-synapse
// values) and touches W only when a step's update would change it (see update() and
// the *_active() tests below). synapses() re-expands (W, Zpre, Zpost) for export.
#pragma once

#include <spice/models/brunel.h>
#include <spice/models/model.h>

namespace spice
{
struct brunel_with_plasticity : model
{
	enum neuron_attr
	{
		V,
		Twait
	};
	enum syn_attr
	{
		W
	};

	struct neuron : ::spice::neuron<float, int>
	{
		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter n, snn_info info, Backend & bak )
		{
			brunel::neuron::init( n, info, bak );
		}

		template <typename Iter, typename Backend>
		SPICE_HD static bool update( Iter n, float const dt, snn_info info, Backend & bak )
		{
			return brunel::neuron::update( n, dt, info, bak );
		}

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int, Iter dst, SynIter && syn, snn_info info, Backend & bak )
		{
			using util::get;
			if( get<Twait>( dst ) <= 0 ) bak.atomic_add( get<V>( dst ), get<W>( syn ) * 20'000 / info.num_neurons );
		}
	};

	struct synapse : ::spice::synapse<float>
	{
		static constexpr bool has_stdp = true;
		// exported as the reference's (W, Zpre, Zpost)
		using export_tuple_t = std::tuple<float, float, float>;

		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter syn, int src, int, snn_info info, Backend & )
		{
			using util::get;
			get<W>( syn ) = src < static_cast<int>( 0.9f * info.num_neurons ) ? 0.0001f : -0.0005f;
		}

		// brunel_with_plasticity.h:129-135, written as a product of a source and a target test
		SPICE_HD static bool plastic_src( int src, snn_info info )
		{
			return src >= info.num_neurons / 2 && src < 9 * info.num_neurons / 10;
		}
		SPICE_HD static bool plastic_dst( int dst, snn_info info ) { return dst < 9 * info.num_neurons / 10; }
		SPICE_HD static bool plastic( int src, int dst, snn_info info )
		{
			return plastic_src( src, info ) && plastic_dst( dst, info );
		}

		// Per-neuron traces: Z <- fma(Z, decay(dt), spiked), starting at trace_init. The
		// reference multiplies by pow(1 - dt / 0.02, nsteps) with nsteps = 1 on its CPU path,
		// and pow(x, 1) == x.
		static constexpr float trace_init = 1.0f;
		SPICE_HD static float trace_decay( float dt ) { return 1 - dt * ( 1.0f / 0.02f ); }

		// One step of the reference's synapse update given this step's traces
		// (brunel_with_plasticity.h:102-127), weights clipped to [0, 0.3 mV].
		template <typename Backend>
		SPICE_HD static float update( float w, bool pre, bool post, float zpre, float zpost, float dt, Backend & bak )
		{
			float const inv_dt = 1.0f / dt;
			return bak.clamp(
			    w - pre * 0.0202f * w * bak.exp( -zpost * inv_dt ) + post * 0.01f * ( 1.0f - w ) * bak.exp( -zpre * inv_dt ),
			    0.0f,
			    0.0003f );
		}

		// For w inside the clip range, update(w, pre, post, ...) == w whenever the
		// depression term is off (pre == false or exp(-zpost/dt) == 0) and the potentiation
		// term is off (post == false or exp(-zpre/dt) == 0). These two tests decide it.
		template <typename Backend>
		SPICE_HD static bool depression_active( float zpost, float dt, Backend & bak )
		{
			return bak.exp( -zpost * ( 1.0f / dt ) ) != 0.0f;
		}
		template <typename Backend>
		SPICE_HD static bool potentiation_active( float zpre, float dt, Backend & bak )
		{
			return bak.exp( -zpre * ( 1.0f / dt ) ) != 0.0f;
		}
	};
};
} // namespace spice
