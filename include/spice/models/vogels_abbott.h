// Vogels-Abbott conductance-based LIF network, the reference's parameter set
// (spice/models/vogels_abbott.h:9-91). The arithmetic below keeps the reference's
// operation order term by term: results are bit-identical to its CPU simulator when both
// sides compile without floating-point contraction.
#pragma once

#include <spice/models/model.h>

namespace spice
{
struct vogels_abbott : model
{
	struct neuron : ::spice::neuron<float, float, float, int>
	{
		enum attr
		{
			V,
			Gex,
			Gin,
			Twait
		};

		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter n, snn_info, Backend & )
		{
			using util::get;
			get<V>( n ) = -0.06f; // resting potential, volt
			get<Gex>( n ) = 0.0f;
			get<Gin>( n ) = 0.0f;
			get<Twait>( n ) = 0;
		}

		template <typename Iter, typename Backend>
		SPICE_HD static bool update( Iter n, float const dt, snn_info, Backend & )
		{
			using util::get;
			int const t_refractory = 50; // steps
			float const v_rest = -0.06f;
			float const v_thresh = -0.05f;
			float const inv_tau_mem = 1.0f / 0.02f;
			float const e_exc = 0.0f;
			float const e_inh = -0.08f;
			float const i_bg = 0.02f;
			float const inv_tau_exc = 1.0f / 0.005f;
			float const inv_tau_inh = 1.0f / 0.01f;

			bool fired = false;
			if( --get<Twait>( n ) <= 0 )
			{
				if( get<V>( n ) > v_thresh )
				{
					get<V>( n ) = v_rest;
					get<Twait>( n ) = t_refractory;
					fired = true;
				}
				else
				{
					float const v = get<V>( n );
					get<V>( n ) +=
					    ( ( v_rest - v ) + get<Gex>( n ) * ( e_exc - v ) + get<Gin>( n ) * ( e_inh - v ) + i_bg ) *
					    ( dt * inv_tau_mem );
				}
			}
			get<Gex>( n ) -= get<Gex>( n ) * ( dt * inv_tau_exc );
			get<Gin>( n ) -= get<Gin>( n ) * ( dt * inv_tau_inh );
			return fired;
		}

		SPICE_HD static int excitatory_count( snn_info info ) { return static_cast<int>( 0.8f * info.num_neurons ); }

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int src, Iter dst, SynIter &&, snn_info info, Backend & bak )
		{
			using util::get;
			float const n2 = static_cast<float>( static_cast<long long>( info.num_neurons ) * info.num_neurons );
			float const w_exc = 0.4f * 16'000'000 / n2;
			float const w_inh = 5.1f * 16'000'000 / n2;
			if( src < excitatory_count( info ) )
				bak.atomic_add( get<Gex>( dst ), w_exc );
			else
				bak.atomic_add( get<Gin>( dst ), w_inh );
		}

		// two input classes: excitatory sources [0, 0.8 N), inhibitory [0.8 N, N)
		static constexpr int input_classes = 2;
		SPICE_HD static int input_class( int src, snn_info info ) { return src < excitatory_count( info ) ? 0 : 1; }
		SPICE_HD static int class_source( int cls, snn_info info ) { return cls == 0 ? 0 : excitatory_count( info ); }
	};
};
} // namespace spice
