// Brunel network: the first half of the neurons are Poisson sources firing at 20 Hz, the
// rest are current-based LIF neurons (spice/models/brunel.h:9-83). Operation order follows
// the reference term by term.
#pragma once

#include <spice/models/model.h>

namespace spice
{
struct brunel : model
{
	struct neuron : ::spice::neuron<float, int>
	{
		enum attr
		{
			V,
			Twait
		};

		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter n, snn_info, Backend & )
		{
			using util::get;
			get<V>( n ) = 0.0f;
			get<Twait>( n ) = 0;
		}

		template <typename Iter, typename Backend>
		SPICE_HD static bool update( Iter n, float const dt, snn_info info, Backend & bak )
		{
			using util::get;
			float const inv_tau_mem = static_cast<float>( 1.0 / 0.02 );
			float const v_rest = 0.0f;
			int const t_refractory = 20; // steps
			float const v_thresh = 0.02f;

			if( n.id() < static_cast<unsigned>( info.num_neurons / 2 ) ) // Poisson source
			{
				float const rate = 20; // Hz
				return bak.rand() < ( rate * dt );
			}
			if( --get<Twait>( n ) <= 0 )
			{
				if( get<V>( n ) > v_thresh )
				{
					get<V>( n ) = v_rest;
					get<Twait>( n ) = t_refractory;
					return true;
				}
				get<V>( n ) += ( v_rest - get<V>( n ) ) * ( dt * inv_tau_mem );
			}
			return false;
		}

		SPICE_HD static int excitatory_count( snn_info info ) { return static_cast<int>( 0.9f * info.num_neurons ); }

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int src, Iter dst, SynIter &&, snn_info info, Backend & bak )
		{
			using util::get;
			if( get<Twait>( dst ) <= 0 )
			{
				float const w_exc = 0.0001f * 20'000 / info.num_neurons;
				float const w_inh = -0.0005f * 20'000 / info.num_neurons;
				bak.atomic_add( get<V>( dst ), src < excitatory_count( info ) ? w_exc : w_inh );
			}
		}

		// excitatory sources [0, 0.9 N), inhibitory [0.9 N, N)
		static constexpr int input_classes = 2;
		SPICE_HD static int input_class( int src, snn_info info ) { return src < excitatory_count( info ) ? 0 : 1; }
		SPICE_HD static int class_source( int cls, snn_info info ) { return cls == 0 ? 0 : excitatory_count( info ); }
	};
};
} // namespace spice
