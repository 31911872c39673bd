// Brunel network with the benchmark configuration's constants: after a spike the LIF
// neurons reset to 10 mV, and the synaptic efficacies are fixed, J = 0.1 mV excitatory and
// -0.5 mV inhibitory (g = 5). The reference's model (spice/models/brunel.h) resets to its
// resting potential, 0 mV (:48-54), and scales J by 20,000 / N (:70-75). The Poisson
// population (the first N / 2 neurons at 20 Hz), the 20 mV threshold, the 20 ms membrane
// time constant with leak towards 0 mV and the 20-step refractory period are the
// reference's, in the same operation order.
#pragma once

#include <spice/models/brunel.h>

namespace spice
{
struct brunel_fixed : model
{
	struct neuron : brunel::neuron
	{
		template <typename Iter, typename Backend>
		SPICE_HD static bool update( Iter n, float const dt, snn_info info, Backend & bak )
		{
			using util::get;
			float const inv_tau_mem = static_cast<float>( 1.0 / 0.02 );
			float const v_rest = 0.0f;
			float const v_reset = 0.01f;
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
					get<V>( n ) = v_reset;
					get<Twait>( n ) = t_refractory;
					return true;
				}
				get<V>( n ) += ( v_rest - get<V>( n ) ) * ( dt * inv_tau_mem );
			}
			return false;
		}

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int src, Iter dst, SynIter &&, snn_info info, Backend & bak )
		{
			using util::get;
			if( get<Twait>( dst ) <= 0 )
			{
				float const w_exc = 0.0001f;  // 0.1 mV
				float const w_inh = -0.0005f; // -0.5 mV
				bak.atomic_add( get<V>( dst ), src < excitatory_count( info ) ? w_exc : w_inh );
			}
		}
	};
};
} // namespace spice
