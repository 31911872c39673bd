// Brunel network with pair STDP and the benchmark configuration's depression amplitude
// A- = 0.012; the reference's model uses 0.0202 (spice/models/brunel_with_plasticity.h:
// 121-126). Everything else -- the neurons, the weights' initial values (0.1 mV
// excitatory, -0.5 mV inhibitory) and their clip range [0, 0.3 mV], A+ = 0.01, the 20 ms
// trace time constants, which synapses are plastic -- is the reference model's, in the
// same operation order.
#pragma once

#include <spice/models/brunel_with_plasticity.h>

namespace spice
{
struct brunel_with_plasticity_a012 : model
{
	struct neuron : brunel_with_plasticity::neuron
	{
	};

	struct synapse : brunel_with_plasticity::synapse
	{
		template <typename Backend>
		SPICE_HD static float update( float w, bool pre, bool post, float zpre, float zpost, float dt, Backend & bak )
		{
			float const inv_dt = 1.0f / dt;
			return bak.clamp(
			    w - pre * 0.012f * w * bak.exp( -zpost * inv_dt ) + post * 0.01f * ( 1.0f - w ) * bak.exp( -zpre * inv_dt ),
			    0.0f,
			    0.0003f );
		}
	};
};
} // namespace spice
