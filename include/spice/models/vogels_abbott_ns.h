// Vogels-Abbott network with the benchmark configuration's constants: conductance
// increments of 0.27 nS (excitatory) and 4.5 nS (inhibitory), and membrane potentials
// initialised uniformly in [-60, -50) mV. The reference's model (spice/models/vogels_abbott.h)
// keeps its conductances relative to the leak conductance (Gex, Gin are dimensionless:
// V += ((Vrest - V) + Gex (Eex - V) + Gin (Ein - V) + Ibg) dt / tau) and scales them as
// 0.4 * 16e6 / N^2 and 5.1 * 16e6 / N^2 (:76-82) with V = -60 mV at start (:24-29). Here the
// increments are 0.27 nS and 4.5 nS over the 10 nS leak of a 200 pF, 20 ms membrane, i.e.
// 0.027 and 0.45, and V starts at -60 mV + 10 mV x u with u the neuron's counter-based draw
// (the Backend's rand() at initialisation). Update, refractoriness and the operation order
// are the reference model's.
#pragma once

#include <spice/models/vogels_abbott.h>

namespace spice
{
struct vogels_abbott_ns : model
{
	struct neuron : vogels_abbott::neuron
	{
		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter n, snn_info, Backend & bak )
		{
			using util::get;
			float const v_rest = -0.06f, v_thresh = -0.05f;
			get<V>( n ) = v_rest + ( v_thresh - v_rest ) * bak.rand();
			get<Gex>( n ) = 0.0f;
			get<Gin>( n ) = 0.0f;
			get<Twait>( n ) = 0;
		}

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int src, Iter dst, SynIter &&, snn_info info, Backend & bak )
		{
			using util::get;
			float const g_leak = 10.0f;          // nS
			float const w_exc = 0.27f / g_leak;  // 0.27 nS
			float const w_inh = 4.5f / g_leak;   // 4.5 nS
			if( src < excitatory_count( info ) )
				bak.atomic_add( get<Gex>( dst ), w_exc );
			else
				bak.atomic_add( get<Gin>( dst ), w_inh );
		}
	};
};
} // namespace spice
