// TEST MODEL -- defined only for the tests of the generic window kernel (window_ordered).
//
// A current-based LIF neuron driven by a per-neuron bias, whose synapses carry a static
// weight each: receive() adds the synapse's own weight, so the input sum depends on every
// synapse and on the order of the additions. It has no input classes, so the counting
// kernels cannot run it. It is written against the model concept only
// (spice/models/model.h): the same header compiles into a build of the B200 library
// (spice_b200.build.build_user) and, as the oracle, into the reference's CPU simulator
// (oracle/Makefile, target `user`).
#pragma once

#include <spice/models/model.h>
#include <spice/snn_info.h>

#if defined( __CUDACC__ )
#define WLIF_HD __host__ __device__
#else
#define WLIF_HD
#endif

namespace test_models
{
struct weighted_lif : ::spice::model
{
	struct neuron : ::spice::neuron<float, float, int>
	{
		enum attr
		{
			V,
			I,
			Twait
		};

		template <typename Iter, typename Backend>
		WLIF_HD static void init( Iter n, ::spice::snn_info, Backend & )
		{
			using ::spice::util::get;
			get<V>( n ) = 0.0f;
			get<I>( n ) = 0.0f;
			get<Twait>( n ) = 0;
		}

		template <typename Iter, typename Backend>
		WLIF_HD static bool update( Iter n, float const dt, ::spice::snn_info, Backend & )
		{
			using ::spice::util::get;
			float const inv_tau_mem = 1.0f / 0.02f;
			float const inv_tau_syn = 1.0f / 0.005f;
			float const v_thresh = 0.02f;
			int const t_ref = 20; // steps
			// bias 21-29 mV: every neuron fires on its own, at its own rate
			float const bias = 0.021f + 0.00008f * static_cast<float>( ( static_cast<int>( n.id() ) * 37 ) % 101 );

			bool fired = false;
			if( --get<Twait>( n ) <= 0 )
			{
				if( get<V>( n ) > v_thresh )
				{
					get<V>( n ) = 0.0f;
					get<Twait>( n ) = t_ref;
					fired = true;
				}
				else
					get<V>( n ) += ( bias - get<V>( n ) + get<I>( n ) ) * ( dt * inv_tau_mem );
			}
			get<I>( n ) -= get<I>( n ) * ( dt * inv_tau_syn );
			return fired;
		}

		template <typename Iter, typename SynIter, typename Backend>
		WLIF_HD static void receive( int, Iter dst, SynIter && syn, ::spice::snn_info, Backend & bak )
		{
			using ::spice::util::get;
			bak.atomic_add( get<I>( dst ), get<0>( syn ) );
		}
	};

	struct synapse : ::spice::synapse<float>
	{
		// excitatory sources (the first 80 %) 0.4-2 mV, inhibitory ones -2 to -10 mV, by a
		// hash of the pair
		template <typename Iter, typename Backend>
		WLIF_HD static void init( Iter syn, int src, int dst, ::spice::snn_info info, Backend & )
		{
			using ::spice::util::get;
			float const w = 0.0004f * static_cast<float>( 1 + ( src * 7 + dst * 13 ) % 5 );
			get<0>( syn ) = src < static_cast<int>( 0.8f * info.num_neurons ) ? w : -5.0f * w;
		}

		// static weights: never updated
		template <typename Iter, typename Backend>
		WLIF_HD static void update( Iter &&, int, bool, bool, float, ::spice::snn_info, Backend & )
		{
		}
		WLIF_HD static bool plastic( int, int, ::spice::snn_info ) { return false; }
	};
};
} // namespace test_models
