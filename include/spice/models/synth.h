// Synthetic benchmark model: one population, every neuron fires with probability 0.005
// per step and counts its arrivals (spice/models/synth.h:12-43).
#pragma once

#include <spice/models/model.h>

namespace spice
{
struct synth : model
{
	struct neuron : ::spice::neuron<int>
	{
		enum attr
		{
			N
		};

		template <typename Iter, typename Backend>
		SPICE_HD static void init( Iter n, snn_info, Backend & )
		{
			using util::get;
			get<N>( n ) = 0;
		}

		template <typename Iter, typename Backend>
		SPICE_HD static bool update( Iter, float const, snn_info, Backend & bak )
		{
			return bak.rand() < 0.005f;
		}

		template <typename Iter, typename SynIter, typename Backend>
		SPICE_HD static void receive( int, Iter dst, SynIter &&, snn_info, Backend & bak )
		{
			using util::get;
			bak.atomic_add( get<N>( dst ), 1 );
		}

		static constexpr int input_classes = 1;
		SPICE_HD static int input_class( int, snn_info ) { return 0; }
		SPICE_HD static int class_source( int, snn_info ) { return 0; }
	};
};
} // namespace spice
