// spice::snn<Model> -- the abstract net interface of the reference (spice/snn.h:16-45):
// step(std::vector<int>* out), num_neurons(), num_synapses(), dt(), delay(), info(),
// adj(), neurons(), synapses(). Host-only, header-only.
#pragma once

#include <spice/snn_info.h>

#include <cstddef>
#include <utility>
#include <vector>

namespace spice
{
template <typename Model>
class snn
{
public:
	virtual ~snn() = default;

	virtual void step( std::vector<int> * out_spikes = nullptr ) = 0;

	virtual std::size_t num_neurons() const = 0;
	virtual std::size_t num_synapses() const = 0;
	virtual float dt() const = 0;
	virtual int delay() const = 0;
	snn_info info() const { return { static_cast<int>( num_neurons() ) }; }

	// (edges, width)
	virtual std::pair<std::vector<int>, std::size_t> adj() const = 0;
	virtual std::vector<typename Model::neuron::tuple_t> neurons() const = 0;
	virtual std::vector<typename Model::synapse::export_tuple_t> synapses() const = 0;
};
} // namespace spice
