// spice::cuda::snn<Model> -- the single-GPU net of the reference (spice/cuda/snn.h:16-77),
// as a header-only C++17 wrapper over the C ABI of libspice_b200.so (include/spice_b200.h).
// Link with -lspice_b200. Errors are thrown as the reference throws them:
// std::invalid_argument for bad arguments, std::bad_alloc for device allocation failures,
// std::runtime_error for everything else.
#pragma once

#include <spice/models/brunel.h>
#include <spice/models/brunel_fixed.h>
#include <spice/models/brunel_with_plasticity.h>
#include <spice/models/brunel_with_plasticity_a012.h>
#include <spice/models/synth.h>
#include <spice/models/vogels_abbott.h>
#include <spice/models/vogels_abbott_ns.h>
#include <spice/snn.h>
#include <spice/util/layout.h>
#include <spice_b200.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace spice
{
namespace cuda
{
template <typename Model>
struct model_id;
template <>
struct model_id<vogels_abbott> : std::integral_constant<int, SPK_VOGELS_ABBOTT>
{
};
template <>
struct model_id<brunel> : std::integral_constant<int, SPK_BRUNEL>
{
};
template <>
struct model_id<brunel_with_plasticity> : std::integral_constant<int, SPK_BRUNEL_PLUS>
{
};
template <>
struct model_id<synth> : std::integral_constant<int, SPK_SYNTH>
{
};
template <>
struct model_id<vogels_abbott_ns> : std::integral_constant<int, SPK_VOGELS_ABBOTT_NS>
{
};
template <>
struct model_id<brunel_fixed> : std::integral_constant<int, SPK_BRUNEL_FIXED>
{
};
template <>
struct model_id<brunel_with_plasticity_a012> : std::integral_constant<int, SPK_BRUNEL_PLUS_A012>
{
};

inline void check( int status )
{
	if( status == SPK_OK ) return;
	std::string const msg = spk_last_error();
	if( status == SPK_ERR_INVALID ) throw std::invalid_argument( msg );
	if( status == SPK_ERR_NOMEM ) throw std::bad_alloc();
	throw std::runtime_error( msg );
}

template <typename Model>
class snn : public ::spice::snn<Model>
{
public:
	using neuron_tuple = typename Model::neuron::tuple_t;
	using synapse_tuple = typename Model::synapse::export_tuple_t;

	// snn(layout, dt, delay) (spice/cuda/snn.h:20-25); seed keys the Poisson draws,
	// graph_seed the counter-based graph generator
	snn( util::layout const & desc, float dt, int delay = 1, std::uint64_t seed = 1, std::uint64_t graph_seed = 1337, int device = 0 )
	{
		std::vector<std::uint64_t> pops;
		std::vector<int> src, dst;
		std::vector<float> p;
		flatten_to_pops( desc, pops, src, dst, p );
		spk_layout_desc d{ (int)pops.size(), pops.data(), (int)src.size(), src.data(), dst.data(), p.data() };
		check( spk_net_create( &_net, model_id<Model>::value, &d, dt, delay, seed, graph_seed, device ) );
	}

	// snn(adj, width, dt, delay) (spice/cuda/snn.h:26-32)
	snn( std::vector<int> const & adj, std::size_t width, float dt, int delay = 1, std::uint64_t seed = 1, int device = 0 )
	{
		if( width == 0 || adj.size() % width ) throw std::invalid_argument( "adjacency size is not a multiple of width" );
		check( spk_net_create_from_adj( &_net, model_id<Model>::value, adj.data(), adj.size() / width, width, dt, delay, seed, device ) );
	}

	// snn(const spice::snn<Model>&) (spice/cuda/snn.h:33): same graph and state
	explicit snn( ::spice::snn<Model> const & other, std::uint64_t seed = 1, int device = 0 )
	    : snn( other.adj().first, other.adj().second, other.dt(), other.delay(), seed, device )
	{
		set_neurons( other.neurons() );
		if constexpr( std::tuple_size_v<synapse_tuple> > 0 ) set_synapses( other.synapses() );
	}

	// a copy is a new net with the same graph and state (the conversion constructor)
	snn( snn const & other )
	    : snn( static_cast<::spice::snn<Model> const &>( other ) )
	{
	}
	snn & operator=( snn const & ) = delete;
	~snn() override
	{
		if( _net ) spk_net_destroy( _net );
	}

	void step( std::vector<int> * out = nullptr ) override
	{
		if( !out )
		{
			check( spk_net_step( _net, nullptr, 0, nullptr ) );
			return;
		}
		out->resize( num_neurons() );
		std::uint64_t count = 0;
		check( spk_net_step( _net, out->data(), out->size(), &count ) );
		out->resize( count );
	}

	// nsteps x step(nullptr): one cooperative launch, or CUDA-graph windows
	void run( std::uint64_t nsteps ) { check( spk_net_run( _net, nsteps ) ); }

	std::size_t num_neurons() const override { return info().num_neurons; }
	std::size_t num_synapses() const override { return info().num_synapses; }
	float dt() const override { return info().dt; }
	int delay() const override { return info().delay; }

	std::pair<std::vector<int>, std::size_t> adj() const override
	{
		auto const i = info();
		std::vector<int> e( i.num_synapses );
		check( spk_net_adj( _net, e.data(), e.size() ) );
		return { std::move( e ), i.width };
	}

	std::vector<neuron_tuple> neurons() const override { return gather<neuron_tuple>( num_neurons(), &spk_net_neurons ); }
	std::vector<synapse_tuple> synapses() const override
	{
		if constexpr( std::tuple_size_v<synapse_tuple> == 0 )
			return {};
		else
			return gather<synapse_tuple>( num_synapses(), &spk_net_synapses );
	}

	void set_neurons( std::vector<neuron_tuple> const & v ) { scatter( v, &spk_net_set_neurons ); }
	void set_synapses( std::vector<synapse_tuple> const & v ) { scatter( v, &spk_net_set_synapses ); }

	spk_net_info info() const
	{
		spk_net_info i{};
		check( spk_net_get_info( _net, &i ) );
		return i;
	}
	spk_net * handle() const { return _net; }

	// everything the net needs to continue bit for bit (edges, state, spikes in flight,
	// clock, lazy-STDP state); restore() makes a net continuing from it
	std::vector<unsigned char> checkpoint() const
	{
		std::uint64_t size = 0;
		check( spk_net_checkpoint( _net, nullptr, 0, &size ) );
		std::vector<unsigned char> buf( size );
		check( spk_net_checkpoint( _net, buf.data(), buf.size(), &size ) );
		return buf;
	}
	static snn restore( std::vector<unsigned char> const & buf, int device = 0 )
	{
		spk_net * h = nullptr;
		check( spk_net_restore( &h, buf.data(), buf.size(), device ) );
		spk_net_info i{};
		int const st = spk_net_get_info( h, &i );
		if( st != SPK_OK || i.model != model_id<Model>::value )
		{
			spk_net_destroy( h );
			throw std::invalid_argument( "the checkpoint holds another model" );
		}
		return snn( h );
	}
	snn( snn && other ) noexcept
	    : _net( std::exchange( other._net, nullptr ) )
	{
	}

private:
	explicit snn( spk_net * h )
	    : _net( h )
	{
	}
	spk_net * _net = nullptr;

	static void flatten_to_pops( util::layout const & l, std::vector<std::uint64_t> & pops, std::vector<int> & src, std::vector<int> & dst, std::vector<float> & p )
	{
		for( auto x : l.populations() ) pops.push_back( x );
		for( auto const & c : l.population_connections() )
		{
			src.push_back( (int)std::get<0>( c ) );
			dst.push_back( (int)std::get<1>( c ) );
			p.push_back( std::get<2>( c ) );
		}
	}

	template <typename Tuple, typename F>
	std::vector<Tuple> gather( std::size_t n, F f ) const
	{
		constexpr std::size_t k = std::tuple_size_v<Tuple>;
		std::vector<std::vector<std::uint32_t>> cols( k, std::vector<std::uint32_t>( n ) );
		void * ptrs[k > 0 ? k : 1];
		for( std::size_t i = 0; i < k; i++ ) ptrs[i] = cols[i].data();
		check( f( _net, ptrs ) );
		std::vector<Tuple> out( n );
		fill<Tuple>( out, cols, std::make_index_sequence<k>() );
		return out;
	}

	template <typename Tuple, std::size_t... I>
	static void fill( std::vector<Tuple> & out, std::vector<std::vector<std::uint32_t>> const & cols, std::index_sequence<I...> )
	{
		for( std::size_t r = 0; r < out.size(); r++ )
			( ( std::memcpy( &std::get<I>( out[r] ), &cols[I][r], 4 ) ), ... );
	}

	template <typename Tuple, typename F>
	void scatter( std::vector<Tuple> const & v, F f )
	{
		constexpr std::size_t k = std::tuple_size_v<Tuple>;
		std::vector<std::vector<std::uint32_t>> cols( k, std::vector<std::uint32_t>( v.size() ) );
		put<Tuple>( v, cols, std::make_index_sequence<k>() );
		void * ptrs[k > 0 ? k : 1];
		for( std::size_t i = 0; i < k; i++ ) ptrs[i] = cols[i].data();
		check( f( _net, ptrs ) );
	}

	template <typename Tuple, std::size_t... I>
	static void put( std::vector<Tuple> const & v, std::vector<std::vector<std::uint32_t>> & cols, std::index_sequence<I...> )
	{
		for( std::size_t r = 0; r < v.size(); r++ )
			( ( std::memcpy( &cols[I][r], &std::get<I>( v[r] ), 4 ) ), ... );
	}
};
} // namespace cuda
} // namespace spice
