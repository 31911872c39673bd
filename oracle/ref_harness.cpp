// TEST INFRASTRUCTURE ONLY -- a C-ABI wrapper around the reference's own cpu::snn, compiled
// from the reference sources (never copied) into oracle/_ref/libspice_ref*.so by
// oracle/Makefile. The RNG shim in oracle/shim/ replaces the Poisson stream with the
// counter-based one (see that header). Used by tests/golden/make_golden.py to produce the
// committed golden fixtures, by the oracle tests to pin the restatement, and by bench.py's
// reference arm as the CPU baseline (the reference's single-core simulator).
#include <spice/cpu/snn.h>
#include <spice/models/brunel.h>
#include <spice/models/brunel_with_plasticity.h>
#include <spice/models/synth.h>
#include <spice/models/vogels_abbott.h>
#include <spice/util/adj_list.h>
#include <spice/util/layout.h>

// A model of the tests compiled in as model 7 (the `user` target of oracle/Makefile): the
// reference's snn and cpu::snn definitions are included here, instead of linking snn.cpp and
// snn.h.cpp, so that both can be instantiated for it.
#if defined( SPK_USER_MODEL_HEADER ) && defined( SPK_USER_MODEL )
#include <spice/cpu/snn.h.cpp>
#include <spice/snn.cpp>
#include SPK_USER_MODEL_HEADER
template class spice::snn<SPK_USER_MODEL>;
template class spice::cpu::snn<SPK_USER_MODEL>;
#define SPK_HAS_USER_MODEL 1
#endif

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <stdexcept>
#include <tuple>
#include <type_traits>
#include <vector>

namespace
{
thread_local std::string g_err;
uint64_t g_generate_calls = 0; // adj_list::generate seeds its stream with 1337 + call index

spice::util::layout make_layout( int npops, uint64_t const * pops, int nconn, int const * csrc, int const * cdst, float const * cp )
{
	std::vector<size_t> p( pops, pops + npops );
	std::vector<std::tuple<size_t, size_t, float>> c;
	for( int i = 0; i < nconn; i++ ) c.emplace_back( (size_t)csrc[i], (size_t)cdst[i], cp[i] );
	return spice::util::layout( p, c );
}

struct net_base
{
	virtual ~net_base() = default;
	virtual int step( int * out, int cap ) = 0;
	virtual uint64_t num_neurons() const = 0;
	virtual uint64_t width() const = 0;
	virtual void adj( int * out ) const = 0;
	virtual void neurons( void ** attrs ) const = 0;
	virtual uint64_t num_synapse_attrs() const = 0;
	virtual void synapses( void ** attrs ) const = 0;
};

template <typename Tuple, size_t... I>
void scatter_tuple( std::vector<Tuple> const & v, void ** attrs, std::index_sequence<I...> )
{
	( [&] {
		using T = std::tuple_element_t<I, Tuple>;
		T * dst = static_cast<T *>( attrs[I] );
		for( size_t k = 0; k < v.size(); k++ ) dst[k] = std::get<I>( v[k] );
	}(),
	  ... );
}

// cpu::snn keeps its graph and state private and has no constructor from an adjacency
// (spice/cpu/snn.h:16-46). The explicit-instantiation rule (template arguments of an
// explicit instantiation are not access-checked) gives the harness pointers to those three
// members, so a reference net can start from a given graph and state: the GPU net's state
// at the same step, for parity checks at sizes where running the reference from step 0 to
// a steady state takes too long.
template <typename Tag, auto Member>
struct member_access
{
	friend auto member_pointer( Tag ) { return Member; }
};
template <typename Model>
struct graph_tag
{
	friend auto member_pointer( graph_tag );
};
template <typename Model>
struct neurons_tag
{
	friend auto member_pointer( neurons_tag );
};
template <typename Model>
struct synapses_tag
{
	friend auto member_pointer( synapses_tag );
};
template <typename Model>
struct spikes_tag
{
	friend auto member_pointer( spikes_tag );
};
template <typename Model>
struct istep_tag
{
	friend auto member_pointer( istep_tag );
};
template <typename Model>
struct simtime_tag
{
	friend auto member_pointer( simtime_tag );
};
#define SPICE_HARNESS_ACCESS( M )                                                                             \
	template struct member_access<graph_tag<M>, &spice::cpu::snn<M>::_graph>;                                \
	template struct member_access<neurons_tag<M>, &spice::cpu::snn<M>::_neurons>;                            \
	template struct member_access<synapses_tag<M>, &spice::cpu::snn<M>::_synapses>;                          \
	template struct member_access<spikes_tag<M>, &spice::cpu::snn<M>::_spikes>;                              \
	template struct member_access<istep_tag<M>, &spice::snn<M>::_i>;                                         \
	template struct member_access<simtime_tag<M>, &spice::snn<M>::_simtime>;
SPICE_HARNESS_ACCESS( spice::vogels_abbott )
SPICE_HARNESS_ACCESS( spice::brunel )
SPICE_HARNESS_ACCESS( spice::brunel_with_plasticity )
SPICE_HARNESS_ACCESS( spice::synth )
#if defined( SPK_HAS_USER_MODEL )
SPICE_HARNESS_ACCESS( SPK_USER_MODEL )
#endif
#undef SPICE_HARNESS_ACCESS

template <typename Tuple, size_t... I>
void gather_tuple( std::vector<Tuple> & v, void * const * attrs, std::index_sequence<I...> )
{
	( [&] {
		using T = std::tuple_element_t<I, Tuple>;
		T const * src = static_cast<T const *>( attrs[I] );
		for( size_t k = 0; k < v.size(); k++ ) std::get<I>( v[k] ) = src[k];
	}(),
	  ... );
}

template <typename Model>
struct net : net_base
{
	spice::cpu::snn<Model> impl;
	std::vector<int> buf;

	net( spice::util::layout const & l, float dt, int delay )
	    : impl( l, dt, delay )
	{
	}

	// a net of n neurons without synapses, then the given graph (n x width ELL) and state
	// (one array per attribute, in the model's attribute order) put in its place; with
	// step0 > 0 the net stands at step step0: its simulated clock advanced by step0 steps
	// and the spikes of the steps [step0 - nq, step0) in flight (counts[nq], ids)
	net( uint64_t n,
	     uint64_t width,
	     int const * edges,
	     void * const * neuron_attrs,
	     void * const * synapse_attrs,
	     float dt,
	     int delay,
	     uint64_t step0,
	     int nq,
	     uint32_t const * counts,
	     int const * ids )
	    : impl( spice::util::layout( n, 0.0f ), dt, delay )
	{
		auto & base = static_cast<spice::snn<Model> &>( impl );
		base.*member_pointer( istep_tag<Model>{} ) = static_cast<int>( step0 );
		auto & clock = base.*member_pointer( simtime_tag<Model>{} );
		for( uint64_t k = 0; k < step0; k++ ) clock.add( dt );
		auto & spikes = impl.*member_pointer( spikes_tag<Model>{} );
		size_t o = 0;
		for( int q = 0; q < nq; q++ )
		{
			spikes.counts.push_back( counts[q] );
			spikes.ids.insert( spikes.ids.end(), ids + o, ids + o + counts[q] );
			// Brunel+ keeps each step's firing flags in slot step % (delay + 1)
			if( spikes.flags )
				for( uint32_t k = 0; k < counts[q]; k++ )
					( *spikes.flags )[( step0 - nq + q ) % ( delay + 1 )][ids[o + k]] = true;
			o += counts[q];
		}
		auto & graph = impl.*member_pointer( graph_tag<Model>{} );
		graph.edges.assign( edges, edges + n * width );
		graph.adj = spice::util::adj_list( n, width, graph.edges.data() );
		if constexpr( Model::neuron::size > 0 )
		{
			auto & nv = *( impl.*member_pointer( neurons_tag<Model>{} ) );
			using T = typename Model::neuron::tuple_t;
			gather_tuple( nv, neuron_attrs, std::make_index_sequence<std::tuple_size_v<T>>() );
		}
		if constexpr( Model::synapse::size > 0 )
		{
			auto & sv = impl.*member_pointer( synapses_tag<Model>{} );
			sv.emplace( n * width );
			using T = typename Model::synapse::tuple_t;
			gather_tuple( *sv, synapse_attrs, std::make_index_sequence<std::tuple_size_v<T>>() );
		}
	}

	int step( int * out, int cap ) override
	{
		impl.step( &buf );
		int const n = static_cast<int>( buf.size() );
		if( out )
			for( int i = 0; i < n && i < cap; i++ ) out[i] = buf[i];
		return n;
	}
	uint64_t num_neurons() const override { return impl.num_neurons(); }
	uint64_t width() const override { return impl.adj().second; }
	void adj( int * out ) const override
	{
		auto a = impl.adj();
		std::memcpy( out, a.first.data(), a.first.size() * sizeof( int ) );
	}
	void neurons( void ** attrs ) const override
	{
		using T = typename Model::neuron::tuple_t;
		scatter_tuple( impl.neurons(), attrs, std::make_index_sequence<std::tuple_size_v<T>>() );
	}
	uint64_t num_synapse_attrs() const override { return Model::synapse::size; }
	void synapses( void ** attrs ) const override
	{
		using T = typename Model::synapse::tuple_t;
		scatter_tuple( impl.synapses(), attrs, std::make_index_sequence<std::tuple_size_v<T>>() );
	}
};
} // namespace

extern "C" {
char const * ref_last_error() { return g_err.c_str(); }

// Flattened layout as the reference computes it (spice/util/layout.cpp:51-110):
// writes up to `cap` tuples (src_first, src_last, dst_first, dst_last) + p, returns the
// tuple count; *max_degree receives layout::max_degree() (spice/util/layout.cpp:13-38).
int ref_layout(
    int npops,
    uint64_t const * pops,
    int nconn,
    int const * csrc,
    int const * cdst,
    float const * cp,
    int * out_ranges,
    float * out_p,
    int cap,
    uint64_t * max_degree,
    uint64_t * size )
{
	try
	{
		auto l = make_layout( npops, pops, nconn, csrc, cdst, cp );
		int i = 0;
		for( auto const & c : l.connections() )
		{
			if( i < cap )
			{
				out_ranges[4 * i + 0] = std::get<0>( c );
				out_ranges[4 * i + 1] = std::get<1>( c );
				out_ranges[4 * i + 2] = std::get<2>( c );
				out_ranges[4 * i + 3] = std::get<3>( c );
				out_p[i] = std::get<4>( c );
			}
			i++;
		}
		*max_degree = l.max_degree();
		*size = l.size();
		return i;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return -1;
	}
}

// The reference's CPU graph generator (spice/util/adj_list.cpp:49-91). Returns the seed it
// used (1337 + number of earlier generate calls in this process), 0 on error.
uint64_t ref_generate( int npops, uint64_t const * pops, int nconn, int const * csrc, int const * cdst, float const * cp, int * out )
{
	try
	{
		auto l = make_layout( npops, pops, nconn, csrc, cdst, cp );
		std::vector<int> e;
		uint64_t const seed = 1337 + g_generate_calls++;
		spice::util::adj_list::generate( l, e );
		std::memcpy( out, e.data(), e.size() * sizeof( int ) );
		return seed;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return 0;
	}
}

// model: 0 vogels_abbott, 1 brunel, 2 brunel_with_plasticity, 3 synth
void * ref_create(
    int model,
    int npops,
    uint64_t const * pops,
    int nconn,
    int const * csrc,
    int const * cdst,
    float const * cp,
    float dt,
    int delay,
    uint64_t rng_seed )
{
	try
	{
		auto l = make_layout( npops, pops, nconn, csrc, cdst, cp );
		oracle::counter_rng::seed = rng_seed;
		oracle::counter_rng::calls = 0;
		uint64_t const n = l.size();
		oracle::counter_rng::npoisson = ( model == 3 ) ? n : ( n / 2 > 0 ? n / 2 : 1 );
		g_generate_calls++;
		switch( model )
		{
		case 0: return new net<spice::vogels_abbott>( l, dt, delay );
		case 1: return new net<spice::brunel>( l, dt, delay );
		case 2: return new net<spice::brunel_with_plasticity>( l, dt, delay );
		case 3: return new net<spice::synth>( l, dt, delay );
		default: g_err = "invalid model"; return nullptr;
		}
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return nullptr;
	}
}

// A reference net over an imported graph and state (see net's second constructor): the
// graph n x width (rows ascending, INT_MAX padded, as adj() returns it), neuron_attrs one
// array per neuron attribute and, for brunel_with_plasticity, synapse_attrs (W, Zpre,
// Zpost) over all n x width slots. The Poisson stream restarts at step 0 with rng_seed.
// With step0 > 0 the net continues a run at step step0 (clock, Poisson stream and the nq
// steps of spikes in flight, counts[nq] and ids concatenated, oldest first); nq <= delay.
void * ref_create_from_state(
    int model,
    uint64_t n,
    uint64_t width,
    int const * edges,
    void * const * neuron_attrs,
    void * const * synapse_attrs,
    float dt,
    int delay,
    uint64_t rng_seed,
    uint64_t step0,
    int nq,
    uint32_t const * counts,
    int const * ids )
{
	try
	{
		if( nq < 0 || nq > delay || (uint64_t)nq > step0 ) throw std::invalid_argument( "spikes in flight: at most delay steps, none before step 0" );
		oracle::counter_rng::seed = rng_seed;
		oracle::counter_rng::npoisson = ( model == 3 ) ? n : ( n / 2 > 0 ? n / 2 : 1 );
		oracle::counter_rng::calls = step0 * oracle::counter_rng::npoisson;
		g_generate_calls++;
		auto const a = std::make_tuple( n, width, edges, neuron_attrs, synapse_attrs, dt, delay, step0, nq, counts, ids );
		auto make = [&]( auto tag ) -> net_base * {
			using M = typename decltype( tag )::type;
			return std::apply( []( auto... x ) { return new net<M>( x... ); }, a );
		};
		switch( model )
		{
		case 0: return make( std::common_type<spice::vogels_abbott>{} );
		case 1: return make( std::common_type<spice::brunel>{} );
		case 2: return make( std::common_type<spice::brunel_with_plasticity>{} );
		case 3: return make( std::common_type<spice::synth>{} );
#if defined( SPK_HAS_USER_MODEL )
		case 7: return make( std::common_type<SPK_USER_MODEL>{} );
#endif
		default: g_err = "invalid model"; return nullptr;
		}
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return nullptr;
	}
}

void ref_destroy( void * h ) { delete static_cast<net_base *>( h ); }
int ref_step( void * h, int * out, int cap ) { return static_cast<net_base *>( h )->step( out, cap ); }
uint64_t ref_num_neurons( void * h ) { return static_cast<net_base *>( h )->num_neurons(); }
uint64_t ref_width( void * h ) { return static_cast<net_base *>( h )->width(); }
void ref_adj( void * h, int * out ) { static_cast<net_base *>( h )->adj( out ); }
void ref_neurons( void * h, void ** attrs ) { static_cast<net_base *>( h )->neurons( attrs ); }
void ref_synapses( void * h, void ** attrs ) { static_cast<net_base *>( h )->synapses( attrs ); }
uint64_t ref_num_synapse_attrs( void * h ) { return static_cast<net_base *>( h )->num_synapse_attrs(); }
}
