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

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <tuple>
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

template <typename Model>
struct net : net_base
{
	spice::cpu::snn<Model> impl;
	std::vector<int> buf;

	net( spice::util::layout const & l, float dt, int delay )
	    : impl( l, dt, delay )
	{
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

void ref_destroy( void * h ) { delete static_cast<net_base *>( h ); }
int ref_step( void * h, int * out, int cap ) { return static_cast<net_base *>( h )->step( out, cap ); }
uint64_t ref_num_neurons( void * h ) { return static_cast<net_base *>( h )->num_neurons(); }
uint64_t ref_width( void * h ) { return static_cast<net_base *>( h )->width(); }
void ref_adj( void * h, int * out ) { static_cast<net_base *>( h )->adj( out ); }
void ref_neurons( void * h, void ** attrs ) { static_cast<net_base *>( h )->neurons( attrs ); }
void ref_synapses( void * h, void ** attrs ) { static_cast<net_base *>( h )->synapses( attrs ); }
uint64_t ref_num_synapse_attrs( void * h ) { return static_cast<net_base *>( h )->num_synapse_attrs(); }
}
