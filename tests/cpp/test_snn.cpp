// C++17 surface test (restates spice_test/cuda/snn.d.cpp:72-139 against the C++ wrapper):
// construction, conversion constructor, stepping, export. Exit code 0 = pass.
#include <spice/cuda/batch.h>
#include <spice/cuda/snn.h>

#include <cstdio>
#include <cstdlib>

#define EXPECT( x )                                                         \
	do                                                                      \
	{                                                                       \
		if( !( x ) )                                                        \
		{                                                                   \
			std::fprintf( stderr, "%s:%d: %s failed\n", __FILE__, __LINE__, #x ); \
			std::exit( 1 );                                                 \
		}                                                                   \
	} while( 0 )

using namespace spice;

int main()
{
	{ // ctor (spice_test/cuda/snn.d.cpp:75-88)
		cuda::snn<brunel> d( util::layout( 100, 0.1f ), 0.0001f, 15 );
		EXPECT( d.num_neurons() == 100u );
		EXPECT( d.dt() == 0.0001f );
		EXPECT( d.delay() == 15 );
		EXPECT( d.adj().second == d.num_synapses() / 100 );
	}
	{ // conversion ctor: same graph, same state, same spikes
		cuda::snn<vogels_abbott> a( util::layout( 2000, 0.02f ), 0.0001f, 1 );
		cuda::snn<vogels_abbott> b( a );
		EXPECT( a.adj() == b.adj() );
		std::vector<int> sa, sb;
		for( int i = 0; i < 500; i++ )
		{
			a.step( &sa );
			b.step( &sb );
			EXPECT( sa == sb );
		}
		auto na = a.neurons(), nb = b.neurons();
		EXPECT( na == nb );
	}
	{ // plastic model exports the reference's synapse tuple
		cuda::snn<brunel_with_plasticity> d( util::layout( { 200, 200 }, { { 0, 1, 0.1f }, { 1, 1, 0.1f } } ), 0.0001f, 15 );
		d.run( 300 );
		auto s = d.synapses();
		EXPECT( s.size() == d.num_synapses() );
		std::vector<int> out;
		d.step( &out );
	}
	{ // checkpoint / restore: the restored net continues bit for bit
		cuda::snn<brunel> a( util::layout( { 2000, 2000 }, { { 0, 1, 0.1f }, { 1, 1, 0.1f } } ), 0.0001f, 15 );
		a.run( 123 );
		auto b = cuda::snn<brunel>::restore( a.checkpoint() );
		std::vector<int> sa, sb;
		for( int i = 0; i < 100; i++ )
		{
			a.step( &sa );
			b.step( &sb );
			EXPECT( sa == sb );
		}
		EXPECT( a.neurons() == b.neurons() );
		bool thrown = false;
		try
		{
			cuda::snn<vogels_abbott>::restore( a.checkpoint() );
		}
		catch( std::invalid_argument const & )
		{
			thrown = true;
		}
		EXPECT( thrown );
	}
	{ // a batch steps its nets as they step alone; a server job ends with the same state
		util::layout const l( { 1500, 1500 }, { { 0, 1, 0.1f }, { 1, 1, 0.1f } } );
		cuda::snn<brunel> alone( l, 0.0001f, 15, 5 ), in_batch( l, 0.0001f, 15, 5 );
		cuda::batch b;
		b.add( in_batch );
		b.run( 200 );
		alone.run( 200 );
		EXPECT( alone.neurons() == in_batch.neurons() );
		cuda::server srv( 1ull << 32, 100 );
		auto const job = srv.submit<brunel>( l, 250, 0.0001f, 15, 5 );
		srv.wait( job, 60.0 );
		EXPECT( srv.info( job ).state == SPK_JOB_DONE && srv.info( job ).steps_done == 250 );
		EXPECT( srv.stats().done == 1 );
	}
	{ // errors come back as the reference's exception types
		bool thrown = false;
		try
		{
			cuda::snn<brunel> d( util::layout( 10, 0.1f ), 0.0f );
		}
		catch( std::invalid_argument const & )
		{
			thrown = true;
		}
		EXPECT( thrown );
	}
	std::puts( "cpp ok" );
	return 0;
}
