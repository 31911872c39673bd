// C++17 surface test (restates spice_test/cuda/snn.d.cpp:72-139 against the C++ wrapper):
// construction, conversion constructor, stepping, export. Exit code 0 = pass.
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
