// TEST INFRASTRUCTURE ONLY -- the CPU oracle (the checker). Only tests/, the smoke check and
// bench.py's CPU-baseline leg load this library; the product never does.
//
// An independent single-core restatement of the reference's CPU simulator cpu::snn
// (spice/cpu/snn.h.cpp:73-181) and of the pieces it uses:
//   * layout flattening and ELL width      spice/util/layout.cpp:13-38, 51-110
//   * the reference graph generator        spice/util/adj_list.cpp:49-91 with
//     xoroshiro256ss / exprnd / binornd      spice/util/random.h:18-27, 76-113, 117-156
//   * the Kahan-compensated time step      spice/snn.cpp:38-44, spice/util/numeric.h:9-33
//   * the three models                     spice/models/vogels_abbott.h, brunel.h,
//                                          brunel_with_plasticity.h, synth.h
// plus the counter-based pieces the B200 path introduces (same definitions, written
// independently of the GPU code):
//   * Poisson draws rand(step, neuron) = uniform_left_inc(Philox(seed; neuron, step, 0, 'NEUR'))
//   * the Bernoulli ELL generator (philox_generate below)
//
// Everything is templated on the state precision R: R = float reproduces the reference's
// FP32 arithmetic operation by operation (build with -ffp-contract=off); R = double is the
// FP64 oracle run (same inputs, same dt sequence, double state arithmetic).
#include "philox.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <vector>

namespace oracle
{
// threads of the Brunel+ synapse sweep on large nets (ORACLE_THREADS, else the host's)
static int sweep_threads()
{
	char const * e = std::getenv( "ORACLE_THREADS" );
	int const t = e ? std::atoi( e ) : (int)std::thread::hardware_concurrency();
	return std::max( 1, std::min( t, 64 ) );
}

// ---------------------------------------------------------------------------------------
// layout  (spice/util/layout.cpp:51-110, estimate_max_deg :13-38)
// ---------------------------------------------------------------------------------------
struct conn
{
	int src_first, src_last, dst_first, dst_last;
	float p;
};

struct layout
{
	uint64_t n = 0;
	std::vector<conn> conns;
	uint64_t max_degree = 0;
};

static uint64_t estimate_max_degree( std::vector<conn> const & cs )
{
	int src = cs.empty() ? 0 : cs.front().src_first;
	uint64_t result = 0;
	double m = 0.0, s2 = 0.0;
	for( auto const & c : cs )
	{
		if( c.src_first != src )
		{
			result = std::max( result, static_cast<uint64_t>( m + 3 * std::sqrt( s2 ) ) );
			src = c.src_first;
			m = 0.0;
			s2 = 0.0;
		}
		double const range = static_cast<double>( c.dst_last - c.dst_first );
		m += range * c.p;
		s2 += range * c.p * ( 1.0 - c.p );
	}
	return ( std::max( result, static_cast<uint64_t>( m + 3 * std::sqrt( s2 ) ) ) + 31 ) / 32 * 32;
}

static layout make_layout( std::vector<uint64_t> const & pops, std::vector<std::tuple<int, int, float>> cs )
{
	if( pops.empty() ) throw std::invalid_argument( "layout must contain at least 1 population" );
	for( auto p : pops )
		if( p == 0 || p > INT_MAX ) throw std::invalid_argument( "invalid population size" );
	for( auto const & c : cs )
	{
		if( std::get<0>( c ) < 0 || std::get<1>( c ) < 0 || (size_t)std::get<0>( c ) >= pops.size() ||
		    (size_t)std::get<1>( c ) >= pops.size() )
			throw std::invalid_argument( "invalid index in connections matrix" );
		if( !( std::get<2>( c ) >= 0.0f && std::get<2>( c ) <= 1.0f ) )
			throw std::invalid_argument( "invalid connect. prob." );
	}
	std::sort( cs.begin(), cs.end(), []( auto const & a, auto const & b ) {
		return std::get<0>( a ) < std::get<0>( b ) || ( std::get<0>( a ) == std::get<0>( b ) && std::get<1>( a ) < std::get<1>( b ) );
	} );
	for( size_t i = 1; i < cs.size(); i++ )
		if( std::get<0>( cs[i] ) == std::get<0>( cs[i - 1] ) && std::get<1>( cs[i] ) == std::get<1>( cs[i - 1] ) )
			throw std::invalid_argument( "no duplicate edges in connections list allowed" );

	std::vector<uint64_t> first( pops.size() + 1, 0 );
	for( size_t i = 0; i < pops.size(); i++ ) first[i + 1] = first[i] + pops[i];
	layout l;
	l.n = first.back();
	for( auto const & c : cs )
	{
		int const s = std::get<0>( c ), d = std::get<1>( c );
		l.conns.push_back( { (int)first[s], (int)first[s + 1], (int)first[d], (int)first[d + 1], std::get<2>( c ) } );
	}
	l.max_degree = estimate_max_degree( l.conns );
	return l;
}

// ---------------------------------------------------------------------------------------
// reference RNGs  (spice/util/random.h)
// ---------------------------------------------------------------------------------------
static inline uint64_t rotl64( uint64_t x, uint64_t k ) { return ( x << k ) | ( x >> ( 64 - k ) ); }
static inline uint64_t splitmix_hash( uint64_t x ) // random.h:18-27
{
	x = ( x ^ ( x >> 30 ) ) * 0xbf58476d1ce4e5b9llu;
	x = ( x ^ ( x >> 27 ) ) * 0x94d049bb133111ebllu;
	return x ^ ( x >> 31 );
}

struct xoshiro256ss // random.h:76-113
{
	uint64_t s0, s1, s2, s3;
	explicit xoshiro256ss( uint64_t seed )
	{
		s0 = splitmix_hash( seed );
		s1 = splitmix_hash( s0 );
		s2 = splitmix_hash( s1 );
		s3 = splitmix_hash( s2 );
	}
	uint64_t operator()()
	{
		uint64_t const r = rotl64( s1 * 5, 7 ) * 9;
		uint64_t const t = s1 << 17;
		s2 ^= s0;
		s3 ^= s1;
		s1 ^= s2;
		s0 ^= s3;
		s2 ^= t;
		s3 = rotl64( s3, 45 );
		return r;
	}
};

template <typename G>
static float u_left( G & g ) // random.h:117-121
{
	return ( (uint32_t)g() >> 8 ) / 16777216.0f;
}
template <typename G>
static float u_right( G & g ) // random.h:123-128
{
	return ( ( (uint32_t)g() >> 8 ) + 1.0f ) / 16777216.0f;
}
template <typename G>
static float exp_rnd( G & g ) // random.h:130-134
{
	return -logf( u_right( g ) );
}
template <typename G>
static float norm_rnd( G & g, float m, float s ) // random.h:138-145 (host sinpif at :28)
{
	// The radius draw happens before the angle draw (left operand first).
	float const r = sqrtf( -2 * logf( u_right( g ) ) );
	float const a = std::sin( 3.14159265359f * ( 2 * u_left( g ) ) );
	return fmaf( r * a, s, m );
}
template <typename G>
static int bino_rnd( G & g, int n, float p ) // random.h:147-156
{
	return std::min( n, std::max( 0, (int)lrintf( norm_rnd( g, n * p, sqrtf( n * p * ( 1 - p ) ) ) ) ) );
}

// spice/util/adj_list.cpp:49-91
static void reference_generate( layout const & l, uint64_t seed, std::vector<int> & edges )
{
	edges.assign( l.n * l.max_degree, 0 );
	xoshiro256ss gen( seed );
	int const n = (int)l.n;
	size_t offset = 0;
	for( int i = 0; i < n; i++ )
	{
		int total_degree = 0;
		for( auto const & c : l.conns )
		{
			if( i < c.src_first || i >= c.src_last ) continue;
			int const first = c.dst_first;
			int const range = c.dst_last - first;
			int const degree = std::min( (int)( l.max_degree - total_degree ), bino_rnd( gen, range, c.p ) );
			total_degree += degree;
			std::vector<float> pos( degree );
			float total = exp_rnd( gen );
			for( int k = 0; k < degree; k++ )
			{
				pos[k] = total;
				total += exp_rnd( gen );
			}
			float const scale = ( range - degree ) / total;
			for( int k = 0; k < degree; k++ ) edges[offset++] = first + (int)( pos[k] * scale ) + k;
		}
		while( offset < ( i + 1 ) * l.max_degree ) edges[offset++] = INT_MAX;
	}
}

// ---------------------------------------------------------------------------------------
// the counter-based Bernoulli ELL generator of the B200 path
//   row `src`, connection index c (position in the flattened, sorted layout), candidate
//   j in [0, range): u = Philox(seed; src, j / 4, c, 'GRAP').v[j % 4]; the edge src->first+j
//   exists iff u < floor(p * 2^32). Rows are ascending by construction, truncated at the
//   layout width, padded with INT_MAX.
// ---------------------------------------------------------------------------------------
static uint64_t bernoulli_threshold( float p )
{
	double const t = std::floor( (double)p * 4294967296.0 );
	return t >= 4294967296.0 ? 4294967296ull : (uint64_t)t;
}

static void philox_row( layout const & l, uint64_t seed, int src, int * row )
{
	uint64_t const w = l.max_degree;
	uint64_t k = 0;
	for( size_t ci = 0; ci < l.conns.size(); ci++ )
	{
		auto const & c = l.conns[ci];
		if( src < c.src_first || src >= c.src_last ) continue;
		uint64_t const thr = bernoulli_threshold( c.p );
		int const range = c.dst_last - c.dst_first;
		for( int j = 0; j < range && k < w; j += 4 )
		{
			philox_out const r = philox4x32_10(
			    (uint32_t)src, (uint32_t)( j / 4 ), (uint32_t)ci, TAG_GRAPH, (uint32_t)seed, (uint32_t)( seed >> 32 ) );
			for( int q = 0; q < 4 && j + q < range && k < w; q++ )
				if( (uint64_t)r.v[q] < thr ) row[k++] = c.dst_first + j + q;
		}
	}
	for( ; k < w; k++ ) row[k] = INT_MAX;
}

static void philox_generate( layout const & l, uint64_t seed, std::vector<int> & edges )
{
	edges.assign( l.n * l.max_degree, INT_MAX );
	for( uint64_t i = 0; i < l.n; i++ ) philox_row( l, seed, (int)i, edges.data() + i * l.max_degree );
}

// ---------------------------------------------------------------------------------------
// Kahan-compensated clock (spice/snn.cpp:38-44 + spice/util/numeric.h:9-33): the dt each
// step hands to the models is the compensated delta, always computed in float.
// ---------------------------------------------------------------------------------------
struct kahan
{
	float c = 0, sum = 0;
	float add( float d )
	{
		volatile float y = d - c;
		volatile float t = sum + y;
		c = ( t - sum ) - y;
		sum = t;
		return y;
	}
};

// constants: R(double literal) gives the float literal for R=float, a true double otherwise.
template <typename R>
static constexpr R K( double x )
{
	return static_cast<R>( x );
}

// ---------------------------------------------------------------------------------------
// models. Each mirrors the reference struct's arithmetic order exactly.
// ---------------------------------------------------------------------------------------
enum model_id
{
	VOGELS_ABBOTT = 0,
	BRUNEL = 1,
	BRUNEL_PLUS = 2,
	SYNTH = 3,
	// the benchmark configurations' constants (include/spice/models/vogels_abbott_ns.h,
	// brunel_fixed.h, brunel_with_plasticity_a012.h): the model above them, with the
	// differences restated where they apply
	VOGELS_ABBOTT_NS = 4,
	BRUNEL_FIXED = 5,
	BRUNEL_PLUS_A012 = 6
};
constexpr int MODEL_COUNT = 7;

// the reference model a variant differs from
static int base_model( int m )
{
	return m == VOGELS_ABBOTT_NS ? VOGELS_ABBOTT : m == BRUNEL_FIXED ? BRUNEL : m == BRUNEL_PLUS_A012 ? BRUNEL_PLUS : m;
}

template <typename R>
struct state
{
	int model = 0;
	int n = 0;
	// neuron attributes
	std::vector<R> V, Gex, Gin;
	std::vector<int> Twait, Ncount;
	// synapse attributes (Brunel+ only)
	std::vector<R> W, Zpre, Zpost;
};

template <typename R>
struct sim
{
	layout lay;
	uint64_t width = 0;
	std::vector<int> edges;
	std::vector<int> row_len;
	state<R> s;
	float dt;
	int delay;
	uint64_t rng_seed;
	int istep = 0;
	kahan clock;
	std::vector<std::vector<int>> queue; // spike batches, oldest first
	std::vector<std::vector<uint8_t>> flags; // (delay+1) x n, Brunel+ only

	float rnd( int neuron ) const
	{
		return uniform_left_inc( neuron_u32( rng_seed, (uint32_t)neuron, (uint32_t)istep, 0 ) );
	}

	void init_state()
	{
		int const n = s.n;
		switch( base_model( s.model ) )
		{
		case VOGELS_ABBOTT: // vogels_abbott.h:23-33
			s.V.assign( n, K<R>( -0.06 ) );
			if( s.model == VOGELS_ABBOTT_NS ) // uniform in [-60, -50) mV from the initialisation draw
				for( int i = 0; i < n; i++ )
					s.V[i] = K<R>( -0.06 ) + ( K<R>( -0.05 ) - K<R>( -0.06 ) ) *
					                             static_cast<R>( uniform_left_inc( neuron_u32( rng_seed, (uint32_t)i, 0xFFFFFFFFu, 0 ) ) );
			s.Gex.assign( n, R( 0 ) );
			s.Gin.assign( n, R( 0 ) );
			s.Twait.assign( n, 0 );
			break;
		case BRUNEL: // brunel.h:20-28
		case BRUNEL_PLUS: // brunel_with_plasticity.h:27-36
			s.V.assign( n, R( 0 ) );
			s.Twait.assign( n, 0 );
			break;
		case SYNTH: // synth.h:21-27
			s.Ncount.assign( n, 0 );
			break;
		}
		if( base_model( s.model ) == BRUNEL_PLUS ) // brunel_with_plasticity.h:83-100
		{
			s.W.assign( edges.size(), R( 0 ) );
			s.Zpre.assign( edges.size(), R( 0 ) );
			s.Zpost.assign( edges.size(), R( 0 ) );
			int const nexc = static_cast<int>( K<R>( 0.9 ) * n );
			for( int src = 0; src < n; src++ )
				for( int j = 0; j < row_len[src]; j++ )
				{
					size_t const syn = (size_t)src * width + j;
					s.W[syn] = src < nexc ? K<R>( 0.0001 ) : K<R>( -0.0005 );
					s.Zpre[syn] = R( 1 );
					s.Zpost[syn] = R( 1 );
				}
			flags.assign( delay + 1, std::vector<uint8_t>( n, 0 ) );
		}
	}

	// neuron::update for neuron i; returns spiked
	bool update( int i, R dt_ )
	{
		int const n = s.n;
		switch( base_model( s.model ) )
		{
		case VOGELS_ABBOTT:
		{ // vogels_abbott.h:35-71
			int const Tref = 50;
			R const Vrest = K<R>( -0.06 ), Vthres = K<R>( -0.05 ), TmemInv = R( 1 ) / K<R>( 0.02 );
			R const Eex = R( 0 ), Ein = K<R>( -0.08 ), Ibg = K<R>( 0.02 );
			R const TexInv = R( 1 ) / K<R>( 0.005 ), TinInv = R( 1 ) / K<R>( 0.01 );
			R & V = s.V[i];
			R & Gex = s.Gex[i];
			R & Gin = s.Gin[i];
			int & Tw = s.Twait[i];
			bool spiked = false;
			if( --Tw <= 0 )
			{
				if( V > Vthres )
				{
					V = Vrest;
					Tw = Tref;
					spiked = true;
				}
				else
					V += ( ( Vrest - V ) + Gex * ( Eex - V ) + Gin * ( Ein - V ) + Ibg ) * ( dt_ * TmemInv );
			}
			Gex -= Gex * ( dt_ * TexInv );
			Gin -= Gin * ( dt_ * TinInv );
			return spiked;
		}
		case BRUNEL:
		case BRUNEL_PLUS:
		{ // brunel.h:30-62, brunel_with_plasticity.h:38-68
			R const TmemInv = static_cast<R>( 1.0 / 0.02 ), Vrest = R( 0 ), Vthres = K<R>( 0.02 );
			int const Tref = 20;
			if( (uint32_t)i < static_cast<uint32_t>( n / 2 ) )
			{
				R const rate = 20;
				return static_cast<R>( rnd( i ) ) < ( rate * dt_ );
			}
			R & V = s.V[i];
			int & Tw = s.Twait[i];
			if( --Tw <= 0 )
			{
				if( V > Vthres )
				{
					// brunel_fixed resets to 10 mV
					V = s.model == BRUNEL_FIXED ? K<R>( 0.01 ) : Vrest;
					Tw = Tref;
					return true;
				}
				V += ( Vrest - V ) * ( dt_ * TmemInv );
			}
			return false;
		}
		case SYNTH: // synth.h:29-33
			return rnd( i ) < 0.005f;
		}
		return false;
	}

	// neuron::receive(src, dst, syn)
	void receive( int src, int dst, size_t syn )
	{
		int const n = s.n;
		switch( base_model( s.model ) )
		{
		case VOGELS_ABBOTT:
		{ // vogels_abbott.h:73-89; vogels_abbott_ns: 0.27 nS and 4.5 nS over the 10 nS leak
			bool const ns = s.model == VOGELS_ABBOTT_NS;
			R const Wex = ns ? K<R>( 0.27 ) / K<R>( 10 ) : K<R>( 0.4 ) * R( 16000000 ) / static_cast<R>( (int64_t)n * n );
			R const Win = ns ? K<R>( 4.5 ) / K<R>( 10 ) : K<R>( 5.1 ) * R( 16000000 ) / static_cast<R>( (int64_t)n * n );
			int const nexc = static_cast<int>( K<R>( 0.8 ) * n );
			if( src < nexc )
				s.Gex[dst] += Wex;
			else
				s.Gin[dst] += Win;
			break;
		}
		case BRUNEL:
		{ // brunel.h:64-80
			if( s.Twait[dst] <= 0 )
			{
				int const nexc = static_cast<int>( K<R>( 0.9 ) * n );
				// brunel_fixed: J = 0.1 / -0.5 mV, not scaled by 20,000 / N
				bool const fixed = s.model == BRUNEL_FIXED;
				R const Wex = fixed ? K<R>( 0.0001 ) : K<R>( 0.0001 ) * R( 20000 ) / static_cast<R>( n );
				R const Win = fixed ? K<R>( -0.0005 ) : K<R>( -0.0005 ) * R( 20000 ) / static_cast<R>( n );
				s.V[dst] += src < nexc ? Wex : Win;
			}
			break;
		}
		case BRUNEL_PLUS: // brunel_with_plasticity.h:70-77
			if( s.Twait[dst] <= 0 ) s.V[dst] += s.W[syn] * R( 20000 ) / static_cast<R>( n );
			break;
		case SYNTH: // synth.h:35-41
			s.Ncount[dst] += 1;
			break;
		}
	}

	// brunel_with_plasticity.h:102-127 (nsteps = 1 in the CPU sweep)
	void stdp( size_t syn, bool pre, bool post, R dt_ )
	{
		R const TstdpInv = R( 1 ) / K<R>( 0.02 );
		R const dtInv = R( 1 ) / dt_;
		R const decay = static_cast<R>( std::pow( R( 1 ) - dt_ * TstdpInv, R( 1 ) ) );
		R & zpre = s.Zpre[syn];
		R & zpost = s.Zpost[syn];
		R & w = s.W[syn];
		zpre = std::fma( zpre, decay, static_cast<R>( pre ) );
		zpost = std::fma( zpost, decay, static_cast<R>( post ) );
		R const a_minus = s.model == BRUNEL_PLUS_A012 ? K<R>( 0.012 ) : K<R>( 0.0202 );
		R const x = w - pre * a_minus * w * std::exp( -zpost * dtInv ) +
		            post * K<R>( 0.01 ) * ( R( 1 ) - w ) * std::exp( -zpre * dtInv );
		w = std::min( K<R>( 0.0003 ), std::max( R( 0 ), x ) );
	}

	static bool plastic( int src, int dst, int n ) // brunel_with_plasticity.h:129-135
	{
		int const npoisson = n / 2;
		int const nexc = 9 * n / 10;
		return src >= npoisson && src < nexc && dst < nexc;
	}

	// cpu::snn::step (spice/cpu/snn.h.cpp:114-181)
	void step( std::vector<int> & out )
	{
		float const dt_f = clock.add( dt );
		R const dt_ = static_cast<R>( dt_f );
		int const n = s.n;
		int const post = istep % ( delay + 1 );
		int const pre = ( istep + 1 ) % ( delay + 1 );

		if( (int)queue.size() >= delay ) // receive, ascending spike order, ascending dst
		{
			for( int src : queue.front() )
				for( int j = 0; j < row_len[src]; j++ )
					receive( src, edges[(size_t)src * width + j], (size_t)src * width + j );
			queue.erase( queue.begin() );
		}

		out.clear();
		for( int i = 0; i < n; i++ )
		{
			bool const spiked = update( i, dt_ );
			if( base_model( s.model ) == BRUNEL_PLUS ) flags[post][i] = spiked;
			if( spiked ) out.push_back( i );
		}
		queue.push_back( out );

		if( base_model( s.model ) == BRUNEL_PLUS )
		{
			// every synapse's update reads only its own state and the step's flags, so rows
			// are independent: large nets sweep them on several threads (same results)
			auto sweep = [&]( int r0, int r1 ) {
				for( int src = r0; src < r1; src++ )
					for( int j = 0; j < row_len[src]; j++ )
					{
						int const dst = edges[(size_t)src * width + j];
						if( plastic( src, dst, n ) ) stdp( (size_t)src * width + j, flags[pre][src], flags[post][dst], dt_ );
					}
			};
			int const nthreads = (size_t)n * width < ( 1u << 22 ) ? 1 : sweep_threads();
			if( nthreads <= 1 )
				sweep( 0, n );
			else
			{
				std::vector<std::thread> pool;
				for( int k = 0; k < nthreads; k++ )
					pool.emplace_back( sweep, (int)( (long long)n * k / nthreads ), (int)( (long long)n * ( k + 1 ) / nthreads ) );
				for( auto & t : pool ) t.join();
			}
		}
		istep++;
	}
};

struct handle_base
{
	virtual ~handle_base() = default;
};
template <typename R>
struct handle : handle_base
{
	sim<R> s;
};
} // namespace oracle

using namespace oracle;

namespace
{
thread_local std::string g_err;

layout layout_from( int npops, uint64_t const * pops, int nconn, int const * csrc, int const * cdst, float const * cp )
{
	std::vector<uint64_t> p( pops, pops + npops );
	std::vector<std::tuple<int, int, float>> c;
	for( int i = 0; i < nconn; i++ ) c.emplace_back( csrc[i], cdst[i], cp[i] );
	return make_layout( p, c );
}

template <typename R>
sim<R> & S( void * h )
{
	return static_cast<handle<R> *>( h )->s;
}
bool is64( void * h ) { return dynamic_cast<handle<double> *>( static_cast<handle_base *>( h ) ) != nullptr; }
} // namespace

// Neuron attributes in the reference's order, as float64 arrays (ints converted):
// VA (V, Gex, Gin, Twait); Brunel/Brunel+ (V, Twait); synth (N).
template <typename R>
static void export_neurons( sim<R> & s, double ** a )
{
	auto put = [&]( double * dst, auto const & v ) {
		for( size_t i = 0; i < v.size(); i++ ) dst[i] = (double)v[i];
	};
	switch( base_model( s.s.model ) )
	{
	case VOGELS_ABBOTT:
		put( a[0], s.s.V ), put( a[1], s.s.Gex ), put( a[2], s.s.Gin ), put( a[3], s.s.Twait );
		break;
	case BRUNEL:
	case BRUNEL_PLUS: put( a[0], s.s.V ), put( a[1], s.s.Twait ); break;
	case SYNTH: put( a[0], s.s.Ncount ); break;
	}
}
extern "C" {
char const * oracle_last_error() { return g_err.c_str(); }

int oracle_layout(
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
		layout const l = layout_from( npops, pops, nconn, csrc, cdst, cp );
		int i = 0;
		for( auto const & c : l.conns )
		{
			if( i < cap )
			{
				out_ranges[4 * i + 0] = c.src_first;
				out_ranges[4 * i + 1] = c.src_last;
				out_ranges[4 * i + 2] = c.dst_first;
				out_ranges[4 * i + 3] = c.dst_last;
				out_p[i] = c.p;
			}
			i++;
		}
		*max_degree = l.max_degree;
		*size = l.n;
		return i;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return -1;
	}
}

// graph: 0 = reference generator (seed), 1 = Philox Bernoulli generator (seed)
int oracle_generate(
    int graph, uint64_t seed, int npops, uint64_t const * pops, int nconn, int const * csrc, int const * cdst, float const * cp, int * out )
{
	try
	{
		layout const l = layout_from( npops, pops, nconn, csrc, cdst, cp );
		std::vector<int> e;
		if( graph == 0 )
			reference_generate( l, seed, e );
		else
			philox_generate( l, seed, e );
		std::memcpy( out, e.data(), e.size() * sizeof( int ) );
		return 0;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return -1;
	}
}

// one Philox-generated row (random access; used to spot-check GPU graphs at full size)
int oracle_philox_row(
    uint64_t seed, int npops, uint64_t const * pops, int nconn, int const * csrc, int const * cdst, float const * cp, int row, int * out )
{
	try
	{
		layout const l = layout_from( npops, pops, nconn, csrc, cdst, cp );
		philox_row( l, seed, row, out );
		return 0;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return -1;
	}
}

// Create a net. `edges` (n x width ELL, INT_MAX padded) is imported when non-null, as the
// reference's conversion constructor does (spice/cuda/snn.d.cpp:123-143); otherwise the
// graph is generated with `graph` (0 reference generator, 1 Philox) from `graph_seed`.
// precision: 32 or 64.
void * oracle_create(
    int model,
    int precision,
    int npops,
    uint64_t const * pops,
    int nconn,
    int const * csrc,
    int const * cdst,
    float const * cp,
    float dt,
    int delay,
    uint64_t rng_seed,
    int graph,
    uint64_t graph_seed,
    int const * edges,
    uint64_t width )
{
	try
	{
		if( !( dt > 0.0f ) ) throw std::invalid_argument( "dt must be > 0" );
		if( delay < 1 ) throw std::invalid_argument( "delay must be >= 1" );
		if( model < 0 || model >= MODEL_COUNT ) throw std::invalid_argument( "invalid model" );
		auto build = [&]( auto * h ) -> void * {
			auto & s = h->s;
			s.lay = layout_from( npops, pops, nconn, csrc, cdst, cp );
			if( edges )
			{
				s.width = width;
				s.edges.assign( edges, edges + s.lay.n * width );
			}
			else
			{
				s.width = s.lay.max_degree;
				if( graph == 0 )
					reference_generate( s.lay, graph_seed, s.edges );
				else
					philox_generate( s.lay, graph_seed, s.edges );
			}
			s.s.model = model;
			s.s.n = (int)s.lay.n;
			s.row_len.assign( s.lay.n, 0 );
			for( uint64_t i = 0; i < s.lay.n; i++ )
			{
				int const * r = s.edges.data() + i * s.width;
				s.row_len[i] = (int)( std::lower_bound( r, r + s.width, INT_MAX ) - r );
			}
			s.dt = dt;
			s.delay = delay;
			s.rng_seed = rng_seed;
			s.init_state();
			return h;
		};
		if( precision == 64 )
			return build( new handle<double>() );
		return build( new handle<float>() );
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return nullptr;
	}
}

void oracle_destroy( void * h ) { delete static_cast<handle_base *>( h ); }

int oracle_step( void * h, int * out, int cap )
{
	std::vector<int> v;
	if( is64( h ) )
		S<double>( h ).step( v );
	else
		S<float>( h ).step( v );
	for( int i = 0; i < (int)v.size() && i < cap; i++ ) out[i] = v[i];
	return (int)v.size();
}

uint64_t oracle_num_neurons( void * h ) { return is64( h ) ? S<double>( h ).s.n : S<float>( h ).s.n; }
uint64_t oracle_width( void * h ) { return is64( h ) ? S<double>( h ).width : S<float>( h ).width; }
void oracle_adj( void * h, int * out )
{
	auto const & e = is64( h ) ? S<double>( h ).edges : S<float>( h ).edges;
	std::memcpy( out, e.data(), e.size() * sizeof( int ) );
}

void oracle_neurons( void * h, double ** attrs )
{
	if( is64( h ) )
		export_neurons( S<double>( h ), attrs );
	else
		export_neurons( S<float>( h ), attrs );
}

// Brunel+ synapse attributes (W, Zpre, Zpost) over all n x width slots, as float64.
void oracle_synapses( void * h, double ** a )
{
	auto go = [&]( auto & s ) {
		for( size_t i = 0; i < s.s.W.size(); i++ )
		{
			a[0][i] = s.s.W[i];
			a[1][i] = s.s.Zpre[i];
			a[2][i] = s.s.Zpost[i];
		}
	};
	if( is64( h ) )
		go( S<double>( h ) );
	else
		go( S<float>( h ) );
}

// Replace the neuron state (one array per attribute in the reference's order, float32 or
// int32 as the model declares them) and, for Brunel+, the synapse state (W, Zpre, Zpost,
// float32 over all n x width slots): a net that starts from another simulator's state, as
// the conversion constructor does (spice/cuda/snn.d.cpp:201-221).
void oracle_set_state( void * h, void * const * neurons, void * const * synapses )
{
	auto go = [&]( auto & s ) {
		using R = typename std::remove_reference_t<decltype( s.s.V )>::value_type;
		auto fl = [&]( auto & dst, void const * src ) {
			float const * f = static_cast<float const *>( src );
			for( size_t i = 0; i < dst.size(); i++ ) dst[i] = static_cast<R>( f[i] );
		};
		auto in = [&]( std::vector<int> & dst, void const * src ) { std::memcpy( dst.data(), src, dst.size() * 4 ); };
		switch( base_model( s.s.model ) )
		{
		case VOGELS_ABBOTT: fl( s.s.V, neurons[0] ), fl( s.s.Gex, neurons[1] ), fl( s.s.Gin, neurons[2] ), in( s.s.Twait, neurons[3] ); break;
		case BRUNEL:
		case BRUNEL_PLUS: fl( s.s.V, neurons[0] ), in( s.s.Twait, neurons[1] ); break;
		case SYNTH: in( s.s.Ncount, neurons[0] ); break;
		}
		if( base_model( s.s.model ) == BRUNEL_PLUS && synapses ) fl( s.s.W, synapses[0] ), fl( s.s.Zpre, synapses[1] ), fl( s.s.Zpost, synapses[2] );
	};
	if( is64( h ) )
		go( S<double>( h ) );
	else
		go( S<float>( h ) );
}

// Continue a run at step step0: the simulated clock advanced by step0 steps (the Poisson
// draws keyed by the step follow) and the spikes of the steps [step0 - nq, step0) in flight
// (counts[nq], ids concatenated, oldest first; nq <= delay), with their firing flags.
int oracle_set_progress( void * h, uint64_t step0, int nq, uint32_t const * counts, int const * ids )
{
	auto go = [&]( auto & s ) {
		if( nq < 0 || nq > s.delay || (uint64_t)nq > step0 ) throw std::invalid_argument( "spikes in flight: at most delay steps" );
		s.istep = (int)step0;
		s.clock = kahan{};
		for( uint64_t k = 0; k < step0; k++ ) s.clock.add( s.dt );
		s.queue.clear();
		size_t o = 0;
		for( int q = 0; q < nq; q++ )
		{
			s.queue.emplace_back( ids + o, ids + o + counts[q] );
			if( base_model( s.s.model ) == BRUNEL_PLUS )
				for( uint32_t k = 0; k < counts[q]; k++ ) s.flags[( step0 - nq + q ) % ( s.delay + 1 )][ids[o + k]] = 1;
			o += counts[q];
		}
	};
	try
	{
		if( is64( h ) )
			go( S<double>( h ) );
		else
			go( S<float>( h ) );
		return 0;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return -1;
	}
}

// Exact float32 views for bit-level comparisons (precision 32 only).
void oracle_neurons_f32( void * h, void ** a )
{
	auto & s = S<float>( h );
	auto cpy = [&]( void * dst, auto const & v ) { std::memcpy( dst, v.data(), v.size() * 4 ); };
	switch( base_model( s.s.model ) )
	{
	case VOGELS_ABBOTT: cpy( a[0], s.s.V ), cpy( a[1], s.s.Gex ), cpy( a[2], s.s.Gin ), cpy( a[3], s.s.Twait ); break;
	case BRUNEL:
	case BRUNEL_PLUS: cpy( a[0], s.s.V ), cpy( a[1], s.s.Twait ); break;
	case SYNTH: cpy( a[0], s.s.Ncount ); break;
	}
}
void oracle_synapses_f32( void * h, void ** a )
{
	auto & s = S<float>( h );
	std::memcpy( a[0], s.s.W.data(), s.s.W.size() * 4 );
	std::memcpy( a[1], s.s.Zpre.data(), s.s.Zpre.size() * 4 );
	std::memcpy( a[2], s.s.Zpost.data(), s.s.Zpost.size() * 4 );
}

// The Kahan-compensated dt sequence (first `count` steps) for a given dt.
void oracle_dt_sequence( float dt, int count, float * out )
{
	kahan k;
	for( int i = 0; i < count; i++ ) out[i] = k.add( dt );
}

// Philox known-answer check helper.
void oracle_philox( uint32_t const * ctr, uint32_t const * key, uint32_t * out )
{
	philox_out const r = philox4x32_10( ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1] );
	std::memcpy( out, r.v, 16 );
}
}
