// spice::util::layout -- population sizes plus (src_pop, dst_pop, p) connections,
// flattened into (src_first, src_last, dst_first, dst_last, p) index ranges, with the ELL
// row width max_degree() = mean + 3 sigma of the out-degree rounded up to a multiple of 32.
// Same interface and results as the reference (spice/util/layout.h:26-58,
// spice/util/layout.cpp:13-113); the multi-GPU cut()/static_load_balance() helpers are not
// part of the single-GPU path. Host-only, header-only.
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <tuple>
#include <vector>

namespace spice
{
namespace util
{
class layout
{
public:
	// (first src, last src, first dst, last dst, p)
	using edge = std::tuple<int, int, int, int, float>;

	layout( std::size_t num_neurons, float p )
	    : layout( std::vector<std::size_t>{ num_neurons }, { { 0, 0, p } } )
	{
	}

	layout( std::vector<std::size_t> const & pops, std::vector<std::tuple<std::size_t, std::size_t, float>> conns )
	{
		if( pops.empty() ) throw std::invalid_argument( "layout must contain at least 1 (non-empty) population" );
		for( auto p : pops )
			if( p == 0 || p > (std::size_t)INT_MAX ) throw std::invalid_argument( "invalid population size" );
		for( auto const & c : conns )
		{
			if( std::get<0>( c ) >= pops.size() || std::get<1>( c ) >= pops.size() )
				throw std::invalid_argument( "invalid index in connections matrix" );
			if( !( std::get<2>( c ) >= 0.0f && std::get<2>( c ) <= 1.0f ) )
				throw std::invalid_argument( "invalid connect. prob." );
		}
		std::sort( conns.begin(), conns.end(), []( auto const & a, auto const & b ) {
			return std::get<0>( a ) < std::get<0>( b ) || ( std::get<0>( a ) == std::get<0>( b ) && std::get<1>( a ) < std::get<1>( b ) );
		} );
		for( std::size_t i = 1; i < conns.size(); i++ )
			if( std::get<0>( conns[i] ) == std::get<0>( conns[i - 1] ) && std::get<1>( conns[i] ) == std::get<1>( conns[i - 1] ) )
				throw std::invalid_argument( "no duplicate edges in connections list allowed" );

		std::vector<std::size_t> first( pops.size() + 1, 0 );
		for( std::size_t i = 0; i < pops.size(); i++ ) first[i + 1] = first[i] + pops[i];
		if( first.back() > (std::size_t)INT_MAX ) throw std::invalid_argument( "too many neurons" );
		_n = first.back();
		for( auto const & c : conns )
		{
			auto const s = std::get<0>( c ), d = std::get<1>( c );
			_connections.emplace_back( (int)first[s], (int)first[s + 1], (int)first[d], (int)first[d + 1], std::get<2>( c ) );
		}
		_max_degree = estimate_width( _connections );
		_pops = pops;
		_pop_connections = conns;
	}

	std::size_t size() const { return _n; }
	// the constructor's inputs (connections sorted by (src, dst))
	std::vector<std::size_t> const & populations() const { return _pops; }
	std::vector<std::tuple<std::size_t, std::size_t, float>> const & population_connections() const { return _pop_connections; }
	std::vector<edge> const & connections() const { return _connections; }
	std::size_t max_degree() const { return _max_degree; }

	// mean + 3 sigma of the out-degree of the busiest source population (double
	// precision, truncated), rounded up to a multiple of 32
	static std::size_t estimate_width( std::vector<edge> const & cs )
	{
		int src = cs.empty() ? 0 : std::get<0>( cs.front() );
		std::size_t widest = 0;
		double mean = 0.0, var = 0.0;
		auto close_group = [&] { widest = std::max( widest, static_cast<std::size_t>( mean + 3 * std::sqrt( var ) ) ); };
		for( auto const & c : cs )
		{
			if( std::get<0>( c ) != src )
			{
				close_group();
				src = std::get<0>( c );
				mean = 0.0;
				var = 0.0;
			}
			double const range = static_cast<double>( std::get<3>( c ) - std::get<2>( c ) );
			float const p = std::get<4>( c );
			mean += range * p;
			var += range * p * ( 1.0 - p );
		}
		close_group();
		return ( widest + 31 ) / 32 * 32;
	}

private:
	std::size_t _n = 0;
	std::vector<edge> _connections;
	std::size_t _max_degree = 0;
	std::vector<std::size_t> _pops;
	std::vector<std::tuple<std::size_t, std::size_t, float>> _pop_connections;
};
} // namespace util
} // namespace spice
