// spice::cuda::batch and spice::cuda::server -- many nets on one GPU, over the C ABI of
// libspice_b200.so (include/spice_b200.h). The reference steps one snn per object
// (spice/cuda/snn.h:16-77); a batch steps many with shared launches (results identical to
// stepping each alone) and a server admits simulation jobs against a device-memory budget
// and steps them by continuous batching. Errors are thrown as in spice/cuda/snn.h.
#pragma once

#include <spice/cuda/snn.h>

#include <cstdint>
#include <vector>

namespace spice
{
namespace cuda
{
class batch
{
public:
	explicit batch( int device = 0 ) { check( spk_batch_create( &_b, device ) ); }
	batch( batch const & ) = delete;
	batch & operator=( batch const & ) = delete;
	~batch()
	{
		if( _b ) spk_batch_destroy( _b );
	}

	// the net stays owned by the caller; destroying it removes it from the batch
	template <typename Model>
	void add( snn<Model> & net )
	{
		check( spk_batch_add( _b, net.handle() ) );
	}
	template <typename Model>
	void remove( snn<Model> & net )
	{
		check( spk_batch_remove( _b, net.handle() ) );
	}
	// every net of the batch +nsteps steps
	void run( std::uint64_t nsteps ) { check( spk_batch_run( _b, nsteps ) ); }

private:
	spk_batch * _b = nullptr;
};

class server
{
public:
	// maps the budget into the device's stream-ordered pool the jobs' nets are built from
	// (spk_server_create); the destructor hands it back
	server( std::uint64_t budget_bytes, std::uint64_t quantum_steps, int device = 0 )
	{
		check( spk_server_create( &_s, device, budget_bytes, quantum_steps ) );
	}
	server( server const & ) = delete;
	server & operator=( server const & ) = delete;
	~server()
	{
		if( _s ) spk_server_destroy( _s );
	}

	// queue a job; throws std::bad_alloc if it alone exceeds the budget
	template <typename Model>
	std::uint64_t submit(
	    util::layout const & l, std::uint64_t nsteps, float dt, int delay = 1, std::uint64_t seed = 1, std::uint64_t graph_seed = 1337,
	    double timeout_s = 0 )
	{
		std::vector<std::uint64_t> pops;
		std::vector<int> src, dst;
		std::vector<float> p;
		for( auto x : l.populations() ) pops.push_back( x );
		for( auto const & c : l.population_connections() )
		{
			src.push_back( (int)std::get<0>( c ) );
			dst.push_back( (int)std::get<1>( c ) );
			p.push_back( std::get<2>( c ) );
		}
		spk_layout_desc d{ (int)pops.size(), pops.data(), (int)src.size(), src.data(), dst.data(), p.data() };
		std::uint64_t job = 0;
		check( spk_server_submit( _s, model_id<Model>::value, &d, dt, delay, seed, graph_seed, nsteps, timeout_s, &job ) );
		return job;
	}
	spk_job_info info( std::uint64_t job ) const
	{
		spk_job_info i{};
		check( spk_server_job_info( _s, job, &i ) );
		return i;
	}
	// block until the job (0: every job) is finished
	void wait( std::uint64_t job = 0, double timeout_s = -1 ) { check( spk_server_wait( _s, job, timeout_s ) ); }
	void cancel( std::uint64_t job ) { check( spk_server_cancel( _s, job ) ); }
	spk_server_stats stats() const
	{
		spk_server_stats st{};
		check( spk_server_get_stats( _s, &st ) );
		return st;
	}

private:
	spk_server * _s = nullptr;
};
} // namespace cuda
} // namespace spice
