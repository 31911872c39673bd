// Serving loop: simulation jobs submitted at any time, admitted against a device-memory
// budget, stepped together by continuous batching.
//
// The reference has no server; a workload of many nets is a host loop that builds and steps
// one net after another (spice_bench/paper_plots.cpp:184-231). Here a few builder threads
// and one ticker thread per server own the GPU side:
//   builders admit queued jobs in arrival order while their estimated device memory fits
//            the budget (a job larger than the whole budget is refused at submission) and
//            build each admitted job's net, with a tile count sized to its share of the
//            load, while the ticker steps the others;
//   ticker   each tick advances every running job by up to `quantum` steps in one batch
//            run (jobs built since the last tick join it: continuous batching), then
//            retires: finished jobs export their final neuron state to host memory and free
//            their device memory; cancelled, timed-out and failed jobs free theirs too.
// The server is a client of the C ABI only (spk_net_*, spk_batch_*): a job's results are
// those of the same net stepped alone.
#include <spice_b200.h>

#include <cuda_runtime_api.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

// defined in net.cu beside the C ABI: the per-thread error message (spk_last_error), nets
// built from the device's stream-ordered pool, and handing that pool's unused memory back
void spk_set_last_error( std::string const & msg );
int spk_net_create_pooled(
    spk_net ** out, int model, spk_layout_desc const * desc, float dt, int delay, uint64_t seed, uint64_t graph_seed, int device, int tile_target );
void spk_trim_pool( int device );
void spk_reserve_pool( int device, uint64_t bytes );
int spk_net_raise_device_error( spk_net * net );

namespace
{
// models with plastic synapses export synapse attributes (spk_model_attrs)
bool plastic_model( int model )
{
	int na = 0, ns = 0;
	return spk_model_attrs( model, &na, &ns, nullptr, 0 ) == SPK_OK && ns > 0;
}
} // namespace

namespace
{
// builder threads: 2 unless the creator asks (1-8); with jobs queued, a second builder
// overlaps one build's host work with another's kernels. SPK_SERVER_BUILDERS overrides the
// automatic choice (a test hook).
int builders_count( int requested )
{
	int n = requested;
	if( n <= 0 )
	{
		char const * e = getenv( "SPK_SERVER_BUILDERS" );
		n = e ? atoi( e ) : 2;
	}
	return n < 1 ? 1 : ( n > 8 ? 8 : n );
}

int fail( int code, std::string const & msg )
{
	spk_set_last_error( msg );
	return code;
}

struct job
{
	uint64_t id = 0;
	int model = 0;
	std::vector<uint64_t> pops;
	std::vector<int> src, dst;
	std::vector<float> p;
	float dt = 0;
	int delay = 1;
	uint64_t seed = 0, graph_seed = 0, nsteps = 0;
	double timeout_s = 0;

	int state = SPK_JOB_QUEUED;
	int error = SPK_OK;
	std::string message;
	uint64_t done = 0;
	uint64_t reserved = 0; // device bytes held against the budget
	uint64_t num_neurons = 0;
	double t_submit = 0, t_start = -1, t_end = -1;
	bool cancel = false;
	bool raise = false; // fault injection: its net reports a device error at its next tick
	spk_net * net = nullptr;
	double work = 0;                           // expected cost per step (tiling share)
	bool own = false;                          // steps on its own stream, not in the shared launches (Brunel+)
	uint64_t inflight = 0;                     // own-stream steps launched, not yet seen finished
	std::vector<std::vector<uint32_t>> result; // final neuron attributes (4-byte words)

	spk_layout_desc desc() const
	{
		return { (int)pops.size(), pops.data(), (int)src.size(), src.data(), dst.data(), p.data() };
	}
	bool final() const { return state >= SPK_JOB_DONE; }
};

struct server
{
	int device = 0;
	uint64_t budget = 0, quantum = 0;
	int sms = 148;
	spk_batch * batch = nullptr;
	std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

	std::mutex mu;
	std::condition_variable wake, changed;
	bool stop = false;
	uint64_t next_id = 1;
	std::map<uint64_t, std::unique_ptr<job>> jobs;
	std::deque<job *> queue;
	std::vector<job *> building, ready; // admitted: net being built / built, not yet ticked
	std::vector<job *> running;         // in the batch (copy of the ticker's list)
	std::vector<job *> running_t;       // the ticker's own list
	std::condition_variable tick_wake;
	uint64_t in_use = 0, peak = 0, ticks = 0;
	double build_s = 0, tick_s = 0;
	int inject = 0;
	std::vector<std::thread> builders; // builder threads: they admit and build concurrently
	std::thread ticker;

	double now() const { return std::chrono::duration<double>( std::chrono::steady_clock::now() - t0 ).count(); }

	void finish( job & j, int state, int error = SPK_OK, std::string const & msg = {} )
	{
		j.state = state;
		j.error = error;
		j.message = msg;
		j.t_end = now();
		changed.notify_all();
	}

	// tile target of a new job: its share of the SMs by expected work against the jobs
	// already running (one tile at least)
	int tile_target( job const & j ) const
	{
		double total = j.work;
		for( auto * r : running ) total += r->work;
		return std::max( 1, (int)std::lround( sms * j.work / total ) );
	}

	// build the net of an admitted job (lock not held; the ticker adds it to the batch)
	int build( job & j, int target, std::string & msg )
	{
		auto const d = j.desc();
		// from the stream-ordered pool: no device-wide synchronisation while the ticker runs
		int const rc = spk_net_create_pooled( &j.net, j.model, &d, j.dt, j.delay, j.seed, j.graph_seed, device, target );
		if( rc != SPK_OK )
		{
			msg = spk_last_error();
			j.net = nullptr;
		}
		return rc;
	}

	// builder thread: deadlines of queued jobs, admission in arrival order while the head
	// fits the budget, and the admitted jobs' nets (built while the ticker steps others)
	void build_loop()
	{
		std::unique_lock<std::mutex> lk( mu );
		while( !stop )
		{
			double const t = now();
			for( auto it = queue.begin(); it != queue.end(); )
			{
				job & j = **it;
				if( j.cancel || ( j.timeout_s > 0 && t - j.t_submit > j.timeout_s ) )
				{
					finish( j, j.cancel ? SPK_JOB_CANCELLED : SPK_JOB_TIMEOUT );
					it = queue.erase( it );
				}
				else
					++it;
			}
			if( queue.empty() || in_use + queue.front()->reserved > budget )
			{
				wake.wait_for( lk, std::chrono::milliseconds( 20 ) );
				continue;
			}
			job & j = *queue.front();
			queue.pop_front();
			in_use += j.reserved;
			peak = std::max( peak, in_use );
			j.state = SPK_JOB_RUNNING;
			j.t_start = now();
			int const target = tile_target( j );
			bool const injected = inject > 0;
			if( injected ) inject--;
			building.push_back( &j );
			lk.unlock();
			std::string msg;
			double const tb = now();
			int const rc = injected ? ( msg = "injected allocation failure", SPK_ERR_NOMEM ) : build( j, target, msg );
			lk.lock();
			build_s += now() - tb;
			building.erase( std::find( building.begin(), building.end(), &j ) );
			if( rc != SPK_OK )
			{
				in_use -= j.reserved;
				j.reserved = 0;
				finish( j, SPK_JOB_FAILED, rc, msg );
				continue;
			}
			// held against the budget: the estimate, or what the net holds if that is more
			// (admission stays within the budget even where an estimate falls short)
			spk_net_info info{};
			if( spk_net_get_info( j.net, &info ) == SPK_OK && info.device_bytes > j.reserved )
			{
				in_use += info.device_bytes - j.reserved;
				j.reserved = info.device_bytes;
				peak = std::max( peak, in_use );
			}
			ready.push_back( &j );
			tick_wake.notify_all();
		}
	}

	// ticker thread: built jobs join the batch; every tick advances each running job by up
	// to `quantum` steps; finished, failed, cancelled and timed-out jobs leave
	void tick_loop()
	{
		std::unique_lock<std::mutex> lk( mu );
		while( !stop )
		{
			std::vector<job *> joining;
			joining.swap( ready );
			lk.unlock();
			std::vector<std::pair<job *, std::string>> rejected;
			for( auto * j : joining )
			{
				spk_net_info info{};
				if( spk_net_get_info( j->net, &info ) == SPK_OK && spk_batch_add( batch, j->net ) == SPK_OK )
				{
					// nets outside the shared launches (window_counts, window_ordered) run on
					// their own streams, each at its own pace: the ticks of the shared
					// launches do not wait for them; plastic nets share window_plastic_batch
					j->own = !plastic_model( info.model ) && info.slice_pack == 0;
					running_t.push_back( j );
				}
				else
					rejected.push_back( { j, spk_last_error() } );
			}
			for( auto & r : rejected )
			{
				spk_net_destroy( r.first->net );
				r.first->net = nullptr;
			}
			lk.lock();
			for( auto & r : rejected )
			{
				in_use -= r.first->reserved;
				r.first->reserved = 0;
				finish( *r.first, SPK_JOB_FAILED, SPK_ERR_INVALID, r.second );
			}
			running = running_t;
			if( running_t.empty() )
			{
				tick_wake.wait_for( lk, std::chrono::milliseconds( 20 ) );
				continue;
			}
			// one tick: every job of the shared launches up to `quantum` steps, synchronised;
			// own-stream jobs: a finished quantum is counted and the next one launched
			std::vector<spk_net *> nets;
			std::vector<uint64_t> counts;
			std::vector<job *> ticked, owns, raised;
			for( auto * j : running_t )
			{
				if( j->raise )
				{
					raised.push_back( j );
					j->raise = false;
				}
				if( j->own )
					owns.push_back( j );
				else if( !j->cancel && j->done < j->nsteps )
				{
					nets.push_back( j->net );
					counts.push_back( std::min( quantum, j->nsteps - j->done ) );
					ticked.push_back( j );
				}
			}
			lk.unlock();
			for( auto * j : raised ) spk_net_raise_device_error( j->net );
			double const tt = now();
			std::vector<int> status( ticked.size(), SPK_OK );
			std::vector<std::string> msgs( ticked.size() );
			std::vector<int> own_status( owns.size(), SPK_OK );
			std::vector<std::string> own_msgs( owns.size() );
			std::vector<uint64_t> own_done( owns.size(), 0 ), own_launch( owns.size(), 0 );
			bool own_busy = false;
			for( size_t i = 0; i < owns.size(); i++ )
			{
				job & j = *owns[i];
				int idle = 0;
				int r = spk_net_idle( j.net, &idle );
				if( r == SPK_OK && idle && j.inflight ) r = spk_net_sync( j.net ); // its quantum ended: errors?
				if( r != SPK_OK )
				{
					own_status[i] = r;
					own_msgs[i] = spk_last_error();
					continue;
				}
				if( !idle )
				{
					own_busy = true;
					continue;
				}
				own_done[i] = j.inflight;
				uint64_t const left = j.nsteps - j.done - j.inflight;
				if( !j.cancel && left > 0 )
				{
					own_launch[i] = std::min( quantum, left );
					r = spk_net_run( j.net, own_launch[i] );
					if( r != SPK_OK )
					{
						own_status[i] = r;
						own_msgs[i] = spk_last_error();
						own_launch[i] = 0;
					}
					else
						own_busy = true;
				}
			}
			int rc = nets.empty() ? SPK_OK : spk_batch_run_nets( batch, (int)nets.size(), nets.data(), counts.data() );
			std::string const run_msg = rc != SPK_OK ? spk_last_error() : "";
			for( size_t i = 0; i < ticked.size(); i++ )
			{
				status[i] = rc != SPK_OK ? rc : spk_net_sync( nets[i] );
				if( status[i] != SPK_OK ) msgs[i] = rc != SPK_OK ? run_msg : spk_last_error();
			}
			lk.lock();
			ticks++;
			tick_s += now() - tt;
			for( size_t i = 0; i < ticked.size(); i++ )
				if( status[i] == SPK_OK ) ticked[i]->done += counts[i];
			for( size_t i = 0; i < owns.size(); i++ )
			{
				owns[i]->done += own_done[i];
				owns[i]->inflight = own_launch[i] ? own_launch[i] : ( own_done[i] ? 0 : owns[i]->inflight );
			}
			// the same outcome lists for both kinds of jobs
			for( size_t i = 0; i < owns.size(); i++ )
			{
				ticked.push_back( owns[i] );
				status.push_back( own_status[i] );
				msgs.push_back( own_msgs[i] );
			}
			// retire
			double const te = now();
			std::vector<std::pair<job *, int>> leaving; // (job, final state)
			std::vector<int> errs;
			std::vector<std::string> emsgs;
			for( auto it = running_t.begin(); it != running_t.end(); )
			{
				job & j = **it;
				auto const k = std::find( ticked.begin(), ticked.end(), &j ) - ticked.begin();
				int const st = (size_t)k < ticked.size() ? status[k] : SPK_OK;
				int state = -1;
				if( st != SPK_OK ) state = SPK_JOB_FAILED;
				else if( j.done >= j.nsteps ) state = SPK_JOB_DONE;
				else if( j.own && j.inflight ) state = -1; // its quantum still runs
				else if( j.cancel ) state = SPK_JOB_CANCELLED;
				else if( j.timeout_s > 0 && te - j.t_submit > j.timeout_s ) state = SPK_JOB_TIMEOUT;
				if( state < 0 )
				{
					++it;
					continue;
				}
				leaving.push_back( { &j, state } );
				errs.push_back( st );
				emsgs.push_back( (size_t)k < ticked.size() ? msgs[k] : std::string() );
				it = running_t.erase( it );
			}
			running = running_t;
			lk.unlock();
			for( size_t i = 0; i < leaving.size(); i++ )
			{
				job & j = *leaving[i].first;
				if( leaving[i].second == SPK_JOB_DONE )
				{
					spk_net_info info{};
					int na = 0, ns = 0;
					char types[16];
					int r = spk_net_get_info( j.net, &info );
					if( r == SPK_OK ) r = spk_model_attrs( j.model, &na, &ns, types, sizeof types );
					std::vector<std::vector<uint32_t>> res( na, std::vector<uint32_t>( info.num_neurons ) );
					std::vector<void *> ptrs;
					for( auto & a : res ) ptrs.push_back( a.data() );
					if( r == SPK_OK ) r = spk_net_neurons( j.net, ptrs.data() );
					if( r != SPK_OK )
					{
						leaving[i].second = SPK_JOB_FAILED;
						errs[i] = r;
						emsgs[i] = spk_last_error();
					}
					else
					{
						j.result = std::move( res );
						j.num_neurons = info.num_neurons;
					}
				}
				spk_batch_remove( batch, j.net );
				spk_net_destroy( j.net );
				j.net = nullptr;
			}
			lk.lock();
			for( size_t i = 0; i < leaving.size(); i++ )
			{
				job & j = *leaving[i].first;
				in_use -= j.reserved;
				j.reserved = 0;
				finish( j, leaving[i].second, errs[i], emsgs[i] );
			}
			if( !leaving.empty() ) wake.notify_all(); // budget freed
			// only own-stream jobs running, all busy: poll again shortly, not in a spin
			if( nets.empty() && own_busy && leaving.empty() ) tick_wake.wait_for( lk, std::chrono::microseconds( 200 ) );
		}
	}
};
} // namespace

struct spk_server : server
{
};

extern "C" {
int spk_server_create( spk_server ** out, int device, uint64_t budget_bytes, uint64_t quantum_steps )
{
	return spk_server_create_ex( out, device, budget_bytes, quantum_steps, 0 );
}

int spk_server_create_ex( spk_server ** out, int device, uint64_t budget_bytes, uint64_t quantum_steps, int builders )
{
	if( !out ) return fail( SPK_ERR_INVALID, "out is null" );
	if( builders < 0 || builders > 8 ) return fail( SPK_ERR_INVALID, "builders must be 0 (automatic) to 8" );
	*out = nullptr;
	if( budget_bytes == 0 || quantum_steps == 0 ) return fail( SPK_ERR_INVALID, "budget and quantum must be > 0" );
	auto s = std::make_unique<spk_server>();
	s->device = device;
	s->budget = budget_bytes;
	s->quantum = quantum_steps;
	if( cudaDeviceGetAttribute( &s->sms, cudaDevAttrMultiProcessorCount, device ) != cudaSuccess )
		return fail( SPK_ERR_INVALID, "invalid device" );
	int const rc = spk_batch_create( &s->batch, device );
	if( rc != SPK_OK ) return rc;
	// the budget mapped into the pool the nets are built from, before any job runs
	spk_reserve_pool( device, budget_bytes );
	for( int b = 0, nb = builders_count( builders ); b < nb; b++ ) s->builders.emplace_back( [p = s.get()] { p->build_loop(); } );
	s->ticker = std::thread( [p = s.get()] { p->tick_loop(); } );
	*out = s.release();
	return SPK_OK;
}

int spk_server_submit(
    spk_server * s,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    uint64_t nsteps,
    double timeout_s,
    uint64_t * out_job )
{
	if( !s || !desc || !out_job ) return fail( SPK_ERR_INVALID, "null argument" );
	if( nsteps == 0 ) return fail( SPK_ERR_INVALID, "nsteps must be > 0" );
	if( plastic_model( model ) && delay > 63 ) return fail( SPK_ERR_INVALID, "plastic models support delays up to 63 steps" );
	if( desc->npops <= 0 || !desc->pops || desc->nconn < 0 || ( desc->nconn && ( !desc->conn_src || !desc->conn_dst || !desc->conn_p ) ) )
		return fail( SPK_ERR_INVALID, "bad layout descriptor" );
	auto j = std::make_unique<job>();
	j->model = model;
	j->pops.assign( desc->pops, desc->pops + desc->npops );
	j->src.assign( desc->conn_src, desc->conn_src + desc->nconn );
	j->dst.assign( desc->conn_dst, desc->conn_dst + desc->nconn );
	j->p.assign( desc->conn_p, desc->conn_p + desc->nconn );
	j->dt = dt;
	j->delay = delay;
	j->seed = seed;
	j->graph_seed = graph_seed;
	j->nsteps = nsteps;
	j->timeout_s = timeout_s;
	// admission estimate at the largest tiling (one tile per SM), and the job's work share
	uint64_t est = 0;
	auto const d = j->desc();
	int const rc = spk_net_estimate_bytes( model, &d, delay, s->device, 0, &est );
	if( rc != SPK_OK ) return rc;
	double syn = 0, n = 0;
	for( int i = 0; i < desc->nconn; i++ )
		syn += (double)desc->pops[desc->conn_src[i]] * (double)desc->pops[desc->conn_dst[i]] * desc->conn_p[i];
	for( int i = 0; i < desc->npops; i++ ) n += (double)desc->pops[i];
	j->work = syn * 0.01 + 1000.0 * n;
	std::lock_guard<std::mutex> lk( s->mu );
	j->id = s->next_id++;
	j->t_submit = s->now();
	j->reserved = est;
	*out_job = j->id;
	if( est > s->budget )
	{
		j->state = SPK_JOB_REFUSED;
		j->error = SPK_ERR_NOMEM;
		j->message = "the job's device memory exceeds the server's budget";
		j->t_end = j->t_submit;
		j->reserved = 0;
		s->jobs[j->id] = std::move( j );
		return fail( SPK_ERR_NOMEM, "the job's device memory (" + std::to_string( est ) + " B) exceeds the budget" );
	}
	s->queue.push_back( j.get() );
	s->jobs[j->id] = std::move( j );
	s->wake.notify_all();
	return SPK_OK;
}

int spk_server_job_info( spk_server * s, uint64_t id, spk_job_info * out )
{
	if( !s || !out ) return fail( SPK_ERR_INVALID, "null argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	auto it = s->jobs.find( id );
	if( it == s->jobs.end() ) return fail( SPK_ERR_INVALID, "unknown job" );
	job const & j = *it->second;
	std::memset( out, 0, sizeof *out );
	out->state = j.state;
	out->error = j.error;
	out->steps_done = j.done;
	out->steps_total = j.nsteps;
	out->num_neurons = j.num_neurons;
	out->device_bytes = j.reserved;
	out->t_submit = j.t_submit;
	out->t_start = j.t_start;
	out->t_end = j.t_end;
	std::strncpy( out->message, j.message.c_str(), sizeof out->message - 1 );
	return SPK_OK;
}

int spk_server_job_neurons( spk_server * s, uint64_t id, void * const * attrs )
{
	if( !s || !attrs ) return fail( SPK_ERR_INVALID, "null argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	auto it = s->jobs.find( id );
	if( it == s->jobs.end() ) return fail( SPK_ERR_INVALID, "unknown job" );
	job const & j = *it->second;
	if( j.state != SPK_JOB_DONE ) return fail( SPK_ERR_INVALID, "the job has not completed" );
	for( size_t a = 0; a < j.result.size(); a++ )
	{
		if( !attrs[a] ) return fail( SPK_ERR_INVALID, "attribute pointer is null" );
		std::memcpy( attrs[a], j.result[a].data(), j.result[a].size() * 4 );
	}
	return SPK_OK;
}

int spk_server_cancel( spk_server * s, uint64_t id )
{
	if( !s ) return fail( SPK_ERR_INVALID, "null argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	auto it = s->jobs.find( id );
	if( it == s->jobs.end() ) return fail( SPK_ERR_INVALID, "unknown job" );
	it->second->cancel = true;
	s->wake.notify_all();
	return SPK_OK;
}

int spk_server_release( spk_server * s, uint64_t id )
{
	if( !s ) return fail( SPK_ERR_INVALID, "null argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	auto it = s->jobs.find( id );
	if( it == s->jobs.end() ) return fail( SPK_ERR_INVALID, "unknown job" );
	if( !it->second->final() ) return fail( SPK_ERR_INVALID, "the job is still queued or running" );
	s->jobs.erase( it );
	return SPK_OK;
}

int spk_server_wait( spk_server * s, uint64_t id, double timeout_s )
{
	if( !s ) return fail( SPK_ERR_INVALID, "null argument" );
	std::unique_lock<std::mutex> lk( s->mu );
	auto done = [&] {
		if( id == 0 )
		{
			for( auto const & kv : s->jobs )
				if( !kv.second->final() ) return false;
			return true;
		}
		auto it = s->jobs.find( id );
		return it == s->jobs.end() || it->second->final();
	};
	if( id != 0 && !s->jobs.count( id ) ) return fail( SPK_ERR_INVALID, "unknown job" );
	if( timeout_s < 0 )
		s->changed.wait( lk, done );
	else if( !s->changed.wait_for( lk, std::chrono::duration<double>( timeout_s ), done ) )
		return fail( SPK_ERR_TIMEOUT, "wait timed out" );
	return SPK_OK;
}

int spk_server_get_stats( spk_server * s, spk_server_stats * out )
{
	if( !s || !out ) return fail( SPK_ERR_INVALID, "null argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	std::memset( out, 0, sizeof *out );
	for( auto const & kv : s->jobs )
		switch( kv.second->state )
		{
		case SPK_JOB_QUEUED: out->queued++; break;
		case SPK_JOB_RUNNING: out->running++; break;
		case SPK_JOB_DONE: out->done++; break;
		case SPK_JOB_FAILED: out->failed++; break;
		case SPK_JOB_CANCELLED: out->cancelled++; break;
		case SPK_JOB_TIMEOUT: out->timed_out++; break;
		case SPK_JOB_REFUSED: out->refused++; break;
		}
	out->bytes_in_use = s->in_use;
	out->peak_bytes = s->peak;
	out->budget_bytes = s->budget;
	out->ticks = s->ticks;
	out->build_seconds = s->build_s;
	out->tick_seconds = s->tick_s;
	return SPK_OK;
}

int spk_server_inject_alloc_failures( spk_server * s, int count )
{
	if( !s || count < 0 ) return fail( SPK_ERR_INVALID, "bad argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	s->inject = count;
	return SPK_OK;
}

int spk_server_inject_device_error( spk_server * s, uint64_t id )
{
	if( !s ) return fail( SPK_ERR_INVALID, "bad argument" );
	std::lock_guard<std::mutex> lk( s->mu );
	auto it = s->jobs.find( id );
	if( it == s->jobs.end() || it->second->final() ) return fail( SPK_ERR_INVALID, "no such unfinished job" );
	it->second->raise = true;
	return SPK_OK;
}

int spk_server_destroy( spk_server * s )
{
	if( !s ) return SPK_OK;
	{
		std::lock_guard<std::mutex> lk( s->mu );
		s->stop = true;
		s->wake.notify_all();
		s->tick_wake.notify_all();
	}
	for( auto & b : s->builders )
		if( b.joinable() ) b.join();
	if( s->ticker.joinable() ) s->ticker.join();
	for( auto * j : s->ready )
		spk_net_destroy( j->net );
	for( auto * j : s->running_t )
	{
		spk_batch_remove( s->batch, j->net );
		spk_net_destroy( j->net );
		j->net = nullptr;
	}
	spk_batch_destroy( s->batch );
	int const device = s->device;
	delete s;
	spk_trim_pool( device );
	return SPK_OK;
}
}
