// Host orchestrator of one simulated net (the role of spice::cuda::snn,
// spice/cuda/snn.d.cpp) and the C ABI declared in include/spice_b200.h.
//
// One net = one CUDA stream. Steps requested without output are queued and launched in
// windows of up to `delay` steps (one kernel launch advances every tile by the whole
// window); spk_net_run replays a captured CUDA graph of many windows.
#include "kernels.cuh"
#include "flat.cuh"
#include "models.cuh"
#include "ordered.cuh"
#include "plastic.cuh"
#include "slots.cuh"

#include <spice/util/layout.h>
#include <spice_b200.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_err;

struct spk_error : std::runtime_error
{
	int code;
	spk_error( int c, std::string const & m )
	    : std::runtime_error( m )
	    , code( c )
	{
	}
};

void cuda_check( cudaError_t e, char const * what )
{
	if( e == cudaSuccess ) return;
	if( e == cudaErrorMemoryAllocation )
	{
		cudaGetLastError();
		throw spk_error( SPK_ERR_NOMEM, std::string( what ) + ": " + cudaGetErrorString( e ) );
	}
	throw spk_error( SPK_ERR_CUDA, std::string( what ) + ": " + cudaGetErrorString( e ) );
}
#define CK( x ) cuda_check( ( x ), #x )

void require( bool ok, char const * msg )
{
	if( !ok ) throw spk_error( SPK_ERR_INVALID, msg );
}

template <typename F>
int guarded( F && f )
{
	try
	{
		f();
		return SPK_OK;
	}
	catch( spk_error const & e )
	{
		g_err = e.what();
		return e.code;
	}
	catch( std::bad_alloc const & )
	{
		g_err = "host allocation failed";
		return SPK_ERR_NOMEM;
	}
	catch( std::exception const & e )
	{
		g_err = e.what();
		return SPK_ERR_INVALID;
	}
}

// Where a buffer's memory comes from: cudaMalloc (pool null), or a stream-ordered pool on
// `stream`. cudaMalloc and cudaFree synchronise the whole device; the pool synchronises
// nothing beyond the stream, so a net built or freed beside a running batch does not
// wait for the batch's launches.
struct dmem
{
	cudaMemPool_t pool = nullptr;
	cudaStream_t stream = nullptr;
};

// device allocation owned by the net
struct dbuf
{
	void * p = nullptr;
	size_t bytes = 0;
	dmem src{};
	dbuf() = default;
	dbuf( dbuf const & ) = delete;
	dbuf & operator=( dbuf const & ) = delete;
	~dbuf() { reset(); }
	void reset()
	{
		if( p )
		{
			if( src.pool )
				cudaFreeAsync( p, src.stream );
			else
				cudaFree( p );
		}
		p = nullptr;
		bytes = 0;
		src = {};
	}
	void alloc( size_t b, dmem m = {} )
	{
		reset();
		if( b == 0 ) return;
		if( m.pool )
			CK( cudaMallocFromPoolAsync( &p, b, m.pool, m.stream ) );
		else
			CK( cudaMalloc( &p, b ) );
		bytes = b;
		src = m;
	}
	void swap( dbuf & o )
	{
		std::swap( p, o.p );
		std::swap( bytes, o.bytes );
		std::swap( src, o.src );
	}
	template <typename T>
	T * as() const
	{
		return static_cast<T *>( p );
	}
};

// 16-byte pinned host slots for the nets' small device-to-host reads, carved from slabs
// allocated once: a page-locked allocation synchronises the whole device, which a net
// built beside a running batch should not do
class pinned_slots
{
public:
	static unsigned * get()
	{
		std::lock_guard<std::mutex> lk( mu() );
		auto & f = free_list();
		if( f.empty() )
		{
			void * slab = nullptr;
			CK( cudaMallocHost( &slab, SLAB ) );
			for( size_t o = 0; o < SLAB; o += 16 ) f.push_back( reinterpret_cast<unsigned *>( static_cast<char *>( slab ) + o ) );
		}
		unsigned * q = f.back();
		f.pop_back();
		return q;
	}
	static void put( unsigned * q )
	{
		if( !q ) return;
		std::lock_guard<std::mutex> lk( mu() );
		free_list().push_back( q );
	}

private:
	static constexpr size_t SLAB = 64 * 1024;
	static std::mutex & mu()
	{
		static std::mutex m;
		return m;
	}
	static std::vector<unsigned *> & free_list()
	{
		static std::vector<unsigned *> f;
		return f;
	}
};

// Scratch device memory ordered on a stream, from a per-device pool that keeps its memory:
// unlike cudaFree, releasing it does not wait for the whole device, so a net built beside
// a running batch does not stall on the batch's launches.
cudaMemPool_t scratch_pool( int device )
{
	static std::mutex m;
	static std::vector<cudaMemPool_t> pools;
	std::lock_guard<std::mutex> lk( m );
	if( (int)pools.size() <= device ) pools.resize( device + 1, nullptr );
	if( !pools[device] )
	{
		cudaMemPoolProps props{};
		props.allocType = cudaMemAllocationTypePinned;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id = device;
		CK( cudaMemPoolCreate( &pools[device], &props ) );
		unsigned long long keep = ~0ull;
		CK( cudaMemPoolSetAttribute( pools[device], cudaMemPoolAttrReleaseThreshold, &keep ) );
	}
	return pools[device];
}
struct sbuf
{
	void * p = nullptr;
	cudaStream_t s = nullptr;
	sbuf( size_t b, cudaStream_t st, int device )
	    : s( st )
	{
		if( b ) CK( cudaMallocFromPoolAsync( &p, b, scratch_pool( device ), s ) );
	}
	sbuf( sbuf const & ) = delete;
	sbuf & operator=( sbuf const & ) = delete;
	~sbuf()
	{
		if( p ) cudaFreeAsync( p, s );
	}
	template <typename T>
	T * as() const
	{
		return static_cast<T *>( p );
	}
};

// A kernel's dynamic shared-memory limit on `device` (the current device), set once: the
// value depends on the kernel and the device only, so nets configured later (beside
// running launches of the same kernel) make no further driver call for it.
void set_smem_limit( void const * kernel, int device, int bytes )
{
	static std::mutex m;
	static std::map<std::pair<void const *, int>, int> done;
	std::lock_guard<std::mutex> lk( m );
	auto it = done.find( { kernel, device } );
	if( it != done.end() && it->second == bytes ) return;
	CK( cudaFuncSetAttribute( kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes ) );
	done[{ kernel, device }] = bytes;
}

// restores the caller's current device on scope exit
struct device_guard
{
	int prev = -1;
	explicit device_guard( int dev )
	{
		CK( cudaGetDevice( &prev ) );
		if( prev != dev ) CK( cudaSetDevice( dev ) );
	}
	~device_guard()
	{
		if( prev >= 0 ) cudaSetDevice( prev );
	}
};

// Idle streams of the serving loop's nets kept for reuse, per device (all of the greatest
// priority). Creating a stream beside running work took milliseconds in the serving loop,
// so the stream of a destroyed net (its work synchronised, its buffers' releases issued
// on it) serves the next such net of the device; later work on it is ordered after those
// releases. Nets outside the server do not use it: measured alone, their destruction
// took twice as long with recycled streams.
class stream_recycler
{
public:
	// a stream of the current device, `device`
	static cudaStream_t take( int device )
	{
		{
			std::lock_guard<std::mutex> lk( mu() );
			auto & v = idle()[device];
			if( !v.empty() )
			{
				cudaStream_t const s = v.back();
				v.pop_back();
				return s;
			}
		}
		int least = 0, greatest = 0;
		CK( cudaDeviceGetStreamPriorityRange( &least, &greatest ) );
		cudaStream_t s = nullptr;
		CK( cudaStreamCreateWithPriority( &s, cudaStreamNonBlocking, greatest ) );
		return s;
	}
	static void give( int device, cudaStream_t s )
	{
		std::lock_guard<std::mutex> lk( mu() );
		auto & v = idle()[device];
		if( v.size() < KEEP )
			v.push_back( s );
		else
			cudaStreamDestroy( s );
	}

private:
	static constexpr size_t KEEP = 256;
	static std::mutex & mu()
	{
		static std::mutex m;
		return m;
	}
	static std::map<int, std::vector<cudaStream_t>> & idle()
	{
		static std::map<int, std::vector<cudaStream_t>> m;
		return m;
	}
};

spk::model_traits describe( int model )
{
	spk::model_traits t{};
	if( !spk::with_model( model, [&]( auto tag ) { t = spk::traits_of<typename decltype( tag )::type>(); } ) )
		throw spk_error( SPK_ERR_INVALID, "invalid model" );
	return t;
}

bool plastic_of( int model ) { return describe( model ).plastic; }
int classes_of( int model ) { return describe( model ).classes; }
int neuron_attrs_of( int model ) { return describe( model ).neuron_attrs; }

// body( model_tag<Model> ) for the net's model (a valid id: checked at creation)
template <typename F>
void dispatch( int model, F && body )
{
	if( !spk::with_model( model, std::forward<F>( body ) ) ) throw spk_error( SPK_ERR_INVALID, "invalid model" );
}

spice::util::layout to_layout( spk_layout_desc const * d )
{
	require( d != nullptr, "layout descriptor is null" );
	require( d->npops > 0 && d->pops, "layout must contain at least 1 (non-empty) population" );
	require( d->nconn >= 0 && ( d->nconn == 0 || ( d->conn_src && d->conn_dst && d->conn_p ) ), "bad connection arrays" );
	std::vector<size_t> pops( d->pops, d->pops + d->npops );
	std::vector<std::tuple<size_t, size_t, float>> cs;
	for( int i = 0; i < d->nconn; i++ )
	{
		require( d->conn_src[i] >= 0 && d->conn_dst[i] >= 0, "invalid index in connections matrix" );
		cs.emplace_back( (size_t)d->conn_src[i], (size_t)d->conn_dst[i], d->conn_p[i] );
	}
	return spice::util::layout( pops, cs );
}

unsigned long long bernoulli_threshold( float p )
{
	double const t = std::floor( (double)p * 4294967296.0 );
	return t >= 4294967296.0 ? 4294967296ull : (unsigned long long)t;
}

struct tile_cfg
{
	int threads, npt, tile, ntiles;
};

// Tiles of threads * npt destination neurons, one CTA each. Every tile scans every
// arrival of a step, so fewer, larger tiles do less redundant work: prefer the fewest
// waves of CTAs over the SMs, then the best fill of the last wave, then larger tiles.
// Small nets use 128-neuron tiles.
tile_cfg choose_tiles( long long n, int sms, int max_tile, int max_npt )
{
	tile_cfg best{ 128, 1, 128, (int)( ( n + 127 ) / 128 ) };
	if( n <= 128LL * sms ) return best;
	long long best_waves = LLONG_MAX;
	double best_eff = -1;
	for( int npt : { 4, 2, 1 } )
		for( int threads = 64; npt <= max_npt && threads <= 512; threads += 32 )
		{
			long long const T = (long long)threads * npt;
			if( T > max_tile ) continue;
			long long const ntiles = ( n + T - 1 ) / T;
			long long const waves = ( ntiles + sms - 1 ) / sms;
			double const eff = (double)n / ( (double)waves * sms * T );
			if( waves < best_waves || ( waves == best_waves && eff > best_eff + 1e-6 ) ||
			    ( waves == best_waves && eff > best_eff - 1e-6 && T > best.tile ) )
			{
				best_waves = waves;
				best_eff = eff;
				best = { threads, npt, (int)T, (int)ntiles };
			}
		}
	return best;
}

// Tiles of a plastic net, one neuron per thread. Every tile scans every arrival of a step,
// so a net whose tiles of up to 512 neurons fit one per SM keeps those (one CTA per SM); a
// larger net takes tiles of up to PL_THREADS neurons for PL_CTAS_PER_SM CTAs per SM, all
// resident at once, instead of a second wave of CTAs. At Brunel+ 5e8 (100,000 neurons):
// 285 tiles of 352, 0.52-0.54 wall/bio against 0.64 for the same tiles one CTA per SM
// (two waves).
tile_cfg plastic_tiles( long long n, int sms )
{
	tile_cfg const one = choose_tiles( n, sms, 512, 1 );
	if( one.ntiles <= sms ) return one;
	return choose_tiles( n, spk::PL_CTAS_PER_SM * sms, spk::PL_THREADS, 1 );
}
} // namespace

namespace
{
void summaries_from_ring( spk_net & net );
}

// A net's build choices: spk_net_options with every automatic field resolved (the
// environment's test overrides applied to automatic fields only).
struct build_opts
{
	int tile_target = 0;   // 0: one tile per SM
	bool direct = false;   // per-step kernels instead of the window kernels
	bool kernel_auto = true; // the kernel is the automatic choice (no field value, no test override)
	bool ordered = false;  // the generic window_ordered kernel for any non-plastic model
	bool pack16 = false;   // 16-bit slice indices even where 10-bit ones fit
	bool uniform = false;  // equal tiles instead of cost-balanced ones
	bool windowed = false; // no persistent launch
	bool flat_sync = false; // window_flat without its step pipeline
	int slots = 0;         // 0: variable slices; 1: fixed slots where they fit; 2, 4, 8: exactly
	                       // these slots (a restored slotted net)
};

build_opts resolve_opts( spk_net_options const * o )
{
	spk_net_options d;
	spk_net_options_init( &d );
	if( o ) d = *o;
	require( d.tile_target >= 0, "tile target must be >= 0" );
	auto env_is = []( char const * name, char const * value ) {
		char const * e = getenv( name );
		return e && !strcmp( e, value );
	};
	auto pick = [&]( int field, char const * name, char const * on, char const * off, bool dflt ) {
		if( field >= 0 ) return field != 0;
		if( env_is( name, on ) ) return true;
		if( env_is( name, off ) ) return false;
		return dflt;
	};
	require( d.slice_bits == -1 || d.slice_bits == 10 || d.slice_bits == 16, "slice_bits must be 10 or 16" );
	build_opts r;
	r.tile_target = d.tile_target;
	require( d.kernel >= -1 && d.kernel <= 2, "kernel must be 0 (window), 1 (direct) or 2 (ordered)" );
	char const * ke = getenv( "SPK_KERNEL" );
	int const kernel = d.kernel >= 0 ? d.kernel : !ke ? 0 : !strcmp( ke, "direct" ) ? 1 : !strcmp( ke, "ordered" ) ? 2 : 0;
	r.direct = kernel == 1;
	r.kernel_auto = d.kernel < 0 && !ke;
	r.ordered = kernel == 2;
	r.pack16 = d.slice_bits >= 0 ? d.slice_bits == 16 : env_is( "SPK_PACK", "16" );
	r.uniform = pick( d.tiling, "SPK_TILES", "uniform", "balanced", false );
	r.windowed = !pick( d.persistent, "SPK_PERSIST", "1", "0", true );
	r.flat_sync = !pick( d.pipelined, "SPK_FLAT_SYNC", "0", "1", true );
	r.slots = pick( d.slots, "SPK_SLOTS", "1", "0", false ) ? 1 : 0;
	return r;
}

struct spk_net
{
	// owns `stream` (destroyed, or handed back to the device's stream_recycler if it came
	// from there); the first member, so destroyed last: buffers from the pool are released
	// on the stream when the members after it are destroyed
	struct stream_owner
	{
		int device = 0;
		bool recycle = false;
		cudaStream_t s = nullptr;
		~stream_owner()
		{
			if( !s ) return;
			if( recycle )
				stream_recycler::give( device, s );
			else
				cudaStreamDestroy( s );
		}
	} owner;
	int model = 0;
	int device = 0;
	int sms = 148;
	build_opts opts; // build choices (resolved spk_net_options)
	cudaStream_t stream = nullptr;
	cudaMemPool_t pool = nullptr; // null: cudaMalloc; else the net's buffers come from this pool on `stream`
	long long n = 0, width = 0;
	int delay = 1;
	float dt = 0;
	unsigned long long seed = 0;
	tile_cfg tc{};
	std::vector<spk::conn_dev> conns;

	dbuf edges, pivots, tile_first, ring_ids, ring_cnt, clock, dt_ring, err, conns_dev;
	std::vector<int> tile_first_host; // [ntiles + 1]
	dbuf attr[spk::MAX_ATTRS];
	dbuf syn[spk::MAX_ATTRS]; // static synapse attributes (window_ordered models), [n x width] each
	bool ordered = false;     // window_ordered: every arrival through the model's receive(), in order
	dbuf gather_ids, gather_cnt, cursor, gather_done, rec_ids, rec_cnt;
	spk::plastic_state plast; // plastic models only

	unsigned long long steps = 0;   // steps requested so far
	unsigned long long launched = 0; // steps launched
	unsigned long long kernel_launches = 0; // simulation kernel launches (graph replays counted per window)
	int ring_slots = 0;                      // steps the spike ring holds (2 delay; more for recording runs)
	unsigned * host_count = nullptr; // pinned (a pinned_slots slot)

	cudaGraphExec_t graph = nullptr;
	int graph_windows = 0, graph_len = 0;
	// window kernel of non-plastic models: window_flat (staged arrival table, work-balanced
	// tiles, neuron state in shared memory) where it applies, else window_counts
	bool flat = false;
	int flat_tmax = 0;   // the largest tile of the flat tiling
	int flat_smem = 0;   // dynamic shared memory of a window_flat launch
	dbuf slices, slice_rec; // tile-major 16-bit slices, [n][ntiles] records
	dbuf tile_inputs;       // [ntiles] tiles with incoming synapses
	int flat_sync = 0;      // window_flat without its step pipeline (opts.flat_sync)
	int producers = spk::FLAT_PRODUCERS; // window_flat's producer warps (spk_net_set_producer_warps)
	int pack = 8;           // slice indices per 16-byte vector: 8 (16-bit) or 12 (10-bit)
	dbuf done_step;         // [ntiles] last step each tile has published (window_flat)
	// window_slots (10-bit nets whose slices fit fixed slots, section on slots in slots.cuh):
	// slot_vecs > 0 selects it over window_flat; the slots, the tiles' indices among the
	// tiles with inputs and the spike-summary ring
	int slot_vecs = 0, tin = 0;
	int slot_smem = 0; // dynamic shared memory of a window_slots launch
	dbuf slot_data, tile_in, summ;
	bool persistent = false; // run() as one cooperative window_flat launch (delay >= 6)
	// failure-detection tests (SPK_TEST_WAIT_LIMIT, SPK_TEST_WITHHOLD_TILE at creation): a
	// shorter bounded wait, and a tile that never publishes its steps so that the waits of
	// the tiles reading it run out and the launch ends with ERR_TIMEOUT in the error word
	int wait_limit = spk::WAIT_LIMIT;
	int withhold_tile = -1;
	std::vector<double> seg_start, seg_cost; // expected work per neuron stretch (tiling)
	spk_batch * batch = nullptr;             // the batch holding this net, if any

	~spk_net()
	{
		if( graph ) cudaGraphExecDestroy( graph );
		pinned_slots::put( host_count );
	}

	dmem mem() const { return { pool, stream }; }

	spk::net_params params() const
	{
		spk::net_params p{};
		p.n = (int)n;
		p.width = (int)width;
		p.delay = delay;
		p.tile = tc.tile;
		p.ntiles = tc.ntiles;
		p.ring = ring_slots;
		p.seed = seed;
		p.edges = edges.as<int const>();
		p.pivots = pivots.as<unsigned const>();
		p.tile_first = tile_first.as<int const>();
		for( int i = 0; i < spk::MAX_ATTRS; i++ ) p.attr[i] = attr[i].p;
		for( int i = 0; i < spk::MAX_ATTRS; i++ ) p.syn_attr[i] = syn[i].p;
		p.ring_ids = ring_ids.as<int>();
		p.ring_cnt = ring_cnt.as<unsigned>();
		p.clock = clock.as<spk::clock_state>();
		p.dt_ring = dt_ring.as<float>();
		p.err = err.as<int>();
		p.slices = slices.as<uint4 const>();
		p.slice_rec = slice_rec.as<uint2 const>();
		p.tile_inputs = tile_inputs.as<int const>();
		p.flat_sync = flat_sync;
		p.producers = producers;
		p.pack = pack;
		p.done_step = done_step.as<long long>();
		p.wait_limit = wait_limit;
		p.withhold_tile = withhold_tile;
		p.slots = slot_data.as<uint4 const>();
		p.tile_in = tile_in.as<int const>();
		p.tin = tin;
		p.slot_vecs = slot_vecs;
		p.summ = summ.as<int>();
		return p;
	}

	size_t device_bytes() const
	{
		size_t b = edges.bytes + pivots.bytes + tile_first.bytes + ring_ids.bytes + ring_cnt.bytes + clock.bytes + dt_ring.bytes + err.bytes +
		           conns_dev.bytes + gather_ids.bytes + gather_cnt.bytes + cursor.bytes + gather_done.bytes + rec_ids.bytes +
		           rec_cnt.bytes + plast.bytes() + slices.bytes + slice_rec.bytes + tile_inputs.bytes + done_step.bytes +
		           slot_data.bytes + tile_in.bytes + summ.bytes;
		for( auto const & a : attr ) b += a.bytes;
		for( auto const & a : syn ) b += a.bytes;
		return b;
	}

	int classes() const { return classes_of( model ); }
	int neuron_attrs() const { return neuron_attrs_of( model ); }

	int window_smem() const
	{
		if( flat ) return slot_vecs ? slot_smem : flat_smem;
		int const classes = this->classes();
		size_t const head = ( (size_t)classes * tc.tile + tc.ntiles + 1 ) * 4;
		size_t b = ( ( head + 15 ) & ~(size_t)15 ) + (size_t)spk::SPIKE_BATCH * 16;
		if( plastic_of( model ) ) b = spk::plastic_window_smem( tc.tile, tc.ntiles, tc.threads );
		if( ordered ) b = spk::ordered_window_smem( tc.tile, tc.ntiles );
		return (int)b;
	}

	// every kernel a launch can use, with its shared-memory size set (once, outside any
	// stream capture)
	template <typename Model, typename F>
	void with_window_kernel( F && f )
	{
		if constexpr( Model::synapse::has_stdp )
		{
			// one neuron per thread (plastic_tiles); two CTAs per SM where the tiles need it
			if( plastic_two_per_sm() )
				f( spk::window_plastic<Model, 1, spk::PL_CTAS_PER_SM> );
			else
				f( spk::window_plastic<Model, 1, 1> );
		}
		else
		{
			if( ordered )
				switch( tc.npt )
				{
				case 2: f( spk::window_ordered<Model, 2> ); break;
				default: f( spk::window_ordered<Model, 1> ); break;
				}
			else if constexpr( spk::is_flat_model<Model> )
				switch( tc.npt )
				{
				case 4: f( spk::window_counts<Model, 4> ); break;
				case 2: f( spk::window_counts<Model, 2> ); break;
				default: f( spk::window_counts<Model, 1> ); break;
				}
		}
	}

	template <typename Model>
	void configure_model()
	{
		int const smem = window_smem();
		if constexpr( spk::is_flat_model<Model> )
			if( flat )
			{
				// all the shared memory a CTA can have: what the fixed parts leave over
				// becomes slice buffers
				int optin = 0;
				CK( cudaDeviceGetAttribute( &optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device ) );
				cudaFuncAttributes fa{};
				CK( cudaFuncGetAttributes( &fa, spk::window_flat<Model> ) );
				flat_smem = optin - (int)fa.sharedSizeBytes;
				require( (size_t)flat_smem >= spk::flat_smem_bytes( classes(), neuron_attrs(), flat_tmax ), "shared memory too small for the tiling" );
				cudaFuncAttributes fb{};
				CK( cudaFuncGetAttributes( &fb, spk::window_flat_batch<Model> ) );
				require( (int)fb.sharedSizeBytes <= (int)fa.sharedSizeBytes + (int)sizeof( spk::net_params ) + 256, "batched kernel shared memory" );
				flat_smem = std::min( flat_smem, optin - (int)fb.sharedSizeBytes );
				set_smem_limit( (void const *)spk::window_flat<Model>, device, flat_smem );
				set_smem_limit( (void const *)spk::window_flat_batch<Model>, device, flat_smem );
				cudaFuncAttributes fs{}, fsb{};
				CK( cudaFuncGetAttributes( &fs, spk::window_slots<Model> ) );
				CK( cudaFuncGetAttributes( &fsb, spk::window_slots_batch<Model> ) );
				slot_smem = optin - (int)std::max( fs.sharedSizeBytes, fsb.sharedSizeBytes );
				set_smem_limit( (void const *)spk::window_slots<Model>, device, slot_smem );
				set_smem_limit( (void const *)spk::window_slots_batch<Model>, device, slot_smem );
				// one launch for a whole run: every tile's CTA resident at once (cooperative
				// launch), and the step pipeline never waits on a step not yet simulated
				int coop = 0, per_sm = 0;
				CK( cudaDeviceGetAttribute( &coop, cudaDevAttrCooperativeLaunch, device ) );
				if( slot_vecs )
					CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, spk::window_slots<Model>, tc.threads, slot_smem ) );
				else
					CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, spk::window_flat<Model>, tc.threads, flat_smem ) );
				persistent = coop && (long long)per_sm * sms >= tc.ntiles && !opts.windowed;
				return;
			}
		// the limit is per kernel, shared by every net: set it to all a CTA can have, so a
		// net configured later with smaller needs does not lower it under an earlier net's
		int optin = 0;
		CK( cudaDeviceGetAttribute( &optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device ) );
		auto full_limit = [&]( void const * kernel ) {
			cudaFuncAttributes fa{};
			CK( cudaFuncGetAttributes( &fa, kernel ) );
			int const limit = optin - (int)fa.sharedSizeBytes;
			set_smem_limit( kernel, device, limit );
			return limit;
		};
		with_window_kernel<Model>( [&]( auto kernel ) { require( smem <= full_limit( (void const *)kernel ), "shared memory too small for the tiling" ); } );
		// a batch's shared launches of plastic nets (either form)
		if constexpr( spk::is_plastic_model<Model> )
		{
			int const one = full_limit( (void const *)spk::window_plastic_batch<Model, 1> );
			int const two = full_limit( (void const *)spk::window_plastic_batch<Model, spk::PL_CTAS_PER_SM> );
			require( smem <= std::min( one, two ), "shared memory too small for the tiling" );
		}
	}

	void configure()
	{
		dispatch( model, [&]( auto tag ) { configure_model<typename decltype( tag )::type>(); } );
	}

	template <typename Model>
	void launch_window_model( int L )
	{
		auto const p = params();
		int const smem = window_smem();
		if constexpr( Model::synapse::has_stdp )
		{
			auto const q = plast.params();
			with_window_kernel<Model>( [&]( auto kernel ) { kernel<<<tc.ntiles, tc.threads, smem, stream>>>( p, q, L, dt ); } );
		}
		else if( flat )
		{
			if constexpr( spk::is_flat_model<Model> )
			{
				if( slot_vecs )
					spk::window_slots<Model><<<tc.ntiles, tc.threads, smem, stream>>>( p, L, dt, smem );
				else
					spk::window_flat<Model><<<tc.ntiles, tc.threads, smem, stream>>>( p, L, dt, smem );
			}
		}
		else
			with_window_kernel<Model>( [&]( auto kernel ) { kernel<<<tc.ntiles, tc.threads, smem, stream>>>( p, L, dt ); } );
		CK( cudaGetLastError() );
	}

	void launch_window( int L )
	{
		dispatch( model, [&]( auto tag ) { launch_window_model<typename decltype( tag )::type>( L ); } );
	}

	int max_window() const { return std::min( delay, spk::MAX_WINDOW ); }

	// window_plastic's two-CTAs-per-SM form: more tiles than SMs, each of at most PL_THREADS
	bool plastic_two_per_sm() const { return tc.ntiles > sms && tc.threads <= spk::PL_THREADS; }

	// launch every queued step
	void flush()
	{
		while( launched < steps )
		{
			int const L = (int)std::min<unsigned long long>( steps - launched, (unsigned long long)max_window() );
			launch_window( L );
			launched += L;
			kernel_launches++;
		}
	}

	void check_device_error()
	{
		int e = 0;
		CK( cudaMemcpyAsync( &e, err.p, sizeof( int ), cudaMemcpyDeviceToHost, stream ) );
		CK( cudaStreamSynchronize( stream ) );
		if( e ) throw spk_error( SPK_ERR_DEVICE, "device error flag " + std::to_string( e ) );
	}

	void sync()
	{
		flush();
		check_device_error();
	}

	// dense ascending spikes of the `count` steps just launched -> ids (device), counts
	void gather( int count, int * ids, unsigned * counts, unsigned long long cap, long long rec_base )
	{
		spk::raster_totals<<<( count + 7 ) / 8, 256, 0, stream>>>(
		    ring_cnt.as<unsigned>(), tc.ntiles, ring_slots, clock.as<spk::clock_state>(), count, counts + rec_base );
		CK( cudaGetLastError() );
		spk::gather_raster<<<count, 256, 0, stream>>>(
		    ring_ids.as<int>(),
		    ring_cnt.as<unsigned>(),
		    (int)n,
		    tile_first.as<int>(),
		    tc.ntiles,
		    ring_slots,
		    clock.as<spk::clock_state>(),
		    count,
		    counts + rec_base,
		    cursor.as<unsigned long long>(),
		    gather_done.as<unsigned>(),
		    ids,
		    cap,
		    err.as<int>() );
		CK( cudaGetLastError() );
	}

	// Enlarge the spike ring to `slots` steps (window_flat nets, all steps launched): the
	// last ring_slots steps' spikes move to their slots of the larger ring, so a
	// persistent run of up to slots - 2 delay steps leaves every step it simulated in
	// the ring for one gather at the end.
	void grow_ring( int slots )
	{
		if( slots <= ring_slots ) return;
		require( !plastic_of( model ) && launched == steps, "ring growth of a non-plastic net between runs" );
		dbuf ids, cnt;
		ids.alloc( (size_t)slots * n * 4, mem() );
		cnt.alloc( (size_t)slots * tc.ntiles * 4, mem() );
		CK( cudaMemsetAsync( cnt.p, 0, cnt.bytes, stream ) );
		CK( cudaMemsetAsync( ids.p, 0, ids.bytes, stream ) );
		long long const t = (long long)launched;
		for( long long st = std::max( 0LL, t - ring_slots ); st < t; st++ )
		{
			long long const from = st % ring_slots, to = st % slots;
			CK( cudaMemcpyAsync( ids.as<int>() + to * n, ring_ids.as<int>() + from * n, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream ) );
			CK( cudaMemcpyAsync( cnt.as<unsigned>() + to * tc.ntiles, ring_cnt.as<unsigned>() + from * tc.ntiles, (size_t)tc.ntiles * 4,
			                     cudaMemcpyDeviceToDevice, stream ) );
		}
		CK( cudaStreamSynchronize( stream ) );
		ring_ids.swap( ids );
		ring_cnt.swap( cnt );
		ring_slots = slots;
		if( slot_vecs )
		{
			summaries_from_ring( *this );
			CK( cudaStreamSynchronize( stream ) );
		}
		if( graph ) cudaGraphExecDestroy( graph ); // captured the old ring
		graph = nullptr;
	}

	void build_graph_exec( int windows, int len )
	{
		if( graph && graph_windows == windows && graph_len == len ) return;
		if( graph ) cudaGraphExecDestroy( graph );
		graph = nullptr;
		cudaGraph_t g;
		CK( cudaStreamBeginCapture( stream, cudaStreamCaptureModeThreadLocal ) );
		for( int w = 0; w < windows; w++ ) launch_window( len );
		CK( cudaStreamEndCapture( stream, &g ) );
		cudaError_t const e = cudaGraphInstantiate( &graph, g, 0 );
		cudaGraphDestroy( g );
		CK( e );
		graph_windows = windows;
		graph_len = len;
	}

	// all of a run's steps as cooperative launches of window_flat (section on persistence in
	// flat.cuh)
	template <typename Model>
	void launch_persistent_model( int L )
	{
		if constexpr( spk::is_flat_model<Model> )
		{
			auto p = params();
			// window_flat's step pipeline looks five steps ahead, which needs delay >= 6;
			// shorter delays run every step on the synchronous path (each step waits for the
			// steps it reads). window_slots looks five steps ahead (its nets have delay >= 7).
			if( !slot_vecs && delay < 6 ) p.flat_sync = 1;
			int smem = slot_vecs ? slot_smem : flat_smem;
			float d = dt;
			void * args[] = { &p, &L, &d, &smem };
			void const * kernel = slot_vecs ? (void const *)spk::window_slots<Model> : (void const *)spk::window_flat<Model>;
			CK( cudaLaunchCooperativeKernel( kernel, dim3( tc.ntiles ), dim3( tc.threads ), args, (size_t)smem, stream ) );
		}
	}
	void launch_persistent( int L )
	{
		dispatch( model, [&]( auto tag ) { launch_persistent_model<typename decltype( tag )::type>( L ); } );
	}

	void run( unsigned long long nsteps )
	{
		flush();
		if( persistent )
		{
			while( nsteps > 0 )
			{
				int const L = (int)std::min<unsigned long long>( nsteps, 1u << 30 );
				steps += L;
				launch_persistent( L );
				kernel_launches++;
				launched += L;
				nsteps -= L;
			}
			return;
		}
		int const len = max_window();
		unsigned long long const windows = std::min<unsigned long long>( nsteps / len, 512 );
		if( windows >= 2 )
		{
			build_graph_exec( (int)windows, len );
			unsigned long long const per_graph = windows * len;
			while( nsteps >= per_graph )
			{
				CK( cudaGraphLaunch( graph, stream ) );
				kernel_launches += windows;
				nsteps -= per_graph;
				steps += per_graph;
				launched += per_graph;
			}
		}
		steps += nsteps;
		flush();
	}
};

namespace
{
template <typename Model>
void init_model( spk_net & net )
{
	auto const p = net.params();
	int const blocks = (int)std::min<long long>( 4 * net.sms, ( net.n + 255 ) / 256 );
	spk::init_neurons<Model><<<std::max( 1, blocks ), 256, 0, net.stream>>>( p );
	CK( cudaGetLastError() );
	if constexpr( Model::synapse::has_stdp ) spk::init_plastic<Model>( p, net.plast, net.dt, net.sms, net.stream );
	else if constexpr( Model::synapse::size > 0 )
		if( net.n * net.width > 0 )
		{
			spk::init_synapses<Model><<<4 * net.sms, 256, 0, net.stream>>>( p );
			CK( cudaGetLastError() );
		}
}

void init_state( spk_net & net )
{
	dispatch( net.model, [&]( auto tag ) { init_model<typename decltype( tag )::type>( net ); } );
}

// Work per neuron, piecewise constant: neurons [start, next start) cost `cost` each.
struct cost_segment
{
	long long start;
	double cost;
};

// one neuron update against one synapse of in-degree, for tile balancing. Measured on
// B200 (Brunel, 1e9 synapses): a Poisson source (one counter-RNG draw per step) costs
// about as much per window as 1000 synapses of in-degree of a receiving neuron.
constexpr double UPDATE_COST = 1000.0;

// expected in-degree of every neuron of a layout (constant over stretches of populations)
std::vector<cost_segment> layout_costs( spice::util::layout const & l )
{
	std::vector<long long> cuts{ 0, (long long)l.size() };
	for( auto const & c : l.connections() )
	{
		cuts.push_back( std::get<2>( c ) );
		cuts.push_back( std::get<3>( c ) );
	}
	std::sort( cuts.begin(), cuts.end() );
	cuts.erase( std::unique( cuts.begin(), cuts.end() ), cuts.end() );
	std::vector<cost_segment> segs;
	for( size_t i = 0; i + 1 < cuts.size(); i++ )
	{
		double in = 0;
		for( auto const & c : l.connections() )
			if( std::get<2>( c ) <= cuts[i] && cuts[i] < std::get<3>( c ) ) in += (double)( std::get<1>( c ) - std::get<0>( c ) ) * std::get<4>( c );
		segs.push_back( { cuts[i], UPDATE_COST + in } );
	}
	return segs;
}

// synapses of a net from its cost segments (each neuron's in-degree above the update cost)
double segment_synapses( std::vector<cost_segment> const & segs, long long n )
{
	double syn = 0;
	for( size_t i = 0; i < segs.size(); i++ )
	{
		long long const end = i + 1 < segs.size() ? segs[i + 1].start : n;
		syn += (double)( end - segs[i].start ) * ( segs[i].cost - UPDATE_COST );
	}
	return syn;
}

// The automatic kernel of a net with input classes at delay 1: window_counts (one launch
// per step from a CUDA graph) for nets of up to this many synapses, window_flat above. At
// delay 1 window_flat's persistent launch waits for every tile's spikes each step, about
// 9 us; measured on B200, 1e4-step runs: VA 5,000 and 20,000 neurons 6.3 / 6.7 us per
// step with window_counts against 8.8 / 9.3 us, Brunel 20,000 (2e7 synapses) 10.0 against
// 9.9 us, Brunel 1e8 22.8 against 11.1 us. At delay 3 and above window_flat is as fast or
// faster throughout.
constexpr double PER_STEP_MAX_SYNAPSES = 1e7;

// exact in-degree of every neuron of an imported ELL graph (edges already validated)
std::vector<cost_segment> adjacency_costs( int const * edges, long long n, long long width )
{
	std::vector<int> in( n, 0 );
	for( long long e = 0; e < n * width; e++ )
		if( edges[e] != INT_MAX ) in[edges[e]]++;
	std::vector<cost_segment> segs;
	for( long long i = 0; i < n; i++ )
		if( i == 0 || in[i] != in[i - 1] ) segs.push_back( { i, UPDATE_COST + in[i] } );
	return segs;
}

// Cut [0, n) into contiguous tiles of about equal work, aiming at no more tiles than SMs
// (every tile with inputs scans every arrival of a step). Tiles never mix neurons with
// and without incoming synapses (cost == UPDATE_COST): tiles with inputs hold at most
// tmax_in neurons, tiles without at most tmax_free (they keep only neuron state).
std::vector<int> balanced_tiles( std::vector<cost_segment> const & segs, long long n, int sms, int tmax_in, int tmax_free )
{
	auto seg_end = [&]( size_t i ) { return i + 1 < segs.size() ? segs[i + 1].start : n; };
	auto is_free = [&]( size_t i ) { return segs[i].cost <= UPDATE_COST; };
	double total = 0;
	for( size_t i = 0; i < segs.size(); i++ ) total += ( seg_end( i ) - segs[i].start ) * segs[i].cost;
	auto cut = [&]( double target ) {
		std::vector<int> first{ 0 };
		long long start = 0;
		double acc = 0;
		for( size_t i = 0; i < segs.size(); i++ )
		{
			double const c = std::max( segs[i].cost, 1e-9 );
			long long pos = segs[i].start;
			long long const e = seg_end( i );
			int const tmax = is_free( i ) ? tmax_free : tmax_in;
			if( i > 0 && is_free( i ) != is_free( i - 1 ) && pos > start ) // no mixed tiles
			{
				first.push_back( (int)pos );
				start = pos;
				acc = 0;
			}
			while( pos < e )
			{
				long long const room = tmax - ( pos - start );
				long long fit = (long long)std::floor( ( target - acc ) / c );
				if( pos == start ) fit = std::max( fit, 1LL );
				long long const take = std::min( { e - pos, room, std::max( fit, 0LL ) } );
				if( take <= 0 ) // this tile is full: the next one starts here
				{
					first.push_back( (int)pos );
					start = pos;
					acc = 0;
					continue;
				}
				pos += take;
				acc += take * c;
				if( ( acc >= target * ( 1 - 1e-12 ) || pos - start >= tmax ) && pos < n )
				{
					first.push_back( (int)pos );
					start = pos;
					acc = 0;
				}
			}
		}
		if( first.back() != (int)n ) first.push_back( (int)n );
		return first;
	};
	// small nets: at least 256 neurons' worth of work per tile
	double target = std::max( total / sms, 256.0 * total / std::max<long long>( n, 1 ) );
	std::vector<int> best = cut( target );
	for( int it = 0; it < 400 && (int)best.size() - 1 > sms; it++ )
	{
		target *= 1.01;
		best = cut( target );
	}
	return best;
}

std::vector<int> uniform_tiles( long long n, int tile )
{
	std::vector<int> f;
	for( long long d = 0; d < n; d += tile ) f.push_back( (int)d );
	f.push_back( (int)n );
	return f;
}

void set_tiles( spk_net & net, std::vector<int> const & first )
{
	net.tile_first_host = first;
	net.tc.ntiles = (int)first.size() - 1;
	net.tile_first.alloc( first.size() * 4, net.mem() );
	// on the net's stream (non-blocking: a plain cudaMemcpy from pageable memory may return
	// before its DMA lands, unordered with the net's kernels)
	CK( cudaMemcpyAsync( net.tile_first.p, first.data(), first.size() * 4, cudaMemcpyHostToDevice, net.stream ) );
	CK( cudaStreamSynchronize( net.stream ) );
}

// window_flat's tiling of n neurons into at most about `target` work-balanced tiles (target
// = the SM count for a net alone; fewer for a net that shares the GPU in a batch): the
// tiles' first neurons and the shared-memory span of the largest tile with inputs; false
// if the net does not fit window_flat.
bool plan_flat( int model,
                int device,
                long long n,
                long long width,
                std::vector<cost_segment> const & segs,
                int target,
                build_opts const & o,
                std::vector<int> & first,
                int & span,
                int & pack )
{
	int optin = 0;
	CK( cudaDeviceGetAttribute( &optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device ) );
	int const classes = classes_of( model ), attrs = neuron_attrs_of( model );
	// largest tile whose counters, state, tables and minimal slice ring fit (with room for
	// the kernel's static shared memory), and whose counter indices fit 16 bits
	// a slice holds at most min(tile, row width) targets, and its length must fit 12 bits
	int tmax = width <= spk::FLAT_MAX_SLICE ? spk::FLAT_MAX_TILE_WIDE : spk::FLAT_MAX_TILE;
	while( tmax >= 128 && ( spk::flat_smem_bytes( classes, attrs, tmax ) + 4096 > (size_t)optin || (long long)classes * tmax >= spk::SLICE_PAD ) )
		tmax -= 32;
	// tiles without inputs keep only their neuron state and fired bits
	int const tmax_free = (int)std::max<long long>( tmax, ( ( optin - 4096LL ) * 32 / ( 32LL * 4 * attrs + 8 ) ) / 32 * 32 );
	if( tmax < 128 ) return false;
	bool const uniform = o.uniform;
	auto cut = [&]( int tmax_in ) {
		return uniform ? uniform_tiles( n, std::min( tmax_in, 1024 ) ) : balanced_tiles( segs, n, std::max( 1, target ), tmax_in, tmax_free );
	};
	// the largest tile with inputs sets the shared-memory floor (tiles without inputs need
	// less than it per neuron)
	auto input_span = [&]( std::vector<int> const & f, int tmax_in ) {
		int sp = 0;
		size_t si = 0;
		for( size_t i = 0; i + 1 < f.size(); i++ )
		{
			while( si + 1 < segs.size() && segs[si + 1].start <= f[i] ) si++;
			if( segs[si].cost > UPDATE_COST || f[i + 1] - f[i] <= tmax_in ) sp = std::max( sp, f[i + 1] - f[i] );
		}
		return sp;
	};
	first = cut( tmax );
	if( (int)first.size() >= spk::FLAT_PC ) return false;
	span = input_span( first, tmax );
	// 10-bit slices (twelve indices per vector instead of eight) when every counter index
	// fits below SLICE_PAD10: tiles with inputs capped at (SLICE_PAD10 - 1) / classes
	// neurons, taken if that needs no more tiles (o.pack16 keeps 16-bit slices)
	pack = 8;
	int const cap10 = (int)( ( spk::SLICE_PAD10 - 1 ) / std::max( 1, classes ) );
	if( !o.pack16 && cap10 >= 128 )
	{
		if( (long long)classes * span < (long long)spk::SLICE_PAD10 )
			pack = 12;
		else
		{
			std::vector<int> const f10 = cut( std::min( tmax, cap10 ) );
			int const s10 = input_span( f10, std::min( tmax, cap10 ) );
			if( f10.size() <= first.size() && (long long)classes * s10 < (long long)spk::SLICE_PAD10 )
			{
				first = f10;
				span = s10;
				pack = 12;
			}
		}
	}
	return true;
}

// plan_flat applied to a net: sets net.flat and the tiles
bool flat_tiling( spk_net & net, std::vector<cost_segment> const & segs, int target )
{
	std::vector<int> first;
	int span = 0, pack = 8;
	if( !plan_flat( net.model, net.device, net.n, net.width, segs, target, net.opts, first, span, pack ) ) return false;
	net.flat = true;
	net.pack = pack;
	net.flat_tmax = ( span + 31 ) / 32 * 32;
	net.tc = { spk::FLAT_THREADS, 1, net.flat_tmax, (int)first.size() - 1 };
	set_tiles( net, first );
	return true;
}

// buffers + pivots; edges must be filled before build_pivots is enqueued
void allocate_buffers( spk_net & net );

void allocate( spk_net & net, long long n, long long width, std::vector<cost_segment> const & segs )
{
	require( n > 0 && n <= INT_MAX, "invalid neuron count" );
	require( width >= 0 && width % 32 == 0, "width must be a multiple of 32" );
	require( n * std::max<long long>( width, 1 ) < ( 1LL << 40 ), "graph too large" );
	net.n = n;
	net.width = width;
	int dev_sms = 0;
	CK( cudaDeviceGetAttribute( &dev_sms, cudaDevAttrMultiProcessorCount, net.device ) );
	net.sms = dev_sms;
	spk::model_traits const md = describe( net.model );
	net.ordered = !md.plastic && ( md.ordered || net.opts.ordered );
	net.tc = md.plastic ? plastic_tiles( n, dev_sms )
	         : net.ordered ? choose_tiles( n, dev_sms, spk::ORD_MAX_TILE, 2 )
	                       : choose_tiles( n, dev_sms, 2048, 4 );

	// window kernel and tiling: window_flat with work-balanced tiles (opts.uniform keeps
	// equal tiles, opts.direct selects window_counts)
	net.seg_start.clear();
	net.seg_cost.clear();
	for( auto const & g : segs )
	{
		net.seg_start.push_back( (double)g.start );
		net.seg_cost.push_back( g.cost );
	}
	net.flat = false;
	int const target = net.opts.tile_target;
	bool const per_step = net.opts.kernel_auto && net.delay == 1 && segment_synapses( segs, n ) <= PER_STEP_MAX_SYNAPSES;
	if( !md.plastic && !net.ordered && !net.opts.direct && !per_step ) flat_tiling( net, segs, target > 0 ? target : dev_sms );
	if( !net.flat ) set_tiles( net, uniform_tiles( n, net.tc.tile ) );
	net.ring_slots = 2 * net.delay;
	allocate_buffers( net );
}

// every per-net buffer for the net's size, tiling and ring (edges, pivots, ring, clock,
// neuron state, gather buffers, plastic state), then the kernels' configuration
void allocate_buffers( spk_net & net )
{
	long long const n = net.n, width = net.width;
	spk::model_traits const md = describe( net.model );
	net.edges.alloc( (size_t)( n * width ) * 4, net.mem() );
	net.pivots.alloc( (size_t)n * ( net.tc.ntiles + 1 ) * 4, net.mem() );
	net.ring_ids.alloc( (size_t)net.ring_slots * n * 4, net.mem() );
	net.ring_cnt.alloc( (size_t)net.ring_slots * net.tc.ntiles * 4, net.mem() );
	net.clock.alloc( sizeof( spk::clock_state ), net.mem() );
	net.dt_ring.alloc( spk::DT_RING * 4, net.mem() );
	net.err.alloc( 4, net.mem() );
	for( int i = 0; i < md.neuron_attrs; i++ ) net.attr[i].alloc( (size_t)n * 4, net.mem() );
	net.gather_ids.alloc( (size_t)n * 4, net.mem() );
	net.gather_cnt.alloc( 4, net.mem() );
	net.cursor.alloc( 8, net.mem() );
	net.gather_done.alloc( 4, net.mem() );
	CK( cudaMemsetAsync( net.ring_cnt.p, 0, net.ring_cnt.bytes, net.stream ) );
	// spike ids start as valid neuron ids: a tile that reads a slot before its publication
	// (only after a wait ran out) still indexes inside every table
	CK( cudaMemsetAsync( net.ring_ids.p, 0, net.ring_ids.bytes, net.stream ) );
	CK( cudaMemsetAsync( net.clock.p, 0, net.clock.bytes, net.stream ) );
	CK( cudaMemsetAsync( net.err.p, 0, 4, net.stream ) );
	CK( cudaMemsetAsync( net.cursor.p, 0, 8, net.stream ) );
	CK( cudaMemsetAsync( net.gather_done.p, 0, 4, net.stream ) );
	if( plastic_of( net.model ) ) net.plast.allocate( n, width, net.tc.ntiles, net.delay, net.stream, net.pool );
	else
		for( int i = 0; i < md.synapse_attrs; i++ )
		{
			// zero on padding slots, as the reference's value-initialised synapse vector
			net.syn[i].alloc( (size_t)( n * width ) * 4, net.mem() );
			CK( cudaMemsetAsync( net.syn[i].p, 0, net.syn[i].bytes, net.stream ) );
		}
	if( !net.host_count ) net.host_count = pinned_slots::get();
	net.configure();
}

template <typename Model>
void fill_slices( spk_net & net, sbuf const & bases )
{
	if constexpr( spk::is_flat_model<Model> )
	{
		int const blocks = (int)( ( net.n * 32 + 255 ) / 256 );
		spk::slice_fill<Model><<<blocks, 256, 0, net.stream>>>(
		    (int)net.n, (int)net.width, net.tc.ntiles, net.edges.as<int>(), net.pivots.as<unsigned>(), net.tile_first.as<int>(),
		    bases.as<unsigned long long>(), net.slice_rec.as<uint2>(), net.slices.as<unsigned short>(), net.pack );
		CK( cudaGetLastError() );
	}
}

template <typename Model>
void fill_slots( spk_net & net )
{
	if constexpr( spk::is_flat_model<Model> )
	{
		int const blocks = (int)( ( net.n * 32 + 255 ) / 256 );
		spk::slot_fill<Model><<<blocks, 256, 0, net.stream>>>(
		    (int)net.n, (int)net.width, net.tc.ntiles, net.edges.as<int>(), net.pivots.as<unsigned>(), net.tile_first.as<int>(),
		    net.tile_in.as<int>(), net.tin, net.slot_vecs, net.slot_data.as<uint4>() );
		CK( cudaGetLastError() );
	}
}

// the spike-summary ring of a slotted net, rebuilt from its spike ring (after a restore or
// when the ring grows)
void summaries_from_ring( spk_net & net )
{
	if( !net.slot_vecs ) return;
	net.summ.alloc( (size_t)net.ring_slots * net.tc.ntiles * spk::SUM_W * 4, net.mem() );
	long long const warps = (long long)net.ring_slots * net.tc.ntiles;
	spk::summ_from_ring<<<(int)( ( warps * 32 + 255 ) / 256 ), 256, 0, net.stream>>>(
	    net.ring_ids.as<int>(), net.ring_cnt.as<unsigned>(), (int)net.n, net.tc.ntiles, net.ring_slots, net.tile_first.as<int>(),
	    net.summ.as<int>() );
	CK( cudaGetLastError() );
}

// Fixed slots (window_slots) instead of variable slices, on request only (a checkpoint of
// a slotted net, SPK_SLOTS=1): for 10-bit nets with delay >= 7 whose longest slice fits 8
// vectors and whose step's arrivals fit the shared memory. On the 1e9-synapse Brunel net
// (slots of 8 vectors) a step takes 6.47 us against window_flat's 6.22 us, so the
// variable slices stay the default.
bool plan_slots( spk_net & net )
{
	net.slot_vecs = 0;
	net.tin = 0;
	net.slot_data.reset();
	net.tile_in.reset();
	net.summ.reset();
	int const want = net.opts.slots; // 0: none; 1: where they fit; else exactly this many vectors
	int const nt = net.tc.ntiles;
	require( want <= 1 || net.pack == 12, "checkpoint slots do not fit this device" );
	if( want == 0 || net.pack != 12 || net.delay < 7 || net.width == 0 ) return false;
	std::vector<int> in( nt ), idx( nt, -1 );
	CK( cudaMemcpyAsync( in.data(), net.tile_inputs.p, (size_t)nt * 4, cudaMemcpyDeviceToHost, net.stream ) );
	sbuf mx( 4, net.stream, net.device );
	CK( cudaMemsetAsync( mx.p, 0, 4, net.stream ) );
	spk::slice_max<<<4 * net.sms, 256, 0, net.stream>>>( (int)net.n, nt, net.pivots.as<unsigned>(), mx.as<unsigned>() );
	CK( cudaGetLastError() );
	unsigned longest = 0;
	CK( cudaMemcpyAsync( &longest, mx.p, 4, cudaMemcpyDeviceToHost, net.stream ) );
	CK( cudaStreamSynchronize( net.stream ) );
	int tin = 0;
	for( int j = 0; j < nt; j++ )
		if( in[j] ) idx[j] = tin++;
	int S = 2;
	while( S < 8 && (unsigned)S * 12 < longest ) S *= 2;
	if( tin == 0 || (unsigned)S * 12 < longest ) return false;
	spk::slot_geom const g = spk::slot_layout( net.classes(), net.neuron_attrs(), net.flat_tmax, nt, S, net.slot_smem );
	bool const fits = g.ecap >= spk::SLOT_MIN_ECAP && spk::slot_layout_end( g, S ) <= (size_t)net.slot_smem;
	require( want <= 1 || ( fits && S == want ), "checkpoint slots do not fit this device" );
	if( !fits ) return false;
	net.slot_vecs = S;
	net.tin = tin;
	net.tile_in.alloc( (size_t)nt * 4, net.mem() );
	CK( cudaMemcpyAsync( net.tile_in.p, idx.data(), (size_t)nt * 4, cudaMemcpyHostToDevice, net.stream ) );
	net.slot_data.alloc( (size_t)net.n * tin * S * 16, net.mem() );
	dispatch( net.model, [&]( auto tag ) { fill_slots<typename decltype( tag )::type>( net ); } );
	summaries_from_ring( net );
	CK( cudaStreamSynchronize( net.stream ) ); // idx is freed on return
	return true;
}

// the tile-major slices of window_flat, from the ELL rows and their pivots
void build_slices( spk_net & net )
{
	int const nt = net.tc.ntiles;
	long long const n = net.n;
	net.slice_rec.alloc( (size_t)n * nt * sizeof( uint2 ), net.mem() );
	net.tile_inputs.alloc( (size_t)nt * 4, net.mem() );
	CK( cudaMemsetAsync( net.tile_inputs.p, 0, net.tile_inputs.bytes, net.stream ) );
	sbuf rows( (size_t)n * 4, net.stream, net.device ), bases( (size_t)n * 8, net.stream, net.device );
	std::vector<unsigned> rv( n );
	std::vector<unsigned long long> base( n );
	// vectors per (src, tile), their prefix along each row, and the rows' totals
	int const blocks = (int)( ( n * 32 + 255 ) / 256 );
	spk::slice_vectors<<<4 * net.sms, 256, 0, net.stream>>>( (int)n, nt, net.pivots.as<unsigned>(), net.slice_rec.as<uint2>(), net.pack );
	CK( cudaGetLastError() );
	spk::slice_row_offsets<<<blocks, 256, 0, net.stream>>>( (int)n, nt, net.slice_rec.as<uint2>(), rows.as<unsigned>(), net.tile_inputs.as<int>() );
	CK( cudaGetLastError() );
	CK( cudaMemcpyAsync( rv.data(), rows.p, (size_t)n * 4, cudaMemcpyDeviceToHost, net.stream ) );
	CK( cudaStreamSynchronize( net.stream ) );
	unsigned long long all = 0;
	for( long long s = 0; s < n; s++ )
	{
		base[s] = all;
		all += rv[s];
	}
	require( all < ( 1ULL << 32 ), "graph too large for 32-bit slice records" );
	net.flat_sync = net.opts.flat_sync;
	net.done_step.alloc( (size_t)nt * sizeof( long long ), net.mem() );
	CK( cudaMemsetAsync( net.done_step.p, 0xFF, net.done_step.bytes, net.stream ) ); // -1: nothing published
	if( plan_slots( net ) )
	{
		net.slice_rec.reset();
		net.slices.reset();
		CK( cudaStreamSynchronize( net.stream ) );
		net.configure(); // the persistent launch of window_slots
		return;
	}
	net.slices.alloc( std::max<size_t>( (size_t)all * 16, 16 ), net.mem() );
	CK( cudaMemcpyAsync( bases.p, base.data(), (size_t)n * 8, cudaMemcpyHostToDevice, net.stream ) );
	dispatch( net.model, [&]( auto tag ) { fill_slices<typename decltype( tag )::type>( net, bases ); } );
	CK( cudaStreamSynchronize( net.stream ) ); // rows and bases are freed on return
}

void enqueue_pivots( spk_net & net )
{
	if( net.n == 0 ) return;
	int const blocks = (int)( ( net.n * 32 + 255 ) / 256 );
	if( net.width > 0 )
		spk::build_pivots<<<blocks, 256, 0, net.stream>>>(
		    (int)net.n, (int)net.width, net.tile_first.as<int>(), net.tc.ntiles, net.edges.as<int>(), net.pivots.as<unsigned>() );
	else
		CK( cudaMemsetAsync( net.pivots.p, 0, net.pivots.bytes, net.stream ) );
	CK( cudaGetLastError() );
	if( net.flat ) build_slices( net );
}

// device memory a recording run may give the spike ring (run_record of persistent nets)
constexpr long long RECORD_RING_BYTES = 1LL << 30;

// Re-tile a net that has not been stepped yet for about `target` tiles (batching): tiles,
// pivots, slices and the per-tile buffers are rebuilt from the unchanged edges.
void retile( spk_net & net, int target )
{
	require( net.steps == 0 && net.launched == 0, "a net is re-tiled before its first step" );
	if( !net.flat ) return; // window_counts and window_plastic keep their fixed tiles
	std::vector<cost_segment> segs;
	for( size_t i = 0; i < net.seg_start.size(); i++ ) segs.push_back( { (long long)net.seg_start[i], net.seg_cost[i] } );
	CK( cudaStreamSynchronize( net.stream ) );
	require( flat_tiling( net, segs, target ), "tiling failed" );
	net.pivots.alloc( (size_t)net.n * ( net.tc.ntiles + 1 ) * 4, net.mem() );
	net.ring_cnt.alloc( (size_t)net.ring_slots * net.tc.ntiles * 4, net.mem() );
	CK( cudaMemsetAsync( net.ring_cnt.p, 0, net.ring_cnt.bytes, net.stream ) );
	enqueue_pivots( net );
	if( net.graph ) cudaGraphExecDestroy( net.graph );
	net.graph = nullptr;
	net.configure();
	CK( cudaStreamSynchronize( net.stream ) );
}

void enqueue_generate( cudaStream_t s, spice::util::layout const & l, unsigned long long seed, int * d_edges, dbuf & conns_dev, dmem m = {} )
{
	std::vector<spk::conn_dev> cs;
	for( auto const & c : l.connections() )
		cs.push_back( { std::get<0>( c ), std::get<1>( c ), std::get<2>( c ), std::get<3>( c ), bernoulli_threshold( std::get<4>( c ) ) } );
	long long const n = (long long)l.size(), w = (long long)l.max_degree();
	if( n == 0 || w == 0 ) return;
	conns_dev.alloc( std::max<size_t>( cs.size(), 1 ) * sizeof( spk::conn_dev ), m );
	if( !cs.empty() ) CK( cudaMemcpyAsync( conns_dev.p, cs.data(), cs.size() * sizeof( spk::conn_dev ), cudaMemcpyHostToDevice, s ) );
	int const blocks = (int)( ( n * 32 + 255 ) / 256 );
	spk::generate_ell<<<blocks, 256, 0, s>>>( (int)n, (int)w, (int)cs.size(), conns_dev.as<spk::conn_dev>(), seed, d_edges );
	CK( cudaGetLastError() );
}

// ELL rows as the reference keeps them (spice/util/adj_list.cpp:28-46): every row strictly
// ascending, every target in [0, n), INT_MAX padding only at the end of a row. The
// pivot and slice builders rely on it, so imported graphs are checked on the host first.
void validate_edges( int32_t const * edges, uint64_t n, uint64_t width )
{
	for( uint64_t i = 0; i < n; i++ )
	{
		int prev = -1;
		bool pad = false;
		for( uint64_t j = 0; j < width; j++ )
		{
			int const v = edges[i * width + j];
			if( v == INT_MAX )
			{
				pad = true;
				continue;
			}
			require( !pad, "edges: padding must end a row" );
			require( v > prev && (uint64_t)v < n, "edges: rows must be strictly ascending and in range" );
			prev = v;
		}
	}
}

// Upper estimate of the device memory a net of this layout holds once built (the buffers
// of allocate, build_slices and the plastic state; slices bounded by one 16-byte vector per
// 8 or 12 synapses plus one per non-empty (source, tile) pair, at 5 % above the expected
// synapse count), each buffer rounded up to the allocator's 2 MiB granule.
size_t estimate_bytes( int model, spice::util::layout const & l, int delay, int device, build_opts const & o )
{
	long long const n = (long long)l.size(), w = (long long)l.max_degree();
	double syn = 0;
	for( auto const & c : l.connections() )
		syn += (double)( std::get<1>( c ) - std::get<0>( c ) ) * (double)( std::get<3>( c ) - std::get<2>( c ) ) * std::get<4>( c );
	syn = std::min( syn * 1.05, (double)n * w );
	int sms = 0;
	CK( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, device ) );
	spk::model_traits const md = describe( model );
	int const attrs = md.neuron_attrs;
	bool flat = false;
	long long T = 0;
	int pack = 8;
	if( !md.plastic && ( md.ordered || o.ordered ) )
		T = choose_tiles( n, sms, spk::ORD_MAX_TILE, 2 ).ntiles;
	else if( !md.plastic )
	{
		std::vector<int> first;
		int span = 0;
		std::vector<cost_segment> const segs = layout_costs( l );
		bool const per_step = o.kernel_auto && delay == 1 && segment_synapses( segs, n ) <= PER_STEP_MAX_SYNAPSES;
		if( !o.direct && !per_step && plan_flat( model, device, n, w, segs, o.tile_target > 0 ? o.tile_target : sms, o, first, span, pack ) )
		{
			flat = true;
			T = (long long)first.size() - 1;
		}
		else
			T = choose_tiles( n, sms, 2048, 4 ).ntiles;
	}
	else
		T = plastic_tiles( n, sms ).ntiles;
	std::vector<double> b = { (double)n * w * 4,
	                          (double)n * ( T + 1 ) * 4,
	                          2.0 * delay * n * 4,
	                          2.0 * delay * T * 4,
	                          64,
	                          spk::DT_RING * 4.0,
	                          4,
	                          (double)n * 4,
	                          4,
	                          8,
	                          4,
	                          4096 };
	for( int i = 0; i < attrs; i++ ) b.push_back( (double)n * 4 );
	if( !md.plastic )
		for( int i = 0; i < md.synapse_attrs; i++ ) b.push_back( (double)n * w * 4 );
	if( flat )
	{
		b.push_back( (double)n * T * 8 );
		b.push_back( 16.0 * ( std::ceil( syn / pack ) + std::min( (double)n * T, syn ) ) );
		if( o.slots && pack == 12 && delay >= 7 )
		{
			// fixed slots (on request): at most 8 vectors per (source, tile) pair, built
			// beside the slice records, and the spike-summary ring
			b.push_back( 128.0 * n * T );
			b.push_back( 2.0 * delay * T * spk::SUM_W * 4 );
			b.push_back( (double)T * 4 );
		}
		b.push_back( (double)T * 8 );
		b.push_back( (double)T * 4 );
	}
	if( plastic_of( model ) )
	{
		b.push_back( (double)n * w * 4 );
		for( int i = 0; i < 8; i++ ) b.push_back( (double)n * 4 );
		b.push_back( (double)n * 8 );
		b.push_back( 2.0 * delay * n * 16 );
		b.push_back( 2.0 * delay * n * 16 );
		b.push_back( 2.0 * delay * T * 4 );
		b.push_back( 2.0 * delay * T * 4 );
	}
	double const granule = 2.0 * 1024 * 1024;
	double total = 0;
	for( double x : b ) total += std::ceil( x / granule ) * granule;
	return (size_t)total;
}

// ------------------------------------------------------------------------------------
// checkpoints: everything a net needs to continue bit for bit, in host memory
// ------------------------------------------------------------------------------------
// Layout: ckpt_header, tile_first[ntiles + 1] (int32), then per buffer { u32 id, u64 bytes,
// bytes }. Derived buffers (pivots, slices, slice records) are rebuilt from the edges and
// tiles on restore; the spike ring, clock and (Brunel+) the lazy-STDP state are kept, so
// spikes in flight and pending weight updates survive.
struct ckpt_header
{
	char magic[8];
	uint32_t version;
	int32_t model;
	int64_t n, width;
	int32_t delay;
	float dt;
	uint64_t seed, steps;
	int32_t ntiles, flat, pack, ring_slots, flat_tmax, threads, npt, tile; // flat: 1 window_flat, 2 window_ordered
	int32_t nbufs, slot_vecs; // window_slots' vectors per slot (0: variable slices)
};
constexpr char CKPT_MAGIC[8] = { 'S', 'P', 'K', 'C', 'K', 'P', 'T', '1' };

// the checkpointed buffers of a net, by id (the same order on save and restore)
std::vector<std::pair<uint32_t, void *>> ckpt_buffers( spk_net & net )
{
	std::vector<std::pair<uint32_t, void *>> b;
	auto add = [&]( uint32_t id, auto & buf ) { b.push_back( { id, static_cast<void *>( &buf ) } ); };
	add( 1, net.edges );
	spk::model_traits const md = describe( net.model );
	for( int i = 0; i < md.neuron_attrs; i++ ) add( 10 + i, net.attr[i] );
	if( !md.plastic )
		for( int i = 0; i < md.synapse_attrs; i++ ) add( 30 + i, net.syn[i] );
	add( 20, net.ring_ids );
	add( 21, net.ring_cnt );
	add( 22, net.clock );
	add( 23, net.dt_ring );
	if( net.flat ) add( 24, net.done_step );
	return b;
}
std::vector<std::pair<uint32_t, spk::plastic_state::buf *>> ckpt_plastic( spk_net & net )
{
	auto & q = net.plast;
	if( !plastic_of( net.model ) ) return {};
	return { { 40, &q.W },        { 41, &q.za },         { 42, &q.zpre },       { 43, &q.zpost },     { 44, &q.hist },
	         { 45, &q.rf_a },     { 46, &q.zrf_a },      { 47, &q.rf_c },       { 48, &q.zrf_c },     { 49, &q.ring_meta },
	         { 50, &q.flush_ring }, { 51, &q.flush_cnt }, { 52, &q.ring_pot } };
}

// The contents a restored net's kernels index with, checked on the host before any
// device work: the edges (as an imported graph), the tiling and kernel shape against
// what the builders can produce, the spike ring's per-tile segments and, for Brunel+,
// the lazy-STDP rings and row states. A corrupted or hand-edited checkpoint is refused
// with SPK_ERR_INVALID instead of sending a kernel outside its buffers.
using ckpt_dir = std::vector<std::tuple<uint32_t, uint64_t, unsigned char const *>>;
unsigned char const * ckpt_find( ckpt_dir const & dir, uint32_t id, uint64_t bytes )
{
	for( auto const & d : dir )
		if( std::get<0>( d ) == id )
		{
			require( std::get<1>( d ) == bytes, "checkpoint buffer size differs from the net's" );
			return std::get<2>( d );
		}
	throw spk_error( SPK_ERR_INVALID, "checkpoint lacks a buffer" );
}
template <typename T>
std::vector<T> ckpt_read( ckpt_dir const & dir, uint32_t id, uint64_t count )
{
	std::vector<T> v( count );
	if( count ) std::memcpy( v.data(), ckpt_find( dir, id, count * sizeof( T ) ), count * sizeof( T ) );
	return v;
}
void validate_checkpoint( ckpt_header const & h, std::vector<int> const & first, ckpt_dir const & dir )
{
	uint64_t const n = (uint64_t)h.n, width = (uint64_t)h.width;
	int const T = h.ntiles;
	bool const plastic = plastic_of( h.model );
	// the graph
	int32_t const * edges = n * width ? reinterpret_cast<int32_t const *>( ckpt_find( dir, 1, n * width * 4 ) ) : nullptr;
	if( edges )
	{
		// read in place when aligned (the directory keeps buffers at 4-byte offsets)
		std::vector<int32_t> copy;
		int32_t const * e = edges;
		if( reinterpret_cast<uintptr_t>( edges ) % alignof( int32_t ) )
		{
			copy.resize( n * width );
			std::memcpy( copy.data(), edges, n * width * 4 );
			e = copy.data();
		}
		validate_edges( e, n, width );
		// tiles that receive synapses
		std::vector<char> in_tile( T, 0 );
		std::vector<char> target( n, 0 );
		for( uint64_t k = 0; k < n * width; k++ )
			if( e[k] != INT_MAX ) target[e[k]] = 1;
		for( int j = 0; j < T; j++ )
			for( int d = first[j]; d < first[j + 1] && !in_tile[j]; d++ ) in_tile[j] = target[d];
		if( h.flat == 1 )
		{
			unsigned const pad = h.pack == 12 ? spk::SLICE_PAD10 : spk::SLICE_PAD;
			for( int j = 0; j < T; j++ )
				if( in_tile[j] )
				{
					long long const span = first[j + 1] - first[j];
					require( span <= h.flat_tmax && (long long)classes_of( h.model ) * span < (long long)pad,
					         "checkpoint tiling does not fit its kernel: a tile with inputs exceeds the tile limit" );
				}
		}
	}
	require( h.slot_vecs == 0 || ( h.flat == 1 && h.pack == 12 && h.delay >= 7 && ( h.slot_vecs == 2 || h.slot_vecs == 4 || h.slot_vecs == 8 ) ),
	         "checkpoint tiling does not fit its kernel: slots" );
	// the kernel shape
	spk::model_traits const md = describe( h.model );
	require( h.flat >= 0 && h.flat <= 2 && ( h.flat != 1 || md.classes > 0 ) && ( h.flat == 2 || !md.ordered ) && ( h.flat != 2 || !plastic ),
	         "checkpoint kernel does not fit the model" );
	if( h.flat == 2 )
		require( ( h.npt == 1 || h.npt == 2 ) && h.threads >= 32 && h.threads <= 512 && h.threads % 32 == 0 && h.tile == h.threads * h.npt &&
		             h.tile <= spk::ORD_MAX_TILE && first == uniform_tiles( h.n, h.tile ),
		         "checkpoint tiling does not fit its kernel" );
	else if( h.flat )
	{
		require( !plastic && T + 1 < spk::FLAT_PC && h.threads == spk::FLAT_THREADS && h.npt == 1 && h.tile == h.flat_tmax &&
		             h.flat_tmax >= 32 && h.flat_tmax <= ( h.width <= spk::FLAT_MAX_SLICE ? spk::FLAT_MAX_TILE_WIDE : spk::FLAT_MAX_TILE ) &&
		             h.flat_tmax % 32 == 0,
		         "checkpoint tiling does not fit its kernel" );
	}
	else
	{
		require( ( h.npt == 1 || h.npt == 2 || h.npt == 4 ) && h.threads >= 32 && h.threads <= 512 && h.threads % 32 == 0 &&
		             h.tile == h.threads * h.npt && h.tile <= ( plastic ? 512 : 2048 ) && ( !plastic || h.npt == 1 ) &&
		             first == uniform_tiles( h.n, h.tile ),
		         "checkpoint tiling does not fit its kernel" );
	}
	// the spike ring: per slot and tile, an ascending run of the tile's own neurons
	uint64_t const slots = (uint64_t)h.ring_slots;
	auto const cnt = ckpt_read<uint32_t>( dir, 21, slots * T );
	auto const ids = ckpt_read<int32_t>( dir, 20, slots * n );
	auto check_segments = [&]( std::vector<uint32_t> const & counts, auto && id_at, char const * what ) {
		for( uint64_t sl = 0; sl < counts.size() / T; sl++ )
			for( int j = 0; j < T; j++ )
			{
				uint32_t const c = counts[sl * T + j];
				require( c <= (uint32_t)( first[j + 1] - first[j] ), what );
				int prev = first[j] - 1;
				for( uint32_t k = 0; k < c; k++ )
				{
					int const v = id_at( sl * n + first[j] + k );
					require( v > prev && v < first[j + 1], what );
					prev = v;
				}
			}
	};
	check_segments( cnt, [&]( uint64_t i ) { return ids[i]; }, "checkpoint spike ring is inconsistent" );
	if( !plastic ) return;
	// Brunel+: the flush ring's sources and every replay window at most the history's 64
	// steps; row states pending no longer than the forced flush allows
	struct ent
	{
		int32_t a, b, c, d;
	};
	uint64_t const ps = 2ull * h.delay;
	require( slots == ps, "checkpoint spike ring is inconsistent" );
	auto const fcnt = ckpt_read<uint32_t>( dir, 51, ps * T );
	auto const fring = ckpt_read<ent>( dir, 50, ps * n );
	auto const meta = ckpt_read<ent>( dir, 49, ps * n );
	check_segments( fcnt, [&]( uint64_t i ) { return fring[i].a; }, "checkpoint flush ring is inconsistent" );
	for( uint64_t sl = 0; sl < ps; sl++ )
		for( int j = 0; j < T; j++ )
		{
			for( uint32_t k = 0; k < fcnt[sl * T + j]; k++ )
				require( fring[sl * n + first[j] + k].b >= 0 && fring[sl * n + first[j] + k].b <= 64, "checkpoint flush ring is inconsistent" );
			for( uint32_t k = 0; k < cnt[sl * T + j]; k++ )
				require( ( meta[sl * n + first[j] + k].a & 0xff ) <= 64, "checkpoint spike ring is inconsistent" );
		}
	long long const now = (long long)h.steps;
	auto const rf_a = ckpt_read<int32_t>( dir, 45, n );
	auto const rf_c = ckpt_read<int32_t>( dir, 47, n );
	for( uint64_t i = 0; i < n; i++ )
	{
		require( rf_a[i] == -1 || ( rf_a[i] >= 0 && rf_a[i] >= now + h.delay - 64 && rf_a[i] <= now + h.delay ),
		         "checkpoint STDP row state is inconsistent" );
		require( rf_c[i] == -1 || ( rf_c[i] >= 0 && rf_c[i] >= now - 64 && rf_c[i] <= now + h.delay ),
		         "checkpoint STDP row state is inconsistent" );
	}
}

// pooled: the net's buffers come from the device's stream-ordered pool and its stream
// from the stream_recycler (the serving loop's nets); otherwise cudaMalloc and a stream
// of its own, destroyed with the net
spk_net * new_net( int model, float dt, int delay, unsigned long long seed, int device, bool pooled = false )
{
	describe( model );
	require( dt > 0.0f, "dt must be > 0" );
	require( delay >= 1, "delay must be >= 1" );
	require( !plastic_of( model ) || delay <= spk::PL_MAX_DELAY, "plastic models support delays up to 63 steps" );
	int ndev = 0;
	CK( cudaGetDeviceCount( &ndev ) );
	require( device >= 0 && device < ndev, "invalid device" );
	auto net = std::make_unique<spk_net>();
	net->model = model;
	net->device = device;
	net->opts = resolve_opts( nullptr ); // the automatic choices (creators with options replace them)
	CK( cudaDeviceGetAttribute( &net->sms, cudaDevAttrMultiProcessorCount, device ) );
	net->dt = dt;
	net->delay = delay;
	net->seed = seed;
	device_guard g( device ); // the stream belongs to the net's device
	// a net's own work (building it, its windows, exports) at the highest stream priority:
	// beside the long shared launches of a batch its CTAs start as soon as an SM frees up
	net->owner.device = device;
	net->owner.recycle = pooled;
	if( pooled )
		net->owner.s = stream_recycler::take( device );
	else
	{
		int least = 0, greatest = 0;
		CK( cudaDeviceGetStreamPriorityRange( &least, &greatest ) );
		CK( cudaStreamCreateWithPriority( &net->owner.s, cudaStreamNonBlocking, greatest ) );
	}
	net->stream = net->owner.s;
	if( pooled ) net->pool = scratch_pool( device );
	if( char const * w = getenv( "SPK_TEST_WAIT_LIMIT" ) ) net->wait_limit = std::max( 1, atoi( w ) );
	if( char const * h = getenv( "SPK_TEST_WITHHOLD_TILE" ) ) net->withhold_tile = atoi( h );
	return net.release();
}
} // namespace

// ------------------------------------------------------------------------------------
// batching: many independent window_flat nets stepped by shared launches
// ------------------------------------------------------------------------------------
struct spk_batch
{
	// the nets of one model: stepped by their own launches on their own stream, so the
	// models' launches overlap
	struct group
	{
		cudaStream_t stream = nullptr;
		cudaEvent_t ev = nullptr;
		dbuf d_params, d_jobs, d_pls;
		std::vector<spk::net_params> h_params, c_params; // this run's / on the device
		std::vector<spk::plastic_params> h_pls, c_pls;   // plastic groups
		std::vector<int4> h_jobs, c_jobs;
		std::vector<std::pair<int, int>> c_launches; // rounds of the captured graph
		cudaGraphExec_t graph = nullptr;             // the rounds of the last job table
		void drop_graph()
		{
			if( graph ) cudaGraphExecDestroy( graph );
			graph = nullptr;
			c_launches.clear();
		}
	};
	int device = 0;
	std::vector<spk_net *> nets;
	// by model id and kernel: window_flat, window_slots, window_plastic (one CTA per SM, up to
	// 512 threads), then window_plastic in its two-CTAs-per-SM form for tiles of 257 to
	// PL_THREADS, up to 128 and 129 to 256 neurons (a launch is as wide as its widest tile:
	// narrow tiles in narrow launches, so several of their CTAs share an SM)
	static constexpr int KINDS = 6;
	group groups[KINDS * spk::MODEL_COUNT];

	~spk_batch()
	{
		for( auto * net : nets ) net->batch = nullptr;
		for( auto & g : groups )
		{
			g.drop_graph();
			if( g.ev ) cudaEventDestroy( g.ev );
			if( g.stream ) cudaStreamDestroy( g.stream );
		}
	}

	// stepped by the shared launches (window_flat_batch, window_slots_batch,
	// window_plastic_batch); window_counts and window_ordered nets run their own windows
	static bool shared( spk_net const & net ) { return ( net.flat && !plastic_of( net.model ) ) || plastic_of( net.model ); }
	static int kind( spk_net const & net )
	{
		if( plastic_of( net.model ) )
		{
			int const w = net.tc.threads;
			return w <= 128 ? 4 : w <= 256 ? 5 : w <= spk::PL_THREADS ? 3 : 2;
		}
		return net.slot_vecs ? 1 : 0;
	}

	template <typename Model>
	static void launch_model( group & g, int4 const * jobs, int njobs, int smem, int kind, int threads )
	{
		auto const * params = g.d_params.as<spk::net_params const>();
		if constexpr( spk::is_flat_model<Model> )
		{
			if( kind == 1 )
				spk::window_slots_batch<Model><<<njobs, spk::FLAT_THREADS, smem, g.stream>>>( params, jobs, smem );
			else
				spk::window_flat_batch<Model><<<njobs, spk::FLAT_THREADS, smem, g.stream>>>( params, jobs, smem );
			CK( cudaGetLastError() );
		}
		else if constexpr( spk::is_plastic_model<Model> )
		{
			auto const * pls = g.d_pls.as<spk::plastic_params const>();
			if( kind >= 3 )
				spk::window_plastic_batch<Model, spk::PL_CTAS_PER_SM><<<njobs, threads, smem, g.stream>>>( params, pls, jobs );
			else
				spk::window_plastic_batch<Model, 1><<<njobs, threads, smem, g.stream>>>( params, pls, jobs );
			CK( cudaGetLastError() );
		}
	}

	// advance the nets of one model by nsteps: rounds of one launch, every tile of every net
	// running up to its own window (delay) of steps per round
	void run_group( group & g, int model, int kind, std::vector<spk_net *> const & gn, std::vector<unsigned long long> const & counts )
	{
		for( auto * net : gn )
		{
			net->flush();
			CK( cudaEventRecord( g.ev, net->stream ) );
			CK( cudaStreamWaitEvent( g.stream, g.ev, 0 ) );
		}
		g.h_params.resize( gn.size() );
		for( size_t i = 0; i < gn.size(); i++ ) g.h_params[i] = gn[i]->params();
		bool const plastic = kind >= 2;
		g.h_pls.resize( plastic ? gn.size() : 0 );
		for( size_t i = 0; i < g.h_pls.size(); i++ ) g.h_pls[i] = gn[i]->plast.params();
		// all rounds' jobs (net, tile, steps, dt) at once; a round whose windows equal the
		// previous round's reuses its jobs
		std::vector<unsigned long long> left = counts;
		std::vector<std::pair<int, int>> launches; // (first job, count)
		g.h_jobs.clear();
		std::vector<int> L( gn.size(), 0 ), prevL;
		for( bool more = std::any_of( left.begin(), left.end(), []( unsigned long long x ) { return x > 0; } ); more; )
		{
			more = false;
			for( size_t i = 0; i < gn.size(); i++ )
				L[i] = left[i] ? (int)std::min<unsigned long long>( left[i], (unsigned long long)gn[i]->max_window() ) : 0;
			if( L == prevL )
				launches.push_back( launches.back() );
			else
			{
				int const first = (int)g.h_jobs.size();
				for( size_t i = 0; i < gn.size(); i++ )
					if( L[i] )
					{
						int dtbits;
						std::memcpy( &dtbits, &gn[i]->dt, 4 );
						for( int j = 0; j < gn[i]->tc.ntiles; j++ ) g.h_jobs.push_back( make_int4( (int)i, j, L[i], dtbits ) );
					}
				launches.push_back( { first, (int)g.h_jobs.size() - first } );
				prevL = L;
			}
			for( size_t i = 0; i < gn.size(); i++ )
			{
				left[i] -= L[i];
				more = more || left[i];
			}
		}
		size_t const pb = g.h_params.size() * sizeof( spk::net_params ), jb = g.h_jobs.size() * sizeof( int4 );
		size_t const qb = g.h_pls.size() * sizeof( spk::plastic_params );
		if( g.d_params.bytes < pb || g.d_jobs.bytes < jb || g.d_pls.bytes < qb )
		{
			CK( cudaStreamSynchronize( g.stream ) ); // launches reading the old ones
			g.drop_graph();                          // captured the old buffers
			g.c_params.clear();
			g.c_jobs.clear();
			g.c_pls.clear();
		}
		if( g.d_params.bytes < pb ) g.d_params.alloc( pb );
		if( g.d_jobs.bytes < jb ) g.d_jobs.alloc( jb );
		if( g.d_pls.bytes < qb ) g.d_pls.alloc( qb );
		// pageable sources: each copy returns once its source is staged, and the stream
		// orders it after the previous run's launches that read the same buffers; a table
		// equal to the one on the device is not sent again
		auto same = []( auto const & a, auto const & b ) {
			return a.size() == b.size() && ( a.empty() || !std::memcmp( a.data(), b.data(), a.size() * sizeof( a[0] ) ) );
		};
		if( !same( g.h_params, g.c_params ) )
		{
			CK( cudaMemcpyAsync( g.d_params.p, g.h_params.data(), pb, cudaMemcpyHostToDevice, g.stream ) );
			g.c_params = g.h_params;
		}
		if( !same( g.h_jobs, g.c_jobs ) )
		{
			CK( cudaMemcpyAsync( g.d_jobs.p, g.h_jobs.data(), jb, cudaMemcpyHostToDevice, g.stream ) );
			g.c_jobs = g.h_jobs;
			g.drop_graph();
		}
		if( !same( g.h_pls, g.c_pls ) )
		{
			CK( cudaMemcpyAsync( g.d_pls.p, g.h_pls.data(), qb, cudaMemcpyHostToDevice, g.stream ) );
			g.c_pls = g.h_pls;
		}
		// launch shape: window_flat's fixed one, or the widest plastic tile and the largest
		// shared-memory carve-up at that width
		int threads = spk::FLAT_THREADS, smem = kind == 1 ? gn[0]->slot_smem : gn[0]->flat_smem;
		if( plastic )
		{
			threads = 32;
			for( auto * net : gn ) threads = std::max( threads, net->tc.threads );
			smem = 0;
			for( auto * net : gn ) smem = std::max( smem, spk::plastic_window_smem( net->tc.tile, net->tc.ntiles, threads ) );
		}
		auto launch_all = [&] {
			for( auto const & l : launches )
			{
				int4 const * jobs = g.d_jobs.as<int4 const>() + l.first;
				dispatch( model, [&]( auto tag ) { launch_model<typename decltype( tag )::type>( g, jobs, l.second, smem, kind, threads ); } );
			}
		};
		// the rounds as one CUDA graph, captured once per job table and round sequence and
		// replayed by later runs of the same nets and step counts (serving ticks, loops)
		if( launches.size() < 2 )
			launch_all();
		else
		{
			if( g.graph && g.c_launches != launches ) g.drop_graph();
			if( !g.graph )
			{
				cudaGraph_t cg;
				CK( cudaStreamBeginCapture( g.stream, cudaStreamCaptureModeThreadLocal ) );
				launch_all();
				CK( cudaStreamEndCapture( g.stream, &cg ) );
				cudaError_t const e = cudaGraphInstantiate( &g.graph, cg, 0 );
				cudaGraphDestroy( cg );
				CK( e );
				g.c_launches = launches;
			}
			CK( cudaGraphLaunch( g.graph, g.stream ) );
		}
		for( size_t i = 0; i < gn.size(); i++ )
		{
			gn[i]->steps += counts[i];
			gn[i]->launched += counts[i];
			gn[i]->kernel_launches += ( counts[i] + gn[i]->max_window() - 1 ) / gn[i]->max_window(); // shared launches
		}
		CK( cudaEventRecord( g.ev, g.stream ) );
		for( auto * net : gn ) CK( cudaStreamWaitEvent( net->stream, g.ev, 0 ) );
	}

	// advance nets[i] by counts[i] steps (members of the batch)
	void run( std::vector<spk_net *> const & which, std::vector<unsigned long long> const & counts )
	{
		// nets outside the shared kernels (window_counts, window_ordered) run their own
		// windows on their own streams, concurrently with the shared launches
		std::vector<spk_net *> gn[KINDS * spk::MODEL_COUNT];
		std::vector<unsigned long long> gc[KINDS * spk::MODEL_COUNT];
		for( size_t i = 0; i < which.size(); i++ )
		{
			if( counts[i] == 0 ) continue;
			if( shared( *which[i] ) )
			{
				int const gi = KINDS * which[i]->model + kind( *which[i] );
				gn[gi].push_back( which[i] );
				gc[gi].push_back( counts[i] );
			}
			else
				which[i]->run( counts[i] );
		}
		for( int m = 0; m < KINDS * spk::MODEL_COUNT; m++ )
			if( !gn[m].empty() ) run_group( groups[m], m / KINDS, m % KINDS, gn[m], gc[m] );
	}
};

namespace
{
int create_net(
    spk_net ** out,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    int device,
    spk_net_options const * opts,
    bool pooled )
{
	return guarded( [&] {
		require( out != nullptr, "out is null" );
		*out = nullptr;
		build_opts const o = resolve_opts( opts );
		auto const l = to_layout( desc );
		std::unique_ptr<spk_net> net( new_net( model, dt, delay, seed, device, pooled ) );
		net->opts = o;
		device_guard g( device );
		allocate( *net, (long long)l.size(), (long long)l.max_degree(), layout_costs( l ) );
		enqueue_generate( net->stream, l, graph_seed, net->edges.as<int>(), net->conns_dev, net->mem() );
		enqueue_pivots( *net );
		init_state( *net );
		CK( cudaStreamSynchronize( net->stream ) );
		*out = net.release();
	} );
}

void detach( spk_batch * b, spk_net * net )
{
	b->nets.erase( std::remove( b->nets.begin(), b->nets.end(), net ), b->nets.end() );
	net->batch = nullptr;
}
} // namespace

void spk_set_last_error( std::string const & msg ) { g_err = msg; }

// The serving loop's fault injection (spk_server_inject_device_error): the net's device
// error word as a kernel sets it when a bounded wait runs out, so that its next
// synchronisation reports SPK_ERR_DEVICE.
int spk_net_raise_device_error( spk_net * net )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		device_guard g( net->device );
		int const bits = spk::ERR_TIMEOUT;
		CK( cudaMemcpyAsync( net->err.p, &bits, sizeof bits, cudaMemcpyHostToDevice, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

// A net whose buffers come from the device's stream-ordered pool (on the net's stream):
// neither building nor destroying it synchronises the device, so the server's builder
// does not wait for the launches of the nets it steps meanwhile.
int spk_net_create_pooled(
    spk_net ** out, int model, spk_layout_desc const * desc, float dt, int delay, uint64_t seed, uint64_t graph_seed, int device, int tile_target )
{
	if( tile_target < 0 ) return guarded( [] { require( false, "tile target must be >= 0" ); } );
	spk_net_options o;
	spk_net_options_init( &o );
	o.tile_target = tile_target;
	return create_net( out, model, desc, dt, delay, seed, graph_seed, device, &o, true );
}

// Maps up to `bytes` (at most the device's free memory less 1 GiB) into the device's
// stream-ordered pool ahead of use: the pool keeps released memory, so nets built from it
// later reuse mapped memory instead of growing the pool beside running work (growing it
// took tens of milliseconds per net in the serving loop). Best effort: a failed
// reservation leaves the pool to grow on demand.
void spk_reserve_pool( int device, uint64_t bytes )
{
	int ndev = 0;
	if( cudaGetDeviceCount( &ndev ) != cudaSuccess || device < 0 || device >= ndev ) return;
	try
	{
		device_guard g( device );
		size_t free_b = 0, total_b = 0;
		if( cudaMemGetInfo( &free_b, &total_b ) != cudaSuccess ) return;
		size_t const margin = (size_t)1 << 30;
		size_t const size = std::min<size_t>( bytes, free_b > margin ? free_b - margin : 0 );
		if( size == 0 ) return;
		cudaStream_t s = stream_recycler::take( device );
		void * p = nullptr;
		if( cudaMallocFromPoolAsync( &p, size, scratch_pool( device ), s ) == cudaSuccess ) cudaFreeAsync( p, s );
		cudaGetLastError();
		cudaStreamSynchronize( s );
		stream_recycler::give( device, s );
	}
	catch( ... )
	{
		cudaGetLastError();
	}
}

// hands the pool's unused memory back to the device (after a server's nets are gone)
void spk_trim_pool( int device )
{
	int ndev = 0;
	if( cudaGetDeviceCount( &ndev ) != cudaSuccess || device < 0 || device >= ndev ) return;
	cudaMemPoolTrimTo( scratch_pool( device ), 0 );
}

extern "C" {
char const * spk_last_error( void ) { return g_err.c_str(); }

int spk_layout_flatten(
    spk_layout_desc const * desc, int * out_ranges, float * out_p, int cap, int * out_count, uint64_t * out_size, uint64_t * out_max_degree )
{
	return guarded( [&] {
		auto const l = to_layout( desc );
		int i = 0;
		for( auto const & c : l.connections() )
		{
			if( i < cap )
			{
				if( out_ranges )
				{
					out_ranges[4 * i + 0] = std::get<0>( c );
					out_ranges[4 * i + 1] = std::get<1>( c );
					out_ranges[4 * i + 2] = std::get<2>( c );
					out_ranges[4 * i + 3] = std::get<3>( c );
				}
				if( out_p ) out_p[i] = std::get<4>( c );
			}
			i++;
		}
		if( out_count ) *out_count = i;
		if( out_size ) *out_size = l.size();
		if( out_max_degree ) *out_max_degree = l.max_degree();
	} );
}

int spk_generate_adj_list( void * stream, spk_layout_desc const * desc, uint64_t seed, int32_t * d_edges )
{
	return guarded( [&] {
		auto const l = to_layout( desc );
		require( d_edges != nullptr || l.size() * l.max_degree() == 0, "edges pointer is null" );
		cudaStream_t const s = static_cast<cudaStream_t>( stream );
		static thread_local dbuf conns; // kept alive until the next call on this thread
		CK( cudaStreamSynchronize( s ) );
		enqueue_generate( s, l, seed, d_edges, conns );
	} );
}

int spk_net_create( spk_net ** out, int model, spk_layout_desc const * desc, float dt, int delay, uint64_t seed, uint64_t graph_seed, int device )
{
	return spk_net_create_ex( out, model, desc, dt, delay, seed, graph_seed, device, 0 );
}

int spk_net_create_ex(
    spk_net ** out, int model, spk_layout_desc const * desc, float dt, int delay, uint64_t seed, uint64_t graph_seed, int device, int tile_target )
{
	if( tile_target < 0 ) return guarded( [] { require( false, "tile target must be >= 0" ); } );
	spk_net_options o;
	spk_net_options_init( &o );
	o.tile_target = tile_target;
	return create_net( out, model, desc, dt, delay, seed, graph_seed, device, &o, false );
}

int spk_net_create_opts(
    spk_net ** out, int model, spk_layout_desc const * desc, float dt, int delay, uint64_t seed, uint64_t graph_seed, int device, spk_net_options const * opts )
{
	return create_net( out, model, desc, dt, delay, seed, graph_seed, device, opts, false );
}

void spk_net_options_init( spk_net_options * o )
{
	if( !o ) return;
	o->tile_target = 0;
	o->kernel = o->slice_bits = o->tiling = o->persistent = o->pipelined = o->slots = -1;
}

int spk_net_estimate_bytes_opts( int model, spk_layout_desc const * desc, int delay, int device, spk_net_options const * opts, uint64_t * out_bytes )
{
	return guarded( [&] {
		require( out_bytes != nullptr, "out is null" );
		require( delay >= 1, "invalid delay" );
		describe( model );
		auto const l = to_layout( desc );
		*out_bytes = estimate_bytes( model, l, delay, device, resolve_opts( opts ) );
	} );
}

int spk_net_estimate_bytes( int model, spk_layout_desc const * desc, int delay, int device, int tile_target, uint64_t * out_bytes )
{
	if( tile_target < 0 ) return guarded( [] { require( false, "invalid delay or tile target" ); } );
	spk_net_options o;
	spk_net_options_init( &o );
	o.tile_target = tile_target;
	return spk_net_estimate_bytes_opts( model, desc, delay, device, &o, out_bytes );
}

int spk_net_create_from_adj(
    spk_net ** out, int model, int32_t const * edges, uint64_t num_neurons, uint64_t width, float dt, int delay, uint64_t seed, int device )
{
	return guarded( [&] {
		require( out != nullptr, "out is null" );
		*out = nullptr;
		require( edges != nullptr || num_neurons * width == 0, "edges is null" );
		std::unique_ptr<spk_net> net( new_net( model, dt, delay, seed, device ) );
		device_guard g( device );
		validate_edges( edges, num_neurons, width );
		allocate( *net, (long long)num_neurons, (long long)width, adjacency_costs( edges, (long long)num_neurons, (long long)width ) );
		if( num_neurons * width )
			CK( cudaMemcpyAsync( net->edges.p, edges, num_neurons * width * 4, cudaMemcpyHostToDevice, net->stream ) );
		enqueue_pivots( *net );
		init_state( *net );
		CK( cudaStreamSynchronize( net->stream ) );
		*out = net.release();
	} );
}

int spk_net_set_neurons( spk_net * net, void * const * attrs )
{
	return guarded( [&] {
		require( net && attrs, "null argument" );
		device_guard g( net->device );
		net->flush();
		spk::model_traits const md = describe( net->model );
		for( int i = 0; i < md.neuron_attrs; i++ )
			CK( cudaMemcpyAsync( net->attr[i].p, attrs[i], (size_t)net->n * 4, cudaMemcpyHostToDevice, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_set_synapses( spk_net * net, void * const * attrs )
{
	return guarded( [&] {
		require( net && attrs, "null argument" );
		device_guard g( net->device );
		net->flush();
		spk::model_traits const md = describe( net->model );
		if( md.synapse_attrs == 0 ) return;
		require( net->steps == 0, "synapse state can only be imported before the first step" );
		dispatch( net->model, [&]( auto tag ) {
			using M = typename decltype( tag )::type;
			if constexpr( spk::is_plastic_model<M> )
				net->plast.import<M>( net->params(), static_cast<float const *>( attrs[0] ), static_cast<float const *>( attrs[1] ),
				                      static_cast<float const *>( attrs[2] ), net->dt, net->sms, net->stream );
			else
				for( int i = 0; i < md.synapse_attrs; i++ )
					CK( cudaMemcpyAsync( net->syn[i].p, attrs[i], net->syn[i].bytes, cudaMemcpyHostToDevice, net->stream ) );
		} );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_destroy( spk_net * net )
{
	return guarded( [&] {
		if( !net ) return;
		if( net->batch ) detach( net->batch, net );
		{
			device_guard g( net->device );
			cudaStreamSynchronize( net->stream );
		}
		delete net;
	} );
}

int spk_net_step( spk_net * net, int32_t * out_ids, uint64_t cap, uint64_t * out_count )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		device_guard g( net->device );
		net->steps++;
		if( !out_ids && !out_count )
		{
			if( net->steps - net->launched >= (unsigned long long)net->max_window() ) net->flush();
			return;
		}
		net->flush();
		CK( cudaMemsetAsync( net->cursor.p, 0, 8, net->stream ) );
		net->gather( 1, net->gather_ids.as<int>(), net->gather_cnt.as<unsigned>(), (unsigned long long)net->n, 0 );
		CK( cudaMemcpyAsync( net->host_count, net->gather_cnt.p, 4, cudaMemcpyDeviceToHost, net->stream ) );
		net->check_device_error();
		uint64_t const c = net->host_count[0];
		if( out_count ) *out_count = c;
		if( !out_ids ) return;
		if( c > cap ) throw spk_error( SPK_ERR_CAPACITY, "spike buffer too small" );
		if( c ) CK( cudaMemcpyAsync( out_ids, net->gather_ids.p, c * 4, cudaMemcpyDeviceToHost, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_run( spk_net * net, uint64_t nsteps )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		device_guard g( net->device );
		net->run( nsteps );
	} );
}

int spk_net_run_record( spk_net * net, uint64_t nsteps, uint32_t * counts, int32_t * ids, uint64_t ids_cap, uint64_t * out_total )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		require( counts != nullptr || nsteps == 0, "counts is null" );
		device_guard g( net->device );
		net->flush();
		if( nsteps == 0 )
		{
			if( out_total ) *out_total = 0;
			return;
		}
		if( net->rec_ids.bytes < std::max<uint64_t>( ids_cap, 1 ) * 4 ) net->rec_ids.alloc( std::max<uint64_t>( ids_cap, 1 ) * 4, net->mem() );
		if( net->rec_cnt.bytes < nsteps * 4 ) net->rec_cnt.alloc( nsteps * 4, net->mem() );
		CK( cudaMemsetAsync( net->cursor.p, 0, 8, net->stream ) );
		// non-plastic nets record in chunks: a chunk's steps (one persistent launch, or its
		// windows replayed from a CUDA graph) into a ring enlarged to hold the chunk (bounded
		// to RECORD_RING_BYTES), then one gather per chunk; plastic nets, whose lazy-STDP
		// rings have 2 delay slots, gather every window
		long long chunk = 0;
		if( !plastic_of( net->model ) )
		{
			long long const per_slot = net->n * 4 + (long long)net->tc.ntiles * 4;
			long long const fit = RECORD_RING_BYTES / per_slot - 2LL * net->delay;
			chunk = std::min<long long>( { (long long)nsteps, fit, 1LL << 20 } );
			if( chunk < 4LL * net->max_window() ) chunk = 0;
			else net->grow_ring( (int)( chunk + 2 * net->delay ) );
		}
		uint64_t done = 0;
		while( done < nsteps )
		{
			int const L = (int)std::min<uint64_t>( nsteps - done, chunk > 0 ? (uint64_t)chunk : (uint64_t)net->max_window() );
			if( chunk > 0 && !net->persistent )
				net->run( L ); // the chunk's windows (counted there)
			else
			{
				net->steps += L;
				if( chunk > 0 )
					net->launch_persistent( L );
				else
					net->launch_window( L );
				net->launched += L;
				net->kernel_launches++;
			}
			net->gather( L, net->rec_ids.as<int>(), net->rec_cnt.as<unsigned>(), ids_cap, (long long)done );
			done += L;
		}
		unsigned long long total = 0;
		CK( cudaMemcpyAsync( net->host_count, net->cursor.p, 8, cudaMemcpyDeviceToHost, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
		std::memcpy( &total, net->host_count, 8 );
		if( out_total ) *out_total = total;
		int e = 0;
		CK( cudaMemcpy( &e, net->err.p, 4, cudaMemcpyDeviceToHost ) );
		if( e & spk::ERR_OVERFLOW )
		{
			CK( cudaMemsetAsync( net->err.p, 0, 4, net->stream ) );
			throw spk_error( SPK_ERR_CAPACITY, "spike raster buffer too small" );
		}
		if( e ) throw spk_error( SPK_ERR_DEVICE, "device error flag " + std::to_string( e ) );
		CK( cudaMemcpyAsync( counts, net->rec_cnt.p, nsteps * 4, cudaMemcpyDeviceToHost, net->stream ) );
		if( total && ids ) CK( cudaMemcpyAsync( ids, net->rec_ids.p, total * 4, cudaMemcpyDeviceToHost, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_stream( spk_net * net, void ** out_stream )
{
	return guarded( [&] {
		require( net && out_stream, "null argument" );
		device_guard g( net->device );
		net->flush();
		*out_stream = net->stream;
	} );
}

int spk_net_idle( spk_net * net, int * out_idle )
{
	return guarded( [&] {
		require( net != nullptr && out_idle != nullptr, "null argument" );
		device_guard g( net->device );
		net->flush();
		cudaError_t const e = cudaStreamQuery( net->stream );
		if( e != cudaErrorNotReady ) CK( e );
		*out_idle = e == cudaSuccess ? 1 : 0;
	} );
}

int spk_net_sync( spk_net * net )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		device_guard g( net->device );
		net->sync();
	} );
}

int spk_net_get_info( spk_net * net, spk_net_info * out )
{
	return guarded( [&] {
		require( net && out, "null argument" );
		out->model = net->model;
		out->device = net->device;
		out->num_neurons = (uint64_t)net->n;
		out->num_synapses = (uint64_t)( net->n * net->width );
		out->width = (uint64_t)net->width;
		out->delay = net->delay;
		out->dt = net->dt;
		out->steps = net->steps;
		out->tile_size = (uint64_t)net->tc.tile;
		out->num_tiles = (uint64_t)net->tc.ntiles;
		out->device_bytes = net->device_bytes();
		out->kernel_launches = net->kernel_launches;
		out->persistent = net->persistent ? 1 : 0;
		out->slice_pack = net->flat ? net->pack : 0;
		out->slot_vecs = net->slot_vecs;
	} );
}

int spk_net_adj( spk_net * net, int32_t * out, uint64_t cap )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		uint64_t const need = (uint64_t)( net->n * net->width );
		if( cap < need ) throw spk_error( SPK_ERR_CAPACITY, "adjacency buffer too small" );
		device_guard g( net->device );
		net->sync();
		if( need ) CK( cudaMemcpyAsync( out, net->edges.p, need * 4, cudaMemcpyDeviceToHost, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_neurons( spk_net * net, void * const * attrs )
{
	return guarded( [&] {
		require( net && attrs, "null argument" );
		device_guard g( net->device );
		net->sync();
		spk::model_traits const md = describe( net->model );
		for( int i = 0; i < md.neuron_attrs; i++ )
			CK( cudaMemcpyAsync( attrs[i], net->attr[i].p, (size_t)net->n * 4, cudaMemcpyDeviceToHost, net->stream ) );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_synapses( spk_net * net, void * const * attrs )
{
	return guarded( [&] {
		require( net && attrs, "null argument" );
		device_guard g( net->device );
		net->sync();
		spk::model_traits const md = describe( net->model );
		if( md.synapse_attrs == 0 ) return;
		dispatch( net->model, [&]( auto tag ) {
			using M = typename decltype( tag )::type;
			if constexpr( spk::is_plastic_model<M> )
				CK( net->plast.export_synapses<M>( net->params(), static_cast<float *>( attrs[0] ), static_cast<float *>( attrs[1] ),
				                                   static_cast<float *>( attrs[2] ), net->sms, net->stream ) );
			else
				for( int i = 0; i < md.synapse_attrs; i++ )
					CK( cudaMemcpyAsync( attrs[i], net->syn[i].p, net->syn[i].bytes, cudaMemcpyDeviceToHost, net->stream ) );
		} );
		CK( cudaStreamSynchronize( net->stream ) );
	} );
}

int spk_net_checkpoint( spk_net * net, void * buf, uint64_t cap, uint64_t * out_bytes )
{
	return guarded( [&] {
		require( net != nullptr && out_bytes != nullptr, "null argument" );
		device_guard g( net->device );
		net->sync(); // every queued step launched, and no device error
		auto const bufs = ckpt_buffers( *net );
		auto const pl = ckpt_plastic( *net );
		uint64_t total = sizeof( ckpt_header ) + ( net->tile_first_host.size() ) * 4;
		for( auto const & x : bufs ) total += 12 + static_cast<dbuf *>( x.second )->bytes;
		for( auto const & x : pl ) total += 12 + x.second->bytes;
		*out_bytes = total;
		if( buf == nullptr ) return; // size query
		require( cap >= total, "checkpoint buffer too small" );
		ckpt_header h{};
		std::memcpy( h.magic, CKPT_MAGIC, 8 );
		h.version = 1;
		h.model = net->model;
		h.n = net->n;
		h.width = net->width;
		h.delay = net->delay;
		h.dt = net->dt;
		h.seed = net->seed;
		h.steps = net->steps;
		h.ntiles = net->tc.ntiles;
		h.flat = net->flat ? 1 : net->ordered ? 2 : 0;
		h.pack = net->pack;
		h.ring_slots = net->ring_slots;
		h.flat_tmax = net->flat_tmax;
		h.threads = net->tc.threads;
		h.npt = net->tc.npt;
		h.tile = net->tc.tile;
		h.nbufs = (int32_t)( bufs.size() + pl.size() );
		h.slot_vecs = net->slot_vecs;
		unsigned char * o = static_cast<unsigned char *>( buf );
		std::memcpy( o, &h, sizeof h );
		o += sizeof h;
		std::memcpy( o, net->tile_first_host.data(), net->tile_first_host.size() * 4 );
		o += net->tile_first_host.size() * 4;
		auto put = [&]( uint32_t id, void const * dev, uint64_t bytes ) {
			std::memcpy( o, &id, 4 );
			std::memcpy( o + 4, &bytes, 8 );
			o += 12;
			if( bytes ) CK( cudaMemcpy( o, dev, bytes, cudaMemcpyDeviceToHost ) );
			o += bytes;
		};
		for( auto const & x : bufs ) put( x.first, static_cast<dbuf *>( x.second )->p, static_cast<dbuf *>( x.second )->bytes );
		for( auto const & x : pl ) put( x.first, x.second->p, x.second->bytes );
	} );
}

int spk_net_restore( spk_net ** out, void const * buf, uint64_t size, int device )
{
	return guarded( [&] {
		require( out != nullptr && buf != nullptr, "null argument" );
		*out = nullptr;
		require( size >= sizeof( ckpt_header ), "checkpoint truncated" );
		ckpt_header h;
		std::memcpy( &h, buf, sizeof h );
		require( !std::memcmp( h.magic, CKPT_MAGIC, 8 ) && h.version == 1, "not a checkpoint of this library" );
		describe( h.model );
		require( h.n > 0 && h.n <= INT_MAX && h.width >= 0 && h.width % 32 == 0 && h.delay >= 1 && h.ntiles >= 1 &&
		             h.ring_slots >= 2 * h.delay && ( h.pack == 8 || h.pack == 12 ),
		         "checkpoint header is inconsistent" );
		uint64_t const tiles_bytes = (uint64_t)( h.ntiles + 1 ) * 4;
		require( size >= sizeof h + tiles_bytes, "checkpoint truncated" );
		unsigned char const * in = static_cast<unsigned char const *>( buf ) + sizeof h;
		std::vector<int> first( h.ntiles + 1 );
		std::memcpy( first.data(), in, tiles_bytes );
		in += tiles_bytes;
		require( first[0] == 0 && first[h.ntiles] == h.n, "checkpoint tiling is inconsistent" );
		for( int i = 0; i < h.ntiles; i++ ) require( first[i] < first[i + 1], "checkpoint tiling is inconsistent" );
		// read the buffer directory first: every size and index checked before any device work
		ckpt_dir dir;
		unsigned char const * end = static_cast<unsigned char const *>( buf ) + size;
		for( int b = 0; b < h.nbufs; b++ )
		{
			require( end - in >= 12, "checkpoint truncated" );
			uint32_t id;
			uint64_t bytes;
			std::memcpy( &id, in, 4 );
			std::memcpy( &bytes, in + 4, 8 );
			in += 12;
			require( (uint64_t)( end - in ) >= bytes, "checkpoint truncated" );
			dir.emplace_back( id, bytes, in );
			in += bytes;
		}
		validate_checkpoint( h, first, dir );

		std::unique_ptr<spk_net> net( new_net( h.model, h.dt, h.delay, h.seed, device ) );
		device_guard g( device );
		net->n = h.n;
		net->width = h.width;
		CK( cudaDeviceGetAttribute( &net->sms, cudaDevAttrMultiProcessorCount, device ) );
		net->flat = h.flat == 1;
		net->ordered = h.flat == 2;
		net->pack = h.pack;
		net->flat_tmax = h.flat_tmax;
		net->tc = { h.threads, h.npt, h.tile, h.ntiles };
		net->opts.slots = h.slot_vecs; // the saved net's kernel and layout
		set_tiles( *net, first );
		net->ring_slots = h.ring_slots;
		allocate_buffers( *net );
		auto find = [&]( uint32_t id, uint64_t bytes ) { return ckpt_find( dir, id, bytes ); };
		// tiles without inputs keep only their state in shared memory: it must fit the
		// window kernel's shared memory (configured by allocate_buffers)
		if( net->flat )
			for( int j = 0; j < h.ntiles; j++ )
				require( spk::flat_state_bytes( net->neuron_attrs(), first[j + 1] - first[j] ) <= (size_t)net->flat_smem,
				         "checkpoint tiling does not fit its kernel: a tile exceeds the shared memory" );
		// edges first: the pivots and slices are rebuilt from them (which resets the
		// publication flags), then the state over them
		dbuf & e = net->edges;
		// every upload on the net's stream, ahead of the kernels that read it (a plain
		// cudaMemcpy from pageable memory may return before its DMA lands)
		if( e.bytes ) CK( cudaMemcpyAsync( e.p, find( 1, e.bytes ), e.bytes, cudaMemcpyHostToDevice, net->stream ) );
		enqueue_pivots( *net );
		CK( cudaStreamSynchronize( net->stream ) );
		for( auto const & x : ckpt_buffers( *net ) )
		{
			dbuf & d = *static_cast<dbuf *>( x.second );
			if( x.first == 1 || d.bytes == 0 ) continue;
			CK( cudaMemcpyAsync( d.p, find( x.first, d.bytes ), d.bytes, cudaMemcpyHostToDevice, net->stream ) );
		}
		for( auto const & x : ckpt_plastic( *net ) )
			if( x.second->bytes )
				CK( cudaMemcpyAsync( x.second->p, find( x.first, x.second->bytes ), x.second->bytes, cudaMemcpyHostToDevice, net->stream ) );
		summaries_from_ring( *net ); // slotted nets: the summaries of the restored ring
		CK( cudaStreamSynchronize( net->stream ) );
		net->steps = net->launched = h.steps;
		net->configure();
		*out = net.release();
	} );
}

int spk_model_attrs( int model, int * num_neuron_attrs, int * num_synapse_attrs, char * types, int types_cap )
{
	return guarded( [&] {
		spk::model_traits const md = describe( model );
		if( num_neuron_attrs ) *num_neuron_attrs = md.neuron_attrs;
		if( num_synapse_attrs ) *num_synapse_attrs = md.synapse_attrs;
		if( types && types_cap > 0 )
		{
			std::strncpy( types, md.types, (size_t)types_cap - 1 );
			types[types_cap - 1] = 0;
		}
	} );
}
}

// ---------------------------------------------------------------------------------------
// Graph generation without any allocation (spk_generate_adj_list_static).
//
// Some callers cannot allocate device memory: code running inside a framework whose
// caching allocator owns the whole device (a raw cudaMalloc there steals memory the pool
// has already budgeted and can fail at an arbitrary point), and latency-critical loops
// that cannot afford the device-wide synchronisation cudaMalloc / cudaFree imply. For
// them this variant keeps the generator's connection table in a fixed device array of
// this file instead of a fresh allocation. The host side flattens the layout in
// per-thread static arrays (no heap, about 36 KiB kept off the caller's stack), and the
// table reaches the device array through kernel parameters: each launch of
// store_static_conns carries its own copy of up to STATIC_CHUNK connections, so nothing
// on the device side ever refers to host memory of the call.
// ---------------------------------------------------------------------------------------
namespace
{
constexpr int STATIC_MAX_CONNECTIONS = 1024; // 24 KiB of device memory per GPU, held until exit
constexpr int STATIC_MAX_POPULATIONS = 1024;

__device__ __align__( 256 ) spk::conn_dev g_static_conns[STATIC_MAX_CONNECTIONS];

// device address of g_static_conns, looked up once per device (host code may not use the
// symbol itself: on the host it is only a stand-in, not a device address)
constexpr int MAX_DEVICES = 64;
void * g_static_conns_ptr[MAX_DEVICES] = {};
std::mutex g_static_mutex;

// a piece of the connection table, passed by value as a kernel parameter (3 KiB, inside
// the 4 KiB parameter space of every launch)
constexpr int STATIC_CHUNK = 128;
struct static_chunk
{
	spk::conn_dev c[STATIC_CHUNK];
};
__global__ void store_static_conns( static_chunk chunk, int offset, int count, spk::conn_dev * dst )
{
	int const i = threadIdx.x;
	if( i < count ) dst[offset + i] = chunk.c[i];
}

void * static_conns_address( int device )
{
	require( device >= 0 && device < MAX_DEVICES, "device index out of range" );
	std::lock_guard<std::mutex> lock( g_static_mutex );
	if( !g_static_conns_ptr[device] )
	{
		void * p = nullptr;
		CK( cudaGetSymbolAddress( &p, g_static_conns ) );
		g_static_conns_ptr[device] = p;
	}
	return g_static_conns_ptr[device];
}
} // namespace

extern "C" int spk_generate_adj_list_static( void * stream, spk_layout_desc const * d, uint64_t seed, int32_t * d_edges )
{
	return guarded( [&] {
		require( d != nullptr, "layout descriptor is null" );
		require( d->npops > 0 && d->pops, "layout must contain at least 1 (non-empty) population" );
		require( d->npops <= STATIC_MAX_POPULATIONS, "spk_generate_adj_list_static: at most 1024 populations" );
		require( d->nconn >= 0 && d->nconn <= STATIC_MAX_CONNECTIONS, "spk_generate_adj_list_static: at most 1024 connections" );
		require( d->nconn == 0 || ( d->conn_src && d->conn_dst && d->conn_p ), "bad connection arrays" );

		// the layout, flattened exactly as spice::util::layout does, in per-thread arrays
		static thread_local unsigned long long first[STATIC_MAX_POPULATIONS + 1];
		static thread_local int order[STATIC_MAX_CONNECTIONS];
		static thread_local spk::conn_dev table[STATIC_MAX_CONNECTIONS];
		first[0] = 0;
		for( int i = 0; i < d->npops; i++ )
		{
			require( d->pops[i] > 0 && d->pops[i] <= (uint64_t)INT_MAX, "invalid population size" );
			first[i + 1] = first[i] + d->pops[i];
		}
		require( first[d->npops] <= (unsigned long long)INT_MAX, "too many neurons" );
		for( int i = 0; i < d->nconn; i++ )
		{
			require( d->conn_src[i] >= 0 && d->conn_src[i] < d->npops && d->conn_dst[i] >= 0 && d->conn_dst[i] < d->npops,
			         "invalid index in connections matrix" );
			require( d->conn_p[i] >= 0.0f && d->conn_p[i] <= 1.0f, "invalid connect. prob." );
			order[i] = i;
		}
		auto less = [&]( int a, int b ) {
			return d->conn_src[a] < d->conn_src[b] || ( d->conn_src[a] == d->conn_src[b] && d->conn_dst[a] < d->conn_dst[b] );
		};
		for( int i = 1; i < d->nconn; i++ ) // insertion sort: no temporary buffer
			for( int j = i; j > 0 && less( order[j], order[j - 1] ); j-- ) std::swap( order[j], order[j - 1] );
		for( int i = 1; i < d->nconn; i++ )
			require( less( order[i - 1], order[i] ), "no duplicate edges in connections list allowed" );

		for( int i = 0; i < d->nconn; i++ )
		{
			int const c = order[i], s = d->conn_src[c], t = d->conn_dst[c];
			table[i] = { (int)first[s], (int)first[s + 1], (int)first[t], (int)first[t + 1], bernoulli_threshold( d->conn_p[c] ) };
		}
		// width: mean + 3 sigma of the busiest source population, rounded up to 32
		size_t widest = 0;
		double mean = 0.0, var = 0.0;
		int src = d->nconn ? table[0].src_first : 0;
		for( int i = 0; i < d->nconn; i++ )
		{
			if( table[i].src_first != src )
			{
				widest = std::max( widest, static_cast<size_t>( mean + 3 * std::sqrt( var ) ) );
				src = table[i].src_first;
				mean = var = 0.0;
			}
			double const range = static_cast<double>( table[i].dst_last - table[i].dst_first );
			float const p = d->conn_p[order[i]];
			mean += range * p;
			var += range * p * ( 1.0 - p );
		}
		widest = std::max( widest, static_cast<size_t>( mean + 3 * std::sqrt( var ) ) );
		long long const n = (long long)first[d->npops], w = (long long)( ( widest + 31 ) / 32 * 32 );
		require( d_edges != nullptr || n * w == 0, "edges pointer is null" );
		if( n * w == 0 ) return;

		int device = 0;
		CK( cudaGetDevice( &device ) );
		void * conns = static_conns_address( device );
		cudaStream_t const s = static_cast<cudaStream_t>( stream );
		// the table in pieces of STATIC_CHUNK connections, each launch holding its own copy
		for( int o = 0; o < d->nconn; o += STATIC_CHUNK )
		{
			static_chunk chunk{};
			int const count = std::min( STATIC_CHUNK, d->nconn - o );
			std::memcpy( chunk.c, table + o, (size_t)count * sizeof( spk::conn_dev ) );
			store_static_conns<<<1, STATIC_CHUNK, 0, s>>>( chunk, o, count, static_cast<spk::conn_dev *>( conns ) );
			CK( cudaGetLastError() );
		}
		int const blocks = (int)( ( n * 32 + 255 ) / 256 );
		spk::generate_ell<<<blocks, 256, 0, s>>>( (int)n, (int)w, d->nconn, static_cast<spk::conn_dev const *>( conns ), seed, d_edges );
		CK( cudaGetLastError() );
	} );
}

extern "C" {
int spk_net_set_producer_warps( spk_net * net, int warps )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		require( warps >= spk::FLAT_MIN_PRODUCERS && warps <= spk::FLAT_MAX_PRODUCERS, "producer warps must be 4 to 24" );
		device_guard g( net->device );
		net->flush(); // launches already queued keep the split they were captured with
		net->producers = warps;
		if( net->graph ) cudaGraphExecDestroy( net->graph ); // captured the old parameters
		net->graph = nullptr;
	} );
}

int spk_net_set_tile_target( spk_net * net, int target )
{
	return guarded( [&] {
		require( net != nullptr, "net is null" );
		require( target >= 1, "tile target must be >= 1" );
		device_guard g( net->device );
		retile( *net, target );
	} );
}

int spk_batch_create( spk_batch ** out, int device )
{
	return guarded( [&] {
		require( out != nullptr, "out is null" );
		int ndev = 0;
		CK( cudaGetDeviceCount( &ndev ) );
		require( device >= 0 && device < ndev, "invalid device" );
		device_guard g( device );
		auto b = std::make_unique<spk_batch>();
		b->device = device;
		for( auto & g : b->groups )
		{
			int least = 0, greatest = 0;
			CK( cudaDeviceGetStreamPriorityRange( &least, &greatest ) );
			CK( cudaStreamCreateWithPriority( &g.stream, cudaStreamNonBlocking, least ) );
			CK( cudaEventCreateWithFlags( &g.ev, cudaEventDisableTiming ) );
		}
		*out = b.release();
	} );
}

int spk_batch_add( spk_batch * b, spk_net * net )
{
	return guarded( [&] {
		require( b != nullptr && net != nullptr, "null argument" );
		require( net->device == b->device, "the net lives on another device" );
		require( net->batch == nullptr, "the net belongs to a batch already" );
		// window_flat's batched launches have one shared-memory size (plastic launches take
		// theirs from their nets)
		if( net->flat )
			for( auto * o : b->nets )
				require( !o->flat || ( o->flat_smem == net->flat_smem && o->slot_smem == net->slot_smem ),
				         "nets of a batch share one kernel configuration" );
		b->nets.push_back( net );
		net->batch = b;
	} );
}

int spk_batch_remove( spk_batch * b, spk_net * net )
{
	return guarded( [&] {
		require( b != nullptr && net != nullptr, "null argument" );
		require( net->batch == b, "the net is not in the batch" );
		detach( b, net );
	} );
}

int spk_batch_run( spk_batch * b, uint64_t nsteps )
{
	return guarded( [&] {
		require( b != nullptr, "batch is null" );
		device_guard g( b->device );
		b->run( b->nets, std::vector<unsigned long long>( b->nets.size(), nsteps ) );
	} );
}

int spk_batch_run_nets( spk_batch * b, int count, spk_net * const * nets, uint64_t const * nsteps )
{
	return guarded( [&] {
		require( b != nullptr, "batch is null" );
		require( count >= 0 && ( count == 0 || ( nets && nsteps ) ), "bad net arrays" );
		std::vector<spk_net *> which( nets, nets + count );
		for( auto * n : which ) require( n != nullptr && n->batch == b, "a net is not in the batch" );
		std::vector<spk_net *> sorted = which;
		std::sort( sorted.begin(), sorted.end() );
		require( std::adjacent_find( sorted.begin(), sorted.end() ) == sorted.end(), "a net is listed twice" );
		device_guard g( b->device );
		b->run( which, std::vector<unsigned long long>( nsteps, nsteps + count ) );
	} );
}

int spk_batch_destroy( spk_batch * b )
{
	return guarded( [&] {
		if( !b ) return;
		device_guard g( b->device );
		for( auto & gr : b->groups ) cudaStreamSynchronize( gr.stream );
		delete b;
	} );
}
}
