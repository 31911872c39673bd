// sm_100a kernels of the simulation path.
//
// Data layout in HBM (one net):
//   edges    int32 [n x width]      ELL rows, ascending, INT_MAX padded (the reference's
//                                   adjacency format, spice/util/adj_list.cpp:28-46)
//   pivots   uint32 [n x (ntiles+1)] pivots[src][j] = first position in row src whose
//                                   target is >= tile_first[j] (row slice of tile j)
//   attr[k]  neuron attribute k, structure of arrays
//   ring_ids int32 [2*delay x n]    spike queue: slot s holds, per tile j, the ids that
//                                   fired in tile j at a step t with t % (2 delay) == s,
//                                   ascending, in the segment [j*tile, j*tile + count)
//   ring_cnt uint32 [2*delay x ntiles]
//
// Execution: the destination neurons are cut into `ntiles` contiguous tiles
// [tile_first[j], tile_first[j + 1]), one CTA per tile. A spike fired at step t reaches its targets at step t + delay, so all the
// arrivals of the steps [t0, t0 + L) with L <= delay were fired before t0: one launch
// advances every tile by L steps with no grid-wide synchronisation inside the launch
// (the kernel boundary is the only barrier, once per window). The ring has 2*delay slots
// so that slots written inside a window never alias the slots read in it.
#pragma once

#include "device_common.cuh"

#include <spice/models/model.h>
#include <spice/snn_info.h>

#include <climits>
#include <cstdint>
#include <type_traits>

namespace spk
{
using spice::snn_info;

constexpr int MAX_ATTRS = 8;
constexpr int MAX_WINDOW = 64;  // steps per launch
constexpr int SPIKE_BATCH = 1024; // arrivals staged in shared memory at a time
constexpr int DT_RING = 128;    // per-step dt history (>= MAX_WINDOW)

enum error_bits
{
	ERR_BAD_TARGET = 1, // an edge pointed outside its tile slice (corrupt pivots/graph)
	ERR_OVERFLOW = 2,
	ERR_TIMEOUT = 4     // a wait for another tile's spikes gave up (window_flat)
};
constexpr int WAIT_LIMIT = 1 << 20; // polls of a bounded wait (about a second)

struct conn_dev
{
	int src_first, src_last, dst_first, dst_last;
	unsigned long long thr; // floor(p * 2^32)
};

struct net_params
{
	int n, width, delay, tile, ntiles, ring;
	unsigned long long seed;
	int const * edges;
	unsigned const * pivots;
	int const * tile_first; // [ntiles + 1] first neuron of every tile
	void * attr[MAX_ATTRS];
	void * syn_attr[MAX_ATTRS]; // static synapse attribute k, [n x width] parallel to edges (window_ordered)
	int * ring_ids;
	unsigned * ring_cnt;
	clock_state * clock;
	float * dt_ring;
	int * err;
	uint4 const * slices;    // tile-major slices of counter indices (window_flat)
	uint2 const * slice_rec; // [n][ntiles] { first vector, length } (window_flat)
	int const * tile_inputs; // [ntiles] 1 if the tile has incoming synapses (window_flat)
	int pack;                // indices per 16-byte slice vector: 8 (16-bit) or 12 (10-bit)
	int flat_sync;           // window_flat: every step on the synchronous path
	int producers;           // window_flat: producer warps, the publisher included (the rest count and update)
	long long * done_step;   // [ntiles] last step whose spikes the tile has published
	int wait_limit;          // polls of a bounded wait before it gives up (WAIT_LIMIT)
	int withhold_tile;       // failure-detection tests: this tile never publishes (-1: none)
	// fixed slots (window_slots): S vectors per (source, tile with inputs), the index of
	// every tile among the tiles with inputs (-1: none) and their number; spike summaries
	// [ring][ntiles][32]: count and first 31 ids of every (step, tile)
	uint4 const * slots;
	int const * tile_in;
	int tin, slot_vecs;
	int * summ;
};

template <typename T>
__device__ __forceinline__ T from_bits( int x )
{
	if constexpr( sizeof( T ) == 4 && std::is_floating_point<T>::value )
		return __int_as_float( x );
	else
		return static_cast<T>( x );
}
__device__ __forceinline__ int to_bits( float x ) { return __float_as_int( x ); }
__device__ __forceinline__ int to_bits( int x ) { return x; }

// ------------------------------------------------------------------------------------
// attribute load / store between SoA arrays and register tuples
// ------------------------------------------------------------------------------------
template <typename Decl, int I = 0>
struct attrs_io
{
	template <typename Tup>
	__device__ __forceinline__ static void load( Tup & t, void * const * a, long long i )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			tuple_at<I>::get( t ) = static_cast<T const *>( a[I] )[i];
			attrs_io<Decl, I + 1>::load( t, a, i );
		}
	}
	template <typename Tup>
	__device__ __forceinline__ static void store( Tup & t, void * const * a, long long i )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			static_cast<T *>( a[I] )[i] = tuple_at<I>::get( t );
			attrs_io<Decl, I + 1>::store( t, a, i );
		}
	}
	// four consecutive neurons with one 16-byte access per attribute
	template <typename Tup>
	__device__ __forceinline__ static void load4( Tup * t, void * const * a, long long i )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			static_assert( sizeof( T ) == 4, "attributes are 32-bit" );
			int4 const v = *reinterpret_cast<int4 const *>( static_cast<T const *>( a[I] ) + i );
			tuple_at<I>::get( t[0] ) = from_bits<T>( v.x );
			tuple_at<I>::get( t[1] ) = from_bits<T>( v.y );
			tuple_at<I>::get( t[2] ) = from_bits<T>( v.z );
			tuple_at<I>::get( t[3] ) = from_bits<T>( v.w );
			attrs_io<Decl, I + 1>::load4( t, a, i );
		}
	}
	template <typename Tup>
	__device__ __forceinline__ static void store4( Tup * t, void * const * a, long long i )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			int4 v;
			v.x = to_bits( tuple_at<I>::get( t[0] ) );
			v.y = to_bits( tuple_at<I>::get( t[1] ) );
			v.z = to_bits( tuple_at<I>::get( t[2] ) );
			v.w = to_bits( tuple_at<I>::get( t[3] ) );
			*reinterpret_cast<int4 *>( static_cast<T *>( a[I] ) + i ) = v;
			attrs_io<Decl, I + 1>::store4( t, a, i );
		}
	}
};

// ------------------------------------------------------------------------------------
// clock: every CTA derives the window's dt sequence from the clock state; the CTA that
// finishes last advances the clock (all CTAs have read it by then).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void window_clock_begin( net_params const & p, int L, float dt, float * s_dt, long long * s_t0, float * s_c, float * s_sum )
{
	if( threadIdx.x == 0 )
	{
		clock_state const cs = *p.clock;
		float c = cs.c, sum = cs.sum;
		for( int k = 0; k < L; k++ ) s_dt[k] = kahan_add( c, sum, dt );
		*s_t0 = cs.step;
		*s_c = c;
		*s_sum = sum;
		if( blockIdx.x == 0 )
			for( int k = 0; k < L; k++ ) p.dt_ring[( cs.step + k ) % DT_RING] = s_dt[k];
	}
	__syncthreads();
}

// Publication of a tile's spikes (window_flat): after the ring entries of step t are
// written, every writer fences and the tile's flag is released; a reader acquires the flag
// before it reads the ring. A wait polls with a limit, then flags ERR_TIMEOUT and returns.
__device__ __forceinline__ void publish_step( net_params const & p, int tile, long long t )
{
	asm volatile( "st.release.gpu.global.s64 [%0], %1;" ::"l"( p.done_step + tile ), "l"( t ) : "memory" );
}
__device__ __forceinline__ long long published( net_params const & p, int i )
{
	long long v;
	asm volatile( "ld.acquire.gpu.global.s64 %0, [%1];" : "=l"( v ) : "l"( p.done_step + i ) : "memory" );
	return v;
}
__device__ __forceinline__ void wait_published( net_params const & p, int i, long long t )
{
	if( t < 0 ) return;
	for( int it = 0; published( p, i ) < t; it++ )
	{
		// after one wait has given up, every other wait of the launch returns at once
		if( it >= p.wait_limit || ( *(int volatile *)p.err & ERR_TIMEOUT ) )
		{
			atomicOr( p.err, ERR_TIMEOUT );
			return;
		}
		__nanosleep( 256 );
	}
}

// every tile has published step t: lanes of a warp read the flags of tiles lane, lane + 32,
// ... at once (relaxed), one acquire fence when all are there, else the bounded wait
__device__ __forceinline__ void warp_wait_all_published( net_params const & p, long long t )
{
	if( t < 0 ) return;
	bool ok = true;
	for( int i = threadIdx.x & 31; i < p.ntiles; i += 32 )
	{
		long long v;
		asm volatile( "ld.relaxed.gpu.global.s64 %0, [%1];" : "=l"( v ) : "l"( p.done_step + i ) : "memory" );
		ok = ok && v >= t;
	}
	if( __all_sync( 0xffffffffu, ok ) )
		asm volatile( "fence.acq_rel.gpu;" ::: "memory" );
	else
		for( int i = threadIdx.x & 31; i < p.ntiles; i += 32 ) wait_published( p, i, t );
	__syncwarp();
}

__device__ __forceinline__ void window_clock_end( net_params const & p, int L, long long t0, float c, float sum )
{
	__syncthreads();
	if( threadIdx.x == 0 )
	{
		__threadfence();
		unsigned const prev = atomicAdd( &p.clock->done, 1u );
		if( prev == (unsigned)p.ntiles - 1 ) // the net's last CTA (batched launches run several nets)
		{
			p.clock->step = t0 + L;
			p.clock->c = c;
			p.clock->sum = sum;
			p.clock->done = 0;
			__threadfence();
		}
	}
}

// The exclusive prefix over the source tiles' entry counts of ring slot `slot` (pref[0..ntiles]),
// and the slot's total.
__device__ __forceinline__ int stage_prefix( net_params const & p, unsigned const * cnt_ring, int slot, int * pref, int * scratch )
{
	int running = 0;
	for( int base = 0; base < p.ntiles; base += blockDim.x )
	{
		int const i = base + threadIdx.x;
		int const c = i < p.ntiles ? (int)cnt_ring[(long long)slot * p.ntiles + i] : 0;
		int tot;
		int const ex = block_exclusive_scan( c, scratch, &tot );
		if( i < p.ntiles ) pref[i] = running + ex;
		running += tot;
	}
	if( threadIdx.x == 0 ) pref[p.ntiles] = running;
	__syncthreads();
	return running;
}

__device__ __forceinline__ int find_tile( int const * pref, int ntiles, int g )
{
	int lo = 0, hi = ntiles;
	while( hi - lo > 1 )
	{
		int const mid = ( lo + hi ) >> 1;
		if( pref[mid] <= g )
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

// ------------------------------------------------------------------------------------
// arrivals of one step into this tile: stage (src, slice bounds, class) of up to
// SPIKE_BATCH spikes, then one warp per spike walks the row slice and bumps the
// per-(target, class) counters with shared-memory atomics.
// Returns nothing; counters `cnt` (classes x tile) must be zero on entry.
// ------------------------------------------------------------------------------------
template <typename Neuron>
__device__ __forceinline__ void deliver_counts(
    net_params const & p, int slot_in, int tile, int d0, int d1, unsigned * cnt, int * pref, int4 * sb, int * scratch )
{
	int const tid = threadIdx.x;
	snn_info const info{ p.n };

	// per-source-tile counts -> exclusive prefix (pref[0..ntiles])
	int running = 0;
	for( int base = 0; base < p.ntiles; base += blockDim.x )
	{
		int const i = base + tid;
		int const c = i < p.ntiles ? (int)p.ring_cnt[(long long)slot_in * p.ntiles + i] : 0;
		int tot;
		int const ex = block_exclusive_scan( c, scratch, &tot );
		if( i < p.ntiles ) pref[i] = running + ex;
		running += tot;
	}
	if( tid == 0 ) pref[p.ntiles] = running;
	__syncthreads();
	int const total = running;

	int const warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
	int const span = d1 - d0;
	for( int b0 = 0; b0 < total; b0 += SPIKE_BATCH )
	{
		int const m = min( SPIKE_BATCH, total - b0 );
		for( int x = tid; x < m; x += blockDim.x )
		{
			int const g = b0 + x;
			int lo = 0, hi = p.ntiles; // largest i with pref[i] <= g
			while( hi - lo > 1 )
			{
				int const mid = ( lo + hi ) >> 1;
				if( pref[mid] <= g )
					lo = mid;
				else
					hi = mid;
			}
			int const src = p.ring_ids[(long long)slot_in * p.n + __ldg( p.tile_first + lo ) + ( g - pref[lo] )];
			unsigned const * pv = p.pivots + (long long)src * ( p.ntiles + 1 ) + tile;
			sb[x] = make_int4( src, (int)__ldg( pv ), (int)__ldg( pv + 1 ), Neuron::input_class( src, info ) );
		}
		__syncthreads();
		for( int x = warp; x < m; x += nw )
		{
			int4 const e = sb[x];
			int const * row = p.edges + (long long)e.x * p.width;
			unsigned * cc = cnt + e.w * p.tile;
			for( int j = e.y + lane; j < e.z; j += 32 )
			{
				int const local = __ldg( row + j ) - d0;
				if( (unsigned)local < (unsigned)span )
					atomicAdd( cc + local, 1u );
				else
					atomicOr( p.err, ERR_BAD_TARGET );
			}
		}
		__syncthreads();
	}
}

// ------------------------------------------------------------------------------------
// the window kernel for models with input classes (non-plastic): counts -> receive replay
// -> update -> ordered spike compaction, L steps per launch.
// ------------------------------------------------------------------------------------
template <typename Model, int NPT>
__global__ void __launch_bounds__( 512, 1 ) window_counts( net_params p, int L, float dt )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	constexpr int C = N::input_classes;
	static_assert( C >= 1, "window_counts needs a model with input classes" );

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;

	int const T = p.tile;
	unsigned * cnt = reinterpret_cast<unsigned *>( smem );
	int * pref = reinterpret_cast<int *>( cnt + C * T );
	int4 * sb = reinterpret_cast<int4 *>( smem + ( ( ( C * T + p.ntiles + 1 ) * 4 + 15 ) & ~15 ) );

	int const tile = blockIdx.x, tid = threadIdx.x;
	int const d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 );
	snn_info const info{ p.n };

	window_clock_begin( p, L, dt, s_dt, &s_t0, &s_c, &s_sum );

	Tup st[NPT];
	long long const i0 = (long long)d0 + NPT * tid;
	if( NPT == 4 && i0 + 3 < d1 )
		attrs_io<N>::load4( st, p.attr, i0 );
	else
#pragma unroll
		for( int q = 0; q < NPT; q++ )
			if( i0 + q < d1 ) attrs_io<N>::load( st[q], p.attr, i0 + q );

	for( int k = 0; k < L; k++ )
	{
		long long const t = s_t0 + k;
		bool const arrivals = t >= p.delay;
		if( arrivals )
		{
			for( int x = tid; x < C * T; x += blockDim.x ) cnt[x] = 0;
			__syncthreads();
			deliver_counts<N>( p, (int)( ( t - p.delay ) % p.ring ), tile, d0, d1, cnt, pref, sb, scratch );
		}

		unsigned fired = 0;
#pragma unroll
		for( int q = 0; q < NPT; q++ )
		{
			long long const i = i0 + q;
			if( i < d1 )
			{
				reg_iter<Tup> it{ st[q], (uint32_t)i };
				device_backend bak( p.seed, (uint32_t)i, (uint32_t)t );
				if( arrivals )
#pragma unroll
					for( int c = 0; c < C; c++ )
					{
						unsigned const m = cnt[c * T + NPT * tid + q];
						if( m )
						{
							repeat_backend rb( p.seed, (uint32_t)i, (uint32_t)t, m );
							N::receive( N::class_source( c, info ), it, null_syn_iter{}, info, rb );
						}
					}
				if( N::update( it, s_dt[k], info, bak ) ) fired |= 1u << q;
			}
		}

		int total;
		int off = block_exclusive_scan( __popc( fired ), scratch, &total );
		int const slot_out = (int)( t % p.ring );
		int * out = p.ring_ids + (long long)slot_out * p.n + d0;
#pragma unroll
		for( int q = 0; q < NPT; q++ )
			if( ( fired >> q ) & 1u ) out[off++] = (int)( i0 + q );
		if( tid == 0 ) p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)total;
	}

	if( NPT == 4 && i0 + 3 < d1 )
		attrs_io<N>::store4( st, p.attr, i0 );
	else
#pragma unroll
		for( int q = 0; q < NPT; q++ )
			if( i0 + q < d1 ) attrs_io<N>::store( st[q], p.attr, i0 + q );

	window_clock_end( p, L, s_t0, s_c, s_sum );
}

// ------------------------------------------------------------------------------------
// graph generation: one warp per row, Bernoulli trials from Philox, warp-scan compaction
// keeps rows ascending; truncation at `width`; INT_MAX padding with 16-byte stores.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__( 256 ) generate_ell( int n, int width, int nconn, conn_dev const * conns, unsigned long long seed, int * edges )
{
	int const warp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( warp >= n ) return;
	int const src = warp;
	int * row = edges + (long long)src * width;
	uint32_t const k0 = (uint32_t)seed, k1 = (uint32_t)( seed >> 32 );
	int k = 0;
	for( int ci = 0; ci < nconn && k < width; ci++ )
	{
		conn_dev const c = conns[ci];
		if( src < c.src_first || src >= c.src_last ) continue;
		int const range = c.dst_last - c.dst_first;
		for( int base = 0; base < range && k < width; base += 128 )
		{
			int const j0 = base + 4 * lane;
			unsigned bits = 0;
			if( j0 < range )
			{
				u32x4 const r = philox4x32_10( { (uint32_t)src, (uint32_t)( j0 >> 2 ), (uint32_t)ci, TAG_GRAPH }, k0, k1 );
				bits = ( (unsigned long long)r.x < c.thr ? 1u : 0u ) | ( ( j0 + 1 < range && (unsigned long long)r.y < c.thr ) ? 2u : 0u ) |
				       ( ( j0 + 2 < range && (unsigned long long)r.z < c.thr ) ? 4u : 0u ) |
				       ( ( j0 + 3 < range && (unsigned long long)r.w < c.thr ) ? 8u : 0u );
			}
			int const cntl = __popc( bits );
			int const incl = warp_inclusive_scan( cntl );
			int pos = k + incl - cntl;
#pragma unroll
			for( int q = 0; q < 4; q++ )
				if( ( bits >> q ) & 1u )
				{
					if( pos < width ) row[pos] = c.dst_first + j0 + q;
					pos++;
				}
			k = min( width, k + __shfl_sync( 0xffffffffu, incl, 31 ) );
		}
	}
	// padding: scalar up to a 4-aligned position, then int4 stores
	int const a = min( width, ( k + 3 ) & ~3 );
	if( lane < a - k ) row[k + lane] = INT_MAX;
	int4 const pad = make_int4( INT_MAX, INT_MAX, INT_MAX, INT_MAX );
	for( int e = a + 4 * lane; e < width; e += 128 ) *reinterpret_cast<int4 *>( row + e ) = pad;
}

// pivots[src][j] = lower_bound(row src, tile_first[j]) for j = 0..ntiles; one warp per row.
__global__ void __launch_bounds__( 256 ) build_pivots( int n, int width, int const * tile_first, int ntiles, int const * edges, unsigned * pivots )
{
	int const warp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( warp >= n ) return;
	int const * row = edges + (long long)warp * width;
	unsigned * out = pivots + (long long)warp * ( ntiles + 1 );
	for( int j = lane; j <= ntiles; j += 32 )
	{
		long long const key = tile_first[j];
		int lo = 0, hi = width; // first position with row[pos] >= key
		while( lo < hi )
		{
			int const mid = ( lo + hi ) >> 1;
			if( (long long)__ldg( row + mid ) >= key )
				hi = mid;
			else
				lo = mid + 1;
		}
		out[j] = (unsigned)lo;
	}
}

// neuron::init for all neurons
template <typename Model>
__global__ void init_neurons( net_params p )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	snn_info const info{ p.n };
	for( long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < p.n; i += (long long)gridDim.x * blockDim.x )
	{
		Tup t{};
		reg_iter<Tup> it{ t, (uint32_t)i };
		device_backend bak( p.seed, (uint32_t)i, 0xFFFFFFFFu );
		N::init( it, info, bak );
		attrs_io<N>::store( t, p.attr, i );
	}
}

// spikes per step of the `count` steps just simulated (the clock already advanced past
// them): totals[k] = sum over tiles of the step's ring counts; one warp per step
__global__ void raster_totals( unsigned const * ring_cnt, int ntiles, int ring, clock_state const * clock, int count, unsigned * totals )
{
	int const k = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( k >= count ) return;
	long long const t0 = clock->step - count;
	int const slot = (int)( ( t0 + k ) % ring );
	unsigned c = 0;
	for( int i = lane; i < ntiles; i += 32 ) c += ring_cnt[(long long)slot * ntiles + i];
	for( int o = 16; o > 0; o >>= 1 ) c += __shfl_xor_sync( ~0u, c, o );
	if( lane == 0 ) totals[k] = c;
}

// Dense raster of the `count` steps just simulated: step k's spikes (ascending: tiles in
// order, each tile's ids ascending) go to out_ids at cursor + (spikes of steps < k); the
// last block advances the cursor. totals = raster_totals of the same steps.
__global__ void gather_raster(
    int const * ring_ids,
    unsigned const * ring_cnt,
    int n,
    int const * tile_first,
    int ntiles,
    int ring,
    clock_state const * clock,
    int count,
    unsigned const * totals,
    unsigned long long * cursor,
    unsigned * done,
    int * out_ids,
    unsigned long long out_cap,
    int * err )
{
	__shared__ int scratch[33];
	__shared__ long long s_base;
	__shared__ long long s_off, s_grand;
	int const k = blockIdx.x, tid = threadIdx.x;
	long long const t0 = clock->step - count;
	// offset of step k = spikes of the steps before it; grand = all of them
	long long before = 0, grand = 0;
	for( int s = tid; s < count; s += blockDim.x )
	{
		long long const c = totals[s];
		grand += c;
		if( s < k ) before += c;
	}
	for( int o = 16; o > 0; o >>= 1 )
	{
		before += __shfl_xor_sync( ~0u, before, o );
		grand += __shfl_xor_sync( ~0u, grand, o );
	}
	__shared__ long long s_red[2][32];
	if( ( tid & 31 ) == 0 )
	{
		s_red[0][tid >> 5] = before;
		s_red[1][tid >> 5] = grand;
	}
	__syncthreads();
	if( tid == 0 )
	{
		long long b = 0, g = 0;
		for( int w = 0; w < (int)( blockDim.x >> 5 ); w++ )
		{
			b += s_red[0][w];
			g += s_red[1][w];
		}
		s_base = (long long)*cursor;
		s_off = b;
		s_grand = g;
	}
	__syncthreads();
	int const slot = (int)( ( t0 + k ) % ring );
	int running = 0;
	for( int base = 0; base < ntiles; base += blockDim.x )
	{
		int const i = base + tid;
		int const c = i < ntiles ? (int)ring_cnt[(long long)slot * ntiles + i] : 0;
		int tot;
		int const ex = block_exclusive_scan( c, scratch, &tot );
		long long const dst = s_base + s_off + running + ex;
		for( int r = 0; r < c; r++ )
		{
			if( (unsigned long long)( dst + r ) < out_cap )
				out_ids[dst + r] = ring_ids[(long long)slot * n + tile_first[i] + r];
			else
				atomicOr( err, ERR_OVERFLOW );
		}
		running += tot;
	}
	if( tid == 0 )
	{
		__threadfence();
		unsigned const prev = atomicAdd( done, 1u );
		if( prev == gridDim.x - 1 )
		{
			*cursor = (unsigned long long)( s_base + s_grand );
			*done = 0;
			__threadfence();
		}
	}
}

} // namespace spk
