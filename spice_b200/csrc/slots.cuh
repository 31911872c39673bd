// Window kernel over fixed slots (non-plastic models with input classes), the step
// pipeline of window_flat with fewer, aligned requests per step.
//
// Data layout ("slots"). Every (source row, tile with inputs) pair owns one fixed slot of
// S 16-byte vectors (S = 2, 4 or 8: the smallest power of two that holds the net's longest
// slice) at slots[(src * tin + ti) * S]: the row's targets inside the tile as 10-bit
// counter indices class(src) * span + (target - d0), twelve to a vector (three per 32-bit
// word, pad 0x3FF), and the slice length in the two spare top bits of the first vector's
// four words. A tile finds the slice of a spiking source from the source's id alone, so
// the per-(source, tile) records of window_flat (one more dependent load per arrival) are
// gone, and a slot of 128 bytes is one aligned line. Rows stay source-major: the tiles'
// slots of one row are one contiguous stretch, fetched from DRAM once.
//
// Spike summaries. Besides the ring of spike ids, every tile writes per step one 128-byte
// record { count, first 31 ids } (the `summ` ring). A tile reads the first 16 bytes of
// every source tile's record of a step (count and three ids: all of a tile of 511
// receiving neurons in almost every step) and, a step later, the rest of the records of
// the few tiles that fired more, instead of per-source-tile counts and then every id.
//
// Pipeline (tiles with inputs). While the consumer warps count step k, the producer warps
//   - load the record heads of step k + 3 and the rest of step k + 2's records, then lay
//     out step k + 2's arrivals (a place per source tile from one shared atomic, then its
//     ids: the order of a step's arrivals does not change its integer counts),
//   - copy the slots of step k + 1's arrivals into the slot ring, right after step k's,
// and the publisher warp compacts step k - 1 into the spike ring and its record, publishing
// it (fence, then the tile's flag) every P = min(4, delay - 5) steps, and, when the records
// the producers load next are not yet known to be published, waits for several steps at
// once. The consumers count every slot with up to S threads, each slot's length (in its
// first vector) telling which vectors hold indices. A step whose arrivals and the previous
// step's do not fit the ring together, or a source tile with more than 31 spikes, runs
// alone: its ids from the spike ring, its slots in pieces of a whole ring; the pipeline
// restarts after it. Persistent runs need delay >= 6 (the nets use it from delay 7): every
// wait then targets a step that every tile at the waiting tile's step or later has
// published.
#pragma once

#include "flat.cuh"

namespace spk
{
constexpr int SLOT_PRODUCERS = 8; // producer warps, the publisher warp included (the last)
constexpr int SUM_W = 32;         // ints per summary record: count + first 31 ids
constexpr int SLOT_MIN_ECAP = 64; // arrivals per step a ring half holds at least
constexpr int SLOT_MAX_ECAP = 1024;

// the slice length kept in the spare bits of a slot's first vector
__host__ __device__ __forceinline__ unsigned slot_len( uint4 v )
{
	return ( v.x >> 30 ) | ( ( v.y >> 30 ) << 2 ) | ( ( v.z >> 30 ) << 4 ) | ( ( v.w >> 30 ) << 6 );
}

// Shared-memory layout of a window_slots CTA with inputs, after the fixed part of
// window_flat (state, fired bits, counters): summaries [2][ntiles][SUM_W], spare
// [ntiles + 1], entry lists [2][2 ecap] (source ids) and the slot ring [2 ecap][S] vectors.
struct slot_geom
{
	size_t sum, soff, ent, vl, ring;
	int ecap;
};
__host__ __device__ inline slot_geom slot_layout( int classes, int attrs, int span, int ntiles, int S, int smem_bytes )
{
	slot_geom g{};
	size_t b = flat_state_bytes( attrs, span ) + (size_t)classes * span * 4;
	b = ( b + 15 ) & ~(size_t)15;
	g.sum = b;
	b += (size_t)2 * ntiles * SUM_W * 4;
	g.soff = b;
	b += ( ( (size_t)ntiles + 1 ) * 4 + 15 ) & ~(size_t)15;
	long long const per = 4LL * 4 + 2LL * S * 16; // bytes per arrival of capacity
	long long const room = (long long)smem_bytes - (long long)b - 64;
	int ecap = room > 0 ? (int)( room / per ) : 0;
	ecap = ecap > SLOT_MAX_ECAP ? SLOT_MAX_ECAP : ecap & ~7;
	g.ecap = ecap;
	g.ent = b;
	b += (size_t)2 * ( 2 * ecap ) * 4; // two lists of 2 ecap ids
	b = ( b + 15 ) & ~(size_t)15;
	g.vl = b;
	g.ring = b;
	return g;
}
// the end of a window_slots CTA's shared memory (the slot ring's end)
__host__ __device__ inline size_t slot_layout_end( slot_geom const & g, int S ) { return g.ring + (size_t)2 * g.ecap * S * 16; }

// ------------------------------------------------------------------------------------
// building the slots (once per net)
// ------------------------------------------------------------------------------------
// longest (source, tile) slice of the net, from the pivots
__global__ void slice_max( int n, int ntiles, unsigned const * pivots, unsigned * out )
{
	unsigned m = 0;
	long long const total = (long long)n * ntiles;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x )
	{
		long long const src = e / ntiles, j = e % ntiles;
		unsigned const * pv = pivots + src * ( ntiles + 1 ) + j;
		m = max( m, pv[1] - pv[0] );
	}
	for( int o = 16; o; o >>= 1 ) m = max( m, __shfl_xor_sync( 0xffffffffu, m, o ) );
	if( ( threadIdx.x & 31 ) == 0 && m ) atomicMax( out, m );
}

// one warp per source row: every input tile's slot (indices, pads, the length bits)
template <typename Model>
__global__ void __launch_bounds__( 256 ) slot_fill(
    int n, int width, int ntiles, int const * edges, unsigned const * pivots, int const * tile_first, int const * tile_in, int tin, int S,
    uint4 * slots )
{
	using N = typename Model::neuron;
	snn_info const info{ n };
	int const warp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( warp >= n ) return;
	int const src = warp;
	int const cls = N::input_class( src, info );
	int const * row = edges + (long long)src * width;
	unsigned const * pv = pivots + (long long)src * ( ntiles + 1 );
	int const words = 4 * S;
	for( int j = 0; j < ntiles; j++ )
	{
		int const ti = tile_in[j];
		if( ti < 0 ) continue;
		int const d0 = tile_first[j], span = tile_first[j + 1] - d0;
		unsigned const lo = pv[j], len = pv[j + 1] - lo;
		unsigned * out = reinterpret_cast<unsigned *>( slots + ( (long long)src * tin + ti ) * S );
		for( int w = lane; w < words; w += 32 )
		{
			unsigned word = 0;
			for( int f = 0; f < 3; f++ )
			{
				int const e = 3 * w + f;
				unsigned const x = e < (int)len ? (unsigned)( cls * span + ( row[lo + e] - d0 ) ) : SLICE_PAD10;
				word |= x << ( 10 * f );
			}
			if( w < 4 ) word |= ( ( len >> ( 2 * w ) ) & 3u ) << 30;
			out[w] = word;
		}
	}
}

// barrier of the producer warps (SLOT_PRODUCERS - 1 warps before the publisher warp)
__device__ __forceinline__ void bar_sync_slot_producers() { asm volatile( "bar.sync 3, %0;\n" ::"r"( 32 * ( SLOT_PRODUCERS - 1 ) ) : "memory" ); }

// ------------------------------------------------------------------------------------
// window kernel
// ------------------------------------------------------------------------------------
template <typename Model>
__device__ __forceinline__ void window_slots_body( net_params const & p, int const tile, int L, float dt, int smem_bytes )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	constexpr int C = N::input_classes;
	static_assert( C >= 1, "window_slots needs a model with input classes" );
	constexpr int DT_AHEAD = MAX_WINDOW / 2;

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	// per step s (index s & 7): arrivals, too large for the pipeline; per ring half: vectors
	__shared__ long long s_known; // latest step every tile has published (the publisher's cache)
	// per parity of a step: its arrivals and vectors (counted with shared atomics: the order
	// of a step's arrivals does not change its integer counts), a source tile with more ids
	// than its record holds
	__shared__ int ecnt[4], eover[4], rbase[4], bigf[4];

	int const tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	int const nwc = nw - SLOT_PRODUCERS, ncons = nwc * 32;
	int const d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	int const words = ( span + 31 ) >> 5;
	int const ti = __ldg( p.tile_in + tile ); // this tile's index among the tiles with inputs
	bool const inputs = ti >= 0;
	int const S = p.slot_vecs;
	snn_info const info{ p.n };

	unsigned char * state = smem;
	unsigned * bits2 = reinterpret_cast<unsigned *>( state + (size_t)N::size * span * 4 );
	unsigned * cnt = bits2 + 2 * words;
	slot_geom const g = slot_layout( C, (int)N::size, span, p.ntiles, S, smem_bytes );
	int * sum = reinterpret_cast<int *>( smem + g.sum );                      // [2][ntiles][SUM_W]
	int * ent = reinterpret_cast<int *>( smem + g.ent );                      // [2][2 ecap]
	uint4 * const ring = reinterpret_cast<uint4 *>( smem + g.ring );          // [2][ecap][S]
	int const ecap = g.ecap;

	if( tid == 0 )
	{
		clock_state const cs = *p.clock;
		float c = cs.c, sm = cs.sum;
		for( int k = 0; k < min( L, DT_AHEAD ); k++ )
		{
			s_dt[k % MAX_WINDOW] = kahan_add( c, sm, dt );
			if( tile == 0 ) p.dt_ring[( cs.step + k ) % DT_RING] = s_dt[k % MAX_WINDOW];
		}
		s_t0 = cs.step;
		s_c = c;
		s_sum = sm;
	}
	__syncthreads();
	long long const t0 = s_t0;
	auto advance_clock = [&]( int k ) {
		int const ka = k + DT_AHEAD;
		if( tid == 0 && ka < L )
		{
			float c = s_c, sm = s_sum;
			float const d = kahan_add( c, sm, dt );
			s_dt[ka % MAX_WINDOW] = d;
			s_c = c;
			s_sum = sm;
			if( tile == 0 ) p.dt_ring[( t0 + ka ) % DT_RING] = d;
		}
	};
	smem_state<N>::from_global( p.attr, d0, span, state );
	if( inputs )
		for( int x = tid; x < C * span; x += nt ) cnt[x] = 0;
	__syncthreads();

	auto update = [&]( int k, int nws ) {
		long long const t = t0 + k;
		bool const arrivals = inputs && t >= p.delay;
		unsigned * bits = bits2 + ( k & 1 ) * words;
		float const dtk = s_dt[k % MAX_WINDOW];
		for( int base = warp * 32; base < span; base += nws * 32 )
		{
			int const local = base + lane;
			bool fired = false;
			if( local < span )
			{
				Tup st;
				smem_state<N>::load( st, state, span, local );
				uint32_t const i = (uint32_t)( d0 + local );
				reg_iter<Tup> it{ st, i };
				if( arrivals )
#pragma unroll
					for( int c = 0; c < C; c++ )
					{
						unsigned const m = cnt[c * span + local];
						if( m )
						{
							cnt[c * span + local] = 0u;
							repeat_backend rb( p.seed, i, (uint32_t)t, m );
							N::receive( N::class_source( c, info ), it, null_syn_iter{}, info, rb );
						}
					}
				device_backend bak( p.seed, i, (uint32_t)t );
				fired = N::update( it, dtk, info, bak );
				smem_state<N>::store( st, state, span, local );
			}
			unsigned const word = __ballot_sync( 0xffffffffu, fired );
			if( lane == 0 ) bits[base >> 5] = word;
		}
	};
	auto compact = [&]( int k, bool publish = true ) { compact_step( p, bits2 + ( k & 1 ) * words, words, d0, tile, t0 + k, lane, publish ); };

	if( !inputs )
	{
		// no arrivals: every warp updates, the last warp compacts the step before while the
		// others update the next one (its bits are in the other half)
		for( int k = 0; k < L; k++ )
		{
			advance_clock( k );
			update( k, nw );
			__syncthreads();
			if( warp == nw - 1 )
			{
				warp_wait_all_published( p, t0 + k - p.delay );
				compact( k );
			}
		}
		__syncthreads();
	}
	else
	{
		// every index of the E slots from ring slot `b0` on (wrapping around the ring of R
		// slots), T threads per slot (T a power of two: as many as the threads allow, at most
		// S): a slot's length (its first vector) tells how many vectors hold indices
		auto count_slots = [&]( int b0, int E, int t, int nthr ) {
			if( E <= 0 ) return;
			int lt = 0;
			while( ( 1 << lt ) < S && ( 2 << lt ) * E <= nthr ) lt++;
			int const T = 1 << lt, RR = 2 * ecap;
#pragma unroll 1
			for( int x = t; x < E * T; x += nthr )
			{
				int const e = x >> lt, h = x & ( T - 1 );
				int r = b0 + e;
				if( r >= RR ) r -= RR;
				uint4 const * sl = ring + (size_t)r * S;
				int const nv = min( S, (int)( slot_len( sl[0] ) + 11 ) / 12 );
				for( int v = h; v < nv; v += T ) count_vector<12>( cnt, sl[v] );
			}
		};
		// publication every P steps (each publication covers the steps before it)
		int const P = min( 4, p.delay - 5 );
		auto compact_lazy = [&]( int k ) { compact( k, ( ( t0 + k ) % P ) == P - 1 || k == L - 1 ); };
		int const R = 2 * ecap; // the slot ring: consecutive steps' arrivals follow each other
		int k = 0;
		while( k < L )
		{
			int const kb = k; // the pipeline (re)starts at step kb
			// producer work during step j (the prologue: j < kb, every thread): threads
			// [0, npt) of numbering pt; `all` when every warp of the CTA takes part
			auto produce = [&]( int j, int pt, int npt, bool all ) {
				int const s3 = j + 3, sa = j + 2, sb = j + 1;
				bool const do_sa = sa >= kb && sa < L;
				// step sb's place in the ring: after step j's arrivals (none before kb); too
				// many arrivals for the ring, or more ids than a record holds: the step runs alone
				int const eb = ecnt[sb & 3];
				int const prev = sb > kb ? ecnt[j & 3] : 0;
				int const base = sb > kb ? ( rbase[j & 3] + prev ) % R : 0;
				bool const big = eover[sb & 3] || eb + prev > R;
				bool const do_a = sb >= kb && sb < L && !big;
				if( pt == 0 )
				{
					bigf[sb & 3] = big;
					rbase[sb & 3] = base;
					ecnt[sa & 3] = 0;
					eover[sa & 3] = 0;
				}
				// the first 16 bytes (count, three ids) of every summary record of step s3 (none
				// before `delay`); in the prologue every thread first waits for the step's
				// publication (later steps: checked by the publisher warp ahead of time)
				if( s3 >= kb && s3 < L )
				{
					long long const t = t0 + s3;
					int * sd = sum + ( s3 & 1 ) * p.ntiles * SUM_W;
					if( t >= p.delay )
					{
						int const * src = p.summ + ( ( t - p.delay ) % p.ring ) * (long long)p.ntiles * SUM_W;
						for( int i = pt; i < p.ntiles; i += npt )
						{
							if( all ) wait_published( p, i, t - p.delay );
							cp_async16( sd + i * SUM_W, src + i * SUM_W );
						}
					}
					else
						for( int i = pt; i < p.ntiles; i += npt ) sd[i * SUM_W] = 0;
				}
				// the rest of the records of step sa whose tile fired more than three neurons
				if( do_sa && t0 + sa >= p.delay )
				{
					int * sd = sum + ( sa & 1 ) * p.ntiles * SUM_W;
					int const * src = p.summ + ( ( t0 + sa - p.delay ) % p.ring ) * (long long)p.ntiles * SUM_W;
					for( int i = pt; i < p.ntiles; i += npt )
					{
						int const need = min( SUM_W, sd[i * SUM_W] + 1 ); // ints of the record in use
						for( int v = 4; v < need; v += 4 ) cp_async16( sd + i * SUM_W + v, src + i * SUM_W + v );
					}
				}
				// the slots of step sb's arrivals, S lanes per arrival
				if( do_a )
				{
					int const * es = ent + ( sb & 1 ) * ecap * 2;
					int const q = pt % S, groups = npt / S;
					for( int e = pt / S; e < eb; e += groups )
					{
						int r = base + e;
						if( r >= R ) r -= R;
						cp_async16( ring + (size_t)r * S + q, p.slots + ( (long long)es[e] * p.tin + ti ) * S + q );
					}
				}
				cp_async_commit();
				cp_async_wait_all();
				if( all )
					__syncthreads();
				else
					bar_sync_slot_producers();
				// step sa's arrivals: a place in its entry list per source tile from one shared
				// atomic (the order of a step's arrivals does not change its integer counts),
				// then the tile's ids
				if( do_sa )
				{
					int const * sd = sum + ( sa & 1 ) * p.ntiles * SUM_W;
					int * es = ent + ( sa & 1 ) * ecap * 2;
					for( int i = pt; i < p.ntiles; i += npt )
					{
						int const c = sd[i * SUM_W];
						if( c == 0 ) continue;
						if( c > SUM_W - 1 ) eover[sa & 3] = 1; // more ids than the record holds
						int const o = atomicAdd( &ecnt[sa & 3], c );
						int const cc = min( c, SUM_W - 1 );
						for( int r = 0; r < cc && o + r < R; r++ ) es[o + r] = sd[i * SUM_W + 1 + r];
					}
				}
			};

			int ks = L; // a step for the synchronous path, if any
			if( !p.flat_sync )
			{
				for( int j = kb - 3; j < kb; j++ )
				{
					produce( j, tid, nt, true );
					__syncthreads();
				}
				// the publication of the step whose summaries the producers load during step
				// kb (later ones: checked by the publisher warp ahead of time)
				if( kb + 3 < L && t0 + kb + 3 >= p.delay )
					for( int i = tid; i < p.ntiles; i += nt ) wait_published( p, i, t0 + kb + 3 - p.delay );
				if( tid == 0 ) s_known = t0 + kb + 3 - p.delay;
				__syncthreads();
				for( ; k < L; k++ )
				{
					if( bigf[k & 3] )
					{
						ks = k; // this step takes the synchronous path
						break;
					}
					advance_clock( k );
					if( warp < nwc )
					{
						if( t0 + k >= p.delay ) count_slots( rbase[k & 3], ecnt[k & 3], tid, ncons );
						bar_sync_first( ncons ); // counts complete
						update( k, nwc );
					}
					else if( warp == nw - 1 )
					{
						// the publisher warp: step k - 1's spikes and summary (published every P
						// steps, fenced); then, when the summaries the producers load next step
						// are not known to be published, a wait for several steps at once
						if( k > kb ) compact_lazy( k - 1 );
						long long const need = t0 + k + 4 - p.delay;
						if( k + 4 < L && need >= 0 && need > s_known )
						{
							long long const demand = min( t0 + k - P - 1, need + 7 );
							warp_wait_all_published( p, demand );
							if( lane == 0 ) s_known = demand;
						}
					}
					else
						produce( k, tid - ncons, nt - ncons - 32, false );
					__syncthreads(); // step k updated, step k + 1's slots in the ring
				}
				if( k > kb && warp == nw - 1 ) compact( k - 1 ); // the last pipelined step, published
				__syncthreads();
			}
			else
				ks = k;
			if( ks >= L ) break;

			// ------------------------------------------------------------ the synchronous path
			// step ks alone: its arrivals' ids from the spike ring, their slots in pieces of up
			// to a whole ring (both halves), each counted before the next is copied
			advance_clock( ks );
			long long const t = t0 + ks;
			if( t >= p.delay )
			{
				int const slot_in = (int)( ( t - p.delay ) % p.ring );
				int * pref = sum; // [ntiles + 1] per-source-tile prefix of the step's spikes
				for( int i = tid; i < p.ntiles; i += nt ) wait_published( p, i, t - p.delay );
				__syncthreads();
				int running = 0;
				for( int base = 0; base < p.ntiles; base += nt )
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
				int const M = running, R = 2 * ecap;
				for( int b0 = 0; b0 < M; b0 += R )
				{
					int const m = min( R, M - b0 );
					for( int x = tid; x < m; x += nt )
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
						uint4 const * from = p.slots + ( (long long)src * p.tin + ti ) * S;
						for( int v = 0; v < S; v++ ) cp_async16( ring + (size_t)x * S + v, from + v );
					}
					cp_async_commit();
					cp_async_wait_all();
					__syncthreads();
					count_slots( 0, m, tid, nt );
					__syncthreads();
				}
			}
			__syncthreads();
			update( ks, nw );
			__syncthreads();
			if( warp == nw - 1 ) compact( ks );
			__syncthreads();
			k = ks + 1;
		}
	}

	smem_state<N>::to_global( p.attr, d0, span, state );
	window_clock_end( p, L, t0, s_c, s_sum );
}

template <typename Model>
__global__ void __launch_bounds__( FLAT_THREADS, 1 ) window_slots( net_params p, int L, float dt, int smem_bytes )
{
	window_slots_body<Model>( p, blockIdx.x, L, dt, smem_bytes );
}

// many nets of one model in one launch (batching), as window_flat_batch
template <typename Model>
__global__ void __launch_bounds__( FLAT_THREADS, 1 ) window_slots_batch( net_params const * nets, int4 const * jobs, int smem_bytes )
{
	__shared__ net_params s_p;
	int4 const j = jobs[blockIdx.x];
	if( threadIdx.x == 0 ) s_p = nets[j.x];
	__syncthreads();
	if( j.z > 0 ) window_slots_body<Model>( s_p, j.y, j.z, __int_as_float( j.w ), smem_bytes );
}
} // namespace spk

namespace spk
{
// the summary ring from the spike ring (a restored or enlarged ring): one warp per
// (slot, tile)
__global__ void summ_from_ring( int const * ring_ids, unsigned const * ring_cnt, int n, int ntiles, int slots, int const * tile_first, int * summ )
{
	long long const w = ( blockIdx.x * (long long)blockDim.x + threadIdx.x ) >> 5;
	int const lane = threadIdx.x & 31;
	if( w >= (long long)slots * ntiles ) return;
	int const s = (int)( w / ntiles ), i = (int)( w % ntiles );
	unsigned const c = ring_cnt[w];
	int * o = summ + w * SUM_W;
	int const * ids = ring_ids + (long long)s * n + tile_first[i];
	if( lane == 0 ) o[0] = (int)c;
	if( lane < SUM_W - 1 && (unsigned)lane < c ) o[1 + lane] = ids[lane];
}
} // namespace spk
