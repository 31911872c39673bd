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
// Spike summaries. Besides the ring of spike ids, every tile publishes per step one
// 128-byte record { count, first 31 ids } (the `summ` ring). A tile reads a step's
// records of all source tiles in one burst of aligned lines instead of per-source-tile
// counts and then ids.
//
// Pipeline (tiles with inputs). While the consumer warps count step k, the producer warps
//   - load the summary records of step k + 2 and lay out its arrivals (a scan of the
//     counts, then every source tile's ids into the step's entry list),
//   - copy the slots of step k + 1's arrivals into half (k + 1) & 1 of the slot ring and,
//     once they landed, list the vectors that hold indices (from each slot's length),
// and the publisher warp compacts step k - 1 into the spike ring and its summary, fences
// and publishes it, then checks the publication of step k + 3 for the producers' next
// loads. A step with more arrivals than a ring half, or a source tile with more than 31
// spikes, takes the direct path of window_counts (ELL rows) alone; the pipeline restarts
// after it. Persistent runs need delay >= 4: every wait then targets a step before the
// waiting tile's own.
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
// window_flat (state, fired bits, counters): summaries [2][ntiles][SUM_W], their scanned
// offsets [ntiles + 1], entry lists [2][ecap] (source ids), vector lists [2][ecap * S]
// (16-bit ring vector indices) and the slot ring [2][ecap][S] vectors.
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
	long long const per = 2LL * 4 + 2LL * S * 2 + 2LL * S * 16; // bytes per arrival of capacity
	long long const room = (long long)smem_bytes - (long long)b - 64;
	int ecap = room > 0 ? (int)( room / per ) : 0;
	ecap = ecap > SLOT_MAX_ECAP ? SLOT_MAX_ECAP : ecap & ~7;
	g.ecap = ecap;
	g.ent = b;
	b += (size_t)2 * ecap * 4;
	g.vl = b;
	b += ( (size_t)2 * ecap * S * 2 + 15 ) & ~(size_t)15;
	g.ring = b;
	return g;
}

// the direct path's scratch (per-source-tile prefix, staged arrivals) lives in the ring
__host__ __device__ inline size_t slot_direct_scratch( int ntiles )
{
	return ( ( ( (size_t)ntiles + 1 ) * 4 + 15 ) & ~(size_t)15 ) + (size_t)SPIKE_BATCH * 16;
}

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
	__shared__ int m_e[8], m_big[8];
	__shared__ int vcnt[2];
	__shared__ int wsum[32];
	__shared__ int s_big;

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
	int * soff = reinterpret_cast<int *>( smem + g.soff );                    // [ntiles + 1]
	int * ent = reinterpret_cast<int *>( smem + g.ent );                      // [2][ecap]
	unsigned short * vl = reinterpret_cast<unsigned short *>( smem + g.vl ); // [2][ecap * S]
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
	auto compact = [&]( int k ) { compact_step( p, bits2 + ( k & 1 ) * words, words, d0, tile, t0 + k, lane ); };

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
		int k = 0;
		while( k < L )
		{
			int const kb = k; // the pipeline (re)starts at step kb
			// producer work during step j (the prologue: j < kb, every thread): threads
			// [0, npt) of numbering pt; `all` when every warp of the CTA takes part
			auto produce = [&]( int j, int pt, int npt, bool all ) {
				int const sa = j + 2, sb = j + 1;
				bool const do_s = sa >= kb && sa < L;
				bool const do_a = sb >= kb && sb < L && !m_big[sb & 7];
				if( pt == 0 )
				{
					vcnt[sb & 1] = 0;
					s_big = 0;
				}
				// summaries of step sa (none before `delay`): eight lanes per source tile; in
				// the prologue every lane first waits for the step's publication (later steps:
				// checked by the publisher warp during the step before)
				if( do_s )
				{
					long long const t = t0 + sa;
					int * sd = sum + ( sa & 1 ) * p.ntiles * SUM_W;
					if( t >= p.delay )
					{
						int const * src = p.summ + ( ( t - p.delay ) % p.ring ) * (long long)p.ntiles * SUM_W;
						int const q = pt & 7;
						for( int i = pt >> 3; i < p.ntiles; i += npt >> 3 )
						{
							if( all ) wait_published( p, i, t - p.delay );
							cp_async16( sd + i * SUM_W + 4 * q, src + i * SUM_W + 4 * q );
						}
					}
					else
						for( int i = pt; i < p.ntiles; i += npt ) sd[i * SUM_W] = 0;
				}
				// slots of step sb's arrivals into ring half sb & 1: S lanes per arrival
				if( do_a )
				{
					int const E = m_e[sb & 7];
					int const * es = ent + ( sb & 1 ) * ecap;
					uint4 * rh = ring + (size_t)( sb & 1 ) * ecap * S;
					int const q = pt % S, groups = npt / S;
					for( int e = pt / S; e < E; e += groups )
						cp_async16( rh + e * S + q, p.slots + ( (long long)es[e] * p.tin + ti ) * S + q );
				}
				cp_async_commit();
				cp_async_wait_all();
				if( all )
					__syncthreads();
				else
					bar_sync_slot_producers();
				// the vectors of step sb that hold indices, from every slot's length
				if( do_a )
				{
					int const E = m_e[sb & 7];
					uint4 const * rh = ring + (size_t)( sb & 1 ) * ecap * S;
					unsigned short * vo = vl + ( sb & 1 ) * ecap * S;
					int const rbase = ( sb & 1 ) * ecap * S;
					for( int e0 = pt - lane; e0 < E; e0 += npt )
					{
						int const e = e0 + lane;
						int nv = 0;
						if( e < E ) nv = min( S, (int)( slot_len( rh[e * S] ) + 11 ) / 12 );
						int const incl = warp_inclusive_scan( nv );
						int base = 0;
						if( lane == 31 && incl ) base = atomicAdd( &vcnt[sb & 1], incl );
						base = __shfl_sync( 0xffffffffu, base, 31 );
						int const o = base + incl - nv;
						for( int v = 0; v < nv; v++ ) vo[o + v] = (unsigned short)( rbase + e * S + v );
					}
				}
				// step sa: counts -> offsets of its arrivals (a scan over the source tiles),
				// then every source tile's ids into the entry list
				if( do_s )
				{
					int const * sd = sum + ( sa & 1 ) * p.ntiles * SUM_W;
					int const nwp = npt >> 5, pw = pt >> 5;
					int run = 0;
					for( int i0 = 0; i0 < p.ntiles; i0 += npt )
					{
						int const i = i0 + pt;
						int const c = i < p.ntiles ? sd[i * SUM_W] : 0;
						if( c > SUM_W - 1 ) s_big = 1; // more ids than the record holds
						int const incl = warp_inclusive_scan( c );
						if( lane == 31 ) wsum[pw] = incl;
						if( all )
							__syncthreads();
						else
							bar_sync_slot_producers();
						int before = run;
						for( int w = 0; w < pw; w++ ) before += wsum[w];
						if( i < p.ntiles ) soff[i] = before + incl - c;
						for( int w = 0; w < nwp; w++ ) run += wsum[w];
						if( all )
							__syncthreads();
						else
							bar_sync_slot_producers();
					}
					bool const big = s_big != 0; // set before the scan's barriers
					if( pt == 0 )
					{
						soff[p.ntiles] = run;
						m_e[sa & 7] = run;
						m_big[sa & 7] = big || run > ecap;
					}
					if( !big && run <= ecap )
					{
						int * es = ent + ( sa & 1 ) * ecap;
						for( int i = pt; i < p.ntiles; i += npt )
						{
							int const c = sd[i * SUM_W], o = soff[i];
							for( int r = 0; r < c; r++ ) es[o + r] = sd[i * SUM_W + 1 + r];
						}
					}
				}
			};

			int ks = L; // a step for the direct path, if any
			if( !p.flat_sync )
			{
				for( int j = kb - 2; j < kb; j++ )
				{
					produce( j, tid, nt, true );
					__syncthreads();
				}
				// the publication of the step whose summaries the producers load during step
				// kb (later ones: checked by the publisher warp a step ahead)
				if( kb + 2 < L && t0 + kb + 2 >= p.delay )
					for( int i = tid; i < p.ntiles; i += nt ) wait_published( p, i, t0 + kb + 2 - p.delay );
				__syncthreads();
				for( ; k < L; k++ )
				{
					if( m_big[k & 7] )
					{
						ks = k;
						break;
					}
					advance_clock( k );
					if( warp < nwc )
					{
						if( t0 + k >= p.delay )
						{
							int const v = vcnt[k & 1];
							unsigned short const * vo = vl + ( k & 1 ) * ecap * S;
#pragma unroll 2
							for( int x = tid; x < v; x += ncons ) count_vector<12>( cnt, ring[vo[x]] );
						}
						bar_sync_first( ncons ); // counts complete
						update( k, nwc );
					}
					else if( warp == nw - 1 )
					{
						// the publisher warp: step k - 1's spikes and summary, fenced, then its
						// flag; then the publication of the step whose summaries the producers
						// load during the next step
						if( k > kb ) compact( k - 1 );
						if( k + 3 < L && t0 + k + 3 >= p.delay ) warp_wait_all_published( p, t0 + k + 3 - p.delay );
					}
					else
						produce( k, tid - ncons, nt - ncons - 32, false );
					__syncthreads(); // step k updated, step k + 1's slots in the ring
				}
				if( k > kb && warp == nw - 1 ) compact( k - 1 ); // the last pipelined step
				__syncthreads();
			}
			else
				ks = k;
			if( ks >= L ) break;

			// ------------------------------------------------------------ the direct path
			// step ks alone from the ELL rows (window_counts' path), its scratch in the ring
			advance_clock( ks );
			long long const t = t0 + ks;
			if( t >= p.delay )
			{
				int * pref = reinterpret_cast<int *>( ring );
				int4 * sbuf = reinterpret_cast<int4 *>( reinterpret_cast<unsigned char *>( ring ) + ( ( ( p.ntiles + 1 ) * 4 + 15 ) & ~15 ) );
				net_params q = p;
				q.tile = span; // counter rows are span long
				for( int i = tid; i < p.ntiles; i += nt ) wait_published( p, i, t - p.delay );
				__syncthreads();
				deliver_counts<N>( q, (int)( ( t - p.delay ) % p.ring ), tile, d0, d1, cnt, pref, sbuf, scratch );
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
