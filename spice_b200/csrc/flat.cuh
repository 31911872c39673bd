// Window kernel for models with input classes (non-plastic), shaped by measurement.
//
// Same results as window_counts (kernels.cuh). Per launch -- one delay window of L steps --
// a CTA owns one tile of destination neurons [tile_first[j], tile_first[j + 1]):
//   1. Staging. All arrivals of the window fired before it started, so the CTA stages the
//      window's whole arrival table (source, slice start, slice length of the row
//      restricted to the tile) in shared memory with three rounds of parallel loads
//      (per-tile spike counts, spike ids, pivots) instead of a latency chain per step.
//   2. Counting. Per step, warps take batches of FLAT_U arrivals; lane l loads elements
//      l, l + 32, ... of every slice (coalesced 128-byte loads), the next batch's loads
//      are issued before the current batch is counted, and every target is counted per
//      (target, input class) with shared-memory atomics.
//   3. Update. The tile's neuron state lives in shared memory for the whole window; the
//      counts are replayed through the model's receive() and the model updates every
//      neuron; fired neurons are compacted in ascending order into the spike ring.
// Keeping the state in shared memory lets tile sizes follow the work (balanced tiles):
// a population without inputs costs little per neuron and gets few, large tiles.
//
// Measured on B200 (Brunel, 1e9 synapses): slices of a few hundred bytes make 1-D bulk
// (TMA) copies issue-bound at about 90 cycles per copy on the issuing warp, and four-
// element vector loads per lane spend their time on per-element bounds arithmetic; the
// element-per-lane form above is several times faster than either.
#pragma once

#include "kernels.cuh"

namespace spk
{
#ifndef SPK_FLAT_U
#define SPK_FLAT_U 4
#endif
#ifndef SPK_FLAT_R
#define SPK_FLAT_R 4
#endif
constexpr int FLAT_U = SPK_FLAT_U;  // arrivals per warp batch
constexpr int FLAT_R = SPK_FLAT_R;  // 32-element rounds per arrival held in registers
constexpr int FLAT_ENT_CAP = 8192;  // staged arrivals per segment of a window
constexpr int FLAT_SCRATCH = 4096;  // per-(step, source tile) counts staged at once
constexpr int FLAT_MAX_TILE = 4064; // slice lengths fit the table's 12-bit field
constexpr long long FLAT_MAX_WIDTH = 1 << 20; // slice starts fit the table's 20-bit field

// shared memory of a launch: table, staging scratch, counters [classes][tmax],
// fired bits [tmax / 32], neuron state [attrs][tmax]
inline size_t flat_smem_bytes( int classes, int attrs, int tmax )
{
	return (size_t)FLAT_ENT_CAP * 8 + (size_t)FLAT_SCRATCH * 4 + (size_t)classes * tmax * 4 + (size_t)tmax / 8 + (size_t)attrs * tmax * 4;
}

// Stage the arrivals of the steps [ks, L) of the window starting at t0, as many whole
// steps as fit ENT_CAP. Returns ke: steps [ks, ke) are staged (ke == ks: step ks alone
// exceeds the table). step_begin[k - ks] = first table entry of step k, k in [ks, ke].
// table[g] = { source id, slice start | slice length << 20 }.
__device__ __forceinline__ int stage_table(
    net_params const & p, unsigned * cnts, int cnts_cap, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int * scratch )
{
	int const tid = threadIdx.x, nt = blockDim.x;
	int const ksteps = min( L - ks, max( 1, ( cnts_cap - 1 ) / max( 1, p.ntiles ) ) );
	int const M = ksteps * p.ntiles;

	// 1. per-(step, source tile) spike counts (none before `delay`)
	for( int q = tid; q < M; q += nt )
	{
		int const k = ks + q / p.ntiles, i = q % p.ntiles;
		long long const t = t0 + k;
		cnts[q] = t >= p.delay ? p.ring_cnt[(long long)( ( t - p.delay ) % p.ring ) * p.ntiles + i] : 0u;
	}
	__syncthreads();
	// 2. in-place exclusive scan over the flattened array, contiguous runs per thread
	int const per = ( M + nt - 1 ) / nt;
	int const q0 = min( M, tid * per ), q1 = min( M, q0 + per );
	int run = 0;
	for( int q = q0; q < q1; q++ ) run += (int)cnts[q];
	int total;
	int base = block_exclusive_scan( run, scratch, &total );
	for( int q = q0; q < q1; q++ )
	{
		int const c = (int)cnts[q];
		cnts[q] = (unsigned)base;
		base += c;
	}
	if( tid == 0 ) cnts[M] = (unsigned)total;
	__syncthreads();
	// 3. whole steps that fit
	int ke = ks;
	while( ke < ks + ksteps )
	{
		int const end = ( ke + 1 - ks ) < ksteps ? (int)cnts[( ke + 1 - ks ) * p.ntiles] : total;
		if( end > FLAT_ENT_CAP ) break;
		ke++;
	}
	for( int k = ks + tid; k <= ke; k += nt ) step_begin[k - ks] = ( k - ks ) < ksteps ? (int)cnts[( k - ks ) * p.ntiles] : total;
	int const nent = ( ke - ks ) < ksteps ? (int)cnts[( ke - ks ) * p.ntiles] : total;
	// 4. spike ids: one thread per (step, source tile)
	for( int q = tid; q < ( ke - ks ) * p.ntiles; q += nt )
	{
		int const k = ks + q / p.ntiles, i = q % p.ntiles;
		int const b = (int)cnts[q], c = (int)cnts[q + 1] - b;
		if( c == 0 ) continue;
		long long const t = t0 + k;
		int const * seg = p.ring_ids + (long long)( ( t - p.delay ) % p.ring ) * p.n + __ldg( p.tile_first + i );
		for( int r = 0; r < c; r++ ) table[b + r].x = seg[r];
	}
	__syncthreads();
	// 5. this tile's slice of every arriving row
	for( int g = tid; g < nent; g += nt )
	{
		int const src = table[g].x;
		unsigned const * pv = p.pivots + (long long)src * ( p.ntiles + 1 ) + tile;
		unsigned const lo = __ldg( pv ), hi = __ldg( pv + 1 );
		table[g].y = (int)( lo | ( ( hi - lo ) << 20 ) );
	}
	__syncthreads();
	return ke;
}

// arrival x of the table: pointer to its slice, slice length, source id
__device__ __forceinline__ int const * flat_entry( net_params const & p, int2 const * table, int x, int & len, int & src )
{
	int2 const en = table[x];
	src = en.x;
	len = (int)( (unsigned)en.y >> 20 );
	return p.edges + (long long)en.x * p.width + ( (unsigned)en.y & 0xFFFFFu );
}

// lane `lane` loads elements lane + 32 r, r < FLAT_R, of the slices of arrivals
// [x, x + FLAT_U) (coalesced 128-byte warp loads); longer slices finish in flat_count
__device__ __forceinline__ void flat_load( net_params const & p, int2 const * table, int x, int xe, int lane, int * v )
{
#pragma unroll
	for( int u = 0; u < FLAT_U; u++ )
	{
		int len = 0, src = 0;
		int const * row = p.edges;
		if( x + u < xe ) row = flat_entry( p, table, x + u, len, src );
#pragma unroll
		for( int r = 0; r < FLAT_R; r++ )
		{
			int const j = r * 32 + lane;
			v[u * FLAT_R + r] = j < len ? __ldg( row + j ) : 0;
		}
	}
}

__device__ __forceinline__ void flat_count_one( net_params const & p, unsigned * cc, int target, int d0, int span )
{
	unsigned const local = (unsigned)( target - d0 );
	if( local < (unsigned)span )
		atomicAdd( cc + local, 1u );
	else
		atomicOr( p.err, ERR_BAD_TARGET );
}

// count the targets of arrivals [x, x + FLAT_U) per (target, input class)
template <typename N>
__device__ __forceinline__ void flat_count(
    net_params const & p, int2 const * table, int x, int xe, int lane, int const * v, unsigned * cnt, int tmax, int d0, int span, snn_info info )
{
#pragma unroll
	for( int u = 0; u < FLAT_U; u++ )
	{
		if( x + u < xe )
		{
			int len, src;
			int const * row = flat_entry( p, table, x + u, len, src );
			unsigned * cc = cnt + N::input_class( src, info ) * tmax;
#pragma unroll
			for( int r = 0; r < FLAT_R; r++ )
				if( r * 32 + lane < len ) flat_count_one( p, cc, v[u * FLAT_R + r], d0, span );
			for( int j = FLAT_R * 32 + lane; j < len; j += 32 ) flat_count_one( p, cc, __ldg( row + j ), d0, span );
		}
	}
}

// neuron state of the tile: shared memory [attrs][tmax] <-> registers / global memory
template <typename Decl, int I = 0>
struct smem_state
{
	template <typename Tup>
	__device__ __forceinline__ static void load( Tup & t, unsigned char const * base, int tmax, int local )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			tuple_at<I>::get( t ) = reinterpret_cast<T const *>( base + (size_t)I * tmax * 4 )[local];
			smem_state<Decl, I + 1>::load( t, base, tmax, local );
		}
	}
	template <typename Tup>
	__device__ __forceinline__ static void store( Tup & t, unsigned char * base, int tmax, int local )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			reinterpret_cast<T *>( base + (size_t)I * tmax * 4 )[local] = tuple_at<I>::get( t );
			smem_state<Decl, I + 1>::store( t, base, tmax, local );
		}
	}
	__device__ __forceinline__ static void from_global( void * const * a, long long d0, int span, unsigned char * base, int tmax )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			static_assert( sizeof( T ) == 4, "attributes are 32-bit" );
			T const * g = static_cast<T const *>( a[I] ) + d0;
			T * sh = reinterpret_cast<T *>( base + (size_t)I * tmax * 4 );
			for( int x = threadIdx.x; x < span; x += blockDim.x ) sh[x] = g[x];
			smem_state<Decl, I + 1>::from_global( a, d0, span, base, tmax );
		}
	}
	__device__ __forceinline__ static void to_global( void * const * a, long long d0, int span, unsigned char const * base, int tmax )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			T * g = static_cast<T *>( a[I] ) + d0;
			T const * sh = reinterpret_cast<T const *>( base + (size_t)I * tmax * 4 );
			for( int x = threadIdx.x; x < span; x += blockDim.x ) g[x] = sh[x];
			smem_state<Decl, I + 1>::to_global( a, d0, span, base, tmax );
		}
	}
};
template <typename Model>
__global__ void __launch_bounds__( 512, 1 ) window_flat( net_params p, int L, float dt, int tmax )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	constexpr int C = N::input_classes;
	static_assert( C >= 1, "window_flat needs a model with input classes" );

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	__shared__ int step_begin[MAX_WINDOW + 1];

	int2 * table = reinterpret_cast<int2 *>( smem );                    // [FLAT_ENT_CAP]
	unsigned * cnts = reinterpret_cast<unsigned *>( table + FLAT_ENT_CAP ); // [FLAT_SCRATCH]
	unsigned * cnt = cnts + FLAT_SCRATCH;                                 // [C][tmax]
	unsigned * bits = cnt + C * tmax;                                     // [tmax / 32]
	unsigned char * state = reinterpret_cast<unsigned char *>( bits + tmax / 32 ); // [attrs][tmax]

	int const tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	int const tile = blockIdx.x, d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	snn_info const info{ p.n };

	window_clock_begin( p, L, dt, s_dt, &s_t0, &s_c, &s_sum );
	long long const t0 = s_t0;
	smem_state<N>::from_global( p.attr, d0, span, state, tmax );
	__syncthreads();

	int ks = 0;
	while( ks < L )
	{
		int const ke = stage_table( p, cnts, FLAT_SCRATCH, table, tile, t0, ks, L, step_begin, scratch );
		int const kend = ke > ks ? ke : ks + 1; // ke == ks: step ks goes the direct way

		for( int k = ks; k < kend; k++ )
		{
			long long const t = t0 + k;
			bool const arrivals = t >= p.delay;
			if( arrivals )
			{
				for( int x = tid; x < C * tmax; x += nt ) cnt[x] = 0;
				__syncthreads();
				if( ke == ks )
				{
					// more arrivals than the table holds: the direct path of window_counts,
					// its scratch in the (unused) table
					int * pref = reinterpret_cast<int *>( table );
					int4 * sb = reinterpret_cast<int4 *>( smem + ( ( ( p.ntiles + 1 ) * 4 + 15 ) & ~15 ) );
					net_params q = p;
					q.tile = tmax; // counter rows are tmax long
					deliver_counts<N>( q, (int)( ( t - p.delay ) % p.ring ), tile, d0, d1, cnt, pref, sb, scratch );
				}
				else
				{
					int const eb = step_begin[k - ks], ee = step_begin[k + 1 - ks];
					int const stride = nw * FLAT_U;
					int va[FLAT_U * FLAT_R], vb[FLAT_U * FLAT_R];
					int x = eb + warp * FLAT_U;
					if( x < ee ) flat_load( p, table, x, ee, lane, va );
					for( ; x < ee; x += stride )
					{
						int const xn = x + stride;
						if( xn < ee ) flat_load( p, table, xn, ee, lane, vb );
						flat_count<N>( p, table, x, ee, lane, va, cnt, tmax, d0, span, info );
#pragma unroll
						for( int u = 0; u < FLAT_U * FLAT_R; u++ ) va[u] = vb[u];
					}
					__syncthreads();
				}
			}

			// update: warp w owns neurons [32 w, 32 w + 32) + 32 nw * round; one bit word each
			for( int base = warp * 32; base < span; base += nw * 32 )
			{
				int const local = base + lane;
				bool fired = false;
				if( local < span )
				{
					Tup st;
					smem_state<N>::load( st, state, tmax, local );
					uint32_t const i = (uint32_t)( d0 + local );
					reg_iter<Tup> it{ st, i };
					if( arrivals )
#pragma unroll
						for( int c = 0; c < C; c++ )
						{
							unsigned const m = cnt[c * tmax + local];
							if( m )
							{
								repeat_backend rb( p.seed, i, (uint32_t)t, m );
								N::receive( N::class_source( c, info ), it, null_syn_iter{}, info, rb );
							}
						}
					device_backend bak( p.seed, i, (uint32_t)t );
					fired = N::update( it, s_dt[k], info, bak );
					smem_state<N>::store( st, state, tmax, local );
				}
				unsigned const word = __ballot_sync( 0xffffffffu, fired );
				if( lane == 0 ) bits[base >> 5] = word;
			}
			__syncthreads();
			// ascending compaction: thread t emits the fired ids of words [t per, t per + per)
			int const words = ( span + 31 ) >> 5;
			int const per = ( words + nt - 1 ) / nt;
			int const w0 = min( words, tid * per ), w1 = min( words, w0 + per );
			int mine = 0;
			for( int w = w0; w < w1; w++ ) mine += __popc( bits[w] );
			int total;
			int off = block_exclusive_scan( mine, scratch, &total );
			int const slot_out = (int)( t % p.ring );
			int * out = p.ring_ids + (long long)slot_out * p.n + d0;
			for( int w = w0; w < w1; w++ )
			{
				unsigned m = bits[w];
				while( m )
				{
					int const b = __ffs( m ) - 1;
					m &= m - 1;
					out[off++] = d0 + ( w << 5 ) + b;
				}
			}
			if( tid == 0 ) p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)total;
			__syncthreads(); // bits and counters are rewritten next step
		}
		ks = kend;
	}

	smem_state<N>::to_global( p.attr, d0, span, state, tmax );
	window_clock_end( p, L, t0, s_c, s_sum );
}
} // namespace spk
