// Window kernel for models with input classes (non-plastic), shaped by measurement.
//
// Same results as window_counts (kernels.cuh). Per launch -- one delay window of L steps --
// a CTA owns one tile of destination neurons [tile_first[j], tile_first[j + 1]).
//
// Data layout ("slices"). Besides the ELL rows, the net keeps every row's part inside
// every tile as a slice of counter indices, class(src) * span + (target - d0), padded to a
// whole 16-byte vector: eight 16-bit indices per vector (pad SLICE_PAD), or, when every
// index of the net fits 10 bits, twelve (three per 32-bit word, pad SLICE_PAD10). A row's
// slices lie contiguously in tile order (source-major), and rec[src * ntiles + tile] =
// { first vector, length }. A CTA reads 1.33 or 2 bytes per synapse, already in the form
// its counters are indexed by; and since all tiles fetch their slices of the same spiking
// rows at about the same time, each row is one contiguous stretch of DRAM.
//
// All arrivals of a window fired before it started, so a step's arrivals can be prepared
// steps ahead. The CTA splits into FLAT_PRODUCERS producer warps and consumer warps. While
// the consumers work on step k, the producers
//   - copy the slices of step k + 1 into a shared-memory ring with cp.async,
//   - load the slice records of step k + 2's arrivals and lay out their ring offsets,
//   - load the spike ids of step k + 3 (the per-source-tile spike counts, scanned),
//   - load the per-source-tile spike counts of step k + 4,
// each stage one global-memory round trip that a whole step hides, while the last warp
// compacts the fired neurons of step k - 1 in ascending order into the spike ring and
// publishes them. The consumers count
// step k from the ring, one 16-byte vector per thread at a time with a shared-memory
// atomic per index; a consumer-only barrier; then they replay the counts through the
// model's receive(), update every neuron and zero the counters they consumed. The tile's
// neuron state stays in shared memory for the whole window; one block-wide barrier per
// step. A step with more arrivals than a step table holds, or more slices than the ring,
// switches the rest of the window to a synchronous path (window-wide staging, slices in
// pieces or the direct path of window_counts).
// Keeping the state in shared memory lets tile sizes follow the work (balanced tiles): a
// population without inputs costs little per neuron and gets few, large tiles.
//
// Measured on B200 (Brunel, 1e9 synapses): scattered 16-byte copies issue at about one per
// cycle per SM, and since all tiles issue theirs at the same moment the burst runs near
// HBM bandwidth; issued by the warps that then count, it sat on every step's critical
// path, and staging a whole window before its first step cost more than the steps.
#pragma once

#include "kernels.cuh"

namespace spk
{
constexpr int FLAT_THREADS = 1024;    // threads of a window_flat CTA (one CTA per SM)
#ifndef SPK_FLAT_PRODUCERS
#define SPK_FLAT_PRODUCERS 12
#endif
constexpr int FLAT_PRODUCERS = SPK_FLAT_PRODUCERS; // warps that stage, copy slices and compact spikes (default)
constexpr int FLAT_MIN_PRODUCERS = 4;  // two scanning warps and the publisher at least
constexpr int FLAT_MAX_PRODUCERS = 24; // eight consumer warps at least
constexpr int FLAT_PC = 1032;         // per-source-tile counts of one step (ntiles + 1 <= FLAT_PC)
constexpr int FLAT_STEP_CAP = 1024;   // arrivals of one step the pipeline stages
constexpr int FLAT_ENT_CAP = 6144;    // arrivals per segment of the synchronous path
constexpr int FLAT_SCRATCH = 2560;    // per-(step, source tile) counts it stages at once (>= threads)
constexpr int FLAT_MAX_TILE = 4064;   // slice lengths fit the table's 12-bit field
// a slice is no longer than its row's ELL width either: nets of width <= FLAT_MAX_SLICE may
// take tiles up to FLAT_MAX_TILE_WIDE (shared memory permitting)
constexpr int FLAT_MAX_SLICE = 4095;
constexpr int FLAT_MAX_TILE_WIDE = 16352;
constexpr int FLAT_MIN_BUF = 512;     // vectors per buffer at least (one slice of a full tile)
constexpr int FLAT_P_BITS = 20;       // vector offsets inside a step held in the table
constexpr unsigned short SLICE_PAD = 0xFFFFu;
constexpr unsigned SLICE_PAD10 = 0x3FFu; // 10-bit packing: indices < SLICE_PAD10
static_assert( FLAT_SCRATCH >= FLAT_THREADS, "staging keeps one prefix per thread in the scratch" );
static_assert( FLAT_STEP_CAP <= ( 1 << FLAT_P_BITS ), "step offsets fit the table" );

// shared memory of a CTA: neuron state [attrs][span], fired bits [2][words]; tiles with
// inputs add counters [classes][span], the per-step staging ring (counts [4][FLAT_PC],
// tables [4][FLAT_STEP_CAP]) and the slice ring in what is left (the synchronous path
// keeps its table, scratch and buffer there)
__host__ __device__ inline size_t flat_state_bytes( int attrs, int span )
{
	return (size_t)attrs * span * 4 + 2 * ( ( (size_t)span + 31 ) / 32 ) * 4;
}
__host__ __device__ inline size_t flat_fixed_bytes( int classes, int attrs, int span )
{
	size_t b = flat_state_bytes( attrs, span ) + (size_t)classes * span * 4;
	b = ( b + 15 ) & ~(size_t)15;
	return b + (size_t)4 * FLAT_PC * 4 + (size_t)4 * FLAT_STEP_CAP * 8;
}
inline size_t flat_smem_bytes( int classes, int attrs, int tmax )
{
	return flat_fixed_bytes( classes, attrs, tmax ) + (size_t)FLAT_ENT_CAP * 8 + (size_t)FLAT_SCRATCH * 4 + (size_t)FLAT_MIN_BUF * 16;
}

// ------------------------------------------------------------------------------------
// building the slices (once per net)
// ------------------------------------------------------------------------------------
// 16-byte vectors of a slice of `len` indices, `per` (8 or 12) to a vector
__host__ __device__ __forceinline__ unsigned slice_vecs( unsigned len, int per ) { return per == 12 ? ( len + 11 ) / 12 : ( len + 7 ) >> 3; }

// vectors of every (src, tile) slice, from the ELL pivots, into rec[].x; rec[].y = length
__global__ void slice_vectors( int n, int ntiles, unsigned const * pivots, uint2 * rec, int per )
{
	long long const total = (long long)n * ntiles;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x )
	{
		long long const src = e / ntiles, j = e % ntiles;
		unsigned const * pv = pivots + src * ( ntiles + 1 ) + j;
		unsigned const len = pv[1] - pv[0];
		rec[e] = make_uint2( slice_vecs( len, per ), len );
	}
}

// one warp per source row: rec[src][tile].x <- exclusive prefix over the row's tiles of the
// vector counts (row-relative), row_vectors[src] <- the row's vectors; tile_inputs[tile]
// <- 1 if any row has synapses in the tile
__global__ void slice_row_offsets( int n, int ntiles, uint2 * rec, unsigned * row_vectors, int * tile_inputs )
{
	int const warp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( warp >= n ) return;
	uint2 * r = rec + (long long)warp * ntiles;
	unsigned carry = 0;
	for( int j0 = 0; j0 < ntiles; j0 += 32 )
	{
		int const j = j0 + lane;
		uint2 const e = j < ntiles ? r[j] : make_uint2( 0u, 0u );
		unsigned incl = e.x;
		for( int o = 1; o < 32; o <<= 1 )
		{
			unsigned const y = __shfl_up_sync( 0xffffffffu, incl, o );
			if( lane >= o ) incl += y;
		}
		if( j < ntiles )
		{
			r[j].x = carry + incl - e.x;
			if( e.y && !*(int volatile *)( tile_inputs + j ) ) atomicOr( tile_inputs + j, 1 );
		}
		carry += __shfl_sync( 0xffffffffu, incl, 31 );
	}
	if( lane == 0 ) row_vectors[warp] = carry;
}

// one warp per source row: rebase rec[] to global vector indices (the row's first vector
// row_base[src] plus the row-relative offset) and write every slice
template <typename Model>
__global__ void __launch_bounds__( 256 ) slice_fill(
    int n, int width, int ntiles, int const * edges, unsigned const * pivots, int const * tile_first,
    unsigned long long const * row_base, uint2 * rec, unsigned short * slices, int per )
{
	using N = typename Model::neuron;
	snn_info const info{ n };
	int const warp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5, lane = threadIdx.x & 31;
	if( warp >= n ) return;
	int const src = warp;
	int const cls = N::input_class( src, info );
	int const * row = edges + (long long)src * width;
	unsigned const * pv = pivots + (long long)src * ( ntiles + 1 );
	for( int j = 0; j < ntiles; j++ )
	{
		uint2 const r = rec[(long long)src * ntiles + j];
		unsigned long long const first = row_base[src] + r.x;
		__syncwarp();
		if( lane == 0 ) rec[(long long)src * ntiles + j] = make_uint2( (unsigned)first, r.y );
		if( r.y == 0 ) continue;
		int const d0 = tile_first[j], span = tile_first[j + 1] - d0;
		unsigned const lo = pv[j];
		if( per == 12 )
		{
			// three 10-bit indices per 32-bit word, bits 0-9, 10-19, 20-29
			unsigned * out = reinterpret_cast<unsigned *>( slices ) + first * 4;
			int const words = (int)slice_vecs( r.y, 12 ) * 4;
			for( int w = lane; w < words; w += 32 )
			{
				unsigned word = 0;
				for( int f = 0; f < 3; f++ )
				{
					int const e = 3 * w + f;
					unsigned const x = e < (int)r.y ? (unsigned)( cls * span + ( row[lo + e] - d0 ) ) : SLICE_PAD10;
					word |= x << ( 10 * f );
				}
				out[w] = word;
			}
		}
		else
		{
			unsigned short * out = slices + first * 8;
			int const padded = (int)( ( r.y + 7 ) & ~7u );
			for( int e = lane; e < padded; e += 32 )
				out[e] = e < (int)r.y ? (unsigned short)( cls * span + ( row[lo + e] - d0 ) ) : SLICE_PAD;
		}
	}
}

// per-(step, source tile) spike counts of steps [ks, ks + ksteps) of the window starting
// at t0 (none before `delay`) into cnts[(k - ks) * ntiles + tile], eight loads in flight
// per thread; ends with a barrier
__device__ __forceinline__ void load_counts( net_params const & p, unsigned * cnts, long long t0, int ks, int ksteps, int * )
{
	constexpr int B = 8;
	int const tid = threadIdx.x, nt = blockDim.x;
	int const M = ksteps * p.ntiles;
	for( int q0 = tid; q0 < M; q0 += B * nt )
	{
		unsigned v[B];
#pragma unroll
		for( int b = 0; b < B; b++ )
		{
			int const q = q0 + b * nt;
			v[b] = 0u;
			if( q < M )
			{
				int const k = ks + q / p.ntiles, i = q % p.ntiles;
				long long const t = t0 + k;
				if( t >= p.delay )
				{
					wait_published( p, i, t - p.delay );
					v[b] = __ldcg( p.ring_cnt + (long long)( ( t - p.delay ) % p.ring ) * p.ntiles + i );
				}
			}
		}
#pragma unroll
		for( int b = 0; b < B; b++ )
			if( q0 + b * nt < M ) cnts[q0 + b * nt] = v[b];
	}
	__syncthreads();
}

// ------------------------------------------------------------------------------------
// window kernel
// ------------------------------------------------------------------------------------
// table[g] = { first vector of the slice, length | vector offset inside its step << 12 }
__device__ __forceinline__ int ent_len( int2 e ) { return e.y & 0xFFF; }
__device__ __forceinline__ int ent_vec( int2 e, int per ) { return (int)slice_vecs( (unsigned)ent_len( e ), per ); }
__device__ __forceinline__ int ent_off( int2 e ) { return (int)( (unsigned)e.y >> 12 ); }

// how a staged segment runs
enum seg_mode
{
	SEG_PIPE = 0,   // steps [ks, ke) each fit a slice buffer: producers and consumers
	SEG_PIECES = 1, // step ks alone, its slices in several buffer loads
	SEG_DIRECT = 2  // step ks alone, counted from the ELL rows (window_counts' path)
};

__device__ __forceinline__ int stage_arrivals(
    net_params const & p, unsigned * cnts, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int & nent_out, int * scratch );
__device__ __forceinline__ int stage_offsets(
    int2 * table, int ks, int ke, int nent, int * step_begin, int * step_vec, int * run_first, int * scratch, int bufv, int pack, int & mode );

// Stage the arrivals of the steps [ks, L) of the window starting at t0 (the synchronous
// path), as many whole steps as fit FLAT_ENT_CAP, and set the segment's mode. Returns the
// segment's end ke.
// step_begin[k - ks] = first entry of step k and step_vec[k - ks] = first vector of step
// k counted from the segment start, for k in [ks, ke].
__device__ __forceinline__ int stage_table(
    net_params const & p, unsigned * cnts, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int * step_vec,
    int * scratch, int bufv, int & mode )
{
	int nent = 0;
	int const ke = stage_arrivals( p, cnts, table, tile, t0, ks, L, step_begin, nent, scratch );
	if( ke == ks )
	{
		mode = SEG_DIRECT; // step ks alone exceeds the table
		return ks + 1;
	}
	return stage_offsets( table, ks, ke, nent, step_begin, step_vec, reinterpret_cast<int *>( cnts ), scratch, bufv, p.pack, mode );
}

// Per-CTA staging of whole steps: the (step, source tile) prefix, then every arrival's
// spike id and slice record. Returns ke.
__device__ __forceinline__ int stage_arrivals(
    net_params const & p, unsigned * cnts, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int & nent_out, int * scratch )
{
	constexpr int B = 8; // loads in flight per thread
	int const tid = threadIdx.x, nt = blockDim.x;
	int const ksteps = min( L - ks, max( 1, ( FLAT_SCRATCH - 1 ) / max( 1, p.ntiles ) ) );
	int const M = ksteps * p.ntiles;

	// 1. per-(step, source tile) spike counts
	load_counts( p, cnts, t0, ks, ksteps, scratch );
	// 2. in-place exclusive scan over the flattened array, contiguous runs per thread
	{
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
	}
	__syncthreads();
	// 3. whole steps that fit the table
	int ke = ks;
	while( ke < ks + ksteps && (int)cnts[( ke + 1 - ks ) * p.ntiles] <= FLAT_ENT_CAP ) ke++;
	for( int k = tid; k <= ke - ks; k += nt ) step_begin[k] = (int)cnts[k * p.ntiles];
	int const mq = ( ke - ks ) * p.ntiles;
	int const nent = (int)cnts[mq];
	// 4. entry g -> its (step, source tile) pair, spike id, slice record; every thread owns
	//    a contiguous run of entries and walks the pairs along it
	int const per = ( nent + nt - 1 ) / nt;
	int const g0 = min( nent, tid * per ), g1 = min( nent, g0 + per );
	if( g0 < g1 )
	{
		int q = 0, hi = mq; // last pair q with cnts[q] <= g0
		while( hi - q > 1 )
		{
			int const mid = ( q + hi ) >> 1;
			if( (int)cnts[mid] <= g0 )
				q = mid;
			else
				hi = mid;
		}
		for( int gb = g0; gb < g1; gb += B )
		{
			int src[B];
#pragma unroll
			for( int b = 0; b < B; b++ )
			{
				int const g = gb + b;
				src[b] = 0;
				if( g < g1 )
				{
					while( (int)cnts[q + 1] <= g ) q++;
					int const k = ks + q / p.ntiles, i = q % p.ntiles;
					long long const t = t0 + k;
					src[b] = __ldcg( p.ring_ids + (long long)( ( t - p.delay ) % p.ring ) * p.n + __ldg( p.tile_first + i ) + ( g - (int)cnts[q] ) );
				}
			}
			uint2 r[B];
#pragma unroll
			for( int b = 0; b < B; b++ ) r[b] = gb + b < g1 ? __ldg( p.slice_rec + (long long)src[b] * p.ntiles + tile ) : make_uint2( 0, 0 );
#pragma unroll
			for( int b = 0; b < B; b++ )
				if( gb + b < g1 ) table[gb + b] = make_int2( (int)r[b].x, (int)r[b].y );
		}
	}
	__syncthreads();
	nent_out = nent;
	return ke;
}


// Vector offsets of the staged arrivals: prefix over the segment, then relative to each
// step (table[g].y = length | offset << 12), step_vec[k - ks] = first vector of step k.
// The segment ends before the first step whose vectors exceed a slice buffer (`bufv`);
// if that is step ks, it runs alone: in pieces, or directly if its offsets do not fit
// FLAT_P_BITS. Returns the segment's end and sets `mode`.
__device__ __forceinline__ int stage_offsets(
    int2 * table, int ks, int ke, int nent, int * step_begin, int * step_vec, int * run_first, int * scratch, int bufv, int pack, int & mode )
{
	int const tid = threadIdx.x, nt = blockDim.x;
	int const per = ( nent + nt - 1 ) / nt;
	int const g0 = min( nent, tid * per ), g1 = min( nent, g0 + per );
	int run = 0;
	for( int g = g0; g < g1; g++ ) run += ent_vec( table[g], pack );
	int vtotal;
	int const my_first = block_exclusive_scan( run, scratch, &vtotal );
	run_first[tid] = my_first;
	__syncthreads();
	for( int k = tid; k <= ke - ks; k += nt )
	{
		int const g = step_begin[k];
		int v = vtotal;
		if( g < nent )
		{
			int const owner = g / per;
			v = run_first[owner];
			for( int h = owner * per; h < g; h++ ) v += ent_vec( table[h], pack );
		}
		step_vec[k] = v;
	}
	__syncthreads();
	if( g0 < g1 )
	{
		int k = 0;
		int v = my_first;
		for( int g = g0; g < g1; g++ )
		{
			while( step_begin[k + 1] <= g ) k++;
			int2 e = table[g];
			unsigned const rel = (unsigned)( v - step_vec[k] );
			int const nv = ent_vec( e, pack );
			e.y = ent_len( e ) | (int)( ( rel & ( ( 1u << FLAT_P_BITS ) - 1 ) ) << 12 );
			table[g] = e;
			v += nv;
		}
	}
	int kfit = ks;
	while( kfit < ke && step_vec[kfit + 1 - ks] - step_vec[kfit - ks] <= bufv ) kfit++;
	__syncthreads();
	if( kfit > ks )
	{
		mode = SEG_PIPE;
		return kfit;
	}
	mode = step_vec[1] - step_vec[0] < ( 1 << FLAT_P_BITS ) ? SEG_PIECES : SEG_DIRECT;
	return ks + 1;
}

// one past the last entry of the piece starting at entry `a` of a step whose entries end
// at `e`: the entries whose vectors fit one buffer of `bufv` vectors together
__device__ __forceinline__ int piece_end( int2 const * table, int a, int e, int bufv, int pack )
{
	int const pa = ent_off( table[a] );
	int lo = a, hi = e; // f(g) = off(g) + vec(g) - pa <= bufv holds for g = a
	while( hi - lo > 1 )
	{
		int const mid = ( lo + hi ) >> 1;
		int2 const m = table[mid];
		if( ent_off( m ) + ent_vec( m, pack ) - pa <= bufv )
			lo = mid;
		else
			hi = mid;
	}
	return lo + 1;
}

// vectors of the piece [a, b) of a step whose entries end at e (step_vectors in all)
__device__ __forceinline__ int piece_vectors( int2 const * table, int a, int b, int e, int step_vectors )
{
	if( a >= b ) return 0;
	return ( b < e ? ent_off( table[b] ) : step_vectors ) - ent_off( table[a] );
}

__device__ __forceinline__ void cp_async16( void * dst, void const * src )
{
	unsigned const d = (unsigned)__cvta_generic_to_shared( dst );
	asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"( d ), "l"( src ) : "memory" );
}
__device__ __forceinline__ void cp_async8( void * dst, void const * src )
{
	unsigned const d = (unsigned)__cvta_generic_to_shared( dst );
	asm volatile( "cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"( d ), "l"( src ) : "memory" );
}
__device__ __forceinline__ void cp_async4( void * dst, void const * src )
{
	unsigned const d = (unsigned)__cvta_generic_to_shared( dst );
	asm volatile( "cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"( d ), "l"( src ) : "memory" );
}
__device__ __forceinline__ void cp_async_commit() { asm volatile( "cp.async.commit_group;\n" ::: "memory" ); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile( "cp.async.wait_group 0;\n" ::: "memory" ); }
__device__ __forceinline__ void cp_async_wait_but_one() { asm volatile( "cp.async.wait_group 1;\n" ::: "memory" ); }

// copy the slices of entries [a, b) into buf, by threads [0, nthreads) of the caller's
// numbering `t`: groups of 4 lanes per entry, lane q copies vectors q, q + 4, ...
__device__ __forceinline__ void issue_piece( net_params const & p, int2 const * table, int a, int b, uint4 * buf, int t, int nthreads )
{
	if( a >= b ) return;
	int const pa = ent_off( table[a] );
	int const q = t & 3, groups = nthreads >> 2;
	for( int g = a + ( t >> 2 ); g < b; g += groups )
	{
		int2 const e = table[g];
		int const nv = ent_vec( e, p.pack );
		uint4 const * src = p.slices + (unsigned)e.x;
		uint4 * dst = buf + ( ent_off( e ) - pa );
		for( int j = q; j < nv; j += 4 ) cp_async16( dst + j, src + j );
	}
}

__device__ __forceinline__ void count_index( unsigned * cnt, unsigned x )
{
	if( x != SLICE_PAD ) atomicAdd( cnt + x, 1u );
}
__device__ __forceinline__ void count_index10( unsigned * cnt, unsigned x )
{
	if( x != SLICE_PAD10 ) atomicAdd( cnt + x, 1u );
}

// one counter increment per index of a slice vector (eight 16-bit or twelve 10-bit ones)
template <int PER>
__device__ __forceinline__ void count_vector( unsigned * cnt, uint4 const w )
{
	if constexpr( PER == 12 )
	{
		unsigned const q[4] = { w.x, w.y, w.z, w.w };
#pragma unroll
		for( int i = 0; i < 4; i++ )
		{
			count_index10( cnt, q[i] & 0x3FFu );
			count_index10( cnt, ( q[i] >> 10 ) & 0x3FFu );
			count_index10( cnt, ( q[i] >> 20 ) & 0x3FFu );
		}
	}
	else
	{
		count_index( cnt, w.x & 0xFFFFu );
		count_index( cnt, w.x >> 16 );
		count_index( cnt, w.y & 0xFFFFu );
		count_index( cnt, w.y >> 16 );
		count_index( cnt, w.z & 0xFFFFu );
		count_index( cnt, w.z >> 16 );
		count_index( cnt, w.w & 0xFFFFu );
		count_index( cnt, w.w >> 16 );
	}
}

// count every index of the `V` vectors in buf, by threads [0, nthreads) of numbering `t`
__device__ __forceinline__ void count_buffer( uint4 const * buf, int V, unsigned * cnt, int t, int nthreads, int pack )
{
	if( pack == 12 )
	{
#pragma unroll 2
		for( int v = t; v < V; v += nthreads ) count_vector<12>( cnt, buf[v] );
	}
	else
	{
#pragma unroll 2
		for( int v = t; v < V; v += nthreads ) count_vector<8>( cnt, buf[v] );
	}
}

// barrier of the first `threads` threads (whole warps) of the CTA
__device__ __forceinline__ void bar_sync_first( int threads ) { asm volatile( "bar.sync 1, %0;\n" ::"r"( threads ) : "memory" ); }
// barrier of the producer warps (producers - 1 warps before the last one, which compacts
// and publishes)
__device__ __forceinline__ void bar_sync_producers( int producers ) { asm volatile( "bar.sync 2, %0;\n" ::"r"( 32 * ( producers - 1 ) ) : "memory" ); }

// ascending compaction of a step's fired bits into the spike ring, by one warp: 32 words
// per round, a warp scan of their counts gives every word's offset; then the step is
// published to the other tiles
__device__ __forceinline__ void compact_step(
    net_params const & p, unsigned const * bits, int words, int d0, int tile, long long t, int lane, bool publish = true )
{
	int const slot_out = (int)( t % p.ring );
	int * out = p.ring_ids + (long long)slot_out * p.n + d0;
	// the step's summary record (nets with slots): count, then the first 31 ids
	int * summ = p.summ ? p.summ + ( (long long)slot_out * p.ntiles + tile ) * 32 : nullptr;
	int done = 0;
	for( int w0 = 0; w0 < words; w0 += 32 )
	{
		int const w = w0 + lane;
		unsigned m = w < words ? bits[w] : 0u;
		int const c = __popc( m );
		int const incl = warp_inclusive_scan( c );
		int off = done + incl - c;
		while( m )
		{
			int const b = __ffs( m ) - 1;
			m &= m - 1;
			int const id = d0 + ( w << 5 ) + b;
			if( summ && off < 31 ) summ[1 + off] = id;
			out[off++] = id;
		}
		done += __shfl_sync( 0xffffffffu, incl, 31 );
	}
	if( lane == 0 )
	{
		p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)done;
		if( summ ) summ[0] = done;
	}
	// every lane's ring writes, then the flag that publishes them (and every step before:
	// a caller may publish only every few steps)
	if( !publish ) return;
	__threadfence();
	__syncwarp();
	if( lane == 0 && tile != p.withhold_tile ) publish_step( p, tile, t );
}

// neuron state of the tile: shared memory [attrs][span] <-> registers / global memory
template <typename Decl, int I = 0>
struct smem_state
{
	template <typename Tup>
	__device__ __forceinline__ static void load( Tup & t, unsigned char const * base, int span, int local )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			tuple_at<I>::get( t ) = reinterpret_cast<T const *>( base + (size_t)I * span * 4 )[local];
			smem_state<Decl, I + 1>::load( t, base, span, local );
		}
	}
	template <typename Tup>
	__device__ __forceinline__ static void store( Tup & t, unsigned char * base, int span, int local )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			reinterpret_cast<T *>( base + (size_t)I * span * 4 )[local] = tuple_at<I>::get( t );
			smem_state<Decl, I + 1>::store( t, base, span, local );
		}
	}
	__device__ __forceinline__ static void from_global( void * const * a, long long d0, int span, unsigned char * base )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			static_assert( sizeof( T ) == 4, "attributes are 32-bit" );
			T const * g = static_cast<T const *>( a[I] ) + d0;
			T * sh = reinterpret_cast<T *>( base + (size_t)I * span * 4 );
			constexpr int B = 8; // loads in flight per thread
			int const nt = blockDim.x;
			for( int x0 = threadIdx.x; x0 < span; x0 += B * nt )
			{
				T v[B];
#pragma unroll
				for( int b = 0; b < B; b++ )
					if( x0 + b * nt < span ) v[b] = g[x0 + b * nt];
#pragma unroll
				for( int b = 0; b < B; b++ )
					if( x0 + b * nt < span ) sh[x0 + b * nt] = v[b];
			}
			smem_state<Decl, I + 1>::from_global( a, d0, span, base );
		}
	}
	__device__ __forceinline__ static void to_global( void * const * a, long long d0, int span, unsigned char const * base )
	{
		if constexpr( I < (int)Decl::size )
		{
			using T = typename Decl::template type<I>;
			T * g = static_cast<T *>( a[I] ) + d0;
			T const * sh = reinterpret_cast<T const *>( base + (size_t)I * span * 4 );
			for( int x = threadIdx.x; x < span; x += blockDim.x ) g[x] = sh[x];
			smem_state<Decl, I + 1>::to_global( a, d0, span, base );
		}
	}
};


// Launches of up to `delay` steps read only spikes of earlier launches. A longer launch
// (a cooperative launch: every CTA resident) reads spikes other tiles publish during it:
// before staging a step, a tile waits until every source tile has published the step
// `delay` earlier. With the pipeline checking five steps ahead that is a step before its
// own current one (delay >= 6), so the slowest tile never waits and every wait ends.
// Shorter delays run such launches on the synchronous path only (flat_sync): a step is
// staged after every tile has published the steps it reads, all before the current one.
template <typename Model>
__device__ __forceinline__ void window_flat_body( net_params const & p, int const tile, int L, float dt, int smem_bytes )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	constexpr int C = N::input_classes;
	static_assert( C >= 1, "window_flat needs a model with input classes" );
	constexpr int DT_AHEAD = MAX_WINDOW / 2; // compensated dt computed this many steps ahead

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW]; // dt of step k at k % MAX_WINDOW
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	__shared__ int step_begin[MAX_WINDOW + 1];
	__shared__ int step_vec[MAX_WINDOW + 1];
	// per-step staging results, slot s & 7: arrivals, vectors, ring offset, too large
	__shared__ int m_e[8], m_v[8], m_off[8], m_big[8];

	int const tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	int const nwc = nw - p.producers, ncons = nwc * 32; // consumer warps first, then producers
	int const d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	int const words = ( span + 31 ) >> 5;
	bool const inputs = __ldg( p.tile_inputs + tile ) != 0; // else no arrival ever reaches the tile
	snn_info const info{ p.n };

	unsigned char * state = smem;                                                          // [attrs][span]
	unsigned * bits2 = reinterpret_cast<unsigned *>( state + (size_t)N::size * span * 4 ); // [2][words]
	unsigned * cnt = bits2 + 2 * words;                                                    // [C][span], inputs only
	size_t const fixed = flat_fixed_bytes( C, (int)N::size, span );
	int * pcnt = reinterpret_cast<int *>( smem + fixed - (size_t)4 * FLAT_PC * 4 - (size_t)4 * FLAT_STEP_CAP * 8 ); // [4][FLAT_PC]
	int2 * ent = reinterpret_cast<int2 *>( pcnt + 4 * FLAT_PC );                           // [4][FLAT_STEP_CAP]
	uint4 * const ring = reinterpret_cast<uint4 *>( smem + fixed );
	int const rb = inputs ? (int)( ( (size_t)smem_bytes - fixed ) / 16 ) : 0; // ring vectors

	// the simulated clock: thread 0 advances the Kahan-compensated dt DT_AHEAD steps ahead
	if( tid == 0 )
	{
		clock_state const cs = *p.clock;
		float c = cs.c, sum = cs.sum;
		for( int k = 0; k < min( L, DT_AHEAD ); k++ )
		{
			s_dt[k % MAX_WINDOW] = kahan_add( c, sum, dt );
			if( tile == 0 ) p.dt_ring[( cs.step + k ) % DT_RING] = s_dt[k % MAX_WINDOW];
		}
		s_t0 = cs.step;
		s_c = c;
		s_sum = sum;
	}
	__syncthreads();
	long long const t0 = s_t0;
	auto advance_clock = [&]( int k ) { // at step k, by thread 0: the dt of step k + DT_AHEAD
		int const ka = k + DT_AHEAD;
		if( tid == 0 && ka < L )
		{
			float c = s_c, sum = s_sum;
			float const d = kahan_add( c, sum, dt );
			s_dt[ka % MAX_WINDOW] = d;
			s_c = c;
			s_sum = sum;
			if( tile == 0 ) p.dt_ring[( t0 + ka ) % DT_RING] = d;
		}
	};
	smem_state<N>::from_global( p.attr, d0, span, state );
	// counters start at zero; the update zeroes every counter it consumes
	if( inputs )
		for( int x = tid; x < C * span; x += nt ) cnt[x] = 0;
	__syncthreads();

	// update of step k by warps [0, nws): warp w owns neurons [32 w, 32 w + 32) + 32 nws r,
	// one fired-bit word each (bits of step k in half k & 1)
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
				// the ring slot of step t held step t - 2 delay: wait until every tile has
				// published step t - delay, so none still stages from the overwritten step
				// (tiles with inputs are bounded by their own waits)
				warp_wait_all_published( p, t0 + k - p.delay );
				compact( k );
			}
		}
		__syncthreads();
	}
	else
	{
		int k = 0; // next step to simulate
		while( k < L )
		{
			// ------------------------------------------------------------ pipelined steps
			int const kb = k; // the pipeline (re)starts at step kb
			// producer work during step j (j < kb: the prologue): every stage's loads go out
			// as asynchronous copies at once, one wait, then the scans that lay out the
			// next stages
			auto produce = [&]( int j, int pt, int npt, bool all ) {
				// slices of step j + 1: entry g's vectors to ring[(off + offset(g) + v) mod rb]
				int const sa = j + 1;
				bool const do_a = sa >= kb && sa < L && !m_big[sa & 7];
				if( do_a )
				{
					int2 const * e1 = ent + ( sa & 3 ) * FLAT_STEP_CAP;
					int const ea = m_e[sa & 7], oa = m_off[sa & 7];
					int const q = pt & 3, groups = npt >> 2;
					for( int g = pt >> 2; g < ea; g += groups )
					{
						int2 const e = e1[g];
						int const nv = ent_vec( e, p.pack );
						uint4 const * src = p.slices + (unsigned)e.x;
						int o = oa + ent_off( e ) + q;
						if( o >= rb ) o -= rb;
						for( int v = q; v < nv; v += 4 )
						{
							cp_async16( ring + o, src + v );
							o += 4;
							if( o >= rb ) o -= rb;
						}
					}
				}
				// slice records of step j + 2's arrivals, over their spike ids
				int const sb = j + 2;
				bool const do_b = sb >= kb && sb < L && !m_big[sb & 7];
				if( do_b )
				{
					int2 * e2 = ent + ( sb & 3 ) * FLAT_STEP_CAP;
					int const eb = m_e[sb & 7];
					for( int g = pt; g < eb; g += npt ) cp_async8( e2 + g, p.slice_rec + (long long)e2[g].x * p.ntiles + tile );
				}
				// spike ids of step j + 3 (its per-source-tile counts are scanned), one source
				// tile per thread
				int const sc = j + 3;
				if( sc >= kb && sc < L && !m_big[sc & 7] )
				{
					int const * pc = pcnt + ( sc & 3 ) * FLAT_PC;
					int2 * e3 = ent + ( sc & 3 ) * FLAT_STEP_CAP;
					long long const slot = ( ( t0 + sc - p.delay ) % p.ring ) * (long long)p.n;
					// source tile i's spikes are ring_ids[slot + tile_first[i] + r], r < its count
					for( int i = pt; i < p.ntiles; i += npt )
					{
						int const g0 = pc[i], g1 = pc[i + 1];
						if( g0 == g1 ) continue;
						int const * ids = p.ring_ids + slot + __ldg( p.tile_first + i );
						for( int r = 0; r < g1 - g0; r++ ) cp_async4( &e3[g0 + r].x, ids + r );
					}
				}
				// per-source-tile spike counts of step j + 4 (none before `delay`): every
				// source tile has published the step they fired in (checked during the step
				// before, or here in the prologue)
				int const sd = j + 4;
				bool const do_d = sd >= kb && sd < L;
				if( do_d )
				{
					int * pc = pcnt + ( sd & 3 ) * FLAT_PC;
					long long const t = t0 + sd;
					for( int i = pt; i < p.ntiles; i += npt )
					{
						if( t >= p.delay )
						{
							if( j < kb ) wait_published( p, i, t - p.delay );
							cp_async4( pc + i, p.ring_cnt + ( ( t - p.delay ) % p.ring ) * p.ntiles + i );
						}
						else
							pc[i] = 0;
					}
				}
				// publication of the spikes step j + 5 reads (a step before its own one for
				// delay >= 6: no wait in practice): checked here in the prologue, by the
				// publisher warp during the pipelined steps
				if( all && j + 5 >= kb && j + 5 < L && j + 5 + t0 >= p.delay )
					for( int i = pt; i < p.ntiles; i += npt ) wait_published( p, i, t0 + j + 5 - p.delay );
				cp_async_commit();
				cp_async_wait_all();
				if( all )
					__syncthreads();
				else
					bar_sync_producers( p.producers );
				// the two scans, one warp each, while another producer warp compacts
				int const pw = pt >> 5;
				if( do_b && pw == 0 )
				{
					// ring layout of step j + 2: per-entry vector offsets and the step's place
					int2 * e2 = ent + ( sb & 3 ) * FLAT_STEP_CAP;
					int const eb = m_e[sb & 7];
					int carry = 0;
					// four entries per lane and round (two 16-byte loads)
					for( int g0 = 0; g0 < eb; g0 += 128 )
					{
						int const g = g0 + 4 * lane;
						int4 const a01 = g < eb ? reinterpret_cast<int4 const *>( e2 )[g >> 1] : make_int4( 0, 0, 0, 0 );
						int4 const a23 = g + 2 < eb ? reinterpret_cast<int4 const *>( e2 )[( g >> 1 ) + 1] : make_int4( 0, 0, 0, 0 );
						int2 e[4] = { make_int2( a01.x, a01.y ), make_int2( a01.z, a01.w ), make_int2( a23.x, a23.y ), make_int2( a23.z, a23.w ) };
						int nv[4], sum = 0;
#pragma unroll
						for( int u = 0; u < 4; u++ )
						{
							nv[u] = g + u < eb ? ent_vec( e[u], p.pack ) : 0;
							sum += nv[u];
						}
						int const incl = warp_inclusive_scan( sum );
						int off = carry + incl - sum;
#pragma unroll
						for( int u = 0; u < 4; u++ )
							if( g + u < eb )
							{
								e2[g + u] = make_int2( e[u].x, ent_len( e[u] ) | ( off << 12 ) );
								off += nv[u];
							}
						carry += __shfl_sync( 0xffffffffu, incl, 31 );
					}
					if( lane == 0 )
					{
						int const prev_v = sb > kb ? m_v[( sb - 1 ) & 7] : 0, prev_off = sb > kb ? m_off[( sb - 1 ) & 7] : 0;
						m_v[sb & 7] = carry;
						int o = prev_off + prev_v;
						if( o >= rb ) o -= rb;
						m_off[sb & 7] = o;
						// two steps live in the ring at once: the one counted and the one copied
						if( carry + prev_v > rb || carry >= ( 1 << FLAT_P_BITS ) ) m_big[sb & 7] = 1;
					}
				}
				if( do_d && pw == 1 )
				{
					// exclusive prefix of step j + 4's per-source-tile counts: its arrivals
					int * pc = pcnt + ( sd & 3 ) * FLAT_PC;
					int carry = 0;
					for( int i0 = 0; i0 < p.ntiles; i0 += 32 )
					{
						int const i = i0 + lane;
						int const c = i < p.ntiles ? pc[i] : 0;
						int const incl = warp_inclusive_scan( c );
						if( i < p.ntiles ) pc[i] = carry + incl - c;
						carry += __shfl_sync( 0xffffffffu, incl, 31 );
					}
					if( lane == 0 )
					{
						pc[p.ntiles] = carry;
						m_e[sd & 7] = carry;
						m_big[sd & 7] = carry > FLAT_STEP_CAP ? 1 : 0;
					}
				}
			};

			int ks = L; // first step of a synchronous stretch, if any
			if( !p.flat_sync )
			{
				for( int j = kb - 4; j < kb; j++ )
				{
					// the prologue: every warp stages (nobody counts yet)
					produce( j, tid, nt, true );
					__syncthreads();
				}
				for( ; k < L; k++ )
				{
					if( m_big[k & 7] )
					{
						ks = k; // this step takes the synchronous path
						break;
					}
					advance_clock( k );
					if( warp < nwc )
					{
						if( t0 + k >= p.delay )
						{
							// count the ring region [off, off + V) of step k
							int const v = m_v[k & 7], o = m_off[k & 7];
							if( p.pack == 12 )
							{
#pragma unroll 2
								for( int x = tid; x < v; x += ncons )
								{
									int y = o + x;
									if( y >= rb ) y -= rb;
									count_vector<12>( cnt, ring[y] );
								}
							}
							else
							{
#pragma unroll 2
								for( int x = tid; x < v; x += ncons )
								{
									int y = o + x;
									if( y >= rb ) y -= rb;
									count_vector<8>( cnt, ring[y] );
								}
							}
						}
						bar_sync_first( ncons ); // counts complete
						update( k, nwc );
					}
					else if( warp == nw - 1 )
					{
						// the publisher warp: step k - 1's spikes to the ring, fenced, then its
						// flag (the fence waits for the stores; no producer waits on it); then
						// the publication of the spikes step k + 5 reads, for the producers'
						// next step (relaxed reads of every flag, one acquire fence)
						if( k > kb ) compact( k - 1 );
						if( k + 5 < L && t0 + k + 5 >= p.delay ) warp_wait_all_published( p, t0 + k + 5 - p.delay );
					}
					else
						produce( k, tid - ncons, nt - ncons - 32, false );
					__syncthreads(); // step k updated, step k + 1's slices in the ring
				}
				if( k > kb && warp == nw - 1 ) compact( k - 1 ); // the last pipelined step
				__syncthreads();
			}
			else
				ks = k;
			if( ks >= L ) break;

			// ------------------------------------------------------------ synchronous steps
			// staging of whole steps (those whose spikes are published already: fewer than
			// `delay` steps ahead), table, scratch and buffer in the slice ring; back to the
			// pipeline after the first segment unless every step goes this way
			int2 * table = reinterpret_cast<int2 *>( ring );
			unsigned * cnts = reinterpret_cast<unsigned *>( table + FLAT_ENT_CAP );
			uint4 * buf = reinterpret_cast<uint4 *>( cnts + FLAT_SCRATCH );
			int const bufv = rb - ( FLAT_ENT_CAP * 8 + FLAT_SCRATCH * 4 ) / 16;
			int mode;
			int const ke = stage_table( p, cnts, table, tile, t0, ks, min( L, ks + p.delay ), step_begin, step_vec, scratch, bufv, mode );
			for( int kk = ks; kk < ke; kk++ )
			{
				advance_clock( kk );
				long long const t = t0 + kk;
				if( t >= p.delay )
				{
					if( mode == SEG_DIRECT )
					{
						// the direct path of window_counts, its scratch in the (unused) table
						int * pref = reinterpret_cast<int *>( table );
						int4 * sbuf = reinterpret_cast<int4 *>( reinterpret_cast<unsigned char *>( table ) + ( ( ( p.ntiles + 1 ) * 4 + 15 ) & ~15 ) );
						net_params q = p;
						q.tile = span; // counter rows are span long
						for( int i = tid; i < p.ntiles; i += nt ) wait_published( p, i, t - p.delay );
						__syncthreads();
						deliver_counts<N>( q, (int)( ( t - p.delay ) % p.ring ), tile, d0, d1, cnt, pref, sbuf, scratch );
					}
					else
					{
						// slices in pieces that fit the buffer
						int const e = step_begin[kk + 1 - ks];
						int const sv = step_vec[kk + 1 - ks] - step_vec[kk - ks];
						for( int a = step_begin[kk - ks], b = a; b < e; )
						{
							a = b;
							b = piece_end( table, a, e, bufv, p.pack );
							issue_piece( p, table, a, b, buf, tid, nt );
							cp_async_commit();
							cp_async_wait_all();
							__syncthreads();
							count_buffer( buf, piece_vectors( table, a, b, e, sv ), cnt, tid, nt, p.pack );
							__syncthreads();
						}
					}
				}
				__syncthreads();
				update( kk, nw );
				__syncthreads();
				if( warp == nw - 1 ) compact( kk );
				__syncthreads();
			}
			k = ke;
		}
	}

	smem_state<N>::to_global( p.attr, d0, span, state );
	window_clock_end( p, L, t0, s_c, s_sum );
}

// one net: CTA j runs tile j
template <typename Model>
__global__ void __launch_bounds__( FLAT_THREADS, 1 ) window_flat( net_params p, int L, float dt, int smem_bytes )
{
	window_flat_body<Model>( p, blockIdx.x, L, dt, smem_bytes );
}

// Many independent nets of one model in one launch (batching): CTA b runs tile jobs[b].y
// of net jobs[b].x for jobs[b].z steps of dt __int_as_float(jobs[b].w); every net's steps
// read only spikes of earlier launches (jobs[b].z <= that net's delay).
template <typename Model>
__global__ void __launch_bounds__( FLAT_THREADS, 1 ) window_flat_batch( net_params const * nets, int4 const * jobs, int smem_bytes )
{
	__shared__ net_params s_p;
	int4 const j = jobs[blockIdx.x];
	if( threadIdx.x == 0 ) s_p = nets[j.x];
	__syncthreads();
	if( j.z > 0 ) window_flat_body<Model>( s_p, j.y, j.z, __int_as_float( j.w ), smem_bytes );
}
} // namespace spk
