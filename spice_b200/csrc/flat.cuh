// Window kernel for models with input classes (non-plastic), shaped by measurement.
//
// Same results as window_counts (kernels.cuh). Per launch -- one delay window of L steps --
// a CTA owns one tile of destination neurons [tile_first[j], tile_first[j + 1]).
//
// Data layout ("slices"). Besides the ELL rows, the net keeps every row's part inside
// every tile as a slice of 16-bit counter indices, class(src) * span + (target - d0),
// padded with SLICE_PAD to a whole 16-byte vector. A tile's slices lie contiguously in
// ascending source order, and rec[src * ntiles + tile] = { first vector, length }. So a
// CTA reads only its own tile's region, two bytes per synapse, already in the form its
// counters are indexed by.
//
//   1. Staging. All arrivals of the window fired before it started, so the CTA stages the
//      window's arrival table (first vector, length, vector offset inside the step) in
//      shared memory: per-(step, source tile) spike counts, spike ids, slice records.
//   2. Prefetch. The slices of step k + 2 are copied into one of two shared-memory
//      buffers with cp.async while step k is updated, so the loads of a step overlap the
//      work of the step before it.
//   3. Counting. Threads walk the step's buffer one 16-byte vector at a time and count
//      every index with a shared-memory atomic. A step larger than a buffer is counted in
//      pieces that are loaded synchronously.
//   4. Update. The tile's neuron state lives in shared memory for the whole window; the
//      counts are replayed through the model's receive(), the model updates every neuron
//      and the counters it consumed are zeroed; fired neurons are compacted in ascending
//      order into the spike ring. Two barriers per step.
// Keeping the state in shared memory lets tile sizes follow the work (balanced tiles): a
// population without inputs costs little per neuron and gets few, large tiles.
//
// Measured on B200 (Brunel, 1e9 synapses): with 4-byte row loads issued one step at a
// time the counting phase waited on memory for most of a step; the layout and the
// two-step-ahead copies remove both the wait and half the bytes.
#pragma once

#include "kernels.cuh"

namespace spk
{
constexpr int FLAT_THREADS = 1024;  // threads of a window_flat CTA (one CTA per SM)
constexpr int FLAT_ENT_CAP = 8192;  // staged arrivals per segment of a window
constexpr int FLAT_SCRATCH = 4096;  // per-(step, source tile) counts staged at once
constexpr int FLAT_MAX_TILE = 4064; // slice lengths fit the table's 12-bit field
constexpr int FLAT_MIN_BUF = 512;   // vectors per buffer at least (one slice of a full tile)
constexpr int FLAT_P_BITS = 20;     // vector offsets inside a step held in the table
constexpr int FLAT_STAGE_CAP = 16384; // arrivals per window stage_window stages
constexpr unsigned short SLICE_PAD = 0xFFFFu;

// shared memory of a CTA: neuron state [attrs][span], fired bits [2][words]; tiles with
// inputs add counters [classes][span], the arrival table, staging scratch and two slice
// buffers in what is left
__host__ __device__ inline size_t flat_state_bytes( int attrs, int span )
{
	return (size_t)attrs * span * 4 + 2 * ( ( (size_t)span + 31 ) / 32 ) * 4;
}
__host__ __device__ inline size_t flat_fixed_bytes( int classes, int attrs, int span )
{
	size_t b = flat_state_bytes( attrs, span ) + (size_t)classes * span * 4;
	b = ( b + 15 ) & ~(size_t)15;
	return b + (size_t)FLAT_ENT_CAP * 8 + (size_t)FLAT_SCRATCH * 4;
}
inline size_t flat_smem_bytes( int classes, int attrs, int tmax )
{
	return flat_fixed_bytes( classes, attrs, tmax ) + (size_t)2 * FLAT_MIN_BUF * 16;
}

// ------------------------------------------------------------------------------------
// building the slices (once per net)
// ------------------------------------------------------------------------------------
// 16-byte vectors of a slice of `len` targets: a list of 16-bit indices (dense == 0) or
// a bitmap of the tile's `words` receiving 32-neuron words (dense == 1, none if len == 0)
__host__ __device__ inline unsigned slice_vecs( unsigned len, int words, int dense )
{
	if( !dense ) return ( len + 7 ) >> 3;
	return len ? (unsigned)( ( words + 3 ) / 4 ) : 0u;
}

// lowest and highest tile-local target of every tile over all rows (tiles without
// inputs keep lo = INT_MAX)
__global__ void tile_target_range(
    int n, int width, int ntiles, int const * edges, unsigned const * pivots, int const * tile_first, int * lo, int * hi )
{
	long long const total = (long long)n * ntiles;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x )
	{
		long long const src = e / ntiles;
		int const j = (int)( e % ntiles );
		unsigned const * pv = pivots + src * ( ntiles + 1 ) + j;
		if( pv[1] > pv[0] )
		{
			int const * row = edges + src * width;
			atomicMin( lo + j, row[pv[0]] - tile_first[j] );
			atomicMax( hi + j, row[pv[1] - 1] - tile_first[j] );
		}
	}
}

// vectors of every (src, tile) slice, from the ELL pivots, into rec[].x; rec[].y = length
__global__ void slice_vectors( int n, int ntiles, unsigned const * pivots, int2 const * bm_range, int dense, uint2 * rec )
{
	long long const total = (long long)n * ntiles;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x )
	{
		long long const src = e / ntiles, j = e % ntiles;
		unsigned const * pv = pivots + src * ( ntiles + 1 ) + j;
		unsigned const len = pv[1] - pv[0];
		rec[e] = make_uint2( slice_vecs( len, bm_range[j].y, dense ), len );
	}
}

// per tile (one CTA of 1024 threads each): rec[src][tile].x <- exclusive prefix over src
// of the vector counts (tile-relative), totals[tile] <- the tile's vectors
__global__ void __launch_bounds__( 1024 ) slice_offsets( int n, int ntiles, uint2 * rec, unsigned long long * totals )
{
	__shared__ unsigned long long s_run[1024];
	int const j = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
	long long const per = ( (long long)n + nt - 1 ) / nt;
	long long const s0 = min( (long long)n, tid * per ), s1 = min( (long long)n, s0 + per );
	unsigned long long run = 0;
	for( long long s = s0; s < s1; s++ ) run += rec[s * ntiles + j].x;
	s_run[tid] = run;
	__syncthreads();
	if( tid < 32 )
	{
		// 64-bit exclusive scan of the per-thread sums: lane l owns nt / 32 consecutive ones
		int const chunk = nt / 32;
		unsigned long long acc = 0;
		for( int i = 0; i < chunk; i++ ) acc += s_run[tid * chunk + i];
		unsigned long long incl = acc;
		for( int o = 1; o < 32; o <<= 1 )
		{
			unsigned long long const y = __shfl_up_sync( 0xffffffffu, incl, o );
			if( tid >= o ) incl += y;
		}
		unsigned long long base = incl - acc;
		for( int i = 0; i < chunk; i++ )
		{
			unsigned long long const v = s_run[tid * chunk + i];
			s_run[tid * chunk + i] = base;
			base += v;
		}
		if( tid == 31 ) totals[j] = incl;
	}
	__syncthreads();
	unsigned long long off = s_run[tid];
	for( long long s = s0; s < s1; s++ )
	{
		uint2 & r = rec[s * ntiles + j];
		unsigned const v = r.x;
		r.x = (unsigned)off;
		off += v;
	}
}

// one warp per source row: rebase rec[] to global vector indices and write every slice.
// Lists: rec.y = length. Bitmaps: rec.y = 1 | class << 1 for a slice with targets, 0 else.
template <typename Model, bool Dense>
__global__ void __launch_bounds__( 256 ) slice_fill(
    int n, int width, int ntiles, int const * edges, unsigned const * pivots, int const * tile_first, int2 const * bm_range,
    unsigned long long const * tile_base, uint2 * rec, unsigned short * slices )
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
		unsigned long long const first = tile_base[j] + r.x;
		unsigned const y = Dense ? ( r.y ? 1u | (unsigned)cls << 1 : 0u ) : r.y;
		__syncwarp();
		if( lane == 0 ) rec[(long long)src * ntiles + j] = make_uint2( (unsigned)first, y );
		if( r.y == 0 ) continue;
		int const d0 = tile_first[j], span = tile_first[j + 1] - d0;
		unsigned const lo = pv[j];
		if constexpr( Dense )
		{
			unsigned * out = reinterpret_cast<unsigned *>( slices ) + first * 4;
			int2 const br = bm_range[j];
			int const padded = (int)slice_vecs( r.y, br.y, 1 ) * 4;
			for( int e = lane; e < padded; e += 32 ) out[e] = 0u;
			__syncwarp();
			for( int e = lane; e < (int)r.y; e += 32 )
			{
				int const local = row[lo + e] - d0 - 32 * br.x;
				atomicOr( out + ( local >> 5 ), 1u << ( local & 31 ) );
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

// ------------------------------------------------------------------------------------
// stage_window: the arrivals of the next window for every tile at once
// ------------------------------------------------------------------------------------
// Runs before window_flat. All CTAs compute the window's (step, source tile) prefix; then
// each takes chunks of `chunk` arrivals, reads every arrival's record row rec[src][*]
// (contiguous, coalesced) into shared memory and writes it out transposed, one run of
// `chunk` consecutive entries per tile: wtab[tile][g] = rec[src_g][tile]. A window_flat
// CTA then loads its table as one contiguous run instead of one scattered record load per
// arrival. wsteps[k] = first entry of step k (k <= L), wsteps[MAX_WINDOW + 1] = 1 if the
// window fits ecap (else window_flat stages by itself).
inline size_t stage_window_smem( int ntiles, int chunk ) { return (size_t)FLAT_SCRATCH * 4 + (size_t)chunk * ( ntiles * 8 + 4 ); }

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
				if( t >= p.delay ) v[b] = __ldcg( p.ring_cnt + (long long)( ( t - p.delay ) % p.ring ) * p.ntiles + i );
			}
		}
#pragma unroll
		for( int b = 0; b < B; b++ )
			if( q0 + b * nt < M ) cnts[q0 + b * nt] = v[b];
	}
	__syncthreads();
}

__global__ void __launch_bounds__( 256 ) stage_window( net_params p, int L, int chunk )
{
	extern __shared__ __align__( 16 ) unsigned char smem[];
	__shared__ int scratch[33];
	unsigned * pref = reinterpret_cast<unsigned *>( smem );                 // [FLAT_SCRATCH]
	uint2 * srec = reinterpret_cast<uint2 *>( pref + FLAT_SCRATCH );        // [chunk][ntiles]
	int * ssrc = reinterpret_cast<int *>( srec + (size_t)chunk * p.ntiles ); // [chunk]
	int const tid = threadIdx.x, nt = blockDim.x, nti = p.ntiles;
	int const M = L * nti;
	if( M + 1 > FLAT_SCRATCH )
	{
		if( blockIdx.x == 0 && tid == 0 ) p.wsteps[MAX_WINDOW + 1] = 0;
		return;
	}
	long long const t0 = __ldcg( &p.clock->step );
	load_counts( p, pref, t0, 0, L, scratch );
	int total;
	{
		int const per = ( M + nt - 1 ) / nt;
		int const q0 = min( M, tid * per ), q1 = min( M, q0 + per );
		int run = 0;
		for( int q = q0; q < q1; q++ ) run += (int)pref[q];
		int base = block_exclusive_scan( run, scratch, &total );
		for( int q = q0; q < q1; q++ )
		{
			int const c = (int)pref[q];
			pref[q] = (unsigned)base;
			base += c;
		}
		if( tid == 0 ) pref[M] = (unsigned)total;
	}
	__syncthreads();
	bool const fits = total <= p.ecap;
	if( blockIdx.x == 0 )
	{
		for( int k = tid; k <= L; k += nt ) p.wsteps[k] = (int)pref[k * nti];
		if( tid == 0 ) p.wsteps[MAX_WINDOW + 1] = fits ? 1 : 0;
	}
	if( !fits ) return;
	for( int g0 = blockIdx.x * chunk; g0 < total; g0 += gridDim.x * chunk )
	{
		int const m = min( chunk, total - g0 );
		if( tid < m )
		{
			int const g = g0 + tid;
			int q = 0, hi = M; // last pair q with pref[q] <= g
			while( hi - q > 1 )
			{
				int const mid = ( q + hi ) >> 1;
				if( (int)pref[mid] <= g )
					q = mid;
				else
					hi = mid;
			}
			int const k = q / nti, i = q % nti;
			long long const t = t0 + k;
			ssrc[tid] = __ldcg( p.ring_ids + (long long)( ( t - p.delay ) % p.ring ) * p.n + __ldg( p.tile_first + i ) + ( g - (int)pref[q] ) );
		}
		__syncthreads();
		constexpr int B = 8;
		int const items = m * nti;
		for( int x0 = tid; x0 < items; x0 += B * nt )
		{
			uint2 v[B];
#pragma unroll
			for( int b = 0; b < B; b++ )
			{
				int const x = x0 + b * nt;
				if( x < items ) v[b] = __ldg( p.slice_rec + (long long)ssrc[x / nti] * nti + x % nti );
			}
#pragma unroll
			for( int b = 0; b < B; b++ )
				if( x0 + b * nt < items ) srec[x0 + b * nt] = v[b];
		}
		__syncthreads();
		for( int x = tid; x < nti * chunk; x += nt )
		{
			int const j = x / chunk, e = x % chunk;
			if( e < m ) p.wtab[(long long)j * p.ecap + g0 + e] = srec[e * nti + j];
		}
		__syncthreads();
	}
}

// ------------------------------------------------------------------------------------
// window kernel
// ------------------------------------------------------------------------------------
// table[g] = { first vector of the slice, low | vector offset inside its step << 12 } with
// low = length (lists) or 1 | class << 1 for a bitmap with targets (bitmaps: `wv` vectors
// each; wv == 0 selects lists)
__device__ __forceinline__ int ent_low( int2 e ) { return e.y & 0xFFF; }
__device__ __forceinline__ int ent_vec( int2 e, int wv ) { return wv ? ( ent_low( e ) & 1 ) * wv : ( ent_low( e ) + 7 ) >> 3; }
__device__ __forceinline__ int ent_cls( int2 e ) { return ( ent_low( e ) >> 1 ) & 7; }
__device__ __forceinline__ int ent_off( int2 e ) { return (int)( (unsigned)e.y >> 12 ); }

__device__ __forceinline__ int stage_arrivals(
    net_params const & p, unsigned * cnts, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int & nent_out, int * scratch );
__device__ __forceinline__ int stage_offsets(
    int2 * table, int ks, int ke, int nent, int * step_begin, int * step_vec, int * run_first, int * scratch, int wv );

// Stage the arrivals of the steps [ks, L) of the window starting at t0, as many whole
// steps as fit FLAT_ENT_CAP and keep their vector offsets within FLAT_P_BITS. Returns
// ke: steps [ks, ke) are staged (ke == ks: step ks goes the direct way).
// step_begin[k - ks] = first entry of step k and step_vec[k - ks] = first vector of step
// k counted from the segment start, for k in [ks, ke].
__device__ __forceinline__ int stage_table(
    net_params const & p, unsigned * cnts, int2 * table, int tile, long long t0, int ks, int L, int * step_begin, int * step_vec,
    int * scratch, int wv )
{
	constexpr int B = 8; // loads in flight per thread
	int const tid = threadIdx.x, nt = blockDim.x;
	int ke = ks, nent = 0;
	if( p.ecap > 0 && __ldcg( p.wsteps + MAX_WINDOW + 1 ) )
	{
		// staged by stage_window: whole steps that fit the table, one contiguous run
		for( int k = ks + tid; k <= L; k += nt ) step_vec[k - ks] = __ldcg( p.wsteps + k ); // scratch use
		__syncthreads();
		int const base = step_vec[0];
		while( ke < L && step_vec[ke + 1 - ks] - base <= FLAT_ENT_CAP ) ke++;
		nent = step_vec[ke - ks] - base;
		__syncthreads();
		for( int k = tid; k <= ke - ks; k += nt ) step_begin[k] = step_vec[k] - base;
		uint2 const * src = p.wtab + (long long)tile * p.ecap + base;
		for( int g0 = tid; g0 < nent; g0 += B * nt )
		{
			uint2 v[B];
#pragma unroll
			for( int b = 0; b < B; b++ )
				if( g0 + b * nt < nent ) v[b] = __ldcg( src + g0 + b * nt );
#pragma unroll
			for( int b = 0; b < B; b++ )
				if( g0 + b * nt < nent ) table[g0 + b * nt] = make_int2( (int)v[b].x, (int)v[b].y );
		}
		__syncthreads();
	}
	else
		ke = stage_arrivals( p, cnts, table, tile, t0, ks, L, step_begin, nent, scratch );
	return stage_offsets( table, ks, ke, nent, step_begin, step_vec, reinterpret_cast<int *>( cnts ), scratch, wv );
}

// Per-CTA staging (when stage_window did not run or the window did not fit): the
// (step, source tile) prefix, then every arrival's spike id and slice record. Returns ke.
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
// A step whose vectors do not fit the offset field ends the segment before it; returns
// the segment's end.
__device__ __forceinline__ int stage_offsets(
    int2 * table, int ks, int ke, int nent, int * step_begin, int * step_vec, int * run_first, int * scratch, int wv )
{
	int const tid = threadIdx.x, nt = blockDim.x;
	int const per = ( nent + nt - 1 ) / nt;
	int const g0 = min( nent, tid * per ), g1 = min( nent, g0 + per );
	int run = 0;
	for( int g = g0; g < g1; g++ ) run += ent_vec( table[g], wv );
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
			for( int h = owner * per; h < g; h++ ) v += ent_vec( table[h], wv );
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
			int const nv = ent_vec( e, wv );
			e.y = ent_low( e ) | (int)( ( rel & ( ( 1u << FLAT_P_BITS ) - 1 ) ) << 12 );
			table[g] = e;
			v += nv;
		}
	}
	// 6. a step whose vectors do not fit the offset field ends the segment before it
	int kfit = ks;
	while( kfit < ke && step_vec[kfit + 1 - ks] - step_vec[kfit - ks] < ( 1 << FLAT_P_BITS ) ) kfit++;
	__syncthreads();
	return kfit;
}

// one past the last entry of the piece starting at entry `a` of a step whose entries end
// at `e`: the entries whose vectors fit one buffer of `bufv` vectors together
__device__ __forceinline__ int piece_end( int2 const * table, int a, int e, int bufv, int wv )
{
	int const pa = ent_off( table[a] );
	int lo = a, hi = e; // f(g) = off(g) + vec(g) - pa <= bufv holds for g = a
	while( hi - lo > 1 )
	{
		int const mid = ( lo + hi ) >> 1;
		int2 const m = table[mid];
		if( ent_off( m ) + ent_vec( m, wv ) - pa <= bufv )
			lo = mid;
		else
			hi = mid;
	}
	return lo + 1;
}

__device__ __forceinline__ void cp_async16( void * dst, void const * src )
{
	unsigned const d = (unsigned)__cvta_generic_to_shared( dst );
	asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"( d ), "l"( src ) : "memory" );
}
__device__ __forceinline__ void cp_async_commit() { asm volatile( "cp.async.commit_group;\n" ::: "memory" ); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile( "cp.async.wait_group 0;\n" ::: "memory" ); }

// copy the slices of entries [a, b) into buf: groups of 8 lanes per entry, lane q copies
// vectors q, q + 8, ... (a warp instruction touches 4 slices, not 32)
__device__ __forceinline__ void issue_piece( net_params const & p, int2 const * table, int a, int b, uint4 * buf, int wv )
{
	if( a >= b ) return;
	int const pa = ent_off( table[a] );
	int const q = threadIdx.x & 7, groups = blockDim.x >> 3;
	for( int g = a + (int)( threadIdx.x >> 3 ); g < b; g += groups )
	{
		int2 const e = table[g];
		int const nv = ent_vec( e, wv );
		uint4 const * src = p.slices + (unsigned)e.x;
		uint4 * dst = buf + ( ent_off( e ) - pa );
		for( int j = q; j < nv; j += 8 ) cp_async16( dst + j, src + j );
	}
}

__device__ __forceinline__ void count_index( unsigned * cnt, unsigned x )
{
	if( x != SLICE_PAD ) atomicAdd( cnt + x, 1u );
}

// count every index of the `V` vectors in buf
__device__ __forceinline__ void count_buffer( uint4 const * buf, int V, unsigned * cnt )
{
#pragma unroll 2
	for( int v = threadIdx.x; v < V; v += blockDim.x )
	{
		uint4 const w = buf[v];
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

// vectors of the piece [a, b) of a step whose entries end at e (step_vectors in all)
__device__ __forceinline__ int piece_vectors( int2 const * table, int a, int b, int e, int step_vectors )
{
	if( a >= b ) return 0;
	return ( b < e ? ent_off( table[b] ) : step_vectors ) - ent_off( table[a] );
}

// 32 x 32 bit transpose across a warp: afterwards bit j of lane l is bit l of lane j
__device__ __forceinline__ unsigned warp_transpose32( unsigned x, int lane )
{
#pragma unroll
	for( int s = 16; s >= 1; s >>= 1 )
	{
		unsigned const m = s == 16 ? 0x0000FFFFu : s == 8 ? 0x00FF00FFu : s == 4 ? 0x0F0F0F0Fu : s == 2 ? 0x33333333u : 0x55555555u;
		unsigned const y = __shfl_xor_sync( 0xffffffffu, x, s );
		// lanes with bit s set keep their high halves and take the partner's high halves
		// shifted down, the others keep their low halves and take the partner's low halves
		// shifted up (~m >> s == m for these masks)
		bool const up = lane & s;
		unsigned const keep = up ? ~m : m;
		unsigned const z = up ? y >> s : y << s;
		x = ( x & keep ) | ( z & ~keep );
	}
	return x;
}

// Bitmap counting. Slots [s0, s1) lie in `buf` from slot `base` on, `ww` words each. For
// bitmap word w, lane l adds the words of slots s0 + l, s0 + l + 32, ... into four bit
// planes (a per-bit counter up to 15), in rounds of 15 slots per lane; transposing a plane
// makes lane l's popcount the number of planes' bits l over all lanes. Returns this lane's
// count for bit `lane` of word w.
__device__ __forceinline__ unsigned bitmap_count( unsigned const * buf, int base, int s0, int s1, int ww, int w, int lane )
{
	unsigned total = 0;
	for( int r0 = s0; r0 < s1; r0 += 15 * 32 )
	{
		int const r1 = min( s1, r0 + 15 * 32 );
		unsigned p0 = 0, p1 = 0, p2 = 0, p3 = 0;
		for( int s = r0 + lane; s < r1; s += 32 )
		{
			unsigned c = buf[( s - base ) * ww + w];
			unsigned t = p0 & c;
			p0 ^= c;
			c = t;
			t = p1 & c;
			p1 ^= c;
			c = t;
			t = p2 & c;
			p2 ^= c;
			p3 ^= t; // no carry out: a lane adds at most 15 words
		}
		// planes needed for the largest lane count (uniform across the warp)
		int const most = ( r1 - r0 + 31 ) >> 5;
		if( most >= 8 )
		{
			unsigned const a = warp_transpose32( p0, lane ), b = warp_transpose32( p1, lane ), c = warp_transpose32( p2, lane ),
			               d = warp_transpose32( p3, lane );
			total += __popc( a ) + ( __popc( b ) << 1 ) + ( __popc( c ) << 2 ) + ( __popc( d ) << 3 );
		}
		else if( most >= 4 )
		{
			unsigned const a = warp_transpose32( p0, lane ), b = warp_transpose32( p1, lane ), c = warp_transpose32( p2, lane );
			total += __popc( a ) + ( __popc( b ) << 1 ) + ( __popc( c ) << 2 );
		}
		else if( most >= 2 )
		{
			unsigned const a = warp_transpose32( p0, lane ), b = warp_transpose32( p1, lane );
			total += __popc( a ) + ( __popc( b ) << 1 );
		}
		else
			total += __popc( warp_transpose32( p0, lane ) );
	}
	return total;
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

template <typename Model, bool Dense>
__global__ void __launch_bounds__( FLAT_THREADS, 1 ) window_flat( net_params p, int L, float dt, int smem_bytes )
{
	using N = typename Model::neuron;
	using Tup = typename N::template apply<reg_tuple>;
	constexpr int C = N::input_classes;
	static_assert( C >= 1, "window_flat needs a model with input classes" );
	static_assert( !Dense || C <= 4, "bitmap slices carry up to four input classes" );

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	__shared__ int step_begin[MAX_WINDOW + 1];
	__shared__ int step_vec[MAX_WINDOW + 1];
	__shared__ int s_cslots[MAX_WINDOW][4]; // bitmaps: slots of every input class per step

	int const tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	int const tile = blockIdx.x, d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	int const words = ( span + 31 ) >> 5;
	// bitmaps: words [bw0, bw0 + bwn) of the tile hold all its targets, wv vectors each
	int2 const brange = Dense ? __ldg( p.bm_range + tile ) : make_int2( 0, 0 );
	int const bw0 = brange.x, bwn = brange.y;
	int const wv = Dense ? max( 1, ( bwn + 3 ) >> 2 ) : 0;
	bool const inputs = __ldg( p.tile_inputs + tile ) != 0; // else no arrival ever reaches the tile
	snn_info const info{ p.n };

	unsigned char * state = smem;                                                          // [attrs][span]
	unsigned * bits2 = reinterpret_cast<unsigned *>( state + (size_t)N::size * span * 4 ); // [2][words]
	unsigned * cnt = bits2 + 2 * words;                                                    // [C][span], inputs only
	size_t const fixed = flat_fixed_bytes( C, (int)N::size, span );
	int2 * table = reinterpret_cast<int2 *>( smem + fixed - (size_t)FLAT_ENT_CAP * 8 - (size_t)FLAT_SCRATCH * 4 );
	unsigned * cnts = reinterpret_cast<unsigned *>( table + FLAT_ENT_CAP );
	int const bufv = (int)( ( (size_t)smem_bytes - fixed ) / 32 );
	uint4 * const buf0 = reinterpret_cast<uint4 *>( smem + fixed );
	uint4 * const buf1 = buf0 + bufv;

	window_clock_begin( p, L, dt, s_dt, &s_t0, &s_c, &s_sum );
	long long const t0 = s_t0;
	smem_state<N>::from_global( p.attr, d0, span, state );
	// counters start at zero; the update phase zeroes every counter it consumes
	if( inputs )
		for( int x = tid; x < C * span; x += nt ) cnt[x] = 0;
	__syncthreads();

	int ks = 0;
	while( ks < L )
	{
		int const ke = inputs ? stage_table( p, cnts, table, tile, t0, ks, L, step_begin, step_vec, scratch, wv ) : L;
		bool const direct = ke == ks; // step ks alone exceeds the table
		int const kend = direct ? ks + 1 : ke;
		bool const piped = inputs && !direct; // slices flow through the two buffers
		if( Dense && piped )
		{
			// bitmaps of every input class per step (slots ascend with the source id, and so
			// does the class)
			for( int x = tid; x < ( kend - ks ) * 4; x += nt ) s_cslots[x >> 2][x & 3] = 0;
			__syncthreads();
			int const nent = step_begin[kend - ks];
			for( int g = tid; g < nent; g += nt )
			{
				int2 const e = table[g];
				if( ent_low( e ) & 1 )
				{
					int lo = 0, hi = kend - ks; // step of g: last k with step_begin[k] <= g
					while( hi - lo > 1 )
					{
						int const mid = ( lo + hi ) >> 1;
						if( step_begin[mid] <= g )
							lo = mid;
						else
							hi = mid;
					}
					atomicAdd( &s_cslots[lo][ent_cls( e )], 1 );
				}
			}
			__syncthreads();
		}

		// first piece [a, b) of step k
		auto first_piece = [&]( int k, int & a, int & b ) {
			a = step_begin[k - ks];
			int const e = step_begin[k + 1 - ks];
			b = a < e ? piece_end( table, a, e, bufv, wv ) : a;
		};
		if( piped )
		{
			// the first pieces of steps ks and ks + 1 in flight before the loop
			for( int k = ks; k < min( ks + 2, kend ); k++ )
			{
				int a, b;
				first_piece( k, a, b );
				issue_piece( p, table, a, b, ( k & 1 ) ? buf1 : buf0, wv );
			}
			cp_async_commit();
			cp_async_wait_all();
			__syncthreads();
		}

		for( int k = ks; k < kend; k++ )
		{
			long long const t = t0 + k;
			bool const arrivals = t >= p.delay;
			uint4 * const bk = ( k & 1 ) ? buf1 : buf0;
			if( inputs && arrivals )
			{
				if( direct )
				{
					// the direct path of window_counts, its scratch in the (unused) table
					int * pref = reinterpret_cast<int *>( table );
					int4 * sb = reinterpret_cast<int4 *>( reinterpret_cast<unsigned char *>( table ) + ( ( ( p.ntiles + 1 ) * 4 + 15 ) & ~15 ) );
					net_params q = p;
					q.tile = span; // counter rows are span long
					deliver_counts<N>( q, (int)( ( t - p.delay ) % p.ring ), tile, d0, d1, cnt, pref, sb, scratch );
				}
				else
				{
					int const e = step_begin[k + 1 - ks];
					int const sv = step_vec[k + 1 - ks] - step_vec[k - ks];
					// bitmaps: the warp that owns word w counts it for all classes; the
					// counts land in the counter rows the update reads
					auto count_piece = [&]( int a, int b ) {
						if constexpr( Dense )
						{
							if( a >= b ) return;
							int const slot0 = ent_off( table[a] ) / wv;
							int const slot1 = ( b < e ? ent_off( table[b] ) : sv ) / wv;
							unsigned const * bw = reinterpret_cast<unsigned const *>( bk );
							// class 0 = all slots minus the other classes (fewer planes to move).
							// Warp `warp` counts the tile words it updates below (warp + r nw),
							// so no barrier is needed between counting and the update.
							for( int tw = warp; tw < bw0 + bwn; tw += nw )
							{
								if( tw < bw0 ) continue;
								int const w = tw - bw0;
								int const local = ( tw << 5 ) + lane;
								unsigned rest = 0;
								int c0 = s_cslots[k - ks][0];
#pragma unroll
								for( int c = 1; c < C; c++ )
								{
									int const c1 = c0 + s_cslots[k - ks][c];
									int const lo = max( c0, slot0 ), hi = min( c1, slot1 );
									if( lo < hi )
									{
										unsigned const m = bitmap_count( bw, slot0, lo, hi, wv * 4, w, lane );
										if( local < span ) cnt[c * span + local] += m;
										rest += m;
									}
									c0 = c1;
								}
								unsigned const all = bitmap_count( bw, slot0, slot0, slot1, wv * 4, w, lane );
								if( local < span ) cnt[local] += all - rest;
							}
						}
						else
							count_buffer( bk, piece_vectors( table, a, b, e, sv ), cnt );
					};
					int a, b;
					first_piece( k, a, b );
					count_piece( a, b );
					while( b < e ) // the rest of a step larger than a buffer
					{
						__syncthreads(); // bk is free
						a = b;
						b = piece_end( table, a, e, bufv, wv );
						issue_piece( p, table, a, b, bk, wv );
						cp_async_commit();
						cp_async_wait_all();
						__syncthreads();
						count_piece( a, b );
					}
				}
			}
			// counts complete (bitmaps: every warp counted its own words, no barrier needed)
			if( !Dense || !piped ) __syncthreads();
			unsigned * bits = bits2 + ( k & 1 ) * words; // the compaction of step k - 1 reads the other half

			// update: warp w owns neurons [32 w, 32 w + 32) + 32 nw * round; one bit word each
			for( int base = warp * 32; base < span; base += nw * 32 )
			{
				int const local = base + lane;
				bool fired = false;
				if( local < span )
				{
					Tup st;
					smem_state<N>::load( st, state, span, local );
					uint32_t const i = (uint32_t)( d0 + local );
					reg_iter<Tup> it{ st, i };
					if( inputs && arrivals )
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
					fired = N::update( it, s_dt[k], info, bak );
					smem_state<N>::store( st, state, span, local );
				}
				unsigned const word = __ballot_sync( 0xffffffffu, fired );
				if( lane == 0 ) bits[base >> 5] = word;
			}
			if( piped ) cp_async_wait_all(); // this thread's copies for step k + 1
			__syncthreads();                 // fired bits and step k + 1's slices complete
			if( piped && k + 2 < kend )
			{
				// step k + 2 into the buffer step k was counted from (done: barrier above)
				int a, b;
				first_piece( k + 2, a, b );
				issue_piece( p, table, a, b, bk, wv );
				cp_async_commit();
			}
			// ascending compaction by the last warp, without a further barrier: 32 words per
			// round, a warp scan of their counts gives every word's offset. The other warps
			// go on to the next step's counting; bits are rewritten only after the next
			// step's first barrier, and counters were zeroed where they were consumed.
			if( warp == nw - 1 )
			{
				int const slot_out = (int)( t % p.ring );
				int * out = p.ring_ids + (long long)slot_out * p.n + d0;
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
						out[off++] = d0 + ( w << 5 ) + b;
					}
					done += __shfl_sync( 0xffffffffu, incl, 31 );
				}
				if( lane == 0 ) p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)done;
			}
		}
		ks = kend;
		__syncthreads(); // compaction reads of bits are done before the next segment or the exit
	}

	smem_state<N>::to_global( p.attr, d0, span, state );
	window_clock_end( p, L, t0, s_c, s_sum );
}
} // namespace spk
