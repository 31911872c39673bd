// The generic window kernel: non-plastic models without input classes, and models whose
// synapses carry static attributes (a per-synapse weight, say). Every arrival goes through
// the model's own receive( src, dst, syn, info, backend ), per target in the order of the
// reference's CPU simulator (spice/cpu/snn.h.cpp:111-127: the step's spikes in ascending
// id, each row's synapses in ascending position), so a receive() that adds floats gives
// the CPU simulator's sums bit for bit. The reference's GPU form (_gather,
// spice/cuda/algorithm.cu:340-384) applies the same receives with atomics in whatever order
// the threads reach them.
//
// Per step and tile: the step's arrivals (ascending source ids: tiles are ascending id
// ranges and every tile's ring segment is ascending) are staged in batches of ORD_STAGE
// (source, row slice); in chunks of 32, one warp per arrival walks the arrival's row slice
// and records, per (arrival, target), the synapse's position in the row and a bit in the
// target's mask; then every target's thread applies the chunk's arrivals in ascending bit
// order. Rows are strictly ascending, so a target occurs at most once in an arrival's
// slice. The receive() and update() of one neuron run in the thread that owns it, so a
// Backend's atomic_add is a plain add.
#pragma once

#include "kernels.cuh"

namespace spk
{
constexpr int ORD_CHUNK = 32;
constexpr int ORD_STAGE = 256;     // staged arrivals per batch
constexpr int ORD_MAX_TILE = 1024; // neurons per tile (2 per thread at most)
constexpr int ORD_AHEAD = 8;       // arrivals per warp of a chunk with their rows loaded ahead (4 warps cover a chunk)

// attribute I of the synapse at edge position e (the reference's synapse id src * width + j,
// spice/util/adj_list.cpp:40-46), in the net's structure-of-arrays synapse attributes
template <typename Syn, bool Writable>
struct syn_ref_iter
{
	void * const * a;
	long long e;
	template <int I>
	__device__ __forceinline__ auto & get() const
	{
		using T = typename Syn::template type<I>;
		if constexpr( Writable )
			return static_cast<T *>( a[I] )[e];
		else
			return static_cast<T const *>( a[I] )[e];
	}
};

// dynamic shared memory of a window_ordered launch: positions [ORD_CHUNK][tile], masks
// [tile], the source tiles' prefix [ntiles + 1], staged arrivals [ORD_STAGE]
__host__ __device__ inline size_t ordered_window_smem( int tile, int ntiles )
{
	size_t b = ( (size_t)ORD_CHUNK * tile + tile + ntiles + 1 ) * 4;
	return ( ( b + 15 ) & ~(size_t)15 ) + (size_t)ORD_STAGE * 16;
}

template <typename Model, int NPT>
__global__ void __launch_bounds__( 512, 1 ) window_ordered( net_params p, int L, float dt )
{
	using N = typename Model::neuron;
	using S = typename Model::synapse;
	using Tup = typename N::template apply<reg_tuple>;
	static_assert( !S::has_stdp, "window_ordered runs models without plasticity" );

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	__shared__ int s_src[ORD_CHUNK];

	int const T = p.tile, tid = threadIdx.x;
	int const warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
	int const tile = blockIdx.x, d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	snn_info const info{ p.n };
	int * pos = reinterpret_cast<int *>( smem );                            // [ORD_CHUNK][T]
	unsigned * mask = reinterpret_cast<unsigned *>( pos + ORD_CHUNK * T ); // [T]
	int * pref = reinterpret_cast<int *>( mask + T );                     // [ntiles + 1]
	int4 * sb = reinterpret_cast<int4 *>( smem + ( ( ( (size_t)ORD_CHUNK * T + T + p.ntiles + 1 ) * 4 + 15 ) & ~(size_t)15 ) );

	window_clock_begin( p, L, dt, s_dt, &s_t0, &s_c, &s_sum );

	Tup st[NPT];
	long long const i0 = (long long)d0 + NPT * tid;
#pragma unroll
	for( int q = 0; q < NPT; q++ )
		if( i0 + q < d1 ) attrs_io<N>::load( st[q], p.attr, i0 + q );
	for( int x = tid; x < T; x += blockDim.x ) mask[x] = 0u;
	__syncthreads();

	for( int k = 0; k < L; k++ )
	{
		long long const t = s_t0 + k;
		if( t >= p.delay )
		{
			int const slot_in = (int)( ( t - p.delay ) % p.ring );
			int const total = stage_prefix( p, p.ring_cnt, slot_in, pref, scratch );
			for( int b0 = 0; b0 < total; b0 += ORD_STAGE )
			{
				int const m = min( ORD_STAGE, total - b0 );
				for( int x = tid; x < m; x += blockDim.x )
				{
					int const g = b0 + x;
					int const si = find_tile( pref, p.ntiles, g );
					int const src = p.ring_ids[(long long)slot_in * p.n + __ldg( p.tile_first + si ) + ( g - pref[si] )];
					unsigned const * pv = p.pivots + (long long)src * ( p.ntiles + 1 ) + tile;
					sb[x] = make_int4( src, (int)__ldg( pv ), (int)__ldg( pv + 1 ), 0 );
				}
				__syncthreads();
				for( int c0 = 0; c0 < m; c0 += ORD_CHUNK )
				{
					int const mc = min( ORD_CHUNK, m - c0 );
					if( tid < mc ) s_src[tid] = sb[c0 + tid].x;
					// the warp's arrivals of the chunk (x = warp, warp + nw, ...): the first two
					// targets per lane of each row slice loaded before any is recorded, so the
					// rows' loads overlap; the rest of a longer slice is loaded as it is walked
					int pd[ORD_AHEAD][2];
#pragma unroll
					for( int u = 0; u < ORD_AHEAD; u++ )
					{
						int const x = warp + u * nw;
						pd[u][0] = pd[u][1] = -1;
						if( x < mc )
						{
							int4 const e = sb[c0 + x];
#pragma unroll
							for( int h = 0; h < 2; h++ )
							{
								int const j = e.y + lane + 32 * h;
								if( j < e.z ) pd[u][h] = __ldg( p.edges + (long long)e.x * p.width + j );
							}
						}
					}
					auto record = [&]( int x, bool ahead, int d1st, int d2nd ) {
						int4 const e = sb[c0 + x];
						int const * row = p.edges + (long long)e.x * p.width;
						for( int j = e.y + lane; j < e.z; j += 32 )
						{
							int const it = ( j - e.y - lane ) >> 5;
							int const d = ahead && it < 2 ? ( it == 0 ? d1st : d2nd ) : __ldg( row + j );
							int const local = d - d0;
							if( (unsigned)local >= (unsigned)span )
							{
								atomicOr( p.err, ERR_BAD_TARGET );
								continue;
							}
							pos[x * T + local] = j;
							atomicOr( mask + local, 1u << x );
						}
					};
#pragma unroll
					for( int u = 0; u < ORD_AHEAD; u++ )
						if( warp + u * nw < mc ) record( warp + u * nw, true, pd[u][0], pd[u][1] );
					for( int x = warp + ORD_AHEAD * nw; x < mc; x += nw ) record( x, false, 0, 0 ); // CTAs of < 4 warps
					__syncthreads();
					// every target applies its arrivals of the chunk in ascending source order
#pragma unroll
					for( int q = 0; q < NPT; q++ )
					{
						int const local = NPT * tid + q;
						if( i0 + q >= d1 ) continue;
						unsigned mm = mask[local];
						if( !mm ) continue;
						mask[local] = 0u;
						reg_iter<Tup> it{ st[q], (uint32_t)( i0 + q ) };
						device_backend bak( p.seed, (uint32_t)( i0 + q ), (uint32_t)t );
						// four arrivals at a time, in ascending source order: their synapses'
						// attribute loads (inside receive) are independent of each other
						while( mm )
						{
							constexpr int RX = 4;
							int bs[RX];
							int nb = 0;
#pragma unroll
							for( int u = 0; u < RX; u++ )
								if( mm )
								{
									bs[u] = __ffs( mm ) - 1;
									mm &= mm - 1;
									nb = u + 1;
								}
#pragma unroll
							for( int u = 0; u < RX; u++ )
								if( u < nb )
								{
									int const src = s_src[bs[u]];
									N::receive( src, it, syn_ref_iter<S, false>{ p.syn_attr, (long long)src * p.width + pos[bs[u] * T + local] }, info, bak );
								}
						}
					}
					__syncthreads();
				}
			}
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
				if( N::update( it, s_dt[k], info, bak ) ) fired |= 1u << q;
			}
		}
		// the step's spikes, ascending, into the tile's ring segment
		int total;
		int off = block_exclusive_scan( __popc( fired ), scratch, &total );
		int const slot_out = (int)( t % p.ring );
		int * out = p.ring_ids + (long long)slot_out * p.n + d0;
#pragma unroll
		for( int q = 0; q < NPT; q++ )
			if( ( fired >> q ) & 1u ) out[off++] = (int)( i0 + q );
		if( tid == 0 ) p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)total;
	}

#pragma unroll
	for( int q = 0; q < NPT; q++ )
		if( i0 + q < d1 ) attrs_io<N>::store( st[q], p.attr, i0 + q );
	window_clock_end( p, L, s_t0, s_c, s_sum );
}

// Synapse::init for every synapse (non-pad edge slot) of the net: the reference's
// _process_spikes<INIT_SYNS> (spice/cuda/algorithm.cu:238-313) and its CPU twin
// (spice/cpu/snn.h.cpp:90-103). The attribute arrays are zero where an edge slot is padding,
// as the reference's value-initialised synapse vector. A rand() in Synapse::init draws
// from the counter stream keyed (seed ^ SYN_INIT_KEY, source, position in the row).
constexpr unsigned long long SYN_INIT_KEY = 0x53594e494e495431ull;
template <typename Model>
__global__ void __launch_bounds__( 256 ) init_synapses( net_params p )
{
	using S = typename Model::synapse;
	snn_info const info{ p.n };
	long long const total = (long long)p.n * p.width;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x )
	{
		int const dst = p.edges[e];
		if( dst == INT_MAX ) continue;
		int const src = (int)( e / p.width ), j = (int)( e % p.width );
		device_backend bak( p.seed ^ SYN_INIT_KEY, (uint32_t)src, (uint32_t)j );
		S::init( syn_ref_iter<S, true>{ p.syn_attr, e }, src, dst, info, bak );
	}
}
} // namespace spk
