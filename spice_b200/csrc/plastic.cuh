// Lazy event-driven pair STDP (models whose synapse declares has_stdp), B200 form of the
// reference's spike-triggered replay (spice/cuda/algorithm.cu:238-313) with the results of
// its CPU sweep (spice/cpu/snn.h.cpp:161-179).
//
// Reference semantics, per step t and plastic synapse (s, d):
//   Zpre  <- fma(Zpre,  c_t, x_s(t - delay))      (the source's delayed spike: "pre")
//   Zpost <- fma(Zpost, c_t, x_d(t))              ("post")
//   W     <- F_t(W, pre, post, Zpre, Zpost)       (after the step's receive and update)
// Zpre / Zpost are per-neuron traces (see brunel_with_plasticity.h): they are updated for
// every neuron every step, exactly. W is touched only when F_t is not the identity:
//   * a pre event at step t (the row of s arrives at t) changes W only if d is
//     "post-active" (exp(-Zpost_d(t)/dt) != 0) or d fires at t while s is "pre-active";
//     the tile holding d applies it at t + 1 ("completion"), once x_d(t), Zpost_d(t) exist;
//   * a post event of d at step tau changes W only while s is pre-active at tau
//     (exp(-Zpre_s(tau)/dt) != 0, i.e. s has been silent for a long time). Those are
//     replayed lazily from d's 64-step spike history when the row of s is next touched:
//     at its next arrival, or at a forced "flush" touch that the owner of s schedules at
//     most 63 steps after the first pre-active step of the pending window.
// Every touch of row s is announced by the tile that owns neuron s, `delay` steps ahead,
// through the spike ring (arrivals) or the flush ring, with the trace values the touching
// tiles need (so no tile reads state another tile writes during the same launch).
//
// The input sum of a plastic model depends on the per-synapse weights, so it is reduced in
// the reference's order: arrivals are processed in chunks of 32 in ascending source order,
// each chunk records its weights per (arrival, target) and a per-target bit mask in
// shared memory, and every target then adds its inputs in ascending source order.
#pragma once

#include "kernels.cuh"

#include <algorithm>
#include <vector>

namespace spk
{
constexpr int PL_CHUNK = 32;
constexpr int PL_MAX_TILE = 1024;
// window_plastic comes in two register budgets: one CTA of up to 512 threads per SM (118
// registers a thread), and two CTAs of up to PL_THREADS threads per SM (at most 85
// registers; the kernel then needs 76, with no spills), for nets whose tiles do not fit one
// per SM. The two-per-SM form runs single small nets about 6 % slower, so it is used only
// where it saves a wave of CTAs.
constexpr int PL_THREADS = 384;
constexpr int PL_CTAS_PER_SM = 2;
constexpr int PL_STAGE = 256;     // staged arrivals per batch
constexpr int PL_FLUSH_AT = 63;   // longest replay window (bits of the spike history)
constexpr int PL_MAX_DELAY = 63;

struct plastic_params
{
	float * W;                 // [n x width] weights, parallel to edges
	float * za;                // Zpre_s(now - 1 + delay): the owner's look-ahead trace
	float * zpre;              // Zpre_s(now - 1)
	float * zpost;             // Zpost_d(now - 1)
	unsigned long long * hist; // bit j: fired at step now - 1 - j
	int * rf_a;                // look-ahead row state: first pre-active step of the pending window (-1: none)
	float * zrf_a;             //   Zpre at rf_a - 1
	int * rf_c;                // the same row state as of now (for export)
	float * zrf_c;
	int4 * ring_meta;          // per spike, parallel to ring_ids: {rf_off | pot << 8, zrf bits, zpre_t bits, 0}
	int4 * flush_ring;         // [2 delay x n]: {src, rf_off, zrf bits, 0}, one segment per tile
	unsigned * flush_cnt;      // [2 delay x ntiles]
	unsigned * ring_pot;       // [2 delay x ntiles]: some arrival entry of the tile segment has pot set
};

struct stage_e
{
	int src, lo, hi, meta;
	float zrf, zt;
};

// The row-state machine: called for every touch step tp of a plastic source with
// arrive = x_s(tp - delay), z_prev = Zpre_s(tp - 1), z_new = Zpre_s(tp), pa = s is
// pre-active at tp. Returns 1 for an arrival entry, 2 for a flush entry, 0 for none;
// rf_off / zrf describe the entry's replay window [tp - rf_off, tp - 1].
__device__ __forceinline__ int row_step( int & rf, float & zrf, bool arrive, float z_prev, bool pa, long long tp, int & rf_off, float & zrf_out )
{
	if( arrive )
	{
		rf_off = rf >= 0 ? (int)( tp - rf ) : 0;
		zrf_out = zrf;
		rf = -1;
		return 1;
	}
	if( rf >= 0 && tp - rf >= PL_FLUSH_AT )
	{
		rf_off = (int)( tp - rf );
		zrf_out = zrf;
		if( pa )
		{
			rf = (int)tp;
			zrf = z_prev;
		}
		else
			rf = -1;
		return 2;
	}
	if( rf < 0 && pa )
	{
		rf = (int)tp;
		zrf = z_prev;
	}
	rf_off = 0;
	return 0;
}

__device__ __forceinline__ float dt_at( long long tau, long long t0, float const * s_dt, float const * dt_ring )
{
	return tau >= t0 ? s_dt[tau - t0] : dt_ring[tau % DT_RING];
}

// Replays the post events of one synapse over [tp - rf_off, tp - 1]: hb holds d's firing
// bits (bit j = step tp - 1 - j), zwin[i] = Zpre_s(tp - rf_off + i).
template <typename Syn, typename Backend>
__device__ __forceinline__ float replay_post(
    float w, unsigned long long hb, int rf_off, long long tp, float const * zwin, long long t0, float const * s_dt, float const * dt_ring, Backend & bak )
{
	while( hb )
	{
		int const j = 63 - __clzll( (long long)hb ); // oldest event first
		hb &= ~( 1ull << j );
		long long const tau = tp - 1 - j;
		w = Syn::update( w, false, true, zwin[tau - ( tp - rf_off )], 1.0f, dt_at( tau, t0, s_dt, dt_ring ), bak );
	}
	return w;
}

// entries [b0, b0 + m) of the spike slot -> sb (src, slice bounds, meta)
__device__ __forceinline__ void stage_spikes( net_params const & p, plastic_params const & q, int slot, int tile, int const * pref, int b0, int m, stage_e * sb )
{
	for( int x = threadIdx.x; x < m; x += blockDim.x )
	{
		int const g = b0 + x;
		int const st = find_tile( pref, p.ntiles, g );
		long long const pos = (long long)slot * p.n + __ldg( p.tile_first + st ) + ( g - pref[st] );
		int const src = p.ring_ids[pos];
		int4 const meta = q.ring_meta[pos];
		unsigned const * pv = p.pivots + (long long)src * ( p.ntiles + 1 ) + tile;
		sb[x] = { src, (int)__ldg( pv ), (int)__ldg( pv + 1 ), meta.x, __int_as_float( meta.y ), __int_as_float( meta.z ) };
	}
}

__device__ __forceinline__ void stage_flushes( net_params const & p, plastic_params const & q, int slot, int tile, int const * pref, int b0, int m, stage_e * sb )
{
	for( int x = threadIdx.x; x < m; x += blockDim.x )
	{
		int const g = b0 + x;
		int const st = find_tile( pref, p.ntiles, g );
		int4 const f = q.flush_ring[(long long)slot * p.n + __ldg( p.tile_first + st ) + ( g - pref[st] )];
		unsigned const * pv = p.pivots + (long long)f.x * ( p.ntiles + 1 ) + tile;
		sb[x] = { f.x, (int)__ldg( pv ), (int)__ldg( pv + 1 ), f.y, __int_as_float( f.z ), 0.0f };
	}
}

// Zpre_s over a replay window: zwin[i] = Zpre_s(tp - rf_off + i), no arrivals inside.
template <typename Syn>
__device__ __forceinline__ void window_trace( float zrf, int rf_off, long long tp, long long t0, float const * s_dt, float const * dt_ring, float * zwin )
{
	float z = zrf;
	for( int i = 0; i < rf_off; i++ )
	{
		long long const tau = tp - rf_off + i;
		z = fmaf( z, Syn::trace_decay( dt_at( tau, t0, s_dt, dt_ring ) ), 0.0f );
		zwin[i] = z;
	}
}

// The window step of tile `tile` of a plastic net (L steps of dt): the body of
// window_plastic and window_plastic_batch. Tiles of up to blockDim.x * NPT neurons.
template <typename Model, int NPT>
__device__ __forceinline__ void window_plastic_body( net_params const & p, plastic_params const & q, int const tile, int L, float dt )
{
	using N = typename Model::neuron;
	using Syn = typename Model::synapse;
	using Tup = typename N::template apply<reg_tuple>;

	extern __shared__ __align__( 128 ) unsigned char smem[];
	__shared__ int scratch[33];
	__shared__ float s_dt[2 * MAX_WINDOW];
	__shared__ long long s_t0;
	__shared__ float s_c, s_sum;
	__shared__ int s_flags; // bit 0: some plastic target post-active at t-1; bit 1: some target fired at t-1
	__shared__ int s_src[PL_CHUNK];

	int const T = p.tile, tid = threadIdx.x;
	int const warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
	int const d0 = __ldg( p.tile_first + tile ), d1 = __ldg( p.tile_first + tile + 1 ), span = d1 - d0;
	snn_info const info{ p.n };

	// shared memory carve-up (sizes: see plastic_window_smem)
	float * wT = reinterpret_cast<float *>( smem );                                   // [PL_CHUNK][T]
	unsigned * mask = reinterpret_cast<unsigned *>( wT + PL_CHUNK * T );             // [T]
	unsigned long long * sh_hist = reinterpret_cast<unsigned long long *>( mask + T ); // [T] (8-aligned: T % 2 == 0)
	float * sh_zpost = reinterpret_cast<float *>( sh_hist + T );                     // [T]
	unsigned char * sh_dpa = reinterpret_cast<unsigned char *>( sh_zpost + T );      // [T]
	int * pref = reinterpret_cast<int *>( sh_dpa + ( ( T + 15 ) & ~15 ) );            // [ntiles + 1]
	stage_e * sb = reinterpret_cast<stage_e *>( pref + ( ( p.ntiles + 1 + 3 ) & ~3 ) ); // [PL_STAGE]
	float * zwin = reinterpret_cast<float *>( sb + PL_STAGE );                        // [nwarps][64]

	// clock: the window's dt plus `delay` steps of look-ahead for the owners' traces
	if( tid == 0 )
	{
		clock_state const cs = *p.clock;
		float c = cs.c, sum = cs.sum;
		for( int k = 0; k < L; k++ ) s_dt[k] = kahan_add( c, sum, dt );
		s_c = c;
		s_sum = sum;
		float c2 = c, sum2 = sum;
		for( int k = L; k < L + p.delay; k++ ) s_dt[k] = kahan_add( c2, sum2, dt );
		s_t0 = cs.step;
		if( tile == 0 )
			for( int k = 0; k < L; k++ ) p.dt_ring[( cs.step + k ) % DT_RING] = s_dt[k];
	}
	__syncthreads();
	long long const t0 = s_t0;

	// per-neuron state into registers / shared memory
	Tup st[NPT];
	float za[NPT], zpre[NPT];
	int rfa[NPT], rfc[NPT];
	float zrfa[NPT], zrfc[NPT];
	long long const i0 = (long long)d0 + NPT * tid;
	int any_pa = 0, any_fired = 0;
#pragma unroll
	for( int k = 0; k < NPT; k++ )
	{
		long long const i = i0 + k;
		int const local = NPT * tid + k;
		if( i < d1 )
		{
			attrs_io<N>::load( st[k], p.attr, i );
			za[k] = q.za[i];
			zpre[k] = q.zpre[i];
			rfa[k] = q.rf_a[i];
			zrfa[k] = q.zrf_a[i];
			rfc[k] = q.rf_c[i];
			zrfc[k] = q.zrf_c[i];
			unsigned long long const h = q.hist[i];
			float const zp = q.zpost[i];
			sh_hist[local] = h;
			sh_zpost[local] = zp;
			device_backend bak( p.seed, (uint32_t)i, 0u );
			bool const dpa = t0 >= 1 && Syn::plastic_dst( (int)i, info ) &&
			                 Syn::depression_active( zp, p.dt_ring[( t0 - 1 + DT_RING ) % DT_RING], bak );
			sh_dpa[local] = dpa;
			any_pa |= dpa;
			any_fired |= (int)( h & 1ull );
		}
		else if( local < T )
		{
			sh_hist[local] = 0;
			sh_zpost[local] = 0;
			sh_dpa[local] = 0;
		}
	}
	for( int x = tid; x < T; x += blockDim.x ) mask[x] = 0;
	if( tid == 0 ) s_flags = 0;
	__syncthreads();
	if( any_pa ) atomicOr( &s_flags, 1 );
	if( any_fired ) atomicOr( &s_flags, 2 );
	__syncthreads();

	for( int k = 0; k < L; k++ )
	{
		long long const t = t0 + k;
		float const dt_t = s_dt[k];

		// ---- completion of the pre events of step t-1 (rows that arrived at t-1) ----
		if( t - 1 >= p.delay )
		{
			int const slot_c = (int)( ( t - 1 - p.delay ) % p.ring );
			bool pot_any = false;
			if( s_flags & 2 )
				for( int i = lane; i < p.ntiles; i += 32 ) pot_any |= q.ring_pot[(long long)slot_c * p.ntiles + i] != 0;
			pot_any = __any_sync( 0xffffffffu, pot_any );
			bool const need = ( s_flags & 1 ) || ( ( s_flags & 2 ) && pot_any );
			// `need` may differ between warps only through pot_any, which every warp computed
			// from the same data: uniform.
			if( need )
			{
				float const dt_c = dt_at( t - 1, t0, s_dt, p.dt_ring );
				int const total = stage_prefix( p, p.ring_cnt, slot_c, pref, scratch );
				for( int b0 = 0; b0 < total; b0 += PL_STAGE )
				{
					int const m = min( PL_STAGE, total - b0 );
					stage_spikes( p, q, slot_c, tile, pref, b0, m, sb );
					__syncthreads();
					for( int x = warp; x < m; x += nw )
					{
						stage_e const e = sb[x];
						if( !Syn::plastic_src( e.src, info ) ) continue;
						bool const pot = ( e.meta >> 8 ) & 1;
						int const * row = p.edges + (long long)e.src * p.width;
						float * wrow = q.W + (long long)e.src * p.width;
						device_backend bak( p.seed, (uint32_t)e.src, (uint32_t)t );
						for( int j = e.lo + lane; j < e.hi; j += 32 )
						{
							int const d = __ldg( row + j );
							int const local = d - d0;
							if( (unsigned)local >= (unsigned)span || !Syn::plastic_dst( d, info ) ) continue;
							bool const x_d = sh_hist[local] & 1ull;
							if( !sh_dpa[local] && !( x_d && pot ) ) continue;
							float const w = wrow[j];
							float const w2 = Syn::update( w, true, x_d, e.zt, sh_zpost[local], dt_c, bak );
							if( __float_as_int( w2 ) != __float_as_int( w ) ) wrow[j] = w2;
						}
					}
					__syncthreads();
				}
			}
		}

		// ---- flush touches of step t: replay post events of pre-active rows ----
		if( t >= p.delay )
		{
			int const slot_in = (int)( ( t - p.delay ) % p.ring );
			int const total = stage_prefix( p, q.flush_cnt, slot_in, pref, scratch );
			for( int b0 = 0; b0 < total; b0 += PL_STAGE )
			{
				int const m = min( PL_STAGE, total - b0 );
				stage_flushes( p, q, slot_in, tile, pref, b0, m, sb );
				__syncthreads();
				for( int x = warp; x < m; x += nw )
				{
					stage_e const e = sb[x];
					int const rf_off = e.meta & 0xff;
					float * zw = zwin + warp * 64;
					if( lane == 0 ) window_trace<Syn>( e.zrf, rf_off, t, t0, s_dt, p.dt_ring, zw );
					__syncwarp();
					int const * row = p.edges + (long long)e.src * p.width;
					float * wrow = q.W + (long long)e.src * p.width;
					device_backend bak( p.seed, (uint32_t)e.src, (uint32_t)t );
					unsigned long long const wm = rf_off >= 64 ? ~0ull : ( ( 1ull << rf_off ) - 1 );
					for( int j = e.lo + lane; j < e.hi; j += 32 )
					{
						int const d = __ldg( row + j );
						int const local = d - d0;
						if( (unsigned)local >= (unsigned)span || !Syn::plastic_dst( d, info ) ) continue;
						unsigned long long const hb = sh_hist[local] & wm;
						if( !hb ) continue;
						float const w = wrow[j];
						float const w2 = replay_post<Syn>( w, hb, rf_off, t, zw, t0, s_dt, p.dt_ring, bak );
						if( __float_as_int( w2 ) != __float_as_int( w ) ) wrow[j] = w2;
					}
					__syncwarp();
				}
				__syncthreads();
			}
		}

		// ---- arrivals of step t: replay pending post events, then ordered receive ----
		bool const arrivals = t >= p.delay;
		if( arrivals )
		{
			int const slot_in = (int)( ( t - p.delay ) % p.ring );
			int const total = stage_prefix( p, p.ring_cnt, slot_in, pref, scratch );
			for( int b0 = 0; b0 < total; b0 += PL_STAGE )
			{
				int const m = min( PL_STAGE, total - b0 );
				stage_spikes( p, q, slot_in, tile, pref, b0, m, sb );
				__syncthreads();
				// chunks of `chunk` arrivals, PL_AH per warp, each with its row slice's first two
				// elements per lane loaded ahead: a chunk's loads are issued while the chunk
				// before it is walked and received, so their latency overlaps that work (a
				// chunk's rows are other sources than the chunk before it: no weight it loads is
				// one that chunk writes)
				constexpr int PL_AH = 4;
				int const chunk = min( PL_CHUNK, PL_AH * nw );
				int pdA[PL_AH][2], pdB[PL_AH][2];
				float pwA[PL_AH][2], pwB[PL_AH][2];
				auto preload = [&]( int cc0, int( &pd )[PL_AH][2], float( &pw )[PL_AH][2] ) {
					int const cmc = min( chunk, m - cc0 );
#pragma unroll
					for( int u = 0; u < PL_AH; u++ )
					{
						int const x = warp + u * nw;
#pragma unroll
						for( int h = 0; h < 2; h++ )
						{
							pd[u][h] = -1;
							pw[u][h] = 0.0f;
						}
						if( x < cmc )
						{
							stage_e const e = sb[cc0 + x];
#pragma unroll
							for( int h = 0; h < 2; h++ )
							{
								int const j = e.lo + lane + 32 * h;
								if( j < e.hi )
								{
									pd[u][h] = __ldg( p.edges + (long long)e.src * p.width + j );
									pw[u][h] = q.W[(long long)e.src * p.width + j];
								}
							}
						}
					}
				};
				preload( 0, pdA, pwA );
				for( int c0 = 0; c0 < m; c0 += chunk )
				{
					int const mc = min( chunk, m - c0 );
					if( tid < mc ) s_src[tid] = sb[c0 + tid].src;
					if( c0 + chunk < m ) preload( c0 + chunk, pdB, pwB );
					// spike x of the chunk into its weight column; (d1st, w1st) = its first slice
					// element if loaded ahead (ahead1st)
					auto arrive = [&]( int x, bool ahead1st, int d1st, float w1st, int d2nd, float w2nd ) {
						stage_e const e = sb[c0 + x];
						int const rf_off = e.meta & 0xff;
						bool const replay = rf_off > 0 && Syn::plastic_src( e.src, info );
						float * zw = zwin + warp * 64;
						if( replay )
						{
							if( lane == 0 ) window_trace<Syn>( e.zrf, rf_off, t, t0, s_dt, p.dt_ring, zw );
							__syncwarp();
						}
						int const * row = p.edges + (long long)e.src * p.width;
						float * wrow = q.W + (long long)e.src * p.width;
						float * wcol = wT + x * T;
						unsigned const bit = 1u << x;
						device_backend bak( p.seed, (uint32_t)e.src, (uint32_t)t );
						unsigned long long const wm = rf_off >= 64 ? ~0ull : ( ( 1ull << rf_off ) - 1 );
						for( int j = e.lo + lane; j < e.hi; j += 32 )
						{
							int const it = ( j - e.lo - lane ) >> 5; // 0: first element of this lane, 1: second
							bool const ahead = ahead1st && it < 2;
							int const d = ahead ? ( it == 0 ? d1st : d2nd ) : __ldg( row + j );
							int const local = d - d0;
							if( (unsigned)local >= (unsigned)span )
							{
								atomicOr( p.err, ERR_BAD_TARGET );
								continue;
							}
							float w = ahead ? ( it == 0 ? w1st : w2nd ) : wrow[j];
							if( replay && Syn::plastic_dst( d, info ) )
							{
								unsigned long long const hb = sh_hist[local] & wm;
								if( hb )
								{
									float const w2 = replay_post<Syn>( w, hb, rf_off, t, zw, t0, s_dt, p.dt_ring, bak );
									if( __float_as_int( w2 ) != __float_as_int( w ) ) wrow[j] = w2;
									w = w2;
								}
							}
							wcol[local] = w;
							atomicOr( mask + local, bit );
						}
						if( replay ) __syncwarp();
					};
#pragma unroll
					for( int u = 0; u < PL_AH; u++ ) // every arrival of the chunk (chunk <= PL_AH * nw)
						if( warp + u * nw < mc ) arrive( warp + u * nw, true, pdA[u][0], pwA[u][0], pdA[u][1], pwA[u][1] );
					__syncthreads();
					// every target adds its inputs in ascending source order
#pragma unroll
					for( int kk = 0; kk < NPT; kk++ )
					{
						int const local = NPT * tid + kk;
						if( i0 + kk < d1 )
						{
							unsigned mm = mask[local];
							if( mm )
							{
								reg_iter<Tup> it{ st[kk], (uint32_t)( i0 + kk ) };
								device_backend bak( p.seed, (uint32_t)( i0 + kk ), (uint32_t)t );
								// four arrivals at a time: their weights loaded together, then the
								// receives in ascending source order (the loads and the parts of
								// receive that do not touch the neuron's state overlap)
								while( mm )
								{
									constexpr int RX = 4;
									int bs[RX];
									float ws[RX];
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
										if( u < nb ) ws[u] = wT[bs[u] * T + local];
#pragma unroll
									for( int u = 0; u < RX; u++ )
										if( u < nb ) N::receive( s_src[bs[u]], it, weight_iter{ ws[u] }, info, bak );
								}
								mask[local] = 0;
							}
						}
					}
					__syncthreads();
#pragma unroll
					for( int u = 0; u < PL_AH; u++ )
#pragma unroll
						for( int h = 0; h < 2; h++ )
						{
							pdA[u][h] = pdB[u][h];
							pwA[u][h] = pwB[u][h];
						}
				}
			}
		}

		// ---- neuron update, traces, row-state machines, entries ----
		unsigned fired = 0, flushed = 0;
		int4 meta[NPT];
		int4 fl[NPT];
		bool pot_tile = false;
		int apa = 0, afi = 0;
		float const c_t = Syn::trace_decay( dt_t );
		long long const ta = t + p.delay; // look-ahead touch step
		float const dt_a = s_dt[k + p.delay];
		float const c_a = Syn::trace_decay( dt_a );
#pragma unroll
		for( int kk = 0; kk < NPT; kk++ )
		{
			long long const i = i0 + kk;
			int const local = NPT * tid + kk;
			meta[kk] = make_int4( 0, 0, 0, 0 );
			fl[kk] = make_int4( 0, 0, 0, 0 );
			if( i < d1 )
			{
				reg_iter<Tup> it{ st[kk], (uint32_t)i };
				device_backend bak( p.seed, (uint32_t)i, (uint32_t)t );
				bool const x = N::update( it, dt_t, info, bak );
				unsigned long long const h = ( sh_hist[local] << 1 ) | ( x ? 1ull : 0ull );
				float const zp = fmaf( sh_zpost[local], c_t, x ? 1.0f : 0.0f );
				bool const dpa = Syn::plastic_dst( (int)i, info ) && Syn::depression_active( zp, dt_t, bak );
				sh_hist[local] = h;
				sh_zpost[local] = zp;
				sh_dpa[local] = dpa;
				apa |= dpa;
				afi |= x;
				if( x ) fired |= 1u << kk;

				if( Syn::plastic_src( (int)i, info ) )
				{
					// row state as of now (t): arrivals are this neuron's spikes of t - delay
					bool const arr = ( h >> p.delay ) & 1ull;
					float const zn = fmaf( zpre[kk], c_t, arr ? 1.0f : 0.0f );
					int off_c;
					float zr_c;
					row_step( rfc[kk], zrfc[kk], arr, zpre[kk], Syn::potentiation_active( zn, dt_t, bak ), t, off_c, zr_c );
					zpre[kk] = zn;
					// look-ahead row state (touch step t + delay): decides the entries
					float const zan = fmaf( za[kk], c_a, x ? 1.0f : 0.0f );
					bool const pa = Syn::potentiation_active( zan, dt_a, bak );
					int off;
					float zr;
					int const kind = row_step( rfa[kk], zrfa[kk], x, za[kk], pa, ta, off, zr );
					za[kk] = zan;
					if( kind == 1 )
					{
						meta[kk] = make_int4( off | ( pa ? 0x100 : 0 ), __float_as_int( zr ), __float_as_int( zan ), 0 );
						pot_tile |= pa;
					}
					else if( kind == 2 )
					{
						fl[kk] = make_int4( (int)i, off, __float_as_int( zr ), 0 );
						flushed |= 1u << kk;
					}
				}
				else
				{
					bool const arr = ( h >> p.delay ) & 1ull;
					zpre[kk] = fmaf( zpre[kk], c_t, arr ? 1.0f : 0.0f );
					za[kk] = fmaf( za[kk], c_a, x ? 1.0f : 0.0f );
				}
			}
		}
		if( tid == 0 ) s_flags = 0;
		int total;
		int off = block_exclusive_scan( __popc( fired ), scratch, &total ); // syncs: s_flags reset visible
		if( apa ) atomicOr( &s_flags, 1 );
		if( afi ) atomicOr( &s_flags, 2 );
		int const slot_out = (int)( t % p.ring );
		long long const seg = (long long)slot_out * p.n + d0;
#pragma unroll
		for( int kk = 0; kk < NPT; kk++ )
			if( ( fired >> kk ) & 1u )
			{
				p.ring_ids[seg + off] = (int)( i0 + kk );
				q.ring_meta[seg + off] = meta[kk];
				off++;
			}
		int ftotal;
		int foff = block_exclusive_scan( __popc( flushed ), scratch, &ftotal );
#pragma unroll
		for( int kk = 0; kk < NPT; kk++ )
			if( ( flushed >> kk ) & 1u ) q.flush_ring[seg + foff++] = fl[kk];
		int const pot_sum = __syncthreads_or( pot_tile );
		if( tid == 0 )
		{
			p.ring_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)total;
			q.flush_cnt[(long long)slot_out * p.ntiles + tile] = (unsigned)ftotal;
			q.ring_pot[(long long)slot_out * p.ntiles + tile] = pot_sum ? 1u : 0u;
		}
		__syncthreads();
	}

	// write back
#pragma unroll
	for( int k = 0; k < NPT; k++ )
	{
		long long const i = i0 + k;
		int const local = NPT * tid + k;
		if( i < d1 )
		{
			attrs_io<N>::store( st[k], p.attr, i );
			q.za[i] = za[k];
			q.zpre[i] = zpre[k];
			q.rf_a[i] = rfa[k];
			q.zrf_a[i] = zrfa[k];
			q.rf_c[i] = rfc[k];
			q.zrf_c[i] = zrfc[k];
			q.hist[i] = sh_hist[local];
			q.zpost[i] = sh_zpost[local];
		}
	}
	window_clock_end( p, L, t0, s_c, s_sum );
}

template <typename Model, int NPT, int CTAS>
__global__ void __launch_bounds__( CTAS == 1 ? 512 : PL_THREADS, CTAS ) window_plastic( net_params p, plastic_params q, int L, float dt )
{
	window_plastic_body<Model, NPT>( p, q, blockIdx.x, L, dt );
}

// Many plastic nets of one model in one launch (batching): CTA b runs tile jobs[b].y of net
// jobs[b].x (parameters nets[], pls[]) for jobs[b].z steps of dt __int_as_float(jobs[b].w),
// one neuron per thread. The launch has as many threads as its widest tile (at most
// PL_THREADS for the two-CTAs-per-SM form); a narrower tile leaves the rest of its threads
// idle. Every net's steps read only spikes of earlier launches (jobs[b].z <= its delay).
template <typename Model, int CTAS>
__global__ void __launch_bounds__( CTAS == 1 ? 512 : PL_THREADS, CTAS )
    window_plastic_batch( net_params const * nets, plastic_params const * pls, int4 const * jobs )
{
	__shared__ net_params s_p;
	__shared__ plastic_params s_q;
	int4 const j = jobs[blockIdx.x];
	if( threadIdx.x == 0 )
	{
		s_p = nets[j.x];
		s_q = pls[j.x];
	}
	__syncthreads();
	if( j.z > 0 ) window_plastic_body<Model, 1>( s_p, s_q, j.y, j.z, __int_as_float( j.w ) );
}

// synapse::init for every edge (pads 0), per-neuron traces at their initial value.
template <typename Model>
__global__ void init_plastic_kernel( net_params p, plastic_params q )
{
	using Syn = typename Model::synapse;
	snn_info const info{ p.n };
	long long const nthreads = (long long)gridDim.x * blockDim.x;
	long long const gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	for( long long e = gid; e < (long long)p.n * p.width; e += nthreads )
	{
		int const src = (int)( e / p.width );
		int const dst = p.edges[e];
		float w = 0.0f;
		if( dst != INT_MAX )
		{
			weight_iter_rw it{ w };
			device_backend bak( p.seed, (uint32_t)src, 0u );
			Syn::init( it, src, dst, info, bak );
		}
		q.W[e] = w;
	}
	for( long long i = gid; i < p.n; i += nthreads )
	{
		q.zpre[i] = Syn::trace_init;
		q.zpost[i] = Syn::trace_init;
	}
}

// Look-ahead state at step 0 from Zpre(-1) = q.zpre: nothing arrives before step `delay`,
// so the owner's row-state machine runs over the touch steps 0 .. delay-1 without arrivals.
template <typename Model>
__global__ void init_lookahead( net_params p, plastic_params q, float dt )
{
	using Syn = typename Model::synapse;
	snn_info const info{ p.n };
	long long const nthreads = (long long)gridDim.x * blockDim.x;
	for( long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < p.n; i += nthreads )
	{
		device_backend bak( p.seed, (uint32_t)i, 0u );
		float z = q.zpre[i];
		int rf = -1;
		float zrf = 0.0f;
		float c = 0.0f, sum = 0.0f;
		for( int tp = 0; tp < p.delay; tp++ )
		{
			float const d = kahan_add( c, sum, dt );
			float const zn = fmaf( z, Syn::trace_decay( d ), 0.0f );
			if( Syn::plastic_src( (int)i, info ) )
			{
				int off;
				float zr;
				row_step( rf, zrf, false, z, Syn::potentiation_active( zn, d, bak ), tp, off, zr );
			}
			z = zn;
		}
		q.za[i] = z;
		q.hist[i] = 0ull;
		q.rf_a[i] = rf;
		q.zrf_a[i] = zrf;
		q.rf_c[i] = -1;
		q.zrf_c[i] = 0.0f;
	}
}

// Settled weights for export: W plus every event still pending at `now` (the completion
// of arrivals at now - 1 and the replay window of pre-active rows), written to `out`.
template <typename Model>
__global__ void settle_weights( net_params p, plastic_params q, float * out )
{
	using Syn = typename Model::synapse;
	snn_info const info{ p.n };
	__shared__ float zw[64];
	long long const now = p.clock->step;
	int const src = blockIdx.x;
	if( !Syn::plastic_src( src, info ) ) return;
	int const rf = q.rf_c[src];
	// hist bit j: fired at now - 1 - j; an arrival at now - 1 fired at now - 1 - delay
	bool const arrived_last = now - 1 >= p.delay && ( ( q.hist[src] >> p.delay ) & 1ull );
	int const rf_off = ( rf >= 0 && rf <= now - 1 ) ? (int)( now - rf ) : 0;
	if( !arrived_last && rf_off == 0 ) return;
	device_backend bak( p.seed, (uint32_t)src, (uint32_t)now );
	float const dt_last = now >= 1 ? p.dt_ring[( now - 1 ) % DT_RING] : 0.0f;
	if( rf_off > 0 && threadIdx.x == 0 )
	{
		float z = q.zrf_c[src];
		for( int i = 0; i < rf_off; i++ )
		{
			long long const tau = now - rf_off + i;
			z = fmaf( z, Syn::trace_decay( p.dt_ring[tau % DT_RING] ), 0.0f );
			zw[i] = z;
		}
	}
	__syncthreads();
	float const zt = q.zpre[src];
	bool const pot = arrived_last && Syn::potentiation_active( zt, dt_last, bak );
	int const * row = p.edges + (long long)src * p.width;
	for( int j = threadIdx.x; j < p.width; j += blockDim.x )
	{
		int const d = row[j];
		if( d == INT_MAX || !Syn::plastic_dst( d, info ) ) continue;
		long long const e = (long long)src * p.width + j;
		float w = out[e];
		unsigned long long const h = q.hist[d];
		if( arrived_last )
		{
			// the pending completion of the arrival at now - 1; the replay window of an
			// arrival row starts after it
			bool const x_d = h & 1ull;
			bool const dpa = Syn::depression_active( q.zpost[d], dt_last, bak );
			if( dpa || ( x_d && pot ) ) w = Syn::update( w, true, x_d, zt, q.zpost[d], dt_last, bak );
		}
		else
		{
			unsigned long long const wm = rf_off >= 64 ? ~0ull : ( ( 1ull << rf_off ) - 1 );
			unsigned long long hb = h & wm;
			while( hb )
			{
				int const jj = 63 - __clzll( (long long)hb );
				hb &= ~( 1ull << jj );
				long long const tau = now - 1 - jj;
				w = Syn::update( w, false, true, zw[tau - ( now - rf_off )], 1.0f, p.dt_ring[tau % DT_RING], bak );
			}
		}
		out[e] = w;
	}
}

// Reference-shaped synapse export, one trace at a time (which = 0: Zpre, 1: Zpost) per
// slot: plastic synapses carry the per-neuron trace, other valid synapses its initial
// value (the reference never updates them), padding slots 0.
template <typename Model>
__global__ void expand_trace( net_params p, plastic_params q, int which, float * out )
{
	using Syn = typename Model::synapse;
	snn_info const info{ p.n };
	long long const nthreads = (long long)gridDim.x * blockDim.x;
	for( long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)p.n * p.width; e += nthreads )
	{
		int const src = (int)( e / p.width );
		int const dst = p.edges[e];
		float v = 0.0f;
		if( dst != INT_MAX ) v = Syn::plastic( src, dst, info ) ? ( which == 0 ? q.zpre[src] : q.zpost[dst] ) : Syn::trace_init;
		out[e] = v;
	}
}

inline int plastic_window_smem( int tile, int ntiles, int threads )
{
	size_t b = (size_t)PL_CHUNK * tile * 4 + (size_t)tile * 4 + (size_t)tile * 8 + (size_t)tile * 4 + ( ( tile + 15 ) & ~15 );
	b += (size_t)( ( ntiles + 1 + 3 ) & ~3 ) * 4;
	b += (size_t)PL_STAGE * sizeof( stage_e );
	b += (size_t)( threads / 32 ) * 64 * 4;
	return (int)b;
}

// device buffers of the plastic state
struct plastic_state
{
	// from cudaMalloc, or (pool set) from a stream-ordered pool on stream s
	struct buf
	{
		void * p = nullptr;
		size_t bytes = 0;
		cudaMemPool_t pool = nullptr;
		cudaStream_t s = nullptr;
		~buf() { release(); }
		void release()
		{
			if( p )
			{
				if( pool )
					cudaFreeAsync( p, s );
				else
					cudaFree( p );
			}
			p = nullptr;
			bytes = 0;
		}
		void alloc( size_t b, cudaMemPool_t from, cudaStream_t on )
		{
			release();
			if( !b ) return;
			cudaError_t const e = from ? cudaMallocFromPoolAsync( &p, b, from, on ) : cudaMalloc( &p, b );
			if( e != cudaSuccess )
			{
				p = nullptr;
				cudaGetLastError();
				throw std::bad_alloc();
			}
			bytes = b;
			pool = from;
			s = on;
		}
	};
	buf W, za, zpre, zpost, hist, rf_a, zrf_a, rf_c, zrf_c, ring_meta, flush_ring, flush_cnt, ring_pot, tmp;
	bool active = false;
	cudaMemPool_t pool = nullptr; // where the buffers come from (null: cudaMalloc)
	cudaStream_t stream = nullptr;

	size_t bytes() const
	{
		return W.bytes + za.bytes + zpre.bytes + zpost.bytes + hist.bytes + rf_a.bytes + zrf_a.bytes + rf_c.bytes + zrf_c.bytes +
		       ring_meta.bytes + flush_ring.bytes + flush_cnt.bytes + ring_pot.bytes + tmp.bytes;
	}

	void allocate( long long n, long long width, int ntiles, int delay, cudaStream_t stream, cudaMemPool_t from )
	{
		active = true;
		pool = from;
		this->stream = stream;
		W.alloc( (size_t)( n * width ) * 4, pool, stream );
		za.alloc( n * 4, pool, stream );
		zpre.alloc( n * 4, pool, stream );
		zpost.alloc( n * 4, pool, stream );
		hist.alloc( n * 8, pool, stream );
		rf_a.alloc( n * 4, pool, stream );
		zrf_a.alloc( n * 4, pool, stream );
		rf_c.alloc( n * 4, pool, stream );
		zrf_c.alloc( n * 4, pool, stream );
		ring_meta.alloc( (size_t)2 * delay * n * 16, pool, stream );
		flush_ring.alloc( (size_t)2 * delay * n * 16, pool, stream );
		flush_cnt.alloc( (size_t)2 * delay * ntiles * 4, pool, stream );
		ring_pot.alloc( (size_t)2 * delay * ntiles * 4, pool, stream );
		// on the net's stream, ahead of the kernels that read them
		cudaMemsetAsync( flush_cnt.p, 0, flush_cnt.bytes, stream );
		cudaMemsetAsync( ring_pot.p, 0, ring_pot.bytes, stream );
	}

	plastic_params params() const
	{
		plastic_params q{};
		q.W = static_cast<float *>( W.p );
		q.za = static_cast<float *>( za.p );
		q.zpre = static_cast<float *>( zpre.p );
		q.zpost = static_cast<float *>( zpost.p );
		q.hist = static_cast<unsigned long long *>( hist.p );
		q.rf_a = static_cast<int *>( rf_a.p );
		q.zrf_a = static_cast<float *>( zrf_a.p );
		q.rf_c = static_cast<int *>( rf_c.p );
		q.zrf_c = static_cast<float *>( zrf_c.p );
		q.ring_meta = static_cast<int4 *>( ring_meta.p );
		q.flush_ring = static_cast<int4 *>( flush_ring.p );
		q.flush_cnt = static_cast<unsigned *>( flush_cnt.p );
		q.ring_pot = static_cast<unsigned *>( ring_pot.p );
		return q;
	}

	// W from the reference's (W, Zpre, Zpost) tuples; the per-neuron traces from the
	// per-synapse Zpre / Zpost of plastic synapses (equal per neuron when they come from a
	// net in the reference's state); only before the first step.
	template <typename Model>
	void import( net_params const & p, float const * w, float const * zpre_syn, float const * zpost_syn, float dt, int sms, cudaStream_t s )
	{
		using Syn = typename Model::synapse;
		snn_info const info{ p.n };
		long long const ne = (long long)p.n * p.width;
		std::vector<int> edges( (size_t)ne );
		if( ne ) cudaMemcpyAsync( edges.data(), p.edges, ne * 4, cudaMemcpyDeviceToHost, s );
		cudaStreamSynchronize( s );
		std::vector<float> zpre_n( p.n, Syn::trace_init ), zpost_n( p.n, Syn::trace_init );
		for( long long e = 0; e < ne; e++ )
		{
			int const src = (int)( e / p.width ), dst = edges[e];
			if( dst == INT_MAX || !Syn::plastic( src, dst, info ) ) continue;
			zpre_n[src] = zpre_syn[e];
			zpost_n[dst] = zpost_syn[e];
		}
		if( ne ) cudaMemcpyAsync( W.p, w, ne * 4, cudaMemcpyHostToDevice, s );
		cudaMemcpyAsync( zpre.p, zpre_n.data(), p.n * 4, cudaMemcpyHostToDevice, s );
		cudaMemcpyAsync( zpost.p, zpost_n.data(), p.n * 4, cudaMemcpyHostToDevice, s );
		init_lookahead<Model><<<4 * sms, 256, 0, s>>>( p, params(), dt );
		cudaStreamSynchronize( s );
	}

	// Reference-shaped export: settled weights (pending events applied, the net's own
	// state untouched) and the re-expanded traces.
	template <typename Model>
	cudaError_t export_synapses( net_params const & p, float * w, float * zpre_syn, float * zpost_syn, int sms, cudaStream_t s )
	{
		long long const ne = (long long)p.n * p.width;
		if( ne == 0 ) return cudaSuccess;
		if( tmp.bytes < (size_t)ne * 4 ) tmp.alloc( (size_t)ne * 4, pool, stream );
		float * t = static_cast<float *>( tmp.p );
		cudaMemcpyAsync( t, W.p, ne * 4, cudaMemcpyDeviceToDevice, s );
		settle_weights<Model><<<p.n, 256, 0, s>>>( p, params(), t );
		cudaMemcpyAsync( w, t, ne * 4, cudaMemcpyDeviceToHost, s );
		expand_trace<Model><<<4 * sms, 256, 0, s>>>( p, params(), 0, t );
		cudaMemcpyAsync( zpre_syn, t, ne * 4, cudaMemcpyDeviceToHost, s );
		expand_trace<Model><<<4 * sms, 256, 0, s>>>( p, params(), 1, t );
		cudaMemcpyAsync( zpost_syn, t, ne * 4, cudaMemcpyDeviceToHost, s );
		return cudaStreamSynchronize( s );
	}
};

template <typename Model>
void init_plastic( net_params const & p, plastic_state & ps, float dt, int sms, cudaStream_t s )
{
	init_plastic_kernel<Model><<<4 * sms, 256, 0, s>>>( p, ps.params() );
	init_lookahead<Model><<<4 * sms, 256, 0, s>>>( p, ps.params(), dt );
}
} // namespace spk
