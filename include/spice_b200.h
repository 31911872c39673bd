/* spice_b200 -- C ABI of the B200 simulation path.
 *
 * A C-ABI shared library (libspice_b200.so) over hand-written sm_100a kernels. The C++17
 * class template spice::cuda::snn<Model> (include/spice/cuda/snn.h) is a thin wrapper over
 * these calls, and the Python package spice_b200 binds them with ctypes. Every function
 * returns an spk_status; on failure spk_last_error() holds a message (per host thread).
 * Nothing here takes or returns torch types, C++ objects or CUDA handles other than a
 * cudaStream_t passed as void*.
 */
#ifndef SPICE_B200_H
#define SPICE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum spk_status
{
	SPK_OK = 0,
	SPK_ERR_INVALID = 1,  /* bad argument (the reference throws std::invalid_argument)      */
	SPK_ERR_CUDA = 2,     /* CUDA runtime error (the reference throws std::runtime_error)    */
	SPK_ERR_NOMEM = 3,    /* device allocation failed (the reference throws std::bad_alloc)  */
	SPK_ERR_DEVICE = 4,   /* a kernel reported an error through the net's device error word */
	SPK_ERR_CAPACITY = 5, /* an output buffer is too small; *count tells the size needed    */
	SPK_ERR_TIMEOUT = 6   /* a host-side wait ran out (spk_server_wait)                      */
} spk_status;

typedef enum spk_model
{
	SPK_VOGELS_ABBOTT = 0, /* spice/models/vogels_abbott.h          */
	SPK_BRUNEL = 1,        /* spice/models/brunel.h                 */
	SPK_BRUNEL_PLUS = 2,   /* spice/models/brunel_with_plasticity.h */
	SPK_SYNTH = 3,         /* spice/models/synth.h                  */
	/* the same models with the benchmark configurations' constants (no reference
	   counterpart; see each header): */
	SPK_VOGELS_ABBOTT_NS = 4, /* include/spice/models/vogels_abbott_ns.h: 0.27 / 4.5 nS, V uniform in [-60, -50) mV */
	SPK_BRUNEL_FIXED = 5,     /* include/spice/models/brunel_fixed.h: reset 10 mV, J = 0.1 / -0.5 mV */
	SPK_BRUNEL_PLUS_A012 = 6, /* include/spice/models/brunel_with_plasticity_a012.h: A- = 0.012 */
	/* a model of the user's, compiled into a build of the library with
	   -DSPK_USER_MODEL_HEADER='"header.h"' -DSPK_USER_MODEL=its::type (spice_b200.build.build_user);
	   absent (SPK_ERR_INVALID) from the default build */
	SPK_USER_MODEL_ID = 7
} spk_model;

/* Population sizes and (src_pop, dst_pop, p) connection list: the arguments of
 * spice::util::layout(pops, connections) (spice/util/layout.h:30-33). */
typedef struct spk_layout_desc
{
	int npops;
	uint64_t const * pops;
	int nconn;
	int const * conn_src;
	int const * conn_dst;
	float const * conn_p;
} spk_layout_desc;

typedef struct spk_net spk_net;

typedef struct spk_net_info
{
	int model;
	int device;
	uint64_t num_neurons;  /* snn::num_neurons()  (spice/snn.h:24)                       */
	uint64_t num_synapses; /* snn::num_synapses() = num_neurons * width (spice/snn.h:25) */
	uint64_t width;        /* ELL row width = layout::max_degree()                      */
	int delay;             /* snn::delay()  (spice/snn.h:27)                             */
	float dt;              /* snn::dt()     (spice/snn.h:26)                             */
	uint64_t steps;        /* steps taken so far                                         */
	uint64_t tile_size;    /* destination neurons per tile (one CTA each)                */
	uint64_t num_tiles;
	uint64_t device_bytes; /* device memory held by the net                              */
	uint64_t kernel_launches; /* simulation kernel launches so far (a CUDA graph's replay
	                             counts each window; a batch counts its shared launches)  */
	int persistent;        /* 1: spk_net_run advances the net in one cooperative launch */
	int slice_pack;        /* window_flat slices: 8 (16-bit) or 12 (10-bit) indices per
	                          16-byte vector; 0 for the other window kernels            */
	int slot_vecs;         /* window_slots: 16-byte vectors per fixed (source, tile) slot;
	                          0 when the net keeps variable slices                     */
} spk_net_info;

/* Message of the last failed call on this host thread ("" if none). */
char const * spk_last_error( void );

/* Flattened layout: replaces spice::util::layout's constructor and accessors
 * (spice/util/layout.cpp:51-110, size()/connections()/max_degree() at :111-113).
 * Writes up to `cap` tuples (src_first, src_last, dst_first, dst_last) to out_ranges and
 * their probabilities to out_p; *out_count = number of connections. */
int spk_layout_flatten(
    spk_layout_desc const * desc,
    int * out_ranges,
    float * out_p,
    int cap,
    int * out_count,
    uint64_t * out_size,
    uint64_t * out_max_degree );

/* Generate the ELL adjacency of `desc` on the device into d_edges
 * (size * max_degree int32, rows ascending, INT_MAX padded), asynchronously on `stream`.
 * Replaces spice::cuda::generate_adj_list (spice/cuda/algorithm.h:15). The generator is
 * counter-based: edge src->dst exists iff Philox(seed; src, j/4, conn, 'GRAP')[j%4] <
 * floor(p * 2^32) for candidate j = dst - dst_first, truncated at the row width. */
int spk_generate_adj_list( void * stream, spk_layout_desc const * desc, uint64_t seed, int32_t * d_edges );

/* Allocation-free variant of spk_generate_adj_list: the same graph for the same layout and
 * seed, for callers that must not allocate device memory -- code inside a framework whose
 * caching allocator owns the device (a raw cudaMalloc takes memory behind the pool's back
 * and can fail mid-run), or latency-critical loops that cannot pay the device-wide
 * synchronisation of cudaMalloc/cudaFree. No counterpart in the reference.
 * The connection table goes to a fixed device array of the library (24 KiB per GPU, held
 * until the process exits): at most 1024 connections and 1024 populations, larger layouts
 * are rejected with SPK_ERR_INVALID. d_edges (size * max_degree int32) is the caller's.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current: make it before any stream capture. Every call on a device
 * shares the one array and leaves its table there; calls whose copies and kernels overlap
 * on the GPU (different streams) race on it, so order them. The stream must belong to the
 * current device. */
int spk_generate_adj_list_static( void * stream, spk_layout_desc const * desc, uint64_t seed, int32_t * d_edges );

/* cuda::snn<Model>(layout, dt, delay) (spice/cuda/snn.h:20-25, spice/cuda/snn.d.cpp:136-165):
 * allocates the net on `device`, generates the graph from `graph_seed`, initialises
 * neurons and synapses. `seed` keys the per-(step, neuron) Poisson draws. */
int spk_net_create(
    spk_net ** out,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    int device );

/* spk_net_create with the number of window_flat tiles chosen for about `tile_target`
 * (0 = one per SM, the default): a net that shares the GPU with others (a batch, a server)
 * takes fewer CTAs. Results do not depend on the tiling. */
int spk_net_create_ex(
    spk_net ** out,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    int device,
    int tile_target );

/* Build choices of a net. A field at -1 is chosen automatically; for such a field the
 * environment variable named beside it, where set, overrides the automatic choice (a test
 * hook: an explicit field value always wins). Results never depend on these choices: they
 * select kernels and data layouts that all compute the same integer spike counts. */
typedef struct spk_net_options
{
    int tile_target; /* window_flat tiles: about this many; 0 = one per SM */
    int kernel;      /* SPK_KERNEL: 0 = window kernels (window_flat where the model allows), 1 = window_counts ("direct"),
                        automatic: window_flat, except window_counts at delay 1 for nets of at most 1e7 synapses,
                        2 = window_ordered ("ordered": the generic kernel, every arrival through the model's receive()
                        in the reference CPU simulator's order; the only kernel of models without input classes or with
                        synapse attributes, and of no plastic model) */
    int slice_bits;  /* SPK_PACK: 10 = 10-bit target indices where every index fits (12 to a vector), 16 = 16-bit (8 to a vector) */
    int tiling;      /* SPK_TILES: 0 = tiles balanced by per-neuron cost, 1 = equal tiles ("uniform") */
    int persistent;  /* SPK_PERSIST: 1 = one cooperative launch per run when every tile's CTA is resident, 0 = windowed launches */
    int pipelined;   /* SPK_FLAT_SYNC (inverted): 1 = window_flat's step pipeline, 0 = every step synchronous */
    int slots;       /* SPK_SLOTS: 1 = fixed slots (window_slots) where they fit, 0 = variable slices (the automatic choice) */
} spk_net_options;

/* Every field automatic (-1), tile_target 0. */
void spk_net_options_init( spk_net_options * opts );

/* spk_net_create with explicit build choices (`opts` null: all automatic). */
int spk_net_create_opts(
    spk_net ** out,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    int device,
    spk_net_options const * opts );

/* Upper estimate of the device memory (bytes) a net of this model, layout, delay and tile
 * target would hold once built: what a server admits against its memory budget. */
int spk_net_estimate_bytes( int model, spk_layout_desc const * desc, int delay, int device, int tile_target, uint64_t * out_bytes );

/* spk_net_estimate_bytes for a net built with `opts` (null: all automatic). */
int spk_net_estimate_bytes_opts( int model, spk_layout_desc const * desc, int delay, int device, spk_net_options const * opts, uint64_t * out_bytes );

/* cuda::snn<Model>(adj, width, dt, delay) (spice/cuda/snn.h:26-32, spice/cuda/snn.d.cpp:167-199):
 * imports an ELL adjacency (num_neurons x width int32, rows ascending, INT_MAX padded,
 * width a multiple of 32) from host memory and initialises neurons and synapses. */
int spk_net_create_from_adj(
    spk_net ** out,
    int model,
    int32_t const * edges,
    uint64_t num_neurons,
    uint64_t width,
    float dt,
    int delay,
    uint64_t seed,
    int device );

/* Import neuron / synapse state from host memory, one array per attribute in the model's
 * attribute order (float or int32, num_neurons resp. num_synapses entries). With
 * spk_net_create_from_adj this is the conversion constructor cuda::snn(const snn&)
 * (spice/cuda/snn.d.cpp:201-221). For brunel_with_plasticity the synapse attributes are
 * the reference's (W, Zpre, Zpost); Zpre / Zpost must be consistent per neuron. */
int spk_net_set_neurons( spk_net * net, void * const * attrs );
int spk_net_set_synapses( spk_net * net, void * const * attrs );

int spk_net_destroy( spk_net * net );

/* snn::step(std::vector<int>* out) (spice/snn.h:22, spice/cuda/snn.d.cpp:224-289).
 * With out_ids == NULL the step is queued and launched together with later steps (in
 * windows of up to `delay` steps, identical results). With out_ids != NULL all queued
 * steps and this one run, and the ids that fired this step are copied out in ascending
 * order; *out_count receives their number (SPK_ERR_CAPACITY if > cap). */
int spk_net_step( spk_net * net, int32_t * out_ids, uint64_t cap, uint64_t * out_count );

/* Advance `nsteps` steps: the same as nsteps calls of step(nullptr). Non-plastic nets
 * whose tiles fit the GPU at once run them as one cooperative launch (tiles wait, bounded,
 * for the spikes they read); other nets as delay-step windows replayed from a CUDA graph.
 * spk_net_info reports which (persistent) and the launches made (kernel_launches). */
int spk_net_run( spk_net * net, uint64_t nsteps );

/* Advance `nsteps` steps and return their spike raster to host memory: counts[k] = number
 * of spikes of step k, ids = all spike ids concatenated in step order (ascending within a
 * step). *out_total = total spikes; SPK_ERR_CAPACITY (state advanced, nothing copied) if
 * it exceeds ids_cap. */
int spk_net_run_record( spk_net * net, uint64_t nsteps, uint32_t * counts, int32_t * ids, uint64_t ids_cap, uint64_t * out_total );

/* The CUDA stream (cudaStream_t) every kernel of this net runs on, for callers that order
 * their own work or record events against it. Queued steps are launched first. The stream
 * belongs to the library: do not destroy it (spk_net_destroy does; a server's nets hand
 * theirs on to the server's later nets). */
int spk_net_stream( spk_net * net, void ** out_stream );

/* Wait for all queued work; reports device-side errors. */
int spk_net_sync( spk_net * net );

/* Queued steps launched; *out_idle = 1 if the net's stream has finished all its work
 * (without waiting; device-side errors are reported by spk_net_sync). */
int spk_net_idle( spk_net * net, int * out_idle );

int spk_net_get_info( spk_net * net, spk_net_info * out );

/* snn::adj() (spice/snn.h:31): the ELL edges (num_neurons * width int32). */
int spk_net_adj( spk_net * net, int32_t * out, uint64_t cap );

/* snn::neurons() / snn::synapses() (spice/snn.h:32-33) as structure-of-arrays: one host
 * array per attribute, model attribute order. */
int spk_net_neurons( spk_net * net, void * const * attrs );
int spk_net_synapses( spk_net * net, void * const * attrs );

/* Checkpoints. The reference's snapshot is adj() + neurons() + synapses() and the
 * conversion constructor (spice/cuda/snn.d.cpp:123-143), which drops the spikes in flight
 * and the lazy-STDP history. A checkpoint keeps everything a net needs to continue bit
 * for bit: edges, neuron state, the spike ring and its publication flags, the simulated
 * clock and, for Brunel+, the lazy-STDP state; derived tables are rebuilt on restore.
 * spk_net_checkpoint with buf == NULL returns the size in *out_bytes; otherwise it writes
 * that many bytes (SPK_ERR_INVALID if cap is smaller). spk_net_restore makes a new net on
 * `device` that continues where the saved one stood (same tiling; the checkpoint is
 * validated before any device work). */
int spk_net_checkpoint( spk_net * net, void * buf, uint64_t cap, uint64_t * out_bytes );
int spk_net_restore( spk_net ** out, void const * buf, uint64_t size, int device );

/* Attribute counts of a model's neuron and synapse tuples (as exported above) and, per
 * attribute, 'f' (float32) or 'i' (int32) in types (neuron attributes, then synapse). */
int spk_model_attrs( int model, int * num_neuron_attrs, int * num_synapse_attrs, char * types, int types_cap );

/* ---- batching: many independent nets stepped together ------------------------------
 * The reference steps one net per snn object (spice/cuda/snn.d.cpp:224-289); a workload
 * of many small nets is a host loop over them (spice_bench/paper_plots.cpp:184-231). A
 * batch advances all its nets by the same number of steps with shared kernel launches:
 * each launch runs every tile of every net of one model for up to that net's delay in
 * steps, one CTA per (net, tile). Results are identical to stepping each net alone. */
typedef struct spk_batch spk_batch;

/* Re-tile a net, before its first step, into about `target` tiles (>= 1): a net sharing
 * the GPU with others in a batch takes fewer CTAs than a net alone (one per SM). */
int spk_net_set_tile_target( spk_net * net, int target );

/* window_flat's split of its 32 warps: `warps` (4-24, default 12) stage the next steps'
 * arrivals and copy their slices (the last of them compacts and publishes the tile's
 * spikes), the rest count arrivals and update neurons. A tuning choice for nets of
 * different sizes (the batch autotuner sets it per size bucket); results do not depend on
 * it. Nets of the other kernels ignore it. */
int spk_net_set_producer_warps( spk_net * net, int warps );

int spk_batch_create( spk_batch ** out, int device );
/* Nets of any model, on the batch's device; a net belongs to at most one batch. The nets
 * of one model share launches (window_flat_batch, window_slots_batch, window_plastic_batch:
 * one CTA per (net, tile), a round of up to each net's delay in steps); nets of the generic
 * kernel (window_ordered) and of window_counts run their own windows beside them. */
int spk_batch_add( spk_batch * batch, spk_net * net );
int spk_batch_remove( spk_batch * batch, spk_net * net );
/* Advance every net of the batch by `nsteps` steps (asynchronous against the host up to
 * the launches; each net's own stream is ordered after them, so spk_net_sync and the
 * state exports of a net see the batch's steps). */
int spk_batch_run( spk_batch * batch, uint64_t nsteps );
/* Advance nets[i] (members of the batch, each listed once) by nsteps[i] steps. */
int spk_batch_run_nets( spk_batch * batch, int count, spk_net * const * nets, uint64_t const * nsteps );
int spk_batch_destroy( spk_batch * batch );

/* ---- serving: jobs admitted against a device-memory budget, continuously batched ----
 * A server owns builder threads (they build admitted jobs' nets), a ticker thread (it
 * steps the batch) and one batch on `device`. Submitted jobs queue in
 * arrival order; the head is admitted when its estimated device memory
 * (spk_net_estimate_bytes) fits the budget beside the running jobs, and its net is built
 * with a tile count sized to its share of the load. Every tick advances each running job
 * by up to `quantum_steps` steps in one batch run; jobs admitted meanwhile join the next
 * tick. A completed job's final neuron state is kept in host memory (same values as the
 * net stepped alone) and its device memory is freed at once. */
typedef struct spk_server spk_server;

typedef enum spk_job_state
{
	SPK_JOB_QUEUED = 0,
	SPK_JOB_RUNNING = 1,
	SPK_JOB_DONE = 2,
	SPK_JOB_FAILED = 3,    /* building or stepping failed: error and message say why   */
	SPK_JOB_CANCELLED = 4,
	SPK_JOB_TIMEOUT = 5,   /* the job's deadline passed before it completed            */
	SPK_JOB_REFUSED = 6    /* larger than the whole budget: refused at submission      */
} spk_job_state;

typedef struct spk_job_info
{
	int state;             /* spk_job_state                                             */
	int error;             /* spk_status of a failed or refused job                     */
	uint64_t steps_done;
	uint64_t steps_total;
	uint64_t num_neurons;  /* of a completed job (its state's length)                  */
	uint64_t device_bytes; /* held against the budget while queued for admission / running */
	double t_submit;       /* seconds since the server was created                      */
	double t_start;        /* admission (-1 before)                                     */
	double t_end;          /* completion, failure, cancellation or timeout (-1 before)  */
	char message[160];
} spk_job_info;

typedef struct spk_server_stats
{
	uint64_t queued, running, done, failed, cancelled, timed_out, refused;
	uint64_t bytes_in_use, peak_bytes, budget_bytes;
	uint64_t ticks;
	double build_seconds; /* building admitted jobs' nets (builder thread)          */
	double tick_seconds;  /* ticks: batch runs until every stepped net synchronised */
} spk_server_stats;

/* Starts the builder threads (two) and the ticker. The
 * budget (at most the device's free memory less 1 GiB) is mapped into the device's
 * stream-ordered memory pool first, and the jobs' nets are built from that pool, so
 * neither building nor freeing a net synchronises the device; creation takes about 2-3.5 s
 * for 150 GB, and spk_server_destroy hands the memory back. */
int spk_server_create( spk_server ** out, int device, uint64_t budget_bytes, uint64_t quantum_steps );
/* spk_server_create with `builders` builder threads (1-8; 0 = automatic: two, or the test
 * override SPK_SERVER_BUILDERS). */
int spk_server_create_ex( spk_server ** out, int device, uint64_t budget_bytes, uint64_t quantum_steps, int builders );
/* Queue a job: the arguments of spk_net_create, its number of steps and a deadline in
 * seconds from submission (0 = none). SPK_ERR_NOMEM (and a job in state REFUSED) if the
 * job alone exceeds the budget. */
int spk_server_submit(
    spk_server * server,
    int model,
    spk_layout_desc const * desc,
    float dt,
    int delay,
    uint64_t seed,
    uint64_t graph_seed,
    uint64_t nsteps,
    double timeout_s,
    uint64_t * out_job );
int spk_server_job_info( spk_server * server, uint64_t job, spk_job_info * out );
/* Final neuron state of a completed job, one host array per attribute (spk_model_attrs). */
int spk_server_job_neurons( spk_server * server, uint64_t job, void * const * attrs );
int spk_server_cancel( spk_server * server, uint64_t job );
/* Forget a finished job (frees its host results). */
int spk_server_release( spk_server * server, uint64_t job );
/* Block until `job` (0 = every job) is finished; timeout_s < 0 waits without limit,
 * otherwise SPK_ERR_TIMEOUT when it runs out. */
int spk_server_wait( spk_server * server, uint64_t job, double timeout_s );
int spk_server_get_stats( spk_server * server, spk_server_stats * out );
/* Fault injection on the host: the next `count` admissions fail as an allocation failure
 * would (the job ends FAILED with SPK_ERR_NOMEM; the server carries on). */
int spk_server_inject_alloc_failures( spk_server * server, int count );
/* Fault injection on the host: at the job's next tick its net reports a device error, as
 * when a kernel's bounded wait runs out (its error word set); the job ends FAILED with
 * SPK_ERR_DEVICE and the other jobs carry on. SPK_ERR_INVALID for an unknown or finished
 * job. */
int spk_server_inject_device_error( spk_server * server, uint64_t job );
/* Stops both threads; queued and running jobs are dropped. */
int spk_server_destroy( spk_server * server );

#ifdef __cplusplus
}
#endif

#endif /* SPICE_B200_H */
