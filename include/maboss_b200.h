/*
 * maboss_b200.h -- C ABI of the B200 (sm_100a) trajectory engine for stochastic Boolean
 * networks (MaBoSS semantics).
 *
 * This is the boundary that replaces, for the trajectory hot path, the C++ classes of the
 * reference implementation (paths relative to the reference project):
 *   driver            src/parser/driver.h:14-56          -> mb_model_*
 *   generator         src/generator.h:7-23               -> mb_model_generate_code
 *   kernel_compiler   src/kernel_compiler.h:8-20         -> mb_context_*, mb_module_*
 *   kernel_wrapper    src/kernel.h:5-23                  -> mb_launch_*
 *   simulation_runner src/simulation_runner.h:8-24       -> mb_run*, mb_result_*
 *   stats plugins     src/statistics/stats.h:15-29,
 *                     window_average_small.h, final_states.h, fixed_states.h -> mb_launch_*_stats,
 *                     mb_result_* and the CSV writers
 *
 * Conventions:
 *   - every function returns an mb_status (MB_OK == 0) and never exits the process; the
 *     message of the last failure on the calling thread is returned by mb_last_error();
 *   - handles are opaque; pointers are plain host or device pointers, sizes are explicit;
 *   - device entry points take an explicit CUDA stream (cudaStream_t passed as void*);
 *     NULL means the context's own stream;
 *   - trajectory buffers are Structure-of-Arrays (SoA) with a row stride equal to the batch
 *     capacity B:  states[(slot * W + word) * B + traj], times[slot * B + traj],
 *     entropies[slot * B + traj], last_states[word * B + traj]
 *     (the reference uses Array-of-Structures [traj][slot][word]).
 */
#ifndef MABOSS_B200_H
#define MABOSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mb_status;
#define MB_OK 0
#define MB_ERR_INVALID 1   /* bad argument or handle */
#define MB_ERR_PARSE 2     /* malformed .bnd/.cfg or semantic model error */
#define MB_ERR_COMPILE 3   /* NVRTC compilation failure (log in mb_last_error) */
#define MB_ERR_CUDA 4      /* CUDA runtime/driver failure */
#define MB_ERR_LIMIT 5     /* size beyond a supported maximum, or out of device memory */
#define MB_ERR_NO_DEVICE 6 /* no usable sm_100 device */
#define MB_ERR_INTERNAL 7

typedef struct mb_model_s* mb_model;     /* parsed model            (reference: driver) */
typedef struct mb_context_s* mb_context; /* device + stream         (reference: kernel_compiler's context) */
typedef struct mb_module_s* mb_module;   /* compiled model kernels  (reference: kernel_compiler's module) */
typedef struct mb_result_s* mb_result;   /* statistics of one run   (reference: stats_composite after finalize) */

/* Run modes. */
#define MB_MODE_FUSED_EXACT 0 /* persistent kernel; bit-exact trajectories with the reference CUDA build */
#define MB_MODE_FUSED_FAST 1  /* persistent kernel; Philox streams; statistically equivalent */
#define MB_MODE_EPOCH 2       /* buffered 100-slot epochs through SoA trajectory buffers */
#define MB_MODE_EPOCH_DENSE 3 /* the same with the reference's per-step evaluation of every node's rate
                                 function (for comparisons with the reference algorithm; same results) */

/* Trajectory status byte (src/trajectory_status.h:3-8). */
#define MB_STATUS_CONTINUE 0
#define MB_STATUS_FINISHED 1
#define MB_STATUS_FIXED_POINT 2

const char* mb_version(void);
const char* mb_last_error(void);

/* ------------------------------------------------------------------ models (driver) */

/* driver::parse(bnd_file, cfg_file), src/parser/driver.cpp:16-31. */
mb_status mb_model_parse_files(const char* bnd_path, const char* cfg_path, mb_model* out);
/* Same, from in-memory text. */
mb_status mb_model_parse_text(const char* bnd_text, const char* cfg_text, mb_model* out);
mb_status mb_model_free(mb_model m);

/* driver::nodes (src/parser/driver.h:43): count, names, node_t::istate and node_t::is_internal
 * (src/parser/parse_types.h:16-29). */
mb_status mb_model_num_nodes(mb_model m, int* n);
mb_status mb_model_node_name(mb_model m, int i, char* buf, size_t cap, size_t* len);
mb_status mb_model_node_info(mb_model m, int i, float* istate, int* is_internal);
mb_status mb_model_set_istate(mb_model m, int i, float istate);

/* driver::constants and driver::variables (src/parser/driver.h:41-42). Missing constants read
 * as 0 like std::map::operator[] in src/main.cpp:128-132; missing variables are an error. */
/* Opt-in front-end change, no counterpart in the reference: every node attribute defined more than
 * once (in the .bnd and again in the .cfg) takes its last definition. The reference keeps the first
 * (src/parser/driver.cpp:65-77 appends the .cfg's attribute, src/parser/parse_types.cpp:6-13 returns
 * the first match), so by default a .cfg cannot override a .bnd rate or logic; call this after
 * parsing (before compiling) to let it. */
mb_status mb_model_apply_cfg_overrides(mb_model m);
mb_status mb_model_get_constant(mb_model m, const char* name, float* value);
mb_status mb_model_set_constant(mb_model m, const char* name, float value);
mb_status mb_model_get_variable(mb_model m, const char* name, float* value);
mb_status mb_model_set_variable(mb_model m, const char* name, float value);
mb_status mb_model_num_variables(mb_model m, int* n);
mb_status mb_model_variable_name(mb_model m, int i, char* buf, size_t cap, size_t* len);
/* Names of driver::constants in map order (the defaults of src/parser/driver.cpp:7-14 included). */
mb_status mb_model_num_constants(mb_model m, int* n);
mb_status mb_model_constant_name(mb_model m, int i, char* buf, size_t cap, size_t* len);

/* generator::generate_code(), src/generator.cpp:11-55. Writes the generated CUDA source
 * (NUL-terminated, truncated to cap) and its full length. */
mb_status mb_model_generate_code(mb_model m, char* buf, size_t cap, size_t* len);

/* ------------------------------------------------------------------ device / JIT (kernel_compiler) */

/* kernel_compiler::kernel_compiler(), src/kernel_compiler.cpp:46-52 (binds the primary context of
 * `device` instead of creating a private context). */
mb_status mb_context_create(int device, mb_context* out);
mb_status mb_context_free(mb_context c);
mb_status mb_context_stream(mb_context c, void** stream);
mb_status mb_context_sm_count(mb_context c, int* sm_count);

/* kernel_compiler::compile_simulation(code, discrete_time), src/kernel_compiler.cpp:61-164:
 * NVRTC-compiles generated code together with the engine kernels for sm_100a. */
mb_status mb_module_compile(mb_context c, const char* generated_code, mb_module* out);
/* Generate + compile in one call; the module keeps the model's layout. */
mb_status mb_module_compile_model(mb_context c, mb_model m, mb_module* out);
mb_status mb_module_free(mb_module mod);
/* NVRTC compilation of generated code + every engine kernel family for sm_100a without a
 * device (build checks); writes the total cubin size and the compiler log. */
mb_status mb_jit_check(const char* generated_code, size_t* cubin_size, char* log, size_t cap);
mb_status mb_module_state_size(mb_module mod, int* state_size, int* state_words);
/* NVRTC log of the compilation (may be empty). */
mb_status mb_module_log(mb_module mod, char* buf, size_t cap, size_t* len);

/* Device memory and synchronisation on the context's device, so that host code above this ABI
 * needs no CUDA runtime of its own (the reference allocates with thrust::device_malloc and copies
 * with cudaMemcpy, src/simulation_runner.cu:65-98). mb_memcpy copies in any direction (host or
 * device pointers) on `stream` and waits for it; mb_synchronize waits for all work on the device. */
mb_status mb_device_malloc(mb_context c, size_t bytes, void** ptr);
mb_status mb_device_free(mb_context c, void* ptr);
mb_status mb_memcpy(mb_context c, void* stream, void* dst, const void* src, size_t bytes);
mb_status mb_memset_async(mb_context c, void* stream, void* ptr, int value, size_t bytes);
mb_status mb_synchronize(mb_context c);
/* The context a module was compiled for. */
mb_status mb_module_context(mb_module mod, mb_context* out);

/* ------------------------------------------------------------------ kernel entry points (kernel_wrapper) */
/* Size in bytes of one per-trajectory random state (curandState, XORWOW). */
size_t mb_rand_state_size(void);

/* initialize_random, src/jit_kernels/simulation.cu:23-32: curand_init(seed, first + i, 0). */
mb_status mb_launch_initialize_random(mb_module mod, void* stream, int n, unsigned long long seed,
                                      unsigned long long first, void* rands);
/* initialize_initial_state, src/jit_kernels/simulation.cu:34-71 (SoA last_states). */
mb_status mb_launch_initialize_initial_state(mb_module mod, void* stream, int n, int stride,
                                             const float* initial_probs, uint32_t* last_states,
                                             float* last_times, void* rands);
/* simulate, src/generator.cpp:189-203 + src/jit_kernels/simulation.cu:77-164 (SoA buffers,
 * `traj_len` slots per epoch); adds the number of recorded steps to *transitions (device u64).
 * For models whose rates all have the @logic form the kernel keeps incremental unstable sets instead
 * of evaluating every rate function per step; trajectories are the same. */
mb_status mb_launch_simulate(mb_module mod, void* stream, int n, int stride, int traj_len,
                             uint32_t* last_states, float* last_times, void* rands,
                             uint32_t* traj_states, float* traj_times, float* traj_entropies,
                             uint8_t* statuses, unsigned long long* transitions);

/* Device-side statistics accumulators of one run (window_average_small_stats,
 * final_states_stats, fixed_states_stats). */
typedef struct mb_stats_s* mb_stats;
/* window_average_small_stats ctor (src/statistics/window_average_small.cpp:7-41) + the other two:
 * windows = ceil(max_time / time_tick); non-internal mask given as node indices. */
mb_status mb_stats_create(mb_module mod, float time_tick, float max_time, int discrete_time,
                          const int* noninternal_nodes, int n_noninternal, long long sample_count,
                          mb_stats* out);
/* The same with only some of the three accumulators (a bitwise OR of MB_STATS_*): one stats plugin
 * of src/statistics/ each (window_average_small_stats, final_states_stats, fixed_states_stats)
 * without the device memory of the other two. Launching the statistics of a missing section returns
 * MB_ERR_INVALID. time_tick, max_time and the non-internal nodes are ignored without MB_STATS_WINDOWS
 * and MB_STATS_FINAL (pass 1, 1 and none). */
#define MB_STATS_WINDOWS 1u
#define MB_STATS_FINAL 2u
#define MB_STATS_FIXED 4u
#define MB_STATS_ALL 7u
mb_status mb_stats_create_sections(mb_module mod, float time_tick, float max_time, int discrete_time,
                                   const int* noninternal_nodes, int n_noninternal, long long sample_count,
                                   unsigned sections, mb_stats* out);
mb_status mb_stats_free(mb_stats st);
/* window_average_small{,_discrete}, src/jit_kernels/window_average_small.cu:50-136 */
mb_status mb_launch_window_average_stats(mb_stats st, void* stream, int n, int stride, int traj_len,
                                         const uint32_t* traj_states, const float* traj_times,
                                         const float* traj_entropies);
/* final_states, src/jit_kernels/final_states.cu:9-21 */
mb_status mb_launch_final_states_stats(mb_stats st, void* stream, int n, int stride,
                                       const uint32_t* last_states, const uint8_t* statuses);
/* fixed_states_stats::process_batch, src/statistics/fixed_states.cu:84-125 */
mb_status mb_launch_fixed_states_stats(mb_stats st, void* stream, int n, int stride,
                                       const uint32_t* last_states, const uint8_t* statuses);
/* stats::finalize (device -> host); the result is independent of the stats object. */
mb_status mb_stats_finalize(mb_stats st, long long n_trajectories, mb_result* out);

/* The epoch batch's partition, src/simulation_runner.cu:126-139 (thrust::stable_partition of
 * last_states and thrust::partition of last_times and the random states by status == CONTINUE):
 * copies the CONTINUE trajectories of [0, n), in their order, to the front of a second buffer set
 * (out_states SoA [word * stride + j], out_times, out_rands; these must not overlap the inputs) and
 * writes their number to the device word *kept. `scratch` is device memory of
 * mb_partition_scratch_size(n) bytes. Finished slots are not carried over: new trajectories get
 * fresh random states from mb_launch_initialize_random (the reference reuses a freed slot's state). */
size_t mb_partition_scratch_size(int n);
mb_status mb_launch_partition(mb_module mod, void* stream, int n, int stride, const uint8_t* statuses,
                              const uint32_t* last_states, const float* last_times, const void* rands,
                              uint32_t* out_states, float* out_times, void* out_rands, void* scratch,
                              unsigned* kept);

/* Fixed-point statistics for callers that cannot allocate device memory. No counterpart in the
 * reference. Same result as mb_launch_fixed_states_stats followed by mb_stats_finalize (the
 * distinct FIXED_POINT states among the n trajectories and how many trajectories ended in each),
 * but the work table is a static 8 MiB device array inside this library instead of memory allocated
 * per call, so the call itself allocates nothing: use it from code whose device memory belongs to
 * someone else (a framework's caching allocator that owns the whole device, a process with a fixed
 * memory budget) or where a cudaMalloc would stall the device.
 *   inputs  (device): last_states[word * stride + i] and statuses[i] for i < n (SoA, as the kernels write them)
 *   outputs (device): out_states[j * state_words + w] and out_counts[j] for j < *out_n, in no particular
 *                     order; *out_n (host) is the number of distinct fixed points
 * Limits: state_words <= 64 (2048 nodes); at most P/2 distinct fixed points, P the largest power of
 * two with P * (20 + 4 * state_words) + 256 <= 8 MiB (131072 for 1 word, 16384 for 32 words); larger
 * inputs return MB_ERR_LIMIT with a message and *out_n = -1 (the count is unknown). When only
 * out_cap is too small, the call returns MB_ERR_LIMIT with *out_n = the number of distinct fixed
 * points and the first out_cap of them written. Runs on `stream` and synchronises it.
 * The device is the calling thread's current device (cudaGetDevice), not the stream's: make every
 * call with the stream's device current. The first call on a device, and the first call after that
 * device's context changed (cudaDeviceReset), looks up the array's device address in the current
 * context; make that call before any stream capture. Every call reuses the same array and clears it first, so
 * calls that overlap on the GPU (other streams, other host threads) race: serialise them. Every GPU
 * that loads the library holds the 8 MiB until the process exits. */
mb_status mb_fixed_states_noalloc(void* stream, int n, int stride, int state_words, const uint32_t* last_states,
                                  const uint8_t* statuses, uint32_t* out_states, unsigned* out_counts,
                                  int out_cap, int* out_n);

/* ------------------------------------------------------------------ whole runs (simulation_runner) */

typedef struct mb_run_config_s
{
    int mode;                      /* MB_MODE_* */
    long long sample_count;        /* number of trajectories */
    unsigned long long seed;       /* seed_pseudorandom */
    unsigned long long first_traj; /* random-stream id of trajectory 0 (sharding / replicas) */
    int traj_len;                  /* epoch length (reference: trajectory_len_limit = 100) */
    int batch_limit;               /* epoch batch (reference: trajectory_batch_limit = 1e6) */
    int block;                     /* threads per block (multiple of 32, <= 256) */
    int blocks_per_sm;             /* 0 = occupancy calculator */
    int fixed_capacity_log2;       /* fixed-point table capacity, 0 = automatic */
    long long stats_trajectories;  /* 0, or the trajectory count of the whole job when this run is one
                                      shard of it: window sums then use the job's fixed-point scale,
                                      so that mb_result_merge of the shards is exact */
    int bin_capacity_log2;         /* more than 20 non-internal nodes: log2 of the sparse-bin table size
                                      (24 bytes a slot), 0 = automatic (4 (T+1) n slots, 2^16 to 2^28) */
    int refill_reuse_rng;          /* epoch modes with more trajectories than one batch: 0 (default), a refilled
                                      slot's trajectory gets its own random stream (trajectory id); 1, it
                                      continues the random state of the trajectory that finished in that slot,
                                      in the order thrust::partition leaves them, as the reference does
                                      (simulation_runner.cu:126-153): the reference's results for n > batch */
} mb_run_config;

/* Defaults from the model's .cfg constants: mode FUSED_EXACT, traj_len 100, batch 1e6. */
mb_status mb_run_config_default(mb_model m, mb_run_config* cfg);

/* simulation_runner(n, N, seed, initial_probs).run_simulation(...) with the three built-in stats
 * plugins (src/main.cpp:54-83). The module must come from mb_module_compile_model. */
mb_status mb_run(mb_module mod, const mb_run_config* cfg, mb_result* out);

/* The run constants of a module compiled from generated code alone (mb_module_compile), which
 * the reference hands to simulation_runner (src/simulation_runner.h:17: sample count, seed,
 * initial probabilities) and to the statistics plugins (src/main.cpp:65-74: time_tick, max_time,
 * discrete_time, non-internal mask). */
typedef struct mb_run_params_s
{
    float time_tick;
    float max_time;
    int discrete_time;
    const float* initial_probs;    /* host, one per node */
    int n_nodes;
    const int* noninternal_nodes;  /* host, node indices in increasing order */
    int n_noninternal;
} mb_run_params;
/* mb_run for a module from mb_module_compile: cfg->sample_count and cfg->seed are used as given. */
mb_status mb_run_module(mb_module mod, const mb_run_config* cfg, const mb_run_params* params, mb_result* out);

/* Launch-shape autotuner of the fused modes (no counterpart in the reference, whose launches are
 * fixed at 256 threads): times candidate shapes (threads per block, resident blocks per SM; fewer
 * blocks than fit leave more L1 to the model tables) on a slice of the run's own trajectories and
 * writes the fastest into cfg->block and cfg->blocks_per_sm. *transitions_per_s (optional) is its
 * probe rate; up to `cap` candidates are reported fastest first in shapes[3 * i + {0, 1}] (block,
 * blocks per SM) with their rates in rates[i] (both optional). */
mb_status mb_autotune(mb_module mod, mb_run_config* cfg, float* transitions_per_s, int* shapes, float* rates,
                      int cap, int* n_shapes);

/* A run with device buffers allocated once (the reference allocates them per
 * simulation_runner::run_simulation, simulation_runner.cu:65-82). mb_runner_launch clears the
 * accumulators and enqueues the simulation on `stream` without synchronising (fused modes; the
 * epoch mode synchronises once per epoch); mb_runner_result waits and copies the statistics back. */
typedef struct mb_runner_s* mb_runner;
mb_status mb_runner_create(mb_module mod, const mb_run_config* cfg, mb_runner* out);
mb_status mb_runner_launch(mb_runner r, void* stream);
mb_status mb_runner_result(mb_runner r, void* stream, mb_result* out);
/* number of engine kernels the last mb_runner_launch enqueued */
mb_status mb_runner_kernel_launches(mb_runner r, unsigned* n);
mb_status mb_runner_free(mb_runner r);

/* ------------------------------------------------------------------ batched variants, gradients */
/* Many parameter variants of one or more networks (of different sizes) in one persistent launch.
 * No counterpart in the reference, which bakes $variables into the generated code and needs one
 * process and one compilation per variant (src/parser/expressions.cpp:211-214). Networks must have
 * rates of the form `rate_up = @logic ? U : 0; rate_down = @logic ? 0 : D` (U, D expressions of
 * $variables), at most 2048 nodes, at most 12 logic inputs per node. Variants take exact float
 * variable values (no 6-digit rounding) and run the fast-mode algorithm; a variant without
 * overrides equals MB_MODE_FUSED_FAST of the same model bit for bit. Trajectory i of a variant uses
 * random stream first_traj + i of `seed`: variants with equal first_traj share random numbers. */
typedef struct mb_batch_s* mb_batch;
mb_status mb_batch_create(mb_context c, mb_batch* out);
mb_status mb_batch_free(mb_batch b);
mb_status mb_batch_add_model(mb_batch b, mb_model m, int* net);
mb_status mb_batch_add_variant(mb_batch b, int net, const char* const* names, const float* values, int n_values,
                               long long n_traj, unsigned long long first_traj, int* variant);
mb_status mb_batch_run(mb_batch b, unsigned long long seed, float* kernel_ms);
/* a copy of variant `v`'s statistics after mb_batch_run */
mb_status mb_batch_result(mb_batch b, int v, mb_result* out);
/* Run options (both on by default). use_graph: the first run of a batch captures everything a run
 * does on the device (clearing the accumulators, the persistent kernel, the compaction of every
 * variant's fixed points, the copies of every statistic into pinned host memory) as one CUDA graph,
 * and later runs replay it with the new seed. autotune: before that capture, the launch shape
 * (threads per block, resident blocks per SM) is chosen by timing candidates on the batch itself.
 * Changing the batch (add_model / add_variant) drops the graph and the chosen shape. */
mb_status mb_batch_set_options(mb_batch b, int use_graph, int autotune);
/* A batch of one network runs by default kernels compiled for that network (NVRTC on its first run:
 * the network's sizes and tables are compile-time, the variants' rates and derivatives stay runtime,
 * so mb_batch_set_variables needs no recompilation); on = 0 selects the ahead-of-time kernels that
 * take any set of networks. Both give the same results. No counterpart in the reference (it has no
 * batched runs). */
mb_status mb_batch_set_specialize(mb_batch b, int on);
/* The launch shape of the last run, the node count of its graph (0 without one) and the number of
 * launch shapes timed by the autotuner so far. */
mb_status mb_batch_info(mb_batch b, int* block, int* blocks_per_sm, unsigned* grid, unsigned* graph_nodes,
                        int* tuned_shapes);
/* Shape `i` of the autotuner's timings: gradient run or not, threads per block, blocks per SM, kernel ms. */
mb_status mb_batch_tuning(mb_batch b, int i, int* gradient, int* block, int* blocks_per_sm, float* kernel_ms);
/* Gradients on a batch (the engine of mb_gradient kept across calls: buffers, launch shapes and
 * graphs are reused). mb_batch_add_variant_grad adds a variant like mb_batch_add_variant whose
 * gradient with respect to the $variables grad_params is computed by mb_batch_run_gradient.
 * mb_batch_set_variables gives variant v new values of some of its $variables in place (its rate
 * tables are recomputed and uploaded; prepared runs stay valid). mb_batch_run_gradient runs the
 * batch once with cotangents (cotangents[v]: variant v's [windows * 2^k] array, NULL for zeros;
 * n_cotangents = the number of variants): forward statistics (mb_batch_result) and, per variant,
 * the vector-Jacobian product that mb_batch_gradient copies out (n_grad = its length, at most cap
 * values written). Same estimator, trajectories and scaling as mb_gradient. */
mb_status mb_batch_add_variant_grad(mb_batch b, int net, const char* const* names, const float* values,
                                    int n_values, long long n_traj, unsigned long long first_traj,
                                    const char* const* grad_params, int n_grad, int* variant);
/* Mutant analysis (a TODO of the reference, README.md "Next steps"; no counterpart in its code): a
 * variant of network `net` in which each listed node is forced on (on[i] != 0) or off: its initial
 * state is 1 or 0 and both of its rates are 0, so it never changes; the other nodes evolve as in the
 * model (with the given $variable values). All single-node mutants of a network run in one launch.
 * Equal, bit for bit, to MB_MODE_FUSED_FAST of the model with those nodes' rates and istate edited. */
mb_status mb_batch_add_mutant(mb_batch b, int net, const char* const* names, const float* values, int n_values,
                              long long n_traj, unsigned long long first_traj, const char* const* nodes,
                              const int* on, int n_mutants, int* variant);
mb_status mb_batch_set_variables(mb_batch b, int v, const char* const* names, const float* values, int n_values);
mb_status mb_batch_run_gradient(mb_batch b, unsigned long long seed, const double* const* cotangents,
                                int n_cotangents, float* kernel_ms);
mb_status mb_batch_gradient(mb_batch b, int v, double* grad, int cap, int* n_grad);

/* Score-function (likelihood-ratio) gradient of L = sum_{w,s} cotangent[w * 2^k + s] * P_w(s) with
 * respect to the $variables `params` (set to `values`), P_w(s) the window probabilities of
 * n_traj trajectories (fast-mode algorithm, seed `seed`, streams 0..n_traj-1): grad[p] = dL/dparam_p,
 * estimated on the same trajectories as the forward statistics written to *forward (optional).
 * Continuous time: causal score sum_{jumps <= t} dlog a_j - int_0^t d a_0 weighted by the
 * occupancy; discrete time: step score sum (dlog a_j - d a_0 / a_0). No counterpart in the reference. */
mb_status mb_gradient(mb_context c, mb_model m, const char* const* params, const float* values, int n_params,
                      long long n_traj, unsigned long long seed, const double* cotangent, double* grad,
                      mb_result* forward);

/* ------------------------------------------------------------------ results */
mb_status mb_result_free(mb_result r);
/* dims: windows, bins (2^k; 0 for a sparse result), non-internal count k, state words W, node count N.
 * With 21 to 112 non-internal nodes (the reference's limit is 20, src/main.cpp:142-146) the result
 * is sparse: window probabilities and final states exist only for the states that occurred, through
 * mb_result_sparse_*; the dense getters (window probabilities, raw window sums, final counts) fail. */
mb_status mb_result_dims(mb_result r, int* windows, int* bins, int* noninternal, int* state_words, int* nodes);
mb_status mb_result_transitions(mb_result r, unsigned long long* transitions);
/* Trajectory count, time constants and non-internal node indices ([k], may be NULL) of a result. */
mb_status mb_result_info(mb_result r, long long* n_trajectories, int* discrete_time, float* time_tick,
                         float* max_time, int* noninternal_nodes);
/* kernel_ms: simulation + statistics kernels; total_ms: the whole run on the device */
mb_status mb_result_timing(mb_result r, float* kernel_ms, float* total_ms, int* epochs);
/* Window probabilities [windows * bins] (window_average_small.cpp:126-140) and TH [windows]. */
mb_status mb_result_window_probs(mb_result r, double* probs);
mb_status mb_result_window_entropy(mb_result r, double* th);
/* Raw accumulators: continuous occupancy in fixed point (value * 2^exponent) or discrete counts. */
mb_status mb_result_window_raw(mb_result r, long long* occupancy, unsigned* counts, long long* entropy,
                               int* occupancy_exponent, int* entropy_exponent);
mb_status mb_result_final_counts(mb_result r, unsigned* counts);
/* 1 when the result's windows are stored as sparse entries: more than 20 non-internal nodes, or a
 * dense histogram of at least 2^24 cells (windows x 2^k) of which at most a quarter are non-zero (only
 * those cells are copied from the device; final states stay dense). The sparse getters then give the
 * entries; the dense getters still work for the latter (they write zeros and scatter the entries).
 * No counterpart in the reference (its window_average_small_stats::finalize copies the whole
 * histogram, window_average_small.cpp:91-108). */
mb_status mb_result_windows_sparse(mb_result r, int* sparse);
/* Sparse results: entry counts and the number of bin additions lost to a full table (0 means exact). */
mb_status mb_result_sparse_size(mb_result r, long long* window_entries, long long* final_entries,
                                unsigned* bin_overflow);
/* Window entries sorted by window then non-internal index (bit i = i-th non-internal node, at most 112
 * nodes, two uint64 per index: bits 0-63, then 64-127): raw sums (fixed point as in
 * mb_result_window_raw) and probabilities; any output may be NULL. Final states: the same indices. */
mb_status mb_result_sparse_windows(mb_result r, int* windows, uint64_t* states, long long* raw, double* probs);
mb_status mb_result_sparse_final(mb_result r, uint64_t* states, unsigned* counts);
mb_status mb_result_num_fixed(mb_result r, int* n, unsigned* overflow);
mb_status mb_result_fixed(mb_result r, int i, uint32_t* state_words, unsigned* count);

/* Output writers: <prefix>_probtraj.csv (window_average_small.cpp:181-250) and <prefix>_fp.csv
 * (fixed_states.cu:154-187); visualize() text of all three plugins (stdout format of
 * src/main.cpp:85-99). Node names come from the model. */
mb_status mb_result_write_csv(mb_result r, mb_model m, const char* prefix);
/* Opt-in, no counterpart in the reference (final_states_stats::write_csv writes nothing,
 * src/statistics/final_states.cpp:70): the final-state distribution to <prefix>_finalprob.csv in the
 * MB_FORMAT_CSV_FINAL_STATES layout. */
mb_status mb_result_write_final_csv(mb_result r, mb_model m, const char* prefix);
mb_status mb_result_visualize(mb_result r, mb_model m, char* buf, size_t cap, size_t* len);
/* A result from raw accumulators (for instance the per-rank sums of a sharded run after a
 * collective). Window sums are fixed point: occupancy = time * 2^occupancy_exponent (continuous),
 * entropy = sum of h * slice * 2^entropy_exponent (discrete: h * 2^entropy_exponent); the exponents
 * are those mb_result_window_raw reports. Fixed points may come in any order and with repeats (their
 * counts are summed). */
typedef struct mb_result_desc_s
{
    int n_nodes;
    int n_windows;
    int discrete_time;
    float time_tick;
    float max_time;
    const int* noninternal_nodes;  /* increasing node indices, at most 20 */
    int n_noninternal;
    long long n_trajectories;
    int occupancy_exponent;
    int entropy_exponent;
    const long long* occupancy;    /* continuous: [n_windows * 2^k] */
    const unsigned* counts;        /* discrete:   [n_windows * 2^k] */
    const long long* entropy;      /* [n_windows] */
    const unsigned* final_counts;  /* [2^k] */
    int n_fixed;
    const uint32_t* fixed_states;  /* [n_fixed * ceil(n_nodes / 32)] */
    const unsigned* fixed_counts;  /* [n_fixed] */
    unsigned long long transitions;
} mb_result_desc;
mb_status mb_result_create(const mb_result_desc* desc, mb_result* out);
/* The statistics of the union of disjoint trajectory sets: the shards of one job, run with the
 * same mb_run_config.stats_trajectories (the reference has one process per job; its final sum
 * over shards would be simulation_runner's accumulation across batches). Integer sums, so the
 * merge of shards [0, a) and [a, n) equals one run of [0, n) bit for bit. */
mb_status mb_result_merge(const mb_result* parts, int n_parts, mb_result* out);

/* One plugin's output with caller-given node names (stats::visualize / stats::write_csv of
 * src/statistics/stats.h:26-27): section MB_SECTION_FINAL (visualize: "final points:"; csv: empty,
 * as final_states.cpp:70 writes no file), MB_SECTION_FIXED (fixed_states.cu:127-187) or
 * MB_SECTION_WINDOWS (window_average_small.cpp:142-250). */
#define MB_SECTION_FINAL 0
#define MB_SECTION_FIXED 1
#define MB_SECTION_WINDOWS 2
#define MB_FORMAT_VISUALIZE 0
#define MB_FORMAT_CSV 1
/* Opt-in, no counterpart in the reference: MB_SECTION_FINAL as a CSV file ("Final States (n)",
 * "Proba<TAB>State", one line per final state in non-internal index order); other sections as
 * MB_FORMAT_CSV. */
#define MB_FORMAT_CSV_FINAL_STATES 2
mb_status mb_result_format(mb_result r, int section, int format, const char* const* node_names, int n_names,
                           char* buf, size_t cap, size_t* len);

#ifdef __cplusplus
}
#endif

#endif /* MABOSS_B200_H */
