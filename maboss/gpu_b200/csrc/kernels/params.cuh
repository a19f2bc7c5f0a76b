// Kernel parameter blocks shared by the host runtime and the NVRTC-compiled engine.
// Plain-old-data only: the host passes these structs by value through cuLaunchKernel.
#pragma once

struct __align__(16) mb_key128
{
	unsigned long long lo, hi;
};

// Statistics sinks shared by all kernels.
struct mb_stats_params
{
	int n_windows;		  // T = ceil(max_time / tick)
	unsigned n_bins;	  // S = 2^k
	float win_tick;		  // window size (exact host float, window_average_small.cpp:305)
	int h_in_smem;		  // transition-entropy sums privatised per block in shared memory
	double fx;			  // occupancy scale 2^e
	double fx_h;		  // transition-entropy scale 2^eh
	long long* win_occ;	  // [T*S] continuous occupancy (fixed point)
	unsigned* win_cnt;	  // [T*S] discrete counts
	long long* win_h;	  // [T] transition-entropy sums (fixed point)
	unsigned* final_cnt;  // [S]
	mb_key128* fp_keys;	  // [cap] fixed-point hash keys (0 = empty)
	unsigned* fp_counts;  // [cap]
	unsigned* fp_states;  // [cap * W]
	unsigned fp_mask;	  // cap - 1 (cap is a power of two)
	unsigned* fp_overflow;
	// more than 20 non-internal nodes: window sums (continuous occupancy or discrete counts) and, at
	// window T, final-state counts in a hash table keyed by (window + 1, 64-bit non-internal index)
	mb_key128* bin_keys;  // [cap] ({0, 0} = empty)
	long long* bin_vals;  // [cap]
	unsigned bin_mask;	  // cap - 1
	unsigned* bin_overflow;
};

struct mb_fused_params
{
	mb_stats_params st;
	const float* istate;			 // [N] initial probabilities
	unsigned long long seed;		 // seed_pseudorandom
	unsigned long long first_traj;	 // global id of trajectory 0 of this launch (RNG subsequence)
	unsigned n_traj;				 // trajectories of this launch
	int traj_len;					 // epoch length L emulated in exact mode (0 = none)
	unsigned long long* next_traj;	 // work counter (zeroed by the host)
	unsigned long long* transitions; // executed simulate iterations
	unsigned* errors;				 // trajectories stopped because the total rate was not finite
	void* rands;					 // exact mode: curandState of trajectory t at [t], initialised by a
									 // separate mb_initialize_random launch, or null (curand_init inline)
};
