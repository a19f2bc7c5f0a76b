// Fixed-point statistics without any device allocation.
//
// mb_fixed_states_noalloc collects the distinct fixed-point states of a batch of trajectories and
// how many trajectories ended in each, like mb_launch_fixed_states_stats + mb_stats_finalize, but
// its hash table lives in one static device array of this library instead of memory the engine
// allocates. It is meant for callers that must not allocate device memory themselves or through
// us: code running under a caching allocator that owns every byte of the device (a framework's
// memory pool), processes with a fixed memory budget, or sections where cudaMalloc would
// synchronise the device. The caller passes device inputs and device outputs; nothing else is
// allocated. Compiled ahead of time with nvcc for sm_100a; it does not depend on the model, only on
// the number of state words.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "maboss_b200.h"

namespace {

// Scratch capacity: the whole table (keys, counts, states, counters) must fit in this many bytes.
constexpr size_t MB_NOALLOC_SCRATCH_BYTES = 8u << 20; // 8 MiB
constexpr int MB_NOALLOC_MAX_WORDS = 64;			  // states of up to 2048 nodes

// The table. Every GPU that loads this library holds these 8 MiB until the process exits.
static __device__ __align__(256) unsigned char mb_noalloc_scratch[MB_NOALLOC_SCRATCH_BYTES];

struct __align__(16) key128
{
	unsigned long long lo, hi;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
	x ^= x >> 30;
	x *= 0xbf58476d1ce4e5b9ull;
	x ^= x >> 27;
	x *= 0x94d049bb133111ebull;
	x ^= x >> 31;
	return x;
}

// layout of the scratch for `cap` slots of `words` state words
struct table
{
	key128* keys;
	unsigned* counts;
	unsigned* states;
	unsigned* counters; // [0] overflow, [1] records written
	unsigned mask;
};

__host__ __device__ inline size_t table_bytes(unsigned cap, int words)
{
	return (size_t)cap * (sizeof(key128) + sizeof(unsigned) + sizeof(unsigned) * words) + 256;
}

__device__ table make_table(unsigned char* base, unsigned cap, int words)
{
	table t;
	t.keys = reinterpret_cast<key128*>(base);
	t.counts = reinterpret_cast<unsigned*>(base + (size_t)cap * sizeof(key128));
	t.states = t.counts + cap;
	t.counters = t.states + (size_t)cap * words;
	t.mask = cap - 1;
	return t;
}

// 128-bit key: the state itself for up to 3 words, else two independent 64-bit hashes; the top
// bit is set so that an all-zero key marks an empty slot.
__device__ key128 state_key(const unsigned* st, int words)
{
	key128 k;
	if (words <= 3)
	{
		k.lo = (unsigned long long)st[0] | (words > 1 ? (unsigned long long)st[1] << 32 : 0ull);
		k.hi = (words > 2 ? (unsigned long long)st[2] : 0ull) | (1ull << 63);
		return k;
	}
	unsigned long long a = 0x243f6a8885a308d3ull, b = 0x13198a2e03707344ull;
	for (int w = 0; w < words; w++)
	{
		a = mix64(a ^ ((unsigned long long)st[w] + 0x9e3779b97f4a7c15ull * (w + 1)));
		b = mix64(b + ((unsigned long long)st[w] ^ (0xc2b2ae3d27d4eb4full * (w + 7))));
	}
	k.lo = a;
	k.hi = b | (1ull << 63);
	return k;
}

__global__ void clear_table(unsigned char* base, unsigned cap, int words)
{
	const table t = make_table(base, cap, words);
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < cap)
	{
		t.keys[i].lo = 0;
		t.keys[i].hi = 0;
		t.counts[i] = 0;
	}
	if (i < 2)
		t.counters[i] = 0;
}

// one thread per trajectory: FIXED_POINT states go into the table (bounded linear probing)
__global__ void insert_fixed(unsigned char* base, unsigned cap, int words, int n, int stride,
							 const uint32_t* __restrict__ last_states, const uint8_t* __restrict__ statuses)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || statuses[i] != MB_STATUS_FIXED_POINT)
		return;
	const table t = make_table(base, cap, words);
	unsigned st[MB_NOALLOC_MAX_WORDS];
	for (int w = 0; w < words; w++)
		st[w] = last_states[(size_t)w * stride + i];
	const key128 key = state_key(st, words);
	const unsigned h = (unsigned)mix64(key.lo ^ mix64(key.hi));
	key128 empty;
	empty.lo = 0;
	empty.hi = 0;
	for (unsigned probe = 0; probe <= t.mask; probe++)
	{
		const unsigned slot = (h + probe) & t.mask;
		const key128 prev = atomicCAS(t.keys + slot, empty, key);
		if (prev.lo == 0ull && prev.hi == 0ull)
		{
			for (int w = 0; w < words; w++)
				t.states[(size_t)slot * words + w] = st[w];
			atomicAdd(t.counts + slot, 1u);
			return;
		}
		if (prev.lo == key.lo && prev.hi == key.hi)
		{
			atomicAdd(t.counts + slot, 1u);
			return;
		}
	}
	atomicAdd(t.counters, 1u); // table full
}

// compact the occupied slots into the caller's arrays (records beyond out_cap are only counted)
__global__ void extract_fixed(unsigned char* base, unsigned cap, int words, uint32_t* __restrict__ out_states,
							  unsigned* __restrict__ out_counts, int out_cap)
{
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= cap)
		return;
	const table t = make_table(base, cap, words);
	const key128 k = t.keys[i];
	if (k.lo == 0ull && k.hi == 0ull)
		return;
	// wait-free: every occupied slot takes one output position
	const unsigned o = atomicAdd(t.counters + 1, 1u);
	if ((int)o >= out_cap)
		return;
	for (int w = 0; w < words; w++)
		out_states[(size_t)o * words + w] = t.states[(size_t)i * words + w];
	out_counts[o] = t.counts[i];
}


// Driver-API functions resolved through the runtime (this library does not link libcuda).
typedef int (*ctx_get_current_fn)(void** ctx);
typedef int (*ctx_get_id_fn)(void* ctx, unsigned long long* id);

template <typename F>
F driver_function(const char* name)
{
	void* p = nullptr;
	cudaDriverEntryPointQueryResult q;
	if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess
		|| q != cudaDriverEntryPointSuccess)
		return nullptr;
	return reinterpret_cast<F>(p);
}

// Device address of the scratch array in the current context. It is looked up with
// cudaGetSymbolAddress the first time a device is used and again whenever that device's current
// context has changed (cuCtxGetId gives every context of the process its own id, so a context
// created after cudaDeviceReset or a primary-context reset is never served the old address).
void* scratch_address(int device, cudaError_t& err)
{
	static std::mutex mu;
	static void* addr[256] = { nullptr };
	static unsigned long long ctx_id[256] = { 0 };
	static ctx_get_current_fn get_current = driver_function<ctx_get_current_fn>("cuCtxGetCurrent");
	static ctx_get_id_fn get_id = driver_function<ctx_get_id_fn>("cuCtxGetId");
	std::lock_guard<std::mutex> lk(mu);
	err = cudaSuccess;
	if (device < 0 || device >= 256)
	{
		err = cudaErrorInvalidDevice;
		return nullptr;
	}
	// before the runtime has bound a context to this thread there is no current context: id 0,
	// and cudaGetSymbolAddress (which binds the device's primary context) runs again next time
	unsigned long long id = 0;
	void* ctx = nullptr;
	if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0)
		id = 0; // no id available: look the address up on every call
	if (!addr[device] || id == 0 || id != ctx_id[device])
	{
		void* p = nullptr;
		err = cudaGetSymbolAddress(&p, mb_noalloc_scratch);
		if (err != cudaSuccess)
			return nullptr;
		addr[device] = p;
		ctx_id[device] = id;
	}
	return addr[device];
}

unsigned table_capacity(int state_words)
{
	unsigned cap = 1u << 30;
	while (cap > 1 && table_bytes(cap, state_words) > MB_NOALLOC_SCRATCH_BYTES)
		cap >>= 1;
	return cap;
}

} // namespace

namespace mb {
void set_last_error(const std::string& message); // api.cpp: the message mb_last_error() returns
}

namespace {

mb_status fail(mb_status s, const std::string& msg)
{
	mb::set_last_error(msg);
	return s;
}

} // namespace

extern "C" {

mb_status mb_fixed_states_noalloc(void* stream, int n, int stride, int state_words, const uint32_t* last_states,
								  const uint8_t* statuses, uint32_t* out_states, unsigned* out_counts, int out_cap,
								  int* out_n)
{
	mb::set_last_error("");
	if (n < 0 || stride < n || out_cap < 0 || !out_n)
		return fail(MB_ERR_INVALID, "mb_fixed_states_noalloc: bad n, stride, out_cap or out_n");
	if (state_words < 1 || state_words > MB_NOALLOC_MAX_WORDS)
		return fail(MB_ERR_LIMIT, "mb_fixed_states_noalloc: state_words must be in [1, " +
									  std::to_string(MB_NOALLOC_MAX_WORDS) + "] (networks of up to " +
									  std::to_string(32 * MB_NOALLOC_MAX_WORDS) + " nodes)");
	if (n > 0 && (!last_states || !statuses))
		return fail(MB_ERR_INVALID, "mb_fixed_states_noalloc: null input buffer");
	if (out_cap > 0 && (!out_states || !out_counts))
		return fail(MB_ERR_INVALID, "mb_fixed_states_noalloc: null output buffer");
	int device = 0;
	cudaError_t e = cudaGetDevice(&device);
	if (e != cudaSuccess)
		return fail(MB_ERR_CUDA, std::string("mb_fixed_states_noalloc: ") + cudaGetErrorString(e));
	unsigned char* base = static_cast<unsigned char*>(scratch_address(device, e));
	if (!base)
		return fail(MB_ERR_CUDA, std::string("mb_fixed_states_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
	const unsigned cap = table_capacity(state_words);
	cudaStream_t s = static_cast<cudaStream_t>(stream);

	// the array keeps the previous call's table: clear it first
	// grid sizes in size_t: n may be close to INT_MAX
	const unsigned table_blocks = (unsigned)(((size_t)cap + 255) / 256);
	clear_table<<<table_blocks, 256, 0, s>>>(base, cap, state_words);
	if (n > 0)
		insert_fixed<<<(unsigned)(((size_t)n + 255) / 256), 256, 0, s>>>(base, cap, state_words, n, stride,
																		 last_states, statuses);
	extract_fixed<<<table_blocks, 256, 0, s>>>(base, cap, state_words, out_states, out_counts, out_cap);
	e = cudaGetLastError();
	if (e != cudaSuccess)
		return fail(MB_ERR_CUDA, std::string("mb_fixed_states_noalloc: launch: ") + cudaGetErrorString(e));

	// counters back to the host (a copy into host stack memory, no allocation)
	const size_t counters_offset = (size_t)cap * (sizeof(key128) + sizeof(unsigned) + sizeof(unsigned) * state_words);
	unsigned counters[2] = { 0, 0 };
	e = cudaMemcpyAsync(counters, base + counters_offset, sizeof counters, cudaMemcpyDeviceToHost, s);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(s);
	if (e != cudaSuccess)
		return fail(MB_ERR_CUDA, std::string("mb_fixed_states_noalloc: ") + cudaGetErrorString(e));
	if (counters[0] != 0 || counters[1] > cap / 2)
	{
		// the table overflowed: the number of distinct fixed points is unknown
		*out_n = -1;
		return fail(MB_ERR_LIMIT, "mb_fixed_states_noalloc: more distinct fixed points than the static table holds (" +
									  std::to_string(cap / 2) + " for " + std::to_string(state_words) + " state words)");
	}
	*out_n = (int)counters[1];
	if ((int)counters[1] > out_cap)
		return fail(MB_ERR_LIMIT, "mb_fixed_states_noalloc: " + std::to_string(counters[1]) +
									  " distinct fixed points do not fit in out_cap = " + std::to_string(out_cap));
	return MB_OK;
}

} // extern "C"
