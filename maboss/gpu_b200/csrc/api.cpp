// C ABI (include/maboss_b200.h) over the C++ runtime. Every entry point catches exceptions
// and turns them into status codes with a thread-local message.
#include "maboss_b200.h"

#include <curand_kernel.h>

#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <thread>

#include "batch.h"
#include "codegen.h"
#include "model.h"
#include "output.h"
#include "runtime.h"
#include "sparse_bins.h"

struct mb_model_s
{
	mb::model_t model;
};
struct mb_context_s
{
	std::unique_ptr<mb::context> ctx;
};
struct mb_module_s
{
	std::unique_ptr<mb::module> mod;
	mb_context ctx = nullptr;
};
struct mb_result_s
{
	std::unique_ptr<mb::result> res;
};
struct mb_stats_s
{
	mb::stats_state st;
};
struct mb_runner_s
{
	std::unique_ptr<mb::runner> rn;
};
struct mb_batch_s
{
	std::unique_ptr<mb::batch_engine> b;
	bool ran = false;
};

namespace {

thread_local std::string g_last_error;

template <typename F>
mb_status guard(F&& f)
{
	try
	{
		g_last_error.clear();
		f();
		return MB_OK;
	}
	catch (const mb::engine_error& e)
	{
		g_last_error = e.what();
		return e.code;
	}
	catch (const mb::model_error& e)
	{
		g_last_error = e.what();
		return MB_ERR_PARSE;
	}
	catch (const std::bad_alloc&)
	{
		g_last_error = "out of host memory";
		return MB_ERR_LIMIT;
	}
	catch (const std::exception& e)
	{
		g_last_error = e.what();
		return MB_ERR_INTERNAL;
	}
	catch (...)
	{
		g_last_error = "unknown error";
		return MB_ERR_INTERNAL;
	}
}

void need(bool cond, const char* msg)
{
	if (!cond)
		throw mb::engine_error(MB_ERR_INVALID, msg);
}

void copy_out(const std::string& s, char* buf, size_t cap, size_t* len)
{
	if (len)
		*len = s.size();
	if (buf && cap)
	{
		size_t n = std::min(cap - 1, s.size());
		std::memcpy(buf, s.data(), n);
		buf[n] = '\0';
	}
}

cudaStream_t stream_of(mb::context* ctx, void* s) { return s ? (cudaStream_t)s : ctx->stream; }

std::vector<std::string> names_of(const mb::model_t& m)
{
	std::vector<std::string> n;
	for (auto& x : m.nodes)
		n.push_back(x.name);
	return n;
}

} // namespace

namespace mb {
// lets entry points outside this file report through mb_last_error()
void set_last_error(const std::string& message) { g_last_error = message; }
} // namespace mb

extern "C" {

const char* mb_version(void) { return "maboss_b200 0.1 (sm_100a)"; }
const char* mb_last_error(void) { return g_last_error.c_str(); }

// ------------------------------------------------------------------ models

mb_status mb_model_parse_files(const char* bnd_path, const char* cfg_path, mb_model* out)
{
	return guard([&] {
		need(bnd_path && cfg_path && out, "null argument");
		auto m = std::make_unique<mb_model_s>();
		mb::parse_model_files(m->model, bnd_path, cfg_path);
		*out = m.release();
	});
}

mb_status mb_model_parse_text(const char* bnd_text, const char* cfg_text, mb_model* out)
{
	return guard([&] {
		need(bnd_text && cfg_text && out, "null argument");
		auto m = std::make_unique<mb_model_s>();
		mb::parse_bnd(m->model, bnd_text, "<bnd>");
		mb::parse_cfg(m->model, cfg_text, "<cfg>");
		*out = m.release();
	});
}

mb_status mb_model_free(mb_model m)
{
	delete m;
	return MB_OK;
}

mb_status mb_model_num_nodes(mb_model m, int* n)
{
	return guard([&] {
		need(m && n, "null argument");
		*n = (int)m->model.nodes.size();
	});
}

mb_status mb_model_node_name(mb_model m, int i, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(m && i >= 0 && i < (int)m->model.nodes.size(), "bad node index");
		copy_out(m->model.nodes[i].name, buf, cap, len);
	});
}

mb_status mb_model_node_info(mb_model m, int i, float* istate, int* is_internal)
{
	return guard([&] {
		need(m && i >= 0 && i < (int)m->model.nodes.size(), "bad node index");
		if (istate)
			*istate = m->model.nodes[i].istate;
		if (is_internal)
			*is_internal = m->model.is_internal(i) ? 1 : 0;
	});
}

mb_status mb_model_set_istate(mb_model m, int i, float istate)
{
	return guard([&] {
		need(m && i >= 0 && i < (int)m->model.nodes.size(), "bad node index");
		m->model.nodes[i].istate = istate;
	});
}

mb_status mb_model_apply_cfg_overrides(mb_model m)
{
	return guard([&] {
		need(m, "null model");
		mb::apply_cfg_overrides(m->model);
	});
}

mb_status mb_model_get_constant(mb_model m, const char* name, float* value)
{
	return guard([&] {
		need(m && name && value, "null argument");
		*value = m->model.constant(name);
	});
}

mb_status mb_model_set_constant(mb_model m, const char* name, float value)
{
	return guard([&] {
		need(m && name, "null argument");
		m->model.constants[name] = value;
	});
}

mb_status mb_model_get_variable(mb_model m, const char* name, float* value)
{
	return guard([&] {
		need(m && name && value, "null argument");
		auto it = m->model.variables.find(name);
		if (it == m->model.variables.end())
			throw mb::engine_error(MB_ERR_INVALID, std::string("unknown variable ") + name);
		*value = it->second;
	});
}

mb_status mb_model_set_variable(mb_model m, const char* name, float value)
{
	return guard([&] {
		need(m && name && name[0] == '$', "variable names start with '$'");
		m->model.variables[name] = value;
	});
}

mb_status mb_model_num_variables(mb_model m, int* n)
{
	return guard([&] {
		need(m && n, "null argument");
		*n = (int)m->model.variables.size();
	});
}

mb_status mb_model_variable_name(mb_model m, int i, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(m && i >= 0 && i < (int)m->model.variables.size(), "bad variable index");
		auto it = m->model.variables.begin();
		std::advance(it, i);
		copy_out(it->first, buf, cap, len);
	});
}

mb_status mb_model_num_constants(mb_model m, int* n)
{
	return guard([&] {
		need(m && n, "null argument");
		*n = (int)m->model.constants.size();
	});
}

mb_status mb_model_constant_name(mb_model m, int i, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(m && i >= 0 && i < (int)m->model.constants.size(), "bad constant index");
		auto it = m->model.constants.begin();
		std::advance(it, i);
		copy_out(it->first, buf, cap, len);
	});
}

mb_status mb_model_generate_code(mb_model m, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(m, "null model");
		copy_out(mb::generate_code(m->model), buf, cap, len);
	});
}

// ------------------------------------------------------------------ context / modules

mb_status mb_context_create(int device, mb_context* out)
{
	return guard([&] {
		need(out, "null argument");
		auto c = std::make_unique<mb_context_s>();
		c->ctx = std::make_unique<mb::context>(device);
		*out = c.release();
	});
}

mb_status mb_context_free(mb_context c)
{
	delete c;
	return MB_OK;
}

mb_status mb_context_stream(mb_context c, void** stream)
{
	return guard([&] {
		need(c && stream, "null argument");
		*stream = (void*)c->ctx->stream;
	});
}

mb_status mb_context_sm_count(mb_context c, int* sm_count)
{
	return guard([&] {
		need(c && sm_count, "null argument");
		*sm_count = c->ctx->sm_count;
	});
}

mb_status mb_module_compile(mb_context c, const char* code, mb_module* out)
{
	return guard([&] {
		need(c && code && out, "null argument");
		auto m = std::make_unique<mb_module_s>();
		m->ctx = c;
		m->mod = mb::compile_module(*c->ctx, code);
		*out = m.release();
	});
}

mb_status mb_module_compile_model(mb_context c, mb_model model, mb_module* out)
{
	return guard([&] {
		need(c && model && out, "null argument");
		auto m = std::make_unique<mb_module_s>();
		m->ctx = c;
		mb::model_layout L = mb::analyze_model(model->model);
		m->mod = mb::compile_module(*c->ctx, mb::generate_code(model->model));
		m->mod->layout = std::move(L);
		m->mod->has_layout = true;
		*out = m.release();
	});
}

mb_status mb_jit_check(const char* generated_code, size_t* cubin_size, char* log, size_t cap)
{
	return guard([&] {
		need(generated_code, "null code");
		std::string all;
		size_t total = 0;
		for (int f = 0; f < mb::FAMILY_COUNT; f++)
		{
			std::string lg;
			total += mb::compile_cubin(generated_code, lg, f).size();
			all += lg;
		}
		if (cubin_size)
			*cubin_size = total;
		copy_out(all, log, cap, nullptr);
	});
}

mb_status mb_module_free(mb_module mod)
{
	delete mod;
	return MB_OK;
}

mb_status mb_module_state_size(mb_module mod, int* state_size, int* state_words)
{
	return guard([&] {
		need(mod, "null module");
		if (state_size)
			*state_size = mod->mod->state_size;
		if (state_words)
			*state_words = mod->mod->state_words;
	});
}

mb_status mb_module_log(mb_module mod, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(mod, "null module");
		copy_out(mod->mod->log, buf, cap, len);
	});
}

mb_status mb_module_context(mb_module mod, mb_context* out)
{
	return guard([&] {
		need(mod && out, "null argument");
		*out = mod->ctx;
	});
}

mb_status mb_device_malloc(mb_context c, size_t bytes, void** ptr)
{
	return guard([&] {
		need(c && ptr, "null argument");
		MB_CUDA(cudaSetDevice(c->ctx->device));
		*ptr = nullptr;
		if (bytes == 0)
			return;
		const cudaError_t e = cudaMalloc(ptr, bytes);
		if (e == cudaErrorMemoryAllocation)
		{
			cudaGetLastError();
			throw mb::engine_error(MB_ERR_LIMIT, "out of device memory (" + std::to_string(bytes) + " bytes)");
		}
		MB_CUDA(e);
	});
}

mb_status mb_device_free(mb_context c, void* ptr)
{
	return guard([&] {
		need(c, "null context");
		if (!ptr)
			return;
		MB_CUDA(cudaSetDevice(c->ctx->device));
		MB_CUDA(cudaFree(ptr));
	});
}

mb_status mb_memcpy(mb_context c, void* stream, void* dst, const void* src, size_t bytes)
{
	return guard([&] {
		need(c && (bytes == 0 || (dst && src)), "null argument");
		if (bytes == 0)
			return;
		MB_CUDA(cudaSetDevice(c->ctx->device));
		cudaStream_t s = stream_of(c->ctx.get(), stream);
		MB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
		MB_CUDA(cudaStreamSynchronize(s));
	});
}

mb_status mb_memset_async(mb_context c, void* stream, void* ptr, int value, size_t bytes)
{
	return guard([&] {
		need(c && (bytes == 0 || ptr), "null argument");
		if (bytes == 0)
			return;
		MB_CUDA(cudaSetDevice(c->ctx->device));
		MB_CUDA(cudaMemsetAsync(ptr, value, bytes, stream_of(c->ctx.get(), stream)));
	});
}

mb_status mb_synchronize(mb_context c)
{
	return guard([&] {
		need(c, "null context");
		MB_CUDA(cudaSetDevice(c->ctx->device));
		MB_CUDA(cudaDeviceSynchronize());
	});
}

// ------------------------------------------------------------------ kernel entry points

size_t mb_rand_state_size(void) { return sizeof(curandState); }

mb_status mb_launch_initialize_random(mb_module mod, void* stream, int n, unsigned long long seed,
									  unsigned long long first, void* rands)
{
	return guard([&] {
		need(mod && n >= 0 && (rands || n == 0), "bad argument");
		if (n == 0)
			return;
		mb::module& m = *mod->mod;
		MB_CUDA(cudaSetDevice(m.ctx->device));
		if (!m.init_random)
			m.ensure(mb::FAMILY_EPOCH);
		int per = mb::init_random_per(n);
		void* a[] = { &n, &seed, &first, &rands, &per };
		mb::launch(m.init_random, mb::init_random_blocks(n, per), 256, 0, stream_of(m.ctx, stream), a);
	});
}

mb_status mb_launch_initialize_initial_state(mb_module mod, void* stream, int n, int stride,
											 const float* initial_probs, uint32_t* last_states, float* last_times,
											 void* rands)
{
	return guard([&] {
		need(mod && n >= 0 && stride >= n, "bad argument");
		if (n == 0)
			return;
		need(initial_probs && last_states && last_times && rands, "null buffer");
		mb::module& m = *mod->mod;
		MB_CUDA(cudaSetDevice(m.ctx->device));
		m.ensure_any();
		void* a[] = { &n, &stride, &initial_probs, &last_states, &last_times, &rands };
		mb::launch(m.init_state, (n + 255) / 256, 256, 0, stream_of(m.ctx, stream), a);
	});
}

mb_status mb_launch_simulate(mb_module mod, void* stream, int n, int stride, int traj_len, uint32_t* last_states,
							 float* last_times, void* rands, uint32_t* traj_states, float* traj_times,
							 float* traj_entropies, uint8_t* statuses, unsigned long long* transitions)
{
	return guard([&] {
		need(mod && n >= 0 && stride >= n && traj_len >= 2, "bad argument");
		if (n == 0)
			return;
		need(last_states && last_times && rands && traj_states && traj_times && traj_entropies && statuses &&
				 transitions,
			 "null buffer");
		mb::module& m = *mod->mod;
		MB_CUDA(cudaSetDevice(m.ctx->device));
		mb::simulate_epoch(m, false, stream_of(m.ctx, stream), n, stride, traj_len, last_states, last_times, rands,
						   traj_states, traj_times, traj_entropies, statuses, transitions);
	});
}

mb_status mb_stats_create_sections(mb_module mod, float time_tick, float max_time, int discrete_time,
								   const int* noninternal_nodes, int n_noninternal, long long sample_count,
								   unsigned sections, mb_stats* out)
{
	return guard([&] {
		need(mod && out && n_noninternal >= 0 && (noninternal_nodes || n_noninternal == 0), "bad argument");
		mb::module& m = *mod->mod;
		MB_CUDA(cudaSetDevice(m.ctx->device));
		auto s = std::make_unique<mb_stats_s>();
		std::vector<int> ni(noninternal_nodes, noninternal_nodes + n_noninternal);
		s->st.init(m, time_tick, max_time, discrete_time != 0, ni, sample_count, 0, m.ctx->stream, sections);
		MB_CUDA(cudaStreamSynchronize(m.ctx->stream));
		*out = s.release();
	});
}

mb_status mb_stats_create(mb_module mod, float time_tick, float max_time, int discrete_time,
						  const int* noninternal_nodes, int n_noninternal, long long sample_count, mb_stats* out)
{
	return mb_stats_create_sections(mod, time_tick, max_time, discrete_time, noninternal_nodes, n_noninternal,
									sample_count, MB_STATS_ALL, out);
}

mb_status mb_stats_free(mb_stats st)
{
	delete st;
	return MB_OK;
}

mb_status mb_launch_window_average_stats(mb_stats st, void* stream, int n, int stride, int traj_len,
										 const uint32_t* traj_states, const float* traj_times,
										 const float* traj_entropies)
{
	return guard([&] {
		need(st && n >= 0 && stride >= n && traj_len >= 2, "bad argument");
		if (n == 0)
			return;
		need(traj_states && traj_times && traj_entropies, "null buffer");
		MB_CUDA(cudaSetDevice(st->st.mod->ctx->device));
		st->st.window_batch(stream_of(st->st.mod->ctx, stream), n, stride, traj_len, traj_states, traj_times,
							traj_entropies);
	});
}

mb_status mb_launch_final_states_stats(mb_stats st, void* stream, int n, int stride, const uint32_t* last_states,
									   const uint8_t* statuses)
{
	return guard([&] {
		need(st && n >= 0 && stride >= n, "bad argument");
		if (n == 0)
			return;
		need(last_states && statuses, "null buffer");
		MB_CUDA(cudaSetDevice(st->st.mod->ctx->device));
		st->st.final_batch(stream_of(st->st.mod->ctx, stream), n, stride, last_states, statuses);
	});
}

mb_status mb_launch_fixed_states_stats(mb_stats st, void* stream, int n, int stride, const uint32_t* last_states,
									   const uint8_t* statuses)
{
	return guard([&] {
		need(st && n >= 0 && stride >= n, "bad argument");
		if (n == 0)
			return;
		need(last_states && statuses, "null buffer");
		MB_CUDA(cudaSetDevice(st->st.mod->ctx->device));
		st->st.fixed_batch(stream_of(st->st.mod->ctx, stream), n, stride, last_states, statuses);
	});
}

mb_status mb_stats_finalize(mb_stats st, long long n_trajectories, mb_result* out)
{
	return guard([&] {
		need(st && out, "null argument");
		MB_CUDA(cudaSetDevice(st->st.mod->ctx->device));
		MB_CUDA(cudaDeviceSynchronize());
		auto r = std::make_unique<mb_result_s>();
		r->res = st->st.finalize(n_trajectories, st->st.mod->ctx->stream);
		*out = r.release();
	});
}

size_t mb_partition_scratch_size(int n) { return mb::partition_scratch_bytes(n); }

mb_status mb_launch_partition(mb_module mod, void* stream, int n, int stride, const uint8_t* statuses,
							  const uint32_t* last_states, const float* last_times, const void* rands,
							  uint32_t* out_states, float* out_times, void* out_rands, void* scratch, unsigned* kept)
{
	return guard([&] {
		need(mod && n >= 0 && stride >= n && kept && scratch, "bad argument");
		need(n == 0 || (statuses && last_states && last_times && rands && out_states && out_times && out_rands),
			 "null buffer");
		mb::module& m = *mod->mod;
		MB_CUDA(cudaSetDevice(m.ctx->device));
		mb::partition(m, stream_of(m.ctx, stream), n, stride, statuses, last_states, last_times, rands, out_states,
					  out_times, out_rands, scratch, kept);
	});
}

// ------------------------------------------------------------------ whole runs

mb_status mb_run_config_default(mb_model m, mb_run_config* cfg)
{
	return guard([&] {
		need(m && cfg, "null argument");
		mb_run_config c{};
		c.mode = MB_MODE_FUSED_EXACT;
		c.sample_count = (long long)m->model.constant("sample_count");
		c.seed = (unsigned long long)m->model.constant("seed_pseudorandom");
		c.first_traj = 0;
		c.traj_len = 100;
		c.batch_limit = 1000000;
		c.block = 256;
		c.blocks_per_sm = 0;
		c.fixed_capacity_log2 = 0;
		c.stats_trajectories = 0;
		c.bin_capacity_log2 = 0;
		c.refill_reuse_rng = 0;
		*cfg = c;
	});
}

namespace {
mb::run_config to_config(mb_module mod, const mb_run_config* cfg)
{
	need(mod->mod->has_layout, "whole runs need a module from mb_module_compile_model");
	mb::run_config c = mb::config_from_layout(mod->mod->layout, cfg->mode);
	c.sample_count = cfg->sample_count;
	c.seed = cfg->seed;
	c.first_traj = cfg->first_traj;
	c.traj_len = cfg->traj_len > 0 ? cfg->traj_len : 100;
	c.batch_limit = cfg->batch_limit > 0 ? cfg->batch_limit : 1000000;
	c.block = cfg->block > 0 ? cfg->block : 256;
	c.blocks_per_sm = cfg->blocks_per_sm;
	c.fixed_capacity_log2 = cfg->fixed_capacity_log2;
	c.stats_trajectories = cfg->stats_trajectories;
	c.bin_capacity_log2 = cfg->bin_capacity_log2;
	c.refill_reuse_rng = cfg->refill_reuse_rng != 0;
	return c;
}
} // namespace

mb_status mb_autotune(mb_module mod, mb_run_config* cfg, float* transitions_per_s, int* shapes, float* rates,
					  int cap, int* n_shapes)
{
	return guard([&] {
		need(mod && cfg, "null argument");
		const std::vector<mb::tuned_shape> t = mb::autotune(*mod->mod, to_config(mod, cfg));
		cfg->block = t.front().block;
		cfg->blocks_per_sm = t.front().blocks_per_sm;
		if (transitions_per_s)
			*transitions_per_s = (float)t.front().transitions_per_s;
		if (n_shapes)
			*n_shapes = (int)t.size();
		for (int i = 0; i < cap && i < (int)t.size(); i++)
		{
			if (shapes)
			{
				shapes[3 * i] = t[i].block;
				shapes[3 * i + 1] = t[i].blocks_per_sm;
				shapes[3 * i + 2] = 0;
			}
			if (rates)
				rates[i] = (float)t[i].transitions_per_s;
		}
	});
}

mb_status mb_runner_create(mb_module mod, const mb_run_config* cfg, mb_runner* out)
{
	return guard([&] {
		need(mod && cfg && out, "null argument");
		auto r = std::make_unique<mb_runner_s>();
		r->rn = std::make_unique<mb::runner>(*mod->mod, to_config(mod, cfg));
		*out = r.release();
	});
}

mb_status mb_runner_launch(mb_runner r, void* stream)
{
	return guard([&] {
		need(r, "null runner");
		r->rn->launch(stream_of(r->rn->mod->ctx, stream));
	});
}

mb_status mb_runner_result(mb_runner r, void* stream, mb_result* out)
{
	return guard([&] {
		need(r && out, "null argument");
		auto res = std::make_unique<mb_result_s>();
		res->res = r->rn->collect(stream_of(r->rn->mod->ctx, stream));
		*out = res.release();
	});
}

mb_status mb_runner_kernel_launches(mb_runner r, unsigned* n)
{
	return guard([&] {
		need(r && n, "null argument");
		*n = r->rn->kernel_launches();
	});
}

mb_status mb_runner_free(mb_runner r)
{
	delete r;
	return MB_OK;
}

mb_status mb_run_module(mb_module mod, const mb_run_config* cfg, const mb_run_params* params, mb_result* out)
{
	return guard([&] {
		need(mod && cfg && params && out, "null argument");
		const mb::module& m = *mod->mod;
		need(params->n_nodes == m.state_size && params->initial_probs, "one initial probability per node is needed");
		need(params->n_noninternal >= 0 && (params->noninternal_nodes || params->n_noninternal == 0),
			 "bad non-internal nodes");
		mb::run_config c;
		c.mode = cfg->mode;
		c.max_time = params->max_time;
		c.time_tick = params->time_tick;
		c.discrete_time = params->discrete_time != 0;
		c.istate.assign(params->initial_probs, params->initial_probs + params->n_nodes);
		c.noninternal_nodes.assign(params->noninternal_nodes, params->noninternal_nodes + params->n_noninternal);
		for (size_t i = 0; i < c.noninternal_nodes.size(); i++)
			need(c.noninternal_nodes[i] >= 0 && c.noninternal_nodes[i] < m.state_size &&
					 (i == 0 || c.noninternal_nodes[i] > c.noninternal_nodes[i - 1]),
				 "non-internal nodes must be increasing node indices");
		c.sample_count = cfg->sample_count;
		c.seed = cfg->seed;
		c.first_traj = cfg->first_traj;
		c.traj_len = cfg->traj_len > 0 ? cfg->traj_len : 100;
		c.batch_limit = cfg->batch_limit > 0 ? cfg->batch_limit : 1000000;
		c.block = cfg->block > 0 ? cfg->block : 256;
		c.blocks_per_sm = cfg->blocks_per_sm;
		c.fixed_capacity_log2 = cfg->fixed_capacity_log2;
		c.stats_trajectories = cfg->stats_trajectories;
		c.bin_capacity_log2 = cfg->bin_capacity_log2;
		c.refill_reuse_rng = cfg->refill_reuse_rng != 0;
		auto r = std::make_unique<mb_result_s>();
		r->res = mb::run(*mod->mod, c);
		*out = r.release();
	});
}

mb_status mb_run(mb_module mod, const mb_run_config* cfg, mb_result* out)
{
	return guard([&] {
		need(mod && cfg && out, "null argument");
		mb::run_config c = to_config(mod, cfg);
		auto r = std::make_unique<mb_result_s>();
		r->res = mb::run(*mod->mod, c);
		*out = r.release();
	});
}

// ------------------------------------------------------------------ batches and gradients

mb_status mb_batch_create(mb_context c, mb_batch* out)
{
	return guard([&] {
		need(c && out, "null argument");
		auto b = std::make_unique<mb_batch_s>();
		b->b = std::make_unique<mb::batch_engine>(*c->ctx);
		*out = b.release();
	});
}

mb_status mb_batch_free(mb_batch b)
{
	delete b;
	return MB_OK;
}

mb_status mb_batch_add_model(mb_batch b, mb_model m, int* net)
{
	return guard([&] {
		need(b && m && net, "null argument");
		*net = b->b->add_model(m->model);
	});
}

namespace {
std::map<std::string, float> overrides_of(const char* const* names, const float* values, int n)
{
	std::map<std::string, float> o;
	for (int i = 0; i < n; i++)
	{
		need(names && names[i] && values, "null variable name or value");
		o[names[i]] = values[i];
	}
	return o;
}
} // namespace

mb_status mb_batch_add_variant(mb_batch b, int net, const char* const* names, const float* values, int n_values,
							   long long n_traj, unsigned long long first_traj, int* variant)
{
	return guard([&] {
		need(b && variant && n_values >= 0, "bad argument");
		*variant = b->b->add_variant(net, overrides_of(names, values, n_values), n_traj, first_traj);
	});
}

mb_status mb_batch_add_variant_grad(mb_batch b, int net, const char* const* names, const float* values,
									int n_values, long long n_traj, unsigned long long first_traj,
									const char* const* grad_params, int n_grad, int* variant)
{
	return guard([&] {
		need(b && variant && n_values >= 0 && n_grad >= 0, "bad argument");
		std::vector<std::string> gp;
		for (int i = 0; i < n_grad; i++)
		{
			need(grad_params && grad_params[i], "null gradient parameter name");
			gp.push_back(grad_params[i]);
		}
		need(net >= 0 && net < (int)b->b->nets.size(), "bad network index");
		const mb::model_t& m = b->b->nets[net]->model;
		for (auto& g : gp)
			need(m.variables.count(g) != 0, "unknown gradient parameter");
		*variant = b->b->add_variant(net, overrides_of(names, values, n_values), n_traj, first_traj, gp);
	});
}

mb_status mb_batch_add_mutant(mb_batch b, int net, const char* const* names, const float* values, int n_values,
							  long long n_traj, unsigned long long first_traj, const char* const* nodes,
							  const int* on, int n_mutants, int* variant)
{
	return guard([&] {
		need(b && variant && n_values >= 0 && n_mutants >= 0, "bad argument");
		std::map<std::string, bool> mut;
		for (int i = 0; i < n_mutants; i++)
		{
			need(nodes && nodes[i] && on, "null mutant node name or state");
			mut[nodes[i]] = on[i] != 0;
		}
		*variant = b->b->add_variant(net, overrides_of(names, values, n_values), n_traj, first_traj, {}, mut);
	});
}

mb_status mb_batch_set_variables(mb_batch b, int v, const char* const* names, const float* values, int n_values)
{
	return guard([&] {
		need(b && n_values >= 0, "bad argument");
		b->b->set_variables(v, overrides_of(names, values, n_values));
	});
}

mb_status mb_batch_run_gradient(mb_batch b, unsigned long long seed, const double* const* cotangents,
								int n_cotangents, float* kernel_ms)
{
	return guard([&] {
		need(b, "null batch");
		mb::batch_engine& e = *b->b;
		need(n_cotangents == (int)e.vars_.size() && (cotangents || n_cotangents == 0),
			 "one cotangent per variant");
		std::vector<std::vector<double>> cot(e.vars_.size());
		for (size_t i = 0; i < e.vars_.size(); i++)
		{
			const mb::model_layout& L = e.nets[e.vars_[i]->net]->L;
			const size_t cells = (size_t)L.windows() << L.noninternal_nodes.size();
			cot[i] = cotangents[i] ? std::vector<double>(cotangents[i], cotangents[i] + cells)
								   : std::vector<double>(cells, 0.0);
		}
		e.run(seed, &cot);
		b->ran = true;
		if (kernel_ms)
			*kernel_ms = e.kernel_ms;
	});
}

mb_status mb_batch_gradient(mb_batch b, int v, double* grad, int cap, int* n_grad)
{
	return guard([&] {
		need(b && b->ran, "run the batch first");
		need(v >= 0 && v < (int)b->b->vars_.size(), "bad variant index");
		const std::vector<double>& g = b->b->vars_[v]->grad;
		need(cap >= 0 && (grad || cap == 0), "bad argument");
		for (int i = 0; i < cap && i < (int)g.size(); i++)
			grad[i] = g[i];
		if (n_grad)
			*n_grad = (int)g.size();
	});
}

mb_status mb_batch_set_options(mb_batch b, int use_graph, int autotune)
{
	return guard([&] {
		need(b, "null batch");
		b->b->use_graph = use_graph != 0;
		b->b->autotune = autotune != 0;
	});
}

mb_status mb_batch_set_specialize(mb_batch b, int on)
{
	return guard([&] {
		need(b, "null batch");
		b->b->specialize = on != 0;
	});
}

mb_status mb_batch_info(mb_batch b, int* block, int* blocks_per_sm, unsigned* grid, unsigned* graph_nodes,
						int* tuned_shapes)
{
	return guard([&] {
		need(b, "null batch");
		const mb::batch_engine& e = *b->b;
		if (block)
			*block = e.last_block;
		if (blocks_per_sm)
			*blocks_per_sm = e.last_per_sm;
		if (grid)
			*grid = e.last_grid;
		if (graph_nodes)
			*graph_nodes = e.use_graph ? e.graph_nodes : 0u;
		if (tuned_shapes)
			*tuned_shapes = (int)e.tuning.size();
	});
}

mb_status mb_batch_tuning(mb_batch b, int i, int* gradient, int* block, int* blocks_per_sm, float* kernel_ms)
{
	return guard([&] {
		need(b && i >= 0 && i < (int)b->b->tuning.size(), "bad tuning index");
		const auto& t = b->b->tuning[i];
		if (gradient)
			*gradient = t.grad ? 1 : 0;
		if (block)
			*block = t.block;
		if (blocks_per_sm)
			*blocks_per_sm = t.blocks_per_sm;
		if (kernel_ms)
			*kernel_ms = t.kernel_ms;
	});
}

mb_status mb_batch_run(mb_batch b, unsigned long long seed, float* kernel_ms)
{
	return guard([&] {
		need(b, "null batch");
		b->b->run(seed);
		b->ran = true;
		if (kernel_ms)
			*kernel_ms = b->b->kernel_ms;
	});
}

mb_status mb_batch_result(mb_batch b, int v, mb_result* out)
{
	return guard([&] {
		need(b && out && b->ran, "run the batch first");
		need(v >= 0 && v < (int)b->b->vars_.size(), "bad variant index");
		auto r = std::make_unique<mb_result_s>();
		r->res = std::make_unique<mb::result>(*b->b->vars_[v]->res);
		*out = r.release();
	});
}

mb_status mb_gradient(mb_context c, mb_model m, const char* const* params, const float* values, int n_params,
					  long long n_traj, unsigned long long seed, const double* cotangent, double* grad,
					  mb_result* forward)
{
	return guard([&] {
		need(c && m && cotangent && n_params >= 0 && (grad || n_params == 0), "bad argument");
		mb::batch_engine be(*c->ctx);
		// one run of a throw-away engine: neither a CUDA graph nor timed candidate shapes would be
		// used again; the default shape is 128 threads with as many blocks as fit
		be.use_graph = false;
		be.autotune = false;
		const int net = be.add_model(m->model);
		std::vector<std::string> names;
		for (int i = 0; i < n_params; i++)
		{
			need(params && params[i], "null parameter name");
			names.push_back(params[i]);
		}
		const int v = be.add_variant(net, overrides_of(params, values, n_params), n_traj, 0, names);
		const mb::model_layout& L = be.nets[net]->L;
		const size_t cells = (size_t)L.windows() << L.noninternal_nodes.size();
		std::vector<std::vector<double>> cot(1, std::vector<double>(cotangent, cotangent + cells));
		be.run(seed, &cot);
		for (int i = 0; i < n_params; i++)
			grad[i] = be.vars_[v]->grad[i];
		if (forward)
		{
			auto r = std::make_unique<mb_result_s>();
			r->res = std::move(be.vars_[v]->res);
			*forward = r.release();
		}
	});
}

// ------------------------------------------------------------------ results

mb_status mb_result_free(mb_result r)
{
	delete r;
	return MB_OK;
}

mb_status mb_result_dims(mb_result r, int* windows, int* bins, int* noninternal, int* state_words, int* nodes)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		if (windows)
			*windows = x.n_windows;
		if (bins)
			*bins = (int)x.n_bins;
		if (noninternal)
			*noninternal = (int)x.noninternal_nodes.size();
		if (state_words)
			*state_words = x.state_words;
		if (nodes)
			*nodes = x.state_size;
	});
}

mb_status mb_result_transitions(mb_result r, unsigned long long* t)
{
	return guard([&] {
		need(r && t, "null argument");
		*t = r->res->transitions;
	});
}

mb_status mb_result_timing(mb_result r, float* kernel_ms, float* total_ms, int* epochs)
{
	return guard([&] {
		need(r, "null result");
		if (kernel_ms)
			*kernel_ms = r->res->kernel_ms;
		if (total_ms)
			*total_ms = r->res->total_ms;
		if (epochs)
			*epochs = r->res->epochs;
	});
}

mb_status mb_result_window_probs(mb_result r, double* probs)
{
	return guard([&] {
		need(r && probs, "null argument");
		const mb::result& x = *r->res;
		need(x.sections & MB_STATS_WINDOWS, "the result has no window statistics");
		need(!x.wide, "sparse result (more than 20 non-internal nodes): use mb_result_sparse_windows");
		if (x.compact)
		{
			// zeros, then the stored (non-zero) cells
			std::memset(probs, 0, (size_t)x.n_windows * x.n_bins * sizeof(double));
			mb::parallel_ranges(x.sp_w.size(), (int)std::thread::hardware_concurrency(), [&](size_t a, size_t e) {
				for (size_t i = a; i < e; i++)
					probs[(size_t)x.sp_w[i] * x.n_bins + (size_t)x.sp_idx[i]] = x.n_traj > 0 ? x.sparse_prob(i) : 0.0;
			});
			return;
		}
		for (int w = 0; w < x.n_windows; w++)
			for (unsigned b = 0; b < x.n_bins; b++)
				probs[(size_t)w * x.n_bins + b] = x.n_traj > 0 ? x.window_prob(w, b) : 0.0;
	});
}

mb_status mb_result_window_entropy(mb_result r, double* th)
{
	return guard([&] {
		need(r && th, "null argument");
		const mb::result& x = *r->res;
		need(x.sections & MB_STATS_WINDOWS, "the result has no window statistics");
		for (int w = 0; w < x.n_windows; w++)
			th[w] = x.n_traj > 0 ? x.window_th(w) : 0.0;
	});
}

mb_status mb_result_window_raw(mb_result r, long long* occupancy, unsigned* counts, long long* entropy, int* occ_exp,
							   int* ent_exp)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		if (x.compact)
		{
			// the dense arrays from the stored (non-zero) cells
			const size_t cells = (size_t)x.n_windows * x.n_bins;
			if (occupancy && !x.discrete_time)
			{
				std::memset(occupancy, 0, cells * sizeof(long long));
				for (size_t i = 0; i < x.sp_w.size(); i++)
					occupancy[(size_t)x.sp_w[i] * x.n_bins + (size_t)x.sp_idx[i]] = x.sp_val[i];
			}
			if (counts && x.discrete_time)
			{
				std::memset(counts, 0, cells * sizeof(unsigned));
				for (size_t i = 0; i < x.sp_w.size(); i++)
					counts[(size_t)x.sp_w[i] * x.n_bins + (size_t)x.sp_idx[i]] = (unsigned)x.sp_val[i];
			}
		}
		if (occupancy && !x.win_occ.empty())
			std::memcpy(occupancy, x.win_occ.data(), x.win_occ.size() * sizeof(long long));
		if (counts && !x.win_cnt.empty())
			std::memcpy(counts, x.win_cnt.data(), x.win_cnt.size() * sizeof(unsigned));
		if (entropy && !x.win_h.empty())
			std::memcpy(entropy, x.win_h.data(), x.win_h.size() * sizeof(long long));
		if (occ_exp)
			*occ_exp = (int)std::lround(std::log2(x.fx));
		if (ent_exp)
			*ent_exp = (int)std::lround(std::log2(x.fx_h));
	});
}

mb_status mb_result_final_counts(mb_result r, unsigned* counts)
{
	return guard([&] {
		need(r && counts, "null argument");
		need(r->res->sections & MB_STATS_FINAL, "the result has no final-state statistics");
		need(!r->res->wide, "sparse result (more than 20 non-internal nodes): use mb_result_sparse_final");
		std::memcpy(counts, r->res->final_cnt.data(), r->res->final_cnt.size() * sizeof(unsigned));
	});
}

mb_status mb_result_windows_sparse(mb_result r, int* sparse)
{
	return guard([&] {
		need(r && sparse, "null argument");
		*sparse = r->res->sparse_windows() ? 1 : 0;
	});
}

mb_status mb_result_sparse_size(mb_result r, long long* window_entries, long long* final_entries,
								unsigned* bin_overflow)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		if (window_entries)
			*window_entries = (long long)x.sp_w.size();
		if (final_entries)
			*final_entries = (long long)x.fin_idx.size();
		if (bin_overflow)
			*bin_overflow = x.bin_overflow;
	});
}

mb_status mb_result_sparse_windows(mb_result r, int* windows, uint64_t* states, long long* raw, double* probs)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		// independent entries (tens of millions for a large job): copied by host threads
		mb::parallel_ranges(x.sp_w.size(), (int)std::thread::hardware_concurrency(), [&](size_t a, size_t e) {
			for (size_t i = a; i < e; i++)
			{
				if (windows)
					windows[i] = x.sp_w[i];
				if (states)
				{
					states[2 * i] = (uint64_t)x.sp_idx[i];
					states[2 * i + 1] = (uint64_t)(x.sp_idx[i] >> 64);
				}
				if (raw)
					raw[i] = x.sp_val[i];
				if (probs)
					probs[i] = x.sparse_prob(i);
			}
		});
	});
}

mb_status mb_result_sparse_final(mb_result r, uint64_t* states, unsigned* counts)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		for (size_t i = 0; i < x.fin_idx.size(); i++)
		{
			if (states)
			{
				states[2 * i] = (uint64_t)x.fin_idx[i];
				states[2 * i + 1] = (uint64_t)(x.fin_idx[i] >> 64);
			}
			if (counts)
				counts[i] = x.fin_cnt[i];
		}
	});
}

mb_status mb_result_num_fixed(mb_result r, int* n, unsigned* overflow)
{
	return guard([&] {
		need(r, "null result");
		if (n)
			*n = (int)r->res->fixed_counts.size();
		if (overflow)
			*overflow = r->res->fixed_overflow;
	});
}

mb_status mb_result_fixed(mb_result r, int i, uint32_t* state_words, unsigned* count)
{
	return guard([&] {
		need(r && i >= 0 && i < (int)r->res->fixed_counts.size(), "bad fixed-point index");
		const mb::result& x = *r->res;
		if (state_words)
			std::memcpy(state_words, x.fixed_states.data() + (size_t)i * x.state_words, x.state_words * sizeof(uint32_t));
		if (count)
			*count = x.fixed_counts[i];
	});
}

mb_status mb_result_write_csv(mb_result r, mb_model m, const char* prefix)
{
	return guard([&] {
		need(r && m && prefix, "null argument");
		need(r->res->sections == MB_STATS_ALL, "the result lacks some of the three statistics");
		need((int)m->model.nodes.size() == r->res->state_size, "model does not match the result");
		const auto names = names_of(m->model);
		{
			std::ofstream f(std::string(prefix) + "_probtraj.csv");
			if (!f)
				throw mb::engine_error(MB_ERR_INVALID, std::string("cannot write ") + prefix + "_probtraj.csv");
			f << mb::format_probtraj_csv(*r->res, names);
		}
		{
			std::ofstream f(std::string(prefix) + "_fp.csv");
			if (!f)
				throw mb::engine_error(MB_ERR_INVALID, std::string("cannot write ") + prefix + "_fp.csv");
			f << mb::format_fp_csv(*r->res, names);
		}
	});
}

mb_status mb_result_write_final_csv(mb_result r, mb_model m, const char* prefix)
{
	return guard([&] {
		need(r && m && prefix, "null argument");
		need(r->res->sections & MB_STATS_FINAL, "the result has no final-state statistics");
		need((int)m->model.nodes.size() == r->res->state_size, "model does not match the result");
		std::ofstream f(std::string(prefix) + "_finalprob.csv");
		if (!f)
			throw mb::engine_error(MB_ERR_INVALID, std::string("cannot write ") + prefix + "_finalprob.csv");
		f << mb::format_final_csv(*r->res, names_of(m->model));
	});
}

mb_status mb_result_info(mb_result r, long long* n_trajectories, int* discrete_time, float* time_tick,
						 float* max_time, int* noninternal_nodes)
{
	return guard([&] {
		need(r, "null result");
		const mb::result& x = *r->res;
		if (n_trajectories)
			*n_trajectories = x.n_traj;
		if (discrete_time)
			*discrete_time = x.discrete_time ? 1 : 0;
		if (time_tick)
			*time_tick = x.time_tick;
		if (max_time)
			*max_time = x.max_time;
		if (noninternal_nodes)
			std::copy(x.noninternal_nodes.begin(), x.noninternal_nodes.end(), noninternal_nodes);
	});
}

mb_status mb_result_create(const mb_result_desc* d, mb_result* out)
{
	return guard([&] {
		need(d && out, "null argument");
		need(d->n_nodes > 0 && d->n_windows > 0 && d->n_trajectories >= 0, "bad dimensions");
		need(d->n_noninternal >= 0 && d->n_noninternal <= 20 && (d->noninternal_nodes || d->n_noninternal == 0),
			 "at most 20 non-internal nodes");
		need(d->time_tick > 0.f && d->max_time > 0.f, "max_time and time_tick must be positive");
		need(d->occupancy_exponent >= 0 && d->occupancy_exponent <= 100 && d->entropy_exponent >= 0 &&
				 d->entropy_exponent <= 100,
			 "exponents must be in [0, 100]");
		need(d->n_fixed >= 0 && (d->n_fixed == 0 || (d->fixed_states && d->fixed_counts)), "bad fixed points");
		need(d->entropy && d->final_counts && (d->discrete_time ? d->counts != nullptr : d->occupancy != nullptr),
			 "null accumulator");
		auto r = std::make_unique<mb::result>();
		r->state_size = d->n_nodes;
		r->state_words = (d->n_nodes + 31) / 32;
		r->n_windows = d->n_windows;
		r->n_bins = 1u << d->n_noninternal;
		r->n_traj = d->n_trajectories;
		r->discrete_time = d->discrete_time != 0;
		r->time_tick = d->time_tick;
		r->max_time = d->max_time;
		r->noninternal_nodes.assign(d->noninternal_nodes, d->noninternal_nodes + d->n_noninternal);
		for (size_t i = 0; i < r->noninternal_nodes.size(); i++)
			need(r->noninternal_nodes[i] >= 0 && r->noninternal_nodes[i] < d->n_nodes &&
					 (i == 0 || r->noninternal_nodes[i] > r->noninternal_nodes[i - 1]),
				 "non-internal nodes must be increasing node indices");
		r->fx = std::ldexp(1.0, d->occupancy_exponent);
		r->fx_h = std::ldexp(1.0, d->entropy_exponent);
		const size_t cells = (size_t)d->n_windows * r->n_bins;
		if (r->discrete_time)
			r->win_cnt.assign(d->counts, d->counts + cells);
		else
			r->win_occ.assign(d->occupancy, d->occupancy + cells);
		r->win_h.assign(d->entropy, d->entropy + d->n_windows);
		r->final_cnt.assign(d->final_counts, d->final_counts + r->n_bins);
		r->transitions = d->transitions;
		std::map<std::vector<unsigned>, unsigned long long> fixed;
		const int W = r->state_words;
		for (int j = 0; j < d->n_fixed; j++)
			fixed[std::vector<unsigned>(d->fixed_states + (size_t)j * W, d->fixed_states + (size_t)(j + 1) * W)] +=
				d->fixed_counts[j];
		std::vector<unsigned> st, cn;
		for (auto& [state, count] : fixed)
		{
			st.insert(st.end(), state.begin(), state.end());
			cn.push_back((unsigned)count);
		}
		mb::set_fixed_sorted(*r, st, cn);
		auto h = std::make_unique<mb_result_s>();
		h->res = std::move(r);
		*out = h.release();
	});
}

mb_status mb_result_merge(const mb_result* parts, int n_parts, mb_result* out)
{
	return guard([&] {
		need(parts && n_parts > 0 && out, "bad argument");
		std::vector<const mb::result*> rs;
		for (int i = 0; i < n_parts; i++)
		{
			need(parts[i] && parts[i]->res, "null result");
			rs.push_back(parts[i]->res.get());
		}
		auto h = std::make_unique<mb_result_s>();
		h->res = mb::merge_results(rs);
		*out = h.release();
	});
}

mb_status mb_result_format(mb_result r, int section, int format, const char* const* node_names, int n_names,
						   char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(r && (node_names || n_names == 0), "null argument");
		const mb::result& res = *r->res;
		need(n_names == res.state_size, "one name per node is needed");
		need(format == MB_FORMAT_VISUALIZE || format == MB_FORMAT_CSV || format == MB_FORMAT_CSV_FINAL_STATES,
			 "unknown format");
		std::vector<std::string> names(node_names, node_names + n_names);
		std::string text;
		switch (section)
		{
		case MB_SECTION_FINAL:
			need(res.sections & MB_STATS_FINAL, "the result has no final-state statistics");
			if (format == MB_FORMAT_VISUALIZE)
				text = mb::format_final_visualize(res, names);
			else if (format == MB_FORMAT_CSV_FINAL_STATES)
				text = mb::format_final_csv(res, names);
			break;
		case MB_SECTION_FIXED:
			need(res.sections & MB_STATS_FIXED, "the result has no fixed-point statistics");
			text = format == MB_FORMAT_VISUALIZE ? mb::format_fixed_visualize(res, names) : mb::format_fp_csv(res, names);
			break;
		case MB_SECTION_WINDOWS:
			need(res.sections & MB_STATS_WINDOWS, "the result has no window statistics");
			text = format == MB_FORMAT_VISUALIZE ? mb::format_windows_visualize(res, names)
												 : mb::format_probtraj_csv(res, names);
			break;
		default:
			need(false, "unknown section");
		}
		copy_out(text, buf, cap, len);
	});
}

mb_status mb_result_visualize(mb_result r, mb_model m, char* buf, size_t cap, size_t* len)
{
	return guard([&] {
		need(r && m, "null argument");
		need(r->res->sections == MB_STATS_ALL, "the result lacks some of the three statistics");
		need((int)m->model.nodes.size() == r->res->state_size, "model does not match the result");
		copy_out(mb::format_visualize(*r->res, names_of(m->model)), buf, cap, len);
	});
}

} // extern "C"
