// MaBoSS.GPU command line (same usage as the reference's src/main.cpp:101-169), written against
// the C ABI only.
//
//   MaBoSS.GPU [options] [-o prefix] model.bnd model.cfg
//     -o prefix        write <prefix>_probtraj.csv and <prefix>_fp.csv instead of printing
//     --mode M         exact (default; bit-exact with the reference), fast, or epoch (buffered)
//     --device D       CUDA device ordinal (default 0)
//     --emit-code      print the generated CUDA source and exit (no GPU needed)
//     --stats          print transitions and timings to stderr
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "maboss_b200.h"

namespace {

int fail(const char* what)
{
	std::cerr << what << ": " << mb_last_error() << std::endl;
	return 1;
}

void usage()
{
	std::cout << "Usage: MaBoSS.GPU [--mode exact|fast|epoch] [--device D] [--emit-code] [--stats] [-o prefix] "
				 "bnd_file cfg_file"
			  << std::endl;
}

} // namespace

int main(int argc, char** argv)
{
	std::vector<std::string> args(argv + 1, argv + argc);
	std::string prefix, mode = "exact";
	int device = 0;
	bool emit = false, stats = false;
	std::vector<std::string> files;
	for (size_t i = 0; i < args.size(); i++)
	{
		const std::string& a = args[i];
		if (a == "-o" && i + 1 < args.size())
			prefix = args[++i];
		else if (a == "--mode" && i + 1 < args.size())
			mode = args[++i];
		else if (a == "--device" && i + 1 < args.size())
			device = std::stoi(args[++i]);
		else if (a == "--emit-code")
			emit = true;
		else if (a == "--stats")
			stats = true;
		else if (!a.empty() && a[0] == '-')
		{
			usage();
			return 1;
		}
		else
			files.push_back(a);
	}
	if (files.size() != 2)
	{
		usage();
		return 1;
	}

	mb_model model = nullptr;
	if (mb_model_parse_files(files[0].c_str(), files[1].c_str(), &model) != MB_OK)
		return fail("parse");

	if (emit)
	{
		size_t len = 0;
		if (mb_model_generate_code(model, nullptr, 0, &len) != MB_OK)
			return fail("generate");
		std::string code(len + 1, '\0');
		mb_model_generate_code(model, &code[0], code.size(), &len);
		code.resize(len);
		std::fwrite(code.data(), 1, code.size(), stdout);
		mb_model_free(model);
		return 0;
	}

	int n = 0;
	mb_model_num_nodes(model, &n);
	int noninternal = 0;
	for (int i = 0; i < n; i++)
	{
		int internal = 0;
		mb_model_node_info(model, i, nullptr, &internal);
		noninternal += internal ? 0 : 1;
	}
	// src/main.cpp:142-146
	if (noninternal > 20)
	{
		std::cerr << "This executable supports a maximum of 20 non-internal nodes." << std::endl;
		return 1;
	}

	mb_context ctx = nullptr;
	if (mb_context_create(device, &ctx) != MB_OK)
		return fail("device");
	mb_module mod = nullptr;
	if (mb_module_compile_model(ctx, model, &mod) != MB_OK)
		return fail("compile");
	mb_run_config cfg;
	mb_run_config_default(model, &cfg);
	cfg.mode = mode == "fast" ? MB_MODE_FUSED_FAST : mode == "epoch" ? MB_MODE_EPOCH : MB_MODE_FUSED_EXACT;
	mb_result res = nullptr;
	if (mb_run(mod, &cfg, &res) != MB_OK)
		return fail("run");

	if (stats)
	{
		unsigned long long t = 0;
		float kms = 0, tms = 0;
		int epochs = 0;
		mb_result_transitions(res, &t);
		mb_result_timing(res, &kms, &tms, &epochs);
		std::cerr << "transitions: " << t << "  kernel_ms: " << kms << "  total_ms: " << tms << "  epochs: " << epochs
				  << "  transitions/s: " << (kms > 0 ? (double)t / (kms * 1e-3) : 0.0) << std::endl;
	}

	if (!prefix.empty())
	{
		if (mb_result_write_csv(res, model, prefix.c_str()) != MB_OK)
			return fail("write");
	}
	else
	{
		size_t len = 0;
		mb_result_visualize(res, model, nullptr, 0, &len);
		std::string text(len + 1, '\0');
		mb_result_visualize(res, model, &text[0], text.size(), &len);
		text.resize(len);
		std::fwrite(text.data(), 1, text.size(), stdout);
	}
	mb_result_free(res);
	mb_module_free(mod);
	mb_context_free(ctx);
	mb_model_free(model);
	return 0;
}
