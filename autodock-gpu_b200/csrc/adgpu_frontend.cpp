// adgpu_frontend.cpp -- C ABI of the front end (include/adgpu_b200.h).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>
#include "adgpu_prep.h"

namespace adgpu {
adgpu_status fail(adgpu_status st, const std::string& msg);
}
using namespace adgpu;

extern "C" {

adgpu_status adgpu_grid_read(const char* fld_path, adgpu_grid** out)
{
	if (!fld_path || !out) return fail(ADGPU_ERR_ARG, "null argument");
	adgpu_grid* g = new (std::nothrow) adgpu_grid;
	if (!g) return fail(ADGPU_ERR_ARG, "out of host memory");
	adgpu_status st = grid_read(fld_path, g->g);
	if (st != ADGPU_OK) { delete g; return st; }
	*out = g;
	return ADGPU_OK;
}

adgpu_status adgpu_grid_from_values(const int dims[3], double spacing, const double origin[3], int num_maps,
                                    const char* const* types, const float* values, adgpu_grid** out)
{
	if (!dims || !origin || !types || !values || !out) return fail(ADGPU_ERR_ARG, "null argument");
	if (num_maps < 3 || strcmp(types[num_maps - 2], "e") || strcmp(types[num_maps - 1], "d"))
		return fail(ADGPU_ERR_ARG, "maps must be type maps followed by e and d");
	for (int k = 0; k < 3; k++)
		if (dims[k] < 2 || dims[k] > 256) return fail(ADGPU_ERR_LIMIT, "grid dimensions must be 2..256");
	if (spacing <= 0 || spacing > 1) return fail(ADGPU_ERR_ARG, "grid spacing must be in (0, 1]");
	adgpu_grid* g = new (std::nothrow) adgpu_grid;
	if (!g) return fail(ADGPU_ERR_ARG, "out of host memory");
	for (int k = 0; k < 3; k++) { g->g.dims[k] = dims[k]; g->g.origin[k] = origin[k]; }
	g->g.spacing = spacing;
	g->g.num_map_atypes = num_maps - 2;
	for (int m = 0; m < num_maps; m++) g->g.types.push_back(types[m]);
	size_t n = (size_t)dims[0] * dims[1] * dims[2] * num_maps;
	g->g.values.assign(values, values + n);
	*out = g;
	return ADGPU_OK;
}

void adgpu_grid_free(adgpu_grid* grid) { delete grid; }

adgpu_status adgpu_grid_save(const adgpu_grid* grid, const char* path)
{
	if (!grid || !path) return fail(ADGPU_ERR_ARG, "null argument");
	return grid_save(grid->g, path);
}

adgpu_status adgpu_grid_load(const char* path, adgpu_grid** out)
{
	if (!path || !out) return fail(ADGPU_ERR_ARG, "null argument");
	adgpu_grid* g = new (std::nothrow) adgpu_grid;
	if (!g) return fail(ADGPU_ERR_ARG, "out of host memory");
	adgpu_status st = grid_load(path, g->g);
	if (st != ADGPU_OK) { delete g; return st; }
	*out = g;
	return ADGPU_OK;
}

adgpu_status adgpu_grid_info(const adgpu_grid* grid, int dims[3], double* spacing, double origin[3], int* num_map_atypes)
{
	if (!grid) return fail(ADGPU_ERR_ARG, "null grid");
	for (int k = 0; k < 3; k++) {
		if (dims) dims[k] = grid->g.dims[k];
		if (origin) origin[k] = grid->g.origin[k];
	}
	if (spacing) *spacing = grid->g.spacing;
	if (num_map_atypes) *num_map_atypes = grid->g.num_map_atypes;
	return ADGPU_OK;
}

adgpu_status adgpu_grid_reference_layout(const adgpu_grid* grid, float* out, size_t n_floats)
{
	if (!grid || !out) return fail(ADGPU_ERR_ARG, "null argument");
	const Grid& g = grid->g;
	size_t need = (size_t)4 * g.types.size() * g.dims[0] * g.dims[1] * g.dims[2];
	if (n_floats != need) return fail(ADGPU_ERR_ARG, "output size must be 4*num_maps*X*Y*Z floats");
	memset(out, 0, need * sizeof(float));
	grid_reference_layout(g, out);
	return ADGPU_OK;
}

adgpu_status adgpu_dockpars_default(adgpu_dockpars* dp, double spacing, int pop_size)
{
	if (!dp) return fail(ADGPU_ERR_ARG, "null dockpars");
	if (pop_size < 2 || pop_size > ADGPU_MAX_POPSIZE) return fail(ADGPU_ERR_LIMIT, "pop_size must be 2..2048");
	if (spacing <= 0 || spacing > 1) return fail(ADGPU_ERR_ARG, "grid spacing must be in (0, 1]");
	dockpars_defaults(*dp, spacing, pop_size);
	return ADGPU_OK;
}

adgpu_status adgpu_ligand_prepare(const adgpu_grid* grid, const char* ligand_pdbqt, const char* flexres_pdbqt,
                                  const adgpu_dockpars* run, const uint32_t seed[3], int num_runs, adgpu_ligand** out)
{
	if (!grid || !run || !seed || !out) return fail(ADGPU_ERR_ARG, "null argument");
	if (!ligand_pdbqt && !flexres_pdbqt) return fail(ADGPU_ERR_ARG, "no ligand or flexible residue");
	if (num_runs < 0 || num_runs > ADGPU_MAX_RUNS) return fail(ADGPU_ERR_LIMIT, "num_runs must be 0..8192");
	if (run->pop_size < 2 || run->pop_size > ADGPU_MAX_POPSIZE) return fail(ADGPU_ERR_LIMIT, "pop_size must be 2..2048");
	adgpu_ligand* l = new (std::nothrow) adgpu_ligand;
	if (!l) return fail(ADGPU_ERR_ARG, "out of host memory");
	adgpu_status st = prepare_ligand(grid->g, ligand_pdbqt ? ligand_pdbqt : "", flexres_pdbqt ? flexres_pdbqt : "",
	                                 *run, seed, num_runs, l->p);
	if (st != ADGPU_OK) { delete l; return st; }
	*out = l;
	return ADGPU_OK;
}

void adgpu_ligand_free(adgpu_ligand* lig) { delete lig; }

adgpu_status adgpu_ligand_prepare_batch(const adgpu_grid* grid, const char* const* ligand_pdbqt,
                                        const char* const* flexres_pdbqt, uint32_t count, const adgpu_dockpars* run,
                                        const uint32_t* seeds, int num_runs, int nthreads, adgpu_ligand** out,
                                        adgpu_status* status)
{
	if (!grid || !ligand_pdbqt || !run || !seeds || !out || !status) return fail(ADGPU_ERR_ARG, "null argument");
	if (num_runs < 0 || num_runs > ADGPU_MAX_RUNS) return fail(ADGPU_ERR_LIMIT, "num_runs must be 0..8192");
	if (run->pop_size < 2 || run->pop_size > ADGPU_MAX_POPSIZE) return fail(ADGPU_ERR_LIMIT, "pop_size must be 2..2048");
	for (uint32_t i = 0; i < count; i++) { out[i] = nullptr; status[i] = ADGPU_ERR_STATE; }
	unsigned hw = std::max(1u, std::thread::hardware_concurrency());
	unsigned nt = nthreads > 0 ? (unsigned)nthreads : hw;
	nt = std::max(1u, std::min<unsigned>(nt, count));
	std::atomic<uint32_t> next(0);
	std::vector<std::string> why(count);     // a worker's error text (the last error is per thread)
	auto work = [&]() {
		for (uint32_t i; (i = next.fetch_add(1)) < count;) {
			const char* lt = ligand_pdbqt[i];
			const char* ft = flexres_pdbqt ? flexres_pdbqt[i] : nullptr;
			if (!lt && !ft) { status[i] = ADGPU_ERR_ARG; continue; }
			adgpu_ligand* l = new (std::nothrow) adgpu_ligand;
			if (!l) { status[i] = ADGPU_ERR_ARG; continue; }
			adgpu_status st = prepare_ligand(grid->g, lt ? lt : "", ft ? ft : "", *run, seeds + 3 * (size_t)i, num_runs, l->p);
			if (st != ADGPU_OK) { delete l; status[i] = st; why[i] = adgpu_last_error(); continue; }
			out[i] = l;
			status[i] = ADGPU_OK;
		}
	};
	std::vector<std::thread> pool;
	for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
	work();
	for (auto& t : pool) t.join();
	for (uint32_t i = 0; i < count; i++)
		if (status[i] != ADGPU_OK)
			return fail(status[i], "ligand " + std::to_string(i) + " could not be prepared" +
			                           (why[i].empty() ? std::string() : ": " + why[i]));
	return ADGPU_OK;
}

adgpu_status adgpu_ligand_tables(const adgpu_ligand* lig, adgpu_dockpars* dockpars, adgpu_kc_interintra* interintra,
                                 adgpu_kc_intracontrib* intracontrib, adgpu_kc_intra* intra, adgpu_kc_rotlist* rotlist,
                                 adgpu_kc_conform* conform, adgpu_kc_grads* grads)
{
	if (!lig) return fail(ADGPU_ERR_ARG, "null ligand");
	const Prepared& p = lig->p;
	if (dockpars) *dockpars = p.dockpars;
	if (interintra) *interintra = p.interintra;
	if (intracontrib) {
		memset(intracontrib, 0, sizeof(*intracontrib));
		memcpy(intracontrib->intraE_contributors_const, p.pairs.data(), p.pairs.size() * sizeof(uint32_t));
	}
	if (intra) *intra = p.intra;
	if (rotlist) {
		memset(rotlist, 0, sizeof(*rotlist));
		memcpy(rotlist->rotlist_const, p.rotlist.data(), p.rotlist.size() * sizeof(int));
	}
	if (conform) *conform = p.conform;
	if (grads) *grads = p.grads;
	return ADGPU_OK;
}

adgpu_status adgpu_ligand_population(const adgpu_ligand* lig, float* initpop, size_t n_floats, uint32_t* prng, size_t n_states)
{
	if (!lig) return fail(ADGPU_ERR_ARG, "null ligand");
	const Prepared& p = lig->p;
	if (initpop) {
		if (n_floats != p.initpop.size()) return fail(ADGPU_ERR_ARG, "initpop size must be runs*pop_size*64");
		memcpy(initpop, p.initpop.data(), n_floats * sizeof(float));
	}
	if (prng) {
		if (n_states != p.prng.size()) return fail(ADGPU_ERR_ARG, "prng size must be runs*pop_size*64");
		memcpy(prng, p.prng.data(), n_states * sizeof(uint32_t));
	}
	return ADGPU_OK;
}

}  // extern "C"
