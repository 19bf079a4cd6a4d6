/*
 * ref_prepare.cpp -- drives the reference's own host front end (compiled from
 * host/src/*.cpp of AutoDock-GPU where they lie) to turn .fld/.map/.pdbqt
 * inputs plus a command line into the exact tables the reference hands to
 * its kernel API.  TEST INFRASTRUCTURE ONLY (oracle side).
 *
 * Sequence restated from the reference:
 *   initial_commandpars + get_filelist        host/src/main.cpp:104-107
 *   setup()                                   host/src/main.cpp:333 -> host/src/setup.cpp:60
 *   gen_initpop_and_reflig, LocalRNG seeds    host/src/performdocking.cpp.Cuda:302-317
 *   prepare_const_fields_for_gpu              host/src/performdocking.cpp.Cuda:352-361
 *   GpuDockparameters fill                    host/src/performdocking.cpp.Cuda:413-463
 */
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <cstdint>
#include "filelist.hpp"
#include "processgrid.h"
#include "processligand.h"
#include "getparameters.h"
#include "setup.hpp"
#include "calcenergy.h"
#include "processresult.h"

/* GpuDockparameters, cuda/GpuData.h:74-110 (kept byte-identical). */
typedef struct {
	int num_of_atoms, true_ligand_atoms, num_of_atypes, num_of_map_atypes, num_of_intraE_contributors;
	int gridsize_x, gridsize_y, gridsize_z, gridsize_x_times_y, gridsize_x_times_y_times_z;
	float grid_spacing;
	int rotbondlist_length;
	float coeff_elec, elec_min_distance, coeff_desolv;
	int pop_size, num_of_genes;
	float tournament_rate, crossover_rate, mutation_rate, abs_max_dmov, abs_max_dang, lsearch_rate, smooth;
	unsigned int num_of_lsentities;
	float rho_lower_bound, base_dmov_mul_sqrt3, base_dang_mul_sqrt3;
	unsigned int cons_limit, max_num_of_iters;
	float qasp, adam_beta1, adam_beta2, adam_epsilon;
} RefDockpars;

struct RefJob {
	RefDockpars dockpars;
	kernelconstant_interintra interintra;
	kernelconstant_intracontrib intracontrib;
	kernelconstant_intra intra;
	kernelconstant_rotlist rotlist;
	kernelconstant_conform conform;
	kernelconstant_grads grads;
	std::vector<float> grid;
	std::vector<float> initpop;
	std::vector<uint32_t> prng;
	int num_runs = 0;
	int num_rotbonds = 0;
	int num_rotcyc = 0;
	unsigned long nev = 0;
	unsigned long ngen = 0;
	char lsmet[8] = {0};
	float grid_origin[3] = {0, 0, 0};
	float grid_size_angstrom[3] = {0, 0, 0};
	std::vector<int32_t> bonds;        // [N*N] bond matrix of the prepared ligand
	std::vector<int32_t> rigid;        // [N] rigid structure ids
	std::vector<int32_t> contrib;      // [N*N] intramolecular contributor matrix
	// kept for result processing (process_result's inputs)
	std::unique_ptr<Liganddata> lig_ref;   // sim_state.myligand_reference
	std::unique_ptr<Liganddata> lig_init;  // myligand_init (coordinates as read)
	std::unique_ptr<Liganddata> xray;
	Dockpars mypars;
	Gridinfo gridinfo;
};

/* GpuData layout of cuda/GpuData.h:112-136, with plain pointer members. */
struct RefGpuData {
	int devnum, devid, preallocated_gridsize;
	RefDockpars dockpars;
	void* pKerconst_interintra;
	void* pKerconst_intracontrib;
	void* pKerconst_intra;
	void* pKerconst_rotlist;
	void* pKerconst_conform;
	void* pKerconst_grads;
	float* pMem_fgrids;
	int* pMem_evals_of_new_entities;
	int* pMem_gpu_evals_of_runs;
	uint32_t* pMem_prng_states;
	int* pMem_rotbonds_const;
	int* pMem_rotbonds_atoms_const;
	int* pMem_num_rotating_atoms_per_rotbond_const;
	unsigned int warpmask, warpbits;
};

extern "C" void adgpu_ref_set_gpudata(const void* data);

extern "C" {

typedef struct {
	int num_of_atoms, true_ligand_atoms, num_of_rotbonds, num_of_genes, num_of_intraE_contributors;
	int num_of_rotcyc, pop_size, num_of_runs, num_of_lsentities, num_of_map_atypes;
	int gridsize[3];
	float spacing;
	float grid_origin[3];
	unsigned long nev, ngen;
	char lsmet[8];
} adgpu_ref_info;

void* adgpu_ref_job_create(int argc, char** argv)
{
	FileList filelist;
	Dockpars initial_pars;
	Gridinfo initial_grid;
	if (initial_commandpars(&argc, argv, &initial_pars, &initial_grid, filelist) != 0) return nullptr;
	if (get_filelist(&argc, argv, &initial_pars, &initial_grid, filelist) != 0) return nullptr;
	Dockpars mypars = initial_pars;
	Gridinfo* mygrid = &initial_grid;
	if (filelist.used) {
		mypars = filelist.mypars[0];
		mygrid = &filelist.mygrids[mypars.filelist_grid_idx];
	}
	Liganddata* lig_init = new Liganddata;
	Liganddata* xray = new Liganddata;
	if (setup(mygrid, &mypars, *lig_init, *xray, filelist, 0, argc, argv) != 0) {
		delete lig_init; delete xray; return nullptr;
	}
	RefJob* job = new RefJob;
	job->num_runs = (int)mypars.num_of_runs;
	size_t npop = (size_t)mypars.num_of_runs * mypars.pop_size;
	job->initpop.assign(npop * GENOTYPE_LENGTH_IN_GLOBMEM, 0.0f);
	Liganddata* lig = new Liganddata;
	*lig = *lig_init;
	gen_initpop_and_reflig(&mypars, job->initpop.data(), lig, mygrid);
	job->prng.resize(npop * NUM_OF_THREADS_PER_BLOCK);
	LocalRNG r(mypars.seed);
	for (size_t i = 0; i < job->prng.size(); i++) job->prng[i] = r.random_uint();
	if (prepare_const_fields_for_gpu(lig, &mypars, &job->interintra, &job->intracontrib, &job->intra,
	                                 &job->rotlist, &job->conform, &job->grads) != 0) {
		delete lig; delete lig_init; delete xray; delete job; return nullptr;
	}
	job->grid.assign(mygrid->grids.begin(), mygrid->grids.end());
	RefDockpars& d = job->dockpars;
	memset(&d, 0, sizeof(d));
	d.num_of_atoms = lig->num_of_atoms;
	d.true_ligand_atoms = (int)lig->true_ligand_atoms;
	d.num_of_atypes = lig->num_of_atypes;
	d.num_of_map_atypes = mygrid->num_of_map_atypes;
	d.num_of_intraE_contributors = (int)lig->num_of_intraE_contributors;
	d.gridsize_x = mygrid->size_xyz[0];
	d.gridsize_y = mygrid->size_xyz[1];
	d.gridsize_z = mygrid->size_xyz[2];
	d.gridsize_x_times_y = d.gridsize_x * d.gridsize_y;
	d.gridsize_x_times_y_times_z = d.gridsize_x * d.gridsize_y * d.gridsize_z;
	d.grid_spacing = (float)mygrid->spacing;
	d.rotbondlist_length = (int)NUM_OF_THREADS_PER_BLOCK * lig->num_of_rotcyc;
	d.coeff_elec = (float)mypars.coeffs.scaled_AD4_coeff_elec;
	d.elec_min_distance = (float)mypars.elec_min_distance;
	d.coeff_desolv = (float)mypars.coeffs.AD4_coeff_desolv;
	d.pop_size = (int)mypars.pop_size;
	d.num_of_genes = lig->num_of_rotbonds + 6;
	d.tournament_rate = mypars.tournament_rate / 100.0f;
	d.crossover_rate = mypars.crossover_rate / 100.0f;
	d.mutation_rate = mypars.mutation_rate / 100.f;
	d.abs_max_dang = mypars.abs_max_dang;
	d.abs_max_dmov = mypars.abs_max_dmov;
	d.qasp = mypars.qasp;
	d.smooth = mypars.smooth;
	d.lsearch_rate = mypars.lsearch_rate;
	d.adam_beta1 = mypars.adam_beta1;
	d.adam_beta2 = mypars.adam_beta2;
	d.adam_epsilon = mypars.adam_epsilon;
	if (d.lsearch_rate != 0.0f) {
		d.num_of_lsentities = (unsigned int)(mypars.lsearch_rate / 100.0 * mypars.pop_size + 0.5);
		d.rho_lower_bound = mypars.rho_lower_bound;
		d.base_dmov_mul_sqrt3 = mypars.base_dmov_mul_sqrt3;
		d.base_dang_mul_sqrt3 = mypars.base_dang_mul_sqrt3;
		d.cons_limit = (unsigned int)mypars.cons_limit;
		d.max_num_of_iters = (unsigned int)mypars.max_num_of_iters;
	}
	job->num_rotbonds = lig->num_of_rotbonds;
	job->num_rotcyc = lig->num_of_rotcyc;
	job->nev = mypars.num_of_energy_evals;
	job->ngen = mypars.num_of_generations;
	strncpy(job->lsmet, mypars.ls_method, sizeof(job->lsmet) - 1);
	for (int i = 0; i < 3; i++) job->grid_origin[i] = (float)mygrid->origo_real_xyz[i];
	{
		int n = lig->num_of_atoms;
		job->bonds.resize((size_t)n * n); job->contrib.resize((size_t)n * n); job->rigid.resize(n);
		for (int a = 0; a < n; a++) {
			job->rigid[a] = lig->atom_rigid_structures[a];
			for (int b = 0; b < n; b++) {
				job->bonds[(size_t)a * n + b] = lig->bonds[a][b];
				job->contrib[(size_t)a * n + b] = lig->intraE_contributors[a][b];
			}
		}
	}
	job->lig_ref.reset(lig);
	job->lig_init.reset(lig_init);
	job->xray.reset(xray);
	job->mypars = mypars;
	job->gridinfo = *mygrid;
	return job;
}

void adgpu_ref_job_free(void* h) { delete (RefJob*)h; }

int adgpu_ref_job_info(void* h, adgpu_ref_info* out)
{
	RefJob* j = (RefJob*)h;
	memset(out, 0, sizeof(*out));
	out->num_of_atoms = j->dockpars.num_of_atoms;
	out->true_ligand_atoms = j->dockpars.true_ligand_atoms;
	out->num_of_rotbonds = j->num_rotbonds;
	out->num_of_genes = j->dockpars.num_of_genes;
	out->num_of_intraE_contributors = j->dockpars.num_of_intraE_contributors;
	out->num_of_rotcyc = j->num_rotcyc;
	out->pop_size = j->dockpars.pop_size;
	out->num_of_runs = j->num_runs;
	out->num_of_lsentities = (int)j->dockpars.num_of_lsentities;
	out->num_of_map_atypes = j->dockpars.num_of_map_atypes;
	out->gridsize[0] = j->dockpars.gridsize_x;
	out->gridsize[1] = j->dockpars.gridsize_y;
	out->gridsize[2] = j->dockpars.gridsize_z;
	out->spacing = j->dockpars.grid_spacing;
	for (int i = 0; i < 3; i++) out->grid_origin[i] = j->grid_origin[i];
	out->nev = j->nev;
	out->ngen = j->ngen;
	memcpy(out->lsmet, j->lsmet, sizeof(out->lsmet));
	return 0;
}

/* Pointer to, and size of, one of the job's tables. */
void* adgpu_ref_job_blob(void* h, const char* name, size_t* nbytes)
{
	RefJob* j = (RefJob*)h;
	std::string n(name);
#define BLOB(key, ptr, sz) if (n == key) { *nbytes = (sz); return (void*)(ptr); }
	BLOB("dockpars", &j->dockpars, sizeof(j->dockpars));
	BLOB("interintra", &j->interintra, sizeof(j->interintra));
	BLOB("intracontrib", &j->intracontrib, sizeof(j->intracontrib));
	BLOB("intra", &j->intra, sizeof(j->intra));
	BLOB("rotlist", &j->rotlist, sizeof(j->rotlist));
	BLOB("conform", &j->conform, sizeof(j->conform));
	BLOB("grads", &j->grads, sizeof(j->grads));
	BLOB("grid", j->grid.data(), j->grid.size() * sizeof(float));
	BLOB("initpop", j->initpop.data(), j->initpop.size() * sizeof(float));
	BLOB("prng", j->prng.data(), j->prng.size() * sizeof(uint32_t));
	BLOB("bonds", j->bonds.data(), j->bonds.size() * sizeof(int32_t));
	BLOB("rigid", j->rigid.data(), j->rigid.size() * sizeof(int32_t));
	BLOB("contrib", j->contrib.data(), j->contrib.size() * sizeof(int32_t));
#undef BLOB
	*nbytes = 0;
	return nullptr;
}

/* Points the emulated kernels at this job's tables (host memory stands in
 * for device memory), with caller-owned PRNG states and eval counters, and
 * an optional override of the docking parameters. */
int adgpu_ref_job_bind(void* h, const void* dockpars_override, uint32_t* prng_states,
                       int* evals_of_new_entities, int* evals_of_runs)
{
	RefJob* j = (RefJob*)h;
	RefGpuData g;
	memset(&g, 0, sizeof(g));
	g.dockpars = dockpars_override ? *(const RefDockpars*)dockpars_override : j->dockpars;
	g.pKerconst_interintra = &j->interintra;
	g.pKerconst_intracontrib = &j->intracontrib;
	g.pKerconst_intra = &j->intra;
	g.pKerconst_rotlist = &j->rotlist;
	g.pKerconst_conform = &j->conform;
	g.pKerconst_grads = &j->grads;
	g.pMem_fgrids = j->grid.data();
	g.pMem_evals_of_new_entities = evals_of_new_entities;
	g.pMem_gpu_evals_of_runs = evals_of_runs;
	g.pMem_prng_states = prng_states;
	g.pMem_rotbonds_const = j->grads.rotbonds;
	g.pMem_rotbonds_atoms_const = j->grads.rotbonds_atoms;
	g.pMem_num_rotating_atoms_per_rotbond_const = j->grads.num_rotating_atoms_per_rotbond;
	g.warpmask = 31;
	g.warpbits = 5;
	adgpu_ref_set_gpudata(&g);
	return 0;
}

size_t adgpu_ref_sizeof_refgpudata(void) { return sizeof(RefGpuData); }

/* The reference's own map reading (get_gridinfo + get_gridvalues,
 * host/src/processgrid.cpp:28-253) of a .maps.fld; returns the number of
 * floats read (the replicated layout), or -1. */
long adgpu_ref_read_grid(const char* fld_path)
{
	Gridinfo g;
	if (get_gridinfo(fld_path, &g) != 0) return -1;
	if (get_gridvalues(&g) != 0) return -1;
	return (long)g.grids.size();
}

/* One run's Ligandresult fields (host/inc/processresult.h:40-58). */
typedef struct {
	float inter_e, interflex_e, inter_e_elec, intra_e, intraflex_e, rmsd_from_ref, rmsd_from_cluster_center;
	int cluster_id, cluster_subrank, output, run_number;
} adgpu_ref_run_result;

static Dockpars result_pars(const RefJob* j, int num_runs, float rmsd_tol, int symmetry, int clustering, int ncp)
{
	Dockpars mp = j->mypars;
	mp.num_of_runs = num_runs;
	mp.gen_finalpop = false;
	mp.gen_best = false;
	mp.gen_pdbs = 0;
	mp.output_dlg = false;
	mp.output_xml = false;
	mp.contact_analysis = false;
	mp.xml2dlg = false;
	mp.rmsd_tolerance = rmsd_tol;
	mp.handle_symmetry = symmetry != 0;
	mp.calc_clustering = clustering != 0;
	mp.nr_cluster_poses = ncp;
	if (!mp.resname) mp.resname = (char*)"oracle";
	return mp;
}

/* process_result (host/src/processresult.cpp:1312-1363) with every file
 * output switched off: arrange_result + make_resfiles per run, then
 * generate_output's ordering and clustering.  pops/energies are sorted in
 * place as the reference sorts them.  xyz: num_runs*N*3 best-pose
 * coordinates; peratom: num_runs*N*2 (vdW, elec). */
int adgpu_ref_process_result(void* h, float* pops, float* energies, int num_runs, float rmsd_tol, int symmetry,
                             int clustering, int ncp, adgpu_ref_run_result* out, double* xyz, float* peratom)
{
	RefJob* j = (RefJob*)h;
	Dockpars mp = result_pars(j, num_runs, rmsd_tol, symmetry, clustering, ncp);
	const int P = (int)mp.pop_size, N = j->lig_ref->num_of_atoms;
	IntraTables tables(j->lig_ref.get(), mp.coeffs.scaled_AD4_coeff_elec, mp.coeffs.AD4_coeff_desolv, mp.qasp,
	                   mp.nr_mod_atype_pairs, mp.mod_atype_pairs);
	std::vector<Ligandresult> res(num_runs);
	float best_energy_of_all = 1000000000000.0;
	int argc = 1;
	char name[] = "oracle";
	char* argv[] = {name, nullptr};
	for (int r = 0; r < num_runs; r++) {
		float* pr = pops + (size_t)r * P * GENOTYPE_LENGTH_IN_GLOBMEM;
		float* er = energies + (size_t)r * P;
		arrange_result(pr, er, P);
		make_resfiles(pr, er, &tables, j->lig_ref.get(), j->lig_init.get(), j->xray.get(), &mp, 0, 0, &j->gridinfo,
		              &argc, argv, 0, r, best_energy_of_all, &res[r]);
	}
	generate_output(res.data(), num_runs, &tables, j->lig_init.get(), j->xray.get(), &mp, &j->gridinfo, &argc, argv,
	                0.0, 0, 0, 0.0, 0.0);
	for (int r = 0; r < num_runs; r++) {
		const Ligandresult& L = res[r];
		adgpu_ref_run_result& o = out[r];
		o.inter_e = L.interE; o.interflex_e = L.interflexE; o.inter_e_elec = L.interE_elec; o.intra_e = L.intraE;
		o.intraflex_e = L.intraflexE; o.rmsd_from_ref = L.rmsd_from_ref; o.rmsd_from_cluster_center = L.rmsd_from_cluscent;
		o.cluster_id = L.clus_id; o.cluster_subrank = L.clus_subrank; o.output = L.output ? 1 : 0;
		o.run_number = L.run_number;
		for (int a = 0; a < N; a++) {
			if (xyz) for (int k = 0; k < 3; k++) xyz[((size_t)r * N + a) * 3 + k] = L.atom_idxyzq[a][k + 1];
			if (peratom) {
				peratom[((size_t)r * N + a) * 2] = L.peratom_vdw[a];
				peratom[((size_t)r * N + a) * 2 + 1] = L.peratom_elec[a];
			}
		}
	}
	return 0;
}

/* make_resfiles' per-entity body (host/src/processresult.cpp:421-475) for n
 * genotypes, as the final-population report computes it: out[3*i] =
 * intraE + intraflexE, out[3*i+1] = interE + interflexE, out[3*i+2] = RMSD
 * from the input ligand. */
int adgpu_ref_rescore(void* h, const float* genotypes, int n, int symmetry, float* out)
{
	RefJob* j = (RefJob*)h;
	Dockpars mp = result_pars(j, 1, 2.0f, symmetry, 1, 0);
	IntraTables tables(j->lig_ref.get(), mp.coeffs.scaled_AD4_coeff_elec, mp.coeffs.AD4_coeff_desolv, mp.qasp,
	                   mp.nr_mod_atype_pairs, mp.mod_atype_pairs);
	Liganddata* ref = j->lig_ref.get();
	const Liganddata* inp = j->lig_init.get();
	std::unique_ptr<Liganddata> work(new Liganddata(*ref));
	for (int i = 0; i < n; i++) {
		memcpy(work->atom_idxyzq, ref->atom_idxyzq, sizeof(ref->atom_idxyzq));
		change_conform_f(work.get(), &j->gridinfo, genotypes + (size_t)i * GENOTYPE_LENGTH_IN_GLOBMEM, 0);
		float intraflexE = 0, interflexE = 0;
		float interE = calc_interE_f(&j->gridinfo, work.get(), 0.0005, 0, intraflexE);
		scale_ligand(work.get(), j->gridinfo.spacing);
		float intraE = calc_intraE_f(work.get(), 8, mp.smooth, 0, mp.elec_min_distance, &tables, 0, interflexE);
		move_ligand(work.get(), j->gridinfo.origo_real_xyz, j->gridinfo.origo_real_xyz);
		double rmsd = calc_rmsd(inp->atom_idxyzq, work->atom_idxyzq,
		                        (!inp->true_ligand_atoms) ? inp->num_of_atoms : inp->true_ligand_atoms, mp.handle_symmetry);
		out[3 * i] = intraE + intraflexE;
		out[3 * i + 1] = interE + interflexE;
		out[3 * i + 2] = (float)rmsd;
	}
	return 0;
}

}  // extern "C"
