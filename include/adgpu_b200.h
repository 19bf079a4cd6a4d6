/*
 * adgpu_b200.h -- C ABI of the B200-native AutoDock-GPU LGA hot path.
 *
 * Two layers are declared here:
 *
 *  1. The reference's kernel API, restated as `extern "C"` entry points with
 *     plain pointers.  A host program that today calls AutoDock-GPU's
 *     cuda/kernels.cu API (declared in host/src/performdocking.cpp.Cuda:40-84)
 *     can call these instead, with the same GpuData contents and the same
 *     buffers.  libadgpu_b200 also exports the original C++-linkage names
 *     (SetKernelsGpuData, gpu_calc_initpop, ...) so the reference host objects
 *     link against it unchanged; those wrappers keep the reference's
 *     print-and-exit error convention (cuda/GpuData.h:40-72), while the
 *     adgpu_* entry points below return an adgpu_status instead.
 *
 *  2. A batch/serving API (adgpu_engine_*) with no reference counterpart:
 *     many ligands with uneven atom/torsion counts, each with its own runs,
 *     docked by one persistent launch over device-resident receptor maps.
 *
 * Memory ownership follows the reference: the caller allocates every buffer
 * it passes (device pointers unless stated otherwise); the library owns only
 * the repacked copies of the constant tables and grid that it builds inside
 * adgpu_set_kernels_gpu_data / adgpu_engine_* calls.
 *
 * Layout types below must stay byte-identical to the reference's:
 *   adgpu_dockpars            == GpuDockparameters          (cuda/GpuData.h:74-110)
 *   adgpu_gpudata             == GpuData                    (cuda/GpuData.h:112-136)
 *   adgpu_kc_interintra       == kernelconstant_interintra  (host/inc/calcenergy.h:88-94)
 *   adgpu_kc_intracontrib     == kernelconstant_intracontrib(host/inc/calcenergy.h:96-99)
 *   adgpu_kc_intra            == kernelconstant_intra       (host/inc/calcenergy.h:101-110)
 *   adgpu_kc_rotlist          == kernelconstant_rotlist     (host/inc/calcenergy.h:112-115)
 *   adgpu_kc_conform          == kernelconstant_conform     (host/inc/calcenergy.h:117-122)
 *   adgpu_kc_grads            == kernelconstant_grads       (host/inc/calcenergy.h:124-136)
 * so that a GpuData filled by the reference host program can be handed over
 * as-is.  Limits are the reference's (common/defines.h:83-95).
 */
#ifndef ADGPU_B200_H
#define ADGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADGPU_MAX_ATOMS        256
#define ADGPU_MAX_ATYPES       32
#define ADGPU_MAX_ROTBONDS     57
#define ADGPU_MAX_INTRAE       (ADGPU_MAX_ATOMS * ADGPU_MAX_ATOMS)
#define ADGPU_MAX_ROTATIONS    (ADGPU_MAX_ATOMS * ADGPU_MAX_ROTBONDS)
#define ADGPU_MAX_POPSIZE      2048
#define ADGPU_MAX_RUNS         8192
#define ADGPU_GENOTYPE_STRIDE  64     /* floats per genotype in global memory */
#define ADGPU_MAX_GENES        (ADGPU_MAX_ROTBONDS + 6)

typedef enum {
	ADGPU_OK = 0,
	ADGPU_ERR_ARG = 1,        /* bad argument (null pointer, size out of range) */
	ADGPU_ERR_CUDA = 2,       /* a CUDA runtime call failed; see adgpu_last_error() */
	ADGPU_ERR_NOT_READY = 3,  /* adgpu_set_kernels_gpu_data has not been called */
	ADGPU_ERR_LIMIT = 4,      /* a reference limit (atoms, genes, runs ...) exceeded */
	ADGPU_ERR_BUDGET = 5,     /* request does not fit the engine's memory budget */
	ADGPU_ERR_STATE = 6,      /* call not valid in the object's current state */
	ADGPU_ERR_TIMEOUT = 7     /* a bounded device wait gave up; kernel returned early */
} adgpu_status;

typedef struct {
	int          num_of_atoms;
	int          true_ligand_atoms;
	int          num_of_atypes;
	int          num_of_map_atypes;
	int          num_of_intraE_contributors;
	int          gridsize_x;
	int          gridsize_y;
	int          gridsize_z;
	int          gridsize_x_times_y;
	int          gridsize_x_times_y_times_z;
	float        grid_spacing;
	int          rotbondlist_length;
	float        coeff_elec;
	float        elec_min_distance;
	float        coeff_desolv;
	int          pop_size;
	int          num_of_genes;
	float        tournament_rate;
	float        crossover_rate;
	float        mutation_rate;
	float        abs_max_dmov;
	float        abs_max_dang;
	float        lsearch_rate;
	float        smooth;
	unsigned int num_of_lsentities;
	float        rho_lower_bound;
	float        base_dmov_mul_sqrt3;
	float        base_dang_mul_sqrt3;
	unsigned int cons_limit;
	unsigned int max_num_of_iters;
	float        qasp;
	float        adam_beta1;
	float        adam_beta2;
	float        adam_epsilon;
} adgpu_dockpars;

typedef struct {
	float    atom_charges_const  [ADGPU_MAX_ATOMS];
	uint32_t atom_types_const    [ADGPU_MAX_ATOMS];
	uint32_t atom_types_map_const[ADGPU_MAX_ATOMS];
	char     ignore_inter_const  [ADGPU_MAX_ATOMS];
} adgpu_kc_interintra;

typedef struct {
	uint32_t intraE_contributors_const[2 * ADGPU_MAX_INTRAE];
} adgpu_kc_intracontrib;

typedef struct {
	unsigned int   atom_types_reqm_const[ADGPU_MAX_ATYPES];
	unsigned short VWpars_exp_const     [ADGPU_MAX_ATYPES * ADGPU_MAX_ATYPES];
	float          reqm_AB_const        [ADGPU_MAX_ATYPES * ADGPU_MAX_ATYPES];
	float          VWpars_AC_const      [ADGPU_MAX_ATYPES * ADGPU_MAX_ATYPES];
	float          VWpars_BD_const      [ADGPU_MAX_ATYPES * ADGPU_MAX_ATYPES];
	float          dspars_S_const       [ADGPU_MAX_ATYPES];
	float          dspars_V_const       [ADGPU_MAX_ATYPES];
} adgpu_kc_intra;

typedef struct {
	int rotlist_const[ADGPU_MAX_ROTATIONS];
} adgpu_kc_rotlist;

typedef struct {
	float ref_coords_const             [3 * ADGPU_MAX_ATOMS];
	float rotbonds_moving_vectors_const[3 * ADGPU_MAX_ROTBONDS];
	float rotbonds_unit_vectors_const  [3 * ADGPU_MAX_ROTBONDS];
} adgpu_kc_conform;

typedef struct {
	int rotbonds                      [2 * ADGPU_MAX_ROTBONDS];
	int rotbonds_atoms                [ADGPU_MAX_ATOMS * ADGPU_MAX_ROTBONDS];
	int num_rotating_atoms_per_rotbond[ADGPU_MAX_ROTBONDS];
} adgpu_kc_grads;

/* Rotation-list element bits (common/calcenergy_basic.h:31-36). */
#define ADGPU_RLIST_ATOMID_MASK   0x000000FF
#define ADGPU_RLIST_RBONDID_MASK  0x0000FF00
#define ADGPU_RLIST_RBONDID_SHIFT 8
#define ADGPU_RLIST_FIRSTROT_MASK 0x00010000
#define ADGPU_RLIST_GENROT_MASK   0x00020000
#define ADGPU_RLIST_DUMMY_MASK    0x00040000

typedef struct {
	int                     devnum;
	int                     devid;
	int                     preallocated_gridsize;
	adgpu_dockpars          dockpars;
	adgpu_kc_interintra*    pKerconst_interintra;
	adgpu_kc_intracontrib*  pKerconst_intracontrib;
	adgpu_kc_intra*         pKerconst_intra;
	adgpu_kc_rotlist*       pKerconst_rotlist;
	adgpu_kc_conform*       pKerconst_conform;
	adgpu_kc_grads*         pKerconst_grads;
	float*                  pMem_fgrids;
	int*                    pMem_evals_of_new_entities;
	int*                    pMem_gpu_evals_of_runs;
	uint32_t*               pMem_prng_states;
	int*                    pMem_rotbonds_const;
	int*                    pMem_rotbonds_atoms_const;
	int*                    pMem_num_rotating_atoms_per_rotbond_const;
	unsigned int            warpmask;
	unsigned int            warpbits;
} adgpu_gpudata;

/* ---------------------------------------------------------------------------
 * Layer 1: the reference kernel API.
 *
 * All calls are synchronous like the reference's (its LAUNCHERROR macro
 * synchronises after every launch, cuda/GpuData.h:49-62): results are
 * visible to the host on return.  `threads` is accepted for signature
 * compatibility; it names the reference's block size, which fixes how the
 * per-thread PRNG states in pMem_prng_states are indexed (blockIdx*threads+tid,
 * cuda/auxiliary_genetic.cu:37).  The library reproduces that indexing no
 * matter how many device threads it actually assigns to one pose.
 * ------------------------------------------------------------------------- */

/* Replaces SetKernelsGpuData, cuda/kernels.cu:126-132.  Copies *data (device
 * pointers inside) and builds the library's repacked tables and 8-corner grid
 * from the pointed-to device buffers.  Must be called again whenever those
 * buffers change. */
adgpu_status adgpu_set_kernels_gpu_data(const adgpu_gpudata* data);

/* Replaces GetKernelsGpuData, cuda/kernels.cu:134-139. */
adgpu_status adgpu_get_kernels_gpu_data(adgpu_gpudata* data);

/* Replaces gpu_calc_initpop, cuda/kernel1.cu:57-63.  blocks = runs*pop_size. */
adgpu_status adgpu_calc_initpop(uint32_t blocks, uint32_t threads,
                                float* conformations_current, float* energies_current);

/* Replaces gpu_sum_evals, cuda/kernel2.cu:54-58.  blocks = runs. */
adgpu_status adgpu_sum_evals(uint32_t blocks, uint32_t threads);

/* Replaces gpu_gen_and_eval_newpops, cuda/kernel4.cu:307-318.  blocks = runs*pop_size. */
adgpu_status adgpu_gen_and_eval_newpops(uint32_t blocks, uint32_t threads,
                                        float* conformations_current, float* energies_current,
                                        float* conformations_next, float* energies_next);

/* Replaces gpu_perform_LS (Solis-Wets), cuda/kernel3.cu:311-320.  blocks = runs*num_of_lsentities. */
adgpu_status adgpu_perform_ls(uint32_t blocks, uint32_t threads,
                              float* conformations_next, float* energies_next);

/* Replaces gpu_gradient_minAD (ADADELTA), cuda/kernel_ad.cu:396-405. */
adgpu_status adgpu_gradient_minad(uint32_t blocks, uint32_t threads,
                                  float* conformations_next, float* energies_next);

/* Replaces gpu_gradient_minAdam (ADAM), cuda/kernel_adam.cu:399-408. */
adgpu_status adgpu_gradient_minadam(uint32_t blocks, uint32_t threads,
                                    float* conformations_next, float* energies_next);

/* FIRE local search.  The reference has it only as an OpenCL kernel
 * (gradient_minFire, device/kernel_fire.cl:76-895) launched from
 * host/src/performdocking.cpp.OpenCL; same launch shape as the others. */
adgpu_status adgpu_gradient_minfire(uint32_t blocks, uint32_t threads,
                                    float* conformations_next, float* energies_next);

/* Scores `n` genotypes (stride ADGPU_GENOTYPE_STRIDE floats, device memory)
 * with the energy-only scorer (gpu_calc_energy, cuda/calcenergy.cu:114-453)
 * or, if gradients != NULL, with the merged energy+gradient scorer
 * (gpu_calc_energrad, cuda/calcMergeEneGra.cu:48-900); gradients has the same
 * stride as genotypes.  The reference has no stand-alone entry point for its
 * scorer; this is the unit the per-pose parity tests drive. */
adgpu_status adgpu_score_genotypes(uint32_t n, const float* genotypes,
                                   float* energies, float* gradients);

/* The scorer's energy split into its terms, for n genotypes (device
 * buffers; no reference counterpart, the parity tests' per-term view):
 * energies[n], and terms[8n] per genotype = intermolecular type-map,
 * electrostatic and desolvation energies, intramolecular vdW/H-bond,
 * electrostatic, desolvation and CG-G0 energies, and the number of atoms
 * outside the grid (each adds the 2^24 penalty to the energy only). */
adgpu_status adgpu_score_terms(uint32_t n, const float* genotypes, float* energies, float* terms);

/* The same scoring as adgpu_score_genotypes, for callers that may not
 * allocate device memory: a host whose memory is all handed out by its own
 * pool, or a process with every byte of the device already reserved.  It has
 * no counterpart in the reference.  It takes the reference-layout GpuData
 * directly (adgpu_set_kernels_gpu_data is not needed) and repacks its tables
 * on the device into one fixed 1 MiB device array compiled into the library,
 * reading the grid in the caller's layout; it calls neither cudaMalloc nor
 * cudaFree.  Ligands whose repacked tables exceed 1 MiB (about 30,000
 * intramolecular pairs) are rejected with ADGPU_ERR_LIMIT.  The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress),
 * so make it before any stream capture.  There is one array per device:
 * calls that overlap on the GPU (from several host threads) race on it.
 * Runs on the legacy default stream and returns once its own kernels have
 * finished (it synchronises that stream, not the whole device). */
adgpu_status adgpu_score_genotypes_noalloc(const adgpu_gpudata* data, uint32_t n,
                                           const float* genotypes, float* energies,
                                           float* gradients);

/* Device-resident docking loop for one ligand: the generation loop of
 * docking_with_gpu (host/src/performdocking.cpp.Cuda:684-831) without host
 * round trips.  Runs generations (GA + the LS method `lsmet`: 0 sw, 1 ad,
 * 2 adam, 3 fire) until the mean evaluations per run reach `max_evals` or
 * `max_gens` generations have passed (check_progress,
 * host/src/performdocking.cpp.Cuda:908-942), on the `num_runs` populations
 * already resident in conformations1/energies1 (initpop and sum_evals must
 * have run, as in the reference).  On return the final
 * population is in the buffers reported through *final_is_second (0: 1, 1: 2)
 * and *generations holds the number of generations executed.
 * With a 100 % local-search rate (num_of_lsentities == pop_size, the
 * reference's default) the loop is one persistent launch in which every run
 * starts its next generation as soon as its own local searches end, up to
 * three generations ahead of the stop test; generations run past the stop are
 * discarded, so populations, energies, evaluation counts and the generation
 * count are those of the generation-synchronous loop (only the PRNG states
 * and the per-entity evaluation counters keep the discarded generations'
 * draws).  Otherwise, or with ADGPU_DOCK_PIPELINE=0 in the environment of
 * adgpu_set_kernels_gpu_data, it graph-captures the per-generation launch
 * sequence.  Uses the legacy default stream; returns when the loop has
 * ended. */
adgpu_status adgpu_dock_resident(int lsmet, uint32_t num_runs, uint64_t max_evals, uint32_t max_gens,
                                 float* conformations1, float* energies1,
                                 float* conformations2, float* energies2,
                                 int* final_is_second, uint32_t* generations);

/* adgpu_dock_resident with the reference's AutoStop (--autostop 1,
 * host/inc/autostop.hpp:169-222, applied as in
 * host/src/performdocking.cpp.Cuda:689-698): every `as_frequency`
 * generations (--asfreq) the convergence test runs on the device on the
 * current energies, and the loop ends once it is satisfied (standard
 * deviation of the best energies below `stopstd`, --stopstd) and the total
 * evaluations exceed `min_as_evals` (the reference's heuristics minimum; 0
 * without heuristics).  *autostopped reports whether it triggered.  The
 * reference copies all energies to the host for each test; here nothing
 * leaves the device until the loop ends. */
adgpu_status adgpu_dock_resident_autostop(int lsmet, uint32_t num_runs, uint64_t max_evals, uint32_t max_gens,
                                          uint32_t as_frequency, float stopstd, uint64_t min_as_evals,
                                          float* conformations1, float* energies1,
                                          float* conformations2, float* energies2,
                                          int* final_is_second, uint32_t* generations, int* autostopped);

/* Accounting of the last adgpu_dock_resident call on this process (no
 * counterpart in the reference). */
typedef struct {
	int      pipelined;               /* 1: the pipelined loop ran; 0: the per-generation launches */
	int      threads_per_pose;        /* pipelined loop: threads per pose group */
	int      pose_groups;             /* pipelined loop: pose groups of the launch */
	uint32_t generations;             /* generations run (as reported by the call) */
	uint32_t generations_discarded;   /* most generations any run ran past the stop */
	uint64_t tasks;                   /* GA chunks and local searches executed */
	uint64_t parks;                   /* times a run waited for a stop test before its next generation */
	uint64_t evals_executed;          /* evaluations executed, those of discarded generations included */
	int      buffers;                 /* population buffers (look-ahead + 1 generations) */
	int      pad;
	double   busy_s;                  /* summed time pose groups spent on tasks */
	double   span_s;                  /* first pose group start to last pose group exit */
} adgpu_dock_stats;

adgpu_status adgpu_dock_stats_get(adgpu_dock_stats* out);

/* ---------------------------------------------------------------------------
 * Front end: the input side of the path.  Reads AutoDock-4 grid maps and
 * prepares PDBQT ligands (with optional flexible residues) into the
 * reference-layout tables above, as the reference host does before it calls
 * the kernel API.  Base AD4 atom types only (no derived types or modified
 * pairs).  Host memory throughout.
 * ------------------------------------------------------------------------- */
typedef struct adgpu_grid_s adgpu_grid;
typedef struct adgpu_ligand_s adgpu_ligand;

/* Replaces get_gridinfo + get_gridvalues (host/src/processgrid.cpp:28-253):
 * reads a .maps.fld and its .map files (type maps, then e, then d). */
adgpu_status adgpu_grid_read(const char* fld_path, adgpu_grid** out);

/* Builds a grid from values[map][z][y][x] (num_maps = type maps + e + d,
 * types[] names the type maps followed by "e" and "d"). */
adgpu_status adgpu_grid_from_values(const int dims[3], double spacing, const double origin[3], int num_maps,
                                    const char* const* types, const float* values, adgpu_grid** out);
void adgpu_grid_free(adgpu_grid* grid);

/* Binary grid cache (no reference counterpart; the reference re-reads the
 * text maps for every job, host/src/processgrid.cpp:186-253): the parsed
 * maps written once and loaded with one read. */
adgpu_status adgpu_grid_save(const adgpu_grid* grid, const char* path);
adgpu_status adgpu_grid_load(const char* path, adgpu_grid** out);
adgpu_status adgpu_grid_info(const adgpu_grid* grid, int dims[3], double* spacing, double origin[3], int* num_map_atypes);

/* The grid in the reference's device layout (4 floats per point per map,
 * host/src/processgrid.cpp:244-248); n_floats must be 4*num_maps*X*Y*Z. */
adgpu_status adgpu_grid_reference_layout(const adgpu_grid* grid, float* out, size_t n_floats);

/* Reference defaults for every run parameter (host/inc/getparameters.h:66-145),
 * scaled as docking_with_gpu does (host/src/performdocking.cpp.Cuda:413-463). */
adgpu_status adgpu_dockpars_default(adgpu_dockpars* dp, double spacing, int pop_size);

/* Replaces init_liganddata + parse_liganddata + gen_initpop_and_reflig +
 * prepare_const_fields_for_gpu (host/src/processligand.cpp:40-1322,
 * host/src/getparameters.cpp:2543-2631, host/src/calcenergy.cpp:31-488).
 * ligand_pdbqt / flexres_pdbqt are file contents (either may be NULL, not
 * both); run supplies the run parameters; seed is the reference's --seed
 * triple, so the initial population and LCG states equal the reference's. */
adgpu_status adgpu_ligand_prepare(const adgpu_grid* grid, const char* ligand_pdbqt, const char* flexres_pdbqt,
                                  const adgpu_dockpars* run, const uint32_t seed[3], int num_runs,
                                  adgpu_ligand** out);
void adgpu_ligand_free(adgpu_ligand* lig);

/* adgpu_ligand_prepare for `count` ligands on nthreads host threads (0: all
 * cores); flexres_pdbqt may be NULL (no flexible residues) or hold NULLs;
 * seeds holds 3 words per ligand.  out[i] / status[i] per ligand; returns the
 * first failure's status, or ADGPU_OK when every ligand was prepared.  In
 * the reference each job's setup (files read, tables prepared) runs in the
 * pipeline thread that then docks it (host/src/main.cpp:303-345). */
adgpu_status adgpu_ligand_prepare_batch(const adgpu_grid* grid, const char* const* ligand_pdbqt,
                                        const char* const* flexres_pdbqt, uint32_t count, const adgpu_dockpars* run,
                                        const uint32_t* seeds, int num_runs, int nthreads, adgpu_ligand** out,
                                        adgpu_status* status);

/* Copies the prepared tables out (any pointer may be NULL). */
adgpu_status adgpu_ligand_tables(const adgpu_ligand* lig, adgpu_dockpars* dockpars,
                                 adgpu_kc_interintra* interintra, adgpu_kc_intracontrib* intracontrib,
                                 adgpu_kc_intra* intra, adgpu_kc_rotlist* rotlist,
                                 adgpu_kc_conform* conform, adgpu_kc_grads* grads);

/* Initial population (runs*pop_size*64 floats) and per-thread LCG states
 * (runs*pop_size*64 uint32) of the prepared ligand. */
adgpu_status adgpu_ligand_population(const adgpu_ligand* lig, float* initpop, size_t n_floats,
                                     uint32_t* prng, size_t n_states);

/* ---------------------------------------------------------------------------
 * Result processing: the output side of the path, on the device.  Replaces
 * the computations of process_result (host/src/processresult.cpp:1312-1363):
 * arrange_result (:31-59) orders each run's final population by energy;
 * make_resfiles (:336-531) rebuilds poses from genotypes (change_conform_f,
 * host/src/processligand.cpp:1592-1664), re-scores them with the host
 * scorer (calc_interE_f :1796-2055, calc_intraE_f :2058-2331, with the
 * IntraTables lookup tables, host/inc/processligand.h:324-364) and takes the
 * RMSD from the input ligand (calc_rmsd :1441-1489); generate_output
 * (:655-804) orders the runs by that energy and clusters them by RMSD.  The
 * .dlg/.xml/.pdbqt writing stays with the caller.  Arithmetic follows the
 * reference host code operation by operation (IEEE single and double, no
 * contraction), so the results agree with it to the last bit except where
 * the device's double sin/cos round differently from the host's.
 * ------------------------------------------------------------------------- */
typedef struct {
	float  rmsd_tolerance;       /* --rmstol, Angstrom (2.0) */
	int    handle_symmetry;      /* --hsym (1) */
	int    calc_clustering;      /* --clustering (1) */
	int    nr_cluster_poses;     /* poses output per cluster (>= 0; 0: all) */
	int    free_roaming_ligand;  /* 1 for a ligand (cluster energies without intraE), 0 for flexres only */
	int    rescore_entities;     /* 1: every entity (the final-population report), 0: each run's best only */
	double coeff_tors;           /* AD4 torsional free-energy coefficient (0.2983, unbound model 0) */
} adgpu_result_params;

typedef struct {                 /* one run: its best entity after ordering (Ligandresult) */
	float  inter_e;              /* ligand-receptor (map) energy */
	float  interflex_e;          /* ligand-flexres energy */
	float  inter_e_elec;         /* electrostatic part of inter_e */
	float  intra_e;              /* intramolecular energy */
	float  intraflex_e;          /* flexres-receptor (map) energy */
	float  rmsd_from_ref;        /* from the input ligand, Angstrom */
	float  rmsd_from_cluster_center;
	float  energy;               /* the population energy (scorer) of the run's best entity */
	int    run_number;           /* 1-based */
	int    cluster_id;           /* 1-based; 0 without clustering */
	int    cluster_subrank;      /* 1-based rank inside the cluster */
	int    output;               /* pose is output under nr_cluster_poses */
	int    energy_rank;          /* position of the run in the energy order (0-based) */
} adgpu_run_result;

typedef struct {
	int    size;
	int    best_run;             /* run_number of the cluster's lowest-energy member */
	double best_energy;          /* kcal/mol, with the torsional term */
	double sum_energy;           /* over members; mean = sum_energy / size */
} adgpu_cluster;

adgpu_status adgpu_result_params_default(adgpu_result_params* params);

/* populations (num_runs*pop_size*64 floats) and energies (num_runs*pop_size)
 * are DEVICE buffers holding the final populations; on return each run's
 * entities are ordered by energy in place, as arrange_result leaves them.
 * grid_reference_layout is the DEVICE grid of the kernel API
 * (adgpu_gpudata.pMem_fgrids).  Host outputs: runs[num_runs]; clusters
 * (num_runs entries available) with *num_clusters; best_xyz (may be NULL):
 * num_runs*N*3 doubles, each run's best pose in Angstrom; peratom (may be
 * NULL): num_runs*N*2 floats (vdW + desolvation, elec) of each best pose, as
 * make_resfiles reports them per atom; entities (may be
 * NULL; needs rescore_entities): num_runs*pop_size*3 floats (intra, inter
 * and RMSD of every entity, as the final-population report prints them). */
adgpu_status adgpu_process_result(const adgpu_ligand* lig, const float* grid_reference_layout,
                                  float* populations, float* energies, uint32_t num_runs,
                                  const adgpu_result_params* params, adgpu_run_result* runs,
                                  adgpu_cluster* clusters, int* num_clusters,
                                  double* best_xyz, float* peratom, float* entities);

/* ---------------------------------------------------------------------------
 * Layer 2: batch / serving engine (no counterpart in the reference, which
 * docks one ligand at a time through the layer-1 API).
 *
 * Receptor maps stay resident; each submitted request (a prepared ligand
 * with its runs) keeps its populations, energies, eval counters and PRNG
 * states on the device until its result is taken.  adgpu_engine_tick
 * advances every admitted run by up to gens_per_tick generations, or until
 * tick_ms has passed, in one persistent launch per local-search method whose
 * pose groups take tasks (one entity of a run's generation: its GA step and
 * its local search) from the runs' own counters, least advanced run first
 * (or, with priority 1, the oldest request's runs first);
 * between ticks requests can be submitted and results taken (continuous
 * batching).  Each run stops on its own budget (evals >=
 * max_evals or generations >= max_gens), so a request's result does not
 * depend on what else is running or on where ticks end.
 * ------------------------------------------------------------------------- */
typedef struct adgpu_engine_s adgpu_engine;

typedef struct {
	size_t memory_budget_bytes;  /* device bytes for receptors + requests; 0: 80% of free memory */
	int    threads_per_pose;     /* 32, 64 or 128; 0: 32; -1: tuned per ligand size class */
	int    gens_per_tick;        /* generations per tick; <= 0: run every admitted run to completion */
	int    device;               /* CUDA device ordinal */
	float  tick_ms;              /* > 0: a tick also ends after this long: no pose group takes a new task after it */
	float  idle_timeout_ms;      /* a pose group that finds no task for this long while runs are active ends
	                                the tick with ADGPU_ERR_TIMEOUT; 0: 2000 */
	int    priority;             /* which run a free pose group serves: 0 the least advanced run (a batch
	                                finishes together); 1 a run of the oldest admitted request, least
	                                advanced first among its runs (a stream: requests finish in order,
	                                lower latency); results are the same either way */
} adgpu_engine_config;

typedef struct {
	int      receptor;           /* id from adgpu_engine_add_receptor */
	int      lsmet;              /* 0 sw, 1 ad, 2 adam, 3 fire */
	uint64_t max_evals;          /* evaluations per run */
	uint32_t max_gens;           /* generations per run; 0: unlimited */
} adgpu_request_params;

typedef struct {
	uint64_t submitted, completed, cancelled, ticks;
	size_t   bytes_used, bytes_budget;
	int      active;
	/* Worker accounting over all ticks: time pose groups spent on tasks, and
	 * pose groups x (first worker start .. last worker exit) per class and
	 * tick; busy / span is the engine kernel's worker utilisation. */
	double   worker_busy_s, worker_span_s;
	uint64_t tasks;
	double   kernel_s;                /* device time of the engine launches (CUDA events) */
} adgpu_engine_stats;

adgpu_status adgpu_engine_create(const adgpu_engine_config* cfg, adgpu_engine** out);
void adgpu_engine_destroy(adgpu_engine* engine);
/* Uploads a receptor's maps once (8-corner cell records); returns its id. */
adgpu_status adgpu_engine_add_receptor(adgpu_engine* engine, const adgpu_grid* grid, int* receptor_id);
/* Admits a request; ADGPU_ERR_BUDGET when its device state does not fit now
 * (retry after taking results).  The ligand must have been prepared against
 * a grid equal to the receptor's, with num_runs > 0. */
adgpu_status adgpu_engine_submit(adgpu_engine* engine, const adgpu_ligand* ligand, const adgpu_request_params* params,
                                 uint64_t* request_id);
/* One engine step (see above); *completed = requests finished in it. */
adgpu_status adgpu_engine_tick(adgpu_engine* engine, int* completed);
/* Ticks until every admitted request has finished. */
adgpu_status adgpu_engine_run(adgpu_engine* engine);
adgpu_status adgpu_engine_poll(adgpu_engine* engine, uint64_t request_id, int* done);
/* Drops a request between ticks, finished or not, and frees its device
 * state (no result is kept). */
adgpu_status adgpu_engine_cancel(adgpu_engine* engine, uint64_t request_id);
/* Failure injection for tests: every run of the request stops handing out
 * tasks, as if all of its open phase had been taken by pose groups that never
 * finish, so the next tick's pose groups find nothing to do while the runs
 * stay active and the tick returns ADGPU_ERR_TIMEOUT after idle_timeout_ms
 * (the device-side wait limit at work).  adgpu_engine_cancel clears it. */
adgpu_status adgpu_engine_inject_stall(adgpu_engine* engine, uint64_t request_id);
/* Result of a finished request (any output may be NULL): best energy and
 * genotype of each run's final population, evals and generations per run,
 * submit-to-finish latency.  Frees the request's device state. */
adgpu_status adgpu_engine_result(adgpu_engine* engine, uint64_t request_id, float* best_energies,
                                 float* best_genotypes, int* evals, uint32_t* generations, double* latency_s);
/* adgpu_process_result on a finished request's final populations (call it
 * before adgpu_engine_result, which frees them); the request's ligand and
 * the receptor's resident maps are used.  final_population (runs*pop*64
 * floats) and final_energies (runs*pop), host, may be NULL: the populations
 * ordered as arrange_result leaves them. */
adgpu_status adgpu_engine_process_result(adgpu_engine* engine, uint64_t request_id, const adgpu_result_params* params,
                                         adgpu_run_result* runs, adgpu_cluster* clusters, int* num_clusters,
                                         double* best_xyz, float* peratom, float* entities, float* final_population,
                                         float* final_energies);
adgpu_status adgpu_engine_stats_get(adgpu_engine* engine, adgpu_engine_stats* out);
/* Threads per pose the engine chose for a request, and its run count. */
adgpu_status adgpu_engine_request_info(adgpu_engine* engine, uint64_t request_id, int* threads_per_pose, int* runs);

/* Text of the last error recorded on this thread (never NULL). */
const char* adgpu_last_error(void);

/* Library version string. */
const char* adgpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ADGPU_B200_H */
