// adgpu_prep.h -- the engine's front end: AutoDock-4 inputs to reference-layout tables.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/adgpu_b200.h"

namespace adgpu {

// Grid maps as read from a .maps.fld: values[map][z][y][x] with the type maps
// first and the e and d maps last (the .fld order the reference requires).
struct Grid {
	int dims[3] = {0, 0, 0};
	double spacing = 0.0;
	double origin[3] = {0, 0, 0};
	int num_map_atypes = 0;
	std::vector<std::string> types;
	std::vector<float> values;
};

// What result processing needs beyond the kernel tables, in the precision the
// reference's host scorer and pose builder use (double coordinates and pair
// parameters; host/src/processligand.cpp:1592-1690, 1796-2331): the
// reference orientation, the coordinates as read, the torsion tree and the
// per-type-pair van der Waals parameters.
struct PostLigand {
	int natoms = 0, true_lig_atoms = 0, nrot = 0, ntypes = 0, true_lig_rotbonds = 0;
	double origin[3] = {0, 0, 0};         // grid origin, Angstrom
	double spacing = 0.0;
	std::vector<double> ref_xyz;          // N*3, grid units, reference orientation
	std::vector<double> input_xyz;        // N*3, Angstrom, as read from the PDBQT
	std::vector<double> charge;           // N
	std::vector<int> type;                // N, ligand type index
	std::vector<int> map;                 // N, grid map of the type (-1: none)
	std::vector<uint8_t> ignore_inter;    // N
	std::vector<uint64_t> rot_mask;       // N, bit r: the atom turns with torsion r
	std::vector<double> rot_move, rot_unit;          // NR*3, grid units
	std::vector<double> reqm_AB, vw_A, vw_B, vw_C, vw_D;  // NT*NT
	std::vector<uint8_t> is_hb;           // NT*NT
	std::vector<int> vw_index;            // NT: base type index (atom_types_reqm)
	std::vector<double> solpar, volume;   // NT
};

// A ligand (plus optional flexible residues) prepared for docking: the tables
// prepare_const_fields_for_gpu would produce, the initial population and the
// per-thread LCG seeds of a reference run with the same --seed.
struct Prepared {
	adgpu_dockpars dockpars{};
	adgpu_kc_interintra interintra{};
	std::vector<uint32_t> pairs;       // 2 * num_of_intraE_contributors
	adgpu_kc_intra intra{};
	std::vector<int> rotlist;          // rotbondlist_length entries (64-thread rows)
	adgpu_kc_conform conform{};
	adgpu_kc_grads grads{};
	int num_rotbonds = 0;
	int num_rotcyc = 0;
	std::vector<float> initpop;        // runs * pop_size * 64
	std::vector<uint32_t> prng;        // runs * pop_size * 64
	PostLigand post;
};

}  // namespace adgpu

// The opaque handles of the C ABI.
struct adgpu_grid_s { adgpu::Grid g; };
struct adgpu_ligand_s { adgpu::Prepared p; };

namespace adgpu {

adgpu_status grid_read(const char* fld_path, Grid& g);
adgpu_status grid_save(const Grid& g, const char* path);
adgpu_status grid_load(const char* path, Grid& g);
void grid_reference_layout(const Grid& g, float* out);      // 4 * nmaps * X*Y*Z floats
void grid_cell_records(const Grid& g, float* out);          // (X-1)(Y-1)(Z-1) * nmaps * 8 floats
adgpu_status prepare_ligand(const Grid& grid, const std::string& ligand_text, const std::string& flexres_text,
                            const adgpu_dockpars& run, const uint32_t seed[3], int num_runs, Prepared& out);
void dockpars_defaults(adgpu_dockpars& dp, double spacing, int pop_size);

}  // namespace adgpu
