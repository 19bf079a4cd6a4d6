// adgpu_tables.h -- repacking of the reference's per-ligand constant tables
// (kernelconstant_*, host/inc/calcenergy.h:88-136) and grid maps into the
// engine's device layout (LigDev, adgpu_device.cuh).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/adgpu_b200.h"
#include "adgpu_device.cuh"

namespace adgpu {

adgpu_status fail(adgpu_status st, const std::string& msg);
adgpu_status cuda_fail(cudaError_t e, const char* what);

// Host-side packed tables of one ligand (offsets are into `blob`).
struct PackedLigand {
	int natoms = 0, nlig = 0, ngenes = 0, ntors = 0, npairs = 0, ntoritems = 0;
	int npairs2 = 0, ngpairs = 0;     // two-pair records (AD4 pairs), PairRec entries (other exponents)
	std::vector<uint8_t> blob;
	size_t off_atom_xyzq = 0, off_atom_info = 0, off_chain_len = 0, off_chain = 0;
	size_t off_tors_uv = 0, off_tors_mv = 0, off_tors_ends = 0, off_tor_items = 0, off_pairs2 = 0, off_gpairs = 0;
	size_t off_f3_bias = 0;           // per-atom start of the fixed-point forces (LigDev::f3_bias)
	// cost model inputs (algorithmic work per evaluation)
	long rot_ops = 0;     // torsion rotations + general rotations applied per pose
};

// Device copy of a packed ligand plus its relaid-out grid.
struct LigandTables {
	LigDev dev{};
	void* dmem = nullptr;
	size_t dmem_bytes = 0;
	float* dgrid = nullptr;
	size_t dgrid_bytes = 0;
	bool own_grid = true;
	PackedLigand packed;
	LigandTables() = default;
	LigandTables(const LigandTables&) = delete;
	LigandTables& operator=(const LigandTables&) = delete;
	~LigandTables();
	void release();
};

// Builds the packed ligand from host copies of the reference tables.
adgpu_status pack_ligand(const adgpu_dockpars& dp, const adgpu_kc_interintra& ii, const uint32_t* pairs,
                         const adgpu_kc_intra& kin, const int* rotlist, const adgpu_kc_conform& cf,
                         const int* rotbonds, const int* rotbonds_atoms, const int* nrot_per_rotbond,
                         PackedLigand& out);

// Uploads a packed ligand (tables only; grid pointers left unset).
adgpu_status upload_ligand(const PackedLigand& p, LigandTables& t);
// LigDev table pointers for a packed blob already copied to device address dbase.
void place_ligand(const PackedLigand& p, const void* dbase, LigDev& L);

// Fills the grid fields of a LigDev from the dockpars and a cell-record grid.
void set_grid_fields(LigDev& L, const adgpu_dockpars& dp, const float* cell_grid);

// Relays out a reference-layout grid (device memory) into cell records
// (device memory, allocated here; caller frees with cudaFree).
adgpu_status relayout_grid(const float* ref_grid_dev, const adgpu_dockpars& dp, float** out, size_t* out_bytes,
                           cudaStream_t stream);

// Size in bytes of the cell-record grid for these dimensions.
size_t cell_grid_bytes(int gx, int gy, int gz, int num_map_atypes);

// Everything adgpu_set_kernels_gpu_data needs: D2H copy of the tables a
// GpuData points to, repack, upload, grid relayout.
adgpu_status build_ligand_tables_from_device(const adgpu_gpudata& d, LigandTables& t);

}  // namespace adgpu
