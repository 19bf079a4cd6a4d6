// adgpu_tables.cu -- repacking of the reference's per-ligand tables into the
// engine's device layout, and the grid relayout.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <algorithm>
#include "adgpu_tables.h"
#include <vector>

namespace adgpu {

__global__ void relayout_grid_kernel(const float* __restrict__ ref, float* __restrict__ out,
                                     int gx, int gy, int gz, int nmaps, int num_map_atypes);

LigandTables::~LigandTables() { release(); }

void LigandTables::release()
{
	if (dmem) cudaFree(dmem);
	if (dgrid && own_grid) cudaFree(dgrid);
	dmem = nullptr; dgrid = nullptr; dmem_bytes = 0; dgrid_bytes = 0;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

size_t cell_grid_bytes(int gx, int gy, int gz, int num_map_atypes)
{
	return (size_t)(gx - 1) * (gy - 1) * (gz - 1) * (size_t)(num_map_atypes + 2) * 8 * sizeof(float);
}

// Couples of pairs for the scorer's pair loop.  A thread takes two pairs per
// step from one record: pair A, of an aligned group of 32 (one warp
// instruction), and pair B, of the next group.  When both pairs share their
// first atom, that atom's force from the two is summed in registers and added
// with one set of shared-memory atomics instead of two, and its position is
// loaded once.  Pairs are coupled at shared atoms: each atom, lowest degree
// first, couples its still-uncoupled pairs two by two (a pair's orientation is
// free: its terms do not depend on it and the force update is antisymmetric,
// x1 - x2 = -(x2 - x1) with symmetric fixed-point rounding); a pair left over
// gets an empty partner (both atoms the same, zero coefficients).
struct Couple { uint32_t c; int a, b; };   // shared atom; pair indices (b < 0: empty)

static uint32_t partner(const uint32_t* pairs, int p, uint32_t c)
{
	return pairs[2 * p] == c ? pairs[2 * p + 1] : pairs[2 * p];
}

static void couple_pairs(const uint32_t* pairs, int Q, int N, std::vector<Couple>& out)
{
	out.clear();
	std::vector<std::vector<int>> inc(N);
	for (int p = 0; p < Q; p++) { inc[pairs[2 * p]].push_back(p); inc[pairs[2 * p + 1]].push_back(p); }
	std::vector<int> order(N);
	for (int v = 0; v < N; v++) order[v] = v;
	std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return inc[x].size() < inc[y].size(); });
	std::vector<uint8_t> used(Q, 0);
	for (int v : order) {
		int pending = -1;
		for (int p : inc[v]) {
			if (used[p]) continue;
			if (pending < 0) { pending = p; continue; }
			out.push_back({(uint32_t)v, pending, p});
			used[pending] = used[p] = 1;
			pending = -1;
		}
	}
	for (int p = 0; p < Q; p++)
		if (!used[p]) out.push_back({pairs[2 * p], p, -1});
}

// Slots of the couples: one record per couple, records in blocks of 32 (a
// warp's step).  Couples sorted by the bank of their shared atom are dealt
// round-robin over the blocks, which spreads every bank's couples evenly;
// then within each block a couple swaps its A and B pairs while that lowers
// the largest bank count of the A partners plus that of the B partners (the
// shared atoms' atomics are one instruction per block, the partners' two).
static void order_couples(const uint32_t* pairs, std::vector<Couple>& cs, std::vector<uint32_t>& pos)
{
	const int n = (int)cs.size();
	pos.assign(n, 0);
	if (n == 0) return;
	std::vector<int> idx(n);
	for (int i = 0; i < n; i++) idx[i] = i;
	std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return (cs[x].c & 31) < (cs[y].c & 31); });
	const int G = (n + 31) / 32;
	std::vector<std::vector<int>> blocks(G);
	int g = 0;
	for (int i : idx) {
		while ((int)blocks[g].size() >= (g == G - 1 ? n - 32 * (G - 1) : 32)) g = (g + 1) % G;
		blocks[g].push_back(i);
		g = (g + 1) % G;
	}
	auto pb = [&](const Couple& c, bool first) {
		const int p = first ? c.a : c.b;
		return (int)((p < 0 ? c.c : partner(pairs, p, c.c)) & 31);
	};
	auto cost = [&](const std::vector<int>& blk) {
		int ca[32] = {0}, cb[32] = {0}, ma = 0, mb = 0;
		for (int i : blk) {
			ma = std::max(ma, ++ca[pb(cs[i], true)]);
			mb = std::max(mb, ++cb[pb(cs[i], false)]);
		}
		return ma + mb;
	};
	for (int gi = 0; gi < G; gi++) {
		std::vector<int>& blk = blocks[gi];
		int best = cost(blk);
		for (int pass = 0; pass < 4; pass++) {
			bool improved = false;
			for (int i : blk) {
				std::swap(cs[i].a, cs[i].b);
				const int c = cost(blk);
				if (c < best) { best = c; improved = true; }
				else std::swap(cs[i].a, cs[i].b);
			}
			if (!improved) break;
		}
		for (size_t k = 0; k < blk.size(); k++) pos[blk[k]] = (uint32_t)(32 * gi + k);
	}
}

adgpu_status pack_ligand(const adgpu_dockpars& dp, const adgpu_kc_interintra& ii, const uint32_t* pairs,
                         const adgpu_kc_intra& kin, const int* rotlist, const adgpu_kc_conform& cf,
                         const int* rotbonds, const int* rotbonds_atoms, const int* nrot, PackedLigand& out)
{
	const int N = dp.num_of_atoms, NG = dp.num_of_genes, NT = NG - 6, Q = dp.num_of_intraE_contributors;
	if (N <= 0 || N > ADGPU_MAX_ATOMS) return fail(ADGPU_ERR_LIMIT, "num_of_atoms out of range 1..256");
	if (NG < 6 || NG > ADGPU_MAX_GENES) return fail(ADGPU_ERR_LIMIT, "num_of_genes out of range 6..63");
	if (dp.true_ligand_atoms < 0 || dp.true_ligand_atoms > N) return fail(ADGPU_ERR_ARG, "true_ligand_atoms out of range");
	if (Q < 0 || Q > ADGPU_MAX_INTRAE) return fail(ADGPU_ERR_LIMIT, "num_of_intraE_contributors out of range");
	if (dp.num_of_atypes <= 0 || dp.num_of_atypes > ADGPU_MAX_ATYPES) return fail(ADGPU_ERR_LIMIT, "num_of_atypes out of range");
	if (dp.rotbondlist_length < 0 || dp.rotbondlist_length > ADGPU_MAX_ROTATIONS) return fail(ADGPU_ERR_LIMIT, "rotbondlist_length out of range");
	if (dp.num_of_map_atypes <= 0 || dp.num_of_map_atypes + 2 > 255) return fail(ADGPU_ERR_LIMIT, "num_of_map_atypes out of range");
	out = PackedLigand();
	out.natoms = N; out.nlig = dp.true_ligand_atoms; out.ngenes = NG; out.ntors = NT; out.npairs = Q;

	// per-atom rotation chains from the rotation list: every non-dummy entry of
	// atom a, in list order (host/src/calcenergy.cpp:387-488 orders them
	// torsions first, the general rotation last)
	std::vector<std::vector<uint8_t>> chains(N);
	std::vector<bool> genrot(N, false);
	for (int k = 0; k < dp.rotbondlist_length; k++) {
		int el = rotlist[k];
		if (el & ADGPU_RLIST_DUMMY_MASK) continue;
		int a = el & ADGPU_RLIST_ATOMID_MASK;
		if (a >= N) return fail(ADGPU_ERR_ARG, "rotation list names an atom beyond num_of_atoms");
		if (el & ADGPU_RLIST_GENROT_MASK) {
			if (genrot[a]) return fail(ADGPU_ERR_ARG, "rotation list applies the general rotation twice");
			genrot[a] = true;
		} else {
			if (genrot[a]) return fail(ADGPU_ERR_ARG, "rotation list rotates an atom about a torsion after the general rotation");
			int rb = (el & ADGPU_RLIST_RBONDID_MASK) >> ADGPU_RLIST_RBONDID_SHIFT;
			if (rb >= NT) return fail(ADGPU_ERR_ARG, "rotation list names a torsion beyond num_of_genes-6");
			chains[a].push_back((uint8_t)rb);
		}
	}
	// torsion items
	std::vector<uint32_t> items;
	for (int k = 0; k < NT; k++) {
		if (nrot[k] < 0 || nrot[k] > N) return fail(ADGPU_ERR_ARG, "num_rotating_atoms_per_rotbond out of range");
		if (rotbonds[2 * k] < 0 || rotbonds[2 * k] >= N || rotbonds[2 * k + 1] < 0 || rotbonds[2 * k + 1] >= N)
			return fail(ADGPU_ERR_ARG, "rotbond atom out of range");
		for (int c = 0; c < nrot[k]; c++) {
			int la = rotbonds_atoms[ADGPU_MAX_ATOMS * k + c];
			if (la < 0 || la >= N) return fail(ADGPU_ERR_ARG, "rotating atom out of range");
			items.push_back(((uint32_t)k << 8) | (uint32_t)la);
		}
	}
	out.ntoritems = (int)items.size();
	size_t nchain = 0;
	for (auto& c : chains) nchain += c.size();
	if (nchain > 65535) return fail(ADGPU_ERR_LIMIT, "rotation chains too long");

	// layout of the blob
	size_t o = 0;
	out.off_atom_xyzq = o; o = align_up(o + (size_t)N * 16, 16);
	out.off_atom_info = o; o = align_up(o + (size_t)N * 4, 16);
	out.off_chain_len = o; o = align_up(o + (size_t)N, 16);
	out.off_chain = o; o = align_up(o + std::max<size_t>(nchain, 1), 16);
	out.off_tors_uv = o; o = align_up(o + (size_t)std::max(NT, 1) * 16, 16);
	out.off_tors_mv = o; o = align_up(o + (size_t)std::max(NT, 1) * 16, 16);
	out.off_tors_ends = o; o = align_up(o + (size_t)std::max(NT, 1) * 8, 16);
	out.off_tor_items = o; o = align_up(o + std::max<size_t>(items.size(), 1) * 4, 16);
	// intramolecular pairs: the AD4 ones (m = 12, n = 6 or 10) into
	// two-pair records (pair2_set), the others (modified pair potentials) one to a PairRec
	const int nat = dp.num_of_atypes;
	std::vector<uint32_t> std_pairs;          // (a1, a2) of the AD4 pairs
	std::vector<int> std_idx, gen_idx;        // their indices in the reference's list
	for (int p = 0; p < Q; p++) {
		uint32_t a1 = pairs[2 * p], a2 = pairs[2 * p + 1];
		if (a1 >= (uint32_t)N || a2 >= (uint32_t)N) return fail(ADGPU_ERR_ARG, "intramolecular pair atom out of range");
		uint32_t t1 = ii.atom_types_const[a1], t2 = ii.atom_types_const[a2];
		if (t1 >= (uint32_t)nat || t2 >= (uint32_t)nat) return fail(ADGPU_ERR_ARG, "atom type out of range");
		unsigned short exps = kin.VWpars_exp_const[t1 * (uint32_t)nat + t2];
		uint32_t m = (exps & 0xFF00) >> 8, n = exps & 0xFF;
		if (m == 12 && (n == 6 || n == 10)) {
			std_idx.push_back(p);
			std_pairs.push_back(a1);
			std_pairs.push_back(a2);
		} else {
			gen_idx.push_back(p);
		}
	}
	const int Qs = (int)std_idx.size(), Qg = (int)gen_idx.size();
	std::vector<Couple> couples;
	couple_pairs(std_pairs.data(), Qs, N, couples);
	out.npairs2 = (int)(couples.size() + 31) / 32 * 32;
	out.ngpairs = Qg;
	out.off_pairs2 = o; o = align_up(o + (size_t)std::max(out.npairs2, 1) * 64, 16);
	out.off_gpairs = o; o = align_up(o + (size_t)std::max(Qg, 1) * sizeof(PairRec), 16);
	out.off_f3_bias = o; o = align_up(o + (size_t)N * 4, 16);
	out.blob.assign(o, 0);
	uint8_t* B = out.blob.data();

	float4* xyzq = reinterpret_cast<float4*>(B + out.off_atom_xyzq);
	uint32_t* info = reinterpret_cast<uint32_t*>(B + out.off_atom_info);
	uint8_t* clen = B + out.off_chain_len;
	uint8_t* chain = B + out.off_chain;
	size_t cpos = 0;
	for (int a = 0; a < N; a++) {
		xyzq[a] = make_float4(cf.ref_coords_const[3 * a], cf.ref_coords_const[3 * a + 1], cf.ref_coords_const[3 * a + 2],
		                      ii.atom_charges_const[a]);
		uint32_t mt = ii.atom_types_map_const[a];
		bool ignore = ii.ignore_inter_const[a] > 0;
		if (!ignore && mt >= (uint32_t)dp.num_of_map_atypes) return fail(ADGPU_ERR_ARG, "atom map type out of range");
		uint32_t slot = ignore ? 0u : (2u + mt);
		info[a] = slot | (ignore ? 0x100u : 0u) | (genrot[a] ? 0x200u : 0u) | ((uint32_t)cpos << 16);
		clen[a] = (uint8_t)chains[a].size();
		for (uint8_t k : chains[a]) chain[cpos++] = k;
		out.rot_ops += (long)chains[a].size() + (genrot[a] && a < dp.true_ligand_atoms ? 1 : 0);
		if (ii.atom_types_const[a] >= (uint32_t)dp.num_of_atypes) return fail(ADGPU_ERR_ARG, "atom type out of range");
	}
	float4* uv = reinterpret_cast<float4*>(B + out.off_tors_uv);
	float4* mv = reinterpret_cast<float4*>(B + out.off_tors_mv);
	int2* ends = reinterpret_cast<int2*>(B + out.off_tors_ends);
	for (int k = 0; k < NT; k++) {
		uv[k] = make_float4(cf.rotbonds_unit_vectors_const[3 * k], cf.rotbonds_unit_vectors_const[3 * k + 1], cf.rotbonds_unit_vectors_const[3 * k + 2], 0.f);
		mv[k] = make_float4(cf.rotbonds_moving_vectors_const[3 * k], cf.rotbonds_moving_vectors_const[3 * k + 1], cf.rotbonds_moving_vectors_const[3 * k + 2], 0.f);
		ends[k] = make_int2(rotbonds[2 * k], rotbonds[2 * k + 1]);
	}
	// torsion items in warp-interleaved order (interleave_pos), pairs in
	// couples sharing their first atom, in bank-spread blocks (order_couples)
	uint32_t* it_out = reinterpret_cast<uint32_t*>(B + out.off_tor_items);
	for (size_t i = 0; i < items.size(); i++) it_out[interleave_pos((uint32_t)i, (uint32_t)items.size())] = items[i];
	// pair terms in the reference's operand order: desolvation prefactor,
	// Coulomb factor; G = 50 for CG-G0 pairs (ATYPE_CG_IDX 24 / ATYPE_G0_IDX 25)
	auto fields = [&](int p, float& ac, float& bd, float& reqm, float& dsolv_pref, float& qq, float& vbond) {
		uint32_t a1 = pairs[2 * p], a2 = pairs[2 * p + 1];
		uint32_t t1 = ii.atom_types_const[a1], t2 = ii.atom_types_const[a2];
		uint32_t idx = t1 * (uint32_t)nat + t2;
		uint32_t h1 = kin.atom_types_reqm_const[t1], h2 = kin.atom_types_reqm_const[t2];
		bool cgg0 = (h1 == 24 && h2 == 25) || (h1 == 25 && h2 == 24);
		float q1 = ii.atom_charges_const[a1], q2 = ii.atom_charges_const[a2];
		ac = kin.VWpars_AC_const[idx];
		bd = kin.VWpars_BD_const[idx];
		reqm = kin.reqm_AB_const[idx];
		dsolv_pref = (kin.dspars_S_const[t1] + dp.qasp * std::fabs(q1)) * kin.dspars_V_const[t2] +
		             (kin.dspars_S_const[t2] + dp.qasp * std::fabs(q2)) * kin.dspars_V_const[t1];
		qq = dp.coeff_elec * q1 * q2;
		vbond = cgg0 ? 50.0f : 0.0f;
	};
	float4* pr2 = reinterpret_cast<float4*>(B + out.off_pairs2);
	for (int r = 0; r < out.npairs2; r++) pair2_pad(pr2, (uint32_t)r, (uint32_t)N);
	std::vector<uint32_t> slot;
	order_couples(std_pairs.data(), couples, slot);
	for (size_t k = 0; k < couples.size(); k++) {
		const Couple& cp = couples[k];
		for (uint32_t h = 0; h < 2; h++) {
			const int q = h ? cp.b : cp.a;                 // index into the AD4 list
			if (q < 0) {
				pair2_set(pr2, slot[k], h, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, cp.c | (cp.c << 8));
				continue;
			}
			const int p = std_idx[q];
			const uint32_t a1 = pairs[2 * p], a2 = pairs[2 * p + 1];
			const uint32_t n = kin.VWpars_exp_const[ii.atom_types_const[a1] * (uint32_t)nat + ii.atom_types_const[a2]] & 0xFF;
			float ac, bd, reqm, dsp, qq, vb;
			fields(p, ac, bd, reqm, dsp, qq, vb);
			pair2_set(pr2, slot[k], h, ac, n == 6 ? bd : 0.0f, n == 10 ? bd : 0.0f, reqm, dp.coeff_desolv * dsp, qq, vb,
			          cp.c | (partner(std_pairs.data(), q, cp.c) << 8));
		}
	}
	// couple_force adds kRoundBits (mod 2^32) for each record's second atoms
	// and subtracts it twice for the shared atom, padding included: each atom
	// starts at minus the sum over the records as the kernel reads them
	std::vector<int32_t> offsets(N, 0);
	for (int r = 0; r < out.npairs2; r++) {
		const float4 q3 = pr2[pair2_quad((uint32_t)r, 3)];
		uint32_t ija, ijb;
		std::memcpy(&ija, &q3.z, 4);
		std::memcpy(&ijb, &q3.w, 4);
		offsets[ija & 0xFFu] -= 2;
		offsets[ija >> 8] += 1;
		offsets[ijb >> 8] += 1;
	}
	int32_t* f3b = reinterpret_cast<int32_t*>(B + out.off_f3_bias);
	for (int a = 0; a < N; a++) {
		const uint32_t v = 0u - (uint32_t)offsets[a] * kRoundBits;
		std::memcpy(&f3b[a], &v, 4);
	}
	PairRec* gpr = reinterpret_cast<PairRec*>(B + out.off_gpairs);
	for (int i = 0; i < Qg; i++) {
		const int p = gen_idx[i];
		uint32_t a1 = pairs[2 * p], a2 = pairs[2 * p + 1];
		unsigned short exps = kin.VWpars_exp_const[ii.atom_types_const[a1] * (uint32_t)nat + ii.atom_types_const[a2]];
		uint32_t m = (exps & 0xFF00) >> 8, n = exps & 0xFF;
		PairRec r;
		fields(p, r.ac, r.bd, r.reqm, r.dsolv_pref, r.qq, r.vbond);
		r.ij = a1 | (a2 << 8) | (m << 16) | (n << 24);
		r.pad = 0;
		gpr[i] = r;
	}
	return ADGPU_OK;
}

adgpu_status upload_ligand(const PackedLigand& p, LigandTables& t)
{
	if (t.dmem && t.dmem_bytes < p.blob.size()) { cudaFree(t.dmem); t.dmem = nullptr; t.dmem_bytes = 0; }
	if (!t.dmem) {
		cudaError_t e = cudaMalloc(&t.dmem, p.blob.size());
		if (e != cudaSuccess) return cuda_fail(e, "ligand tables");
		t.dmem_bytes = p.blob.size();
	}
	cudaError_t e = cudaMemcpy(t.dmem, p.blob.data(), p.blob.size(), cudaMemcpyHostToDevice);
	if (e != cudaSuccess) return cuda_fail(e, "ligand tables upload");
	place_ligand(p, t.dmem, t.dev);
	t.packed = p;
	return ADGPU_OK;
}

void place_ligand(const PackedLigand& p, const void* dbase, LigDev& L)
{
	const uint8_t* D = static_cast<const uint8_t*>(dbase);
	L.natoms = p.natoms; L.nlig = p.nlig; L.ngenes = p.ngenes; L.ntors = p.ntors; L.npairs = p.npairs; L.ntoritems = p.ntoritems;
	L.atom_xyzq = reinterpret_cast<const float4*>(D + p.off_atom_xyzq);
	L.atom_info = reinterpret_cast<const uint32_t*>(D + p.off_atom_info);
	L.chain_len = D + p.off_chain_len;
	L.chain = D + p.off_chain;
	L.tors_uv = reinterpret_cast<const float4*>(D + p.off_tors_uv);
	L.tors_mv = reinterpret_cast<const float4*>(D + p.off_tors_mv);
	L.tors_ends = reinterpret_cast<const int2*>(D + p.off_tors_ends);
	L.tor_items = reinterpret_cast<const uint32_t*>(D + p.off_tor_items);
	L.npairs2 = p.npairs2; L.ngpairs = p.ngpairs;
	L.coupled = 1;
	L.pairs2 = reinterpret_cast<const float4*>(D + p.off_pairs2);
	L.gpairs = reinterpret_cast<const PairRec*>(D + p.off_gpairs);
	L.f3_bias = reinterpret_cast<const int*>(D + p.off_f3_bias);
}

void set_grid_fields(LigDev& L, const adgpu_dockpars& dp, const float* cell_grid)
{
	L.map_e = 0;
	L.gx = dp.gridsize_x; L.gy = dp.gridsize_y; L.gz = dp.gridsize_z;
	L.cells_x = dp.gridsize_x - 1;
	L.cells_xy = (dp.gridsize_x - 1) * (dp.gridsize_y - 1);
	L.rec_floats = 8 * (dp.num_of_map_atypes + 2);
	L.spacing = dp.grid_spacing;
	L.inv_spacing = 1.0f / dp.grid_spacing;
	L.coeff_desolv = dp.coeff_desolv;
	L.elec_min_distance = dp.elec_min_distance;
	L.half_smooth = 0.5f * dp.smooth;
	L.grid = cell_grid;
}

adgpu_status relayout_grid(const float* ref_grid_dev, const adgpu_dockpars& dp, float** out, size_t* out_bytes, cudaStream_t stream)
{
	if (dp.gridsize_x < 2 || dp.gridsize_y < 2 || dp.gridsize_z < 2 || dp.gridsize_x > 256 || dp.gridsize_y > 256 || dp.gridsize_z > 256)
		return fail(ADGPU_ERR_LIMIT, "grid dimensions out of range 2..256");
	size_t bytes = cell_grid_bytes(dp.gridsize_x, dp.gridsize_y, dp.gridsize_z, dp.num_of_map_atypes);
	if (*out == nullptr || *out_bytes < bytes) {
		if (*out) cudaFree(*out);
		*out = nullptr;
		cudaError_t e = cudaMalloc(out, bytes);
		if (e != cudaSuccess) return cuda_fail(e, "cell grid");
		*out_bytes = bytes;
	}
	int nmaps = dp.num_of_map_atypes + 2;
	relayout_grid_kernel<<<148 * 8, 256, 0, stream>>>(ref_grid_dev, *out, dp.gridsize_x, dp.gridsize_y, dp.gridsize_z, nmaps, dp.num_of_map_atypes);
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "grid relayout launch");
	return ADGPU_OK;
}

adgpu_status build_ligand_tables_from_device(const adgpu_gpudata& d, LigandTables& t)
{
	const adgpu_dockpars& dp = d.dockpars;
	if (!d.pKerconst_interintra || !d.pKerconst_intracontrib || !d.pKerconst_intra || !d.pKerconst_rotlist ||
	    !d.pKerconst_conform || !d.pMem_fgrids || !d.pMem_rotbonds_const || !d.pMem_rotbonds_atoms_const ||
	    !d.pMem_num_rotating_atoms_per_rotbond_const)
		return fail(ADGPU_ERR_ARG, "GpuData has a null table pointer");
	if (dp.num_of_intraE_contributors < 0 || dp.num_of_intraE_contributors > ADGPU_MAX_INTRAE ||
	    dp.rotbondlist_length < 0 || dp.rotbondlist_length > ADGPU_MAX_ROTATIONS)
		return fail(ADGPU_ERR_LIMIT, "table sizes out of range");
	adgpu_kc_interintra ii;
	adgpu_kc_intra kin;
	adgpu_kc_conform cf;
	std::vector<uint32_t> pairs(2 * (size_t)std::max(dp.num_of_intraE_contributors, 1));
	std::vector<int> rotlist(std::max(dp.rotbondlist_length, 1));
	std::vector<int> rb(2 * ADGPU_MAX_ROTBONDS), rba((size_t)ADGPU_MAX_ATOMS * ADGPU_MAX_ROTBONDS), nrot(ADGPU_MAX_ROTBONDS);
	struct { void* dst; const void* src; size_t n; } cps[] = {
		{&ii, d.pKerconst_interintra, sizeof(ii)},
		{&kin, d.pKerconst_intra, sizeof(kin)},
		{&cf, d.pKerconst_conform, sizeof(cf)},
		{pairs.data(), d.pKerconst_intracontrib, 2 * (size_t)dp.num_of_intraE_contributors * 4},
		{rotlist.data(), d.pKerconst_rotlist, (size_t)dp.rotbondlist_length * 4},
		{rb.data(), d.pMem_rotbonds_const, rb.size() * 4},
		{rba.data(), d.pMem_rotbonds_atoms_const, rba.size() * 4},
		{nrot.data(), d.pMem_num_rotating_atoms_per_rotbond_const, nrot.size() * 4},
	};
	for (auto& c : cps) {
		if (c.n == 0) continue;
		cudaError_t e = cudaMemcpy(c.dst, c.src, c.n, cudaMemcpyDeviceToHost);
		if (e != cudaSuccess) return cuda_fail(e, "reading GpuData tables");
	}
	PackedLigand p;
	adgpu_status st = pack_ligand(dp, ii, pairs.data(), kin, rotlist.data(), cf, rb.data(), rba.data(), nrot.data(), p);
	if (st != ADGPU_OK) return st;
	st = upload_ligand(p, t);
	if (st != ADGPU_OK) return st;
	t.own_grid = true;
	st = relayout_grid(d.pMem_fgrids, dp, &t.dgrid, &t.dgrid_bytes, 0);
	if (st != ADGPU_OK) return st;
	cudaError_t e = cudaDeviceSynchronize();
	if (e != cudaSuccess) return cuda_fail(e, "grid relayout");
	set_grid_fields(t.dev, dp, t.dgrid);
	return ADGPU_OK;
}

}  // namespace adgpu
