// adgpu_noalloc.cu -- a scorer entry point that allocates no device memory.
//
// adgpu_score_genotypes needs the library's repacked copy of a ligand's
// tables and its cell-record grid, which adgpu_set_kernels_gpu_data
// allocates with cudaMalloc.  Some callers cannot allocate at all: a host
// that owns all device memory through its own pool and forbids foreign
// allocations, or a process whose device memory is already fully reserved.
// For them,
// adgpu_score_genotypes_noalloc repacks the caller's reference-layout tables
// on the device into one fixed, file-scope device array and reads the
// caller's grid in its own layout, so the only memory it touches besides its
// inputs and outputs is that array.
#include <cuda_runtime.h>
#include <mutex>
#include <string>

#include "adgpu_kernels.cuh"

namespace adgpu {
adgpu_status fail(adgpu_status st, const std::string& msg);
adgpu_status cuda_fail(cudaError_t e, const char* what);
}

using namespace adgpu;

// 1 MiB of scratch: the repacked tables of one ligand (about 30,000
// intramolecular pairs at most).  Every device that loads the library holds
// this array until the process exits.
static constexpr size_t kNoAllocScratchBytes = 1u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

struct NoAllocLayout {
	size_t ligdev = 0, status = 0, xyzq = 0, info = 0, clen = 0, chain = 0, uv = 0, mv = 0, ends = 0, items = 0, pairs = 0;
	size_t pairs_bytes = 0;      // two-pair records of the AD4 pairs from the front, PairRec entries from the back
	size_t total = 0;
};

size_t up16(size_t v) { return (v + 15) / 16 * 16; }

NoAllocLayout layout_for(const adgpu_dockpars& dp)
{
	const size_t N = dp.num_of_atoms, NT = dp.num_of_genes - 6, Q = dp.num_of_intraE_contributors;
	NoAllocLayout l;
	size_t o = 0;
	l.ligdev = o; o = up16(o + sizeof(LigDev));
	l.status = o; o = up16(o + 16);
	l.xyzq = o; o = up16(o + N * 16);
	l.info = o; o = up16(o + N * 4);
	l.clen = o; o = up16(o + N);
	l.chain = o; o = up16(o + (size_t)dp.rotbondlist_length + 1);
	l.uv = o; o = up16(o + (NT + 1) * 16);
	l.mv = o; o = up16(o + (NT + 1) * 16);
	l.ends = o; o = up16(o + (NT + 1) * 8);
	l.items = o; o = up16(o + N * (NT + 1) * 4);
	// AD4 pairs take pair2_records(Qs) * 64 <= 32 * Qs + 2048 bytes and the
	// others 32 * Qg, so this holds any split of the Q pairs
	l.pairs = o; l.pairs_bytes = (size_t)pair2_records((uint32_t)Q) * 64 + 32 * 64;
	o = up16(o + l.pairs_bytes);
	l.total = o;
	return l;
}

// Repacks the reference tables (device memory) into the scratch array: the
// device-side twin of pack_ligand (adgpu_tables.cu), with the same float
// operations (no contraction) so the packed values are bit-identical.
__global__ void __launch_bounds__(256) noalloc_repack_kernel(adgpu_gpudata d, LigDev L, NoAllocLayout lay)
{
	unsigned char* base = g_noalloc_scratch;
	int* status = reinterpret_cast<int*>(base + lay.status);
	const adgpu_dockpars& dp = d.dockpars;
	const int N = dp.num_of_atoms, NT = dp.num_of_genes - 6, Q = dp.num_of_intraE_contributors;
	__shared__ int s_start[ADGPU_MAX_ATOMS + 1];
	__shared__ int s_istart[ADGPU_MAX_ROTBONDS + 1];
	if (threadIdx.x == 0) status[0] = 0;
	__syncthreads();
	const int* rl = d.pKerconst_rotlist->rotlist_const;
	float4* xyzq = reinterpret_cast<float4*>(base + lay.xyzq);
	uint32_t* info = reinterpret_cast<uint32_t*>(base + lay.info);
	uint8_t* clen = base + lay.clen;
	uint8_t* chain = base + lay.chain;
	// pass 1: torsion rotations per atom, and the general-rotation flag
	for (int a = threadIdx.x; a < N; a += blockDim.x) {
		int cnt = 0;
		bool genrot = false;
		for (int k = 0; k < dp.rotbondlist_length; k++) {
			int el = rl[k];
			if ((el & ADGPU_RLIST_DUMMY_MASK) || (el & ADGPU_RLIST_ATOMID_MASK) != a) continue;
			if (el & ADGPU_RLIST_GENROT_MASK) {
				if (genrot) status[0] = 1;
				genrot = true;
			} else {
				if (genrot) status[0] = 1;
				int rb = (el & ADGPU_RLIST_RBONDID_MASK) >> ADGPU_RLIST_RBONDID_SHIFT;
				if (rb >= NT) status[0] = 1;
				cnt++;
			}
		}
		s_start[a + 1] = cnt;
		clen[a] = (uint8_t)cnt;
		info[a] = genrot ? 0x200u : 0u;
	}
	// a rotation-list entry must name one of the atoms (the repack on the
	// host rejects the same, adgpu_tables.cu)
	for (int k = threadIdx.x; k < dp.rotbondlist_length; k += blockDim.x) {
		const int el = rl[k];
		if (!(el & ADGPU_RLIST_DUMMY_MASK) && (el & ADGPU_RLIST_ATOMID_MASK) >= N) status[0] = 1;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		s_start[0] = 0;
		for (int a = 0; a < N; a++) s_start[a + 1] += s_start[a];
		s_istart[0] = 0;
		const int* nrot = d.pMem_num_rotating_atoms_per_rotbond_const;
		for (int k = 0; k < NT; k++) {
			int n = nrot[k];
			if (n < 0 || n > N) { status[0] = 1; n = 0; }
			s_istart[k + 1] = s_istart[k] + n;
		}
	}
	__syncthreads();
	// pass 2: chains, per-atom records
	const adgpu_kc_interintra* ii = d.pKerconst_interintra;
	const float* ref = d.pKerconst_conform->ref_coords_const;
	for (int a = threadIdx.x; a < N; a += blockDim.x) {
		int pos = s_start[a];
		for (int k = 0; k < dp.rotbondlist_length; k++) {
			int el = rl[k];
			if ((el & ADGPU_RLIST_DUMMY_MASK) || (el & ADGPU_RLIST_ATOMID_MASK) != a || (el & ADGPU_RLIST_GENROT_MASK)) continue;
			chain[pos++] = (uint8_t)((el & ADGPU_RLIST_RBONDID_MASK) >> ADGPU_RLIST_RBONDID_SHIFT);
		}
		xyzq[a] = make_float4(ref[3 * a], ref[3 * a + 1], ref[3 * a + 2], ii->atom_charges_const[a]);
		uint32_t mt = ii->atom_types_map_const[a];
		bool ignore = ii->ignore_inter_const[a] > 0;
		if (!ignore && mt >= (uint32_t)dp.num_of_map_atypes) status[0] = 1;
		if (ii->atom_types_const[a] >= (uint32_t)dp.num_of_atypes) status[0] = 1;
		info[a] |= (ignore ? 0x100u : (2u + mt)) | ((uint32_t)s_start[a] << 16);
	}
	// torsions
	const float* cuv = d.pKerconst_conform->rotbonds_unit_vectors_const;
	const float* cmv = d.pKerconst_conform->rotbonds_moving_vectors_const;
	float4* uv = reinterpret_cast<float4*>(base + lay.uv);
	float4* mv = reinterpret_cast<float4*>(base + lay.mv);
	int2* ends = reinterpret_cast<int2*>(base + lay.ends);
	uint32_t* items = reinterpret_cast<uint32_t*>(base + lay.items);
	for (int k = threadIdx.x; k < NT; k += blockDim.x) {
		uv[k] = make_float4(cuv[3 * k], cuv[3 * k + 1], cuv[3 * k + 2], 0.f);
		mv[k] = make_float4(cmv[3 * k], cmv[3 * k + 1], cmv[3 * k + 2], 0.f);
		int a1 = d.pMem_rotbonds_const[2 * k], a2 = d.pMem_rotbonds_const[2 * k + 1];
		if (a1 < 0 || a1 >= N || a2 < 0 || a2 >= N) status[0] = 1;
		ends[k] = make_int2(a1, a2);
		for (int c = 0; c < s_istart[k + 1] - s_istart[k]; c++) {
			int la = d.pMem_rotbonds_atoms_const[ADGPU_MAX_ATOMS * k + c];
			if (la < 0 || la >= N) { status[0] = 1; la = 0; }
			items[interleave_pos((uint32_t)(s_istart[k] + c), (uint32_t)s_istart[NT])] = ((uint32_t)k << 8) | (uint32_t)la;
		}
	}
	// intramolecular pairs: the AD4 ones (m = 12, n = 6 or 10) into
	// two-pair records in warp-interleaved order (interleave_pos), the others one to
	// a PairRec; each thread takes a contiguous chunk, and a scan of the
	// per-chunk counts of other-exponent pairs gives every pair its index
	const uint32_t* pairs = d.pKerconst_intracontrib->intraE_contributors_const;
	const adgpu_kc_intra* kin = d.pKerconst_intra;
	const uint32_t nat = (uint32_t)dp.num_of_atypes;
	__shared__ int s_gen[257];
	const int chunk = (Q + (int)blockDim.x - 1) / (int)blockDim.x;
	const int p0 = min(Q, (int)threadIdx.x * chunk), p1 = min(Q, p0 + chunk);
	auto exps_of = [&](int p, uint32_t& a1, uint32_t& a2, uint32_t& t1, uint32_t& t2) {
		a1 = pairs[2 * p]; a2 = pairs[2 * p + 1];
		if (a1 >= (uint32_t)N || a2 >= (uint32_t)N) { status[0] = 1; a1 = a2 = 0; }
		t1 = ii->atom_types_const[a1]; t2 = ii->atom_types_const[a2];
		if (t1 >= nat || t2 >= nat) { status[0] = 1; t1 = t2 = 0; }
		return (uint32_t)kin->VWpars_exp_const[t1 * nat + t2];
	};
	auto is_ad4 = [](uint32_t exps) { const uint32_t m = (exps & 0xFF00) >> 8, n = exps & 0xFF; return m == 12 && (n == 6 || n == 10); };
	int ngen = 0;
	for (int p = p0; p < p1; p++) {
		uint32_t a1, a2, t1, t2;
		if (!is_ad4(exps_of(p, a1, a2, t1, t2))) ngen++;
	}
	s_gen[threadIdx.x + 1] = ngen;
	__syncthreads();
	if (threadIdx.x == 0) {
		s_gen[0] = 0;
		for (int i = 0; i < (int)blockDim.x; i++) s_gen[i + 1] += s_gen[i];
	}
	__syncthreads();
	const int Qg = s_gen[blockDim.x], Qs = Q - Qg;
	const uint32_t nrec = pair2_records((uint32_t)Qs);
	float4* pr2 = reinterpret_cast<float4*>(base + lay.pairs);
	PairRec* gpr = reinterpret_cast<PairRec*>(base + lay.pairs + lay.pairs_bytes - (size_t)Qg * sizeof(PairRec));
	for (uint32_t r = threadIdx.x; r < nrec; r += blockDim.x) pair2_pad(pr2, r, (uint32_t)N);
	__syncthreads();
	int gi = s_gen[threadIdx.x];
	for (int p = p0; p < p1; p++) {
		uint32_t a1, a2, t1, t2;
		const uint32_t exps = exps_of(p, a1, a2, t1, t2);
		const uint32_t m = (exps & 0xFF00) >> 8, n = exps & 0xFF;
		const uint32_t idx = t1 * nat + t2;
		const uint32_t h1 = kin->atom_types_reqm_const[t1], h2 = kin->atom_types_reqm_const[t2];
		const bool cgg0 = (h1 == 24 && h2 == 25) || (h1 == 25 && h2 == 24);
		const float q1 = ii->atom_charges_const[a1], q2 = ii->atom_charges_const[a2];
		const float ac = kin->VWpars_AC_const[idx], bd = kin->VWpars_BD_const[idx], reqm = kin->reqm_AB_const[idx];
		const float dsp = __fadd_rn(__fmul_rn(__fadd_rn(kin->dspars_S_const[t1], __fmul_rn(dp.qasp, fabsf(q1))), kin->dspars_V_const[t2]),
		                            __fmul_rn(__fadd_rn(kin->dspars_S_const[t2], __fmul_rn(dp.qasp, fabsf(q2))), kin->dspars_V_const[t1]));
		const float qq = __fmul_rn(__fmul_rn(dp.coeff_elec, q1), q2);
		const float vb = cgg0 ? 50.0f : 0.0f;
		if (is_ad4(exps)) {
			uint32_t rec, h;
			pair2_slot(interleave_pos((uint32_t)(p - gi), (uint32_t)Qs), &rec, &h);
			pair2_set(pr2, rec, h, ac, n == 6 ? bd : 0.0f, n == 10 ? bd : 0.0f, reqm, __fmul_rn(dp.coeff_desolv, dsp), qq,
			          vb, a1 | (a2 << 8));
		} else {
			PairRec r;
			r.ac = ac; r.bd = bd; r.reqm = reqm; r.dsolv_pref = dsp; r.qq = qq; r.vbond = vb;
			r.ij = a1 | (a2 << 8) | (m << 16) | (n << 24);
			r.pad = 0;
			gpr[gi++] = r;
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		L.ntoritems = s_istart[NT];
		L.npairs2 = (int)nrec; L.ngpairs = Qg;
		L.pairs2 = pr2; L.gpairs = gpr;
		*reinterpret_cast<LigDev*>(base + lay.ligdev) = L;
	}
}

template <bool GRAD>
__global__ void __launch_bounds__(128) noalloc_score_kernel(size_t ligdev_off, adgpu_dockpars dp, uint32_t n,
                                                             const float* genotypes, float* energies, float* gradients)
{
	__shared__ LigDev sL;
	if (threadIdx.x == 0) sL = *reinterpret_cast<const LigDev*>(g_noalloc_scratch + ligdev_off);
	__syncthreads();
	extern __shared__ __align__(16) char smem[];
	const int local = threadIdx.x / 32;
	const int bytes = group_smem_bytes(sL.natoms, sL.ntors, 64, 32);
	GroupSmem S = carve_group(smem + local * bytes, sL.natoms, sL.ntors, 64, 32);
	Group<32> G;
	G.rank = threadIdx.x % 32;
	G.bar_id = 1 + local;
	G.red = S.red;
	const int NG = dp.num_of_genes;
	for (uint32_t b = blockIdx.x * 4 + local; b < n; b += gridDim.x * 4) {
		for (int k = G.rank; k < NG; k += 32) S.gen[k] = genotypes[(size_t)b * kGenotypeStride + k];
		G.sync();
		const float e = score_pose<32, GRAD, true>(sL, S.gen, S.grad, S.pose, G);
		if (GRAD)
			for (int k = G.rank; k < NG; k += 32) gradients[(size_t)b * kGenotypeStride + k] = S.grad[k];
		if (G.rank == 0) energies[b] = e;
		G.sync();
	}
}

// Device address of the scratch array, looked up once per device.
std::mutex g_sym_mu;
void* g_sym_addr[64] = {nullptr};

}  // namespace

extern "C" adgpu_status adgpu_score_genotypes_noalloc(const adgpu_gpudata* data, uint32_t n, const float* genotypes,
                                                      float* energies, float* gradients)
{
	if (!data || !genotypes || !energies) return fail(ADGPU_ERR_ARG, "null argument");
	const adgpu_dockpars& dp = data->dockpars;
	if (!data->pKerconst_interintra || !data->pKerconst_intracontrib || !data->pKerconst_intra ||
	    !data->pKerconst_rotlist || !data->pKerconst_conform || !data->pMem_fgrids || !data->pMem_rotbonds_const ||
	    !data->pMem_rotbonds_atoms_const || !data->pMem_num_rotating_atoms_per_rotbond_const)
		return fail(ADGPU_ERR_ARG, "GpuData has a null table pointer");
	if (dp.num_of_atoms <= 0 || dp.num_of_atoms > ADGPU_MAX_ATOMS || dp.num_of_genes < 6 || dp.num_of_genes > ADGPU_MAX_GENES ||
	    dp.num_of_intraE_contributors < 0 || dp.num_of_intraE_contributors > ADGPU_MAX_INTRAE ||
	    dp.rotbondlist_length < 0 || dp.rotbondlist_length > ADGPU_MAX_ROTATIONS || dp.num_of_atypes <= 0 ||
	    dp.num_of_atypes > ADGPU_MAX_ATYPES || dp.true_ligand_atoms < 0 || dp.true_ligand_atoms > dp.num_of_atoms ||
	    dp.num_of_map_atypes <= 0 || dp.num_of_map_atypes > ADGPU_MAX_ATYPES ||
	    dp.gridsize_x < 2 || dp.gridsize_y < 2 || dp.gridsize_z < 2)
		return fail(ADGPU_ERR_LIMIT, "docking parameters out of the reference's limits");
	const NoAllocLayout lay = layout_for(dp);
	if (lay.total > kNoAllocScratchBytes)
		return fail(ADGPU_ERR_LIMIT, "ligand needs " + std::to_string(lay.total) +
		                             " bytes of scratch; adgpu_score_genotypes_noalloc holds at most 1048576 "
		                             "(about 30,000 intramolecular pairs); use adgpu_score_genotypes");
	if (n == 0) return ADGPU_OK;
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return cuda_fail(e, "current device");
	if (dev < 0 || dev >= 64) return fail(ADGPU_ERR_ARG, "device ordinal beyond 63");
	void* scratch = nullptr;
	{
		std::lock_guard<std::mutex> lk(g_sym_mu);
		if (!g_sym_addr[dev]) {
			e = cudaGetSymbolAddress(&g_sym_addr[dev], g_noalloc_scratch);
			if (e != cudaSuccess) { g_sym_addr[dev] = nullptr; return cuda_fail(e, "scratch symbol address"); }
		}
		scratch = g_sym_addr[dev];
	}
	unsigned char* base = static_cast<unsigned char*>(scratch);
	LigDev L;
	memset(&L, 0, sizeof(L));
	L.natoms = dp.num_of_atoms; L.nlig = dp.true_ligand_atoms; L.ngenes = dp.num_of_genes; L.ntors = dp.num_of_genes - 6;
	L.npairs = dp.num_of_intraE_contributors;
	L.atom_xyzq = reinterpret_cast<const float4*>(base + lay.xyzq);
	L.atom_info = reinterpret_cast<const uint32_t*>(base + lay.info);
	L.chain_len = base + lay.clen;
	L.chain = base + lay.chain;
	L.tors_uv = reinterpret_cast<const float4*>(base + lay.uv);
	L.tors_mv = reinterpret_cast<const float4*>(base + lay.mv);
	L.tors_ends = reinterpret_cast<const int2*>(base + lay.ends);
	L.tor_items = reinterpret_cast<const uint32_t*>(base + lay.items);
	L.gx = dp.gridsize_x; L.gy = dp.gridsize_y; L.gz = dp.gridsize_z;
	L.cells_x = dp.gridsize_x - 1;
	L.cells_xy = (dp.gridsize_x - 1) * (dp.gridsize_y - 1);
	L.rec_floats = 8 * (dp.num_of_map_atypes + 2);
	L.spacing = dp.grid_spacing;
	L.inv_spacing = 1.0f / dp.grid_spacing;
	L.coeff_desolv = dp.coeff_desolv;
	L.elec_min_distance = dp.elec_min_distance;
	L.half_smooth = 0.5f * dp.smooth;
	L.grid = data->pMem_fgrids;          // the caller's grid, reference layout
	noalloc_repack_kernel<<<1, 256>>>(*data, L, lay);
	e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "repack launch");
	int status = 0;
	e = cudaMemcpy(&status, base + lay.status, sizeof(int), cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return cuda_fail(e, "repack");
	if (status) return fail(ADGPU_ERR_ARG, "GpuData tables hold an index out of range");
	const int bytes = group_smem_bytes(L.natoms, L.ntors, 64, 32) * 4;
	auto k = gradients ? noalloc_score_kernel<true> : noalloc_score_kernel<false>;
	if (bytes > 48 * 1024) {
		e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
		if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
	}
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	unsigned grid = (n + 3) / 4;
	if (grid > (unsigned)sms * 8) grid = sms * 8;
	k<<<grid, 128, bytes>>>(lay.ligdev, dp, n, genotypes, energies, gradients);
	e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "score launch");
	// both kernels ran on the legacy default stream: wait for them only
	e = cudaStreamSynchronize(cudaStreamLegacy);
	if (e != cudaSuccess) return cuda_fail(e, "score");
	return ADGPU_OK;
}
