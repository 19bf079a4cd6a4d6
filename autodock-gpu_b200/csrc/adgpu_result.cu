// adgpu_result.cu -- result processing on the device (include/adgpu_b200.h,
// "Result processing"): each run's final population ordered by energy, poses
// rebuilt from genotypes and re-scored with the reference's host scorer, the
// RMSD from the input ligand, and the runs clustered by RMSD.
//
// This file is compiled without flush-to-zero and without multiply-add
// contraction (build.py): its single- and double-precision arithmetic is the
// IEEE arithmetic of the reference's host code, which it follows operation by
// operation, in the same order, so that the energies, RMSDs and cluster
// assignments are the ones the reference's process_result computes.  The one
// source of difference is the double-precision sin/cos of the pose builder,
// which may round differently from the host's libm in the last place.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include "adgpu_prep.h"
#include "adgpu_result.h"
#include "adgpu_tables.h"
#include "adgpu_nvtx.h"

namespace adgpu {
namespace {

constexpr int kTab = 2048;                 // IntraTables distance tables, 0.01..20.48 A
constexpr int kWarps = 4;                  // rescoring warps per CTA
constexpr double kPi = 3.14159265359;      // PI, host/inc/miscellaneous.h:51
constexpr float kGbond = 50.0f;            // G, common/defines.h:108
constexpr int kCG = 24, kG0 = 25;          // ATYPE_CG_IDX, ATYPE_G0_IDX, common/defines.h:71-72
constexpr float kOutOfGridTol = 0.0005f;   // outofgrid_tolerance of make_resfiles' calc_interE_f calls
constexpr float kDcutoff = 8.0f;           // dcutoff of make_resfiles' calc_intraE_f calls

struct PostDev {
	int N, NL, NR, NT, Q, P;
	int gx, gy, gz, nmaps;                 // grid points, type maps
	int rmsd_atoms, symmetry, rescore_all;
	int cells;                             // grid layout: 0 reference (4 floats per point per map), 1 cell records
	const float* grid;
	const double *ref_xyz, *input_xyz, *charge, *rot_move, *rot_unit;
	const double *reqm, *vA, *vB, *vC, *vD, *solpar, *volume;
	const unsigned long long* rot_mask;
	const float *r6, *r10, *r12, *repsr, *desolv, *qasp_absq;
	const int *type, *map, *vwidx;
	const unsigned char *ignore, *is_hb;
	const unsigned int* pairs;
	double movvec[3];                      // get_movvec_to_origo of the reference orientation
	double spacing, origin[3];
	float smooth, elec_min_distance;
};

struct RunRec {                            // per run, written by the rescoring of its best entity
	float inter, intraflex, intra, interflex, elec, rmsd, energy;
	float crmsd;
	int clus, subrank, output, rank;
};

// ---------------------------------------------------------------------------
// arrange_result (host/src/processresult.cpp:31-59): a stable ascending bubble
// sort of each run's entities by energy.  A NaN energy compares false both
// ways, so it never moves and the entities on either side of it are sorted
// separately; each entity's destination is its rank inside its NaN-free
// segment (ties keep their order).
// ---------------------------------------------------------------------------
__device__ int stable_rank(const float* e, int n, int i)
{
	const float x = e[i];
	if (isnan(x)) return i;
	int s = i;
	while (s > 0 && !isnan(e[s - 1])) s--;
	int rank = s;
	for (int j = s; j < n && !isnan(e[j]); j++) rank += (e[j] < x) || (e[j] == x && j < i);
	return rank;
}

__global__ void __launch_bounds__(256) arrange_kernel(float* pop, float* energies, float* scratch, int P)
{
	extern __shared__ float sh_e[];
	int* dst = reinterpret_cast<int*>(sh_e + P);
	const size_t r = blockIdx.x;
	float* E = energies + r * P;
	float* G = pop + r * P * 64;
	float* S = scratch + r * P * 64;
	for (int i = threadIdx.x; i < P; i += blockDim.x) sh_e[i] = E[i];
	__syncthreads();
	for (int i = threadIdx.x; i < P; i += blockDim.x) dst[i] = stable_rank(sh_e, P, i);
	__syncthreads();
	for (int k = threadIdx.x; k < P * 64; k += blockDim.x) S[(size_t)dst[k >> 6] * 64 + (k & 63)] = G[k];
	for (int i = threadIdx.x; i < P; i += blockDim.x) E[dst[i]] = sh_e[i];
	__syncthreads();
	for (int k = threadIdx.x; k < P * 64; k += blockDim.x) G[k] = S[k];
}

// ---------------------------------------------------------------------------
// Pose building: change_conform (host/src/processligand.cpp:1607-1664) with
// rotate (host/src/miscellaneous.cpp:150-256): the point is moved by
// -movvec, turned by the quaternion q = (cos a/2, sin a/2 n) as q v q^-1
// (the products written out with v's and the result's scalar parts zero),
// and moved back.
// ---------------------------------------------------------------------------
__device__ void rotate_point(double p[3], const double mv[3], const double n[3], double c, double s)
{
	p[0] = p[0] - mv[0];
	p[1] = p[1] - mv[1];
	p[2] = p[2] - mv[2];
	const double lq = c, lx = s * n[0], ly = s * n[1], lz = s * n[2];
	const double rq = lq, rx = -1 * lx, ry = -1 * ly, rz = -1 * lz;
	const double tq = 0 - lx * p[0] - ly * p[1] - lz * p[2];
	const double tx = lq * p[0] + 0 + ly * p[2] - lz * p[1];
	const double ty = lq * p[1] - lx * p[2] + 0 + lz * p[0];
	const double tz = lq * p[2] + lx * p[1] - ly * p[0] + 0;
	p[0] = tq * rx + tx * rq + ty * rz - tz * ry;
	p[1] = tq * ry - tx * rz + ty * rq + tz * rx;
	p[2] = tq * rz + tx * ry - ty * rx + tz * rq;
	p[0] = p[0] + mv[0];
	p[1] = p[1] + mv[1];
	p[2] = p[2] + mv[2];
}

__device__ __forceinline__ double dist2(const double* a, const double* b)
{
	const double s1 = a[0] - b[0], s2 = a[1] - b[1], s3 = a[2] - b[2];
	return s1 * s1 + s2 * s2 + s3 * s3;
}

// calc_rmsd (host/src/processligand.cpp:1441-1489) of pose xyz against ref:
// with symmetry, each atom's squared distance to the nearest reference atom
// of its type (100000 when there is none).  Per-atom terms in parallel, the
// sum in atom order on lane 0, the result broadcast to the warp.
__device__ double warp_rmsd(const double* xyz, const double* ref, const int* type, int n, int symmetry, int lane)
{
	double sum = 0.0;
	for (int base = 0; base < n; base += 32) {
		const int a = base + lane;
		double m = 0.0;
		if (a < n) {
			if (symmetry) {
				m = 100000;
				for (int b = 0; b < n; b++)
					if (type[a] == type[b]) {
						const double d2 = dist2(xyz + 3 * a, ref + 3 * b);
						if (d2 < m) m = d2;
					}
			} else m = dist2(xyz + 3 * a, ref + 3 * a);
		}
		for (int k = 0; k < 32; k++) {
			const double mk = __shfl_sync(0xffffffffu, m, k);
			if (lane == 0 && base + k < n) sum += mk;
		}
	}
	return __shfl_sync(0xffffffffu, sqrt(sum / (unsigned)n), 0);
}

// ---------------------------------------------------------------------------
// Re-scoring, one warp per entity: the per-entity body of make_resfiles
// (host/src/processresult.cpp:421-475): change_conform_f, calc_interE_f in
// grid units, scale_ligand to Angstrom, calc_intraE_f, move_ligand to the
// grid's origin, calc_rmsd.  Per-atom and per-pair terms are computed by the
// lanes; the energies are summed on lane 0 in the reference's atom and pair
// order, so the float sums round as the host's do.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kWarps * 32)
rescore_kernel(PostDev D, const float* pop, const float* energies, int ntask, RunRec* runs, double* best_xyz,
               float* peratom, float* entities)
{
	extern __shared__ double sh_w[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int N = D.N, NL = D.NL, NR = D.NR;
	double* xyz = sh_w + (size_t)warp * (3 * N + 2 * NR + 8);
	double* trig = xyz + 3 * N;                // cos, sin of each torsion's half angle; genrot axis, cos, sin
	const size_t g3_4 = ((size_t)D.gx * D.gy * D.gz) << 2;
	for (int task = blockIdx.x * kWarps + warp; task < ntask; task += gridDim.x * kWarps) {
		const int run = D.rescore_all ? task / D.P : task;
		const int ent = D.rescore_all ? task % D.P : 0;
		const float* g = pop + ((size_t)run * D.P + ent) * 64;
		// half-angle sines and cosines (rotate computes them per call; same values)
		for (int rb = lane; rb < NR; rb += 32) {
			const double ang = (double)g[6 + rb];
			const double half = ang / 2 / 180 * kPi;
			trig[2 * rb] = cos(half);
			trig[2 * rb + 1] = sin(half);
		}
		if (lane == 0) {
			const double phi = ((double)g[3]) / 180 * kPi, theta = ((double)g[4]) / 180 * kPi;
			double* gr = trig + 2 * NR;
			gr[0] = sin(theta) * cos(phi);
			gr[1] = sin(theta) * sin(phi);
			gr[2] = cos(theta);
			const double half = (double)g[5] / 2 / 180 * kPi;
			gr[3] = cos(half);
			gr[4] = sin(half);
		}
		__syncwarp();
		const double* gr = trig + 2 * NR;
		const double zero[3] = {0.0, 0.0, 0.0};
		for (int a = lane; a < N; a += 32) {
			double p[3] = {D.ref_xyz[3 * a], D.ref_xyz[3 * a + 1], D.ref_xyz[3 * a + 2]};
			if (a < NL) for (int k = 0; k < 3; k++) p[k] += D.movvec[k];
			const unsigned long long m = D.rot_mask[a];
			for (int rb = 0; rb < NR; rb++)
				if ((m >> rb) & 1ull) rotate_point(p, D.rot_move + 3 * rb, D.rot_unit + 3 * rb, trig[2 * rb], trig[2 * rb + 1]);
			if (a < NL) {
				rotate_point(p, zero, gr, gr[3], gr[4]);
				for (int k = 0; k < 3; k++) p[k] += (double)g[k];
			}
			for (int k = 0; k < 3; k++) xyz[3 * a + k] = p[k];
		}
		__syncwarp();

		// calc_interE_f (host/src/processligand.cpp:1796-2055)
		const bool best = ent == 0;
		float interE = 0.0f, intraflexE = 0.0f, elecE = 0.0f;
		for (int base = 0; base < N; base += 32) {
			const int a = base + lane;
			int kind = 0;                      // 0: not counted, 1: outside the grid, 2: interpolated
			float val = 0.0f, vd = 0.0f, e = 0.0f;   // vd: vdW + desolvation (the per-atom vdW the reference reports)
			if (a < N && !D.ignore[a]) {
				float x = (float)xyz[3 * a], y = (float)xyz[3 * a + 1], z = (float)xyz[3 * a + 2];
				const float q = (float)D.charge[a];
				const float X1 = (float)(D.gx - 1), Y1 = (float)(D.gy - 1), Z1 = (float)(D.gz - 1);
				bool out = x < 0 || x >= X1 || y < 0 || y >= Y1 || z < 0 || z >= Z1;
				if (out) {
					if (x < 0) x += kOutOfGridTol;
					if (y < 0) y += kOutOfGridTol;
					if (z < 0) z += kOutOfGridTol;
					if (x >= X1) x -= kOutOfGridTol;
					if (y >= Y1) y -= kOutOfGridTol;
					if (z >= Z1) z -= kOutOfGridTol;
					out = x < 0 || x >= X1 || y < 0 || y >= Y1 || z < 0 || z >= Z1;
				}
				if (out) {
					val += 16777216;
					kind = 1;
				} else {
					const int xl = (int)floorf(x), yl = (int)floorf(y), zl = (int)floorf(z);
					// the 8 corner values of each map in idx_000 .. idx_111 order: 8 consecutive
					// floats from the point in the reference layout; the cell's record (e, d,
					// type maps) in the engine's layout, the same values in the same order
					const float *cv, *ce, *cd;
					if (D.cells) {
						const float* rec = D.grid + (size_t)(xl + yl * (D.gx - 1) + zl * (D.gx - 1) * (D.gy - 1)) *
						                            (size_t)(D.nmaps + 2) * 8;
						cv = rec + (size_t)(2 + D.map[a]) * 8;
						ce = rec;
						cd = rec + 8;
					} else {
						const float* c0 = D.grid + ((size_t)(unsigned)(xl + yl * D.gx + zl * D.gx * D.gy) << 2);
						cv = c0 + (size_t)D.map[a] * g3_4;
						ce = c0 + (size_t)D.nmaps * g3_4;
						cd = ce + g3_4;
					}
					const float dx = x - xl, omdx = 1.0f - dx;
					const float dy = y - yl, omdy = 1.0f - dy;
					const float dz = z - zl, omdz = 1.0f - dz;
					float w[8];
					w[0] = omdx * omdy * omdz; w[1] = omdx * dy * omdz; w[2] = omdx * omdy * dz; w[3] = omdx * dy * dz;
					w[4] = dx * omdy * omdz;   w[5] = dx * dy * omdz;   w[6] = dx * omdy * dz;   w[7] = dx * dy * dz;
					auto interp = [&](const float* c) {
						return c[0] * w[0] + c[1] * w[1] + c[2] * w[2] + c[3] * w[3] + c[4] * w[4] + c[5] * w[5] +
						       c[6] * w[6] + c[7] * w[7];
					};
					const float v = interp(cv);
					val += v;
					e = q * interp(ce);
					val += e;
					const float ed = fabsf(q) * interp(cd);
					val += ed;
					// AD4_desolv_peratom_vdW is defined (host/src/processligand.cpp:30, 2041-2043)
					vd = v + ed;
					kind = 2;
				}
			}
			if (best && a < N) {
				float* pa = peratom + ((size_t)run * N + a) * 2;
				pa[0] = kind == 2 ? vd : (kind == 1 ? 100000.0f : 0.0f);
				pa[1] = kind == 2 ? e : (kind == 1 ? 100000.0f : 0.0f);
			}
			for (int k = 0; k < 32; k++) {
				const float vk = __shfl_sync(0xffffffffu, val, k), ek = __shfl_sync(0xffffffffu, e, k);
				const int kk = __shfl_sync(0xffffffffu, kind, k);
				if (lane == 0 && kk) {
					if (base + k < NL) interE += vk;
					else intraflexE += vk;
					if (kk == 2 && base + k < NL) elecE += ek;
				}
			}
		}

		// scale_ligand to Angstrom (the grid's spacing)
		for (int a = lane; a < N; a += 32)
			for (int k = 0; k < 3; k++) xyz[3 * a + k] *= D.spacing;
		__syncwarp();

		// calc_intraE_f (host/src/processligand.cpp:2058-2331), without
		// modified pairs (the front end has none) and without contact analysis
		float vW = 0.0f, el = 0.0f, desolv = 0.0f, interflexE = 0.0f;
		const float delta = 0.5f * D.smooth;
		for (int base = 0; base < D.Q; base += 32) {
			const int pi = base + lane;
			int fl = 0;                         // 1: CG-G0 term, 2: vdW/H-bond term, 4: elec+desolv, 8: ligand-flexres pair
			float t_cg = 0.0f, t_vdw = 0.0f, t_a = 0.0f, t_b = 0.0f;
			if (pi < D.Q) {
				const int i = (int)D.pairs[2 * pi], j = (int)D.pairs[2 * pi + 1];
				if (((i >= NL) + (j >= NL)) & 1) fl |= 8;
				float dist = (float)sqrt(dist2(xyz + 3 * i, xyz + 3 * j));
				int did = (int)floorf((100.0f * dist) + 0.5f) - 1;
				if (did < 0) did = 0;
				const int t1 = D.type[i], t2 = D.type[j], tp = t1 * D.NT + t2;
				const int v1 = D.vwidx[t1], v2 = D.vwidx[t2];
				if ((v1 == kCG && v2 == kG0) || (v1 == kG0 && v2 == kCG)) {
					fl |= 1;
					t_cg = kGbond * dist;
				}
				if (dist < kDcutoff) {
					const float opt = (float)D.reqm[tp];
					float sd;
					if (dist <= (opt - delta)) sd = dist + delta;
					else if (dist < (opt + delta)) sd = opt;
					else sd = dist - delta;
					int sid = (int)floorf((100.0f * sd) + 0.5f) - 1;
					if (sid < 0) sid = 0;
					float vdw1, vdw2;
					if (D.is_hb[tp]) {
						vdw1 = (float)(D.vC[tp] * D.r12[sid]);
						vdw2 = (float)(D.vD[tp] * D.r10[sid]);
					} else {
						vdw1 = (float)(D.vA[tp] * D.r12[sid]);
						vdw2 = (float)(D.vB[tp] * D.r6[sid]);
					}
					fl |= 2;
					t_vdw = vdw1 - vdw2;
				}
				if (dist < 20.48) {
					int eid = did;
					if (dist < D.elec_min_distance) {
						dist = D.elec_min_distance;
						eid = (int)floor((100 * dist) + 0.5) - 1;
						// the reference reads outside its table here when elec_min_distance < 0.005
						eid = eid < 0 ? 0 : (eid >= kTab ? kTab - 1 : eid);
					}
					const float s1 = (float)(D.solpar[t1] + D.qasp_absq[i]);
					const float s2 = (float)(D.solpar[t2] + D.qasp_absq[j]);
					const float w1 = (float)D.volume[t1], w2 = (float)D.volume[t2];
					const float q1q2 = (float)((double)(float)D.charge[i] * D.charge[j]);
					t_a = q1q2 * D.repsr[eid];
					t_b = (s1 * w2 + s2 * w1) * D.desolv[eid];
					fl |= 4;
				}
			}
			for (int k = 0; k < 32; k++) {
				const int fk = __shfl_sync(0xffffffffu, fl, k);
				const float ck = __shfl_sync(0xffffffffu, t_cg, k), vk = __shfl_sync(0xffffffffu, t_vdw, k);
				const float ak = __shfl_sync(0xffffffffu, t_a, k), bk = __shfl_sync(0xffffffffu, t_b, k);
				if (lane == 0 && fk) {
					const bool flex = fk & 8;
					// the CG-G0 term goes the other way round from the others
					// (host/src/processligand.cpp:2142-2145)
					if (fk & 1) { if (flex) vW += ck; else interflexE += ck; }
					if (fk & 2) { if (flex) interflexE += vk; else vW += vk; }
					if (fk & 4) {
						if (flex) interflexE += ak + bk;
						else { el += ak; desolv += bk; }
					}
				}
			}
		}
		const float intraE = vW + el + desolv;

		// move_ligand by the grid's origin (ligand and flexible residues)
		for (int a = lane; a < N; a += 32)
			for (int k = 0; k < 3; k++) xyz[3 * a + k] += D.origin[k];
		__syncwarp();
		double rmsd = 0.0;
		if (best || D.rescore_all)
			rmsd = warp_rmsd(xyz, D.input_xyz, D.type, D.rmsd_atoms, D.symmetry, lane);
		if (lane == 0) {
			if (entities) {
				float* o = entities + ((size_t)run * D.P + ent) * 3;
				o[0] = intraE + intraflexE;
				o[1] = interE + interflexE;
				o[2] = (float)rmsd;
			}
			if (best) {
				RunRec& R = runs[run];
				R.inter = interE; R.intraflex = intraflexE; R.intra = intraE; R.interflex = interflexE;
				R.elec = elecE; R.rmsd = (float)rmsd; R.energy = energies[(size_t)run * D.P];
				R.crmsd = 0.0f; R.clus = 0; R.subrank = 0; R.output = 1; R.rank = 0;
			}
		}
		if (best)
			for (int a = lane; a < N; a += 32)
				for (int k = 0; k < 3; k++) best_xyz[((size_t)run * N + a) * 3 + k] = xyz[3 * a + k];
		__syncwarp();
	}
}

// ---------------------------------------------------------------------------
// generate_output's ordering and clustering (host/src/processresult.cpp:
// 688-804): runs ordered by energy (inter + interflex, plus intra terms for
// flexible residues alone) with the same NaN-segment stable ranking; then
// each run in that order joins the first cluster whose centre (its first
// member) lies within the RMSD tolerance, or founds a new one.  The RMSDs to
// all current centres are taken in parallel (one warp per centre); the scan
// over runs stays in order.  Cluster statistics: one thread per cluster.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
cluster_kernel(PostDev D, int R, RunRec* runs, const double* best_xyz, double* en, int* order, int* centers,
               double* crmsd, double tol, int calc, int ncp, int free_roaming, double torsional,
               adgpu_cluster* clusters, int* nclus)
{
	__shared__ int s_found, s_K;
	__shared__ double s_rmsd;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
	for (int r = tid; r < R; r += blockDim.x) {
		double e = (double)(runs[r].inter + runs[r].interflex);
		if (!free_roaming) e += (double)(runs[r].intra + runs[r].intraflex);
		en[r] = e;
	}
	__syncthreads();
	for (int r = tid; r < R; r += blockDim.x) {
		double x = en[r];
		int rank;
		if (isnan(x)) rank = r;
		else {
			int s = r;
			while (s > 0 && !isnan(en[s - 1])) s--;
			rank = s;
			for (int j = s; j < R && !isnan(en[j]); j++) rank += (en[j] < x) || (en[j] == x && j < r);
		}
		order[rank] = r;
		runs[r].rank = rank;
	}
	__syncthreads();
	if (!calc) {
		if (tid == 0) *nclus = 0;
		return;
	}
	const int n = D.rmsd_atoms, N = D.N;
	if (tid == 0) {
		const int c0 = order[0];
		runs[c0].clus = 1;
		runs[c0].crmsd = 0.0f;
		centers[0] = c0;
		s_K = 1;
	}
	__syncthreads();
	for (int w = 1; w < R; w++) {
		const int i = order[w];
		const int K = s_K;
		for (int c = warp; c < K; c += nwarps)
			crmsd[c] = warp_rmsd(best_xyz + (size_t)i * N * 3, best_xyz + (size_t)centers[c] * N * 3, D.type, n,
			                     D.symmetry, lane);
		__syncthreads();
		if (tid == 0) {
			int f = -1;
			for (int c = 0; c < K; c++)
				if (crmsd[c] <= tol) { f = c; break; }
			s_found = f;
			s_rmsd = f >= 0 ? crmsd[f] : 0.0;
		}
		__syncthreads();
		if (tid == 0) {
			if (s_found >= 0) {
				runs[i].clus = s_found + 1;
				runs[i].crmsd = (float)s_rmsd;
			} else {
				centers[K] = i;
				runs[i].clus = K + 1;
				runs[i].crmsd = 0.0f;
				s_K = K + 1;
			}
		}
		__syncthreads();
	}
	const int K = s_K;
	for (int c = tid; c < K; c += blockDim.x) {
		int sub = 0;
		double sum = 0.0, bestE = 0.0;
		int best_run = 0;
		for (int u = 0; u < R; u++) {
			const int j = order[u];
			if (runs[j].clus != c + 1) continue;
			sub++;
			sum += runs[j].inter + runs[j].interflex + torsional;
			if (!free_roaming) sum += runs[j].intra + runs[j].intraflex;
			runs[j].subrank = sub;
			runs[j].output = !((ncp > 0) && (sub > ncp)) && (ncp >= 0);
			if (sub == 1) {
				bestE = runs[j].inter + runs[j].interflex + torsional;
				if (!free_roaming) bestE += runs[j].intra + runs[j].intraflex;
				best_run = j + 1;
				runs[j].output = 1;
			}
		}
		clusters[c].size = sub;
		clusters[c].best_run = best_run;
		clusters[c].best_energy = bestE;
		clusters[c].sum_energy = sum;
	}
	if (tid == 0) *nclus = K;
}

// IntraTables' distance tables (calc_distdep_tables_f,
// host/src/processligand.cpp:1543-1570) on the host, with the host's libm as
// the reference computes them: 1/r^6, 1/r^10, 1/r^12, the distance-dependent
// dielectric elec factor and the desolvation gaussian at r = 0.01 .. 20.48 A.
double ddd_mehler_solmajer(double d)
{
	// Mehler & Solmajer (1991) sigmoidal dielectric with AutoDock's constants
	// (host/src/processligand.cpp:1491-1512): the constants are long double
	// literals held in doubles, and the denominator is formed in long double.
	const double lambda = 0.003627L, epsilon0 = 78.4L, A = -8.5525L, rk = 7.7839L;
	const double B = epsilon0 - A;
	const double lambda_B = -lambda * B;
	const double eps = A + B / (1.0L + rk * exp(lambda_B * d));
	return eps;
}

void distance_tables(float* r6, float* r10, float* r12, float* repsr, float* desolv, float coeff_elec, float coeff_desolv)
{
	float dist = 0;
	const float sigma = 3.6f;
	for (int i = 0; i < kTab; i++) {
		dist += 0.01;
		r6[i] = 1 / powf(dist, 6);
		r10[i] = 1 / powf(dist, 10);
		r12[i] = 1 / powf(dist, 12);
		repsr[i] = (float)coeff_elec / (dist * ddd_mehler_solmajer(dist));
		desolv[i] = coeff_desolv * expf(-1 * dist * dist / (2 * sigma * sigma));
	}
}

template <class T>
size_t put(std::vector<unsigned char>& blob, const T* src, size_t n)
{
	size_t off = (blob.size() + 15) / 16 * 16;
	blob.resize(off + n * sizeof(T));
	if (n) memcpy(blob.data() + off, src, n * sizeof(T));
	return off;
}

}  // namespace
}  // namespace adgpu

using namespace adgpu;

extern "C" {

adgpu_status adgpu_result_params_default(adgpu_result_params* p)
{
	if (!p) return fail(ADGPU_ERR_ARG, "null argument");
	memset(p, 0, sizeof(*p));
	p->rmsd_tolerance = 2.0f;
	p->handle_symmetry = 1;
	p->calc_clustering = 1;
	p->nr_cluster_poses = 0;
	p->free_roaming_ligand = 1;
	p->rescore_entities = 0;
	p->coeff_tors = 0.2983;
	return ADGPU_OK;
}

}  // extern "C"

namespace adgpu {

adgpu_status process_result_core(const PostLigand& L, const uint32_t* pairs, const adgpu_dockpars& dp,
                                 const float* grid, int grid_cells, float* populations, float* energies,
                                 uint32_t num_runs, const adgpu_result_params* params, adgpu_run_result* runs_out,
                                 adgpu_cluster* clusters_out, int* num_clusters, double* best_xyz, float* peratom,
                                 float* entities, cudaStream_t st, cudaMemPool_t pool)
{
	if (!grid || !populations || !energies || !params || !runs_out || !clusters_out || !num_clusters)
		return fail(ADGPU_ERR_ARG, "null argument");
	if (num_runs == 0 || num_runs > ADGPU_MAX_RUNS) return fail(ADGPU_ERR_LIMIT, "num_runs must be 1..8192");
	if (L.natoms <= 0) return fail(ADGPU_ERR_STATE, "ligand carries no result-processing data");
	if (params->nr_cluster_poses < 0)
		return fail(ADGPU_ERR_ARG, "nr_cluster_poses < 0 (poses chosen by contact analysis) is not supported");
	if (entities && !params->rescore_entities) return fail(ADGPU_ERR_ARG, "entities output needs rescore_entities");
	const int N = L.natoms, NR = L.nrot, NT = L.ntypes, P = dp.pop_size, R = (int)num_runs;
	const int Q = dp.num_of_intraE_contributors;

	// host side: constant tables (IntraTables) and the packed ligand
	std::vector<float> tab(5 * kTab);
	distance_tables(tab.data(), tab.data() + kTab, tab.data() + 2 * kTab, tab.data() + 3 * kTab, tab.data() + 4 * kTab,
	                dp.coeff_elec, dp.coeff_desolv);
	std::vector<float> qabs(N);
	for (int i = 0; i < N; i++) qabs[i] = dp.qasp * fabs(L.charge[i]);        // calc_q_tables_f
	std::vector<unsigned char> blob;
	const size_t o_ref = put(blob, L.ref_xyz.data(), 3 * N), o_in = put(blob, L.input_xyz.data(), 3 * N),
	             o_q = put(blob, L.charge.data(), N), o_mv = put(blob, L.rot_move.data(), 3 * NR),
	             o_un = put(blob, L.rot_unit.data(), 3 * NR), o_reqm = put(blob, L.reqm_AB.data(), NT * NT),
	             o_A = put(blob, L.vw_A.data(), NT * NT), o_B = put(blob, L.vw_B.data(), NT * NT),
	             o_C = put(blob, L.vw_C.data(), NT * NT), o_D = put(blob, L.vw_D.data(), NT * NT),
	             o_sp = put(blob, L.solpar.data(), NT), o_vol = put(blob, L.volume.data(), NT),
	             o_mask = put(blob, L.rot_mask.data(), N), o_tab = put(blob, tab.data(), tab.size()),
	             o_qa = put(blob, qabs.data(), N), o_ty = put(blob, L.type.data(), N), o_map = put(blob, L.map.data(), N),
	             o_vw = put(blob, L.vw_index.data(), NT), o_ig = put(blob, L.ignore_inter.data(), N),
	             o_hb = put(blob, L.is_hb.data(), NT * NT), o_pr = put(blob, pairs, 2 * (size_t)Q);
	// device scratch
	const size_t n_pop = (size_t)R * P * 64;
	size_t off = (blob.size() + 255) / 256 * 256;
	auto take = [&](size_t bytes) { size_t o = off; off = (off + bytes + 255) / 256 * 256; return o; };
	const size_t o_scr = take(n_pop * 4), o_runs = take((size_t)R * sizeof(RunRec)), o_bx = take((size_t)R * N * 3 * 8),
	             o_pa = take((size_t)R * N * 2 * 4), o_ent = take(params->rescore_entities ? (size_t)R * P * 3 * 4 : 0),
	             o_en = take((size_t)R * 8), o_ord = take((size_t)R * 4), o_cen = take((size_t)R * 4),
	             o_cr = take((size_t)R * 8), o_cl = take((size_t)R * sizeof(adgpu_cluster)), o_nc = take(4);

	unsigned char* d = nullptr;
	auto done = [&](cudaError_t err, const char* what) {
		if (d) cudaFreeAsync(d, st);
		cudaStreamSynchronize(st);
		return err == cudaSuccess ? ADGPU_OK : cuda_fail(err, what);
	};
	cudaError_t e = pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d), off, pool, st)
	                     : cudaMallocAsync(reinterpret_cast<void**>(&d), off, st);
	if (e != cudaSuccess) { d = nullptr; return done(e, "result scratch"); }
	e = cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, st);
	if (e != cudaSuccess) return done(e, "result tables");

	PostDev D;
	memset(&D, 0, sizeof(D));
	D.N = N; D.NL = L.true_lig_atoms; D.NR = NR; D.NT = NT; D.Q = Q; D.P = P;
	D.gx = dp.gridsize_x; D.gy = dp.gridsize_y; D.gz = dp.gridsize_z; D.nmaps = dp.num_of_map_atypes;
	D.rmsd_atoms = L.true_lig_atoms ? L.true_lig_atoms : N;
	D.symmetry = params->handle_symmetry ? 1 : 0;
	D.rescore_all = params->rescore_entities ? 1 : 0;
	D.cells = grid_cells ? 1 : 0;
	D.grid = grid;
	D.ref_xyz = (const double*)(d + o_ref); D.input_xyz = (const double*)(d + o_in); D.charge = (const double*)(d + o_q);
	D.rot_move = (const double*)(d + o_mv); D.rot_unit = (const double*)(d + o_un);
	D.reqm = (const double*)(d + o_reqm); D.vA = (const double*)(d + o_A); D.vB = (const double*)(d + o_B);
	D.vC = (const double*)(d + o_C); D.vD = (const double*)(d + o_D);
	D.solpar = (const double*)(d + o_sp); D.volume = (const double*)(d + o_vol);
	D.rot_mask = (const unsigned long long*)(d + o_mask);
	const float* T = (const float*)(d + o_tab);
	D.r6 = T; D.r10 = T + kTab; D.r12 = T + 2 * kTab; D.repsr = T + 3 * kTab; D.desolv = T + 4 * kTab;
	D.qasp_absq = (const float*)(d + o_qa);
	D.type = (const int*)(d + o_ty); D.map = (const int*)(d + o_map); D.vwidx = (const int*)(d + o_vw);
	D.ignore = d + o_ig; D.is_hb = d + o_hb; D.pairs = (const unsigned int*)(d + o_pr);
	// get_movvec_to_origo of the reference orientation (host/src/processligand.cpp:1363-1387)
	if (L.true_lig_atoms > 0) {
		double t[3] = {0, 0, 0};
		for (int i = 0; i < L.true_lig_atoms; i++) for (int k = 0; k < 3; k++) t[k] += L.ref_xyz[3 * i + k];
		for (int k = 0; k < 3; k++) D.movvec[k] = -1 * t[k] / L.true_lig_atoms;
	}
	D.spacing = L.spacing;
	for (int k = 0; k < 3; k++) D.origin[k] = L.origin[k];
	D.smooth = dp.smooth;
	D.elec_min_distance = dp.elec_min_distance;

	RunRec* d_runs = (RunRec*)(d + o_runs);
	double* d_bx = (double*)(d + o_bx);
	float* d_pa = (float*)(d + o_pa);
	float* d_ent = params->rescore_entities ? (float*)(d + o_ent) : nullptr;
	adgpu_cluster* d_cl = (adgpu_cluster*)(d + o_cl);
	int* d_nc = (int*)(d + o_nc);

	arrange_kernel<<<R, 256, (size_t)P * 8, st>>>(populations, energies, (float*)(d + o_scr), P);
	const int ntask = params->rescore_entities ? R * P : R;
	const size_t wsm = (size_t)kWarps * (3 * N + 2 * NR + 8) * sizeof(double);
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const int blocks = std::min((ntask + kWarps - 1) / kWarps, sms * 8);
	rescore_kernel<<<blocks, kWarps * 32, wsm, st>>>(D, populations, energies, ntask, d_runs, d_bx, d_pa, d_ent);
	cluster_kernel<<<1, 1024, 0, st>>>(D, R, d_runs, d_bx, (double*)(d + o_en), (int*)(d + o_ord), (int*)(d + o_cen),
	                                   (double*)(d + o_cr), (double)params->rmsd_tolerance, params->calc_clustering ? 1 : 0,
	                                   params->nr_cluster_poses, params->free_roaming_ligand ? 1 : 0,
	                                   params->coeff_tors * L.true_lig_rotbonds, d_cl, d_nc);
	e = cudaGetLastError();
	if (e != cudaSuccess) return done(e, "result kernels");
	std::vector<RunRec> h_runs(R);
	e = cudaMemcpyAsync(h_runs.data(), d_runs, R * sizeof(RunRec), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaMemcpyAsync(clusters_out, d_cl, R * sizeof(adgpu_cluster), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaMemcpyAsync(num_clusters, d_nc, 4, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess && best_xyz) e = cudaMemcpyAsync(best_xyz, d_bx, (size_t)R * N * 3 * 8, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess && peratom) e = cudaMemcpyAsync(peratom, d_pa, (size_t)R * N * 2 * 4, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess && entities) e = cudaMemcpyAsync(entities, d_ent, (size_t)R * P * 3 * 4, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (e != cudaSuccess) return done(e, "result download");
	for (int r = 0; r < R; r++) {
		const RunRec& s = h_runs[r];
		adgpu_run_result& o = runs_out[r];
		o.inter_e = s.inter; o.interflex_e = s.interflex; o.inter_e_elec = s.elec; o.intra_e = s.intra;
		o.intraflex_e = s.intraflex; o.rmsd_from_ref = s.rmsd; o.rmsd_from_cluster_center = s.crmsd; o.energy = s.energy;
		o.run_number = r + 1; o.cluster_id = s.clus; o.cluster_subrank = s.subrank; o.output = s.output;
		o.energy_rank = s.rank;
	}
	return done(cudaSuccess, "");
}


}  // namespace adgpu

extern "C" {

adgpu_status adgpu_process_result(const adgpu_ligand* lig, const float* grid_reference_layout, float* populations,
                                  float* energies, uint32_t num_runs, const adgpu_result_params* params,
                                  adgpu_run_result* runs_out, adgpu_cluster* clusters_out, int* num_clusters,
                                  double* best_xyz, float* peratom, float* entities)
{
	adgpu::NvtxRange nvtx_range("adgpu_process_result");
	if (!lig) return fail(ADGPU_ERR_ARG, "null argument");
	// a blocking stream: ordered after the caller's work on the legacy
	// default stream (where the kernel API and torch's default stream write
	// the final populations)
	cudaStream_t st = nullptr;
	cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamDefault);
	if (e != cudaSuccess) return cuda_fail(e, "stream");
	// scratch from a pool of this library that keeps its memory between calls
	// (one per device), so repeated calls do not go back to the driver
	static std::mutex pool_mu;
	static cudaMemPool_t pools[64] = {};
	cudaMemPool_t pool = nullptr;
	int dev = 0;
	if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
		std::lock_guard<std::mutex> lk(pool_mu);
		if (!pools[dev]) {
			cudaMemPoolProps props{};
			props.allocType = cudaMemAllocationTypePinned;
			props.location.type = cudaMemLocationTypeDevice;
			props.location.id = dev;
			if (cudaMemPoolCreate(&pools[dev], &props) == cudaSuccess) {
				uint64_t keep = 256ull << 20;
				cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
			} else {
				pools[dev] = nullptr;
				cudaGetLastError();
			}
		}
		pool = pools[dev];
	}
	adgpu_status rc = process_result_core(lig->p.post, lig->p.pairs.data(), lig->p.dockpars, grid_reference_layout, 0,
	                                      populations, energies, num_runs, params, runs_out, clusters_out, num_clusters,
	                                      best_xyz, peratom, entities, st, pool);
	cudaStreamDestroy(st);
	return rc;
}

}  // extern "C"
