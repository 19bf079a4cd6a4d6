/*
 * adgpu_oracle.c -- CPU restatement of AutoDock-GPU's LGA hot path (plain C).
 *
 * TEST INFRASTRUCTURE ONLY (see adgpu_oracle.h).  Each function names the
 * reference lines it restates.  One pose is scored by one CPU thread, in
 * program order; where the reference's result depends on its thread layout
 * (which LCG state a draw uses; the warp arg-min of the elitist selection)
 * that layout is emulated with `threads` virtual lanes.
 */
#define _GNU_SOURCE
#include "adgpu_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- constants (common/calcenergy_basic.h, common/defines.h, cuda/GpuData.h) */
#define DEG_TO_RAD        0.0174533f
#define PI_FLOAT          ((float)M_PI)
#define PI_TIMES_2        (2.0f * PI_FLOAT)
#define INV_PI_TIMES_2    (1.0f / (PI_TIMES_2))
#define ATYPE_CG_IDX      24
#define ATYPE_G0_IDX      25
#define G_CG_G0           50.0f
#define TERMSCALE         1024.0f
#define ONEOVERTERMSCALE  (1.0f / 1024.0f)
#define MAXTERM           8192.0f
#define MAXENERGY         (FLT_MAX / 100.0f)
#define INFINITESIMAL_RADIAN 1E-3f
#define HALF_INFINITESIMAL_RADIAN (0.5f * INFINITESIMAL_RADIAN)
#define INV_INFINITESIMAL_RADIAN (1.0f / INFINITESIMAL_RADIAN)
#define SCFACTOR_ANGSTROM_RADIAN (1.0f / (DEG_TO_RAD * DEG_TO_RAD))
#define LS_EXP_FACTOR     2.0f
#define LS_CONT_FACTOR    0.5f
#define GSTRIDE           ADGPU_GENOTYPE_STRIDE

typedef struct { float x, y, z; } f3;
typedef struct { float x, y, z, w; } f4;
typedef struct { int x, y, z; } i3;

/* ---- small helpers (cuda/calcenergy.cu:31-109) ------------------------- */

/* fmod_pi2, cuda/calcenergy.cu:43-46 */
static float fmod_pi2(float x) { return x - (float)(int)(INV_PI_TIMES_2 * x) * PI_TIMES_2; }

/* fast_acos, cuda/calcenergy.cu:48-65: the reference's polynomial+sqrt fit of
 * acos; kept identical because the orientation gradient is defined through it. */
static float fast_acos(float cosine)
{
	const float a = 9.78056e-05f, b = -0.00104588f, c = 0.00418716f, d = -0.00314347f;
	const float e = 2.74084f, f = 0.370388f, o = -(a + b + c + d);
	float x = fabsf(cosine);
	float x2 = x * x, x3 = x2 * x, x4 = x3 * x;
	float ac = (((o * x4 + a) * x3 + b) * x2 + c) * x + d
	           + e * sqrtf(2.0f - sqrtf(2.0f + 2.0f * x)) - f * sqrtf(2.0f - 2.0f * x);
	return copysignf(ac, cosine) + (float)(cosine < 0.0f) * PI_FLOAT;
}

/* cross, cuda/calcenergy.cu:67-85 */
static f3 cross3(f3 u, f3 v)
{
	f3 r = { u.y * v.z - v.y * u.z, v.x * u.z - u.x * v.z, u.x * v.y - v.x * u.y };
	return r;
}

/* quaternion_multiply, cuda/calcenergy.cu:87-94 */
static f4 qmul(f4 a, f4 b)
{
	f4 r = { a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
	         a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
	         a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
	         a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z };
	return r;
}

/* quaternion_rotate, cuda/calcenergy.cu:95-109 */
static f3 qrot(f3 v, f4 q)
{
	f3 qv = { q.x, q.y, q.z };
	f3 z = cross3(qv, v);
	z.x *= 2.0f; z.y *= 2.0f; z.z *= 2.0f;
	f3 c = cross3(qv, z);
	f3 r = { v.x + z.x * q.w + c.x, v.y + z.y * q.w + c.y, v.z + z.z * q.w + c.z };
	return r;
}

static int quant(float v)   /* lrintf(clamp(TERMSCALE*v)) as used throughout calcMergeEneGra.cu */
{
	return (int)lrintf(fminf(MAXTERM, fmaxf(-MAXTERM, TERMSCALE * v)));
}

/* ---- pose build (cuda/calcMergeEneGra.cu:92-190) ------------------------ */
static void build_pose(const adgpu_gpudata* d, const float* g, f3* xyz, f4* genrot_q, f3* genrot_mv,
                       float* sin_theta_out, float* sin_half_out, float* is_theta_gt_pi)
{
	const adgpu_dockpars* dp = &d->dockpars;
	const float* ref = d->pKerconst_conform->ref_coords_const;
	for (int a = 0; a < dp->num_of_atoms; a++) {
		xyz[a].x = ref[3 * a]; xyz[a].y = ref[3 * a + 1]; xyz[a].z = ref[3 * a + 2];
	}
	float phi = g[3] * DEG_TO_RAD, theta = g[4] * DEG_TO_RAD, rotangle = g[5] * DEG_TO_RAD;
	f4 gq = { 0, 0, 0, 1 };
	f3 gm = { 0, 0, 0 };
	float sin_theta = 0.0f, sin_half = 0.0f;
	if (dp->true_ligand_atoms) {
		gm.x = g[0]; gm.y = g[1]; gm.z = g[2];
		sin_theta = sinf(theta);
		float cos_theta = cosf(theta);
		sin_half = sinf(rotangle * 0.5f);
		gq.x = sin_half * sin_theta * cosf(phi);
		gq.y = sin_half * sin_theta * sinf(phi);
		gq.z = sin_half * cos_theta;
		gq.w = cosf(rotangle * 0.5f);
	}
	if (genrot_q) *genrot_q = gq;
	if (genrot_mv) *genrot_mv = gm;
	if (sin_theta_out) *sin_theta_out = sin_theta;
	if (sin_half_out) *sin_half_out = sin_half;
	if (is_theta_gt_pi) *is_theta_gt_pi = 1.0f - 2.0f * (float)(sin_theta < 0.0f);
	const int* rl = d->pKerconst_rotlist->rotlist_const;
	const float* uv = d->pKerconst_conform->rotbonds_unit_vectors_const;
	const float* mv = d->pKerconst_conform->rotbonds_moving_vectors_const;
	/* rows of the rotation list are dependency ordered (host/src/calcenergy.cpp:387-488),
	 * so walking the list in order is a valid serialisation of the reference's row loop */
	for (int k = 0; k < dp->rotbondlist_length; k++) {
		int el = rl[k];
		if (el & ADGPU_RLIST_DUMMY_MASK) continue;
		int atom = el & ADGPU_RLIST_ATOMID_MASK;
		f3 p = xyz[atom];
		f4 q; f3 m;
		if (atom < dp->true_ligand_atoms) { q = gq; m = gm; }
		else { q.x = q.y = q.z = 0.0f; q.w = 1.0f; m.x = m.y = m.z = 0.0f; }
		if ((el & ADGPU_RLIST_GENROT_MASK) == 0) {
			int rb = (el & ADGPU_RLIST_RBONDID_MASK) >> ADGPU_RLIST_RBONDID_SHIFT;
			float ang = g[6 + rb] * DEG_TO_RAD * 0.5f;
			float s = sinf(ang);
			q.x = s * uv[3 * rb]; q.y = s * uv[3 * rb + 1]; q.z = s * uv[3 * rb + 2];
			q.w = cosf(ang);
			m.x = mv[3 * rb]; m.y = mv[3 * rb + 1]; m.z = mv[3 * rb + 2];
			p.x -= m.x; p.y -= m.y; p.z -= m.z;
		}
		f3 r = qrot(p, q);
		xyz[atom].x = r.x + m.x; xyz[atom].y = r.y + m.y; xyz[atom].z = r.z + m.z;
	}
}

/* ---- scorer -------------------------------------------------------------- */
void oracle_score(const adgpu_gpudata* d, const float* genotype, float* energy_out, float* fgrad, float* terms)
{
	const adgpu_dockpars* dp = &d->dockpars;
	const adgpu_kc_interintra* ii = d->pKerconst_interintra;
	const adgpu_kc_intra* kin = d->pKerconst_intra;
	const uint32_t* pairs = d->pKerconst_intracontrib->intraE_contributors_const;
	f3 xyz[ADGPU_MAX_ATOMS];
	i3 grad[ADGPU_MAX_ATOMS];
	int ggene[ADGPU_MAX_GENES + 1];
	float t[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
	f4 gq; f3 gm;
	float sin_theta, sin_half, is_theta_gt_pi;
	const int want_grad = fgrad != NULL;

	build_pose(d, genotype, xyz, &gq, &gm, &sin_theta, &sin_half, &is_theta_gt_pi);
	memset(grad, 0, sizeof(grad));
	memset(ggene, 0, sizeof(ggene));
	double e_sum = 0.0;   /* only the final value is compared; sum order is not the reference's */
	float energy = 0.0f;

	/* inter-molecular, cuda/calcMergeEneGra.cu:195-413 and cuda/calcenergy.cu:236-333 */
	const uint32_t g1 = (uint32_t)dp->gridsize_x, g2 = (uint32_t)dp->gridsize_x_times_y;
	const uint32_t g3 = (uint32_t)dp->gridsize_x_times_y_times_z;
	const float inv_sp = 1.0f / dp->grid_spacing;
	for (int a = 0; a < dp->num_of_atoms; a++) {
		if (ii->ignore_inter_const[a] > 0) continue;
		float x = xyz[a].x, y = xyz[a].y, z = xyz[a].z;
		float q = ii->atom_charges_const[a];
		uint32_t ty = ii->atom_types_map_const[a];
		if (x < 0 || y < 0 || z < 0 || x >= dp->gridsize_x - 1 || y >= dp->gridsize_y - 1 || z >= dp->gridsize_z - 1) {
			energy += 16777216.0f;
			t[7] += 1.0f;
			grad[a].x += 16777216; grad[a].y += 16777216; grad[a].z += 16777216;
			continue;
		}
		float xl = floorf(x), yl = floorf(y), zl = floorf(z);
		uint64_t cell = (uint64_t)(uint32_t)xl + (uint64_t)(uint32_t)yl * g1 + (uint64_t)(uint32_t)zl * g2;
		const float* base = d->pMem_fgrids + (cell << 2);
		float dx = x - xl, omdx = 1.0f - dx, dy = y - yl, omdy = 1.0f - dy, dz = z - zl, omdz = 1.0f - dz;
		float w[8];
		w[0] = omdx * omdy * omdz; w[1] = omdx * dy * omdz; w[2] = omdx * omdy * dz; w[3] = omdx * dy * dz;
		w[4] = dx * omdy * omdz;   w[5] = dx * dy * omdz;   w[6] = dx * omdy * dz;   w[7] = dx * dy * dz;
		float gx = 0, gy = 0, gz = 0;
		for (int m = 0; m < 3; m++) {
			uint64_t map = (m == 0) ? ty : (uint64_t)dp->num_of_map_atypes + (m - 1);
			const float* c = base + ((map * g3) << 2);
			float v = c[0] * w[0] + c[1] * w[1] + c[2] * w[2] + c[3] * w[3] + c[4] * w[4] + c[5] * w[5] + c[6] * w[6] + c[7] * w[7];
			float s = (m == 0) ? 1.0f : (m == 1 ? q : fabsf(q));
			float e = (m == 0) ? v : s * v;
			energy += e;
			t[m] += e;
			if (want_grad) {
				/* idx 0..7 = 000, 010, 001, 011, 100, 110, 101, 111 (common/defines.h:52-62) */
				float cx = omdz * (omdy * (c[4] - c[0]) + dy * (c[5] - c[1])) + dz * (omdy * (c[6] - c[2]) + dy * (c[7] - c[3]));
				float cy = omdz * (omdx * (c[1] - c[0]) + dx * (c[5] - c[4])) + dz * (omdx * (c[3] - c[2]) + dx * (c[7] - c[6]));
				float cz = omdy * (omdx * (c[2] - c[0]) + dx * (c[6] - c[4])) + dy * (omdx * (c[3] - c[1]) + dx * (c[7] - c[5]));
				if (m == 0) { gx = cx * inv_sp; gy = cy * inv_sp; gz = cz * inv_sp; }
				else {
					float q1 = (m == 1) ? q * inv_sp : fabsf(q * inv_sp);
					gx += q1 * cx; gy += q1 * cy; gz += q1 * cz;
				}
			}
		}
		if (want_grad) { grad[a].x += quant(gx); grad[a].y += quant(gy); grad[a].z += quant(gz); }
	}

	/* intra-molecular, cuda/calcMergeEneGra.cu:418-602 and cuda/calcenergy.cu:336-446 */
	const float delta_distance = 0.5f * dp->smooth;
	for (int p = 0; p < dp->num_of_intraE_contributors; p++) {
		uint32_t a1 = pairs[2 * p], a2 = pairs[2 * p + 1];
		float subx = xyz[a1].x - xyz[a2].x, suby = xyz[a1].y - xyz[a2].y, subz = xyz[a1].z - xyz[a2].z;
		float dist = sqrtf(subx * subx + suby * suby + subz * subz);
		float r = dist * dp->grid_spacing;
		uint32_t t1 = ii->atom_types_const[a1], t2 = ii->atom_types_const[a2];
		uint32_t h1 = kin->atom_types_reqm_const[t1], h2 = kin->atom_types_reqm_const[t2];
		float vbond = G_CG_G0 * (float)(((h1 == ATYPE_CG_IDX) && (h2 == ATYPE_G0_IDX)) || ((h1 == ATYPE_G0_IDX) && (h2 == ATYPE_CG_IDX)));
		float pg = vbond;
		energy += vbond * r;
		t[6] += vbond * r;
		if (r < 8.0f) {
			uint32_t idx = t1 * (uint32_t)dp->num_of_atypes + t2;
			unsigned short exps = kin->VWpars_exp_const[idx];
			int m = (exps & 0xFF00) >> 8, n = exps & 0xFF;
			float opt = kin->reqm_AB_const[idx];
			float delta = opt - r, sd;
			if (fabsf(delta) >= delta_distance) sd = r + copysignf(delta_distance, delta);
			else sd = opt;
			float rmn = powf(sd, (float)(m - n)), rm = powf(sd, (float)(-m));
			float AC = kin->VWpars_AC_const[idx], BD = kin->VWpars_BD_const[idx];
			float ev = (AC - rmn * BD) * rm;
			energy += ev;
			t[3] += ev;
			pg += ((float)n * BD * rmn - (float)m * AC) * rm / sd;
		}
		if (r < 20.48f) {
			if (r < dp->elec_min_distance) r = dp->elec_min_distance;
			float q1 = ii->atom_charges_const[a1], q2 = ii->atom_charges_const[a2];
			float d2 = r * r;
			float desolv = ((kin->dspars_S_const[t1] + dp->qasp * fabsf(q1)) * kin->dspars_V_const[t2] +
			                (kin->dspars_S_const[t2] + dp->qasp * fabsf(q2)) * kin->dspars_V_const[t1]) *
			               (dp->coeff_desolv * (12.96f - 0.1063f * d2 * (1.0f - 0.001947f * d2)) /
			                (12.96f + d2 * (0.4137f + d2 * (0.00357f + 0.000112f * d2))));
			float shift = r + 1.26366f;
			float s2 = shift * shift;
			float diel = 1.10859f / s2 + 0.010358f;
			float es = dp->coeff_elec * q1 * q2 / r;
			energy += diel * es + desolv;
			t[4] += diel * es;
			t[5] += desolv;
			pg += -(es / r) * diel - es * 2.21718f / (s2 * shift) - 0.0771605f * r * desolv;
		}
		if (want_grad) {
			float gdd = -pg / dist;
			int ix = quant(subx * gdd), iy = quant(suby * gdd), iz = quant(subz * gdd);
			grad[a1].x -= ix; grad[a1].y -= iy; grad[a1].z -= iz;
			grad[a2].x += ix; grad[a2].y += iy; grad[a2].z += iz;
		}
	}
	(void)e_sum;
	*energy_out = energy;
	if (terms) memcpy(terms, t, sizeof(t));
	if (!want_grad) return;

	/* torque and total force over the ligand, cuda/calcMergeEneGra.cu:608-661 */
	f3 torque = { 0, 0, 0 };
	float gx = 0, gy = 0, gz = 0;
	for (int a = 0; a < dp->true_ligand_atoms; a++) {
		f3 r = { (xyz[a].x - gm.x) * dp->grid_spacing, (xyz[a].y - gm.y) * dp->grid_spacing, (xyz[a].z - gm.z) * dp->grid_spacing };
		f3 f = { ONEOVERTERMSCALE * (float)grad[a].x, ONEOVERTERMSCALE * (float)grad[a].y, ONEOVERTERMSCALE * (float)grad[a].z };
		gx += f.x; gy += f.y; gz += f.z;
		f3 tr = cross3(r, f);
		torque.x += tr.x; torque.y += tr.y; torque.z += tr.z;
	}
	if (dp->true_ligand_atoms) {
		/* translation genes, :676-689 */
		ggene[0] = quant(gx * dp->grid_spacing);
		ggene[1] = quant(gy * dp->grid_spacing);
		ggene[2] = quant(gz * dp->grid_spacing);
		/* orientation genes, :695-815 */
		float phi = genotype[3] * DEG_TO_RAD, theta = genotype[4] * DEG_TO_RAD, rotangle = genotype[5] * DEG_TO_RAD;
		float tl = sqrtf(torque.x * torque.x + torque.y * torque.y + torque.z * torque.z);
		float oscale = (tl < INFINITESIMAL_RADIAN) ? 1.0f : tl * INV_INFINITESIMAL_RADIAN;
		float tscale = (tl < INFINITESIMAL_RADIAN) ? 0.5f - tl * tl / 48.0f : sinf(HALF_INFINITESIMAL_RADIAN) / tl;
		f4 qt = { torque.x * tscale, torque.y * tscale, torque.z * tscale,
		          (tl < INFINITESIMAL_RADIAN) ? 1.0f - tl * tl * 0.125f : cosf(HALF_INFINITESIMAL_RADIAN) };
		f4 target = qmul(qt, gq);
		float cur_phi = fmod_pi2(PI_TIMES_2 + phi);
		float cur_theta = fmod_pi2(PI_TIMES_2 + theta);
		float cur_rot = fmod_pi2(PI_TIMES_2 + rotangle);
		float tgt_rot = 2.0f * fast_acos(target.w);
		float sin_ang = sqrtf(1.0f - target.w * target.w);
		float tgt_theta = PI_TIMES_2 + is_theta_gt_pi * fast_acos(target.z / sin_ang);
		float tgt_phi = fmod_pi2(atan2f(is_theta_gt_pi * target.y, is_theta_gt_pi * target.x) + PI_TIMES_2);
		float gphi = oscale * (fmod_pi2(tgt_phi - cur_phi + PI_FLOAT) - PI_FLOAT);
		float gth = oscale * (fmod_pi2(tgt_theta - cur_theta + PI_FLOAT) - PI_FLOAT);
		float grot = oscale * (fmod_pi2(tgt_rot - cur_rot + PI_FLOAT) - PI_FLOAT);
		float corr = 4.0f * sin_half * sin_half;
		ggene[3] = quant(gphi * sin_theta * sin_theta * corr * DEG_TO_RAD);
		ggene[4] = quant(gth * corr * DEG_TO_RAD);
		ggene[5] = quant(grot * DEG_TO_RAD);
	}
	/* torsion genes, cuda/calcMergeEneGra.cu:819-880 */
	int ntors = dp->num_of_genes - 6;
	const int* rb = d->pKerconst_grads->rotbonds;
	const int* rba = d->pKerconst_grads->rotbonds_atoms;
	const int* nrot = d->pKerconst_grads->num_rotating_atoms_per_rotbond;
	for (int k = 0; k < ntors; k++) {
		int a1 = rb[2 * k], a2 = rb[2 * k + 1];
		f3 ref = xyz[a1];
		f3 ax = { xyz[a2].x - ref.x, xyz[a2].y - ref.y, xyz[a2].z - ref.z };
		float l = 1.0f / sqrtf(ax.x * ax.x + ax.y * ax.y + ax.z * ax.z);
		ax.x *= l; ax.y *= l; ax.z *= l;
		for (int c = 0; c < nrot[k]; c++) {
			int la = rba[ADGPU_MAX_ATOMS * k + c];
			f3 r = { xyz[la].x - ref.x, xyz[la].y - ref.y, xyz[la].z - ref.z };
			f3 f = { ONEOVERTERMSCALE * (float)grad[la].x, ONEOVERTERMSCALE * (float)grad[la].y, ONEOVERTERMSCALE * (float)grad[la].z };
			f3 tq = cross3(r, f);
			float on_axis = (ax.x * tq.x + ax.y * tq.y + ax.z * tq.z) * dp->grid_spacing;
			ggene[6 + k] += quant(on_axis * DEG_TO_RAD);
		}
	}
	/* fixed point -> float, then Angstrom/radian scaling, :883-899 */
	for (int gi = 0; gi < dp->num_of_genes; gi++) {
		fgrad[gi] = ONEOVERTERMSCALE * (float)ggene[gi];
		if (gi >= 3) fgrad[gi] *= dp->grid_spacing * dp->grid_spacing * SCFACTOR_ANGSTROM_RADIAN;
	}
}

/* ---- threading helper ----------------------------------------------------- */
typedef void (*block_fn)(const void* ctx, uint32_t block);
typedef struct { const void* ctx; block_fn fn; uint32_t blocks; uint32_t next; pthread_mutex_t mu; } pool_t;

static void* pool_worker(void* arg)
{
	pool_t* p = (pool_t*)arg;
	for (;;) {
		pthread_mutex_lock(&p->mu);
		uint32_t b = p->next++;
		pthread_mutex_unlock(&p->mu);
		if (b >= p->blocks) break;
		p->fn(p->ctx, b);
	}
	return NULL;
}

static void run_blocks(const void* ctx, block_fn fn, uint32_t blocks, int nthreads)
{
	if (nthreads <= 1 || blocks < 2) {
		for (uint32_t b = 0; b < blocks; b++) fn(ctx, b);
		return;
	}
	if ((uint32_t)nthreads > blocks) nthreads = (int)blocks;
	pool_t p = { ctx, fn, blocks, 0, PTHREAD_MUTEX_INITIALIZER };
	pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
	for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, pool_worker, &p);
	for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
	free(th);
}

/* ---- PRNG (cuda/auxiliary_genetic.cu:29-79) ---------------------------- */
static inline uint32_t lcg(uint32_t* states, uint32_t idx)
{
	uint32_t s = 1103515245u * states[idx] + 12345u;
	states[idx] = s;
	return s;
}
static inline float lcgf(uint32_t* states, uint32_t idx)
{
	return ((float)lcg(states, idx) / 4294967296.0f) * 0.999999f;
}
static inline void map_angle(float* a)
{
	while (*a >= 360.0f) *a -= 360.0f;
	while (*a < 0.0f) *a += 360.0f;
}

/* ---- kernel1 / kernel2 ------------------------------------------------------ */
typedef struct { const adgpu_gpudata* d; uint32_t threads; const float* cc; const float* ec; float* cn; float* en; } kctx;

static void initpop_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	float e;
	oracle_score(k->d, k->cn + (size_t)b * GSTRIDE, &e, NULL, NULL);
	k->en[b] = e;
	k->d->pMem_evals_of_new_entities[b] = 1;
}

/* gpu_calc_initpop_kernel, cuda/kernel1.cu:26-55 */
void oracle_calc_initpop(const adgpu_gpudata* d, uint32_t blocks, float* conf_cur, float* e_cur, int nthreads)
{
	kctx k = { d, 0, NULL, NULL, conf_cur, e_cur };
	run_blocks(&k, initpop_block, blocks, nthreads);
}

/* gpu_sum_evals_kernel, cuda/kernel2.cu:26-52 */
void oracle_sum_evals(const adgpu_gpudata* d, uint32_t blocks)
{
	for (uint32_t b = 0; b < blocks; b++) {
		int s = 0;
		for (int e = 0; e < d->dockpars.pop_size; e++) s += d->pMem_evals_of_new_entities[b * d->dockpars.pop_size + e];
		d->pMem_gpu_evals_of_runs[b] += s;
	}
}

/* ---- kernel4: one GA generation (cuda/kernel4.cu:28-304) --------------------- */

/* WARPMINIMUMEXCHANGE / WARPMINIMUM2 of cuda/kernels.cu:47-64 on 32 lanes:
 * a compare-exchange network after which lane 0 holds the minimum. */
static void warp_minimum2(float* v, int* k)
{
	for (int mask = 1; mask < 32; mask <<= 1) {
		float nv[32]; int nk[32];
		for (int t = 0; t < 32; t++) {
			int o = t ^ mask;
			float v1 = v[t], v2 = v[o];
			int flag = ((v1 < v2) ^ (t > o)) && (v1 != v2);
			nk[t] = flag ? k[t] : k[o];
			nv[t] = flag ? v1 : v2;
		}
		memcpy(v, nv, sizeof(nv)); memcpy(k, nk, sizeof(nk));
	}
}

static void ga_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	const adgpu_gpudata* d = k->d;
	const adgpu_dockpars* dp = &d->dockpars;
	const int P = dp->pop_size, T = (int)k->threads, NG = dp->num_of_genes;
	uint32_t* st = d->pMem_prng_states;
	if (b % (uint32_t)P == 0) {
		/* elitism: per-thread scan, warp arg-min, then warp 0 over the warps' minima */
		int nwarps = (T + 31) / 32;
		float wbest_e[32]; int wbest_id[32];
		for (int w = 0; w < nwarps; w++) {
			float v[32]; int id[32];
			for (int l = 0; l < 32; l++) {
				int t = w * 32 + l;
				if (t < P && t < T) { id[l] = (int)b + t; v[l] = k->ec[b + t]; }
				else { id[l] = -1; v[l] = FLT_MAX; }
				if (t < T)
					for (int i = (int)b + T + t; i < (int)b + P; i += T) {
						float e = k->ec[i];
						if (e < v[l]) { id[l] = i; v[l] = e; }
					}
			}
			warp_minimum2(v, id);
			wbest_id[w] = id[0];
			wbest_e[w] = fminf(MAXENERGY, v[0]);
		}
		float v[32]; int id[32];
		for (int l = 0; l < 32; l++) {
			if (l < T / 32) { id[l] = wbest_id[l]; v[l] = wbest_e[l]; }
			else { id[l] = -1; v[l] = FLT_MAX; }
		}
		warp_minimum2(v, id);
		k->en[b] = v[0];
		d->pMem_evals_of_new_entities[b] = 0;
		for (int i = 0; i < NG; i++) k->cn[(size_t)b * GSTRIDE + i] = k->cc[(size_t)id[0] * GSTRIDE + i];
		return;
	}
	float rn[10];
	for (int i = 0; i < 10; i++) rn[i] = lcgf(st, b * (uint32_t)T + (uint32_t)(i % T));
	int run = (int)b / P;
	int cand[4]; float ce[4];
	for (int i = 0; i < 4; i++) {
		cand[i] = (int)((float)P * rn[i]);
		ce[i] = k->ec[run * P + cand[i]];
	}
	int par[2];
	for (int i = 0; i < 2; i++) {
		if (ce[2 * i] < ce[2 * i + 1]) par[i] = (rn[4 + i] < dp->tournament_rate) ? cand[2 * i] : cand[2 * i + 1];
		else par[i] = (rn[4 + i] < dp->tournament_rate) ? cand[2 * i + 1] : cand[2 * i];
	}
	float off[ADGPU_MAX_GENES];
	const float* p0 = k->cc + (size_t)(run * P + par[0]) * GSTRIDE;
	const float* p1 = k->cc + (size_t)(run * P + par[1]) * GSTRIDE;
	if (rn[6] < dp->crossover_rate) {
		int cp0 = (int)((float)(NG - 1) * rn[7]), cp1 = (int)((float)(NG - 1) * rn[8]);
		if (cp1 < cp0) { int tmp = cp1; cp1 = cp0; cp0 = tmp; }
		for (int g = 0; g < NG; g++) {
			if (cp0 != cp1) off[g] = (g <= cp0 || g > cp1) ? p0[g] : p1[g];
			else off[g] = (g <= cp0) ? p0[g] : p1[g];
		}
	} else {
		for (int g = 0; g < NG; g++) off[g] = p0[g];
	}
	/* mutation: gene g is handled by lane g % T, in gene order per lane */
	for (int lane = 0; lane < T; lane++)
		for (int g = lane; g < NG; g += T) {
			uint32_t si = b * (uint32_t)T + (uint32_t)lane;
			if (lcgf(st, si) < dp->mutation_rate) {
				if (g < 3) off[g] += dp->abs_max_dmov * (2.0f * lcgf(st, si) - 1.0f);
				else { off[g] += dp->abs_max_dang * (2.0f * lcgf(st, si) - 1.0f); map_angle(&off[g]); }
			}
		}
	float e;
	oracle_score(d, off, &e, NULL, NULL);
	k->en[b] = e;
	d->pMem_evals_of_new_entities[b] = 1;
	for (int g = 0; g < NG; g++) k->cn[(size_t)b * GSTRIDE + g] = off[g];
}

void oracle_gen_and_eval_newpops(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                                 const float* conf_cur, const float* e_cur, float* conf_next, float* e_next,
                                 int nthreads)
{
	kctx k = { d, threads, conf_cur, e_cur, conf_next, e_next };
	run_blocks(&k, ga_block, blocks, nthreads);
}

/* ---- local searches ---------------------------------------------------------- */

/* entity selection shared by every LS kernel, e.g. cuda/kernel_ad.cu:116-127 */
static int ls_entity(const adgpu_gpudata* d, uint32_t b, uint32_t threads)
{
	const adgpu_dockpars* dp = &d->dockpars;
	int ent = (int)(b % dp->num_of_lsentities);
	if (ent == 0 && 100.0f * lcgf(d->pMem_prng_states, b * threads) > dp->lsearch_rate)
		ent = (int)dp->num_of_lsentities;
	return ent;
}

/* gpu_perform_LS_kernel (Solis-Wets, SWAT3), cuda/kernel3.cu:30-308 */
static void sw_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	const adgpu_gpudata* d = k->d;
	const adgpu_dockpars* dp = &d->dockpars;
	const uint32_t T = k->threads;
	uint32_t* st = d->pMem_prng_states;
	int run = (int)(b / dp->num_of_lsentities);
	int ent = ls_entity(d, b, T);
	size_t off = (size_t)(run * dp->pop_size + ent) * GSTRIDE;
	float cur_e = k->en[run * dp->pop_size + ent];
	float rho = 1.0f;
	int succ = 0, fail = 0, iters = 0, evals = 0;
	float gen[ADGPU_MAX_GENES], cand[ADGPU_MAX_GENES], dev[ADGPU_MAX_GENES], bias[ADGPU_MAX_GENES];
	const int NG = dp->num_of_genes;
	for (int g = 0; g < NG; g++) { gen[g] = k->cn[off + g]; bias[g] = 0.0f; cand[g] = gen[g]; dev[g] = 0.0f; }
	const int gs = (dp->true_ligand_atoms == 0) * 6;
	const float lig_scale = 1.0f / sqrtf((float)dp->num_of_atoms);
	const float gene_scale = 1.0f / sqrtf((float)NG);
	while (iters < (int)dp->max_num_of_iters && rho > dp->rho_lower_bound) {
		for (uint32_t lane = 0; lane < T; lane++)
			for (int g = gs + (int)lane; g < NG; g += (int)T) {
				uint32_t si = b * T + lane;
				float r1 = lcgf(st, si);
				float r2 = lcgf(st, si);
				dev[g] = rho * (2.0f * r1 - 1.0f) * (float)(r2 < gene_scale);
				if (g < 3) dev[g] *= dp->base_dmov_mul_sqrt3;
				else if (g < 6) dev[g] *= dp->base_dang_mul_sqrt3 * lig_scale;
				else dev[g] *= dp->base_dang_mul_sqrt3 * gene_scale;
			}
		for (int g = gs; g < NG; g++) cand[g] = gen[g] + dev[g] + bias[g];
		float ce;
		oracle_score(d, cand, &ce, NULL, NULL);
		evals++;
		if (ce < cur_e) {
			for (int g = gs; g < NG; g++) { gen[g] = cand[g]; bias[g] = 0.6f * bias[g] + 0.4f * dev[g]; }
			cur_e = ce; succ++; fail = 0;
		} else {
			for (int g = gs; g < NG; g++) cand[g] = gen[g] - dev[g] - bias[g];
			oracle_score(d, cand, &ce, NULL, NULL);
			evals++;
			if (ce < cur_e) {
				for (int g = gs; g < NG; g++) { gen[g] = cand[g]; bias[g] = 0.6f * bias[g] - 0.4f * dev[g]; }
				cur_e = ce; succ++; fail = 0;
			} else {
				for (int g = gs; g < NG; g++) bias[g] = 0.5f * bias[g];
				succ = 0; fail++;
			}
		}
		iters++;
		if (succ >= (int)dp->cons_limit) { rho *= LS_EXP_FACTOR; succ = 0; }
		else if (fail >= (int)dp->cons_limit) { rho *= LS_CONT_FACTOR; fail = 0; }
	}
	d->pMem_evals_of_new_entities[run * dp->pop_size + ent] += evals;
	k->en[run * dp->pop_size + ent] = cur_e;
	for (int g = gs; g < NG; g++) {
		if (g >= 3) map_angle(&gen[g]);
		k->cn[off + g] = gen[g];
	}
}

void oracle_perform_ls(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads, float* conf_next, float* e_next, int nthreads)
{
	kctx k = { d, threads, NULL, NULL, conf_next, e_next };
	run_blocks(&k, sw_block, blocks, nthreads);
}

/* gpu_gradient_minAD_kernel (ADADELTA, rho 0.8, eps 1e-2, success/fail stop), cuda/kernel_ad.cu:60-393 */
static void ad_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	const adgpu_gpudata* d = k->d;
	const adgpu_dockpars* dp = &d->dockpars;
	const float RHO = 0.8f, EPS = 1e-2f;
	int run = (int)(b / dp->num_of_lsentities);
	int ent = ls_entity(d, b, k->threads);
	size_t off = (size_t)(run * dp->pop_size + ent) * GSTRIDE;
	const int NG = dp->num_of_genes;
	float gen[ADGPU_MAX_GENES], best[ADGPU_MAX_GENES], grad[ADGPU_MAX_GENES], sqd[ADGPU_MAX_GENES], sqg[ADGPU_MAX_GENES];
	for (int g = 0; g < NG; g++) { gen[g] = k->cn[off + g]; grad[g] = 0; sqg[g] = 0; sqd[g] = 0; best[g] = gen[g]; }
	float best_e = INFINITY, energy, rho = 1.0f;
	int succ = 0, fail = 0;
	uint32_t it = 0;
	do {
		oracle_score(d, gen, &energy, grad, NULL);
		for (int g = 0; g < NG; g++) {
			if (energy < best_e) best[g] = gen[g];
			sqg[g] = RHO * sqg[g] + (1.0f - RHO) * grad[g] * grad[g];
			float delta = -1.0f * grad[g] * sqrtf((float)(sqd[g] + EPS) / (float)(sqg[g] + EPS));
			sqd[g] = RHO * sqd[g] + (1.0f - RHO) * delta * delta;
			gen[g] += delta;
		}
		it++;
		if (energy < best_e) { best_e = energy; succ++; fail = 0; }
		else { succ = 0; fail++; }
		if (succ >= 4) { rho *= LS_EXP_FACTOR; succ = 0; }
		else if (fail >= 4) { rho *= LS_CONT_FACTOR; fail = 0; }
	} while (it < dp->max_num_of_iters && rho > 0.01f);
	for (int g = 3; g < NG; g++) map_angle(&best[g]);
	for (int g = 0; g < NG; g++) k->cn[off + g] = best[g];
	d->pMem_evals_of_new_entities[run * dp->pop_size + ent] += (int)it;
	k->en[run * dp->pop_size + ent] = best_e;
}

void oracle_gradient_minad(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads, float* conf_next, float* e_next, int nthreads)
{
	kctx k = { d, threads, NULL, NULL, conf_next, e_next };
	run_blocks(&k, ad_block, blocks, nthreads);
}

/* gpu_gradient_minAdam_kernel (bias-corrected ADAM, fixed iteration count), cuda/kernel_adam.cu:55-396 */
static void adam_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	const adgpu_gpudata* d = k->d;
	const adgpu_dockpars* dp = &d->dockpars;
	int run = (int)(b / dp->num_of_lsentities);
	int ent = ls_entity(d, b, k->threads);
	size_t off = (size_t)(run * dp->pop_size + ent) * GSTRIDE;
	const int NG = dp->num_of_genes;
	float gen[ADGPU_MAX_GENES], best[ADGPU_MAX_GENES], grad[ADGPU_MAX_GENES], mt[ADGPU_MAX_GENES], vt[ADGPU_MAX_GENES];
	for (int g = 0; g < NG; g++) { gen[g] = k->cn[off + g]; grad[g] = 0; mt[g] = 0; vt[g] = 0; best[g] = gen[g]; }
	float best_e = INFINITY, energy;
	uint32_t it = 0;
	do {
		oracle_score(d, gen, &energy, grad, NULL);
		float b1p = 1.0f - powf(dp->adam_beta1, 1.0f + (float)it);
		float b2p = 1.0f - powf(dp->adam_beta2, 1.0f + (float)it);
		for (int g = 0; g < NG; g++) {
			if (energy < best_e) best[g] = gen[g];
			mt[g] = dp->adam_beta1 * mt[g] + (1.0f - dp->adam_beta1) * grad[g];
			vt[g] = dp->adam_beta2 * vt[g] + (1.0f - dp->adam_beta2) * grad[g] * grad[g];
			float mp = mt[g] / b1p, vp = vt[g] / b2p;
			gen[g] -= mp / (sqrtf(vp) + dp->adam_epsilon);
		}
		it++;
		if (energy < best_e) best_e = energy;
	} while (it < dp->max_num_of_iters);
	for (int g = 3; g < NG; g++) map_angle(&best[g]);
	for (int g = 0; g < NG; g++) k->cn[off + g] = best[g];
	d->pMem_evals_of_new_entities[run * dp->pop_size + ent] += (int)it;
	k->en[run * dp->pop_size + ent] = best_e;
}

void oracle_gradient_minadam(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads, float* conf_next, float* e_next, int nthreads)
{
	kctx k = { d, threads, NULL, NULL, conf_next, e_next };
	run_blocks(&k, adam_block, blocks, nthreads);
}

/* gradient_minFire (FIRE), device/kernel_fire.cl:76-895.  The initial gradient
 * is taken from the merged scorer (the OpenCL kernel calls its separate
 * gradient-only routine, device/calcgradient.cl:109, for that one step). */
static void fire_block(const void* c, uint32_t b)
{
	const kctx* k = (const kctx*)c;
	const adgpu_gpudata* d = k->d;
	const adgpu_dockpars* dp = &d->dockpars;
	const float DT_INC = 1.2f, DT_DEC = 0.8f, ALPHA_START = 0.2f, ALPHA_DEC = 0.99f;
	const float DT_MAX = 10.0f, DT_MIN = 1e-6f;
	const uint32_t SUCCESS_MIN = 5;
	int run = (int)(b / dp->num_of_lsentities);
	int ent = ls_entity(d, b, k->threads);
	size_t off = (size_t)(run * dp->pop_size + ent) * GSTRIDE;
	const int NG = dp->num_of_genes;
	float gen[ADGPU_MAX_GENES], grad[ADGPU_MAX_GENES], cgen[ADGPU_MAX_GENES], cgrad[ADGPU_MAX_GENES];
	float vel[ADGPU_MAX_GENES], best[ADGPU_MAX_GENES];
	float energy = k->en[run * dp->pop_size + ent], ce, dummy;
	for (int g = 0; g < NG; g++) gen[g] = k->cn[off + g];
	oracle_score(d, gen, &dummy, grad, NULL);
	float alpha = ALPHA_START, dt = DT_MAX / 3.0f;
	uint32_t count_success = 0, it = 0;
	float s = 0.0f;
	for (int g = 0; g < NG; g++) s += grad[g] * grad[g];
	float inv = ALPHA_START * (1.0f / sqrtf(s));
	for (int g = 0; g < NG; g++) vel[g] = -grad[g] * inv;
	float best_e = energy;
	for (int g = 0; g < NG; g++) best[g] = gen[g];
	do {
		for (int g = 0; g < NG; g++) cgen[g] = gen[g] + dt * vel[g];
		oracle_score(d, cgen, &ce, cgrad, NULL);
		float power = 0.0f;
		for (int g = 0; g < NG; g++) power += -cgrad[g] * vel[g];
		if (power < 0.0f) {
			s = 0.0f;
			for (int g = 0; g < NG; g++) s += grad[g] * grad[g];
			inv = ALPHA_START * (1.0f / sqrtf(s));
			for (int g = 0; g < NG; g++) vel[g] = -grad[g] * inv;
			count_success = 0;
			alpha = ALPHA_START;
			dt = dt * DT_DEC;
		} else {
			count_success++;
			if (count_success > SUCCESS_MIN) {
				dt = fminf(dt * DT_INC, DT_MAX);
				alpha = alpha * ALPHA_DEC;
			}
		}
		energy = ce;
		for (int g = 0; g < NG; g++) { gen[g] = cgen[g]; grad[g] = cgrad[g]; }
		s = 0.0f;
		for (int g = 0; g < NG; g++) s += grad[g] * grad[g];
		float inv_gn = 1.0f / sqrtf(s);
		float vn = 0.0f;
		for (int g = 0; g < NG; g++) vn += vel[g] * vel[g];
		vn = sqrtf(vn);
		float vdg = alpha * vn * inv_gn;
		for (int g = 0; g < NG; g++) vel[g] = (1.0f - alpha) * vel[g] - grad[g] * vdg;
		it++;
		if (energy < best_e) {
			best_e = energy;
			for (int g = 0; g < NG; g++) best[g] = gen[g];
		}
	} while (it < dp->max_num_of_iters && dt > DT_MIN);
	d->pMem_evals_of_new_entities[run * dp->pop_size + ent] += (int)it;
	k->en[run * dp->pop_size + ent] = best_e;
	for (int g = 3; g < NG; g++) map_angle(&best[g]);
	for (int g = 0; g < NG; g++) k->cn[off + g] = best[g];
}

void oracle_gradient_minfire(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads, float* conf_next, float* e_next, int nthreads)
{
	kctx k = { d, threads, NULL, NULL, conf_next, e_next };
	run_blocks(&k, fire_block, blocks, nthreads);
}

/* ---- batch scorer ------------------------------------------------------------- */
typedef struct { const adgpu_gpudata* d; const float* g; float* e; float* gr; } sctx;
static void score_block(const void* c, uint32_t b)
{
	const sctx* s = (const sctx*)c;
	oracle_score(s->d, s->g + (size_t)b * GSTRIDE, &s->e[b], s->gr ? s->gr + (size_t)b * GSTRIDE : NULL, NULL);
}

void oracle_score_batch(const adgpu_gpudata* d, uint32_t n, const float* genotypes, float* energies, float* gradients, int nthreads)
{
	sctx s = { d, genotypes, energies, gradients };
	run_blocks(&s, score_block, n, nthreads);
}
