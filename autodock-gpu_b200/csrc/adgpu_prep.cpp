// adgpu_prep.cpp -- the input side of the hot path: AutoDock-4 grid maps and
// PDBQT ligands/flexible residues turned into the reference-layout tables the
// kernel API consumes, restated from the reference's host front end:
//   .fld/.map reading            host/src/processgrid.cpp:28-253
//   ligand/flexres parsing       host/src/processligand.cpp:40-193, 1124-1322
//   bond perception              host/src/processligand.cpp:459-733
//   intramolecular pair list     host/src/processligand.cpp:250-457
//   vdW/H-bond/desolv parameters host/src/processligand.cpp:749-1066 (AD4.1 tables)
//   torsion vectors              host/src/processligand.cpp:1068-1122
//   initial population           host/src/getparameters.cpp:2543-2631
//   table packing + rotation list host/src/calcenergy.cpp:31-488
// Only the base AD4 atom types are supported (no --derivtype / --modpair).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>
#include <atomic>
#include <string>
#include <vector>
#include <algorithm>
#include "adgpu_prep.h"

namespace adgpu {

adgpu_status fail(adgpu_status st, const std::string& msg);

// ---------------------------------------------------------------------------
// CMWC4096 generator (G. Marsaglia, "Random number generators", JMASM 2(1), 2003),
// seeded the way the reference seeds its host generator (LocalRNG,
// host/inc/miscellaneous.h:146-219) so equal seeds give equal populations.
// ---------------------------------------------------------------------------
class Cmwc4096 {
	uint32_t Q[4096], i = 4095, c = 362436;
	static constexpr uint32_t kPhi = 0x9e3779b9u;
public:
	explicit Cmwc4096(const uint32_t seed[3])
	{
		uint32_t x = seed[0], y, z;
		if (!seed[2]) {
			if (!seed[1]) { y = x + kPhi; z = x + kPhi + kPhi; }
			else { y = seed[1]; z = y + kPhi; }
		} else { y = seed[1]; z = seed[2]; }
		Q[0] = x; Q[1] = y + kPhi; Q[2] = z + kPhi;
		for (uint32_t j = 3; j < 4096; j++) Q[j] = Q[j - 3] ^ Q[j - 2] ^ kPhi ^ j;
		i = 4095; c = 362436;
		do c = next(); while (c >= 809430660u);
		i = 4095;
	}
	uint32_t next()
	{
		const uint64_t a = 18782ULL;
		const uint32_t m = 0xfffffffeu;
		i = (i + 1) & 4095;
		uint64_t t = a * Q[i] + c;
		c = (uint32_t)(t >> 32);
		uint32_t x = (uint32_t)t + c;
		if (x < c) { x++; c++; }
		return (Q[i] = m - x);
	}
	float next_float()
	{
		float r = 0.0f;
		while (r <= 0.0f || r >= 1.0f) r = (float)next() / 4294967295.0f;
		return r;
	}
};

// ---------------------------------------------------------------------------
// grid maps
// ---------------------------------------------------------------------------

// AutoGrid map values: integer part and decimal part accumulated separately
// and joined with one float division (the reference's map2float,
// host/src/miscellaneous.cpp:30-71, so values are bit-identical).
static float parse_map_value(const char* c)
{
	float result;
	bool negative = false;
	if (*c == '-') { negative = true; c++; }
	int len = (int)strlen(c);
	if (len > 9) {
		const char* dp = strchr(c, '.');
		if (dp) {
			int d = (int)(dp - c);
			if (d > 9 || len - d > 9) {
				result = strtof(c, nullptr);
				return negative ? -result : result;
			}
		}
	}
	int number = 0;
	while (*c >= '0' && *c <= '9') { number = number * 10 + (*c - '0'); c++; }
	if (*c == '.') c++;
	int decimal = 0, denom = 1;
	while (*c >= '0' && *c <= '9') { decimal = decimal * 10 + (*c - '0'); denom *= 10; c++; }
	result = (float)number + (float)decimal / ((float)denom);
	return negative ? -result : result;
}

static std::string dirname_of(const std::string& p)
{
	size_t k = p.find_last_of('/');
	return k == std::string::npos ? std::string() : p.substr(0, k);
}

adgpu_status grid_read(const char* fld_path, Grid& g)
{
	std::ifstream fp(fld_path);
	if (!fp) return fail(ADGPU_ERR_ARG, std::string("cannot open fld file ") + fld_path);
	g = Grid();
	std::string line;
	int npts[3] = {0, 0, 0};
	double center[3] = {0, 0, 0};
	std::vector<std::string> files;
	char tmp[256];
	while (std::getline(fp, line)) {
		if (sscanf(line.c_str(), "%255s", tmp) != 1) continue;
		std::string key(tmp);
		if (key == "#SPACING") sscanf(line.c_str() + 8, "%lf", &g.spacing);
		else if (key == "#NELEMENTS") sscanf(line.c_str() + 10, "%d %d %d", &npts[0], &npts[1], &npts[2]);
		else if (key == "#CENTER") sscanf(line.c_str() + 7, "%lf %lf %lf", &center[0], &center[1], &center[2]);
		if (line.find("label=") == 0) {
			sscanf(line.c_str() + 6, "%255s", tmp);
			char* sep = strchr(tmp, '-');
			if (sep) *sep = '\0';
			else { tmp[1] = '\0'; tmp[0] = (char)tolower(tmp[0]); }
			g.types.push_back(tmp);
		}
		if (key == "variable") {
			size_t f = line.find("file=");
			if (f == std::string::npos) return fail(ADGPU_ERR_ARG, "fld: map file names cannot be read");
			sscanf(line.c_str() + f + 5, "%255s", tmp);
			files.push_back(tmp);
		}
	}
	if (g.spacing <= 0 || g.spacing > 1) return fail(ADGPU_ERR_ARG, "fld: grid spacing must be in (0, 1] A");
	for (int k = 0; k < 3; k++) {
		g.dims[k] = npts[k] + 1;
		if (g.dims[k] < 2 || g.dims[k] > 256) return fail(ADGPU_ERR_LIMIT, "fld: each grid dimension must be 2..256 points");
		g.origin[k] = center[k] - (double)npts[k] * 0.5 * g.spacing;
	}
	if (files.size() != g.types.size()) return fail(ADGPU_ERR_ARG, "fld: map labels and file names mismatched");
	if (g.types.size() < 3 || g.types[g.types.size() - 2] != "e" || g.types.back() != "d")
		return fail(ADGPU_ERR_ARG, "fld: expected type maps followed by the e and d maps");
	g.num_map_atypes = (int)g.types.size() - 2;
	const size_t n = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
	g.values.assign(n * g.types.size(), 0.0f);
	const std::string dir = dirname_of(fld_path);
	// One map per thread: each file is read whole, its lines are cut in place
	// (newline -> NUL, so every value is parsed from the same text a line
	// reader would give it) and parsed in order.
	std::vector<std::string> errors(files.size());
	auto read_map = [&](size_t m) {
		const std::string fn = dir.empty() ? files[m] : dir + "/" + files[m];
		FILE* f = fopen(fn.c_str(), "rb");
		if (!f) { errors[m] = "cannot open grid map " + fn; return; }
		std::vector<char> buf;
		char chunk[1 << 16];
		size_t got;
		while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
		fclose(f);
		buf.push_back('\0');
		char* c = buf.data();
		char* end = c + buf.size() - 1;
		auto next_line = [&](char*& ln) -> bool {
			if (c >= end) return false;
			ln = c;
			char* nl = static_cast<char*>(memchr(c, '\n', (size_t)(end - c)));
			if (nl) { *nl = '\0'; c = nl + 1; } else c = end;
			return true;
		};
		char* ln = nullptr;
		do {
			if (!next_line(ln)) { errors[m] = "grid map preamble too short: " + fn; return; }
		} while (strncmp(ln, "CENTER", 6) != 0);
		float* out = g.values.data() + m * n;
		for (size_t p = 0; p < n; p++) {
			if (!next_line(ln)) { errors[m] = "grid map too short: " + fn; return; }
			out[p] = parse_map_value(ln);
		}
	};
	const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
	std::atomic<size_t> next_map(0);
	std::vector<std::thread> pool;
	for (unsigned t = 0; t < std::min<size_t>(hw, files.size()); t++)
		pool.emplace_back([&]() { for (size_t m; (m = next_map.fetch_add(1)) < files.size();) read_map(m); });
	for (auto& t : pool) t.join();
	for (auto& e : errors)
		if (!e.empty()) return fail(ADGPU_ERR_ARG, e);
	return ADGPU_OK;
}

// Binary grid cache: "ADGPUGRD", version, dims, spacing, origin, map count,
// map names (NUL-padded to 8 bytes), then values[map][z][y][x] as float32.
static const char kGridMagic[8] = {'A', 'D', 'G', 'P', 'U', 'G', 'R', 'D'};

adgpu_status grid_save(const Grid& g, const char* path)
{
	FILE* f = fopen(path, "wb");
	if (!f) return fail(ADGPU_ERR_ARG, std::string("cannot create grid cache ") + path);
	const int32_t version = 1, nm = (int32_t)g.types.size();
	bool ok = fwrite(kGridMagic, 1, 8, f) == 8 && fwrite(&version, 4, 1, f) == 1 && fwrite(g.dims, 4, 3, f) == 3 &&
	          fwrite(&g.spacing, 8, 1, f) == 1 && fwrite(g.origin, 8, 3, f) == 3 && fwrite(&nm, 4, 1, f) == 1;
	for (int m = 0; ok && m < nm; m++) {
		char name[8] = {0};
		strncpy(name, g.types[m].c_str(), 7);
		ok = fwrite(name, 1, 8, f) == 8;
	}
	if (ok) ok = fwrite(g.values.data(), 4, g.values.size(), f) == g.values.size();
	ok = (fclose(f) == 0) && ok;
	return ok ? ADGPU_OK : fail(ADGPU_ERR_ARG, std::string("writing grid cache failed: ") + path);
}

adgpu_status grid_load(const char* path, Grid& g)
{
	FILE* f = fopen(path, "rb");
	if (!f) return fail(ADGPU_ERR_ARG, std::string("cannot open grid cache ") + path);
	g = Grid();
	char magic[8];
	int32_t version = 0, nm = 0;
	bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kGridMagic, 8) == 0 && fread(&version, 4, 1, f) == 1 &&
	          version == 1 && fread(g.dims, 4, 3, f) == 3 && fread(&g.spacing, 8, 1, f) == 1 &&
	          fread(g.origin, 8, 3, f) == 3 && fread(&nm, 4, 1, f) == 1 && nm >= 3 && nm <= ADGPU_MAX_ATYPES + 2;
	for (int k = 0; ok && k < 3; k++) ok = g.dims[k] >= 2 && g.dims[k] <= 256;
	for (int m = 0; ok && m < nm; m++) {
		char name[9] = {0};
		ok = fread(name, 1, 8, f) == 8;
		g.types.push_back(name);
	}
	if (ok) {
		g.values.resize((size_t)g.dims[0] * g.dims[1] * g.dims[2] * nm);
		ok = fread(g.values.data(), 4, g.values.size(), f) == g.values.size();
	}
	fclose(f);
	if (!ok) return fail(ADGPU_ERR_ARG, std::string("not a valid grid cache: ") + path);
	if (g.types[nm - 2] != "e" || g.types[nm - 1] != "d") return fail(ADGPU_ERR_ARG, "grid cache: maps must end with e, d");
	g.num_map_atypes = nm - 2;
	return ADGPU_OK;
}

void grid_reference_layout(const Grid& g, float* out)
{
	const int gx = g.dims[0], gy = g.dims[1], gz = g.dims[2];
	const size_t n = (size_t)gx * gy * gz;
	const size_t g1 = gx, g2 = (size_t)gx * gy;
	for (size_t m = 0; m < g.types.size(); m++) {
		const float* v = g.values.data() + m * n;
		float* base = out + m * n * 4;
		for (int z = 0; z < gz; z++)
			for (int y = 0; y < gy; y++)
				for (int x = 0; x < gx; x++) {
					size_t p = x + y * g1 + z * g2;
					float val = v[p];
					base[4 * p] = val;
					// duplicates so the 8 corners of a cell are 8 consecutive floats
					// (host/src/processgrid.cpp:244-248)
					if (y > 0) base[4 * (p - g1) + 1] = val;
					if (z > 0) base[4 * (p - g2) + 2] = val;
					if (y > 0 && z > 0) base[4 * (p - g2 - g1) + 3] = val;
				}
	}
}

void grid_cell_records(const Grid& g, float* out)
{
	const int gx = g.dims[0], gy = g.dims[1], gz = g.dims[2];
	const size_t n = (size_t)gx * gy * gz;
	const int nm = (int)g.types.size(), M = g.num_map_atypes;
	size_t rec = 0;
	for (int z = 0; z < gz - 1; z++)
		for (int y = 0; y < gy - 1; y++)
			for (int x = 0; x < gx - 1; x++, rec++) {
				float* r = out + rec * nm * 8;
				for (int s = 0; s < nm; s++) {
					int map = s == 0 ? M : (s == 1 ? M + 1 : s - 2);
					const float* v = g.values.data() + (size_t)map * n;
					auto at = [&](int dx, int dy, int dz) { return v[(x + dx) + (size_t)(y + dy) * gx + (size_t)(z + dz) * gx * gy]; };
					float* o = r + s * 8;
					o[0] = at(0, 0, 0); o[1] = at(0, 1, 0); o[2] = at(0, 0, 1); o[3] = at(0, 1, 1);
					o[4] = at(1, 0, 0); o[5] = at(1, 1, 0); o[6] = at(1, 0, 1); o[7] = at(1, 1, 1);
				}
			}
}

// ---------------------------------------------------------------------------
// ligand preparation
// ---------------------------------------------------------------------------

// AD4.1 parameters per atom type (AD4.1_bound.dat, as tabulated in
// host/src/processligand.cpp:775-880): Rii, epsii, Rij_hb, epsij_hb, vol, solpar.
struct TypeParams { const char* name; double reqm, eps, reqm_hb, eps_hb, vol, solpar; };
static const TypeParams kTypes[] = {
	{"H", 2.00, 0.020, 0.0, 0.0, 0.0000, 0.00051}, {"HD", 2.00, 0.020, 0.0, 1.0, 0.0000, 0.00051},
	{"HS", 2.00, 0.020, 0.0, 1.0, 0.0000, 0.00051}, {"C", 4.00, 0.150, 0.0, 0.0, 33.5103, -0.00143},
	{"A", 4.00, 0.150, 0.0, 0.0, 33.5103, -0.00052}, {"N", 3.50, 0.160, 0.0, 0.0, 22.4493, -0.00162},
	{"NA", 3.50, 0.160, 1.9, 5.0, 22.4493, -0.00162}, {"NS", 3.50, 0.160, 1.9, 5.0, 22.4493, -0.00162},
	{"OA", 3.20, 0.200, 1.9, 5.0, 17.1573, -0.00251}, {"OS", 3.20, 0.200, 1.9, 5.0, 17.1573, -0.00251},
	{"F", 3.09, 0.080, 0.0, 0.0, 15.4480, -0.00110}, {"MG", 1.30, 0.875, 0.0, 0.0, 1.5600, -0.00110},
	{"P", 4.20, 0.200, 0.0, 0.0, 38.7924, -0.00110}, {"SA", 4.00, 0.200, 2.5, 1.0, 33.5103, -0.00214},
	{"S", 4.00, 0.200, 0.0, 0.0, 33.5103, -0.00214}, {"CL", 4.09, 0.276, 0.0, 0.0, 35.8235, -0.00110},
	{"CA", 1.98, 0.550, 0.0, 0.0, 2.7700, -0.00110}, {"MN", 1.30, 0.875, 0.0, 0.0, 2.1400, -0.00110},
	{"FE", 1.30, 0.010, 0.0, 0.0, 1.8400, -0.00110}, {"ZN", 1.48, 0.550, 0.0, 0.0, 1.7000, -0.00110},
	{"BR", 4.33, 0.389, 0.0, 0.0, 42.5661, -0.00110}, {"I", 4.72, 0.550, 0.0, 0.0, 55.0585, -0.00110},
	{"SI", 4.10, 0.200, 0.0, 0.0, 35.8235, -0.00143}, {"B", 3.84, 0.155, 0.0, 0.0, 29.6478, -0.00152},
	{"CG", 4.00, 0.150, 0.0, 0.0, 33.5103, -0.00143}, {"G0", 0.00, 0.000, 0.0, 0.0, 0.0000, 0.00000},
	{"W", 0.00, 0.000, 0.0, 0.0, 0.0000, 0.00000}, {"CX", 4.00, 0.150, 0.0, 0.0, 33.5103, -0.00143},
	{"NX", 3.50, 0.160, 0.0, 0.0, 22.4493, -0.00162}, {"OX", 3.20, 0.200, 1.9, 5.0, 17.1573, -0.00251},
};
constexpr int kNumTypes = 30;
constexpr int kCG = 24, kG0 = 25;

static bool ci_prefix2_equal(const char* a, const char* b)
{
	// two-character, case-insensitive match in which a shorter string matches
	// only if the other one ends at the same place (the reference's strincmp(.., 2))
	int count = 1;
	char c1 = *a, c2 = *b;
	while (c1 && c2 && count < 2) {
		if (toupper(c1) != toupper(c2)) return false;
		a++; b++; c1 = *a; c2 = *b; count++;
	}
	return toupper(c1) == toupper(c2);
}

static int type_index(const std::string& t)
{
	for (int i = 0; i < kNumTypes; i++) {
		if (ci_prefix2_equal(kTypes[i].name, t.c_str())) return i;
		if (kTypes[i].name[1] == '0' && kTypes[i].name[0] == toupper(t[0])) return i;
	}
	return -1;
}

static bool is_acceptor(const std::string& t) { return t == "NA" || t == "NS" || t == "OA" || t == "OS" || t == "SA"; }
static bool is_hbond(const std::string& a, const std::string& b)
{
	return ((a == "HD" || a == "HS") && is_acceptor(b)) || ((b == "HD" || b == "HS") && is_acceptor(a));
}

// bond-length class of an atom type for bond perception (host/src/processligand.cpp:465-489)
static int bond_class(const std::string& t, int* nameid)
{
	static const char* names[22] = {"C", "A", "Hx", "Nx", "Ox", "F", "MG", "P", "Sx", "CL", "CA", "MN", "FE", "ZN", "BR", "I", "CG", "G0", "W", "CX", "SI", "B"};
	static const int cls[22] = {0, 0, 3, 1, 2, 4, 4, 5, 6, 4, 4, 4, 4, 4, 4, 4, 0, 0, 2, 0, 6, 0};
	int id = 22;
	for (int i = 0; i < 22; i++) {
		if (names[i][1] == 'x' || names[i][1] == '0') {
			if (names[i][0] == toupper(t[0])) id = i;
		} else if (ci_prefix2_equal(names[i], t.c_str())) id = i;
	}
	*nameid = id;
	return id < 22 ? cls[id] : -1;
}

struct Atom {
	double xyz[3];
	double q;
	int type;            // index into the ligand's type list
	int lig_id;          // ligand/residue number (0 ligand, 1.. flex residues)
	int rigid;           // rigid structure id
	bool ignore_inter;
};

static void trim_range(const std::string& s, size_t a, size_t b, std::string& out)
{
	out.clear();
	for (size_t i = a; i < b && i < s.size(); i++)
		if (!isspace((unsigned char)s[i])) out.push_back(s[i]);
}

static double field_double(const std::string& s, size_t a, size_t len)
{
	if (a >= s.size()) return 0.0;
	return atof(s.substr(a, len).c_str());
}

static bool is_atom_record(const std::string& line)
{
	char tmp[32];
	if (sscanf(line.c_str(), "%31s", tmp) != 1) return false;
	return !strcmp(tmp, "ATOM") || !strcmp(tmp, "HETATM");
}

adgpu_status prepare_ligand(const Grid& grid, const std::string& ligand_text, const std::string& flexres_text,
                            const adgpu_dockpars& run, const uint32_t seed[3], int num_runs, Prepared& out)
{
	out = Prepared();
	std::vector<std::string> lines[2];
	{
		std::istringstream a(ligand_text), b(flexres_text);
		std::string l;
		while (std::getline(a, l)) lines[0].push_back(l);
		while (std::getline(b, l)) lines[1].push_back(l);
	}
	const bool has_lig = !lines[0].empty(), has_flex = !lines[1].empty();
	if (!has_lig && !has_flex) return fail(ADGPU_ERR_ARG, "no ligand or flexible residue given");

	// atom types in order of first appearance (init_liganddata)
	std::vector<std::string> types;
	for (int f = 0; f < 2; f++)
		for (auto& line : lines[f]) {
			if (!is_atom_record(line)) continue;
			std::string t;
			trim_range(line, 77, 80, t);
			if (std::find(types.begin(), types.end(), t) == types.end()) {
				if ((int)types.size() >= ADGPU_MAX_ATYPES) return fail(ADGPU_ERR_LIMIT, "more than 32 atom types");
				types.push_back(t);
			}
		}
	const int NT = (int)types.size();
	std::vector<int> vw(NT), map_of_type(NT, -1);
	for (int t = 0; t < NT; t++) {
		vw[t] = type_index(types[t]);
		if (vw[t] < 0) return fail(ADGPU_ERR_ARG, "unknown atom type " + types[t]);
		for (int m = 0; m < grid.num_map_atypes; m++)
			if (grid.types[m] == types[t]) { map_of_type[t] = m; break; }
		if (map_of_type[t] < 0 && types[t][0] != 'G') return fail(ADGPU_ERR_ARG, "no grid map for atom type " + types[t]);
	}

	// atoms, torsion tree (parse_liganddata)
	std::vector<Atom> atoms;
	struct Branch { int a, b, state; };
	std::vector<Branch> branches;
	std::vector<std::array<int, 2>> rotbonds;                      // in ENDBRANCH order
	std::vector<std::vector<int>> atom_branches;                   // open branches per atom (branch order)
	int rigid_cur = 1, rigid_top = 1, ligand_count = 0, true_lig_atoms = 0, true_lig_rotbonds = 0;
	for (int f = 0; f < 2; f++) {
		int first_serial = 1;
		bool first_atom = true;
		int atom_rot_start = (int)atoms.size(), flex_root = (int)atoms.size();
		size_t branch_start = f == 0 ? 0 : branches.size();
		for (auto& line : lines[f]) {
			char tmp[32];
			if (sscanf(line.c_str(), "%31s", tmp) != 1) continue;
			std::string key(tmp);
			if (f > 0 && key == "ROOT") {
				ligand_count++;
				flex_root = (int)atoms.size();
				atom_rot_start = (int)atoms.size();
				branch_start = branches.size();
				first_atom = true;
			}
			if (key == "ATOM" || key == "HETATM") {
				if ((int)atoms.size() >= ADGPU_MAX_ATOMS) return fail(ADGPU_ERR_LIMIT, "more than 256 atoms");
				if (first_atom) { sscanf(line.c_str() + 6, "%d", &first_serial); first_atom = false; }
				Atom at;
				at.xyz[0] = field_double(line, 30, 8);
				at.xyz[1] = field_double(line, 38, 8);
				at.xyz[2] = field_double(line, 46, 8);
				at.q = line.size() > 70 ? strtod(line.c_str() + 70, nullptr) : 0.0;   // "%lf" from column 70
				std::string t;
				trim_range(line, 77, 80, t);
				at.type = (int)(std::find(types.begin(), types.end(), t) - types.begin());
				at.lig_id = ligand_count;
				at.rigid = rigid_cur;
				at.ignore_inter = (t[0] == 'G') || (f > 0 && (int)atoms.size() - flex_root < 2);
				std::vector<int> open;
				for (size_t i = branch_start; i < branches.size(); i++)
					if (branches[i].state == 1) open.push_back((int)i);
				atom_branches.push_back(open);
				atoms.push_back(at);
			}
			if (key == "BRANCH") {
				if (branches.size() >= ADGPU_MAX_ROTBONDS) return fail(ADGPU_ERR_LIMIT, "more than 57 rotatable bonds");
				int a = 0, b = 0;
				sscanf(line.c_str() + 6, "%d %d", &a, &b);
				branches.push_back({a + atom_rot_start - first_serial, b + atom_rot_start - first_serial, 1});
				rigid_top++;
				rigid_cur = rigid_top;
			}
			if (key == "ENDBRANCH") {
				int a = 0, b = 0;
				sscanf(line.c_str() + 9, "%d %d", &a, &b);
				a += atom_rot_start - first_serial;
				b += atom_rot_start - first_serial;
				rotbonds.push_back({a, b});
				for (size_t i = branch_start; i < branches.size(); i++)
					if (branches[i].a == a && branches[i].b == b) branches[i].state = 2;
				rigid_cur--;
			}
		}
		rigid_top++;
		rigid_cur = rigid_top;
		if (f == 0) { true_lig_atoms = (int)atoms.size(); true_lig_rotbonds = (int)branches.size(); }
	}
	const int N = (int)atoms.size(), NR = (int)branches.size();
	if (N == 0) return fail(ADGPU_ERR_ARG, "no atoms");
	if ((int)rotbonds.size() != NR) return fail(ADGPU_ERR_ARG, "BRANCH/ENDBRANCH records unbalanced");
	// atom_rotbonds in ENDBRANCH order
	std::vector<std::vector<char>> atom_rot(N, std::vector<char>(NR, 0));
	for (int i = 0; i < NR; i++)
		for (int j = 0; j < NR; j++)
			if (rotbonds[i][0] == branches[j].a && rotbonds[i][1] == branches[j].b)
				for (int k = 0; k < N; k++)
					if (std::find(atom_branches[k].begin(), atom_branches[k].end(), j) != atom_branches[k].end()) atom_rot[k][i] = 1;
	for (auto& rb : rotbonds)
		if (rb[0] < 0 || rb[0] >= N || rb[1] < 0 || rb[1] >= N) return fail(ADGPU_ERR_ARG, "BRANCH names an atom that does not exist");

	// bonds by distance (get_bonds with the AD4_BOND_DISTS table the reference
	// compiles in, host/src/processligand.cpp:27,529-567): Handbook of Chemistry
	// and Physics bond-length ranges widened by 0.1 A, 0.9-2.1 A otherwise
	double mind[7][7], maxd[7][7];
	const double tol = 0.1;
	for (int i = 0; i < 7; i++) for (int j = 0; j < 7; j++) { mind[i][j] = 0.9 - tol; maxd[i][j] = 2.1 + tol; }
	enum { Cc = 0, Nc = 1, Oc = 2, Hc = 3, Xc = 4, Pc = 5, Sc = 6 };
	auto setmm = [&](int a, int b, double lo, double hi) {
		mind[a][b] = lo - tol; maxd[a][b] = hi + tol;
		if (a != b) { mind[b][a] = mind[a][b]; maxd[b][a] = maxd[a][b]; }
	};
	setmm(Cc, Cc, 1.20, 1.545); setmm(Cc, Nc, 1.1, 1.479); setmm(Cc, Oc, 1.15, 1.47); setmm(Cc, Hc, 1.022, 1.12);
	setmm(Cc, Xc, 0.9, 1.545); setmm(Cc, Pc, 1.85, 1.89); setmm(Cc, Sc, 1.55, 1.835);
	setmm(Nc, Nc, 1.0974, 1.128); setmm(Nc, Oc, 1.0619, 1.25); setmm(Nc, Hc, 1.004, 1.041); setmm(Nc, Xc, 0.9, 1.041);
	setmm(Nc, Pc, 1.4910, 1.4910); setmm(Nc, Sc, 1.58, 1.672);
	setmm(Oc, Oc, 1.208, 1.51); setmm(Oc, Hc, 0.955, 1.0289); setmm(Oc, Xc, 0.955, 2.1); setmm(Oc, Pc, 1.36, 1.67);
	setmm(Oc, Sc, 1.41, 1.47);
	setmm(Hc, Hc, 100., -100.); setmm(Hc, Xc, 0.9, 1.5); setmm(Hc, Pc, 1.40, 1.44); setmm(Hc, Sc, 1.325, 1.3455);
	setmm(Xc, Xc, 0.9, 2.1); setmm(Xc, Pc, 0.9, 2.1); setmm(Xc, Sc, 1.325, 2.1);
	setmm(Pc, Pc, 2.18, 2.23); setmm(Pc, Sc, 1.83, 1.88); setmm(Sc, Sc, 2.03, 2.05);
	std::vector<std::vector<char>> bonds(N, std::vector<char>(N, 0));
	for (int a1 = 0; a1 < N - 1; a1++)
		for (int a2 = a1 + 1; a2 < N; a2++) {
			if (atoms[a1].lig_id != atoms[a2].lig_id) continue;
			const std::string &t1 = types[atoms[a1].type], &t2 = types[atoms[a2].type];
			int n1, n2;
			int c1 = bond_class(t1, &n1), c2 = bond_class(t2, &n2);
			if (c1 < 0 || c2 < 0) return fail(ADGPU_ERR_ARG, "ligand atom type unknown to bond perception");
			double dx = atoms[a1].xyz[0] - atoms[a2].xyz[0], dy = atoms[a1].xyz[1] - atoms[a2].xyz[1], dz = atoms[a1].xyz[2] - atoms[a2].xyz[2];
			double d = sqrt(dx * dx + dy * dy + dz * dz);
			if (n1 == 18 || n2 == 18) continue;   // W is never bonded
			if (d >= mind[c1][c2] && d <= maxd[c1][c2]) { bonds[a1][a2] = bonds[a2][a1] = 1; }
			else if (n1 == 16 && n2 == 16 && t1.substr(2) == t2.substr(2)) { bonds[a1][a2] = bonds[a2][a1] = 2; }
		}

	// intramolecular contributors (get_intraE_contributors, 5 cases)
	std::vector<std::vector<char>> contrib(N, std::vector<char>(N, 1));
	for (int i = 0; i < N; i++) contrib[i][i] = 0;
	for (int i = 0; i < N - 1; i++)
		for (int j = i + 1; j < N; j++)
			if (atoms[i].rigid == atoms[j].rigid) contrib[i][j] = contrib[j][i] = 0;
	std::vector<char> nb(N), nbt(N);
	for (int i = 0; i < N; i++) {
		for (int j = 0; j < N; j++) nb[j] = bonds[i][j] > 0;
		for (int pass = 0; pass < 2; pass++) {
			nbt = nb;
			for (int j = 0; j < N; j++)
				if (nb[j]) for (int k = 0; k < N; k++) if (bonds[j][k] > 0) nbt[k] = 1;
			nb = nbt;
		}
		for (int j = 0; j < N; j++) if (nb[j]) contrib[i][j] = contrib[j][i] = 0;
		const std::string& ti = types[atoms[i].type];
		for (int j = 0; j < N; j++) {
			const std::string& tj = types[atoms[j].type];
			if (ti[0] == 'G' || tj[0] == 'G') contrib[i][j] = contrib[j][i] = 0;
			bool cg_g = ti.compare(0, 2, "CG") == 0 && tj[0] == 'G';
			bool g_cg = ti[0] == 'G' && tj.compare(0, 2, "CG") == 0;
			if (bonds[i][j] == 0 && (cg_g || g_cg)) {
				bool match = cg_g ? ti.substr(2) == tj.substr(1) : ti.substr(1) == tj.substr(2);
				contrib[i][j] = contrib[j][i] = match ? 1 : 0;
			}
		}
	}
	for (int r = 0; r < NR; r++) {
		int a = rotbonds[r][0], b = rotbonds[r][1];
		int A = atoms[a].rigid, B = atoms[b].rigid;
		for (int i = 0; i < N; i++) {
			if (atoms[i].rigid == A) contrib[i][b] = contrib[b][i] = 0;
			if (atoms[i].rigid == B) contrib[i][a] = contrib[a][i] = 0;
		}
	}
	for (int r1 = 0; r1 < NR - 1; r1++)
		for (int r2 = r1 + 1; r2 < NR; r2++) {
			int a = rotbonds[r1][0], b = rotbonds[r1][1], a2 = rotbonds[r2][0], b2 = rotbonds[r2][1];
			auto R = [&](int x) { return atoms[x].rigid; };
			if (R(a) == R(a2)) contrib[b][b2] = contrib[b2][b] = 0;
			if (R(a) == R(b2)) contrib[b][a2] = contrib[a2][b] = 0;
			if (R(b) == R(a2)) contrib[a][b2] = contrib[b2][a] = 0;
			if (R(b) == R(b2)) contrib[a][a2] = contrib[a2][a] = 0;
		}
	for (int i = 0; i < N - 1; i++)
		for (int j = i + 1; j < N; j++)
			if (types[atoms[i].type] == "W" || types[atoms[j].type] == "W") contrib[i][j] = contrib[j][i] = 0;

	// vdW / H-bond / desolvation parameters (get_VWpars with the unbound model 0 coefficients)
	const double coeff_vdw = 0.1662, coeff_hb = 0.1209;
	adgpu_kc_intra& kin = out.intra;
	memset(&kin, 0, sizeof(kin));
	PostLigand& pl = out.post;
	pl.ntypes = NT;
	pl.reqm_AB.assign(NT * NT, 0.0); pl.vw_A.assign(NT * NT, 0.0); pl.vw_B.assign(NT * NT, 0.0);
	pl.vw_C.assign(NT * NT, 0.0); pl.vw_D.assign(NT * NT, 0.0); pl.is_hb.assign(NT * NT, 0);
	pl.vw_index.resize(NT); pl.solpar.resize(NT); pl.volume.resize(NT);
	for (int t1 = 0; t1 < NT; t1++) {
		kin.atom_types_reqm_const[t1] = (unsigned)vw[t1];
		kin.dspars_S_const[t1] = (float)kTypes[vw[t1]].solpar;
		kin.dspars_V_const[t1] = (float)kTypes[vw[t1]].vol;
		pl.vw_index[t1] = vw[t1];
		pl.solpar[t1] = kTypes[vw[t1]].solpar;
		pl.volume[t1] = kTypes[vw[t1]].vol;
		for (int t2 = 0; t2 < NT; t2++) {
			const TypeParams &p1 = kTypes[vw[t1]], &p2 = kTypes[vw[t2]];
			int idx = t1 * NT + t2;
			double A = 0, B = 0;
			if (is_hbond(types[t1], types[t2])) {
				double eps12 = coeff_hb * p1.eps_hb * p2.eps_hb;
				double reqm12 = p1.reqm_hb + p2.reqm_hb;
				kin.VWpars_exp_const[idx] = (12 << 8) + 10;
				kin.reqm_AB_const[idx] = (float)reqm12;
				A = 5 * eps12 * pow(reqm12, 12);
				B = 6 * eps12 * pow(reqm12, 10);
				pl.reqm_AB[idx] = reqm12; pl.vw_C[idx] = A; pl.vw_D[idx] = B; pl.is_hb[idx] = 1;
			} else {
				double eps12 = coeff_vdw * sqrt(p1.eps * p2.eps);
				double reqm12 = 0.5 * (p1.reqm + p2.reqm);
				kin.VWpars_exp_const[idx] = (12 << 8) + 6;
				kin.reqm_AB_const[idx] = (float)reqm12;
				bool cgcg = vw[t1] == kCG && vw[t2] == kCG && types[t1].substr(2) == types[t2].substr(2);
				if (!cgcg) { A = eps12 * pow(reqm12, 12); B = 2 * eps12 * pow(reqm12, 6); }
				pl.reqm_AB[idx] = reqm12; pl.vw_A[idx] = A; pl.vw_B[idx] = B;
			}
			kin.VWpars_AC_const[idx] = (float)A;
			kin.VWpars_BD_const[idx] = (float)B;
		}
	}
	(void)kG0;

	pl.natoms = N; pl.true_lig_atoms = true_lig_atoms; pl.nrot = NR; pl.true_lig_rotbonds = true_lig_rotbonds;
	pl.spacing = grid.spacing;
	for (int k = 0; k < 3; k++) pl.origin[k] = grid.origin[k];
	pl.input_xyz.resize(3 * N); pl.charge.resize(N); pl.type.resize(N); pl.map.resize(N);
	pl.ignore_inter.resize(N); pl.rot_mask.assign(N, 0);
	for (int i = 0; i < N; i++) {
		for (int k = 0; k < 3; k++) pl.input_xyz[3 * i + k] = atoms[i].xyz[k];
		pl.charge[i] = atoms[i].q;
		pl.type[i] = atoms[i].type;
		pl.map[i] = map_of_type[atoms[i].type];
		pl.ignore_inter[i] = atoms[i].ignore_inter ? 1 : 0;
		for (int r = 0; r < NR; r++) if (atom_rot[i][r]) pl.rot_mask[i] |= 1ull << r;
	}

	// reference orientation: ligand centred on the origin, flex residues in grid
	// coordinates, all scaled to grid units (gen_initpop_and_reflig tail)
	double mv[3] = {0, 0, 0};
	if (true_lig_atoms > 0) {
		for (int i = 0; i < true_lig_atoms; i++) for (int k = 0; k < 3; k++) mv[k] += atoms[i].xyz[k];
		for (int k = 0; k < 3; k++) mv[k] = -1 * mv[k] / true_lig_atoms;
	}
	for (int i = 0; i < N; i++)
		for (int k = 0; k < 3; k++) {
			if (i < true_lig_atoms) atoms[i].xyz[k] += mv[k];
			else atoms[i].xyz[k] += -grid.origin[k];
			atoms[i].xyz[k] *= 1.0 / grid.spacing;
		}

	// tables (prepare_const_fields_for_gpu)
	adgpu_kc_interintra& ii = out.interintra;
	memset(&ii, 0, sizeof(ii));
	for (int m = 0; m < ADGPU_MAX_ATOMS; m++) ii.ignore_inter_const[m] = 1;
	for (int i = 0; i < N; i++) {
		ii.atom_charges_const[i] = (float)atoms[i].q;
		ii.atom_types_const[i] = (uint32_t)atoms[i].type;
		ii.atom_types_map_const[i] = (uint32_t)map_of_type[atoms[i].type];
		ii.ignore_inter_const[i] = atoms[i].ignore_inter ? 1 : 0;
	}
	out.pairs.clear();
	for (int i = 0; i < N - 1; i++)
		for (int j = i + 1; j < N; j++)
			if (contrib[i][j] == 1) { out.pairs.push_back((uint32_t)i); out.pairs.push_back((uint32_t)j); }
	if (out.pairs.size() / 2 > (size_t)ADGPU_MAX_INTRAE) return fail(ADGPU_ERR_LIMIT, "too many intramolecular pairs");
	adgpu_kc_conform& cf = out.conform;
	memset(&cf, 0, sizeof(cf));
	for (int i = 0; i < N; i++) for (int k = 0; k < 3; k++) cf.ref_coords_const[3 * i + k] = (float)atoms[i].xyz[k];
	pl.ref_xyz.resize(3 * N);
	for (int i = 0; i < N; i++) for (int k = 0; k < 3; k++) pl.ref_xyz[3 * i + k] = atoms[i].xyz[k];
	pl.rot_move.assign(3 * NR, 0.0); pl.rot_unit.assign(3 * NR, 0.0);
	for (int r = 0; r < NR; r++) {
		const double* A = atoms[rotbonds[r][0]].xyz;
		const double* B = atoms[rotbonds[r][1]].xyz;
		double u[3], d = 0;
		for (int k = 0; k < 3; k++) { u[k] = B[k] - A[k]; }
		d = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
		if (d == 0.0) return fail(ADGPU_ERR_ARG, "rotatable bond of zero length");
		for (int k = 0; k < 3; k++) { u[k] /= d; if (u[k] >= 1) u[k] = 0.999999; }
		// moving vector: from the origin to its projection on the bond axis (vec_point2line)
		double L2 = pow(B[0] - A[0], 2) + pow(B[1] - A[1], 2) + pow(B[2] - A[2], 2);
		double tt = 0;
		for (int k = 0; k < 3; k++) tt += (B[k] - A[k]) * (0.0 - A[k]);
		tt = tt / L2;
		for (int k = 0; k < 3; k++) {
			double proj = tt * (B[k] - A[k]) + A[k];
			cf.rotbonds_moving_vectors_const[3 * r + k] = (float)(proj - 0.0);
			cf.rotbonds_unit_vectors_const[3 * r + k] = (float)u[k];
			pl.rot_move[3 * r + k] = proj - 0.0;
			pl.rot_unit[3 * r + k] = u[k];
		}
	}
	adgpu_kc_grads& gr = out.grads;
	memset(&gr, 0, sizeof(gr));
	for (int r = 0; r < NR; r++) {
		gr.rotbonds[2 * r] = rotbonds[r][0];
		gr.rotbonds[2 * r + 1] = rotbonds[r][1];
		int c = 0;
		for (int j = 0; j < N; j++)
			if (atom_rot[j][r]) gr.rotbonds_atoms[ADGPU_MAX_ATOMS * r + c++] = j;
		gr.num_rotating_atoms_per_rotbond[r] = c;
	}
	// rotation list for a 64-thread block (gen_rotlist): rows of 64 independent
	// rotations; each atom's torsions in increasing id, then the general rotation
	{
		const int TH = 64;
		std::vector<int> nreq(std::max(N, TH), 0), order(N);
		std::vector<bool> first(N, true);
		for (int a = 0; a < N; a++) {
			order[a] = a;
			nreq[a] = 1;
			for (int r = 0; r < NR; r++) if (atom_rot[a][r]) nreq[a]++;
		}
		auto reorder = [&]() {
			for (int j = 0; j < N - 1; j++)
				for (int i = N - 2; i >= j; i--)
					if (nreq[i + 1] > nreq[i]) { std::swap(nreq[i], nreq[i + 1]); std::swap(order[i], order[i + 1]); }
		};
		out.rotlist.clear();
		reorder();
		int cycles = 0;
		while (nreq[0] != 0) {
			if ((int)out.rotlist.size() >= ADGPU_MAX_ROTATIONS) return fail(ADGPU_ERR_LIMIT, "too many rotations");
			for (int p = 0; p < TH; p++) {
				int el;
				if (nreq[p] == 0) el = ADGPU_RLIST_DUMMY_MASK;
				else {
					int a = order[p];
					el = a & ADGPU_RLIST_ATOMID_MASK;
					if (nreq[p] == 1) el |= ADGPU_RLIST_GENROT_MASK;
					else {
						int remaining = nreq[p] - 1, cand = NR - 1;
						for (;;) {
							if (cand < 0) return fail(ADGPU_ERR_ARG, "rotation list construction failed");
							if (atom_rot[a][cand]) { if (remaining == 1) break; remaining--; }
							cand--;
						}
						el |= (cand << ADGPU_RLIST_RBONDID_SHIFT) & ADGPU_RLIST_RBONDID_MASK;
					}
					if (first[a]) el |= ADGPU_RLIST_FIRSTROT_MASK;
					first[a] = false;
					nreq[p]--;
				}
				out.rotlist.push_back(el);
			}
			reorder();
			cycles++;
		}
		out.num_rotcyc = cycles;
	}

	// docking parameters: run settings from `run`, ligand/grid fields filled here
	adgpu_dockpars& dp = out.dockpars;
	dp = run;
	dp.num_of_atoms = N;
	dp.true_ligand_atoms = true_lig_atoms;
	dp.num_of_atypes = NT;
	dp.num_of_map_atypes = grid.num_map_atypes;
	dp.num_of_intraE_contributors = (int)(out.pairs.size() / 2);
	dp.gridsize_x = grid.dims[0]; dp.gridsize_y = grid.dims[1]; dp.gridsize_z = grid.dims[2];
	dp.gridsize_x_times_y = grid.dims[0] * grid.dims[1];
	dp.gridsize_x_times_y_times_z = grid.dims[0] * grid.dims[1] * grid.dims[2];
	dp.grid_spacing = (float)grid.spacing;
	dp.rotbondlist_length = 64 * out.num_rotcyc;
	dp.num_of_genes = NR + 6;
	out.num_rotbonds = NR;

	// initial population and per-thread LCG seeds (gen_initpop_and_reflig;
	// host/src/performdocking.cpp.Cuda:306-317)
	if (num_runs > 0) {
		const int P = run.pop_size;
		out.initpop.assign((size_t)num_runs * P * ADGPU_GENOTYPE_STRIDE, 0.0f);
		Cmwc4096 r(seed);
		const double box[3] = {(grid.dims[0] - 1) * grid.spacing, (grid.dims[1] - 1) * grid.spacing, (grid.dims[2] - 1) * grid.spacing};
		const float PI_F = (float)M_PI;
		for (size_t e = 0; e < (size_t)num_runs * P; e++) {
			float* g = out.initpop.data() + e * ADGPU_GENOTYPE_STRIDE;
			for (int k = 0; k < 3; k++) g[k] = (float)(r.next_float() * box[k] / grid.spacing);
			// float/double mix as in the reference (float arguments go to the float overloads)
			float u1 = r.next_float(), u2 = r.next_float(), u3 = r.next_float();
			const float twopi = 2.0f * PI_F;
			float qw = (float)(sqrt(1.0 - u1) * sinf(twopi * u2));
			float qx = (float)(sqrt(1.0 - u1) * cosf(twopi * u2));
			float qy = (float)(sqrtf(u1) * sinf(twopi * u3));
			float qz = (float)(sqrtf(u1) * cosf(twopi * u3));
			float rot = (float)(2.0 * acosf(qw));
			float s = (float)sqrt(1.0 - (qw * qw));
			float x, y, z;
			if (s < 0.001) { x = qx; y = qy; z = qz; }
			else { x = qx / s; y = qy / s; z = qz / s; }
			float theta = acosf(z), phi = atan2f(y, x);
			g[3] = phi / 0.0174533f;
			g[4] = theta / 0.0174533f;
			g[5] = rot / 0.0174533f;
			for (int k = 6; k < ADGPU_MAX_ROTBONDS + 6; k++) g[k] = r.next_float() * 360;
		}
		Cmwc4096 r2(seed);
		out.prng.resize((size_t)num_runs * P * 64);
		for (auto& v : out.prng) v = r2.next();
	}
	return ADGPU_OK;
}

void dockpars_defaults(adgpu_dockpars& dp, double spacing, int pop_size)
{
	// command-line defaults (host/inc/getparameters.h:66-145, host/src/getparameters.cpp:1399-1400)
	// scaled as docking_with_gpu does (host/src/performdocking.cpp.Cuda:413-463)
	memset(&dp, 0, sizeof(dp));
	dp.coeff_elec = (float)(332.06363f * 0.1406);
	dp.elec_min_distance = 0.01f;
	dp.coeff_desolv = (float)0.1322;
	dp.pop_size = pop_size;
	dp.tournament_rate = 60 / 100.0f;
	dp.crossover_rate = 80 / 100.0f;
	dp.mutation_rate = 2 / 100.f;
	dp.abs_max_dang = 90;
	dp.abs_max_dmov = (float)(6.0 / spacing);
	dp.qasp = 0.01097f;
	dp.smooth = 0.5f;
	dp.lsearch_rate = 100;
	dp.adam_beta1 = 0.9f;
	dp.adam_beta2 = 0.999f;
	dp.adam_epsilon = 1.0e-8f;
	dp.num_of_lsentities = (unsigned int)(100 / 100.0 * pop_size + 0.5);
	dp.rho_lower_bound = 0.01f;
	dp.base_dmov_mul_sqrt3 = (float)(2.0 / spacing * sqrt(3.0));
	dp.base_dang_mul_sqrt3 = (float)(75.0 * sqrt(3.0));
	dp.cons_limit = 4;
	dp.max_num_of_iters = 300;
}

}  // namespace adgpu
