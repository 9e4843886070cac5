/* TEST INFRASTRUCTURE ONLY -- the loader of the Star Schema Benchmark tables
 * that dbgen (data/ssb/dbgen, built from its sources by the Makefile here)
 * writes, into the integer columns the reference's queries read.
 *
 *     ssb_load <tbl_dir> <out_dir>
 *
 * reads <tbl_dir>/{lineorder,supplier,customer,part,date}.tbl ('|'-separated
 * text, one row per line) and writes each column the SSB queries use as raw
 * little-endian int32 to <out_dir>/<column>.i32.  The integer encoding is the
 * reference's (data/ssb/loader/convert.py, then load_modified.c):
 *   - numeric fields are parsed as decimal integers (load_modified.c strtol);
 *   - nation and region names become their index in convert.py's lists
 *     (convert.py:1-40; note the list is not alphabetical);
 *   - a city becomes nation * 10 + the city's last digit (convert.py:55,71);
 *   - MFGR#m -> m - 1; category MFGR#mc -> mfgr * 5 + (mc % 10 - 1); brand
 *     MFGR#mcbb -> category * 40 + (bb - 1) (convert.py:82-88).
 * The parse runs in parallel over newline-aligned slices of each file. */
#define _GNU_SOURCE
#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

static const char* const kNations[25] = {
    "ALGERIA", "ARGENTINA", "BRAZIL",  "CANADA",       "EGYPT",   "ETHIOPIA", "FRANCE",         "GERMANY",
    "INDIA",   "INDONESIA", "IRAN",    "IRAQ",         "JAPAN",   "JORDAN",   "KENYA",          "MOROCCO",
    "MOZAMBIQUE", "PERU",   "CHINA",   "ROMANIA",      "SAUDI ARABIA", "VIETNAM", "RUSSIA",     "UNITED KINGDOM",
    "UNITED STATES"};
static const char* const kRegions[5] = {"AFRICA", "AMERICA", "ASIA", "EUROPE", "MIDDLE EAST"};

typedef struct {
	const char* p;
	size_t      n;
} Field;

static void die(const char* what, const char* arg) {
	fprintf(stderr, "ssb_load: %s %s\n", what, arg ? arg : "");
	exit(1);
}

static int32_t to_int(Field f) {
	int64_t v = 0;
	int     neg = 0;
	size_t  i   = 0;
	if (i < f.n && f.p[i] == '-') {
		neg = 1;
		++i;
	}
	for (; i < f.n && f.p[i] >= '0' && f.p[i] <= '9'; ++i) { v = v * 10 + (f.p[i] - '0'); }
	return (int32_t)(neg ? -v : v);
}

static int index_of(Field f, const char* const* names, int n) {
	while (f.n && f.p[f.n - 1] == ' ') { --f.n; }
	for (int i = 0; i < n; ++i) {
		if (strlen(names[i]) == f.n && memcmp(names[i], f.p, f.n) == 0) { return i; }
	}
	die("unknown name in", "nation/region field");
	return -1;
}

/* The integer after the last '#' of a field (MFGR#1221 -> 1221, as a string). */
static Field after_hash(Field f) {
	size_t i = f.n;
	while (i > 0 && f.p[i - 1] != '#') { --i; }
	Field r = {f.p + i, f.n - i};
	return r;
}

/* Splits one line into up to max fields; returns the count. */
static int split(const char* line, const char* end, Field* out, int max) {
	int         k = 0;
	const char* s = line;
	for (const char* p = line; p < end && k < max; ++p) {
		if (*p == '|') {
			out[k].p = s;
			out[k].n = (size_t)(p - s);
			++k;
			s = p + 1;
		}
	}
	return k;
}

typedef struct {
	const char* data;
	size_t      size;
} Map;

static Map map_file(const char* path) {
	int fd = open(path, O_RDONLY);
	if (fd < 0) { die("cannot open", path); }
	struct stat st;
	if (fstat(fd, &st) != 0) { die("cannot stat", path); }
	Map m = {NULL, (size_t)st.st_size};
	if (m.size) {
		m.data = mmap(NULL, m.size, PROT_READ, MAP_PRIVATE, fd, 0);
		if (m.data == MAP_FAILED) { die("cannot map", path); }
		madvise((void*)m.data, m.size, MADV_SEQUENTIAL);
	}
	close(fd);
	return m;
}

enum { kMaxCols = 9, kMaxSlices = 256 };

/* One table: per line, fill one value per output column. */
typedef void (*RowFn)(const Field* f, int nf, int32_t* vals);

static void load_table(const char* tbl_dir, const char* file, const char* out_dir, const char* const* names, int n_cols,
                       int n_fields, RowFn fn) {
	char path[4096];
	snprintf(path, sizeof(path), "%s/%s", tbl_dir, file);
	Map m = map_file(path);
	int nt = (int)sysconf(_SC_NPROCESSORS_ONLN);
	if (nt < 1) { nt = 1; }
	if (nt > kMaxSlices) { nt = kMaxSlices; }
	if (m.size < (size_t)nt * 4096u) { nt = 1; }
	/* newline-aligned slices */
	size_t start[kMaxSlices + 1];
	start[0] = 0;
	for (int t = 1; t < nt; ++t) {
		size_t s = m.size / (size_t)nt * (size_t)t;
		while (s < m.size && m.data[s - 1] != '\n') { ++s; }
		start[t] = s;
	}
	start[nt] = m.size;
	size_t rows[kMaxSlices + 1];
#pragma omp parallel for num_threads(nt)
	for (int t = 0; t < nt; ++t) {
		size_t r = 0;
		for (size_t i = start[t]; i < start[t + 1]; ++i) { r += m.data[i] == '\n'; }
		rows[t] = r;
	}
	size_t off[kMaxSlices + 1];
	off[0] = 0;
	for (int t = 0; t < nt; ++t) { off[t + 1] = off[t] + rows[t]; }
	const size_t total = off[nt];
	int32_t*     cols[kMaxCols];
	for (int c = 0; c < n_cols; ++c) {
		cols[c] = malloc(total * sizeof(int32_t) + 4);
		if (!cols[c]) { die("out of memory for", file); }
	}
	int bad = 0;
#pragma omp parallel for num_threads(nt) reduction(| : bad)
	for (int t = 0; t < nt; ++t) {
		size_t      r = off[t];
		const char* p = m.data + start[t];
		const char* e = m.data + start[t + 1];
		Field       f[24];
		int32_t     vals[kMaxCols];
		while (p < e) {
			const char* nl = memchr(p, '\n', (size_t)(e - p));
			if (!nl) { nl = e; }
			const int nf = split(p, nl, f, 24);
			if (nf < n_fields) {
				bad = 1;
			} else {
				fn(f, nf, vals);
				for (int c = 0; c < n_cols; ++c) { cols[c][r] = vals[c]; }
			}
			++r;
			p = nl + 1;
		}
	}
	if (bad) { die("short line in", file); }
	for (int c = 0; c < n_cols; ++c) {
		snprintf(path, sizeof(path), "%s/%s.i32", out_dir, names[c]);
		FILE* o = fopen(path, "wb");
		if (!o || fwrite(cols[c], sizeof(int32_t), total, o) != total || fclose(o) != 0) { die("cannot write", path); }
		free(cols[c]);
	}
	if (m.size) { munmap((void*)m.data, m.size); }
	printf("%s %zu rows\n", file, total);
}

/* lineorder: orderkey 0, linenumber 1, custkey 2, partkey 3, suppkey 4,
 * orderdate 5, orderpriority 6, shippriority 7, quantity 8, extendedprice 9,
 * ordtotalprice 10, discount 11, revenue 12, supplycost 13, tax 14,
 * commitdate 15, shipmode 16 (load_modified.c lineorder()). */
static const char* const kLo[9] = {"lo_custkey",  "lo_partkey",  "lo_suppkey", "lo_orderdate", "lo_quantity",
                                   "lo_extendedprice", "lo_discount", "lo_revenue", "lo_supplycost"};
static void lo_row(const Field* f, int nf, int32_t* v) {
	(void)nf;
	static const int idx[9] = {2, 3, 4, 5, 8, 9, 11, 12, 13};
	for (int i = 0; i < 9; ++i) { v[i] = to_int(f[idx[i]]); }
}

/* supplier / customer: key 0, name 1, address 2, city 3, nation 4, region 5 */
static const char* const kSupp[4] = {"s_suppkey", "s_city", "s_nation", "s_region"};
static const char* const kCust[4] = {"c_custkey", "c_city", "c_nation", "c_region"};
static void geo_row(const Field* f, int nf, int32_t* v) {
	(void)nf;
	v[0]                = to_int(f[0]);
	const int nation    = index_of(f[4], kNations, 25);
	const Field city    = f[3];
	const char  digit   = city.n ? city.p[city.n - 1] : '0';
	v[1]                = nation * 10 + (digit - '0');
	v[2]                = nation;
	v[3]                = index_of(f[5], kRegions, 5);
}

/* part: partkey 0, name 1, mfgr 2, category 3, brand1 4, ... */
static const char* const kPart[4] = {"p_partkey", "p_mfgr", "p_category", "p_brand1"};
static void part_row(const Field* f, int nf, int32_t* v) {
	(void)nf;
	v[0]             = to_int(f[0]);
	const int mfgr   = to_int(after_hash(f[2])) - 1;
	const int cat    = mfgr * 5 + (to_int(after_hash(f[3])) % 10 - 1);
	Field     brand  = after_hash(f[4]);
	Field     tail   = {brand.p + 2, brand.n >= 2 ? brand.n - 2 : 0};
	v[1]             = mfgr;
	v[2]             = cat;
	v[3]             = cat * 40 + (to_int(tail) - 1);
}

/* date: datekey 0, date 1, dayofweek 2, month 3, year 4, yearmonthnum 5,
 * yearmonth 6, daynuminweek 7, daynuminmonth 8, daynuminyear 9,
 * monthnuminyear 10, weeknuminyear 11, ... */
static const char* const kDate[4] = {"d_datekey", "d_year", "d_yearmonthnum", "d_weeknuminyear"};
static void date_row(const Field* f, int nf, int32_t* v) {
	(void)nf;
	v[0] = to_int(f[0]);
	v[1] = to_int(f[4]);
	v[2] = to_int(f[5]);
	v[3] = to_int(f[11]);
}

int main(int argc, char** argv) {
	if (argc != 3) {
		fprintf(stderr, "usage: ssb_load <tbl_dir> <out_dir>\n");
		return 2;
	}
	load_table(argv[1], "lineorder.tbl", argv[2], kLo, 9, 17, lo_row);
	load_table(argv[1], "supplier.tbl", argv[2], kSupp, 4, 7, geo_row);
	load_table(argv[1], "customer.tbl", argv[2], kCust, 4, 8, geo_row);
	load_table(argv[1], "part.tbl", argv[2], kPart, 4, 9, part_row);
	load_table(argv[1], "date.tbl", argv[2], kDate, 4, 17, date_row);
	return 0;
}
