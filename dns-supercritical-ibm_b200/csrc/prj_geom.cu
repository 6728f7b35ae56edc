// prj_geom.cu -- readers of a reference case's geometry folder (host only).
//
// The reference's pre-processor (src/pycode/calc_bands.py) writes the wall-normal
// tables of a case as text files in ./geom_data: the first line holds the row
// count, then one row per line of space-separated values (calc_bands.py:358-364).
// The solver reads one column of such a file with read_column_r8
// (src/mod_utils.f90:14-35): the rows n_prev .. n_prev+n-1 of column icol, and it
// stops when that range runs past the row count.  The general parameters come
// from geom_data/base_params.txt, one list-directed record per line
// (src/inc_set_read_params.f90:14-45); text after the values of a record is
// ignored, as list-directed input ignores the rest of a record.
//
// Values are parsed with strtod, which rounds correctly: a file written with
// Python's str of each float (the shortest string that reads back to the same
// double) reads back to the bands calc_bands.py computed, bit for bit.
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/projection.h"
#include "prj_internal.h"

namespace {

int gfail(int code, const char* fmt, ...) {
    char buf[768];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return prj::record_error(code, buf);
}

// all lines of a text file
bool read_lines(const char* path, std::vector<std::string>* out) {
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    std::string cur;
    char buf[4096];
    while (std::fgets(buf, sizeof(buf), f)) {
        cur += buf;
        if (!cur.empty() && cur.back() == '\n') {
            cur.pop_back();
            if (!cur.empty() && cur.back() == '\r') cur.pop_back();
            out->push_back(cur);
            cur.clear();
        }
    }
    if (!cur.empty()) out->push_back(cur);
    std::fclose(f);
    return true;
}

// the first `want` numbers of a record; false if it holds fewer
bool parse_record(const std::string& line, int want, double* vals) {
    const char* p = line.c_str();
    for (int i = 0; i < want; i++) {
        while (*p == ' ' || *p == '\t' || *p == ',') p++;
        if (!*p) return false;
        char* end = nullptr;
        errno = 0;
        const double v = std::strtod(p, &end);
        if (end == p || errno == ERANGE) return false;
        vals[i] = v;
        p = end;
    }
    return true;
}

bool parse_ints(const std::string& line, int want, long long* vals) {
    const char* p = line.c_str();
    for (int i = 0; i < want; i++) {
        while (*p == ' ' || *p == '\t' || *p == ',') p++;
        if (!*p) return false;
        char* end = nullptr;
        errno = 0;
        const long long v = std::strtoll(p, &end, 10);
        if (end == p || errno == ERANGE) return false;
        vals[i] = v;
        p = end;
    }
    return true;
}

std::string join(const char* dir, const char* name) {
    std::string s(dir ? dir : ".");
    if (!s.empty() && s.back() != '/') s += '/';
    return s + name;
}

}  // namespace

extern "C" {

int prj_geom_read_column(const char* path, int icol, int n, int n_prev, double* out) {
    if (!path || !out) return gfail(PRJ_ERR_ARG, "NULL path or output");
    if (icol < 0 || icol > 3) return gfail(PRJ_ERR_ARG, "Unrecognized icol value %d (0..3)", icol);
    if (n < 0 || n_prev < 0) return gfail(PRJ_ERR_ARG, "n = %d, n_prev = %d must be >= 0", n, n_prev);
    std::vector<std::string> lines;
    if (!read_lines(path, &lines)) return gfail(PRJ_ERR_ARG, "cannot open %s", path);
    long long nb = 0;
    if (lines.empty() || !parse_ints(lines[0], 1, &nb) || nb < 0)
        return gfail(PRJ_ERR_ARG, "%s: the first line must hold the row count", path);
    if ((long long)n_prev + n - 1 >= nb)
        return gfail(PRJ_ERR_ARG, "%s: mismatch in (n_prev, n, nb) = (%d, %d, %lld)", path, n_prev, n, nb);
    if ((long long)lines.size() < nb + 1)
        return gfail(PRJ_ERR_ARG, "%s: %lld rows announced, %zu present", path, nb, lines.size() - 1);
    double vals[4];
    for (int k = 0; k < n; k++) {
        const std::string& row = lines[(size_t)n_prev + k + 1];
        if (!parse_record(row, icol + 1, vals))
            return gfail(PRJ_ERR_ARG, "%s: row %d has fewer than %d values", path, n_prev + k, icol + 1);
        out[k] = vals[icol];
    }
    return PRJ_OK;
}

int prj_geom_read_bands(const char* geom_dir, int ny, double* a, double* b, double* c, double* a00, double* b00,
                        double* c00) {
    if (ny < 1) return gfail(PRJ_ERR_ARG, "ny = %d must be >= 1", ny);
    const std::string f = join(geom_dir, "P_band_abc.dat"), f00 = join(geom_dir, "P_band_abc_00.dat");
    double* dst[6] = {a, b, c, a00, b00, c00};
    for (int i = 0; i < 6; i++) {
        const int rc = prj_geom_read_column((i < 3 ? f : f00).c_str(), i % 3, ny, 0, dst[i]);
        if (rc) return rc;
    }
    return PRJ_OK;
}

int prj_geom_read_metrics(const char* geom_dir, int ny, double* inv_dy_p, double* dPdy_lo, double* dPdy_hi) {
    if (ny < 1) return gfail(PRJ_ERR_ARG, "ny = %d must be >= 1", ny);
    int rc = prj_geom_read_column(join(geom_dir, "inv_dy_p.dat").c_str(), 0, ny, 0, inv_dy_p);
    if (rc) return rc;
    const std::string f = join(geom_dir, "dPdy_ddy_lh.dat");
    if ((rc = prj_geom_read_column(f.c_str(), 0, ny, 0, dPdy_lo))) return rc;
    return prj_geom_read_column(f.c_str(), 1, ny, 0, dPdy_hi);
}

int prj_geom_read_base_params(const char* path, prj_case_params* out) {
    if (!path || !out) return gfail(PRJ_ERR_ARG, "NULL path or output");
    std::vector<std::string> L;
    if (!read_lines(path, &L)) return gfail(PRJ_ERR_ARG, "cannot open %s", path);
    if (L.size() < 14) return gfail(PRJ_ERR_ARG, "%s: %zu records, at least 14 expected", path, L.size());
    long long g[3], rough[2], nst[1], inc[1];
    double ns_dt[2], dxz[2], wb[4], wt[4];
    if (!parse_ints(L[0], 3, g) || !parse_ints(L[1], 2, rough) || !parse_ints(L[2], 1, nst) ||
        !parse_record(L[2], 2, ns_dt) || !parse_record(L[3], 2, dxz) || !parse_record(L[11], 4, wb) ||
        !parse_record(L[12], 4, wt) || !parse_ints(L[13], 1, inc))
        return gfail(PRJ_ERR_ARG, "%s: a record holds fewer values than base_params.txt has", path);
    std::memset(out, 0, sizeof(*out));
    out->nx = (int)g[0];
    out->nz = (int)g[1];
    out->ny = (int)g[2];
    out->use_rough_surf = (int)rough[0];
    out->nstep = nst[0];
    out->dtmax = ns_dt[1];
    out->dx = dxz[0];
    out->dz = dxz[1];
    out->wall_U_bot = wb[0];
    out->wall_V_bot = wb[1];
    out->wall_W_bot = wb[2];
    out->wall_U_top = wt[0];
    out->wall_V_top = wt[1];
    out->wall_W_top = wt[2];
    out->use_incompressible = (int)inc[0];
    if (out->nx < 1 || out->nz < 1 || out->ny < 1 || !(out->dx > 0) || !(out->dz > 0))
        return gfail(PRJ_ERR_ARG, "%s: grid %d x %d x %d with dx=%g dz=%g is not a valid case", path, out->nx, out->nz,
                     out->ny, out->dx, out->dz);
    return PRJ_OK;
}

}  // extern "C"
