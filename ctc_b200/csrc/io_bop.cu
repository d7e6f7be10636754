// Particle files in the bop format and the restart files built on it (host
// code).
//
// A bop file NAME is a text header NAME.bop and a values file NAME.values.
// The header holds the record count on its first line, then the lines
// "DATA_FILE: <values file, relative to the header's folder>",
// "DATA_FORMAT: float|int|ascii|iascii" and "VARIABLES: <names>", as the
// external bop library writes them (its files under the reference's
// post/*/data show the layout).  float/int values are raw little-endian 4-byte
// words, nvars per record; ascii/iascii are whitespace-separated text.
//
// restart_write_pp/ii and restart_read_pp/ii (src/io/restart/imp/main.h)
// name the file base/code/ID with ID "templ" (-1), "final" (-2) or %05d, the
// particles as BopFLOAT "x y z vx vy vz", the integers as BopINT "i".
// io_bop_parts/ids/colors (src/io/bop/imp/main.h) write
// dump_base/bop/name-%05d, positions shifted to the box's edge
// (local2global of one rank: x + (0 + 1/2) L in float).
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/ctc_b200.h"
#include "api_util.h"

using ctc::fail;

namespace {

std::string dir_of(const std::string &p) {
    const size_t k = p.rfind('/');
    return k == std::string::npos ? std::string() : p.substr(0, k);
}
std::string base_of(const std::string &p) {
    const size_t k = p.rfind('/');
    return k == std::string::npos ? p : p.substr(k + 1);
}

int mkdir_p(const std::string &d) {   // creates d and its parents
    if (d.empty()) return 0;
    struct stat sb;
    if (stat(d.c_str(), &sb) == 0) return S_ISDIR(sb.st_mode) ? 0 : -1;
    if (mkdir_p(dir_of(d))) return -1;
    return (mkdir(d.c_str(), 0755) == 0 || errno == EEXIST) ? 0 : -1;
}

std::string restart_name(const char *base, const char *code, int id) {
    char idc[32];
    if (id == CTC_RESTART_TEMPL) snprintf(idc, sizeof(idc), "templ");
    else if (id == CTC_RESTART_FINAL) snprintf(idc, sizeof(idc), "final");
    else snprintf(idc, sizeof(idc), "%05d", id);
    return std::string(base) + "/" + code + "/" + idc;
}

int nwords(const char *vars) {
    int n = 0;
    for (const char *c = vars; *c;) {
        while (*c == ' ') c++;
        if (!*c) break;
        n++;
        while (*c && *c != ' ') c++;
    }
    return n;
}

}  // namespace

extern "C" int ctc_bop_write(const char *name, long n, int type, const char *vars, const void *data) {
    if (!name || n < 0 || (type != CTC_BOP_FLOAT && type != CTC_BOP_INT) || !vars || (n > 0 && !data))
        return fail(CTC_ERR_ARG, "ctc_bop_write: bad arguments");
    const int nv = nwords(vars);
    if (nv <= 0) return fail(CTC_ERR_ARG, "ctc_bop_write: no variables");
    const std::string nm(name), hname = nm + ".bop", vname = nm + ".values";
    if (mkdir_p(dir_of(nm))) return fail(CTC_ERR_ARG, "ctc_bop_write: cannot create the folder of %s", name);
    FILE *f = fopen(hname.c_str(), "w");
    if (!f) return fail(CTC_ERR_ARG, "ctc_bop_write: cannot open %s", hname.c_str());
    bool ok = fprintf(f, "%ld\nDATA_FILE: %s\nDATA_FORMAT: %s\nVARIABLES: %s\n", n, base_of(vname).c_str(),
                      type == CTC_BOP_FLOAT ? "float" : "int", vars) > 0;
    ok = (fclose(f) == 0) && ok;
    f = fopen(vname.c_str(), "wb");
    if (!f) return fail(CTC_ERR_ARG, "ctc_bop_write: cannot open %s", vname.c_str());
    const size_t cnt = (size_t)n * nv;
    ok = ok && (cnt == 0 || fwrite(data, 4, cnt, f) == cnt);
    ok = (fclose(f) == 0) && ok;
    return ok ? CTC_OK : fail(CTC_ERR_ARG, "ctc_bop_write: write failed on %s", name);
}

extern "C" int ctc_bop_read(const char *header, long cap, long *pn, int *ptype, int *pnvars, void *data) {
    if (!header || !pn) return fail(CTC_ERR_ARG, "ctc_bop_read: bad arguments");
    FILE *f = fopen(header, "r");
    if (!f) return fail(CTC_ERR_ARG, "ctc_bop_read: cannot open %s", header);
    long n = -1;
    std::string dfile, fmt, vars;
    char line[4096];
    if (fgets(line, sizeof(line), f)) n = strtol(line, nullptr, 10);
    while (fgets(line, sizeof(line), f)) {
        std::string s(line);
        while (!s.empty() && (s.back() == '\n' || s.back() == '\r' || s.back() == ' ')) s.pop_back();
        auto val = [&](const char *key) -> const char * {
            const size_t k = strlen(key);
            if (s.compare(0, k, key) != 0) return nullptr;
            const char *v = s.c_str() + k;
            while (*v == ' ') v++;
            return v;
        };
        if (const char *v = val("DATA_FILE:")) dfile = v;
        else if (const char *v = val("DATA_FORMAT:")) fmt = v;
        else if (const char *v = val("VARIABLES:")) vars = v;
    }
    fclose(f);
    const int nv = nwords(vars.c_str());
    const bool bin = fmt == "float" || fmt == "int", txt = fmt == "ascii" || fmt == "iascii";
    if (n < 0 || dfile.empty() || nv <= 0 || !(bin || txt))
        return fail(CTC_ERR_ARG, "ctc_bop_read: malformed header %s", header);
    *pn = n;
    if (ptype) *ptype = (fmt == "float" || fmt == "ascii") ? CTC_BOP_FLOAT : CTC_BOP_INT;
    if (pnvars) *pnvars = nv;
    if (!data) return CTC_OK;   // header only
    const size_t cnt = (size_t)n * nv;
    if ((long)cnt > cap) return fail(CTC_ERR_CAPACITY, "ctc_bop_read: %ld values > capacity %ld", (long)cnt, cap);
    const std::string d = dir_of(header), vpath = (dfile[0] == '/' || d.empty()) ? dfile : d + "/" + dfile;
    f = fopen(vpath.c_str(), bin ? "rb" : "r");
    if (!f) return fail(CTC_ERR_ARG, "ctc_bop_read: cannot open %s", vpath.c_str());
    bool ok = true;
    if (bin) ok = cnt == 0 || fread(data, 4, cnt, f) == cnt;
    else if (fmt == "ascii")
        for (size_t i = 0; ok && i < cnt; i++) ok = fscanf(f, "%f", (float *)data + i) == 1;
    else
        for (size_t i = 0; ok && i < cnt; i++) ok = fscanf(f, "%d", (int *)data + i) == 1;
    fclose(f);
    return ok ? CTC_OK : fail(CTC_ERR_ARG, "ctc_bop_read: short values file %s", vpath.c_str());
}

extern "C" int ctc_restart_write_pp(const char *base, const char *code, int id, long n, const float *pp) {
    if (!base || !code) return fail(CTC_ERR_ARG, "ctc_restart_write_pp: bad arguments");
    return ctc_bop_write(restart_name(base, code, id).c_str(), n, CTC_BOP_FLOAT, "x y z vx vy vz", pp);
}

extern "C" int ctc_restart_write_ii(const char *base, const char *code, int id, long n, const int *ii) {
    if (!base || !code) return fail(CTC_ERR_ARG, "ctc_restart_write_ii: bad arguments");
    return ctc_bop_write(restart_name(base, code, id).c_str(), n, CTC_BOP_INT, "i", ii);
}

static int restart_read(const char *base, const char *code, int id, int want_type, int want_nv, long cap, long *n,
                        void *out) {
    if (!base || !code || !n) return fail(CTC_ERR_ARG, "restart read: bad arguments");
    const std::string h = restart_name(base, code, id) + ".bop";
    int type = 0, nv = 0;
    int rc = ctc_bop_read(h.c_str(), 0, n, &type, &nv, nullptr);
    if (rc) return rc;
    if (type != want_type || nv != want_nv)
        return fail(CTC_ERR_ARG, "restart read: %s holds %d %s values a record", h.c_str(), nv,
                    type == CTC_BOP_FLOAT ? "float" : "int");
    return out ? ctc_bop_read(h.c_str(), cap * want_nv, n, nullptr, nullptr, out) : CTC_OK;
}

extern "C" int ctc_restart_read_pp(const char *base, const char *code, int id, long cap, long *n, float *pp) {
    return restart_read(base, code, id, CTC_BOP_FLOAT, 6, cap, n, pp);
}

extern "C" int ctc_restart_read_ii(const char *base, const char *code, int id, long cap, long *n, int *ii) {
    return restart_read(base, code, id, CTC_BOP_INT, 1, cap, n, ii);
}

static std::string dump_name(const char *dump_base, const char *name, int id) {
    char tail[64];
    snprintf(tail, sizeof(tail), "-%05d", id);
    return std::string(dump_base) + "/bop/" + name + tail;
}

extern "C" int ctc_io_bop_parts(const char *dump_base, const char *name, int id, long n, const float *pp,
                                const float *ff, int LX, int LY, int LZ) {
    if (!dump_base || !name || n < 0 || (n > 0 && !pp)) return fail(CTC_ERR_ARG, "ctc_io_bop_parts: bad arguments");
    const int nr = ff ? 9 : 6;
    const float o[3] = {0.5f * (float)LX, 0.5f * (float)LY, 0.5f * (float)LZ};
    std::vector<float> w((size_t)n * nr);
    for (size_t i = 0; i < (size_t)n; i++) {
        float *q = w.data() + i * nr;
        for (int k = 0; k < 3; k++) q[k] = o[k] + pp[6 * i + k];    // (0 + 0.5f) * L + x
        for (int k = 3; k < 6; k++) q[k] = pp[6 * i + k];
        if (ff)
            for (int k = 0; k < 3; k++) q[6 + k] = ff[3 * i + k];
    }
    return ctc_bop_write(dump_name(dump_base, name, id).c_str(), n, CTC_BOP_FLOAT,
                         ff ? "x y z vx vy vz fx fy fz" : "x y z vx vy vz", w.data());
}

extern "C" int ctc_io_bop_ints(const char *dump_base, const char *name, int id, long n, const int *ii, int colors) {
    if (!dump_base || !name || n < 0 || (n > 0 && !ii)) return fail(CTC_ERR_ARG, "ctc_io_bop_ints: bad arguments");
    return ctc_bop_write(dump_name(dump_base, name, id).c_str(), n, CTC_BOP_INT, colors ? "color" : "ids", ii);
}
