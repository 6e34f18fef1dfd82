// io.cpp -- output and input formats of one quantity (host side).
//
// The formats of the reference's ovf/ and dump/ packages, written from the engine's
// internal (Z,Y,X) SoA float32 layout [comp][n0][n1][n2]:
//   OVF 2.0  (ovf/ovf2_output.go:34-161): text header, "Binary 4" little-endian or "Text";
//   OMF 1.0  (ovf/omf_output.go:34-206): text header, "Binary 4" big-endian or "Text";
//   dump     (dump/writer.go:34-97, engine/format_dump.go:40-62): 64-bit header words,
//            the raw float32 list, CRC-64 (ISO polynomial, Go's hash/crc64) of the frame.
// Cells are written x fastest (user axes), i.e. in the internal C order, and vector
// components in user order (internal component 2 first), as the reference's loops do.
// Readers: OMF/OVF (ovf/omf_input.go:27-260, extended to OVF 2.0 headers) and dump
// (dump/reader.go:28-131).
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mm_b200.h"

namespace mm {
int report_error(int code, const char* msg);
}

namespace {

// ---------------------------------------------------------------- number formatting
// Go's fmt %v of a float: the shortest digits that round-trip at the value's own
// precision (float32 or float64), in strconv's 'g' form, which uses the exponent form
// when the decimal exponent is < -4 or >= 6.
template <typename F>
std::string go_float(F v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "+Inf" : "-Inf";
    if (v == 0) return std::signbit(v) ? "-0" : "0";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    *r.ptr = 0;
    // buf = [-]d[.ddd]e(+|-)xx
    std::string s(buf);
    const bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    const size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    const int x = std::stoi(s.substr(e + 1));
    std::string digits;
    for (char c : mant)
        if (c != '.') digits += c;
    std::string out;
    if (x < -4 || x >= 6) {
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char eb[16];
        snprintf(eb, sizeof eb, "e%c%02d", x < 0 ? '-' : '+', x < 0 ? -x : x);
        out += eb;
    } else {
        const int nd = (int)digits.size(), dp = x + 1;
        if (dp <= 0) out = "0." + std::string(-dp, '0') + digits;
        else if (dp >= nd) out = digits + std::string(dp - nd, '0');
        else out = digits.substr(0, dp) + "." + digits.substr(dp);
    }
    return neg ? "-" + out : out;
}

// "# Key: v1 v2 ...\n" (hdr of ovf/omf_output.go:197-200: Fprint then Fprintln, whose
// operands are separated by single spaces)
struct Out {
    FILE* f;
    void line(const std::string& s) { fputs(s.c_str(), f); fputc('\n', f); }
    void hdr(const std::string& key, const std::string& v) { line("# " + key + ": " + v); }
};

// user-order component c of internal array (reference SwapIndex)
inline int swap_comp(int c, int ncomp) { return ncomp == 3 ? 2 - c : c; }

void data_values(const float* data, int ncomp, const int n[3], std::vector<float>& out) {
    const long long N = (long long)n[0] * n[1] * n[2];
    out.resize((size_t)N * ncomp);
    for (long long i = 0; i < N; i++)
        for (int c = 0; c < ncomp; c++) out[(size_t)i * ncomp + c] = data[swap_comp(c, ncomp) * N + i];
}

void write_text_data(FILE* f, const std::vector<float>& v, int ncomp) {
    std::string line;
    for (size_t i = 0; i < v.size(); i += ncomp) {
        line.clear();
        for (int c = 0; c < ncomp; c++) line += go_float(v[i + c]) + " ";
        line += "\n";
        fputs(line.c_str(), f);
    }
}

void write_bin4(FILE* f, std::vector<float>& v, bool big_endian) {
    float ctrl = 1234567.0f;  // OMF_CONTROL_NUMBER
    auto put = [&](float* p, size_t n) {
        if (big_endian)
            for (size_t i = 0; i < n; i++) {
                uint32_t u;
                memcpy(&u, p + i, 4);
                u = __builtin_bswap32(u);
                memcpy(p + i, &u, 4);
            }
        fwrite(p, 4, n, f);
    };
    put(&ctrl, 1);
    put(v.data(), v.size());
}

std::string go_vec_line(std::initializer_list<std::string> parts) {
    std::string s;
    for (auto& p : parts) s += (s.empty() ? "" : " ") + p;
    return s;
}

// ---------------------------------------------------------------- CRC-64 (Go hash/crc64, ISO)
struct Crc64 {
    uint64_t tab[256];
    uint64_t crc = 0;
    Crc64() {
        const uint64_t poly = 0xD800000000000000ULL;  // crc64.ISO, reversed representation
        for (int i = 0; i < 256; i++) {
            uint64_t c = (uint64_t)i;
            for (int k = 0; k < 8; k++) c = (c & 1) ? (c >> 1) ^ poly : c >> 1;
            tab[i] = c;
        }
    }
    void update(const void* p, size_t n) {
        const unsigned char* b = (const unsigned char*)p;
        uint64_t c = ~crc;
        for (size_t i = 0; i < n; i++) c = tab[(uint8_t)c ^ b[i]] ^ (c >> 8);
        crc = ~c;
    }
};

}  // namespace

// ---------------------------------------------------------------- C-ABI
extern "C" MM_API uint64_t mm_crc64_iso(const void* data, size_t n) {
    Crc64 c;
    c.update(data, n);
    return c.crc;
}

extern "C" MM_API int mm_write_field(const char* path, int format, const float* data, int ncomp, const int n[3],
                                     const double cell[3], double time, const char* name, const char* unit) {
    if (!path || !data || !n || !cell || (ncomp != 1 && ncomp != 3))
        return mm::report_error(MM_ERR_ARG, "mm_write_field: bad argument");
    const std::string qn = name ? name : "", qu = unit ? unit : "";
    const bool dump = format == MM_FMT_DUMP;
    FILE* f = fopen(path, dump ? "ab" : "wb");
    if (!f) return mm::report_error(MM_ERR_ARG, ("cannot open " + std::string(path)).c_str());
    Out o{f};
    // user axes: x = internal 2, z = internal 0
    const int X = 2, Y = 1, Z = 0;
    if (format == MM_FMT_OVF2_BIN4 || format == MM_FMT_OVF2_TEXT) {
        o.line("# OOMMF OVF 2.0");
        o.line("#");
        o.hdr("Segment count", "1");
        o.line("#");
        o.hdr("Begin", "Segment");
        o.hdr("Begin", "Header");
        o.line("#");
        o.hdr("Title", "mumax data");
        o.hdr("meshtype", "rectangular");
        o.hdr("meshunit", "m");
        o.hdr("xmin", "0");
        o.hdr("ymin", "0");
        o.hdr("zmin", "0");
        o.hdr("xmax", go_float(cell[X] * (double)n[X]));
        o.hdr("ymax", go_float(cell[Y] * (double)n[Y]));
        o.hdr("zmax", go_float(cell[Z] * (double)n[Z]));
        o.hdr("valuedim", std::to_string(ncomp));
        const std::string u = qu.empty() ? "1" : qu;
        if (ncomp == 1) {
            o.hdr("valuelabels", qn);
            o.hdr("valueunits", u);
        } else {
            o.hdr("valuelabels", go_vec_line({qn + "_x", qn + "_y", qn + "_z"}));
            o.hdr("valueunits", go_vec_line({u, u, u}));
        }
        o.line("# Desc: Stage simulation time:  " + go_float(time) + "  s");
        o.line("# Desc: Total simulation time:  " + go_float(time) + "  s");
        o.hdr("xbase", go_float(cell[X] / 2));
        o.hdr("ybase", go_float(cell[Y] / 2));
        o.hdr("zbase", go_float(cell[Z] / 2));
        o.hdr("xnodes", std::to_string(n[X]));
        o.hdr("ynodes", std::to_string(n[Y]));
        o.hdr("znodes", std::to_string(n[Z]));
        o.hdr("xstepsize", go_float(cell[X]));
        o.hdr("ystepsize", go_float(cell[Y]));
        o.hdr("zstepsize", go_float(cell[Z]));
        o.line("#");
        o.hdr("End", "Header");
        o.line("#");
        const std::string df = format == MM_FMT_OVF2_BIN4 ? "Binary 4" : "Text";
        o.hdr("Begin", "Data " + df);
        std::vector<float> v;
        data_values(data, ncomp, n, v);
        if (format == MM_FMT_OVF2_BIN4) write_bin4(f, v, false);
        else write_text_data(f, v, ncomp);
        o.hdr("End", "Data " + df);
        o.hdr("End", "Segment");
    } else if (format == MM_FMT_OMF_BIN4 || format == MM_FMT_OMF_TEXT) {
        o.hdr("OOMMF", "rectangular mesh v1.0");
        o.hdr("Segment count", "1");
        o.hdr("Begin", "Segment");
        o.hdr("Begin", "Header");
        o.hdr("Desc", "Time :  " + go_float(time));
        o.hdr("Title", qn);
        o.hdr("meshtype", "rectangular");
        o.hdr("meshunit", "m");
        o.hdr("xbase", go_float(cell[X] / 2));
        o.hdr("ybase", go_float(cell[Y] / 2));
        o.hdr("zbase", go_float(cell[Z] / 2));
        o.hdr("xstepsize", go_float(cell[X]));
        o.hdr("ystepsize", go_float(cell[Y]));
        o.hdr("zstepsize", go_float(cell[Z]));
        o.hdr("xmin", "0");
        o.hdr("ymin", "0");
        o.hdr("zmin", "0");
        o.hdr("xmax", go_float(cell[X] * (double)n[X]));
        o.hdr("ymax", go_float(cell[Y] * (double)n[Y]));
        o.hdr("zmax", go_float(cell[Z] * (double)n[Z]));
        o.hdr("xnodes", std::to_string(n[X]));
        o.hdr("ynodes", std::to_string(n[Y]));
        o.hdr("znodes", std::to_string(n[Z]));
        o.hdr("ValueRangeMinMag", "1e-08");
        o.hdr("ValueRangeMaxMag", "1");
        o.hdr("valueunit", qu);
        o.hdr("valuemultiplier", "1");
        o.hdr("End", "Header");
        const std::string df = format == MM_FMT_OMF_BIN4 ? "Binary 4" : "Text";
        o.hdr("Begin", "Data " + df);
        std::vector<float> v;
        data_values(data, ncomp, n, v);
        if (format == MM_FMT_OMF_BIN4) write_bin4(f, v, true);
        else write_text_data(f, v, ncomp);
        o.hdr("End", "Data " + df);
        o.hdr("End", "Segment");
    } else if (dump) {
        Crc64 crc;
        auto w = [&](const void* p, size_t nb) {
            crc.update(p, nb);
            fwrite(p, 1, nb, f);
        };
        auto wstr = [&](const std::string& s) {
            char b[8] = {0};
            memcpy(b, s.data(), s.size() < 8 ? s.size() : 8);
            w(b, 8);
        };
        auto wu = [&](uint64_t x) { w(&x, 8); };
        auto wd = [&](double x) { w(&x, 8); };
        wstr("#dump002");
        wu((uint64_t)ncomp);
        for (int i = 0; i < 3; i++) wu((uint64_t)n[i]);
        for (int i = 0; i < 3; i++) wd(cell[i]);  // internal order, not swapped (format_dump.go:58)
        wstr("m");
        wd(time);
        wstr("s");
        wstr(qn);
        wstr(qu);
        wu(4);  // FLOAT32
        w(data, sizeof(float) * (size_t)ncomp * n[0] * n[1] * n[2]);
        const uint64_t h = crc.crc;
        fwrite(&h, 8, 1, f);
    } else {
        fclose(f);
        return mm::report_error(MM_ERR_ARG, "mm_write_field: unknown format");
    }
    const bool bad = ferror(f) != 0;
    fclose(f);
    if (bad) return mm::report_error(MM_ERR_ARG, ("write error on " + std::string(path)).c_str());
    return MM_OK;
}

// ---------------------------------------------------------------- readers
namespace {

std::string lower(std::string s) {
    for (auto& c : s) c = (char)tolower((unsigned char)c);
    return s;
}
std::string trim(const std::string& s, const char* set) {
    size_t a = s.find_first_not_of(set), b = s.find_last_not_of(set);
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

bool read_line(FILE* f, std::string& line) {
    line.clear();
    int c;
    while ((c = fgetc(f)) != EOF) {
        if (c == '\n') return true;
        line += (char)c;
    }
    return !line.empty();
}

}  // namespace

// Reads the first field of an OMF 1.0 / OVF 2.0 ("Binary 4" or "Text") or dump file
// into data [ncomp][n0][n1][n2] (internal order; may be NULL to query the sizes).
extern "C" MM_API int mm_read_field(const char* path, float* data, long long capacity, int* ncomp, int n[3],
                                    double* time) {
    if (!path || !ncomp || !n) return mm::report_error(MM_ERR_ARG, "mm_read_field: bad argument");
    FILE* f = fopen(path, "rb");
    if (!f) return mm::report_error(MM_ERR_ARG, ("cannot open " + std::string(path)).c_str());
    char magic[8] = {0};
    size_t got = fread(magic, 1, 8, f);
    auto fail = [&](const std::string& msg) {
        fclose(f);
        return mm::report_error(MM_ERR_ARG, (std::string(path) + ": " + msg).c_str());
    };
    if (got == 8 && memcmp(magic, "#dump002", 8) == 0) {
        Crc64 crc;
        crc.update(magic, 8);
        auto ru = [&](uint64_t& x) {
            bool ok = fread(&x, 8, 1, f) == 1;
            crc.update(&x, 8);
            return ok;
        };
        uint64_t comps, sz[3], prec, w;
        double step[3], t;
        bool ok = ru(comps);
        for (int i = 0; i < 3; i++) ok = ru(sz[i]) && ok;
        for (int i = 0; i < 3; i++) { ok = ru(w) && ok; memcpy(&step[i], &w, 8); }
        ok = ru(w) && ok;  // mesh unit
        ok = ru(w) && ok;
        memcpy(&t, &w, 8);
        for (int i = 0; i < 3; i++) ok = ru(w) && ok;  // time unit, label, unit
        ok = ru(prec) && ok;
        if (!ok) return fail("truncated dump header");
        if (prec != 4) return fail("dump precision is not float32");
        *ncomp = (int)comps;
        for (int i = 0; i < 3; i++) n[i] = (int)sz[i];
        if (time) *time = t;
        const long long total = (long long)comps * sz[0] * sz[1] * sz[2];
        if (!data) { fclose(f); return MM_OK; }
        if (total > capacity) return fail("buffer too small");
        if ((long long)fread(data, 4, (size_t)total, f) != total) return fail("truncated dump data");
        crc.update(data, 4 * (size_t)total);
        uint64_t stored;
        if (fread(&stored, 8, 1, f) != 1) return fail("missing dump CRC");
        if (stored != 0 && stored != crc.crc) return fail("dump CRC error");
        fclose(f);
        return MM_OK;
    }
    // OMF / OVF text header
    fseek(f, 0, SEEK_SET);
    std::string line;
    int nodes[3] = {0, 0, 0}, dim = 3;
    bool v2 = false;
    double t = 0;
    std::string fmt, dfmt;
    bool first = true;
    while (read_line(f, line)) {
        std::string body = trim(line, "# \r\t");
        if (first) { v2 = lower(body).find("ovf 2.0") != std::string::npos; first = false; }
        const size_t colon = body.find(':');
        if (colon == std::string::npos) continue;
        const std::string key = lower(trim(body.substr(0, colon), "# \t"));
        const std::string val = trim(body.substr(colon + 1), "# \t\r");
        if (key == "xnodes") nodes[2] = atoi(val.c_str());
        else if (key == "ynodes") nodes[1] = atoi(val.c_str());
        else if (key == "znodes") nodes[0] = atoi(val.c_str());
        else if (key == "valuedim") dim = atoi(val.c_str());
        else if (key == "desc") {
            const std::string lv = lower(val);
            size_t p = lv.find("time");
            size_t c2 = val.find(':', p == std::string::npos ? 0 : p);
            if (p != std::string::npos && c2 != std::string::npos) t = atof(val.c_str() + c2 + 1);
        } else if (key == "begin" && lower(val).rfind("data", 0) == 0) {
            std::string rest = trim(val.substr(4), " \t");
            const size_t sp = rest.find(' ');
            fmt = lower(rest.substr(0, sp));
            dfmt = sp == std::string::npos ? "" : trim(rest.substr(sp + 1), " \t");
            break;
        }
    }
    if (fmt.empty()) return fail("no data section");
    if (nodes[0] < 1 || nodes[1] < 1 || nodes[2] < 1) return fail("missing xnodes/ynodes/znodes");
    *ncomp = dim;
    for (int i = 0; i < 3; i++) n[i] = nodes[i];
    if (time) *time = t;
    if (!data) { fclose(f); return MM_OK; }
    const long long N = (long long)nodes[0] * nodes[1] * nodes[2];
    if (N * dim > capacity) return fail("buffer too small");
    if (fmt == "binary") {
        if (dfmt != "4") return fail("only Binary 4 is supported");
        auto rd = [&](float& v) {
            uint32_t u;
            if (fread(&u, 4, 1, f) != 1) return false;
            if (!v2) u = __builtin_bswap32(u);  // OMF 1.0 is big-endian (omf_input.go:113)
            memcpy(&v, &u, 4);
            return true;
        };
        float ctrl;
        if (!rd(ctrl)) return fail("truncated data");
        if (ctrl != 1234567.0f) return fail("invalid control number");
        for (long long i = 0; i < N; i++)
            for (int c = 0; c < dim; c++)
                if (!rd(data[swap_comp(c, dim) * N + i])) return fail("truncated data");
    } else if (fmt == "text") {
        for (long long i = 0; i < N; i++)
            for (int c = 0; c < dim; c++)
                if (fscanf(f, "%f", &data[swap_comp(c, dim) * N + i]) != 1) return fail("bad text data");
    } else {
        return fail("unknown data format " + fmt);
    }
    fclose(f);
    return MM_OK;
}
