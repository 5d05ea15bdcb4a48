// io.cpp -- the reference's state files (new_dynamics.cpp:123-139, 228-236)
// and input files (helpers.h:299-340 read_points), plus a binary
// equivalent of the state file.
//
// Text: every value is written as the default-formatted C++ stream writes a
// double (%g with 6 significant digits, the "C" locale), here by
// std::to_chars(general, 6), which produces the same characters.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fss.h"

namespace fss {
void set_last_error(const std::string& msg);
}

namespace {

int iofail(int code, const std::string& m) {
    fss::set_last_error(m);
    return code;
}

// One double as `os << x` writes it by default.
inline char* put_g6(char* p, double x) {
    if (std::isnan(x)) {  // glibc's %g: "nan" / "-nan"
        const char* s = std::signbit(x) ? "-nan" : "nan";
        const size_t l = std::strlen(s);
        std::memcpy(p, s, l);
        return p + l;
    }
    if (std::isinf(x)) {
        const char* s = x < 0 ? "-inf" : "inf";
        const size_t l = std::strlen(s);
        std::memcpy(p, s, l);
        return p + l;
    }
    return std::to_chars(p, p + 32, x, std::chars_format::general, 6).ptr;
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

// Next line of `f` into `line` (without the newline); false at the end.
bool next_line(FILE* f, std::string& line) {
    line.clear();
    int c;
    while ((c = std::fgetc(f)) != EOF && c != '\n') line.push_back(char(c));
    return !(c == EOF && line.empty());
}

// The first `count` comma-separated fields of `line` as doubles (stod:
// leading blanks skipped, the longest valid prefix parsed); false when a
// field is missing or has no number.
bool fields(const std::string& line, int count, double* out) {
    size_t pos = 0;
    for (int j = 0; j < count; j++) {
        if (pos > line.size()) return false;
        size_t end = line.find(',', pos);
        if (end == std::string::npos) end = line.size();
        const std::string w = line.substr(pos, end - pos);
        char* stop = nullptr;
        out[j] = std::strtod(w.c_str(), &stop);
        if (stop == w.c_str()) return false;
        pos = end + 1;
    }
    return true;
}

constexpr char kBinMagic[8] = {'F', 'S', 'S', 'S', 'T', 'A', 'T', '1'};

}  // namespace

extern "C" {

int fss_state_csv_append(const char* path, int64_t n, const double* state5, const double* area) {
    if (!path || n < 0 || (n > 0 && (!state5 || !area))) return iofail(FSS_ERR_INVALID, "bad state file arguments");
    File out;
    out.f = std::fopen(path, "ab");
    if (!out.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    std::vector<char> buf(size_t(1) << 20);
    size_t used = 0;
    for (int64_t i = 0; i < n; i++) {
        if (buf.size() - used < 6 * 40) {
            if (std::fwrite(buf.data(), 1, used, out.f) != used) return iofail(FSS_ERR_INVALID, "write failed");
            used = 0;
        }
        char* p = buf.data() + used;
        for (int c = 0; c < 5; c++) {
            p = put_g6(p, state5[5 * i + c]);
            *p++ = ',';
        }
        p = put_g6(p, area[i]);
        *p++ = '\n';
        used = size_t(p - buf.data());
    }
    if (std::fwrite(buf.data(), 1, used, out.f) != used) return iofail(FSS_ERR_INVALID, "write failed");
    return FSS_OK;
}

int fss_point_count_append(const char* path, int64_t n) {
    if (!path) return iofail(FSS_ERR_INVALID, "null path");
    File out;
    out.f = std::fopen(path, "ab");
    if (!out.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    if (std::fprintf(out.f, "%lld\n", (long long)n) < 0) return iofail(FSS_ERR_INVALID, "write failed");
    return FSS_OK;
}

int fss_output_name(char* buf, int64_t cap, int64_t point_count, const char* init_cond, int use_fast,
                    int tree_levels, int use_amr, int use_mpi, int use_remesh, int64_t time_steps) {
    if (!buf || cap < 1 || !init_cond) return iofail(FSS_ERR_INVALID, "bad name arguments");
    std::string s = std::to_string(point_count) + "_" + init_cond + "_";
    s += use_fast ? "fast_" + std::to_string(tree_levels) : std::string("direct");
    if (use_amr) s += "_amr";
    if (use_mpi) s += "_mpi";
    if (use_remesh) s += "_remesh";
    s += "_" + std::to_string(time_steps);
    if (int64_t(s.size()) + 1 > cap) return iofail(FSS_ERR_CAPACITY, "name buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return FSS_OK;
}

int fss_state_bin_append(const char* path, int64_t n, const double* state5, const double* area) {
    if (!path || n < 0 || (n > 0 && (!state5 || !area))) return iofail(FSS_ERR_INVALID, "bad state file arguments");
    File out;
    out.f = std::fopen(path, "ab");
    if (!out.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    const int64_t hdr = n;
    bool ok = std::fwrite(kBinMagic, 1, 8, out.f) == 8 && std::fwrite(&hdr, 8, 1, out.f) == 1;
    std::vector<double> row(size_t(6) * std::min<int64_t>(n, 65536));
    for (int64_t i0 = 0; ok && i0 < n; i0 += 65536) {
        const int64_t m = std::min<int64_t>(65536, n - i0);
        for (int64_t i = 0; i < m; i++) {
            std::memcpy(&row[6 * i], state5 + 5 * (i0 + i), 5 * sizeof(double));
            row[6 * i + 5] = area[i0 + i];
        }
        ok = std::fwrite(row.data(), sizeof(double), size_t(6 * m), out.f) == size_t(6 * m);
    }
    return ok ? FSS_OK : iofail(FSS_ERR_INVALID, "write failed");
}

int fss_state_bin_read(const char* path, int64_t step, int64_t cap, double* state5, double* area, int64_t* n_out) {
    if (!path || step < 0 || !n_out) return iofail(FSS_ERR_INVALID, "bad state file arguments");
    File in;
    in.f = std::fopen(path, "rb");
    if (!in.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    for (int64_t s = 0;; s++) {
        char magic[8];
        int64_t n = 0;
        if (std::fread(magic, 1, 8, in.f) != 8 || std::fread(&n, 8, 1, in.f) != 1)
            return iofail(FSS_ERR_INVALID, "no such step in the state file");
        if (std::memcmp(magic, kBinMagic, 8) != 0 || n < 0) return iofail(FSS_ERR_INVALID, "not a state file");
        if (s < step) {
            if (std::fseek(in.f, long(6 * sizeof(double) * n), SEEK_CUR) != 0)
                return iofail(FSS_ERR_INVALID, "truncated state file");
            continue;
        }
        *n_out = n;
        if (n > cap) return iofail(FSS_ERR_CAPACITY, "state arrays too small");
        std::vector<double> row(6);
        for (int64_t i = 0; i < n; i++) {
            if (std::fread(row.data(), sizeof(double), 6, in.f) != 6)
                return iofail(FSS_ERR_INVALID, "truncated state file");
            if (state5) std::memcpy(state5 + 5 * i, row.data(), 5 * sizeof(double));
            if (area) area[i] = row[5];
        }
        return FSS_OK;
    }
}

int fss_read_points_csv(const char* path, int64_t n, double* state5) {
    if (!path || n < 0 || (n > 0 && !state5)) return iofail(FSS_ERR_INVALID, "bad arguments");
    File in;
    in.f = std::fopen(path, "rb");
    if (!in.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    std::string line;
    for (int64_t i = 0; i < n; i++) {
        double v[4];
        if (!next_line(in.f, line) || !fields(line, 4, v))
            return iofail(FSS_ERR_INVALID, "points file: line " + std::to_string(i + 1));
        for (int j = 0; j < 4; j++) state5[5 * i + j] = v[j];
    }
    return FSS_OK;
}

int fss_read_tris_csv(const char* path, int64_t ntri, int32_t* tris) {
    if (!path || ntri < 0 || (ntri > 0 && !tris)) return iofail(FSS_ERR_INVALID, "bad arguments");
    File in;
    in.f = std::fopen(path, "rb");
    if (!in.f) return iofail(FSS_ERR_INVALID, std::string("cannot open ") + path);
    std::string line;
    for (int64_t t = 0; t < ntri; t++) {
        double v[3];
        if (!next_line(in.f, line) || !fields(line, 3, v))
            return iofail(FSS_ERR_INVALID, "triangles file: line " + std::to_string(t + 1));
        for (int j = 0; j < 3; j++) tris[3 * t + j] = int32_t(v[j]);  // stod, then int
    }
    return FSS_OK;
}

int fss_read_vert_tris_csv(const char* lists_path, const char* counts_path, int64_t n, int32_t* off, int32_t* adj,
                           int64_t cap) {
    if (!lists_path || !counts_path || n < 0 || !off) return iofail(FSS_ERR_INVALID, "bad arguments");
    File fl, fc;
    fl.f = std::fopen(lists_path, "rb");
    fc.f = std::fopen(counts_path, "rb");
    if (!fl.f || !fc.f) return iofail(FSS_ERR_INVALID, "cannot open the vert_tris files");
    std::string line;
    int64_t a = 0;
    off[0] = 0;
    for (int64_t i = 0; i < n; i++) {
        double cnt;
        if (!next_line(fc.f, line) || !fields(line, 1, &cnt) || !(cnt >= 0))
            return iofail(FSS_ERR_INVALID, "vert_tri_count file: line " + std::to_string(i + 1));
        const int k = int(cnt);
        std::vector<double> v(size_t(std::max(k, 1)));
        if (!next_line(fl.f, line) || (k > 0 && !fields(line, k, v.data())))
            return iofail(FSS_ERR_INVALID, "vert_tris file: line " + std::to_string(i + 1));
        if (a + k > cap) return iofail(FSS_ERR_CAPACITY, "adjacency array too small");
        for (int j = 0; j < k; j++) adj[a++] = int32_t(v[j]);
        off[i + 1] = int32_t(a);
    }
    return FSS_OK;
}

}  // extern "C"
