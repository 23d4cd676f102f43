// obj_oracle.cpp - CPU restatement of the reference's OBJ ingest.  TEST INFRASTRUCTURE ONLY.
//
// Part of the parity oracle (oracle/liblvbh_oracle.so): only tests/ and bench.py's CPU-baseline
// arm use it, as the checker; the product library never does.
//
// Restates, in the reference's order, what happens between a dropped .obj file and the build:
//   OBJFile.parse()        scripts/obj/obj-file-parser.js:19-67  (lines split on '\n', comments
//                          cut at '#', runs of whitespace collapsed, keyword lower-cased, the
//                          statements' checks that throw), _parseVertexCoords (:110-116),
//                          _parsePolygon (:153-186), _parseLine (:132-151), _parseGroup (:104-108),
//                          _parseSmoothShadingStatement (:196-201), _currentModel (:80-89)
//   parseObj()             scripts/obj/parse-obj.js:3-88  (model 0's faces fan-triangulated from
//                          their first vertex, y and z swapped, bounds over the faces' vertices
//                          with Math.min / Math.max, two floor triangles at z_min + .01)
//   build()                scripts/bvh/build-bvh.js:14-21 stores the doubles into a
//                          Float32Array (round to nearest, ties to even).
// JavaScript semantics kept: parseFloat takes the longest decimal prefix and rounds correctly
// (glibc strtod on exactly that prefix), parseInt takes an optional sign, a 0x / 0X prefix
// switching to base 16, and the longest digit prefix (NaN if none), Math.min / Math.max
// propagate NaN and order -0 below +0, array indices must be integers in range.  Whitespace is
// JavaScript's `\s` over the UTF-8 text (js_space); other bytes count as ordinary characters.
//
// Parity status: unpinned against a run of the reference (no JavaScript engine in this image).

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

// Bytes of the JavaScript `\s` character (WhiteSpace or LineTerminator) at s[i] in UTF-8, 0 if
// none: ASCII \t \n \v \f \r and space, U+00A0, U+1680, U+2000-200A, U+2028, U+2029, U+202F,
// U+205F, U+3000, U+FEFF.  readAsText decodes the file as UTF-8 and turns a broken sequence into
// U+FFFD before any lead byte, so whitespace is exactly these byte sequences wherever they
// start.
size_t js_space(const std::string &s, size_t i) {
    const unsigned char c = (unsigned char)s[i];
    if (c == ' ' || (c >= 9 && c <= 13)) return 1;
    auto at = [&](size_t k) -> int { return i + k < s.size() ? (unsigned char)s[i + k] : -1; };
    if (c == 0xC2 && at(1) == 0xA0) return 2;
    const int c1 = at(1), c2 = at(2);
    if (c == 0xE1 && c1 == 0x9A && c2 == 0x80) return 3;
    if (c == 0xE2 && c1 == 0x80 && ((c2 >= 0x80 && c2 <= 0x8A) || c2 == 0xA8 || c2 == 0xA9 || c2 == 0xAF)) return 3;
    if (c == 0xE2 && c1 == 0x81 && c2 == 0x9F) return 3;
    if (c == 0xE3 && c1 == 0x80 && c2 == 0x80) return 3;
    if (c == 0xEF && c1 == 0xBB && c2 == 0xBF) return 3;
    return 0;
}

// parseFloat of a whitespace-free token.
double js_parse_float(const std::string &s) {
    size_t i = 0;
    bool neg = false;
    if (i < s.size() && (s[i] == '+' || s[i] == '-')) { neg = s[i] == '-'; ++i; }
    if (s.compare(i, 8, "Infinity") == 0) return neg ? -INFINITY : INFINITY;
    const size_t start = i;
    size_t digits = 0;
    while (i < s.size() && s[i] >= '0' && s[i] <= '9') { ++i; ++digits; }
    if (i < s.size() && s[i] == '.') {
        ++i;
        while (i < s.size() && s[i] >= '0' && s[i] <= '9') { ++i; ++digits; }
    }
    if (digits == 0) return NAN;
    size_t end = i;
    if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
        size_t j = i + 1;
        if (j < s.size() && (s[j] == '+' || s[j] == '-')) ++j;
        size_t ed = 0;
        while (j < s.size() && s[j] >= '0' && s[j] <= '9') { ++j; ++ed; }
        if (ed) end = j;
    }
    const std::string lit = s.substr(start, end - start);
    const double v = std::strtod(lit.c_str(), nullptr);
    return neg ? -v : v;
}

// parseInt of a whitespace-free token, radix undefined.
double js_parse_int(const std::string &s) {
    size_t i = 0;
    bool neg = false;
    if (i < s.size() && (s[i] == '+' || s[i] == '-')) { neg = s[i] == '-'; ++i; }
    int radix = 10;
    if (i + 1 < s.size() && s[i] == '0' && (s[i + 1] == 'x' || s[i + 1] == 'X')) { radix = 16; i += 2; }
    double v = 0.0;
    size_t digits = 0;
    for (; i < s.size(); ++i) {
        int d;
        const char c = s[i];
        if (c >= '0' && c <= '9') d = c - '0';
        else if (radix == 16 && c >= 'a' && c <= 'f') d = c - 'a' + 10;
        else if (radix == 16 && c >= 'A' && c <= 'F') d = c - 'A' + 10;
        else break;
        v = v * radix + d;  // exact while below 2^53, the range any valid index lies in
        ++digits;
    }
    if (!digits) return NAN;
    return neg ? -v : v;
}

inline double js_min(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return NAN;
    if (a == 0.0 && b == 0.0) return std::signbit(a) ? a : b;
    return a < b ? a : b;
}
inline double js_max(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return NAN;
    if (a == 0.0 && b == 0.0) return std::signbit(a) ? b : a;
    return a > b ? a : b;
}

std::string lower(std::string s) {
    for (char &c : s) if (c >= 'A' && c <= 'Z') c = (char)(c - 'A' + 'a');
    return s;
}

std::vector<std::string> split(const std::string &s, char sep) {
    std::vector<std::string> out;
    size_t a = 0;
    for (;;) {
        const size_t b = s.find(sep, a);
        if (b == std::string::npos) { out.push_back(s.substr(a)); break; }
        out.push_back(s.substr(a, b - a));
        a = b + 1;
    }
    return out;
}

struct V3 { double x, y, z; };
struct FaceV { double idx; };
struct Model {
    std::vector<V3> vertices;
    std::vector<std::vector<double>> faces;  // resolved vertex indices (1-based, may be bad)
};

}  // namespace

extern "C" {

// OBJ text -> triangle soup as parseObj + build() produce it.  Returns 0, or -1 where the
// reference throws (err_line: 1-based line of the statement, 0 for a failure after parsing).
// tri_out (12 floats per triangle) may be NULL or too small: *num_tris is always set, the
// triangles are written only when cap_tris suffices.  bounds6: the BOUNDS doubles.
int oracle_parse_obj(const char *text, uint64_t bytes, float *tri_out, uint64_t cap_tris,
                     uint64_t *num_tris, double *bounds6, int64_t *err_line) {
    *err_line = 0;
    *num_tris = 0;
    const std::string all(text, text + bytes);
    std::vector<Model> models;
    auto current = [&]() -> Model & {
        if (models.empty()) models.emplace_back();
        return models.back();
    };
    size_t pos = 0;
    int64_t line_no = 0;
    for (;;) {
        const size_t nl = all.find('\n', pos);
        std::string line = all.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos);
        ++line_no;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::vector<std::string> items;
        {
            // line.replace(/\s+/g, ' ').trim().split(' ')
            size_t i = 0;
            while (i < line.size()) {
                while (i < line.size()) {
                    const size_t w = js_space(line, i);
                    if (!w) break;
                    i += w;
                }
                if (i >= line.size()) break;
                size_t j = i;
                while (j < line.size() && !js_space(line, j)) ++j;
                items.push_back(line.substr(i, j - i));
                i = j;
            }
            if (items.empty()) items.push_back("");
        }
        const std::string kw = lower(items[0]);
        const size_t nitems = items.size();
        if (kw == "o") {
            models.emplace_back();
        } else if (kw == "g") {
            if (nitems != 2) { *err_line = line_no; return -1; }
        } else if (kw == "v") {
            const double x = nitems >= 2 ? js_parse_float(items[1]) : 0.0;
            const double y = nitems >= 3 ? js_parse_float(items[2]) : 0.0;
            const double z = nitems >= 4 ? js_parse_float(items[3]) : 0.0;
            current().vertices.push_back({x, y, z});
        } else if (kw == "vt" || kw == "vn") {
            current();
        } else if (kw == "l") {
            if (nitems - 1 < 2) { *err_line = line_no; return -1; }
            for (size_t i = 1; i < nitems; ++i)
                if (split(items[i], '/').size() > 2) { *err_line = line_no; return -1; }
            current();
        } else if (kw == "s") {
            if (nitems != 2) { *err_line = line_no; return -1; }
        } else if (kw == "f") {
            if (nitems - 1 < 3) { *err_line = line_no; return -1; }
            std::vector<double> face;
            for (size_t i = 1; i < nitems; ++i) {
                const std::vector<std::string> parts = split(items[i], '/');
                if (parts.size() > 3) { *err_line = line_no; return -1; }
                double vi = js_parse_int(parts[0]);
                if (vi == 0.0) { *err_line = line_no; return -1; }
                if (vi < 0.0) vi = (double)current().vertices.size() + 1.0 + vi;
                face.push_back(vi);
            }
            current().faces.push_back(face);
        }
        if (nl == std::string::npos) break;
        pos = nl + 1;
    }
    if (models.empty()) { *err_line = 0; return -1; }  // output.models[0] is undefined
    const Model &m = models[0];
    double xmin = 1e30, ymin = 1e30, zmin = 1e30, xmax = -1e30, ymax = -1e30, zmax = -1e30;
    std::vector<float> tri;
    uint64_t nt = 0;
    auto fetch = [&](double idx, V3 &v) -> bool {
        const double k = idx - 1.0;
        if (!(k >= 0.0) || k != std::floor(k) || k >= (double)m.vertices.size()) return false;
        v = m.vertices[(size_t)k];
        return true;
    };
    const float pad = (float)3.1415;  // the double 3.1415 stored to a Float32Array
    for (const auto &f : m.faces) {
        V3 r;
        if (!fetch(f[0], r)) { *err_line = 0; return -1; }
        // vr_x = .x, vr_z = .y, vr_y = .z
        const double rx = r.x, ry = r.z, rz = r.y;
        xmin = js_min(xmin, rx); ymin = js_min(ymin, ry); zmin = js_min(zmin, rz);
        xmax = js_max(xmax, rx); ymax = js_max(ymax, ry); zmax = js_max(zmax, rz);
        for (size_t y = 1; y + 1 < f.size(); ++y) {
            V3 a, b;
            if (!fetch(f[y], a) || !fetch(f[y + 1], b)) { *err_line = 0; return -1; }
            const double ax = a.x, ay = a.z, az = a.y, bx = b.x, by = b.z, bz = b.y;
            xmin = js_min(ax, js_min(xmin, bx)); ymin = js_min(ay, js_min(ymin, by));
            zmin = js_min(az, js_min(zmin, bz));
            xmax = js_max(ax, js_max(xmax, bx)); ymax = js_max(ay, js_max(ymax, by));
            zmax = js_max(az, js_max(zmax, bz));
            const float t[12] = {(float)rx, (float)ry, (float)rz, pad, (float)ax, (float)ay,
                                 (float)az, pad, (float)bx, (float)by, (float)bz, pad};
            tri.insert(tri.end(), t, t + 12);
            ++nt;
        }
    }
    const double fh = zmin + .01, fs = 10000.;
    const double floor_v[6][3] = {{-fs, -fs, fh}, {fs, -fs, fh}, {-fs, fs, fh},
                                  {fs, -fs, fh},  {fs, fs, fh},  {-fs, fs, fh}};
    for (int v = 0; v < 6; ++v) {
        tri.push_back((float)floor_v[v][0]);
        tri.push_back((float)floor_v[v][1]);
        tri.push_back((float)floor_v[v][2]);
        tri.push_back(pad);
    }
    nt += 2;
    *num_tris = nt;
    bounds6[0] = xmin; bounds6[1] = ymin; bounds6[2] = zmin;
    bounds6[3] = xmax; bounds6[4] = ymax; bounds6[5] = zmax;
    if (tri_out && cap_tris >= nt) std::memcpy(tri_out, tri.data(), tri.size() * sizeof(float));
    return 0;
}

}  // extern "C"
