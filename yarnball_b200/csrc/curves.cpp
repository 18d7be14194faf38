// curves.cpp - scene construction from curve files and JSON scene descriptions (host).
//
//   resample_cmr      Resample::resampleCMR and helpers   io/resample.h:10-187
//   yb_read_bcc       readFromBCC                          io/reader.cpp:49-97
//   yb_read_obj       readFromOBJ                          io/reader.cpp:99-156
//   yb_read_poly      readFromPoly                         io/reader.cpp:158-293
//   create_from_curves createFromCurves                    io/reader.cpp:13-47
//   yb_build_from_json buildFromJSON                       io/jsonBuilder.cpp:8-172
//   yb_glue_endpoints  Sim::glueEndpoints                  io/jsonBuilder.cpp:174-212
//
// The Catmull-Rom resampler runs in double with the reference's operation order (glm::mix(x,
// y, a) = x (1 - a) + y a; this file is built with -ffp-contract=off), so resampled curves are
// reproducible bit for bit.  Where the reference indexes outside a list (resampling fewer than
// 4 control points, end alignment of short lists, the merge blend) the library stays inside it;
// where its order is unspecified (which way a closed .poly loop is walked, in which order glued
// endpoints are applied) the library fixes one: segment order in the file, ascending endpoint
// index.  The nearest-vertex search of glueEndpoints runs on the GPU.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "yarnball_b200.h"

namespace yb {
// Nearest vertex of each endpoint (k_glue.cu).
cudaError_t glue_nearest(const float* pos4, int n, const int* endpoints, const int* lo, const int* hi, int count,
                         unsigned long long* keys);
}

namespace {

thread_local std::string g_ioError;

yb_status io_fail(yb_status st, const std::string& msg) {
    g_ioError = msg;
    return st;
}

struct P3 {
    float x, y, z;
};
struct D3 {
    double x, y, z;
};

// ---- Catmull-Rom resampling (resample.h) -------------------------------------------------

inline D3 mix3(const D3& a, const D3& b, double t) {
    return {a.x * (1.0 - t) + b.x * t, a.y * (1.0 - t) + b.y * t, a.z * (1.0 - t) + b.z * t};
}

inline double len2(const D3& a, const D3& b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return (dx * dx + dy * dy) + dz * dz;
}

// Kit::cmrSpline (Common.h:683-694): uniform Catmull-Rom as repeated linear interpolation.
D3 cmr_spline(const D3& p0, const D3& p1, const D3& p2, const D3& p3, double t) {
    const D3 a0 = mix3(p0, p1, t + 1);
    const D3 a1 = mix3(p1, p2, t + 0);
    const D3 a2 = mix3(p2, p3, t - 1);
    const D3 b0 = mix3(a0, a1, (t + 1) * 0.5);
    const D3 b1 = mix3(a1, a2, (t + 0) * 0.5);
    return mix3(b0, b1, t);
}

D3 sample_curve(const std::vector<P3>& c, double t) {
    int si = (int)std::floor(t);
    si = std::min(std::max(si, 1), (int)c.size() - 3);
    auto d = [&](int k) { return D3{c[k].x, c[k].y, c[k].z}; };
    return cmr_spline(d(si - 1), d(si), d(si + 1), d(si + 2), t - si);
}

// Parameter values spaced `tar` apart along the curve from `start` to `end` (either way).
std::vector<double> resample_coords(const std::vector<P3>& c, double start, double end, double tar) {
    std::vector<double> ts;
    const double MIN_STEP = 0.2;
    const bool up = end > start;
    const double step = up ? MIN_STEP : -MIN_STEP;
    const double r2 = tar * tar;
    double i = start;
    D3 last = sample_curve(c, i);
    ts.push_back(i);
    while (up ? i < end : i > end) {
        i += step;
        const D3 pos = sample_curve(c, i);
        double l0 = len2(pos, last);
        if (l0 > r2) {
            // overshoot: place the point at distance tar with 8 secant steps from (i, l0)
            l0 = std::sqrt(l0);
            double lo = i - step, hi = i;
            if (lo > hi) std::swap(lo, hi);
            const double t0 = i;
            i -= 0.5 * step;
            for (int k = 0; k < 8; k++) {
                const double d = std::sqrt(len2(sample_curve(c, i), last));
                i += (i - t0) * (tar - d) / (d - l0);
            }
            i = std::min(std::max(i, lo), hi);
            ts.push_back(i);
            last = sample_curve(c, i);
        }
    }
    if (ts.size() == 1) {
        ts.push_back(end);
    } else {
        // land the last point on `end`, spreading the change over the last 8 intervals
        const double d = std::sqrt(len2(sample_curve(c, ts.back()), sample_curve(c, end)));
        double dt = ts.back() - ts[ts.size() - 2];
        if (d > 0.5 * tar)
            ts.push_back(end);
        else
            ts.back() = end;
        dt -= ts.back() - ts[ts.size() - 2];
        const int N = std::min((int)ts.size(), 8);
        for (int k = 0; k < N; k++) {
            const long at = (long)ts.size() - 2 - k;
            if (at >= 0) ts[at] -= dt * (N - k) / (double)N;
        }
    }
    return ts;
}

// Forward and backward passes joined where their parameters agree best (resample.h:85-141).
std::vector<double> two_direction(const std::vector<P3>& c, double start, double end, double tar) {
    const std::vector<double> fwd = resample_coords(c, start, end, tar);
    const std::vector<double> bwd = resample_coords(c, end, start, tar);
    const int B = 8;
    if ((int)fwd.size() <= 4 * B || (int)bwd.size() <= 4 * B) return fwd;
    double minErr = std::numeric_limits<double>::infinity();
    int sx = 2 * B, sy = 2 * B;
    int j = (int)bwd.size() - 1 - B;
    for (int i = B; i < (int)fwd.size() - 8; i++) {
        const double t = fwd[i];
        while (j > 0 && bwd[j] < t) j--;
        const double t0 = bwd[j + 1];
        if (minErr > std::fabs(t - t0)) {
            minErr = std::fabs(t - t0);
            sx = i;
            sy = j + 1;
        }
        const double t1 = bwd[j];
        if (minErr > std::fabs(t1 - t)) {
            minErr = std::fabs(t1 - t);
            sx = i;
            sy = j;
        }
    }
    std::vector<double> merged(fwd.begin(), fwd.begin() + sx);
    const double mid = 0.5 * (fwd[sx] + bwd[sy]);
    merged.push_back(mid);
    for (int k = sy - 1; k >= 0; k--) merged.push_back(bwd[k]);
    double dt = fwd[sx] - mid;
    for (int k = 0; k < B; k++) {
        const int at = sx - k - 1;
        if (at >= 0 && at < (int)merged.size()) merged[at] -= dt * (B - k) / (1. + B);
    }
    dt = bwd[sy] - mid;
    for (int k = 0; k < B; k++) {
        const int at = sx + k + 1;
        if (at >= 0 && at < (int)merged.size()) merged[at] -= dt * (B - k) / (1. + B);
    }
    return merged;
}

std::vector<P3> resample_cmr(const std::vector<P3>& c, double start, double end, double tar) {
    if (c.size() < 4) return c;  // a Catmull-Rom segment needs 4 control points
    auto max_err = [&](const std::vector<double>& ts, double target, double* total) {
        double err = 0, sum = 0;
        D3 last = sample_curve(c, ts[0]);
        for (size_t i = 1; i < ts.size(); i++) {
            const D3 pos = sample_curve(c, ts[i]);
            const double l = std::sqrt(len2(pos, last));
            err = std::max(err, std::fabs(l - target));
            sum += l;
            last = pos;
        }
        if (total) *total = sum;
        return err;
    };
    // Two passes: the first gives the mean spacing, the second resamples at that spacing;
    // the one with the smaller worst deviation wins (resample.h:143-187).
    const std::vector<double> ts0 = two_direction(c, start, end, tar);
    double total = 0;
    const double err0 = max_err(ts0, tar, &total);
    const double avg = total / (double)(ts0.size() - 1);
    const std::vector<double> ts1 = two_direction(c, start, end, avg);
    const double err1 = max_err(ts1, avg, nullptr);
    const std::vector<double>& ts = err0 < err1 ? ts0 : ts1;
    std::vector<P3> out(ts.size());
    for (size_t i = 0; i < ts.size(); i++) {
        const D3 p = sample_curve(c, ts[i]);
        out[i] = {(float)p.x, (float)p.y, (float)p.z};
    }
    return out;
}

// vec3(T * vec4(p, 1)) for a column-major 4x4 matrix, in glm's order of operations.
P3 transform_point(const float* T, const P3& p) {
    float r[3];
    for (int i = 0; i < 3; i++) {
        const float a = T[0 + i] * p.x + T[4 + i] * p.y;
        const float b = T[8 + i] * p.z + T[12 + i] * 1.0f;
        r[i] = a + b;
    }
    return {r[0], r[1], r[2]};
}

// ---- createFromCurves -------------------------------------------------------------------

yb_status create_from_curves(const std::vector<std::vector<P3>>& curves, const std::vector<bool>& closed,
                             yb_sim** out) {
    size_t total = 0;
    for (const auto& c : curves) total += c.size();
    if (total > (size_t)INT32_MAX) return io_fail(YB_ERR_INVALID_ARGUMENT, "too many vertices");
    yb_sim* S = nullptr;
    yb_status st = yb_create((int32_t)total, &S);
    if (st != YB_OK) return io_fail(st, yb_status_string(st));
    yb_vertex* v = nullptr;
    float *q = nullptr, *qr = nullptr, *vel = nullptr;
    yb_host_arrays(S, &v, &q, &qr, &vel);
    int off = 0;
    for (size_t i = 0; i < curves.size(); i++) {
        const auto& c = curves[i];
        for (size_t j = 0; j < c.size(); j++) {
            v[off + j].pos[0] = c[j].x;
            v[off + j].pos[1] = c[j].y;
            v[off + j].pos[2] = c[j].z;
        }
        v[off + c.size() - 1].flags = 0;
        if (closed[i]) {
            v[off].connectionIndex = off + (int)c.size() - 1;
            v[off + c.size() - 1].connectionIndex = off;
        }
        off += (int)c.size();
    }
    *out = S;
    return YB_OK;
}

// ---- readers ----------------------------------------------------------------------------

const float* identity_or(const float* T, float* tmp) {
    if (T) return T;
    for (int i = 0; i < 16; i++) tmp[i] = (i % 5 == 0) ? 1.f : 0.f;
    return tmp;
}

yb_status read_bcc(const char* path, float target, const float* T, bool breakUp, bool allowResample, yb_sim** out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(YB_ERR_IO, "Could not open file");
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, &std::fclose);
    unsigned char h[64];
    if (std::fread(h, 1, 64, f) != 64) return io_fail(YB_ERR_FORMAT, "Unsupported BCC file");
    if (h[0] != 'B' || h[1] != 'C' || h[2] != 'C' || h[3] != 0x44) return io_fail(YB_ERR_FORMAT, "Unsupported BCC file");
    const bool polyline = h[4] == 'P' && h[5] == 'L';
    if (!polyline && (h[4] != 'C' || h[5] != '0'))
        return io_fail(YB_ERR_FORMAT, "Not polyline or uniform CMR spline");
    if (h[6] != 3) return io_fail(YB_ERR_FORMAT, "Only curves in 3D are supported");
    uint64_t curveCount = 0;
    std::memcpy(&curveCount, h + 8, 8);
    std::vector<std::vector<P3>> curves;
    std::vector<bool> closed;
    for (uint64_t i = 0; i < curveCount; i++) {
        int32_t m = 0;
        if (std::fread(&m, 4, 1, f) != 1) return io_fail(YB_ERR_FORMAT, "truncated BCC file");
        const bool isClosed = m < 0;
        if (m == INT32_MIN) return io_fail(YB_ERR_FORMAT, "truncated BCC file");
        m = m < 0 ? -m : m;
        std::vector<P3> pts(m);
        if (m && std::fread(pts.data(), 12, (size_t)m, f) != (size_t)m)
            return io_fail(YB_ERR_FORMAT, "truncated BCC file");
        for (auto& p : pts) p = transform_point(T, p);
        if (allowResample && !polyline) pts = resample_cmr(pts, 1, (double)pts.size() - 2, target);
        if (m < 3) continue;
        closed.push_back(isClosed && !breakUp);
        curves.push_back(std::move(pts));
    }
    return create_from_curves(curves, closed, out);
}

yb_status read_obj(const char* path, float target, const float* T, bool breakUp, bool allowResample, yb_sim** out) {
    std::ifstream file(path);
    if (!file.is_open()) return io_fail(YB_ERR_IO, "Could not open file.");
    std::vector<P3> vertices;
    std::vector<std::vector<int>> lines;
    std::string line;
    while (std::getline(file, line)) {
        std::istringstream iss(line);
        std::string prefix;
        iss >> prefix;
        if (prefix == "v") {
            P3 p{0, 0, 0};
            iss >> p.x >> p.y >> p.z;
            vertices.push_back(transform_point(T, p));
        } else if (prefix == "l") {
            std::vector<int> idx;
            int k;
            while (iss >> k) idx.push_back(k);
            if (!idx.empty()) lines.push_back(std::move(idx));
        }
    }
    std::vector<std::vector<P3>> curves;
    std::vector<bool> closed;
    for (const auto& idx : lines) {
        std::vector<P3> c;
        c.reserve(idx.size());
        bool isClosed = idx.front() == idx.back();
        for (int k : idx) {
            if (k < 1 || k > (int)vertices.size()) return io_fail(YB_ERR_FORMAT, "OBJ line index out of range");
            c.push_back(vertices[k - 1]);
        }
        if (breakUp && isClosed) {
            c.pop_back();
            isClosed = false;
        }
        if (allowResample) c = resample_cmr(c, 1, (double)c.size() - 2, target);
        if (c.size() < 4) continue;
        curves.push_back(std::move(c));
        closed.push_back(isClosed);
    }
    return create_from_curves(curves, closed, out);
}

yb_status read_poly(const char* path, float target, const float* T, bool breakUp, bool allowResample, yb_sim** out) {
    std::ifstream file(path);
    if (!file.is_open()) return io_fail(YB_ERR_IO, "Could not open file.");
    std::string line;
    bool isPoint = true;
    std::vector<P3> points;
    std::vector<std::pair<int, int>> segs;
    while (std::getline(file, line)) {
        std::istringstream iss(line);
        if (line == "POINTS") {
            isPoint = true;
            continue;
        } else if (line == "POLYS") {
            isPoint = false;
            continue;
        } else if (line == "END") {
            break;
        }
        int id;
        char colon;
        if (isPoint) {
            float x, y, z;
            if (!(iss >> id >> colon >> x >> y >> z) || colon != ':')
                return io_fail(YB_ERR_FORMAT, "Error parsing .poly. Point parse error.");
            points.push_back(transform_point(T, P3{x, y, z}));
            if (id != (int)points.size()) return io_fail(YB_ERR_FORMAT, "Error parsing .poly. Point id mismatch.");
        } else {
            int a, b;
            if (!(iss >> id >> colon >> a >> b) || colon != ':')
                return io_fail(YB_ERR_FORMAT, "Error parsing .poly. Segment parse error.");
            if (a < 1 || b < 1 || a > (int)points.size() || b > (int)points.size())
                return io_fail(YB_ERR_FORMAT, "Error parsing .poly. Segment index out of range.");
            segs.push_back({a - 1, b - 1});
        }
    }
    // Neighbours of each point in segment order.
    const int np = (int)points.size();
    std::vector<std::vector<int>> nbr(np);
    for (const auto& s : segs) {
        nbr[s.first].push_back(s.second);
        nbr[s.second].push_back(s.first);
    }
    std::vector<std::vector<P3>> curves;
    std::vector<bool> closed;
    std::vector<char> visited(np, 0);
    // open curves: walk from every end point
    for (int i = 0; i < np; i++) {
        if (visited[i]) continue;
        if (nbr[i].size() > 2) return io_fail(YB_ERR_FORMAT, "Graphs not allowed.");
        if (nbr[i].size() > 1) continue;
        std::vector<P3> c;
        int cur = i;
        while (!visited[cur]) {
            visited[cur] = 1;
            c.push_back(points[cur]);
            if (nbr[cur].empty()) break;
            for (int x : nbr[cur])
                if (!visited[x]) {
                    cur = x;
                    break;
                }
        }
        if (c.size() < 4) continue;
        // as in the reference, open curves are resampled even when resampling is off
        c = resample_cmr(c, 1, (double)c.size() - 2, target);
        curves.push_back(std::move(c));
        closed.push_back(false);
    }
    // closed curves: every remaining point has exactly two neighbours
    for (int i = 0; i < np; i++) {
        if (visited[i]) continue;
        if (nbr[i].size() != 2) return io_fail(YB_ERR_FORMAT, "Graphs not allowed.");
        std::vector<P3> c;
        int cur = i;
        while (true) {
            visited[cur] = 1;
            c.push_back(points[cur]);
            bool found = false, isEnd = false;
            for (int x : nbr[cur]) {
                if (!visited[x]) {
                    cur = x;
                    found = true;
                    break;
                }
                if (x == i) isEnd = true;
            }
            if (!found) {
                if (!isEnd) return io_fail(YB_ERR_FORMAT, "Closed curve not closed.");
                break;
            }
        }
        if (allowResample) c = resample_cmr(c, 1, (double)c.size() - 2, target);
        if (c.size() < 4) continue;
        curves.push_back(std::move(c));
        closed.push_back(!breakUp);
    }
    return create_from_curves(curves, closed, out);
}

// ---- a small JSON reader (the subset jsoncpp's default reader accepts in scene files:
// comments and trailing commas allowed) --------------------------------------------------

struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal& operator[](const char* key) const {
        static const JVal null;
        if (kind != Obj) return null;
        for (const auto& kv : obj)
            if (kv.first == key) return kv.second;
        return null;
    }
    const JVal& operator[](int i) const {
        static const JVal null;
        if (kind != Arr || i < 0 || (size_t)i >= arr.size()) return null;
        return arr[i];
    }
    bool isNull() const { return kind == Null; }
    size_t size() const { return kind == Arr ? arr.size() : (kind == Obj ? obj.size() : 0); }
    double asDouble() const { return kind == Num ? num : (kind == Bool ? (b ? 1.0 : 0.0) : 0.0); }
    float asFloat() const { return (float)asDouble(); }
    int asInt() const { return kind == Num ? (int)num : (kind == Bool ? (b ? 1 : 0) : 0); }
    bool asBool() const { return kind == Bool ? b : (kind == Num ? num != 0 : false); }
};

struct JParser {
    const std::string& s;
    size_t p = 0;
    std::string err;
    explicit JParser(const std::string& text) : s(text) {}

    void skip() {
        while (p < s.size()) {
            const char c = s[p];
            if (std::isspace((unsigned char)c)) {
                p++;
            } else if (c == '/' && p + 1 < s.size() && s[p + 1] == '/') {
                while (p < s.size() && s[p] != '\n') p++;
            } else if (c == '/' && p + 1 < s.size() && s[p + 1] == '*') {
                const size_t e = s.find("*/", p + 2);
                p = e == std::string::npos ? s.size() : e + 2;
            } else {
                break;
            }
        }
    }
    bool fail(const char* m) {
        if (err.empty()) err = std::string(m) + " at offset " + std::to_string(p);
        return false;
    }
    bool parse_string(std::string& out) {
        p++;  // opening quote
        while (p < s.size() && s[p] != '"') {
            if (s[p] == '\\' && p + 1 < s.size()) {
                const char e = s[p + 1];
                out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e);
                p += 2;
            } else {
                out.push_back(s[p++]);
            }
        }
        if (p >= s.size()) return fail("unterminated string");
        p++;
        return true;
    }
    bool parse(JVal& v, int depth = 0) {
        if (depth > 64) return fail("nesting too deep");
        skip();
        if (p >= s.size()) return fail("unexpected end");
        const char c = s[p];
        if (c == '{') {
            v.kind = JVal::Obj;
            p++;
            while (true) {
                skip();
                if (p < s.size() && s[p] == '}') { p++; return true; }
                if (p >= s.size() || s[p] != '"') return fail("expected a key");
                std::string key;
                if (!parse_string(key)) return false;
                skip();
                if (p >= s.size() || s[p] != ':') return fail("expected ':'");
                p++;
                JVal child;
                if (!parse(child, depth + 1)) return false;
                v.obj.push_back({key, std::move(child)});
                skip();
                if (p < s.size() && s[p] == ',') { p++; continue; }
                if (p < s.size() && s[p] == '}') { p++; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JVal::Arr;
            p++;
            while (true) {
                skip();
                if (p < s.size() && s[p] == ']') { p++; return true; }
                JVal child;
                if (!parse(child, depth + 1)) return false;
                v.arr.push_back(std::move(child));
                skip();
                if (p < s.size() && s[p] == ',') { p++; continue; }
                if (p < s.size() && s[p] == ']') { p++; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JVal::Str;
            return parse_string(v.str);
        }
        if (s.compare(p, 4, "true") == 0) { v.kind = JVal::Bool; v.b = true; p += 4; return true; }
        if (s.compare(p, 5, "false") == 0) { v.kind = JVal::Bool; v.b = false; p += 5; return true; }
        if (s.compare(p, 4, "null") == 0) { v.kind = JVal::Null; p += 4; return true; }
        const char* start = s.c_str() + p;
        char* end = nullptr;
        const double x = std::strtod(start, &end);
        if (end == start) return fail("unexpected character");
        v.kind = JVal::Num;
        v.num = x;
        p += (size_t)(end - start);
        return true;
    }
};

bool ends_with(const std::string& s, const char* suf) {
    const size_t n = std::strlen(suf);
    return s.size() > n && s.compare(s.size() - n, n, suf) == 0;
}

}  // namespace

namespace yb {
void set_io_error(const std::string& msg) { g_ioError = msg; }
}  // namespace yb

// =========================================================================================
extern "C" {

const char* yb_last_io_error(void) { return g_ioError.c_str(); }

yb_status yb_resample_cmr(const float* points, int32_t count, double start, double end, double targetSegLen,
                          float* out, int32_t capacity, int32_t* outCount) {
    if (!points || count < 0 || !outCount || !(targetSegLen > 0)) return YB_ERR_INVALID_ARGUMENT;
    std::vector<P3> c(count);
    std::memcpy(c.data(), points, sizeof(P3) * (size_t)count);
    const std::vector<P3> r = resample_cmr(c, start, end, targetSegLen);
    *outCount = (int32_t)r.size();
    if (!out || capacity < (int32_t)r.size()) return out ? YB_ERR_SCRATCH_TOO_SMALL : YB_OK;
    std::memcpy(out, r.data(), sizeof(P3) * r.size());
    return YB_OK;
}

yb_status yb_read_bcc(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                      int32_t allowResample, yb_sim** out) {
    if (!path || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    float tmp[16];
    return read_bcc(path, targetSegLen, identity_or(transform, tmp), breakUpClosedCurves != 0, allowResample != 0, out);
}

yb_status yb_read_obj(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                      int32_t allowResample, yb_sim** out) {
    if (!path || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    float tmp[16];
    return read_obj(path, targetSegLen, identity_or(transform, tmp), breakUpClosedCurves != 0, allowResample != 0, out);
}

yb_status yb_read_poly(const char* path, float targetSegLen, const float transform[16], int32_t breakUpClosedCurves,
                       int32_t allowResample, yb_sim** out) {
    if (!path || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    float tmp[16];
    return read_poly(path, targetSegLen, identity_or(transform, tmp), breakUpClosedCurves != 0, allowResample != 0,
                     out);
}

yb_status yb_glue_endpoints(yb_sim* S, float searchRadius) {
    if (!S) return YB_ERR_INVALID_ARGUMENT;
    yb_vertex* v = nullptr;
    float *q = nullptr, *qr = nullptr, *vel = nullptr;
    yb_host_arrays(S, &v, &q, &qr, &vel);
    int32_t n = 0, numScenes = 0, prec = 0;
    yb_info(S, &n, &numScenes, &prec);
    // Endpoints (exactly one of hasPrev / hasNext, jsonBuilder.cpp:177-183) and the vertex
    // range searched for each: its own scene.
    std::vector<int> ends, lo, hi;
    for (int32_t s = 0; s < numScenes; s++) {
        int32_t first = 0, count = 0;
        yb_scene_range(S, s, &first, &count);
        for (int i = first; i < first + count; i++) {
            const bool hasPrev = i > first && (v[i - 1].flags & YB_HAS_NEXT) != 0;
            const bool hasNext = (v[i].flags & YB_HAS_NEXT) != 0;
            if (hasPrev != hasNext) {
                ends.push_back(i);
                lo.push_back(first);
                hi.push_back(first + count);
            }
        }
    }
    if (ends.empty()) return YB_OK;
    std::vector<float> pos4(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
        pos4[4 * i] = v[i].pos[0];
        pos4[4 * i + 1] = v[i].pos[1];
        pos4[4 * i + 2] = v[i].pos[2];
        pos4[4 * i + 3] = 0.f;
    }
    std::vector<unsigned long long> keys(ends.size());
    const cudaError_t e =
        yb::glue_nearest(pos4.data(), n, ends.data(), lo.data(), hi.data(), (int)ends.size(), keys.data());
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? YB_ERR_OUT_OF_MEMORY : YB_ERR_CUDA;
    // Apply in ascending endpoint order; both ends must still be free (jsonBuilder.cpp:201-208).
    for (size_t k = 0; k < ends.size(); k++) {
        if (keys[k] == ~0ull) continue;
        uint32_t bits = (uint32_t)(keys[k] >> 32);
        float minDist;
        std::memcpy(&minDist, &bits, 4);
        const int j = (int)(keys[k] & 0xffffffffu);
        const int i = ends[k];
        if (!(minDist <= searchRadius)) continue;
        if (v[j].connectionIndex < 0 && v[i].connectionIndex < 0) {
            v[j].connectionIndex = i;
            v[i].connectionIndex = j;
            for (int a = 0; a < 3; a++) v[j].pos[a] = v[i].pos[a] = 0.5f * (v[i].pos[a] + v[j].pos[a]);
        }
    }
    return YB_OK;
}

yb_status yb_build_from_json(const char* path, yb_sim** out) {
    if (!path || !out) return YB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::ifstream file(path, std::ifstream::binary);
    if (!file.is_open()) return io_fail(YB_ERR_IO, "Error opening file");
    std::stringstream ss;
    ss << file.rdbuf();
    const std::string text = ss.str();
    JParser jp(text);
    JVal root;
    if (!jp.parse(root)) return io_fail(YB_ERR_FORMAT, "Error parsing the JSON file: " + jp.err);

    const std::string dataPath = root["curveFile"].str;
    float T[16] = {0};
    T[0] = T[5] = T[10] = 0.01f;  // centimetres to metres
    T[15] = 1.f;
    if (!root["transform"].isNull()) {
        const JVal& t = root["transform"];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 4; j++) T[4 * j + i] = t[i][j].asFloat();
    }
    const bool resample = !root["resampleLength"].isNull();
    const float segLen = root["resampleLength"].asFloat();
    const bool breakUp = root["breakUpClosedCurves"].isNull() ? false : root["breakUpClosedCurves"].asBool();

    yb_sim* S = nullptr;
    yb_status st;
    if (ends_with(dataPath, ".poly"))
        st = read_poly(dataPath.c_str(), segLen, T, breakUp, resample, &S);
    else if (ends_with(dataPath, ".obj"))
        st = read_obj(dataPath.c_str(), segLen, T, breakUp, resample, &S);
    else
        st = read_bcc(dataPath.c_str(), segLen, T, breakUp, resample, &S);
    if (st != YB_OK) return st;
    std::unique_ptr<yb_sim, void (*)(yb_sim*)> guard(S, &yb_destroy);

    yb_meta m;
    yb_get_meta(S, 0, &m);
    float maxH = 0;
    yb_get_max_h(S, &maxH);
    if (!root["curveRadius"].isNull()) {
        const float r = root["curveRadius"].asFloat();
        const float ratio = 0.05f;
        m.radius = ratio * r;
        m.barrierThickness = 2 * (1 - ratio) * r;
    }
    const JVal& sim = root["simulation"];
    double density = 1., kStretch = 5e5, kBend = 1e-1;
    if (!sim.isNull()) {
        if (!sim["density"].isNull()) density = sim["density"].asFloat();
        if (!sim["frictionCoeff"].isNull()) m.frictionCoeff = sim["frictionCoeff"].asFloat();
        if (!sim["kStretch"].isNull()) kStretch = sim["kStretch"].asFloat();
        if (!sim["kBend"].isNull()) kBend = sim["kBend"].asFloat();
        if (!sim["kCollision"].isNull()) m.kCollision = sim["kCollision"].asFloat();
        if (!sim["kFriction"].isNull()) m.kFriction = sim["kFriction"].asFloat();
        if (!sim["damping"].isNull()) m.damping = sim["damping"].asFloat();
        if (!sim["gravity"].isNull()) {
            const JVal& g = sim["gravity"];
            m.gravity[0] = g[0].asFloat();
            m.gravity[1] = g[1].asFloat();
            m.gravity[2] = g[2].asFloat();
        }
        if (!sim["drag"].isNull()) m.drag = sim["drag"].asFloat();
        if (!sim["maxTimeStep"].isNull()) maxH = sim["maxTimeStep"].asFloat();
        if (!sim["numIterations"].isNull()) m.numItr = sim["numIterations"].asInt();
        if (!sim["detectionPeriod"].isNull()) m.detectionPeriod = sim["detectionPeriod"].asInt();
        if (!sim["detectionScaler"].isNull()) m.detectionScaler = sim["detectionScaler"].asFloat();
        if (!sim["stepLimit"].isNull()) m.useStepSizeLimit = sim["stepLimit"].asBool() ? 1 : 0;
        if (!sim["velStepLimit"].isNull()) m.useVelocityRadius = sim["velStepLimit"].asBool() ? 1 : 0;
        if (!sim["bvhRebuildPeriod"].isNull()) m.bvhRebuildPeriod = sim["bvhRebuildPeriod"].asFloat();
    }
    if ((st = yb_set_meta(S, 0, &m)) != YB_OK) return st;
    if ((st = yb_set_max_h(S, maxH)) != YB_OK) return st;
    if ((st = yb_configure(S, (float)density)) != YB_OK) return st;
    if ((st = yb_set_kstretch(S, -1, (float)kStretch)) != YB_OK) return st;
    if ((st = yb_set_kbend(S, -1, (float)kBend)) != YB_OK) return st;

    if (!root["glueEndpoints"].isNull()) {
        const float radius = root["glueEndpoints"].asFloat();
        if (radius >= 0 && (st = yb_glue_endpoints(S, radius)) != YB_OK) return st;
    }
    yb_vertex* v = nullptr;
    float *q = nullptr, *qr = nullptr, *vel = nullptr;
    yb_host_arrays(S, &v, &q, &qr, &vel);
    yb_get_meta(S, 0, &m);
    const int n = m.numVerts;
    const JVal& borders = root["fixBorders"];
    if (borders.kind == JVal::Arr && borders.size() == 6) {
        float bd[6];
        for (int i = 0; i < 6; i++) bd[i] = borders[i].asFloat();
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int i = 0; i < n; i++)
            for (int a = 0; a < 3; a++) {
                mn[a] = v[i].pos[a] < mn[a] ? v[i].pos[a] : mn[a];
                mx[a] = mx[a] < v[i].pos[a] ? v[i].pos[a] : mx[a];
            }
        const float pad = 0.01f * m.radius;
        for (int a = 0; a < 3; a++) {
            mn[a] -= pad;
            mx[a] += pad;
        }
        mx[0] -= bd[0]; mn[0] += bd[1];
        mx[1] -= bd[2]; mn[1] += bd[3];
        mx[2] -= bd[4]; mn[2] += bd[5];
        for (int i = 0; i < n; i++) {
            bool inside = true;
            for (int a = 0; a < 3; a++) inside = inside && mn[a] <= v[i].pos[a] && v[i].pos[a] <= mx[a];
            if (!inside) v[i].invMass = 0;
        }
    }
    const JVal& fix = root["fixVertex"];
    if (fix.kind == JVal::Arr) {
        for (int i = 0; i < (int)fix.size(); i++) {
            const JVal& e = fix[i];
            if (e.kind == JVal::Arr) {
                if (e.size() < 3) continue;
                const float p[3] = {e[0].asFloat(), e[1].asFloat(), e[2].asFloat()};
                auto dist2 = [&](int j) {
                    const float dx = v[j].pos[0] - p[0], dy = v[j].pos[1] - p[1], dz = v[j].pos[2] - p[2];
                    return (dx * dx + dy * dy) + dz * dz;
                };
                if (e.size() >= 4) {  // pin everything inside the sphere
                    float r2 = e[3].asFloat();
                    r2 *= r2;
                    for (int j = 0; j < n; j++)
                        if (dist2(j) < r2) v[j].invMass = 0;
                } else {  // pin the closest vertex
                    float best = INFINITY;
                    int closest = -1;
                    for (int j = 0; j < n; j++) {
                        const float d2 = dist2(j);
                        if (d2 < best) {
                            best = d2;
                            closest = j;
                        }
                    }
                    if (closest >= 0) v[closest].invMass = 0;
                }
            } else {
                const int j = e.asInt();
                if (j < 0 || j >= n) return io_fail(YB_ERR_FORMAT, "fixVertex index out of range");
                v[j].invMass = 0;
            }
        }
    }
    if ((st = yb_upload(S)) != YB_OK) return st;
    *out = guard.release();
    return YB_OK;
}

}  // extern "C"
