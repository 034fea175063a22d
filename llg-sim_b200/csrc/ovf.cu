// ovf.cu — OOMMF OVF 2.0 rectangular-mesh writers (ovf.rs:54-251).
//
// write_ovf2_rectangular_text (:54-151): MuMax-like header with {:.16e} extents
// and one "{:.10e} {:.10e} {:.10e}" line per cell, x fastest.
// write_ovf2_rectangular_binary4 (:153-251): header with {:.17e} extents, the
// check value 1234567.0f, then x, y, z of every cell as little-endian f32.
//
// The byte stream has to be the reference's for other tools to read the files
// alike; the code that produces it is this project's own.  Rust's `{:.Ne}`
// prints the correctly rounded mantissa (ties to even) and the exponent without
// sign padding ("e-9", "e0", "e5"); C's %.*e gives the same digits, and the
// exponent is rewritten.
//
// For a solver's resident state the binary4 payload is packed on the GPU
// (SoA -> AoS f32, 12 bytes per cell, the f64 -> f32 conversion rounding to
// nearest as Rust's `as f32` does) and copied to the host once; the text
// format needs the FP64 values and reads the state as llg_get_state does.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../../include/llg_b200.h"
#include "build_api.h"

namespace {

std::string rust_exp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*e", prec, v);
    char* e = std::strchr(buf, 'e');
    const long ex = std::strtol(e + 1, nullptr, 10);
    *e = '\0';
    return std::string(buf) + "e" + std::to_string(ex);
}

int fail(int code, const char* msg) {
    llg_set_error_message(msg);
    return code;
}

// create_dir_all of the parent directory (ensure_parent_dir, ovf.rs:47-52)
bool ensure_parent_dir(const char* path) {
    std::string p(path);
    const size_t slash = p.find_last_of('/');
    if (slash == std::string::npos || slash == 0) return true;
    const std::string dir = p.substr(0, slash);
    for (size_t i = 1; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            const std::string part = dir.substr(0, i);
            if (mkdir(part.c_str(), 0777) != 0 && errno != EEXIST) return false;
        }
    }
    return true;
}

const char* str_or_empty(const char* s) { return s ? s : ""; }

struct Writer {
    FILE* f = nullptr;
    bool ok = true;
    explicit Writer(const char* path) : f(std::fopen(path, "wb")) { ok = f != nullptr; }
    ~Writer() {
        if (f) std::fclose(f);
    }
    void line(const std::string& s) {
        if (!ok) return;
        ok = std::fwrite(s.data(), 1, s.size(), f) == s.size() && std::fputc('\n', f) != EOF;
    }
    void bytes(const void* p, size_t n) {
        if (ok && n) ok = std::fwrite(p, 1, n, f) == n;
    }
    bool close() {
        if (!f) return false;
        const bool good = ok && std::fflush(f) == 0;
        const bool closed = std::fclose(f) == 0;
        f = nullptr;
        return good && closed;
    }
};

std::string labels_line(const char* key, const char* const v[3]) {
    return std::string("# ") + key + ": " + str_or_empty(v[0]) + " " + str_or_empty(v[1]) + " " + str_or_empty(v[2]);
}

// Data lines "{:.10e} {:.10e} {:.10e}" formatted in parallel chunks, written in order.
void write_text_data(Writer& w, const double* m, long long n) {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const long long chunk = 16384;
    const long long nchunks = (n + chunk - 1) / chunk;
    for (long long c0 = 0; c0 < nchunks && w.ok; c0 += hw) {
        const long long c1 = std::min<long long>(nchunks, c0 + hw);
        std::vector<std::string> out(c1 - c0);
        std::vector<std::thread> th;
        for (long long c = c0; c < c1; ++c)
            th.emplace_back([&, c]() {
                std::string& s = out[c - c0];
                const long long a = c * chunk, b = std::min(n, a + chunk);
                s.reserve((size_t)(b - a) * 54);
                for (long long i = a; i < b; ++i) {
                    s += rust_exp(m[3 * i], 10);
                    s += ' ';
                    s += rust_exp(m[3 * i + 1], 10);
                    s += ' ';
                    s += rust_exp(m[3 * i + 2], 10);
                    s += '\n';
                }
            });
        for (auto& t : th) t.join();
        for (auto& s : out) w.bytes(s.data(), s.size());
    }
}

int write_text(const char* path, const llg_grid* g, const double* m, const llg_ovf_meta* meta) {
    if (!ensure_parent_dir(path)) return fail(LLG_ERR_INVALID, "cannot create the parent directory");
    Writer w(path);
    if (!w.ok) return fail(LLG_ERR_INVALID, "cannot create the OVF file");
    const long long nx = g->nx, ny = g->ny, nz = 1;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    w.line("# OOMMF OVF 2.0");
    w.line("# Segment count: 1");
    w.line("# Begin: Segment");
    w.line("# Begin: Header");
    w.line(std::string("# Title: ") + str_or_empty(meta->title));
    w.line("# meshtype: rectangular");
    w.line("# meshunit: m");
    w.line("# xmin: " + rust_exp(0.0, 16));
    w.line("# ymin: " + rust_exp(0.0, 16));
    w.line("# zmin: " + rust_exp(0.0, 16));
    w.line("# xmax: " + rust_exp((double)nx * dx, 16));
    w.line("# ymax: " + rust_exp((double)ny * dy, 16));
    w.line("# zmax: " + rust_exp((double)nz * dz, 16));
    w.line("# valuedim: 3");
    w.line(labels_line("valuelabels", meta->valuelabels));
    w.line(labels_line("valueunits", meta->valueunits));
    for (int i = 0; i < meta->n_desc; ++i) w.line(std::string("# Desc: ") + str_or_empty(meta->desc_lines[i]));
    w.line("# xbase: " + rust_exp(0.5 * dx, 16));
    w.line("# ybase: " + rust_exp(0.5 * dy, 16));
    w.line("# zbase: " + rust_exp(0.5 * dz, 16));
    w.line("# xnodes: " + std::to_string(nx));
    w.line("# ynodes: " + std::to_string(ny));
    w.line("# znodes: " + std::to_string(nz));
    w.line("# xstepsize: " + rust_exp(dx, 16));
    w.line("# ystepsize: " + rust_exp(dy, 16));
    w.line("# zstepsize: " + rust_exp(dz, 16));
    w.line("# End: Header");
    w.line("# Begin: Data Text");
    write_text_data(w, m, nx * ny);
    w.line("# End: Data Text");
    w.line("# End: Segment");
    return w.close() ? LLG_OK : fail(LLG_ERR_INVALID, "OVF write failed");
}

// payload: 3*nx*ny little-endian f32 values (x, y, z per cell)
int write_binary4(const char* path, const llg_grid* g, const float* payload, const llg_ovf_meta* meta) {
    if (!ensure_parent_dir(path)) return fail(LLG_ERR_INVALID, "cannot create the parent directory");
    Writer w(path);
    if (!w.ok) return fail(LLG_ERR_INVALID, "cannot create the OVF file");
    const long long nx = g->nx, ny = g->ny;
    const double dx = g->dx, dy = g->dy, dz = g->dz;
    w.line("# OOMMF OVF 2.0");
    w.line("# Segment count: 1");
    w.line("# Begin: Segment");
    w.line("# Begin: Header");
    w.line(std::string("# Title: ") + str_or_empty(meta->title));
    for (int i = 0; i < meta->n_desc; ++i) w.line(std::string("# Desc: ") + str_or_empty(meta->desc_lines[i]));
    w.line("# meshunit: m");
    w.line("# meshtype: rectangular");
    w.line("# xbase: " + rust_exp(0.5 * dx, 17));
    w.line("# ybase: " + rust_exp(0.5 * dy, 17));
    w.line("# zbase: " + rust_exp(0.5 * dz, 17));
    w.line("# xstepsize: " + rust_exp(dx, 17));
    w.line("# ystepsize: " + rust_exp(dy, 17));
    w.line("# zstepsize: " + rust_exp(dz, 17));
    w.line("# xnodes: " + std::to_string(nx));
    w.line("# ynodes: " + std::to_string(ny));
    w.line("# znodes: 1");
    w.line("# xmin: 0");
    w.line("# xmax: " + rust_exp((double)nx * dx, 17));
    w.line("# ymin: 0");
    w.line("# ymax: " + rust_exp((double)ny * dy, 17));
    w.line("# zmin: 0");
    w.line("# zmax: " + rust_exp(dz, 17));
    w.line("# valuedim: 3");
    w.line(labels_line("valuelabels", meta->valuelabels));
    w.line(labels_line("valueunits", meta->valueunits));
    w.line("# End: Header");
    w.line("# Begin: Data Binary 4");
    const float check = 1234567.0f;   // OVF2 binary4 check value
    w.bytes(&check, 4);                // x86-64 and the GPU are little-endian
    w.bytes(payload, sizeof(float) * 3 * (size_t)(nx * ny));
    w.line("");
    w.line("# End: Data Binary 4");
    w.line("# End: Segment");
    w.line("# End: File");
    return w.close() ? LLG_OK : fail(LLG_ERR_INVALID, "OVF write failed");
}

int check_args(const char* path, const llg_grid* g, const llg_ovf_meta* meta, int32_t format) {
    if (!path || !g || !meta) return fail(LLG_ERR_INVALID, "null argument");
    if (g->nx < 1 || g->ny < 1) return fail(LLG_ERR_INVALID, "bad grid");
    if (meta->n_desc < 0 || (meta->n_desc > 0 && !meta->desc_lines)) return fail(LLG_ERR_INVALID, "bad desc lines");
    if (format != LLG_OVF_TEXT && format != LLG_OVF_BINARY4) return fail(LLG_ERR_INVALID, "unknown OVF format");
    return LLG_OK;
}

}  // namespace

namespace llg {

int ovf2_write_packed(const char* path, const llg_grid* g, const float* payload, const llg_ovf_meta* meta) {
    int rc = check_args(path, g, meta, LLG_OVF_BINARY4);
    return rc ? rc : write_binary4(path, g, payload, meta);
}

}  // namespace llg

extern "C" {

int llg_ovf2_write(const char* path, const llg_grid* g, const double* m_aos, const llg_ovf_meta* meta,
                   int32_t format) {
    int rc = check_args(path, g, meta, format);
    if (rc) return rc;
    if (!m_aos) return fail(LLG_ERR_INVALID, "null m");
    if (format == LLG_OVF_TEXT) return write_text(path, g, m_aos, meta);
    const size_t n = (size_t)(g->nx * g->ny);
    std::vector<float> payload(3 * n);
    for (size_t i = 0; i < 3 * n; ++i) payload[i] = (float)m_aos[i];
    return write_binary4(path, g, payload.data(), meta);
}

int llg_ovf_format_exp(double v, int32_t precision, char* buf, int64_t len) {
    if (!buf || len < 1 || precision < 0 || precision > 40) return fail(LLG_ERR_INVALID, "bad argument");
    const std::string s = rust_exp(v, precision);
    if ((int64_t)s.size() + 1 > len) return fail(LLG_ERR_INVALID, "buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return LLG_OK;
}

}  // extern "C"
