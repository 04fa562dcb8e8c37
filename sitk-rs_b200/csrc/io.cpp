// MetaImage reader (io/meta_image.rs read / parse_header), for 3-D scalar volumes, so
// the metric can be fed from files as well as from synthetic data.
//
// The header is `Key = Value` lines up to and including ElementDataFile (MetaIO's
// terminateRead field); a repeated key keeps its last value. Aliases resolve in
// MetaIO's fixed order, not the file's: origin Offset, then Position, then Origin;
// direction Orientation, then Rotation, then TransformMatrix (Position, Origin,
// Orientation and Rotation only at FileFormatVersion 0, the default); byte order
// ElementByteOrderMSB, then BinaryDataByteOrderMSB. A boolean is true when its first
// character is T, t or 1. ElementDataFile LOCAL (any case) puts the pixels after the
// header; any other name is a file beside the header. CompressedData marks a zlib (or
// gzip) stream; a LOCAL compressed header must carry CompressedDataSize (without it
// the reference refuses, since MetaIO would inflate the header text). Not read here,
// and refused by name: other dimensions than 3, more than one channel, LIST slice
// files.
#include <zlib.h>

#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"

namespace mi {
namespace {

struct MetaHeader {
    int64_t size[3];
    double spacing[3], origin[3], direction[9];
    mi_dtype dtype;
    int esize;
    bool big_endian = false, compressed = false, has_csize = false;
    uint64_t csize = 0;
    std::string data_file;
    size_t data_offset = 0;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

bool met_bool(const std::string& v) { return !v.empty() && (v[0] == 'T' || v[0] == 't' || v[0] == '1'); }

bool parse_doubles(const std::string& v, std::vector<double>& out) {
    out.clear();
    std::istringstream is(v);
    std::string tok;
    while (is >> tok) {
        char* end = nullptr;
        const double d = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str() || *end != '\0') return false;
        out.push_back(d);
    }
    return true;
}

const std::string* last(const std::vector<std::pair<std::string, std::string>>& f, const char* key) {
    for (auto it = f.rbegin(); it != f.rend(); ++it)
        if (it->first == key) return &it->second;
    return nullptr;
}

// io/meta_image.rs:214-228
bool element_type(const std::string& s, mi_dtype& t, int& size) {
    struct E {
        const char* name;
        mi_dtype t;
        int size;
    };
    static const E table[] = {{"MET_UCHAR", MI_U8, 1},       {"MET_CHAR", MI_I8, 1},     {"MET_USHORT", MI_U16, 2},
                              {"MET_SHORT", MI_I16, 2},      {"MET_UINT", MI_U32, 4},    {"MET_INT", MI_I32, 4},
                              {"MET_ULONG_LONG", MI_U64, 8}, {"MET_ULONG", MI_U64, 8},   {"MET_LONG_LONG", MI_I64, 8},
                              {"MET_LONG", MI_I64, 8},       {"MET_FLOAT", MI_F32, 4},   {"MET_DOUBLE", MI_F64, 8}};
    for (const E& e : table)
        if (s == e.name) {
            t = e.t;
            size = e.size;
            return true;
        }
    return false;
}

// scan_fields + parse_header (io/meta_image.rs:448-560)
bool parse_header(const std::string& bytes, MetaHeader& h, std::string& why) {
    std::vector<std::pair<std::string, std::string>> fields;
    size_t pos = 0;
    for (;;) {
        const size_t nl = bytes.find('\n', pos);
        if (nl == std::string::npos) {
            why = "no ElementDataFile line";
            return false;
        }
        std::string line = bytes.substr(pos, nl - pos);
        while (!line.empty() && line.back() == '\r') line.pop_back();
        const size_t eq = line.find('=');
        if (eq == std::string::npos) {
            why = "header line without '='";
            return false;
        }
        const std::string key = trim(line.substr(0, eq)), value = trim(line.substr(eq + 1));
        fields.emplace_back(key, value);
        pos = nl + 1;
        if (key == "ElementDataFile") break;
    }
    h.data_offset = pos;
    const std::string* v = last(fields, "NDims");
    if (!v || std::atoi(v->c_str()) != 3 || trim(*v) != std::to_string(std::atoi(v->c_str()))) {
        why = v ? "only 3-D images are read (NDims = " + *v + ")" : "missing NDims";
        return false;
    }
    std::vector<double> list;
    v = last(fields, "DimSize");
    if (!v || !parse_doubles(*v, list) || list.size() != 3) {
        why = "bad DimSize";
        return false;
    }
    for (int d = 0; d < 3; ++d) {
        if (list[d] < 1 || list[d] != (double)(int64_t)list[d]) {
            why = "bad DimSize";
            return false;
        }
        h.size[d] = (int64_t)list[d];
    }
    v = last(fields, "ElementType");
    if (!v || !element_type(*v, h.dtype, h.esize)) {
        why = v ? "unsupported ElementType " + *v : "missing ElementType";
        return false;
    }
    for (int d = 0; d < 3; ++d) h.spacing[d] = 1.0;
    if ((v = last(fields, "ElementSpacing"))) {
        if (!parse_doubles(*v, list) || list.size() != 3) {
            why = "bad ElementSpacing";
            return false;
        }
        for (int d = 0; d < 3; ++d) h.spacing[d] = list[d];
    }
    const std::string* ffv = last(fields, "FileFormatVersion");
    const bool legacy = !ffv || trim(*ffv) == "0";
    for (int d = 0; d < 3; ++d) h.origin[d] = 0.0;
    for (const char* key : {"Offset", "Position", "Origin"}) {
        if (!(legacy || std::strcmp(key, "Offset") == 0)) continue;
        if ((v = last(fields, key))) {
            if (!parse_doubles(*v, list) || list.size() != 3) {
                why = std::string("bad ") + key;
                return false;
            }
            for (int d = 0; d < 3; ++d) h.origin[d] = list[d];
        }
    }
    for (int i = 0; i < 9; ++i) h.direction[i] = (i % 4 == 0) ? 1.0 : 0.0;
    for (const char* key : {"Orientation", "Rotation", "TransformMatrix"}) {
        if (!(legacy || std::strcmp(key, "TransformMatrix") == 0)) continue;
        if ((v = last(fields, key))) {
            if (!parse_doubles(*v, list) || list.size() != 9) {
                why = std::string("bad ") + key;
                return false;
            }
            for (int i = 0; i < 9; ++i) h.direction[i] = list[i];
        }
    }
    if ((v = last(fields, "ElementNumberOfChannels")) && trim(*v) != "1") {
        why = "vector images (ElementNumberOfChannels = " + *v + ") are not read";
        return false;
    }
    for (const char* key : {"ElementByteOrderMSB", "BinaryDataByteOrderMSB"})
        if ((v = last(fields, key))) h.big_endian = met_bool(*v);
    if ((v = last(fields, "CompressedData"))) h.compressed = met_bool(*v);
    if ((v = last(fields, "CompressedDataSize"))) {
        char* end = nullptr;
        const unsigned long long c = std::strtoull(trim(*v).c_str(), &end, 10);
        if (end && *end == '\0' && !trim(*v).empty()) {
            h.has_csize = true;
            h.csize = c;
        }
    }
    h.data_file = *last(fields, "ElementDataFile");
    return true;
}

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

// inflate a zlib or gzip stream (inflateInit2 with 47, as MetaIO) into exactly `want` bytes
bool inflate_exact(const char* src, size_t n, size_t want, std::string& out) {
    out.assign(want, '\0');
    z_stream s;
    std::memset(&s, 0, sizeof(s));
    if (inflateInit2(&s, 47) != Z_OK) return false;
    s.next_in = reinterpret_cast<Bytef*>(const_cast<char*>(src));
    s.avail_in = (uInt)n;
    s.next_out = reinterpret_cast<Bytef*>(&out[0]);
    s.avail_out = (uInt)want;
    const int r = inflate(&s, Z_FINISH);
    const size_t got = want - s.avail_out;
    inflateEnd(&s);
    return (r == Z_STREAM_END || r == Z_OK || r == Z_BUF_ERROR) && got == want;
}

// The pixels of a header as host bytes of its element type, little-endian.
mi_status read_pixels(mi_context* ctx, const std::string& path, MetaHeader& h, std::string& data) {
    std::string bytes;
    if (!read_file(path, bytes)) return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "cannot read " + path)
                                            : MI_ERR_INVALID_ARGUMENT;
    std::string why;
    if (!parse_header(bytes, h, why))
        return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "MetaImage header: " + why) : MI_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)(h.size[0] * h.size[1] * h.size[2]);
    const size_t want = n * (size_t)h.esize;
    std::string lower = h.data_file;
    for (auto& c : lower) c = (char)std::tolower((unsigned char)c);
    std::string raw;
    if (lower == "local") {
        if (h.compressed && !h.has_csize)
            return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT,
                                   "CompressedData = True with no CompressedDataSize in a LOCAL header")
                       : MI_ERR_INVALID_ARGUMENT;
        raw = bytes.substr(h.data_offset);
    } else if (h.data_file.compare(0, 4, "LIST") == 0) {
        return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "ElementDataFile = LIST is not read")
                   : MI_ERR_INVALID_ARGUMENT;
    } else {
        std::string file = h.data_file;
        if (file.empty() || file[0] != '/') {
            const size_t slash = path.find_last_of('/');
            file = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/" + file;
        }
        if (!read_file(file, raw))
            return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "cannot read " + file) : MI_ERR_INVALID_ARGUMENT;
    }
    if (h.compressed) {
        const size_t csize = h.has_csize ? (size_t)h.csize : raw.size();
        if (csize > raw.size() || !inflate_exact(raw.data(), csize, want, data))
            return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "compressed pixel data is truncated or corrupt")
                       : MI_ERR_INVALID_ARGUMENT;
    } else {
        if (raw.size() < want)
            return ctx ? set_error(ctx, MI_ERR_INVALID_ARGUMENT, "pixel data is truncated") : MI_ERR_INVALID_ARGUMENT;
        data = raw.substr(0, want);
    }
    if (h.big_endian && h.esize > 1)
        for (size_t i = 0; i < n; ++i) {
            char* p = &data[i * (size_t)h.esize];
            for (int a = 0, b = h.esize - 1; a < b; ++a, --b) std::swap(p[a], p[b]);
        }
    return MI_OK;
}

template <class T>
void widen(const char* src, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) {
        T x;
        std::memcpy(&x, src + i * sizeof(T), sizeof(T));
        dst[i] = (float)(double)x;  // the upload cast of every scalar type
    }
}

void to_float(const MetaHeader& h, const std::string& data, float* dst, size_t n) {
    const char* s = data.data();
    switch (h.dtype) {
        case MI_U8: widen<uint8_t>(s, n, dst); break;
        case MI_I8: widen<int8_t>(s, n, dst); break;
        case MI_U16: widen<uint16_t>(s, n, dst); break;
        case MI_I16: widen<int16_t>(s, n, dst); break;
        case MI_U32: widen<uint32_t>(s, n, dst); break;
        case MI_I32: widen<int32_t>(s, n, dst); break;
        case MI_U64: widen<uint64_t>(s, n, dst); break;
        case MI_I64: widen<int64_t>(s, n, dst); break;
        case MI_F32: widen<float>(s, n, dst); break;
        default: widen<double>(s, n, dst); break;
    }
}

void to_geometry(const MetaHeader& h, mi_geometry* g) {
    for (int d = 0; d < 3; ++d) {
        g->size[d] = h.size[d];
        g->spacing[d] = h.spacing[d];
        g->origin[d] = h.origin[d];
    }
    for (int i = 0; i < 9; ++i) g->direction[i] = h.direction[i];
}

}  // namespace
}  // namespace mi

extern "C" {

mi_status mi_image_read_meta_host(const char* path, mi_geometry* geometry, float* dst, size_t n_elements) {
    if (!path || !geometry) return MI_ERR_INVALID_ARGUMENT;
    mi::MetaHeader h;
    std::string data;
    mi_status s = mi::read_pixels(nullptr, path, h, data);
    if (s != MI_OK) return s;
    mi::to_geometry(h, geometry);
    const size_t n = (size_t)(h.size[0] * h.size[1] * h.size[2]);
    if (!dst) return MI_OK;  // geometry only
    if (n_elements < n) return MI_ERR_INVALID_ARGUMENT;
    mi::to_float(h, data, dst, n);
    return MI_OK;
}

mi_status mi_image_read_meta(mi_context* ctx, const char* path, mi_image** out) {
    if (!ctx || !path || !out) return MI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    mi::MetaHeader h;
    std::string data;
    mi_status s = mi::read_pixels(ctx, path, h, data);
    if (s != MI_OK) return s;
    mi_geometry g;
    mi::to_geometry(h, &g);
    return mi_image_upload(ctx, data.data(), h.dtype, &g, out);
}

}  // extern "C"
