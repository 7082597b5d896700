// Reading reconstructions back (round trip of the save path): the .txt info
// parse of the viewer and Volume<float>::loadFromBinaryFile, plus the
// cross-section previews of Volume::getVolumeCrossSection.

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../ctb_internal.h"
#include "reconstructor.h"

namespace ctb {
namespace {

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return char(std::tolower(c)); });
    return s;
}

// QString::toULongLong: the whole field is an unsigned decimal number.
bool to_ull(const std::string& s, unsigned long long* v) {
    if (s.empty()) return false;
    char* e = nullptr;
    const unsigned long long r = std::strtoull(s.c_str(), &e, 10);
    if (*e != '\0' || s[0] == '-' || s[0] == '+' || std::isspace((unsigned char)s[0])) return false;
    *v = r;
    return true;
}

size_t type_size(int dt) {
    switch (dt) {
        case CTB_DT_FLOAT32: return 4;
        case CTB_DT_DOUBLE64: return 8;
        case CTB_DT_UINT8: case CTB_DT_INT8: return 1;
        case CTB_DT_UINT16: case CTB_DT_INT16: return 2;
        case CTB_DT_UINT32: case CTB_DT_INT32: return 4;
    }
    return 0;
}

float convert(const unsigned char* p, int dt, bool swap) {
    unsigned char b[8];
    const size_t n = type_size(dt);
    for (size_t i = 0; i < n; ++i) b[i] = swap ? p[n - 1 - i] : p[i];
    switch (dt) {
        case CTB_DT_FLOAT32: { float v; std::memcpy(&v, b, 4); return v; }
        case CTB_DT_DOUBLE64: { double v; std::memcpy(&v, b, 8); return float(v); }
        case CTB_DT_UINT8: return float(b[0]);
        case CTB_DT_INT8: return float(int8_t(b[0]));
        case CTB_DT_UINT16: { uint16_t v; std::memcpy(&v, b, 2); return float(v); }
        case CTB_DT_INT16: { int16_t v; std::memcpy(&v, b, 2); return float(v); }
        case CTB_DT_UINT32: { uint32_t v; std::memcpy(&v, b, 4); return float(v); }
        case CTB_DT_INT32: { int32_t v; std::memcpy(&v, b, 4); return float(v); }
    }
    return 0.0f;
}

}  // namespace

int cross_section_of(const float* v, int X, int Y, int Z, int axis, int index, float* out, int* rows, int* cols) {
    auto at = [&](size_t x, size_t y, size_t z) { return v[(z * Y + y) * X + x]; };
    int R, C;
    if (axis == CTB_AXIS_X) { R = Z; C = Y; if (index < 0 || index >= X) return CTB_ERR_ARG; }
    else if (axis == CTB_AXIS_Y) { R = Z; C = X; if (index < 0 || index >= Y) return CTB_ERR_ARG; }
    else { R = X; C = Y; if (index < 0 || index >= Z) return CTB_ERR_ARG; }
    if (rows) *rows = R;
    if (cols) *cols = C;
    if (!out) return CTB_OK;
    for (int r = 0; r < R; ++r)
        for (int c = 0; c < C; ++c) {
            float val;
            if (axis == CTB_AXIS_X) val = at(index, c, R - 1 - r);
            else if (axis == CTB_AXIS_Y) val = at(C - 1 - c, index, R - 1 - r);
            else val = at(r, c, index);
            out[size_t(r) * C + c] = val;
        }
    return CTB_OK;
}

int Reconstructor::cross_section(int axis, int index, float* out, int* rows, int* cols) const {
    const int X = vol_dims_[0], Y = vol_dims_[1], Z = vol_dims_[2];
    if (X == 0 || !volume_.p) return CTB_ERR_ARG;
    return cross_section_of(static_cast<const float*>(volume_.p), X, Y, Z, axis, index, out, rows, cols);
}

}  // namespace ctb

extern "C" {

int ctb_read_volume_info(const char* txt_path, int* x, int* y, int* z, int* index_order, int* byte_order) {
    using namespace ctb;
    if (!txt_path) { set_global_error("null path"); return CTB_ERR_ARG; }
    std::ifstream in(txt_path);
    if (!in.good()) { set_global_error("The info file could not be opened."); return CTB_ERR_IO; }
    unsigned long long xs = 0, ys = 0, zs = 0;
    bool bo_found = false, io_found = false;
    int bo = CTB_LITTLE_ENDIAN, io = CTB_Z_FASTEST;
    std::string line;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        const std::string l = lower(line);
        unsigned long long* target = nullptr;
        if (l.find("x size:") != std::string::npos) target = &xs;
        else if (l.find("y size:") != std::string::npos) target = &ys;
        else if (l.find("z size:") != std::string::npos) target = &zs;
        if (target) {
            std::stringstream ss(line);
            std::string part;
            while (std::getline(ss, part, '\t')) {
                unsigned long long v;
                if (to_ull(part, &v)) *target = v;
            }
        } else if (l.find("byte order:") != std::string::npos) {
            bo_found = true;
            if (l.find("big endian") != std::string::npos) bo = CTB_BIG_ENDIAN;
        } else if (l.find("index order:") != std::string::npos) {
            io_found = true;
            if (l.find("x fastest") != std::string::npos) io = CTB_X_FASTEST;
        }
    }
    if (x) *x = int(xs);
    if (y) *y = int(ys);
    if (z) *z = int(zs);
    if (index_order) *index_order = io;
    if (byte_order) *byte_order = bo;
    if (!(xs > 0 && ys > 0 && zs > 0 && bo_found && io_found)) {
        set_global_error("The info file does not contain the volume dimensions, byte order and index order.");
        return CTB_ERR_ARG;
    }
    return CTB_OK;
}

int ctb_load_volume(const char* raw_path, int x, int y, int z, int index_order, int byte_order, int data_type,
                    size_t header_offset, int mirror_x, int mirror_y, int mirror_z, float* out) {
    using namespace ctb;
    const size_t es = type_size(data_type);
    if (!raw_path || !out || x <= 0 || y <= 0 || z <= 0 || es == 0) {
        set_global_error("ctb_load_volume: invalid arguments");
        return CTB_ERR_ARG;
    }
    FILE* f = std::fopen(raw_path, "rb");
    if (!f) { set_global_error("Could not open the file. Maybe your path does not exist."); return CTB_ERR_IO; }
    std::fseek(f, 0, SEEK_END);
    const long long actual = std::ftell(f);
    const size_t n = size_t(x) * y * z;
    const size_t expected = n * es + header_offset;
    if (actual < 0 || size_t(actual) < expected) {
        std::fclose(f);
        set_global_error("The size of the file does not fit the given parameters. Expected filesize: " +
                         std::to_string(expected) + " Actual filesize: " + std::to_string(actual));
        return CTB_ERR_IO;
    }
    std::fseek(f, long(header_offset), SEEK_SET);
    // file order: Z_FASTEST walks x (outer) -> y -> z, X_FASTEST walks z -> y -> x
    const int outer_n = index_order == CTB_X_FASTEST ? z : x;
    const int inner_n = index_order == CTB_X_FASTEST ? x : z;
    std::vector<unsigned char> buf(size_t(y) * inner_n * es);
    const bool swap = byte_order == CTB_BIG_ENDIAN;
    for (int o = 0; o < outer_n; ++o) {
        if (std::fread(buf.data(), 1, buf.size(), f) != buf.size()) {
            std::fclose(f);
            set_global_error("An error occured while reading from the disk.");
            return CTB_ERR_IO;
        }
        for (int yy = 0; yy < y; ++yy)
            for (int i = 0; i < inner_n; ++i) {
                int xx = index_order == CTB_X_FASTEST ? i : o;
                int zz = index_order == CTB_X_FASTEST ? o : i;
                int yv = yy;
                if (mirror_x) xx = x - xx - 1;
                if (mirror_y) yv = y - yv - 1;
                if (mirror_z) zz = z - zz - 1;
                out[(size_t(zz) * y + yv) * x + xx] = convert(&buf[(size_t(yy) * inner_n + i) * es], data_type, swap);
            }
    }
    std::fclose(f);
    return CTB_OK;
}

}  // extern "C"
