#include "image_io.h"

#include <zlib.h>

#include <algorithm>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>

#include "../../../include/ctb.h"

namespace ctb {

namespace {

bool read_file(const std::string& path, std::vector<uint8_t>* buf, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) {
        *err = "cannot open";
        return false;
    }
    f.seekg(0, std::ios::end);
    const std::streamoff n = f.tellg();
    if (n <= 0) {
        *err = "empty file";
        return false;
    }
    f.seekg(0, std::ios::beg);
    buf->resize(size_t(n));
    f.read(reinterpret_cast<char*>(buf->data()), n);
    if (!f) {
        *err = "read failed";
        return false;
    }
    return true;
}

size_t sample_bytes(int type) { return type == CTB_U8 ? 1 : type == CTB_U16 ? 2 : 4; }

// ----------------------------------------------------------------- PGM (P5)
struct PgmHeader {
    int w = 0, h = 0, maxval = 0;
    size_t offset = 0;
};

bool pgm_header(const std::vector<uint8_t>& b, PgmHeader* hd, std::string* err) {
    if (b.size() < 2 || b[0] != 'P' || b[1] != '5') {
        *err = "not a binary PGM";
        return false;
    }
    size_t i = 2;
    int vals[3];
    for (int k = 0; k < 3; ++k) {
        while (i < b.size()) {  // skip whitespace and comments
            if (b[i] == '#') {
                while (i < b.size() && b[i] != '\n') ++i;
            } else if (b[i] == ' ' || b[i] == '\t' || b[i] == '\n' || b[i] == '\r') {
                ++i;
            } else {
                break;
            }
        }
        long v = 0;
        bool any = false;
        while (i < b.size() && b[i] >= '0' && b[i] <= '9') {
            v = v * 10 + (b[i] - '0');
            any = true;
            ++i;
            if (v > (1L << 30)) break;
        }
        if (!any) {
            *err = "malformed PGM header";
            return false;
        }
        vals[k] = int(v);
    }
    ++i;  // single whitespace before the raster
    hd->w = vals[0];
    hd->h = vals[1];
    hd->maxval = vals[2];
    hd->offset = i;
    if (hd->w <= 0 || hd->h <= 0 || hd->maxval <= 0 || hd->maxval > 65535) {
        *err = "unsupported PGM size or maxval";
        return false;
    }
    return true;
}

// ----------------------------------------------------------------- TIFF
struct TiffInfo {
    int w = 0, h = 0, bps = 0, spp = 1, fmt = 1, comp = 1, photo = 1, planar = 1, predictor = 1;
    long rows_per_strip = -1;
    std::vector<uint64_t> offsets, counts;
    bool be = false;
};

struct Reader {
    const std::vector<uint8_t>& b;
    bool be;
    bool ok = true;
    uint32_t u16(size_t o) {
        if (o + 2 > b.size()) { ok = false; return 0; }
        return be ? (uint32_t(b[o]) << 8) | b[o + 1] : (uint32_t(b[o + 1]) << 8) | b[o];
    }
    uint32_t u32(size_t o) {
        if (o + 4 > b.size()) { ok = false; return 0; }
        return be ? (uint32_t(b[o]) << 24) | (uint32_t(b[o + 1]) << 16) | (uint32_t(b[o + 2]) << 8) | b[o + 3]
                  : (uint32_t(b[o + 3]) << 24) | (uint32_t(b[o + 2]) << 16) | (uint32_t(b[o + 1]) << 8) | b[o];
    }
};

bool tiff_info(const std::vector<uint8_t>& b, TiffInfo* t, std::string* err) {
    if (b.size() < 8 || !((b[0] == 'I' && b[1] == 'I') || (b[0] == 'M' && b[1] == 'M'))) {
        *err = "not a TIFF";
        return false;
    }
    t->be = b[0] == 'M';
    Reader r{b, t->be};
    if (r.u16(2) != 42) {
        *err = "not a classic TIFF";
        return false;
    }
    const size_t ifd = r.u32(4);
    const uint32_t n = r.u16(ifd);
    if (!r.ok) {
        *err = "truncated TIFF";
        return false;
    }
    for (uint32_t k = 0; k < n; ++k) {
        const size_t e = ifd + 2 + 12 * size_t(k);
        const uint32_t tag = r.u16(e), typ = r.u16(e + 2), cnt = r.u32(e + 4);
        auto value = [&](uint32_t idx) -> uint64_t {
            const size_t sz = typ == 3 ? 2 : 4;
            const size_t base = (sz * cnt <= 4) ? e + 8 : r.u32(e + 8);
            return typ == 3 ? r.u16(base + idx * 2) : r.u32(base + idx * 4);
        };
        switch (tag) {
            case 256: t->w = int(value(0)); break;
            case 257: t->h = int(value(0)); break;
            case 258: t->bps = int(value(0)); break;
            case 259: t->comp = int(value(0)); break;
            case 262: t->photo = int(value(0)); break;
            case 273: t->offsets.resize(cnt); for (uint32_t i = 0; i < cnt; ++i) t->offsets[i] = value(i); break;
            case 277: t->spp = int(value(0)); break;
            case 278: t->rows_per_strip = long(value(0)); break;
            case 279: t->counts.resize(cnt); for (uint32_t i = 0; i < cnt; ++i) t->counts[i] = value(i); break;
            case 284: t->planar = int(value(0)); break;
            case 317: t->predictor = int(value(0)); break;
            case 339: t->fmt = int(value(0)); break;
            default: break;
        }
    }
    if (!r.ok) {
        *err = "truncated TIFF directory";
        return false;
    }
    if (t->w <= 0 || t->h <= 0 || t->offsets.empty()) {
        *err = "TIFF without size or strips";
        return false;
    }
    // none, LZW, Deflate (two codes), PackBits; horizontal differencing for integers
    if (t->comp != 1 && t->comp != 5 && t->comp != 8 && t->comp != 32946 && t->comp != 32773) {
        *err = "unsupported TIFF compression " + std::to_string(t->comp);
        return false;
    }
    if (t->predictor != 1 && !(t->predictor == 2 && t->fmt == 1)) {
        *err = "unsupported TIFF predictor " + std::to_string(t->predictor);
        return false;
    }
    if (t->counts.size() != t->offsets.size() && t->comp != 1) {
        *err = "TIFF strip byte counts missing";
        return false;
    }
    // colour (RGB, RGBA) is read as cv::imread(GRAYSCALE) does: converted to gray
    const bool color = t->spp == 3 || t->spp == 4;
    if (!(t->spp == 1 || (color && t->photo == 2 && t->planar == 1 && (t->bps == 8 || t->bps == 16)))) {
        *err = "unsupported TIFF sample layout (" + std::to_string(t->spp) + " samples per pixel)";
        return false;
    }
    return true;
}

// cv::cvtColor RGB -> gray in 14-bit fixed point (R 4899, G 9617, B 1868), the
// conversion cv::imread(IMREAD_GRAYSCALE) applies to colour TIFF images.
template <typename T>
void rgb_to_gray(const T* src, int channels, size_t n, T* dst) {
    for (size_t i = 0; i < n; ++i) {
        const T* p = src + i * channels;
        dst[i] = T((uint32_t(p[0]) * 4899u + uint32_t(p[1]) * 9617u + uint32_t(p[2]) * 1868u + 8192u) >> 14);
    }
}

// TIFF LZW (compression 5): MSB-first codes of 9..12 bits, clear 256, end 257,
// the code width grows one code early (when the next free code reaches 2^n - 1).
// Codes are read from a bit buffer refilled a byte at a time, and every table
// entry is kept as (offset, length) of a place in the output where its string
// already stands: an entry is the previous string plus the first byte of the
// current one, which the output holds contiguously, so emitting a code is one
// copy from earlier output (1.9x faster than reading bit by bit and walking
// prefix chains, on 16-bit noise).
bool lzw_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t cap, std::string* err) {
    static thread_local uint32_t off[4096];
    static thread_local uint16_t len[4096];
    size_t out = 0, ip = 0;
    uint64_t bits = 0;
    int nbits = 0, width = 9, next = 258, prev = -1;
    size_t prev_off = 0, prev_len = 0;
    while (out < cap) {
        while (nbits < width && ip < n) {
            bits = (bits << 8) | src[ip++];
            nbits += 8;
        }
        if (nbits < width) break;  // running out of data ends the strip
        const int code = int((bits >> (nbits - width)) & ((1u << width) - 1u));
        nbits -= width;
        if (code == 257) break;
        if (code == 256) {
            width = 9;
            next = 258;
            prev = -1;
            continue;
        }
        const size_t start = out;
        size_t l;
        if (prev < 0) {
            if (code > 255) { *err = "corrupt LZW data"; return false; }
            dst[out++] = uint8_t(code);
            prev = code;
            prev_off = start;
            prev_len = 1;
            continue;
        }
        if (code > next || next >= 4096) { *err = "corrupt LZW data"; return false; }
        if (code < 256) {
            l = 1;
            dst[out++] = uint8_t(code);
        } else if (code < next) {
            l = len[code];
            if (out + l > cap) break;
            const uint8_t* from = dst + off[code];
            for (size_t k = 0; k < l; ++k) dst[out + k] = from[k];
            out += l;
        } else {  // the entry being made: previous string plus its own first byte
            l = prev_len + 1;
            if (out + l > cap) break;
            for (size_t k = 0; k < prev_len; ++k) dst[out + k] = dst[prev_off + k];
            dst[out + prev_len] = dst[prev_off];
            out += l;
        }
        off[next] = uint32_t(prev_off);
        len[next] = uint16_t(prev_len + 1);
        ++next;
        prev = code;
        prev_off = start;
        prev_len = l;
        if (next + 1 >= (1 << width) && width < 12) ++width;
    }
    if (out != cap) { *err = "LZW strip shorter than its rows"; return false; }
    return true;
}

// PackBits (compression 32773).
bool packbits_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t cap, std::string* err) {
    size_t i = 0, out = 0;
    while (i < n && out < cap) {
        const int8_t h = int8_t(src[i++]);
        if (h >= 0) {
            const size_t k = size_t(h) + 1;
            if (i + k > n || out + k > cap) break;
            std::memcpy(dst + out, src + i, k);
            i += k;
            out += k;
        } else if (h != -128) {
            const size_t k = size_t(1 - h);
            if (i >= n || out + k > cap) break;
            std::memset(dst + out, src[i++], k);
            out += k;
        }
    }
    if (out != cap) { *err = "PackBits strip shorter than its rows"; return false; }
    return true;
}

int tiff_type(const TiffInfo& t) {
    if (t.bps == 8 && t.fmt == 1) return CTB_U8;
    if (t.bps == 16 && t.fmt == 1) return CTB_U16;
    if (t.bps == 32 && t.fmt == 3) return CTB_F32;
    return 0;
}

// ----------------------------------------------------------------- PNG
uint32_t be32(const uint8_t* p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

struct PngInfo {
    int w = 0, h = 0, depth = 0, color = 0, interlace = 0;
    std::vector<uint8_t> idat;
};

bool png_info(const std::vector<uint8_t>& b, PngInfo* p, bool want_data, std::string* err) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (b.size() < 33 || std::memcmp(b.data(), sig, 8) != 0) {
        *err = "not a PNG";
        return false;
    }
    size_t i = 8;
    bool have_ihdr = false;
    while (i + 12 <= b.size()) {
        const uint32_t len = be32(&b[i]);
        const char* type = reinterpret_cast<const char*>(&b[i + 4]);
        if (i + 12 + size_t(len) > b.size()) {
            *err = "truncated PNG chunk";
            return false;
        }
        const uint8_t* data = &b[i + 8];
        if (std::memcmp(type, "IHDR", 4) == 0 && len >= 13) {
            p->w = int(be32(data));
            p->h = int(be32(data + 4));
            p->depth = data[8];
            p->color = data[9];
            p->interlace = data[12];
            have_ihdr = true;
            if (!want_data) break;
        } else if (std::memcmp(type, "IDAT", 4) == 0) {
            p->idat.insert(p->idat.end(), data, data + len);
        } else if (std::memcmp(type, "IEND", 4) == 0) {
            break;
        }
        i += 12 + size_t(len);
    }
    if (!have_ihdr) {
        *err = "PNG without IHDR";
        return false;
    }
    // gray (0), RGB (2), gray + alpha (4), RGBA (6); palettes are not read
    if (p->color != 0 && p->color != 2 && p->color != 4 && p->color != 6) {
        *err = "palette PNG is not supported";
        return false;
    }
    if (p->interlace != 0) {
        *err = "interlaced PNG is not supported";
        return false;
    }
    if (p->depth != 8 && p->depth != 16) {
        *err = "only 8/16-bit PNG is supported";
        return false;
    }
    return true;
}

int png_channels(int color) { return color == 2 ? 3 : color == 4 ? 2 : color == 6 ? 4 : 1; }

bool png_decode(PngInfo& p, void* dst, std::string* err) {
    const int ch = png_channels(p.color);
    const size_t bps = p.depth / 8;            // bytes per sample
    const size_t bpp = bps * ch;               // bytes per pixel (filter unit)
    const size_t stride = size_t(p.w) * bpp;
    std::vector<uint8_t> raw((stride + 1) * size_t(p.h));
    uLongf out_len = uLongf(raw.size());
    if (uncompress(raw.data(), &out_len, p.idat.data(), uLong(p.idat.size())) != Z_OK || out_len != raw.size()) {
        *err = "PNG inflate failed";
        return false;
    }
    std::vector<uint8_t> prev(stride, 0), cur(stride);
    uint8_t* out = static_cast<uint8_t*>(dst);
    for (int r = 0; r < p.h; ++r) {
        const uint8_t f = raw[size_t(r) * (stride + 1)];
        const uint8_t* src = &raw[size_t(r) * (stride + 1) + 1];
        for (size_t c = 0; c < stride; ++c) {
            const int a = c >= bpp ? cur[c - bpp] : 0, up = prev[c], ul = c >= bpp ? prev[c - bpp] : 0;
            int v = src[c];
            switch (f) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += up; break;
                case 3: v += (a + up) / 2; break;
                case 4: {
                    const int pp = a + up - ul, pa = std::abs(pp - a), pb = std::abs(pp - up), pc = std::abs(pp - ul);
                    v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? up : ul);
                    break;
                }
                default: *err = "bad PNG filter"; return false;
            }
            cur[c] = uint8_t(v);
        }
        // samples of this row (big-endian 16-bit), then one gray value per pixel:
        // gray + alpha keeps the gray sample, colour goes through the gray formula
        auto sample = [&](int c, int k) -> uint32_t {
            const size_t o = size_t(c) * bpp + size_t(k) * bps;
            return bps == 1 ? cur[o] : (uint32_t(cur[o]) << 8) | cur[o + 1];
        };
        for (int c = 0; c < p.w; ++c) {
            uint32_t g = sample(c, 0);
            if (ch >= 3) g = (sample(c, 0) * 4899u + sample(c, 1) * 9617u + sample(c, 2) * 1868u + 8192u) >> 14;
            if (bps == 1) out[size_t(r) * p.w + c] = uint8_t(g);
            else reinterpret_cast<uint16_t*>(out)[size_t(r) * p.w + c] = uint16_t(g);
        }
        std::swap(prev, cur);
    }
    return true;
}

}  // namespace

namespace {

bool probe_buf(const std::vector<uint8_t>& b, int* width, int* height, int* type, std::string* err) {
    if (b.size() >= 2 && b[0] == 'P' && b[1] == '5') {
        PgmHeader hd;
        if (!pgm_header(b, &hd, err)) return false;
        *width = hd.w; *height = hd.h; *type = hd.maxval < 256 ? CTB_U8 : CTB_U16;
        return true;
    }
    if (b.size() >= 4 && (b[0] == 'I' || b[0] == 'M')) {
        TiffInfo t;
        if (!tiff_info(b, &t, err)) return false;
        *width = t.w; *height = t.h; *type = tiff_type(t);
        if (!*type) { *err = "unsupported TIFF sample format"; return false; }
        return true;
    }
    if (b.size() >= 8 && b[0] == 137 && b[1] == 'P') {
        PngInfo p;
        if (!png_info(b, &p, false, err)) return false;
        *width = p.w; *height = p.h; *type = p.depth == 8 ? CTB_U8 : CTB_U16;
        return true;
    }
    *err = "unsupported image format";
    return false;
}

bool decode_buf(const std::vector<uint8_t>& b, int width, int height, int type, void* dst, std::string* err) {
    const size_t n = size_t(width) * height;
    if (b.size() >= 2 && b[0] == 'P' && b[1] == '5') {
        PgmHeader hd;
        if (!pgm_header(b, &hd, err)) return false;
        const int t = hd.maxval < 256 ? CTB_U8 : CTB_U16;
        if (hd.w != width || hd.h != height || t != type) { *err = "size or depth differs"; return false; }
        if (b.size() < hd.offset + n * sample_bytes(t)) { *err = "truncated PGM raster"; return false; }
        const uint8_t* src = b.data() + hd.offset;
        if (t == CTB_U8) {
            std::memcpy(dst, src, n);
        } else {
            uint16_t* o = static_cast<uint16_t*>(dst);
            for (size_t i = 0; i < n; ++i) o[i] = uint16_t((src[2 * i] << 8) | src[2 * i + 1]);
        }
        return true;
    }
    if (b.size() >= 4 && (b[0] == 'I' || b[0] == 'M')) {
        TiffInfo t;
        if (!tiff_info(b, &t, err)) return false;
        const int ty = tiff_type(t);
        if (t.w != width || t.h != height || ty != type) { *err = "size or depth differs"; return false; }
        const size_t sb = sample_bytes(ty), spp = size_t(t.spp), row = size_t(width) * sb * spp;
        const long rps = t.rows_per_strip > 0 ? t.rows_per_strip : height;
        std::vector<uint8_t> interleaved(spp > 1 ? n * sb * spp : 0);
        uint8_t* o = spp > 1 ? interleaved.data() : static_cast<uint8_t*>(dst);
        size_t written = 0;
        for (size_t s = 0; s < t.offsets.size() && written < n * sb * spp; ++s) {
            const size_t rows = std::min<size_t>(size_t(rps), size_t(height) - s * size_t(rps));
            const size_t bytes = rows * row;
            if (t.comp == 1) {
                if (t.offsets[s] + bytes > b.size()) { *err = "truncated TIFF strip"; return false; }
                std::memcpy(o + written, b.data() + t.offsets[s], bytes);
            } else {
                if (t.offsets[s] + t.counts[s] > b.size()) { *err = "truncated TIFF strip"; return false; }
                const uint8_t* src = b.data() + t.offsets[s];
                const size_t cn = size_t(t.counts[s]);
                if (t.comp == 5) {
                    if (!lzw_decode(src, cn, o + written, bytes, err)) return false;
                } else if (t.comp == 32773) {
                    if (!packbits_decode(src, cn, o + written, bytes, err)) return false;
                } else {  // Deflate: a zlib stream per strip
                    uLongf got = uLongf(bytes);
                    if (uncompress(o + written, &got, src, uLong(cn)) != Z_OK || got != bytes) {
                        *err = "TIFF Deflate strip failed to inflate";
                        return false;
                    }
                }
            }
            written += bytes;
        }
        if (written != n * sb * spp) { *err = "TIFF strips do not cover the image"; return false; }
        if (t.be && sb > 1) {
            for (size_t i = 0; i < n * spp; ++i) std::reverse(o + i * sb, o + (i + 1) * sb);
        }
        if (t.predictor == 2) {  // horizontal differencing, per sample channel, within each row
            const size_t rs = size_t(width) * spp;
            for (int r = 0; r < height; ++r) {
                if (sb == 1) {
                    uint8_t* v = o + size_t(r) * rs;
                    for (size_t i = spp; i < rs; ++i) v[i] = uint8_t(v[i] + v[i - spp]);
                } else {
                    uint16_t* v = reinterpret_cast<uint16_t*>(o) + size_t(r) * rs;
                    for (size_t i = spp; i < rs; ++i) v[i] = uint16_t(v[i] + v[i - spp]);
                }
            }
        }
        if (spp > 1) {
            if (sb == 1) rgb_to_gray(o, int(spp), n, static_cast<uint8_t*>(dst));
            else rgb_to_gray(reinterpret_cast<const uint16_t*>(o), int(spp), n, static_cast<uint16_t*>(dst));
        }
        return true;
    }
    if (b.size() >= 8 && b[0] == 137 && b[1] == 'P') {
        PngInfo p;
        if (!png_info(b, &p, true, err)) return false;
        const int t = p.depth == 8 ? CTB_U8 : CTB_U16;
        if (p.w != width || p.h != height || t != type) { *err = "size or depth differs"; return false; }
        return png_decode(p, dst, err);
    }
    *err = "unsupported image format";
    return false;
}

}  // namespace

bool probe_image(const std::string& path, int* width, int* height, int* type, std::string* err) {
    std::vector<uint8_t> b;
    return read_file(path, &b, err) && probe_buf(b, width, height, type, err);
}

bool decode_image_into(const std::string& path, int width, int height, int type, void* dst, std::string* err) {
    std::vector<uint8_t> b;
    return read_file(path, &b, err) && decode_buf(b, width, height, type, dst, err);
}

int load_image_into(const std::string& path, int width, int height, int type, void* dst, std::string* err) {
    std::vector<uint8_t> b;
    int w = 0, h = 0, t = 0;
    if (!read_file(path, &b, err) || !probe_buf(b, &w, &h, &t, err)) return kLoadUnreadable;
    if (w != width || h != height) return kLoadOtherSize;
    if (t != type) return kLoadOtherDepth;
    return decode_buf(b, width, height, type, dst, err) ? kLoadOk : kLoadUnreadable;
}

bool decode_image(const std::string& path, Image* img, std::string* err) {
    if (!probe_image(path, &img->width, &img->height, &img->type, err)) return false;
    img->data.resize(size_t(img->width) * img->height * sample_bytes(img->type));
    return decode_image_into(path, img->width, img->height, img->type, img->data.data(), err);
}

}  // namespace ctb
