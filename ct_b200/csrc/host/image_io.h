// Projection image decoding for the CSV ingest path.
//
// The reference decodes with cv::imread(GRAYSCALE | ANYDEPTH)
// (Ct/CtVolume.cpp:20-33) and accepts 8-bit, 16-bit and 32-bit float images
// (:247). This decoder covers the lossless single-channel formats CT
// projection exports use: binary PGM (P5, 8/16-bit, big-endian samples as in
// the Netpbm specification), baseline TIFF (uncompressed, strips, II or MM byte
// order, 8/16-bit unsigned or 32-bit IEEE float) and PNG (8/16-bit grayscale,
// non-interlaced, zlib).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ctb {

struct Image {
    int width = 0, height = 0;
    int type = 0;               // CTB_U8, CTB_U16 or CTB_F32
    std::vector<uint8_t> data;  // row-major, native-endian samples
};

// The size and sample type from the header. Returns false with a message.
bool probe_image(const std::string& path, int* width, int* height, int* type, std::string* err);

// Decodes the image into dst (width*height samples of `type`), which must be
// large enough. Returns false with a message on failure.
bool decode_image_into(const std::string& path, int width, int height, int type, void* dst, std::string* err);
// Both in one read of the file: the image's size and depth must be the given
// ones (the projections of one scan), then its samples go to dst.
enum { kLoadOk = 0, kLoadUnreadable = 1, kLoadOtherSize = 2, kLoadOtherDepth = 3 };
int load_image_into(const std::string& path, int width, int height, int type, void* dst, std::string* err);

bool decode_image(const std::string& path, Image* img, std::string* err);

}  // namespace ctb
