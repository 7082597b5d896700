// saveVolumeToBinaryFile (Ct/CtVolume.cpp:634-721) and
// Volume<float>::saveToBinaryFile (Common/Volume.h:476-574).
//
// Writes <base>.txt (reconstruction info), <base>.vgi (VG Studio header with
// the volume's min/max) and the raw float32 file in the requested index order
// and byte order. The raw data is converted in parallel blocks and written in
// large chunks instead of one QDataStream call per voxel.

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "reconstructor.h"

namespace ctb {

namespace {

std::string base_name(const std::string& path) {  // QFileInfo::baseName: up to the first '.'
    size_t s = path.find_last_of('/');
    std::string f = s == std::string::npos ? path : path.substr(s + 1);
    size_t d = f.find('.');
    return d == std::string::npos ? f : f.substr(0, d);
}
std::string file_name(const std::string& path) {
    size_t s = path.find_last_of('/');
    return s == std::string::npos ? path : path.substr(s + 1);
}
std::string dir_of(const std::string& path) {
    size_t s = path.find_last_of('/');
    return s == std::string::npos ? std::string() : path.substr(0, s + 1);
}

// QTextStream << float / QString::arg(double): %g with 6 significant digits.
std::string g6(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%g", v);
    return b;
}
std::string f3(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.3f", v);
    return b;
}

}  // namespace

int Reconstructor::save(const std::string& path, int index_order, int byte_order) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    const int X = vol_dims_[0], Y = vol_dims_[1], Z = vol_dims_[2];
    const std::string dir = dir_of(path), base = base_name(path), fname = file_name(path);
    {
        FILE* f = std::fopen((dir + base + ".txt").c_str(), "wb");
        if (!f) return fail(CTB_ERR_IO, "Could not write the info file.");
        std::string s;
        s += fname + "\n\n";
        s += "[Image dimensions]\n";
        s += "U resolution:\t\t" + std::to_string(det_.width) + "\n";
        s += "V resolution:\t\t" + std::to_string(det_.height) + "\n\n";
        s += "[Reconstruction parameters]\n";
        s += "FCD:\t\t\t\t\t" + g6(det_.fcd) + "\n";
        s += "Pixel size:\t\t\t" + g6(float(pixel_size_)) + "\n";
        s += "U offset:\t\t\t" + g6(det_.u_offset) + "\n";
        s += "X range relative:\t[" + f3(rel_[0]) + " - " + f3(rel_[1]) + "]\n";
        s += "Y range relative:\t[" + f3(rel_[2]) + " - " + f3(rel_[3]) + "]\n";
        s += "Z range relative:\t[" + f3(rel_[4]) + " - " + f3(rel_[5]) + "]\n";
        s += "X range:\t\t\t[" + std::to_string(grid_.x_from) + ".." + std::to_string(grid_.x_to) + "]\n";
        s += "Y range:\t\t\t[" + std::to_string(grid_.y_from) + ".." + std::to_string(grid_.y_to) + "]\n";
        s += "Z range:\t\t\t[" + std::to_string(grid_.z_from) + ".." + std::to_string(grid_.z_to) + "]\n\n";
        s += "[Volume dimensions]\n";
        s += "X size:\t\t\t\t" + std::to_string(X) + "\n";
        s += "Y size:\t\t\t\t" + std::to_string(Y) + "\n";
        s += "Z size:\t\t\t\t" + std::to_string(Z) + "\n\n";
        s += "[Data format]\n";
        s += "Data type:\t\t\t32bit IEEE 754 float\n";
        s += byte_order == CTB_LITTLE_ENDIAN ? "Byte order:\t\t\tLittle endian\n" : "Byte order:\t\t\tBig endian\n";
        s += index_order == CTB_Z_FASTEST ? "Index order:\t\tZ fastest" : "Index order:\t\tX fastest";
        std::fwrite(s.data(), 1, s.size(), f);
        std::fclose(f);
    }
    // volume min/max (Volume::calculateMinMax, Common/Volume.h:192-217); an empty
    // volume reports 0 0 as Volume::min()/max() do.
    float vmin = 0, vmax = 0;
    const float* v = static_cast<const float*>(volume_.p);
    const size_t n = size_t(X) * Y * Z;
    if (n > 0 && v) {
        const unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<float> mins(T, FLT_MAX), maxs(T, -FLT_MAX);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < T; ++t)
            th.emplace_back([&, t] {
                float a = FLT_MAX, b = -FLT_MAX;
                for (size_t i = t * n / T; i < (t + 1) * n / T; ++i) { a = std::min(a, v[i]); b = std::max(b, v[i]); }
                mins[t] = a; maxs[t] = b;
            });
        for (auto& x : th) x.join();
        vmin = *std::min_element(mins.begin(), mins.end());
        vmax = *std::max_element(maxs.begin(), maxs.end());
    }
    {
        FILE* f = std::fopen((dir + base + ".vgi").c_str(), "wb");
        if (!f) return fail(CTB_ERR_IO, "Could not write the vgi file.");
        const std::string sz = std::to_string(X) + " " + std::to_string(Y) + " " + std::to_string(Z);
        const std::string range = g6(vmin) + " " + g6(vmax);
        const std::string res = g6(float(pixel_size_));
        std::string s = "{volume1}\n[representation]\nsize = " + sz + "\nbitsperelement = 32\ndatatype = float\n"
                        "datarange = " + range + "\n[file1]\nFileFormat = raw\nSize = " + sz + "\nName = ./" + fname +
                        "\nbitsperelement = 32\ndatatype = float\ndatarange = " + range +
                        "\n{volumeprimitive}\n[geometry]\nclipbox = 0 0 0 " + sz + "\nstatus = visible\nresolution = " +
                        res + " " + res + " " + res + "\nunit = mm\n[volume]\nvolume = volume1\n";
        std::fwrite(s.data(), 1, s.size(), f);
        std::fclose(f);
    }
    if (n == 0 || !v) return fail(CTB_ERR_ARG, "Did not save the volume, because it appears to be empty.");
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(CTB_ERR_IO, "Could not open the file. Maybe your path does not exist. No files were written.");
    // convert one x-slab (Z_FASTEST) or one z-slab (X_FASTEST) block at a time
    const size_t block = index_order == CTB_Z_FASTEST ? size_t(Y) * Z : size_t(X) * Y;
    const size_t nblocks = index_order == CTB_Z_FASTEST ? size_t(X) : size_t(Z);
    const size_t per = std::max<size_t>(1, (size_t(64) << 20) / (block * 4));
    std::vector<uint32_t> buf(block * per);
    for (size_t b0 = 0; b0 < nblocks; b0 += per) {
        if (stop_) { std::fclose(f); return fail(CTB_INTERRUPTED, "User interrupted. Stopping."); }
        const size_t nb = std::min(per, nblocks - b0);
        const unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < T; ++t)
            th.emplace_back([&, t] {
                for (size_t k = t; k < nb; k += T) {
                    const size_t ob = b0 + k;
                    uint32_t* o = buf.data() + k * block;
                    if (index_order == CTB_Z_FASTEST) {  // ob = x
                        for (int y = 0; y < Y; ++y)
                            for (int z = 0; z < Z; ++z) {
                                float val = v[(size_t(z) * Y + y) * X + ob];
                                std::memcpy(&o[size_t(y) * Z + z], &val, 4);
                            }
                    } else {
                        std::memcpy(o, v + ob * block, block * 4);
                    }
                    if (byte_order == CTB_BIG_ENDIAN)
                        for (size_t i = 0; i < block; ++i) o[i] = __builtin_bswap32(o[i]);
                }
            });
        for (auto& x : th) x.join();
        if (std::fwrite(buf.data(), 4, nb * block, f) != nb * block) {
            std::fclose(f);
            return fail(CTB_ERR_IO, "An error occured while writing to the disk. Maybe there is not enough free disk space.");
        }
        progress(2, 100.0 * double(b0 + nb) / double(nblocks));
    }
    std::fclose(f);
    return CTB_OK;
}

}  // namespace ctb
