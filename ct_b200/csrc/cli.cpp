// ctb -- console front end with the option set of the reference's console
// mode (Ct/main.cpp:53-234): -i/-o, -f, -n, -c, -d, -w, -m, -e, -j, -b,
// --xmin..--zmax, -h. As in the reference, the default index order is
// X fastest (Ct/main.cpp:62) although the help text says zfastest, -j only
// switches when given "zfastest" (:174), and an unknown filter name keeps
// ramlak (:123-129). The call order is load -> bounds -> filter ->
// reconstruct -> save (:220-227).
//
// Engine extensions: --precision fp32|fp16|bf16, --pad 1|2,
// --grid X,Y,Z,voxel_pitch, --slab N.

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ctb.h"

namespace {

void usage() {
    std::printf(
        "Usage: ctb [parameters]\n"
        "Parameters:\n"
        "\t-i [path]\tFile path to the input config file. Long: --input.\n"
        "\t-o [path]\tFile path for the output file. Long: --output.\n"
        "\t-b \t\tOptional. Run with background priority (no effect on Linux). Long: --background.\n"
        "\t-f [option] \tOptional. Sets the preprocessing filter. Options are 'ramlak', 'shepplogan' and\n"
        "\t\t\t'hann'. Long: --filter. Default: ramlak\n"
        "\t-n \t\tOptional. Disables CUDA (not available: this engine reconstructs on the GPU). Long: --nocuda.\n"
        "\t-c \t\tOptional. CPU preprocessing (ignored: preprocessing runs on the GPU). Long: --cpuPreprocessing.\n"
        "\t-d 0,1,..,n \tOptional. CUDA devices; each reconstructs a share of the z slices.\n"
        "\t\t\tLong: --cudadevices. Default: 0\n"
        "\t-w x,y \t\tOptional. Exponents of the multiprocessor and memory-bandwidth shares in the\n"
        "\t\t\tper-device weights. Long: --weights. Default: 1,1\n"
        "\t-m [number] \tOptional. VRAM to spare in Mb. Long: --cudasparememory. Default: 200\n"
        "\t-e [option] \tOptional. Byte order of the output, 'littleendian' or 'bigendian'. Long: --byteorder.\n"
        "\t-j [option] \tOptional. Index order of the output, 'zfastest' or 'xfastest'. Long: --indexorder.\n"
        "\t-h \t\tDisplay this help. Long: --help.\n"
        "\t--xmin/--xmax/--ymin/--ymax/--zmin/--zmax 0..1\tOptional. Bounds of the reconstructed part.\n"
        "\t--precision fp32|fp16|bf16\tOptional. Storage of the projections (arithmetic is FP32).\n"
        "\t--pad 1|2\tOptional. 1: reference filter (no padding); 2: zero padding to 2W.\n"
        "\t--grid X,Y,Z,pitch\tOptional. Grid size and voxel pitch in detector pixels.\n"
        "\t--slab N\tOptional. z-slab height of the streamed output.\n");
}

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return char(std::tolower(c)); });
    return s;
}

bool parse_double(int argc, char** argv, int i, double* out) {
    if (i >= argc) return false;
    *out = std::strtod(argv[i], nullptr);
    return true;
}

void progress(int stage, double pct, void*) {
    static const char* names[] = {"Loading", "Reconstructing", "Saving"};
    std::printf("\r%s: %.0f%%", names[stage < 0 || stage > 2 ? 0 : stage], pct);
    std::fflush(stdout);
    if (pct >= 100.0) std::printf("\n");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2 || !std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help")) {
        usage();
        return argc < 2 ? 1 : 0;
    }
    std::string input, output;
    bool have_in = false, have_out = false, nocuda = false;
    int filter = CTB_RAMLAK, order = CTB_X_FASTEST, endian = CTB_LITTLE_ENDIAN, store = CTB_FP32;
    int pad = 1, slab = 0;
    std::vector<int> devices{0};
    double mp_coef = 1, bw_coef = 1;
    double spare = 200, xmin = 0, xmax = 1, ymin = 0, ymax = 1, zmin = 0, zmax = 1;
    int gx = 0, gy = 0, gz = 0;
    double gvs = 1;
    std::string filter_name = "Ram-Lak";
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--xmin") parse_double(argc, argv, ++i, &xmin);
        else if (a == "--xmax") parse_double(argc, argv, ++i, &xmax);
        else if (a == "--ymin") parse_double(argc, argv, ++i, &ymin);
        else if (a == "--ymax") parse_double(argc, argv, ++i, &ymax);
        else if (a == "--zmin") parse_double(argc, argv, ++i, &zmin);
        else if (a == "--zmax") parse_double(argc, argv, ++i, &zmax);
        else if (a == "-f" || a == "--filter") {
            if (++i < argc) {
                const std::string f = lower(argv[i]);
                if (f == "shepplogan") { filter = CTB_SHEPPLOGAN; filter_name = "Shepp-Logan"; }
                else if (f == "hann") { filter = CTB_HANN; filter_name = "Hann"; }
            }
        } else if (a == "-i" || a == "--input") {
            if (++i < argc) { input = argv[i]; have_in = true; }
        } else if (a == "-o" || a == "--output") {
            if (++i < argc) { output = argv[i]; have_out = true; }
        } else if (a == "-b" || a == "--background") {
        } else if (a == "-n" || a == "--nocuda") {
            nocuda = true;
        } else if (a == "-c" || a == "--cpuPreprocessing") {
        } else if (a == "-d" || a == "--cudadevices") {
            if (++i < argc) {
                std::string list = argv[i];
                if (list.empty()) {
                    std::printf("When using the flag -d you have to specify at least one device ID.\n");
                    return 1;
                }
                devices.clear();
                size_t at = 0;
                while (true) {
                    const size_t comma = list.find(',', at);
                    devices.push_back(std::atoi(list.substr(at, comma - at).c_str()));
                    if (comma == std::string::npos) break;
                    at = comma + 1;
                }
            }
        } else if (a == "-m" || a == "--cudasparememory") {
            parse_double(argc, argv, ++i, &spare);
        } else if (a == "-e" || a == "--byteorder") {
            if (++i < argc && lower(argv[i]) == "bigendian") endian = CTB_BIG_ENDIAN;
        } else if (a == "-j" || a == "--indexorder") {
            if (++i < argc && lower(argv[i]) == "zfastest") order = CTB_Z_FASTEST;
        } else if (a == "-w" || a == "--weights") {
            if (++i < argc) {
                const std::string w = argv[i];
                if (std::count(w.begin(), w.end(), ',') != 1) {
                    std::printf("When using the flag -w you have to specify exactly two coefficients.\n");
                    return 1;
                }
                mp_coef = std::strtod(w.c_str(), nullptr);
                bw_coef = std::strtod(w.c_str() + w.find(',') + 1, nullptr);
            }
        } else if (a == "--precision") {
            if (++i < argc) {
                const std::string p = lower(argv[i]);
                store = p == "fp16" ? CTB_FP16 : p == "bf16" ? CTB_BF16 : CTB_FP32;
            }
        } else if (a == "--pad") {
            if (++i < argc) pad = std::atoi(argv[i]);
        } else if (a == "--slab") {
            if (++i < argc) slab = std::atoi(argv[i]);
        } else if (a == "--grid") {
            if (++i < argc && std::sscanf(argv[i], "%d,%d,%d,%lf", &gx, &gy, &gz, &gvs) != 4) {
                std::printf("--grid expects X,Y,Z,pitch\n");
                return 1;
            }
        } else {
            std::printf("Unknown or misplaced parameter %s.\n", argv[i]);
            return 1;
        }
    }
    if (!have_in || !have_out) {
        std::printf("You must provide a file path to the config file as input as well as a file path for the output.\n");
        return 1;
    }
    if (nocuda) {
        std::printf("CPU reconstruction is not part of this engine; remove -n to reconstruct on the GPU.\n");
        return 1;
    }
    std::printf("\nBeginning reconstruction.\n\tInput:\t\t\t%s\n\tOutput:\t\t\t%s\n\tFilter type:\t\t%s\n",
                input.c_str(), output.c_str(), filter_name.c_str());
    ctb_ctx* ctx = nullptr;
    if (ctb_create(&ctx) != CTB_OK) return 1;
    auto fail = [&](const char* what) {
        std::printf("\n%s: %s\n", what, ctb_last_error(ctx));
        ctb_destroy(ctx);
        return 1;
    };
    ctb_set_progress_callback(ctx, progress, nullptr);
    if (ctb_set_devices(ctx, devices.data(), int(devices.size())) != CTB_OK)
        std::printf("%s\n", ctb_last_error(ctx));  // the previous selection stays, as in the reference
    ctb_set_gpu_coefficients(ctx, mp_coef, bw_coef);
    ctb_set_gpu_spare_memory(ctx, size_t(spare));
    ctb_set_precision(ctx, store);
    if (ctb_set_pad(ctx, pad) != CTB_OK) return fail("pad");
    if (slab > 0) ctb_set_slab_height(ctx, slab);
    if (ctb_load_csv(ctx, input.c_str()) != CTB_OK) return fail("load");
    if (gx > 0 && ctb_set_grid(ctx, gx, gy, gz, float(gvs)) != CTB_OK) return fail("grid");
    if (ctb_set_volume_bounds(ctx, float(xmin), float(xmax), float(ymin), float(ymax), float(zmin), float(zmax)) !=
        CTB_OK)
        std::printf("ERROR: the lower and upper bounds must not be identical.\n");
    int X = 0, Y = 0, Z = 0;
    ctb_get_volume_size(ctx, &X, &Y, &Z);
    std::printf("\nThe resulting volume dimensions will be:\n\n\t%dx%dx%d (x:y:z)\n\n", X, Y, Z);
    ctb_set_filter(ctx, filter);
    if (ctb_reconstruct(ctx) != CTB_OK) return fail("reconstruction");
    ctb_timings t;
    ctb_get_timings(ctx, &t);
    std::printf("Volume successfully reconstructed (%.3fs, %.1f GUPS)\n", t.total_s,
                t.total_s > 0 ? t.voxel_views / t.total_s / 1e9 : 0.0);
    if (ctb_save_volume(ctx, output.c_str(), order, endian) != CTB_OK) return fail("save");
    std::printf("Volume successfully saved.\n");
    ctb_destroy(ctx);
    return 0;
}
