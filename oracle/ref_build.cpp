// ref_build.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Builds oracle/_ref/libct_ref.so from the reference's own CPU reconstruction
// code: oracle/Makefile cuts these line ranges of Ct/CtVolume.cpp, unchanged,
// into oracle/_ref/*.inc, and this file compiles them as members of a
// stand-in for ct::CtVolume that holds the same data members with the same
// types (Ct/CtVolume.h:218-258) and reads the projections from memory instead
// of image files:
//
//   frag_units.inc     :169-172   FCD and uOffset divided by the pixel size
//   frag_grid.inc      :306-327   relative heights, angle direction, grid
//                                 rule, updateBoundaries, cross-section index
//   frag_radius.inc    :370-373   getReconstructionCylinderRadius
//   frag_bounds.inc    :487-500   setVolumeBounds
//   frag_sinogram.inc  :742-767   makeHeightOffsetRelative, correctAngleDirection
//   frag_preproc.inc   :787-885   prepareProjection, preprocessImage,
//                                 convertTo32bit, applyFeldkampWeight, W,
//                                 applyFourierFilter, applyLogScaling, windows
//   frag_core.inc      :923-1054  reconstructionCore, bilinearInterpolation
//   frag_coords.inc    :1399-1466 updateBoundaries, coordinate transforms
//
// The OpenCV and Qt names those lines use come from ref_shim.h. Only the
// parity tests and bench.py's reference leg load the library.

#include "ref_shim.h"

namespace ct {

#ifdef CTREF_FLOAT_MATH
// The reference calls sqrt, sin and cos unqualified on float arguments (W
// :828-830, the view angle :953-955). Where the float overloads are visible
// in the global namespace (MSVC's <cmath>; libstdc++ once <math.h> is
// included) they resolve to the platform's sqrtf / sinf / cosf. sqrtf is
// correctly rounded everywhere; sinf and cosf are not (glibc's differ from
// the correctly rounded value in the last bit for a few percent of angles,
// and other libraries differ elsewhere), so the stand-ins here return the
// correctly rounded values, which is also what the oracle and the engine use.
inline float sqrt(float x) { return std::sqrt(x); }
inline double sqrt(double x) { return std::sqrt(x); }
inline float sin(float x) { return float(std::sin(double(x))); }
inline double sin(double x) { return std::sin(x); }
inline float cos(float x) { return float(std::cos(double(x))); }
inline double cos(double x) { return std::cos(x); }
#endif

enum class FilterType { RAMLAK, SHEPP_LOGAN, HANN };
enum class Axis { X, Y, Z };

// Volume<float> as the CPU path uses it: Z_FASTEST storage, slicePtr(x) the
// start of the y-z plane of x (Common/Volume.h:313-316).
template <typename T>
class Volume {
public:
    void reinitialise(size_t x, size_t y, size_t z, T v) {
        xs_ = x;
        ys_ = y;
        zs_ = z;
        data_.assign(x * y * z, v);
    }
    T* slicePtr(size_t outer) { return data_.data() + outer * ys_ * zs_; }
    T* data() { return data_.data(); }
    size_t size() const { return data_.size(); }

private:
    size_t xs_ = 0, ys_ = 0, zs_ = 0;
    std::vector<T> data_;
};

class CtVolume {
public:
    struct Projection {
        QString imagePath;
        double angle;
        double heightOffset;
        // the image in memory instead of on disk
        const void* pixels = nullptr;
        int depth = CV_16U, rows = 0, cols = 0;
        cv::Mat getImage() const {
            cv::Mat m(rows, cols, depth);
            const size_t bytes = size_t(rows) * cols * (depth == CV_8U ? 1 : depth == CV_16U ? 2 : 4);
            std::memcpy(m.data, pixels, bytes);
            return m;
        }
    };

    // ------------------------------------------------ the reference's lines
    unsigned int getReconstructionCylinderRadius() const;
    void setVolumeBounds(float xFrom, float xTo, float yFrom, float yTo, float zFrom, float zTo);
    void makeHeightOffsetRelative();
    void correctAngleDirection(std::string rotationDirection);
    cv::Mat prepareProjection(unsigned int index, bool multithreading = false) const;
    void preprocessImage(cv::Mat& image, bool multithreading = false) const;
    void convertTo32bit(cv::Mat& img) const;
    void applyFeldkampWeight(cv::Mat& image, bool multithreading = false) const;
    static float W(float D, float u, float v);
    static void applyFourierFilter(cv::Mat& image, FilterType filterType, bool multithreading = false);
    void applyLogScaling(cv::Mat& image) const;
    static float ramLakWindowFilter(float n, float N);
    static float sheppLoganWindowFilter(float n, float N);
    static float hannWindowFilter(float n, float N);
    bool reconstructionCore();
    static float bilinearInterpolation(float u, float v, float u0v0, float u1v0, float u0v1, float u1v1);
    void updateBoundaries();
    float worldToVolumeX(float xCoord) const;
    float worldToVolumeY(float yCoord) const;
    float worldToVolumeZ(float zCoord) const;
    float volumeToWorldX(float xCoord) const;
    float volumeToWorldY(float yCoord) const;
    float volumeToWorldZ(float zCoord) const;
    float imageToMatU(float uCoord) const;
    float imageToMatV(float vCoord) const;
    float matToImageU(float uCoord) const;
    float matToImageV(float vCoord) const;

    // ------------------------------------------------ the load sequence
    // sinogramFromImages after the CSV header was read (:169-172) and after
    // the images were checked (:306-327), in the reference's order.
    void convert_units() {
#include "frag_units.inc"
    }
    void finish_loading(std::string rotationDirection) {
#include "frag_grid.inc"
    }

    // Qt signal and preview stand-ins (never reached: emitSignals is false)
    cv::Mat getVolumeCrossSection(Axis, unsigned int) const { return cv::Mat(); }
    void reconstructionProgress(double, cv::Mat) const {}

    // ------------------------------------------------ data members (types of Ct/CtVolume.h:218-258)
    std::vector<Projection> sinogram;
    unsigned int xSize = 0, ySize = 0, zSize = 0;
    unsigned int imageWidth = 0, imageHeight = 0;
    int imageType;
    float FCD = 0;
    float pixelSize = 0;
    float uOffset = 0;
    float baseIntensity = 0;
    FilterType filterType = FilterType::RAMLAK;
    unsigned int projectionStep = 1;
    bool emitSignals = false;
    unsigned int crossSectionIndex = 0;
    Axis crossSectionAxis = Axis::Z;
    mutable std::atomic<bool> stopActiveProcess{false};
    float xFrom_float = 0, xTo_float = 1;
    float yFrom_float = 0, yTo_float = 1;
    float zFrom_float = 0, zTo_float = 1;
    Volume<float> volume;
    unsigned int xFrom = 0, xTo = 0;
    unsigned int yFrom = 0, yTo = 0;
    unsigned int zFrom = 0, zTo = 0;
    unsigned int xMax = 0, yMax = 0, zMax = 0;
    mutable std::mutex exclusiveFunctionsMutex;
    std::string lastErrorMessage;
    float xPrecomputed;
    float yPrecomputed;
    float zPrecomputed;
    float uPrecomputed;
    float vPrecomputed;
};

#include "frag_radius.inc"
#include "frag_bounds.inc"
#include "frag_sinogram.inc"
#include "frag_preproc.inc"
#include "frag_core.inc"
#include "frag_coords.inc"

}  // namespace ct

namespace {

// The reference's console output (progress lines) is not wanted in tests.
struct QuietCout {
    std::streambuf* old;
    std::ofstream null;
    QuietCout() : old(std::cout.rdbuf()), null("/dev/null") { std::cout.rdbuf(null.rdbuf()); }
    ~QuietCout() { std::cout.rdbuf(old); }
};

int cv_depth(int bits) { return bits == 8 ? CV_8U : bits == 16 ? CV_16U : CV_32F; }

// Loads a scan the way sinogramFromImages does once the CSV was parsed.
void load(ct::CtVolume& c, const void* images, int bits, int n, int W, int H, const double* angles_deg,
          const double* heights_mm, double pixel_size, double u_offset_mm, double fcd_mm, double base,
          const char* rotation) {
    c.pixelSize = float(pixel_size);
    c.uOffset = float(u_offset_mm);
    c.FCD = float(fcd_mm);
    c.baseIntensity = float(base);
    c.convert_units();
    const size_t bytes = size_t(W) * H * (bits == 8 ? 1 : bits == 16 ? 2 : 4);
    for (int i = 0; i < n; ++i) {
        ct::CtVolume::Projection p;
        p.imagePath = QString("projection " + std::to_string(i));
        p.angle = angles_deg[i];
        p.heightOffset = heights_mm ? heights_mm[i] : 0.0;
        p.pixels = static_cast<const unsigned char*>(images) + bytes * i;
        p.depth = cv_depth(bits);
        p.rows = H;
        p.cols = W;
        c.sinogram.push_back(p);
    }
    c.imageWidth = unsigned(W);
    c.imageHeight = unsigned(H);
    c.imageType = cv_depth(bits);
    c.finish_loading(rotation);
}

}  // namespace

extern "C" {

// Whole CPU reconstruction through the reference's own code: load (units,
// relative heights in mm, angle direction "cw"/"ccw", grid rule), bounds
// rel6 = {xmin, xmax, ymin, ymax, zmin, zmax} (NULL: whole grid), filter
// 0/1/2, skip projections, then reconstructionCore into a Z_FASTEST volume.
// dims receives xMax, yMax, zMax. With vol == NULL and run == 0 only dims are
// set; with vol == NULL and run != 0 the reconstruction runs and its volume is
// dropped. seconds: steady-clock time of what reconstructVolume does for the
// CPU path (:553-573): the zeroed volume (reinitialise) and reconstructionCore.
// Returns 0 on success.
int ref_reconstruct(const void* images, int bits, int n_views, int W, int H, const double* angles_deg,
                    const double* heights_mm, double pixel_size, double u_offset_mm, double fcd_mm, double base,
                    const char* rotation, const float* rel6, int filter, unsigned skip, float* vol, int* dims,
                    double* seconds, int run) {
    QuietCout quiet;
    ct::CtVolume c;
    try {
        load(c, images, bits, n_views, W, H, angles_deg, heights_mm, pixel_size, u_offset_mm, fcd_mm, base,
             rotation);
        if (rel6) c.setVolumeBounds(rel6[0], rel6[1], rel6[2], rel6[3], rel6[4], rel6[5]);
        c.filterType = ct::FilterType(filter);
        c.projectionStep = skip + 1;   // setSkipProjections (:539-541)
        dims[0] = int(c.xMax);
        dims[1] = int(c.yMax);
        dims[2] = int(c.zMax);
        if (!vol && !run) return 0;
        const auto t0 = std::chrono::steady_clock::now();
        c.volume.reinitialise(c.xMax, c.yMax, c.zMax, 0);
        const bool ok = c.reconstructionCore();
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        if (!ok) return 2;
        if (vol) std::memcpy(vol, c.volume.data(), c.volume.size() * sizeof(float));
    } catch (const std::exception&) {
        return 1;
    }
    return 0;
}

// The reference's preprocessing of one projection (prepareProjection:
// convertTo32bit, applyLogScaling, applyFeldkampWeight, applyFourierFilter)
// for a scan loaded as in ref_reconstruct; out: H x W floats.
int ref_prepare_projection(const void* images, int bits, int n_views, int W, int H, const double* angles_deg,
                           double pixel_size, double fcd_mm, double base, int filter, int index, float* out) {
    QuietCout quiet;
    ct::CtVolume c;
    try {
        load(c, images, bits, n_views, W, H, angles_deg, nullptr, pixel_size, 0.0, fcd_mm, base, "ccw");
        c.filterType = ct::FilterType(filter);
        cv::Mat m = c.prepareProjection(unsigned(index), false);
        std::memcpy(out, m.data, size_t(W) * H * sizeof(float));
    } catch (const std::exception&) {
        return 1;
    }
    return 0;
}

// Corrected angles (degrees) and relative height offsets (pixels) after the
// reference's makeHeightOffsetRelative and correctAngleDirection.
int ref_fix_sinogram(int n_views, const double* angles_deg, const double* heights_mm, double pixel_size,
                     const char* rotation, double* angles_out, double* heights_px_out) {
    ct::CtVolume c;
    c.pixelSize = float(pixel_size);
    for (int i = 0; i < n_views; ++i) {
        ct::CtVolume::Projection p;
        p.angle = angles_deg[i];
        p.heightOffset = heights_mm ? heights_mm[i] : 0.0;
        c.sinogram.push_back(p);
    }
    c.makeHeightOffsetRelative();
    c.correctAngleDirection(rotation);
    for (int i = 0; i < n_views; ++i) {
        angles_out[i] = c.sinogram[i].angle;
        heights_px_out[i] = c.sinogram[i].heightOffset;
    }
    return 0;
}

}  // extern "C"
