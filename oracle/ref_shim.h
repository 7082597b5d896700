// ref_shim.h -- TEST INFRASTRUCTURE ONLY.
//
// The few OpenCV and Qt names that the reference's CPU reconstruction path
// (Ct/CtVolume.cpp) touches, written here from their documented behaviour so
// that those source lines compile unchanged without OpenCV 3.1 and Qt 5,
// which this machine does not have. ref_build.cpp includes the reference's
// lines (cut out of Ct/CtVolume.cpp by oracle/Makefile into oracle/_ref/)
// after this header and builds oracle/_ref/libct_ref.so, the reference's own
// loops run as the oracle's pin.
//
// What the shims stand for (third-party arithmetic, restated):
//  * cv::Mat: a 2-D single-channel (or 2-channel float) image with row
//    pointers, Mat::convertTo(dst, CV_32F, alpha, beta) for 8U/16U input with
//    a float working type (dst = float(src) * float(alpha) + float(beta)), and
//    Mat *= s (dst = src * float(s)), as OpenCV's cvtScale does for float.
//  * cv::dft(DFT_COMPLEX_OUTPUT | DFT_ROWS): the full complex spectrum of
//    each row, computed in double and rounded to float; cv::idft(DFT_ROWS |
//    DFT_REAL_OUTPUT): the unnormalised inverse of the Hermitian spectrum given
//    by bins 0..W/2 (bins above W/2 ignored), computed in double and rounded to
//    float. Both pinned against cv2 by the fixtures in tests/golden.
//  * cv::log: the natural logarithm of each float sample (OpenCV's differs
//    from the correctly rounded one by at most 2 ulp, pinned in tests/golden).
//  * cv::Vec2f *= float: each component times the float factor.
//  * QString: a std::string holder with toStdString().
//  * Qt's `emit`: an empty macro, as in Qt.
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <chrono>
#include <ctime>
#include <fstream>
#include <future>
#include <iostream>
#include <memory>
#include <mutex>
#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

#define emit

#define CV_8U 0
#define CV_16U 2
#define CV_32F 5
#define CV_32FC1 5
#define CV_32FC2 13
#define CV_Assert(expr)                                                              \
    do {                                                                             \
        if (!(expr)) throw std::runtime_error("assertion failed: " #expr);           \
    } while (0)

namespace cv {

enum { DFT_INVERSE = 1, DFT_ROWS = 4, DFT_COMPLEX_OUTPUT = 16, DFT_REAL_OUTPUT = 32 };

template <typename T, int n>
struct Vec {
    T val[n];
    T& operator[](int i) { return val[i]; }
    const T& operator[](int i) const { return val[i]; }
};
template <typename T, int n>
inline Vec<T, n>& operator*=(Vec<T, n>& a, float alpha) {
    for (int i = 0; i < n; ++i) a.val[i] = T(a.val[i] * alpha);
    return a;
}
typedef Vec<float, 2> Vec2f;

class Mat {
public:
    int rows = 0, cols = 0;
    unsigned char* data = nullptr;

    Mat() {}
    Mat(int r, int c, int type) { create(r, c, type); }

    void create(int r, int c, int type) {
        rows = r;
        cols = c;
        type_ = type;
        buf_ = std::make_shared<std::vector<unsigned char>>(size_t(r) * c * elem_size(type));
        data = buf_->data();
    }
    int type() const { return type_; }
    int depth() const { return type_ & 7; }
    int channels() const { return (type_ >> 3) + 1; }
    size_t step() const { return size_t(cols) * elem_size(type_); }
    template <typename T>
    T* ptr(int r) { return reinterpret_cast<T*>(data + size_t(r) * step()); }
    template <typename T>
    const T* ptr(int r) const { return reinterpret_cast<const T*>(data + size_t(r) * step()); }

    // 8U / 16U / 32F -> 32F with scale and shift (float working type)
    void convertTo(Mat& dst, int rtype, double alpha = 1.0, double beta = 0.0) const {
        CV_Assert(rtype == CV_32F && channels() == 1);
        Mat out(rows, cols, CV_32F);
        const float a = float(alpha), b = float(beta);
        const size_t n = size_t(rows) * cols;
        float* o = reinterpret_cast<float*>(out.data);
        for (size_t i = 0; i < n; ++i) {
            float s;
            if (depth() == CV_8U) s = float(data[i]);
            else if (depth() == CV_16U) s = float(reinterpret_cast<const uint16_t*>(data)[i]);
            else s = reinterpret_cast<const float*>(data)[i];
            o[i] = s * a + b;
        }
        dst = out;
    }
    Mat& operator*=(double s) {
        CV_Assert(depth() == CV_32F);
        const float f = float(s);
        const size_t n = size_t(rows) * cols * channels();
        float* p = reinterpret_cast<float*>(data);
        for (size_t i = 0; i < n; ++i) p[i] = p[i] * f;
        return *this;
    }

private:
    static size_t elem_size(int type) {
        const int d = type & 7, cn = (type >> 3) + 1;
        return size_t(cn) * (d == CV_8U ? 1 : d == CV_16U ? 2 : 4);
    }
    int type_ = -1;
    std::shared_ptr<std::vector<unsigned char>> buf_;
};

namespace detail {
using cd = std::complex<double>;

// Unnormalised DFT of one sequence (forward sign -1, inverse +1): radix-2
// for powers of two, Bluestein's chirp-z transform for other lengths. Tables
// are built once per length and thread.
struct Pow2Plan {
    std::vector<cd> tw;            // exp(-2 pi i k / n), k < n/2
    std::vector<uint32_t> rev;     // bit reversal
    explicit Pow2Plan(size_t n) : tw(n / 2), rev(n) {
        for (size_t k = 0; k < n / 2; ++k) tw[k] = std::polar(1.0, -2.0 * M_PI * double(k) / double(n));
        for (size_t i = 1, j = 0; i < n; ++i) {
            size_t bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            rev[i] = uint32_t(j);
        }
    }
    void run(cd* a, size_t n, bool inverse) const {
        for (size_t i = 1; i < n; ++i)
            if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        for (size_t len = 2; len <= n; len <<= 1) {
            const size_t half = len / 2, stride = n / len;
            for (size_t i = 0; i < n; i += len)
                for (size_t k = 0; k < half; ++k) {
                    const cd w = inverse ? std::conj(tw[k * stride]) : tw[k * stride];
                    const cd u = a[i + k], v = a[i + k + half] * w;
                    a[i + k] = u + v;
                    a[i + k + half] = u - v;
                }
        }
    }
};

struct Plan {
    size_t n = 0, m = 0;
    std::shared_ptr<Pow2Plan> p2;
    std::vector<cd> chirp, bfft;   // Bluestein: exp(-i pi k^2 / n) and the FFT of its conjugate
    explicit Plan(size_t n_) : n(n_) {
        if (n && !(n & (n - 1))) {
            m = n;
            p2 = std::make_shared<Pow2Plan>(n);
            return;
        }
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
        p2 = std::make_shared<Pow2Plan>(m);
        chirp.resize(n);
        for (size_t k = 0; k < n; ++k)
            chirp[k] = std::polar(1.0, -M_PI * double((unsigned long long)k * k % (2ull * n)) / double(n));
        bfft.assign(m, cd(0, 0));
        bfft[0] = std::conj(chirp[0]);
        for (size_t k = 1; k < n; ++k) bfft[k] = bfft[m - k] = std::conj(chirp[k]);
        p2->run(bfft.data(), m, false);
    }
    void run(std::vector<cd>& x, bool inverse) const {
        if (m == n) {
            p2->run(x.data(), n, inverse);
            return;
        }
        if (inverse)
            for (auto& v : x) v = std::conj(v);
        std::vector<cd> a(m, cd(0, 0));
        for (size_t k = 0; k < n; ++k) a[k] = x[k] * chirp[k];
        p2->run(a.data(), m, false);
        for (size_t k = 0; k < m; ++k) a[k] *= bfft[k];
        p2->run(a.data(), m, true);
        for (size_t k = 0; k < n; ++k) x[k] = a[k] * chirp[k] / double(m);
        if (inverse)
            for (auto& v : x) v = std::conj(v);
    }
};

inline void dft_any(std::vector<cd>& x, bool inverse) {
    thread_local std::vector<std::shared_ptr<Plan>> plans;
    std::shared_ptr<Plan> plan;
    for (auto& p : plans)
        if (p->n == x.size()) plan = p;
    if (!plan) {
        plan = std::make_shared<Plan>(x.size());
        plans.push_back(plan);
    }
    plan->run(x, inverse);
}
}  // namespace detail

inline void dft(const Mat& src, Mat& dst, int flags) {
    CV_Assert(src.depth() == CV_32F && src.channels() == 1 && (flags & DFT_COMPLEX_OUTPUT) && (flags & DFT_ROWS));
    Mat out(src.rows, src.cols, CV_32FC2);
    std::vector<detail::cd> x(src.cols);
    for (int r = 0; r < src.rows; ++r) {
        const float* in = src.ptr<float>(r);
        for (int c = 0; c < src.cols; ++c) x[c] = detail::cd(in[c], 0.0);
        detail::dft_any(x, false);
        float* o = out.ptr<float>(r);
        for (int c = 0; c < src.cols; ++c) {
            o[2 * c] = float(x[c].real());
            o[2 * c + 1] = float(x[c].imag());
        }
    }
    dst = out;
}

inline void idft(const Mat& src, Mat& dst, int flags) {
    CV_Assert(src.depth() == CV_32F && src.channels() == 2 && (flags & DFT_REAL_OUTPUT) && (flags & DFT_ROWS));
    const int W = src.cols;
    Mat out(src.rows, W, CV_32F);
    std::vector<detail::cd> x(W);
    for (int r = 0; r < src.rows; ++r) {
        const float* in = src.ptr<float>(r);
        // Hermitian spectrum from bins 0..W/2
        for (int k = 0; k <= W / 2; ++k) x[k] = detail::cd(in[2 * k], in[2 * k + 1]);
        x[0] = detail::cd(x[0].real(), 0.0);
        if (W % 2 == 0) x[W / 2] = detail::cd(x[W / 2].real(), 0.0);
        for (int k = 1; k < (W + 1) / 2; ++k) x[W - k] = std::conj(x[k]);
        detail::dft_any(x, true);
        float* o = out.ptr<float>(r);
        for (int c = 0; c < W; ++c) o[c] = float(x[c].real());
    }
    dst = out;
}

inline void log(const Mat& src, Mat& dst) {
    CV_Assert(src.depth() == CV_32F);
    Mat out(src.rows, src.cols, src.type());
    const size_t n = size_t(src.rows) * src.cols * src.channels();
    const float* s = reinterpret_cast<const float*>(src.data);
    float* o = reinterpret_cast<float*>(out.data);
    for (size_t i = 0; i < n; ++i) o[i] = std::log(s[i]);
    dst = out;
}

}  // namespace cv

class QString {
public:
    QString() {}
    QString(const std::string& s) : s_(s) {}
    std::string toStdString() const { return s_; }

private:
    std::string s_;
};
