// A stand-in for the few parts of OpenCV's cv::Mat that the drop-in headers
// (include/stereo/*.h) use, so their cv::Mat overloads compile and run in a
// test where OpenCV's C++ headers and libraries are absent.  Test
// infrastructure only: 2-D, contiguous, reference-counted by shared_ptr.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#define CV_8U 0
#define CV_16S 3
#define CV_32F 5
#define CV_64F 6
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << 3))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_16SC1 CV_MAKETYPE(CV_16S, 1)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_64FC1 CV_MAKETYPE(CV_64F, 1)

namespace cv {

using uchar = unsigned char;

struct Size {
    int width = 0, height = 0;
    bool operator==(const Size& o) const { return width == o.width && height == o.height; }
    bool operator!=(const Size& o) const { return !(*this == o); }
};

class Mat {
public:
    Mat() = default;
    Mat(int r, int c, int t) { create(r, c, t); }

    void create(int r, int c, int t) {
        if (buf_ && rows == r && cols == c && type_ == t) return;
        rows = r;
        cols = c;
        type_ = t;
        step[0] = (size_t)c * elemSize();
        step[1] = elemSize();
        buf_ = std::make_shared<std::vector<uchar>>((size_t)r * step[0]);
        data = buf_->data();
    }
    Mat clone() const {
        Mat m;
        if (empty()) return m;
        m.create(rows, cols, type_);
        std::memcpy(m.data, data, (size_t)rows * step[0]);
        return m;
    }
    bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
    bool isContinuous() const { return true; }
    int type() const { return type_; }
    int channels() const { return (type_ >> 3) + 1; }
    size_t elemSize() const {
        const int depth = type_ & 7;
        const size_t b = depth == CV_8U ? 1 : depth == CV_16S ? 2 : depth == CV_32F ? 4 : 8;
        return b * channels();
    }
    Size size() const { return Size{cols, rows}; }
    template <typename T> T* ptr(int r = 0) { return reinterpret_cast<T*>(data + (size_t)r * step[0]); }
    template <typename T> const T* ptr(int r = 0) const {
        return reinterpret_cast<const T*>(data + (size_t)r * step[0]);
    }
    template <typename T> T& at(int r, int c) { return ptr<T>(r)[c]; }
    template <typename T> const T& at(int r, int c) const { return ptr<T>(r)[c]; }

    int rows = 0, cols = 0;
    uchar* data = nullptr;
    size_t step[2] = {0, 0};

private:
    int type_ = 0;
    std::shared_ptr<std::vector<uchar>> buf_;
};

// L2 norm of a CV_64FC1 matrix (CameraParams::computeDerivedValues uses it on T)
inline double norm(const Mat& m) {
    double s = 0;
    for (int r = 0; r < m.rows; ++r)
        for (int c = 0; c < m.cols; ++c) s += m.at<double>(r, c) * m.at<double>(r, c);
    return std::sqrt(s);
}

}  // namespace cv
