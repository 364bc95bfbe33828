/*
 * Stand-in for the OpenCV headers that 3DI's hot-path sources include (funcs.h, newfuncs.h,
 * config.h). TEST INFRASTRUCTURE ONLY: it lets the reference's own kernels compile for the
 * oracle's pinning build (oracle/_ref/) without OpenCV, which is not installed here.
 *
 * Those files use OpenCV only in host helpers that show or save images
 * (funcs.cu:1137-1247) and in eulerAnglesToRotationMatrix (newfuncs.cu:720-747); the pinning
 * driver calls none of them. Every function below therefore only has to compile: each one
 * aborts if it is ever reached.
 */
#ifndef TDI_REFSTUB_OPENCV_CORE_HPP
#define TDI_REFSTUB_OPENCV_CORE_HPP

#include <cstdlib>
#include <string>
#include <vector>   /* the real header brings in <vector>; config.h relies on it */

#define CV_32F 5

namespace cv {

[[noreturn]] inline void refstub_unreachable() { std::abort(); }

struct Scalar {
    double v[4];
    static Scalar all(double) { refstub_unreachable(); }
};

struct Rect {
    int x, y, width, height;
    Rect(int x_, int y_, int w_, int h_) : x(x_), y(y_), width(w_), height(h_) {}
};

class Mat {
public:
    int rows = 0, cols = 0;
    unsigned char *data = nullptr;
    Mat() {}
    Mat(int, int, int) { refstub_unreachable(); }
    Mat(int, int, int, const Scalar &) { refstub_unreachable(); }
    Mat t() const { refstub_unreachable(); }
    Mat operator()(const Rect &) const { refstub_unreachable(); }
    /* OpenCV takes an output proxy that binds to temporaries such as m(rect) */
    void copyTo(const Mat &) const { refstub_unreachable(); }
    Mat &setTo(const Scalar &) { refstub_unreachable(); }
};

inline Mat operator-(const Mat &, double) { refstub_unreachable(); }
inline Mat operator/(const Mat &, double) { refstub_unreachable(); }
inline Mat operator*(double, const Mat &) { refstub_unreachable(); }
inline Mat operator*(float, const Mat &) { refstub_unreachable(); }
inline Mat operator*(const Mat &, const Mat &) { refstub_unreachable(); }

template <typename T>
class Mat_ : public Mat {
public:
    struct Init {
        template <typename U> Init &operator,(const U &) { return *this; }
        operator Mat() const { refstub_unreachable(); }
    };
    Mat_(int, int) { refstub_unreachable(); }
    template <typename U> Init operator<<(const U &) { refstub_unreachable(); }
};

template <typename T, int n>
struct Vec {
    T val[n];
    T &operator[](int i) { return val[i]; }
    const T &operator[](int i) const { return val[i]; }
};
typedef Vec<float, 3> Vec3f;

inline void minMaxLoc(const Mat &, double *, double *) { refstub_unreachable(); }
inline void transpose(const Mat &, Mat &) { refstub_unreachable(); }

}  // namespace cv

#endif
