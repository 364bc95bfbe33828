/* Stand-in for <opencv2/imgcodecs.hpp> (see core.hpp in this directory): test infrastructure only. */
#ifndef TDI_REFSTUB_OPENCV_IMGCODECS_HPP
#define TDI_REFSTUB_OPENCV_IMGCODECS_HPP
#include "core.hpp"
namespace cv {
inline bool imwrite(const std::string &, const Mat &) { refstub_unreachable(); }
}
#endif
