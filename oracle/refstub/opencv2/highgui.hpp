/* Stand-in for <opencv2/highgui.hpp> (see core.hpp in this directory): test infrastructure only. */
#ifndef TDI_REFSTUB_OPENCV_HIGHGUI_HPP
#define TDI_REFSTUB_OPENCV_HIGHGUI_HPP
#include "core.hpp"
namespace cv {
inline void imshow(const std::string &, const Mat &) { refstub_unreachable(); }
inline int waitKey(int = 0) { refstub_unreachable(); }
}
#endif
