/* Stand-in for <opencv2/imgproc.hpp> (see core.hpp in this directory): test infrastructure only. */
#ifndef TDI_REFSTUB_OPENCV_IMGPROC_HPP
#define TDI_REFSTUB_OPENCV_IMGPROC_HPP
#include "core.hpp"
#endif
