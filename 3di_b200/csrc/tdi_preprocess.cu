// Device preprocessing of raw video frames into the fitting crops: the steps of
// InputData::get_resized_frame (input_data.cu:43-53) and of the crop in
// VideoFitter::fit_to_video_frame (video_fitter.cu:537-550), fused per crop pixel.
//
// The reference runs them through OpenCV 4 on the host:
//   cv::cvtColor(frame, gray, cv::COLOR_BGR2GRAY)  8-bit: (3735 B + 19235 G + 9798 R + 2^14) >> 15
//   gray.convertTo(gray, CV_32FC1); gray /= 255    convertTo with scale: v * (float)(1/255.)
//   cv::resize(gray, gray, Size(), c, c)           INTER_LINEAR on floats (OpenCV's own code)
//   cv::copyMakeBorder(..., 0, DIMY, 0, DIMX, ...)  zeros right and below
//   gray(Rect(x0, y0, 256, 256)).t()               the crop, column-major (x * 256 + y)
// The bilinear resize follows OpenCV's generic path: for destination column X,
// fx = (float)((X + 0.5) / c - 0.5) (double arithmetic), sx = floor(fx), weights 1 - fx and
// fx as floats; columns left of the image use sx = 0 with weight 0 on the second tap, columns
// at or past the last source column take that column alone; rows use the same coordinate
// with both row indices clamped to the image and the weights left as computed. Each pass is
// two float products and one float sum, in that order. (OpenCV built with Intel IPP takes
// IPP's resize instead, whose rounding differs by up to a few units in the last place.)

namespace tdi {

constexpr int PP_TILE = 32;                 // crop tile of 32 x 32 pixels per block
constexpr int PP_ROWS = 8;                  // block of 32 x 8 threads

struct PrepFrame {
    const uint8_t *bgr;                     // device copy of the image
    int64_t row_bytes;
    int32_t width, height;                  // source size
    int32_t rw, rh;                         // resized size (OpenCV's rounding)
    double inv;                             // 1 / resize coefficient
    int32_t x0, y0;                         // crop origin in the resized image
};

__device__ __forceinline__ float gray_at(const PrepFrame &p, int r, int c)
{
    const uint8_t *q = p.bgr + (size_t)r * p.row_bytes + 3 * (size_t)c;
    const uint32_t y8 = ((uint32_t)q[0] * 3735u + (uint32_t)q[1] * 19235u + (uint32_t)q[2] * 9798u + 16384u) >> 15;
    return (float)y8 * (float)(1.0 / 255.0);
}

// Resized image value at (X, Y), X < rw, Y < rh.
__device__ float resized_at(const PrepFrame &p, int X, int Y)
{
    float fx = (float)(((double)X + 0.5) * p.inv - 0.5);
    int sx = (int)floorf(fx);
    fx -= (float)sx;
    bool single = false;
    if (sx < 0) { fx = 0.0f; sx = 0; }
    if (sx + 1 >= p.width) { single = true; fx = 0.0f; sx = p.width - 1; }
    const float a0 = 1.0f - fx, a1 = fx;
    float fy = (float)(((double)Y + 0.5) * p.inv - 0.5);
    const int sy = (int)floorf(fy);
    fy -= (float)sy;
    const float b0 = 1.0f - fy, b1 = fy;
    const int r0 = sy < 0 ? 0 : (sy < p.height ? sy : p.height - 1);
    const int r1 = sy + 1 < 0 ? 0 : (sy + 1 < p.height ? sy + 1 : p.height - 1);
    float h[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int r = k == 0 ? r0 : r1;
        if (single) {
            h[k] = gray_at(p, r, sx);
        } else {
            const float t0 = gray_at(p, r, sx) * a0;
            const float t1 = gray_at(p, r, sx + 1) * a1;
            h[k] = t0 + t1;
        }
    }
    const float u0 = h[0] * b0, u1 = h[1] * b1;
    return u0 + u1;
}

// One 32 x 32 tile of one frame's crop: values formed along image rows, written along the
// crop's columns (the crop is stored x-major) through a shared-memory transpose.
__global__ void __launch_bounds__(PP_TILE * PP_ROWS) k_preprocess(const PrepFrame *frames, float *targets)
{
    const PrepFrame p = frames[blockIdx.z];
    __shared__ float tile[PP_TILE][PP_TILE + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int xb = blockIdx.x * PP_TILE, yb = blockIdx.y * PP_TILE;
    for (int j = ty; j < PP_TILE; j += PP_ROWS) {
        const int X = p.x0 + xb + tx, Y = p.y0 + yb + j;   // in the padded resized image
        tile[j][tx] = (X < p.rw && Y < p.rh) ? resized_at(p, X, Y) : 0.0f;
    }
    __syncthreads();
    float *out = targets + (size_t)blockIdx.z * NPIX;
    for (int j = ty; j < PP_TILE; j += PP_ROWS) out[(size_t)(xb + j) * DIM + yb + tx] = tile[tx][j];
}

}  // namespace tdi
