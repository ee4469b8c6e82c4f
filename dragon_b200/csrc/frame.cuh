// Enumeration of the ghost frame of a padded 2D array: the points of the
// padded index range outside a box. The 2D MHD step copies its output
// buffers' frame (mhd2d_copy_frame, step_mhd.cuh) instead of whole arrays.
// Plain C++ like fluid.cuh, so the CPU test suite compiles the same code.
#pragma once

#include "fluid.cuh"

namespace dgpu {

// Point k of the frame of the box [bi0, bi1) x [bj0, bj1) inside the padded
// range [lo_i, hi_i) x [lo_j, hi_j): the rows above and below the box, then
// the columns left and right of it. False past the last point.
DHD bool frame_point(long long k, int lo_i, int hi_i, int lo_j, int hi_j, int bi0, int bi1, int bj0, int bj1, int& i,
                     int& j) {
    const long long W = hi_j - lo_j;
    const long long top = (long long)(bi0 - lo_i) * W;
    if (k < top) {
        i = lo_i + (int)(k / W);
        j = lo_j + (int)(k % W);
        return true;
    }
    k -= top;
    const long long bot = (long long)(hi_i - bi1) * W;
    if (k < bot) {
        i = bi1 + (int)(k / W);
        j = lo_j + (int)(k % W);
        return true;
    }
    k -= bot;
    const int sl = bj0 - lo_j, side = sl + (hi_j - bj1);
    if (side <= 0 || k >= (long long)(bi1 - bi0) * side) return false;
    i = bi0 + (int)(k / side);
    const int c = (int)(k % side);
    j = c < sl ? lo_j + c : bj1 + (c - sl);
    return true;
}

DHD long long frame_count(int lo_i, int hi_i, int lo_j, int hi_j, int bi0, int bi1, int bj0, int bj1) {
    return (long long)(hi_i - lo_i) * (hi_j - lo_j) - (long long)(bi1 - bi0) * (bj1 - bj0);
}

// Frame points of the cells and of the three face-B components, in that order.
DHD long long mhd2d_frame_points(long long nx, long long ny, long long g) {
    const long long cells = (nx + 2 * g) * (ny + 2 * g) - nx * ny;
    const long long faces = (nx + 1 + 2 * g) * (ny + 1 + 2 * g);
    return cells + (faces - (nx + 1) * ny) + (faces - nx * (ny + 1)) + (faces - nx * ny);
}

}  // namespace dgpu
