// Block-list data movement on the device: every re-layout of a site tensor
// (resize, column/row concatenation, zero padding, sector stacking) is a list
// of rectangle copies between two packed slabs, done in one launch.
#pragma once

#include <vector>

#include "common.cuh"

namespace dmrg {

struct RectCopy {
    int64_t src_off;
    int64_t dst_off;
    int src_ld;
    int dst_ld;
    int rows;
    int cols;
    double scale;
};

// dst[dst_off + i*dst_ld + j] = scale * src[src_off + i*src_ld + j] for every task.
// `scratch` keeps the uploaded task list alive until the launch has run.
// Every rectangle is checked against src_size / dst_size (doubles) first.
int launch_rect_copies(const std::vector<RectCopy>& tasks, const double* src, int64_t src_size, double* dst,
                       int64_t dst_size, DeviceBuffer& scratch, cudaStream_t st);

// x *= s (s read on the device)
int launch_scale_by(double* x, int64_t n, const double* s, bool inverse, cudaStream_t st);

}  // namespace dmrg
