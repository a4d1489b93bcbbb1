// Host helpers shared by the C-ABI translation units (definitions in krr_abi.cu): the
// reference's argument validation, parameter packing and launch-shape selection.
#pragma once

#include "../../include/kerrray_cuda.h"
#include "krr_launch.h"

namespace krr_host {

int fail(int code, const char* fmt, ...);
int validate_options(const krr_options* o);
int validate_spacetime(double mass, double spin);
int validate_grid(const krr_camera* c);
int pixel_range(const krr_image& im, long long* first, long long* count);
int check_precision(int32_t precision, const krr_options* o);
krr::Params make_params(double mass, double spin, const krr_options* o);
int make_frame(double mass, double spin, const krr_camera* c, krr::Frame& F);
krr::Outputs to_outputs(const krr_result* r);
const krr::Variant* variants_for(int32_t precision, const krr_options* o, int* count);
int sm_count_of(int device);

}  // namespace krr_host
