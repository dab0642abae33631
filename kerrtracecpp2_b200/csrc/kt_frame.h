// kt_frame.h -- host-side frame preparation shared by the C ABI layer.
#pragma once

#include <string>

#include "../../include/kerrtrace.h"
#include "kt_machines.cuh"

namespace kt {

double host_r_horizon(const Metric& g);
double host_r_cosmo(const Metric& g);
// rh: host_r_horizon(g)
double host_r_isco(const Metric& g, double rh);

// Validate `d`, apply the reference's fallback rules and clamps, fill the
// kernel constants `f` and (optionally) the public derived record.
kt_status prepare_frame(const kt_frame_desc* d, Frame* f, kt_frame_derived* dv, std::string* err);

ColourConst make_colour(const Frame& f, const kt_color_params& cp);

}  // namespace kt
