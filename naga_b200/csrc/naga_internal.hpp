// Internal host-side declarations shared by the translation units of
// libnaga_b200.so.
#pragma once
#include "naga_b200.h"

#include <cstdint>
#include <string>
#include <vector>

namespace naga {

// thread-local error message; returns rc so callers can `return set_error(..)`
int set_error(int rc, const std::string& msg);
void clear_error();

struct GridScene {
    int dim = 0;
    double h = 0;
    int64_t n_bulk = 0, n_layer = 0, n_boundary = 0;
    std::vector<float> points;   // [N][dim]
    std::vector<float> normals;  // [n_boundary][dim]
    std::vector<float> sigma;    // [n_layer]
    std::vector<int64_t> grid_index;
};

int build_grid_scene(const naga_grid_spec& spec, GridScene& out);
int build_box_scene(const naga_box_grid_spec& spec, GridScene& out);

}  // namespace naga
