// The facade's primitive classes used the way NAGA's example programs use
// them: examples/radial_point_interpolation_3d.cu:128-157 (segmentation,
// nearest neighbours, create_interpolator, interpolate) and
// examples/nonlocal_divergence_3d.cu:113-125 (divergence operator create /
// apply, in double), plus the device-pointer forms (caller-owned memory
// wrapped by device_array::view) and the batched inverse on device arrays.
// Writes its results as raw arrays into the directory given as argv[1];
// tests/test_gpu_facade.py compares them with the Python binding and the
// oracle.
#include <naga/naga.hpp>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace {
template <class T>
void dump(const std::string& dir, const char* name, const std::vector<T>& v) {
    FILE* f = std::fopen((dir + "/" + name).c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write output");
    std::fwrite(v.data(), sizeof(T), v.size(), f);
    std::fclose(f);
}

template <class T>
std::vector<T> grid(size_t m, T spacing) {
    std::vector<T> g(3 * m * m * m);
    for (size_t i = 0; i < m * m * m; ++i) {
        g[3 * i + 0] = (T)(i % m) * spacing;
        g[3 * i + 1] = (T)((i / m) % m) * spacing;
        g[3 * i + 2] = (T)(i / (m * m)) * spacing;
    }
    return g;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    const float pi = 3.14159265358979f;

    // ---- radial point interpolation (radial_point_interpolation_3d.cu)
    const unsigned support_size = 32;
    const size_t m = 24, mi = 17;
    const float spacing = 2 * pi / (float)(m - 1), ispacing = 2 * pi / (float)(mi - 1);
    std::vector<float> src = grid<float>(m, spacing), qry = grid<float>(mi, ispacing);
    std::vector<float> values(m * m * m);
    for (size_t i = 0; i < values.size(); ++i)
        values[i] = std::sin(src[3 * i]) * std::cos(src[3 * i + 1]) * src[3 * i + 2];

    // source points in caller-owned device memory, viewed without a copy
    float* raw_src = nullptr;
    if (cudaMalloc((void**)&raw_src, sizeof(float) * src.size()) != cudaSuccess) return 3;
    cudaMemcpy(raw_src, src.data(), sizeof(float) * src.size(), cudaMemcpyHostToDevice);
    auto source_grid = naga::device_array<float>::view(raw_src, src.size());
    auto interp_grid = naga::device_array<float>::from_host(qry);
    auto source_values = naga::device_array<float>::from_host(values);
    naga::device_array<float> interp_values(mi * mi * mi);

    naga::segmentation::nd_cubic_segmentation<float, 3> source_segmentation(source_grid, support_size);
    auto [distances_squared, indices] = naga::segmentation::batched_nearest_neighbors(
        support_size, naga::default_point_map<float, 3>{interp_grid}, source_segmentation);
    auto interpolator = naga::interpolation::radial_point_method<>::create_interpolator<3>(
        source_grid, indices, naga::default_point_map<float, 3>{interp_grid}, spacing);
    interpolator.interpolate(source_values, interp_values).get();
    interpolator.interpolate(source_values, interp_values).get();

    dump(dir, "seg_sizes.u32", source_segmentation.partition_sizes().to_host());
    dump(dir, "seg_indices.u32", source_segmentation.indices().to_host());
    std::vector<float> seg_meta = {source_segmentation.partition_width(), (float)source_segmentation.shape()[0],
                                   (float)source_segmentation.shape()[1], (float)source_segmentation.shape()[2]};
    dump(dir, "seg_meta.f32", seg_meta);
    dump(dir, "knn_idx.u32", indices.to_host());
    dump(dir, "knn_d2.f32", distances_squared.to_host());
    dump(dir, "rpim_weights.f32", interpolator.weights().to_host());
    dump(dir, "rpim_values.f32", interp_values.to_host());

    // a partition's indices through get_partition, against the index list
    {
        auto sizes = source_segmentation.partition_sizes().to_host();
        auto offs = source_segmentation.partition_index_offsets().to_host();
        auto all = source_segmentation.indices().to_host();
        const float probe[3] = {1.0f, 2.0f, 3.0f};
        size_t lin = source_segmentation.linear_index(source_segmentation.get_partition_index(probe));
        auto part = source_segmentation.get_partition(lin);
        if (part.size() != sizes[lin]) return 4;
        for (size_t t = 0; t < part.size(); ++t)
            if (part[t] != all[offs[lin] + t]) return 5;
    }

    // ---- nonlocal divergence (nonlocal_divergence_3d.cu), double and float
    const size_t md = 20;
    const double dspacing = 2 * 3.14159265358979323846 / (double)(md - 1);
    std::vector<double> dgrid = grid<double>(md, dspacing);
    std::vector<double> dvals(dgrid.size());
    for (size_t i = 0; i < md * md * md; ++i) {
        dvals[3 * i + 0] = std::sin(dgrid[3 * i + 0]);
        dvals[3 * i + 1] = 0;
        dvals[3 * i + 2] = std::cos(dgrid[3 * i + 2]);
    }
    auto source_d = naga::device_array<double>::from_host(dgrid);
    auto values_d = naga::device_array<double>::from_host(dvals);
    naga::device_array<double> div_d(md * md * md);
    auto divergence = naga::nonlocal_calculus::divergence_operator<double, 3>::create(source_d);
    divergence.apply(values_d, div_d);
    divergence.apply(values_d, div_d);
    dump(dir, "div_f64.f64", div_d.to_host());
    dump(dir, "div_idx.u32", divergence.support_indices().to_host());
    // the same operator through operator_builder, as NAGA's example builds it
    naga::nonlocal_calculus::operator_builder<double, 3> builder(source_d);
    auto built = builder.create<naga::nonlocal_calculus::divergence_operator>();
    naga::device_array<double> div_b(md * md * md);
    built.apply(values_d, div_b);
    if (div_b.to_host() != div_d.to_host()) return 10;

    std::vector<float> fgrid(dgrid.begin(), dgrid.end()), fvals(dvals.begin(), dvals.end());
    auto source_f = naga::device_array<float>::from_host(fgrid);
    auto values_f = naga::device_array<float>::from_host(fvals);
    naga::device_array<float> div_f(md * md * md);
    auto divergence_f = naga::nonlocal_calculus::divergence_operator<float, 3>::create(source_f);
    divergence_f.apply(values_f, div_f, 0.25f);
    dump(dir, "div_f32_offset.f32", div_f.to_host());
    // override_query_size pads the stencil with zero rows, as NAGA's
    auto padded = naga::nonlocal_calculus::divergence_operator<float, 3>::create(source_f, source_f, md * md * md + 5);
    auto pw = padded.weights().to_host();
    for (size_t i = md * md * md * 32 * 3; i < pw.size(); ++i)
        if (pw[i] != 0.f) return 6;
    bool threw = false;
    try {
        naga::nonlocal_calculus::divergence_operator<float, 3>::create(source_f, interp_grid);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    if (!threw) return 7;

    // ---- batched inverse on device arrays (batched_matrix_inversion.cu:47-70)
    std::vector<double> A = {2, 1, 0, 1, 3, 1, 0, 1, 4};  // symmetric, column-major = row-major
    auto dA = naga::device_array<double>::from_host(A);
    naga::device_array<double> dX(9);
    naga::device_array<int> info(1);
    naga::linalg::batched_matrix_inverse(dA, dX, 3, info).get();
    auto X = dX.to_host();
    if (info.to_host()[0] != 0) return 8;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int t = 0; t < 3; ++t) s += A[i + 3 * t] * X[t + 3 * j];
            if (std::fabs(s - (i == j ? 1.0 : 0.0)) > 1e-12) return 9;
        }

    cudaFree(raw_src);
    std::printf("ok\n");
    return 0;
}
