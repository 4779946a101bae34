// Exercises include/cbct_gadgetron.hpp the way xray/cuCBOS_reconstruct.cpp uses
// CBSubsetOperator: setup on an acquisition, mult_M / mult_MH over all subsets,
// and the device-resident OS-MOM solve.  Inputs and outputs are raw float32
// files; tests/test_dropin.py checks them against the FP64 oracle.
//
// usage: dropin_main <io_dir> nx ny nz lx ly lz W H fov_u fov_v SAD SDD P subsets
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "cbct_gadgetron.hpp"

using namespace Gadgetron;

static std::vector<float> read_f32(const std::string& path, size_t n) {
  std::vector<float> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(float));
  if (!f) throw std::runtime_error("cannot read " + path);
  return v;
}

static void write_f32(const std::string& path, const float* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), n * sizeof(float));
}

static void download(const cuNDArray<float>& a, std::vector<float>& h) {
  h.resize(a.get_number_of_elements());
  if (cudaMemcpy(h.data(), a.get_data_ptr(), a.bytes(), cudaMemcpyDeviceToHost) != cudaSuccess)
    throw std::runtime_error("cudaMemcpy failed");
}

int main(int argc, char** argv) {
  if (argc != 16) {
    std::fprintf(stderr, "usage: %s io_dir nx ny nz lx ly lz W H fov_u fov_v SAD SDD P subsets\n", argv[0]);
    return 2;
  }
  try {
    const std::string dir = argv[1];
    const size_t nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]);
    const floatd3 L(std::atof(argv[5]), std::atof(argv[6]), std::atof(argv[7]));
    const size_t W = std::atoi(argv[8]), H = std::atoi(argv[9]);
    const floatd2 fov(std::atof(argv[10]), std::atof(argv[11]));
    const float SAD = std::atof(argv[12]), SDD = std::atof(argv[13]);
    const size_t P = std::atoi(argv[14]);
    const int subsets = std::atoi(argv[15]);

    auto acq = boost::make_shared<CBCT_acquisition>();
    auto geo = acq->get_geometry();
    geo->set_SAD(SAD);
    geo->set_SDD(SDD);
    geo->set_FOV(fov);
    std::vector<float> ang = read_f32(dir + "/angles.f32", P);
    std::vector<float> off = read_f32(dir + "/offsets.f32", 2 * P);
    std::vector<floatd2> offsets(P);
    for (size_t i = 0; i < P; ++i) offsets[i] = floatd2(off[2 * i], off[2 * i + 1]);
    geo->set_angles(ang);
    geo->set_offsets(offsets);
    auto proj = boost::make_shared<hoCuNDArray<float>>(std::vector<size_t>{W, H, P});
    std::vector<float> b = read_f32(dir + "/b.f32", W * H * P);
    std::copy(b.begin(), b.end(), proj->get_data_ptr());
    acq->set_projections(proj);

    auto E = boost::make_shared<CBSubsetOperatorB200>(subsets);
    E->setup(acq, L);
    std::vector<size_t> is_dims{nx, ny, nz};
    E->set_domain_dimensions(&is_dims);

    // permuted geometry (the reference mutates the acquisition the same way)
    write_f32(dir + "/angles_perm.f32", geo->get_angles().data(), P);
    std::vector<float> offp(2 * P);
    for (size_t i = 0; i < P; ++i) {
      offp[2 * i] = geo->get_offsets()[i][0];
      offp[2 * i + 1] = geo->get_offsets()[i][1];
    }
    write_f32(dir + "/offsets_perm.f32", offp.data(), 2 * P);

    std::vector<size_t> pd{W, H, P};
    cuNDArray<float> projections(&pd);
    cudaMemcpy(projections.get_data_ptr(), acq->get_projections()->get_data_ptr(), projections.bytes(),
               cudaMemcpyHostToDevice);

    // mult_M of a given image over all subsets, then mult_MH back
    std::vector<float> x = read_f32(dir + "/x.f32", nx * ny * nz);
    cuNDArray<float> img(&is_dims), img2(&is_dims), ax(&pd);
    cudaMemcpy(img.get_data_ptr(), x.data(), img.bytes(), cudaMemcpyHostToDevice);
    E->mult_M(&img, &ax, false);
    E->mult_MH(&ax, &img2, false);
    std::vector<float> h;
    download(ax, h);
    write_f32(dir + "/ax.f32", h.data(), h.size());
    download(img2, h);
    write_f32(dir + "/atax.f32", h.data(), h.size());

    // OS-MOM, 2 iterations, positivity (cuCBOS_reconstruct.cpp defaults)
    auto z = E->solve_osmom(&projections, 2, true);
    download(*z, h);
    write_f32(dir + "/z.f32", h.data(), h.size());
    std::printf("dropin ok: %zu views in %d subsets\n", P, subsets);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
