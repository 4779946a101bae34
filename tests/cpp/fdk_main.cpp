// Runs the FDK recipe of xray/FDK_reconstruct_3d.cpp:124-161 with
// hoCuConebeamProjectionOperatorB200 in place of hoCuConebeamProjectionOperator,
// call for call: setup on the acquisition and binning, filtered
// back-projection on, mult_MH of the projections into the volume, mult_M of
// the volume, and the least-squares rescale by dot(A x, p) / dot(A x, A x).
// Inputs and outputs are raw float32 files; tests/test_dropin.py checks them
// against the FP64 oracle.
//
// usage: fdk_main <io_dir> nx ny nz lx ly lz W H fov_u fov_v SAD SDD P batch [filter]
//   filter = 1: read filter.f32 (W+1 floats) and pass it to set_frequency_filter
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

int main(int argc, char** argv) {
  if (argc != 16 && argc != 17) {
    std::fprintf(stderr, "usage: %s io_dir nx ny nz lx ly lz W H fov_u fov_v SAD SDD P batch [filter]\n", argv[0]);
    return 2;
  }
  try {
    const std::string dir = argv[1];
    const size_t nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]);
    const floatd3 is_dims_in_mm(std::atof(argv[5]), std::atof(argv[6]), std::atof(argv[7]));
    const size_t W = std::atoi(argv[8]), H = std::atoi(argv[9]);
    const floatd2 fov(std::atof(argv[10]), std::atof(argv[11]));
    const float SAD = std::atof(argv[12]), SDD = std::atof(argv[13]);
    const size_t P = std::atoi(argv[14]);
    const unsigned batch = std::atoi(argv[15]);
    const bool custom_filter = argc == 17 && std::atoi(argv[16]) != 0;

    auto acquisition = boost::make_shared<CBCT_acquisition>();
    auto geo = acquisition->get_geometry();
    geo->set_SAD(SAD);
    geo->set_SDD(SDD);
    geo->set_FOV(fov);
    std::vector<float> ang = read_f32(dir + "/angles.f32", P);
    std::vector<float> off = read_f32(dir + "/offsets.f32", 2 * P);
    std::vector<floatd2> offsets(P);
    for (size_t i = 0; i < P; ++i) offsets[i] = floatd2(off[2 * i], off[2 * i + 1]);
    geo->set_angles(ang);
    geo->set_offsets(offsets);
    auto p = boost::make_shared<hoCuNDArray<float>>(std::vector<size_t>{W, H, P});
    std::vector<float> b = read_f32(dir + "/b.f32", W * H * P);
    std::copy(b.begin(), b.end(), p->get_data_ptr());
    acquisition->set_projections(p);
    std::vector<unsigned int> all(P);
    for (size_t i = 0; i < P; ++i) all[i] = (unsigned)i;
    auto binning = boost::make_shared<CBCT_binning>(std::vector<std::vector<unsigned int>>(1, all));

    // FDK_reconstruct_3d.cpp:128-161
    std::vector<size_t> is_dims = {nx, ny, nz};
    hoCuNDArray<float> fdk_3d(&is_dims);
    hoCuNDArray<float> projections(*acquisition->get_projections());

    boost::shared_ptr<hoCuConebeamProjectionOperatorB200> E(new hoCuConebeamProjectionOperatorB200());
    E->setup(acquisition, binning, is_dims_in_mm);
    E->set_use_filtered_backprojection(true);
    E->set_num_projections_per_batch(batch);
    if (custom_filter) {
      std::vector<float> f = read_f32(dir + "/filter.f32", W + 1);
      std::vector<size_t> fd{W + 1};
      auto filt = boost::make_shared<cuNDArray<float>>(&fd);
      cudaMemcpy(filt->get_data_ptr(), f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
      E->set_frequency_filter(filt);
    }

    E->mult_MH(&projections, &fdk_3d);
    write_f32(dir + "/fdk_raw.f32", fdk_3d.get_data_ptr(), fdk_3d.get_number_of_elements());
    hoCuNDArray<float> tmp_proj(projections.get_dimensions());
    E->mult_M(&fdk_3d, &tmp_proj, false);
    float scaler = dot(&tmp_proj, &projections) / dot(&tmp_proj, &tmp_proj);
    fdk_3d *= scaler;

    write_f32(dir + "/fdk.f32", fdk_3d.get_data_ptr(), fdk_3d.get_number_of_elements());
    write_f32(dir + "/ax.f32", tmp_proj.get_data_ptr(), tmp_proj.get_number_of_elements());
    std::printf("fdk ok: scaler %.9g\n", scaler);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
