// Drives the binned device-array drop-ins the way gt-tomography's 4-D drivers
// (xray/cuCBOSMOM.cpp, cuCBOS_reconstruct.cpp with a binning file) use
// cuConebeamProjectionOperator and CBSubsetOperator:
//   1. cuConebeamProjectionOperatorB200: setup with a binning (the
//      acquisition's projections permuted into bin order), mult_M of a 4-D
//      image (one volume per bin), mult_MH of the result back;
//   2. CBSubsetOperatorB200: setup with the same binning on a fresh
//      acquisition, mult_M of subset 0, and the device-resident OS-MOM solve
//      of all bins.
// Inputs and outputs are raw float32 / int32 files; tests/test_dropin.py checks
// them against the FP64 oracle.
//
// usage: bins_main <io_dir> nx ny nz lx ly lz W H fov_u fov_v SAD SDD P subsets
//   reads angles.f32, offsets.f32, b.f32 (W*H*P, acquisition order), x.f32
//   (nx*ny*nz*2), view_bin.i32 (P ints in {0,1})
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "cbct_gadgetron.hpp"

using namespace Gadgetron;

template <class T>
static std::vector<T> read_raw(const std::string& path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
  if (!f) throw std::runtime_error("cannot read " + path);
  return v;
}

template <class T>
static void write_raw(const std::string& path, const T* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), n * sizeof(T));
}

static void download(const cuNDArray<float>& a, std::vector<float>& h) {
  h.resize(a.get_number_of_elements());
  if (cudaMemcpy(h.data(), a.get_data_ptr(), a.bytes(), cudaMemcpyDeviceToHost) != cudaSuccess)
    throw std::runtime_error("cudaMemcpy failed");
}

static boost::shared_ptr<CBCT_acquisition> acquisition(const std::string& dir, size_t W, size_t H, size_t P, floatd2 fov,
                                                       float SAD, float SDD) {
  auto acq = boost::make_shared<CBCT_acquisition>();
  auto geo = acq->get_geometry();
  geo->set_SAD(SAD);
  geo->set_SDD(SDD);
  geo->set_FOV(fov);
  std::vector<float> ang = read_raw<float>(dir + "/angles.f32", P);
  std::vector<float> off = read_raw<float>(dir + "/offsets.f32", 2 * P);
  std::vector<floatd2> offsets(P);
  for (size_t i = 0; i < P; ++i) offsets[i] = floatd2(off[2 * i], off[2 * i + 1]);
  geo->set_angles(ang);
  geo->set_offsets(offsets);
  auto proj = boost::make_shared<hoCuNDArray<float>>(std::vector<size_t>{W, H, P});
  std::vector<float> b = read_raw<float>(dir + "/b.f32", W * H * P);
  std::copy(b.begin(), b.end(), proj->get_data_ptr());
  acq->set_projections(proj);
  return acq;
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
    std::vector<int32_t> vb = read_raw<int32_t>(dir + "/view_bin.i32", P);
    std::vector<std::vector<unsigned int>> bins(2);
    for (size_t i = 0; i < P; ++i) bins[vb[i]].push_back((unsigned)i);
    auto binning = boost::make_shared<CBCT_binning>(bins);
    std::vector<size_t> dims4{nx, ny, nz, 2};
    std::vector<float> x = read_raw<float>(dir + "/x.f32", nx * ny * nz * 2);
    cuNDArray<float> img(&dims4), back(&dims4);
    cudaMemcpy(img.get_data_ptr(), x.data(), img.bytes(), cudaMemcpyHostToDevice);
    std::vector<float> h;

    // 1. the binned device-array operator
    {
      auto acq = acquisition(dir, W, H, P, fov, SAD, SDD);
      cuConebeamProjectionOperatorB200 E;
      E.setup(acq, binning, L);
      E.set_domain_dimensions(&dims4);
      std::vector<size_t> pd{W, H, P};
      cuNDArray<float> ax(&pd);
      E.mult_M(&img, &ax);
      E.mult_MH(&ax, &back);
      download(ax, h);
      write_raw(dir + "/op_ax.f32", h.data(), h.size());
      download(back, h);
      write_raw(dir + "/op_atax.f32", h.data(), h.size());
      write_raw(dir + "/op_b_perm.f32", acq->get_projections()->get_data_ptr(), W * H * P);
    }
    // 2. the binned subset operator and its OS-MOM solve
    {
      auto acq = acquisition(dir, W, H, P, fov, SAD, SDD);
      auto E = boost::make_shared<CBSubsetOperatorB200>(subsets);
      E->setup(acq, binning, L);
      E->set_domain_dimensions(&dims4);
      write_raw(dir + "/sub_angles.f32", acq->get_geometry()->get_angles().data(), P);
      std::vector<float> offp(2 * P);
      for (size_t i = 0; i < P; ++i) {
        offp[2 * i] = acq->get_geometry()->get_offsets()[i][0];
        offp[2 * i + 1] = acq->get_geometry()->get_offsets()[i][1];
      }
      write_raw(dir + "/sub_offsets.f32", offp.data(), 2 * P);
      auto d0 = *E->get_codomain_dimensions(0);
      cuNDArray<float> a0(&d0);
      E->mult_M(&img, &a0, 0, false);
      download(a0, h);
      write_raw(dir + "/sub_ax0.f32", h.data(), h.size());
      std::vector<size_t> pd{W, H, P};
      cuNDArray<float> projections(&pd);
      cudaMemcpy(projections.get_data_ptr(), acq->get_projections()->get_data_ptr(), projections.bytes(),
                 cudaMemcpyHostToDevice);
      auto z = E->solve_osmom(&projections, 2, true);
      download(*z, h);
      write_raw(dir + "/sub_z.f32", h.data(), h.size());
    }
    std::printf("bins ok: %zu views, 2 bins, %d subsets\n", P, subsets);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
